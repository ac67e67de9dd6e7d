"""Named workloads of the geodesic hot path, with their sizes.

kerr_small_64   a=0.9 Kerr-Schild, camera r=1000 M at 60 deg, 64x64 rays over
                +-20 M, RK4 to affine parameter -2000 M (64 dumps of -31.25 M,
                1000 substeps each, i.e. a 1/32 M step cap), FP64, no transfer.
torus_rt_1024   a=0.998, 17 deg, 1024x1024 rays over +-20 M at r=1000 M, same
                step control, transfer at nu = 1, 2, 4, 8 through the analytic
                power-law torus; kappa is frozen so that tau(nu=1) = 1 along
                the central ray (ray 512*1024+512).
numerical_128   128^3 FP32 boosted Kerr-Schild grid (a=0.7, v=0.3 along x) on
                [-40, 40]^3 with the n=3 fisheye map, levels t=0 and t=10 M;
                512x512 camera at r=200 M, 45 deg, mixed precision.
"""
TORUS_KAPPA = 125.8988  # 1 / tau(nu=1) of the central ray with kappa = 1

KERR_SMALL_64 = dict(
    a_spin=0.9, w_img=40.0, h_img=40.0, r_obs=1000.0, i_obs=60.0, j_obs=0.0,
    n_width=64, n_height=64, t_init=0.0, dt_dump=-31.25, n_sub=1000, n_dump=64,
    nu=(),
)

TORUS_RT_1024 = dict(
    a_spin=0.998, w_img=40.0, h_img=40.0, r_obs=1000.0, i_obs=17.0, j_obs=0.0,
    n_width=1024, n_height=1024, t_init=0.0, dt_dump=-31.25, n_sub=1000, n_dump=64,
    nu=(1.0, 2.0, 4.0, 8.0), torus_n0=1.0, torus_kappa=TORUS_KAPPA, torus_hr=0.3,
)


SURVEY_SEED = 20261203


def survey(n=256, seed=SURVEY_SEED, side_lo=32, side_hi=512):
    """survey_256: n renders with side log-uniform in [side_lo, side_hi]
    (pixels log-uniform in 32^2..512^2), spin U[0, 0.998], inclination
    U[5, 85] deg, camera distance U[100, 1000] M (numpy PCG64, seeded); each
    uses the torus_rt_1024 torus at 4 frequencies and its step control."""
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(seed))
    side = np.rint(np.exp(rng.uniform(np.log(side_lo), np.log(side_hi), n))).astype(int)
    a = rng.uniform(0.0, 0.998, n)
    inc = rng.uniform(5.0, 85.0, n)
    robs = rng.uniform(100.0, 1000.0, n)
    out = []
    for k in range(n):
        c = dict(TORUS_RT_1024)
        c.update(a_spin=float(a[k]), i_obs=float(inc[k]), r_obs=float(robs[k]),
                 n_width=int(side[k]), n_height=int(side[k]))
        out.append(c)
    return out


NUMERICAL_128 = dict(        # 128^3 grid, two levels, 512^2 camera at 200 M, 45 deg
    a_spin=0.0, r_obs=200.0, i_obs=45.0, j_obs=0.0, w_img=80.0, h_img=80.0,
    n_width=512, n_height=512, t_init=0.0, dt_dump=-10.0, n_dump=30, n_sub=100,
    nu=(), spacetime=1)
NUMERICAL_GRID = dict(n=128, box=40.0, a=0.7, v=0.3, axis=1, t1=0.0, t2=10.0)

SERVE_SEED = 20261204
SERVE_GRID_N = 256          # 256^3 FP32 boosted KS, one time level: 3.5 GB resident
SERVE_GRID_BOX = 40.0
NUMERICAL_BASE = dict(       # numerical-spacetime camera of the serving mix
    a_spin=0.0, r_obs=200.0, w_img=80.0, h_img=80.0, j_obs=0.0, t_init=0.0,
    dt_dump=-10.0, n_dump=30, n_sub=100, nu=(), spacetime=1)


def serve_requests(n, seed=SERVE_SEED):
    """serve_mix request stream: 70% analytic torus renders (side log-uniform
    64..1024, spin U[0, 0.998], inclination U[5, 85] deg, camera at 1000 M)
    and 30% numerical-spacetime renders on the shared boosted-KS grid (side
    log-uniform 64..512, inclination U[5, 85] deg, camera at 200 M, affine
    range -300 M in steps of 0.01 M)."""
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        numerical = rng.uniform() < 0.3
        inc = float(rng.uniform(5.0, 85.0))
        if numerical:
            side = int(np.rint(np.exp(rng.uniform(np.log(64), np.log(512)))))
            c = dict(NUMERICAL_BASE, i_obs=inc, n_width=side, n_height=side)
        else:
            side = int(np.rint(np.exp(rng.uniform(np.log(64), np.log(1024)))))
            c = dict(TORUS_RT_1024, a_spin=float(rng.uniform(0.0, 0.998)), i_obs=inc,
                     n_width=side, n_height=side)
        out.append(c)
    return out


def scaled(cfg, side):
    """The same workload on a side x side camera (parity-test sizes)."""
    c = dict(cfg)
    c["n_width"] = side
    c["n_height"] = side
    return c
