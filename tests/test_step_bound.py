"""The mixed kernel's far-field step shortcut (gray_b200/csrc/kernels_mixed.cu,
start_dump and ticks): beyond x^2+y^2+z^2-a^2 >= r2_far the kernel takes the
capped step without evaluating the radius root.  The shortcut is exact only
if, wherever it fires, the full FP32 tick rule (KS.cl:48-61 radius and
epsilon, phys.cl:60-61 via driver.cl:93) would also give the capped step.
This checks that on the CPU, with the rule's FP32 arithmetic emulated in
numpy float32, over random spins, dump intervals, substep counts and
positions just beyond the bound.  No GPU is involved."""
import numpy as np

INT_MAX = 2**31 - 1
f32 = np.float32


def bound(a, dt, n_sub):
    """start_dump's per-interval constants, in the same FP64 arithmetic."""
    n = (INT_MAX // n_sub) * n_sub
    dts = dt / n_sub
    dh_cap = int(dts / dt * n)
    cdt = f32(n / abs(dt))
    rp = 1.0 + np.sqrt(1.0 - a * a)
    e_cap = np.sqrt(dh_cap / (0.01 * float(cdt)))
    r_far = 1.01 * (rp + e_cap) + 1.0
    return f32(r_far * r_far), dh_cap, cdt, f32(rp)


def full_rule(a, x, y, z, dh_cap, cdt, rp):
    """ticks() without the shortcut, in float32 (exact square roots stand in
    for the approximate ones; the bound's 1% margin covers both)."""
    aa = f32(a * a)
    zz = z * z
    kk = f32(0.5) * ((x * x + (y * y + zz)) - aa)
    rr = np.sqrt(kk * kk + aa * zz) + kk
    eps = np.sqrt(rr) - rp
    want = f32(0.01) * eps * eps * cdt
    dh = np.where(want < f32(dh_cap), np.floor(want), dh_cap)
    return eps, dh


def test_shortcut_gives_the_capped_step_wherever_it_fires():
    rng = np.random.default_rng(11)
    fired = 0
    for _ in range(200):
        a = rng.uniform(0.0, 0.999)
        dt = rng.choice([-1.0, 1.0]) * 10 ** rng.uniform(-1, 2)
        n_sub = int(10 ** rng.uniform(1, 4))
        r2_far, dh_cap, cdt, rp = bound(a, dt, n_sub)
        # positions at and just beyond the bound, in every direction
        m = 2000
        d = rng.standard_normal((m, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        q2 = float(r2_far) + a * a + np.abs(rng.standard_normal(m)) * rng.choice([1e-6, 1e-2, 1.0])
        p = (d * np.sqrt(q2)[:, None]).astype(np.float32)
        x, y, z = p[:, 0], p[:, 1], p[:, 2]
        aa = f32(a * a)
        fires = (x * x + (y * y + z * z)) - aa >= r2_far
        eps, dh = full_rule(a, x, y, z, dh_cap, cdt, rp)
        assert np.all(eps[fires] >= 1.0)       # no FP64 island, no stop
        assert np.all(dh[fires] == dh_cap)     # the capped step, as the shortcut returns
        fired += int(fires.sum())
    assert fired > 100000
