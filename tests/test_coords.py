"""Output coordinates (KS.cl:63-153): spherical Kerr-Schild and
Boyer-Lindquist events and vectors of an analytic render's state.

CPU: the oracle's restatement against geometry -- the inverse of the
Kerr-Schild Cartesian map, the vector transform as the derivative of the
event transform along u, and null rays staying null in the Boyer-Lindquist
metric.  The default follows the metric of down(); the as-written form
(KS.cl's phi convention and getBLu lines) inverts the other handedness and
fails the null test.
GPU: gray_read_coords against the oracle on traced rays (the vector parts
use only +, *, /, sqrt and agree bit for bit; the events call acos, atan2
and log, whose last bits differ between CUDA and glibc)."""
import numpy as np
import pytest

import oracle as O
from gray_b200 import api

A = 0.9


def ks_event(r, th, ph, a=A):
    """x + iy = (r + i a) e^(i phi) sin(theta), z = r cos(theta): the event
    of the metric of KS.cl:91-114 (down())."""
    return np.array([(r * np.cos(ph) - a * np.sin(ph)) * np.sin(th),
                     (r * np.sin(ph) + a * np.cos(ph)) * np.sin(th), r * np.cos(th)])


def bl_metric(r, th, a=A):
    S = r * r + a * a * np.cos(th) ** 2
    D = r * r - 2 * r + a * a
    s2 = np.sin(th) ** 2
    g = np.zeros((4, 4))
    g[0, 0] = -(1 - 2 * r / S)
    g[0, 3] = g[3, 0] = -2 * a * r * s2 / S
    g[1, 1] = S / D
    g[2, 2] = S
    g[3, 3] = (r * r + a * a + 2 * a * a * r * s2 / S) * s2
    return g


def traced_states(n=24):
    cfg = dict(a_spin=A, r_obs=60.0, i_obs=60.0, w_img=24.0, h_img=24.0, n_width=6,
               n_height=4, dt_dump=-10.0, n_dump=4, n_sub=64)
    out, info, _ = O.trace(cfg, np.arange(n))
    return cfg, out, info


def test_spherical_ks_inverts_the_cartesian_map():
    rng = np.random.default_rng(3)
    for _ in range(50):
        r, th, ph = rng.uniform(1.5, 50), rng.uniform(0.05, 3.09), rng.uniform(-3.1, 3.1)
        c = O.coords(A, np.r_[2.5, ks_event(r, th, ph), 1, 0, 0, 0], "sph")
        assert np.allclose(c[:4], [2.5, r, th, ph], rtol=1e-12, atol=1e-12)
        # KS.cl:68-69 as written inverts the event of spin -a
        w = O.coords(A, np.r_[2.5, ks_event(r, th, ph, -A), 1, 0, 0, 0], "sph",
                     as_written=True)
        assert np.allclose(w[:4], [2.5, r, th, ph], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("system", ["sph", "bl"])
def test_vectors_are_derivatives_of_events(system):
    rng = np.random.default_rng(4)
    for _ in range(20):
        q = np.r_[rng.uniform(-5, 5), ks_event(rng.uniform(3, 30), rng.uniform(0.3, 2.8),
                                               rng.uniform(-3, 3))]
        u = np.r_[1.0, rng.normal(size=3)]
        e = 1e-6 * np.linalg.norm(q)
        fd = (O.coords(A, np.r_[q + e * u, u], system)[:4] -
              O.coords(A, np.r_[q - e * u, u], system)[:4]) / (2 * e)
        an = O.coords(A, np.r_[q, u], system)[4:]
        assert np.allclose(an, fd, rtol=1e-6, atol=1e-7)
        fw = (O.coords(A, np.r_[q + e * u, u], system, as_written=True)[:4] -
              O.coords(A, np.r_[q - e * u, u], system, as_written=True)[:4]) / (2 * e)
        aw = O.coords(A, np.r_[q, u], system, as_written=True)[4:]
        if system == "sph":  # KS.cl:63-71 and 116-133 agree with each other
            assert np.allclose(aw, fw, rtol=1e-6, atol=1e-7)
        else:  # KS.cl:148-151 as written is not the derivative of getBL
            assert np.max(np.abs(aw - fw)) > 1e-3


def test_bl_matching_conventions():
    q = np.r_[4.0, ks_event(10.0, 1.0, 0.5)]
    c = O.coords(A, np.r_[q, 1, 0, 0, 0], "bl", r_match=10.0)
    assert c[0] == pytest.approx(4.0, abs=1e-13)  # t_BL = t_KS at r_match
    far = O.coords(A, np.r_[q[0], ks_event(1e9, 1.0, 0.5), 1, 0, 0, 0], "bl")
    assert far[3] == pytest.approx(0.5, abs=1e-8)  # phi matched at infinity


def test_null_rays_stay_null_in_boyer_lindquist():
    _, out, info = traced_states()
    for s, i in zip(out, info):
        if not np.all(np.isfinite(s)):
            continue
        c = O.coords(A, s[:8], "bl")
        g = bl_metric(c[1], c[2])
        uu, scale = c[4:] @ g @ c[4:], np.abs(c[4:]) @ np.abs(g) @ np.abs(c[4:])
        assert abs(uu) <= 1e-9 * scale + abs(i)
        aw = O.coords(A, s[:8], "bl", as_written=True)
        assert abs(aw[4:] @ g @ aw[4:]) > 1e-6 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("system,flags", [(api.COORDS_SPH_KS, 0), (api.COORDS_BL, 0),
                                          (api.COORDS_BL, api.COORDS_AS_WRITTEN)])
def test_device_coords_match_oracle(ctx, system, flags):
    cfg, _, _ = traced_states()
    r = ctx.render(dict(cfg, precision=api.PREC_FP64))
    try:
        r.run()
        s, _ = r.state(api.LAYOUT_AOS)
        got = r.coords(system, r_match=12.0, flags=flags)
    finally:
        r.close()
    name = "sph" if system == api.COORDS_SPH_KS else "bl"
    ref = np.array([O.coords(A, x[:8], name, r_match=12.0, as_written=bool(flags))
                    for x in s]).T
    fin = np.all(np.isfinite(ref), axis=0)
    assert fin.mean() > 0.5 and np.array_equal(fin, np.all(np.isfinite(got), axis=0))
    assert np.array_equal(got[4:, fin], ref[4:, fin])  # vectors: bit for bit
    assert np.array_equal(got[1, fin], ref[1, fin])    # r: sqrt only
    assert np.allclose(got[[0, 2, 3]][:, fin], ref[[0, 2, 3]][:, fin], rtol=1e-14, atol=1e-14)


@pytest.mark.gpu
def test_coords_arguments(ctx):
    r = ctx.render(dict(n_width=4, n_height=4, a_spin=A, n_dump=1))
    try:
        with pytest.raises(api.GrayError) as e:
            r.coords()  # no state yet
        assert e.value.status == api.ESTATE
        r.icond()
        for kw in (dict(system=7), dict(r_match=1.2), dict(flags=4)):  # r_match inside r_+
            with pytest.raises(api.GrayError) as e:
                r.coords(**kw)
            assert e.value.status == api.EINVAL
    finally:
        r.close()
