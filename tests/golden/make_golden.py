"""Generate golden vectors from the reference's own Python spacetime code.

The reference (luxsrc/gray) ships no golden vectors for the geodesic path.
Its Python tool tools/boosted_ks.py, however, evaluates the boosted
Kerr-Schild metric (boosted_ks.py:120-186) and its Christoffel symbols by
dual-number differentiation (boosted_ks.py:191-275); tools/generate_data.py
uses it to write numerical spacetimes.  This script imports that module
unmodified and records:

  boosted_ks_points.json  g_ij (10) and Gamma^i_jk (40) at sample events for
                          several (a, boost) pairs, boost along z as the tool
                          hard-wires it;
  ks_rk4_rays.json        short classical-RK4 integrations of
                          du^mu/dl = -Gamma^mu_ab u^a u^b with the tool's
                          Christoffels (boost 0, i.e. plain Kerr-Schild).

It also checks, writing nothing, that the log K_2 table the library
generates (gray_b200/csrc/make_logk2.py) holds the same numbers as the
table of sim-org/rt.cl:51-67.

Run from the repository root:
    python tests/golden/make_golden.py <path/to/reference>/tools
The fixtures are committed; the tests never need the reference at run time.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_tool(tools_dir):
    sys.path.insert(0, tools_dir)
    import boosted_ks  # noqa: E402  (the reference's unmodified module)
    return boosted_ks


IDX_G = [(i, j, k) for i in range(4) for j in range(4) for k in range(j, 4)]
IDX_M = [(i, j) for i in range(4) for j in range(i, 4)]


def fields(bk, m, a, v, q):
    P = (m, a, v)
    X = tuple(float(c) for c in q)
    gam = [bk.Christoffel(P, X, *ind) for ind in IDX_G]
    met = [bk.metric(P, X, *ind) for ind in IDX_M]
    return [float(x) for x in gam], [float(x) for x in met]


def accel(bk, a, s):
    """-Gamma^mu_ab u^a u^b from the tool's Christoffels (boost 0)."""
    P = (1.0, a, 0.0)
    X = tuple(float(c) for c in s[:4])
    u = s[4:]
    acc = np.zeros(4)
    for mu in range(4):
        tot = 0.0
        for al in range(4):
            for be in range(4):
                j, k = min(al, be), max(al, be)
                tot += bk.Christoffel(P, X, mu, j, k) * u[al] * u[be]
        acc[mu] = -tot
    return acc


def rhs(bk, a, s):
    return np.concatenate([s[4:], accel(bk, a, s)])


def rk4(bk, a, s, h):
    k1 = rhs(bk, a, s)
    k2 = rhs(bk, a, s + 0.5 * h * k1)
    k3 = rhs(bk, a, s + 0.5 * h * k2)
    k4 = rhs(bk, a, s + h * k3)
    return s + h * (k1 + 2 * (k2 + k3) + k4) / 6.0


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference>/tools  (the reference's tools directory)")
    tools = sys.argv[1]
    bk = load_tool(tools)
    rng = np.random.default_rng(20261203)

    cases = []
    for (a, v) in [(0.0, 0.0), (0.9, 0.0), (0.998, 0.0), (0.7, 0.3), (0.6, 0.5)]:
        for _ in range(12):
            # events away from the ring singularity and the horizon
            while True:
                r = rng.uniform(2.5, 60.0)
                th = np.arccos(rng.uniform(-1, 1))
                ph = rng.uniform(0, 2 * np.pi)
                x, y, z = r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)
                if np.sqrt(x * x + y * y) > 1.5 or abs(z) > 1.5:
                    break
            t = rng.uniform(-5.0, 5.0)
            q = [t, x, y, z]
            gam, met = fields(bk, 1.0, a, v, q)
            cases.append({"m": 1.0, "a": a, "v": v, "axis": 3, "q": q,
                          "gamma": gam, "g": met})
    with open(os.path.join(HERE, "boosted_ks_points.json"), "w") as f:
        json.dump({"source": "tools/boosted_ks.py metric() and Christoffel()",
                   "cases": cases}, f, indent=1)

    rays = []
    for (a, q, d, h, n) in [
        (0.9, [0.0, 30.0, 4.0, 10.0], [-0.8, 0.1, -0.2], 0.05, 12),
        (0.998, [0.0, -6.0, 7.0, 3.0], [0.3, -0.9, -0.1], 0.02, 12),
        (0.0, [0.0, 12.0, 0.0, 5.0], [-1.0, 0.2, 0.0], 0.1, 12),
    ]:
        # direction made null with u^t = 1 in flat space; the RK4 pin does
        # not need the curved null condition
        d = np.array(d) / np.linalg.norm(d)
        s0 = np.array(q + [1.0] + list(d))
        s = s0.copy()
        for _ in range(n):
            s = rk4(bk, a, s, h)
        rays.append({"a": a, "s0": list(map(float, s0)), "h": h, "n": n,
                     "s": list(map(float, s))})
    with open(os.path.join(HERE, "ks_rk4_rays.json"), "w") as f:
        json.dump({"source": "classical RK4 on -Gamma u u from tools/boosted_ks.py",
                   "rays": rays}, f, indent=1)
    print("wrote", len(cases), "field cases and", len(rays), "rays")
    check_logk2(os.path.join(os.path.dirname(os.path.abspath(tools)), "sim-org", "rt.cl"))


def check_logk2(rt_cl):
    import re
    sys.path.insert(0, os.path.join(HERE, "..", "..", "gray_b200", "csrc"))
    import make_logk2  # noqa: E402
    src = open(rt_cl).read()
    body = re.search(r"log_K2it_tab\[\]\s*=\s*\{(.*?)\}", src, re.S).group(1)
    ref = np.array([float(x) for x in body.split(",")])
    ours = np.array([float(make_logk2.fmt(x)) for x in make_logk2.values()])
    assert np.array_equal(ref, ours), np.max(np.abs(ref - ours))
    print("log K_2 table: %d values identical to %s" % (ref.size, "sim-org/rt.cl"))


if __name__ == "__main__":
    main()
