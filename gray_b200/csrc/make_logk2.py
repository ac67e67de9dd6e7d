"""Writes logk2_table.h: log K_2(1/Theta_e) on the log-spaced Theta_e grid
T_MIN * (T_MAX / T_MIN)^(i / T_GRID), i = 0..T_GRID, with T_MIN = 0.1,
T_MAX = 100, T_GRID = 60 -- the grid the synchrotron emissivity
interpolates on (rt.cl:41-78).  The values come from the modified Bessel
function itself (scipy.special.kn), not from a copied table, rounded the
way rt.cl:51-67 publishes its table (13 characters: ten decimals, nine
when the value has two integer digits), so that the interpolation reads
the same numbers the reference does.

    python gray_b200/csrc/make_logk2.py
"""
import os

import numpy as np
from scipy.special import kn

T_MIN, T_MAX, T_GRID = 0.1, 100.0, 60


def values():
    te = T_MIN * (T_MAX / T_MIN) ** (np.arange(T_GRID + 1) / T_GRID)
    return np.log(kn(2, 1.0 / te))


def fmt(x):
    return "%+.9f" % x if abs(x) >= 10 else "%+.10f" % x


def render():
    v = values()
    rows = [", ".join(fmt(x) for x in v[i:i + 4]) for i in range(0, len(v), 4)]
    return ("/* Generated by make_logk2.py: log K_2(1/Theta_e) at Theta_e =\n"
            " * 0.1 * 1000^(i/60), i = 0..60 (scipy.special.kn), rounded to\n"
            " * 13 characters as rt.cl:51-67 publishes the table. */\n"
            "#ifndef GRAY_LOGK2_TABLE_H\n#define GRAY_LOGK2_TABLE_H\n"
            "#define GRAY_LOGK2_N %d\n" % (T_GRID + 1) +
            "#define GRAY_LOGK2_VALUES \\\n" +
            ", \\\n".join("\t" + r for r in rows) + "\n#endif\n")


def main():
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "logk2_table.h")
    with open(out, "w") as f:
        f.write(render())


if __name__ == "__main__":
    main()
