"""Algorithmic work per accepted RK4 ray-step, counted from the kernel source.

Counting rule: an FMA is 2 FLOP; every add, multiply, divide, square root,
reciprocal, reciprocal square root, exp/exp2/log2/pow is 1 FLOP; negation
and copies are free.  Counts assume the ray is inside the emission region
(r > r_isco, timelike Keplerian flow, shift > 0), which holds for nearly
every step of the torus workloads; outside it the transfer part is skipped.

Mixed kernel (gray_b200/csrc/kernels_mixed.cu), per call; the geodesic is
integrated in Hamiltonian form on (x^mu, k_i) with k_t conserved:
  ks_ham          93   (head 32: radius root, f, df/dr and the explicit
                        df/dz with 2 rsqrt + 2 rcp; l, L = l^mu k_mu,
                        dL/dr and the force G d_i r + f L (explicit d_i L),
                        and dx^mu/dl 61)
  torus_rt        33 + 4 per frequency  (Keplerian flow and shift from
                        k_mu 23; the density in log2, -1.5 lg2 r plus the
                        Gaussian from z/r of the geodesic part, and dtau_0 as
                        one ex2 10; per frequency
                        one ex2 of the summed log2 factors, with n0 and
                        nu_i^-0.7 folded into a per-ray constant 4); only
                        tau_0 is integrated, the other optical depths are
                        (nu_0/nu_i)^2 times it
  RK4 + Kahan     per integrated real: stages 2 + 4 + 4, final 2 + 4
                  (Kahan) = 16, plus 3 scalars; 7 + (n_freq + 1) reals
  step control    6   (far from the hole, nearly every step of these
                        workloads: x^2+y^2+z^2-a^2 against the per-interval
                        bound beyond which the step is the cap; near it the
                        FP32 radius root and the n/|dt| tick rule add 17)

FP64 kernel (gray_b200/csrc/kernels_fp64.cu), per call:
  ks_rhs64        196  (5 divides and 2 sqrt counted as 1 each)
  torus_rt64      49 + 5 per frequency  (pow and exp counted as 1 each)
  RK4             per component 2 + 2 + 2 + 6 = 12, plus 2 scalars
  step control    16 + 4 for the integer-tick arithmetic

The reference's own comments count the same KS RHS as about 205 FLOP
(KS.cl:310-374), counting its divides the same way.
"""


def mixed_per_step(n_freq, transfer=True):
    ni = 7 + (n_freq + 1 if n_freq else 0)
    rhs = 93 + ((33 + 4 * n_freq) if (transfer and n_freq) else 0)
    return 4 * rhs + 16 * ni + 3 + 6


def fp64_per_step(n_freq, transfer=True):
    nd = 8 + 2 * n_freq
    rhs = 196 + ((49 + 5 * n_freq) if (transfer and n_freq) else 0)
    return 4 * rhs + 12 * nd + 2 + 20


def state_bytes_per_ray(n_freq):
    """HBM traffic of one persistent launch per ray: FP64 initial state in,
    FP64 final state and the getuu diagnostic out."""
    nd = 8 + 2 * n_freq
    return 8 * nd + 8 * nd + 8
