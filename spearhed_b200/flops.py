"""Algorithmic work per accepted pair, counted from the pair kernels' arithmetic.

Counting rule: one FP32 (or FP64) add, multiply, compare-select or min/max is 1
flop; a fused multiply-add is 2; a reciprocal square root, reciprocal or
division is 1.  Candidate tests that are rejected by the cull are not counted
(they are reported separately as cull efficiency, CULL_FLOPS_PER_CANDIDATE each),
and the artificial-viscosity terms, evaluated branch-free for every pair but
nonzero only for approaching ones, are not counted either, so the figures are
lower bounds.  s_j is counted even where equal smoothing lengths let the kernel
reuse s_i.

Wendland C2 kernel (the benchmark workload's kernel):
  density pass, per accepted pair (pair_kernels.cu, kDensity sum over the list):
    displacement with stencil shift: 3 x (fma + sub)             9
    r^2: mul + 2 fma                                             5
    rsqrt, r = r2 * invR                                         2
    W: x = r/h (1), (1-x/2) (2), squares (2), (1+2x) (2), * (1),
       sigma/h^3 * (1)                                            9
    m_j * W and accumulate (fma)                                  2
                                                                 27
  force pass, SPMHD variant, per accepted pair (kForce<K, T, 2 or 3>):
    displacement + r^2 + rsqrt + r                               16
    s_i: x (1), shape (6), dwnorm * shape * invR (2)              9
    s_j: 1/h_j (1), h-powers and norms (4), x (1), shape (6), (2) 14
    isotropic pressure term m_j (P~_i s_i + P~_j s_j)             4
    v_ij (3), v_ij . r (5)                                        8
    acceleration accumulate (3 fma)                               6
    m_j s_i and D accumulate                                      3
    signal speed (w, min, fma, max)                               6
    B_i . r, B_j . r                                             10
    c_i, c_j                                                      5
    anisotropic stress accumulate (3 x (mul + fma + add))        12
    tensile sum, m_j s_i (B_i . r), induction (3 fma)             9
    div B accumulate                                              3
    Dedner gradient term and accumulate                          10
                                                                115
The SPH pair-interaction metric counts logical pair passes per step: density (1),
hydro/AV (1) and SPMHD/Dedner (1); one fused force kernel evaluates the last
two, so one accepted pair of that kernel is two pair interactions.
"""

DENSITY_FLOPS = {"cubic": 27, "quintic": 33, "wendland_c2": 27}
FORCE_FLOPS = {  # by physics variant
    "hydro": 70,        # reference inviscid hydro: geometry 16 + s_i 9 + s_j 14 + iso 4 + v 8 + acc 6 + D 3 + vsig 6 + ...
    "hydro_av": 70,     # viscosity branch not counted (see above)
    "mhd": 115,
}
PASSES_PER_STEP = {"hydro": 2, "hydro_av": 2, "mhd": 3}
# cull test of one (target, staged source) candidate: 3 differences, 3 squares,
# 2 adds for r^2 and the r^2 - R^2 whose sign is the acceptance bit
CULL_FLOPS_PER_CANDIDATE = 9
