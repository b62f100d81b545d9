"""Algorithmic FLOP model of the Rys-quadrature J/K build, per angular class.

The count is what the Rys algorithm needs, not what a given kernel happens to
execute (an FMA counts as 2 FLOPs).  Per primitive quartet of class
(la lb | lc ld) with n = (la+lb+lc+ld)//2 + 1 roots:

  setup            30       p+q, rho, T, prefactor, P-A, Q-C, P-Q
  roots R(n)       n = 1: 40, n = 2: 70, n = 3: 160 (Boys Taylor + downward
                   recursion + closed-form Jacobi eigenproblem), n >= 4: 2n * 38
                   (degree-11 Clenshaw per root/weight)
  per root         15       B00, B10, B01, C00, C00' (3 axes)
  per root, axis   4 * ((la+lb+1)(lc+ld+1) - 1)                 vertical recursion
                   2 * sum_{d=1..ld} (la+lb+1)(lc+ld+1-d)        ket transfer
                   2 * sum_{b=1..lb} (la+lb+1-b)(lc+1)(ld+1)     bra transfer
  per root         3 * Nc   (Ix*Iy, *Iz, accumulate), Nc = product of
                   Cartesian shell sizes
Per contracted quartet and symmetric density: 12 * Nc digestion FLOPs
(J: 2 FMA, K: 4 FMA per integral).
"""
from __future__ import annotations


def ncart(l):
    return (l + 1) * (l + 2) // 2


def nroots(la, lb, lc, ld):
    return (la + lb + lc + ld) // 2 + 1


def root_flops(n):
    return {1: 40, 2: 70, 3: 160}.get(n, 2 * n * 38)


def per_primitive_quartet(la, lb, lc, ld):
    n = nroots(la, lb, lc, ld)
    lab, lcd = la + lb, lc + ld
    vrr = 4 * ((lab + 1) * (lcd + 1) - 1)
    hrr_ket = 2 * sum((lab + 1) * (lcd + 1 - d) for d in range(1, ld + 1))
    hrr_bra = 2 * sum((lab + 1 - b) * (lc + 1) * (ld + 1) for b in range(1, lb + 1))
    nc = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    return 30 + root_flops(n) + n * (15 + 3 * (vrr + hrr_bra + hrr_ket) + 3 * nc)


def per_quartet_digestion(la, lb, lc, ld, ndens=1):
    return 12 * ncart(la) * ncart(lb) * ncart(lc) * ncart(ld) * ndens


def class_flops(cls, prim_quartets, quartets, ndens=1):
    la, lb, lc, ld = cls
    return prim_quartets * per_primitive_quartet(la, lb, lc, ld) + \
        quartets * per_quartet_digestion(la, lb, lc, ld, ndens)
