"""Generate rys_tables.h: Rys quadrature roots/weights and Boys-function grids.

Written from the mathematics, not from any existing integral library:

* Boys function  F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt
                        = 1F1(m+1/2; m+3/2; -T) / (2m+1)      (mpmath, 60 digits)
* Rys quadrature: for the weight exp(-T t^2) on t in [0,1], written in
  x = t^2, the ordinary moments are mu_k = F_k(T).  The three-term recurrence
  of the orthogonal polynomials comes from Gautschi's Chebyshev algorithm
  (W. Gautschi, "Orthogonal Polynomials: Computation and Approximation", 2004,
  sec. 2.1.7) run in 60-digit arithmetic (the map is ill-conditioned, so the
  extra digits absorb it), and the nodes x_i and weights w_i come from the
  Golub-Welsch eigen-decomposition of the Jacobi matrix.
* For T in [k, k+1), k < K_n, each x_i(T) and w_i(T) is a degree-11
  Chebyshev series in s = 2(T-k)-1 (coefficients from Chebyshev-node
  interpolation; relative error ~2e-16, checked below).
* For T >= K_n the large-T limit is used: the weight exp(-T t^2) on [0, inf)
  gives x_i = s_i^2 / T and w_i = h_i / sqrt(T), with s_i the n positive
  Gauss-Hermite nodes of order 2n and h_i their weights.  K_n is the first
  integer beyond which that limit is accurate to 4e-16 relative.
* Boys grid: F_m(k/20) for k = 0..800 and m = 0..BOYS_MMAX+7, used by a
  Taylor expansion about the nearest grid point (|dT| <= 0.025, 8 terms).

Usage: python gradscf_b200/csrc/gen_tables.py   (writes rys_tables.h here)
"""
from __future__ import annotations

import multiprocessing as mproc
from pathlib import Path

import mpmath as mp

RYS_MAX_N = 8
DEG = 11
BOYS_STEP_INV = 20
BOYS_TMAX = 40
BOYS_MMAX = 16          # highest order evaluated through the Taylor grid
BOYS_TERMS = 8
DPS = 60


def boys(m, t):
    t = mp.mpf(t)
    if t == 0:
        return mp.mpf(1) / (2 * m + 1)
    return mp.hyp1f1(m + mp.mpf(1) / 2, m + mp.mpf(3) / 2, -t) / (2 * m + 1)


def rys(n, t):
    mp.mp.dps = DPS
    mu = [boys(k, t) for k in range(2 * n)]
    sig_prev = [mp.mpf(0)] * (2 * n)
    sig = mu[:]
    alpha, beta = [mu[1] / mu[0]], [mu[0]]
    for k in range(1, n):
        new = [mp.mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l]
        alpha.append(new[k + 1] / new[k] - sig[k] / sig[k - 1])
        beta.append(new[k] / sig[k - 1])
        sig_prev, sig = sig, new
    jac = mp.zeros(n)
    for i in range(n):
        jac[i, i] = alpha[i]
        if i + 1 < n:
            jac[i, i + 1] = jac[i + 1, i] = mp.sqrt(beta[i + 1])
    e, v = mp.eigsy(jac)
    order = sorted(range(n), key=lambda i: e[i])
    return [e[i] for i in order], [beta[0] * v[0, i] ** 2 for i in order]


def hermite_half(n):
    """Positive Gauss-Hermite nodes/weights of order 2n (Golub-Welsch)."""
    mp.mp.dps = DPS
    m = 2 * n
    jac = mp.zeros(m)
    for k in range(1, m):
        jac[k - 1, k] = jac[k, k - 1] = mp.sqrt(mp.mpf(k) / 2)
    e, v = mp.eigsy(jac)
    out = sorted([(e[i], mp.sqrt(mp.pi) * v[0, i] ** 2) for i in range(m) if e[i] > 0])
    return [s for s, _ in out], [h for _, h in out]


def asym(n, t, herm):
    s, h = herm
    t = mp.mpf(t)
    return [si ** 2 / t for si in s], [hi / mp.sqrt(t) for hi in h]


def find_asym_start(n):
    mp.mp.dps = DPS
    herm = hermite_half(n)
    k = 4
    while True:
        ok = True
        for t in [k + d for d in (0, 0.5, 1, 3, 7, 15, 31)]:
            x, w = rys(n, t)
            xa, wa = asym(n, t, herm)
            err = max(max(abs(a / b - 1) for a, b in zip(xa, x)), max(abs(a / b - 1) for a, b in zip(wa, w)))
            if err > 4e-16:
                ok = False
                break
        if ok:
            return k, herm
        k += 1


def cheb_coeffs(vals):
    nn = len(vals)
    c = []
    for j in range(nn):
        c.append(2 * mp.fsum(vals[k] * mp.cos(mp.pi * j * (k + mp.mpf(1) / 2) / nn) for k in range(nn)) / nn)
    c[0] /= 2
    return c


def table_for(n):
    mp.mp.dps = DPS
    kmax, herm = find_asym_start(n)
    nodes = [mp.cos(mp.pi * (k + mp.mpf(1) / 2) / (DEG + 1)) for k in range(DEG + 1)]
    coeffs = []   # [interval][coef][func]
    worst = 0.0
    for iv in range(kmax):
        samples = [rys(n, iv + (s + 1) / 2) for s in nodes]
        funcs = [[smp[0][i] for smp in samples] for i in range(n)] + \
                [[smp[1][i] for smp in samples] for i in range(n)]
        cs = [cheb_coeffs(f) for f in funcs]
        coeffs.append([[float(cs[f][c]) for f in range(2 * n)] for c in range(DEG + 1)])
        for s in (-1.0, -0.37, 0.21, 0.9):
            x, w = rys(n, iv + (s + 1) / 2)
            exact = [float(v) for v in x + w]
            for f in range(2 * n):
                b1 = b2 = 0.0
                for c in range(DEG, 0, -1):
                    b1, b2 = coeffs[-1][c][f] + 2 * s * b1 - b2, b1
                val = coeffs[-1][0][f] + s * b1 - b2
                worst = max(worst, abs(val / exact[f] - 1))
    return n, kmax, coeffs, [float(v) for v in herm[0]], [float(v) for v in herm[1]], worst


def boys_grid():
    mp.mp.dps = DPS
    rows = []
    for k in range(BOYS_TMAX * BOYS_STEP_INV + 1):
        t = mp.mpf(k) / BOYS_STEP_INV
        rows.append([float(boys(m, t)) for m in range(BOYS_MMAX + BOYS_TERMS)])
    return rows


def hx(v):
    return float(v).hex()


def main():
    with mproc.get_context("spawn").Pool(min(8, RYS_MAX_N)) as pool:
        results = pool.map(table_for, range(1, RYS_MAX_N + 1))
    grid = boys_grid()
    lines = ["// Generated by gen_tables.py -- do not edit.  Rys roots/weights as",
             "// piecewise Chebyshev series on unit T intervals, large-T Hermite limits,",
             "// and a Boys-function Taylor grid.  See gen_tables.py for the method.",
             "#pragma once",
             f"#define RYS_MAX_N {RYS_MAX_N}",
             f"#define RYS_NCOEF {DEG + 1}",
             f"#define BOYS_STEP_INV {BOYS_STEP_INV}",
             f"#define BOYS_TMAX {BOYS_TMAX}",
             f"#define BOYS_MMAX {BOYS_MMAX}",
             f"#define BOYS_TERMS {BOYS_TERMS}",
             f"#define BOYS_NCOL {BOYS_MMAX + BOYS_TERMS}",
             f"#define BOYS_NROW {BOYS_TMAX * BOYS_STEP_INV + 1}"]
    nints = [0] * (RYS_MAX_N + 1)
    offsets = [0] * (RYS_MAX_N + 2)
    flat = []
    for n, kmax, coeffs, s, h, worst in results:
        nints[n] = kmax
        offsets[n] = len(flat)
        for iv in coeffs:
            for c in iv:
                flat.extend(c)
        print(f"n={n}: {kmax} intervals, max rel err {worst:.2e}")
    offsets[RYS_MAX_N + 1] = len(flat)
    lines.append("static const int kRysIntervals[RYS_MAX_N + 1] = {" + ",".join(map(str, nints)) + "};")
    lines.append("static const int kRysOffset[RYS_MAX_N + 2] = {" + ",".join(map(str, offsets[:RYS_MAX_N + 2])) + "};")
    lines.append(f"#define RYS_TABLE_SIZE {len(flat)}")
    lines.append("static const double kRysTable[RYS_TABLE_SIZE] = {")
    for i in range(0, len(flat), 4):
        lines.append("  " + ",".join(hx(v) for v in flat[i:i + 4]) + ",")
    lines.append("};")
    asym_r = [[0.0] * RYS_MAX_N for _ in range(RYS_MAX_N + 1)]
    asym_w = [[0.0] * RYS_MAX_N for _ in range(RYS_MAX_N + 1)]
    for n, kmax, coeffs, s, h, worst in results:
        for i in range(n):
            asym_r[n][i] = s[i] ** 2
            asym_w[n][i] = h[i]
    lines.append("static const double kRysAsymR[(RYS_MAX_N + 1) * RYS_MAX_N] = {")
    for row in asym_r:
        lines.append("  " + ",".join(hx(v) for v in row) + ",")
    lines.append("};")
    lines.append("static const double kRysAsymW[(RYS_MAX_N + 1) * RYS_MAX_N] = {")
    for row in asym_w:
        lines.append("  " + ",".join(hx(v) for v in row) + ",")
    lines.append("};")
    lines.append("static const double kBoysGrid[BOYS_NROW * BOYS_NCOL] = {")
    for row in grid:
        lines.append("  " + ",".join(hx(v) for v in row) + ",")
    lines.append("};")
    out = Path(__file__).with_name("rys_tables.h")
    out.write_text("\n".join(lines) + "\n")
    print(f"wrote {out} ({out.stat().st_size} bytes, {len(flat)} Rys coefficients)")


if __name__ == "__main__":
    main()
