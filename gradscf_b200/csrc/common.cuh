// Shared device code: class traits, Cartesian component tables, the Boys
// function and Rys roots/weights (tables generated by gen_tables.py).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#define B200JK_PI 3.14159265358979323846
// 2 pi^(5/2): prefactor of the (ss|ss) integral, 2 pi^2.5 / (p q sqrt(p+q)).
#define B200JK_ERI_C0 34.98683665524972497

namespace b200jk {

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Cartesian component ordering of libcint: lx descending, then ly descending
// (xx, xy, xz, yy, yz, zz for d).  Index i of shell l -> exponents.
__host__ __device__ constexpr int cart_lx(int l, int i) {
  int lx = l, k = i;
  while (k > l - lx) { k -= l - lx + 1; --lx; }
  return lx;
}
__host__ __device__ constexpr int cart_ly(int l, int i) {
  int lx = l, k = i;
  while (k > l - lx) { k -= l - lx + 1; --lx; }
  return l - lx - k;
}
__host__ __device__ constexpr int cart_lz(int l, int i) {
  return l - cart_lx(l, i) - cart_ly(l, i);
}

// Compile-time loop: f(std::integral_constant<int, I>) for I in [B, E), so
// indices derived from I are constant expressions (register arrays stay in
// registers).
template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

// The same over [0, N) as one fold expression (no recursion depth, so long
// loops stay inlined).
template <typename F, int... I>
__device__ __forceinline__ void static_for_seq(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for_n(F&& f) {
  static_for_seq(f, std::make_integer_sequence<int, N>{});
}

template <int LA, int LB, int LC, int LD>
struct ClassInfo {
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  static constexpr int NAB = NA * NB, NCD = NC * ND, NOUT = NAB * NCD;
  static constexpr int LAB = LA + LB, LCD = LC + LD, L = LAB + LCD;
  static constexpr int NROOT = L / 2 + 1;
  static constexpr int NG = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
  static constexpr int NV = (LAB + 1) * (LCD + 1);
};

__host__ __device__ constexpr int binom(int n, int k) {
  int r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

template <typename R> __device__ __forceinline__ R dexp(R x);
template <> __device__ __forceinline__ double dexp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float dexp<float>(float x) { return __expf(x); }
template <typename R> __device__ __forceinline__ R dsqrt(R x);
template <> __device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }
// FP32 quartets need ~1e-7 relative accuracy: hardware approximations (a
// few ulp) instead of the IEEE-rounded sequences; arguments are positive.
template <> __device__ __forceinline__ float dsqrt<float>(float x) { return x * rsqrtf(x); }
template <typename R> __device__ __forceinline__ R drsqrt(R x);
template <> __device__ __forceinline__ double drsqrt<double>(double x) { return rsqrt(x); }
template <> __device__ __forceinline__ float drsqrt<float>(float x) { return rsqrtf(x); }

// Device-resident lookup tables (see gen_tables.py for their definition).
struct Tables {
  const double* rys;        // Chebyshev coefficients, [n][interval][coef][2n]
  const float* rys_f;       // same, float
  const int* rys_off;       // offset of each n in rys
  const int* rys_nint;      // number of tabulated unit intervals per n
  const double* asym_r;     // [n][RYS_MAX_N] large-T root numerators s_i^2
  const double* asym_w;     // [n][RYS_MAX_N] large-T weight numerators h_i
  const double* boys;       // [row][col] F_col(row / BOYS_STEP_INV)
  const float* boys_f;
  const double* c2s;        // per l: [kTW][kTW] output transform (cart->sph or cart factor)
  // Per-order Taylor tables for the closed-form roots: for M = 1, 3, 5 (table
  // (M-1)/2), row k holds F_{M+i}(k/20) / i!, i = 0..7 -- one aligned 64-byte
  // (double) / 32-byte (float) row per lookup.
  const double* boys_m;
  const float* boys_m_f;
  // FP32 copies at spacing 1/10 (401 rows of 8, terms F_{M+i}/i!), staged in
  // shared memory by the FP32 register path.
  const float* boys_s_f;
};

// Output-transform table layout: per l a kTW x kTW block, row = raw Cartesian
// component, column = output function (up to 10 for Cartesian f).
constexpr int kTW = 10;
constexpr int kTS = kTW * kTW;

// Boys function F_0..F_M(T) into f[0..M], M in {1, 3, 5}.
// T < 40: Taylor expansion of F_M about the nearest grid point (spacing
// 1/20; 8 terms in FP64, 5 in FP32) followed by the stable downward recursion
//   F_m = (2 T F_{m+1} + e^{-T}) / (2m + 1).
// T >= 40: F_0 = sqrt(pi/T)/2 and the stable upward recursion
//   F_{m+1} = ((2m+1) F_m - e^{-T}) / (2T).
// (Taylor/downward scheme: Gill, Johnson & Pople, Int. J. Quantum Chem. 40, 745 (1991).)
// Division-free: constant divisors are multiplications by folded reciprocals.
template <int M, typename R, int SINV = 20, int NT = (sizeof(R) == 8 ? 8 : 5)>
__device__ __forceinline__ void boys_fn(R t, R* f, const R* tab) {
  // tab: this order's table, rows of 8 at spacing 1/SINV over [0, 40]
  if (t < R(40)) {
    const int k = min(max(__float2int_rn(float(t) * float(SINV)), 0), 40 * SINV);
    const R dt = R(k) * R(1.0 / SINV) - t;          // -(t - t_k)
    const R* row = tab + k * 8;
    R c[8];
    if constexpr (sizeof(R) == 8) {
      const double4 a = reinterpret_cast<const double4*>(row)[0];
      const double4 b = reinterpret_cast<const double4*>(row)[1];
      c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w; c[4] = b.x; c[5] = b.y; c[6] = b.z; c[7] = b.w;
    } else {
      const float4 a = reinterpret_cast<const float4*>(row)[0];
      const float4 b = reinterpret_cast<const float4*>(row)[1];
      c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w; c[4] = b.x; c[5] = b.y; c[6] = b.z; c[7] = b.w;
    }
    R acc = c[NT - 1];
#pragma unroll
    for (int i = NT - 2; i >= 0; --i) acc = c[i] + acc * dt;
    f[M] = acc;
    const R e = dexp<R>(-t);
    const R t2 = t + t;
#pragma unroll
    for (int m = M - 1; m >= 0; --m) f[m] = (t2 * f[m + 1] + e) * R(1.0 / (2 * m + 1));
  } else {
    const R e = dexp<R>(-t);
    const R rs = drsqrt<R>(t);
    f[0] = R(0.886226925452758014) * rs;      // sqrt(pi)/2 / sqrt(t)
    const R inv2t = R(0.5) * rs * rs;
#pragma unroll
    for (int m = 0; m < M; ++m) f[m + 1] = (R(2 * m + 1) * f[m] - e) * inv2t;
  }
}

template <typename R> __device__ __forceinline__ R drcp(R x);
template <> __device__ __forceinline__ double drcp<double>(double x) { return 1.0 / x; }
template <> __device__ __forceinline__ float drcp<float>(float x) { return __fdividef(1.0f, x); }

// Rys nodes x_i = t_i^2 and weights w_i for N <= 3 from the Boys moments
// mu_k = F_k(T) (k < 2N): Gautschi's Chebyshev algorithm gives the Jacobi
// matrix (alpha_k, beta_k); its eigenvalues are the nodes and
// w_i = F_0 / sum_k p_k(x_i)^2 with the orthonormal recurrence polynomials
// p_k.  N = 2 is a closed-form quadratic; N = 3 solves the cubic by the
// trigonometric formula in float and polishes each node with two Newton
// steps in R.  Max relative error vs 60-digit values: 2e-15 (N <= 2),
// 2e-14 (N = 3), both in FP64.
template <int N, typename R, int SINV = 20, int NT = (sizeof(R) == 8 ? 8 : 5)>
__device__ __forceinline__ void rys_small(R t, R* x, R* w, const R* tab) {
  // tab: Taylor table of order M = 2N - 1
  if (N == 1) {
    R f[2];
    boys_fn<1, R, SINV, NT>(t, f, tab);
    w[0] = f[0];
    x[0] = f[1] * drcp<R>(f[0]);
  } else if (N == 2) {
    R f[4];
    boys_fn<3, R, SINV, NT>(t, f, tab);
    const R inv0 = drcp<R>(f[0]);
    const R a0 = f[1] * inv0;
    const R s11 = f[2] - a0 * f[1];
    const R s12 = f[3] - a0 * f[2];
    const R a1 = s12 * drcp<R>(s11) - a0;
    const R b1 = s11 * inv0;
    const R mid = R(0.5) * (a0 + a1), hd = R(0.5) * (a0 - a1);
    const R rad = dsqrt<R>(hd * hd + b1);
    const R xp = mid + rad;
    const R xm = (a0 * a1 - b1) * drcp<R>(xp);
    x[0] = xm;
    x[1] = xp;
    const R dm = xm - a0, dp = xp - a0;
    const R fb = f[0] * b1;
    w[0] = fb * drcp<R>(b1 + dm * dm);
    w[1] = fb * drcp<R>(b1 + dp * dp);
  } else {
    R f[6];
    boys_fn<5, R, SINV, NT>(t, f, tab);
    const R inv0 = drcp<R>(f[0]);
    const R a0 = f[1] * inv0;
    const R s11 = f[2] - a0 * f[1], s12 = f[3] - a0 * f[2];
    const R s13 = f[4] - a0 * f[3], s14 = f[5] - a0 * f[4];
    const R i11 = drcp<R>(s11);
    const R a1 = s12 * i11 - a0;
    const R b1 = s11 * inv0;
    const R s22 = s13 - a1 * s12 - b1 * f[2];
    const R s23 = s14 - a1 * s13 - b1 * f[3];
    const R a2 = s23 * drcp<R>(s22) - s12 * i11;
    const R b2 = s22 * i11;
    const R c2 = -(a0 + a1 + a2);
    const R c1 = a0 * a1 + a0 * a2 + a1 * a2 - b1 - b2;
    const R c0 = -a0 * a1 * a2 + a0 * b2 + a2 * b1;
    const R m = c2 * R(-1.0 / 3.0);
    const R d0 = a0 - m, d1 = a1 - m, d2 = a2 - m;
    const R p = R(-0.5) * (d0 * d0 + d1 * d1 + d2 * d2 + R(2) * (b1 + b2));
    const R q = -(d0 * d1 * d2 - d0 * b2 - d2 * b1);
    const float r = dsqrt<float>(float(-p) * (1.0f / 3.0f));
    const float cth = fminf(fmaxf(__fdividef(-float(q), 2.0f * r * r * r), -1.0f), 1.0f);
    const float th = acosf(cth) * (1.0f / 3.0f);
    const R sb1 = dsqrt<R>(b1), sb2 = dsqrt<R>(b2);
    const R isb1 = drcp<R>(sb1), isb2 = drcp<R>(sb2);
    R lam[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      R l = R(2.0f * r * __cosf(th - 2.0943951023931955f * float(k))) + m;   // polished below
      const R dpi = R(1.0f / float((R(3) * l + R(2) * c2) * l + c1));
#pragma unroll
      for (int it = 0; it < 2; ++it) l -= (((l + c2) * l + c1) * l + c0) * dpi;
      lam[k] = l;
    }
    // theta in [0, pi/3]: k = 0 gives the largest node, k = 2 the smallest
    x[0] = lam[2];
    x[1] = lam[1];
    x[2] = lam[0];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const R p1 = (x[i] - a0) * isb1;
      const R p2 = ((x[i] - a1) * p1 - sb1) * isb2;
      w[i] = f[0] * drcp<R>(R(1) + p1 * p1 + p2 * p2);
    }
  }
}

// One Rys function (root or weight index fidx of N) from the Chebyshev table.
template <typename R>
__device__ __forceinline__ R rys_cheb(const R* tab, int off, int nfun, int fidx, int interval, R s) {
  const R* c = tab + off + interval * 12 * nfun + fidx;
  R b1 = R(0), b2 = R(0);
  const R s2 = s + s;
#pragma unroll
  for (int k = 11; k >= 1; --k) {
    const R b0 = c[k * nfun] + s2 * b1 - b2;
    b2 = b1;
    b1 = b0;
  }
  return c[0] + s * b1 - b2;
}

template <typename R> struct TableSel;
template <> struct TableSel<double> {
  static __device__ __forceinline__ const double* rys(const Tables& t) { return t.rys; }
  static __device__ __forceinline__ const double* boys(const Tables& t) { return t.boys_m; }
};
template <> struct TableSel<float> {
  static __device__ __forceinline__ const float* rys(const Tables& t) { return t.rys_f; }
  static __device__ __forceinline__ const float* boys(const Tables& t) { return t.boys_m_f; }
};

// All N nodes/weights by one thread: closed forms for N <= 3, the
// Chebyshev table (or the large-T Hermite limit) above.
template <int N, typename R>
__device__ __forceinline__ void rys_roots(R t, R* x, R* w, const Tables& tb) {
  if (N <= 3) {
    rys_small<N, R>(t, x, w, TableSel<R>::boys(tb) + (N - 1) * 801 * 8);
    return;
  }
  const int nint = tb.rys_nint[N];
  if (t >= R(nint)) {
    const R rt = drcp<R>(t), rs = drsqrt<R>(t);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      x[i] = R(tb.asym_r[N * 8 + i]) * rt;
      w[i] = R(tb.asym_w[N * 8 + i]) * rs;
    }
    return;
  }
  const int k = min(max(int(t), 0), nint - 1);
  const R s = R(2) * (t - R(k)) - R(1);
  const R* tab = TableSel<R>::rys(tb);
  const int off = tb.rys_off[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    x[i] = rys_cheb<R>(tab, off, 2 * N, i, k, s);
    w[i] = rys_cheb<R>(tab, off, 2 * N, N + i, k, s);
  }
}

// One of the 2N functions (index f: nodes 0..N-1 then weights) -- used when
// several threads share one primitive quartet.
template <int N, typename R>
__device__ __forceinline__ R rys_one(R t, int f, const Tables& tb) {
  // several lanes share the quartet: for N >= 3 each lane evaluates one
  // Chebyshev series of the same interval (near-broadcast reads) instead of
  // every lane running the closed-form solve
  if (N <= 2) {
    R x[N], w[N];
    rys_small<N, R>(t, x, w, TableSel<R>::boys(tb) + (N - 1) * 801 * 8);
    R v = x[0];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      if (f == i) v = x[i];
      if (f == N + i) v = w[i];
    }
    return v;
  }
  const int nint = tb.rys_nint[N];
  if (t >= R(nint)) {
    if (f < N) return R(tb.asym_r[N * 8 + f]) / t;
    return R(tb.asym_w[N * 8 + f - N]) * drsqrt<R>(t);
  }
  const int k = min(max(int(t), 0), nint - 1);
  const R s = R(2) * (t - R(k)) - R(1);
  return rys_cheb<R>(TableSel<R>::rys(tb), tb.rys_off[N], 2 * N, f, k, s);
}

// 2D Rys integrals of one (root, axis): VRR to V[e][f] (e <= LA+LB,
// f <= LC+LD) from
//   V[e+1][f] = C00 V[e][f] + e B10 V[e-1][f] + f B00 V[e][f-1]
//   V[e][f+1] = C0p V[e][f] + f B01 V[e][f-1] + e B00 V[e-1][f]
// then the horizontal transfers, ket first then bra:
//   W[e][c][d+1] = W[e][c+1][d] + CD W[e][c][d],
//   G[a][b+1][cd] = G[a+1][b][cd] + AB G[a][b][cd]
// (AB = A - B, CD = C - D along the axis).  G layout:
// ((a*(LB+1)+b)*(LC+1)+c)*(LD+1)+d.
template <int LA, int LB, int LC, int LD, typename R, typename GPtr>
__device__ __forceinline__ void build_g(R c00, R c0p, R b10, R b01, R b00, R g00, R ab, R cd,
                                        GPtr G) {
  constexpr int LAB = LA + LB, LCD = LC + LD;
  R v[LAB + 1][LCD + 1];
  v[0][0] = g00;
  if (LAB > 0) v[1][0] = c00 * g00;
#pragma unroll
  for (int e = 1; e < LAB; ++e) v[e + 1][0] = c00 * v[e][0] + R(e) * b10 * v[e - 1][0];
#pragma unroll
  for (int f = 0; f < LCD; ++f) {
#pragma unroll
    for (int e = 0; e <= LAB; ++e) {
      R val = c0p * v[e][f];
      if (f > 0) val += R(f) * b01 * v[e][f - 1];
      if (e > 0) val += R(e) * b00 * v[e - 1][f];
      v[e][f + 1] = val;
    }
  }
  // ket transfer: w[e][c][d], c <= LCD - d
  R w[LAB + 1][LCD + 1][LD + 1];
#pragma unroll
  for (int e = 0; e <= LAB; ++e) {
#pragma unroll
    for (int c = 0; c <= LCD; ++c) w[e][c][0] = v[e][c];
#pragma unroll
    for (int d = 1; d <= LD; ++d)
#pragma unroll
      for (int c = 0; c <= LCD - d; ++c) w[e][c][d] = w[e][c + 1][d - 1] + cd * w[e][c][d - 1];
  }
  // bra transfer per (c, d)
#pragma unroll
  for (int c = 0; c <= LC; ++c)
#pragma unroll
    for (int d = 0; d <= LD; ++d) {
      R y[LAB + 1][LB + 1];
#pragma unroll
      for (int a = 0; a <= LAB; ++a) y[a][0] = w[a][c][d];
#pragma unroll
      for (int b = 1; b <= LB; ++b)
#pragma unroll
        for (int a = 0; a <= LAB - b; ++a) y[a][b] = y[a + 1][b - 1] + ab * y[a][b - 1];
#pragma unroll
      for (int a = 0; a <= LA; ++a)
#pragma unroll
        for (int b = 0; b <= LB; ++b) G[((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d] = y[a][b];
    }
}

// The same table with the recursion held in memory instead of registers:
// the vertical recursion advances one f column at a time (two columns in
// registers), the ket transfer runs in `w` ((LAB+1)(LCD+1)(LD+1) values,
// shared or local memory) and the bra transfer per (c, d) keeps one column
// of LAB+1 values.  For large classes, whose register-held recursion would
// cap the occupancy of the whole kernel.
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void build_g_mem(R c00, R c0p, R b10, R b01, R b00, R g00, R ab, R cd, R* G,
                                            R* w) {
  constexpr int LAB = LA + LB, LCD = LC + LD;
  auto W = [&](int e, int c, int d) -> R& { return w[(e * (LCD + 1) + c) * (LD + 1) + d]; };
  R prev[LAB + 1], cur[LAB + 1];
  cur[0] = g00;
  if (LAB > 0) cur[1] = c00 * g00;
#pragma unroll
  for (int e = 1; e < LAB; ++e) cur[e + 1] = c00 * cur[e] + R(e) * b10 * cur[e - 1];
#pragma unroll
  for (int e = 0; e <= LAB; ++e) {
    W(e, 0, 0) = cur[e];
    prev[e] = R(0);
  }
#pragma unroll
  for (int f = 0; f < LCD; ++f) {
    R next[LAB + 1];
#pragma unroll
    for (int e = 0; e <= LAB; ++e) {
      R val = c0p * cur[e];
      if (f > 0) val += R(f) * b01 * prev[e];
      if (e > 0) val += R(e) * b00 * cur[e - 1];
      next[e] = val;
    }
#pragma unroll
    for (int e = 0; e <= LAB; ++e) {
      prev[e] = cur[e];
      cur[e] = next[e];
      W(e, f + 1, 0) = next[e];
    }
  }
#pragma unroll
  for (int e = 0; e <= LAB; ++e)
#pragma unroll
    for (int d = 1; d <= LD; ++d)
#pragma unroll
      for (int c = 0; c <= LCD - d; ++c) W(e, c, d) = W(e, c + 1, d - 1) + cd * W(e, c, d - 1);
#pragma unroll
  for (int c = 0; c <= LC; ++c)
#pragma unroll
    for (int d = 0; d <= LD; ++d) {
      R y[LAB + 1];
#pragma unroll
      for (int e = 0; e <= LAB; ++e) y[e] = W(e, c, d);
#pragma unroll
      for (int b = 0; b <= LB; ++b) {
#pragma unroll
        for (int a = 0; a <= LA; ++a) G[((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d] = y[a];
        if (b < LB) {
#pragma unroll
          for (int a = 0; a + b < LAB; ++a) y[a] = y[a + 1] + ab * y[a];
        }
      }
    }
}

}  // namespace b200jk
