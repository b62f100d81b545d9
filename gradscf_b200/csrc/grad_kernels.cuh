// Coordinate VJP of J/K: sum over canonical screened quartets of
//   dE = sum_abcd d(ab|cd)/dR * Gamma_abcd,
// Gamma = the eight-permutation symmetrisation (times the degeneracy scale
// s of load_quartet) of  Jbar_ab D_cd + Kbar_ac D_bd  (the reference's
// transposed contraction, csrc/direct_jk_geometry.cc:68-84, which runs over
// all n^4 entries instead).  Derivatives recomputed, never stored:
//   d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x}  (same for B, C),
//   d/dD = -(d/dA + d/dB + d/dC)  (translational invariance).
// Team layout as the J/K team path: 2D integrals with raised bra/ket
// indices in shared memory, each lane owns a strided slice of the Cartesian
// block, nine gradient partials per lane reduced across the team.
#pragma once
#include "jk_kernels.cuh"

namespace b200jk {

template <int LA, int LB, int LC, int LD, int TEAM>
struct GradCfg {
  using CI = ClassInfo<LA, LB, LC, LD>;
  static constexpr int NROOT = (CI::L + 1) / 2 + 1;
  static constexpr int NG = (LA + 2) * (LB + 2) * (LC + 2) * (LD + 1);
  static constexpr int NK = (CI::NOUT + TEAM - 1) / TEAM;
  static constexpr int ELEMS = 3 * NROOT * NG + 2 * NROOT;
  static constexpr size_t bytes() { return (size_t)ELEMS * 8; }
  __host__ __device__ static constexpr int idx(int a, int b, int c, int d) {
    return ((a * (LB + 2) + b) * (LC + 2) + c) * (LD + 1) + d;
  }
};

// Raw Cartesian Gamma of one AO quartet (a, b, c, d), summed over batches.
__device__ __forceinline__ double gamma_abcd(const JKArgs& args, long long base, int n, int a, int b,
                                             int c, int d) {
  double gsum = 0.0;
  for (int e = 0; e < args.gnb; ++e) {
    const double* D = args.dens + e * args.dstride + base;
    const double* J = args.cot_j ? args.cot_j + e * args.dstride + base : nullptr;
    const double* K = args.cot_k ? args.cot_k + e * args.dstride + base : nullptr;
#define M_(X, i, j) X[(long long)(i) * n + (j)]
    if (J)
      gsum += (M_(J, a, b) + M_(J, b, a)) * (M_(D, c, d) + M_(D, d, c)) +
              (M_(J, c, d) + M_(J, d, c)) * (M_(D, a, b) + M_(D, b, a));
    if (K)
      gsum += M_(K, a, c) * M_(D, b, d) + M_(K, c, a) * M_(D, d, b) + M_(K, b, c) * M_(D, a, d) +
              M_(K, c, b) * M_(D, d, a) + M_(K, a, d) * M_(D, b, c) + M_(K, d, a) * M_(D, c, b) +
              M_(K, b, d) * M_(D, a, c) + M_(K, d, b) * M_(D, c, a);
#undef M_
  }
  return gsum;
}

// Ket range of a coordinate-VJP work item for the requested precision slice
// (split_mode 1: the kets before the item's FP32 boundary, 2: from it on).
__device__ __forceinline__ void grad_ket_range(const JKArgs& args, int item, const int4 w, int& kb, int& ke) {
  kb = w.y;
  ke = w.z;
  if (args.split_mode != 0) {
    const int s = args.split[item];
    if (args.split_mode == 1) ke = min(ke, s);
    else kb = max(kb, s);
  }
}

// One primitive quartet's scalars in precision R (FP32 quartets: the pair
// data stored relative to A and C, centre differences formed in FP64).
template <typename R>
__device__ __forceinline__ void grad_prim(const JKArgs& args, const QuartetGeom& g, int i, int j, PrimQ<R>& s) {
  const float3 ac = make_float3(float(g.ax - g.cx), float(g.ay - g.cy), float(g.az - g.cz));
  prim_any<R>(g, ac, PrimData<R>::a(args, i), PrimData<R>::b(args, i), PrimData<R>::a(args, j),
              PrimData<R>::b(args, j), s);
}

template <int LA, int LB, int LC, int LD, int TEAM, typename R>
__global__ void grad_team_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GC = GradCfg<LA, LB, LC, LD, TEAM>;
  constexpr int N = GC::NROOT;
  constexpr int NG = GC::NG;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x % TEAM;
  const int team = threadIdx.x / TEAM;
  const int nteams = blockDim.x / TEAM;
  const unsigned mask =
      TEAM == 32 ? 0xffffffffu : (((1u << TEAM) - 1u) << ((threadIdx.x % 32) / TEAM * TEAM));
  R* G = reinterpret_cast<R*>(smem_raw) + (size_t)team * GC::ELEMS;
  R* roots = G + 3 * N * NG;
  const int4 w = args.work[blockIdx.x];
  const int bra = args.bra_pairs[w.x];
  int kb, ke;
  grad_ket_range(args, blockIdx.x, w, kb, ke);
  for (int k = kb + team; k < ke; k += nteams) {
    QuartetGeom g;
    load_quartet(args, bra, args.ket_pairs[k], g);
    const long long base = args.mol_base[g.mol];
    const int n = args.mol_n[g.mol];
    R gam[GC::NK];
    int exps[GC::NK];   // packed exponent digits of (a, b, c, d) per axis
#pragma unroll
    for (int q = 0; q < GC::NK; ++q) {
      const int o = lane + q * TEAM;
      gam[q] = R(0);
      exps[q] = -1;
      if (o < CI::NOUT) {
        const int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
        const int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
        gam[q] = R(g.scale * gamma_abcd(args, base, n, g.aoA + ia, g.aoB + ib, g.aoC + ic, g.aoD + id));
        exps[q] = ia | (ib << 4) | (ic << 8) | (id << 12);
      }
    }
    R dA[3] = {0, 0, 0}, dB[3] = {0, 0, 0}, dC[3] = {0, 0, 0};
    for (int i = g.ppa; i < g.ppa + g.npa; ++i) {
      const R alpha = R(args.pp_exp[i].x), beta = R(args.pp_exp[i].y);
      for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
        PrimQ<R> s;
        grad_prim<R>(args, g, i, j, s);
        const R gamma_c = R(args.pp_exp[j].x);
        for (int f = lane; f < 2 * N; f += TEAM) roots[f] = rys_one<N, R>(s.t, f, args.tb);
        __syncwarp(mask);
        for (int tsk = lane; tsk < 3 * N; tsk += TEAM) {
          const int r = tsk / 3, ax = tsk - 3 * r;
          RootCoef<R> rc;
          root_coef<R>(s, roots[r], rc);
          const R abd = R(ax == 0 ? g.abx : (ax == 1 ? g.aby : g.abz));
          const R cdd = R(ax == 0 ? g.cdx : (ax == 1 ? g.cdy : g.cdz));
          const R g00 = ax == 2 ? roots[N + r] * s.pref : R(1);
          build_g<LA + 1, LB + 1, LC + 1, LD, R>(rc.c00[ax], rc.c0p[ax], rc.b10, rc.b01, rc.b00, g00, abd, cdd,
                                                 G + (r * 3 + ax) * NG);
        }
        __syncwarp(mask);
#pragma unroll
        for (int q = 0; q < GC::NK; ++q) {
          if (exps[q] < 0 || gam[q] == R(0)) continue;
          const int ia = exps[q] & 15, ib = (exps[q] >> 4) & 15, ic = (exps[q] >> 8) & 15, id = exps[q] >> 12;
          const int la[3] = {cart_lx(LA, ia), cart_ly(LA, ia), cart_lz(LA, ia)};
          const int lb[3] = {cart_lx(LB, ib), cart_ly(LB, ib), cart_lz(LB, ib)};
          const int lc[3] = {cart_lx(LC, ic), cart_ly(LC, ic), cart_lz(LC, ic)};
          const int ld[3] = {cart_lx(LD, id), cart_ly(LD, id), cart_lz(LD, id)};
          for (int r = 0; r < N; ++r) {
            R v[3], fa[3], fb[3], fc[3];
#pragma unroll
            for (int x = 0; x < 3; ++x) {
              const R* Gx = G + (r * 3 + x) * NG;
              const int a = la[x], b = lb[x], c = lc[x], d = ld[x];
              v[x] = Gx[GC::idx(a, b, c, d)];
              fa[x] = R(2) * alpha * Gx[GC::idx(a + 1, b, c, d)] - (a ? R(a) * Gx[GC::idx(a - 1, b, c, d)] : R(0));
              fb[x] = R(2) * beta * Gx[GC::idx(a, b + 1, c, d)] - (b ? R(b) * Gx[GC::idx(a, b - 1, c, d)] : R(0));
              fc[x] = R(2) * gamma_c * Gx[GC::idx(a, b, c + 1, d)] - (c ? R(c) * Gx[GC::idx(a, b, c - 1, d)] : R(0));
            }
            const R gq = gam[q];
            const R yz = v[1] * v[2], xz = v[0] * v[2], xy = v[0] * v[1];
            dA[0] += gq * fa[0] * yz; dA[1] += gq * fa[1] * xz; dA[2] += gq * fa[2] * xy;
            dB[0] += gq * fb[0] * yz; dB[1] += gq * fb[1] * xz; dB[2] += gq * fb[2] * xy;
            dC[0] += gq * fc[0] * yz; dC[1] += gq * fc[1] * xz; dC[2] += gq * fc[2] * xy;
          }
        }
        __syncwarp(mask);
      }
    }
    // reduce the nine partials over the team; lane 0 adds to the four centres
#pragma unroll
    for (int x = 0; x < 3; ++x)
#pragma unroll
      for (int off = TEAM / 2; off > 0; off >>= 1) {
        dA[x] += __shfl_down_sync(mask, dA[x], off, TEAM);
        dB[x] += __shfl_down_sync(mask, dB[x], off, TEAM);
        dC[x] += __shfl_down_sync(mask, dC[x], off, TEAM);
      }
    if (lane == 0) {
      double* gA = args.grad + 3LL * args.ws_atm[g.A];
      double* gB = args.grad + 3LL * args.ws_atm[g.B];
      double* gC = args.grad + 3LL * args.ws_atm[g.C];
      double* gD = args.grad + 3LL * args.ws_atm[g.D];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        atomicAdd(gA + x, double(dA[x]));
        atomicAdd(gB + x, double(dB[x]));
        atomicAdd(gC + x, double(dC[x]));
        atomicAdd(gD + x, -(double(dA[x]) + double(dB[x]) + double(dC[x])));
      }
    }
  }
}

}  // namespace b200jk

namespace b200jk {

// ---------------------------------------------------------------------------
// Block-wide coordinate VJP for the large classes (NOUT > 256, i.e. d and f
// shells): the whole block works on one quartet at a time.  Gamma of every
// element is staged in shared memory once per quartet; per primitive
// quartet the raised 2D tables of every root and axis are built in shared
// memory (build_g_mem, one thread per table, recursion scratch in shared
// memory so the kernel's register count stays that of the accumulation);
// the threads then stride over the elements, each summing the nine centre
// partials, which are block-reduced per quartet.
// ---------------------------------------------------------------------------
template <int LA, int LB, int LC, int LD>
struct GradBlk {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GC = GradCfg<LA, LB, LC, LD, 1>;
  static constexpr int THREADS = 128;
  static constexpr int N = GC::NROOT, NG = GC::NG;
  static constexpr int LAB = LA + LB + 2, LCD = LC + LD + 1;
  static constexpr int NW = (LAB + 1) * (LCD + 1) * (LD + 1);   // recursion scratch per table
  static constexpr int G_OFF = 0, R_OFF = 3 * N * NG, W_OFF = R_OFF + 2 * N, GAM_OFF = W_OFF + 3 * N * NW;
  static constexpr int ELEMS = GAM_OFF + CI::NOUT;
  static constexpr size_t bytes() { return (size_t)ELEMS * 8; }   // FP64; FP32 takes half
  static constexpr bool OK = CI::NOUT > 256 && bytes() <= 220 * 1024;
};

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) grad_block_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GB = GradBlk<LA, LB, LC, LD>;
  using GC = GradCfg<LA, LB, LC, LD, 1>;
  constexpr int N = GB::N, NG = GB::NG;
  extern __shared__ __align__(16) unsigned char gsm_raw[];
  R* gsm = reinterpret_cast<R*>(gsm_raw);
  R* G = gsm + GB::G_OFF;
  R* roots = gsm + GB::R_OFF;
  R* scratch = gsm + GB::W_OFF;
  R* gam = gsm + GB::GAM_OFF;
  __shared__ double red[9][GB::THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int4 w = args.work[blockIdx.x];
  const int bra = args.bra_pairs[w.x];
  int kb, ke;
  grad_ket_range(args, blockIdx.x, w, kb, ke);
  for (int k = kb; k < ke; ++k) {
    QuartetGeom g;
    load_quartet(args, bra, args.ket_pairs[k], g);
    const long long base = args.mol_base[g.mol];
    const int n = args.mol_n[g.mol];
    for (int o = tid; o < CI::NOUT; o += GB::THREADS) {
      const int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
      const int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
      gam[o] = R(g.scale * gamma_abcd(args, base, n, g.aoA + ia, g.aoB + ib, g.aoC + ic, g.aoD + id));
    }
    R dA[3] = {0, 0, 0}, dB[3] = {0, 0, 0}, dC[3] = {0, 0, 0};
    for (int i = g.ppa; i < g.ppa + g.npa; ++i) {
      const R alpha = R(args.pp_exp[i].x), beta = R(args.pp_exp[i].y);
      for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
        PrimQ<R> s;
        grad_prim<R>(args, g, i, j, s);
        const R gamma_c = R(args.pp_exp[j].x);
        __syncthreads();   // the previous primitive quartet's tables are no longer read
        if (tid < 2 * N) roots[tid] = rys_one<N, R>(s.t, tid, args.tb);
        __syncthreads();
        if (tid < 3 * N) {
          const int r = tid / 3, ax = tid - 3 * r;
          RootCoef<R> rc;
          root_coef<R>(s, roots[r], rc);
          const R abd = R(ax == 0 ? g.abx : (ax == 1 ? g.aby : g.abz));
          const R cdd = R(ax == 0 ? g.cdx : (ax == 1 ? g.cdy : g.cdz));
          const R g00 = ax == 2 ? roots[N + r] * s.pref : R(1);
          build_g_mem<LA + 1, LB + 1, LC + 1, LD, R>(rc.c00[ax], rc.c0p[ax], rc.b10, rc.b01, rc.b00, g00, abd, cdd,
                                                    G + tid * NG, scratch + tid * GB::NW);
        }
        __syncthreads();
        for (int o = tid; o < CI::NOUT; o += GB::THREADS) {
          const R gq = gam[o];
          if (gq == R(0)) continue;
          const int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
          const int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
          const int la[3] = {cart_lx(LA, ia), cart_ly(LA, ia), cart_lz(LA, ia)};
          const int lb[3] = {cart_lx(LB, ib), cart_ly(LB, ib), cart_lz(LB, ib)};
          const int lc[3] = {cart_lx(LC, ic), cart_ly(LC, ic), cart_lz(LC, ic)};
          const int ld[3] = {cart_lx(LD, id), cart_ly(LD, id), cart_lz(LD, id)};
#pragma unroll 2
          for (int r = 0; r < N; ++r) {
            R v[3], fa[3], fb[3], fc[3];
#pragma unroll
            for (int x = 0; x < 3; ++x) {
              const R* Gx = G + (r * 3 + x) * NG;
              const int a = la[x], b = lb[x], c = lc[x], d = ld[x];
              v[x] = Gx[GC::idx(a, b, c, d)];
              fa[x] = R(2) * alpha * Gx[GC::idx(a + 1, b, c, d)] - (a ? R(a) * Gx[GC::idx(a - 1, b, c, d)] : R(0));
              fb[x] = R(2) * beta * Gx[GC::idx(a, b + 1, c, d)] - (b ? R(b) * Gx[GC::idx(a, b - 1, c, d)] : R(0));
              fc[x] = R(2) * gamma_c * Gx[GC::idx(a, b, c + 1, d)] - (c ? R(c) * Gx[GC::idx(a, b, c - 1, d)] : R(0));
            }
            const R yz = gq * v[1] * v[2], xz = gq * v[0] * v[2], xy = gq * v[0] * v[1];
            dA[0] += fa[0] * yz; dA[1] += fa[1] * xz; dA[2] += fa[2] * xy;
            dB[0] += fb[0] * yz; dB[1] += fb[1] * xz; dB[2] += fb[2] * xy;
            dC[0] += fc[0] * yz; dC[1] += fc[1] * xz; dC[2] += fc[2] * xy;
          }
        }
      }
    }
    // block reduction of the nine partials; thread 0 adds to the four centres
    double part[9] = {double(dA[0]), double(dA[1]), double(dA[2]), double(dB[0]), double(dB[1]),
                      double(dB[2]), double(dC[0]), double(dC[1]), double(dC[2])};
#pragma unroll
    for (int q = 0; q < 9; ++q) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) part[q] += __shfl_down_sync(0xffffffffu, part[q], off);
      if (lane == 0) red[q][warp] = part[q];
    }
    __syncthreads();
    if (tid == 0) {
      double sum[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        sum[q] = 0.0;
        for (int wi = 0; wi < GB::THREADS / 32; ++wi) sum[q] += red[q][wi];
      }
      double* gA = args.grad + 3LL * args.ws_atm[g.A];
      double* gB = args.grad + 3LL * args.ws_atm[g.B];
      double* gC = args.grad + 3LL * args.ws_atm[g.C];
      double* gD = args.grad + 3LL * args.ws_atm[g.D];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        atomicAdd(gA + x, sum[x]);
        atomicAdd(gB + x, sum[3 + x]);
        atomicAdd(gC + x, sum[6 + x]);
        atomicAdd(gD + x, -(sum[x] + sum[3 + x] + sum[6 + x]));
      }
    }
    __syncthreads();   // red and gam are rewritten by the next quartet
  }
}

// Register-path coordinate VJP for small classes: one lane per ket of a
// work item (warp-granular items as the J/K register path), the raised 2D
// integrals of one root in registers, nine derivative partials per lane;
// the bra-centre partials (A, B fixed per warp) are warp-reduced.
template <int LA, int LB, int LC, int LD>
struct GradReg {
  using CI = ClassInfo<LA, LB, LC, LD>;
  static constexpr int NGR = (LA + 2) * (LB + 2) * (LC + 2) * (LD + 1);
#ifndef B200JK_GRAD_REG_LIMIT
#define B200JK_GRAD_REG_LIMIT 96  // measured: (H2O)8 cc-pVTZ gradient 510 -> 479 ms
#endif
  static constexpr bool OK = 3 * NGR + CI::NOUT <= B200JK_GRAD_REG_LIMIT;
};

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128, 3) grad_reg_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GC = GradCfg<LA, LB, LC, LD, 1>;
  using GI = GIdx<LA + 1, LB + 1, LC + 1, LD>;
  constexpr int N = GC::NROOT;
  constexpr int NGR = GradReg<LA, LB, LC, LD>::NGR;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x * 4 + warp;
  if (item >= args.nwork) return;
  const int4 w = args.work[item];
  const int bra = args.bra_pairs[w.x];
  double bA[3] = {0, 0, 0}, bB[3] = {0, 0, 0};
  int atA = 0, atB = 0;
  int kb, ke;
  grad_ket_range(args, item, w, kb, ke);
  for (int k0 = kb; k0 < ke; k0 += 32) {
    const bool active = k0 + lane < ke;
    const int k = active ? k0 + lane : ke - 1;
    QuartetGeom g;
    load_quartet(args, bra, args.ket_pairs[k], g);
    atA = args.ws_atm[g.A];
    atB = args.ws_atm[g.B];
    const long long base = args.mol_base[g.mol];
    const int n = args.mol_n[g.mol];
    R gam[CI::NOUT];
    static_for<0, CI::NOUT>([&](auto O) {
      constexpr int o = decltype(O)::value;
      constexpr int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
      constexpr int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
      gam[o] = active ? R(g.scale * gamma_abcd(args, base, n, g.aoA + ia, g.aoB + ib, g.aoC + ic, g.aoD + id)) : R(0);
    });
    R dA[3] = {0, 0, 0}, dB[3] = {0, 0, 0}, dC[3] = {0, 0, 0};
    for (int i = g.ppa; i < g.ppa + g.npa; ++i) {
      const R alpha = R(args.pp_exp[i].x), beta = R(args.pp_exp[i].y);
      for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
        PrimQ<R> s;
        grad_prim<R>(args, g, i, j, s);
        const R gamma_c = R(args.pp_exp[j].x);
        R x[N], wt[N];
        rys_roots<N, R>(s.t, x, wt, args.tb);
#pragma unroll
        for (int r = 0; r < N; ++r) {
          RootCoef<R> rc;
          root_coef<R>(s, x[r], rc);
          R G[3][NGR];
          build_g<LA + 1, LB + 1, LC + 1, LD, R>(rc.c00[0], rc.c0p[0], rc.b10, rc.b01, rc.b00, R(1), R(g.abx),
                                                 R(g.cdx), G[0]);
          build_g<LA + 1, LB + 1, LC + 1, LD, R>(rc.c00[1], rc.c0p[1], rc.b10, rc.b01, rc.b00, R(1), R(g.aby),
                                                 R(g.cdy), G[1]);
          build_g<LA + 1, LB + 1, LC + 1, LD, R>(rc.c00[2], rc.c0p[2], rc.b10, rc.b01, rc.b00, wt[r] * s.pref,
                                                 R(g.abz), R(g.cdz), G[2]);
          static_for<0, CI::NOUT>([&](auto O) {
            constexpr int o = decltype(O)::value;
            constexpr int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
            constexpr int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
            R v[3], fa[3], fb[3], fc[3];
            static_for<0, 3>([&](auto X) {
              constexpr int ax = decltype(X)::value;
              constexpr int a = ax == 0 ? cart_lx(LA, ia) : ax == 1 ? cart_ly(LA, ia) : cart_lz(LA, ia);
              constexpr int b = ax == 0 ? cart_lx(LB, ib) : ax == 1 ? cart_ly(LB, ib) : cart_lz(LB, ib);
              constexpr int c = ax == 0 ? cart_lx(LC, ic) : ax == 1 ? cart_ly(LC, ic) : cart_lz(LC, ic);
              constexpr int d = ax == 0 ? cart_lx(LD, id) : ax == 1 ? cart_ly(LD, id) : cart_lz(LD, id);
              v[ax] = G[ax][GI::idx(a, b, c, d)];
              fa[ax] = R(2) * alpha * G[ax][GI::idx(a + 1, b, c, d)];
              fb[ax] = R(2) * beta * G[ax][GI::idx(a, b + 1, c, d)];
              fc[ax] = R(2) * gamma_c * G[ax][GI::idx(a, b, c + 1, d)];
              if constexpr (a > 0) fa[ax] -= R(a) * G[ax][GI::idx(a - 1, b, c, d)];
              if constexpr (b > 0) fb[ax] -= R(b) * G[ax][GI::idx(a, b - 1, c, d)];
              if constexpr (c > 0) fc[ax] -= R(c) * G[ax][GI::idx(a, b, c - 1, d)];
            });
            const R gq = gam[o];
            const R yz = v[1] * v[2], xz = v[0] * v[2], xy = v[0] * v[1];
            dA[0] += gq * fa[0] * yz; dA[1] += gq * fa[1] * xz; dA[2] += gq * fa[2] * xy;
            dB[0] += gq * fb[0] * yz; dB[1] += gq * fb[1] * xz; dB[2] += gq * fb[2] * xy;
            dC[0] += gq * fc[0] * yz; dC[1] += gq * fc[1] * xz; dC[2] += gq * fc[2] * xy;
          });
        }
      }
    }
    if (active) {
      double* gC = args.grad + 3LL * args.ws_atm[g.C];
      double* gD = args.grad + 3LL * args.ws_atm[g.D];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        atomicAdd(gC + x, double(dC[x]));
        atomicAdd(gD + x, -(double(dA[x]) + double(dB[x]) + double(dC[x])));
        bA[x] += double(dA[x]);
        bB[x] += double(dB[x]);
      }
    }
  }
#pragma unroll
  for (int x = 0; x < 3; ++x)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      bA[x] += __shfl_down_sync(0xffffffffu, bA[x], off);
      bB[x] += __shfl_down_sync(0xffffffffu, bB[x], off);
    }
  if (lane == 0) {
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      atomicAdd(args.grad + 3LL * atA + x, bA[x]);
      atomicAdd(args.grad + 3LL * atB + x, bB[x]);
    }
  }
}

// Warp-per-quartet coordinate VJP for the classes between the lane kernel
// and the block kernel (up to 48 KB of tables per warp).  Per primitive
// quartet the raised 2D tables of every (root, axis) are built in shared
// memory (build_g_mem, recursion scratch in shared memory, so the kernel's
// registers stay those of the accumulation), then turned into derivative
// tables: for every unraised (a, b, c, d) tuple the four values
// (G, 2 alpha G(a+1) - a G(a-1), 2 beta G(b+1) - b G(b-1),
// 2 gamma G(c+1) - c G(c-1)) side by side, so an element's nine partials at
// one root take six 16-byte shared loads.  Lanes stride over the elements;
// Gamma is staged in shared memory once per quartet.
template <int LA, int LB, int LC, int LD>
struct GradWarp {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GC = GradCfg<LA, LB, LC, LD, 1>;
  static constexpr int N = GC::NROOT, NGR = GC::NG;
  static constexpr int NGU = CI::NG;                                     // unraised tuples
  static constexpr int NW = (LA + LB + 3) * (LC + LD + 2) * (LD + 1);   // build_g_mem scratch
  static constexpr int D_OFF = (3 * N * NGR + 3) / 4 * 4;                // 16-byte aligned in FP32 and FP64
  // the derivative tables overwrite the recursion scratch (dead by then)
  static constexpr int DW = 3 * N * NGU * 4 > 3 * N * NW ? 3 * N * NGU * 4 : 3 * N * NW;
  static constexpr int GAM_OFF = D_OFF + DW;
  static constexpr int R_OFF = GAM_OFF + CI::NOUT;
  static constexpr int ELEMS = (R_OFF + 2 * N + 3) / 4 * 4;
  static constexpr int WARPS = 4;
  static constexpr int NK = (CI::NOUT + 31) / 32;
  static constexpr size_t bytes() { return (size_t)WARPS * ELEMS * sizeof(double); }   // FP64; FP32 takes half
  // the classes where it beat the team / block kernel, measured per class
  // on (H2O)16 cc-pVTZ (one VJP, serial launches): (21|21) 1.39x, (31|30)
  // 1.61x, (33|10) 1.42x, (30|30) 1.38x, (33|00) 1.30x, (31|20) 1.25x,
  // (31|11) 1.22x, (33|20) 1.20x, (32|10) 1.18x, (22|20) 1.12x, (32|30)
  // 1.08x, (22|11) 1.05x, (30|22) 1.04x, (31|21) 1.03x, (22|21) 1.02x;
  // elsewhere it was slower (to 0.69x) and is not used
  static constexpr bool PICK = (LA == 2 && LB == 1 && LC == 2 && LD == 1) || (LA == 3 && LB == 1 && LC == 3 && LD == 0) ||
                               (LA == 3 && LB == 3 && LC == 1 && LD == 0) || (LA == 3 && LB == 0 && LC == 3 && LD == 0) ||
                               (LA == 3 && LB == 3 && LC == 0 && LD == 0) || (LA == 3 && LB == 1 && LC == 2 && LD == 0) ||
                               (LA == 3 && LB == 1 && LC == 1 && LD == 1) || (LA == 3 && LB == 3 && LC == 2 && LD == 0) ||
                               (LA == 3 && LB == 2 && LC == 1 && LD == 0) || (LA == 2 && LB == 2 && LC == 2 && LD == 0) ||
                               (LA == 3 && LB == 2 && LC == 3 && LD == 0) || (LA == 2 && LB == 2 && LC == 1 && LD == 1) ||
                               (LA == 3 && LB == 0 && LC == 2 && LD == 2) || (LA == 3 && LB == 1 && LC == 2 && LD == 1) ||
                               (LA == 2 && LB == 2 && LC == 2 && LD == 1);
  static constexpr bool OK = PICK && NGU <= 256 && ELEMS * sizeof(double) <= 48 * 1024;
};

// Four derivative-table values (G, f_A, f_B, f_C) stored side by side: one
// 16-byte access in FP32, two in FP64.
template <typename R> struct Quad;
template <> struct Quad<double> {
  static __device__ __forceinline__ void st(double* p, double a, double b, double c, double d) {
    reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
    reinterpret_cast<double2*>(p)[1] = make_double2(c, d);
  }
  static __device__ __forceinline__ void ld(const double* p, double& a, double& b, double& c, double& d) {
    const double2 x = reinterpret_cast<const double2*>(p)[0], y = reinterpret_cast<const double2*>(p)[1];
    a = x.x; b = x.y; c = y.x; d = y.y;
  }
};
template <> struct Quad<float> {
  static __device__ __forceinline__ void st(float* p, float a, float b, float c, float d) {
    *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
  }
  static __device__ __forceinline__ void ld(const float* p, float& a, float& b, float& c, float& d) {
    const float4 x = *reinterpret_cast<const float4*>(p);
    a = x.x; b = x.y; c = x.z; d = x.w;
  }
};

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) grad_warp_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GW = GradWarp<LA, LB, LC, LD>;
  using GC = GradCfg<LA, LB, LC, LD, 1>;
  constexpr int N = GW::N, NGR = GW::NGR, NGU = GW::NGU;
  extern __shared__ __align__(16) unsigned char wsm_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  R* G = reinterpret_cast<R*>(wsm_raw) + warp * GW::ELEMS;
  R* D = G + GW::D_OFF;
  R* scratch = D;
  R* gam = G + GW::GAM_OFF;
  R* roots = G + GW::R_OFF;
  // the lane's elements: unraised tuple index per axis, 8 bits each
  int tix[GW::NK];
#pragma unroll
  for (int q = 0; q < GW::NK; ++q) {
    const int o = lane + 32 * q;
    tix[q] = 0;
    if (o < CI::NOUT) {
      const int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
      const int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
      const int tx = GIdx<LA, LB, LC, LD>::idx(cart_lx(LA, ia), cart_lx(LB, ib), cart_lx(LC, ic), cart_lx(LD, id));
      const int ty = GIdx<LA, LB, LC, LD>::idx(cart_ly(LA, ia), cart_ly(LB, ib), cart_ly(LC, ic), cart_ly(LD, id));
      const int tz = GIdx<LA, LB, LC, LD>::idx(cart_lz(LA, ia), cart_lz(LB, ib), cart_lz(LC, ic), cart_lz(LD, id));
      tix[q] = tx | (ty << 8) | (tz << 16);
    }
  }
  const int4 w = args.work[blockIdx.x];
  const int bra = args.bra_pairs[w.x];
  int kb, ke;
  grad_ket_range(args, blockIdx.x, w, kb, ke);
  for (int k = kb + warp; k < ke; k += GW::WARPS) {
    QuartetGeom g;
    load_quartet(args, bra, args.ket_pairs[k], g);
    const long long base = args.mol_base[g.mol];
    const int n = args.mol_n[g.mol];
    for (int o = lane; o < CI::NOUT; o += 32) {
      const int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
      const int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
      gam[o] = R(g.scale * gamma_abcd(args, base, n, g.aoA + ia, g.aoB + ib, g.aoC + ic, g.aoD + id));
    }
    R dA[3] = {0, 0, 0}, dB[3] = {0, 0, 0}, dC[3] = {0, 0, 0};
    for (int i = g.ppa; i < g.ppa + g.npa; ++i) {
      const R alpha = R(args.pp_exp[i].x), beta = R(args.pp_exp[i].y);
      for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
        PrimQ<R> s;
        grad_prim<R>(args, g, i, j, s);
        const R gamma_c = R(args.pp_exp[j].x);
        __syncwarp();   // the previous primitive quartet's tables are no longer read
        if (lane < 2 * N) roots[lane] = rys_one<N, R>(s.t, lane, args.tb);
        __syncwarp();
        if (lane < 3 * N) {
          const int r = lane / 3, ax = lane - 3 * r;
          RootCoef<R> rc;
          root_coef<R>(s, roots[r], rc);
          const R abd = R(ax == 0 ? g.abx : (ax == 1 ? g.aby : g.abz));
          const R cdd = R(ax == 0 ? g.cdx : (ax == 1 ? g.cdy : g.cdz));
          const R g00 = ax == 2 ? roots[N + r] * s.pref : R(1);
          build_g_mem<LA + 1, LB + 1, LC + 1, LD, R>(rc.c00[ax], rc.c0p[ax], rc.b10, rc.b01, rc.b00, g00, abd, cdd,
                                                    G + lane * NGR, scratch + lane * GW::NW);
        }
        __syncwarp();
        const R e2a = R(2) * alpha, e2b = R(2) * beta, e2c = R(2) * gamma_c;
        for (int e = lane; e < 3 * N * NGU; e += 32) {
          const int tbl = e / NGU, tt = e - tbl * NGU;
          const int d = tt % (LD + 1), c = (tt / (LD + 1)) % (LC + 1);
          const int b = (tt / ((LD + 1) * (LC + 1))) % (LB + 1), a = tt / ((LD + 1) * (LC + 1) * (LB + 1));
          const R* Gt = G + tbl * NGR;
          const R v = Gt[GC::idx(a, b, c, d)];
          R fa = e2a * Gt[GC::idx(a + 1, b, c, d)];
          R fb = e2b * Gt[GC::idx(a, b + 1, c, d)];
          R fc = e2c * Gt[GC::idx(a, b, c + 1, d)];
          if (a) fa -= R(a) * Gt[GC::idx(a - 1, b, c, d)];
          if (b) fb -= R(b) * Gt[GC::idx(a, b - 1, c, d)];
          if (c) fc -= R(c) * Gt[GC::idx(a, b, c - 1, d)];
          Quad<R>::st(D + 4 * e, v, fa, fb, fc);
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < GW::NK; ++q) {
          const int o = lane + 32 * q;
          if (o >= CI::NOUT) break;
          const R gq = gam[o];
          if (gq == R(0)) continue;
          const int tx = tix[q] & 255, ty = (tix[q] >> 8) & 255, tz = tix[q] >> 16;
#pragma unroll 2
          for (int r = 0; r < N; ++r) {
            const R* Dr = D + 4 * (3 * r * NGU);
            R vx, ax, bx, cx, vy, ay, by, cy, vz, az, bz, cz;
            Quad<R>::ld(Dr + 4 * tx, vx, ax, bx, cx);
            Quad<R>::ld(Dr + 4 * (NGU + ty), vy, ay, by, cy);
            Quad<R>::ld(Dr + 4 * (2 * NGU + tz), vz, az, bz, cz);
            const R yz = gq * vy * vz, xz = gq * vx * vz, xy = gq * vx * vy;
            dA[0] += ax * yz; dA[1] += ay * xz; dA[2] += az * xy;
            dB[0] += bx * yz; dB[1] += by * xz; dB[2] += bz * xy;
            dC[0] += cx * yz; dC[1] += cy * xz; dC[2] += cz * xy;
          }
        }
      }
    }
    // warp reduction of the nine partials; lane 0 adds to the four centres
    double part[9] = {double(dA[0]), double(dA[1]), double(dA[2]), double(dB[0]), double(dB[1]),
                      double(dB[2]), double(dC[0]), double(dC[1]), double(dC[2])};
#pragma unroll
    for (int x = 0; x < 9; ++x)
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) part[x] += __shfl_down_sync(0xffffffffu, part[x], off);
    if (lane == 0) {
      double* gA = args.grad + 3LL * args.ws_atm[g.A];
      double* gB = args.grad + 3LL * args.ws_atm[g.B];
      double* gC = args.grad + 3LL * args.ws_atm[g.C];
      double* gD = args.grad + 3LL * args.ws_atm[g.D];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        atomicAdd(gA + x, part[x]);
        atomicAdd(gB + x, part[3 + x]);
        atomicAdd(gC + x, part[6 + x]);
        atomicAdd(gD + x, -(part[x] + part[3 + x] + part[6 + x]));
      }
    }
    __syncwarp();   // Gamma is rewritten by the next quartet
  }
}

// Per-lane coordinate VJP for the mid-size classes (NOUT <= 90): one lane
// per ket of a work item as the register path, Gamma of the lane's quartet
// in a private column of shared memory (conflict-free: element-major,
// lane-minor), and per root the derivative tables of one centre at a time
// in registers -- raised in a for d/dA, in b for d/dB, in c for d/dC (three
// smaller tables instead of one raised in all three, so a table set fits
// the registers).  Every index is a compile-time constant.
template <int LA, int LB, int LC, int LD>
struct GradLane {
  using CI = ClassInfo<LA, LB, LC, LD>;
  static constexpr int NGA = (LA + 2) * (LB + 1) * (LC + 1) * (LD + 1);
  static constexpr int NGB = (LA + 1) * (LB + 2) * (LC + 1) * (LD + 1);
  static constexpr int NGC = (LA + 1) * (LB + 1) * (LC + 2) * (LD + 1);
  static constexpr int NGMAX = NGA > NGB ? (NGA > NGC ? NGA : NGC) : (NGB > NGC ? NGB : NGC);
  static constexpr int THREADS = 128;
  static constexpr size_t bytes() { return (size_t)CI::NOUT * THREADS * sizeof(double); }   // FP64; FP32 half
#ifndef B200JK_GRAD_LANE_TABLES
#define B200JK_GRAD_LANE_TABLES 90   // doubles of one centre's three tables
#endif
  // measured on (H2O)16 cc-pVTZ: 1.5-2.6x over the team kernel up to 90
  // elements, slower than the register kernel on its classes and than the
  // team kernel on 108-element blocks
  static constexpr bool OK = !GradReg<LA, LB, LC, LD>::OK && CI::NOUT <= 90 && 3 * NGMAX <= B200JK_GRAD_LANE_TABLES;
};

// One shared-memory load the compiler keeps in place: each centre pass
// re-reads Gamma instead of holding NOUT values live across the passes.
__device__ __forceinline__ double lds_keep(const double* p) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"((unsigned)__cvta_generic_to_shared(p)));
  return v;
}
__device__ __forceinline__ float lds_keep(const float* p) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"((unsigned)__cvta_generic_to_shared(p)));
  return v;
}

// d/dX of one centre (X = 0: A, 1: B, 2: C) for every element of the lane's
// quartet at one root: tables raised in X's index, Gamma from the lane's
// shared-memory column, partials into d[3].
template <int LA, int LB, int LC, int LD, int X, typename R>
__device__ __forceinline__ void grad_lane_centre(const RootCoef<R>& rc, R g00, const QuartetGeom& g, R expo,
                                                 const R* __restrict__ gam, R* d) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  constexpr int RA = LA + (X == 0), RB = LB + (X == 1), RC = LC + (X == 2);
  using GI = GIdx<RA, RB, RC, LD>;
  constexpr int NGX = (RA + 1) * (RB + 1) * (RC + 1) * (LD + 1);
  R G[3][NGX];
  build_g<RA, RB, RC, LD, R>(rc.c00[0], rc.c0p[0], rc.b10, rc.b01, rc.b00, R(1), R(g.abx), R(g.cdx), G[0]);
  build_g<RA, RB, RC, LD, R>(rc.c00[1], rc.c0p[1], rc.b10, rc.b01, rc.b00, R(1), R(g.aby), R(g.cdy), G[1]);
  build_g<RA, RB, RC, LD, R>(rc.c00[2], rc.c0p[2], rc.b10, rc.b01, rc.b00, g00, R(g.abz), R(g.cdz), G[2]);
  const R e2 = R(2) * expo;
  // compile-time element indices: the tables stay in registers
  static_for_n<CI::NOUT>([&](auto O) {
    constexpr int o = decltype(O)::value;
    constexpr int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
    constexpr int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
    R v[3], f[3];
    static_for_n<3>([&](auto AX) {
      constexpr int ax = decltype(AX)::value;
      constexpr int a = ax == 0 ? cart_lx(LA, ia) : ax == 1 ? cart_ly(LA, ia) : cart_lz(LA, ia);
      constexpr int b = ax == 0 ? cart_lx(LB, ib) : ax == 1 ? cart_ly(LB, ib) : cart_lz(LB, ib);
      constexpr int c = ax == 0 ? cart_lx(LC, ic) : ax == 1 ? cart_ly(LC, ic) : cart_lz(LC, ic);
      constexpr int dd = ax == 0 ? cart_lx(LD, id) : ax == 1 ? cart_ly(LD, id) : cart_lz(LD, id);
      constexpr int n = X == 0 ? a : X == 1 ? b : c;   // the raised index
      v[ax] = G[ax][GI::idx(a, b, c, dd)];
      f[ax] = e2 * G[ax][GI::idx(a + (X == 0), b + (X == 1), c + (X == 2), dd)];
      if constexpr (n > 0) f[ax] -= R(n) * G[ax][GI::idx(a - (X == 0), b - (X == 1), c - (X == 2), dd)];
    });
    const R gq = lds_keep(gam + o * GradLane<LA, LB, LC, LD>::THREADS);
    d[0] += gq * f[0] * (v[1] * v[2]);
    d[1] += gq * f[1] * (v[0] * v[2]);
    d[2] += gq * f[2] * (v[0] * v[1]);
  });
}

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) grad_lane_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GC = GradCfg<LA, LB, LC, LD, 1>;
  using GL = GradLane<LA, LB, LC, LD>;
  constexpr int N = GC::NROOT;
  extern __shared__ __align__(16) unsigned char s_gam_raw[];   // [NOUT][THREADS]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x * (GL::THREADS / 32) + warp;
  if (item >= args.nwork) return;
  R* gam = reinterpret_cast<R*>(s_gam_raw) + threadIdx.x;
  const int4 w = args.work[item];
  const int bra = args.bra_pairs[w.x];
  double bA[3] = {0, 0, 0}, bB[3] = {0, 0, 0};
  int atA = 0, atB = 0;
  int kb, ke;
  grad_ket_range(args, item, w, kb, ke);
  for (int k0 = kb; k0 < ke; k0 += 32) {
    const bool active = k0 + lane < ke;
    const int k = active ? k0 + lane : ke - 1;
    QuartetGeom g;
    load_quartet(args, bra, args.ket_pairs[k], g);
    atA = args.ws_atm[g.A];
    atB = args.ws_atm[g.B];
    const long long base = args.mol_base[g.mol];
    const int n = args.mol_n[g.mol];
    for (int o = 0; o < CI::NOUT; ++o) {
      const int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
      const int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
      gam[o * GL::THREADS] =
          active ? R(g.scale * gamma_abcd(args, base, n, g.aoA + ia, g.aoB + ib, g.aoC + ic, g.aoD + id)) : R(0);
    }
    R dA[3] = {0, 0, 0}, dB[3] = {0, 0, 0}, dC[3] = {0, 0, 0};
    for (int i = g.ppa; i < g.ppa + g.npa; ++i) {
      const R alpha = R(args.pp_exp[i].x), beta = R(args.pp_exp[i].y);
      for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
        PrimQ<R> s;
        grad_prim<R>(args, g, i, j, s);
        const R gamma_c = R(args.pp_exp[j].x);
        R x[N], wt[N];
        rys_roots<N, R>(s.t, x, wt, args.tb);
        // one (root, centre) pass per iteration, not unrolled: one centre's
        // tables are live at a time
#pragma unroll 1
        for (int tsk = 0; tsk < 3 * N; ++tsk) {
          const int r = tsk / 3, cx = tsk - 3 * r;
          RootCoef<R> rc;
          root_coef<R>(s, x[r], rc);
          const R g00 = wt[r] * s.pref;
          if (cx == 0) grad_lane_centre<LA, LB, LC, LD, 0, R>(rc, g00, g, alpha, gam, dA);
          else if (cx == 1) grad_lane_centre<LA, LB, LC, LD, 1, R>(rc, g00, g, beta, gam, dB);
          else grad_lane_centre<LA, LB, LC, LD, 2, R>(rc, g00, g, gamma_c, gam, dC);
        }
      }
    }
    if (active) {
      double* gC = args.grad + 3LL * args.ws_atm[g.C];
      double* gD = args.grad + 3LL * args.ws_atm[g.D];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        atomicAdd(gC + x, double(dC[x]));
        atomicAdd(gD + x, -(double(dA[x]) + double(dB[x]) + double(dC[x])));
        bA[x] += double(dA[x]);
        bB[x] += double(dB[x]);
      }
    }
  }
#pragma unroll
  for (int x = 0; x < 3; ++x)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      bA[x] += __shfl_down_sync(0xffffffffu, bA[x], off);
      bB[x] += __shfl_down_sync(0xffffffffu, bB[x], off);
    }
  if (lane == 0) {
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      atomicAdd(args.grad + 3LL * atA + x, bA[x]);
      atomicAdd(args.grad + 3LL * atB + x, bB[x]);
    }
  }
}

}  // namespace b200jk
