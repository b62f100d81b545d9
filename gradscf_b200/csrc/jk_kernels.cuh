// Direct J/K shell-quartet kernels, one template instantiation per
// angular-momentum class (LA>=LB | LC>=LD), FP64 or FP32 arithmetic.
//
// Work decomposition: the significant shell pairs of one pair class are
// sorted by Schwarz bound (descending) -- the "bra list"; for a class pair
// (X,Y) every bra pair p of X meets the leading kets of Y whose bound passes
// Q_p Q_q >= cut (and q <= p when X == Y).  A work item is (bra position,
// ket range); one CUDA block takes one item.
//
// Digestion (all in the raw Cartesian basis, densities pre-transformed):
// with s = (A==B ? 1/2:1)(C==D ? 1/2:1)(pq ? 1/2:1) the unique quartet adds
//   MJ[a][b] += 2s sum_cd V D_cd,   MJ[c][d] += 2s sum_ab V D_ab,
//   MK[a][c] += s sum_bd V D_bd,    MK[a][d] += s sum_bc V D_bc,
//   MK[b][c] += s sum_ad V D_ad,    MK[b][d] += s sum_ac V D_ac,
// and the caller finalises J = MJ + MJ^T, K = MK +/- MK^T (symmetric /
// antisymmetric density part).  That is the reference's eight-permutation
// scatter (csrc/direct_jk.cc:50-75) folded by the symmetry of D.
#pragma once
#include "common.cuh"

namespace b200jk {

struct JKArgs {
  const int4* sh_info;       // (cart offset in molecule, l, molecule, unused)
  const double4* sh_xyz;     // centre
  const int4* pair_info;     // (shell A, shell B, first primitive pair, count)
  const double4* pp_data;    // primitive pair: (Px, Py, Pz, p = a+b)
  const double2* pp_aux;     // (exp(-ab/p |AB|^2) c_a c_b / p, 1/(2p))
  const float4* pp_f;        // FP32 copy: (P - A, p)
  const float2* pp_f2;       // FP32 copy: (K/p, 1/(2p))
  const long long* mol_base; // offset of the molecule's n x n block
  const int* mol_n;          // Cartesian AO count of the molecule
  const int* bra_pairs;      // sorted pair ids of the bra class
  const int* ket_pairs;      // sorted pair ids of the ket class
  // per list position: (Ax, Ay, Az, molecule), A - B, (first primitive
  // pair, count, Cartesian offset of A, of B); same_list: bra list == ket list
  const double4 *bra_ra, *bra_ab, *ket_ra, *ket_ab;
  const int4 *bra_ix, *ket_ix;
  // grouped lists: (diag, 0, aoA1, aoB1), (aoA2, aoB2, aoA3, aoB3) per position
  const int4 *bra_gx, *bra_gy, *ket_gx, *ket_gy;
  const double4* pp_c;       // per primitive pair: coefficients of up to 4 combinations
  const float4* pp_cf;       // the same in FP32
  int same_list;
  double omega2;             // long-range erf(omega r)/r operator: omega^2 (0: full Coulomb)
  const int4* work;          // (bra position, ket begin, ket end, unused)
  int nwork;
  const int* split;          // per work item: first ket computed in FP32
  int split_mode;            // 0 all kets, 1 kets below split, 2 kets from split
  const double* dens;        // [ndm][dstride] Cartesian effective densities
  const float* dens_f;       // the same in FP32 (used by FP32 quartets)
  double* vj;                // [nsym][dstride]
  double* vk;                // [ndm][dstride]
  long long dstride;
  int ndm, nsym, with_j, with_k;
  Tables tb;
  double* q_out;             // Schwarz mode: per pair max |(ab|ab)| in output basis
  int* status;               // device error word (0 = ok)
  // coordinate VJP
  const double2* pp_exp;     // primitive pair: (exponent on A, exponent on B)
  const double* cot_j;       // raw Cartesian J cotangents [gnb][dstride] (or null)
  const double* cot_k;       // raw Cartesian K cotangents (or null)
  int gnb;                   // density / cotangent batches
  // bra-group register path: bra order -> list position, Schwarz bounds per
  // list position, per-item density bound, Schwarz and FP32 cuts
  const int* bra_bord;
  const double* bra_q;
  const double* ket_q;
  const double* item_m;
  double cutoff, fp32_cut;
  int* queue;                // persistent kernels: the launch's item counter (zeroed before it)
  // split builds: FP64 quartets listed one per lane (bra position, ket
  // position), the list length, its capacity, and per bra-group item a flag
  // set when its FP64 quartets are in the list (the bra-group launch skips it)
  const int2* flat;
  const unsigned long long* flat_n;
  int flat_cap;
  const int* item_skip;
  const int* ws_atm;         // atm row of each work shell's centre
  double* grad;              // (atm rows, 3)
  // coordinate JVP / Hessian-vector products: directions, (atm rows, 3)
  const double* geo_u;
  const double* geo_v;
};

template <typename R> struct DensSel;
template <> struct DensSel<double> {
  static __device__ __forceinline__ const double* get(const JKArgs& a) { return a.dens; }
};
template <> struct DensSel<float> {
  static __device__ __forceinline__ const float* get(const JKArgs& a) { return a.dens_f; }
};

template <int LA, int LB, int LC, int LD>
struct GIdx {
  __host__ __device__ static constexpr int idx(int a, int b, int c, int d) {
    return ((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d;
  }
};

// Ket range of a work item for the requested precision slice.
__device__ __forceinline__ void ket_range(const JKArgs& args, const int4 w, int& kb, int& ke) {
  kb = w.y;
  ke = w.z;
  if (args.split_mode != 0) {
    const int s = args.split[blockIdx.x];
    if (args.split_mode == 1) ke = min(ke, s);
    else kb = max(kb, s);
  }
}

// Quartet-level geometry shared by both paths.
struct QuartetGeom {
  int A, B, C, D;
  int ppa, npa, ppc, npc;
  double ax, ay, az, cx, cy, cz;
  double abx, aby, abz, cdx, cdy, cdz;
  int aoA, aoB, aoC, aoD, mol;
  double scale;
  double omega2;   // erf-attenuated operator: omega^2 (0: full Coulomb)
};

__device__ __forceinline__ void load_quartet(const JKArgs& args, int bra, int ket, QuartetGeom& g) {
  const int4 pb = args.pair_info[bra];
  const int4 pk = args.pair_info[ket];
  g.A = pb.x; g.B = pb.y; g.ppa = pb.z; g.npa = pb.w;
  g.C = pk.x; g.D = pk.y; g.ppc = pk.z; g.npc = pk.w;
  const double4 ra = args.sh_xyz[g.A], rb = args.sh_xyz[g.B];
  const double4 rc = args.sh_xyz[g.C], rd = args.sh_xyz[g.D];
  g.ax = ra.x; g.ay = ra.y; g.az = ra.z;
  g.cx = rc.x; g.cy = rc.y; g.cz = rc.z;
  g.abx = ra.x - rb.x; g.aby = ra.y - rb.y; g.abz = ra.z - rb.z;
  g.cdx = rc.x - rd.x; g.cdy = rc.y - rd.y; g.cdz = rc.z - rd.z;
  const int4 ia = args.sh_info[g.A], ib = args.sh_info[g.B];
  const int4 ic = args.sh_info[g.C], id = args.sh_info[g.D];
  g.aoA = ia.x; g.aoB = ib.x; g.aoC = ic.x; g.aoD = id.x; g.mol = ia.z;
  double s = 1.0;
  if (g.A == g.B) s *= 0.5;
  if (g.C == g.D) s *= 0.5;
  if (bra == ket) s *= 0.5;
  g.scale = s;
  g.omega2 = args.omega2;
}

// Bra side of a work item from the per-position records (loaded once per warp).
struct BraRec {
  double4 ra, ab;
  int4 ix;
  int pos;
};

__device__ __forceinline__ BraRec load_bra(const JKArgs& args, int pos) {
  return BraRec{args.bra_ra[pos], args.bra_ab[pos], args.bra_ix[pos], pos};
}

// Quartet from the bra record and the ket at list position kpos: three
// coalesced loads per lane, no dependent table lookups.  The shell ids
// A..D are not filled (the J/K paths address by Cartesian offset).
__device__ __forceinline__ void load_quartet_rec(const JKArgs& args, const BraRec& b, int kpos,
                                                 QuartetGeom& g) {
  const double4 rc = args.ket_ra[kpos], cd = args.ket_ab[kpos];
  const int4 kx = args.ket_ix[kpos];
  g.A = g.B = g.C = g.D = -1;
  g.ppa = b.ix.x; g.npa = b.ix.y; g.ppc = kx.x; g.npc = kx.y;
  g.ax = b.ra.x; g.ay = b.ra.y; g.az = b.ra.z;
  g.cx = rc.x; g.cy = rc.y; g.cz = rc.z;
  g.abx = b.ab.x; g.aby = b.ab.y; g.abz = b.ab.z;
  g.cdx = cd.x; g.cdy = cd.y; g.cdz = cd.z;
  g.aoA = b.ix.z; g.aoB = b.ix.w; g.aoC = kx.z; g.aoD = kx.w;
  g.mol = (int)b.ra.w;
  double s = 1.0;
  if (b.ix.z == b.ix.w) s *= 0.5;
  if (kx.z == kx.w) s *= 0.5;
  if (args.same_list && kpos == b.pos) s *= 0.5;
  g.scale = s;
  g.omega2 = args.omega2;
}

// Per primitive quartet scalars.
template <typename R>
struct PrimQ {
  R pq_inv, q_pq, p_pq;      // 1/(p+q), q/(p+q), p/(p+q)
  R inv2p, inv2q;            // 1/(2p), 1/(2q)
  R pax, pay, paz, qcx, qcy, qcz, pqx, pqy, pqz;
  R t, pref;
  R theta;                   // omega^2 / (omega^2 + rho) for erf(omega r)/r, else 1
};

// erf(omega r)/r (libcint's PTR_RANGE_OMEGA > 0): with theta = omega^2 /
// (omega^2 + pq/(p+q)) the Boys functions become theta^(m+1/2) F_m(theta T),
// i.e. Rys roots at theta T, nodes t^2 scaled by theta (root_coef) and
// weights by sqrt(theta) (folded into pref).
template <typename R>
__device__ __forceinline__ void apply_range(double omega2, R p, R q, R ipq, PrimQ<R>& s) {
  s.theta = R(1);
  if (omega2 > 0.0) {
    const R w2 = R(omega2);
    const R th = w2 / (w2 + p * q * ipq);
    s.t *= th;
    s.pref *= dsqrt<R>(th);
    s.theta = th;
  }
}

// Division-free: pref = 2 pi^2.5 (K_ab/p)(K_cd/q) / sqrt(p+q) with the
// per-pair factors precomputed; 1/(p+q) = rsqrt(p+q)^2.
template <typename R>
__device__ __forceinline__ void prim_setup(const QuartetGeom& g, const double4 P, const double2 PA,
                                           const double4 Q, const double2 QA, PrimQ<R>& s) {
  if constexpr (sizeof(R) == 4) {
    // FP32 quartets: centre differences in FP64, the rest in FP32.
    const float p = float(P.w), q = float(Q.w);
    const float pq = p + q;
    const float rs = rsqrtf(pq);
    const float ipq = rs * rs;
    const float pqx = float(P.x - Q.x), pqy = float(P.y - Q.y), pqz = float(P.z - Q.z);
    s.t = p * q * ipq * (pqx * pqx + pqy * pqy + pqz * pqz);
    s.pref = float(B200JK_ERI_C0) * float(PA.x) * float(QA.x) * rs;
    s.pq_inv = ipq;
    s.q_pq = q * ipq;
    s.p_pq = p * ipq;
    s.inv2p = float(PA.y);
    s.inv2q = float(QA.y);
    s.pax = float(P.x - g.ax); s.pay = float(P.y - g.ay); s.paz = float(P.z - g.az);
    s.qcx = float(Q.x - g.cx); s.qcy = float(Q.y - g.cy); s.qcz = float(Q.z - g.cz);
    s.pqx = pqx; s.pqy = pqy; s.pqz = pqz;
    apply_range<R>(g.omega2, R(p), R(q), R(ipq), s);
    return;
  }
  const double p = P.w, q = Q.w;
  const double pq = p + q;
  const double rs = rsqrt(pq);
  const double ipq = rs * rs;
  const double pqx = P.x - Q.x, pqy = P.y - Q.y, pqz = P.z - Q.z;
  const double t = p * q * ipq * (pqx * pqx + pqy * pqy + pqz * pqz);
  s.t = R(t);
  s.pref = R(B200JK_ERI_C0 * PA.x * QA.x * rs);
  s.pq_inv = R(ipq);
  s.q_pq = R(q * ipq);
  s.p_pq = R(p * ipq);
  s.inv2p = R(PA.y);
  s.inv2q = R(QA.y);
  s.pax = R(P.x - g.ax); s.pay = R(P.y - g.ay); s.paz = R(P.z - g.az);
  s.qcx = R(Q.x - g.cx); s.qcy = R(Q.y - g.cy); s.qcz = R(Q.z - g.cz);
  s.pqx = R(pqx); s.pqy = R(pqy); s.pqz = R(pqz);
  apply_range<R>(g.omega2, R(p), R(q), R(ipq), s);
}

// FP32 quartets: per-primitive data stored relative to the shell centre in
// FP32, P - Q = (A - C) + (P - A) - (Q - C) with A - C formed once per quartet.
__device__ __forceinline__ void prim_setup_f(const float3 ac, const float4 P, const float2 PA,
                                             const float4 Q, const float2 QA, PrimQ<float>& s,
                                             double omega2) {
  const float p = P.w, q = Q.w;
  const float pq = p + q;
  const float rs = rsqrtf(pq);
  const float ipq = rs * rs;
  const float pqx = ac.x + P.x - Q.x, pqy = ac.y + P.y - Q.y, pqz = ac.z + P.z - Q.z;
  s.t = p * q * ipq * (pqx * pqx + pqy * pqy + pqz * pqz);
  s.pref = float(B200JK_ERI_C0) * PA.x * QA.x * rs;
  s.pq_inv = ipq;
  s.q_pq = q * ipq;
  s.p_pq = p * ipq;
  s.inv2p = PA.y;
  s.inv2q = QA.y;
  s.pax = P.x; s.pay = P.y; s.paz = P.z;
  s.qcx = Q.x; s.qcy = Q.y; s.qcz = Q.z;
  s.pqx = pqx; s.pqy = pqy; s.pqz = pqz;
  apply_range<float>(omega2, p, q, ipq, s);
}

// Primitive-pair storage type per precision (bra cache and ket reads).
template <typename R> struct PrimData;
template <> struct PrimData<double> {
  using A = double4;
  using B = double2;
  static __device__ __forceinline__ A a(const JKArgs& x, int i) { return x.pp_data[i]; }
  static __device__ __forceinline__ B b(const JKArgs& x, int i) { return x.pp_aux[i]; }
};
template <> struct PrimData<float> {
  using A = float4;
  using B = float2;
  static __device__ __forceinline__ A a(const JKArgs& x, int i) { return x.pp_f[i]; }
  static __device__ __forceinline__ B b(const JKArgs& x, int i) { return x.pp_f2[i]; }
};

template <typename R>
__device__ __forceinline__ void prim_any(const QuartetGeom& g, const float3 ac,
                                         const typename PrimData<R>::A P, const typename PrimData<R>::B PA,
                                         const typename PrimData<R>::A Q, const typename PrimData<R>::B QA,
                                         PrimQ<R>& s) {
  if constexpr (sizeof(R) == 4) prim_setup_f(ac, P, PA, Q, QA, s, g.omega2);
  else prim_setup<double>(g, P, PA, Q, QA, s);
}

// Rys coefficients of one root for the three axes.
template <typename R>
struct RootCoef {
  R b00, b10, b01;
  R c00[3], c0p[3];
};

template <typename R>
__device__ __forceinline__ void root_coef(const PrimQ<R>& s, R u0, RootCoef<R>& rc) {
  const R u = u0 * s.theta;  // node t^2 (scaled for the erf-attenuated operator)
  const R up = u * s.pq_inv;
  rc.b00 = R(0.5) * up;
  rc.b10 = s.inv2p - s.inv2p * u * s.q_pq;
  rc.b01 = s.inv2q - s.inv2q * u * s.p_pq;
  const R uq = u * s.q_pq, upp = u * s.p_pq;
  rc.c00[0] = s.pax - uq * s.pqx;
  rc.c00[1] = s.pay - uq * s.pqy;
  rc.c00[2] = s.paz - uq * s.pqz;
  rc.c0p[0] = s.qcx + upp * s.pqx;
  rc.c0p[1] = s.qcy + upp * s.pqy;
  rc.c0p[2] = s.qcz + upp * s.pqz;
}

__device__ __forceinline__ long long dm_index(const JKArgs& args, int mol, int a, int b) {
  return args.mol_base[mol] + (long long)a * args.mol_n[mol] + b;
}

// ---------------------------------------------------------------------------
// Register path: one thread per quartet, the whole Cartesian block in registers.
// ---------------------------------------------------------------------------
#ifndef B200JK_REG_UNROLL
#define B200JK_REG_UNROLL 2
#endif
constexpr int kRegUnroll = B200JK_REG_UNROLL;   // bra primitives interleaved per step (ILP)
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void quartet_block_reg(const JKArgs& args, const QuartetGeom& g,
                                                  const typename PrimData<R>::A* bpp,
                                                  const typename PrimData<R>::B* baux, R* out,
                                                  const float* s_boys) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GI = GIdx<LA, LB, LC, LD>;
  constexpr int N = CI::NROOT;
#pragma unroll
  for (int o = 0; o < CI::NOUT; ++o) out[o] = R(0);
  // ket primitive in registers (outer), bra primitives broadcast from
  // shared memory (inner): one global read per ket primitive pair.
  const float3 ac = make_float3(float(g.ax - g.cx), float(g.ay - g.cy), float(g.az - g.cz));
  // the next ket primitive is fetched while the current one is in use
  auto Qn = PrimData<R>::a(args, g.ppc);
  auto QAn = PrimData<R>::b(args, g.ppc);
  for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
    const auto Q = Qn;
    const auto QA = QAn;
    if (j + 1 < g.ppc + g.npc) {
      Qn = PrimData<R>::a(args, j + 1);
      QAn = PrimData<R>::b(args, j + 1);
    }
#pragma unroll(kRegUnroll)
    for (int i = 0; i < g.npa; ++i) {
      PrimQ<R> s;
      prim_any<R>(g, ac, bpp[i], baux[i], Q, QA, s);
      R x[N], w[N];
      if constexpr (sizeof(R) == 4 && N <= 3)
        rys_small<N, float, 10, 6>(s.t, x, w, s_boys);   // shared-memory Taylor rows
      else
        rys_roots<N, R>(s.t, x, w, args.tb);
#pragma unroll
      for (int r = 0; r < N; ++r) {
        RootCoef<R> rc;
        root_coef<R>(s, x[r], rc);
        R gx[CI::NG], gy[CI::NG], gz[CI::NG];
        build_g<LA, LB, LC, LD, R>(rc.c00[0], rc.c0p[0], rc.b10, rc.b01, rc.b00, R(1), R(g.abx),
                                   R(g.cdx), gx);
        build_g<LA, LB, LC, LD, R>(rc.c00[1], rc.c0p[1], rc.b10, rc.b01, rc.b00, R(1), R(g.aby),
                                   R(g.cdy), gy);
        build_g<LA, LB, LC, LD, R>(rc.c00[2], rc.c0p[2], rc.b10, rc.b01, rc.b00, w[r] * s.pref,
                                   R(g.abz), R(g.cdz), gz);
        static_for<0, CI::NOUT>([&](auto O) {
          constexpr int o = decltype(O)::value;
          constexpr int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
          constexpr int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
          constexpr int jx = GI::idx(cart_lx(LA, ia), cart_lx(LB, ib), cart_lx(LC, ic), cart_lx(LD, id));
          constexpr int jy = GI::idx(cart_ly(LA, ia), cart_ly(LB, ib), cart_ly(LC, ic), cart_ly(LD, id));
          constexpr int jz = GI::idx(cart_lz(LA, ia), cart_lz(LB, ib), cart_lz(LC, ic), cart_lz(LD, id));
          out[o] += gx[jx] * gy[jy] * gz[jz];
        });
      }
    }
  }
}

// Density elements one quartet digests, in a fixed order: D[c][d] (J of the
// bra), D[a][b] (J of the ket), then D[b][d], D[b][c], D[a][d], D[a][c] (the
// four exchange terms).  Small classes fetch them into registers before the
// primitive loop so the loads overlap the integral evaluation.
template <int LA, int LB, int LC, int LD>
struct DigestMap {
  using CI = ClassInfo<LA, LB, LC, LD>;
  static constexpr int NA = CI::NA, NB = CI::NB, NC = CI::NC, ND = CI::ND;
  static constexpr int OJ1 = 0, OJ2 = NC * ND, OK1 = OJ2 + NA * NB, OK2 = OK1 + NB * ND,
                       OK3 = OK2 + NB * NC, OK4 = OK3 + NA * ND, TOTAL = OK4 + NA * NC;
};

#ifndef B200JK_PRELOAD_MAX
#define B200JK_PRELOAD_MAX 0   // measured on (H2O)32 cc-pVDZ: no gain from preloading
#endif

template <int LA, int LB, int LC, int LD, typename R>
struct DensPre {
  using M = DigestMap<LA, LB, LC, LD>;
  static constexpr bool ON = M::TOTAL <= B200JK_PRELOAD_MAX;
  R v[ON ? M::TOTAL : 1];
  __device__ __forceinline__ void load(const JKArgs& args, const QuartetGeom& g) {
    if constexpr (ON) {
      const R* dm = DensSel<R>::get(args) + args.mol_base[g.mol];
      const int n = args.mol_n[g.mol];
      auto at = [&](int r, int c) { return __ldg(dm + (long long)r * n + c); };
#pragma unroll
      for (int c = 0; c < M::NC; ++c)
#pragma unroll
        for (int d = 0; d < M::ND; ++d) v[M::OJ1 + c * M::ND + d] = at(g.aoC + c, g.aoD + d);
#pragma unroll
      for (int a = 0; a < M::NA; ++a)
#pragma unroll
        for (int b = 0; b < M::NB; ++b) v[M::OJ2 + a * M::NB + b] = at(g.aoA + a, g.aoB + b);
#pragma unroll
      for (int b = 0; b < M::NB; ++b) {
#pragma unroll
        for (int d = 0; d < M::ND; ++d) v[M::OK1 + b * M::ND + d] = at(g.aoB + b, g.aoD + d);
#pragma unroll
        for (int c = 0; c < M::NC; ++c) v[M::OK2 + b * M::NC + c] = at(g.aoB + b, g.aoC + c);
      }
#pragma unroll
      for (int a = 0; a < M::NA; ++a) {
#pragma unroll
        for (int d = 0; d < M::ND; ++d) v[M::OK3 + a * M::ND + d] = at(g.aoA + a, g.aoD + d);
#pragma unroll
        for (int c = 0; c < M::NC; ++c) v[M::OK4 + a * M::NC + c] = at(g.aoA + a, g.aoC + c);
      }
    }
  }
};

// J[a][b] of the block's bra pair for density 0 goes to `jab` (reduced by
// the caller) when acc_j is set; everything else is an atomic add.  Density
// elements come from `pre` (density 0 of small classes) or are read where
// they are used (L1/L2 resident).
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void digest_reg(const JKArgs& args, const QuartetGeom& g, const R* out,
                                           bool acc_j, bool active, double* s_jab_row,
                                           const DensPre<LA, LB, LC, LD, R>& pre) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using M = DigestMap<LA, LB, LC, LD>;
  constexpr bool PRE = DensPre<LA, LB, LC, LD, R>::ON;
  constexpr int NA = CI::NA, NB = CI::NB, NC = CI::NC, ND = CI::ND;
  const double s = g.scale;
  const long long base = args.mol_base[g.mol];
  const int n = args.mol_n[g.mol];
  // per-quartet contractions in R (FP32 quartets: FP32 accumulation per
  // quartet); the J/K matrices themselves are accumulated in FP64.
  const R* dens = DensSel<R>::get(args);
#define V_(a, b, c, d) (out[(((a) * NB + (b)) * NC + (c)) * ND + (d)])
  for (int e = 0; e < args.ndm; ++e) {
    const R* dm = dens + e * args.dstride + base;
    const bool use_pre = PRE && e == 0;
    auto dv = [&](int slot, int r, int c) -> R {
      if constexpr (PRE) {
        if (use_pre) return pre.v[slot];
      }
      return __ldg(dm + (long long)r * n + c);
    };
    if (args.with_j && e < args.nsym) {
      double* vj = args.vj + e * args.dstride + base;
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          R acc = R(0);
#pragma unroll
          for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int d = 0; d < ND; ++d) acc += V_(a, b, c, d) * dv(M::OJ1 + c * ND + d, g.aoC + c, g.aoD + d);
          if (acc_j && e == 0) {
            // bra-block J of density 0: warp-reduced here, added once per work item
            double v = active ? 2.0 * s * double(acc) : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if ((threadIdx.x & 31) == 0) s_jab_row[a * NB + b] += v;
          } else if (active) {
            atomicAdd(vj + (long long)(g.aoA + a) * n + g.aoB + b, 2.0 * s * double(acc));
          }
        }
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          R acc = R(0);
#pragma unroll
          for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int b = 0; b < NB; ++b) acc += V_(a, b, c, d) * dv(M::OJ2 + a * NB + b, g.aoA + a, g.aoB + b);
          if (active) atomicAdd(vj + (long long)(g.aoC + c) * n + g.aoD + d, 2.0 * s * double(acc));
        }
    }
    if (args.with_k) {
      double* vk = args.vk + e * args.dstride + base;
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          R acc = R(0);
#pragma unroll
          for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int d = 0; d < ND; ++d) acc += V_(a, b, c, d) * dv(M::OK1 + b * ND + d, g.aoB + b, g.aoD + d);
          if (active) atomicAdd(vk + (long long)(g.aoA + a) * n + g.aoC + c, s * double(acc));
        }
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          R acc = R(0);
#pragma unroll
          for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int c = 0; c < NC; ++c) acc += V_(a, b, c, d) * dv(M::OK2 + b * NC + c, g.aoB + b, g.aoC + c);
          if (active) atomicAdd(vk + (long long)(g.aoA + a) * n + g.aoD + d, s * double(acc));
        }
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          R acc = R(0);
#pragma unroll
          for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int d = 0; d < ND; ++d) acc += V_(a, b, c, d) * dv(M::OK3 + a * ND + d, g.aoA + a, g.aoD + d);
          if (active) atomicAdd(vk + (long long)(g.aoB + b) * n + g.aoC + c, s * double(acc));
        }
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          R acc = R(0);
#pragma unroll
          for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int c = 0; c < NC; ++c) acc += V_(a, b, c, d) * dv(M::OK4 + a * NC + c, g.aoA + a, g.aoC + c);
          if (active) atomicAdd(vk + (long long)(g.aoB + b) * n + g.aoD + d, s * double(acc));
        }
    }
  }
#undef V_
}

// Occupancy target of the register path from its estimated register need.
template <int LA, int LB, int LC, int LD, typename R, int NACC = ClassInfo<LA, LB, LC, LD>::NOUT>
struct RegMinBlocks {
  using CI = ClassInfo<LA, LB, LC, LD>;
  // estimated live registers: accumulators + one root's 2D integrals + ~70 for
  // addresses, primitive scalars and digestion (FP64 values take two)
  static constexpr int EST = (sizeof(R) == 8 ? 2 : 1) * (NACC + 3 * CI::NG) + 70;
  static constexpr int base = EST <= 84 ? 6 : (EST <= 100 ? 5 : (EST <= 124 ? 4 : (EST <= 160 ? 3 : 2)));
#ifndef B200JK_MINB_DELTA
#define B200JK_MINB_DELTA 0
#endif
  static constexpr int value = base + B200JK_MINB_DELTA < 1 ? 1 : base + B200JK_MINB_DELTA;
};

constexpr int kBraPrimCache = 64;
constexpr int kRegWarps = 4;   // warps per block; each warp owns one work item

// Register path, warp-granular: warp w of block b takes work item 4b+w,
// caches its bra primitive pairs in a per-warp shared slot, processes its
// kets 32 at a time, and reduces the bra-block J of density 0 with shuffles.
// No block-wide barrier.
template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128, (RegMinBlocks<LA, LB, LC, LD, R>::value))
    jk_reg_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using PA_t = typename PrimData<R>::A;
  using PB_t = typename PrimData<R>::B;
  __shared__ PA_t s_pp[kRegWarps][kBraPrimCache];
  __shared__ PB_t s_aux[kRegWarps][kBraPrimCache];
  __shared__ double s_jab[kRegWarps][CI::NAB];
  // FP32 path with closed-form roots: this order's Taylor table (12.8 KB)
  constexpr bool kSharedBoys = sizeof(R) == 4 && CI::NROOT <= 3;
  __shared__ __align__(16) float s_boys[kSharedBoys ? 401 * 8 : 4];
  if constexpr (kSharedBoys) {
    const float4* src = reinterpret_cast<const float4*>(args.tb.boys_s_f + (CI::NROOT - 1) * 401 * 8);
    float4* dst = reinterpret_cast<float4*>(s_boys);
    for (int i = threadIdx.x; i < 401 * 2; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x * kRegWarps + warp;
  if (item >= args.nwork) return;
  const int4 w = args.work[item];
  int kb = w.y, ke = w.z;
  if (args.split_mode != 0) {
    const int sp = args.split[item];
    if (args.split_mode == 1) ke = min(ke, sp);
    else kb = max(kb, sp);
  }
  if (kb >= ke) return;
  const BraRec br = load_bra(args, w.x);
  const int ppb = br.ix.x, npb = br.ix.y;
  const bool cached = npb <= kBraPrimCache;
  if (cached)
    for (int i = lane; i < npb; i += 32) {
      s_pp[warp][i] = PrimData<R>::a(args, ppb + i);
      s_aux[warp][i] = PrimData<R>::b(args, ppb + i);
    }
  const bool acc_j = args.with_j && args.nsym == 1;
  for (int i = lane; i < CI::NAB; i += 32) s_jab[warp][i] = 0.0;
  __syncwarp();
  const PA_t* bpp = cached ? s_pp[warp] : (sizeof(R) == 4 ? (const PA_t*)(args.pp_f + ppb)
                                                         : (const PA_t*)(args.pp_data + ppb));
  const PB_t* baux = cached ? s_aux[warp] : (sizeof(R) == 4 ? (const PB_t*)(args.pp_f2 + ppb)
                                                           : (const PB_t*)(args.pp_aux + ppb));
  QuartetGeom g;
  for (int k0 = kb; k0 < ke; k0 += 32) {
    // lanes past the range recompute the last ket with their output masked,
    // so the whole warp takes part in the J shuffles
    const bool active = k0 + lane < ke;
    const int k = active ? k0 + lane : ke - 1;
    load_quartet_rec(args, br, k, g);
    DensPre<LA, LB, LC, LD, R> pre;
    pre.load(args, g);
    R out[CI::NOUT];
    quartet_block_reg<LA, LB, LC, LD, R>(args, g, bpp, baux, out, s_boys);
    digest_reg<LA, LB, LC, LD, R>(args, g, out, acc_j, active, s_jab[warp], pre);
  }
  if (acc_j) {
    __syncwarp();
    const int mol = (int)br.ra.w;
    double* vj = args.vj + args.mol_base[mol];
    const int n = args.mol_n[mol];
    for (int ab = lane; ab < CI::NAB; ab += 32) {
      const double v = s_jab[warp][ab];
      if (v != 0.0) atomicAdd(vj + (long long)(br.ix.z + ab / CI::NB) * n + br.ix.w + ab % CI::NB, v);
    }
  }
}

// ---------------------------------------------------------------------------
// Register path over bra groups.  A work item is (bras [g0, g0 + gn) of the
// bra order, which share molecule, primitive-pair count and shell A; kets
// [kb, ke) of one ket run).  Lane = ket; for each 32-ket pass the warp walks
// the group's bras, so the contributions whose targets are the same for
// every bra of the pass -- K[a][c], K[a][d] (rows of the common shell A,
// columns of the lane's ket) and J[c][d] (the lane's ket) -- are summed in
// registers over the bras (R precision: FP32 quartets accumulate in FP32
// per pass, i.e. per quartet batch) and added to memory once per pass.
// Only K[b][c], K[b][d] (rows of each bra's own B) go to memory per quartet,
// and J[a][b] once per bra and pass after a warp reduction.  The density
// elements of row block A and of the lane's ket (D_cd, D_ad, D_ac) are read
// once per pass.  Screening (Q_bra Q_ket >= cut), the canonical order (ket
// position <= bra position when bra and ket come from one list) and the
// precision slice (FP32 when Q_bra Q_ket M_item < fp32_cut) are per-lane
// masks; a bra none of whose quartets is active in the pass is skipped.
// Densities after the first (nb > 1 or a nonsymmetric density) are
// digested quartet by quartet.
// ---------------------------------------------------------------------------
// One quartet's digestion of density e with every target added to memory.
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void digest_one(const JKArgs& args, const QuartetGeom& g, const R* out, int e) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  constexpr int NA = CI::NA, NB = CI::NB, NC = CI::NC, ND = CI::ND;
  const double s = g.scale;
  const long long base = args.mol_base[g.mol];
  const int n = args.mol_n[g.mol];
  const R* dm = DensSel<R>::get(args) + e * args.dstride + base;
  auto dv = [&](int r, int c) -> R { return __ldg(dm + (long long)r * n + c); };
#define V_(a, b, c, d) (out[(((a) * NB + (b)) * NC + (c)) * ND + (d)])
  if (args.with_j && e < args.nsym) {
    double* vj = args.vj + e * args.dstride + base;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        R acc = R(0);
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int d = 0; d < ND; ++d) acc += V_(a, b, c, d) * dv(g.aoC + c, g.aoD + d);
        atomicAdd(vj + (long long)(g.aoA + a) * n + g.aoB + b, 2.0 * s * double(acc));
      }
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        R acc = R(0);
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
          for (int b = 0; b < NB; ++b) acc += V_(a, b, c, d) * dv(g.aoA + a, g.aoB + b);
        atomicAdd(vj + (long long)(g.aoC + c) * n + g.aoD + d, 2.0 * s * double(acc));
      }
  }
  if (args.with_k) {
    double* vk = args.vk + e * args.dstride + base;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        R acc = R(0);
#pragma unroll
        for (int b = 0; b < NB; ++b)
#pragma unroll
          for (int d = 0; d < ND; ++d) acc += V_(a, b, c, d) * dv(g.aoB + b, g.aoD + d);
        atomicAdd(vk + (long long)(g.aoA + a) * n + g.aoC + c, s * double(acc));
      }
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        R acc = R(0);
#pragma unroll
        for (int b = 0; b < NB; ++b)
#pragma unroll
          for (int c = 0; c < NC; ++c) acc += V_(a, b, c, d) * dv(g.aoB + b, g.aoC + c);
        atomicAdd(vk + (long long)(g.aoA + a) * n + g.aoD + d, s * double(acc));
      }
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        R acc = R(0);
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
          for (int d = 0; d < ND; ++d) acc += V_(a, b, c, d) * dv(g.aoA + a, g.aoD + d);
        atomicAdd(vk + (long long)(g.aoB + b) * n + g.aoC + c, s * double(acc));
      }
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        R acc = R(0);
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
          for (int c = 0; c < NC; ++c) acc += V_(a, b, c, d) * dv(g.aoA + a, g.aoC + c);
        atomicAdd(vk + (long long)(g.aoB + b) * n + g.aoD + d, s * double(acc));
      }
  }
#undef V_
}

template <int LA, int LB, int LC, int LD>
struct GrpAcc {
  using CI = ClassInfo<LA, LB, LC, LD>;
  // per-lane sums over a pass: J[c][d], K[a][c], K[a][d]
  static constexpr int OJ = 0, OKC = CI::NC * CI::ND, OKD = OKC + CI::NA * CI::NC, N = OKD + CI::NA * CI::ND;
};

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128, (RegMinBlocks<LA, LB, LC, LD, R>::value))
    jk_grp_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GA = GrpAcc<LA, LB, LC, LD>;
  using PA_t = typename PrimData<R>::A;
  using PB_t = typename PrimData<R>::B;
  constexpr int NA = CI::NA, NB = CI::NB, NC = CI::NC, ND = CI::ND;
  __shared__ PA_t s_pp[kRegWarps][kBraPrimCache];
  __shared__ PB_t s_aux[kRegWarps][kBraPrimCache];
  // the pass sums live in shared memory, one private column per lane
  __shared__ R s_acc[kRegWarps][GA::N <= 32 ? GA::N : 1][32];
  constexpr bool kSharedBoys = sizeof(R) == 4 && CI::NROOT <= 3;
  __shared__ __align__(16) float s_boys[kSharedBoys ? 401 * 8 : 4];
  if constexpr (kSharedBoys) {
    const float4* src = reinterpret_cast<const float4*>(args.tb.boys_s_f + (CI::NROOT - 1) * 401 * 8);
    float4* dst = reinterpret_cast<float4*>(s_boys);
    for (int i = threadIdx.x; i < 401 * 2; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // persistent warps: items are taken from the launch's queue in list order
  // (the host sorts them by cost, longest first)
  for (;;) {
  int item = 0;
  if (lane == 0) item = atomicAdd(args.queue, 1);
  item = __shfl_sync(0xffffffffu, item, 0);
  if (item >= args.nwork) break;
  if (args.item_skip && args.item_skip[item]) continue;   // its FP64 quartets run from the flat list
  const int4 w = args.work[item];  // (bra-order begin, bra count, ket begin, ket end)
  const double qm = args.split_mode != 0 ? args.item_m[item] : 0.0;
  const double cut = args.cutoff;
  const int* __restrict__ bord = args.bra_bord;
  // the common A shell: Cartesian offset and molecule from the first bra
  const int p0 = bord[w.x];
  const int aoA = args.bra_ix[p0].z;
  const int mol = (int)args.bra_ra[p0].w;
  const long long mbase = args.mol_base[mol];
  const int n = args.mol_n[mol];
  const R* dm0 = DensSel<R>::get(args) + mbase;
  auto dv = [&](int r, int c) -> R { return __ldg(dm0 + (long long)r * n + c); };
  const bool doj = args.with_j != 0 && args.nsym > 0, dok = args.with_k != 0;
  R(*acc)[32] = s_acc[warp];
  for (int k0 = w.z; k0 < w.w; k0 += 32) {
    const bool valid = k0 + lane < w.w;
    const int k = valid ? k0 + lane : w.w - 1;
    const double qk = args.ket_q[k];
    const double4 kra = args.ket_ra[k], kab = args.ket_ab[k];
    const int4 kix = args.ket_ix[k];
    const int aoC = kix.z, aoD = kix.w;
#pragma unroll
    for (int i = 0; i < GA::N; ++i) acc[i][lane] = R(0);
    bool any = false;
    for (int bi = 0; bi < w.y; ++bi) {
      const int pos = bord[w.x + bi];
      const double qq = args.bra_q[pos] * qk;
      bool act = valid && qq >= cut && (!args.same_list || k <= pos);
      if (args.split_mode == 1) act = act && !(qq * qm < args.fp32_cut);
      else if (args.split_mode == 2) act = act && (qq * qm < args.fp32_cut);
      if (!__any_sync(0xffffffffu, act)) continue;
      any = any || act;
      const BraRec br = load_bra(args, pos);
      const int ppb = br.ix.x, npb = br.ix.y;
      const bool cached = npb <= kBraPrimCache;
      __syncwarp();
      if (cached)
        for (int i = lane; i < npb; i += 32) {
          s_pp[warp][i] = PrimData<R>::a(args, ppb + i);
          s_aux[warp][i] = PrimData<R>::b(args, ppb + i);
        }
      __syncwarp();
      const PA_t* bpp = cached ? s_pp[warp] : (sizeof(R) == 4 ? (const PA_t*)(args.pp_f + ppb)
                                                             : (const PA_t*)(args.pp_data + ppb));
      const PB_t* baux = cached ? s_aux[warp] : (sizeof(R) == 4 ? (const PB_t*)(args.pp_f2 + ppb)
                                                               : (const PB_t*)(args.pp_aux + ppb));
      QuartetGeom g;
      g.A = g.B = g.C = g.D = -1;
      g.ppa = ppb; g.npa = npb; g.ppc = kix.x; g.npc = kix.y;
      g.ax = br.ra.x; g.ay = br.ra.y; g.az = br.ra.z;
      g.cx = kra.x; g.cy = kra.y; g.cz = kra.z;
      g.abx = br.ab.x; g.aby = br.ab.y; g.abz = br.ab.z;
      g.cdx = kab.x; g.cdy = kab.y; g.cdz = kab.z;
      g.aoA = aoA; g.aoB = br.ix.w; g.aoC = aoC; g.aoD = aoD;
      g.mol = mol;
      g.scale = (aoA == br.ix.w ? 0.5 : 1.0) * (aoC == aoD ? 0.5 : 1.0) * (args.same_list && k == pos ? 0.5 : 1.0);
      g.omega2 = args.omega2;
      R out[CI::NOUT];
      quartet_block_reg<LA, LB, LC, LD, R>(args, g, bpp, baux, out, s_boys);
      const int aoB = br.ix.w;
      const R sR = act ? R(g.scale) : R(0);
#define V_(a, b, c, d) (out[(((a) * NB + (b)) * NC + (c)) * ND + (d)])
      if (doj) {
        // J[a][b] of this bra: warp-reduced, one add per element and pass
        double* vj = args.vj + mbase;
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
          for (int b = 0; b < NB; ++b) {
            R s = R(0);
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
              for (int d = 0; d < ND; ++d) s += V_(a, b, c, d) * dv(aoC + c, aoD + d);
            double v = 2.0 * double(sR) * double(s);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0 && v != 0.0) atomicAdd(vj + (long long)(aoA + a) * n + aoB + b, v);
          }
        // J[c][d] of the lane's ket, summed over the bras
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            R s = R(0);
#pragma unroll
            for (int a = 0; a < NA; ++a)
#pragma unroll
              for (int b = 0; b < NB; ++b) s += V_(a, b, c, d) * dv(aoA + a, aoB + b);
            acc[GA::OJ + c * ND + d][lane] += R(2) * sR * s;
          }
      }
      if (dok) {
        double* vk = args.vk + mbase;
        // K[a][c] += s sum_bd V D_bd, K[a][d] += s sum_bc V D_bc (pass sums)
#pragma unroll
        for (int a = 0; a < NA; ++a) {
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            R s = R(0);
#pragma unroll
            for (int b = 0; b < NB; ++b)
#pragma unroll
              for (int d = 0; d < ND; ++d) s += V_(a, b, c, d) * dv(aoB + b, aoD + d);
            acc[GA::OKC + a * NC + c][lane] += sR * s;
          }
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            R s = R(0);
#pragma unroll
            for (int b = 0; b < NB; ++b)
#pragma unroll
              for (int c = 0; c < NC; ++c) s += V_(a, b, c, d) * dv(aoB + b, aoC + c);
            acc[GA::OKD + a * ND + d][lane] += sR * s;
          }
        }
        // K[b][c], K[b][d]: rows of this bra's B, added per quartet
        if (act) {
#pragma unroll
          for (int b = 0; b < NB; ++b) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              R s = R(0);
#pragma unroll
              for (int a = 0; a < NA; ++a)
#pragma unroll
                for (int d = 0; d < ND; ++d) s += V_(a, b, c, d) * dv(aoA + a, aoD + d);
              atomicAdd(vk + (long long)(aoB + b) * n + aoC + c, double(sR) * double(s));
            }
#pragma unroll
            for (int d = 0; d < ND; ++d) {
              R s = R(0);
#pragma unroll
              for (int a = 0; a < NA; ++a)
#pragma unroll
                for (int c = 0; c < NC; ++c) s += V_(a, b, c, d) * dv(aoA + a, aoC + c);
              atomicAdd(vk + (long long)(aoB + b) * n + aoD + d, double(sR) * double(s));
            }
          }
        }
      }
#undef V_
      if (act)
        for (int e = 1; e < args.ndm; ++e) digest_one<LA, LB, LC, LD, R>(args, g, out, e);
    }
    // the pass sums of density 0: J[c][d], K[a][c], K[a][d]
    if (any) {
      if (doj) {
        double* vj = args.vj + mbase;
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int d = 0; d < ND; ++d)
            atomicAdd(vj + (long long)(aoC + c) * n + aoD + d, double(acc[GA::OJ + c * ND + d][lane]));
      }
      if (dok) {
        double* vk = args.vk + mbase;
#pragma unroll
        for (int a = 0; a < NA; ++a) {
#pragma unroll
          for (int c = 0; c < NC; ++c)
            atomicAdd(vk + (long long)(aoA + a) * n + aoC + c, double(acc[GA::OKC + a * NC + c][lane]));
#pragma unroll
          for (int d = 0; d < ND; ++d)
            atomicAdd(vk + (long long)(aoA + a) * n + aoD + d, double(acc[GA::OKD + a * ND + d][lane]));
        }
      }
    }
  }
  }  // items
}

// ---------------------------------------------------------------------------
// Register path on grouped lists: a bra entry carries GB contraction
// combinations of its parent shell pair and a ket entry GK; the primitive
// pairs are shared by the combinations and carry their coefficients
// (pp_c), so each primitive quartet is evaluated once and added, weighted,
// to the GB*GK contracted blocks.  Every combination is digested like a
// quartet of work shells; a diagonal parent pair (A and B the same shell)
// holds both orders of its combinations, each digested with weight 1/2.
// ---------------------------------------------------------------------------
template <typename R> struct CoefSel;
template <> struct CoefSel<double> {
  using T = double4;
  static __device__ __forceinline__ T get(const JKArgs& a, int i) { return a.pp_c[i]; }
};
template <> struct CoefSel<float> {
  using T = float4;
  static __device__ __forceinline__ T get(const JKArgs& a, int i) { return a.pp_cf[i]; }
};
template <int K, typename C4>
__device__ __forceinline__ auto comp(const C4& v) {
  if constexpr (K == 0) return v.x;
  else if constexpr (K == 1) return v.y;
  else if constexpr (K == 2) return v.z;
  else return v.w;
}

// PRESUM: the bra combinations are summed over the bra primitives first and
// the ket coefficients applied once per ket primitive (GB NO + GB GK NO / npa
// multiply-adds per primitive quartet instead of GB GK NO): used by the flat
// FP64 kernel, whose quartets are the heavily contracted core ones (its FP64
// slice went from 14.9 to 8.4 ms per C1 split build); the bra-group kernels
// keep the direct form, which measured up to 14% faster on their classes.
template <int LA, int LB, int LC, int LD, typename R, int GB, int GK, bool PRESUM = false>
__device__ __forceinline__ void quartet_block_gen(const JKArgs& args, const QuartetGeom& g,
                                                  const typename PrimData<R>::A* bpp,
                                                  const typename PrimData<R>::B* baux,
                                                  const typename CoefSel<R>::T* bco, R* out,
                                                  const float* s_boys) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GI = GIdx<LA, LB, LC, LD>;
  constexpr int N = CI::NROOT, NO = CI::NOUT;
#pragma unroll
  for (int o = 0; o < GB * GK * NO; ++o) out[o] = R(0);
  const float3 ac = make_float3(float(g.ax - g.cx), float(g.ay - g.cy), float(g.az - g.cz));
  auto Qn = PrimData<R>::a(args, g.ppc);
  auto QAn = PrimData<R>::b(args, g.ppc);
  auto Cn = CoefSel<R>::get(args, g.ppc);
  for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
    const auto Q = Qn;
    const auto QA = QAn;
    const auto CK = Cn;
    if (j + 1 < g.ppc + g.npc) {
      Qn = PrimData<R>::a(args, j + 1);
      QAn = PrimData<R>::b(args, j + 1);
      Cn = CoefSel<R>::get(args, j + 1);
    }
    R sb[PRESUM ? GB * NO : 1];
#pragma unroll
    for (int o = 0; o < (PRESUM ? GB * NO : 1); ++o) sb[o] = R(0);
    for (int i = 0; i < g.npa; ++i) {
      PrimQ<R> s;
      prim_any<R>(g, ac, bpp[i], baux[i], Q, QA, s);
      R x[N], w[N];
      if constexpr (sizeof(R) == 4 && N <= 3)
        rys_small<N, float, 10, 6>(s.t, x, w, s_boys);
      else
        rys_roots<N, R>(s.t, x, w, args.tb);
      R tmp[NO];
#pragma unroll
      for (int o = 0; o < NO; ++o) tmp[o] = R(0);
#pragma unroll
      for (int r = 0; r < N; ++r) {
        RootCoef<R> rc;
        root_coef<R>(s, x[r], rc);
        R gx[CI::NG], gy[CI::NG], gz[CI::NG];
        build_g<LA, LB, LC, LD, R>(rc.c00[0], rc.c0p[0], rc.b10, rc.b01, rc.b00, R(1), R(g.abx),
                                   R(g.cdx), gx);
        build_g<LA, LB, LC, LD, R>(rc.c00[1], rc.c0p[1], rc.b10, rc.b01, rc.b00, R(1), R(g.aby),
                                   R(g.cdy), gy);
        build_g<LA, LB, LC, LD, R>(rc.c00[2], rc.c0p[2], rc.b10, rc.b01, rc.b00, w[r] * s.pref,
                                   R(g.abz), R(g.cdz), gz);
        static_for<0, NO>([&](auto O) {
          constexpr int o = decltype(O)::value;
          constexpr int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
          constexpr int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
          constexpr int jx = GI::idx(cart_lx(LA, ia), cart_lx(LB, ib), cart_lx(LC, ic), cart_lx(LD, id));
          constexpr int jy = GI::idx(cart_ly(LA, ia), cart_ly(LB, ib), cart_ly(LC, ic), cart_ly(LD, id));
          constexpr int jz = GI::idx(cart_lz(LA, ia), cart_lz(LB, ib), cart_lz(LC, ic), cart_lz(LD, id));
          tmp[o] += gx[jx] * gy[jy] * gz[jz];
        });
      }
      const auto CB = bco[i];
      if constexpr (PRESUM) {
        static_for<0, GB>([&](auto BI) {
          constexpr int b = decltype(BI)::value;
          const R cb = R(comp<b>(CB));
#pragma unroll
          for (int o = 0; o < NO; ++o) sb[b * NO + o] += cb * tmp[o];
        });
      } else {
        static_for<0, GB>([&](auto BI) {
          constexpr int b = decltype(BI)::value;
          const R cb = R(comp<b>(CB));
          static_for<0, GK>([&](auto KI) {
            constexpr int k = decltype(KI)::value;
            const R wgt = cb * R(comp<k>(CK));
#pragma unroll
            for (int o = 0; o < NO; ++o) out[(b * GK + k) * NO + o] += wgt * tmp[o];
          });
        });
      }
    }
    if constexpr (PRESUM) {
      static_for<0, GB>([&](auto BI) {
        constexpr int b = decltype(BI)::value;
        static_for<0, GK>([&](auto KI) {
          constexpr int k = decltype(KI)::value;
          const R ck = R(comp<k>(CK));
#pragma unroll
          for (int o = 0; o < NO; ++o) out[(b * GK + k) * NO + o] += ck * sb[b * NO + o];
        });
      });
    }
  }
}

template <int LA, int LB, int LC, int LD, typename R, int GB, int GK>
__global__ void __launch_bounds__(128, (RegMinBlocks<LA, LB, LC, LD, R,
                                                     (GB * GK + 1) * ClassInfo<LA, LB, LC, LD>::NOUT>::value))
    jk_reg_gen_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using PA_t = typename PrimData<R>::A;
  using PB_t = typename PrimData<R>::B;
  using C4 = typename CoefSel<R>::T;
  constexpr int NO = CI::NOUT;
  __shared__ PA_t s_pp[kRegWarps][kBraPrimCache];
  __shared__ PB_t s_aux[kRegWarps][kBraPrimCache];
  __shared__ C4 s_co[kRegWarps][kBraPrimCache];
  __shared__ double s_jab[kRegWarps][GB * CI::NAB];
  constexpr bool kSharedBoys = sizeof(R) == 4 && CI::NROOT <= 3;
  __shared__ __align__(16) float s_boys[kSharedBoys ? 401 * 8 : 4];
  if constexpr (kSharedBoys) {
    const float4* src = reinterpret_cast<const float4*>(args.tb.boys_s_f + (CI::NROOT - 1) * 401 * 8);
    float4* dst = reinterpret_cast<float4*>(s_boys);
    for (int i = threadIdx.x; i < 401 * 2; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x * kRegWarps + warp;
  if (item >= args.nwork) return;
  const int4 w = args.work[item];
  int kb = w.y, ke = w.z;
  if (args.split_mode != 0) {
    const int sp = args.split[item];
    if (args.split_mode == 1) ke = min(ke, sp);
    else kb = max(kb, sp);
  }
  if (kb >= ke) return;
  const BraRec br = load_bra(args, w.x);
  const int ppb = br.ix.x, npb = br.ix.y;
  // bra combinations: Cartesian offsets of A and B, parent-diagonal flag
  int aoA[GB], aoB[GB];
  bool bdiag;
  {
    int4 gx = make_int4(br.ix.z == br.ix.w, 0, 0, 0), gy = make_int4(0, 0, 0, 0);
    if constexpr (GB > 1) {
      gx = args.bra_gx[w.x];
      gy = args.bra_gy[w.x];
    }
    const int a4[4] = {br.ix.z, gx.z, gy.x, gy.z}, b4[4] = {br.ix.w, gx.w, gy.y, gy.w};
#pragma unroll
    for (int b = 0; b < GB; ++b) { aoA[b] = a4[b]; aoB[b] = b4[b]; }
    bdiag = gx.x != 0;
  }
  const bool cached = npb <= kBraPrimCache;
  if (cached)
    for (int i = lane; i < npb; i += 32) {
      s_pp[warp][i] = PrimData<R>::a(args, ppb + i);
      s_aux[warp][i] = PrimData<R>::b(args, ppb + i);
      s_co[warp][i] = CoefSel<R>::get(args, ppb + i);
    }
  const bool acc_j = args.with_j && args.nsym == 1;
  for (int i = lane; i < GB * CI::NAB; i += 32) s_jab[warp][i] = 0.0;
  __syncwarp();
  const PA_t* bpp = cached ? s_pp[warp] : (sizeof(R) == 4 ? (const PA_t*)(args.pp_f + ppb)
                                                         : (const PA_t*)(args.pp_data + ppb));
  const PB_t* baux = cached ? s_aux[warp] : (sizeof(R) == 4 ? (const PB_t*)(args.pp_f2 + ppb)
                                                           : (const PB_t*)(args.pp_aux + ppb));
  const C4* bco = cached ? s_co[warp] : (sizeof(R) == 4 ? (const C4*)(args.pp_cf + ppb)
                                                       : (const C4*)(args.pp_c + ppb));
  QuartetGeom g;
  for (int k0 = kb; k0 < ke; k0 += 32) {
    const bool active = k0 + lane < ke;
    const int k = active ? k0 + lane : ke - 1;
    load_quartet_rec(args, br, k, g);
    int aoC[GK], aoD[GK];
    bool kdiag;
    {
      int4 gx = make_int4(g.aoC == g.aoD, 0, 0, 0), gy = make_int4(0, 0, 0, 0);
      if constexpr (GK > 1) {
        gx = args.ket_gx[k];
        gy = args.ket_gy[k];
      }
      const int c4[4] = {g.aoC, gx.z, gy.x, gy.z}, d4[4] = {g.aoD, gx.w, gy.y, gy.w};
#pragma unroll
      for (int c = 0; c < GK; ++c) { aoC[c] = c4[c]; aoD[c] = d4[c]; }
      kdiag = gx.x != 0;
    }
    const double sbk = (bdiag ? 0.5 : 1.0) * (kdiag ? 0.5 : 1.0) * (args.same_list && k == w.x ? 0.5 : 1.0);
    R out[GB * GK * NO];
    quartet_block_gen<LA, LB, LC, LD, R, GB, GK>(args, g, bpp, baux, bco, out, s_boys);
#pragma unroll
    for (int b = 0; b < GB; ++b)
#pragma unroll
      for (int c = 0; c < GK; ++c) {
        QuartetGeom gc = g;
        gc.aoA = aoA[b]; gc.aoB = aoB[b]; gc.aoC = aoC[c]; gc.aoD = aoD[c];
        gc.scale = sbk;
        DensPre<LA, LB, LC, LD, R> pre;
        pre.load(args, gc);
        digest_reg<LA, LB, LC, LD, R>(args, gc, out + (b * GK + c) * NO, acc_j, active,
                                      s_jab[warp] + b * CI::NAB, pre);
      }
  }
  if (acc_j) {
    __syncwarp();
    const int mol = (int)br.ra.w;
    double* vj = args.vj + args.mol_base[mol];
    const int n = args.mol_n[mol];
#pragma unroll
    for (int b = 0; b < GB; ++b)
      for (int ab = lane; ab < CI::NAB; ab += 32) {
        const double v = s_jab[warp][b * CI::NAB + ab];
        if (v != 0.0) atomicAdd(vj + (long long)(aoA[b] + ab / CI::NB) * n + aoB[b] + ab % CI::NB, v);
      }
  }
}

// ---------------------------------------------------------------------------
// The register path over bra groups on grouped lists: bra entries carry GB
// contraction combinations (whose A shells the whole group shares) and ket
// entries GK; each primitive quartet is evaluated once for all GB x GK
// combination blocks (quartet_block_gen), and every block is digested as in
// jk_grp_kernel: J[c][d], K[a][c], K[a][d] summed per lane over the pass's
// bras, one sum set per (bra combination, ket combination).
// ---------------------------------------------------------------------------
template <int LA, int LB, int LC, int LD, int GB, int GK>
struct GrpGenAcc {
  using CI = ClassInfo<LA, LB, LC, LD>;
  static constexpr int OJ = 0;                                  // [GK][NC*ND]
  static constexpr int OKC = GK * CI::NC * CI::ND;              // [GB][GK][NA*NC]
  static constexpr int OKD = OKC + GB * GK * CI::NA * CI::NC;   // [GB][GK][NA*ND]
  static constexpr int N = OKD + GB * GK * CI::NA * CI::ND;
};

template <int LA, int LB, int LC, int LD, typename R, int GB, int GK>
__global__ void __launch_bounds__(128, (RegMinBlocks<LA, LB, LC, LD, R,
                                                     (GB * GK + 1) * ClassInfo<LA, LB, LC, LD>::NOUT>::value))
    jk_grp_gen_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using GA = GrpGenAcc<LA, LB, LC, LD, GB, GK>;
  using PA_t = typename PrimData<R>::A;
  using PB_t = typename PrimData<R>::B;
  using C4 = typename CoefSel<R>::T;
  constexpr int NA = CI::NA, NB = CI::NB, NC = CI::NC, ND = CI::ND, NO = CI::NOUT;
  __shared__ PA_t s_pp[kRegWarps][kBraPrimCache];
  __shared__ PB_t s_aux[kRegWarps][kBraPrimCache];
  __shared__ C4 s_co[kRegWarps][kBraPrimCache];
  // the pass sums (GA::N values of 32 lanes per warp) in dynamic shared
  // memory, sized by the launcher
  extern __shared__ __align__(16) unsigned char s_acc_raw[];
  R(*s_acc)[GA::N][32] = reinterpret_cast<R(*)[GA::N][32]>(s_acc_raw);
  constexpr bool kSharedBoys = sizeof(R) == 4 && CI::NROOT <= 3;
  __shared__ __align__(16) float s_boys[kSharedBoys ? 401 * 8 : 4];
  if constexpr (kSharedBoys) {
    const float4* src = reinterpret_cast<const float4*>(args.tb.boys_s_f + (CI::NROOT - 1) * 401 * 8);
    float4* dst = reinterpret_cast<float4*>(s_boys);
    for (int i = threadIdx.x; i < 401 * 2; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // persistent warps: items are taken from the launch's queue in list order
  // (the host sorts them by cost, longest first)
  for (;;) {
  int item = 0;
  if (lane == 0) item = atomicAdd(args.queue, 1);
  item = __shfl_sync(0xffffffffu, item, 0);
  if (item >= args.nwork) break;
  if (args.item_skip && args.item_skip[item]) continue;   // its FP64 quartets run from the flat list
  const int4 w = args.work[item];  // (bra-order begin, bra count, ket begin, ket end)
  const double qm = args.split_mode != 0 ? args.item_m[item] : 0.0;
  const double cut = args.cutoff;
  const int* __restrict__ bord = args.bra_bord;
  // the group's A shells, one per bra combination (shared by every bra of the group)
  const int p0 = bord[w.x];
  int aoA[GB];
  {
    const int4 ix = args.bra_ix[p0];
    int4 gx = make_int4(0, 0, 0, 0), gy = make_int4(0, 0, 0, 0);
    if constexpr (GB > 1) {
      gx = args.bra_gx[p0];
      gy = args.bra_gy[p0];
    }
    const int a4[4] = {ix.z, gx.z, gy.x, gy.z};
#pragma unroll
    for (int b = 0; b < GB; ++b) aoA[b] = a4[b];
  }
  const int mol = (int)args.bra_ra[p0].w;
  const long long mbase = args.mol_base[mol];
  const int n = args.mol_n[mol];
  const R* dm0 = DensSel<R>::get(args) + mbase;
  auto dv = [&](int r, int c) -> R { return __ldg(dm0 + (long long)r * n + c); };
  const bool doj = args.with_j != 0 && args.nsym > 0, dok = args.with_k != 0;
  R(*acc)[32] = s_acc[warp];
  for (int k0 = w.z; k0 < w.w; k0 += 32) {
    const bool valid = k0 + lane < w.w;
    const int k = valid ? k0 + lane : w.w - 1;
    const double qk = args.ket_q[k];
    const double4 kra = args.ket_ra[k], kab = args.ket_ab[k];
    const int4 kix = args.ket_ix[k];
    int aoC[GK], aoD[GK];
    bool kdiag;
    {
      int4 gx = make_int4(kix.z == kix.w, 0, 0, 0), gy = make_int4(0, 0, 0, 0);
      if constexpr (GK > 1) {
        gx = args.ket_gx[k];
        gy = args.ket_gy[k];
      }
      const int c4[4] = {kix.z, gx.z, gy.x, gy.z}, d4[4] = {kix.w, gx.w, gy.y, gy.w};
#pragma unroll
      for (int c = 0; c < GK; ++c) { aoC[c] = c4[c]; aoD[c] = d4[c]; }
      kdiag = gx.x != 0;
    }
#pragma unroll
    for (int i = 0; i < GA::N; ++i) acc[i][lane] = R(0);
    bool any = false;
    for (int bi = 0; bi < w.y; ++bi) {
      const int pos = bord[w.x + bi];
      const double qq = args.bra_q[pos] * qk;
      bool act = valid && qq >= cut && (!args.same_list || k <= pos);
      if (args.split_mode == 1) act = act && !(qq * qm < args.fp32_cut);
      else if (args.split_mode == 2) act = act && (qq * qm < args.fp32_cut);
      if (!__any_sync(0xffffffffu, act)) continue;
      any = any || act;
      const BraRec br = load_bra(args, pos);
      const int ppb = br.ix.x, npb = br.ix.y;
      int aoB[GB];
      bool bdiag;
      {
        int4 gx = make_int4(br.ix.z == br.ix.w, 0, 0, 0), gy = make_int4(0, 0, 0, 0);
        if constexpr (GB > 1) {
          gx = args.bra_gx[pos];
          gy = args.bra_gy[pos];
        }
        const int b4[4] = {br.ix.w, gx.w, gy.y, gy.w};
#pragma unroll
        for (int b = 0; b < GB; ++b) aoB[b] = b4[b];
        bdiag = gx.x != 0;
      }
      const bool cached = npb <= kBraPrimCache;
      __syncwarp();
      if (cached)
        for (int i = lane; i < npb; i += 32) {
          s_pp[warp][i] = PrimData<R>::a(args, ppb + i);
          s_aux[warp][i] = PrimData<R>::b(args, ppb + i);
          s_co[warp][i] = CoefSel<R>::get(args, ppb + i);
        }
      __syncwarp();
      const PA_t* bpp = cached ? s_pp[warp] : (sizeof(R) == 4 ? (const PA_t*)(args.pp_f + ppb)
                                                             : (const PA_t*)(args.pp_data + ppb));
      const PB_t* baux = cached ? s_aux[warp] : (sizeof(R) == 4 ? (const PB_t*)(args.pp_f2 + ppb)
                                                               : (const PB_t*)(args.pp_aux + ppb));
      const C4* bco = cached ? s_co[warp] : (sizeof(R) == 4 ? (const C4*)(args.pp_cf + ppb)
                                                           : (const C4*)(args.pp_c + ppb));
      QuartetGeom g;
      g.A = g.B = g.C = g.D = -1;
      g.ppa = ppb; g.npa = npb; g.ppc = kix.x; g.npc = kix.y;
      g.ax = br.ra.x; g.ay = br.ra.y; g.az = br.ra.z;
      g.cx = kra.x; g.cy = kra.y; g.cz = kra.z;
      g.abx = br.ab.x; g.aby = br.ab.y; g.abz = br.ab.z;
      g.cdx = kab.x; g.cdy = kab.y; g.cdz = kab.z;
      g.mol = mol;
      g.omega2 = args.omega2;
      const double sbk = (bdiag ? 0.5 : 1.0) * (kdiag ? 0.5 : 1.0) * (args.same_list && k == pos ? 0.5 : 1.0);
      R out[GB * GK * NO];
      quartet_block_gen<LA, LB, LC, LD, R, GB, GK>(args, g, bpp, baux, bco, out, s_boys);
      const R sR = act ? R(sbk) : R(0);
#pragma unroll
      for (int b = 0; b < GB; ++b)
#pragma unroll
        for (int c = 0; c < GK; ++c) {
          const R* o = out + (b * GK + c) * NO;
          const int oA = aoA[b], oB = aoB[b], oC = aoC[c], oD = aoD[c];
#define V_(a, bb, cc, d) (o[(((a) * NB + (bb)) * NC + (cc)) * ND + (d)])
          if (doj) {
            double* vj = args.vj + mbase;
#pragma unroll
            for (int a = 0; a < NA; ++a)
#pragma unroll
              for (int bb = 0; bb < NB; ++bb) {
                R s = R(0);
#pragma unroll
                for (int cc = 0; cc < NC; ++cc)
#pragma unroll
                  for (int d = 0; d < ND; ++d) s += V_(a, bb, cc, d) * dv(oC + cc, oD + d);
                double v = 2.0 * double(sR) * double(s);
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
                if (lane == 0 && v != 0.0) atomicAdd(vj + (long long)(oA + a) * n + oB + bb, v);
              }
#pragma unroll
            for (int cc = 0; cc < NC; ++cc)
#pragma unroll
              for (int d = 0; d < ND; ++d) {
                R s = R(0);
#pragma unroll
                for (int a = 0; a < NA; ++a)
#pragma unroll
                  for (int bb = 0; bb < NB; ++bb) s += V_(a, bb, cc, d) * dv(oA + a, oB + bb);
                acc[GA::OJ + c * NC * ND + cc * ND + d][lane] += R(2) * sR * s;
              }
          }
          if (dok) {
            double* vk = args.vk + mbase;
#pragma unroll
            for (int a = 0; a < NA; ++a) {
#pragma unroll
              for (int cc = 0; cc < NC; ++cc) {
                R s = R(0);
#pragma unroll
                for (int bb = 0; bb < NB; ++bb)
#pragma unroll
                  for (int d = 0; d < ND; ++d) s += V_(a, bb, cc, d) * dv(oB + bb, oD + d);
                acc[GA::OKC + (b * GK + c) * NA * NC + a * NC + cc][lane] += sR * s;
              }
#pragma unroll
              for (int d = 0; d < ND; ++d) {
                R s = R(0);
#pragma unroll
                for (int bb = 0; bb < NB; ++bb)
#pragma unroll
                  for (int cc = 0; cc < NC; ++cc) s += V_(a, bb, cc, d) * dv(oB + bb, oC + cc);
                acc[GA::OKD + (b * GK + c) * NA * ND + a * ND + d][lane] += sR * s;
              }
            }
            if (act) {
#pragma unroll
              for (int bb = 0; bb < NB; ++bb) {
#pragma unroll
                for (int cc = 0; cc < NC; ++cc) {
                  R s = R(0);
#pragma unroll
                  for (int a = 0; a < NA; ++a)
#pragma unroll
                    for (int d = 0; d < ND; ++d) s += V_(a, bb, cc, d) * dv(oA + a, oD + d);
                  atomicAdd(vk + (long long)(oB + bb) * n + oC + cc, double(sR) * double(s));
                }
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                  R s = R(0);
#pragma unroll
                  for (int a = 0; a < NA; ++a)
#pragma unroll
                    for (int cc = 0; cc < NC; ++cc) s += V_(a, bb, cc, d) * dv(oA + a, oC + cc);
                  atomicAdd(vk + (long long)(oB + bb) * n + oD + d, double(sR) * double(s));
                }
              }
            }
          }
#undef V_
          if (act) {
            QuartetGeom gc = g;
            gc.aoA = oA; gc.aoB = oB; gc.aoC = oC; gc.aoD = oD;
            gc.scale = sbk;
            for (int e = 1; e < args.ndm; ++e) digest_one<LA, LB, LC, LD, R>(args, gc, o, e);
          }
        }
    }
    if (any) {
      if (doj) {
        double* vj = args.vj + mbase;
#pragma unroll
        for (int c = 0; c < GK; ++c)
#pragma unroll
          for (int cc = 0; cc < NC; ++cc)
#pragma unroll
            for (int d = 0; d < ND; ++d)
              atomicAdd(vj + (long long)(aoC[c] + cc) * n + aoD[c] + d, double(acc[GA::OJ + c * NC * ND + cc * ND + d][lane]));
      }
      if (dok) {
        double* vk = args.vk + mbase;
#pragma unroll
        for (int b = 0; b < GB; ++b)
#pragma unroll
          for (int c = 0; c < GK; ++c)
#pragma unroll
            for (int a = 0; a < NA; ++a) {
#pragma unroll
              for (int cc = 0; cc < NC; ++cc)
                atomicAdd(vk + (long long)(aoA[b] + a) * n + aoC[c] + cc,
                          double(acc[GA::OKC + (b * GK + c) * NA * NC + a * NC + cc][lane]));
#pragma unroll
              for (int d = 0; d < ND; ++d)
                atomicAdd(vk + (long long)(aoA[b] + a) * n + aoD[c] + d,
                          double(acc[GA::OKD + (b * GK + c) * NA * ND + a * ND + d][lane]));
            }
      }
    }
  }
  }  // items
}

// ---------------------------------------------------------------------------
// FP64 slice of a split build, for the bra-group items whose FP64 quartets
// are few (the leading kets of the leading bras, where the bra-group path
// would keep most lanes of a pass idle): border_kernel lists them as (bra
// position, ket position) and this kernel gives each lane one quartet, its
// block in registers and every digested element an atomic add.  Plain lists
// (GB = GK = 1) and grouped lists, digested as the bra-group kernels do.
// ---------------------------------------------------------------------------
template <int LA, int LB, int LC, int LD, int GB, int GK>
__global__ void __launch_bounds__(128) jk_flat_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  constexpr int NO = CI::NOUT;
  const int n = (int)min(*args.flat_n, (unsigned long long)args.flat_cap);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int2 q = args.flat[i];
    if (q.x < 0) continue;   // space of a reservation that did not fit
    const BraRec br = load_bra(args, q.x);
    QuartetGeom g;
    load_quartet_rec(args, br, q.y, g);
    const double4* bpp = args.pp_data + g.ppa;
    const double2* baux = args.pp_aux + g.ppa;
    if constexpr (GB == 1 && GK == 1) {
      double out[NO];
      quartet_block_reg<LA, LB, LC, LD, double>(args, g, bpp, baux, out, nullptr);
      for (int e = 0; e < args.ndm; ++e) digest_one<LA, LB, LC, LD, double>(args, g, out, e);
    } else {
      int aoA[GB], aoB[GB], aoC[GK], aoD[GK];
      bool bdiag, kdiag;
      {
        int4 gx = make_int4(br.ix.z == br.ix.w, 0, 0, 0), gy = make_int4(0, 0, 0, 0);
        if constexpr (GB > 1) {
          gx = args.bra_gx[q.x];
          gy = args.bra_gy[q.x];
        }
        const int a4[4] = {br.ix.z, gx.z, gy.x, gy.z}, b4[4] = {br.ix.w, gx.w, gy.y, gy.w};
#pragma unroll
        for (int b = 0; b < GB; ++b) { aoA[b] = a4[b]; aoB[b] = b4[b]; }
        bdiag = gx.x != 0;
      }
      {
        const int4 kix = args.ket_ix[q.y];
        int4 gx = make_int4(kix.z == kix.w, 0, 0, 0), gy = make_int4(0, 0, 0, 0);
        if constexpr (GK > 1) {
          gx = args.ket_gx[q.y];
          gy = args.ket_gy[q.y];
        }
        const int c4[4] = {kix.z, gx.z, gy.x, gy.z}, d4[4] = {kix.w, gx.w, gy.y, gy.w};
#pragma unroll
        for (int c = 0; c < GK; ++c) { aoC[c] = c4[c]; aoD[c] = d4[c]; }
        kdiag = gx.x != 0;
      }
      double out[GB * GK * NO];
      quartet_block_gen<LA, LB, LC, LD, double, GB, GK, true>(args, g, bpp, baux, args.pp_c + g.ppa, out, nullptr);
      const double sbk = (bdiag ? 0.5 : 1.0) * (kdiag ? 0.5 : 1.0) * (args.same_list && q.y == q.x ? 0.5 : 1.0);
#pragma unroll
      for (int b = 0; b < GB; ++b)
#pragma unroll
        for (int c = 0; c < GK; ++c) {
          QuartetGeom gc = g;
          gc.aoA = aoA[b]; gc.aoB = aoB[b]; gc.aoC = aoC[c]; gc.aoD = aoD[c];
          gc.scale = sbk;
          for (int e = 0; e < args.ndm; ++e) digest_one<LA, LB, LC, LD, double>(args, gc, out + (b * GK + c) * NO, e);
        }
    }
  }
}

// ---------------------------------------------------------------------------
// Team path: TEAM lanes of one warp share a quartet.  Rys functions and the
// 3*NROOT (root, axis) 2D-integral tables are built cooperatively in shared
// memory; each lane accumulates a strided slice of the Cartesian block; the
// contracted block is staged in shared memory for digestion (one atomic per
// digested element).  Blocks larger than TEAM*NK are done in passes.
// ---------------------------------------------------------------------------
template <int LA, int LB, int LC, int LD, int TEAM>
struct TeamCfg {
  using CI = ClassInfo<LA, LB, LC, LD>;
  static constexpr int NK_MAX = 48;
  static constexpr int NK = (CI::NOUT + TEAM - 1) / TEAM < NK_MAX ? (CI::NOUT + TEAM - 1) / TEAM : NK_MAX;
  static constexpr int PASS = TEAM * NK;
  static constexpr int NPASS = (CI::NOUT + PASS - 1) / PASS;
  static constexpr int G_ELEMS = 3 * CI::NROOT * CI::NG;
  static constexpr int ROOT_ELEMS = 2 * CI::NROOT;
  // G region (+ roots) and the staged block V; V may alias G in one pass.
  static constexpr int GR = G_ELEMS + ROOT_ELEMS;
  static constexpr int ELEMS = NPASS == 1 ? (GR > CI::NOUT ? GR : CI::NOUT) : GR + CI::NOUT;
};

template <int LA, int LB, int LC, int LD, typename R, int TEAM>
__device__ __forceinline__ void team_block(const JKArgs& args, const QuartetGeom& g, R* sm,
                                           double* vsm, int lane, unsigned mask) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using TC = TeamCfg<LA, LB, LC, LD, TEAM>;
  using GI = GIdx<LA, LB, LC, LD>;
  constexpr int N = CI::NROOT;
  constexpr int NG = CI::NG;
  R* G = sm;
  R* roots = sm + TC::G_ELEMS;
  for (int pass = 0; pass < TC::NPASS; ++pass) {
    R acc[TC::NK];
    int ixyz[TC::NK];
#pragma unroll
    for (int k = 0; k < TC::NK; ++k) {
      acc[k] = R(0);
      const int o = pass * TC::PASS + lane + k * TEAM;
      if (o < CI::NOUT) {
        const int id = o % CI::ND, ic = (o / CI::ND) % CI::NC;
        const int ib = (o / CI::NCD) % CI::NB, ia = o / (CI::NCD * CI::NB);
        const int jx = GI::idx(cart_lx(LA, ia), cart_lx(LB, ib), cart_lx(LC, ic), cart_lx(LD, id));
        const int jy = GI::idx(cart_ly(LA, ia), cart_ly(LB, ib), cart_ly(LC, ic), cart_ly(LD, id));
        const int jz = GI::idx(cart_lz(LA, ia), cart_lz(LB, ib), cart_lz(LC, ic), cart_lz(LD, id));
        ixyz[k] = jx | (jy << 10) | (jz << 20);
      } else {
        ixyz[k] = -1;
      }
    }
    for (int i = g.ppa; i < g.ppa + g.npa; ++i) {
      const double4 P = args.pp_data[i];
      const double2 PA = args.pp_aux[i];
      for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
        PrimQ<R> s;
        prim_setup<R>(g, P, PA, args.pp_data[j], args.pp_aux[j], s);
        for (int f = lane; f < 2 * N; f += TEAM) roots[f] = rys_one<N, R>(s.t, f, args.tb);
        __syncwarp(mask);
        for (int tsk = lane; tsk < 3 * N; tsk += TEAM) {
          const int r = tsk / 3, ax = tsk - 3 * r;
          RootCoef<R> rc;
          root_coef<R>(s, roots[r], rc);
          const R abd = ax == 0 ? R(g.abx) : (ax == 1 ? R(g.aby) : R(g.abz));
          const R cdd = ax == 0 ? R(g.cdx) : (ax == 1 ? R(g.cdy) : R(g.cdz));
          const R g00 = ax == 2 ? roots[N + r] * s.pref : R(1);
          build_g<LA, LB, LC, LD, R>(rc.c00[ax], rc.c0p[ax], rc.b10, rc.b01, rc.b00, g00, abd, cdd,
                                     G + (r * 3 + ax) * NG);
        }
        __syncwarp(mask);
#pragma unroll
        for (int k = 0; k < TC::NK; ++k) {
          if (ixyz[k] >= 0) {
            const int jx = ixyz[k] & 1023, jy = (ixyz[k] >> 10) & 1023, jz = ixyz[k] >> 20;
            R a = acc[k];
#pragma unroll
            for (int r = 0; r < N; ++r)
              a += G[(r * 3) * NG + jx] * G[(r * 3 + 1) * NG + jy] * G[(r * 3 + 2) * NG + jz];
            acc[k] = a;
          }
        }
        __syncwarp(mask);
      }
    }
    // stage this pass into V (double)
#pragma unroll
    for (int k = 0; k < TC::NK; ++k) {
      const int o = pass * TC::PASS + lane + k * TEAM;
      if (o < CI::NOUT) vsm[o] = double(acc[k]);
    }
    __syncwarp(mask);
  }
}

template <int LA, int LB, int LC, int LD, int TEAM>
__device__ __forceinline__ void team_digest(const JKArgs& args, const QuartetGeom& g,
                                            const double* V, int lane) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  constexpr int NA = CI::NA, NB = CI::NB, NC = CI::NC, ND = CI::ND;
  constexpr int T0 = NA * NB, T1 = T0 + NC * ND, T2 = T1 + NA * NC, T3 = T2 + NA * ND,
                T4 = T3 + NB * NC, T5 = T4 + NB * ND;
  const double s = g.scale;
  const long long base = args.mol_base[g.mol];
  const int n = args.mol_n[g.mol];
  for (int e = 0; e < args.ndm; ++e) {
    const double* dm = args.dens + e * args.dstride + base;
    const bool doj = args.with_j && e < args.nsym;
    double* vj = doj ? args.vj + e * args.dstride + base : nullptr;
    double* vk = args.vk + e * args.dstride + base;
    for (int t = lane; t < T5; t += TEAM) {
      double acc = 0.0;
      if (t < T1) {
        if (!doj) continue;
        if (t < T0) {
          const int a = t / NB, b = t % NB;
          for (int c = 0; c < NC; ++c)
            for (int d = 0; d < ND; ++d)
              acc += V[((a * NB + b) * NC + c) * ND + d] * dm[(long long)(g.aoC + c) * n + g.aoD + d];
          atomicAdd(vj + (long long)(g.aoA + a) * n + g.aoB + b, 2.0 * s * acc);
        } else {
          const int c = (t - T0) / ND, d = (t - T0) % ND;
          for (int a = 0; a < NA; ++a)
            for (int b = 0; b < NB; ++b)
              acc += V[((a * NB + b) * NC + c) * ND + d] * dm[(long long)(g.aoA + a) * n + g.aoB + b];
          atomicAdd(vj + (long long)(g.aoC + c) * n + g.aoD + d, 2.0 * s * acc);
        }
        continue;
      }
      if (!args.with_k) continue;
      if (t < T2) {
        const int a = (t - T1) / NC, c = (t - T1) % NC;
        for (int b = 0; b < NB; ++b)
          for (int d = 0; d < ND; ++d)
            acc += V[((a * NB + b) * NC + c) * ND + d] * dm[(long long)(g.aoB + b) * n + g.aoD + d];
        atomicAdd(vk + (long long)(g.aoA + a) * n + g.aoC + c, s * acc);
      } else if (t < T3) {
        const int a = (t - T2) / ND, d = (t - T2) % ND;
        for (int b = 0; b < NB; ++b)
          for (int c = 0; c < NC; ++c)
            acc += V[((a * NB + b) * NC + c) * ND + d] * dm[(long long)(g.aoB + b) * n + g.aoC + c];
        atomicAdd(vk + (long long)(g.aoA + a) * n + g.aoD + d, s * acc);
      } else if (t < T4) {
        const int b = (t - T3) / NC, c = (t - T3) % NC;
        for (int a = 0; a < NA; ++a)
          for (int d = 0; d < ND; ++d)
            acc += V[((a * NB + b) * NC + c) * ND + d] * dm[(long long)(g.aoA + a) * n + g.aoD + d];
        atomicAdd(vk + (long long)(g.aoB + b) * n + g.aoC + c, s * acc);
      } else {
        const int b = (t - T4) / ND, d = (t - T4) % ND;
        for (int a = 0; a < NA; ++a)
          for (int c = 0; c < NC; ++c)
            acc += V[((a * NB + b) * NC + c) * ND + d] * dm[(long long)(g.aoA + a) * n + g.aoC + c];
        atomicAdd(vk + (long long)(g.aoB + b) * n + g.aoD + d, s * acc);
      }
    }
  }
}

template <int LA, int LB, int LC, int LD, typename R, int TEAM>
struct TeamSmem {
  using TC = TeamCfg<LA, LB, LC, LD, TEAM>;
  // bytes per team: R-typed G/roots region, then (if not aliased) a double V region
  __host__ __device__ static constexpr size_t bytes() {
    return TC::NPASS == 1
               ? ((size_t)TC::GR * sizeof(R) > (size_t)ClassInfo<LA, LB, LC, LD>::NOUT * 8
                      ? (size_t)TC::GR * sizeof(R)
                      : (size_t)ClassInfo<LA, LB, LC, LD>::NOUT * 8)
               : (((size_t)TC::GR * sizeof(R) + 15) / 16) * 16 +
                     (size_t)ClassInfo<LA, LB, LC, LD>::NOUT * 8;
  }
  __host__ __device__ static constexpr size_t vofs() {
    return TC::NPASS == 1 ? 0 : (((size_t)TC::GR * sizeof(R) + 15) / 16) * 16;
  }
};

template <int LA, int LB, int LC, int LD, typename R, int TEAM>
__global__ void jk_team_kernel(JKArgs args) {
  using SM = TeamSmem<LA, LB, LC, LD, R, TEAM>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x % TEAM;
  const int team = threadIdx.x / TEAM;
  const int nteams = blockDim.x / TEAM;
  const unsigned mask =
      TEAM == 32 ? 0xffffffffu : (((1u << TEAM) - 1u) << ((threadIdx.x % 32) / TEAM * TEAM));
  unsigned char* mine = smem_raw + (size_t)team * SM::bytes();
  R* sm = reinterpret_cast<R*>(mine);
  double* vsm = reinterpret_cast<double*>(mine + SM::vofs());
  const int4 w = args.work[blockIdx.x];
  int kb, ke;
  ket_range(args, w, kb, ke);
  const BraRec br = load_bra(args, w.x);
  for (int k = kb + team; k < ke; k += nteams) {
    QuartetGeom g;
    load_quartet_rec(args, br, k, g);
    team_block<LA, LB, LC, LD, R, TEAM>(args, g, sm, vsm, lane, mask);
    team_digest<LA, LB, LC, LD, TEAM>(args, g, vsm, lane);
    __syncwarp(mask);
  }
}

// ---------------------------------------------------------------------------
// Tile path for mid-size classes (ket shells up to d): a team of NAB lanes
// per quartet, lane (a, b) owning one bra Cartesian pair and every ket pair
// (c, d) of the block, so each root costs it 3 (LC+1)(LD+1) shared reads for
// NC*ND outputs.  Kets of a work item share their primitive count and the
// bra is fixed, so all teams of a block run the primitive loop in lockstep
// (block barriers, no divergence).  Digestion stages the contracted block in
// shared memory and spreads the target elements over the team.
// ---------------------------------------------------------------------------
template <int LA, int LB, int LC, int LD, typename R>
struct TileCfg {
  using CI = ClassInfo<LA, LB, LC, LD>;
  static constexpr int TEAM = CI::NAB;
  static constexpr int Q = (128 / TEAM) > 0 ? (128 / TEAM) : 1;      // quartets per block
  static constexpr int THREADS = Q * TEAM;
  static constexpr int N = CI::NROOT;
  static constexpr int NG = CI::NG;
  static constexpr int KSTR = (LC + 1) * (LD + 1);                     // ket part of a G row
  // per quartet slot: G (3N*NG R), roots (2N R), staged block (NOUT double)
  static constexpr size_t G_BYTES = ((size_t)(3 * N * NG + 2 * N) * sizeof(R) + 15) / 16 * 16;
  static constexpr size_t SLOT = G_BYTES + (size_t)CI::NOUT * 8;
  static constexpr size_t bytes() { return SLOT * Q; }
};

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) jk_tile_kernel(JKArgs args) {
  using CI = ClassInfo<LA, LB, LC, LD>;
  using TC = TileCfg<LA, LB, LC, LD, R>;
  using GI = GIdx<LA, LB, LC, LD>;
  constexpr int N = TC::N, NG = TC::NG, TEAM = TC::TEAM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 w = args.work[blockIdx.x];
  int kb, ke;
  ket_range(args, w, kb, ke);
  if (kb >= ke) return;
  const int team = threadIdx.x / TEAM, lane = threadIdx.x % TEAM;
  R* G = reinterpret_cast<R*>(smem_raw + (size_t)team * TC::SLOT);
  R* roots = G + 3 * N * NG;
  double* V = reinterpret_cast<double*>(smem_raw + (size_t)team * TC::SLOT + TC::G_BYTES);
  const BraRec br = load_bra(args, w.x);
  // this lane's bra Cartesian pair
  const int ia = lane / CI::NB, ib = lane % CI::NB;
  const int bx = GI::idx(cart_lx(LA, ia), cart_lx(LB, ib), 0, 0);
  const int by = GI::idx(cart_ly(LA, ia), cart_ly(LB, ib), 0, 0);
  const int bz = GI::idx(cart_lz(LA, ia), cart_lz(LB, ib), 0, 0);
  for (int k0 = kb; k0 < ke; k0 += TC::Q) {
    const bool active = k0 + team < ke;
    QuartetGeom g;
    load_quartet_rec(args, br, active ? k0 + team : ke - 1, g);
    R acc[CI::NCD];
#pragma unroll
    for (int q = 0; q < CI::NCD; ++q) acc[q] = R(0);
    for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
      const double4 Qd = args.pp_data[j];
      const double2 QA = args.pp_aux[j];
      for (int i = g.ppa; i < g.ppa + g.npa; ++i) {
        PrimQ<R> s;
        prim_setup<R>(g, args.pp_data[i], args.pp_aux[i], Qd, QA, s);
        for (int f = lane; f < 2 * N; f += TEAM) roots[f] = rys_one<N, R>(s.t, f, args.tb);
        __syncthreads();
        for (int tsk = lane; tsk < 3 * N; tsk += TEAM) {
          const int r = tsk / 3, ax = tsk - 3 * r;
          RootCoef<R> rc;
          root_coef<R>(s, roots[r], rc);
          const R abd = ax == 0 ? R(g.abx) : (ax == 1 ? R(g.aby) : R(g.abz));
          const R cdd = ax == 0 ? R(g.cdx) : (ax == 1 ? R(g.cdy) : R(g.cdz));
          const R g00 = ax == 2 ? roots[N + r] * s.pref : R(1);
          build_g<LA, LB, LC, LD, R>(rc.c00[ax], rc.c0p[ax], rc.b10, rc.b01, rc.b00, g00, abd, cdd,
                                     G + (r * 3 + ax) * NG);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < N; ++r) {
          R vx[TC::KSTR], vy[TC::KSTR], vz[TC::KSTR];
          const R* gx = G + (r * 3) * NG + bx;
          const R* gy = G + (r * 3 + 1) * NG + by;
          const R* gz = G + (r * 3 + 2) * NG + bz;
#pragma unroll
          for (int q = 0; q < TC::KSTR; ++q) { vx[q] = gx[q]; vy[q] = gy[q]; vz[q] = gz[q]; }
          static_for<0, CI::NCD>([&](auto O) {
            constexpr int cd = decltype(O)::value;
            constexpr int ic = cd / CI::ND, id = cd % CI::ND;
            constexpr int jx = cart_lx(LC, ic) * (LD + 1) + cart_lx(LD, id);
            constexpr int jy = cart_ly(LC, ic) * (LD + 1) + cart_ly(LD, id);
            constexpr int jz = cart_lz(LC, ic) * (LD + 1) + cart_lz(LD, id);
            acc[cd] += vx[jx] * vy[jy] * vz[jz];
          });
        }
        __syncthreads();
      }
    }
#pragma unroll
    for (int q = 0; q < CI::NCD; ++q) V[lane * CI::NCD + q] = double(acc[q]);
    __syncthreads();
    if (active) team_digest<LA, LB, LC, LD, TEAM>(args, g, V, lane);
    __syncthreads();
  }
}

// Schwarz bound of one work pair: max over output-basis AO pairs (a,b) of
// |(ab|ab)| (csrc/coulomb_shells.h:60-77 uses the same diagonal), one team
// per pair.  c2s[l] holds the 10x7 output transform of shell l.
template <int LA, int LB, int TEAM>
__global__ void schwarz_kernel(JKArgs args, int npairs, int cart) {
  using SM = TeamSmem<LA, LB, LA, LB, double, TEAM>;
  using CI = ClassInfo<LA, LB, LA, LB>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x % TEAM;
  const int team = threadIdx.x / TEAM;
  const int nteams = blockDim.x / TEAM;
  const unsigned mask =
      TEAM == 32 ? 0xffffffffu : (((1u << TEAM) - 1u) << ((threadIdx.x % 32) / TEAM * TEAM));
  unsigned char* mine = smem_raw + (size_t)team * SM::bytes();
  double* sm = reinterpret_cast<double*>(mine);
  double* V = reinterpret_cast<double*>(mine + SM::vofs());
  const int pos = blockIdx.x * nteams + team;
  if (pos >= npairs) return;
  const int pair = args.bra_pairs[pos];
  QuartetGeom g;
  load_quartet(args, pair, pair, g);
  team_block<LA, LB, LA, LB, double, TEAM>(args, g, sm, V, lane, mask);
  const int nfa = cart ? CI::NA : 2 * LA + 1, nfb = cart ? CI::NB : 2 * LB + 1;
  const double* ta = args.tb.c2s + LA * kTS;
  const double* tb = args.tb.c2s + LB * kTS;
  double best = 0.0;
  for (int t = lane; t < nfa * nfb; t += TEAM) {
    const int fa = t / nfb, fb = t % nfb;
    double acc = 0.0;
    for (int a1 = 0; a1 < CI::NA; ++a1) {
      const double x1 = ta[a1 * kTW + fa];
      if (x1 == 0.0) continue;
      for (int b1 = 0; b1 < CI::NB; ++b1) {
        const double y1 = tb[b1 * kTW + fb];
        if (y1 == 0.0) continue;
        for (int a2 = 0; a2 < CI::NA; ++a2) {
          const double x2 = ta[a2 * kTW + fa];
          if (x2 == 0.0) continue;
          for (int b2 = 0; b2 < CI::NB; ++b2) {
            const double y2 = tb[b2 * kTW + fb];
            if (y2 == 0.0) continue;
            acc += x1 * y1 * x2 * y2 * V[((a1 * CI::NB + b1) * CI::NA + a2) * CI::NB + b2];
          }
        }
      }
    }
    best = fmax(best, fabs(acc));
  }
  for (int off = TEAM / 2; off > 0; off >>= 1) best = fmax(best, __shfl_down_sync(mask, best, off, TEAM));
  if (lane == 0) args.q_out[pair] = best;
}

}  // namespace b200jk

namespace b200jk {

// ---------------------------------------------------------------------------
// Packed ERI producer (the reference's packed_eri, csrc/packed_eri.cc): the
// team path's contracted Cartesian block of one quartet, transformed index
// by index to the output basis in shared memory and written to s4 (np x np)
// or s8 (np(np+1)/2 pairs of pairs) storage, np = n(n+1)/2, pair(i,j) =
// i(i+1)/2 + j for i >= j.  Every element of the block is written (equal
// values at symmetric positions), so the shell quartets of the canonical
// traversal cover the whole array.
// ---------------------------------------------------------------------------
// dst[..., f, ...] = sum_c src[..., c, ...] T[c][f] along `axis` of dims[4].
__device__ __forceinline__ void transform_axis(const double* src, double* dst, const int* dims, int axis,
                                               const double* T, int nf, int lane, int team) {
  int od[4] = {dims[0], dims[1], dims[2], dims[3]};
  od[axis] = nf;
  const int total = od[0] * od[1] * od[2] * od[3];
  int sstride = 1;
  for (int x = 3; x > axis; --x) sstride *= dims[x];
  for (int e = lane; e < total; e += team) {
    int r = e, idx[4];
    for (int x = 3; x >= 0; --x) {
      idx[x] = r % od[x];
      r /= od[x];
    }
    const int f = idx[axis];
    idx[axis] = 0;
    const int s0 = ((idx[0] * dims[1] + idx[1]) * dims[2] + idx[2]) * dims[3] + idx[3];
    double acc = 0.0;
    for (int c = 0; c < dims[axis]; ++c) {
      const double t = T[c * kTW + f];
      if (t != 0.0) acc += t * src[s0 + c * sstride];
    }
    dst[e] = acc;
  }
}

__device__ __forceinline__ long long pair_idx(long long i, long long j) {
  return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

template <int LA, int LB, int LC, int LD, int TEAM>
__global__ void eri_store_kernel(JKArgs args, int cart, int layout, double* __restrict__ out, long long npair) {
  using SM = TeamSmem<LA, LB, LC, LD, double, TEAM>;
  using CI = ClassInfo<LA, LB, LC, LD>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x % TEAM;
  const int team = threadIdx.x / TEAM;
  const int nteams = blockDim.x / TEAM;
  const unsigned mask =
      TEAM == 32 ? 0xffffffffu : (((1u << TEAM) - 1u) << ((threadIdx.x % 32) / TEAM * TEAM));
  const size_t per_team = SM::bytes() + (size_t)CI::NOUT * 8;
  unsigned char* mine = smem_raw + (size_t)team * per_team;
  double* sm = reinterpret_cast<double*>(mine);
  double* V = reinterpret_cast<double*>(mine + SM::vofs());
  double* W = reinterpret_cast<double*>(mine + SM::bytes());  // second buffer of NOUT doubles
  const int4 w = args.work[blockIdx.x];
  const int bra = args.bra_pairs[w.x];
  const int nf[4] = {cart ? CI::NA : 2 * LA + 1, cart ? CI::NB : 2 * LB + 1, cart ? CI::NC : 2 * LC + 1,
                     cart ? CI::ND : 2 * LD + 1};
  const double* T[4] = {args.tb.c2s + LA * kTS, args.tb.c2s + LB * kTS, args.tb.c2s + LC * kTS,
                        args.tb.c2s + LD * kTS};
  for (int k = w.y + team; k < w.z; k += nteams) {
    QuartetGeom g;
    load_quartet(args, bra, args.ket_pairs[k], g);
    team_block<LA, LB, LC, LD, double, TEAM>(args, g, sm, V, lane, mask);
    // V (Cartesian a,b,c,d) -> output basis, innermost index first
    int dims[4] = {CI::NA, CI::NB, CI::NC, CI::ND};
    double* src = V;
    double* dst = W;
    for (int axis = 3; axis >= 0; --axis) {
      transform_axis(src, dst, dims, axis, T[axis], nf[axis], lane, TEAM);
      __syncwarp(mask);
      dims[axis] = nf[axis];
      double* t = src;
      src = dst;
      dst = t;
    }
    const int o[4] = {args.sh_info[g.A].w, args.sh_info[g.B].w, args.sh_info[g.C].w, args.sh_info[g.D].w};
    const int total = nf[0] * nf[1] * nf[2] * nf[3];
    for (int e = lane; e < total; e += TEAM) {
      const int fd = e % nf[3], fc = (e / nf[3]) % nf[2], fb = (e / (nf[3] * nf[2])) % nf[1];
      const int fa = e / (nf[3] * nf[2] * nf[1]);
      const long long ab = pair_idx(o[0] + fa, o[1] + fb), cd = pair_idx(o[2] + fc, o[3] + fd);
      const double v = src[e];
      if (layout == 0) {
        out[ab * npair + cd] = v;
        out[cd * npair + ab] = v;
      } else {
        out[pair_idx(ab, cd)] = v;
      }
    }
    __syncwarp(mask);
  }
}

}  // namespace b200jk
