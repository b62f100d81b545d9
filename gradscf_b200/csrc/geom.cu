// Coordinate products of J/K beyond the gradient: the directional JVP of
// order 1 and 2 and the order-2 VJP (Hessian-vector product), replacing the
// reference's gradscf_direct_jk_geometry_{jvp_cpu_v1, vjp_cpu_v2} with order
// 1 and 2 (csrc/direct_jk_geometry.cc:8-99 over the entries of
// csrc/eri_geometry_entries.h:6-31 and csrc/geometry_contraction.h:7-53).
//
// With u, v coordinate directions (one 3-vector per atm row) and, for one
// canonical quartet with centres A, B, C, D, the translation-invariant
// reductions u~_P = u_P - u_D (P = A, B, C), the kernels evaluate
//   W1 = (u~ . d)(ab|cd),   W2 = (u~ . d)(v~ . d)(ab|cd)
// -- the first and second directional derivatives of the ERI block, which
// keep its eight-fold permutational symmetry, so the JVPs digest W1 / W2
// into J and K exactly as the J/K build digests (ab|cd) -- and, for the VJP,
//   T_{P,x} = sum_abcd Gamma_abcd d/dP_x (u~ . d)(ab|cd),  P = A, B, C,
//   T_{D,x} = -(T_{A,x} + T_{B,x} + T_{C,x}),
// Gamma the eight-permutation contraction of the cotangents with D (as in
// the gradient kernel).  Derivatives act on the 2D Rys integrals with the
// primitive exponents (d/dA_x phi_a = 2 alpha phi_{a+1} - a phi_{a-1}, twice
// for the second derivatives), computed from one table raised by two on A, B
// and C; nothing is stored.
//
// One generic kernel for every class (runtime angular momenta): a warp per
// quartet, the 2D tables of one root at a time in shared memory (three
// lanes build the x, y, z tables), every lane accumulating a strided slice
// of the Cartesian block in registers, in passes of 32 x kGeoNK elements.
// These products serve vibrational analysis, not the SCF loop: the kernel
// favours one code path for all classes over per-class tuning.
#include <cuda_runtime.h>

#include "grad_kernels.cuh"
#include "plan.h"

namespace b200jk {

namespace {

constexpr int kGeoWarps = 4;
constexpr int kGeoNK = 8;   // elements per lane per pass

struct GeoShape {
  int la, lb, lc, ld;
  int na, nb, nc, nd, nout;
  int a2, b2, c2, d1;      // raised table extents: la+3, lb+3, lc+3, ld+1
  int lab, lcd;            // la+lb+4, lc+ld+2 (VRR extents of the raised table)
  int ng;                  // table size per (root, axis)
  int nw;                  // HRR scratch per (root, axis): (lab+1)(lcd+1)(ld+1)
  int nroot;
};

__host__ __device__ inline GeoShape geo_shape(int la, int lb, int lc, int ld) {
  GeoShape s;
  s.la = la; s.lb = lb; s.lc = lc; s.ld = ld;
  s.na = ncart(la); s.nb = ncart(lb); s.nc = ncart(lc); s.nd = ncart(ld);
  s.nout = s.na * s.nb * s.nc * s.nd;
  s.a2 = la + 3; s.b2 = lb + 3; s.c2 = lc + 3; s.d1 = ld + 1;
  s.lab = la + lb + 4; s.lcd = lc + ld + 2;
  s.ng = s.a2 * s.b2 * s.c2 * s.d1;
  s.nw = (s.lab + 1) * (s.lcd + 1) * s.d1;
  s.nroot = (la + lb + lc + ld + 2) / 2 + 1;
  return s;
}

// doubles of shared memory per warp: roots/weights, three tables, three scratch areas
__host__ __device__ inline int geo_warp_doubles(const GeoShape& s) { return 16 + 3 * s.ng + 3 * s.nw; }

__device__ __forceinline__ double rys_one_rt(int n, double t, int f, const Tables& tb) {
  switch (n) {
    case 1: return rys_one<1, double>(t, f, tb);
    case 2: return rys_one<2, double>(t, f, tb);
    case 3: return rys_one<3, double>(t, f, tb);
    case 4: return rys_one<4, double>(t, f, tb);
    case 5: return rys_one<5, double>(t, f, tb);
    case 6: return rys_one<6, double>(t, f, tb);
    case 7: return rys_one<7, double>(t, f, tb);
    default: return rys_one<8, double>(t, f, tb);
  }
}

// The raised 2D table of one (root, axis): the VRR and horizontal transfers
// of build_g with runtime extents, G[((a*b2 + b)*c2 + c)*d1 + d] for
// a < a2, b < b2, c < c2, d < d1.  `w` is scratch of s.nw doubles.
__device__ void build_g_rt(const GeoShape& s, double c00, double c0p, double b10, double b01, double b00,
                           double g00, double ab, double cd, double* G, double* w) {
  const int LAB = s.lab, LCD = s.lcd, LD = s.ld;
  auto W = [&](int e, int c, int d) -> double& { return w[(e * (LCD + 1) + c) * (LD + 1) + d]; };
  // VRR into W[e][f][0]
  W(0, 0, 0) = g00;
  if (LAB > 0) W(1, 0, 0) = c00 * g00;
  for (int e = 1; e < LAB; ++e) W(e + 1, 0, 0) = c00 * W(e, 0, 0) + e * b10 * W(e - 1, 0, 0);
  for (int f = 0; f < LCD; ++f)
    for (int e = 0; e <= LAB; ++e) {
      double val = c0p * W(e, f, 0);
      if (f > 0) val += f * b01 * W(e, f - 1, 0);
      if (e > 0) val += e * b00 * W(e - 1, f, 0);
      W(e, f + 1, 0) = val;
    }
  // ket transfer
  for (int e = 0; e <= LAB; ++e)
    for (int d = 1; d <= LD; ++d)
      for (int c = 0; c <= LCD - d; ++c) W(e, c, d) = W(e, c + 1, d - 1) + cd * W(e, c, d - 1);
  // bra transfer per (c, d): y_b[a] over a = 0..LAB-b, y_{b+1}[a] = y_b[a+1] + ab y_b[a]
  for (int c = 0; c < s.c2; ++c)
    for (int d = 0; d < s.d1; ++d) {
      double y[16];
      for (int e = 0; e <= LAB; ++e) y[e] = W(e, c, d);
      for (int b = 0; b < s.b2; ++b) {
        for (int a = 0; a < s.a2; ++a) G[((a * s.b2 + b) * s.c2 + c) * s.d1 + d] = y[a];
        if (b + 1 < s.b2)
          for (int a = 0; a + b + 1 <= LAB; ++a) y[a] = y[a + 1] + ab * y[a];
      }
    }
}

struct AxisDer {
  double i, dA, dB, dC, dAA, dBB, dCC, dAB, dAC, dBC;
};

// Derivatives along one axis of the 2D integral with exponents (a, b, c, d):
// d/dP (P = A, B, C) and the second derivatives, from the raised table.
__device__ __forceinline__ AxisDer axis_der(const GeoShape& s, const double* G, int a, int b, int c, int d,
                                            double al, double be, double ga, bool second) {
  auto at = [&](int x, int y, int z) { return G[((x * s.b2 + y) * s.c2 + z) * s.d1 + d]; };
  AxisDer r;
  r.i = at(a, b, c);
  const double am = a ? a * at(a - 1, b, c) : 0.0, bm = b ? b * at(a, b - 1, c) : 0.0,
               cm = c ? c * at(a, b, c - 1) : 0.0;
  r.dA = 2.0 * al * at(a + 1, b, c) - am;
  r.dB = 2.0 * be * at(a, b + 1, c) - bm;
  r.dC = 2.0 * ga * at(a, b, c + 1) - cm;
  if (!second) return r;
  r.dAA = 4.0 * al * al * at(a + 2, b, c) - 2.0 * al * (2 * a + 1) * r.i + (a > 1 ? a * (a - 1) * at(a - 2, b, c) : 0.0);
  r.dBB = 4.0 * be * be * at(a, b + 2, c) - 2.0 * be * (2 * b + 1) * r.i + (b > 1 ? b * (b - 1) * at(a, b - 2, c) : 0.0);
  r.dCC = 4.0 * ga * ga * at(a, b, c + 2) - 2.0 * ga * (2 * c + 1) * r.i + (c > 1 ? c * (c - 1) * at(a, b, c - 2) : 0.0);
  // mixed: (2x f(+1) - n f(-1)) on two indices
  auto mix = [&](int p1, int q1) {
    // p1, q1 select the two indices: 0 = a, 1 = b, 2 = c
    const int e[3] = {a, b, c};
    const double ex[3] = {al, be, ga};
    double acc = 0.0;
    for (int sp = 0; sp < 2; ++sp)
      for (int sq = 0; sq < 2; ++sq) {
        int idx[3] = {a, b, c};
        double f;
        if (sp == 0) { idx[p1] += 1; f = 2.0 * ex[p1]; } else { if (!e[p1]) continue; idx[p1] -= 1; f = -e[p1]; }
        if (sq == 0) { idx[q1] += 1; f *= 2.0 * ex[q1]; } else { if (!e[q1]) continue; idx[q1] -= 1; f *= -e[q1]; }
        acc += f * at(idx[0], idx[1], idx[2]);
      }
    return acc;
  };
  r.dAB = mix(0, 1);
  r.dAC = mix(0, 2);
  r.dBC = mix(1, 2);
  return r;
}

// Directional combinations along one axis: U = sum_P u_P dP, UV = sum_PQ u_P v_Q dPQ,
// and dP U = sum_Q u_Q dPQ.
__device__ __forceinline__ double dirv(const AxisDer& r, const double* u) {
  return u[0] * r.dA + u[1] * r.dB + u[2] * r.dC;
}
__device__ __forceinline__ double dir2(const AxisDer& r, const double* u, const double* v) {
  return u[0] * v[0] * r.dAA + u[1] * v[1] * r.dBB + u[2] * v[2] * r.dCC +
         (u[0] * v[1] + u[1] * v[0]) * r.dAB + (u[0] * v[2] + u[2] * v[0]) * r.dAC +
         (u[1] * v[2] + u[2] * v[1]) * r.dBC;
}
__device__ __forceinline__ void dP_dir(const AxisDer& r, const double* u, double* out) {
  out[0] = u[0] * r.dAA + u[1] * r.dAB + u[2] * r.dAC;
  out[1] = u[0] * r.dAB + u[1] * r.dBB + u[2] * r.dBC;
  out[2] = u[0] * r.dAC + u[1] * r.dBC + u[2] * r.dCC;
}

}  // namespace

// mode 0: JVP order 1, 1: JVP order 2, 2: VJP order 2.
// JKArgs: dens (raw Cartesian D), vj/vk accumulators (JVP), cot_j/cot_k +
// gnb (VJP), grad (VJP output), geo_u / geo_v (atm rows x 3).
__global__ void __launch_bounds__(32 * kGeoWarps) geom_team_kernel(JKArgs args, int la, int lb, int lc, int ld,
                                                                   int mode) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const GeoShape S = geo_shape(la, lb, lc, ld);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* base = reinterpret_cast<double*>(smem_raw) + (size_t)warp * geo_warp_doubles(S);
  double* roots = base;
  double* G = base + 16;
  double* Wsc = G + 3 * S.ng;
  const int4 w = args.work[blockIdx.x];
  const int bra = args.bra_pairs[w.x];
  const bool second = mode != 0;
  for (int k = w.y + warp; k < w.z; k += kGeoWarps) {
    QuartetGeom g;
    load_quartet(args, bra, args.ket_pairs[k], g);
    const long long mbase = args.mol_base[g.mol];
    const int n = args.mol_n[g.mol];
    const int atA = args.ws_atm[g.A], atB = args.ws_atm[g.B], atC = args.ws_atm[g.C], atD = args.ws_atm[g.D];
    // reduced directions per axis: ut[axis][P], P = A, B, C
    double ut[3][3], vt[3][3];
    for (int x = 0; x < 3; ++x) {
      const double uD = args.geo_u[3 * atD + x];
      ut[x][0] = args.geo_u[3 * atA + x] - uD;
      ut[x][1] = args.geo_u[3 * atB + x] - uD;
      ut[x][2] = args.geo_u[3 * atC + x] - uD;
      if (mode == 1) {
        const double vD = args.geo_v[3 * atD + x];
        vt[x][0] = args.geo_v[3 * atA + x] - vD;
        vt[x][1] = args.geo_v[3 * atB + x] - vD;
        vt[x][2] = args.geo_v[3 * atC + x] - vD;
      } else {
        vt[x][0] = vt[x][1] = vt[x][2] = 0.0;
      }
    }
    double T[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // VJP: [P][axis]
    for (int p0 = 0; p0 < S.nout; p0 += 32 * kGeoNK) {
      double acc[kGeoNK], gam[kGeoNK];
      int el[kGeoNK];
#pragma unroll
      for (int q = 0; q < kGeoNK; ++q) {
        const int o = p0 + lane + 32 * q;
        acc[q] = 0.0;
        gam[q] = 0.0;
        el[q] = o < S.nout ? o : -1;
        if (mode == 2 && o < S.nout) {
          const int id = o % S.nd, ic = (o / S.nd) % S.nc, ib = (o / (S.nd * S.nc)) % S.nb,
                    ia = o / (S.nd * S.nc * S.nb);
          gam[q] = g.scale * gamma_abcd(args, mbase, n, g.aoA + ia, g.aoB + ib, g.aoC + ic, g.aoD + id);
        }
      }
      for (int i = g.ppa; i < g.ppa + g.npa; ++i) {
        const double4 P = args.pp_data[i];
        const double2 PA = args.pp_aux[i];
        const double al = args.pp_exp[i].x, be = args.pp_exp[i].y;
        for (int j = g.ppc; j < g.ppc + g.npc; ++j) {
          PrimQ<double> s;
          prim_setup<double>(g, P, PA, args.pp_data[j], args.pp_aux[j], s);
          const double ga = args.pp_exp[j].x;
          if (lane < 2 * S.nroot) roots[lane] = rys_one_rt(S.nroot, s.t, lane, args.tb);
          __syncwarp();
          for (int r = 0; r < S.nroot; ++r) {
            if (lane < 3) {
              RootCoef<double> rc;
              root_coef<double>(s, roots[r], rc);
              const double abd = lane == 0 ? g.abx : (lane == 1 ? g.aby : g.abz);
              const double cdd = lane == 0 ? g.cdx : (lane == 1 ? g.cdy : g.cdz);
              const double g00 = lane == 2 ? roots[S.nroot + r] * s.pref : 1.0;
              build_g_rt(S, rc.c00[lane], rc.c0p[lane], rc.b10, rc.b01, rc.b00, g00, abd, cdd, G + lane * S.ng,
                         Wsc + lane * S.nw);
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < kGeoNK; ++q) {
              const int o = el[q];
              if (o < 0 || (mode == 2 && gam[q] == 0.0)) continue;
              const int id = o % S.nd, ic = (o / S.nd) % S.nc, ib = (o / (S.nd * S.nc)) % S.nb,
                        ia = o / (S.nd * S.nc * S.nb);
              AxisDer ax[3];
              const int exa[3] = {cart_lx(la, ia), cart_ly(la, ia), cart_lz(la, ia)};
              const int exb[3] = {cart_lx(lb, ib), cart_ly(lb, ib), cart_lz(lb, ib)};
              const int exc[3] = {cart_lx(lc, ic), cart_ly(lc, ic), cart_lz(lc, ic)};
              const int exd[3] = {cart_lx(ld, id), cart_ly(ld, id), cart_lz(ld, id)};
              for (int x = 0; x < 3; ++x)
                ax[x] = axis_der(S, G + x * S.ng, exa[x], exb[x], exc[x], exd[x], al, be, ga, second);
              if (mode == 0) {
                acc[q] += dirv(ax[0], ut[0]) * ax[1].i * ax[2].i + ax[0].i * dirv(ax[1], ut[1]) * ax[2].i +
                          ax[0].i * ax[1].i * dirv(ax[2], ut[2]);
              } else if (mode == 1) {
                double U[3], V[3], UV[3];
                for (int x = 0; x < 3; ++x) {
                  U[x] = dirv(ax[x], ut[x]);
                  V[x] = dirv(ax[x], vt[x]);
                  UV[x] = dir2(ax[x], ut[x], vt[x]);
                }
                const double I0 = ax[0].i, I1 = ax[1].i, I2 = ax[2].i;
                acc[q] += UV[0] * I1 * I2 + I0 * UV[1] * I2 + I0 * I1 * UV[2] + (U[0] * V[1] + V[0] * U[1]) * I2 +
                          (U[0] * V[2] + V[0] * U[2]) * I1 + (U[1] * V[2] + V[1] * U[2]) * I0;
              } else {
                // d/dP_x (u~ . d): the x factor takes dP, the others their plain / directional value
                double U[3], dPU[3][3];
                for (int x = 0; x < 3; ++x) {
                  U[x] = dirv(ax[x], ut[x]);
                  dP_dir(ax[x], ut[x], dPU[x]);
                }
                const double gq = gam[q];
                for (int x = 0; x < 3; ++x) {
                  const int y = (x + 1) % 3, z = (x + 2) % 3;
                  const double rest = U[y] * ax[z].i + ax[y].i * U[z];
                  const double plain = ax[y].i * ax[z].i;
                  const double dP[3] = {ax[x].dA, ax[x].dB, ax[x].dC};
                  for (int P = 0; P < 3; ++P) T[P][x] += gq * (dPU[x][P] * plain + dP[P] * rest);
                }
              }
            }
            __syncwarp();
          }
        }
      }
      if (mode != 2) {
        // digest this pass's elements: the derivative block has the ERI's
        // permutational symmetry, so it enters J/K as (ab|cd) does
        const double sc = g.scale;
        for (int q = 0; q < kGeoNK; ++q) {
          const int o = el[q];
          if (o < 0) continue;
          const int id = o % S.nd, ic = (o / S.nd) % S.nc, ib = (o / (S.nd * S.nc)) % S.nb,
                    ia = o / (S.nd * S.nc * S.nb);
          const int a = g.aoA + ia, b = g.aoB + ib, c = g.aoC + ic, d = g.aoD + id;
          const double v = acc[q];
          for (int e = 0; e < args.ndm; ++e) {
            const double* dm = args.dens + e * args.dstride + mbase;
            if (args.with_j && e < args.nsym) {
              double* vj = args.vj + e * args.dstride + mbase;
              atomicAdd(vj + (long long)a * n + b, 2.0 * sc * v * dm[(long long)c * n + d]);
              atomicAdd(vj + (long long)c * n + d, 2.0 * sc * v * dm[(long long)a * n + b]);
            }
            if (args.with_k) {
              double* vk = args.vk + e * args.dstride + mbase;
              atomicAdd(vk + (long long)a * n + c, sc * v * dm[(long long)b * n + d]);
              atomicAdd(vk + (long long)a * n + d, sc * v * dm[(long long)b * n + c]);
              atomicAdd(vk + (long long)b * n + c, sc * v * dm[(long long)a * n + d]);
              atomicAdd(vk + (long long)b * n + d, sc * v * dm[(long long)a * n + c]);
            }
          }
        }
      }
    }
    if (mode == 2) {
      for (int P = 0; P < 3; ++P)
        for (int x = 0; x < 3; ++x)
          for (int off = 16; off > 0; off >>= 1) T[P][x] += __shfl_down_sync(0xffffffffu, T[P][x], off);
      if (lane == 0) {
        for (int x = 0; x < 3; ++x) {
          atomicAdd(args.grad + 3LL * atA + x, T[0][x]);
          atomicAdd(args.grad + 3LL * atB + x, T[1][x]);
          atomicAdd(args.grad + 3LL * atC + x, T[2][x]);
          atomicAdd(args.grad + 3LL * atD + x, -(T[0][x] + T[1][x] + T[2][x]));
        }
      }
    }
  }
}

// Shared memory of one launch for class (la, lb | lc, ld), or 0 if it does not fit.
size_t geom_smem_bytes(int la, int lb, int lc, int ld) {
  const GeoShape s = geo_shape(la, lb, lc, ld);
  const size_t bytes = (size_t)geo_warp_doubles(s) * 8 * kGeoWarps;
  return bytes <= 227 * 1024 ? bytes : 0;
}

int launch_geom(const JKArgs& args, int la, int lb, int lc, int ld, int mode, cudaStream_t st) {
  if (args.nwork <= 0) return 0;
  const size_t smem = geom_smem_bytes(la, lb, lc, ld);
  if (!smem) return (int)cudaErrorInvalidConfiguration;
  static std::atomic<uint64_t> smem_done{0};
  // the largest class sets the attribute once per device
  smem_opt_in(geom_team_kernel, 227 * 1024, smem_done);
  geom_team_kernel<<<args.nwork, 32 * kGeoWarps, smem, st>>>(args, la, lb, lc, ld, mode);
  return (int)cudaGetLastError();
}

}  // namespace b200jk
