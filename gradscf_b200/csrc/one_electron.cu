// One-electron integrals (overlap, kinetic, nuclear attraction) and the
// one-electron part of the RHF nuclear gradient, on the plan's shells.
//
// Overlap and kinetic use the Obara-Saika 1D recursions
//   S(i+1,j) = PA S(i,j) + [i S(i-1,j) + j S(i,j-1)] / 2p
//   S(i,j+1) = PB S(i,j) + [i S(i-1,j) + j S(i,j-1)] / 2p
//   K(i,j)   = -1/2 [ j(j-1) S(i,j-2) - 2b(2j+1) S(i,j) + 4b^2 S(i,j+2) ]
// with the product prefactor (pi/p)^(3/2) exp(-ab/p |AB|^2).  Nuclear
// attraction uses Rys quadrature with the same roots as the ERIs:
//   (a| 1/|r-C| |b) = 2 pi/p K_ab sum_r w_r Ix Iy Iz,  T = p |PC|^2,
//   I(i+1,0) = (PA - u PC) I(i,0) + i (1-u)/(2p) I(i-1,0),
//   I(i,j+1) = I(i+1,j) + AB I(i,j).
// Centre derivatives: d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x};
// the operator derivative of the nuclear attraction follows from
// translational invariance, dC = -(dA + dB).
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/b200jk.h"
#include "common.cuh"
#include "dispatch.h"
#include "plan.h"
#include "one_electron.h"

namespace b200jk {


template <int IMAX, int JMAX>
__device__ __forceinline__ void os_overlap(double pa, double pb, double i2p, double (&s)[IMAX + 1][JMAX + 1]) {
  s[0][0] = 1.0;
#pragma unroll
  for (int i = 0; i < IMAX; ++i) s[i + 1][0] = pa * s[i][0] + (i > 0 ? i * i2p * s[i - 1][0] : 0.0);
#pragma unroll
  for (int j = 0; j < JMAX; ++j)
#pragma unroll
    for (int i = 0; i <= IMAX; ++i) {
      double v = pb * s[i][j];
      if (i > 0) v += i * i2p * s[i - 1][j];
      if (j > 0) v += j * i2p * s[i][j - 1];
      s[i][j + 1] = v;
    }
}

// Kinetic 1D integral <i| -1/2 d^2/dx^2 |j> from the overlap table (needs j+2).
template <int IMAX, int JMAX>
__device__ __forceinline__ double os_kin(const double (&s)[IMAX + 1][JMAX + 1], int i, int j, double b) {
  double v = -2.0 * b * (2 * j + 1) * s[i][j] + 4.0 * b * b * s[i][j + 2];
  if (j >= 2) v += j * (j - 1) * s[i][j - 2];
  return -0.5 * v;
}

// 1D nuclear-attraction tables for one root: I(i, j), i <= IMAX, j <= JMAX.
template <int IMAX, int JMAX>
__device__ __forceinline__ void rys_1e(double c00, double b10, double ab, double (&g)[IMAX + 1][JMAX + 1]) {
  double v[IMAX + JMAX + 1];
  v[0] = 1.0;
#pragma unroll
  for (int e = 0; e < IMAX + JMAX; ++e) v[e + 1] = c00 * v[e] + (e > 0 ? e * b10 * v[e - 1] : 0.0);
  double y[IMAX + JMAX + 1][JMAX + 1];
#pragma unroll
  for (int e = 0; e <= IMAX + JMAX; ++e) y[e][0] = v[e];
#pragma unroll
  for (int j = 1; j <= JMAX; ++j)
#pragma unroll
    for (int e = 0; e <= IMAX + JMAX - j; ++e) y[e][j] = y[e + 1][j - 1] + ab * y[e][j - 1];
#pragma unroll
  for (int i = 0; i <= IMAX; ++i)
#pragma unroll
    for (int j = 0; j <= JMAX; ++j) g[i][j] = y[i][j];
}

// 1D centre derivatives along one axis: overlap (sp) and kinetic (kp) for
// d/dA of the bra index la, and (sq, kq) for d/dB of the ket index lb.
template <int IMAX, int JMAX>
__device__ __forceinline__ void axis_deriv(const double (&t)[IMAX + 1][JMAX + 1], int la, int lb, double al,
                                           double be, double& sp, double& kp, double& sq, double& kq) {
  sp = 2 * al * t[la + 1][lb] - (la ? la * t[la - 1][lb] : 0.0);
  kp = 2 * al * os_kin<IMAX, JMAX>(t, la + 1, lb, be) - (la ? la * os_kin<IMAX, JMAX>(t, la - 1, lb, be) : 0.0);
  sq = 2 * be * t[la][lb + 1] - (lb ? lb * t[la][lb - 1] : 0.0);
  kq = 2 * be * os_kin<IMAX, JMAX>(t, la, lb + 1, be) - (lb ? lb * os_kin<IMAX, JMAX>(t, la, lb - 1, be) : 0.0);
}

// Value kernel: one thread per (pair, bra Cartesian component).  DERIV
// selects the gradient contraction instead of the matrix output.
template <int LA, int LB, bool DERIV>
__global__ void one_electron_kernel(OneArgs args) {
  constexpr int NA = ncart(LA), NB = ncart(LB);
  constexpr int D = DERIV ? 1 : 0;
  constexpr int IM = LA + D, JM = LB + D;            // angular range needed
  constexpr int NR = (IM + JM) / 2 + 1;              // Rys roots for V
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int pidx = gid / NA, ia = gid % NA;
  if (pidx >= args.npairs) return;
  const int4 pr = args.pair_info[args.pairs[pidx]];
  const int A = pr.x, B = pr.y;
  const int4 sa = args.ws_info[A], sb = args.ws_info[B];
  const double4 ra = args.ws_xyz[A], rb = args.ws_xyz[B];
  const double abx = ra.x - rb.x, aby = ra.y - rb.y, abz = ra.z - rb.z;
  const double ab2 = abx * abx + aby * aby + abz * abz;
  int lxa = 0, lya = 0, lza = 0;
#pragma unroll
  for (int i = 0; i < NA; ++i)
    if (i == ia) { lxa = cart_lx(LA, i); lya = cart_ly(LA, i); lza = cart_lz(LA, i); }
  const int mol = sa.z;
  const int atm0 = args.mol_atm_off[mol], natm = args.mol_natm[mol];
  const int n = args.mol_n[mol];
  const long long base = args.mol_base[mol];
  double s_out[NB], t_out[NB], v_out[NB];
#pragma unroll
  for (int j = 0; j < NB; ++j) s_out[j] = t_out[j] = v_out[j] = 0.0;
  // gradient accumulators: d/dA and d/dB (3 each)
  double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
  double dmr[NB], wmr[NB];
  const double fac = (A == B) ? 1.0 : 2.0;   // (a,b) and (b,a) for distinct shells
  if (DERIV) {
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const long long idx = base + (long long)(sa.x + ia) * n + sb.x + j;
      dmr[j] = fac * args.dm[idx];
      wmr[j] = fac * args.wm[idx];
    }
  }
  for (int ip = args.prim_off[A]; ip < args.prim_off[A + 1]; ++ip) {
    const double2 pa_ = args.prim[ip];
    for (int jp = args.prim_off[B]; jp < args.prim_off[B + 1]; ++jp) {
      const double2 pb_ = args.prim[jp];
      const double al = pa_.x, be = pb_.x;
      const double p = al + be, ip2 = 0.5 / p;
      const double kab = exp(-al * be / p * ab2) * pa_.y * pb_.y;
      if (kab == 0.0) continue;
      const double Px = (al * ra.x + be * rb.x) / p, Py = (al * ra.y + be * rb.y) / p,
                   Pz = (al * ra.z + be * rb.z) / p;
      const double pre_s = kab * B200JK_PI / p * sqrt(B200JK_PI / p);
      // overlap / kinetic tables (j up to JM + 2 for the kinetic operator)
      double sx[IM + 1][JM + 3], sy[IM + 1][JM + 3], sz[IM + 1][JM + 3];
      os_overlap<IM, JM + 2>(Px - ra.x, Px - rb.x, ip2, sx);
      os_overlap<IM, JM + 2>(Py - ra.y, Py - rb.y, ip2, sy);
      os_overlap<IM, JM + 2>(Pz - ra.z, Pz - rb.z, ip2, sz);
      // nuclear attraction: 1D tables per nucleus and root
      for (int c = 0; c < natm; ++c) {
        const double4 C = args.atoms[atm0 + c];
        if (C.w == 0.0) continue;
        const double pcx = Px - C.x, pcy = Py - C.y, pcz = Pz - C.z;
        const double tt = p * (pcx * pcx + pcy * pcy + pcz * pcz);
        double x[NR], w[NR];
        rys_roots<NR, double>(tt, x, w, args.tb);
        const double pre_v = -C.w * 2.0 * B200JK_PI / p * kab;
        double gC[3] = {0, 0, 0};
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const double u = x[r];
          const double b10 = (1.0 - u) * ip2;
          double ix[IM + 1][JM + 1], iy[IM + 1][JM + 1], iz[IM + 1][JM + 1];
          rys_1e<IM, JM>(Px - ra.x - u * pcx, b10, abx, ix);
          rys_1e<IM, JM>(Py - ra.y - u * pcy, b10, aby, iy);
          rys_1e<IM, JM>(Pz - ra.z - u * pcz, b10, abz, iz);
          const double wr = w[r] * pre_v;
#pragma unroll
          for (int jb = 0; jb < NB; ++jb) {
            const int bx = cart_lx(LB, jb), by = cart_ly(LB, jb), bz = cart_lz(LB, jb);
            if (!DERIV) {
              v_out[jb] += wr * ix[lxa][bx] * iy[lya][by] * iz[lza][bz];
            } else {
              // d/dA and d/dB of (a|V_C|b); dC = -(dA + dB)
              const double dx = dmr[jb] * wr;
              const double ga0 = 2 * al * ix[lxa + 1][bx] * iy[lya][by] * iz[lza][bz] -
                                 (lxa ? lxa * ix[lxa - 1][bx] * iy[lya][by] * iz[lza][bz] : 0.0);
              const double ga1 = 2 * al * ix[lxa][bx] * iy[lya + 1][by] * iz[lza][bz] -
                                 (lya ? lya * ix[lxa][bx] * iy[lya - 1][by] * iz[lza][bz] : 0.0);
              const double ga2 = 2 * al * ix[lxa][bx] * iy[lya][by] * iz[lza + 1][bz] -
                                 (lza ? lza * ix[lxa][bx] * iy[lya][by] * iz[lza - 1][bz] : 0.0);
              const double gb0 = 2 * be * ix[lxa][bx + 1] * iy[lya][by] * iz[lza][bz] -
                                 (bx ? bx * ix[lxa][bx - 1] * iy[lya][by] * iz[lza][bz] : 0.0);
              const double gb1 = 2 * be * ix[lxa][bx] * iy[lya][by + 1] * iz[lza][bz] -
                                 (by ? by * ix[lxa][bx] * iy[lya][by - 1] * iz[lza][bz] : 0.0);
              const double gb2 = 2 * be * ix[lxa][bx] * iy[lya][by] * iz[lza][bz + 1] -
                                 (bz ? bz * ix[lxa][bx] * iy[lya][by] * iz[lza][bz - 1] : 0.0);
              gA[0] += dx * ga0; gA[1] += dx * ga1; gA[2] += dx * ga2;
              gB[0] += dx * gb0; gB[1] += dx * gb1; gB[2] += dx * gb2;
              gC[0] -= dx * (ga0 + gb0); gC[1] -= dx * (ga1 + gb1); gC[2] -= dx * (ga2 + gb2);
            }
          }
        }
        if (DERIV) {
          double* g = args.grad + (long long)(atm0 + c) * 3;
          atomicAdd(g, gC[0]); atomicAdd(g + 1, gC[1]); atomicAdd(g + 2, gC[2]);
        }
      }
#pragma unroll
      for (int jb = 0; jb < NB; ++jb) {
        const int bx = cart_lx(LB, jb), by = cart_ly(LB, jb), bz = cart_lz(LB, jb);
        if (!DERIV) {
          s_out[jb] += pre_s * sx[lxa][bx] * sy[lya][by] * sz[lza][bz];
          t_out[jb] += pre_s * (os_kin<IM, JM + 2>(sx, lxa, bx, be) * sy[lya][by] * sz[lza][bz] +
                                sx[lxa][bx] * os_kin<IM, JM + 2>(sy, lya, by, be) * sz[lza][bz] +
                                sx[lxa][bx] * sy[lya][by] * os_kin<IM, JM + 2>(sz, lza, bz, be));
        } else {
          // overlap derivative (weighted by W) and kinetic derivative (weighted by D)
          const double s0 = sx[lxa][bx], s1 = sy[lya][by], s2 = sz[lza][bz];
          const double t0 = os_kin<IM, JM + 2>(sx, lxa, bx, be);
          const double t1 = os_kin<IM, JM + 2>(sy, lya, by, be);
          const double t2 = os_kin<IM, JM + 2>(sz, lza, bz, be);
          double spa[3], kpa[3], spb[3], kpb[3];
          axis_deriv<IM, JM + 2>(sx, lxa, bx, al, be, spa[0], kpa[0], spb[0], kpb[0]);
          axis_deriv<IM, JM + 2>(sy, lya, by, al, be, spa[1], kpa[1], spb[1], kpb[1]);
          axis_deriv<IM, JM + 2>(sz, lza, bz, al, be, spa[2], kpa[2], spb[2], kpb[2]);
          const double so[3] = {s1 * s2, s0 * s2, s0 * s1};          // other-axis overlaps
          const double to[3] = {t1 * s2 + s1 * t2, t0 * s2 + s0 * t2, t0 * s1 + s0 * t1};
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            gA[k] += pre_s * (dmr[jb] * (kpa[k] * so[k] + spa[k] * to[k]) - wmr[jb] * spa[k] * so[k]);
            gB[k] += pre_s * (dmr[jb] * (kpb[k] * so[k] + spb[k] * to[k]) - wmr[jb] * spb[k] * so[k]);
          }
        }
      }
    }
  }
  if (!DERIV) {
#pragma unroll
    for (int jb = 0; jb < NB; ++jb) {
      const long long ab = base + (long long)(sa.x + ia) * n + sb.x + jb;
      const long long ba = base + (long long)(sb.x + jb) * n + sa.x + ia;
      args.out_s[ab] = s_out[jb]; args.out_t[ab] = t_out[jb]; args.out_v[ab] = v_out[jb];
      args.out_s[ba] = s_out[jb]; args.out_t[ba] = t_out[jb]; args.out_v[ba] = v_out[jb];
    }
  } else {
    double* ga = args.grad + (long long)args.ws_atm[A] * 3;
    double* gb = args.grad + (long long)args.ws_atm[B] * 3;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      atomicAdd(ga + k, gA[k]);
      atomicAdd(gb + k, gB[k]);
    }
  }
}

template <int LA, int LB, bool DERIV>
static void launch_one(const OneArgs& a, cudaStream_t st) {
  if (a.npairs == 0) return;
  const long long threads = (long long)a.npairs * ncart(LA);
  one_electron_kernel<LA, LB, DERIV><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a);
}

void launch_one_electron(int pc, bool deriv, const OneArgs& a, cudaStream_t st) {
#define B200JK_ONE(PC, LA, LB) \
  case PC: deriv ? launch_one<LA, LB, true>(a, st) : launch_one<LA, LB, false>(a, st); break;
  switch (pc) {
    B200JK_ONE(0, 0, 0) B200JK_ONE(1, 1, 0) B200JK_ONE(2, 1, 1) B200JK_ONE(3, 2, 0)
    B200JK_ONE(4, 2, 1) B200JK_ONE(5, 2, 2) B200JK_ONE(6, 3, 0) B200JK_ONE(7, 3, 1)
    B200JK_ONE(8, 3, 2) B200JK_ONE(9, 3, 3)
  }
#undef B200JK_ONE
}

}  // namespace b200jk
