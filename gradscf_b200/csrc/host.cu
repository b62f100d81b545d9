// Plan construction, basis transforms, J/K orchestration and the C ABI.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <unordered_map>
#include <set>
#include <functional>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/b200jk.h"
#include "jk_kernels.cuh"
#include "plan.h"
#include "rys_tables.h"

namespace b200jk {

// ---------------------------------------------------------------- errors
static thread_local std::string g_error;
void set_error(const std::string& msg) { g_error = msg; }

struct Failure {
  int code;
  std::string msg;
};

#define CUDA_OK(expr)                                                                   \
  do {                                                                                  \
    cudaError_t _e = (expr);                                                            \
    if (_e != cudaSuccess)                                                              \
      throw Failure{B200JK_INTERNAL, std::string(#expr) + ": " + cudaGetErrorString(_e)}; \
  } while (0)

static void invalid(const std::string& m) { throw Failure{B200JK_INVALID_ARGUMENT, m}; }

// ---------------------------------------------------------------- dispatch
const DispatchTable& dispatch() {
  static DispatchTable table;
  static std::once_flag once;
  std::call_once(once, [] {
#define B200JK_CALL_REG(x, y) register_jk_class_##x##_##y(table);
    B200JK_FOR_EACH_CLASS_PAIR(B200JK_CALL_REG)
#undef B200JK_CALL_REG
  });
  return table;
}

// ---------------------------------------------------------------- transforms
// Output transform of shell l: column f of row c is the coefficient of raw
// Cartesian component c (x^lx y^ly z^lz times the normalised radial part) in
// output function f.  Spherical: real solid harmonics r^l Y_lm, m = -l..l
// (p: x, y, z), with the closed form of Helgaker, Jorgensen & Olsen,
// "Molecular Electronic-Structure Theory" eq. 6.4.47-6.4.50, times
// sqrt((2l+1)/4pi).  Cartesian: libcint keeps the angular factors
// 1/(2 sqrt(pi)) and sqrt(3/(4 pi)) on s and p functions and none above.
static double fact(int n) { double r = 1; for (int i = 2; i <= n; ++i) r *= i; return r; }
static double binomd(int n, int k) { return (k < 0 || k > n) ? 0.0 : fact(n) / (fact(k) * fact(n - k)); }

static void output_transform(int l, int cart, double* t /* [10][10] */) {
  std::fill(t, t + kTS, 0.0);
  const int nc = (l + 1) * (l + 2) / 2;
  if (cart) {
    const double f = l == 0 ? 0.282094791773878143 : (l == 1 ? 0.488602511902919921 : 1.0);
    for (int c = 0; c < nc; ++c) t[c * kTW + c] = f;
    return;
  }
  const double norm = std::sqrt((2 * l + 1) / (4 * M_PI));
  for (int m = -l; m <= l; ++m) {
    const int am = std::abs(m);
    int col = m + l;
    if (l == 1) col = m == 1 ? 0 : (m == -1 ? 1 : 2);
    const double nlm = 1.0 / (std::pow(2.0, am) * fact(l)) *
                       std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
    for (int tt = 0; tt <= (l - am) / 2; ++tt)
      for (int u = 0; u <= tt; ++u)
        for (int v2 = (m < 0 ? 1 : 0); v2 <= am; v2 += 2) {
          const int sgn_exp = tt + (v2 - (m < 0 ? 1 : 0)) / 2;
          const double coef = (sgn_exp % 2 ? -1.0 : 1.0) * std::pow(0.25, tt) * binomd(l, tt) *
                              binomd(l - tt, am + tt) * binomd(tt, u) * binomd(am, v2);
          const int px = 2 * tt + am - 2 * u - v2, py = 2 * u + v2, pz = l - 2 * tt - am;
          const int c = (l - px) * (l - px + 1) / 2 + pz;
          (void)py;
          t[c * kTW + col] += norm * nlm * coef;
        }
  }
}

// ---------------------------------------------------------------- tables
struct DeviceTables {
  Tables t{};
  DevBuf rys, rys_f, off, nint, ar, aw, boys, boys_f, c2s_sph, c2s_cart, boys_m, boys_m_f, boys_s_f;
  Tables sph, cartt;
};

static std::mutex g_tables_mu;
static std::map<int, DeviceTables*> g_tables;

static DeviceTables& tables_for(int device) {
  std::lock_guard<std::mutex> lock(g_tables_mu);
  auto it = g_tables.find(device);
  if (it != g_tables.end()) return *it->second;
  auto* d = new DeviceTables();
  auto up = [](DevBuf& b, const void* src, size_t n) {
    CUDA_OK(b.ensure(n));
    CUDA_OK(cudaMemcpy(b.ptr, src, n, cudaMemcpyHostToDevice));
  };
  up(d->rys, kRysTable, sizeof(kRysTable));
  std::vector<float> rf(kRysTable, kRysTable + RYS_TABLE_SIZE);
  up(d->rys_f, rf.data(), rf.size() * sizeof(float));
  up(d->off, kRysOffset, sizeof(kRysOffset));
  up(d->nint, kRysIntervals, sizeof(kRysIntervals));
  up(d->ar, kRysAsymR, sizeof(kRysAsymR));
  up(d->aw, kRysAsymW, sizeof(kRysAsymW));
  up(d->boys, kBoysGrid, sizeof(kBoysGrid));
  std::vector<float> bf(kBoysGrid, kBoysGrid + BOYS_NROW * BOYS_NCOL);
  up(d->boys_f, bf.data(), bf.size() * sizeof(float));
  {
    // per-order Taylor rows: F_{M+i}(k/20) / i!, M = 1, 3, 5
    std::vector<double> bm(3 * 801 * 8);
    for (int mi = 0; mi < 3; ++mi)
      for (int k = 0; k < 801; ++k) {
        double fact_i = 1.0;
        for (int i = 0; i < 8; ++i) {
          if (i > 0) fact_i *= i;
          bm[(mi * 801 + k) * 8 + i] = kBoysGrid[k * BOYS_NCOL + (2 * mi + 1) + i] / fact_i;
        }
      }
    up(d->boys_m, bm.data(), bm.size() * sizeof(double));
    std::vector<float> bs(3 * 401 * 8);
    for (int mi = 0; mi < 3; ++mi)
      for (int k = 0; k < 401; ++k)
        for (int i = 0; i < 8; ++i) bs[(mi * 401 + k) * 8 + i] = float(bm[(mi * 801 + 2 * k) * 8 + i]);
    up(d->boys_s_f, bs.data(), bs.size() * sizeof(float));
    std::vector<float> bmf(bm.begin(), bm.end());
    up(d->boys_m_f, bmf.data(), bmf.size() * sizeof(float));
  }
  std::vector<double> cs(4 * kTS), cc(4 * kTS);
  for (int l = 0; l <= 3; ++l) {
    output_transform(l, 0, cs.data() + l * kTS);
    output_transform(l, 1, cc.data() + l * kTS);
  }
  up(d->c2s_sph, cs.data(), cs.size() * sizeof(double));
  up(d->c2s_cart, cc.data(), cc.size() * sizeof(double));
  Tables base{};
  base.rys = d->rys.as<double>();
  base.rys_f = d->rys_f.as<float>();
  base.rys_off = d->off.as<int>();
  base.rys_nint = d->nint.as<int>();
  base.asym_r = d->ar.as<double>();
  base.asym_w = d->aw.as<double>();
  base.boys = d->boys.as<double>();
  base.boys_f = d->boys_f.as<float>();
  base.boys_m = d->boys_m.as<double>();
  base.boys_m_f = d->boys_m_f.as<float>();
  base.boys_s_f = d->boys_s_f.as<float>();
  d->sph = base;
  d->sph.c2s = d->c2s_sph.as<double>();
  d->cartt = base;
  d->cartt.c2s = d->c2s_cart.as<double>();
  g_tables[device] = d;
  return *d;
}

static Tables plan_tables(const Plan& p) {
  DeviceTables& d = tables_for(p.device);
  return p.cart ? d.cartt : d.sph;
}

// ---------------------------------------------------------------- small kernels
// Input densities (output basis, packed per molecule) -> raw Cartesian
// effective densities: symmetric part (all nb) then, if hermi == 0, the
// antisymmetric part.  Also flags a nonfinite density in *status.
__global__ void density_in_kernel(const double* __restrict__ din, int nb, int hermi,
                                  double* __restrict__ dout, long long out_stride,
                                  long long cart_stride, const long long* mol_out_base,
                                  const int* mol_nout, const long long* mol_cart_base,
                                  const int* mol_ncart, const int* cart_ws, const int4* ws_info,
                                  const int* mol_cart_ao, const double* c2s, int* status) {
  const int mol = blockIdx.y;
  const int e = blockIdx.z;
  const int nc = mol_ncart[mol];
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)nc * nc) return;
  const int i = (int)(idx / nc), j = (int)(idx % nc);
  const int no = mol_nout[mol];
  const int wi = cart_ws[mol_cart_ao[mol] + i], wj = cart_ws[mol_cart_ao[mol] + j];
  const int4 si = ws_info[wi], sj = ws_info[wj];
  const int ci = i - si.x, cj = j - sj.x;
  const double* ti = c2s + si.y * kTS + ci * kTW;
  const double* tj = c2s + sj.y * kTS + cj * kTW;
  const double* d = din + (long long)e * out_stride + mol_out_base[mol];
  double sym = 0.0, anti = 0.0;
  bool finite = true;
  for (int fa = 0; fa < kTW; ++fa) {
    const double x = ti[fa];
    if (x == 0.0) continue;
    for (int fb = 0; fb < kTW; ++fb) {
      const double y = tj[fb];
      if (y == 0.0) continue;
      const double dab = d[(long long)(si.w + fa) * no + sj.w + fb];
      const double dba = d[(long long)(sj.w + fb) * no + si.w + fa];
      finite = finite && isfinite(dab);
      sym += x * y * (dab + dba);
      anti += x * y * (dab - dba);
    }
  }
  if (!finite) atomicOr(status, 1);
  const long long o = mol_cart_base[mol] + (long long)i * nc + j;
  dout[(long long)e * cart_stride + o] = 0.5 * sym;
  if (!hermi) dout[(long long)(nb + e) * cart_stride + o] = 0.5 * anti;
}

// MJ/MK (raw Cartesian, unsymmetrised) -> J/K in the output basis.
__global__ void jk_out_kernel(const double* __restrict__ vj, const double* __restrict__ vk, int nb,
                              int hermi, int with_j, int with_k, double* __restrict__ out,
                              long long out_stride, long long cart_stride,
                              const long long* mol_out_base, const int* mol_nout,
                              const long long* mol_cart_base, const int* mol_ncart,
                              const int* out_ws, const int4* ws_info, const int* mol_out_ao,
                              const double* c2s) {
  const int mol = blockIdx.y;
  const int e = blockIdx.z;
  const int no = mol_nout[mol];
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)no * no) return;
  const int a = (int)(idx / no), b = (int)(idx % no);
  const int wa = out_ws[mol_out_ao[mol] + a], wb = out_ws[mol_out_ao[mol] + b];
  const int4 sa = ws_info[wa], sb = ws_info[wb];
  const int fa = a - sa.w, fb = b - sb.w;
  const int na = (sa.y + 1) * (sa.y + 2) / 2, nbf = (sb.y + 1) * (sb.y + 2) / 2;
  const double* ta = c2s + sa.y * kTS;
  const double* tb = c2s + sb.y * kTS;
  const int nc = mol_ncart[mol];
  const long long cb = mol_cart_base[mol];
  double jv = 0.0, kv = 0.0;
  for (int i = 0; i < na; ++i) {
    const double x = ta[i * kTW + fa];
    if (x == 0.0) continue;
    const int ci = sa.x + i;
    for (int j = 0; j < nbf; ++j) {
      const double y = tb[j * kTW + fb];
      if (y == 0.0) continue;
      const int cj = sb.x + j;
      const long long ij = cb + (long long)ci * nc + cj, ji = cb + (long long)cj * nc + ci;
      if (with_j) {
        const double* m = vj + (long long)e * cart_stride;
        jv += x * y * (m[ij] + m[ji]);
      }
      if (with_k) {
        const double* m = vk + (long long)e * cart_stride;
        double v = m[ij] + m[ji];
        if (!hermi) {
          const double* ma = vk + (long long)(nb + e) * cart_stride;
          v += ma[ij] - ma[ji];
        }
        kv += x * y * v;
      }
    }
  }
  const long long o = mol_out_base[mol] + (long long)a * no + b;
  if (with_j) out[(long long)e * out_stride + o] = jv;
  if (with_k) out[(long long)((with_j ? nb : 0) + e) * out_stride + o] = kv;
}

// Output-basis matrices -> raw Cartesian, X_raw = T X T^T (no symmetrisation).
__global__ void mat_in_kernel(const double* __restrict__ xin, double* __restrict__ xout,
                              long long out_stride, long long cart_stride,
                              const long long* mol_out_base, const int* mol_nout,
                              const long long* mol_cart_base, const int* mol_ncart,
                              const int* cart_ws, const int4* ws_info, const int* mol_cart_ao,
                              const double* c2s) {
  const int mol = blockIdx.y;
  const int e = blockIdx.z;
  const int nc = mol_ncart[mol];
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)nc * nc) return;
  const int i = (int)(idx / nc), j = (int)(idx % nc);
  const int no = mol_nout[mol];
  const int wi = cart_ws[mol_cart_ao[mol] + i], wj = cart_ws[mol_cart_ao[mol] + j];
  const int4 si = ws_info[wi], sj = ws_info[wj];
  const double* ti = c2s + si.y * kTS + (i - si.x) * kTW;
  const double* tj = c2s + sj.y * kTS + (j - sj.x) * kTW;
  const double* x = xin + (long long)e * out_stride + mol_out_base[mol];
  double v = 0.0;
  for (int fa = 0; fa < kTW; ++fa) {
    if (ti[fa] == 0.0) continue;
    for (int fb = 0; fb < kTW; ++fb)
      if (tj[fb] != 0.0) v += ti[fa] * tj[fb] * x[(long long)(si.w + fa) * no + sj.w + fb];
  }
  xout[(long long)e * cart_stride + mol_cart_base[mol] + (long long)i * nc + j] = v;
}

// Raw Cartesian matrix -> output basis, M_out = T^T M T (no symmetrisation).
__global__ void cart_to_out_kernel(const double* __restrict__ m, double* __restrict__ out,
                                   const long long* mol_out_base, const int* mol_nout,
                                   const long long* mol_cart_base, const int* mol_ncart,
                                   const int* out_ws, const int4* ws_info, const int* mol_out_ao,
                                   const double* c2s) {
  const int mol = blockIdx.y;
  const int no = mol_nout[mol];
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)no * no) return;
  const int a = (int)(idx / no), b = (int)(idx % no);
  const int wa = out_ws[mol_out_ao[mol] + a], wb = out_ws[mol_out_ao[mol] + b];
  const int4 sa = ws_info[wa], sb = ws_info[wb];
  const int fa = a - sa.w, fb = b - sb.w;
  const int na = (sa.y + 1) * (sa.y + 2) / 2, nbf = (sb.y + 1) * (sb.y + 2) / 2;
  const double* ta = c2s + sa.y * kTS;
  const double* tb = c2s + sb.y * kTS;
  const int nc = mol_ncart[mol];
  const long long cb = mol_cart_base[mol];
  double v = 0.0;
  for (int i = 0; i < na; ++i) {
    const double x = ta[i * kTW + fa];
    if (x == 0.0) continue;
    for (int j = 0; j < nbf; ++j) {
      const double y = tb[j * kTW + fb];
      if (y == 0.0) continue;
      v += x * y * m[cb + (long long)(sa.x + i) * nc + sb.x + j];
    }
  }
  out[mol_out_base[mol] + (long long)a * no + b] = v;
}

__global__ void to_float_kernel(const double* __restrict__ x, float* __restrict__ y, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = float(x[i]);
}

__global__ void maxabs_kernel(const double* __restrict__ x, long long n, double* out) {
  double m = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = fabs(x[i]);
    if (v > m) m = v;
  }
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0 && m > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(out), (unsigned long long)__double_as_longlong(m));
}

// max |D| over every row of the effective Cartesian densities (all sets), by
// global Cartesian row; one warp per row.
__global__ void rowmax_kernel(const double* __restrict__ dens, int ndm, long long dstride,
                              const long long* __restrict__ mol_base, const int* __restrict__ mol_n,
                              const int* __restrict__ mol_ao_off, const int* __restrict__ cart_ws,
                              const int4* __restrict__ ws_info, int nrows, double* __restrict__ rowmax) {
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= nrows) return;
  const int m = ws_info[cart_ws[row]].z;
  const int n = mol_n[m];
  const long long base = mol_base[m] + (long long)(row - mol_ao_off[m]) * n;
  double v = 0.0;
  for (int e = 0; e < ndm; ++e)
    for (int j = lane; j < n; j += 32) v = fmax(v, fabs(dens[e * dstride + base + j]));
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  if (lane == 0) rowmax[row] = v;
}

// Split-precision coordinate VJP, per Cartesian row i: 8 nb v_i^2 with
// v_i = max(|D|, 2|Jbar|, 2|Kbar|) over row i and column i of every batch.
// Each Gamma term of a quartet (ab|cd) is a cotangent element times a
// density element, each with an index in A, B or C: 8 terms Jbar x D (J_ab
// D_cd, J_cd D_ab and transposes) and 8 terms Kbar x D per batch, so
// |Gamma| <= 8 nb max|D| (max|Jbar| + max|Kbar|) <= 8 nb V^2 with V the
// largest v_i over the rows of A, B and C (the rows the item bound of
// split_kernel takes).
__global__ void grad_rowmax_kernel(const double* __restrict__ dens, const double* __restrict__ cj,
                                   const double* __restrict__ ck, int nb, long long dstride,
                                   const long long* __restrict__ mol_base, const int* __restrict__ mol_n,
                                   const int* __restrict__ mol_ao_off, const int* __restrict__ cart_ws,
                                   const int4* __restrict__ ws_info, int nrows, double* __restrict__ rowmax) {
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= nrows) return;
  const int m = ws_info[cart_ws[row]].z;
  const int n = mol_n[m];
  const long long i = row - mol_ao_off[m];
  double v = 0.0;
  for (int e = 0; e < nb; ++e)
    for (int x = 0; x < 3; ++x) {
      const double* X = x == 0 ? dens : (x == 1 ? cj : ck);
      if (!X) continue;
      const double w = x == 0 ? 1.0 : 2.0;
      const double* M = X + e * dstride + mol_base[m];
      for (int j = lane; j < n; j += 32) v = fmax(v, w * fmax(fabs(M[i * n + j]), fabs(M[(long long)j * n + i])));
    }
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  if (lane == 0) rowmax[row] = 8.0 * nb * v * v;
}

// Density bound of the quartets of one work item: every density element a
// quartet (ab|cd) digests (D_cd, D_ab, D_bd, D_bc, D_ad, D_ac) lies in a row
// of shell A, B or C, so max |D| over those rows bounds them; over the
// item's kets (and every contraction combination of grouped entries).
struct SplitLists {
  const int4 *bix, *bgx, *bgy;
  const double* kmax;  // per ket position: max |D| over its C rows
  const double4* bra;
  int gb, na, nb;
};

__device__ __forceinline__ double rows_max(const double* rowmax, int base, int off, int n) {
  double v = 0.0;
  for (int i = 0; i < n; ++i) v = fmax(v, rowmax[base + off + i]);
  return v;
}

// Per list position: max |D| over the rows of its A shell (every combination).
__global__ void posmax_kernel(const int4* __restrict__ ix, const int4* __restrict__ gx,
                              const int4* __restrict__ gy, const int* __restrict__ nco,
                              const double4* __restrict__ ra, int npos, int na,
                              const double* __restrict__ rowmax, const int* __restrict__ mol_ao_off,
                              double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npos) return;
  const int base = mol_ao_off[(int)ra[k].w];
  const int g = nco ? nco[k] : 1;
  double v = rows_max(rowmax, base, ix[k].z, na);
  if (g > 1) {
    const int4 x = gx[k], y = gy[k];
    v = fmax(v, rows_max(rowmax, base, x.z, na));
    if (g > 2) v = fmax(v, fmax(rows_max(rowmax, base, y.x, na), rows_max(rowmax, base, y.z, na)));
  }
  out[k] = v;
}

// Per work item: first ket position of its range computed in FP32,
// Q_bra * Q_ket * max|D over the rows the item's quartets touch| < fp32_cut
// (ket bounds sorted descending, so the FP32 kets are a suffix).
__global__ void split_kernel(const int4* __restrict__ work, const double* __restrict__ bra_q,
                             const double* __restrict__ ket_q, const double* __restrict__ rowmax,
                             const int* __restrict__ mol_ao_off, SplitLists L, double fp32_cut,
                             int nwork, int* __restrict__ split) {
  // one warp per item: the lanes take the item's kets, then lane 0 searches
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= nwork) return;
  const int4 w = work[i];
  const int base = mol_ao_off[(int)L.bra[w.x].w];
  double dmax = 0.0;
  if (lane < L.gb) {
    const int4 ix = L.bix[w.x];
    const int4 gx = L.gb > 1 ? L.bgx[w.x] : make_int4(0, 0, 0, 0);
    const int4 gy = L.gb > 1 ? L.bgy[w.x] : make_int4(0, 0, 0, 0);
    const int a = lane == 0 ? ix.z : lane == 1 ? gx.z : lane == 2 ? gy.x : gy.z;
    const int b = lane == 0 ? ix.w : lane == 1 ? gx.w : lane == 2 ? gy.y : gy.w;
    dmax = fmax(rows_max(rowmax, base, a, L.na), rows_max(rowmax, base, b, L.nb));
  }
  for (int k = w.y + lane; k < w.z; k += 32) dmax = fmax(dmax, L.kmax[k]);
  for (int off = 16; off > 0; off >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
  if (lane != 0) return;
  const double f = bra_q[w.x] * dmax;
  int lo = w.y, hi = w.z;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ket_q[mid] * f < fp32_cut) hi = mid;
    else lo = mid + 1;
  }
  split[i] = lo;
}

// Per bra-group work item: max |D| over the rows its quartets touch -- the
// common A shell, every bra's B shell, every ket's C shell (one warp per item).
__global__ void grp_split_kernel(const int4* __restrict__ work, int nwork, const int* __restrict__ bord,
                                 const int4* __restrict__ bix, const int4* __restrict__ bgx,
                                 const int4* __restrict__ bgy, int gb, const double4* __restrict__ bra,
                                 const double* __restrict__ kmax, const double* __restrict__ rowmax,
                                 const int* __restrict__ mol_ao_off, int na, int nb, double* __restrict__ m_out) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= nwork) return;
  const int4 w = work[i];
  const int p0 = bord[w.x];
  const int base = mol_ao_off[(int)bra[p0].w];
  double dmax = 0.0;
  for (int b = lane; b < w.y; b += 32) {
    const int pos = bord[w.x + b];
    const int4 ix = bix[pos];
    const int4 gx = gb > 1 ? bgx[pos] : make_int4(0, 0, 0, 0);
    const int4 gy = gb > 1 ? bgy[pos] : make_int4(0, 0, 0, 0);
    const int ao[4] = {ix.z, gx.z, gy.x, gy.z}, bo[4] = {ix.w, gx.w, gy.y, gy.w};
    for (int c = 0; c < gb; ++c)
      dmax = fmax(dmax, fmax(rows_max(rowmax, base, ao[c], na), rows_max(rowmax, base, bo[c], nb)));
  }
  for (int k = w.z + lane; k < w.w; k += 32) dmax = fmax(dmax, kmax[k]);
  for (int off = 16; off > 0; off >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
  if (lane == 0) m_out[i] = dmax;
}

// Split builds, per bra-group item (one warp): its FP64 quartets (Q_bra
// Q_ket >= cut, canonical, not Q_bra Q_ket M_item < fp32_cut -- the
// bra-group kernels' own tests) are appended to the flat list and the item
// is flagged so the bra-group FP64 launch skips it (the FP64 quartets of an
// item are the leading kets of its leading bras: on the bra-group path most
// lanes of their passes idle).  A reservation past the list's capacity is
// filled with (-1, -1) and its item stays on the bra-group path.  Kets of an
// item are sorted by bound (descending), so a bra's scan stops at the first
// pass that starts in FP32.
__global__ void border_kernel(const int4* __restrict__ work, int nwork, const int* __restrict__ bord,
                              const double* __restrict__ bra_q, const double* __restrict__ ket_q,
                              const double* __restrict__ item_m, int same_list, double cut, double fp32_cut,
                              int2* __restrict__ flat, unsigned long long* __restrict__ flat_n, int cap,
                              int* __restrict__ skip) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= nwork) return;
  const int4 w = work[i];
  const double qm = item_m[i];
  auto scan = [&](auto&& visit) {
    for (int bi = 0; bi < w.y; ++bi) {
      const int pos = bord[w.x + bi];
      const double qb = bra_q[pos];
      for (int k0 = w.z; k0 < w.w; k0 += 32) {
        const double q0 = qb * ket_q[k0];
        if (q0 < cut || q0 * qm < fp32_cut) break;   // this pass and the later ones hold no FP64 quartet
        const int k = k0 + lane;
        bool act = false;
        if (k < w.w) {
          const double qq = qb * ket_q[k];
          act = qq >= cut && (!same_list || k <= pos) && !(qq * qm < fp32_cut);
        }
        visit(pos, k, act, __ballot_sync(0xffffffffu, act));
      }
    }
  };
  int count = 0;
  scan([&](int, int, bool, unsigned b) { count += __popc(b); });
  if (count == 0) {
    if (lane == 0) skip[i] = 1;
    return;
  }
  // 64-bit reservation counter: the counts of one build can pass 2^31
  long long base = 0;
  if (lane == 0) base = (long long)atomicAdd(flat_n, (unsigned long long)count);
  base = __shfl_sync(0xffffffffu, base, 0);
  if (base + count > (long long)cap) {
    for (long long j = base + lane; j < (long long)cap && j < base + count; j += 32) flat[j] = make_int2(-1, -1);
    if (lane == 0) skip[i] = 0;
    return;
  }
  int at = (int)base;
  scan([&](int pos, int k, bool act, unsigned b) {
    if (act) flat[at + __popc(b & ((1u << lane) - 1u))] = make_int2(pos, k);
    at += __popc(b);
  });
  if (lane == 0) skip[i] = 1;
}

// ---------------------------------------------------------------- plan creation
static int ncart_of(int l) { return (l + 1) * (l + 2) / 2; }
static int pc_la_host(int pc) { return pc == 0 ? 0 : pc <= 2 ? 1 : pc <= 5 ? 2 : 3; }

struct PrimPair {
  double4 data;
  double k;
};

static void validate_tables(const b200jk_molecule& m, int cart) {
  // csrc/tables.h:40-75
  if (m.natm < 0 || m.nbas < 1 || m.nenv < 20 || (cart != 0 && cart != 1) || !m.atm || !m.bas || !m.env)
    invalid("Invalid libcint table dimensions or operator");
  for (int i = 0; i < m.nenv; ++i)
    if (!std::isfinite(m.env[i])) invalid("Native integral env must be finite");
  if (m.env[8] > std::sqrt(std::numeric_limits<double>::max()) / 2.0)
    invalid("omega exceeds the safe float64 squared range");
  // env[8] (libcint PTR_RANGE_OMEGA): omega > 0 selects erf(omega r)/r, as the
  // reference's long-range J/K sets it (plan.py:86-87); the short-range
  // (omega < 0) operator is not built
  if (m.env[8] < 0.0) throw Failure{B200JK_UNSUPPORTED, "Short-range (omega < 0) J/K is not built on the B200 path"};
  for (int a = 0; a < m.natm; ++a) {
    const int32_t* row = m.atm + a * 6;
    if (row[1] < 20 || row[1] + 3 > m.nenv || row[2] != 1)
      invalid("Native backend requires valid point nuclei");
  }
  for (int s = 0; s < m.nbas; ++s) {
    const int32_t* row = m.bas + s * 8;
    const int l = row[1], np = row[2], nc = row[3];
    if (row[0] < 0 || row[0] >= m.natm || l < 0 || l > 12 || np < 1 || np > 64 || nc < 1 || nc > 64 ||
        row[4] != 0 || row[5] < 20 || row[5] + np > m.nenv || row[6] < 20 ||
        (long long)row[6] + (long long)np * nc > m.nenv)
      invalid("Invalid or unsupported libcint basis table");
    for (int p = 0; p < np; ++p)
      if (m.env[row[5] + p] <= 0.0) invalid("Gaussian exponents must be positive");
    if (l > kMaxL)
      throw Failure{B200JK_UNSUPPORTED, "Angular momentum above f (l > 3) is not built on the B200 path"};
  }
}

static void upload(DevBuf& b, const void* src, size_t n) {
  CUDA_OK(b.ensure(n));
  if (n) CUDA_OK(cudaMemcpy(b.ptr, src, n, cudaMemcpyHostToDevice));
}

// Bra/ket class lists of a class pair: pair ids and per-position records.
static void set_lists(JKArgs& a, const Plan& p, const ClassPairWork& W) {
  const ClassList& X = p.classes[W.x];
  const ClassList& Y = p.classes[W.y];
  a.bra_pairs = X.d_pairs.as<int>();
  a.ket_pairs = Y.d_pairs.as<int>();
  a.bra_ra = X.d_ra.as<double4>();
  a.bra_ab = X.d_ab.as<double4>();
  a.bra_ix = X.d_ix.as<int4>();
  a.ket_ra = Y.d_ra.as<double4>();
  a.ket_ab = Y.d_ab.as<double4>();
  a.ket_ix = Y.d_ix.as<int4>();
  a.same_list = W.x == W.y;
}

// The J/K launches of one class pair: its buckets on grouped lists, or its
// expanded work items.
struct JKUnit {
  const DevBuf* work;
  int nwork;
  DevBuf* split;
  const ClassList* X;
  const ClassList* Y;
  int gb, gk;
  std::vector<int4>* h_items;
  GroupWork* grp;   // non-null: the unit runs the register path over bra groups
};

template <typename F>
static void for_each_unit(Plan& p, ClassPairWork& W, F&& f) {
  auto active = [](GroupWork& G) { return G.h_items.empty() ? &G.all_items : &G.h_items; };
  if (!W.buckets.empty()) {
    const ClassList* X = W.grouped_x ? &p.grouped[W.x] : &p.classes[W.x];
    const ClassList* Y = W.grouped_y ? &p.grouped[W.y] : &p.classes[W.y];
    for (auto* B : W.buckets) {
      if (B->use_grp)
        f(JKUnit{&B->grp.work, B->grp.nwork, &B->grp.m, X, Y, B->gb, B->gk, active(B->grp), &B->grp});
      else
        f(JKUnit{&B->work, B->nwork, &B->split, X, Y, B->gb, B->gk, B->h_items.empty() ? &B->all_items : &B->h_items,
                 nullptr});
    }
  } else if (W.use_grp) {
    f(JKUnit{&W.grp.work, W.grp.nwork, &W.grp.m, &p.classes[W.x], &p.classes[W.y], 1, 1, active(W.grp), &W.grp});
  } else {
    f(JKUnit{&W.work, W.nwork, &W.split, &p.classes[W.x], &p.classes[W.y], 1, 1,
             W.h_items.empty() ? &W.all_items : &W.h_items, nullptr});
  }
}

static void set_unit_lists(JKArgs& a, const JKUnit& u, bool same) {
  a.bra_pairs = u.X->d_pairs.as<int>();
  a.ket_pairs = u.Y->d_pairs.as<int>();
  a.bra_ra = u.X->d_ra.as<double4>();
  a.bra_ab = u.X->d_ab.as<double4>();
  a.bra_ix = u.X->d_ix.as<int4>();
  a.bra_gx = u.X->d_gx.as<int4>();
  a.bra_gy = u.X->d_gy.as<int4>();
  a.ket_ra = u.Y->d_ra.as<double4>();
  a.ket_ab = u.Y->d_ab.as<double4>();
  a.ket_ix = u.Y->d_ix.as<int4>();
  a.ket_gx = u.Y->d_gx.as<int4>();
  a.ket_gy = u.Y->d_gy.as<int4>();
  a.bra_bord = u.X->d_bord.as<int>();
  a.bra_q = u.X->d_q.as<double>();
  a.ket_q = u.Y->d_q.as<double>();
  a.same_list = same;
}

static int gen_slot(int gb, int gk) {
  auto k = [](int g) { return g == 1 ? 0 : (g == 2 ? 1 : 2); };
  return k(gb) * 3 + k(gk);
}

static JKArgs base_args(const Plan& p) {
  JKArgs a{};
  a.sh_info = p.d_ws_info.as<int4>();
  a.sh_xyz = p.d_ws_xyz.as<double4>();
  a.pair_info = p.d_pair_info.as<int4>();
  a.pp_data = p.d_pp_data.as<double4>();
  a.pp_aux = p.d_pp_aux.as<double2>();
  a.pp_exp = p.d_pp_exp.as<double2>();
  a.pp_f = p.d_pp_f.as<float4>();
  a.pp_f2 = p.d_pp_f2.as<float2>();
  a.pp_c = p.d_pp_c.as<double4>();
  a.omega2 = p.omega * p.omega;
  a.pp_cf = p.d_pp_cf.as<float4>();
  a.ws_atm = p.d_ws_atm.as<int>();
  a.mol_base = p.d_mol_base_cart.as<long long>();
  a.mol_n = p.d_mol_ncart.as<int>();
  a.tb = plan_tables(p);
  a.status = p.d_status.as<int>();
  a.cutoff = p.cutoff;
  return a;
}

// (bra position, ket run [lo, hi)) of every bra: the Schwarz-screened
// prefix of each ket run of the bra's molecule, canonical when X == Y
template <typename F>
static void for_each_run(const ClassList& X, const ClassList& Y, bool same, double cut, F&& emit) {
  for (int bp = 0; bp < (int)X.q.size(); ++bp) {
    const int m = X.mol_pos[bp];
    const double qb = X.q[bp];
    for (const int2 seg : Y.segs[m]) {
      const int lo = seg.x;
      if (same && lo > bp) break;  // canonical: ket position <= bra position
      int hi = seg.y;
      if (cut > 0) {
        int a = lo, b = seg.y;  // first ket with qb*qk < cut (bounds sorted descending)
        while (a < b) {
          const int mid = (a + b) >> 1;
          if (qb * Y.q[mid] < cut) b = mid;
          else a = mid + 1;
        }
        hi = a;
      }
      if (same) hi = std::min(hi, bp + 1);
      if (hi > lo) emit(bp, lo, hi);
    }
  }
}

#ifndef B200JK_TILE_CHUNK
#define B200JK_TILE_CHUNK 64   // kets per tile-path work item (measured best of 16/32/64)
#endif
#ifndef B200JK_REG_CHUNK
#define B200JK_REG_CHUNK 64    // kets per register-path work item (two 32-ket passes of a warp)
#endif
#ifndef B200JK_HEAVY_PQ
#define B200JK_HEAVY_PQ 64  // primitive quartets per quartet from which items take 32 kets (measured)
#endif

// register path: items of heavy quartets (many primitive pairs on both
// sides) take one 32-ket pass, so long items do not form the launch's tail
static int reg_chunk(long long npa, long long npc) {
  return npa * npc >= (long long)(B200JK_HEAVY_PQ) ? 32 : B200JK_REG_CHUNK;
}

static void upload_items(DevBuf& work, DevBuf& split, const std::vector<int4>& items) {
  CUDA_OK(work.ensure(std::max<size_t>(items.size(), 1) * sizeof(int4)));
  if (!items.empty())
    CUDA_OK(cudaMemcpy(work.ptr, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CUDA_OK(split.ensure(std::max<size_t>(items.size(), 1) * sizeof(int)));
}

#ifndef B200JK_GRP_BRAS
#define B200JK_GRP_BRAS 16   // bras per bra-group work item
#endif
#ifndef B200JK_GRP_CHUNK
#define B200JK_GRP_CHUNK 64  // kets per bra-group work item
#endif

// First ket position in [lo, hi) of a Q-descending run with qb * Q < cut.
static int screen_end(const ClassList& Y, int lo, int hi, double qb, double cut) {
  if (cut <= 0) return hi;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (qb * Y.q[mid] < cut) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Work items of the register path over bra groups: for every group of X's
// bra order (entries with `gb` combinations) and every ket run of Y in the
// same molecule (entries with `gk` combinations), the kets any bra of the
// group meets (its Schwarz prefix, and at most its own position when X and
// Y are one list), cut into chunks.
static void fill_group(GroupWork& G, const ClassList& X, const ClassList& Y, bool same, double cut, int chunk,
                       int gb, int gk) {
  G.all_items.clear();
  G.h_items.clear();
  G.item_cost.clear();
  G.quartets = G.prim_quartets = 0;
  auto nco = [](const ClassList& L, int i) { return L.nco.empty() ? 1 : L.nco[i]; };
  std::vector<int> hp;
  for (size_t gi = 0; gi + 1 < X.gbeg.size(); ++gi) {
    const int g0 = X.gbeg[gi], g1 = X.gbeg[gi + 1];
    const int first = X.bord[g0];
    if (nco(X, first) != gb) continue;
    const int m = X.mol_pos[first];
    for (int c0 = g0; c0 < g1; c0 += B200JK_GRP_BRAS) {
      const int c1 = std::min(g1, c0 + B200JK_GRP_BRAS);
      for (const int2 seg : Y.segs[m]) {
        const int lo = seg.x;
        if (nco(Y, lo) != gk) continue;
        hp.assign(c1 - c0, lo);
        int hi = lo;
        for (int i = c0; i < c1; ++i) {
          const int pos = X.bord[i];
          int h = screen_end(Y, lo, seg.y, X.q[pos], cut);
          if (same) h = std::min(h, pos + 1);
          h = std::max(h, lo);
          hp[i - c0] = h;
          hi = std::max(hi, h);
          G.quartets += (long long)(h - lo) * gb * gk;
          G.prim_quartets += (long long)X.npp_pos[pos] * (Y.npp_prefix[h] - Y.npp_prefix[lo]);
        }
        // staircase: the bras a ket meets are the chunk's first cnt(k) bras
        // (bounds sorted descending); split [lo, hi) where cnt drops, so the
        // lanes of a pass are mostly active for every bra the item lists --
        // steps shorter than a pass stay merged with the wider range before
        // them.  With one list (X == Y) the canonical cap can break the
        // order; the kernel's per-lane mask covers it.
        int s = lo;
        while (s < hi) {
          int cnt = 0;
          for (int i = c0; i < c1; ++i)
            if (hp[i - c0] > s) cnt = i - c0 + 1;
          if (cnt == 0) break;
          // the range ends where the first listed bra stops, but runs at least a pass
          int e = hi;
          for (int i = c0; i < c0 + cnt; ++i)
            if (hp[i - c0] > s) e = std::min(e, std::max(hp[i - c0], s + 32));
          e = std::min(e, hi);
          for (int b0 = s; b0 < e; b0 += chunk) {
            const int b1 = std::min(e, b0 + chunk);
            long long cost = 0;
            for (int i = c0; i < c0 + cnt; ++i) {
              const int h = std::min(std::max(hp[i - c0], b0), b1);
              cost += (long long)X.npp_pos[X.bord[i]] * (Y.npp_prefix[h] - Y.npp_prefix[b0]);
            }
            if (cost == 0) continue;
            G.all_items.push_back(make_int4(c0, cnt, b0, b1));
            G.item_cost.push_back(cost);
          }
          s = e;
        }
      }
    }
  }
  // longest first: the persistent kernels take items in list order
  {
    std::vector<int> ord(G.all_items.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return G.item_cost[a] > G.item_cost[b]; });
    std::vector<int4> items(ord.size());
    std::vector<int64_t> cost(ord.size());
    for (size_t i = 0; i < ord.size(); ++i) {
      items[i] = G.all_items[ord[i]];
      cost[i] = G.item_cost[ord[i]];
    }
    G.all_items = std::move(items);
    G.item_cost = std::move(cost);
  }
  G.nwork = (int)G.all_items.size();
  CUDA_OK(G.work.ensure(std::max<size_t>(G.all_items.size(), 1) * sizeof(int4)));
  if (!G.all_items.empty())
    CUDA_OK(cudaMemcpy(G.work.ptr, G.all_items.data(), G.all_items.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CUDA_OK(G.m.ensure(std::max<size_t>(G.all_items.size(), 1) * sizeof(double)));
  // the FP64 flat list of split builds: room for 1/16 of the group's (bra,
  // ket) pairs, at most 2^21; items that do not fit keep the bra-group path
  const long long pairs = G.quartets / std::max(1, gb * gk);
  G.flat_cap = (int)std::min<long long>(pairs / 16 + 4096, 1LL << 21);
  CUDA_OK(G.flat.ensure((size_t)G.flat_cap * sizeof(int2)));
  CUDA_OK(G.flat_n.ensure(sizeof(unsigned long long)));
  CUDA_OK(G.skip.ensure(std::max<size_t>(G.all_items.size(), 1) * sizeof(int)));
}

// (Re)build the work items of class pair W: the expanded items and, where
// both precisions' kernels take grouped lists, the grouped buckets.
// `force` > 0 sets the ket chunk of the items the J/K build launches on the
// register path (the autotuner's knob); 0 keeps the default rule.
static void fill_items(Plan& p, ClassPairWork& W, int force) {
  const auto& disp = dispatch();
  const int x = W.x, y = W.y;
  const ClassList& X = p.classes[x];
  const ClassList& Y = p.classes[y];
  const int cls = quartet_class(x, y);
  const double cut = p.cutoff;
  W.grouped_x = disp.grouped[cls] && !p.grouped[x].q.empty();
  W.grouped_y = disp.grouped[cls] && !p.grouped[y].q.empty();
  const bool grouped = W.grouped_x || W.grouped_y;
  const int chunk0 = disp.reg_path[cls] ? B200JK_REG_CHUNK : std::max(8, 4 * (128 / disp.team[cls]));
  std::vector<int4> items;
  W.quartets = W.prim_quartets = 0;
  W.item_cost.clear();
  for_each_run(X, Y, x == y, cut, [&](int bp, int lo, int hi) {
    const long long npa = X.npp_pos[bp];
    int chunk = chunk0;
    if (disp.tile[cls] && B200JK_TILE_CHUNK > 0) chunk = B200JK_TILE_CHUNK;
    else if (disp.reg_path[cls]) chunk = (force > 0 && !grouped) ? force : reg_chunk(npa, Y.npp_pos[lo]);
    W.quartets += hi - lo;
    W.prim_quartets += npa * (Y.npp_prefix[hi] - Y.npp_prefix[lo]);
    for (int s = lo; s < hi; s += chunk) {
      const int e = std::min(hi, s + chunk);
      items.push_back(make_int4(bp, s, e, 0));
      W.item_cost.push_back(npa * (Y.npp_prefix[e] - Y.npp_prefix[s]));
    }
  });
  W.nwork = (int)items.size();
  ++p.layout_gen;
  upload_items(W.work, W.split, items);
  W.h_items.clear();  // unsharded: the active items are all_items
  W.all_items = std::move(items);
  for (auto* B : W.buckets) delete B;
  W.buckets.clear();
  const bool grp = disp.grp64[cls] && disp.grp32[cls];
  const int gchunk0 = force > 0 ? force : B200JK_GRP_CHUNK;
  W.use_grp = grp && !grouped;
  if (W.use_grp) fill_group(W.grp, X, Y, x == y, cut, gchunk0, 1, 1);
  if (!grouped) return;
  const ClassList& GX = W.grouped_x ? p.grouped[x] : X;
  const ClassList& GY = W.grouped_y ? p.grouped[y] : Y;
  std::map<std::pair<int, int>, GenBucket*> by;
  for_each_run(GX, GY, x == y, cut, [&](int bp, int lo, int hi) {
    const int gb = GX.nco.empty() ? 1 : GX.nco[bp];
    const int gk = GY.nco.empty() ? 1 : GY.nco[lo];
    GenBucket*& B = by[{gb, gk}];
    if (!B) {
      B = new GenBucket();
      B->gb = gb;
      B->gk = gk;
    }
    const long long npa = GX.npp_pos[bp];
    B->quartets += (long long)(hi - lo) * gb * gk;
    B->prim_quartets += npa * (GY.npp_prefix[hi] - GY.npp_prefix[lo]);
    const int gchunk = force > 0 ? force : reg_chunk(npa, GY.npp_pos[lo]);
    for (int s = lo; s < hi; s += gchunk) {
      const int e = std::min(hi, s + gchunk);
      B->all_items.push_back(make_int4(bp, s, e, 0));
      B->item_cost.push_back(npa * (GY.npp_prefix[e] - GY.npp_prefix[s]) * (gb * gk > 1 ? 2 : 1));
    }
  });
  for (auto& kv : by) {
    GenBucket* B = kv.second;
    B->h_items.clear();
    B->nwork = (int)B->all_items.size();
    upload_items(B->work, B->split, B->all_items);
    const bool bgrp = (B->gb == 1 && B->gk == 1) ? grp
                                                    : (disp.grpg64[cls][gen_slot(B->gb, B->gk)] != nullptr &&
                                                       disp.grpg32[cls][gen_slot(B->gb, B->gk)] != nullptr);
    if (bgrp) {
      B->use_grp = true;
      fill_group(B->grp, GX, GY, x == y, cut, gchunk0, B->gb, B->gk);
    }
    W.buckets.push_back(B);
  }
}

// Restrict class pair W to the plan's shard: contiguous cost-balanced blocks
// of every item list (expanded items and grouped buckets).
static void apply_shard(Plan& p, ClassPairWork& W) {
  const int rank = p.shard_rank, world = p.shard_world;
  ++p.layout_gen;
  auto shard = [&](const std::vector<int4>& all, const std::vector<int64_t>& cost, DevBuf& work,
                   std::vector<int4>& h, int& nwork, long long& q, long long& pq, long long qmul) {
    const int64_t n = (int64_t)all.size();
    std::vector<int32_t> owner(n);
    if (b200jk_partition_items(cost.data(), n, world, owner.data()) != 0)
      throw Failure{B200JK_INTERNAL, "work-item partition failed"};
    std::vector<int4> mine;
    q = pq = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (owner[i] != rank) continue;
      if (world > 1) mine.push_back(all[i]);
      q += (long long)(all[i].z - all[i].y) * qmul;
      pq += cost[i];
    }
    const std::vector<int4>& act = world > 1 ? mine : all;
    nwork = (int)act.size();
    if (!act.empty())  // the buffer holds the full list, so it is never reallocated
      CUDA_OK(cudaMemcpy(work.ptr, act.data(), act.size() * sizeof(int4), cudaMemcpyHostToDevice));
    h = std::move(mine);  // empty when unsharded: the active items are then `all`
  };
  shard(W.all_items, W.item_cost, W.work, W.h_items, W.nwork, W.quartets, W.prim_quartets, 1);
  for (auto* B : W.buckets)
    shard(B->all_items, B->item_cost, B->work, B->h_items, B->nwork, B->quartets, B->prim_quartets,
          (long long)B->gb * B->gk);
  // bra-group items: the same contiguous cost-balanced blocks (their quartet
  // counts stay those of the whole class pair; the expanded items carry the shard's)
  auto shard_grp = [&](GroupWork& G) {
    long long q = 0, pq = 0;
    std::vector<int4> h;
    int nw = 0;
    shard(G.all_items, G.item_cost, G.work, h, nw, q, pq, 0);
    G.h_items = std::move(h);
    G.nwork = nw;
  };
  if (W.use_grp) shard_grp(W.grp);
  for (auto* B : W.buckets)
    if (B->use_grp) shard_grp(B->grp);
}

// Bra order and groups of a class list (register path over bra groups).
static void build_bra_order(ClassList& L) {
  const int n = (int)L.q.size();
  L.bord.resize(n);
  std::iota(L.bord.begin(), L.bord.end(), 0);
  auto nco = [&](int i) { return L.nco.empty() ? 1 : L.nco[i]; };
  auto key_less = [&](int a, int b) {
    if (L.mol_pos[a] != L.mol_pos[b]) return L.mol_pos[a] < L.mol_pos[b];
    if (nco(a) != nco(b)) return nco(a) < nco(b);
    if (L.npp_pos[a] != L.npp_pos[b]) return L.npp_pos[a] < L.npp_pos[b];
    return L.aoa_pos[a] < L.aoa_pos[b];
  };
  // list order breaks ties: Q descending within a group
  std::sort(L.bord.begin(), L.bord.end(), [&](int a, int b) { return key_less(a, b) || (!key_less(b, a) && a < b); });
  L.gbeg.clear();
  for (int i = 0; i < n; ++i)
    if (i == 0 || key_less(L.bord[i - 1], L.bord[i])) L.gbeg.push_back(i);
  L.gbeg.push_back(n);
  upload(L.d_bord, L.bord.data(), (size_t)n * sizeof(int));
}

// One entry of a grouped list (pair classes (l, 0)): a parent shell pair
// with nco contraction combinations (work shells ws[k] on A, wsb[k] on B).
struct GenEntry {
  int cls = 0, mol = 0, diag = 0, pair = -1, nco = 1, ppoff = 0, npp = 0;
  int ws[4] = {0, 0, 0, 0}, wsb[4] = {0, 0, 0, 0};
  long long pkey = 0;  // parent pair: max parent id * nparent + min parent id
};

static Plan* build_plan(const b200jk_molecule* mols, int nmol, int cart, double cut, int device) {
  if (nmol < 1 || !mols) invalid("At least one molecule is required");
  if (!std::isfinite(cut) || cut < 0) invalid("Invalid Schwarz cutoff");
  if (cart != 0 && cart != 1) invalid("cart must be 0 or 1");
  for (int m = 0; m < nmol; ++m) validate_tables(mols[m], cart);
  CUDA_OK(cudaSetDevice(device));
  auto plan = std::make_unique<Plan>();
  Plan& p = *plan;
  p.device = device;
  p.cart = cart;
  p.omega = mols[0].env[8];
  for (int m = 1; m < nmol; ++m)
    if (mols[m].env[8] != p.omega) invalid("All molecules of a batch need the same range parameter env[8]");
  p.cutoff = cut;
  p.nmol = nmol;
  // ---- work shells (one per contraction column of every shell)
  std::vector<int> parent_base(nmol + 1, 0);
  int atm_base = 0;
  for (int m = 0; m < nmol; ++m) {
    const auto& M = mols[m];
    parent_base[m + 1] = parent_base[m] + M.nbas;
    int out = 0, cartn = 0;
    p.mol_atm_off.push_back(atm_base);
    for (int a = 0; a < M.natm; ++a) {
      const double* r = M.env + M.atm[a * 6 + 1];
      p.atom_xyzq.push_back(make_double4(r[0], r[1], r[2], (double)M.atm[a * 6 + 0]));
    }
    for (int s = 0; s < M.nbas; ++s) {
      const int32_t* row = M.bas + s * 8;
      const int l = row[1], np = row[2], nc = row[3];
      const double* r = M.env + M.atm[row[0] * 6 + 1];
      const int nf = cart ? ncart_of(l) : 2 * l + 1;
      for (int c = 0; c < nc; ++c) {
        p.ws_info.push_back(make_int4(cartn, l, m, out + c * nf));
        p.ws_xyz.push_back(make_double4(r[0], r[1], r[2], 0.0));
        p.ws_parent.push_back(parent_base[m] + s);
        p.ws_atm.push_back(atm_base + row[0]);
        p.ws_nprim.push_back(np);
        p.ws_prim_off.push_back((int)p.ws_exp.size());
        for (int q = 0; q < np; ++q) {
          p.ws_exp.push_back(M.env[row[5] + q]);
          p.ws_coef.push_back(M.env[row[6] + c * np + q]);
        }
        cartn += ncart_of(l);
      }
      out += nc * nf;
    }
    p.mol_nout.push_back(out);
    p.mol_ncart.push_back(cartn);
    p.mol_natm.push_back(M.natm);
    atm_base += M.natm;
  }
  p.total_atm = atm_base;
  p.nws = (int)p.ws_info.size();
  long long ob = 0, cb = 0;
  for (int m = 0; m < nmol; ++m) {
    p.mol_out_base.push_back(ob);
    p.mol_cart_base.push_back(cb);
    ob += (long long)p.mol_nout[m] * p.mol_nout[m];
    cb += (long long)p.mol_ncart[m] * p.mol_ncart[m];
  }
  p.out_stride = ob;
  p.cart_stride = cb;
  // ---- shell pairs and primitive pairs
  std::vector<double4> pp_data;
  std::vector<double2> pp_aux, pp_exp;
  std::vector<float4> pp_f;
  std::vector<float2> pp_f2;
  int ws0 = 0;
  for (int m = 0; m < nmol; ++m) {
    int wsn = ws0;
    while (wsn < p.nws && p.ws_info[wsn].z == m) ++wsn;
    for (int i = ws0; i < wsn; ++i)
      for (int j = ws0; j <= i; ++j) {
        int A = i, B = j;
        if (p.ws_info[B].y > p.ws_info[A].y) std::swap(A, B);
        const double4 ra = p.ws_xyz[A], rb = p.ws_xyz[B];
        const double ab2 = (ra.x - rb.x) * (ra.x - rb.x) + (ra.y - rb.y) * (ra.y - rb.y) +
                           (ra.z - rb.z) * (ra.z - rb.z);
        const int off = (int)pp_data.size();
        for (int ia = 0; ia < p.ws_nprim[A]; ++ia)
          for (int ib = 0; ib < p.ws_nprim[B]; ++ib) {
            const double a = p.ws_exp[p.ws_prim_off[A] + ia], b = p.ws_exp[p.ws_prim_off[B] + ib];
            const double ca = p.ws_coef[p.ws_prim_off[A] + ia], cbv = p.ws_coef[p.ws_prim_off[B] + ib];
            const double pe = a + b;
            const double expo = a * b / pe * ab2;
            if (expo > 40.0 || ca == 0.0 || cbv == 0.0) continue;  // exp(-40) ~ 4e-18
            pp_data.push_back(make_double4((a * ra.x + b * rb.x) / pe, (a * ra.y + b * rb.y) / pe,
                                           (a * ra.z + b * rb.z) / pe, pe));
            pp_aux.push_back(make_double2(std::exp(-expo) * ca * cbv / pe, 0.5 / pe));
            pp_exp.push_back(make_double2(a, b));
            pp_f.push_back(make_float4(float(pp_data.back().x - ra.x), float(pp_data.back().y - ra.y),
                                       float(pp_data.back().z - ra.z), float(pe)));
            pp_f2.push_back(make_float2(float(pp_aux.back().x), float(0.5 / pe)));
          }
        const int cnt = (int)pp_data.size() - off;
        if (cnt == 0) continue;
        p.pair_info.push_back(make_int4(A, B, off, cnt));
        p.pair_class.push_back(pair_class(p.ws_info[A].y, p.ws_info[B].y));
      }
    ws0 = wsn;
  }
  p.npair = (int)p.pair_info.size();
  // every primitive pair of the expanded list carries its contraction
  // coefficients inside K: combination coefficients (1, 0, 0, 0)
  std::vector<double4> pp_c(pp_data.size(), make_double4(1.0, 0.0, 0.0, 0.0));
  // ---- grouped entries (pair classes (l, 0)): one entry per parent shell
  // pair carrying its contraction combinations, so primitive quartets shared
  // by the combinations are evaluated once.  Entries with a single
  // combination are the expanded pairs themselves.
  std::unordered_map<long long, int> ws_pair_id;  // key: max(ws) * nws + min(ws)
  ws_pair_id.reserve(2 * (size_t)p.npair + 1);
  auto ws_key = [&](int a, int b) { return (long long)std::max(a, b) * p.nws + std::min(a, b); };
  for (int q = 0; q < p.npair; ++q) ws_pair_id[ws_key(p.pair_info[q].x, p.pair_info[q].y)] = q;
  std::vector<int> parent_ws0;  // first work shell of every parent shell
  for (int w = 0; w < p.nws; ++w)
    if (w == 0 || p.ws_parent[w] != p.ws_parent[w - 1]) parent_ws0.push_back(w);
  std::vector<int> parent_nc(parent_ws0.size());
  for (size_t i = 0; i < parent_ws0.size(); ++i)
    parent_nc[i] = (i + 1 < parent_ws0.size() ? parent_ws0[i + 1] : p.nws) - parent_ws0[i];
  std::vector<GenEntry> gen;
  for (size_t pa = 0; pa < parent_ws0.size(); ++pa)
    for (size_t pb = 0; pb <= pa; ++pb) {
      int PA = (int)pa, PB = (int)pb;
      const int la = p.ws_info[parent_ws0[PA]].y, lb = p.ws_info[parent_ws0[PB]].y;
      if (p.ws_info[parent_ws0[PA]].z != p.ws_info[parent_ws0[PB]].z) continue;  // other molecule
      if (lb > la) std::swap(PA, PB);
      if (std::min(la, lb) != 0) continue;  // grouped lists hold pair classes (l, 0) only
      const int nca = parent_nc[PA], ncb = parent_nc[PB];
      GenEntry base{};
      base.cls = pair_class(std::max(la, lb), 0);
      base.mol = p.ws_info[parent_ws0[PA]].z;
      base.diag = PA == PB;
      base.pkey = (long long)std::max(p.ws_parent[parent_ws0[PA]], p.ws_parent[parent_ws0[PB]]) * parent_base[nmol] +
                  std::min(p.ws_parent[parent_ws0[PA]], p.ws_parent[parent_ws0[PB]]);
      if (nca * ncb == 1) {
        int A = parent_ws0[PA], B = parent_ws0[PB];
        auto it = ws_pair_id.find(ws_key(A, B));
        if (it == ws_pair_id.end()) continue;  // every primitive pair screened out
        base.pair = it->second;
        base.nco = 1;
        const int4 pi = p.pair_info[base.pair];
        base.ws[0] = pi.x;
        base.wsb[0] = pi.y;
        base.ppoff = pi.z;
        base.npp = pi.w;
        gen.push_back(base);
        continue;
      }
      // ordered combinations (column of A, column of B), cut into runs of
      // 4 (pair class (0,0)) or 2, then 2, then 1
      std::vector<int2> combos;
      for (int ca = 0; ca < nca; ++ca)
        for (int cb = 0; cb < ncb; ++cb) combos.push_back(make_int2(ca, cb));
      const int gmax = base.cls == 0 ? 4 : 2;
      size_t c0 = 0;
      while (c0 < combos.size()) {
        const size_t rem = combos.size() - c0;
        const int g = rem >= (size_t)gmax ? gmax : (rem >= 2 ? 2 : 1);
        GenEntry e = base;
        e.pair = -1;
        e.nco = g;
        const int A0 = parent_ws0[PA], B0 = parent_ws0[PB];
        for (int k = 0; k < g; ++k) {
          e.ws[k] = A0 + combos[c0 + k].x;
          e.wsb[k] = B0 + combos[c0 + k].y;
        }
        const double4 ra = p.ws_xyz[A0], rb = p.ws_xyz[B0];
        const double ab2 = (ra.x - rb.x) * (ra.x - rb.x) + (ra.y - rb.y) * (ra.y - rb.y) +
                           (ra.z - rb.z) * (ra.z - rb.z);
        e.ppoff = (int)pp_data.size();
        for (int ia = 0; ia < p.ws_nprim[A0]; ++ia)
          for (int ib = 0; ib < p.ws_nprim[B0]; ++ib) {
            const double a = p.ws_exp[p.ws_prim_off[A0] + ia], b = p.ws_exp[p.ws_prim_off[B0] + ib];
            const double pe = a + b;
            const double expo = a * b / pe * ab2;
            if (expo > 40.0) continue;
            double c[4] = {0.0, 0.0, 0.0, 0.0};
            bool any = false;
            for (int k = 0; k < g; ++k) {
              c[k] = p.ws_coef[p.ws_prim_off[e.ws[k]] + ia] * p.ws_coef[p.ws_prim_off[e.wsb[k]] + ib];
              any = any || c[k] != 0.0;
            }
            if (!any) continue;
            double kk = std::exp(-expo) / pe;
            if (g == 1) {  // a lone combination keeps its coefficient in K
              kk *= c[0];
              c[0] = 1.0;
            }
            const double4 P = make_double4((a * ra.x + b * rb.x) / pe, (a * ra.y + b * rb.y) / pe,
                                           (a * ra.z + b * rb.z) / pe, pe);
            pp_data.push_back(P);
            pp_aux.push_back(make_double2(kk, 0.5 / pe));
            pp_exp.push_back(make_double2(a, b));
            pp_f.push_back(make_float4(float(P.x - ra.x), float(P.y - ra.y), float(P.z - ra.z), float(pe)));
            pp_f2.push_back(make_float2(float(kk), float(0.5 / pe)));
            pp_c.push_back(make_double4(c[0], c[1], c[2], c[3]));
          }
        e.npp = (int)pp_data.size() - e.ppoff;
        if (e.npp > 0) gen.push_back(e);
        c0 += g;
      }
    }
  // ---- device upload
  upload(p.d_ws_info, p.ws_info.data(), p.ws_info.size() * sizeof(int4));
  upload(p.d_ws_xyz, p.ws_xyz.data(), p.ws_xyz.size() * sizeof(double4));
  upload(p.d_pair_info, p.pair_info.data(), p.pair_info.size() * sizeof(int4));
  upload(p.d_pp_data, pp_data.data(), pp_data.size() * sizeof(double4));
  upload(p.d_pp_aux, pp_aux.data(), pp_aux.size() * sizeof(double2));
  upload(p.d_pp_exp, pp_exp.data(), pp_exp.size() * sizeof(double2));
  upload(p.d_pp_f, pp_f.data(), pp_f.size() * sizeof(float4));
  upload(p.d_pp_f2, pp_f2.data(), pp_f2.size() * sizeof(float2));
  {
    std::vector<float4> pp_cf(pp_c.size());
    for (size_t i = 0; i < pp_c.size(); ++i)
      pp_cf[i] = make_float4(float(pp_c[i].x), float(pp_c[i].y), float(pp_c[i].z), float(pp_c[i].w));
    upload(p.d_pp_c, pp_c.data(), pp_c.size() * sizeof(double4));
    upload(p.d_pp_cf, pp_cf.data(), pp_cf.size() * sizeof(float4));
  }
  upload(p.d_mol_base_cart, p.mol_cart_base.data(), nmol * sizeof(long long));
  upload(p.d_mol_ncart, p.mol_ncart.data(), nmol * sizeof(int));
  upload(p.d_mol_base_out, p.mol_out_base.data(), nmol * sizeof(long long));
  upload(p.d_mol_nout, p.mol_nout.data(), nmol * sizeof(int));
  {
    std::vector<int> cart_ws, out_ws;
    for (int w = 0; w < p.nws; ++w) {
      const int l = p.ws_info[w].y;
      for (int c = 0; c < ncart_of(l); ++c) cart_ws.push_back(w);
      for (int c = 0; c < (cart ? ncart_of(l) : 2 * l + 1); ++c) out_ws.push_back(w);
    }
    upload(p.d_cart_ws, cart_ws.data(), cart_ws.size() * sizeof(int));
    upload(p.d_out_ws, out_ws.data(), out_ws.size() * sizeof(int));
  }
  upload(p.d_atoms, p.atom_xyzq.data(), p.atom_xyzq.size() * sizeof(double4));
  upload(p.d_ws_atm, p.ws_atm.data(), p.ws_atm.size() * sizeof(int));
  {
    std::vector<double2> ec(p.ws_exp.size());
    for (size_t i = 0; i < ec.size(); ++i) ec[i] = make_double2(p.ws_exp[i], p.ws_coef[i]);
    upload(p.d_ws_prim, ec.data(), ec.size() * sizeof(double2));
    std::vector<int> off = p.ws_prim_off;
    off.push_back((int)p.ws_exp.size());
    upload(p.d_ws_prim_off, off.data(), off.size() * sizeof(int));
    upload(p.d_mol_atm, p.mol_atm_off.data(), nmol * sizeof(int));
    upload(p.d_mol_natm, p.mol_natm.data(), nmol * sizeof(int));
  }
  CUDA_OK(p.d_status.ensure(sizeof(int)));
  CUDA_OK(cudaMemset(p.d_status.ptr, 0, sizeof(int)));
  CUDA_OK(p.d_maxd.ensure(sizeof(double)));
  // ---- Schwarz bounds on the device, one launch per pair class
  std::vector<std::vector<int>> by_class(kPairClasses);
  for (int q = 0; q < p.npair; ++q) by_class[p.pair_class[q]].push_back(q);
  for (int c = 0; c < kPairClasses; ++c) {
    p.n_all_pairs[c] = (int)by_class[c].size();
    if (p.n_all_pairs[c]) upload(p.d_all_pairs[c], by_class[c].data(), by_class[c].size() * sizeof(int));
  }
  // molecule AO starts (global Cartesian / output AO index) for the transforms
  {
    std::vector<int> v(2 * nmol);
    int c = 0, o = 0;
    for (int m = 0; m < nmol; ++m) {
      v[m] = c;
      v[nmol + m] = o;
      c += p.mol_ncart[m];
      o += p.mol_nout[m];
    }
    upload(p.d_mol_ao_off, v.data(), v.size() * sizeof(int));
    CUDA_OK(p.d_rowmax.ensure((size_t)std::max(c, 1) * sizeof(double)));
  }
  CUDA_OK(p.d_q_work.ensure(std::max(p.npair, 1) * sizeof(double)));
  {
    std::vector<DevBuf> lists(kPairClasses);
    for (int c = 0; c < kPairClasses; ++c) {
      if (by_class[c].empty()) continue;
      upload(lists[c], by_class[c].data(), by_class[c].size() * sizeof(int));
      JKArgs a = base_args(p);
      a.bra_pairs = lists[c].as<int>();
      a.q_out = p.d_q_work.as<double>();
      const int rc = dispatch().schwarz[c](a, (int)by_class[c].size(), cart, 0);
      if (rc) throw Failure{B200JK_INTERNAL, std::string("Schwarz launch failed: ") + cudaGetErrorString((cudaError_t)rc)};
    }
    CUDA_OK(cudaDeviceSynchronize());
  }
  std::vector<double> qw(p.npair);
  if (p.npair) CUDA_OK(cudaMemcpy(qw.data(), p.d_q_work.ptr, p.npair * sizeof(double), cudaMemcpyDeviceToHost));
  // parent-pair bound: max over the work pairs of the parent pair
  // (parent key max * nparent + min)
  const long long npar = (long long)parent_base[nmol];
  std::unordered_map<long long, double> parent;
  parent.reserve(2 * (size_t)p.npair + 1);
  auto pkey = [&](int q) {
    int a = p.ws_parent[p.pair_info[q].x], b = p.ws_parent[p.pair_info[q].y];
    if (a < b) std::swap(a, b);
    return (long long)a * npar + b;
  };
  for (int q = 0; q < p.npair; ++q) {
    auto k = pkey(q);
    auto it = parent.find(k);
    if (it == parent.end()) parent[k] = qw[q];
    else it->second = std::max(it->second, qw[q]);
  }
  p.pair_q.resize(p.npair);
  std::vector<double> qmax_mol(nmol, 0.0);
  for (int q = 0; q < p.npair; ++q) {
    p.pair_q[q] = std::sqrt(parent[pkey(q)]);
    const int m = p.ws_info[p.pair_info[q].x].z;
    qmax_mol[m] = std::max(qmax_mol[m], p.pair_q[q]);
  }
  // ---- class lists: significant pairs sorted by (molecule, Q desc, id)
  for (int c = 0; c < kPairClasses; ++c) {
    ClassList& L = p.classes[c];
    std::vector<int> ids;
    for (int q : by_class[c]) {
      const int m = p.ws_info[p.pair_info[q].x].z;
      if (cut > 0 && p.pair_q[q] * qmax_mol[m] < cut) continue;  // coulomb_shells.h:203
      ids.push_back(q);
    }
    // Order: molecule, then primitive-pair count (so a warp's kets share
    // their contraction length), then Q descending (screening prefix).
    std::sort(ids.begin(), ids.end(), [&](int a, int b) {
      const int ma = p.ws_info[p.pair_info[a].x].z, mb = p.ws_info[p.pair_info[b].x].z;
      if (ma != mb) return ma < mb;
      if (p.pair_info[a].w != p.pair_info[b].w) return p.pair_info[a].w < p.pair_info[b].w;
      if (p.pair_q[a] != p.pair_q[b]) return p.pair_q[a] > p.pair_q[b];
      return a < b;
    });
    L.pairs = ids;
    L.q.resize(ids.size());
    for (size_t i = 0; i < ids.size(); ++i) L.q[i] = p.pair_q[ids[i]];
    L.npp_prefix.assign(ids.size() + 1, 0);
    for (size_t i = 0; i < ids.size(); ++i) L.npp_prefix[i + 1] = L.npp_prefix[i] + p.pair_info[ids[i]].w;
    L.npp_pos.resize(ids.size());
    L.mol_pos.resize(ids.size());
    for (size_t i = 0; i < ids.size(); ++i) {
      L.npp_pos[i] = p.pair_info[ids[i]].w;
      L.mol_pos[i] = p.ws_info[p.pair_info[ids[i]].x].z;
    }
    L.mol_begin.assign(nmol + 1, 0);
    for (int q : ids) L.mol_begin[p.ws_info[p.pair_info[q].x].z + 1]++;
    for (int m = 0; m < nmol; ++m) L.mol_begin[m + 1] += L.mol_begin[m];
    L.segs.assign(nmol, {});
    for (size_t i = 0; i < ids.size();) {
      size_t j = i + 1;
      const int m = p.ws_info[p.pair_info[ids[i]].x].z;
      while (j < ids.size() && p.ws_info[p.pair_info[ids[j]].x].z == m &&
             p.pair_info[ids[j]].w == p.pair_info[ids[i]].w)
        ++j;
      L.segs[m].push_back(make_int2((int)i, (int)j));
      i = j;
    }
    upload(L.d_pairs, ids.data(), ids.size() * sizeof(int));
    upload(L.d_q, L.q.data(), L.q.size() * sizeof(double));
    std::vector<double4> ra(ids.size()), ab(ids.size());
    std::vector<int4> ix(ids.size());
    for (size_t i = 0; i < ids.size(); ++i) {
      const int4 pi = p.pair_info[ids[i]];
      const double4 a = p.ws_xyz[pi.x], b = p.ws_xyz[pi.y];
      ra[i] = make_double4(a.x, a.y, a.z, (double)p.ws_info[pi.x].z);
      ab[i] = make_double4(a.x - b.x, a.y - b.y, a.z - b.z, 0.0);
      ix[i] = make_int4(pi.z, pi.w, p.ws_info[pi.x].x, p.ws_info[pi.y].x);
    }
    upload(L.d_ra, ra.data(), ra.size() * sizeof(double4));
    upload(L.d_ab, ab.data(), ab.size() * sizeof(double4));
    upload(L.d_ix, ix.data(), ix.size() * sizeof(int4));
    CUDA_OK(L.d_kmax.ensure(std::max<size_t>(ids.size(), 1) * sizeof(double)));
    L.aoa_pos.resize(ids.size());
    for (size_t i = 0; i < ids.size(); ++i) L.aoa_pos[i] = ix[i].z;
    build_bra_order(L);

  }
  // the combinations of the grouped entries cover exactly the expanded
  // work pairs of their classes (checked once per plan, on the host)
  {
    std::vector<long long> want, got;  // (class, work-shell pair) keys
    const long long span = (long long)p.nws * p.nws;
    for (int q = 0; q < p.npair; ++q) {
      const int c = p.pair_class[q];
      if (c == 0 || c == 1 || c == 3 || c == 6) want.push_back(c * span + ws_key(p.pair_info[q].x, p.pair_info[q].y));
    }
    for (const GenEntry& e : gen)
      for (int k = 0; k < e.nco; ++k) got.push_back(e.cls * span + ws_key(e.ws[k], e.wsb[k]));
    std::sort(want.begin(), want.end());
    std::sort(got.begin(), got.end());
    got.erase(std::unique(got.begin(), got.end()), got.end());
    if (!std::includes(got.begin(), got.end(), want.begin(), want.end()))
      throw Failure{B200JK_INTERNAL, "grouped pair list misses a work pair"};
  }
  std::vector<double> gen_q(gen.size());
  for (size_t i = 0; i < gen.size(); ++i) gen_q[i] = std::sqrt(parent[gen[i].pkey]);
  // ---- grouped lists: same screening and order, plus the number of
  // combinations (runs of equal (combinations, primitive pairs) per molecule)
  for (int c = 0; c < kPairClasses; ++c) {
    std::vector<int> ids;
    bool any_gen = false;
    for (size_t i = 0; i < gen.size(); ++i) {
      if (gen[i].cls != c) continue;
      const double q = gen_q[i];
      if (cut > 0 && q * qmax_mol[gen[i].mol] < cut) continue;
      ids.push_back((int)i);
      any_gen = any_gen || gen[i].nco > 1;
    }
    if (!any_gen) continue;  // identical to the expanded list
    auto qof = [&](int i) { return gen_q[i]; };
    std::sort(ids.begin(), ids.end(), [&](int a, int b) {
      const GenEntry &ea = gen[a], &eb = gen[b];
      if (ea.mol != eb.mol) return ea.mol < eb.mol;
      if (ea.nco != eb.nco) return ea.nco < eb.nco;
      if (ea.npp != eb.npp) return ea.npp < eb.npp;
      const double qa = qof(a), qb = qof(b);
      if (qa != qb) return qa > qb;
      return a < b;
    });
    ClassList& L = p.grouped[c];
    const size_t n = ids.size();
    L.pairs.assign(n, -1);
    L.q.resize(n);
    L.nco.resize(n);
    L.npp_pos.resize(n);
    L.mol_pos.resize(n);
    L.npp_prefix.assign(n + 1, 0);
    std::vector<double4> ra(n), ab(n);
    std::vector<int4> ix(n), gx(n), gy(n);
    for (size_t i = 0; i < n; ++i) {
      const GenEntry& e = gen[ids[i]];
      L.pairs[i] = e.pair;
      L.q[i] = qof(ids[i]);
      L.nco[i] = e.nco;
      L.npp_pos[i] = e.npp;
      L.mol_pos[i] = e.mol;
      L.npp_prefix[i + 1] = L.npp_prefix[i] + e.npp;
      const double4 a = p.ws_xyz[e.ws[0]], b = p.ws_xyz[e.wsb[0]];
      ra[i] = make_double4(a.x, a.y, a.z, (double)e.mol);
      ab[i] = make_double4(a.x - b.x, a.y - b.y, a.z - b.z, 0.0);
      int ao[4], bo[4];
      for (int k = 0; k < 4; ++k) {
        ao[k] = k < e.nco ? p.ws_info[e.ws[k]].x : 0;
        bo[k] = k < e.nco ? p.ws_info[e.wsb[k]].x : 0;
      }
      const int diag = e.nco == 1 ? (ao[0] == bo[0]) : e.diag;
      ix[i] = make_int4(e.ppoff, e.npp, ao[0], bo[0]);
      gx[i] = make_int4(diag, 0, ao[1], bo[1]);
      gy[i] = make_int4(ao[2], bo[2], ao[3], bo[3]);
    }
    L.mol_begin.assign(nmol + 1, 0);
    for (size_t i = 0; i < n; ++i) L.mol_begin[L.mol_pos[i] + 1]++;
    for (int m = 0; m < nmol; ++m) L.mol_begin[m + 1] += L.mol_begin[m];
    L.segs.assign(nmol, {});
    for (size_t i = 0; i < n;) {
      size_t j = i + 1;
      while (j < n && L.mol_pos[j] == L.mol_pos[i] && L.nco[j] == L.nco[i] && L.npp_pos[j] == L.npp_pos[i]) ++j;
      L.segs[L.mol_pos[i]].push_back(make_int2((int)i, (int)j));
      i = j;
    }
    upload(L.d_q, L.q.data(), n * sizeof(double));
    upload(L.d_ra, ra.data(), n * sizeof(double4));
    upload(L.d_ab, ab.data(), n * sizeof(double4));
    upload(L.d_ix, ix.data(), n * sizeof(int4));
    upload(L.d_gx, gx.data(), n * sizeof(int4));
    upload(L.d_gy, gy.data(), n * sizeof(int4));
    upload(L.d_nco, L.nco.data(), n * sizeof(int));
    CUDA_OK(L.d_kmax.ensure(std::max<size_t>(n, 1) * sizeof(double)));
    L.aoa_pos.resize(n);
    for (size_t i = 0; i < n; ++i)
      L.aoa_pos[i] = (long long)ix[i].z | ((long long)gx[i].z << 16) | ((long long)gy[i].x << 32) |
                     ((long long)gy[i].z << 48);
    build_bra_order(L);
  }
  // ---- work items per class pair (X >= Y)
  for (int x = 0; x < kPairClasses; ++x)
    for (int y = 0; y <= x; ++y) {
      if (p.classes[x].pairs.empty() || p.classes[y].pairs.empty()) continue;
      auto* W = new ClassPairWork();
      W->x = x;
      W->y = y;
      W->nbra = (int)p.classes[x].pairs.size();
      fill_items(p, *W, 0);
      if (W->nwork == 0) { delete W; continue; }
      p.work.push_back(W);
    }
  // ---- quartet count on the reference's shells (parent pairs, canonical)
  {
    long long total = 0;
    std::vector<std::vector<double>> pq(nmol);
    // parent pair bounds per molecule
    std::unordered_map<long long, char> seen;
    seen.reserve(2 * (size_t)p.npair + 1);
    for (int q = 0; q < p.npair; ++q)
      if (seen.emplace(pkey(q), 1).second) pq[p.ws_info[p.pair_info[q].x].z].push_back(p.pair_q[q]);
    for (int m = 0; m < nmol; ++m) {
      auto& v = pq[m];
      std::sort(v.begin(), v.end(), std::greater<double>());
      for (size_t a = 0; a < v.size(); ++a) {
        if (cut <= 0) { total += (long long)a + 1; continue; }
        // count b <= a (in sorted order) with v[a]*v[b] >= cut: all b < a have v[b] >= v[a]
        size_t lo = 0, hi = a + 1;
        while (lo < hi) {
          const size_t mid = (lo + hi) / 2;
          if (v[a] * v[mid] < cut) hi = mid;
          else lo = mid + 1;
        }
        total += (long long)lo;
      }
    }
    p.quartets = total;
  }
  CUDA_OK(p.d_queue.ensure(kQueueSlots * sizeof(int)));
  for (int i = 0; i < kAuxStreams; ++i) {
    CUDA_OK(cudaStreamCreateWithFlags(&p.aux[i], cudaStreamNonBlocking));
    CUDA_OK(cudaEventCreateWithFlags(&p.join_ev[i], cudaEventDisableTiming));
  }
  CUDA_OK(cudaEventCreateWithFlags(&p.fork_ev, cudaEventDisableTiming));
  return plan.release();
}

}  // namespace b200jk
#include "one_electron.h"
namespace b200jk {

static OneArgs one_args(const Plan& p) {
  OneArgs a{};
  a.pair_info = p.d_pair_info.as<int4>();
  a.ws_info = p.d_ws_info.as<int4>();
  a.ws_xyz = p.d_ws_xyz.as<double4>();
  a.prim = p.d_ws_prim.as<double2>();
  a.prim_off = p.d_ws_prim_off.as<int>();
  a.atoms = p.d_atoms.as<double4>();
  a.mol_atm_off = p.d_mol_atm.as<int>();
  a.mol_natm = p.d_mol_natm.as<int>();
  a.mol_base = p.d_mol_base_cart.as<long long>();
  a.mol_n = p.d_mol_ncart.as<int>();
  a.ws_atm = p.d_ws_atm.as<int>();
  a.tb = plan_tables(p);
  return a;
}

// ---------------------------------------------------------------- J/K execution
static void ensure_scratch(Plan& p, int nb) {
  if (p.scratch_nb >= nb) return;
  CUDA_OK(p.d_dens.ensure((size_t)2 * nb * p.cart_stride * sizeof(double)));
  CUDA_OK(p.d_vj.ensure((size_t)nb * p.cart_stride * sizeof(double)));
  CUDA_OK(p.d_vk.ensure((size_t)2 * nb * p.cart_stride * sizeof(double)));
  CUDA_OK(p.d_dens_f.ensure((size_t)2 * nb * p.cart_stride * sizeof(float)));
  p.scratch_nb = nb;
}

static int max_nc(const Plan& p) { return *std::max_element(p.mol_ncart.begin(), p.mol_ncart.end()); }
static int max_no(const Plan& p) { return *std::max_element(p.mol_nout.begin(), p.mol_nout.end()); }

void check_jk_args(const Plan& p, const double* d_in, int nb, const double* d_out, int with_j,
                   int with_k, int precision, double fp32_cut) {
  (void)p;
  if (nb < 1) invalid("Direct J/K requires at least one density");
  if ((with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) || !(with_j || with_k))
    invalid("Direct J/K requires at least one selected operator");
  if (precision != B200JK_FP64 && precision != B200JK_SPLIT) invalid("Unknown precision mode");
  if (precision == B200JK_SPLIT && !(fp32_cut >= 0 && std::isfinite(fp32_cut))) invalid("Invalid fp32_cut");
  if (!d_in || !d_out) invalid("Null density or output pointer");
}

// The FP32/FP64 boundary of every item of class pair W (split mode); the
// row maxima of the effective densities are in p.d_rowmax.
static void split_units(Plan& p, ClassPairWork& W, double fp32_cut, cudaStream_t st) {
  const int la = pc_la_host(W.x), lb = W.x - la * (la + 1) / 2, lc = pc_la_host(W.y);
  for_each_unit(p, W, [&](const JKUnit& u) {
    if (u.nwork == 0) return;  // nothing of this class pair on this shard
    (void)lc;
    if (u.grp) {
      grp_split_kernel<<<(u.nwork + 3) / 4, 128, 0, st>>>(
          u.work->as<int4>(), u.nwork, u.X->d_bord.as<int>(), u.X->d_ix.as<int4>(), u.X->d_gx.as<int4>(),
          u.X->d_gy.as<int4>(), u.gb, u.X->d_ra.as<double4>(),
          u.Y->d_kmax.as<double>(), p.d_rowmax.as<double>(), p.d_mol_ao_off.as<int>(), ncart_of(la),
          ncart_of(lb), u.split->as<double>());
      CUDA_OK(cudaGetLastError());
      if (u.grp->flat_cap > 0 && dispatch().flat64[quartet_class(W.x, W.y)][gen_slot(u.gb, u.gk)]) {
        CUDA_OK(cudaMemsetAsync(u.grp->flat_n.ptr, 0, sizeof(unsigned long long), st));
        border_kernel<<<(u.nwork + 3) / 4, 128, 0, st>>>(
            u.work->as<int4>(), u.nwork, u.X->d_bord.as<int>(), u.X->d_q.as<double>(), u.Y->d_q.as<double>(),
            u.split->as<double>(), W.x == W.y, p.cutoff, fp32_cut, u.grp->flat.as<int2>(),
            u.grp->flat_n.as<unsigned long long>(), u.grp->flat_cap, u.grp->skip.as<int>());
        CUDA_OK(cudaGetLastError());
      }
      return;
    }
    SplitLists L{u.X->d_ix.as<int4>(), u.X->d_gx.as<int4>(), u.X->d_gy.as<int4>(), u.Y->d_kmax.as<double>(),
                 u.X->d_ra.as<double4>(), u.gb, ncart_of(la), ncart_of(lb)};
    split_kernel<<<(u.nwork + 3) / 4, 128, 0, st>>>(u.work->as<int4>(), u.X->d_q.as<double>(),
                                                       u.Y->d_q.as<double>(), p.d_rowmax.as<double>(),
                                                       p.d_mol_ao_off.as<int>(), L, fp32_cut, u.nwork,
                                                       u.split->as<int>());
    CUDA_OK(cudaGetLastError());
  });
}

// The J/K kernels of class pair W (both slices in split mode), on the
// densities and accumulators already set in `a`.
// `only`: -1 launches every slice of `precision`; 1 only the FP64 slice and
// 2 only the FP32 slice of a split build.
static void launch_units(Plan& p, ClassPairWork& W, JKArgs a, int precision, cudaStream_t st,
                         bool allow_profiling, int only = -1) {
  const auto& disp = dispatch();
  const int cls = quartet_class(W.x, W.y);
  for_each_unit(p, W, [&](const JKUnit& u) {
    if (u.nwork == 0) return;
    set_unit_lists(a, u, W.x == W.y);
    a.work = u.work->as<int4>();
    a.nwork = u.nwork;
    a.split = u.grp ? nullptr : u.split->as<int>();
    a.item_m = u.grp ? u.split->as<double>() : nullptr;
    const bool plain = u.gb == 1 && u.gk == 1;
    const int gs = gen_slot(u.gb, u.gk);
    const JKLauncher l64 = u.grp ? (plain ? disp.grp64[cls] : disp.grpg64[cls][gs])
                                 : (plain ? disp.jk64[cls] : disp.jkg64[cls][gs]);
    const JKLauncher l32 = u.grp ? (plain ? disp.grp32[cls] : disp.grpg32[cls][gs])
                                 : (plain ? disp.jk32[cls] : disp.jkg32[cls][gs]);
    if (!l64 || !l32) throw Failure{B200JK_INTERNAL, "no kernel for this contraction grouping"};
    const JKLauncher lflat = u.grp ? disp.flat64[cls][gs] : nullptr;
    auto launch = [&](int mode, bool fp32) {
      a.split_mode = mode;
      // the FP64 slice of a split build: the flat list first, then the
      // bra-group items it does not hold
      const bool flat = mode == 1 && lflat && u.grp->flat_cap > 0;
      a.flat = flat ? u.grp->flat.as<int2>() : nullptr;
      a.flat_n = flat ? u.grp->flat_n.as<unsigned long long>() : nullptr;
      a.flat_cap = flat ? u.grp->flat_cap : 0;
      a.item_skip = flat ? u.grp->skip.as<int>() : nullptr;
      if (u.grp) {
        // a zeroed work-queue counter of its own (slots cycle over the plan's pool)
        int* q = p.d_queue.as<int>() + (p.next_queue++ % kQueueSlots);
        CUDA_OK(cudaMemsetAsync(q, 0, sizeof(int), st));
        a.queue = q;
      }
      ProfileEvent ev{cls, fp32 ? 1 : 0, nullptr, nullptr};
      if (p.profiling && allow_profiling) {
        CUDA_OK(cudaEventCreate(&ev.start));
        CUDA_OK(cudaEventCreate(&ev.stop));
        CUDA_OK(cudaEventRecord(ev.start, st));
      }
      int rc = flat ? lflat(a, st) : 0;
      if (rc == 0) rc = fp32 ? l32(a, st) : l64(a, st);
      if (rc) throw Failure{B200JK_INTERNAL, std::string("J/K launch failed: ") + cudaGetErrorString((cudaError_t)rc)};
      if (p.profiling && allow_profiling) {
        CUDA_OK(cudaEventRecord(ev.stop, st));
        p.events.push_back(ev);
      }
    };
    if (precision == B200JK_FP64) {
      launch(0, false);
    } else {
      if (only != 2) launch(1, false);
      if (only != 1) launch(2, true);
    }
  });
}

// Primitive quartets a class pair's J/K launches evaluate (scheduling weight).
static long long jk_cost(const ClassPairWork& W) {
  if (W.buckets.empty()) return W.prim_quartets;
  long long c = 0;
  for (const auto* B : W.buckets) c += B->prim_quartets;
  return c;
}

// The class-pair launches of one build spread over the caller's stream and
// the plan's auxiliary streams (forked from and joined back into `st`): the
// launches are independent (J/K accumulate atomically), so their tails and
// low-occupancy kernels overlap.  Longest-first onto the least-loaded
// stream; in split builds the FP64 slices share one auxiliary stream.
static void launch_all(Plan& p, JKArgs a, int precision, cudaStream_t st) {
  CUDA_OK(cudaEventRecord(p.fork_ev, st));
  for (int i = 0; i < kAuxStreams; ++i) CUDA_OK(cudaStreamWaitEvent(p.aux[i], p.fork_ev, 0));
  cudaStream_t streams[kAuxStreams + 1] = {st};
  for (int i = 0; i < kAuxStreams; ++i) streams[i + 1] = p.aux[i];
  std::vector<std::pair<long long, ClassPairWork*>> order;
  for (auto* W : p.work) order.push_back({jk_cost(*W), W});
  std::sort(order.begin(), order.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  const bool split = precision == B200JK_SPLIT;  // split builds: stream 1 carries the FP64 slices
  std::vector<long long> load(kAuxStreams + 1, 0);
  for (auto& [cost, W] : order) {
    int best = -1;
    for (int i = 0; i <= kAuxStreams; ++i) {
      if (split && i == 1) continue;
      if (best < 0 || load[i] < load[best]) best = i;
    }
    load[best] += cost;
    launch_units(p, *W, a, precision, streams[best], false, split ? 2 : -1);
    if (split) launch_units(p, *W, a, precision, streams[1], false, 1);
  }
  for (int i = 0; i < kAuxStreams; ++i) {
    CUDA_OK(cudaEventRecord(p.join_ev[i], p.aux[i]));
    CUDA_OK(cudaStreamWaitEvent(st, p.join_ev[i], 0));
  }
}

// The J/K pipeline on caller-provided scratch: dens/dens_f hold (hermi ? nb :
// 2nb) Cartesian matrices, vj nb, vk (hermi ? nb : 2nb); nothing is allocated
// here when profiling is off.
// Densities in (output basis) -> raw Cartesian effective densities (status
// word flags a nonfinite density); J/K accumulators zeroed.
static void jk_prologue(Plan& p, const double* d_in, int nb, int hermi, int with_j, int with_k,
                        cudaStream_t st, double* s_dens, double* s_vj, double* s_vk) {
  const int ndm = hermi ? nb : 2 * nb;
  const Tables tb = plan_tables(p);
  const int nc = max_nc(p);
  const long long n2 = (long long)nc * nc;
  dim3 grid((unsigned)((n2 + 255) / 256), p.nmol, nb);
  density_in_kernel<<<grid, 256, 0, st>>>(
      d_in, nb, hermi, s_dens, p.out_stride, p.cart_stride,
      p.d_mol_base_out.as<long long>(), p.d_mol_nout.as<int>(), p.d_mol_base_cart.as<long long>(),
      p.d_mol_ncart.as<int>(), p.d_cart_ws.as<int>(), p.d_ws_info.as<int4>(), p.d_mol_ao_off.as<int>(), tb.c2s,
      p.d_status.as<int>());
  CUDA_OK(cudaGetLastError());
  if (with_j) CUDA_OK(cudaMemsetAsync(s_vj, 0, (size_t)nb * p.cart_stride * sizeof(double), st));
  if (with_k) CUDA_OK(cudaMemsetAsync(s_vk, 0, (size_t)ndm * p.cart_stride * sizeof(double), st));
}

// MJ/MK accumulators -> J/K in the output basis (d_out fully overwritten).
static void jk_epilogue(Plan& p, int nb, int hermi, int with_j, int with_k, double* d_out, cudaStream_t st,
                        const double* s_vj, const double* s_vk) {
  const Tables tb = plan_tables(p);
  const int no = max_no(p);
  const long long n2 = (long long)no * no;
  dim3 grid((unsigned)((n2 + 255) / 256), p.nmol, nb);
  jk_out_kernel<<<grid, 256, 0, st>>>(
      s_vj, s_vk, nb, hermi, with_j, with_k, d_out, p.out_stride,
      p.cart_stride, p.d_mol_base_out.as<long long>(), p.d_mol_nout.as<int>(),
      p.d_mol_base_cart.as<long long>(), p.d_mol_ncart.as<int>(), p.d_out_ws.as<int>(),
      p.d_ws_info.as<int4>(), p.d_mol_ao_off.as<int>() + p.nmol, tb.c2s);
  CUDA_OK(cudaGetLastError());
}

void run_jk_core(Plan& p, const double* d_in, int nb, double* d_out, int with_j, int with_k,
                 int hermi, int precision, double fp32_cut, cudaStream_t st, double* s_dens,
                 float* s_dens_f, double* s_vj, double* s_vk, bool allow_profiling) {
  const int ndm = hermi ? nb : 2 * nb;
  jk_prologue(p, d_in, nb, hermi, with_j, with_k, st, s_dens, s_vj, s_vk);
  if (precision == B200JK_SPLIT) {
    to_float_kernel<<<592, 256, 0, st>>>(s_dens, s_dens_f,
                                         (long long)ndm * p.cart_stride);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaMemsetAsync(p.d_maxd.ptr, 0, sizeof(double), st));
    maxabs_kernel<<<592, 256, 0, st>>>(d_in, (long long)nb * p.out_stride, p.d_maxd.as<double>());
    CUDA_OK(cudaGetLastError());
    const int nrows = (int)(p.d_rowmax.bytes / sizeof(double));
    rowmax_kernel<<<(nrows + 7) / 8, 256, 0, st>>>(s_dens, ndm, p.cart_stride, p.d_mol_base_cart.as<long long>(),
                                                  p.d_mol_ncart.as<int>(), p.d_mol_ao_off.as<int>(),
                                                  p.d_cart_ws.as<int>(), p.d_ws_info.as<int4>(), nrows,
                                                  p.d_rowmax.as<double>());
    CUDA_OK(cudaGetLastError());
    for (int c = 0; c < kPairClasses; ++c)
      for (ClassList* Lp : {&p.classes[c], &p.grouped[c]}) {
        const int npos = (int)Lp->q.size();
        if (npos == 0) continue;
        posmax_kernel<<<(npos + 127) / 128, 128, 0, st>>>(
            Lp->d_ix.as<int4>(), Lp->d_gx.as<int4>(), Lp->d_gy.as<int4>(), Lp->d_nco.as<int>(),
            Lp->d_ra.as<double4>(), npos, ncart_of(pc_la_host(c)), p.d_rowmax.as<double>(),
            p.d_mol_ao_off.as<int>(), Lp->d_kmax.as<double>());
        CUDA_OK(cudaGetLastError());
      }
    for (auto* W : p.work) split_units(p, *W, fp32_cut, st);
    p.last_fp32_cut = fp32_cut;
  }
  JKArgs a = base_args(p);
  a.dens = s_dens;
  a.dens_f = s_dens_f;
  a.vj = s_vj;
  a.vk = s_vk;
  a.dstride = p.cart_stride;
  a.ndm = ndm;
  a.nsym = nb;
  a.with_j = with_j;
  a.with_k = with_k;
  a.fp32_cut = fp32_cut;
  if (p.profiling && allow_profiling) {
    // serial, so that every class-pair launch is timed alone
    for (auto* W : p.work) launch_units(p, *W, a, precision, st, true);
  } else {
    launch_all(p, a, precision, st);
  }
  jk_epilogue(p, nb, hermi, with_j, with_k, d_out, st, s_vj, s_vk);
}

static void run_jk(Plan& p, const double* d_in, int nb, double* d_out, int with_j, int with_k,
                   int hermi, int precision, double fp32_cut, cudaStream_t st) {
  check_jk_args(p, d_in, nb, d_out, with_j, with_k, precision, fp32_cut);
  CUDA_OK(cudaSetDevice(p.device));
  ensure_scratch(p, nb);
  run_jk_core(p, d_in, nb, d_out, with_j, with_k, hermi, precision, fp32_cut, st, p.d_dens.as<double>(),
              p.d_dens_f.as<float>(), p.d_vj.as<double>(), p.d_vk.as<double>(), true);
}

template <typename F>
static int guarded(F&& f) {
  try {
    f();
    g_error.clear();
    return B200JK_OK;
  } catch (const Failure& e) {
    g_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_error = "host allocation failed";
    return B200JK_INTERNAL;
  } catch (const std::exception& e) {
    g_error = e.what();
    return B200JK_INTERNAL;
  }
}

int guarded_call(const std::function<void()>& f) { return guarded(f); }
void fail_invalid(const std::string& m) { invalid(m); }

}  // namespace b200jk

using namespace b200jk;

extern "C" {

const char* b200jk_last_error(void) { return g_error.c_str(); }

int b200jk_plan_create(const b200jk_molecule* mols, int32_t nmol, int32_t cart, double schwarz_cut,
                       int32_t device, b200jk_plan** out) {
  return guarded([&] {
    if (!out) invalid("Null output handle");
    *out = nullptr;
    Plan* p = build_plan(mols, nmol, cart, schwarz_cut, device);
    *out = new b200jk_plan{p};
  });
}

void b200jk_plan_destroy(b200jk_plan* plan) {
  if (!plan) return;
  cudaSetDevice(plan->p->device);
  delete plan->p;
  delete plan;
}

int b200jk_plan_nao(const b200jk_plan* plan, int32_t mol, int32_t* nao) {
  return guarded([&] {
    if (!plan || !nao || mol < 0 || mol >= plan->p->nmol) invalid("Invalid plan query");
    *nao = plan->p->mol_nout[mol];
  });
}

int b200jk_plan_quartets(const b200jk_plan* plan, int64_t* count) {
  return guarded([&] {
    if (!plan || !count) invalid("Invalid plan query");
    *count = plan->p->quartets;
  });
}

int b200jk_plan_block_offsets(const b200jk_plan* plan, int64_t* offsets) {
  return guarded([&] {
    if (!plan || !offsets) invalid("Invalid plan query");
    for (int m = 0; m < plan->p->nmol; ++m) offsets[m] = plan->p->mol_out_base[m];
  });
}

int b200jk_direct_jk(b200jk_plan* plan, const double* d_density, int32_t nb, double* d_out,
                     int32_t with_j, int32_t with_k, int32_t hermi, int32_t precision,
                     double fp32_cut, void* stream) {
  return guarded([&] {
    if (!plan) invalid("Null plan");
    run_jk(*plan->p, d_density, nb, d_out, with_j, with_k, hermi ? 1 : 0, precision, fp32_cut,
           (cudaStream_t)stream);
  });
}

// A captured build owns its scratch (effective densities, J/K accumulators),
// so later calls on the plan with more densities, which grow the plan's own
// scratch, leave the graph's pointers valid.  The plan's work-item arrays are
// shared: the graph records their generation and refuses to replay once
// autotune or set_shard has rebuilt them.
struct b200jk_graph {
  b200jk_plan* plan = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long layout_gen = 0;
  DevBuf dens, dens_f, vj, vk;
};

int b200jk_graph_create(b200jk_plan* plan, const double* d_density, int32_t nb, double* d_out,
                        int32_t with_j, int32_t with_k, int32_t hermi, int32_t precision,
                        double fp32_cut, b200jk_graph** out) {
  return guarded([&] {
    if (!plan || !out) invalid("Null plan or output handle");
    *out = nullptr;
    Plan& p = *plan->p;
    check_jk_args(p, d_density, nb, d_out, with_j, with_k, precision, fp32_cut);
    CUDA_OK(cudaSetDevice(p.device));
    std::unique_ptr<b200jk_graph> g(new b200jk_graph());
    g->plan = plan;
    const size_t cs = (size_t)p.cart_stride, ndm = hermi ? (size_t)nb : 2 * (size_t)nb;
    CUDA_OK(g->dens.ensure(ndm * cs * sizeof(double)));
    CUDA_OK(g->dens_f.ensure(ndm * cs * sizeof(float)));
    CUDA_OK(g->vj.ensure((size_t)nb * cs * sizeof(double)));
    CUDA_OK(g->vk.ensure(ndm * cs * sizeof(double)));
    cudaStream_t st;
    CUDA_OK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    auto build = [&] {
      run_jk_core(p, d_density, nb, d_out, with_j, with_k, hermi ? 1 : 0, precision, fp32_cut, st,
                  g->dens.as<double>(), g->dens_f.as<float>(), g->vj.as<double>(), g->vk.as<double>(),
                  false);
    };
    // one eager build first: first-use kernel attributes are set outside capture
    try {
      build();
    } catch (...) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
      throw;
    }
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      build();
    } catch (...) {
      cudaStreamEndCapture(st, &g->graph);
      if (g->graph) cudaGraphDestroy(g->graph);
      g->graph = nullptr;
      cudaStreamDestroy(st);
      throw;
    }
    CUDA_OK(cudaStreamEndCapture(st, &g->graph));
    cudaStreamDestroy(st);
    const cudaError_t e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g->graph);
      g->graph = nullptr;
      throw Failure{B200JK_INTERNAL, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
    }
    g->layout_gen = p.layout_gen;
    *out = g.release();
  });
}

int b200jk_graph_launch(b200jk_graph* g, void* stream) {
  return guarded([&] {
    if (!g) invalid("Null graph");
    if (g->layout_gen != g->plan->p->layout_gen)
      invalid("The plan's work items were rebuilt (autotune or set_shard) after this graph was "
              "captured; destroy the graph and create a new one");
    CUDA_OK(cudaSetDevice(g->plan->p->device));
    CUDA_OK(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  });
}

void b200jk_graph_destroy(b200jk_graph* g) {
  if (!g) return;
  cudaSetDevice(g->plan->p->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
}

int b200jk_check_status(b200jk_plan* plan, void* stream) {
  return guarded([&] {
    if (!plan) invalid("Null plan");
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    CUDA_OK(cudaStreamSynchronize((cudaStream_t)stream));
    int st = 0;
    CUDA_OK(cudaMemcpy(&st, p.d_status.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemset(p.d_status.ptr, 0, sizeof(int)));
    if (st & 1) invalid("Nonfinite density");
    if (st) throw Failure{B200JK_INTERNAL, "device status " + std::to_string(st)};
  });
}

int b200jk_direct_jk_tables(const int32_t* atm, int32_t natm, const int32_t* bas, int32_t nbas,
                            const double* env, int32_t nenv, const double* d_density, int32_t nb,
                            int32_t n, double* d_out, int32_t cart, double cutoff, int32_t workers,
                            int32_t with_j, int32_t with_k, void* stream) {
  return guarded([&] {
    // the handler's order of checks (csrc/direct_jk.cc:15-24): workers,
    // operator flags, tables, shapes, then the density values
    if (workers < 1) invalid("Direct J/K workers must be positive");
    if ((with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) || !(with_j || with_k))
      invalid("Direct J/K requires at least one selected operator");
    int dev = 0;
    CUDA_OK(cudaGetDevice(&dev));
    b200jk_molecule m{atm, natm, bas, nbas, env, nenv};
    std::unique_ptr<Plan> p(build_plan(&m, 1, cart, cutoff, dev));
    if (nb < 0 || n != p->mol_nout[0]) invalid("Direct J/K shape mismatch");
    if (nb == 0) return;  // an empty batch: the handler writes nothing either
    run_jk(*p, d_density, nb, d_out, with_j, with_k, 0, B200JK_FP64, 0.0, (cudaStream_t)stream);
    CUDA_OK(cudaStreamSynchronize((cudaStream_t)stream));
    int st = 0;
    CUDA_OK(cudaMemcpy(&st, p->d_status.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    if (st & 1) invalid("Nonfinite density");
  });
}

int b200jk_partition_items(const int64_t* cost, int64_t n, int32_t world, int32_t* owner) {
  return guarded([&] {
    if (n < 0 || world < 1 || (n > 0 && (!cost || !owner))) invalid("Invalid partition request");
    long double total = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (cost[i] < 0) invalid("Negative work-item cost");
      total += (long double)cost[i];
    }
    // contiguous blocks: item i goes to the rank that owns the midpoint of
    // its cost interval in [0, total)
    long double before = 0;
    for (int64_t i = 0; i < n; ++i) {
      int r;
      if (total > 0) r = (int)((before + 0.5L * (long double)cost[i]) * world / total);
      else r = (int)((i * (int64_t)world) / n);
      owner[i] = std::min(std::max(r, 0), world - 1);
      before += (long double)cost[i];
    }
  });
}

int b200jk_plan_autotune(b200jk_plan* plan, const double* d_density, int32_t nb, int32_t hermi,
                         int32_t precision, double fp32_cut, int32_t reps, void* stream, int32_t* chunks) {
  return guarded([&] {
    if (!plan) invalid("Invalid plan");
    if (reps < 1) invalid("autotune needs reps >= 1");
    Plan& p = *plan->p;
    cudaStream_t st = (cudaStream_t)stream;
    check_jk_args(p, d_density, nb, d_density, 1, 1, precision, fp32_cut);
    CUDA_OK(cudaSetDevice(p.device));
    ensure_scratch(p, nb);
    // one full build on the plan's scratch prepares the effective densities
    // and the FP32 boundary input (max |D|); its result is discarded
    DevBuf out;
    CUDA_OK(out.ensure((size_t)2 * nb * p.out_stride * sizeof(double)));
    run_jk_core(p, d_density, nb, out.as<double>(), 1, 1, hermi, precision, fp32_cut, st, p.d_dens.as<double>(),
                p.d_dens_f.as<float>(), p.d_vj.as<double>(), p.d_vk.as<double>(), false);
    JKArgs a = base_args(p);
    a.dens = p.d_dens.as<double>();
    a.dens_f = p.d_dens_f.as<float>();
    a.vj = p.d_vj.as<double>();
    a.vk = p.d_vk.as<double>();
    a.dstride = p.cart_stride;
    a.ndm = hermi ? nb : 2 * nb;
    a.nsym = nb;
    a.with_j = 1;
    a.with_k = 1;
    a.fp32_cut = fp32_cut;
    const auto& disp = dispatch();
    cudaEvent_t e0, e1;
    CUDA_OK(cudaEventCreate(&e0));
    CUDA_OK(cudaEventCreate(&e1));
    if (chunks) std::fill(chunks, chunks + kQuartetClasses, -1);
    for (auto* W : p.work) {
      const int cls = quartet_class(W->x, W->y);
      if (!disp.reg_path[cls]) continue;  // tile / team items keep their sizes
      int best = 0;
      float best_ms = 0.f;
      for (const int cand : {32, 64, 128}) {
        fill_items(p, *W, cand);
        apply_shard(p, *W);
        if (precision == B200JK_SPLIT) split_units(p, *W, fp32_cut, st);
        launch_units(p, *W, a, precision, st, false);  // warm-up
        CUDA_OK(cudaEventRecord(e0, st));
        for (int r = 0; r < reps; ++r) launch_units(p, *W, a, precision, st, false);
        CUDA_OK(cudaEventRecord(e1, st));
        CUDA_OK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
        if (best == 0 || ms < best_ms) {
          best = cand;
          best_ms = ms;
        }
      }
      fill_items(p, *W, best);
      apply_shard(p, *W);
      W->chunk = best;
      if (chunks) chunks[cls] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CUDA_OK(cudaStreamSynchronize(st));
  });
}

int b200jk_plan_launches(const b200jk_plan* plan, int32_t precision, int64_t* count) {
  return guarded([&] {
    if (!plan || !count) invalid("Invalid plan query");
    const Plan& p = *plan->p;
    long long units = 0, lists = 0, flat = 0;
    const auto& disp = dispatch();
    for (auto* W : p.work)
      for_each_unit(const_cast<Plan&>(p), *W, [&](const JKUnit& u) {
        units += u.nwork > 0;
        flat += u.nwork > 0 && u.grp && u.grp->flat_cap > 0 &&
                disp.flat64[quartet_class(W->x, W->y)][gen_slot(u.gb, u.gk)] != nullptr;
      });
    for (int c = 0; c < kPairClasses; ++c) lists += !p.classes[c].q.empty() + !p.grouped[c].q.empty();
    // density_in + jk_out; split: to_float, maxabs, rowmax, one row-max pass
    // per list, one boundary kernel and two J/K slices per unit, and per
    // bra-group unit the flat-list builder and the flat FP64 kernel
    *count = precision == B200JK_SPLIT ? 2 + 3 + lists + 3 * units + 2 * flat : 2 + units;
  });
}

int b200jk_plan_set_shard(b200jk_plan* plan, int32_t rank, int32_t world) {
  return guarded([&] {
    if (!plan) invalid("Invalid plan");
    if (world < 1 || rank < 0 || rank >= world) invalid("Invalid shard (rank, world)");
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    CUDA_OK(cudaDeviceSynchronize());
    p.shard_rank = rank;
    p.shard_world = world;
    for (auto* W : p.work) apply_shard(p, *W);
  });
}

int b200jk_plan_class_stats(const b200jk_plan* plan, int64_t* quartets, int64_t* prim_quartets) {
  return guarded([&] {
    if (!plan || !quartets || !prim_quartets) invalid("Invalid plan query");
    std::fill(quartets, quartets + kQuartetClasses, 0);
    std::fill(prim_quartets, prim_quartets + kQuartetClasses, 0);
    for (auto* W : plan->p->work) {
      const int c = quartet_class(W->x, W->y);
      if (W->buckets.empty()) {
        quartets[c] += W->quartets;
        prim_quartets[c] += W->prim_quartets;
      }
      for (auto* B : W->buckets) {  // grouped: digested quartets, primitive quartets evaluated
        quartets[c] += B->quartets;
        prim_quartets[c] += B->prim_quartets;
      }
    }
  });
}

int b200jk_plan_split_stats(b200jk_plan* plan, void* stream, int64_t* q64, int64_t* q32,
                            int64_t* pq64, int64_t* pq32) {
  return guarded([&] {
    if (!plan || !q64 || !q32 || !pq64 || !pq32) invalid("Invalid plan query");
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    CUDA_OK(cudaStreamSynchronize((cudaStream_t)stream));
    for (int c = 0; c < kQuartetClasses; ++c) q64[c] = q32[c] = pq64[c] = pq32[c] = 0;
    for (auto* W : p.work) {
      const int c = quartet_class(W->x, W->y);
      for_each_unit(p, *W, [&](const JKUnit& u) {
        if (u.nwork == 0) return;
        if (u.grp) {
          // per bra of each item: screened, canonical kets, FP64 while
          // Q_bra Q_ket M_item >= fp32_cut (a prefix of the Q-descending run)
          std::vector<double> m(u.nwork);
          CUDA_OK(cudaMemcpy(m.data(), u.split->ptr, u.nwork * sizeof(double), cudaMemcpyDeviceToHost));
          const ClassList& X = *u.X;
          const ClassList& Y = *u.Y;
          const auto& pre = Y.npp_prefix;
          const bool same = W->x == W->y;
          for (int i = 0; i < u.nwork; ++i) {
            const int4 it = (*u.h_items)[i];
            for (int b = 0; b < it.y; ++b) {
              const int pos = X.bord[it.x + b];
              const double qb = X.q[pos];
              int h = screen_end(Y, it.z, it.w, qb, p.cutoff);
              if (same) h = std::min(h, pos + 1);
              h = std::max(h, it.z);
              int s = it.z, e = h;  // first FP32 ket
              while (s < e) {
                const int mid = (s + e) >> 1;
                if (qb * Y.q[mid] * m[i] < p.last_fp32_cut) e = mid;
                else s = mid + 1;
              }
              const long long npa = X.npp_pos[pos];
              const long long combos = (long long)u.gb * u.gk;
              q64[c] += (s - it.z) * combos;
              q32[c] += (h - s) * combos;
              pq64[c] += npa * (pre[s] - pre[it.z]);
              pq32[c] += npa * (pre[h] - pre[s]);
            }
          }
          return;
        }
        std::vector<int> split(u.nwork);
        CUDA_OK(cudaMemcpy(split.data(), u.split->ptr, u.nwork * sizeof(int), cudaMemcpyDeviceToHost));
        const auto& pre = u.Y->npp_prefix;
        const long long combos = (long long)u.gb * u.gk;
        for (int i = 0; i < u.nwork; ++i) {
          const int4 it = (*u.h_items)[i];
          const int lo = it.y, hi = it.z;
          const int sp = std::min(std::max(split[i], lo), hi);
          const long long npa = u.X->npp_pos[it.x];
          q64[c] += (sp - lo) * combos;
          q32[c] += (hi - sp) * combos;
          pq64[c] += npa * (pre[sp] - pre[lo]);
          pq32[c] += npa * (pre[hi] - pre[sp]);
        }
      });
    }
  });
}

int b200jk_plan_border_stats(b200jk_plan* plan, void* stream, int64_t* listed, int64_t* overflow) {
  return guarded([&] {
    if (!plan || !listed || !overflow) invalid("Invalid plan query");
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    CUDA_OK(cudaStreamSynchronize((cudaStream_t)stream));
    *listed = *overflow = 0;
    for (auto* W : p.work)
      for_each_unit(p, *W, [&](const JKUnit& u) {
        if (u.nwork == 0 || !u.grp || u.grp->flat_cap <= 0) return;
        unsigned long long n = 0;
        CUDA_OK(cudaMemcpy(&n, u.grp->flat_n.ptr, sizeof(n), cudaMemcpyDeviceToHost));
        const long long cap = u.grp->flat_cap;
        *listed += std::min((long long)n, cap);
        *overflow += std::max(0LL, (long long)n - cap);
      });
  });
}

int b200jk_int1e(b200jk_plan* plan, int32_t which, double* d_out, void* stream) {
  return guarded([&] {
    if (!plan || !d_out || which < 0 || which > 2) invalid("Invalid one-electron request");
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_OK(p.d_one_scratch.ensure((size_t)3 * p.cart_stride * sizeof(double)));
    double* raw = p.d_one_scratch.as<double>();
    CUDA_OK(cudaMemsetAsync(raw, 0, (size_t)3 * p.cart_stride * sizeof(double), st));
    OneArgs a = one_args(p);
    a.out_s = raw;
    a.out_t = raw + p.cart_stride;
    a.out_v = raw + 2 * p.cart_stride;
    for (int c = 0; c < kPairClasses; ++c) {
      a.pairs = p.d_all_pairs[c].as<int>();
      a.npairs = p.n_all_pairs[c];
      launch_one_electron(c, false, a, st);
      CUDA_OK(cudaGetLastError());
    }
    const Tables tb = plan_tables(p);
    const int no = max_no(p);
    dim3 grid((unsigned)(((long long)no * no + 255) / 256), p.nmol);
    cart_to_out_kernel<<<grid, 256, 0, st>>>(raw + which * p.cart_stride, d_out,
        p.d_mol_base_out.as<long long>(), p.d_mol_nout.as<int>(), p.d_mol_base_cart.as<long long>(),
        p.d_mol_ncart.as<int>(), p.d_out_ws.as<int>(), p.d_ws_info.as<int4>(),
        p.d_mol_ao_off.as<int>() + p.nmol, tb.c2s);
    CUDA_OK(cudaGetLastError());
  });
}

int b200jk_int1e_grad(b200jk_plan* plan, const double* d_density, const double* d_energy_weighted,
                      double* d_grad, void* stream) {
  return guarded([&] {
    if (!plan || !d_density || !d_energy_weighted || !d_grad) invalid("Invalid one-electron gradient request");
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_OK(p.d_one_dens.ensure((size_t)2 * p.cart_stride * sizeof(double)));
    double* raw = p.d_one_dens.as<double>();
    const Tables tb = plan_tables(p);
    const int nc = max_nc(p);
    const double* ins[2] = {d_density, d_energy_weighted};
    for (int k = 0; k < 2; ++k) {
      dim3 grid((unsigned)(((long long)nc * nc + 255) / 256), p.nmol, 1);
      density_in_kernel<<<grid, 256, 0, st>>>(
          ins[k], 1, 1, raw + k * p.cart_stride, p.out_stride, p.cart_stride,
          p.d_mol_base_out.as<long long>(), p.d_mol_nout.as<int>(), p.d_mol_base_cart.as<long long>(),
          p.d_mol_ncart.as<int>(), p.d_cart_ws.as<int>(), p.d_ws_info.as<int4>(),
          p.d_mol_ao_off.as<int>(), tb.c2s, p.d_status.as<int>());
      CUDA_OK(cudaGetLastError());
    }
    CUDA_OK(cudaMemsetAsync(d_grad, 0, (size_t)p.total_atm * 3 * sizeof(double), st));
    OneArgs a = one_args(p);
    a.dm = raw;
    a.wm = raw + p.cart_stride;
    a.grad = d_grad;
    for (int c = 0; c < kPairClasses; ++c) {
      a.pairs = p.d_all_pairs[c].as<int>();
      a.npairs = p.n_all_pairs[c];
      launch_one_electron(c, true, a, st);
      CUDA_OK(cudaGetLastError());
    }
  });
}

int b200jk_packed_eri(b200jk_plan* plan, int32_t layout, double* d_out, int64_t out_size, void* stream) {
  return guarded([&] {
    if (!plan || !d_out) invalid("Invalid packed ERI request");
    Plan& p = *plan->p;
    if (p.nmol != 1) invalid("Packed ERIs are built for one-molecule plans");
    if (layout != 0 && layout != 1) invalid("Packed ERI layout must be 0 (s4) or 1 (s8)");
    const long long n = p.mol_nout[0], np = n * (n + 1) / 2;
    const long long size = layout == 0 ? np * np : np * (np + 1) / 2;
    if (out_size != size) invalid("Packed ERI shape mismatch");  // csrc/packed_eri.cc:7-9
    CUDA_OK(cudaSetDevice(p.device));
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_OK(cudaMemsetAsync(d_out, 0, (size_t)size * sizeof(double), st));
    JKArgs a = base_args(p);
    const auto& disp = dispatch();
    for (auto* W : p.work) {
      if (W->nwork == 0) continue;
      const int cls = quartet_class(W->x, W->y);
      set_lists(a, p, *W);
      a.work = W->work.as<int4>();
      a.nwork = W->nwork;
      const int rc = disp.store[cls](a, p.cart, layout, d_out, np, st);
      if (rc) throw Failure{B200JK_INTERNAL, std::string("packed ERI launch failed: ") + cudaGetErrorString((cudaError_t)rc)};
    }
  });
}

int b200jk_direct_jk_geom_vjp(b200jk_plan* plan, const double* d_density, int32_t nb,
                              const double* d_cot, int32_t with_j, int32_t with_k, double* d_grad,
                              void* stream) {
  return b200jk_direct_jk_geom_vjp_precision(plan, d_density, nb, d_cot, with_j, with_k, B200JK_FP64, 0.0, d_grad,
                                             stream);
}

int b200jk_direct_jk_geom_vjp_precision(b200jk_plan* plan, const double* d_density, int32_t nb,
                                        const double* d_cot, int32_t with_j, int32_t with_k, int32_t precision,
                                        double fp32_cut, double* d_grad, void* stream) {
  return guarded([&] {
    if (!plan || !d_density || !d_cot || !d_grad || nb < 1) invalid("Invalid direct J/K geometry product");
    if ((with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) || !(with_j || with_k))
      invalid("Invalid direct J/K geometry product");
    if (precision != B200JK_FP64 && precision != B200JK_SPLIT) invalid("Unknown precision mode");
    if (precision == B200JK_SPLIT && !(fp32_cut >= 0 && std::isfinite(fp32_cut))) invalid("Invalid fp32_cut");
    const bool split = precision == B200JK_SPLIT;
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    cudaStream_t st = (cudaStream_t)stream;
    ensure_scratch(p, nb);
    const Tables tb = plan_tables(p);
    // raw Cartesian D (d_dens), J cotangent (d_vj) and K cotangent (d_vk)
    const int nc = max_nc(p);
    dim3 grid((unsigned)(((long long)nc * nc + 255) / 256), p.nmol, nb);
    auto to_raw = [&](const double* src, double* dst) {
      mat_in_kernel<<<grid, 256, 0, st>>>(src, dst, p.out_stride, p.cart_stride,
          p.d_mol_base_out.as<long long>(), p.d_mol_nout.as<int>(), p.d_mol_base_cart.as<long long>(),
          p.d_mol_ncart.as<int>(), p.d_cart_ws.as<int>(), p.d_ws_info.as<int4>(), p.d_mol_ao_off.as<int>(),
          tb.c2s);
      CUDA_OK(cudaGetLastError());
    };
    to_raw(d_density, p.d_dens.as<double>());
    if (with_j) to_raw(d_cot, p.d_vj.as<double>());
    if (with_k) to_raw(d_cot + (size_t)(with_j ? nb : 0) * p.out_stride, p.d_vk.as<double>());
    CUDA_OK(cudaMemsetAsync(d_grad, 0, (size_t)p.total_atm * 3 * sizeof(double), st));
    if (split) {
      // per item the first ket whose quartets run in FP32: Q_bra Q_ket M_item < fp32_cut
      // with M_item bounding |Gamma| over the item (grad_rowmax_kernel)
      const int nrows = (int)(p.d_rowmax.bytes / sizeof(double));
      grad_rowmax_kernel<<<(nrows + 7) / 8, 256, 0, st>>>(
          p.d_dens.as<double>(), with_j ? p.d_vj.as<double>() : nullptr, with_k ? p.d_vk.as<double>() : nullptr, nb,
          p.cart_stride, p.d_mol_base_cart.as<long long>(), p.d_mol_ncart.as<int>(), p.d_mol_ao_off.as<int>(),
          p.d_cart_ws.as<int>(), p.d_ws_info.as<int4>(), nrows, p.d_rowmax.as<double>());
      CUDA_OK(cudaGetLastError());
      for (int c = 0; c < kPairClasses; ++c) {
        ClassList& L = p.classes[c];
        const int npos = (int)L.q.size();
        if (npos == 0) continue;
        posmax_kernel<<<(npos + 127) / 128, 128, 0, st>>>(L.d_ix.as<int4>(), L.d_gx.as<int4>(), L.d_gy.as<int4>(),
                                                         L.d_nco.as<int>(), L.d_ra.as<double4>(), npos,
                                                         ncart_of(pc_la_host(c)), p.d_rowmax.as<double>(),
                                                         p.d_mol_ao_off.as<int>(), L.d_kmax.as<double>());
        CUDA_OK(cudaGetLastError());
      }
      for (auto* W : p.work) {
        if (W->nwork == 0) continue;
        const ClassList& X = p.classes[W->x];
        const ClassList& Y = p.classes[W->y];
        const int la = pc_la_host(W->x), lb = W->x - la * (la + 1) / 2;
        SplitLists L{X.d_ix.as<int4>(), X.d_gx.as<int4>(), X.d_gy.as<int4>(), Y.d_kmax.as<double>(),
                     X.d_ra.as<double4>(), 1, ncart_of(la), ncart_of(lb)};
        split_kernel<<<(W->nwork + 3) / 4, 128, 0, st>>>(W->work.as<int4>(), X.d_q.as<double>(), Y.d_q.as<double>(),
                                                        p.d_rowmax.as<double>(), p.d_mol_ao_off.as<int>(), L,
                                                        fp32_cut, W->nwork, W->split.as<int>());
        CUDA_OK(cudaGetLastError());
      }
    }
    JKArgs a = base_args(p);
    a.dens = p.d_dens.as<double>();
    a.dstride = p.cart_stride;
    a.cot_j = with_j ? p.d_vj.as<double>() : nullptr;
    a.cot_k = with_k ? p.d_vk.as<double>() : nullptr;
    a.gnb = nb;
    a.grad = d_grad;
    const auto& disp = dispatch();
    // class pairs longest-first over the caller's and the auxiliary streams
    // (serial while profiling, so each launch is timed alone)
    const int nstreams = p.profiling ? 1 : kAuxStreams + 1;
    cudaStream_t streams[kAuxStreams + 1] = {st};
    for (int i = 0; i < kAuxStreams; ++i) streams[i + 1] = p.aux[i];
    if (nstreams > 1) {
      CUDA_OK(cudaEventRecord(p.fork_ev, st));
      for (int i = 0; i < kAuxStreams; ++i) CUDA_OK(cudaStreamWaitEvent(p.aux[i], p.fork_ev, 0));
    }
    std::vector<std::pair<long long, ClassPairWork*>> order;
    for (auto* W : p.work) order.push_back({W->prim_quartets, W});
    std::sort(order.begin(), order.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    std::vector<long long> load(nstreams, 0);
    for (auto& [cost, W] : order) {
      if (W->nwork == 0) continue;
      int best = 0;
      for (int i = 1; i < nstreams; ++i)
        if (load[i] < load[best]) best = i;
      load[best] += cost;
      cudaStream_t ls = streams[best];
      const int cls = quartet_class(W->x, W->y);
      set_lists(a, p, *W);
      a.work = W->work.as<int4>();
      a.nwork = W->nwork;
      a.split = W->split.as<int>();
      // FP64 (all kets, or the kets before each item's FP32 boundary), then the FP32 slice
      for (int slice = 0; slice < (split ? 2 : 1); ++slice) {
        a.split_mode = split ? slice + 1 : 0;
        ProfileEvent ev{cls, slice, nullptr, nullptr};
        if (p.profiling) {
          CUDA_OK(cudaEventCreate(&ev.start));
          CUDA_OK(cudaEventCreate(&ev.stop));
          CUDA_OK(cudaEventRecord(ev.start, ls));
        }
        const GradLauncher lg = slice == 0 ? disp.grad64[cls] : disp.grad32[cls];
        const int rc = lg(a, ls);
        if (rc)
          throw Failure{B200JK_INTERNAL, std::string("gradient launch failed (class pair ") + std::to_string(W->x) +
                                             "," + std::to_string(W->y) + "): " + cudaGetErrorString((cudaError_t)rc)};
        if (p.profiling) {
          CUDA_OK(cudaEventRecord(ev.stop, ls));
          p.events.push_back(ev);
        }
      }
    }
    if (nstreams > 1)
      for (int i = 0; i < kAuxStreams; ++i) {
        CUDA_OK(cudaEventRecord(p.join_ev[i], p.aux[i]));
        CUDA_OK(cudaStreamWaitEvent(st, p.join_ev[i], 0));
      }
  });
}

// The geometry-product kernel (mode 0/1: JVP of order 1/2, 2: order-2 VJP)
// of every class pair's expanded work items, on `a` as prepared by the caller.
static void launch_geom_all(Plan& p, JKArgs a, int mode, cudaStream_t st) {
  for (auto* W : p.work) {
    if (W->nwork == 0) continue;
    const int la = pc_la_host(W->x), lb = W->x - la * (la + 1) / 2;
    const int lc = pc_la_host(W->y), ld = W->y - lc * (lc + 1) / 2;
    if (!geom_smem_bytes(la, lb, lc, ld)) throw Failure{B200JK_UNSUPPORTED, "class too large for the geometry products"};
    set_lists(a, p, *W);
    a.work = W->work.as<int4>();
    a.nwork = W->nwork;
    a.split_mode = 0;
    const int rc = launch_geom(a, la, lb, lc, ld, mode, st);
    if (rc) throw Failure{B200JK_INTERNAL, std::string("geometry product launch failed: ") + cudaGetErrorString((cudaError_t)rc)};
  }
}

int b200jk_direct_jk_geom_jvp(b200jk_plan* plan, const double* d_density, int32_t nb, int32_t hermi,
                              const double* d_u, const double* d_v, int32_t with_j, int32_t with_k,
                              double* d_out, void* stream) {
  return guarded([&] {
    if (!plan || !d_density || !d_u || !d_out || nb < 1) invalid("Invalid direct J/K geometry product");
    if ((with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) || !(with_j || with_k))
      invalid("Invalid direct J/K geometry product");
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    cudaStream_t st = (cudaStream_t)stream;
    ensure_scratch(p, nb);
    const int hm = hermi ? 1 : 0;
    jk_prologue(p, d_density, nb, hm, with_j, with_k, st, p.d_dens.as<double>(), p.d_vj.as<double>(),
                p.d_vk.as<double>());
    JKArgs a = base_args(p);
    a.dens = p.d_dens.as<double>();
    a.vj = p.d_vj.as<double>();
    a.vk = p.d_vk.as<double>();
    a.dstride = p.cart_stride;
    a.ndm = hm ? nb : 2 * nb;
    a.nsym = nb;
    a.with_j = with_j;
    a.with_k = with_k;
    a.geo_u = d_u;
    a.geo_v = d_v;
    launch_geom_all(p, a, d_v ? 1 : 0, st);
    jk_epilogue(p, nb, hm, with_j, with_k, d_out, st, p.d_vj.as<double>(), p.d_vk.as<double>());
  });
}

int b200jk_direct_jk_geom_hvp(b200jk_plan* plan, const double* d_density, int32_t nb, const double* d_u,
                              const double* d_cot, int32_t with_j, int32_t with_k, double* d_grad,
                              void* stream) {
  return guarded([&] {
    if (!plan || !d_density || !d_u || !d_cot || !d_grad || nb < 1) invalid("Invalid direct J/K geometry product");
    if ((with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) || !(with_j || with_k))
      invalid("Invalid direct J/K geometry product");
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    cudaStream_t st = (cudaStream_t)stream;
    ensure_scratch(p, nb);
    const Tables tb = plan_tables(p);
    const int nc = max_nc(p);
    dim3 grid((unsigned)(((long long)nc * nc + 255) / 256), p.nmol, nb);
    auto to_raw = [&](const double* src, double* dst) {
      mat_in_kernel<<<grid, 256, 0, st>>>(src, dst, p.out_stride, p.cart_stride,
          p.d_mol_base_out.as<long long>(), p.d_mol_nout.as<int>(), p.d_mol_base_cart.as<long long>(),
          p.d_mol_ncart.as<int>(), p.d_cart_ws.as<int>(), p.d_ws_info.as<int4>(), p.d_mol_ao_off.as<int>(),
          tb.c2s);
      CUDA_OK(cudaGetLastError());
    };
    to_raw(d_density, p.d_dens.as<double>());
    if (with_j) to_raw(d_cot, p.d_vj.as<double>());
    if (with_k) to_raw(d_cot + (size_t)(with_j ? nb : 0) * p.out_stride, p.d_vk.as<double>());
    CUDA_OK(cudaMemsetAsync(d_grad, 0, (size_t)p.total_atm * 3 * sizeof(double), st));
    JKArgs a = base_args(p);
    a.dens = p.d_dens.as<double>();
    a.dstride = p.cart_stride;
    a.cot_j = with_j ? p.d_vj.as<double>() : nullptr;
    a.cot_k = with_k ? p.d_vk.as<double>() : nullptr;
    a.gnb = nb;
    a.grad = d_grad;
    a.geo_u = d_u;
    launch_geom_all(p, a, 2, st);
  });
}

int b200jk_plan_set_profiling(b200jk_plan* plan, int32_t on) {
  return guarded([&] {
    if (!plan) invalid("Null plan");
    plan->p->profiling = on != 0;
  });
}

int b200jk_plan_profile(b200jk_plan* plan, double* ms64, double* ms32, int32_t* launches) {
  return guarded([&] {
    if (!plan || !ms64 || !ms32 || !launches) invalid("Invalid plan query");
    Plan& p = *plan->p;
    CUDA_OK(cudaSetDevice(p.device));
    for (int c = 0; c < kQuartetClasses; ++c) { ms64[c] = ms32[c] = 0.0; launches[c] = 0; }
    for (auto& e : p.events) {
      CUDA_OK(cudaEventSynchronize(e.stop));
      float ms = 0.f;
      CUDA_OK(cudaEventElapsedTime(&ms, e.start, e.stop));
      (e.fp32 ? ms32 : ms64)[e.cls] += ms;
      launches[e.cls] += 1;
      cudaEventDestroy(e.start);
      cudaEventDestroy(e.stop);
    }
    p.events.clear();
  });
}

}  // extern "C"
