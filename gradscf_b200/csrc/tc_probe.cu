// Measured tensor-core decision for the high-l horizontal transfer.
//
// The bra transfer of the Rys 2D integrals maps, for one (root, axis,
// ket) column, the vertical-recursion values W[e], e = 0..LA+LB, to
// G[a][b] = sum_e H_AB[(a, b)][e] W[e] -- a linear map that depends only on
// A - B, so for one bra pair (one work item) it is the same matrix for every
// ket and root: a GEMM  G (NAB x ncol) = H (NAB x (LAB+1)) W ((LAB+1) x ncol).
// The recursion computes the same result with far fewer operations
// (y_{b+1}[a] = y_b[a+1] + AB y_b[a]).  This probe times both on the f x f
// bra of the cc-pVTZ f-shell classes (LA = LB = 3: 16 outputs from 7 inputs
// per column, FP64):
//   variant 0: the recursion, one column per thread, in registers;
//   variant 1: the GEMM on the FP64 tensor cores (mma.sync m8n8k4 DMMA: two
//              8-row output tiles, K = 7 padded to 8, 8 columns per warp step).
// Both read W from and write G to shared memory, as the tile kernel does.
// No counterpart in the reference (CPU only).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "b200jk.h"
#include "plan.h"

namespace b200jk {
namespace {

constexpr int kLA = 3, kLB = 3, kLAB = kLA + kLB, kNE = kLAB + 1;   // 7 inputs
constexpr int kNAB = (kLA + 1) * (kLB + 1);                          // 16 outputs
constexpr int kCols = 128;                                           // columns per block pass

// H[(a,b)][e] of the recursion for one AB (host and device)
__host__ __device__ inline void transfer_matrix(double ab, double* H /* [16][8] */) {
  for (int i = 0; i < kNAB * 8; ++i) H[i] = 0.0;
  // track each y_b[a] as a combination of W[0..6]
  double y[kNE][8];
  for (int e = 0; e < kNE; ++e)
    for (int k = 0; k < 8; ++k) y[e][k] = e == k ? 1.0 : 0.0;
  for (int b = 0; b <= kLB; ++b) {
    for (int a = 0; a <= kLA; ++a)
      for (int k = 0; k < 8; ++k) H[(a * (kLB + 1) + b) * 8 + k] = y[a][k];
    if (b < kLB)
      for (int a = 0; a + b < kLAB; ++a)
        for (int k = 0; k < 8; ++k) y[a][k] = y[a + 1][k] + ab * y[a][k];
  }
}

// variant 0: recursion per column
__global__ void hrr_scalar_kernel(const double* __restrict__ w_in, double* __restrict__ g_out, int ncol,
                                  double ab, int reps) {
  __shared__ double W[kNE][kCols];
  __shared__ double G[kNAB][kCols];
  for (int base = blockIdx.x * kCols; base < ncol; base += gridDim.x * kCols) {
    const int n = min(kCols, ncol - base);
    for (int i = threadIdx.x; i < kNE * kCols; i += blockDim.x) {
      const int e = i / kCols, c = i % kCols;
      W[e][c] = c < n ? w_in[(long long)e * ncol + base + c] : 0.0;
    }
    __syncthreads();
    // volatile shared accesses: every repetition really reads and writes
    volatile double(*Wv)[kCols] = W;
    volatile double(*Gv)[kCols] = G;
    for (int r = 0; r < reps; ++r)
      for (int c = threadIdx.x; c < kCols; c += blockDim.x) {
        double y[kNE];
#pragma unroll
        for (int e = 0; e < kNE; ++e) y[e] = Wv[e][c];
#pragma unroll
        for (int b = 0; b <= kLB; ++b) {
#pragma unroll
          for (int a = 0; a <= kLA; ++a) Gv[a * (kLB + 1) + b][c] = y[a];
          if (b < kLB) {
#pragma unroll
            for (int a = 0; a + b < kLAB; ++a) y[a] = y[a + 1] + ab * y[a];
          }
        }
      }
    __syncthreads();
    for (int i = threadIdx.x; i < kNAB * kCols; i += blockDim.x) {
      const int o = i / kCols, c = i % kCols;
      if (c < n) g_out[(long long)o * ncol + base + c] = G[o][c];
    }
    __syncthreads();
  }
}

// variant 1: FP64 tensor cores.  m8n8k4 fragments (PTX ISA, .f64): A 8x4
// row-major, lane holds A[lane/4][lane%4]; B 4x8 column-major, lane holds
// B[lane%4][lane/4]; C/D 8x8, lane holds D[lane/4][2(lane%4) + {0,1}].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void hrr_dmma_kernel(const double* __restrict__ w_in, double* __restrict__ g_out, int ncol,
                                double ab, int reps) {
  __shared__ double W[8][kCols];    // row 7 is the K padding (zero)
  __shared__ double G[kNAB][kCols];
  __shared__ double H[kNAB * 8];
  if (threadIdx.x == 0) transfer_matrix(ab, H);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int base = blockIdx.x * kCols; base < ncol; base += gridDim.x * kCols) {
    const int n = min(kCols, ncol - base);
    for (int i = threadIdx.x; i < 8 * kCols; i += blockDim.x) {
      const int e = i / kCols, c = i % kCols;
      W[e][c] = (e < kNE && c < n) ? w_in[(long long)e * ncol + base + c] : 0.0;
    }
    __syncthreads();
    // per lane: its A fragments of both 8-row tiles and both k-steps
    double a[2][2];
#pragma unroll
    for (int t = 0; t < 2; ++t)
#pragma unroll
      for (int k = 0; k < 2; ++k) a[t][k] = H[(t * 8 + (lane >> 2)) * 8 + k * 4 + (lane & 3)];
    volatile double(*Wv)[kCols] = W;
    volatile double(*Gv)[kCols] = G;
    for (int r = 0; r < reps; ++r)
      for (int c0 = warp * 8; c0 < kCols; c0 += nwarp * 8) {
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          double d0 = 0.0, d1 = 0.0;
#pragma unroll
          for (int k = 0; k < 2; ++k) dmma(d0, d1, a[t][k], Wv[k * 4 + (lane & 3)][c0 + (lane >> 2)]);
          const int row = t * 8 + (lane >> 2), col = c0 + 2 * (lane & 3);
          Gv[row][col] = d0;
          Gv[row][col + 1] = d1;
        }
      }
    __syncthreads();
    for (int i = threadIdx.x; i < kNAB * kCols; i += blockDim.x) {
      const int o = i / kCols, c = i % kCols;
      if (c < n) g_out[(long long)o * ncol + base + c] = G[o][c];
    }
    __syncthreads();
  }
}

}  // namespace
}  // namespace b200jk

extern "C" int b200jk_measure_bra_transfer(int32_t ncol, int32_t reps, double* ns_per_column, double* max_abs_diff,
                                           void* stream) {
  using namespace b200jk;
  return guarded_call([&] {
    if (ncol < 1 || reps < 1 || !ns_per_column || !max_abs_diff) fail_invalid("Invalid probe request");
    cudaStream_t st = (cudaStream_t)stream;
    auto ok = [](cudaError_t e) {
      if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    };
    std::vector<double> hw((size_t)kNE * ncol);
    unsigned long long s = 88172645463325252ull;
    for (auto& v : hw) {
      s ^= s << 13; s ^= s >> 7; s ^= s << 17;
      v = (double)(s >> 11) / 9007199254740992.0 - 0.5;
    }
    const double ab = -1.3717;
    double *dw = nullptr, *dg0 = nullptr, *dg1 = nullptr;
    ok(cudaMalloc(&dw, hw.size() * sizeof(double)));
    ok(cudaMalloc(&dg0, (size_t)kNAB * ncol * sizeof(double)));
    ok(cudaMalloc(&dg1, (size_t)kNAB * ncol * sizeof(double)));
    ok(cudaMemcpy(dw, hw.data(), hw.size() * sizeof(double), cudaMemcpyHostToDevice));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    const int blocks = std::min((ncol + kCols - 1) / kCols, 4 * sms);
    cudaEvent_t e0, e1;
    ok(cudaEventCreate(&e0));
    ok(cudaEventCreate(&e1));
    float ms[2] = {0.f, 0.f};
    for (int v = 0; v < 2; ++v) {
      double* out = v == 0 ? dg0 : dg1;
      for (int pass = 0; pass < 2; ++pass) {   // warm-up, then timed
        ok(cudaEventRecord(e0, st));
        if (v == 0) hrr_scalar_kernel<<<blocks, 128, 0, st>>>(dw, out, ncol, ab, reps);
        else hrr_dmma_kernel<<<blocks, 128, 0, st>>>(dw, out, ncol, ab, reps);
        ok(cudaGetLastError());
        ok(cudaEventRecord(e1, st));
        ok(cudaEventSynchronize(e1));
        ok(cudaEventElapsedTime(&ms[v], e0, e1));
      }
      ns_per_column[v] = (double)ms[v] * 1e6 / ((double)ncol * reps);
    }
    std::vector<double> g0((size_t)kNAB * ncol), g1((size_t)kNAB * ncol);
    ok(cudaMemcpy(g0.data(), dg0, g0.size() * sizeof(double), cudaMemcpyDeviceToHost));
    ok(cudaMemcpy(g1.data(), dg1, g1.size() * sizeof(double), cudaMemcpyDeviceToHost));
    double md = 0.0;
    for (size_t i = 0; i < g0.size(); ++i) md = std::fmax(md, std::fabs(g0[i] - g1[i]));
    *max_abs_diff = md;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(dw);
    cudaFree(dg0);
    cudaFree(dg1);
  });
}
