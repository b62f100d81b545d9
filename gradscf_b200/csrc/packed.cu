// J/K from packed ERIs (the reference's PackedJK, csrc/packed_jk.cc:6-80):
// s8 storage (np(np+1)/2 values, np = n(n+1)/2) or s4 (np x np), any real
// density batch (nonsymmetric allowed), output (with_j + with_k, nb, n, n)
// overwritten.  One warp per pair row ab: the row's contributions to
// J[a][b] are warp-reduced, every other element is an atomic add.
#include <cuda_runtime.h>

#include <cmath>
#include <stdexcept>
#include <string>

#include "b200jk.h"
#include "plan.h"

namespace b200jk {
namespace {

// i >= j with pair = i(i+1)/2 + j
__device__ __forceinline__ void unpair(long long pr, int& i, int& j) {
  long long r = (long long)((sqrt(8.0 * (double)pr + 1.0) - 1.0) * 0.5);
  while (r * (r + 1) / 2 > pr) --r;
  while ((r + 1) * (r + 2) / 2 <= pr) ++r;
  i = (int)r;
  j = (int)(pr - r * (r + 1) / 2);
}

__global__ void packed_jk_kernel(const double* __restrict__ eri, int layout, int n, long long np,
                                 const double* __restrict__ dens, int nb, double* __restrict__ out,
                                 int with_j, int with_k) {
  const long long ab = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (ab >= np) return;
  int a, b;
  unpair(ab, a, b);
  const long long nn = (long long)n * n;
  const double* row = layout == 1 ? eri + ab * (ab + 1) / 2 : eri + ab * np;
  for (int e = 0; e < nb; ++e) {
    const double* D = dens + e * nn;
    double* J = with_j ? out + e * nn : nullptr;
    double* K = with_k ? out + ((long long)with_j * nb + e) * nn : nullptr;
    double jab = 0.0;
    const double dab = D[(long long)a * n + b] + (a != b ? D[(long long)b * n + a] : 0.0);
    for (long long cd = lane; cd <= ab; cd += 32) {
      int c, d;
      unpair(cd, c, d);
      const double v = row[cd];
      if (v == 0.0) continue;
      if (J) {
        jab += v * (D[(long long)c * n + d] + (c != d ? D[(long long)d * n + c] : 0.0));
        if (ab != cd) {
          const double jcd = v * dab;
          atomicAdd(J + (long long)c * n + d, jcd);
          if (c != d) atomicAdd(J + (long long)d * n + c, jcd);
        }
      }
      if (K) {
        atomicAdd(K + (long long)a * n + c, v * D[(long long)b * n + d]);
        if (c != d) atomicAdd(K + (long long)a * n + d, v * D[(long long)b * n + c]);
        if (a != b) atomicAdd(K + (long long)b * n + c, v * D[(long long)a * n + d]);
        if (a != b && c != d) atomicAdd(K + (long long)b * n + d, v * D[(long long)a * n + c]);
        if (ab != cd) {
          atomicAdd(K + (long long)c * n + a, v * D[(long long)d * n + b]);
          if (a != b) atomicAdd(K + (long long)c * n + b, v * D[(long long)d * n + a]);
          if (c != d) atomicAdd(K + (long long)d * n + a, v * D[(long long)c * n + b]);
          if (a != b && c != d) atomicAdd(K + (long long)d * n + b, v * D[(long long)c * n + a]);
        }
      }
    }
    if (J) {
      for (int off = 16; off > 0; off >>= 1) jab += __shfl_down_sync(0xffffffffu, jab, off);
      if (lane == 0 && jab != 0.0) {
        atomicAdd(J + (long long)a * n + b, jab);
        if (a != b) atomicAdd(J + (long long)b * n + a, jab);
      }
    }
  }
}

}  // namespace
}  // namespace b200jk

extern "C" int b200jk_packed_jk(const double* d_eri, int32_t layout, int64_t eri_size, int32_t n,
                                const double* d_density, int32_t nb, double* d_out, int32_t with_j,
                                int32_t with_k, void* stream) {
  return b200jk::guarded_call([&] {
    if ((with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) || !(with_j || with_k))
      b200jk::fail_invalid("Packed J/K requires at least one selected operator");
    if (!d_eri || !d_density || !d_out || n < 1 || nb < 1 || (layout != 0 && layout != 1))
      b200jk::fail_invalid("Packed J/K dimensions do not match");
    const long long np = (long long)n * (n + 1) / 2;
    if (eri_size != (layout == 1 ? np * (np + 1) / 2 : np * np))
      b200jk::fail_invalid("Packed J/K dimensions do not match");  // csrc/packed_jk.cc:18-22
    cudaStream_t st = (cudaStream_t)stream;
    const size_t outn = (size_t)(with_j + with_k) * nb * n * n;
    cudaError_t e = cudaMemsetAsync(d_out, 0, outn * sizeof(double), st);
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    const long long warps = np;
    b200jk::packed_jk_kernel<<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(d_eri, layout, n, np, d_density, nb,
                                                                        d_out, with_j, with_k);
    e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
  });
}
