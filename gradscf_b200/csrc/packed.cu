// J/K from packed ERIs (the reference's PackedJK, csrc/packed_jk.cc:6-80):
// s8 storage (np(np+1)/2 values, np = n(n+1)/2) or s4 (np x np), any real
// density batch (nonsymmetric allowed), output (with_j + with_k, nb, n, n)
// overwritten.  One warp per pair row ab (packed_jk_kernel below).
#include <cuda_runtime.h>

#include <atomic>
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

// One block (one warp) per pair row ab = (a, b), a >= b: the row's
// elements (ab|cd), cd <= ab, are read once, contiguously, for every
// density.  Its exchange contributions all land in rows a, b and columns
// a, b of K: they are summed in shared memory (K[a][.], K[b][.], K[.][a],
// K[.][b], one column per density) and added to K once per row.  The loop
// runs over c with the lanes on d, so terms indexed by d go to distinct
// shared addresses and terms indexed by c are warp-reduced first.  J[a][b]
// is warp-reduced; J[c][d] (cd < ab) takes one add per element into the
// pair-packed accumulator `jp`, unfolded by packed_j_out_kernel.
__global__ void packed_jk_kernel(const double* __restrict__ eri, int layout, int n, long long np,
                                 const double* __restrict__ dens, int nb, double* __restrict__ out,
                                 double* __restrict__ jp, int with_j, int with_k) {
  extern __shared__ double sk[];  // [nb][4][n]: K[a][x], K[b][x], K[x][a], K[x][b]
  const long long ab = blockIdx.x;
  const int lane = threadIdx.x;
  if (ab >= np) return;
  int a, b;
  unpair(ab, a, b);
  const long long nn = (long long)n * n;
  const double* row = layout == 1 ? eri + ab * (ab + 1) / 2 : eri + ab * np;
  if (with_k)
    for (int i = lane; i < 4 * n * nb; i += 32) sk[i] = 0.0;
  __syncwarp();
  double jab[4] = {0.0, 0.0, 0.0, 0.0};   // densities in chunks of 4 (J[a][b])
  for (int e0 = 0; e0 < nb; e0 += 4) {
    const int ne = min(4, nb - e0);
    for (int c = 0; c <= a; ++c) {
      const int dmax = c == a ? b : c;
      double rc[4][4];   // [density][K[a][c], K[b][c], K[c][a], K[c][b]] for this c
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) rc[x][y] = 0.0;
      for (int d = lane; d <= dmax; d += 32) {
        const long long cd = (long long)c * (c + 1) / 2 + d;
        const double v = row[cd];
        if (v == 0.0) continue;
        const bool offd = c != d, offab = a != b, notdiag = ab != cd;
        for (int q = 0; q < ne; ++q) {
          const int e = e0 + q;
          const double* D = dens + e * nn;
          if (with_j) {
            jab[q] += v * (D[(long long)c * n + d] + (offd ? D[(long long)d * n + c] : 0.0));
            if (notdiag)
              atomicAdd(jp + (long long)e * np + cd, v * (D[(long long)a * n + b] + (offab ? D[(long long)b * n + a] : 0.0)));
          }
          if (with_k) {
            double* s = sk + (long long)e * 4 * n;
            rc[q][0] += v * D[(long long)b * n + d];                          // K[a][c]
            if (offd) s[d] += v * D[(long long)b * n + c];                    // K[a][d]
            if (offab) {
              rc[q][1] += v * D[(long long)a * n + d];                        // K[b][c]
              if (offd) s[n + d] += v * D[(long long)a * n + c];              // K[b][d]
            }
            if (notdiag) {
              rc[q][2] += v * D[(long long)d * n + b];                        // K[c][a]
              if (offab) rc[q][3] += v * D[(long long)d * n + a];             // K[c][b]
              if (offd) {
                s[2 * n + d] += v * D[(long long)c * n + b];                  // K[d][a]
                if (offab) s[3 * n + d] += v * D[(long long)c * n + a];       // K[d][b]
              }
            }
          }
        }
      }
      if (with_k) {
        for (int q = 0; q < ne; ++q)
#pragma unroll
          for (int y = 0; y < 4; ++y) {
            double v = rc[q][y];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0) sk[(long long)(e0 + q) * 4 * n + y * n + c] += v;
          }
      }
      __syncwarp();
    }
    if (with_j) {
      for (int q = 0; q < ne; ++q) {
        double v = jab[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0 && v != 0.0) atomicAdd(jp + (long long)(e0 + q) * np + ab, v);
        jab[q] = 0.0;
      }
    }
  }
  if (!with_k) return;
  __syncwarp();
  // the row's exchange sums: rows a, b and columns a, b of every density's K
  for (int e = 0; e < nb; ++e) {
    double* K = out + ((long long)with_j * nb + e) * nn;
    const double* s = sk + (long long)e * 4 * n;
    for (int x = lane; x < n; x += 32) {
      if (s[x] != 0.0) atomicAdd(K + (long long)a * n + x, s[x]);
      if (s[2 * n + x] != 0.0) atomicAdd(K + (long long)x * n + a, s[2 * n + x]);
      if (a != b) {
        if (s[n + x] != 0.0) atomicAdd(K + (long long)b * n + x, s[n + x]);
        if (s[3 * n + x] != 0.0) atomicAdd(K + (long long)x * n + b, s[3 * n + x]);
      }
    }
  }
}

// J[i][j] = J[j][i] = jp[pair(i, j)] for every density.
__global__ void packed_j_out_kernel(const double* __restrict__ jp, int n, long long np, int nb,
                                    double* __restrict__ out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nn = (long long)n * n;
  if (idx >= nn * nb) return;
  const int e = (int)(idx / nn);
  const long long r = idx - e * nn;
  const int i = (int)(r / n), j = (int)(r % n);
  const long long pr = i >= j ? (long long)i * (i + 1) / 2 + j : (long long)j * (j + 1) / 2 + i;
  out[idx] = jp[(long long)e * np + pr];
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
    const size_t smem = with_k ? (size_t)4 * n * nb * sizeof(double) : 0;
    if (smem > 200 * 1024)
      b200jk::fail_invalid("Packed J/K: n x nb too large for the per-row exchange sums (n * nb <= 6400)");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t outn = (size_t)(with_j + with_k) * nb * n * n;
    cudaError_t e = cudaMemsetAsync(d_out, 0, outn * sizeof(double), st);
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    // pair-packed J accumulator (stream-ordered allocation, freed on the stream after use)
    double* jp = nullptr;
    if (with_j) {
      e = cudaMallocAsync(reinterpret_cast<void**>(&jp), (size_t)nb * np * sizeof(double), st);
      if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
      e = cudaMemsetAsync(jp, 0, (size_t)nb * np * sizeof(double), st);
      if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    }
    // the attribute is set once per device, to the largest size any call asks for
    static std::atomic<uint64_t> smem_done{0};
    e = b200jk::smem_opt_in(b200jk::packed_jk_kernel, smem > 48 * 1024 ? (size_t)200 * 1024 : smem, smem_done);
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    b200jk::packed_jk_kernel<<<(unsigned)np, 32, smem, st>>>(d_eri, layout, n, np, d_density, nb, d_out, jp,
                                                            with_j, with_k);
    e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    if (with_j) {
      const long long total = (long long)nb * n * n;
      b200jk::packed_j_out_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(jp, n, np, nb, d_out);
      e = cudaGetLastError();
      if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
      e = cudaFreeAsync(jp, st);
      if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    }
  });
}
