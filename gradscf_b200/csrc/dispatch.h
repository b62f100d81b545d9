// Launcher table filled by the per-bra-class translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

namespace b200jk {

struct JKArgs;

constexpr int kMaxL = 3;
constexpr int kPairClasses = (kMaxL + 1) * (kMaxL + 2) / 2;              // 10
constexpr int kQuartetClasses = kPairClasses * (kPairClasses + 1) / 2;   // 55

using JKLauncher = int (*)(const JKArgs&, cudaStream_t);
using SchwarzLauncher = int (*)(const JKArgs&, int npairs, int cart, cudaStream_t);
using GradLauncher = int (*)(const JKArgs&, cudaStream_t);
using StoreLauncher = int (*)(const JKArgs&, int cart, int layout, double* out, long long npair, cudaStream_t);

struct DispatchTable {
  JKLauncher jk64[kQuartetClasses] = {};
  JKLauncher jk32[kQuartetClasses] = {};
  JKLauncher grp64[kQuartetClasses] = {};   // register path over bra groups (null: not built)
  JKLauncher grp32[kQuartetClasses] = {};
  GradLauncher grad64[kQuartetClasses] = {};
  GradLauncher grad32[kQuartetClasses] = {};   // FP32 slice of a split-precision VJP
  StoreLauncher store[kQuartetClasses] = {};   // packed ERI producer
  SchwarzLauncher schwarz[kPairClasses] = {};
  // grouped-list kernels by (bra, ket) combinations: slot 3*g(gb) + g(gk),
  // g(1) = 0, g(2) = 1, g(4) = 2 (slot 0 is the plain kernel above)
  JKLauncher jkg64[kQuartetClasses][9] = {};
  JKLauncher jkg32[kQuartetClasses][9] = {};
  // the same buckets on the bra-group register path (null: not built)
  JKLauncher grpg64[kQuartetClasses][9] = {};
  JKLauncher grpg32[kQuartetClasses][9] = {};
  // FP64 flat-list kernels of split builds, per bucket slot (slot 0: plain);
  // built wherever the bra-group kernels are
  JKLauncher flat64[kQuartetClasses][9] = {};
  bool grouped[kQuartetClasses] = {};    // the class pair takes grouped lists
  bool reg_path[kQuartetClasses] = {};   // either precision runs the register path
  bool tile[kQuartetClasses] = {};       // the FP64 kernel is the tile path
  int team[kQuartetClasses] = {};
};

inline int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }   // la >= lb
inline int quartet_class(int x, int y) { return x * (x + 1) / 2 + y; }      // x >= y

#define B200JK_FOR_EACH_CLASS_PAIR(M) \
  M(0, 0) \
  M(1, 0) \
  M(1, 1) \
  M(2, 0) \
  M(2, 1) \
  M(2, 2) \
  M(3, 0) \
  M(3, 1) \
  M(3, 2) \
  M(3, 3) \
  M(4, 0) \
  M(4, 1) \
  M(4, 2) \
  M(4, 3) \
  M(4, 4) \
  M(5, 0) \
  M(5, 1) \
  M(5, 2) \
  M(5, 3) \
  M(5, 4) \
  M(5, 5) \
  M(6, 0) \
  M(6, 1) \
  M(6, 2) \
  M(6, 3) \
  M(6, 4) \
  M(6, 5) \
  M(6, 6) \
  M(7, 0) \
  M(7, 1) \
  M(7, 2) \
  M(7, 3) \
  M(7, 4) \
  M(7, 5) \
  M(7, 6) \
  M(7, 7) \
  M(8, 0) \
  M(8, 1) \
  M(8, 2) \
  M(8, 3) \
  M(8, 4) \
  M(8, 5) \
  M(8, 6) \
  M(8, 7) \
  M(8, 8) \
  M(9, 0) \
  M(9, 1) \
  M(9, 2) \
  M(9, 3) \
  M(9, 4) \
  M(9, 5) \
  M(9, 6) \
  M(9, 7) \
  M(9, 8) \
  M(9, 9)
#define B200JK_DECLARE_REG(x, y) void register_jk_class_##x##_##y(DispatchTable&);
B200JK_FOR_EACH_CLASS_PAIR(B200JK_DECLARE_REG)
#undef B200JK_DECLARE_REG

const DispatchTable& dispatch();

// Blocks of a persistent launch: the kernel's resident blocks per SM times
// the SM count of the current device (looked up once per device).
template <typename Kernel>
inline int persistent_blocks(Kernel* kernel, int threads, size_t smem, std::atomic<int>* cache /* [64] */) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (dev < 64) {
    const int v = cache[dev].load(std::memory_order_acquire);
    if (v > 0) return v;
  }
  int per_sm = 1, sms = 148;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int v = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  if (dev < 64) cache[dev].store(v, std::memory_order_release);
  return v;
}

// Dynamic shared memory above 48 KB is an opt-in attribute of each kernel in
// each device's context: set it on the current device the first time a
// kernel is launched there (bit d of `done` marks device d; any thread).
// Returns the attribute call's error (cudaSuccess when nothing was needed).
template <typename Kernel>
inline cudaError_t smem_opt_in(Kernel* kernel, size_t bytes, std::atomic<uint64_t>& done) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = dev < 64 ? (uint64_t(1) << dev) : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

}  // namespace b200jk
