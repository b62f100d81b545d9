// b200jk_direct_jk_noalloc: the direct J/K build on a fixed, file-scope
// device scratch array instead of memory allocated at call time.
//
// Who needs it: callers that must not allocate device memory while they
// run -- e.g. an XLA custom call on a stream XLA owns (XLA's allocator, not
// ours, must own every byte it hands out), code that runs inside CUDA stream
// capture, or a host framework with a fixed device-memory budget.  The plan
// (built beforehand by b200jk_plan_create, which does allocate) holds the
// read-only tables; this entry point itself calls no cudaMalloc/cudaFree and
// no allocating library routine.
//
// Limits and sharing: the scratch is B200JK_NOALLOC_SCRATCH_BYTES (16 MiB)
// of static device memory, held by every GPU that loads the library until
// the process exits.  All calls share it and it keeps the last call's
// contents (the J/K accumulators are zeroed at the start of every call), so
// two calls whose work overlaps on the GPU -- different streams, or
// different threads without ordering -- race and corrupt each other's
// results; order them on one stream.  A call also uses the plan's own small
// device state (density row maxima, status word, per-item FP32 boundaries,
// auxiliary streams), so it races with any other build on the same plan
// (b200jk_direct_jk, a graph replay, the geometry VJP) that overlaps it on
// the GPU.  The first call on each device looks up the array's device
// address (cudaGetSymbolAddress) with that device current; make that first
// call before any stream capture.  The caller's current device is restored
// on return.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/b200jk.h"
#include "plan.h"

namespace b200jk {
namespace {

constexpr size_t kScratchDoubles = B200JK_NOALLOC_SCRATCH_BYTES / sizeof(double);
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (looked up once per device,
// with that device current).
double* scratch_address(int device) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (device < 0 || device >= kMaxDevices) fail_invalid("device ordinal out of range");
  if (!g_ptr[device]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
      fail_invalid(std::string("cudaGetSymbolAddress(scratch) failed: ") + cudaGetErrorString(e));
    g_ptr[device] = static_cast<double*>(ptr);
  }
  return g_ptr[device];
}

size_t round256(size_t doubles) { return (doubles + 31) / 32 * 32; }

}  // namespace
}  // namespace b200jk

extern "C" int b200jk_direct_jk_noalloc(b200jk_plan* plan, const double* d_density, int32_t nb,
                                        double* d_out, int32_t with_j, int32_t with_k,
                                        int32_t hermi, int32_t precision, double fp32_cut,
                                        void* stream) {
  using namespace b200jk;
  return guarded_call([&] {
    if (!plan) fail_invalid("Null plan");
    Plan& p = *plan->p;
    check_jk_args(p, d_density, nb, d_out, with_j, with_k, precision, fp32_cut);
    const size_t cs = (size_t)p.cart_stride;
    const size_t ndm = hermi ? (size_t)nb : 2 * (size_t)nb;
    const size_t n_dens = round256(ndm * cs);
    const size_t n_dens_f = precision == B200JK_SPLIT ? round256((ndm * cs + 1) / 2) : 0;
    const size_t n_vj = with_j ? round256((size_t)nb * cs) : 0;
    const size_t n_vk = with_k ? round256(ndm * cs) : 0;
    const size_t need = n_dens + n_dens_f + n_vj + n_vk;
    if (need > kScratchDoubles)
      fail_invalid("b200jk_direct_jk_noalloc: this call needs " + std::to_string(need * 8) +
                   " bytes of scratch, above the fixed " +
                   std::to_string((size_t)B200JK_NOALLOC_SCRATCH_BYTES) +
                   " bytes; use b200jk_direct_jk (which allocates) or fewer densities");
    int caller_device = 0;
    if (cudaGetDevice(&caller_device) != cudaSuccess) fail_invalid("cannot read the current device");
    if (cudaSetDevice(p.device) != cudaSuccess) fail_invalid("cannot select the plan's device");
    // the caller's device is current again when this scope ends, on every path
    struct RestoreDevice {
      int dev;
      ~RestoreDevice() { cudaSetDevice(dev); }
    } restore{caller_device};
    double* base = scratch_address(p.device);
    double* s_dens = base;
    float* s_dens_f = n_dens_f ? reinterpret_cast<float*>(base + n_dens) : nullptr;
    double* s_vj = n_vj ? base + n_dens + n_dens_f : nullptr;
    double* s_vk = n_vk ? base + n_dens + n_dens_f + n_vj : nullptr;
    run_jk_core(p, d_density, nb, d_out, with_j, with_k, hermi ? 1 : 0, precision, fp32_cut,
                (cudaStream_t)stream, s_dens, s_dens_f, s_vj, s_vk, false);
  });
}
