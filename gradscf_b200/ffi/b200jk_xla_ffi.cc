// XLA typed-FFI handler that routes the reference's direct J/K custom call
// to the B200 library on CUDA arrays.
//
// It binds exactly what the reference's CPU handler GradSCFDirectJK binds
// (src/gradscf/integrals/_native/csrc/direct_jk.cc:97-102): Args atm (natm,
// 6) s32, bas (nbas, 8) s32, env f64, density (nb, n, n) f64; Ret (with_j +
// with_k, nb, n, n) f64; Attrs cart, cutoff, workers, with_j, with_k -- with
// Ctx<PlatformStream<cudaStream_t>> in place of the CPU thread pool, so
// registering it as the CUDA target of the same custom-call name
// ("gradscf_direct_jk_cpu_v1", api_version 1) leaves the reference's
// _direct_operator lowering unchanged.
//
// The tables live in device memory on the CUDA platform: they are copied to
// the host on the call's stream (a few KB), and a device plan is kept per
// distinct table content (rebuilt when coordinates change).  The build runs
// on the allocation-free entry point when its fixed scratch suffices --
// XLA owns the stream and every buffer it hands out -- and otherwise on the
// plan's own scratch, which the plan allocates once and keeps.
//
// Build (needs JAX's FFI headers): python -m gradscf_b200.build --ffi
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "b200jk.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

struct PlanKey {
  std::string bytes;  // atm | bas | env contents, cart, cutoff, device
  bool operator<(const PlanKey& o) const { return bytes < o.bytes; }
};

struct PlanHandle {
  b200jk_plan* plan = nullptr;
  ~PlanHandle() { b200jk_plan_destroy(plan); }
};

std::mutex g_mu;
std::map<PlanKey, std::unique_ptr<PlanHandle>> g_plans;

ffi::Error status_error(int rc) {
  const std::string msg = b200jk_last_error();
  if (rc == B200JK_INVALID_ARGUMENT) return ffi::Error::InvalidArgument(msg);
  if (rc == B200JK_UNSUPPORTED) return ffi::Error(ffi::ErrorCode::kUnimplemented, msg);
  return ffi::Error::Internal(msg);
}

ffi::Error B200DirectJKImpl(cudaStream_t stream, ffi::BufferR2<ffi::S32> atm, ffi::BufferR2<ffi::S32> bas,
                            ffi::BufferR1<ffi::F64> env, ffi::BufferR3<ffi::F64> density,
                            ffi::ResultBufferR4<ffi::F64> out, int32_t cart, double cutoff, int32_t workers,
                            int32_t with_j, int32_t with_k) {
  // the reference handler's checks and their order (direct_jk.cc:15-24)
  if (workers < 1) return ffi::Error::InvalidArgument("Direct J/K workers must be positive");
  if ((with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) || !(with_j || with_k))
    return ffi::Error::InvalidArgument("Direct J/K requires at least one selected operator");
  if (atm.dimensions()[1] != 6 || bas.dimensions()[1] != 8)
    return ffi::Error::InvalidArgument("Invalid libcint table dimensions or operator");
  const int natm = (int)atm.dimensions()[0], nbas = (int)bas.dimensions()[0], nenv = (int)env.element_count();
  const int nb = (int)density.dimensions()[0], n = (int)density.dimensions()[1];
  if (density.dimensions()[2] != n || out->dimensions()[0] != with_j + with_k || out->dimensions()[1] != nb ||
      out->dimensions()[2] != n || out->dimensions()[3] != n)
    return ffi::Error::InvalidArgument("Direct J/K shape mismatch");
  std::vector<int32_t> h_atm((size_t)natm * 6), h_bas((size_t)nbas * 8);
  std::vector<double> h_env(nenv);
  cudaMemcpyAsync(h_atm.data(), atm.typed_data(), h_atm.size() * 4, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(h_bas.data(), bas.typed_data(), h_bas.size() * 4, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(h_env.data(), env.typed_data(), h_env.size() * 8, cudaMemcpyDeviceToHost, stream);
  if (cudaStreamSynchronize(stream) != cudaSuccess) return ffi::Error::Internal("cannot read the tables");
  int device = 0;
  cudaGetDevice(&device);
  PlanKey key;
  key.bytes.append(reinterpret_cast<const char*>(h_atm.data()), h_atm.size() * 4);
  key.bytes.append(reinterpret_cast<const char*>(h_bas.data()), h_bas.size() * 4);
  key.bytes.append(reinterpret_cast<const char*>(h_env.data()), h_env.size() * 8);
  key.bytes.append(reinterpret_cast<const char*>(&cart), sizeof cart);
  key.bytes.append(reinterpret_cast<const char*>(&cutoff), sizeof cutoff);
  key.bytes.append(reinterpret_cast<const char*>(&device), sizeof device);
  std::lock_guard<std::mutex> lock(g_mu);
  auto& slot = g_plans[key];
  if (!slot) {
    auto h = std::make_unique<PlanHandle>();
    const b200jk_molecule mol{h_atm.data(), natm, h_bas.data(), nbas, h_env.data(), nenv};
    const int rc = b200jk_plan_create(&mol, 1, cart, cutoff, device, &h->plan);
    if (rc) {
      g_plans.erase(key);
      return status_error(rc);
    }
    slot = std::move(h);
  }
  int32_t nao = 0;
  b200jk_plan_nao(slot->plan, 0, &nao);
  if (nao != n) return ffi::Error::InvalidArgument("Direct J/K shape mismatch");
  int rc = b200jk_direct_jk_noalloc(slot->plan, density.typed_data(), nb, out->typed_data(), with_j, with_k, 0,
                                    B200JK_FP64, 0.0, stream);
  if (rc == B200JK_INVALID_ARGUMENT && std::strstr(b200jk_last_error(), "scratch"))
    rc = b200jk_direct_jk(slot->plan, density.typed_data(), nb, out->typed_data(), with_j, with_k, 0, B200JK_FP64,
                          0.0, stream);
  if (rc) return status_error(rc);
  rc = b200jk_check_status(slot->plan, stream);   // nonfinite density -> InvalidArgument
  return rc ? status_error(rc) : ffi::Error::Success();
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(B200DirectJK, B200DirectJKImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::BufferR2<ffi::S32>>()
                                  .Arg<ffi::BufferR2<ffi::S32>>()
                                  .Arg<ffi::BufferR1<ffi::F64>>()
                                  .Arg<ffi::BufferR3<ffi::F64>>()
                                  .Ret<ffi::BufferR4<ffi::F64>>()
                                  .Attr<int32_t>("cart")
                                  .Attr<double>("cutoff")
                                  .Attr<int32_t>("workers")
                                  .Attr<int32_t>("with_j")
                                  .Attr<int32_t>("with_k"));
