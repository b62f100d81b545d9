// Host-side plan: the device-resident description of one batch of molecules.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "common.cuh"
#include "dispatch.h"

namespace b200jk {

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  cudaError_t ensure(size_t n) {
    if (n <= bytes && ptr) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&ptr, n > 0 ? n : 16);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// Work items of the register path over bra groups (jk_grp_kernel): int4
// (bra-order begin, bra count, ket begin, ket end), the bras sharing
// molecule, combinations, primitive-pair count and shell A, the kets one run
// of equal primitive-pair count; `m` holds each item's density bound (max |D|
// over the rows its quartets touch) for split-precision calls.
struct GroupWork {
  int nwork = 0;
  DevBuf work, m;
  // split builds: the FP64 quartets of items whose FP64 corner is sparse,
  // one int2 (bra position, ket position) each; the list's length; per item
  // a flag (its FP64 quartets are in the list)
  DevBuf flat, flat_n, skip;
  int flat_cap = 0;
  std::vector<int4> h_items, all_items;
  std::vector<int64_t> item_cost;
  long long quartets = 0, prim_quartets = 0;
};

// Work items of a class pair on grouped lists whose bra / ket entries carry
// gb / gk contraction combinations (one kernel instantiation per bucket).
struct GenBucket {
  int gb = 1, gk = 1;
  int nwork = 0;
  DevBuf work, split;
  std::vector<int4> h_items, all_items;
  std::vector<int64_t> item_cost;
  long long quartets = 0, prim_quartets = 0;
  bool use_grp = false;   // the bucket runs the bra-group register path
  GroupWork grp;
};

struct ClassPairWork {
  int x = 0, y = 0;             // bra / ket pair classes
  int nwork = 0;
  int nbra = 0;
  DevBuf work;                  // int4 per work item
  DevBuf split;                 // int per work item: first FP32 ket (filled per call)
  long long quartets = 0;       // significant work-shell quartets in this class pair
  long long prim_quartets = 0;  // their primitive quartets
  std::vector<int4> h_items;    // this rank's items when the plan is sharded (empty: all_items)
  std::vector<int4> all_items;  // every work item of the class pair
  std::vector<int64_t> item_cost;  // primitive quartets per item (all_items order)
  // grouped lists (contraction combinations shared): the J/K work is in
  // `buckets`; `work` still holds the expanded items (coordinate VJP)
  bool grouped_x = false, grouped_y = false;
  int chunk = 0;                // register-path ket chunk chosen by the autotuner (0: default rule)
  std::vector<GenBucket*> buckets;
  bool use_grp = false;         // J/K on the bra-group register path (no buckets)
  GroupWork grp;
  ~ClassPairWork() {
    for (auto* b : buckets) delete b;
  }
};

struct ClassList {
  std::vector<int> pairs;       // pair ids, sorted (molecule, Q desc)
  std::vector<double> q;        // their parent Schwarz bounds
  std::vector<int> mol_begin;   // per molecule: first position (size nmol+1)
  std::vector<std::vector<int2>> segs;  // per molecule: [begin, end) runs of equal primitive-pair count
  std::vector<long long> npp_prefix;  // prefix sums of primitive-pair counts (size+1)
  std::vector<int> npp_pos, mol_pos;  // per position: primitive pairs, molecule
  DevBuf d_pairs, d_q;
  // per list position (coalesced reads by consecutive kets): centre A and
  // molecule (Ax, Ay, Az, mol), A - B, and (first primitive pair, count,
  // Cartesian offset of A, of B) in the molecule
  DevBuf d_ra, d_ab, d_ix;
  // grouped lists only: contraction combinations per entry (1, 2 or 4) and,
  // per position, (diag, 0, aoA1, aoB1) and (aoA2, aoB2, aoA3, aoB3); segs
  // are then runs of equal (combinations, primitive-pair count)
  std::vector<int> nco;
  DevBuf d_gx, d_gy, d_nco;
  DevBuf d_kmax;  // per position: max |D| over the rows of its A shell (split calls)
  // bra order of the bra-group register path: positions sorted by (molecule,
  // combinations, primitive pairs, Cartesian offsets of the combinations' A
  // shells (aoa_pos packs up to four 16-bit offsets), Q desc); gbeg holds the
  // first bra-order index of every group of equal keys (+ the end)
  std::vector<long long> aoa_pos;
  std::vector<int> bord, gbeg;
  DevBuf d_bord;
};

struct ProfileEvent {
  int cls;
  int fp32;
  cudaEvent_t start, stop;
};

#ifndef B200JK_AUX_STREAMS
#define B200JK_AUX_STREAMS 3
#endif
constexpr int kAuxStreams = B200JK_AUX_STREAMS;  // streams besides the caller's for concurrent class-pair launches
constexpr int kQueueSlots = 4096;  // work-queue counters of persistent launches, reused cyclically

struct Plan {
  int device = 0;
  cudaStream_t aux[kAuxStreams] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[kAuxStreams] = {};
  int shard_rank = 0, shard_world = 1;  // active work-item shard
  int cart = 0;
  double cutoff = 0.0;
  double omega = 0.0;   // env[8]: erf(omega r)/r operator when > 0
  int nmol = 0;
  // per molecule
  std::vector<int> mol_nout, mol_ncart, mol_natm, mol_atm_off;
  std::vector<long long> mol_out_base, mol_cart_base;
  long long out_stride = 0, cart_stride = 0;
  int total_atm = 0;
  // work shells
  int nws = 0;
  std::vector<int4> ws_info;     // (cart offset in mol, l, mol, out offset in mol)
  std::vector<double4> ws_xyz;
  std::vector<int> ws_parent;    // global parent shell id
  std::vector<int> ws_atm;       // global atm row of the shell's centre
  std::vector<int> ws_nprim;
  std::vector<double> ws_exp, ws_coef;  // per primitive (flattened), coef of this column
  std::vector<int> ws_prim_off;
  // pairs
  int npair = 0;
  std::vector<int4> pair_info;   // (A, B, pp offset, pp count)
  std::vector<int> pair_class;
  std::vector<double> pair_q;    // parent Schwarz bound
  ClassList classes[kPairClasses];
  ClassList grouped[kPairClasses];  // pair classes (l, 0) only: parent pairs with combinations
  std::vector<ClassPairWork*> work;
  long long quartets = 0;
  // nuclei (for one-electron terms): global atm rows with charge
  std::vector<double4> atom_xyzq; // (x, y, z, charge) per global atm row
  // device tables
  DevBuf d_pp_c, d_pp_cf;          // per primitive pair: combination coefficients (FP64, FP32)
  DevBuf d_rowmax;                 // per Cartesian row (all molecules): max |D| of the last split call
  DevBuf d_ws_info, d_ws_xyz, d_pair_info, d_pp_data, d_pp_aux, d_pp_exp, d_pp_f, d_pp_f2, d_mol_base_cart, d_mol_ncart,
      d_mol_base_out, d_mol_nout, d_cart_ws, d_out_ws, d_status, d_maxd, d_q_work, d_atoms,
      d_ws_atm, d_mol_ao_off, d_ws_prim, d_ws_prim_off;
  // one-electron work: every work pair of each pair class, nuclei ranges
  DevBuf d_all_pairs[kPairClasses];
  int n_all_pairs[kPairClasses] = {};
  DevBuf d_mol_atm, d_mol_natm;
  DevBuf d_one_scratch;           // raw Cartesian S, T, V (3 x cart_stride)
  DevBuf d_one_dens;              // raw Cartesian D, W (2 x cart_stride)
  // scratch
  DevBuf d_dens, d_dens_f, d_vj, d_vk;
  int scratch_nb = 0;
  // bumped whenever device work-item arrays are rebuilt or rewritten
  // (autotune, set_shard): a CUDA graph captured before then is stale
  unsigned long long layout_gen = 0;
  // work-queue counters of the persistent launches: one per unit and slice
  DevBuf d_queue;            // kQueueSlots ints, allocated with the plan
  unsigned next_queue = 0;
  double last_fp32_cut = 0.0;   // fp32_cut of the last split-precision build (split statistics)
  // optional per-class launch timing (CUDA events on the launching stream)
  bool profiling = false;
  std::vector<ProfileEvent> events;
  ~Plan() {
    for (int i = 0; i < kAuxStreams; ++i) {
      if (aux[i]) cudaStreamDestroy(aux[i]);
      if (join_ev[i]) cudaEventDestroy(join_ev[i]);
    }
    if (fork_ev) cudaEventDestroy(fork_ev);
    for (auto* w : work) delete w;
    for (auto& e : events) {
      cudaEventDestroy(e.start);
      cudaEventDestroy(e.stop);
    }
  }
};

void check_jk_args(const Plan& p, const double* d_in, int nb, const double* d_out, int with_j,
                   int with_k, int precision, double fp32_cut);
void run_jk_core(Plan& p, const double* d_in, int nb, double* d_out, int with_j, int with_k,
                 int hermi, int precision, double fp32_cut, cudaStream_t st, double* s_dens,
                 float* s_dens_f, double* s_vj, double* s_vk, bool allow_profiling);
int guarded_call(const std::function<void()>& f);
// coordinate JVP (mode 0: order 1, 1: order 2) and order-2 VJP (mode 2) of
// one class pair's expanded work items (geom.cu)
int launch_geom(const JKArgs& args, int la, int lb, int lc, int ld, int mode, cudaStream_t st);
size_t geom_smem_bytes(int la, int lb, int lc, int ld);
void fail_invalid(const std::string& m);

// Device-wide constant tables (Rys, Boys, c2s) of the current device.
const Tables& device_tables(int device);

void set_error(const std::string& msg);

}  // namespace b200jk

// The C ABI's opaque plan handle.
struct b200jk_plan {
  b200jk::Plan* p;
};
