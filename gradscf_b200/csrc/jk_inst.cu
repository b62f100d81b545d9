// Instantiates the J/K kernels of one class pair (BRA_CLASS >= KET_CLASS,
// compiled once per pair so the classes build in parallel) and registers
// their launchers in the dispatch table.
#include <algorithm>

#include "dispatch.h"
#include "grad_kernels.cuh"
#include "jk_kernels.cuh"

#if !defined(BRA_CLASS) || !defined(KET_CLASS)
#error "compile with -DBRA_CLASS=<0..9> -DKET_CLASS=<0..BRA_CLASS>"
#endif

namespace b200jk {

namespace {

constexpr int pc_la(int pc) { return pc == 0 ? 0 : pc <= 2 ? 1 : pc <= 5 ? 2 : 3; }
constexpr int pc_lb(int pc) { return pc - pc_la(pc) * (pc_la(pc) + 1) / 2; }

// Kernel shape policy: a register path for blocks that fit one thread,
// otherwise a team whose lanes hold about 24 outputs each.
#ifndef B200JK_REG_LIMIT32
#define B200JK_REG_LIMIT32 240
#endif
template <int LA, int LB, int LC, int LD, typename R = double>
struct Policy {
  using CI = ClassInfo<LA, LB, LC, LD>;
  // FP32 blocks take half the registers of FP64 ones: a larger register-path
  // limit (measured on (H2O)32 cc-pVDZ: (11|11), (21|11), (21|20), (22|10)
  // run 3-6x faster there than on the tile path)
  static constexpr int LIMIT = sizeof(R) == 4 ? B200JK_REG_LIMIT32 : 96;
  static constexpr bool REG = (3 * CI::NG + CI::NOUT <= LIMIT) && CI::NROOT <= 3;
  // tile path: kets up to d x d (NCD <= 36), bra pair fits one block; FP32
  // accumulators take half the registers, so FP32 takes kets up to f x s / d x p
#ifndef B200JK_TILE_NCD32
#define B200JK_TILE_NCD32 100   // measured on (H2O)8 cc-pVTZ: split kernels 92.5 -> 84.8 ms
#endif
#ifndef B200JK_TILE_NCD64
#define B200JK_TILE_NCD64 100  // measured on (H2O)8 cc-pVTZ: FP64 kernels 102.0 -> 91.4 ms (despite spills)
#endif
  static constexpr int TILE_NCD = sizeof(R) == 4 ? B200JK_TILE_NCD32 : B200JK_TILE_NCD64;
  static constexpr bool TILE = !REG && CI::NCD <= TILE_NCD && CI::NAB <= 128;
  static constexpr int TEAM = CI::NOUT <= 4 * 24 ? 4 : CI::NOUT <= 8 * 24 ? 8 : CI::NOUT <= 16 * 24 ? 16 : 32;
};

template <int LA, int LB, int LC, int LD, typename R>
int launch_class(const JKArgs& args, cudaStream_t stream) {
  if (args.nwork <= 0) return 0;
  using P = Policy<LA, LB, LC, LD, R>;
  if constexpr (P::REG) {
    jk_reg_kernel<LA, LB, LC, LD, R><<<(args.nwork + kRegWarps - 1) / kRegWarps, 32 * kRegWarps, 0, stream>>>(args);
  } else if constexpr (P::TILE) {
    using TC = TileCfg<LA, LB, LC, LD, R>;
    constexpr size_t smem = TC::bytes();
    static std::atomic<uint64_t> smem_done{0};
    smem_opt_in(jk_tile_kernel<LA, LB, LC, LD, R>, smem, smem_done);
    jk_tile_kernel<LA, LB, LC, LD, R><<<args.nwork, TC::THREADS, smem, stream>>>(args);
  } else {
    constexpr int TEAM = P::TEAM;
    using SM = TeamSmem<LA, LB, LC, LD, R, TEAM>;
    constexpr size_t per_team = SM::bytes();
    int teams = 128 / TEAM;
    while (teams > 1 && per_team * teams > 200 * 1024) --teams;
    const size_t smem = per_team * teams;
    static std::atomic<uint64_t> smem_done{0};
    smem_opt_in(jk_team_kernel<LA, LB, LC, LD, R, TEAM>, smem, smem_done);
    jk_team_kernel<LA, LB, LC, LD, R, TEAM><<<args.nwork, teams * TEAM, smem, stream>>>(args);
  }
  return (int)cudaGetLastError();
}

template <int LA, int LB, int LC, int LD>
int launch_store(const JKArgs& args, int cart, int layout, double* out, long long npair, cudaStream_t stream) {
  if (args.nwork <= 0) return 0;
  using CI = ClassInfo<LA, LB, LC, LD>;
  constexpr int TEAM = Policy<LA, LB, LC, LD>::TEAM;
  using SM = TeamSmem<LA, LB, LC, LD, double, TEAM>;
  constexpr size_t per_team = SM::bytes() + (size_t)CI::NOUT * 8;
  int teams = 128 / TEAM;
  while (teams > 1 && per_team * teams > 200 * 1024) --teams;
  const size_t smem = per_team * teams;
  static std::atomic<uint64_t> smem_done{0};
  smem_opt_in(eri_store_kernel<LA, LB, LC, LD, TEAM>, smem, smem_done);
  eri_store_kernel<LA, LB, LC, LD, TEAM><<<args.nwork, teams * TEAM, smem, stream>>>(args, cart, layout, out, npair);
  return (int)cudaGetLastError();
}

// Persistent launches of the bra-group kernels: at most one wave of resident
// blocks; their warps take items from args.queue (zeroed by the caller).
template <int LA, int LB, int LC, int LD, typename R>
int launch_grp(const JKArgs& args, cudaStream_t stream) {
  if (args.nwork <= 0) return 0;
  static std::atomic<int> resident[64];
  const int wave = persistent_blocks(jk_grp_kernel<LA, LB, LC, LD, R>, 32 * kRegWarps, 0, resident);
  const int blocks = std::min((args.nwork + kRegWarps - 1) / kRegWarps, wave);
  jk_grp_kernel<LA, LB, LC, LD, R><<<blocks, 32 * kRegWarps, 0, stream>>>(args);
  return (int)cudaGetLastError();
}

template <int LA, int LB, int LC, int LD, typename R, int GB, int GK>
int launch_grp_gen(const JKArgs& args, cudaStream_t stream) {
  if (args.nwork <= 0) return 0;
  constexpr size_t smem = (size_t)kRegWarps * GrpGenAcc<LA, LB, LC, LD, GB, GK>::N * 32 * sizeof(R);
  // static caches plus these pass sums pass 48 KB for most buckets: opt in
  // (to at least 64 KB of dynamic shared memory) for every one
  static std::atomic<uint64_t> smem_done{0};
  const cudaError_t ea =
      smem_opt_in(jk_grp_gen_kernel<LA, LB, LC, LD, R, GB, GK>, std::max(smem, (size_t)64 * 1024), smem_done);
  if (ea != cudaSuccess) return (int)ea;
  static std::atomic<int> resident[64];
  const int wave = persistent_blocks(jk_grp_gen_kernel<LA, LB, LC, LD, R, GB, GK>, 32 * kRegWarps, smem, resident);
  const int blocks = std::min((args.nwork + kRegWarps - 1) / kRegWarps, wave);
  jk_grp_gen_kernel<LA, LB, LC, LD, R, GB, GK><<<blocks, 32 * kRegWarps, smem, stream>>>(args);
  return (int)cudaGetLastError();
}

// The FP64 flat list of a split build: its length is on the device, so the
// grid is one wave of resident blocks, sized for the list's capacity.
template <int LA, int LB, int LC, int LD, int GB, int GK>
int launch_flat(const JKArgs& args, cudaStream_t stream) {
  if (args.flat_cap <= 0) return 0;
  static std::atomic<int> resident[64];
  const int wave = persistent_blocks(jk_flat_kernel<LA, LB, LC, LD, GB, GK>, 128, 0, resident);
  const int blocks = std::min((args.flat_cap + 127) / 128, wave);
  jk_flat_kernel<LA, LB, LC, LD, GB, GK><<<blocks, 128, 0, stream>>>(args);
  return (int)cudaGetLastError();
}

template <int LA, int LB, int LC, int LD, typename R, int GB, int GK>
int launch_gen(const JKArgs& args, cudaStream_t stream) {
  if (args.nwork <= 0) return 0;
  jk_reg_gen_kernel<LA, LB, LC, LD, R, GB, GK>
      <<<(args.nwork + kRegWarps - 1) / kRegWarps, 32 * kRegWarps, 0, stream>>>(args);
  return (int)cudaGetLastError();
}

#if BRA_CLASS == KET_CLASS
template <int LA, int LB>
int launch_schwarz(const JKArgs& args, int npairs, int cart, cudaStream_t stream) {
  if (npairs <= 0) return 0;
  constexpr int TEAM = Policy<LA, LB, LA, LB>::TEAM;
  using SM = TeamSmem<LA, LB, LA, LB, double, TEAM>;
  constexpr size_t per_team = SM::bytes();
  int teams = 128 / TEAM;
  while (teams > 1 && per_team * teams > 200 * 1024) --teams;
  const size_t smem = per_team * teams;
  static std::atomic<uint64_t> smem_done{0};
  smem_opt_in(schwarz_kernel<LA, LB, TEAM>, smem, smem_done);
  const int blocks = (npairs + teams - 1) / teams;
  schwarz_kernel<LA, LB, TEAM><<<blocks, teams * TEAM, smem, stream>>>(args, npairs, cart);
  return (int)cudaGetLastError();
}
#endif

// The coordinate VJP of one class pair in precision R (FP32: the split
// slice of small-bound quartets); the kernel family per class is the same
// in both precisions, shared memory scales with sizeof(R).
template <int LA, int LB, int LC, int LD, typename R>
int launch_grad(const JKArgs& args, cudaStream_t stream) {
  if (args.nwork <= 0) return 0;
  constexpr size_t RS = sizeof(R);
#ifndef B200JK_GRAD_LANE
#define B200JK_GRAD_LANE 1
#endif
  if constexpr (B200JK_GRAD_LANE && GradLane<LA, LB, LC, LD>::OK) {
    // mid-size classes: one lane per quartet, Gamma in shared memory
    using GL = GradLane<LA, LB, LC, LD>;
    constexpr size_t smem = GL::bytes() / 8 * RS;
    static std::atomic<uint64_t> smem_done{0};
    const cudaError_t ea = smem_opt_in(grad_lane_kernel<LA, LB, LC, LD, R>, smem, smem_done);
    if (ea != cudaSuccess) return (int)ea;
    grad_lane_kernel<LA, LB, LC, LD, R><<<(args.nwork + GL::THREADS / 32 - 1) / (GL::THREADS / 32), GL::THREADS,
                                          smem, stream>>>(args);
    return (int)cudaGetLastError();
  }
  if constexpr (GradReg<LA, LB, LC, LD>::OK) {
    grad_reg_kernel<LA, LB, LC, LD, R><<<(args.nwork + 3) / 4, 128, 0, stream>>>(args);
    return (int)cudaGetLastError();
  }
#ifndef B200JK_GRAD_WARP
#define B200JK_GRAD_WARP 1
#endif
  if constexpr (B200JK_GRAD_WARP && GradWarp<LA, LB, LC, LD>::OK) {
    // the classes between: one warp per quartet, derivative tables in shared memory
    using GW = GradWarp<LA, LB, LC, LD>;
    constexpr size_t smem = GW::bytes() / 8 * RS;
    static std::atomic<uint64_t> smem_done{0};
    const cudaError_t ea = smem_opt_in(grad_warp_kernel<LA, LB, LC, LD, R>, smem, smem_done);
    if (ea != cudaSuccess) return (int)ea;
    grad_warp_kernel<LA, LB, LC, LD, R><<<args.nwork, 32 * GW::WARPS, smem, stream>>>(args);
    return (int)cudaGetLastError();
  }
#ifndef B200JK_GRAD_BLOCK
#define B200JK_GRAD_BLOCK 1
#endif
  if constexpr (B200JK_GRAD_BLOCK && GradBlk<LA, LB, LC, LD>::OK) {
    // large classes: one quartet per block at a time (block-wide teams)
    using GB = GradBlk<LA, LB, LC, LD>;
    constexpr size_t smem = GB::bytes() / 8 * RS;
    static std::atomic<uint64_t> smem_done{0};
    const cudaError_t ea = smem_opt_in(grad_block_kernel<LA, LB, LC, LD, R>, smem, smem_done);
    if (ea != cudaSuccess) return (int)ea;
    grad_block_kernel<LA, LB, LC, LD, R><<<args.nwork, GB::THREADS, smem, stream>>>(args);
    return (int)cudaGetLastError();
  }
  using CI = ClassInfo<LA, LB, LC, LD>;
  constexpr int TEAM = CI::NOUT <= 8 ? 4 : CI::NOUT <= 64 ? 8 : CI::NOUT <= 256 ? 16 : 32;
  using GC = GradCfg<LA, LB, LC, LD, TEAM>;
  constexpr size_t per_team = GC::bytes() / 8 * RS;
  int teams = 128 / TEAM;
  while (teams > 1 && per_team * teams > 200 * 1024) --teams;
  const size_t smem = per_team * teams;
  static std::atomic<uint64_t> smem_done{0};
  const cudaError_t ea = smem_opt_in(grad_team_kernel<LA, LB, LC, LD, TEAM, R>, smem, smem_done);
  if (ea != cudaSuccess) return (int)ea;
  grad_team_kernel<LA, LB, LC, LD, TEAM, R><<<args.nwork, teams * TEAM, smem, stream>>>(args);
  return (int)cudaGetLastError();
}

constexpr int X = BRA_CLASS;
constexpr int Y = KET_CLASS;
static_assert(Y <= X, "ket class must not exceed bra class");
constexpr int XA = pc_la(X), XB = pc_lb(X);
constexpr int YA = pc_la(Y), YB = pc_lb(Y);

// Grouped lists: both precisions on the register path and an (l, 0) side;
// up to 4 combinations on a (0, 0) pair, 2 on other (l, 0) pairs.
constexpr bool GROUPED = Policy<XA, XB, YA, YB, float>::REG && Policy<XA, XB, YA, YB>::REG && (XB == 0 || YB == 0);

constexpr int gslot(int g) { return g == 1 ? 0 : (g == 2 ? 1 : 2); }

// The register path over bra groups: both precisions on the register path.
#ifndef B200JK_GRP
#define B200JK_GRP 1
#endif
// The per-lane pass sums (GrpAcc::N values of 32 lanes, 4 warps) stay within
// 32 KB of static shared memory in FP64.
constexpr bool GRP = B200JK_GRP && Policy<XA, XB, YA, YB, float>::REG && Policy<XA, XB, YA, YB>::REG &&
                     GrpAcc<XA, XB, YA, YB>::N <= 32;
#ifndef B200JK_GRP_GEN
#define B200JK_GRP_GEN 1
#endif
constexpr bool GRP_GEN = B200JK_GRP_GEN && GRP;

template <int GB, int GK>
void register_gen(DispatchTable& t, int id) {
  constexpr bool okb = GB == 1 || (XB == 0 && (GB == 2 || X == 0));
  constexpr bool okk = GK == 1 || (YB == 0 && (GK == 2 || Y == 0));
  if constexpr (GROUPED && okb && okk && !(GB == 1 && GK == 1)) {
    t.jkg64[id][3 * gslot(GB) + gslot(GK)] = &launch_gen<XA, XB, YA, YB, double, GB, GK>;
    t.jkg32[id][3 * gslot(GB) + gslot(GK)] = &launch_gen<XA, XB, YA, YB, float, GB, GK>;
    // pass sums (N x 32 lanes x 4 warps) in dynamic shared memory.  Up to 26
    // per lane: wider buckets measured 3-8% faster in the FP32 slices with up
    // to 2 ket combinations but 30-48% slower with 4, and the (H2O)64 cc-pVTZ
    // FP64 build 8% slower (11.9 -> 12.9 s), so they keep the per-quartet form
    constexpr int NACC = GrpGenAcc<XA, XB, YA, YB, GB, GK>::N;
    if constexpr (GRP_GEN && NACC <= 26) {
      t.grpg64[id][3 * gslot(GB) + gslot(GK)] = &launch_grp_gen<XA, XB, YA, YB, double, GB, GK>;
      t.grpg32[id][3 * gslot(GB) + gslot(GK)] = &launch_grp_gen<XA, XB, YA, YB, float, GB, GK>;
      t.flat64[id][3 * gslot(GB) + gslot(GK)] = &launch_flat<XA, XB, YA, YB, GB, GK>;
    }
  }
}

}  // namespace

#define CAT4(a, b, c, d) a##b##c##d
#define REG_NAME(x, y) CAT4(register_jk_class_, x, _, y)
void REG_NAME(BRA_CLASS, KET_CLASS)(DispatchTable& t) {
  const int id = X * (X + 1) / 2 + Y;
  t.jk64[id] = &launch_class<XA, XB, YA, YB, double>;
  t.jk32[id] = &launch_class<XA, XB, YA, YB, float>;
  if constexpr (GRP) {
    t.grp64[id] = &launch_grp<XA, XB, YA, YB, double>;
    t.grp32[id] = &launch_grp<XA, XB, YA, YB, float>;
    t.flat64[id][0] = &launch_flat<XA, XB, YA, YB, 1, 1>;
  }
  t.grad64[id] = &launch_grad<XA, XB, YA, YB, double>;
  t.grad32[id] = &launch_grad<XA, XB, YA, YB, float>;
  t.store[id] = &launch_store<XA, XB, YA, YB>;
  t.reg_path[id] = Policy<XA, XB, YA, YB, float>::REG || Policy<XA, XB, YA, YB>::REG;
  t.tile[id] = Policy<XA, XB, YA, YB>::TILE;
  t.grouped[id] = GROUPED;
  register_gen<1, 2>(t, id);
  register_gen<1, 4>(t, id);
  register_gen<2, 1>(t, id);
  register_gen<2, 2>(t, id);
  register_gen<2, 4>(t, id);
  register_gen<4, 1>(t, id);
  register_gen<4, 2>(t, id);
  register_gen<4, 4>(t, id);
  t.team[id] = Policy<XA, XB, YA, YB>::REG ? 1
               : (Policy<XA, XB, YA, YB>::TILE ? TileCfg<XA, XB, YA, YB, double>::THREADS / 4
                                               : Policy<XA, XB, YA, YB>::TEAM);
#if BRA_CLASS == KET_CLASS
  t.schwarz[X] = &launch_schwarz<XA, XB>;
#endif
}

}  // namespace b200jk
