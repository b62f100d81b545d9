/*
 * b200jk -- B200-native (sm_100a) direct-SCF Coulomb/exchange build.
 *
 * Plain C ABI over raw pointers: host arrays for the libcint-layout tables,
 * device pointers (caller-owned, stream-ordered) for densities and results.
 * Every entry point returns 0 on success or a nonzero b200jk_status; the
 * message of the calling thread's last failure is b200jk_last_error().
 *
 * Reference interfaces replaced (paths inside the reference's
 * src/gradscf/integrals/_native/):
 *   GradSCFDirectJK            csrc/direct_jk.cc:97-102   ("gradscf_direct_jk_cpu_v1")
 *   GradSCFDirectJKGeometryVJPParallel
 *                              csrc/direct_jk_geometry.cc:194-201 ("..._geometry_vjp_cpu_v2")
 * Table layout (atm rows of 6 int32, bas rows of 8 int32, env float64) is
 * libcint's, validated as csrc/tables.h:31-76 validates it.
 */
#ifndef B200JK_H
#define B200JK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  B200JK_OK = 0,
  B200JK_INVALID_ARGUMENT = 1, /* reference: ffi::Error::InvalidArgument */
  B200JK_INTERNAL = 2,         /* reference: ffi::Error::Internal (CUDA failure, device status) */
  B200JK_UNSUPPORTED = 3       /* valid input outside this build (l > 3, omega != 0) */
} b200jk_status;

/* Precision of the ERI evaluation.  J/K accumulation is FP64 in every mode. */
typedef enum {
  B200JK_FP64 = 0,  /* every quartet in FP64 */
  B200JK_SPLIT = 1  /* quartets with Q_ij*Q_kl*max|D| < fp32_cut in FP32, the rest FP64 */
} b200jk_precision;

typedef struct b200jk_plan b200jk_plan;

/* One molecule's libcint tables (host memory; copied during plan creation). */
typedef struct {
  const int32_t* atm; int32_t natm;
  const int32_t* bas; int32_t nbas;
  const double* env;  int32_t nenv;
} b200jk_molecule;

/* Message of this thread's last failure ("" if none). */
const char* b200jk_last_error(void);

/* Build a device-resident plan for one molecule or a batch of independent
 * molecules: validated tables, split general contractions, primitive-pair
 * data, Schwarz bounds Q_ij = sqrt(max |(ab|ab)|) (the reference's
 * eri_schwarz_bounds, csrc/coulomb_shells.h:60-77) and the sorted
 * significant-pair lists with their work items for `schwarz_cut`
 * (quartets with Q_ij*Q_kl < schwarz_cut are skipped, as unique_eri does,
 * csrc/coulomb_shells.h:200-212).  Rebuild when coordinates change.
 * `device` is the CUDA ordinal the plan lives on. */
int b200jk_plan_create(const b200jk_molecule* mols, int32_t nmol, int32_t cart,
                       double schwarz_cut, int32_t device, b200jk_plan** out);
void b200jk_plan_destroy(b200jk_plan* plan);

/* Plan facts: output AO count of molecule `mol`, and the number of
 * significant canonical shell quartets (i>=j, k>=l, ij>=kl, Q_ij Q_kl >= cut,
 * counted on the reference's shells) -- the unit of the quartets/s metric. */
int b200jk_plan_nao(const b200jk_plan* plan, int32_t mol, int32_t* nao);
int b200jk_plan_quartets(const b200jk_plan* plan, int64_t* count);
/* Per-molecule output block offsets into the packed density / J / K layout
 * (molecule m occupies [offset[m], offset[m] + nao[m]^2) of each matrix). */
int b200jk_plan_block_offsets(const b200jk_plan* plan, int64_t* offsets);

/* Per angular-momentum class pair (index x(x+1)/2 + y of the pair classes
 * x >= y, pair class l_a(l_a+1)/2 + l_b; 55 entries): significant quartets of
 * split-contraction shells and their primitive quartets.  For the FLOP model. */
int b200jk_plan_class_stats(const b200jk_plan* plan, int64_t* quartets, int64_t* prim_quartets);

/* Multi-GPU sharding of one J/K build (replaces the reference's per-process
 * row-range worker ownership, csrc/direct_jk.cc:26-92, across devices).
 * b200jk_partition_items: host-only; assigns n work items with the given
 * costs to `world` ranks in contiguous, cost-balanced blocks (owner[i] in
 * [0, world)).  b200jk_plan_set_shard: from now on the plan evaluates only
 * rank `rank`'s items of every class pair (costs = primitive quartets), so
 * the J/K it returns is this rank's partial sum; the caller sums the ranks'
 * outputs (one all-reduce).  (0, 1) restores the whole build.  Graphs
 * created before the call must be recreated (their launch is refused). */
int b200jk_partition_items(const int64_t* cost, int64_t n, int32_t world, int32_t* owner);
int b200jk_plan_set_shard(b200jk_plan* plan, int32_t rank, int32_t world);

/* Autotuner for the register-path tile shape (no counterpart in the
 * reference, whose CPU loop has no tiles): for every class pair on the
 * register path, times its kernels on `d_density` (nb packed matrices, the
 * workload the plan will serve, e.g. an SCF iteration's dD) with 32, 64 and
 * 128 kets per work item (`reps` timed launches after one warm-up each) and
 * keeps the fastest.  chunks[55] (or NULL) receives the choice per class pair,
 * -1 where not tuned.  Synchronises `stream`; call it before creating graphs
 * (graphs created earlier must be recreated) and after set_shard. */
int b200jk_plan_autotune(b200jk_plan* plan, const double* d_density, int32_t nb, int32_t hermi,
                         int32_t precision, double fp32_cut, int32_t reps, void* stream, int32_t* chunks);

/* After a B200JK_SPLIT call (synchronises `stream`): per class pair, the
 * quartets and primitive quartets that ran in FP64 and in FP32. */
int b200jk_plan_split_stats(b200jk_plan* plan, void* stream, int64_t* q64, int64_t* q32,
                            int64_t* pq64, int64_t* pq32);

/* After a B200JK_SPLIT call (synchronises `stream`): the FP64 quartets that
 * ran one per lane from the flat lists (`listed`; list slots, including the
 * filler of a reservation that did not fit) and the quartets whose
 * reservation did not fit (`overflow`; they ran on the bra-group path). */
int b200jk_plan_border_stats(b200jk_plan* plan, void* stream, int64_t* listed, int64_t* overflow);

/* Optional CUDA-event timing of every class-pair launch (on the launching
 * stream).  b200jk_plan_profile synchronises, returns per class pair the
 * summed milliseconds of FP64 and FP32 launches and the launch counts since
 * the last read, then resets. */
int b200jk_plan_set_profiling(b200jk_plan* plan, int32_t on);
int b200jk_plan_profile(b200jk_plan* plan, double* ms64, double* ms32, int32_t* launches);

/* Packed four-centre ERIs of a one-molecule plan (replaces packed_eri,
 * csrc/packed_eri.cc:5-14): layout 0 = s4 (np x np), 1 = s8 (np(np+1)/2),
 * np = n(n+1)/2 output AO pairs, pair(i,j) = i(i+1)/2 + j for i >= j.
 * out_size must equal the layout's element count.  d_out is zeroed first;
 * quartets below the plan's Schwarz cut stay zero (the reference uses
 * cut 0 here). */
int b200jk_packed_eri(b200jk_plan* plan, int32_t layout, double* d_out, int64_t out_size, void* stream);

/* J/K from packed ERIs (replaces PackedJK, csrc/packed_jk.cc:6-80): d_eri in
 * the s4 / s8 layout above (eri_size elements), nb real (n, n) densities
 * (nonsymmetric allowed), d_out (with_j + with_k, nb, n, n) overwritten.
 * No plan needed. */
int b200jk_packed_jk(const double* d_eri, int32_t layout, int64_t eri_size, int32_t n,
                     const double* d_density, int32_t nb, double* d_out, int32_t with_j,
                     int32_t with_k, void* stream);

/* Number of kernels one b200jk_direct_jk call launches on this plan (and
 * shard) in `precision` mode. */
int b200jk_plan_launches(const b200jk_plan* plan, int32_t precision, int64_t* count);

/* Probe for the tensor-core decision on the high-l horizontal transfer (no
 * counterpart in the reference): times the f x f bra transfer of the 2D
 * integrals (16 outputs from 7 inputs per root/axis/ket column, FP64) over
 * `ncol` columns x `reps`, as the scalar recursion (ns_per_column[0]) and as a
 * GEMM on the FP64 tensor cores (mma.sync DMMA, ns_per_column[1]), and
 * returns the largest difference between the two results. */
int b200jk_measure_bra_transfer(int32_t ncol, int32_t reps, double* ns_per_column, double* max_abs_diff,
                                void* stream);

/* Measured vector-pipe FMA throughput of the current device in TFLOP/s
 * (fp64 = 1: FP64, 0: FP32) -- the roofline denominator for the ERI kernels. */
int b200jk_measure_fma_peak(int32_t fp64, double* tflops, void* stream);

/* Direct J/K (replaces GradSCFDirectJK, csrc/direct_jk.cc:7-95).
 *   d_density : device, nb packed density sets (nb x sum_m nao_m^2, row-major
 *               per molecule; for one molecule simply (nb, n, n)).  Need not be
 *               symmetric unless hermi = 1 promises it.
 *   d_out     : device, (with_j + with_k, nb, ...) like the reference's result
 *               buffer: J first, then K; fully overwritten.
 *   precision : B200JK_FP64 or B200JK_SPLIT (fp32_cut used only for SPLIT).
 *   stream    : cudaStream_t (NULL = legacy default stream).
 * Asynchronous: returns after enqueueing; a nonfinite density is reported
 * through b200jk_check_status (or by a later synchronous call). */
int b200jk_direct_jk(b200jk_plan* plan, const double* d_density, int32_t nb, double* d_out,
                     int32_t with_j, int32_t with_k, int32_t hermi, int32_t precision,
                     double fp32_cut, void* stream);

/* Allocation-free variant of b200jk_direct_jk.  No counterpart in the
 * reference (its CPU handler allocates per call).  For callers that may not
 * allocate device memory while they run -- an XLA custom call on a stream
 * XLA owns, code inside CUDA stream capture, a host with a fixed memory
 * budget.  Same arguments and results as b200jk_direct_jk, but the scratch
 * (effective densities and J/K accumulators) lives in a static device array
 * of B200JK_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
 * until exit; a call needing more returns B200JK_INVALID_ARGUMENT with the
 * byte counts.  The plan must already exist (plan creation allocates).
 * All calls share the array: calls that overlap on the GPU race, so order
 * them on one stream.  A call also uses the plan's small device state (row
 * maxima, status word, FP32 boundaries), so it also races with any other
 * build on the same plan that overlaps it on the GPU.  The first call on a
 * device looks up the array's address with that device current -- make it
 * before any stream capture.  The caller's current device is restored. */
#define B200JK_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int b200jk_direct_jk_noalloc(b200jk_plan* plan, const double* d_density, int32_t nb, double* d_out,
                             int32_t with_j, int32_t with_k, int32_t hermi, int32_t precision,
                             double fp32_cut, void* stream);

/* CUDA-graph capture of one complete J/K build (density transform, every
 * class-pair kernel, finalisation) for fixed device buffers, replayed once
 * per SCF iteration: the reference runs one FFI call per iteration
 * (scf/rks.py:305-321); here the caller copies the next density into
 * d_density and launches the graph.  Creation allocates the graph's own
 * scratch and runs one eager build before capturing, so later builds on the
 * plan with more densities leave the graph valid.  The graph shares the
 * plan's work items and small device state: do not run another build on the
 * same plan concurrently, and after b200jk_plan_autotune or
 * b200jk_plan_set_shard (which rebuild the work items) b200jk_graph_launch
 * refuses with B200JK_INVALID_ARGUMENT -- destroy and recreate the graph. */
typedef struct b200jk_graph b200jk_graph;
int b200jk_graph_create(b200jk_plan* plan, const double* d_density, int32_t nb, double* d_out,
                        int32_t with_j, int32_t with_k, int32_t hermi, int32_t precision,
                        double fp32_cut, b200jk_graph** out);
int b200jk_graph_launch(b200jk_graph* graph, void* stream);
void b200jk_graph_destroy(b200jk_graph* graph);

/* Synchronise `stream` and turn the plan's device status word into a return
 * code (nonfinite density -> B200JK_INVALID_ARGUMENT), clearing it. */
int b200jk_check_status(b200jk_plan* plan, void* stream);

/* One-shot drop-in with the reference handler's argument list
 * (csrc/direct_jk.cc:7-11 + 97-102): builds a plan, runs FP64 J/K, checks the
 * density, destroys the plan.  `workers` is accepted for ABI parity (must be
 * >= 1) and ignored.  Synchronous. */
int b200jk_direct_jk_tables(const int32_t* atm, int32_t natm, const int32_t* bas, int32_t nbas,
                            const double* env, int32_t nenv, const double* d_density, int32_t nb,
                            int32_t n, double* d_out, int32_t cart, double cutoff, int32_t workers,
                            int32_t with_j, int32_t with_k, void* stream);

/* Coordinate VJP of J/K (replaces gradscf_direct_jk_geometry_vjp_cpu_v2,
 * csrc/direct_jk_geometry.cc:122-182): for cotangents Jbar, Kbar
 * (d_cot: (with_j + with_k, nb, ...), same layout as d_out above) returns
 *   g[R] = sum_abcd d(ab|cd)/dR (Jbar_ab D_cd + Kbar_ac D_bd)
 * for every centre atom row of every molecule's atm table.
 *   d_grad : device, (sum_m natm_m, 3), fully overwritten.
 * Unlike the reference (which demands cutoff 0), the plan's Schwarz cut is
 * applied; a plan built with cut 0 reproduces the reference exactly. */
int b200jk_direct_jk_geom_vjp(b200jk_plan* plan, const double* d_density, int32_t nb,
                              const double* d_cot, int32_t with_j, int32_t with_k, double* d_grad,
                              void* stream);

/* The same VJP in split precision (precision = B200JK_SPLIT): per work item,
 * the quartets with Q_bra Q_ket M < fp32_cut run in FP32, M = 8 nb
 * max(|D|, 2|Jbar|, 2|Kbar|)^2 over the rows and columns of the item's A, B
 * and C shells (a bound on |Gamma|); the rest, and every accumulation across
 * quartets, in FP64.  B200JK_FP64 is b200jk_direct_jk_geom_vjp.  No reference
 * counterpart (the reference's VJP is FP64). */
int b200jk_direct_jk_geom_vjp_precision(b200jk_plan* plan, const double* d_density, int32_t nb,
                                        const double* d_cot, int32_t with_j, int32_t with_k, int32_t precision,
                                        double fp32_cut, double* d_grad, void* stream);

/* Coordinate JVP of J/K (replaces gradscf_direct_jk_geometry_jvp_cpu_v1 with
 * order 1 and 2, csrc/direct_jk_geometry.cc:8-99):
 *   d_v == NULL : d_out = d/du (J, K)           (order 1)
 *   d_v != NULL : d_out = d^2/(du dv) (J, K)    (order 2)
 * at fixed density.  d_u, d_v: device, (sum_m natm_m, 3) coordinate directions
 * per atm row (the coordinate slots of the reference's env-sized
 * direction).  d_density / d_out / hermi as for b200jk_direct_jk.  The
 * plan's Schwarz cut applies (cut 0 reproduces the reference). */
int b200jk_direct_jk_geom_jvp(b200jk_plan* plan, const double* d_density, int32_t nb, int32_t hermi,
                              const double* d_u, const double* d_v, int32_t with_j, int32_t with_k,
                              double* d_out, void* stream);

/* Order-2 coordinate VJP (Hessian-vector product; replaces the order-2 branch
 * of gradscf_direct_jk_geometry_vjp_cpu_v2, csrc/direct_jk_geometry.cc:59-99
 * over csrc/geometry_contraction.h:7-53): for cotangents (Jbar, Kbar) in d_cot
 * (as for b200jk_direct_jk_geom_vjp) and a coordinate direction d_u,
 *   d_grad[R] = d/dR sum(Jbar * dJ/du + Kbar * dK/du),  (sum_m natm_m, 3). */
int b200jk_direct_jk_geom_hvp(b200jk_plan* plan, const double* d_density, int32_t nb, const double* d_u,
                              const double* d_cot, int32_t with_j, int32_t with_k, double* d_grad,
                              void* stream);

/* One-electron matrices in the plan's output basis (sum_m nao_m^2 packed):
 * which = 0 overlap, 1 kinetic, 2 nuclear attraction (atoms with nonzero
 * charge in the atm table, point nuclei). */
int b200jk_int1e(b200jk_plan* plan, int32_t which, double* d_out, void* stream);

/* Gradient of sum_ab [ D_ab h_ab - W_ab S_ab ] with respect to every atm row
 * (h = kinetic + nuclear attraction, including the Hellmann-Feynman operator
 * derivative of the nuclear attraction).  d_grad: (sum_m natm_m, 3), overwritten. */
int b200jk_int1e_grad(b200jk_plan* plan, const double* d_density, const double* d_energy_weighted,
                      double* d_grad, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* B200JK_H */
