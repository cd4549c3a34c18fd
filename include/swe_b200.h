/*
 * swe_b200.h -- C ABI of the B200 (sm_100a) implementation of the RBF-FD
 * shallow-water RK4 hot path of cenamiller/RBF-FD-SWE.
 *
 * Reference interfaces replaced (paths within the reference project):
 *   RK_substep(H, K, F, D, id)     swe_code/main/include/rk4_rbffd_swe.h:8,
 *                                  swe_code/main/rk4_rbffd_swe.c:30-72
 *   eval_RHS_swe(K, F)             swe_code/main/rk4_rbffd_swe.c:189-362
 *                                  (external linkage, not in a header)
 *   RK_substep_ocl(..., substep)   swe_code/ocl/RK_ocl.c:9-51 (device precedent:
 *                                  buffers set once, state device-resident)
 *   static data of PSMD_struct     swe_code/main/include/swe_config.h:187-233
 *   layout macros DM_LIN_ID, VECT_LIN_ID, SVM_LIN_ID
 *                                  swe_code/main/include/swe_config.h:31-54
 *
 * Conventions.  Every entry point returns an int status (SWE_OK = 0) and never
 * exits the process; swe_cuda_last_error() describes the last failure.  Host
 * arrays are owned by the caller and use the caller's compile-time layout
 * (SWE_LAYOUT_* flags and the SIMD tile width), exactly as the reference's
 * LPSMD holds them.  The library owns all device memory and one CUDA stream;
 * calls come from one host thread.  fsize = sizeof(fType): 8 (FP64) or 4 (FP32),
 * which selects the arithmetic precision of the plain form.
 */
#ifndef SWE_B200_H
#define SWE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SWE_OK 0
#define SWE_ERR_ARG 1       /* invalid argument or size                        */
#define SWE_ERR_STATE 2     /* call out of order (e.g. step before init)       */
#define SWE_ERR_CUDA 3      /* CUDA runtime failure                            */
#define SWE_ERR_NOMEM 4     /* device allocation failed or budget exceeded     */
#define SWE_ERR_INDEX 5     /* stencil index outside the patch                 */
#define SWE_ERR_TIMEOUT 6   /* a bounded device wait ran out                   */
#define SWE_ERR_NONFINITE 7 /* NaN/Inf detected by a watchdog reduction        */
#define SWE_ERR_CANCELLED 8 /* request cancelled                               */

/* layout flags: the reference's USE_CFDL / USE_SFDL compile options */
#define SWE_LAYOUT_CFDL 1
#define SWE_LAYOUT_SFDL 2

const char* swe_cuda_last_error(void);

/* Selects the CUDA device for the calling thread's subsequent calls (one
 * process per GPU: call with the local rank before swe_cuda_init). */
int swe_cuda_select_device(int device);

/* ---------------------------------------------------------------------------
 * Plain drop-in form (one state, FP64 or FP32)
 * ------------------------------------------------------------------------- */

/* Uploads the static model data of one patch and canonicalises it for the
 * device.  Replaces the reference's implicit global LPSMD (rk4_rbffd_swe.c:19)
 * and the OpenCL buffer setup (ocl/buffers.c:26-49, main.c:318-322).
 * Arrays are laid out as swe_config.h:31-54 prescribes for `layout` with tile
 * width `simd_length`: x, y, z, f, ghm [compute_size]; p_u, p_v, p_w, gradghm
 * by VECT_LIN_ID; idx, Dx, Dy, Dz, L by DM_LIN_ID with row length padded_nnbr.
 * idx is 0-based and patch-local.  Weight columns j >= nnbr are never read
 * (the reference pads them by replicating the last column,
 * layout/matrix_transformations.c:20-21).  Requires nnbr <= 32.  Re-init
 * replaces the previous patch. */
int swe_cuda_init(int fsize, int layout, int simd_length,
                  int compute_size, int patch_size, int compute_pid_s,
                  int nnbr, int padded_nnbr, double gh0, double dt,
                  const void* x, const void* y, const void* z, const void* f, const void* ghm,
                  const void* p_u, const void* p_v, const void* p_w, const void* gradghm,
                  const int* idx, const void* Dx, const void* Dy, const void* Dz, const void* L);

/* State transfer, H of patch_size*4 values in the init layout (SVM_LIN_ID).
 * set_state writes H only.  The RK registers need no reset: the reference's
 * time loop copies H into K at the start of each attempt (main.c:297,
 * :308-314), and here stage 0 of every step reads H and writes K and D before
 * any later stage reads them, so K and D never carry values across set_state. */
int swe_cuda_set_state(const void* H);
int swe_cuda_get_state(void* H);

/* Parity entry point with eval_RHS_swe semantics: F = RHS(K).  K holds
 * patch_size*4 and F compute_size*4 values, both host pointers in the init
 * layout.  Synchronous. */
int swe_cuda_eval_rhs(const void* K, void* F);

/* One RK4 stage on the device-resident state; same stage semantics as
 * RK_substep (rk4_rbffd_swe.c:30-72).  The RHS, the stage combine and the
 * D/K (or H) update are one fused kernel per stage.  Asynchronous.  As in the
 * reference's time loop, a step calls substeps 0, 1, 2, 3 in order: substep k
 * reads the stage state that substep k-1 wrote. */
int swe_cuda_rk_substep(int substep_id);

/* Halo rows of a patch that is one part of a grid split across ranks (the
 * reference's MPI patches, mpi/init_patches.c:21-92): rows outside
 * compute_pid_s .. compute_pid_s + compute_size - 1 that the compute rows'
 * stencils read.  swe_cuda_rk_substep steps such a patch (H and the K buffers
 * hold all patch rows, D compute rows only, as in the reference); between
 * substeps the caller refreshes the halo rows of the buffer the next substep
 * reads, as the reference's exchange_SVM_halos does after eval_K and update_H
 * (mpi/halos.c:11-35):
 *   swe_cuda_halo_setup   patch rows this rank sends (compute rows) and
 *                         receives (halo rows), host arrays, checked; once;
 *   swe_cuda_halo_pack    the send rows of the buffer substep `substep_id`
 *                         reads -> send_buf, a [n_send][4] device buffer;
 *   swe_cuda_halo_unpack  recv_buf ([n_recv][4], device) -> the receive rows.
 * Pack and unpack are asynchronous on the library's stream (swe_cuda_sync
 * before handing the send buffer to a communication library).  After
 * substep s the next substep is (s + 1) % 4, and its buffer is what to
 * exchange.  Transport is the caller's (swe_b200/shard.py: NCCL send/recv over
 * NVLink, or gloo); nothing here reads another GPU's memory. */
int swe_cuda_halo_setup(const int* send_rows, int n_send, const int* recv_rows, int n_recv);
int swe_cuda_halo_pack(int substep_id, void* send_buf);
int swe_cuda_halo_unpack(int substep_id, const void* recv_buf);

/* nsteps full RK4 steps (4 stages each) from a captured CUDA graph.
 * Asynchronous; requires compute_pid_s == 0 and patch_size == compute_size
 * (no halo rows: a patch with halo rows steps by swe_cuda_rk_substep with
 * halo exchanges between substeps). */
int swe_cuda_step(int nsteps);

/* Waits for all work of the library's stream. */
int swe_cuda_sync(void);

/* Kernel choice.  0 = the bulk-copy pipelined stage kernel (a producer warp
 * streams each tile's weights, indices, pointwise data and state rows into
 * shared memory with cp.async.bulk; tiles of 64 nodes, one CTA per SM, of 32
 * nodes, two CTAs per SM, or of 16 nodes, four CTAs per SM); 1 = the
 * register-streaming kernel; 2 = the node-per-lane kernel (1, 2 or 4 lanes per
 * node, each summing its slots serially, from a tile-transposed copy of the
 * weights and indices).  Kernels 0 and 1 do the same arithmetic in the same
 * order; kernel 2 sums the slots in another order and meets the same error
 * bars; it runs at 3, 4 or 5 CTAs per SM and can bulk-prefetch each warp's
 * contiguous blocks into L2 at its start).  swe_cuda_init times every kernel
 * and shape on the patch, keeps the fastest shape of each, and uses the fastest
 * kernel.  info[9] = {kernel in use (0/1/2), pipelined tile in nodes (0 if
 * unavailable), ns per stage launch of kernel 0 (its fastest tile; stages 0-2
 * chained as in a step), of kernel 1, lanes per node of kernel 2, ns per stage
 * launch of kernel 2 (its fastest
 * shape), kernel 2's L2 prefetch (0/1), kernel 2's CTAs per SM (3/4/5),
 * kernel 2 reads its gather rows as 16-bit offsets from each node's own row
 * (1: every stencil row lies within 32767 rows of its node, as in any
 * RCM-ordered grid; 0: 32-bit indices)}.
 * swe_cuda_select_kernel takes which = 0 / 1 (kernels 0 / 1), 2 / 3 / 4 (the
 * pipelined kernel with 64- / 32- / 16-node tiles), 5 (kernel 2, its current
 * shape) and 6 + s for kernel 2's shape s in 0..17: 1 / 2 / 4 lanes per node
 * for s % 3 = 0 / 1 / 2; for s < 12, 5 CTAs per SM when (s / 3) is odd (else
 * 4) and the L2 prefetch when s >= 6; for s >= 12, 3 CTAs per SM and the L2
 * prefetch when s >= 15. */
int swe_cuda_select_kernel(int which);
int swe_cuda_kernel_info(int* info);
/* Index width of kernel 2's gather rows: 16 (the default whenever every stencil
 * row lies within 32767 rows of its node; SWE_ERR_ARG otherwise) or 32.  The
 * results are the same bits either way; 16 halves the index bytes. */
int swe_cuda_set_index_width(int bits);

/* Timing of the fused stage kernels, measured with CUDA events on the
 * library's stream while enabled.  out[0] = seconds of stage kernels since
 * the last reset, out[1] = stage launches, out[2] = seconds of the last
 * swe_cuda_step call.  Reading synchronises. */
int swe_cuda_set_timing(int enabled);
int swe_cuda_last_timings(double* out);

/* The library's CUDA stream (a cudaStream_t) for callers that want to order
 * their own work or events against it. */
void* swe_cuda_stream(void);

/* FP64 (mass, energy) of the device state with equal node areas 4*pi/n:
 * mass = sum A (h + gh0 - ghm), energy = sum A (0.5 (h+gh0-ghm)|u|^2 + 0.5 (h+gh0)^2).
 * Also the NaN/Inf watchdog (the reference's only such check is the NaN test in
 * verify_output, main.c:451): the sums are written either way, and the call
 * returns SWE_ERR_NONFINITE when either is NaN or Inf, i.e. when any value of
 * the state is. */
int swe_cuda_invariants(double* mass_energy);

/* Frees all device memory and the stream. */
int swe_cuda_finalize(void);

/* ---------------------------------------------------------------------------
 * History output of the plain form
 * ------------------------------------------------------------------------- */

/* The writer the reference declares but never implements (USE_HIST:
 * runtime_params.c:24-27 reads SWE_OUTPUT_FILE and SWE_HIST_INT,
 * swe_config.h:112-115 holds them; nothing writes).  After swe_hist_open,
 * every `interval` completed RK4 steps (swe_cuda_step, or swe_cuda_rk_substep
 * with substep 3; counted from the last swe_cuda_set_state) the state is
 * appended to `path` -- the same values swe_cuda_get_state returns, in the
 * caller's layout -- without stopping the time loop: the copy runs on its own
 * stream and a writer thread does the file I/O (at most 4 snapshots in
 * flight).  Format: a 64-byte header {char "SWEHIST1"[8]; int32 value bytes;
 * int32 interval; int64 values per record; double dt; int32 layout flags;
 * int32 SIMD length; 24 zero bytes}, then per record {int64 step; double
 * step * dt; values}.  swe_hist_close writes what is queued and closes the
 * file (swe_cuda_init and swe_cuda_finalize also close it).  stats[4] =
 * {open (0/1), records written, bytes written, steps since set_state}. */
int swe_hist_open(const char* path, int interval);
int swe_hist_close(void);
int swe_hist_stats(long long* stats);

/* ---------------------------------------------------------------------------
 * Input generator on the GPU (grids beyond the shipped N=2562 file)
 * ------------------------------------------------------------------------- */

/* No reference counterpart: the reference reads its binary input
 * (io/input.c:189-414) and does not ship the tool that produced it.  All
 * pointers are device pointers.
 * swe_gen_stencils: X [n][3] FP64 unit vectors -> idx [n][k] int32, 0-based, the
 *   k nearest nodes by chordal distance, self first, then by distance, ties by
 *   node index (k <= 32).
 * swe_gen_weights: unit-sphere RBF-FD weights D [4][n][k] FP64 (Dx, Dy, Dz, L)
 *   for those stencils: PHS r^7 + degree-4 tangent-plane polynomials for the
 *   projected gradient, r^9 on tangent-plane distances for Delta^4; one local
 *   solve (partial pivoting) per node and operator set.  The reader's scaling
 *   (Dx/a, L*gamma; input.c:314-319) is applied later, as for a file. */
int swe_gen_stencils(int n, int k, const double* X, int* idx);
int swe_gen_weights(int n, int k, const double* X, const int* idx, double* D);

/* Self-test of the bounded waits (no reference counterpart).  Launches one block
 * that waits on an mbarrier nothing arrives on, with the time-bounded wait the
 * pipelined kernels use; returns SWE_ERR_TIMEOUT once it gave up after about
 * limit_s (0 < limit_s <= 2), with the context still usable.  waited_s (may
 * be NULL) receives the time the kernel waited. */
int swe_selftest_wait_timeout(double limit_s, double* waited_s);

/* ---------------------------------------------------------------------------
 * Batched-ensemble form (members share one grid; tcgen05 tensor cores)
 * ------------------------------------------------------------------------- */

/* No single reference counterpart: the reference steps one state at a time
 * (RK_substep, rk4_rbffd_swe.c:30-72); this form steps `members` (32 or 64)
 * states of the same grid together.  Static arrays are the canonical FP64
 * ones in natural node order -- idx [n][nnbr] 0-based, Dx, Dy, Dz, L [n][nnbr]
 * already scaled as input.c:314-319 scales them, x, y, z, f, ghm [n],
 * p_u, p_v, p_w, gradghm [n][3].  The library reorders nodes along a
 * space-filling curve internally; states are exchanged as [members][n][4]
 * FP64 in natural order.
 * Precision: stencil products in 3xTF32 (or split BF16, see
 * swe_ens_set_precision) on tcgen05 with FP32 accumulation;
 * u, v, w and the stage states K in FP32; the RK4 accumulation of h (base
 * state and D register) in FP64; invariants in FP64.
 * Device memory: besides the member states (about 40 B per node and member),
 * the static weights are kept split for the tensor cores, about 11.7 KB per
 * node for both tile shapes and all three precisions together (1.91 GB at
 * N=163842). */
int swe_ens_init(int members, int n, int nnbr, double gh0, double dt, const int* idx,
                 const double* Dx, const double* Dy, const double* Dz, const double* L,
                 const double* x, const double* y, const double* z, const double* f,
                 const double* ghm, const double* p_u, const double* p_v, const double* p_w,
                 const double* gradghm);
int swe_ens_set_state(const double* H);
int swe_ens_get_state(double* H);
/* F = RHS(K) for all members (the same stencil math in the same precision);
 * K and F are [members][n][4] FP64 host arrays in natural order. */
int swe_ens_eval_rhs(const double* K, double* F);
/* nsteps RK4 steps of every member (captured CUDA graph of the four stage
 * kernels); swe_ens_stage runs one stage, same semantics as RK_substep. */
int swe_ens_step(int nsteps);
int swe_ens_stage(int substep_id);
/* Autotuner: times one RK4 step of every kernel variant -- tile shape (32-node
 * tiles, M = 128, or 16-node tiles, M = 64; 3xTF32 only) x members per CTA (64
 * or 32) -- in the current precision on the live state, restores the state and
 * keeps the fastest.  ms_per_step[4] (may be NULL) receives the timings in the
 * order (tile, members per CTA) = (32, 64), (32, 32), (16, 64), (16, 32), -1
 * where a variant does not apply.  config[6] = {tile nodes, members per CTA,
 * largest neighbour set of a tile, tiles, precision, 16-row chunks of
 * neighbour rows over all tiles}. */
int swe_ens_tune(double* ms_per_step);
int swe_ens_config(int* config);
/* Forces one variant (tile_nodes 32 or 16, members_per_cta 64 or 32). */
int swe_ens_use_variant(int tile_nodes, int members_per_cta);
/* Precision of the stencil products: 0 = 3xTF32 (default; hi = x rounded to
 * TF32, lo = x - hi kept in FP32 and read by the tensor core at TF32
 * precision, |x - hi - lo| <= 2^-21 |x|), 1 = split BF16 (2^-17), 2 = split
 * FP16 (2^-22 within FP16's range), all with FP32 accumulation and the same
 * FP64 h accumulation.  Split FP16 scales each weight row by a power of two and
 * each state field by one taken from the largest |value| of that field (the
 * velocities share one), again after every step: a field may grow 8-fold
 * within one step before FP16 overflows, which swe_ens_invariants then reports
 * as SWE_ERR_NONFINITE.  Splits 1 and 2 use 32-node tiles. */
int swe_ens_set_precision(int precision);
/* FP64 (mass, energy) per member, [members][2], definitions as swe_cuda_invariants;
 * SWE_ERR_NONFINITE (message naming the first such member) when a member's sums
 * are NaN or Inf. */
int swe_ens_invariants(double* mass_energy);
int swe_ens_sync(void);
int swe_ens_set_timing(int enabled);
int swe_ens_last_timings(double* out);
void* swe_ens_stream(void);
int swe_ens_finalize(void);

/* ---------------------------------------------------------------------------
 * Serving form (continuous batching of forecast requests)
 * ------------------------------------------------------------------------- */

/* No reference counterpart (the reference runs one solve per process).
 * swe_srv_start reserves `budget_bytes` of device memory as the arena that
 * requests are admitted into, and starts the scheduler thread and the
 * persistent kernel.  Grids are registered once (canonical FP64 arrays as for
 * swe_ens_init, in the node order the caller wants them stepped) and stay
 * resident; swe_srv_add_grid returns a grid id >= 0 or -status.
 * swe_srv_submit queues a request (1..32 members, nsteps RK4 steps, initial
 * states [members][n][4] FP64, copied at once) and returns its id >= 0 or
 * -status; requests run as soon as arena space frees up, stepped together in
 * the FP64 plain-form arithmetic.  swe_srv_poll returns 0 while queued or
 * running, 1 when done, 2 when cancelled (times[2] = seconds from submission
 * to admission and to completion, -1 until known); swe_srv_fetch copies the
 * final states and forgets the request.  swe_srv_stats fills out[10] =
 * {kernel launches, admitted, completed, arena bytes in use, peak bytes in
 * use, budget, work items done (an item is one stage of one node chunk for
 * up to two members of a request), queued requests, running requests,
 * dependency-wait failures}.
 *
 * Failure path.  Every wait of the persistent kernel is bounded.  A work item
 * waits for its request's previous stage at most the dependency limit (10 s,
 * swe_srv_set_dep_limit changes it; 1 ms .. 1 h).  When a wait runs out the
 * kernel stops claiming work and ends; every request whose work was queued
 * then fails (swe_srv_poll returns -SWE_ERR_TIMEOUT naming it), while queued
 * and later requests run normally on a relaunched kernel.
 * swe_srv_test_withhold(request, stage_index) is a test hook: the first work
 * item of that stage (step * 4 + stage; chunk 0, members 0-1) of that request
 * (of the next request submitted, when request < 0) is never queued, so the
 * next stage's wait runs out. */
int swe_srv_start(double budget_bytes, int max_requests);
int swe_srv_add_grid(int n, int nnbr, double gh0, double dt, const int* idx,
                     const double* Dx, const double* Dy, const double* Dz, const double* L,
                     const double* x, const double* y, const double* z, const double* f,
                     const double* ghm, const double* p_u, const double* p_v, const double* p_w,
                     const double* gradghm);
int swe_srv_submit(int grid, int members, int nsteps, const double* H0);
int swe_srv_poll(int request, double* times);
int swe_srv_fetch(int request, double* H);
int swe_srv_cancel(int request);
int swe_srv_stats(double* out);
int swe_srv_stop(void);
int swe_srv_set_dep_limit(double seconds);
int swe_srv_test_withhold(int request, int stage_index);

/* ---------------------------------------------------------------------------
 * Plain form without device allocation
 * ------------------------------------------------------------------------- */

/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (device memory owned by an outer framework's pool; loops where an
 * allocation's implicit device synchronisation is not allowed): nsteps RK4
 * steps of one state, like swe_cuda_step, with every array a device pointer
 * the caller owns -- idx [n][nnbr] (0-based), Dx, Dy, Dz, L [n][nnbr],
 * x, y, z, f, ghm [n], p_u, p_v, p_w, gradghm [n][3], and H [n][4]
 * (u, v, w, h per node; updated in place) -- in fType of fsize bytes, with
 * Dx, Dy, Dz already divided by a and L multiplied by gamma (the reader's
 * scaling).  The K and D registers live in a static device array of
 * SWE_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit, so n <= SWE_NOALLOC_SCRATCH_BYTES / (12 * fsize) nodes (43690 FP64,
 * 87381 FP32); larger n returns SWE_ERR_ARG.  Nothing here allocates.  The
 * first call on a device looks up the array's address, so make it before any
 * stream capture.  Calls share the array: calls that overlap on the GPU race
 * and must be serialised by the caller.  Kernels go to `stream` (a
 * cudaStream_t, NULL for the default stream); the call returns once they are
 * enqueued.  Every idx entry must lie in 0..n-1.  The kernels check each one
 * as they gather: an entry outside that range is never dereferenced (the node's
 * own row is read in its place, so that call's results are wrong) and the
 * first one is recorded.  A call with nsteps = 0 steps nothing: it waits for
 * `stream` and returns SWE_ERR_INDEX, naming the recorded (node, slot, value)
 * in swe_cuda_last_error(), if any earlier call met such an entry (clearing
 * the record), else SWE_OK. */
#define SWE_NOALLOC_SCRATCH_BYTES (4u << 20)
int swe_cuda_step_noalloc(int fsize, int n, int nnbr, double gh0, double dt, const int* idx,
                          const void* Dx, const void* Dy, const void* Dz, const void* L,
                          const void* x, const void* y, const void* z, const void* f, const void* ghm,
                          const void* p_u, const void* p_v, const void* p_w, const void* gradghm,
                          void* H, int nsteps, void* stream);

/* ---------------------------------------------------------------------------
 * Host utilities (no device work)
 * ------------------------------------------------------------------------- */

/* Reverse Cuthill-McKee node order of the stencil graph, the same permutation
 * as the reference's rcm_mapping (swe_code/rcm/rcm.c:9-62): mapping[new] = old.
 * idx is [n][nnbr], 0-based, self first. */
int swe_host_rcm_mapping(int n, int nnbr, const int* idx, int* mapping);

/* Reverse Cuthill-McKee-style order computed on the current device, for callers
 * that need a bandwidth-reducing order fast (serving admission of new grids, large
 * N): breadth-first from node 0 one level at a time, in parallel within a level;
 * each level sorted by (position of the node's first parent in the order, stencil
 * slot); reversed at the end.  It replaces the ordering step of rcm_mapping
 * (swe_code/rcm/rcm.c:9-62) but not its exact permutation: the reference sorts each
 * node's children by their count of still-unmapped neighbours, a sequential
 * dependency.  Its bandwidth, as print_max_bandwidth (rcm.c:68-96) measures it, is
 * of the same size.  mapping[new] = old; idx [n][nnbr] host array, 0-based, self
 * first; needs 0 < n < 2^24 and breadth-first levels of at most 16384 nodes
 * (SWE_ERR_ARG otherwise, or for a disconnected stencil graph). */
int swe_dev_rcm_mapping(int n, int nnbr, const int* idx, int* mapping);

/* Number of kernels this library has launched since load (all forms). */
long long swe_b200_kernel_launches(void);

#ifdef __cplusplus
}
#endif

/* Convenience for reference host code that already includes swe_config.h:
 * forwards one PSMD_struct with the build's own layout options. */
#if defined(SWE_CONFIG_H) && !defined(__cplusplus)
static inline int swe_cuda_init_psmd(const PSMD_struct* p) {
    int layout = 0;
#ifdef USE_CFDL
    layout |= SWE_LAYOUT_CFDL;
#endif
#ifdef USE_SFDL
    layout |= SWE_LAYOUT_SFDL;
#endif
    return swe_cuda_init((int)sizeof(fType), layout, SIMD_LENGTH, p->compute_size, p->patch_size,
                         p->compute_pid_s, p->Nnbr, p->padded_Nnbr, (double)p->gh0, (double)p->dt,
                         p->x, p->y, p->z, p->f, p->ghm, p->p_u, p->p_v, p->p_w, p->gradghm,
                         p->idx, p->Dx, p->Dy, p->Dz, p->L);
}
#endif

#endif /* SWE_B200_H */
