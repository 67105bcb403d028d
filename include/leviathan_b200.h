/*
 * leviathan_b200.h -- C ABI of the B200 engine for the delayed Kuramoto
 * network with prediction-gated Hebbian plasticity and a homeostatic gain
 * controller (LEVIATHAN core engine step).
 *
 * Two layers are exported by libleviathan_b200.so:
 *
 *  1. The reference's own C ABI, symbol for symbol (leviathan_init ...
 *     leviathan_free).  A binding written against the reference
 *     (src/bindings/leviathan_pybind11.cpp:10-25) links against this library
 *     unchanged.  Unlike the reference, no call ever terminates the process:
 *     failures are recorded and readable through lev_last_error().
 *
 *  2. The lev_* status-code ABI.  Every function returns LEV_OK (0) or a
 *     negative LEV_ERR_* code; lev_last_error() returns a message for the
 *     calling thread.  It adds batched networks (many independent networks in
 *     one launch), step blocks (n steps per call, CUDA-graph replayed), full
 *     state checkpoint / restore and per-network parameters.
 *
 * Plain pointers and sizes only; all host pointers are borrowed for the
 * duration of the call.  Device pointers appear only in the *_dev functions.
 * A handle is not thread-safe: concurrent calls on one handle are not
 * supported (same as the reference).
 */
#ifndef LEVIATHAN_B200_H
#define LEVIATHAN_B200_H

#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
#define LEV_OK 0
#define LEV_ERR_ARG (-1)     /* invalid argument (size, range, null)        */
#define LEV_ERR_CUDA (-2)    /* CUDA runtime error                          */
#define LEV_ERR_STATE (-3)   /* call not valid in the current handle state  */
#define LEV_ERR_NOMEM (-4)   /* device or host allocation failed            */

/* Arithmetic of the transcendental calls inside the step.
 * LEV_MATH_REFERENCE uses the same fast sin/cos intrinsic as the reference
 * kernels (leviathan_kernel.cu:152,195) so results track the reference
 * engine; LEV_MATH_ACCURATE uses correctly-ranged sincosf for the edge and
 * order-parameter terms (lower error against an FP64 transcription). */
#define LEV_MATH_REFERENCE 0
#define LEV_MATH_ACCURATE 1

/* Physics parameters of one network.  Defaults (lev_default_params) are the
 * constants hard-coded in leviathan_init (leviathan_kernel.cu:282-296) and
 * the literal g_rest = 1.5 of leviathan_step (leviathan_kernel.cu:433). */
typedef struct LevParams {
  float eta;       /* Hebbian learning rate                 (0.01)  */
  float lam;       /* weight decay                          (0.001) */
  float gamma;     /* prediction-error gating               (0.05)  */
  float alpha_eps; /* prediction-error feedback on phase    (0.1)   */
  float kappa_w;   /* predictor frequency adaptation        (0.01)  */
  float w_min;     /* weight clamp                          (0.0)   */
  float w_max;     /*                                       (2.0)   */
  float g;         /* initial global coupling gain          (1.5)   */
  float r0;        /* controller target order parameter     (0.5)   */
  float beta;      /* controller gain rate                  (0.01)  */
  float mu;        /* controller relaxation rate            (0.01)  */
  float g_rest;    /* controller resting gain               (1.5)   */
  float g_min;     /* gain clamp                            (0.1)   */
  float g_max;     /*                                       (5.0)   */
  int32_t gain_controller; /* 1 = on (default), 0 = off             */
  int32_t reserved;
} LevParams;

typedef struct LevEngine LevEngine;

/* Message of the last failed lev_* / leviathan_* call on this thread. */
const char *lev_last_error(void);

/* Library version string. */
const char *lev_version(void);

/* Fill *p with the reference defaults. */
void lev_default_params(LevParams *p);

/* ------------------------------------------------------------------------ */
/* Construction                                                              */
/* ------------------------------------------------------------------------ */

/* One network.  Replaces leviathan_init (leviathan_kernel.cu:270-389).
 * E = row_ptr[N].  Arrays: row_ptr[N+1] (non-decreasing, row_ptr[0]=0),
 * col_idx[E] in [0,N), delays[E] in [0,max_delay], weights[E], theta[N],
 * theta_hat[N], omega[N].  omega_hat starts equal to omega
 * (leviathan_kernel.cu:350); every ring slot starts equal to theta
 * (init_buffer_kernel, leviathan_kernel.cu:79-90).  max_delay in [0,255]
 * (delays are uint8), N in [1, 2^24).  params may be NULL (defaults).
 * math_mode is LEV_MATH_REFERENCE or LEV_MATH_ACCURATE.  The engine runs on
 * the CUDA device that is current at the call.  The edge arrays are read for
 * row_ptr[N] entries while the rest of row_ptr is still being checked (as
 * the reference, which takes E from row_ptr[N], leviathan_kernel.cu:278):
 * they must hold that many. */
int lev_create(LevEngine **out, int32_t N, int32_t max_delay,
               const int32_t *row_ptr, const int32_t *col_idx,
               const uint8_t *delays, const float *weights,
               const float *theta, const float *theta_hat,
               const float *omega, const LevParams *params,
               int32_t math_mode);

/* Many independent networks in one engine (packed CSR with per-network
 * offsets).  No reference counterpart: the reference runs one engine per
 * network (experiments/phase_sweep.py:25-59 drives one network serially).
 * Arrays are the per-network arrays concatenated in network order:
 * row_ptr_cat holds num_nets local row_ptr arrays of N[n]+1 entries each
 * (values local to the network), the edge arrays hold sum(E[n]) entries,
 * the node arrays sum(N[n]).  params holds num_nets entries (NULL: all
 * defaults). */
int lev_batch_create(LevEngine **out, int32_t num_nets, const int32_t *N,
                     const int32_t *max_delay, const int32_t *row_ptr_cat,
                     const int32_t *col_idx_cat, const uint8_t *delays_cat,
                     const float *weights_cat, const float *theta_cat,
                     const float *theta_hat_cat, const float *omega_cat,
                     const LevParams *params, int32_t math_mode);

/* Replaces leviathan_free (leviathan_kernel.cu:455-478).  The engine's
 * device memory goes back to this library's per-device memory pool, which
 * keeps it for the next engine created in the process (no driver
 * allocation then); lev_trim_memory returns the pooled memory to the device. */
int lev_destroy(LevEngine *h);
int lev_trim_memory(void);

/* Wall-clock milliseconds of the phases of the engine's creation (no
 * reference counterpart; for tuning construction): ms_out[8] = host-side
 * validation and layout, and kernel set-up (both on a helper thread, while
 * the caller's CSR edge arrays are already being staged to a temporary
 * device buffer); the stream and the device allocations; the mapped host
 * buffer of r; small uploads (descriptors, tile lists); the staged pass (the
 * edge arrays, overlapping the first two phases, then the node arrays: host
 * threads copy them into pinned buffers and issue the DMAs); the launches
 * of the SELL-32 packing (which validates columns and delays) and of the
 * ring fill; the wait for every DMA, the packing and the fill. */
int lev_create_profile(const LevEngine *h, double *ms_out);

/* Shape queries. */
int lev_num_nets(const LevEngine *h, int32_t *out);
int lev_total_nodes(const LevEngine *h, int64_t *out);
int lev_total_edges(const LevEngine *h, int64_t *out);
int lev_net_shape(const LevEngine *h, int32_t net, int32_t *N, int64_t *E,
                  int32_t *max_delay);

/* ------------------------------------------------------------------------ */
/* Stepping                                                                  */
/* ------------------------------------------------------------------------ */

/* One step of every network.  Replaces leviathan_step
 * (leviathan_kernel.cu:391-438): predictor, delayed gather + coupling +
 * Hebbian update, integration + ring write, order parameter r, gain
 * controller.  r_out[num_nets] receives r of theta(t+1) per network
 * (may be NULL).  Synchronous, like the reference.  When every degree class
 * takes two steps per launch, a call that starts a pair also computes the
 * next step up to its integrate into shadow buffers (the engine state is
 * exactly that after this step); the next call, with the same dt and no
 * state-writing call in between, only finishes it.  Results are bitwise the
 * same either way; the first such call allocates one more SELL weight array
 * and two node arrays. */
int lev_step(LevEngine *h, float dt, float *r_out);

/* n steps of every network in one call; the step loop is replayed from a
 * CUDA graph.  r_out[n*num_nets] (step-major) receives r per step and
 * network (may be NULL).  Synchronous. */
int lev_step_n(LevEngine *h, float dt, int32_t n, float *r_out);

/* Asynchronous variant of lev_step_n for timing and device-side pipelines:
 * enqueues n steps on the engine stream and returns.  r values stay on the
 * device; lev_sync waits for completion. */
int lev_step_n_async(LevEngine *h, float dt, int32_t n);
int lev_sync(LevEngine *h);

/* Engine stream as a cudaStream_t cast to void*. */
int lev_get_stream(LevEngine *h, void **stream);

/* ------------------------------------------------------------------------ */
/* State access                                                              */
/* ------------------------------------------------------------------------ */

/* theta of all nodes (concatenated over networks).  Replaces
 * leviathan_get_theta (leviathan_kernel.cu:440-443). */
int lev_get_theta(LevEngine *h, float *theta_out);

/* Upload theta of all nodes and refill every ring slot with it (θ̂, ω̂, w
 * untouched).  Replaces leviathan_set_theta (leviathan_kernel.cu:445-453). */
int lev_set_theta(LevEngine *h, const float *theta_in);

/* Per-network variants (n in [0,num_nets)). */
int lev_get_theta_net(LevEngine *h, int32_t net, float *theta_out);
int lev_set_theta_net(LevEngine *h, int32_t net, const float *theta_in);

/* Edge weights (concatenated).  lev_reset_weights replaces
 * leviathan_reset_weights (leviathan_kernel.cu:492-497). */
int lev_get_weights(LevEngine *h, float *w_out);
int lev_reset_weights(LevEngine *h, const float *w_in);

/* Predictor state (concatenated): theta_hat, omega_hat; and omega. */
int lev_get_predictor(LevEngine *h, float *theta_hat_out,
                      float *omega_hat_out);
int lev_set_predictor(LevEngine *h, const float *theta_hat_in,
                      const float *omega_hat_in);
int lev_get_omega(LevEngine *h, float *omega_out);
int lev_set_omega(LevEngine *h, const float *omega_in);

/* Delay ring of one network exported in the reference layout:
 * ring_out[N*(max_delay+1)], node-major, slot s of node j at
 * ring_out[j*(max_delay+1)+s], slot of theta(t) = t mod (max_delay+1)
 * (leviathan_kernel.cu:142-143,192).  *buf_idx receives that slot index. */
int lev_get_ring(LevEngine *h, int32_t net, float *ring_out,
                 int32_t *buf_idx);
/* Inverse of lev_get_ring: restores the ring and the slot index. */
int lev_set_ring(LevEngine *h, int32_t net, const float *ring_in,
                 int32_t buf_idx);

/* Steps taken by a network since creation. */
int lev_get_step_count(LevEngine *h, int32_t net, int64_t *t);

/* Gain g and last order parameter r of a network.  Replace
 * leviathan_set_gain / leviathan_get_gain (leviathan_kernel.cu:480-482). */
int lev_set_gain(LevEngine *h, int32_t net, float g);
int lev_get_gain(LevEngine *h, int32_t net, float *g);
int lev_get_r(LevEngine *h, int32_t net, float *r);

/* Replaces leviathan_set_gain_controller (leviathan_kernel.cu:484-486). */
int lev_set_gain_controller(LevEngine *h, int32_t net, int32_t enabled);

/* Parameters of one network (net = -1: all networks). */
int lev_set_params(LevEngine *h, int32_t net, const LevParams *p);
int lev_get_params(LevEngine *h, int32_t net, LevParams *p);

/* Arithmetic mode (LEV_MATH_*), switchable between steps. */
int lev_set_math_mode(LevEngine *h, int32_t math_mode);

/* Device bytes held by the engine.  Replaces leviathan_get_vram_usage
 * (leviathan_kernel.cu:488-490), which returns a formula; this returns the
 * bytes actually allocated. */
int lev_get_vram_usage(const LevEngine *h, size_t *bytes);

/* ------------------------------------------------------------------------ */
/* Autotuner (no reference counterpart)                                      */
/* ------------------------------------------------------------------------ */

/* The step kernel is compiled in several variants (edges per lane in flight,
 * software pipelining, occupancy target).  An engine groups its networks in
 * three degree classes by mean SELL slice length (<= 14, <= 26, larger); each
 * class has its own tile list and variant.  Threads per row is fixed at one:
 * the reference's CSR-order row sum needs a single thread per row. */
int lev_num_variants(void);
int lev_variant_info(int32_t v, int32_t *unroll, int32_t *pipelined,
                     int32_t *min_blocks);
int lev_class_info(const LevEngine *h, int32_t c, int32_t *ntiles,
                   float *mean_slice_len, int64_t *edges, int32_t *variant);
int lev_set_variant(LevEngine *h, int32_t c, int32_t v);

/* Cluster-resident path (no reference counterpart): a single network whose
 * edges, node state and delay ring fit in the shared memory of one
 * thread-block cluster (<= 16 CTAs of <= 1024 rows) is stepped by
 * lev_step_n / lev_step_n_async with one launch per block of steps, delayed
 * phases of other CTAs' nodes read through distributed shared memory, one
 * cluster barrier per step.  Results are bitwise those of the per-step
 * kernel.  Eligibility is decided at creation; lev_set_cluster_mode(h, 0)
 * forces the per-step kernel. */
int lev_cluster_info(const LevEngine *h, int32_t *eligible, int32_t *enabled,
                     int32_t *ctas, int32_t *rows_per_cta, int64_t *smem_bytes);
int lev_set_cluster_mode(LevEngine *h, int32_t enabled);

/* Grid-resident path (no reference counterpart): a single network whose CTAs
 * (64, 128 or 256 rows each, four lanes per row, its edges and node state in
 * shared memory) can all be resident at once is stepped by lev_step_n /
 * lev_step_n_async with one cooperative launch per block of steps; the delay
 * ring stays in global memory (L2) and one grid barrier orders each step.
 * The barrier wait is bounded; a timeout makes lev_step_n / lev_sync return
 * LEV_ERR_CUDA and disables the path.  Results are bitwise those of the
 * per-step kernel.  The cluster path takes precedence when both are enabled.
 * lev_grid_info: enabled = eligible and allowed (the path step blocks use;
 * 0 after a timeout); rows_per_cta in use; eligible_rows_mask = OR of the
 * eligible rows-per-CTA values.  lev_set_grid_mode: enabled 0 forces the
 * per-step kernel; rows_per_cta 0 keeps the current choice. */
int lev_grid_info(const LevEngine *h, int32_t *eligible, int32_t *enabled, int32_t *ctas,
                  int32_t *rows_per_cta, int64_t *smem_bytes, int32_t *eligible_rows_mask);
int lev_set_grid_mode(LevEngine *h, int32_t enabled, int32_t rows_per_cta);

/* Bound of the grid-barrier waits of the grid-resident step blocks (no
 * reference counterpart).  limit_ns (1 us .. 60 s, default 2 s): longest
 * time one wait may take before the kernel gives up, sets the error flag and
 * returns.  extra_arrivals: 0 in normal use; a positive value makes every
 * wait expect that many more arrivals than the grid makes, so the block's
 * first wait runs out -- for tests of the timeout path, which then neither
 * faults nor hangs the GPU.  After a timeout at the first wait every CTA has
 * done the block's first step into its shared memory and one ring slot that
 * no step of the restored state reads, and has written nothing else back:
 * the engine keeps the state it had before the block. */
int lev_set_grid_wait(LevEngine *h, uint64_t limit_ns, uint32_t extra_arrivals);

/* Two steps per launch (no reference counterpart).  When no delay of the
 * engine is 0, step t+1's predictor and edge work need only the row's own
 * theta(t+1) and ring slots written before step t, so step blocks
 * (lev_step_n / lev_step_n_async) walk each row's edges for steps t and t+1
 * in one launch and finish step t+1's integrate, which needs the gain
 * g(t+1) and so the global r(t+1), in a short node-only launch.  The
 * edge streams then leave HBM once per two steps.  `deep` variants keep two
 * groups of edges in flight per lane.
 * Results are bitwise those of one step per launch.  lev_autotune times the pair variants of each
 * degree class against its best one-step variant and keeps pairs only where
 * they are faster; pair_variant -1 means one step per launch for that class.
 * lev_step (single steps, and the reference ABI) uses the same pair launches
 * as speculative single steps: the call that starts a pair leaves the state
 * of its own step and keeps the next step's work in shadow buffers for the
 * following call (see lev_step). */
int lev_num_pair_variants(void);
int lev_pair_variant_info(int32_t v, int32_t *unroll, int32_t *min_blocks,
                          int32_t *deep);
/* Threads per row of pair variant v (1, or 4: the row's SELL entries split
 * over four lanes, for low-degree networks; the coupling sum is formed in
 * CSR order from the four lanes' terms, bitwise as with one lane).  The
 * autotuner searches this dimension with the others, per degree class. */
int lev_pair_variant_lanes(int32_t v, int32_t *lanes);
int lev_pair_info(const LevEngine *h, int32_t c, int32_t *eligible, int32_t *enabled,
                  int32_t *pair_variant, float *pair_ms, float *step_ms);
int lev_set_pair_mode(LevEngine *h, int32_t enabled);
int lev_set_pair_variant(LevEngine *h, int32_t c, int32_t v);

/* Launch durations for profiling (no reference counterpart): runs n rounds
 * of two launch phases on the engine stream, each bracketed by CUDA events,
 * and advances the simulation by 2n steps.  With two steps per launch in use
 * ms_out[0] is the mean duration of the pair_kernel phase and ms_out[1] of
 * the finish_kernel phase; otherwise both are one-step launches.  (All
 * degree classes launch within a phase.) */
int lev_time_launches(LevEngine *h, float dt, int32_t n, float *ms_out);

/* Times every variant on every non-empty class of this engine
 * (trial_steps steps each, after two warm-up steps), keeps the fastest per
 * class, remembers it for later engines of the process with a similar class,
 * and restores the engine state afterwards (device-side snapshot, so the
 * simulation is unaffected).  variant_out[3] (may be NULL) receives the
 * choices, ms_out[3 * lev_num_variants()] (may be NULL) the ms per step of
 * every trial (0 for empty classes). */
int lev_autotune(LevEngine *h, float dt, int32_t trial_steps,
                 int32_t *variant_out, float *ms_out);

/* ------------------------------------------------------------------------ */
/* Adjoint: gradients through T steps (no reference counterpart)             */
/* ------------------------------------------------------------------------ */

/* Differentiable run of an engine's networks from the phases and predictor
 * phases the engine holds when the adjoint is created, with
 * omega_hat(0) = omega (leviathan_kernel.cu:350), every ring slot =
 * theta(0), and the inputs: omega[total nodes], w0[total edges] (CSR order of
 * the engine's inputs), K[num_nets] (the gain g(0)), and an optional drive
 * u[T][total nodes] added to d theta / dt.  The forward pass checkpoints the
 * state every `segment` steps; backward recomputes each segment and runs one
 * reverse kernel per step.  All array arguments of lev_adj_forward /
 * lev_adj_backward are DEVICE pointers (float32) on the engine's device.
 * The drive array passed to lev_adj_forward must stay valid until
 * lev_adj_backward returns. */
typedef struct LevAdjoint LevAdjoint;
int lev_adj_create(LevAdjoint **out, LevEngine *h, int32_t segment,
                   int32_t max_steps);
int lev_adj_destroy(LevAdjoint *a);
int lev_adj_bytes(const LevAdjoint *a, size_t *bytes);
/* r_out[T][num_nets]: r after each step; theta_out[T][total nodes] (may be
 * NULL): phases after each step. */
int lev_adj_forward(LevAdjoint *a, float dt, int32_t T, const float *omega,
                    const float *w0_csr, const float *K, const float *drive,
                    float *r_out, float *theta_out);
/* dLdr[T][num_nets] (may be NULL), dLdtheta[T][total nodes] (may be NULL);
 * outputs (each may be NULL): grad_omega[total nodes], grad_w0[total edges]
 * (CSR order), grad_K[num_nets], grad_drive[T][total nodes]. */
int lev_adj_backward(LevAdjoint *a, const float *dLdr, const float *dLdtheta,
                     float *grad_omega, float *grad_w0_csr, float *grad_K,
                     float *grad_drive);
/* dL/dtheta(0) of the last backward pass, [total nodes] (device). */
int lev_adj_grad_theta0(LevAdjoint *a, float *grad_theta0);

/* Reservoir terms fused into the adjoint's forward and reverse kernels
 * (device pointers, kept until replaced; NULL pairs disable a term):
 *   drive    u_i(t) = win[i] * x[t][network of i]      (win [total nodes],
 *            x [T][num_nets]) added to d theta_i / dt;
 *   readout  y[t][n] = sum_{i in n} ra[i] cos theta_i(t+1) + rb[i] sin theta_i(t+1)
 *            written to y_out[T][num_nets] by lev_adj_forward.
 * Set before lev_adj_forward.  For the backward pass set dL/dy [T][num_nets]
 * and the accumulators grad_win, grad_ra, grad_rb [total nodes] (zeroed by
 * lev_adj_backward, each may be NULL) with lev_adj_set_reservoir_grads. */
int lev_adj_set_reservoir(LevAdjoint *a, const float *win, const float *x,
                          const float *ra, const float *rb, float *y_out);
int lev_adj_set_reservoir_grads(LevAdjoint *a, const float *dLdy,
                                float *grad_win, float *grad_ra,
                                float *grad_rb);

/* Grid-resident segments (no reference counterpart): for a single network
 * whose CTAs (64, 128 or 256 rows, four lanes per row) can all be resident
 * at once, each checkpoint segment is one cooperative launch forward (with
 * the recording of the backward recompute) and one backward, with a bounded
 * grid barrier per step; a timeout makes lev_adj_forward / lev_adj_backward
 * return LEV_ERR_CUDA.  Not used with the reservoir readout (ra, rb).  The
 * forward trajectory is bitwise that of the per-step kernels; gradients
 * agree to rounding (sums over a row's edges and over CTAs in another
 * order).  lev_adj_set_grid_mode: enabled 0 forces per-step launches;
 * rows_per_cta 0 keeps the current choice.  When a second segment record set
 * fits and both CTA groups fit on the device at once, the backward pass
 * recomputes segment k-1 and reverses segment k in ONE paired launch (two
 * CTA groups, one barrier counter each); *paired tells whether it does;
 * lev_adj_set_grid_pairing(a, 0) makes the two separate launches again. */
int lev_adj_grid_info(const LevAdjoint *a, int32_t *eligible, int32_t *enabled,
                      int32_t *rows_per_cta, int32_t *eligible_rows_mask, int32_t *paired);
int lev_adj_set_grid_mode(LevAdjoint *a, int32_t enabled, int32_t rows_per_cta);
int lev_adj_set_grid_pairing(LevAdjoint *a, int32_t enabled);
/* Bound of the adjoint's grid-barrier waits, as lev_set_grid_wait. */
int lev_adj_set_grid_wait(LevAdjoint *a, uint64_t limit_ns, uint32_t extra_arrivals);

/* Self-test of the phase wraps (no reference counterpart; checks this
 * library's division-free evaluation of the wraps of
 * leviathan_kernel.cu:105,146,188).  Runs, on the current device, both
 * wraps for all 2^32 float inputs against the same expressions with IEEE
 * division; *mismatch_pm / *mismatch_02 receive the number of inputs whose
 * results differ in any bit (0 expected). */
int lev_selftest_wraps(uint64_t *mismatch_pm, uint64_t *mismatch_02);

/* ------------------------------------------------------------------------ */
/* One network split over several GPUs (halo engine)                         */
/* ------------------------------------------------------------------------ */

/* Replaces the reference's multi-GPU engine (multigpu_init / multigpu_step,
 * leviathan_multigpu.cu:123-238, whose halo kernels :97-115 are never
 * launched and whose step averages per-GPU |r| on the host) and the halo
 * lists of its partitioner (python/partition.py:45-170, which drops every
 * edge that crosses partitions, :121).
 *
 * The network's rows are cut into contiguous ranges of whole 256-row tiles;
 * a partition engine holds one range ("own" rows, N of them, starting at
 * global row 256 * tile_off_global) and ring columns for the n_halo other
 * nodes its rows read ("halo" nodes).  Its CSR is the own rows' part of the
 * network's CSR with columns renumbered: own node j -> j - 256 *
 * tile_off_global, halo node -> N + its position in the partition's halo
 * list; edge order within a row is kept, so every coupling sum is that of
 * the single-GPU engine.  theta_halo[n_halo] are the halo nodes' phases
 * (every ring slot of a halo column starts equal to them).  N_global and
 * ntiles_global = ceil(N_global / 256) describe the whole network.  Every
 * partition but the last owns a multiple of 256 rows.
 *
 * One step, all on the engine stream (lev_get_stream), device pointers:
 *   lev_part_step_begin  predictor, edges, integrate and own ring columns;
 *                        writes this partition's tile partials of
 *                        (sum cos, sum sin) to partials[tile_off_global ..
 *                        + own tiles) of a float2[ntiles_global] array;
 *   (caller)             all-gather the partials of every partition into
 *                        one float2[ntiles_global] array;
 *   lev_part_step_end    r of the whole network from that array in the
 *                        reference's order and the gain controller: every
 *                        partition gets the same r and g, bitwise those of
 *                        the single-GPU engine; r is also written to *r_dev
 *                        (device, may be NULL);
 *   lev_part_pack        out[k] = theta(t+1) of own node idx[k];
 *   (caller)             send / receive to the peers;
 *   lev_part_unpack      halo column idx[k] of the ring slot of theta(t+1)
 *                        := in[k], before the next step.
 * Indices out of range are skipped.  lev_set_theta / lev_get_theta work on
 * the own nodes; lev_part_fill_halo(theta_halo host) refills every ring slot
 * of the halo columns (the rest of set_theta).  lev_step, lev_step_n,
 * autotuning, hub monitors and the adjoint are refused (LEV_ERR_STATE). */
int lev_part_create(LevEngine **out, int32_t N, int32_t n_halo, int32_t max_delay,
                    const int32_t *row_ptr, const int32_t *col_idx,
                    const uint8_t *delays, const float *weights,
                    const float *theta, const float *theta_hat,
                    const float *omega, const float *theta_halo,
                    int32_t N_global, int32_t tile_off_global,
                    int32_t ntiles_global, const LevParams *params,
                    int32_t math_mode);
int lev_part_info(const LevEngine *h, int32_t *n_halo, int32_t *N_global,
                  int32_t *tile_off_global, int32_t *ntiles_global);
int lev_part_step_begin(LevEngine *h, float dt, void *partials_dev);
int lev_part_step_end(LevEngine *h, float dt, const void *partials_all_dev,
                      float *r_dev);
int lev_part_pack(LevEngine *h, const int32_t *idx_dev, int32_t n, float *out_dev);
int lev_part_unpack(LevEngine *h, const int32_t *idx_dev, int32_t n,
                    const float *in_dev);
int lev_part_fill_halo(LevEngine *h, const float *theta_halo);

/* Two steps per pair of launches for a partition (no zero delay, a one-lane
 * pair variant: lev_part_pairs tells), bitwise the one-step sequence:
 *   lev_part_pair_begin(partials)  step t in full and step t+1 up to its
 *                                  integrate; partials of r(t+1)
 *   all-gather, lev_part_step_end  r(t+1), g(t+1) on every rank
 *   lev_part_pack, send/recv, lev_part_unpack   theta(t+1) into the halo
 *                                  (before the finish overwrites theta)
 *   lev_part_pair_finish(partials) the integrate of step t+1; partials of
 *                                  r(t+2)
 *   all-gather, lev_part_step_end  r(t+2), g(t+2)
 *   lev_part_pack, send/recv, lev_part_unpack   theta(t+2) into the halo.
 * The next pair reads halo slots t+1 and t+2 only (no delay is 0). */
int lev_part_pairs(const LevEngine *h, int32_t *eligible);
int lev_part_pair_begin(LevEngine *h, float dt, void *partials_dev);
int lev_part_pair_finish(LevEngine *h, float dt, void *partials_dev);

/* ------------------------------------------------------------------------ */
/* Allocation-free step                                                      */
/* ------------------------------------------------------------------------ */

/* No counterpart in the reference (the reference engine always allocates its
 * own state, leviathan_kernel.cu:315-368).
 *
 * For callers that cannot call cudaMalloc -- code whose device memory is
 * owned by a memory planner or a framework allocator that must account for
 * every byte, or a fixed-budget / real-time loop where cudaMalloc (which can
 * synchronise the device and stall other streams) is not acceptable.  The
 * caller owns every buffer; this call allocates nothing and frees nothing.
 *
 * One step of one network, enqueued on `stream` (a cudaStream_t; NULL = the
 * legacy default stream); returns after the launch.  Same arithmetic and
 * results as lev_step.  All array arguments are DEVICE pointers on the
 * current device:
 *   row_ptr[N+1], col_idx[E], delays[E]   CSR topology: E = row_ptr[N],
 *                                         col < N, delay <= max_delay.  No
 *                                         error is raised for an edge whose
 *                                         col or delay is out of range: it is
 *                                         skipped (no ring read, nothing added
 *                                         to the coupling sum, its weight left
 *                                         unchanged).  Every pointer must be
 *                                         non-NULL, also when E = 0.
 *   weights[E], theta[N], theta_hat[N], omega_hat[N]   state, updated
 *   omega[N]                              natural frequencies
 *   ring[(max_delay+2)*N]                 delay ring, slot-major: slot s of
 *                                         node j at ring[s*N + j]; theta(t)
 *                                         is in slot t mod (max_delay+2);
 *                                         fill every slot with theta before
 *                                         the first step (t = 0)
 *   gain[1]   in: g for this step; out: g after the gain controller
 *   r_out[1]  out: order parameter of the new phases
 * t is the step index of the current phases (0 for the first call; the
 * caller adds 1 after each call).  params is a host pointer (NULL:
 * defaults).
 *
 * Scratch (one float2 per 256-node tile and a counter) lives in a fixed
 * device array built into the library: N is limited to 4,194,304 nodes
 * (LEV_ERR_ARG beyond), and every GPU that loads the library holds that
 * array (about 128 KiB) until the process exits.  All calls share it and it
 * keeps the last call's contents (the counter is cleared by each call), so
 * calls whose kernels overlap on the GPU -- on different streams, or from
 * different threads -- race and must not be issued.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture. */
int lev_step_noalloc(int32_t N, int32_t max_delay, int64_t t,
                     const int32_t *row_ptr, const int32_t *col_idx,
                     const uint8_t *delays, float *weights, float *theta,
                     float *theta_hat, const float *omega, float *omega_hat,
                     float *ring, float *gain, float *r_out,
                     const LevParams *params, float dt, int32_t math_mode,
                     void *stream);

/* ------------------------------------------------------------------------ */
/* Topology and initial state on the device                                  */
/* ------------------------------------------------------------------------ */

/* Seeded Watts-Strogatz graph built on the current device (replaces the
 * host networkx/scipy construction of python/leviathan_h100.py:34-55): ring
 * lattice of k/2 neighbours per side, every lattice edge rewired with
 * probability p to a uniform target avoiding self-loops and multi-edges;
 * canonical symmetric CSR (columns sorted), E = N*k.  Initial state drawn
 * per position: delays uniform in [delay_lo, delay_hi], weights uniform in
 * [w_lo, w_hi), theta uniform in [0, 2pi), omega ~ Normal(mean, std).
 * Deterministic for a seed.  Outputs are HOST arrays: row_ptr[N+1],
 * col_idx[E], delays[E], weights[E], theta[N], omega[N]. */
int lev_gen_ws(int32_t N, int32_t k, double p, uint64_t seed,
               int32_t delay_lo, int32_t delay_hi, float w_lo, float w_hi,
               float omega_mean, float omega_std, int32_t *row_ptr,
               int32_t *col_idx, uint8_t *delays, float *weights,
               float *theta, float *omega);

/* ------------------------------------------------------------------------ */
/* Hub-phase transition counts: the integrated-information front-end         */
/* ------------------------------------------------------------------------ */

/* The reference estimates a transition probability matrix of up to 10 "hub"
 * nodes for its integrated-information solver: after every step the hub
 * phases are binarised (bit i set when hub i's phase, taken modulo
 * 6.2831853f into [0, 2pi), exceeds 3.1415926f) and the transition from the
 * previous state is counted (binarize_and_accumulate_kernel,
 * leviathan_phi_kernel.cu:60-92; in python/leviathan_iit_integration.py:
 * 244-250 after a full host snapshot of all phases every step).  A LevHubs
 * monitor counts the same transitions.  Attached to an engine it observes
 * every step of one network inside the step's own reduction (no snapshot,
 * no extra launch); standalone it observes a phase array in device memory,
 * like phi_accumulate.  The integrated-information solver itself is not part
 * of this library.
 *
 * lev_hubs_create    replaces phi_init (:243-287): num_hubs in [1, 10],
 *                    hub_idx[num_hubs] node indices; S = 2^num_hubs states.
 * lev_attach_hubs    every later step of network `net` of h is observed
 *                    (m = NULL detaches).  While attached, the cluster-
 *                    resident path is not used and lev_hubs_accumulate is
 *                    refused.
 * lev_hubs_accumulate replaces phi_accumulate (:289-298): one observation
 *                    of theta_dev (device pointer; every hub index must be
 *                    inside it) on `stream` (NULL: the monitor's own stream).
 * lev_hubs_reset     replaces phi_reset (:337-345): counts 0, no previous
 *                    state, no observations.
 * lev_hubs_read      counts[S*S] (row = previous state), totals[S], the
 *                    last state (-1 before any observation) and the number
 *                    of observations (phi_get_transition_count, :347-349);
 *                    each output may be NULL.  Waits for the feeding engine.
 * lev_hubs_destroy   replaces phi_free (:351-367); detaches first. */
typedef struct LevHubs LevHubs;
int lev_hubs_create(LevHubs **out, int32_t num_hubs, const int32_t *hub_idx);
int lev_attach_hubs(LevEngine *h, int32_t net, LevHubs *m);
int lev_hubs_accumulate(LevHubs *m, const float *theta_dev, void *stream);
int lev_hubs_reset(LevHubs *m);
int lev_hubs_read(LevHubs *m, uint64_t *counts, uint64_t *totals, int32_t *prev_state,
                  int64_t *observed);
int lev_hubs_destroy(LevHubs *m);

/* ------------------------------------------------------------------------ */
/* Reference C ABI (leviathan_kernel.cu:21-499), same symbols and signatures */
/* ------------------------------------------------------------------------ */
typedef struct LeviathanHandle LeviathanHandle;

/* leviathan_kernel.cu:270.  Returns NULL on failure (reference: exit(1)). */
LeviathanHandle *leviathan_init(int N, int max_delay, int *h_row_ptr,
                                int *h_col_idx, uint8_t *h_delays,
                                float *h_weights, float *h_theta,
                                float *h_theta_hat, float *h_omega);
/* leviathan_kernel.cu:391.  Returns NaN on failure. */
float leviathan_step(LeviathanHandle *handle, float dt);
/* leviathan_kernel.cu:440 */
void leviathan_get_theta(LeviathanHandle *handle, float *h_theta);
/* leviathan_kernel.cu:445 */
void leviathan_set_theta(LeviathanHandle *handle, float *h_theta);
/* leviathan_kernel.cu:455 */
void leviathan_free(LeviathanHandle *handle);
/* leviathan_kernel.cu:480 */
void leviathan_set_gain(LeviathanHandle *handle, float g);
/* leviathan_kernel.cu:482 */
float leviathan_get_gain(LeviathanHandle *handle);
/* leviathan_kernel.cu:484 */
void leviathan_set_gain_controller(LeviathanHandle *handle, bool enabled);
/* leviathan_kernel.cu:488 */
size_t leviathan_get_vram_usage(LeviathanHandle *handle);
/* leviathan_kernel.cu:492 */
void leviathan_reset_weights(LeviathanHandle *handle, float *h_weights);

/* The engine behind a reference-ABI handle (for mixing both layers). */
LevEngine *leviathan_engine(LeviathanHandle *handle);

#ifdef __cplusplus
}
#endif

#endif /* LEVIATHAN_B200_H */
