// lev_kernels.cuh -- sm_100a device code of the LEVIATHAN core engine step.
//
// One launch of step_kernel advances every network of an engine by one step.
// It fuses what the reference does in four launches plus a host round trip
// (leviathan_kernel.cu:391-438):
//   prep_kernel              :93-111   predictor, prediction error eps
//   csr_physics_kernel       :114-167  delayed gather, coupling sum, Hebbian
//   integrate_and_reduce     :170-234  phase integration, ring write, block r
//   final_reduce_r_kernel    :237-264  order parameter r
//   host gain controller     :431-435  g update (moved on device)
//
// Work unit: a tile of 256 consecutive rows (nodes) of one network, one CTA
// of 256 threads per tile, one thread per row -- the reference's mapping
// (leviathan_kernel.cu:124, 354).  The block partial sums of cos/sin, and so
// r, are formed over the same node groups in the same tree order.
//
// Layout in HBM (per network, packed over networks by offsets):
//   row_ptr  int32 [N+1]        local CSR offsets (as given by the caller)
//   sl_cd    uint32[...]        (col_idx << 8) | delay, SELL-32 layout
//   sl_w     f32   [...]        plastic weights, SELL-32 layout, in place
//   theta, theta_hat, omega, omega_hat  f32 [N]
//   ring     f32   [bsi/4][Np][4] delay ring, bsi = max_delay + 2 (rounded up
//                               to a multiple of 4 for the allocation), Np = N
//                               rounded up to 32: slots 4m .. 4m+3 of a node
//                               side by side (ring_pos), so the two walks of a
//                               pair launch find slots t-d and t+1-d in one
//                               16-byte group for three delays in four
//
// SELL-32 (sliced ELLPACK, slice height 32): rows are grouped in slices of
// 32 consecutive rows; a slice stores its rows' edges column-major, entry k
// of the slice's row l at sl_off[slice] + 32*k + l, for k below the slice's
// largest degree sl_len[slice] (shorter rows are padded with an inert entry).
// Each warp owns one slice and each lane one row, so every load of the edge
// streams is a coalesced 128-byte warp access, no lane ever searches for its
// row, and a lane walks its row's edges in CSR order -- the order and the
// fused multiply-add of the reference's per-row sum (:137-154), so the
// coupling sum is bitwise the reference's.
//
// The ring has one slot more than the reference's max_delay+1: step t reads
// slots (t-d) mod bsi for d in [0,max_delay] and writes theta(t+1) to slot
// (t+1) mod bsi, which no read of the same step touches.  The reference
// relies on separate launches for that ordering (:398 then :408); with the
// extra slot one launch per step is race-free for every delay in
// [0,max_delay] and the gathered values are identical.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

namespace lev {

constexpr int kTile = 256;    // rows per CTA == threads per CTA
constexpr int kChunk = 4096;  // edges staged in shared memory per pass (CSR kernels)

// step_kernel is instantiated for several (U, PIPE, MINB) variants, chosen per
// engine (and per degree class of a batch) by the autotuner in lev_engine.cu:
//   U     edges per lane whose loads are in flight together ("vector width")
//   PIPE  1: the next group's edge-stream loads overlap this group's gathers
//   MINB  resident CTAs per SM the register budget is sized for

struct NetDesc {
  long long node_off;  // first node in the packed node arrays
  long long edge_off;  // first edge in CSR order (packed over networks)
  long long ring_off;  // first float of the ring (multiple of 32)
  long long rp_off;    // first entry of the local row_ptr (N+1 entries)
  long long slice_base;  // first SELL slice of this network
  long long aux_off;     // first float of the network's adjoint ring (adjoint only)
  int N;
  int Np;         // ring row pitch
  int bsi;        // ring slots = max_delay + 2
  int max_delay;  // reference ring has max_delay + 1 slots
  int ntiles;     // 256-row tiles of this network
  int part_off;   // first partial-sum slot
  int tile_off;   // first tile (CTA) of this network in the grid
  int dist;       // 1: partition of a network split over GPUs (lev_part.cuh):
                  // step_kernel stops after the tile partials, which go to
                  // their global tile positions (part_off = first global tile)
  float eta, lam, gamma, alpha, kappa_w, w_min, w_max, r0;
  float beta, mu, g_rest, g_min, g_max;
  int ctrl;
  int pad1, pad2;
};

struct NetState {
  float g;          // gain used by the next step
  float r;          // order parameter after the last step
  int cur;          // ring slot holding theta(t)   = t mod bsi
  unsigned ticket;  // CTAs of the running step that have finished
  long long t;      // steps taken
  int rbuf;         // reference ring slot of theta(t) = t mod (max_delay+1)
  int rpos;         // next row of the r history
};

// Hub-phase transition counter: the front-end of the reference's integrated-
// information solver (binarize_and_accumulate_kernel,
// leviathan_phi_kernel.cu:60-92), fed by the engine after every step of one
// network instead of by a host snapshot of all phases.
constexpr int kMaxHubs = 10;  // the reference solver's limit (1024 states)
struct HubMonitor {
  int net;                     // watched network (-1: standalone)
  int num_hubs;                // 1 .. kMaxHubs
  int hub[kMaxHubs];           // hub node indices, local to the network
  int prev;                    // state after the previous observation, -1 before the first
  int pad;
  long long observed;          // observations (accumulate calls)
  unsigned long long *counts;  // [S][S] transitions prev -> state, S = 2^num_hubs
  unsigned long long *totals;  // [S] transitions out of each state
};

// One observation (binarize_and_accumulate_kernel, leviathan_phi_kernel.cu:
// 67-91): bit i of the state is set when hub i's phase, taken modulo
// 6.2831853f into [0, 2pi), exceeds 3.1415926f; the transition from the
// previous state is counted.  One thread; theta read through L2 because
// other CTAs of the same launch may have written it.
__device__ __forceinline__ void hub_observe(HubMonitor *hm, const float *theta) {
  int state = 0;
  for (int i = 0; i < hm->num_hubs; ++i) {
    float phase = __ldcg(theta + hm->hub[i]);
    phase = fmodf(phase, 6.2831853f);
    if (phase < 0) phase += 6.2831853f;
    if (phase > 3.1415926f) state |= (1 << i);
  }
  const int S = 1 << hm->num_hubs;
  const int prev = hm->prev;
  if (prev >= 0 && prev < S) {
    hm->counts[(long long)prev * S + state] += 1ull;
    hm->totals[prev] += 1ull;
  }
  hm->prev = state;
  hm->observed += 1;
}

struct StepArgs {
  const NetDesc *nets;
  NetState *st;
  const int2 *tiles;  // (network, first local row)
  const int *row_ptr;
  const long long *sl_off;  // per slice: first entry (multiple of 32)
  const int *sl_len;        // per slice: largest degree
  const uint32_t *sl_cd;
  float *sl_w;
  float *theta;
  float *theta_hat;
  const float *omega;
  float *omega_hat;
  float *ring;
  float2 *partials;
  float *r_hist;  // [r_cap][num_nets] on device, or null
  float *r_host;  // [num_nets] in mapped host memory, or null
  int r_cap;
  int num_nets;
  float dt;
  int reverse;  // 1: CTAs walk the tile list backwards (alternating sweeps)
  float2 *pend;  // [nodes] (coupling sum, eps) of a half-done step (lev_pair.cuh)
  HubMonitor *hubs;  // observes hub phases after every step of hubs->net, or null
  // speculative second step (lev_pair.cuh), or null: pair_kernel writes step
  // t+1's new weights to w2 (SELL) and its predictor (theta_hat, omega_hat
  // after step t+1) to thh2 / omh2, leaving the engine state exactly that
  // after step t; finish_kernel moves thh2 / omh2 in
  float *w2;
  float *thh2;
  float *omh2;
};

// ---------------------------------------------------------------------------
// Arithmetic shared with the reference.  The expressions are written in the
// same form as leviathan_kernel.cu so that nvcc forms the same fused
// multiply-adds; see the line cited at each use.
// ---------------------------------------------------------------------------
constexpr float kTwoPi = 2.0f * CUDART_PI_F;
constexpr float kInvTwoPi = 0x1.45f306p-3f;  // RN(1 / kTwoPi)

// x / kTwoPi, correctly rounded, without a division: q0 = RN(x * 1/c) is
// corrected once with the exact remainder x - q0*c (one fma) -- the
// division-by-a-known-divisor scheme of P. Markstein (IBM J. Res. Dev. 34,
// 1990) and N. Brisebarre, J.-M. Muller, S. K. Raina (IEEE Trans. Comput.
// 53(8), 2004).  For |x| >= 2^-100 the two phase wraps below computed with it
// are bitwise identical to the same wraps computed with IEEE division, for
// every float input; tiny |x| take the IEEE division.  lev_selftest_wraps()
// re-checks that over all 2^32 inputs on the device.
__device__ __forceinline__ float div_two_pi(float x) {
  if (fabsf(x) < 0x1p-100f) return x / kTwoPi;
  const float q0 = __fmul_rn(x, kInvTwoPi);
  const float rem = __fmaf_rn(-q0, kTwoPi, x);
  return __fmaf_rn(rem, kInvTwoPi, q0);
}

__device__ __forceinline__ float wrap_pm_pi(float diff) {
  // symmetric wrap to [-pi, pi): leviathan_kernel.cu:105 and :146
  return diff - floorf(div_two_pi(diff) + 0.5f) * kTwoPi;
}

__device__ __forceinline__ float wrap_0_2pi(float x) {
  // wrap to [0, 2pi): leviathan_kernel.cu:188
  return x - floorf(div_two_pi(x)) * kTwoPi;
}

template <int MATH>
__device__ __forceinline__ void lev_sincos(float x, float *s, float *c) {
  if (MATH == 0) {
    __sincosf(x, s, c);  // reference: leviathan_kernel.cu:152,195
  } else {
    sincosf(x, s, c);
  }
}

// Host gain controller of leviathan_step (leviathan_kernel.cu:431-435),
// evaluated with one rounding per operation like the x86 host code (no
// contraction), then clamped with fmax/fmin.
__device__ __forceinline__ float gain_controller(float g, float r, float dt,
                                                 const NetDesc &nd) {
  float t1 = __fsub_rn(nd.r0, r);
  float t2 = __fmul_rn(nd.beta, t1);
  float t3 = __fsub_rn(g, nd.g_rest);
  float t4 = __fmul_rn(nd.mu, t3);
  float t5 = __fsub_rn(t2, t4);
  float t6 = __fmul_rn(dt, t5);
  float gn = __fadd_rn(g, t6);
  return fmaxf(nd.g_min, fminf(nd.g_max, gn));
}

// Ring gather: read-only (non-coherent) path.  The slot written by the same
// launch is never read by it (see the ring note at the top).
__device__ __forceinline__ float ld_ring(const float *p) { return __ldg(p); }

// Float index of slot `slot` of node `col` in a network's ring: groups of
// four slots (4m .. 4m+3) of a node side by side (16 bytes).  The second
// walk of a pair launch reads slot t+1-d where the first read t-d; they
// share a group unless t-d = 3 mod 4, so three quarters of the second
// walk's gathers -- the rewired edges' DRAM misses included -- find the word
// the first walk fetched.  Measured per pair launch at N = 10^6, k = 32:
// slot-major rows 307 us, pairs of slots 284.7 us, groups of four 277 us,
// groups of eight 284 us (a warp's gather of 32 consecutive nodes in one
// slot then spans 32 sectors).  slots * Np < 2^32 is checked at creation.
__host__ __device__ __forceinline__ unsigned ring_pos(int slot, unsigned col, int Np) {
  return ((unsigned)(slot >> 2) * (unsigned)Np + col) * 4u + (unsigned)(slot & 3);
}

// Slots allocated per node: bsi rounded up to whole groups of four.
__host__ __device__ __forceinline__ int ring_slots(int bsi) { return (bsi + 3) & ~3; }

// ---------------------------------------------------------------------------
// The fused step.
// ---------------------------------------------------------------------------
template <int MATH, int U, int PIPE, int MINB>
__global__ void __launch_bounds__(kTile, MINB) step_kernel(const StepArgs a) {
  __shared__ float s_rc[32];
  __shared__ float s_rs[32];
  __shared__ int s_last;

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int tix = a.reverse ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
  const int2 tile = a.tiles[tix];
  const NetDesc nd = a.nets[tile.x];
  NetState *ns = a.st + tile.x;

  const int N = nd.N;
  const int row0 = tile.y;
  const int row = row0 + tid;
  const bool live = row < N;
  const long long gi = nd.node_off + row;
  const float dt = a.dt;
  const int bsi = nd.bsi;
  const int Np = nd.Np;
  const int cur = ns->cur;
  const float g = ns->g;
  const float *ring = a.ring + nd.ring_off;

  // ---- predictor (prep_kernel, leviathan_kernel.cu:100-110) ----------------
  float th = 0.0f, eps = 0.0f;
  int deg = 0;
  if (live) {
    th = a.theta[gi];
    const float thh = a.theta_hat[gi];
    const float wh = a.omega_hat[gi];
    float diff = th - thh;
    diff = wrap_pm_pi(diff);
    eps = sinf(diff);
    a.theta_hat[gi] = thh + dt * wh;
    a.omega_hat[gi] = wh + nd.kappa_w * dt * eps;
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }
  const float my_eps = fabsf(eps);

  // ---- edges of this lane's row (csr_physics_kernel, :126-165) -------------
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  float local_sum = 0.0f;
  const int slice_row0 = row0 + 32 * warp;
  if (slice_row0 < N) {  // warp-uniform
    const long long s = nd.slice_base + (slice_row0 >> 5);
    const int len = a.sl_len[s];
    const long long base = a.sl_off[s] + lane;
    const uint32_t *cdp = a.sl_cd + base;
    float *wp = a.sl_w + base;
    if constexpr (PIPE) {
    // software-pipelined: the edge streams of group k0+U are in flight
    // while the ring gathers and math of group k0 run
    uint32_t p[U];
    float wv[U], dj[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      p[u] = (u < len) ? __ldcs(cdp + 32 * u) : 0u;
      wv[u] = (u < len) ? __ldcs(wp + 32 * u) : 0.0f;
    }
    for (int k0 = 0; k0 < len; k0 += U) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int slot = cur - (int)(p[u] & 255u);
        slot += (slot < 0) ? bsi : 0;
        dj[u] = ld_ring(ring + ring_pos(slot, p[u] >> 8, Np));
      }
      uint32_t pn[U];
      float wn[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + U + u;
        pn[u] = (k < len) ? __ldcs(cdp + 32 * k) : 0u;
        wn[u] = (k < len) ? __ldcs(wp + 32 * k) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (k0 + u < deg) {
          const float delayed_j = dj[u];
          float diff = delayed_j - th;
          diff = wrap_pm_pi(diff);
          float w = wv[u];
          float sin_diff, cos_diff;
          lev_sincos<MATH>(diff, &sin_diff, &cos_diff);
          local_sum += w * sin_diff;
          float dw = dt * (eta * cos_diff * (1.0f - gamma * my_eps) - lam * w);
          w += dw;
          if (!isfinite(w)) w = w_min;
          w = fmaxf(w_min, fminf(w_max, w));
          __stcs(wp + 32 * (k0 + u), w);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        p[u] = pn[u];
        wv[u] = wn[u];
      }
    }
    } else {
    for (int k0 = 0; k0 < len; k0 += U) {
      // all U entries' stream loads, then all U ring gathers, are issued
      // before the dependent math so their latencies overlap
      uint32_t p[U];
      float wv[U], dj[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (k0 + u < len) {  // warp-uniform
          p[u] = __ldcs(cdp + 32 * (k0 + u));
          wv[u] = __ldcs(wp + 32 * (k0 + u));
        } else {
          p[u] = 0u;
          wv[u] = 0.0f;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int slot = cur - (int)(p[u] & 255u);
        slot += (slot < 0) ? bsi : 0;
        // slot * Np + col < 2^32 is checked when the engine is created
        dj[u] = ld_ring(ring + ring_pos(slot, p[u] >> 8, Np));
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (k0 + u < deg) {
          const float delayed_j = dj[u];
          float diff = delayed_j - th;
          diff = wrap_pm_pi(diff);
          float w = wv[u];
          float sin_diff, cos_diff;
          lev_sincos<MATH>(diff, &sin_diff, &cos_diff);
          local_sum += w * sin_diff;
          float dw = dt * (eta * cos_diff * (1.0f - gamma * my_eps) - lam * w);
          w += dw;
          if (!isfinite(w)) w = w_min;
          w = fmaxf(w_min, fminf(w_max, w));
          __stcs(wp + 32 * (k0 + u), w);
        }
      }
    }
    }
  }

  // ---- integrate (integrate_and_reduce_kernel, leviathan_kernel.cu:182-196)
  int nxt = cur + 1;
  if (nxt == bsi) nxt = 0;
  float my_cos = 0.0f, my_sin = 0.0f;
  if (live) {
    float inc = dt * (a.omega[gi] + g * local_sum - nd.alpha * eps);
    float x = th + inc;
    x = wrap_0_2pi(x);
    if (!isfinite(x)) x = 0.0f;
    a.theta[gi] = x;
    a.ring[nd.ring_off + ring_pos(nxt, row, Np)] = x;
    lev_sincos<MATH>(x, &my_sin, &my_cos);
  }

  // ---- block partial of (sum cos, sum sin) (leviathan_kernel.cu:198-233) ---
  const unsigned mask = 0xffffffffu;
#pragma unroll
  for (int off = 16; off > 0; off /= 2) {
    my_cos += __shfl_down_sync(mask, my_cos, off);
    my_sin += __shfl_down_sync(mask, my_sin, off);
  }
  if (lane == 0) {
    s_rc[warp] = my_cos;
    s_rs[warp] = my_sin;
  }
  __syncthreads();
  if (warp == 0) {
    my_cos = (lane < (kTile / 32)) ? s_rc[lane] : 0.0f;
    my_sin = (lane < (kTile / 32)) ? s_rs[lane] : 0.0f;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      my_cos += __shfl_down_sync(mask, my_cos, off);
      my_sin += __shfl_down_sync(mask, my_sin, off);
    }
    if (lane == 0) {
      a.partials[nd.part_off + row0 / kTile] = make_float2(my_cos, my_sin);
      if (nd.dist) {
        s_last = 0;  // r of the whole network: part_finish_kernel
      } else {
        __threadfence();
        const unsigned prev = atomicAdd(&ns->ticket, 1u);
        s_last = (prev == (unsigned)(nd.ntiles - 1));
      }
    }
  }
  __syncthreads();
  if (!s_last) return;

  // ---- last CTA of this network: r and the gain controller ----------------
  // (final_reduce_r_kernel, leviathan_kernel.cu:242-263; controller :431-435)
  __threadfence();
  if (warp == 0) {
    float sum_cos = 0.0f, sum_sin = 0.0f;
    const float2 *part = a.partials + nd.part_off;
    for (int k = lane; k < nd.ntiles; k += 32) {
      const float2 v = __ldcg(part + k);
      sum_cos += v.x;
      sum_sin += v.y;
    }
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      sum_cos += __shfl_down_sync(mask, sum_cos, off);
      sum_sin += __shfl_down_sync(mask, sum_sin, off);
    }
    if (lane == 0) {
      float inv_N = 1.0f / (float)N;
      float r = sqrtf(sum_cos * sum_cos + sum_sin * sum_sin) * inv_N;
      const float gn = nd.ctrl ? gain_controller(g, r, dt, nd) : g;
      ns->g = gn;
      ns->r = r;
      ns->cur = nxt;
      int rb = ns->rbuf + 1;
      if (rb == nd.max_delay + 1) rb = 0;
      ns->rbuf = rb;
      ns->t = ns->t + 1;
      ns->ticket = 0u;
      if (a.r_host) a.r_host[tile.x] = r;
      if (a.r_hist) {
        const int k = ns->rpos;
        if (k < a.r_cap) a.r_hist[(long long)k * a.num_nets + tile.x] = r;
        ns->rpos = k + 1;
      }
      if (a.hubs && a.hubs->net == tile.x) hub_observe(a.hubs, a.theta + nd.node_off);
    }
  }
}

// ---------------------------------------------------------------------------
// Layout conversion and helpers
// ---------------------------------------------------------------------------

// Every ring slot of nodes col0 .. col0+N-1 := theta (init_buffer_kernel,
// leviathan_kernel.cu:79-90).  pairs 1: the engine's ring (ring_pos);
// pairs 0: a slot-major ring [bsi][Np] (the adjoint's own rings).
__global__ void ring_fill_kernel(const float *__restrict__ theta,
                                 float *__restrict__ ring, int N, int Np,
                                 int bsi, int col0, int pairs) {
  const long long total = (long long)bsi * N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
       k < total; k += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(k / N);
    const int i = (int)(k - (long long)s * N);
    if (pairs)
      ring[ring_pos(s, (unsigned)(col0 + i), Np)] = theta[i];
    else
      ring[(long long)s * Np + col0 + i] = theta[i];
  }
}

// CSR -> SELL-32 for one network: entry k of row i goes to
// sl_off[slice_base + i/32] + 32k + i%32.  One thread per row.
// mode 0: pack (col, delay) into sl_cd and copy weights, validating
//         col in [0,ncols) and delay <= max_delay (bits 1, 2 of *err); bit 4
//         reports a zero delay (ncols = N, or N plus the halo columns of a
//         partition, lev_part.cuh);
// mode 1: weights only, CSR -> SELL;   mode 2: weights only, SELL -> CSR.
__global__ void sell_convert_kernel(int mode, const int *__restrict__ row_ptr,
                                    int N, int ncols, long long slice_base,
                                    const long long *__restrict__ sl_off,
                                    const int *__restrict__ col,
                                    const uint8_t *__restrict__ delays,
                                    float *__restrict__ w_csr,
                                    uint32_t *__restrict__ sl_cd,
                                    float *__restrict__ sl_w, int max_delay,
                                    unsigned *__restrict__ err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    const int e0 = row_ptr[i], e1 = row_ptr[i + 1];
    const long long base = sl_off[slice_base + (i >> 5)] + (i & 31);
    unsigned bad = 0u;
    for (int e = e0; e < e1; ++e) {
      const long long idx = base + 32LL * (e - e0);
      if (mode == 0) {
        const int c = col[e];
        const int d = delays[e];
        if (c < 0 || c >= ncols) bad |= 1u;
        if (d > max_delay) bad |= 2u;
        if (d == 0) bad |= 4u;  // not an error: rules out two steps per launch
        sl_cd[idx] = ((uint32_t)c << 8) | (uint32_t)d;
        sl_w[idx] = w_csr[e];
      } else if (mode == 1) {
        sl_w[idx] = w_csr[e];
      } else {
        w_csr[e] = sl_w[idx];
      }
    }
    if (bad) atomicOr(err, bad);
  }
}

// CSR -> SELL-32 of every network of an engine at creation, one warp per
// slice: lane l takes row l of the slice and writes its entries k = 0 ..
// len-1 (len: the slice's longest row) at sl_off[s] + 32k + l, so each k is
// one contiguous 128-byte store per warp; entries past the row's degree are
// padding (node 0, delay 0, weight 0: read, never used).  The CSR arrays
// (concatenated over networks, as the caller passed them) were copied to the
// device as they are.  Validation as sell_convert_kernel: bit 1 a column
// outside [0, ncols) (ncols = N, plus the halo columns of a partition for
// network 0), bit 2 a delay above max_delay, bit 4 a zero delay (not an
// error: it rules out two steps per launch).
__global__ void sell_pack_kernel(const NetDesc *__restrict__ nets,
                                 const int *__restrict__ slice_net, long long slices,
                                 const long long *__restrict__ sl_off,
                                 const int *__restrict__ sl_len,
                                 const int *__restrict__ row_ptr,
                                 const int *__restrict__ col,
                                 const uint8_t *__restrict__ delays,
                                 const float *__restrict__ w, int n_ext,
                                 uint32_t *__restrict__ sl_cd, float *__restrict__ sl_w,
                                 unsigned *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  unsigned bad = 0u;
  for (long long s = warp0; s < slices; s += nwarps) {  // warp-uniform
    const int n = slice_net[s];
    const NetDesc &nd = nets[n];
    const int N = nd.N;
    const int row = (int)(s - nd.slice_base) * 32 + lane;
    const unsigned ncols = (unsigned)(N + (n == 0 ? n_ext : 0));
    const unsigned md = (unsigned)nd.max_delay;
    int e0 = 0, deg = 0;
    if (row < N) {
      const int *rp = row_ptr + nd.rp_off + row;
      e0 = rp[0];
      deg = rp[1] - e0;
    }
    const long long eb = nd.edge_off + e0;
    const long long base = sl_off[s] + lane;
    const int len = sl_len[s];
    for (int k = 0; k < len; ++k) {
      uint32_t word = 0u;
      float wv = 0.0f;
      if (k < deg) {
        const int c = col[eb + k];
        const unsigned d = delays[eb + k];
        bad |= (unsigned)((unsigned)c >= ncols) | ((unsigned)(d > md) << 1) |
               ((unsigned)(d == 0u) << 2);
        word = ((uint32_t)c << 8) | d;
        wv = w[eb + k];
      }
      sl_cd[base + 32LL * k] = word;
      sl_w[base + 32LL * k] = wv;
    }
  }
  bad = __reduce_or_sync(0xffffffffu, bad);
  if (lane == 0 && bad) atomicOr(err, bad);
}

// r-history row counters := 0 (first node of every captured step block).
__global__ void reset_rpos_kernel(NetState *st, int num_nets) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < num_nets;
       n += gridDim.x * blockDim.x)
    st[n].rpos = 0;
}

// Exhaustive check of the division-free phase wraps: for every float bit
// pattern x, wrap_pm_pi(x) and wrap_0_2pi(x) against the same expressions
// with IEEE division (leviathan_kernel.cu:105,146,188).  counts[0], counts[1]
// receive the numbers of inputs whose results differ in any bit (NaN equal
// to NaN).
__global__ void selftest_wraps_kernel(unsigned long long *counts) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long bad_pm = 0, bad_02 = 0;
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
       k < (1ull << 32); k += stride) {
    const float x = __uint_as_float((unsigned int)k);
    const float ref_pm = x - floorf(x / kTwoPi + 0.5f) * kTwoPi;
    const float ref_02 = x - floorf(x / kTwoPi) * kTwoPi;
    const float got_pm = wrap_pm_pi(x);
    const float got_02 = wrap_0_2pi(x);
    const bool nan_pm = isnan(ref_pm) && isnan(got_pm);
    const bool nan_02 = isnan(ref_02) && isnan(got_02);
    bad_pm += (!nan_pm && __float_as_uint(ref_pm) != __float_as_uint(got_pm));
    bad_02 += (!nan_02 && __float_as_uint(ref_02) != __float_as_uint(got_02));
  }
  if (bad_pm) atomicAdd(counts + 0, bad_pm);
  if (bad_02) atomicAdd(counts + 1, bad_02);
}

}  // namespace lev
