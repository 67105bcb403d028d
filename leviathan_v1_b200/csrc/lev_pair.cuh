// lev_pair.cuh -- two engine steps per pass over the edge streams.
//
// Why two steps fit in one launch.  Step t of the reference
// (leviathan_kernel.cu:391-438) needs, for row i:
//   * theta_i(t), theta_hat_i(t), omega_hat_i(t)          (own row)
//   * theta_j(t - d) for every edge (i, j, d)             (ring, d >= 0)
//   * the gain g(t)                                       (global: r(t))
// and produces theta_i(t+1).  When every delay is at least 1, step t+1's
// predictor and edge work (coupling sum S_i(t+1), eps_i(t+1), weights
// w(t+2)) need only theta_i(t+1) -- computed by the same thread -- and
// theta_j(t+1-d) with t+1-d <= t, which the ring held before the launch.
// Only the integrate of step t+1 needs a global value, g(t+1), which depends
// on r(t+1) over all nodes.  So:
//
//   pair_kernel   step t complete (predictor, edges, integrate, tile
//                 partials of r(t+1)) and step t+1 without its integrate: the
//                 row's edges are walked twice back to back, the second
//                 walk re-reading col/delay/weight from cache; S_i(t+1) and
//                 eps_i(t+1) are parked in `pend`.
//   reduce_kernel r(t+1) from the partials, controller -> g(t+1).
//   finish_kernel the integrate of step t+1 with g(t+1), partials of r(t+2);
//                 then reduce_kernel again.
//
// Each SELL entry (col/delay word, weight read and write) then leaves HBM
// once per two steps, and the ring lines a tile gathers serve both steps
// while they are in L2.  Every value is computed by the same expression, in
// the same order, as step_kernel computes it, so the trajectory is bitwise
// the one-step-per-launch trajectory (and the reference's).
//
// Ring hazards: pair_kernel writes theta(t+1) to slot (t+1) mod bsi.  Step t
// reads slots t-d, d in [0, max_delay]; step t+1 reads slots t+1-d,
// d in [1, max_delay]; with bsi = max_delay + 2 neither touches slot t+1.
// finish_kernel writes slot (t+2) mod bsi = t - max_delay, read only by the
// previous launch.  Networks with a zero delay take one step per launch.
#pragma once

#include "lev_kernels.cuh"

namespace lev {

// Block partial of (sum cos, sum sin) of one 256-node tile in the
// reference's tree order (leviathan_kernel.cu:198-233): warp shuffle trees,
// then warp 0 over the eight warp sums.  All threads of the CTA call it.
__device__ __forceinline__ void tile_partial(const StepArgs &a, const NetDesc &nd, int row0,
                                             float my_cos, float my_sin, float *s_rc,
                                             float *s_rs) {
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
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
    if (lane == 0) a.partials[nd.part_off + row0 / kTile] = make_float2(my_cos, my_sin);
  }
}

constexpr int kReduceThreads = 1024;
constexpr int kPartChunk = 4096;  // partials staged in shared memory per round

// r and the gain controller of one network per CTA, after a pair_kernel or
// finish_kernel launch has written every tile partial: the one-warp
// lane-strided sums and shuffle tree of final_reduce_r_kernel
// (leviathan_kernel.cu:242-263) -- lane l adds partials l, l+32, ... in turn
// -- with the partials first staged in shared memory by the whole CTA, so
// the sequential adds do not wait on L2; then the controller (:431-435) and
// the ring / step-count advance.  nets: the networks of the launch's class.
__global__ void __launch_bounds__(kReduceThreads) reduce_kernel(const StepArgs a,
                                                                const int *nets) {
  __shared__ float2 s_part[kPartChunk];
  const int tid = threadIdx.x;
  const int net = nets[blockIdx.x];
  const NetDesc nd = a.nets[net];
  NetState *ns = a.st + net;
  // network state read up front, off the partial-sum critical path
  NetState st;
  if (tid == 0) st = *ns;
  const int ntiles = nd.ntiles;
  const float2 *part = a.partials + nd.part_off;
  float sum_cos = 0.0f, sum_sin = 0.0f;
  for (int c0 = 0; c0 < ntiles; c0 += kPartChunk) {
    const int n = min(kPartChunk, ntiles - c0);
    for (int k = tid; k < n; k += kReduceThreads) s_part[k] = part[c0 + k];
    __syncthreads();
    if (tid < 32) {
#pragma unroll 8
      for (int k = tid; k < n; k += 32) {
        const float2 v = s_part[k];
        sum_cos += v.x;
        sum_sin += v.y;
      }
    }
    __syncthreads();
  }
  if (tid < 32) {
    const unsigned mask = 0xffffffffu;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      sum_cos += __shfl_down_sync(mask, sum_cos, off);
      sum_sin += __shfl_down_sync(mask, sum_sin, off);
    }
    if (tid == 0) {
      float inv_N = 1.0f / (float)nd.N;
      float r = sqrtf(sum_cos * sum_cos + sum_sin * sum_sin) * inv_N;
      const float g = st.g;
      st.g = nd.ctrl ? gain_controller(g, r, a.dt, nd) : g;
      st.r = r;
      const int nxt = st.cur + 1;
      st.cur = (nxt == nd.bsi) ? 0 : nxt;
      const int rb = st.rbuf + 1;
      st.rbuf = (rb == nd.max_delay + 1) ? 0 : rb;
      st.t = st.t + 1;
      if (a.r_host) a.r_host[net] = r;
      if (a.r_hist) {
        if (st.rpos < a.r_cap) a.r_hist[(long long)st.rpos * a.num_nets + net] = r;
        st.rpos = st.rpos + 1;
      }
      *ns = st;
      if (a.hubs && a.hubs->net == net) hub_observe(a.hubs, a.theta + nd.node_off);
    }
  }
}

__device__ __forceinline__ int nxt_slot(int cur, int bsi) {
  int nxt = cur + 1;
  return nxt == bsi ? 0 : nxt;
}

// One step's walk over a lane's SELL row (csr_physics_kernel,
// leviathan_kernel.cu:126-165): delayed phases from ring slot
// (base - d) mod bsi, coupling sum in CSR order, Hebbian update in place.
//   SECOND = 0: first walk of the launch.  Stream loads stay cached (col /
//               delay in L1 and L2, weights in L2) and the new weights are
//               written to L2 for the second walk.
//   SECOND = 1: second walk (step t+1): last use of the streams; it reads
//               back the weights the first walk wrote (same thread, coherent
//               loads).  Entries past the row's degree gather nothing: a
//               padding entry (node 0, delay 0) would name the slot being
//               written in this launch.
//   DEEP = 0:   one-stage software pipeline (as step_kernel): the stream
//               loads of group k0+U are in flight while group k0 gathers and
//               computes.
//   DEEP = 1:   two stages: while group k0 computes, the gathers of group
//               k0+U (whose col/delay words arrived during the previous
//               group) and the stream loads of group k0+2U are in flight.
// wo: where the second walk writes the new weights (wp: in place).
template <int MATH, int U, int SECOND, int DEEP>
__device__ __forceinline__ float row_walk(const uint32_t *__restrict__ cdp,
                                          float *wp, float *wo, int len, int deg,
                                          const float *__restrict__ ring, int base,
                                          int bsi, int Np, float th, float my_eps,
                                          float dt, const NetDesc &nd) {
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  float local_sum = 0.0f;
  auto load_streams = [&](int k0, uint32_t *p, float *w) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0 + u;
      if (SECOND) {
        p[u] = (k < len) ? __ldcs(cdp + 32 * k) : 0u;
        w[u] = (k < len) ? __ldcs(wp + 32 * k) : 0.0f;
      } else {
        p[u] = (k < len) ? __ldg(cdp + 32 * k) : 0u;
        w[u] = (k < len) ? __ldcg(wp + 32 * k) : 0.0f;
      }
    }
  };
  auto gather = [&](int k0, const uint32_t *p, float *g) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      int slot = base - (int)(p[u] & 255u);
      slot += (slot < 0) ? bsi : 0;
      const float *src = ring + ring_pos(slot, p[u] >> 8, Np);
      if (SECOND)
        g[u] = (k0 + u < deg) ? ld_ring(src) : 0.0f;
      else
        g[u] = ld_ring(src);
    }
  };
  auto compute = [&](int k0, const float *g, const float *wv) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (k0 + u < deg) {
        const float delayed_j = g[u];
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
        if (SECOND)
          __stcs(wo + 32 * (k0 + u), w);
        else
          __stcg(wp + 32 * (k0 + u), w);
      }
    }
  };
  if constexpr (DEEP) {
    uint32_t pb[U];
    float wa[U], wb[U], ga[U], gb[U];
    {
      uint32_t pa[U];
      load_streams(0, pa, wa);
      load_streams(U, pb, wb);
      gather(0, pa, ga);
    }
    for (int k0 = 0; k0 < len; k0 += U) {
      gather(k0 + U, pb, gb);
      uint32_t pc[U];
      float wc[U];
      load_streams(k0 + 2 * U, pc, wc);
      compute(k0, ga, wa);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        ga[u] = gb[u];
        wa[u] = wb[u];
        pb[u] = pc[u];
        wb[u] = wc[u];
      }
    }
  } else {
    uint32_t p[U];
    float wv[U], dj[U];
    load_streams(0, p, wv);
    for (int k0 = 0; k0 < len; k0 += U) {
      gather(k0, p, dj);
      uint32_t pn[U];
      float wn[U];
      load_streams(k0 + U, pn, wn);
      compute(k0, dj, wv);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        p[u] = pn[u];
        wv[u] = wn[u];
      }
    }
  }
  return local_sum;
}

// Step t in full and step t+1 up to its integrate (see the top of the file).
template <int MATH, int U, int MINB, int DEEP>
__global__ void __launch_bounds__(kTile, MINB) pair_kernel(const StepArgs a) {
  __shared__ float s_rc[32];
  __shared__ float s_rs[32];

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
  const int nxt = nxt_slot(cur, bsi);
  const float g = ns->g;
  const float *ring = a.ring + nd.ring_off;

  // ---- step t: predictor (prep_kernel, leviathan_kernel.cu:100-110) --------
  float th = 0.0f, eps = 0.0f, thh = 0.0f, wh = 0.0f;
  int deg = 0;
  if (live) {
    th = a.theta[gi];
    const float thh0 = a.theta_hat[gi];
    const float wh0 = a.omega_hat[gi];
    float diff = th - thh0;
    diff = wrap_pm_pi(diff);
    eps = sinf(diff);
    thh = thh0 + dt * wh0;
    wh = wh0 + nd.kappa_w * dt * eps;
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }

  const int slice_row0 = row0 + 32 * warp;
  const bool slice_live = slice_row0 < N;  // warp-uniform
  int len = 0;
  const uint32_t *cdp = nullptr;
  float *wp = nullptr, *wo = nullptr;
  if (slice_live) {
    const long long s = nd.slice_base + (slice_row0 >> 5);
    len = a.sl_len[s];
    const long long base = a.sl_off[s] + lane;
    cdp = a.sl_cd + base;
    wp = a.sl_w + base;
    wo = (a.w2 ? a.w2 : a.sl_w) + base;
  }

  // ---- step t: edges (csr_physics_kernel, :126-165) -------------------------
  float sum0 = 0.0f;
  if (slice_live)
    sum0 = row_walk<MATH, U, 0, DEEP>(cdp, wp, wp, len, deg, ring, cur, bsi, Np, th, fabsf(eps),
                                      dt, nd);

  // ---- step t: integrate (integrate_and_reduce_kernel, :182-196) ------------
  float my_cos = 0.0f, my_sin = 0.0f;
  float th1 = 0.0f, eps1 = 0.0f;
  if (live) {
    float inc = dt * (a.omega[gi] + g * sum0 - nd.alpha * eps);
    float x = th + inc;
    x = wrap_0_2pi(x);
    if (!isfinite(x)) x = 0.0f;
    th1 = x;
    a.theta[gi] = x;
    a.ring[nd.ring_off + ring_pos(nxt, row, Np)] = x;
    lev_sincos<MATH>(x, &my_sin, &my_cos);
    // ---- step t+1: predictor ------------------------------------------------
    float diff = th1 - thh;
    diff = wrap_pm_pi(diff);
    eps1 = sinf(diff);
    if (a.thh2) {  // speculative: the state stays that after step t
      a.theta_hat[gi] = thh;
      a.omega_hat[gi] = wh;
      a.thh2[gi] = thh + dt * wh;
      a.omh2[gi] = wh + nd.kappa_w * dt * eps1;
    } else {
      a.theta_hat[gi] = thh + dt * wh;
      a.omega_hat[gi] = wh + nd.kappa_w * dt * eps1;
    }
  }

  // ---- step t+1: edges; the integrate waits for g(t+1) (finish_kernel) ------
  float sum1 = 0.0f;
  if (slice_live)
    sum1 = row_walk<MATH, U, 1, DEEP>(cdp, wp, wo, len, deg, ring, nxt, bsi, Np, th1,
                                      fabsf(eps1), dt, nd);
  if (live) a.pend[gi] = make_float2(sum1, eps1);

  // ---- partial of r(t+1); reduce_kernel forms r(t+1), g(t+1) ----------------
  tile_partial(a, nd, row0, my_cos, my_sin, s_rc, s_rs);
}

// ---------------------------------------------------------------------------
// Four lanes per row: the threads-per-row dimension of the autotuner.  A row
// of a low-degree network is only a few SELL entries long, so one lane per
// row leaves most of the gathers' latency exposed; four lanes per row keep
// four times as many rows' loads in flight per SM.  CTA = 1024 threads = one
// 256-row tile (the same tiles and tile partials as pair_kernel); warp w
// holds rows 8w .. 8w+7 of the tile, lane 4r + q of the warp is lane q of
// row r, and lane q takes the row's SELL entries q, q+4, q+8, ...  Eight
// rows' entries k are 32 contiguous bytes of the slice, so every stream load
// of a warp is four full 32-byte sectors.  Each entry's arithmetic is that of
// row_walk; the row's first lane forms the coupling sum in CSR order from the
// other lanes' terms (shuffled to it in entry order), with the same fused
// multiply-add, so the sum -- and the whole trajectory -- is bitwise that of
// one lane per row.
// ---------------------------------------------------------------------------
template <int MATH, int U, int SECOND>
__device__ __forceinline__ float row_walk4(const uint32_t *__restrict__ cdp,
                                           float *wp, float *wo, int len, int deg,
                                           const float *__restrict__ ring, int base,
                                           int bsi, int Np, float th, float my_eps,
                                           float dt, const NetDesc &nd, int q, int lead) {
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  const unsigned mask = 0xffffffffu;
  float local_sum = 0.0f;
  for (int kb = 0; kb < len; kb += 4 * U) {  // len: the slice's, warp-uniform
    uint32_t p[U];
    float wv[U], dj[U], sn[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb + 4 * u + q;
      if (SECOND) {
        p[u] = (k < deg) ? __ldcs(cdp + 32 * k) : 0u;
        wv[u] = (k < deg) ? __ldcs(wp + 32 * k) : 0.0f;
      } else {
        p[u] = (k < deg) ? __ldg(cdp + 32 * k) : 0u;
        wv[u] = (k < deg) ? __ldcg(wp + 32 * k) : 0.0f;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      int slot = base - (int)(p[u] & 255u);
      slot += (slot < 0) ? bsi : 0;
      const float *src = ring + ring_pos(slot, p[u] >> 8, Np);
      dj[u] = (kb + 4 * u + q < deg) ? ld_ring(src) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb + 4 * u + q;
      sn[u] = 0.0f;
      if (k < deg) {
        const float delayed_j = dj[u];
        float diff = delayed_j - th;
        diff = wrap_pm_pi(diff);
        float w = wv[u];
        float sin_diff, cos_diff;
        lev_sincos<MATH>(diff, &sin_diff, &cos_diff);
        sn[u] = sin_diff;
        float dw = dt * (eta * cos_diff * (1.0f - gamma * my_eps) - lam * w);
        w += dw;
        if (!isfinite(w)) w = w_min;
        w = fmaxf(w_min, fminf(w_max, w));
        if (SECOND)
          __stcs(wo + 32 * k, w);
        else
          __stcg(wp + 32 * k, w);
      }
    }
    // the row sum in CSR order on the row's first lane (entry kb + e is
    // lane e % 4's slot e / 4)
#pragma unroll
    for (int e = 0; e < 4 * U; ++e) {
      const int src = lead + (e & 3);
      const float w = __shfl_sync(mask, wv[e >> 2], src);
      const float sin_diff = __shfl_sync(mask, sn[e >> 2], src);
      if (kb + e < deg) local_sum += w * sin_diff;
    }
  }
  return local_sum;
}

template <int MATH, int U, int MINB>
__global__ void __launch_bounds__(4 * kTile, MINB) pair4_kernel(const StepArgs a) {
  __shared__ float s_rc[32];
  __shared__ float s_rs[32];
  __shared__ float s_oc[kTile];
  __shared__ float s_os[kTile];

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int q = lane & 3, lead = lane & ~3;
  const int rloc = 8 * warp + (lane >> 2);  // row within the tile
  const unsigned mask = 0xffffffffu;
  const int tix = a.reverse ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
  const int2 tile = a.tiles[tix];
  const NetDesc nd = a.nets[tile.x];
  NetState *ns = a.st + tile.x;

  const int N = nd.N;
  const int row0 = tile.y;
  const int row = row0 + rloc;
  const bool live = row < N;
  const long long gi = nd.node_off + row;
  const float dt = a.dt;
  const int bsi = nd.bsi;
  const int Np = nd.Np;
  const int cur = ns->cur;
  const int nxt = nxt_slot(cur, bsi);
  const float g = ns->g;
  const float *ring = a.ring + nd.ring_off;

  // ---- step t: predictor (every lane of the row; the first one writes) ----
  float th = 0.0f, eps = 0.0f, thh = 0.0f, wh = 0.0f;
  int deg = 0;
  if (live) {
    th = a.theta[gi];
    const float thh0 = a.theta_hat[gi];
    const float wh0 = a.omega_hat[gi];
    float diff = th - thh0;
    diff = wrap_pm_pi(diff);
    eps = sinf(diff);
    thh = thh0 + dt * wh0;
    wh = wh0 + nd.kappa_w * dt * eps;
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }

  const int slice_row0 = row0 + 32 * (warp >> 2);
  const bool slice_live = slice_row0 < N;  // warp-uniform
  int len = 0;
  const uint32_t *cdp = nullptr;
  float *wp = nullptr, *wo = nullptr;
  if (slice_live) {
    const long long s = nd.slice_base + (slice_row0 >> 5);
    len = a.sl_len[s];
    const long long base = a.sl_off[s] + (rloc & 31);
    cdp = a.sl_cd + base;
    wp = a.sl_w + base;
    wo = (a.w2 ? a.w2 : a.sl_w) + base;
  }

  // ---- step t: edges ------------------------------------------------------
  float sum0 = 0.0f;
  if (slice_live)
    sum0 = row_walk4<MATH, U, 0>(cdp, wp, wp, len, deg, ring, cur, bsi, Np, th, fabsf(eps),
                                 dt, nd, q, lead);
  sum0 = __shfl_sync(mask, sum0, lead);

  // ---- step t: integrate; step t+1: predictor ------------------------------
  float my_cos = 0.0f, my_sin = 0.0f;
  float th1 = 0.0f, eps1 = 0.0f;
  if (live) {
    float inc = dt * (a.omega[gi] + g * sum0 - nd.alpha * eps);
    float x = th + inc;
    x = wrap_0_2pi(x);
    if (!isfinite(x)) x = 0.0f;
    th1 = x;
    float diff = th1 - thh;
    diff = wrap_pm_pi(diff);
    eps1 = sinf(diff);
    if (q == 0) {
      a.theta[gi] = x;
      a.ring[nd.ring_off + ring_pos(nxt, row, Np)] = x;
      lev_sincos<MATH>(x, &my_sin, &my_cos);
      if (a.thh2) {  // speculative: the state stays that after step t
        a.theta_hat[gi] = thh;
        a.omega_hat[gi] = wh;
        a.thh2[gi] = thh + dt * wh;
        a.omh2[gi] = wh + nd.kappa_w * dt * eps1;
      } else {
        a.theta_hat[gi] = thh + dt * wh;
        a.omega_hat[gi] = wh + nd.kappa_w * dt * eps1;
      }
    }
  }

  // ---- step t+1: edges; the integrate waits for g(t+1) (finish_kernel) ------
  float sum1 = 0.0f;
  if (slice_live)
    sum1 = row_walk4<MATH, U, 1>(cdp, wp, wo, len, deg, ring, nxt, bsi, Np, th1, fabsf(eps1),
                                 dt, nd, q, lead);
  if (live && q == 0) a.pend[gi] = make_float2(sum1, eps1);

  // ---- partial of r(t+1): the rows' values in row order, then the tree ----
  if (q == 0) {
    s_oc[rloc] = my_cos;
    s_os[rloc] = my_sin;
  }
  __syncthreads();
  const float c = (tid < kTile) ? s_oc[tid] : 0.0f;
  const float sv = (tid < kTile) ? s_os[tid] : 0.0f;
  tile_partial(a, nd, row0, c, sv, s_rc, s_rs);
}

// The integrate of step t+1 (integrate_and_reduce_kernel, :182-196) with
// g(t+1), from the coupling sum and eps that pair_kernel parked, and the tile
// partials of r(t+2).  A CTA takes kFinishTiles consecutive tiles of the
// class's tile list (thread = one row of each), so the loads of all its rows
// are in flight together and the launch is less than one wave deep.
constexpr int kFinishTiles = 4;

template <int MATH>
__global__ void __launch_bounds__(kTile) finish_kernel(const StepArgs a, int ntiles) {
  __shared__ float s_rc[kFinishTiles][32];
  __shared__ float s_rs[kFinishTiles][32];

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  float my_cos[kFinishTiles], my_sin[kFinishTiles];
  float th[kFinishTiles], om[kFinishTiles];
  float2 pe[kFinishTiles];
  int2 tile[kFinishTiles];
#pragma unroll
  for (int q = 0; q < kFinishTiles; ++q) {
    const int t = blockIdx.x * kFinishTiles + q;
    tile[q] = make_int2(-1, 0);
    if (t < ntiles) tile[q] = a.tiles[a.reverse ? ntiles - 1 - t : t];
  }
#pragma unroll
  for (int q = 0; q < kFinishTiles; ++q) {
    my_cos[q] = my_sin[q] = 0.0f;
    th[q] = om[q] = 0.0f;
    pe[q] = make_float2(0.0f, 0.0f);
    if (tile[q].x >= 0) {
      const NetDesc &nd = a.nets[tile[q].x];
      const int row = tile[q].y + tid;
      if (row < nd.N) {
        const long long gi = nd.node_off + row;
        th[q] = a.theta[gi];
        pe[q] = a.pend[gi];
        om[q] = a.omega[gi];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kFinishTiles; ++q) {
    if (tile[q].x < 0) continue;
    const NetDesc &nd = a.nets[tile[q].x];
    const NetState *ns = a.st + tile[q].x;
    const int row = tile[q].y + tid;
    if (row < nd.N) {
      const long long gi = nd.node_off + row;
      const float g = ns->g;
      int nxt = ns->cur + 1;
      if (nxt == nd.bsi) nxt = 0;
      const float local_sum = pe[q].x, eps = pe[q].y;
      float inc = a.dt * (om[q] + g * local_sum - nd.alpha * eps);
      float x = th[q] + inc;
      x = wrap_0_2pi(x);
      if (!isfinite(x)) x = 0.0f;
      a.theta[gi] = x;
      a.ring[nd.ring_off + ring_pos(nxt, row, nd.Np)] = x;
      if (a.thh2) {  // the predictor of a speculative pair
        a.theta_hat[gi] = a.thh2[gi];
        a.omega_hat[gi] = a.omh2[gi];
      }
      lev_sincos<MATH>(x, &my_sin[q], &my_cos[q]);
    }
  }
  // block partials in the tree order of tile_partial, warp q closing tile q
  const unsigned mask = 0xffffffffu;
#pragma unroll
  for (int q = 0; q < kFinishTiles; ++q) {
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      my_cos[q] += __shfl_down_sync(mask, my_cos[q], off);
      my_sin[q] += __shfl_down_sync(mask, my_sin[q], off);
    }
    if (lane == 0) {
      s_rc[q][warp] = my_cos[q];
      s_rs[q][warp] = my_sin[q];
    }
  }
  __syncthreads();
  if (warp < kFinishTiles && tile[warp].x >= 0) {
    float c = (lane < (kTile / 32)) ? s_rc[warp][lane] : 0.0f;
    float sn = (lane < (kTile / 32)) ? s_rs[warp][lane] : 0.0f;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      c += __shfl_down_sync(mask, c, off);
      sn += __shfl_down_sync(mask, sn, off);
    }
    if (lane == 0) {
      const NetDesc &nd = a.nets[tile[warp].x];
      a.partials[nd.part_off + tile[warp].y / kTile] = make_float2(c, sn);
    }
  }
}

}  // namespace lev
