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
//   pair_kernel   step t complete (predictor, edges, integrate, r(t+1),
//                 controller) and step t+1 without its integrate: the
//                 row's edges are walked twice back to back, the second
//                 walk re-reading col/delay/weight from cache; S_i(t+1) and
//                 eps_i(t+1) are parked in `pend`.
//   finish_kernel the integrate of step t+1 with g(t+1), r(t+2), controller.
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

// Block partial of (sum cos, sum sin) in the reference's tree order
// (leviathan_kernel.cu:198-233), completion ticket and, in the last CTA of
// the network, r (:242-263), the gain controller (:431-435) and the ring /
// step-count advance.  The same sequence closes step_kernel.
__device__ __forceinline__ void close_step(const StepArgs &a, const NetDesc &nd,
                                           NetState *ns, int net, int row0,
                                           float my_cos, float my_sin, float g,
                                           int nxt, float *s_rc, float *s_rs,
                                           int *s_last) {
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
    if (lane == 0) {
      a.partials[nd.part_off + row0 / kTile] = make_float2(my_cos, my_sin);
      __threadfence();
      const unsigned prev = atomicAdd(&ns->ticket, 1u);
      *s_last = (prev == (unsigned)(nd.ntiles - 1));
    }
  }
  __syncthreads();
  if (!*s_last) return;

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
      float inv_N = 1.0f / (float)nd.N;
      float r = sqrtf(sum_cos * sum_cos + sum_sin * sum_sin) * inv_N;
      const float gn = nd.ctrl ? gain_controller(g, r, a.dt, nd) : g;
      ns->g = gn;
      ns->r = r;
      ns->cur = nxt;
      int rb = ns->rbuf + 1;
      if (rb == nd.max_delay + 1) rb = 0;
      ns->rbuf = rb;
      ns->t = ns->t + 1;
      ns->ticket = 0u;
      if (a.r_host) a.r_host[net] = r;
      if (a.r_hist) {
        const int k = ns->rpos;
        if (k < a.r_cap) a.r_hist[(long long)k * a.num_nets + net] = r;
        ns->rpos = k + 1;
      }
    }
  }
}

// One step's walk over a lane's SELL row (csr_physics_kernel,
// leviathan_kernel.cu:126-165): delayed phases from ring slot
// (base - d) mod bsi, coupling sum in CSR order, Hebbian update in place.
// Software-pipelined like step_kernel: the stream loads of group k0+U are in
// flight while group k0 gathers and computes.
//   SECOND = 0: first walk of the launch.  Stream loads stay cached (col /
//               delay in L1 and L2, weights in L2) and the new weights are
//               written to L2 for the second walk.
//   SECOND = 1: second walk (step t+1): last use of the streams; it reads
//               back the weights the first walk wrote (same thread, coherent
//               loads).  Entries past the row's degree gather nothing: a
//               padding entry (node 0, delay 0) would name the slot being
//               written in this launch.
template <int MATH, int U, int SECOND>
__device__ __forceinline__ float row_walk(const uint32_t *__restrict__ cdp,
                                          float *__restrict__ wp, int len,
                                          int deg, const float *__restrict__ ring,
                                          int base, int bsi, int Np, float th,
                                          float my_eps, float dt,
                                          const NetDesc &nd) {
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  float local_sum = 0.0f;
  uint32_t p[U];
  float wv[U], dj[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (SECOND) {
      p[u] = (u < len) ? __ldcs(cdp + 32 * u) : 0u;
      wv[u] = (u < len) ? __ldcs(wp + 32 * u) : 0.0f;
    } else {
      p[u] = (u < len) ? __ldg(cdp + 32 * u) : 0u;
      wv[u] = (u < len) ? __ldcg(wp + 32 * u) : 0.0f;
    }
  }
  for (int k0 = 0; k0 < len; k0 += U) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      int slot = base - (int)(p[u] & 255u);
      slot += (slot < 0) ? bsi : 0;
      const float *src = ring + ((unsigned)slot * (unsigned)Np + (p[u] >> 8));
      if (SECOND)
        dj[u] = (k0 + u < deg) ? ld_ring(src) : 0.0f;
      else
        dj[u] = ld_ring(src);
    }
    uint32_t pn[U];
    float wn[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0 + U + u;
      if (SECOND) {
        pn[u] = (k < len) ? __ldcs(cdp + 32 * k) : 0u;
        wn[u] = (k < len) ? __ldcs(wp + 32 * k) : 0.0f;
      } else {
        pn[u] = (k < len) ? __ldg(cdp + 32 * k) : 0u;
        wn[u] = (k < len) ? __ldcg(wp + 32 * k) : 0.0f;
      }
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
        if (SECOND)
          __stcs(wp + 32 * (k0 + u), w);
        else
          __stcg(wp + 32 * (k0 + u), w);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      p[u] = pn[u];
      wv[u] = wn[u];
    }
  }
  return local_sum;
}

// Step t in full and step t+1 up to its integrate (see the top of the file).
template <int MATH, int U, int MINB>
__global__ void __launch_bounds__(kTile, MINB) pair_kernel(const StepArgs a) {
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
  float *wp = nullptr;
  if (slice_live) {
    const long long s = nd.slice_base + (slice_row0 >> 5);
    len = a.sl_len[s];
    const long long base = a.sl_off[s] + lane;
    cdp = a.sl_cd + base;
    wp = a.sl_w + base;
  }

  // ---- step t: edges (csr_physics_kernel, :126-165) -------------------------
  float sum0 = 0.0f;
  if (slice_live)
    sum0 = row_walk<MATH, U, 0>(cdp, wp, len, deg, ring, cur, bsi, Np, th,
                                fabsf(eps), dt, nd);

  // ---- step t: integrate (integrate_and_reduce_kernel, :182-196) ------------
  int nxt = cur + 1;
  if (nxt == bsi) nxt = 0;
  float my_cos = 0.0f, my_sin = 0.0f;
  float th1 = 0.0f, eps1 = 0.0f;
  if (live) {
    float inc = dt * (a.omega[gi] + g * sum0 - nd.alpha * eps);
    float x = th + inc;
    x = wrap_0_2pi(x);
    if (!isfinite(x)) x = 0.0f;
    th1 = x;
    a.theta[gi] = x;
    a.ring[nd.ring_off + (long long)nxt * Np + row] = x;
    lev_sincos<MATH>(x, &my_sin, &my_cos);
    // ---- step t+1: predictor ------------------------------------------------
    float diff = th1 - thh;
    diff = wrap_pm_pi(diff);
    eps1 = sinf(diff);
    a.theta_hat[gi] = thh + dt * wh;
    a.omega_hat[gi] = wh + nd.kappa_w * dt * eps1;
  }

  // ---- step t+1: edges; the integrate waits for g(t+1) (finish_kernel) ------
  float sum1 = 0.0f;
  if (slice_live)
    sum1 = row_walk<MATH, U, 1>(cdp, wp, len, deg, ring, nxt, bsi, Np, th1,
                                fabsf(eps1), dt, nd);
  if (live) a.pend[gi] = make_float2(sum1, eps1);

  // ---- r(t+1), g(t+1) -------------------------------------------------------
  close_step(a, nd, ns, tile.x, row0, my_cos, my_sin, g, nxt, s_rc, s_rs, &s_last);
}

// The integrate of step t+1 (integrate_and_reduce_kernel, :182-196) with
// g(t+1), from the coupling sum and eps that pair_kernel parked; then
// r(t+2) and the controller.
template <int MATH>
__global__ void __launch_bounds__(kTile) finish_kernel(const StepArgs a) {
  __shared__ float s_rc[32];
  __shared__ float s_rs[32];
  __shared__ int s_last;

  const int tid = threadIdx.x;
  const int tix = a.reverse ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
  const int2 tile = a.tiles[tix];
  const NetDesc nd = a.nets[tile.x];
  NetState *ns = a.st + tile.x;

  const int N = nd.N;
  const int row0 = tile.y;
  const int row = row0 + tid;
  const long long gi = nd.node_off + row;
  const float dt = a.dt;
  const int cur = ns->cur;
  const float g = ns->g;
  int nxt = cur + 1;
  if (nxt == nd.bsi) nxt = 0;

  float my_cos = 0.0f, my_sin = 0.0f;
  if (row < N) {
    const float th = a.theta[gi];
    const float2 pe = a.pend[gi];
    const float local_sum = pe.x, eps = pe.y;
    float inc = dt * (a.omega[gi] + g * local_sum - nd.alpha * eps);
    float x = th + inc;
    x = wrap_0_2pi(x);
    if (!isfinite(x)) x = 0.0f;
    a.theta[gi] = x;
    a.ring[nd.ring_off + (long long)nxt * nd.Np + row] = x;
    lev_sincos<MATH>(x, &my_sin, &my_cos);
  }
  close_step(a, nd, ns, tile.x, row0, my_cos, my_sin, g, nxt, s_rc, s_rs, &s_last);
}

}  // namespace lev
