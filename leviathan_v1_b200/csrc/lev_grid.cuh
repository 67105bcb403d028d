// lev_grid.cuh -- grid-resident engine for mid-sized single networks.
// Included once, from lev_engine.cu.
//
// A single network whose CTAs all fit on the device at once (one cooperative
// launch, co-residency guaranteed by the launch) is stepped n times in ONE
// launch:
//   * CTA b owns rows [b*R, b*R + R), four lanes per row (4R threads); its
//     SELL-32 slices (col|delay, weights) and its rows' node state stay in
//     shared memory for the whole launch;
//   * the delay ring stays in global memory, which at these sizes is
//     L2-resident: each step writes theta(t+1) of the CTA's rows to ring slot
//     t+1 through L2, and every gather reads through L2 (ld.global.cg), so no
//     SM reads a stale L1 line of a slot another SM rewrote;
//   * one grid barrier per step (an arrival counter in global memory): a CTA
//     arrives after step t's ring write and warp sums and waits for barrier
//     t before step t+1's integrate, which needs g(t+1) and overwrites ring
//     slot t+2 = t-max_delay (mod max_delay+2), read by step t.  With zero
//     delays step t+1's gathers read slot t+1 and the wait comes before
//     them.  Without, they read slots <= t, ordered by barrier t-1, so the
//     wait for barrier t comes after the predictor and the edge work of step
//     t+1, which hide the barrier's latency;
//   * each warp's shuffle-tree (sum cos, sum sin) of its 32 rows goes to a
//     double-buffered array of warp sums; after the barrier every CTA stages
//     them in shared memory (cp.async, in flight during the next step's edge
//     work), forms the reference's 256-node block sums from eight warp sums
//     (block_tree8) and reduces the blocks in the order of
//     leviathan_kernel.cu:242-263.  All CTAs so compute the same r and gain,
//     which the next step needs only at its integrate.
// Arithmetic and summation order are those of step_kernel: results are
// bitwise the same as stepping with step_kernel.
//
// The barrier's wait is bounded (GridWait, 2 s by default): on a timeout
// the CTA writes 1 to the error flag (mapped host memory), leaves the step
// loop and writes nothing back; the host reports the error.

#pragma once

#include "lev_kernels.cuh"

namespace lev {

constexpr int kGridLPR = 4;                               // lanes per row
constexpr unsigned long long kGridWaitNs = 2000000000ull;  // default wait limit

// Bound of every grid-barrier wait of a launch.  `extra` is 0 in normal use;
// a positive value makes each wait expect that many arrivals more than the
// grid makes, so the first wait runs out after `ns` -- the timeout path can
// then be exercised by a test without faulting or hanging the GPU.
struct GridWait {
  unsigned long long ns;  // limit of one wait, globaltimer nanoseconds
  unsigned extra;
  unsigned pad;
};

struct GridArgs {
  const NetDesc *net;
  NetState *st;
  const int *row_ptr;
  const long long *sl_off;
  const int *sl_len;
  const uint32_t *sl_cd;
  float *sl_w;
  float *theta;
  float *theta_hat;
  const float *omega;
  float *omega_hat;
  float *ring;
  float2 *wsum;      // [2][nwarps]: warp sums of the network's 32-row groups
  unsigned *bar;     // arrival counter, zero at launch
  int early;         // no delay is 0: wait for barrier t after step t+1's edges
  int *err;          // error flag (mapped host memory)
  GridWait wait;     // bound of the barrier waits
  float *r_hist;     // [n] (row rpos + k), or null
  int r_cap;
  int n_steps;
  int nwarps;        // 8 * 256-node blocks, rounded up to even
  int edge_cap;      // SELL entries per CTA the shared memory was sized for
  float dt;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void cp_async_cg16(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Grid barrier, split in two.  Arrive: every thread of the CTA calls it
// after its writes; thread 0 adds one arrival with release semantics, which
// (after the CTA barrier) publishes the writes of the whole CTA.
__device__ __forceinline__ void grid_arrive(unsigned *bar) {
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
}

// Wait: every thread of the CTA calls it; thread 0 waits (acquire) until
// `target` arrivals (plus gw.extra), at most gw.ns.  Returns false after a
// timeout, in every thread.
__device__ __forceinline__ bool grid_wait(unsigned *bar, unsigned target, int *err, int *s_ok,
                                          const GridWait &gw) {
  if (threadIdx.x == 0) {
    const unsigned long long t0 = global_ns();
    while (ld_acquire_gpu(bar) < target + gw.extra) {
      if (global_ns() - t0 > gw.ns) {
        *reinterpret_cast<volatile int *>(err) = 1;
        *s_ok = 0;
        break;
      }
    }
  }
  __syncthreads();
  return *reinterpret_cast<volatile int *>(s_ok) != 0;
}

// shared memory layout (bytes, from the dynamic base):
//   s_ws   float2 [nwarps]    staged warp sums of the previous step
//   th, thh, om, omh  float [R]
//   ord    float  [2R]        the rows' (cos, sin) in row order
//   sloff, sllen  int [R/32]
//   cd     uint32 [edge_cap]
//   w      float  [edge_cap]
// R: rows per CTA (64, 128 or 256); U: edges per lane in flight together.
template <int MATH, int R, int U>
__global__ void __launch_bounds__(kGridLPR * R, 256 / R) grid_kernel(const GridArgs a) {
  constexpr int LPR = kGridLPR;
  constexpr int nslices = R / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ float s_g;
  __shared__ int s_ok;

  const NetDesc nd = *a.net;
  const int cta = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = tid & (LPR - 1);
  const int rloc = tid / LPR;
  const int lead = lane & ~(LPR - 1);
  const unsigned mask = 0xffffffffu;
  const int N = nd.N, bsi = nd.bsi, Np = nd.Np;
  const int row0 = cta * R;
  const int row = row0 + rloc;
  const bool live = row < N;
  const int nwarps = a.nwarps;

  float2 *s_ws = reinterpret_cast<float2 *>(smem);
  float *s_th = reinterpret_cast<float *>(s_ws + nwarps);
  float *s_thh = s_th + R;
  float *s_om = s_thh + R;
  float *s_omh = s_om + R;
  float *s_ord = s_omh + R;
  int *sloff = reinterpret_cast<int *>(s_ord + 2 * R);
  int *sllen = sloff + nslices;
  uint32_t *s_cd = reinterpret_cast<uint32_t *>(sllen + nslices);
  float *s_w = reinterpret_cast<float *>(s_cd + a.edge_cap);

  // ---- load this CTA's part of the network --------------------------------
  const long long sl0 = nd.slice_base + row0 / 32;
  const int my_slices = max(0, min(nslices, (N - row0 + 31) / 32));
  const long long ebase = my_slices ? a.sl_off[sl0] : 0;
  long long eend = ebase;
  for (int s = tid; s < nslices; s += blockDim.x) {
    if (s < my_slices) {
      sloff[s] = (int)(a.sl_off[sl0 + s] - ebase);
      sllen[s] = a.sl_len[sl0 + s];
    } else {
      sloff[s] = 0;
      sllen[s] = 0;
    }
  }
  if (my_slices) eend = a.sl_off[sl0 + my_slices - 1] + 32LL * a.sl_len[sl0 + my_slices - 1];
  const int nent = (int)(eend - ebase);
  for (int k = tid; k < nent; k += blockDim.x) {
    s_cd[k] = a.sl_cd[ebase + k];
    s_w[k] = a.sl_w[ebase + k];
  }
  int deg = 0;
  if (live) {
    const long long gi = nd.node_off + row;
    if (q == 0) {
      s_th[rloc] = a.theta[gi];
      s_thh[rloc] = a.theta_hat[gi];
      s_om[rloc] = a.omega[gi];
      s_omh[rloc] = a.omega_hat[gi];
    }
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }
  const NetState ns = *a.st;
  int cur = ns.cur, rbuf = ns.rbuf;
  float g = ns.g, r = ns.r;
  const int nblocks = (N + kTile - 1) / kTile;
  const float *ring = a.ring + nd.ring_off;
  float *ring_w = a.ring + nd.ring_off;
  const float dt = a.dt;
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  // the warp's 8 rows share one SELL slice
  const int wslice = (warp * (32 / LPR)) / 32;
  const bool slice_live = row0 + wslice * 32 < N;
  if (tid == 0) s_ok = 1;
  __syncthreads();

  const unsigned G = gridDim.x;
  // warp sums of step s into shared memory (warp 0), after barrier s
  auto stage_sums = [&](int s) {
    if (warp == 0) {
      const float2 *src = a.wsum + (s & 1) * nwarps;
      for (int c = lane; c < nwarps / 2; c += 32) cp_async_cg16(s_ws + 2 * c, src + 2 * c);
      cp_async_commit();
    }
  };
  int step = 0;
  bool ok = true;
  for (; step < a.n_steps; ++step) {
    // with zero delays: barrier step-1 before the gathers; the warp sums are
    // in flight during the predictor and the edge work
    if (step > 0 && !a.early) {
      if (!(ok = grid_wait(a.bar, (unsigned)step * G, a.err, &s_ok, a.wait))) break;
      stage_sums(step - 1);
    }
    // ---- predictor (row's first lane) --------------------------------------
    float th = 0.0f, eps = 0.0f;
    if (live && q == 0) {
      th = s_th[rloc];
      const float thh = s_thh[rloc];
      const float wh = s_omh[rloc];
      float diff = th - thh;
      diff = wrap_pm_pi(diff);
      eps = sinf(diff);
      s_thh[rloc] = thh + dt * wh;
      s_omh[rloc] = wh + nd.kappa_w * dt * eps;
    }
    th = __shfl_sync(mask, th, lead);
    eps = __shfl_sync(mask, eps, lead);
    const float my_eps = fabsf(eps);
    // ---- edges: lane q takes entries q, q+4, ...; the sum in CSR order -----
    float local_sum = 0.0f;
    if (slice_live) {
      const int len = sllen[wslice];
      const int base = sloff[wslice] + (rloc & 31);
      for (int kb = 0; kb < len; kb += LPR * U) {
        uint32_t p[U];
        float wv[U], dj[U], sn[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int k = kb + LPR * u + q;
          const bool in = k < deg;
          p[u] = in ? s_cd[base + 32 * k] : 0u;
          wv[u] = in ? s_w[base + 32 * k] : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          int slot = cur - (int)(p[u] & 255u);
          slot += (slot < 0) ? bsi : 0;
          dj[u] = __ldcg(ring + ring_pos(slot, p[u] >> 8, Np));
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int k = kb + LPR * u + q;
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
            s_w[base + 32 * k] = w;
          }
        }
#pragma unroll
        for (int e = 0; e < LPR * U; ++e) {
          const int srcl = lead + (e % LPR);
          const float w = __shfl_sync(mask, wv[e / LPR], srcl);
          const float sin_diff = __shfl_sync(mask, sn[e / LPR], srcl);
          if (kb + e < deg) local_sum += w * sin_diff;  // the expression of cluster_kernel
        }
      }
    }
    // ---- r and gain of the previous step (warp 0, from the staged sums) ----
    if (step > 0) {
      if (a.early) {
        if (!(ok = grid_wait(a.bar, (unsigned)step * G, a.err, &s_ok, a.wait))) break;
        stage_sums(step - 1);
      }
      if (warp == 0) {
        cp_async_wait_all();
        __syncwarp();
        const float2 sums = cluster_sums(s_ws, nblocks, lane);
        if (lane == 0) {
          float inv_N = 1.0f / (float)N;
          r = sqrtf(sums.x * sums.x + sums.y * sums.y) * inv_N;
          if (nd.ctrl) g = gain_controller(g, r, dt, nd);
          s_g = g;
          if (cta == 0 && a.r_hist) {
            const int k = ns.rpos + step - 1;
            if (k < a.r_cap) a.r_hist[k] = r;
          }
        }
      }
      __syncthreads();
      g = s_g;
    }
    // ---- integrate (row's first lane) --------------------------------------
    int nxt = cur + 1;
    if (nxt == bsi) nxt = 0;
    if (q == 0) {
      float my_cos = 0.0f, my_sin = 0.0f;
      if (live) {
        float inc = dt * (s_om[rloc] + g * local_sum - nd.alpha * eps);
        float x = th + inc;
        x = wrap_0_2pi(x);
        if (!isfinite(x)) x = 0.0f;
        s_th[rloc] = x;
        __stcg(ring_w + ring_pos(nxt, row, Np), x);
        lev_sincos<MATH>(x, &my_sin, &my_cos);
      }
      s_ord[rloc] = my_cos;
      s_ord[R + rloc] = my_sin;
    }
    __syncthreads();
    // ---- warp sums in row order (leviathan_kernel.cu:198-214) --------------
    if (tid < R) {
      float c = s_ord[tid], sn = s_ord[R + tid];
#pragma unroll
      for (int off = 16; off > 0; off /= 2) {
        c += __shfl_down_sync(mask, c, off);
        sn += __shfl_down_sync(mask, sn, off);
      }
      if (lane == 0) __stcg(a.wsum + (step & 1) * nwarps + row0 / 32 + warp, make_float2(c, sn));
    }
    cur = nxt;
    rbuf = (rbuf + 1 == nd.max_delay + 1) ? 0 : rbuf + 1;
    grid_arrive(a.bar);
  }
  // CTA 0 needs every warp sum of the last step
  if (ok && a.n_steps > 0 && cta == 0) ok = grid_wait(a.bar, (unsigned)a.n_steps * G, a.err, &s_ok, a.wait);
  if (!ok) return;  // barrier timeout: the host reports it
  // ---- r of the last step (CTA 0), then write the state back ---------------
  if (a.n_steps > 0 && cta == 0 && warp == 0) {
    const float2 *src = a.wsum + ((a.n_steps - 1) & 1) * nwarps;
    for (int k = lane; k < nwarps; k += 32) s_ws[k] = __ldcg(src + k);
    __syncwarp();
    const float2 sums = cluster_sums(s_ws, nblocks, lane);
    if (lane == 0) {
      float inv_N = 1.0f / (float)N;
      r = sqrtf(sums.x * sums.x + sums.y * sums.y) * inv_N;
      if (nd.ctrl) g = gain_controller(g, r, dt, nd);
      if (a.r_hist) {
        const int k = ns.rpos + a.n_steps - 1;
        if (k < a.r_cap) a.r_hist[k] = r;
      }
      NetState o = ns;
      o.g = g;
      o.r = r;
      o.cur = cur;
      o.rbuf = rbuf;
      o.t = ns.t + a.n_steps;
      o.rpos = ns.rpos + a.n_steps;
      o.ticket = 0u;
      *a.st = o;
    }
  }
  if (live && q == 0) {
    const long long gi = nd.node_off + row;
    a.theta[gi] = s_th[rloc];
    a.theta_hat[gi] = s_thh[rloc];
    a.omega_hat[gi] = s_omh[rloc];
  }
  for (int k = tid; k < nent; k += blockDim.x) a.sl_w[ebase + k] = s_w[k];
}

}  // namespace lev
