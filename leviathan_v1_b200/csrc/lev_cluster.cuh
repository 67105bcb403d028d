// lev_cluster.cuh -- cluster-resident engine for small networks.  Included
// once, from lev_engine.cu.
//
// A network of up to 16 x 1024 nodes whose edges, node state and delay ring
// fit in the shared memory of one thread-block cluster (up to 16 CTAs, one per
// SM, 227 KB each) is stepped n times in ONE launch:
//   * CTA r of the cluster owns rows [r*R, r*R + R), R a multiple of 32, one
//     thread per row; its SELL-32 slices (col|delay, weights), its node state
//     and its rows of every ring slot live in its shared memory;
//   * a delayed phase of a node owned by another CTA is read from that CTA's
//     shared memory (distributed shared memory, cluster.map_shared_rank);
//   * one cluster barrier per step, split into an arrival after step t's
//     ring write and warp sums and a wait before step t+1's integrate (which
//     needs g(t+1) and overwrites ring slot t+2 = t-max_delay, read by step
//     t).  Without zero delays step t+1's gathers read slots <= t, ordered by
//     the barrier of step t-1, so the predictor and the edge work of step t+1
//     run while the barrier of step t completes; with zero delays the wait
//     comes before the gathers (with max_delay+2 ring slots, reads and the
//     write of one step never touch the same slot);
//   * each warp's shuffle-tree (sum cos, sum sin) of its 32 rows goes to a
//     double-buffered array in CTA 0; after the barrier every CTA forms the
//     256-node block sums from eight warp sums with the arithmetic of the
//     reference's block tree (leviathan_kernel.cu:198-233) and reduces the
//     blocks in the order of :242-263, so all CTAs compute the same r and
//     gain without a second barrier.  A 256-node block may thus span CTAs,
//     and a small network spreads over up to 16 SMs.
// Arithmetic and summation order are those of step_kernel: results are
// bitwise the same as stepping with step_kernel.

#include <cooperative_groups.h>

namespace lev {

constexpr int kClusterMax = 16;     // CTAs per cluster (non-portable size)
constexpr int kClusterRowsMax = 1024;
constexpr int kClusterWarpsMax = kClusterMax * kClusterRowsMax / 32;  // 512

// Sum of one 256-node block from its eight warp sums v[0..7], with the
// arithmetic of the reference's second-level tree (leviathan_kernel.cu:
// 216-233: warp 0 takes the eight warp sums in lanes 0-7, zeros elsewhere,
// then shuffle-down adds at offsets 16, 8, 4, 2, 1): the first two levels add
// zeros (which turns -0 into +0), then (v0+v4, ...), then pairs, then one.
__device__ __forceinline__ float block_tree8(const float *v) {
  float z[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) z[i] = __fadd_rn(__fadd_rn(v[i], 0.0f), 0.0f);
  const float a0 = __fadd_rn(z[0], z[4]), a1 = __fadd_rn(z[1], z[5]);
  const float a2 = __fadd_rn(z[2], z[6]), a3 = __fadd_rn(z[3], z[7]);
  return __fadd_rn(__fadd_rn(a0, a2), __fadd_rn(a1, a3));
}

// r of one step from the warp sums wsum[nwarps_blocks * 8] (one warp: lane l
// adds blocks l, l+32, ..., then the shuffle tree), as final_reduce_r_kernel
// (leviathan_kernel.cu:242-263) over the reference's block partials.
__device__ __forceinline__ float2 cluster_sums(const float2 *wsum, int nblocks, int lane) {
  float sum_cos = 0.0f, sum_sin = 0.0f;
  for (int b = lane; b < nblocks; b += 32) {
    float vc[8], vs[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float2 v = wsum[b * 8 + i];
      vc[i] = v.x;
      vs[i] = v.y;
    }
    sum_cos += block_tree8(vc);
    sum_sin += block_tree8(vs);
  }
  const unsigned mask = 0xffffffffu;
#pragma unroll
  for (int off = 16; off > 0; off /= 2) {
    sum_cos += __shfl_down_sync(mask, sum_cos, off);
    sum_sin += __shfl_down_sync(mask, sum_sin, off);
  }
  return make_float2(sum_cos, sum_sin);
}

struct ClusterArgs {
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
  float *r_hist;  // [n] (row rpos + k), or null
  int r_cap;
  int n_steps;
  int R;          // rows per CTA (a power of two, 32 .. 1024)
  int lgR;        // log2(R)
  int edge_cap;   // SELL entries per CTA the shared memory was sized for
  int early;      // no delay is 0: wait for step t's barrier after step t+1's edges
  float dt;
};

// Split cluster barrier (every thread of every CTA of the cluster): arrival
// with release semantics, wait with acquire semantics.
__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// shared memory layout (bytes, from the dynamic base):
//   wsum   float2 [2][kClusterWarpsMax]        warp sums (used in CTA 0)
//   sloff  int    [R/32]   slice start (relative to the CTA's first entry)
//   sllen  int    [R/32]
//   th, thh, om, omh  float [R]
//   ring   float  [bsi][R]
//   cd     uint32 [edge_cap]
//   w      float  [edge_cap]
// MAXR: largest rows per CTA of the instantiation (the register budget);
// U: edges per lane whose gathers are in flight together.
template <int MATH, int MAXR, int U>
__global__ void __launch_bounds__(MAXR, 1) cluster_kernel(const ClusterArgs a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem[];

  const NetDesc nd = *a.net;
  const int rank = (int)cluster.block_rank();
  const int R = a.R;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N = nd.N, bsi = nd.bsi, Np = nd.Np;
  const int row0 = rank * R;
  const int row = row0 + tid;
  const bool live = (tid < R) && (row < N);
  const int nslices = R / 32;

  float2 *wsum = reinterpret_cast<float2 *>(smem);
  int *sloff = reinterpret_cast<int *>(wsum + 2 * kClusterWarpsMax);
  int *sllen = sloff + nslices;
  float *s_th = reinterpret_cast<float *>(sllen + nslices);
  float *s_thh = s_th + R;
  float *s_om = s_thh + R;
  float *s_omh = s_om + R;
  float *s_ring = s_omh + R;
  uint32_t *s_cd = reinterpret_cast<uint32_t *>(s_ring + (size_t)bsi * R);
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
    s_th[tid] = a.theta[gi];
    s_thh[tid] = a.theta_hat[gi];
    s_om[tid] = a.omega[gi];
    s_omh[tid] = a.omega_hat[gi];
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }
  for (int s = 0; s < bsi; ++s)
    if (live) s_ring[(size_t)s * R + tid] = a.ring[nd.ring_off + ring_pos(s, row, Np)];
  NetState ns = *a.st;
  int cur = ns.cur, rbuf = ns.rbuf;
  float g = ns.g, r = ns.r;
  const int nblocks = (N + kTile - 1) / kTile;
  // warps past the network's last row contribute zero sums to their block
  if (rank == 0)
    for (int k = tid; k < 2 * kClusterWarpsMax; k += blockDim.x) wsum[k] = make_float2(0.0f, 0.0f);
  const float dt = a.dt;
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  const unsigned mask = 0xffffffffu;
  cluster.sync();

  float2 *wsum0 = cluster.map_shared_rank(wsum, 0);
  __shared__ float s_g;
  for (int step = 0; step < a.n_steps; ++step) {
    // with zero delays: step-1's barrier before the gathers
    if (step > 0 && !a.early) cluster_wait();
    // ---- predictor --------------------------------------------------------
    float th = 0.0f, eps = 0.0f;
    if (live) {
      th = s_th[tid];
      const float thh = s_thh[tid];
      const float wh = s_omh[tid];
      float diff = th - thh;
      diff = wrap_pm_pi(diff);
      eps = sinf(diff);
      s_thh[tid] = thh + dt * wh;
      s_omh[tid] = wh + nd.kappa_w * dt * eps;
    }
    const float my_eps = fabsf(eps);
    // ---- edges --------------------------------------------------------------
    float local_sum = 0.0f;
    if (warp < my_slices) {
      const int len = sllen[warp];
      const int base = sloff[warp] + lane;
      for (int k0 = 0; k0 < len; k0 += U) {
        uint32_t p[U];
        float wv[U], dj[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const bool in = k0 + u < deg;
          p[u] = in ? s_cd[base + 32 * (k0 + u)] : 0u;
          wv[u] = in ? s_w[base + 32 * (k0 + u)] : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          int slot = cur - (int)(p[u] & 255u);
          slot += (slot < 0) ? bsi : 0;
          const int j = (int)(p[u] >> 8);
          const int owner = j >> a.lgR;
          const int loc = j & (R - 1);
          const float *src = (owner == rank) ? s_ring : cluster.map_shared_rank(s_ring, owner);
          dj[u] = src[(size_t)slot * R + loc];
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
            s_w[base + 32 * (k0 + u)] = w;
          }
        }
      }
    }
    // ---- r and gain of the previous step: warp 0 of every CTA reduces the
    // block partials (same order everywhere) and shares g with its CTA ----
    if (step > 0) {
      if (a.early) cluster_wait();
      if (warp == 0) {
        const float2 sums =
            cluster_sums(wsum0 + ((step - 1) & 1) * kClusterWarpsMax, nblocks, lane);
        const float sum_cos = sums.x, sum_sin = sums.y;
        if (lane == 0) {
          float inv_N = 1.0f / (float)N;
          r = sqrtf(sum_cos * sum_cos + sum_sin * sum_sin) * inv_N;
          if (nd.ctrl) g = gain_controller(g, r, dt, nd);
          s_g = g;
          if (rank == 0 && a.r_hist) {
            const int k = ns.rpos + step - 1;
            if (k < a.r_cap) a.r_hist[k] = r;
          }
        }
      }
      __syncthreads();
      g = s_g;
    }
    // ---- integrate ----------------------------------------------------------
    int nxt = cur + 1;
    if (nxt == bsi) nxt = 0;
    float my_cos = 0.0f, my_sin = 0.0f;
    if (live) {
      float inc = dt * (s_om[tid] + g * local_sum - nd.alpha * eps);
      float x = th + inc;
      x = wrap_0_2pi(x);
      if (!isfinite(x)) x = 0.0f;
      s_th[tid] = x;
      s_ring[(size_t)nxt * R + tid] = x;
      lev_sincos<MATH>(x, &my_sin, &my_cos);
    }
    // ---- warp sums of (cos, sin), first level of the block tree
    // (leviathan_kernel.cu:198-214), to CTA 0 ------------------------------
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      my_cos += __shfl_down_sync(mask, my_cos, off);
      my_sin += __shfl_down_sync(mask, my_sin, off);
    }
    if (lane == 0)
      wsum0[(step & 1) * kClusterWarpsMax + row0 / 32 + warp] = make_float2(my_cos, my_sin);
    cur = nxt;
    rbuf = (rbuf + 1 == nd.max_delay + 1) ? 0 : rbuf + 1;
    cluster_arrive();
  }
  if (a.n_steps > 0) cluster_wait();
  // ---- r of the last step, then write the state back ------------------------
  if (a.n_steps > 0) {
    const float2 sums =
        cluster_sums(wsum0 + ((a.n_steps - 1) & 1) * kClusterWarpsMax, nblocks, lane);
    const float sum_cos = __shfl_sync(mask, sums.x, 0);
    const float sum_sin = __shfl_sync(mask, sums.y, 0);
    float inv_N = 1.0f / (float)N;
    r = sqrtf(sum_cos * sum_cos + sum_sin * sum_sin) * inv_N;
    if (nd.ctrl) g = gain_controller(g, r, dt, nd);
    if (rank == 0 && tid == 0) {
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
  if (live) {
    const long long gi = nd.node_off + row;
    a.theta[gi] = s_th[tid];
    a.theta_hat[gi] = s_thh[tid];
    a.omega_hat[gi] = s_omh[tid];
    for (int s = 0; s < bsi; ++s)
      a.ring[nd.ring_off + ring_pos(s, row, Np)] = s_ring[(size_t)s * R + tid];
  }
  for (int k = tid; k < nent; k += blockDim.x) a.sl_w[ebase + k] = s_w[k];
  // no CTA may leave while a peer can still read its shared memory
  cluster.sync();
}

// The cluster-resident step with four lanes per row (CTA = 4R threads, R up
// to 128, lanes 4r .. 4r+3 on row r).  The row's first lane runs the node work and forms the
// coupling sum in CSR order from the per-edge terms the row's lanes computed
// (shuffled, same expression); the warp-level trees of the block sums read
// the rows' values from shared memory in row order.  Bitwise the results of
// cluster_kernel and step_kernel.  Shared memory as cluster_kernel plus
// ord float [2][R] after omh.
template <int MATH, int U>
__global__ void __launch_bounds__(4 * 128, 1) cluster_split_kernel(const ClusterArgs a) {
  namespace cg = cooperative_groups;
  constexpr int LPR = 4;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem[];

  const NetDesc nd = *a.net;
  const int rank = (int)cluster.block_rank();
  const int R = a.R;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = tid & (LPR - 1);
  const int rloc = tid / LPR;
  const int lead = lane & ~(LPR - 1);
  const unsigned mask = 0xffffffffu;
  const int N = nd.N, bsi = nd.bsi, Np = nd.Np;
  const int row0 = rank * R;
  const int row = row0 + rloc;
  const bool live = row < N;
  const int nslices = R / 32;

  float2 *wsum = reinterpret_cast<float2 *>(smem);
  int *sloff = reinterpret_cast<int *>(wsum + 2 * kClusterWarpsMax);
  int *sllen = sloff + nslices;
  float *s_th = reinterpret_cast<float *>(sllen + nslices);
  float *s_thh = s_th + R;
  float *s_om = s_thh + R;
  float *s_omh = s_om + R;
  float *s_ord = s_omh + R;
  float *s_ring = s_ord + 2 * R;
  uint32_t *s_cd = reinterpret_cast<uint32_t *>(s_ring + (size_t)bsi * R);
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
  for (int s = q; s < bsi; s += LPR)
    if (live) s_ring[(size_t)s * R + rloc] = a.ring[nd.ring_off + ring_pos(s, row, Np)];
  NetState ns = *a.st;
  int cur = ns.cur, rbuf = ns.rbuf;
  float g = ns.g, r = ns.r;
  const int nblocks = (N + kTile - 1) / kTile;
  if (rank == 0)
    for (int k = tid; k < 2 * kClusterWarpsMax; k += blockDim.x) wsum[k] = make_float2(0.0f, 0.0f);
  const float dt = a.dt;
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  // the warp's 8 rows share one SELL slice
  const int wslice = (warp * (32 / LPR)) / 32;
  const bool slice_live = row0 + wslice * 32 < N;
  cluster.sync();

  float2 *wsum0 = cluster.map_shared_rank(wsum, 0);
  __shared__ float s_g;
  for (int step = 0; step < a.n_steps; ++step) {
    // with zero delays: step-1's barrier before the gathers
    if (step > 0 && !a.early) cluster_wait();
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
          const int j = (int)(p[u] >> 8);
          const int owner = j >> a.lgR;
          const int loc = j & (R - 1);
          const float *src = (owner == rank) ? s_ring : cluster.map_shared_rank(s_ring, owner);
          dj[u] = src[(size_t)slot * R + loc];
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
    // ---- r and gain of the previous step (warp 0 of every CTA) -------------
    if (step > 0) {
      if (a.early) cluster_wait();
      if (warp == 0) {
        const float2 sums =
            cluster_sums(wsum0 + ((step - 1) & 1) * kClusterWarpsMax, nblocks, lane);
        if (lane == 0) {
          float inv_N = 1.0f / (float)N;
          r = sqrtf(sums.x * sums.x + sums.y * sums.y) * inv_N;
          if (nd.ctrl) g = gain_controller(g, r, dt, nd);
          s_g = g;
          if (rank == 0 && a.r_hist) {
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
        s_ring[(size_t)nxt * R + rloc] = x;
        lev_sincos<MATH>(x, &my_sin, &my_cos);
      }
      s_ord[rloc] = my_cos;
      s_ord[R + rloc] = my_sin;
    }
    __syncthreads();
    // ---- warp sums in row order to CTA 0 (leviathan_kernel.cu:198-214) ----
    if (tid < R) {
      float c = s_ord[tid], sn = s_ord[R + tid];
#pragma unroll
      for (int off = 16; off > 0; off /= 2) {
        c += __shfl_down_sync(mask, c, off);
        sn += __shfl_down_sync(mask, sn, off);
      }
      if (lane == 0)
        wsum0[(step & 1) * kClusterWarpsMax + row0 / 32 + warp] = make_float2(c, sn);
    }
    cur = nxt;
    rbuf = (rbuf + 1 == nd.max_delay + 1) ? 0 : rbuf + 1;
    cluster_arrive();
  }
  if (a.n_steps > 0) cluster_wait();
  // ---- r of the last step, then write the state back ------------------------
  if (a.n_steps > 0) {
    const float2 sums =
        cluster_sums(wsum0 + ((a.n_steps - 1) & 1) * kClusterWarpsMax, nblocks, lane);
    const float sum_cos = __shfl_sync(mask, sums.x, 0);
    const float sum_sin = __shfl_sync(mask, sums.y, 0);
    float inv_N = 1.0f / (float)N;
    r = sqrtf(sum_cos * sum_cos + sum_sin * sum_sin) * inv_N;
    if (nd.ctrl) g = gain_controller(g, r, dt, nd);
    if (rank == 0 && tid == 0) {
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
  if (live) {
    const long long gi = nd.node_off + row;
    if (q == 0) {
      a.theta[gi] = s_th[rloc];
      a.theta_hat[gi] = s_thh[rloc];
      a.omega_hat[gi] = s_omh[rloc];
    }
    for (int s = q; s < bsi; s += LPR)
      a.ring[nd.ring_off + ring_pos(s, row, Np)] = s_ring[(size_t)s * R + rloc];
  }
  for (int k = tid; k < nent; k += blockDim.x) a.sl_w[ebase + k] = s_w[k];
  // no CTA may leave while a peer can still read its shared memory
  cluster.sync();
}

}  // namespace lev
