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
// per tile; 256 = the reference block size (leviathan_kernel.cu:354) so the
// block partial sums of cos/sin, and therefore r, are formed over the same
// node groups and in the same tree order as the reference.
//
// Layout in HBM (per network, packed over networks by offsets):
//   row_ptr  int32 [N+1]      local CSR offsets (as given by the caller)
//   cd       uint32[E]        (col_idx << 8) | delay  -- one 4-byte word
//   w        f32   [E]        plastic weights, updated in place
//   theta, theta_hat, omega, omega_hat  f32 [N]
//   ring     f32   [bsi][Np]  slot-major delay ring, bsi = max_delay + 2,
//                             Np = N rounded up to 32 (128-byte rows)
//
// The ring has one slot more than the reference's max_delay+1: step t reads
// slots (t-d) mod bsi for d in [0,max_delay] and writes theta(t+1) to slot
// (t+1) mod bsi, which no read of the same step touches.  The reference
// relies on separate launches for that ordering (:398 then :408); with the
// extra slot one launch per step is race-free for every delay in
// [0,max_delay] and the gathered values are identical.
//
// Edge phase: edges of the tile are processed flat (4 consecutive edges per
// thread per iteration, 16-byte loads of cd and w, coalesced across the
// warp); each edge finds its row in the staged row_ptr slice.  The coupling
// term sum_e w_e*sin(d_e) of a row is then accumulated by the row's thread in
// CSR order from shared memory, the same order and the same fused
// multiply-add as the reference's per-row loop (:137-154).
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

namespace lev {

constexpr int kTile = 256;    // rows per CTA == threads per CTA
constexpr int kChunk = 4096;  // edges staged in shared memory per pass

struct NetDesc {
  long long node_off;  // first node in the packed node arrays
  long long edge_off;  // first edge in the packed edge arrays
  long long ring_off;  // first float of the ring (multiple of 32)
  long long rp_off;    // first entry of the local row_ptr (N+1 entries)
  int N;
  int Np;         // ring row pitch
  int bsi;        // ring slots = max_delay + 2
  int max_delay;  // reference ring has max_delay + 1 slots
  int ntiles;     // 256-row tiles of this network
  int part_off;   // first partial-sum slot
  int tile_off;   // first tile (CTA) of this network in the grid
  int pad0;
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

struct StepArgs {
  const NetDesc *nets;
  NetState *st;
  const int2 *tiles;  // (network, first local row)
  const int *row_ptr;
  const uint32_t *cd;
  float *w;
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
};

// ---------------------------------------------------------------------------
// Arithmetic shared with the reference.  The expressions are written in the
// same form as leviathan_kernel.cu so that nvcc forms the same fused
// multiply-adds; see the line cited at each use.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float wrap_pm_pi(float diff) {
  // symmetric wrap to [-pi, pi): leviathan_kernel.cu:105 and :146
  const float TWO_PI = 2.0f * CUDART_PI_F;
  return diff - floorf(diff / TWO_PI + 0.5f) * TWO_PI;
}

__device__ __forceinline__ float wrap_0_2pi(float x) {
  // wrap to [0, 2pi): leviathan_kernel.cu:188
  const float TWO_PI = 2.0f * CUDART_PI_F;
  return x - floorf(x / TWO_PI) * TWO_PI;
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

// ---------------------------------------------------------------------------
// The fused step.
// ---------------------------------------------------------------------------
template <int MATH>
__global__ void __launch_bounds__(kTile, 3) step_kernel(const StepArgs a) {
  __shared__ int s_rp[kTile + 1];
  __shared__ float s_th[kTile];
  __shared__ float s_ae[kTile];
  __shared__ float2 s_ws[kChunk];
  __shared__ float s_rc[32];
  __shared__ float s_rs[32];
  __shared__ int s_last;

  const int tid = threadIdx.x;
  const int2 tile = a.tiles[blockIdx.x];
  const NetDesc nd = a.nets[tile.x];
  NetState *ns = a.st + tile.x;

  const int N = nd.N;
  const int row0 = tile.y;
  const int nrows = min(kTile, N - row0);
  const long long node0 = nd.node_off + row0;
  const float dt = a.dt;
  const int bsi = nd.bsi;
  const int Np = nd.Np;
  const int cur = ns->cur;
  const float g = ns->g;
  float *ring = a.ring + nd.ring_off;

  // ---- stage this tile's row_ptr slice ------------------------------------
  const int *rp = a.row_ptr + nd.rp_off + row0;
  for (int k = tid; k <= nrows; k += kTile) s_rp[k] = __ldg(rp + k);

  // ---- predictor (prep_kernel, leviathan_kernel.cu:100-110) ----------------
  float th = 0.0f, eps = 0.0f;
  if (tid < nrows) {
    const long long gi = node0 + tid;
    th = a.theta[gi];
    const float thh = a.theta_hat[gi];
    const float wh = a.omega_hat[gi];
    float diff = th - thh;
    diff = wrap_pm_pi(diff);
    eps = sinf(diff);
    a.theta_hat[gi] = thh + dt * wh;
    a.omega_hat[gi] = wh + nd.kappa_w * dt * eps;
  }
  s_th[tid] = th;
  s_ae[tid] = fabsf(eps);
  __syncthreads();

  // ---- edges (csr_physics_kernel, leviathan_kernel.cu:126-165) -------------
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  const long long eoff = nd.edge_off;
  const long long gbeg = eoff + s_rp[0];
  const long long gend = eoff + s_rp[nrows];
  const int my_rs = (tid < nrows) ? s_rp[tid] : 0;
  const int my_re = (tid < nrows) ? s_rp[tid + 1] : 0;

  float local_sum = 0.0f;
  int rlo = 0;  // row search lower bound, monotone in the edge index
  const long long vstart = (gbeg < gend) ? (gbeg & ~3LL) : gend;
  for (long long vc = vstart; vc < gend; vc += kChunk) {
    const long long cend = min(vc + (long long)kChunk, gend);
    for (long long g4 = vc + 4LL * tid; g4 < cend; g4 += 4LL * kTile) {
      const uint4 p = __ldcs(reinterpret_cast<const uint4 *>(a.cd + g4));
      const float4 wv = __ldcs(reinterpret_cast<const float4 *>(a.w + g4));
      const uint32_t pq[4] = {p.x, p.y, p.z, p.w};
      const float wq[4] = {wv.x, wv.y, wv.z, wv.w};
      float wn[4] = {wv.x, wv.y, wv.z, wv.w};
      // row of the first valid edge of this vector
      const long long efirst = g4 > gbeg ? g4 : gbeg;
      const int lef = (int)(efirst - eoff);
      int lo = rlo, hi = nrows;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s_rp[mid] <= lef) lo = mid; else hi = mid;
      }
      int r = lo;
      bool full = true;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const long long ge = g4 + q;
        if (ge < gbeg || ge >= cend) { full = false; continue; }
        const int le = (int)(ge - eoff);
        while (s_rp[r + 1] <= le) ++r;
        const int j = (int)(pq[q] >> 8);
        const int d = (int)(pq[q] & 255u);
        int slot = cur - d;
        slot += (slot < 0) ? bsi : 0;
        const float delayed_j = __ldg(ring + (long long)slot * Np + j);
        float diff = delayed_j - s_th[r];
        diff = wrap_pm_pi(diff);
        float w = wq[q];
        float sin_diff, cos_diff;
        lev_sincos<MATH>(diff, &sin_diff, &cos_diff);
        s_ws[ge - vc] = make_float2(w, sin_diff);
        const float my_eps = s_ae[r];
        float dw = dt * (eta * cos_diff * (1.0f - gamma * my_eps) - lam * w);
        w += dw;
        if (!isfinite(w)) w = w_min;
        w = fmaxf(w_min, fminf(w_max, w));
        wn[q] = w;
      }
      rlo = r;
      if (full) {
        __stcs(reinterpret_cast<float4 *>(a.w + g4),
               make_float4(wn[0], wn[1], wn[2], wn[3]));
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const long long ge = g4 + q;
          if (ge >= gbeg && ge < cend) a.w[ge] = wn[q];
        }
      }
    }
    __syncthreads();
    // coupling sum of this thread's row, CSR order (leviathan_kernel.cu:154)
    if (tid < nrows) {
      const long long b = max(eoff + my_rs, vc);
      const long long e = min(eoff + my_re, cend);
      for (long long x = b; x < e; ++x) {
        const float2 v = s_ws[x - vc];
        local_sum += v.x * v.y;
      }
    }
    __syncthreads();
  }

  // ---- integrate (integrate_and_reduce_kernel, leviathan_kernel.cu:182-196)
  int nxt = cur + 1;
  if (nxt == bsi) nxt = 0;
  float my_cos = 0.0f, my_sin = 0.0f;
  if (tid < nrows) {
    const long long gi = node0 + tid;
    float inc = dt * (a.omega[gi] + g * local_sum - nd.alpha * eps);
    float x = th + inc;
    x = wrap_0_2pi(x);
    if (!isfinite(x)) x = 0.0f;
    a.theta[gi] = x;
    ring[(long long)nxt * Np + row0 + tid] = x;
    lev_sincos<MATH>(x, &my_sin, &my_cos);
  }

  // ---- block partial of (sum cos, sum sin) (leviathan_kernel.cu:198-233) ---
  const unsigned mask = 0xffffffffu;
#pragma unroll
  for (int off = 16; off > 0; off /= 2) {
    my_cos += __shfl_down_sync(mask, my_cos, off);
    my_sin += __shfl_down_sync(mask, my_sin, off);
  }
  const int lane = tid & 31, warp = tid >> 5;
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
      s_last = (prev == (unsigned)(nd.ntiles - 1));
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
    }
  }
}

// ---------------------------------------------------------------------------
// Helpers
// ---------------------------------------------------------------------------

// Every ring slot of every node := theta (init_buffer_kernel,
// leviathan_kernel.cu:79-90, in the slot-major layout).
__global__ void ring_fill_kernel(const float *__restrict__ theta,
                                 float *__restrict__ ring, int N, int Np,
                                 int bsi) {
  const long long total = (long long)bsi * N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
       k < total; k += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(k / N);
    const int i = (int)(k - (long long)s * N);
    ring[(long long)s * Np + i] = theta[i];
  }
}

// cd[e] := (col[e] << 8) | delay[e], in place over cd (which holds col on
// entry).  Out-of-range columns or delays set bits of *err.
__global__ void pack_edges_kernel(uint32_t *__restrict__ cd,
                                  const uint8_t *__restrict__ delays,
                                  long long E, int N, int max_delay,
                                  unsigned *__restrict__ err) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
       e += (long long)gridDim.x * blockDim.x) {
    const int col = (int)cd[e];
    const int d = delays[e];
    unsigned bad = 0u;
    if (col < 0 || col >= N) bad |= 1u;
    if (d > max_delay) bad |= 2u;
    if (bad) atomicOr(err, bad);
    cd[e] = ((uint32_t)col << 8) | (uint32_t)d;
  }
}

// r-history row counters := 0 (first node of every captured step block).
__global__ void reset_rpos_kernel(NetState *st, int num_nets) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < num_nets;
       n += gridDim.x * blockDim.x)
    st[n].rpos = 0;
}

}  // namespace lev
