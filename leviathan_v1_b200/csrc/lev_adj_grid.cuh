// lev_adj_grid.cuh -- grid-resident adjoint kernels for single networks whose
// CTAs all fit on the device at once.  Included once, from lev_engine.cu,
// after lev_grid.cuh and lev_adjoint.cuh.
//
// One cooperative launch runs a whole checkpoint segment:
//   adj_grid_fwd_kernel  the forward steps of the segment with the recording
//                        hooks of adj_fwd_kernel (pre-step theta_hat, post-step
//                        weights, per-step (g, r, sum cos, sum sin), r, theta),
//                        the grid_kernel scheme: rows' state and SELL slices
//                        in shared memory, the ring in L2, warp sums and one
//                        grid barrier per step.  Bitwise the trajectory of
//                        adj_fwd_kernel and of the engine.
//   adj_grid_bwd_kernel  the reverse steps of the segment, last to first, with
//                        the arithmetic of adj_bwd_split_kernel.  The adjoint
//                        node state (lam_theta, lam_theta_hat, lam_omega_hat,
//                        the omega gradient) and lam_w stay in shared memory;
//                        the adjoint ring takes the red.add scatters in global
//                        memory.  lam_g(s) = lam_g(s+1) dg/dg + sum_i lam_th'_i
//                        dt S_i: every CTA writes its part, and after the grid
//                        barrier every CTA adds the parts in the same order.
//                        One barrier per reverse step orders the scatters into
//                        slot s+1 before reverse step s reads it.  Only lam_g
//                        needs the barrier of the step reversed just before:
//                        the history, weight and trace loads of step s, the
//                        first group of its edge loads and, without zero
//                        delays, its adjoint-ring slot (whose scatters came
//                        from steps s+2 and later) are issued before the wait.
// Both use the bounded barrier of lev_grid.cuh (error flag on a timeout).

#pragma once

namespace lev {

struct AdjGridFwdArgs {
  const NetDesc *net;  // adjoint copy: bsi = C + max_delay + 2
  NetState *st;
  const int *row_ptr;
  const long long *sl_off;
  const int *sl_len;
  const uint32_t *sl_cd;
  const float *w_in;   // SELL weights before the first step
  float *w_out;        // after the last step (may alias w_in)
  float *w_rec;        // weights after step k at w_rec + k*SL, or null
  float *theta;
  float *theta_hat;
  const float *omega;
  float *omega_hat;
  float *ring;
  const float *drive;  // drive of step k at drive + k*N, or null
  const float *win;    // reservoir drive u_i = win_i * xin[k], or null
  const float *xin;
  float *thh_rec;      // theta_hat before step k at thh_rec + k*N, or null
  float4 *trace;       // (g, r, sum cos, sum sin) of step k at trace[k], or null
  float *r_out;        // r after step k at r_out[k], or null
  float *theta_out;    // theta after step k at theta_out + k*N, or null
  float2 *wsum;        // [2][nwarps]
  unsigned *bar;
  int *err;
  GridWait wait;  // bound of the barrier waits
  // the segment's checkpoint (theta, theta_hat, omega_hat, SELL weights, the
  // last max_delay+1 ring slots as [m][N], g): ck_mode 1 writes it from the
  // initial state (forward pass); 2 takes the initial state from it and
  // refills ring slots 0..max_delay, the unwrapped segment ring (backward
  // recompute), then w0_out (if not null) receives the initial weights
  int ck_mode;
  float *ck_theta, *ck_thh, *ck_omh, *ck_w, *ck_ring, *ck_g;
  float *w0_out;
  long long SL;
  int early;           // no delay is 0
  int nwarps;
  int edge_cap;
  int n_steps;
  float dt;
};

// R rows per CTA, four lanes per row; U edges per lane in flight together.
// Shared memory: s_ws float2[nwarps], th/thh/om/omh float[R], ord float[2R],
// sloff/sllen int[R/32], cd uint32[edge_cap], w float[edge_cap].
// The body runs as CTA `cta` of a group of G CTAs (the whole grid, or one
// half of a paired launch).
template <int MATH, int R, int U>
__device__ __forceinline__ void adj_grid_fwd_body(const AdjGridFwdArgs &a, const int cta,
                                                  const unsigned G, unsigned char *smem) {
  constexpr int LPR = kGridLPR;
  constexpr int nslices = R / 32;
  __shared__ float s_g;
  __shared__ int s_ok;

  const NetDesc nd = *a.net;
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
  const bool restore = a.ck_mode == 2;
  const float *w_src = restore ? a.ck_w : a.w_in;
  for (int k = tid; k < nent; k += blockDim.x) {
    s_cd[k] = a.sl_cd[ebase + k];
    const float w = w_src[ebase + k];
    s_w[k] = w;
    if (a.ck_mode == 1) a.ck_w[ebase + k] = w;
    if (restore && a.w0_out) a.w0_out[ebase + k] = w;
  }
  const long long gi = nd.node_off + row;
  int deg = 0;
  if (live) {
    if (q == 0) {
      const float th0 = restore ? a.ck_theta[gi] : a.theta[gi];
      const float thh0 = restore ? a.ck_thh[gi] : a.theta_hat[gi];
      const float omh0 = restore ? a.ck_omh[gi] : a.omega_hat[gi];
      s_th[rloc] = th0;
      s_thh[rloc] = thh0;
      s_om[rloc] = a.omega[gi];
      s_omh[rloc] = omh0;
      if (a.ck_mode == 1) {
        a.ck_theta[gi] = th0;
        a.ck_thh[gi] = thh0;
        a.ck_omh[gi] = omh0;
      }
    }
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }
  NetState ns;
  if (restore) {
    // the state of a restored segment (adj_state_kernel mode 2)
    ns.g = a.ck_g[0];
    ns.r = 0.0f;
    ns.cur = nd.max_delay;
    ns.ticket = 0u;
    ns.t = 0;
    ns.rbuf = 0;
    ns.rpos = 0;
  } else {
    ns = *a.st;
  }
  if (a.ck_mode == 1) {
    // ring window: theta(t - m) -> ck_ring[m][N], m = 0..max_delay
    if (live)
      for (int m = q; m <= nd.max_delay; m += LPR) {
        int slot = ns.cur - m;
        slot += (slot < 0) ? nd.bsi : 0;
        a.ck_ring[(long long)m * N + row] = a.ring[nd.ring_off + (long long)slot * nd.Np + row];
      }
    if (cta == 0 && tid == 0) a.ck_g[0] = ns.g;
  }
  int cur = ns.cur;
  float g = ns.g, r = ns.r;
  const int nblocks = (N + kTile - 1) / kTile;
  const float *ring = a.ring + nd.ring_off;
  float *ring_w = a.ring + nd.ring_off;
  const float dt = a.dt;
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  const int wslice = (warp * (32 / LPR)) / 32;
  const bool slice_live = row0 + wslice * 32 < N;
  if (tid == 0) s_ok = 1;
  __syncthreads();
  // restored segment: theta(s0 - m) -> ring slot max_delay - m of every row,
  // read by every CTA's first gathers: one grid barrier before step 0
  unsigned base = 0;
  if (restore) {
    if (live)
      for (int m = q; m <= nd.max_delay; m += LPR)
        __stcg(ring_w + (long long)(nd.max_delay - m) * Np + row, a.ck_ring[(long long)m * N + row]);
    grid_arrive(a.bar);
    if (!grid_wait(a.bar, G, a.err, &s_ok, a.wait)) return;
    base = G;
  }

  auto stage_sums = [&](int s) {
    if (warp == 0) {
      const float2 *src = a.wsum + (s & 1) * nwarps;
      for (int c = lane; c < nwarps / 2; c += 32) cp_async_cg16(s_ws + 2 * c, src + 2 * c);
      cp_async_commit();
    }
  };
  // r of step s-1 and the gain of step s (warp 0, lane 0 holds the result);
  // CTA 0 records the previous step
  auto reduce_prev = [&](int s) {
    if (warp == 0) {
      cp_async_wait_all();
      __syncwarp();
      const float2 sums = cluster_sums(s_ws, nblocks, lane);
      if (lane == 0) {
        float inv_N = 1.0f / (float)N;
        r = sqrtf(sums.x * sums.x + sums.y * sums.y) * inv_N;
        const float gn = nd.ctrl ? gain_controller(g, r, dt, nd) : g;
        if (cta == 0) {
          if (a.trace) a.trace[s - 1] = make_float4(g, r, sums.x, sums.y);
          if (a.r_out) a.r_out[s - 1] = r;
        }
        g = gn;
        s_g = g;
      }
    }
  };

  int step = 0;
  bool ok = true;
  for (; step < a.n_steps; ++step) {
    if (step > 0 && !a.early) {
      if (!(ok = grid_wait(a.bar, base + (unsigned)step * G, a.err, &s_ok, a.wait))) break;
      stage_sums(step - 1);
    }
    // ---- predictor (row's first lane) --------------------------------------
    float th = 0.0f, eps = 0.0f;
    if (live && q == 0) {
      th = s_th[rloc];
      const float thh = s_thh[rloc];
      const float wh = s_omh[rloc];
      if (a.thh_rec) a.thh_rec[(long long)step * N + gi] = thh;
      float diff = th - thh;
      diff = wrap_pm_pi(diff);
      eps = sinf(diff);
      s_thh[rloc] = thh + dt * wh;
      s_omh[rloc] = wh + nd.kappa_w * dt * eps;
    }
    th = __shfl_sync(mask, th, lead);
    eps = __shfl_sync(mask, eps, lead);
    const float my_eps = fabsf(eps);
    // ---- edges -------------------------------------------------------------
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
          dj[u] = __ldcg(ring + (size_t)slot * Np + (int)(p[u] >> 8));
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
          if (kb + e < deg) local_sum += w * sin_diff;  // the expression of adj_fwd_kernel
        }
      }
    }
    if (step > 0) {
      if (a.early) {
        if (!(ok = grid_wait(a.bar, base + (unsigned)step * G, a.err, &s_ok, a.wait))) break;
        stage_sums(step - 1);
      }
      reduce_prev(step);
      __syncthreads();
      g = s_g;
    }
    // ---- integrate (row's first lane) --------------------------------------
    int nxt = cur + 1;
    if (nxt == bsi) nxt = 0;
    if (q == 0) {
      float my_cos = 0.0f, my_sin = 0.0f;
      if (live) {
        float inc;
        if (a.drive || a.win) {
          float u = 0.0f;
          if (a.drive) u += a.drive[(long long)step * N + gi];
          if (a.win) u += a.win[gi] * a.xin[step];
          inc = dt * (s_om[rloc] + g * local_sum - nd.alpha * eps + u);
        } else {
          inc = dt * (s_om[rloc] + g * local_sum - nd.alpha * eps);
        }
        float x = th + inc;
        x = wrap_0_2pi(x);
        if (!isfinite(x)) x = 0.0f;
        s_th[rloc] = x;
        __stcg(ring_w + (size_t)nxt * Np + row, x);
        if (a.theta_out) a.theta_out[(long long)step * N + gi] = x;
        lev_sincos<MATH>(x, &my_sin, &my_cos);
      }
      s_ord[rloc] = my_cos;
      s_ord[R + rloc] = my_sin;
    }
    __syncthreads();
    // ---- post-step weights, warp sums ---------------------------------------
    if (a.w_rec) {
      float *wr = a.w_rec + (long long)step * a.SL + ebase;
      for (int k = tid; k < nent; k += blockDim.x) wr[k] = s_w[k];
    }
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
    grid_arrive(a.bar);
  }
  if (ok && a.n_steps > 0 && cta == 0)
    ok = grid_wait(a.bar, base + (unsigned)a.n_steps * G, a.err, &s_ok, a.wait);
  if (!ok) return;
  if (a.n_steps > 0 && cta == 0 && warp == 0) {
    const float2 *src = a.wsum + ((a.n_steps - 1) & 1) * nwarps;
    for (int c = lane; c < nwarps / 2; c += 32) cp_async_cg16(s_ws + 2 * c, src + 2 * c);
    cp_async_commit();
    reduce_prev(a.n_steps);
    if (lane == 0) {
      NetState o = ns;
      o.g = g;
      o.r = r;
      o.cur = cur;
      o.t = ns.t + a.n_steps;
      o.ticket = 0u;
      *a.st = o;
    }
  }
  if (live && q == 0) {
    a.theta[gi] = s_th[rloc];
    a.theta_hat[gi] = s_thh[rloc];
    a.omega_hat[gi] = s_omh[rloc];
  }
  for (int k = tid; k < nent; k += blockDim.x) a.w_out[ebase + k] = s_w[k];
}

struct AdjGridBwdArgs {
  const NetDesc *net;  // adjoint copy (ring_off: history ring, aux_off: adjoint ring)
  const int *row_ptr;
  const long long *sl_off;
  const int *sl_len;
  const uint32_t *sl_cd;
  const float *w_hist;   // weights before step seg_start + k at w_hist + k*SL
  const float *H;        // history ring: theta(tau) at slot tau - seg_start + max_delay
  const float *thh_hist; // theta_hat before step seg_start + k at thh_hist + k*N
  const float4 *trace;   // (g_s, r_{s+1}, sum cos, sum sin) of step seg_start + k at trace[k]
  const float *dLdr;     // dL/dr(s+1) at dLdr[s], or null
  const float *dLdth;    // dL/dtheta(s+1) at dLdth + s*N, or null
  float *grad_drive;     // at grad_drive + s*N, or null
  const float *win;      // reservoir drive (xin[s]); grad_win accumulated; or null
  const float *xin;
  float *grad_win;
  float *lam_th;
  float *lam_thh;
  float *lam_omh;
  float *lam_w;          // SELL
  float *adj_ring;
  float *lam_g;          // [1]: in lam_g(seg_end), out lam_g(seg_start)
  float *grad_omega;     // accumulated
  float *lgp;            // [2][group CTAs rounded up to 4] per-CTA lam_g parts
  unsigned *bar;
  int *err;
  GridWait wait;  // bound of the barrier waits
  int early;             // no delay is 0: slot s+1 is complete one barrier earlier
  long long SL;
  long long seg_start;
  int n_steps;           // reverse steps seg_start + n_steps - 1 .. seg_start
  int edge_cap;
  float dt;
};

// R rows per CTA, four lanes per row; U edges per lane in flight together.
// Shared memory: lt/lthh/lomh/go float[R], lgp float[G rounded up to 4],
// sloff/sllen int[R/32], cd uint32[edge_cap], lw float[edge_cap].
template <int MATH, int R, int U>
__device__ __forceinline__ void adj_grid_bwd_body(const AdjGridBwdArgs &a, const int cta,
                                                  const unsigned G, unsigned char *smem) {
  constexpr int LPR = kGridLPR;
  constexpr int nslices = R / 32;
  __shared__ float s_red[32];
  __shared__ float s_lg;
  __shared__ int s_ok;

  const NetDesc nd = *a.net;
  const int gpad = ((int)G + 3) & ~3;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = tid & (LPR - 1);
  const int rloc = tid / LPR;
  const int lead = lane & ~(LPR - 1);
  const unsigned mask = 0xffffffffu;
  const int N = nd.N, Np = nd.Np;
  const int row0 = cta * R;
  const int row = row0 + rloc;
  const bool live = row < N;
  const long long gi = nd.node_off + row;
  const int bsa = nd.max_delay + 2;
  const float *H = a.H + nd.ring_off;
  float *AR = a.adj_ring + nd.aux_off;

  float *s_lt = reinterpret_cast<float *>(smem);
  float *s_lthh = s_lt + R;
  float *s_lomh = s_lthh + R;
  float *s_go = s_lomh + R;
  float *s_lgp = s_go + R;
  int *sloff = reinterpret_cast<int *>(s_lgp + gpad);
  int *sllen = sloff + nslices;
  uint32_t *s_cd = reinterpret_cast<uint32_t *>(sllen + nslices);
  float *s_lw = reinterpret_cast<float *>(s_cd + a.edge_cap);

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
    s_lw[k] = a.lam_w[ebase + k];
  }
  int deg = 0;
  if (live) {
    if (q == 0) {
      s_lt[rloc] = a.lam_th[gi];
      s_lthh[rloc] = a.lam_thh[gi];
      s_lomh[rloc] = a.lam_omh[gi];
      s_go[rloc] = a.grad_omega[gi];
    }
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }
  const float dt = a.dt;
  const float invN = 1.0f / (float)N;
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  const float decay = 1.0f - dt * lam;
  const int wslice = (warp * (32 / LPR)) / 32;
  const bool slice_live = row0 + wslice * 32 < N;
  float lamg = a.lam_g[0];  // lam_g(s+1) of the next reverse step
  float dgdg_prev = 1.0f;   // dg(s+2)/dg(s+1) of the step reversed before
  if (tid == 0) s_ok = 1;
  __syncthreads();

  // lam_g(s+1) from lam_g(s+2) and the parts of reverse step s+1 (warp 0)
  auto fold_parts = [&](int k) {
    if (warp == 0) {
      const float *src = a.lgp + (k & 1) * gpad;
      for (int c = lane; c < gpad / 4; c += 32) cp_async_cg16(s_lgp + 4 * c, src + 4 * c);
      cp_async_commit();
      cp_async_wait_all();
      __syncwarp();
      float sum = 0.0f;
      for (int c = lane; c < (int)G; c += 32) sum += s_lgp[c];
#pragma unroll
      for (int off = 16; off > 0; off /= 2) sum += __shfl_down_sync(mask, sum, off);
      if (lane == 0) s_lg = lamg * dgdg_prev + sum;
    }
  };

  int k = 0;
  bool ok = true;
  for (; k < a.n_steps; ++k) {
    const long long s = a.seg_start + a.n_steps - 1 - k;
    const int kk = (int)(s - a.seg_start);
    const int hs = kk + nd.max_delay;  // history slot of theta(s)
    const int as_next = pos_mod(s + 1, bsa);
    const int as_s = pos_mod(s, bsa);
    // values of step s that need nothing from the previous reverse step
    const float4 tr = a.trace[kk];
    const float g_s = tr.x, r1 = tr.y;
    float dgdr = 0.0f, dgdg = 1.0f;
    if (nd.ctrl) {
      const float pre = g_s + dt * (nd.beta * (nd.r0 - r1) - nd.mu * (g_s - nd.g_rest));
      const bool free = pre >= nd.g_min && pre <= nd.g_max;
      dgdr = free ? -dt * nd.beta : 0.0f;
      dgdg = free ? 1.0f - dt * nd.mu : 0.0f;
    }
    const float Cm = tr.z * invN, Sm = tr.w * invN;
    float th = 0.0f, eps = 0.0f, diff = 0.0f, sn1 = 0.0f, cs1 = 0.0f, arv = 0.0f;
    float *slot_next = AR + (long long)as_next * Np + row;
    if (live) {
      th = H[(long long)hs * Np + row];
      diff = wrap_pm_pi(th - a.thh_hist[(long long)kk * N + gi]);
      eps = sinf(diff);
      if (q == 0) {
        sincosf(H[(long long)(hs + 1) * Np + row], &sn1, &cs1);
        if (a.early) {
          arv = __ldcg(slot_next);
          __stcg(slot_next, 0.0f);
        }
      }
    }
    // first group of edge loads (nothing in them depends on lam)
    const int len = slice_live ? sllen[wslice] : 0;
    const int base = sloff[wslice] + (rloc & 31);
    const float *w_s = a.w_hist + (long long)kk * a.SL + ebase;
    uint32_t p[U];
    float wv[U], lw[U], dj[U];
    auto load_group = [&](int kb) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = kb + LPR * u + q;
        const bool in = e < deg;
        p[u] = in ? s_cd[base + 32 * e] : 0u;
        wv[u] = in ? __ldg(w_s + base + 32 * e) : 0.0f;
        lw[u] = in ? s_lw[base + 32 * e] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int d = (int)(p[u] & 255u);
        dj[u] = __ldg(H + (long long)(hs - d) * Np + (p[u] >> 8));
      }
    };
    if (len > 0) load_group(0);
    const float dldr = a.dLdr ? a.dLdr[s] : 0.0f;
    // lam_g(s+1): the parts of reverse step s+1, after its barrier
    if (k > 0) {
      if (!(ok = grid_wait(a.bar, (unsigned)k * G, a.err, &s_ok, a.wait))) break;
      fold_parts(k - 1);
      __syncthreads();
      lamg = s_lg;
    }
    dgdg_prev = dgdg;
    const float lam_r = dldr + lamg * dgdr;
    float lt1 = 0.0f;
    if (live && q == 0) {
      // (A) adjoint of theta(s+1), complete; (B) integrate
      if (!a.early) {
        arv = __ldcg(slot_next);
        __stcg(slot_next, 0.0f);
      }
      lt1 = s_lt[rloc] + arv;
      if (r1 > 0.0f) lt1 += lam_r * (Sm * cs1 - Cm * sn1) * invN / r1;
      if (a.dLdth) lt1 += a.dLdth[s * N + gi];
      s_go[rloc] += lt1 * dt;
      if (a.grad_drive) a.grad_drive[s * N + gi] = lt1 * dt;
      if (a.grad_win) a.grad_win[gi] += lt1 * dt * a.xin[s];
    }
    lt1 = __shfl_sync(mask, lt1, lead);
    const float lam_S = lt1 * dt * g_s;
    const float ae = fabsf(eps);
    float S_i = 0.0f, lsum = 0.0f, labs = 0.0f;
    for (int kb = 0; kb < len; kb += LPR * U) {
      if (kb > 0) load_group(kb);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = kb + LPR * u + q;
        if (e < deg) {
          const int j = (int)(p[u] >> 8), d = (int)(p[u] & 255u);
          const float delayed_j = dj[u];
          float dlt = delayed_j - th;
          dlt = wrap_pm_pi(dlt);
          const float w = wv[u];
          float sn, cs;
          lev_sincos<MATH>(dlt, &sn, &cs);
          S_i += w * sn;
          const float w_pre = w + dt * (eta * cs * (1.0f - gamma * ae) - lam * w);
          const float c = (w_pre >= w_min && w_pre <= w_max) ? 1.0f : 0.0f;
          const float lwn = lw[u];
          s_lw[base + 32 * e] = lwn * c * decay + lam_S * sn;
          const float lD = lam_S * w * cs - lwn * c * dt * eta * sn * (1.0f - gamma * ae);
          labs -= lwn * c * dt * eta * gamma * cs;
          const int slot = (as_s - d < 0) ? as_s - d + bsa : as_s - d;
          atomicAdd(AR + (long long)slot * Np + j, lD);
          lsum -= lD;
        }
      }
    }
#pragma unroll
    for (int off = 1; off < LPR; off *= 2) {
      S_i += __shfl_xor_sync(mask, S_i, off);
      lsum += __shfl_xor_sync(mask, lsum, off);
      labs += __shfl_xor_sync(mask, labs, off);
    }
    float lg_part = 0.0f;
    if (live && q == 0) {
      // (D) predictor
      const float sgn = (eps > 0.0f) ? 1.0f : ((eps < 0.0f) ? -1.0f : 0.0f);
      const float lthh1 = s_lthh[rloc], lomh1 = s_lomh[rloc];
      const float leps = -lt1 * dt * nd.alpha + labs * sgn + lomh1 * nd.kappa_w * dt;
      const float ldiff = leps * cosf(diff);
      s_lt[rloc] = lt1 + lsum + ldiff;
      s_lthh[rloc] = lthh1 - ldiff;
      s_lomh[rloc] = lomh1 + lthh1 * dt;
      lg_part = lt1 * dt * S_i;
    }
    // (E) this CTA's part of sum_i lam_th'_i dt S_i
#pragma unroll
    for (int off = 16; off > 0; off /= 2) lg_part += __shfl_down_sync(mask, lg_part, off);
    if (lane == 0) s_red[warp] = lg_part;
    __syncthreads();
    if (warp == 0) {
      lg_part = (lane < (int)(blockDim.x / 32)) ? s_red[lane] : 0.0f;
#pragma unroll
      for (int off = 16; off > 0; off /= 2) lg_part += __shfl_down_sync(mask, lg_part, off);
      if (lane == 0) __stcg(a.lgp + (k & 1) * gpad + cta, lg_part);
    }
    grid_arrive(a.bar);
  }
  if (ok && a.n_steps > 0 && cta == 0) {
    ok = grid_wait(a.bar, (unsigned)a.n_steps * G, a.err, &s_ok, a.wait);
    if (ok) {
      fold_parts(a.n_steps - 1);
      if (tid == 0) a.lam_g[0] = s_lg;
    }
  }
  if (!ok) return;
  if (live && q == 0) {
    a.lam_th[gi] = s_lt[rloc];
    a.lam_thh[gi] = s_lthh[rloc];
    a.lam_omh[gi] = s_lomh[rloc];
    a.grad_omega[gi] = s_go[rloc];
  }
  for (int e = tid; e < nent; e += blockDim.x) a.lam_w[ebase + e] = s_lw[e];
}

template <int MATH, int R, int U>
__global__ void __launch_bounds__(kGridLPR * R, 256 / R)
    adj_grid_fwd_kernel(const AdjGridFwdArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  adj_grid_fwd_body<MATH, R, U>(a, blockIdx.x, gridDim.x, smem);
}

template <int MATH, int R, int U>
__global__ void __launch_bounds__(kGridLPR * R, R == 64 ? 2 : 1)
    adj_grid_bwd_kernel(const AdjGridBwdArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  adj_grid_bwd_body<MATH, R, U>(a, blockIdx.x, gridDim.x, smem);
}

// Paired launch of the backward pass: CTAs [0, gf) recompute segment k-1
// into one record set while CTAs [gf, grid) reverse segment k from the
// other; each group has its own barrier counter and shares the SMs with the
// other, so the two latency-bound step chains overlap.  Every CTA of both
// groups is resident at once (cooperative launch).
template <int MATH, int R, int UF, int UB>
__global__ void __launch_bounds__(kGridLPR * R, 256 / R)
    adj_grid_pair_kernel(const AdjGridFwdArgs f, const AdjGridBwdArgs b, const int gf) {
  extern __shared__ __align__(16) unsigned char smem[];
  if ((int)blockIdx.x < gf)
    adj_grid_fwd_body<MATH, R, UF>(f, blockIdx.x, gf, smem);
  else
    adj_grid_bwd_body<MATH, R, UB>(b, blockIdx.x - gf, gridDim.x - gf, smem);
}

}  // namespace lev
