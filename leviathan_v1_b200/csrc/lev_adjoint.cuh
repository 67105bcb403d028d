// lev_adjoint.cuh -- reverse-mode (adjoint) differentiation of the engine
// step through T steps.  Included once, from lev_engine.cu.
//
// No counterpart in the reference (it has no training path).  The model is
// the reference step (leviathan_kernel.cu:93-264, controller :431-435) with an
// optional additive drive u_i(t) in d theta_i / dt.  The differentiable run
// starts from the engine's (theta, theta_hat) captured at creation, with
// omega_hat(0) = omega (leviathan_kernel.cu:350), every ring slot = theta(0),
// weights w(0) and gain g(0) = K given as inputs; it returns r(t) for
// t = 1..T (and optionally theta(t)).  Backward, given dL/dr(t) (and
// optionally dL/dtheta(t)), returns dL/domega, dL/dw(0), dL/dK and dL/du(t).
//
// Storage: the forward pass checkpoints, every C steps, theta, theta_hat,
// omega_hat, weights, g and the last max_delay+1 ring slots.  Backward walks
// the segments in reverse: it restores a checkpoint, recomputes the
// segment forward (same kernel, bitwise the same trajectory) recording the
// pre-step weights, theta_hat and per-step (g, r, sum cos, sum sin) -- the
// phases themselves stay in an extended ring of C + max_delay + 2 slots --
// and then runs one reverse kernel per step.
//
// Reverse step s (state s -> s+1), per node i (one lane per row, SELL-32):
//   lam_r      = dL/dr(s+1) + lam_g(s+1) * dg(s+1)/dr(s+1)
//   lam_th'    = lam_th_cur + adj_ring[s+1] + lam_r * dr/dtheta_i + dL/dtheta_i(s+1)
//   lam_S      = lam_th' dt g(s);  dL/domega_i += lam_th' dt;  dL/du_i(s) = lam_th' dt
//   per edge e = (i <- j, d), Delta = wrap(theta_j(s-d) - theta_i(s)):
//     c        = 1 if the updated weight was not clamped, else 0
//     lam_w(s) = c (1 - dt lam) lam_w(s+1) + lam_S sin Delta
//     lam_D    = lam_S w cos Delta - c dt eta sin Delta (1 - gamma|eps_i|) lam_w(s+1)
//     adj_ring[s-d][j] += lam_D  (scatter, red.add);  lam_th(s) -= lam_D
//   prep: lam_eps -> lam_diff = lam_eps cos(diff);  lam_th(s) += lam_diff;
//     lam_thh(s) = lam_thh(s+1) - lam_diff;  lam_omh(s) = lam_omh(s+1) + dt lam_thh(s+1)
//   lam_g(s)   = lam_g(s+1) dg(s+1)/dg(s) + sum_i lam_th'_i dt S_i
// The wraps have derivative 1; a clamped weight or gain passes nothing;
// |eps| has derivative sign(eps).  The adjoint ring has max_delay+2 slots so
// the slot finalised at the start of a launch is never one scattered into by
// the same launch (reads of time s+1, writes of times s-max_delay..s).

namespace lev {

struct AdjFwdArgs {
  const NetDesc *nets;  // adjoint copies: bsi = C + max_delay + 2
  NetState *st;
  const int2 *tiles;
  const int *row_ptr;
  const long long *sl_off;
  const int *sl_len;
  const uint32_t *sl_cd;
  const float *w_in;  // SELL weights before the step
  float *w_out;       // after the step (may alias w_in)
  float *theta;
  float *theta_hat;
  const float *omega;
  float *omega_hat;
  float *ring;
  float2 *partials;
  const float *drive;  // [total nodes] for this step, or null
  float *thh_rec;      // theta_hat before the step [total nodes], or null
  float *dj_rec;       // the delayed source phase of every edge this step
                       // (SELL order, entries below the row's degree), or null
  float4 *trace;       // per network (g used, r, sum cos, sum sin), or null
  float *r_out;        // per network r after the step, or null
  float *theta_out;    // theta after the step [total nodes], or null
  // reservoir: drive u_i = win_i * xin[network]; readout
  // y[network] = sum_i ra_i cos theta_i + rb_i sin theta_i (after the step)
  const float *win;    // [total nodes] or null
  const float *xin;    // [num_nets] input of this step
  const float *ra;     // [total nodes] or null
  const float *rb;
  float *ro_partials;  // per tile
  float *y_out;        // per network, or null
  float dt;
};

// Forward step with recording hooks.  Same arithmetic as step_kernel (and
// bitwise the same results when drive is null).  Five CTAs per SM with four
// entries in flight per lane: measured on the batch-64 reservoir (64 × 10⁶
// edges) 0.415 s per 1,000 forward steps, against 0.446 s at three CTAs per
// SM with eight entries, 0.423 s at four with six or eight.
template <int MATH>
__global__ void __launch_bounds__(kTile, 5) adj_fwd_kernel(const AdjFwdArgs a) {
  __shared__ float s_rc[32];
  __shared__ float s_rs[32];
  __shared__ float s_ry[32];
  __shared__ int s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int2 tile = a.tiles[blockIdx.x];
  const NetDesc nd = a.nets[tile.x];
  NetState *ns = a.st + tile.x;
  const int N = nd.N, row0 = tile.y, row = row0 + tid;
  const bool live = row < N;
  const long long gi = nd.node_off + row;
  const float dt = a.dt;
  const int bsi = nd.bsi, Np = nd.Np, cur = ns->cur;
  const float g = ns->g;
  const float *ring = a.ring + nd.ring_off;

  float th = 0.0f, eps = 0.0f;
  int deg = 0;
  if (live) {
    th = a.theta[gi];
    const float thh = a.theta_hat[gi];
    const float wh = a.omega_hat[gi];
    if (a.thh_rec) a.thh_rec[gi] = thh;
    float diff = th - thh;
    diff = wrap_pm_pi(diff);
    eps = sinf(diff);
    a.theta_hat[gi] = thh + dt * wh;
    a.omega_hat[gi] = wh + nd.kappa_w * dt * eps;
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }
  const float my_eps = fabsf(eps);
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  float local_sum = 0.0f;
  const int slice_row0 = row0 + 32 * warp;
  if (slice_row0 < N) {
    const long long s = nd.slice_base + (slice_row0 >> 5);
    const int len = a.sl_len[s];
    const long long base = a.sl_off[s] + lane;
    // software-pipelined like step_kernel: the stream loads of group k0+U
    // are in flight while group k0 gathers and computes
    constexpr int U = 4;
    uint32_t p[U];
    float wv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool in = u < len;
      p[u] = in ? __ldg(a.sl_cd + base + 32 * u) : 0u;
      wv[u] = in ? a.w_in[base + 32 * u] : 0.0f;
    }
    for (int k0 = 0; k0 < len; k0 += U) {
      float dj[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int slot = cur - (int)(p[u] & 255u);
        slot += (slot < 0) ? bsi : 0;
        dj[u] = ld_ring(ring + ((unsigned)slot * (unsigned)Np + (p[u] >> 8)));
      }
      uint32_t pn[U];
      float wn[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool in = k0 + U + u < len;
        pn[u] = in ? __ldg(a.sl_cd + base + 32 * (k0 + U + u)) : 0u;
        wn[u] = in ? a.w_in[base + 32 * (k0 + U + u)] : 0.0f;
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
          a.w_out[base + 32 * (k0 + u)] = w;
          if (a.dj_rec) a.dj_rec[base + 32 * (k0 + u)] = delayed_j;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        p[u] = pn[u];
        wv[u] = wn[u];
      }
    }
  }

  int nxt = cur + 1;
  if (nxt == bsi) nxt = 0;
  float my_cos = 0.0f, my_sin = 0.0f, my_y = 0.0f;
  if (live) {
    float inc;
    if (a.drive || a.win) {
      float u = 0.0f;
      if (a.drive) u += a.drive[gi];
      if (a.win) u += a.win[gi] * a.xin[tile.x];
      inc = dt * (a.omega[gi] + g * local_sum - nd.alpha * eps + u);
    } else {
      inc = dt * (a.omega[gi] + g * local_sum - nd.alpha * eps);
    }
    float x = th + inc;
    x = wrap_0_2pi(x);
    if (!isfinite(x)) x = 0.0f;
    a.theta[gi] = x;
    if (a.theta_out) a.theta_out[gi] = x;
    a.ring[nd.ring_off + (long long)nxt * Np + row] = x;
    lev_sincos<MATH>(x, &my_sin, &my_cos);
    if (a.ra) my_y = a.ra[gi] * my_cos + a.rb[gi] * my_sin;
  }
  const unsigned mask = 0xffffffffu;
#pragma unroll
  for (int off = 16; off > 0; off /= 2) {
    my_cos += __shfl_down_sync(mask, my_cos, off);
    my_sin += __shfl_down_sync(mask, my_sin, off);
    my_y += __shfl_down_sync(mask, my_y, off);
  }
  if (lane == 0) {
    s_rc[warp] = my_cos;
    s_rs[warp] = my_sin;
    s_ry[warp] = my_y;
  }
  __syncthreads();
  if (warp == 0) {
    my_cos = (lane < (kTile / 32)) ? s_rc[lane] : 0.0f;
    my_sin = (lane < (kTile / 32)) ? s_rs[lane] : 0.0f;
    my_y = (lane < (kTile / 32)) ? s_ry[lane] : 0.0f;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      my_cos += __shfl_down_sync(mask, my_cos, off);
      my_sin += __shfl_down_sync(mask, my_sin, off);
      my_y += __shfl_down_sync(mask, my_y, off);
    }
    if (lane == 0) {
      a.partials[nd.part_off + row0 / kTile] = make_float2(my_cos, my_sin);
      if (a.ra) a.ro_partials[nd.part_off + row0 / kTile] = my_y;
      __threadfence();
      const unsigned prev = atomicAdd(&ns->ticket, 1u);
      s_last = (prev == (unsigned)(nd.ntiles - 1));
    }
  }
  __syncthreads();
  if (!s_last) return;
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
      if (a.trace) a.trace[tile.x] = make_float4(g, r, sum_cos, sum_sin);
      if (a.r_out) a.r_out[tile.x] = r;
      if (a.ra && a.y_out) {
        float y = 0.0f;
        for (int k = 0; k < nd.ntiles; ++k) y += __ldcg(a.ro_partials + nd.part_off + k);
        a.y_out[tile.x] = y;
      }
      ns->g = gn;
      ns->r = r;
      ns->cur = nxt;
      ns->t = ns->t + 1;
      ns->ticket = 0u;
    }
  }
}

// The forward step with four lanes per row, for grids under one wave
// (N ~ 10^4: 40 tiles on 148 SMs).  CTA = one 256-row tile, 1024 threads,
// lanes 4r .. 4r+3 of the CTA on row r.  The row's first lane runs the node
// work and forms the coupling sum in CSR order from the per-edge terms its
// three partner lanes and it computed (shuffled), with the same expression;
// the block trees read the rows' values from shared memory in row order.  So
// the results are bitwise those of adj_fwd_kernel (and of step_kernel).
template <int MATH, int U>
__global__ void __launch_bounds__(4 * kTile, 1) adj_fwd_split_kernel(const AdjFwdArgs a) {
  constexpr int LPR = 4;
  __shared__ float s_rc[32];
  __shared__ float s_rs[32];
  __shared__ float s_ry[32];
  __shared__ float s_val[3][kTile];
  __shared__ int s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = tid & (LPR - 1);
  const int rloc = tid / LPR;  // row within the tile
  const int lead = lane & ~(LPR - 1);
  const unsigned mask = 0xffffffffu;
  const int2 tile = a.tiles[blockIdx.x];
  const NetDesc nd = a.nets[tile.x];
  NetState *ns = a.st + tile.x;
  const int N = nd.N, row0 = tile.y, row = row0 + rloc;
  const bool live = row < N;
  const long long gi = nd.node_off + row;
  const float dt = a.dt;
  const int bsi = nd.bsi, Np = nd.Np, cur = ns->cur;
  const float g = ns->g;
  const float *ring = a.ring + nd.ring_off;

  // ---- predictor (row's first lane) ----------------------------------------
  float th = 0.0f, eps = 0.0f;
  int deg = 0;
  if (live) {
    if (q == 0) {
      th = a.theta[gi];
      const float thh = a.theta_hat[gi];
      const float wh = a.omega_hat[gi];
      if (a.thh_rec) a.thh_rec[gi] = thh;
      float diff = th - thh;
      diff = wrap_pm_pi(diff);
      eps = sinf(diff);
      a.theta_hat[gi] = thh + dt * wh;
      a.omega_hat[gi] = wh + nd.kappa_w * dt * eps;
    }
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }
  th = __shfl_sync(mask, th, lead);
  eps = __shfl_sync(mask, eps, lead);
  const float my_eps = fabsf(eps);
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;

  // ---- edges: lane q takes entries q, q+4, ...; the sum in CSR order -------
  float local_sum = 0.0f;
  const int wrow0 = row0 + warp * (32 / LPR);  // the warp's 8 rows share a slice
  if (wrow0 < N) {
    const long long s = nd.slice_base + (wrow0 >> 5);
    const int len = a.sl_len[s];
    const long long base = a.sl_off[s] + (row & 31);
    for (int kb = 0; kb < len; kb += LPR * U) {
      uint32_t p[U];
      float wv[U], dj[U], sn[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = kb + LPR * u + q;
        const bool in = k < len;
        p[u] = in ? __ldg(a.sl_cd + base + 32 * k) : 0u;
        wv[u] = in ? a.w_in[base + 32 * k] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int slot = cur - (int)(p[u] & 255u);
        slot += (slot < 0) ? bsi : 0;
        dj[u] = ld_ring(ring + ((unsigned)slot * (unsigned)Np + (p[u] >> 8)));
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
          a.w_out[base + 32 * k] = w;
        }
      }
#pragma unroll
      for (int e = 0; e < LPR * U; ++e) {
        const int src = lead + (e % LPR);
        const float w = __shfl_sync(mask, wv[e / LPR], src);
        const float sin_diff = __shfl_sync(mask, sn[e / LPR], src);
        if (kb + e < deg) local_sum += w * sin_diff;  // the expression of adj_fwd_kernel
      }
    }
  }

  // ---- integrate (row's first lane) ----------------------------------------
  int nxt = cur + 1;
  if (nxt == bsi) nxt = 0;
  if (q == 0) {
    float my_cos = 0.0f, my_sin = 0.0f, my_y = 0.0f;
    if (live) {
      float inc;
      if (a.drive || a.win) {
        float u = 0.0f;
        if (a.drive) u += a.drive[gi];
        if (a.win) u += a.win[gi] * a.xin[tile.x];
        inc = dt * (a.omega[gi] + g * local_sum - nd.alpha * eps + u);
      } else {
        inc = dt * (a.omega[gi] + g * local_sum - nd.alpha * eps);
      }
      float x = th + inc;
      x = wrap_0_2pi(x);
      if (!isfinite(x)) x = 0.0f;
      a.theta[gi] = x;
      if (a.theta_out) a.theta_out[gi] = x;
      a.ring[nd.ring_off + (long long)nxt * Np + row] = x;
      lev_sincos<MATH>(x, &my_sin, &my_cos);
      if (a.ra) my_y = a.ra[gi] * my_cos + a.rb[gi] * my_sin;
    }
    s_val[0][rloc] = my_cos;
    s_val[1][rloc] = my_sin;
    s_val[2][rloc] = my_y;
  }
  __syncthreads();

  // ---- block partials in row order (leviathan_kernel.cu:198-233) -----------
  if (tid < kTile) {
    float my_cos = s_val[0][tid], my_sin = s_val[1][tid], my_y = s_val[2][tid];
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      my_cos += __shfl_down_sync(mask, my_cos, off);
      my_sin += __shfl_down_sync(mask, my_sin, off);
      my_y += __shfl_down_sync(mask, my_y, off);
    }
    if (lane == 0) {
      s_rc[warp] = my_cos;
      s_rs[warp] = my_sin;
      s_ry[warp] = my_y;
    }
  }
  __syncthreads();
  if (warp == 0) {
    float my_cos = (lane < (kTile / 32)) ? s_rc[lane] : 0.0f;
    float my_sin = (lane < (kTile / 32)) ? s_rs[lane] : 0.0f;
    float my_y = (lane < (kTile / 32)) ? s_ry[lane] : 0.0f;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      my_cos += __shfl_down_sync(mask, my_cos, off);
      my_sin += __shfl_down_sync(mask, my_sin, off);
      my_y += __shfl_down_sync(mask, my_y, off);
    }
    if (lane == 0) {
      a.partials[nd.part_off + row0 / kTile] = make_float2(my_cos, my_sin);
      if (a.ra) a.ro_partials[nd.part_off + row0 / kTile] = my_y;
      __threadfence();
      const unsigned prev = atomicAdd(&ns->ticket, 1u);
      s_last = (prev == (unsigned)(nd.ntiles - 1));
    }
  }
  __syncthreads();
  if (!s_last) return;
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
      if (a.trace) a.trace[tile.x] = make_float4(g, r, sum_cos, sum_sin);
      if (a.r_out) a.r_out[tile.x] = r;
      if (a.ra && a.y_out) {
        float y = 0.0f;
        for (int k = 0; k < nd.ntiles; ++k) y += __ldcg(a.ro_partials + nd.part_off + k);
        a.y_out[tile.x] = y;
      }
      ns->g = gn;
      ns->r = r;
      ns->cur = nxt;
      ns->t = ns->t + 1;
      ns->ticket = 0u;
    }
  }
}

struct AdjBwdArgs {
  const NetDesc *nets;  // adjoint copies (ring_off: history ring, aux_off: adjoint ring)
  const int2 *tiles;
  const int *row_ptr;
  const long long *sl_off;
  const int *sl_len;
  const uint32_t *sl_cd;
  const float *w_s;    // SELL weights before step s
  const float *dj_s;   // delayed source phases of step s (SELL), or null: from H
  const float *H;      // history ring: theta(tau) at slot tau - seg_start + max_delay
  const float *thh_s;  // theta_hat before step s [total nodes]
  const float4 *trace; // per network (g_s, r_{s+1}, sum cos, sum sin)
  const float *dLdr;   // per network dL/dr(s+1), or null
  const float *dLdth;  // [total nodes] dL/dtheta(s+1), or null
  float *lam_th;       // current-phase adjoint: in time s+1, out time s
  float *lam_thh;
  float *lam_omh;
  float *lam_w;        // SELL
  float *adj_ring;
  float *lam_g;        // per network: in lam_g(s+1), out lam_g(s)
  float *grad_omega;   // accumulated
  float *grad_drive;   // [total nodes] for step s, or null
  float2 *partials;    // per tile (lam_g partial, unused)
  unsigned *tickets;   // per network
  // reservoir terms (see AdjFwdArgs); all may be null
  const float *win;
  const float *xin;    // [num_nets] input of step s
  float *grad_win;     // accumulated
  const float *ra;
  const float *rb;
  const float *dLdy;   // [num_nets] dL/dy(s+1)
  float *grad_ra;      // accumulated
  float *grad_rb;
  long long s;         // step being reversed (absolute)
  long long seg_start;
  float dt;
};

__device__ __forceinline__ int pos_mod(long long x, int m) {
  int r = (int)(x % m);
  return r < 0 ? r + m : r;
}

// U: edges per lane whose loads are in flight together; MINB: resident CTAs
// per SM the register budget is sized for.
template <int MATH, int U, int MINB>
__global__ void __launch_bounds__(kTile, MINB) adj_bwd_kernel(const AdjBwdArgs a) {
  __shared__ float s_red[32];
  __shared__ int s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int2 tile = a.tiles[blockIdx.x];
  const NetDesc nd = a.nets[tile.x];
  const int N = nd.N, row0 = tile.y, row = row0 + tid;
  const bool live = row < N;
  const long long gi = nd.node_off + row;
  const float dt = a.dt;
  const int Np = nd.Np;
  const int bsa = nd.max_delay + 2;
  const int hs = (int)(a.s - a.seg_start) + nd.max_delay;  // history slot of theta(s)
  const float *H = a.H + nd.ring_off;
  float *AR = a.adj_ring + nd.aux_off;
  const int as_next = pos_mod(a.s + 1, bsa);
  const int as_s = pos_mod(a.s, bsa);

  // controller derivatives at step s -> s+1
  const float4 tr = a.trace[tile.x];
  const float g_s = tr.x, r1 = tr.y;
  float dgdr = 0.0f, dgdg = 1.0f;
  if (nd.ctrl) {
    const float pre = g_s + dt * (nd.beta * (nd.r0 - r1) - nd.mu * (g_s - nd.g_rest));
    const bool free = pre >= nd.g_min && pre <= nd.g_max;
    dgdr = free ? -dt * nd.beta : 0.0f;
    dgdg = free ? 1.0f - dt * nd.mu : 0.0f;
  }
  const float lam_g1 = a.lam_g[tile.x];
  const float lam_r = (a.dLdr ? a.dLdr[tile.x] : 0.0f) + lam_g1 * dgdr;
  const float invN = 1.0f / (float)N;
  const float Cm = tr.z * invN, Sm = tr.w * invN;

  float lg_part = 0.0f;
  float lt1 = 0.0f, th = 0.0f, eps = 0.0f, diff = 0.0f, lam_S = 0.0f;
  int deg = 0;
  if (live) {
    // (A) adjoint of theta(s+1), complete
    const float th1 = H[(long long)(hs + 1) * Np + row];
    float* slot_next = AR + (long long)as_next * Np + row;
    lt1 = a.lam_th[gi] + *slot_next;
    *slot_next = 0.0f;
    float sn, cs;
    sincosf(th1, &sn, &cs);
    if (r1 > 0.0f) lt1 += lam_r * (Sm * cs - Cm * sn) * invN / r1;
    if (a.dLdth) lt1 += a.dLdth[gi];
    if (a.dLdy) {  // readout y = sum ra cos theta + rb sin theta
      const float gy = a.dLdy[tile.x];
      lt1 += gy * (a.rb[gi] * cs - a.ra[gi] * sn);
      a.grad_ra[gi] += gy * cs;
      a.grad_rb[gi] += gy * sn;
    }
    // (B) integrate
    lam_S = lt1 * dt * g_s;
    a.grad_omega[gi] += lt1 * dt;
    if (a.grad_drive) a.grad_drive[gi] = lt1 * dt;
    if (a.grad_win) a.grad_win[gi] += lt1 * dt * a.xin[tile.x];
    // prep recompute
    th = H[(long long)hs * Np + row];
    diff = wrap_pm_pi(th - a.thh_s[gi]);
    eps = sinf(diff);
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
  }
  const float ae = fabsf(eps);
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  const float decay = 1.0f - dt * lam;
  float S_i = 0.0f, lth = lt1, labs = 0.0f;
  const int slice_row0 = row0 + 32 * warp;
  if (slice_row0 < N) {
    const long long s = nd.slice_base + (slice_row0 >> 5);
    const int len = a.sl_len[s];
    const long long base = a.sl_off[s] + lane;
    // all U entries' stream loads, then all gathers, before the dependent
    // math (measured faster here than a software pipeline of the groups).
    // With dj_s the delayed phases the recompute recorded are one more
    // stream, so a group waits on memory once instead of twice.
    for (int k0 = 0; k0 < len; k0 += U) {
      uint32_t p[U];
      float wv[U], lw[U], dj[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool in = k0 + u < deg;
        p[u] = in ? __ldg(a.sl_cd + base + 32 * (k0 + u)) : 0u;
        wv[u] = in ? a.w_s[base + 32 * (k0 + u)] : 0.0f;
        lw[u] = in ? a.lam_w[base + 32 * (k0 + u)] : 0.0f;
        if (a.dj_s) dj[u] = in ? __ldcs(a.dj_s + base + 32 * (k0 + u)) : 0.0f;
      }
      if (!a.dj_s) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int d = (int)(p[u] & 255u);
          dj[u] = H[(long long)(hs - d) * Np + (p[u] >> 8)];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (k0 + u < deg) {
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
          a.lam_w[base + 32 * (k0 + u)] = lwn * c * decay + lam_S * sn;
          const float lD = lam_S * w * cs - lwn * c * dt * eta * sn * (1.0f - gamma * ae);
          labs -= lwn * c * dt * eta * gamma * cs;
          const int slot = (as_s - d < 0) ? as_s - d + bsa : as_s - d;
          atomicAdd(AR + (long long)slot * Np + j, lD);
          lth -= lD;
        }
      }
    }
  }
  if (live) {
    // (D) predictor
    const float sgn = (eps > 0.0f) ? 1.0f : ((eps < 0.0f) ? -1.0f : 0.0f);
    const float lthh1 = a.lam_thh[gi], lomh1 = a.lam_omh[gi];
    const float leps = -lt1 * dt * nd.alpha + labs * sgn + lomh1 * nd.kappa_w * dt;
    const float ldiff = leps * cosf(diff);
    lth += ldiff;
    a.lam_th[gi] = lth;
    a.lam_thh[gi] = lthh1 - ldiff;
    a.lam_omh[gi] = lomh1 + lthh1 * dt;
    lg_part = lt1 * dt * S_i;
  }
  // (E) lam_g(s) = lam_g(s+1) dg/dg + sum_i lam_th'_i dt S_i
  const unsigned mask = 0xffffffffu;
#pragma unroll
  for (int off = 16; off > 0; off /= 2) lg_part += __shfl_down_sync(mask, lg_part, off);
  if (lane == 0) s_red[warp] = lg_part;
  __syncthreads();
  if (warp == 0) {
    lg_part = (lane < kTile / 32) ? s_red[lane] : 0.0f;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) lg_part += __shfl_down_sync(mask, lg_part, off);
    if (lane == 0) {
      a.partials[nd.part_off + row0 / kTile] = make_float2(lg_part, 0.0f);
      __threadfence();
      const unsigned prev = atomicAdd(a.tickets + tile.x, 1u);
      s_last = (prev == (unsigned)(nd.ntiles - 1));
    }
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (warp == 0) {
    float sum = 0.0f;
    const float2 *part = a.partials + nd.part_off;
    for (int k = lane; k < nd.ntiles; k += 32) sum += __ldcg(part + k).x;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) sum += __shfl_down_sync(mask, sum, off);
    if (lane == 0) {
      a.lam_g[tile.x] = lam_g1 * dgdg + sum;
      a.tickets[tile.x] = 0u;
    }
  }
}

// The reverse step with LPR lanes per row, for grids that leave most SMs idle
// with one lane per row (N ~ 10^4: 40 CTAs on 148 SMs).  Each 256-row tile is
// taken by LPR CTAs of 256/LPR rows; lane q of a row walks the row's SELL
// entries q, q + LPR, ...; the row's sums (coupling sum S_i, the lam_D sum, the
// |eps| term) are combined by shuffles and the node-level work is done by the
// row's first lane.  The per-edge arithmetic is that of adj_bwd_kernel; only
// the order of the sums over a row's edges differs (the gradients agree to
// rounding).  Partials: LPR per tile.
template <int MATH, int LPR, int U>
__global__ void __launch_bounds__(kTile, 4) adj_bwd_split_kernel(const AdjBwdArgs a) {
  constexpr int RPC = kTile / LPR;  // rows per CTA
  __shared__ float s_red[32];
  __shared__ int s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int sub = blockIdx.x % LPR;
  const int2 tile = a.tiles[blockIdx.x / LPR];
  const NetDesc nd = a.nets[tile.x];
  const int q = tid % LPR;
  const int N = nd.N, row0 = tile.y, row = row0 + sub * RPC + tid / LPR;
  const bool live = row < N;
  const long long gi = nd.node_off + row;
  const float dt = a.dt;
  const int Np = nd.Np;
  const int bsa = nd.max_delay + 2;
  const int hs = (int)(a.s - a.seg_start) + nd.max_delay;  // history slot of theta(s)
  const float *H = a.H + nd.ring_off;
  float *AR = a.adj_ring + nd.aux_off;
  const int as_next = pos_mod(a.s + 1, bsa);
  const int as_s = pos_mod(a.s, bsa);
  const unsigned mask = 0xffffffffu;

  const float4 tr = a.trace[tile.x];
  const float g_s = tr.x, r1 = tr.y;
  float dgdr = 0.0f, dgdg = 1.0f;
  if (nd.ctrl) {
    const float pre = g_s + dt * (nd.beta * (nd.r0 - r1) - nd.mu * (g_s - nd.g_rest));
    const bool free = pre >= nd.g_min && pre <= nd.g_max;
    dgdr = free ? -dt * nd.beta : 0.0f;
    dgdg = free ? 1.0f - dt * nd.mu : 0.0f;
  }
  const float lam_g1 = a.lam_g[tile.x];
  const float lam_r = (a.dLdr ? a.dLdr[tile.x] : 0.0f) + lam_g1 * dgdr;
  const float invN = 1.0f / (float)N;
  const float Cm = tr.z * invN, Sm = tr.w * invN;

  float lg_part = 0.0f;
  float lt1 = 0.0f, th = 0.0f, eps = 0.0f, diff = 0.0f;
  int deg = 0;
  if (live) {
    th = H[(long long)hs * Np + row];
    diff = wrap_pm_pi(th - a.thh_s[gi]);
    eps = sinf(diff);
    const int *rp = a.row_ptr + nd.rp_off + row;
    deg = rp[1] - rp[0];
    if (q == 0) {
      // (A) adjoint of theta(s+1), complete; (B) integrate
      const float th1 = H[(long long)(hs + 1) * Np + row];
      float *slot_next = AR + (long long)as_next * Np + row;
      lt1 = a.lam_th[gi] + *slot_next;
      *slot_next = 0.0f;
      float sn, cs;
      sincosf(th1, &sn, &cs);
      if (r1 > 0.0f) lt1 += lam_r * (Sm * cs - Cm * sn) * invN / r1;
      if (a.dLdth) lt1 += a.dLdth[gi];
      if (a.dLdy) {
        const float gy = a.dLdy[tile.x];
        lt1 += gy * (a.rb[gi] * cs - a.ra[gi] * sn);
        a.grad_ra[gi] += gy * cs;
        a.grad_rb[gi] += gy * sn;
      }
      a.grad_omega[gi] += lt1 * dt;
      if (a.grad_drive) a.grad_drive[gi] = lt1 * dt;
      if (a.grad_win) a.grad_win[gi] += lt1 * dt * a.xin[tile.x];
    }
  }
  lt1 = __shfl_sync(mask, lt1, lane & ~(LPR - 1));  // from the row's first lane
  const float lam_S = lt1 * dt * g_s;
  const float ae = fabsf(eps);
  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  const float decay = 1.0f - dt * lam;
  float S_i = 0.0f, lsum = 0.0f, labs = 0.0f;
  // the warp's rows lie in one 32-row SELL slice (32 / LPR consecutive rows)
  const int wrow0 = row0 + sub * RPC + warp * (32 / LPR);
  if (wrow0 < N) {
    const long long s = nd.slice_base + (wrow0 >> 5);
    const int len = a.sl_len[s];
    const long long base = a.sl_off[s] + (row & 31);
    for (int kb = 0; kb < len; kb += LPR * U) {
      uint32_t p[U];
      float wv[U], lw[U], dj[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = kb + LPR * u + q;
        const bool in = k < deg;
        p[u] = in ? __ldg(a.sl_cd + base + 32 * k) : 0u;
        wv[u] = in ? a.w_s[base + 32 * k] : 0.0f;
        lw[u] = in ? a.lam_w[base + 32 * k] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int d = (int)(p[u] & 255u);
        dj[u] = H[(long long)(hs - d) * Np + (p[u] >> 8)];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = kb + LPR * u + q;
        if (k < deg) {
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
          a.lam_w[base + 32 * k] = lwn * c * decay + lam_S * sn;
          const float lD = lam_S * w * cs - lwn * c * dt * eta * sn * (1.0f - gamma * ae);
          labs -= lwn * c * dt * eta * gamma * cs;
          const int slot = (as_s - d < 0) ? as_s - d + bsa : as_s - d;
          atomicAdd(AR + (long long)slot * Np + j, lD);
          lsum -= lD;
        }
      }
    }
  }
#pragma unroll
  for (int off = 1; off < LPR; off *= 2) {
    S_i += __shfl_xor_sync(mask, S_i, off);
    lsum += __shfl_xor_sync(mask, lsum, off);
    labs += __shfl_xor_sync(mask, labs, off);
  }
  if (live && q == 0) {
    // (D) predictor
    const float sgn = (eps > 0.0f) ? 1.0f : ((eps < 0.0f) ? -1.0f : 0.0f);
    const float lthh1 = a.lam_thh[gi], lomh1 = a.lam_omh[gi];
    const float leps = -lt1 * dt * nd.alpha + labs * sgn + lomh1 * nd.kappa_w * dt;
    const float ldiff = leps * cosf(diff);
    a.lam_th[gi] = lt1 + lsum + ldiff;
    a.lam_thh[gi] = lthh1 - ldiff;
    a.lam_omh[gi] = lomh1 + lthh1 * dt;
    lg_part = lt1 * dt * S_i;
  }
  // (E) lam_g(s) = lam_g(s+1) dg/dg + sum_i lam_th'_i dt S_i
#pragma unroll
  for (int off = 16; off > 0; off /= 2) lg_part += __shfl_down_sync(mask, lg_part, off);
  if (lane == 0) s_red[warp] = lg_part;
  __syncthreads();
  const int nparts = nd.ntiles * LPR;
  if (warp == 0) {
    lg_part = (lane < kTile / 32) ? s_red[lane] : 0.0f;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) lg_part += __shfl_down_sync(mask, lg_part, off);
    if (lane == 0) {
      a.partials[(long long)nd.part_off * LPR + (row0 / kTile) * LPR + sub] =
          make_float2(lg_part, 0.0f);
      __threadfence();
      const unsigned prev = atomicAdd(a.tickets + tile.x, 1u);
      s_last = (prev == (unsigned)(nparts - 1));
    }
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (warp == 0) {
    float sum = 0.0f;
    const float2 *part = a.partials + (long long)nd.part_off * LPR;
    for (int k = lane; k < nparts; k += 32) sum += __ldcg(part + k).x;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) sum += __shfl_down_sync(mask, sum, off);
    if (lane == 0) {
      a.lam_g[tile.x] = lam_g1 * dgdg + sum;
      a.tickets[tile.x] = 0u;
    }
  }
}

// Checkpoint of the ring window of every network: mode 0 saves theta(t-m),
// m = 0..max_delay, from the ring (slot (cur - m) mod bsi) into
// ck[m][N] (per network at ck_off); mode 1 writes it back as
// theta(t-m) -> slot max_delay - m of an unwrapped segment ring.
__global__ void adj_ring_ckpt_kernel(int mode, const NetDesc *nets,
                                     const NetState *st, float *ring,
                                     float *ck, const long long *ck_off,
                                     int num_nets) {
  const int n = blockIdx.y;
  if (n >= num_nets) return;
  const NetDesc nd = nets[n];
  const int bs = nd.max_delay + 1;
  const long long total = (long long)bs * nd.N;
  const int cur = st[n].cur;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(k / nd.N);
    const int i = (int)(k - (long long)m * nd.N);
    float *c = ck + ck_off[n] + k;
    if (mode == 0) {
      int slot = cur - m;
      slot += (slot < 0) ? nd.bsi : 0;
      *c = ring[nd.ring_off + (long long)slot * nd.Np + i];
    } else {
      ring[nd.ring_off + (long long)(nd.max_delay - m) * nd.Np + i] = *c;
    }
  }
}

// Final adjoint of theta(0): current part plus every adjoint-ring slot (reads
// of times <= 0 all read theta(0), the value every slot starts with).
__global__ void adj_finalize_kernel(const NetDesc *nets, int num_nets,
                                    const float *lam_th, const float *adj_ring,
                                    float *grad_theta0) {
  const int n = blockIdx.y;
  if (n >= num_nets) return;
  const NetDesc nd = nets[n];
  const int bsa = nd.max_delay + 2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd.N;
       i += gridDim.x * blockDim.x) {
    float v = lam_th[nd.node_off + i];
    for (int s = 0; s < bsa; ++s) v += adj_ring[nd.aux_off + (long long)s * nd.Np + i];
    grad_theta0[nd.node_off + i] = v;
  }
}

__global__ void add_kernel(float *dst, const float *src, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    dst[k] += src[k];
}

}  // namespace lev
