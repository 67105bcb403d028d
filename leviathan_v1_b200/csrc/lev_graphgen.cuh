// lev_graphgen.cuh -- seeded Watts-Strogatz topology and initial state built
// on the device.  Included once, from lev_engine.cu.
//
// The reference builds its topology on the host with networkx and scipy
// (python/leviathan_h100.py:34-45), seconds to minutes at N = 10^6.  Same
// model here: ring lattice of k/2 neighbours per side; each lattice edge
// (u, u+j) is rewired with probability p to (u, w), w uniform, avoiding
// self-loops and multi-edges.  Deterministic for a seed regardless of thread
// timing:
//   * random numbers come from counter-based streams (SplitMix64 finaliser
//     of (seed, stream, counter); G. Steele, D. Lea, C. Flood, OOPSLA 2014);
//   * rewiring proceeds in rounds: every pending edge proposes a target,
//     proposals of the same undirected pair meet in a hash table where the
//     lowest edge index wins (atomicMin), losers and collisions with
//     existing edges propose again in the next round;
//   * the CSR is made canonical (columns sorted per row), so the fill order
//     of the atomics does not matter;
//   * per-edge and per-node initial values are drawn by position.
// The graph is not the one networkx draws for the same seed (different
// random streams); it is the same random-graph model.

namespace lev {

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ unsigned long long rng64(unsigned long long seed,
                                                    unsigned long long stream,
                                                    unsigned long long ctr) {
  return mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) + ctr);
}

// uniform in [0, 1) with 53 random bits
__device__ __forceinline__ double rng_u01(unsigned long long seed,
                                          unsigned long long stream,
                                          unsigned long long ctr) {
  return (double)(rng64(seed, stream, ctr) >> 11) * (1.0 / 9007199254740992.0);
}

// uniform integer in [0, n)
__device__ __forceinline__ unsigned int rng_below(unsigned long long seed,
                                                  unsigned long long stream,
                                                  unsigned long long ctr,
                                                  unsigned int n) {
  return (unsigned int)__umul64hi(rng64(seed, stream, ctr), (unsigned long long)n);
}

struct WsArgs {
  int N, half;
  double p;
  unsigned long long seed;
};

__device__ __forceinline__ bool ws_rewired(const WsArgs &a, long long e) {
  return rng_u01(a.seed, 1, (unsigned long long)e) < a.p;
}

// Is the undirected pair (x, y) a lattice edge that stayed in place?
__device__ __forceinline__ bool ws_kept_lattice(const WsArgs &a, int x, int y) {
  int lo = min(x, y), hi = max(x, y);
  int fwd = hi - lo;             // hi = lo + fwd
  int bwd = lo + a.N - hi;       // lo = hi + bwd (mod N)
  long long e = -1;
  if (fwd >= 1 && fwd <= a.half) e = (long long)lo * a.half + (fwd - 1);
  else if (bwd >= 1 && bwd <= a.half) e = (long long)hi * a.half + (bwd - 1);
  return e >= 0 && !ws_rewired(a, e);
}

struct WsSlot {
  unsigned long long key;  // lo * N + hi + 1 (0 = empty)
  unsigned int owner;      // lowest proposing edge index
  unsigned int accepted;   // 1 once a round settled this pair
};

__device__ __forceinline__ unsigned long long ws_key(int x, int y, int N) {
  return (unsigned long long)min(x, y) * (unsigned long long)N + max(x, y) + 1ull;
}

// final target of every lattice edge; pending list of rewired edges
__global__ void ws_init_kernel(WsArgs a, long long n_lat, int *target,
                               unsigned int *pending, unsigned int *n_pending) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n_lat;
       e += (long long)gridDim.x * blockDim.x) {
    const int u = (int)(e / a.half);
    const int j = (int)(e - (long long)u * a.half) + 1;
    if (ws_rewired(a, e)) {
      target[e] = -1;
      pending[atomicAdd(n_pending, 1u)] = (unsigned int)e;
    } else {
      target[e] = (u + j) % a.N;
    }
  }
}

// round r, phase 1: propose a target; meet the other proposals of the pair
__global__ void ws_propose_kernel(WsArgs a, int round, const unsigned int *pending,
                                  unsigned int n_pending, WsSlot *table,
                                  unsigned long long tmask, long long *cand) {
  for (unsigned int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_pending;
       k += gridDim.x * blockDim.x) {
    const unsigned int e = pending[k];
    const int u = (int)(e / a.half);
    const int w = (int)rng_below(a.seed, 16 + round, e, (unsigned int)a.N);
    cand[k] = -1;
    if (w == u || ws_kept_lattice(a, u, w)) continue;
    const unsigned long long key = ws_key(u, w, a.N);
    unsigned long long h = (key * 0x9E3779B97F4A7C15ull) & tmask;
    for (;;) {  // linear probing; the table is at most 1/4 full
      const unsigned long long prev = atomicCAS(&table[h].key, 0ull, key);
      if (prev == 0ull || prev == key) break;
      h = (h + 1) & tmask;
    }
    if (table[h].accepted) continue;  // settled in an earlier round
    atomicMin(&table[h].owner, e);
    cand[k] = (long long)h;
  }
}

// round r, phase 2: the lowest index of each pair wins; the rest retry
__global__ void ws_resolve_kernel(WsArgs a, int round, const unsigned int *pending,
                                  unsigned int n_pending, WsSlot *table,
                                  const long long *cand, int *target,
                                  unsigned int *next, unsigned int *n_next) {
  for (unsigned int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_pending;
       k += gridDim.x * blockDim.x) {
    const unsigned int e = pending[k];
    const long long h = cand[k];
    if (h >= 0 && table[h].owner == e) {
      target[e] = (int)rng_below(a.seed, 16 + round, e, (unsigned int)a.N);
      table[h].accepted = 1u;
    } else {
      next[atomicAdd(n_next, 1u)] = e;
    }
  }
}

__global__ void ws_degree_kernel(WsArgs a, long long n_lat, const int *target,
                                 int *deg) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n_lat;
       e += (long long)gridDim.x * blockDim.x) {
    const int u = (int)(e / a.half);
    atomicAdd(deg + u, 1);
    atomicAdd(deg + target[e], 1);
  }
}

// exclusive scan of deg[0..N) into row_ptr[0..N] (one block, N <= 2^24)
__global__ void ws_scan_kernel(const int *deg, int *row_ptr, int N) {
  __shared__ long long s_part[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const long long per = (N + T - 1) / T;
  const long long b = t * per, e = min((long long)N, b + per);
  long long sum = 0;
  for (long long i = b; i < e; ++i) sum += deg[i];
  s_part[t] = sum;
  __syncthreads();
  if (t == 0) {
    long long run = 0;
    for (int i = 0; i < T; ++i) {
      const long long v = s_part[i];
      s_part[i] = run;
      run += v;
    }
  }
  __syncthreads();
  long long run = s_part[t];
  for (long long i = b; i < e; ++i) {
    row_ptr[i] = (int)run;
    run += deg[i];
  }
  if (t == T - 1) row_ptr[N] = (int)run;
}

__global__ void ws_fill_kernel(WsArgs a, long long n_lat, const int *target,
                               const int *row_ptr, int *cursor, int *col) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n_lat;
       e += (long long)gridDim.x * blockDim.x) {
    const int u = (int)(e / a.half);
    const int v = target[e];
    col[row_ptr[u] + atomicAdd(cursor + u, 1)] = v;
    col[row_ptr[v] + atomicAdd(cursor + v, 1)] = u;
  }
}

// canonical CSR (columns sorted per row) and the initial state, drawn by
// position: delays U{lo..hi}, weights U[w_lo, w_hi), theta U[0, 2pi),
// omega Normal(mean, std) (Box-Muller)
struct WsStateArgs {
  unsigned long long seed;
  int delay_lo, delay_hi;
  float w_lo, w_hi, omega_mean, omega_std;
};

__global__ void ws_finish_kernel(WsStateArgs s, int N, const int *row_ptr, int *col,
                                 uint8_t *delays, float *weights, float *theta,
                                 float *omega) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int b = row_ptr[i], e = row_ptr[i + 1];
    for (int x = b + 1; x < e; ++x) {  // insertion sort (rows hold ~k entries)
      const int v = col[x];
      int y = x - 1;
      while (y >= b && col[y] > v) {
        col[y + 1] = col[y];
        --y;
      }
      col[y + 1] = v;
    }
    const unsigned span = (unsigned)(s.delay_hi - s.delay_lo + 1);
    for (int x = b; x < e; ++x) {
      delays[x] = (uint8_t)(s.delay_lo + (int)rng_below(s.seed, 8, x, span));
      weights[x] = (float)(s.w_lo + (s.w_hi - s.w_lo) * rng_u01(s.seed, 9, x));
    }
    theta[i] = (float)(2.0 * 3.14159265358979323846 * rng_u01(s.seed, 10, i));
    const double u1 = 1.0 - rng_u01(s.seed, 11, i), u2 = rng_u01(s.seed, 12, i);
    const double z = sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2);
    omega[i] = (float)(s.omega_mean + s.omega_std * z);
  }
}

}  // namespace lev
