// lev_engine.cu -- host side of the C ABI declared in include/leviathan_b200.h.
//
// Owns device memory, the engine stream, the tile list and the CUDA graphs of
// step blocks.  Replaces the host API of the reference engine
// (leviathan_kernel.cu:266-499): every failure returns a status code and
// leaves a message for lev_last_error(); nothing terminates the process.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include "leviathan_b200.h"
#include "lev_kernels.cuh"
#include "lev_pair.cuh"
#include "lev_cluster.cuh"
#include "lev_grid.cuh"  // uses cluster_sums from lev_cluster.cuh
#include "lev_part.cuh"

namespace lev {

static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

#define LEV_TRY_CUDA(call)                                                  \
  do {                                                                      \
    cudaError_t _e = (call);                                                \
    if (_e != cudaSuccess)                                                  \
      return fail(LEV_ERR_CUDA, std::string(#call) + " failed: " +          \
                                    cudaGetErrorString(_e));                \
  } while (0)

// Makes the engine's device current for the scope of an API call and puts
// the caller's device back afterwards.
struct DeviceScope {
  int prev = -1;
  bool switched = false;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) {
      switched = (cudaSetDevice(dev) == cudaSuccess);
    }
  }
  ~DeviceScope() {
    if (switched) cudaSetDevice(prev);
  }
};

struct GraphEntry {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

// Compiled step-kernel variants the autotuner chooses from (see
// step_kernel's template parameters).  Index 0 is the default.
using StepFn = void (*)(StepArgs);
struct StepVariant {
  int U, PIPE, MINB;
  StepFn fn[2];  // [math mode]
};
#define LEV_VARIANT(U, P, M) \
  { U, P, M, { step_kernel<0, U, P, M>, step_kernel<1, U, P, M> } }
static const StepVariant kVariants[] = {
    LEV_VARIANT(12, 1, 3), LEV_VARIANT(8, 1, 3), LEV_VARIANT(16, 0, 3),
    LEV_VARIANT(8, 0, 4),  LEV_VARIANT(4, 1, 4), LEV_VARIANT(6, 1, 4),
};
#undef LEV_VARIANT
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// Two-steps-per-launch variants (lev_pair.cuh): pair_kernel<MATH, U, MINB,
// DEEP> (DEEP: two-stage software pipeline).  Measured on B200: fewer
// resident CTAs with more loads in flight per lane win at large networks
// (the L1 keeps the tile's ring lines and col/delay words between the two
// walks); more CTAs win at the small networks of a sweep.
// LANES: threads per row (1: pair_kernel, 256-thread CTAs; 4: pair4_kernel,
// 1024-thread CTAs for low-degree rows).
struct PairVariant {
  int U, MINB, DEEP, LANES;
  StepFn fn[2];  // [math mode]
};
#define LEV_PAIR_VARIANT(U, M, D) \
  { U, M, D, 1, { pair_kernel<0, U, M, D>, pair_kernel<1, U, M, D> } }
#define LEV_PAIR4_VARIANT(U, M) \
  { U, M, 0, 4, { pair4_kernel<0, U, M>, pair4_kernel<1, U, M> } }
static const PairVariant kPairVariants[] = {
    LEV_PAIR_VARIANT(8, 2, 1), LEV_PAIR_VARIANT(6, 3, 1), LEV_PAIR_VARIANT(8, 3, 0),
    LEV_PAIR_VARIANT(4, 4, 1), LEV_PAIR_VARIANT(10, 2, 1), LEV_PAIR4_VARIANT(2, 1),
    LEV_PAIR4_VARIANT(4, 1),
};
#undef LEV_PAIR_VARIANT
#undef LEV_PAIR4_VARIANT
constexpr int kNumPairVariants = sizeof(kPairVariants) / sizeof(kPairVariants[0]);

// Networks of a batch are grouped by the mean SELL slice length (the
// per-lane edge count): each class has its own tile list and variant.
constexpr int kNumClasses = 3;
inline int degree_class(double mean_slice_len) {
  return mean_slice_len <= 14.0 ? 0 : (mean_slice_len <= 26.0 ? 1 : 2);
}

struct TileClass {
  int ntiles = 0;
  int tile_off = 0;  // first entry of this class in the tile list
  int variant = 0;
  int pair_variant = 0;  // two steps per launch with this variant; -1: one
  double mean_len = 0.0;  // mean slice length of the class
  long long edges = 0;
  int net_off = 0;       // first entry of this class in the class network list
  int nnets = 0;
  float step_ms = 0.0f;  // autotuner: best ms per step, one step per launch
  float pair_ms = 0.0f;  // autotuner: best ms per step, two steps per launch
};

// Autotuner results shared by the engines of a process, keyed by the degree
// class, its mean slice length (rounded) and the size of its tile list
// (power-of-two bucket).
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int>, int> g_tune_cache;
static std::map<std::tuple<int, int, int>, int> g_pair_cache;

inline std::tuple<int, int, int> tune_key(const TileClass &tc, int c) {
  int bucket = 0;
  while ((1 << bucket) < tc.ntiles) ++bucket;
  return std::make_tuple(c, (int)std::lround(tc.mean_len), bucket);
}

}  // namespace lev

using namespace lev;

struct LevHubs;

struct LevEngine {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_nets = 0;
  long long total_nodes = 0;
  long long total_edges = 0;   // sum of E
  long long num_slices = 0;    // SELL-32 slices over all networks
  long long sl_total = 0;      // SELL-32 entries (multiple of 32)
  long long rp_total = 0;
  long long ring_floats = 0;
  int total_tiles = 0;
  int math_mode = LEV_MATH_REFERENCE;
  int sweep = 0;  // direction of the next step's walk over the tiles
  size_t vram = 0;

  std::vector<NetDesc> h_nets;
  std::vector<long long> net_E;

  NetDesc *d_nets = nullptr;
  NetState *d_st = nullptr;
  int2 *d_tiles = nullptr;
  int *d_row_ptr = nullptr;
  long long *d_sl_off = nullptr;
  int *d_sl_len = nullptr;
  uint32_t *d_sl_cd = nullptr;
  float *d_sl_w = nullptr;
  float *d_theta = nullptr;
  float *d_theta_hat = nullptr;
  float *d_omega = nullptr;
  float *d_omega_hat = nullptr;
  float *d_ring = nullptr;
  float2 *d_part = nullptr;

  // two steps per launch (lev_pair.cuh): possible when no delay is 0
  bool pair_ok = false;
  bool use_pairs = true;
  float2 *d_pend = nullptr;  // [total_nodes] parked (coupling sum, eps)
  // speculative pairs of single steps (lev_step): the first call runs the
  // pair kernel with step t+1's weights and predictor going to the spec
  // buffers and returns r(t+1); the next call, if nothing wrote the engine
  // state in between and dt is the same, only finishes step t+1 and swaps the
  // weight buffers (w_flip tells which one is current, for the graph cache)
  bool spec = false;
  uint32_t spec_dt = 0;  // bits of the dt of the pending step
  float *d_w_spec = nullptr, *d_thh_spec = nullptr, *d_omh_spec = nullptr;
  void *spec_block = nullptr;  // the three spec buffers: one allocation from the pool
  size_t spec_bytes = 0;
  int w_flip = 0;
  int *d_class_nets = nullptr;  // networks of each class, class by class
  LevHubs *hubs = nullptr;      // attached hub monitor (lev_attach_hubs)
  // step blocks of engines with several degree classes: one chain of
  // launches per class, forked from and joined back to `stream` in the graph
  cudaStream_t class_stream[kNumClasses] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[kNumClasses] = {nullptr, nullptr, nullptr};

  // r of the last single step, written by the kernel into mapped host memory
  float *h_rmap = nullptr;
  float *d_rmap = nullptr;

  // r history of step blocks
  int block_len = 256;
  float *d_rhist = nullptr;   // [block_len][num_nets]
  float *h_rstage = nullptr;  // pinned staging for lev_step_n
  size_t h_rstage_len = 0;

  std::map<std::tuple<int, uint32_t, int>, GraphEntry> graphs;

  TileClass classes[kNumClasses];

  // cluster-resident path for small single networks (lev_cluster.cuh)
  bool cluster_ok = false;   // eligible and launchable on this device
  bool use_cluster = true;   // may step blocks use it
  int cluster_R = 0, cluster_C = 0, cluster_edge_cap = 0;
  size_t cluster_smem = 0;

  // grid-resident path for mid-sized single networks (lev_grid.cuh): one
  // cooperative launch per step block, rows per CTA 64, 128 or 256
  bool grid_ok = false;      // some rows-per-CTA choice is eligible
  bool use_grid = true;      // may step blocks use it
  int grid_R = 0;            // rows per CTA in use
  bool grid_R_ok[3] = {false, false, false};  // R = 64, 128, 256
  int grid_cap[3] = {0, 0, 0};                // SELL entries per CTA
  size_t grid_smem_R[3] = {0, 0, 0};
  int grid_nwarps = 0;
  float2 *d_gwsum = nullptr;  // [2][grid_nwarps]
  unsigned *d_gbar = nullptr;
  int *h_gerr = nullptr, *d_gerr = nullptr;  // barrier timeout flag (mapped)
  GridWait grid_wait = {kGridWaitNs, 0u, 0u};  // bound of the barrier waits

  // one device allocation holding the arrays sized at creation
  void *slab = nullptr;
  size_t slab_bytes = 0;

  // wall-clock ms of the phases of creation (lev_create_profile)
  double create_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};

  // partition of a network split over GPUs (lev_part.cuh, lev_part_*): own
  // rows stepped here, halo phases in ring columns N .. N + part_halo - 1
  bool part = false;
  int part_halo = 0;
  int part_N_global = 0;
  int part_tile_off = 0;      // first global tile of the partition
  int part_ntiles_global = 0;
};

struct LeviathanHandle {
  LevEngine *eng;
};

// Hub-phase transition counter (HubMonitor on the device).
struct LevHubs {
  int device = 0;
  int num_hubs = 0;
  int S = 0;  // 2^num_hubs states
  HubMonitor *d_mon = nullptr;
  unsigned long long *d_counts = nullptr;  // [S][S]
  unsigned long long *d_totals = nullptr;  // [S]
  cudaStream_t stream = nullptr;           // standalone observations
  LevEngine *engine = nullptr;             // engine that feeds it, if attached
};

namespace {

template <typename T>
int dev_alloc(LevEngine *h, T **p, size_t count) {
  size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(LEV_ERR_NOMEM, std::string("cudaMalloc of ") +
                                   std::to_string(bytes) + " bytes failed: " +
                                   cudaGetErrorString(e));
  }
  h->vram += bytes;
  return LEV_OK;
}

// Device memory of engines comes from one stream-ordered pool per device
// that keeps freed memory for the next engine of the process (creating an
// engine then costs no driver allocation when an earlier one was freed);
// lev_trim_memory gives it back to the device.
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};

cudaError_t engine_pool(int dev, cudaMemPool_t *out) {
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaError_t e = cudaMemPoolCreate(&g_pool[dev], &props);
    if (e != cudaSuccess) {
      g_pool[dev] = nullptr;
      return e;
    }
    uint64_t keep = ~0ull;
    e = cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

// The r of the last single step is written by the kernel into mapped host
// memory.  Engines take 4 KiB slots of one mapped block per process (a
// mapped allocation of its own costs milliseconds); an engine with more
// networks than a slot holds gets its own.
constexpr size_t kMapSlot = 4096;
constexpr int kMapSlots = 256;
struct MappedArena {
  std::mutex mu;
  char *base = nullptr;
  bool used[kMapSlots] = {};
};
MappedArena g_map;

float *mapped_alloc(size_t n_floats) {
  if (n_floats * sizeof(float) <= kMapSlot) {
    std::lock_guard<std::mutex> lk(g_map.mu);
    if (!g_map.base &&
        cudaHostAlloc(reinterpret_cast<void **>(&g_map.base), kMapSlot * kMapSlots,
                      cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      g_map.base = nullptr;
    }
    if (g_map.base)
      for (int k = 0; k < kMapSlots; ++k)
        if (!g_map.used[k]) {
          g_map.used[k] = true;
          return reinterpret_cast<float *>(g_map.base + k * kMapSlot);
        }
  }
  float *p = nullptr;
  if (cudaHostAlloc(reinterpret_cast<void **>(&p), std::max<size_t>(n_floats, 1) * sizeof(float),
                    cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
    return nullptr;
  return p;
}

void mapped_free(float *p) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lk(g_map.mu);
    char *c = reinterpret_cast<char *>(p);
    if (g_map.base && c >= g_map.base && c < g_map.base + kMapSlot * kMapSlots) {
      g_map.used[(c - g_map.base) / kMapSlot] = false;
      return;
    }
  }
  cudaFreeHost(p);
}

void free_engine(LevEngine *h) {
  if (!h) return;
  if (h->hubs) h->hubs->engine = nullptr;
  for (auto &kv : h->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  h->graphs.clear();
  // arrays inside the creation slab go with it (a pointer swapped with a
  // separately allocated buffer, as the speculative weights are, is freed
  // on its own)
  auto dfree = [h](void *p) {
    const char *c = static_cast<const char *>(p);
    const char *b = static_cast<const char *>(h->slab);
    const char *q = static_cast<const char *>(h->spec_block);
    if (p && !(b && c >= b && c < b + h->slab_bytes) &&
        !(q && c >= q && c < q + h->spec_bytes))
      cudaFree(p);
  };
  dfree(h->d_nets);
  dfree(h->d_st);
  dfree(h->d_tiles);
  dfree(h->d_row_ptr);
  dfree(h->d_sl_off);
  dfree(h->d_sl_len);
  dfree(h->d_sl_cd);
  dfree(h->d_sl_w);
  dfree(h->d_theta);
  dfree(h->d_theta_hat);
  dfree(h->d_omega);
  dfree(h->d_omega_hat);
  dfree(h->d_ring);
  dfree(h->d_part);
  dfree(h->d_pend);
  dfree(h->d_w_spec);
  dfree(h->d_thh_spec);
  dfree(h->d_omh_spec);
  dfree(h->d_class_nets);
  dfree(h->d_rhist);
  dfree(h->d_gwsum);
  dfree(h->d_gbar);
  if (h->spec_block) cudaFreeAsync(h->spec_block, h->stream);
  if (h->slab) cudaFreeAsync(h->slab, h->stream);  // back to the engine pool
  if (h->h_gerr) cudaFreeHost(h->h_gerr);
  mapped_free(h->h_rmap);
  if (h->h_rstage) cudaFreeHost(h->h_rstage);
  for (int c = 0; c < kNumClasses; ++c) {
    if (h->class_stream[c]) cudaStreamDestroy(h->class_stream[c]);
    if (h->ev_join[c]) cudaEventDestroy(h->ev_join[c]);
  }
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

void params_to_desc(const LevParams &p, NetDesc *d) {
  d->eta = p.eta;
  d->lam = p.lam;
  d->gamma = p.gamma;
  d->alpha = p.alpha_eps;
  d->kappa_w = p.kappa_w;
  d->w_min = p.w_min;
  d->w_max = p.w_max;
  d->r0 = p.r0;
  d->beta = p.beta;
  d->mu = p.mu;
  d->g_rest = p.g_rest;
  d->g_min = p.g_min;
  d->g_max = p.g_max;
  d->ctrl = p.gain_controller ? 1 : 0;
}

void desc_to_params(const NetDesc &d, float g, LevParams *p) {
  p->eta = d.eta;
  p->lam = d.lam;
  p->gamma = d.gamma;
  p->alpha_eps = d.alpha;
  p->kappa_w = d.kappa_w;
  p->w_min = d.w_min;
  p->w_max = d.w_max;
  p->g = g;
  p->r0 = d.r0;
  p->beta = d.beta;
  p->mu = d.mu;
  p->g_rest = d.g_rest;
  p->g_min = d.g_min;
  p->g_max = d.g_max;
  p->gain_controller = d.ctrl;
  p->reserved = 0;
}

int check_params(const LevParams &p) {
  const float v[] = {p.eta, p.lam, p.gamma, p.alpha_eps, p.kappa_w,
                     p.w_min, p.w_max, p.g, p.r0, p.beta,
                     p.mu, p.g_rest, p.g_min, p.g_max};
  for (float x : v)
    if (!std::isfinite(x)) return fail(LEV_ERR_ARG, "parameter is not finite");
  if (p.w_min > p.w_max) return fail(LEV_ERR_ARG, "w_min > w_max");
  if (p.g_min > p.g_max) return fail(LEV_ERR_ARG, "g_min > g_max");
  return LEV_OK;
}

int launch_fill(LevEngine *h, int n) {
  const NetDesc &nd = h->h_nets[n];
  const long long total = (long long)nd.bsi * nd.N;
  int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  ring_fill_kernel<<<blocks, 256, 0, h->stream>>>(
      h->d_theta + nd.node_off, h->d_ring + nd.ring_off, nd.N, nd.Np, nd.bsi, 0, 1);
  LEV_TRY_CUDA(cudaGetLastError());
  return LEV_OK;
}

StepArgs make_args(LevEngine *h, float dt, float *r_hist, int r_cap,
                   float *r_host) {
  StepArgs a;
  a.nets = h->d_nets;
  a.st = h->d_st;
  a.tiles = h->d_tiles;
  a.row_ptr = h->d_row_ptr;
  a.sl_off = h->d_sl_off;
  a.sl_len = h->d_sl_len;
  a.sl_cd = h->d_sl_cd;
  a.sl_w = h->d_sl_w;
  a.theta = h->d_theta;
  a.theta_hat = h->d_theta_hat;
  a.omega = h->d_omega;
  a.omega_hat = h->d_omega_hat;
  a.ring = h->d_ring;
  a.partials = h->d_part;
  a.r_hist = r_hist;
  a.r_host = r_host;
  a.r_cap = r_cap;
  a.num_nets = h->num_nets;
  a.dt = dt;
  a.reverse = 0;
  a.pend = h->d_pend;
  a.hubs = h->hubs ? h->hubs->d_mon : nullptr;
  a.w2 = nullptr;
  a.thh2 = nullptr;
  a.omh2 = nullptr;
  return a;
}

// The step kernel keeps almost nothing in shared memory; prefer the largest
// L1 carve-out so ring gathers reuse lines across a tile's rows.
int prepare_step_kernels() {
  for (int v = 0; v < kNumVariants; ++v)
    for (int m = 0; m < 2; ++m)
      LEV_TRY_CUDA(cudaFuncSetAttribute(
          reinterpret_cast<const void *>(kVariants[v].fn[m]),
          cudaFuncAttributePreferredSharedMemoryCarveout,
          (int)cudaSharedmemCarveoutMaxL1));
  for (int v = 0; v < kNumPairVariants; ++v)
    for (int m = 0; m < 2; ++m)
      LEV_TRY_CUDA(cudaFuncSetAttribute(
          reinterpret_cast<const void *>(kPairVariants[v].fn[m]),
          cudaFuncAttributePreferredSharedMemoryCarveout,
          (int)cudaSharedmemCarveoutMaxL1));
  return LEV_OK;
}

int launch_class(LevEngine *h, int c, StepArgs a, cudaStream_t s = nullptr) {
  const TileClass &tc = h->classes[c];
  if (tc.ntiles == 0) return LEV_OK;
  if (!s) s = h->stream;
  a.tiles = h->d_tiles + tc.tile_off;
  const int mode = (h->math_mode == LEV_MATH_ACCURATE) ? 1 : 0;
  void *args[] = {&a};
  LEV_TRY_CUDA(cudaLaunchKernel(
      reinterpret_cast<const void *>(kVariants[tc.variant].fn[mode]),
      dim3(tc.ntiles), dim3(kTile), args, 0, s));
  return LEV_OK;
}

// Launches one step: one kernel per degree class, each over its own tiles
// with its own variant.  Successive steps alternate the direction in which
// CTAs walk the tiles, so the ring lines touched at the end of one step are
// the first touched by the next while they are still in L2; results do not
// depend on the direction or on the variant.
int launch_step(LevEngine *h, StepArgs a) {
  a.reverse = h->sweep;
  h->sweep ^= 1;
  for (int c = 0; c < kNumClasses; ++c) {
    int rc = launch_class(h, c, a);
    if (rc != LEV_OK) return rc;
  }
  return LEV_OK;
}

// A pair variant index in range.
bool pair_variant_ok(const LevEngine *, int v) { return v >= 0 && v < kNumPairVariants; }

// Two-steps-per-launch path (lev_pair.cuh) in use for at least one class.
bool pairs_active(const LevEngine *h) {
  if (!h->pair_ok || !h->use_pairs) return false;
  for (int c = 0; c < kNumClasses; ++c)
    if (h->classes[c].ntiles > 0 && h->classes[c].pair_variant >= 0) return true;
  return false;
}

// phase 0: pair_kernel (or a first step_kernel for a class without a pair
// variant); phase 1: finish_kernel (or a second step_kernel).
int launch_pair_tc(LevEngine *h, const TileClass &tc, StepArgs a, int phase,
                   cudaStream_t s = nullptr) {
  if (tc.ntiles == 0) return LEV_OK;
  if (!s) s = h->stream;
  a.tiles = h->d_tiles + tc.tile_off;
  const int mode = (h->math_mode == LEV_MATH_ACCURATE) ? 1 : 0;
  if (tc.pair_variant < 0 || phase == 0) {
    const void *fn =
        tc.pair_variant < 0
            ? reinterpret_cast<const void *>(kVariants[tc.variant].fn[mode])
            : reinterpret_cast<const void *>(kPairVariants[tc.pair_variant].fn[mode]);
    const int lanes = tc.pair_variant < 0 ? 1 : kPairVariants[tc.pair_variant].LANES;
    void *args[] = {&a};
    LEV_TRY_CUDA(cudaLaunchKernel(fn, dim3(tc.ntiles), dim3(lanes * kTile), args, 0, s));
  } else {
    const int blocks = (tc.ntiles + kFinishTiles - 1) / kFinishTiles;
    if (mode)
      finish_kernel<1><<<blocks, kTile, 0, s>>>(a, tc.ntiles);
    else
      finish_kernel<0><<<blocks, kTile, 0, s>>>(a, tc.ntiles);
    LEV_TRY_CUDA(cudaGetLastError());
  }
  if (tc.pair_variant >= 0) {  // r and g of the class's networks
    reduce_kernel<<<tc.nnets, kReduceThreads, 0, s>>>(a, h->d_class_nets + tc.net_off);
    LEV_TRY_CUDA(cudaGetLastError());
  }
  return LEV_OK;
}

int launch_pair_class(LevEngine *h, int c, StepArgs a, int phase, cudaStream_t s = nullptr) {
  return launch_pair_tc(h, h->classes[c], a, phase, s);
}

// When every degree class that has tiles takes two steps per launch with
// the same pair variant, the classes run as one: their tiles are contiguous
// in the tile list (class by class) and the class network list holds every
// network, so one pair, finish and reduce launch each cover the engine.
// That saves the launches and the tail of each class's launch (measured on
// the 512-network sweep: one chain per class forked on three streams
// overlapped little, each launch filling the GPU).
bool merged_pairs(const LevEngine *h, TileClass *out) {
  int v = -2, nbusy = 0, first = -1;
  for (int c = 0; c < kNumClasses; ++c) {
    const TileClass &tc = h->classes[c];
    if (tc.ntiles == 0) continue;
    if (first < 0) first = c;
    ++nbusy;
    if (tc.pair_variant < 0 || (v != -2 && tc.pair_variant != v)) return false;
    v = tc.pair_variant;
  }
  if (nbusy < 2) return false;
  *out = TileClass();
  out->ntiles = h->total_tiles;
  out->tile_off = 0;
  out->variant = h->classes[first].variant;
  out->pair_variant = v;
  out->net_off = 0;
  out->nnets = h->num_nets;
  return true;
}

// Two steps of every class.
int launch_two_steps(LevEngine *h, StepArgs a) {
  for (int phase = 0; phase < 2; ++phase) {
    a.reverse = h->sweep;
    h->sweep ^= 1;
    for (int c = 0; c < kNumClasses; ++c) {
      int rc = launch_pair_class(h, c, a, phase);
      if (rc != LEV_OK) return rc;
    }
  }
  return LEV_OK;
}

// Every class of the engine takes two steps per launch (speculative pairs
// need it: a class stepped by step_kernel updates the weights in place).
bool pairs_all(const LevEngine *h) {
  if (!h->pair_ok || !h->use_pairs) return false;
  for (int c = 0; c < kNumClasses; ++c)
    if (h->classes[c].ntiles > 0 && h->classes[c].pair_variant < 0) return false;
  return true;
}

// Anything that writes the engine state (or the kernels' configuration)
// drops a pending speculative step; the state itself is that after the last
// completed step.
inline void spec_drop(LevEngine *h) { h->spec = false; }

void clear_graphs(LevEngine *h) {
  for (auto &kv : h->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  h->graphs.clear();
}

// The launches of one block of `len` steps (r history rows 0..len-1), on the
// engine stream: recorded into a graph by get_graph, or issued directly.
int issue_block(LevEngine *h, int len, float dt) {
  reset_rpos_kernel<<<1, 128, 0, h->stream>>>(h->d_st, h->num_nets);
  StepArgs a = make_args(h, dt, h->d_rhist, h->block_len, nullptr);
  int rc = LEV_OK;
  const bool pairs = pairs_active(h);
  int busy[kNumClasses], nbusy = 0;
  for (int c = 0; c < kNumClasses; ++c)
    if (h->classes[c].ntiles > 0) busy[nbusy++] = c;
  TileClass merged;
  if (pairs && merged_pairs(h, &merged)) {
    for (int i = 0; i < len && rc == LEV_OK;) {
      if (i + 1 < len) {
        for (int phase = 0; phase < 2 && rc == LEV_OK; ++phase) {
          a.reverse = h->sweep;
          h->sweep ^= 1;
          rc = launch_pair_tc(h, merged, a, phase);
        }
        i += 2;
      } else {
        rc = launch_step(h, a);
        i += 1;
      }
    }
  } else if (nbusy > 1 && h->ev_fork) {
    // the classes' networks are independent: one chain per class, so the
    // classes' launches overlap instead of queueing behind each other
    LEV_TRY_CUDA(cudaEventRecord(h->ev_fork, h->stream));
    const int sweep0 = h->sweep;
    for (int q = 0; q < nbusy; ++q) {
      const int c = busy[q];
      cudaStream_t cs = h->class_stream[c];
      if (rc == LEV_OK && cudaStreamWaitEvent(cs, h->ev_fork, 0) != cudaSuccess)
        rc = fail(LEV_ERR_CUDA, "graph fork failed");
      int sweep = sweep0;
      const bool two = pairs && h->classes[c].pair_variant >= 0;
      for (int i = 0; i < len && rc == LEV_OK;) {
        const int n = (two && i + 1 < len) ? 2 : 1;
        for (int phase = 0; phase < n && rc == LEV_OK; ++phase) {
          a.reverse = sweep;
          sweep ^= 1;
          rc = (n == 2) ? launch_pair_class(h, c, a, phase, cs) : launch_class(h, c, a, cs);
        }
        i += n;
      }
      // join every chain that was forked, even after a failure
      cudaEventRecord(h->ev_join[c], cs);
      cudaStreamWaitEvent(h->stream, h->ev_join[c], 0);
      h->sweep = sweep;
    }
  } else {
    for (int i = 0; i < len && rc == LEV_OK;) {
      if (pairs && i + 1 < len) {
        rc = launch_two_steps(h, a);
        i += 2;
      } else {
        rc = launch_step(h, a);
        i += 1;
      }
    }
  }
  return rc;
}

// Graph of `len` steps keyed by (len, dt, mode).  The first request of a key
// gets *out = null and the caller issues the block directly (a graph pays
// for itself only when replayed: capture and instantiation cost more than
// the launches of one block); the next request records the graph.
int get_graph(LevEngine *h, int len, float dt, cudaGraphExec_t *out) {
  uint32_t dbits;
  std::memcpy(&dbits, &dt, 4);
  auto key = std::make_tuple(len, dbits, h->math_mode + 2 * h->w_flip);
  auto it = h->graphs.find(key);
  if (it != h->graphs.end() && it->second.exec) {
    *out = it->second.exec;
    return LEV_OK;
  }
  if (it == h->graphs.end()) {
    if (h->graphs.size() >= 16) clear_graphs(h);
    h->graphs[key] = GraphEntry();  // seen once
    *out = nullptr;
    return LEV_OK;
  }
  GraphEntry ge;
  LEV_TRY_CUDA(
      cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = issue_block(h, len, dt);
  cudaError_t ce = cudaStreamEndCapture(h->stream, &ge.graph);
  if (rc != LEV_OK) {
    if (ge.graph) cudaGraphDestroy(ge.graph);
    return rc;
  }
  if (ce != cudaSuccess)
    return fail(LEV_ERR_CUDA,
                std::string("graph capture failed: ") + cudaGetErrorString(ce));
  ce = cudaGraphInstantiate(&ge.exec, ge.graph, 0);
  if (ce != cudaSuccess) {
    cudaGraphDestroy(ge.graph);
    return fail(LEV_ERR_CUDA, std::string("graph instantiate failed: ") +
                                  cudaGetErrorString(ce));
  }
  h->graphs[key] = ge;
  *out = ge.exec;
  return LEV_OK;
}

// Cluster kernel for R rows per CTA (measured on B200): up to 128 rows four
// lanes per row (4R threads); 256 rows one lane per row with 24 gathers in
// flight; above, one lane per row with 8.
using ClusterFn = void (*)(ClusterArgs);
ClusterFn cluster_fn(int R, int math_mode) {
  const bool acc = math_mode == LEV_MATH_ACCURATE;
  if (R <= 128) return acc ? cluster_split_kernel<1, 8> : cluster_split_kernel<0, 8>;
  if (R <= 256) return acc ? cluster_kernel<1, 256, 24> : cluster_kernel<0, 256, 24>;
  return acc ? cluster_kernel<1, kClusterRowsMax, 8> : cluster_kernel<0, kClusterRowsMax, 8>;
}
inline int cluster_threads(int R) { return R <= 128 ? 4 * R : R; }

// One launch of the cluster-resident kernel: `len` steps, r history rows
// 0..len-1 in d_rhist.
int launch_cluster(LevEngine *h, float dt, int len) {
  reset_rpos_kernel<<<1, 128, 0, h->stream>>>(h->d_st, h->num_nets);
  ClusterArgs ca;
  ca.net = h->d_nets;
  ca.st = h->d_st;
  ca.row_ptr = h->d_row_ptr;
  ca.sl_off = h->d_sl_off;
  ca.sl_len = h->d_sl_len;
  ca.sl_cd = h->d_sl_cd;
  ca.sl_w = h->d_sl_w;
  ca.theta = h->d_theta;
  ca.theta_hat = h->d_theta_hat;
  ca.omega = h->d_omega;
  ca.omega_hat = h->d_omega_hat;
  ca.ring = h->d_ring;
  ca.r_hist = h->d_rhist;
  ca.r_cap = h->block_len;
  ca.n_steps = len;
  ca.R = h->cluster_R;
  ca.lgR = 0;
  while ((1 << ca.lgR) < h->cluster_R) ++ca.lgR;
  ca.edge_cap = h->cluster_edge_cap;
  ca.early = h->pair_ok ? 1 : 0;  // no delay is 0
  ca.dt = dt;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(h->cluster_C);
  cfg.blockDim = dim3(cluster_threads(h->cluster_R));
  cfg.dynamicSmemBytes = h->cluster_smem;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = h->cluster_C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LEV_TRY_CUDA(cudaLaunchKernelEx(&cfg, cluster_fn(h->cluster_R, h->math_mode), ca));
  return LEV_OK;
}

// Small single networks: choose rows per CTA and check that the cluster
// kernel can run (shared memory, cluster size, occupancy).
void setup_cluster(LevEngine *h, const std::vector<long long> &sl_off,
                   const std::vector<int> &sl_len) {
  h->cluster_ok = false;
  if (h->num_nets != 1) return;
  const NetDesc &d = h->h_nets[0];
  int dev = 0, max_smem = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  if (cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
      cudaSuccess)
    return;
  // the smallest rows-per-CTA that fits (up to 16 CTAs): the most SMs
  for (int R = 32; R <= kClusterRowsMax; R *= 2) {
    const int C = (d.N + R - 1) / R;
    if (C > kClusterMax) continue;
    long long cap = 0;
    for (int c = 0; c < C; ++c) {
      long long e = 0;
      for (int s = c * R / 32; s < std::min<long long>((c + 1) * R / 32, (d.N + 31) / 32); ++s)
        e += 32LL * sl_len[d.slice_base + s];
      cap = std::max(cap, e);
    }
    const size_t smem = sizeof(float2) * 2 * kClusterWarpsMax + sizeof(int) * 2 * (R / 32) +
                        sizeof(float) * (R <= 128 ? 6 : 4) * R +
                        sizeof(float) * (size_t)d.bsi * R + 8 * (size_t)cap;
    if (smem + 1024 > (size_t)max_smem) continue;
    bool ok = true;
    for (int m = 0; m < 2 && ok; ++m) {
      const void *fn = reinterpret_cast<const void *>(
          cluster_fn(R, m ? LEV_MATH_ACCURATE : LEV_MATH_REFERENCE));
      ok = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
               cudaSuccess &&
           cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
               cudaSuccess;
      if (ok) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(C);
        cfg.blockDim = dim3(cluster_threads(R));
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        ok = cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) == cudaSuccess && clusters >= 1;
      }
    }
    cudaGetLastError();  // clear a refused attribute, if any
    if (!ok) continue;
    h->cluster_ok = true;
    h->cluster_R = R;
    h->cluster_C = C;
    h->cluster_edge_cap = (int)cap;
    h->cluster_smem = smem;
    // measured on B200: faster than per-step graph replay up to 256 rows per
    // CTA (N = 4096 on 16 CTAs), slower at 1024; lev_autotune times both
    // and decides per engine
    h->use_cluster = R <= 256;
    return;
  }
}

// Grid kernel for R rows per CTA (64, 128, 256), four lanes per row.
using GridFn = void (*)(GridArgs);
constexpr int kGridRs[3] = {64, 128, 256};
GridFn grid_fn(int R, int math_mode) {
  const bool acc = math_mode == LEV_MATH_ACCURATE;
  if (R == 64) return acc ? grid_kernel<1, 64, 8> : grid_kernel<0, 64, 8>;
  if (R == 128) return acc ? grid_kernel<1, 128, 8> : grid_kernel<0, 128, 8>;
  return acc ? grid_kernel<1, 256, 8> : grid_kernel<0, 256, 8>;
}
inline int grid_r_index(int R) { return R == 64 ? 0 : (R == 128 ? 1 : 2); }

// One cooperative launch of the grid-resident kernel: `len` steps, r history
// rows 0..len-1 in d_rhist.
int launch_grid(LevEngine *h, float dt, int len) {
  reset_rpos_kernel<<<1, 128, 0, h->stream>>>(h->d_st, h->num_nets);
  LEV_TRY_CUDA(cudaMemsetAsync(h->d_gbar, 0, sizeof(unsigned), h->stream));
  const int R = h->grid_R, ri = grid_r_index(R);
  GridArgs ga;
  ga.net = h->d_nets;
  ga.st = h->d_st;
  ga.row_ptr = h->d_row_ptr;
  ga.sl_off = h->d_sl_off;
  ga.sl_len = h->d_sl_len;
  ga.sl_cd = h->d_sl_cd;
  ga.sl_w = h->d_sl_w;
  ga.theta = h->d_theta;
  ga.theta_hat = h->d_theta_hat;
  ga.omega = h->d_omega;
  ga.omega_hat = h->d_omega_hat;
  ga.ring = h->d_ring;
  ga.wsum = h->d_gwsum;
  ga.bar = h->d_gbar;
  ga.early = h->pair_ok ? 1 : 0;  // no delay is 0
  ga.err = h->d_gerr;
  ga.wait = h->grid_wait;
  ga.r_hist = h->d_rhist;
  ga.r_cap = h->block_len;
  ga.n_steps = len;
  ga.nwarps = h->grid_nwarps;
  ga.edge_cap = h->grid_cap[ri];
  ga.dt = dt;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((h->h_nets[0].N + R - 1) / R);
  cfg.blockDim = dim3(kGridLPR * R);
  cfg.dynamicSmemBytes = h->grid_smem_R[ri];
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LEV_TRY_CUDA(cudaLaunchKernelEx(&cfg, grid_fn(R, h->math_mode), ga));
  return LEV_OK;
}

// Mid-sized single networks: for each rows-per-CTA choice, check that every
// CTA of the grid kernel can be resident at once (shared memory, occupancy,
// cooperative launch).  Allocates the warp sums, barrier and error flag.
int setup_grid(LevEngine *h, const std::vector<long long> &sl_off,
               const std::vector<int> &sl_len) {
  h->grid_ok = false;
  if (h->num_nets != 1) return LEV_OK;
  const NetDesc &d = h->h_nets[0];
  int dev = 0, max_smem = 0, coop = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
          cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return LEV_OK;
  }
  if (!coop) return LEV_OK;
  const int nblocks = (d.N + kTile - 1) / kTile;
  const int nwarps = 8 * nblocks;
  for (int ri = 0; ri < 3; ++ri) {
    const int R = kGridRs[ri];
    const int C = (d.N + R - 1) / R;
    if (C < 2) continue;  // one CTA: the cluster path or graph replay
    long long cap = 0;
    for (int c = 0; c < C; ++c) {
      long long e = 0;
      for (int s = c * R / 32; s < std::min<long long>((c + 1) * R / 32, (d.N + 31) / 32); ++s)
        e += 32LL * sl_len[d.slice_base + s];
      cap = std::max(cap, e);
    }
    const size_t smem = sizeof(float2) * nwarps + sizeof(float) * 6 * R +
                        sizeof(int) * 2 * (R / 32) + 8 * (size_t)cap;
    if (smem + 1024 > (size_t)max_smem) continue;
    bool ok = true;
    for (int m = 0; m < 2 && ok; ++m) {
      const void *fn = reinterpret_cast<const void *>(
          grid_fn(R, m ? LEV_MATH_ACCURATE : LEV_MATH_REFERENCE));
      int per_sm = 0;
      ok = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
               cudaSuccess &&
           cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kGridLPR * R, smem) ==
               cudaSuccess &&
           (long long)per_sm * sms >= C;
    }
    cudaGetLastError();  // clear a refused attribute, if any
    if (!ok) continue;
    h->grid_R_ok[ri] = true;
    h->grid_cap[ri] = (int)cap;
    h->grid_smem_R[ri] = smem;
    if (!h->grid_ok) h->grid_R = R;  // the smallest: the most SMs
    h->grid_ok = true;
  }
  if (!h->grid_ok) return LEV_OK;
  h->grid_nwarps = nwarps;
  int rc = dev_alloc(h, &h->d_gwsum, 2 * (size_t)nwarps);
  if (rc == LEV_OK) rc = dev_alloc(h, &h->d_gbar, 1);
  if (rc != LEV_OK) return rc;
  LEV_TRY_CUDA(cudaMemset(h->d_gwsum, 0, sizeof(float2) * 2 * (size_t)nwarps));
  LEV_TRY_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&h->h_gerr), sizeof(int),
                             cudaHostAllocMapped));
  *h->h_gerr = 0;
  LEV_TRY_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&h->d_gerr), h->h_gerr, 0));
  return LEV_OK;
}

// After the stream has drained: a grid barrier that timed out leaves the
// engine state undefined; report it once and stop using the grid path.
int check_grid_error(LevEngine *h) {
  if (h->h_gerr && *reinterpret_cast<volatile int *>(h->h_gerr)) {
    *h->h_gerr = 0;
    h->grid_ok = false;
    return fail(LEV_ERR_CUDA,
                "grid-resident step block: a grid barrier wait timed out; the engine state "
                "is undefined");
  }
  return LEV_OK;
}

// Enqueue n steps as graph replays (or cluster-kernel launches for small
// networks); if stage != null, the r history of every block is copied into
// stage[n][num_nets] (pinned host memory).
int enqueue_steps(LevEngine *h, float dt, int n, float *stage) {
  spec_drop(h);
  int done = 0;
  while (done < n) {
    const int len = std::min(h->block_len, n - done);
    if (h->cluster_ok && h->use_cluster && !h->hubs) {
      int rc = launch_cluster(h, dt, len);
      if (rc != LEV_OK) return rc;
    } else if (h->grid_ok && h->use_grid && !h->hubs) {
      int rc = launch_grid(h, dt, len);
      if (rc != LEV_OK) return rc;
    } else {
      cudaGraphExec_t ex = nullptr;
      int rc = get_graph(h, len, dt, &ex);
      if (rc == LEV_OK && !ex) rc = issue_block(h, len, dt);
      if (rc != LEV_OK) return rc;
      if (ex) LEV_TRY_CUDA(cudaGraphLaunch(ex, h->stream));
    }
    if (stage) {
      LEV_TRY_CUDA(cudaMemcpyAsync(
          stage + (size_t)done * h->num_nets, h->d_rhist,
          sizeof(float) * (size_t)len * h->num_nets, cudaMemcpyDeviceToHost,
          h->stream));
    }
    done += len;
  }
  return LEV_OK;
}

int read_states(LevEngine *h, std::vector<NetState> &st) {
  st.resize(h->num_nets);
  LEV_TRY_CUDA(cudaMemcpyAsync(st.data(), h->d_st,
                               sizeof(NetState) * h->num_nets,
                               cudaMemcpyDeviceToHost, h->stream));
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return LEV_OK;
}

int write_state(LevEngine *h, int n, const NetState &s) {
  LEV_TRY_CUDA(cudaMemcpyAsync(h->d_st + n, &s, sizeof(NetState),
                               cudaMemcpyHostToDevice, h->stream));
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return LEV_OK;
}

// Host <-> device transfers of caller (pageable) memory through pinned
// staging.  The driver moves pageable memory through its own staging at one
// host thread's memcpy speed; here a transfer is cut into jobs of at most
// kStageBytes, and up to kStageThreads host threads each copy a job into a
// pinned buffer of their own and issue its DMA on the engine stream, with
// two buffers per thread so one is filled while the other's DMA runs.  The buffers are allocated on the
// first large transfer of the process (on that device) and kept.
// The staging is bound by host memory: every staged byte is read from the
// caller's array, written to a pinned buffer and read again by the DMA.
// Measured on the B200 box (16 cores, one socket; 300 MB, 2 MB buffers):
// eight threads 7.6 ms with memcpy, sixteen 8.2 ms; with the non-temporal
// copy below (no read-for-ownership of the pinned lines) eight threads
// 6.6 ms.  Page-locking the caller's arrays in place costs 70 ms for 304 MB.
constexpr size_t kStageBytes = 2u << 20;
constexpr int kStageThreads = 8;

// Copy into a pinned staging buffer (dst 16-byte aligned) with streaming
// stores: the lines go to memory without being read first.
void stage_copy_in(void *dst, const void *src, size_t n) {
#if defined(__SSE2__)
  char *d = static_cast<char *>(dst);
  const char *s = static_cast<const char *>(src);
  size_t i = 0;
  for (; i + 64 <= n; i += 64) {
    const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s + i));
    const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s + i + 16));
    const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s + i + 32));
    const __m128i e = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s + i + 48));
    _mm_stream_si128(reinterpret_cast<__m128i *>(d + i), a);
    _mm_stream_si128(reinterpret_cast<__m128i *>(d + i + 16), b);
    _mm_stream_si128(reinterpret_cast<__m128i *>(d + i + 32), c);
    _mm_stream_si128(reinterpret_cast<__m128i *>(d + i + 48), e);
  }
  _mm_sfence();  // the streamed lines are in memory before the DMA is issued
  if (i < n) std::memcpy(d + i, s + i, n - i);
#else
  std::memcpy(dst, src, n);
#endif
}
constexpr int kStageBufs = 2 * kStageThreads;
constexpr int kStageDevices = 64;
struct StagePool {
  std::mutex mu;
  int nbuf = 0;
  void *buf[kStageBufs] = {};
  cudaEvent_t ev[kStageBufs] = {};
};
static StagePool g_stage_pool[kStageDevices];  // one per device, made on first use

struct StageJob {
  int kind;              // 0: H2D copy, 2: D2H copy
  void *dst;
  const void *src;
  size_t bytes;
};

// Runs the jobs on the staging threads.  H2D sources are fully read and D2H
// destinations fully written when this returns (the H2D DMAs may still be in
// flight).
cudaError_t run_stage_jobs(const std::vector<StageJob> &jobs, cudaStream_t s) {
  if (jobs.empty()) return cudaSuccess;
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return ce;
  if (dev < 0 || dev >= kStageDevices) return cudaErrorInvalidDevice;
  StagePool &g_stage = g_stage_pool[dev];
  std::lock_guard<std::mutex> lk(g_stage.mu);
  if (g_stage.nbuf == 0) {
    for (int b = 0; b < kStageBufs; ++b) {
      if (cudaHostAlloc(&g_stage.buf[b], kStageBytes, cudaHostAllocPortable) != cudaSuccess ||
          cudaEventCreateWithFlags(&g_stage.ev[b], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (g_stage.buf[b]) cudaFreeHost(g_stage.buf[b]);
        g_stage.buf[b] = nullptr;
        break;
      }
      cudaEventRecord(g_stage.ev[b], s);  // a first wait returns at once
      g_stage.nbuf = b + 1;
    }
    if (g_stage.nbuf < 2) return cudaErrorMemoryAllocation;
  }
  const long long hw = std::max(2u, std::thread::hardware_concurrency());
  const int nth = (int)std::min({(long long)g_stage.nbuf / 2, hw, (long long)jobs.size()});
  std::atomic<long long> next{0};
  std::atomic<int> failed{(int)cudaSuccess};
  auto worker = [&](int t) {
    if (cudaSetDevice(dev) != cudaSuccess) {
      failed = (int)cudaErrorInvalidDevice;
      return;
    }
    for (int turn = 0;; ++turn) {
      const long long j = next++;
      if (j >= (long long)jobs.size() || failed != (int)cudaSuccess) break;
      const StageJob &job = jobs[j];
      const int b = 2 * t + (turn & 1);
      char *buf = static_cast<char *>(g_stage.buf[b]);
      cudaError_t e = cudaEventSynchronize(g_stage.ev[b]);  // its last DMA is done
      if (e == cudaSuccess && job.kind == 0) {
        stage_copy_in(buf, job.src, job.bytes);
        e = cudaMemcpyAsync(job.dst, buf, job.bytes, cudaMemcpyHostToDevice, s);
      } else if (e == cudaSuccess && job.kind == 2) {
        e = cudaMemcpyAsync(buf, job.src, job.bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaEventRecord(g_stage.ev[b], s);
        if (e == cudaSuccess) e = cudaEventSynchronize(g_stage.ev[b]);
        if (e == cudaSuccess) std::memcpy(job.dst, buf, job.bytes);
      }
      if (e == cudaSuccess) e = cudaEventRecord(g_stage.ev[b], s);
      if (e != cudaSuccess) {
        failed = (int)e;
        break;
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nth; ++t) th.emplace_back(worker, t);
  worker(0);
  for (auto &x : th) x.join();
  return (cudaError_t)failed.load();
}

// Copy jobs of at most `chunk` (<= kStageBytes) bytes for one array (kind 0:
// H2D, 2: D2H).
void add_copy_jobs(std::vector<StageJob> &jobs, int kind, void *dst, const void *src,
                   size_t bytes, size_t chunk = kStageBytes) {
  chunk = std::min(chunk, kStageBytes);
  for (size_t off = 0; off < bytes; off += chunk) {
    StageJob j{};
    j.kind = kind;
    j.dst = static_cast<char *>(dst) + off;
    j.src = static_cast<const char *>(src) + off;
    j.bytes = std::min(chunk, bytes - off);
    jobs.push_back(j);
  }
}

// Staged host -> device copy of one array.
cudaError_t upload(void *dst, const void *src, size_t bytes, cudaStream_t s) {
  if (bytes < 2 * kStageBytes) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  std::vector<StageJob> jobs;
  add_copy_jobs(jobs, 0, dst, src, bytes);
  return run_stage_jobs(jobs, s);
}

// Staged device -> host copy into caller (pageable) memory; synchronous.
// Arrays from 512 KiB on are cut into at least eight chunks, so that the
// copies out of the pinned buffers (and the first-touch page faults of a
// fresh destination) run on several host threads.
cudaError_t download(void *dst, const void *src, size_t bytes, cudaStream_t s) {
  if (bytes < (512u << 10)) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
    return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
  }
  std::vector<StageJob> jobs;
  const size_t chunk = std::max<size_t>(64u << 10, (bytes / 8 + 4095) / 4096 * 4096);
  add_copy_jobs(jobs, 2, dst, const_cast<void *>(src), bytes, chunk);
  cudaError_t e = cudaStreamSynchronize(s);  // the data is complete on the device
  return e == cudaSuccess ? run_stage_jobs(jobs, s) : e;
}

// Every ring slot of halo columns N .. N + n_ext - 1 of network 0 := the
// given host phases (the partition's part of init_buffer_kernel,
// leviathan_kernel.cu:79-90).  Synchronous.
int fill_ext_columns(LevEngine *h, int n_ext, const float *theta_ext) {
  const NetDesc &nd = h->h_nets[0];
  float *d_tmp = nullptr;
  LEV_TRY_CUDA(cudaMalloc(reinterpret_cast<void **>(&d_tmp), sizeof(float) * n_ext));
  cudaError_t e = cudaMemcpyAsync(d_tmp, theta_ext, sizeof(float) * n_ext,
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    const long long total = (long long)nd.bsi * n_ext;
    int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    ring_fill_kernel<<<blocks, 256, 0, h->stream>>>(
        d_tmp, h->d_ring + nd.ring_off, n_ext, nd.Np, nd.bsi, nd.N, 1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d_tmp);
  if (e != cudaSuccess)
    return fail(LEV_ERR_CUDA, std::string("halo ring fill: ") + cudaGetErrorString(e));
  return LEV_OK;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
      .count();
}

int create_impl(LevEngine **out, int num_nets, const int32_t *Ns,
                const int32_t *mds, const int32_t *rp_cat,
                const int32_t *col_cat, const uint8_t *d_cat,
                const float *w_cat, const float *th_cat,
                const float *thh_cat, const float *om_cat,
                const LevParams *params, int math_mode, int n_ext = 0,
                const float *theta_ext = nullptr) {
  // n_ext > 0 (one network only): ring columns N .. N + n_ext - 1 hold the
  // phases of halo nodes of a partition (lev_part.cuh), initially theta_ext;
  // col_idx may then address them
  if (!out) return fail(LEV_ERR_ARG, "out is null");
  if (n_ext < 0 || (n_ext > 0 && (num_nets != 1 || !theta_ext)))
    return fail(LEV_ERR_ARG, "halo columns need one network and their phases");
  *out = nullptr;
  if (num_nets < 1) return fail(LEV_ERR_ARG, "num_nets must be >= 1");
  if (!Ns || !mds || !rp_cat || !th_cat || !thh_cat || !om_cat)
    return fail(LEV_ERR_ARG, "null array argument");
  if (math_mode != LEV_MATH_REFERENCE && math_mode != LEV_MATH_ACCURATE)
    return fail(LEV_ERR_ARG, "math_mode must be 0 (reference) or 1");

  // ---- scalar arguments and sizes from the ends of row_ptr, before any
  // device work: the edge arrays then start moving to the device at once,
  // while a helper thread lays out the engine (a pass over row_ptr that also
  // checks it never decreases) and sets up its kernels
  long long e_total = 0, s_total = 0;
  {
    long long ro = 0;
    for (int n = 0; n < num_nets; ++n) {
      const int N = Ns[n], md = mds[n];
      if (N < 1 || N >= (1 << 24))
        return fail(LEV_ERR_ARG, "network " + std::to_string(n) +
                                     ": N must be in [1, 2^24), got " + std::to_string(N));
      if (md < 0 || md > 255)
        return fail(LEV_ERR_ARG, "network " + std::to_string(n) +
                                     ": max_delay must be in [0,255] (uint8 delays), got " +
                                     std::to_string(md));
      if (rp_cat[ro] != 0)
        return fail(LEV_ERR_ARG, "network " + std::to_string(n) + ": row_ptr[0] must be 0");
      const long long E = rp_cat[ro + N];
      if (E < 0)
        return fail(LEV_ERR_ARG, "network " + std::to_string(n) + ": row_ptr[N] is negative");
      LevParams p;
      if (params) p = params[n]; else lev_default_params(&p);
      const int prc = check_params(p);
      if (prc != LEV_OK) return prc;
      e_total += E;
      s_total += (N + 31) / 32;
      ro += N + 1;
    }
  }
  if (e_total > 0 && (!col_cat || !d_cat || !w_cat))
    return fail(LEV_ERR_ARG, "null edge array argument");

  const auto t_start = std::chrono::steady_clock::now();
  double t_mark = 0.0;
  LevEngine *h = new LevEngine();
  auto lap = [&]() {
    const double t = ms_since(t_start), d = t - t_mark;
    t_mark = t;
    return d;
  };
  h->num_nets = num_nets;
  h->math_mode = math_mode;
  h->h_nets.resize(num_nets);
  h->net_E.resize(num_nets);
  cudaError_t ce = cudaGetDevice(&h->device);
  if (ce != cudaSuccess) {
    delete h;
    return fail(LEV_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(ce));
  }
  ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) {
    delete h;
    return fail(LEV_ERR_CUDA, std::string("cudaStreamCreate failed: ") +
                                  cudaGetErrorString(ce));
  }
  // the temporary device buffer: col [E] | weights [E] | delays [E] |
  // slice -> network [slices] | error word
  char *tmp = nullptr;
  auto cleanup_fail = [&](int code, const std::string &msg) {
    cudaStreamSynchronize(h->stream);
    if (tmp) cudaFreeAsync(tmp, h->stream);
    cudaStreamSynchronize(h->stream);
    free_engine(h);
    return fail(code, msg);
  };
  const long long E1 = std::max<long long>(e_total, 1);
  const size_t off_w = (size_t)(4 * E1 + 255) / 256 * 256;
  const size_t off_dl = off_w + (size_t)(4 * E1 + 255) / 256 * 256;
  const size_t off_sn = off_dl + (size_t)(E1 + 255) / 256 * 256;
  const size_t off_err = off_sn + (size_t)(4 * std::max<long long>(s_total, 1) + 255) / 256 * 256;
  {
    cudaMemPool_t pool = nullptr;
    cudaError_t e = engine_pool(h->device, &pool);
    if (e == cudaSuccess)
      e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&tmp), off_err + 256, pool,
                                  h->stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      tmp = nullptr;
      return cleanup_fail(LEV_ERR_NOMEM, std::string("device allocation of ") +
                                             std::to_string(off_err + 256) +
                                             " bytes failed: " + cudaGetErrorString(e));
    }
  }
  int *t_col = reinterpret_cast<int *>(tmp);
  float *t_w = reinterpret_cast<float *>(tmp + off_w);
  uint8_t *t_dl = reinterpret_cast<uint8_t *>(tmp + off_dl);
  int *t_sn = reinterpret_cast<int *>(tmp + off_sn);
  unsigned *t_err = reinterpret_cast<unsigned *>(tmp + off_err);
  double ms_device = lap();

  // ---- validate shapes and lay out the packed arrays (helper thread) -------
  long long node_off = 0, edge_off = 0, ring_off = 0, rp_off = 0;
  long long slices = 0, sl_total = 0;
  std::vector<long long> h_sl_off;
  std::vector<int> h_sl_len;
  int tiles = 0;
  std::vector<int> slice_net;
  std::vector<int> h_class_nets;
  std::vector<int2> h_tiles;
  auto layout = [&]() -> int {
    for (int n = 0; n < num_nets; ++n) {
      const int N = Ns[n], md = mds[n];
      if (N < 1 || N >= (1 << 24)) {
        return fail(LEV_ERR_ARG, "network " + std::to_string(n) +
                                     ": N must be in [1, 2^24), got " +
                                     std::to_string(N));
      }
      if (md < 0 || md > 255) {
        return fail(LEV_ERR_ARG, "network " + std::to_string(n) +
                                     ": max_delay must be in [0,255] (uint8 "
                                     "delays), got " + std::to_string(md));
      }
      const int32_t *rp = rp_cat + rp_off;
      if (rp[0] != 0) {
        return fail(LEV_ERR_ARG, "network " + std::to_string(n) +
                                     ": row_ptr[0] must be 0");
      }
      const long long E = rp[N];
      NetDesc &d = h->h_nets[n];
      std::memset(&d, 0, sizeof(d));
      d.node_off = node_off;
      d.edge_off = edge_off;
      d.ring_off = ring_off;
      d.rp_off = rp_off;
      d.N = N;
      if ((long long)N + n_ext >= (1LL << 24)) {
        return fail(LEV_ERR_ARG, "N plus halo nodes must be below 2^24");
      }
      d.Np = (N + n_ext + 31) / 32 * 32;
      d.bsi = md + 2;
      d.max_delay = md;
      d.ntiles = (N + kTile - 1) / kTile;
      d.part_off = tiles;
      d.tile_off = tiles;
      LevParams p;
      if (params) p = params[n]; else lev_default_params(&p);
      int rc = check_params(p);
      if (rc != LEV_OK) {
        return rc;
      }
      params_to_desc(p, &d);
      // ring gathers index a network's ring with 32-bit slot * Np + col
      if ((unsigned long long)ring_slots(d.bsi) * (unsigned long long)d.Np >= (1ull << 32)) {
        return fail(LEV_ERR_ARG, "network " + std::to_string(n) +
                                     ": (max_delay + 2) * N must be below 2^32");
      }
      // SELL-32 slices: entry k of row i at sl_off[i/32] + 32k + i%32; the
      // same pass checks that row_ptr never decreases
      d.slice_base = slices;
      const int nsl = (N + 31) / 32;
      h_sl_off.resize((size_t)(slices + nsl));
      h_sl_len.resize((size_t)(slices + nsl));
      int neg = 0;
      for (int q = 0; q < nsl; ++q) {
        const int s0 = 32 * q, s1 = std::min(N, s0 + 32);
        int len = 0, lo = 0;
        for (int i = s0; i < s1; ++i) {
          const int deg = rp[i + 1] - rp[i];
          len = std::max(len, deg);
          lo = std::min(lo, deg);
        }
        neg |= (lo < 0);
        h_sl_off[(size_t)(slices + q)] = sl_total;
        h_sl_len[(size_t)(slices + q)] = len;
        sl_total += 32LL * len;
      }
      slices += nsl;
      if (neg) {
        int i = 0;
        while (rp[i + 1] >= rp[i]) ++i;
        return fail(LEV_ERR_ARG, "network " + std::to_string(n) +
                                     ": row_ptr is decreasing at row " + std::to_string(i));
      }
      h->net_E[n] = E;
      node_off += N;
      edge_off += E;
      ring_off += (long long)ring_slots(d.bsi) * d.Np;
      rp_off += N + 1;
      tiles += d.ntiles;
    }
    h_sl_off.push_back(sl_total);  // one more entry: the end of the last slice
    slice_net.assign((size_t)slices, 0);
    for (int n = 0; n < num_nets; ++n) {
      const NetDesc &d = h->h_nets[n];
      const long long ns = (d.N + 31) / 32;
      for (long long k = 0; k < ns; ++k) slice_net[(size_t)(d.slice_base + k)] = n;
    }
    h->total_nodes = node_off;
    h->total_edges = edge_off;
    h->num_slices = slices;
    h->sl_total = sl_total;
    h->rp_total = rp_off;
    h->ring_floats = ring_off;
    h->total_tiles = tiles;

    // Tile list grouped by degree class (class = mean SELL slice length of the
    // network); within a class, networks keep their order.
    std::vector<int> net_class(num_nets);
    for (int n = 0; n < num_nets; ++n) {
      const NetDesc &d = h->h_nets[n];
      const long long s0 = d.slice_base, ns = (d.N + 31) / 32;
      double sum = 0.0;
      for (long long s = s0; s < s0 + ns; ++s) sum += h_sl_len[s];
      const double mean = ns ? sum / ns : 0.0;
      net_class[n] = degree_class(mean);
      TileClass &tc = h->classes[net_class[n]];
      tc.mean_len = (tc.mean_len * tc.ntiles + mean * d.ntiles) /
                    std::max(1, tc.ntiles + d.ntiles);
      tc.ntiles += d.ntiles;
      tc.edges += h->net_E[n];
    }
    for (int c = 1; c < kNumClasses; ++c)
      h->classes[c].tile_off = h->classes[c - 1].tile_off + h->classes[c - 1].ntiles;
    for (int c = 0; c < kNumClasses; ++c) {
      h->classes[c].net_off = (int)h_class_nets.size();
      for (int n = 0; n < num_nets; ++n)
        if (net_class[n] == c) h_class_nets.push_back(n);
      h->classes[c].nnets = (int)h_class_nets.size() - h->classes[c].net_off;
    }
    h_tiles.assign(tiles, make_int2(0, 0));
    {
      int fill[kNumClasses];
      for (int c = 0; c < kNumClasses; ++c) fill[c] = h->classes[c].tile_off;
      for (int n = 0; n < num_nets; ++n) {
        const NetDesc &d = h->h_nets[n];
        for (int t = 0; t < d.ntiles; ++t)
          h_tiles[fill[net_class[n]]++] = make_int2(n, t * kTile);
      }
    }
    {
      // remembered choices of earlier engines with a similar class
      std::lock_guard<std::mutex> lk(g_tune_mu);
      for (int c = 0; c < kNumClasses; ++c) {
        auto it = g_tune_cache.find(tune_key(h->classes[c], c));
        h->classes[c].variant = (it != g_tune_cache.end()) ? it->second : 0;
        auto ip = g_pair_cache.find(tune_key(h->classes[c], c));
        h->classes[c].pair_variant = (ip != g_pair_cache.end()) ? ip->second : 0;
      }
    }

    return LEV_OK;
  };
  int lrc = LEV_OK;
  std::string lmsg;
  std::thread helper([&] {
    auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = cudaSetDevice(h->device);
    lrc = e == cudaSuccess ? layout()
                           : fail(LEV_ERR_CUDA, std::string("cudaSetDevice failed: ") +
                                                    cudaGetErrorString(e));
    h->create_ms[0] = ms_since(t0);
    t0 = std::chrono::steady_clock::now();
    if (lrc == LEV_OK) lrc = prepare_step_kernels();
    if (lrc == LEV_OK) {
      setup_cluster(h, h_sl_off, h_sl_len);
      lrc = setup_grid(h, h_sl_off, h_sl_len);
    }
    if (lrc == LEV_OK) {
      int nbusy = 0;
      for (int c = 0; c < kNumClasses; ++c) nbusy += h->classes[c].ntiles > 0;
      if (nbusy > 1) {
        bool ok = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) == cudaSuccess;
        for (int c = 0; c < kNumClasses && ok; ++c)
          ok = cudaStreamCreateWithFlags(&h->class_stream[c], cudaStreamNonBlocking) ==
                   cudaSuccess &&
               cudaEventCreateWithFlags(&h->ev_join[c], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) lrc = fail(LEV_ERR_CUDA, "class streams: creation failed");
      }
    }
    h->create_ms[1] = ms_since(t0);
    if (lrc != LEV_OK) lmsg = g_last_error;
  });
  // ---- meanwhile: the edge arrays as they are, through the staging buffers
  cudaError_t se;
  {
    std::vector<StageJob> jobs;
    add_copy_jobs(jobs, 0, t_col, col_cat, sizeof(int32_t) * e_total);
    add_copy_jobs(jobs, 0, t_w, w_cat, sizeof(float) * e_total);
    add_copy_jobs(jobs, 0, t_dl, d_cat, sizeof(uint8_t) * e_total);
    se = run_stage_jobs(jobs, h->stream);
  }
  helper.join();
  double ms_staged = lap();
  if (lrc != LEV_OK) return cleanup_fail(lrc, lmsg);
  if (se != cudaSuccess)
    return cleanup_fail(LEV_ERR_CUDA, std::string("upload failed: ") + cudaGetErrorString(se));
  if (edge_off != e_total || slices != s_total)
    return cleanup_fail(LEV_ERR_ARG, "row_ptr changed during creation");

  int rc = LEV_OK;
  // every array sized here in one device allocation (256-byte aligned
  // parts): one cudaMalloc instead of one per array
  {
    struct Part { void **p; size_t bytes; };
    const Part parts[] = {
        {(void **)&h->d_nets, sizeof(NetDesc) * num_nets},
        {(void **)&h->d_st, sizeof(NetState) * num_nets},
        {(void **)&h->d_tiles, sizeof(int2) * std::max(tiles, 1)},
        {(void **)&h->d_row_ptr, sizeof(int) * rp_off},
        {(void **)&h->d_sl_off, sizeof(long long) * std::max<long long>(slices, 1)},
        {(void **)&h->d_sl_len, sizeof(int) * std::max<long long>(slices, 1)},
        {(void **)&h->d_sl_cd, sizeof(uint32_t) * std::max<long long>(sl_total, 1)},
        {(void **)&h->d_sl_w, sizeof(float) * std::max<long long>(sl_total, 1)},
        {(void **)&h->d_theta, sizeof(float) * node_off},
        {(void **)&h->d_theta_hat, sizeof(float) * node_off},
        {(void **)&h->d_omega, sizeof(float) * node_off},
        {(void **)&h->d_omega_hat, sizeof(float) * node_off},
        {(void **)&h->d_ring, sizeof(float) * ring_off},
        {(void **)&h->d_part, sizeof(float2) * std::max(tiles, 1)},
        {(void **)&h->d_rhist, sizeof(float) * h->block_len * num_nets},
        {(void **)&h->d_class_nets, sizeof(int) * num_nets},
        {(void **)&h->d_pend, sizeof(float2) * node_off},
    };
    size_t total = 0;
    for (const Part &q : parts) total += (q.bytes + 255) / 256 * 256;
    {
      cudaMemPool_t pool = nullptr;
      cudaError_t e = engine_pool(h->device, &pool);
      if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&h->slab, total, pool, h->stream);
      if (e != cudaSuccess) {
        cudaGetLastError();
        h->slab = nullptr;
        rc = fail(LEV_ERR_NOMEM, std::string("device allocation of ") + std::to_string(total) +
                                     " bytes failed: " + cudaGetErrorString(e));
      }
    }
    if (rc == LEV_OK) {
      h->slab_bytes = total;
      h->vram += total;
      char *c = static_cast<char *>(h->slab);
      for (const Part &q : parts) {
        *q.p = c;
        c += (q.bytes + 255) / 256 * 256;
      }
    }
  }
  if (rc != LEV_OK) return cleanup_fail(rc, g_last_error);
  ms_device += lap();
  h->h_rmap = mapped_alloc((size_t)num_nets);
  ce = h->h_rmap ? cudaSuccess : cudaErrorMemoryAllocation;
  if (ce == cudaSuccess)
    ce = cudaHostGetDevicePointer(reinterpret_cast<void **>(&h->d_rmap),
                                  h->h_rmap, 0);
  if (ce != cudaSuccess)
    return cleanup_fail(LEV_ERR_CUDA, std::string("mapped host buffer: ") +
                                          cudaGetErrorString(ce));

  h->create_ms[2] = ms_device;
  h->create_ms[3] = lap();
  // ---- uploads: the node arrays through the staging buffers; the edge
  // arrays, already on the device, are packed into SELL-32 and validated by
  // sell_pack_kernel
  std::vector<NetState> st(num_nets);
  for (int n = 0; n < num_nets; ++n) {
    std::memset(&st[n], 0, sizeof(NetState));
    LevParams p;
    if (params) p = params[n]; else lev_default_params(&p);
    st[n].g = p.g;
  }
  {
    cudaError_t e = cudaMemsetAsync(h->d_ring, 0, sizeof(float) * std::max<long long>(ring_off, 1),
                                    h->stream);
    const struct { void *dst; const void *src; size_t bytes; } small[] = {
        {h->d_nets, h->h_nets.data(), sizeof(NetDesc) * num_nets},
        {h->d_tiles, h_tiles.data(), sizeof(int2) * tiles},
        {h->d_class_nets, h_class_nets.data(), sizeof(int) * num_nets},
        {h->d_st, st.data(), sizeof(NetState) * num_nets},
        {h->d_sl_off, h_sl_off.data(), sizeof(long long) * slices},
        {h->d_sl_len, h_sl_len.data(), sizeof(int) * slices},
        {t_sn, slice_net.data(), sizeof(int) * slices},
    };
    if (e == cudaSuccess) e = cudaMemsetAsync(t_err, 0, sizeof(unsigned), h->stream);
    for (const auto &c : small)
      if (e == cudaSuccess && c.bytes > 0)
        e = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess)
      return cleanup_fail(LEV_ERR_CUDA, std::string("upload failed: ") + cudaGetErrorString(e));
  }
  h->create_ms[4] = lap();
  {
    std::vector<StageJob> jobs;
    add_copy_jobs(jobs, 0, h->d_row_ptr, rp_cat, sizeof(int32_t) * rp_off);
    add_copy_jobs(jobs, 0, h->d_theta, th_cat, sizeof(float) * node_off);
    add_copy_jobs(jobs, 0, h->d_theta_hat, thh_cat, sizeof(float) * node_off);
    add_copy_jobs(jobs, 0, h->d_omega, om_cat, sizeof(float) * node_off);
    cudaError_t e = run_stage_jobs(jobs, h->stream);
    if (e != cudaSuccess)
      return cleanup_fail(LEV_ERR_CUDA, std::string("upload failed: ") + cudaGetErrorString(e));
    h->create_ms[5] = ms_staged + lap();
    // omega_hat starts as omega (leviathan_kernel.cu:350)
    e = cudaMemcpyAsync(h->d_omega_hat, h->d_omega, sizeof(float) * node_off,
                        cudaMemcpyDeviceToDevice, h->stream);
    if (e != cudaSuccess)
      return cleanup_fail(LEV_ERR_CUDA, std::string("upload failed: ") + cudaGetErrorString(e));
    if (slices > 0) {
      const int blocks = (int)std::min<long long>((slices + 7) / 8, 148LL * 16);
      sell_pack_kernel<<<blocks, 256, 0, h->stream>>>(
          h->d_nets, t_sn, slices, h->d_sl_off, h->d_sl_len, h->d_row_ptr, t_col, t_dl, t_w,
          n_ext, h->d_sl_cd, h->d_sl_w, t_err);
      e = cudaGetLastError();
      if (e != cudaSuccess)
        return cleanup_fail(LEV_ERR_CUDA, std::string("SELL packing: ") + cudaGetErrorString(e));
    }
  }
  for (int n = 0; n < num_nets; ++n) {
    int r2 = launch_fill(h, n);
    if (r2 != LEV_OK) return cleanup_fail(r2, g_last_error);
  }
  h->create_ms[6] = lap();
  {
    // waits for the DMAs and the packing (pageable destination)
    unsigned herr = 0u;
    cudaError_t e = cudaMemcpyAsync(&herr, t_err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                    h->stream);
    if (e != cudaSuccess)
      return cleanup_fail(LEV_ERR_CUDA, std::string("upload failed: ") + cudaGetErrorString(e));
    if (herr & 1u) return cleanup_fail(LEV_ERR_ARG, "col_idx out of range [0, N)");
    if (herr & 2u) return cleanup_fail(LEV_ERR_ARG, "delay larger than max_delay");
    h->pair_ok = !(herr & 4u);
    cudaFreeAsync(tmp, h->stream);  // back to the engine pool
    tmp = nullptr;
  }
  if (n_ext > 0) {
    int r2 = fill_ext_columns(h, n_ext, theta_ext);
    if (r2 != LEV_OK) return cleanup_fail(r2, g_last_error);
  }
  ce = cudaStreamSynchronize(h->stream);
  if (ce != cudaSuccess)
    return cleanup_fail(LEV_ERR_CUDA,
                        std::string("engine init failed: ") + cudaGetErrorString(ce));
  h->create_ms[7] = lap();
  *out = h;
  return LEV_OK;
}

}  // namespace

// ===========================================================================
// lev_* ABI
// ===========================================================================
extern "C" {

const char *lev_last_error(void) { return g_last_error.c_str(); }

const char *lev_version(void) { return "leviathan_b200 1.0 (sm_100a)"; }

void lev_default_params(LevParams *p) {
  if (!p) return;
  // leviathan_kernel.cu:282-296 and the literal 1.5 at :433
  p->eta = 0.01f;
  p->lam = 0.001f;
  p->gamma = 0.05f;
  p->alpha_eps = 0.1f;
  p->kappa_w = 0.01f;
  p->w_min = 0.0f;
  p->w_max = 2.0f;
  p->g = 1.5f;
  p->r0 = 0.5f;
  p->beta = 0.01f;
  p->mu = 0.01f;
  p->g_rest = 1.5f;
  p->g_min = 0.1f;
  p->g_max = 5.0f;
  p->gain_controller = 1;
  p->reserved = 0;
}

int lev_create(LevEngine **out, int32_t N, int32_t max_delay,
               const int32_t *row_ptr, const int32_t *col_idx,
               const uint8_t *delays, const float *weights,
               const float *theta, const float *theta_hat,
               const float *omega, const LevParams *params,
               int32_t math_mode) {
  return create_impl(out, 1, &N, &max_delay, row_ptr, col_idx, delays,
                     weights, theta, theta_hat, omega, params, math_mode);
}

int lev_batch_create(LevEngine **out, int32_t num_nets, const int32_t *N,
                     const int32_t *max_delay, const int32_t *row_ptr_cat,
                     const int32_t *col_idx_cat, const uint8_t *delays_cat,
                     const float *weights_cat, const float *theta_cat,
                     const float *theta_hat_cat, const float *omega_cat,
                     const LevParams *params, int32_t math_mode) {
  return create_impl(out, num_nets, N, max_delay, row_ptr_cat, col_idx_cat,
                     delays_cat, weights_cat, theta_cat, theta_hat_cat,
                     omega_cat, params, math_mode);
}

int lev_destroy(LevEngine *h) {
  if (!h) return LEV_OK;
  DeviceScope ds(h->device);
  cudaStreamSynchronize(h->stream);
  free_engine(h);
  return LEV_OK;
}

int lev_num_nets(const LevEngine *h, int32_t *out) {
  if (!h || !out) return fail(LEV_ERR_ARG, "null argument");
  *out = h->num_nets;
  return LEV_OK;
}

int lev_total_nodes(const LevEngine *h, int64_t *out) {
  if (!h || !out) return fail(LEV_ERR_ARG, "null argument");
  *out = h->total_nodes;
  return LEV_OK;
}

int lev_total_edges(const LevEngine *h, int64_t *out) {
  if (!h || !out) return fail(LEV_ERR_ARG, "null argument");
  *out = h->total_edges;
  return LEV_OK;
}

int lev_net_shape(const LevEngine *h, int32_t net, int32_t *N, int64_t *E,
                  int32_t *max_delay) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (net < 0 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  if (N) *N = h->h_nets[net].N;
  if (E) *E = h->net_E[net];
  if (max_delay) *max_delay = h->h_nets[net].max_delay;
  return LEV_OK;
}

int lev_step(LevEngine *h, float dt, float *r_out) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (h->part) return fail(LEV_ERR_STATE, "partition engine: step with lev_part_step_begin / lev_part_step_end");
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  DeviceScope ds(h->device);
  StepArgs a = make_args(h, dt, nullptr, 0, h->d_rmap);
  int rc = LEV_OK;
  uint32_t dbits;
  std::memcpy(&dbits, &dt, 4);
  if (pairs_all(h)) {
    if (h->spec && h->spec_dt == dbits) {
      // the speculative step t+1: its integrate, then the weights it wrote
      a.thh2 = h->d_thh_spec;
      a.omh2 = h->d_omh_spec;
      a.reverse = h->sweep;
      h->sweep ^= 1;
      for (int c = 0; c < kNumClasses && rc == LEV_OK; ++c) rc = launch_pair_class(h, c, a, 1);
      h->spec = false;
      if (rc != LEV_OK) return rc;
      std::swap(h->d_sl_w, h->d_w_spec);
      h->w_flip ^= 1;
    } else {
      h->spec = false;
      if (!h->d_w_spec) {
        // one block from the engine pool (a driver allocation of this size
        // costs milliseconds; the pool usually has it from earlier engines)
        const size_t nw = ((size_t)std::max<long long>(h->sl_total, 1) + 63) / 64 * 64;
        const size_t nn = ((size_t)std::max<long long>(h->total_nodes, 1) + 63) / 64 * 64;
        const size_t bytes = sizeof(float) * (nw + 2 * nn);
        cudaMemPool_t pool = nullptr;
        cudaError_t e = engine_pool(h->device, &pool);
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&h->spec_block, bytes, pool, h->stream);
        if (e != cudaSuccess) {
          cudaGetLastError();
          h->spec_block = nullptr;
          return fail(LEV_ERR_NOMEM, std::string("device allocation of ") +
                                         std::to_string(bytes) + " bytes failed: " +
                                         cudaGetErrorString(e));
        }
        h->spec_bytes = bytes;
        h->vram += bytes;
        float *f = static_cast<float *>(h->spec_block);
        h->d_w_spec = f;
        h->d_thh_spec = f + nw;
        h->d_omh_spec = f + nw + nn;
        // padding entries (never written by a walk) as in the live buffer
        LEV_TRY_CUDA(cudaMemcpyAsync(h->d_w_spec, h->d_sl_w,
                                     sizeof(float) * std::max<long long>(h->sl_total, 1),
                                     cudaMemcpyDeviceToDevice, h->stream));
      }
      // step t in full and step t+1 up to its integrate, into the spec buffers
      a.w2 = h->d_w_spec;
      a.thh2 = h->d_thh_spec;
      a.omh2 = h->d_omh_spec;
      a.reverse = h->sweep;
      h->sweep ^= 1;
      for (int c = 0; c < kNumClasses && rc == LEV_OK; ++c) rc = launch_pair_class(h, c, a, 0);
      if (rc != LEV_OK) return rc;
      h->spec = true;
      h->spec_dt = dbits;
    }
  } else {
    rc = launch_step(h, a);
    if (rc != LEV_OK) return rc;
  }
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  if (r_out) {
    const volatile float *src = h->h_rmap;
    for (int n = 0; n < h->num_nets; ++n) r_out[n] = src[n];
  }
  return LEV_OK;
}

int lev_step_n(LevEngine *h, float dt, int32_t n, float *r_out) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (h->part) return fail(LEV_ERR_STATE, "partition engine: step with lev_part_step_begin / lev_part_step_end");
  if (n < 0) return fail(LEV_ERR_ARG, "n must be >= 0");
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  if (n == 0) return LEV_OK;
  DeviceScope ds(h->device);
  float *stage = nullptr;
  if (r_out) {
    const size_t need = (size_t)n * h->num_nets;
    if (h->h_rstage_len < need) {
      if (h->h_rstage) cudaFreeHost(h->h_rstage);
      h->h_rstage = nullptr;
      h->h_rstage_len = 0;
      LEV_TRY_CUDA(cudaMallocHost(reinterpret_cast<void **>(&h->h_rstage),
                                  sizeof(float) * need));
      h->h_rstage_len = need;
    }
    stage = h->h_rstage;
  }
  int rc = enqueue_steps(h, dt, n, stage);
  if (rc != LEV_OK) return rc;
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  rc = check_grid_error(h);
  if (rc != LEV_OK) return rc;
  if (r_out)
    std::memcpy(r_out, stage, sizeof(float) * (size_t)n * h->num_nets);
  return LEV_OK;
}

int lev_step_n_async(LevEngine *h, float dt, int32_t n) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (h->part) return fail(LEV_ERR_STATE, "partition engine: step with lev_part_step_begin / lev_part_step_end");
  if (n < 0) return fail(LEV_ERR_ARG, "n must be >= 0");
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  DeviceScope ds(h->device);
  return enqueue_steps(h, dt, n, nullptr);
}

int lev_sync(LevEngine *h) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  DeviceScope ds(h->device);
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return check_grid_error(h);
}

int lev_get_stream(LevEngine *h, void **stream) {
  if (!h || !stream) return fail(LEV_ERR_ARG, "null argument");
  *stream = reinterpret_cast<void *>(h->stream);
  return LEV_OK;
}

static int copy_nodes(LevEngine *h, float *dst_host, const float *src_dev,
                      long long off, long long count) {
  LEV_TRY_CUDA(download(dst_host, src_dev + off, sizeof(float) * count, h->stream));
  return LEV_OK;
}

static int upload_nodes(LevEngine *h, float *dst_dev, const float *src_host,
                        long long off, long long count) {
  LEV_TRY_CUDA(upload(dst_dev + off, src_host, sizeof(float) * count, h->stream));
  return LEV_OK;
}

int lev_get_theta(LevEngine *h, float *theta_out) {
  if (!h || !theta_out) return fail(LEV_ERR_ARG, "null argument");
  DeviceScope ds(h->device);
  return copy_nodes(h, theta_out, h->d_theta, 0, h->total_nodes);
}

int lev_get_theta_net(LevEngine *h, int32_t net, float *theta_out) {
  if (!h || !theta_out) return fail(LEV_ERR_ARG, "null argument");
  if (net < 0 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  DeviceScope ds(h->device);
  const NetDesc &d = h->h_nets[net];
  return copy_nodes(h, theta_out, h->d_theta, d.node_off, d.N);
}

int lev_set_theta(LevEngine *h, const float *theta_in) {
  if (h) spec_drop(h);
  if (!h || !theta_in) return fail(LEV_ERR_ARG, "null argument");
  DeviceScope ds(h->device);
  int rc = upload_nodes(h, h->d_theta, theta_in, 0, h->total_nodes);
  for (int n = 0; n < h->num_nets && rc == LEV_OK; ++n) rc = launch_fill(h, n);
  if (rc != LEV_OK) return rc;
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return LEV_OK;
}

int lev_set_theta_net(LevEngine *h, int32_t net, const float *theta_in) {
  if (h) spec_drop(h);
  if (!h || !theta_in) return fail(LEV_ERR_ARG, "null argument");
  if (net < 0 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  DeviceScope ds(h->device);
  const NetDesc &d = h->h_nets[net];
  int rc = upload_nodes(h, h->d_theta, theta_in, d.node_off, d.N);
  if (rc == LEV_OK) rc = launch_fill(h, net);
  if (rc != LEV_OK) return rc;
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return LEV_OK;
}

// Weights between the caller's CSR order and the engine's SELL-32 layout,
// through a temporary device buffer in CSR order (mode 1: CSR -> SELL,
// mode 2: SELL -> CSR).
static int convert_weights(LevEngine *h, float *d_csr, int mode) {
  for (int n = 0; n < h->num_nets; ++n) {
    const NetDesc &d = h->h_nets[n];
    if (h->net_E[n] == 0) continue;
    int blocks = (int)std::min<long long>((d.N + 255) / 256, 148LL * 16);
    sell_convert_kernel<<<blocks, 256, 0, h->stream>>>(
        mode, h->d_row_ptr + d.rp_off, d.N, d.N, d.slice_base, h->d_sl_off,
        nullptr, nullptr, d_csr + d.edge_off, h->d_sl_cd, h->d_sl_w,
        d.max_delay, nullptr);
  }
  LEV_TRY_CUDA(cudaGetLastError());
  return LEV_OK;
}

int lev_get_weights(LevEngine *h, float *w_out) {
  if (!h || (!w_out && h->total_edges > 0))
    return fail(LEV_ERR_ARG, "null argument");
  DeviceScope ds(h->device);
  if (h->total_edges == 0) return LEV_OK;
  float *tmp = nullptr;
  LEV_TRY_CUDA(cudaMalloc(&tmp, sizeof(float) * h->total_edges));
  int rc = convert_weights(h, tmp, 2);
  if (rc == LEV_OK) rc = copy_nodes(h, w_out, tmp, 0, h->total_edges);
  cudaFree(tmp);
  return rc;
}

int lev_reset_weights(LevEngine *h, const float *w_in) {
  if (h) spec_drop(h);
  if (!h || (!w_in && h->total_edges > 0))
    return fail(LEV_ERR_ARG, "null argument");
  DeviceScope ds(h->device);
  if (h->total_edges == 0) return LEV_OK;
  float *tmp = nullptr;
  LEV_TRY_CUDA(cudaMalloc(&tmp, sizeof(float) * h->total_edges));
  int rc = upload_nodes(h, tmp, w_in, 0, h->total_edges);
  if (rc == LEV_OK) rc = convert_weights(h, tmp, 1);
  cudaError_t ce = cudaStreamSynchronize(h->stream);
  cudaFree(tmp);
  if (rc != LEV_OK) return rc;
  if (ce != cudaSuccess)
    return fail(LEV_ERR_CUDA, std::string("reset_weights: ") + cudaGetErrorString(ce));
  return LEV_OK;
}

int lev_selftest_wraps(uint64_t *mismatch_pm, uint64_t *mismatch_02) {
  unsigned long long *d = nullptr;
  LEV_TRY_CUDA(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
  unsigned long long hc[2] = {0, 0};
  cudaError_t e = cudaMemset(d, 0, sizeof(hc));
  if (e == cudaSuccess) {
    selftest_wraps_kernel<<<148 * 8, 256>>>(d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(hc, d, sizeof(hc), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess)
    return fail(LEV_ERR_CUDA, std::string("selftest: ") + cudaGetErrorString(e));
  if (mismatch_pm) *mismatch_pm = hc[0];
  if (mismatch_02) *mismatch_02 = hc[1];
  return LEV_OK;
}

int lev_get_predictor(LevEngine *h, float *theta_hat_out,
                      float *omega_hat_out) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  DeviceScope ds(h->device);
  int rc = LEV_OK;
  if (theta_hat_out)
    rc = copy_nodes(h, theta_hat_out, h->d_theta_hat, 0, h->total_nodes);
  if (rc == LEV_OK && omega_hat_out)
    rc = copy_nodes(h, omega_hat_out, h->d_omega_hat, 0, h->total_nodes);
  return rc;
}

int lev_set_predictor(LevEngine *h, const float *theta_hat_in,
                      const float *omega_hat_in) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  spec_drop(h);
  DeviceScope ds(h->device);
  int rc = LEV_OK;
  if (theta_hat_in)
    rc = upload_nodes(h, h->d_theta_hat, theta_hat_in, 0, h->total_nodes);
  if (rc == LEV_OK && omega_hat_in)
    rc = upload_nodes(h, h->d_omega_hat, omega_hat_in, 0, h->total_nodes);
  if (rc != LEV_OK) return rc;
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return LEV_OK;
}

int lev_get_omega(LevEngine *h, float *omega_out) {
  if (!h || !omega_out) return fail(LEV_ERR_ARG, "null argument");
  DeviceScope ds(h->device);
  return copy_nodes(h, omega_out, h->d_omega, 0, h->total_nodes);
}

int lev_set_omega(LevEngine *h, const float *omega_in) {
  if (h) spec_drop(h);
  if (!h || !omega_in) return fail(LEV_ERR_ARG, "null argument");
  DeviceScope ds(h->device);
  int rc = upload_nodes(h, h->d_omega, omega_in, 0, h->total_nodes);
  if (rc != LEV_OK) return rc;
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return LEV_OK;
}

int lev_get_ring(LevEngine *h, int32_t net, float *ring_out,
                 int32_t *buf_idx) {
  if (!h || !ring_out) return fail(LEV_ERR_ARG, "null argument");
  if (net < 0 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  DeviceScope ds(h->device);
  std::vector<NetState> st;
  int rc = read_states(h, st);
  if (rc != LEV_OK) return rc;
  const NetDesc &d = h->h_nets[net];
  std::vector<float> ri((size_t)ring_slots(d.bsi) * d.Np);
  LEV_TRY_CUDA(cudaMemcpyAsync(ri.data(), h->d_ring + d.ring_off,
                               sizeof(float) * ri.size(),
                               cudaMemcpyDeviceToHost, h->stream));
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  const int bs = d.max_delay + 1;
  const int cur = st[net].cur, rb = st[net].rbuf;
  for (int m = 0; m <= d.max_delay; ++m) {
    const int si = ((cur - m) % d.bsi + d.bsi) % d.bsi;
    const int sr = ((rb - m) % bs + bs) % bs;
    for (int j = 0; j < d.N; ++j) ring_out[(size_t)j * bs + sr] = ri[ring_pos(si, j, d.Np)];
  }
  if (buf_idx) *buf_idx = rb;
  return LEV_OK;
}

int lev_set_ring(LevEngine *h, int32_t net, const float *ring_in,
                 int32_t buf_idx) {
  if (h) spec_drop(h);
  if (!h || !ring_in) return fail(LEV_ERR_ARG, "null argument");
  if (net < 0 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  const NetDesc &d = h->h_nets[net];
  const int bs = d.max_delay + 1;
  if (buf_idx < 0 || buf_idx >= bs)
    return fail(LEV_ERR_ARG, "buf_idx out of range [0, max_delay]");
  DeviceScope ds(h->device);
  std::vector<NetState> st;
  int rc = read_states(h, st);
  if (rc != LEV_OK) return rc;
  std::vector<float> ri((size_t)ring_slots(d.bsi) * d.Np, 0.0f);
  const int cur = st[net].cur;
  for (int m = 0; m <= d.max_delay; ++m) {
    const int si = ((cur - m) % d.bsi + d.bsi) % d.bsi;
    const int sr = ((buf_idx - m) % bs + bs) % bs;
    for (int j = 0; j < d.N; ++j) ri[ring_pos(si, j, d.Np)] = ring_in[(size_t)j * bs + sr];
  }
  LEV_TRY_CUDA(cudaMemcpyAsync(h->d_ring + d.ring_off, ri.data(),
                               sizeof(float) * ri.size(),
                               cudaMemcpyHostToDevice, h->stream));
  NetState s = st[net];
  s.rbuf = buf_idx;
  return write_state(h, net, s);
}

int lev_get_step_count(LevEngine *h, int32_t net, int64_t *t) {
  if (!h || !t) return fail(LEV_ERR_ARG, "null argument");
  if (net < 0 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  DeviceScope ds(h->device);
  std::vector<NetState> st;
  int rc = read_states(h, st);
  if (rc != LEV_OK) return rc;
  *t = st[net].t;
  return LEV_OK;
}

int lev_set_gain(LevEngine *h, int32_t net, float g) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (net < -1 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  DeviceScope ds(h->device);
  std::vector<NetState> st;
  int rc = read_states(h, st);
  if (rc != LEV_OK) return rc;
  for (int n = 0; n < h->num_nets; ++n) {
    if (net >= 0 && n != net) continue;
    st[n].g = g;
  }
  LEV_TRY_CUDA(cudaMemcpyAsync(h->d_st, st.data(),
                               sizeof(NetState) * h->num_nets,
                               cudaMemcpyHostToDevice, h->stream));
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return LEV_OK;
}

int lev_get_gain(LevEngine *h, int32_t net, float *g) {
  if (!h || !g) return fail(LEV_ERR_ARG, "null argument");
  if (net < 0 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  DeviceScope ds(h->device);
  std::vector<NetState> st;
  int rc = read_states(h, st);
  if (rc != LEV_OK) return rc;
  *g = st[net].g;
  return LEV_OK;
}

int lev_get_r(LevEngine *h, int32_t net, float *r) {
  if (!h || !r) return fail(LEV_ERR_ARG, "null argument");
  if (net < 0 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  DeviceScope ds(h->device);
  std::vector<NetState> st;
  int rc = read_states(h, st);
  if (rc != LEV_OK) return rc;
  *r = st[net].r;
  return LEV_OK;
}

int lev_set_gain_controller(LevEngine *h, int32_t net, int32_t enabled) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (net < -1 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  DeviceScope ds(h->device);
  for (int n = 0; n < h->num_nets; ++n) {
    if (net >= 0 && n != net) continue;
    h->h_nets[n].ctrl = enabled ? 1 : 0;
  }
  LEV_TRY_CUDA(cudaMemcpyAsync(h->d_nets, h->h_nets.data(),
                               sizeof(NetDesc) * h->num_nets,
                               cudaMemcpyHostToDevice, h->stream));
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return LEV_OK;
}

int lev_set_params(LevEngine *h, int32_t net, const LevParams *p) {
  if (h) spec_drop(h);
  if (!h || !p) return fail(LEV_ERR_ARG, "null argument");
  if (net < -1 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  int rc = check_params(*p);
  if (rc != LEV_OK) return rc;
  DeviceScope ds(h->device);
  std::vector<NetState> st;
  rc = read_states(h, st);
  if (rc != LEV_OK) return rc;
  for (int n = 0; n < h->num_nets; ++n) {
    if (net >= 0 && n != net) continue;
    params_to_desc(*p, &h->h_nets[n]);
    st[n].g = p->g;
  }
  LEV_TRY_CUDA(cudaMemcpyAsync(h->d_nets, h->h_nets.data(),
                               sizeof(NetDesc) * h->num_nets,
                               cudaMemcpyHostToDevice, h->stream));
  LEV_TRY_CUDA(cudaMemcpyAsync(h->d_st, st.data(),
                               sizeof(NetState) * h->num_nets,
                               cudaMemcpyHostToDevice, h->stream));
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  return LEV_OK;
}

int lev_get_params(LevEngine *h, int32_t net, LevParams *p) {
  if (!h || !p) return fail(LEV_ERR_ARG, "null argument");
  if (net < 0 || net >= h->num_nets)
    return fail(LEV_ERR_ARG, "network index out of range");
  float g = 0.0f;
  int rc = lev_get_gain(h, net, &g);
  if (rc != LEV_OK) return rc;
  desc_to_params(h->h_nets[net], g, p);
  return LEV_OK;
}

int lev_set_math_mode(LevEngine *h, int32_t math_mode) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  spec_drop(h);
  if (math_mode != LEV_MATH_REFERENCE && math_mode != LEV_MATH_ACCURATE)
    return fail(LEV_ERR_ARG, "math_mode must be 0 (reference) or 1");
  h->math_mode = math_mode;
  return LEV_OK;
}

int lev_cluster_info(const LevEngine *h, int32_t *eligible, int32_t *enabled,
                     int32_t *ctas, int32_t *rows_per_cta, int64_t *smem_bytes) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (eligible) *eligible = h->cluster_ok ? 1 : 0;
  if (enabled) *enabled = h->use_cluster ? 1 : 0;
  if (ctas) *ctas = h->cluster_C;
  if (rows_per_cta) *rows_per_cta = h->cluster_R;
  if (smem_bytes) *smem_bytes = (int64_t)h->cluster_smem;
  return LEV_OK;
}

int lev_set_cluster_mode(LevEngine *h, int32_t enabled) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  h->use_cluster = enabled != 0;
  return LEV_OK;
}

int lev_grid_info(const LevEngine *h, int32_t *eligible, int32_t *enabled, int32_t *ctas,
                  int32_t *rows_per_cta, int64_t *smem_bytes, int32_t *eligible_rows_mask) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  const int R = h->grid_R;
  const int ri = grid_r_index(R);
  if (eligible) *eligible = h->grid_ok ? 1 : 0;
  if (enabled) *enabled = (h->grid_ok && h->use_grid) ? 1 : 0;  // in use by step blocks
  if (ctas) *ctas = (h->grid_ok && R > 0) ? (h->h_nets[0].N + R - 1) / R : 0;
  if (rows_per_cta) *rows_per_cta = h->grid_ok ? R : 0;
  if (smem_bytes) *smem_bytes = h->grid_ok ? (int64_t)h->grid_smem_R[ri] : 0;
  if (eligible_rows_mask) {
    int m = 0;
    for (int i = 0; i < 3; ++i)
      if (h->grid_R_ok[i]) m |= kGridRs[i];
    *eligible_rows_mask = m;
  }
  return LEV_OK;
}

int lev_set_grid_mode(LevEngine *h, int32_t enabled, int32_t rows_per_cta) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (rows_per_cta != 0) {
    if (rows_per_cta != 64 && rows_per_cta != 128 && rows_per_cta != 256)
      return fail(LEV_ERR_ARG, "rows_per_cta must be 0, 64, 128 or 256");
    if (!h->grid_R_ok[grid_r_index(rows_per_cta)])
      return fail(LEV_ERR_ARG, "rows_per_cta not eligible for this engine");
    h->grid_R = rows_per_cta;
  }
  h->use_grid = enabled != 0;
  return LEV_OK;
}

static int check_wait_args(uint64_t limit_ns, uint32_t extra) {
  if (limit_ns < 1000ull || limit_ns > 60000000000ull)
    return fail(LEV_ERR_ARG, "limit_ns must be in [1 us, 60 s]");
  if (extra > 1024u) return fail(LEV_ERR_ARG, "extra_arrivals must be <= 1024");
  return LEV_OK;
}

int lev_set_grid_wait(LevEngine *h, uint64_t limit_ns, uint32_t extra_arrivals) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  int rc = check_wait_args(limit_ns, extra_arrivals);
  if (rc != LEV_OK) return rc;
  h->grid_wait.ns = limit_ns;
  h->grid_wait.extra = extra_arrivals;
  return LEV_OK;
}

int lev_trim_memory(void) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (int d = 0; d < kMaxDevices; ++d)
    if (g_pool[d]) LEV_TRY_CUDA(cudaMemPoolTrimTo(g_pool[d], 0));
  return LEV_OK;
}

int lev_create_profile(const LevEngine *h, double *ms_out) {
  if (!h || !ms_out) return fail(LEV_ERR_ARG, "null argument");
  for (int k = 0; k < 8; ++k) ms_out[k] = h->create_ms[k];
  return LEV_OK;
}

int lev_num_variants(void) { return kNumVariants; }

int lev_num_pair_variants(void) { return kNumPairVariants; }

int lev_pair_variant_info(int32_t v, int32_t *unroll, int32_t *min_blocks,
                          int32_t *deep) {
  if (v < 0 || v >= kNumPairVariants) return fail(LEV_ERR_ARG, "pair variant out of range");
  if (unroll) *unroll = kPairVariants[v].U;
  if (min_blocks) *min_blocks = kPairVariants[v].MINB;
  if (deep) *deep = kPairVariants[v].DEEP;
  return LEV_OK;
}

int lev_pair_variant_lanes(int32_t v, int32_t *lanes) {
  if (v < 0 || v >= kNumPairVariants || !lanes) return fail(LEV_ERR_ARG, "bad pair variant");
  *lanes = kPairVariants[v].LANES;
  return LEV_OK;
}

int lev_pair_info(const LevEngine *h, int32_t c, int32_t *eligible, int32_t *enabled,
                  int32_t *pair_variant, float *pair_ms, float *step_ms) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (c < 0 || c >= kNumClasses) return fail(LEV_ERR_ARG, "class out of range");
  const TileClass &tc = h->classes[c];
  if (eligible) *eligible = h->pair_ok ? 1 : 0;
  if (enabled) *enabled = pairs_active(h) ? 1 : 0;
  if (pair_variant) *pair_variant = tc.pair_variant;
  if (pair_ms) *pair_ms = tc.pair_ms;
  if (step_ms) *step_ms = tc.step_ms;
  return LEV_OK;
}

int lev_set_pair_mode(LevEngine *h, int32_t enabled) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  spec_drop(h);
  if ((enabled != 0) != h->use_pairs) {
    DeviceScope ds(h->device);
    cudaStreamSynchronize(h->stream);
    clear_graphs(h);
    h->use_pairs = enabled != 0;
  }
  return LEV_OK;
}

int lev_set_pair_variant(LevEngine *h, int32_t c, int32_t v) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  spec_drop(h);
  if (c < 0 || c >= kNumClasses) return fail(LEV_ERR_ARG, "class out of range");
  if (v < -1 || v >= kNumPairVariants)
    return fail(LEV_ERR_ARG, "pair variant out of range (-1 turns pairs off)");
  if (h->classes[c].pair_variant != v) {
    DeviceScope ds(h->device);
    cudaStreamSynchronize(h->stream);
    clear_graphs(h);
    h->classes[c].pair_variant = v;
  }
  return LEV_OK;
}

int lev_time_launches(LevEngine *h, float dt, int32_t n, float *ms_out) {
  if (h) spec_drop(h);
  if (!h || !ms_out) return fail(LEV_ERR_ARG, "null argument");
  if (h->part) return fail(LEV_ERR_STATE, "partition engine: not supported");
  if (n < 1) return fail(LEV_ERR_ARG, "n must be >= 1");
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  DeviceScope ds(h->device);
  const bool pairs = pairs_active(h);
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  int rc = LEV_OK;
  for (int i = 0; i < 3 && rc == LEV_OK; ++i)
    if (cudaEventCreate(&ev[i]) != cudaSuccess) rc = fail(LEV_ERR_CUDA, "event creation failed");
  StepArgs a = make_args(h, dt, nullptr, 0, nullptr);
  double sum[2] = {0.0, 0.0};
  for (int i = 0; i < n && rc == LEV_OK; ++i) {
    float ms0 = 0.0f, ms1 = 0.0f;
    for (int phase = 0; phase < 2 && rc == LEV_OK; ++phase) {
      cudaEventRecord(ev[phase], h->stream);
      a.reverse = h->sweep;
      h->sweep ^= 1;
      for (int c = 0; c < kNumClasses && rc == LEV_OK; ++c)
        rc = pairs ? launch_pair_class(h, c, a, phase) : launch_class(h, c, a);
    }
    cudaEventRecord(ev[2], h->stream);
    if (rc != LEV_OK) break;
    if (cudaEventSynchronize(ev[2]) != cudaSuccess) {
      rc = fail(LEV_ERR_CUDA, "timed launches failed");
      break;
    }
    cudaEventElapsedTime(&ms0, ev[0], ev[1]);
    cudaEventElapsedTime(&ms1, ev[1], ev[2]);
    sum[0] += ms0;
    sum[1] += ms1;
  }
  for (int i = 0; i < 3; ++i)
    if (ev[i]) cudaEventDestroy(ev[i]);
  if (rc != LEV_OK) return rc;
  ms_out[0] = (float)(sum[0] / n);
  ms_out[1] = (float)(sum[1] / n);
  return LEV_OK;
}

int lev_variant_info(int32_t v, int32_t *unroll, int32_t *pipelined,
                     int32_t *min_blocks) {
  if (v < 0 || v >= kNumVariants) return fail(LEV_ERR_ARG, "variant out of range");
  if (unroll) *unroll = kVariants[v].U;
  if (pipelined) *pipelined = kVariants[v].PIPE;
  if (min_blocks) *min_blocks = kVariants[v].MINB;
  return LEV_OK;
}

int lev_class_info(const LevEngine *h, int32_t c, int32_t *ntiles,
                   float *mean_slice_len, int64_t *edges, int32_t *variant) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (c < 0 || c >= kNumClasses) return fail(LEV_ERR_ARG, "class out of range");
  const TileClass &tc = h->classes[c];
  if (ntiles) *ntiles = tc.ntiles;
  if (mean_slice_len) *mean_slice_len = (float)tc.mean_len;
  if (edges) *edges = tc.edges;
  if (variant) *variant = tc.variant;
  return LEV_OK;
}

int lev_set_variant(LevEngine *h, int32_t c, int32_t v) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  spec_drop(h);
  if (c < 0 || c >= kNumClasses) return fail(LEV_ERR_ARG, "class out of range");
  if (v < 0 || v >= kNumVariants) return fail(LEV_ERR_ARG, "variant out of range");
  if (h->classes[c].variant != v) {
    DeviceScope ds(h->device);
    cudaStreamSynchronize(h->stream);
    clear_graphs(h);
    h->classes[c].variant = v;
  }
  return LEV_OK;
}

// Device-side copy of the evolving state (weights, node state, ring,
// per-network state) so tuning trials leave the simulation untouched.
struct StateSnapshot {
  float *w = nullptr, *th = nullptr, *thh = nullptr, *wh = nullptr,
        *ring = nullptr;
  NetState *st = nullptr;
  void release() {
    cudaFree(w);
    cudaFree(th);
    cudaFree(thh);
    cudaFree(wh);
    cudaFree(ring);
    cudaFree(st);
    w = th = thh = wh = ring = nullptr;
    st = nullptr;
  }
};

static int snapshot_copy(LevEngine *h, StateSnapshot &s, bool save) {
  auto cp = [&](void *dst_save, void *live, size_t bytes) -> cudaError_t {
    return save ? cudaMemcpyAsync(dst_save, live, bytes, cudaMemcpyDeviceToDevice, h->stream)
                : cudaMemcpyAsync(live, dst_save, bytes, cudaMemcpyDeviceToDevice, h->stream);
  };
  const size_t nn = sizeof(float) * h->total_nodes;
  cudaError_t e = cp(s.w, h->d_sl_w, sizeof(float) * std::max<long long>(h->sl_total, 1));
  if (e == cudaSuccess) e = cp(s.th, h->d_theta, nn);
  if (e == cudaSuccess) e = cp(s.thh, h->d_theta_hat, nn);
  if (e == cudaSuccess) e = cp(s.wh, h->d_omega_hat, nn);
  if (e == cudaSuccess) e = cp(s.ring, h->d_ring, sizeof(float) * h->ring_floats);
  if (e == cudaSuccess) e = cp(s.st, h->d_st, sizeof(NetState) * h->num_nets);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return fail(LEV_ERR_CUDA, std::string("state snapshot: ") + cudaGetErrorString(e));
  return LEV_OK;
}

int lev_autotune(LevEngine *h, float dt, int32_t trial_steps,
                 int32_t *variant_out, float *ms_out) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (h->part) return fail(LEV_ERR_STATE, "partition engine: not supported");
  spec_drop(h);
  if (trial_steps < 1) return fail(LEV_ERR_ARG, "trial_steps must be >= 1");
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  DeviceScope ds(h->device);
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  StateSnapshot snap;
  const size_t nn = sizeof(float) * std::max<long long>(h->total_nodes, 1);
  if (cudaMalloc(&snap.w, sizeof(float) * std::max<long long>(h->sl_total, 1)) != cudaSuccess ||
      cudaMalloc(&snap.th, nn) != cudaSuccess || cudaMalloc(&snap.thh, nn) != cudaSuccess ||
      cudaMalloc(&snap.wh, nn) != cudaSuccess ||
      cudaMalloc(&snap.ring, sizeof(float) * std::max<long long>(h->ring_floats, 1)) != cudaSuccess ||
      cudaMalloc(&snap.st, sizeof(NetState) * h->num_nets) != cudaSuccess) {
    snap.release();
    return fail(LEV_ERR_NOMEM, "autotune: no room for a state snapshot");
  }
  int rc = snapshot_copy(h, snap, true);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (rc == LEV_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    rc = fail(LEV_ERR_CUDA, "autotune: event creation failed");
  StepArgs a = make_args(h, dt, nullptr, 0, nullptr);
  for (int c = 0; c < kNumClasses && rc == LEV_OK; ++c) {
    TileClass &tc = h->classes[c];
    if (tc.ntiles == 0) {
      for (int v = 0; v < kNumVariants; ++v)
        if (ms_out) ms_out[c * kNumVariants + v] = 0.0f;
      continue;
    }
    float best = 0.0f;
    int best_v = tc.variant;
    for (int v = 0; v < kNumVariants && rc == LEV_OK; ++v) {
      tc.variant = v;
      for (int i = 0; i < 2 && rc == LEV_OK; ++i) {  // warm-up
        a.reverse = i & 1;
        rc = launch_class(h, c, a);
      }
      if (rc != LEV_OK) break;
      cudaEventRecord(e0, h->stream);
      for (int i = 0; i < trial_steps && rc == LEV_OK; ++i) {
        a.reverse = i & 1;
        rc = launch_class(h, c, a);
      }
      cudaEventRecord(e1, h->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        rc = fail(LEV_ERR_CUDA, "autotune: trial failed");
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= trial_steps;
      if (ms_out) ms_out[c * kNumVariants + v] = ms;
      if (v == 0 || ms < best) {
        best = ms;
        best_v = v;
      }
    }
    tc.variant = best_v;
    tc.step_ms = best;
    if (variant_out) variant_out[c] = best_v;
    // two steps per launch: pair_kernel + finish_kernel per two steps; kept
    // for this class only where it beats the best one-step variant
    if (h->pair_ok && rc == LEV_OK) {
      const int pairs = std::max(1, trial_steps);
      float best_p = 0.0f;
      int best_pv = -1;
      for (int v = 0; v < kNumPairVariants && rc == LEV_OK; ++v) {
        if (!pair_variant_ok(h, v)) continue;
        tc.pair_variant = v;
        for (int ph = 0; ph < 2 && rc == LEV_OK; ++ph) {  // warm-up
          a.reverse = ph;
          rc = launch_pair_class(h, c, a, ph);
        }
        if (rc != LEV_OK) break;
        cudaEventRecord(e0, h->stream);
        for (int i = 0; i < pairs && rc == LEV_OK; ++i)
          for (int ph = 0; ph < 2 && rc == LEV_OK; ++ph) {
            a.reverse = ph;
            rc = launch_pair_class(h, c, a, ph);
          }
        cudaEventRecord(e1, h->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
          rc = fail(LEV_ERR_CUDA, "autotune: pair trial failed");
          break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= 2.0f * pairs;
        if (best_pv < 0 || ms < best_p) {
          best_p = ms;
          best_pv = v;
        }
      }
      tc.pair_ms = best_p;
      tc.pair_variant = (best_pv >= 0 && best_p < best) ? best_pv : -1;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[tune_key(tc, c)] = best_v;
    if (h->pair_ok) g_pair_cache[tune_key(tc, c)] = tc.pair_variant;
  }
  // small and mid-sized single networks: per-step graph replay, the
  // cluster-resident kernel or the grid-resident kernel (each rows-per-CTA
  // choice), whichever is fastest
  if (rc == LEV_OK && (h->cluster_ok || h->grid_ok)) {
    const int n = std::max(trial_steps, 32);
    // mode 0: graph replay, 1: cluster, 2 + ri: grid with kGridRs[ri]
    float best_t = -1.0f;
    int best_m = 0;
    for (int m = 0; m < 5 && rc == LEV_OK; ++m) {
      if (m == 1 && !h->cluster_ok) continue;
      if (m >= 2 && !h->grid_R_ok[m - 2]) continue;
      h->use_cluster = (m == 1);
      h->use_grid = (m >= 2);
      if (m >= 2) h->grid_R = kGridRs[m - 2];
      // warm-up: the first block of a length is issued directly, the second
      // records the graph that the timed block replays
      for (int w = 0; w < 2 && rc == LEV_OK; ++w) rc = enqueue_steps(h, dt, n, nullptr);
      if (rc != LEV_OK) break;
      cudaEventRecord(e0, h->stream);
      rc = enqueue_steps(h, dt, n, nullptr);
      cudaEventRecord(e1, h->stream);
      float t = 0.0f;
      if (rc == LEV_OK && cudaEventSynchronize(e1) == cudaSuccess &&
          cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) {
        if (best_t < 0.0f || t < best_t) {
          best_t = t;
          best_m = m;
        }
      }
      if (rc == LEV_OK) rc = check_grid_error(h);
    }
    h->use_cluster = rc == LEV_OK && best_m == 1;
    h->use_grid = rc == LEV_OK && best_m >= 2;
    if (best_m >= 2) h->grid_R = kGridRs[best_m - 2];
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (rc == LEV_OK) rc = snapshot_copy(h, snap, false);
  else snapshot_copy(h, snap, false);
  snap.release();
  clear_graphs(h);
  return rc;
}

int lev_get_vram_usage(const LevEngine *h, size_t *bytes) {
  if (!h || !bytes) return fail(LEV_ERR_ARG, "null argument");
  *bytes = h->vram;
  return LEV_OK;
}

// ===========================================================================
// Hub-phase transition counter (the reference's integrated-information
// front-end, leviathan_phi_kernel.cu:60-92 and phi_init / phi_accumulate /
// phi_reset / phi_get_transition_count / phi_free, :243-367)
// ===========================================================================
namespace lev {
__global__ void hub_observe_kernel(HubMonitor *m, const float *theta) {
  if (threadIdx.x == 0 && blockIdx.x == 0) hub_observe(m, theta);
}
}  // namespace lev

static int hubs_sync(LevHubs *m) {
  if (m->engine) LEV_TRY_CUDA(cudaStreamSynchronize(m->engine->stream));
  LEV_TRY_CUDA(cudaStreamSynchronize(m->stream));
  return LEV_OK;
}

static int hubs_clear(LevHubs *m) {
  const size_t S = (size_t)m->S;
  LEV_TRY_CUDA(cudaMemsetAsync(m->d_counts, 0, sizeof(unsigned long long) * S * S, m->stream));
  LEV_TRY_CUDA(cudaMemsetAsync(m->d_totals, 0, sizeof(unsigned long long) * S, m->stream));
  const int prev = -1;
  const long long observed = 0;
  LEV_TRY_CUDA(cudaMemcpyAsync(&m->d_mon->prev, &prev, sizeof(int), cudaMemcpyHostToDevice,
                               m->stream));
  LEV_TRY_CUDA(cudaMemcpyAsync(&m->d_mon->observed, &observed, sizeof(long long),
                               cudaMemcpyHostToDevice, m->stream));
  LEV_TRY_CUDA(cudaStreamSynchronize(m->stream));
  return LEV_OK;
}

static void hubs_free(LevHubs *m) {
  cudaFree(m->d_mon);
  cudaFree(m->d_counts);
  cudaFree(m->d_totals);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

extern "C" {

int lev_hubs_create(LevHubs **out, int32_t num_hubs, const int32_t *hub_idx) {
  if (!out || !hub_idx) return fail(LEV_ERR_ARG, "null argument");
  *out = nullptr;
  if (num_hubs < 1 || num_hubs > kMaxHubs)
    return fail(LEV_ERR_ARG, "num_hubs must be in [1, " + std::to_string(kMaxHubs) + "]");
  for (int i = 0; i < num_hubs; ++i)
    if (hub_idx[i] < 0) return fail(LEV_ERR_ARG, "hub index is negative");
  LevHubs *m = new LevHubs();
  m->num_hubs = num_hubs;
  m->S = 1 << num_hubs;
  cudaError_t e = cudaGetDevice(&m->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_mon, sizeof(HubMonitor));
  if (e == cudaSuccess)
    e = cudaMalloc(&m->d_counts, sizeof(unsigned long long) * (size_t)m->S * m->S);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_totals, sizeof(unsigned long long) * m->S);
  if (e != cudaSuccess) {
    hubs_free(m);
    return fail(LEV_ERR_NOMEM, std::string("hub monitor: ") + cudaGetErrorString(e));
  }
  HubMonitor hm;
  std::memset(&hm, 0, sizeof(hm));
  hm.net = -1;
  hm.num_hubs = num_hubs;
  for (int i = 0; i < num_hubs; ++i) hm.hub[i] = hub_idx[i];
  hm.prev = -1;
  hm.counts = m->d_counts;
  hm.totals = m->d_totals;
  e = cudaMemcpy(m->d_mon, &hm, sizeof(hm), cudaMemcpyHostToDevice);
  int rc = e == cudaSuccess ? hubs_clear(m)
                            : fail(LEV_ERR_CUDA, std::string("hub monitor: ") + cudaGetErrorString(e));
  if (rc != LEV_OK) {
    std::string msg = g_last_error;
    hubs_free(m);
    return fail(rc, msg);
  }
  *out = m;
  return LEV_OK;
}

int lev_attach_hubs(LevEngine *h, int32_t net, LevHubs *m) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (h->part) return fail(LEV_ERR_STATE, "partition engine: not supported");
  spec_drop(h);
  DeviceScope ds(h->device);
  LEV_TRY_CUDA(cudaStreamSynchronize(h->stream));
  if (!m) {  // detach
    if (h->hubs) {
      h->hubs->engine = nullptr;
      h->hubs = nullptr;
      clear_graphs(h);
    }
    return LEV_OK;
  }
  if (net < 0 || net >= h->num_nets) return fail(LEV_ERR_ARG, "network out of range");
  if (m->device != h->device) return fail(LEV_ERR_ARG, "hub monitor is on another device");
  if (m->engine && m->engine != h) return fail(LEV_ERR_STATE, "hub monitor fed by another engine");
  HubMonitor hm;
  LEV_TRY_CUDA(cudaMemcpy(&hm, m->d_mon, sizeof(hm), cudaMemcpyDeviceToHost));
  for (int i = 0; i < m->num_hubs; ++i)
    if (hm.hub[i] >= h->h_nets[net].N) return fail(LEV_ERR_ARG, "hub index beyond the network");
  if (h->hubs && h->hubs != m) h->hubs->engine = nullptr;
  hm.net = net;
  LEV_TRY_CUDA(cudaMemcpy(&m->d_mon->net, &hm.net, sizeof(int), cudaMemcpyHostToDevice));
  h->hubs = m;
  m->engine = h;
  clear_graphs(h);
  return LEV_OK;
}

int lev_hubs_accumulate(LevHubs *m, const float *theta_dev, void *stream) {
  if (!m || !theta_dev) return fail(LEV_ERR_ARG, "null argument");
  if (m->engine) return fail(LEV_ERR_STATE, "hub monitor is fed by an engine; detach it first");
  DeviceScope ds(m->device);
  cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : m->stream;
  hub_observe_kernel<<<1, 32, 0, s>>>(m->d_mon, theta_dev);
  LEV_TRY_CUDA(cudaGetLastError());
  if (s != m->stream) LEV_TRY_CUDA(cudaStreamSynchronize(s));
  return LEV_OK;
}

int lev_hubs_reset(LevHubs *m) {
  if (!m) return fail(LEV_ERR_ARG, "null argument");
  DeviceScope ds(m->device);
  int rc = hubs_sync(m);
  return rc != LEV_OK ? rc : hubs_clear(m);
}

int lev_hubs_read(LevHubs *m, uint64_t *counts, uint64_t *totals, int32_t *prev_state,
                  int64_t *observed) {
  if (!m) return fail(LEV_ERR_ARG, "null argument");
  DeviceScope ds(m->device);
  int rc = hubs_sync(m);
  if (rc != LEV_OK) return rc;
  const size_t S = (size_t)m->S;
  if (counts)
    LEV_TRY_CUDA(cudaMemcpy(counts, m->d_counts, sizeof(uint64_t) * S * S, cudaMemcpyDeviceToHost));
  if (totals)
    LEV_TRY_CUDA(cudaMemcpy(totals, m->d_totals, sizeof(uint64_t) * S, cudaMemcpyDeviceToHost));
  HubMonitor hm;
  LEV_TRY_CUDA(cudaMemcpy(&hm, m->d_mon, sizeof(hm), cudaMemcpyDeviceToHost));
  if (prev_state) *prev_state = hm.prev;
  if (observed) *observed = hm.observed;
  return LEV_OK;
}

int lev_hubs_destroy(LevHubs *m) {
  if (!m) return LEV_OK;
  DeviceScope ds(m->device);
  if (m->engine) lev_attach_hubs(m->engine, 0, nullptr);
  hubs_free(m);
  return LEV_OK;
}

}  // extern "C"

// ===========================================================================
// Reference ABI (leviathan_kernel.cu:21-499)
// ===========================================================================
static void report(const char *fn) {
  std::fprintf(stderr, "[leviathan_b200] %s: %s\n", fn, g_last_error.c_str());
}

LeviathanHandle *leviathan_init(int N, int max_delay, int *h_row_ptr,
                                int *h_col_idx, uint8_t *h_delays,
                                float *h_weights, float *h_theta,
                                float *h_theta_hat, float *h_omega) {
  LevEngine *e = nullptr;
  if (lev_create(&e, N, max_delay, h_row_ptr, h_col_idx, h_delays, h_weights,
                 h_theta, h_theta_hat, h_omega, nullptr,
                 LEV_MATH_REFERENCE) != LEV_OK) {
    report("leviathan_init");
    return nullptr;
  }
  LeviathanHandle *h = new LeviathanHandle();
  h->eng = e;
  return h;
}

float leviathan_step(LeviathanHandle *handle, float dt) {
  if (!handle) {
    fail(LEV_ERR_ARG, "null handle");
    return std::numeric_limits<float>::quiet_NaN();
  }
  float r = 0.0f;
  if (lev_step(handle->eng, dt, &r) != LEV_OK) {
    report("leviathan_step");
    return std::numeric_limits<float>::quiet_NaN();
  }
  return r;
}

void leviathan_get_theta(LeviathanHandle *handle, float *h_theta) {
  if (!handle || lev_get_theta(handle->eng, h_theta) != LEV_OK)
    report("leviathan_get_theta");
}

void leviathan_set_theta(LeviathanHandle *handle, float *h_theta) {
  if (!handle || lev_set_theta(handle->eng, h_theta) != LEV_OK)
    report("leviathan_set_theta");
}

void leviathan_free(LeviathanHandle *handle) {
  if (!handle) return;
  lev_destroy(handle->eng);
  delete handle;
}

void leviathan_set_gain(LeviathanHandle *handle, float g) {
  if (!handle || lev_set_gain(handle->eng, 0, g) != LEV_OK)
    report("leviathan_set_gain");
}

float leviathan_get_gain(LeviathanHandle *handle) {
  float g = std::numeric_limits<float>::quiet_NaN();
  if (!handle || lev_get_gain(handle->eng, 0, &g) != LEV_OK)
    report("leviathan_get_gain");
  return g;
}

void leviathan_set_gain_controller(LeviathanHandle *handle, bool enabled) {
  if (!handle ||
      lev_set_gain_controller(handle->eng, 0, enabled ? 1 : 0) != LEV_OK)
    report("leviathan_set_gain_controller");
}

size_t leviathan_get_vram_usage(LeviathanHandle *handle) {
  size_t b = 0;
  if (!handle || lev_get_vram_usage(handle->eng, &b) != LEV_OK)
    report("leviathan_get_vram_usage");
  return b;
}

void leviathan_reset_weights(LeviathanHandle *handle, float *h_weights) {
  if (!handle || lev_reset_weights(handle->eng, h_weights) != LEV_OK)
    report("leviathan_reset_weights");
}

LevEngine *leviathan_engine(LeviathanHandle *handle) {
  return handle ? handle->eng : nullptr;
}

}  // extern "C"

// ===========================================================================
// Adjoint (reverse-mode differentiation through T steps); device code in
// lev_adjoint.cuh.
// ===========================================================================
#include "lev_adjoint.cuh"
#include "lev_adj_grid.cuh"
#include "lev_graphgen.cuh"

namespace lev {
__global__ void ws_table_init_kernel(WsSlot *t, unsigned long long n) {
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
       k < n; k += (unsigned long long)gridDim.x * blockDim.x) {
    t[k].key = 0ull;
    t[k].owner = 0xFFFFFFFFu;
    t[k].accepted = 0u;
  }
}
}  // namespace lev

extern "C" int lev_gen_ws(int32_t N, int32_t k, double p, uint64_t seed,
                          int32_t delay_lo, int32_t delay_hi, float w_lo,
                          float w_hi, float omega_mean, float omega_std,
                          int32_t *row_ptr, int32_t *col_idx, uint8_t *delays,
                          float *weights, float *theta, float *omega) {
  if (N < 3 || N >= (1 << 24)) return fail(LEV_ERR_ARG, "N must be in [3, 2^24)");
  if (k < 2 || (k & 1) || k >= N) return fail(LEV_ERR_ARG, "k must be even, 2 <= k < N");
  if (!(p >= 0.0 && p <= 1.0)) return fail(LEV_ERR_ARG, "p must be in [0, 1]");
  if (delay_lo < 0 || delay_hi > 255 || delay_lo > delay_hi)
    return fail(LEV_ERR_ARG, "delays must satisfy 0 <= lo <= hi <= 255");
  if (!row_ptr || !col_idx || !delays || !weights || !theta || !omega)
    return fail(LEV_ERR_ARG, "null output array");
  const long long half = k / 2, n_lat = (long long)N * half, E = 2 * n_lat;
  if (E >= (1LL << 31)) return fail(LEV_ERR_ARG, "N*k must be below 2^31");
  cudaStream_t s;
  LEV_TRY_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  // table: >= 4x the expected number of rewired edges (load factor <= 1/4)
  unsigned long long tsize = 1024;
  while (tsize < (unsigned long long)(4.0 * p * n_lat + 1024)) tsize <<= 1;
  int *target = nullptr, *deg = nullptr, *rp = nullptr, *cursor = nullptr, *col = nullptr;
  unsigned int *pend[2] = {nullptr, nullptr}, *cnt = nullptr;
  long long *cand = nullptr;
  WsSlot *table = nullptr;
  uint8_t *dl = nullptr;
  float *w = nullptr, *th = nullptr, *om = nullptr;
  std::vector<void *> bufs;
  auto cleanup = [&]() {
    for (void *b : bufs) cudaFree(b);
    cudaStreamDestroy(s);
  };
  auto alloc = [&](void **ptr, size_t bytes) {
    cudaError_t e = cudaMalloc(ptr, std::max<size_t>(bytes, 4));
    if (e == cudaSuccess) bufs.push_back(*ptr);
    return e == cudaSuccess;
  };
  bool ok = alloc((void **)&target, sizeof(int) * n_lat) &&
            alloc((void **)&deg, sizeof(int) * N) &&
            alloc((void **)&rp, sizeof(int) * (N + 1)) &&
            alloc((void **)&cursor, sizeof(int) * N) &&
            alloc((void **)&col, sizeof(int) * E) &&
            alloc((void **)&pend[0], sizeof(unsigned) * n_lat) &&
            alloc((void **)&pend[1], sizeof(unsigned) * n_lat) &&
            alloc((void **)&cnt, sizeof(unsigned) * 2) &&
            alloc((void **)&cand, sizeof(long long) * n_lat) &&
            alloc((void **)&table, sizeof(WsSlot) * tsize) &&
            alloc((void **)&dl, E) && alloc((void **)&w, sizeof(float) * E) &&
            alloc((void **)&th, sizeof(float) * N) && alloc((void **)&om, sizeof(float) * N);
  if (!ok) {
    cleanup();
    return fail(LEV_ERR_NOMEM, "lev_gen_ws: device allocation failed");
  }
  WsArgs a;
  a.N = N;
  a.half = (int)half;
  a.p = p;
  a.seed = seed;
  const int G = 148 * 8, B = 256;
  cudaMemsetAsync(cnt, 0, sizeof(unsigned) * 2, s);
  cudaMemsetAsync(deg, 0, sizeof(int) * N, s);
  cudaMemsetAsync(cursor, 0, sizeof(int) * N, s);
  ws_table_init_kernel<<<G, B, 0, s>>>(table, tsize);
  ws_init_kernel<<<G, B, 0, s>>>(a, n_lat, target, pend[0], cnt);
  unsigned int n_pend = 0;
  cudaMemcpyAsync(&n_pend, cnt, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  cudaError_t ce = cudaStreamSynchronize(s);
  int cur = 0, round = 0;
  while (ce == cudaSuccess && n_pend > 0) {
    if (++round > 200) {
      cleanup();
      return fail(LEV_ERR_ARG, "lev_gen_ws: rewiring did not settle (graph too dense)");
    }
    cudaMemsetAsync(cnt + 1, 0, sizeof(unsigned), s);
    ws_propose_kernel<<<G, B, 0, s>>>(a, round, pend[cur], n_pend, table, tsize - 1, cand);
    ws_resolve_kernel<<<G, B, 0, s>>>(a, round, pend[cur], n_pend, table, cand, target,
                                      pend[cur ^ 1], cnt + 1);
    cudaMemcpyAsync(&n_pend, cnt + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    ce = cudaStreamSynchronize(s);
    cur ^= 1;
  }
  if (ce == cudaSuccess) {
    ws_degree_kernel<<<G, B, 0, s>>>(a, n_lat, target, deg);
    ws_scan_kernel<<<1, 1024, 0, s>>>(deg, rp, N);
    ws_fill_kernel<<<G, B, 0, s>>>(a, n_lat, target, rp, cursor, col);
    WsStateArgs st;
    st.seed = seed ^ 0x5A17E5EEDull;
    st.delay_lo = delay_lo;
    st.delay_hi = delay_hi;
    st.w_lo = w_lo;
    st.w_hi = w_hi;
    st.omega_mean = omega_mean;
    st.omega_std = omega_std;
    ws_finish_kernel<<<G, B, 0, s>>>(st, N, rp, col, dl, w, th, om);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(row_ptr, rp, sizeof(int) * (N + 1), cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(col_idx, col, sizeof(int) * E, cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(delays, dl, E, cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(weights, w, sizeof(float) * E, cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(theta, th, sizeof(float) * N, cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(omega, om, sizeof(float) * N, cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
  cleanup();
  if (ce != cudaSuccess)
    return fail(LEV_ERR_CUDA, std::string("lev_gen_ws: ") + cudaGetErrorString(ce));
  return LEV_OK;
}

namespace lev {

// per-network state set-up: mode 0 init from K (cur 0), mode 1 save g into
// ck, mode 2 restore g from ck with the segment ring position.
__global__ void adj_state_kernel(int mode, const NetDesc *nets, NetState *st,
                                 float *ck_g, const float *K, int num_nets) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < num_nets;
       n += gridDim.x * blockDim.x) {
    if (mode == 1) {
      ck_g[n] = st[n].g;
      continue;
    }
    NetState s;
    s.g = (mode == 0) ? K[n] : ck_g[n];
    s.r = 0.0f;
    s.cur = (mode == 0) ? 0 : nets[n].max_delay;
    s.ticket = 0u;
    s.t = 0;
    s.rbuf = 0;
    s.rpos = 0;
    st[n] = s;
  }
}

}  // namespace lev

struct LevAdjoint {
  LevEngine *e = nullptr;
  int C = 50, Tmax = 0, nseg = 0;
  long long TN = 0, SL = 0;  // total nodes, SELL entries
  int NN = 0;                // networks
  std::vector<NetDesc> h_nets;
  NetDesc *d_nets = nullptr;
  NetState *d_st = nullptr;
  long long ring_floats = 0, aux_floats = 0, ckr_floats = 0;
  long long *d_ck_off = nullptr;
  float *theta0 = nullptr, *theta_hat0 = nullptr;
  float *theta = nullptr, *theta_hat = nullptr, *omega = nullptr,
        *omega_hat = nullptr, *w = nullptr, *ring = nullptr;
  float2 *partials = nullptr, *bpart = nullptr;
  unsigned *tickets = nullptr;
  float *ck_theta = nullptr, *ck_thh = nullptr, *ck_omh = nullptr,
        *ck_w = nullptr, *ck_ring = nullptr, *ck_g = nullptr;
  float *w_hist = nullptr, *thh_hist = nullptr;
  // delayed source phase of every edge in each step of a segment (SELL),
  // recorded by the recompute for the reverse steps of the per-step kernels
  // (grids of more than one wave); null otherwise
  float *dj_hist = nullptr, *dj_hist2 = nullptr;
  float4 *trace = nullptr;
  // second set of segment records (extended ring, weights, theta_hat, trace)
  // so the backward pass recomputes segment k-1 on `rstream` while segment k
  // is reversed on the engine stream; null when it did not fit
  float *ring2 = nullptr, *w_hist2 = nullptr, *thh_hist2 = nullptr;
  float4 *trace2 = nullptr;
  cudaStream_t rstream = nullptr;
  cudaEvent_t ev_rec[2] = {nullptr, nullptr}, ev_rev[2] = {nullptr, nullptr},
              ev_start = nullptr;
  float *lam_th = nullptr, *lam_thh = nullptr, *lam_omh = nullptr,
        *lam_w = nullptr, *adj_ring = nullptr, *lam_g = nullptr,
        *grad_omega_acc = nullptr, *grad_theta0 = nullptr;
  std::vector<void *> allocs;
  size_t bytes = 0;
  int last_T = 0;
  float last_dt = 0.0f;
  const float *drive = nullptr;
  // reservoir (fused drive win * x and cos/sin readout), all device pointers
  const float *res_win = nullptr, *res_x = nullptr, *res_ra = nullptr,
              *res_rb = nullptr;
  float *res_y = nullptr;
  const float *res_dLdy = nullptr;
  float *res_gwin = nullptr, *res_gra = nullptr, *res_grb = nullptr;
  float *ro_partials = nullptr;
  // grid-resident segments (lev_adj_grid.cuh), single networks only
  bool grid_ok = false;
  bool use_grid = true;
  int grid_R = 0;
  bool gR_ok[3] = {false, false, false};  // R = 64, 128, 256
  int g_cap[3] = {0, 0, 0};
  size_t gf_smem[3] = {0, 0, 0}, gb_smem[3] = {0, 0, 0};
  bool gp_ok[3] = {false, false, false};  // paired recompute + reverse launch fits
  bool use_pair = true;
  int g_nwarps = 0, g_gpad = 0;
  float2 *g_wsum = nullptr;
  float *g_lgp = nullptr;
  unsigned *g_bar = nullptr;
  int *h_gerr = nullptr, *d_gerr = nullptr;
  GridWait grid_wait = {kGridWaitNs, 0u, 0u};  // bound of the barrier waits
};

namespace {

template <typename T>
int adj_alloc(LevAdjoint *a, T **p, long long count) {
  size_t b = std::max<long long>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), b);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(LEV_ERR_NOMEM, "adjoint: cudaMalloc of " + std::to_string(b) +
                                   " bytes failed: " + cudaGetErrorString(e));
  }
  a->allocs.push_back(*p);
  a->bytes += b;
  return LEV_OK;
}

void adj_free(LevAdjoint *a) {
  if (!a) return;
  for (void *p : a->allocs) cudaFree(p);
  for (int i = 0; i < 2; ++i) {
    if (a->ev_rec[i]) cudaEventDestroy(a->ev_rec[i]);
    if (a->ev_rev[i]) cudaEventDestroy(a->ev_rev[i]);
  }
  if (a->ev_start) cudaEventDestroy(a->ev_start);
  if (a->rstream) cudaStreamDestroy(a->rstream);
  if (a->h_gerr) cudaFreeHost(a->h_gerr);
  delete a;
}

AdjFwdArgs adj_fwd_args(LevAdjoint *a, float dt) {
  AdjFwdArgs f;
  std::memset(&f, 0, sizeof(f));
  LevEngine *e = a->e;
  f.nets = a->d_nets;
  f.st = a->d_st;
  f.tiles = e->d_tiles;
  f.row_ptr = e->d_row_ptr;
  f.sl_off = e->d_sl_off;
  f.sl_len = e->d_sl_len;
  f.sl_cd = e->d_sl_cd;
  f.w_in = a->w;
  f.w_out = a->w;
  f.theta = a->theta;
  f.theta_hat = a->theta_hat;
  f.omega = a->omega;
  f.omega_hat = a->omega_hat;
  f.ring = a->ring;
  f.partials = a->partials;
  f.dt = dt;
  return f;
}

int adj_launch_fwd(LevAdjoint *a, const AdjFwdArgs &f, cudaStream_t s = nullptr) {
  LevEngine *e = a->e;
  if (!s) s = e->stream;
  const bool acc = e->math_mode == LEV_MATH_ACCURATE;
  if (e->total_tiles <= 148) {  // under one wave: four lanes per row
    if (acc)
      adj_fwd_split_kernel<1, 2><<<e->total_tiles, 4 * kTile, 0, s>>>(f);
    else
      adj_fwd_split_kernel<0, 2><<<e->total_tiles, 4 * kTile, 0, s>>>(f);
  } else if (acc) {
    adj_fwd_kernel<1><<<e->total_tiles, kTile, 0, s>>>(f);
  } else {
    adj_fwd_kernel<0><<<e->total_tiles, kTile, 0, s>>>(f);
  }
  LEV_TRY_CUDA(cudaGetLastError());
  return LEV_OK;
}

// Checkpoint `seg` of the working state: save (forward pass) or restore into
// the working state and the extended ring `ring` (backward recompute).
int adj_ckpt(LevAdjoint *a, int seg, bool save, cudaStream_t s = nullptr,
             float *ring = nullptr) {
  LevEngine *e = a->e;
  if (!s) s = e->stream;
  if (!ring) ring = a->ring;
  const size_t nb = sizeof(float) * a->TN;
  auto cp = [&](float *ck, float *live, size_t bytes) {
    return save ? cudaMemcpyAsync(ck, live, bytes, cudaMemcpyDeviceToDevice, s)
                : cudaMemcpyAsync(live, ck, bytes, cudaMemcpyDeviceToDevice, s);
  };
  LEV_TRY_CUDA(cp(a->ck_theta + (size_t)seg * a->TN, a->theta, nb));
  LEV_TRY_CUDA(cp(a->ck_thh + (size_t)seg * a->TN, a->theta_hat, nb));
  LEV_TRY_CUDA(cp(a->ck_omh + (size_t)seg * a->TN, a->omega_hat, nb));
  LEV_TRY_CUDA(cp(a->ck_w + (size_t)seg * a->SL, a->w,
                  sizeof(float) * std::max<long long>(a->SL, 1)));
  dim3 grid(64, a->NN);
  if (save) {
    adj_state_kernel<<<1, 128, 0, s>>>(1, a->d_nets, a->d_st,
                                       a->ck_g + (size_t)seg * a->NN, nullptr, a->NN);
    adj_ring_ckpt_kernel<<<grid, 256, 0, s>>>(0, a->d_nets, a->d_st, ring,
                                              a->ck_ring + (size_t)seg * a->ckr_floats,
                                              a->d_ck_off, a->NN);
  } else {
    adj_ring_ckpt_kernel<<<grid, 256, 0, s>>>(1, a->d_nets, a->d_st, ring,
                                              a->ck_ring + (size_t)seg * a->ckr_floats,
                                              a->d_ck_off, a->NN);
    adj_state_kernel<<<1, 128, 0, s>>>(2, a->d_nets, a->d_st,
                                       a->ck_g + (size_t)seg * a->NN, nullptr, a->NN);
  }
  LEV_TRY_CUDA(cudaGetLastError());
  return LEV_OK;
}

using AdjGridFwdFn = void (*)(AdjGridFwdArgs);
using AdjGridBwdFn = void (*)(AdjGridBwdArgs);
AdjGridFwdFn adj_grid_fwd_fn(int R, int math_mode) {
  const bool acc = math_mode == LEV_MATH_ACCURATE;
  if (R == 64) return acc ? adj_grid_fwd_kernel<1, 64, 8> : adj_grid_fwd_kernel<0, 64, 8>;
  if (R == 128) return acc ? adj_grid_fwd_kernel<1, 128, 8> : adj_grid_fwd_kernel<0, 128, 8>;
  return acc ? adj_grid_fwd_kernel<1, 256, 8> : adj_grid_fwd_kernel<0, 256, 8>;
}
using AdjGridPairFn = void (*)(AdjGridFwdArgs, AdjGridBwdArgs, int);
AdjGridPairFn adj_grid_pair_fn(int R, int math_mode) {
  const bool acc = math_mode == LEV_MATH_ACCURATE;
  if (R == 64) return acc ? adj_grid_pair_kernel<1, 64, 8, 4> : adj_grid_pair_kernel<0, 64, 8, 4>;
  if (R == 128)
    return acc ? adj_grid_pair_kernel<1, 128, 8, 4> : adj_grid_pair_kernel<0, 128, 8, 4>;
  return acc ? adj_grid_pair_kernel<1, 256, 8, 4> : adj_grid_pair_kernel<0, 256, 8, 4>;
}
AdjGridBwdFn adj_grid_bwd_fn(int R, int math_mode) {
  const bool acc = math_mode == LEV_MATH_ACCURATE;
  if (R == 64) return acc ? adj_grid_bwd_kernel<1, 64, 8> : adj_grid_bwd_kernel<0, 64, 8>;
  if (R == 128) return acc ? adj_grid_bwd_kernel<1, 128, 8> : adj_grid_bwd_kernel<0, 128, 8>;
  return acc ? adj_grid_bwd_kernel<1, 256, 4> : adj_grid_bwd_kernel<0, 256, 4>;
}

// Grid-resident segments for a single network: per rows-per-CTA choice, the
// shared memory of both kernels and whether every CTA can be resident at once.
int adj_setup_grid(LevAdjoint *a, const std::vector<long long> &sl_off,
                   const std::vector<int> &sl_len) {
  a->grid_ok = false;
  if (a->NN != 1) return LEV_OK;
  const NetDesc &d = a->h_nets[0];
  int dev = 0, max_smem = 0, coop = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
          cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return LEV_OK;
  }
  if (!coop) return LEV_OK;
  const int nwarps = 8 * ((d.N + kTile - 1) / kTile);
  int max_gpad = 0;
  for (int ri = 0; ri < 3; ++ri) {
    const int R = kGridRs[ri];
    const int C = (d.N + R - 1) / R;
    if (C < 2) continue;
    const int gpad = (C + 3) & ~3;
    long long cap = 0;
    for (int c = 0; c < C; ++c) {
      long long e = 0;
      for (int s = c * R / 32; s < std::min<long long>((c + 1) * R / 32, (d.N + 31) / 32); ++s)
        e += 32LL * sl_len[d.slice_base + s];
      cap = std::max(cap, e);
    }
    const size_t fsm = sizeof(float2) * nwarps + sizeof(float) * 6 * R +
                       sizeof(int) * 2 * (R / 32) + 8 * (size_t)cap;
    const size_t bsm = sizeof(float) * (4 * R + gpad) + sizeof(int) * 2 * (R / 32) +
                       8 * (size_t)cap;
    if (std::max(fsm, bsm) + 1024 > (size_t)max_smem) continue;
    bool ok = true;
    for (int m = 0; m < 2 && ok; ++m) {
      const int mm = m ? LEV_MATH_ACCURATE : LEV_MATH_REFERENCE;
      const void *ff = reinterpret_cast<const void *>(adj_grid_fwd_fn(R, mm));
      const void *bf = reinterpret_cast<const void *>(adj_grid_bwd_fn(R, mm));
      int pf = 0, pb = 0;
      ok = cudaFuncSetAttribute(ff, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm) ==
               cudaSuccess &&
           cudaFuncSetAttribute(bf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm) ==
               cudaSuccess &&
           cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pf, ff, kGridLPR * R, fsm) ==
               cudaSuccess &&
           cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pb, bf, kGridLPR * R, bsm) ==
               cudaSuccess &&
           (long long)pf * sms >= C && (long long)pb * sms >= C;
    }
    cudaGetLastError();
    if (!ok) continue;
    // the paired backward launch: both groups resident at once
    bool pok = true;
    for (int m = 0; m < 2 && pok; ++m) {
      const void *pf = reinterpret_cast<const void *>(
          adj_grid_pair_fn(R, m ? LEV_MATH_ACCURATE : LEV_MATH_REFERENCE));
      const size_t psm = std::max(fsm, bsm);
      int per_sm = 0;
      pok = cudaFuncSetAttribute(pf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm) ==
                cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pf, kGridLPR * R, psm) ==
                cudaSuccess &&
            (long long)per_sm * sms >= 2LL * C;
    }
    cudaGetLastError();
    a->gp_ok[ri] = pok;
    a->gR_ok[ri] = true;
    a->g_cap[ri] = (int)cap;
    a->gf_smem[ri] = fsm;
    a->gb_smem[ri] = bsm;
    max_gpad = std::max(max_gpad, gpad);
    if (!a->grid_ok) a->grid_R = R;  // the smallest: the most SMs
    a->grid_ok = true;
  }
  if (!a->grid_ok) return LEV_OK;
  a->g_nwarps = nwarps;
  a->g_gpad = max_gpad;
  int rc = adj_alloc(a, &a->g_wsum, 2LL * nwarps);
  if (rc == LEV_OK) rc = adj_alloc(a, &a->g_lgp, 2LL * max_gpad);
  if (rc == LEV_OK) rc = adj_alloc(a, &a->g_bar, 2);
  if (rc != LEV_OK) return rc;
  LEV_TRY_CUDA(cudaMemset(a->g_wsum, 0, sizeof(float2) * 2 * (size_t)nwarps));
  LEV_TRY_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&a->h_gerr), sizeof(int),
                             cudaHostAllocMapped));
  *a->h_gerr = 0;
  LEV_TRY_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&a->d_gerr), a->h_gerr, 0));
  return LEV_OK;
}

// The checkpoint slots of segment `seg` for a grid-resident forward launch
// (mode 1: written from the initial state; 2: the initial state).
void adj_grid_ckpt_args(LevAdjoint *a, int seg, int mode, AdjGridFwdArgs &g) {
  g.ck_mode = mode;
  g.ck_theta = a->ck_theta + (size_t)seg * a->TN;
  g.ck_thh = a->ck_thh + (size_t)seg * a->TN;
  g.ck_omh = a->ck_omh + (size_t)seg * a->TN;
  g.ck_w = a->ck_w + (size_t)seg * a->SL;
  g.ck_ring = a->ck_ring + (size_t)seg * a->ckr_floats;  // one network: offset 0
  g.ck_g = a->ck_g + (size_t)seg * a->NN;
}

inline bool adj_grid_on(const LevAdjoint *a) {
  return a->grid_ok && a->use_grid && a->res_ra == nullptr;
}

int adj_grid_check(LevAdjoint *a) {
  if (a->h_gerr && *reinterpret_cast<volatile int *>(a->h_gerr)) {
    *a->h_gerr = 0;
    a->grid_ok = false;
    return fail(LEV_ERR_CUDA,
                "grid-resident adjoint segment: a grid barrier wait timed out; results are "
                "undefined");
  }
  return LEV_OK;
}

// The fields of a forward segment that do not depend on the segment.
void adj_grid_fill_fwd(LevAdjoint *a, AdjGridFwdArgs &f, int n) {
  LevEngine *e = a->e;
  const int ri = grid_r_index(a->grid_R);
  f.net = a->d_nets;
  f.st = a->d_st;
  f.row_ptr = e->d_row_ptr;
  f.sl_off = e->d_sl_off;
  f.sl_len = e->d_sl_len;
  f.sl_cd = e->d_sl_cd;
  f.theta = a->theta;
  f.theta_hat = a->theta_hat;
  f.omega = a->omega;
  f.omega_hat = a->omega_hat;
  f.wsum = a->g_wsum;
  f.bar = a->g_bar;
  f.err = a->d_gerr;
  f.wait = a->grid_wait;
  f.SL = a->SL;
  f.early = e->pair_ok ? 1 : 0;  // no delay is 0
  f.nwarps = a->g_nwarps;
  f.edge_cap = a->g_cap[ri];
  f.n_steps = n;
}

// One cooperative launch of the grid-resident forward over `n` steps (the
// per-step record pointers of f start at the segment's first step).
int adj_grid_launch_fwd(LevAdjoint *a, AdjGridFwdArgs f, int n, cudaStream_t s) {
  LevEngine *e = a->e;
  const int R = a->grid_R, ri = grid_r_index(R);
  LEV_TRY_CUDA(cudaMemsetAsync(a->g_bar, 0, sizeof(unsigned), s));
  adj_grid_fill_fwd(a, f, n);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((a->h_nets[0].N + R - 1) / R);
  cfg.blockDim = dim3(kGridLPR * R);
  cfg.dynamicSmemBytes = a->gf_smem[ri];
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LEV_TRY_CUDA(cudaLaunchKernelEx(&cfg, adj_grid_fwd_fn(R, e->math_mode), f));
  return LEV_OK;
}

// The fields of a reverse segment that do not depend on the segment.
void adj_grid_fill_bwd(LevAdjoint *a, AdjGridBwdArgs &b) {
  LevEngine *e = a->e;
  const int ri = grid_r_index(a->grid_R);
  b.net = a->d_nets;
  b.row_ptr = e->d_row_ptr;
  b.sl_off = e->d_sl_off;
  b.sl_len = e->d_sl_len;
  b.sl_cd = e->d_sl_cd;
  b.lam_th = a->lam_th;
  b.lam_thh = a->lam_thh;
  b.lam_omh = a->lam_omh;
  b.lam_w = a->lam_w;
  b.adj_ring = a->adj_ring;
  b.lam_g = a->lam_g;
  b.grad_omega = a->grad_omega_acc;
  b.lgp = a->g_lgp;
  b.bar = a->g_bar;
  b.err = a->d_gerr;
  b.wait = a->grid_wait;
  b.early = e->pair_ok ? 1 : 0;  // no delay is 0
  b.SL = a->SL;
  b.edge_cap = a->g_cap[ri];
}

// One cooperative launch of the grid-resident reverse over the steps of b.
int adj_grid_launch_bwd(LevAdjoint *a, AdjGridBwdArgs b, cudaStream_t s) {
  LevEngine *e = a->e;
  const int R = a->grid_R, ri = grid_r_index(R);
  LEV_TRY_CUDA(cudaMemsetAsync(a->g_bar, 0, sizeof(unsigned), s));
  adj_grid_fill_bwd(a, b);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((a->h_nets[0].N + R - 1) / R);
  cfg.blockDim = dim3(kGridLPR * R);
  cfg.dynamicSmemBytes = a->gb_smem[ri];
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LEV_TRY_CUDA(cudaLaunchKernelEx(&cfg, adj_grid_bwd_fn(R, e->math_mode), b));
  return LEV_OK;
}

// The paired backward launch: the forward segment f (n steps) on CTAs
// [0, C), the reverse segment b on CTAs [C, 2C), each group with its own
// barrier counter.
int adj_grid_launch_pair(LevAdjoint *a, AdjGridFwdArgs f, int n, AdjGridBwdArgs b,
                         cudaStream_t s) {
  LevEngine *e = a->e;
  const int R = a->grid_R, ri = grid_r_index(R);
  const int C = (a->h_nets[0].N + R - 1) / R;
  LEV_TRY_CUDA(cudaMemsetAsync(a->g_bar, 0, 2 * sizeof(unsigned), s));
  adj_grid_fill_fwd(a, f, n);
  adj_grid_fill_bwd(a, b);
  f.bar = a->g_bar;
  b.bar = a->g_bar + 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * C);
  cfg.blockDim = dim3(kGridLPR * R);
  cfg.dynamicSmemBytes = std::max(a->gf_smem[ri], a->gb_smem[ri]);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LEV_TRY_CUDA(cudaLaunchKernelEx(&cfg, adj_grid_pair_fn(R, e->math_mode), f, b, C));
  return LEV_OK;
}

}  // namespace

extern "C" {

int lev_adj_create(LevAdjoint **out, LevEngine *e, int32_t segment,
                   int32_t max_steps) {
  if (!out || !e) return fail(LEV_ERR_ARG, "null argument");
  *out = nullptr;
  if (e->part) return fail(LEV_ERR_STATE, "partition engine: not supported");
  if (segment < 1 || max_steps < 1)
    return fail(LEV_ERR_ARG, "segment and max_steps must be >= 1");
  DeviceScope ds(e->device);
  LevAdjoint *a = new LevAdjoint();
  a->e = e;
  a->C = segment;
  a->Tmax = max_steps;
  a->nseg = (max_steps + segment - 1) / segment;
  a->TN = e->total_nodes;
  a->SL = e->sl_total;
  a->NN = e->num_nets;
  a->h_nets = e->h_nets;
  std::vector<long long> ck_off(a->NN);
  for (int n = 0; n < a->NN; ++n) {
    NetDesc &d = a->h_nets[n];
    d.bsi = segment + d.max_delay + 2;
    d.ring_off = a->ring_floats;
    d.aux_off = a->aux_floats;
    a->ring_floats += (long long)d.bsi * d.Np;
    a->aux_floats += (long long)(d.max_delay + 2) * d.Np;
    ck_off[n] = a->ckr_floats;
    a->ckr_floats += (long long)(d.max_delay + 1) * d.N;
    if ((unsigned long long)d.bsi * (unsigned long long)d.Np >= (1ull << 32)) {
      delete a;
      return fail(LEV_ERR_ARG, "adjoint: (segment + max_delay + 2) * N must be below 2^32");
    }
  }
  const long long TN = a->TN, SL = a->SL, NN = a->NN;
  const long long S = a->nseg, C = a->C;
  int rc = LEV_OK;
#define A(ptr, n) \
  if (rc == LEV_OK) rc = adj_alloc(a, &(ptr), (n));
  A(a->d_nets, NN);
  A(a->d_st, NN);
  A(a->d_ck_off, NN);
  A(a->theta0, TN); A(a->theta_hat0, TN);
  A(a->theta, TN); A(a->theta_hat, TN); A(a->omega, TN); A(a->omega_hat, TN);
  A(a->w, SL);
  A(a->ring, a->ring_floats);
  A(a->partials, e->total_tiles);
  A(a->bpart, 4LL * e->total_tiles);  // up to four partials per tile
  A(a->ro_partials, e->total_tiles);
  A(a->tickets, NN);
  A(a->ck_theta, S * TN); A(a->ck_thh, S * TN); A(a->ck_omh, S * TN);
  A(a->ck_w, S * SL);
  A(a->ck_ring, S * a->ckr_floats);
  A(a->ck_g, S * NN);
  A(a->w_hist, (C + 1) * SL);
  A(a->thh_hist, C * TN);
  A(a->trace, C * NN);
  const bool dj_rec = e->total_tiles > 148;  // adj_fwd_kernel / adj_bwd_kernel
  if (dj_rec) A(a->dj_hist, C * SL);
  A(a->lam_th, TN); A(a->lam_thh, TN); A(a->lam_omh, TN);
  A(a->lam_w, SL);
  A(a->adj_ring, a->aux_floats);
  A(a->lam_g, NN);
  A(a->grad_omega_acc, TN);
  A(a->grad_theta0, TN);
  if (rc == LEV_OK && S > 1) {
    // optional second record set; without it the backward pass runs the
    // recompute and the reverse steps of each segment one after the other
    size_t fr = 0, tot = 0;
    const size_t need = sizeof(float) * ((size_t)a->ring_floats + (size_t)(C + 1) * SL +
                                         (size_t)C * TN + (dj_rec ? (size_t)C * SL : 0)) +
                        sizeof(float4) * (size_t)C * NN;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && need + (256ull << 20) < fr) {
      A(a->ring2, a->ring_floats);
      A(a->w_hist2, (C + 1) * SL);
      if (dj_rec) A(a->dj_hist2, C * SL);
      A(a->thh_hist2, C * TN);
      A(a->trace2, C * NN);
      if (rc == LEV_OK &&
          (cudaStreamCreateWithFlags(&a->rstream, cudaStreamNonBlocking) != cudaSuccess ||
           cudaEventCreateWithFlags(&a->ev_rec[0], cudaEventDisableTiming) != cudaSuccess ||
           cudaEventCreateWithFlags(&a->ev_rec[1], cudaEventDisableTiming) != cudaSuccess ||
           cudaEventCreateWithFlags(&a->ev_rev[0], cudaEventDisableTiming) != cudaSuccess ||
           cudaEventCreateWithFlags(&a->ev_rev[1], cudaEventDisableTiming) != cudaSuccess ||
           cudaEventCreateWithFlags(&a->ev_start, cudaEventDisableTiming) != cudaSuccess))
        rc = fail(LEV_ERR_CUDA, "adjoint: stream or event creation failed");
    }
  }
#undef A
  if (rc == LEV_OK && NN == 1) {
    std::vector<long long> h_off(e->num_slices);
    std::vector<int> h_len(e->num_slices);
    if (cudaMemcpy(h_off.data(), e->d_sl_off, sizeof(long long) * e->num_slices,
                   cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(h_len.data(), e->d_sl_len, sizeof(int) * e->num_slices,
                   cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = fail(LEV_ERR_CUDA, "adjoint: reading the SELL slice table failed");
    else
      rc = adj_setup_grid(a, h_off, h_len);
  }
  if (rc != LEV_OK) {
    std::string msg = g_last_error;
    adj_free(a);
    return fail(rc, msg);
  }
  cudaStream_t s = e->stream;
  cudaError_t ce = cudaMemcpyAsync(a->d_nets, a->h_nets.data(), sizeof(NetDesc) * NN,
                                   cudaMemcpyHostToDevice, s);
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(a->d_ck_off, ck_off.data(), sizeof(long long) * NN,
                         cudaMemcpyHostToDevice, s);
  // initial conditions: the engine's current phases and predictor phases
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(a->theta0, e->d_theta, sizeof(float) * TN,
                         cudaMemcpyDeviceToDevice, s);
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(a->theta_hat0, e->d_theta_hat, sizeof(float) * TN,
                         cudaMemcpyDeviceToDevice, s);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(a->tickets, 0, sizeof(unsigned) * NN, s);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
  if (ce != cudaSuccess) {
    adj_free(a);
    return fail(LEV_ERR_CUDA, std::string("adjoint set-up: ") + cudaGetErrorString(ce));
  }
  *out = a;
  return LEV_OK;
}

int lev_adj_destroy(LevAdjoint *a) {
  if (!a) return LEV_OK;
  DeviceScope ds(a->e->device);
  cudaStreamSynchronize(a->e->stream);
  adj_free(a);
  return LEV_OK;
}

int lev_adj_bytes(const LevAdjoint *a, size_t *bytes) {
  if (!a || !bytes) return fail(LEV_ERR_ARG, "null argument");
  *bytes = a->bytes;
  return LEV_OK;
}

int lev_adj_forward(LevAdjoint *a, float dt, int32_t T, const float *omega,
                    const float *w0_csr, const float *K, const float *drive,
                    float *r_out, float *theta_out) {
  if (!a || !omega || !w0_csr || !K || !r_out)
    return fail(LEV_ERR_ARG, "null argument");
  if (T < 1 || T > a->Tmax)
    return fail(LEV_ERR_ARG, "T must be in [1, max_steps]");
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  LevEngine *e = a->e;
  DeviceScope ds(e->device);
  cudaStream_t s = e->stream;
  const size_t nb = sizeof(float) * a->TN;
  LEV_TRY_CUDA(cudaMemcpyAsync(a->theta, a->theta0, nb, cudaMemcpyDeviceToDevice, s));
  LEV_TRY_CUDA(cudaMemcpyAsync(a->theta_hat, a->theta_hat0, nb, cudaMemcpyDeviceToDevice, s));
  LEV_TRY_CUDA(cudaMemcpyAsync(a->omega, omega, nb, cudaMemcpyDeviceToDevice, s));
  // omega_hat starts as omega (leviathan_kernel.cu:350)
  LEV_TRY_CUDA(cudaMemcpyAsync(a->omega_hat, omega, nb, cudaMemcpyDeviceToDevice, s));
  LEV_TRY_CUDA(cudaMemsetAsync(a->w, 0, sizeof(float) * std::max<long long>(a->SL, 1), s));
  for (int n = 0; n < a->NN; ++n) {
    const NetDesc &d = a->h_nets[n];
    if (e->net_E[n] == 0) continue;
    int blocks = (int)std::min<long long>((d.N + 255) / 256, 148LL * 16);
    sell_convert_kernel<<<blocks, 256, 0, s>>>(
        1, e->d_row_ptr + d.rp_off, d.N, d.N, d.slice_base, e->d_sl_off, nullptr,
        nullptr, const_cast<float *>(w0_csr) + d.edge_off, e->d_sl_cd, a->w,
        d.max_delay, nullptr);
    const long long total = (long long)d.bsi * d.N;
    int fb = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    ring_fill_kernel<<<fb, 256, 0, s>>>(a->theta0 + d.node_off, a->ring + d.ring_off,
                                       d.N, d.Np, d.bsi, 0, 0);  // slot-major
  }
  adj_state_kernel<<<1, 128, 0, s>>>(0, a->d_nets, a->d_st, nullptr, K, a->NN);
  LEV_TRY_CUDA(cudaGetLastError());
  if (adj_grid_on(a)) {
    // one cooperative launch per checkpoint segment, which also writes the
    // segment's checkpoint
    for (int t0 = 0; t0 < T; t0 += a->C) {
      const int n = std::min(a->C, T - t0);
      AdjGridFwdArgs g;
      std::memset(&g, 0, sizeof(g));
      adj_grid_ckpt_args(a, t0 / a->C, 1, g);
      g.w_in = a->w;
      g.w_out = a->w;
      g.ring = a->ring;
      g.drive = drive ? drive + (size_t)t0 * a->TN : nullptr;
      if (a->res_win) {
        g.win = a->res_win;
        g.xin = a->res_x + (size_t)t0 * a->NN;
      }
      g.r_out = r_out + (size_t)t0 * a->NN;
      g.theta_out = theta_out ? theta_out + (size_t)t0 * a->TN : nullptr;
      g.dt = dt;
      int rc = adj_grid_launch_fwd(a, g, n, s);
      if (rc != LEV_OK) return rc;
    }
    LEV_TRY_CUDA(cudaStreamSynchronize(s));
    int rc = adj_grid_check(a);
    if (rc != LEV_OK) return rc;
    a->last_T = T;
    a->last_dt = dt;
    a->drive = drive;
    return LEV_OK;
  }
  AdjFwdArgs f = adj_fwd_args(a, dt);
  f.drive = nullptr;
  for (int t = 0; t < T; ++t) {
    if (t % a->C == 0) {
      int rc = adj_ckpt(a, t / a->C, true);
      if (rc != LEV_OK) return rc;
    }
    f.drive = drive ? drive + (size_t)t * a->TN : nullptr;
    f.r_out = r_out + (size_t)t * a->NN;
    f.theta_out = theta_out ? theta_out + (size_t)t * a->TN : nullptr;
    if (a->res_win) {
      f.win = a->res_win;
      f.xin = a->res_x + (size_t)t * a->NN;
    }
    if (a->res_ra) {
      f.ra = a->res_ra;
      f.rb = a->res_rb;
      f.ro_partials = a->ro_partials;
      f.y_out = a->res_y ? a->res_y + (size_t)t * a->NN : nullptr;
    }
    int rc = adj_launch_fwd(a, f);
    if (rc != LEV_OK) return rc;
  }
  LEV_TRY_CUDA(cudaStreamSynchronize(s));
  a->last_T = T;
  a->last_dt = dt;
  a->drive = drive;
  return LEV_OK;
}

int lev_adj_backward(LevAdjoint *a, const float *dLdr, const float *dLdtheta,
                     float *grad_omega, float *grad_w0_csr, float *grad_K,
                     float *grad_drive) {
  if (!a) return fail(LEV_ERR_ARG, "null handle");
  if (a->last_T < 1) return fail(LEV_ERR_STATE, "lev_adj_backward before lev_adj_forward");
  LevEngine *e = a->e;
  DeviceScope ds(e->device);
  cudaStream_t s = e->stream;
  const int T = a->last_T;
  const float dt = a->last_dt;
  const size_t nb = sizeof(float) * a->TN;
  const size_t wb = sizeof(float) * std::max<long long>(a->SL, 1);
  LEV_TRY_CUDA(cudaMemsetAsync(a->lam_th, 0, nb, s));
  LEV_TRY_CUDA(cudaMemsetAsync(a->lam_thh, 0, nb, s));
  LEV_TRY_CUDA(cudaMemsetAsync(a->lam_omh, 0, nb, s));
  LEV_TRY_CUDA(cudaMemsetAsync(a->grad_omega_acc, 0, nb, s));
  LEV_TRY_CUDA(cudaMemsetAsync(a->lam_w, 0, wb, s));
  LEV_TRY_CUDA(cudaMemsetAsync(a->adj_ring, 0, sizeof(float) * std::max<long long>(a->aux_floats, 1), s));
  LEV_TRY_CUDA(cudaMemsetAsync(a->lam_g, 0, sizeof(float) * a->NN, s));
  LEV_TRY_CUDA(cudaMemsetAsync(a->tickets, 0, sizeof(unsigned) * a->NN, s));
  if (a->res_gwin) LEV_TRY_CUDA(cudaMemsetAsync(a->res_gwin, 0, nb, s));
  if (a->res_gra) LEV_TRY_CUDA(cudaMemsetAsync(a->res_gra, 0, nb, s));
  if (a->res_grb) LEV_TRY_CUDA(cudaMemsetAsync(a->res_grb, 0, nb, s));
  const int nseg = (T + a->C - 1) / a->C;
  const int mode = (e->math_mode == LEV_MATH_ACCURATE) ? 1 : 0;
  if (adj_grid_on(a)) {
    // Segments last to first.  Segment k's records go to set k & 1 when a
    // second set exists.  Recompute of segment k-1 and reverse of segment k
    // share one paired launch when both groups fit on the device; otherwise
    // each segment is recomputed, then reversed, in launches of their own.
    const bool two = a->ring2 != nullptr;
    const bool paired = two && a->use_pair && a->gp_ok[grid_r_index(a->grid_R)] && nseg > 1;
    float *rings[2] = {a->ring, two ? a->ring2 : a->ring};
    float *whs[2] = {a->w_hist, two ? a->w_hist2 : a->w_hist};
    float *ths[2] = {a->thh_hist, two ? a->thh_hist2 : a->thh_hist};
    float4 *trs[2] = {a->trace, two ? a->trace2 : a->trace};
    auto seg_len = [&](int seg) { return std::min(T, seg * a->C + a->C) - seg * a->C; };
    // the recompute of segment `seg` (restored from its checkpoint by the
    // launch itself) into its record set
    auto prep_fwd = [&](int seg, AdjGridFwdArgs &g) -> int {
      const int s0 = seg * a->C, n = seg_len(seg), k = paired ? (seg & 1) : 0;
      std::memset(&g, 0, sizeof(g));
      adj_grid_ckpt_args(a, seg, 2, g);
      g.w0_out = whs[k];
      g.w_in = whs[k];
      g.w_rec = whs[k] + a->SL;
      g.w_out = whs[k] + (size_t)n * a->SL;
      g.ring = rings[k];
      g.drive = a->drive ? a->drive + (size_t)s0 * a->TN : nullptr;
      if (a->res_win) {
        g.win = a->res_win;
        g.xin = a->res_x + (size_t)s0 * a->NN;
      }
      g.thh_rec = ths[k];
      g.trace = trs[k];
      g.dt = dt;
      return LEV_OK;
    };
    auto prep_bwd = [&](int seg, AdjGridBwdArgs &b) {
      const int k = paired ? (seg & 1) : 0;
      std::memset(&b, 0, sizeof(b));
      b.w_hist = whs[k];
      b.H = rings[k];
      b.thh_hist = ths[k];
      b.trace = trs[k];
      b.dLdr = dLdr;
      b.dLdth = dLdtheta;
      b.grad_drive = grad_drive;
      if (a->res_win) {
        b.win = a->res_win;
        b.xin = a->res_x;
        b.grad_win = a->res_gwin;
      }
      b.seg_start = (long long)seg * a->C;
      b.n_steps = seg_len(seg);
      b.dt = dt;
    };
    AdjGridFwdArgs g;
    AdjGridBwdArgs b;
    int rc = LEV_OK;
    if (paired) {
      rc = prep_fwd(nseg - 1, g);
      if (rc == LEV_OK) rc = adj_grid_launch_fwd(a, g, seg_len(nseg - 1), s);
      for (int seg = nseg - 1; seg >= 0 && rc == LEV_OK; --seg) {
        prep_bwd(seg, b);
        if (seg > 0) {
          rc = prep_fwd(seg - 1, g);
          if (rc == LEV_OK) rc = adj_grid_launch_pair(a, g, seg_len(seg - 1), b, s);
        } else {
          rc = adj_grid_launch_bwd(a, b, s);
        }
      }
    } else {
      for (int seg = nseg - 1; seg >= 0 && rc == LEV_OK; --seg) {
        rc = prep_fwd(seg, g);
        if (rc == LEV_OK) rc = adj_grid_launch_fwd(a, g, seg_len(seg), s);
        prep_bwd(seg, b);
        if (rc == LEV_OK) rc = adj_grid_launch_bwd(a, b, s);
      }
    }
    if (rc != LEV_OK) return rc;
  } else {
  // Segment k-1 is recomputed (stream rs, record set (k-1)&1) while segment k
  // is reversed (engine stream, record set k&1), when the second set exists.
  const bool overlap = a->rstream != nullptr && nseg > 1;
  float *rings[2] = {a->ring, overlap ? a->ring2 : a->ring};
  float *whs[2] = {a->w_hist, overlap ? a->w_hist2 : a->w_hist};
  float *ths[2] = {a->thh_hist, overlap ? a->thh_hist2 : a->thh_hist};
  float4 *trs[2] = {a->trace, overlap ? a->trace2 : a->trace};
  float *djs[2] = {a->dj_hist, overlap ? a->dj_hist2 : a->dj_hist};
  cudaStream_t rs = overlap ? a->rstream : s;
  if (overlap) {
    LEV_TRY_CUDA(cudaEventRecord(a->ev_start, s));
    LEV_TRY_CUDA(cudaStreamWaitEvent(rs, a->ev_start, 0));
  }
  // recompute a segment forward, recording what its reverse steps need
  auto recompute = [&](int seg) -> int {
    const int buf = seg & 1;
    const int s0 = seg * a->C, s1 = std::min(T, s0 + a->C);
    int rc = adj_ckpt(a, seg, false, rs, rings[buf]);
    if (rc != LEV_OK) return rc;
    LEV_TRY_CUDA(cudaMemcpyAsync(whs[buf], a->w, wb, cudaMemcpyDeviceToDevice, rs));
    AdjFwdArgs f = adj_fwd_args(a, dt);
    f.ring = rings[buf];
    for (int t = s0; t < s1; ++t) {
      const int k = t - s0;
      f.w_in = whs[buf] + (size_t)k * a->SL;
      f.w_out = whs[buf] + (size_t)(k + 1) * a->SL;
      f.thh_rec = ths[buf] + (size_t)k * a->TN;
      f.dj_rec = djs[buf] ? djs[buf] + (size_t)k * a->SL : nullptr;
      f.trace = trs[buf] + (size_t)k * a->NN;
      f.drive = a->drive ? a->drive + (size_t)t * a->TN : nullptr;
      f.r_out = nullptr;
      f.theta_out = nullptr;
      if (a->res_win) {
        f.win = a->res_win;
        f.xin = a->res_x + (size_t)t * a->NN;
      }
      rc = adj_launch_fwd(a, f, rs);
      if (rc != LEV_OK) return rc;
    }
    if (overlap) LEV_TRY_CUDA(cudaEventRecord(a->ev_rec[buf], rs));
    return LEV_OK;
  };
  bool rev_recorded[2] = {false, false};
  int rc = recompute(nseg - 1);
  if (rc != LEV_OK) return rc;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int buf = seg & 1;
    const int s0 = seg * a->C, s1 = std::min(T, s0 + a->C);
    if (overlap) LEV_TRY_CUDA(cudaStreamWaitEvent(s, a->ev_rec[buf], 0));
    // reverse steps
    AdjBwdArgs b;
    std::memset(&b, 0, sizeof(b));
    b.nets = a->d_nets;
    b.tiles = e->d_tiles;
    b.row_ptr = e->d_row_ptr;
    b.sl_off = e->d_sl_off;
    b.sl_len = e->d_sl_len;
    b.sl_cd = e->d_sl_cd;
    b.H = rings[buf];
    b.lam_th = a->lam_th;
    b.lam_thh = a->lam_thh;
    b.lam_omh = a->lam_omh;
    b.lam_w = a->lam_w;
    b.adj_ring = a->adj_ring;
    b.lam_g = a->lam_g;
    b.grad_omega = a->grad_omega_acc;
    b.partials = a->bpart;
    b.tickets = a->tickets;
    b.seg_start = s0;
    b.dt = dt;
    for (int t = s1 - 1; t >= s0; --t) {
      const int k = t - s0;
      b.s = t;
      b.w_s = whs[buf] + (size_t)k * a->SL;
      b.dj_s = djs[buf] ? djs[buf] + (size_t)k * a->SL : nullptr;
      b.thh_s = ths[buf] + (size_t)k * a->TN;
      b.trace = trs[buf] + (size_t)k * a->NN;
      b.dLdr = dLdr ? dLdr + (size_t)t * a->NN : nullptr;
      b.dLdth = dLdtheta ? dLdtheta + (size_t)t * a->TN : nullptr;
      b.grad_drive = grad_drive ? grad_drive + (size_t)t * a->TN : nullptr;
      if (a->res_win) {
        b.win = a->res_win;
        b.xin = a->res_x + (size_t)t * a->NN;
        b.grad_win = a->res_gwin;
      }
      if (a->res_ra && a->res_dLdy) {
        b.ra = a->res_ra;
        b.rb = a->res_rb;
        b.dLdy = a->res_dLdy + (size_t)t * a->NN;
        b.grad_ra = a->res_gra;
        b.grad_rb = a->res_grb;
      }
      // measured on B200: grids of many waves (batch-64 reservoir) run best
      // at 5 CTAs/SM with 6 edges in flight per lane (fwd+bwd 1.75-1.77 s;
      // 4 CTAs/SM with 4 edges 2.00 s, 6 with 4 1.77 s, 7 or 8 spill: 2.00 s);
      // a grid of one partial wave (N = 10^4) with four lanes per row
      if (e->total_tiles <= 148) {
        const int g4 = e->total_tiles * 4;
        if (mode) adj_bwd_split_kernel<1, 4, 2><<<g4, kTile, 0, s>>>(b);
        else adj_bwd_split_kernel<0, 4, 2><<<g4, kTile, 0, s>>>(b);
      } else if (e->total_tiles > 3 * 148 * 2) {
        if (mode) adj_bwd_kernel<1, 6, 5><<<e->total_tiles, kTile, 0, s>>>(b);
        else adj_bwd_kernel<0, 6, 5><<<e->total_tiles, kTile, 0, s>>>(b);
      } else {
        if (mode) adj_bwd_kernel<1, 8, 3><<<e->total_tiles, kTile, 0, s>>>(b);
        else adj_bwd_kernel<0, 8, 3><<<e->total_tiles, kTile, 0, s>>>(b);
      }
      LEV_TRY_CUDA(cudaGetLastError());
    }
    if (overlap) {
      LEV_TRY_CUDA(cudaEventRecord(a->ev_rev[buf], s));
      rev_recorded[buf] = true;
    }
    if (seg > 0) {
      // the record set of segment seg-1 was last read by the reverse of seg+1
      const int nbuf = (seg - 1) & 1;
      if (overlap && rev_recorded[nbuf])
        LEV_TRY_CUDA(cudaStreamWaitEvent(rs, a->ev_rev[nbuf], 0));
      rc = recompute(seg - 1);
      if (rc != LEV_OK) return rc;
    }
  }
  }  // per-step launches
  // gradients
  dim3 grid(64, a->NN);
  adj_finalize_kernel<<<grid, 256, 0, s>>>(a->d_nets, a->NN, a->lam_th, a->adj_ring,
                                           a->grad_theta0);
  if (grad_omega) {
    // omega enters directly and through omega_hat(0) = omega
    LEV_TRY_CUDA(cudaMemcpyAsync(grad_omega, a->grad_omega_acc, nb, cudaMemcpyDeviceToDevice, s));
    add_kernel<<<148, 256, 0, s>>>(grad_omega, a->lam_omh, a->TN);
  }
  if (grad_w0_csr) {
    for (int n = 0; n < a->NN; ++n) {
      const NetDesc &d = a->h_nets[n];
      if (e->net_E[n] == 0) continue;
      int blocks = (int)std::min<long long>((d.N + 255) / 256, 148LL * 16);
      sell_convert_kernel<<<blocks, 256, 0, s>>>(
          2, e->d_row_ptr + d.rp_off, d.N, d.N, d.slice_base, e->d_sl_off, nullptr, nullptr,
          grad_w0_csr + d.edge_off, e->d_sl_cd, a->lam_w, d.max_delay, nullptr);
    }
  }
  if (grad_K)
    LEV_TRY_CUDA(cudaMemcpyAsync(grad_K, a->lam_g, sizeof(float) * a->NN,
                                 cudaMemcpyDeviceToDevice, s));
  LEV_TRY_CUDA(cudaGetLastError());
  LEV_TRY_CUDA(cudaStreamSynchronize(s));
  return adj_grid_check(a);
}

int lev_adj_grid_info(const LevAdjoint *a, int32_t *eligible, int32_t *enabled,
                      int32_t *rows_per_cta, int32_t *eligible_rows_mask, int32_t *paired) {
  if (!a) return fail(LEV_ERR_ARG, "null handle");
  if (eligible) *eligible = a->grid_ok ? 1 : 0;
  if (enabled) *enabled = adj_grid_on(a) ? 1 : 0;
  if (rows_per_cta) *rows_per_cta = a->grid_ok ? a->grid_R : 0;
  if (paired)
    *paired = (adj_grid_on(a) && a->use_pair && a->ring2 != nullptr &&
               a->gp_ok[grid_r_index(a->grid_R)]) ? 1 : 0;
  if (eligible_rows_mask) {
    int m = 0;
    for (int i = 0; i < 3; ++i)
      if (a->gR_ok[i]) m |= kGridRs[i];
    *eligible_rows_mask = m;
  }
  return LEV_OK;
}

int lev_adj_set_grid_wait(LevAdjoint *a, uint64_t limit_ns, uint32_t extra_arrivals) {
  if (!a) return fail(LEV_ERR_ARG, "null handle");
  int rc = check_wait_args(limit_ns, extra_arrivals);
  if (rc != LEV_OK) return rc;
  a->grid_wait.ns = limit_ns;
  a->grid_wait.extra = extra_arrivals;
  return LEV_OK;
}

int lev_adj_set_grid_pairing(LevAdjoint *a, int32_t enabled) {
  if (!a) return fail(LEV_ERR_ARG, "null handle");
  a->use_pair = enabled != 0;
  return LEV_OK;
}

int lev_adj_set_grid_mode(LevAdjoint *a, int32_t enabled, int32_t rows_per_cta) {
  if (!a) return fail(LEV_ERR_ARG, "null handle");
  if (rows_per_cta != 0) {
    if (rows_per_cta != 64 && rows_per_cta != 128 && rows_per_cta != 256)
      return fail(LEV_ERR_ARG, "rows_per_cta must be 0, 64, 128 or 256");
    if (!a->gR_ok[grid_r_index(rows_per_cta)])
      return fail(LEV_ERR_ARG, "rows_per_cta not eligible for this adjoint");
    a->grid_R = rows_per_cta;
  }
  a->use_grid = enabled != 0;
  return LEV_OK;
}

int lev_adj_set_reservoir(LevAdjoint *a, const float *win, const float *x,
                          const float *ra, const float *rb, float *y_out) {
  if (!a) return fail(LEV_ERR_ARG, "null handle");
  if ((win == nullptr) != (x == nullptr))
    return fail(LEV_ERR_ARG, "win and x must be given together");
  if ((ra == nullptr) != (rb == nullptr))
    return fail(LEV_ERR_ARG, "ra and rb must be given together");
  a->res_win = win;
  a->res_x = x;
  a->res_ra = ra;
  a->res_rb = rb;
  a->res_y = y_out;
  return LEV_OK;
}

int lev_adj_set_reservoir_grads(LevAdjoint *a, const float *dLdy,
                                float *grad_win, float *grad_ra,
                                float *grad_rb) {
  if (!a) return fail(LEV_ERR_ARG, "null handle");
  if (grad_win && !a->res_win)
    return fail(LEV_ERR_STATE, "no input weights set (lev_adj_set_reservoir)");
  if ((dLdy || grad_ra || grad_rb) && !a->res_ra)
    return fail(LEV_ERR_STATE, "no readout set (lev_adj_set_reservoir)");
  a->res_dLdy = dLdy;
  a->res_gwin = grad_win;
  a->res_gra = grad_ra;
  a->res_grb = grad_rb;
  return LEV_OK;
}

int lev_adj_grad_theta0(LevAdjoint *a, float *grad_theta0) {
  if (!a || !grad_theta0) return fail(LEV_ERR_ARG, "null argument");
  DeviceScope ds(a->e->device);
  LEV_TRY_CUDA(cudaMemcpyAsync(grad_theta0, a->grad_theta0, sizeof(float) * a->TN,
                               cudaMemcpyDeviceToDevice, a->e->stream));
  LEV_TRY_CUDA(cudaStreamSynchronize(a->e->stream));
  return LEV_OK;
}

}  // extern "C"

// ===========================================================================
// Partition of a network split over GPUs (lev_part.cuh)
// ===========================================================================
extern "C" {

int lev_part_create(LevEngine **out, int32_t N, int32_t n_halo, int32_t max_delay,
                    const int32_t *row_ptr, const int32_t *col_idx,
                    const uint8_t *delays, const float *weights,
                    const float *theta, const float *theta_hat,
                    const float *omega, const float *theta_halo,
                    int32_t N_global, int32_t tile_off_global,
                    int32_t ntiles_global, const LevParams *params,
                    int32_t math_mode) {
  if (!out) return fail(LEV_ERR_ARG, "out is null");
  *out = nullptr;
  if (n_halo < 0) return fail(LEV_ERR_ARG, "n_halo must be >= 0");
  if (n_halo > 0 && !theta_halo) return fail(LEV_ERR_ARG, "theta_halo is null");
  if (N < 1 || N_global < N || tile_off_global < 0 || ntiles_global < 1 ||
      (long long)tile_off_global * kTile + N > (long long)N_global ||
      ntiles_global != (N_global + kTile - 1) / kTile)
    return fail(LEV_ERR_ARG,
                "partition: need 1 <= N, rows [256 * tile_off_global, + N) inside "
                "N_global, ntiles_global = ceil(N_global / 256)");
  if ((long long)tile_off_global * kTile + N < (long long)N_global && N % kTile != 0)
    return fail(LEV_ERR_ARG, "partition: every partition but the last must own whole "
                             "256-row tiles");
  // a halo column that no edge reads is allowed (its phases are just kept)
  LevEngine *h = nullptr;
  int rc = create_impl(&h, 1, &N, &max_delay, row_ptr, col_idx, delays, weights,
                       theta, theta_hat, omega, params, math_mode, n_halo,
                       theta_halo);
  if (rc != LEV_OK) return rc;
  DeviceScope ds(h->device);
  h->part = true;
  h->part_halo = n_halo;
  h->part_N_global = N_global;
  h->part_tile_off = tile_off_global;
  h->part_ntiles_global = ntiles_global;
  // steps driven by the host (lev_part_step_*, lev_part_pair_*) with the
  // whole-network reduction on gathered partials: none of the block paths;
  // pair_ok (no zero delay) stays as creation found it
  h->cluster_ok = false;
  h->use_cluster = false;
  h->grid_ok = false;
  h->use_grid = false;
  h->h_nets[0].dist = 1;
  h->h_nets[0].part_off = tile_off_global;
  cudaError_t e = cudaMemcpyAsync(h->d_nets, h->h_nets.data(), sizeof(NetDesc),
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    free_engine(h);
    return fail(LEV_ERR_CUDA, std::string("partition set-up: ") + cudaGetErrorString(e));
  }
  *out = h;
  return LEV_OK;
}

static int part_check(const LevEngine *h) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (!h->part) return fail(LEV_ERR_STATE, "not a partition engine (lev_part_create)");
  return LEV_OK;
}

int lev_part_info(const LevEngine *h, int32_t *n_halo, int32_t *N_global,
                  int32_t *tile_off_global, int32_t *ntiles_global) {
  if (!h) return fail(LEV_ERR_ARG, "null handle");
  if (n_halo) *n_halo = h->part ? h->part_halo : 0;
  if (N_global) *N_global = h->part ? h->part_N_global : (int32_t)h->total_nodes;
  if (tile_off_global) *tile_off_global = h->part ? h->part_tile_off : 0;
  if (ntiles_global) *ntiles_global = h->part ? h->part_ntiles_global : h->total_tiles;
  return h->part ? LEV_OK : fail(LEV_ERR_STATE, "not a partition engine");
}

int lev_part_step_begin(LevEngine *h, float dt, void *partials_dev) {
  int rc = part_check(h);
  if (rc != LEV_OK) return rc;
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  if (!partials_dev) return fail(LEV_ERR_ARG, "partials buffer is null");
  DeviceScope ds(h->device);
  StepArgs a = make_args(h, dt, nullptr, 0, nullptr);
  a.partials = static_cast<float2 *>(partials_dev);
  a.hubs = nullptr;
  return launch_step(h, a);
}

int lev_part_step_end(LevEngine *h, float dt, const void *partials_all_dev,
                      float *r_dev) {
  int rc = part_check(h);
  if (rc != LEV_OK) return rc;
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  if (!partials_all_dev) return fail(LEV_ERR_ARG, "partials buffer is null");
  DeviceScope ds(h->device);
  part_finish_kernel<<<1, kReduceThreads, 0, h->stream>>>(
      h->d_nets, h->d_st, static_cast<const float2 *>(partials_all_dev),
      h->part_ntiles_global, h->part_N_global, dt, r_dev, h->d_rmap);
  LEV_TRY_CUDA(cudaGetLastError());
  return LEV_OK;
}

// The single degree class of a partition engine that takes two steps per
// launch with a one-lane pair variant, or -1.
static int part_pair_class(const LevEngine *h) {
  if (!pairs_all(h)) return -1;
  for (int c = 0; c < kNumClasses; ++c) {
    const TileClass &tc = h->classes[c];
    if (tc.ntiles > 0) return kPairVariants[tc.pair_variant].LANES == 1 ? c : -1;
  }
  return -1;
}

int lev_part_pairs(const LevEngine *h, int32_t *eligible) {
  int rc = part_check(h);
  if (rc != LEV_OK) return rc;
  if (!eligible) return fail(LEV_ERR_ARG, "null argument");
  *eligible = part_pair_class(h) >= 0 ? 1 : 0;
  return LEV_OK;
}

// Two steps of a partition per pair of launches, as the single engine takes
// them (lev_pair.cuh), with the whole-network reduction of each step done by
// lev_part_step_end on the all-gathered partials instead of reduce_kernel.
int lev_part_pair_begin(LevEngine *h, float dt, void *partials_dev) {
  int rc = part_check(h);
  if (rc != LEV_OK) return rc;
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  if (!partials_dev) return fail(LEV_ERR_ARG, "partials buffer is null");
  const int c = part_pair_class(h);
  if (c < 0) return fail(LEV_ERR_STATE, "partition engine: two steps per launch not eligible");
  DeviceScope ds(h->device);
  StepArgs a = make_args(h, dt, nullptr, 0, nullptr);
  a.partials = static_cast<float2 *>(partials_dev);
  a.hubs = nullptr;
  a.reverse = h->sweep;
  h->sweep ^= 1;
  const TileClass &tc = h->classes[c];
  a.tiles = h->d_tiles + tc.tile_off;
  const int mode = (h->math_mode == LEV_MATH_ACCURATE) ? 1 : 0;
  void *args[] = {&a};
  LEV_TRY_CUDA(cudaLaunchKernel(reinterpret_cast<const void *>(kPairVariants[tc.pair_variant].fn[mode]),
                                dim3(tc.ntiles), dim3(kTile), args, 0, h->stream));
  return LEV_OK;
}

int lev_part_pair_finish(LevEngine *h, float dt, void *partials_dev) {
  int rc = part_check(h);
  if (rc != LEV_OK) return rc;
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "dt is not finite");
  if (!partials_dev) return fail(LEV_ERR_ARG, "partials buffer is null");
  const int c = part_pair_class(h);
  if (c < 0) return fail(LEV_ERR_STATE, "partition engine: two steps per launch not eligible");
  DeviceScope ds(h->device);
  StepArgs a = make_args(h, dt, nullptr, 0, nullptr);
  a.partials = static_cast<float2 *>(partials_dev);
  a.hubs = nullptr;
  a.reverse = h->sweep;
  h->sweep ^= 1;
  const TileClass &tc = h->classes[c];
  a.tiles = h->d_tiles + tc.tile_off;
  const int blocks = (tc.ntiles + kFinishTiles - 1) / kFinishTiles;
  if (h->math_mode == LEV_MATH_ACCURATE)
    finish_kernel<1><<<blocks, kTile, 0, h->stream>>>(a, tc.ntiles);
  else
    finish_kernel<0><<<blocks, kTile, 0, h->stream>>>(a, tc.ntiles);
  LEV_TRY_CUDA(cudaGetLastError());
  return LEV_OK;
}

int lev_part_pack(LevEngine *h, const int32_t *idx_dev, int32_t n, float *out_dev) {
  int rc = part_check(h);
  if (rc != LEV_OK) return rc;
  if (n < 0) return fail(LEV_ERR_ARG, "n must be >= 0");
  if (n == 0) return LEV_OK;
  if (!idx_dev || !out_dev) return fail(LEV_ERR_ARG, "null device pointer");
  DeviceScope ds(h->device);
  const int blocks = std::min((n + 255) / 256, 148 * 8);
  part_pack_kernel<<<blocks, 256, 0, h->stream>>>(h->d_theta, h->h_nets[0].N, idx_dev, n,
                                                  out_dev);
  LEV_TRY_CUDA(cudaGetLastError());
  return LEV_OK;
}

int lev_part_unpack(LevEngine *h, const int32_t *idx_dev, int32_t n, const float *in_dev) {
  int rc = part_check(h);
  if (rc != LEV_OK) return rc;
  if (n < 0) return fail(LEV_ERR_ARG, "n must be >= 0");
  if (n == 0) return LEV_OK;
  if (!idx_dev || !in_dev) return fail(LEV_ERR_ARG, "null device pointer");
  DeviceScope ds(h->device);
  const NetDesc &nd = h->h_nets[0];
  const int blocks = std::min((n + 255) / 256, 148 * 8);
  part_unpack_kernel<<<blocks, 256, 0, h->stream>>>(h->d_st, h->d_ring + nd.ring_off, nd.N,
                                                    nd.Np, h->part_halo, idx_dev, n, in_dev);
  LEV_TRY_CUDA(cudaGetLastError());
  return LEV_OK;
}

int lev_part_fill_halo(LevEngine *h, const float *theta_halo) {
  int rc = part_check(h);
  if (rc != LEV_OK) return rc;
  if (h->part_halo == 0) return LEV_OK;
  if (!theta_halo) return fail(LEV_ERR_ARG, "theta_halo is null");
  DeviceScope ds(h->device);
  return fill_ext_columns(h, h->part_halo, theta_halo);
}

}  // extern "C"

// ===========================================================================
// Allocation-free step: lev_step_noalloc
//
// For callers that cannot call cudaMalloc: code whose device memory is owned
// by a memory planner or a framework allocator that must see every byte,
// fixed-budget or real-time loops in which cudaMalloc (which may synchronise
// the device and stall other streams) is not acceptable.  Such a caller keeps
// the whole network state in its own device buffers; this entry point only
// reads and writes them.  The step needs global scratch (one float2 partial
// sum per 256-node tile and a completion ticket); it lives in the file-scope
// device array below, of fixed size, which every GPU that loads this library
// holds until the process exits.
// ===========================================================================
namespace lev {

// Largest network the allocation-free step accepts (nodes).
constexpr int kNoAllocMaxNodes = 1 << 22;  // 4,194,304
constexpr int kNoAllocMaxTiles = kNoAllocMaxNodes / kTile;  // 16,384
// [0, 2*kNoAllocMaxTiles): float2 partial sums; [2*kNoAllocMaxTiles]: ticket
constexpr int kNoAllocWords = 2 * kNoAllocMaxTiles + 64;

static __device__ __align__(256) unsigned int g_noalloc_scratch[kNoAllocWords];

struct NoAllocArgs {
  const int *row_ptr;
  const int *col_idx;
  const uint8_t *delays;
  float *w;
  float *theta;
  float *theta_hat;
  const float *omega;
  float *omega_hat;
  float *ring;  // [max_delay + 2][N]
  float *gain;  // in: g for this step, out: g after the controller
  float *r_out;
  unsigned int *scratch;  // device address of g_noalloc_scratch
  NetDesc nd;             // parameters (offsets unused)
  int cur;                // ring slot of theta(t) = t mod (max_delay + 2)
  float dt;
};

// Same arithmetic as step_kernel (one network, caller-owned buffers,
// unpacked col_idx / delays, ring pitch N); scratch in g_noalloc_scratch.
template <int MATH>
__global__ void __launch_bounds__(kTile) noalloc_step_kernel(const NoAllocArgs a) {
  __shared__ int s_rp[kTile + 1];
  __shared__ float s_th[kTile];
  __shared__ float s_ae[kTile];
  __shared__ float2 s_ws[kChunk];
  __shared__ float s_rc[32];
  __shared__ float s_rs[32];
  __shared__ int s_last;

  const NetDesc &nd = a.nd;
  const int tid = threadIdx.x;
  const int N = nd.N;
  const int row0 = blockIdx.x * kTile;
  const int nrows = min(kTile, N - row0);
  const float dt = a.dt;
  const int bsi = nd.bsi;
  const int cur = a.cur;
  const float g = *a.gain;
  float2 *partials = reinterpret_cast<float2 *>(a.scratch);
  unsigned *ticket = a.scratch + 2 * kNoAllocMaxTiles;

  for (int k = tid; k <= nrows; k += kTile) s_rp[k] = a.row_ptr[row0 + k];
  float th = 0.0f, eps = 0.0f;
  if (tid < nrows) {
    const int gi = row0 + tid;
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

  const float eta = nd.eta, gamma = nd.gamma, lam = nd.lam;
  const float w_min = nd.w_min, w_max = nd.w_max;
  const int ebeg = s_rp[0], eend = s_rp[nrows];
  const int my_rs = (tid < nrows) ? s_rp[tid] : 0;
  const int my_re = (tid < nrows) ? s_rp[tid + 1] : 0;
  float local_sum = 0.0f;
  for (int c0 = ebeg; c0 < eend; c0 += kChunk) {
    const int c1 = min(c0 + kChunk, eend);
    int r = 0;
    for (int e = c0 + tid; e < c1; e += kTile) {
      int lo = r, hi = nrows;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s_rp[mid] <= e) lo = mid; else hi = mid;
      }
      r = lo;
      const int j = a.col_idx[e];
      const int d = a.delays[e];
      float w = a.w[e];
      float sin_diff = 0.0f;
      if ((unsigned)j < (unsigned)N && d <= nd.max_delay) {
        int slot = cur - d;
        slot += (slot < 0) ? bsi : 0;
        const float delayed_j = a.ring[(long long)slot * N + j];
        float diff = delayed_j - s_th[r];
        diff = wrap_pm_pi(diff);
        float cos_diff;
        lev_sincos<MATH>(diff, &sin_diff, &cos_diff);
        s_ws[e - c0] = make_float2(w, sin_diff);
        const float my_eps = s_ae[r];
        float dw = dt * (eta * cos_diff * (1.0f - gamma * my_eps) - lam * w);
        w += dw;
        if (!isfinite(w)) w = w_min;
        w = fmaxf(w_min, fminf(w_max, w));
        a.w[e] = w;
      } else {
        s_ws[e - c0] = make_float2(0.0f, 0.0f);  // out-of-range edge: skipped
      }
    }
    __syncthreads();
    if (tid < nrows) {
      const int b = max(my_rs, c0), e = min(my_re, c1);
      for (int x = b; x < e; ++x) {
        const float2 v = s_ws[x - c0];
        local_sum += v.x * v.y;
      }
    }
    __syncthreads();
  }

  int nxt = cur + 1;
  if (nxt == bsi) nxt = 0;
  float my_cos = 0.0f, my_sin = 0.0f;
  if (tid < nrows) {
    const int gi = row0 + tid;
    float inc = dt * (a.omega[gi] + g * local_sum - nd.alpha * eps);
    float x = th + inc;
    x = wrap_0_2pi(x);
    if (!isfinite(x)) x = 0.0f;
    a.theta[gi] = x;
    a.ring[(long long)nxt * N + gi] = x;
    lev_sincos<MATH>(x, &my_sin, &my_cos);
  }
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
      partials[blockIdx.x] = make_float2(my_cos, my_sin);
      __threadfence();
      const unsigned prev = atomicAdd(ticket, 1u);
      s_last = (prev == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (warp == 0) {
    float sum_cos = 0.0f, sum_sin = 0.0f;
    for (int k = lane; k < (int)gridDim.x; k += 32) {
      const float2 v = __ldcg(partials + k);
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
      *a.gain = nd.ctrl ? gain_controller(g, r, dt, nd) : g;
      *a.r_out = r;
      *ticket = 0u;
    }
  }
}

// Device address of g_noalloc_scratch per device, looked up on the first
// call made with that device current.  Atomic: two threads making their first
// call on one device at once both store the same address.
constexpr int kNoAllocMaxDevices = 64;
static std::atomic<unsigned int *> g_noalloc_addr[kNoAllocMaxDevices] = {};

}  // namespace lev

extern "C" int lev_step_noalloc(int32_t N, int32_t max_delay, int64_t t,
                                const int32_t *row_ptr, const int32_t *col_idx,
                                const uint8_t *delays, float *weights,
                                float *theta, float *theta_hat,
                                const float *omega, float *omega_hat,
                                float *ring, float *gain, float *r_out,
                                const LevParams *params, float dt,
                                int32_t math_mode, void *stream) {
  if (N < 1 || N > kNoAllocMaxNodes)
    return fail(LEV_ERR_ARG,
                "lev_step_noalloc: N must be in [1, " +
                    std::to_string(kNoAllocMaxNodes) +
                    "] (size of the built-in scratch), got " + std::to_string(N));
  if (max_delay < 0 || max_delay > 255)
    return fail(LEV_ERR_ARG, "lev_step_noalloc: max_delay must be in [0,255]");
  if (t < 0) return fail(LEV_ERR_ARG, "lev_step_noalloc: t must be >= 0");
  if (!row_ptr || !col_idx || !delays || !weights || !theta || !theta_hat ||
      !omega || !omega_hat || !ring || !gain || !r_out)
    return fail(LEV_ERR_ARG, "lev_step_noalloc: null device pointer");
  if (!std::isfinite(dt)) return fail(LEV_ERR_ARG, "lev_step_noalloc: dt is not finite");
  if (math_mode != LEV_MATH_REFERENCE && math_mode != LEV_MATH_ACCURATE)
    return fail(LEV_ERR_ARG, "lev_step_noalloc: math_mode must be 0 or 1");
  LevParams p;
  if (params) p = *params; else lev_default_params(&p);
  int rc = check_params(p);
  if (rc != LEV_OK) return rc;

  int dev = 0;
  LEV_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(LEV_ERR_ARG, "lev_step_noalloc: device ordinal too large");
  unsigned int *scratch = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (!scratch) {
    void *addr = nullptr;
    LEV_TRY_CUDA(cudaGetSymbolAddress(&addr, g_noalloc_scratch));
    scratch = static_cast<unsigned int *>(addr);
    g_noalloc_addr[dev].store(scratch, std::memory_order_release);
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

  NoAllocArgs a;
  std::memset(&a, 0, sizeof(a));
  a.row_ptr = row_ptr;
  a.col_idx = col_idx;
  a.delays = delays;
  a.w = weights;
  a.theta = theta;
  a.theta_hat = theta_hat;
  a.omega = omega;
  a.omega_hat = omega_hat;
  a.ring = ring;
  a.gain = gain;
  a.r_out = r_out;
  a.scratch = scratch;
  a.nd.N = N;
  a.nd.bsi = max_delay + 2;
  a.nd.max_delay = max_delay;
  params_to_desc(p, &a.nd);
  a.cur = (int)(t % (int64_t)(max_delay + 2));
  a.dt = dt;
  // the ticket must start at zero even if an earlier call was interrupted
  LEV_TRY_CUDA(cudaMemsetAsync(scratch + 2 * kNoAllocMaxTiles, 0,
                               sizeof(unsigned int), s));
  const int tiles = (N + kTile - 1) / kTile;
  if (math_mode == LEV_MATH_ACCURATE)
    noalloc_step_kernel<1><<<tiles, kTile, 0, s>>>(a);
  else
    noalloc_step_kernel<0><<<tiles, kTile, 0, s>>>(a);
  LEV_TRY_CUDA(cudaGetLastError());
  return LEV_OK;
}
