// lev_part.cuh -- one partition of a network split over several GPUs.
//
// The network's rows are cut into contiguous ranges of whole 256-row tiles,
// one range per GPU.  A partition engine steps its own rows with step_kernel
// (one network, NetDesc::dist = 1); the sources of its incoming edges that
// other partitions own ("halo" nodes) get ring columns N .. N + n_halo - 1
// after its own N columns, so every delayed gather stays a local ring read.
// Per step, outside these kernels (the host issues the collectives on the
// engine stream):
//   1. step_kernel: predictor, edges, integrate, own ring columns, and the
//      partition's tile partials of (sum cos, sum sin) written at their
//      GLOBAL tile positions of a partials array of the whole network;
//   2. all-gather of the tile partials (8 bytes per 256 nodes);
//   3. part_finish_kernel: r of the whole network from the gathered partials
//      in the reference's order (final_reduce_r_kernel,
//      leviathan_kernel.cu:242-263) and the gain controller (:431-435) --
//      every partition computes the same r and g bit for bit, and they are
//      those of the single-GPU engine because the tiles are the same;
//   4. part_pack_kernel: theta(t+1) of own nodes that peers need;
//   5. send/recv to the peers;
//   6. part_unpack_kernel: received theta(t+1) into the halo columns of ring
//      slot t+1, before the next step reads it (a delay-0 edge reads it).
// With no zero delay, two steps go per pair of launches instead: pair_kernel
// (steps t and t+1 but the last integrate; partials of r(t+1)), 2.-6. for
// step t+1, finish_kernel (the integrate of t+1; partials of r(t+2)), 2.-6.
// for step t+2 -- the next pair reads halo slots t+2 and older only.
// This replaces the reference's multi-GPU stub (leviathan_multigpu.cu:97-115,
// whose pack/unpack kernels are never launched, and :218-238, which averages
// per-GPU |r| on the host) and its partitioner, which drops every edge that
// crosses partitions (python/partition.py:121).
#pragma once

#include "lev_kernels.cuh"
#include "lev_pair.cuh"  // kReduceThreads, kPartChunk

namespace lev {

// r and g of the whole network from the partials of all its tiles, with the
// arithmetic of step_kernel's last CTA (lane l of one warp adds partials l,
// l+32, ... in turn, then the shuffle tree); advances the ring slot and step
// count.  One CTA of kReduceThreads: the partials are first staged in shared
// memory by the whole CTA, as reduce_kernel does, so the warp's sequential
// adds do not wait on L2 (a network of 10^6 nodes has 3,907 tiles).
__global__ void __launch_bounds__(kReduceThreads)
    part_finish_kernel(const NetDesc *nets, NetState *st, const float2 *__restrict__ partials,
                       int ntiles_global, int N_global, float dt, float *r_dev, float *r_host) {
  __shared__ float2 s_part[kPartChunk];
  const int tid = threadIdx.x;
  const NetDesc nd = nets[0];
  NetState *ns = st;
  const unsigned mask = 0xffffffffu;
  float sum_cos = 0.0f, sum_sin = 0.0f;
  for (int c0 = 0; c0 < ntiles_global; c0 += kPartChunk) {
    const int n = min(kPartChunk, ntiles_global - c0);
    for (int k = tid; k < n; k += kReduceThreads) s_part[k] = partials[c0 + k];
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
  if (tid >= 32) return;
#pragma unroll
  for (int off = 16; off > 0; off /= 2) {
    sum_cos += __shfl_down_sync(mask, sum_cos, off);
    sum_sin += __shfl_down_sync(mask, sum_sin, off);
  }
  if (tid == 0) {
    const float g = ns->g;
    float inv_N = 1.0f / (float)N_global;
    float r = sqrtf(sum_cos * sum_cos + sum_sin * sum_sin) * inv_N;
    const float gn = nd.ctrl ? gain_controller(g, r, dt, nd) : g;
    ns->g = gn;
    ns->r = r;
    int nxt = ns->cur + 1;
    if (nxt == nd.bsi) nxt = 0;
    ns->cur = nxt;
    int rb = ns->rbuf + 1;
    if (rb == nd.max_delay + 1) rb = 0;
    ns->rbuf = rb;
    ns->t = ns->t + 1;
    if (r_dev) *r_dev = r;
    if (r_host) *r_host = r;
  }
}

// out[k] = theta[idx[k]] (own nodes, after the step); an index outside
// [0, N) is skipped and its output left unwritten.
__global__ void part_pack_kernel(const float *__restrict__ theta, int N,
                                 const int *__restrict__ idx, int n,
                                 float *__restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += gridDim.x * blockDim.x) {
    const int j = idx[k];
    if ((unsigned)j < (unsigned)N) out[k] = theta[j];
  }
}

// Halo column N + idx[k] of the ring slot holding theta(t+1) := in[k]; an
// index outside [0, n_halo) is skipped.
__global__ void part_unpack_kernel(const NetState *st, float *__restrict__ ring,
                                   int N, int Np, int n_halo,
                                   const int *__restrict__ idx, int n,
                                   const float *__restrict__ in) {
  const int cur = st->cur;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += gridDim.x * blockDim.x) {
    const int j = idx[k];
    if ((unsigned)j < (unsigned)n_halo) ring[ring_pos(cur, (unsigned)(N + j), Np)] = in[k];
  }
}

}  // namespace lev
