// reduce.cuh -- single-launch grid reductions with a device-side finalize.
//
// Every block reduces its NRED per-thread doubles (warp shuffles, then one
// value per warp in shared memory) and writes them to its partial slot
// partials[(rhs * nslots + slot) * NRED + k].  The last block to arrive (an
// atomic ticket on `counter`) sums, for each right-hand side, its nslots
// partials in a fixed strided order followed by a fixed shuffle / shared-memory
// tree, so the result does not depend on which block finished last, and hands
// the totals to f.finalize(rhs, tot) on the device.  The ticket is reset for
// the next launch on the same stream.  A functor with a member
// finalize_warp(rhs, tot, lane) has it run by the 32 lanes of warp 0 instead
// (scalar updates over many independent entries, e.g. the shifts of a
// multi-shift solve, then take one round of global-memory latency, not one
// per entry).
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

namespace clg {

template <class F, class = void>
struct has_warp_finalize : std::false_type {};
template <class F>
struct has_warp_finalize<F, std::void_t<decltype(&F::finalize_warp)>> : std::true_type {};

// The last block's part: totals per right-hand side -> f.finalize.  Called by
// every thread of that block (at most 256 threads, 8 warps).
template <int NRED, class F>
__device__ __forceinline__ void grid_final_reduce(const F& f, unsigned nslots, int nrhs, const double* partials,
                                                  unsigned* counter, const int64_t* rhs_sites = nullptr) {
  __shared__ double sm[NRED][8];
  __shared__ double tot[NRED];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  // U independent partial loads in flight per thread and step (fixed order)
  constexpr int U = NRED >= 8 ? 1 : 8 / NRED;
  if constexpr (!has_warp_finalize<F>::value) {
    // several right-hand sides: warp w sums and finalises rhs w, w + nw, ...
    // (each finalize touches only its own rhs's state), so the finalize
    // latencies of up to nw right-hand sides overlap and no block barrier
    // separates them
    if (nrhs > 1) {
      for (int r = warp; r < nrhs; r += nw) {
        double s[NRED];
#pragma unroll
        for (int k = 0; k < NRED; ++k) s[k] = 0.0;
        const double* pr = partials + (int64_t)r * nslots * NRED;
        const unsigned ns = rhs_sites ? (unsigned)min((int64_t)nslots, (rhs_sites[r] + blockDim.x - 1) / blockDim.x)
                                      : nslots;
        for (unsigned b0 = lane; b0 < ns; b0 += U * 32) {
          double v[U][NRED];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const unsigned b = b0 + u * 32;
#pragma unroll
            for (int k = 0; k < NRED; ++k) v[u][k] = b < ns ? __ldcg(pr + (int64_t)b * NRED + k) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k = 0; k < NRED; ++k) s[k] += v[u][k];
        }
#pragma unroll
        for (int k = 0; k < NRED; ++k) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_down_sync(0xffffffffu, s[k], o);
        }
        if (lane == 0) f.finalize(r, s);
      }
      __syncthreads();
      if (threadIdx.x == 0) *counter = 0u;
      return;
    }
  }
  for (int r = 0; r < nrhs; ++r) {
    double s[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) s[k] = 0.0;
    const double* pr = partials + (int64_t)r * nslots * NRED;
    // a batch of lattices: only the slots that hold sites of this rhs's lattice wrote a partial
    const unsigned ns = rhs_sites ? (unsigned)min((int64_t)nslots, (rhs_sites[r] + blockDim.x - 1) / blockDim.x)
                                  : nslots;
    for (unsigned b0 = threadIdx.x; b0 < ns; b0 += U * blockDim.x) {
      double v[U][NRED];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const unsigned b = b0 + u * blockDim.x;
#pragma unroll
        for (int k = 0; k < NRED; ++k) v[u][k] = b < ns ? __ldcg(pr + (int64_t)b * NRED + k) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int k = 0; k < NRED; ++k) s[k] += v[u][k];
    }
#pragma unroll
    for (int k = 0; k < NRED; ++k) {
      double v = s[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) sm[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < NRED) {
      double v = 0.0;
      for (int w = 0; w < nw; ++w) v += sm[threadIdx.x][w];
      tot[threadIdx.x] = v;
    }
    __syncthreads();
    if constexpr (has_warp_finalize<F>::value) {
      if (threadIdx.x < 32) f.finalize_warp(r, tot, (int)threadIdx.x);
    } else {
      if (threadIdx.x == 0) f.finalize(r, tot);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// Block partials + ticket + (last block) final reduction.  `contribute` must be
// uniform over the block: a block that does not contribute (its right-hand
// side is finished) writes no partial and only takes its ticket, so the caller's
// finalize must ignore the totals of such right-hand sides.
template <int NRED, class F>
__device__ __forceinline__ void grid_reduce_finalize(double (&acc)[NRED], const F& f, int rhs, unsigned slot,
                                                     unsigned nslots, int nrhs, double* partials, unsigned* counter,
                                                     bool contribute = true, const int64_t* rhs_sites = nullptr) {
  __shared__ double sm[NRED][8];
  __shared__ bool last;
  if (contribute) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NRED; ++k) {
      double v = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) sm[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < NRED) {
      double v = 0.0;
      for (int w = 0; w < nw; ++w) v += sm[threadIdx.x][w];
      partials[((int64_t)rhs * nslots + slot) * NRED + threadIdx.x] = v;
      // only the partials must be visible to the last block before the ticket
      __threadfence();
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(counter, 1u);
    last = (t == nslots * (unsigned)nrhs - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  grid_final_reduce<NRED>(f, nslots, nrhs, partials, counter, rhs_sites);
}

// Two-level form for grids with many blocks per right-hand side (the hop
// epilogues: one block per 64-256 sites, thousands per right-hand side).  A
// block computes R right-hand sides (rhs[0..R), R = 1 or 2, the unit `unit`
// of nunits); acc holds NRED values per member, c[i] says whether member i
// contributes and has[i] whether it exists (the second member of the last
// pair of an odd count does not).  The slots of each unit are grouped by
// `group`; the block that completes a group (ticket counter[1 + unit *
// ngroups + g]) sums the group's partials in slot order and writes each
// member's group total to gpart[(rhs * ngroups + g) * NRED + k]; the block
// that completes the last group of all (ticket counter[0]) runs
// grid_final_reduce over the group totals.  No block reads more than `group`
// partials per right-hand side, every sum has a fixed order (deterministic),
// and the tickets are reset for the next launch.  In a batch of lattices
// (rhs_sites, R = 1) a group sums only the slots holding this rhs's sites.
template <int NRED, int R, class F>
__device__ __forceinline__ void grid_reduce_finalize2(double (&acc)[R * NRED], const F& f, const int (&rhs)[R],
                                                      const bool (&c)[R], const bool (&has)[R], unsigned unit,
                                                      unsigned nunits, unsigned slot, unsigned nslots, int nrhs,
                                                      unsigned group, double* partials, double* gpart,
                                                      unsigned* counter, const int64_t* rhs_sites = nullptr) {
  __shared__ double sm[R * NRED][8];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  bool any = false;
#pragma unroll
  for (int i = 0; i < R; ++i) any = any || c[i];
  if (any) {
#pragma unroll
    for (int k = 0; k < R * NRED; ++k) {
      double v = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) sm[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < R * NRED) {
      const int i = threadIdx.x / NRED, k = threadIdx.x % NRED;
      bool ci = c[0];
#pragma unroll
      for (int j = 1; j < R; ++j)
        if (i == j) ci = c[j];
      if (ci) {
        double v = 0.0;
        for (int w = 0; w < nw; ++w) v += sm[threadIdx.x][w];
        int ri = rhs[0];
#pragma unroll
        for (int j = 1; j < R; ++j)
          if (i == j) ri = rhs[j];
        partials[((int64_t)ri * nslots + slot) * NRED + k] = v;
        __threadfence();
      }
    }
    __syncthreads();
  }
  const unsigned ngroups = (nslots + group - 1) / group;
  const unsigned g = slot / group;
  const unsigned g0 = g * group;
  const unsigned gs = min(group, nslots - g0);
  unsigned* gc = counter + 1 + (int64_t)unit * ngroups + g;
  if (threadIdx.x == 0) last = atomicAdd(gc, 1u) == gs - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // this block completed group g of its unit: each member's total, in slot order
#pragma unroll
  for (int i = 0; i < R; ++i) {
    if (!has[i]) continue;  // uniform over the block
    unsigned ns = gs;
    if (rhs_sites) {
      const int64_t used = (rhs_sites[rhs[i]] + blockDim.x - 1) / blockDim.x;
      ns = used <= (int64_t)g0 ? 0u : (unsigned)min((int64_t)gs, used - (int64_t)g0);
    }
    double s[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) s[k] = 0.0;
    const double* pg = partials + ((int64_t)rhs[i] * nslots + g0) * NRED;
    for (unsigned b = threadIdx.x; b < ns; b += blockDim.x)
#pragma unroll
      for (int k = 0; k < NRED; ++k) s[k] += __ldcg(pg + (int64_t)b * NRED + k);
    __syncthreads();  // sm is reused
#pragma unroll
    for (int k = 0; k < NRED; ++k) {
      double v = s[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) sm[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < NRED) {
      double v = 0.0;
      for (int w = 0; w < nw; ++w) v += sm[threadIdx.x][w];
      gpart[((int64_t)rhs[i] * ngroups + g) * NRED + threadIdx.x] = v;
      __threadfence();
    }
  }
  if (threadIdx.x == 0) *gc = 0u;
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == ngroups * nunits - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  grid_final_reduce<NRED>(f, ngroups, nrhs, gpart, counter);
}

// The two-level reduction for blocks that each cover every right-hand side of
// one slot (the tile hops): each block has written partials[(rhs * nslots +
// blockIdx.x) * NRED + k] for the right-hand sides it computed (with a fence).
// The block that completes a group of `group` slots (ticket counter[1 + g])
// sums the group's partials per right-hand side in slot order (warp w takes
// rhs w, w + nwarps, ...) into gpart[(rhs * ngroups + g) * NRED + k]; the block
// that completes the last group runs grid_final_reduce over the group totals.
// Every block of the grid must call this (it has barriers).
template <int NRED, class F>
__device__ __forceinline__ void tile_reduce_finalize(const F& f, unsigned nslots, int nrhs, unsigned group,
                                                     const double* partials, double* gpart, unsigned* counter) {
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  const unsigned ngroups = (nslots + group - 1) / group;
  const unsigned g = blockIdx.x / group;
  const unsigned g0 = g * group;
  const unsigned gs = min(group, nslots - g0);
  unsigned* gc = counter + 1 + g;
  if (threadIdx.x == 0) last = atomicAdd(gc, 1u) == gs - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int r = warp; r < nrhs; r += nw) {
    double s[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) s[k] = 0.0;
    const double* pg = partials + ((int64_t)r * nslots + g0) * NRED;
    for (unsigned b = lane; b < gs; b += 32)
#pragma unroll
      for (int k = 0; k < NRED; ++k) s[k] += __ldcg(pg + (int64_t)b * NRED + k);
#pragma unroll
    for (int k = 0; k < NRED; ++k) {
      double v = s[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) gpart[((int64_t)r * ngroups + g) * NRED + k] = v;
    }
    if (lane == 0) __threadfence();
  }
  if (threadIdx.x == 0) *gc = 0u;
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == ngroups - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  grid_final_reduce<NRED>(f, ngroups, nrhs, gpart, counter);
}

// The same for a block that computes two right-hand sides (rhs0 with acc[0,
// NRED), rhs1 with acc[NRED, 2 NRED)); c0 / c1 say which of them contribute
// (each uniform over the block).  nblocks is the grid's total block count.
template <int NRED, class F>
__device__ __forceinline__ void grid_reduce_finalize_pair(double (&acc)[2 * NRED], const F& f, int rhs0, int rhs1,
                                                          bool c0, bool c1, unsigned slot, unsigned nslots,
                                                          unsigned nblocks, int nrhs, double* partials,
                                                          unsigned* counter) {
  __shared__ double sm[2 * NRED][8];
  __shared__ bool last;
  if (c0 || c1) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < 2 * NRED; ++k) {
      double v = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) sm[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 2 * NRED) {
      const bool second = threadIdx.x >= NRED;
      const int k = second ? threadIdx.x - NRED : threadIdx.x;
      if (second ? c1 : c0) {
        double v = 0.0;
        for (int w = 0; w < nw; ++w) v += sm[threadIdx.x][w];
        partials[((int64_t)(second ? rhs1 : rhs0) * nslots + slot) * NRED + k] = v;
        __threadfence();
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(counter, 1u);
    last = (t == nblocks - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  grid_final_reduce<NRED>(f, nslots, nrhs, partials, counter);
}

}  // namespace clg
