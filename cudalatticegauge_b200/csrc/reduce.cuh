// reduce.cuh -- single-launch grid reductions with a device-side finalize.
//
// Every block reduces its NRED per-thread doubles (warp shuffles, then one
// value per warp in shared memory) and writes them to its partial slot
// partials[(rhs * nslots + slot) * NRED + k].  The last block to arrive (an
// atomic ticket on `counter`) sums, for each right-hand side, its nslots
// partials in a fixed strided order followed by a fixed shuffle / shared-memory
// tree, so the result does not depend on which block finished last, and hands
// the totals to f.finalize(rhs, tot) on the device.  The ticket is reset for
// the next launch on the same stream.
#pragma once
#include <cuda_runtime.h>

namespace clg {

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
    if (threadIdx.x == 0) f.finalize(r, tot);
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
