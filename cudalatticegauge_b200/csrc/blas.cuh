// blas.cuh -- fused site-wise field kernels with single-pass FP64 reductions.
//
// The reference issues one kernel per BLAS op and reduces every dot product
// with log2(V) tree launches plus a blocking copy to the host
// (Core/CudaHelper.cu:183-190, 697-710).  Here a functor F describes what one
// site does (load / combine / store, accumulate NRED doubles); one launch
// covers every right-hand side (grid.y) and every site of the requested
// checkerboards, reduces with warp shuffles, and the last block to finish sums
// the block partials in a fixed order (deterministic) and runs F::finalize on
// the device, so solver scalars never leave the GPU.
#pragma once
#include <type_traits>

#include "field_io.cuh"
#include "internal.h"
#include "reduce.cuh"

namespace clg {

template <int NRED, class F>
__global__ void __launch_bounds__(256)
    site_reduce_kernel(F f, int64_t nsites, int first_parity, int64_t Vh, double* partials, unsigned* counter) {
  const int rhs = blockIdx.y;
  pdl_launch_dependents();
  pdl_wait();
  double acc[NRED > 0 ? NRED : 1];
#pragma unroll
  for (int k = 0; k < (NRED > 0 ? NRED : 1); ++k) acc[k] = 0.0;
  if (f.active(rhs)) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nsites; i += (int64_t)gridDim.x * blockDim.x) {
      const int pi = (int)(i / Vh);
      const int64_t h = i - (int64_t)pi * Vh;
      f(rhs, first_parity + pi, h, acc);
    }
  }
  if constexpr (NRED > 0)
    grid_reduce_finalize<NRED>(acc, f, rhs, blockIdx.x, gridDim.x, (int)gridDim.y, partials, counter);
}

// The same over a batch of lattices (clg_solve_lattices): right-hand side r
// holds rhs_vh[r] sites per checkerboard, the rest of the padded range is
// skipped (it stays zero).
template <int NRED, class F>
__global__ void __launch_bounds__(256)
    site_reduce_batch_kernel(F f, int64_t nsites, int first_parity, int64_t Vh, double* partials, unsigned* counter,
                             const int64_t* rhs_vh) {
  const int rhs = blockIdx.y;
  pdl_launch_dependents();
  pdl_wait();
  double acc[NRED > 0 ? NRED : 1];
#pragma unroll
  for (int k = 0; k < (NRED > 0 ? NRED : 1); ++k) acc[k] = 0.0;
  if (f.active(rhs)) {
    const int64_t vr = rhs_vh[rhs];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nsites; i += (int64_t)gridDim.x * blockDim.x) {
      const int pi = (int)(i / Vh);
      const int64_t h = i - (int64_t)pi * Vh;
      if (h < vr) f(rhs, first_parity + pi, h, acc);
    }
  }
  if constexpr (NRED > 0)
    grid_reduce_finalize<NRED>(acc, f, rhs, blockIdx.x, gridDim.x, (int)gridDim.y, partials, counter);
}

// Launch F over the checkerboards [first_parity, first_parity + nparity) of all nrhs.
template <int NRED, class F>
clg_status launch_sites(clg_context_s* ctx, const F& f, int first_parity, int nparity, int64_t Vh, int nrhs) {
  const int bs = 256;
  const int64_t nsites = (int64_t)nparity * Vh;
  int64_t nb = (nsites + bs - 1) / bs;
  // wide reductions use fewer, longer-running blocks: each block's shuffle tree
  // and its NRED partials are then amortised over more sites
  const int64_t per_sm = NRED > 4 ? 2 : 8;
  const int64_t cap = (int64_t)ctx->num_sms * per_sm / (nrhs > 0 ? nrhs : 1) + 1;
  if (NRED > 0 && nb > cap) nb = cap;
  if (nb > 65535 * 64) nb = 65535 * 64;
  if (NRED > 0) {
    clg_status st = ensure_reduction(ctx, nb * nrhs * (NRED > 0 ? NRED : 1));
    if (st) return st;
  }
  dim3 grid((unsigned)nb, (unsigned)nrhs);
  cudaError_t e;
  if (ctx->batch_vh && Vh == ctx->batch_vh_stride && nrhs == ctx->batch_nrhs)
    e = launch_pdl(ctx, site_reduce_batch_kernel<NRED, F>, grid, dim3(bs), 0, f, nsites, first_parity, Vh,
                   ctx->red_partials, ctx->red_counter, (const int64_t*)ctx->batch_vh);
  else
    e = launch_pdl(ctx, site_reduce_kernel<NRED, F>, grid, dim3(bs), 0, f, nsites, first_parity, Vh,
                   ctx->red_partials, ctx->red_counter);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("site kernel: ") + cudaGetErrorString(e));
  return CLG_SUCCESS;
}

// Call fn(P, NC) with compile-time precision / colour-spin count.
template <class Fn>
clg_status with_pn(int prec, int nc, Fn&& fn) {
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  using N12 = std::integral_constant<int, 12>;
  using N3 = std::integral_constant<int, 3>;
  if (nc == 12) {
    if (prec == 0) return fn(I0{}, N12{});
    if (prec == 1) return fn(I1{}, N12{});
    return fn(I2{}, N12{});
  }
  if (prec == 0) return fn(I0{}, N3{});
  if (prec == 1) return fn(I1{}, N3{});
  return fn(I2{}, N3{});
}

// Device-side view of a field for the functors.
struct DField {
  char* data;
  float* norm;
  int64_t blk, rstride, nrstride;
  int first_parity;
  int64_t Vh;
  __device__ __forceinline__ char* base(int rhs, int p) const {
    return data + (int64_t)rhs * rstride + (int64_t)(p - first_parity) * blk;
  }
  __device__ __forceinline__ float* nbase(int rhs, int p) const {
    return norm ? norm + (int64_t)rhs * nrstride + (int64_t)(p - first_parity) * Vh : nullptr;
  }
};
inline DField dfield(const FieldRef& r) {
  DField d;
  d.data = r.data;
  d.norm = r.norm;
  d.blk = r.blk;
  d.rstride = r.rstride;
  d.nrstride = r.nrstride;
  d.first_parity = r.first_parity;
  d.Vh = r.Vh;
  return d;
}

template <int P, int NC, typename AT>
__device__ __forceinline__ void ldv(const DField& f, int rhs, int p, int64_t h, cpx<AT> v[NC]) {
  load_site<P, NC, AT>(f.base(rhs, p), f.nbase(rhs, p), f.Vh, h, v);
}
template <int P, int NC, typename AT>
__device__ __forceinline__ void stv(const DField& f, int rhs, int p, int64_t h, const cpx<AT> v[NC]) {
  store_site<P, NC, AT>(f.base(rhs, p), f.nbase(rhs, p), f.Vh, h, v);
}

template <int NC, typename AT>
__device__ __forceinline__ void acc_dot(const cpx<AT> a[NC], const cpx<AT> b[NC], double* acc) {
  AT re = 0, im = 0;
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    re += a[k].x * b[k].x + a[k].y * b[k].y;
    im += a[k].x * b[k].y - a[k].y * b[k].x;
  }
  acc[0] += (double)re;
  acc[1] += (double)im;
}
template <int NC, typename AT>
__device__ __forceinline__ double site_norm2(const cpx<AT> a[NC]) {
  AT s = 0;
#pragma unroll
  for (int k = 0; k < NC; ++k) s += a[k].x * a[k].x + a[k].y * a[k].y;
  return (double)s;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

}  // namespace clg
