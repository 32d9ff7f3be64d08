// noalloc.cu -- clg_dot_noalloc: the field inner product <a, b> without any
// device allocation.
//
// clg_dot allocates a small device buffer for its result and may grow the
// context's reduction scratch with cudaMalloc.  Some callers cannot allow that:
// code that hands all device memory to its own pool up front and must not see
// the free memory change mid-run, code running under a hard device-memory
// budget, or a hot loop that cannot take the device-wide synchronisation that
// cudaMalloc / cudaFree imply.  This variant keeps its block partials, arrival
// counter and result in one file-scope __device__ array of fixed size, so a
// call allocates nothing: it launches the same reduction kernel as clg_dot and
// copies 2*nrhs doubles back to the caller's host buffer.
//
// Limits and rules of use:
//  - at most CLG_DOT_NOALLOC_MAX_RHS (64) right-hand sides; the block partials
//    must fit in the array (checked, CLG_ERR_BAD_ARG otherwise);
//  - every loaded GPU holds the 64 KiB array until the process exits;
//  - clg_context_create looks up the array's device address
//    (cudaGetSymbolAddress, with the context's device current) and loads this
//    file's kernels (cudaFuncGetAttributes).  Under CUDA's lazy module
//    loading that is the moment the array and the kernel code take device
//    memory, so it happens when the context is made, never inside
//    clg_dot_noalloc: a caller that hands the rest of the GPU to its own pool
//    after creating the context sees no allocation from this entry point;
//  - all calls share the array and it keeps the last call's contents; the
//    arrival counter is cleared at the start of every call; two calls that
//    overlap on the GPU (different streams or contexts, same device) race on
//    the array and give wrong results.
#include <mutex>

#include "blas.cuh"

namespace {

constexpr int kMaxRhs = 64;
constexpr int kScratchDoubles = 8192;    // 64 KiB
constexpr int kResultOff = 0;            // 2 * kMaxRhs doubles: the results
constexpr int kCounterOff = 2 * kMaxRhs; // one 8-byte slot: the arrival counter
constexpr int kPartialOff = 256;         // block partials from here on
constexpr int kMaxDevices = 128;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// Device address of the array on ctx's device (looked up once per device).
clg_status scratch_address(clg_context_s* ctx, double** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  const int dev = ctx->device;
  if (dev < 0 || dev >= kMaxDevices) return ctx->fail(CLG_ERR_BAD_ARG, "clg_dot_noalloc: device index out of range");
  if (!g_addr[dev]) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return ctx->fail(CLG_ERR_CUDA, "clg_dot_noalloc: cudaGetDevice failed");
    if (cur != dev && cudaSetDevice(dev) != cudaSuccess) return ctx->fail(CLG_ERR_CUDA, "clg_dot_noalloc: cudaSetDevice failed");
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (cur != dev) cudaSetDevice(cur);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return ctx->fail(clg::cuda_status(e), std::string("clg_dot_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return CLG_SUCCESS;
}

template <int P, int NC>
struct DotNoAllocF {
  clg::DField a, b;
  double* out;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int rhs, int p, int64_t h, double* acc) const {
    using AT = typename clg::AccT<P>::T;
    clg::cpx<AT> va[NC], vb[NC];
    clg::ldv<P, NC, AT>(a, rhs, p, h, va);
    clg::ldv<P, NC, AT>(b, rhs, p, h, vb);
    clg::acc_dot<NC, AT>(va, vb, acc);
  }
  __device__ void finalize(int rhs, const double* s) const {
    out[2 * rhs] = s[0];
    out[2 * rhs + 1] = s[1];
  }
};

}  // namespace

using namespace clg;

namespace clg {
// Called once by clg_context_create with the context's device current.
clg_status noalloc_prepare(clg_context_s* ctx) {
  double* base = nullptr;
  if (clg_status st = scratch_address(ctx, &base)) return st;
  cudaFuncAttributes fa;
  cudaError_t e = cudaSuccess;
  for (int prec = 0; prec < 3 && e == cudaSuccess; ++prec)
    for (int nc : {12, 3}) {
      with_pn(prec, nc, [&](auto P, auto NC) -> clg_status {
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, site_reduce_kernel<2, DotNoAllocF<P.value, NC.value>>);
        return CLG_SUCCESS;
      });
    }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return ctx->fail(cuda_status(e), std::string("clg_dot_noalloc set-up: ") + cudaGetErrorString(e));
  }
  return CLG_SUCCESS;
}
}  // namespace clg

extern "C" clg_status clg_dot_noalloc(clg_field a, clg_field b, double* re_im) {
  if (!a || !b || !re_im || a->lat != b->lat || a->kind != b->kind || a->subset != b->subset || a->nrhs != b->nrhs ||
      a->prec != b->prec)
    return CLG_ERR_BAD_ARG;
  // pending asynchronous imports are reordered from their own staging (no allocation)
  if (clg_status st = clg::settle(a)) return st;
  if (clg_status st = clg::settle(b)) return st;
  clg_context_s* ctx = a->lat->ctx;
  const int nrhs = a->nrhs;
  if (nrhs > kMaxRhs)
    return ctx->fail(CLG_ERR_BAD_ARG, "clg_dot_noalloc: at most 64 right-hand sides (the scratch array is fixed)");
  // same grid as the allocating path, so the two give the same sums
  const FieldRef fa = a->ref(), fb = b->ref();
  const int bs = 256;
  const int64_t nsites = (int64_t)fa.nparity * fa.Vh;
  int64_t nb = (nsites + bs - 1) / bs;
  const int64_t cap = (int64_t)ctx->num_sms * 8 / nrhs + 1;
  if (nb > cap) nb = cap;
  if (nb * nrhs * 2 > kScratchDoubles - kPartialOff)
    return ctx->fail(CLG_ERR_BAD_ARG, "clg_dot_noalloc: block partials exceed the fixed 64 KiB scratch array");
  double* base = nullptr;
  clg_status st = scratch_address(ctx, &base);
  if (st) return st;
  unsigned* counter = reinterpret_cast<unsigned*>(base + kCounterOff);
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(double), ctx->stream);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("clg_dot_noalloc: ") + cudaGetErrorString(e));
  st = with_pn(fa.prec, fa.nc, [&](auto P, auto NC) -> clg_status {
    DotNoAllocF<P.value, NC.value> f{dfield(fa), dfield(fb), base + kResultOff};
    dim3 grid((unsigned)nb, (unsigned)nrhs);
    site_reduce_kernel<2, DotNoAllocF<P.value, NC.value>>
        <<<grid, bs, 0, ctx->stream>>>(f, nsites, fa.first_parity, fa.Vh, base + kPartialOff, counter);
    ctx->kernels++;
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return ctx->fail(cuda_status(le), std::string("clg_dot_noalloc launch: ") + cudaGetErrorString(le));
    return CLG_SUCCESS;
  });
  if (st) return st;
  e = cudaMemcpyAsync(re_im, base + kResultOff, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("clg_dot_noalloc: ") + cudaGetErrorString(e));
  return CLG_SUCCESS;
}
