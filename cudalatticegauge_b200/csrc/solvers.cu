// solvers.cu -- CSLASolver::Solve (SparseLinearAlgebra/CSLASolver.h:42-50) on the B200.
//
// Structure of one solve of  A x = b  (A = D, D^+, D D^+, M_ee, ...):
//   outer loop in FP64 (defect correction / iterative refinement):
//       r = b - A x            (FP64 operator, FP64 reductions)
//       stop when |r| <= tol_true_rel |b| for every right-hand side
//       e ~= A^{-1} r          (inner Krylov solve in the inner precision)
//       x += e
//   the inner solve of D (Wilson or staggered) goes through the even-odd Schur
//   complement (Docs/SparseLinearAlgebra/evenodd.tex:11-16); its Krylov method is
//   GMRES(k) (CSolverGMRES.cpp:111-358), BiCGStab (CSolverBiCGstab.cpp:403-607)
//   or CG, with every scalar on the device and the iterations replayed from
//   CUDA graphs.  All right-hand sides of a field are solved together: one
//   launch per step covers every rhs, finished ones are skipped.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "dslash.cuh"
#include "krylov.cuh"

namespace clg {

__global__ void gm_solve_y(KState* st, int nrhs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  KState& k = st[r];
  if (k.done || k.j == 0) return;
  const int m = k.j;
  for (int i = m - 1; i >= 0; --i) {
    double2 acc = k.g[i];
    for (int l = i + 1; l < m; ++l) {
      const double2 p = cmul(k.H[i * GM_MAXK + l], k.y[l]);
      acc.x -= p.x;
      acc.y -= p.y;
    }
    k.y[i] = cdiv(acc, k.H[i * GM_MAXK + i]);
  }
  for (int i = 0; i < m; ++i) k.y[i] = make_double2(k.y[i].x * k.s[i], k.y[i].y * k.s[i]);
  if (k.resid_est * k.resid_est <= k.tol2 * k.rr0) k.status = ST_CONVERGED;
}

namespace {

__global__ void gm_finish(KState* st, int nrhs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  KState& k = st[r];
  if (k.done) return;
  if (k.status != ST_RUNNING) k.done = k.skip = 1;
  k.j = 0;
}

__global__ void kstate_reset(KState* st, const int* outer_done, int nrhs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  KState& k = st[r];
  const int d = outer_done[r];
  k.done = k.skip = d;
  k.conv_s = 0;
  k.status = d ? ST_CONVERGED : ST_RUNNING;
  k.iters = 0;
  k.j = 0;
  k.rr = k.rr0 = 0.0;
  k.best = 1e300;
  k.since = 0;
}

// Control of the device-side inner loop (a CUDA-graph WHILE node whose body is
// one chunk of iterations followed by loop_cond).
struct LoopCtl {
  int cap;         // operator applications allowed per rhs in this inner solve
  int max_chunks;  // hard bound on the chunks of one inner solve
  int chunks;      // chunks run so far
  int pad;
};

// Keeps looping while some right-hand side is unfinished, under its budget
// and has improved its residual within the last `patience` chunks -- the
// host-side rules of iterate(), evaluated on the device.
__global__ void loop_cond(KState* st, int nrhs, LoopCtl* ctl, int patience, cudaGraphConditionalHandle h) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  ctl->chunks += 1;
  unsigned go = 0;
  if (ctl->chunks < ctl->max_chunks) {
    for (int r = 0; r < nrhs; ++r) {
      KState& k = st[r];
      if (k.done || k.iters >= ctl->cap) continue;
      const double cur = k.rr > 0 ? k.rr : k.resid_est * k.resid_est;
      if (cur < 0.9 * k.best) {
        k.best = cur;
        k.since = 0;
      } else if (++k.since >= patience) {
        continue;
      }
      go = 1;
    }
  }
  cudaGraphSetConditional(h, go);
}

struct Summary {
  int done, status, iters, pad;
  double rr, rr0, resid_est, pad2;
};

// A few bytes between device memory and a solve's mapped pinned host buffers,
// moved by one warp instead of a copy engine: a copy engine busy with a large
// transfer queued on another stream (an overlapped field import or export of
// 100 MB) holds a small copy back until that transfer has ended.
__global__ void small_copy_kernel(uint32_t* dst, const uint32_t* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

__global__ void kstate_summary(const KState* st, Summary* out, int nrhs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  const KState& k = st[r];
  out[r].done = k.done;
  out[r].status = k.status;
  out[r].iters = k.iters;
  out[r].rr = k.rr;
  out[r].rr0 = k.rr0;
  out[r].resid_est = k.resid_est;
}

// x64 += e (converted), r64 = b64 - r64 are plain BLAS; this adds a lower-precision
// correction into the FP64 iterate for the rhs still running.
template <int PS, int NC>
struct AddConv {
  DField x, e;
  const int* skip;
  __device__ bool active(int r) const { return !skip[r]; }
  __device__ void operator()(int rhs, int p, int64_t h, double*) const {
    cpx<double> vx[NC], ve[NC];
    load_site<P64, NC, double>(x.base(rhs, p), nullptr, x.Vh, h, vx);
    load_site<PS, NC, double>(e.base(rhs, p), e.nbase(rhs, p), e.Vh, h, ve);
#pragma unroll
    for (int k = 0; k < NC; ++k) vx[k] = vx[k] + ve[k];
    store_site<P64, NC, double>(x.base(rhs, p), nullptr, x.Vh, h, vx);
  }
  __device__ void finalize(int, const double*) const {}
};

// r = b - r ; |r|^2
template <int NC>
struct Resid {
  DField b, r;
  double* out;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int rhs, int p, int64_t h, double* acc) const {
    cpx<double> vb[NC], vr[NC];
    load_site<P64, NC, double>(b.base(rhs, p), nullptr, b.Vh, h, vb);
    load_site<P64, NC, double>(r.base(rhs, p), nullptr, r.Vh, h, vr);
#pragma unroll
    for (int k = 0; k < NC; ++k) vr[k] = vb[k] - vr[k];
    store_site<P64, NC, double>(r.base(rhs, p), nullptr, r.Vh, h, vr);
    acc[0] += site_norm2<NC, double>(vr);
  }
  __device__ void finalize(int rhs, const double* s) const { out[rhs] = s[0]; }
};

// out += sigma_r * scale_r * in  (the shift of a shifted system; scale for lazily normalised inputs)
template <int P, int NC>
struct ShiftAdd {
  DField out, in;
  const double2* shift;
  const double* scale;
  int sstride;
  const int* skip;
  int kstride;
  __device__ bool active(int r) const { return !(skip && skip[(int64_t)r * kstride]); }
  __device__ void operator()(int rhs, int p, int64_t h, double*) const {
    using AT = typename AccT<P>::T;
    double2 sg = shift[rhs];
    if (scale) {
      const double sc = scale[(int64_t)rhs * sstride];
      sg = make_double2(sg.x * sc, sg.y * sc);
    }
    cpx<AT> vo[NC], vi[NC];
    ldv<P, NC, AT>(out, rhs, p, h, vo);
    ldv<P, NC, AT>(in, rhs, p, h, vi);
    const cpx<AT> c = mk<AT>((AT)sg.x, (AT)sg.y);
#pragma unroll
    for (int k = 0; k < NC; ++k) vo[k] = vo[k] + c * vi[k];
    stv<P, NC, AT>(out, rhs, p, h, vo);
  }
  __device__ void finalize(int, const double*) const {}
};

template <int P, int NC>
struct CopySkip {
  DField d, s;
  const int* skip;
  __device__ bool active(int r) const { return !skip[r]; }
  __device__ void operator()(int rhs, int p, int64_t h, double*) const {
    using AT = typename AccT<P>::T;
    cpx<AT> v[NC];
    ldv<P, NC, AT>(s, rhs, p, h, v);
    stv<P, NC, AT>(d, rhs, p, h, v);
  }
  __device__ void finalize(int, const double*) const {}
};

// ------------------------------------------------------------------ owned fields
struct Owned {
  FieldRef ref;
  void* data = nullptr;
  float* norm = nullptr;
  Owned() = default;
  Owned(const Owned&) = delete;
  Owned& operator=(const Owned&) = delete;
  ~Owned() {
    dfree(data);
    dfree(norm);
  }
  // allocates once; a cached workspace calls it again with the same shape
  clg_status alloc(clg_context_s* ctx, int prec, int nc, int nparity, int first_parity, int nrhs, int64_t Vh) {
    if (data) return CLG_SUCCESS;
    const int64_t blk = Vh * site_bytes_of(prec, nc);
    clg_status st = dalloc(ctx, &data, (size_t)blk * nparity * nrhs);
    if (st) return st;
    // zeroed once: in a batch of lattices the sites past a lattice's own
    // checkerboard are padding that every kernel leaves (or keeps) at zero
    cudaMemsetAsync(data, 0, (size_t)blk * nparity * nrhs, ctx->stream);
    if (prec == CLG_PREC_HALF) {
      st = dalloc(ctx, (void**)&norm, (size_t)Vh * nparity * nrhs * sizeof(float));
      if (st) return st;
      cudaMemsetAsync(norm, 0, (size_t)Vh * nparity * nrhs * sizeof(float), ctx->stream);
    }
    ref.data = (char*)data;
    ref.norm = norm;
    ref.blk = blk;
    ref.rstride = blk * nparity;
    ref.nrstride = norm ? Vh * nparity : 0;
    ref.nparity = nparity;
    ref.first_parity = first_parity;
    ref.prec = prec;
    ref.nc = nc;
    ref.nrhs = nrhs;
    ref.Vh = Vh;
    return CLG_SUCCESS;
  }
};

// internal Krylov operator M_ee^+ M_ee (CGNR for D^+ solves); not part of the C ABI
constexpr int OP_MEEDAG_MEE = 100;

bool hermitian_op(int op) {
  return op == CLG_OP_DDDAG || op == CLG_OP_DDDAG_EE || op == CLG_OP_MEE_MEEDAG || op == OP_MEEDAG_MEE;
}
// operator applications one Krylov-operator application stands for
int op_weight(int op) { return (op == CLG_OP_MEE_MEEDAG || op == OP_MEEDAG_MEE || op == CLG_OP_DDDAG) ? 2 : 1; }

}  // namespace

}  // namespace clg

using namespace clg;

namespace {

// Everything one solve needs, allocated per call.
struct Work : public SolveCacheBase {
  std::string key;  // shape of the solve this workspace was built for
  clg_context_s* ctx;
  clg_gauge_s* U;
  int kind, op, P, nc, nrhs;
  double param;
  int64_t Vh;
  const clg_solver_params* prm;
  // FP64 outer vectors and inner-precision Schur vectors (allocated on first use)
  Owned x64, b64, r64, t64, tf, te, rP, eP, yP, bS, yS;
  // device state
  KState* st = nullptr;
  Summary* sum_d = nullptr;
  Summary* sum_h = nullptr;
  int* outer_done_d = nullptr;
  double* tol_d = nullptr;
  double* red_d = nullptr;   // per-rhs reduction outputs
  double* host_buf = nullptr;
  // device addresses of sum_h and host_buf (mapped pinned memory), or nullptr
  // where the device cannot address them (then the copy engines move them)
  Summary* sum_hd = nullptr;
  double* host_buf_d = nullptr;
  double2* shift_dev = nullptr;  // per-rhs shift sigma_r: the system is (op + sigma_r) x_r = b_r
  // Krylov operator temporaries (precision P)
  Owned kt_odd, kt_even, kt_full;
  // Krylov vectors per graph slot: they persist for the whole solve so a
  // captured graph stays valid across defect-correction cycles
  std::map<int, std::vector<std::unique_ptr<Owned>>> kv;
  // graphs
  std::vector<cudaGraphExec_t> graphs;
  std::vector<int64_t> graph_kernels;  // kernel nodes per graph (for the launch count)
  // device-side inner loops (WHILE node around one chunk + loop_cond) per slot
  std::vector<cudaGraphExec_t> loops;
  std::vector<int64_t> loop_kernels;  // kernel nodes per loop body
  std::vector<char> loop_failed;      // building the loop failed once: host-driven chunks
  LoopCtl* ctl_d = nullptr;
  LoopCtl* ctl_h = nullptr;           // pinned
  int total_iters = 0;
  int inner_cap = 1 << 30;  // operator applications allowed in the current inner solve
  clg_status kvec(int slot, int idx, int np, int fp, FieldRef& out) {
    auto& v = kv[slot];
    while ((int)v.size() <= idx) v.emplace_back(nullptr);
    if (!v[idx]) {
      v[idx].reset(new Owned());
      clg_status s = v[idx]->alloc(ctx, P, nc, np, fp, nrhs, Vh);
      if (s) {
        v[idx].reset();
        return s;
      }
    }
    out = v[idx]->ref;
    return CLG_SUCCESS;
  }
  ~Work() {
    for (auto g : graphs)
      if (g) cudaGraphExecDestroy(g);
    for (auto g : loops)
      if (g) cudaGraphExecDestroy(g);
    dfree(ctl_d);
    if (ctl_h) cudaFreeHost(ctl_h);
    dfree(st);
    dfree(sum_d);
    dfree(outer_done_d);
    dfree(tol_d);
    dfree(red_d);
    dfree(shift_dev);
    if (sum_h) cudaFreeHost(sum_h);
    if (host_buf) cudaFreeHost(host_buf);
  }
};

// dst <- src, `bytes` (a multiple of 4) between device memory and a mapped
// pinned host buffer, in stream order on the context stream
static cudaError_t small_copy(clg_context_s* ctx, void* dst, const void* src, size_t bytes) {
  small_copy_kernel<<<1, 32, 0, ctx->stream>>>(static_cast<uint32_t*>(dst), static_cast<const uint32_t*>(src),
                                               (int)(bytes / 4));
  ctx->kernels++;
  return cudaGetLastError();
}

// host_buf[0, bytes) <- device memory, in stream order
static cudaError_t to_host(Work& w, const void* src, size_t bytes) {
  if (w.host_buf_d) return small_copy(w.ctx, w.host_buf_d, src, bytes);
  return cudaMemcpyAsync(w.host_buf, src, bytes, cudaMemcpyDeviceToHost, w.ctx->stream);
}

clg_status read_summary(Work& w) {
  // the summary kernel writes the host buffer directly where it is mapped
  kstate_summary<<<(w.nrhs + 63) / 64, 64, 0, w.ctx->stream>>>(w.st, w.sum_hd ? w.sum_hd : w.sum_d, w.nrhs);
  w.ctx->kernels++;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && !w.sum_hd)
    e = cudaMemcpyAsync(w.sum_h, w.sum_d, sizeof(Summary) * w.nrhs, cudaMemcpyDeviceToHost, w.ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(w.ctx->stream);
  if (e != cudaSuccess) return w.ctx->fail(cuda_status(e), std::string("solver sync: ") + cudaGetErrorString(e));
  return CLG_SUCCESS;
}

// Krylov operator K on fields of precision P: out = K in (optionally * scale_dev[rhs])
clg_status kapply_base(Work& w, int op, const FieldRef& out, const FieldRef& in, const double* scale, int sstride,
                       const int* skip, int kstride) {
  const double2 one = make_double2(1, 0);
  if (op == CLG_OP_MEE_MEEDAG || op == OP_MEEDAG_MEE) {
    const bool mdag_first = op == CLG_OP_MEE_MEEDAG;  // M (M^+ in)  or  M^+ (M in)
    clg_status s = apply_op(w.ctx, mdag_first ? CLG_OP_MEE_DAG : CLG_OP_MEE, w.U, w.kind, w.param, w.kt_even.ref, in,
                            &w.kt_odd.ref, one, w.nrhs, nullptr, 0, skip, kstride);
    if (s) return s;
    return apply_op(w.ctx, mdag_first ? CLG_OP_MEE : CLG_OP_MEE_DAG, w.U, w.kind, w.param, out, w.kt_even.ref,
                    &w.kt_odd.ref, one, w.nrhs, scale, sstride, skip, kstride);
  }
  const FieldRef* tmp = (op == CLG_OP_DDDAG || op == CLG_OP_DD) ? &w.kt_full.ref : &w.kt_odd.ref;
  return apply_op(w.ctx, op, w.U, w.kind, w.param, out, in, tmp, one, w.nrhs, scale, sstride, skip, kstride);
}

clg_status kapply(Work& w, int op, const FieldRef& out, const FieldRef& in, const double* scale, int sstride,
                  const int* skip, int kstride) {
  clg_status s = kapply_base(w, op, out, in, scale, sstride, skip, kstride);
  if (s || !w.shift_dev) return s;
  return with_pn(out.prec, out.nc, [&](auto PP, auto NN) {
    ShiftAdd<PP.value, NN.value> f{dfield(out), dfield(in), w.shift_dev, scale, sstride, skip, kstride};
    return launch_sites<0>(w.ctx, f, out.first_parity, out.nparity, out.Vh, w.nrhs);
  });
}

// Run `body` (one iteration or one cycle) repeatedly until every rhs is done
// or the budget runs out.  Chunks after the first are replayed from a CUDA graph.
// The rest of an inner solve as one graph launch: a WHILE node whose body is
// `chunk` iterations and loop_cond.  Built on first use per graph slot (the
// body is captured into the node's body graph); afterwards one launch and one
// host read per inner solve.  CLG_ERR_UNSUPPORTED: the loop could not be built
// (the caller falls back to host-driven chunks).
template <class Body>
clg_status run_device_loop(Work& w, int slot, int chunk, int max_chunks, int patience, Body& body) {
  clg_context_s* ctx = w.ctx;
  while ((int)w.loops.size() <= slot) {
    w.loops.push_back(nullptr);
    w.loop_kernels.push_back(0);
    w.loop_failed.push_back(0);
  }
  if (w.loop_failed[slot]) return CLG_ERR_UNSUPPORTED;
  if (!w.ctl_d) {
    if (clg_status s = dalloc(ctx, (void**)&w.ctl_d, sizeof(LoopCtl))) return s;
    if (cudaMallocHost((void**)&w.ctl_h, sizeof(LoopCtl)) != cudaSuccess) {
      w.ctl_h = nullptr;
      return ctx->fail(CLG_ERR_OOM, "loop control (pinned)");
    }
  }
  if (!w.loops[slot]) {
    cudaGraph_t g = nullptr;
    cudaGraphConditionalHandle h;
    cudaGraphNodeParams np = {};
    cudaGraphNode_t node;
    bool ok = cudaGraphCreate(&g, 0) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = h;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      ok = cudaGraphAddNode(&node, g, nullptr, 0, &np) == cudaSuccess;
    }
    clg_status s = CLG_SUCCESS;
    if (ok) ok = cudaStreamBeginCaptureToGraph(ctx->stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      // captured launches run per loop pass: count them from the passes run
      const int64_t k0 = ctx->kernels;
      const bool pdl = ctx->pdl;
      ctx->pdl = false;  // plain stream order inside the loop body
      for (int i = 0; i < chunk && !s; ++i) s = body();
      if (!s) {
        loop_cond<<<1, 32, 0, ctx->stream>>>(w.st, w.nrhs, w.ctl_d, patience, h);
        ctx->kernels++;
      }
      ctx->pdl = pdl;
      w.loop_kernels[slot] = ctx->kernels - k0;
      ctx->kernels = k0;
      cudaGraph_t out = nullptr;
      ok = cudaStreamEndCapture(ctx->stream, &out) == cudaSuccess && !s;
      cudaGraphExec_t ex = nullptr;
      if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
      if (ok) w.loops[slot] = ex;
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    if (s) return s;
    if (!ok) {
      w.loop_failed[slot] = 1;
      return CLG_ERR_UNSUPPORTED;
    }
  }
  w.ctl_h->cap = w.inner_cap;
  w.ctl_h->max_chunks = max_chunks;
  w.ctl_h->chunks = 0;
  cudaError_t e = cudaMemcpyAsync(w.ctl_d, w.ctl_h, sizeof(LoopCtl), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaGraphLaunch(w.loops[slot], ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w.ctl_h, w.ctl_d, sizeof(LoopCtl), cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("device loop: ") + cudaGetErrorString(e));
  if (clg_status s = read_summary(w)) return s;  // synchronises the stream
  ctx->kernels += (int64_t)w.ctl_h->chunks * w.loop_kernels[slot];
  return CLG_SUCCESS;
}

template <class Body>
clg_status iterate(Work& w, int graph_slot, int chunk, int max_chunks, Body&& body, bool device_loop = false) {
  const bool graphs = w.prm->use_graphs && w.ctx->stream != nullptr;
  while ((int)w.graphs.size() <= graph_slot) w.graphs.push_back(nullptr);
  while ((int)w.graph_kernels.size() <= graph_slot) w.graph_kernels.push_back(0);
  // stagnation guard: an inner solve ends when no running rhs has improved its
  // residual (recursive, or the GMRES estimate) for `patience` chunks
  std::vector<double> best(w.nrhs, 1e300);
  std::vector<int> since(w.nrhs, 0);
  const int patience = std::max(8, 400 / std::max(chunk, 1));
  for (int c = 0; c < max_chunks; ++c) {
    clg_status s = CLG_SUCCESS;
    // after the first (eager) chunk, the rest of the inner solve on the device
    if (device_loop && graphs && w.ctx->device_loops && c > 0) {
      s = run_device_loop(w, graph_slot, chunk, max_chunks - c, patience, body);
      if (s != CLG_ERR_UNSUPPORTED) return s;
      s = CLG_SUCCESS;
    }
    if (graphs && c > 0 && !w.graphs[graph_slot]) {
      cudaGraph_t g = nullptr;
      if (cudaStreamBeginCapture(w.ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        // captured launches do not run here: count them once per replay instead
        const int64_t k0 = w.ctx->kernels;
        for (int i = 0; i < chunk && !s; ++i) s = body();
        w.graph_kernels[graph_slot] = w.ctx->kernels - k0;
        w.ctx->kernels = k0;
        cudaError_t e = cudaStreamEndCapture(w.ctx->stream, &g);
        if (!s && e == cudaSuccess && g) {
          cudaGraphExec_t ex = nullptr;
          if (cudaGraphInstantiate(&ex, g, 0) == cudaSuccess) w.graphs[graph_slot] = ex;
        }
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (s) return s;
      } else {
        cudaGetLastError();
      }
    }
    if (graphs && w.graphs[graph_slot]) {
      cudaError_t e = cudaGraphLaunch(w.graphs[graph_slot], w.ctx->stream);
      if (e != cudaSuccess) return w.ctx->fail(cuda_status(e), std::string("graph launch: ") + cudaGetErrorString(e));
      w.ctx->kernels += w.graph_kernels[graph_slot];
    } else {
      for (int i = 0; i < chunk && !s; ++i) s = body();
      if (s) return s;
    }
    s = read_summary(w);
    if (s) return s;
    bool all = true, stalled = true;
    int most = 0;
    for (int r = 0; r < w.nrhs; ++r) {
      const Summary& q = w.sum_h[r];
      all = all && q.done;
      most = std::max(most, q.iters);
      if (q.done) continue;
      const double cur = q.rr > 0 ? q.rr : q.resid_est * q.resid_est;
      if (cur < 0.9 * best[r]) {
        best[r] = cur;
        since[r] = 0;
      } else {
        since[r]++;
      }
      stalled = stalled && since[r] >= patience;
    }
    if (all || stalled || most >= w.inner_cap) break;
  }
  return CLG_SUCCESS;
}

// GMRES multi-dot of column j with a reduction exactly 2(j+1) wide
template <int PV, int NV, int J>
clg_status launch_gm_dots(clg_context_s* ctx, const VList& vl, const FieldRef& wv, KState* st, int j, int fp, int np,
                          int64_t Vh, int nrhs) {
  if constexpr (J < GM_MAXK) {
    if (j == J) return launch_sites<2 * (J + 1)>(ctx, GmDotsJ<PV, NV, J>{vl, dfield(wv), st}, fp, np, Vh, nrhs);
    return launch_gm_dots<PV, NV, J + 1>(ctx, vl, wv, st, j, fp, np, Vh, nrhs);
  } else {
    return ctx->fail(CLG_ERR_BAD_ARG, "GMRES column index out of range");
  }
}

// ------------------------------------------------------------------ Krylov methods
// Solve K x = b (precision P, the subset of b) for every rhs not marked in outer_done.
// ------------------------------------------------------------------ fused CG on the Wilson normal equations
// CG on A = M_ee M_ee^+ (CLG_OP_MEE_MEEDAG) or M_ee^+ M_ee (OP_MEEDAG_MEE)
// without a shift: one iteration is the four Schur hops of A p with the CG
// vector work in the epilogues of the second and fourth (CgHopAlpha,
// CgHopUpdate), then p = r + beta p.
bool fused_cg(const Work& w, int op) {
  return w.ctx->fused_cg && w.kind == CLG_FERMION_WILSON && !w.shift_dev &&
         (op == CLG_OP_MEE_MEEDAG || op == OP_MEEDAG_MEE);
}

// the paired FP16 form: config = block | variant << 16 as in launch_wilson_pair
template <bool DAG, class E>
cudaError_t launch_hop_pair_epi(clg_context_s* ctx, const HopArgs& a, const E& e, int cfg) {
  const int bs = cfg & 0xffff;
  const unsigned npairs = (unsigned)(a.nrhs + 1) / 2u;
  const int64_t nslots = (a.g.Vh + bs - 1) / bs;
  dim3 grid((unsigned)(nslots * npairs));
  const unsigned group = red_group(nslots, npairs);
  double* gpart = ctx->red_partials + nslots * a.nrhs * E::NRED;
  if ((cfg >> 16) == 1)
    return launch_pdl(ctx, wilson_hop_pair_epi_kernel<DAG, 256, 2, E>, grid, dim3(bs), 0, a, e, ctx->red_partials,
                      gpart, ctx->red_counter, group);
  return launch_pdl(ctx, wilson_hop_pair_epi_kernel<DAG, 256, 1, E>, grid, dim3(bs), 0, a, e, ctx->red_partials,
                    gpart, ctx->red_counter, group);
}

// the tile form (wilson_hop_tile16_epi_kernel): config as in launch_wilson_tile
// the tensor-core form (wilson_hop_mma16_epi_kernel): config as in launch_wilson_mma
template <bool DAG, class E>
cudaError_t launch_hop_mma_epi(clg_context_s* ctx, const HopArgs& a0, const E& e, int cfg) {
  HopArgs a = a0;
  const int v = (cfg >> 16) - 24;
  a.tile_rows = (v & 2) ? tile_rows(a.g, a.nrhs, MMA_TS) : 0;
  const int64_t nslots = (a.g.Vh + MMA_TS - 1) / MMA_TS;
  const unsigned group = red_group(nslots, 1);
  double* gpart = ctx->red_partials + nslots * a.nrhs * E::NRED;
  const size_t smem = sizeof(Mma16Smem);
  auto go = [&](void (*kernel)(HopArgs, E, double*, double*, unsigned*, unsigned)) {
    if (const cudaError_t err = opt_in_smem((const void*)kernel, smem)) return err;
    return launch_pdl(ctx, kernel, dim3((unsigned)nslots), dim3(256), smem, a, e, ctx->red_partials, gpart,
                      ctx->red_counter, group);
  };
  if (v & 1) return go(wilson_hop_mma16_epi_kernel<DAG, 2, E>);
  return go(wilson_hop_mma16_epi_kernel<DAG, 1, E>);
}

template <bool DAG, class E>
cudaError_t launch_hop_tile_epi(clg_context_s* ctx, const HopArgs& a0, const E& e, int cfg) {
  if ((cfg >> 16) >= 24) return launch_hop_mma_epi<DAG>(ctx, a0, e, cfg);
  const int bs = cfg & 0xffff;
  HopArgs a = a0;
  a.tile_rows = ((cfg >> 16) & 2) ? tile_rows(a.g, a.nrhs) : 0;
  const int64_t nslots = (a.g.Vh + TILE16 - 1) / TILE16;
  const unsigned group = red_group(nslots, 1);
  double* gpart = ctx->red_partials + nslots * a.nrhs * E::NRED;
  int v = cfg >> 16;
  // an epilogue that loads vectors of its own (the CG update: x, r, p) spills
  // under the 72- and 64-register caps: it keeps the 80-register form
  if (v >= 20 && !E::STORE) v = 17 + (v & 2);
  if (v >= 20) {  // at most 128 threads: 72 or (v odd) 64 registers
    if (bs > 128) return cudaErrorInvalidConfiguration;
    if (v & 1)
      return launch_pdl(ctx, wilson_hop_tile16_epi_kernel<DAG, 8, E, false, 128>, dim3((unsigned)nslots), dim3(bs),
                        0, a, e, ctx->red_partials, gpart, ctx->red_counter, group);
    return launch_pdl(ctx, wilson_hop_tile16_epi_kernel<DAG, 7, E, false, 128>, dim3((unsigned)nslots), dim3(bs), 0,
                      a, e, ctx->red_partials, gpart, ctx->red_counter, group);
  }
  if (v & 1)
    return launch_pdl(ctx, wilson_hop_tile16_epi_kernel<DAG, 3, E>, dim3((unsigned)nslots), dim3(bs), 0, a, e,
                      ctx->red_partials, gpart, ctx->red_counter, group);
  return launch_pdl(ctx, wilson_hop_tile16_epi_kernel<DAG, 2, E>, dim3((unsigned)nslots), dim3(bs), 0, a, e,
                    ctx->red_partials, gpart, ctx->red_counter, group);
}

// the FP64 / FP32 tile form (wilson_hop_tileN_epi_kernel): config as in launch_wilson_tileN
template <int P, int RECON, bool DAG, class E>
cudaError_t launch_hop_tileN_epi(clg_context_s* ctx, const HopArgs& a0, const E& e, int cfg) {
  constexpr int CAP = P == P64 ? 2 : 3;
  const int bs = cfg & 0xffff;
  HopArgs a = a0;
  a.tile_rows = ((cfg >> 16) & 2) ? tile_rows(a.g, a.nrhs, TILE16, spinor_bytes<P>()) : 0;
  const int64_t nslots = (a.g.Vh + TILE16 - 1) / TILE16;
  const unsigned group = red_group(nslots, 1);
  double* gpart = ctx->red_partials + nslots * a.nrhs * E::NRED;
  if ((cfg >> 16) & 1)
    return launch_pdl(ctx, wilson_hop_tileN_epi_kernel<P, RECON, DAG, CAP, E>, dim3((unsigned)nslots), dim3(bs), 0,
                      a, e, ctx->red_partials, gpart, ctx->red_counter, group);
  return launch_pdl(ctx, wilson_hop_tileN_epi_kernel<P, RECON, DAG, 1, E>, dim3((unsigned)nslots), dim3(bs), 0, a,
                    e, ctx->red_partials, gpart, ctx->red_counter, group);
}

// a batch of lattices in the tile form (wilson_hop_tile16_epi_kernel /
// wilson_hop_tileN_epi_kernel with BATCH): one block per tile of one lattice
template <int P, int RECON, bool DAG, class E>
cudaError_t launch_hop_batch_tile_epi(clg_context_s* ctx, const HopArgs& a, const E& e) {
  constexpr int CAP = P == P64 ? 2 : 3;
  const int64_t nslots = a.btiles;
  const unsigned group = red_group(nslots, 1);
  double* gpart = ctx->red_partials + nslots * a.nrhs * E::NRED;
  const dim3 grid((unsigned)nslots), block(128);
  if constexpr (P == P16)
    return launch_pdl(ctx, wilson_hop_tile16_epi_kernel<DAG, CAP, E, true>, grid, block, 0, a, e, ctx->red_partials,
                      gpart, ctx->red_counter, group);
  else
    return launch_pdl(ctx, wilson_hop_tileN_epi_kernel<P, RECON, DAG, CAP, E, true>, grid, block, 0, a, e,
                      ctx->red_partials, gpart, ctx->red_counter, group);
}

template <int P, int RECON, bool DAG, class E>
cudaError_t launch_hop_epi(clg_context_s* ctx, const HopArgs& a, const E& e, int bs) {
  const int64_t nslots = (a.g.Vh + bs - 1) / bs;
  dim3 grid((unsigned)(nslots * a.nrhs));
  const unsigned group = red_group(nslots, a.nrhs);
  double* gpart = ctx->red_partials + nslots * a.nrhs * E::NRED;
  constexpr int MINB = P == P64 ? 1 : 3;
  if (a.seg)  // a batch of lattices
    return launch_pdl(ctx, wilson_hop_epi_kernel<P, RECON, DAG, 256, MINB, E, true>, grid, dim3(bs), 0, a, e,
                      ctx->red_partials, gpart, ctx->red_counter, group);
  return launch_pdl(ctx, wilson_hop_epi_kernel<P, RECON, DAG, 256, MINB, E>, grid, dim3(bs), 0, a, e,
                    ctx->red_partials, gpart, ctx->red_counter, group);
}

// out_e = in_e - kappa^2 H_eo^(dag) t_o with epilogue e (E::STORE decides
// whether out_e is written)
template <int P, class E>
clg_status schur_hop_epi(Work& w, bool dag, const FieldRef& t_odd, const FieldRef& in_even, const FieldRef& out_even,
                         const E& e, const int* skip, int ks) {
  clg_context_s* ctx = w.ctx;
  HopSpec s;
  s.kind = CLG_FERMION_WILSON;
  s.prec = P;
  s.dagger = dag;
  s.out_parity = 0;
  s.in = t_odd;
  s.out = out_even;
  s.x = &in_even;
  s.a = make_double2(-w.param * w.param, 0.0);
  s.xa = make_double2(1.0, 0.0);
  s.scale_dev = nullptr;
  s.scale_stride = 0;
  s.skip_dev = skip;
  s.skip_stride = ks;
  s.nrhs = w.nrhs;
  HopArgs a;
  if (clg_status st = make_hop_args(ctx, w.U, s, a)) return st;
  if (a.seg && a.btile) {  // a batch of lattices: the tile form
    if (clg_status st = ensure_reduction(ctx, red2_doubles(a.btiles, w.nrhs, 1, E::NRED))) return st;
    cudaError_t berr;
    if constexpr (P == P64)
      berr = dag ? launch_hop_batch_tile_epi<P, 18, true>(ctx, a, e) : launch_hop_batch_tile_epi<P, 18, false>(ctx, a, e);
    else
      berr = dag ? launch_hop_batch_tile_epi<P, 12, true>(ctx, a, e) : launch_hop_batch_tile_epi<P, 12, false>(ctx, a, e);
    if (berr != cudaSuccess) return ctx->fail(cuda_status(berr), std::string("fused hop: ") + cudaGetErrorString(berr));
    return CLG_SUCCESS;
  }
  // the block size tuned for the plain hop of the same kind (the hops on the
  // odd checkerboard of each iteration run first and are tuned)
  HopSpec plain = s;
  plain.x = nullptr;
  const int bs = tuned_hop_block(ctx, w.U, plain, P == P64 ? 64 : 128);
  if constexpr (P == P16) {
    const int tcfg = w.nrhs >= 2 && !a.seg ? tuned_hop_tile_config(ctx, w.U, plain, -1) : -1;
    if (tcfg >= 0) {
      const int64_t nslots = (w.Vh + ((tcfg >> 16) >= 24 ? MMA_TS : TILE16) - 1) / ((tcfg >> 16) >= 24 ? MMA_TS : TILE16);
      if (clg_status st = ensure_reduction(ctx, red2_doubles(nslots, w.nrhs, 1, E::NRED))) return st;
      const cudaError_t terr = dag ? launch_hop_tile_epi<true>(ctx, a, e, tcfg) : launch_hop_tile_epi<false>(ctx, a, e, tcfg);
      if (terr != cudaSuccess) return ctx->fail(cuda_status(terr), std::string("fused hop: ") + cudaGetErrorString(terr));
      return CLG_SUCCESS;
    }
    const int pcfg = tuned_hop_pair_config(ctx, w.U, plain, -1);
    const bool pair = ctx->hop_pair_mode == 1 || (ctx->hop_pair_mode == 2 && pcfg >= 0);
    if (w.nrhs >= 2 && pair && !a.seg) {
      const int cfg = pcfg >= 0 ? pcfg : 128;
      const int pbs = cfg & 0xffff;
      // partials are indexed [rhs][slot]: nslots x nrhs of them
      if (clg_status st = ensure_reduction(ctx, red2_doubles((w.Vh + pbs - 1) / pbs, w.nrhs, (w.nrhs + 1) / 2, E::NRED)))
        return st;
      const cudaError_t perr = dag ? launch_hop_pair_epi<true>(ctx, a, e, cfg) : launch_hop_pair_epi<false>(ctx, a, e, cfg);
      if (perr != cudaSuccess) return ctx->fail(cuda_status(perr), std::string("fused hop: ") + cudaGetErrorString(perr));
      return CLG_SUCCESS;
    }
  }
  if constexpr (P != P16) {
    // the tile form, when the autotuner chose it for the plain hop
    const int pc = w.nrhs >= 2 && !a.seg ? tuned_hop_config(ctx, w.U, plain, -1) : -1;
    if (pc >= 0 && (pc >> 16) >= 16) {
      const int64_t nslots = (w.Vh + TILE16 - 1) / TILE16;
      if (clg_status st = ensure_reduction(ctx, red2_doubles(nslots, w.nrhs, 1, E::NRED))) return st;
      cudaError_t terr;
      if constexpr (P == P64)
        terr = dag ? launch_hop_tileN_epi<P, 18, true>(ctx, a, e, pc) : launch_hop_tileN_epi<P, 18, false>(ctx, a, e, pc);
      else if (w.U->recon32 == 12)
        terr = dag ? launch_hop_tileN_epi<P, 12, true>(ctx, a, e, pc) : launch_hop_tileN_epi<P, 12, false>(ctx, a, e, pc);
      else
        terr = dag ? launch_hop_tileN_epi<P, 18, true>(ctx, a, e, pc) : launch_hop_tileN_epi<P, 18, false>(ctx, a, e, pc);
      if (terr != cudaSuccess) return ctx->fail(cuda_status(terr), std::string("fused hop: ") + cudaGetErrorString(terr));
      return CLG_SUCCESS;
    }
  }
  if (clg_status st = ensure_reduction(ctx, red2_doubles((w.Vh + bs - 1) / bs, w.nrhs, w.nrhs, E::NRED))) return st;
  cudaError_t err;
  if constexpr (P == P64) {
    err = dag ? launch_hop_epi<P, 18, true>(ctx, a, e, bs) : launch_hop_epi<P, 18, false>(ctx, a, e, bs);
  } else if constexpr (P == P32) {
    if (w.U->recon32 == 12)
      err = dag ? launch_hop_epi<P, 12, true>(ctx, a, e, bs) : launch_hop_epi<P, 12, false>(ctx, a, e, bs);
    else
      err = dag ? launch_hop_epi<P, 18, true>(ctx, a, e, bs) : launch_hop_epi<P, 18, false>(ctx, a, e, bs);
  } else {
    err = dag ? launch_hop_epi<P, 12, true>(ctx, a, e, bs) : launch_hop_epi<P, 12, false>(ctx, a, e, bs);
  }
  if (err != cudaSuccess) return ctx->fail(cuda_status(err), std::string("fused hop: ") + cudaGetErrorString(err));
  return CLG_SUCCESS;
}

// t_o = H_oe^(dag) in_e
}  // namespace (a kernel's template argument must not have internal linkage)

// The outer residual of a Wilson D / D^+ solve fused into the FP64 hop that
// computes D x on parity par: r = b - D x is stored in FP64 and in the inner
// precision PI (the next inner solve's right-hand side), and |r|^2 goes to
// out[rhs] (the first parity sets it, the second adds), so neither the
// separate residual pass nor the copy to the inner precision reads r again.
template <int PI>
struct ResidHop {
  static constexpr int NRED = 1;
  static constexpr bool STORE = false;
  DField b, r, rp;
  int par;
  bool first;
  double* out;
  template <typename AT>
  __device__ void site(int rhs, int64_t h, const cpx<AT> dx[12], double* red) const {
    cpx<double> v[12];
    ldv<P64, 12, double>(b, rhs, par, h, v);
#pragma unroll
    for (int k = 0; k < 12; ++k) v[k] = mk<double>(v[k].x - (double)dx[k].x, v[k].y - (double)dx[k].y);
    stv<P64, 12, double>(r, rhs, par, h, v);
    using AI = typename AccT<PI>::T;
    cpx<AI> vi[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) vi[k] = mk<AI>((AI)v[k].x, (AI)v[k].y);
    stv<PI, 12, AI>(rp, rhs, par, h, vi);
    red[0] += site_norm2<12, double>(v);
  }
  __device__ void finalize(int rhs, const double* s) const { out[rhs] = first ? s[0] : out[rhs] + s[0]; }
};

namespace {

template <int PI>
clg_status fused_residual_t(Work& w, bool dag, const FieldRef& b, const FieldRef& x, const FieldRef& r,
                            const FieldRef& rp, double* out) {
  clg_context_s* ctx = w.ctx;
  for (int par = 0; par < 2; ++par) {
    HopSpec s{};
    s.kind = CLG_FERMION_WILSON;
    s.prec = CLG_PREC_DOUBLE;
    s.dagger = dag;
    s.out_parity = par;
    s.in = x;
    s.out = r;  // not written by the hop (ResidHop::STORE is false): the epilogue stores r
    s.x = &x;
    s.a = make_double2(-w.param, 0.0);
    s.xa = make_double2(1.0, 0.0);
    s.nrhs = w.nrhs;
    HopArgs a;
    if (clg_status st = make_hop_args(ctx, w.U, s, a)) return st;
    const ResidHop<PI> e{dfield(b), dfield(r), dfield(rp), par, par == 0, out};
    HopSpec plain = s;
    plain.x = nullptr;
    const int pc = tuned_hop_config(ctx, w.U, plain, -1);
    cudaError_t err;
    if (w.nrhs >= 2 && pc >= 0 && (pc >> 16) >= 16) {
      const int64_t nslots = (w.Vh + TILE16 - 1) / TILE16;
      if (clg_status st = ensure_reduction(ctx, red2_doubles(nslots, w.nrhs, 1, 1))) return st;
      err = dag ? launch_hop_tileN_epi<P64, 18, true>(ctx, a, e, pc) : launch_hop_tileN_epi<P64, 18, false>(ctx, a, e, pc);
    } else {
      const int bs = tuned_hop_block(ctx, w.U, plain, 64);
      if (clg_status st = ensure_reduction(ctx, red2_doubles((w.Vh + bs - 1) / bs, w.nrhs, w.nrhs, 1))) return st;
      err = dag ? launch_hop_epi<P64, 18, true>(ctx, a, e, bs) : launch_hop_epi<P64, 18, false>(ctx, a, e, bs);
    }
    if (err != cudaSuccess) return ctx->fail(cuda_status(err), std::string("residual hop: ") + cudaGetErrorString(err));
  }
  return CLG_SUCCESS;
}

clg_status fused_residual(Work& w, bool dag, const FieldRef& b, const FieldRef& x, const FieldRef& r,
                          const FieldRef& rp, double* out) {
  return w.P == CLG_PREC_HALF     ? fused_residual_t<P16>(w, dag, b, x, r, rp, out)
         : w.P == CLG_PREC_SINGLE ? fused_residual_t<P32>(w, dag, b, x, r, rp, out)
                                  : fused_residual_t<P64>(w, dag, b, x, r, rp, out);
}

clg_status schur_hop_odd(Work& w, bool dag, const FieldRef& in_even, const FieldRef& t_odd, const int* skip, int ks) {
  HopSpec s;
  s.kind = CLG_FERMION_WILSON;
  s.prec = t_odd.prec;
  s.dagger = dag;
  s.out_parity = 1;
  s.in = in_even;
  s.out = t_odd;
  s.x = nullptr;
  s.a = make_double2(1.0, 0.0);
  s.xa = make_double2(0.0, 0.0);
  s.scale_dev = nullptr;
  s.scale_stride = 0;
  s.skip_dev = skip;
  s.skip_stride = ks;
  s.nrhs = w.nrhs;
  return hop(w.ctx, w.U, s);
}

// one CG iteration on A = M M^+ (m_dag_first) or M^+ M, fused as described above.
// Folding p = r + beta p into the second hop as well (hops on r, u = M^+ p
// carried as u = M^+ r + beta u, 4 kernels per iteration) measured no faster on
// the 32^3x16 FP16-inner solve: 13.44-13.72 against 13.26-13.36 ms (the
// epilogue re-reads r and spills at the 80-register cap)
template <int P>
clg_status cg_fused_iteration(Work& w, int op, const FieldRef& x, const FieldRef& r, const FieldRef& p,
                              const int* skip, int ks) {
  const bool d1 = op == CLG_OP_MEE_MEEDAG;  // the factor applied first is M^+
  const FieldRef& to = w.kt_odd.ref;
  const FieldRef& te = w.kt_even.ref;
  clg_status s;
  if ((s = schur_hop_odd(w, d1, p, to, skip, ks))) return s;
  if ((s = schur_hop_epi<P>(w, d1, to, p, te, CgHopAlpha<P>{w.st, op_weight(op)}, skip, ks))) return s;
  if ((s = schur_hop_odd(w, !d1, te, to, skip, ks))) return s;
  return schur_hop_epi<P>(w, !d1, to, te, te, CgHopUpdate<P>{dfield(x), dfield(r), dfield(p), w.st}, skip, ks);
}

clg_status krylov(Work& w, int op, const FieldRef& x, const FieldRef& b, int slot_base) {
  clg_context_s* ctx = w.ctx;
  const int nrhs = w.nrhs;
  kstate_reset<<<(nrhs + 63) / 64, 64, 0, ctx->stream>>>(w.st, w.outer_done_d, nrhs);
  ctx->kernels++;
  const int ks = (int)(sizeof(KState) / sizeof(int));
  const int* skip = &w.st[0].skip;
  const int fp = b.first_parity, np = b.nparity;
  const int64_t Vh = b.Vh;
  const int method = w.prm->kind;
  struct Ref {
    FieldRef ref;
  };
  int vidx = 0;
  auto vec = [&](Ref& o) { return w.kvec(slot_base, vidx++, np, fp, o.ref); };

  if (method == CLG_SOLVER_BICGSTAB || (method == CLG_SOLVER_CG && !hermitian_op(op))) {
    if (method == CLG_SOLVER_CG) return ctx->fail(CLG_ERR_BAD_ARG, "CG needs a Hermitian operator (DDdagger forms)");
    Ref r, rh, p, v, t;
    clg_status s;
    if ((s = vec(r)) || (s = vec(rh)) || (s = vec(p)) || (s = vec(v)) || (s = vec(t))) return s;
    s = with_pn(w.P, w.nc, [&](auto PP, auto NN) -> clg_status {
      constexpr int PV = PP.value, NV = NN.value;
      BiInit<PV, NV> init{dfield(b), dfield(x), dfield(r.ref), dfield(rh.ref), dfield(p.ref), w.st, w.tol_d};
      clg_status q = launch_sites<1>(ctx, init, fp, np, Vh, nrhs);
      if (q) return q;
      auto body = [&]() -> clg_status {
        clg_status e;
        if ((e = kapply(w, op, v.ref, p.ref, nullptr, 0, skip, ks))) return e;
        if ((e = launch_sites<2>(ctx, BiAlpha<PV, NV>{dfield(rh.ref), dfield(v.ref), w.st}, fp, np, Vh, nrhs))) return e;
        if ((e = launch_sites<1>(ctx, BiS<PV, NV>{dfield(r.ref), dfield(v.ref), w.st}, fp, np, Vh, nrhs))) return e;
        if ((e = kapply(w, op, t.ref, r.ref, nullptr, 0, skip, ks))) return e;
        if ((e = launch_sites<3>(ctx, BiOmega<PV, NV>{dfield(t.ref), dfield(r.ref), w.st}, fp, np, Vh, nrhs))) return e;
        BiUpdate<PV, NV> up{dfield(x), dfield(p.ref), dfield(r.ref), dfield(t.ref), dfield(rh.ref), w.st};
        if ((e = launch_sites<3>(ctx, up, fp, np, Vh, nrhs))) return e;
        return launch_sites<0>(ctx, BiP<PV, NV>{dfield(p.ref), dfield(r.ref), dfield(v.ref), w.st}, fp, np, Vh, nrhs);
      };
      const int chunk = 8;
      return iterate(w, slot_base + 0, chunk, w.prm->max_iterations / (2 * chunk) + 2, body);
    });
    return s;
  }

  if (method == CLG_SOLVER_CG) {
    Ref r, p, q;
    clg_status s;
    if ((s = vec(r)) || (s = vec(p)) || (s = vec(q))) return s;
    return with_pn(w.P, w.nc, [&](auto PP, auto NN) -> clg_status {
      constexpr int PV = PP.value, NV = NN.value;
      CgInit<PV, NV> init{dfield(b), dfield(x), dfield(r.ref), dfield(p.ref), w.st, w.tol_d};
      clg_status e = launch_sites<1>(ctx, init, fp, np, Vh, nrhs);
      if (e) return e;
      const bool fused = NV == 12 && fused_cg(w, op);
      auto body = [&]() -> clg_status {
        clg_status e2;
        if (fused) {
          if constexpr (NV == 12)
            if ((e2 = cg_fused_iteration<PV>(w, op, x, r.ref, p.ref, skip, ks))) return e2;
        } else {
          if ((e2 = kapply(w, op, q.ref, p.ref, nullptr, 0, skip, ks))) return e2;
          CgAlpha<PV, NV> ca{dfield(p.ref), dfield(q.ref), w.st, op_weight(op)};
          if ((e2 = launch_sites<2>(ctx, ca, fp, np, Vh, nrhs))) return e2;
          CgUpdate<PV, NV> up{dfield(x), dfield(r.ref), dfield(p.ref), dfield(q.ref), w.st};
          if ((e2 = launch_sites<1>(ctx, up, fp, np, Vh, nrhs))) return e2;
        }
        return launch_sites<0>(ctx, CgP<PV, NV>{dfield(p.ref), dfield(r.ref), w.st}, fp, np, Vh, nrhs);
      };
      // 8 iterations per chunk: an inner solve overshoots its convergence by
      // fewer (skipped) iterations; measured on the 32^3x16 FP16-inner solve
      // against chunks of 4, 12 and 16 (65.5, 66.0, 67.2 -> 69.8 solves/s)
      const int chunk = 8;
      return iterate(w, slot_base + 1, chunk, w.prm->max_iterations / chunk + 2, body, true);
    });
  }

  if (method == CLG_SOLVER_GMRES) {
    const int k = std::min(std::max(w.prm->max_dim, 1), GM_MAXK);
    Ref V[GM_MAXK + 1], wv;
    clg_status s;
    for (int i = 0; i <= k; ++i)
      if ((s = vec(V[i]))) return s;
    if ((s = vec(wv))) return s;
    if ((s = blas_zero(ctx, x))) return s;
    return with_pn(w.P, w.nc, [&](auto PP, auto NN) -> clg_status {
      constexpr int PV = PP.value, NV = NN.value;
      VList vl;
      for (int i = 0; i <= GM_MAXK; ++i) vl.v[i] = dfield(V[std::min(i, k)].ref);
      // first cycle start (x = 0)
      GmStart<PV, NV> st0{dfield(b), dfield(wv.ref), dfield(V[0].ref), w.st, 0, w.tol_d, 1};
      clg_status e = launch_sites<1>(ctx, st0, fp, np, Vh, nrhs);
      if (e) return e;
      bool first_cycle = true;
      auto cycle = [&]() -> clg_status {
        clg_status e2;
        if (!first_cycle) {
          // restart: V'_0 = b - K x
          if ((e2 = kapply(w, op, wv.ref, x, nullptr, 0, &w.st[0].done, ks))) return e2;
          GmStart<PV, NV> sr{dfield(b), dfield(wv.ref), dfield(V[0].ref), w.st, 1, w.tol_d, 0};
          if ((e2 = launch_sites<1>(ctx, sr, fp, np, Vh, nrhs))) return e2;
        }
        for (int j = 0; j < k; ++j) {
          if ((e2 = kapply(w, op, wv.ref, V[j].ref, &w.st[0].s[j], (int)(sizeof(KState) / sizeof(double)), skip, ks)))
            return e2;
          if ((e2 = launch_gm_dots<PV, NV, 0>(ctx, vl, wv.ref, w.st, j, fp, np, Vh, nrhs))) return e2;
          if ((e2 = launch_sites<1>(ctx, GmOrtho<PV, NV>{vl, dfield(wv.ref), w.st, j}, fp, np, Vh, nrhs))) return e2;
        }
        gm_solve_y<<<(nrhs + 63) / 64, 64, 0, ctx->stream>>>(w.st, nrhs);
        ctx->kernels++;
        if ((e2 = launch_sites<0>(ctx, GmUpdate<PV, NV>{vl, dfield(x), w.st, k}, fp, np, Vh, nrhs))) return e2;
        gm_finish<<<(nrhs + 63) / 64, 64, 0, ctx->stream>>>(w.st, nrhs);
        ctx->kernels++;
        return CLG_SUCCESS;
      };
      // the first cycle runs eagerly (it has no restart prologue); later cycles replay a graph
      e = cycle();
      if (e) return e;
      first_cycle = false;
      e = read_summary(w);
      if (e) return e;
      bool all = true;
      for (int r = 0; r < nrhs; ++r) all = all && w.sum_h[r].done;
      if (all) return CLG_SUCCESS;
      return iterate(w, slot_base + 2, 1, w.prm->max_iterations / k + 2, cycle);
    });
  }
  return ctx->fail(CLG_ERR_UNSUPPORTED, "solver kind not available for clg_solve");
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

clg_status clg_solver_default_params(int kind, clg_solver_params* p) {
  if (!p) return CLG_ERR_BAD_ARG;
  std::memset(p, 0, sizeof(*p));
  p->kind = kind;
  p->max_dim = 12;          // TestSuit_FermionUpdator.yaml:529-645 (GMRES MaxDim 12)
  p->restart = 100;
  p->accuracy = 1e-20;
  p->absolute_accuracy = 0;
  p->deviation_step = 10;   // CSolverBiCGstab.cpp:33-93 keys
  p->max_step = 100;
  p->small_rho = 1e-30;
  p->inner_precision = CLG_PREC_SINGLE;
  p->tol_true_rel = 1e-10;
  // multi-shift CG: the shared iteration leaves FP64 for the inner precision
  // once |r| <= inner_tol |b|
  p->inner_tol = kind == CLG_SOLVER_CGM ? 1e-4 : 1e-5;
  p->max_iterations = 200000;
  p->max_outer = 40;
  p->even_odd = 1;
  p->use_graphs = 1;
  if (kind == CLG_SOLVER_GCRODR || kind == CLG_SOLVER_GMRESMDR) {
    p->max_dim = 10;  // CSolverGCRODR.cpp:67-90: MDim 10, KDim MDim - 2
    p->kdim = 8;
    p->inner_precision = CLG_PREC_DOUBLE;
  }
  return CLG_SUCCESS;
}

clg_status clg_solver_create(clg_context ctx, const clg_solver_params* p, clg_solver* out) {
  if (!ctx || !p || !out) return CLG_ERR_BAD_ARG;
  if (p->kind < 0 || p->kind > CLG_SOLVER_GMRES_MS || p->inner_precision < 0 || p->inner_precision > 2 ||
      !(p->tol_true_rel > 0) || p->max_iterations < 1 || p->max_outer < 1)
    return ctx->fail(CLG_ERR_BAD_ARG, "invalid solver parameters");
  if ((p->kind == CLG_SOLVER_GMRES || p->kind == CLG_SOLVER_NESTED_MS) && (p->max_dim < 1 || p->max_dim > GM_MAXK))
    return ctx->fail(CLG_ERR_UNSUPPORTED, "GMRES MaxDim must be in [1, 16] on the device");
  if ((p->kind == CLG_SOLVER_FOM_MS || p->kind == CLG_SOLVER_GMRES_MS) &&
      (p->max_dim < 2 || p->max_dim > 32 || p->restart < 1))
    return ctx->fail(CLG_ERR_BAD_ARG, "multi-shift FOM / GMRES: MaxDim in [2, 32], Restart >= 1");
  if ((p->kind == CLG_SOLVER_GCRODR || p->kind == CLG_SOLVER_GMRESMDR) &&
      (p->max_dim < 5 || p->max_dim > 32 || p->kdim < 0 || (p->kdim > 0 && (p->kdim < 2 || p->kdim > p->max_dim - 2)) ||
       p->deflation < CLG_DEFLATION_SVD || p->deflation > CLG_DEFLATION_HEV))
    return ctx->fail(CLG_ERR_BAD_ARG, "GCRO-DR: MDim in [5, 32], KDim in [2, MDim - 2], deflation SVD / REV / HEV");
  clg_solver_s* s = new clg_solver_s();
  s->ctx = ctx;
  s->p = *p;
  *out = s;
  return CLG_SUCCESS;
}

clg_status clg_solver_destroy(clg_solver s) {
  if (!s) return CLG_ERR_BAD_ARG;
  delete s;
  return CLG_SUCCESS;
}

clg_status clg_solve(clg_solver S, clg_field X, clg_field B, clg_gauge U, int op, clg_field X0, clg_solve_info* info) {
  if (!S || !X || !B || !U || !info) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = S->ctx;
  if (X->lat != B->lat || U->lat != B->lat || X->kind != B->kind || X->subset != B->subset || X->nrhs != B->nrhs ||
      (X0 && (X0->lat != B->lat || X0->subset != B->subset || X0->nrhs != B->nrhs || X0->kind != B->kind)))
    return ctx->fail(CLG_ERR_BAD_ARG, "solve: field shapes differ");
  if (S->p.kind == CLG_SOLVER_CGM || S->p.kind == CLG_SOLVER_FOM_MS || S->p.kind == CLG_SOLVER_NESTED_MS ||
      S->p.kind == CLG_SOLVER_BICGSTAB_MS || S->p.kind == CLG_SOLVER_GMRES_MS)
    return ctx->fail(CLG_ERR_BAD_ARG, "multi-shift solvers are called through clg_solve_multishift");
  if (S->p.kind == CLG_SOLVER_GCRODR || S->p.kind == CLG_SOLVER_GMRESMDR) return gcrodr_solve(S, X, B, U, op, X0, info);
  for (clg_field f : {X, B, X0})
    if (f)
      if (clg_status st = settle(f)) return st;
  SolveReq q;
  q.cache = &S->cache;
  q.ctx = ctx;
  q.prm = &S->p;
  q.U = U;
  q.lat = B->lat;
  q.kind = B->kind;
  q.param = B->param;
  q.op = op;
  q.subset = B->subset;
  q.nrhs = B->nrhs;
  q.b = B->ref();
  FieldRef x0r;
  if (X0) {
    x0r = X0->ref();
    q.x0 = &x0r;
  }
  q.xout.push_back(X->ref());
  q.info = info;
  return solve_core(q);
}

}  // extern "C"

clg_status clg::solve_core(const SolveReq& q) {
  clg_context_s* ctx = q.ctx;
  clg_gauge_s* U = q.U;
  const int op = q.op;
  const double t0 = now_s();
  clg_solve_info* info = q.info;
  const bool full = q.subset == CLG_SUBSET_FULL;
  const bool wilson = q.kind == CLG_FERMION_WILSON;
  const bool even_ops = op == CLG_OP_MEE || op == CLG_OP_MEE_DAG || op == CLG_OP_MEE_MEEDAG || op == CLG_OP_DDDAG_EE;
  if (even_ops == full) return ctx->fail(CLG_ERR_BAD_ARG, "solve: Schur operators act on EVEN fields, D forms on FULL");
  if (!(op == CLG_OP_D || op == CLG_OP_DDAG || op == CLG_OP_DDDAG || even_ops))
    return ctx->fail(CLG_ERR_UNSUPPORTED, "solve: operator not supported");
  if ((op == CLG_OP_MEE || op == CLG_OP_MEE_DAG || op == CLG_OP_MEE_MEEDAG) && !wilson)
    return ctx->fail(CLG_ERR_BAD_ARG, "MEE forms are Wilson operators");
  if (op == CLG_OP_DDDAG_EE && wilson) return ctx->fail(CLG_ERR_BAD_ARG, "DDDAG_EE is the staggered Schur operator");
  if (q.shifts && (op == CLG_OP_D || op == CLG_OP_DDAG) && q.prm->kind == CLG_SOLVER_CG)
    return ctx->fail(CLG_ERR_BAD_ARG, "CG needs a Hermitian operator");

  clg_status s = CLG_SUCCESS;
  const int P = q.prm->inner_precision;
  if ((s = gauge_prepare(U, P))) return s;
  const L2LinkWindow l2(ctx, U, P);
  // The workspace (buffers, pinned memory, captured graphs) lives in the solver
  // and is reused while the shape of the solve and the gauge arrays stay the same.
  const std::string key =
      std::to_string((uintptr_t)q.lat) + "/" + std::to_string(q.kind) + "/" + std::to_string(q.subset) + "/" +
      std::to_string(q.nrhs) + "/" + std::to_string(op) + "/" + std::to_string(P) + "/" + std::to_string(q.prm->kind) +
      "/" + std::to_string(q.prm->max_dim) + "/" + std::to_string(q.prm->even_odd) + "/" +
      std::to_string(q.prm->use_graphs) + "/" + std::to_string((uintptr_t)U) + "/" +
      std::to_string((uintptr_t)U->u64[0]) + "/" + std::to_string((uintptr_t)U->u32[0]) + "/" +
      std::to_string((uintptr_t)U->u16[0]) + "/" + std::to_string(q.shifts != nullptr) + "/" +
      std::to_string(q.b_broadcast) + "/" + std::to_string(q.param);
  std::unique_ptr<Work> local;
  Work* wp = nullptr;
  if (q.cache) {
    Work* cw = dynamic_cast<Work*>(q.cache->get());
    if (!cw || cw->key != key) {
      cudaStreamSynchronize(ctx->stream);
      q.cache->reset();
      cw = new Work();
      q.cache->reset(cw);
    }
    wp = cw;
  } else {
    local.reset(new Work());
    wp = local.get();
  }
  Work& w = *wp;
  w.key = key;
  w.ctx = ctx;
  w.U = U;
  w.kind = q.kind;
  w.op = op;
  w.P = P;
  w.nc = q.kind == CLG_FERMION_WILSON ? 12 : 3;
  w.nrhs = q.nrhs;
  w.param = q.param;
  w.Vh = q.lat->g.Vh;
  w.prm = q.prm;
  const int nrhs = w.nrhs;
  const clg_solver_params* prm = q.prm;
  if (!w.st) {
    if ((s = dalloc(ctx, (void**)&w.st, sizeof(KState) * nrhs)) ||
        (s = dalloc(ctx, (void**)&w.sum_d, sizeof(Summary) * nrhs)) ||
        (s = dalloc(ctx, (void**)&w.outer_done_d, sizeof(int) * nrhs)) ||
        (s = dalloc(ctx, (void**)&w.tol_d, sizeof(double) * nrhs)) ||
        (s = dalloc(ctx, (void**)&w.red_d, sizeof(double) * 2 * nrhs)))
      return s;
    if (cudaMallocHost((void**)&w.sum_h, sizeof(Summary) * nrhs) != cudaSuccess ||
        cudaMallocHost((void**)&w.host_buf, sizeof(double) * 4 * nrhs + 64) != cudaSuccess)
      return ctx->fail(CLG_ERR_OOM, "pinned host buffer");
    if (cudaHostGetDevicePointer((void**)&w.sum_hd, w.sum_h, 0) != cudaSuccess ||
        cudaHostGetDevicePointer((void**)&w.host_buf_d, w.host_buf, 0) != cudaSuccess) {
      cudaGetLastError();
      w.sum_hd = nullptr;
      w.host_buf_d = nullptr;
    }
  }
  cudaMemsetAsync(w.st, 0, sizeof(KState) * nrhs, ctx->stream);

  // Schur (even-odd) path for D / D^+ on full fields; Wilson DD^+ = two Schur solves
  const bool schur =
      full && prm->even_odd && !q.shifts && (op == CLG_OP_D || op == CLG_OP_DDAG || (op == CLG_OP_DDDAG && wilson));
  if (q.shifts) {
    if (!w.shift_dev && (s = dalloc(ctx, (void**)&w.shift_dev, sizeof(double2) * nrhs))) return s;
    if (cudaMemcpyAsync(w.shift_dev, q.shifts, sizeof(double2) * nrhs, cudaMemcpyHostToDevice, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      return ctx->fail(CLG_ERR_CUDA, "solve: shifts upload");
  }
  const int kop_d = wilson ? CLG_OP_MEE : CLG_OP_DDDAG_EE;
  const int kop_ddag = wilson ? CLG_OP_MEE_DAG : CLG_OP_DDDAG_EE;
  const int64_t Vh = w.Vh;
  const int nc = w.nc;

  // FP64 outer vectors
  Owned &x64 = w.x64, &b64 = w.b64, &r64 = w.r64, &t64 = w.t64;
  const int npar = full ? 2 : 1;
  if ((s = x64.alloc(ctx, 0, nc, npar, 0, nrhs, Vh)) || (s = b64.alloc(ctx, 0, nc, npar, 0, nrhs, Vh)) ||
      (s = r64.alloc(ctx, 0, nc, npar, 0, nrhs, Vh)))
    return s;
  if ((s = t64.alloc(ctx, 0, nc, full ? 2 : 1, full ? 0 : 1, nrhs, Vh))) return s;
  // inner-precision vectors
  // CG on a Wilson D / D^+ solve: the Schur system through its normal equations
  // (CGNE: M M^+ y = b, x = M^+ y; CGNR for D^+: M^+ M y = b, x = M y)
  const bool cgne = schur && wilson && prm->kind == CLG_SOLVER_CG;
  Owned &rP = w.rP, &eP = w.eP, &yP = w.yP, &bS = w.bS, &yS = w.yS;
  if ((s = rP.alloc(ctx, w.P, nc, npar, 0, nrhs, Vh)) || (s = eP.alloc(ctx, w.P, nc, npar, 0, nrhs, Vh))) return s;
  if (schur) {
    if ((s = bS.alloc(ctx, w.P, nc, 1, 0, nrhs, Vh))) return s;
    if (op == CLG_OP_DDDAG && (s = yP.alloc(ctx, w.P, nc, 2, 0, nrhs, Vh))) return s;
    if (cgne && (s = yS.alloc(ctx, w.P, nc, 1, 0, nrhs, Vh))) return s;
  }
  if ((s = w.kt_odd.alloc(ctx, w.P, nc, 1, 1, nrhs, Vh))) return s;
  if ((op == CLG_OP_MEE_MEEDAG || cgne) && (s = w.kt_even.alloc(ctx, w.P, nc, 1, 0, nrhs, Vh))) return s;
  if (!schur && op == CLG_OP_DDDAG && (s = w.kt_full.alloc(ctx, w.P, nc, 2, 0, nrhs, Vh))) return s;

  // b64 = B, x64 = X0 or 0
  if (q.b_broadcast) {
    for (int r = 0; r < nrhs; ++r)
      if ((s = blas_copy(ctx, b64.ref.rhs_view(r, 1), q.b.rhs_view(0, 1)))) return s;
  } else if ((s = blas_copy(ctx, b64.ref, q.b))) {
    return s;
  }
  if (q.x0) s = blas_copy(ctx, x64.ref, *q.x0);
  else s = blas_zero(ctx, x64.ref);
  if (s) return s;
  if ((s = blas_norm2(ctx, b64.ref, w.red_d))) return s;
  std::vector<double> bn2(nrhs), rn2(nrhs);
  if (to_host(w, w.red_d, sizeof(double) * nrhs) != cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return ctx->fail(CLG_ERR_CUDA, "solve: reading |b|");
  for (int r = 0; r < nrhs; ++r) bn2[r] = w.host_buf[r];

  const double tol = prm->tol_true_rel;
  std::vector<int> done(nrhs, 0), outer_count(nrhs, 0), status(nrhs, CLG_ERR_NOT_CONVERGED), iters(nrhs, 0);
  std::vector<int> inner_fail(nrhs, 0);
  const double2 one = make_double2(1, 0);
  // floor of the inner tolerance per precision.  FP16 on the 32^3x16 solve:
  // 2e-3 -> 230 applications in 5 outer cycles, 13.5 ms; 1e-3 -> 238 / 5,
  // 14.2 ms; 5e-4 -> 240 / 4, 13.4 ms; 2e-4 -> 244 / 4, 13.3 ms (within run noise)
  const double lo_tol = w.P == CLG_PREC_DOUBLE ? 1e-14 : (w.P == CLG_PREC_SINGLE ? 1e-6 : 2e-3);
  const char* venv = std::getenv("CLG_VERBOSE");
  const bool verbose = venv && venv[0] == '1';
  int outer = 0;
  // the residual fused into the FP64 hop (Wilson D / D^+ on full fields, no
  // shift, one lattice) from the second cycle on: the first cycle runs the
  // plain hops, which also time their launch configuration
  const bool fuse_resid = ctx->fused_resid && wilson && full && nc == 12 && !w.shift_dev && !U->seg &&
                          (op == CLG_OP_D || op == CLG_OP_DDAG);
  bool rp_ready = false;
  for (;; ++outer) {
    // r = b - A x  (FP64, true residual)
    rp_ready = false;
    if (fuse_resid && outer > 0) {
      if ((s = fused_residual(w, op == CLG_OP_DDAG, b64.ref, x64.ref, r64.ref, rP.ref, w.red_d))) return s;
      rp_ready = true;
      goto residual_done;
    }
    {
    const FieldRef* tmp = (op == CLG_OP_DDDAG) ? nullptr : &t64.ref;
    Owned& tf = w.tf;
    if (op == CLG_OP_DDDAG) {
      if ((s = tf.alloc(ctx, 0, nc, 2, 0, nrhs, Vh))) return s;
      tmp = &tf.ref;
    }
    if (op == CLG_OP_MEE_MEEDAG) {
      Owned& te = w.te;
      if ((s = te.alloc(ctx, 0, nc, 1, 0, nrhs, Vh))) return s;
      if ((s = apply_op(ctx, CLG_OP_MEE_DAG, U, w.kind, w.param, te.ref, x64.ref, &t64.ref, one, nrhs))) return s;
      if ((s = apply_op(ctx, CLG_OP_MEE, U, w.kind, w.param, r64.ref, te.ref, &t64.ref, one, nrhs))) return s;
      if ((s = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? CLG_SUCCESS : CLG_ERR_CUDA)) return s;
    } else {
      if ((s = apply_op(ctx, op, U, w.kind, w.param, r64.ref, x64.ref, tmp, one, nrhs))) return s;
    }
    if (w.shift_dev) {
      s = with_pn(0, nc, [&](auto PP, auto NN) {
        ShiftAdd<PP.value, NN.value> f{dfield(r64.ref), dfield(x64.ref), w.shift_dev, nullptr, 0, nullptr, 0};
        return launch_sites<0>(ctx, f, 0, npar, Vh, nrhs);
      });
      if (s) return s;
    }
    s = with_pn(0, nc, [&](auto, auto NN) {
      return launch_sites<1>(ctx, Resid<NN.value>{dfield(b64.ref), dfield(r64.ref), w.red_d}, 0, npar, Vh, nrhs);
    });
    if (s) return s;
    }
  residual_done:
    if (to_host(w, w.red_d, sizeof(double) * nrhs) != cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      return ctx->fail(CLG_ERR_CUDA, "solve: reading |r|");
    bool all = true;
    for (int r = 0; r < nrhs; ++r) {
      rn2[r] = w.host_buf[r];
      if (!done[r]) {
        const bool ok = bn2[r] == 0.0 ? rn2[r] == 0.0 : std::sqrt(rn2[r]) <= tol * std::sqrt(bn2[r]);
        if (ok) {
          done[r] = 1;
          status[r] = CLG_SUCCESS;
        } else if (!(rn2[r] == rn2[r])) {
          done[r] = 1;
          status[r] = CLG_ERR_BREAKDOWN;
        }
      }
      all = all && done[r];
    }
    if (all || outer >= prm->max_outer) break;
    int budget_left = 0;
    for (int r = 0; r < nrhs; ++r)
      if (!done[r]) budget_left = std::max(budget_left, prm->max_iterations - iters[r]);
    if (budget_left <= 0) break;
    w.inner_cap = budget_left;
    // inner tolerances
    for (int r = 0; r < nrhs; ++r) {
      double want = done[r] ? 1.0 : 0.5 * tol * std::sqrt(bn2[r] / std::max(rn2[r], 1e-300));
      if (w.P != CLG_PREC_DOUBLE) want = std::max(want, prm->inner_tol);
      w.host_buf[r] = std::min(0.5, std::max(want, lo_tol));
      ((int*)(w.host_buf + nrhs))[r] = done[r];
      if (!done[r]) outer_count[r]++;
    }
    if (w.host_buf_d) {
      small_copy(ctx, w.tol_d, w.host_buf_d, sizeof(double) * nrhs);
      small_copy(ctx, w.outer_done_d, w.host_buf_d + nrhs, sizeof(int) * nrhs);
    } else {
      cudaMemcpyAsync(w.tol_d, w.host_buf, sizeof(double) * nrhs, cudaMemcpyHostToDevice, ctx->stream);
      cudaMemcpyAsync(w.outer_done_d, w.host_buf + nrhs, sizeof(int) * nrhs, cudaMemcpyHostToDevice, ctx->stream);
    }
    // e ~= A^{-1} r in the inner precision
    if (!rp_ready && (s = blas_copy(ctx, rP.ref, r64.ref))) return s;
    auto schur_solve = [&](bool dag, const FieldRef& rhs, const FieldRef& sol) -> clg_status {
      clg_status q;
      FieldRef rhs_e = rhs.parity_view(0), rhs_o = rhs.parity_view(1);
      FieldRef sol_e = sol.parity_view(0), sol_o = sol.parity_view(1);
      // bS = rhs_e + kappa H_eo rhs_o  (Wilson) ; m rhs_e -/+ H_eo rhs_o (staggered D / D^+)
      HopSpec h1{};
      h1.kind = w.kind;
      h1.prec = w.P;
      h1.dagger = dag && wilson;
      h1.out_parity = 0;
      h1.in = rhs_o;
      h1.out = bS.ref;
      h1.x = &rhs_e;
      h1.a = wilson ? make_double2(w.param, 0) : make_double2(dag ? 1.0 : -1.0, 0);
      h1.xa = wilson ? one : make_double2(w.param, 0);
      h1.skip_dev = w.outer_done_d;
      h1.skip_stride = 1;
      h1.nrhs = nrhs;
      if ((q = hop(ctx, U, h1))) return q;
      if (cgne) {
        // M M^+ y = bS, sol_e = M^+ y   (D^+: M^+ M y = bS, sol_e = M y)
        if ((q = krylov(w, dag ? OP_MEEDAG_MEE : CLG_OP_MEE_MEEDAG, yS.ref, bS.ref, dag ? 10 : 0))) return q;
        if ((q = apply_op(ctx, dag ? CLG_OP_MEE : CLG_OP_MEE_DAG, U, w.kind, w.param, sol_e, yS.ref, &w.kt_odd.ref, one,
                          nrhs, nullptr, 0, w.outer_done_d, 1)))
          return q;
      } else if ((q = krylov(w, dag ? kop_ddag : kop_d, sol_e, bS.ref, dag ? 10 : 0))) {
        return q;
      }
      // sol_o = rhs_o + kappa H_oe sol_e (Wilson) ; (rhs_o -/+ H_oe sol_e) / m (staggered)
      HopSpec h2 = h1;
      h2.out_parity = 1;
      h2.in = sol_e;
      h2.out = sol_o;
      h2.x = &rhs_o;
      h2.a = wilson ? make_double2(w.param, 0) : make_double2((dag ? 1.0 : -1.0) / w.param, 0);
      h2.xa = wilson ? one : make_double2(1.0 / w.param, 0);
      return hop(ctx, U, h2);
    };
    if (schur) {
      if (op == CLG_OP_DDDAG) {
        if ((s = schur_solve(false, rP.ref, yP.ref))) return s;
        s = schur_solve(true, yP.ref, eP.ref);
      } else {
        s = schur_solve(op == CLG_OP_DDAG, rP.ref, eP.ref);
      }
    } else {
      s = krylov(w, op, eP.ref, rP.ref, 0);
    }
    if (s) return s;
    if ((s = read_summary(w))) return s;
    for (int r = 0; r < nrhs; ++r) {
      if (done[r]) continue;
      iters[r] += w.sum_h[r].iters;
      if (w.sum_h[r].status == ST_BREAKDOWN) inner_fail[r]++;
      if (verbose)  // the reference logs per-restart deviations at PARANOIAC level (CSolverGMRES.cpp:234,246)
        std::fprintf(stderr, "clg_solve outer %d rhs %d: |r|/|b| = %.3e, inner tol %.1e, inner applications %d, "
                     "inner status %d, inner |r|/|r0| = %.3e\n", outer, r, std::sqrt(rn2[r] / std::max(bn2[r], 1e-300)),
                     w.host_buf[r], w.sum_h[r].iters, w.sum_h[r].status,
                     w.sum_h[r].rr0 > 0 ? std::sqrt((w.sum_h[r].rr > 0 ? w.sum_h[r].rr : w.sum_h[r].resid_est * w.sum_h[r].resid_est) / w.sum_h[r].rr0) : 0.0);
    }
    // x += e
    s = with_pn(w.P, nc, [&](auto PP, auto NN) {
      AddConv<PP.value, NN.value> f{dfield(x64.ref), dfield(eP.ref), w.outer_done_d};
      return launch_sites<0>(ctx, f, 0, npar, Vh, nrhs);
    });
    if (s) return s;
  }
  // write the solution
  if (q.xout.size() == 1) {
    if ((s = blas_copy(ctx, q.xout[0], x64.ref))) return s;
  } else {
    for (int r = 0; r < nrhs && r < (int)q.xout.size(); ++r)
      if ((s = blas_copy(ctx, q.xout[r], x64.ref.rhs_view(r, 1)))) return s;
  }
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return ctx->fail(CLG_ERR_CUDA, "solve: final sync");
  const double t1 = now_s();
  clg_status overall = CLG_SUCCESS;
  for (int r = 0; r < nrhs; ++r) {
    info[r].status = status[r];
    if (status[r] != CLG_SUCCESS && inner_fail[r] && status[r] == CLG_ERR_NOT_CONVERGED) info[r].status = CLG_ERR_BREAKDOWN;
    info[r].iterations = iters[r];
    info[r].restarts = 0;
    info[r].outer = outer_count[r];
    info[r].true_rel_residual = bn2[r] > 0 ? std::sqrt(rn2[r] / bn2[r]) : std::sqrt(rn2[r]);
    info[r].seconds = t1 - t0;
    if (info[r].status != CLG_SUCCESS && overall == CLG_SUCCESS) overall = info[r].status;
  }
  return overall;
}
