// api.cu -- the C ABI (include/clg_b200.h): contexts, lattices, gauge and
// fermion fields, operator application (CField::ApplyOperator,
// Data/Field/CField.h:203) and field BLAS.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "blas.cuh"
#include "internal.h"

namespace clg {

clg_status gauge_generate(clg_gauge_s* U, int init, uint64_t seed, uint32_t fid, double eps);
clg_status gauge_reorder(clg_gauge_s* U, double* dev_buf, int layout, int to_device);
clg_status field_reorder(clg_field_s* f, int rhs, double* dev_buf, int to_device);
clg_status field_stream(clg_field_s* f, int rhs, double* host_dev, int to_device, cudaStream_t s);
clg_status field_source(clg_field_s* f, int rhs, int kind, uint64_t seed, uint32_t fid, int64_t site, int comp);
clg_status gauge_plaquette(clg_gauge_s* U, double* host_out);
clg_status gauge_unitarity(clg_gauge_s* U, double* host_out);

clg_status cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return CLG_SUCCESS;
  if (e == cudaErrorMemoryAllocation) return CLG_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return CLG_ERR_NO_DEVICE;
  return CLG_ERR_CUDA;
}

int64_t site_bytes_of(int prec, int nc) { return (int64_t)nc * (prec == 0 ? 16 : (prec == 1 ? 8 : 4)); }

clg_status dalloc(clg_context_s* ctx, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return CLG_SUCCESS;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return ctx->fail(cuda_status(e), std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
  }
  return CLG_SUCCESS;
}
void dfree(void* p) {
  if (p) cudaFree(p);
}

// bytes of one right-hand side of a host (FP64 lexicographic) field array
static size_t host_rhs_bytes(const clg_field_s* f) { return (size_t)f->lat->g.V * f->nc() * 2 * sizeof(double); }

// The device address of a host buffer that the SMs can read and write
// directly (pinned, mapped into the device's address space, 16-byte aligned),
// for a field that takes the zero-copy path (FP64, CLG_ZERO_COPY=1), or
// nullptr: pageable memory and other fields go through a device slot.
static double* mapped_host(const clg_field_s* f, const void* p) {
  const clg_context_s* ctx = f->lat->ctx;
  if (!ctx->zero_copy || f->prec != CLG_PREC_DOUBLE || (reinterpret_cast<uintptr_t>(p) & 15)) return nullptr;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // not a pointer the runtime knows: pageable
    return nullptr;
  }
  if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
  return static_cast<double*>(a.devicePointer);
}

// copy stream, staging slots (unless the transfer is zero-copy) and events of
// the asynchronous transfers
static clg_status xfer_prepare(clg_field_s* f, bool import, bool slot) {
  clg_context_s* ctx = f->lat->ctx;
  if (!ctx->copy_stream && cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    ctx->copy_stream = nullptr;
    return ctx->fail(CLG_ERR_CUDA, "copy stream");
  }
  void*& buf = import ? f->xin : f->xout;
  if (slot && !buf)
    if (clg_status st = dalloc(ctx, &buf, host_rhs_bytes(f) * f->nrhs)) return st;
  auto make = [&](std::vector<cudaEvent_t>& v) -> bool {
    if (!v.empty()) return true;
    v.assign(f->nrhs, nullptr);
    for (auto& e : v)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
    return true;
  };
  const bool ok = import ? (make(f->in_copied) && make(f->in_consumed)) : (make(f->out_ready) && make(f->out_copied));
  if (!ok) return ctx->fail(CLG_ERR_CUDA, "transfer events");
  if (import && f->in_pending.empty()) f->in_pending.assign(f->nrhs, 0);
  if (!import && f->out_pending.empty()) f->out_pending.assign(f->nrhs, 0);
  return CLG_SUCCESS;
}

// Orders the context stream after the field's asynchronous transfers: an
// import's data is in the field (reordered out of its slot, or written in
// place), and no zero-copy export still reads it.  Every entry point that
// reads or writes a field calls this first.
clg_status settle(clg_field_s* f) {
  clg_context_s* ctx = f->lat->ctx;
  for (int r = 0; r < (int)f->out_pending.size(); ++r) {
    if (!f->out_pending[r]) continue;
    f->out_pending[r] = 0;
    if (cudaStreamWaitEvent(ctx->stream, f->out_copied[r], 0) != cudaSuccess)
      return ctx->fail(CLG_ERR_CUDA, "export: wait for the copy");
  }
  for (int r = 0; r < (int)f->in_pending.size(); ++r) {
    if (!f->in_pending[r]) continue;
    const bool in_place = f->in_pending[r] == 2;
    f->in_pending[r] = 0;
    if (cudaStreamWaitEvent(ctx->stream, f->in_copied[r], 0) != cudaSuccess)
      return ctx->fail(CLG_ERR_CUDA, "import: wait for the copy");
    if (in_place) continue;
    double* slot = reinterpret_cast<double*>(static_cast<char*>(f->xin) + r * host_rhs_bytes(f));
    if (clg_status st = field_reorder(f, r, slot, 1)) return st;
    if (cudaEventRecord(f->in_consumed[r], ctx->stream) != cudaSuccess) return ctx->fail(CLG_ERR_CUDA, "import event");
  }
  return CLG_SUCCESS;
}

static clg_status staging_buffer(clg_context_s* ctx, size_t bytes, double** p) {
  if (bytes > ctx->staging_bytes) {
    if (ctx->staging) {
      cudaStreamSynchronize(ctx->stream);
      dfree(ctx->staging);
      ctx->staging = nullptr;
      ctx->staging_bytes = 0;
    }
    clg_status st = dalloc(ctx, &ctx->staging, bytes);
    if (st) return st;
    ctx->staging_bytes = bytes;
  }
  *p = static_cast<double*>(ctx->staging);
  return CLG_SUCCESS;
}

clg_status ensure_reduction(clg_context_s* ctx, int64_t doubles) {
  if (doubles <= ctx->red_capacity) return CLG_SUCCESS;
  if (stream_capturing(ctx->stream))
    return ctx->fail(CLG_ERR_BAD_ARG, "reduction scratch must be sized before stream capture");
  int64_t n = doubles < 65536 ? 65536 : doubles;
  if (ctx->red_partials) {
    cudaStreamSynchronize(ctx->stream);
    dfree(ctx->red_partials);
    ctx->red_partials = nullptr;
    ctx->red_capacity = 0;
  }
  clg_status st = dalloc(ctx, (void**)&ctx->red_partials, (size_t)n * sizeof(double));
  if (st) return st;
  ctx->red_capacity = n;
  return CLG_SUCCESS;
}

bool stream_capturing(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return cs != cudaStreamCaptureStatusNone;
}

// ------------------------------------------------------------------ operators
static double2 c2(double re, double im) { return make_double2(re, im); }
static double2 cmulh(double2 a, double2 b) { return c2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

static clg_status hop1(clg_context_s* ctx, const clg_gauge_s* U, int kind, bool dagger, int out_parity,
                       const FieldRef& in, const FieldRef& out, const FieldRef* x, double2 a, double2 xa, int nrhs,
                       const double* scale_dev, int scale_stride, const int* skip_dev, int skip_stride) {
  HopSpec s;
  s.kind = kind;
  s.prec = out.prec;
  s.dagger = dagger;
  s.out_parity = out_parity;
  s.in = in;
  s.out = out;
  s.x = x;
  s.a = a;
  s.xa = xa;
  s.scale_dev = scale_dev;
  s.scale_stride = scale_stride;
  s.skip_dev = skip_dev;
  s.skip_stride = skip_stride;
  s.nrhs = nrhs;
  return hop(ctx, U, s);
}

clg_status apply_op(clg_context_s* ctx, int op, const clg_gauge_s* U, int kind, double param, const FieldRef& out,
                    const FieldRef& in, const FieldRef* tmp, double2 coeff, int nrhs, const double* scale_dev,
                    int scale_stride, const int* skip_dev, int skip_stride) {
  const bool wilson = kind == CLG_FERMION_WILSON;
  const double2 one = c2(1, 0);
  clg_status st = CLG_SUCCESS;
  auto need_tmp = [&](int parity) -> bool { return tmp && tmp->has_parity(parity) && tmp->prec == out.prec; };
  switch (op) {
    case CLG_OP_D:
    case CLG_OP_DDAG: {
      if (out.nparity != 2 || in.nparity != 2) return ctx->fail(CLG_ERR_BAD_ARG, "D needs full fields");
      if (out.data == in.data) return ctx->fail(CLG_ERR_BAD_ARG, "D: in-place needs a temporary (use clg_apply)");
      const bool dag = op == CLG_OP_DDAG;
      // Wilson: out_p = in_p - kappa H in_(1-p); staggered: out_p = 2am in_p +/- H in_(1-p)
      const double2 a = wilson ? cmulh(coeff, c2(-param, 0)) : cmulh(coeff, c2(dag ? -1.0 : 1.0, 0));
      const double2 xa = wilson ? coeff : cmulh(coeff, c2(param, 0));
      for (int p = 0; p < 2; ++p) {
        FieldRef x = in;
        st = hop1(ctx, U, kind, dag && wilson, p, in, out, &x, a, xa, nrhs, scale_dev, scale_stride, skip_dev, skip_stride);
        if (st) return st;
      }
      return CLG_SUCCESS;
    }
    case CLG_OP_DDDAG:
    case CLG_OP_DD: {
      if (!tmp || tmp->nparity != 2) return ctx->fail(CLG_ERR_BAD_ARG, "DDdagger needs a full temporary");
      st = apply_op(ctx, op == CLG_OP_DDDAG ? CLG_OP_DDAG : CLG_OP_D, U, kind, param, *tmp, in, nullptr, one, nrhs,
                    nullptr, 0, skip_dev, skip_stride);
      if (st) return st;
      return apply_op(ctx, CLG_OP_D, U, kind, param, out, *tmp, nullptr, coeff, nrhs, scale_dev, scale_stride, skip_dev, skip_stride);
    }
    case CLG_OP_MEE:
    case CLG_OP_MEE_DAG:
    case CLG_OP_DDDAG_EE: {
      if (op == CLG_OP_DDDAG_EE && wilson) return ctx->fail(CLG_ERR_BAD_ARG, "DDDAG_EE is the staggered Schur operator");
      if (op != CLG_OP_DDDAG_EE && !wilson) return ctx->fail(CLG_ERR_BAD_ARG, "MEE is the Wilson Schur operator");
      if (!need_tmp(1)) return ctx->fail(CLG_ERR_BAD_ARG, "Schur operator needs an odd temporary");
      if (out.data == in.data) return ctx->fail(CLG_ERR_BAD_ARG, "Schur operator: in-place needs a temporary");
      const bool dag = op == CLG_OP_MEE_DAG;
      st = hop1(ctx, U, kind, dag, 1, in, *tmp, nullptr, one, c2(0, 0), nrhs, nullptr, 0, skip_dev, skip_stride);
      if (st) return st;
      // Wilson: out_e = in_e - kappa^2 H_eo tmp ; staggered: out_e = (2am)^2 in_e - H_eo tmp
      const double2 a = wilson ? cmulh(coeff, c2(-param * param, 0)) : cmulh(coeff, c2(-1.0, 0));
      const double2 xa = wilson ? coeff : cmulh(coeff, c2(param * param, 0));
      FieldRef x = in;
      return hop1(ctx, U, kind, dag, 0, *tmp, out, &x, a, xa, nrhs, scale_dev, scale_stride, skip_dev, skip_stride);
    }
    case CLG_OP_MEE_MEEDAG:
      return ctx->fail(CLG_ERR_BAD_ARG, "MEE_MEEDAG is composed by the caller with two temporaries");
    case CLG_OP_DEO:
    case CLG_OP_DOE: {
      const int p = op == CLG_OP_DEO ? 0 : 1;
      return hop1(ctx, U, kind, false, p, in, out, nullptr, coeff, c2(0, 0), nrhs, scale_dev, scale_stride, skip_dev, skip_stride);
    }
    default:
      return ctx->fail(CLG_ERR_BAD_ARG, "unknown operator");
  }
}

}  // namespace clg

using namespace clg;

// ================================================================== C ABI
namespace {

bool valid_prec(int p) { return p >= 0 && p <= 2; }

// scratch field with the shape of f (cached per context by shape key)
struct Scratch {
  void* data = nullptr;
  float* norm = nullptr;
  FieldRef ref;
};

clg_status make_like(clg_context_s* ctx, const clg_field_s* f, int nparity, int first_parity, Scratch& s) {
  const int64_t Vh = f->lat->g.Vh;
  const int64_t blk = Vh * site_bytes_of(f->prec, f->nc());
  clg_status st = dalloc(ctx, &s.data, (size_t)blk * nparity * f->nrhs);
  if (st) return st;
  if (f->prec == CLG_PREC_HALF) {
    st = dalloc(ctx, (void**)&s.norm, (size_t)Vh * nparity * f->nrhs * sizeof(float));
    if (st) {
      dfree(s.data);
      return st;
    }
  }
  s.ref.data = (char*)s.data;
  s.ref.norm = s.norm;
  s.ref.blk = blk;
  s.ref.rstride = blk * nparity;
  s.ref.nrstride = s.norm ? Vh * nparity : 0;
  s.ref.nparity = nparity;
  s.ref.first_parity = first_parity;
  s.ref.prec = f->prec;
  s.ref.nc = f->nc();
  s.ref.nrhs = f->nrhs;
  s.ref.Vh = Vh;
  return CLG_SUCCESS;
}
void free_scratch(Scratch& s) {
  dfree(s.data);
  dfree(s.norm);
  s.data = nullptr;
  s.norm = nullptr;
}

clg_status sync_status(clg_context_s* ctx) {
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), cudaGetErrorString(e));
  return CLG_SUCCESS;
}

// errors of the launches issued so far, without waiting for them
clg_status launch_status(clg_context_s* ctx) {
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), cudaGetErrorString(e));
  return CLG_SUCCESS;
}

}  // namespace

extern "C" {

const char* clg_status_string(clg_status s) {
  switch (s) {
    case CLG_SUCCESS: return "success";
    case CLG_ERR_BAD_ARG: return "bad argument";
    case CLG_ERR_CUDA: return "CUDA error";
    case CLG_ERR_OOM: return "out of device memory";
    case CLG_ERR_NOT_CONVERGED: return "solver did not converge";
    case CLG_ERR_BREAKDOWN: return "Krylov breakdown";
    case CLG_ERR_TIMEOUT: return "device wait timed out";
    case CLG_ERR_UNSUPPORTED: return "unsupported";
    case CLG_ERR_NO_DEVICE: return "no suitable CUDA device";
    default: return "unknown status";
  }
}

clg_status clg_context_create(int device, void* stream, clg_context* out) {
  if (!out) return CLG_ERR_BAD_ARG;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return CLG_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) return CLG_ERR_BAD_ARG;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return CLG_ERR_CUDA;
  if (prop.major < 10) return CLG_ERR_NO_DEVICE;  // the kernels are built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return CLG_ERR_CUDA;
  clg_context_s* ctx = new clg_context_s();
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  ctx->max_window = prop.accessPolicyMaxWindowSize > 0 ? (size_t)prop.accessPolicyMaxWindowSize : 0;
  ctx->max_persist = prop.persistingL2CacheMaxSize > 0 ? (size_t)prop.persistingL2CacheMaxSize : 0;
  ctx->l2_bytes = prop.l2CacheSize > 0 ? (size_t)prop.l2CacheSize : 0;
  if (const char* t = std::getenv("CLG_L2_WINDOW")) ctx->l2_window = t[0] != '0';
  if (const char* t = std::getenv("CLG_DEVICE_LOOP")) ctx->device_loops = t[0] == '1';
  if (const char* t = std::getenv("CLG_ZERO_COPY")) ctx->zero_copy = t[0] == '1';
  if (const char* t = std::getenv("CLG_XFER_BLOCKS")) ctx->xfer_blocks = std::max(1, std::min(4096, std::atoi(t)));
  // CLG_AUTOTUNE=0 keeps the default block size (reproducible profiling runs)
  if (const char* t = std::getenv("CLG_AUTOTUNE")) ctx->tuning_enabled = t[0] != '0';
  if (const char* t = std::getenv("CLG_FUSED_CG")) ctx->fused_cg = t[0] != '0';
  if (const char* t = std::getenv("CLG_FUSED_RESID")) ctx->fused_resid = t[0] != '0';
  if (const char* t = std::getenv("CLG_HOP_PAIR")) {
    int variant = -1, bs = 0;
    if (std::sscanf(t, "%d:%d", &variant, &bs) == 2 && (variant == 0 || variant == 1) &&
        (bs == 64 || bs == 128 || bs == 256)) {
      ctx->hop_pair_mode = 1;
      ctx->hop_pair_config = bs | (variant << 16);
    } else {
      ctx->hop_pair_mode = t[0] == '1' ? 1 : (t[0] == '0' ? 0 : 2);
    }
  }
  if (const char* t = std::getenv("CLG_HOP_TILE")) {
    int warps = 0, variant = -1;
    if (std::sscanf(t, "%d:%d", &warps, &variant) == 2 && warps >= 1 && warps <= 8 && variant >= 0 &&
        (variant <= 3 || (variant <= 7 && warps <= 4))) {
      ctx->hop_pair_mode = 3;
      ctx->hop_tile_config = (32 * warps) | ((16 + variant) << 16);
    } else if (std::sscanf(t, "%d:%d", &warps, &variant) == 2 && warps == 8 && variant >= 8 && variant <= 11) {
      ctx->hop_pair_mode = 3;
      ctx->hop_tile_config = 256 | ((24 + variant - 8) << 16);
    }
  }
  if (const char* t = std::getenv("CLG_HOP_MMA")) ctx->hop_mma = t[0] != '0';
  // CLG_TUNE_FILE: the autotuner's choices ("<key>=<config>" lines) are read
  // from this file when the context is created and written back when it is
  // destroyed, so a later run (a profiler's, whose timings would mislead the
  // autotuner) launches exactly the kernels an earlier run chose
  if (const char* t = std::getenv("CLG_TUNE_FILE")) {
    ctx->tune_file = t;
    if (FILE* f = std::fopen(t, "r")) {
      char line[512];
      while (std::fgets(line, sizeof line, f)) {
        char* eq = std::strrchr(line, '=');
        if (!eq) continue;
        *eq = 0;
        ctx->tuned[line] = std::atoi(eq + 1);
      }
      std::fclose(f);
    }
  }
  if (const char* t = std::getenv("CLG_PDL")) ctx->pdl = t[0] != '0';
  if (const char* t = std::getenv("CLG_HOP_CONFIG")) {
    int variant = -1, bs = 0;
    if (std::sscanf(t, "%d:%d", &variant, &bs) == 2 && variant >= 0 && variant <= 3 &&
        (bs == 64 || bs == 128 || bs == 256))
      ctx->hop_config = bs | (variant << 16);
    // the FP64 / FP32 tile form: variants 16..19, 32 x (1..8) threads
    else if (std::sscanf(t, "%d:%d", &variant, &bs) == 2 && variant >= 16 && variant <= 19 && bs >= 32 &&
             bs <= 256 && bs % 32 == 0)
      ctx->hop_config = bs | (variant << 16);
  }
  if (stream) {
    ctx->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete ctx;
      return CLG_ERR_CUDA;
    }
    ctx->own_stream = true;
  }
  if (dalloc(ctx, (void**)&ctx->red_counter, sizeof(unsigned) * (1 + kRedGroups)) ||
      cudaMemset(ctx->red_counter, 0, sizeof(unsigned) * (1 + kRedGroups)) != cudaSuccess ||
      ensure_reduction(ctx, 65536)) {
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    dfree(ctx->red_counter);
    delete ctx;
    return CLG_ERR_OOM;
  }
  if (clg_status st = noalloc_prepare(ctx)) {
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    dfree(ctx->red_partials);
    dfree(ctx->red_counter);
    delete ctx;
    return st;
  }
  *out = ctx;
  return CLG_SUCCESS;
}

clg_status clg_context_destroy(clg_context ctx) {
  if (!ctx) return CLG_ERR_BAD_ARG;
  cudaStreamSynchronize(ctx->stream);
  if (!ctx->tune_file.empty()) {
    if (FILE* f = std::fopen(ctx->tune_file.c_str(), "w")) {
      for (const auto& kv : ctx->tuned) std::fprintf(f, "%s=%d\n", kv.first.c_str(), kv.second);
      std::fclose(f);
    }
  }
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  if (ctx->persist_set) {  // give the persisting L2 carve-out back
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
    cudaGetLastError();
  }
  dfree(ctx->red_partials);
  dfree(ctx->red_counter);
  dfree(ctx->staging);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return CLG_SUCCESS;
}

clg_status clg_context_set_stream(clg_context ctx, void* stream) {
  if (!ctx) return CLG_ERR_BAD_ARG;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  ctx->own_stream = false;
  if (stream) {
    ctx->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return CLG_ERR_CUDA;
    ctx->own_stream = true;
  }
  return CLG_SUCCESS;
}

clg_status clg_context_synchronize(clg_context ctx) {
  if (!ctx) return CLG_ERR_BAD_ARG;
  return sync_status(ctx);
}

const char* clg_last_error(clg_context ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

clg_status clg_context_kernel_count(clg_context ctx, int64_t* count) {
  if (!ctx || !count) return CLG_ERR_BAD_ARG;
  *count = ctx->kernels;
  return CLG_SUCCESS;
}

clg_status clg_context_tuned(clg_context ctx, char* buf, size_t len, size_t* needed) {
  if (!ctx || !needed || (len && !buf)) return CLG_ERR_BAD_ARG;
  std::string out;
  for (const auto& kv : ctx->tuned) out += kv.first + "=" + std::to_string(kv.second) + "\n";
  *needed = out.size();
  if (len) {
    const size_t n = std::min(len - 1, out.size());
    std::memcpy(buf, out.data(), n);
    buf[n] = 0;
  }
  return CLG_SUCCESS;
}

clg_status clg_lattice_create(clg_context ctx, const int dims[4], const int bc[4], clg_lattice* out) {
  if (!ctx || !dims || !out) return CLG_ERR_BAD_ARG;
  *out = nullptr;
  clg_lattice_s* lat = new clg_lattice_s();
  lat->ctx = ctx;
  int64_t V = 1;
  for (int k = 0; k < 4; ++k) {
    if (dims[k] < 2 || (dims[k] & 1)) {
      delete lat;
      // odd extents break the even-odd split (Docs/SparseLinearAlgebra/evenodd.tex:52)
      return ctx->fail(CLG_ERR_UNSUPPORTED, "lattice extents must be even and >= 2");
    }
    lat->g.L[k] = dims[k];
    lat->g.dL[k].set((unsigned)dims[k]);
    lat->g.bc[k] = bc ? (bc[k] < 0 ? -1 : 1) : (k == 3 ? -1 : 1);
    V *= dims[k];
  }
  if (V >= ((int64_t)1 << 31)) {
    delete lat;
    return ctx->fail(CLG_ERR_UNSUPPORTED, "lattice volume must be below 2^31 sites (32-bit site indices)");
  }
  lat->g.V = V;
  lat->g.Vh = V / 2;
  *out = lat;
  return CLG_SUCCESS;
}

clg_status clg_lattice_destroy(clg_lattice lat) {
  if (!lat) return CLG_ERR_BAD_ARG;
  delete lat;
  return CLG_SUCCESS;
}

// ------------------------------------------------------------------ gauge
clg_status clg_gauge_create(clg_lattice lat, clg_gauge* out) {
  if (!lat || !out) return CLG_ERR_BAD_ARG;
  *out = nullptr;
  clg_context_s* ctx = lat->ctx;
  clg_gauge_s* g = new clg_gauge_s();
  g->lat = lat;
  const size_t bytes = (size_t)lat->g.Vh * 4 * 9 * sizeof(double2);
  for (int p = 0; p < 2; ++p) {
    clg_status st = dalloc(ctx, &g->u64[p], bytes);
    if (st) {
      dfree(g->u64[0]);
      delete g;
      return st;
    }
  }
  clg_status st = gauge_generate(g, CLG_GAUGE_IDENTITY, 0, 0, 0.0);
  if (st) return st;
  g->su3 = true;
  g->unitarity = 0.0;
  *out = g;
  return CLG_SUCCESS;
}

clg_status clg_gauge_destroy(clg_gauge g) {
  if (!g) return CLG_ERR_BAD_ARG;
  cudaStreamSynchronize(g->lat->ctx->stream);
  for (int p = 0; p < 2; ++p) dfree(g->u64[p]);
  dfree(g->u32[0]);  // one allocation holds both parities of a low-precision copy
  dfree(g->u16[0]);
  delete g;
  return CLG_SUCCESS;
}

static clg_status refresh_unitarity(clg_gauge_s* g) {
  double u = 0;
  clg_status st = gauge_unitarity(g, &u);
  if (st) return st;
  g->unitarity = u;
  g->su3 = u < 1e-12;
  g->dirty_lowp = true;
  return CLG_SUCCESS;
}

clg_status clg_gauge_import(clg_gauge g, const double* data, int layout, int on_device) {
  if (!g || !data || (layout != CLG_LAYOUT_CLGBIN && layout != CLG_LAYOUT_BRIDGEPP)) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = g->lat->ctx;
  const size_t bytes = (size_t)g->lat->g.V * 4 * 18 * sizeof(double);
  double* buf = nullptr;
  clg_status st = dalloc(ctx, (void**)&buf, bytes);
  if (st) return st;
  cudaError_t e = cudaMemcpyAsync(buf, data, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  ctx->stream);
  if (e != cudaSuccess) st = ctx->fail(cuda_status(e), cudaGetErrorString(e));
  if (!st) st = gauge_reorder(g, buf, layout, 1);
  if (!st) st = sync_status(ctx);
  dfree(buf);
  if (!st) st = refresh_unitarity(g);
  return st;
}

clg_status clg_gauge_export(clg_gauge g, double* data, int on_device) {
  if (!g || !data) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = g->lat->ctx;
  const size_t bytes = (size_t)g->lat->g.V * 4 * 18 * sizeof(double);
  double* buf = nullptr;
  clg_status st = dalloc(ctx, (void**)&buf, bytes);
  if (st) return st;
  st = gauge_reorder(g, buf, CLG_LAYOUT_CLGBIN, 0);
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(data, buf, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    ctx->stream);
    if (e != cudaSuccess) st = ctx->fail(cuda_status(e), cudaGetErrorString(e));
  }
  if (!st) st = sync_status(ctx);
  dfree(buf);
  return st;
}

clg_status clg_gauge_random(clg_gauge g, int init, uint64_t seed, uint32_t field_id, double eps) {
  if (!g || init < 0 || init > CLG_GAUGE_ZERO) return CLG_ERR_BAD_ARG;
  clg_status st = gauge_generate(g, init, seed, field_id, eps);
  if (!st) st = refresh_unitarity(g);
  return st;
}

clg_status clg_gauge_plaquette(clg_gauge g, double* out) {
  if (!g || !out) return CLG_ERR_BAD_ARG;
  return gauge_plaquette(g, out);
}

clg_status clg_gauge_unitarity(clg_gauge g, double* out) {
  if (!g || !out) return CLG_ERR_BAD_ARG;
  clg_status st = refresh_unitarity(g);
  if (!st) *out = g->unitarity;
  return st;
}

// ------------------------------------------------------------------ fields
clg_status clg_field_create(clg_lattice lat, int kind, int subset, int precision, int nrhs, double param,
                            clg_field* out) {
  if (!lat || !out || (kind != CLG_FERMION_WILSON && kind != CLG_FERMION_STAGGERED) ||
      (subset != CLG_SUBSET_FULL && subset != CLG_SUBSET_EVEN) || !valid_prec(precision) || nrhs < 1 || nrhs > 4096)
    return CLG_ERR_BAD_ARG;
  *out = nullptr;
  clg_context_s* ctx = lat->ctx;
  clg_field_s* f = new clg_field_s();
  f->lat = lat;
  f->kind = kind;
  f->subset = subset;
  f->prec = precision;
  f->nrhs = nrhs;
  f->param = param;
  f->blk = lat->g.Vh * site_bytes_of(precision, f->nc());
  clg_status st = dalloc(ctx, (void**)&f->data, (size_t)f->blk * f->nparity() * nrhs);
  if (!st && precision == CLG_PREC_HALF)
    st = dalloc(ctx, (void**)&f->norm, (size_t)lat->g.Vh * f->nparity() * nrhs * sizeof(float));
  if (!st) st = blas_zero(ctx, f->ref());
  if (st) {
    dfree(f->data);
    dfree(f->norm);
    delete f;
    return st;
  }
  *out = f;
  return CLG_SUCCESS;
}

clg_status clg_field_destroy(clg_field f) {
  if (!f) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = f->lat->ctx;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  for (auto* v : {&f->in_copied, &f->in_consumed, &f->out_ready, &f->out_copied})
    for (cudaEvent_t e : *v)
      if (e) cudaEventDestroy(e);
  dfree(f->xin);
  dfree(f->xout);
  dfree(f->data);
  dfree(f->norm);
  delete f;
  return CLG_SUCCESS;
}

clg_status clg_field_set_param(clg_field f, double param) {
  if (!f) return CLG_ERR_BAD_ARG;
  f->param = param;
  return CLG_SUCCESS;
}

clg_status clg_field_import(clg_field f, int rhs, const double* data, int on_device) {
  if (!f || !data || rhs < 0 || rhs >= f->nrhs) return CLG_ERR_BAD_ARG;
  if (clg_status st = settle(f)) return st;
  clg_context_s* ctx = f->lat->ctx;
  const size_t bytes = (size_t)f->lat->g.V * f->nc() * 2 * sizeof(double);
  double* buf = nullptr;
  clg_status st = CLG_SUCCESS;
  if (on_device) {
    buf = const_cast<double*>(data);
  } else {
    st = staging_buffer(ctx, bytes, &buf);
    if (st) return st;
    cudaError_t e = cudaMemcpyAsync(buf, data, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) st = ctx->fail(cuda_status(e), cudaGetErrorString(e));
  }
  if (!st) st = field_reorder(f, rhs, buf, 1);
  // the caller may reuse or free its buffer once this returns
  if (!st) st = sync_status(ctx);
  return st;
}

clg_status clg_field_export(clg_field f, int rhs, double* data, int on_device) {
  if (!f || !data || rhs < 0 || rhs >= f->nrhs) return CLG_ERR_BAD_ARG;
  if (clg_status st = settle(f)) return st;
  clg_context_s* ctx = f->lat->ctx;
  const size_t bytes = (size_t)f->lat->g.V * f->nc() * 2 * sizeof(double);
  double* buf = nullptr;
  clg_status st = CLG_SUCCESS;
  if (on_device) {
    buf = data;
  } else {
    st = staging_buffer(ctx, bytes, &buf);
    if (st) return st;
  }
  st = field_reorder(f, rhs, buf, 0);
  if (!on_device && !st) {
    cudaError_t e = cudaMemcpyAsync(data, buf, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) st = ctx->fail(cuda_status(e), cudaGetErrorString(e));
  }
  // the data is complete (and readable from any stream) once this returns
  if (!st) st = sync_status(ctx);
  return st;
}

clg_status clg_field_random(clg_field f, int rhs, int kind, uint64_t seed, uint32_t field_id, int64_t site, int comp) {
  if (!f || rhs < 0 || rhs >= f->nrhs || kind < 0 || kind > CLG_SOURCE_Z4) return CLG_ERR_BAD_ARG;
  if (kind == CLG_SOURCE_POINT && (site < 0 || site >= f->lat->g.V || comp < 0 || comp >= f->nc())) return CLG_ERR_BAD_ARG;
  if (clg_status st = settle(f)) return st;
  return field_source(f, rhs, kind, seed, field_id, site, comp);
}

clg_status clg_field_import_async(clg_field f, int rhs, const double* data) {
  if (!f || !data || rhs < 0 || rhs >= f->nrhs) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = f->lat->ctx;
  double* direct = mapped_host(f, data);
  if (clg_status st = xfer_prepare(f, true, !direct)) return st;
  if (direct) {
    // the field is rewritten on the copy stream once the work queued on the
    // context stream so far (which may read or write it) has finished
    if (clg_status st = settle(f)) return st;
    cudaError_t e = cudaEventRecord(f->in_consumed[rhs], ctx->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_stream, f->in_consumed[rhs], 0);
    if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("import_async: ") + cudaGetErrorString(e));
    if (clg_status st = field_stream(f, rhs, direct, 1, ctx->copy_stream)) return st;
    e = cudaEventRecord(f->in_copied[rhs], ctx->copy_stream);
    if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("import_async: ") + cudaGetErrorString(e));
    f->in_pending[rhs] = 2;
    return CLG_SUCCESS;
  }
  const size_t bytes = host_rhs_bytes(f);
  char* slot = static_cast<char*>(f->xin) + rhs * bytes;
  // the slot is overwritten only after the last reorder out of it
  cudaError_t e = cudaStreamWaitEvent(ctx->copy_stream, f->in_consumed[rhs], 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(slot, data, bytes, cudaMemcpyHostToDevice, ctx->copy_stream);
  if (e == cudaSuccess) e = cudaEventRecord(f->in_copied[rhs], ctx->copy_stream);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("import_async: ") + cudaGetErrorString(e));
  f->in_pending[rhs] = 1;
  return CLG_SUCCESS;
}

clg_status clg_field_export_async(clg_field f, int rhs, double* data) {
  if (!f || !data || rhs < 0 || rhs >= f->nrhs) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = f->lat->ctx;
  if (clg_status st = settle(f)) return st;
  double* direct = mapped_host(f, data);
  if (clg_status st = xfer_prepare(f, false, !direct)) return st;
  if (direct) {
    // read on the copy stream after the work queued so far; later work on the
    // field waits for the read (settle)
    cudaError_t e = cudaEventRecord(f->out_ready[rhs], ctx->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_stream, f->out_ready[rhs], 0);
    if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("export_async: ") + cudaGetErrorString(e));
    if (clg_status st = field_stream(f, rhs, direct, 0, ctx->copy_stream)) return st;
    e = cudaEventRecord(f->out_copied[rhs], ctx->copy_stream);
    if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("export_async: ") + cudaGetErrorString(e));
    f->out_pending[rhs] = 1;
    return CLG_SUCCESS;
  }
  const size_t bytes = host_rhs_bytes(f);
  double* slot = reinterpret_cast<double*>(static_cast<char*>(f->xout) + rhs * bytes);
  // the slot is refilled only after its last copy to the host
  cudaError_t e = cudaStreamWaitEvent(ctx->stream, f->out_copied[rhs], 0);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), "export_async: wait");
  if (clg_status st = field_reorder(f, rhs, slot, 0)) return st;
  e = cudaEventRecord(f->out_ready[rhs], ctx->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_stream, f->out_ready[rhs], 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(data, slot, bytes, cudaMemcpyDeviceToHost, ctx->copy_stream);
  if (e == cudaSuccess) e = cudaEventRecord(f->out_copied[rhs], ctx->copy_stream);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("export_async: ") + cudaGetErrorString(e));
  return CLG_SUCCESS;
}

clg_status clg_field_wait(clg_field f) {
  if (!f) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = f->lat->ctx;
  for (auto* v : {&f->in_copied, &f->out_copied})
    for (cudaEvent_t ev : *v) {
      const cudaError_t e = cudaEventSynchronize(ev);
      if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("field wait: ") + cudaGetErrorString(e));
    }
  return CLG_SUCCESS;
}

clg_status clg_field_copy(clg_field dst, clg_field src) {
  if (!dst || !src || dst->lat != src->lat || dst->kind != src->kind || dst->subset != src->subset ||
      dst->nrhs != src->nrhs)
    return CLG_ERR_BAD_ARG;
  if (clg_status st = settle(dst)) return st;
  if (clg_status st = settle(src)) return st;
  return blas_copy(dst->lat->ctx, dst->ref(), src->ref());
}

// ------------------------------------------------------------------ operators
static clg_status check_pair(const clg_field_s* out, const clg_field_s* in, const clg_gauge_s* g) {
  if (!out || !in || !g) return CLG_ERR_BAD_ARG;
  if (out->lat != in->lat || g->lat != in->lat || out->kind != in->kind || out->prec != in->prec ||
      out->nrhs != in->nrhs)
    return CLG_ERR_BAD_ARG;
  return CLG_SUCCESS;
}

static double2 coeff_of(int ct, double re, double im) {
  switch (ct) {
    case CLG_COEFF_MINUS: return make_double2(-1, 0);
    case CLG_COEFF_REAL: return make_double2(re, 0);
    case CLG_COEFF_COMPLEX: return make_double2(re, im);
    default: return make_double2(1, 0);
  }
}

static bool op_on_even(int op) { return op == CLG_OP_MEE || op == CLG_OP_MEE_DAG || op == CLG_OP_MEE_MEEDAG || op == CLG_OP_DDDAG_EE; }

clg_status clg_apply_to(int op, clg_field out, clg_field in, clg_gauge g, int coeff_type, double cre, double cim) {
  clg_status st = check_pair(out, in, g);
  if (st) return st;
  if ((st = settle(out)) || (st = settle(in))) return st;
  clg_context_s* ctx = in->lat->ctx;
  if (op < 0 || op > CLG_OP_DDDAG_EE) return ctx->fail(CLG_ERR_BAD_ARG, "unknown operator");
  if (op_on_even(op)) {
    if (in->subset != CLG_SUBSET_EVEN || out->subset != CLG_SUBSET_EVEN)
      return ctx->fail(CLG_ERR_BAD_ARG, "Schur operators act on EVEN fields");
  } else if (op == CLG_OP_DEO || op == CLG_OP_DOE) {
    if (in->subset != CLG_SUBSET_FULL || out->subset != CLG_SUBSET_FULL)
      return ctx->fail(CLG_ERR_BAD_ARG, "hopping blocks act on FULL fields");
  } else if (in->subset != CLG_SUBSET_FULL || out->subset != CLG_SUBSET_FULL) {
    return ctx->fail(CLG_ERR_BAD_ARG, "D / D^+ act on FULL fields");
  }
  st = gauge_prepare(g, in->prec);
  if (st) return st;
  const double2 coeff = coeff_of(coeff_type, cre, cim);
  Scratch t1, t2;
  FieldRef o = out->ref(), i = in->ref();
  const bool alias = out->data == in->data;
  if (alias) {
    st = make_like(ctx, in, in->nparity(), 0, t2);
    if (st) return st;
    st = blas_copy(ctx, t2.ref, i);
    i = t2.ref;
  }
  if (!st) {
    if (op == CLG_OP_DDDAG || op == CLG_OP_DD) {
      st = make_like(ctx, in, 2, 0, t1);
      if (!st) st = apply_op(ctx, op, g, in->kind, in->param, o, i, &t1.ref, coeff, in->nrhs);
    } else if (op_on_even(op)) {
      st = make_like(ctx, in, 1, 1, t1);
      if (!st) {
        if (op == CLG_OP_MEE_MEEDAG) {
          Scratch t3;
          st = make_like(ctx, in, 1, 0, t3);
          if (!st) st = apply_op(ctx, CLG_OP_MEE_DAG, g, in->kind, in->param, t3.ref, i, &t1.ref, make_double2(1, 0), in->nrhs);
          if (!st) st = apply_op(ctx, CLG_OP_MEE, g, in->kind, in->param, o, t3.ref, &t1.ref, coeff, in->nrhs);
          if (!st) st = sync_status(ctx);
          free_scratch(t3);
        } else {
          st = apply_op(ctx, op, g, in->kind, in->param, o, i, &t1.ref, coeff, in->nrhs);
        }
      }
    } else if (op == CLG_OP_DEO || op == CLG_OP_DOE) {
      // the other checkerboard of out is left unchanged
      st = apply_op(ctx, op, g, in->kind, in->param, o, i, nullptr, coeff, in->nrhs);
    } else {
      st = apply_op(ctx, op, g, in->kind, in->param, o, i, nullptr, coeff, in->nrhs);
    }
  }
  // Operators that needed scratch fields wait for their kernels before the
  // scratch is released; the others return once launched, like any stream
  // operation, and can be captured into a CUDA graph.
  if (!st) st = (t1.data || t2.data) ? sync_status(ctx) : launch_status(ctx);
  free_scratch(t1);
  free_scratch(t2);
  return st;
}

clg_status clg_apply(int op, clg_field inout, clg_gauge g, int coeff_type, double cre, double cim) {
  return clg_apply_to(op, inout, inout, g, coeff_type, cre, cim);
}

// ------------------------------------------------------------------ BLAS
static clg_status read_dev(clg_context_s* ctx, double* host, const double* dev, size_t n) {
  cudaError_t e = cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), cudaGetErrorString(e));
  return CLG_SUCCESS;
}

clg_status clg_dot(clg_field a, clg_field b, double* re_im) {
  if (!a || !b || !re_im || a->lat != b->lat || a->kind != b->kind || a->subset != b->subset || a->nrhs != b->nrhs ||
      a->prec != b->prec)
    return CLG_ERR_BAD_ARG;
  if (clg_status st = settle(a)) return st;
  if (clg_status st = settle(b)) return st;
  clg_context_s* ctx = a->lat->ctx;
  double* d = nullptr;
  clg_status st = dalloc(ctx, (void**)&d, sizeof(double) * 2 * a->nrhs);
  if (!st) st = blas_dot(ctx, a->ref(), b->ref(), d);
  if (!st) st = read_dev(ctx, re_im, d, 2 * a->nrhs);
  dfree(d);
  return st;
}

clg_status clg_norm2(clg_field a, double* out) {
  if (!a || !out) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = a->lat->ctx;
  double* d = nullptr;
  clg_status st = dalloc(ctx, (void**)&d, sizeof(double) * a->nrhs);
  if (!st) st = blas_norm2(ctx, a->ref(), d);
  if (!st) st = read_dev(ctx, out, d, a->nrhs);
  dfree(d);
  return st;
}

clg_status clg_axpy(clg_field y, double are, double aim, clg_field x) {
  if (!y || !x || y->lat != x->lat || y->kind != x->kind || y->subset != x->subset || y->nrhs != x->nrhs ||
      y->prec != x->prec)
    return CLG_ERR_BAD_ARG;
  clg_status st = settle(y);
  if (!st) st = settle(x);
  if (st) return st;
  st = blas_axpby(y->lat->ctx, y->ref(), make_double2(are, aim), x->ref(), make_double2(1, 0));
  return st ? st : sync_status(y->lat->ctx);
}

clg_status clg_scale(clg_field y, double are, double aim) {
  if (!y) return CLG_ERR_BAD_ARG;
  clg_status st = settle(y);
  if (!st) st = blas_axpby(y->lat->ctx, y->ref(), make_double2(0, 0), y->ref(), make_double2(are, aim));
  return st ? st : sync_status(y->lat->ctx);
}

clg_status clg_zero(clg_field y) {
  if (!y) return CLG_ERR_BAD_ARG;
  clg_status st = settle(y);
  if (!st) st = blas_zero(y->lat->ctx, y->ref());
  return st ? st : sync_status(y->lat->ctx);
}

}  // extern "C"
