// internal.h -- host-side object model behind the C ABI (include/clg_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/clg_b200.h"
#include "clg_common.cuh"

namespace clg {

clg_status cuda_status(cudaError_t e);

// A view of one field: (rhs, parity) block at data + rhs*rstride + (p-first_parity)*blk.
struct FieldRef {
  char* data = nullptr;
  float* norm = nullptr;   // FP16 per-site norms, same block structure in floats
  int64_t blk = 0;         // bytes of one parity block
  int64_t rstride = 0;     // bytes between right-hand sides
  int64_t nrstride = 0;    // floats between right-hand sides (norms)
  int nparity = 1;         // 2 = full field, 1 = single checkerboard
  int first_parity = 0;    // parity of block 0
  int prec = 0;
  int nc = 12;             // complex per site (12 Wilson, 3 staggered)
  int nrhs = 1;
  int64_t Vh = 0;
  __host__ __device__ char* base(int rhs, int p) const {
    return data + (int64_t)rhs * rstride + (int64_t)(p - first_parity) * blk;
  }
  __host__ __device__ float* nbase(int rhs, int p) const {
    return norm ? norm + (int64_t)rhs * nrstride + (int64_t)(p - first_parity) * Vh : nullptr;
  }
  bool has_parity(int p) const { return p >= first_parity && p < first_parity + nparity; }
  FieldRef parity_view(int p) const {
    FieldRef r = *this;
    r.data = data + (int64_t)(p - first_parity) * blk;
    r.norm = norm ? norm + (int64_t)(p - first_parity) * Vh : nullptr;
    r.first_parity = p;
    r.nparity = 1;
    return r;
  }
  FieldRef rhs_view(int r0, int n) const {
    FieldRef r = *this;
    r.data = data + (int64_t)r0 * rstride;
    r.norm = norm ? norm + (int64_t)r0 * nrstride : nullptr;
    r.nrhs = n;
    return r;
  }
};

int64_t site_bytes_of(int prec, int nc);

}  // namespace clg

struct clg_context_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string last_error;
  int num_sms = 148;
  int64_t kernels = 0;
  // reduction scratch (device): partial sums and the arrival counter
  // reduction scratch: block partials (and the group totals of the two-level
  // reductions) in red_partials; red_counter[0] is the grid ticket, and
  // red_counter[1 .. kRedGroups] the group tickets (grid_reduce_finalize2)
  double* red_partials = nullptr;
  int64_t red_capacity = 0;  // doubles
  unsigned int* red_counter = nullptr;
  // device staging buffer of host field imports/exports (grow-only; one FP64
  // lexicographic field).  Kept across calls so that a host round trip costs
  // two copies and a reorder, not a cudaMalloc/cudaFree pair.
  void* staging = nullptr;
  size_t staging_bytes = 0;
  // stream of the asynchronous host transfers (created on first use)
  cudaStream_t copy_stream = nullptr;
  // CLG_ZERO_COPY=1: asynchronous transfers of FP64 fields from/to pinned
  // host memory are made by CLG_XFER_BLOCKS blocks on the copy stream reading
  // or writing the host buffer directly, instead of a copy engine into a
  // device slot plus a reorder.  Off by default: beside a 32^3x16 solve (13.8
  // ms) the two 100 MB transfers per solve cost 0.85 ms with 8 blocks, 1.6 ms
  // with 16 (the blocks take SM room from the solve), 0.8 ms by copy engine
  bool zero_copy = false;
  int xfer_blocks = 8;
  // block size chosen per kernel variant by the autotuner
  std::map<std::string, int> tuned;
  bool tuning_enabled = true;
  // CLG_HOP_CONFIG="<variant>:<block>" pins the Wilson hop launch (variant 3: FP64 capped at 128;
  // 0 plain, 1 register-capped; block 64, 128 or 256); -1 lets the autotuner choose
  int hop_config = -1;
  // CG on the Wilson normal equations fuses its vector work into the Schur
  // hops, and multi-shift CG on the staggered (DD^+)_ee its (p, A p) (FP64 /
  // FP32 iterations); CLG_FUSED_CG=0 runs the separate kernels instead
  bool fused_cg = true;
  // the outer residual r = b - D x of Wilson solves fused into the FP64 hop
  // (with |r|^2 and the inner-precision copy); CLG_FUSED_RESID=0: separate passes
  bool fused_resid = true;
  // FP16 Wilson hops over two or more right-hand sides: one right-hand side
  // per thread (the right-hand sides interleaved over the blocks, links shared
  // through L2), two per thread (wilson_hop_pair_kernel: one link load and
  // reconstruction per pair, planar half2 arithmetic) or a tile of 32 sites
  // for all right-hand sides (wilson_hop_tile16_kernel: links staged once per
  // tile in shared memory).  hop_pair_mode 2 (the default) lets the autotuner
  // time the three forms per operator and lattice (the right-hand-side-per-
  // thread and site-tiling axes); CLG_HOP_PAIR=0 keeps one, =1 forces two,
  // "<variant>:<block>" pins the paired launch (variant 0 uncapped, 1 capped at
  // 128 registers).  Measured on 32^3x16 / 32^3x32 the two are within a few
  // per cent (13.6 against 13.4 us per rhs at 8 rhs, 27.2 against 27.5 at 28).
  // CLG_HOP_TILE="<warps>:<variant>" forces the tile form (mode 3;
  // wilson_hop_tile16_kernel; variants 0-3: bit 0 capped at 80 registers, bit
  // 1 the blocked tile order; 4-7 (at most 4 warps): capped at 72, bit 0 at
  // 64 instead, bit 1 the blocked order);
  // the autotuner of mode 2 times it with the other two
  int hop_pair_mode = 2;
  int hop_tile_config = -1;
  // the tensor-core form of the FP16 hop (wilson_hop_mma16_kernel) among the
  // autotuner's candidates: CLG_HOP_MMA=1 (off by default: measured 1.91 ms
  // against 0.63 ms for the tile form on 28 rhs of 32^3x32, bound by the
  // latency of its three barrier-separated phases at 16 warps per SM).
  // CLG_HOP_TILE variants 8..11 force it (variant bit 0: two blocks per SM,
  // bit 1: the blocked tile order)
  bool hop_mma = false;
  std::string tune_file;  // CLG_TUNE_FILE (empty: none)
  // set by clg_solve_lattices for the duration of its solve: the per-rhs
  // checkerboard sizes (device) of the padded batch, whose site kernels skip
  // the padding (launches with this stride and right-hand-side count)
  const int64_t* batch_vh = nullptr;
  int64_t batch_vh_stride = 0;
  int batch_nrhs = 0;
  int hop_pair_config = -1;
  // hops and site kernels are launched with programmatic stream serialization
  // (they overlap the previous kernel's drain); CLG_PDL=0 launches them plainly
  bool pdl = true;
  // solves keep the low-precision link copy in a persisting L2 window
  // (CLG_L2_WINDOW=0 turns it off); device limits queried at creation
  bool l2_window = true;
  // CLG_DEVICE_LOOP=1: CG inner solves loop on the device (CUDA-graph WHILE
  // node) after their first chunk, instead of one host check per chunk.  Off
  // by default: on the 32^3x16 FP16-inner solve it measured no faster
  // (70.2 / 71.7 against 71.2 / 74.5 solves/s), the host checks being cheap
  bool device_loops = false;
  size_t max_window = 0, max_persist = 0, persist_set = 0, l2_bytes = 0;
  clg_status fail(clg_status s, const std::string& msg) {
    last_error = msg;
    return s;
  }
};

struct clg_lattice_s {
  clg_context_s* ctx = nullptr;
  clg::Geom g;
};

namespace clg {
struct HopSeg;     // dslash.cuh
struct BatchTile;  // dslash.cuh
}

struct clg_gauge_s {
  clg_lattice_s* lat = nullptr;
  // a batch of lattices (clg_solve_lattices): per right-hand side geometry and
  // link arrays on the device; lat is then the batch's padded virtual lattice
  const clg::HopSeg* seg = nullptr;
  const int64_t* seg_vh = nullptr;  // per right-hand side checkerboard sizes (device)
  // the batch's tiles of 32 sites per lattice (device; the tile-form hops)
  const clg::BatchTile* btile = nullptr;
  int nbtile = 0;
  int64_t btiles = 0;
  // per parity link arrays [mu][chunk][h]
  void* u64[2] = {nullptr, nullptr};   // FP64, 18 reals
  void* u32[2] = {nullptr, nullptr};   // FP32, 12 reals (SU(3)) or 18
  void* u16[2] = {nullptr, nullptr};   // FP16, 12 reals (SU(3) only)
  int recon32 = 12;
  bool su3 = false;
  bool dirty_lowp = true;  // low-precision copies need a rebuild
  double unitarity = -1.0;
};

struct clg_field_s {
  clg_lattice_s* lat = nullptr;
  int kind = CLG_FERMION_WILSON;
  int subset = CLG_SUBSET_FULL;
  int prec = CLG_PREC_DOUBLE;
  int nrhs = 1;
  double param = 0.0;
  char* data = nullptr;
  float* norm = nullptr;
  int64_t blk = 0;
  // asynchronous host transfers: FP64 lexicographic staging per rhs, and per
  // rhs the events that order the copy stream against the context stream
  void* xin = nullptr;                       // import staging (nrhs slots)
  void* xout = nullptr;                      // export staging (nrhs slots)
  std::vector<cudaEvent_t> in_copied;        // H2D of a slot finished (copy stream)
  std::vector<cudaEvent_t> in_consumed;      // reorder out of a slot finished (context stream)
  std::vector<cudaEvent_t> out_ready;        // reorder into a slot finished (context stream)
  std::vector<cudaEvent_t> out_copied;       // D2H of a slot finished (copy stream)
  std::vector<char> in_pending;              // 1: slot copied, not yet reordered; 2: written in place
  std::vector<char> out_pending;             // a zero-copy export may still be reading the field
  int nparity() const { return subset == CLG_SUBSET_FULL ? 2 : 1; }
  int nc() const { return kind == CLG_FERMION_WILSON ? 12 : 3; }
  clg::FieldRef ref() const {
    clg::FieldRef r;
    r.data = data;
    r.norm = norm;
    r.blk = blk;
    r.rstride = blk * nparity();
    r.nrstride = norm ? (int64_t)nparity() * lat->g.Vh : 0;
    r.nparity = nparity();
    r.first_parity = 0;
    r.prec = prec;
    r.nc = nc();
    r.nrhs = nrhs;
    r.Vh = lat->g.Vh;
    return r;
  }
};

namespace clg {

// Queue the pending asynchronous imports of f on the context stream (every
// entry point that takes a field calls it before using the field).
clg_status settle(clg_field_s* f);
// clg_dot_noalloc's one-time set-up on a new context's device (noalloc.cu)
clg_status noalloc_prepare(clg_context_s* ctx);

// ------------------------------------------------------------ device allocation
clg_status dalloc(clg_context_s* ctx, void** p, size_t bytes);
void dfree(void* p);
clg_status ensure_reduction(clg_context_s* ctx, int64_t doubles);
// Group tickets of the two-level reductions, and the group size for nunits x
// nslots blocks (at least 64 slots, doubled until the tickets fit)
constexpr int64_t kRedGroups = 65536;
inline unsigned red_group(int64_t nslots, int64_t nunits) {
  int64_t g = 64;
  while (((nslots + g - 1) / g) * nunits > kRedGroups) g *= 2;
  return (unsigned)g;
}
// scratch doubles of a two-level reduction: block partials then group totals
inline int64_t red2_doubles(int64_t nslots, int nrhs, int nunits, int nred) {
  const int64_t ng = (nslots + red_group(nslots, nunits) - 1) / red_group(nslots, nunits);
  return (nslots + ng) * nrhs * nred;
}

// ------------------------------------------------------------ launch helpers
bool stream_capturing(cudaStream_t s);

// Launch a kernel that follows the pdl_launch_dependents / pdl_wait protocol
// (clg_common.cuh) on the context stream, with programmatic stream
// serialization when the context allows it.  Counts the launch.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(clg_context_s* ctx, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       Args&&... args) {
  ctx->kernels++;
  if (!ctx->pdl) {
    kernel<<<grid, block, smem, ctx->stream>>>(std::forward<Args>(args)...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
// Opt kernel fn into `bytes` of dynamic shared memory (above the 48 KB
// default), once per kernel and device.
inline cudaError_t opt_in_smem(const void* fn, size_t bytes) {
  static std::mutex m;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  if (cudaError_t e = cudaGetDevice(&dev)) return e;
  std::lock_guard<std::mutex> lk(m);
  auto it = done.find({fn, dev});
  if (it != done.end() && it->second >= bytes) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done[{fn, dev}] = bytes;
  return e;
}

// Autotuner: the launch configuration for kernel variant `key`.  On first use
// (outside stream capture, when the launch is idempotent) each candidate
// (a block size, optionally combined with a register-capped kernel variant) is
// timed with CUDA events on the context stream and the fastest is cached.
template <class Go>
int tune_block(clg_context_s* ctx, const std::string& key, bool can_repeat, Go&& go,
               const std::vector<int>& cand = {64, 128, 256, 512}, int fallback = 128,
               std::map<int, float>* times = nullptr) {
  auto it = ctx->tuned.find(key);
  if (it != ctx->tuned.end()) return it->second;
  if (!ctx->tuning_enabled || !can_repeat || stream_capturing(ctx->stream)) return fallback;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return fallback;
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return fallback; }
  int best = fallback;
  float best_ms = 1e30f;
  for (int bs : cand) {
    if (go(bs) != cudaSuccess) continue;  // warm-up / validity
    cudaEventRecord(e0, ctx->stream);
    for (int r = 0; r < 3; ++r) go(bs);
    cudaEventRecord(e1, ctx->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (times) (*times)[bs] = ms;
    if (ms < best_ms) { best_ms = ms; best = bs; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
  ctx->tuned[key] = best;
  return best;
}

// ------------------------------------------------------------ operators (dslash.cu)
// A single checkerboard hop:  out_p = xa * x_p + a * H in_(1-p)  [ * scale_dev[rhs] ]
struct HopSpec {
  int kind;        // CLG_FERMION_WILSON / STAGGERED
  int prec;
  bool dagger;     // Wilson H^+ (ignored for staggered: the sign is in `a`)
  int out_parity;
  FieldRef in;     // must hold parity 1-out_parity
  FieldRef out;    // must hold out_parity
  const FieldRef* x;  // nullable, must hold out_parity
  double2 a, xa;
  const double* scale_dev;
  int scale_stride;
  const int* skip_dev;
  int skip_stride;
  int nrhs;
};
clg_status hop(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s);
// the kernel arguments of a hop (checked as hop() checks them), for callers
// that launch a fused variant themselves
struct HopArgs;
clg_status make_hop_args(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, HopArgs& a);
// block size the autotuner chose for this hop (fallback if not tuned yet)
int tuned_hop_block(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, int fallback);
// the tuned launch configuration (block | variant << 16) of the paired FP16 hop
int tuned_hop_pair_config(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, int fallback);
// the autotuner's configuration (block | variant << 16) of this hop (FP64 /
// FP32: variants from 16 on are the tile form)
int tuned_hop_config(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, int fallback);
// the tile form's configuration (block | variant << 16), when the tile form is
// forced or was the autotuner's choice for this hop
int tuned_hop_tile_config(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, int fallback);
clg_status gauge_prepare(clg_gauge_s* U, int prec);  // builds the FP32 / FP16 copies on first use
// address range of the link copy the hops of precision `prec` read (nullptr, 0 if none)
void gauge_link_range(const clg_gauge_s* U, int prec, const void** base, size_t* bytes);

// While alive, the link copy of precision `prec` is a persisting L2 access
// window on the context stream (kernels and captured graph nodes launched on
// it keep those lines resident), so streaming traffic -- the solve's own
// vectors, or copy-engine transfers of neighbouring steps -- does not evict
// the links every hop reads.
struct L2LinkWindow {
  clg_context_s* ctx;
  bool set = false;
  L2LinkWindow(clg_context_s* c, const clg_gauge_s* U, int prec);
  ~L2LinkWindow();
};

// ------------------------------------------------------------ operator composition (api.cu)
// out = coeff * op(in) on fields of one precision. tmp: scratch with at least
// the parity the operator needs (nullable: allocated internally).
clg_status apply_op(clg_context_s* ctx, int op, const clg_gauge_s* U, int kind, double param,
                    const FieldRef& out, const FieldRef& in, const FieldRef* tmp, double2 coeff, int nrhs,
                    const double* scale_dev = nullptr, int scale_stride = 0, const int* skip_dev = nullptr,
                    int skip_stride = 1);

// ------------------------------------------------------------ BLAS (blas.cu)
clg_status blas_dot(clg_context_s* ctx, const FieldRef& a, const FieldRef& b, double* dev_out);  // 2*nrhs doubles
clg_status blas_norm2(clg_context_s* ctx, const FieldRef& a, double* dev_out);                    // nrhs doubles
clg_status blas_axpby(clg_context_s* ctx, const FieldRef& y, double2 a, const FieldRef& x, double2 b);  // y = a x + b y
clg_status blas_copy(clg_context_s* ctx, const FieldRef& dst, const FieldRef& src);               // converts precision
clg_status blas_zero(clg_context_s* ctx, const FieldRef& y);
// dst <- src for FP64 fields that differ only in their chunk stride Vh: the
// first min(Vh) sites of every parity block (a lattice inside a padded batch)
clg_status blas_copy_strided(clg_context_s* ctx, const FieldRef& dst, const FieldRef& src);

// ------------------------------------------------------------ solves (solvers.cu)
// Workspace a solver keeps between calls (buffers, pinned host memory, captured
// CUDA graphs); rebuilt when the shape of the solve changes.
struct SolveCacheBase {
  virtual ~SolveCacheBase() {}
};

// One batched solve of (op + shift_r) x_r = b_r, r < nrhs, to prm->tol_true_rel
// through the FP64 defect-correction loop.
struct SolveReq {
  std::unique_ptr<SolveCacheBase>* cache = nullptr;  // solver-owned workspace slot (nullable)
  clg_context_s* ctx = nullptr;
  const clg_solver_params* prm = nullptr;
  clg_gauge_s* U = nullptr;
  clg_lattice_s* lat = nullptr;
  int kind = 0;
  double param = 0.0;
  int op = 0;
  int subset = 0;
  int nrhs = 1;
  FieldRef b;                  // nrhs right-hand sides, or one copied to every rhs
  bool b_broadcast = false;
  const FieldRef* x0 = nullptr;      // start vectors (any precision), nullable
  const double2* shifts = nullptr;   // host, nrhs complex shifts, nullable
  std::vector<FieldRef> xout;        // one field holding nrhs, or nrhs single fields
  clg_solve_info* info = nullptr;
};
clg_status solve_core(const SolveReq& q);

}  // namespace clg

struct clg_solver_s {
  clg_context_s* ctx = nullptr;
  clg_solver_params p;
  std::unique_ptr<clg::SolveCacheBase> cache;        // single-shift solves
  std::unique_ptr<clg::SolveCacheBase> cache_shift;  // multi-shift refinement
  std::unique_ptr<clg::SolveCacheBase> cache_cgm;    // multi-shift CG vectors, state, graph
  std::unique_ptr<clg::SolveCacheBase> cache_gcro;   // GCRO-DR vectors and the recycled subspace
  std::unique_ptr<clg::SolveCacheBase> cache_fom;    // multi-shift FOM basis and solutions
  std::unique_ptr<clg::SolveCacheBase> cache_batch;  // a batch of lattices: table, padded fields, workspace
  // X = (DD^+)^-1 phi and Y = D^+ X of clg_wilson_fermion_force
  clg_field force_x = nullptr, force_y = nullptr;
  // phi_i = (DD^+ + b_i)^-1 phi and phi_id = D0 phi_i of clg_ks_fermion_force
  std::vector<clg_field> ks_phi_i, ks_phi_id;
  ~clg_solver_s() {
    if (force_x) clg_field_destroy(force_x);
    if (force_y) clg_field_destroy(force_y);
    for (clg_field f : ks_phi_i) clg_field_destroy(f);
    for (clg_field f : ks_phi_id) clg_field_destroy(f);
  }
};

namespace clg {
// GCRO-DR (gcrodr.cu)
clg_status gcrodr_solve(::clg_solver_s* S, clg_field_s* X, clg_field_s* B, clg_gauge_s* U, int op, clg_field_s* X0,
                        clg_solve_info* info);
}  // namespace clg
