// C ABI of n4b200: context, workspace planning, launches.
//
// The reference drives every step from the host with per-iteration
// cudaMalloc/cudaFree, device-wide synchronisations and host FFTs
// (cudaN4.cu:1418-1747).  Here a run is four stream-ordered launches with no
// host round trip: prologue (threshold/shrink/log), the N4 kernel (all levels
// and iterations on the device), per-axis tables, and the fused full-
// resolution correction.  Workspaces are owned by the context and only grow.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "n4_kernels.cuh"

using namespace n4;

namespace {

thread_local std::string g_err;

n4_status_t fail(n4_status_t s, const std::string &msg) {
  g_err = msg;
  return s;
}

}  // namespace

// shared with the encoder translation unit
n4_status_t n4_record_error(n4_status_t s, const char *msg) { return fail(s, msg); }
// defined in the encoder translation unit
int n4_encoder_capacity(const n4_encoder_t *enc);
// kernels one n4_encoder_predict call of batch B launches
int n4_encoder_predict_launches(const n4_encoder_t *enc, int B);

namespace {

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      cudaGetLastError();                                                                \
      return fail(e_ == cudaErrorMemoryAllocation ? N4_ERR_OOM : N4_ERR_CUDA,            \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                   \
    }                                                                                    \
  } while (0)

#define TRY(expr)                                \
  do {                                           \
    n4_status_t s_ = (expr);                     \
    if (s_ != N4_OK) return s_;                  \
  } while (0)

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  n4_status_t ensure(size_t bytes, const char *what) {
    if (bytes <= cap) return N4_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    bytes = align_up(std::max<size_t>(bytes, 256), 256);
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(N4_ERR_OOM, std::string("cudaMalloc failed for ") + what);
    }
    cap = bytes;
    return N4_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class T> T *as() const { return (T *)p; }
};

// One slot of the descriptor upload ring: pinned host staging + device copy
// + an event recorded after the last kernel that reads the slot.
struct Slot {
  char *h = nullptr;
  DevBuf d;
  size_t cap = 0;
  cudaEvent_t ev = nullptr;
  bool pending = false;
  // report bookkeeping of the run that used the slot
  int nrep = 0;
  size_t off_rep = 0, off_flags = 0;
  std::vector<int> path, csize, perm;   // per descriptor: path, cluster size, caller's index
};

// Autotuner key: lattice, levels, bins and the fitting-grid size of every
// volume of the run, in order.
using TuneKey = std::vector<int>;
struct TuneVal {
  int grid;   // 1 = whole-GPU path
  int K;      // CTAs per cluster
  int nt;     // threads per CTA
  int corr;   // correction tile shape (index into kCorrectShape)
  int nsub;   // overlapped sub-batches (0: the default rule)
  int taper;  // 1: the first and last sub-batch half the size of the others
  int adapt;  // > 0: each sub-batch on the smallest cluster size >= adapt its volumes fit
};

constexpr int kStaticSmemReserve = 1024;
constexpr int kSlots = 4;
constexpr int kMaxSub = 4;   // sub-batches of a pipelined batch
constexpr int kHostLanes = 4;   // lanes of n4_run_batched_host

}  // namespace

struct n4_context {
  int device = 0;
  int nsm = 0;
  int max_smem = 0;
  DevBuf imlog, tables, big, red, bar;
  DevBuf s1, s2, s3, s4, s5;   // component scratch
  DevBuf warm_x, warm_lat;     // learned warm start: network inputs, predicted lattices
  DevBuf h_im, h_mask, h_out, h_lat, h_bias, h_warm;   // host-run staging
  // pipelined host batches: one stream and one device staging slot per lane
  DevBuf hb;
  cudaStream_t hst[kHostLanes] = {};
  cudaEvent_t hev[kHostLanes] = {};
  cudaEvent_t hclock[2] = {};
  Slot slots[kSlots];
  int next_slot = 0;
  int last_slot = -1;
  cudaStream_t last_stream = nullptr;
  cudaEvent_t last_done = nullptr;
  std::map<TuneKey, TuneVal> tune;
  // standalone components: (fx, fy, fz, ncpt, field alignment) -> fit shape,
  // (fx, fy, fz, ncpt) -> evaluation (correction) tile shape
  std::map<std::vector<int>, int> fit_tune, eval_tune;
  // max co-resident clusters per (threads, cluster size, shared bytes)
  std::map<std::tuple<int, int, int>, int> cluster_cap;
  // sub-batch pipeline: N4 launches on two high-priority streams, prologues
  // and warm starts on one low-priority stream, corrections on another
  cudaStream_t pipe[5] = {};   // N4 (2), prologues and pooling, corrections, encoder
  cudaEvent_t pev[24] = {};
  // profiling
  int profiling = 0;
  cudaEvent_t ev[5] = {};
  int prof_launches = 0;
  long long prof_fit = 0, prof_full = 0;
  int prof_fit_shape = -1, prof_corr_shape = -1;   // shapes of the last profiled call
  bool prof_valid = false;
};

struct n4_batch_graph;

namespace {

// ------------------------------------------------------------------ params
struct Dims {
  int FX, FY, FZ;   // full resolution
  int X, Y, Z;      // fitting grid
};

int npad_of(int bins) {
  double e = std::ceil(std::log((double)bins) / std::log(2.0)) + 1.0;
  return (int)(std::pow(2.0, e) + 0.5);
}

// float4 I/O is used only when rows are whole float4s and every pointer is 16-byte aligned.
int vec4_ok(int fz, const void *a, const void *b, const void *c) {
  auto al = [](const void *p) { return ((uintptr_t)p & 15u) == 0; };
  return (fz % 4 == 0) && fz <= 1024 && al(a) && al(b) && al(c) ? 1 : 0;
}

int final_nc(unsigned nc0, unsigned levels) { return (int)(((nc0 - 3) << (levels - 1)) + 3); }

n4_status_t check_params(const n4_params_t *p) {
  if (!p) return fail(N4_ERR_INVALID_ARG, "params is NULL");
  if (p->SplineOrder != 3) return fail(N4_ERR_UNSUPPORTED_SPLINE_ORDER, "only cubic B-splines (SplineOrder 3) are supported");
  if (p->NumberOfHistogramBins < 2 || p->NumberOfHistogramBins > 1024)
    return fail(N4_ERR_INVALID_ARG, "NumberOfHistogramBins must be in [2, 1024]");
  if (p->NumberOfFittingLevels < 1 || p->NumberOfFittingLevels > N4_MAX_LEVELS)
    return fail(N4_ERR_INVALID_ARG, "NumberOfFittingLevels must be in [1, 8]");
  if (p->NumberOfControlPoints_x < 4 || p->NumberOfControlPoints_y < 4 || p->NumberOfControlPoints_z < 4)
    return fail(N4_ERR_INVALID_ARG, "at least 4 control points per axis are required");
  const int ncx = final_nc(p->NumberOfControlPoints_x, p->NumberOfFittingLevels);
  const int ncy = final_nc(p->NumberOfControlPoints_y, p->NumberOfFittingLevels);
  const int ncz = final_nc(p->NumberOfControlPoints_z, p->NumberOfFittingLevels);
  if (ncx > 1024 || ncy > 1024 || ncz > kMaxNcz || (long long)ncx * ncy * ncz > (1 << 20))
    return fail(N4_ERR_TOO_LARGE, "final lattice too large (z control points <= 64, total <= 2^20)");
  if (p->ShrinkFactor < 1 || p->ShrinkFactor > 16) return fail(N4_ERR_INVALID_ARG, "ShrinkFactor must be in [1, 16]");
  if (!(p->WienerFilterNoise >= 0.0f) || !(p->BiasFieldFullWidthAtHalfMaximum > 0.0f))
    return fail(N4_ERR_INVALID_ARG, "WienerFilterNoise must be >= 0 and the FWHM > 0");
  if (!(p->FitEpsilon >= 0.0f)) return fail(N4_ERR_INVALID_ARG, "FitEpsilon must be >= 0");
  for (unsigned l = 0; l < p->NumberOfFittingLevels; ++l)
    if (p->MaximumNumberOfIterations[l] > 1000000u) return fail(N4_ERR_INVALID_ARG, "too many iterations");
  if (((p->flags >> 8) & 31u) > 16u) return fail(N4_ERR_INVALID_ARG, "cluster size must be in [1, 16]");
  return N4_OK;
}

n4_status_t make_dims(const n4_params_t *p, unsigned fx, unsigned fy, unsigned fz, Dims &d) {
  const unsigned s = p->ShrinkFactor;
  if (fx == 0 || fy == 0 || fz == 0) return fail(N4_ERR_INVALID_ARG, "empty volume");
  if (fx % s || fy % s || fz % s) return fail(N4_ERR_INVALID_ARG, "dimensions must be multiples of ShrinkFactor");
  if ((unsigned long long)fx * fy * fz >= (1ull << 40)) return fail(N4_ERR_TOO_LARGE, "volume too large");
  // the correction indexes full-resolution rows (fx * fy of them) in 32 bits
  if ((unsigned long long)fx * fy >= (1ull << 32)) return fail(N4_ERR_TOO_LARGE, "more than 2^32 - 1 rows (fx * fy)");
  d.FX = (int)fx; d.FY = (int)fy; d.FZ = (int)fz;
  d.X = (int)(fx / s); d.Y = (int)(fy / s); d.Z = (int)(fz / s);
  if (d.Z > 1024) return fail(N4_ERR_TOO_LARGE, "fitting grid rows longer than 1024 voxels (raise ShrinkFactor)");
  if ((long long)d.X * d.Y * d.Z >= (1ll << 22) * 1024) return fail(N4_ERR_TOO_LARGE, "fitting grid too large");
  return N4_OK;
}

// The decimal number a float parameter was written as (0.01f -> 0.01), so
// that the FP64 parts of the algorithm use the same constants as N4.py.
double decimal_of(float f) {
  char buf[32];
  std::snprintf(buf, sizeof(buf), "%.7g", (double)f);
  return std::strtod(buf, nullptr);
}

Params make_dev_params(const n4_params_t *p) {
  Params r{};
  r.bins = (int)p->NumberOfHistogramBins;
  r.wiener = decimal_of(p->WienerFilterNoise);
  r.fwhm = decimal_of(p->BiasFieldFullWidthAtHalfMaximum);
  r.thr = decimal_of(p->ConvergenceThreshold);
  r.eps = p->FitEpsilon;
  r.zero_den = (p->flags & N4_FLAG_FIT_ZERO_DEN) ? 1 : 0;
  r.ddof1 = (p->flags & N4_FLAG_CV_DDOF1) ? 1 : 0;
  for (unsigned l = 0; l < N4_MAX_LEVELS; ++l)
    r.iters[l] = l < p->NumberOfFittingLevels ? (int)p->MaximumNumberOfIterations[l] : 0;
  return r;
}

// Workspace layout for a group of K CTAs over the given fitting grids.
Plan make_plan(const n4_params_t *p, int K, const std::vector<Dims> &vols, bool grid) {
  Plan pl{};
  pl.levels = (int)p->NumberOfFittingLevels;
  pl.nc0x = (int)p->NumberOfControlPoints_x;
  pl.nc0y = (int)p->NumberOfControlPoints_y;
  pl.nc0z = (int)p->NumberOfControlPoints_z;
  pl.NCX = final_nc(p->NumberOfControlPoints_x, p->NumberOfFittingLevels);
  pl.NCY = final_nc(p->NumberOfControlPoints_y, p->NumberOfFittingLevels);
  pl.NCZ = final_nc(p->NumberOfControlPoints_z, p->NumberOfFittingLevels);
  pl.NLAT = pl.NCX * pl.NCY * pl.NCZ;
  pl.bins = (int)p->NumberOfHistogramBins;
  pl.npad = npad_of(pl.bins);
  pl.hoff = (int)(0.5 * (pl.npad - pl.bins));
  long long slab = 0, rows_max = 0, nvxl = 0;
  for (const Dims &d : vols) {
    pl.Xmax = std::max(pl.Xmax, d.X);
    pl.Ymax = std::max(pl.Ymax, d.Y);
    pl.Zmax = std::max(pl.Zmax, d.Z);
    const long long rows = (long long)d.X * d.Y;
    // grid: contiguous rows; cluster: whole x-planes, ceil(X / K) per CTA
    const long long rpc = grid ? (rows + K - 1) / K : ((long long)d.X + K - 1) / K * d.Y;
    rows_max = std::max(rows_max, rpc);
    slab = std::max(slab, rpc * d.Z);
    // the y contraction spans every x-plane a CTA touches: all of them when
    // rows are interleaved (cluster), a contiguous range otherwise (grid)
    nvxl = std::max(nvxl, grid ? (rpc - 1) / d.Y + 2 : ((long long)d.X + K - 1) / K);
  }
  pl.slab_floats = (int)slab;
  pl.rows_max = (int)rows_max;
  pl.nvxl = (int)nvxl;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o = align_up(o + bytes, 16); return (int)r; };
  pl.o_ax = take(axis_bytes(pl.Xmax, pl.NCX - 3));
  pl.o_ay = take(axis_bytes(pl.Ymax, pl.NCY - 3));
  pl.o_az = take(axis_bytes(pl.Zmax, pl.NCZ - 3));
  pl.o_L = take((size_t)pl.NLAT * 4);
  pl.o_D = take((size_t)pl.NLAT * 4);
  pl.o_den = take((size_t)pl.NLAT * 4);
  pl.o_tmp = take((size_t)pl.NLAT * 4);
  pl.o_aux = take((size_t)pl.NLAT * 4);
  // cluster path: the histogram copies and the two FFT work buffers share
  // the Gd region (see Plan::alias_sharpen); grid path: shared memory
  const size_t hist_bytes = (size_t)kHistCopies * pl.bins * 4, fft_bytes = (size_t)pl.npad * 16;
  pl.alias_sharpen = grid ? 0 : 1;
  if (grid) {
    pl.o_hist = take(hist_bytes);
    pl.o_fa = take(fft_bytes);
    pl.o_fb = take(fft_bytes);
  }
  pl.o_H64 = take((size_t)pl.bins * 8);
  pl.o_R2 = take((size_t)pl.bins * 8);   // the residual's per-bin linear form
  pl.o_E = take((size_t)pl.bins * 8);
  pl.o_tw = take((size_t)pl.npad * 16);
  pl.o_ff = grid ? take((size_t)pl.npad * 8) : 0;   // cluster: in the Gd region
  pl.o_red = take(160 * 8);
  pl.o_misc = take(64);
  pl.sm_bytes = (int)align_up(o, 128);
  o = 0;
  pl.b_imlog = take(((size_t)pl.slab_floats + 8) * 4);   // logU (cluster: the staged rows first)
  pl.a_fa = 0;
  pl.a_fb = (int)fft_bytes;
  pl.a_hist = (int)(2 * fft_bytes);
  pl.a_ff = pl.a_hist;   // written by the sharpening after the histogram copies are merged
  const size_t ff_bytes = (size_t)pl.npad * 8;
  pl.b_Gd = take(std::max((size_t)pl.rows_max * pl.NCZ * 4, grid ? 0 : 2 * fft_bytes + std::max(hist_bytes, ff_bytes)));
  pl.b_T2 = take((size_t)pl.nvxl * pl.NCY * pl.NCZ * 4);
  pl.b_slotA = take(sizeof(Stats));
  pl.b_slotB = take((size_t)pl.bins * 8);
  pl.b_slotC = take((size_t)pl.NLAT * 4);
  pl.b_slice = take(std::max((size_t)(pl.NLAT + K - 1) / K * 4, (size_t)(pl.bins + K - 1) / K * 8));
  pl.big_bytes = (int)align_up(o, 128);
  return pl;
}

bool cluster_fits(const n4_context *ctx, const Plan &pl) {
  return (long long)pl.sm_bytes + pl.big_bytes + kStaticSmemReserve <= ctx->max_smem;
}

// Dynamic shared memory granted to k_n4_cluster<NT> per device.  The
// attribute belongs to the function (process-wide), not to a context, so the
// record is process-wide too and the grant only ever grows.
constexpr int kMaxDev = 64;
std::mutex g_attr_mu;
int g_attr_smem[kMaxDev][3];   // per thread count: 512, 768, 1024

template <int NT>
n4_status_t grant_cluster_smem(n4_context *ctx, int smem) {
  static_assert(NT == 512 || NT == 768 || NT == 1024, "engine thread counts");
  if (ctx->device < 0 || ctx->device >= kMaxDev) return fail(N4_ERR_INVALID_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_attr_mu);
  int &granted = g_attr_smem[ctx->device][NT == 512 ? 0 : (NT == 768 ? 1 : 2)];
  if (smem > granted) {
    CK(cudaFuncSetAttribute(k_n4_cluster<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CK(cudaFuncSetAttribute(k_n4_cluster<NT>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    granted = smem;
  }
  return N4_OK;
}

template <int NT>
n4_status_t cluster_capacity(n4_context *ctx, int K, int smem, int *nclusters) {
  auto kern = k_n4_cluster<NT>;
  TRY(grant_cluster_smem<NT>(ctx, smem));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(K);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = K;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  CK(cudaOccupancyMaxActiveClusters(&n, kern, &cfg));
  *nclusters = n;
  return N4_OK;
}

n4_status_t capacity(n4_context *ctx, int nt, int K, int smem, int *n) {
  const auto key = std::make_tuple(nt, K, smem);
  auto it = ctx->cluster_cap.find(key);
  if (it != ctx->cluster_cap.end()) { *n = it->second; return N4_OK; }
  TRY(nt == 1024 ? cluster_capacity<1024>(ctx, K, smem, n)
                  : nt == 768 ? cluster_capacity<768>(ctx, K, smem, n) : cluster_capacity<512>(ctx, K, smem, n));
  ctx->cluster_cap[key] = *n;
  return N4_OK;
}

// Largest cluster (<= 16 CTAs) whose per-CTA share of every volume fits.
n4_status_t choose_cluster(n4_context *ctx, const n4_params_t *p, const std::vector<Dims> &vols, int nt,
                           int *K_out) {
  *K_out = 0;
  for (int K : {16, 12, 8, 6, 4, 2, 1}) {
    Plan pl = make_plan(p, K, vols, false);
    if (!cluster_fits(ctx, pl)) continue;
    int n = 0;
    TRY(capacity(ctx, nt, K, pl.sm_bytes + pl.big_bytes, &n));
    if (n > 0) { *K_out = K; return N4_OK; }
  }
  return N4_OK;
}

// Volumes (indices into dims) that run on a cluster of K CTAs: one launch
// shares one shared-memory layout, sized by the maxima over its volumes, so
// volumes are added largest first while that layout still fits; the others
// go to `rest`.
std::vector<int> cluster_subset(const n4_context *ctx, const n4_params_t *p, const std::vector<Dims> &dims,
                                const std::vector<int> &idx, int K, std::vector<int> *rest) {
  std::vector<int> order = idx, fit;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return (long long)dims[a].X * dims[a].Y * dims[a].Z > (long long)dims[b].X * dims[b].Y * dims[b].Z;
  });
  std::vector<Dims> sub;
  for (int i : order) {
    sub.push_back(dims[i]);
    if (cluster_fits(ctx, make_plan(p, K, sub, false))) {
      fit.push_back(i);
    } else {
      sub.pop_back();
      if (rest) rest->push_back(i);
    }
  }
  std::sort(fit.begin(), fit.end());
  if (rest) std::sort(rest->begin(), rest->end());
  return fit;
}

// ------------------------------------------------------------------ upload ring
struct Upload {
  Slot *slot;
  int index;
  size_t off;
  char *h() const { return slot->h; }
  template <class T> T *hp(size_t o) const { return (T *)(slot->h + o); }
  template <class T> T *dp(size_t o) const { return (T *)((char *)slot->d.p + o); }
};

n4_status_t acquire_slot(n4_context *ctx, size_t bytes, Upload &u) {
  const int i = ctx->next_slot;
  ctx->next_slot = (ctx->next_slot + 1) % kSlots;
  Slot &s = ctx->slots[i];
  if (!s.ev) CK(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
  if (s.pending) { CK(cudaEventSynchronize(s.ev)); s.pending = false; }
  if (bytes > s.cap) {
    if (s.h) cudaFreeHost(s.h);
    s.h = nullptr;
    s.cap = 0;
    const size_t cap = align_up(std::max<size_t>(bytes, 1 << 16), 4096);
    CK(cudaMallocHost((void **)&s.h, cap));
    TRY(s.d.ensure(cap, "descriptor slot"));
    s.cap = cap;
  }
  std::memset(s.h, 0, bytes);
  u.slot = &s;
  u.index = i;
  u.off = 0;
  return N4_OK;
}

// Order this run after the context's previous run (which may be on another stream).
n4_status_t begin_run(n4_context *ctx, cudaStream_t st) {
  CK(cudaSetDevice(ctx->device));
  if (!ctx->last_done) CK(cudaEventCreateWithFlags(&ctx->last_done, cudaEventDisableTiming));
  if (ctx->last_slot >= 0 && st != ctx->last_stream) CK(cudaStreamWaitEvent(st, ctx->last_done, 0));
  return N4_OK;
}

n4_status_t end_run(n4_context *ctx, cudaStream_t st, Upload &u) {
  CK(cudaEventRecord(u.slot->ev, st));
  CK(cudaEventRecord(ctx->last_done, st));
  u.slot->pending = true;
  ctx->last_slot = u.index;
  ctx->last_stream = st;
  return N4_OK;
}

n4_status_t prof_mark(n4_context *ctx, int k, cudaStream_t st) {
  if (!ctx->profiling) return N4_OK;
  if (!ctx->ev[k]) CK(cudaEventCreate(&ctx->ev[k]));
  CK(cudaEventRecord(ctx->ev[k], st));
  return N4_OK;
}

// ------------------------------------------------------------------ the run
struct RunVol {
  const float *im;
  const void *mask;            // float or byte (N4_FLAG_MASK_U8)
  float *out, *lat, *bias;
  const float *warm;
  float *im_w;
  void *mask_w;
  Dims d;
};

// Workspaces of the whole-GPU path for one volume (sized before any capture).
n4_status_t ensure_grid_workspace(n4_context *ctx, const n4_params_t *p, const Dims &d) {
  std::vector<Dims> one{d};
  Plan pl = make_plan(p, ctx->nsm, one, true);
  TRY(ctx->big.ensure((size_t)pl.big_bytes * ctx->nsm, "grid workspace"));
  TRY(ctx->red.ensure(std::max((size_t)pl.bins * 8, (size_t)pl.NLAT * 4) + 64, "grid reduction"));
  TRY(ctx->bar.ensure(64, "grid barrier"));
  return N4_OK;
}

// Cooperative launch of the whole-GPU N4 kernel with NT threads per CTA.
template <int NT>
n4_status_t launch_grid_kernel(GridArgs &a, int nblk, int smem, cudaStream_t st) {
  CK(cudaFuncSetAttribute(k_n4_grid<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int occ = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_n4_grid<NT>, NT, smem));
  if (occ < 1) return fail(N4_ERR_TOO_LARGE, "grid kernel does not fit on an SM");
  void *args[] = {&a};
  CK(cudaLaunchCooperativeKernel((void *)k_n4_grid<NT>, dim3(nblk), dim3(NT), args, smem, st));
  return N4_OK;
}

n4_status_t launch_grid_path(n4_context *ctx, const n4_params_t *p, const Params &pr, const RunVol &rv,
                             const VolJob &job0, int nt, cudaStream_t st) {
  std::vector<Dims> one{rv.d};
  int nblk = ctx->nsm;
  Plan pl = make_plan(p, nblk, one, true);
  if (pl.sm_bytes + kStaticSmemReserve > ctx->max_smem)
    return fail(N4_ERR_TOO_LARGE, "histogram/lattice workspace exceeds shared memory");
  if ((long long)pl.rows_max * rv.d.Z >= (1ll << 22))
    return fail(N4_ERR_TOO_LARGE, "fitting grid too large for one GPU (raise ShrinkFactor)");
  TRY(ctx->big.ensure((size_t)pl.big_bytes * nblk, "grid workspace"));
  TRY(ctx->red.ensure(std::max((size_t)pl.bins * 8, (size_t)pl.NLAT * 4) + 64, "grid reduction"));
  TRY(ctx->bar.ensure(64, "grid barrier"));
  CK(cudaMemsetAsync(ctx->bar.p, 0, 64, st));
  GridArgs a{};
  a.pl = pl;
  a.pr = pr;
  a.job = job0;
  a.big_base = ctx->big.as<char>();
  a.big_stride = pl.big_bytes;
  a.bar.count = ctx->bar.as<unsigned>();
  a.bar.gen = ctx->bar.as<unsigned>() + 1;
  a.bar.err = (int *)ctx->bar.as<unsigned>() + 2;
  a.bar.nblocks = nblk;
  a.red_global = ctx->red.as<float>();
  const int smem = pl.sm_bytes;
  if (nt == 1024) return launch_grid_kernel<1024>(a, nblk, smem, st);
  if (nt == 768) return launch_grid_kernel<768>(a, nblk, smem, st);
  return launch_grid_kernel<512>(a, nblk, smem, st);
}

template <int NT>
n4_status_t launch_cluster_kernel(n4_context *ctx, const ClusterArgs &a, int K, int nclusters, int smem,
                                  cudaStream_t st) {
  auto kern = k_n4_cluster<NT>;
  TRY(grant_cluster_smem<NT>(ctx, smem));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(K * nclusters);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = K;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, kern, a));
  return N4_OK;
}

struct Choice {
  bool grid;
  int K, nt;
  int corr = -1;   // correction tile shape; -1: the recorded or default one
  int nsub = 0;    // overlapped sub-batches; 0: the recorded count or the default rule
  int taper = 0;   // 1: first and last sub-batch half-size (three or more sub-batches)
  int adapt = 0;   // > 0: per sub-batch, the smallest cluster size >= adapt that holds its volumes
};

// Autotuner key: first-level lattice, levels, bins, shrink factor and the
// fitting-grid size of every volume (with the shrink factor, the
// full-resolution size the correction runs over).
TuneKey tune_key(const n4_params_t *p, const std::vector<Dims> &vols) {
  TuneKey k{(int)p->NumberOfControlPoints_x, (int)p->NumberOfControlPoints_y, (int)p->NumberOfControlPoints_z,
            (int)p->NumberOfFittingLevels, (int)p->NumberOfHistogramBins, (int)p->ShrinkFactor, (int)vols.size()};
  // the volumes' sizes in a canonical order: a run plans its volumes largest
  // first, whatever order the caller passes them in
  std::vector<std::tuple<int, int, int>> sz;
  for (const Dims &d : vols) sz.emplace_back(d.X, d.Y, d.Z);
  std::sort(sz.begin(), sz.end());
  for (const auto &t : sz) { k.push_back(std::get<0>(t)); k.push_back(std::get<1>(t)); k.push_back(std::get<2>(t)); }
  return k;
}

n4_status_t choose_path(n4_context *ctx, const n4_params_t *p, const std::vector<Dims> &vols, bool batch,
                        Choice &c) {
  const Dims &d0 = vols[0];
  c.nt = (p->flags & N4_FLAG_CTA_512) ? 512 : 1024;
  c.grid = false;
  c.K = 0;
  (void)d0;
  (void)batch;
  const int forced_k = (int)((p->flags >> 8) & 31u);
  if (forced_k) {
    if (p->flags & N4_FLAG_FORCE_GRID) return fail(N4_ERR_INVALID_ARG, "cluster size given with FORCE_GRID");
    Plan pl = make_plan(p, forced_k, vols, false);
    int cap = 0;
    if (cluster_fits(ctx, pl)) TRY(capacity(ctx, c.nt, forced_k, pl.sm_bytes + pl.big_bytes, &cap));
    if (cap < 1) return fail(N4_ERR_TOO_LARGE, "a volume does not fit a cluster of the requested size");
    c.K = forced_k;
    return N4_OK;
  }
  if (!(p->flags & (N4_FLAG_FORCE_GRID | N4_FLAG_FORCE_CLUSTER))) {
    auto it = ctx->tune.find(tune_key(p, vols));
    if (it != ctx->tune.end()) {
      c.grid = it->second.grid != 0;
      c.K = it->second.K;
      c.corr = it->second.corr;
      c.nsub = it->second.nsub;
      c.taper = it->second.taper;
      c.adapt = it->second.adapt;
      if (!(p->flags & N4_FLAG_CTA_512)) c.nt = it->second.nt;
      return N4_OK;
    }
  }
  if (!(p->flags & N4_FLAG_FORCE_GRID)) TRY(choose_cluster(ctx, p, vols, c.nt, &c.K));
  if (c.K == 0) {
    if (p->flags & N4_FLAG_FORCE_CLUSTER) return fail(N4_ERR_TOO_LARGE, "volume does not fit a thread-block cluster");
    c.grid = true;
  }
  return N4_OK;
}

// Core of n4_run / n4_run_batched: every pointer is a device pointer.
// A run's plan: the execution path of every volume and the layout of its
// descriptor buffer (volume descriptors, reports, flags, work-queue counter).
struct Prepared {
  int n = 0;
  Params pr{};
  Choice ch{};
  std::vector<int> in_cluster, in_grid, path, csize;
  std::vector<Dims> dims;
  std::vector<RunVol> rvs;
  std::vector<size_t> imlog_off, tab_off;
  int NCX = 0, NCY = 0, NCZ = 0;
  size_t o_pro = 0, o_pst = 0, o_job = 0, o_ord = 0, o_tab = 0, o_cor = 0, o_tst = 0, o_rep = 0, o_flg = 0,
         o_q = 0, o_pool = 0, bytes = 0;
  n4_encoder_t *enc = nullptr;   // learned warm start run inside the batch
  int enc_batch = 0;             // predictions per encoder call
  long long fit_total = 0, tiles = 0;
  int corr = kCorrectDefault;    // correction tile shape
  int nsub = 1;                  // sub-batches (volume ranges sub_lo[k] .. sub_lo[k + 1])
  std::vector<int> sub_lo;
  std::vector<int> subK;         // cluster size of each sub-batch (empty: ch.K for all)
  std::vector<int> perm;         // descriptor k holds the caller's volume perm[k]
};

// Descriptor buffer: pinned host staging and its device copy.
struct DescBuf {
  char *h = nullptr;
  char *d = nullptr;
  template <class T> T *hp(size_t o) const { return (T *)(h + o); }
  template <class T> T *dp(size_t o) const { return (T *)(d + o); }
};

// Choose paths, size the workspaces and lay out the descriptors.
n4_status_t plan_run(n4_context *ctx, const n4_params_t *p, const std::vector<RunVol> &rvs, const Choice *forced,
                     Prepared &P, n4_encoder_t *enc = nullptr) {
  const int n = (int)rvs.size();
  P.n = n;
  // descriptors hold the volumes largest first (fitting voxels), so that
  // sub-batches, which are contiguous descriptor ranges, end with the small
  // ones and the last launch's tail is short; reports go back in the
  // caller's order
  P.perm.resize(n);
  for (int i = 0; i < n; ++i) P.perm[i] = i;
  std::stable_sort(P.perm.begin(), P.perm.end(), [&](int a, int b) {
    const Dims &x = rvs[a].d, &y = rvs[b].d;
    return (long long)x.X * x.Y * x.Z > (long long)y.X * y.Y * y.Z;
  });
  P.rvs.resize(n);
  for (int i = 0; i < n; ++i) P.rvs[i] = rvs[P.perm[i]];
  if (enc) {
    if (p->NumberOfControlPoints_x != 4 || p->NumberOfControlPoints_y != 4 || p->NumberOfControlPoints_z != 4)
      return fail(N4_ERR_INVALID_ARG, "the warm-start encoder predicts 4x4x4 first-level lattices");
    for (const RunVol &r : P.rvs)
      if (r.warm) return fail(N4_ERR_INVALID_ARG, "warm lattices are predicted by the encoder: pass none");
    TRY(ctx->warm_x.ensure((size_t)n * kPoolCells * 2, "warm-start inputs"));
    TRY(ctx->warm_lat.ensure((size_t)n * 64 * 4, "warm-start lattices"));
    for (int i = 0; i < n; ++i) P.rvs[i].warm = ctx->warm_lat.as<float>() + 64 * i;
    P.enc = enc;
    P.enc_batch = n4_encoder_capacity(enc);
    if (P.enc_batch < 1) return fail(N4_ERR_INVALID_ARG, "encoder has no batch capacity");
  }
  P.pr = make_dev_params(p);
  for (const RunVol &r : P.rvs) P.dims.push_back(r.d);
  const std::vector<Dims> &dims = P.dims;
  Choice ch{};
  if (forced) ch = *forced;
  else TRY(choose_path(ctx, p, dims, n > 1, ch));
  if (!ch.grid) {
    for (int i = 0; i < n; ++i) P.in_cluster.push_back(i);
  } else if (n == 1) {
    P.in_grid.push_back(0);
  } else {
    // batch with volumes too large for a cluster: the largest cluster size
    // (the smallest per-CTA share) takes every volume its shared-memory
    // layout can hold, the whole-GPU path the rest
    std::vector<int> all(n), rest;
    for (int i = 0; i < n; ++i) all[i] = i;
    P.in_cluster = cluster_subset(ctx, p, dims, all, 16, &rest);
    P.in_grid = rest;
    if (!P.in_cluster.empty()) {
      std::vector<Dims> sub;
      for (int i : P.in_cluster) sub.push_back(dims[i]);
      const Plan pl = make_plan(p, 16, sub, false);
      int cap = 0;
      TRY(capacity(ctx, 1024, 16, pl.sm_bytes + pl.big_bytes, &cap));
      if (cap > 0) {
        ch.grid = false;
        ch.nt = 1024;
        ch.K = 16;
      } else {
        for (int i : P.in_cluster) P.in_grid.push_back(i);
        std::sort(P.in_grid.begin(), P.in_grid.end());
        P.in_cluster.clear();
      }
    }
  }
  if (!ch.grid && n > 1 && !(p->flags & N4_FLAG_CLUSTER_SIZE(31))) {
    // a recorded cluster size (autotuner): volumes whose share does not fit
    // a CTA of that cluster run on the whole-GPU path
    std::vector<int> rest;
    P.in_cluster = cluster_subset(ctx, p, dims, P.in_cluster, ch.K, &rest);
    for (int i : rest) P.in_grid.push_back(i);
  }
  P.ch = ch;
  P.corr = (ch.corr >= 0 && ch.corr < kCorrectShapes) ? ch.corr : kCorrectDefault;
  for (int i : P.in_grid) TRY(ensure_grid_workspace(ctx, p, dims[i]));
  P.path.assign(n, 0);
  P.csize.assign(n, 0);
  for (int i : P.in_cluster) { P.path[i] = 1; P.csize[i] = ch.K; }
  for (int i : P.in_grid) { P.path[i] = 2; P.csize[i] = ctx->nsm; }
  // sub-batches (cluster-path batches only): by default one per two waves of
  // the clusters that fit at once, so that every sub-batch keeps them busy
  P.nsub = 1;
  const int want_sub = (int)((p->flags >> 16) & 7u);
  if (P.in_grid.empty() && n > 1 && want_sub != 1) {
    int S = want_sub ? want_sub : ch.nsub;
    if (S == 0) {
      const Plan pl = make_plan(p, ch.K, dims, false);
      int cap = 0;
      TRY(capacity(ctx, ch.nt, ch.K, pl.sm_bytes + pl.big_bytes, &cap));
      S = cap > 0 ? n / (2 * cap) : 1;
    }
    P.nsub = std::max(1, std::min(std::min(S, kMaxSub), n));
  }
  P.sub_lo.resize(P.nsub + 1);
  if (P.nsub >= 3 && ch.taper && !want_sub) {
    // half-size first and last sub-batches: the first N4 launch starts after a
    // shorter prologue, and a shorter correction follows the last one
    const int S = P.nsub;
    for (int k = 0; k <= S; ++k) {
      const int w2 = k == 0 ? 0 : (k == S ? 2 * (S - 1) : 2 * k - 1);   // twice the cumulative weight
      P.sub_lo[k] = (int)((long long)n * w2 / (2 * (S - 1)));
    }
  } else {
    for (int k = 0; k <= P.nsub; ++k) P.sub_lo[k] = (int)((long long)n * k / P.nsub);
  }
  // a split of few volumes can leave a sub-batch empty (4 volumes tapered
  // over 4: 0,0,2,3,4); drop it, no launch may see an empty sub-batch
  P.sub_lo.erase(std::unique(P.sub_lo.begin(), P.sub_lo.end()), P.sub_lo.end());
  P.nsub = (int)P.sub_lo.size() - 1;
  // per-sub-batch cluster sizes: the volumes are planned largest first, so
  // later sub-batches hold smaller volumes and may take smaller clusters,
  // more of them side by side; their launches overlap the earlier ones'
  // tails on the other engine stream
  P.subK.clear();
  const int want_floor = (int)((p->flags >> 19) & 31u);
  if (want_floor) ch.adapt = want_floor;
  if (ch.adapt > 0 && P.nsub > 1 && P.in_grid.empty()) {
    for (int k = 0; k < P.nsub; ++k) {
      std::vector<Dims> sub(dims.begin() + P.sub_lo[k], dims.begin() + P.sub_lo[k + 1]);
      int Kk = 0;
      for (int K : {2, 4, 6, 8, 12, 16}) {
        if (K < ch.adapt) continue;
        const Plan pl = make_plan(p, K, sub, false);
        int cap = 0;
        if (cluster_fits(ctx, pl)) TRY(capacity(ctx, ch.nt, K, pl.sm_bytes + pl.big_bytes, &cap));
        if (cap > 0) { Kk = K; break; }
      }
      P.subK.push_back(Kk > 0 ? Kk : ch.K);
      for (int i = P.sub_lo[k]; i < P.sub_lo[k + 1]; ++i) P.csize[i] = P.subK[k];
    }
  }
  // workspaces
  P.NCX = final_nc(p->NumberOfControlPoints_x, p->NumberOfFittingLevels);
  P.NCY = final_nc(p->NumberOfControlPoints_y, p->NumberOfFittingLevels);
  P.NCZ = final_nc(p->NumberOfControlPoints_z, p->NumberOfFittingLevels);
  P.imlog_off.resize(n);
  P.tab_off.resize(n);
  size_t imlog_bytes = 0, tab_bytes = 0;
  for (int i = 0; i < n; ++i) {
    P.imlog_off[i] = imlog_bytes;
    imlog_bytes = align_up(imlog_bytes + (size_t)dims[i].X * dims[i].Y * dims[i].Z * 4 + 64, 256);
    P.tab_off[i] = tab_bytes;
    tab_bytes += align_up(axis_bytes(dims[i].FX, P.NCX - 3), 256) + align_up(axis_bytes(dims[i].FY, P.NCY - 3), 256) +
                 align_up(axis_bytes(dims[i].FZ, P.NCZ - 3), 256);
  }
  TRY(ctx->imlog.ensure(imlog_bytes, "fitting grid"));
  TRY(ctx->tables.ensure(tab_bytes, "axis tables"));
  size_t o = 0;
  auto take = [&](size_t b) { size_t r = o; o = align_up(o + b, 16); return r; };
  P.o_pro = take(sizeof(PrologueVol) * n);
  P.o_pst = take(8 * n);
  P.o_job = take(sizeof(VolJob) * n);
  P.o_ord = take(4 * n);
  P.o_tab = take(sizeof(TableJob) * 3 * n);
  P.o_cor = take(sizeof(CorrectVol) * n);
  P.o_tst = take(8 * n);
  P.o_rep = take(sizeof(n4_report_t) * n);
  P.o_flg = take(4 * n);
  P.o_q = take(16 * kMaxSub);
  P.o_pool = take(sizeof(PoolJob) * n);
  P.bytes = o;
  return N4_OK;
}

// Fill the descriptors (host side of `B`, which must hold P.bytes zeroed bytes).
void fill_descriptors(n4_context *ctx, const n4_params_t *p, Prepared &P, const DescBuf &B) {
  const int n = P.n;
  PrologueVol *pv = B.hp<PrologueVol>(P.o_pro);
  long long *pst = B.hp<long long>(P.o_pst);
  VolJob *jb = B.hp<VolJob>(P.o_job);
  int *ord = B.hp<int>(P.o_ord);
  TableJob *tj = B.hp<TableJob>(P.o_tab);
  CorrectVol *cv = B.hp<CorrectVol>(P.o_cor);
  long long *tst = B.hp<long long>(P.o_tst);
  n4_report_t *rep = B.hp<n4_report_t>(P.o_rep);
  long long fit_total = 0, tiles = 0;
  char *tabs = ctx->tables.as<char>();
  for (int i = 0; i < n; ++i) {
    const RunVol &r = P.rvs[i];
    const Dims &d = P.dims[i];
    float *il = (float *)(ctx->imlog.as<char>() + P.imlog_off[i]);
    pv[i] = PrologueVol{r.im, r.mask, r.im_w, r.mask_w, d.FX, d.FY, d.FZ, (int)p->ShrinkFactor,
                        d.X, d.Y, d.Z, il, fit_total, (p->flags & N4_FLAG_MASK_U8) ? 1 : 0};
    pst[i] = fit_total;
    fit_total += (long long)d.X * d.Y * d.Z;
    jb[i] = VolJob{d.X, d.Y, d.Z, il, r.warm, r.lat, B.dp<n4_report_t>(P.o_rep) + i};
    B.hp<PoolJob>(P.o_pool)[i] = PoolJob{il, d.X, d.Y, d.Z};
    char *tx = tabs + P.tab_off[i];
    char *ty = tx + align_up(axis_bytes(d.FX, P.NCX - 3), 256);
    char *tz = ty + align_up(axis_bytes(d.FY, P.NCY - 3), 256);
    tj[3 * i] = TableJob{tx, d.FX, P.NCX};
    tj[3 * i + 1] = TableJob{ty, d.FY, P.NCY};
    tj[3 * i + 2] = TableJob{tz, d.FZ, P.NCZ};
    cv[i] = CorrectVol{r.im, r.out, r.bias, r.lat, tx, ty, tz, d.FX, d.FY, d.FZ, P.NCX, P.NCY, P.NCZ, tiles,
                       vec4_ok(d.FZ, r.im, r.out, r.bias)};
    tst[i] = tiles;
    const long long rt = kCorrectShape[P.corr].rows;
    tiles += ((long long)d.FX * d.FY + rt - 1) / rt;
    std::memset(&rep[i], 0, sizeof(n4_report_t));
    rep[i].status = -1;
  }
  P.fit_total = fit_total;
  P.tiles = tiles;
  // longest-first order of each sub-batch's cluster queue, the sub-batches
  // one after the other
  std::vector<int> order;
  const int nsub = P.sub_lo.empty() ? 1 : P.nsub;
  for (int k = 0; k < nsub; ++k) {
    const int lo = P.sub_lo.empty() ? 0 : P.sub_lo[k], hi = P.sub_lo.empty() ? n : P.sub_lo[k + 1];
    std::vector<int> part;
    for (int i : P.in_cluster)
      if (i >= lo && i < hi) part.push_back(i);
    std::stable_sort(part.begin(), part.end(), [&](int a, int b) {
      const Dims &x = P.dims[a], &y = P.dims[b];
      return (long long)x.X * x.Y * x.Z > (long long)y.X * y.Y * y.Z;
    });
    order.insert(order.end(), part.begin(), part.end());
  }
  for (size_t k = 0; k < order.size(); ++k) ord[k] = order[k];
}

// k_prologue over the volumes [lo, hi) of a run: the vectorised variant for
// shrink 2 or 4 when every row of those volumes is aligned for it, else the
// scalar one (the same values either way).
void launch_prologue(const n4_params_t *p, const Prepared &P, const DescBuf &B, int lo, int hi, long long g0,
                     long long count, int blocks, cudaStream_t st) {
  int S = (int)p->ShrinkFactor;
  const bool u8 = (p->flags & N4_FLAG_MASK_U8) != 0;
  if (S != 2 && S != 4) S = 0;
  for (int i = lo; i < hi && S; ++i) {
    const Dims &d = P.dims[i];
    if ((long long)d.X * d.Y * d.Z >= (1ll << 31) || ((uintptr_t)P.rvs[i].im % (4 * S)) != 0 ||
        (P.rvs[i].mask && ((uintptr_t)P.rvs[i].mask % (u8 ? S : 4 * S)) != 0))
      S = 0;
  }
  const PrologueVol *pv = B.dp<PrologueVol>(P.o_pro) + lo;
  const long long *pst = B.dp<long long>(P.o_pst) + lo;
  int *flg = B.dp<int>(P.o_flg) + lo;
  // A grid of more than one wave is cut to whole waves of the variant's
  // resident CTAs: every CTA runs the same number of grid-stride passes, so a
  // last partial wave would run as long as a full one on a fraction of the SMs
  // (148 x 16 CTAs of k_prologue<2>, 5 resident per SM, were 3.2 waves).
  int nb = std::max(blocks, 1), dev = 0, nsm = 0, per_sm = 0;
  if (cudaGetDevice(&dev) == cudaSuccess &&
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
      (S == 4   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_prologue<4>, 256, 0)
       : S == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_prologue<2>, 256, 0)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_prologue<0>, 256, 0)) == cudaSuccess &&
      nsm > 0 && per_sm > 0 && nb > nsm * per_sm)
    nb = nb / (nsm * per_sm) * (nsm * per_sm);
  if (S == 4) k_prologue<4><<<nb, 256, 0, st>>>(pv, pst, hi - lo, g0, count, p->low_value, flg);
  else if (S == 2) k_prologue<2><<<nb, 256, 0, st>>>(pv, pst, hi - lo, g0, count, p->low_value, flg);
  else k_prologue<0><<<nb, 256, 0, st>>>(pv, pst, hi - lo, g0, count, p->low_value, flg);
}

// Network inputs of the warm start from the prologue's fitting grids.
n4_status_t enqueue_pool(n4_context *ctx, const Prepared &P, const DescBuf &B, __nv_bfloat16 *d_x, cudaStream_t st) {
  const long long cells = (long long)P.n * kPoolCells;
  const int blocks = (int)std::min<long long>((cells + 255) / 256, (long long)ctx->nsm * 16);
  k_pool_fitgrid<<<blocks, 256, 0, st>>>(B.dp<PoolJob>(P.o_pool), P.n, d_x);
  CK(cudaGetLastError());
  return N4_OK;
}

// The cluster kernel over the queue ord[o0 .. o0 + njobs) with queue counter q.
n4_status_t launch_engine(n4_context *ctx, const n4_params_t *p, const Prepared &P, const DescBuf &B, int o0,
                          int njobs, int q, cudaStream_t st) {
  // one shared-memory layout for every launch of the run, or, with
  // per-sub-batch cluster sizes, the layout of this sub-batch's volumes
  const bool own = !P.subK.empty();
  const int K = own ? P.subK[q] : P.ch.K;
  std::vector<Dims> sub;
  if (own) {
    for (int j = o0; j < o0 + njobs; ++j) sub.push_back(P.dims[j]);
  } else {
    for (int i : P.in_cluster) sub.push_back(P.dims[i]);
  }
  Plan pl = make_plan(p, K, sub, false);
  const int smem = pl.sm_bytes + pl.big_bytes;
  int cap = 0;
  TRY(capacity(ctx, P.ch.nt, K, smem, &cap));
  if (cap < 1) return fail(N4_ERR_TOO_LARGE, "no cluster of this size fits on the device");
  ClusterArgs a{};
  a.pl = pl;
  a.pr = P.pr;
  a.jobs = B.dp<VolJob>(P.o_job);
  a.order = B.dp<int>(P.o_ord) + o0;
  a.njobs = njobs;
  a.queue = B.dp<int>(P.o_q) + 4 * q;
  a.use_tma = 1;
  const int ncl = std::min<int>(cap, njobs);
  if (P.ch.nt == 1024) TRY(launch_cluster_kernel<1024>(ctx, a, K, ncl, smem, st));
  else if (P.ch.nt == 768) TRY(launch_cluster_kernel<768>(ctx, a, K, ncl, smem, st));
  else TRY(launch_cluster_kernel<512>(ctx, a, K, ncl, smem, st));
  return N4_OK;
}

n4_status_t ensure_pipe(n4_context *ctx) {
  if (ctx->pipe[0]) return N4_OK;
  int least = 0, greatest = 0;
  CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  for (int i = 0; i < 5; ++i)
    CK(cudaStreamCreateWithPriority(&ctx->pipe[i], cudaStreamNonBlocking, i < 2 ? greatest : least));
  for (cudaEvent_t &e : ctx->pev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return N4_OK;
}

// A cluster-path batch as P.nsub sub-batches (descriptors already on the
// device; capturable).  Sub-batch k's N4 launch waits only for its own
// prologue and warm start, and runs on stream pipe[k % 2], so that it can
// start on the SMs the previous launch frees while that launch's last volumes
// finish; the prologues and pooling run in order on pipe[2], the encoder
// calls on pipe[4] (sub-batch k's after its pooling, beside sub-batch k+1's
// prologue: measured on 48 uneven volumes, the encoder calls in line with the
// prologues delayed the last N4 launch by 0.4 ms) and the corrections on
// pipe[3], on the SMs the clusters leave free (the N4 streams have the
// higher priority; measured, it makes no difference).  Every kernel reads
// and writes only its own volumes' buffers; st waits for all five streams.
// k_correct over `tiles` tiles from t0 with tile shape `shape`.
n4_status_t launch_correct(int shape, long long tiles, int ncz, cudaStream_t st, const CorrectVol *vols,
                           const long long *tile_starts, int nvol, long long t0, float low, bool log_only = false) {
  if (tiles <= 0) return N4_OK;
  const CorrectShape cs = kCorrectShape[shape];
  const size_t smem = correct_smem_bytes(cs.rows, ncz);
  const unsigned g = (unsigned)tiles;
  if (log_only) {
    if (cs.threads == 512) k_correct<512, true><<<g, 512, smem, st>>>(vols, tile_starts, nvol, t0, low, cs.rows);
    else k_correct<256, true><<<g, 256, smem, st>>>(vols, tile_starts, nvol, t0, low, cs.rows);
  } else {
    if (cs.threads == 512) k_correct<512, false><<<g, 512, smem, st>>>(vols, tile_starts, nvol, t0, low, cs.rows);
    else k_correct<256, false><<<g, 256, smem, st>>>(vols, tile_starts, nvol, t0, low, cs.rows);
  }
  CK(cudaGetLastError());
  return N4_OK;
}

n4_status_t enqueue_pipelined(n4_context *ctx, const n4_params_t *p, const Prepared &P, const DescBuf &B,
                              cudaStream_t st) {
  TRY(ensure_pipe(ctx));
  const int S = P.nsub;
  cudaStream_t side = ctx->pipe[2], corr = ctx->pipe[3], encs = ctx->pipe[4];
  // events: 0 fork, 1 tables, 2+k inputs of sub-batch k ready (prologue, or
  // encoder), 6+k N4 k, 10+i join of pipe[i], 16+k pooling k
  cudaEvent_t *ev = ctx->pev;
  CK(cudaEventRecord(ev[0], st));
  for (cudaStream_t s2 : ctx->pipe) CK(cudaStreamWaitEvent(s2, ev[0], 0));
  const int n = P.n;
  const long long *pst = B.hp<long long>(P.o_pst), *tst = B.hp<long long>(P.o_tst);
  int launches = 0;
  k_axis_tables<<<3 * n, 256, 0, side>>>(B.dp<TableJob>(P.o_tab));
  CK(cudaGetLastError());
  CK(cudaEventRecord(ev[1], side));
  CK(cudaStreamWaitEvent(corr, ev[1], 0));
  ++launches;
  for (int k = 0; k < S; ++k) {
    const int lo = P.sub_lo[k], hi = P.sub_lo[k + 1], nk = hi - lo;
    const long long g0 = pst[lo], g1 = hi < n ? pst[hi] : P.fit_total;
    const int blocks = (int)std::min<long long>((g1 - g0 + 255) / 256, (long long)ctx->nsm * 16);
    launch_prologue(p, P, B, lo, hi, g0, g1 - g0, blocks, side);
    CK(cudaGetLastError());
    ++launches;
    if (p->ShrinkFactor > 1 && (p->flags & N4_FLAG_INPLACE_THRESH)) {
      for (int i = lo; i < hi; ++i) {
        const long long nf = (long long)P.dims[i].FX * P.dims[i].FY * P.dims[i].FZ;
        if (P.rvs[i].im_w) {
          k_threshold_inplace<<<(int)std::min<long long>((nf + 255) / 256, ctx->nsm * 16LL), 256, 0, side>>>(
              P.rvs[i].im_w, P.rvs[i].mask_w, (p->flags & N4_FLAG_MASK_U8) ? 1 : 0, nf, p->low_value);
          CK(cudaGetLastError());
          ++launches;
        }
      }
    }
    if (P.enc) {
      __nv_bfloat16 *x = (__nv_bfloat16 *)ctx->warm_x.p;
      const long long cells = (long long)nk * kPoolCells;
      const int pb = (int)std::min<long long>((cells + 255) / 256, (long long)ctx->nsm * 16);
      k_pool_fitgrid<<<pb, 256, 0, side>>>(B.dp<PoolJob>(P.o_pool) + lo, nk, x + (size_t)lo * kPoolCells);
      CK(cudaGetLastError());
      ++launches;
      CK(cudaEventRecord(ev[16 + k], side));
      CK(cudaStreamWaitEvent(encs, ev[16 + k], 0));
      for (int c0 = lo; c0 < hi; c0 += P.enc_batch) {
        const int nb = std::min(P.enc_batch, hi - c0);
        TRY(n4_encoder_predict(P.enc, x + (size_t)c0 * kPoolCells, nb, ctx->warm_lat.as<float>() + 64 * c0, encs));
        launches += n4_encoder_predict_launches(P.enc, nb);
      }
      CK(cudaEventRecord(ev[2 + k], encs));
    } else {
      CK(cudaEventRecord(ev[2 + k], side));
    }
    // sub-batch k's N4 launch and correction are enqueued right after its
    // inputs, so that the device need not wait for the host to enqueue the
    // later sub-batches' prologues and encoder calls first
    cudaStream_t es = ctx->pipe[k & 1];
    CK(cudaStreamWaitEvent(es, ev[2 + k], 0));
    TRY(launch_engine(ctx, p, P, B, lo, nk, k, es));
    CK(cudaEventRecord(ev[6 + k], es));
    ++launches;
    const long long t0 = tst[lo], t1 = hi < n ? tst[hi] : P.tiles;
    CK(cudaStreamWaitEvent(corr, ev[6 + k], 0));
    TRY(launch_correct(P.corr, t1 - t0, P.NCZ, corr, B.dp<CorrectVol>(P.o_cor) + lo, B.dp<long long>(P.o_tst) + lo,
                       hi - lo, t0, p->low_value));
    ++launches;
  }
  for (int i = 0; i < 5; ++i) {
    CK(cudaEventRecord(ev[10 + i], ctx->pipe[i]));
    CK(cudaStreamWaitEvent(st, ev[10 + i], 0));
  }
  ctx->prof_launches = launches;
  ctx->prof_fit = P.fit_total;
  ctx->prof_full = 0;
  for (const Dims &d : P.dims) ctx->prof_full += (long long)d.FX * d.FY * d.FZ;
  ctx->prof_fit_shape = -1;
  ctx->prof_corr_shape = P.corr;
  return N4_OK;
}

// The launches of a run (descriptors already on the device); capturable.
n4_status_t enqueue_run(n4_context *ctx, const n4_params_t *p, const Prepared &P, const DescBuf &B, cudaStream_t st,
                        bool profile) {
  if (!profile && P.nsub > 1) return enqueue_pipelined(ctx, p, P, B, st);
  const int n = P.n;
  int launches = 0;
  if (profile) TRY(prof_mark(ctx, 0, st));
  {
    ++launches;
    const int blocks = (int)std::min<long long>((P.fit_total + 255) / 256, (long long)ctx->nsm * 16);
    launch_prologue(p, P, B, 0, n, 0, P.fit_total, blocks, st);
    CK(cudaGetLastError());
    if (p->ShrinkFactor > 1 && (p->flags & N4_FLAG_INPLACE_THRESH)) {
      for (int i = 0; i < n; ++i) {
        const long long nf = (long long)P.dims[i].FX * P.dims[i].FY * P.dims[i].FZ;
        if (P.rvs[i].im_w) {
          k_threshold_inplace<<<(int)std::min<long long>((nf + 255) / 256, ctx->nsm * 16LL), 256, 0, st>>>(
              P.rvs[i].im_w, P.rvs[i].mask_w, (p->flags & N4_FLAG_MASK_U8) ? 1 : 0, nf, p->low_value);
          ++launches;
          CK(cudaGetLastError());
        }
      }
    }
  }
  if (P.enc) {
    // learned warm start: pooled fitting grids -> encoder -> first-level lattices
    TRY(enqueue_pool(ctx, P, B, (__nv_bfloat16 *)ctx->warm_x.p, st));
    ++launches;
    for (int c0 = 0; c0 < n; c0 += P.enc_batch) {
      const int nb = std::min(P.enc_batch, n - c0);
      TRY(n4_encoder_predict(P.enc, (const __nv_bfloat16 *)ctx->warm_x.p + (size_t)c0 * kPoolCells, nb,
                             ctx->warm_lat.as<float>() + 64 * c0, st));
      launches += n4_encoder_predict_launches(P.enc, nb);
    }
  }
  if (profile) TRY(prof_mark(ctx, 1, st));
  if (!P.subK.empty()) {
    // per-sub-batch cluster sizes: one launch per sub-batch, in order
    for (int k = 0; k < P.nsub; ++k) {
      TRY(launch_engine(ctx, p, P, B, P.sub_lo[k], P.sub_lo[k + 1] - P.sub_lo[k], k, st));
      ++launches;
    }
  } else if (!P.in_cluster.empty()) {
    TRY(launch_engine(ctx, p, P, B, 0, (int)P.in_cluster.size(), 0, st));
    ++launches;
  }
  for (int i : P.in_grid) {
    VolJob j = B.hp<VolJob>(P.o_job)[i];
    TRY(launch_grid_path(ctx, p, P.pr, P.rvs[i], j, P.ch.nt ? P.ch.nt : 1024, st));
    ++launches;
  }
  if (profile) TRY(prof_mark(ctx, 2, st));
  k_axis_tables<<<3 * n, 256, 0, st>>>(B.dp<TableJob>(P.o_tab));
  CK(cudaGetLastError());
  if (profile) TRY(prof_mark(ctx, 3, st));
  TRY(launch_correct(P.corr, P.tiles, P.NCZ, st, B.dp<CorrectVol>(P.o_cor), B.dp<long long>(P.o_tst), n, 0,
                     p->low_value));
  if (profile) TRY(prof_mark(ctx, 4, st));
  launches += 2;
  ctx->prof_launches = launches;
  ctx->prof_fit = P.fit_total;
  ctx->prof_full = 0;
  for (const Dims &d : P.dims) ctx->prof_full += (long long)d.FX * d.FY * d.FZ;
  ctx->prof_fit_shape = -1;
  ctx->prof_corr_shape = P.corr;
  return N4_OK;
}

// Core of n4_run / n4_run_batched: every pointer is a device pointer.
n4_status_t run_volumes(n4_context *ctx, const n4_params_t *p, const std::vector<RunVol> &rvs, cudaStream_t st,
                        const Choice *forced, n4_encoder_t *enc = nullptr) {
  Prepared P;
  TRY(plan_run(ctx, p, rvs, forced, P, enc));
  Upload u;
  TRY(acquire_slot(ctx, P.bytes, u));
  DescBuf B{u.slot->h, (char *)u.slot->d.p};
  fill_descriptors(ctx, p, P, B);
  TRY(begin_run(ctx, st));
  CK(cudaMemcpyAsync(B.d, B.h, P.bytes, cudaMemcpyHostToDevice, st));
  TRY(enqueue_run(ctx, p, P, B, st, ctx->profiling != 0));
  ctx->prof_valid = ctx->profiling != 0;
  Slot &slot = *u.slot;
  slot.nrep = P.n;
  slot.off_rep = P.o_rep;
  slot.off_flags = P.o_flg;
  slot.path = P.path;
  slot.csize = P.csize;
  slot.perm = P.perm;
  // reports back to the slot's pinned buffer
  CK(cudaMemcpyAsync(B.h + P.o_rep, B.d + P.o_rep, sizeof(n4_report_t) * P.n, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(B.h + P.o_flg, B.d + P.o_flg, 4 * P.n, cudaMemcpyDeviceToHost, st));
  return end_run(ctx, st, u);
}

// The reports of the run that used descriptor slot `slot` (waits for it).
n4_status_t collect_slot(n4_context *ctx, int slot, n4_report_t *out, int n);

n4_status_t collect(n4_context *ctx, n4_report_t *out, int n) {
  if (ctx->last_slot < 0) return fail(N4_ERR_INVALID_ARG, "no run to synchronise with");
  return collect_slot(ctx, ctx->last_slot, out, n);
}

n4_status_t collect_slot(n4_context *ctx, int slot, n4_report_t *out, int n) {
  Slot &s = ctx->slots[slot];
  CK(cudaEventSynchronize(s.ev));
  s.pending = false;
  const n4_report_t *rep = (const n4_report_t *)(s.h + s.off_rep);
  const int *flg = (const int *)(s.h + s.off_flags);
  n4_status_t worst = N4_OK;
  for (int i = 0; i < s.nrep; ++i) {
    n4_report_t r = rep[i];
    if (r.status == -1) r.status = N4_ERR_CUDA;
    if (r.status == N4_OK && flg[i]) r.status = N4_ERR_NONFINITE;
    r.path = s.path[i];
    r.cluster_size = s.csize[i];
    if (out && s.perm[i] < n) out[s.perm[i]] = r;
    if (r.status != N4_OK && worst == N4_OK) worst = (n4_status_t)r.status;
  }
  if (worst != N4_OK) return fail(worst, std::string("volume failed: ") + n4_status_string(worst));
  return N4_OK;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

void n4_params_default(n4_params_t *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->NumberOfHistogramBins = 200;
  p->WienerFilterNoise = 0.01f;
  p->BiasFieldFullWidthAtHalfMaximum = 0.15f;
  p->NumberOfControlPoints_x = p->NumberOfControlPoints_y = p->NumberOfControlPoints_z = 4;
  p->NumberOfFittingLevels = 4;
  for (int l = 0; l < N4_MAX_LEVELS; ++l) p->MaximumNumberOfIterations[l] = 50;
  p->ConvergenceThreshold = 0.001f;
  p->low_value = 10.0f;
  p->ShrinkFactor = 1;
  p->SplineOrder = 3;
  p->FitEpsilon = 1e-3f;
  p->flags = 0;
}

n4_status_t n4_lattice_dims(const n4_params_t *p, unsigned int dims[3], size_t *count) {
  TRY(check_params(p));
  const int x = final_nc(p->NumberOfControlPoints_x, p->NumberOfFittingLevels);
  const int y = final_nc(p->NumberOfControlPoints_y, p->NumberOfFittingLevels);
  const int z = final_nc(p->NumberOfControlPoints_z, p->NumberOfFittingLevels);
  if (dims) { dims[0] = x; dims[1] = y; dims[2] = z; }
  if (count) *count = (size_t)x * y * z;
  return N4_OK;
}

n4_status_t n4_fitting_dims(const n4_params_t *p, unsigned int fx, unsigned int fy, unsigned int fz,
                            unsigned int dims[3]) {
  TRY(check_params(p));
  Dims d;
  TRY(make_dims(p, fx, fy, fz, d));
  if (dims) { dims[0] = (unsigned)d.X; dims[1] = (unsigned)d.Y; dims[2] = (unsigned)d.Z; }
  return N4_OK;
}

const char *n4_status_string(int s) {
  switch (s) {
    case N4_OK: return "ok";
    case N4_ERR_INVALID_ARG: return "invalid argument";
    case N4_ERR_UNSUPPORTED_SPLINE_ORDER: return "unsupported spline order";
    case N4_ERR_EMPTY_MASK: return "empty mask";
    case N4_ERR_OOM: return "out of device memory";
    case N4_ERR_CUDA: return "CUDA error";
    case N4_ERR_TIMEOUT: return "device wait timed out";
    case N4_ERR_NONFINITE: return "non-finite intensity in the mask";
    case N4_ERR_TOO_LARGE: return "request exceeds a supported limit";
    case N4_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char *n4_last_error_string(void) { return g_err.c_str(); }
const char *n4_version(void) { return "n4b200 1.0 (sm_100a)"; }

n4_status_t n4_create(n4_context_t **out, int device) {
  if (!out) return fail(N4_ERR_INVALID_ARG, "ctx is NULL");
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(N4_ERR_NO_DEVICE, "no CUDA device available");
  }
  if (device < 0 || device >= count) return fail(N4_ERR_INVALID_ARG, "bad device index");
  CK(cudaSetDevice(device));
  int major = 0;
  CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  if (major != 10) return fail(N4_ERR_NO_DEVICE, "n4b200 is built for sm_100a (B200) only");
  n4_context *c = new n4_context();
  c->device = device;
  CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
  CK(cudaDeviceGetAttribute(&c->max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  // the largest correction tile: 512 rows of kMaxNcz z control points
  const int corr_smem = (int)correct_smem_bytes(512, kMaxNcz);
  if (cudaFuncSetAttribute(k_correct<256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, corr_smem) != cudaSuccess ||
      cudaFuncSetAttribute(k_correct<512, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, corr_smem) != cudaSuccess ||
      cudaFuncSetAttribute(k_correct<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, corr_smem) != cudaSuccess ||
      cudaFuncSetAttribute(k_correct<512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, corr_smem) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return fail(N4_ERR_CUDA, "cannot raise the correction kernel's shared-memory limit");
  }
  *out = c;
  return N4_OK;
}

n4_status_t n4_destroy(n4_context_t *c) {
  if (!c) return N4_OK;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  for (DevBuf *b : {&c->imlog, &c->tables, &c->big, &c->red, &c->bar, &c->s1, &c->s2, &c->s3, &c->s4,
                    &c->s5, &c->h_im, &c->h_mask, &c->h_out, &c->h_lat, &c->h_bias, &c->h_warm, &c->warm_x,
                    &c->warm_lat, &c->hb})
    b->release();
  for (cudaEvent_t e : c->hev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : c->hclock)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : c->hst)
    if (s) cudaStreamDestroy(s);
  for (Slot &s : c->slots) {
    if (s.h) cudaFreeHost(s.h);
    s.d.release();
    if (s.ev) cudaEventDestroy(s.ev);
  }
  if (c->last_done) cudaEventDestroy(c->last_done);
  for (cudaEvent_t e : c->ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : c->pev)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : c->pipe)
    if (s) cudaStreamDestroy(s);
  delete c;
  return N4_OK;
}

n4_status_t n4_run(n4_context_t *ctx, const n4_params_t *p, const float *d_im, const float *d_mask,
                   unsigned int fx, unsigned int fy, unsigned int fz, float *d_im_normalized, float *d_lattice,
                   float *d_bias_field, const float *d_warm_lattice, void *stream, n4_report_t *report) {
  if (!ctx) return fail(N4_ERR_INVALID_ARG, "ctx is NULL");
  TRY(check_params(p));
  if (!d_im || !d_im_normalized || !d_lattice) return fail(N4_ERR_INVALID_ARG, "NULL input/output pointer");
  RunVol r{};
  TRY(make_dims(p, fx, fy, fz, r.d));
  r.im = d_im;
  r.mask = d_mask;
  r.out = d_im_normalized;
  r.lat = d_lattice;
  r.bias = d_bias_field;
  r.warm = d_warm_lattice;
  if (p->flags & N4_FLAG_INPLACE_THRESH) { r.im_w = const_cast<float *>(d_im); r.mask_w = const_cast<float *>(d_mask); }
  std::vector<RunVol> v{r};
  TRY(run_volumes(ctx, p, v, (cudaStream_t)stream, nullptr));
  if (report) return collect(ctx, report, 1);
  return N4_OK;
}

n4_status_t n4_run_batched(n4_context_t *ctx, const n4_params_t *p, int n, const n4_volume_t *vols, void *stream,
                           n4_report_t *reports) {
  if (!ctx || !vols || n < 1) return fail(N4_ERR_INVALID_ARG, "bad batch");
  TRY(check_params(p));
  std::vector<RunVol> v(n);
  for (int i = 0; i < n; ++i) {
    const n4_volume_t &q = vols[i];
    if (!q.im || !q.im_normalized || !q.lattice) return fail(N4_ERR_INVALID_ARG, "NULL pointer in batch");
    TRY(make_dims(p, q.fx, q.fy, q.fz, v[i].d));
    v[i].im = q.im;
    v[i].mask = q.mask;
    v[i].out = q.im_normalized;
    v[i].lat = q.lattice;
    v[i].bias = q.bias_field;
    v[i].warm = q.warm_lattice;
  }
  TRY(run_volumes(ctx, p, v, (cudaStream_t)stream, nullptr));
  if (reports) return collect(ctx, reports, n);
  return N4_OK;
}

n4_status_t n4_run_batched_warm(n4_context_t *ctx, const n4_params_t *p, int n, const n4_volume_t *vols,
                                n4_encoder_t *enc, void *stream, n4_report_t *reports) {
  if (!ctx || !vols || n < 1 || !enc) return fail(N4_ERR_INVALID_ARG, "bad batch");
  TRY(check_params(p));
  std::vector<RunVol> v(n);
  for (int i = 0; i < n; ++i) {
    const n4_volume_t &q = vols[i];
    if (!q.im || !q.im_normalized || !q.lattice) return fail(N4_ERR_INVALID_ARG, "NULL pointer in batch");
    TRY(make_dims(p, q.fx, q.fy, q.fz, v[i].d));
    v[i].im = q.im;
    v[i].mask = q.mask;
    v[i].out = q.im_normalized;
    v[i].lat = q.lattice;
    v[i].bias = q.bias_field;
    v[i].warm = q.warm_lattice;
  }
  TRY(run_volumes(ctx, p, v, (cudaStream_t)stream, nullptr, enc));
  if (reports) return collect(ctx, reports, n);
  return N4_OK;
}

n4_status_t n4_warm_inputs(n4_context_t *ctx, const n4_params_t *p, int n, const n4_volume_t *vols, void *d_x,
                           void *stream) {
  if (!ctx || !vols || n < 1 || !d_x) return fail(N4_ERR_INVALID_ARG, "bad arguments");
  TRY(check_params(p));
  std::vector<RunVol> v(n);
  for (int i = 0; i < n; ++i) {
    const n4_volume_t &q = vols[i];
    if (!q.im) return fail(N4_ERR_INVALID_ARG, "NULL image in batch");
    TRY(make_dims(p, q.fx, q.fy, q.fz, v[i].d));
    v[i].im = q.im;
    v[i].mask = q.mask;
  }
  // the prologue and the pooling of a run, without the run
  Prepared P;
  const Choice grid_only{true, 0, 1024};
  P.n = n;
  P.rvs = v;
  P.ch = grid_only;
  for (const RunVol &r : v) P.dims.push_back(r.d);
  P.NCX = P.NCY = P.NCZ = 4;
  P.imlog_off.resize(n);
  P.tab_off.assign(n, 0);
  size_t imlog_bytes = 0;
  for (int i = 0; i < n; ++i) {
    P.imlog_off[i] = imlog_bytes;
    imlog_bytes = align_up(imlog_bytes + (size_t)v[i].d.X * v[i].d.Y * v[i].d.Z * 4 + 64, 256);
  }
  TRY(ctx->imlog.ensure(imlog_bytes, "fitting grid"));
  size_t o = 0;
  auto take = [&](size_t b) { size_t r = o; o = align_up(o + b, 16); return r; };
  P.o_pro = take(sizeof(PrologueVol) * n);
  P.o_pst = take(8 * n);
  P.o_flg = take(4 * n);
  P.o_pool = take(sizeof(PoolJob) * n);
  P.bytes = o;
  Upload u;
  TRY(acquire_slot(ctx, P.bytes, u));
  DescBuf B{u.slot->h, (char *)u.slot->d.p};
  long long fit_total = 0;
  for (int i = 0; i < n; ++i) {
    const Dims &d = v[i].d;
    float *il = (float *)(ctx->imlog.as<char>() + P.imlog_off[i]);
    B.hp<PrologueVol>(P.o_pro)[i] = PrologueVol{v[i].im, v[i].mask, nullptr, nullptr, d.FX, d.FY, d.FZ,
                                                (int)p->ShrinkFactor, d.X, d.Y, d.Z, il, fit_total,
                                                (p->flags & N4_FLAG_MASK_U8) ? 1 : 0};
    B.hp<long long>(P.o_pst)[i] = fit_total;
    B.hp<PoolJob>(P.o_pool)[i] = PoolJob{il, d.X, d.Y, d.Z};
    fit_total += (long long)d.X * d.Y * d.Z;
  }
  cudaStream_t st = (cudaStream_t)stream;
  TRY(begin_run(ctx, st));
  CK(cudaMemcpyAsync(B.d, B.h, P.bytes, cudaMemcpyHostToDevice, st));
  const int blocks = (int)std::min<long long>((fit_total + 255) / 256, (long long)ctx->nsm * 16);
  launch_prologue(p, P, B, 0, n, 0, fit_total, blocks, st);
  CK(cudaGetLastError());
  TRY(enqueue_pool(ctx, P, B, (__nv_bfloat16 *)d_x, st));
  u.slot->nrep = 0;
  return end_run(ctx, st, u);
}

n4_status_t n4_autotune(n4_context_t *ctx, const n4_params_t *p, int n, const n4_volume_t *vols, void *stream,
                        n4_tune_report_t *report) {
  if (!ctx || !vols || n < 1) return fail(N4_ERR_INVALID_ARG, "bad batch");
  TRY(check_params(p));
  if (p->flags & (N4_FLAG_FORCE_GRID | N4_FLAG_FORCE_CLUSTER | N4_FLAG_CLUSTER_SIZE(31) | N4_FLAG_CTA_512))
    return fail(N4_ERR_INVALID_ARG,
                "autotuning chooses the path itself: clear the FORCE, cluster-size and thread flags");
  std::vector<RunVol> v(n);
  std::vector<Dims> dims(n);
  for (int i = 0; i < n; ++i) {
    const n4_volume_t &q = vols[i];
    if (!q.im || !q.im_normalized || !q.lattice) return fail(N4_ERR_INVALID_ARG, "NULL pointer in batch");
    TRY(make_dims(p, q.fx, q.fy, q.fz, v[i].d));
    v[i].im = q.im;
    v[i].mask = q.mask;
    v[i].out = q.im_normalized;
    v[i].lat = q.lattice;
    v[i].bias = q.bias_field;
    v[i].warm = q.warm_lattice;
    dims[i] = v[i].d;
  }
  CK(cudaSetDevice(ctx->device));
  // candidates: every cluster size whose per-CTA share of every volume fits,
  // and the whole-GPU path for a single volume
  // a size that leaves more volumes to the whole-GPU path than another size
  // does cannot be faster: only sizes that keep the most volumes on clusters
  size_t most = 0;
  for (int K : {16, 12, 8, 6, 4, 2}) {
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    most = std::max(most, cluster_subset(ctx, p, dims, all, K, nullptr).size());
  }
  std::vector<Choice> cand;
  for (int K : {16, 12, 8, 6, 4, 2}) {
    // the volumes whose per-CTA share fits this cluster size (the others
    // take the whole-GPU path in a run with this choice)
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    const std::vector<int> fit = cluster_subset(ctx, p, dims, all, K, nullptr);
    if (fit.empty() || fit.size() < most) continue;
    std::vector<Dims> sub;
    for (int i : fit) sub.push_back(dims[i]);
    Plan pl = make_plan(p, K, sub, false);
    for (int nt : {1024, 768, 512}) {
      int cap = 0;
      TRY(capacity(ctx, nt, K, pl.sm_bytes + pl.big_bytes, &cap));
      if (cap > 0) cand.push_back(Choice{false, K, nt});
    }
  }
  if (n == 1) {
    cand.push_back(Choice{true, 0, 1024});
    cand.push_back(Choice{true, 0, 768});
    cand.push_back(Choice{true, 0, 512});
  }
  if ((int)cand.size() > N4_TUNE_MAX) cand.resize(N4_TUNE_MAX);
  cudaStream_t st = (cudaStream_t)stream;
  const int saved_prof = ctx->profiling;
  ctx->profiling = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  n4_status_t status = N4_OK;
  n4_tune_report_t rep{};
  int best = -1;
  float best_ms = 0.0f;
  std::vector<n4_report_t> reps(n);
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    status = fail(N4_ERR_CUDA, "cudaEventCreate failed");
  }
  for (size_t c = 0; c < cand.size() && status == N4_OK; ++c) {
    const Choice &ch = cand[c];
    constexpr int kReps = 2;
    n4_status_t s = run_volumes(ctx, p, v, st, &ch);   // untimed first run
    if (s == N4_OK) s = collect(ctx, reps.data(), n);
    if (s == N4_ERR_TOO_LARGE) continue;                // e.g. a grid the device cannot hold
    if (s != N4_OK) { status = s; break; }
    if (cudaEventRecord(e0, st) != cudaSuccess) { status = fail(N4_ERR_CUDA, "cudaEventRecord failed"); break; }
    for (int r = 0; r < kReps && s == N4_OK; ++r) s = run_volumes(ctx, p, v, st, &ch);
    if (s == N4_OK && cudaEventRecord(e1, st) != cudaSuccess) s = fail(N4_ERR_CUDA, "cudaEventRecord failed");
    if (s == N4_OK) s = collect(ctx, reps.data(), n);
    if (s != N4_OK) { status = s; break; }
    // the run's own completion event precedes e1 on the stream: wait for e1
    float ms = 0.0f;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
      status = fail(N4_ERR_CUDA, "event timing failed");
      break;
    }
    ms /= kReps;
    const int k = rep.candidates++;
    rep.cluster_size[k] = ch.grid ? 0 : ch.K;
    rep.threads[k] = ch.nt;
    rep.ms[k] = ms;
    if (best < 0 || ms < best_ms) { best = k; best_ms = ms; }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  ctx->profiling = saved_prof;
  if (status != N4_OK) return status;
  if (best < 0) return fail(N4_ERR_TOO_LARGE, "no execution path fits these volumes");
  rep.chosen = best;
  const int K = rep.cluster_size[best];
  // correction tile shapes on the chosen path: the correction stage's device
  // time (profiling events around it) of one run per shape, the fastest of
  // two runs each
  Choice ch{K == 0, K, rep.threads[best]};
  ctx->profiling = 1;
  for (int k = 0; k < kCorrectShapes && status == N4_OK; ++k) {
    ch.corr = k;
    float ms = 0.0f;
    for (int r = 0; r < 2 && status == N4_OK; ++r) {
      status = run_volumes(ctx, p, v, st, &ch);
      if (status == N4_OK) status = collect(ctx, reps.data(), n);
      n4_timings_t t{};
      if (status == N4_OK) status = n4_last_timings(ctx, &t);
      if (status == N4_OK && (r == 0 || t.stage_ms[3] < ms)) ms = t.stage_ms[3];
    }
    if (status != N4_OK) break;
    rep.corr_rows[k] = kCorrectShape[k].rows;
    rep.corr_threads[k] = kCorrectShape[k].threads;
    rep.corr_ms[k] = ms;
    rep.corr_candidates = k + 1;
    if (k == 0 || ms < rep.corr_ms[rep.corr_chosen]) rep.corr_chosen = k;
  }
  ctx->profiling = 0;
  // overlapped sub-batches (cluster path, batches of two or more): 1 to 4,
  // each timed over two runs on the chosen configuration and tile; then, on
  // the best split and on 4 tapered sub-batches, per-sub-batch cluster sizes
  // (each sub-batch on the smallest size >= a floor that holds its volumes)
  // for every floor that gives sizes not timed yet
  int best_sub = 0, best_taper = 0, best_adapt = 0;
  if (status == N4_OK && K > 0 && n > 1) {
    ch.corr = rep.corr_chosen;
    float best_sub_ms = 0.0f;
    struct SubCand { int S, taper, adapt; };
    std::vector<std::vector<int>> seen;   // split and per-volume cluster sizes of the candidates timed
    // one candidate: an untimed run, then two timed ones; a per-sub-batch
    // candidate whose split and sizes repeat a timed one is skipped
    auto time_split = [&](const SubCand &sc) {
      ch.nsub = sc.S;
      ch.taper = sc.taper;
      ch.adapt = sc.adapt;
      status = run_volumes(ctx, p, v, st, &ch);   // untimed
      if (status == N4_OK) status = collect(ctx, reps.data(), n);
      if (status != N4_OK) return;
      std::vector<int> sig{sc.S, sc.taper};
      for (int i = 0; i < n; ++i) sig.push_back(reps[i].cluster_size);
      for (const auto &q : seen)
        if (sc.adapt > 0 && q == sig) return;
      seen.push_back(sig);
      if (rep.sub_candidates >= N4_TUNE_MAX) return;
      if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        status = fail(N4_ERR_CUDA, "cudaEventCreate failed");
        return;
      }
      if (cudaEventRecord(e0, st) != cudaSuccess) status = fail(N4_ERR_CUDA, "cudaEventRecord failed");
      for (int r = 0; r < 2 && status == N4_OK; ++r) status = run_volumes(ctx, p, v, st, &ch);
      if (status == N4_OK && cudaEventRecord(e1, st) != cudaSuccess) status = fail(N4_ERR_CUDA, "cudaEventRecord failed");
      if (status == N4_OK) status = collect(ctx, reps.data(), n);
      float ms = 0.0f;
      if (status == N4_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        status = fail(N4_ERR_CUDA, "event timing failed");
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      e0 = e1 = nullptr;
      if (status != N4_OK) return;
      const int k = rep.sub_candidates++;
      rep.sub_ms[k] = ms / 2;
      rep.sub_count[k] = sc.S;
      rep.sub_tapered[k] = sc.taper;
      rep.sub_adapt[k] = sc.adapt;
      if (k == 0 || ms / 2 < best_sub_ms) {
        best_sub = sc.S; best_taper = sc.taper; best_adapt = sc.adapt;
        best_sub_ms = ms / 2;
        rep.sub_chosen = k;
      }
    };
    // 1..4 even sub-batches, then 3 and 4 with half-size ends
    for (int S = 1; S <= std::min(kMaxSub, n) && status == N4_OK; ++S) time_split({S, 0, 0});
    if (n >= 4) {
      if (status == N4_OK) time_split({3, 1, 0});
      if (status == N4_OK) time_split({4, 1, 0});
    }
    // per-sub-batch cluster sizes on the best split so far and on 4 tapered
    const int s0 = best_sub, t0 = best_taper;
    for (int fl : {2, 4, 6, 8}) {
      if (status == N4_OK && s0 > 1) time_split({s0, t0, fl});
      if (status == N4_OK && n >= 4 && !(s0 == 4 && t0 == 1)) time_split({4, 1, fl});
    }
  }
  ctx->profiling = saved_prof;
  ctx->prof_valid = false;
  if (status != N4_OK) return status;
  ctx->tune[tune_key(p, dims)] =
      TuneVal{K == 0 ? 1 : 0, K, rep.threads[best], rep.corr_chosen, best_sub, best_taper, best_adapt};
  if (report) *report = rep;
  return N4_OK;
}

n4_status_t n4_set_profiling(n4_context_t *ctx, int enable) {
  if (!ctx) return fail(N4_ERR_INVALID_ARG, "ctx is NULL");
  ctx->profiling = enable ? 1 : 0;
  ctx->prof_valid = false;
  return N4_OK;
}

n4_status_t n4_last_timings(n4_context_t *ctx, n4_timings_t *t) {
  if (!ctx || !t) return fail(N4_ERR_INVALID_ARG, "NULL argument");
  if (!ctx->prof_valid) return fail(N4_ERR_INVALID_ARG, "no profiled run");
  CK(cudaEventSynchronize(ctx->ev[4]));
  for (int k = 0; k < 4; ++k) CK(cudaEventElapsedTime(&t->stage_ms[k], ctx->ev[k], ctx->ev[k + 1]));
  t->launches = ctx->prof_launches;
  t->fit_voxels = ctx->prof_fit;
  t->full_voxels = ctx->prof_full;
  const int fs = ctx->prof_fit_shape, cs = ctx->prof_corr_shape;
  t->fit_rows = fs >= 0 ? kFitShape[fs].rows : -1;
  t->fit_step = fs >= 0 ? kFitShape[fs].step : -1;
  t->fit_depth = fs >= 0 ? kFitShape[fs].depth : -1;
  t->correct_rows = cs >= 0 ? kCorrectShape[cs].rows : -1;
  t->correct_threads = cs >= 0 ? kCorrectShape[cs].threads : -1;
  return N4_OK;
}

n4_status_t n4_sync(n4_context_t *ctx, n4_report_t *reports, int n) {
  if (!ctx) return fail(N4_ERR_INVALID_ARG, "ctx is NULL");
  return collect(ctx, reports, n);
}

n4_status_t n4_run_host(n4_context_t *ctx, const n4_params_t *p, const float *h_im, const float *h_mask,
                        unsigned int fx, unsigned int fy, unsigned int fz, float *h_im_normalized, float *h_lattice,
                        float *h_bias_field, const float *h_warm_lattice, n4_report_t *report) {
  if (!ctx) return fail(N4_ERR_INVALID_ARG, "ctx is NULL");
  TRY(check_params(p));
  if (!h_im || !h_im_normalized || !h_lattice) return fail(N4_ERR_INVALID_ARG, "NULL input/output pointer");
  Dims d;
  TRY(make_dims(p, fx, fy, fz, d));
  CK(cudaSetDevice(ctx->device));
  size_t nlat = 0;
  TRY(n4_lattice_dims(p, nullptr, &nlat));
  const size_t nv = (size_t)fx * fy * fz;
  const size_t nwarm = (size_t)p->NumberOfControlPoints_x * p->NumberOfControlPoints_y * p->NumberOfControlPoints_z;
  TRY(ctx->h_im.ensure(nv * 4, "input"));
  TRY(ctx->h_out.ensure(nv * 4, "output"));
  TRY(ctx->h_lat.ensure(nlat * 4, "lattice"));
  const size_t mask_bytes = nv * ((p->flags & N4_FLAG_MASK_U8) ? 1 : 4);
  if (h_mask) TRY(ctx->h_mask.ensure(mask_bytes, "mask"));
  if (h_bias_field) TRY(ctx->h_bias.ensure(nv * 4, "bias"));
  if (h_warm_lattice) TRY(ctx->h_warm.ensure(nwarm * 4, "warm lattice"));
  cudaStream_t st = nullptr;
  CK(cudaMemcpyAsync(ctx->h_im.p, h_im, nv * 4, cudaMemcpyHostToDevice, st));
  if (h_mask) CK(cudaMemcpyAsync(ctx->h_mask.p, h_mask, mask_bytes, cudaMemcpyHostToDevice, st));
  if (h_warm_lattice) CK(cudaMemcpyAsync(ctx->h_warm.p, h_warm_lattice, nwarm * 4, cudaMemcpyHostToDevice, st));
  n4_report_t rep;
  n4_status_t s = n4_run(ctx, p, ctx->h_im.as<float>(), h_mask ? ctx->h_mask.as<float>() : nullptr, fx, fy, fz,
                         ctx->h_out.as<float>(), ctx->h_lat.as<float>(), h_bias_field ? ctx->h_bias.as<float>() : nullptr,
                         h_warm_lattice ? ctx->h_warm.as<float>() : nullptr, st, &rep);
  if (report) *report = rep;
  if (s != N4_OK && s != N4_ERR_EMPTY_MASK && s != N4_ERR_NONFINITE) return s;
  CK(cudaMemcpyAsync(h_im_normalized, ctx->h_out.p, nv * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h_lattice, ctx->h_lat.p, nlat * 4, cudaMemcpyDeviceToHost, st));
  if (h_bias_field) CK(cudaMemcpyAsync(h_bias_field, ctx->h_bias.p, nv * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return s;
}

n4_status_t n4_run_batched_host(n4_context_t *ctx, const n4_params_t *p, int n, const n4_volume_t *vols, int per,
                                n4_encoder_t *enc, n4_report_t *reports, float *device_ms) {
  if (!ctx || !vols || n < 1 || per < 0) return fail(N4_ERR_INVALID_ARG, "bad batch");
  TRY(check_params(p));
  CK(cudaSetDevice(ctx->device));
  size_t nlat = 0;
  TRY(n4_lattice_dims(p, nullptr, &nlat));
  const size_t nwarm = (size_t)p->NumberOfControlPoints_x * p->NumberOfControlPoints_y * p->NumberOfControlPoints_z;
  const size_t mask_b = (p->flags & N4_FLAG_MASK_U8) ? 1 : 4;
  size_t vmax = 0;
  bool any_mask = false, any_bias = false, any_warm = false;
  for (int i = 0; i < n; ++i) {
    const n4_volume_t &q = vols[i];
    if (!q.im || !q.im_normalized || !q.lattice) return fail(N4_ERR_INVALID_ARG, "NULL pointer in batch");
    Dims d;
    TRY(make_dims(p, q.fx, q.fy, q.fz, d));
    vmax = std::max(vmax, (size_t)q.fx * q.fy * q.fz);
    any_mask |= q.mask != nullptr;
    any_bias |= q.bias_field != nullptr;
    any_warm |= q.warm_lattice != nullptr;
  }
  if (enc && any_warm) return fail(N4_ERR_INVALID_ARG, "warm lattices are predicted by the encoder: pass none");
  if (per == 0) per = std::min(n, 8);
  per = std::min(per, n);
  // one staging slot per lane: per volumes of input, mask, output, bias, lattice, warm lattice
  auto al = [](size_t b) { return align_up(b, 256); };
  const size_t vin = al(vmax * 4), vmask = any_mask ? al(vmax * mask_b) : 0, vout = al(vmax * 4),
               vbias = any_bias ? al(vmax * 4) : 0, vlat = al(nlat * 4), vwarm = any_warm ? al(nwarm * 4) : 0;
  const size_t per_vol = vin + vmask + vout + vbias + vlat + vwarm;
  constexpr int L = kHostLanes;
  TRY(ctx->hb.ensure((size_t)L * per * per_vol, "host-batch staging"));
  for (cudaStream_t &s2 : ctx->hst)
    if (!s2) CK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
  for (cudaEvent_t &e : ctx->hev)
    if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (cudaEvent_t &e : ctx->hclock)
    if (!e) CK(cudaEventCreate(&e));
  // every lane starts after the context's earlier work and after the clock
  cudaStream_t lane0 = ctx->hst[0];
  if (ctx->last_done && ctx->last_slot >= 0) CK(cudaStreamWaitEvent(lane0, ctx->last_done, 0));
  CK(cudaEventRecord(ctx->hclock[0], lane0));
  for (int l = 1; l < L; ++l) CK(cudaStreamWaitEvent(ctx->hst[l], ctx->hclock[0], 0));
  const int nsb = (n + per - 1) / per;
  std::vector<int> run_slot(nsb, -1);
  n4_status_t worst = N4_OK;
  auto harvest = [&](int k) -> n4_status_t {
    if (k < 0 || run_slot[k] < 0) return N4_OK;
    const int lo = k * per, cnt = std::min(per, n - lo);
    n4_status_t st = collect_slot(ctx, run_slot[k], reports ? reports + lo : nullptr, cnt);
    run_slot[k] = -1;
    if (st == N4_ERR_CUDA || st == N4_ERR_TIMEOUT) return st;
    if (st != N4_OK && worst == N4_OK) worst = st;
    return N4_OK;
  };
  for (int k = 0; k < nsb; ++k) {
    // sub-batch k on lane k % L: its uploads, its run and its downloads in
    // that lane's stream order (so the lane's staging slot is free again once
    // its previous downloads are done); the runs of successive sub-batches
    // are ordered by the context (each waits for the previous run, not for
    // its downloads), and the copies of the other lanes overlap them
    const int l = k % L, lo = k * per, cnt = std::min(per, n - lo);
    cudaStream_t st = ctx->hst[l];
    char *base = (char *)ctx->hb.p + (size_t)l * per * per_vol;
    std::vector<RunVol> rvs(cnt);
    for (int j = 0; j < cnt; ++j) {
      const n4_volume_t &q = vols[lo + j];
      const size_t nv = (size_t)q.fx * q.fy * q.fz;
      char *v = base + (size_t)j * per_vol;
      float *im = (float *)v, *mk = (float *)(v + vin), *out = (float *)(v + vin + vmask),
            *bias = (float *)(v + vin + vmask + vout), *lat = (float *)(v + vin + vmask + vout + vbias),
            *warm = (float *)(v + vin + vmask + vout + vbias + vlat);
      CK(cudaMemcpyAsync(im, q.im, nv * 4, cudaMemcpyHostToDevice, st));
      if (q.mask) CK(cudaMemcpyAsync(mk, q.mask, nv * mask_b, cudaMemcpyHostToDevice, st));
      if (q.warm_lattice) CK(cudaMemcpyAsync(warm, q.warm_lattice, nwarm * 4, cudaMemcpyHostToDevice, st));
      RunVol &r = rvs[j];
      TRY(make_dims(p, q.fx, q.fy, q.fz, r.d));
      r.im = im;
      r.mask = q.mask ? mk : nullptr;
      r.out = out;
      r.lat = lat;
      r.bias = q.bias_field ? bias : nullptr;
      r.warm = q.warm_lattice ? warm : nullptr;
    }
    // the run's descriptor slot is the one run k - kSlots used: take that
    // run's reports first
    TRY(harvest(k - kSlots));
    TRY(run_volumes(ctx, p, rvs, st, nullptr, enc));
    run_slot[k] = ctx->last_slot;
    for (int j = 0; j < cnt; ++j) {
      const n4_volume_t &q = vols[lo + j];
      const size_t nv = (size_t)q.fx * q.fy * q.fz;
      const RunVol &r = rvs[j];
      CK(cudaMemcpyAsync(q.im_normalized, r.out, nv * 4, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(q.lattice, r.lat, nlat * 4, cudaMemcpyDeviceToHost, st));
      if (q.bias_field) CK(cudaMemcpyAsync(q.bias_field, r.bias, nv * 4, cudaMemcpyDeviceToHost, st));
    }
  }
  // join the lanes on lane 0
  for (int l = 1; l < L; ++l) {
    CK(cudaEventRecord(ctx->hev[l], ctx->hst[l]));
    CK(cudaStreamWaitEvent(lane0, ctx->hev[l], 0));
  }
  CK(cudaEventRecord(ctx->hclock[1], lane0));
  // later work of this context waits for the downloads
  CK(cudaEventRecord(ctx->last_done, lane0));
  ctx->last_stream = lane0;
  for (int k = std::max(0, nsb - kSlots); k < nsb; ++k) TRY(harvest(k));
  CK(cudaEventSynchronize(ctx->hclock[1]));
  if (device_ms) CK(cudaEventElapsedTime(device_ms, ctx->hclock[0], ctx->hclock[1]));
  if (worst != N4_OK) return fail(worst, std::string("volume failed: ") + n4_status_string(worst));
  return N4_OK;
}

}  // extern "C"

struct n4_batch_graph {
  n4_context *ctx = nullptr;
  Prepared P;
  n4_params_t params{};
  char *h_desc = nullptr, *d_desc = nullptr, *h_rep = nullptr;
  size_t rep_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t done = nullptr;
  bool launched = false;
  int launches = 0;   // kernel launches recorded in the graph
};

static void graph_free(n4_batch_graph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->done) cudaEventDestroy(g->done);
  if (g->h_desc) cudaFreeHost(g->h_desc);
  if (g->h_rep) cudaFreeHost(g->h_rep);
  if (g->d_desc) cudaFree(g->d_desc);
  delete g;
}

extern "C" {

static n4_status_t graph_create(n4_context_t *ctx, const n4_params_t *p, int n, const n4_volume_t *vols,
                                n4_encoder_t *enc, n4_batch_graph_t **out) {
  if (!ctx || !vols || n < 1 || !out) return fail(N4_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  TRY(check_params(p));
  CK(cudaSetDevice(ctx->device));
  std::vector<RunVol> v(n);
  for (int i = 0; i < n; ++i) {
    const n4_volume_t &q = vols[i];
    if (!q.im || !q.im_normalized || !q.lattice) return fail(N4_ERR_INVALID_ARG, "NULL pointer in batch");
    TRY(make_dims(p, q.fx, q.fy, q.fz, v[i].d));
    v[i].im = q.im; v[i].mask = q.mask; v[i].out = q.im_normalized; v[i].lat = q.lattice;
    v[i].bias = q.bias_field; v[i].warm = q.warm_lattice;
  }
  n4_batch_graph *g = new n4_batch_graph();
  g->ctx = ctx;
  g->params = *p;
  n4_status_t s = plan_run(ctx, p, v, nullptr, g->P, enc);
  if (s != N4_OK) { graph_free(g); return s; }
  const Prepared &P = g->P;
  g->rep_bytes = P.o_flg + 4 * (size_t)P.n - P.o_rep;
  cudaError_t e;
  if ((e = cudaMallocHost((void **)&g->h_desc, P.bytes)) || (e = cudaMallocHost((void **)&g->h_rep, g->rep_bytes)) ||
      (e = cudaMalloc((void **)&g->d_desc, P.bytes)) || (e = cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming))) {
    graph_free(g);
    return fail(N4_ERR_OOM, cudaGetErrorString(e));
  }
  std::memset(g->h_desc, 0, P.bytes);
  std::memset(g->h_rep, 0, g->rep_bytes);
  DescBuf B{g->h_desc, g->d_desc};
  fill_descriptors(ctx, p, g->P, B);
  if (P.nsub > 1 && (s = ensure_pipe(ctx)) != N4_OK) { graph_free(g); return s; }
  cudaStream_t cs;
  CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  s = N4_OK;
  if ((e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed)) != cudaSuccess) {
    s = fail(N4_ERR_CUDA, cudaGetErrorString(e));
  } else {
    // every replay starts from the pristine descriptors (reports, queue counter)
    if ((e = cudaMemcpyAsync(B.d, B.h, P.bytes, cudaMemcpyHostToDevice, cs)) != cudaSuccess)
      s = fail(N4_ERR_CUDA, cudaGetErrorString(e));
    if (s == N4_OK) s = enqueue_run(ctx, p, P, B, cs, false);
    g->launches = ctx->prof_launches;
    if (s == N4_OK &&
        (e = cudaMemcpyAsync(g->h_rep, B.d + P.o_rep, g->rep_bytes, cudaMemcpyDeviceToHost, cs)) != cudaSuccess)
      s = fail(N4_ERR_CUDA, cudaGetErrorString(e));
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(cs, &graph);
    if (s == N4_OK && e != cudaSuccess) s = fail(N4_ERR_CUDA, cudaGetErrorString(e));
    g->graph = graph;
    if (s == N4_OK && (e = cudaGraphInstantiate(&g->exec, graph, 0)) != cudaSuccess)
      s = fail(N4_ERR_CUDA, cudaGetErrorString(e));
  }
  cudaStreamDestroy(cs);
  cudaGetLastError();
  if (s != N4_OK) { graph_free(g); return s; }
  *out = g;
  return N4_OK;
}

n4_status_t n4_batch_graph_create(n4_context_t *ctx, const n4_params_t *p, int n, const n4_volume_t *vols,
                                  n4_batch_graph_t **out) {
  return graph_create(ctx, p, n, vols, nullptr, out);
}

n4_status_t n4_batch_graph_create_warm(n4_context_t *ctx, const n4_params_t *p, int n, const n4_volume_t *vols,
                                       n4_encoder_t *enc, n4_batch_graph_t **out) {
  if (!enc) return fail(N4_ERR_INVALID_ARG, "encoder is NULL");
  return graph_create(ctx, p, n, vols, enc, out);
}

n4_status_t n4_batch_graph_launch(n4_batch_graph_t *g, void *stream) {
  if (!g) return fail(N4_ERR_INVALID_ARG, "graph is NULL");
  CK(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  CK(cudaEventRecord(g->done, (cudaStream_t)stream));
  g->launched = true;
  return N4_OK;
}

n4_status_t n4_batch_graph_sync(n4_batch_graph_t *g, n4_report_t *reports, int n) {
  if (!g) return fail(N4_ERR_INVALID_ARG, "graph is NULL");
  if (!g->launched) return fail(N4_ERR_INVALID_ARG, "graph not launched");
  CK(cudaEventSynchronize(g->done));
  const Prepared &P = g->P;
  const n4_report_t *rep = (const n4_report_t *)g->h_rep;
  const int *flg = (const int *)(g->h_rep + (P.o_flg - P.o_rep));
  n4_status_t worst = N4_OK;
  for (int i = 0; i < P.n; ++i) {
    n4_report_t r = rep[i];
    if (r.status == -1) r.status = N4_ERR_CUDA;
    if (r.status == N4_OK && flg[i]) r.status = N4_ERR_NONFINITE;
    r.path = P.path[i];
    r.cluster_size = P.csize[i];
    if (reports && P.perm[i] < n) reports[P.perm[i]] = r;
    if (r.status != N4_OK && worst == N4_OK) worst = (n4_status_t)r.status;
  }
  if (worst != N4_OK) return fail(worst, std::string("volume failed: ") + n4_status_string(worst));
  return N4_OK;
}

n4_status_t n4_batch_graph_info(const n4_batch_graph_t *g, int *kernel_launches, int *sub_batches) {
  if (!g) return fail(N4_ERR_INVALID_ARG, "graph is NULL");
  if (kernel_launches) *kernel_launches = g->launches;
  if (sub_batches) *sub_batches = g->P.nsub;
  return N4_OK;
}

n4_status_t n4_batch_graph_destroy(n4_batch_graph_t *g) {
  if (!g) return N4_OK;
  cudaSetDevice(g->ctx->device);
  if (g->launched) cudaEventSynchronize(g->done);
  graph_free(g);
  return N4_OK;
}

// ---------------------------------------------------------------- components
// Whether fit shape `k` can run on this field: 8-voxel (32-byte) register
// steps need Z % 8 == 0 and field and mask on 32-byte boundaries, 4-voxel
// (16-byte) steps Z % 4 == 0 and 16-byte boundaries, both a z table within
// the default 48 KB of shared memory (Z <= 1024); the scalar kernel runs on
// anything.  Every shape computes the same sums in the same order (bitwise).
static bool fit_shape_ok(int k, const float *field, const float *mask, int Z) {
  const uintptr_t al = (uintptr_t)field | (uintptr_t)mask;
  const FitShape f = kFitShape[k];
  if (f.step == 16) return Z % 16 == 0 && Z <= kFitZMaxD && (al & 63u) == 0;
  if (f.step == 8) return Z % 8 == 0 && Z <= kFitZMaxD && (al & 31u) == 0;
  if (f.step == 4) return Z % 4 == 0 && Z <= kFitZMaxD && (al & 15u) == 0;
  return true;
}

static int fit_default_shape(const float *field, const float *mask, int Z) {
  if (fit_shape_ok(kFitDefault8, field, mask, Z)) return kFitDefault8;
  if (fit_shape_ok(kFitDefault4, field, mask, Z)) return kFitDefault4;
  return kFitScalar;
}

// Component autotuner keys: field and lattice sizes (and, for the fit, the
// alignment class of field and mask, which decides the shapes that can run).
static std::vector<int> fit_key(unsigned fx, unsigned fy, unsigned fz, unsigned nx, unsigned ny, unsigned nz,
                                const float *field, const float *mask) {
  const uintptr_t al = (uintptr_t)field | (uintptr_t)mask;
  const int cls = (al & 63u) == 0 ? 64 : ((al & 31u) == 0 ? 32 : ((al & 15u) == 0 ? 16 : 4));
  return {(int)fx, (int)fy, (int)fz, (int)nx, (int)ny, (int)nz, cls};
}
static std::vector<int> eval_key(unsigned fx, unsigned fy, unsigned fz, unsigned nx, unsigned ny, unsigned nz) {
  return {(int)fx, (int)fy, (int)fz, (int)nx, (int)ny, (int)nz};
}

extern "C++" {
template <int S, int D, int R>
static void fit_rows_as(const float *field, const float *mask, long long rows, int Z, const Axis &az, float *t1n,
                        float *t1d, cudaStream_t st) {
  k_fit_rows_v5<S, D, R><<<(unsigned)((rows + R - 1) / R), R, kFitTableBytes(Z), st>>>(field, mask, rows, Z, az, t1n,
                                                                                      t1d);
}
}  // extern "C++"

// z contraction of a standalone fit with shape `k` (fit_shape_ok must hold).
static void launch_fit_rows(int k, const float *field, const float *mask, long long rows, int Z, const Axis &az,
                            float *t1n, float *t1d, cudaStream_t st) {
  switch (k) {
    case 0: fit_rows_as<8, 3, 64>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 1: fit_rows_as<8, 2, 64>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 2: fit_rows_as<8, 4, 64>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 3: fit_rows_as<8, 3, 32>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 4: fit_rows_as<8, 3, 128>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 5: fit_rows_as<8, 2, 128>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 6: fit_rows_as<4, 6, 64>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 7: fit_rows_as<4, 4, 64>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 8: fit_rows_as<4, 6, 128>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 10: fit_rows_as<16, 2, 64>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 11: fit_rows_as<16, 2, 32>(field, mask, rows, Z, az, t1n, t1d, st); break;
    case 12: fit_rows_as<16, 2, 128>(field, mask, rows, Z, az, t1n, t1d, st); break;
    default:
      k_fit_rows<<<(unsigned)((rows + kFitRows - 1) / kFitRows), kFitRows, 0, st>>>(field, mask, rows, Z, az, t1n,
                                                                                     t1d);
  }
}
static_assert(kFitShapes == 13, "launch_fit_rows covers every fit shape");

// Sizes a standalone fit accepts: every extent below 2^31 (the kernels take
// them as int), at most 2^36 field voxels and 4096 control points per axis,
// so that the row and plane sums (fx*fy*ncpt_z, fx*ncpt_y*ncpt_z floats)
// cannot wrap.
static n4_status_t check_fit_sizes(unsigned ncpt_x, unsigned ncpt_y, unsigned ncpt_z, unsigned fx, unsigned fy,
                                   unsigned fz) {
  if (ncpt_x < 4 || ncpt_y < 4 || ncpt_z < 4 || !fx || !fy || !fz) return fail(N4_ERR_INVALID_ARG, "bad sizes");
  if (fx > 0x7fffffffu || fy > 0x7fffffffu || fz > 0x7fffffffu) return fail(N4_ERR_TOO_LARGE, "extent >= 2^31");
  if ((unsigned long long)fx * fy * fz >= (1ull << 36)) return fail(N4_ERR_TOO_LARGE, "field too large");
  if (ncpt_x > 4096 || ncpt_y > 4096 || ncpt_z > 4096)
    return fail(N4_ERR_TOO_LARGE, "more than 4096 control points along an axis");
  return N4_OK;
}

static n4_status_t component_tables(n4_context_t *ctx, unsigned fx, unsigned fy, unsigned fz, unsigned nx, unsigned ny,
                                    unsigned nz, cudaStream_t st, Axis &ax, Axis &ay, Axis &az) {
  const size_t bx = align_up(axis_bytes(fx, nx - 3), 256), by = align_up(axis_bytes(fy, ny - 3), 256),
               bz = align_up(axis_bytes(fz, nz - 3), 256);
  TRY(ctx->s5.ensure(bx + by + bz + sizeof(TableJob) * 3 + 256, "tables"));
  char *base = ctx->s5.as<char>();
  TableJob tj[3] = {{base, (int)fx, (int)nx}, {base + bx, (int)fy, (int)ny}, {base + bx + by, (int)fz, (int)nz}};
  Upload u;
  TRY(acquire_slot(ctx, sizeof(tj), u));
  std::memcpy(u.h(), tj, sizeof(tj));
  TRY(begin_run(ctx, st));
  CK(cudaMemcpyAsync(u.slot->d.p, u.slot->h, sizeof(tj), cudaMemcpyHostToDevice, st));
  k_axis_tables<<<3, 256, 0, st>>>(u.dp<TableJob>(0));
  CK(cudaGetLastError());
  u.slot->nrep = 0;
  TRY(end_run(ctx, st, u));
  ax = axis_at(base, fx, nx);
  ay = axis_at(base + bx, fy, ny);
  az = axis_at(base + bx + by, fz, nz);
  return N4_OK;
}

n4_status_t n4_fit_bspline3d(n4_context_t *ctx, const float *d_field, const float *d_mask, unsigned int ncpt_x,
                             unsigned int ncpt_y, unsigned int ncpt_z, unsigned int fx, unsigned int fy,
                             unsigned int fz, float eps, int zero_den, float *d_lattice, void *stream) {
  if (!ctx || !d_field || !d_lattice) return fail(N4_ERR_INVALID_ARG, "NULL pointer");
  TRY(check_fit_sizes(ncpt_x, ncpt_y, ncpt_z, fx, fy, fz));
  cudaStream_t st = (cudaStream_t)stream;
  Axis ax, ay, az;
  TRY(component_tables(ctx, fx, fy, fz, ncpt_x, ncpt_y, ncpt_z, st, ax, ay, az));
  const size_t t1 = (size_t)fx * fy * ncpt_z, t2 = (size_t)fx * ncpt_y * ncpt_z;
  TRY(ctx->s1.ensure(t1 * 8, "fit rows"));
  TRY(ctx->s2.ensure(t2 * 8, "fit planes"));
  float *t1n = ctx->s1.as<float>(), *t1d = t1n + t1, *t2n = ctx->s2.as<float>(), *t2d = t2n + t2;
  const int gb = ctx->nsm * 8;
  const long long rows = (long long)fx * fy;
  const bool prof = ctx->profiling != 0;
  int shape = fit_default_shape(d_field, d_mask, (int)fz);
  auto it = ctx->fit_tune.find(fit_key(fx, fy, fz, ncpt_x, ncpt_y, ncpt_z, d_field, d_mask));
  if (it != ctx->fit_tune.end() && fit_shape_ok(it->second, d_field, d_mask, (int)fz)) shape = it->second;
  if (prof) TRY(prof_mark(ctx, 0, st));
  launch_fit_rows(shape, d_field, d_mask, rows, fz, az, t1n, t1d, st);
  if (prof) TRY(prof_mark(ctx, 1, st));
  k_fit_planes<<<(int)std::min<size_t>((t2 + 255) / 256, gb), 256, 0, st>>>(t1n, t1d, fx, fy, ay, ncpt_z, t2n, t2d);
  if (prof) TRY(prof_mark(ctx, 2, st));
  const int nlat = ncpt_x * ncpt_y * ncpt_z;
  k_fit_final<<<(nlat + 255) / 256, 256, 0, st>>>(t2n, t2d, fx, ax, ncpt_y, ncpt_z, eps, zero_den, d_lattice);
  if (prof) { TRY(prof_mark(ctx, 3, st)); TRY(prof_mark(ctx, 4, st)); }
  CK(cudaGetLastError());
  ctx->prof_launches = 4;
  ctx->prof_fit = (long long)fx * fy * fz;
  ctx->prof_full = 0;
  ctx->prof_fit_shape = shape;
  ctx->prof_corr_shape = -1;
  ctx->prof_valid = prof;
  return N4_OK;
}

n4_status_t n4_evaluate_bspline3d(n4_context_t *ctx, const float *d_lattice, unsigned int ncpt_x, unsigned int ncpt_y,
                                  unsigned int ncpt_z, unsigned int fx, unsigned int fy, unsigned int fz,
                                  float *d_fitted, void *stream) {
  if (!ctx || !d_lattice || !d_fitted) return fail(N4_ERR_INVALID_ARG, "NULL pointer");
  if (ncpt_x < 4 || ncpt_y < 4 || ncpt_z < 4 || !fx || !fy || !fz) return fail(N4_ERR_INVALID_ARG, "bad sizes");
  if (ncpt_z > (unsigned)kMaxNcz) return fail(N4_ERR_TOO_LARGE, "at most 64 control points along z");
  cudaStream_t st = (cudaStream_t)stream;
  Axis ax, ay, az;
  if (ctx->profiling) TRY(prof_mark(ctx, 0, st));
  TRY(component_tables(ctx, fx, fy, fz, ncpt_x, ncpt_y, ncpt_z, st, ax, ay, az));
  CorrectVol cv{nullptr, d_fitted, nullptr, d_lattice, (char *)ax.s, (char *)ay.s, (char *)az.s,
                (int)fx, (int)fy, (int)fz, (int)ncpt_x, (int)ncpt_y, (int)ncpt_z, 0,
                vec4_ok((int)fz, nullptr, d_fitted, nullptr)};
  int shape = kCorrectDefault;
  auto it = ctx->eval_tune.find(eval_key(fx, fy, fz, ncpt_x, ncpt_y, ncpt_z));
  if (it != ctx->eval_tune.end()) shape = it->second;
  const long long rt = kCorrectShape[shape].rows;
  const long long tiles = ((long long)fx * fy + rt - 1) / rt;
  Upload u;
  TRY(acquire_slot(ctx, sizeof(cv) + 16, u));
  std::memcpy(u.h(), &cv, sizeof(cv));
  TRY(begin_run(ctx, st));
  CK(cudaMemcpyAsync(u.slot->d.p, u.slot->h, sizeof(cv) + 16, cudaMemcpyHostToDevice, st));
  const size_t so = align_up(sizeof(cv), 16);
  const bool prof = ctx->profiling != 0;
  if (prof) TRY(prof_mark(ctx, 1, st));
  TRY(launch_correct(shape, tiles, (int)ncpt_z, st, u.dp<CorrectVol>(0), u.dp<long long>(so), 1, 0, 0.0f, true));
  if (prof) { TRY(prof_mark(ctx, 2, st)); TRY(prof_mark(ctx, 3, st)); TRY(prof_mark(ctx, 4, st)); }
  ctx->prof_launches = 2;
  ctx->prof_fit = 0;
  ctx->prof_full = (long long)fx * fy * fz;
  ctx->prof_fit_shape = -1;
  ctx->prof_corr_shape = shape;
  ctx->prof_valid = prof;
  u.slot->nrep = 0;
  return end_run(ctx, st, u);
}

n4_status_t n4_autotune_components(n4_context_t *ctx, const float *d_field, const float *d_mask, unsigned int ncpt_x,
                                   unsigned int ncpt_y, unsigned int ncpt_z, unsigned int fx, unsigned int fy,
                                   unsigned int fz, float *d_lattice, float *d_out, void *stream,
                                   n4_component_tune_t *report) {
  if (!ctx || !d_field || !d_lattice || !d_out) return fail(N4_ERR_INVALID_ARG, "NULL pointer");
  TRY(check_fit_sizes(ncpt_x, ncpt_y, ncpt_z, fx, fy, fz));
  if (ncpt_z > (unsigned)kMaxNcz) return fail(N4_ERR_TOO_LARGE, "at most 64 control points along z");
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  Axis ax, ay, az;
  TRY(component_tables(ctx, fx, fy, fz, ncpt_x, ncpt_y, ncpt_z, st, ax, ay, az));
  const size_t t1 = (size_t)fx * fy * ncpt_z;
  TRY(ctx->s1.ensure(t1 * 8, "fit rows"));
  float *t1n = ctx->s1.as<float>(), *t1d = t1n + t1;
  // a 256 MiB buffer read before every timed launch evicts its inputs from L2
  const size_t evict_bytes = 256u << 20;
  TRY(ctx->s4.ensure(evict_bytes + 256, "L2 eviction buffer"));
  CK(cudaMemsetAsync(ctx->s4.p, 0, evict_bytes + 256, st));
  const float4 *ev_buf = (const float4 *)ctx->s4.p;
  float *sink = (float *)((char *)ctx->s4.p + evict_bytes);
  const long long rows = (long long)fx * fy;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    return fail(N4_ERR_CUDA, "cudaEventCreate failed");
  }
  // time `launch` three times after an eviction each; the fastest in ms
  auto timed = [&](auto &&launch, float *ms) -> n4_status_t {
    launch();   // warm-up (and the first launch of the kernel)
    float best = 0.0f;
    for (int r = 0; r < 3; ++r) {
      k_read_evict<<<ctx->nsm * 4, 512, 0, st>>>(ev_buf, (long long)(evict_bytes / 16), sink);
      CK(cudaEventRecord(e0, st));
      launch();
      CK(cudaEventRecord(e1, st));
      CK(cudaGetLastError());
      CK(cudaEventSynchronize(e1));
      float t = 0.0f;
      CK(cudaEventElapsedTime(&t, e0, e1));
      if (r == 0 || t < best) best = t;
    }
    *ms = best;
    return N4_OK;
  };
  n4_component_tune_t rep{};
  n4_status_t status = N4_OK;
  for (int k = 0; k < kFitShapes && status == N4_OK && rep.fit_candidates < N4_TUNE_MAX; ++k) {
    if (!fit_shape_ok(k, d_field, d_mask, (int)fz)) continue;
    float ms = 0.0f;
    status = timed([&] { launch_fit_rows(k, d_field, d_mask, rows, (int)fz, az, t1n, t1d, st); }, &ms);
    if (status != N4_OK) break;
    const int c = rep.fit_candidates++;
    rep.fit_step[c] = kFitShape[k].step;
    rep.fit_depth[c] = kFitShape[k].depth;
    rep.fit_rows[c] = kFitShape[k].rows;
    rep.fit_ms[c] = ms;
    if (c == 0 || ms < rep.fit_ms[rep.fit_chosen]) { rep.fit_chosen = c; rep.fit_shape = k; }
  }
  // the evaluation candidates write d_out from the lattice the fit produces
  if (status == N4_OK)
    status = n4_fit_bspline3d(ctx, d_field, d_mask, ncpt_x, ncpt_y, ncpt_z, fx, fy, fz, 1e-3f, 0, d_lattice, stream);
  Upload u;
  if (status == N4_OK) status = acquire_slot(ctx, sizeof(CorrectVol) + 16, u);
  if (status == N4_OK) {
    CorrectVol cv{nullptr, d_out, nullptr, d_lattice, (char *)ax.s, (char *)ay.s, (char *)az.s,
                  (int)fx, (int)fy, (int)fz, (int)ncpt_x, (int)ncpt_y, (int)ncpt_z, 0,
                  vec4_ok((int)fz, nullptr, d_out, nullptr)};
    std::memcpy(u.h(), &cv, sizeof(cv));
    status = begin_run(ctx, st);
    if (status == N4_OK && cudaMemcpyAsync(u.slot->d.p, u.slot->h, sizeof(cv) + 16, cudaMemcpyHostToDevice, st) !=
                               cudaSuccess)
      status = fail(N4_ERR_CUDA, "descriptor upload failed");
    const size_t so = align_up(sizeof(cv), 16);
    for (int k = 0; k < kCorrectShapes && status == N4_OK; ++k) {
      const long long rt = kCorrectShape[k].rows;
      const long long tiles = ((long long)fx * fy + rt - 1) / rt;
      float ms = 0.0f;
      n4_status_t ls = N4_OK;
      status = timed([&] { ls = launch_correct(k, tiles, (int)ncpt_z, st, u.dp<CorrectVol>(0),
                                               u.dp<long long>(so), 1, 0, 0.0f, true); }, &ms);
      if (status == N4_OK) status = ls;
      if (status != N4_OK) break;
      const int c = rep.eval_candidates++;
      rep.eval_rows[c] = kCorrectShape[k].rows;
      rep.eval_threads[c] = kCorrectShape[k].threads;
      rep.eval_ms[c] = ms;
      if (c == 0 || ms < rep.eval_ms[rep.eval_chosen]) { rep.eval_chosen = c; rep.eval_shape = k; }
    }
    u.slot->nrep = 0;
    if (status == N4_OK) status = end_run(ctx, st, u);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status != N4_OK) return status;
  ctx->fit_tune[fit_key(fx, fy, fz, ncpt_x, ncpt_y, ncpt_z, d_field, d_mask)] = rep.fit_shape;
  ctx->eval_tune[eval_key(fx, fy, fz, ncpt_x, ncpt_y, ncpt_z)] = rep.eval_shape;
  if (report) *report = rep;
  return N4_OK;
}

n4_status_t n4_upsample_lattice3d(n4_context_t *ctx, const float *d_lattice, unsigned int ncpt_x, unsigned int ncpt_y,
                                  unsigned int ncpt_z, float *d_lattice_upsample, void *stream) {
  if (!ctx || !d_lattice || !d_lattice_upsample) return fail(N4_ERR_INVALID_ARG, "NULL pointer");
  if (ncpt_x < 4 || ncpt_y < 4 || ncpt_z < 4) return fail(N4_ERR_INVALID_ARG, "at least 4 control points per axis");
  CK(cudaSetDevice(ctx->device));
  k_refine<<<1, 256, 0, (cudaStream_t)stream>>>(d_lattice, ncpt_x, ncpt_y, ncpt_z, d_lattice_upsample);
  CK(cudaGetLastError());
  return N4_OK;
}

n4_status_t n4_sharpen_image(n4_context_t *ctx, const float *d_before, const float *d_mask, unsigned int n,
                             unsigned int bins, float wiener, float fwhm, float *d_after, float *bin_min,
                             float *bin_max, float *h_E) {
  if (!ctx || !d_before || !d_after || n == 0) return fail(N4_ERR_INVALID_ARG, "bad arguments");
  if (bins < 2 || bins > 1024) return fail(N4_ERR_INVALID_ARG, "bins must be in [2, 1024]");
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = nullptr;
  const int nb = std::min<int>((int)((n + 255) / 256), ctx->nsm * 8);
  TRY(ctx->s1.ensure((size_t)nb * 8 + 64, "partials"));
  TRY(ctx->s2.ensure((size_t)bins * 16 + 64, "histogram"));
  TRY(ctx->s3.ensure(64, "statistics"));
  float *part = ctx->s1.as<float>();
  double *stats = ctx->s3.as<double>();
  unsigned long long *hist = ctx->s2.as<unsigned long long>();
  double *E = (double *)(hist + bins);
  k_minmax<<<nb, 256, 0, st>>>(d_before, d_mask, n, part);
  k_minmax_final<<<1, 256, 0, st>>>(part, nb, bins, stats);
  CK(cudaMemsetAsync(hist, 0, (size_t)bins * 8, st));
  // one block sees at most (grid-stride trips) x 256 voxels
  const int shift = hist_shift_for(((long long)n + (long long)nb * 256 - 1) / ((long long)nb * 256) * 256);
  k_hist<<<nb, 256, bins * 4, st>>>(d_before, d_mask, n, stats, bins, shift, hist);
  const int npad = npad_of(bins), hoff = (int)(0.5 * (npad - bins));
  const int smem = npad * (16 * 3 + 8) + bins * 16;
  CK(cudaFuncSetAttribute(k_sharpen, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_sharpen<<<1, 512, smem, st>>>(hist, stats, bins, shift, npad, hoff, decimal_of(wiener), decimal_of(fwhm), E);
  k_remap<<<nb, 256, 0, st>>>(d_before, d_mask, n, stats, E, bins, d_after);
  CK(cudaGetLastError());
  double hs[4];
  std::vector<double> hE(bins);
  CK(cudaMemcpyAsync(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(hE.data(), E, (size_t)bins * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (bin_min) *bin_min = (float)hs[0];
  if (bin_max) *bin_max = (float)hs[1];
  if (h_E) for (unsigned b = 0; b < bins; ++b) h_E[b] = (float)hE[b];
  if (!(hs[0] <= hs[1])) return fail(N4_ERR_EMPTY_MASK, "no voxel in the mask");
  return N4_OK;
}

n4_status_t n4_convergence(n4_context_t *ctx, const float *d_field1, const float *d_field2, const float *d_mask,
                           unsigned int n, int ddof, double *cv) {
  if (!ctx || !d_field1 || !d_field2 || !cv || n == 0) return fail(N4_ERR_INVALID_ARG, "bad arguments");
  CK(cudaSetDevice(ctx->device));
  const int nb = std::min<int>((int)((n + 255) / 256), ctx->nsm * 4);
  TRY(ctx->s1.ensure((size_t)nb * 24, "partials"));
  k_cv<<<nb, 256>>>(d_field1, d_field2, d_mask, n, ctx->s1.as<double>());
  CK(cudaGetLastError());
  std::vector<double> part((size_t)nb * 3);
  CK(cudaMemcpy(part.data(), ctx->s1.p, part.size() * 8, cudaMemcpyDeviceToHost));
  double s0 = 0, s1 = 0, c = 0;
  for (int b = 0; b < nb; ++b) { s0 += part[3 * b]; s1 += part[3 * b + 1]; c += part[3 * b + 2]; }
  if (c < 1.0) return fail(N4_ERR_EMPTY_MASK, "no voxel in the mask");
  const double m = s0 / c;
  double var = s1 / c - m * m;
  if (ddof) var = c > 1.0 ? var * c / (c - 1.0) : 0.0;
  *cv = std::sqrt(var > 0 ? var : 0.0) / (1.0 + m);
  return N4_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- no-allocation fit
// Fixed device scratch for n4_fit_bspline3d_noalloc: the three axis tables,
// T1 (numerator/denominator per field row and z control point) and T2 (per
// x voxel and (y, z) control point).  Every entry the fit reads is written
// earlier in the same call, so nothing in it has to start at zero.
namespace {

constexpr size_t kNoAllocScratchBytes = 8u << 20;   // 8 MiB per device
static __device__ __align__(256) unsigned char g_fit_scratch[kNoAllocScratchBytes];

// The array's device address, looked up once per CUDA context: a context
// made after cudaDeviceReset loads the module again, possibly elsewhere, so
// the cached address is keyed by the context's process-unique id as well as
// the device ordinal.
constexpr int kMaxDevices = 64;
struct ScratchAddr {
  unsigned long long ctx_id = 0;   // 0: not looked up yet
  void *ptr = nullptr;
};
ScratchAddr g_fit_scratch_addr[kMaxDevices];
std::mutex g_fit_scratch_mu;

// Unique id of the current CUDA context (cuCtxGetCurrent + cuCtxGetId through
// the runtime's driver entry points, so the library needs no -lcuda).
n4_status_t current_context_id(unsigned long long *id) {
  using GetCurrent = int (*)(void **);
  using GetId = int (*)(void *, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (!get_current || !get_id) {
    void *a = nullptr, *b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess)
      return fail(N4_ERR_CUDA, "cuCtxGetCurrent/cuCtxGetId not available from the driver");
    get_current = (GetCurrent)a;
    get_id = (GetId)b;
  }
  void *ctx = nullptr;
  if (get_current(&ctx) != 0 || !ctx) return fail(N4_ERR_CUDA, "no current CUDA context");
  if (get_id(ctx, id) != 0) return fail(N4_ERR_CUDA, "cuCtxGetId failed");
  return N4_OK;
}

// The three tables of one call, passed by value (no descriptor upload).
__global__ void k_axis_tables_by_value(TableJob jx, TableJob jy, TableJob jz) {
  const TableJob t = blockIdx.x == 0 ? jx : (blockIdx.x == 1 ? jy : jz);
  build_axis(axis_at(t.base, t.n, t.nc));
}

}  // namespace

extern "C" {

n4_status_t n4_fit_bspline3d_noalloc(const float *d_field, const float *d_mask, unsigned int ncpt_x,
                                     unsigned int ncpt_y, unsigned int ncpt_z, unsigned int fx, unsigned int fy,
                                     unsigned int fz, float eps, int zero_den, float *d_lattice, void *stream) {
  if (!d_field || !d_lattice) return fail(N4_ERR_INVALID_ARG, "NULL pointer");
  TRY(check_fit_sizes(ncpt_x, ncpt_y, ncpt_z, fx, fy, fz));
  const size_t bx = align_up(axis_bytes(fx, ncpt_x - 3), 256), by = align_up(axis_bytes(fy, ncpt_y - 3), 256),
               bz = align_up(axis_bytes(fz, ncpt_z - 3), 256);
  const size_t t1 = (size_t)fx * fy * ncpt_z, t2 = (size_t)fx * ncpt_y * ncpt_z;
  const size_t need = bx + by + bz + align_up(t1 * 8, 256) + align_up(t2 * 8, 256);
  if (need > kNoAllocScratchBytes) {
    char msg[160];
    std::snprintf(msg, sizeof(msg),
                  "n4_fit_bspline3d_noalloc needs %zu bytes of scratch; its fixed scratch holds %zu "
                  "(use n4_fit_bspline3d)", need, kNoAllocScratchBytes);
    return fail(N4_ERR_TOO_LARGE, msg);
  }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(N4_ERR_INVALID_ARG, "device ordinal out of range");
  CK(cudaSetDevice(dev));   // makes the device's primary context current (CUDA 12 initialises it here)
  unsigned long long cid = 0;
  TRY(current_context_id(&cid));
  char *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_fit_scratch_mu);
    ScratchAddr &a = g_fit_scratch_addr[dev];
    if (a.ctx_id != cid) {   // once per device and context: the scratch's device address
      void *p = nullptr;
      CK(cudaGetSymbolAddress(&p, g_fit_scratch));
      a.ptr = p;
      a.ctx_id = cid;
    }
    base = (char *)a.ptr;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const TableJob jx{base, (int)fx, (int)ncpt_x}, jy{base + bx, (int)fy, (int)ncpt_y},
      jz{base + bx + by, (int)fz, (int)ncpt_z};
  k_axis_tables_by_value<<<3, 256, 0, st>>>(jx, jy, jz);
  const Axis ax = axis_at(jx.base, fx, ncpt_x), ay = axis_at(jy.base, fy, ncpt_y), az = axis_at(jz.base, fz, ncpt_z);
  float *t1n = (float *)(base + bx + by + bz), *t1d = t1n + t1;
  float *t2n = (float *)(base + bx + by + bz + align_up(t1 * 8, 256)), *t2d = t2n + t2;
  const long long rows = (long long)fx * fy;
  launch_fit_rows(fit_default_shape(d_field, d_mask, (int)fz), d_field, d_mask, rows, fz, az, t1n, t1d, st);
  k_fit_planes<<<(int)std::min<size_t>((t2 + 255) / 256, 148 * 8), 256, 0, st>>>(t1n, t1d, fx, fy, ay, ncpt_z, t2n,
                                                                                   t2d);
  const int nlat = ncpt_x * ncpt_y * ncpt_z;
  k_fit_final<<<(nlat + 255) / 256, 256, 0, st>>>(t2n, t2d, fx, ax, ncpt_y, ncpt_z, eps, zero_den, d_lattice);
  CK(cudaGetLastError());
  return N4_OK;
}

}  // extern "C"
