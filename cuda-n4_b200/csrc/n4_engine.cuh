// The N4 iteration for one volume, executed by a group of CTAs that share
// the volume's rows (cudaN4.cu:1418-1747, N4.py:276-332).
//
// A group is either a thread-block cluster (the volume lives in the
// cluster's distributed shared memory; partials are exchanged through DSMEM;
// hardware cluster barriers) or the whole grid of a cooperative launch (the
// volume lives in global memory/L2; partials are exchanged through global
// memory; a bounded software barrier).  The algorithm below is written once
// for both.
//
// Per level, with L the control lattice, D its last update and Gd = rows(D)
// the per-row partial evaluation of D (x/y contracted, one value per z
// control point), the slab holds logU, one float per fitting voxel:
//   reset   logU = im_log - eval(rows(L))    (level start, warm-start trial)
//   pass A  logU -= eval(Gd): the previous update applied, its convergence
//           value, masked min/max of logU                   (group reduce)
//   pass B  fractional histogram of logU                        (group reduce)
//           Wiener sharpening map E (every CTA, in shared memory)
//   pass C  residual R = logU - remap(logU)
//   fit     separable contraction of R with the fit weights     (group reduce)
//   update  D = num / (den + eps), L += D, Gd = rows(D)
// logU follows L by the same updates, applied per voxel: eval is linear, so
// logU = im_log - eval(rows(L)) up to FP32 rounding, which the reset at every
// level start clears.
#pragma once
#include <cooperative_groups.h>
#include <new>
#include <type_traits>

#include "n4_device.cuh"

namespace cg = cooperative_groups;

namespace n4 {

// Fixed-point scale 2^shift of one volume's histogram: the largest shift
// (<= 24) for which no 32-bit bin of a histogram copy can overflow.  A copy
// (one per 8th warp) receives at most an 8th of a CTA's voxels plus 160.  It
// depends on the volume and the group size alone (not on the other volumes of
// a batch), so a volume gets bitwise the same result in any batch.
__host__ __device__ inline int volume_hist_shift(int X, int Y, int Z, int K, bool grid) {
  const long long rows = (long long)X * Y;
  const long long rpc = grid ? (rows + K - 1) / K : ((long long)X + K - 1) / K * Y;
  return hist_shift_for((rpc * Z + 7) / 8 + 160);
}

// Voxels (or rows) whose loads a thread issues together in the voxel passes:
// 4 on the whole-GPU path, whose rows are read from L2/HBM; 1 on the cluster
// path, whose rows are in shared memory (measured: batching there only adds
// registers and instructions).
template <bool Grid> struct RowBatch { static constexpr int n = Grid ? 4 : 1; };
#define kNaN __int_as_float(0x7fc00000)

// ------------------------------------------------------------------ layout
// Byte offsets of one CTA's workspace.  "sm" offsets are always in shared
// memory; "big" offsets are in shared memory for the cluster path and in a
// per-CTA slice of global memory for the grid path.
struct Plan {
  // limits
  int levels, nc0x, nc0y, nc0z, NCX, NCY, NCZ, NLAT;
  int Xmax, Ymax, Zmax, slab_floats, rows_max, nvxl;
  int bins, npad, hoff;
  // shared
  int o_ax, o_ay, o_az, o_L, o_D, o_den, o_tmp, o_aux, o_hist, o_H64, o_R2, o_E;
  int o_fa, o_fb, o_tw, o_ff, o_red, o_misc;
  int sm_bytes;
  // big
  int b_imlog, b_Gd, b_T2, b_slotA, b_slotB, b_slotC, b_slice, big_bytes;
  // cluster path: the FFT work buffers, the histogram copies and the
  // Gaussian's transform (which the sharpening writes after the copies are
  // merged, over them) live in the Gd region, dead from the end of pass A
  // until the update, at these offsets
  int alias_sharpen, a_fa, a_fb, a_hist, a_ff;
};

struct Params {
  int bins;
  double wiener, fwhm, thr;   // decimal values of the float parameters
  float eps;
  int zero_den, ddof1;
  int iters[N4_MAX_LEVELS];
};

struct VolJob {
  int X, Y, Z;                  // fitting-resolution dimensions
  const float *imlog;           // [X*Y*Z] log intensity, NaN outside the mask
  const float *warm;            // first-level lattice or nullptr
  float *lattice_out;           // final lattice
  n4_report_t *report;
};

// Statistics exchanged after pass A: min, max, sum y, sum y^2.
struct Stats { double v[4]; };

// ------------------------------------------------------------------ groups
struct ClusterGroup {
  __device__ int rank() const { return (int)cg::this_cluster().block_rank(); }
  __device__ int size() const { return (int)cg::this_cluster().num_blocks(); }
  __device__ bool sync() const { cg::this_cluster().sync(); return true; }
  template <class T> __device__ const T *peer(const T *p, int r) const {
    return cg::this_cluster().map_shared_rank(const_cast<T *>(p), r);
  }
  template <class T> __device__ T load(const T *p) const { return *p; }
  static constexpr bool kGrid = false;
};

struct GridGroup {
  GridBarrier bar;
  char *big_base;      // per-CTA big regions, stride big_stride
  size_t big_stride;
  __device__ int rank() const { return (int)blockIdx.x; }
  __device__ int size() const { return (int)gridDim.x; }
  __device__ bool sync() const { return bar.sync(); }
  template <class T> __device__ const T *peer(const T *p, int r) const {
    const char *mine = big_base + (size_t)blockIdx.x * big_stride;
    return (const T *)(big_base + (size_t)r * big_stride + ((const char *)p - mine));
  }
  template <class T> __device__ T load(const T *p) const { return __ldcg(p); }
  static constexpr bool kGrid = true;
};

// ------------------------------------------------------------------ phase timers
// Compile with -DN4_PHASE_TIMERS to print, per volume, the cycles thread 0
// of the first CTA spends between phase marks (measurement builds only).  The
// counters live in shared memory, so that the timed build allocates the
// kernel's registers as the product build does.
#ifdef N4_PHASE_TIMERS
#define N4_MARK(k)                                                     \
  do {                                                                 \
    if (threadIdx.x == 0) {                                            \
      const long long t_ = clock64();                                  \
      ph_acc[k] += t_ - ph_acc[PH_N];                                  \
      ph_acc[PH_N] = t_;                                               \
    }                                                                  \
  } while (0)
#else
#define N4_MARK(k) do { } while (0)
#endif
enum { PH_SETUP, PH_A, PH_B, PH_SHARP, PH_C, PH_FIT, PH_UPDATE, PH_A_LOOP, PH_A_RED, PH_B_ZERO, PH_B_LOOP, PH_B_MERGE,
       PH_B_RED, PH_F_T1, PH_F_T2, PH_F_P, PH_F_RED, PH_N };
#ifdef N4_PHASE_TIMERS
__shared__ long long ph_acc[PH_N + 1];   // per-phase cycles, then the last mark
#endif

// ------------------------------------------------------------------ engine
// The Engine's fields are uniform over the CTA.  Whole-GPU path: one object
// per CTA in shared memory (EngineSlot), its fields written by thread 0 only
// (construction, run, set_level, each followed by a barrier); held in
// registers, the ~50 fields (pointers of the axis tables and work arrays)
// stay live through every pass and push the voxel loops into local-memory
// spills (measured: 512x512x320 in 6.2 ms instead of 6.5).  Cluster path: one
// object per thread, every thread writing its own copy (measured: the shared
// object made the 256x256x176 batch 11 % slower, its loops reloading fields
// after every shared-memory store or atomic).
template <class Group>
struct Engine {
  static constexpr int kRB = RowBatch<Group::kGrid>::n;
  static constexpr bool kShared = Group::kGrid;   // the object lives in shared memory
  // the threads that write the fields, and the barrier that publishes them
  __device__ __forceinline__ bool writer() const { return !kShared || threadIdx.x == 0; }
  __device__ __forceinline__ void publish() const { if (kShared) __syncthreads(); }
  Group g;
  const Plan &pl;
  const Params &pr;
  char *sm;
  char *big;
  float *red_global;   // grid path: [NLAT] / [bins] slice-reduction buffer
  // volume
  int X, Y, Z, nrow, rank, K;
  // rows of this CTA: grid path, contiguous rows r0 + rl; cluster path,
  // whole x-planes vx = rank + m * K (m = rl / Y), interleaved over the group
  int r0, nplane;
  int hshift;   // fixed-point scale of this volume's histogram
  FastDiv divZ;
  float *logu;         // [nrow][Z] logU of the local rows (NaN outside the mask)
  const float *src;    // the job's log volume (global memory), read by reset
  // level
  int ncx, ncy, ncz, nlat;
  Axis ax, ay, az;
  // smem views
  float *L, *D, *den, *tmp, *aux;
  double *E, *Ff;
  float2 *R2;          // the residual's per-bin linear form (residual_lin)
  unsigned *hist;
  unsigned long long *H64;
  double2 *fa, *fb, *tw;
  double *red;
  float *Gd, *T2, *slotC;
  Stats *slotA;
  unsigned long long *slotB;

  __device__ Engine(const Group &g_, const Plan &p, const Params &r, char *sm_, char *big_, float *rg)
      : g(g_), pl(p), pr(r), sm(sm_), big(big_), red_global(rg) {
    L = (float *)(sm + pl.o_L); D = (float *)(sm + pl.o_D); den = (float *)(sm + pl.o_den);
    tmp = (float *)(sm + pl.o_tmp); aux = (float *)(sm + pl.o_aux);
    hist = (unsigned *)(sm + pl.o_hist); H64 = (unsigned long long *)(sm + pl.o_H64);
    R2 = (float2 *)(sm + pl.o_R2); E = (double *)(sm + pl.o_E);
    fa = (double2 *)(sm + pl.o_fa); fb = (double2 *)(sm + pl.o_fb); tw = (double2 *)(sm + pl.o_tw);
    Ff = (double *)(sm + pl.o_ff); red = (double *)(sm + pl.o_red);
    Gd = (float *)(big + pl.b_Gd); T2 = (float *)(big + pl.b_T2);
    logu = (float *)(big + pl.b_imlog);
    if (pl.alias_sharpen) {
      fa = (double2 *)(big + pl.b_Gd + pl.a_fa); fb = (double2 *)(big + pl.b_Gd + pl.a_fb);
      hist = (unsigned *)(big + pl.b_Gd + pl.a_hist);
      Ff = (double *)(big + pl.b_Gd + pl.a_ff);
    }
    slotA = (Stats *)(big + pl.b_slotA); slotB = (unsigned long long *)(big + pl.b_slotB);
    slotC = (float *)(big + pl.b_slotC);
  }

  // ---- level geometry
  __device__ void set_level(int level) {
    if (writer()) {
      ncx = ((pl.nc0x - 3) << level) + 3;
      ncy = ((pl.nc0y - 3) << level) + 3;
      ncz = ((pl.nc0z - 3) << level) + 3;
      nlat = ncx * ncy * ncz;
      ax = axis_at(sm + pl.o_ax, X, ncx);
      ay = axis_at(sm + pl.o_ay, Y, ncy);
      az = axis_at(sm + pl.o_az, Z, ncz);
    }
    publish();
    build_axis(ax);
    build_axis(ay);
    build_axis(az);
    __syncthreads();
  }

  __device__ __forceinline__ void row_xy(int rl, int &vx, int &vy) const {
    if (Group::kGrid) {
      const int row = r0 + rl;
      vx = row / Y;
      vy = row - vx * Y;
    } else {
      const int m = rl / Y;
      vx = rank + m * K;
      vy = rl - m * Y;
    }
  }

  // ---- rows(lat) -> Gt: x/y contraction of the lattice for every local row
  __device__ void rowtab(const float *lat, float *Gt) {
    const int ntask = nrow * ncz;
    for (int t = threadIdx.x; t < ntask; t += blockDim.x) {
      const int rl = t / ncz, cz = t - rl * ncz;
      int vx, vy;
      row_xy(rl, vx, vy);
      const int sx = ax.s[vx], sy = ay.s[vy];
      const float4 wx = ax.w[vx], wy = ay.w[vy];
      const float wxa[4] = {wx.x, wx.y, wx.z, wx.w};
      const float wya[4] = {wy.x, wy.y, wy.z, wy.w};
      float acc = 0.0f;
#pragma unroll
      for (int jx = 0; jx < 4; ++jx) {
        const float *lp = lat + ((sx + jx) * ncy + sy) * ncz + cz;
        float s = 0.0f;
#pragma unroll
        for (int jy = 0; jy < 4; ++jy) s = __fmaf_rn(wya[jy], lp[jy * ncz], s);
        acc = __fmaf_rn(wxa[jx], s, acc);
      }
      Gt[t] = acc;
    }
  }

  // x-planes this CTA holds rows of: cluster, vx = rank + m*K for m < nplane
  // (local rows m*Y .. m*Y + Y - 1); grid, the planes r0/Y .. (r0+nrow-1)/Y
  __device__ __forceinline__ int nplanes_local() const {
    if (Group::kGrid) return nrow > 0 ? (r0 + nrow - 1) / Y - r0 / Y + 1 : 0;
    return nplane;
  }
  __device__ __forceinline__ int plane_vx(int m) const { return Group::kGrid ? r0 / Y + m : rank + m * K; }

  // rowtab(lat, Gt) after a lattice update, through the x-contracted planes:
  // per local x-plane, X[cy][cz] = sum_jx wx lat[sx+jx][cy][cz] (into aux,
  // free outside the warm-start trial), then per row Gt[cz] = sum_jy wy
  // X[sy+jy][cz]: 8 loads and multiply-adds per entry instead of 32.  Falls
  // back to rowtab when the planes' slices do not fit in a lattice-sized
  // buffer.  The caller synchronises.
  __device__ void rowtab_planes(const float *lat, float *Gt) {
    const int np = nplanes_local(), slice = ncy * ncz;
    if ((long long)np * slice > pl.NLAT) { rowtab(lat, Gt); return; }
    float *Xp = aux;
    for (int t = threadIdx.x; t < np * slice; t += blockDim.x) {
      const int m = t / slice, c = t - m * slice;
      const int vx = plane_vx(m);
      const int sx = ax.s[vx];
      const float4 wx = ax.w[vx];
      const float *pa = lat + (size_t)sx * slice + c;
      float a = __fmul_rn(wx.x, pa[0]);
      a = __fmaf_rn(wx.y, pa[slice], a);
      a = __fmaf_rn(wx.z, pa[2 * slice], a);
      Xp[t] = __fmaf_rn(wx.w, pa[3 * slice], a);
    }
    __syncthreads();
    const int vx0 = Group::kGrid ? r0 / Y : 0;
    for (int t = threadIdx.x; t < nrow * ncz; t += blockDim.x) {
      const int rl = t / ncz, cz = t - rl * ncz;
      int vx, vy;
      row_xy(rl, vx, vy);
      const int m = Group::kGrid ? vx - vx0 : rl / Y;
      const int sy = ay.s[vy];
      const float4 wy = ay.w[vy];
      const float *xa = Xp + m * slice + sy * ncz + cz;
      float a = __fmul_rn(wy.x, xa[0]);
      a = __fmaf_rn(wy.y, xa[ncz], a);
      a = __fmaf_rn(wy.z, xa[2 * ncz], a);
      Gt[t] = __fmaf_rn(wy.w, xa[3 * ncz], a);
    }
  }

  // First voxel of local row rl in the job's log volume: grid, contiguous
  // rows r0 + rl; cluster, plane vx = rank + m*K, row vy of it
  __device__ __forceinline__ const float *src_row(int rl) const {
    if (Group::kGrid) return src + (size_t)(r0 + rl) * Z;
    const int m = rl / Y;
    return src + ((size_t)(rank + m * K) * Y + (rl - m * Y)) * Z;
  }

  // logU = im_log - eval(rows(lat)) for every local voxel, im_log read from
  // the slab itself when `staged` (the cluster kernel's bulk copy of the
  // volume, before the first reset), else from the job's log volume in
  // global memory; rows(lat) goes through the Gd region (free at every
  // reset: level start, warm-start trial).
  __device__ void reset(const float *lat, bool staged = false) {
    rowtab(lat, Gd);
    __syncthreads();
    const int n = nrow * Z;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int rl = (int)divZ.div((unsigned)i), vz = i - rl * Z;
      const float v = staged ? logu[i] : src_row(rl)[vz];
      logu[i] = isnan(v) ? v : __fsub_rn(v, eval(Gd, rl, vz));
    }
    __syncthreads();
  }

  __device__ __forceinline__ float eval(const float *Gt, int rl, int vz) const {
    return dot4(az.w[vz], Gt + rl * ncz + az.s[vz]);
  }

  // ---- group reductions
  // Stats: every CTA reads all K slots in the same order.
  __device__ bool reduce_stats(const double in[4], double out[4]) {
    if (threadIdx.x == 0) { for (int i = 0; i < 4; ++i) slotA->v[i] = in[i]; }
    if (!g.sync()) return false;
    if (threadIdx.x < 32) {
      float mn = INFINITY, mx = -INFINITY;
      double s0 = 0.0, s1 = 0.0;
      for (int k = threadIdx.x; k < K; k += 32) {
        const Stats *p = g.peer(slotA, k);
        mn = fminf(mn, (float)g.load(&p->v[0]));
        mx = fmaxf(mx, (float)g.load(&p->v[1]));
        s0 += g.load(&p->v[2]);
        s1 += g.load(&p->v[3]);
      }
      mn = warp_min(mn); mx = warp_max(mx); s0 = warp_sum(s0); s1 = warp_sum(s1);
      if (threadIdx.x == 0) { red[0] = mn; red[1] = mx; red[2] = s0; red[3] = s1; }
    }
    __syncthreads();
    for (int i = 0; i < 4; ++i) out[i] = red[i];
    __syncthreads();
    return true;
  }

  // Sum of every CTA's `mine[0..n)` into `out` (shared), identical in all
  // CTAs, each entry summed over the CTAs in rank order.  Cluster: after one
  // barrier every CTA reads all K partials through DSMEM (a partial is written
  // again only after later barriers of the iteration, by which time every
  // peer has read it).  Grid: each CTA reduces one slice over all peers, then
  // every CTA gathers the slices; slices live in a buffer of their own, so a
  // CTA may modify `out` while slower peers are still gathering.
  // Sum over the group's K partials of entry c, in rank order: exact for the
  // integer histogram, Kahan-compensated for the fit's float partials.
  struct Acc64 {
    unsigned long long s = 0;
    __device__ __forceinline__ void add(unsigned long long x) { s += x; }
    __device__ __forceinline__ unsigned long long value() const { return s; }
  };
  template <class T> using AccOf = typename std::conditional<std::is_same<T, float>::value, KahanSum, Acc64>::type;

  template <class T>
  __device__ bool allreduce(const T *mine, T *out, int n) {
    if (!g.sync()) return false;
    if (!Group::kGrid) {
      for (int c = threadIdx.x; c < n; c += blockDim.x) {
        AccOf<T> acc;
#pragma unroll 4
        for (int k = 0; k < K; ++k) acc.add(*(g.peer(mine, k) + c));
        out[c] = acc.value();
      }
      __syncthreads();
      return true;
    }
    const int per = (n + K - 1) / K;
    const int c0 = rank * per, c1 = min(n, c0 + per);
    T *slice = Group::kGrid ? (T *)red_global : (T *)(big + pl.b_slice);
    // one warp per entry of the slice: lane l sums the partials of CTAs
    // l, l + 32, ... (compensated for floats), then a fixed shuffle tree adds
    // the lanes, so that the K loads of an entry are in flight together
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int c = c0 + warp; c < c1; c += nwarp) {
      AccOf<T> acc;
      for (int k = lane; k < K; k += 32) acc.add(g.load(g.peer(mine, k) + c));
      T v = acc.value();
#pragma unroll
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
      if (lane == 0) slice[Group::kGrid ? c : c - c0] = v;
    }
    if (!g.sync()) return false;
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      if (Group::kGrid) {
        out[c] = __ldcg(slice + c);
      } else {
        const int owner = c / per;
        out[c] = *(g.peer(slice, owner) + (c - owner * per));
      }
    }
    __syncthreads();
    return true;
  }

  // ---- separable fit contraction of the local rows into slotC (full lattice)
  // num: the residuals left by pass C with weights w^3/sum w^2; den: the mask
  // with weights w^2 (N4.py:224-236).
  //   T1[row][cz]   z contraction: one thread per (row, z-span) accumulates
  //                 the span's 4 targets in registers; spans s = phi mod 4
  //                 never share a target, so 4 phases add without atomics in
  //                 a fixed order
  //   T2[vx][cy][cz] y contraction over the CTA's rows of each x-plane
  //   slotC[c]       x contraction (the CTA's partial lattice)
  // then the group all-reduce of the partial lattices.  The sums across rows
  // (y, x and over the CTAs) are Kahan-compensated: a control point of the
  // 256x256x160 grid gathers ~5e5 voxels through them.  The sum within a row
  // covers one span (at most Z / spans voxels, fixed order) and is plain FP32.
  __device__ void contract(bool num_mode, const BinMap *bm = nullptr, bool degenerate = false) {
    float *T1 = Gd;   // Gd is dead between pass A and the next update
    const int nt1 = nrow * ncz;
    // whole-GPU path, few spans per row (coarse levels): the (row, span) tasks
    // leave most of the CTA's threads idle (443 rows of 160 voxels for 1024
    // threads at 512x512x320), so each span is cut in two halves, summed by
    // two threads into two tables (the second after the first in Gd, when it
    // fits) that are added at the end.  (On the cluster path, rows of ~44
    // voxels, the extra tasks and the final pass cost more than they save.)
    const int gd_floats = (pl.b_T2 - pl.b_Gd) / 4;
    const int halves = (Group::kGrid && az.nsp <= 4 && 2 * nt1 <= gd_floats) ? 2 : 1;
    float *T1b = T1 + nt1;
    for (int t = threadIdx.x; t < halves * nt1; t += blockDim.x) T1[t] = 0.0f;
    __syncthreads();
    const float4 *W4 = num_mode ? az.p4 : az.q4;
    for (int phase = 0; phase < 4; ++phase) {
      const int nsp = phase < az.nsp ? (az.nsp - phase + 3) / 4 : 0;   // spans phase, phase+4, ...
      const int per_row = nsp * halves;
      const int ntask = nrow * per_row;
      for (int t = threadIdx.x; t < ntask; t += blockDim.x) {
        const int rl = t / per_row, rem = t - rl * per_row;
        const int sp = phase + 4 * (halves == 2 ? rem >> 1 : rem), h = halves == 2 ? rem & 1 : 0;
        int lo = az.lo[sp], hi = az.hi[sp];
        if (halves == 2) {
          const int mid = (lo + hi) >> 1;
          if (h) lo = mid;
          else hi = mid;
        }
        float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
        if (num_mode) {
          // residual R = logU - E(logU) of each masked voxel
          const float *iv = logu + (size_t)rl * Z;
          if constexpr (kRB == 1) {
            for (int vz = lo; vz < hi; ++vz) {
              const float lu = iv[vz];
              if (isnan(lu)) continue;
              const float r = degenerate ? 0.0f : residual_of(*bm, lu, R2, E, pr.bins);
              const float4 w = W4[vz];
              a0 = __fmaf_rn(w.x, r, a0); a1 = __fmaf_rn(w.y, r, a1);
              a2 = __fmaf_rn(w.z, r, a2); a3 = __fmaf_rn(w.w, r, a3);
            }
          } else
          // kRB voxels at a time: their loads are issued before the
          // first is used; the terms are added in voxel order
          for (int vb = lo; vb < hi; vb += kRB) {
            float v[kRB];
#pragma unroll
            for (int u = 0; u < kRB; ++u) v[u] = vb + u < hi ? iv[vb + u] : kNaN;
#pragma unroll
            for (int u = 0; u < kRB; ++u) {
              if (isnan(v[u])) continue;
              const int vz = vb + u;
              const float lu = v[u];
              const float r = degenerate ? 0.0f : residual_of(*bm, lu, R2, E, pr.bins);
              const float4 w = W4[vz];
              a0 = __fmaf_rn(w.x, r, a0); a1 = __fmaf_rn(w.y, r, a1);
              a2 = __fmaf_rn(w.z, r, a2); a3 = __fmaf_rn(w.w, r, a3);
            }
          }
        } else {
          const float *iv = logu + (size_t)rl * Z;
          if constexpr (kRB == 1) {
            for (int vz = lo; vz < hi; ++vz) {
              if (isnan(iv[vz])) continue;
              const float4 w = W4[vz];
              a0 += w.x; a1 += w.y; a2 += w.z; a3 += w.w;
            }
          } else
          for (int vb = lo; vb < hi; vb += kRB) {
            float v[kRB];
#pragma unroll
            for (int u = 0; u < kRB; ++u) v[u] = vb + u < hi ? iv[vb + u] : kNaN;
#pragma unroll
            for (int u = 0; u < kRB; ++u) {
              if (isnan(v[u])) continue;
              const float4 w = W4[vb + u];
              a0 += w.x; a1 += w.y; a2 += w.z; a3 += w.w;
            }
          }
        }
        float *t1 = (h ? T1b : T1) + rl * ncz + sp;
        t1[0] += a0; t1[1] += a1; t1[2] += a2; t1[3] += a3;
      }
      __syncthreads();
    }
    if (halves == 2) {
      for (int t = threadIdx.x; t < nt1; t += blockDim.x) T1[t] = __fadd_rn(T1[t], T1b[t]);
      __syncthreads();
    }
    N4_MARK(PH_F_T1);
    const float *PY = num_mode ? ay.p : ay.q;
    const float *PX = num_mode ? ax.p : ax.q;
    if (Group::kGrid) {
      // contiguous rows: planes vx0..vx1, partially covered at both ends
      const int vx0 = r0 / Y, vx1 = (r0 + nrow - 1) / Y;
      const int nt2 = (vx1 - vx0 + 1) * ncy * ncz;
      for (int t = threadIdx.x; t < nt2; t += blockDim.x) {
        const int cz = t % ncz, cy = (t / ncz) % ncy, xl = t / (ncz * ncy);
        const int rb = (vx0 + xl) * Y - r0;   // local row of (vx, 0)
        KahanSum acc, acc2;   // two chains (alternate rows), merged at the end
        for (int j = 0; j < 4; ++j) {
          const int sp = cy - j;
          if (sp < 0 || sp >= ay.nsp) continue;
          const int lo = max(ay.lo[sp], -rb), hi = min(ay.hi[sp], nrow - rb);
          const float *wy = PY + j * Y;
          int vy = lo;
          for (; vy + 1 < hi; vy += 2) {
            acc.add_prod(wy[vy], T1[(rb + vy) * ncz + cz]);
            acc2.add_prod(wy[vy + 1], T1[(rb + vy + 1) * ncz + cz]);
          }
          if (vy < hi) acc.add_prod(wy[vy], T1[(rb + vy) * ncz + cz]);
        }
        acc.merge(acc2);
        T2[t] = acc.value();
      }
      __syncthreads();
      N4_MARK(PH_F_T2);
      for (int c = threadIdx.x; c < nlat; c += blockDim.x) {
        const int cz = c % ncz, cy = (c / ncz) % ncy, cx = c / (ncz * ncy);
        KahanSum acc;
        for (int j = 0; j < 4; ++j) {
          const int sp = cx - j;
          if (sp < 0 || sp >= ax.nsp) continue;
          const int lo = max(ax.lo[sp], vx0), hi = min(ax.hi[sp], vx1 + 1);
          const float *wx = PX + j * X;
          for (int vx = lo; vx < hi; ++vx) acc.add_prod(wx[vx], T2[((vx - vx0) * ncy + cy) * ncz + cz]);
        }
        slotC[c] = acc.value();
      }
      return;
    }
    // whole planes vx = rank + m*K: y contraction per local plane
    const int nt2 = nplane * ncy * ncz;
    for (int t = threadIdx.x; t < nt2; t += blockDim.x) {
      const int cz = t % ncz, cy = (t / ncz) % ncy, m = t / (ncz * ncy);
      const float *t1 = T1 + (size_t)m * Y * ncz + cz;
      KahanSum acc, acc2;   // two chains (alternate rows), merged at the end
      for (int j = 0; j < 4; ++j) {
        const int sp = cy - j;
        if (sp < 0 || sp >= ay.nsp) continue;
        const float *wy = PY + j * Y;
        int vy = ay.lo[sp];
        const int hi = ay.hi[sp];
        for (; vy + 1 < hi; vy += 2) {
          acc.add_prod(wy[vy], t1[vy * ncz]);
          acc2.add_prod(wy[vy + 1], t1[(vy + 1) * ncz]);
        }
        if (vy < hi) acc.add_prod(wy[vy], t1[vy * ncz]);
      }
      acc.merge(acc2);
      T2[t] = acc.value();
    }
    __syncthreads();
    N4_MARK(PH_F_T2);
    for (int c = threadIdx.x; c < nlat; c += blockDim.x) {
      const int cz = c % ncz, cy = (c / ncz) % ncy, cx = c / (ncz * ncy);
      KahanSum acc;
      for (int j = 0; j < 4; ++j) {
        const int sp = cx - j;
        if (sp < 0 || sp >= ax.nsp) continue;
        const float *wx = PX + j * X;
        // local planes inside [lo, hi): vx = rank + m*K
        const int lo = ax.lo[sp], hi = ax.hi[sp];
        int m = lo <= rank ? 0 : (lo - rank + K - 1) / K;
        for (int vx = rank + m * K; vx < hi; vx += K, ++m) acc.add_prod(wx[vx], T2[(m * ncy + cy) * ncz + cz]);
      }
      slotC[c] = acc.value();
    }
  }

  // ---- pass A: the previous update's convergence sums from eval(Gd) (when
  // need_cv), applied to logU (when apply: logU -= eval(Gd)), and the masked
  // min/max of logU
  __device__ bool pass_a(bool need_cv, bool apply, double st[4]) {
    float vmin = INFINITY, vmax = -INFINITY;
    double sy = 0.0, syy = 0.0;
    const int per = (int)blockDim.x / Z;   // whole rows per sweep: each thread keeps one z
    if (per > 0) {
      const int rs = (int)threadIdx.x / Z, vz = (int)threadIdx.x - rs * Z;
      if (rs < per) {
        const float4 w = az.w[vz];
        const int sz = az.s[vz];
        if constexpr (kRB == 1) {
          for (int rl = rs; rl < nrow; rl += per) {
            float lu = logu[rl * Z + vz];
            if (isnan(lu)) continue;   // outside the mask
            if (need_cv) {
              const float ed = dot4(w, Gd + rl * ncz + sz);
              const float y = expm1_conv(-ed);
              sy += (double)y;
              syy += (double)y * (double)y;
              if (apply) {
                lu = __fsub_rn(lu, ed);
                logu[rl * Z + vz] = lu;
              }
            }
            vmin = fminf(vmin, lu);
            vmax = fmaxf(vmax, lu);
          }
        } else
        // kRB rows at a time: their loads are all issued before the
        // first of them is used; the values are then taken in row order
        for (int rb = rs; rb < nrow; rb += kRB * per) {
          float v[kRB], evd[kRB];
#pragma unroll
          for (int u = 0; u < kRB; ++u) {
            const int rl = rb + u * per;
            v[u] = rl < nrow ? logu[rl * Z + vz] : kNaN;
          }
#pragma unroll
          for (int u = 0; u < kRB; ++u) {
            const int rl = rb + u * per;
            evd[u] = (!isnan(v[u]) && need_cv) ? dot4(w, Gd + rl * ncz + sz) : 0.0f;
          }
#pragma unroll
          for (int u = 0; u < kRB; ++u) {
            if (isnan(v[u])) continue;   // outside the mask
            float lu = v[u];
            if (need_cv) {
              const float y = expm1_conv(-evd[u]);
              sy += (double)y;
              syy += (double)y * (double)y;
              if (apply) {
                lu = __fsub_rn(lu, evd[u]);
                logu[(rb + u * per) * Z + vz] = lu;
              }
            }
            vmin = fminf(vmin, lu);
            vmax = fmaxf(vmax, lu);
          }
        }
      }
    } else {
      const int n = nrow * Z;
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        float lu = logu[i];
        if (isnan(lu)) continue;
        if (need_cv) {
          const int rl = (int)divZ.div((unsigned)i), vz = i - rl * Z;
          const float ed = eval(Gd, rl, vz);
          const float y = expm1_conv(-ed);
          sy += (double)y;
          syy += (double)y * (double)y;
          if (apply) {
            lu = __fsub_rn(lu, ed);
            logu[i] = lu;
          }
        }
        vmin = fminf(vmin, lu);
        vmax = fmaxf(vmax, lu);
      }
    }
    double loc[4];
    block_reduce4(vmin, vmax, sy, syy, red + 8, loc);
    if (threadIdx.x == 0) for (int i = 0; i < 4; ++i) red[4 + i] = loc[i];
    __syncthreads();
    for (int i = 0; i < 4; ++i) loc[i] = red[4 + i];
    __syncthreads();
    N4_MARK(PH_A_LOOP);
    const bool ok = reduce_stats(loc, st);
    N4_MARK(PH_A_RED);
    return ok;
  }

  // ---- pass B + sharpening: histogram of logU over the group, then E
  __device__ bool pass_b(const BinMap &bm) {
    const int bins = pr.bins, shift = hshift;
    const double scale = ldexp(1.0, shift);
    for (int i = threadIdx.x; i < kHistCopies * bins; i += blockDim.x) hist[i] = 0u;
    __syncthreads();
    N4_MARK(PH_B_ZERO);
    unsigned *hc = hist + ((threadIdx.x >> 5) % kHistCopies) * bins;
    const int n = nrow * Z;   // the local voxels in order: lanes take consecutive voxels
    if constexpr (kRB == 1) {
      for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        int key = -1;
        unsigned qlo = 0, qhi = 0;
        if (i < n) {
          const float lu = logu[i];
          if (!isnan(lu)) key = hist_bin_of(bm, lu, bins, scale, qlo, qhi);
        }
        if (key >= 0) {
          atomicAdd(&hc[key], qlo);
          if (qhi) atomicAdd(&hc[key + 1], qhi);
        }
      }
    } else {
      // kRB voxels per thread at a time, their loads issued first
      for (int base = 0; base < n; base += kRB * blockDim.x) {
        float v[kRB];
#pragma unroll
        for (int u = 0; u < kRB; ++u) {
          const int i = base + u * (int)blockDim.x + (int)threadIdx.x;
          v[u] = i < n ? logu[i] : kNaN;
        }
#pragma unroll
        for (int u = 0; u < kRB; ++u) {
          if (isnan(v[u])) continue;
          unsigned qlo = 0, qhi = 0;
          const int key = hist_bin_of(bm, v[u], bins, scale, qlo, qhi);
          if (key >= 0) {
            atomicAdd(&hc[key], qlo);
            if (qhi) atomicAdd(&hc[key + 1], qhi);
          }
        }
      }
    }
    __syncthreads();
    N4_MARK(PH_B_LOOP);
    for (int b = threadIdx.x; b < bins; b += blockDim.x) {
      unsigned long long s = 0;
      for (int c = 0; c < kHistCopies; ++c) s += hist[c * bins + b];
      slotB[b] = s;
    }
    __syncthreads();
    N4_MARK(PH_B_MERGE);
    if (!allreduce(slotB, H64, bins)) return false;
    N4_MARK(PH_B_RED);
    N4_MARK(PH_B);
    const double inv = ldexp(1.0, -shift);
    const unsigned long long *h64 = H64;
    SharpenBufs sb{fa, fb, tw, Ff};
    sharpen_map([=](int b) { return (double)h64[b] * inv; }, bins, pl.npad, pl.hoff, bm.binMin, bm.slope,
                pr.wiener, pr.fwhm, sb, E, R2);
    N4_MARK(PH_SHARP);
    return true;
  }

  // ---- one sharpen + fit step from the current logU; leaves the update in D
  __device__ bool fit_step(const double st[4]) {
    // bin range of the masked logU (N4.py:14-15); st holds FP32 values
    const double bmin = st[0], bmax = st[1];
    const double slope = (bmax - bmin) / (double)(pr.bins - 1);
    const bool degenerate = !(slope > 0.0) || !isfinite(slope);
    const BinMap bm(bmin, degenerate ? 1.0 : slope, pr.bins);
    if (!degenerate) { if (!pass_b(bm)) return false; }
    N4_MARK(PH_C);
    contract(true, &bm, degenerate);   // the residual is formed inside the z contraction
    __syncthreads();
    N4_MARK(PH_F_P);
    if (!allreduce(slotC, D, nlat)) return false;
    N4_MARK(PH_F_RED);
    for (int c = threadIdx.x; c < nlat; c += blockDim.x) {
      const float nu = D[c], de = den[c];
      D[c] = pr.zero_den ? (de != 0.0f ? nu / de : 0.0f) : nu / (de + pr.eps);
    }
    __syncthreads();
    return true;
  }

  __device__ float cv_from(const double st[4], double nfg) const {
    const double mean_y = st[2] / nfg;
    double var = st[3] / nfg - mean_y * mean_y;
    if (pr.ddof1) var = nfg > 1.0 ? var * nfg / (nfg - 1.0) : 0.0;
    return (float)(sqrt(var > 0.0 ? var : 0.0) / (1.0 + mean_y));
  }

  // ---- the whole volume (logU of the local rows in the big region's slab;
  // im_log read from job.imlog; cluster path: the slab holds the local rows
  // of im_log on entry)
  __device__ void run(const VolJob &job) {
    if (writer()) {
      X = job.X; Y = job.Y; Z = job.Z;
      rank = g.rank(); K = g.size();
      if constexpr (Group::kGrid) {  // contiguous rows: the volume lives in global memory
        r0 = (int)((long long)X * Y * rank / K);
        nrow = (int)((long long)X * Y * (rank + 1) / K) - r0;
        nplane = 0;
      } else {                       // interleaved planes: every CTA samples the whole volume
        r0 = 0;
        nplane = X > rank ? (X - rank + K - 1) / K : 0;
        nrow = nplane * Y;
      }
      divZ = FastDiv((unsigned)Z);
      hshift = volume_hist_shift(X, Y, Z, K, Group::kGrid);
      src = job.imlog;
    }
    publish();
    const bool lead = (rank == 0 && threadIdx.x == 0);
    n4_report_t *rep = job.report;
    if (lead) { rep->device_begin_ns = global_ns(); rep->device_end_ns = 0; rep->sm = sm_id(); }

#ifdef N4_PHASE_TIMERS
    if (threadIdx.x == 0) {
      for (int k = 0; k < PH_N; ++k) ph_acc[k] = 0;
      ph_acc[PH_N] = clock64();
    }
#endif
    fft_twiddles(tw, pl.npad);
    // foreground count of the group
    float cnt = 0.0f;
    double cntd = 0.0;
    for (int i = threadIdx.x; i < nrow * Z; i += blockDim.x) {
      const int rl = (int)divZ.div((unsigned)i);
      cnt += isnan(Group::kGrid ? src_row(rl)[i - rl * Z] : logu[i]) ? 0.0f : 1.0f;   // cluster: staged
    }
    cntd = cnt;
    double loc[4], st[4];
    block_reduce4(0.0f, 0.0f, cntd, 0.0, red + 8, loc);
    if (threadIdx.x == 0) red[4] = loc[2];
    __syncthreads();
    loc[0] = 0.0; loc[1] = 0.0; loc[2] = red[4]; loc[3] = 0.0;
    __syncthreads();
    if (!reduce_stats(loc, st)) { if (lead) rep->status = N4_ERR_TIMEOUT; return; }
    const double nfg = st[2];
    if (lead) { rep->foreground = (long long)nfg; rep->levels = 0; rep->warm_start_used = 0; }
    if (nfg < 1.0) {
      if (rank == 0) {
        for (int c = threadIdx.x; c < pl.NLAT; c += blockDim.x) job.lattice_out[c] = 0.0f;
        if (threadIdx.x == 0) rep->status = N4_ERR_EMPTY_MASK;
      }
      return;
    }

    // first-level lattice
    set_level(0);
    for (int c = threadIdx.x; c < nlat; c += blockDim.x) L[c] = job.warm ? job.warm[c] : 0.0f;
    __syncthreads();

    for (int level = 0; level < pl.levels; ++level) {
      if (level > 0) {
        const int pcx = ncx, pcy = ncy, pcz = ncz;
        refine_lattice(L, pcx, pcy, pcz, tmp);
        __syncthreads();
        set_level(level);
        for (int c = threadIdx.x; c < nlat; c += blockDim.x) L[c] = tmp[c];
        __syncthreads();
      }
      // logU of this level's lattice, then the constant denominator of the fit
      reset(L, level == 0 && !Group::kGrid);
      contract(false);
      if (!allreduce(slotC, den, nlat)) goto timeout;
      const int maxIt = pr.iters[level];
      int it = 0;
      float cv = 1e10f;
      if (level == 0 && job.warm && maxIt > 0) {
        // warm start: one iteration from the warm lattice and one from zero;
        // keep the one whose first convergence value is not larger.  Each
        // arm starts from a reset and leaves logU one update (D, in Gd)
        // behind L, as the main loop expects after an iteration.
        float cvs[2];
        for (int arm = 0; arm < 2; ++arm) {
          for (int c = threadIdx.x; c < nlat; c += blockDim.x) L[c] = arm == 0 ? job.warm[c] : 0.0f;
          __syncthreads();
          if (arm == 1) reset(L);   // arm 0 starts from the level's reset (L = warm)
          if (!pass_a(false, false, st)) goto timeout;
          if (!fit_step(st)) goto timeout;
          rowtab(D, Gd);
          for (int c = threadIdx.x; c < nlat; c += blockDim.x) L[c] += D[c];
          __syncthreads();
          if (!pass_a(true, false, st)) goto timeout;   // the update's CV; logU not advanced
          cvs[arm] = cv_from(st, nfg);
          if (arm == 0) {   // keep the warm result in aux, its update in tmp
            for (int c = threadIdx.x; c < nlat; c += blockDim.x) { aux[c] = L[c]; tmp[c] = D[c]; }
            __syncthreads();
          }
        }
        const bool use_warm = cvs[0] <= cvs[1];
        if (use_warm) {
          // logU back to the warm lattice, L and D to the warm arm's update
          reset(job.warm);
          for (int c = threadIdx.x; c < nlat; c += blockDim.x) { L[c] = aux[c]; D[c] = tmp[c]; }
          __syncthreads();
          rowtab_planes(D, Gd);
          __syncthreads();
        }
        cv = use_warm ? cvs[0] : cvs[1];
        it = 1;
        if (lead) {
          rep->warm_start_used = use_warm ? 1 : 0;
          rep->first_cv_warm = cvs[0];
          rep->first_cv_plain = cvs[1];
        }
      }
      N4_MARK(PH_SETUP);
      for (;;) {
        if (!pass_a(it > 0, it > 0, st)) goto timeout;   // applies the last update
        N4_MARK(PH_A);
        if (it > 0) cv = cv_from(st, nfg);
        if (!((double)cv > pr.thr) || it >= maxIt) break;
        if (!fit_step(st)) goto timeout;
        for (int c = threadIdx.x; c < nlat; c += blockDim.x) L[c] += D[c];
        __syncthreads();
        rowtab_planes(D, Gd);
        __syncthreads();
        N4_MARK(PH_UPDATE);
        ++it;
      }
      if (lead) { rep->iterations[level] = it; rep->final_cv[level] = cv; rep->levels = level + 1; }
    }
    if (rank == 0) {
      for (int c = threadIdx.x; c < nlat; c += blockDim.x) job.lattice_out[c] = L[c];
      if (threadIdx.x == 0) { rep->status = N4_OK; rep->device_end_ns = global_ns(); }
    }
#ifdef N4_PHASE_TIMERS
    if (lead)
      printf("N4PHASE K=%d nt=%d setup=%lld A=%lld Aloop=%lld Ared=%lld Bzero=%lld Bloop=%lld Bmerge=%lld Bred=%lld "
             "Bconv=%lld sharp=%lld C=%lld T1=%lld T2=%lld P=%lld Fred=%lld update=%lld\n",
             K, (int)blockDim.x, ph_acc[PH_SETUP], ph_acc[PH_A], ph_acc[PH_A_LOOP], ph_acc[PH_A_RED],
             ph_acc[PH_B_ZERO], ph_acc[PH_B_LOOP], ph_acc[PH_B_MERGE], ph_acc[PH_B_RED], ph_acc[PH_B],
             ph_acc[PH_SHARP], ph_acc[PH_C], ph_acc[PH_F_T1], ph_acc[PH_F_T2], ph_acc[PH_F_P], ph_acc[PH_F_RED],
             ph_acc[PH_UPDATE]);
#endif
    return;
  timeout:
    if (lead) rep->status = N4_ERR_TIMEOUT;
  }
};

// Shared-memory home of a CTA's Engine on the whole-GPU path: thread 0
// constructs it, then every thread of the CTA uses the same object.
template <class Group>
struct EngineSlot {
  static_assert(Engine<Group>::kShared, "only the whole-GPU path keeps its Engine in shared memory");
  alignas(16) unsigned char raw[sizeof(Engine<Group>)];
  __device__ Engine<Group> &make(const Group &g, const Plan &p, const Params &r, char *sm, char *big, float *rg) {
    if (threadIdx.x == 0) new (raw) Engine<Group>(g, p, r, sm, big, rg);
    __syncthreads();
    return *reinterpret_cast<Engine<Group> *>(raw);
  }
};

}  // namespace n4
