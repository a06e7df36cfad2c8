// Kernels of n4b200 (sm_100a).
//
//   k_prologue        full resolution -> fitting grid: threshold, shrink, log
//                     (cudaN4.cu:639-652, 131-147; N4.py:284-287)
//   k_n4_cluster      persistent N4 over a queue of volumes, one thread-block
//                     cluster per volume, the volume resident in DSMEM
//   k_n4_grid         N4 on one large volume with the whole GPU
//   k_axis_tables     per-axis B-spline tables in global memory
//   k_correct         final dense evaluation at full resolution fused with
//                     im / exp(b) and the optional exp(b) output
//                     (cudaN4.cu:1697-1729, N4.py:329-330)
//   k_fit_*           standalone separable B-spline fit (FitBspline3D)
//   k_refine          lattice refinement (upsampleLattice3D_gpu)
//   k_minmax/k_hist/k_sharpen/k_remap   standalone sharpenImage
//   k_cv              standalone convergence measurement
#pragma once
#include <cuda_bf16.h>

#include "n4_engine.cuh"

namespace n4 {

// ------------------------------------------------------------------ prologue
struct PrologueVol {
  const float *im;          // full resolution
  const void *mask;         // float or byte mask (mask_u8), may be null
  float *im_w;              // optional in-place threshold write-back
  void *mask_w;             //   (the mask in its own type)
  int FX, FY, FZ, s;        // full dims, shrink
  int X, Y, Z;              // fitting dims
  float *imlog;             // [X*Y*Z]
  long long start;          // first fitting voxel of this volume in the batch
  int mask_u8;              // mask and mask_w hold uint8_t
};

__device__ __forceinline__ bool mask_on(const void *m, int u8, long long i) {
  return u8 ? ((const unsigned char *)m)[i] != 0 : ((const float *)m)[i] != 0.0f;
}
__device__ __forceinline__ void mask_clear(void *m, int u8, long long i) {
  if (u8) ((unsigned char *)m)[i] = 0;
  else ((float *)m)[i] = 0.0f;
}

__device__ __forceinline__ int find_volume(const long long *starts, int n, long long gi) {
  int lo = 0, hi = n - 1;
  while (lo < hi) { int m = (lo + hi + 1) >> 1; if (starts[m] <= gi) lo = m; else hi = m - 1; }
  return lo;
}

// Rows of S consecutive voxels loaded as one vector: S floats, or S mask bytes.
template <int S> struct VecF;
template <> struct VecF<2> { using T = float2; };
template <> struct VecF<4> { using T = float4; };
template <int S> struct VecB;
template <> struct VecB<2> { using T = uchar2; };
template <> struct VecB<4> { using T = uchar4; };
__device__ __forceinline__ float vget(const float2 &v, int i) { return i == 0 ? v.x : v.y; }
__device__ __forceinline__ float vget(const float4 &v, int i) { return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w; }
__device__ __forceinline__ unsigned char vget(const uchar2 &v, int i) { return i == 0 ? v.x : v.y; }
__device__ __forceinline__ unsigned char vget(const uchar4 &v, int i) {
  return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// Fitting voxels g0 .. g0 + total - 1 of a batch (numbered as in
// PrologueVol::start) of the volumes vols[0 .. nvol); a non-finite voxel inside
// the mask sets flag_nonfinite[v] of its volume v.  S = 0: any shrink factor,
// scalar loads.  S = 2 or 4: that shrink factor, every volume with fewer than
// 2^31 fitting voxels and its rows of S voxels aligned to S floats (S bytes for
// a byte mask): the block's S*S rows are read as one vector load per row and
// array, all requested before they are summed, in the scalar path's order
// (the same sums, bitwise).  The loads' latency bounds S = 0 and 2, so both
// ask for 6 resident CTAs per SM (40 registers); S = 4 needs 62 for its
// 16-row batches and keeps 4.
template <int S>
__global__ void __launch_bounds__(256, S == 4 ? 4 : 6) k_prologue(const PrologueVol *vols, const long long *starts,
                                                                  int nvol, long long g0, long long total, float low,
                                                                  int *flag_nonfinite) {
  const long long end = g0 + total;
  for (long long gi = g0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; gi < end;
       gi += (long long)gridDim.x * blockDim.x) {
    const int v = find_volume(starts, nvol, gi);
    const PrologueVol &P = vols[v];
    float out;
    if constexpr (S == 0) {
      const long long li = gi - P.start;
      const int z = (int)(li % P.Z), y = (int)((li / P.Z) % P.Y), x = (int)(li / ((long long)P.Z * P.Y));
      const int s = P.s;
      if (s == 1) {
        const float val = P.im[li];
        const bool m = (P.mask ? mask_on(P.mask, P.mask_u8, li) : true) && val > low;
        if (m && !isfinite(val)) atomicExch(flag_nonfinite + v, 1);
        out = m ? logf(val) : __int_as_float(0x7fc00000);
        if (P.im_w && !(val > low)) { P.im_w[li] = 0.0f; if (P.mask_w) mask_clear(P.mask_w, P.mask_u8, li); }
      } else {
        float sum = 0.0f;
        int cnt = 0;
        for (int dx = 0; dx < s; ++dx)
          for (int dy = 0; dy < s; ++dy) {
            const long long rowb = ((long long)(x * s + dx) * P.FY + (y * s + dy)) * P.FZ + (long long)z * s;
            for (int dz = 0; dz < s; ++dz) {
              const float val = P.im[rowb + dz];
              const bool m = (P.mask ? mask_on(P.mask, P.mask_u8, rowb + dz) : true) && val > low;
              if (m) { sum += val; ++cnt; if (!isfinite(val)) atomicExch(flag_nonfinite + v, 1); }
            }
          }
        const float mean = cnt ? sum / (float)cnt : 0.0f;
        out = (2 * cnt > s * s * s && mean > low) ? logf(mean) : __int_as_float(0x7fc00000);
      }
      P.imlog[li] = out;
    } else {
      using VF = typename VecF<S>::T;
      using VB = typename VecB<S>::T;
      const unsigned li = (unsigned)(gi - P.start);
      const unsigned Z = (unsigned)P.Z, Y = (unsigned)P.Y;
      const unsigned q = li / Z, z = li - q * Z, x = q / Y, y = q - x * Y;
      const size_t FY = (size_t)P.FY, FZ = (size_t)P.FZ;
      // rows in batches of kB: the batch's loads are all requested before its
      // values are summed; the mask becomes one bit per voxel on arrival
      constexpr int kB = 4;
      float sum = 0.0f;
      int cnt = 0;
      bool bad = false;
#pragma unroll
      for (int r0 = 0; r0 < S * S; r0 += kB) {
        VF iv[kB];
        unsigned bits = 0;
#pragma unroll
        for (int j = 0; j < kB; ++j) {
          const int r = r0 + j;
          const size_t rowb = ((size_t)(x * S + r / S) * FY + (y * S + r % S)) * FZ + (size_t)z * S;
          iv[j] = *(const VF *)(P.im + rowb);
          unsigned mb = (1u << S) - 1u;
          if (P.mask && P.mask_u8) {
            const VB m = *(const VB *)((const unsigned char *)P.mask + rowb);
            mb = 0;
#pragma unroll
            for (int d = 0; d < S; ++d) mb |= (vget(m, d) != 0 ? 1u : 0u) << d;
          } else if (P.mask) {
            const VF m = *(const VF *)((const float *)P.mask + rowb);
            mb = 0;
#pragma unroll
            for (int d = 0; d < S; ++d) mb |= (vget(m, d) != 0.0f ? 1u : 0u) << d;
          }
          bits |= mb << (S * j);
        }
#pragma unroll
        for (int j = 0; j < kB; ++j)
#pragma unroll
          for (int d = 0; d < S; ++d) {
            const float val = vget(iv[j], d);
            const bool m = ((bits >> (S * j + d)) & 1u) && val > low;
            if (m) { sum += val; ++cnt; bad |= !isfinite(val); }
          }
      }
      if (bad) atomicExch(flag_nonfinite + v, 1);
      const float mean = cnt ? sum / (float)cnt : 0.0f;
      out = (2 * cnt > S * S * S && mean > low) ? logf(mean) : __int_as_float(0x7fc00000);
      P.imlog[li] = out;
    }
  }
}

// In-place threshold of the caller's full-resolution buffers (shrink > 1).
__global__ void k_threshold_inplace(float *im, void *mask, int mask_u8, long long n, float low) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (!(im[i] > low)) { im[i] = 0.0f; if (mask) mask_clear(mask, mask_u8, i); }
  }
}

// ------------------------------------------------------------------ warm-start input
// Input of the learned warm start: each volume's masked log fitting grid
// (the prologue's output, NaN outside the mask) averaged over 32x32x24
// adaptive cells [i*X/32, ceil((i+1)*X/32)) per axis, stored as BF16
// [volume][32][32][24].  A cell without a masked voxel is 0.
constexpr int kPoolX = 32, kPoolY = 32, kPoolZ = 24;
constexpr int kPoolCells = kPoolX * kPoolY * kPoolZ;

struct PoolJob {
  const float *imlog;
  int X, Y, Z;
};

__global__ void k_pool_fitgrid(const PoolJob *jobs, int nvol, __nv_bfloat16 *out) {
  const long long total = (long long)nvol * kPoolCells;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(t / kPoolCells), cell = (int)(t - (long long)v * kPoolCells);
    const PoolJob J = jobs[v];
    const int k = cell % kPoolZ, j = (cell / kPoolZ) % kPoolY, i = cell / (kPoolZ * kPoolY);
    const int x0 = i * J.X / kPoolX, x1 = ((i + 1) * J.X + kPoolX - 1) / kPoolX;
    const int y0 = j * J.Y / kPoolY, y1 = ((j + 1) * J.Y + kPoolY - 1) / kPoolY;
    const int z0 = k * J.Z / kPoolZ, z1 = ((k + 1) * J.Z + kPoolZ - 1) / kPoolZ;
    float s = 0.0f, c = 0.0f;
    for (int x = x0; x < x1; ++x)
      for (int y = y0; y < y1; ++y) {
        const float *row = J.imlog + ((long long)x * J.Y + y) * J.Z;
        for (int z = z0; z < z1; ++z) {
          const float val = row[z];
          if (!isnan(val)) { s += val; c += 1.0f; }
        }
      }
    out[t] = __float2bfloat16(c > 0.0f ? s / c : 0.0f);
  }
}

// ------------------------------------------------------------------ N4 kernels
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// Bounded wait for the given phase of an mbarrier; 1 when it completed.
__device__ unsigned mbar_wait(unsigned long long *mbar, unsigned phase) {
  unsigned done = 0;
  unsigned long long spins = 0;
  while (!done) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(mbar)), "r"(phase)
        : "memory");
    if (!done && ++spins > kSpinLimit) break;
  }
  return done;
}

// Stage rows rank, rank + K, ... of a [rows][Z] volume into consecutive
// shared-memory rows.  Rows whose size is a multiple of 16 bytes go by 1-D
// bulk (TMA) copies completing on an mbarrier; others by plain loads.  Every
// wait is bounded; returns false on timeout.
__device__ bool stage_rows(const float *src, int rank, int K, int nrow, int Z, float *dst,
                           unsigned long long *mbar, unsigned &phase, bool use_tma) {
  const bool bulk = use_tma && (Z % 4 == 0) && (((uintptr_t)src & 15u) == 0) && nrow > 0;
  if (!bulk) {
    for (int i = threadIdx.x; i < nrow * Z; i += blockDim.x) {
      const int rl = i / Z, z = i - rl * Z;
      dst[i] = src[(size_t)(rank + rl * K) * Z + z];
    }
    __syncthreads();
    return true;
  }
  const unsigned row_bytes = (unsigned)Z * 4u;
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)),
                 "r"(row_bytes * (unsigned)nrow)
                 : "memory");
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int rl = threadIdx.x; rl < nrow; rl += 32) {
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_u32(dst + (size_t)rl * Z)),
          "l"(src + (size_t)(rank + rl * K) * Z), "r"(row_bytes), "r"(smem_u32(mbar))
          : "memory");
    }
  }
  const unsigned done = mbar_wait(mbar, phase);
  phase ^= 1u;
  __syncthreads();
  return done != 0;
}

struct ClusterArgs {
  Plan pl;
  Params pr;
  const VolJob *jobs;
  const int *order;
  int njobs;
  int *queue;
  int use_tma;
};

template <int NT>
__global__ void __launch_bounds__(NT, 1) k_n4_cluster(const __grid_constant__ ClusterArgs a) {
  extern __shared__ __align__(128) char smem[];
  __shared__ Plan s_pl;
  __shared__ Params s_pr;
  __shared__ int s_job;
  __shared__ __align__(8) unsigned long long s_mbar;
  if (threadIdx.x == 0) {
    s_pl = a.pl;
    s_pr = a.pr;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_mbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  ClusterGroup g;
  char *sm = smem;
  char *big = smem + s_pl.sm_bytes;
  unsigned phase = 0;
  for (;;) {
    if (g.rank() == 0 && threadIdx.x == 0) s_job = atomicAdd(a.queue, 1);
    g.sync();
    const int j = *g.peer(&s_job, 0);
    g.sync();
    if (j >= a.njobs) break;
    const VolJob &job = a.jobs[a.order[j]];
    const int rank = g.rank(), K = g.size();
    const int nplane = job.X > rank ? (job.X - rank + K - 1) / K : 0;
    float *slab = (float *)(big + s_pl.b_imlog);
    // planes rank, rank + K, ... (each Y*Z contiguous floats)
    int ok = stage_rows(job.imlog, rank, K, nplane, job.Y * job.Z, slab, &s_mbar, phase, a.use_tma != 0) ? 1 : 0;
    if (!ok && threadIdx.x == 0) job.report->status = N4_ERR_TIMEOUT;
    // all CTAs of the cluster must agree before starting the volume
    __shared__ int s_ok;
    if (threadIdx.x == 0) s_ok = ok;
    g.sync();
    int all_ok = 1;
    for (int k = 0; k < g.size(); ++k) all_ok &= *g.peer(&s_ok, k);
    g.sync();
    if (!all_ok) {
      // a bulk copy did not complete in time: wait once more (bounded) for
      // this CTA's copies still in flight, then stop taking volumes
      if (!ok) mbar_wait(&s_mbar, phase ^ 1u);
      break;
    }
    Engine<ClusterGroup> e(g, s_pl, s_pr, sm, big, nullptr);
    e.run(job);   // the slab holds the staged rows
  }
}

struct GridArgs {
  Plan pl;
  Params pr;
  VolJob job;
  char *big_base;
  size_t big_stride;
  GridBarrier bar;
  float *red_global;
};

template <int NT>
__global__ void __launch_bounds__(NT, 1) k_n4_grid(const __grid_constant__ GridArgs a) {
  extern __shared__ __align__(128) char smem[];
  __shared__ Plan s_pl;
  __shared__ Params s_pr;
  if (threadIdx.x == 0) { s_pl = a.pl; s_pr = a.pr; }
  __syncthreads();
  GridGroup g{a.bar, a.big_base, a.big_stride};
  char *big = a.big_base + (size_t)blockIdx.x * a.big_stride;
  __shared__ EngineSlot<GridGroup> s_eng;
  Engine<GridGroup> &e = s_eng.make(g, s_pl, s_pr, smem, big, a.red_global);
  e.run(a.job);
}

// ------------------------------------------------------------------ tables
struct TableJob {
  char *base;     // axis table memory
  int n, nc;
};

__global__ void k_axis_tables(const TableJob *jobs) {
  const TableJob t = jobs[blockIdx.x];
  build_axis(axis_at(t.base, t.n, t.nc));
}

// ------------------------------------------------------------------ final correction
struct CorrectVol {
  const float *im;       // full resolution input (null: output the log field)
  float *out;            // im / exp(b)  or b
  float *bias;           // optional exp(b)
  const float *lattice;
  char *tx, *ty, *tz;    // axis tables (full resolution, final lattice)
  int FX, FY, FZ, ncx, ncy, ncz;
  long long tile0;       // first row tile of this volume in the batch
  int vec4;              // FZ % 4 == 0 and every pointer 16-byte aligned
};

constexpr int kMaxNcz = 64;
constexpr int kLxMax = 2048;    // x-contracted lattice slice ncy*ncz held per x-plane

// Tile shapes of the correction: full-resolution rows per tile and threads
// per CTA.  The autotuner times them per workload; kCorrectDefault is used
// when nothing is recorded.
struct CorrectShape {
  int rows, threads;
};
constexpr int kCorrectShapes = 6;
constexpr CorrectShape kCorrectShape[kCorrectShapes] = {{128, 256}, {64, 256}, {256, 256},
                                                         {512, 256}, {256, 512}, {512, 512}};
constexpr int kCorrectDefault = 0;
// Dynamic shared memory of a correction CTA: the two x-contracted planes and
// the tile's row contractions [rows][ncz].
__host__ __device__ inline size_t correct_smem_bytes(int rows, int ncz) {
  return (size_t)(2 * kLxMax + rows * ncz) * sizeof(float);
}

// One CTA per tile of `rt` full-resolution rows (vy fastest within
// an x-plane).  Contraction of the lattice for the tile's rows into shared
// memory, separable: per x-plane the tile touches, Lx[cy][cz] =
// sum_jx wx L[sx+jx][cy][cz]; per row, G[r][cz] = sum_jy wy Lx[sy+jy][cz]
// (a tile spanning more than two planes, or a slice larger than kLxMax,
// contracts each row directly).  Then z is evaluated per voxel with float4
// I/O.  HBM traffic: read im, write out (+ bias).
constexpr int kCorrectPre = 3;   // rows of input float4s a thread loads per step (two steps in flight)

// Tile `tile` of a batch (numbered as in CorrectVol::tile0) of the volumes
// vols[0 .. nvol); Gs and Lx in shared memory.  kLog: every volume's im is
// null and the log field is the output (its own instantiation: no input
// registers held).
template <bool kLog>
__device__ __forceinline__ void correct_tile(const CorrectVol *vols, const long long *tile_starts, int nvol,
                                             long long tile, float low, int rt, float *Gs, float *Lx) {
  const int v = find_volume(tile_starts, nvol, tile);
  const CorrectVol &C = vols[v];
  const Axis ax = axis_at(C.tx, C.FX, C.ncx), ay = axis_at(C.ty, C.FY, C.ncy), az = axis_at(C.tz, C.FZ, C.ncz);
  const long long rows = (long long)C.FX * C.FY;
  const long long row0 = (tile - C.tile0) * (long long)rt;
  const int nr = (int)min((long long)rt, rows - row0);
  const int ncz = C.ncz, ncy = C.ncy;
  const int FZ = C.FZ;
  const long long base = row0 * FZ;
  // float4 path: each thread owns 4 consecutive z (weights in registers) and
  // rows r_first, r_first + rpp, ...; it requests kCorrectPre input float4s
  // per step, the first ones before the barrier that ends the contraction
  const bool vec = C.vec4 != 0;
  const int nz4 = vec ? FZ >> 2 : 1;
  const int rpp = vec ? (int)blockDim.x / nz4 : 0;          // rows per pass (nz4 <= 256)
  const bool act = vec && (int)threadIdx.x < rpp * nz4;
  const int z = act ? ((int)threadIdx.x % nz4) * 4 : 0;
  const int r_first = act ? (int)threadIdx.x / nz4 : 0;
  {
    const unsigned FY = (unsigned)C.FY;
    const unsigned rw0 = (unsigned)row0;                     // rows of one volume < 2^32
    const int vxa = (int)(rw0 / FY), vxb = (int)((rw0 + (unsigned)nr - 1u) / FY);
    const int slice = ncy * ncz;
    if (vxb - vxa <= 1 && slice <= kLxMax) {
      const int np = vxb - vxa + 1;
      for (int t = threadIdx.x; t < np * slice; t += blockDim.x) {
        const int pl = t >= slice ? 1 : 0, c = t - pl * slice;
        const int vx = vxa + pl;
        const int sx = ax.s[vx];
        const float4 wx = ax.w[vx];
        const float *lp = C.lattice + (size_t)sx * slice + c;
        float acc = __fmul_rn(wx.x, __ldg(lp));
        acc = __fmaf_rn(wx.y, __ldg(lp + slice), acc);
        acc = __fmaf_rn(wx.z, __ldg(lp + 2 * slice), acc);
        Lx[t] = __fmaf_rn(wx.w, __ldg(lp + 3 * slice), acc);
      }
      __syncthreads();
      // entry (r, cz) at t = r * lanes + cz, lanes the power of two >= ncz
      // (no divisions); rows past the first plane's end continue in the next
      const int lsh = ncz <= 16 ? 4 : (ncz <= 32 ? 5 : 6);
      const int vy0 = (int)(rw0 - (unsigned)vxa * FY);
      for (int t = threadIdx.x; t < (nr << lsh); t += blockDim.x) {
        const int r = t >> lsh, cz = t & ((1 << lsh) - 1);
        if (cz >= ncz) continue;
        int vy = vy0 + r, pl = 0;
        if (vy >= (int)FY) { vy -= (int)FY; pl = 1; }
        const float *lx = Lx + pl * slice + ay.s[vy] * ncz + cz;
        const float4 wy = ay.w[vy];
        float acc = __fmul_rn(wy.x, lx[0]);
        acc = __fmaf_rn(wy.y, lx[ncz], acc);
        acc = __fmaf_rn(wy.z, lx[2 * ncz], acc);
        Gs[r * ncz + cz] = __fmaf_rn(wy.w, lx[3 * ncz], acc);
      }
    } else {
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
      for (int r = warp; r < nr; r += nwarp) {
        const unsigned row = rw0 + (unsigned)r;
        const int vx = (int)(row / FY), vy = (int)(row - (unsigned)vx * FY);
        const int sx = ax.s[vx], sy = ay.s[vy];
        const float4 wx = ax.w[vx], wy = ay.w[vy];
        const float wxa[4] = {wx.x, wx.y, wx.z, wx.w}, wya[4] = {wy.x, wy.y, wy.z, wy.w};
        for (int cz = lane; cz < ncz; cz += 32) {
          float lxv[4];
#pragma unroll
          for (int jy = 0; jy < 4; ++jy) {
            const float *lp = C.lattice + ((size_t)sx * ncy + sy + jy) * ncz + cz;
            float acc = __fmul_rn(wxa[0], __ldg(lp));
#pragma unroll
            for (int jx = 1; jx < 4; ++jx) acc = __fmaf_rn(wxa[jx], __ldg(lp + (size_t)jx * ncy * ncz), acc);
            lxv[jy] = acc;
          }
          float acc = __fmul_rn(wya[0], lxv[0]);
#pragma unroll
          for (int jy = 1; jy < 4; ++jy) acc = __fmaf_rn(wya[jy], lxv[jy], acc);
          Gs[r * ncz + cz] = acc;
        }
      }
    }
  }
  float4 xin[kCorrectPre];
  if (!kLog && act) {
#pragma unroll
    for (int k = 0; k < kCorrectPre; ++k) {
      const int r = r_first + k * rpp;
      xin[k] = r < nr ? __ldcs((const float4 *)(C.im + base + (long long)r * FZ + z)) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  __syncthreads();
  if (vec) {
    if (!act) return;
    int sz[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) sz[k] = az.s[z + k];
    // When the thread's 4 voxels lie in at most two spans (spans of >= 4
    // voxels), every row needs only G[s0 .. s0+4]: voxel q's value is
    // sum_j c[q][j] G[s0+j] with its 4 weights shifted by sz[q] - s0 and a
    // zero beside them, the same products and additions in the same order
    // as dot4 (a zero weight adds an exact zero).  5 shared loads per row
    // instead of 16.
    const int s0 = sz[0];
    const bool two = sz[3] - s0 <= 1;
    const bool has5 = s0 + 4 < ncz;
    float cq[4][5];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 w = az.w[z + q];
      const bool sh = sz[q] != s0;
      cq[q][0] = sh ? 0.0f : w.x;
      cq[q][1] = sh ? w.x : w.y;
      cq[q][2] = sh ? w.y : w.z;
      cq[q][3] = sh ? w.z : w.w;
      cq[q][4] = sh ? w.w : 0.0f;
    }
    // the thread's 4 voxels of the row whose contraction starts at g: the
    // two-span form above, or the general form (weights re-read, short spans)
    auto eval_two = [&](const float *g, float (&bz)[4]) {
      const float g0 = g[s0], g1 = g[s0 + 1], g2 = g[s0 + 2], g3 = g[s0 + 3];
      const float g4 = has5 ? g[s0 + 4] : 0.0f;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float b = __fmul_rn(cq[q][0], g0);
        b = __fmaf_rn(cq[q][1], g1, b);
        b = __fmaf_rn(cq[q][2], g2, b);
        b = __fmaf_rn(cq[q][3], g3, b);
        bz[q] = __fmaf_rn(cq[q][4], g4, b);
      }
    };
    auto eval_gen = [&](const float *g, float (&bz)[4]) {
#pragma unroll
      for (int q = 0; q < 4; ++q) bz[q] = dot4(az.w[z + q], g + sz[q]);
    };
    // the thread's rows r_first, r_first + rpp, ...: contractions gstep
    // floats apart, voxels step float4s apart (offsets within the tile < 2^31)
    const int gstep = rpp * ncz, step = rpp * (FZ >> 2);
    const float *g_first = Gs + r_first * ncz;
    const int v_first = r_first * (FZ >> 2) + (z >> 2);
    float4 *out4 = (float4 *)(C.out + base);
    auto rows = [&](auto &&ev) {
      if constexpr (kLog) {
        // the log field only (EvaluateBspline3D): stores, no loads
        const float *g = g_first;
        int v = v_first;
#pragma unroll 4
        for (int r = r_first; r < nr; r += rpp, g += gstep, v += step) {
          float bz[4];
          ev(g, bz);
          __stcs(out4 + v, make_float4(bz[0], bz[1], bz[2], bz[3]));
        }
      } else {
        const float4 *in4 = (const float4 *)(C.im + base);
        float4 *bias4 = C.bias ? (float4 *)(C.bias + base) : nullptr;
        const float *g = g_first;
        int v = v_first;
        for (int rb = r_first; rb < nr; rb += kCorrectPre * rpp, g += kCorrectPre * gstep, v += kCorrectPre * step) {
          // the next step's loads go out before this step's rows are evaluated
          // (double buffering: 4 % faster on the 96-volume bench batch)
          float4 xnx[kCorrectPre];
#pragma unroll
          for (int k = 0; k < kCorrectPre; ++k) {
            const int r = rb + (kCorrectPre + k) * rpp;
            xnx[k] = r < nr ? __ldcs(in4 + v + (kCorrectPre + k) * step) : make_float4(0.f, 0.f, 0.f, 0.f);
          }
#pragma unroll
          for (int k = 0; k < kCorrectPre; ++k) {
            if (rb + k * rpp >= nr) break;
            float bz[4];
            ev(g + k * gstep, bz);
            // im / exp(b) as im * exp(-b): one special-function op per voxel
            // (fast intrinsic, a few ulp); exp(b) only when it is an output
            const float xa[4] = {xin[k].x, xin[k].y, xin[k].z, xin[k].w};
            float o[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) o[q] = xa[q] > low ? xa[q] * __expf(-bz[q]) : 0.0f;
            if (bias4) {
              float e[4];
#pragma unroll
              for (int q = 0; q < 4; ++q) e[q] = __expf(bz[q]);
              __stcs(bias4 + v + k * step, make_float4(e[0], e[1], e[2], e[3]));
            }
            __stcs(out4 + v + k * step, make_float4(o[0], o[1], o[2], o[3]));
          }
#pragma unroll
          for (int k = 0; k < kCorrectPre; ++k) xin[k] = xnx[k];
        }
      }
    };
    if (two) rows(eval_two);
    else rows(eval_gen);
  } else {
    for (int t = threadIdx.x; t < nr * FZ; t += blockDim.x) {
      const int r = t / FZ, zz = t - r * FZ;
      const long long off = base + (long long)r * FZ + zz;
      const float b = dot4(az.w[zz], Gs + r * ncz + az.s[zz]);
      if constexpr (!kLog) {
        const float x = C.im[off];
        C.out[off] = x > low ? x * __expf(-b) : 0.0f;
        if (C.bias) C.bias[off] = __expf(b);
      } else {
        C.out[off] = b;
      }
    }
  }
}

// Tile t0 + blockIdx.x of a batch (numbered as in CorrectVol::tile0, tiles of
// `rt` rows) of the volumes vols[0 .. nvol); dynamic shared memory
// correct_smem_bytes(rt, ncz).  256 threads: 4 CTAs per SM for the log field
// (64 registers), 3 for the correction, whose loads in flight need more.
template <int NT, bool kLog>
__global__ void __launch_bounds__(NT, NT <= 256 ? (kLog ? 4 : 3) : 1) k_correct(const CorrectVol *vols,
                                                                   const long long *tile_starts, int nvol,
                                                                   long long t0, float low, int rt) {
  extern __shared__ __align__(16) float correct_sm[];
  correct_tile<kLog>(vols, tile_starts, nvol, t0 + blockIdx.x, low, rt, correct_sm + 2 * kLxMax, correct_sm);
}

// ------------------------------------------------------------------ standalone fit
constexpr int kFitRows = 128;   // rows per block (one thread each)
constexpr int kFitChunk = 32;   // z voxels staged per step

// T1[row][cz] (numerator and denominator) for every row of the field.  One
// thread per row walks z once with the 4 open targets of its current span in
// registers (a span's voxels feed targets s..s+3; target s is final when the
// walk leaves span s), so every voxel is read once and every target written
// once.  Rows are staged through shared memory in coalesced [rows][32] tiles.
__global__ void __launch_bounds__(kFitRows) k_fit_rows(const float *field, const float *mask, long long rows, int Z,
                                                       Axis az, float *t1n, float *t1d) {
  __shared__ float fs[kFitRows][kFitChunk + 1];
  __shared__ float ms[kFitRows][kFitChunk + 1];
  const long long row0 = (long long)blockIdx.x * kFitRows;
  const int nr = (int)min((long long)kFitRows, rows - row0);
  const int ncz = az.nc;
  const long long my = row0 + threadIdx.x;
  float n0 = 0.f, n1 = 0.f, n2 = 0.f, n3 = 0.f, d0 = 0.f, d1 = 0.f, d2 = 0.f, d3 = 0.f;
  int cur = 0;                                   // span of the open window
  for (int z0 = 0; z0 < Z; z0 += kFitChunk) {
    const int nz = min(kFitChunk, Z - z0);
    __syncthreads();
    for (int i = threadIdx.x; i < nr * kFitChunk; i += blockDim.x) {
      const int r = i / kFitChunk, z = i - r * kFitChunk;
      if (z < nz) {
        const long long g = (row0 + r) * Z + z0 + z;
        fs[r][z] = field[g];
        ms[r][z] = mask ? mask[g] : 1.0f;
      }
    }
    __syncthreads();
    if ((int)threadIdx.x < nr) {
      for (int z = 0; z < nz; ++z) {
        const int vz = z0 + z;
        const int sp = az.s[vz];
        while (cur < sp) {                       // close target `cur`
          t1n[my * ncz + cur] = n0;
          t1d[my * ncz + cur] = d0;
          n0 = n1; n1 = n2; n2 = n3; n3 = 0.f;
          d0 = d1; d1 = d2; d2 = d3; d3 = 0.f;
          ++cur;
        }
        if (ms[threadIdx.x][z] == 0.0f) continue;
        const float f = fs[threadIdx.x][z];
        const float4 p = az.p4[vz], q = az.q4[vz];
        n0 = __fmaf_rn(p.x, f, n0); n1 = __fmaf_rn(p.y, f, n1);
        n2 = __fmaf_rn(p.z, f, n2); n3 = __fmaf_rn(p.w, f, n3);
        d0 += q.x; d1 += q.y; d2 += q.z; d3 += q.w;
      }
    }
  }
  if ((int)threadIdx.x < nr) {
    // flush the open window and any targets after it
    const float nn[4] = {n0, n1, n2, n3}, dd[4] = {d0, d1, d2, d3};
    for (int c = cur; c < ncz; ++c) {
      const int k = c - cur;
      t1n[my * ncz + c] = k < 4 ? nn[k] : 0.0f;
      t1d[my * ncz + c] = k < 4 ? dd[k] : 0.0f;
    }
  }
}

// The same contraction for Z % 4 == 0, Z <= 1024 and 16-byte aligned field
// and mask, built for HBM bandwidth: one thread per row walks its row as in
// k_fit_rows (the sums are bitwise equal: the same fused multiply-adds in the
// same order; masked-out voxels add exact zeros), but reads it straight from
// global memory, S voxels per step and array, with D steps in flight in
// registers.  No shared-memory staging and no barrier after the z table is
// loaded: warps never wait for one another, so the loads of some warps
// overlap the arithmetic of others instead of the whole grid alternating
// between loading and walking.  S = 8 (Z % 8 == 0, 32-byte aligned rows):
// one 32-byte load per array and step, exactly one sector, not kept in L1;
// S = 4: 16-byte loads, the sector's other half served by L1.  R rows
// (threads) per CTA.  Dynamic shared memory: kFitTableBytes(Z) (the z table:
// numerator and denominator weights and the span of every voxel).
constexpr int kFitZMaxD = 1024;

// Shapes of the fit's z contraction: voxels per load step (16: 64-byte steps,
// 8: 32-byte steps, 4: 16-byte steps, 0: the shared-memory staged kernel
// k_fit_rows), steps in
// flight per thread and rows per CTA.  The autotuner times the ones the
// field's alignment allows; kFitDefault8 / kFitDefault4 are used otherwise.
struct FitShape {
  int step, depth, rows;
};
constexpr int kFitShapes = 13;
constexpr FitShape kFitShape[kFitShapes] = {{8, 3, 64},  {8, 2, 64},  {8, 4, 64},  {8, 3, 32},  {8, 3, 128},
                                            {8, 2, 128}, {4, 6, 64},  {4, 4, 64},  {4, 6, 128}, {0, 0, kFitRows},
                                            {16, 2, 64}, {16, 2, 32}, {16, 2, 128}};
constexpr int kFitDefault8 = 0, kFitDefault4 = 6, kFitScalar = 9;
__host__ __device__ inline size_t kFitTableBytes(int Z) { return (size_t)Z * 36; }

template <int S> struct FitStep { float v[S]; };

__device__ __forceinline__ void fit_load(FitStep<8> &x, const float *p) {
  asm("ld.global.nc.L1::no_allocate.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(x.v[0]), "=f"(x.v[1]), "=f"(x.v[2]), "=f"(x.v[3]), "=f"(x.v[4]), "=f"(x.v[5]), "=f"(x.v[6]),
        "=f"(x.v[7])
      : "l"(p));
}
// S = 16: two adjacent 32-byte sectors (one 64-byte DRAM burst) per array and step
__device__ __forceinline__ void fit_load(FitStep<16> &x, const float *p) {
  asm("ld.global.nc.L1::no_allocate.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(x.v[0]), "=f"(x.v[1]), "=f"(x.v[2]), "=f"(x.v[3]), "=f"(x.v[4]), "=f"(x.v[5]), "=f"(x.v[6]),
        "=f"(x.v[7])
      : "l"(p));
  asm("ld.global.nc.L1::no_allocate.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(x.v[8]), "=f"(x.v[9]), "=f"(x.v[10]), "=f"(x.v[11]), "=f"(x.v[12]), "=f"(x.v[13]), "=f"(x.v[14]),
        "=f"(x.v[15])
      : "l"(p + 8));
}
__device__ __forceinline__ void fit_load(FitStep<4> &x, const float *p) {
  asm("ld.global.nc.v4.f32 {%0,%1,%2,%3}, [%4];"
      : "=f"(x.v[0]), "=f"(x.v[1]), "=f"(x.v[2]), "=f"(x.v[3])
      : "l"(p));
}

// One row's walk: the 4 open targets cur..cur+3 (numerator and denominator),
// advanced S voxels at a time in the order of k_fit_rows.
struct FitWalk {
  float n0 = 0.f, n1 = 0.f, n2 = 0.f, n3 = 0.f, d0 = 0.f, d1 = 0.f, d2 = 0.f, d3 = 0.f;
  int cur = 0;             // span of the voxels being walked = first open target
  int end;                 // first voxel after span cur
  float *on, *od;          // the row's targets

  __device__ __forceinline__ void add(float f, float u, const float4 &p, const float4 &w) {
    n0 = __fmaf_rn(p.x, f, n0); n1 = __fmaf_rn(p.y, f, n1);
    n2 = __fmaf_rn(p.z, f, n2); n3 = __fmaf_rn(p.w, f, n3);
    d0 = __fmaf_rn(w.x, u, d0); d1 = __fmaf_rn(w.y, u, d1);
    d2 = __fmaf_rn(w.z, u, d2); d3 = __fmaf_rn(w.w, u, d3);
  }
  // voxels vq .. vq + S - 1 with field fa and mask ma
  template <int S>
  __device__ __forceinline__ void step(const float (&fa)[S], const float (&ma)[S], int vq, const float4 *sp4,
                                       const float4 *sq4, const int *ss, const int *span_hi) {
    if (vq + S > end) {
      // a span ends inside this step: voxel by voxel
#pragma unroll
      for (int j = 0; j < S; ++j) {
        const int sp = ss[vq + j];
        while (cur < sp) {
          on[cur] = n0;
          od[cur] = d0;
          n0 = n1; n1 = n2; n2 = n3; n3 = 0.f;
          d0 = d1; d1 = d2; d2 = d3; d3 = 0.f;
          ++cur;
        }
        const bool in = ma[j] != 0.0f;
        add(in ? fa[j] : 0.0f, in ? 1.0f : 0.0f, sp4[vq + j], sq4[vq + j]);
      }
      end = span_hi[cur];
    } else {
      // the whole step in the open span (the common case)
#pragma unroll
      for (int j = 0; j < S; ++j) {
        const bool in = ma[j] != 0.0f;
        add(in ? fa[j] : 0.0f, in ? 1.0f : 0.0f, sp4[vq + j], sq4[vq + j]);
      }
    }
  }
  // the open window and every target after it
  __device__ __forceinline__ void flush(int ncz) {
    for (int c = cur; c < ncz; ++c) {
      const int k = c - cur;
      on[c] = k == 0 ? n0 : k == 1 ? n1 : k == 2 ? n2 : k == 3 ? n3 : 0.0f;
      od[c] = k == 0 ? d0 : k == 1 ? d1 : k == 2 ? d2 : k == 3 ? d3 : 0.0f;
    }
  }
};

__device__ __forceinline__ void fit_table(const Axis &az, int Z, char *tab) {
  float4 *sp4 = (float4 *)tab, *sq4 = sp4 + Z;
  int *ss = (int *)(sq4 + Z);
  for (int i = threadIdx.x; i < Z; i += blockDim.x) {
    sp4[i] = az.p4[i];
    sq4[i] = az.q4[i];
    ss[i] = az.s[i];
  }
}

template <int S, int D, int R>
__global__ void __launch_bounds__(R, 512 / R) k_fit_rows_v5(const float *__restrict__ field,
                                                              const float *__restrict__ mask, long long rows, int Z,
                                                              Axis az, float *__restrict__ t1n,
                                                              float *__restrict__ t1d) {
  extern __shared__ __align__(16) char fit_tab[];
  const float4 *sp4 = (const float4 *)fit_tab, *sq4 = sp4 + Z;
  const int *ss = (const int *)(sq4 + Z);
  const long long row = (long long)blockIdx.x * R + threadIdx.x;
  const bool live = row < rows;
  const int nq = Z / S;                             // steps per row
  const float *fp = field + (live ? row : 0) * Z;
  const float *mp = mask ? mask + (live ? row : 0) * Z : nullptr;
  FitStep<S> F[D], M[D];
  // the first steps are requested before the table is built
#pragma unroll
  for (int k = 0; k < D; ++k) {
    if (live && k < nq) {
      fit_load(F[k], fp + k * S);
      if (mp) fit_load(M[k], mp + k * S);
    }
  }
  fit_table(az, Z, fit_tab);
  __syncthreads();
  if (!live) return;
  const int ncz = az.nc;
  FitWalk w;
  w.end = az.hi[0];
  w.on = t1n + row * ncz;
  w.od = t1d + row * ncz;
  for (int q0 = 0; q0 < nq; q0 += D) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
      const int q = q0 + k;
      if (q >= nq) break;
      float fa[S], ma[S];
#pragma unroll
      for (int j = 0; j < S; ++j) {
        fa[j] = F[k].v[j];
        ma[j] = mp ? M[k].v[j] : 1.0f;
      }
      // step q is in registers: request step q + D into its slot
      if (q + D < nq) {
        fit_load(F[k], fp + (q + D) * S);
        if (mp) fit_load(M[k], mp + (q + D) * S);
      }
      w.step<S>(fa, ma, S * q, sp4, sq4, ss, az.hi);
    }
  }
  w.flush(ncz);
}

// T2[vx][cy][cz] from T1.
__global__ void k_fit_planes(const float *t1n, const float *t1d, int X, int Y, Axis ay, int ncz,
                             float *t2n, float *t2d) {
  const int ncy = ay.nc;
  const long long ntask = (long long)X * ncy * ncz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntask;
       t += (long long)gridDim.x * blockDim.x) {
    const int cz = (int)(t % ncz), cy = (int)((t / ncz) % ncy);
    const long long vx = t / ((long long)ncz * ncy);
    KahanSum an, ad;
    for (int j = 0; j < 4; ++j) {
      const int sp = cy - j;
      if (sp < 0 || sp >= ay.nsp) continue;
      for (int vy = ay.lo[sp]; vy < ay.hi[sp]; ++vy) {
        const long long i = (vx * Y + vy) * ncz + cz;
        an.add_prod(ay.p[j * Y + vy], t1n[i]);
        ad.add_prod(ay.q[j * Y + vy], t1d[i]);
      }
    }
    t2n[t] = an.value();
    t2d[t] = ad.value();
  }
}

__global__ void k_fit_final(const float *t2n, const float *t2d, int X, Axis ax, int ncy, int ncz,
                            float eps, int zero_den, float *lattice) {
  const int ncx = ax.nc;
  const int nlat = ncx * ncy * ncz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nlat; c += gridDim.x * blockDim.x) {
    const int cz = c % ncz, cy = (c / ncz) % ncy, cx = c / (ncz * ncy);
    KahanSum sn, sd;
    for (int j = 0; j < 4; ++j) {
      const int sp = cx - j;
      if (sp < 0 || sp >= ax.nsp) continue;
      for (int vx = ax.lo[sp]; vx < ax.hi[sp]; ++vx) {
        const long long i = ((long long)vx * ncy + cy) * ncz + cz;
        sn.add_prod(ax.p[j * X + vx], t2n[i]);
        sd.add_prod(ax.q[j * X + vx], t2d[i]);
      }
    }
    const float an = sn.value(), ad = sd.value();
    lattice[c] = zero_den ? (ad != 0.0f ? an / ad : 0.0f) : an / (ad + eps);
  }
}

__global__ void k_refine(const float *in, int ncx, int ncy, int ncz, float *out) {
  refine_lattice(in, ncx, ncy, ncz, out);
}

// ------------------------------------------------------------------ standalone sharpen
__global__ void k_minmax(const float *x, const float *mask, long long n, float *part) {
  float vmin = INFINITY, vmax = -INFINITY;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (mask && mask[i] == 0.0f) continue;
    vmin = fminf(vmin, x[i]);
    vmax = fmaxf(vmax, x[i]);
  }
  __shared__ double scratch[160];
  double out[4];
  block_reduce4(vmin, vmax, 0.0, 0.0, scratch + 8, out);
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = (float)out[0]; part[2 * blockIdx.x + 1] = (float)out[1]; }
}

// stats[0] = min, stats[1] = max, stats[2] = slope, stats[3] = 1 / slope (FP64)
__global__ void k_minmax_final(const float *part, int nb, int bins, double *stats) {
  float vmin = INFINITY, vmax = -INFINITY;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) { vmin = fminf(vmin, part[2 * i]); vmax = fmaxf(vmax, part[2 * i + 1]); }
  __shared__ double scratch[160];
  double out[4];
  block_reduce4(vmin, vmax, 0.0, 0.0, scratch + 8, out);
  if (threadIdx.x == 0) {
    const double slope = (out[1] - out[0]) / (double)(bins - 1);
    stats[0] = out[0];
    stats[1] = out[1];
    stats[2] = slope;
    stats[3] = (slope > 0.0 && isfinite(slope)) ? 1.0 / slope : 0.0;
  }
}

__global__ void k_hist(const float *x, const float *mask, long long n, const double *stats, int bins, int shift,
                       unsigned long long *hist) {
  extern __shared__ unsigned hs[];
  for (int i = threadIdx.x; i < bins; i += blockDim.x) hs[i] = 0u;
  __syncthreads();
  const double inv = stats[3];
  const BinMap bm(stats[0], inv > 0.0 ? stats[2] : 1.0, bins);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = blockIdx.x * (long long)blockDim.x; base < n; base += stride) {
    const long long i = base + threadIdx.x;
    int key = -1;
    unsigned qlo = 0, qhi = 0;
    if (i < n && inv > 0.0 && (!mask || mask[i] != 0.0f)) key = hist_bin(bm.coord(x[i]), bins, ldexp(1.0, shift), qlo, qhi);
    hist_add_warp(hs, bins, key, qlo, qhi);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bins; i += blockDim.x)
    if (hs[i]) atomicAdd(&hist[i], (unsigned long long)hs[i]);
}

__global__ void k_sharpen(const unsigned long long *hist, const double *stats, int bins, int shift, int npad,
                          int hoff, double wiener, double fwhm, double *E_out) {
  extern __shared__ __align__(16) char sm[];
  double2 *fa = (double2 *)sm, *fb = fa + npad, *tw = fb + npad;
  double *Ff = (double *)(tw + npad);
  double *E = Ff + npad;
  fft_twiddles(tw, npad);
  __syncthreads();
  if (stats[3] > 0.0) {
    SharpenBufs sb{fa, fb, tw, Ff};
    const double inv = ldexp(1.0, -shift);
    sharpen_map([=](int b) { return (double)hist[b] * inv; }, bins, npad, hoff, stats[0], stats[2], wiener, fwhm,
                sb, E);
    for (int b = threadIdx.x; b < bins; b += blockDim.x) E_out[b] = E[b];
  } else {
    for (int b = threadIdx.x; b < bins; b += blockDim.x) E_out[b] = 0.0;
  }
}

__global__ void k_remap(const float *x, const float *mask, long long n, const double *stats, const double *E,
                        int bins, float *out) {
  const double inv = stats[3];
  const BinMap bm(stats[0], inv > 0.0 ? stats[2] : 1.0, bins);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (mask && mask[i] == 0.0f) { out[i] = 0.0f; continue; }
    out[i] = inv > 0.0 ? (float)sharpened_value(bm.coord(x[i]), E, bins) : x[i];
  }
}

// ------------------------------------------------------------------ autotuner helper
// Reads n float4s (and writes one value that depends on them, so the reads
// stay): run before a timed kernel to evict its inputs from L2 with clean
// lines, so that the timed kernel reads from HBM and no write-back lands in it.
__global__ void k_read_evict(const float4 *p, long long n, float *sink) {
  float acc = 0.0f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float4 v = __ldcg(p + i);   // normal L2 allocation (a streaming load would be evicted first)
    acc += v.x + v.y + v.z + v.w;
  }
  if (acc == 1.2345678f) *sink = acc;   // practically never true; keeps the loads
}

// ------------------------------------------------------------------ standalone convergence
__global__ void k_cv(const float *f1, const float *f2, const float *mask, long long n, double *part) {
  double s0 = 0.0, s1 = 0.0, c = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (mask && mask[i] == 0.0f) continue;
    const double y = (double)expm1f(__fsub_rn(f1[i], f2[i]));
    s0 += y; s1 += y * y; c += 1.0;
  }
  s0 = warp_sum(s0); s1 = warp_sum(s1); c = warp_sum(c);
  __shared__ double ws[3][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { ws[0][wid] = s0; ws[1][wid] = s1; ws[2][wid] = c; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, d = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += ws[0][w]; b += ws[1][w]; d += ws[2][w]; }
    part[3 * blockIdx.x] = a;
    part[3 * blockIdx.x + 1] = b;
    part[3 * blockIdx.x + 2] = d;
  }
}

}  // namespace n4
