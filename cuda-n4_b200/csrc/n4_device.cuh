// Device helpers shared by every n4b200 kernel (sm_100a).
//
// * per-axis cubic B-spline tables (span index, weights, fit weights),
//   computed in FP64 with the reference's formulas (N4.py:174-181,
//   N4.py:210-222) and stored in FP32;
// * a CTA-level Stockham radix-8/4/2 FFT in shared memory and the Gaussian
//   Wiener-deconvolution sharpening map built on it (N4.py:32-101,
//   cudaN4.cu:733-817);
// * fractional-histogram binning and the piecewise-linear remap
//   (N4.py:14-29, N4.py:103-113);
// * warp/CTA reductions and a bounded software grid barrier.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/n4b200.h"

namespace n4 {

constexpr int kMaxThreads = 1024;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kHistCopies = 8;                   // shared histogram copies per CTA
constexpr int kHistMaxShift = 24;                // fixed-point weight 2^shift, shift <= 24
constexpr unsigned long long kSpinLimit = 1ull << 25;   // bounded waits (~2-4 s)

// ---------------------------------------------------------------- tables
// One axis of the fitting grid at one level.  Arrays live in shared or
// global memory; all pointers are generic.
struct Axis {
  int n;        // voxels along the axis
  int nc;       // control points (= spans + 3)
  int nsp;      // spans
  int *s;       // [n]   span index of each voxel
  float4 *w;    // [n]   cubic weights B0..B3
  float *p;     // [4][n] fit numerator weights  w_j^3 / sum_k w_k^2
  float *q;     // [4][n] fit denominator weights w_j^2
  float4 *p4;   // [n]   the same numerator weights, packed per voxel
  float4 *q4;   // [n]   the same denominator weights, packed per voxel
  int *lo, *hi; // [nsp] voxel range of each span
};

// Byte size of an axis table with `n` voxels and `nsp` spans (16-B multiple).
__host__ __device__ inline size_t axis_bytes(int n, int nsp) {
  size_t b = 0;
  b += ((size_t)n * 4 + 15) / 16 * 16;          // s
  b += (size_t)n * 16;                           // w
  b += (size_t)n * 16 * 2;                       // p, q
  b += (size_t)n * 16 * 2;                       // p4, q4
  b += ((size_t)nsp * 8 + 15) / 16 * 16;         // lo, hi
  return b;
}

__host__ __device__ inline Axis axis_at(char *base, int n, int nc) {
  Axis a;
  a.n = n; a.nc = nc; a.nsp = nc - 3;
  char *p = base;
  a.s = (int *)p;    p += ((size_t)n * 4 + 15) / 16 * 16;
  a.w = (float4 *)p; p += (size_t)n * 16;
  a.p = (float *)p;  p += (size_t)n * 16;
  a.q = (float *)p;  p += (size_t)n * 16;
  a.p4 = (float4 *)p; p += (size_t)n * 16;
  a.q4 = (float4 *)p; p += (size_t)n * 16;
  a.lo = (int *)p;   a.hi = a.lo + a.nsp;
  return a;
}

// Span index of voxel i, as N4.py:210 computes it: floor((i + 0.5) / span)
// with span = n / nspans, all in IEEE FP64 (no contraction).
__device__ __forceinline__ int span_of(int i, double span, int nsp) {
  double u = __dadd_rn((double)i, 0.5);
  int s = (int)floor(__ddiv_rn(u, span));
  return s < 0 ? 0 : (s >= nsp ? nsp - 1 : s);
}

// Fill one axis table with the CTA's threads (caller synchronises).
__device__ void build_axis(const Axis &a) {
  const double span = __ddiv_rn((double)a.n, (double)a.nsp);
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) {
    int s = span_of(i, span, a.nsp);
    double u = __dadd_rn((double)i, 0.5);
    double t = __ddiv_rn(__dsub_rn(u, __dmul_rn((double)s, span)), span);
    double t2 = t * t, t3 = t * t * t, tm = 1.0 - t;
    double w0 = tm * tm * tm / 6.0;
    double w1 = (3.0 * t3 - 6.0 * t2 + 4.0) / 6.0;
    double w2 = (-3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0) / 6.0;
    double w3 = t3 / 6.0;
    double S = w0 * w0 + w1 * w1 + w2 * w2 + w3 * w3;
    a.s[i] = s;
    a.w[i] = make_float4((float)w0, (float)w1, (float)w2, (float)w3);
    a.p[0 * a.n + i] = (float)(w0 * w0 * w0 / S);
    a.p[1 * a.n + i] = (float)(w1 * w1 * w1 / S);
    a.p[2 * a.n + i] = (float)(w2 * w2 * w2 / S);
    a.p[3 * a.n + i] = (float)(w3 * w3 * w3 / S);
    a.q[0 * a.n + i] = (float)(w0 * w0);
    a.q[1 * a.n + i] = (float)(w1 * w1);
    a.q[2 * a.n + i] = (float)(w2 * w2);
    a.q[3 * a.n + i] = (float)(w3 * w3);
    a.p4[i] = make_float4(a.p[i], a.p[a.n + i], a.p[2 * a.n + i], a.p[3 * a.n + i]);
    a.q4[i] = make_float4(a.q[i], a.q[a.n + i], a.q[2 * a.n + i], a.q[3 * a.n + i]);
  }
  // voxel range of every span by binary search on the monotone span index
  for (int sp = threadIdx.x; sp < a.nsp; sp += blockDim.x) {
    int lo = 0, hi = a.n;              // first voxel with span >= sp
    while (lo < hi) { int m = (lo + hi) >> 1; if (span_of(m, span, a.nsp) >= sp) hi = m; else lo = m + 1; }
    int l2 = lo, h2 = a.n;             // first voxel with span >= sp + 1
    while (l2 < h2) { int m = (l2 + h2) >> 1; if (span_of(m, span, a.nsp) >= sp + 1) h2 = m; else l2 = m + 1; }
    a.lo[sp] = lo;
    a.hi[sp] = l2;
  }
}

// b = sum_j w_j g[j] with a fixed association (identical in every pass).
__device__ __forceinline__ float dot4(float4 w, const float *g) {
  float b = __fmul_rn(w.x, g[0]);
  b = __fmaf_rn(w.y, g[1], b);
  b = __fmaf_rn(w.z, g[2], b);
  b = __fmaf_rn(w.w, g[3], b);
  return b;
}

// Exact floor(i / d) for 0 <= i < 2^22 and 1 <= d <= 2^10 via a 32-bit magic.
struct FastDiv {
  unsigned d, m;
  __host__ __device__ FastDiv() : d(1), m(0) {}
  __host__ __device__ explicit FastDiv(unsigned dd) : d(dd), m((unsigned)((0x100000000ull + dd - 1) / dd)) {}
  __device__ __forceinline__ unsigned div(unsigned i) const { return d == 1 ? i : __umulhi(i, m); }
};

// GPU global timer (ns) and the SM this thread runs on.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ int sm_id() {
  unsigned r;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
  return (int)r;
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ float warp_min(float v) {
  for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Kahan-compensated FP32 sum (Kahan, CACM 8(1), 1965): `s` is the running
// sum and `c` the part of the last addition that `s` could not hold, fed
// back into the next term.  The error of a compensated sum of n terms is
// bounded by ~2u sum|x_i| independently of n (u = 2^-24), instead of the
// ~n u sum|x_i| of a plain recursive sum.  The intrinsics keep the compiler
// from contracting or reassociating the steps.
struct KahanSum {
  float s = 0.0f, c = 0.0f;
  __device__ __forceinline__ void add(float x) {
    const float y = __fsub_rn(x, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
  }
  // adds w * x (the product rounded once, inside the first step)
  __device__ __forceinline__ void add_prod(float w, float x) {
    const float y = __fmaf_rn(w, x, -c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
  }
  __device__ __forceinline__ float value() const { return __fsub_rn(s, c); }
  // adds another compensated sum
  __device__ __forceinline__ void merge(const KahanSum &o) { add(o.value()); }
};

// CTA-wide reduction of four values (min, max, sum, sum) into out[0..3] of
// thread 0; `scratch` holds 4 * 32 doubles.  Deterministic order.
__device__ void block_reduce4(float vmin, float vmax, double s0, double s1,
                              double *scratch, double out[4]) {
  vmin = warp_min(vmin); vmax = warp_max(vmax); s0 = warp_sum(s0); s1 = warp_sum(s1);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) {
    scratch[wid] = vmin; scratch[32 + wid] = vmax; scratch[64 + wid] = s0; scratch[96 + wid] = s1;
  }
  __syncthreads();
  if (wid == 0) {
    float a = lane < nw ? (float)scratch[lane] : INFINITY;
    float b = lane < nw ? (float)scratch[32 + lane] : -INFINITY;
    double c = lane < nw ? scratch[64 + lane] : 0.0;
    double d = lane < nw ? scratch[96 + lane] : 0.0;
    a = warp_min(a); b = warp_max(b); c = warp_sum(c); d = warp_sum(d);
    if (lane == 0) { out[0] = a; out[1] = b; out[2] = c; out[3] = d; }
  }
  __syncthreads();
}

// ---------------------------------------------------------------- FFT (FP64)
// The sharpening map is computed in double precision: N4 accumulates the
// residual logU - E(logU), a small difference of O(1) values, so a relative
// error of 1e-6 in E moves the fitted lattice by ~2e-4 after a few dozen
// iterations.  The map is O(bins) work per iteration; every volume-sized
// quantity stays in FP32.
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }  // a * (-i)

__device__ __forceinline__ void dft2(double2 *v) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b); v[1] = csub(a, b);
}
__device__ __forceinline__ void dft4(double2 &v0, double2 &v1, double2 &v2, double2 &v3) {
  double2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = mul_mi(csub(v1, v3));
  v0 = cadd(t0, t2); v2 = csub(t0, t2); v1 = cadd(t1, t3); v3 = csub(t1, t3);
}
__device__ __forceinline__ void dft8(double2 *v) {
  const double c = 0.70710678118654752440;
  double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4(e0, e1, e2, e3);
  dft4(o0, o1, o2, o3);
  o1 = make_double2(c * (o1.x + o1.y), c * (o1.y - o1.x));   // * e^{-i pi/4}
  o2 = mul_mi(o2);                                            // * e^{-i pi/2}
  o3 = make_double2(c * (o3.y - o3.x), -c * (o3.x + o3.y));  // * e^{-3i pi/4}
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

// tw[m] = exp(-2 pi i m / N), m in [0, N).
__device__ void fft_twiddles(double2 *tw, int N) {
  for (int m = threadIdx.x; m < N; m += blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)m / (double)N, &s, &c);
    tw[m] = make_double2(c, s);
  }
}

// One Stockham pass of radix R (Govindaraju et al., SC'08, "High performance
// discrete Fourier transforms on graphics processors"): x -> y.
template <int R>
__device__ void stockham_pass(const double2 *x, double2 *y, int N, int Ns, const double2 *tw) {
  const int T = N / R;
  const int tstep = N / (Ns * R);
  for (int j = threadIdx.x; j < T; j += blockDim.x) {
    const int k = j & (Ns - 1);
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      v[r] = x[j + r * T];
      if (r) v[r] = cmul(v[r], tw[(r * k * tstep) & (N - 1)]);
    }
    if (R == 8) dft8(v);
    else if (R == 4) dft4(v[0], v[1], v[2], v[3]);
    else dft2(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) y[base + r * Ns] = v[r];
  }
}

template <int R> __device__ __forceinline__ void dft_r(double2 *v);
template <> __device__ __forceinline__ void dft_r<2>(double2 *v) { dft2(v); }
template <> __device__ __forceinline__ void dft_r<4>(double2 *v) { dft4(v[0], v[1], v[2], v[3]); }
template <> __device__ __forceinline__ void dft_r<8>(double2 *v) { dft8(v); }

// Largest radix used by the FFT passes (4: five passes for N = 512).
#ifndef N4_FFT_MAX_RADIX
#define N4_FFT_MAX_RADIX 4
#endif
__device__ __forceinline__ int fft_radix(int rem) {
  return (N4_FFT_MAX_RADIX >= 8 && rem % 8 == 0) ? 8 : (rem % 4 == 0 ? 4 : 2);
}

// First Stockham pass (Ns = 1: every twiddle is 1) of an FFT whose input
// x[i] = in(i) is produced on the fly, so that the elementwise step before an
// FFT needs no pass and no barrier of its own.
template <int R, class In>
__device__ void stockham_first(const In &in, double2 *y, int N) {
  const int T = N / R;
  for (int j = threadIdx.x; j < T; j += blockDim.x) {
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in(j + r * T);
    dft_r<R>(v);
#pragma unroll
    for (int r = 0; r < R; ++r) y[j * R + r] = v[r];
  }
}

// Forward FFT (length N = 2^m, 4 <= N <= 4096) of in(0..N): first pass into
// a, then the remaining passes ping-ponging a and b, each ending with a CTA
// barrier.  Returns the buffer that holds the result.
template <class In>
__device__ double2 *fft_from(const In &in, double2 *a, double2 *b, int N, const double2 *tw) {
  const int R0 = fft_radix(N);
  if (R0 == 8) stockham_first<8>(in, a, N);
  else if (R0 == 4) stockham_first<4>(in, a, N);
  else stockham_first<2>(in, a, N);
  __syncthreads();
  int Ns = R0, rem = N / R0;
  while (rem > 1) {
    const int R = fft_radix(rem);
    if (R == 8) stockham_pass<8>(a, b, N, Ns, tw);
    else if (R == 4) stockham_pass<4>(a, b, N, Ns, tw);
    else stockham_pass<2>(a, b, N, Ns, tw);
    __syncthreads();
    double2 *t = a; a = b; b = t;
    Ns *= R;
    rem /= R;
  }
  return a;
}

// ---------------------------------------------------------------- sharpening
struct SharpenBufs {
  double2 *a, *b;    // [N] work buffers
  double2 *tw;       // [N] twiddles (filled by the caller once)
  double *Ff;        // [N] real Fourier transform of the Gaussian
};

// E[0..bins) from the fractional histogram (bin b's weight hv(b)) (N4.py:32-101,
// cudaN4.cu:733-817), all in FP64; all threads of the CTA call it.  Four FFTs;
// each elementwise step is folded into the first pass of the FFT after it.
// R2 (optional): the residual table of residual_lin, R2[b] for b < bins - 1.
template <class HistF>
__device__ void sharpen_map(const HistF &hv, int bins, int N, int off, double binMin, double slope,
                            double wiener, double fwhm, const SharpenBufs &sb, double *E, float2 *R2 = nullptr) {
  const double ln2 = 0.69314718055994530942;
  const double scaledFWHM = fwhm / slope;
  const double expFactor = 4.0 * ln2 / (scaledFWHM * scaledFWHM);
  const double scaleFactor = 2.0 * sqrt(ln2 / 3.14159265358979323846) / scaledFWHM;
  const double invN = 1.0 / (double)N;
  // the periodic Gaussian's N/2 + 1 distinct values, one per thread of the
  // CTA (the first FFT pass has only N/4 threads busy), held in sb.Ff until
  // the second FFT overwrites it with the transform
  for (int d = threadIdx.x; d <= N / 2; d += blockDim.x)
    sb.Ff[d] = scaleFactor * exp(-(double)d * (double)d * expFactor);
  __syncthreads();
  // z = V + i F : the padded histogram and the periodic Gaussian in one FFT
  double2 *Z = fft_from(
      [&](int i) {
        const int d = i <= N / 2 ? i : N - i;
        const double F = sb.Ff[d];
        const double V = (i >= off && i < off + bins) ? hv(i - off) : 0.0;
        return make_double2(V, F);
      },
      sb.a, sb.b, N, sb.tw);
  double2 *W = (Z == sb.a) ? sb.b : sb.a;
  // split the packed transform; Wiener filter Re(conj(Ff)/(|Ff|^2 + w)) with
  // Ff real; conj(Uf), so that the forward FFT inverts
  double2 *Y = fft_from(
      [&](int k) {
        const double2 zk = Z[k], zn = Z[(N - k) & (N - 1)];
        const double2 Vf = make_double2(0.5 * (zk.x + zn.x), 0.5 * (zk.y - zn.y));
        const double Ff = 0.5 * (zk.y + zn.y);
        const double g = Ff / (Ff * Ff + wiener);
        sb.Ff[k] = Ff;
        return make_double2(Vf.x * g, -Vf.y * g);
      },
      W, Z, N, sb.tw);
  double2 *Y2 = (Y == W) ? Z : W;
  // U = max(Re(ifft(Uf)), 0); pack the numerator c_i U_i (real) and U (imaginary)
  double2 *P = fft_from(
      [&](int i) {
        const double U = fmax(Y[i].x * invN, 0.0);
        const double c = binMin + (double)(i - off) * slope;
        return make_double2(c * U, U);
      },
      Y2, Y, N, sb.tw);
  double2 *P2 = (P == Y2) ? Y : Y2;
  // Gaussian smoothing of both: multiply by the (real) Ff, inverse transform
  double2 *S = fft_from(
      [&](int k) {
        const double2 v = P[k];
        const double f = sb.Ff[k];
        return make_double2(v.x * f, -v.y * f);
      },
      P2, P, N, sb.tw);
  auto e_at = [&](int b) {
    const double2 v = S[off + b];
    const double nu = v.x * invN, de = -v.y * invN;
    return (de != 0.0) ? nu / de : 0.0;
  };
  for (int b = threadIdx.x; b < bins; b += blockDim.x) {
    const double e = e_at(b);
    E[b] = e;
    if (R2 && b + 1 < bins)
      R2[b] = make_float2((float)(binMin + (double)b * slope - e), (float)(slope - (e_at(b + 1) - e)));
  }
  __syncthreads();
}

// Float-float arithmetic (a value as the unevaluated sum of two floats, ~48
// significant bits): Knuth's TwoSum and the FMA form of Dekker's TwoProduct
// are error-free, so x - binMin and products keep their rounding errors
// exactly.  The _rn intrinsics keep the compiler from contracting or
// reassociating these sequences.
__device__ __forceinline__ float two_sum(float a, float b, float &err) {
  const float s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  err = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return s;
}

// Bin coordinate of a value, (x - binMin) / slope, in FP64.  The reciprocal
// product is within an ulp of the quotient; near the last bin the quotient
// itself is taken, because there one ulp decides whether the reference
// counts or drops the maximum voxel (N4.py:27).
//
// coord_ff gives the same coordinate from float-float arithmetic as a bin k
// and a fraction f (|error| < 2^-24, the resolution of the histogram's fixed
// point): d = x - binMin exactly by TwoSum (binMin is the minimum of FP32
// values, a float), times 1/slope held as a float-float.  It declines values
// within two bins of the top, which take the FP64 path.
struct BinMap {
  double binMin, slope, inv_slope, top;
  float fmin, ih, il, ff_limit;
  __device__ BinMap(double mn, double sl, int bins)
      : binMin(mn), slope(sl), inv_slope(1.0 / sl), top((double)bins - 1.5), fmin((float)mn),
        ih((float)inv_slope), il((float)(inv_slope - (double)ih)), ff_limit((float)(bins - 2)) {}
  __device__ __forceinline__ double coord(float x) const {
    const double d = (double)x - binMin;
    const double c = d * inv_slope;
    return c > top ? d / slope : c;
  }
  __device__ __forceinline__ bool coord_ff(float x, int &k, float &f) const {
    float dl;
    const float dh = two_sum(x, -fmin, dl);                  // x - binMin = dh + dl exactly
    const float p = __fmul_rn(dh, ih);
    const float pe = __fmaf_rn(dh, ih, -p);                  // p + pe = dh * ih exactly
    const float cl = __fadd_rn(pe, __fmaf_rn(dh, il, __fmul_rn(dl, ih)));
    if (!(p < ff_limit)) return false;                       // near the top bin (or NaN)
    const float kf = floorf(p);
    f = __fadd_rn(__fsub_rn(p, kf), cl);                     // p - kf is exact
    k = (int)kf;
    if (f < 0.0f) { f = __fadd_rn(f, 1.0f); --k; }
    else if (f >= 1.0f) { f = __fsub_rn(f, 1.0f); ++k; }
    if (k < 0) { k = 0; f = 0.0f; }                          // x >= binMin: only rounding reaches here
    return true;
  }
};

// exp(x) - 1 of a convergence term (N4.py:121-126): for |x| < 1/4 its Taylor
// series through x^7 / 7! in Horner form, x + x^2 (1/2! + x (1/3! + ...)),
// whose truncation is below x^7 / 8! < 2^-28 relative and whose last step
// is one fused multiply-add (0.65 ulp at most against FP64 over 2^21 samples
// of the interval); expm1f beyond (first iterations of a level).
__device__ __forceinline__ float expm1_conv(float x) {
  if (fabsf(x) < 0.25f) {
    float p = __fmaf_rn(x, 1.0f / 5040.0f, 1.0f / 720.0f);
    p = __fmaf_rn(p, x, 1.0f / 120.0f);
    p = __fmaf_rn(p, x, 1.0f / 24.0f);
    p = __fmaf_rn(p, x, 1.0f / 6.0f);
    p = __fmaf_rn(p, x, 0.5f);
    return __fmaf_rn(__fmul_rn(x, x), p, x);
  }
  return expm1f(x);
}

// Fractional histogram contribution of one value (N4.py:21-29) from its
// FP64 bin coordinate, as fixed-point weights of 2^shift per voxel (the two
// parts of a split add up to exactly one voxel).  Returns the bin or -1 when
// the value adds nothing.
__device__ __forceinline__ int hist_bin(double c, int bins, double scale, unsigned &qlo, unsigned &qhi) {
  if (!(c >= 0.0) || !(c < (double)bins)) return -1;   // NaN / out of range (defensive)
  const double fc = floor(c);
  const double off = c - fc;
  const int idx = (int)fc;
  const unsigned one = (unsigned)scale;
  if (off == 0.0) { qlo = one; qhi = 0u; return idx; }
  if (idx < bins - 1) {
    qhi = (unsigned)__double2uint_rn(off * scale);
    qlo = one - qhi;
    return idx;
  }
  return -1;                                             // the reference drops it
}

// hist_bin from a coordinate given as bin k (< bins - 1) and fraction f.
__device__ __forceinline__ int hist_bin_ff(int k, float f, double scale, unsigned &qlo, unsigned &qhi) {
  const unsigned one = (unsigned)scale;
  if (f == 0.0f) { qlo = one; qhi = 0u; return k; }
  qhi = min(__float2uint_rn(__fmul_rn(f, (float)scale)), one);
  qlo = one - qhi;
  return k;
}

// The FP64 path of a value near the top bin, out of line: inlined, the
// compiler may evaluate it for every value under a predicate.
__device__ __noinline__ int hist_bin_top(const BinMap &bm, float x, int bins, double scale, unsigned &qlo,
                                         unsigned &qhi) {
  return hist_bin(bm.coord(x), bins, scale, qlo, qhi);
}

// Histogram contribution of one value: float-float below the top two bins.
__device__ __forceinline__ int hist_bin_of(const BinMap &bm, float x, int bins, double scale, unsigned &qlo,
                                           unsigned &qhi) {
  int k;
  float f;
  if (bm.coord_ff(x, k, f)) return hist_bin_ff(k, f, scale, qlo, qhi);
  return hist_bin_top(bm, x, bins, scale, qlo, qhi);
}

// Largest shift <= 24 for which `n` voxels cannot overflow a 32-bit bin.
__host__ __device__ inline int hist_shift_for(long long n) {
  int s = kHistMaxShift;
  while (s > 0 && (unsigned long long)n << s > 0xffffffffull) --s;
  return s;
}

// Warp-aggregated add of one value into a shared 32-bit histogram.  All 32
// lanes must call it (lanes without a value pass key < 0).
__device__ __forceinline__ void hist_add_warp(unsigned *h, int bins, int key, unsigned qlo, unsigned qhi) {
  const unsigned grp = __match_any_sync(kFull, key);
  if (key >= 0) {
    const unsigned slo = __reduce_add_sync(grp, qlo);
    const unsigned shi = __reduce_add_sync(grp, qhi);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(grp) - 1)) {
      atomicAdd(&h[key], slo);
      if (shi && key + 1 < bins) atomicAdd(&h[key + 1], shi);
    }
  }
}

// Piecewise-linear remap through E (N4.py:107-113) from the FP64 bin
// coordinate c of the value.
__device__ __forceinline__ double sharpened_value(double c, const double *E, int bins) {
  const double fc = floor(c);
  int idx = (int)fc;
  if (!(c >= 0.0)) idx = 0;   // unreachable for values >= binMin; keeps the access in range
  if (idx < bins - 1) {
    const double e0 = E[idx], e1 = E[idx + 1];
    return e0 + (e1 - e0) * (c - fc);
  }
  return E[bins - 1];
}

// Residual x - E(x) of the piecewise-linear remap for a value in bin
// k < bins - 1 at fraction f.  With x = binMin + (k + f) slope and
// E(x) = E[k] + f (E[k+1] - E[k]) (N4.py:107-113) the residual is linear in f
// within a bin: x - E(x) = R2[k].x + f R2[k].y, R2[k] = (binMin + k slope -
// E[k], slope - (E[k+1] - E[k])) formed in FP64 by sharpen_map, so the
// cancellation of the O(1) terms happens in FP64.  The fraction's own error
// (~2^-24) moves the result by ~2^-24 |R2[k].y| <= 2^-24 slope.
__device__ __forceinline__ float residual_lin(int k, float f, const float2 *R2) {
  const float2 t = R2[k];
  return __fmaf_rn(f, t.y, t.x);
}

// The FP64 residual of a value near the top bin, out of line: inlined, the
// compiler may evaluate it for every value under a predicate.
__device__ __noinline__ float residual_top(const BinMap &bm, float x, const double *E, int bins) {
  return (float)((double)x - sharpened_value(bm.coord(x), E, bins));
}

// Residual x - E(x) of a masked value (N4.py:107-113): the bin and fraction
// from the float-float coordinate, then the bin's linear form; FP64 in the
// top two bins.  (An FP32 coordinate, error ~2^-24 c, moved the lattice of a
// 32x32x24 volume after 2 x 4 iterations by 1.4e-4 relative, measured with
// the oracle: the bound is 1e-4.)
__device__ __forceinline__ float residual_of(const BinMap &bm, float x, const float2 *R2, const double *E,
                                             int bins) {
  int k;
  float f;
  if (bm.coord_ff(x, k, f)) return residual_lin(k, f, R2);
  return residual_top(bm, x, E, bins);
}

// Refined lattice value at output index (ox, oy, oz) (array indices), from
// the (n+3)-point lattice `L` (Lee, Wolberg, Shin 1997 section 4.2;
// cudaN4.cu:257-339 with its clamped boundary).
__device__ __forceinline__ void refine_taps(int o, int n, int idx[3], float w[3]) {
  const int oi = o - 1;                      // lattice coordinate, from -1
  const int i = (oi >= 0) ? (oi >> 1) : -1;  // floor(oi / 2) for oi >= -1
  const int par = oi - 2 * i;
  for (int k = 0; k < 3; ++k) {
    int c = i - 1 + k;
    c = c < -1 ? -1 : (c > n + 1 ? n + 1 : c);
    idx[k] = c + 1;
  }
  if (par == 0) { w[0] = 0.125f; w[1] = 0.75f; w[2] = 0.125f; }
  else          { w[0] = 0.0f;   w[1] = 0.5f;  w[2] = 0.5f; }
}

__device__ void refine_lattice(const float *L, int ncx, int ncy, int ncz, float *out) {
  const int nx = ncx - 3, ny = ncy - 3, nz = ncz - 3;
  const int mx = 2 * nx + 3, my = 2 * ny + 3, mz = 2 * nz + 3;
  for (int t = threadIdx.x; t < mx * my * mz; t += blockDim.x) {
    int oz = t % mz, oy = (t / mz) % my, ox = t / (mz * my);
    int ix[3], iy[3], iz[3];
    float wx[3], wy[3], wz[3];
    refine_taps(ox, nx, ix, wx);
    refine_taps(oy, ny, iy, wy);
    refine_taps(oz, nz, iz, wz);
    float acc = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          acc += wx[a] * wy[b] * wz[c] * L[(ix[a] * ncy + iy[b]) * ncz + iz[c]];
    out[t] = acc;
  }
}

// ---------------------------------------------------------------- grid barrier
// Sense-counting barrier over all CTAs of a cooperative launch.  Every wait
// is bounded: on timeout (or when another CTA already failed) it records
// N4_ERR_TIMEOUT in *err and returns false.
struct GridBarrier {
  unsigned *count;
  unsigned *gen;
  int *err;
  unsigned nblocks;

  __device__ bool sync() const {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
      volatile unsigned *vgen = gen;
      volatile int *verr = err;
      int ok = (*verr == 0);
      unsigned g0 = *vgen;
      __threadfence();
      unsigned t = atomicAdd(count, 1u);
      if (t == nblocks - 1) {
        atomicExch(count, 0u);
        __threadfence();
        atomicAdd(gen, 1u);
      } else {
        unsigned long long spins = 0;
        while (*vgen == g0) {
          if (*verr != 0) { ok = 0; break; }
          if (++spins > kSpinLimit) { atomicExch(err, (int)N4_ERR_TIMEOUT); ok = 0; break; }
          __nanosleep(64);
        }
      }
      __threadfence();
      s_ok = ok && (*verr == 0);
    }
    __syncthreads();
    return s_ok != 0;
  }
};

}  // namespace n4
