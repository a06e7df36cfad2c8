// Warm-start encoder: a small 3-D convolutional network that predicts the
// first-level 4x4x4 log-bias lattice of N4 from the masked log fitting grid
// average-pooled to 32x32x24.  No counterpart in the reference.
//
//   input 1x32x32x24 -> conv3x3x3/2 16 -> ReLU -> conv 32 -> ReLU -> conv 64
//   -> ReLU -> conv 64 -> ReLU -> (64x2x2x2 = 512) -> linear 64
//
// Every contraction (forward, data gradient, weight gradient) runs on the
// BF16 tensor cores through one implicit-GEMM kernel (mma.sync m16n8k16,
// FP32 accumulate) whose operand tiles are gathered from the activation
// tensors by small index functors.  Activations and weights are BF16, master
// weights, gradients and Adam moments FP32.  Weight gradients reduce over the
// batch with a fixed split-K and a deterministic second pass.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/n4b200.h"

namespace enc {

typedef __nv_bfloat16 bf16;

constexpr int kLayers = 4;
constexpr int kCh[kLayers + 1] = {1, 16, 32, 64, 64};
constexpr int kIn[3] = {32, 32, 24};
constexpr int kOut = 64;          // 4x4x4 lattice
constexpr int kFeat = 64 * 8;     // 64 channels x 2x2x2

__host__ __device__ inline int out_dim(int d) { return (d - 1) / 2 + 1; }   // k3, s2, p1

// ------------------------------------------------------------------ mma
__device__ __forceinline__ void mma_bf16(float c[4], const unsigned a[4], const unsigned b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int BM = 64, BN = 64, BK = 32, PAD = 8;

// Exact floor(k / d) for 0 <= k < 2^24 and 1 <= d < 2^16: with
// M = ceil(2^40 / d), k*M / 2^40 exceeds k/d by less than 2^-16 < 1/d.
struct Div {
  unsigned d;
  unsigned long long M;
  Div() : d(1), M(1ull << 40) {}
  explicit Div(unsigned dd) : d(dd), M(((1ull << 40) + dd - 1) / dd) {}
  __device__ __forceinline__ int q(int k) const { return (int)(((unsigned long long)(unsigned)k * M) >> 40); }
};

// C[m][n] = sum_k A(m,k) B(k,n) over this block's K range; P supplies the
// sizes, the gathers and the store.  128 threads: 4 warps of 32x32.  Tile
// staging: each thread owns half a row of the A tile and half a row of the
// B tile (16 consecutive k), so the row's index decomposition (P::a_row,
// P::b_row) is done once per block and the k decomposition uses constant
// divisors or Div; the 16 values go to shared memory as two 16-byte stores.
template <class P>
__global__ void __launch_bounds__(128) k_igemm(const P p) {
  __shared__ __align__(16) bf16 As[BM][BK + PAD];
  __shared__ __align__(16) bf16 Bs[BN][BK + PAD];
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int kper = ((p.K + gridDim.z - 1) / gridDim.z + BK - 1) / BK * BK;
  const int kb = blockIdx.z * kper, ke = min(p.K, kb + kper);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tig = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int sr = threadIdx.x >> 1, sc = (threadIdx.x & 1) * 16;   // staged row, first column
  const bool a_ok = m0 + sr < p.M, b_ok = n0 + sr < p.N;
  const typename P::ARow ar = p.a_row(a_ok ? m0 + sr : 0);
  const typename P::BRow br = p.b_row(b_ok ? n0 + sr : 0);
  float acc[2][4][4] = {};
  const bf16 zero = __float2bfloat16(0.0f);
  for (int k0 = kb; k0 < ke; k0 += BK) {
    unsigned pa[8], pb[8];   // bf16 pairs, low half first
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
      const int k = k0 + sc + j;
      const bf16 a0 = (a_ok && k < ke) ? p.a(ar, k) : zero, a1 = (a_ok && k + 1 < ke) ? p.a(ar, k + 1) : zero;
      const bf16 b0 = (b_ok && k < ke) ? p.b(br, k) : zero, b1 = (b_ok && k + 1 < ke) ? p.b(br, k + 1) : zero;
      pa[j / 2] = (unsigned)__bfloat16_as_ushort(a0) | ((unsigned)__bfloat16_as_ushort(a1) << 16);
      pb[j / 2] = (unsigned)__bfloat16_as_ushort(b0) | ((unsigned)__bfloat16_as_ushort(b1) << 16);
    }
    *(uint4 *)&As[sr][sc] = make_uint4(pa[0], pa[1], pa[2], pa[3]);
    *(uint4 *)&As[sr][sc + 8] = make_uint4(pa[4], pa[5], pa[6], pa[7]);
    *(uint4 *)&Bs[sr][sc] = make_uint4(pb[0], pb[1], pb[2], pb[3]);
    *(uint4 *)&Bs[sr][sc + 8] = make_uint4(pb[4], pb[5], pb[6], pb[7]);
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      unsigned af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + 16 * i + g;
        af[i][0] = *(const unsigned *)&As[r][kk + 2 * tig];
        af[i][1] = *(const unsigned *)&As[r + 8][kk + 2 * tig];
        af[i][2] = *(const unsigned *)&As[r][kk + 2 * tig + 8];
        af[i][3] = *(const unsigned *)&As[r + 8][kk + 2 * tig + 8];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + 8 * j + g;
        bfr[j][0] = *(const unsigned *)&Bs[c][kk + 2 * tig];
        bfr[j][1] = *(const unsigned *)&Bs[c][kk + 2 * tig + 8];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int m = m0 + wm + 16 * i + g + (e >= 2 ? 8 : 0);
        const int n = n0 + wn + 8 * j + 2 * tig + (e & 1);
        if (m < p.M && n < p.N) p.store(m, n, blockIdx.z, acc[i][j][e]);
      }
}

// ------------------------------------------------------------------ problems
struct Shape {
  int B, Ci, D, H, W, Co, Do, Ho, Wo;
  __host__ __device__ int in_pos() const { return D * H * W; }
  __host__ __device__ int out_pos() const { return Do * Ho * Wo; }
};

// Output position decomposition (b, od, oh, ow) of a flat index.
struct PosDiv {
  Div op, hw, w;
  PosDiv() {}
  PosDiv(int out_pos, int hwo, int wo) : op(out_pos), hw(hwo), w(wo) {}
};

// y = relu(conv(x, w) + bias): M = B*outpos, N = Co, K = Ci*27
struct ConvFwd {
  int M, N, K;
  Shape s;
  const bf16 *x, *w;
  const float *bias;
  bf16 *y;
  int relu;
  struct ARow { const bf16 *xb; int id0, ih0, iw0; };   // batch image, corner of the 3x3x3 window
  struct BRow { const bf16 *wn; };
  __device__ ARow a_row(int m) const {
    const int op = s.out_pos();
    const int b = m / op, r = m - b * op;
    const int od = r / (s.Ho * s.Wo), oh = (r / s.Wo) % s.Ho, ow = r % s.Wo;
    return ARow{x + (size_t)b * s.Ci * s.in_pos(), 2 * od - 1, 2 * oh - 1, 2 * ow - 1};
  }
  __device__ bf16 a(const ARow &R, int k) const {
    const int ci = k / 27, t = k - ci * 27;
    const int id = R.id0 + t / 9, ih = R.ih0 + (t / 3) % 3, iw = R.iw0 + t % 3;
    if (id < 0 || id >= s.D || ih < 0 || ih >= s.H || iw < 0 || iw >= s.W) return __float2bfloat16(0.0f);
    return R.xb[((size_t)ci * s.D + id) * s.H * s.W + ih * s.W + iw];
  }
  __device__ BRow b_row(int n) const { return BRow{w + (size_t)n * K}; }
  __device__ bf16 b(const BRow &R, int k) const { return R.wn[k]; }
  __device__ void store(int m, int n, int, float v) const {
    const int op = s.out_pos();
    const int b = m / op, r = m - b * op;
    v += bias[n];
    if (relu) v = fmaxf(v, 0.0f);
    y[((size_t)b * s.Co + n) * op + r] = __float2bfloat16(v);
  }
};

// dy masked by the ReLU of the forward output
__device__ __forceinline__ float dact(const bf16 *dy, const bf16 *y, size_t i, int relu) {
  const float g = __bfloat162float(dy[i]);
  return (relu && __bfloat162float(y[i]) <= 0.0f) ? 0.0f : g;
}

// dx = conv_transpose(dy', w): M = B*inpos, N = Ci, K = Co*27
struct ConvDgrad {
  int M, N, K;
  Shape s;
  const bf16 *dy, *y, *w;
  bf16 *dx;
  int relu;
  struct ARow { size_t base; int pd0, ph0, pw0; };   // batch offset in dy, input position + 1
  struct BRow { int n; };
  __device__ ARow a_row(int m) const {
    const int ip = s.in_pos();
    const int b = m / ip, r = m - b * ip;
    const int id = r / (s.H * s.W), ih = (r / s.W) % s.H, iw = r % s.W;
    return ARow{(size_t)b * s.Co * s.out_pos(), id + 1, ih + 1, iw + 1};
  }
  __device__ bf16 a(const ARow &R, int k) const {
    const int co = k / 27, t = k - co * 27;
    const int pd = R.pd0 - t / 9, ph = R.ph0 - (t / 3) % 3, pw = R.pw0 - t % 3;
    if ((pd | ph | pw) & 1) return __float2bfloat16(0.0f);   // also rejects odd negatives
    const int od = pd >> 1, oh = ph >> 1, ow = pw >> 1;
    if (pd < 0 || ph < 0 || pw < 0 || od >= s.Do || oh >= s.Ho || ow >= s.Wo) return __float2bfloat16(0.0f);
    const size_t i = R.base + (size_t)co * s.out_pos() + (od * s.Ho + oh) * s.Wo + ow;
    return __float2bfloat16(dact(dy, y, i, relu));
  }
  __device__ BRow b_row(int n) const { return BRow{n}; }
  __device__ bf16 b(const BRow &R, int k) const {
    const int co = k / 27, t = k - co * 27;
    return w[((size_t)co * s.Ci + R.n) * 27 + t];
  }
  __device__ void store(int m, int n, int, float v) const {
    const int ip = s.in_pos();
    const int b = m / ip, r = m - b * ip;
    dx[((size_t)b * s.Ci + n) * ip + r] = __float2bfloat16(v);
  }
};

// dw partials: M = Co, N = Ci*27, K = B*outpos (split over blockIdx.z)
struct ConvWgrad {
  int M, N, K;
  Shape s;
  const bf16 *x, *dy, *y;
  float *part;   // [splits][Co][Ci*27]
  int relu;
  PosDiv pd;     // decomposition of a position index k into (b, od, oh, ow)
  struct ARow { int m; };
  struct BRow { int ci, kd, kh, kw; };
  __device__ ARow a_row(int m) const { return ARow{m}; }
  __device__ bf16 a(const ARow &R, int k) const {
    const int op = s.out_pos();
    const int b = pd.op.q(k), r = k - b * op;
    return __float2bfloat16(dact(dy, y, ((size_t)b * s.Co + R.m) * op + r, relu));
  }
  __device__ BRow b_row(int n) const {
    const int ci = n / 27, t = n - ci * 27;
    return BRow{ci, t / 9 - 1, (t / 3) % 3 - 1, t % 3 - 1};
  }
  __device__ bf16 b(const BRow &R, int k) const {
    const int op = s.out_pos();
    const int bb = pd.op.q(k), r = k - bb * op;
    const int od = pd.hw.q(r), r2 = r - od * s.Ho * s.Wo;
    const int oh = pd.w.q(r2), ow = r2 - oh * s.Wo;
    const int id = 2 * od + R.kd, ih = 2 * oh + R.kh, iw = 2 * ow + R.kw;
    if (id < 0 || id >= s.D || ih < 0 || ih >= s.H || iw < 0 || iw >= s.W) return __float2bfloat16(0.0f);
    return x[(((size_t)bb * s.Ci + R.ci) * s.D + id) * s.H * s.W + ih * s.W + iw];
  }
  __device__ void store(int m, int n, int z, float v) const { part[((size_t)z * M + m) * N + n] = v; }
};

// linear y = x W^T + bias: M = B, N = out, K = in
struct LinFwd {
  int M, N, K;
  const bf16 *x, *w;
  const float *bias;
  float *y;
  struct ARow { const bf16 *r; };
  struct BRow { const bf16 *r; };
  __device__ ARow a_row(int m) const { return ARow{x + (size_t)m * K}; }
  __device__ bf16 a(const ARow &R, int k) const { return R.r[k]; }
  __device__ BRow b_row(int n) const { return BRow{w + (size_t)n * K}; }
  __device__ bf16 b(const BRow &R, int k) const { return R.r[k]; }
  __device__ void store(int m, int n, int, float v) const { y[(size_t)m * N + n] = v + bias[n]; }
};
// dx = dy W: M = B, N = in, K = out
struct LinDgrad {
  int M, N, K;
  const bf16 *dy, *w;
  bf16 *dx;
  struct ARow { const bf16 *r; };
  struct BRow { int n; };
  __device__ ARow a_row(int m) const { return ARow{dy + (size_t)m * K}; }
  __device__ bf16 a(const ARow &R, int k) const { return R.r[k]; }
  __device__ BRow b_row(int n) const { return BRow{n}; }
  __device__ bf16 b(const BRow &R, int k) const { return w[(size_t)k * N + R.n]; }
  __device__ void store(int m, int n, int, float v) const { dx[(size_t)m * N + n] = __float2bfloat16(v); }
};
// dW = dy^T x: M = out, N = in, K = B
struct LinWgrad {
  int M, N, K;
  const bf16 *dy, *x;
  float *part;
  struct ARow { int m; };
  struct BRow { int n; };
  __device__ ARow a_row(int m) const { return ARow{m}; }
  __device__ bf16 a(const ARow &R, int k) const { return dy[(size_t)k * M + R.m]; }
  __device__ BRow b_row(int n) const { return BRow{n}; }
  __device__ bf16 b(const BRow &R, int k) const { return x[(size_t)k * N + R.n]; }
  __device__ void store(int m, int n, int z, float v) const { part[((size_t)z * M + m) * N + n] = v; }
};

// ------------------------------------------------------------------ small kernels
__global__ void k_sum_splits(const float *part, int splits, int n, float *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[(size_t)z * n + i];
    out[i] = s;
  }
}

// A forward GEMM split over K: each block stores its partial sums (the
// wrapper's store), then k_finish adds the splits in order and applies the
// layer's own store (bias, ReLU, BF16 for the convolutions).  The forward's
// small layers (conv3, conv4, the linear head: 1 to 6 blocks of 64x64) would
// otherwise walk 16-54 K steps in one block each.
template <class P>
struct Partial : P {
  float *part;   // [splits][M][N]
  __device__ void store(int m, int n, int z, float v) const { part[((size_t)z * this->M + m) * this->N + n] = v; }
};

template <class P>
__global__ void k_finish(const P p, const float *part, int splits) {
  const long long mn = (long long)p.M * p.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < mn; i += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[z * mn + i];
    p.store((int)(i / p.N), (int)(i % p.N), 0, s);
  }
}

// bias gradient: sum of dy' over batch and positions, one block per channel
__global__ void k_bias_grad(const bf16 *dy, const bf16 *y, int B, int C, int pos, int relu, float *db) {
  const int c = blockIdx.x;
  float s = 0.0f;
  for (int i = threadIdx.x; i < B * pos; i += blockDim.x) {
    const int b = i / pos, r = i - b * pos;
    s += dact(dy, y, ((size_t)b * C + c) * pos + r, relu);
  }
  __shared__ float red[32];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    db[c] = t;
  }
}

// loss = mean((y - t)^2); dy = 2 (y - t) / n (bf16); one block
__global__ void k_mse(const float *y, const float *t, int n, float *loss, bf16 *dy) {
  float s = 0.0f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float d = y[i] - t[i];
    s += d * d;
    dy[i] = __float2bfloat16(2.0f * d / (float)n);
  }
  __shared__ float red[32];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float u = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) u += red[w];
    *loss = u / (float)n;
  }
}

__global__ void k_adam(float *p, const float *gr, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2, bf16 *pb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = gr[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float w = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = w;
    pb[i] = __float2bfloat16(w);
  }
}

__global__ void k_to_bf16(const float *a, int n, bf16 *b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = __float2bfloat16(a[i]);
}

// ------------------------------------------------------------------ host side
template <class P>
cudaError_t run_gemm(const P &p, int splits, cudaStream_t st) {
  dim3 grid((p.M + BM - 1) / BM, (p.N + BN - 1) / BN, splits);
  k_igemm<P><<<grid, 128, 0, st>>>(p);
  return cudaGetLastError();
}

// Splits of a forward GEMM: enough blocks for about two per SM, at least two
// K steps per split, within the partials buffer (cap floats).
inline int fwd_splits(int M, int N, int K, size_t cap) {
  const long long tiles = (long long)((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  const int steps = (K + BK - 1) / BK;
  long long s = std::max<long long>(1, 296 / tiles);
  s = std::min<long long>(s, std::max(1, steps / 2));
  while (s > 1 && (size_t)s * M * N > cap) --s;
  return (int)s;
}

// A forward layer: one pass, or split over K into `part` and finished in order.
template <class P>
cudaError_t run_forward(const P &p, float *part, size_t cap, cudaStream_t st) {
  const int splits = fwd_splits(p.M, p.N, p.K, cap);
  if (splits == 1) return run_gemm(p, 1, st);
  Partial<P> q;
  static_cast<P &>(q) = p;
  q.part = part;
  cudaError_t e = run_gemm(q, splits, st);
  if (e != cudaSuccess) return e;
  const long long mn = (long long)p.M * p.N;
  k_finish<P><<<(int)std::min<long long>((mn + 255) / 256, 1024), 256, 0, st>>>(p, part, splits);
  return cudaGetLastError();
}

struct Layout {
  // parameter offsets (floats) in the flat parameter vector
  size_t w[kLayers + 1], b[kLayers + 1], total;
  Shape s[kLayers];
  Layout(int B) {
    int d = kIn[0], h = kIn[1], wd = kIn[2];
    size_t o = 0;
    for (int l = 0; l < kLayers; ++l) {
      s[l] = Shape{B, kCh[l], d, h, wd, kCh[l + 1], out_dim(d), out_dim(h), out_dim(wd)};
      w[l] = o; o += (size_t)kCh[l + 1] * kCh[l] * 27;
      b[l] = o; o += kCh[l + 1];
      d = out_dim(d); h = out_dim(h); wd = out_dim(wd);
    }
    w[kLayers] = o; o += (size_t)kOut * kFeat;
    b[kLayers] = o; o += kOut;
    total = o;
  }
};

}  // namespace enc

using namespace enc;

struct n4_encoder {
  int device = 0;
  int max_batch = 0;
  size_t nparam = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   // FP32 master, grad, moments
  bf16 *pb = nullptr;                                             // BF16 weights
  bf16 *act[kLayers + 1] = {};                                    // activations (act[0] = input copy)
  bf16 *dact_[kLayers + 1] = {};                                  // activation gradients
  float *out = nullptr, *tgt = nullptr, *loss = nullptr;
  bf16 *dout = nullptr;
  float *part = nullptr;
  size_t part_cap = 0;
  long long step = 0;
};

// records the message returned by n4_last_error_string (n4_api.cu)
n4_status_t n4_record_error(n4_status_t s, const char *msg);

// largest batch one n4_encoder_predict call takes (used by n4_api.cu)
int n4_encoder_capacity(const n4_encoder_t *enc) { return enc ? enc->max_batch : 0; }

// kernels one n4_encoder_predict call of batch B launches (used by n4_api.cu):
// a GEMM per layer and the head, and a finishing pass for each split one
int n4_encoder_predict_launches(const n4_encoder_t *enc, int B) {
  if (!enc || B < 1) return 0;
  const enc::Layout L(B);
  int n = enc::kLayers + 1;
  for (int l = 0; l < enc::kLayers; ++l)
    n += enc::fwd_splits(B * L.s[l].out_pos(), L.s[l].Co, L.s[l].Ci * 27, enc->part_cap) > 1 ? 1 : 0;
  n += enc::fwd_splits(B, enc::kOut, enc::kFeat, enc->part_cap) > 1 ? 1 : 0;
  return n;
}

namespace {
n4_status_t efail(n4_status_t s, const std::string &m) { return n4_record_error(s, m.c_str()); }
#define ECK(x)                                                                              \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) { cudaGetLastError(); return efail(N4_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); } \
  } while (0)
constexpr int kSplitsMax = 128;

int wgrad_splits(long long K) { return (int)std::min<long long>(kSplitsMax, std::max<long long>(1, K / 2048)); }
}  // namespace

extern "C" {

size_t n4_encoder_num_params(void) { return Layout(1).total; }

n4_status_t n4_encoder_create(n4_encoder_t **out, int device, int max_batch) {
  if (!out || max_batch < 1 || max_batch > 4096) return efail(N4_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  ECK(cudaSetDevice(device));
  n4_encoder *e = new n4_encoder();
  e->device = device;
  e->max_batch = max_batch;
  Layout L(max_batch);
  e->nparam = L.total;
  size_t n = L.total;
  auto fail_free = [&](cudaError_t err) {
    n4_encoder_destroy(e);
    return efail(err == cudaErrorMemoryAllocation ? N4_ERR_OOM : N4_ERR_CUDA, cudaGetErrorString(err));
  };
  cudaError_t err;
  if ((err = cudaMalloc(&e->p, n * 4)) || (err = cudaMalloc(&e->g, n * 4)) || (err = cudaMalloc(&e->m, n * 4)) ||
      (err = cudaMalloc(&e->v, n * 4)) || (err = cudaMalloc(&e->pb, n * 2)))
    return fail_free(err);
  cudaMemset(e->m, 0, n * 4);
  cudaMemset(e->v, 0, n * 4);
  cudaMemset(e->p, 0, n * 4);
  cudaMemset(e->pb, 0, n * 2);
  for (int l = 0; l <= kLayers; ++l) {
    const size_t sz = l == 0 ? (size_t)max_batch * L.s[0].in_pos() : (size_t)max_batch * L.s[l - 1].Co * L.s[l - 1].out_pos();
    if ((err = cudaMalloc(&e->act[l], sz * 2)) || (err = cudaMalloc(&e->dact_[l], sz * 2))) return fail_free(err);
  }
  if ((err = cudaMalloc(&e->out, (size_t)max_batch * kOut * 4)) || (err = cudaMalloc(&e->tgt, (size_t)max_batch * kOut * 4)) ||
      (err = cudaMalloc(&e->loss, 16)) || (err = cudaMalloc(&e->dout, (size_t)max_batch * kOut * 2)))
    return fail_free(err);
  // split-K partials: the largest weight gradient times the splits
  size_t need = 0;
  for (int l = 0; l < kLayers; ++l) {
    const long long K = (long long)max_batch * L.s[l].out_pos();
    need = std::max(need, (size_t)wgrad_splits(K) * L.s[l].Co * L.s[l].Ci * 27);
  }
  need = std::max(need, (size_t)wgrad_splits(max_batch) * kOut * kFeat);
  // and the forward's split layers at every batch size up to max_batch
  const size_t unbounded = ~(size_t)0;
  for (int b = 1; b <= max_batch; ++b) {
    const Layout Lb(b);
    for (int l = 0; l < kLayers; ++l) {
      const int M = b * Lb.s[l].out_pos(), N = Lb.s[l].Co;
      need = std::max(need, (size_t)fwd_splits(M, N, Lb.s[l].Ci * 27, unbounded) * M * N);
    }
    need = std::max(need, (size_t)fwd_splits(b, kOut, kFeat, unbounded) * b * kOut);
  }
  if ((err = cudaMalloc(&e->part, need * 4))) return fail_free(err);
  e->part_cap = need;
  *out = e;
  return N4_OK;
}

n4_status_t n4_encoder_destroy(n4_encoder_t *e) {
  if (!e) return N4_OK;
  cudaSetDevice(e->device);
  cudaDeviceSynchronize();
  for (void *q : {(void *)e->p, (void *)e->g, (void *)e->m, (void *)e->v, (void *)e->pb, (void *)e->out, (void *)e->tgt,
                  (void *)e->loss, (void *)e->dout, (void *)e->part})
    if (q) cudaFree(q);
  for (int l = 0; l <= kLayers; ++l) {
    if (e->act[l]) cudaFree(e->act[l]);
    if (e->dact_[l]) cudaFree(e->dact_[l]);
  }
  delete e;
  return N4_OK;
}

n4_status_t n4_encoder_set_params(n4_encoder_t *e, const float *h_params, size_t n) {
  if (!e || !h_params || n != e->nparam) return efail(N4_ERR_INVALID_ARG, "parameter count mismatch");
  ECK(cudaSetDevice(e->device));
  ECK(cudaMemcpy(e->p, h_params, n * 4, cudaMemcpyHostToDevice));
  ECK(cudaMemset(e->m, 0, n * 4));
  ECK(cudaMemset(e->v, 0, n * 4));
  k_to_bf16<<<256, 256>>>(e->p, (int)n, e->pb);
  ECK(cudaGetLastError());
  e->step = 0;
  ECK(cudaDeviceSynchronize());
  return N4_OK;
}

n4_status_t n4_encoder_get_params(n4_encoder_t *e, float *h_params, float *h_grads, size_t n) {
  if (!e || n != e->nparam) return efail(N4_ERR_INVALID_ARG, "parameter count mismatch");
  ECK(cudaSetDevice(e->device));
  ECK(cudaDeviceSynchronize());
  if (h_params) ECK(cudaMemcpy(h_params, e->p, n * 4, cudaMemcpyDeviceToHost));
  if (h_grads) ECK(cudaMemcpy(h_grads, e->g, n * 4, cudaMemcpyDeviceToHost));
  return N4_OK;
}

static n4_status_t forward(n4_encoder *e, const void *d_x, int B, cudaStream_t st) {
  Layout L(B);
  ECK(cudaMemcpyAsync(e->act[0], d_x, (size_t)B * L.s[0].in_pos() * 2, cudaMemcpyDeviceToDevice, st));
  for (int l = 0; l < kLayers; ++l) {
    const Shape &s = L.s[l];
    ConvFwd p{B * s.out_pos(), s.Co, s.Ci * 27, s, e->act[l], e->pb + L.w[l], e->p + L.b[l], e->act[l + 1], 1};
    ECK(run_forward(p, e->part, e->part_cap, st));
  }
  LinFwd lf{B, kOut, kFeat, e->act[kLayers], e->pb + L.w[kLayers], e->p + L.b[kLayers], e->out};
  ECK(run_forward(lf, e->part, e->part_cap, st));
  return N4_OK;
}

n4_status_t n4_encoder_predict(n4_encoder_t *e, const void *d_x, int B, float *d_out, void *stream) {
  if (!e || !d_x || !d_out || B < 1 || B > e->max_batch) return efail(N4_ERR_INVALID_ARG, "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  ECK(cudaSetDevice(e->device));
  n4_status_t s = forward(e, d_x, B, st);
  if (s != N4_OK) return s;
  ECK(cudaMemcpyAsync(d_out, e->out, (size_t)B * kOut * 4, cudaMemcpyDeviceToDevice, st));
  return N4_OK;
}

// Forward + backward on one batch; gradients in the encoder; optionally an
// Adam step (lr > 0).  *h_loss (nullable) receives the batch MSE.
n4_status_t n4_encoder_train_step(n4_encoder_t *e, const void *d_x, const float *d_target, int B, float lr,
                                  float *h_loss, void *stream) {
  if (!e || !d_x || !d_target || B < 1 || B > e->max_batch) return efail(N4_ERR_INVALID_ARG, "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  ECK(cudaSetDevice(e->device));
  n4_status_t s = forward(e, d_x, B, st);
  if (s != N4_OK) return s;
  Layout L(B);
  k_mse<<<1, 256, 0, st>>>(e->out, d_target, B * kOut, e->loss, e->dout);
  ECK(cudaGetLastError());
  // linear head
  {
    const int splits = wgrad_splits(B);
    LinWgrad wg{kOut, kFeat, B, e->dout, e->act[kLayers], e->part};
    ECK(run_gemm(wg, splits, st));
    k_sum_splits<<<64, 256, 0, st>>>(e->part, splits, kOut * kFeat, e->g + L.w[kLayers]);
    // bias gradient = column sums of dout (positions = 1, no activation)
    k_bias_grad<<<kOut, 256, 0, st>>>(e->dout, e->dout, B, kOut, 1, 0, e->g + L.b[kLayers]);
    LinDgrad dg{B, kFeat, kOut, e->dout, e->pb + L.w[kLayers], e->dact_[kLayers]};
    ECK(run_gemm(dg, 1, st));
  }
  for (int l = kLayers - 1; l >= 0; --l) {
    const Shape &sh = L.s[l];
    const long long K = (long long)B * sh.out_pos();
    const int splits = wgrad_splits(K);
    ConvWgrad wg{sh.Co, sh.Ci * 27, (int)K, sh, e->act[l], e->dact_[l + 1], e->act[l + 1], e->part, 1,
                 PosDiv(sh.out_pos(), sh.Ho * sh.Wo, sh.Wo)};
    ECK(run_gemm(wg, splits, st));
    k_sum_splits<<<64, 256, 0, st>>>(e->part, splits, sh.Co * sh.Ci * 27, e->g + L.w[l]);
    k_bias_grad<<<sh.Co, 256, 0, st>>>(e->dact_[l + 1], e->act[l + 1], B, sh.Co, sh.out_pos(), 1, e->g + L.b[l]);
    if (l > 0) {
      ConvDgrad dg{B * sh.in_pos(), sh.Ci, sh.Co * 27, sh, e->dact_[l + 1], e->act[l + 1], e->pb + L.w[l], e->dact_[l], 1};
      ECK(run_gemm(dg, 1, st));
    }
  }
  ECK(cudaGetLastError());
  if (lr > 0.0f) {
    ++e->step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)e->step), c2 = 1.0f - powf(b2, (float)e->step);
    k_adam<<<256, 256, 0, st>>>(e->p, e->g, e->m, e->v, (int)e->nparam, lr, b1, b2, 1e-8f, c1, c2, e->pb);
    ECK(cudaGetLastError());
  }
  if (h_loss) {
    ECK(cudaMemcpyAsync(h_loss, e->loss, 4, cudaMemcpyDeviceToHost, st));
    ECK(cudaStreamSynchronize(st));
  }
  return N4_OK;
}

// Network input for one volume: [32][32][24] BF16 written to d_x.
}  // extern "C"
