// pruner.cu: the learned partition / mode pruner -- its features, its network (forward and
// backward), loss and optimiser, and the masks it proposes (include/celv2_pruner.h).
//
// The network is small (55,080 parameters, ~1 MFLOP per superblock); every layer is an im2col
// (convolutions) plus one GEMM on the tensor cores: operands rounded to BF16, mma.sync m16n8k16
// with FP32 accumulators, bias and ReLU in the epilogue. The backward pass is the same GEMM with
// transposed strides, a gather col2im, ReLU masks and column sums for the biases.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

#include "celv2_pruner.h"
#include "kernels.h"

namespace celv2cu {

void set_last_error(const std::string& msg);

namespace nn {

constexpr int kF = CELV2_PRUNER_FEATURES, kOut = CELV2_PRUNER_OUTPUTS;
// parameter offsets
constexpr int kW1 = 0, kB1 = kW1 + 16 * 9, kW2 = kB1 + 16, kB2 = kW2 + 32 * 144, kW3 = kB2 + 32, kB3 = kW3 + 32 * 288,
              kW4 = kB3 + 32, kB4 = kW4 + 64 * 632, kW5 = kB4 + 64, kB5 = kW5 + kOut * 64, kParams = kB5 + kOut;
static_assert(kParams == CELV2_PRUNER_PARAMS, "parameter count");
// forward cache, floats per sample, in this order
constexpr int kCols1 = 256 * 9, kA1 = 256 * 16, kCols2 = 64 * 144, kA2 = 64 * 32, kCols3 = 16 * 288, kA3 = 16 * 32,
              kH0 = 632, kA4 = 64, kLogits = kOut;
static_assert(kCols1 + kA1 + kCols2 + kA2 + kCols3 + kA3 + kH0 + kA4 + kLogits == CELV2_PRUNER_ACTS, "cache size");
// backward workspace, floats per sample
constexpr int kDz4 = 64, kDh0 = 512, kDcols3 = 4608, kDz2 = 2048, kDcols2 = 9216, kDz1 = 4096;
static_assert(kDz4 + kDh0 + kDcols3 + kDz2 + kDcols2 + kDz1 == CELV2_PRUNER_WORK, "workspace size");

struct Cache {  // the forward cache of a batch, segment by segment
  float *cols1, *a1, *cols2, *a2, *cols3, *a3, *h0, *a4, *logits;
  Cache(float* base, long long b) {
    cols1 = base;
    a1 = cols1 + b * kCols1;
    cols2 = a1 + b * kA1;
    a2 = cols2 + b * kCols2;
    cols3 = a2 + b * kA2;
    a3 = cols3 + b * kCols3;
    h0 = a3 + b * kA3;
    a4 = h0 + b * kH0;
    logits = a4 + b * kA4;
  }
};

// ---- GEMM: C[m][n] = act(sum_k bf16(A[m][k]) * bf16(B[k][n]) + bias[n]) (+ C if accumulate) ----
// Element (m, k) of A at A[m * a_sm + k * a_sk], (k, n) of B at B[k * b_sk + n * b_sn], (m, n) of C
// at C[m * c_sm + n * c_sn]: transposes are strides. CTA tile 64 x 64, four warps of 32 x 32, K in
// steps of 16 staged as BF16 in shared memory; out-of-range elements load as zero.
constexpr int kTm = 64, kTn = 64, kTk = 16, kPad = 8;

// Split K (gridDim.z > 1): CTA z takes K range [z * kc, (z + 1) * kc) and adds its partial sums
// atomically into C (zero beforehand; no ReLU; the bias comes from z == 0).
__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const float* __restrict__ A, long long a_sm,
                                              long long a_sk, const float* __restrict__ B, long long b_sk,
                                              long long b_sn, float* C, long long c_sm, long long c_sn,
                                              const float* __restrict__ bias, int relu, int accumulate, int kc) {
  __shared__ __align__(16) __nv_bfloat16 As[kTm][kTk + kPad];  // [m][k]
  __shared__ __align__(16) __nv_bfloat16 Bs[kTn][kTk + kPad];  // [n][k]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.x * kTm, n0 = blockIdx.y * kTn;
  const int kbeg = blockIdx.z * kc, kend = min(K, kbeg + kc);
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.f;
  for (int k0 = kbeg; k0 < kend; k0 += kTk) {
#pragma unroll
    for (int e = tid; e < kTm * kTk; e += 128) {
      const int r = e / kTk, c = e % kTk, m = m0 + r, k = k0 + c;
      As[r][c] = __float2bfloat16_rn(m < M && k < kend ? A[m * a_sm + k * a_sk] : 0.f);
    }
#pragma unroll
    for (int e = tid; e < kTn * kTk; e += 128) {
      const int r = e / kTk, c = e % kTk, n = n0 + r, k = k0 + c;
      Bs[r][c] = __float2bfloat16_rn(n < N && k < kend ? B[k * b_sk + n * b_sn] : 0.f);
    }
    __syncthreads();
    uint32_t af[2][4], bfr[4][2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int r = wm + i * 16 + g;
      af[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][2 * t]);
      af[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][2 * t]);
      af[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][2 * t + 8]);
      af[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][2 * t + 8]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int n = wn + j * 8 + g;
      bfr[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[n][2 * t]);
      bfr[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[n][2 * t + 8]);
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};"
            : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
            : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bfr[j][0]), "r"(bfr[j][1]));
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int m = m0 + wm + i * 16 + g + (q >> 1) * 8, n = n0 + wn + j * 8 + 2 * t + (q & 1);
        if (m >= M || n >= N) continue;
        float v = acc[i][j][q] + (bias && blockIdx.z == 0 ? bias[n] : 0.f);
        float* dst = C + m * c_sm + n * c_sn;
        if (gridDim.z > 1) {
          atomicAdd(dst, v);
          continue;
        }
        if (relu) v = fmaxf(v, 0.f);
        *dst = accumulate ? *dst + v : v;
      }
}

// split > 1: C must hold zeros (or the sum to add to), and no ReLU.
void gemm(int M, int N, int K, const float* A, long long a_sm, long long a_sk, const float* B, long long b_sk,
          long long b_sn, float* C, long long c_sm, long long c_sn, const float* bias, bool relu, bool accumulate,
          cudaStream_t st, int split = 1) {
  const int kc = ((K + split - 1) / split + kTk - 1) / kTk * kTk;
  const dim3 grid((M + kTm - 1) / kTm, (N + kTn - 1) / kTn, (K + kc - 1) / kc);
  k_gemm<<<grid, 128, 0, st>>>(M, N, K, A, a_sm, a_sk, B, b_sk, b_sn, C, c_sm, c_sn, bias, relu, accumulate, kc);
}

// The K split of a weight-gradient GEMM (long K = batch x positions, small M x N): ~2048 per CTA.
int wsplit(long long K) {
  const long long s = (K + 2047) / 2048;
  return (int)(s < 1 ? 1 : s > 1024 ? 1024 : s);
}

// ---- im2col / col2im for 3x3 convolutions, padding 1, NHWC activations ----
// cols[(b * Ho + oy) * Wo + ox][(ky * 3 + kx) * C + c] = X[b][oy * s + ky - 1][ox * s + kx - 1][c]
__global__ void k_im2col(const float* __restrict__ X, long long sample_stride, int H, int W, int C, int s,
                         float* __restrict__ cols, long long total) {
  const int Ho = (H - 1) / s + 1, Wo = (W - 1) / s + 1, K = 9 * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long row = i / K;
    const int col = (int)(i - row * K), tap = col / C, c = col - tap * C, ky = tap / 3, kx = tap - ky * 3;
    const long long b = row / (Ho * Wo);
    const int p = (int)(row - b * Ho * Wo), oy = p / Wo, ox = p - oy * Wo;
    const int y = oy * s + ky - 1, x = ox * s + kx - 1;
    cols[i] = (y >= 0 && y < H && x >= 0 && x < W) ? X[b * sample_stride + ((long long)y * W + x) * C + c] : 0.f;
  }
}

// dX[b][y][x][c] = sum of dcols over the (output position, tap) pairs that read (y, x)
__global__ void k_col2im(const float* __restrict__ dcols, int H, int W, int C, int s, float* __restrict__ dX,
                         long long total) {
  const int Ho = (H - 1) / s + 1, Wo = (W - 1) / s + 1, K = 9 * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / ((long long)H * W * C);
    const int r = (int)(i - b * H * W * C), c = r % C, px = r / C, y = px / W, x = px - y * W;
    float sum = 0.f;
    for (int ky = 0; ky < 3; ky++) {
      const int ty = y + 1 - ky;
      if (ty < 0 || ty % s) continue;
      const int oy = ty / s;
      if (oy >= Ho) continue;
      for (int kx = 0; kx < 3; kx++) {
        const int tx = x + 1 - kx;
        if (tx < 0 || tx % s) continue;
        const int ox = tx / s;
        if (ox >= Wo) continue;
        sum += dcols[((b * Ho + oy) * Wo + ox) * K + (ky * 3 + kx) * C + c];
      }
    }
    dX[i] = sum;
  }
}

// h0[b] = a3[b] (512) ++ x[b][256 .. 376)
__global__ void k_concat(const float* __restrict__ a3, const float* __restrict__ x, float* __restrict__ h0, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / kH0;
    const int k = (int)(i - b * kH0);
    h0[i] = k < 512 ? a3[b * 512 + k] : x[b * kF + 256 + (k - 512)];
  }
}

__global__ void k_relu(float* a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = fmaxf(a[i], 0.f);
}

// dz = da where the activation is positive (ReLU backward; in place allowed)
__global__ void k_relu_bwd(const float* __restrict__ act, const float* da, float* dz, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dz[i] = act[i] > 0.f ? da[i] : 0.f;
}

// db[n] += sum over rows of dz[m][n] (N <= 64 columns, one thread each; blocks take row strides)
__global__ void k_colsum(const float* __restrict__ dz, long long M, int N, float* db) {
  const int n = threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (long long m = blockIdx.x; m < M; m += gridDim.x) s += dz[m * N + n];
  atomicAdd(db + n, s);
}

__global__ void k_bce(const float* __restrict__ z, const float* __restrict__ y, const float* __restrict__ w, int n,
                      float inv_batch, float* __restrict__ dz, float* loss) {
  __shared__ float part[256];
  float l = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float v = z[i], t = y[i], wt = w[i];
    const float sig = 1.f / (1.f + expf(-v));
    l += wt * (fmaxf(v, 0.f) - v * t + log1pf(expf(-fabsf(v))));
    dz[i] = wt * (sig - t) * inv_batch;
  }
  part[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, part[0] * inv_batch);
}

__global__ void k_adam(float* p, const float* __restrict__ g, float* m, float* v, int n, float lr, float b1, float b2,
                       float eps, float wd, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi, v[i] = vi;
    p[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i]);
  }
}

int grid_for(long long n) {
  const long long g = (n + 255) / 256;
  return (int)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

void forward(const float* P, const float* x, int batch, float* acts, cudaStream_t st) {
  const long long b = batch;
  Cache c(acts, b);
  k_im2col<<<grid_for(b * kCols1), 256, 0, st>>>(x, kF, 16, 16, 1, 1, c.cols1, b * kCols1);
  gemm((int)(b * 256), 16, 9, c.cols1, 9, 1, P + kW1, 1, 9, c.a1, 16, 1, P + kB1, true, false, st);
  k_im2col<<<grid_for(b * kCols2), 256, 0, st>>>(c.a1, kA1, 16, 16, 16, 2, c.cols2, b * kCols2);
  gemm((int)(b * 64), 32, 144, c.cols2, 144, 1, P + kW2, 1, 144, c.a2, 32, 1, P + kB2, true, false, st);
  k_im2col<<<grid_for(b * kCols3), 256, 0, st>>>(c.a2, kA2, 8, 8, 32, 2, c.cols3, b * kCols3);
  gemm((int)(b * 16), 32, 288, c.cols3, 288, 1, P + kW3, 1, 288, c.a3, 32, 1, P + kB3, true, false, st);
  k_concat<<<grid_for(b * kH0), 256, 0, st>>>(c.a3, x, c.h0, b * kH0);
  // the dense layer's K (632) in 8 slices on separate CTAs (few rows, many columns of K), then ReLU
  cudaMemsetAsync(c.a4, 0, (size_t)b * kA4 * sizeof(float), st);
  gemm(batch, 64, 632, c.h0, 632, 1, P + kW4, 1, 632, c.a4, 64, 1, P + kB4, false, false, st, 8);
  k_relu<<<grid_for(b * kA4), 256, 0, st>>>(c.a4, b * kA4);
  gemm(batch, kOut, 64, c.a4, 64, 1, P + kW5, 1, 64, c.logits, kOut, 1, P + kB5, false, false, st);
}

void backward(const float* P, int batch, const float* acts, const float* dlogits, float* work, float* G,
              cudaStream_t st) {
  const long long b = batch;
  Cache c(const_cast<float*>(acts), b);
  float* dz4 = work;
  float* dh0 = dz4 + b * kDz4;
  float* dcols3 = dh0 + b * kDh0;
  float* dz2 = dcols3 + b * kDcols3;
  float* dcols2 = dz2 + b * kDz2;
  float* dz1 = dcols2 + b * kDcols2;
  cudaMemsetAsync(G, 0, kParams * sizeof(float), st);  // the bias sums accumulate
  // dense 64 -> kOut
  gemm(kOut, 64, batch, dlogits, 1, kOut, c.a4, 64, 1, G + kW5, 64, 1, nullptr, false, false, st, wsplit(b));
  k_colsum<<<grid_for(b), 64, 0, st>>>(dlogits, b, kOut, G + kB5);
  gemm(batch, 64, kOut, dlogits, kOut, 1, P + kW5, 64, 1, dz4, 64, 1, nullptr, false, false, st);
  k_relu_bwd<<<grid_for(b * 64), 256, 0, st>>>(c.a4, dz4, dz4, b * 64);
  // dense 632 -> 64 (the gradient reaches only the convolution part of its input)
  gemm(64, 632, batch, dz4, 1, 64, c.h0, 632, 1, G + kW4, 632, 1, nullptr, false, false, st, wsplit(b));
  k_colsum<<<grid_for(b), 64, 0, st>>>(dz4, b, 64, G + kB4);
  gemm(batch, 512, 64, dz4, 64, 1, P + kW4, 632, 1, dh0, 512, 1, nullptr, false, false, st);
  k_relu_bwd<<<grid_for(b * 512), 256, 0, st>>>(c.a3, dh0, dh0, b * 512);  // dz3, (b * 16) x 32
  // conv 32 -> 32, stride 2
  gemm(32, 288, (int)(b * 16), dh0, 1, 32, c.cols3, 288, 1, G + kW3, 288, 1, nullptr, false, false, st, wsplit(b * 16));
  k_colsum<<<grid_for(b * 16), 64, 0, st>>>(dh0, b * 16, 32, G + kB3);
  gemm((int)(b * 16), 288, 32, dh0, 32, 1, P + kW3, 288, 1, dcols3, 288, 1, nullptr, false, false, st);
  k_col2im<<<grid_for(b * kDz2), 256, 0, st>>>(dcols3, 8, 8, 32, 2, dz2, b * kDz2);
  k_relu_bwd<<<grid_for(b * kDz2), 256, 0, st>>>(c.a2, dz2, dz2, b * kDz2);
  // conv 16 -> 32, stride 2
  gemm(32, 144, (int)(b * 64), dz2, 1, 32, c.cols2, 144, 1, G + kW2, 144, 1, nullptr, false, false, st, wsplit(b * 64));
  k_colsum<<<grid_for(b * 64), 64, 0, st>>>(dz2, b * 64, 32, G + kB2);
  gemm((int)(b * 64), 144, 32, dz2, 32, 1, P + kW2, 144, 1, dcols2, 144, 1, nullptr, false, false, st);
  k_col2im<<<grid_for(b * kDz1), 256, 0, st>>>(dcols2, 16, 16, 16, 2, dz1, b * kDz1);
  k_relu_bwd<<<grid_for(b * kDz1), 256, 0, st>>>(c.a1, dz1, dz1, b * kDz1);
  // conv 1 -> 16
  gemm(16, 9, (int)(b * 256), dz1, 1, 16, c.cols1, 9, 1, G + kW1, 9, 1, nullptr, false, false, st, wsplit(b * 256));
  k_colsum<<<grid_for(b * 256), 64, 0, st>>>(dz1, b * 256, 16, G + kB1);
}

}  // namespace nn

// ---- features and masks (the engine side) ----

// One CTA (128 threads) per superblock of one job: the luma at level 2, the level-1 cost map per
// reference, presence flags and lambda (include/celv2_pruner.h).
__global__ void __launch_bounds__(128) k_features(const FrameJob* __restrict__ jobp, float* __restrict__ out) {
  const FrameJob& job = *jobp;
  const int sb = blockIdx.x, tid = threadIdx.x;
  const int sby = sb / job.sb_cols, sbx = sb - sby * job.sb_cols;
  float* f = out + (long long)sb * nn::kF;
  __shared__ float red[128];
  const DevPlane l2 = job.cur.lv[2];
  int v0 = at(l2, sby * 16 + (tid >> 4), sbx * 16 + (tid & 15));
  int v1 = at(l2, sby * 16 + 8 + (tid >> 4), sbx * 16 + (tid & 15));
  red[tid] = (float)(v0 + v1);
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (tid < s) red[tid] += red[tid + s];
    __syncthreads();
  }
  const float mean = red[0] / 256.f;
  f[tid] = ((float)v0 - mean) / 64.f;
  f[128 + tid] = ((float)v1 - mean) / 64.f;
  if (tid < kMaxRefs * 16) {
    const int r = tid >> 4, cell = tid & 15;
    float v = 0.f;
    if (r < job.nrefs) {
      const int cols = job.fcols[1], rows = job.frows[1];
      const int cx = min(sbx * 4 + (cell & 3), cols - 1), cy = min(sby * 4 + (cell >> 2), rows - 1);
      const int m = job.field[r][1][cy * cols + cx], mx = mv_x(m), my = mv_y(m);
      const DevPlane cur = job.cur.lv[1], ref = job.ref[r].lv[1];
      int sad = 0;
      for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) sad += abs(at(cur, cy * 8 + i, cx * 8 + j) - at(ref, cy * 8 + my + i, cx * 8 + mx + j));
      v = log2f(1.f + (float)sad) / 14.f;
    }
    f[256 + tid] = v;
  }
  if (tid < kMaxRefs) f[368 + tid] = tid < job.nrefs ? 1.f : 0.f;
  if (tid == 0) f[375] = log2f((float)(job.lam > 1 ? job.lam : 1)) / 20.f;
}

void launch_features(const FrameJob* djob, int nsb, float* out, cudaStream_t st) {
  k_features<<<nsb, 128, 0, st>>>(djob, out);
}

// The keep word (include/celv2_decision.h) of one superblock from its logits: reference r kept
// where sigmoid >= th.ref (the likeliest reference always), intra where >= th.intra, block level l
// where >= th.level (the likeliest level always), and with intra the modes DC, V, H (their scoring
// costs next to nothing) and each other mode m where >= th.mode; everything where one of the
// reference, intra or level outputs lies within th.band of its threshold (the fallback to the full
// search).
__device__ __forceinline__ uint32_t mask_word(const float* z, int nrefs, const PrunerThresholds& th) {
  unsigned k = 0;
  int best = 0, lbest = 0;
  float pbest = -1.f, plbest = -1.f;
  bool unsure = false;
  for (int r = 0; r < nrefs; r++) {
    const float p = 1.f / (1.f + expf(-z[r]));
    if (p >= th.ref) k |= 1u << r;
    if (p > pbest) pbest = p, best = r;
    unsure |= fabsf(p - th.ref) < th.band;
  }
  k |= 1u << best;
  const float pi = 1.f / (1.f + expf(-z[7]));
  if (pi >= th.intra) k |= CELV2_KEEP_INTRA;
  unsure |= fabsf(pi - th.intra) < th.band;
  for (int l = 0; l < 4; l++) {
    const float p = 1.f / (1.f + expf(-z[8 + l]));
    if (p >= th.level) k |= CELV2_KEEP_LEVEL(l);
    if (p > plbest) plbest = p, lbest = l;
    unsure |= fabsf(p - th.level) < th.band;
  }
  k |= CELV2_KEEP_LEVEL(lbest);
  if (k & CELV2_KEEP_INTRA) {
    k |= CELV2_KEEP_MODE(0) | CELV2_KEEP_MODE(1) | CELV2_KEEP_MODE(2);
    for (int m = 3; m < kModes; m++)
      if (1.f / (1.f + expf(-z[12 + m - 3])) >= th.mode) k |= CELV2_KEEP_MODE(m);
  }
  return unsure ? 0xFFFFFFFFu : k;
}

__global__ void k_masks(const float* __restrict__ logits, int nsb, int nrefs, PrunerThresholds th,
                        uint32_t* __restrict__ keep) {
  const int sb = blockIdx.x * blockDim.x + threadIdx.x;
  if (sb >= nsb) return;
  keep[sb] = mask_word(logits + (long long)sb * nn::kOut, nrefs, th);
}

void launch_masks(const float* logits, int nsb, int nrefs, const PrunerThresholds& th, uint32_t* keep,
                  cudaStream_t st) {
  k_masks<<<(nsb + 127) / 128, 128, 0, st>>>(logits, nsb, nrefs, th, keep);
}

void pruner_forward(const float* params, const float* x, int batch, float* acts, cudaStream_t st) {
  nn::forward(params, x, batch, acts, st);
}

// ---- the engine's inference: the whole network for one superblock per CTA, then its mask ----
// The same arithmetic as nn::forward (BF16 operands, FP32 sums; only the order of the sums
// differs): the 3x3 convolution 1 -> 16 and the dense layers on the CUDA cores (bf16-rounded
// operands), the two strided convolutions (85% of the FLOPs) as mma.sync m16n8k16 tiles whose A
// operand is read straight from the previous activation in shared memory (an implicit im2col).
// Weights: bf16 copies made once (infer_weights), W4 transposed so a CTA's 64 threads read rows.
namespace nn {
constexpr int kIW2 = 0, kIW3 = kIW2 + 32 * 144, kIW4 = kIW3 + 32 * 288, kIWs = kIW4 + 632 * 64;  // bf16 elements

__global__ void k_infer_weights(const float* __restrict__ P, __nv_bfloat16* __restrict__ Wb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kIWs; i += gridDim.x * blockDim.x) {
    float v;
    if (i < kIW3) v = P[kW2 + i];
    else if (i < kIW4) v = P[kW3 + (i - kIW3)];
    else {
      const int r = i - kIW4, k = r / 64, o = r - k * 64;  // W4t[k][o] = W4[o][k]
      v = P[kW4 + o * 632 + k];
    }
    Wb[i] = __float2bfloat16_rn(v);
  }
}

__device__ __forceinline__ float rbf(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__global__ void __launch_bounds__(128) k_infer(const float* __restrict__ P, const __nv_bfloat16* __restrict__ Wb,
                                               const float* __restrict__ feats, int nrefs, PrunerThresholds th,
                                               uint32_t* __restrict__ keep) {
  __shared__ float xr[kF];                            // the features, bf16-rounded
  __shared__ __align__(16) __nv_bfloat16 a1[256][16];  // conv1 output, (y, x) rows, channels
  __shared__ __align__(16) __nv_bfloat16 a2[64][32];
  __shared__ float h0[632], a4[64], part[128];
  __shared__ float logits[kOut];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const float* x = feats + (long long)blockIdx.x * kF;
  for (int i = tid; i < kF; i += 128) xr[i] = rbf(x[i]);
  __syncthreads();
  // conv 3x3 1 -> 16, stride 1
  for (int e = tid; e < 256 * 16; e += 128) {
    const int p = e >> 4, c = e & 15, y = p >> 4, xx = p & 15;
    float s = 0.f;
#pragma unroll
    for (int ky = 0; ky < 3; ky++)
#pragma unroll
      for (int kx = 0; kx < 3; kx++) {
        const int iy = y + ky - 1, ix = xx + kx - 1;
        if (iy >= 0 && iy < 16 && ix >= 0 && ix < 16) s += xr[iy * 16 + ix] * rbf(P[kW1 + c * 9 + ky * 3 + kx]);
      }
    a1[p][c] = __float2bfloat16_rn(fmaxf(s + P[kB1 + c], 0.f));
  }
  __syncthreads();
  // conv 3x3 16 -> 32, stride 2: rows = 64 output positions (warp w: 16w..16w+15), K = tap x 16
  {
    float acc[4][4] = {};
    const int r0 = warp * 16 + g, r1 = r0 + 8;
    for (int tap = 0; tap < 9; tap++) {
      const int ky = tap / 3, kx = tap - ky * 3;
      uint32_t a[4];
      const int iy0 = (r0 >> 3) * 2 + ky - 1, ix0 = (r0 & 7) * 2 + kx - 1;
      const int iy1 = (r1 >> 3) * 2 + ky - 1, ix1 = (r1 & 7) * 2 + kx - 1;
      const bool in0 = iy0 >= 0 && iy0 < 16 && ix0 >= 0 && ix0 < 16, in1 = iy1 >= 0 && iy1 < 16 && ix1 >= 0 && ix1 < 16;
      const uint32_t* q0 = reinterpret_cast<const uint32_t*>(a1[in0 ? iy0 * 16 + ix0 : 0]);
      const uint32_t* q1 = reinterpret_cast<const uint32_t*>(a1[in1 ? iy1 * 16 + ix1 : 0]);
      a[0] = in0 ? q0[t] : 0u, a[1] = in1 ? q1[t] : 0u, a[2] = in0 ? q0[t + 4] : 0u, a[3] = in1 ? q1[t + 4] : 0u;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const uint32_t* w = reinterpret_cast<const uint32_t*>(Wb + kIW2 + (j * 8 + g) * 144 + tap * 16);
        mma16816(acc[j], a, __ldg(w + t), __ldg(w + t + 4));
      }
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = q < 2 ? r0 : r1, n = j * 8 + 2 * t + (q & 1);
        a2[r][n] = __float2bfloat16_rn(fmaxf(acc[j][q] + P[kB2 + n], 0.f));
      }
  }
  __syncthreads();
  // conv 3x3 32 -> 32, stride 2: 16 output positions, warp w: output channels 8w..8w+7, K = tap x 32
  {
    float acc[4] = {};
    const int r0 = g, r1 = g + 8;
    for (int s = 0; s < 18; s++) {
      const int tap = s >> 1, c0 = (s & 1) * 16, ky = tap / 3, kx = tap - ky * 3;
      uint32_t a[4];
      const int iy0 = (r0 >> 2) * 2 + ky - 1, ix0 = (r0 & 3) * 2 + kx - 1;
      const int iy1 = (r1 >> 2) * 2 + ky - 1, ix1 = (r1 & 3) * 2 + kx - 1;
      const bool in0 = iy0 >= 0 && iy0 < 8 && ix0 >= 0 && ix0 < 8, in1 = iy1 >= 0 && iy1 < 8 && ix1 >= 0 && ix1 < 8;
      const uint32_t* q0 = reinterpret_cast<const uint32_t*>(&a2[in0 ? iy0 * 8 + ix0 : 0][c0]);
      const uint32_t* q1 = reinterpret_cast<const uint32_t*>(&a2[in1 ? iy1 * 8 + ix1 : 0][c0]);
      a[0] = in0 ? q0[t] : 0u, a[1] = in1 ? q1[t] : 0u, a[2] = in0 ? q0[t + 4] : 0u, a[3] = in1 ? q1[t + 4] : 0u;
      const uint32_t* w = reinterpret_cast<const uint32_t*>(Wb + kIW3 + (warp * 8 + g) * 288 + tap * 32 + c0);
      mma16816(acc, a, __ldg(w + t), __ldg(w + t + 4));
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int r = q < 2 ? r0 : r1, n = warp * 8 + 2 * t + (q & 1);
      h0[r * 32 + n] = rbf(fmaxf(acc[q] + P[kB3 + n], 0.f));  // the dense layer reads it as BF16
    }
  }
  for (int i = tid; i < 120; i += 128) h0[512 + i] = xr[256 + i];
  __syncthreads();
  // dense 632 -> 64: thread (o, half) sums half of the row
  {
    const int o = tid & 63, half = tid >> 6;
    float s = 0.f;
    for (int k = half * 316; k < half * 316 + 316; k++) s += h0[k] * __bfloat162float(Wb[kIW4 + k * 64 + o]);
    part[tid] = s;
  }
  __syncthreads();
  if (tid < 64) a4[tid] = rbf(fmaxf(part[tid] + part[tid + 64] + P[kB4 + tid], 0.f));
  __syncthreads();
  // dense 64 -> kOut: warp w, lanes sum over the 64 inputs for outputs w, w + 4, ...
  for (int o = warp; o < kOut; o += 4) {
    float s = a4[lane] * rbf(P[kW5 + o * 64 + lane]) + a4[lane + 32] * rbf(P[kW5 + o * 64 + lane + 32]);
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    if (lane == 0) logits[o] = s + P[kB5 + o];
  }
  __syncthreads();
  if (tid == 0) keep[blockIdx.x] = mask_word(logits, nrefs, th);  // k_masks' rule
}
}  // namespace nn

// bf16 copies of the convolution and dense weights the inference kernel reads (nn::kIWs elements)
size_t infer_weight_elems() { return nn::kIWs; }
void infer_weights(const float* params, void* wb, cudaStream_t st) {
  nn::k_infer_weights<<<nn::grid_for(nn::kIWs), 256, 0, st>>>(params, static_cast<__nv_bfloat16*>(wb));
}
void launch_infer(const float* params, const void* wb, const float* feats, int nsb, int nrefs,
                  const PrunerThresholds& th, uint32_t* keep, cudaStream_t st) {
  nn::k_infer<<<nsb, 128, 0, st>>>(params, static_cast<const __nv_bfloat16*>(wb), feats, nrefs, th, keep);
}

}  // namespace celv2cu

using namespace celv2cu;

namespace {

int fail(const char* what, cudaError_t e) {
  set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return CELV2_ECUDA;
}

}  // namespace

extern "C" {

int celv2_pruner_forward(const float* params, const float* x, int batch, float* acts, void* stream) {
  if (!params || !x || !acts || batch <= 0) {
    set_last_error("pruner_forward: null buffer or empty batch");
    return CELV2_EINVAL;
  }
  nn::forward(params, x, batch, acts, static_cast<cudaStream_t>(stream));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CELV2_OK : fail("pruner_forward", e);
}

int celv2_pruner_backward(const float* params, int batch, const float* acts, const float* dlogits, float* work,
                          float* grads, void* stream) {
  if (!params || !acts || !dlogits || !work || !grads || batch <= 0) {
    set_last_error("pruner_backward: null buffer or empty batch");
    return CELV2_EINVAL;
  }
  nn::backward(params, batch, acts, dlogits, work, grads, static_cast<cudaStream_t>(stream));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CELV2_OK : fail("pruner_backward", e);
}

int celv2_pruner_bce(const float* logits, const float* labels, const float* weights, int batch, float* dlogits,
                     float* loss, void* stream) {
  if (!logits || !labels || !weights || !dlogits || !loss || batch <= 0) {
    set_last_error("pruner_bce: null buffer or empty batch");
    return CELV2_EINVAL;
  }
  const int n = batch * nn::kOut;
  nn::k_bce<<<nn::grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(logits, labels, weights, n,
                                                                             1.f / (float)batch, dlogits, loss);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CELV2_OK : fail("pruner_bce", e);
}

int celv2_pruner_adam(float* params, const float* grads, float* m, float* v, int n, float lr, float beta1,
                      float beta2, float eps, float weight_decay, int step, void* stream) {
  if (!params || !grads || !m || !v || n <= 0 || step < 1) {
    set_last_error("pruner_adam: null buffer, empty or step < 1");
    return CELV2_EINVAL;
  }
  double c1 = 1.0, c2 = 1.0;
  for (int i = 0; i < step && i < 100000; i++) c1 *= beta1, c2 *= beta2;
  nn::k_adam<<<nn::grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      params, grads, m, v, n, lr, beta1, beta2, eps, weight_decay, (float)(1.0 - c1), (float)(1.0 - c2));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CELV2_OK : fail("pruner_adam", e);
}

}  // extern "C"
