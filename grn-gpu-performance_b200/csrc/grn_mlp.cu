// grn_mlp.cu -- kernels of the surrogate fitness model: a 128-256-256-256-1
// ReLU MLP over a padded encoding of a GRN model, predicting log(error).
//
// GEMMs use the tensor cores with BF16 operands and FP32 accumulation
// (mma.sync m16n8k16); everything else (bias, ReLU masks, loss, reductions,
// Adam) is plain FP32 SIMT.  No reference counterpart: the reference
// simulates every offspring.

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "grn_mlp.h"

namespace grn {
namespace {

// ---- tensor-core GEMM --------------------------------------------------
//
// C[m][n] = sum_k A(m, k) * B(n, k) for A element (m, k) at A[m*a_rs + k*a_cs]
// and B element (n, k) at B[n*b_rs + k*b_cs], so row-major, transposed and
// column-major operands are all one kernel.  A block computes a 64 x 64 tile
// with 4 warps (2 x 2, 32 x 32 each); K advances 32 at a time through
// shared memory (zero-filled past the edges), fragments come from ldmatrix.

constexpr int kTM = 64, kTN = 64, kTK = 32;
constexpr int kLds = kTK + 8;  // padded shared row (halves): no ldmatrix bank conflicts

struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16 *A;
  int64_t a_rs, a_cs;
  const __nv_bfloat16 *B;
  int64_t b_rs, b_cs;
  // epilogue
  int epi;
  float *Cf;                  // FP32 output (kEpiF32)
  __nv_bfloat16 *Cb;          // BF16 output (kEpiBiasRelu, kEpiMask)
  int64_t ldc;
  const float *bias;          // [N] (kEpiBiasRelu)
  const __nv_bfloat16 *mask;  // [M][ldc] (kEpiMask): keep where mask > 0
};

__device__ __forceinline__ void ldmatrix_x4(uint32_t (&r)[4], const void *p) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ void ldmatrix_x2(uint32_t (&r)[2], const void *p) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];"
               : "=r"(r[0]), "=r"(r[1])
               : "r"(a));
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4],
                                         const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) gemm_bf16_kernel(const GemmArgs g) {
  __shared__ __align__(16) __nv_bfloat16 sa[kTM][kLds];
  __shared__ __align__(16) __nv_bfloat16 sb[kTN][kLds];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;  // warp's 32 x 32 sub-tile
  const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
  float acc[2][4][4] = {};
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  for (int k0 = 0; k0 < g.K; k0 += kTK) {
    for (int i = tid; i < kTM * kTK; i += 128) {
      const int r = i / kTK, c = i % kTK;
      const int m = m0 + r, k = k0 + c;
      sa[r][c] = (m < g.M && k < g.K) ? g.A[m * g.a_rs + k * g.a_cs] : zero;
      const int n = n0 + r;
      sb[r][c] = (n < g.N && k < g.K) ? g.B[n * g.b_rs + k * g.b_cs] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTK; kk += 16) {
      uint32_t af[2][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        // 16 x 16 A sub-tile: lanes 0-15 rows 0-15 at k, lanes 16-31 at k + 8
        const int row = wm * 32 + i * 16 + (lane & 15);
        const int col = kk + (lane >> 4) * 8;
        ldmatrix_x4(af[i], &sa[row][col]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        // 8 x 16 B sub-tile (n rows, k columns): lanes 0-7 at k, 8-15 at k + 8
        const int row = wn * 32 + j * 8 + (lane & 7);
        const int col = kk + ((lane >> 3) & 1) * 8;
        ldmatrix_x2(bf[j], &sb[row][col]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();
  }
  // Epilogue.  Accumulator element (row, col) of m16n8: c0, c1 at
  // (lane / 4, 2 * (lane % 4) + {0, 1}), c2, c3 eight rows below.
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const int m = m0 + wm * 32 + i * 16 + (lane >> 2) + (h >> 1) * 8;
        const int n = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + (h & 1);
        if (m >= g.M || n >= g.N) continue;
        float v = acc[i][j][h];
        const int64_t o = (int64_t)m * g.ldc + n;
        if (g.epi == kEpiF32) {
          g.Cf[o] = v;
        } else if (g.epi == kEpiBiasRelu) {
          v += g.bias[n];
          g.Cb[o] = __float2bfloat16(v > 0.0f ? v : 0.0f);
        } else {  // kEpiMask
          g.Cb[o] = __float2bfloat16(__bfloat162float(g.mask[o]) > 0.0f ? v : 0.0f);
        }
      }
}

// ---- small kernels -----------------------------------------------------

// y[b] = h[b] . w + b0 (output layer), FP32 accumulate; one warp per row.
__global__ void output_forward_kernel(int B, int K, const __nv_bfloat16 *h, const float *w,
                                      const float *b0, float *y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= B) return;
  float s = 0.0f;
  for (int k = lane; k < K; k += 32) s += __bfloat162float(h[(int64_t)warp * K + k]) * w[k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[warp] = s + b0[0];
}

// Loss 1/B sum (y - t)^2 and dy = 2 (y - t) / B.
__global__ void loss_kernel(int B, const float *y, const float *t, float *dy, double *loss) {
  __shared__ double part[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    const float d = y[i] - t[i];
    dy[i] = 2.0f * d / (float)B;
    s += (double)d * d;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = part[0] / B;
}

// Gradients of the output layer: dw[k] = sum_b dy[b] h[b][k], db = sum dy,
// and dz[b][k] = dy[b] w[k] where h[b][k] > 0 (BF16, next backward GEMM).
__global__ void output_backward_kernel(int B, int K, const __nv_bfloat16 *h, const float *w,
                                       const float *dy, float *dw, float *db,
                                       __nv_bfloat16 *dz) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < K) {
    float s = 0.0f;
    for (int b = 0; b < B; ++b) {
      const float hv = __bfloat162float(h[(int64_t)b * K + k]);
      s += dy[b] * hv;
      dz[(int64_t)b * K + k] = __float2bfloat16(hv > 0.0f ? dy[b] * w[k] : 0.0f);
    }
    dw[k] = s;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float s = 0.0f;
    for (int b = 0; b < B; ++b) s += dy[b];
    db[0] = s;
  }
}

// db[n] = sum_b dz[b][n] (bias gradients of the hidden layers).
__global__ void column_sum_kernel(int B, int N, const __nv_bfloat16 *dz, float *db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.0f;
  for (int b = 0; b < B; ++b) s += __bfloat162float(dz[(int64_t)b * N + n]);
  db[n] = s;
}

// Adam on FP32 master weights; refreshes the BF16 copy.
__global__ void adam_kernel(int n, float *w, const float *g, float *m, float *v, float lr,
                            float b1, float b2, float eps, float c1, float c2,
                            __nv_bfloat16 *wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(int n, const float *x, __nv_bfloat16 *y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16(x[i]);
}

// out[r] = src[idx[r]] rows of `width` (training minibatch gather).
__global__ void gather_rows_kernel(int rows, int width, const int32_t *idx,
                                   const __nv_bfloat16 *src, const float *tsrc,
                                   __nv_bfloat16 *dst, float *tdst) {
  const int r = blockIdx.x;
  if (r >= rows) return;
  const int64_t s = idx[r];
  for (int c = threadIdx.x; c < width; c += blockDim.x)
    dst[(int64_t)r * width + c] = src[s * width + c];
  if (threadIdx.x == 0) tdst[r] = tsrc[s];
}

}  // namespace

cudaError_t mlp_gemm(int M, int N, int K, const __nv_bfloat16 *A, int64_t a_rs, int64_t a_cs,
                     const __nv_bfloat16 *B, int64_t b_rs, int64_t b_cs, int epi, float *Cf,
                     __nv_bfloat16 *Cb, int64_t ldc, const float *bias,
                     const __nv_bfloat16 *mask, cudaStream_t st) {
  GemmArgs g{M, N, K, A, a_rs, a_cs, B, b_rs, b_cs, epi, Cf, Cb, ldc, bias, mask};
  dim3 grid((N + kTN - 1) / kTN, (M + kTM - 1) / kTM);
  gemm_bf16_kernel<<<grid, 128, 0, st>>>(g);
  return cudaGetLastError();
}

cudaError_t mlp_output_forward(int B, int K, const __nv_bfloat16 *h, const float *w,
                               const float *b0, float *y, cudaStream_t st) {
  output_forward_kernel<<<(B * 32 + 255) / 256, 256, 0, st>>>(B, K, h, w, b0, y);
  return cudaGetLastError();
}

cudaError_t mlp_loss(int B, const float *y, const float *t, float *dy, double *loss,
                     cudaStream_t st) {
  loss_kernel<<<1, 256, 0, st>>>(B, y, t, dy, loss);
  return cudaGetLastError();
}

cudaError_t mlp_output_backward(int B, int K, const __nv_bfloat16 *h, const float *w,
                                const float *dy, float *dw, float *db, __nv_bfloat16 *dz,
                                cudaStream_t st) {
  output_backward_kernel<<<(K + 127) / 128, 128, 0, st>>>(B, K, h, w, dy, dw, db, dz);
  return cudaGetLastError();
}

cudaError_t mlp_column_sum(int B, int N, const __nv_bfloat16 *dz, float *db, cudaStream_t st) {
  column_sum_kernel<<<(N + 127) / 128, 128, 0, st>>>(B, N, dz, db);
  return cudaGetLastError();
}

cudaError_t mlp_adam(int n, float *w, const float *g, float *m, float *v, float lr, float b1,
                     float b2, float eps, int t, __nv_bfloat16 *wb, cudaStream_t st) {
  const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
  adam_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, w, g, m, v, lr, b1, b2, eps, c1, c2, wb);
  return cudaGetLastError();
}

cudaError_t mlp_to_bf16(int n, const float *x, __nv_bfloat16 *y, cudaStream_t st) {
  to_bf16_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, x, y);
  return cudaGetLastError();
}

cudaError_t mlp_gather_rows(int rows, int width, const int32_t *idx, const __nv_bfloat16 *src,
                            const float *tsrc, __nv_bfloat16 *dst, float *tdst,
                            cudaStream_t st) {
  if (rows == 0) return cudaSuccess;
  gather_rows_kernel<<<rows, 128, 0, st>>>(rows, width, idx, src, tsrc, dst, tdst);
  return cudaGetLastError();
}

}  // namespace grn
