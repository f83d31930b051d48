// grn_mlp.cu -- kernels of the surrogate fitness model: a 128-256-256-256-1
// ReLU MLP over a padded encoding of a GRN model, predicting log(error).
//
// This file holds the warp-level mma.sync GEMM (BF16 operands, FP32
// accumulation; the legacy tensor-core path, kept to cross-check the
// tcgen05 GEMM of grn_umma.cu) and the small kernels around the GEMMs:
// output layer, loss, ReLU-backward of the last layer, bias-gradient row
// sums, Adam, and the row gathers and transposes that give the tcgen05 GEMM
// K-major operands.  Every reduction adds in a fixed order, so training is
// deterministic.  No reference counterpart: the reference simulates every
// offspring.

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
  __nv_bfloat16 *Ct;          // optional transposed BF16 output, Ct[n*ldt + m]
  int64_t ldt;
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
        } else {
          if (g.epi == kEpiBiasRelu) {
            v += g.bias[n];
            v = v > 0.0f ? v : 0.0f;
          } else {  // kEpiMask
            v = __bfloat162float(g.mask[o]) > 0.0f ? v : 0.0f;
          }
          g.Cb[o] = __float2bfloat16(v);
          if (g.Ct) g.Ct[(int64_t)n * g.ldt + m] = __float2bfloat16(v);
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

// Loss 1/B sum (y - t)^2, dy = 2 (y - t) / B and db = sum dy; one block of
// kLossThreads, tree sums in a fixed order.  The operands do not alias, so
// a thread's loads are all issued before its first store.
constexpr int kLossThreads = 1024;

__global__ void __launch_bounds__(kLossThreads)
    loss_kernel(int B, const float *__restrict__ y, const float *__restrict__ t,
                float *__restrict__ dy, double *__restrict__ loss, float *__restrict__ db,
                int *__restrict__ adam_step) {
  __shared__ double part[kLossThreads];
  __shared__ float dpart[kLossThreads];
  double s = 0.0;
  float sd = 0.0f;
#pragma unroll 4
  for (int i = threadIdx.x; i < B; i += kLossThreads) {
    const float d = y[i] - t[i];
    const float g = 2.0f * d / (float)B;
    dy[i] = g;
    sd += g;
    s += (double)d * d;
  }
  part[threadIdx.x] = s;
  dpart[threadIdx.x] = sd;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      part[threadIdx.x] += part[threadIdx.x + o];
      dpart[threadIdx.x] += dpart[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double l = part[0] / B;
    loss[0] = l;
    loss[1] += l;
    db[0] = dpart[0];
    if (adam_step) *adam_step += 1;  // the Adam step this minibatch takes
  }
}

// 32 x 32 tiles through shared memory, blocks of 32 x 8 threads: each
// thread moves four elements of a tile row-wise, then four column-wise, so
// that the row-major and the transposed stores are both coalesced.
constexpr int kTile = 32;

// Gradient of the last hidden layer's pre-activation: dz[b][k] =
// h[b][k] > 0 ? dy[b] w[k] : 0 (BF16), and dzT[k][b].
__global__ void output_backward_kernel(int B, int K, const __nv_bfloat16 *h, const float *w,
                                       const float *dy, __nv_bfloat16 *dz, __nv_bfloat16 *dzT,
                                       int64_t ldt) {
  __shared__ __nv_bfloat16 tile[kTile][kTile + 2];
  const int b0 = blockIdx.x * kTile, k0 = blockIdx.y * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int k = k0 + tx;
  const float wk = k < K ? w[k] : 0.0f;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = ty + 8 * i, b = b0 + r;
    __nv_bfloat16 v = __float2bfloat16(0.0f);
    if (b < B && k < K) {
      const float hv = __bfloat162float(h[(int64_t)b * K + k]);
      v = __float2bfloat16(hv > 0.0f ? dy[b] * wk : 0.0f);
      dz[(int64_t)b * K + k] = v;
    }
    tile[r][tx] = v;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int c = ty + 8 * i, b = b0 + tx;
    if (k0 + c < K && b < B) dzT[(int64_t)(k0 + c) * ldt + b] = tile[tx][c];
  }
}

// Rows to BF16: row r is row idx[r] of the BF16 matrix src_b (a gather), or
// row r of the FP32 matrix src_f; tdst[r] = tsrc[idx[r]] when gathering.
// dstT (optional) receives the transpose.
__global__ void rows_to_bf16_kernel(int rows, int width, const int32_t *idx,
                                    const __nv_bfloat16 *src_b, const float *src_f,
                                    const float *tsrc, __nv_bfloat16 *dst, float *tdst,
                                    __nv_bfloat16 *dstT, int64_t ldt) {
  __shared__ __nv_bfloat16 tile[kTile][kTile + 2];
  const int r0 = blockIdx.x * kTile, c0 = blockIdx.y * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int c = c0 + tx;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = ty + 8 * i, row = r0 + r;
    __nv_bfloat16 v = __float2bfloat16(0.0f);
    if (row < rows) {
      const int64_t s = idx ? (int64_t)idx[row] : (int64_t)row;
      if (c < width) {
        v = idx ? src_b[s * width + c] : __float2bfloat16(src_f[s * width + c]);
        dst[(int64_t)row * width + c] = v;
      }
      if (idx && tdst && blockIdx.y == 0 && tx == 0) tdst[row] = tsrc[s];
    }
    tile[r][tx] = v;
  }
  if (!dstT) return;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int cc = ty + 8 * i, row = r0 + tx;
    if (c0 + cc < width && row < rows) dstT[(int64_t)(c0 + cc) * ldt + row] = tile[tx][cc];
  }
}

// dst[c][r] = src[r][c].
__global__ void transpose_kernel(int rows, int cols, const __nv_bfloat16 *src, int64_t lds,
                                 __nv_bfloat16 *dst, int64_t ldd) {
  __shared__ __nv_bfloat16 tile[kTile][kTile + 2];
  const int r0 = blockIdx.x * kTile, c0 = blockIdx.y * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = ty + 8 * i;
    tile[r][tx] = (r0 + r < rows && c0 + tx < cols) ? src[(int64_t)(r0 + r) * lds + c0 + tx]
                                                    : __float2bfloat16(0.0f);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int cc = ty + 8 * i;
    if (c0 + cc < cols && r0 + tx < rows) dst[(int64_t)(c0 + cc) * ldd + r0 + tx] = tile[tx][cc];
  }
}

struct RowSumJobs {
  MlpRowSum j[4];
};

// out[r] = sum_c X[r][c] (x w[c]): one block of 256 threads per row and
// job; each thread adds a fixed strided subset, then a fixed-order tree.
__global__ void __launch_bounds__(256) row_sums_kernel(const RowSumJobs jobs, int cols,
                                                       int64_t ldx) {
  __shared__ float part[256];
  // Selected without a dynamic index into the parameter block (which would
  // copy it to local memory).
  const unsigned y = blockIdx.y;
  const MlpRowSum jb = y == 0 ? jobs.j[0] : y == 1 ? jobs.j[1] : y == 2 ? jobs.j[2] : jobs.j[3];
  const __nv_bfloat16 *x = jb.X + (int64_t)blockIdx.x * ldx;
  float s = 0.0f;
  const bool vec = (cols & 7) == 0 && (ldx & 7) == 0 && ((uintptr_t)jb.X & 15) == 0 &&
                   (!jb.w || ((uintptr_t)jb.w & 15) == 0);
  if (vec) {
    for (int c = threadIdx.x * 8; c < cols; c += 256 * 8) {
      const uint4 u = *reinterpret_cast<const uint4 *>(x + c);
      const __nv_bfloat162 *p = reinterpret_cast<const __nv_bfloat162 *>(&u);
      float e[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float2 f = __bfloat1622float2(p[q]);
        e[2 * q] = f.x;
        e[2 * q + 1] = f.y;
      }
      if (jb.w) {
        const float4 w0 = *reinterpret_cast<const float4 *>(jb.w + c);
        const float4 w1 = *reinterpret_cast<const float4 *>(jb.w + c + 4);
        e[0] *= w0.x, e[1] *= w0.y, e[2] *= w0.z, e[3] *= w0.w;
        e[4] *= w1.x, e[5] *= w1.y, e[6] *= w1.z, e[7] *= w1.w;
      }
      s += ((e[0] + e[1]) + (e[2] + e[3])) + ((e[4] + e[5]) + (e[6] + e[7]));
    }
  } else {
    for (int c = threadIdx.x; c < cols; c += 256) {
      const float v = __bfloat162float(x[c]);
      s += jb.w ? v * jb.w[c] : v;
    }
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) jb.out[blockIdx.x] = part[0];
}

// Adam on FP32 master weights, step t = *adam_step (device memory, so that
// a captured training step replays as is); refreshes the BF16 copy and the
// transposed BF16 copies of the square matrices listed in tr.
__global__ void adam_kernel(int n, float *w, const float *g, float *m, float *v, float lr,
                            float b1, float b2, float eps, const int *adam_step,
                            __nv_bfloat16 *wb, const MlpTransposed tr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float t = (float)*adam_step;
  const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (!wb) return;
  const __nv_bfloat16 wv = __float2bfloat16(wi);
  wb[i] = wv;
  const int64_t nn = (int64_t)tr.n * tr.n;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int64_t o = i - tr.offset[j];
    if (tr.dst[j] && o >= 0 && o < nn) {
      const int r = (int)(o / tr.n), c = (int)(o - (int64_t)r * tr.n);
      tr.dst[j][(int64_t)c * tr.n + r] = wv;
    }
  }
}

__global__ void to_bf16_kernel(int n, const float *x, __nv_bfloat16 *y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16(x[i]);
}

dim3 tile_grid(int rows, int cols) {
  return dim3((rows + kTile - 1) / kTile, (cols + kTile - 1) / kTile);
}

}  // namespace

cudaError_t mlp_gemm(const MlpGemm &p, cudaStream_t st) {
  if (p.M < 1 || p.N < 1 || p.K < 1) return cudaErrorInvalidValue;
  GemmArgs g{p.M, p.N, p.K, p.A, p.lda, 1, p.B, p.ldb, 1, p.epi, p.Cf, p.Cb, p.ldc,
             p.bias, p.mask, p.Ct, p.ldt};
  dim3 grid((p.N + kTN - 1) / kTN, (p.M + kTM - 1) / kTM);
  gemm_bf16_kernel<<<grid, 128, 0, st>>>(g);
  return cudaGetLastError();
}

cudaError_t mlp_output_forward(int B, int K, const __nv_bfloat16 *h, const float *w,
                               const float *b0, float *y, cudaStream_t st) {
  if (B < 1) return cudaSuccess;
  output_forward_kernel<<<(B * 32 + 255) / 256, 256, 0, st>>>(B, K, h, w, b0, y);
  return cudaGetLastError();
}

cudaError_t mlp_loss(int B, const float *y, const float *t, float *dy, double *loss, float *db,
                     int *adam_step, cudaStream_t st) {
  loss_kernel<<<1, kLossThreads, 0, st>>>(B, y, t, dy, loss, db, adam_step);
  return cudaGetLastError();
}

cudaError_t mlp_output_backward(int B, int K, const __nv_bfloat16 *h, const float *w,
                                const float *dy, __nv_bfloat16 *dz, __nv_bfloat16 *dzT,
                                int64_t ldt, cudaStream_t st) {
  if (B < 1 || K < 1) return cudaSuccess;
  output_backward_kernel<<<tile_grid(B, K), dim3(kTile, 8), 0, st>>>(B, K, h, w, dy, dz, dzT,
                                                                     ldt);
  return cudaGetLastError();
}

cudaError_t mlp_row_sums(int n_jobs, const MlpRowSum *jobs, int rows, int cols, int64_t ldx,
                         cudaStream_t st) {
  if (n_jobs < 1 || n_jobs > 4 || rows < 1) return cudaErrorInvalidValue;
  RowSumJobs j{};
  for (int i = 0; i < n_jobs; ++i) j.j[i] = jobs[i];
  row_sums_kernel<<<dim3(rows, n_jobs), 256, 0, st>>>(j, cols, ldx);
  return cudaGetLastError();
}

cudaError_t mlp_adam(int n, float *w, const float *g, float *m, float *v, float lr, float b1,
                     float b2, float eps, const int *adam_step, __nv_bfloat16 *wb,
                     const MlpTransposed &tr, cudaStream_t st) {
  adam_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, w, g, m, v, lr, b1, b2, eps, adam_step, wb,
                                               tr);
  return cudaGetLastError();
}

cudaError_t mlp_to_bf16(int n, const float *x, __nv_bfloat16 *y, cudaStream_t st) {
  to_bf16_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, x, y);
  return cudaGetLastError();
}

cudaError_t mlp_transpose(int rows, int cols, const __nv_bfloat16 *src, int64_t lds,
                          __nv_bfloat16 *dst, int64_t ldd, cudaStream_t st) {
  if (rows < 1 || cols < 1) return cudaSuccess;
  transpose_kernel<<<tile_grid(rows, cols), dim3(kTile, 8), 0, st>>>(rows, cols, src, lds, dst,
                                                                     ldd);
  return cudaGetLastError();
}

cudaError_t mlp_gather_rows(int rows, int width, const int32_t *idx, const __nv_bfloat16 *src,
                            const float *tsrc, __nv_bfloat16 *dst, float *tdst,
                            __nv_bfloat16 *dstT, int64_t ldt, cudaStream_t st) {
  if (rows < 1) return cudaSuccess;
  rows_to_bf16_kernel<<<tile_grid(rows, width), dim3(kTile, 8), 0, st>>>(
      rows, width, idx, src, nullptr, tsrc, dst, tdst, dstT, ldt);
  return cudaGetLastError();
}

cudaError_t mlp_convert_rows(int rows, int width, const float *src, __nv_bfloat16 *dst,
                             __nv_bfloat16 *dstT, int64_t ldt, cudaStream_t st) {
  if (rows < 1) return cudaSuccess;
  rows_to_bf16_kernel<<<tile_grid(rows, width), dim3(kTile, 8), 0, st>>>(
      rows, width, nullptr, nullptr, src, nullptr, dst, nullptr, dstT, ldt);
  return cudaGetLastError();
}

}  // namespace grn
