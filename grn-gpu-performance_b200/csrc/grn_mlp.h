// grn_mlp.h -- launch interface of the surrogate MLP kernels (grn_mlp.cu,
// grn_umma.cu).
#ifndef GRN_MLP_H_
#define GRN_MLP_H_

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace grn {

enum MlpEpilogue {
  kEpiF32 = 0,       // C = acc (FP32)
  kEpiBiasRelu = 1,  // C = relu(acc + bias[n]) (BF16)
  kEpiMask = 2       // C = mask > 0 ? acc : 0 (BF16; ReLU backward)
};

// C[m][n] = sum_k A[m][k] B[n][k], both operands K-major (row m of A at
// A + m*lda, row n of B at B + n*ldb); BF16 operands, FP32 accumulation.
// The BF16 epilogues can also store the transposed result,
// Ct[n*ldt + m] = C[m][n].
struct MlpGemm {
  int M, N, K;
  const __nv_bfloat16 *A;
  int64_t lda;
  const __nv_bfloat16 *B;
  int64_t ldb;
  int epi;
  float *Cf;                  // FP32 output (kEpiF32)
  __nv_bfloat16 *Cb;          // BF16 output (kEpiBiasRelu, kEpiMask)
  int64_t ldc;
  __nv_bfloat16 *Ct;          // optional transposed BF16 output
  int64_t ldt;
  const float *bias;          // [N] (kEpiBiasRelu)
  const __nv_bfloat16 *mask;  // [M][ldc] (kEpiMask): keep where mask > 0
};

// The GEMM on warp-level mma.sync (the legacy tensor-core path).
cudaError_t mlp_gemm(const MlpGemm &p, cudaStream_t st);
// The GEMM on the tcgen05 tensor cores with TMA loads (grn_umma.cu).  An
// FP32 GEMM with few output tiles and a long K is split over K into ranges
// whose partial tiles go to `work` (up to work_elems floats) and are then
// added in range order.  Sets *error_flag (device) to 1 if a wait for the
// tensor core or a load timed out.  Operand rows must start on 16 bytes
// (lda, ldb multiples of 8, 16-byte aligned bases): cudaErrorInvalidValue
// otherwise.
cudaError_t mlp_gemm_tc(const MlpGemm &p, float *work, size_t work_elems, int *error_flag,
                        cudaStream_t st);

// y[b] = h[b] . w + b0 (the output layer).
cudaError_t mlp_output_forward(int B, int K, const __nv_bfloat16 *h, const float *w,
                               const float *b0, float *y, cudaStream_t st);
// dy = 2 (y - t) / B; loss[0] = mean (y - t)^2, loss[1] += loss[0];
// db[0] = sum dy (the output bias gradient); *adam_step += 1 unless null
// (a training step's count of Adam steps, read by mlp_adam).
cudaError_t mlp_loss(int B, const float *y, const float *t, float *dy, double *loss, float *db,
                     int *adam_step, cudaStream_t st);
// dz[b][k] = h[b][k] > 0 ? dy[b] w[k] : 0 (BF16), and its transpose dzT[k][b].
cudaError_t mlp_output_backward(int B, int K, const __nv_bfloat16 *h, const float *w,
                                const float *dy, __nv_bfloat16 *dz, __nv_bfloat16 *dzT,
                                int64_t ldt, cudaStream_t st);
// Up to four row reductions in one launch: out_j[r] = sum_c X_j[r][c] (x w[c]
// when w_j is set) for r < rows, c < cols; a fixed summation order.
struct MlpRowSum {
  const __nv_bfloat16 *X;
  const float *w;
  float *out;
};
cudaError_t mlp_row_sums(int n_jobs, const MlpRowSum *jobs, int rows, int cols, int64_t ldx,
                         cudaStream_t st);
// Square n x n blocks of the parameter vector, starting at offset[j], whose
// BF16 transpose Adam also writes to dst[j] (skipped where dst[j] is null).
struct MlpTransposed {
  int64_t offset[2];
  __nv_bfloat16 *dst[2];
  int n;
};
// One Adam step on the FP32 parameters w (moments m, v; step number
// *adam_step, in device memory), refreshing their BF16 copy wb and the
// transposed copies of tr.
cudaError_t mlp_adam(int n, float *w, const float *g, float *m, float *v, float lr, float b1,
                     float b2, float eps, const int *adam_step, __nv_bfloat16 *wb,
                     const MlpTransposed &tr, cudaStream_t st);
cudaError_t mlp_to_bf16(int n, const float *x, __nv_bfloat16 *y, cudaStream_t st);
// dst[c][r] = src[r][c] for a rows x cols BF16 matrix.
cudaError_t mlp_transpose(int rows, int cols, const __nv_bfloat16 *src, int64_t lds,
                          __nv_bfloat16 *dst, int64_t ldd, cudaStream_t st);
// Row r of dst (width columns) = row idx[r] of src, tdst[r] = tsrc[idx[r]];
// dstT (optional) receives the transpose, dstT[c*ldt + r].
cudaError_t mlp_gather_rows(int rows, int width, const int32_t *idx, const __nv_bfloat16 *src,
                            const float *tsrc, __nv_bfloat16 *dst, float *tdst,
                            __nv_bfloat16 *dstT, int64_t ldt, cudaStream_t st);
// FP32 rows to BF16 (dst) and optionally their transpose (dstT).
cudaError_t mlp_convert_rows(int rows, int width, const float *src, __nv_bfloat16 *dst,
                             __nv_bfloat16 *dstT, int64_t ldt, cudaStream_t st);

}  // namespace grn

#endif  // GRN_MLP_H_
