// grn_mlp.h -- launch interface of the surrogate MLP kernels (grn_mlp.cu).
#ifndef GRN_MLP_H_
#define GRN_MLP_H_

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace grn {

enum MlpEpilogue {
  kEpiF32 = 0,       // C = acc (FP32)
  kEpiBiasRelu = 1,  // C = relu(acc + bias[n]) (BF16)
  kEpiMask = 2       // C = mask > 0 ? acc : 0 (BF16; ReLU backward)
};

// C[m][n] = sum_k A(m,k) B(n,k), A(m,k) = A[m*a_rs + k*a_cs],
// B(n,k) = B[n*b_rs + k*b_cs]; BF16 operands, FP32 accumulation.
cudaError_t mlp_gemm(int M, int N, int K, const __nv_bfloat16 *A, int64_t a_rs, int64_t a_cs,
                     const __nv_bfloat16 *B, int64_t b_rs, int64_t b_cs, int epi, float *Cf,
                     __nv_bfloat16 *Cb, int64_t ldc, const float *bias,
                     const __nv_bfloat16 *mask, cudaStream_t st);
// The same GEMM on the tcgen05 tensor cores (grn_umma.cu); sets
// *error_flag (device) to 1 if a wait for the tensor core timed out.
cudaError_t mlp_gemm_tc(int M, int N, int K, const __nv_bfloat16 *A, int64_t a_rs, int64_t a_cs,
                        const __nv_bfloat16 *B, int64_t b_rs, int64_t b_cs, int epi, float *Cf,
                        __nv_bfloat16 *Cb, int64_t ldc, const float *bias,
                        const __nv_bfloat16 *mask, int *error_flag, cudaStream_t st);
cudaError_t mlp_output_forward(int B, int K, const __nv_bfloat16 *h, const float *w,
                               const float *b0, float *y, cudaStream_t st);
cudaError_t mlp_loss(int B, const float *y, const float *t, float *dy, double *loss,
                     cudaStream_t st);
cudaError_t mlp_output_backward(int B, int K, const __nv_bfloat16 *h, const float *w,
                                const float *dy, float *dw, float *db, __nv_bfloat16 *dz,
                                cudaStream_t st);
cudaError_t mlp_column_sum(int B, int N, const __nv_bfloat16 *dz, float *db, cudaStream_t st);
cudaError_t mlp_adam(int n, float *w, const float *g, float *m, float *v, float lr, float b1,
                     float b2, float eps, int t, __nv_bfloat16 *wb, cudaStream_t st);
cudaError_t mlp_to_bf16(int n, const float *x, __nv_bfloat16 *y, cudaStream_t st);
cudaError_t mlp_gather_rows(int rows, int width, const int32_t *idx, const __nv_bfloat16 *src,
                            const float *tsrc, __nv_bfloat16 *dst, float *tdst,
                            cudaStream_t st);

}  // namespace grn

#endif  // GRN_MLP_H_
