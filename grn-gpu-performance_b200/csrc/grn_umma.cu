// grn_umma.cu -- the surrogate MLP's GEMMs on the fifth-generation tensor
// cores (tcgen05.mma, kind::f16: BF16 x BF16 -> FP32 in tensor memory).
//
// C[m][n] = sum_k A(m, k) B(n, k) with A(m, k) = A[m*a_rs + k*a_cs] and
// B(n, k) = B[n*b_rs + k*b_cs], so row-major, transposed and column-major
// operands are one kernel.  A CTA computes a 128 x 64 tile (the MLP's
// GEMMs are small: narrow tiles give more CTAs) with 4 warps:
//   - the block gathers a 128 x 64 slice of A and a 64 x 64 slice of B into
//     shared memory in the K-major, non-swizzled core-matrix layout the
//     tensor core reads (8 rows x 16 bytes per core matrix; zero fill past
//     the edges), then fences the generic writes for the async proxy;
//   - one thread issues the slice's four K = 16 MMAs on shared-memory
//     descriptors and commits them to an mbarrier; every thread waits for it
//     (bounded) before the next slice reuses the buffers;
//   - the accumulator lives in tensor memory (warp 0 allocates 64 columns):
//     row m of the tile is lane m, so warp w reads rows 32w .. 32w + 31 with
//     tcgen05.ld and applies the epilogue (FP32 store, bias + ReLU to BF16,
//     or the ReLU-backward mask to BF16).
// Descriptor and instruction-descriptor bit fields follow the PTX ISA's
// tcgen05 shared-memory descriptor and kind::f16 instruction descriptor.

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "grn_mlp.h"

namespace grn {
namespace {

constexpr int kTM = 128;  // tile rows (M of one MMA, cta_group::1)
constexpr int kKC = 64;   // K per shared-memory slice (four K = 16 MMAs)

struct UmmaArgs {
  int M, N, K;
  const __nv_bfloat16 *A;
  int64_t a_rs, a_cs;
  const __nv_bfloat16 *B;
  int64_t b_rs, b_cs;
  int epi;
  float *Cf;
  __nv_bfloat16 *Cb;
  int64_t ldc;
  const float *bias;
  const __nv_bfloat16 *mask;
  int *error_flag;  // set to 1 if a wait for the tensor core timed out
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, no swizzle: start address,
// leading byte offset (between the two 8-element K halves of an MMA's
// K = 16), stride byte offset (between 8-row groups), all in 16-byte units;
// descriptor version 1 (bits 46-47), base offset 0, layout type 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9 and 10-12 = 1), both K-major (bits 15, 16 = 0),
// N / 8 at bits 17-22, M / 16 at bits 24-28.
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait (about one second): false on a time-out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 0; i < (1u << 30); ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > 1000000000ull) return false;
  }
  return false;
}

// Core-matrix offset (in elements) of element (row r, column c) of a
// K-major slice with kKC columns: core matrix (r / 8, c / 8) is 64
// contiguous elements, row-major inside.
__device__ __forceinline__ int cm_offset(int r, int c) {
  return ((r >> 3) * (kKC / 8) + (c >> 3)) * 64 + (r & 7) * 8 + (c & 7);
}

// Gathers rows [r0, r0 + ROWS) x columns [k0, k0 + kKC) of X (element (r, k)
// at X[r*rs + k*cs]) into a K-major core-matrix slice, zero past rows / ks.
// K-contiguous operands move 8 elements (one core-matrix row, 16 bytes) per
// load; row-contiguous (transposed) ones 8 rows of one column per load.
template <int ROWS>
__device__ __forceinline__ void fill_slice(__nv_bfloat16 *s, const __nv_bfloat16 *X, int64_t rs,
                                           int64_t cs, int r0, int nr, int k0, int nk,
                                           int tid) {
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  if (cs == 1 && (rs & 7) == 0 && ((uintptr_t)X & 15) == 0) {
    for (int i = tid; i < ROWS * (kKC / 8); i += 128) {
      const int r = i / (kKC / 8), c8 = (i - r * (kKC / 8)) * 8;
      const int row = r0 + r, k = k0 + c8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (row < nr && k + 8 <= nk) {
        v = *reinterpret_cast<const uint4 *>(X + row * rs + k);
      } else if (row < nr) {
        __nv_bfloat16 t[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) t[j] = k + j < nk ? X[row * rs + k + j] : zero;
        v = *reinterpret_cast<const uint4 *>(t);
      }
      *reinterpret_cast<uint4 *>(s + cm_offset(r, c8)) = v;
    }
  } else if (rs == 1 && (cs & 7) == 0 && ((uintptr_t)X & 15) == 0) {
    for (int i = tid; i < (ROWS / 8) * kKC; i += 128) {
      const int c = i / (ROWS / 8), r8 = (i - c * (ROWS / 8)) * 8;
      const int row = r0 + r8, k = k0 + c;
      __nv_bfloat16 t[8];
      if (k < nk && row + 8 <= nr) {
        *reinterpret_cast<uint4 *>(t) = *reinterpret_cast<const uint4 *>(X + row + k * cs);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) t[j] = (k < nk && row + j < nr) ? X[row + j + k * cs] : zero;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) s[cm_offset(r8 + j, c)] = t[j];
    }
  } else {
    for (int i = tid; i < ROWS * kKC; i += 128) {
      const int r = i / kKC, c = i - (i / kKC) * kKC;
      const int row = r0 + r, k = k0 + c;
      s[cm_offset(r, c)] = (row < nr && k < nk) ? X[row * rs + k * cs] : zero;
    }
  }
}

template <int BN>
__global__ void __launch_bounds__(128) umma_gemm_kernel(const UmmaArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __nv_bfloat16 *sa = reinterpret_cast<__nv_bfloat16 *>(smem);
  __nv_bfloat16 *sb = sa + kTM * kKC;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sb + BN * kKC);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTM, n0 = blockIdx.y * BN;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  const uint32_t bar_addr = smem_u32(bar);
  bool ok = true;
  uint32_t phase = 0;

  for (int k0 = 0; k0 < g.K && ok; k0 += kKC) {
    fill_slice<kTM>(sa, g.A, g.a_rs, g.a_cs, m0, g.M, k0, g.K, tid);
    fill_slice<BN>(sb, g.B, g.b_rs, g.b_cs, n0, g.N, k0, g.K, tid);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t idesc = instr_desc(kTM, BN);
      const uint32_t lbo = 128, sbo = (kKC / 8) * 128;  // bytes
#pragma unroll
      for (int ks = 0; ks < kKC / 16; ++ks) {
        const uint64_t ad = smem_desc(smem_u32(sa) + ks * 256, lbo, sbo);
        const uint64_t bd = smem_desc(smem_u32(sb) + ks * 256, lbo, sbo);
        const uint32_t acc = (k0 > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u),
            "r"(0u));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              bar_addr)
          : "memory");
    }
    ok = mbar_wait(bar_addr, phase);
    phase ^= 1u;
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;");
  }

  if (ok) {
    const int m = m0 + warp * 32 + lane;  // TMEM lane = tile row
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
          "%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, "
          "%26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
            "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
            "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
            "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < g.M) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int n = n0 + c0 + j;
          if (n >= g.N) break;
          float x = __uint_as_float(v[j]);
          const int64_t o = (int64_t)m * g.ldc + n;
          if (g.epi == kEpiF32) {
            g.Cf[o] = x;
          } else if (g.epi == kEpiBiasRelu) {
            x += g.bias[n];
            g.Cb[o] = __float2bfloat16(x > 0.0f ? x : 0.0f);
          } else {
            g.Cb[o] = __float2bfloat16(__bfloat162float(g.mask[o]) > 0.0f ? x : 0.0f);
          }
        }
      }
    }
  } else {
    // A slice's MMAs did not complete in time: wait once more (bounded) so
    // that none is in flight when the accumulator is freed, and report.
    mbar_wait(bar_addr, phase ^ 1u);
    if (tid == 0) atomicExch(g.error_flag, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
  }
}

template <int BN>
size_t umma_smem_bytes() {
  return (size_t)(kTM + BN) * kKC * sizeof(__nv_bfloat16) + 16;
}

}  // namespace

cudaError_t mlp_gemm_tc(int M, int N, int K, const __nv_bfloat16 *A, int64_t a_rs, int64_t a_cs,
                        const __nv_bfloat16 *B, int64_t b_rs, int64_t b_cs, int epi, float *Cf,
                        __nv_bfloat16 *Cb, int64_t ldc, const float *bias,
                        const __nv_bfloat16 *mask, int *error_flag, cudaStream_t st) {
  if (M < 1 || N < 1 || K < 1 || !error_flag) return cudaErrorInvalidValue;
  UmmaArgs g{M, N, K, A, a_rs, a_cs, B, b_rs, b_cs, epi, Cf, Cb, ldc, bias, mask, error_flag};
  // 128 x 64 tiles: more CTAs for the MLP's small GEMMs than 128 x 256 ones.
  const size_t smem = umma_smem_bytes<64>();
  cudaError_t e = cudaFuncSetAttribute(umma_gemm_kernel<64>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  umma_gemm_kernel<64><<<dim3((M + kTM - 1) / kTM, (N + 63) / 64), 128, smem, st>>>(g);
  return cudaGetLastError();
}

}  // namespace grn
