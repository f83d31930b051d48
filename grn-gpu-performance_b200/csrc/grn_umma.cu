// grn_umma.cu -- the surrogate MLP's GEMMs on the fifth-generation tensor
// cores (tcgen05.mma, kind::f16: BF16 x BF16 -> FP32 in tensor memory),
// fed by TMA.
//
// C[m][n] = sum_k A[m][k] B[n][k] with both operands K-major (the MLP keeps
// transposed copies of the activations, gradients and weights that its
// backward GEMMs read, written by the epilogues that produce them).  A CTA
// computes a 128 x 64 tile with 4 warps and a 4-stage shared-memory ring:
//   - thread 0 (producer) loads 64-wide K slices of A (128 rows) and B (64
//     rows) with cp.async.bulk.tensor (128-byte swizzle, zero fill past the
//     edges) into the next stage once that stage's "empty" barrier has
//     flipped, and arms the stage's "full" barrier with the byte count;
//   - thread 32 (MMA issuer) waits for "full", issues the slice's four
//     K = 16 MMAs on shared-memory descriptors and commits them to the
//     stage's "empty" barrier, so a load waits for the tensor core only when
//     the ring wraps; after the last slice it commits to "done";
//   - all 4 warps wait for "done" and read the accumulator (tile row m =
//     TMEM lane m; warp w reads lanes 32w .. 32w + 31) with tcgen05.ld for
//     the epilogue: FP32 store, bias + ReLU to BF16, or the ReLU-backward
//     mask to BF16, each row written with 16-byte stores, plus an optional
//     transposed BF16 copy (coalesced across the warp's 32 rows).
// Split K: blockIdx.z takes K range z.  With more than one range, each CTA
// stores its FP32 partial tile to a workspace and a second kernel adds the
// ranges in order, so the result is deterministic.  The weight-gradient
// GEMMs (256 x 256 outputs, K = the batch) need it: 8 tiles alone would
// leave most SMs idle.
// Every wait is bounded (about a second); on a time-out the CTA waits again
// (bounded) for its loads and MMAs in flight, frees its tensor memory, sets
// the error flag and returns.
// Descriptor and instruction-descriptor bit fields follow the PTX ISA's
// tcgen05 shared-memory descriptor and kind::f16 instruction descriptor.

#include <cuda.h>  // CUtensorMap and the tensor-map encoder's types (no libcuda link)
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "grn_mlp.h"

namespace grn {
namespace {

constexpr int kTM = 128;     // tile rows (M of one MMA, cta_group::1)
constexpr int kBN = 64;      // tile columns
constexpr int kKC = 64;      // K per stage: 128 bytes of BF16, the swizzle span
constexpr int kStages = 4;
constexpr int kABytes = kTM * kKC * 2;
constexpr int kBBytes = kBN * kKC * 2;
constexpr int kStageBytes = kABytes + kBBytes;
// 1 KB of slack to align the ring to the 1024-byte swizzle atom, the ring,
// the barriers (full, empty per stage; done) and four control words.
constexpr size_t kSmemBytes = 1024 + (size_t)kStages * kStageBytes + 8 * (2 * kStages + 1) + 16;
constexpr int kTargetCtas = 148;  // split K until about one CTA per SM runs
constexpr int kMinSlices = 2;     // K slices per range at least

struct UmmaArgs {
  int M, N, K;
  int k_split;  // K range of one blockIdx.z (a multiple of kKC)
  int epi;
  float *Cf;
  __nv_bfloat16 *Cb;
  int64_t ldc;
  __nv_bfloat16 *Ct;
  int64_t ldt;
  const float *bias;
  const __nv_bfloat16 *mask;
  float *work;      // split-K partial tiles [z][M][N]; null without a split
  int *error_flag;  // set to 1 if a wait timed out
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major with the 128-byte swizzle: start
// address, leading byte offset (unused for swizzled K-major; 16 bytes),
// stride byte offset 1024 (between 8-row groups), all in 16-byte units;
// descriptor version 1 (bits 46-47), base offset 0, swizzle mode 2
// (128-byte, bits 61-63).  The ring's stages start on 1024-byte boundaries;
// an MMA's K = 16 step inside the 128-byte row moves the start by 32 bytes.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
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

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

// 2-D tiled TMA load of the box at (x = K offset, y = row) into shared
// memory, completing on the mbarrier's transaction count.  No multicast.
__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x,
                                         int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
  const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&p);
}

// Epilogue of 32 consecutive columns nb .. nb + nn - 1 of tile row m.
__device__ __forceinline__ void store_row(const UmmaArgs &g, int m, int nb, int nn,
                                          const uint32_t (&v)[32]) {
  float x[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) x[j] = __uint_as_float(v[j]);
  if (g.work || g.epi == kEpiF32) {
    float *dst = g.work ? g.work + ((int64_t)blockIdx.z * g.M + m) * g.N + nb
                        : g.Cf + (int64_t)m * g.ldc + nb;
    if (nn == 32 && ((uintptr_t)dst & 15) == 0) {
#pragma unroll
      for (int q = 0; q < 8; ++q)
        reinterpret_cast<float4 *>(dst)[q] =
            make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < nn) dst[j] = x[j];
    }
    return;
  }
  if (g.epi == kEpiBiasRelu) {
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (j < nn) {
        const float y = x[j] + g.bias[nb + j];
        x[j] = y > 0.0f ? y : 0.0f;
      }
  } else {  // kEpiMask
    const __nv_bfloat16 *mk = g.mask + (int64_t)m * g.ldc + nb;
    if (nn == 32 && ((uintptr_t)mk & 15) == 0) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint4 u = reinterpret_cast<const uint4 *>(mk)[q];
        const __nv_bfloat162 *p = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float2 f = __bfloat1622float2(p[e]);
          x[8 * q + 2 * e] = f.x > 0.0f ? x[8 * q + 2 * e] : 0.0f;
          x[8 * q + 2 * e + 1] = f.y > 0.0f ? x[8 * q + 2 * e + 1] : 0.0f;
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < nn) x[j] = __bfloat162float(mk[j]) > 0.0f ? x[j] : 0.0f;
    }
  }
  __nv_bfloat16 *dst = g.Cb + (int64_t)m * g.ldc + nb;
  if (nn == 32 && ((uintptr_t)dst & 15) == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      reinterpret_cast<uint4 *>(dst)[q] =
          make_uint4(bf16x2(x[8 * q], x[8 * q + 1]), bf16x2(x[8 * q + 2], x[8 * q + 3]),
                     bf16x2(x[8 * q + 4], x[8 * q + 5]), bf16x2(x[8 * q + 6], x[8 * q + 7]));
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (j < nn) dst[j] = __float2bfloat16(x[j]);
  }
  if (g.Ct) {
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (j < nn) g.Ct[(int64_t)(nb + j) * g.ldt + m] = __float2bfloat16(x[j]);
  }
}

__global__ void __launch_bounds__(128) umma_gemm_kernel(const __grid_constant__ CUtensorMap ta,
                                                        const __grid_constant__ CUtensorMap tb,
                                                        const UmmaArgs g) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t ring = (raw + 1023u) & ~1023u;
  unsigned char *smem = smem_raw + (ring - raw);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kStages * kStageBytes);
  // ctl[0] tensor-memory address, ctl[1] failure, ctl[2] slices loaded,
  // ctl[3] slices consumed by the MMA issuer.
  volatile int *ctl = reinterpret_cast<volatile int *>(bars + 2 * kStages + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTM, n0 = blockIdx.y * kBN;
  const int kbeg = blockIdx.z * g.k_split;
  const int nk = (min(g.K, kbeg + g.k_split) - kbeg + kKC - 1) / kKC;
  const uint32_t sa = ring, sb = ring + kStages * kABytes;
  const uint32_t full = smem_u32(bars), empty = full + 8 * kStages, done = full + 16 * kStages;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32((const void *)ctl)),
                 "r"(kBN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < 2 * kStages + 1; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full + 8 * i));
    ctl[1] = 0;
    ctl[2] = 0;
    ctl[3] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = (uint32_t)ctl[0];

  if (tid == 0) {
    int i = 0;
    for (; i < nk; ++i) {
      const int s = i % kStages;
      if (i >= kStages && !mbar_wait(empty + 8 * s, ((i / kStages) - 1) & 1)) break;
      const int k0 = kbeg + i * kKC;
      mbar_expect_tx(full + 8 * s, kStageBytes);
      tma_load(sa + s * kABytes, &ta, full + 8 * s, k0, m0);
      tma_load(sb + s * kBBytes, &tb, full + 8 * s, k0, n0);
    }
    ctl[2] = i;
    if (i < nk) ctl[1] = 1;
  } else if (tid == 32) {
    const uint32_t idesc = instr_desc(kTM, kBN);
    int i = 0;
    for (; i < nk; ++i) {
      const int s = i % kStages;
      if (!mbar_wait(full + 8 * s, (i / kStages) & 1)) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int ks = 0; ks < kKC / 16; ++ks) {
        const uint64_t ad = sw128_desc(sa + s * kABytes + ks * 32);
        const uint64_t bd = sw128_desc(sb + s * kBBytes + ks * 32);
        const uint32_t acc = (i > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
                tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      mma_commit(empty + 8 * s);
    }
    // Arrives once every MMA issued above has completed.
    mma_commit(done);
    ctl[3] = i;
    if (i < nk) ctl[1] = 1;
  }

  const bool waited = mbar_wait(done, 0);
  const bool ok = __syncthreads_and(waited) && ctl[1] == 0;
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    const int m = m0 + warp * 32 + lane;  // TMEM lane = tile row
#pragma unroll 1
    for (int c0 = 0; c0 < kBN; c0 += 32) {
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
      const int nb = n0 + c0;
      if (m < g.M && nb < g.N) store_row(g, m, nb, min(32, g.N - nb), v);
    }
  } else {
    // Something timed out: wait (bounded) for the loads the MMA issuer did
    // not consume and for the MMAs, so nothing is in flight when the CTA
    // frees its tensor memory and exits, then report.
    if (tid == 0) {
      for (int i = ctl[3]; i < ctl[2]; ++i)
        mbar_wait(full + 8 * (i % kStages), (i / kStages) & 1);
      atomicExch(g.error_flag, 1);
    }
    if (!waited) mbar_wait(done, 0);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN));
  }
}

// C[m][n] = sum over z (in order) of work[z][m][n].
__global__ void splitk_sum_kernel(int split, int M, int N, const float *work, float *C,
                                  int64_t ldc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t mn = (int64_t)M * N;
  if (i >= mn) return;
  float s = 0.0f;
  for (int z = 0; z < split; ++z) s += work[z * mn + i];
  const int64_t m = i / N;
  C[m * ldc + (i - m * N)] = s;
}

// cuTensorMapEncodeTiled (CUDA 12.0 ABI), found through the runtime so the
// library needs no link against the driver library.
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                 const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                 const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static const EncodeTiled fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (EncodeTiled) nullptr;
    }
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// A K-major BF16 operand of `rows` rows and K columns, row stride ld: the
// map loads boxes of kKC columns x box_rows rows with the 128-byte swizzle
// and zero fill outside the matrix.  TMA needs a 16-byte aligned base and a
// row stride that is a multiple of 16 bytes; every box starts at a K offset
// that is a multiple of kKC (128 bytes).
bool operand_map(EncodeTiled enc, CUtensorMap *map, const __nv_bfloat16 *ptr, int rows, int K,
                 int64_t ld, int box_rows) {
  if (!ptr || ((uintptr_t)ptr & 15) != 0 || (ld & 7) != 0 || ld < K) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(__nv_bfloat16)};
  const cuuint32_t box[2] = {(cuuint32_t)kKC, (cuuint32_t)box_rows};
  const cuuint32_t elem[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(ptr), dims,
             strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

}  // namespace

cudaError_t mlp_gemm_tc(const MlpGemm &p, float *work, size_t work_elems, int *error_flag,
                        cudaStream_t st) {
  if (p.M < 1 || p.N < 1 || p.K < 1 || !error_flag) return cudaErrorInvalidValue;
  const EncodeTiled enc = encoder();
  if (!enc) return cudaErrorNotSupported;
  CUtensorMap ta, tb;
  if (!operand_map(enc, &ta, p.A, p.M, p.K, p.lda, kTM) ||
      !operand_map(enc, &tb, p.B, p.N, p.K, p.ldb, kBN))
    return cudaErrorInvalidValue;
  const int tiles = ((p.M + kTM - 1) / kTM) * ((p.N + kBN - 1) / kBN);
  const int slices = (p.K + kKC - 1) / kKC;
  int split = 1;
  if (p.epi == kEpiF32 && work && tiles < kTargetCtas) {
    split = std::min(slices / kMinSlices, (kTargetCtas + tiles - 1) / tiles);
    while (split > 1 && (size_t)split * p.M * p.N > work_elems) --split;
    if (split < 1) split = 1;
  }
  const int per = ((slices + split - 1) / split) * kKC;
  split = (p.K + per - 1) / per;  // every range non-empty
  UmmaArgs g{p.M, p.N, p.K, per, p.epi, p.Cf, p.Cb, p.ldc, p.Ct, p.ldt, p.bias, p.mask,
             split > 1 ? work : nullptr, error_flag};
  cudaError_t e = cudaFuncSetAttribute(umma_gemm_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmemBytes);
  if (e != cudaSuccess) return e;
  const dim3 grid((p.M + kTM - 1) / kTM, (p.N + kBN - 1) / kBN, split);
  umma_gemm_kernel<<<grid, 128, kSmemBytes, st>>>(ta, tb, g);
  e = cudaGetLastError();
  if (e != cudaSuccess || split == 1) return e;
  const int64_t mn = (int64_t)p.M * p.N;
  splitk_sum_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, st>>>(split, p.M, p.N, work, p.Cf,
                                                                   p.ldc);
  return cudaGetLastError();
}

}  // namespace grn
