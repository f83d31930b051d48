// grn_sim_kernel.cu -- persistent batched GRN simulation + fitness kernels
// for sm_100a.
//
// Replaces the reference's simulateModelKernel
// (Src/GPUSimulator/modelsimulatordevice.cu:154-251), which runs one model
// per launch on one 1024-thread CTA with FP64 state in global memory and a
// function-pointer op interpreter.  Here:
//   - one persistent grid evaluates a whole batch; each CTA pulls the next
//     model from an atomic work counter (the host orders models by cost,
//     longest first);
//   - a model's state lives in shared memory for all Euler steps (planar
//     [gene][y][x] FP32, rows padded to float4 groups), double buffered
//     (one barrier per step); genes that do not fit use the same code on
//     double-buffered global-memory slots, and grids too large for shared
//     memory stream bands of rows through it (or split across a cluster);
//   - each thread owns float4 groups of 4 cells along x; up/down
//     neighbours come from 128-bit loads, left/right ones from 32-bit loads
//     next to the group (every padded row ends in zero cells, so a row's
//     borders read 0 without tests);
//   - regulation is evaluated in exponent form (grn_packed.h): lg2 once per
//     regulator gene and cell, one FMA + compare/select per link, and
//     ex2 + rcp once per regulated gene, on the MUFU pipe;
//   - the step's max |rate| (early-exit test) is a warp max on the float
//     bits plus one shared-memory pass; fitness sums are FP64.
// Semantics follow the reference CPU simulator
// (Src/Simulator/modelsimulator.cpp:205-280), not the reference GPU kernel:
// every cell is updated (the GPU kernel drops W*H mod 1024 cells,
// modelsimulatordevice.cu:44-47) and a zero rate keeps the current value
// (the GPU kernel's double buffer keeps a two-steps-old one, :178).

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/grn_gpu.h"
#include "grn_packed.h"
#include "grn_sim.h"

// GRN_BOUNDS_CHECK=1 builds the bounds-checked library
// (lib/libgrn_b200_checked.so): every state access is checked (see chk).
#ifndef GRN_BOUNDS_CHECK
#define GRN_BOUNDS_CHECK 0
#endif

namespace grn {
namespace {

namespace cg = cooperative_groups;

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxCluster = 16;

// ---- MUFU instructions (PTX ISA: lg2/ex2/rcp .approx.ftz.f32) ----------
__device__ __forceinline__ float lg2_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// ---- paired FP32 arithmetic (PTX ISA: add/mul/fma .rn.f32x2, sm_100+) ---
// Two lanes per instruction, each rounded exactly like its scalar
// counterpart, so results are bit-identical to fmaf / + / *.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  float2 d;
  asm("{.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  float2 d;
  asm("{.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 lo2(const float4 &v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4 &v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }

// ---- bulk copies and mbarriers (PTX ISA; streaming schedule) -----------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
// One bulk copy global -> this CTA's shared memory, completing on `bar`.
// Both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for the phase with `parity` to complete, giving up after about one
// second (a bulk copy of a band takes microseconds): false on a time-out,
// which the caller reports through the error flag instead of hanging.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 0; i < (1u << 30); ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > 1000000000ull) return false;
  }
  return false;
}
// Orders this thread's generic-proxy accesses before later async-proxy
// (bulk copy) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Shared-memory copy of one model record.
struct ModelSmem {
  PackedHeader hdr;
  PackedGene genes[GRN_MAX_GENES];
  PackedLink links[GRN_MAX_LINKS];
};
constexpr int kModelWords = sizeof(ModelSmem) / 16;
static_assert(sizeof(ModelSmem) % 16 == 0, "model smem is whole words");

// Dense form of a fast model's regulation, built in shared memory when the
// model is loaded: for gene p, the regulator slots of its OR links and of
// its AND links as bitmasks, and the (a, b) of the link from slot k at
// ab[p][k].  Hill-coefficient-0 links (constant term 0) fold into or_init
// (min with 0) and and_floor (max with 0).
struct DenseGene {
  uint32_t or_slots;
  uint32_t and_slots;
  float or_init;    // +inf, or 0 with a constant OR term
  float and_floor;  // -inf, or 0 with a constant AND term
};
struct DenseSmem {
  DenseGene gene[GRN_MAX_GENES];
  float2 ab[GRN_MAX_GENES][GRN_MAX_GENES];
};
static_assert(sizeof(DenseSmem) % 16 == 0, "dense table is whole words");

// Fixed shared-memory layout in front of the state planes.
constexpr size_t kDenseOffset = sizeof(ModelSmem);
constexpr size_t kRedOffset = kDenseOffset + sizeof(DenseSmem);  // float [2][32]
constexpr size_t kDredOffset = kRedOffset + 2 * 32 * 4;  // double [32]
constexpr size_t kWorkOffset = kDredOffset + 32 * 8;     // int [2]
// Cluster exchange slots: per-CTA step maxima float [2][kMaxCluster] (by
// step parity) and per-CTA fitness sums double [kMaxCluster].
constexpr size_t kCmaxOffset = kWorkOffset + 16;
constexpr size_t kCsumOffset = kCmaxOffset + 2 * kMaxCluster * 4;
// Two mbarriers of the streaming schedule's copy stages, then its copy
// time-out flag (int).
constexpr size_t kMbarOffset = (kCsumOffset + kMaxCluster * 8 + 15) & ~size_t(15);
constexpr size_t kStreamFailOffset = kMbarOffset + 16;
// Bounds-checked build only: the regions that state accesses are checked
// against (CheckRegions).
constexpr size_t kCheckOffset = (kStreamFailOffset + 16 + 15) & ~size_t(15);
constexpr size_t kCheckBytes = GRN_BOUNDS_CHECK ? 64 : 0;
constexpr size_t kStateOffset = (kCheckOffset + kCheckBytes + 127) & ~size_t(127);

__device__ __forceinline__ float4 f4(float v) { return make_float4(v, v, v, v); }

// ---- bounds-checked build ----------------------------------------------
//
// With GRN_BOUNDS_CHECK every state access goes through chk: the N floats
// at p must lie inside the block's shared-memory state area (from the state
// offset to the end of the dynamic shared memory) or the launch's global
// state slots, and a float4 access must be 16-byte aligned.  An access that
// is not is redirected to a scratch float4 (nothing outside the buffers is
// touched) and sets the error flag to 3, which the host reports as
// GRN_ERR_KERNEL.  Without it chk is the identity.  This stands in for a
// memory checker: the GPU tests run every schedule through the checked
// library on small grids.
struct CheckRegions {
  const float *sm_lo, *sm_hi;  // shared-memory state area
  const float *gl_lo, *gl_hi;  // global state slots of the whole launch
  int32_t *flag;
  float4 scratch;              // target of redirected accesses
};
static_assert(sizeof(CheckRegions) <= 64, "check regions fit their slot");

extern __shared__ __align__(128) unsigned char grn_dyn_smem[];

__device__ __forceinline__ bool check_span(const float *p, long n) {
  const CheckRegions &c = *reinterpret_cast<const CheckRegions *>(grn_dyn_smem + kCheckOffset);
  return (p >= c.sm_lo && p + n <= c.sm_hi) || (c.gl_lo && p >= c.gl_lo && p + n <= c.gl_hi);
}

__device__ __forceinline__ void check_failed() {
  CheckRegions &c = *reinterpret_cast<CheckRegions *>(grn_dyn_smem + kCheckOffset);
  atomicCAS(c.flag, 0, 3);
}

template <int N>
__device__ __forceinline__ float *chk(const float *p) {
#if GRN_BOUNDS_CHECK
  const bool aligned = N < 4 || (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
  if (!aligned || !check_span(p, N)) {
    check_failed();
    CheckRegions &c = *reinterpret_cast<CheckRegions *>(grn_dyn_smem + kCheckOffset);
    return reinterpret_cast<float *>(&c.scratch);
  }
#endif
  return const_cast<float *>(p);
}

// A bulk copy's source and destination spans (floats); false (and the flag)
// if either leaves its buffer, in which case the copy is not issued.
__device__ __forceinline__ bool chk_copy(const float *dst, const float *src, long n) {
#if GRN_BOUNDS_CHECK
  if (!check_span(dst, n) || !check_span(src, n)) {
    check_failed();
    return false;
  }
#endif
  (void)dst;
  (void)src;
  (void)n;
  return true;
}

// ---- regulation ------------------------------------------------------
//
// A gene's regulation is 1 / (1 + 2^V), V combined in exponent space over
// its links (grn_packed.h).  Two combine modes:
//   fast   min / max (fminf / fmaxf).  Identical to the reference whenever
//          no link term is NaN, which holds for models with finite K > 0,
//          finite Hill coefficients and 0 < K^n <= 1e300 on bounded
//          non-negative states (flag kFlagFast, which the host also clears
//          for a step size that could leave the state unbounded, and the
//          context's fast_ok for the initial states).
//   exact  the reference's comparison order (simopor.cpp:20-22,
//          simopand.cpp:20-22 with MathAlgo::max/min): a NaN term on
//          either side yields the new term; a NaN start makes the first
//          link's term the initial value ("first used link writes
//          ratios[p]", modelsimulator.cpp:156-192).

// Reference OR (Hill max) in exponent space: keep the running v only if it
// is strictly smaller.
__device__ __forceinline__ float comb_or(float run, float t) { return (run < t) ? run : t; }
// Reference AND (Hill min) in exponent space.
__device__ __forceinline__ float comb_and(float run, float t) { return (run > t) ? run : t; }

enum CombMode { kOrFast, kAndFast, kOrExact, kAndExact };

template <int MODE>
__device__ __forceinline__ float comb(float run, float t) {
  if constexpr (MODE == kOrFast) return fminf(run, t);
  else if constexpr (MODE == kAndFast) return fmaxf(run, t);
  else if constexpr (MODE == kOrExact) return comb_or(run, t);
  else return comb_and(run, t);
}

template <int MODE>
__device__ __forceinline__ void comb4(float4 &v, float a, const float4 &x, float b) {
  v.x = comb<MODE>(v.x, fmaf(a, x.x, b));
  v.y = comb<MODE>(v.y, fmaf(a, x.y, b));
  v.z = comb<MODE>(v.z, fmaf(a, x.z, b));
  v.w = comb<MODE>(v.w, fmaf(a, x.w, b));
}

// Applies one link to the running exponents of NI groups.  The regulator
// slot is the same for every thread of the block; each case carries the
// link's whole work so that the switch stays a (uniform) branch rather than
// a select chain over all registers.
template <int NI, int GMAX, int MODE>
__device__ __forceinline__ void apply_link(float4 (&v)[NI], const PackedLink &lk,
                                           const float4 (&lg)[NI][GMAX]) {
#define GRN_CASE(k)                                                   \
  case k:                                                             \
    if constexpr (GMAX > k) {                                         \
      _Pragma("unroll") for (int i = 0; i < NI; ++i)                  \
          comb4<MODE>(v[i], lk.a, lg[i][k], lk.b);                    \
    }                                                                 \
    break;
  switch (lk.slot) {
    GRN_CASE(0) GRN_CASE(1) GRN_CASE(2) GRN_CASE(3)
    GRN_CASE(4) GRN_CASE(5) GRN_CASE(6) GRN_CASE(7)
    GRN_CASE(8) GRN_CASE(9) GRN_CASE(10) GRN_CASE(11)
    GRN_CASE(12) GRN_CASE(13) GRN_CASE(14) GRN_CASE(15)
    default:  // kConstSlot: lg2 value 0, a = b = 0 (Hill coefficient 0)
#pragma unroll
      for (int i = 0; i < NI; ++i) comb4<MODE>(v[i], lk.a, f4(0.0f), lk.b);
      break;
  }
#undef GRN_CASE
}

// Regulation of one gene for NI groups.
template <int NI, int GMAX, bool EXACT>
__device__ __forceinline__ void regulation(const ModelSmem &M, const PackedGene &g,
                                           const float4 (&lg)[NI][GMAX], float4 (&h)[NI]) {
  const int n_or = g.n_or, n = g.n_or + g.n_and;
  if (n == 0) {  // OpZero
#pragma unroll
    for (int i = 0; i < NI; ++i) h[i] = f4(0.0f);
    return;
  }
  float4 v[NI];
  // exact: a NaN start makes the first term the initial value; fast: min
  // over OR terms, then max with each AND term.
  const float v0 = EXACT ? __int_as_float(0x7fc00000)
                         : (n_or > 0 ? __int_as_float(0x7f800000) : __int_as_float(0xff800000));
#pragma unroll
  for (int i = 0; i < NI; ++i) v[i] = f4(v0);
  const PackedLink *L = M.links + g.link_begin;
  int l = 0;
  for (; l < n_or; ++l) apply_link<NI, GMAX, EXACT ? kOrExact : kOrFast>(v, L[l], lg);
  for (; l < n; ++l) apply_link<NI, GMAX, EXACT ? kAndExact : kAndFast>(v, L[l], lg);
#pragma unroll
  for (int i = 0; i < NI; ++i) {
    h[i].x = rcp_approx(1.0f + ex2_approx(v[i].x));
    h[i].y = rcp_approx(1.0f + ex2_approx(v[i].y));
    h[i].z = rcp_approx(1.0f + ex2_approx(v[i].z));
    h[i].w = rcp_approx(1.0f + ex2_approx(v[i].w));
  }
}

// Regulation of gene p for NI groups from the dense table (fast models):
// regulator slots are a compile-time loop, so the lg2 values are read with
// fixed register indices and no per-link dispatch is needed.  The result is
// the fast combine's: min over OR terms, then max with each AND term (terms
// are never NaN for fast models, and min/max are order-free).
// Fast-path combine of one link into 4 running exponents: the terms
// a * lg2(x) + b for two cells per instruction, then min (OR) or max (AND).
template <bool AND>
__device__ __forceinline__ void comb4_fast(float4 &v, float2 ab, const float4 &x) {
  const float2 t01 = fma2(f2(ab.x), lo2(x), f2(ab.y));
  const float2 t23 = fma2(f2(ab.x), hi2(x), f2(ab.y));
  if (AND) {
    v.x = fmaxf(v.x, t01.x);
    v.y = fmaxf(v.y, t01.y);
    v.z = fmaxf(v.z, t23.x);
    v.w = fmaxf(v.w, t23.y);
  } else {
    v.x = fminf(v.x, t01.x);
    v.y = fminf(v.y, t01.y);
    v.z = fminf(v.z, t23.x);
    v.w = fminf(v.w, t23.y);
  }
}

template <int NI, int GMAX>
__device__ __forceinline__ void regulation_dense(const ModelSmem &M, const DenseSmem &D, int p,
                                                 const float4 (&lg)[NI][GMAX],
                                                 float4 (&h)[NI]) {
  const PackedGene &g = M.genes[p];
  if (g.n_or + g.n_and == 0) {  // OpZero
#pragma unroll
    for (int i = 0; i < NI; ++i) h[i] = f4(0.0f);
    return;
  }
  const DenseGene dg = D.gene[p];
  float4 v[NI];
#pragma unroll
  for (int i = 0; i < NI; ++i) v[i] = f4(dg.or_init);
  const uint32_t os = dg.or_slots, as = dg.and_slots;
#pragma unroll
  for (int k = 0; k < GMAX; ++k) {
    if ((os >> k) == 0u) break;
    if ((os >> k) & 1u) {
      const float2 ab = D.ab[p][k];
#pragma unroll
      for (int i = 0; i < NI; ++i) comb4_fast<false>(v[i], ab, lg[i][k]);
    }
  }
  if (g.n_or == 0) {
#pragma unroll
    for (int i = 0; i < NI; ++i) v[i] = f4(dg.and_floor);
  } else {
#pragma unroll
    for (int i = 0; i < NI; ++i) {
      v[i].x = fmaxf(v[i].x, dg.and_floor);
      v[i].y = fmaxf(v[i].y, dg.and_floor);
      v[i].z = fmaxf(v[i].z, dg.and_floor);
      v[i].w = fmaxf(v[i].w, dg.and_floor);
    }
  }
#pragma unroll
  for (int k = 0; k < GMAX; ++k) {
    if ((as >> k) == 0u) break;
    if ((as >> k) & 1u) {
      const float2 ab = D.ab[p][k];
#pragma unroll
      for (int i = 0; i < NI; ++i) comb4_fast<true>(v[i], ab, lg[i][k]);
    }
  }
#pragma unroll
  for (int i = 0; i < NI; ++i) {
    const float2 e01 = add2(f2(1.0f), make_float2(ex2_approx(v[i].x), ex2_approx(v[i].y)));
    const float2 e23 = add2(f2(1.0f), make_float2(ex2_approx(v[i].z), ex2_approx(v[i].w)));
    h[i].x = rcp_approx(e01.x);
    h[i].y = rcp_approx(e01.y);
    h[i].z = rcp_approx(e23.x);
    h[i].w = rcp_approx(e23.y);
  }
}

// Builds the dense table of a fast model (one thread per gene).
__device__ __forceinline__ void build_dense(const ModelSmem &M, DenseSmem &D, int tid) {
  const int G = M.hdr.n_genes;
  if (tid < G) {
    const PackedGene g = M.genes[tid];
    DenseGene dg;
    dg.or_slots = 0u;
    dg.and_slots = 0u;
    dg.or_init = __int_as_float(0x7f800000);
    dg.and_floor = __int_as_float(0xff800000);
    for (int l = 0; l < g.n_or + g.n_and; ++l) {
      const PackedLink lk = M.links[g.link_begin + l];
      const bool is_or = l < g.n_or;
      if (lk.slot == kConstSlot) {
        if (is_or) dg.or_init = fminf(dg.or_init, 0.0f);
        else dg.and_floor = fmaxf(dg.and_floor, 0.0f);
      } else {
        if (is_or) dg.or_slots |= 1u << lk.slot;
        else dg.and_slots |= 1u << lk.slot;
        D.ab[tid][lk.slot] = make_float2(lk.a, lk.b);
      }
    }
    D.gene[tid] = dg;
  }
}

// ---- geometry ----------------------------------------------------------
//
// A state plane holds the W x H grid as rows of RS = row_floats(W) floats
// (whole float4 groups, ending in at least one zero cell) plus one zero row
// above and one below:
// PS = (H + 2) * RS floats, row y at (y + 1) * RS.  The zero rows make the
// up/down neighbours of the first and last rows read +0.0, which leaves the
// reference's neighbour sum unchanged.  Steps write data groups only; when W
// is not a multiple of 4 the cells past W of a row's last group are written
// as 0, otherwise a zero group ends the row: either way the cell after a
// row's last cell, and the cell before the next row's first, read 0.
//
// A cluster-split launch gives each CTA of a cluster a band of rows
// [y0, y0 + H) of the Hg-row grid, held the same way: one halo row above and
// one below (the neighbouring bands' edge rows, pushed into them after every
// step, or zero at the grid border).
struct Geom {
  int W, H, Wg, RS, PS, Q;
  int y0, Hg;  // first grid row of the band, grid height
};

// One float4 group a thread owns, with everything a step needs about its
// position (computed once per launch for fixed items).
struct Item {
  int base;           // float offset of the group in a plane
  float4 tot;         // existing neighbours of each cell (reference `total`)
  bool valid;         // the group exists (an index past the end is clamped
                      // onto the last group, computed and not stored)
  bool v1, v2, v3;    // cells 1..3 of the group exist (cell 0 always does)
};

__device__ __forceinline__ Item make_item(int y, int gx, bool valid, const Geom &g) {
  Item it;
  it.valid = valid;
  it.base = (y + 1) * g.RS + 4 * gx;
  const int x0 = 4 * gx;
  const int yg = y + g.y0;
  const float tv = (yg > 0 ? 1.0f : 0.0f) + (yg < g.Hg - 1 ? 1.0f : 0.0f);
  it.tot.x = tv + (x0 > 0 ? 1.0f : 0.0f) + (x0 + 1 < g.W ? 1.0f : 0.0f);
  it.tot.y = tv + 1.0f + (x0 + 2 < g.W ? 1.0f : 0.0f);
  it.tot.z = tv + 1.0f + (x0 + 3 < g.W ? 1.0f : 0.0f);
  it.tot.w = tv + 1.0f + (x0 + 4 < g.W ? 1.0f : 0.0f);
  it.v1 = x0 + 1 < g.W;
  it.v2 = x0 + 2 < g.W;
  it.v3 = x0 + 3 < g.W;
  return it;
}

__device__ __forceinline__ Item item_at(int q, const Geom &g) {
  const bool valid = q < g.Q;
  const int qc = valid ? q : g.Q - 1;
  const int y = qc / g.Wg;
  return make_item(y, qc - y * g.Wg, valid, g);
}

__device__ __forceinline__ int cell_offset(const Geom &g, int y, int x) {
  return (y + 1) * g.RS + x;
}

// Euler update of one cell (modelsimulator.cpp:224-275).
//   r = lim*h - deg*c (+ dif*(s - tot*c) for diffusing genes)
// exact: the reference's guard on the diffusion term, "a zero rate keeps
// the value", the minConc clamp and a NaN-ignoring max.
// fast (minConc 0 and a non-negative finite state, host-checked): the guard
// only ever skips adding dif*0, a zero rate gives c + dt*0 = c, and the
// clamp is a max with 0, so these simplify without changing any result.
template <bool EXACT>
__device__ __forceinline__ float update_cell(float c, float h, float lim, float deg,
                                             float dif, bool diffuses, float s, float tot,
                                             float dt, float min_conc, float &mx) {
  float r = fmaf(-deg, c, lim * h);
  if constexpr (EXACT) {
    if (diffuses && (s > 0.0f || (tot > 0.0f && c > 0.0f))) r = fmaf(dif, fmaf(-tot, c, s), r);
    float nc = c;
    if (r != 0.0f) {  // NaN counts as non-zero, like the reference's `if (ratio)`
      nc = fmaf(dt, r, c);
      nc = (nc < min_conc) ? 0.0f : nc;
      const float ar = fabsf(r);
      mx = (ar > mx) ? ar : mx;  // a NaN rate never raises the max
    }
    return nc;
  } else {
    if (diffuses) r = fmaf(dif, fmaf(-tot, c, s), r);
    mx = fmaxf(mx, fabsf(r));
    return fmaxf(fmaf(dt, r, c), 0.0f);
  }
}

// New values of one gene for NI groups; `cur` points at the gene's current
// plane (shared or global memory).  `mx` takes the max |rate| of the valid
// groups' real cells.  HPAIR: the fast path adds the horizontal neighbours
// as FP32 pairs (else as scalar adds; the same roundings).
template <int NI, int GMAX, bool EXACT, bool RAGGED, bool HPAIR>
__device__ __forceinline__ void gene_update(const ModelSmem &M, const DenseSmem &D, int p,
                                            const PackedGene &gn,
                                            const float4 (&lg)[NI][GMAX], const float *cur,
                                            const Geom &g, const Item (&it)[NI], float dt,
                                            float min_conc, float &mx, float4 (&nv)[NI]) {
  float4 h[NI];
  if constexpr (EXACT)
    regulation<NI, GMAX, true>(M, gn, lg, h);
  else
    regulation_dense<NI, GMAX>(M, D, p, lg, h);
  const bool diffuses = gn.dif > 0.0f;  // uniform: the same gene for the whole block
  if constexpr (!EXACT) {
    // Fast path (update_cell<false>) on cell pairs: the same roundings,
    // two cells per FP32 instruction.
#pragma unroll
    for (int i = 0; i < NI; ++i) {
      const float4 c = *reinterpret_cast<const float4 *>(chk<4>(cur + it[i].base));
      float2 r01 = fma2(f2(-gn.deg), lo2(c), mul2(f2(gn.lim), lo2(h[i])));
      float2 r23 = fma2(f2(-gn.deg), hi2(c), mul2(f2(gn.lim), hi2(h[i])));
      if (diffuses) {
        const float4 up = *reinterpret_cast<const float4 *>(chk<4>(cur + it[i].base - g.RS));
        const float4 dn = *reinterpret_cast<const float4 *>(chk<4>(cur + it[i].base + g.RS));
        // Row borders read the zero cells that end every padded row.
        const float lft = *chk<1>(cur + it[i].base - 1);
        const float rgt = *chk<1>(cur + it[i].base + 4);
        // Reference order: x-1, x+1, y-1, y+1.  Scalar adds suit the step
        // with two groups per thread and the streaming step (the pairs'
        // operands straddle the float4's register pairs); paired adds the
        // steps with one group per thread (measured on the walking step).
        float2 s01, s23;
        if constexpr (!HPAIR) {
          s01 = add2(add2(make_float2(lft + c.y, c.x + c.z), lo2(up)), lo2(dn));
          s23 = add2(add2(make_float2(c.y + c.w, c.z + rgt), hi2(up)), hi2(dn));
        } else {
          s01 = add2(add2(add2(make_float2(lft, c.x), make_float2(c.y, c.z)), lo2(up)), lo2(dn));
          s23 = add2(add2(add2(make_float2(c.y, c.z), make_float2(c.w, rgt)), hi2(up)), hi2(dn));
        }
        r01 = fma2(f2(gn.dif), fma2(make_float2(-it[i].tot.x, -it[i].tot.y), lo2(c), s01), r01);
        r23 = fma2(f2(gn.dif), fma2(make_float2(-it[i].tot.z, -it[i].tot.w), hi2(c), s23), r23);
      }
      const float2 n01 = fma2(f2(dt), r01, lo2(c));
      const float2 n23 = fma2(f2(dt), r23, hi2(c));
      nv[i] = make_float4(fmaxf(n01.x, 0.0f), fmaxf(n01.y, 0.0f), fmaxf(n23.x, 0.0f),
                          fmaxf(n23.y, 0.0f));
      float m = fabsf(r01.x);
      float m1 = fabsf(r01.y), m2 = fabsf(r23.x), m3 = fabsf(r23.y);
      if constexpr (RAGGED) {
        // Cells past W are padding: kept at 0, never part of the max.
        if (!it[i].v1) { nv[i].y = 0.0f; m1 = 0.0f; }
        if (!it[i].v2) { nv[i].z = 0.0f; m2 = 0.0f; }
        if (!it[i].v3) { nv[i].w = 0.0f; m3 = 0.0f; }
      }
      if (it[i].valid) mx = fmaxf(fmaxf(mx, m), fmaxf(fmaxf(m1, m2), m3));
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < NI; ++i) {
    const float4 c = *reinterpret_cast<const float4 *>(chk<4>(cur + it[i].base));
    float4 s = f4(0.0f);
    if (diffuses) {
      const float4 up = *reinterpret_cast<const float4 *>(chk<4>(cur + it[i].base - g.RS));
      const float4 dn = *reinterpret_cast<const float4 *>(chk<4>(cur + it[i].base + g.RS));
      const float lft = *chk<1>(cur + it[i].base - 1);  // zero cells at the row borders
      const float rgt = *chk<1>(cur + it[i].base + 4);
      // Reference order: x-1, x+1, y-1, y+1.
      s.x = ((lft + c.y) + up.x) + dn.x;
      s.y = ((c.x + c.z) + up.y) + dn.y;
      s.z = ((c.y + c.w) + up.z) + dn.z;
      s.w = ((c.z + rgt) + up.w) + dn.w;
    }
    float m = 0.0f, m1 = 0.0f, m2 = 0.0f, m3 = 0.0f;
    nv[i].x = update_cell<EXACT>(c.x, h[i].x, gn.lim, gn.deg, gn.dif, diffuses, s.x,
                                 it[i].tot.x, dt, min_conc, m);
    nv[i].y = update_cell<EXACT>(c.y, h[i].y, gn.lim, gn.deg, gn.dif, diffuses, s.y,
                                 it[i].tot.y, dt, min_conc, RAGGED ? m1 : m);
    nv[i].z = update_cell<EXACT>(c.z, h[i].z, gn.lim, gn.deg, gn.dif, diffuses, s.z,
                                 it[i].tot.z, dt, min_conc, RAGGED ? m2 : m);
    nv[i].w = update_cell<EXACT>(c.w, h[i].w, gn.lim, gn.deg, gn.dif, diffuses, s.w,
                                 it[i].tot.w, dt, min_conc, RAGGED ? m3 : m);
    if constexpr (RAGGED) {
      // Cells past W are padding: kept at 0, never part of the max.
      if (!it[i].v1) { nv[i].y = 0.0f; m1 = 0.0f; }
      if (!it[i].v2) { nv[i].z = 0.0f; m2 = 0.0f; }
      if (!it[i].v3) { nv[i].w = 0.0f; m3 = 0.0f; }
      m = fmaxf(fmaxf(m, m1), fmaxf(m2, m3));
    }
    if (it[i].valid) mx = fmaxf(mx, m);
  }
}

// Block-wide max of a non-negative, non-NaN float (bit order == value
// order).  `parity` alternates two buffers so that one barrier per step
// suffices.
template <int NT>
__device__ __forceinline__ float block_max(float v, float *red, int parity, int lane,
                                           int warp) {
  const unsigned bits = __reduce_max_sync(kFull, __float_as_uint(v));
  float *r = red + parity * 32;
  if (lane == 0) r[warp] = __uint_as_float(bits);
  __syncthreads();
  // One warp value per lane, then a warp max (redux) in every warp.
  const unsigned mine = lane < NT / 32 ? __float_as_uint(r[lane]) : 0u;
  return __uint_as_float(__reduce_max_sync(kFull, mine));
}

// Block-wide FP64 sum; every thread gets the same value (fixed order).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *dred, int lane, int warp) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  if (lane == 0) dred[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < NT / 32; ++w) s += dred[w];
  return s;
}

// Where a model's state lives during one step: genes p < n_sm are double
// buffered in shared-memory planes p and p + n_sm; the others in the
// block's global slot, planes p and p + GMAX.  `par` selects the buffer
// holding the current values.
struct StatePtrs {
  float *sm;   // shared-memory planes
  float *gl;   // global-memory slot
  int n_sm;    // genes held in shared memory
};

template <int GMAX>
__device__ __forceinline__ float *plane_of(const StatePtrs &sp, const Geom &g, int p, int par) {
  return p < sp.n_sm ? sp.sm + (p + (par ? sp.n_sm : 0)) * g.PS
                     : sp.gl + (p + (par ? GMAX : 0)) * g.PS;
}

// New values of all genes of NI groups: shared-memory genes first, then
// global-memory genes (two loops so that each uses its own load path).
// GMAX is the launch's gene capacity (the global slot layout); GS >= the
// model's gene count bounds the regulator slots the step evaluates (the
// unrolled slot loops cost GS steps per gene whatever the links).
template <int NI, int GMAX, int GS, bool EXACT, bool RAGGED>
__device__ __forceinline__ void group_step(const ModelSmem &M, const DenseSmem &D,
                                           const StatePtrs &sp,
                                           const Geom &g, const Item (&it)[NI], int par,
                                           float dt, float min_conc, float &mx) {
  const int G = M.hdr.n_genes;
  const uint32_t lg_mask = M.hdr.lg_mask;
  const float *sm_cur = sp.sm + (par ? sp.n_sm : 0) * g.PS;
  float *sm_nxt = sp.sm + (par ? 0 : sp.n_sm) * g.PS;
  const float *gl_cur = sp.gl + (par ? GMAX : 0) * g.PS;
  float *gl_nxt = sp.gl + (par ? 0 : GMAX) * g.PS;
  // lg2 of the genes' current values.  The fast path takes it for every
  // gene of the model (a uniform bound, no per-slot test; its dense slot
  // masks read only the regulators) and zeroes the slots past the model's
  // genes; the exact path takes it for the regulators only (lg_mask) and
  // keeps the other slots 0 for its slot switch.
  float4 lg[NI][GS];
#pragma unroll
  for (int k = 0; k < GS; ++k) {
    if (EXACT || k >= G) {
#pragma unroll
      for (int i = 0; i < NI; ++i) lg[i][k] = f4(0.0f);
    }
    if (k < G && (!EXACT || ((lg_mask >> k) & 1u))) {
      const float *pl = (k < sp.n_sm ? sm_cur : gl_cur) + k * g.PS;
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        const float4 c = *reinterpret_cast<const float4 *>(chk<4>(pl + it[i].base));
        lg[i][k].x = lg2_approx(c.x);
        lg[i][k].y = lg2_approx(c.y);
        lg[i][k].z = lg2_approx(c.z);
        lg[i][k].w = lg2_approx(c.w);
      }
    }
  }
  for (int p = 0; p < sp.n_sm; ++p) {
    const PackedGene gn = M.genes[p];
    float4 nv[NI];
    gene_update<NI, GS, EXACT, RAGGED, (NI == 1)>(M, D, p, gn, lg, sm_cur + p * g.PS, g, it, dt,
                                                  min_conc, mx, nv);
#pragma unroll
    for (int i = 0; i < NI; ++i)
      if (it[i].valid) *reinterpret_cast<float4 *>(chk<4>(sm_nxt + p * g.PS + it[i].base)) = nv[i];
  }
  for (int p = sp.n_sm; p < G; ++p) {
    const PackedGene gn = M.genes[p];
    float4 nv[NI];
    gene_update<NI, GS, EXACT, RAGGED, (NI == 1)>(M, D, p, gn, lg, gl_cur + p * g.PS, g, it, dt,
                                                  min_conc, mx, nv);
#pragma unroll
    for (int i = 0; i < NI; ++i)
      if (it[i].valid) *reinterpret_cast<float4 *>(chk<4>(gl_nxt + p * g.PS + it[i].base)) = nv[i];
  }
}

// The fast path of one step, with the slot bound fitted to the model's gene
// count (a uniform branch per model).
template <int NI, int GMAX, bool RAGGED>
__device__ __forceinline__ void group_step_fast(const ModelSmem &M, const DenseSmem &D,
                                                const StatePtrs &sp, const Geom &g,
                                                const Item (&it)[NI], int par, float dt,
                                                float min_conc, float &mx) {
  const int G = M.hdr.n_genes;
  if (GMAX > 2 && G <= 2)
    group_step<NI, GMAX, (GMAX < 2 ? GMAX : 2), false, RAGGED>(M, D, sp, g, it, par, dt,
                                                               min_conc, mx);
  else if (GMAX > 4 && G <= 4)
    group_step<NI, GMAX, (GMAX < 4 ? GMAX : 4), false, RAGGED>(M, D, sp, g, it, par, dt,
                                                               min_conc, mx);
  else if (GMAX > 6 && G <= 6)
    group_step<NI, GMAX, (GMAX < 6 ? GMAX : 6), false, RAGGED>(M, D, sp, g, it, par, dt,
                                                               min_conc, mx);
  else
    group_step<NI, GMAX, GMAX, false, RAGGED>(M, D, sp, g, it, par, dt, min_conc, mx);
}

// ---- streaming schedule -------------------------------------------------
//
// For grids whose planes do not fit shared memory: every plane lives in the
// block's global slot and each step walks the grid in bands of R rows.  A
// band's rows plus one halo row above and below, of every gene, arrive in a
// shared-memory stage by bulk copies (the TMA engine's cp.async.bulk, one
// per gene, completing on the stage's mbarrier) while the previous band is
// computed from the other stage; new values go straight to the global slot.
// The step's arithmetic is the other schedules' (gene_update), so states
// are bit-identical.

// New values of all genes of NI groups of one band (stage planes of
// gb.PS floats), written to the global next-state planes.
// `out` addresses the band's cells as a plane does: cell (x, local row y)
// of gene p at out + p * gps + (y + 1) * RS + x.
template <int NI, int GS, bool EXACT, bool RAGGED>
__device__ __forceinline__ void band_group_step(const ModelSmem &M, const DenseSmem &D,
                                                const float *stage, int G, const Geom &gb,
                                                const Item (&it)[NI], float *out, size_t gps,
                                                float dt, float min_conc, float &mx) {
  const uint32_t lg_mask = M.hdr.lg_mask;
  float4 lg[NI][GS];
#pragma unroll
  for (int k = 0; k < GS; ++k) {
    if (EXACT || k >= G) {
#pragma unroll
      for (int i = 0; i < NI; ++i) lg[i][k] = f4(0.0f);
    }
    if (k < G && (!EXACT || ((lg_mask >> k) & 1u))) {
      const float *pl = stage + k * gb.PS;
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        const float4 c = *reinterpret_cast<const float4 *>(chk<4>(pl + it[i].base));
        lg[i][k].x = lg2_approx(c.x);
        lg[i][k].y = lg2_approx(c.y);
        lg[i][k].z = lg2_approx(c.z);
        lg[i][k].w = lg2_approx(c.w);
      }
    }
  }
  for (int p = 0; p < G; ++p) {
    float4 nv[NI];
    gene_update<NI, GS, EXACT, RAGGED, false>(M, D, p, M.genes[p], lg, stage + p * gb.PS, gb, it,
                                              dt, min_conc, mx, nv);
#pragma unroll
    for (int i = 0; i < NI; ++i)
      if (it[i].valid) *reinterpret_cast<float4 *>(chk<4>(out + p * gps + it[i].base)) = nv[i];
  }
}

template <int NI, int GMAX, bool RAGGED>
__device__ __forceinline__ void band_group_step_any(bool exact, const ModelSmem &M,
                                                    const DenseSmem &D, const float *stage, int G,
                                                    const Geom &gb, const Item (&it)[NI],
                                                    float *out, size_t gps, float dt,
                                                    float min_conc, float &mx) {
  if (exact)
    band_group_step<NI, GMAX, true, RAGGED>(M, D, stage, G, gb, it, out, gps, dt, min_conc,
                                            mx);
  else if (GMAX > 2 && G <= 2)
    band_group_step<NI, (GMAX < 2 ? GMAX : 2), false, RAGGED>(M, D, stage, G, gb, it, out,
                                                              gps, dt, min_conc, mx);
  else if (GMAX > 4 && G <= 4)
    band_group_step<NI, (GMAX < 4 ? GMAX : 4), false, RAGGED>(M, D, stage, G, gb, it, out,
                                                              gps, dt, min_conc, mx);
  else if (GMAX > 6 && G <= 6)
    band_group_step<NI, (GMAX < 6 ? GMAX : 6), false, RAGGED>(M, D, stage, G, gb, it, out,
                                                              gps, dt, min_conc, mx);
  else
    band_group_step<NI, GMAX, false, RAGGED>(M, D, stage, G, gb, it, out, gps, dt, min_conc,
                                             mx);
}

// One Euler step of the streaming schedule.  Stages alternate by band; the
// copy of band b + 2 is issued (thread 0) once every thread has finished
// band b.  mphase holds each stage's next wait parity across steps.
// Returns false (the same in every thread) if a copy did not complete in
// time; the copies still in flight have then been waited for (bounded).
// A thread whose wait runs out raises *fail and computes its band from
// whatever the stage holds; the band's one barrier then makes the decision
// block-wide (the model's results are discarded on that path).  *fail is 0
// on entry and is never cleared: the kernel returns after a failure.
template <int NT, int GMAX, bool RAGGED>
__device__ bool stream_step(const SimArgs &A, const ModelSmem &M, const DenseSmem &D,
                            const StatePtrs &sp, const Geom &g, int G, int par, bool exact,
                            float dt, float min_conc, float &mx, uint64_t *bars,
                            uint32_t &mphase, volatile int *fail, int R) {
  const int nb = (g.H + R - 1) / R;
  const int SPS = (R + 2) * g.RS;
  float *stage0 = sp.sm;
  const size_t gps = (size_t)g.PS;
  const float *gl_cur = sp.gl + (par ? GMAX : 0) * gps;
  float *gl_nxt = sp.gl + (par ? 0 : GMAX) * gps;
  auto issue = [&](int b) {
    float *st = stage0 + (b & 1) * GMAX * SPS;
    const int rows = min(R + 2, g.H + 2 - b * R);  // plane rows b*R .. b*R + rows - 1
    const uint32_t bytes = (uint32_t)rows * g.RS * 4u;
    fence_proxy_async_shared();
    mbar_expect_tx(bars + (b & 1), bytes * (uint32_t)G);
    for (int p = 0; p < G; ++p) {
      float *dst = st + p * SPS;
      const float *src = gl_cur + p * gps + (size_t)b * R * g.RS;
      if (chk_copy(dst, src, (long)rows * g.RS)) bulk_g2s(dst, src, bytes, bars + (b & 1));
    }
  };
  // Test hook: withhold band 1's copy, so that its wait runs out.
  const bool withhold = A.test_hooks & kHookWithholdBandCopy;
  if (threadIdx.x == 0) {
    issue(0);
    if (nb > 1 && !withhold) issue(1);
  }
  for (int b = 0; b < nb; ++b) {
    const int s = b & 1;
    const uint32_t parity = (mphase >> s) & 1u;
    if (!mbar_wait(bars + s, parity)) *fail = 1;
    mphase ^= 1u << s;
    Geom gb = g;
    gb.y0 = b * R;
    gb.H = min(R, g.H - b * R);
    gb.PS = SPS;
    gb.Q = gb.H * g.Wg;
    const float *st = stage0 + s * GMAX * SPS;
    const int n_it = (gb.Q + NT - 1) / NT;
    for (int i = 0; i < n_it; ++i) {  // the same count in every thread (barriers follow)
      const Item it[1] = {item_at(threadIdx.x + i * NT, gb)};
      band_group_step_any<1, GMAX, RAGGED>(exact, M, D, st, G, gb, it,
                                            gl_nxt + (size_t)gb.y0 * g.RS, gps, dt, min_conc,
                                            mx);
    }
    __syncthreads();  // stage s is free again; *fail is the same for every thread
    if (*fail) {
      // Bounded second waits for copies that may still be in flight: the
      // timed-out one (unless withheld) and the one issued ahead.
      if (!withhold) mbar_wait(bars + s, parity);
      if (b + 1 < nb) mbar_wait(bars + (s ^ 1), (mphase >> (s ^ 1)) & 1u);
      return false;
    }
    if (threadIdx.x == 0 && b + 2 < nb) issue(b + 2);
  }
  fence_proxy_async_global();  // this step's writes before the next step's copies
  return true;
}

// ---- temporal blocking: two Euler steps per pass over the state --------
//
// The streaming schedule reads and writes every plane once per step.  This
// variant (kernel ST == 2) advances the state two steps per pass.  A band
// of R output rows (grid rows [bR, bR + R)) needs the current state of
// grid rows [bR - 2, bR + R + 2): plane rows [bR - 1, bR + R + 3), clipped
// to the plane, arrive in one shared-memory stage by bulk copies.  Step one
// computes grid rows [bR - 1, bR + R] (clipped to the grid) from the stage
// into an intermediate buffer of R + 2 rows -- the band and one halo row on
// either side, which the neighbouring bands compute as well; step two
// computes the band from the intermediate and writes it to the global
// next-state planes.  The copy of band b + 1 is issued once step one of band
// b has read the stage, so it overlaps step two.  Both steps run
// band_group_step, the one-step schedules' arithmetic, so states are
// bit-identical to them.  Shared memory: G * (R + 4) stage rows and
// G * (R + 2) intermediate rows (R = A.band_rows); the same space holds the
// one-step schedule's two stages of R + 1 + 2 rows, which the kernel uses
// for a single step (an odd last step, or a first step after which the
// simulation stops).
//
// mx1 / mx2 receive the threads' max |rate| of the first / second step.
// Returns false (the same in every thread) if a copy did not complete in
// time, after a bounded wait for the copy still in flight.
template <int NT, int GMAX, bool RAGGED>
__device__ bool stream_step2(const SimArgs &A, const ModelSmem &M, const DenseSmem &D,
                             const StatePtrs &sp, const Geom &g, int G, int par, bool exact,
                             float dt, float min_conc, float &mx1, float &mx2, uint64_t *bars,
                             uint32_t &mphase, volatile int *fail) {
  const int R = A.band_rows;
  const int nb = (g.H + R - 1) / R;
  const int SPS = (R + 4) * g.RS;   // stage plane stride: plane rows bR-1 .. bR+R+2
  const int IPS = (R + 2) * g.RS;   // intermediate plane stride: grid rows bR-1 .. bR+R
  float *stage = sp.sm;
  float *inter = sp.sm + (size_t)GMAX * SPS;
  const size_t gps = (size_t)g.PS;
  const float *gl_cur = sp.gl + (par ? GMAX : 0) * gps;
  float *gl_nxt = sp.gl + (par ? 0 : GMAX) * gps;
  auto issue = [&](int b) {
    const int p0 = max(b * R - 1, 0);               // first plane row copied
    const int p1 = min(b * R + R + 3, g.H + 2);     // one past the last
    const int off = p0 - (b * R - 1);               // its stage row (1 for band 0)
    const uint32_t bytes = (uint32_t)(p1 - p0) * g.RS * 4u;
    fence_proxy_async_shared();
    mbar_expect_tx(bars, bytes * (uint32_t)G);
    for (int p = 0; p < G; ++p) {
      float *dst = stage + p * SPS + off * g.RS;
      const float *src = gl_cur + p * gps + (size_t)p0 * g.RS;
      if (chk_copy(dst, src, (long)(p1 - p0) * g.RS)) bulk_g2s(dst, src, bytes, bars);
    }
  };
  if (threadIdx.x == 0) issue(0);
  for (int b = 0; b < nb; ++b) {
    const uint32_t parity = mphase & 1u;
    if (!mbar_wait(bars, parity)) *fail = 1;
    mphase ^= 1u;
    // Step one: grid rows [y1, y1 + h1) into the intermediate.
    const int y1 = max(b * R - 1, 0);
    const int h1 = min(b * R + R, g.H - 1) - y1 + 1;
    Geom g1 = g;
    g1.y0 = y1;
    g1.H = h1;
    g1.PS = SPS;
    g1.Q = h1 * g.Wg;
    // Stage row of grid row y is y - bR + 2; g1's row 0 is grid row y1 - 1.
    const float *st1 = stage + (y1 - b * R + 1) * g.RS;
    float *out1 = inter + (y1 - b * R) * g.RS;  // cell rows land at y - (bR - 1)
    const int n1 = (g1.Q + NT - 1) / NT;
    for (int i = 0; i < n1; ++i) {
      const Item it[1] = {item_at(threadIdx.x + i * NT, g1)};
      band_group_step_any<1, GMAX, RAGGED>(exact, M, D, st1, G, g1, it, out1, (size_t)IPS, dt,
                                            min_conc, mx1);
    }
    // Intermediate rows outside the grid are the planes' zero rows.
    const int zlo = (b == 0) ? 0 : -1;                            // grid row -1
    const int zhi = (b * R + R >= g.H) ? g.H - (b * R - 1) : -1;  // grid row H
    for (int i = threadIdx.x; i < 2 * G * g.RS; i += NT) {
      const int z = i / (G * g.RS), r = i - z * G * g.RS;
      const int row = z == 0 ? zlo : zhi;
      if (row < 0) continue;
      const int p = r / g.RS, x = r - p * g.RS;
      *chk<1>(inter + p * IPS + row * g.RS + x) = 0.0f;
    }
    __syncthreads();  // the stage is free; the intermediate is complete
    if (*fail) {
      mbar_wait(bars, parity);  // bounded second wait for the copy still in flight
      return false;
    }
    if (threadIdx.x == 0 && b + 1 < nb) issue(b + 1);
    // Step two: the band's rows from the intermediate.
    Geom g2 = g;
    g2.y0 = b * R;
    g2.H = min(R, g.H - b * R);
    g2.PS = IPS;
    g2.Q = g2.H * g.Wg;
    const int n2 = (g2.Q + NT - 1) / NT;
    for (int i = 0; i < n2; ++i) {
      const Item it[1] = {item_at(threadIdx.x + i * NT, g2)};
      band_group_step_any<1, GMAX, RAGGED>(exact, M, D, inter, G, g2, it,
                                            gl_nxt + (size_t)g2.y0 * g.RS, gps, dt, min_conc,
                                            mx2);
    }
    __syncthreads();  // the intermediate is free again
  }
  fence_proxy_async_global();  // this pass's writes before the next pass's copies
  return true;
}

// Pushes the edge rows of the new buffer (`nxt`) of every gene into the
// neighbouring bands' halo rows: the first row to the band above (its row
// Hb + 1), the last row to the band below (its row 0).  Shared-memory planes
// are reached through the cluster's distributed shared memory, global slots
// directly (a cluster's CTAs are consecutive blocks).
template <int NT, int GMAX>
__device__ __forceinline__ void push_halos(const SimArgs &A, const StatePtrs &sp, const Geom &g,
                                           int G, int nxt, int rank, int C, int Hb) {
  cg::cluster_group cl = cg::this_cluster();
  const int n4 = g.RS / 4;
  for (int i = threadIdx.x; i < G * 2 * n4; i += NT) {
    const int p = i / (2 * n4), rem = i - p * 2 * n4;
    const int dir = rem / n4, c = rem - dir * n4;
    const int dst = dir == 0 ? rank - 1 : rank + 1;
    if (dst < 0 || dst >= C) continue;
    float *pl = plane_of<GMAX>(sp, g, p, nxt);
    const float4 v =
        *reinterpret_cast<const float4 *>(chk<4>(pl + (dir == 0 ? 1 : g.H) * g.RS + 4 * c));
    const int off = (dir == 0 ? Hb + 1 : 0) * g.RS + 4 * c;
    float *dpl = p < sp.n_sm
                     ? cl.map_shared_rank(chk<4>(pl + off), (unsigned)dst)  // checked locally
                     : chk<4>(A.gstate + (size_t)(blockIdx.x - rank + dst) * (size_t)A.slot_floats +
                              (pl - sp.gl) + off);
    *reinterpret_cast<float4 *>(dpl) = v;
  }
}

// Copies the first min(G, A.state_planes) genes' current values of the
// block's rows into dst ([plane][H][W], unpadded).
template <int NT, int GMAX>
__device__ __forceinline__ void write_planes(const SimArgs &A, const StatePtrs &sp, const Geom &g,
                                          int G, int par, float *dst) {
  const int planes_out = min(G, A.state_planes);
  for (int i = threadIdx.x; i < planes_out * g.W * g.H; i += NT) {
    const int kk = i / (g.W * g.H), r = i - kk * g.W * g.H;
    const int y = r / g.W, x = r - y * g.W;
    dst[((size_t)kk * g.Hg + g.y0 + y) * g.W + x] =
        *chk<1>(plane_of<GMAX>(sp, g, kk, par) + cell_offset(g, y, x));
  }
}

// Cluster-wide combine of one value per CTA: CTA `rank` stores v into slot
// `rank` of every CTA's array, then the cluster barrier (which also orders
// the halo rows pushed before it).  Every CTA then reads the same C slots.
template <typename T>
__device__ __forceinline__ void cluster_share(T *slots, T v, int rank, int C) {
  cg::cluster_group cl = cg::this_cluster();
  if ((int)threadIdx.x < C) *cl.map_shared_rank(slots + rank, threadIdx.x) = v;
  cl.sync();
}

// The simulation kernel.
//   NT      threads per block
//   GMAX    most genes (products in use) per model
//   ITEMS   float4 groups each thread owns when LOOP is false (geometry
//           computed once per launch)
//   LOOP    grids with more groups than NT * ITEMS: each thread walks its
//           groups with incrementally updated geometry
//   RAGGED  W is not a multiple of 4
//   TRACE   writes trace frames (trace_out) during the step loop; only the
//           variants compiled for it carry that code
//   ST      streaming schedule: planes in the global slot, bands of
//           A.band_rows rows staged through shared memory by bulk copies
//   CL      cluster-split: a cluster of C CTAs (launch attribute) simulates
//           one model at a time, CTA r owning rows [r*Hb, r*Hb + Hb) with
//           Hb = ceil(H / C).  Every CTA of a cluster takes the same branches
//           and passes the same cluster barriers: the model index, the step
//           max and the fitness sum are shared values, identical bits in
//           every CTA.
template <int NT, int GMAX, int ITEMS, bool LOOP, bool RAGGED, bool CL, bool TRACE, int ST>
__global__ void __launch_bounds__(NT, (NT >= 512 ? 1 : 2)) sim_kernel(const SimArgs A) {
  extern __shared__ __align__(128) unsigned char smem[];
  ModelSmem &M = *reinterpret_cast<ModelSmem *>(smem);
  DenseSmem &D = *reinterpret_cast<DenseSmem *>(smem + kDenseOffset);
  float *s_red = reinterpret_cast<float *>(smem + kRedOffset);
  double *s_dred = reinterpret_cast<double *>(smem + kDredOffset);
  int *s_work = reinterpret_cast<int *>(smem + kWorkOffset);
  float *s_cmax = reinterpret_cast<float *>(smem + kCmaxOffset);
  double *s_csum = reinterpret_cast<double *>(smem + kCsumOffset);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int rank = 0, C = 1;
  if constexpr (CL) {
    rank = (int)cg::this_cluster().block_rank();
    C = (int)cg::this_cluster().num_blocks();
  }
  const int Hb = (A.H + C - 1) / C;  // band rows (the last band may be shorter)
  Geom g;
  g.W = A.W;
  g.Hg = A.H;
  g.y0 = rank * Hb;
  g.H = min(A.H - g.y0, Hb);
  g.Wg = A.Wg;
  g.RS = row_floats(A.W);
  g.PS = (Hb + 2) * g.RS;
  g.Q = g.H * A.Wg;
  const float dt = A.dt, min_conc = A.min_conc;
  uint4 *Mw = reinterpret_cast<uint4 *>(smem);

  StatePtrs sp;
  sp.sm = reinterpret_cast<float *>(smem + kStateOffset);
  sp.gl = A.gstate ? A.gstate + (size_t)blockIdx.x * (size_t)A.slot_floats : nullptr;

#if GRN_BOUNDS_CHECK
  if (tid == 0) {
    CheckRegions &cr = *reinterpret_cast<CheckRegions *>(smem + kCheckOffset);
    uint32_t dyn = 0;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    cr.sm_lo = sp.sm;
    cr.sm_hi = reinterpret_cast<const float *>(smem + dyn);
    cr.gl_lo = A.gstate;
    cr.gl_hi = A.gstate ? A.gstate + (size_t)gridDim.x * (size_t)A.slot_floats : nullptr;
    cr.flag = A.error_flag;
  }
  __syncthreads();
#endif

  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kMbarOffset);
  volatile int *s_stream_fail = reinterpret_cast<volatile int *>(smem + kStreamFailOffset);
  uint32_t mphase = 0;  // streaming: next wait parity of each stage
  if constexpr (ST) {
    if (tid == 0) {
      mbar_init(bars, 1);
      mbar_init(bars + 1, 1);
      mbar_init_fence();
      *s_stream_fail = 0;
    }
    __syncthreads();
  }

  // Fixed items: geometry once per launch.
  Item items[LOOP ? 1 : ITEMS];
  if constexpr (!LOOP) {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) items[i] = item_at(tid + i * NT, g);
  }
  // Walking items: per-iteration stride (ITEMS * NT groups) in (row, group
  // column).
  const int dy = (ITEMS * NT) / g.Wg, dgx = ITEMS * NT - dy * g.Wg;
  const int n_iter = (g.Q + ITEMS * NT - 1) / (ITEMS * NT);
  // Items per thread of a full band: the same in every CTA of a cluster.
  const int n_iter_band = (Hb * g.Wg + NT - 1) / NT;

  for (int iter = 0;; ++iter) {
    int m;
    if constexpr (CL) {
      // Rank 0 hands the next model to every CTA of the cluster.  Two slots
      // by iteration parity: a CTA may still be reading this iteration's
      // slot when rank 0 (past the next cluster barrier at the earliest)
      // writes the following one.
      int *slot = s_work + (iter & 1);
      if (rank == 0 && tid == 0) {
        const int v = atomicAdd(A.work_counter, 1);
        for (int r = 0; r < C; ++r) *cg::this_cluster().map_shared_rank(slot, r) = v;
      }
      cg::this_cluster().sync();
      m = *slot;
    } else {
      if (tid == 0) *s_work = atomicAdd(A.work_counter, 1);
      __syncthreads();
      m = *s_work;
    }
    if (m >= A.n_models) break;
    const uint4 *rec = A.packed + A.offsets[m];
    {
      const uint4 w0 = rec[0];
      const int G0 = (int)(short)(w0.y & 0xffff);
      const int L0 = (int)(short)(w0.y >> 16);
      // Counts outside the format's limits: copy the header alone (the model
      // is rejected below) rather than read past the record.
      const bool sane = G0 >= 0 && G0 <= GRN_MAX_GENES && L0 >= 0 && L0 <= GRN_MAX_LINKS;
      const int words = sane ? 1 + G0 + L0 : 1;
      // Header and genes keep their word; links move to ModelSmem::links.
      for (int w = tid; w < words; w += NT) {
        const int dst = (w <= G0) ? w : w - 1 - G0 + 1 + GRN_MAX_GENES;
        if (dst < kModelWords) Mw[dst] = rec[w];
      }
    }
    __syncthreads();
    const int G = M.hdr.n_genes;
    const int orig = M.hdr.orig_index;
    sp.n_sm = min(G, A.planes / 2);
    const bool exact = !(A.fast_ok && (M.hdr.flags & kFlagFast) &&
                         G <= GRN_MAX_GENES);
    const bool bad = G < 1 || G > GMAX || M.hdr.n_links < 0 ||
                     M.hdr.n_links > GRN_MAX_LINKS || (sp.n_sm < G && sp.gl == nullptr) ||
                     (!LOOP && n_iter_band > ITEMS) ||
                     (ST && (A.band_rows < 1 || sp.gl == nullptr || A.planes != 0));
    if (bad) {
      if (tid == 0 && rank == 0) {
        atomicExch(A.error_flag, 1);
        A.raw_error[orig] = __longlong_as_double(0x7ff8000000000000ll);
        if (A.steps) A.steps[orig] = 0;
      }
      if constexpr (CL) cg::this_cluster().sync();
      else __syncthreads();
      continue;
    }

    if (!exact) {
      build_dense(M, D, tid);
      __syncthreads();
    }

    double error = 0.0, change_sum = 0.0;
    int steps_total = 0;
    const double max_err = A.max_error[orig];

    for (int e = 0; e < A.n_exp && error <= max_err; ++e) {
      // Initial state, both buffers of every gene: input morphogen planes
      // from the experiment, the other products 0 (simstate.cpp:64-90);
      // zero rows and padding cells 0.
      // A band's halo rows start as the neighbouring grid rows.
      const float *init = A.initial + (size_t)e * A.n_in * A.W * A.H;
      for (int i = tid; i < 2 * G * g.PS; i += NT) {
        const int kb = i / g.PS, r = i - kb * g.PS;
        const int kk = kb < G ? kb : kb - G;  // gene of this plane
        const int rr = r / g.RS, x = r - rr * g.RS;
        const int y = g.y0 - 1 + rr;  // grid row
        float v = 0.0f;
        if (kk < A.n_in && y >= 0 && y < g.Hg && x < g.W)
          v = init[((size_t)kk * g.Hg + y) * g.W + x];
        float *pl = plane_of<GMAX>(sp, g, kk, kb < G ? 0 : 1);
        *chk<1>(pl + r) = v;
      }
      if constexpr (ST == 2) {
        // The two-step pass's intermediate buffer: its rows' trailing zero
        // cells are never written by a step, so they start at 0 here (the
        // one-step pass's stage copies that may land there carry the
        // planes' zero cells in the same columns).
        float *inter = sp.sm + (size_t)GMAX * (A.band_rows + 4) * g.RS;
        for (int i = tid; i < GMAX * (A.band_rows + 2) * g.RS; i += NT) *chk<1>(inter + i) = 0.0f;
      }
      if constexpr (ST) fence_proxy_async_global();  // before the first bulk copies
      if constexpr (CL) cg::this_cluster().sync();
      else __syncthreads();

      // Trace frames: the state after every trace_every-th step, frame 0
      // the initial state.  A frame reads the current buffer while the
      // next step writes the other one.
      float *trace = nullptr;
      if constexpr (TRACE) {
        trace = A.trace_out + ((size_t)orig * A.n_exp + e) * A.trace_frames * A.state_planes *
                                  g.W * g.Hg;
        write_planes<NT, GMAX>(A, sp, g, G, 0, trace);
      }

      double change = 1.0;
      int step = 0;
      int par = 0;  // buffer holding the current values
      while (step < A.n_steps && change > A.min_conc_change) {
        float mx = 0.0f;
        int adv = 1;  // Euler steps this iteration advanced
        if constexpr (ST == 2) {
          // Two steps per pass while two remain.  If the first step's change
          // already ends the simulation, that step is run alone again (the
          // one-step pass, R + 1 rows per band in the same shared memory),
          // so the state is the one after exactly one step.
          bool ok;
          if (step + 2 <= A.n_steps) {
            float mx2 = 0.0f;
            ok = stream_step2<NT, GMAX, RAGGED>(A, M, D, sp, g, G, par, exact, dt, min_conc, mx,
                                                mx2, bars, mphase, s_stream_fail);
            if (ok) {
              const float b1 = block_max<NT>(mx, s_red, par ^ 1, lane, warp);
              if ((double)b1 > A.min_conc_change) {
                mx = mx2;
                adv = 2;
              } else {
                mx = 0.0f;
                ok = stream_step<NT, GMAX, RAGGED>(A, M, D, sp, g, G, par, exact, dt, min_conc,
                                                   mx, bars, mphase, s_stream_fail,
                                                   A.band_rows + 1);
              }
            }
          } else {
            ok = stream_step<NT, GMAX, RAGGED>(A, M, D, sp, g, G, par, exact, dt, min_conc, mx,
                                               bars, mphase, s_stream_fail, A.band_rows + 1);
          }
          if (!ok) {
            if (tid == 0) {
              atomicExch(A.error_flag, 2);
              A.raw_error[orig] = __longlong_as_double(0x7ff8000000000000ll);
            }
            return;  // every thread of the block: the decision is block-uniform
          }
        } else if constexpr (ST) {
          if (!stream_step<NT, GMAX, RAGGED>(A, M, D, sp, g, G, par, exact, dt, min_conc, mx,
                                              bars, mphase, s_stream_fail, A.band_rows)) {
            if (tid == 0) {
              atomicExch(A.error_flag, 2);
              A.raw_error[orig] = __longlong_as_double(0x7ff8000000000000ll);
            }
            return;  // every thread of the block: the decision is block-uniform
          }
        } else if constexpr (!LOOP) {
          // All ITEMS groups of the thread at once (items past the grid are
          // clamped duplicates and store nothing).
          if (exact)
            group_step<ITEMS, GMAX, GMAX, true, RAGGED>(M, D, sp, g, items, par, dt, min_conc,
                                                        mx);
          else
            group_step_fast<ITEMS, GMAX, RAGGED>(M, D, sp, g, items, par, dt, min_conc, mx);
        } else {
          // ITEMS groups per iteration (more loads in flight), each
          // advanced by ITEMS * NT groups.
          int y[ITEMS], gx[ITEMS];
#pragma unroll
          for (int j = 0; j < ITEMS; ++j) {
            y[j] = (tid + j * NT) / g.Wg;
            gx[j] = (tid + j * NT) - y[j] * g.Wg;
          }
          for (int i = 0; i < n_iter; ++i) {
            Item it[ITEMS];
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
              const int q = tid + (i * ITEMS + j) * NT;
              it[j] = q < g.Q ? make_item(y[j], gx[j], true, g) : item_at(q, g);
            }
            if (exact)
              group_step<ITEMS, GMAX, GMAX, true, RAGGED>(M, D, sp, g, it, par, dt, min_conc,
                                                          mx);
            else
              group_step_fast<ITEMS, GMAX, RAGGED>(M, D, sp, g, it, par, dt, min_conc, mx);
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
              y[j] += dy;
              gx[j] += dgx;
              if (gx[j] >= g.Wg) {
                gx[j] -= g.Wg;
                ++y[j];
              }
            }
          }
        }
        float bm = block_max<NT>(mx, s_red, par, lane, warp);
        if constexpr (CL) {
          push_halos<NT, GMAX>(A, sp, g, G, par ^ 1, rank, C, Hb);
          cluster_share(s_cmax + par * kMaxCluster, bm, rank, C);
          bm = 0.0f;
          for (int r = 0; r < C; ++r) bm = fmaxf(bm, s_cmax[par * kMaxCluster + r]);
        }
        change = (double)bm;
        par ^= 1;
        step += adv;
        if constexpr (TRACE) {
          if (step % A.trace_every == 0 && step / A.trace_every < A.trace_frames)
            write_planes<NT, GMAX>(A, sp, g, G, par,
                                   trace + (size_t)(step / A.trace_every) * A.state_planes *
                                               g.W * g.Hg);
        }
      }
      steps_total += step;
      change_sum += change;
      if (A.state_out)  // final state of this experiment, unpadded [gene][y][x]
        write_planes<NT, GMAX>(A, sp, g, G, par,
                               A.state_out + ((size_t)orig * A.n_exp + e) * A.state_planes *
                                                 g.W * g.Hg);

      // Fitness of the experiment (simstate.cpp:135-158), FP64 sums.
      const float *tgt = A.target + (size_t)e * A.n_target * A.W * A.H;
      double acc = 0.0;
      for (int i = tid; i < g.W * g.H; i += NT) {
        const int y = i / g.W, x = i - y * g.W;
        for (int kk = 0; kk < A.n_target; ++kk) {
          const double a = *chk<1>(plane_of<GMAX>(sp, g, A.n_in + kk, par) + cell_offset(g, y, x));
          const double b = tgt[((size_t)kk * g.Hg + g.y0 + y) * g.W + x];
          if (A.fitness_kind == GRN_FITNESS_MSE) {
            acc += (a - b) * (a - b);
          } else {
            const double sub = fabs(a - b) - A.dist_threshold;
            if (sub > 0) acc += log(1.0 + sub);
          }
        }
      }
      double dist = block_sum<NT>(acc, s_dred, lane, warp);
      if constexpr (CL) {
        cluster_share(s_csum, dist, rank, C);
        dist = 0.0;
        for (int r = 0; r < C; ++r) dist += s_csum[r];
      }
      if (A.fitness_kind == GRN_FITNESS_MSE)
        dist /= (double)g.W * g.Hg * A.n_target;
      else
        dist /= (double)(g.W * g.Hg);
      // Non-convergence penalty on the running change sum
      // (evaluatormorphogens.cpp:62-65).
      if (change_sum > A.min_conc_change) dist += change_sum - A.min_conc_change;
      error += dist / A.n_exp;
    }
    if (tid == 0 && rank == 0) {
      A.raw_error[orig] = error;
      if (A.steps) A.steps[orig] = steps_total;
    }
    __syncthreads();
  }
}

// ---- variant table -----------------------------------------------------

typedef void (*KernelFn)(const SimArgs);

struct VariantEntry {
  KernelVariant v;
  KernelFn fn;
};

#define GRN_VARIANT_X(NT, GMAX, ITEMS, LOOP, CL, TR, ST)                                   \
  {{NT, GMAX, ITEMS, LOOP, false, CL, TR, ST},                                            \
   &sim_kernel<NT, GMAX, ITEMS, LOOP, false, CL, TR, ST>},                                \
  {{NT, GMAX, ITEMS, LOOP, true, CL, TR, ST}, &sim_kernel<NT, GMAX, ITEMS, LOOP, true, CL, TR, ST>}
#define GRN_VARIANT_T(NT, GMAX, ITEMS, LOOP, CL, TR) \
  GRN_VARIANT_X(NT, GMAX, ITEMS, LOOP, CL, TR, 0)
#define GRN_VARIANT(NT, GMAX, ITEMS, LOOP, CL) GRN_VARIANT_T(NT, GMAX, ITEMS, LOOP, CL, false)

const VariantEntry kVariants[] = {
    GRN_VARIANT(256, 4, 1, false, false),  GRN_VARIANT(256, 8, 1, false, false),
    GRN_VARIANT(256, 16, 1, false, false), GRN_VARIANT(512, 4, 2, false, false),
    GRN_VARIANT(512, 8, 2, false, false),
    GRN_VARIANT(512, 8, 1, true, false),   GRN_VARIANT(512, 16, 1, true, false),
    GRN_VARIANT(256, 4, 1, true, false),
    // cluster-split
    GRN_VARIANT(512, 8, 1, false, true),
    GRN_VARIANT(512, 8, 1, true, true),    GRN_VARIANT(512, 16, 1, true, true),
    // trace frames (one model at a time: any grid, any gene count)
    GRN_VARIANT_T(256, 16, 1, true, false, true),
    // streaming (bands staged by bulk copies)
    GRN_VARIANT_X(512, 8, 1, true, false, false, 1),
    GRN_VARIANT_X(512, 16, 1, true, false, false, 1),
    // streaming with temporal blocking: two Euler steps per pass
    GRN_VARIANT_X(512, 8, 1, true, false, false, 2),
    GRN_VARIANT_X(512, 16, 1, true, false, false, 2),
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

const VariantEntry *find_variant(const KernelVariant &v) {
  for (int i = 0; i < kNumVariants; ++i) {
    const KernelVariant &k = kVariants[i].v;
    if (k.threads == v.threads && k.gmax == v.gmax && k.items == v.items &&
        k.loop == v.loop && k.ragged == v.ragged && k.cluster == v.cluster &&
        k.trace == v.trace && k.stream == v.stream)
      return &kVariants[i];
  }
  return nullptr;
}

}  // namespace

size_t sim_fixed_smem_bytes() { return kStateOffset; }

int sim_variant_count() { return kNumVariants; }

KernelVariant sim_variant(int i) { return kVariants[i].v; }

cudaError_t sim_occupancy(const KernelVariant &v, size_t smem_bytes, int *blocks_per_sm) {
  const VariantEntry *e = find_variant(v);
  if (!e) return cudaErrorInvalidValue;
  cudaError_t err =
      cudaFuncSetAttribute(e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (err != cudaSuccess) {
    *blocks_per_sm = 0;
    cudaGetLastError();
    return cudaSuccess;
  }
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, e->fn, v.threads,
                                                       smem_bytes);
}

cudaError_t sim_cluster_occupancy(const KernelVariant &v, size_t smem_bytes, int cluster,
                                  int *clusters) {
  *clusters = 0;
  const VariantEntry *e = find_variant(v);
  if (!e || !v.cluster || cluster < 2 || cluster > kMaxCluster) return cudaErrorInvalidValue;
  if (cudaFuncSetAttribute(e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) !=
          cudaSuccess ||
      cudaFuncSetAttribute(e->fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
          cudaSuccess) {
    cudaGetLastError();
    return cudaSuccess;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster, 1, 1);
  cfg.blockDim = dim3(v.threads, 1, 1);
  cfg.dynamicSmemBytes = smem_bytes;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaOccupancyMaxActiveClusters(clusters, e->fn, &cfg) != cudaSuccess) {
    *clusters = 0;
    cudaGetLastError();
  }
  return cudaSuccess;
}

cudaError_t sim_launch(const LaunchPlan &plan, const SimArgs &args, cudaStream_t stream) {
  const VariantEntry *e = find_variant(plan.v);
  if (!e) return cudaErrorInvalidValue;
  if (plan.v.cluster != (plan.cluster > 1)) return cudaErrorInvalidValue;
  cudaError_t err = cudaFuncSetAttribute(e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)plan.smem_bytes);
  if (err != cudaSuccess) return err;
  if (plan.cluster > 1) {
    // Whole clusters only, each band non-empty.
    const int hb = (args.H + plan.cluster - 1) / plan.cluster;
    if (plan.cluster > kMaxCluster || plan.blocks % plan.cluster != 0 ||
        (plan.cluster - 1) * hb >= args.H)
      return cudaErrorInvalidValue;
    err = cudaFuncSetAttribute(e->fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (err != cudaSuccess) return err;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(plan.blocks, 1, 1);
    cfg.blockDim = dim3(plan.v.threads, 1, 1);
    cfg.dynamicSmemBytes = plan.smem_bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = plan.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, e->fn, args);
  }
  e->fn<<<plan.blocks, plan.v.threads, plan.smem_bytes, stream>>>(args);
  return cudaGetLastError();
}

}  // namespace grn
