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
//     [gene][y][x] FP32, rows padded to float4 groups), either double
//     buffered (one barrier per step) or single buffered with the new values
//     held in registers (two barriers per step); grids too large for shared
//     memory use the same code on double-buffered global-memory slots;
//   - each thread owns float4 groups of 4 cells along x; left/right
//     neighbours come from warp shuffles (lanes hold consecutive groups),
//     up/down neighbours from 128-bit loads;
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

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/grn_gpu.h"
#include "grn_packed.h"
#include "grn_sim.h"

namespace grn {
namespace {

constexpr unsigned kFull = 0xffffffffu;

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

// Shared-memory copy of one model record.
struct ModelSmem {
  PackedHeader hdr;
  PackedGene genes[GRN_MAX_GENES];
  PackedLink links[GRN_MAX_LINKS];
};
constexpr int kModelWords = sizeof(ModelSmem) / 16;
static_assert(sizeof(ModelSmem) % 16 == 0, "model smem is whole words");

// Fixed shared-memory layout in front of the state planes.
constexpr size_t kRedOffset = sizeof(ModelSmem);         // float [2][32]
constexpr size_t kDredOffset = kRedOffset + 2 * 32 * 4;  // double [32]
constexpr size_t kWorkOffset = kDredOffset + 32 * 8;     // int
constexpr size_t kStateOffset = (kWorkOffset + 16 + 127) & ~size_t(127);

__device__ __forceinline__ float4 f4(float v) { return make_float4(v, v, v, v); }

// Regulator lg2 values of one float4 group for a runtime slot.  The slot is
// the same for every thread of the block, so the switch is a uniform branch.
template <int GMAX>
__device__ __forceinline__ float4 pick_slot(const float4 (&lg)[GMAX], int slot) {
#define GRN_CASE(k)                       \
  case k:                                 \
    if constexpr (GMAX > k) return lg[k]; \
    break;
  switch (slot) {
    GRN_CASE(0) GRN_CASE(1) GRN_CASE(2) GRN_CASE(3)
    GRN_CASE(4) GRN_CASE(5) GRN_CASE(6) GRN_CASE(7)
    GRN_CASE(8) GRN_CASE(9) GRN_CASE(10) GRN_CASE(11)
    GRN_CASE(12) GRN_CASE(13) GRN_CASE(14) GRN_CASE(15)
    default: break;
  }
#undef GRN_CASE
  return f4(0.0f);  // kConstSlot: lg2 value 0 (Hill coefficient 0)
}

// Reference OR (Hill max, simopor.cpp:20-22 with MathAlgo::max) in exponent
// space: keep the running v only if it is strictly smaller; a NaN on either
// side yields the new term, as the reference's comparison does.
__device__ __forceinline__ float comb_or(float run, float t) { return (run < t) ? run : t; }
// Reference AND (Hill min, simopand.cpp:20-22 with MathAlgo::min).
__device__ __forceinline__ float comb_and(float run, float t) { return (run > t) ? run : t; }

// Regulation value of gene p for one float4 group: the result of the
// reference's op list for the product (modelsimulator.cpp:156-192).
template <int GMAX>
__device__ __forceinline__ float4 regulation(const ModelSmem &M, int p,
                                             const float4 (&lg)[GMAX]) {
  const PackedGene &g = M.genes[p];
  const int n_or = g.n_or, n_and = g.n_and;
  if (n_or + n_and == 0) return f4(0.0f);  // OpZero
  const float qnan = __int_as_float(0x7fc00000);
  // A NaN start makes the first link's term the initial value, which is the
  // reference's "first used link writes ratios[p]".
  float4 v = f4(qnan);
  const PackedLink *L = M.links + g.link_begin;
  for (int l = 0; l < n_or; ++l) {
    const PackedLink lk = L[l];
    const float4 x = pick_slot<GMAX>(lg, lk.slot);
    v.x = comb_or(v.x, fmaf(lk.a, x.x, lk.b));
    v.y = comb_or(v.y, fmaf(lk.a, x.y, lk.b));
    v.z = comb_or(v.z, fmaf(lk.a, x.z, lk.b));
    v.w = comb_or(v.w, fmaf(lk.a, x.w, lk.b));
  }
  for (int l = n_or; l < n_or + n_and; ++l) {
    const PackedLink lk = L[l];
    const float4 x = pick_slot<GMAX>(lg, lk.slot);
    v.x = comb_and(v.x, fmaf(lk.a, x.x, lk.b));
    v.y = comb_and(v.y, fmaf(lk.a, x.y, lk.b));
    v.z = comb_and(v.z, fmaf(lk.a, x.z, lk.b));
    v.w = comb_and(v.w, fmaf(lk.a, x.w, lk.b));
  }
  float4 h;
  h.x = rcp_approx(1.0f + ex2_approx(v.x));
  h.y = rcp_approx(1.0f + ex2_approx(v.y));
  h.z = rcp_approx(1.0f + ex2_approx(v.z));
  h.w = rcp_approx(1.0f + ex2_approx(v.w));
  return h;
}

// Rate, diffusion and Euler update of one cell
// (modelsimulator.cpp:224-275).  A missing neighbour is passed as +0.0,
// which leaves the reference's running sum unchanged.
__device__ __forceinline__ float update_cell(float c, float h, float lim,
                                             float deg, float dif, float left,
                                             float right, float up, float down,
                                             float tot, float dt,
                                             float min_conc, bool valid,
                                             float &mx) {
  float r = fmaf(lim, h, -deg * c);
  if (dif > 0.0f) {
    const float s = ((left + right) + up) + down;
    if (s > 0.0f || (tot > 0.0f && c > 0.0f)) r = fmaf(dif, fmaf(-tot, c, s), r);
  }
  float nc = c;
  if (r != 0.0f) {  // NaN counts as non-zero, like the reference's `if (ratio)`
    nc = fmaf(dt, r, c);
    nc = (nc < min_conc) ? 0.0f : nc;
    const float ar = fabsf(r);
    if (valid) mx = (ar > mx) ? ar : mx;  // a NaN rate never raises the max
  }
  return valid ? nc : 0.0f;
}

// Geometry of the state: W x H cells, rows padded to Wp = 4 * Wg floats,
// planes of P = H * Wp floats, Q = H * Wg float4 groups per plane.
struct Geom {
  int W, H, Wg, Wp, P, Q;
};

struct GroupPos {
  int q;       // group index, clamped into [0, Q)
  int y, x0;   // row and first column
  bool valid;  // the group exists (q < Q before clamping)
};

__device__ __forceinline__ GroupPos group_pos(int q, const Geom &g) {
  GroupPos p;
  p.valid = q < g.Q;
  p.q = p.valid ? q : g.Q - 1;
  p.y = p.q / g.Wg;
  p.x0 = (p.q - p.y * g.Wg) * 4;
  return p;
}

// Cell-position facts of one float4 group shared by all its genes.
struct GroupCells {
  bool v0, v1, v2, v3;       // cell exists (x < W and group valid)
  bool has_up, has_dn;       // neighbour rows exist
  bool has_l, has_r;         // neighbour groups exist in the row
  bool r0, r1, r2;           // right neighbour of cells 0..2 exists
  float t0, t1, t2, t3;      // number of existing neighbours per cell
};

__device__ __forceinline__ GroupCells group_cells(const GroupPos &gp, const Geom &g) {
  GroupCells c;
  const int W = g.W;
  c.v0 = gp.valid && gp.x0 + 0 < W;
  c.v1 = gp.valid && gp.x0 + 1 < W;
  c.v2 = gp.valid && gp.x0 + 2 < W;
  c.v3 = gp.valid && gp.x0 + 3 < W;
  c.has_up = gp.y > 0;
  c.has_dn = gp.y < g.H - 1;
  c.has_l = gp.x0 > 0;
  c.has_r = gp.x0 + 4 < W;
  c.r0 = gp.x0 + 1 < W;
  c.r1 = gp.x0 + 2 < W;
  c.r2 = gp.x0 + 3 < W;
  const float tv = (c.has_up ? 1.0f : 0.0f) + (c.has_dn ? 1.0f : 0.0f);
  c.t0 = tv + (c.has_l ? 1.0f : 0.0f) + (c.r0 ? 1.0f : 0.0f);
  c.t1 = tv + 1.0f + (c.r1 ? 1.0f : 0.0f);
  c.t2 = tv + 1.0f + (c.r2 ? 1.0f : 0.0f);
  c.t3 = tv + 1.0f + (c.has_r ? 1.0f : 0.0f);
  return c;
}

// lg2 of the current value of every regulator gene of one group.
template <int GMAX>
__device__ __forceinline__ void group_lg(const ModelSmem &M, const float *st,
                                         int plane_shift_planes, int n_dbuf,
                                         const Geom &g, int base,
                                         float4 (&lg)[GMAX]) {
  const int G = M.hdr.n_genes;
  const uint32_t lg_mask = M.hdr.lg_mask;
#pragma unroll
  for (int k = 0; k < GMAX; ++k) {
    lg[k] = f4(0.0f);
    if (k < G && ((lg_mask >> k) & 1u)) {
      const int plane = (k < n_dbuf) ? k + plane_shift_planes : k;
      const float4 c = *reinterpret_cast<const float4 *>(st + plane * g.P + base);
      lg[k].x = lg2_approx(c.x);
      lg[k].y = lg2_approx(c.y);
      lg[k].z = lg2_approx(c.z);
      lg[k].w = lg2_approx(c.w);
    }
  }
}

// New value of gene p for one float4 group whose current plane is `pl`.
// All lanes of a warp call this together (it shuffles).  Updates mx with the
// max |rate| over valid cells.
template <int GMAX>
__device__ __forceinline__ float4 gene_update(const ModelSmem &M, int p,
                                              const float4 (&lg)[GMAX],
                                              const float *pl, const Geom &g,
                                              const GroupPos &gp,
                                              const GroupCells &cc, int lane,
                                              float dt, float min_conc,
                                              float &mx) {
  const float4 h = regulation<GMAX>(M, p, lg);
  const PackedGene &gn = M.genes[p];
  const float lim = gn.lim, deg = gn.deg, dif = gn.dif;
  const int base = gp.q * 4;
  const float4 c = *reinterpret_cast<const float4 *>(pl + base);
  float4 up = f4(0.0f), dn = f4(0.0f);
  float lft = 0.0f, rgt = 0.0f;
  if (dif > 0.0f) {  // uniform: the same gene for the whole block
    if (cc.has_up) up = *reinterpret_cast<const float4 *>(pl + base - g.Wp);
    if (cc.has_dn) dn = *reinterpret_cast<const float4 *>(pl + base + g.Wp);
    lft = __shfl_up_sync(kFull, c.w, 1);
    rgt = __shfl_down_sync(kFull, c.x, 1);
    // Lanes 0 and 31 have no in-warp neighbour group.
    if (lane == 0 && cc.has_l) lft = pl[base - 1];
    if (lane == 31 && cc.has_r) rgt = pl[base + 4];
    if (!cc.has_l) lft = 0.0f;
    if (!cc.has_r) rgt = 0.0f;
  }
  float4 nv;
  nv.x = update_cell(c.x, h.x, lim, deg, dif, lft, cc.r0 ? c.y : 0.0f, up.x,
                     dn.x, cc.t0, dt, min_conc, cc.v0, mx);
  nv.y = update_cell(c.y, h.y, lim, deg, dif, c.x, cc.r1 ? c.z : 0.0f, up.y,
                     dn.y, cc.t1, dt, min_conc, cc.v1, mx);
  nv.z = update_cell(c.z, h.z, lim, deg, dif, c.y, cc.r2 ? c.w : 0.0f, up.z,
                     dn.z, cc.t2, dt, min_conc, cc.v2, mx);
  nv.w = update_cell(c.w, h.w, lim, deg, dif, c.z, rgt, up.w, dn.w, cc.t3, dt,
                     min_conc, cc.v3, mx);
  return nv;
}

// Block-wide max of a non-negative, non-NaN float (bit order == value
// order).  `parity` alternates two buffers so that one barrier per step
// suffices.
template <int NT>
__device__ __forceinline__ float block_max(float v, float *red, int parity,
                                           int lane, int warp) {
  const unsigned bits = __reduce_max_sync(kFull, __float_as_uint(v));
  float *r = red + parity * 32;
  if (lane == 0) r[warp] = __uint_as_float(bits);
  __syncthreads();
  float m = r[0];
#pragma unroll
  for (int w = 1; w < NT / 32; ++w) m = fmaxf(m, r[w]);
  return m;
}

// Block-wide FP64 sum; every thread gets the same value (fixed order).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *dred, int lane,
                                            int warp) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  if (lane == 0) dred[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < NT / 32; ++w) s += dred[w];
  return s;
}

// The simulation kernel.
//   NT     threads per block
//   GMAX   most genes (products in use) per model
//   ITEMS  float4 groups per thread when genes are held in registers
//   NREG   most genes whose new values are held in registers across the
//          barrier (the others are double buffered in spare planes)
//   GSTATE state in global-memory slots instead of shared memory
//
// State planes: genes 0..G-1 start in planes 0..G-1.  With S = planes - G
// spare planes, genes p < min(S, G) are double buffered: their current
// plane is p on even steps and G + p on odd steps.  Genes p >= S keep plane
// p and their new values wait in registers until all reads are done.
template <int NT, int GMAX, int ITEMS, int NREG, bool GSTATE>
__global__ void __launch_bounds__(NT, (NT >= 512 ? 1 : 2))
    sim_kernel(const SimArgs A) {
  extern __shared__ __align__(128) unsigned char smem[];
  ModelSmem &M = *reinterpret_cast<ModelSmem *>(smem);
  float *s_red = reinterpret_cast<float *>(smem + kRedOffset);
  double *s_dred = reinterpret_cast<double *>(smem + kDredOffset);
  int *s_work = reinterpret_cast<int *>(smem + kWorkOffset);
  float *state;
  if constexpr (GSTATE)
    state = A.gstate + (size_t)blockIdx.x * (size_t)A.slot_floats;
  else
    state = reinterpret_cast<float *>(smem + kStateOffset);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  Geom g;
  g.W = A.W;
  g.H = A.H;
  g.Wg = A.Wg;
  g.Wp = A.Wg * 4;
  g.P = A.H * g.Wp;
  g.Q = A.H * A.Wg;
  const int n_iter = (g.Q + NT - 1) / NT;  // same for every thread
  const float dt = A.dt, min_conc = A.min_conc;
  uint4 *Mw = reinterpret_cast<uint4 *>(smem);

  for (;;) {
    if (tid == 0) *s_work = atomicAdd(A.work_counter, 1);
    __syncthreads();
    const int m = *s_work;
    if (m >= A.n_models) break;
    const uint4 *rec = A.packed + A.offsets[m];
    {
      const uint4 w0 = rec[0];
      const int G0 = (int)(short)(w0.y & 0xffff);
      const int L0 = (int)(short)(w0.y >> 16);
      const int words = 1 + G0 + L0;
      // Header and genes keep their word; links move to ModelSmem::links.
      for (int w = tid; w < words; w += NT) {
        const int dst = (w <= G0) ? w : w - 1 - G0 + 1 + GRN_MAX_GENES;
        if (dst < kModelWords) Mw[dst] = rec[w];
      }
    }
    __syncthreads();
    const int G = M.hdr.n_genes;
    const int orig = M.hdr.orig_index;
    const int S = GSTATE ? G : max(0, A.planes - G);  // spare planes
    const int n_dbuf = min(S, G);                       // double-buffered genes
    const int n_reg = G - n_dbuf;                       // register-held genes
    bool bad = G < 1 || G > GMAX || M.hdr.n_links < 0 ||
               M.hdr.n_links > GRN_MAX_LINKS || n_reg > NREG ||
               (n_reg > 0 && n_iter > ITEMS) || (!GSTATE && G > A.planes);
    if (bad) {
      if (tid == 0) {
        atomicExch(A.error_flag, 1);
        A.raw_error[orig] = __longlong_as_double(0x7ff8000000000000ll);
        if (A.steps) A.steps[orig] = 0;
      }
      __syncthreads();
      continue;
    }

    double error = 0.0, change_sum = 0.0;
    int steps_total = 0;
    const double max_err = A.max_error[orig];

    for (int e = 0; e < A.n_exp && error <= max_err; ++e) {
      // Initial state: input morphogen planes from the experiment, the
      // other products 0 (simstate.cpp:64-90).  Padding cells are 0.
      const float *init = A.initial + (size_t)e * A.n_in * A.W * A.H;
      for (int i = tid; i < G * g.P; i += NT) {
        const int k = i / g.P, r = i - k * g.P;
        const int y = r / g.Wp, x = r - y * g.Wp;
        float v = 0.0f;
        if (k < A.n_in && x < g.W) v = init[((size_t)k * g.H + y) * g.W + x];
        state[i] = v;
      }
      __syncthreads();

      double change = 1.0;
      int step = 0;
      int parity = 0;  // double-buffered genes live in planes G.. on odd steps
      while (step < A.n_steps && change > A.min_conc_change) {
        const int cur_shift = parity ? G : 0;   // plane offset of current values
        const int nxt_shift = parity ? 0 : G;   // plane offset of next values
        float mx = 0.0f;
        if constexpr (NREG == 0) {
          for (int it = 0; it < n_iter; ++it) {
            const GroupPos gp = group_pos(tid + it * NT, g);
            const GroupCells cc = group_cells(gp, g);
            float4 lg[GMAX];
            group_lg<GMAX>(M, state, cur_shift, n_dbuf, g, gp.q * 4, lg);
            for (int p = 0; p < G; ++p) {
              const float4 nv = gene_update<GMAX>(M, p, lg, state + (p + cur_shift) * g.P,
                                                  g, gp, cc, lane, dt, min_conc, mx);
              if (gp.valid)
                *reinterpret_cast<float4 *>(state + (p + nxt_shift) * g.P + gp.q * 4) = nv;
            }
          }
          change = (double)block_max<NT>(mx, s_red, parity, lane, warp);
        } else {
          float4 nreg[ITEMS][NREG];
#pragma unroll
          for (int it = 0; it < ITEMS; ++it) {
            if (it < n_iter) {
              const GroupPos gp = group_pos(tid + it * NT, g);
              const GroupCells cc = group_cells(gp, g);
              float4 lg[GMAX];
              group_lg<GMAX>(M, state, cur_shift, n_dbuf, g, gp.q * 4, lg);
              for (int p = 0; p < n_dbuf; ++p) {
                const float4 nv = gene_update<GMAX>(M, p, lg, state + (p + cur_shift) * g.P,
                                                    g, gp, cc, lane, dt, min_conc, mx);
                if (gp.valid)
                  *reinterpret_cast<float4 *>(state + (p + nxt_shift) * g.P + gp.q * 4) = nv;
              }
#pragma unroll
              for (int r = 0; r < NREG; ++r) {
                const int p = n_dbuf + r;
                if (r < n_reg)
                  nreg[it][r] = gene_update<GMAX>(M, p, lg, state + p * g.P, g, gp, cc,
                                                  lane, dt, min_conc, mx);
              }
            }
          }
          change = (double)block_max<NT>(mx, s_red, parity, lane, warp);
          if (n_reg > 0) {
#pragma unroll
            for (int it = 0; it < ITEMS; ++it) {
              if (it < n_iter) {
                const GroupPos gp = group_pos(tid + it * NT, g);
                if (gp.valid) {
#pragma unroll
                  for (int r = 0; r < NREG; ++r)
                    if (r < n_reg)
                      *reinterpret_cast<float4 *>(state + (n_dbuf + r) * g.P + gp.q * 4) =
                          nreg[it][r];
                }
              }
            }
            __syncthreads();
          }
        }
        parity ^= 1;
        ++step;
      }
      steps_total += step;
      change_sum += change;
      if (A.state_out) {
        // Final state of this experiment, unpadded [gene][y][x].
        const int fin = parity ? G : 0;
        const int planes_out = min(G, A.state_planes);
        float *so = A.state_out + ((size_t)orig * A.n_exp + e) * A.state_planes * g.W * g.H;
        for (int i = tid; i < planes_out * g.W * g.H; i += NT) {
          const int k = i / (g.W * g.H), r = i - k * g.W * g.H;
          const int y = r / g.W, x = r - y * g.W;
          const int plane = k < n_dbuf ? k + fin : k;
          so[i] = state[plane * g.P + y * g.Wp + x];
        }
      }

      // Fitness of the experiment (simstate.cpp:135-158), FP64 sums.
      const float *tgt = A.target + (size_t)e * A.n_target * A.W * A.H;
      const int fin_shift = parity ? G : 0;
      double acc = 0.0;
      for (int q = tid; q < g.Q; q += NT) {
        const int y = q / g.Wg, x0 = (q - y * g.Wg) * 4;
        for (int j = 0; j < 4; ++j) {
          const int x = x0 + j;
          if (x >= g.W) break;
          for (int k = 0; k < A.n_target; ++k) {
            const int gene = A.n_in + k;
            const int plane = gene < n_dbuf ? gene + fin_shift : gene;
            const double a = state[plane * g.P + q * 4 + j];
            const double b = tgt[((size_t)k * g.H + y) * g.W + x];
            if (A.fitness_kind == GRN_FITNESS_MSE) {
              acc += (a - b) * (a - b);
            } else {
              const double sub = fabs(a - b) - A.dist_threshold;
              if (sub > 0) acc += log(1.0 + sub);
            }
          }
        }
      }
      double dist = block_sum<NT>(acc, s_dred, lane, warp);
      if (A.fitness_kind == GRN_FITNESS_MSE)
        dist /= (double)g.W * g.H * A.n_target;
      else
        dist /= (double)(g.W * g.H);
      // Non-convergence penalty on the running change sum
      // (evaluatormorphogens.cpp:62-65).
      if (change_sum > A.min_conc_change) dist += change_sum - A.min_conc_change;
      error += dist / A.n_exp;
    }
    if (tid == 0) {
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

#define GRN_SMEM_VARIANT(NT, GMAX, ITEMS, NREG)            \
  {{GRN_SCHEDULE_SMEM_1BUF, NT, GMAX, ITEMS, NREG, false}, \
   &sim_kernel<NT, GMAX, ITEMS, NREG, false>}
#define GRN_GLOBAL_VARIANT(NT, GMAX) \
  {{GRN_SCHEDULE_GLOBAL, NT, GMAX, 1, 0, true}, &sim_kernel<NT, GMAX, 1, 0, true>}

const VariantEntry kVariants[] = {
    GRN_SMEM_VARIANT(256, 4, 1, 0),   GRN_SMEM_VARIANT(256, 8, 1, 0),
    GRN_SMEM_VARIANT(256, 16, 1, 0),  GRN_SMEM_VARIANT(512, 4, 1, 0),
    GRN_SMEM_VARIANT(512, 8, 1, 0),   GRN_SMEM_VARIANT(512, 16, 1, 0),
    GRN_SMEM_VARIANT(1024, 4, 1, 0),  GRN_SMEM_VARIANT(256, 8, 1, 4),
    GRN_SMEM_VARIANT(512, 8, 2, 4),   GRN_SMEM_VARIANT(256, 4, 4, 4),
    GRN_SMEM_VARIANT(512, 4, 2, 4),   GRN_SMEM_VARIANT(256, 16, 1, 8),
    GRN_GLOBAL_VARIANT(256, 16),      GRN_GLOBAL_VARIANT(512, 8),
    GRN_GLOBAL_VARIANT(512, 16),
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

const VariantEntry *find_variant(const KernelVariant &v) {
  for (int i = 0; i < kNumVariants; ++i) {
    const KernelVariant &k = kVariants[i].v;
    if (k.threads == v.threads && k.gmax == v.gmax && k.items == v.items &&
        k.nreg == v.nreg && k.global_state == v.global_state)
      return &kVariants[i];
  }
  return nullptr;
}

}  // namespace

size_t sim_fixed_smem_bytes() { return kStateOffset; }

int sim_variant_count() { return kNumVariants; }

KernelVariant sim_variant(int i) { return kVariants[i].v; }

cudaError_t sim_occupancy(const KernelVariant &v, size_t smem_bytes,
                          int *blocks_per_sm) {
  const VariantEntry *e = find_variant(v);
  if (!e) return cudaErrorInvalidValue;
  cudaError_t err = cudaFuncSetAttribute(
      e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (err != cudaSuccess) {
    *blocks_per_sm = 0;
    cudaGetLastError();
    return cudaSuccess;
  }
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, e->fn,
                                                       v.threads, smem_bytes);
}

cudaError_t sim_launch(const LaunchPlan &plan, const SimArgs &args,
                       cudaStream_t stream) {
  const VariantEntry *e = find_variant(plan.v);
  if (!e) return cudaErrorInvalidValue;
  cudaError_t err = cudaFuncSetAttribute(
      e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan.smem_bytes);
  if (err != cudaSuccess) return err;
  e->fn<<<plan.blocks, plan.v.threads, plan.smem_bytes, stream>>>(args);
  return cudaGetLastError();
}

}  // namespace grn
