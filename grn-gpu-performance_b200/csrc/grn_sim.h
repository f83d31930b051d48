// grn_sim.h -- launch interface between the host evaluator and the
// simulation kernels (grn_sim_kernel.cu).  Internal to the library.
#ifndef GRN_SIM_H_
#define GRN_SIM_H_

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "grn_packed.h"

namespace grn {

// Everything a simulation launch reads or writes.  Pointers are device
// pointers.
struct SimArgs {
  const uint4 *packed;       // model records (grn_packed.h)
  const int32_t *offsets;    // [n_models] first word of each record
  int32_t n_models;
  int32_t n_exp;             // experiments
  int32_t n_in;              // input morphogens (initial channels)
  int32_t n_target;          // target morphogens
  int32_t W, H;              // grid width (x) and height (y)
  int32_t Wg;                // float4 groups per row = ceil(W / 4)
  int32_t n_steps;           // max Euler steps per experiment
  int32_t fitness_kind;      // grn_fitness_kind
  int32_t planes;            // shared-memory state planes per block (even)
  int32_t fast_ok;           // experiments allow the fast path (non-negative
                             // finite initial state, minConc >= 0)
  float dt;
  float min_conc;
  double min_conc_change;
  double dist_threshold;
  const float *initial;      // [n_exp][n_in][H][W]
  const float *target;       // [n_exp][n_target][H][W]
  const double *max_error;   // [caller index]
  double *raw_error;         // [caller index] out
  int32_t *steps;            // [caller index] out, may be null
  int32_t *work_counter;     // zeroed before the launch
  int32_t *error_flag;       // set non-zero on an internal error
  float *gstate;             // global state slots, one per block (or null)
  int64_t slot_floats;       // floats per global state slot
  float *state_out;          // optional final states
                             // [caller index][n_exp][state_planes][H][W]
  int32_t state_planes;
  int32_t trace_every;       // steps between trace frames (frame 0: initial)
  float *trace_out;          // optional trace frames [caller index][n_exp]
                             // [trace_frames][state_planes][H][W]
  int32_t trace_frames;
  int32_t band_rows;         // streaming schedule: rows per staged band
  int32_t test_hooks;        // kHook* bits (tests of the error paths)
};

// Test hooks (grn_set_test_hooks): make a bounded wait run out on purpose.
constexpr int32_t kHookWithholdBandCopy = 1;  // streaming: band 1's copy is never issued

// One compiled kernel variant.
struct KernelVariant {
  int threads;  // threads per block
  int gmax;     // most genes a model may have
  int items;    // float4 groups each thread owns (fixed items)
  bool loop;    // threads walk the grid's groups (any grid size)
  bool ragged;  // compiled for W not a multiple of 4
  bool cluster; // cluster-split: a cluster of CTAs per model, one band of
                // rows each
  bool trace;   // writes trace frames (SimArgs::trace_out)
  int stream;   // 0; 1 streaming schedule (SimArgs::band_rows); 2 streaming
                // with two Euler steps per pass (temporal blocking)
};

// Launch plan chosen by the host.
struct LaunchPlan {
  KernelVariant v;
  int schedule;          // grn_schedule actually used
  int blocks;            // persistent grid size
  int planes;            // state planes in shared memory (even; may be 0)
  size_t smem_bytes;     // dynamic shared memory
  int blocks_per_sm;
  int64_t slot_floats;   // floats of one block's global state slot (0: none)
  int cluster;           // CTAs per cluster (1: one CTA per model)
  int band_rows;         // streaming schedule: rows per staged band (else 0)
};

#ifdef __CUDACC__
#define GRN_HOST_DEVICE __host__ __device__
#else
#define GRN_HOST_DEVICE
#endif

// Floats of one padded state row: W rounded up to float4 groups, plus one
// zero group when W is a multiple of 4, so that every row ends in at least
// one zero cell (the right border of its last cell and the left border of
// the next row's first cell).
GRN_HOST_DEVICE inline int row_floats(int W) {
  return 4 * ((W + 3) / 4) + (W % 4 == 0 ? 4 : 0);
}

// Floats of one state plane of a W x H grid: padded rows plus a zero row
// above and below (see the kernel's Geom).  With a cluster of C CTAs per
// model a CTA's plane holds a band of ceil(H / C) rows.
inline int64_t plane_floats(int W, int H, int cluster = 1) {
  return (int64_t)((H + cluster - 1) / cluster + 2) * row_floats(W);
}

// Bytes of shared memory a block needs besides the state planes.
size_t sim_fixed_smem_bytes();

// Number of compiled variants and their descriptions.
int sim_variant_count();
KernelVariant sim_variant(int i);

// Occupancy of a variant with `smem_bytes` dynamic shared memory: resident
// blocks per SM (0 if it does not fit).  Sets the function's max dynamic
// shared memory attribute as a side effect.
cudaError_t sim_occupancy(const KernelVariant &v, size_t smem_bytes,
                          int *blocks_per_sm);

// Cluster-split variant: resident clusters of `cluster` CTAs on the device
// (0 if it does not fit).
cudaError_t sim_cluster_occupancy(const KernelVariant &v, size_t smem_bytes, int cluster,
                                  int *clusters);

// Launches a variant; the caller has zeroed args.work_counter on `stream`.
cudaError_t sim_launch(const LaunchPlan &plan, const SimArgs &args,
                       cudaStream_t stream);

}  // namespace grn

#endif  // GRN_SIM_H_
