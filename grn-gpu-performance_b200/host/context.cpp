// context.cpp -- the C ABI of include/grn_gpu.h.
//
// Host side of the evaluator: the B200 counterpart of the reference's
// CEvaluatorMorphogens + CModelSimulator (Src/GPUSimulator/*.cpp).  One
// context = one device + one stream; experiments are uploaded once; a batch
// is compiled on the host (pack.cpp), copied from pinned staging buffers,
// simulated by one persistent kernel launch and read back as raw errors,
// which are rounded here exactly as the reference's evaluate does.

#include <cuda_runtime.h>

#include <sched.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <array>
#include <deque>
#include <map>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/grn_gpu.h"
#include "../csrc/grn_sim.h"
#include "pack.h"
#include "trace.h"

namespace {

using grn::LaunchPlan;
using grn::PackedHost;

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
};

struct HostBuf {
  void *p = nullptr;
  size_t cap = 0;
};

// Scratch of one in-flight evaluation: device buffers, pinned staging and a
// completion event.
struct Job {
  DevBuf d_words, d_offsets, d_maxerr, d_raw, d_steps, d_flag;
  HostBuf h_words, h_offsets, h_maxerr, h_raw, h_steps, h_flag;
  cudaEvent_t ev_start = nullptr, ev_kernel = nullptr, ev_done = nullptr;
  cudaGraphExec_t exec = nullptr;  // graph mode: this job's instantiated graph
  // Results of an asynchronous submission.
  int tag = 0;
  int n_models = 0;
  double *error_out = nullptr;
  double *raw_out = nullptr;
  std::vector<double> max_error;
  int64_t cells = 0;
};

}  // namespace

struct grn_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  grn_sim_params p{};
  std::string last_error;
  int n_sm = 0;
  int smem_optin = 0;
  int n_exp = 0;
  DevBuf d_initial, d_target, d_counter, d_gstate;
  DevBuf d_sample;  // autotuning: offsets of the sampled records
  // grn_run_packed's error flag: sticky across launches, read and cleared by
  // grn_run_packed_status.
  DevBuf d_packed_flag;
  Job sync_job;
  std::deque<Job *> pending;
  std::vector<Job *> free_jobs;
  int forced_schedule = GRN_SCHEDULE_AUTO;
  int forced_threads = 0;
  int forced_cluster = 0;
  int test_hooks = 0;   // grn_set_test_hooks
  bool graphs = false;  // evaluations replay one CUDA graph per job
  int host_threads = 0;  // threads compiling a batch (0: the CPUs this process may use)
  // Measured autotuning of GRN_SCHEDULE_AUTO: the fastest plan timed on a
  // sample of the first batch of each shape, by (W, H, max genes, max links,
  // experiments, fast path, batch-size bucket).
  bool autotune = true;
  struct Tuned {
    grn::KernelVariant v;
    int cluster, planes;
    double ms;
  };
  std::map<std::array<int, 7>, Tuned> tuned;
  std::string last_tuning;  // the last autotuning's candidates and times
  int n_tunings = 0;         // autotuning runs so far
  double tuning_ms = 0;      // their host wall time
  // minConc is 0 and the uploaded initial states are finite, non-negative
  // and at most 1e6: the kernel's fast path then gives the same results as
  // the exact one for every model whose step size keeps its state bounded
  // (see the kernel's update_cell and euler_bounded).
  bool fast_ok = false;
};

struct grn_packed {
  grn_ctx *ctx = nullptr;
  PackedHost host;
  DevBuf d_words, d_offsets;
  int64_t cell_bound = 0;
};

namespace {

grn_status fail(grn_ctx *ctx, grn_status s, const std::string &msg) {
  if (ctx) ctx->last_error = msg;
  return s;
}

// The kernel's error flag: 1 a model record it cannot run, 2 a bounded
// wait for a bulk copy that ran out (streaming schedule), 3 a state access
// outside its buffer (bounds-checked build only).
grn_status kernel_flag_error(grn_ctx *ctx, int32_t flag) {
  return fail(ctx, GRN_ERR_KERNEL,
              flag == 3   ? "bounds check: a simulation kernel state access fell outside its buffer"
              : flag == 2 ? "the simulation kernel's wait for a bulk copy timed out"
                          : "the simulation kernel rejected a model record");
}

grn_status cuda_fail(grn_ctx *ctx, cudaError_t e, const char *what) {
  std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
  return fail(ctx, e == cudaErrorMemoryAllocation ? GRN_ERR_OUT_OF_MEMORY : GRN_ERR_CUDA, msg);
}

#define GRN_CUDA(ctx, expr)                               \
  do {                                                    \
    cudaError_t e__ = (expr);                             \
    if (e__ != cudaSuccess) return cuda_fail(ctx, e__, #expr); \
  } while (0)

grn_status ensure_dev(grn_ctx *ctx, DevBuf *b, size_t bytes) {
  if (bytes <= b->cap) return GRN_OK;
  if (ctx->test_hooks & GRN_TEST_FAIL_DEVICE_ALLOC)
    return fail(ctx, GRN_ERR_OUT_OF_MEMORY, "device allocation refused (test hook)");
  if (b->p) cudaFree(b->p);
  b->p = nullptr;
  b->cap = 0;
  size_t cap = std::max<size_t>(bytes + bytes / 4, 256);
  GRN_CUDA(ctx, cudaMalloc(&b->p, cap));
  b->cap = cap;
  return GRN_OK;
}

grn_status ensure_host(grn_ctx *ctx, HostBuf *b, size_t bytes) {
  if (bytes <= b->cap) return GRN_OK;
  if (b->p) cudaFreeHost(b->p);
  b->p = nullptr;
  b->cap = 0;
  size_t cap = std::max<size_t>(bytes + bytes / 4, 256);
  GRN_CUDA(ctx, cudaHostAlloc(&b->p, cap, cudaHostAllocDefault));
  b->cap = cap;
  return GRN_OK;
}

void free_job(Job *j) {
  for (DevBuf *b : {&j->d_words, &j->d_offsets, &j->d_maxerr, &j->d_raw, &j->d_steps, &j->d_flag})
    if (b->p) cudaFree(b->p);
  for (HostBuf *b : {&j->h_words, &j->h_offsets, &j->h_maxerr, &j->h_raw, &j->h_steps, &j->h_flag})
    if (b->p) cudaFreeHost(b->p);
  for (cudaEvent_t e : {j->ev_start, j->ev_kernel, j->ev_done})
    if (e) cudaEventDestroy(e);
  if (j->exec) cudaGraphExecDestroy(j->exec);
}

grn_status check_params(const grn_sim_params *p) {
  if (!p) return GRN_ERR_INVALID_ARGUMENT;
  if (p->dim_x < 1 || p->dim_y < 1 || p->dim_x > 4096 || p->dim_y > 4096)
    return GRN_ERR_INVALID_ARGUMENT;
  if (p->n_input_morphogens < 0 || p->n_input_morphogens > GRN_MAX_INPUT_MORPHOGENS)
    return GRN_ERR_INVALID_ARGUMENT;
  if (p->n_target_morphogens < 0 || p->n_target_morphogens > 3)
    return GRN_ERR_INVALID_ARGUMENT;
  if (p->n_input_morphogens + p->n_target_morphogens > GRN_MAX_GENES)
    return GRN_ERR_INVALID_ARGUMENT;
  if (p->num_sim_steps < 0 || p->error_precision < 0 || p->error_precision > 17)
    return GRN_ERR_INVALID_ARGUMENT;
  if (p->fitness_kind != GRN_FITNESS_REF_LOGTHRESH && p->fitness_kind != GRN_FITNESS_MSE)
    return GRN_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(p->dt)) return GRN_ERR_INVALID_ARGUMENT;
  return GRN_OK;
}

grn_status check_batch(grn_ctx *ctx, const grn_model_batch *b) {
  if (!b || b->n_models < 0) return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "null batch");
  if (b->n_models == 0) return GRN_OK;
  if (!b->product_offsets || !b->link_offsets)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "null offsets");
  if (b->product_offsets[0] != 0 || b->link_offsets[0] != 0)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "offsets must start at 0");
  for (int m = 0; m < b->n_models; ++m) {
    if (b->product_offsets[m + 1] < b->product_offsets[m] ||
        b->link_offsets[m + 1] < b->link_offsets[m])
      return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "offsets must not decrease");
  }
  if (b->product_offsets[b->n_models] > 0 && !b->products)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "null products");
  if (b->link_offsets[b->n_models] > 0 && !b->links)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "null links");
  return GRN_OK;
}

// Threads that compile a batch: the context's setting, else the CPUs this
// process may run on (its affinity mask: several ranks of one node each get
// their share when a launcher pins them).
int host_threads(const grn_ctx *ctx) {
  if (ctx->host_threads > 0) return ctx->host_threads;
  cpu_set_t set;
  if (sched_getaffinity(0, sizeof set, &set) == 0) {
    const int n = CPU_COUNT(&set);
    if (n > 0) return n;
  }
  const unsigned n = std::thread::hardware_concurrency();
  return n ? (int)n : 1;
}

// Autotuner, first stage: every compiled kernel variant that can run the
// batch is scored by its resident useful threads per SM (occupancy x
// threads that own a group), fixed items preferred over walking ones and
// all-shared-memory state over state spilling to global slots.
// Every feasible launch plan for a batch, with the heuristic throughput
// score of each.
// Rows per staged band of the streaming schedule: two stages of
// gmax x (rows + 2) padded rows must fit the shared memory left over, one
// stage's bytes must stay below the mbarrier transaction limit (2^20), and
// a multiple of NT / Wg rows keeps every thread busy when Wg divides NT.
int stream_rows(int W, int H, int gmax, size_t room, int threads) {
  const int Wg = (W + 3) / 4;
  const size_t row_bytes = (size_t)grn::row_floats(W) * sizeof(float);
  long r = (long)(room / (2 * gmax * row_bytes)) - 2;
  r = std::min<long>(r, H);
  while (r > 1 && (size_t)gmax * (r + 2) * row_bytes >= (size_t)1 << 20) --r;
  if (r < 1) return 0;
  if (threads % Wg == 0 && r >= threads / Wg) r -= r % (threads / Wg);
  return (int)r;
}

// Output rows per band of the two-steps-per-pass streaming variant: its
// stage holds R + 4 rows of every gene and its intermediate R + 2, i.e.
// gmax * (2R + 6) rows (the one-step pass it falls back to uses the same
// space as two stages of R + 3 rows).  Rows of a pass's step one are a
// multiple of the block's threads where that is possible.
int stream2_rows(int W, int H, int gmax, size_t room, int threads) {
  const int Wg = (W + 3) / 4;
  const size_t row_bytes = (size_t)grn::row_floats(W) * sizeof(float);
  long r = ((long)(room / (gmax * row_bytes)) - 6) / 2;
  r = std::min<long>(r, H);
  // One pass's copies complete on one mbarrier (transaction count < 2^20).
  while (r > 1 && (size_t)gmax * (r + 4) * row_bytes >= (size_t)1 << 20) --r;
  if (r < 1) return 0;
  if (threads % Wg == 0) {
    const long per = threads / Wg;  // rows per full pass of the block's threads
    if (r + 2 >= per && (r + 2) % per != 0) r -= (r + 2) % per;
  }
  return r >= 1 ? (int)r : 0;
}

grn_status enumerate_plans(grn_ctx *ctx, int max_genes, int n_models, bool trace,
                           std::vector<std::pair<double, LaunchPlan>> *out) {
  const int W = ctx->p.dim_x, H = ctx->p.dim_y;
  const int Wg = (W + 3) / 4;
  const bool ragged = (W % 4) != 0;
  const size_t fixed = grn::sim_fixed_smem_bytes();
  const size_t optin = (size_t)ctx->smem_optin;
  // A trace runs on the trace variants whatever schedule is forced.
  const int sched = trace ? GRN_SCHEDULE_WALK_ITEMS : ctx->forced_schedule;
  static const int kClusterSizes[] = {2, 4, 8, 16};
  out->clear();
  const int nv = grn::sim_variant_count();
  for (int i = 0; i < nv; ++i) {
    const grn::KernelVariant v = grn::sim_variant(i);
    if (v.gmax < max_genes || v.ragged != ragged || v.trace != trace) continue;
    if (ctx->forced_threads && !trace && v.threads != ctx->forced_threads) continue;
    if (v.stream) {
      // Streaming: only where the planes do not all fit shared memory.
      const int own = v.stream == 2 ? GRN_SCHEDULE_STREAM2 : GRN_SCHEDULE_STREAM;
      if (sched != GRN_SCHEDULE_AUTO && sched != own) continue;
      const size_t plane_bytes = (size_t)grn::plane_floats(W, H) * sizeof(float);
      const int fit = optin > fixed ? (int)((optin - fixed) / plane_bytes) & ~1 : 0;
      if (sched == GRN_SCHEDULE_AUTO && fit / 2 >= max_genes) continue;
      const size_t room = optin > fixed ? optin - fixed : 0;
      const int R = v.stream == 2 ? stream2_rows(W, H, v.gmax, room, v.threads)
                                  : stream_rows(W, H, v.gmax, room, v.threads);
      if (R < 1) continue;
      const size_t rows = v.stream == 2 ? (size_t)v.gmax * (2 * R + 6)
                                        : (size_t)2 * v.gmax * (R + 2);
      const size_t smem = fixed + rows * grn::row_floats(W) * sizeof(float);
      int per_sm = 0;
      GRN_CUDA(ctx, grn::sim_occupancy(v, smem, &per_sm));
      const int ctas = per_sm * ctx->n_sm;
      if (ctas < 1) continue;
      LaunchPlan plan{};
      plan.v = v;
      plan.schedule = own;
      plan.planes = 0;
      plan.smem_bytes = smem;
      plan.blocks_per_sm = per_sm;
      plan.slot_floats = 2LL * v.gmax * grn::plane_floats(W, H);
      plan.cluster = 1;
      plan.band_rows = R;
      plan.blocks = std::max(1, std::min(n_models, ctas));
      const double busy = (double)std::min(ctas, n_models) * std::min(v.threads, R * Wg);
      // Heuristic rank below the walking / all-global plans (faster only where the
      // slots' traffic leaves L2); the autotuner measures it against them.
      out->push_back({busy * 0.6 - 1e-3 * v.gmax, plan});
      continue;
    }
    if (sched == GRN_SCHEDULE_STREAM || sched == GRN_SCHEDULE_STREAM2) continue;
    if (sched == GRN_SCHEDULE_CLUSTER && !v.cluster) continue;
    if (sched != GRN_SCHEDULE_AUTO && sched != GRN_SCHEDULE_CLUSTER && v.cluster) continue;
    if (sched == GRN_SCHEDULE_FIXED_ITEMS && v.loop) continue;
    if ((sched == GRN_SCHEDULE_WALK_ITEMS || sched == GRN_SCHEDULE_GLOBAL) && !v.loop) continue;
    for (int ci = 0; ci < (v.cluster ? 4 : 1); ++ci) {
      const int C = v.cluster ? kClusterSizes[ci] : 1;
      if (v.cluster && ctx->forced_cluster && C != ctx->forced_cluster) continue;
      const int Hb = (H + C - 1) / C;
      if (C > 1 && (C - 1) * Hb >= H) continue;  // every band non-empty
      const int Qb = Hb * Wg;
      if (!v.loop && Qb > v.threads * v.items) continue;
      const size_t plane_bytes = (size_t)grn::plane_floats(W, H, C) * sizeof(float);
      int fit = optin > fixed ? (int)((optin - fixed) / plane_bytes) : 0;
      fit &= ~1;
      // Under AUTO a walking variant whose genes spill is also offered with
      // every plane in global memory (the L1 then caches more of them).
      const int smem_planes = std::min(fit, 2 * max_genes);
      const bool offer_global = sched == GRN_SCHEDULE_AUTO && v.loop && C == 1 &&
                                smem_planes / 2 < max_genes && smem_planes > 0;
      for (int gv = 0; gv < (offer_global ? 2 : 1); ++gv) {
        const int planes = (sched == GRN_SCHEDULE_GLOBAL || gv == 1) ? 0 : smem_planes;
        const bool spills = planes / 2 < max_genes;
        const size_t smem = fixed + planes * plane_bytes;
        int ctas = 0, per_sm = 0;  // resident CTAs on the device
        if (C == 1) {
          GRN_CUDA(ctx, grn::sim_occupancy(v, smem, &per_sm));
          ctas = per_sm * ctx->n_sm;
        } else {
          int clusters = 0;
          GRN_CUDA(ctx, grn::sim_cluster_occupancy(v, smem, C, &clusters));
          ctas = clusters * C;
          per_sm = 1;
        }
        if (ctas < 1) continue;
        // Throughput model: busy threads (no more CTAs than models need),
        // fixed items ahead of walking ones, and a penalty for genes kept in
        // global memory -- mild while every resident CTA's slot fits in L2.
        const double busy = (double)std::min(ctas, n_models * C) * std::min(v.threads, Qb);
        const double spill_frac = spills ? 1.0 - (double)(planes / 2) / max_genes : 0.0;
        const double slot_bytes = spills ? 2.0 * v.gmax * plane_bytes : 0.0;
        const bool l2 = slot_bytes * ctas <= 80e6;
        double score = busy * (v.loop ? 1.0 : 1.25) * (1.0 - (l2 ? 0.3 : 0.7) * spill_frac);
        // One cluster barrier per step costs about as much as a step of a
        // small band (measured): clusters only as a last resort unmeasured.
        if (C > 1) score *= 0.3 - 0.01 * C;
        if (gv == 1) score *= 0.9;
        score -= 1e-3 * v.gmax;  // prefer the tighter register footprint
        LaunchPlan plan{};
        plan.v = v;
        plan.schedule = C > 1                                      ? GRN_SCHEDULE_CLUSTER
                        : (sched == GRN_SCHEDULE_GLOBAL || gv == 1) ? GRN_SCHEDULE_GLOBAL
                        : v.loop                                    ? GRN_SCHEDULE_WALK_ITEMS
                                                                    : GRN_SCHEDULE_FIXED_ITEMS;
        plan.planes = planes;
        plan.smem_bytes = smem;
        plan.blocks_per_sm = per_sm;
        plan.slot_floats = spills ? 2LL * v.gmax * grn::plane_floats(W, H, C) : 0;
        plan.cluster = C;
        plan.blocks = C > 1 ? C * std::max(1, std::min(n_models, ctas / C))
                            : std::max(1, std::min(n_models, ctas));
        out->push_back({score, plan});
      }
    }
  }
  if (out->empty())
    return fail(ctx, GRN_ERR_CAPACITY, "no kernel variant holds " + std::to_string(max_genes) +
                                           " genes on this grid with this schedule");
  std::stable_sort(out->begin(), out->end(),
                   [](const std::pair<double, LaunchPlan> &a,
                      const std::pair<double, LaunchPlan> &b) { return a.first > b.first; });
  return GRN_OK;
}

grn_status choose_plan(grn_ctx *ctx, int max_genes, int n_models, LaunchPlan *out) {
  std::vector<std::pair<double, LaunchPlan>> plans;
  grn_status s = enumerate_plans(ctx, max_genes, n_models, false, &plans);
  if (s != GRN_OK) return s;
  *out = plans[0].second;
  return GRN_OK;
}

bool same_plan(const LaunchPlan &a, const grn::KernelVariant &v, int cluster, int planes) {
  return a.v.threads == v.threads && a.v.gmax == v.gmax && a.v.items == v.items &&
         a.v.loop == v.loop && a.v.ragged == v.ragged && a.v.cluster == v.cluster &&
         a.v.stream == v.stream &&
         a.cluster == cluster && a.planes == planes;
}

// Launches the simulation of `n_models` packed records already on the
// device.  `stream` may differ from the context's stream.
// Sets the plan's state planes and global state slots in `a` (allocating
// the slots if they grew).
grn_status bind_state(grn_ctx *ctx, const LaunchPlan &plan, grn::SimArgs *a) {
  a->planes = plan.planes;
  a->band_rows = plan.band_rows;
  a->gstate = nullptr;
  a->slot_floats = 0;
  if (plan.slot_floats > 0) {
    grn_status s =
        ensure_dev(ctx, &ctx->d_gstate, (size_t)plan.slot_floats * plan.blocks * sizeof(float));
    if (s != GRN_OK) return s;
    a->gstate = static_cast<float *>(ctx->d_gstate.p);
    a->slot_floats = plan.slot_floats;
  }
  return GRN_OK;
}

// Enqueues one launch whose arguments bind_state has completed: the work
// counter reset and the kernel (no allocation, no synchronisation).
grn_status enqueue_plan(grn_ctx *ctx, const LaunchPlan &plan, const grn::SimArgs &a,
                        cudaStream_t stream) {
  GRN_CUDA(ctx, cudaMemsetAsync(ctx->d_counter.p, 0, sizeof(int32_t), stream));
  GRN_CUDA(ctx, grn::sim_launch(plan, a, stream));
  return GRN_OK;
}

grn_status launch_plan(grn_ctx *ctx, const LaunchPlan &plan, grn::SimArgs a, cudaStream_t stream) {
  grn_status s = bind_state(ctx, plan, &a);
  if (s != GRN_OK) return s;
  return enqueue_plan(ctx, plan, a, stream);
}

// Measured autotuning: times the feasible plans (best heuristic scores
// first, at most 8) on the batch's first models -- the most expensive ones,
// the host orders records by cost -- with the step count capped.  Every
// candidate is launched once untimed (first-launch costs, and the GPU's
// clock ramp before any timing), then timed in three interleaved rounds,
// keeping each candidate's fastest launch, so that no candidate is favoured
// by when it ran.  A candidate replaces the heuristic's first choice only if
// it is at least 3% faster.  The sample launches write outputs of the
// sampled models that the real launch then overwrites.  Synchronises
// `stream` once per new batch shape.
// The autotuner's cache key: grid, the kernels' gene capacity class (4, 8
// or 16 genes), a coarse link class (the balance of work per cell),
// experiments, fast path, and the batch size when it is below two models
// per SM.  The exact gene and link counts are left out: a search's batches
// vary in them from one generation to the next (its population grows), and
// each new key costs a tuning run.  A kept plan is reused only where it is
// among the batch's own candidates (same variant, cluster and planes),
// else the batch is tuned again.
std::array<int, 7> tune_key(const grn_ctx *ctx, int n_models, int max_genes, int max_links) {
  const int genes_class = max_genes <= 4 ? 4 : max_genes <= 8 ? 8 : 16;
  const int links_class = max_links <= 8 ? 0 : max_links <= 32 ? 1 : 2;
  const int bucket = n_models >= 2 * ctx->n_sm ? 0 : n_models;
  return {ctx->p.dim_x, ctx->p.dim_y, genes_class, links_class, ctx->n_exp,
          ctx->fast_ok ? 1 : 0, bucket};
}

// The plan kept for this key, if it is among the batch's candidates.
bool cached_plan(const grn_ctx *ctx, const std::vector<std::pair<double, LaunchPlan>> &plans,
                 const std::array<int, 7> &key, LaunchPlan *out) {
  const auto it = ctx->tuned.find(key);
  if (it == ctx->tuned.end()) return false;
  for (const auto &c : plans)
    if (same_plan(c.second, it->second.v, it->second.cluster, it->second.planes)) {
      *out = c.second;
      return true;
    }
  return false;
}

grn_status autotune_plan(grn_ctx *ctx, const std::vector<std::pair<double, LaunchPlan>> &plans,
                         const grn::SimArgs &a, int n_models, const int32_t *h_offsets,
                         cudaStream_t stream, LaunchPlan *out) {
  grn::TraceRange trace_range("grn autotune");
  grn::SimArgs t = a;
  // About 2^29 cell-updates per sample launch: up to 8 models per SM (so
  // that, as in the full batch, the slowest block's last model is a small
  // part of the launch), at least 2 per SM, at least 128 steps (past the
  // first steps' atypical speed while states are still mostly zero).
  const double budget = (double)(1u << 29);
  const double model_cells = (double)a.W * a.H * std::max(1, a.n_exp);
  const int by_budget = (int)std::min(1e9, budget / (128.0 * model_cells));
  t.n_models = std::min(n_models, std::max(2 * ctx->n_sm, std::min(8 * ctx->n_sm, by_budget)));
  t.n_steps = std::min(a.n_steps,
                       std::max(128, (int)std::min(1e6, budget / (t.n_models * model_cells))));
  if (h_offsets && n_models > t.n_models) {
    // Records are in decreasing cost: sample across the whole batch, not
    // just its most expensive head, so the sample's mix of model sizes is
    // the batch's.
    std::vector<int32_t> pick(t.n_models);
    for (int i = 0; i < t.n_models; ++i)
      pick[i] = h_offsets[(int64_t)i * n_models / t.n_models];
    grn_status ss = ensure_dev(ctx, &ctx->d_sample, pick.size() * sizeof(int32_t));
    if (ss != GRN_OK) return ss;
    GRN_CUDA(ctx, cudaMemcpyAsync(ctx->d_sample.p, pick.data(), pick.size() * sizeof(int32_t),
                                  cudaMemcpyHostToDevice, stream));
    GRN_CUDA(ctx, cudaStreamSynchronize(stream));  // `pick` is pageable and local
    t.offsets = static_cast<const int32_t *>(ctx->d_sample.p);
  }
  t.state_out = nullptr;
  t.state_planes = 0;
  const int n_try = std::min<int>((int)plans.size(), 8);
  std::vector<LaunchPlan> cand;
  for (int i = 0; i < n_try; ++i) {
    LaunchPlan ps = plans[i].second;
    const int C = std::max(1, ps.cluster);
    // resident CTAs for the full batch (>= the sample's need)
    ps.blocks = std::max(C, std::min(ps.blocks, C * t.n_models));
    ps.blocks -= ps.blocks % C;
    cand.push_back(ps);
  }
  std::vector<cudaEvent_t> ev(2 * n_try, nullptr);
  grn_status s = GRN_OK;
  for (auto &e : ev)
    if (s == GRN_OK && cudaEventCreate(&e) != cudaSuccess) s = fail(ctx, GRN_ERR_CUDA, "event");
  std::vector<double> best_ms(n_try, 1e30);
  for (int i = 0; i < n_try && s == GRN_OK; ++i) s = launch_plan(ctx, cand[i], t, stream);
  for (int round = 0; round < 3 && s == GRN_OK; ++round) {
    for (int i = 0; i < n_try && s == GRN_OK; ++i) {
      if (cudaEventRecord(ev[2 * i], stream) != cudaSuccess) s = fail(ctx, GRN_ERR_CUDA, "event");
      if (s == GRN_OK) s = launch_plan(ctx, cand[i], t, stream);
      if (s == GRN_OK && cudaEventRecord(ev[2 * i + 1], stream) != cudaSuccess)
        s = fail(ctx, GRN_ERR_CUDA, "event");
    }
    if (s == GRN_OK && cudaStreamSynchronize(stream) != cudaSuccess)
      s = fail(ctx, GRN_ERR_CUDA, "autotune timing");
    for (int i = 0; i < n_try && s == GRN_OK; ++i) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]) == cudaSuccess)
        best_ms[i] = std::min(best_ms[i], (double)ms);
    }
  }
  for (auto &e : ev)
    if (e) cudaEventDestroy(e);
  if (s != GRN_OK) return s;
  // The first plan in the heuristic's order whose sample time is within 3%
  // of the fastest: a short sample separates near-ties poorly (the walking
  // and the all-global plans of a spilled grid time alike on 128 steps,
  // while over a full run the walking one is 12% faster).
  int fastest = 0;
  for (int i = 1; i < n_try; ++i)
    if (best_ms[i] < best_ms[fastest]) fastest = i;
  int best = fastest;
  for (int i = 0; i < fastest; ++i)
    if (best_ms[i] <= 1.03 * best_ms[fastest]) {
      best = i;
      break;
    }
  std::string rep;
  for (int i = 0; i < n_try; ++i) {
    const LaunchPlan &p = cand[i];
    char line[200];
    std::snprintf(line, sizeof line,
                  "%s schedule %d threads %d gmax %d items %d cluster %d planes %d band %d "
                  "blocks %d ms %.4f\n",
                  i == best ? "*" : " ", p.schedule, p.v.threads, p.v.gmax, p.v.items,
                  std::max(1, p.cluster), p.planes, p.band_rows, p.blocks, best_ms[i]);
    rep += line;
  }
  ctx->last_tuning = rep;
  if (best_ms[best] >= 1e30) return fail(ctx, GRN_ERR_CUDA, "autotune timed no plan");
  *out = plans[best].second;
  return GRN_OK;
}

// Optional outputs of a launch: final states, trace frames, one experiment.
struct LaunchExtras {
  float *states = nullptr;  // [model][n_exp][state_planes][H][W]
  int state_planes = 0;
  float *trace = nullptr;   // [model][n_exp][trace_frames][state_planes][H][W]
  int trace_every = 0, trace_frames = 0;
  int experiment = -1;      // >= 0: simulate only this experiment
  const int32_t *host_offsets = nullptr;  // host copy of the record offsets
                                          // (autotuning samples across the batch)
};

// Chooses the plan of a launch of `n_models` packed records already on the
// device (timing candidate plans on `stream` the first time a batch shape is
// seen) and fills its arguments, state slots bound: everything but
// enqueueing it.
grn_status prepare_packed(grn_ctx *ctx, const uint4 *d_words, const int32_t *d_offsets,
                          int n_models, int max_genes, int max_links,
                          const double *d_max_error, double *d_raw, int32_t *d_steps,
                          int32_t *d_flag, cudaStream_t stream, LaunchPlan *plan_out,
                          grn::SimArgs *args_out, const LaunchExtras &ex) {
  if (ctx->n_exp < 1) return fail(ctx, GRN_ERR_NO_EXPERIMENTS, "no experiments uploaded");
  const bool trace = ex.trace != nullptr;
  std::vector<std::pair<double, LaunchPlan>> plans;
  grn_status s = enumerate_plans(ctx, max_genes, n_models, trace, &plans);
  if (s != GRN_OK) return s;
  LaunchPlan plan = plans[0].second;
  const int W = ctx->p.dim_x, H = ctx->p.dim_y, Wg = (W + 3) / 4;
  grn::SimArgs a{};
  a.packed = d_words;
  a.offsets = d_offsets;
  a.n_models = n_models;
  a.n_exp = ctx->n_exp;
  a.n_in = ctx->p.n_input_morphogens;
  a.n_target = ctx->p.n_target_morphogens;
  a.W = W;
  a.H = H;
  a.Wg = Wg;
  a.n_steps = ctx->p.num_sim_steps;
  a.fitness_kind = ctx->p.fitness_kind;
  a.planes = plan.planes;
  a.dt = (float)ctx->p.dt;
  a.min_conc = (float)ctx->p.min_conc;
  a.min_conc_change = ctx->p.min_conc_change;
  a.dist_threshold = ctx->p.dist_error_threshold;
  a.initial = static_cast<const float *>(ctx->d_initial.p);
  a.target = static_cast<const float *>(ctx->d_target.p);
  a.max_error = d_max_error;
  a.raw_error = d_raw;
  a.steps = d_steps;
  a.work_counter = static_cast<int32_t *>(ctx->d_counter.p);
  a.error_flag = d_flag;
  a.state_out = ex.states;
  a.state_planes = ex.state_planes;
  a.trace_out = ex.trace;
  a.trace_every = ex.trace_every;
  a.trace_frames = ex.trace_frames;
  a.fast_ok = ctx->fast_ok ? 1 : 0;
  a.test_hooks = ctx->test_hooks;
  if (ex.experiment >= 0) {
    const size_t cells = (size_t)W * H;
    a.initial += (size_t)ex.experiment * a.n_in * cells;
    a.target += (size_t)ex.experiment * a.n_target * cells;
    a.n_exp = 1;
  }
  if (!trace && ctx->forced_schedule == GRN_SCHEDULE_AUTO && ctx->autotune && plans.size() > 1) {
    const std::array<int, 7> key = tune_key(ctx, n_models, max_genes, max_links);
    if (!cached_plan(ctx, plans, key, &plan)) {
      const auto t0 = std::chrono::steady_clock::now();
      s = autotune_plan(ctx, plans, a, n_models, ex.host_offsets, stream, &plan);
      if (s != GRN_OK) return s;
      ctx->n_tunings += 1;
      char kl[128];
      std::snprintf(kl, sizeof kl,
                    "# key: grid %dx%d, gene class %d, link class %d, experiments %d, fast %d, "
                    "batch bucket %d\n",
                    key[0], key[1], key[2], key[3], key[4], key[5], key[6]);
      ctx->last_tuning = kl + ctx->last_tuning;
      ctx->tuning_ms +=
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      ctx->tuned[key] = grn_ctx::Tuned{plan.v, plan.cluster, plan.planes, 0.0};
    }
  }
  s = bind_state(ctx, plan, &a);
  if (s != GRN_OK) return s;
  *plan_out = plan;
  *args_out = a;
  return GRN_OK;
}

// Launches the simulation of `n_models` packed records already on the
// device.  `stream` may differ from the context's stream.
grn_status launch_packed(grn_ctx *ctx, const uint4 *d_words, const int32_t *d_offsets,
                         int n_models, int max_genes, int max_links,
                         const double *d_max_error, double *d_raw, int32_t *d_steps,
                         int32_t *d_flag, cudaStream_t stream, LaunchPlan *plan_out,
                         const LaunchExtras &ex = LaunchExtras()) {
  if (n_models == 0) return GRN_OK;
  LaunchPlan plan;
  grn::SimArgs a;
  grn_status s = prepare_packed(ctx, d_words, d_offsets, n_models, max_genes, max_links,
                                d_max_error, d_raw, d_steps, d_flag, stream, &plan, &a, ex);
  if (s != GRN_OK) return s;
  s = enqueue_plan(ctx, plan, a, stream);
  if (s != GRN_OK) return s;
  if (plan_out) *plan_out = plan;
  return GRN_OK;
}

// The autotuner has not yet chosen a plan for this batch shape.
// (The same test as prepare_packed's: a key without a kept plan, or a kept
// plan that is not among this batch's candidates.)
bool tuning_needed(grn_ctx *ctx, int n_models, int max_genes, int max_links) {
  if (ctx->forced_schedule != GRN_SCHEDULE_AUTO || !ctx->autotune) return false;
  std::vector<std::pair<double, LaunchPlan>> plans;
  if (enumerate_plans(ctx, max_genes, n_models, false, &plans) != GRN_OK) return false;
  if (plans.size() <= 1) return false;
  LaunchPlan p;
  return !cached_plan(ctx, plans, tune_key(ctx, n_models, max_genes, max_links), &p);
}

void fill_launch_stats(grn_eval_stats *stats, int n, std::chrono::steady_clock::time_point t0,
                       std::chrono::steady_clock::time_point t1, size_t h2d, size_t d2h,
                       const LaunchPlan &plan) {
  std::memset(stats, 0, sizeof *stats);
  stats->n_models = n;
  stats->pack_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  stats->h2d_bytes = (int64_t)h2d;
  stats->d2h_bytes = (int64_t)d2h;
  stats->schedule = plan.schedule;
  stats->threads_per_block = plan.v.threads;
  stats->blocks = plan.blocks;
  stats->cluster_size = std::max(1, plan.cluster);
}

// Graph mode: the job's copy-in, kernel, copy-out and timing events as one
// CUDA graph, captured from the stream and replayed.  A job keeps its
// instantiated graph; the next capture only updates its parameters (sizes,
// kernel arguments) when the plan keeps the graph's shape, else it is
// instantiated again.  Plan selection (with any autotuning) stays outside
// the capture.
grn_status enqueue_job_graph(grn_ctx *ctx, Job *j, int n, const PackedHost &ph, size_t wb,
                             size_t ob, size_t eb, size_t sb, LaunchPlan *plan_out) {
  cudaStream_t st = ctx->stream;
  LaunchPlan plan{};
  grn::SimArgs a{};
  grn_status s = prepare_packed(ctx, static_cast<const uint4 *>(j->d_words.p),
                                static_cast<const int32_t *>(j->d_offsets.p), n, ph.max_genes,
                                ph.max_links, static_cast<const double *>(j->d_maxerr.p),
                                static_cast<double *>(j->d_raw.p),
                                static_cast<int32_t *>(j->d_steps.p),
                                static_cast<int32_t *>(j->d_flag.p), st, &plan, &a,
                                LaunchExtras());
  if (s != GRN_OK) return s;
  GRN_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  chk(cudaMemcpyAsync(j->d_words.p, j->h_words.p, wb, cudaMemcpyHostToDevice, st));
  chk(cudaMemcpyAsync(j->d_offsets.p, j->h_offsets.p, ob, cudaMemcpyHostToDevice, st));
  chk(cudaMemcpyAsync(j->d_maxerr.p, j->h_maxerr.p, eb, cudaMemcpyHostToDevice, st));
  chk(cudaMemsetAsync(j->d_flag.p, 0, 4, st));
  chk(cudaEventRecordWithFlags(j->ev_start, st, cudaEventRecordExternal));
  if (e == cudaSuccess) s = enqueue_plan(ctx, plan, a, st);
  chk(cudaEventRecordWithFlags(j->ev_kernel, st, cudaEventRecordExternal));
  chk(cudaMemcpyAsync(j->h_raw.p, j->d_raw.p, eb, cudaMemcpyDeviceToHost, st));
  chk(cudaMemcpyAsync(j->h_steps.p, j->d_steps.p, sb, cudaMemcpyDeviceToHost, st));
  chk(cudaMemcpyAsync(j->h_flag.p, j->d_flag.p, 4, cudaMemcpyDeviceToHost, st));
  chk(cudaEventRecordWithFlags(j->ev_done, st, cudaEventRecordExternal));
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(st, &graph);
  if (s != GRN_OK || e != cudaSuccess || ec != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (s != GRN_OK) return s;
    return cuda_fail(ctx, e != cudaSuccess ? e : ec, "graph capture");
  }
  bool updated = false;
  if (j->exec) {
    cudaGraphExecUpdateResultInfo info;
    updated = cudaGraphExecUpdate(j->exec, graph, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();
      cudaGraphExecDestroy(j->exec);
      j->exec = nullptr;
    }
  }
  if (!updated) e = cudaGraphInstantiate(&j->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    j->exec = nullptr;
    return cuda_fail(ctx, e, "cudaGraphInstantiate");
  }
  GRN_CUDA(ctx, cudaGraphLaunch(j->exec, st));
  *plan_out = plan;
  return GRN_OK;
}

// Compiles a batch and enqueues copy-in, kernel and copy-out on the
// context's stream into job `j`.
grn_status enqueue_job(grn_ctx *ctx, Job *j, const grn_model_batch *batch,
                       const double *max_error, grn_eval_stats *stats) {
  grn_status s = check_batch(ctx, batch);
  if (s != GRN_OK) return s;
  if (!max_error) return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "null max_error");
  if (ctx->n_exp < 1) return fail(ctx, GRN_ERR_NO_EXPERIMENTS, "no experiments uploaded");
  const int n = batch->n_models;
  j->n_models = n;
  auto t0 = std::chrono::steady_clock::now();
  PackedHost ph;
  std::string err;
  s = grn::pack_batch(batch, ctx->p.n_input_morphogens + ctx->p.n_target_morphogens,
                      (float)ctx->p.dt, ctx->p.num_sim_steps,
                      host_threads(ctx), &ph, &err);
  if (s != GRN_OK) return fail(ctx, s, err);
  auto t1 = std::chrono::steady_clock::now();
  if (n == 0) return GRN_OK;
  const size_t wb = ph.words.size() * sizeof(uint4), ob = n * sizeof(int32_t);
  const size_t eb = n * sizeof(double), sb = n * sizeof(int32_t);
  if ((s = ensure_dev(ctx, &j->d_words, wb)) || (s = ensure_dev(ctx, &j->d_offsets, ob)) ||
      (s = ensure_dev(ctx, &j->d_maxerr, eb)) || (s = ensure_dev(ctx, &j->d_raw, eb)) ||
      (s = ensure_dev(ctx, &j->d_steps, sb)) || (s = ensure_dev(ctx, &j->d_flag, 4)) ||
      (s = ensure_host(ctx, &j->h_words, wb)) || (s = ensure_host(ctx, &j->h_offsets, ob)) ||
      (s = ensure_host(ctx, &j->h_maxerr, eb)) || (s = ensure_host(ctx, &j->h_raw, eb)) ||
      (s = ensure_host(ctx, &j->h_steps, sb)) || (s = ensure_host(ctx, &j->h_flag, 4)))
    return s;
  if (!j->ev_start) {
    GRN_CUDA(ctx, cudaEventCreate(&j->ev_start));
    GRN_CUDA(ctx, cudaEventCreate(&j->ev_kernel));
    GRN_CUDA(ctx, cudaEventCreate(&j->ev_done));
  }
  std::memcpy(j->h_words.p, ph.words.data(), wb);
  if (ctx->test_hooks & GRN_TEST_CORRUPT_RECORD) {
    // Gene count 0 in the first record's header (PackedHeader::n_genes).
    auto *hdr = reinterpret_cast<grn::PackedHeader *>(static_cast<uint4 *>(j->h_words.p) +
                                                      ph.offsets[0]);
    hdr->n_genes = 0;
  }
  std::memcpy(j->h_offsets.p, ph.offsets.data(), ob);
  std::memcpy(j->h_maxerr.p, max_error, eb);
  cudaStream_t st = ctx->stream;
  if (ctx->graphs && !tuning_needed(ctx, n, ph.max_genes, ph.max_links)) {
    LaunchPlan plan{};
    s = enqueue_job_graph(ctx, j, n, ph, wb, ob, eb, sb, &plan);
    if (s != GRN_OK) return s;
    j->cells = (int64_t)ctx->p.dim_x * ctx->p.dim_y;
    if (stats) fill_launch_stats(stats, n, t0, t1, wb + ob + eb, eb + sb + 4, plan);
    return GRN_OK;
  }
  GRN_CUDA(ctx, cudaMemcpyAsync(j->d_words.p, j->h_words.p, wb, cudaMemcpyHostToDevice, st));
  GRN_CUDA(ctx, cudaMemcpyAsync(j->d_offsets.p, j->h_offsets.p, ob, cudaMemcpyHostToDevice, st));
  GRN_CUDA(ctx, cudaMemcpyAsync(j->d_maxerr.p, j->h_maxerr.p, eb, cudaMemcpyHostToDevice, st));
  GRN_CUDA(ctx, cudaMemsetAsync(j->d_flag.p, 0, 4, st));
  // Plan first (a new batch shape is autotuned here, on the copied
  // records), so that the kernel events time the real launch only.
  LaunchPlan plan{};
  grn::SimArgs a{};
  LaunchExtras ex;
  ex.host_offsets = ph.offsets.data();
  s = prepare_packed(ctx, static_cast<const uint4 *>(j->d_words.p),
                     static_cast<const int32_t *>(j->d_offsets.p), n, ph.max_genes,
                     ph.max_links, static_cast<const double *>(j->d_maxerr.p),
                     static_cast<double *>(j->d_raw.p), static_cast<int32_t *>(j->d_steps.p),
                     static_cast<int32_t *>(j->d_flag.p), st, &plan, &a, ex);
  if (s != GRN_OK) return s;
  GRN_CUDA(ctx, cudaEventRecord(j->ev_start, st));
  s = enqueue_plan(ctx, plan, a, st);
  if (s != GRN_OK) return s;
  GRN_CUDA(ctx, cudaEventRecord(j->ev_kernel, st));
  GRN_CUDA(ctx, cudaMemcpyAsync(j->h_raw.p, j->d_raw.p, eb, cudaMemcpyDeviceToHost, st));
  GRN_CUDA(ctx, cudaMemcpyAsync(j->h_steps.p, j->d_steps.p, sb, cudaMemcpyDeviceToHost, st));
  GRN_CUDA(ctx, cudaMemcpyAsync(j->h_flag.p, j->d_flag.p, 4, cudaMemcpyDeviceToHost, st));
  GRN_CUDA(ctx, cudaEventRecord(j->ev_done, st));
  j->cells = (int64_t)ctx->p.dim_x * ctx->p.dim_y;
  if (stats) fill_launch_stats(stats, n, t0, t1, wb + ob + eb, eb + sb + 4, plan);
  return GRN_OK;
}

// Reads back a finished job: rounding as CEvaluatorMorphogens::evaluate
// (cevaluatormorphogens.cpp:233-245).
grn_status finish_job(grn_ctx *ctx, Job *j, const double *max_error, double *error_out,
                      double *raw_out, grn_eval_stats *stats) {
  const int n = j->n_models;
  if (n == 0) return GRN_OK;
  if (*static_cast<int32_t *>(j->h_flag.p) != 0)
    return kernel_flag_error(ctx, *static_cast<int32_t *>(j->h_flag.p));
  const double *raw = static_cast<const double *>(j->h_raw.p);
  const int32_t *steps = static_cast<const int32_t *>(j->h_steps.p);
  int64_t total_steps = 0;
  for (int m = 0; m < n; ++m) {
    if (error_out) error_out[m] = grn_round_error(raw[m], max_error[m], ctx->p.error_precision);
    if (raw_out) raw_out[m] = raw[m];
    total_steps += steps[m];
  }
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, j->ev_start, j->ev_kernel);
    stats->kernel_ms = ms;
    stats->total_steps = total_steps;
    stats->cell_updates = total_steps * j->cells;
  }
  return GRN_OK;
}

}  // namespace

extern "C" {

int grn_abi_version(void) { return GRN_ABI_VERSION; }

const char *grn_status_str(grn_status s) {
  switch (s) {
    case GRN_OK: return "GRN_OK";
    case GRN_ERR_INVALID_ARGUMENT: return "GRN_ERR_INVALID_ARGUMENT";
    case GRN_ERR_NO_DEVICE: return "GRN_ERR_NO_DEVICE";
    case GRN_ERR_CUDA: return "GRN_ERR_CUDA";
    case GRN_ERR_OUT_OF_MEMORY: return "GRN_ERR_OUT_OF_MEMORY";
    case GRN_ERR_MODEL: return "GRN_ERR_MODEL";
    case GRN_ERR_CAPACITY: return "GRN_ERR_CAPACITY";
    case GRN_ERR_NO_EXPERIMENTS: return "GRN_ERR_NO_EXPERIMENTS";
    case GRN_ERR_TIMEOUT: return "GRN_ERR_TIMEOUT";
    case GRN_ERR_NOT_FOUND: return "GRN_ERR_NOT_FOUND";
    case GRN_ERR_KERNEL: return "GRN_ERR_KERNEL";
  }
  return "GRN_ERR_UNKNOWN";
}

const char *grn_last_error(const grn_ctx *ctx) {
  return ctx ? ctx->last_error.c_str() : "";
}

double grn_round_error(double raw, double max_error, int precision) {
  // CEvaluatorMorphogens::evaluate + MathAlgo::ceilS (Src/Common/mathalgo.h:55-62).
  if (raw > max_error) return 100;
  if (raw == 0.0) return 0.0;
  const double factor = std::pow(10.0, precision - std::ceil(std::log10(std::fabs(raw))));
  return std::ceil(raw * factor) / factor;
}

grn_status grn_create(grn_ctx **out, int device, const grn_sim_params *params) {
  if (!out) return GRN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  grn_status s = check_params(params);
  if (s != GRN_OK) return s;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev < 1) {
    cudaGetLastError();
    return GRN_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n_dev) return GRN_ERR_NO_DEVICE;
  grn_ctx *ctx = new (std::nothrow) grn_ctx();
  if (!ctx) return GRN_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  ctx->p = *params;
  auto bail = [&](grn_status st) {
    grn_destroy(ctx);
    return st;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bail(GRN_ERR_NO_DEVICE);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(GRN_ERR_CUDA);
  cudaDeviceGetAttribute(&ctx->n_sm, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&ctx->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (ensure_dev(ctx, &ctx->d_counter, 16) != GRN_OK) return bail(GRN_ERR_OUT_OF_MEMORY);
  *out = ctx;
  return GRN_OK;
}

grn_status grn_destroy(grn_ctx *ctx) {
  if (!ctx) return GRN_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (Job *j : ctx->pending) {
    free_job(j);
    delete j;
  }
  for (Job *j : ctx->free_jobs) {
    free_job(j);
    delete j;
  }
  free_job(&ctx->sync_job);
  for (DevBuf *b : {&ctx->d_initial, &ctx->d_target, &ctx->d_counter, &ctx->d_gstate,
                    &ctx->d_sample, &ctx->d_packed_flag})
    if (b->p) cudaFree(b->p);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return GRN_OK;
}

static_assert(grn::kHookWithholdBandCopy == GRN_TEST_WITHHOLD_BAND_COPY, "test hook bits");

grn_status grn_autotune_report(const grn_ctx *ctx, char *buf, int buf_len) {
  if (!ctx || !buf || buf_len < 1) return GRN_ERR_INVALID_ARGUMENT;
  char head[96];
  std::snprintf(head, sizeof head, "# autotuning runs %d, %.1f ms in all; the last one:\n",
                ctx->n_tunings, ctx->tuning_ms);
  const std::string rep = head + ctx->last_tuning;
  std::snprintf(buf, (size_t)buf_len, "%s", rep.c_str());
  return (int)rep.size() < buf_len ? GRN_OK : GRN_ERR_CAPACITY;
}

grn_status grn_set_test_hooks(grn_ctx *ctx, int hooks) {
  if (!ctx || (hooks & ~(GRN_TEST_WITHHOLD_BAND_COPY | GRN_TEST_FAIL_DEVICE_ALLOC |
                         GRN_TEST_CORRUPT_RECORD)))
    return GRN_ERR_INVALID_ARGUMENT;
  ctx->test_hooks = hooks;
  return GRN_OK;
}

grn_status grn_set_host_threads(grn_ctx *ctx, int n_threads) {
  if (!ctx || n_threads < 0) return GRN_ERR_INVALID_ARGUMENT;
  ctx->host_threads = n_threads;
  return GRN_OK;
}

grn_status grn_set_graphs(grn_ctx *ctx, int enable) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  ctx->graphs = enable != 0;
  return GRN_OK;
}

grn_status grn_set_autotune(grn_ctx *ctx, int enable) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  ctx->autotune = enable != 0;
  ctx->tuned.clear();
  return GRN_OK;
}

grn_status grn_set_cluster_size(grn_ctx *ctx, int cluster_size) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (cluster_size != 0 && cluster_size != 2 && cluster_size != 4 && cluster_size != 8 &&
      cluster_size != 16)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "cluster size must be 0, 2, 4, 8 or 16");
  ctx->forced_cluster = cluster_size;
  return GRN_OK;
}

grn_status grn_set_schedule(grn_ctx *ctx, int schedule, int threads_per_block) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (schedule < GRN_SCHEDULE_AUTO || schedule > GRN_SCHEDULE_STREAM2 || threads_per_block < 0)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "bad schedule");
  ctx->forced_schedule = schedule;
  ctx->forced_threads = threads_per_block;
  return GRN_OK;
}

grn_status grn_set_experiments(grn_ctx *ctx, int n_experiments, const double *initial,
                               const double *target) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (n_experiments < 1 || n_experiments > GRN_MAX_EXPERIMENTS || !initial || !target)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "bad experiments");
  cudaSetDevice(ctx->device);
  const size_t plane = (size_t)ctx->p.dim_x * ctx->p.dim_y;
  const size_t ni = n_experiments * ctx->p.n_input_morphogens * plane;
  const size_t nt = n_experiments * ctx->p.n_target_morphogens * plane;
  std::vector<float> fi(ni), ft(nt);
  for (size_t i = 0; i < ni; ++i) fi[i] = (float)initial[i];
  for (size_t i = 0; i < nt; ++i) ft[i] = (float)target[i];
  grn_status s;
  if ((s = ensure_dev(ctx, &ctx->d_initial, std::max<size_t>(ni, 1) * sizeof(float))) ||
      (s = ensure_dev(ctx, &ctx->d_target, std::max<size_t>(nt, 1) * sizeof(float))))
    return s;
  if (ni) GRN_CUDA(ctx, cudaMemcpyAsync(ctx->d_initial.p, fi.data(), ni * sizeof(float),
                                        cudaMemcpyHostToDevice, ctx->stream));
  if (nt) GRN_CUDA(ctx, cudaMemcpyAsync(ctx->d_target.p, ft.data(), nt * sizeof(float),
                                        cudaMemcpyHostToDevice, ctx->stream));
  GRN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->n_exp = n_experiments;
  // The fast path's bound on the state (the kernel's euler_bounded) also
  // needs the initial values below kFastMaxInitial.
  constexpr double kFastMaxInitial = 1.0e6;
  bool ok = ctx->p.min_conc == 0.0;
  for (size_t i = 0; ok && i < ni; ++i) {
    const double v = fi[i];  // the value the kernel starts from
    ok = std::isfinite(v) && v >= 0 && v <= kFastMaxInitial;
  }
  ctx->fast_ok = ok;
  return GRN_OK;
}

grn_status grn_decode_rgb(int dim_x, int dim_y, int n_channels, const uint32_t *pixels,
                          double *out) {
  if (dim_x < 1 || dim_y < 1 || n_channels < 0 || n_channels > 3 || !pixels || !out)
    return GRN_ERR_INVALID_ARGUMENT;
  // SimState::loadMorphologyImage (Src/Simulator/simstate.cpp:71-90):
  // scanline j fills row H-1-j; channel k is byte (16 - 8k) of 0xAARRGGBB.
  const size_t plane = (size_t)dim_x * dim_y;
  for (int j = 0; j < dim_y; ++j)
    for (int i = 0; i < dim_x; ++i) {
      const uint32_t color = pixels[(size_t)j * dim_x + i];
      for (int k = 0; k < n_channels; ++k)
        out[k * plane + (size_t)(dim_y - j - 1) * dim_x + i] =
            (double)((color >> (16 - 8 * k)) & 0xffu) / 255.0;
    }
  return GRN_OK;
}

grn_status grn_set_experiments_rgb(grn_ctx *ctx, int n_experiments, const uint32_t *input_pixels,
                                   const uint32_t *target_pixels) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (n_experiments < 1 || n_experiments > GRN_MAX_EXPERIMENTS || !input_pixels || !target_pixels)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "bad experiments");
  const int W = ctx->p.dim_x, H = ctx->p.dim_y;
  const int ni = ctx->p.n_input_morphogens, nt = ctx->p.n_target_morphogens;
  const size_t plane = (size_t)W * H;
  std::vector<double> init((size_t)n_experiments * ni * plane), tgt((size_t)n_experiments * nt * plane);
  for (int e = 0; e < n_experiments; ++e) {
    grn_decode_rgb(W, H, ni, input_pixels + e * plane, init.data() + e * ni * plane);
    grn_decode_rgb(W, H, nt, target_pixels + e * plane, tgt.data() + e * nt * plane);
  }
  return grn_set_experiments(ctx, n_experiments, init.data(), tgt.data());
}

grn_status grn_evaluate_batch(grn_ctx *ctx, const grn_model_batch *batch, const double *max_error,
                              double *error_out, double *raw_error_out, grn_eval_stats *stats) {
  grn::TraceRange trace_range("grn_evaluate_batch");
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (!error_out && !raw_error_out)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "no output buffer");
  cudaSetDevice(ctx->device);
  grn_status s = enqueue_job(ctx, &ctx->sync_job, batch, max_error, stats);
  if (s != GRN_OK) return s;
  if (batch->n_models == 0) return GRN_OK;
  GRN_CUDA(ctx, cudaEventSynchronize(ctx->sync_job.ev_done));
  return finish_job(ctx, &ctx->sync_job, max_error, error_out, raw_error_out, stats);
}

grn_status grn_evaluate_states(grn_ctx *ctx, const grn_model_batch *batch, const double *max_error,
                               double *raw_error_out, float *states_out, int max_planes) {
  grn::TraceRange trace_range("grn_evaluate_states");
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  grn_status s = check_batch(ctx, batch);
  if (s != GRN_OK) return s;
  if (!max_error || !states_out || max_planes < 1)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "bad states request");
  if (ctx->n_exp < 1) return fail(ctx, GRN_ERR_NO_EXPERIMENTS, "no experiments uploaded");
  const int n = batch->n_models;
  if (n == 0) return GRN_OK;
  cudaSetDevice(ctx->device);
  PackedHost ph;
  std::string err;
  s = grn::pack_batch(batch, ctx->p.n_input_morphogens + ctx->p.n_target_morphogens,
                      (float)ctx->p.dt, ctx->p.num_sim_steps,
                      host_threads(ctx), &ph, &err);
  if (s != GRN_OK) return fail(ctx, s, err);
  Job &j = ctx->sync_job;
  const size_t wb = ph.words.size() * sizeof(uint4), ob = n * sizeof(int32_t);
  const size_t eb = n * sizeof(double);
  const size_t sb = (size_t)n * ctx->n_exp * max_planes * ctx->p.dim_x * ctx->p.dim_y * sizeof(float);
  DevBuf d_states;
  if ((s = ensure_dev(ctx, &j.d_words, wb)) || (s = ensure_dev(ctx, &j.d_offsets, ob)) ||
      (s = ensure_dev(ctx, &j.d_maxerr, eb)) || (s = ensure_dev(ctx, &j.d_raw, eb)) ||
      (s = ensure_dev(ctx, &j.d_steps, ob)) || (s = ensure_dev(ctx, &j.d_flag, 4)) ||
      (s = ensure_dev(ctx, &d_states, sb)))
    return s;
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  chk(cudaMemcpyAsync(j.d_words.p, ph.words.data(), wb, cudaMemcpyHostToDevice, st));
  chk(cudaMemcpyAsync(j.d_offsets.p, ph.offsets.data(), ob, cudaMemcpyHostToDevice, st));
  chk(cudaMemcpyAsync(j.d_maxerr.p, max_error, eb, cudaMemcpyHostToDevice, st));
  chk(cudaMemsetAsync(j.d_flag.p, 0, 4, st));
  chk(cudaMemsetAsync(d_states.p, 0, sb, st));
  if (e == cudaSuccess) {
    s = launch_packed(ctx, static_cast<const uint4 *>(j.d_words.p),
                      static_cast<const int32_t *>(j.d_offsets.p), n, ph.max_genes, ph.max_links,
                      static_cast<const double *>(j.d_maxerr.p), static_cast<double *>(j.d_raw.p),
                      static_cast<int32_t *>(j.d_steps.p), static_cast<int32_t *>(j.d_flag.p), st,
                      nullptr, [&] {
                        LaunchExtras x;
                        x.states = static_cast<float *>(d_states.p);
                        x.state_planes = max_planes;
                        x.host_offsets = ph.offsets.data();
                        return x;
                      }());
    int32_t flag = 0;
    chk(cudaMemcpyAsync(states_out, d_states.p, sb, cudaMemcpyDeviceToHost, st));
    if (raw_error_out) chk(cudaMemcpyAsync(raw_error_out, j.d_raw.p, eb, cudaMemcpyDeviceToHost, st));
    chk(cudaMemcpyAsync(&flag, j.d_flag.p, 4, cudaMemcpyDeviceToHost, st));
    chk(cudaStreamSynchronize(st));
    if (s == GRN_OK && e == cudaSuccess && flag)
      s = kernel_flag_error(ctx, flag);
  }
  cudaFree(d_states.p);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "grn_evaluate_states");
  return s;
}

grn_status grn_evaluate(grn_ctx *ctx, const grn_product *products, int n_products,
                        const grn_link *links, int n_links, double max_error, double *error_out) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (!error_out || n_products < 0 || n_links < 0 || (n_products && !products) ||
      (n_links && !links))
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "bad model");
  const int32_t po[2] = {0, n_products}, lo[2] = {0, n_links};
  grn_model_batch b{};
  b.n_models = 1;
  b.product_offsets = po;
  b.products = products;
  b.link_offsets = lo;
  b.links = links;
  return grn_evaluate_batch(ctx, &b, &max_error, error_out, nullptr, nullptr);
}

grn_status grn_submit(grn_ctx *ctx, int tag, const grn_model_batch *batch, const double *max_error,
                      double *error_out, double *raw_error_out) {
  grn::TraceRange trace_range("grn_submit");
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (!error_out && !raw_error_out)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "no output buffer");
  cudaSetDevice(ctx->device);
  Job *j;
  if (!ctx->free_jobs.empty()) {
    j = ctx->free_jobs.back();
    ctx->free_jobs.pop_back();
  } else {
    j = new (std::nothrow) Job();
    if (!j) return fail(ctx, GRN_ERR_OUT_OF_MEMORY, "job");
  }
  grn_status s = enqueue_job(ctx, j, batch, max_error, nullptr);
  if (s != GRN_OK) {
    ctx->free_jobs.push_back(j);
    return s;
  }
  j->tag = tag;
  j->error_out = error_out;
  j->raw_out = raw_error_out;
  j->max_error.assign(max_error, max_error + batch->n_models);
  ctx->pending.push_back(j);
  return GRN_OK;
}

grn_status grn_wait_any(grn_ctx *ctx, int timeout_ms, int *tag_out) {
  grn::TraceRange trace_range("grn_wait_any");
  if (!ctx || !tag_out) return GRN_ERR_INVALID_ARGUMENT;
  if (ctx->pending.empty()) return fail(ctx, GRN_ERR_NOT_FOUND, "nothing submitted");
  cudaSetDevice(ctx->device);
  auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    for (auto it = ctx->pending.begin(); it != ctx->pending.end(); ++it) {
      Job *j = *it;
      cudaError_t q = j->n_models ? cudaEventQuery(j->ev_done) : cudaSuccess;
      if (q == cudaErrorNotReady) continue;
      ctx->pending.erase(it);
      ctx->free_jobs.push_back(j);
      if (q != cudaSuccess) return cuda_fail(ctx, q, "cudaEventQuery");
      *tag_out = j->tag;
      return finish_job(ctx, j, j->max_error.data(), j->error_out, j->raw_out, nullptr);
    }
    if (timeout_ms >= 0) {
      auto el = std::chrono::steady_clock::now() - t0;
      if (std::chrono::duration<double, std::milli>(el).count() >= timeout_ms)
        return fail(ctx, GRN_ERR_TIMEOUT, "no submitted batch finished in time");
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

grn_status grn_pack(grn_ctx *ctx, const grn_model_batch *batch, grn_packed **out) {
  grn::TraceRange trace_range("grn_pack");
  if (!ctx || !out) return GRN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  grn_status s = check_batch(ctx, batch);
  if (s != GRN_OK) return s;
  cudaSetDevice(ctx->device);
  grn_packed *pk = new (std::nothrow) grn_packed();
  if (!pk) return fail(ctx, GRN_ERR_OUT_OF_MEMORY, "packed");
  pk->ctx = ctx;
  std::string err;
  s = grn::pack_batch(batch, ctx->p.n_input_morphogens + ctx->p.n_target_morphogens,
                      (float)ctx->p.dt, ctx->p.num_sim_steps,
                      host_threads(ctx), &pk->host, &err);
  if (s != GRN_OK) {
    delete pk;
    return fail(ctx, s, err);
  }
  const size_t wb = std::max<size_t>(pk->host.words.size(), 1) * sizeof(uint4);
  const size_t ob = std::max<size_t>(pk->host.offsets.size(), 1) * sizeof(int32_t);
  if ((s = ensure_dev(ctx, &pk->d_words, wb)) || (s = ensure_dev(ctx, &pk->d_offsets, ob))) {
    grn_packed_free(pk);
    return s;
  }
  if (!pk->host.words.empty()) {
    cudaMemcpy(pk->d_words.p, pk->host.words.data(), pk->host.words.size() * sizeof(uint4),
               cudaMemcpyHostToDevice);
    cudaError_t e = cudaMemcpy(pk->d_offsets.p, pk->host.offsets.data(),
                               pk->host.offsets.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      grn_packed_free(pk);
      return cuda_fail(ctx, e, "cudaMemcpy packed");
    }
  }
  pk->cell_bound = (int64_t)batch->n_models * std::max(ctx->n_exp, 1) * ctx->p.num_sim_steps *
                   ctx->p.dim_x * ctx->p.dim_y;
  *out = pk;
  return GRN_OK;
}

grn_status grn_packed_free(grn_packed *pk) {
  if (!pk) return GRN_OK;
  if (pk->ctx) cudaSetDevice(pk->ctx->device);
  if (pk->d_words.p) cudaFree(pk->d_words.p);
  if (pk->d_offsets.p) cudaFree(pk->d_offsets.p);
  delete pk;
  return GRN_OK;
}

grn_status grn_packed_get_info(const grn_packed *pk, grn_packed_info *info) {
  if (!pk || !info) return GRN_ERR_INVALID_ARGUMENT;
  std::memset(info, 0, sizeof *info);
  const PackedHost &h = pk->host;
  info->n_models = h.n_models;
  info->device_bytes = (int64_t)(h.words.size() * sizeof(uint4) + h.offsets.size() * 4);
  info->cell_update_bound = pk->cell_bound;
  const int64_t cells = (int64_t)pk->ctx->p.dim_x * pk->ctx->p.dim_y;
  info->sfu_ops_per_step = h.sfu_per_cell_step * cells;
  info->max_genes = h.max_genes;
  info->max_links = h.max_links;
  info->mean_genes = h.n_models ? h.sum_genes / h.n_models : 0;
  info->mean_links = h.n_models ? h.sum_links / h.n_models : 0;
  info->mean_dif_genes = h.n_models ? h.sum_dif_genes / h.n_models : 0;
  info->alg_sfu_ops_per_step = h.alg_sfu_per_cell_step * cells;
  info->alg_fp32_ops_per_step = h.alg_fp32_per_cell_step * cells;
  return GRN_OK;
}

grn_status grn_trace_model(grn_ctx *ctx, const grn_product *products, int n_products,
                           const grn_link *links, int n_links, int experiment, int every,
                           int max_frames, int max_planes, float *frames_out, int *n_frames,
                           int32_t *labels_out) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (n_products < 0 || n_links < 0 || (n_products && !products) || (n_links && !links) ||
      every < 1 || max_frames < 1 || max_planes < 1 || !frames_out || !n_frames)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "bad trace arguments");
  if (ctx->n_exp < 1) return fail(ctx, GRN_ERR_NO_EXPERIMENTS, "no experiments uploaded");
  if (experiment < 0 || experiment >= ctx->n_exp)
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "no such experiment");
  cudaSetDevice(ctx->device);
  const int n_morph = ctx->p.n_input_morphogens + ctx->p.n_target_morphogens;
  int32_t po[2] = {0, n_products}, lo[2] = {0, n_links};
  grn_model_batch b{};
  b.n_models = 1;
  b.product_offsets = po;
  b.products = products;
  b.link_offsets = lo;
  b.links = links;
  PackedHost ph;
  std::string err;
  grn_status s =
      grn::pack_batch(&b, n_morph, (float)ctx->p.dt, ctx->p.num_sim_steps, 1, &ph, &err);
  if (s != GRN_OK) return fail(ctx, s, err);
  const size_t cells = (size_t)ctx->p.dim_x * ctx->p.dim_y;
  const size_t fb = (size_t)max_frames * max_planes * cells * sizeof(float);
  Job &j = ctx->sync_job;
  DevBuf d_trace;
  const size_t wb = ph.words.size() * sizeof(uint4);
  if ((s = ensure_dev(ctx, &j.d_words, wb)) || (s = ensure_dev(ctx, &j.d_offsets, 4)) ||
      (s = ensure_dev(ctx, &j.d_maxerr, 8)) || (s = ensure_dev(ctx, &j.d_raw, 8)) ||
      (s = ensure_dev(ctx, &j.d_steps, 4)) || (s = ensure_dev(ctx, &j.d_flag, 4)) ||
      (s = ensure_dev(ctx, &d_trace, fb)))
    return s;
  cudaStream_t st = ctx->stream;
  const double never = 1e300;  // no abandon
  int32_t steps = 0, flag = 0;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  chk(cudaMemcpyAsync(j.d_words.p, ph.words.data(), wb, cudaMemcpyHostToDevice, st));
  chk(cudaMemcpyAsync(j.d_offsets.p, ph.offsets.data(), 4, cudaMemcpyHostToDevice, st));
  chk(cudaMemcpyAsync(j.d_maxerr.p, &never, 8, cudaMemcpyHostToDevice, st));
  chk(cudaMemsetAsync(j.d_flag.p, 0, 4, st));
  chk(cudaMemsetAsync(d_trace.p, 0, fb, st));
  if (e == cudaSuccess) {
    LaunchExtras x;
    x.state_planes = max_planes;
    x.trace = static_cast<float *>(d_trace.p);
    x.trace_every = every;
    x.trace_frames = max_frames;
    x.experiment = experiment;
    s = launch_packed(ctx, static_cast<const uint4 *>(j.d_words.p),
                      static_cast<const int32_t *>(j.d_offsets.p), 1, ph.max_genes, ph.max_links,
                      static_cast<const double *>(j.d_maxerr.p), static_cast<double *>(j.d_raw.p),
                      static_cast<int32_t *>(j.d_steps.p), static_cast<int32_t *>(j.d_flag.p), st,
                      nullptr, x);
    chk(cudaMemcpyAsync(frames_out, d_trace.p, fb, cudaMemcpyDeviceToHost, st));
    chk(cudaMemcpyAsync(&steps, j.d_steps.p, 4, cudaMemcpyDeviceToHost, st));
    chk(cudaMemcpyAsync(&flag, j.d_flag.p, 4, cudaMemcpyDeviceToHost, st));
    chk(cudaStreamSynchronize(st));
  }
  cudaFree(d_trace.p);
  if (s != GRN_OK) return s;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "trace");
  if (flag) return kernel_flag_error(ctx, flag);
  *n_frames = std::min(max_frames, steps / every + 1);
  if (labels_out) {
    const std::vector<int> labels = grn::labels_in_use(links, n_links, n_morph);
    for (int i = 0; i < max_planes; ++i)
      labels_out[i] = i < (int)labels.size() ? labels[i] : -1;
  }
  return GRN_OK;
}

grn_status grn_run_packed(grn_ctx *ctx, const grn_packed *pk, const double *d_max_error,
                          double *d_raw_error, int32_t *d_steps, void *cuda_stream) {
  grn::TraceRange trace_range("grn_run_packed");
  if (!ctx || !pk || pk->ctx != ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (pk->host.n_models > 0 && (!d_max_error || !d_raw_error))
    return fail(ctx, GRN_ERR_INVALID_ARGUMENT, "null device pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->stream;
  if (!ctx->d_packed_flag.p) {
    // The flag starts at 0 and stays set until grn_run_packed_status reads it.
    grn_status s = ensure_dev(ctx, &ctx->d_packed_flag, 4);
    if (s != GRN_OK) return s;
    GRN_CUDA(ctx, cudaMemsetAsync(ctx->d_packed_flag.p, 0, 4, st));
  }
  LaunchExtras ex;
  ex.host_offsets = pk->host.offsets.data();
  return launch_packed(ctx, static_cast<const uint4 *>(pk->d_words.p),
                       static_cast<const int32_t *>(pk->d_offsets.p), pk->host.n_models,
                       pk->host.max_genes, pk->host.max_links, d_max_error, d_raw_error, d_steps,
                       static_cast<int32_t *>(ctx->d_packed_flag.p), st, nullptr, ex);
}

grn_status grn_run_packed_status(grn_ctx *ctx, void *cuda_stream) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  if (!ctx->d_packed_flag.p) return GRN_OK;  // nothing launched yet
  cudaSetDevice(ctx->device);
  cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->stream;
  int32_t flag = 0;
  GRN_CUDA(ctx, cudaMemcpyAsync(&flag, ctx->d_packed_flag.p, 4, cudaMemcpyDeviceToHost, st));
  GRN_CUDA(ctx, cudaMemsetAsync(ctx->d_packed_flag.p, 0, 4, st));
  GRN_CUDA(ctx, cudaStreamSynchronize(st));
  return flag != 0 ? kernel_flag_error(ctx, flag) : GRN_OK;
}

}  // extern "C"

extern "C" grn_status grn_model_costs(const grn_model_batch *batch, int n_morphogens,
                                      double *cost_out) {
  if (!batch || !cost_out || batch->n_models < 0 || n_morphogens < 0 ||
      (batch->n_models > 0 && (!batch->product_offsets || !batch->link_offsets)))
    return GRN_ERR_INVALID_ARGUMENT;
  for (int m = 0; m < batch->n_models; ++m) {
    const int p0 = batch->product_offsets[m], p1 = batch->product_offsets[m + 1];
    const int l0 = batch->link_offsets[m], l1 = batch->link_offsets[m + 1];
    if (p1 < p0 || l1 < l0) return GRN_ERR_INVALID_ARGUMENT;
    std::vector<uint4> rec;
    grn::ModelCost cost;
    std::string err;
    const grn_status s = grn::pack_model(batch->products + p0, p1 - p0, batch->links + l0,
                                         l1 - l0, n_morphogens, m, &rec, &cost, &err);
    if (s != GRN_OK) return s;
    cost_out[m] = cost.cost;
  }
  return GRN_OK;
}

extern "C" grn_status grn_describe_model(const grn_product *products, int n_products,
                                         const grn_link *links, int n_links, int n_morphogens,
                                         char *buf, int buf_len) {
  if (!buf || buf_len < 1 || n_products < 0 || n_links < 0 || (n_products && !products) ||
      (n_links && !links) || n_morphogens < 0)
    return GRN_ERR_INVALID_ARGUMENT;
  std::vector<uint4> rec;
  grn::ModelCost cost;
  std::string err;
  grn_status s = grn::pack_model(products, n_products, links, n_links, n_morphogens, 0, &rec,
                                 &cost, &err);
  if (s != GRN_OK) return s;
  grn::PackedHeader hdr;
  std::memcpy(&hdr, rec.data(), sizeof hdr);
  std::string out;
  char line[256];
  std::snprintf(line, sizeof line, "model genes %d links %d lg_mask %u\n", hdr.n_genes,
                hdr.n_links, hdr.lg_mask);
  out += line;
  const std::vector<int> labels = grn::labels_in_use(links, n_links, n_morphogens);
  for (int i = 0; i < hdr.n_genes; ++i) {
    grn::PackedGene g;
    std::memcpy(&g, rec.data() + 1 + i, sizeof g);
    std::snprintf(line, sizeof line, "gene %d label %d lim %.9g deg %.9g dif %.9g or %d and %d\n",
                  i, labels[i], g.lim, g.deg, g.dif, g.n_or, g.n_and);
    out += line;
    for (int l = 0; l < g.n_or + g.n_and; ++l) {
      grn::PackedLink k;
      std::memcpy(&k, rec.data() + 1 + hdr.n_genes + g.link_begin + l, sizeof k);
      std::snprintf(line, sizeof line, "link %d slot %d a %.9g b %.9g\n", i, k.slot, k.a, k.b);
      out += line;
    }
  }
  if ((int)out.size() + 1 > buf_len) return GRN_ERR_CAPACITY;
  std::memcpy(buf, out.c_str(), out.size() + 1);
  return GRN_OK;
}
