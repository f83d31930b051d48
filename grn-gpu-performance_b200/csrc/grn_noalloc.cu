// grn_noalloc.cu -- grn_evaluate_batch_noalloc: batch evaluation that
// allocates no device memory.
//
// Some callers cannot allocate GPU memory: a host application that has
// already divided the whole device memory among its components and hands
// this library only the buffers it owns, or a long-running search loop that
// must never block in, or fail out of, the device allocator halfway through
// a run.  For them this entry point runs the same simulation kernel as
// grn_evaluate_batch, but everything the kernel needs beyond the caller's
// inputs and outputs -- the work counter, the error flag, the compiled model
// records and the per-block state slots of genes that do not fit in shared
// memory -- lives in one file-scope device array of GRN_NOALLOC_SCRATCH_BYTES.
// The array is reserved on a GPU when this module is loaded there; with
// CUDA's lazy module loading (the default) that is the first call on that
// device, which looks the array's address up.  A caller that divides the
// device memory itself should make that first call (a call with no models
// is enough) before it does.
//
// The array is shared by every call on a device and keeps the previous
// call's contents; each call clears the counter and flag it relies on (the
// kernel itself initialises every state plane before use).  Two calls whose
// work overlaps on the GPU (different streams, or one enqueued before the
// previous one finished on another stream) race on the array.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "../../include/grn_gpu.h"
#include "../host/pack.h"
#include "grn_sim.h"

namespace grn {
namespace {

// Reserved on each GPU when the module loads there, for the life of the
// process.
static __device__ __align__(256) unsigned char g_noalloc_scratch[GRN_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side stand-in; the address comes from
// cudaGetSymbolAddress, looked up once per device with that device current.
cudaError_t scratch_address(int device, void **out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// The scratch array starts with the kernel's work counter and error flag.
constexpr size_t kFlagOffset = sizeof(int32_t);

grn_status cuda_status(cudaError_t e) {
  return e == cudaErrorMemoryAllocation ? GRN_ERR_OUT_OF_MEMORY : GRN_ERR_CUDA;
}

grn_status put_error(char *buf, int len, grn_status s, const std::string &msg) {
  if (buf && len > 0) {
    std::snprintf(buf, (size_t)len, "%s", msg.c_str());
  }
  return s;
}

}  // namespace
}  // namespace grn

extern "C" grn_status grn_evaluate_batch_noalloc(
    const grn_sim_params *params, int n_experiments, const float *d_initial,
    const float *d_target, const grn_model_batch *batch, const double *d_max_error,
    double *d_raw_error, int32_t *d_steps, void *cuda_stream, char *err_buf, int err_buf_len) {
  using namespace grn;
  if (err_buf && err_buf_len > 0) err_buf[0] = '\0';
  if (!params || !batch || batch->n_models < 0 || n_experiments < 1 ||
      n_experiments > GRN_MAX_EXPERIMENTS || (batch->n_models > 0 && (!d_max_error || !d_raw_error)) ||
      (params->n_input_morphogens > 0 && !d_initial) || (params->n_target_morphogens > 0 && !d_target))
    return put_error(err_buf, err_buf_len, GRN_ERR_INVALID_ARGUMENT, "null or out-of-range argument");
  if (params->dim_x < 1 || params->dim_y < 1 || params->num_sim_steps < 0 ||
      params->n_input_morphogens < 0 || params->n_input_morphogens > GRN_MAX_INPUT_MORPHOGENS ||
      params->n_target_morphogens < 0 || params->n_target_morphogens > 3 ||
      (params->fitness_kind != GRN_FITNESS_REF_LOGTHRESH && params->fitness_kind != GRN_FITNESS_MSE))
    return put_error(err_buf, err_buf_len, GRN_ERR_INVALID_ARGUMENT, "bad simulation parameters");

  // Set-up first, even for an empty batch: looking the array up loads the
  // module, which reserves the array on this device.
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
    return put_error(err_buf, err_buf_len, GRN_ERR_NO_DEVICE, "no current CUDA device");
  void *scratch = nullptr;
  cudaError_t e = scratch_address(device, &scratch);
  if (e != cudaSuccess)
    return put_error(err_buf, err_buf_len, cuda_status(e),
                     std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  if (batch->n_models == 0) return GRN_OK;
  if (!batch->product_offsets || !batch->link_offsets || batch->product_offsets[0] != 0 ||
      batch->link_offsets[0] != 0)
    return put_error(err_buf, err_buf_len, GRN_ERR_INVALID_ARGUMENT, "bad batch offsets");

  // Compile the batch on the host (host memory only).
  PackedHost ph;
  std::string perr;
  unsigned hw = std::thread::hardware_concurrency();
  grn_status s = pack_batch(batch, params->n_input_morphogens + params->n_target_morphogens,
                            (float)params->dt, params->num_sim_steps, hw ? (int)hw : 1, &ph,
                            &perr);
  if (s != GRN_OK) return put_error(err_buf, err_buf_len, s, perr);

  // Scratch layout: [counter, flag] | records | offsets | state slots.
  const size_t words_off = 256;
  const size_t words_bytes = ph.words.size() * sizeof(uint4);
  const size_t offs_off = align_up(words_off + words_bytes, 256);
  const size_t offs_bytes = ph.offsets.size() * sizeof(int32_t);
  const size_t slots_off = align_up(offs_off + offs_bytes, 256);
  if (slots_off > (size_t)GRN_NOALLOC_SCRATCH_BYTES)
    return put_error(err_buf, err_buf_len, GRN_ERR_CAPACITY,
                     "compiled batch needs " + std::to_string(slots_off) +
                         " bytes of scratch, more than GRN_NOALLOC_SCRATCH_BYTES (" +
                         std::to_string((long long)GRN_NOALLOC_SCRATCH_BYTES) + ")");

  // Kernel variant: fixed items when the grid fits a block's threads, state
  // planes in shared memory as far as they fit, by occupancy.
  int n_sm = 0, optin = 0;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  const int W = params->dim_x, H = params->dim_y, Wg = (W + 3) / 4, Q = H * Wg;
  const bool ragged = (W % 4) != 0;
  const size_t plane_bytes = (size_t)plane_floats(W, H) * sizeof(float);
  const size_t fixed = sim_fixed_smem_bytes();
  int fit = (size_t)optin > fixed ? (int)(((size_t)optin - fixed) / plane_bytes) : 0;
  fit &= ~1;
  const int gmax = ph.max_genes;
  LaunchPlan best{};
  best.cluster = 1;
  double best_score = -1;
  for (int i = 0; i < sim_variant_count(); ++i) {
    const KernelVariant v = sim_variant(i);
    if (v.cluster || v.trace || v.stream || v.gmax < gmax || v.ragged != ragged || (!v.loop && Q > v.threads * v.items))
      continue;
    const int planes = std::min(fit, 2 * gmax);
    const size_t smem = fixed + planes * plane_bytes;
    int occ = 0;
    if (sim_occupancy(v, smem, &occ) != cudaSuccess || occ < 1) continue;
    const double score = (double)occ * std::min(v.threads, Q) * (v.loop ? 1.0 : 1.25) - 1e-3 * v.gmax;
    if (score > best_score) {
      best_score = score;
      best.v = v;
      best.schedule = v.loop ? GRN_SCHEDULE_WALK_ITEMS : GRN_SCHEDULE_FIXED_ITEMS;
      best.planes = planes;
      best.smem_bytes = smem;
      best.blocks_per_sm = occ;
      best.slot_floats = planes / 2 < gmax ? 2LL * v.gmax * plane_floats(W, H) : 0;
    }
  }
  if (best_score < 0)
    return put_error(err_buf, err_buf_len, GRN_ERR_CAPACITY,
                     "no kernel variant holds " + std::to_string(gmax) + " genes on this grid");
  int blocks = std::max(1, std::min(batch->n_models, n_sm * best.blocks_per_sm));
  if (best.slot_floats > 0) {
    // As many persistent blocks as the scratch has state slots for.
    const size_t slot_bytes = (size_t)best.slot_floats * sizeof(float);
    const size_t room = (size_t)GRN_NOALLOC_SCRATCH_BYTES - slots_off;
    const size_t n_slots = room / slot_bytes;
    if (n_slots < 1)
      return put_error(err_buf, err_buf_len, GRN_ERR_CAPACITY,
                       "one block's state slot needs " + std::to_string(slot_bytes) +
                           " bytes, more than the " + std::to_string(room) +
                           " bytes left of GRN_NOALLOC_SCRATCH_BYTES");
    blocks = std::min<int>(blocks, (int)std::min<size_t>(n_slots, 1 << 20));
  }
  best.blocks = blocks;

  unsigned char *base = static_cast<unsigned char *>(scratch);
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  // Pageable source buffers: each copy has read its source when it returns.
  e = cudaMemcpyAsync(base + words_off, ph.words.data(), words_bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + offs_off, ph.offsets.data(), offs_bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(base, 0, 2 * sizeof(int32_t), st);  // counter, flag
  if (e != cudaSuccess)
    return put_error(err_buf, err_buf_len, cuda_status(e),
                     std::string("copy into scratch: ") + cudaGetErrorString(e));

  SimArgs a{};
  a.packed = reinterpret_cast<const uint4 *>(base + words_off);
  a.offsets = reinterpret_cast<const int32_t *>(base + offs_off);
  a.n_models = batch->n_models;
  a.n_exp = n_experiments;
  a.n_in = params->n_input_morphogens;
  a.n_target = params->n_target_morphogens;
  a.W = W;
  a.H = H;
  a.Wg = Wg;
  a.n_steps = params->num_sim_steps;
  a.fitness_kind = params->fitness_kind;
  a.planes = best.planes;
  // Exact arithmetic path only: checking the caller's device-resident
  // initial states for the fast path would need a device pass.
  a.fast_ok = 0;
  a.dt = (float)params->dt;
  a.min_conc = (float)params->min_conc;
  a.min_conc_change = params->min_conc_change;
  a.dist_threshold = params->dist_error_threshold;
  a.initial = d_initial;
  a.target = d_target;
  a.max_error = d_max_error;
  a.raw_error = d_raw_error;
  a.steps = d_steps;
  a.work_counter = reinterpret_cast<int32_t *>(base);
  a.error_flag = reinterpret_cast<int32_t *>(base + kFlagOffset);
  if (best.slot_floats > 0) {
    a.gstate = reinterpret_cast<float *>(base + slots_off);
    a.slot_floats = best.slot_floats;
  }
  e = sim_launch(best, a, st);
  if (e != cudaSuccess)
    return put_error(err_buf, err_buf_len, cuda_status(e),
                     std::string("kernel launch: ") + cudaGetErrorString(e));
  return GRN_OK;
}

extern "C" grn_status grn_evaluate_batch_noalloc_status(void *cuda_stream, char *err_buf,
                                                        int err_buf_len) {
  using namespace grn;
  if (err_buf && err_buf_len > 0) err_buf[0] = '\0';
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
    return put_error(err_buf, err_buf_len, GRN_ERR_NO_DEVICE, "no current CUDA device");
  void *scratch = nullptr;
  cudaError_t e = scratch_address(device, &scratch);
  if (e != cudaSuccess)
    return put_error(err_buf, err_buf_len, cuda_status(e),
                     std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  int32_t flag = 0;
  e = cudaMemcpyAsync(&flag, static_cast<unsigned char *>(scratch) + kFlagOffset, sizeof flag,
                      cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return put_error(err_buf, err_buf_len, cuda_status(e),
                     std::string("reading the error flag: ") + cudaGetErrorString(e));
  if (flag == 0) return GRN_OK;
  return put_error(err_buf, err_buf_len, GRN_ERR_KERNEL,
                   flag == 3   ? "bounds check: a simulation kernel state access fell outside "
                                 "its buffer"
                   : flag == 2 ? "the simulation kernel's wait for a bulk copy timed out"
                               : "the simulation kernel rejected a model record");
}
