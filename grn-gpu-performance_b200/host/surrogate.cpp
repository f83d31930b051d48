// surrogate.cpp -- surrogate fitness model: encoding of GRN models, and the
// host side of training and inference of a 128-256-256-256-1 ReLU MLP whose
// GEMMs run on the tensor cores (csrc/grn_mlp.cu).  It predicts log(error)
// of a model from its compiled program so that the island search can
// simulate only the most promising offspring.  No reference counterpart.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/grn_gpu.h"
#include "../csrc/grn_mlp.h"
#include "pack.h"
#include "trace.h"

namespace {

constexpr int kF = GRN_SURROGATE_FEATURES;  // 128
constexpr int kH = GRN_SURROGATE_HIDDEN;    // 256
// Parameter layout (FP32 master copy; the BF16 mirror has the same layout).
constexpr int64_t kW1 = 0, kB1 = kW1 + (int64_t)kH * kF;
constexpr int64_t kW2 = kB1 + kH, kB2 = kW2 + (int64_t)kH * kH;
constexpr int64_t kW3 = kB2 + kH, kB3 = kW3 + (int64_t)kH * kH;
constexpr int64_t kW4 = kB3 + kH, kB4 = kW4 + kH;
constexpr int64_t kP = kB4 + 1;
static_assert(kP == GRN_SURROGATE_PARAMS, "parameter count");

#define GRN_CK(expr)                                   \
  do {                                                 \
    cudaError_t e__ = (expr);                          \
    if (e__ != cudaSuccess) return GRN_ERR_CUDA;       \
  } while (0)

}  // namespace

struct grn_surrogate {
  int device = 0;
  cudaStream_t st = nullptr;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  __nv_bfloat16 *wb = nullptr;
  __nv_bfloat16 *w2t = nullptr, *w3t = nullptr;  // transposed BF16 W2, W3
  int bmax = 0;
  // Minibatch activations and gradients, row-major [bmax][width], and their
  // transposes [width][bmax] (the K-major operands of the weight gradients).
  __nv_bfloat16 *x = nullptr, *h1 = nullptr, *h2 = nullptr, *h3 = nullptr;
  __nv_bfloat16 *dz1 = nullptr, *dz2 = nullptr, *dz3 = nullptr;
  __nv_bfloat16 *xT = nullptr, *h1T = nullptr, *h2T = nullptr, *h3T = nullptr;
  __nv_bfloat16 *dz1T = nullptr, *dz2T = nullptr, *dz3T = nullptr;
  float *xf = nullptr;  // FP32 staging of uploaded rows [bmax][kF]
  float *y = nullptr, *t = nullptr, *dy = nullptr;
  double *loss = nullptr;  // [0] last minibatch, [1] sum over a training call
  float *work = nullptr;   // split-K partial tiles of the weight gradients
  size_t work_elems = 0;
  int32_t *idx = nullptr;
  int idx_cap = 0;
  int cap = 0, count = 0, head = 0;  // dataset ring buffer
  __nv_bfloat16 *dx = nullptr;
  float *dt = nullptr;
  int step = 0;
  int *d_step = nullptr;   // Adam steps taken (device; the captured step reads it)
  std::mt19937_64 rng;
  // One training step (forward, backward, Adam) captured as a CUDA graph for
  // this batch size, learning rate and tensor-core path.
  cudaGraphExec_t train_exec = nullptr;
  int graph_B = 0;
  float graph_lr = 0;
  bool graph_tc = true;
  bool tcgen05 = true;     // GEMMs on tcgen05 (else mma.sync)
  int *d_err = nullptr;    // set by a tcgen05 GEMM whose wait timed out
};

namespace {

grn::MlpGemm gemm_args(int M, int N, int K, const __nv_bfloat16 *A, int64_t lda,
                       const __nv_bfloat16 *B, int64_t ldb) {
  grn::MlpGemm p{};
  p.M = M;
  p.N = N;
  p.K = K;
  p.A = A;
  p.lda = lda;
  p.B = B;
  p.ldb = ldb;
  return p;
}

// One GEMM of the MLP on the selected tensor-core path.
cudaError_t gemm(grn_surrogate *s, const grn::MlpGemm &p) {
  if (s->tcgen05) return grn::mlp_gemm_tc(p, s->work, s->work_elems, s->d_err, s->st);
  return grn::mlp_gemm(p, s->st);
}

// Reads and clears the tcgen05 time-out flag (after the stream is synced).
grn_status check_err(grn_surrogate *s) {
  int e = 0;
  GRN_CK(cudaMemcpy(&e, s->d_err, sizeof e, cudaMemcpyDeviceToHost));
  if (!e) return GRN_OK;
  GRN_CK(cudaMemset(s->d_err, 0, sizeof e));
  return GRN_ERR_KERNEL;
}

// Hidden layers and output of the rows in s->x; `train` also stores the
// transposed activations that the weight gradients read.
grn_status forward(grn_surrogate *s, int B, bool train) {
  using namespace grn;
  const int64_t T = s->bmax;
  const __nv_bfloat16 *in[3] = {s->x, s->h1, s->h2};
  __nv_bfloat16 *out[3] = {s->h1, s->h2, s->h3}, *outT[3] = {s->h1T, s->h2T, s->h3T};
  const int64_t wo[3] = {kW1, kW2, kW3}, bo[3] = {kB1, kB2, kB3};
  for (int l = 0; l < 3; ++l) {
    const int K = l == 0 ? kF : kH;
    MlpGemm p = gemm_args(B, kH, K, in[l], K, s->wb + wo[l], K);
    p.epi = kEpiBiasRelu;
    p.Cb = out[l];
    p.ldc = kH;
    p.bias = s->w + bo[l];
    if (train) {
      p.Ct = outT[l];
      p.ldt = T;
    }
    GRN_CK(gemm(s, p));
  }
  GRN_CK(mlp_output_forward(B, kH, s->h3, s->w + kW4, s->w + kB4, s->y, s->st));
  return GRN_OK;
}

// Loss and gradients of a minibatch already in s->x / s->xT / s->t (after
// forward with train set); `adam` counts the Adam step that follows.
grn_status backward(grn_surrogate *s, int B, bool adam) {
  using namespace grn;
  cudaStream_t st = s->st;
  const int64_t T = s->bmax;
  GRN_CK(mlp_loss(B, s->y, s->t, s->dy, s->loss, s->g + kB4, adam ? s->d_step : nullptr, st));
  GRN_CK(mlp_output_backward(B, kH, s->h3, s->w + kW4, s->dy, s->dz3, s->dz3T, T, st));
  // Per hidden layer l = 3, 2, 1: dW_l = dZ_l^T H_(l-1) (K = the batch, from
  // the transposed copies), and for l > 1 dZ_(l-1) = (dZ_l W_l) * [H_(l-1) > 0].
  const __nv_bfloat16 *dzT[3] = {s->dz1T, s->dz2T, s->dz3T};
  const __nv_bfloat16 *hT[3] = {s->xT, s->h1T, s->h2T};
  const __nv_bfloat16 *dz[3] = {s->dz1, s->dz2, s->dz3};
  const __nv_bfloat16 *hprev[3] = {s->x, s->h1, s->h2};
  const __nv_bfloat16 *wt[3] = {nullptr, s->w2t, s->w3t};
  __nv_bfloat16 *dzo[3] = {nullptr, s->dz1, s->dz2}, *dzoT[3] = {nullptr, s->dz1T, s->dz2T};
  const int64_t wo[3] = {kW1, kW2, kW3};
  for (int l = 2; l >= 0; --l) {
    const int N = l == 0 ? kF : kH;
    MlpGemm p = gemm_args(kH, N, B, dzT[l], T, hT[l], T);
    p.epi = kEpiF32;
    p.Cf = s->g + wo[l];
    p.ldc = N;
    GRN_CK(gemm(s, p));
    if (l == 0) break;
    p = gemm_args(B, kH, kH, dz[l], kH, wt[l], kH);
    p.epi = kEpiMask;
    p.Cb = dzo[l];
    p.ldc = kH;
    p.mask = hprev[l];
    p.Ct = dzoT[l];
    p.ldt = T;
    GRN_CK(gemm(s, p));
  }
  // Output weights and hidden biases: sums over the batch of the transposes.
  const MlpRowSum jobs[4] = {{s->h3T, s->dy, s->g + kW4},
                             {s->dz3T, nullptr, s->g + kB3},
                             {s->dz2T, nullptr, s->g + kB2},
                             {s->dz1T, nullptr, s->g + kB1}};
  GRN_CK(mlp_row_sums(4, jobs, kH, B, T, st));
  return GRN_OK;
}

// Refreshes the transposed BF16 weights the backward GEMMs read (after the
// parameters are set; Adam refreshes them after each step).
grn_status transpose_weights(grn_surrogate *s) {
  GRN_CK(grn::mlp_transpose(kH, kH, s->wb + kW2, kH, s->w2t, kH, s->st));
  GRN_CK(grn::mlp_transpose(kH, kH, s->wb + kW3, kH, s->w3t, kH, s->st));
  return GRN_OK;
}

// Forward, backward and Adam on the minibatch in s->x / s->xT / s->t.
grn_status train_step_body(grn_surrogate *s, int B, float lr) {
  grn_status st = forward(s, B, true);
  if (st == GRN_OK) st = backward(s, B, true);
  if (st != GRN_OK) return st;
  const grn::MlpTransposed tr{{kW2, kW3}, {s->w2t, s->w3t}, kH};
  GRN_CK(grn::mlp_adam((int)kP, s->w, s->g, s->m, s->v, lr, 0.9f, 0.999f, 1e-8f, s->d_step,
                       s->wb, tr, s->st));
  return GRN_OK;
}

void drop_train_graph(grn_surrogate *s) {
  if (s->train_exec) cudaGraphExecDestroy(s->train_exec);
  s->train_exec = nullptr;
}

// One training step.  The first step of a (batch size, learning rate,
// tensor-core path) runs its 16 launches directly -- which also loads every
// kernel's module -- and is then captured as a graph; later steps replay it
// (the kernels' arguments do not change; the Adam step count is read from
// device memory).
grn_status train_step(grn_surrogate *s, int B, float lr) {
  if (s->train_exec && s->graph_B == B && s->graph_lr == lr && s->graph_tc == s->tcgen05) {
    GRN_CK(cudaGraphLaunch(s->train_exec, s->st));
    return GRN_OK;
  }
  drop_train_graph(s);
  grn_status st = train_step_body(s, B, lr);
  if (st != GRN_OK) return st;
  GRN_CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeRelaxed));
  st = train_step_body(s, B, lr);
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(s->st, &graph);
  cudaError_t ei = cudaSuccess;
  if (st == GRN_OK && ec == cudaSuccess) ei = cudaGraphInstantiate(&s->train_exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (st != GRN_OK || ec != cudaSuccess || ei != cudaSuccess) {
    s->train_exec = nullptr;
    cudaGetLastError();
    return st != GRN_OK ? st : GRN_ERR_CUDA;
  }
  s->graph_B = B;
  s->graph_lr = lr;
  s->graph_tc = s->tcgen05;
  return GRN_OK;
}

// One Adam step on the training-set rows d_idx[0..B) (device indices).
grn_status train_minibatch(grn_surrogate *s, const int32_t *d_idx, int B, float lr) {
  GRN_CK(grn::mlp_gather_rows(B, kF, d_idx, s->dx, s->dt, s->x, s->t, s->xT, s->bmax, s->st));
  const grn_status st = train_step(s, B, lr);
  if (st == GRN_OK) s->step += 1;
  return st;
}

// Runs minibatch i on the sizes[i] training-set rows that follow in idx.
// Indices go to the device in chunks of whole minibatches, and the losses
// add up on the device: one host synchronisation per call.
grn_status run_minibatches(grn_surrogate *s, const std::vector<int32_t> &idx,
                           const std::vector<int> &sizes, float lr, double *mean_loss) {
  GRN_CK(cudaMemsetAsync(s->loss + 1, 0, sizeof(double), s->st));
  size_t pos = 0, b = 0;
  while (b < sizes.size()) {
    size_t e = b, rows = 0;
    while (e < sizes.size() && rows + sizes[e] <= (size_t)s->idx_cap) rows += sizes[e++];
    GRN_CK(cudaMemcpyAsync(s->idx, idx.data() + pos, rows * sizeof(int32_t),
                           cudaMemcpyHostToDevice, s->st));
    size_t off = 0;
    for (; b < e; ++b) {
      const grn_status st = train_minibatch(s, s->idx + off, sizes[b], lr);
      if (st != GRN_OK) return st;
      off += sizes[b];
    }
    pos += rows;
  }
  double l = 0;
  GRN_CK(cudaMemcpyAsync(&l, s->loss + 1, sizeof l, cudaMemcpyDeviceToHost, s->st));
  GRN_CK(cudaStreamSynchronize(s->st));
  if (mean_loss) *mean_loss = sizes.empty() ? 0 : l / sizes.size();
  return GRN_OK;
}

// n <= bmax FP32 rows of kF features from the host to BF16 rows at dst (and
// their transpose at dstT, if set), through the FP32 staging buffer.
grn_status stage_rows(grn_surrogate *s, const float *features, int n, __nv_bfloat16 *dst,
                      __nv_bfloat16 *dstT) {
  GRN_CK(cudaMemcpyAsync(s->xf, features, (size_t)n * kF * sizeof(float), cudaMemcpyHostToDevice,
                         s->st));
  GRN_CK(grn::mlp_convert_rows(n, kF, s->xf, dst, dstT, s->bmax, s->st));
  return GRN_OK;
}

}  // namespace

extern "C" {

grn_status grn_encode_models(const grn_model_batch *batch, int n_morphogens, float *features) {
  if (!batch || !features || batch->n_models < 0 || n_morphogens < 0)
    return GRN_ERR_INVALID_ARGUMENT;
  for (int m = 0; m < batch->n_models; ++m) {
    float *f = features + (size_t)m * kF;
    std::memset(f, 0, sizeof(float) * kF);
    const int p0 = batch->product_offsets[m], p1 = batch->product_offsets[m + 1];
    const int l0 = batch->link_offsets[m], l1 = batch->link_offsets[m + 1];
    std::vector<uint4> rec;
    grn::ModelCost cost;
    std::string err;
    const grn_status s = grn::pack_model(batch->products + p0, p1 - p0, batch->links + l0,
                                         l1 - l0, n_morphogens, m, &rec, &cost, &err);
    if (s != GRN_OK) return s;
    grn::PackedHeader hdr;
    std::memcpy(&hdr, rec.data(), sizeof hdr);
    // 8 genes x (lim, deg, dif, in use), then 24 links x (regulator slot / 8,
    // K, signed Hill coefficient / 5, +-(regulated gene + 1) / 8 with the sign
    // - for AND and + for OR), links in program order (each gene's OR links,
    // then its AND links).  K and n come back from the exponent form
    // a = -n_signed, b = -a * lg2(K).
    int li = 0;
    for (int gi = 0; gi < hdr.n_genes; ++gi) {
      grn::PackedGene g;
      std::memcpy(&g, rec.data() + 1 + gi, sizeof g);
      if (gi < 8) {
        f[4 * gi + 0] = g.lim;
        f[4 * gi + 1] = g.deg;
        f[4 * gi + 2] = g.dif;
        f[4 * gi + 3] = 1.0f;
      }
      for (int l = 0; l < g.n_or + g.n_and && li < 24; ++l, ++li) {
        grn::PackedLink lk;
        std::memcpy(&lk, rec.data() + 1 + hdr.n_genes + g.link_begin + l, sizeof lk);
        float *q = f + 32 + 4 * li;
        const bool konst = lk.slot == grn::kConstSlot;
        q[0] = konst ? -0.125f : lk.slot / 8.0f;
        const float k = (konst || lk.a == 0.0f) ? 0.0f : std::exp2(-lk.b / lk.a);
        q[1] = std::isfinite(k) ? std::min(k, 4.0f) : 4.0f;
        q[2] = -lk.a / 5.0f;
        q[3] = (l < g.n_or ? 1.0f : -1.0f) * (gi + 1) / 8.0f;
      }
    }
  }
  return GRN_OK;
}

grn_status grn_surrogate_create(int device, uint64_t seed, int capacity, grn_surrogate **out) {
  if (!out || capacity < 1) return GRN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) {
    cudaGetLastError();
    return GRN_ERR_NO_DEVICE;
  }
  grn_surrogate *s = new (std::nothrow) grn_surrogate();
  if (!s) return GRN_ERR_OUT_OF_MEMORY;
  s->device = device;
  s->rng.seed(seed);
  s->cap = capacity;
  s->bmax = 8192;
  cudaSetDevice(device);
  bool ok = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) == cudaSuccess;
  auto alloc = [&](void **p, size_t bytes) {
    if (ok && cudaMalloc(p, bytes) != cudaSuccess) ok = false;
  };
  alloc((void **)&s->w, kP * 4);
  alloc((void **)&s->g, kP * 4);
  alloc((void **)&s->m, kP * 4);
  alloc((void **)&s->v, kP * 4);
  alloc((void **)&s->wb, kP * 2);
  alloc((void **)&s->w2t, (size_t)kH * kH * 2);
  alloc((void **)&s->w3t, (size_t)kH * kH * 2);
  const size_t B = s->bmax;
  for (__nv_bfloat16 **p : {&s->x, &s->xT}) alloc((void **)p, B * kF * 2);
  for (__nv_bfloat16 **p : {&s->h1, &s->h2, &s->h3, &s->dz1, &s->dz2, &s->dz3, &s->h1T, &s->h2T,
                            &s->h3T, &s->dz1T, &s->dz2T, &s->dz3T})
    alloc((void **)p, B * kH * 2);
  alloc((void **)&s->xf, B * kF * 4);
  alloc((void **)&s->y, B * 4);
  alloc((void **)&s->t, B * 4);
  alloc((void **)&s->dy, B * 4);
  alloc((void **)&s->loss, 2 * sizeof(double));
  // Split-K workspace: 32 partial 256 x 256 FP32 tiles.
  s->work_elems = (size_t)32 * kH * kH;
  alloc((void **)&s->work, s->work_elems * 4);
  s->idx_cap = 16 * s->bmax;
  alloc((void **)&s->idx, (size_t)s->idx_cap * 4);
  alloc((void **)&s->dx, (size_t)capacity * kF * 2);
  alloc((void **)&s->dt, (size_t)capacity * 4);
  alloc((void **)&s->d_err, sizeof(int));
  if (ok && cudaMemset(s->d_err, 0, sizeof(int)) != cudaSuccess) ok = false;
  alloc((void **)&s->d_step, sizeof(int));
  if (ok && cudaMemset(s->d_step, 0, sizeof(int)) != cudaSuccess) ok = false;
  if (!ok) {
    grn_surrogate_destroy(s);
    return GRN_ERR_OUT_OF_MEMORY;
  }
  // He initialisation for the ReLU layers, small output layer, zero biases.
  std::vector<float> w(kP, 0.0f);
  auto init = [&](int64_t off, int rows, int fan_in, float scale) {
    std::normal_distribution<float> nd(0.0f, scale * std::sqrt(2.0f / fan_in));
    for (int64_t i = 0; i < (int64_t)rows * fan_in; ++i) w[off + i] = nd(s->rng);
  };
  init(kW1, kH, kF, 1.0f);
  init(kW2, kH, kH, 1.0f);
  init(kW3, kH, kH, 1.0f);
  init(kW4, 1, kH, 0.5f);
  w[kB4] = -1.0f;  // typical log(error) of random models
  if (grn_surrogate_set_params(s, w.data(), (int)kP) != GRN_OK) {
    grn_surrogate_destroy(s);
    return GRN_ERR_CUDA;
  }
  *out = s;
  return GRN_OK;
}

grn_status grn_surrogate_destroy(grn_surrogate *s) {
  if (!s) return GRN_OK;
  cudaSetDevice(s->device);
  if (s->st) cudaStreamSynchronize(s->st);
  drop_train_graph(s);
  for (void *p : {(void *)s->w, (void *)s->g, (void *)s->m, (void *)s->v, (void *)s->wb,
                  (void *)s->w2t, (void *)s->w3t, (void *)s->x, (void *)s->h1, (void *)s->h2,
                  (void *)s->h3, (void *)s->dz1, (void *)s->dz2, (void *)s->dz3, (void *)s->xT,
                  (void *)s->h1T, (void *)s->h2T, (void *)s->h3T, (void *)s->dz1T,
                  (void *)s->dz2T, (void *)s->dz3T, (void *)s->xf, (void *)s->y, (void *)s->t,
                  (void *)s->dy, (void *)s->loss, (void *)s->work, (void *)s->idx, (void *)s->dx,
                  (void *)s->dt, (void *)s->d_err, (void *)s->d_step})
    if (p) cudaFree(p);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
  return GRN_OK;
}

grn_status grn_surrogate_set_params(grn_surrogate *s, const float *params, int n) {
  if (!s || !params || n != kP) return GRN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  GRN_CK(cudaMemcpyAsync(s->w, params, kP * 4, cudaMemcpyHostToDevice, s->st));
  GRN_CK(cudaMemsetAsync(s->m, 0, kP * 4, s->st));
  GRN_CK(cudaMemsetAsync(s->v, 0, kP * 4, s->st));
  GRN_CK(cudaMemsetAsync(s->d_step, 0, sizeof(int), s->st));
  GRN_CK(grn::mlp_to_bf16((int)kP, s->w, s->wb, s->st));
  const grn_status ts = transpose_weights(s);
  if (ts != GRN_OK) return ts;
  GRN_CK(cudaStreamSynchronize(s->st));
  s->step = 0;
  return GRN_OK;
}

grn_status grn_surrogate_params(grn_surrogate *s, float *out, int n) {
  if (!s || !out || n != kP) return GRN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  GRN_CK(cudaMemcpyAsync(out, s->w, kP * 4, cudaMemcpyDeviceToHost, s->st));
  GRN_CK(cudaStreamSynchronize(s->st));
  return GRN_OK;
}

grn_status grn_surrogate_add_data(grn_surrogate *s, const float *features, const float *log_error,
                                  int n) {
  if (!s || n < 0 || (n > 0 && (!features || !log_error))) return GRN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  for (int i = 0; i < n;) {
    const int chunk = std::min({n - i, s->cap - s->head, s->bmax});
    const grn_status st = stage_rows(s, features + (size_t)i * kF, chunk,
                                     s->dx + (size_t)s->head * kF, nullptr);
    if (st != GRN_OK) return st;
    GRN_CK(cudaMemcpyAsync(s->dt + s->head, log_error + i, chunk * 4, cudaMemcpyHostToDevice,
                           s->st));
    s->head = (s->head + chunk) % s->cap;
    s->count = std::min(s->cap, s->count + chunk);
    i += chunk;
  }
  GRN_CK(cudaStreamSynchronize(s->st));
  return GRN_OK;
}

int grn_surrogate_data_count(const grn_surrogate *s) { return s ? s->count : 0; }

grn_status grn_surrogate_train(grn_surrogate *s, int epochs, int batch_size, float lr,
                               double *mean_loss) {
  grn::TraceRange trace_range("grn_surrogate_train");
  if (!s || epochs < 0 || batch_size < 1 || batch_size > s->bmax || !(lr > 0))
    return GRN_ERR_INVALID_ARGUMENT;
  if (s->count == 0) return GRN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  std::vector<int32_t> perm(s->count), idx;
  std::vector<int> sizes;
  idx.reserve((size_t)epochs * s->count);
  for (int e = 0; e < epochs; ++e) {
    for (int i = 0; i < s->count; ++i) perm[i] = i;
    std::shuffle(perm.begin(), perm.end(), s->rng);
    idx.insert(idx.end(), perm.begin(), perm.end());
    for (int b0 = 0; b0 < s->count; b0 += batch_size)
      sizes.push_back(std::min(batch_size, s->count - b0));
  }
  const grn_status st = run_minibatches(s, idx, sizes, lr, mean_loss);
  if (st != GRN_OK) return st;
  return check_err(s);
}

grn_status grn_surrogate_train_batches(grn_surrogate *s, int n_batches, int batch_size, float lr,
                                       double *mean_loss) {
  grn::TraceRange trace_range("grn_surrogate_train_batches");
  if (!s || n_batches < 0 || batch_size < 1 || batch_size > s->bmax || !(lr > 0))
    return GRN_ERR_INVALID_ARGUMENT;
  if (s->count == 0) return GRN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  const int B = std::min(batch_size, s->count);
  std::vector<int32_t> idx((size_t)n_batches * B);
  std::uniform_int_distribution<int32_t> pick(0, s->count - 1);
  for (auto &i : idx) i = pick(s->rng);
  const grn_status st = run_minibatches(s, idx, std::vector<int>(n_batches, B), lr, mean_loss);
  if (st != GRN_OK) return st;
  return check_err(s);
}

grn_status grn_surrogate_predict(grn_surrogate *s, const float *features, int n, float *out) {
  grn::TraceRange trace_range("grn_surrogate_predict");
  if (!s || n < 0 || (n > 0 && (!features || !out))) return GRN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  for (int i = 0; i < n; i += s->bmax) {
    const int B = std::min(s->bmax, n - i);
    grn_status st = stage_rows(s, features + (size_t)i * kF, B, s->x, nullptr);
    if (st == GRN_OK) st = forward(s, B, false);
    if (st != GRN_OK) return st;
    GRN_CK(cudaMemcpyAsync(out + i, s->y, B * 4, cudaMemcpyDeviceToHost, s->st));
    GRN_CK(cudaStreamSynchronize(s->st));
  }
  return check_err(s);
}

// Checkpoint layout (host byte order): magic, version, parameter count,
// capacity, count, head, host step, the sampling RNG (std::mt19937_64 text
// form), then the FP32 weights, Adam's two moments and step, and the
// training set's first `count` rows (BF16 features, FP32 targets) when the
// ring has not wrapped, else all `capacity` rows.
grn_status grn_surrogate_checkpoint(grn_surrogate *s, void *buf, size_t cap, size_t *size) {
  if (!s || !size) return GRN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  const int rows = s->count < s->cap ? s->count : s->cap;
  std::ostringstream rng_text;
  rng_text << s->rng;
  const std::string rt = rng_text.str();
  const size_t head_bytes = 8 + 4 * 7 + 8 + rt.size();
  const size_t total = head_bytes + 3 * (size_t)kP * 4 + 4 + (size_t)rows * (kF * 2 + 4);
  *size = total;
  if (!buf) return GRN_OK;
  if (cap < total) return GRN_ERR_CAPACITY;
  char *o = static_cast<char *>(buf);
  auto put = [&](const void *p, size_t n) {
    std::memcpy(o, p, n);
    o += n;
  };
  const uint32_t version = 1;
  const int32_t hdr[6] = {(int32_t)kP, s->cap, s->count, s->head, s->step, s->tcgen05 ? 1 : 0};
  const uint64_t rlen = rt.size();
  put("GRNSURCK", 8);
  put(&version, 4);
  put(hdr, sizeof hdr);
  put(&rlen, 8);
  put(rt.data(), rt.size());
  GRN_CK(cudaMemcpyAsync(o, s->w, kP * 4, cudaMemcpyDeviceToHost, s->st));
  GRN_CK(cudaMemcpyAsync(o + kP * 4, s->m, kP * 4, cudaMemcpyDeviceToHost, s->st));
  GRN_CK(cudaMemcpyAsync(o + 2 * kP * 4, s->v, kP * 4, cudaMemcpyDeviceToHost, s->st));
  GRN_CK(cudaMemcpyAsync(o + 3 * kP * 4, s->d_step, 4, cudaMemcpyDeviceToHost, s->st));
  char *d = o + 3 * kP * 4 + 4;
  GRN_CK(cudaMemcpyAsync(d, s->dx, (size_t)rows * kF * 2, cudaMemcpyDeviceToHost, s->st));
  GRN_CK(cudaMemcpyAsync(d + (size_t)rows * kF * 2, s->dt, (size_t)rows * 4,
                         cudaMemcpyDeviceToHost, s->st));
  GRN_CK(cudaStreamSynchronize(s->st));
  return GRN_OK;
}

grn_status grn_surrogate_restore(grn_surrogate *s, const void *buf, size_t size) {
  if (!s || !buf) return GRN_ERR_INVALID_ARGUMENT;
  const char *p = static_cast<const char *>(buf), *end = p + size;
  auto get = [&](void *v, size_t n) {
    if ((size_t)(end - p) < n) return false;
    std::memcpy(v, p, n);
    p += n;
    return true;
  };
  char magic[8];
  uint32_t version = 0;
  int32_t hdr[6];
  uint64_t rlen = 0;
  if (!get(magic, 8) || std::memcmp(magic, "GRNSURCK", 8) != 0 || !get(&version, 4) ||
      version != 1 || !get(hdr, sizeof hdr) || !get(&rlen, 8) || rlen > (1u << 16) ||
      (size_t)(end - p) < rlen)
    return GRN_ERR_INVALID_ARGUMENT;
  const int cap = hdr[1], count = hdr[2], head = hdr[3];
  if (hdr[0] != (int32_t)kP || cap != s->cap || count < 0 || count > cap || head < 0 ||
      head >= cap)
    return GRN_ERR_INVALID_ARGUMENT;
  std::mt19937_64 rng;
  {
    std::istringstream i(std::string(p, (size_t)rlen));
    if (!(i >> rng)) return GRN_ERR_INVALID_ARGUMENT;
  }
  p += rlen;
  const int rows = count < cap ? count : cap;
  if ((size_t)(end - p) != 3 * (size_t)kP * 4 + 4 + (size_t)rows * (kF * 2 + 4))
    return GRN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  GRN_CK(cudaStreamSynchronize(s->st));
  drop_train_graph(s);
  GRN_CK(cudaMemcpyAsync(s->w, p, kP * 4, cudaMemcpyHostToDevice, s->st));
  GRN_CK(cudaMemcpyAsync(s->m, p + kP * 4, kP * 4, cudaMemcpyHostToDevice, s->st));
  GRN_CK(cudaMemcpyAsync(s->v, p + 2 * kP * 4, kP * 4, cudaMemcpyHostToDevice, s->st));
  GRN_CK(cudaMemcpyAsync(s->d_step, p + 3 * kP * 4, 4, cudaMemcpyHostToDevice, s->st));
  const char *d = p + 3 * kP * 4 + 4;
  GRN_CK(cudaMemcpyAsync(s->dx, d, (size_t)rows * kF * 2, cudaMemcpyHostToDevice, s->st));
  GRN_CK(cudaMemcpyAsync(s->dt, d + (size_t)rows * kF * 2, (size_t)rows * 4,
                         cudaMemcpyHostToDevice, s->st));
  GRN_CK(grn::mlp_to_bf16((int)kP, s->w, s->wb, s->st));
  const grn_status ts = transpose_weights(s);
  if (ts != GRN_OK) return ts;
  GRN_CK(cudaStreamSynchronize(s->st));
  s->count = count;
  s->head = head;
  s->step = hdr[4];
  s->tcgen05 = hdr[5] != 0;
  s->rng = rng;
  return GRN_OK;
}

grn_status grn_surrogate_use_tcgen05(grn_surrogate *s, int enable) {
  if (!s) return GRN_ERR_INVALID_ARGUMENT;
  s->tcgen05 = enable != 0;
  return GRN_OK;
}

grn_status grn_surrogate_gradients(grn_surrogate *s, const float *features,
                                   const float *log_error, int n, float *grads, double *loss) {
  if (!s || !features || !log_error || !grads || n < 1 || n > s->bmax)
    return GRN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(s->device);
  grn_status st = stage_rows(s, features, n, s->x, s->xT);
  if (st != GRN_OK) return st;
  GRN_CK(cudaMemcpyAsync(s->t, log_error, n * 4, cudaMemcpyHostToDevice, s->st));
  st = forward(s, n, true);
  if (st == GRN_OK) st = backward(s, n, false);
  if (st != GRN_OK) return st;
  GRN_CK(cudaMemcpyAsync(grads, s->g, kP * 4, cudaMemcpyDeviceToHost, s->st));
  double l = 0;
  GRN_CK(cudaMemcpyAsync(&l, s->loss, 8, cudaMemcpyDeviceToHost, s->st));
  GRN_CK(cudaStreamSynchronize(s->st));
  if (loss) *loss = l;
  return check_err(s);
}

}  // extern "C"
