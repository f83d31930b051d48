// pack.h -- host compiler from genome-form models to packed programs.
#ifndef GRN_HOST_PACK_H_
#define GRN_HOST_PACK_H_

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/grn_gpu.h"
#include "../csrc/grn_packed.h"

namespace grn {

struct ModelCost {
  int genes = 0;      // products in use
  int links = 0;      // links in the program
  int lg_genes = 0;   // genes read by some link (lg2 per cell)
  int reg_genes = 0;  // genes with a non-zero regulation (ex2 + rcp per cell)
  int dif_genes = 0;  // diffusing genes
  double cost = 0;    // relative work of one cell-step
};

// Compiles one model (CModelSimulator::loadModel,
// Src/GPUSimulator/cmodelsimulator.cpp:114-227) and appends its record to
// `out`.  Returns GRN_OK, GRN_ERR_MODEL (a label in use has no product) or
// GRN_ERR_CAPACITY (more than GRN_MAX_GENES / GRN_MAX_LINKS).
grn_status pack_model(const grn_product *products, int n_products,
                      const grn_link *links, int n_links, int n_morphogens,
                      int orig_index, std::vector<uint4> *out,
                      ModelCost *cost, std::string *err);

// Sorted labels in use: the morphogens and, transitively, their regulators
// (Model::calcProductLabelsInUse, Src/Model/model.cpp:243-270); the order of
// a compiled model's genes.
std::vector<int> labels_in_use(const grn_link *links, int n_links, int n_morphogens);

// A whole batch, records ordered by decreasing cost so that the persistent
// kernel's work queue hands out the longest models first.
struct PackedHost {
  std::vector<uint4> words;
  std::vector<int32_t> offsets;  // [n_models] first word of each record
  int n_models = 0;
  int max_genes = 0;
  int max_links = 0;
  double sum_genes = 0;
  double sum_links = 0;
  int64_t sfu_per_cell_step = 0;  // sum over models of lg + 2 * reg genes
  int64_t fma_per_cell_step = 0;  // rough FP32-pipe op count, summed
  double sum_dif_genes = 0;
  int64_t alg_sfu_per_cell_step = 0;   // sum of 3 L (reference formulation)
  int64_t alg_fp32_per_cell_step = 0;  // sum of 6 L + 7 G + 8 G_dif
};

// Packs a batch for runs of n_steps explicit Euler steps of size dt.  The
// fast-path flag of each record also requires the Euler update to stay
// bounded at that step size (euler_bounded).
grn_status pack_batch(const grn_model_batch *batch, int n_morphogens, float dt, int n_steps,
                      int n_threads, PackedHost *out, std::string *err);

// Largest growth of a state value over a run that the fast path accepts.
constexpr float kFastMaxGrowth = 1.0e6f;

// Whether the explicit Euler update of these genes stays finite and
// non-negative.  With dt >= 0, deg >= 0 and dt*(deg + 4*dif) <= 1 for every
// gene, the update of a cell is a combination with non-negative weights of
// its old value, its neighbours and dt*lim*h (h in [0, 1]), so no value goes
// negative and the largest value grows by at most dt*max(lim, 0) per step.
// Bounding that growth over the run (kFastMaxGrowth) and the initial state
// (the context's fast_ok) keeps every x^n and K^n far from overflow.  A
// model outside the bound -- an unstable step such as dt*dif > 1/4, where a
// checkerboard mode grows until cells overflow to inf and NaN -- runs the
// exact path, which keeps the reference's inf / NaN behaviour
// (modelsimulator.cpp:262-275, simstate.cpp:147-151).
bool euler_bounded(const PackedGene *genes, int n_genes, float dt, int n_steps);

}  // namespace grn

#endif  // GRN_HOST_PACK_H_
