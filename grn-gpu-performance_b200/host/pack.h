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

grn_status pack_batch(const grn_model_batch *batch, int n_morphogens,
                      int n_threads, PackedHost *out, std::string *err);

}  // namespace grn

#endif  // GRN_HOST_PACK_H_
