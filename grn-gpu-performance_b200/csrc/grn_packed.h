// grn_packed.h -- packed program format of a compiled GRN model, shared by
// the host compiler (host/pack.cpp) and the simulation kernels.
//
// A model's regulation program (the reference builds it as a list of SimOp /
// CSimOp objects, Src/Simulator/modelsimulator.cpp:71-203 and
// Src/GPUSimulator/cmodelsimulator.cpp:114-227) is stored as one record of
// 16-byte words:
//
//   word 0            PackedHeader
//   words 1 .. G      PackedGene, one per product in use (sorted labels)
//   words G+1 .. G+L  PackedLink, the used links of gene 0, then gene 1, ...
//                     each gene's OR links first, then its AND links, each
//                     group in the model's link order
//
// Hill terms are stored in "exponent form".  For regulator value x,
//   activation  x^n / (x^n + K^n) = 1 / (1 + 2^v),  v = -n*lg2(x) + n*lg2(K)
//   repression  K^n / (x^n + K^n) = 1 / (1 + 2^v),  v =  n*lg2(x) - n*lg2(K)
// so a link is (a, b) with v = a*lg2(x) + b.  1/(1+2^v) falls as v rises,
// hence the reference's OR (max of Hill values) is the min of the v's and
// its AND (min of Hill values) is the max of the v's, and a gene's whole
// regulation is 1/(1 + 2^V) with V combined in v-space: two transcendental
// operations per gene instead of three per link.
#ifndef GRN_PACKED_H_
#define GRN_PACKED_H_

#include <stdint.h>

namespace grn {

// Regulator slot of a link whose Hill coefficient is 0: the reference
// evaluates pow(x, 0) = 1 for every x, i.e. a constant Hill value 1/2, so
// the link reads the constant lg2 value 0 with a = b = 0.
constexpr int kConstSlot = 255;

// Header flags.
constexpr uint32_t kFlagNone = 0u;
// Every link has a finite K > 0, a finite Hill coefficient n <= 32 and
// 0 < K^n <= 1e300, every gene finite rates, and no (regulator, regulated)
// pair repeats: on a bounded non-negative state no link term can be NaN, so
// the kernel may combine terms with min/max over a dense per-gene table of
// regulator slots (see the kernel's regulation).  pack_batch also clears
// the flag where the run's step size could leave the state unbounded
// (euler_bounded in host/pack.h), so the kernel tests only the flag.
constexpr uint32_t kFlagFast = 1u;

struct alignas(16) PackedHeader {
  int32_t orig_index;  // position of the model in the caller's batch
  int16_t n_genes;     // G: products in use
  int16_t n_links;     // L: links in the program
  uint32_t lg_mask;    // bit g set: gene g is read by some link (needs lg2)
  uint32_t flags;
};

struct alignas(16) PackedGene {
  float lim;           // production rate
  float deg;           // degradation rate
  float dif;           // diffusion constant, 0 if the product does not diffuse
  uint16_t link_begin; // first link of this gene, relative to the link block
  uint8_t n_or;        // OR links (processed first)
  uint8_t n_and;       // AND links; n_or + n_and == 0 means regulation 0
};

struct alignas(16) PackedLink {
  int32_t slot;        // regulator product index, or kConstSlot
  float a;             // v = a * lg2(x) + b
  float b;
  int32_t reserved;
};

static_assert(sizeof(PackedHeader) == 16, "packed header is one word");
static_assert(sizeof(PackedGene) == 16, "packed gene is one word");
static_assert(sizeof(PackedLink) == 16, "packed link is one word");

// Words of one model record.
inline int record_words(int n_genes, int n_links) { return 1 + n_genes + n_links; }

}  // namespace grn

#endif  // GRN_PACKED_H_
