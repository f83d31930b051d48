// pack.cpp -- host compiler from genome-form models to packed programs.
#include "pack.h"
#include "trace.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>

namespace grn {

namespace {

bool contains(const std::vector<int> &v, int x) {
  return std::find(v.begin(), v.end(), x) != v.end();
}

}  // namespace

std::vector<int> labels_in_use(const grn_link *links, int n_links, int n_morphogens) {
  std::vector<int> labels;
  for (int i = 0; i < n_morphogens; ++i) labels.push_back(i);
  for (size_t h = 0; h < labels.size(); ++h)
    for (int l = 0; l < n_links; ++l)
      if (links[l].regulated == labels[h] && !contains(labels, links[l].regulator))
        labels.push_back(links[l].regulator);
  std::sort(labels.begin(), labels.end());
  return labels;
}

grn_status pack_model(const grn_product *products, int n_products,
                      const grn_link *links, int n_links, int n_morphogens,
                      int orig_index, std::vector<uint4> *out,
                      ModelCost *cost, std::string *err) {
  // Labels in use: every morphogen, and every regulator of a label in use
  // (Model::calcProductLabelsInUse, Src/Model/model.cpp:243-270).
  std::vector<int> labels;
  labels.reserve(16);
  for (int i = 0; i < n_morphogens; ++i) labels.push_back(i);
  for (size_t h = 0; h < labels.size(); ++h) {
    const int lab = labels[h];
    for (int l = 0; l < n_links; ++l)
      if (links[l].regulated == lab && !contains(labels, links[l].regulator))
        labels.push_back(links[l].regulator);
    if ((int)labels.size() > GRN_MAX_GENES) {
      if (err) *err = "model " + std::to_string(orig_index) + ": more than " +
                      std::to_string(GRN_MAX_GENES) + " products in use";
      return GRN_ERR_CAPACITY;
    }
  }
  std::sort(labels.begin(), labels.end());  // qSort(labels_)
  const int G = (int)labels.size();
  auto index_of = [&](int lab) {
    return (int)(std::lower_bound(labels.begin(), labels.end(), lab) - labels.begin());
  };

  PackedHeader hdr{};
  hdr.orig_index = orig_index;
  hdr.n_genes = (int16_t)G;
  hdr.lg_mask = 0;
  hdr.flags = kFlagFast;  // cleared below if a link or rate could make NaN
  std::vector<PackedGene> genes(G);
  std::vector<PackedLink> plinks;
  plinks.reserve(n_links);
  ModelCost c;
  c.genes = G;

  for (int i = 0; i < G; ++i) {
    // Model::prodWithLabel: first product with the label (model.cpp:227-240).
    const grn_product *prod = nullptr;
    for (int p = 0; p < n_products; ++p)
      if (products[p].label == labels[i]) {
        prod = &products[p];
        break;
      }
    if (!prod) {
      if (err) *err = "model " + std::to_string(orig_index) + ": label " +
                      std::to_string(labels[i]) + " is in use but has no product";
      return GRN_ERR_MODEL;
    }
    PackedGene &g = genes[i];
    g.lim = (float)prod->lim;
    g.deg = (float)prod->deg;
    // The product diffuses iff dif > 0 (cmodelsimulator.cpp:143-147).
    g.dif = prod->dif > 0 ? (float)prod->dif : 0.0f;
    if (!std::isfinite(g.lim) || !std::isfinite(g.deg) || !std::isfinite(g.dif))
      hdr.flags &= ~kFlagFast;
    if (g.dif > 0) ++c.dif_genes;

    // OR links first, then AND links, each in model link order; a link is
    // used if its regulator is in use (cmodelsimulator.cpp:150-167).
    bool any_activator = false;
    std::vector<const grn_link *> or_l, and_l;
    for (int l = 0; l < n_links; ++l) {
      const grn_link &lk = links[l];
      if (lk.regulated != labels[i]) continue;
      if (std::binary_search(labels.begin(), labels.end(), lk.regulator)) {
        if (lk.is_and) and_l.push_back(&lk);
        else or_l.push_back(&lk);
      }
      if (lk.hill_coef >= 0) any_activator = true;
    }
    g.link_begin = (uint16_t)plinks.size();
    g.n_or = 0;
    g.n_and = 0;
    // No activator at all: regulation 0 (OpZero, cmodelsimulator.cpp:168-172);
    // no used link: also 0 (:216-217).
    if (!any_activator) continue;
    auto emit = [&](const grn_link *lk) {
      PackedLink pl{};
      // createHillOpForLink (cmodelsimulator.cpp:221-227): hillCoef >= 0 is
      // activation with n = hillCoef, else repression with n = -hillCoef.
      const bool act = lk->hill_coef >= 0;
      const double n = act ? lk->hill_coef : -1.0 * lk->hill_coef;
      if (!std::isfinite(n) || !(lk->dis_const > 0) || !std::isfinite(lk->dis_const) ||
          !std::isfinite((float)(n * std::log2(lk->dis_const))))
        hdr.flags &= ~kFlagFast;
      // The reference computes K^n once in FP64 (simophillact.cpp:9-12) and
      // then x^n / (x^n + K^n): a K^n that underflows to 0 or overflows makes
      // 0/0 or inf/inf there, which the exponent form would not reproduce.
      // With n <= 32 and a bounded state (the kernel's euler_bounded) x^n
      // stays below 1e202, so x^n + K^n is finite when K^n <= 1e300.
      if (n > 0) {
        const double kn = std::pow(lk->dis_const, n);
        if (!(kn > 0) || !(kn <= 1e300) || n > 32) hdr.flags &= ~kFlagFast;
      }
      if (n == 0) {
        pl.slot = kConstSlot;  // pow(x, 0) = pow(K, 0) = 1: Hill value 1/2
        pl.a = 0.0f;
        pl.b = 0.0f;
      } else {
        // lg2 of the reference's K^n = pow(K, n) (simophillact.cpp:9-12):
        // n * lg2(K) for a positive K; for K <= 0 lg2 of pow(K, n) itself
        // (positive for an even integer n, NaN -- as the reference's Hill
        // value then is for every x -- for a negative or NaN power).  A K^n
        // of 0 is -inf, so that x = 0 gives the reference's 0/0 = NaN; a
        // repression K^n that overflows is NaN (the reference's inf/inf).
        // A negative K^n (odd integer n) makes the Hill term x^n/(x^n + K^n)
        // non-monotone, which exponent form cannot hold: its term is NaN.
        const double kn = std::pow(lk->dis_const, n);
        double lk2;
        if (kn == 0) lk2 = -HUGE_VAL;
        else if (lk->dis_const > 0) lk2 = n * std::log2(lk->dis_const);
        else lk2 = kn > 0 ? std::log2(kn) : std::nan("");
        if (!act && kn == HUGE_VAL) lk2 = std::nan("");
        pl.slot = index_of(lk->regulator);
        pl.a = (float)(act ? -n : n);
        pl.b = (float)(act ? lk2 : -lk2);
        hdr.lg_mask |= 1u << pl.slot;
      }
      plinks.push_back(pl);
    };
    for (const grn_link *lk : or_l) emit(lk);
    for (const grn_link *lk : and_l) emit(lk);
    g.n_or = (uint8_t)or_l.size();
    g.n_and = (uint8_t)and_l.size();
    if ((int)plinks.size() > GRN_MAX_LINKS || or_l.size() > 255 || and_l.size() > 255) {
      if (err) *err = "model " + std::to_string(orig_index) + ": more than " +
                      std::to_string(GRN_MAX_LINKS) + " used links";
      return GRN_ERR_CAPACITY;
    }
    if (g.n_or + g.n_and > 0) ++c.reg_genes;
  }
  // The kernel's dense regulation holds one link per (regulated, regulator)
  // pair; a model with a repeated pair takes the exact path.
  for (size_t i = 0; i < plinks.size() && (hdr.flags & kFlagFast); ++i)
    for (size_t j = i + 1; j < plinks.size(); ++j)
      if (plinks[i].slot == plinks[j].slot && plinks[i].slot != kConstSlot) {
        // same slot twice within one gene's link range?
        int gi = -1, gj = -1;
        for (int q = 0; q < G; ++q) {
          const int b = genes[q].link_begin, e = b + genes[q].n_or + genes[q].n_and;
          if ((int)i >= b && (int)i < e) gi = q;
          if ((int)j >= b && (int)j < e) gj = q;
        }
        if (gi == gj) {
          hdr.flags &= ~kFlagFast;
          break;
        }
      }
  hdr.n_links = (int16_t)plinks.size();
  c.links = (int)plinks.size();
  c.lg_genes = __builtin_popcount(hdr.lg_mask);
  // Relative cost of one cell-step: MUFU ops weigh 8 issue slots' worth of
  // pipe time, a link ~5 instructions, a gene ~16.
  c.cost = 8.0 * (c.lg_genes + 2 * c.reg_genes) / 4.0 + 5.0 * c.links + 16.0 * G;

  const size_t w0 = out->size();
  out->resize(w0 + record_words(G, (int)plinks.size()));
  uint4 *w = out->data() + w0;
  std::memcpy(w, &hdr, sizeof hdr);
  if (G) std::memcpy(w + 1, genes.data(), sizeof(PackedGene) * G);
  if (!plinks.empty())
    std::memcpy(w + 1 + G, plinks.data(), sizeof(PackedLink) * plinks.size());
  if (cost) *cost = c;
  return GRN_OK;
}

bool euler_bounded(const PackedGene *genes, int n_genes, float dt, int n_steps) {
  bool ok = dt >= 0.0f;
  for (int p = 0; p < n_genes; ++p) {
    const PackedGene &g = genes[p];
    ok = ok && g.deg >= 0.0f && dt * (g.deg + 4.0f * g.dif) <= 1.0f &&
         (float)n_steps * dt * std::max(g.lim, 0.0f) <= kFastMaxGrowth;
  }
  return ok;
}

grn_status pack_batch(const grn_model_batch *batch, int n_morphogens, float dt, int n_steps,
                      int n_threads, PackedHost *out, std::string *err) {
  grn::TraceRange trace_range("grn pack_batch");
  const int n = batch->n_models;
  std::vector<std::vector<uint4>> recs(n);
  std::vector<ModelCost> costs(n);
  std::atomic<int> next{0};
  std::atomic<int> status{GRN_OK};
  std::string first_err;
  std::atomic<bool> err_taken{false};
  auto worker = [&]() {
    for (;;) {
      const int m = next.fetch_add(1);
      if (m >= n || status.load() != GRN_OK) break;
      const int p0 = batch->product_offsets[m], p1 = batch->product_offsets[m + 1];
      const int l0 = batch->link_offsets[m], l1 = batch->link_offsets[m + 1];
      std::string e;
      grn_status s = pack_model(batch->products + p0, p1 - p0, batch->links + l0,
                                l1 - l0, n_morphogens, m, &recs[m], &costs[m], &e);
      if (s == GRN_OK) {
        // The fast path also needs a bounded Euler step at this dt.
        PackedHeader hdr;
        std::memcpy(&hdr, recs[m].data(), sizeof hdr);
        std::vector<PackedGene> genes(hdr.n_genes);
        if (hdr.n_genes > 0)
          std::memcpy(genes.data(), recs[m].data() + 1, sizeof(PackedGene) * hdr.n_genes);
        if ((hdr.flags & kFlagFast) && !euler_bounded(genes.data(), hdr.n_genes, dt, n_steps)) {
          hdr.flags &= ~kFlagFast;
          std::memcpy(recs[m].data(), &hdr, sizeof hdr);
        }
      }
      if (s != GRN_OK) {
        bool expected = false;
        if (err_taken.compare_exchange_strong(expected, true)) first_err = e;
        status.store(s);
      }
    }
  };
  if (n_threads < 1) n_threads = 1;
  if (n < 256) n_threads = 1;
  n_threads = std::min(n_threads, 16);
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; ++t) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
  if (status.load() != GRN_OK) {
    if (err) *err = first_err;
    return (grn_status)status.load();
  }

  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return costs[a].cost > costs[b].cost; });
  size_t total = 0;
  for (int m = 0; m < n; ++m) total += recs[m].size();
  out->words.clear();
  out->words.reserve(total);
  out->offsets.resize(n);
  out->n_models = n;
  out->max_genes = out->max_links = 0;
  out->sum_genes = out->sum_links = 0;
  out->sfu_per_cell_step = out->fma_per_cell_step = 0;
  out->sum_dif_genes = 0;
  out->alg_sfu_per_cell_step = out->alg_fp32_per_cell_step = 0;
  for (int i = 0; i < n; ++i) {
    const int m = order[i];
    out->offsets[i] = (int32_t)out->words.size();
    out->words.insert(out->words.end(), recs[m].begin(), recs[m].end());
    const ModelCost &c = costs[m];
    out->max_genes = std::max(out->max_genes, c.genes);
    out->max_links = std::max(out->max_links, c.links);
    out->sum_genes += c.genes;
    out->sum_links += c.links;
    out->sfu_per_cell_step += c.lg_genes + 2 * c.reg_genes;
    out->fma_per_cell_step += 2 * c.links + 6 * c.genes + 6 * c.dif_genes;
    out->sum_dif_genes += c.dif_genes;
    out->alg_sfu_per_cell_step += 3 * c.links;
    out->alg_fp32_per_cell_step += 6 * c.links + 7 * c.genes + 8 * c.dif_genes;
  }
  return GRN_OK;
}

}  // namespace grn
