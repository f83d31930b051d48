// evolution.cpp -- island evolutionary search on top of a batched evaluator.
//
// Model operators restate Src/Model/model.cpp (cross :21-85, copyLinks
// :120-184, createRandom :285-315, duplicateProduct :317-333, mutate
// :499-547, removeExcess :550-574), Src/Model/modelprod.cpp:14-59 and
// Src/Model/modellink.cpp:10-53.  Where the reference iterates a QSet (hash
// order) this code iterates labels in ascending order.  The search restates
// SearchAlgoDetCrowd (Src/Search/searchalgodetcrowd.cpp:54-147) and the
// migration of Search (Src/Search/search.cpp:263-311), synchronously: every
// generation all demes reproduce, all children are evaluated in one batch
// (the GPU evaluator runs them in one persistent launch), then each deme
// selects and, every migration_period generations, random deme pairs mix.

#include "evolution.h"
#include "trace.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <sstream>
#include <string>
#include <thread>

namespace grn {

namespace {

bool has(const std::vector<int> &v, int x) { return std::find(v.begin(), v.end(), x) != v.end(); }

std::vector<int> product_labels(const GModel &m) {
  std::vector<int> l;
  for (const auto &p : m.prods)
    if (!has(l, p.label)) l.push_back(p.label);
  std::sort(l.begin(), l.end());
  return l;
}

// ModelProd(nMorphogens, label) (modelprod.cpp:14-24, zeroInit :61-70).
grn_product random_product(Rng &rng, int label, int n_morph) {
  grn_product p{};
  p.label = label;
  p.init = (label == 0 && n_morph > 0) ? -1 : (label == 1 && n_morph > 1) ? -2
         : (label == 2 && n_morph > 2) ? -3 : 0;
  p.lim = rng.rand01();
  p.deg = rng.rand01();
  if (rng.rand100() < 10) p.dif = rng.rand01();
  else p.dif = 0;
  return p;
}

// ModelLink(regulator, regulated) with isActivation = false
// (modellink.cpp:10-22).
grn_link random_link(Rng &rng, int regulator, int regulated) {
  grn_link l{};
  l.regulator = regulator;
  l.regulated = regulated;
  l.dis_const = rng.rand01();
  if (rng.rand_bool()) l.hill_coef = rng.rand15();
  else l.hill_coef = -1.0 * rng.rand15();
  l.is_and = (l.hill_coef < 0) || rng.rand_bool();
  return l;
}

// Model::removeLink(regulator, regulated): the first matching link.
void remove_link(GModel *m, int regulator, int regulated) {
  for (size_t i = 0; i < m->links.size(); ++i)
    if (m->links[i].regulator == regulator && m->links[i].regulated == regulated) {
      m->links.erase(m->links.begin() + i);
      return;
    }
}

void add_or_replace_random_link(Rng &rng, GModel *m, int regulator, int regulated) {
  remove_link(m, regulator, regulated);
  m->links.push_back(random_link(rng, regulator, regulated));
}

bool find_link(const GModel &m, int regulator, int regulated) {
  for (const auto &l : m.links)
    if (l.regulator == regulator && l.regulated == regulated) return true;
  return false;
}

void remove_links_of(GModel *m, int label) {
  m->links.erase(std::remove_if(m->links.begin(), m->links.end(),
                                [&](const grn_link &l) {
                                  return l.regulator == label || l.regulated == label;
                                }),
                 m->links.end());
}

// Model::removeProductWithLabel (model.cpp:352-371).
void remove_product_with_label(GModel *m, int label) {
  for (size_t i = 0; i < m->prods.size(); ++i)
    if (m->prods[i].label == label) {
      m->prods.erase(m->prods.begin() + i);
      remove_links_of(m, label);
      return;
    }
}

// Model::distributeProducts (model.cpp:87-99): each label goes to the
// second set with probability 1/2.
void distribute(Rng &rng, const std::vector<int> &from, std::vector<int> *to1,
                std::vector<int> *to2) {
  for (int l : from) {
    if (rng.rand100() < 50) to2->push_back(l);
    else to1->push_back(l);
  }
}

std::vector<int> set_union(const std::vector<int> &a, const std::vector<int> &b) {
  std::vector<int> u = a;
  for (int x : b)
    if (!has(u, x)) u.push_back(x);
  std::sort(u.begin(), u.end());
  return u;
}

// Model::copyProductsAndLinks (model.cpp:101-184).
void copy_products_and_links(Rng &rng, GModel *to, const GModel &from1,
                             const std::vector<int> &products1, const GModel &from2,
                             const std::vector<int> &products2, int n_morph) {
  for (const auto &p : from1.prods)
    if (has(products1, p.label)) to->prods.push_back(p);
  for (const auto &p : from2.prods)
    if (has(products2, p.label)) to->prods.push_back(p);
  auto regulators = [&](const std::vector<int> &ps) {
    std::vector<int> r = ps;
    std::sort(r.begin(), r.end());
    r.erase(std::remove_if(r.begin(), r.end(), [&](int l) { return l < n_morph; }), r.end());
    return r;
  };
  const std::vector<int> reg1 = regulators(products1), reg2 = regulators(products2);
  for (const auto &l : from1.links) {
    if (!has(products1, l.regulated)) continue;
    if (has(products1, l.regulator) || has(products2, l.regulator)) {
      to->links.push_back(l);
    } else if (!reg2.empty()) {
      const int nr = reg2[rng.rand_int((int)reg2.size())];
      if (!find_link(from1, nr, l.regulated)) {
        grn_link c = l;
        c.regulator = nr;
        to->links.push_back(c);
      }
    }
  }
  for (const auto &l : from2.links) {
    if (!has(products2, l.regulated)) continue;
    if (has(products2, l.regulator) || has(products1, l.regulator)) {
      to->links.push_back(l);
    } else if (!reg1.empty()) {
      const int nr = reg1[rng.rand_int((int)reg1.size())];
      if (!find_link(from2, nr, l.regulated)) {
        grn_link c = l;
        c.regulator = nr;
        to->links.push_back(c);
      }
    }
  }
}

}  // namespace

std::vector<int> labels_in_use(const GModel &m, int n_morph) {
  std::vector<int> in_use;
  for (int i = 0; i < n_morph; ++i) in_use.push_back(i);
  for (size_t h = 0; h < in_use.size(); ++h)
    for (const auto &l : m.links)
      if (l.regulated == in_use[h] && !has(in_use, l.regulator)) in_use.push_back(l.regulator);
  std::sort(in_use.begin(), in_use.end());
  return in_use;
}

GModel ModelOps::create_random(Rng &rng, int n_products) const {
  // Model::createRandom (model.cpp:285-315).
  GModel m;
  for (int i = 0; i < n_products; ++i) m.prods.push_back(random_product(rng, i, n_morph));
  for (int i = 0; i < n_products; ++i) {
    const int n_reg = rng.rand_int(1 + n_products);
    for (int j = 0; j < n_reg; ++j) add_or_replace_random_link(rng, &m, i, rng.rand_int(n_products));
  }
  return m;
}

void ModelOps::cross(Rng &rng, const GModel &p1, const GModel &p2, GModel *c1,
                     GModel *c2) const {
  // Model::cross (model.cpp:21-85).
  const std::vector<int> l1 = product_labels(p1), l2 = product_labels(p2);
  std::vector<int> common, only1, only2;
  for (int l : l1) (has(l2, l) ? common : only1).push_back(l);
  for (int l : l2)
    if (!has(l1, l)) only2.push_back(l);
  std::vector<int> copied, swapped, e11, e12, e22, e21;
  distribute(rng, common, &copied, &swapped);
  distribute(rng, only1, &e11, &e12);
  distribute(rng, only2, &e22, &e21);
  GModel a, b;
  copy_products_and_links(rng, &a, p1, set_union(copied, e11), p2, set_union(swapped, e21), n_morph);
  copy_products_and_links(rng, &b, p2, set_union(copied, e22), p1, set_union(swapped, e12), n_morph);
  if (copied.size() + e11.size() < swapped.size() + e21.size()) std::swap(a, b);
  remove_excess(rng, &a);
  remove_excess(rng, &b);
  *c1 = std::move(a);
  *c2 = std::move(b);
}

void ModelOps::remove_excess(Rng &rng, GModel *m) const {
  // Model::removeExcess (model.cpp:550-574), nMinProducts = nMorphogens.
  if (n_max_prods > -1) {
    std::vector<int> in_use = labels_in_use(*m, n_morph);
    const int n_remove = (int)in_use.size() - n_max_prods;
    if (n_remove > 0) {
      in_use.erase(std::remove_if(in_use.begin(), in_use.end(),
                                  [&](int l) { return l >= 0 && l < n_morph; }),
                   in_use.end());
      for (int i = 0; i < n_remove && !in_use.empty(); ++i) {
        const int k = rng.rand_int((int)in_use.size());
        remove_product_with_label(m, in_use[k]);
        in_use.erase(in_use.begin() + k);
      }
    }
  }
  if (n_max_links > -1) {
    const std::vector<int> in_use = labels_in_use(*m, n_morph);
    std::vector<int> used;  // indices of links in use, model order
    for (size_t i = 0; i < m->links.size(); ++i)
      if (has(in_use, m->links[i].regulator) && has(in_use, m->links[i].regulated))
        used.push_back((int)i);
    const int n_remove = (int)used.size() - n_max_links;
    std::vector<char> drop(m->links.size(), 0);
    for (int i = 0; i < n_remove; ++i) {
      const int k = rng.rand_int((int)used.size());
      drop[used[k]] = 1;
      used.erase(used.begin() + k);
    }
    size_t w = 0;
    for (size_t i = 0; i < m->links.size(); ++i)
      if (!drop[i]) m->links[w++] = m->links[i];
    m->links.resize(w);
  }
}

void ModelOps::mutate(Rng &rng, LabelSource &labels, GModel *m) const {
  // Model::mutate (model.cpp:499-547); nMinProducts = nMorphogens.
  for (int i = (int)m->prods.size() - 1; i >= 0; --i) {
    const int label = m->prods[i].label;
    if (rng.rand100() < 1) {
      // duplicateProduct (model.cpp:317-333)
      grn_product np = m->prods[i];
      np.init = 0;
      np.label = labels.take();
      m->prods.push_back(np);
      add_or_replace_random_link(rng, m, np.label,
                                 m->prods[rng.rand_int((int)m->prods.size())].label);
      const std::vector<int> ls = product_labels(*m);
      const int n_choice = (int)m->prods.size() - n_morph;
      if (n_choice > 0)
        add_or_replace_random_link(rng, m, ls[n_morph + rng.rand_int(n_choice)], np.label);
    }
    if (label >= n_morph && rng.rand1000() < 15) {
      // removeProduct(i) (model.cpp:336-350)
      m->prods.erase(m->prods.begin() + i);
      remove_links_of(m, label);
    }
  }
  for (int i = (int)m->links.size() - 1; i >= 0; --i) {
    if (rng.rand100() < 1) {
      // duplicateLink (model.cpp:472-483)
      grn_link nl = m->links[i];
      const int n = (int)m->prods.size();
      const int regulator = m->prods[rng.rand_int(n)].label;
      const int regulated = m->prods[rng.rand_int(n)].label;
      remove_link(m, regulator, regulated);
      nl.regulator = regulator;
      nl.regulated = regulated;
      m->links.push_back(nl);
    }
    if (rng.rand1000() < 15 && i < (int)m->links.size()) m->links.erase(m->links.begin() + i);
  }
  remove_excess(rng, m);
  // Parameter mutations with probability 1% each (modelprod.cpp:43-59,
  // modellink.cpp:30-41).
  for (auto &p : m->prods) {
    if (rng.rand100() < 1) p.lim = rng.rand01();
    if (rng.rand100() < 1) p.deg = rng.rand01();
    if (rng.rand100() < 1) {
      if (rng.rand_bool()) p.dif = rng.rand01();
      else p.dif = 0;
    }
  }
  for (auto &l : m->links) {
    if (rng.rand100() < 1) l.dis_const = rng.rand01();
    if (rng.rand100() < 1) {
      if (rng.rand_bool()) l.hill_coef = rng.rand15();
      else l.hill_coef = -1.0 * rng.rand15();
    }
    if (l.hill_coef < 0) l.is_and = 1;
    else if (rng.rand100() < 1) l.is_and = rng.rand_bool();
  }
}

int ModelOps::complexity_in_use(const GModel &m) const {
  // Model::calcComplexityInUse (model.cpp:590-611).
  const std::vector<int> in_use = labels_in_use(m, n_morph);
  int c = 0;
  for (const auto &p : m.prods)
    if (has(in_use, p.label)) c += 1 + (p.dif > 0);
  for (const auto &l : m.links)
    if (has(in_use, l.regulator) && has(in_use, l.regulated)) c += 1;
  return c;
}

}  // namespace grn

// ------------------------------------------------------------- the search

namespace {

using grn::GModel;

struct Individual {
  GModel model;
  double error = -1;
  double parent_error = 1000;  // Individual.cpp:19-25: random individuals
  int complexity = 0;
  bool clone = false;  // same simulated program as its paired parent
  const Individual *parent = nullptr;  // paired parent of a child (this generation)
};

struct Deme {
  std::vector<Individual> pop;
  std::vector<Individual> children;
  std::vector<int> perm;  // randPopulationInd_, shuffled in place every generation
  grn::Rng rng{0};
  grn::LabelSource labels{11, 1};
};

}  // namespace

namespace {
struct Flight;  // one half of the demes' children in evaluation (pipelined mode)
}  // namespace

struct grn_evolution {
  grn_evolution_params p{};
  grn::ModelOps ops{};
  grn_error_calculator_fn fn = nullptr;
  void *user = nullptr;
  grn_ctx *ctx = nullptr;  // GPU evaluator (raw errors available), or null
  grn_surrogate *sur = nullptr;
  bool sur_audit = false;  // also simulate the children the surrogate rejects
  int sur_score = GRN_SCORE_PAIRED;  // grn_evolution_set_surrogate_score
  bool skip_clones = false;
  double sim_fraction = 0.25;
  int min_train = 2048, batches = 32, batch = 512;
  float lr = 1e-3f;
  std::vector<Deme> demes;
  grn::Rng search_rng{0};
  int generation = -1;
  std::string last_error;
  // Pipelined mode: demes [0, n/2) and [n/2, n) alternate on the GPU.
  bool pipelined = false;
  bool primed = false;  // both halves' children are in flight
  std::unique_ptr<Flight> flights[2];
  ~grn_evolution();
};

namespace {

// Models of `inds` as one grn_model_batch (views into the vectors).
struct FlatBatch {
  std::vector<int32_t> po{0}, lo{0};
  std::vector<grn_product> prods;
  std::vector<grn_link> links;
  grn_model_batch b{};
  explicit FlatBatch(const std::vector<Individual *> &inds) {
    for (Individual *ind : inds) {
      prods.insert(prods.end(), ind->model.prods.begin(), ind->model.prods.end());
      links.insert(links.end(), ind->model.links.begin(), ind->model.links.end());
      po.push_back((int32_t)prods.size());
      lo.push_back((int32_t)links.size());
    }
    b.n_models = (int32_t)inds.size();
    b.product_offsets = po.data();
    b.products = prods.empty() ? nullptr : prods.data();
    b.link_offsets = lo.data();
    b.links = links.empty() ? nullptr : links.data();
  }
};

// Evaluates `inds` with max error = their parent's error.  raw_out gets the
// unrounded errors when the GPU evaluator is used, else the rounded ones.
grn_status evaluate_all(grn_evolution *evo, std::vector<Individual *> &inds,
                        std::vector<double> *raw_out) {
  grn::TraceRange trace_range("grn evaluate children");
  FlatBatch fb(inds);
  std::vector<double> max_err, err(inds.size()), raw(inds.size());
  for (Individual *ind : inds) max_err.push_back(ind->parent_error);
  grn_status s;
  if (evo->ctx)
    s = grn_evaluate_batch(evo->ctx, &fb.b, max_err.data(), err.data(), raw.data(), nullptr);
  else
    s = evo->fn(evo->user, &fb.b, max_err.data(), err.data());
  if (s != GRN_OK) return s;
  for (size_t i = 0; i < inds.size(); ++i) inds[i]->error = err[i];
  if (raw_out) *raw_out = evo->ctx ? raw : err;
  return GRN_OK;
}

// What the simulation of a model reads, in FP64: the first product of every
// label in use (ascending), then every link whose regulated label is in use,
// in model order.  Models with equal keys have equal errors under any
// deterministic evaluator.
std::vector<double> program_key(const GModel &m, int n_morph) {
  const std::vector<int> in_use = grn::labels_in_use(m, n_morph);
  std::vector<double> k;
  for (int label : in_use) {
    const grn_product *p = nullptr;
    for (const auto &q : m.prods)
      if (q.label == label) {
        p = &q;
        break;
      }
    k.push_back(label);
    if (p) {
      k.push_back(p->lim);
      k.push_back(p->deg);
      k.push_back(p->dif);
    } else {
      k.push_back(std::nan(""));  // never equal: the evaluator reports the error
    }
  }
  for (const auto &l : m.links)
    if (std::binary_search(in_use.begin(), in_use.end(), l.regulated)) {
      k.push_back(l.regulator);
      k.push_back(l.regulated);
      k.push_back(l.dis_const);
      k.push_back(l.hill_coef);
      k.push_back(l.is_and != 0);
    }
  return k;
}

bool same_key(const std::vector<double> &a, const std::vector<double> &b) {
  return a.size() == b.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(double)) == 0 &&
         std::all_of(a.begin(), a.end(), [](double x) { return x == x; });
}

// Adds simulated pairs to the surrogate's training set and trains it.  A
// simulation abandoned past the parent's error leaves a lower bound (the raw
// error reached so far, or the parent's error behind the rounded 100 of a
// callback evaluator); it is kept as the target, so that the set is not
// biased towards children that beat their parents.
grn_status feed_surrogate(grn_evolution *evo, const std::vector<Individual *> &inds,
                          const std::vector<double> &raw, grn_generation_stats *st) {
  grn::TraceRange trace_range("grn surrogate training");
  std::vector<Individual *> keep;
  std::vector<float> target;
  for (size_t i = 0; i < inds.size(); ++i) {
    double r = raw[i];
    if (!evo->ctx && r == 100.0 && inds[i]->parent_error < 100.0) r = inds[i]->parent_error;
    if (!(r > 0) || !std::isfinite(r)) continue;
    keep.push_back(inds[i]);
    target.push_back((float)std::log(r));
  }
  if (!keep.empty()) {
    FlatBatch fb(keep);
    std::vector<float> feat((size_t)keep.size() * GRN_SURROGATE_FEATURES);
    grn_status s = grn_encode_models(&fb.b, evo->ops.n_morph, feat.data());
    if (s == GRN_OK) s = grn_surrogate_add_data(evo->sur, feat.data(), target.data(), (int)keep.size());
    if (s != GRN_OK) return s;
  }
  if (grn_surrogate_data_count(evo->sur) > 0 && evo->batches > 0)
    return grn_surrogate_train_batches(evo->sur, evo->batches, evo->batch, evo->lr,
                                       &st->surrogate_loss);
  return GRN_OK;
}

// Ranks with ties averaged (1-based), for Spearman's rank correlation.
std::vector<double> average_ranks(const std::vector<double> &x) {
  std::vector<int> o(x.size());
  for (size_t i = 0; i < o.size(); ++i) o[i] = (int)i;
  std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return x[a] < x[b]; });
  std::vector<double> r(x.size());
  for (size_t i = 0; i < o.size();) {
    size_t j = i;
    while (j + 1 < o.size() && x[o[j + 1]] == x[o[i]]) ++j;
    for (size_t k = i; k <= j; ++k) r[o[k]] = 0.5 * (double)(i + j) + 1.0;
    i = j + 1;
  }
  return r;
}

double spearman(const std::vector<double> &a, const std::vector<double> &b) {
  if (a.size() < 3) return std::nan("");
  const std::vector<double> ra = average_ranks(a), rb = average_ranks(b);
  const double n = (double)a.size(), mean = (n + 1) / 2;
  double sab = 0, saa = 0, sbb = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    sab += (ra[i] - mean) * (rb[i] - mean);
    saa += (ra[i] - mean) * (ra[i] - mean);
    sbb += (rb[i] - mean) * (rb[i] - mean);
  }
  return saa > 0 && sbb > 0 ? sab / std::sqrt(saa * sbb) : std::nan("");
}

// Quality of one generation's screen, from the simulated children: predicted
// score (log error minus the parent's log error) against the simulated one.
// rho over every simulated child; with an audit (every child simulated), the
// recall of the screen: the share of the truly best k children (k = the
// number it chose) that it chose, and the share of the children that beat
// their parents that it chose.
void screen_quality(const std::vector<Individual *> &todo, const std::vector<float> &pred,
                    const std::vector<char> &chosen, const std::vector<double> &raw_all,
                    const std::vector<char> &simulated, bool audited,
                    grn_generation_stats *st) {
  std::vector<double> p, a;
  std::vector<int> idx;
  for (size_t i = 0; i < todo.size(); ++i) {
    if (!simulated[i]) continue;
    const double r = raw_all[i];
    if (!(r > 0) || !std::isfinite(r)) continue;
    const double lp = std::log(std::max(todo[i]->parent_error, 1e-30));
    p.push_back((double)pred[i] - lp);
    a.push_back(std::log(r) - lp);
    idx.push_back((int)i);
  }
  st->surrogate_rho = spearman(p, a);
  st->surrogate_recall = std::nan("");
  st->surrogate_improver_recall = std::nan("");
  if (!audited || idx.empty()) return;
  size_t k = 0;
  for (char c : chosen) k += c != 0;
  std::vector<int> o(idx.size());
  for (size_t i = 0; i < o.size(); ++i) o[i] = (int)i;
  std::stable_sort(o.begin(), o.end(), [&](int x, int y) { return a[x] < a[y]; });
  size_t hit = 0, top = std::min(k, o.size());
  for (size_t i = 0; i < top; ++i) hit += chosen[idx[o[i]]] != 0;
  st->surrogate_recall = top ? (double)hit / (double)top : std::nan("");
  size_t improvers = 0, kept = 0;
  for (size_t i = 0; i < idx.size(); ++i)
    if (raw_all[idx[i]] < todo[idx[i]]->parent_error) {
      ++improvers;
      kept += chosen[idx[i]] != 0;
    }
  st->surrogate_improver_recall = improvers ? (double)kept / (double)improvers : std::nan("");
}

void fill_stats(grn_evolution *evo, grn_generation_stats *st) {
  double best = 1e300, sum = 0;
  int best_c = 1 << 30;
  long n = 0;
  std::vector<std::pair<double, int>> pts;
  for (const Deme &d : evo->demes)
    for (const Individual &ind : d.pop) {
      sum += ind.error;
      ++n;
      if (ind.error < best || (ind.error == best && ind.complexity < best_c)) {
        best = ind.error;
        best_c = ind.complexity;
      }
      pts.push_back({ind.error, ind.complexity});
    }
  // Non-dominated (error, complexity) points, duplicates included
  // (Search::recalculateParetoFront, search.cpp:349-377).
  std::sort(pts.begin(), pts.end());
  int pareto = 0;
  double last_e = 0;
  int last_c = 1 << 30;
  for (size_t i = 0; i < pts.size(); ++i) {
    if (pts[i].second < last_c || (pts[i].second == last_c && pts[i].first == last_e)) {
      ++pareto;
      last_e = pts[i].first;
      last_c = pts[i].second;
    }
  }
  st->best_error = best;
  st->best_complexity = best_c;
  st->mean_error = n ? sum / n : 0;
  st->pareto_size = pareto;
}

template <class F>
void for_each_deme(grn_evolution *evo, F &&f) {
  const int nd = (int)evo->demes.size();
  int nt = evo->p.n_host_threads > 0 ? evo->p.n_host_threads
                                     : (int)std::max(1u, std::thread::hardware_concurrency());
  nt = std::min(nt, nd);
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t)
    pool.emplace_back([&, t]() {
      for (int d = t; d < nd; d += nt) f(d);
    });
  for (int d = 0; d < nd; d += nt) f(d);
  for (auto &th : pool) th.join();
}

// SearchAlgoDetCrowd::reproduce (searchalgodetcrowd.cpp:63-101).
void reproduce(grn_evolution *evo, Deme &d) {
  d.rng.shuffle(d.perm);
  d.children.clear();
  const int n = (int)d.pop.size();
  for (int i = 0; i + 1 < n; i += 2) {
    const Individual &p1 = d.pop[d.perm[i]], &p2 = d.pop[d.perm[i + 1]];
    Individual c1, c2;
    if (d.rng.rand100() < 75) {
      evo->ops.cross(d.rng, p1.model, p2.model, &c1.model, &c2.model);
    } else {
      c1.model = p1.model;
      c2.model = p2.model;
    }
    evo->ops.mutate(d.rng, d.labels, &c1.model);
    evo->ops.mutate(d.rng, d.labels, &c2.model);
    c1.parent_error = p1.error;
    c2.parent_error = p2.error;
    c1.complexity = evo->ops.complexity_in_use(c1.model);
    c2.complexity = evo->ops.complexity_in_use(c2.model);
    d.children.push_back(std::move(c1));
    d.children.push_back(std::move(c2));
  }
}

// SearchAlgoDetCrowd::chooseNextGeneration (searchalgodetcrowd.cpp:103-147):
// each child replaces its paired parent if its error is not larger.
void choose_next(Deme &d) {
  std::vector<Individual> next;
  next.reserve(d.pop.size());
  const int n = (int)d.pop.size();
  for (int i = 0; i + 1 < n; i += 2) {
    Individual &p1 = d.pop[d.perm[i]], &p2 = d.pop[d.perm[i + 1]];
    Individual &c1 = d.children[i], &c2 = d.children[i + 1];
    next.push_back(c1.error <= p1.error ? std::move(c1) : std::move(p1));
    next.push_back(c2.error <= p2.error ? std::move(c2) : std::move(p2));
  }
  d.pop = std::move(next);
  d.children.clear();
}

// Search::createMigrationPartners + migrateIndividuals (search.cpp:263-311).
void migrate(grn_evolution *evo) {
  const int nd = (int)evo->demes.size();
  std::vector<int> ids(nd);
  for (int i = 0; i < nd; ++i) ids[i] = i;
  evo->search_rng.shuffle(ids);
  for (int i = 0; i + 1 < nd; i += 2) {
    Deme &a = evo->demes[ids[i]], &b = evo->demes[ids[i + 1]];
    const int n = (int)a.pop.size();
    std::vector<int> r(2 * n);
    for (int k = 0; k < 2 * n; ++k) r[k] = k;
    evo->search_rng.shuffle(r);
    std::vector<Individual> all;
    all.reserve(2 * n);
    for (auto &x : a.pop) all.push_back(std::move(x));
    for (auto &x : b.pop) all.push_back(std::move(x));
    a.pop.clear();
    b.pop.clear();
    for (int k = 0; k < n; ++k) a.pop.push_back(std::move(all[r[k]]));
    for (int k = n; k < 2 * n; ++k) b.pop.push_back(std::move(all[r[k]]));
  }
}

grn_status gpu_calculator(void *user, const grn_model_batch *batch, const double *max_error,
                          double *error_out) {
  return grn_evaluate_batch(static_cast<grn_ctx *>(user), batch, max_error, error_out, nullptr,
                            nullptr);
}

double ms_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

// Children of one half of the demes submitted to the GPU evaluator; the
// result arrays stay here until grn_wait_any returns the half's tag.
struct Flight {
  std::vector<Individual *> sim;
  std::unique_ptr<FlatBatch> fb;
  std::vector<double> max_err, err, raw;
  int n_clones = 0;  // children accepted as clones of their parent
  bool active = false;
};

constexpr int kFlightTag = 0x47524e00;  // tags kFlightTag + half

void half_range(const grn_evolution *evo, int half, int *d0, int *d1) {
  const int n = (int)evo->demes.size(), mid = n / 2;
  *d0 = half == 0 ? 0 : mid;
  *d1 = half == 0 ? mid : n;
}

// Reproduces the demes of one half (with clone acceptance) and submits the
// children that need simulating.
grn_status launch_half(grn_evolution *evo, int half, grn_generation_stats *st) {
  int d0, d1;
  half_range(evo, half, &d0, &d1);
  Flight &f = *evo->flights[half];
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  const int nt = std::max(1, std::min(d1 - d0, evo->p.n_host_threads > 0
                                                   ? evo->p.n_host_threads
                                                   : (int)std::thread::hardware_concurrency()));
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&, t] {
      for (int d = d0 + t; d < d1; d += nt) {
        Deme &dm = evo->demes[d];
        reproduce(evo, dm);
        if (!evo->skip_clones) continue;
        for (size_t i = 0; i < dm.children.size(); ++i) {
          Individual &c = dm.children[i];
          const Individual &p = dm.pop[dm.perm[i]];
          c.clone = p.error < 100 && same_key(program_key(c.model, evo->ops.n_morph),
                                              program_key(p.model, evo->ops.n_morph));
          if (c.clone) c.error = p.error;
        }
      }
    });
  for (auto &th : pool) th.join();
  f.sim.clear();
  f.n_clones = 0;
  for (int d = d0; d < d1; ++d)
    for (auto &ind : evo->demes[d].children) {
      if (ind.clone) f.n_clones += 1;
      else f.sim.push_back(&ind);
    }
  f.fb.reset(new FlatBatch(f.sim));
  f.max_err.clear();
  for (Individual *ind : f.sim) f.max_err.push_back(ind->parent_error);
  f.err.assign(f.sim.size(), 0.0);
  f.raw.assign(f.sim.size(), 0.0);
  st->host_ms += ms_since(t0);
  const grn_status s = grn_submit(evo->ctx, kFlightTag + half, &f.fb->b, f.max_err.data(),
                                  f.err.data(), f.raw.data());
  if (s != GRN_OK) return s;
  f.active = true;
  return GRN_OK;
}

// Waits until the half's batch has been evaluated (results in its arrays).
grn_status wait_half(grn_evolution *evo, int half, grn_generation_stats *st) {
  auto t0 = std::chrono::steady_clock::now();
  while (evo->flights[half]->active) {
    int tag = -1;
    const grn_status s = grn_wait_any(evo->ctx, -1, &tag);
    if (s != GRN_OK) return s;
    if (tag == kFlightTag || tag == kFlightTag + 1) evo->flights[tag - kFlightTag]->active = false;
  }
  if (st) st->eval_ms += ms_since(t0);
  return GRN_OK;
}

void settle_half(grn_evolution *evo, int half, grn_generation_stats *st) {
  auto t0 = std::chrono::steady_clock::now();
  Flight &f = *evo->flights[half];
  for (size_t i = 0; i < f.sim.size(); ++i) f.sim[i]->error = f.err[i];
  st->n_evaluated += (int32_t)f.sim.size();
  st->n_clones += f.n_clones;
  int d0, d1;
  half_range(evo, half, &d0, &d1);
  for (int d = d0; d < d1; ++d) choose_next(evo->demes[d]);
  st->host_ms += ms_since(t0);
}

// Drops the children in flight (their parents stay); used before the
// populations are replaced from outside.
grn_status drain(grn_evolution *evo) {
  if (!evo->primed) return GRN_OK;
  for (int h = 0; h < 2; ++h) {
    const grn_status s = wait_half(evo, h, nullptr);
    if (s != GRN_OK) return s;
  }
  for (auto &d : evo->demes) d.children.clear();
  evo->primed = false;
  return GRN_OK;
}

// One generation with the halves' evaluations overlapping the host work:
//   wait half 0, select it, reproduce + submit it (the GPU runs half 1);
//   wait half 1, select it, migrate if due, reproduce + submit half 1
//   (half 0 first if migration held it back).
// The sequence of reproductions, selections and migrations of every deme
// is the synchronous mode's, so the populations are identical.
grn_status pipelined_step(grn_evolution *evo, grn_generation_stats *st) {
  if (!evo->primed) {
    for (int h = 0; h < 2; ++h) {
      const grn_status s = launch_half(evo, h, st);
      if (s != GRN_OK) return s;
    }
    evo->primed = true;
  }
  const bool migrate_now = evo->p.migration_period > 0 && evo->demes.size() > 1 &&
                           (evo->generation + 1) % evo->p.migration_period == 0;
  grn_status s = wait_half(evo, 0, st);
  if (s != GRN_OK) return s;
  settle_half(evo, 0, st);
  if (!migrate_now && (s = launch_half(evo, 0, st)) != GRN_OK) return s;
  if ((s = wait_half(evo, 1, st)) != GRN_OK) return s;
  settle_half(evo, 1, st);
  evo->generation += 1;
  if (migrate_now) {
    migrate(evo);
    st->migrated = 1;
    if ((s = launch_half(evo, 0, st)) != GRN_OK) return s;
  }
  return launch_half(evo, 1, st);
}

}  // namespace

extern "C" {

grn_status grn_evolution_create_cb(const grn_evolution_params *params, int n_morphogens,
                                   grn_error_calculator_fn fn, void *user, grn_evolution **out) {
  if (!params || !fn || !out || params->n_demes < 1 || params->deme_size < 2 ||
      n_morphogens < 1 || params->migration_period < 0)
    return GRN_ERR_INVALID_ARGUMENT;
  grn_evolution *evo = new (std::nothrow) grn_evolution();
  if (!evo) return GRN_ERR_OUT_OF_MEMORY;
  evo->p = *params;
  evo->ops.n_morph = n_morphogens;
  evo->ops.n_max_prods = params->n_max_products;
  evo->ops.n_max_links = params->n_max_links;
  evo->fn = fn;
  evo->user = user;
  evo->search_rng = grn::Rng(params->seed * 0x9E3779B97F4A7C15ull + 0x1234567ull);
  const int pop = params->deme_size + (params->deme_size % 2);  // even, as the reference
  evo->demes.resize(params->n_demes);
  for (int d = 0; d < params->n_demes; ++d) {
    Deme &dm = evo->demes[d];
    dm.rng = grn::Rng(params->seed + 0x51ED27ull * (uint64_t)(d + 1));
    dm.labels = grn::LabelSource{11 + d, params->n_demes};
    dm.perm.resize(pop);
    for (int i = 0; i < pop; ++i) dm.perm[i] = i;
    dm.pop.resize(pop);
  }
  *out = evo;
  return GRN_OK;
}

grn_status grn_evolution_create(const grn_evolution_params *params, int n_morphogens,
                                grn_ctx *ctx, grn_evolution **out) {
  if (!ctx) return GRN_ERR_INVALID_ARGUMENT;
  grn_status s = grn_evolution_create_cb(params, n_morphogens, gpu_calculator, ctx, out);
  if (s == GRN_OK) (*out)->ctx = ctx;
  return s;
}

grn_status grn_evolution_set_skip_clones(grn_evolution *evo, int enable) {
  if (!evo) return GRN_ERR_INVALID_ARGUMENT;
  evo->skip_clones = enable != 0;
  return GRN_OK;
}

grn_status grn_evolution_set_surrogate(grn_evolution *evo, grn_surrogate *s,
                                       double simulate_fraction, int min_train_pairs,
                                       int batches_per_generation, int batch_size, float lr) {
  if (!evo || (s && (!(simulate_fraction > 0) || simulate_fraction > 1 || min_train_pairs < 1 ||
                     batches_per_generation < 0 || batch_size < 1 || !(lr > 0) ||
                     evo->pipelined)))
    return GRN_ERR_INVALID_ARGUMENT;
  evo->sur = s;
  evo->sim_fraction = simulate_fraction;
  evo->min_train = min_train_pairs;
  evo->batches = batches_per_generation;
  evo->batch = batch_size;
  evo->lr = lr;
  return GRN_OK;
}

grn_status grn_evolution_set_surrogate_score(grn_evolution *evo, int score) {
  if (!evo || (score != GRN_SCORE_PARENT_ERROR && score != GRN_SCORE_PAIRED))
    return GRN_ERR_INVALID_ARGUMENT;
  evo->sur_score = score;
  return GRN_OK;
}

grn_status grn_evolution_set_surrogate_audit(grn_evolution *evo, int enable) {
  if (!evo) return GRN_ERR_INVALID_ARGUMENT;
  evo->sur_audit = enable != 0;
  return GRN_OK;
}

grn_evolution::~grn_evolution() {
  if (primed) drain(this);
}

grn_status grn_evolution_set_pipeline(grn_evolution *evo, int enable) {
  if (!evo) return GRN_ERR_INVALID_ARGUMENT;
  if (enable && (!evo->ctx || evo->sur || evo->demes.size() < 2)) {
    evo->last_error = "pipelining needs the GPU evaluator, no surrogate and two or more demes";
    return GRN_ERR_INVALID_ARGUMENT;
  }
  if (!enable) {
    const grn_status s = drain(evo);
    if (s != GRN_OK) return s;
  }
  for (auto &f : evo->flights)
    if (!f) f.reset(new Flight());
  evo->pipelined = enable != 0;
  return GRN_OK;
}

grn_status grn_evolution_step(grn_evolution *evo, grn_generation_stats *stats) {
  grn::TraceRange trace_range("grn_evolution_step");
  if (!evo) return GRN_ERR_INVALID_ARGUMENT;
  grn_generation_stats st{};
  if (evo->pipelined && evo->generation >= 0) {
    const grn_status s = pipelined_step(evo, &st);
    if (s != GRN_OK) {
      evo->last_error = "pipelined generation failed";
      return s;
    }
    st.generation = evo->generation;
    fill_stats(evo, &st);
    if (stats) *stats = st;
    return GRN_OK;
  }
  auto t0 = std::chrono::steady_clock::now();
  std::vector<Individual *> todo;
  if (evo->generation < 0) {
    // SearchAlgoDetCrowd::calcInitialPopulation: random models with
    // nMinProducts = nMorphogens products (searchalgodetcrowd.cpp:54-61).
    for_each_deme(evo, [&](int d) {
      Deme &dm = evo->demes[d];
      for (auto &ind : dm.pop) {
        ind.model = evo->ops.create_random(dm.rng, evo->ops.n_morph);
        ind.parent_error = 1000;
        ind.complexity = evo->ops.complexity_in_use(ind.model);
      }
    });
    for (auto &d : evo->demes)
      for (auto &ind : d.pop) todo.push_back(&ind);
  } else {
    for_each_deme(evo, [&](int d) {
      Deme &dm = evo->demes[d];
      reproduce(evo, dm);
      for (size_t i = 0; i < dm.children.size(); ++i) dm.children[i].parent = &dm.pop[dm.perm[i]];
      if (!(evo->skip_clones || evo->sur)) return;
      // A child whose simulated program equals its paired parent's has the
      // parent's error: accept it without simulating (neutral drift kept).
      for (size_t i = 0; i < dm.children.size(); ++i) {
        Individual &c = dm.children[i];
        const Individual &p = dm.pop[dm.perm[i]];
        c.parent = &p;
        c.clone = p.error < 100 && same_key(program_key(c.model, evo->ops.n_morph),
                                            program_key(p.model, evo->ops.n_morph));
        if (c.clone) c.error = p.error;
      }
    });
    for (auto &d : evo->demes)
      for (auto &ind : d.children) {
        if (ind.clone) st.n_clones += 1;
        else todo.push_back(&ind);
      }
  }
  st.host_ms = ms_since(t0);
  // Surrogate screening: simulate only the most promising children.
  std::vector<Individual *> sim = todo;
  std::vector<float> pred;
  std::vector<char> chosen;
  const bool screened = evo->sur && evo->generation >= 0 &&
                        grn_surrogate_data_count(evo->sur) >= evo->min_train;
  st.surrogate_rho = st.surrogate_recall = st.surrogate_improver_recall = std::nan("");
  if (screened) {
    auto ts = std::chrono::steady_clock::now();
    FlatBatch fb(todo);
    std::vector<float> feat((size_t)todo.size() * GRN_SURROGATE_FEATURES);
    pred.assign(todo.size(), 0.0f);
    grn_status s = grn_encode_models(&fb.b, evo->ops.n_morph, feat.data());
    if (s == GRN_OK) s = grn_surrogate_predict(evo->sur, feat.data(), (int)todo.size(), pred.data());
    if (s != GRN_OK) return s;
    if (evo->sur_score == GRN_SCORE_PAIRED) {
      // Predicted change against the paired parent: the parent goes through
      // the same network, so the error the network makes on a model family
      // largely cancels between a child and its (near-copy) parent.  The
      // score is shifted to the parent's true log error, so that it reads as
      // a predicted log error.
      std::vector<Individual *> parents(todo.size());
      for (size_t i = 0; i < todo.size(); ++i)
        parents[i] = const_cast<Individual *>(todo[i]->parent ? todo[i]->parent : todo[i]);
      FlatBatch pb(parents);
      std::vector<float> pf((size_t)todo.size() * GRN_SURROGATE_FEATURES), pp(todo.size());
      s = grn_encode_models(&pb.b, evo->ops.n_morph, pf.data());
      if (s == GRN_OK) s = grn_surrogate_predict(evo->sur, pf.data(), (int)todo.size(), pp.data());
      if (s != GRN_OK) return s;
      for (size_t i = 0; i < todo.size(); ++i)
        pred[i] = (float)((double)pred[i] - pp[i] +
                          std::log(std::max(todo[i]->parent_error, 1e-30)));
    }
    std::vector<int> order(todo.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    auto score = [&](int i) {
      return (double)pred[i] - std::log(std::max(todo[i]->parent_error, 1e-30));
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return score(a) < score(b); });
    const size_t n_sim = std::max<size_t>(1, (size_t)std::ceil(evo->sim_fraction * todo.size()));
    chosen.assign(todo.size(), 0);
    for (size_t k = 0; k < n_sim && k < order.size(); ++k) chosen[order[k]] = 1;
    if (!evo->sur_audit) {
      sim.clear();
      for (size_t i = 0; i < todo.size(); ++i)
        if (chosen[i]) sim.push_back(todo[i]);
    }
    st.n_screened = (int32_t)todo.size();
    st.surrogate_ms += ms_since(ts);
  }
  auto t1 = std::chrono::steady_clock::now();
  std::vector<double> raw;
  grn_status s = evaluate_all(evo, sim, &raw);
  st.eval_ms = ms_since(t1);
  if (s != GRN_OK) {
    evo->last_error = "batch evaluation failed";
    return s;
  }
  if (screened) {
    // Quality of the screen on what was simulated; then the rejected
    // children lose to their parents (an audit's extra results only feed
    // the statistics: the search and the training set are the unaudited
    // run's).
    std::vector<double> raw_all(todo.size(), std::nan(""));
    std::vector<char> simulated(todo.size(), 0);
    for (size_t i = 0, j = 0; i < todo.size(); ++i)
      if (evo->sur_audit || chosen[i]) {
        raw_all[i] = raw[j++];
        simulated[i] = 1;
      }
    screen_quality(todo, pred, chosen, raw_all, simulated, evo->sur_audit, &st);
    if (evo->sur_audit) {
      std::vector<Individual *> kept;
      std::vector<double> kept_raw;
      for (size_t i = 0; i < todo.size(); ++i)
        if (chosen[i]) {
          kept.push_back(todo[i]);
          kept_raw.push_back(raw_all[i]);
        }
      sim.swap(kept);
      raw.swap(kept_raw);
      st.n_audited = (int32_t)todo.size();
    }
    for (size_t i = 0; i < todo.size(); ++i)
      if (!chosen[i]) todo[i]->error = HUGE_VAL;  // not simulated: its parent stays
  }
  if (evo->sur) {
    auto ts = std::chrono::steady_clock::now();
    s = feed_surrogate(evo, sim, raw, &st);
    st.surrogate_ms += ms_since(ts);
    if (s != GRN_OK) return s;
  }
  auto t2 = std::chrono::steady_clock::now();
  if (evo->generation >= 0)
    for (auto &d : evo->demes) choose_next(d);
  evo->generation += 1;
  if (evo->p.migration_period > 0 && evo->generation > 0 &&
      evo->generation % evo->p.migration_period == 0 && evo->demes.size() > 1) {
    migrate(evo);
    st.migrated = 1;
  }
  st.host_ms += ms_since(t2);
  st.generation = evo->generation;
  st.n_evaluated = (int32_t)sim.size();
  fill_stats(evo, &st);
  if (stats) *stats = st;
  return GRN_OK;
}

grn_status grn_evolution_individual(const grn_evolution *evo, int deme, int index,
                                    grn_product *products, int max_products, int *n_products,
                                    grn_link *links, int max_links, int *n_links,
                                    double *error, int *complexity) {
  if (!evo || deme < 0 || deme >= (int)evo->demes.size() || index < 0 ||
      index >= (int)evo->demes[deme].pop.size())
    return GRN_ERR_INVALID_ARGUMENT;
  const Individual &ind = evo->demes[deme].pop[index];
  if (n_products) *n_products = (int)ind.model.prods.size();
  if (n_links) *n_links = (int)ind.model.links.size();
  if (error) *error = ind.error;
  if (complexity) *complexity = ind.complexity;
  if (products) {
    if ((int)ind.model.prods.size() > max_products) return GRN_ERR_CAPACITY;
    std::copy(ind.model.prods.begin(), ind.model.prods.end(), products);
  }
  if (links) {
    if ((int)ind.model.links.size() > max_links) return GRN_ERR_CAPACITY;
    std::copy(ind.model.links.begin(), ind.model.links.end(), links);
  }
  return GRN_OK;
}

grn_status grn_evolution_set_individual(grn_evolution *evo, int deme, int index,
                                        const grn_product *products, int n_products,
                                        const grn_link *links, int n_links, double error) {
  if (!evo || deme < 0 || deme >= (int)evo->demes.size() || index < 0 ||
      index >= (int)evo->demes[deme].pop.size() || n_products < 0 || n_links < 0 ||
      (n_products && !products) || (n_links && !links))
    return GRN_ERR_INVALID_ARGUMENT;
  // Children in flight were bred from the populations being changed.
  const grn_status ds = drain(evo);
  if (ds != GRN_OK) return ds;
  Individual &ind = evo->demes[deme].pop[index];
  ind.model.prods.assign(products, products + n_products);
  ind.model.links.assign(links, links + n_links);
  ind.error = error;
  ind.complexity = evo->ops.complexity_in_use(ind.model);
  return GRN_OK;
}

grn_status grn_evolution_set_generation(grn_evolution *evo, int generation) {
  if (!evo || generation < 0) return GRN_ERR_INVALID_ARGUMENT;
  const grn_status ds = drain(evo);
  if (ds != GRN_OK) return ds;
  for (const auto &d : evo->demes)
    for (const auto &ind : d.pop)
      if (ind.model.prods.empty()) {
        evo->last_error = "an individual has no model";
        return GRN_ERR_MODEL;
      }
  evo->generation = generation;
  return GRN_OK;
}

}  // extern "C"

// ---- checkpoint ----------------------------------------------------------
//
// Layout (host byte order, this library's struct layouts): magic, version,
// the search's shape, generation, the search RNG, then per deme its RNG,
// label source, pairing permutation and population (error, parent error,
// complexity, products, links).  RNG states go through the standard
// library's text form of std::mt19937_64.

namespace {

constexpr char kCheckpointMagic[8] = {'G', 'R', 'N', 'E', 'V', 'O', 'C', 'K'};
constexpr uint32_t kCheckpointVersion = 1;

struct Writer {
  std::string out;
  template <class T>
  void pod(const T &v) {
    out.append(reinterpret_cast<const char *>(&v), sizeof v);
  }
  void str(const std::string &v) {
    pod((uint64_t)v.size());
    out += v;
  }
  template <class T>
  void vec(const std::vector<T> &v) {
    pod((uint64_t)v.size());
    if (!v.empty()) out.append(reinterpret_cast<const char *>(v.data()), sizeof(T) * v.size());
  }
};

struct Reader {
  const char *p, *end;
  template <class T>
  bool pod(T *v) {
    if ((size_t)(end - p) < sizeof *v) return false;
    std::memcpy(v, p, sizeof *v);
    p += sizeof *v;
    return true;
  }
  bool str(std::string *v, uint64_t max_len) {
    uint64_t n = 0;
    if (!pod(&n) || n > max_len || (uint64_t)(end - p) < n) return false;
    v->assign(p, (size_t)n);
    p += n;
    return true;
  }
  template <class T>
  bool vec(std::vector<T> *v, uint64_t max_n) {
    uint64_t n = 0;
    if (!pod(&n) || n > max_n || (uint64_t)(end - p) / sizeof(T) < n) return false;
    v->resize((size_t)n);
    if (n) std::memcpy(v->data(), p, sizeof(T) * n);
    p += sizeof(T) * n;
    return true;
  }
};

std::string rng_text(const grn::Rng &r) {
  std::ostringstream o;
  r.save(o);
  return o.str();
}

bool rng_from_text(const std::string &t, grn::Rng *r) {
  std::istringstream i(t);
  return r->load(i);
}

}  // namespace

extern "C" {

grn_status grn_evolution_checkpoint(const grn_evolution *evo, void *buf, size_t cap,
                                    size_t *size) {
  if (!evo || !size) return GRN_ERR_INVALID_ARGUMENT;
  if (evo->primed) return GRN_ERR_INVALID_ARGUMENT;  // children in flight (pipelined)
  Writer w;
  w.out.append(kCheckpointMagic, sizeof kCheckpointMagic);
  w.pod(kCheckpointVersion);
  w.pod(evo->p.n_demes);
  w.pod(evo->p.deme_size);
  w.pod(evo->ops.n_morph);
  w.pod(evo->p.n_max_products);
  w.pod(evo->p.n_max_links);
  w.pod(evo->generation);
  w.str(rng_text(evo->search_rng));
  for (const Deme &d : evo->demes) {
    w.str(rng_text(d.rng));
    w.pod(d.labels.next);
    w.pod(d.labels.stride);
    w.vec(d.perm);
    w.pod((uint64_t)d.pop.size());
    for (const Individual &ind : d.pop) {
      w.pod(ind.error);
      w.pod(ind.parent_error);
      w.pod(ind.complexity);
      w.vec(ind.model.prods);
      w.vec(ind.model.links);
    }
  }
  *size = w.out.size();
  if (!buf) return GRN_OK;
  if (cap < w.out.size()) return GRN_ERR_CAPACITY;
  std::memcpy(buf, w.out.data(), w.out.size());
  return GRN_OK;
}

grn_status grn_evolution_restore(grn_evolution *evo, const void *buf, size_t size) {
  if (!evo || !buf) return GRN_ERR_INVALID_ARGUMENT;
  Reader r{static_cast<const char *>(buf), static_cast<const char *>(buf) + size};
  auto bad = [&](const char *why) {
    evo->last_error = std::string("checkpoint: ") + why;
    return GRN_ERR_INVALID_ARGUMENT;
  };
  char magic[sizeof kCheckpointMagic];
  uint32_t version = 0;
  if (!r.pod(&magic) || std::memcmp(magic, kCheckpointMagic, sizeof magic) != 0 ||
      !r.pod(&version) || version != kCheckpointVersion)
    return bad("not a checkpoint of this version");
  int32_t n_demes = 0, deme_size = 0, n_max_products = 0, n_max_links = 0;
  int n_morph = 0, generation = 0;
  if (!r.pod(&n_demes) || !r.pod(&deme_size) || !r.pod(&n_morph) || !r.pod(&n_max_products) ||
      !r.pod(&n_max_links) || !r.pod(&generation))
    return bad("truncated");
  if (n_demes != evo->p.n_demes || deme_size != evo->p.deme_size ||
      n_morph != evo->ops.n_morph || n_max_products != evo->p.n_max_products ||
      n_max_links != evo->p.n_max_links)
    return bad("the search's shape differs");
  // Parse everything before changing the search.
  constexpr uint64_t kMaxText = 1 << 16, kMaxItems = 1 << 24;
  std::string text;
  grn::Rng search_rng{0};
  if (!r.str(&text, kMaxText) || !rng_from_text(text, &search_rng)) return bad("search RNG");
  std::vector<Deme> demes(evo->demes.size());
  for (Deme &d : demes) {
    uint64_t n_pop = 0;
    if (!r.str(&text, kMaxText) || !rng_from_text(text, &d.rng) || !r.pod(&d.labels.next) ||
        !r.pod(&d.labels.stride) || !r.vec(&d.perm, kMaxItems) || !r.pod(&n_pop) ||
        n_pop != (uint64_t)deme_size)
      return bad("deme state");
    d.pop.resize((size_t)n_pop);
    for (Individual &ind : d.pop) {
      if (!r.pod(&ind.error) || !r.pod(&ind.parent_error) || !r.pod(&ind.complexity) ||
          !r.vec(&ind.model.prods, kMaxItems) || !r.vec(&ind.model.links, kMaxItems))
        return bad("individual");
    }
    for (int v : d.perm)
      if (v < 0 || v >= deme_size) return bad("pairing order");
    if (generation >= 0)
      for (const Individual &ind : d.pop)
        if (ind.model.prods.empty()) return bad("an individual has no model");
  }
  if (r.p != r.end) return bad("trailing bytes");
  const grn_status ds = drain(evo);
  if (ds != GRN_OK) return ds;
  evo->search_rng = search_rng;
  evo->demes.swap(demes);
  evo->generation = generation;
  return GRN_OK;
}

grn_status grn_evolution_best(const grn_evolution *evo, int *deme, int *index) {
  if (!evo || !deme || !index || evo->generation < 0) return GRN_ERR_INVALID_ARGUMENT;
  double best = 1e300;
  int best_c = 1 << 30;
  for (int d = 0; d < (int)evo->demes.size(); ++d)
    for (int i = 0; i < (int)evo->demes[d].pop.size(); ++i) {
      const Individual &ind = evo->demes[d].pop[i];
      if (ind.error < best || (ind.error == best && ind.complexity < best_c)) {
        best = ind.error;
        best_c = ind.complexity;
        *deme = d;
        *index = i;
      }
    }
  return GRN_OK;
}

grn_status grn_evolution_destroy(grn_evolution *evo) {
  delete evo;
  return GRN_OK;
}

}  // extern "C"
