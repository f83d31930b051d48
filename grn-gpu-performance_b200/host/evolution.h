// evolution.h -- island evolutionary search (host side) driving a batched
// fitness evaluator: a Qt-free restatement of the reference's model
// operators (Src/Model/model.cpp, modelprod.cpp, modellink.cpp) and of its
// deterministic-crowding island search (Src/Search/searchalgodetcrowd.cpp,
// Src/Search/search.cpp), run synchronously one generation at a time with
// every deme's children evaluated in one batch.
#ifndef GRN_HOST_EVOLUTION_H_
#define GRN_HOST_EVOLUTION_H_

#include <stdint.h>

#include <istream>
#include <ostream>
#include <random>
#include <vector>

#include "../../include/grn_gpu.h"

namespace grn {

// The reference's MathAlgo random helpers (Src/Common/mathalgo.h:222-286)
// on a seeded mt19937_64.
class Rng {
 public:
  explicit Rng(uint64_t seed) : g_(seed) {}
  bool rand_bool() { return (g_() % 2) == 0; }
  int rand_int(int n) { return (int)(g_() % (uint64_t)n); }
  int rand100() { return std::uniform_int_distribution<int>(0, 99)(g_); }
  int rand1000() { return std::uniform_int_distribution<int>(0, 999)(g_); }
  double rand01() { return std::uniform_real_distribution<double>(0.0, 1.0)(g_); }
  double rand15() { return std::uniform_real_distribution<double>(1.0, 5.0)(g_); }
  // The generator's state in the standard library's text form.
  void save(std::ostream &o) const { o << g_; }
  bool load(std::istream &i) {
    std::mt19937_64 g;
    if (!(i >> g)) return false;
    g_ = g;
    return true;
  }
  template <class T>
  void shuffle(std::vector<T> &v) {  // Durstenfeld, as MathAlgo::shuffle
    for (int i = (int)v.size() - 1; i > 0; --i) {
      int j = (int)(g_() % (uint64_t)(i + 1));
      std::swap(v[i], v[j]);
    }
  }

 private:
  std::mt19937_64 g_;
};

struct GModel {
  std::vector<grn_product> prods;
  std::vector<grn_link> links;
};

// Source of fresh product labels: the reference uses one global counter
// starting after 10 (Model::createNewLabel, model.cpp:373-379); here each
// deme draws from its own interleaved sequence so that parallel demes stay
// deterministic and labels never collide across demes.
struct LabelSource {
  int next;
  int stride;
  int take() {
    int l = next;
    next += stride;
    return l;
  }
};

struct ModelOps {
  int n_morph;     // nMorphogens (also nMinProducts)
  int n_max_prods; // nMaxProducts (-1: no limit)
  int n_max_links; // nMaxLinks (-1: no limit)

  GModel create_random(Rng &rng, int n_products) const;
  void cross(Rng &rng, const GModel &p1, const GModel &p2, GModel *c1, GModel *c2) const;
  void mutate(Rng &rng, LabelSource &labels, GModel *m) const;
  void remove_excess(Rng &rng, GModel *m) const;
  int complexity_in_use(const GModel &m) const;
};

std::vector<int> labels_in_use(const GModel &m, int n_morph);

}  // namespace grn

#endif  // GRN_HOST_EVOLUTION_H_
