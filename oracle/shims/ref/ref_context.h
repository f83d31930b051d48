/*
 * ref_context.h -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * Stand-ins for the reference classes around its CPU fitness path that live
 * in its SQLite persistence layer (Src/DB, Src/Experiment, Src/Search/search.h,
 * Src/Simulator/simparams.h).  The reference's Simulator and
 * EvaluatorMorphogens read only these members of them:
 *
 *   SimParams   size, dt, NumSimSteps, nSims, nInputMorphogens,
 *               nTargetMorphogens, minConc, minConcChange,
 *               distErrorThreshold, errorPrecision
 *               (Src/Simulator/simulator.cpp:12-27,
 *                Src/Search/evaluatormorphogens.cpp:19-36)
 *   Search      simParams(), nExperiments(), experiment(i)
 *   Experiment  inputMorphology(), outputMorphology()
 *   MorphologyImage  image()  (Src/Simulator/simstate.cpp:71-90)
 *
 * Here they are plain objects that the harness (oracle/ref_harness.cpp) fills
 * from its arguments instead of loading them from a database.
 */
#ifndef GRN_REF_CONTEXT_H_
#define GRN_REF_CONTEXT_H_

#include <vector>

#include "qt_subset.h"

namespace LoboLab {

class DB {};
class DBElement {
 public:
  virtual ~DBElement() {}
};

class SimParams {
 public:
  QSize size;
  double dt = 0;
  double dx = 1;
  int NumSimSteps = 0;
  int nSims = 1;
  int nInputMorphogens = 0;
  int nTargetMorphogens = 0;
  int nMaxProducts = 0;
  int nMaxLinks = 0;
  double minConc = 0;
  double minConcChange = 0;
  double distErrorThreshold = 0;
  int errorPrecision = 0;
};

class SearchParams {};

class MorphologyImage {
 public:
  explicit MorphologyImage(const QImage &img) : image_(img) {}
  const QImage &image() const { return image_; }

 private:
  QImage image_;
};

class Experiment {
 public:
  Experiment(MorphologyImage *in, MorphologyImage *out) : in_(in), out_(out) {}
  MorphologyImage *inputMorphology() const { return in_; }
  MorphologyImage *outputMorphology() const { return out_; }

 private:
  MorphologyImage *in_;
  MorphologyImage *out_;
};

class Search {
 public:
  SimParams *simParams() const { return simParams_; }
  int nExperiments() const { return static_cast<int>(experiments_.size()); }
  Experiment *experiment(int i) const { return experiments_[i]; }

  SimParams *simParams_ = nullptr;
  std::vector<Experiment *> experiments_;
};

}  // namespace LoboLab

#endif  // GRN_REF_CONTEXT_H_
