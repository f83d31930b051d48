/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * A C interface over the reference's OWN CPU fitness path, compiled from the
 * unchanged reference sources by oracle/build_ref.py into oracle/_ref/:
 *
 *   Src/Search/evaluatormorphogens.cpp   EvaluatorMorphogens::evaluate
 *   Src/Simulator/simulator.cpp          Simulator::loadModel/simulate
 *   Src/Simulator/modelsimulator.cpp     ModelSimulator::loadModel/simulateStep
 *   Src/Simulator/simop*.cpp             Hill / AND / OR / zero ops
 *   Src/Simulator/simstate.cpp           SimState (image decode, distance)
 *   Src/Model/model*.cpp                 Model text parser, labels in use
 *
 * The Qt and Eigen parts those files use come from oracle/shims/qt, and the
 * database-backed classes around them (Search, SimParams, Experiment,
 * MorphologyImage) from oracle/shims/ref.  Tests use this library to pin the
 * FP64 restatement (oracle/grn_oracle.cpp) and the CUDA path to the
 * reference's own arithmetic; bench.py's reference arm times it.
 *
 * Experiments are given the way the reference stores them: as 32-bit RGB
 * images (0xAARRGGBB per pixel, scan lines top to bottom), decoded by
 * SimState::loadMorphologyImage.  Models are given in the reference's text
 * format (Model::loadFromString); 17 significant digits carry every double
 * exactly.
 *
 * Every function returns 0 on success, a grn_status code otherwise.
 */
#include <atomic>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "Model/model.h"
#include "Model/modelprod.h"
#include "Search/evaluatormorphogens.h"
#include "Simulator/simstate.h"
#include "Simulator/simulator.h"
#include "ref_context.h"

#include "grn_gpu.h"

std::atomic<int> qt_subset_assert_failures(0);

using namespace LoboLab;

namespace {

/* The reference's experiment set: one Search holding SimParams and the
 * input/output images of every experiment. */
struct RefSetup {
  SimParams params;
  std::vector<std::unique_ptr<MorphologyImage>> images;
  std::vector<std::unique_ptr<Experiment>> experiments;
  Search search;

  RefSetup(const grn_sim_params *p, int n_exp, const uint32_t *input_px,
           const uint32_t *target_px) {
    params.size = QSize(p->dim_x, p->dim_y);
    params.dt = p->dt;
    params.NumSimSteps = p->num_sim_steps;
    params.nInputMorphogens = p->n_input_morphogens;
    params.nTargetMorphogens = p->n_target_morphogens;
    params.minConc = p->min_conc;
    params.minConcChange = p->min_conc_change;
    params.distErrorThreshold = p->dist_error_threshold;
    params.errorPrecision = p->error_precision;
    const size_t px = static_cast<size_t>(p->dim_x) * p->dim_y;
    for (int e = 0; e < n_exp; ++e) {
      images.emplace_back(new MorphologyImage(QImage(p->dim_x, p->dim_y, input_px + e * px)));
      MorphologyImage *in = images.back().get();
      MorphologyImage *out = in;
      if (target_px) {
        images.emplace_back(new MorphologyImage(QImage(p->dim_x, p->dim_y, target_px + e * px)));
        out = images.back().get();
      }
      experiments.emplace_back(new Experiment(in, out));
      search.experiments_.push_back(experiments.back().get());
    }
    search.simParams_ = &params;
  }
};

bool params_ok(const grn_sim_params *p) {
  return p && p->dim_x > 0 && p->dim_y > 0 && p->n_input_morphogens >= 0 &&
         p->n_target_morphogens >= 0 &&
         p->n_input_morphogens <= 3 && p->n_target_morphogens <= 3 && p->num_sim_steps >= 0 &&
         p->fitness_kind == GRN_FITNESS_REF_LOGTHRESH;
}

/* Parses a model and checks that every product in use exists (the reference
 * dereferences prodWithLabel's result without a check,
 * modelsimulator.cpp:95-97). */
int parse_model(const char *text, int n_morphogens, Model *model) {
  if (!text) return GRN_ERR_INVALID_ARGUMENT;
  const int before = qt_subset_assert_failures.load();
  QString s(text);
  model->loadFromString(s);
  if (qt_subset_assert_failures.load() != before || model->nProducts() == 0)
    return GRN_ERR_MODEL;
  QSet<int> in_use = model->calcProductLabelsInUse(n_morphogens);
  for (int label : in_use)
    if (!model->prodWithLabel(label)) return GRN_ERR_MODEL;
  return GRN_OK;
}

}  // namespace

extern "C" {

int grnr_assert_failures(void) { return qt_subset_assert_failures.load(); }

double grnr_ceil_s(double n, int digits) { return MathAlgo::ceilS(n, digits); }

/* SimState::loadMorphologyImage: out[k][y][x] for k < n_channels. */
int grnr_decode_rgb(int dim_x, int dim_y, int n_channels, const uint32_t *pixels, double *out) {
  if (dim_x <= 0 || dim_y <= 0 || n_channels < 0 || n_channels > 3 || !pixels || !out)
    return GRN_ERR_INVALID_ARGUMENT;
  SimState st(QSize(dim_x, dim_y), n_channels, 0, 0.0);
  MorphologyImage img(QImage(dim_x, dim_y, pixels));
  st.loadMorphologyImage(img, n_channels);
  for (int k = 0; k < n_channels; ++k)
    for (int y = 0; y < dim_y; ++y)
      for (int x = 0; x < dim_x; ++x)
        out[(static_cast<size_t>(k) * dim_y + y) * dim_x + x] = st.product(k)(x, y);
  return GRN_OK;
}

/* Model::calcProductLabelsInUse, sorted as ModelSimulator::loadModel sorts it. */
int grnr_labels_in_use(const char *text, int n_morphogens, int32_t *labels_out, int max_labels,
                       int *n_out) {
  Model model;
  QString s(text ? text : "");
  if (!text) return GRN_ERR_INVALID_ARGUMENT;
  model.loadFromString(s);
  QList<int> labels = model.calcProductLabelsInUse(n_morphogens).toList();
  qSort(labels);
  if (n_out) *n_out = labels.size();
  if (labels.size() > max_labels) return GRN_ERR_CAPACITY;
  for (int i = 0; i < labels.size(); ++i) labels_out[i] = labels[i];
  return GRN_OK;
}

/* Model::loadFromString followed by Model::toString. */
int grnr_format_model(const char *text, char *buf, int buf_len) {
  if (!text || !buf || buf_len <= 0) return GRN_ERR_INVALID_ARGUMENT;
  Model model;
  QString s(text);
  model.loadFromString(s);
  std::string out = model.toString().str();
  if (static_cast<int>(out.size()) + 1 > buf_len) return GRN_ERR_CAPACITY;
  std::memcpy(buf, out.c_str(), out.size() + 1);
  return GRN_OK;
}

/* One model on one experiment through Simulator: loadModel, loadExperiment,
 * initialize, simulate(n_steps) (Src/Simulator/simulator.cpp:35-63).
 * state_out[k][y][x] gets the final state of the products in use (sorted
 * labels); distance_out (may be NULL) the thresholded log distance of that
 * state to the target image (SimState::negativeLogLikelihood,
 * simstate.cpp:135-158) -- target_px may be NULL when distance_out is. */
int grnr_simulate(const grn_sim_params *p, const uint32_t *input_px, const uint32_t *target_px,
                  const char *model_text, int n_steps, double *state_out, int max_planes,
                  int *n_planes_out, double *change_out, int *steps_out, double *distance_out) {
  if (!params_ok(p) || !input_px || n_steps < 0 || (distance_out && !target_px))
    return GRN_ERR_INVALID_ARGUMENT;
  try {
    RefSetup setup(p, 1, input_px, target_px);
    const int n_morph = p->n_input_morphogens + p->n_target_morphogens;
    Model model;
    int st = parse_model(model_text, n_morph, &model);
    if (st != GRN_OK) return st;
    Simulator sim(setup.search);
    sim.loadModel(&model);
    sim.loadExperiment(setup.search.experiment(0));
    sim.initialize();
    double change = sim.simulate(n_steps);
    const SimState &state = sim.simulatedState();
    const int n_prod = sim.nProducts();
    if (n_planes_out) *n_planes_out = n_prod;
    if (change_out) *change_out = change;
    if (steps_out) *steps_out = sim.currStep();
    if (state_out) {
      if (n_prod > max_planes) return GRN_ERR_CAPACITY;
      for (int k = 0; k < n_prod; ++k)
        for (int y = 0; y < p->dim_y; ++y)
          for (int x = 0; x < p->dim_x; ++x)
            state_out[(static_cast<size_t>(k) * p->dim_y + y) * p->dim_x + x] =
                state.product(k)(x, y);
    }
    if (distance_out) {
      SimState target(setup.params.size, p->n_input_morphogens, p->n_target_morphogens,
                      p->dist_error_threshold);
      target.loadMorphologyImage(*setup.search.experiment(0)->outputMorphology(),
                                 p->n_target_morphogens);
      *distance_out = state.negativeLogLikelihood(target);
    }
  } catch (const std::bad_alloc &) {
    return GRN_ERR_OUT_OF_MEMORY;
  } catch (const std::exception &) {
    return GRN_ERR_INVALID_ARGUMENT;
  }
  return GRN_OK;
}

/* EvaluatorMorphogens::evaluate(model, max_error[i]) for every model, by
 * n_threads workers that each own one EvaluatorMorphogens and take the next
 * model from a shared counter, as the reference's CPU calculator threads do
 * (Src/UI/Evolution/errorcalculatormultithread.cpp:123-229).  error_out[i] is
 * the reference's return value: 100 when the error passed max_error, else the
 * error rounded up to error_precision significant digits. */
int grnr_evaluate_batch(const grn_sim_params *p, int n_exp, const uint32_t *input_px,
                        const uint32_t *target_px, int n_models, const char *const *model_texts,
                        const double *max_error, double *error_out, int n_threads) {
  if (!params_ok(p) || n_exp <= 0 || !input_px || !target_px || n_models < 0 ||
      (n_models > 0 && (!model_texts || !max_error || !error_out)))
    return GRN_ERR_INVALID_ARGUMENT;
  try {
    RefSetup setup(p, n_exp, input_px, target_px);
    const int n_morph = p->n_input_morphogens + p->n_target_morphogens;
    std::vector<std::unique_ptr<Model>> models(static_cast<size_t>(n_models));
    for (int i = 0; i < n_models; ++i) {
      models[i].reset(new Model());
      int st = parse_model(model_texts[i], n_morph, models[i].get());
      if (st != GRN_OK) return st;
    }
    if (n_threads < 1) n_threads = 1;
    if (n_threads > n_models) n_threads = n_models > 0 ? n_models : 1;
    std::atomic<int> next(0);
    auto worker = [&]() {
      EvaluatorMorphogens evaluator(setup.search);
      for (int i = next++; i < n_models; i = next++)
        error_out[i] = evaluator.evaluate(*models[i], max_error[i]);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < n_threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
  } catch (const std::bad_alloc &) {
    return GRN_ERR_OUT_OF_MEMORY;
  } catch (const std::exception &) {
    return GRN_ERR_INVALID_ARGUMENT;
  }
  return GRN_OK;
}

}  // extern "C"
