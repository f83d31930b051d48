// grn_gpu.hpp -- C++17 host layer over the C ABI (grn_gpu.h), in the shape
// of the reference's evaluator classes so that C++ search code can switch to
// the B200 evaluator by changing types, not call sites:
//
//   reference (lobolab/grn-gpu-performance)               here
//   ---------------------------------------------------    -------------------------
//   Model: genome and text form                            grn::Model
//     (Src/Model/model.h; text: Src/Model/model.cpp:627-706)
//   CEvaluatorMorphogens(threadId, search) / evaluate      grn::CEvaluatorMorphogens
//     (Src/GPUSimulator/cevaluatormorphogens.h:21-62)
//   Individual: model, parentError, setError, setSimTime   grn::Individual
//     (Src/Search/individual.h:23-33)
//   ErrorCalculator: process / waitForAnyDeme              grn::ErrorCalculator
//     (Src/Search/errorcalculator.h:13-21)
//   ErrorCalculatorMultiThread's GPU workers               grn::ErrorCalculatorB200
//     (Src/UI/Evolution/errorcalculatormultithread.h:26-112)
//
// std::vector stands in for QList.  Errors: the reference aborts the process
// on a CUDA error (Src/GPUSimulator/cerrorhandle.h:21); this layer throws
// grn::Error with the status and the context's message, and never falls
// back to a CPU path (no usable device: GRN_ERR_NO_DEVICE from the
// evaluator's constructor).  One evaluator (and the calculators using it)
// per host thread, as the reference keeps one CEvaluatorMorphogens per GPU
// worker thread.  Header-only; link against libgrn_b200.so.
#ifndef GRN_GPU_HPP_
#define GRN_GPU_HPP_

#include <chrono>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "grn_gpu.h"

namespace grn {

// A failed C ABI call.
class Error : public std::runtime_error {
 public:
  Error(grn_status status, const std::string &what) : std::runtime_error(what), status_(status) {}
  grn_status status() const { return status_; }

 private:
  grn_status status_;
};

// Throws grn::Error unless s is GRN_OK; the message names the call and, with
// a context, its last error.
inline void check(grn_status s, const grn_ctx *ctx, const char *call) {
  if (s == GRN_OK) return;
  std::string msg = std::string(call) + ": " + grn_status_str(s);
  if (ctx) {
    const char *e = grn_last_error(ctx);
    if (e && *e) msg += " (" + std::string(e) + ")";
  }
  throw Error(s, msg);
}

// A model in genome form: products and links in the reference's order.
struct Model {
  std::vector<grn_product> products;
  std::vector<grn_link> links;

  // Reads the reference's text form, "(label init lim deg dif|...*from to
  // K n isAnd|...)" (Model::loadFromString and operator>>,
  // Src/Model/model.cpp:614-617, 659-706).
  static Model parse(const std::string &text) {
    Model m;
    int np = 0, nl = 0;
    grn_status s = grn_model_parse(text.c_str(), nullptr, 0, &np, nullptr, 0, &nl);
    if (s != GRN_ERR_CAPACITY) check(s, nullptr, "grn_model_parse");
    m.products.resize(np);
    m.links.resize(nl);
    check(grn_model_parse(text.c_str(), m.products.data(), np, &np, m.links.data(), nl, &nl),
          nullptr, "grn_model_parse");
    return m;
  }

  // The text form (Model::toString and operator<<, model.cpp:619-657) with
  // `precision` significant digits (6: the reference's QTextStream default;
  // 17 round-trips every double).
  std::string str(int precision = 6) const {
    int needed = 0;
    grn_status s = grn_model_format(products.data(), (int)products.size(), links.data(),
                                    (int)links.size(), precision, nullptr, 0, &needed);
    if (s != GRN_ERR_CAPACITY) check(s, nullptr, "grn_model_format");
    std::string buf((size_t)needed, '\0');
    check(grn_model_format(products.data(), (int)products.size(), links.data(),
                           (int)links.size(), precision, &buf[0], needed, &needed),
          nullptr, "grn_model_format");
    buf.resize((size_t)needed - 1);  // drop the terminating 0
    return buf;
  }
};

// Models packed into the C ABI's batch form (grn_model_batch).  The view
// points into this object: keep it alive and unchanged while a call reads
// the view.
class Batch {
 public:
  void add(const Model &m) {
    products_.insert(products_.end(), m.products.begin(), m.products.end());
    links_.insert(links_.end(), m.links.begin(), m.links.end());
    product_offsets_.push_back((int32_t)products_.size());
    link_offsets_.push_back((int32_t)links_.size());
  }
  int size() const { return (int)product_offsets_.size() - 1; }
  grn_model_batch view() const {
    grn_model_batch b{};
    b.n_models = size();
    b.product_offsets = product_offsets_.data();
    b.products = products_.data();
    b.link_offsets = link_offsets_.data();
    b.links = links_.data();
    return b;
  }

 private:
  std::vector<int32_t> product_offsets_{0}, link_offsets_{0};
  std::vector<grn_product> products_;
  std::vector<grn_link> links_;
};

// The GPU evaluator of one host thread: a CUDA device, a stream and the
// experiments uploaded once.
class CEvaluatorMorphogens {
 public:
  // The reference's constructor picks the device from the worker thread id
  // and uploads the search's experiment images once per device
  // (cevaluatormorphogens.cpp:35-90, 92-191).  Here the caller names the
  // device and passes the experiments decoded to planar channels:
  //   initial: [n_experiments][n_input_morphogens][dim_y][dim_x]
  //   target:  [n_experiments][n_target_morphogens][dim_y][dim_x]
  CEvaluatorMorphogens(int device, const grn_sim_params &params, int n_experiments,
                       const double *initial, const double *target) {
    check(grn_create(&ctx_, device, &params), nullptr, "grn_create");
    const grn_status s = grn_set_experiments(ctx_, n_experiments, initial, target);
    if (s != GRN_OK) {
      std::string msg = std::string("grn_set_experiments: ") + grn_status_str(s) + " (" +
                        grn_last_error(ctx_) + ")";
      grn_destroy(ctx_);
      throw Error(s, msg);
    }
  }
  ~CEvaluatorMorphogens() { grn_destroy(ctx_); }
  CEvaluatorMorphogens(const CEvaluatorMorphogens &) = delete;
  CEvaluatorMorphogens &operator=(const CEvaluatorMorphogens &) = delete;

  // CEvaluatorMorphogens::evaluate (cevaluatormorphogens.cpp:233-245): 100
  // if the error exceeds maxError, else the error rounded up to the
  // parameters' errorPrecision significant digits.  Synchronous.
  double evaluate(const Model &model, double maxError) {
    double e = 0.0;
    check(grn_evaluate(ctx_, model.products.data(), (int)model.products.size(),
                       model.links.data(), (int)model.links.size(), maxError, &e),
          ctx_, "grn_evaluate");
    return e;
  }

  // Every model of a batch in one launch; the same values evaluate() gives
  // one by one.  maxError: one per model.
  std::vector<double> evaluate(const Batch &batch, const std::vector<double> &maxError) {
    if ((int)maxError.size() != batch.size())
      throw Error(GRN_ERR_INVALID_ARGUMENT, "evaluate: one maxError per model");
    std::vector<double> out((size_t)batch.size());
    const grn_model_batch b = batch.view();
    check(grn_evaluate_batch(ctx_, &b, maxError.data(), out.data(), nullptr, nullptr), ctx_,
          "grn_evaluate_batch");
    return out;
  }

  grn_ctx *ctx() const { return ctx_; }

 private:
  grn_ctx *ctx_ = nullptr;
};

// The fields of the reference's Individual that an ErrorCalculator reads
// (model, parentError: the maxError of its evaluation) and writes (error,
// simTime).
class Individual {
 public:
  explicit Individual(Model model, double parentError = 1000.0)
      : model_(std::move(model)), parentError_(parentError) {}
  const Model &model() const { return model_; }
  double parentError() const { return parentError_; }
  double error() const { return error_; }
  double simTime() const { return simTime_; }
  void setError(double error) { error_ = error; }
  void setSimTime(double simTime) { simTime_ = simTime; }

 private:
  Model model_;
  double parentError_;
  double error_ = -1.0;
  double simTime_ = 0.0;
};

// Src/Search/errorcalculator.h:13-21.
class ErrorCalculator {
 public:
  virtual ~ErrorCalculator() = default;
  // Queues the individuals of deme nDeme for evaluation; returns at once.
  virtual void process(int nDeme, const std::vector<Individual *> &individuals) = 0;
  // Blocks until every individual of some queued deme has its error, and
  // returns that deme.
  virtual int waitForAnyDeme() = 0;
};

// ErrorCalculator on one GPU evaluator.  The reference's
// ErrorCalculatorMultiThread hands individuals one at a time to worker
// threads, each running CEvaluatorMorphogens::evaluate
// (errorcalculatormultithread.cpp:94-120, 185-229).  Here process() compiles
// the whole deme into one batch and submits it as one persistent launch
// (grn_submit, tag = the deme; several demes may be in flight on the
// evaluator's stream), and waitForAnyDeme() takes the first finished deme
// (grn_wait_any), sets every individual's error (maxError = its
// parentError, as the reference's workers pass it) and simTime (the deme's
// wall seconds from process() to completion, divided by its size; the
// reference times each individual's evaluate call), and returns the deme.
class ErrorCalculatorB200 : public ErrorCalculator {
 public:
  explicit ErrorCalculatorB200(CEvaluatorMorphogens &evaluator) : ev_(evaluator) {}
  ~ErrorCalculatorB200() override {
    // Results of demes still in flight land in buffers owned here: wait for
    // every one (each grn_wait_any call retires one submitted batch).
    while (!pending_.empty()) {
      int tag = kNoDeme;
      const grn_status s = grn_wait_any(ev_.ctx(), -1, &tag);
      if (s == GRN_ERR_NOT_FOUND || s == GRN_ERR_INVALID_ARGUMENT) break;
      pending_.erase(tag);
    }
  }

  void process(int nDeme, const std::vector<Individual *> &individuals) override {
    if (pending_.count(nDeme))
      throw Error(GRN_ERR_INVALID_ARGUMENT, "process: deme already queued");
    std::unique_ptr<Deme> d(new Deme);
    d->individuals = individuals;
    d->max_error.reserve(individuals.size());
    Batch batch;
    for (Individual *ind : individuals) {
      batch.add(ind->model());
      d->max_error.push_back(ind->parentError());
    }
    d->error.assign(individuals.size(), 0.0);
    d->t0 = std::chrono::steady_clock::now();
    const grn_model_batch b = batch.view();  // compiled and copied by grn_submit
    check(grn_submit(ev_.ctx(), nDeme, &b, d->max_error.data(), d->error.data(), nullptr),
          ev_.ctx(), "grn_submit");
    pending_[nDeme] = std::move(d);
  }

  int waitForAnyDeme() override {
    int tag = kNoDeme;
    const grn_status s = grn_wait_any(ev_.ctx(), -1, &tag);
    if (s != GRN_OK) {
      pending_.erase(tag);  // a deme whose evaluation failed is retired too
      check(s, ev_.ctx(), "grn_wait_any");
    }
    auto it = pending_.find(tag);
    if (it == pending_.end()) throw Error(GRN_ERR_NOT_FOUND, "waitForAnyDeme: unknown deme");
    Deme &d = *it->second;
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - d.t0).count();
    const size_t n = d.individuals.size();
    for (size_t i = 0; i < n; ++i) {
      d.individuals[i]->setError(d.error[i]);
      d.individuals[i]->setSimTime(secs / (double)n);
    }
    pending_.erase(it);
    return tag;
  }

 private:
  struct Deme {
    std::vector<Individual *> individuals;
    std::vector<double> max_error, error;
    std::chrono::steady_clock::time_point t0;
  };
  static constexpr int kNoDeme = -2147483647 - 1;
  CEvaluatorMorphogens &ev_;
  std::map<int, std::unique_ptr<Deme>> pending_;
};

}  // namespace grn

#endif  // GRN_GPU_HPP_
