// Test driver of the C++ host layer (include/grn_gpu.hpp), built and run by
// tests/test_cpp_layer.py.
//
//   evaluator_layer cpu <model text file>
//     Host-only checks: the model text round-trips through grn::Model, a
//     grn::Batch views its models, and creating an evaluator without a CUDA
//     device throws grn::Error(GRN_ERR_NO_DEVICE).  Prints "ok".
//   evaluator_layer gpu <input file> <output file>
//     Evaluates every model of the input three ways -- one by one through
//     CEvaluatorMorphogens::evaluate, as one batch, and deme by deme through
//     ErrorCalculatorB200 (all demes queued, then waited for) -- and writes
//     "index error_one error_batch error_calculator sim_time" per model.
//
// Input file (text): the grn_sim_params fields (dim_x dim_y n_input
// n_target steps precision fitness dt min_conc min_conc_change
// dist_threshold), n_experiments, the initial values, the target values,
// then "n_models n_demes" and per model its deme, its parent error and its
// text form on one line.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "grn_gpu.hpp"

namespace {

int fail(const std::string &what) {
  std::cerr << "FAIL: " << what << "\n";
  return 1;
}

std::string read_file(const char *path) {
  std::ifstream f(path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

int run_cpu(const char *model_file) {
  std::string text = read_file(model_file);
  while (!text.empty() && (text.back() == '\n' || text.back() == ' ')) text.pop_back();
  const grn::Model m = grn::Model::parse(text);
  if (m.products.empty() || m.links.empty()) return fail("parse: empty model");
  if (m.str(6) != text) return fail("text round trip at 6 digits");
  const grn::Model m17 = grn::Model::parse(m.str(17));
  if (m17.str(6) != text) return fail("text round trip at 17 digits");
  try {
    grn::Model::parse("(1 0 0.5 0.5");
    return fail("malformed text accepted");
  } catch (const grn::Error &e) {
    if (e.status() != GRN_ERR_MODEL) return fail("malformed text: wrong status");
  }
  grn::Batch batch;
  batch.add(m);
  batch.add(m);
  const grn_model_batch v = batch.view();
  if (v.n_models != 2 || v.product_offsets[2] != 2 * (int)m.products.size() ||
      v.link_offsets[1] != (int)m.links.size())
    return fail("batch view");
  grn_sim_params p{};
  p.dim_x = 8;
  p.dim_y = 8;
  p.n_input_morphogens = 1;
  p.n_target_morphogens = 1;
  p.num_sim_steps = 10;
  p.error_precision = 8;
  p.dt = 0.1;
  std::vector<double> init(64, 0.5), tgt(64, 0.0);
  try {
    grn::CEvaluatorMorphogens ev(0, p, 1, init.data(), tgt.data());
    return fail("evaluator created without a device");
  } catch (const grn::Error &e) {
    if (e.status() != GRN_ERR_NO_DEVICE) return fail(std::string("no device: ") + e.what());
  }
  std::cout << "ok\n";
  return 0;
}

int run_gpu(const char *in_path, const char *out_path) {
  std::ifstream in(in_path);
  grn_sim_params p{};
  in >> p.dim_x >> p.dim_y >> p.n_input_morphogens >> p.n_target_morphogens >>
      p.num_sim_steps >> p.error_precision >> p.fitness_kind >> p.dt >> p.min_conc >>
      p.min_conc_change >> p.dist_error_threshold;
  int n_exp = 0;
  in >> n_exp;
  const size_t cells = (size_t)p.dim_x * p.dim_y;
  std::vector<double> init((size_t)n_exp * p.n_input_morphogens * cells);
  std::vector<double> tgt((size_t)n_exp * p.n_target_morphogens * cells);
  for (double &v : init) in >> v;
  for (double &v : tgt) in >> v;
  int n_models = 0, n_demes = 0;
  in >> n_models >> n_demes;
  std::vector<int> deme(n_models);
  std::vector<grn::Individual> inds;
  inds.reserve(n_models);
  for (int i = 0; i < n_models; ++i) {
    double parent = 0.0;
    std::string text;
    in >> deme[i] >> parent;
    std::getline(in >> std::ws, text);
    inds.emplace_back(grn::Model::parse(text), parent);
  }
  if (!in) return fail("input file");

  grn::CEvaluatorMorphogens ev(0, p, n_exp, init.data(), tgt.data());
  std::vector<double> one(n_models), batched;
  for (int i = 0; i < n_models; ++i) one[i] = ev.evaluate(inds[i].model(), inds[i].parentError());
  {
    grn::Batch b;
    std::vector<double> me;
    for (const grn::Individual &ind : inds) {
      b.add(ind.model());
      me.push_back(ind.parentError());
    }
    batched = ev.evaluate(b, me);
  }
  {
    grn::ErrorCalculatorB200 calc(ev);
    std::vector<std::vector<grn::Individual *>> demes(n_demes);
    for (int i = 0; i < n_models; ++i) demes[deme[i]].push_back(&inds[i]);
    for (int d = 0; d < n_demes; ++d) calc.process(d, demes[d]);
    try {
      calc.process(0, demes[0]);
      return fail("a deme queued twice");
    } catch (const grn::Error &e) {
      if (e.status() != GRN_ERR_INVALID_ARGUMENT) return fail("queued twice: wrong status");
    }
    std::vector<int> seen(n_demes, 0);
    for (int k = 0; k < n_demes; ++k) {
      const int d = calc.waitForAnyDeme();
      if (d < 0 || d >= n_demes || seen[d]++) return fail("waitForAnyDeme returned a bad deme");
    }
  }
  std::FILE *out = std::fopen(out_path, "w");
  if (!out) return fail("output file");
  for (int i = 0; i < n_models; ++i)
    std::fprintf(out, "%d %.17g %.17g %.17g %.17g\n", i, one[i], batched[i], inds[i].error(),
                 inds[i].simTime());
  std::fclose(out);
  std::cout << "ok\n";
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    if (argc == 3 && std::string(argv[1]) == "cpu") return run_cpu(argv[2]);
    if (argc == 4 && std::string(argv[1]) == "gpu") return run_gpu(argv[2], argv[3]);
  } catch (const std::exception &e) {
    return fail(e.what());
  }
  std::cerr << "usage: evaluator_layer cpu MODEL_FILE | gpu INPUT OUTPUT\n";
  return 2;
}
