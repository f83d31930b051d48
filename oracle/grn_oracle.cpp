// grn_oracle.cpp -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
//
// FP64 CPU restatement of lobolab/grn-gpu-performance's CPU fitness path.
// Each function names the reference lines it follows.  The code is written
// from the reference's behaviour, Qt- and Eigen-free: std::vector planes in
// [k][y][x] order stand in for the Eigen matrices product(k)(x, y), whose
// column-major storage has the same order.
//
// Parity status: numerics unpinned (see grn_oracle.h).

#include "grn_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <thread>
#include <vector>

namespace {

// MathAlgo::max / min (Src/Common/mathalgo.h:208-216): the operand order
// decides which value a NaN comparison returns, so keep it exactly.
inline double ref_max(double a, double b) { return (a < b) ? b : a; }
inline double ref_min(double a, double b) { return (!(b < a)) ? a : b; }

struct Model {
  std::vector<grn_product> prods;
  std::vector<grn_link> links;
};

// Model::prodWithLabel (Src/Model/model.cpp:227-240): first product with
// the label, in model order.
const grn_product *prod_with_label(const Model &m, int label) {
  for (const auto &p : m.prods)
    if (p.label == label) return &p;
  return nullptr;
}

// Model::calcProductLabelsInUse (Src/Model/model.cpp:243-270) with
// calcProductRegulators (:272-283): morphogen labels 0..nMorph-1 are in use,
// and so is every regulator of a product in use (breadth-first walk).
std::set<int> labels_in_use(const Model &m, int n_morph) {
  std::map<int, std::vector<int>> regulators;
  for (const auto &l : m.links) regulators[l.regulated].push_back(l.regulator);
  std::set<int> in_use;
  std::vector<int> to_visit;
  for (int i = 0; i < n_morph; ++i) {
    in_use.insert(i);
    to_visit.push_back(i);
  }
  for (size_t head = 0; head < to_visit.size(); ++head) {
    auto it = regulators.find(to_visit[head]);
    if (it == regulators.end()) continue;
    for (int r : it->second)
      if (in_use.insert(r).second) to_visit.push_back(r);
  }
  return in_use;
}

// The compiled program of ModelSimulator::loadModel
// (Src/Simulator/modelsimulator.cpp:71-203).
enum OpType { OP_HILL_ACT, OP_HILL_REP, OP_OR, OP_AND, OP_ZERO };
struct Op {
  OpType type;
  int to;      // product index, or -1 for the temporary Hill slot
  int from;    // regulator product index (Hill ops)
  double K;    // dissociation constant (Hill ops)
  double n;    // |hill coefficient| (Hill ops)
  double Kn;   // K^n, precomputed as SimOpHill*::disConstN_ (simophillact.cpp:9-12)
};

struct Program {
  std::vector<int> labels;      // sorted labels in use; index = product index
  std::vector<double> lim, deg;
  std::vector<int> dif_ind;     // diffusing product indices, ascending
  std::vector<double> dif_const;
  std::vector<Op> ops;
};

// ModelSimulator::createHillOpForLink (modelsimulator.cpp:194-203).
Op hill_op(const grn_link &l, int from, int to) {
  Op op;
  op.to = to;
  op.from = from;
  op.K = l.dis_const;
  if (l.hill_coef >= 0) {
    op.type = OP_HILL_ACT;
    op.n = l.hill_coef;
  } else {
    op.type = OP_HILL_REP;
    op.n = -1.0 * l.hill_coef;
  }
  op.Kn = std::pow(op.K, op.n);
  return op;
}

// ModelSimulator::loadModel (modelsimulator.cpp:71-154) and
// createProductOps (:156-192).
int compile(const Model &m, int n_morph, Program *prog) {
  std::set<int> in_use = labels_in_use(m, n_morph);
  prog->labels.assign(in_use.begin(), in_use.end());  // qSort(labels_)
  std::map<int, int> index;
  for (size_t i = 0; i < prog->labels.size(); ++i) index[prog->labels[i]] = (int)i;
  const int np = (int)prog->labels.size();
  prog->lim.assign(np, 0.0);
  prog->deg.assign(np, 0.0);
  prog->dif_ind.clear();
  prog->dif_const.clear();
  prog->ops.clear();
  for (int i = 0; i < np; ++i) {
    const grn_product *prod = prod_with_label(m, prog->labels[i]);
    if (!prod) return GRN_ERR_MODEL;  // the reference dereferences NULL here
    prog->lim[i] = prod->lim;
    prog->deg[i] = prod->deg;
    if (prod->dif > 0) {
      prog->dif_ind.push_back(i);
      prog->dif_const.push_back(prod->dif);
    }
    // Model::linksToLabel keeps model link order (model.cpp:391-399).
    std::vector<const grn_link *> or_links, and_links;
    bool any_activator = false;
    for (const auto &l : m.links) {
      if (l.regulated != prog->labels[i]) continue;
      if (in_use.count(l.regulator)) {
        if (l.is_and) and_links.push_back(&l);
        else or_links.push_back(&l);
      }
      if (l.hill_coef >= 0) any_activator = true;  // used or not
    }
    if (!any_activator) {
      prog->ops.push_back(Op{OP_ZERO, i, 0, 0, 0, 0});
      continue;
    }
    bool temp_used = false;
    for (const grn_link *l : or_links) {
      if (temp_used) {
        prog->ops.push_back(hill_op(*l, index[l->regulator], -1));
        prog->ops.push_back(Op{OP_OR, i, 0, 0, 0, 0});
      } else {
        prog->ops.push_back(hill_op(*l, index[l->regulator], i));
        temp_used = true;
      }
    }
    for (const grn_link *l : and_links) {
      if (temp_used) {
        prog->ops.push_back(hill_op(*l, index[l->regulator], -1));
        prog->ops.push_back(Op{OP_AND, i, 0, 0, 0, 0});
      } else {
        prog->ops.push_back(hill_op(*l, index[l->regulator], i));
        temp_used = true;
      }
    }
    if (!temp_used) prog->ops.push_back(Op{OP_ZERO, i, 0, 0, 0, 0});
  }
  return GRN_OK;
}

struct Sim {
  const grn_sim_params *p;
  const Program *prog;
  int W, H, np;
  std::vector<double> state;       // [np][H][W]
  std::vector<double> old_dif;     // snapshot of diffusing planes
  std::vector<double> old_conc, ratios;
  double temp_hill = 0;

  double &at(int k, int x, int y) { return state[((size_t)k * H + y) * W + x]; }

  // SimOp*::compute (Src/Simulator/simophillact.cpp:17-20,
  // simophillrep.cpp:17-20, simopor.cpp:20-22, simopand.cpp:20-22,
  // simopzero.cpp:15-17).
  void run_ops() {
    for (const Op &op : prog->ops) {
      double *to = op.to < 0 ? &temp_hill : &ratios[op.to];
      switch (op.type) {
        case OP_HILL_ACT: {
          double rcn = std::pow(old_conc[op.from], op.n);
          *to = rcn / (rcn + op.Kn);
          break;
        }
        case OP_HILL_REP: {
          double rcn = std::pow(old_conc[op.from], op.n);
          *to = op.Kn / (rcn + op.Kn);
          break;
        }
        case OP_OR: *to = ref_max(temp_hill, *to); break;
        case OP_AND: *to = ref_min(temp_hill, *to); break;
        case OP_ZERO: *to = 0; break;
      }
    }
  }

  // ModelSimulator::simulateStep (Src/Simulator/modelsimulator.cpp:205-280).
  double step() {
    const double dt = p->dt, min_conc = p->min_conc;
    const int nd = (int)prog->dif_ind.size();
    const size_t plane = (size_t)W * H;
    for (int d = 0; d < nd; ++d)
      std::memcpy(&old_dif[d * plane], &state[prog->dif_ind[d] * plane],
                  plane * sizeof(double));
    double max_change = 0;
    for (int j = 0; j < H; ++j) {
      for (int i = 0; i < W; ++i) {
        for (int k = 0; k < np; ++k) old_conc[k] = at(k, i, j);
        run_ops();
        for (int k = 0; k < np; ++k)
          ratios[k] = prog->lim[k] * ratios[k] - prog->deg[k] * old_conc[k];
        for (int d = 0; d < nd; ++d) {
          const double *prod = &old_dif[d * plane];
          double diffusion = 0, total = 0;
          if (i > 0) { diffusion += prod[j * W + i - 1]; ++total; }
          if (i < W - 1) { diffusion += prod[j * W + i + 1]; ++total; }
          if (j > 0) { diffusion += prod[(j - 1) * W + i]; ++total; }
          if (j < H - 1) { diffusion += prod[(j + 1) * W + i]; ++total; }
          int k = prog->dif_ind[d];
          if (diffusion > 0 || (total > 0 && old_conc[k] > 0))
            ratios[k] += prog->dif_const[d] * (diffusion - total * old_conc[k]);
        }
        for (int k = 0; k < np; ++k) {
          double ratio = ratios[k];
          if (ratio) {
            double c = old_conc[k] + dt * ratio;
            at(k, i, j) = (c < min_conc) ? 0 : c;
            max_change = ref_max(max_change, std::fabs(ratio));
          }
        }
      }
    }
    return max_change;
  }

  // Simulator::initialize + loadExperiment (Src/Simulator/simulator.cpp:43-52,
  // simstate.cpp:64-69): input morphogen planes from the experiment, the
  // other products at 0.
  void init(const double *initial) {
    const size_t plane = (size_t)W * H;
    std::fill(state.begin(), state.end(), 0.0);
    for (int k = 0; k < p->n_input_morphogens && k < np; ++k)
      std::memcpy(&state[k * plane], &initial[k * plane], plane * sizeof(double));
  }

  // Simulator::simulate (Src/Simulator/simulator.cpp:54-63).
  double simulate(int n_steps, int *steps_run) {
    double change = 1;
    int step = 0;
    while (step < n_steps && change > p->min_conc_change) {
      change = this->step();
      ++step;
    }
    *steps_run = step;
    return change;
  }

  // SimState::negativeLogLikelihood(const SimState &) (simstate.cpp:135-158).
  double distance(const double *target) {
    const int n_in = p->n_input_morphogens, n_t = p->n_target_morphogens;
    const size_t plane = (size_t)W * H;
    double dist = 0;
    if (p->fitness_kind == GRN_FITNESS_MSE) {
      for (int i = 0; i < W; ++i)
        for (int j = 0; j < H; ++j)
          for (int k = 0; k < n_t; ++k) {
            double d = at(k + n_in, i, j) - target[k * plane + (size_t)j * W + i];
            dist += d * d;
          }
      return dist / ((double)W * H * n_t);
    }
    for (int i = 0; i < W; ++i)
      for (int j = 0; j < H; ++j)
        for (int k = 0; k < n_t; ++k) {
          double a = at(k + n_in, i, j);
          double b = target[k * plane + (size_t)j * W + i];
          double abs_sub = std::fabs(a - b) - p->dist_error_threshold;
          if (abs_sub > 0) dist += std::log(1 + abs_sub);
        }
    return dist / (W * H);
  }
};

Model make_model(const grn_product *prods, int np, const grn_link *links, int nl) {
  Model m;
  m.prods.assign(prods, prods + np);
  m.links.assign(links, links + nl);
  return m;
}

int check_params(const grn_sim_params *p) {
  if (!p || p->dim_x < 1 || p->dim_y < 1 || p->n_input_morphogens < 0 ||
      p->n_input_morphogens > GRN_MAX_INPUT_MORPHOGENS ||
      p->n_target_morphogens < 0 || p->n_target_morphogens > 3 ||
      p->num_sim_steps < 0)
    return GRN_ERR_INVALID_ARGUMENT;
  return GRN_OK;
}

// EvaluatorMorphogens::evaluate (Src/Search/evaluatormorphogens.cpp:48-76),
// returning the unrounded error; rounding is grno_ceil_s / the caller.
int evaluate_raw(const grn_sim_params *p, int n_exp, const double *initial,
                 const double *target, const Model &m, double max_error,
                 double *raw, int *steps_total) {
  Program prog;
  int st = compile(m, p->n_input_morphogens + p->n_target_morphogens, &prog);
  if (st != GRN_OK) return st;
  Sim sim;
  sim.p = p;
  sim.prog = &prog;
  sim.W = p->dim_x;
  sim.H = p->dim_y;
  sim.np = (int)prog.labels.size();
  const size_t plane = (size_t)sim.W * sim.H;
  sim.state.assign(plane * sim.np, 0.0);
  sim.old_dif.assign(plane * prog.dif_ind.size(), 0.0);
  sim.old_conc.assign(sim.np, 0.0);
  sim.ratios.assign(sim.np, 0.0);
  double error = 0.0, change = 0;
  int steps = 0;
  for (int i = 0; i < n_exp && error <= max_error; ++i) {
    sim.init(initial + (size_t)i * p->n_input_morphogens * plane);
    int s = 0;
    change += sim.simulate(p->num_sim_steps, &s);
    steps += s;
    double exp_error = sim.distance(target + (size_t)i * p->n_target_morphogens * plane);
    if (change > p->min_conc_change) exp_error += (change - p->min_conc_change);
    error += exp_error / n_exp;
  }
  *raw = error;
  if (steps_total) *steps_total = steps;
  return GRN_OK;
}

double ceil_s(double n, int d) {
  if (n == 0.0) return 0.0;
  double factor = std::pow(10.0, d - std::ceil(std::log10(std::fabs(n))));
  return std::ceil(n * factor) / factor;
}

// ---- model text format -------------------------------------------------

struct Reader {
  const char *s;
  size_t pos, len;
  int get() { return pos < len ? (unsigned char)s[pos++] : 0; }
  void unget() { if (pos > 0) --pos; }
  // QTextStream >> int: skips leading whitespace, reads an optional sign and
  // digits.
  bool read_int(int *v) {
    while (pos < len && (s[pos] == ' ' || s[pos] == '\n' || s[pos] == '\t' || s[pos] == '\r')) ++pos;
    size_t start = pos;
    if (pos < len && (s[pos] == '-' || s[pos] == '+')) ++pos;
    while (pos < len && s[pos] >= '0' && s[pos] <= '9') ++pos;
    if (pos == start) return false;
    *v = (int)std::strtol(std::string(s + start, pos - start).c_str(), nullptr, 10);
    return true;
  }
  // Model::parseDouble (Src/Model/model.cpp:690-706): characters up to a
  // ' ', '|', '*' or ')' (left unread), converted as QString::toDouble
  // (0 when the token is not a number).
  double read_double() {
    std::string tok;
    while (pos < len) {
      char c = s[pos];
      if (c == ' ' || c == '|' || c == '*' || c == ')') break;
      tok.push_back(c);
      ++pos;
    }
    if (tok.empty()) return 0.0;
    char *end = nullptr;
    double v = std::strtod(tok.c_str(), &end);
    return (end && *end == '\0') ? v : 0.0;
  }
};

}  // namespace

extern "C" {

int grno_evaluate_batch(const grn_sim_params *params, int n_exp,
                        const double *initial, const double *target,
                        const grn_model_batch *batch, const double *max_error,
                        double *error_out, double *raw_out, int32_t *steps_out,
                        int n_threads) {
  int st = check_params(params);
  if (st != GRN_OK) return st;
  if (!batch || n_exp < 1 || !initial || !target || !max_error || !error_out ||
      batch->n_models < 0)
    return GRN_ERR_INVALID_ARGUMENT;
  const int n = batch->n_models;
  if (n_threads < 1) n_threads = 1;
  if (n_threads > n) n_threads = n > 0 ? n : 1;
  std::atomic<int> next{0};
  std::atomic<int> status{GRN_OK};
  // One model per worker at a time from a shared queue
  // (errorcalculatormultithread.cpp:153-199).
  auto worker = [&]() {
    for (;;) {
      int m = next.fetch_add(1);
      if (m >= n) break;
      int p0 = batch->product_offsets[m], p1 = batch->product_offsets[m + 1];
      int l0 = batch->link_offsets[m], l1 = batch->link_offsets[m + 1];
      Model model = make_model(batch->products + p0, p1 - p0, batch->links + l0, l1 - l0);
      double raw = 0;
      int steps = 0;
      int s = evaluate_raw(params, n_exp, initial, target, model, max_error[m], &raw, &steps);
      if (s != GRN_OK) {
        status.store(s);
        raw = NAN;
      }
      // CEvaluatorMorphogens::evaluate / EvaluatorMorphogens::evaluate
      // final rounding (evaluatormorphogens.cpp:70-73).
      error_out[m] = raw > max_error[m] ? 100 : ceil_s(raw, params->error_precision);
      if (raw_out) raw_out[m] = raw;
      if (steps_out) steps_out[m] = steps;
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; ++t) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
  return status.load();
}

int grno_simulate(const grn_sim_params *params, const double *initial,
                  const grn_product *products, int n_products,
                  const grn_link *links, int n_links, int n_steps,
                  double *state_out, int max_planes, int *n_planes_out,
                  double *change_out, int *steps_out) {
  int st = check_params(params);
  if (st != GRN_OK) return st;
  if (!initial || !products || (n_links > 0 && !links) || !state_out)
    return GRN_ERR_INVALID_ARGUMENT;
  Model m = make_model(products, n_products, links, n_links);
  Program prog;
  st = compile(m, params->n_input_morphogens + params->n_target_morphogens, &prog);
  if (st != GRN_OK) return st;
  Sim sim;
  sim.p = params;
  sim.prog = &prog;
  sim.W = params->dim_x;
  sim.H = params->dim_y;
  sim.np = (int)prog.labels.size();
  if (sim.np > max_planes) return GRN_ERR_CAPACITY;
  const size_t plane = (size_t)sim.W * sim.H;
  sim.state.assign(plane * sim.np, 0.0);
  sim.old_dif.assign(plane * prog.dif_ind.size(), 0.0);
  sim.old_conc.assign(sim.np, 0.0);
  sim.ratios.assign(sim.np, 0.0);
  sim.init(initial);
  int steps = 0;
  double change = sim.simulate(n_steps, &steps);
  std::memcpy(state_out, sim.state.data(), plane * sim.np * sizeof(double));
  if (n_planes_out) *n_planes_out = sim.np;
  if (change_out) *change_out = change;
  if (steps_out) *steps_out = steps;
  return GRN_OK;
}

int grno_labels_in_use(const grn_product *products, int n_products,
                       const grn_link *links, int n_links, int n_morphogens,
                       int32_t *labels_out, int max_labels, int *n_out) {
  if (!products || (n_links > 0 && !links) || !labels_out || !n_out)
    return GRN_ERR_INVALID_ARGUMENT;
  Model m = make_model(products, n_products, links, n_links);
  std::set<int> s = labels_in_use(m, n_morphogens);
  if ((int)s.size() > max_labels) return GRN_ERR_CAPACITY;
  int i = 0;
  for (int l : s) labels_out[i++] = l;
  *n_out = i;
  return GRN_OK;
}

int grno_dump_program(const grn_product *products, int n_products,
                      const grn_link *links, int n_links, int n_morphogens,
                      char *buf, int buf_len) {
  if (!products || (n_links > 0 && !links) || !buf || buf_len < 1)
    return GRN_ERR_INVALID_ARGUMENT;
  Model m = make_model(products, n_products, links, n_links);
  Program prog;
  int st = compile(m, n_morphogens, &prog);
  if (st != GRN_OK) return st;
  std::string out;
  char line[160];
  for (const Op &op : prog.ops) {
    switch (op.type) {
      case OP_HILL_ACT:
        std::snprintf(line, sizeof line, "hillact %d %d %.17g %.17g\n", op.to, op.from, op.K, op.n);
        break;
      case OP_HILL_REP:
        std::snprintf(line, sizeof line, "hillrep %d %d %.17g %.17g\n", op.to, op.from, op.K, op.n);
        break;
      case OP_OR: std::snprintf(line, sizeof line, "or %d\n", op.to); break;
      case OP_AND: std::snprintf(line, sizeof line, "and %d\n", op.to); break;
      case OP_ZERO: std::snprintf(line, sizeof line, "zero %d\n", op.to); break;
    }
    out += line;
  }
  if ((int)out.size() + 1 > buf_len) return GRN_ERR_CAPACITY;
  std::memcpy(buf, out.c_str(), out.size() + 1);
  return GRN_OK;
}

double grno_ceil_s(double n, int digits) { return ceil_s(n, digits); }

int grno_decode_rgb(int dim_x, int dim_y, int n_channels, const uint32_t *pixels,
                    double *out) {
  if (dim_x < 1 || dim_y < 1 || n_channels < 0 || n_channels > 3 || !pixels || !out)
    return GRN_ERR_INVALID_ARGUMENT;
  const size_t plane = (size_t)dim_x * dim_y;
  for (int j = 0; j < dim_y; ++j)        // scanline j
    for (int i = 0; i < dim_x; ++i) {
      uint32_t color = pixels[(size_t)j * dim_x + i];
      for (int k = 0; k < n_channels; ++k)
        out[k * plane + (size_t)(dim_y - j - 1) * dim_x + i] =
            ((double)((color >> (16 - (8 * k))) & 0xff)) / 255.0;
    }
  return GRN_OK;
}

int grno_parse_model(const char *text, grn_product *products, int max_products,
                     int *n_products, grn_link *links, int max_links,
                     int *n_links) {
  if (!text || !products || !n_products || !links || !n_links)
    return GRN_ERR_INVALID_ARGUMENT;
  Reader r{text, 0, std::strlen(text)};
  int np = 0, nl = 0;
  // operator>>(QTextStream &, Model &) (Src/Model/model.cpp:659-688)
  int c = r.get();
  if (c != '(') return GRN_ERR_MODEL;
  while (c != '*') {
    if (np >= max_products) return GRN_ERR_CAPACITY;
    grn_product &p = products[np++];
    std::memset(&p, 0, sizeof p);
    // operator>>(QTextStream &, ModelProd &) (Src/Model/modelprod.cpp:81-106)
    if (!r.read_int(&p.label)) return GRN_ERR_MODEL;
    if (r.get() != ' ') return GRN_ERR_MODEL;
    p.init = r.read_double();
    if (r.get() != ' ') return GRN_ERR_MODEL;
    p.lim = r.read_double();
    if (r.get() != ' ') return GRN_ERR_MODEL;
    p.deg = r.read_double();
    if (r.get() != ' ') return GRN_ERR_MODEL;
    p.dif = r.read_double();
    c = r.get();
    if (c == 0) return GRN_ERR_MODEL;
  }
  c = r.get();
  if (c != ')') {
    r.unget();
    while (c != ')') {
      if (nl >= max_links) return GRN_ERR_CAPACITY;
      grn_link &l = links[nl++];
      std::memset(&l, 0, sizeof l);
      // operator>>(QTextStream &, ModelLink &) (Src/Model/modellink.cpp:63-90)
      if (!r.read_int(&l.regulator)) return GRN_ERR_MODEL;
      if (r.get() != ' ') return GRN_ERR_MODEL;
      if (!r.read_int(&l.regulated)) return GRN_ERR_MODEL;
      if (r.get() != ' ') return GRN_ERR_MODEL;
      l.dis_const = r.read_double();
      if (r.get() != ' ') return GRN_ERR_MODEL;
      l.hill_coef = r.read_double();
      if (r.get() != ' ') return GRN_ERR_MODEL;
      int b = 0;
      if (!r.read_int(&b)) return GRN_ERR_MODEL;
      l.is_and = b != 0;
      c = r.get();
      if (c == 0) return GRN_ERR_MODEL;
    }
  }
  *n_products = np;
  *n_links = nl;
  return GRN_OK;
}

int grno_format_model(const grn_product *products, int n_products,
                      const grn_link *links, int n_links, char *buf,
                      int buf_len) {
  if (!products || (n_links > 0 && !links) || !buf || buf_len < 1)
    return GRN_ERR_INVALID_ARGUMENT;
  // operator<<(QTextStream &, Model &) (Src/Model/model.cpp:627-657); doubles
  // use QTextStream's default 6 significant digits.
  std::string out = "(";
  char tmp[256];
  for (int i = 0; i < n_products; ++i) {
    const grn_product &p = products[i];
    std::snprintf(tmp, sizeof tmp, "%d %g %g %g %g", p.label, p.init, p.lim, p.deg, p.dif);
    if (i) out += '|';
    out += tmp;
  }
  out += '*';
  for (int i = 0; i < n_links; ++i) {
    const grn_link &l = links[i];
    std::snprintf(tmp, sizeof tmp, "%d %d %g %g %d", l.regulator, l.regulated,
                  l.dis_const, l.hill_coef, l.is_and ? 1 : 0);
    if (i) out += '|';
    out += tmp;
  }
  out += ')';
  if ((int)out.size() + 1 > buf_len) return GRN_ERR_CAPACITY;
  std::memcpy(buf, out.c_str(), out.size() + 1);
  return GRN_OK;
}

}  // extern "C"
