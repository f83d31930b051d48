/*
 * grn_oracle.h -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * FP64 CPU restatement of the reference's CPU fitness path
 * (lobolab/grn-gpu-performance, Src/Simulator + Src/Search/evaluatormorphogens.cpp),
 * used only as the checker in tests/, by __graft_entry__.smoke() and as the
 * CPU baseline leg of bench.py.  The product (grn-gpu-performance_b200/) never
 * links or calls it.
 *
 * Parity status: NUMERICS UNPINNED.  The reference cannot be built here (it
 * needs Qt5 and Eigen) and ships no golden fitness values that can be re-run
 * (its only known answer, errorcalculatormultithread.cpp:61-62, needs
 * experiment images from an unshipped database).  The model-text parser and
 * the op-program compiler are pinned against the reference's test-model
 * string fixture; the numerics are cross-checked against a second,
 * independent pure-Python restatement (oracle/pyoracle.py).
 *
 * All functions return grn_status codes from include/grn_gpu.h.
 */
#ifndef GRN_ORACLE_H_
#define GRN_ORACLE_H_

#include "../include/grn_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Evaluates a batch of models with a pool of n_threads worker threads that
 * pull one model at a time from a shared queue, as the reference's CPU
 * workers do (Src/UI/Evolution/errorcalculatormultithread.cpp:153-229).
 *   initial: [n_exp][n_input_morphogens][H][W], target: [n_exp][n_target][H][W]
 *   error_out: rounded fitness (100 if > max_error, else ceilS)
 *   raw_out:   unrounded error (may be NULL)
 *   steps_out: Euler steps run summed over experiments (may be NULL) */
int grno_evaluate_batch(const grn_sim_params *params, int n_exp,
                        const double *initial, const double *target,
                        const grn_model_batch *batch, const double *max_error,
                        double *error_out, double *raw_out, int32_t *steps_out,
                        int n_threads);

/* Simulates one model on one experiment's initial state for at most n_steps
 * steps (early exit on min_conc_change as Simulator::simulate) and returns the
 * final state [n_products][H][W] (state_out must hold GRN_MAX_GENES planes,
 * or more if the model has more products in use: see max_planes). */
int grno_simulate(const grn_sim_params *params, const double *initial,
                  const grn_product *products, int n_products,
                  const grn_link *links, int n_links, int n_steps,
                  double *state_out, int max_planes, int *n_planes_out,
                  double *change_out, int *steps_out);

/* Labels in use, sorted (Model::calcProductLabelsInUse + qSort). */
int grno_labels_in_use(const grn_product *products, int n_products,
                       const grn_link *links, int n_links, int n_morphogens,
                       int32_t *labels_out, int max_labels, int *n_out);

/* Text listing of the compiled op program, one op per line:
 *   "hillact to from K n" / "hillrep to from K n" / "or to" / "and to" /
 *   "zero to", with to = -1 for the temporary Hill slot. */
int grno_dump_program(const grn_product *products, int n_products,
                      const grn_link *links, int n_links, int n_morphogens,
                      char *buf, int buf_len);

/* MathAlgo::ceilS (Src/Common/mathalgo.h:55-62). */
double grno_ceil_s(double n, int digits);

/* SimState::loadMorphologyImage (Src/Simulator/simstate.cpp:71-90). */
int grno_decode_rgb(int dim_x, int dim_y, int n_channels,
                    const uint32_t *pixels, double *out);

/* Model text format (Src/Model/model.cpp:627-706, modelprod.cpp:74-106,
 * modellink.cpp:56-90). */
int grno_parse_model(const char *text, grn_product *products, int max_products,
                     int *n_products, grn_link *links, int max_links,
                     int *n_links);
int grno_format_model(const grn_product *products, int n_products,
                      const grn_link *links, int n_links, char *buf,
                      int buf_len);

#ifdef __cplusplus
}
#endif

#endif /* GRN_ORACLE_H_ */
