/*
 * grn_gpu.h -- C ABI of the B200 GRN fitness evaluator.
 *
 * The evaluator batch-simulates spatial gene-regulatory-network (GRN)
 * reaction-diffusion models with explicit Euler steps on a 2-D grid and scores
 * every model against target expression patterns.  It replaces the GPU
 * evaluator of lobolab/grn-gpu-performance (directory Src/GPUSimulator) and
 * keeps that evaluator's observable behaviour:
 *
 *   reference entry point                               replacement
 *   ---------------------------------------------------  -------------------------
 *   CEvaluatorMorphogens(threadId, search)               grn_create
 *     (Src/GPUSimulator/cevaluatormorphogens.cpp:35-56)
 *   createGPUExperimentDataset / copySimState            grn_set_experiments,
 *     (cevaluatormorphogens.cpp:92-182)                    grn_set_experiments_rgb
 *   CEvaluatorMorphogens::evaluate(model, maxError)      grn_evaluate
 *     (cevaluatormorphogens.cpp:233-245)
 *   CModelSimulator::loadModel + simulateExperiment      grn_pack + grn_run_packed
 *     (Src/GPUSimulator/cmodelsimulator.cpp:114-242)
 *   launchKernel (modelsimulatordevice.cu:253-264)       grn_run_packed
 *   ErrorCalculator::process / waitForAnyDeme            grn_submit / grn_wait_any
 *     (Src/Search/errorcalculator.h:19-20)
 *   ~CEvaluatorMorphogens                                grn_destroy
 *
 * Conventions
 *   - Every function returns a grn_status; nothing aborts the process.  The
 *     reference aborts on any CUDA error (cerrorhandle.h:21); here the caller
 *     decides.  grn_last_error(ctx) gives a one-line description.
 *   - Input buffers are owned by the caller and copied; nothing is retained
 *     after the call returns (except by grn_submit, see there).
 *   - One context per host thread, or external locking.  A context owns one
 *     CUDA stream on one device, like the reference's one evaluator per GPU
 *     worker thread (errorcalculatormultithread.cpp:233-254).
 *   - Grids are planar, row-major: value (x, y) of channel k lives at
 *     [k][y][x] with x < dim_x (width) fastest.  This is the memory order of
 *     the reference CPU simulator's Eigen matrices product(k)(x, y)
 *     (Src/Simulator/modelsimulator.cpp:213-216).
 *   - The product path has no CPU fallback: if no CUDA device is usable,
 *     grn_create returns GRN_ERR_NO_DEVICE.
 */
#ifndef GRN_GPU_H_
#define GRN_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRN_ABI_VERSION 2

/* Capacity limits of the compiled model format.  A model whose products in
 * use or used links exceed these is rejected with GRN_ERR_CAPACITY. */
#define GRN_MAX_GENES 16         /* products in use per model              */
#define GRN_MAX_LINKS 128        /* links from an in-use regulator         */
#define GRN_MAX_INPUT_MORPHOGENS 3  /* R, G, B channels of an input image  */
#define GRN_MAX_EXPERIMENTS 64

typedef enum grn_status {
  GRN_OK = 0,
  GRN_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, bad params     */
  GRN_ERR_NO_DEVICE = 2,        /* no CUDA device / bad device ordinal    */
  GRN_ERR_CUDA = 3,             /* a CUDA runtime call failed             */
  GRN_ERR_OUT_OF_MEMORY = 4,    /* device or pinned host allocation       */
  GRN_ERR_MODEL = 5,            /* incoherent model (missing product ...) */
  GRN_ERR_CAPACITY = 6,         /* model or grid exceeds the kernel limits */
  GRN_ERR_NO_EXPERIMENTS = 7,   /* evaluate before grn_set_experiments    */
  GRN_ERR_TIMEOUT = 8,          /* grn_wait_any ran out of time           */
  GRN_ERR_NOT_FOUND = 9,        /* grn_wait_any with nothing submitted    */
  GRN_ERR_KERNEL = 10           /* the kernel reported an internal error  */
} grn_status;

/* Per-experiment distance between the simulated and the target pattern. */
typedef enum grn_fitness_kind {
  /* The reference's thresholded log distance:
   *   (1/(W*H)) * sum_cells sum_k [|c - t| - theta > 0] * log(1 + |c - t| - theta)
   * (Src/Simulator/simstate.cpp:135-158).  Use this for drop-in parity.     */
  GRN_FITNESS_REF_LOGTHRESH = 0,
  /* Mean squared error over cells and target channels:
   *   (1/(W*H*nTarget)) * sum_cells sum_k (c - t)^2
   * No reference counterpart; the rest of the evaluation (non-convergence
   * penalty, maxError abandon, rounding) is unchanged.                     */
  GRN_FITNESS_MSE = 1
} grn_fitness_kind;

/* Simulation parameters: the fields of the reference SimParams that the
 * fitness path reads (Src/Simulator/simparams.h:25-43). */
typedef struct grn_sim_params {
  int32_t dim_x;                /* SimParams::size.width()                */
  int32_t dim_y;                /* SimParams::size.height()               */
  int32_t n_input_morphogens;   /* SimParams::nInputMorphogens            */
  int32_t n_target_morphogens;  /* SimParams::nTargetMorphogens           */
  int32_t num_sim_steps;        /* SimParams::NumSimSteps (max Euler steps) */
  int32_t error_precision;      /* SimParams::errorPrecision (sig. digits) */
  int32_t fitness_kind;         /* grn_fitness_kind                       */
  int32_t reserved0;
  double dt;                    /* SimParams::dt                          */
  double min_conc;              /* SimParams::minConc                     */
  double min_conc_change;       /* SimParams::minConcChange               */
  double dist_error_threshold;  /* SimParams::distErrorThreshold          */
} grn_sim_params;

/* One gene product of a model (reference ModelProd, Src/Model/modelprod.h). */
typedef struct grn_product {
  int32_t label;   /* product label; labels 0..nMorphogens-1 are morphogens */
  int32_t reserved0;
  double init;     /* ModelProd::init (not read by the simulation)          */
  double lim;      /* production rate                                       */
  double deg;      /* degradation rate                                      */
  double dif;      /* diffusion constant; the product diffuses iff dif > 0  */
} grn_product;

/* One regulatory link (reference ModelLink, Src/Model/modellink.h). */
typedef struct grn_link {
  int32_t regulator;   /* label of the regulating product                  */
  int32_t regulated;   /* label of the regulated product                   */
  double dis_const;    /* Hill dissociation constant K                     */
  double hill_coef;    /* Hill coefficient n; n < 0 means repression       */
  int32_t is_and;      /* 1 = AND regulation, 0 = OR regulation            */
  int32_t reserved0;
} grn_link;

/* A batch of models in genome form: model m owns products
 * [product_offsets[m], product_offsets[m+1]) and links
 * [link_offsets[m], link_offsets[m+1]); both offset arrays have n_models+1
 * entries and start at 0.  Link order inside a model is significant (it is
 * the order of the reference's Model::links_). */
typedef struct grn_model_batch {
  int32_t n_models;
  int32_t reserved0;
  const int32_t *product_offsets;
  const grn_product *products;
  const int32_t *link_offsets;
  const grn_link *links;
} grn_model_batch;

/* Optional statistics of one evaluation call. */
typedef struct grn_eval_stats {
  int64_t n_models;
  int64_t cell_updates;      /* sum over models of steps run x W x H      */
  int64_t total_steps;       /* Euler steps run, summed over models/exps  */
  double kernel_ms;          /* device time of the simulation kernel(s)   */
  double pack_ms;            /* host time compiling the batch             */
  int64_t h2d_bytes;         /* bytes copied host -> device               */
  int64_t d2h_bytes;         /* bytes copied device -> host               */
  int32_t schedule;          /* grn_schedule chosen for the launch        */
  int32_t threads_per_block;
  int32_t blocks;
  int32_t cluster_size;      /* CTAs per model (GRN_SCHEDULE_CLUSTER), else 1 */
} grn_eval_stats;

/* Kernel schedules.  GRN_SCHEDULE_AUTO lets the autotuner pick.  Every
 * schedule double-buffers each gene's state plane: in shared memory as far
 * as it fits, the remaining genes in a per-block global-memory slot. */
typedef enum grn_schedule {
  GRN_SCHEDULE_AUTO = 0,
  GRN_SCHEDULE_FIXED_ITEMS = 1, /* each thread owns fixed float4 groups of
                                   4 cells for the whole launch           */
  GRN_SCHEDULE_WALK_ITEMS = 2,  /* threads walk the grid's groups; any
                                   grid size                              */
  GRN_SCHEDULE_GLOBAL = 3,      /* walking groups, every plane in global
                                   memory                                 */
  GRN_SCHEDULE_CLUSTER = 4,     /* cluster-split: a thread-block cluster
                                   per model, each CTA a band of rows in
                                   its shared memory, halo rows exchanged
                                   through distributed shared memory      */
  GRN_SCHEDULE_STREAM = 5,      /* every plane in global memory; each step
                                   walks bands of rows staged through
                                   shared memory by bulk (TMA) copies,
                                   double-buffered                        */
  GRN_SCHEDULE_STREAM2 = 6      /* as GRN_SCHEDULE_STREAM with temporal
                                   blocking: each pass over the planes
                                   advances two Euler steps (half the
                                   state traffic; step one recomputes one
                                   halo row per band side)                */
} grn_schedule;

typedef struct grn_ctx grn_ctx;
typedef struct grn_packed grn_packed;

/* ---------------------------------------------------------------- context */

/* Creates an evaluator bound to CUDA device `device` with its own stream.
 * Mirrors CEvaluatorMorphogens' constructor (cevaluatormorphogens.cpp:35-56,
 * 64-90), minus the experiment upload, which is grn_set_experiments. */
grn_status grn_create(grn_ctx **out, int device, const grn_sim_params *params);

/* Frees every device and pinned buffer of the context.  Mirrors
 * ~CEvaluatorMorphogens (cevaluatormorphogens.cpp:193-231).  NULL is a no-op. */
grn_status grn_destroy(grn_ctx *ctx);

/* Description of the last error on this context ("" if none). */
const char *grn_last_error(const grn_ctx *ctx);

/* Name of a status code. */
const char *grn_status_str(grn_status status);

/* ABI version compiled into the library (GRN_ABI_VERSION). */
int grn_abi_version(void);

/* Forces a schedule instead of the autotuner's choice (GRN_SCHEDULE_AUTO to
 * restore).  Returns GRN_ERR_CAPACITY later, at launch, if the forced
 * schedule cannot hold the batch. */
grn_status grn_set_schedule(grn_ctx *ctx, int schedule, int threads_per_block);

/* CTAs per cluster for GRN_SCHEDULE_CLUSTER (2, 4, 8 or 16; 0: the
 * autotuner's choice). */
grn_status grn_set_cluster_size(grn_ctx *ctx, int cluster_size);

/* GRN_SCHEDULE_AUTO's plan choice.  enable = 1 (default): measured -- on the
 * first batch of each shape (W, H, most genes, most links, experiments,
 * fast path, batch size below 2 x SMs) up to 8 feasible plans are timed on
 * a sample of the batch (2 to 8 models per SM, spread evenly over its cost
 * order; about 2^29 cell-updates per sample launch, at least 128 steps),
 * in three interleaved rounds after an untimed launch of each; the
 * heuristic's first choice stays unless another plan is 3% faster.  The winner is kept for later
 * batches of that shape (that first call synchronises its stream).
 * enable = 0: an occupancy/spill heuristic, no timing.  Either call clears
 * the cache. */
grn_status grn_set_autotune(grn_ctx *ctx, int enable);

/* The autotuning on this context: a first line starting with '#' that
 * counts the runs so far and their host time, then the last run, one line
 * per timed plan ("*" marks the one kept): schedule, threads, gene
 * capacity, items per thread, cluster size, shared-memory planes, streaming
 * band rows and the fastest sample launch in ms.  GRN_ERR_CAPACITY if it
 * was truncated to buf_len. */
grn_status grn_autotune_report(const grn_ctx *ctx, char *buf, int buf_len);

/* enable = 1: grn_evaluate, grn_evaluate_batch and grn_submit replay one
 * CUDA graph per in-flight job -- copy-in, simulation kernel, copy-out and
 * timing events -- re-captured each call and updated in place (parameters
 * only) while the launch plan keeps its shape, so a generation's GPU work is
 * one graph launch.  A batch shape the autotuner has not timed yet is run
 * once without a graph.  Off by default. */
grn_status grn_set_graphs(grn_ctx *ctx, int enable);

/* Host threads that compile a batch into its packed form (at most 16 are
 * used).  0 (the default): as many as the CPUs this process may run on.
 * Several processes of one node (one per GPU) each want their share. */
grn_status grn_set_host_threads(grn_ctx *ctx, int n_threads);

/* Tests of the error paths only.  GRN_TEST_WITHHOLD_BAND_COPY: the
 * streaming schedule never issues the bulk copy of each step's second band,
 * so the kernel's bounded wait for it runs out (about one second per model),
 * the model's raw error becomes NaN and the call returns GRN_ERR_KERNEL; the
 * context stays usable.  0 restores normal operation. */
#define GRN_TEST_WITHHOLD_BAND_COPY 1
/* GRN_TEST_FAIL_DEVICE_ALLOC: every device allocation the context would make
 * fails, so the call returns GRN_ERR_OUT_OF_MEMORY; buffers it already holds
 * stay usable.  GRN_TEST_CORRUPT_RECORD: the first compiled model record of
 * each call reaches the kernel with a gene count of 0, which the kernel's
 * record check rejects (GRN_ERR_KERNEL, that model's raw error NaN). */
#define GRN_TEST_FAIL_DEVICE_ALLOC 2
#define GRN_TEST_CORRUPT_RECORD 4
grn_status grn_set_test_hooks(grn_ctx *ctx, int hooks);

/* ------------------------------------------------------------ experiments */

/* Uploads the experiments once (the reference uploads them once per device,
 * cevaluatormorphogens.cpp:92-151).
 *   initial: [n_experiments][n_input_morphogens][dim_y][dim_x]
 *   target:  [n_experiments][n_target_morphogens][dim_y][dim_x]
 * Products other than the input morphogens start at 0
 * (Src/Simulator/simstate.cpp:64-69, modelsimulatordevice.cu:134-151). */
grn_status grn_set_experiments(grn_ctx *ctx, int n_experiments,
                               const double *initial, const double *target);

/* Same, from 32-bit 0xAARRGGBB pixels (Qt's QRgb), scanline-major
 * [n_experiments][dim_y][dim_x], the form the reference decodes with QImage.
 * Channel k takes byte (16 - 8k) / 255 and the y axis is flipped, exactly as
 * SimState::loadMorphologyImage (Src/Simulator/simstate.cpp:71-90). */
grn_status grn_set_experiments_rgb(grn_ctx *ctx, int n_experiments,
                                   const uint32_t *input_pixels,
                                   const uint32_t *target_pixels);

/* Decodes 0xAARRGGBB pixels [dim_y][dim_x] into planar channels
 * [n_channels][dim_y][dim_x] with the reference's y flip.  Pure host helper
 * (no device work), exposed so callers can check the decode. */
grn_status grn_decode_rgb(int dim_x, int dim_y, int n_channels,
                          const uint32_t *pixels, double *out);

/* -------------------------------------------------------------- evaluate */

/* Evaluates one model synchronously and returns the reference's fitness:
 * 100 if the error exceeds max_error, else the error rounded UP to
 * error_precision significant digits.  Mirrors
 * CEvaluatorMorphogens::evaluate (cevaluatormorphogens.cpp:233-245). */
grn_status grn_evaluate(grn_ctx *ctx, const grn_product *products,
                        int n_products, const grn_link *links, int n_links,
                        double max_error, double *error_out);

/* Evaluates a batch synchronously in one persistent launch.
 *   max_error:     [n_models] (the parent's error; 1000 for random models)
 *   error_out:     [n_models] rounded fitness as grn_evaluate returns it
 *   raw_error_out: [n_models] unrounded error sum, or NULL
 *   stats:         optional */
grn_status grn_evaluate_batch(grn_ctx *ctx, const grn_model_batch *batch,
                              const double *max_error, double *error_out,
                              double *raw_error_out, grn_eval_stats *stats);

/* Evaluates a batch like grn_evaluate_batch and also returns the final
 * simulated state of every experiment of every model -- the state that
 * SimState::negativeLogLikelihood scores (Src/Simulator/simstate.cpp:135-158)
 * -- for inspection and headless viewers:
 *   states_out: [n_models][n_experiments][max_planes][dim_y][dim_x] FP32,
 *               plane k = product index k (sorted labels in use); planes
 *               beyond a model's products and experiments skipped after
 *               max_error stay 0.
 *   raw_error_out: [n_models] unrounded errors (may be NULL). */
grn_status grn_evaluate_states(grn_ctx *ctx, const grn_model_batch *batch,
                               const double *max_error, double *raw_error_out,
                               float *states_out, int max_planes);

/* Asynchronous form of grn_evaluate_batch, the reference's
 * ErrorCalculator::process(iDeme, individuals) (errorcalculator.h:19).
 * The batch is compiled and copied before the call returns; error_out
 * (and raw_error_out if not NULL) must stay valid until grn_wait_any has
 * returned `tag`. */
grn_status grn_submit(grn_ctx *ctx, int tag, const grn_model_batch *batch,
                      const double *max_error, double *error_out,
                      double *raw_error_out);

/* Blocks until one submitted batch has finished, writes its results and
 * returns its tag: ErrorCalculator::waitForAnyDeme (errorcalculator.h:20).
 * timeout_ms < 0 waits without limit.  GRN_ERR_NOT_FOUND if nothing is
 * pending, GRN_ERR_TIMEOUT if nothing finished in time. */
grn_status grn_wait_any(grn_ctx *ctx, int timeout_ms, int *tag_out);

/* --------------------------------------------------- device-level API ---
 * For callers that keep inputs resident on the device (CUDA graphs,
 * benchmarks).  grn_pack compiles a batch into the packed program format
 * (host work, CModelSimulator::loadModel for every model) and copies it to
 * device memory owned by the returned handle. */
grn_status grn_pack(grn_ctx *ctx, const grn_model_batch *batch,
                    grn_packed **out);
grn_status grn_packed_free(grn_packed *packed);

typedef struct grn_packed_info {
  int64_t n_models;
  int64_t device_bytes;      /* size of the packed program on the device */
  int64_t cell_update_bound; /* n_models * n_experiments * steps * W * H  */
  int64_t sfu_ops_per_step;  /* MUFU ops of one Euler step of all models  */
  int32_t max_genes;         /* largest products-in-use count             */
  int32_t max_links;         /* largest used-link count                   */
  double mean_genes;
  double mean_links;
  double mean_dif_genes;     /* diffusing products in use per model       */
  /* Algorithmic work of one Euler step of all models, counted on the
   * reference formulation: 3 MUFU ops (lg2, ex2, rcp) per used link and
   * cell, and 6 L + 7 G + 8 G_dif FP32 ops per cell (L used links, G
   * products in use, G_dif of them diffusing). */
  int64_t alg_sfu_ops_per_step;
  int64_t alg_fp32_ops_per_step;
} grn_packed_info;
grn_status grn_packed_get_info(const grn_packed *packed, grn_packed_info *info);

/* Launches the simulation of a packed batch on `cuda_stream` (a
 * cudaStream_t; NULL = the context's stream) and returns without waiting.
 * All pointers are device pointers of n_models entries:
 *   d_max_error (in), d_raw_error (out, unrounded error),
 *   d_steps (out, Euler steps run summed over experiments; may be NULL). */
grn_status grn_run_packed(grn_ctx *ctx, const grn_packed *packed,
                          const double *d_max_error, double *d_raw_error,
                          int32_t *d_steps, void *cuda_stream);

/* Waits for the work queued on `cuda_stream` (NULL = the context's stream)
 * and reports whether a grn_run_packed launch of this context flagged an
 * internal error since the previous call: GRN_ERR_KERNEL (grn_last_error
 * says which: a model record the kernel could not run, a bulk-copy wait that
 * timed out, or a bounds-check failure in the checked library), else GRN_OK.
 * The flag is one word per context, shared by launches on every stream, and
 * this call clears it.  A model the kernel rejected also gets a NaN raw
 * error.  The synchronous entry points (grn_evaluate_batch ...) read their
 * own flag and need no such call.  No reference counterpart: the reference
 * aborts the process on any CUDA error (cerrorhandle.h:21). */
grn_status grn_run_packed_status(grn_ctx *ctx, void *cuda_stream);

/* Compiles one model on the host, as grn_pack does, and writes a text
 * listing of its program (no device work):
 *   "model genes G links L lg_mask M\n"
 *   "gene i label LABEL lim LIM deg DEG dif DIF or N_OR and N_AND\n"  (per gene)
 *   "link i slot S a A b B\n"  (per link of gene i, OR links first)
 * Exponent form: a link's Hill value is 1 / (1 + 2^(a*lg2(x) + b)); slot 255
 * is the constant slot of a Hill coefficient 0.  Mirrors the op list the
 * reference builds in CModelSimulator::loadModel
 * (Src/GPUSimulator/cmodelsimulator.cpp:114-227). */
grn_status grn_describe_model(const grn_product *products, int n_products,
                              const grn_link *links, int n_links,
                              int n_morphogens, char *buf, int buf_len);

/* ------------------------------------------------- headless viewer ---
 * Replaces the reference viewer's simulation thread and its image threads
 * (Src/UI/GUICommon/Simulator/simulatorthread.cpp:30-59,
 * cellimagethread.cpp, concentimagethread.cpp) without a display. */

/* Simulates one model on experiment `experiment` and records its state
 * every `every` Euler steps: frames_out [max_frames][max_planes][dim_y][dim_x]
 * (frame 0 the initial state, frame f the state after f * every steps;
 * plane p the p-th product in use, zero past the model's products).
 * *n_frames = frames written (the simulation may stop early); labels_out
 * (optional, [max_planes]) the plane's product label or -1. */
grn_status grn_trace_model(grn_ctx *ctx, const grn_product *products, int n_products,
                           const grn_link *links, int n_links, int experiment, int every,
                           int max_frames, int max_planes, float *frames_out, int *n_frames,
                           int32_t *labels_out);

/* The viewer's cell image of a state (planes [n_planes][height][width], the
 * products in use in label order): morphogens 0..2 as red, green, blue,
 * 255 * min(1, c).  rgb: [height][width][3]. */
grn_status grn_render_cells(const float *planes, int n_planes, int n_morphogens, int width,
                            int height, uint8_t *rgb);
/* The viewer's concentration image: every product adds its palette colour
 * times c / factor, clamped at 255. */
grn_status grn_render_concentrations(const float *planes, int n_planes, int width, int height,
                                     double factor, uint8_t *rgb);
/* Writes rgb [height][width][3] as a binary PPM (P6) file. */
grn_status grn_write_ppm(const char *path, const uint8_t *rgb, int width, int height);

/* ------------------------------------------------------- model text ---
 * The reference's text form of a model (Model::toString / loadFromString,
 * Src/Model/model.cpp:614-706):
 *   "(" product ("|" product)* "*" [link ("|" link)*] ")"
 *   product = "label init lim deg dif", link = "regulator regulated K n isAnd".
 * grn_model_format writes doubles with `precision` significant digits (6 is
 * the reference's QTextStream default; 17 round-trips exactly) and needs
 * *needed bytes including the terminating 0 (GRN_ERR_CAPACITY if buf_len is
 * smaller).  grn_model_parse returns GRN_ERR_MODEL for malformed text and
 * GRN_ERR_CAPACITY (with the counts set) when the arrays are too small. */
grn_status grn_model_format(const grn_product *products, int n_products, const grn_link *links,
                            int n_links, int precision, char *buf, int buf_len, int *needed);
grn_status grn_model_parse(const char *text, grn_product *products, int max_products,
                           int *n_products, grn_link *links, int max_links, int *n_links);

/* Relative simulation work of one cell-step of each model of a batch (host
 * only; the weights the evaluator uses to order its work queue), for
 * splitting a batch into equal-work shards across GPUs. */
grn_status grn_model_costs(const grn_model_batch *batch, int n_morphogens, double *cost_out);

/* ------------------------------------------------- island evolution ---
 * Deterministic-crowding island search over GRN models, the reference's
 * Search + SearchAlgoDetCrowd (Src/Search/search.cpp:101-311,
 * Src/Search/searchalgodetcrowd.cpp:54-147) with its model operators
 * (crossover, mutation, excess removal: Src/Model/model.cpp), run
 * synchronously: every generation all demes reproduce on host threads, all
 * children are evaluated in one batch, each child replaces its paired parent
 * if its error is not larger, and every migration_period generations random
 * deme pairs shuffle their populations together.  Random initial models
 * have the morphogen products only (nMinProducts = nMorphogens). */
typedef struct grn_evolution_params {
  int32_t n_demes;           /* SearchParams::nDemes                       */
  int32_t deme_size;         /* SearchParams::demesSize (rounded up to even) */
  int32_t migration_period;  /* SearchParams::migrationPeriod (0: never)   */
  int32_t n_max_products;    /* SimParams::nMaxProducts in use (-1: any)   */
  int32_t n_max_links;       /* SimParams::nMaxLinks in use (-1: any)      */
  int32_t n_host_threads;    /* crossover/mutation threads (0: all cores)  */
  uint64_t seed;
} grn_evolution_params;

typedef struct grn_generation_stats {
  int32_t generation;        /* 0: the evaluated random populations        */
  int32_t n_evaluated;       /* models evaluated in this generation        */
  double best_error;         /* lowest error of the populations            */
  int32_t best_complexity;   /* complexity in use of that model            */
  int32_t pareto_size;       /* non-dominated (error, complexity) points   */
  double mean_error;
  double host_ms;            /* reproduction, selection, migration         */
  double eval_ms;            /* batch evaluation, wall clock               */
  int32_t migrated;          /* demes exchanged individuals after it       */
  int32_t n_screened;        /* children ranked by the surrogate (else 0)  */
  double surrogate_ms;       /* encode + predict + train, wall clock       */
  double surrogate_loss;     /* mean training loss of this generation      */
  int32_t n_clones;          /* children accepted without simulation       */
  int32_t n_audited;         /* children simulated for the audit (else 0)  */
  /* Quality of a surrogate screen (NaN without one): Spearman's rank
   * correlation of the predicted and the simulated log(error) minus the
   * parent's log(error), over the simulated children (all children under an
   * audit, grn_evolution_set_surrogate_audit); under an audit also the share
   * of the k truly best children that the screen chose (k = the number it
   * chose), and the share of the children that beat their parents that it
   * chose. */
  double surrogate_rho;
  double surrogate_recall;
  double surrogate_improver_recall;
} grn_generation_stats;

/* A batch fitness evaluator: writes the rounded error (100 above
 * max_error[m]) of every model, as ErrorCalculator does
 * (Src/Search/errorcalculator.h:13-21). */
typedef grn_status (*grn_error_calculator_fn)(void *user, const grn_model_batch *batch,
                                              const double *max_error, double *error_out);

typedef struct grn_evolution grn_evolution;

/* A search evaluated on this library's GPU evaluator (ctx must have its
 * experiments uploaded and outlive the search). */
grn_status grn_evolution_create(const grn_evolution_params *params, int n_morphogens,
                                grn_ctx *ctx, grn_evolution **out);
/* A search evaluated by any batch evaluator. */
grn_status grn_evolution_create_cb(const grn_evolution_params *params, int n_morphogens,
                                   grn_error_calculator_fn fn, void *user,
                                   grn_evolution **out);
/* Runs one generation (the first call creates and evaluates the random
 * populations). */
grn_status grn_evolution_step(grn_evolution *evo, grn_generation_stats *stats);
/* Model, error and complexity of individual `index` of deme `deme`
 * (products/links may be NULL to query the sizes). */
grn_status grn_evolution_individual(const grn_evolution *evo, int deme, int index,
                                    grn_product *products, int max_products,
                                    int *n_products, grn_link *links, int max_links,
                                    int *n_links, double *error, int *complexity);
/* Position of the best individual (lowest error, then lowest complexity). */
/* Replaces individual `index` of deme `deme` (migration between searches,
 * e.g. islands on other GPUs): the model and its known error. */
grn_status grn_evolution_set_individual(grn_evolution *evo, int deme, int index,
                                        const grn_product *products, int n_products,
                                        const grn_link *links, int n_links, double error);
/* Pipelined generations (GPU evaluator only, no surrogate, two or more
 * demes): the demes split into two halves whose evaluations alternate on the
 * GPU, each half's selection and reproduction running on the host while the
 * other half is simulated -- the overlap the reference gets from its
 * asynchronous per-deme loop (Search::calcParalEvolution,
 * Src/Search/search.cpp:132-213, with ErrorCalculator::waitForAnyDeme).
 * Every deme sees the same reproductions, selections and migrations as in
 * the synchronous mode, so the populations are identical; the next
 * generation's children are bred at the end of a step.  Changing a
 * population (grn_evolution_set_individual / _set_generation) first drops
 * the children in flight.  Destroy the search before its evaluator. */
grn_status grn_evolution_set_pipeline(grn_evolution *evo, int enable);

/* Resumes a search whose populations were installed with
 * grn_evolution_set_individual: the next grn_evolution_step reproduces from
 * them (instead of creating random populations) as generation
 * `generation` + 1.  GRN_ERR_MODEL if an individual has no model. */
grn_status grn_evolution_set_generation(grn_evolution *evo, int generation);
/* Checkpoint of a search as an opaque byte string: its generation, every
 * deme's population (models, errors, complexities), pairing order, random
 * state and label counter, and the search's own random state (the
 * reference's Search reload, Src/Search/search.cpp:382-434, restores
 * populations only).  grn_evolution_restore into a search created with the
 * same parameters continues exactly as the checkpointed search would have,
 * given a deterministic evaluator.  An attached surrogate is not part of the
 * checkpoint (grn_surrogate_checkpoint saves it).
 * grn_evolution_checkpoint sets *size to the byte count and writes the bytes
 * when buf is not NULL (GRN_ERR_CAPACITY if cap is smaller).  A pipelined
 * search with children in flight cannot be checkpointed
 * (GRN_ERR_INVALID_ARGUMENT): switch pipelining off first.
 * grn_evolution_restore checks the search's shape and the bytes' integrity
 * (GRN_ERR_INVALID_ARGUMENT, the search unchanged) and drops children in
 * flight. */
grn_status grn_evolution_checkpoint(const grn_evolution *evo, void *buf, size_t cap,
                                    size_t *size);
grn_status grn_evolution_restore(grn_evolution *evo, const void *buf, size_t size);
grn_status grn_evolution_best(const grn_evolution *evo, int *deme, int *index);
grn_status grn_evolution_destroy(grn_evolution *evo);

/* Off by default (the reference simulates every child).  When enabled, a
 * child whose simulated program -- the products in use and the links into
 * them, compared bit for bit -- equals its paired parent's takes the
 * parent's error without being simulated; selection is unchanged, because a
 * deterministic evaluator would return that same error.  Always on while a
 * surrogate is attached. */
grn_status grn_evolution_set_skip_clones(grn_evolution *evo, int enable);

/* ------------------------------------------------------ surrogate MLP ---
 * A learned fitness model that pre-screens offspring (no reference
 * counterpart: the reference simulates every child).  A ReLU MLP
 * 128 -> 256 -> 256 -> 256 -> 1 over a padded encoding of a model's compiled
 * program predicts log(error); its GEMMs run on the tensor cores with BF16
 * operands and FP32 accumulation, trained with Adam on (model, error) pairs
 * the simulator produces. */
#define GRN_SURROGATE_FEATURES 128
#define GRN_SURROGATE_HIDDEN 256
#define GRN_SURROGATE_PARAMS 164865  /* W1 b1 W2 b2 W3 b3 w4 b4, FP32 */

typedef struct grn_surrogate grn_surrogate;

/* Encoding [n_models][128]: products in use 0..7 as (lim, deg, dif, 1), then
 * up to 24 used links in program order (per regulated product: OR links,
 * then AND links) as (regulator index / 8 or -1/8 for a constant term,
 * K clipped to [0, 4], signed Hill coefficient / 5, (regulated index + 1) / 8
 * signed - for AND and + for OR); zero padding.  Host only. */
grn_status grn_encode_models(const grn_model_batch *batch, int n_morphogens, float *features);

/* Surrogate on `device` with a training set ring buffer of `capacity` pairs. */
grn_status grn_surrogate_create(int device, uint64_t seed, int capacity, grn_surrogate **out);
grn_status grn_surrogate_destroy(grn_surrogate *s);
/* Appends (encoding, log error) pairs to the training set (oldest dropped
 * past capacity). */
grn_status grn_surrogate_add_data(grn_surrogate *s, const float *features,
                                  const float *log_error, int n);
int grn_surrogate_data_count(const grn_surrogate *s);
/* Adam epochs over the training set; mean minibatch loss in *mean_loss. */
grn_status grn_surrogate_train(grn_surrogate *s, int epochs, int batch_size, float lr,
                               double *mean_loss);
/* n_batches Adam steps on minibatches drawn uniformly from the training set. */
grn_status grn_surrogate_train_batches(grn_surrogate *s, int n_batches, int batch_size, float lr,
                                       double *mean_loss);
/* Predicted log(error) of n encodings. */
grn_status grn_surrogate_predict(grn_surrogate *s, const float *features, int n,
                                 float *log_error_out);
/* FP32 parameters (GRN_SURROGATE_PARAMS values) out / in (in resets Adam). */
grn_status grn_surrogate_params(grn_surrogate *s, float *params, int n);
grn_status grn_surrogate_set_params(grn_surrogate *s, const float *params, int n);
/* The GEMMs' tensor-core path: 1 (default) tcgen05.mma with the accumulator
 * in tensor memory; 0 warp-level mma.sync (both BF16 x BF16 -> FP32).
 * GRN_ERR_KERNEL from a surrogate call means a tcgen05 GEMM's bounded wait
 * for the tensor core ran out. */
grn_status grn_surrogate_use_tcgen05(grn_surrogate *s, int enable);
/* Checkpoint of a surrogate as an opaque byte string: weights, Adam's
 * moments and step, the training set (the rows it holds), the minibatch
 * sampling state and the tensor-core path.  Restored into a surrogate of the
 * same capacity it trains and predicts exactly as the original would have;
 * with grn_evolution_checkpoint it lets a screened search resume exactly.
 * grn_surrogate_checkpoint sets *size and writes the bytes when buf is not
 * NULL (GRN_ERR_CAPACITY if cap is smaller); grn_surrogate_restore rejects
 * other layouts or capacities with GRN_ERR_INVALID_ARGUMENT. */
grn_status grn_surrogate_checkpoint(grn_surrogate *s, void *buf, size_t cap, size_t *size);
grn_status grn_surrogate_restore(grn_surrogate *s, const void *buf, size_t size);
/* Mean squared loss and its parameter gradients on n pairs, no update. */
grn_status grn_surrogate_gradients(grn_surrogate *s, const float *features,
                                   const float *log_error, int n, float *grads, double *loss);

/* Screens offspring with a surrogate: once it holds min_train_pairs
 * simulated pairs, every generation ranks all children by predicted
 * log(error) minus log(parent error) and simulates only the best
 * simulate_fraction of them (the others lose to their parents); the
 * simulated pairs are added to its training set and it takes
 * batches_per_generation Adam steps.  NULL detaches it. */
grn_status grn_evolution_set_surrogate(grn_evolution *evo, grn_surrogate *s,
                                       double simulate_fraction, int min_train_pairs,
                                       int batches_per_generation, int batch_size, float lr);

/* How a screen ranks a child (grn_evolution_set_surrogate_score):
 *   GRN_SCORE_PARENT_ERROR  predicted log(error) of the child minus the
 *                           parent's simulated log(error);
 *   GRN_SCORE_PAIRED        (default) predicted log(error) of the child
 *                           minus the predicted log(error) of its paired
 *                           parent, so that the network's bias on a model
 *                           family cancels between a child and its parent. */
#define GRN_SCORE_PARENT_ERROR 0
#define GRN_SCORE_PAIRED 1
grn_status grn_evolution_set_surrogate_score(grn_evolution *evo, int score);

/* Audit of the surrogate screen: every screened generation also simulates
 * the children the surrogate rejected, to measure the screen's recall
 * (grn_generation_stats).  The search itself is unchanged -- rejected
 * children still lose to their parents and train nothing -- so an audited
 * run follows the unaudited run's trajectory at the full simulation cost. */
grn_status grn_evolution_set_surrogate_audit(grn_evolution *evo, int enable);

/* ------------------------------------------------ no-allocation entry ---
 * Device memory that grn_evaluate_batch_noalloc uses instead of allocating:
 * one array per GPU, reserved when the library's module is loaded on that
 * GPU and held until the process exits.  Under CUDA's lazy module loading
 * (the default) the module loads at the first grn_evaluate_batch_noalloc
 * call on a device; a caller that divides the device memory itself makes
 * that first call (one with no models is enough) before it does. */
#define GRN_NOALLOC_SCRATCH_BYTES (64u << 20)

/* Batch evaluation that allocates no device memory.  No counterpart in the
 * reference (its evaluator allocates per thread and per model size).
 *
 * For callers that cannot allocate GPU memory: a host application that has
 * already divided the device memory among its components and passes this
 * library only buffers it owns, or a long-running search loop that must not
 * block in, or fail out of, the device allocator in the middle of a run.
 *
 * Runs the same simulation kernel as grn_evaluate_batch on the calling
 * thread's current device, asynchronously on `cuda_stream` (NULL = the
 * legacy default stream).  The caller passes every input and output:
 *   d_initial  [n_experiments][n_input_morphogens][dim_y][dim_x]  FP32, device
 *   d_target   [n_experiments][n_target_morphogens][dim_y][dim_x] FP32, device
 *   batch      models in genome form, host memory (compiled on the host)
 *   d_max_error [n_models] device in; d_raw_error [n_models] device out
 *   (unrounded, round with grn_round_error); d_steps [n_models] device out
 *   or NULL.
 * Everything else -- work counter, error flag, compiled records, state slots
 * of genes that do not fit in shared memory -- lives in a fixed device array
 * of GRN_NOALLOC_SCRATCH_BYTES.  A batch whose records do not fit in it, or
 * a grid one block's state slot does not fit in, is rejected with
 * GRN_ERR_CAPACITY and a message in err_buf; when the slots of one block per
 * SM do not fit, fewer persistent blocks run.  No cudaMalloc, cudaFree or
 * other allocating device routine is called.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * Every call shares the array and it keeps the previous call's contents;
 * the call clears what must start at zero.  Calls whose GPU work overlaps
 * (other streams, or other threads) race on the array: serialise them.
 * A model record the kernel rejects yields a NaN raw error, and the
 * kernel's error flag, which grn_evaluate_batch_noalloc_status reads.  Uses
 * the kernel's exact arithmetic path only.  err_buf (may be NULL) receives a
 * one-line description of a failure. */
grn_status grn_evaluate_batch_noalloc(const grn_sim_params *params, int n_experiments,
                                      const float *d_initial, const float *d_target,
                                      const grn_model_batch *batch,
                                      const double *d_max_error, double *d_raw_error,
                                      int32_t *d_steps, void *cuda_stream,
                                      char *err_buf, int err_buf_len);

/* Waits for `cuda_stream` and reads the error flag that the last
 * grn_evaluate_batch_noalloc call on the current device left in the scratch
 * array: GRN_ERR_KERNEL with a description in err_buf if the kernel flagged
 * an error (a model record it could not run, or a bounds-check failure in
 * the checked library), else GRN_OK.  The next call clears the flag.  Like
 * the evaluation it allocates nothing. */
grn_status grn_evaluate_batch_noalloc_status(void *cuda_stream, char *err_buf,
                                             int err_buf_len);

/* Rounds a raw error the way the reference's evaluate does:
 * 100 if raw > max_error, else ceilS(raw, precision)
 * (Src/Common/mathalgo.h:55-62). */
double grn_round_error(double raw_error, double max_error, int precision);

#ifdef __cplusplus
}
#endif

#endif /* GRN_GPU_H_ */
