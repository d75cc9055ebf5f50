/*
 * nebula_cuda.h — C-ABI of the B200 NEBULA-HL stage-two path.
 *
 * The drop-in entry point is nebula_sparse_cuda(): same inputs and the same
 * NebulaFit as edge-rs's
 *   nebula_sparse<T: EdgeFloat>(counts: &CompressedSparse<f64>,
 *       subject_id: &[usize], design: &[T], n_coef: usize,
 *       offset: Option<&[T]>, params: Option<NebulaParams>)
 *       -> Result<NebulaFit, EdgeErrors>            (src/sc/nebula.rs:434-445)
 * and its device twin nebula_sparse_gpu (src/gpu/stage_two.rs:233-265).
 * Plain pointers and sizes only; the caller owns every buffer.
 *
 * Every function returns NB_OK (0) or one NB_ERR_* code; the codes map 1:1
 * onto the EdgeErrors variants this path can raise (src/errors.rs), and `err`
 * (may be NULL) receives the message.
 */
#ifndef NEBULA_CUDA_H
#define NEBULA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (src/errors.rs variant in brackets). */
enum nb_status {
  NB_OK = 0,
  NB_ERR_EMPTY_COUNTS = 1,            /* EmptyCounts */
  NB_ERR_LENGTH_MISMATCH = 2,         /* LengthMismatch */
  NB_ERR_SHAPE_MISMATCH = 3,          /* ShapeMismatch */
  NB_ERR_INVALID_ARGUMENT = 4,        /* InvalidArgument */
  NB_ERR_MUST_BE_POSITIVE = 5,        /* MustBePositive */
  NB_ERR_MALFORMED_SPARSE = 6,        /* MalformedSparse (errors.rs:162) */
  NB_ERR_NO_GENES_AFTER_FILTERING = 7,/* NoGenesAfterFiltering (errors.rs:169) */
  NB_ERR_INVALID_DISPERSION = 8,      /* InvalidDispersion (errors.rs:183) */
  NB_ERR_SUBJECTS_NOT_CONTIGUOUS = 9, /* SubjectsNotContiguous (errors.rs:196) */
  NB_ERR_MISSING_INTERCEPT = 10,      /* MissingIntercept (errors.rs:203) */
  NB_ERR_TOO_FEW_SUBJECTS = 11,       /* TooFewSubjects (errors.rs:207) */
  NB_ERR_INVALID_BOUNDS = 12,         /* InvalidBounds */
  NB_ERR_COEF_OUT_OF_RANGE = 13,      /* CoefOutOfRange */
  NB_ERR_GPU = 14,                    /* Gpu(String) (errors.rs:223) */
  NB_ERR_UNSUPPORTED = 15             /* what the device path refuses, as the
                                         reference's does: reml
                                         (stage_two.rs:242-246) and more than
                                         8 columns (pml_kernel.rs:1208-1212) */
};

/* CompressedSparse<f64> (src/utils/sparse.rs:58-69): u32 indptr/indices,
 * f64 data, a format flag and the (n_genes, n_cells) shape. */
typedef struct nb_csr {
  uint64_t n_genes;
  uint64_t n_cells;
  uint64_t nnz;
  const uint32_t* indptr;  /* n_genes + 1 */
  const uint32_t* indices; /* nnz, cell of each stored value */
  const double* data;      /* nnz, finite and >= 0; zeros may be stored */
  int32_t format;          /* NB_CSR (gene-major) or NB_CSC */
} nb_csr;

enum nb_format { NB_CSR = 0, NB_CSC = 1 };
enum nb_method { NB_METHOD_LN = 0, NB_METHOD_HL = 1 };

/* NebulaParams (src/sc/nebula.rs:207-258). nb_params_default() fills R's
 * defaults: min (1e-4, 1e-4), max (10, 1000), method LN, cutoff_cell 20,
 * kappa 800, cpc 0.005, mincp 5, min_subjects 0, reml off, eps 1e-6. */
typedef struct nb_params {
  double min_subject, min_cell; /* min.0, min.1 */
  double max_subject, max_cell; /* max.0, max.1 */
  int32_t method;               /* nb_method */
  double cutoff_cell;
  double kappa;
  double cpc;
  uint64_t mincp;
  uint64_t min_subjects;
  int32_t reml;
  double eps;
} nb_params;

/* NebulaFit (src/sc/nebula.rs:301-344). Caller-allocated for n_genes rows;
 * the callee fills the first n_kept rows and writes n_kept and n_coef.
 * covariance is packed upper, column-major: (i <= j) at j(j+1)/2 + i. */
typedef struct nb_fit {
  double* coefficients;           /* n_genes * n_coef */
  double* covariance;             /* n_genes * n_coef(n_coef+1)/2 */
  double* se;                     /* n_genes * n_coef */
  double* subject_overdispersion; /* n_genes */
  double* cell_overdispersion;    /* n_genes */
  int32_t* convergence;           /* n_genes */
  uint8_t* sigma_at_bound;        /* n_genes */
  uint64_t* gene_index;           /* n_genes */
  uint64_t n_kept;
  uint64_t n_coef;
} nb_fit;

/* How stage two is started and run. Zero-initialised = the plain cold-start
 * method the reference runs, on the current device.
 *
 * Warm start (no counterpart in the reference) changes two things, and the
 * plain optimisers finish every search unchanged:
 *  - each inner fit of a gene's search after its first step starts its
 *    Newton loop from the gene's previous iterate (beta, log_w) instead of
 *    (beta_start, 0), and takes at least two Newton steps;
 *  - the search itself starts from
 *      warm_start = 1: the warm-start network's prediction (nb_mlp_predict_cuda)
 *                      from the gene's summary features, weights
 *                      `mlp_weights` (NB_MLP_PARAMS floats) or the built-in
 *                      ones when NULL; genes predicted to need the most
 *                      evaluations are posted first;
 *      warm_start = 2: the caller's starts, warm_points[2 * g], [2 * g + 1]
 *                      for input gene g (e.g. a previous fit);
 *      warm_start = 3: stage one's estimate, as the plain method.
 * Results then differ from the plain method's within the search's
 * tolerance. A deterministic sample of audit_percent % of the searched
 * genes also runs plain (cold); where the warm search's best objective is
 * worse than the cold one's by more than 1e-9 relative, the gene keeps the
 * cold result (refit_cold). */
typedef struct nb_options {
  int32_t device;        /* CUDA ordinal; -1 = current device */
  int32_t warm_start;    /* 0 plain, 1 learned, 2 caller's starts, 3 stage one's */
  int32_t host_threads;  /* worker threads stepping the genes' searches; 0 =
                            twice the hardware threads, at most 32 */
  int32_t audit_percent; /* warm start only: share of genes also run cold */
  const float* mlp_weights; /* warm_start 1: NB_MLP_PARAMS floats; NULL = built-in */
  int32_t cluster;       /* CTAs sharing each inner fit in stages two and three
                            (1, 2, 4 or 8); 0 = chosen per call */
  const double* warm_points; /* warm_start 2: n_genes x 2 starts (sigma, gamma) */
  int32_t* evaluations;  /* optional out: stage-two objective evaluations per
                            kept gene (the kept genes' order of nb_fit) */
  double warm_radius;    /* warm start only: the search's initial BOBYQA trust
                            radius as a fraction of NLopt's (the final radius
                            stays NLopt's); 0 = the library default, 1 = NLopt's */
  int32_t dense_sweep;   /* 1: every sweep visits every cell even where the
                            zero-count tables (src/sc/zeros.rs) apply; 0 = use
                            them for categorical designs, as the reference's
                            CPU path does */
  int32_t cold_inner;    /* warm start only: 1 = every inner fit starts its
                            Newton loop cold, from (beta_start, 0), as the
                            plain method's do; with warm_radius 1 and
                            audit_percent 0 a warm search then differs from
                            the plain one only in its start */
} nb_options;

/* Counters of one call (timings in milliseconds of host wall clock, device
 * times from CUDA events on the launching stream). */
typedef struct nb_stats {
  uint64_t rounds;          /* search steps the host took in stages two and three */
  uint64_t requests;        /* inner fits run on the device */
  uint64_t sweeps;          /* cell passes run on the device */
  uint64_t cell_visits;     /* dense + sparse cell visits on the device */
  uint64_t gpu_launches;    /* kernels launched */
  double ms_total, ms_prepare, ms_stage_one, ms_stage_two, ms_stage_three;
  double ms_device;         /* sum of the fit kernels' device times */
  double ms_step_device;    /* device time from the first stage-two copy to the
                               last stage-three copy, CUDA events */
  uint64_t h2d_bytes, d2h_bytes; /* host<->device bytes the call moved */
  uint64_t audited, refit_cold; /* warm start: genes also run cold, and those
                                    that kept the cold result */
  uint64_t fit_slots;       /* fit-kernel CTAs resident at once */
  uint64_t slot_cycles;     /* SM clock cycles the fit CTAs spent on requests */
  uint64_t cluster;         /* CTAs that shared each fit in stages two and three */
  double ms_upload;         /* host wall time of the device upload */
  double ms_busy_span;      /* device time from the first fit's start to the
                               last fit's end in stages two and three */
  uint64_t zero_groups;     /* zero-count groups looked up instead of swept
                               (0: every sweep visits every cell) */
  double ms_ticket_wait;    /* summed over the fits of stages two and three:
                               device time a cluster waited for its ticket's
                               request to be posted and read */
  uint64_t sparse_visits;   /* the positive entries among cell_visits */
} nb_stats;

void nb_params_default(nb_params* params);

/* Drop-in for nebula_sparse (src/sc/nebula.rs:434-445) with every inner
 * penalised fit on the GPU. Returns NB_OK or an NB_ERR_* code. */
int32_t nebula_sparse_cuda(const nb_csr* counts, const uint64_t* subject_id,
                           const double* design, uint32_t n_coef,
                           const double* offset_or_null,
                           const nb_params* params_or_null, nb_fit* out,
                           char* err, size_t err_len);

/* nebula_sparse_cuda with options and counters (either may be NULL). */
int32_t nebula_sparse_cuda_ex(const nb_csr* counts, const uint64_t* subject_id,
                              const double* design, uint32_t n_coef,
                              const double* offset_or_null,
                              const nb_params* params_or_null,
                              const nb_options* options, nb_fit* out,
                              nb_stats* stats, char* err, size_t err_len);

/* nebula_sparse_cuda in two parts, for callers that fit the same inputs
 * more than once or time the device-resident stages alone:
 * nb_session_create validates and preprocesses the inputs, runs stage one and
 * uploads the design, offsets and kept genes' counts to the device;
 * nb_session_fit runs stages two and three on that resident copy and fills
 * `out` exactly as nebula_sparse_cuda does. */
typedef struct nb_session nb_session;
int32_t nb_session_create(const nb_csr* counts, const uint64_t* subject_id,
                          const double* design, uint32_t n_coef,
                          const double* offset_or_null,
                          const nb_params* params_or_null,
                          const nb_options* options, nb_session** out,
                          char* err, size_t err_len);
int32_t nb_session_fit(nb_session* session, nb_fit* out, nb_stats* stats,
                       char* err, size_t err_len);
void nb_session_free(nb_session* session);

/* opt_pml (src/sc/pml.rs:468-508) for a batch of variance points of one
 * gene on the device (the batched twin of the reference's device entry,
 * src/gpu/nebula_gpu.rs:466-594). The design is used as given (already
 * centred), offsets are logs, subject_start has k + 1 boundaries, counts and
 * cells are the positive entries in increasing cell order. Per request:
 * beta_init (n_beta), subject (nebula's sigma[0]), cell (NB size), ord.
 * scalars_out (4 per request): log_likelihood, log_likelihood_prev, log_det,
 * second_order; ints_out (4 per request): status (0 ok, 1 rejected
 * arguments), iterations, backtracks, sweeps. */
int32_t nb_opt_pml_cuda(const double* design, const double* offset,
                        uint64_t n_cells, uint32_t n_beta, const double* counts,
                        const uint32_t* cells, uint64_t n_pos,
                        const uint64_t* subject_start, uint32_t k,
                        const double* subject_total, uint32_t n_requests,
                        const double* beta_init, const double* subject,
                        const double* cell, const int32_t* ord, int32_t reml,
                        double eps, double* beta_out, double* information_out,
                        double* scalars_out, int32_t* ints_out, char* err,
                        size_t err_len);

/* nb_opt_pml_cuda for callers that cannot allocate device memory: an engine
 * whose HBM belongs to its own pool or arena, a real-time loop that cannot
 * take cudaMalloc's implicit synchronisation, a plugin that must not
 * allocate after start-up. It has no counterpart in the reference. Every
 * array argument is a DEVICE pointer (same meaning and layout as
 * nb_opt_pml_cuda; ord may be NULL); the fit's working memory lives in one
 * fixed 2 MiB device array inside this library, so the call allocates
 * nothing. Limits: at most 2048 requests and 8192 subjects per call, else
 * NB_ERR_INVALID_ARGUMENT before any launch. Runs on the calling thread's
 * current device and `stream` (NULL: the default stream), and returns once
 * the outputs are written: it is blocking and cannot be made during stream
 * capture. The first call on a device looks up the array's address and keeps
 * it for the process; calls after cudaDeviceReset on that device are not
 * supported. All calls on a device share
 * the array: calls whose GPU work overlaps race, so issue them one at a
 * time. */
int32_t nb_opt_pml_cuda_noalloc(const double* design, const double* offset,
                                uint64_t n_cells, uint32_t n_beta,
                                const double* counts, const uint32_t* cells,
                                uint64_t n_pos, const uint64_t* subject_start,
                                uint32_t k, const double* subject_total,
                                uint32_t n_requests, const double* beta_init,
                                const double* subject, const double* cell,
                                const int32_t* ord, int32_t reml, double eps,
                                double* beta_out, double* information_out,
                                double* scalars_out, int32_t* ints_out,
                                void* stream, char* err, size_t err_len);

/* The warm-start network (no counterpart in the reference): 12 summary
 * features of a gene -> 64 -> 64 -> 3 (GELU), predicting log(final sigma /
 * stage-one sigma), log(final gamma / stage-one gamma) and log(stage-two
 * evaluations). Parameters: NB_MLP_PARAMS floats, laid out W1 [64][12],
 * b1 [64], W2 [64][64], b2 [64], W3 [3][64], b3 [3], input mean [12], input
 * scale [12] (inputs enter as (x - mean) * scale; the normalisation is not
 * trained). Loss: mean over samples of sum_o w_o (y_o - t_o)^2 / 2 with
 * w = (1, 1, 0.25). The kernels are the project's own; gradients are summed
 * in a fixed order, so results repeat bit for bit. */
#define NB_MLP_FEATURES 12
#define NB_MLP_OUTPUTS 3
#define NB_MLP_PARAMS 5211
/* Xavier-uniform weights from `seed`, zero biases, identity normalisation. */
void nb_mlp_init(uint64_t seed, float* params);
/* The built-in network warm_start = 1 uses when mlp_weights is NULL. */
void nb_mlp_builtin(float* params);
/* out: n x NB_MLP_OUTPUTS predictions for n x NB_MLP_FEATURES features.
 * Inference takes the weight matrices as BF16 values (rounded to nearest
 * even from `params`), biases and normalisation in FP32, FP32 accumulation;
 * training (below) updates FP32 parameters. */
int32_t nb_mlp_predict_cuda(const float* params, const float* features,
                            uint64_t n, float* out, char* err, size_t err_len);
/* The loss over n samples (targets n x NB_MLP_OUTPUTS) and its gradient
 * (NB_MLP_PARAMS floats; zero for the normalisation entries). */
int32_t nb_mlp_gradient_cuda(const float* params, const float* features,
                             const float* targets, uint64_t n, float* grad_out,
                             double* loss_out, char* err, size_t err_len);
/* Adam (lr, betas 0.9/0.999) on mini-batches of `batch` rows of a fresh
 * seeded permutation each epoch, from and into `params`; epoch_loss (may
 * be NULL) receives each epoch's mean batch loss. Each step's four kernels
 * run as one captured CUDA graph. */
int32_t nb_mlp_train_cuda(const float* features, const float* targets,
                          uint64_t n, int32_t epochs, int32_t batch, float lr,
                          uint64_t seed, float* params, double* epoch_loss,
                          char* err, size_t err_len);
/* A session's kept genes: their NB_MLP_FEATURES features (n_kept rows) and
 * stage one's (sigma, gamma) (n_kept x 2); either may be NULL. */
int32_t nb_session_features(nb_session* session, float* features,
                            double* stage_one, uint64_t* n_kept, char* err,
                            size_t err_len);

/* glm_sc_test (src/sc/test.rs:96-200): Wald test of the contrast c per gene,
 * z = c'beta / sqrt(c'Vc), p = chisq_sf(z^2, 1), BH FDR. log_p_value keeps
 * the tail in log space where p underflows. Any output may be NULL. */
int32_t nb_glm_sc_test(const double* coefficients, const double* covariance,
                       uint64_t n_genes, uint64_t n_coef, const double* contrast,
                       double* log_fc, double* se, double* z, double* p_value,
                       double* log_p_value, double* fdr, char* err,
                       size_t err_len);

/* nb_glm_sc_test on the device (src/sc/test.rs:96-200), for fits kept in
 * HBM: coefficients (n_genes x n_coef, n_coef <= 8), the packed covariance
 * and every output are DEVICE pointers (any output may be NULL); contrast is
 * a host array of n_coef. Same arithmetic in the same order as
 * nb_glm_sc_test; erfc and log are CUDA's, so p-values agree with the host's
 * to a few ulps. The BH FDR sorts on the device (its scratch comes from the
 * device's stream-ordered memory pool). Runs on the current device and
 * `stream` (NULL: the default stream) and returns once the outputs are
 * written. */
int32_t nb_glm_sc_test_cuda(const double* coefficients,
                            const double* covariance, uint64_t n_genes,
                            uint64_t n_coef, const double* contrast,
                            double* log_fc, double* se, double* z,
                            double* p_value, double* log_p_value, double* fdr,
                            void* stream, char* err, size_t err_len);

/* The inner fit's Hessian contraction S_r = sum_c w_rc x_c x_c' for a batch
 * of requests (the dense product of their cell weights with the Khatri-Rao
 * square of the design; the reference's fused curvature assembly,
 * src/gpu/pml_kernel.rs:350-515), in one of four arithmetics: 0 FP64 and
 * 1 FP32 on CUDA cores, 2 TF32 and 3 split BF16 (hi.hi + hi.lo + lo.hi,
 * FP32 accumulation) on the tensor cores (tcgen05.mma). design: device
 * n_cells x n_coef FP64 (n_coef <= 8); weights: device n_requests x n_cells
 * FP64 (n_requests <= 128); out: device n_requests x n_coef (n_coef + 1) / 2,
 * entry b (b + 1) / 2 + a = sum_c w_rc x_ca x_cb for a <= b. ms_out (host,
 * 2 doubles, may be NULL): device ms of the contraction kernel, and with the
 * operand conversions. Scratch comes from the device's stream-ordered pool;
 * returns once `out` is written. A precision study: the fits themselves
 * keep this sum in FP64. */
int32_t nb_contract_krx_cuda(int32_t variant, const double* design,
                             uint64_t n_cells, uint32_t n_coef,
                             const double* weights, uint32_t n_requests,
                             double* out, double* ms_out, void* stream,
                             char* err, size_t err_len);

/* Reverse-communication BOBYQA as NLopt 2.7.1 runs it
 * (src/numeric/bobyqa.rs:141-560 BobyqaStepper::{new, ask, tell, result}). */
typedef struct nb_bobyqa nb_bobyqa;
nb_bobyqa* nb_bobyqa_new(const double* x0, const double* lower,
                         const double* upper, uint32_t n, double xtol_rel,
                         uint32_t maxeval);
/* As nb_bobyqa_new with the initial trust radius at radius_scale (0, 1] of
 * NLopt's and the final radius NLopt's (xtol_rel times the unscaled initial
 * radius): the warm search of nb_options.warm_radius. No counterpart in the
 * reference; radius_scale 1 is nb_bobyqa_new. */
nb_bobyqa* nb_bobyqa_new_scaled(const double* x0, const double* lower,
                                const double* upper, uint32_t n,
                                double xtol_rel, uint32_t maxeval,
                                double radius_scale);
int32_t nb_bobyqa_ask(const nb_bobyqa* h, double* x); /* 1: x pending */
void nb_bobyqa_tell(nb_bobyqa* h, double value);
/* returns the NLopt status: 4 xtol, 5 maxeval, 1 success, -4 roundoff */
int32_t nb_bobyqa_result(const nb_bobyqa* h, double* x, double* f,
                         uint32_t* evaluations);
void nb_bobyqa_free(nb_bobyqa* h);

/* The stage-two search the device driver steps for every gene, in reverse
 * communication (src/sc/nebula.rs:1568-1951 StageTwoSearch::{new, ask,
 * tell, order, result}): n = 2 runs BOBYQA over (sigma, gamma), n = 1 the
 * clamped start, a bounded Nelder-Mead and the polish stencils. A
 * non-finite value told at Laplace order ord > 1 restarts the pass at order
 * one; at order one it abandons the search. radius_scale (0, 1] narrows the
 * first BOBYQA pass's initial trust region (1: NLopt's). NULL on invalid
 * arguments. */
typedef struct nb_search nb_search;
nb_search* nb_search_new(const double* start, const double* lower,
                         const double* upper, uint32_t n, uint32_t ord,
                         double radius_scale);
/* How many points are pending (0 once the search is done); copies up to
 * max_points of them, n doubles each, into points (may be NULL). */
uint32_t nb_search_ask(const nb_search* h, double* points, uint32_t max_points);
/* One value per pending point; NB_ERR_LENGTH_MISMATCH otherwise. */
int32_t nb_search_tell(nb_search* h, const double* values, uint32_t n_values);
uint32_t nb_search_order(const nb_search* h); /* the Laplace order under test */
/* 1: done with a minimiser in x (n doubles) and *failed = 1 where BOBYQA
 * ended roundoff-limited (the gene's convergence -50); 0: done, abandoned
 * (no finite pass: the gene keeps stage one's estimates, convergence -50);
 * -1: still running. *evaluations: values told so far. */
int32_t nb_search_result(const nb_search* h, double* x, int32_t* failed,
                         uint32_t* evaluations);
void nb_search_free(nb_search* h);

/* Self-check of the request ring that feeds the persistent kernels (no
 * counterpart in the reference, whose rounds are host-driven launches,
 * src/gpu/stage_two.rs:362-580 search_all). On the current device, `ctas` one-warp CTAs
 * serve n_requests tickets through a ring of `capacity` slots (a power of
 * two; fewer slots than requests exercises slot reuse) with the same device
 * protocol as the fit and stage-one kernels, answering each request with a
 * fixed function of it; *mismatches counts results that differ from it.
 * idle_ms: how long a CTA waits for its ticket's request before it sets the
 * ring's status word and returns (0 = the library's 5 s). With n_requests 0
 * nothing is posted and no stop is requested, so every CTA's wait runs out:
 * the call then returns NB_ERR_GPU ("... waited more than idle_ms for
 * work") without a device fault, and the device stays usable. */
int32_t nb_ring_check_cuda(uint64_t n_requests, uint32_t capacity,
                           uint32_t ctas, uint32_t idle_ms,
                           uint64_t* mismatches, char* err, size_t err_len);

/* Measured FP64 FMA throughput of the current device in TFLOP/s (best of
 * `repeats` launches), the peak the fit kernel's roofline is taken against. */
double nb_measure_fp64_tflops(int repeats);

#ifdef __cplusplus
}
#endif

#endif /* NEBULA_CUDA_H */
