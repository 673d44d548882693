/* h3g.h — C ABI of the B200 codon-likelihood core (libh3g.so).
 *
 * The reference (veg/hyphy-3) exposes its likelihood core only as header-only
 * C++ static functions of hyphy::core::LikelihoodEngine plus a nanobind module;
 * it has no C ABI.  These entry points are what those call sites bind to:
 *
 *   h3g_branch_length_gradients   <- LikelihoodEngine::compute_branch_length_gradients
 *                                    (include/hyphy/core/likelihood.hpp:1102-1211) and
 *                                    _hyphy3.compute_branch_length_gradients
 *                                    (src/python/bindings.cpp:725-732)
 *   h3g_eval                      <- the general engine behind
 *                                    LikelihoodEngine::compute_joint_frechet_gradients
 *                                    (likelihood.hpp:1228-1594) and BUSTED's
 *                                    compute_busted_branch_gradients / evaluate_log_l
 *                                    (include/hyphy/analyses/busted.hpp:509-660, :1138-1429)
 *   h3g_eval_from_P               <- LikelihoodEngine::compute_tree_log_likelihood_from_P
 *                                    (likelihood.hpp:766-806)
 *
 * Conventions.  Plain pointers and sizes; every host array is read or written
 * during the call only.  Matrices are row-major doubles.  Node ids are the
 * reference's Newick creation order (tree.hpp:273-585); per-node vectors have
 * n_nodes entries and the root entry of a gradient is 0.  Every function
 * returns an h3g_status; h3g_last_error() describes the last failure on a
 * context.  No C++ exception crosses this boundary.  A context is bound to one
 * device and one CUDA stream and is not thread-safe: use one per thread.
 */
#ifndef H3G_H
#define H3G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    H3G_OK = 0,
    H3G_ERR_ARG = 1,      /* invalid argument (sizes, topology, missing arrays) */
    H3G_ERR_OOM = 2,      /* device allocation failed */
    H3G_ERR_CUDA = 3,     /* CUDA runtime error or no usable device / kernel image */
    H3G_ERR_NUMERIC = 4,  /* non-finite input parameters or results */
    H3G_ERR_TIMEOUT = 5,  /* a bounded device wait expired */
    H3G_ERR_STATE = 6     /* call order violated (e.g. eval before model_set) */
} h3g_status;

typedef enum {
    H3G_PREC_FP64 = 0,    /* every contraction in FP64 (parity path, 1e-10 of the CPU engine) */
    H3G_PREC_MIXED = 1    /* split-precision tensor-core contractions, FP32 partials, FP64 model/root */
} h3g_precision;

typedef enum {
    H3G_TIME_RAW = 0,        /* P = exp(Q * r_m * t)             (likelihood.hpp:1118-1127) */
    H3G_TIME_NORMALIZED = 1  /* P = exp(Q * r_m * t * 3 / mu)    (likelihood.hpp:1246-1271) */
} h3g_time_mode;

/* what h3g_eval computes */
enum {
    H3G_WANT_LNL = 1u,        /* total log-likelihood (always computed) */
    H3G_WANT_SITE_LNL = 2u,   /* per-pattern log-likelihood */
    H3G_WANT_GRAD_T = 4u,     /* d lnL / d t for every branch */
    H3G_WANT_GRAD_GLOBAL = 8u /* directional, mixture-weight and rate-weight gradients */
};

typedef struct h3g_ctx h3g_ctx;
typedef struct h3g_problem h3g_problem;
typedef struct h3g_batch h3g_batch;

/* Reversible substitution models as eigensystems, P(tau) = U diag(exp(lam*tau)) V,
 * clamped at 0 (rate_matrix.hpp:251-257).  Models [0, K) are mixed at the P
 * level with weights class_w on test branches; models [K, K + has_bg) are mixed
 * with weights bg_w on branches whose is_test entry is 0 (has_bg = 1 with
 * bg_w = NULL: one background model, weight 1). */
typedef struct {
    int S;                    /* states (<= 64; 61 for the universal code) */
    const double* pi;         /* S equilibrium frequencies (root prior) */
    int n_models;             /* K + has_bg */
    const double* Q;          /* n_models * S * S generators */
    const double* lam;        /* n_models * S eigenvalues (clamped <= 0) */
    const double* U;          /* n_models * S * S, U_pi */
    const double* V;          /* n_models * S * S, V_pi = U_pi^-1 */
                              /* lam, U and V all NULL: the device diagonalises every Q_k itself
                                 (symmetrised with pi as rate_matrix.hpp:229-249 does, parallel
                                 cyclic Jacobi in FP64); h3g_model_get_eigensystem reads the result */
    const double* mu;         /* n_models mean rates (used by H3G_TIME_NORMALIZED); NULL with a
                                 device eigensolve: -sum_i pi_i Q_k,ii */
    int K;                    /* test-branch classes */
    const double* class_w;    /* K mixing weights */
    int has_bg;               /* background classes (0: every branch is a test branch) */
    const uint8_t* is_test;   /* n_nodes flags, NULL = every branch is a test branch */
    int M;                    /* synonymous-rate classes (separate pruning passes) */
    const double* rates;      /* M rate multipliers r_m */
    const double* rate_w;     /* M class weights rho_m */
    int time_mode;            /* h3g_time_mode */
    int n_dirs;               /* global gradient directions x */
    const double* dQ;         /* n_dirs * n_models * S * S : dQ_model / dx */
    int precision;            /* h3g_precision */
    int zero_l_sentinel;      /* 1: a pattern with L <= 0 adds weight * -1e20 to lnL (evaluate_log_l);
                                 0: it adds 0 (the gradient entry points) */
    const double* bg_w;       /* has_bg background mixing weights; NULL allowed only when has_bg <= 1 */
    const int32_t* branch_classes;
                              /* NULL, or n_nodes + 1 offsets into the K classes: branch b mixes classes
                                 [branch_classes[b], branch_classes[b + 1]) with weights class_w (a
                                 distribution of its own per branch, as aBSREL's branch-site models,
                                 absrel.hpp:262-310); needs has_bg = 0 and is_test = NULL; the root's
                                 range is ignored.  grad_class_w then holds every class's weight
                                 partial. */
    const double* dQ_model;   /* NULL, or n_models * S * S: one more direction per model k, dQ_model[k]
                                 acting on model k alone (e.g. d/d omega of each branch class); their
                                 gradients follow the n_dirs dense ones in grad_dir (n_dirs + n_models
                                 entries) */
} h3g_model_desc;

typedef struct {
    double lnl;
    double* site_lnl;         /* n_patterns, or NULL */
    double* grad_t;           /* n_nodes, or NULL */
    double* grad_dir;         /* n_dirs, or NULL */
    double* grad_class_w;     /* K partials d lnL / d class_w[k], or NULL */
    double* grad_rate_w;      /* M partials d lnL / d rate_w[m], or NULL */
    double* grad_bg_w;        /* has_bg partials d lnL / d bg_w[j], or NULL */
} h3g_result;

/* Context: one device, one stream (NULL = a private non-blocking stream).
 * h3g_ctx_destroy fails with H3G_ERR_STATE while problems created on it live. */
h3g_status h3g_ctx_create(int device, void* cuda_stream, h3g_ctx** out);
h3g_status h3g_ctx_destroy(h3g_ctx* ctx);
const char* h3g_last_error(const h3g_ctx* ctx);
const char* h3g_version(void);

/* Upload one tree and its compressed site patterns.
 *   parent[n_nodes]       parent id, -1 for the root (exactly one)
 *   leaf_taxon[n_nodes]   alignment row of each leaf, -1 for a leaf without a
 *                         sequence (all-ones partial); ignored for internal nodes
 *   is_leaf[n_nodes]      1 for leaves
 *   states[P * T]         sense index per (pattern, taxon), -1 if unresolved
 *   masks[P * T]          compatible-state bitmask per (pattern, taxon)
 *   weights[P]            pattern multiplicities
 * Children are visited in increasing node id, the reference's child order. */
h3g_status h3g_problem_create(h3g_ctx* ctx, int n_nodes, const int32_t* parent, const uint8_t* is_leaf,
                              const int32_t* leaf_taxon, int n_taxa, int n_patterns, const int8_t* states,
                              const uint64_t* masks, const double* weights, h3g_problem** out);
h3g_status h3g_problem_destroy(h3g_problem* prob);

/* Install a model (copies all arrays; allocates the device workspace). */
h3g_status h3g_model_set(h3g_problem* prob, const h3g_model_desc* desc);

/* One likelihood (+ gradient) evaluation at branch lengths bl[n_nodes]
 * (root entry ignored).  Blocks until results are on the host. */
h3g_status h3g_eval(h3g_problem* prob, const double* bl, unsigned want, h3g_result* out);

/* Log-likelihood from caller-supplied transition matrices P[n_nodes * S * S]
 * (root entry ignored) and root frequencies pi[S]; zero-likelihood patterns
 * contribute weight * -1e20.  site_lnl may be NULL. */
h3g_status h3g_eval_from_P(h3g_problem* prob, int S, const double* P, const double* pi, double* lnl, double* site_lnl);

/* compute_branch_length_gradients in one call: MG94 eigensystem (S, pi, Q, lam,
 * U, V) with raw time, FP64 or mixed precision; grad[n_nodes]. */
h3g_status h3g_branch_length_gradients(h3g_problem* prob, int S, const double* pi, const double* Q, const double* lam,
                                       const double* U, const double* V, const double* bl, int precision,
                                       double* lnl, double* grad);

/* Device time of the last evaluation in milliseconds (CUDA events on the
 * context stream around the launch sequence, host copies included for
 * h3g_eval), and the number of kernel launches it made. */
h3g_status h3g_last_eval_stats(const h3g_problem* prob, double* device_ms, int* n_launches);

/* Bytes the last evaluation copied host->device and device->host. */
h3g_status h3g_last_eval_transfer(const h3g_problem* prob, size_t* h2d_bytes, size_t* d2h_bytes);

/* Device-resident evaluation, for callers that keep inputs and results on the
 * GPU: h3g_stage_branch_lengths copies bl[n_nodes] to the device (blocking);
 * h3g_eval_resident enqueues one evaluation on the context stream and returns
 * without waiting; h3g_read_result waits for it and copies the results out. */
h3g_status h3g_stage_branch_lengths(h3g_problem* prob, const double* bl);
h3g_status h3g_eval_resident(h3g_problem* prob, unsigned want);
h3g_status h3g_read_result(h3g_problem* prob, unsigned want, h3g_result* out);

/* ---------------------------------------------------------------- batches
 * Many independent problems -- genes of uneven taxon count and length, each with
 * its own tree and model -- evaluated together.  The reference evaluates such
 * genes one call at a time (LikelihoodEngine::compute_* per gene,
 * likelihood.hpp:1102-1211, :1228-1594, OpenMP over each gene's 64-pattern
 * tiles, :785-803); here one batch evaluation is one CUDA-graph launch that runs
 * every gene: the genes are spread over n_slots streams by longest-processing-
 * time assignment on nodes x patterns x rate classes, each slot owning one
 * workspace sized for its largest gene (device memory grows with n_slots, not
 * with the number of genes), the slots running concurrently.
 *   h3g_batch_create   takes problems created with h3g_problem_create; their own
 *                      workspaces are released.  Install each one's model with
 *                      h3g_model_set (before or after), all with one precision.
 *                      While in a batch a problem is evaluated only through it
 *                      (its single-problem entry points return H3G_ERR_STATE).
 *   h3g_batch_eval     bl[i] = branch lengths of problem i (n_nodes each);
 *                      results[i] as for h3g_eval.  Blocks until all results
 *                      are on the host.
 *   h3g_batch_destroy  the problems stay valid but need h3g_model_set again.
 * Replaces: a loop of compute_joint_frechet_gradients / compute_branch_length_
 * gradients calls over genes. */
h3g_status h3g_batch_create(h3g_ctx* ctx, int n_problems, h3g_problem* const* problems, int n_slots, h3g_batch** out);
h3g_status h3g_batch_destroy(h3g_batch* batch);
h3g_status h3g_batch_eval(h3g_batch* batch, const double* const* bl, unsigned want, h3g_result* results);
/* Device time of the last batch evaluation in ms (CUDA events around the graph
 * launch, host copies included) and the number of kernel launches in it. */
h3g_status h3g_batch_last_stats(const h3g_batch* batch, double* device_ms, int* n_launches);

/* The eigensystem of model k as installed (given, or solved on the device):
 * lam[S], U[S*S], V[S*S] row-major. */
h3g_status h3g_model_get_eigensystem(h3g_problem* prob, int k, double* lam, double* U, double* V);

/* ---------------------------------------------------------------- tuning
 * Launch shapes that do not change results beyond rounding: the pattern chunk
 * of the A accumulation (more chunks = more CTAs, more partial sums to reduce),
 * the resident CTAs per SM of the mixed path's persistent passes, and the branch
 * groups of the Frechet kernel.  0 in a field = the built-in heuristic.  The
 * reference's counterpart is its fixed tile schedule (busted.hpp:385-401
 * compute_tile_schedule, likelihood.hpp:91-104 optimal_omp_threads).
 * h3g_autotune times the candidates of each field in turn (coordinate descent;
 * reps evaluations each after one warm-up, CUDA events on the context stream),
 * installs the fastest on the problem and records it for the problem's shape
 * (nodes, internal nodes, padded patterns, M, K, models, directions, precision,
 * device): later problems of that shape start from it.  Results are
 * deterministic for a given tuning; tunings differ only in summation order. */
typedef struct {
    int a_chunk;          /* patterns per A-accumulation chunk: a multiple of 128, >= 256 */
    int ctas_per_sm;      /* mixed persistent passes: 1 or 2 resident CTAs per SM */
    int frechet_groups;   /* branch groups of the Frechet kernel: >= 1 */
} h3g_tuning;
h3g_status h3g_problem_set_tuning(h3g_problem* prob, const h3g_tuning* tuning);
h3g_status h3g_problem_get_tuning(const h3g_problem* prob, h3g_tuning* tuning);
/* Times evaluations at branch lengths bl[n_nodes]; best and best_ms may be NULL. */
h3g_status h3g_autotune(h3g_problem* prob, const double* bl, unsigned want, int reps, h3g_tuning* best, double* best_ms);

/* The CUDA stream a context enqueues its work on (the one given to
 * h3g_ctx_create, or its private stream). */
h3g_status h3g_ctx_stream(const h3g_ctx* ctx, void** stream);

/* For pattern-sharded evaluation across GPUs: after h3g_eval_resident, enqueue on
 * the context stream the assembly of that evaluation's results into the caller's
 * DEVICE vector d_vec of 1 + n_nodes + n_dirs + K + M + 1 doubles:
 * [lnl, grad_t, grad_dir, grad_class_w, grad_rate_w, failed] (failed = 1 when a
 * bounded device wait expired).  Every entry is a sum over site patterns, so the
 * vectors of the ranks holding disjoint pattern ranges add up (one all-reduce) to
 * the whole alignment's result, as the reference's per-tile pattern sums do
 * (likelihood.hpp:794-806).  Returns without waiting. */
h3g_status h3g_pack_result_device(h3g_problem* prob, unsigned want, double* d_vec);

/* Limit of the waits the mixed-precision persistent passes make on one another's
 * items: polls before a wait gives up (0 = the default, about 2^22 polls of 64 ns).
 * An expired wait lets the kernel finish, and the evaluation returns
 * H3G_ERR_TIMEOUT (its results are invalid); the next evaluation on the problem
 * starts clean.  unmatched != 0 makes every such wait look for a flag value that
 * no item publishes, so that each one expires: it exists to test this path
 * without a fault or a hang.  No counterpart in the reference (a CPU engine has
 * no device waits). */
h3g_status h3g_problem_set_wait_limit(h3g_problem* prob, uint32_t polls, int unmatched);

/* ------------------------------------------------------ subtree checkpointing
 * The reference keeps every node's inside, outside and message partials for all
 * patterns in host memory (likelihood.hpp:314-340).  Here, when the evaluation
 * workspace of a problem exceeds its memory budget, the tree is cut into blocks
 * (subtrees rooted at checkpoint nodes, each at most about `target` nodes): the
 * inside pass keeps only the checkpoint nodes' partials, and the outside pass
 * recomputes each block's inside partials from its checkpointed children before
 * walking it.  Results are bit-identical to the unbudgeted evaluation (same
 * kernels, same summation order).  Budget 0 = none, but a workspace larger than
 * the device's free memory checkpoints by itself.  target > 0 forces that block
 * size (0 = the largest that fits the budget).  FP64 and mixed precision; not for
 * batch members (their workspaces are the batch's slots). */
typedef struct {
    int32_t active;          /* 1 when the installed workspace is checkpointed */
    int32_t n_blocks;        /* blocks (= checkpoint nodes, the root included) */
    int32_t target;          /* block size target of the plan */
    int32_t n_persistent;    /* partial slots kept through the evaluation */
    int32_t scratch_internal;/* internal-node slots shared by the blocks */
    int32_t scratch_nodes;   /* gradient-operand slots shared by the blocks */
    uint64_t workspace_bytes;/* device bytes of the installed workspace */
    uint64_t full_bytes;     /* device bytes the workspace takes without checkpoints */
} h3g_checkpoint_info;
h3g_status h3g_problem_set_memory_budget(h3g_problem* prob, uint64_t bytes, int target);
h3g_status h3g_problem_checkpoint_info(const h3g_problem* prob, h3g_checkpoint_info* info);
/* The plan alone, on the host (no device needed): for a tree of n_nodes
 * (parent[i] = -1 at the root) and a block size target, fills the per-node arrays
 * that are not NULL: is_checkpoint, block (index of the block that computes the
 * node, blocks in post-order, the root's last), slot_internal (partial slot of an
 * internal node, -1 for leaves) and slot_vf (gradient-operand slot), and
 * counts[4] = {blocks, persistent slots, scratch internal slots, scratch node slots}. */
h3g_status h3g_checkpoint_plan(int n_nodes, const int32_t* parent, const uint8_t* is_leaf, int target,
                               int32_t* is_checkpoint, int32_t* block, int32_t* slot_internal, int32_t* slot_vf,
                               int32_t* counts);

/* Per-stage device time of one evaluation (mean over reps runs, events between
 * stages, no graph): stage_ms[H3G_N_STAGES], stage_launches[H3G_N_STAGES] (may
 * be NULL).  Stage order: H3G_STAGE_NAMES. */
#define H3G_N_STAGES 10
#define H3G_STAGE_NAMES "build_P,prep_mixed,inside,root,outside,accum_A,frechet,hsum,small,dir"
h3g_status h3g_profile_stages(h3g_problem* prob, unsigned want, int reps, double* stage_ms, int* stage_launches);

/* Log-likelihood from caller-supplied transition matrices without allocating
 * any device memory.  No counterpart in the reference: it exists for callers
 * that cannot call cudaMalloc while they run, such as code embedded in a
 * process whose framework already owns the whole device memory pool, or code
 * that must not add allocation-driven synchronisation to a latency path.
 * Same inputs, outputs and results as h3g_eval_from_P, but no context or
 * problem handle: the topology, patterns, matrices P[n_nodes * S * S] and pi[S]
 * are host arrays, lnl and site_lnl (NULL allowed) host outputs, the work runs
 * on cuda_stream (NULL = the legacy default stream) of `device`.
 * All intermediates live in one 32 MiB __device__ array that every GPU loading
 * the library holds until exit; problems needing more (or n_nodes > 1024) are
 * rejected with H3G_ERR_ARG before any work is launched.  The first call on a
 * device resolves the array's address and should come before any stream
 * capture.  Calls share the array: calls that overlap on the GPU race. */
h3g_status h3g_eval_from_P_noalloc(int device, void* cuda_stream, int n_nodes, const int32_t* parent,
                                   const uint8_t* is_leaf, const int32_t* leaf_taxon, int n_taxa, int n_patterns,
                                   const int8_t* states, const uint64_t* masks, const double* weights, int S,
                                   const double* P, const double* pi, double* lnl, double* site_lnl);

/* ---------------------------------------------------------------- FEL
 * Fixed-effects likelihood per-site fits on the device, replacing
 * FELAnalyzer::analyze_pattern / run (include/hyphy/analyses/fel.hpp:326-446,
 * :778-833) for the case where every branch is tested.  Per pattern: the
 * 12-point (alpha, beta) grid, the bounded 2-D Nelder-Mead of the alternative
 * model, the null grid and Brent search on alpha = beta, then LRT and
 * p = erfc(sqrt(LRT / 2)).  Each likelihood evaluation uses the MG94 model
 * Q = Qs + (beta / alpha) Qn with time scaled by alpha, exactly as the
 * reference; all patterns advance together, one batched device evaluation
 * (eigensystems + single-pattern pruning) per optimiser step. */
typedef struct {
    int S;                    /* states (<= 64; 61 for the universal code) */
    const double* pi;         /* S codon frequencies (root prior) */
    const double* Qs;         /* S * S synonymous rates of the base model at alpha = 1, beta = 0 (diagonal ignored) */
    const double* Qn;         /* S * S non-synonymous rates at alpha = 0, beta = 1 (diagonal ignored) */
} h3g_fel_model;

typedef struct {
    double alpha, beta;       /* alternative-model MLE */
    double alpha_null;        /* null-model (alpha = beta) MLE */
    double log_l_alt, log_l_null;
    double lrt, p_value;
    int evaluations;          /* likelihood evaluations used; 0 for an invariant pattern (not fitted) */
    double beta_nuisance;     /* beta on the background branches (h3g_fel_run_tested with a background); else 0 */
} h3g_fel_result;

/* Fit every pattern of prob.  branch_lengths[n_nodes] are in the reference's
 * FEL time (input length x 3 / mean rate of the base model, fel.hpp:230-273);
 * out[n_patterns].  Blocks until done.  The problem's installed model (if
 * any) is left untouched; h3g_last_eval_transfer then reports the bytes the
 * whole run moved between host and device, and h3g_last_eval_stats the run's
 * host wall time and kernel launches. */
h3g_status h3g_fel_run(h3g_problem* prob, const h3g_fel_model* model, const double* branch_lengths, h3g_fel_result* out);

/* As h3g_fel_run with the tested branches given: tested[n_nodes] != 0 marks a
 * tested branch (the root's entry is ignored).  When every branch is tested
 * this is h3g_fel_run.  Otherwise every pattern runs the reference's
 * branch-subset search (FELAnalyzer::analyze_pattern, fel.hpp:462-572): the
 * alternative model has alpha, beta on the tested branches and beta_nuisance
 * on the others (12-point grid, bounded 3-D Nelder-Mead), the null model sets
 * beta = alpha (the initial point and a 7 x 4 grid, bounded 2-D Nelder-Mead).
 * A branch evolves under Q = alpha Qs + beta Qn of its set, i.e. the MG94
 * model Qs + (beta / alpha) Qn with time scaled by alpha; when
 * |beta - beta_nuisance| < 1e-9 both sets use the tested one.  Background
 * branch lengths are converted by the caller (fel.hpp:230-266). */
h3g_status h3g_fel_run_tested(h3g_problem* prob, const h3g_fel_model* model, const double* branch_lengths,
                              const uint8_t* tested, h3g_fel_result* out);

/* ---------------------------------------------------------------- MEME
 * Mixed-effects model of episodic selection per site on the device, replacing
 * MEMEAnalyzer::analyze_pattern / run (include/hyphy/analyses/meme.hpp:166-632,
 * :634-676) with every branch tested (h3g_meme_run_tested below for a
 * tested / background split).  Per pattern: the FEL
 * fit above as the starting point; the alternative model (alpha, omega1, p1,
 * beta+) by the bounded 4-D Nelder-Mead from the reference's start grid; when
 * beta+ > alpha and p+ > 1e-6, the null model (beta+ = alpha) by a 3-D
 * Nelder-Mead, a warm-started alternative refit when the null is better, the
 * mixture LRT p-value 2/3 (0.45 erfc(sqrt(LRT/2)) + 0.55 exp(-LRT/2)) and the
 * empirical Bayes factor of every branch.  A likelihood evaluation mixes the
 * models of omega1 and beta+ / alpha with weights (p1, 1 - p1) at the
 * transition-matrix level on every branch, time scaled by alpha. */
typedef struct {
    double alpha, beta1, p1, beta_plus, p_plus;   /* MEME MLE (beta1 = alpha omega1) */
    double lrt, p_value;
    int branches_under_selection;                 /* branches with EBF >= 100 */
    double total_branch_length;
    double log_l_meme, log_l_fel;
    double p_value_meme_vs_fel;                   /* exp(-LRT(MEME vs FEL) / 2), 1 when MEME is not better */
    double fel_alpha, fel_beta;
    int evaluations;          /* likelihood evaluations of the MEME search (FEL excluded); 0 for an invariant pattern */
    double beta_bg;           /* beta on the background branches (h3g_meme_run_tested with a background); else 0 */
} h3g_meme_result;

/* Fit every pattern of prob; branch_lengths as for h3g_fel_run; out[n_patterns].
 * branch_ebf, when not NULL, receives [n_patterns][n_nodes] empirical Bayes
 * factors (1 for the root, for invariant patterns and where no EBF is computed). */
h3g_status h3g_meme_run(h3g_problem* prob, const h3g_fel_model* model, const double* branch_lengths, h3g_meme_result* out,
                        double* branch_ebf);

/* As h3g_meme_run with the tested branches given (meme.hpp:84-92, :219-632):
 * tested[n_nodes] != 0 marks a branch of the MEME test (the root's entry is
 * ignored); fel_tested[n_nodes] likewise for the FEL baseline of each pattern,
 * NULL when it is the same set (the reference partitions FEL's branches with
 * {T}-tag detection and MEME's without, so the two differ only for "All" on a
 * tagged tree).  With a background, the background branches evolve under
 * Q = alpha Qs + beta_bg Qn: the alternative model adds beta_bg (5-D
 * Nelder-Mead from the start grid with beta_bg = FEL's beta_nuisance), the null
 * model beta+ = alpha keeps it free (4-D), background branches get EBF 1, and
 * the site's tree length weighs them by their own rate. */
h3g_status h3g_meme_run_tested(h3g_problem* prob, const h3g_fel_model* model, const double* branch_lengths,
                               const uint8_t* tested, const uint8_t* fel_tested, h3g_meme_result* out, double* branch_ebf);

/* ---------------------------------------------------------------- nucleotide GTR
 * The nucleotide log-likelihood of LikelihoodEngine::compute_gtr_log_likelihood
 * (include/hyphy/core/likelihood.hpp:181-254) on a problem whose patterns are
 * nucleotide patterns (states 0..3 or -1, masks over A C G T as built by
 * Alignment::to_nucleotide_alignment, alignment.hpp:832-890).  P[n_nodes][4][4]
 * row-major transition matrices (the root's entry ignored), pi[4] the root
 * frequencies.  *lnl = sum over patterns of weight x (log L, or -1e20 when
 * L <= 0), a fixed-order Neumaier sum; site_lnl[n_patterns] (may be NULL) the
 * per-pattern log-likelihoods.  One thread per pattern walks the tree depth-first
 * (FP64, power-of-two rescaling).  Blocks until done. */
h3g_status h3g_nuc_eval_from_P(h3g_problem* prob, const double* P, const double* pi, double* lnl, double* site_lnl);

/* ---------------------------------------------------------------- alignments
 * Alignment::finalize's codon translation, nucleotide counts and pattern
 * compression (include/hyphy/core/alignment.hpp:665-722, :893-911, :1021-1078)
 * on the device.  Each codon column of the in-frame alignment is translated
 * per taxon to a sense-codon state (-1 when ambiguous, a gap or a stop) and a
 * mask of the compatible sense codons (genetic_code.hpp:82-109: IUPAC
 * ambiguity, '!' and all-ambiguous triplets and stops give every sense codon);
 * identical columns (same states and masks) form one site pattern, patterns
 * are numbered in the order of their first site, and the weight of a pattern
 * is its number of sites.  Unambiguous A/C/G/T(U) characters are counted per
 * codon position.  Identity is decided by comparing the translated columns in
 * full, so the result does not depend on the column hash. */
typedef struct {
    int S;                          /* sense codons, 1..63 */
    const int8_t* codon_to_sense;   /* [64] sense index of codon 16 n1 + 4 n2 + n3 (A, C, G, T = 0..3), -1 for a stop */
} h3g_genetic_code;

typedef struct {
    int64_t n_patterns;             /* distinct columns */
    int64_t pos_counts[12];         /* unambiguous nucleotides at codon position p, [p][A C G T] */
    int rounds;                     /* hash rounds used (1 unless hashes of different columns collided) */
    int hash_bits;                  /* in: 0 or 64 for the full column hash; 1..63 keeps only that many bits (tests) */
    int profile;                    /* in: nonzero records device times of the stages into stage_ms */
    double stage_ms[4];             /* translate (k_translate), rounds (hash / insert / verify), numbering (scan),
                                       output (assign / gather); device event times, 0 unless profile */
    int launches;                   /* kernels the call launched */
} h3g_compress_info;

/* seqs: n_taxa rows of n_nuc characters (n_nuc a positive multiple of 3), row i at
 * seqs + i * row_stride, host memory.  n_codons = n_nuc / 3.  Outputs, host memory,
 * sized for n_codons patterns (the first n_patterns rows are written):
 * site_to_pattern[n_codons], pattern_weight[n_codons], pattern_first_site[n_codons]
 * (may be NULL), pattern_states[n_codons * n_taxa] and pattern_masks[n_codons * n_taxa]
 * (pattern-major, as SitePattern::states / ambiguous_masks).  info->hash_bits is read,
 * the rest written.  The context's stream carries the copies and kernels; the call
 * blocks until the results are on the host. */
h3g_status h3g_alignment_compress(h3g_ctx* ctx, int n_taxa, int64_t n_nuc, const char* seqs, size_t row_stride,
                                  const h3g_genetic_code* code, int32_t* site_to_pattern, int32_t* pattern_weight,
                                  int32_t* pattern_first_site, int8_t* pattern_states, uint64_t* pattern_masks,
                                  h3g_compress_info* info);

/* The same with every array in device memory (d_seqs read, the outputs written
 * on the context's stream).  info (host) receives n_patterns and the counts;
 * the call returns once they are known, the outputs complete on the stream. */
h3g_status h3g_alignment_compress_device(h3g_ctx* ctx, int n_taxa, int64_t n_nuc, const char* d_seqs, size_t row_stride,
                                         const h3g_genetic_code* code, int32_t* d_site_to_pattern, int32_t* d_pattern_weight,
                                         int32_t* d_pattern_first_site, int8_t* d_pattern_states, uint64_t* d_pattern_masks,
                                         h3g_compress_info* info);

#ifdef __cplusplus
}
#endif

#endif /* H3G_H */
