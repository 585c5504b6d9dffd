/*
 * nonstationary_mra_b200 -- C ABI of the B200 (sm_100a) MRA hot path.
 *
 * This boundary replaces, for one GPU, the reference's
 *   Approximation::likelihood()      include/class_approximation.hpp:53
 *                                    (src/class_approximation.cpp:466-470)
 *   Approximation::predict()         include/class_approximation.hpp:56
 *                                    (src/class_approximation-predict.cpp:15-200)
 *   evaluate_*covariance()           include/evaluate_covariance.hpp:25,47,71,88
 *   Nonstationary_covariance::get_*  include/class_nonstationary_covariance.hpp:55-64
 * The partition / knots / observation arrays that the reference keeps in
 * `Partition` (include/class_partition.hpp:26-61) are passed in once as flat
 * arrays (mra_structure) and stay resident in HBM; each likelihood evaluation
 * then only takes the covariance parameters (mra_theta).
 *
 * Conventions: plain pointers and sizes, host memory unless a name says
 * otherwise, column-major matrices as in the reference.  Every function
 * returns an mra_status; nothing exits the process (the reference prints and
 * calls exit(); the drop-in C++ host maps statuses to that behaviour).
 * A context is single-threaded and stream-ordered: do not call into the same
 * mra_ctx from two threads at once.
 */
#ifndef MRA_B200_H
#define MRA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MRA_OK = 0,
    MRA_ERR_ARG = 1,       /* invalid argument or inconsistent structure */
    MRA_ERR_CUDA = 2,      /* CUDA runtime error (message in mra_last_error) */
    MRA_ERR_OOM = 3,       /* device allocation failed */
    MRA_ERR_NOT_SPD = 4,   /* a Cholesky pivot was not positive (region in mra_stats) */
    MRA_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up */
    MRA_ERR_STATE = 6,     /* call out of order (e.g. predict without predictions) */
    MRA_ERR_NO_DEVICE = 7  /* no usable sm_100 device */
} mra_status;

/* Distance between points (coordinates are 3 doubles per point, SoA). */
typedef enum {
    MRA_DIST_CHORDAL = 0,      /* (x,y,z) on the unit sphere, |p-q| * dist_scale  (CHORDAL_DISTANCE_FLAG=true)  */
    MRA_DIST_GREAT_CIRCLE = 1, /* (lon,lat) degrees, arccos(...) * dist_scale      (CHORDAL_DISTANCE_FLAG=false) */
    MRA_DIST_EUCLID2D = 2      /* (x,y) planar, |p-q| * dist_scale                  (extension)                   */
} mra_distance;

typedef enum {
    MRA_BASIS_WENDLAND = 0,    /* (1-d)^6 (35d^2+18d+3)/3 for d<1 (reference)      */
    MRA_BASIS_GAUSSIAN = 1     /* exp(-d^2/2) (extension)                          */
} mra_basis;

typedef enum {
    MRA_PRECISION_FP64 = 0,    /* plain FP64 path                                   */
    MRA_PRECISION_MIXED = 1    /* FP32 covariance + tensor-core trailing updates,
                                  FP64 diagonal-block Cholesky and accumulations   */
} mra_precision;

/* Partition tree, knots, observations and (optionally) prediction locations.
 * Interior regions 0..n_interior-1 are levels 0..M-2 in heap order (children
 * of region i are i*J+1..i*J+J, class_approximation.cpp:36-43).  Finest region
 * k (reference index n_interior+k) has parent finest_parent[k]; the finest
 * children of one parent must be a contiguous range, as the reference assumes
 * (childrenStart/childrenEnd, class_partition.cpp:740-770).                    */
typedef struct {
    int32_t J;                     /* NUM_PARTITIONS_J (2 or 4)                     */
    int32_t M;                     /* NUM_LEVELS_M (>= 2)                           */
    int32_t r;                     /* knots per interior region                     */
    int32_t reserved;
    uint64_t n_interior;           /* (J^(M-1)-1)/(J-1)                             */
    uint64_t n_finest;
    const uint64_t* finest_parent; /* [n_finest]                                     */
    const double* knots;           /* [3][n_interior*r]: coordinate c of knot q of
                                      region i at knots[c*n_interior*r + i*r + q]   */
    const uint64_t* obs_offset;    /* [n_finest+1] CSR offsets into observations     */
    const double* obs;             /* [3][n_obs]                                     */
    const double* obs_value;       /* [n_obs] residuals y (knotsResidual)            */
    const uint64_t* pred_offset;   /* [n_finest+1] or NULL                           */
    const double* pred;            /* [3][n_pred] or NULL                            */
} mra_structure;

/* One nonstationary log-field: log f(s) = intercept + sum_k w_k basis(|s-c_k|/len). */
typedef struct {
    uint64_t n_basis;
    const double* centers;         /* [3][n_basis] in the point coordinate system    */
    const double* weights;         /* [n_basis]                                      */
    double intercept;
} mra_field;

typedef struct {
    int32_t nonstationary;         /* NONSTATIONARY_FLAG                             */
    int32_t distance;              /* mra_distance                                   */
    int32_t nu_x2;                 /* 2*nu: 1 = exponential (reference), 3 = Matern 3/2 */
    int32_t basis;                 /* mra_basis                                      */
    double prefactor_exp;          /* e in (b1 b2 / bbar^2)^e: 1.5 (reference), 1.0 (d=2) */
    double dist_scale;             /* 6371 (reference) or 1                          */
    double basis_len;              /* WENDLAND_LEN or Gaussian width                 */
    mra_field field[3];            /* sill (sigma^2), range (beta), nugget (tau^2)   */
} mra_model;

/* Per-evaluation parameters: the six arguments of Approximation's constructor
 * (include/class_approximation.hpp:46) plus optional overrides of the field
 * intercepts/weights (the extension's 19-dimensional theta).                  */
typedef struct {
    double sill, range, nugget;                     /* stationary model          */
    double sill_scale, range_scale, nugget_scale;   /* nonstationary scales      */
    const double* weights[3];      /* NULL: keep the model's weights             */
    const double* intercepts;      /* NULL or [3]: replace the model's intercepts */
} mra_theta;

/* Kernel kinds in mra_stats.timed_kind. */
typedef enum {
    MRA_KERNEL_FIELDS = 0,         /* sigma^2 / beta / tau^2 at every point          */
    MRA_KERNEL_PRIOR_LEVEL = 1,    /* prior of one interior level (timed_level = m)  */
    MRA_KERNEL_FINEST = 2,         /* finest level + level M-2 posterior, per sibling group */
    MRA_KERNEL_POSTERIOR_LEVEL = 3,/* posterior of one interior level                */
    MRA_KERNEL_REDUCE = 4,         /* final log-likelihood sum                       */
    MRA_KERNEL_PREDICT = 5,        /* prediction                                     */
    MRA_KERNEL_CONVERT = 6         /* FP32 -> FP64 widening between the mixed stages */
} mra_kernel_kind;

#define MRA_MAX_TIMED 40

typedef struct {
    double d;                      /* the reference's internal loglikelihood after
                                      likelihood(): sum of log-dets and quadratic forms */
    double loglik;                 /* -0.5 (d + n log(2*3.14159265359))          */
    double ms_total;               /* device time of the last evaluation          */
    double ms_fields, ms_prior, ms_finest, ms_posterior, ms_predict;
    double flop_last;              /* FLOPs of the algorithm run by the last evaluation */
    double flop_reference;         /* FLOPs of the reference's algorithm on the same tree */
    uint64_t bytes_device;         /* device memory held by the context           */
    int64_t bad_region;            /* region of the last MRA_ERR_NOT_SPD, else -1 */
    int32_t kernel_launches;       /* kernels launched by the last evaluation     */
    int32_t graph_replays;
    int32_t n_timed;               /* launches of the last evaluation, in order   */
    int32_t timed_kind[MRA_MAX_TIMED];   /* mra_kernel_kind                        */
    int32_t timed_level[MRA_MAX_TIMED];  /* tree level for per-level kernels, else -1 */
    double timed_ms[MRA_MAX_TIMED];      /* device time of each launch (CUDA events) */
    double timed_flop[MRA_MAX_TIMED];    /* algorithmic FLOPs of each launch          */
    double timed_ms_cov[MRA_MAX_TIMED];  /* of timed_ms, the device time of the prior
                                            level's covariance-block launches (the rest
                                            is its region launches); 0 for other kinds,
                                            -1 where some went untimed */
} mra_stats;

typedef struct mra_ctx mra_ctx;

/* Uploads the structure and model; allocates every device buffer up front. */
mra_status mra_create(const mra_structure* s, const mra_model* m, int32_t precision, mra_ctx** out);
mra_status mra_destroy(mra_ctx* ctx);

/* Sets the parameters for the next evaluations (a 1-10 word host->device copy). */
mra_status mra_set_theta(mra_ctx* ctx, const mra_theta* theta);

/* Replaces the observation values y (n_obs doubles, host memory). */
mra_status mra_set_obs_values(mra_ctx* ctx, const double* y);

/* Prior + posterior: Approximation::likelihood() in likelihood mode.
 * d_out / loglik_out may be NULL. */
mra_status mra_loglik(mra_ctx* ctx, double* d_out, double* loglik_out);

/* Prior + posterior + prediction: Approximation::likelihood() then predict() in
 * prediction mode.  mean/var: n_pred doubles each, in finest-region order (the
 * order of dump_prediction_result, class_approximation.cpp:493-535). */
mra_status mra_predict(mra_ctx* ctx, double* mean, double* var);

/* Captures the evaluation into CUDA graphs: prior -> posterior, which later
 * mra_loglik calls replay, and, when the structure has prediction locations,
 * prior -> posterior (predictive factors kept) -> prediction, which later
 * mra_predict calls replay.  theta and the observation values are read from
 * device memory by the captured kernels, so mra_set_theta / mra_set_obs_values
 * between replays need no recapture. */
mra_status mra_capture_graph(mra_ctx* ctx);

mra_status mra_get_stats(const mra_ctx* ctx, mra_stats* out);

/* Diagnostics, no counterpart in the reference: the parts of d (the reference's
 * internal loglikelihood) from the last evaluation, by where they are computed.
 * out[m], m = 0..M-2: sum over the level-m regions of their posterior terms
 * (-2 log|L_i| + 2 log|L~_i| - v_i^T v_i, or the factored form's equal);
 * out[M-1]: the finest-level terms (y~^T y~ + 2 log|L_Sigma|) together with the
 * level M-2 posterior terms, which one kernel computes.  sum(out) = d up to
 * summation order.  n_out >= M.  Waits for the context's stream. */
mra_status mra_get_terms(mra_ctx* ctx, double* out, int32_t n_out);

/* Draws y from the MRA prior at the current theta:
 * y = sum_j U_{obs,j}^T z_{a_j} + L_Sigma z_k, z_interior [n_interior*r],
 * z_obs [n_obs] standard normals given by the caller (host memory). */
mra_status mra_sample_prior(mra_ctx* ctx, const double* z_interior, const double* z_obs, double* y_out);

/* Covariance blocks with the reference's layout out[i1*n2+i2]
 * (evaluate_covariance.cpp:56-313), computed on the device.  p1/p2 are
 * [3][n] coordinates; the fields come from the model and theta.  Cross block
 * when self == 0, symmetric self block with sigma^2+tau^2 on the diagonal
 * when self != 0 (then p2/n2 are ignored). */
mra_status mra_eval_covariance(const mra_model* m, const mra_theta* theta, const double* p1, uint64_t n1,
                               const double* p2, uint64_t n2, int32_t self, double* out);

/* sigma^2, beta, tau^2 at n points (Nonstationary_covariance::get_* times the
 * scales), computed on the device.  out: [3][n]. */
mra_status mra_eval_fields(const mra_model* m, const mra_theta* theta, const double* p, uint64_t n,
                           double* out);

/* Autotuner of the FP64 products' tile shapes.  No counterpart in the
 * reference.  Times `evals` log-likelihood evaluations of this context (after
 * one warm-up) for each candidate CTA tile width per product-width bucket
 * (products at most 16, at most 32, and more than 32 columns wide; widths of
 * 16, 32 or 64 columns over 64 rows) and keeps the fastest for the device.
 * The choice is per device and shared by every context on it; results are
 * bitwise the same for every choice (each element is accumulated by one thread
 * in the same order).  choice_out (3 ints, may be NULL): the widths in units of
 * 16 columns; ms_out (may be NULL): the best time per evaluation. */
mra_status mra_autotune(mra_ctx* ctx, int32_t evals, int32_t* choice_out, double* ms_out);

/* Selects the CUDA device that the calling thread's next mra_create uses
 * (one process per GPU: call it with the local rank before mra_create). */
mra_status mra_set_device(int32_t device);

/* Device-side timer on the context's stream: mra_timer_stop returns the device
 * time between the two calls, covering every copy and kernel the context issued
 * in between (CUDA events; waits for the stream). */
mra_status mra_timer_start(mra_ctx* ctx);
mra_status mra_timer_stop(mra_ctx* ctx, double* ms);

/* Allocation-free covariance blocks.  No counterpart in the reference.
 *
 * Same result and layout as mra_eval_covariance (out[i1*n2+i2]), for callers
 * that cannot let this library allocate device memory: programs that give all
 * device memory to their own pool or arena, and loops that cannot afford the
 * device-wide synchronisation of cudaMalloc/cudaFree on every call.  Inputs and
 * output are the caller's DEVICE buffers: p1_dev [3][n1] and p2_dev [3][n2]
 * coordinates, out_dev n1*n2 doubles (n1*n1 when self != 0; p2_dev/n2 ignored).
 * The model's basis tables and theta are read from host memory as elsewhere,
 * with cudaMemcpyAsync on `stream` (a cudaStream_t; NULL = the legacy default
 * stream): theta always goes through a pageable buffer of the call, and a copy
 * from pageable memory waits for the stream's earlier work before it starts.
 * Basis tables or weights in pinned (page-locked) host memory are copied
 * asynchronously instead, so they must stay unchanged until the stream has
 * passed this call.  The kernels are queued on `stream`; the call does not wait
 * for them.
 *
 * Scratch lives in one fixed array in device global memory, held by every GPU
 * that loads the library until the process exits; limits: n1 + n2 <=
 * MRA_STATIC_MAX_POINTS points and <= MRA_STATIC_MAX_BASIS basis functions per
 * field, larger requests fail with MRA_ERR_ARG.  The first call on a device
 * looks up that array's device address (once per device, with the device
 * current); make that first call before any stream capture.  Every call uses
 * the same array and overwrites all of it that it reads, so calls that overlap
 * on the GPU (other streams, other host threads) race with each other:
 * serialize them. */
#define MRA_STATIC_MAX_POINTS 32768
#define MRA_STATIC_MAX_BASIS 1024
mra_status mra_eval_covariance_static(const mra_model* m, const mra_theta* theta, const double* p1_dev, uint64_t n1,
                                      const double* p2_dev, uint64_t n2, int32_t self, double* out_dev, void* stream);

/* Sub-tree sharding: one log-likelihood over several GPUs, one process (and
 * context, on the same structure) per GPU.  The tree splits at level s into J^s
 * independent sub-trees, as the reference's MPI build splits its regions among
 * ranks (src/class_partition.cpp:1188-1280) and sums the children's
 * contributions on the parent's rank (src/class_approximation.cpp:186-264).
 *
 *   mra_shard_set(ctx, s, owned)      owned[q] != 0 for the level-s regions q
 *                                     (local index 0..J^s-1) this rank computes;
 *                                     1 <= s <= M-3, FP64 path; owned = NULL
 *                                     returns the context to whole evaluations
 *   mra_shard_loglik_subtrees(ctx)    prior of levels < s (every rank), and the
 *                                     prior, finest level and posterior of levels
 *                                     >= s of the owned sub-trees
 *   mra_shard_record_size/export      the owned region q's record: its output to
 *                                     its parent (the reference's A~ and w~, or the
 *                                     factored F, f) and the log-likelihood terms of
 *                                     its sub-tree, n_doubles doubles of host memory
 *   mra_shard_import                  on the rank that finishes: the records of the
 *                                     regions it does not own
 *   mra_shard_loglik_top(ctx, &d, &l) posterior of levels < s and the sum, on the
 *                                     finishing rank after every import: bitwise the
 *                                     whole evaluation's d (every term is computed by
 *                                     the same kernel code and summed in the same order)
 *
 * Record layout (doubles): [kind (0 dense, 1 factored), rows] then the dense
 * slices (s(s+1)/2 r x r, then s r) or the factored rows (rows x s r, then rows),
 * then the posterior terms of the sub-tree's regions level by level (J^(m-s) for
 * m = s..M-2), then the finest-level terms of its J^(M-2-s) sibling groups.
 * While a context is sharded, mra_loglik, mra_predict, mra_sample_prior and
 * mra_capture_graph return MRA_ERR_STATE. */
mra_status mra_shard_set(mra_ctx* ctx, int32_t split_level, const uint8_t* owned);
mra_status mra_shard_loglik_subtrees(mra_ctx* ctx);
mra_status mra_shard_record_size(const mra_ctx* ctx, uint64_t region, uint64_t* n_doubles);
mra_status mra_shard_export(mra_ctx* ctx, uint64_t region, double* record, uint64_t n_doubles);
mra_status mra_shard_import(mra_ctx* ctx, uint64_t region, const double* record, uint64_t n_doubles);
mra_status mra_shard_loglik_top(mra_ctx* ctx, double* d_out, double* loglik_out);

/* Text of the last error on this thread. */
const char* mra_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MRA_B200_H */
