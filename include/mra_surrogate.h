/*
 * nonstationary_mra_b200 -- C ABI of the parameter-fitting side of the MRA
 * path: the bound-constrained derivative-free optimizer that drives the
 * likelihood, and the MLP surrogate of the log-likelihood that proposes
 * optimizer steps.
 *
 * Optimizer: replaces the reference's dlib::find_min_bobyqa call
 * (src/optimization.cpp:158-192, objective :107-150): minimise f(x) over
 * lower <= x <= upper from x0 with initial trust radius rho_begin down to
 * rho_end and npt interpolation points (the reference uses n = 3 scales,
 * npt = 7, bounds [1e-2, 1e2], rho 0.1 -> 1e-6).  Host code, no GPU.
 *
 * Surrogate: no counterpart in the reference.  An MLP n_in -> 128 -> 128 -> 1
 * with SiLU activations, weights held in BF16 for the forward and backward
 * passes (an FP32 master copy is what Adam updates) and FP32 accumulation,
 * trained on the device by this library's own kernels on (theta, loglik)
 * pairs.
 *
 * Conventions as in mra_b200.h: host pointers, every call returns an
 * mra_status, errors leave a message in mra_last_error().
 */
#ifndef MRA_SURROGATE_H
#define MRA_SURROGATE_H

#include <stdint.h>

#include "mra_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ optimizer */

/* Objective: returns f(x) for x[n]; a non-finite return value or a nonzero
 * *stop ends the run (the best point so far is kept). */
typedef double (*mra_objective_fn)(const double* x, void* user, int32_t* stop);

typedef struct {
    double rho_begin;      /* initial trust-region radius (reference: 0.1)           */
    double rho_end;        /* final radius (reference: 1e-6)                          */
    int32_t npt;           /* interpolation points, n+2 <= npt <= (n+1)(n+2)/2;
                              0 = 2n+1 (reference: 7 for n = 3)                        */
    int32_t max_evals;     /* evaluation budget (reference: MAX_ITERATIONS)           */
} mra_opt_config;

typedef struct {
    double f_best;         /* smallest f seen                                          */
    int32_t evals;         /* objective calls made                                     */
    int32_t status;        /* 0 converged (rho reached rho_end), 1 budget used,
                              2 stopped by the objective, 3 trust region failure      */
    double rho_final;      /* last trust-region radius bound                           */
} mra_opt_result;

/* Minimises f over the box; x (length n) holds x0 on entry and the best point
 * on return.  lower/upper may not be NULL; x0 is clipped into the box. */
mra_status mra_opt_minimize(int32_t n, double* x, const double* lower, const double* upper,
                            const mra_opt_config* cfg, mra_objective_fn f, void* user, mra_opt_result* out);

/* ----------------------------------------------------------------- surrogate */

typedef struct mra_mlp mra_mlp;

/* n_in inputs (1..64), hidden width 128 (the only width built); weights are
 * initialised uniformly in +-sqrt(6/(fan_in+fan_out)), biases zero, from
 * `seed` (a host generator, so the draw does not depend on the device). */
mra_status mra_mlp_create(int32_t n_in, int32_t hidden, uint64_t seed, mra_mlp** out);
mra_status mra_mlp_destroy(mra_mlp* mlp);

/* Number of FP32 parameters: W1 [hidden][n_in], b1 [hidden], W2 [hidden][hidden],
 * b2 [hidden], w3 [hidden], b3 [1], packed in that order (row-major). */
mra_status mra_mlp_num_params(const mra_mlp* mlp, int64_t* n);
mra_status mra_mlp_get_params(mra_mlp* mlp, float* params);
/* Sets the FP32 master parameters (and their BF16 copies); clears Adam's moments. */
mra_status mra_mlp_set_params(mra_mlp* mlp, const float* params);

/* Training set: x [n][n_in], t [n], already standardised by the caller.
 * Replaces the previous set (n <= 65536). */
mra_status mra_mlp_set_data(mra_mlp* mlp, const float* x, const float* t, int64_t n);

/* Full-batch loss (1/n) sum (y - t)^2 and its gradient w.r.t. every parameter
 * (FP32, packed like the parameters) at the current weights. */
mra_status mra_mlp_grad(mra_mlp* mlp, float* grad, float* loss);

/* `steps` full-batch Adam steps (beta1 0.9, beta2 0.999, eps 1e-8) with
 * learning rate lr; *loss_out (may be NULL) = loss before the last step. */
mra_status mra_mlp_train(mra_mlp* mlp, int32_t steps, float lr, float* loss_out);

/* y [n] = network(x [n][n_in]); dydx [n][n_in] (may be NULL) = d y / d x. */
mra_status mra_mlp_predict(mra_mlp* mlp, const float* x, int64_t n, float* y, float* dydx);

#ifdef __cplusplus
}
#endif

#endif /* MRA_SURROGATE_H */
