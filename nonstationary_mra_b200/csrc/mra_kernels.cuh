// Launch interface between the C-ABI layer (mra_api.cu) and the FP64 region
// kernels (mra_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mra_device.cuh"

namespace mra {

// Everything a kernel needs to address the resident structure and buffers.
struct DevTree {
    int J, M, r, L;            // L = M-1 ancestor levels of a finest region
    long n_int, n_fin, n_obs, n_pred;
    long obs0, pred0;          // first obs / pred index in the joint point arrays
    PointSet pts;              // knots | obs | preds, with their fields
    const double* y;           // [n_obs]
    const int64_t* obs_off;    // [n_fin+1]
    const int64_t* pred_off;   // [n_fin+1] (or nullptr)
    const int64_t* fin_anc;    // [n_fin][L] ancestors of each finest region, level 0 first
    const int64_t* fin_order;  // [n_fin] finest regions, most expensive first
    const int64_t* lsig_off;   // [n_fin+1] offsets of the n_k x n_k blocks
    const int64_t* pc_off;     // [n_fin+1] offsets of the n_k x n_p,k prediction blocks
    const int64_t* child_lo;   // [J^(M-2)] first finest child of each level M-2 region
    const int64_t* child_hi;   // one past the last
    int64_t u_off[kMaxLevels]; // offset of level m's U (= G) blocks, m*r*r doubles per region
    // prior
    double* Lprior;            // [n_int][r*r]
    double* U;                 // per level m: [J^m][(m r) x r], ld = m r
    double* Ufin;              // [n_obs][L r]   finest U_{k,j} columns, obs-major
    double* Bhat;              // [n_obs][L r]   B^_k transposed, obs-major
    double* yt;                // [n_obs]        L_Sigma^{-1} y per region
    double* Lsig;              // CSR n_k x n_k  finest Cholesky factors
    double* dfin;              // [n_fin]
    // posterior
    double* Lpost;             // [n_int][r*r]
    double* vpost;             // [n_int][r]
    double* G;                 // same layout as U: [J^m][r x (m r)], ld = r
    double* dpost;             // [n_int]
    double* aout[2];           // ping-pong A~ slices of one level
    double* wout[2];           // ping-pong w~ of one level
    double* ws;                // per-CTA posterior workspace
    long ws_stride;            // doubles per CTA
    // prediction
    double* P;                 // [n_pred][L r]
    double* Bt;                // [n_pred][L r]
    double* Pc;                // CSR n_k x n_p,k
    double* mean;              // [n_pred]
    double* var;               // [n_pred]
    // bookkeeping
    int* queue;                // work-queue counters
    int* err;                  // [0]: status, [1]: region (low), [2]: region (high)
};

__host__ __device__ inline long level_start(int J, int m) {
    long s = 0, p = 1;
    for (int i = 0; i < m; ++i) { s += p; p *= J; }
    return s;
}
__host__ __device__ inline long level_count(int J, int m) {
    long p = 1;
    for (int i = 0; i < m; ++i) p *= J;
    return p;
}
__host__ __device__ inline long n_slices(int m) { return (long)m * (m + 1) / 2; }
// slice index of block (j,k), j <= k < m, row-major over the upper triangle
// (the order of class_approximation.cpp:62-73)
__host__ __device__ inline long slice_index(int m, int j, int k) { return (long)j * m - (long)j * (j - 1) / 2 + (k - j); }

// θ-dependent field evaluation parameters (device pointers)
struct FieldParams {
    int basis;                 // 0 Wendland, 1 Gaussian
    double basis_len;
    long nb[3];
    const double* centers[3];  // [3][nb]
    const double* theta;       // [0..2] scales, [3..5] intercepts, [6..8] stationary sill/range/nugget
    const double* weights[3];  // [nb]
};

// Sets the text returned by mra_last_error() on this thread.
void set_last_error(const char* msg);

void launch_fields(const Geom& g, const FieldParams& fp, const double* c0, const double* c1, const double* c2,
                   long n, double* s2, double* beta, double* t2, cudaStream_t st);
void launch_prior_level(const Geom& g, const DevTree& t, int m, int grid, cudaStream_t st);
void launch_finest(const Geom& g, const DevTree& t, int grid, bool keep_ufin, cudaStream_t st);
void launch_posterior_level(const Geom& g, const DevTree& t, int m, int grid, bool keep_g, cudaStream_t st);
void launch_predict(const Geom& g, const DevTree& t, int grid, cudaStream_t st);
void launch_reduce(const DevTree& t, double* out, cudaStream_t st);
void launch_sample(const DevTree& t, const double* z_int, const double* z_obs, double* y_out, int grid,
                   cudaStream_t st);
void launch_cov_block(const Geom& g, const PointSet& P, long a0, int na, long b0, int nb, bool self, double* out,
                      cudaStream_t st);

}  // namespace mra
