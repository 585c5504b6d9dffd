// Launch interface between the C-ABI layer (mra_api.cu) and the region
// kernels (mra_kernels.cu), templated on the storage type T (double: plain
// FP64 path, float: mixed path).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mra_b200.h"
#include "mra_device.cuh"

namespace mra {

// Everything a kernel needs to address the resident structure and buffers.
template <typename T>
struct DevTree {
    int J, M, r, L;            // L = M-1 ancestor levels of a finest region
    long n_int, n_fin, n_obs, n_pred;
    long obs0, pred0;          // first obs / pred index in the joint point arrays
    int tf;                    // largest subtree (in observations) kept in factored form
    PointSet pts;              // knots | obs | preds, with their fields (FP64)
    const double* y;           // [n_obs]
    const int64_t* obs_off;    // [n_fin+1]
    const int64_t* pred_off;   // [n_fin+1]
    const int64_t* fin_anc;    // [n_fin][L] ancestors of each finest region, level 0 first
    const int64_t* sub_lo;     // [n_int] first observation of each interior region's subtree
    const int64_t* sub_hi;     // [n_int] one past the last
    const int64_t* child_lo;   // [J^(M-2)] first finest child of each level M-2 region
    const int64_t* child_hi;   // one past the last
    const int64_t* par_order;  // [n_fin_items] finest-kernel work items, most expensive first: a value
                               // v < J^(M-3) is the level M-3 unit v, else the level M-2 group v - J^(M-3)
    long n_fin_items;
    const int64_t* pred_order; // [J^(M-2)] level M-2 regions (local index), most expensive prediction work first
    const int64_t* post_order; // [n_int] per level m, at level_start(m): the level's regions (local index),
                               // most expensive posterior step first
    const int8_t* factored;    // [n_int] 1: the region's posterior output is kept as F, f
    const int8_t* active;      // [n_int] sub-tree sharding: 0 = the region belongs to another rank's
                               // sub-tree and is skipped; nullptr: every region is computed
    const int64_t* dslot;      // [n_int] slot of a dense region among its level's dense regions (-1: factored)
    const int64_t* lsig_off;   // [n_fin+1] offsets of the n_k x n_k blocks
    const int64_t* pc_off;     // [n_fin+1] offsets of the n_k x n_p,k prediction blocks
    int64_t u_off[kMaxLevels]; // offset of level m's U (= G) blocks, m*r*r per region
    // prior
    T* Lprior;                 // [n_int][r*r]
    T* Pinv;                   // [n_int][r*r] inverse of each prior factor (L^{-1} applied as a product)
    double* ldprior;           // [n_int] 2 sum log diag of the prior factor
    T* U;                      // per level m: [J^m][(m r) x r], ld = m r
    T* Ufin;                   // [n_obs][L r]   finest U_{k,j} columns, obs-major
    T* Bhat;                   // [n_obs][L r]   B^ transposed, obs-major (the finest F)
    double* yt;                // [n_obs]        L_Sigma^{-1} y (the finest f)
    T* Lsig;                   // CSR n_k x n_k  finest Cholesky factors
    // posterior
    T* Lpost;                  // [n_int][r*r]
    double* vpost;             // [n_int][r]
    T* G;                      // like U: [J^m][r x (m r)], ld = r (prediction mode)
    T* Lpinv;                  // [n_int][r*r] inverse of each posterior factor (FP64 prediction mode, r <= 64), else null
    double* dpost;             // [n_int] posterior log-lik terms
    double* dfin;              // [J^(M-2)] finest-level log-lik terms of each sibling group
    int fuse_post;             // 1: the finest-group kernel also runs the level M-2 posterior
    T* aout[2];                // dense A~ slices of one level's dense regions (by dslot), ping-pong by level parity
    double* wout[2];           // dense w~ of one level's dense regions (by dslot)
    T* Fbuf[2];                // factored F of one level: [n_obs][m r]
    double* fbuf[2];           // factored f of one level: [n_obs]
    T* cbuf;                   // covariance blocks of a chunk of one prior level's regions
    long cbuf_elems;           // its size in elements (a multiple of nothing in particular)
    T* ws;                     // per-CTA workspace (T)
    long ws_stride;
    double* wsd;               // per-CTA workspace (FP64)
    long wsd_stride;
    // prediction
    T* P;                      // [n_pred][L r]
    T* Bt;                     // [n_pred][L r]
    T* Pc;                     // CSR n_k x n_p,k
    double* mean;              // [n_pred]
    double* var;               // [n_pred]
    // bookkeeping
    int* queue;                // work-queue counters (kQueueCounters, zeroed before every evaluation):
                               // [0] finest items, [1] prediction items, [kQueuePost + m] posterior level m
    int* err;                  // [0]: status, [1]: region (low), [2]: region (high)
};

constexpr int kQueuePost = 4;
constexpr int kQueueCounters = kQueuePost + kMaxLevels;

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
template <typename T>
__device__ __forceinline__ bool skipped(const DevTree<T>& t, long region) {
    return t.active && !t.active[region];
}
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

// Validates a model description (kinds in range, positive basis length and
// non-NULL basis tables for nonstationary fields); sets the error text.
mra_status check_model(const mra_model* m);

// Opts the region kernels into their dynamic shared memory size on the current
// device; call before the first launch (and before any stream capture).
cudaError_t prepare_kernels();

// FP64 GEMM tile width per product-width bucket on the current device
// (c_gemm_nw in mra_device.cuh).
cudaError_t set_gemm_tiles(const int nw[3]);

void launch_fields(const Geom& g, const FieldParams& fp, const double* c0, const double* c1, const double* c2,
                   long n, double* s2, double* beta, double* t2, cudaStream_t st);
// Events recorded around each covariance-block launch of a prior level, so
// that the caller can split the level's device time between the covariance
// launches and the region launches.
struct CovTiming {
    cudaEvent_t* ev;  // two per launch: before and after
    int cap;          // launches that can be timed
    int used;         // launches timed so far
    bool capturing;   // record as external nodes of the graph being captured
    bool overflow;    // a launch went untimed (cap reached)
};
// Covariance-block launches and region launches of one prior level, in chunks
// of regions whose blocks fit t.cbuf; returns the number of kernels launched.
template <typename T>
int launch_prior_level(const Geom& g, const DevTree<T>& t, int m, int grid, cudaStream_t st, CovTiming* tm = nullptr);
// The finest groups; returns the number of kernels launched (1).
template <typename T>
int launch_finest_group(const Geom& g, const DevTree<T>& t, int grid, bool keep, cudaStream_t st);
template <typename T>
void launch_posterior_level(const Geom& g, const DevTree<T>& t, int m, int grid, bool keep, cudaStream_t st);
template <typename T>
void launch_predict(const Geom& g, const DevTree<T>& t, int grid, cudaStream_t st);
template <typename T>
void launch_reduce(const DevTree<T>& t, double* out, cudaStream_t st);
// out[i] = (To) in[i]
template <typename Ti, typename To>
void launch_convert(const Ti* in, To* out, long n, cudaStream_t st);
template <typename T>
void launch_sample(const DevTree<T>& t, const double* z_int, const double* z_obs, double* y_out, int grid,
                   cudaStream_t st);
void launch_cov_block(const Geom& g, const PointSet& P, long a0, int na, long b0, int nb, bool self, double* out,
                      cudaStream_t st);

}  // namespace mra
