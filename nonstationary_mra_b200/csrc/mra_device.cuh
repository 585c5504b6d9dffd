// Device-side building blocks of the MRA hot path (sm_100a).
//
//  * covariance entries, following src/evaluate_covariance.cpp:155-313 and the
//    fields of src/class_nonstationary_covariance.cpp:479-573;
//  * CTA-cooperative FP64 dense primitives on column-major operands that may
//    live in global or shared memory: tiled GEMM, blocked left / right
//    triangular solves and a blocked right-looking Cholesky.  One CTA owns one
//    region's problem; the region kernels in mra_kernels.cu are sequences of
//    these calls.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mra {

constexpr int kThreads = 256;   // every region kernel runs 256-thread CTAs
constexpr int kMaxLevels = 16;  // NUM_LEVELS_M upper bound supported by the kernels

// ----------------------------------------------------------------------------
// geometry / covariance model (read-only per evaluation)
// ----------------------------------------------------------------------------
struct Geom {
    int nonstat;        // NONSTATIONARY_FLAG
    int distance;       // 0 chordal xyz, 1 great circle lon/lat degrees, 2 planar xy
    int nu_x2;          // 1: exponential, 3: Matern 3/2
    int pref_kind;      // 0: (x)^1.5, 1: (x)^1, 2: pow(x, pref_exp)
    double pref_exp;
    double dist_scale;
};

struct Pt {
    double c0, c1, c2;
};

__device__ __forceinline__ double point_distance(const Geom& g, const Pt& a, const Pt& b) {
    if (g.distance == 1) {
        // great_circle_dist, evaluate_covariance.cpp:9-25
        const double k = 3.14159265358979323846 / 180.0;
        double lon1 = a.c0 * k, lon2 = b.c0 * k, lat1 = a.c1 * k, lat2 = b.c1 * k;
        double ang = sin(lat1) * sin(lat2) + cos(lat1) * cos(lat2) * cos(lon1 - lon2);
        ang = ang > 1.0 ? 1.0 : (ang < -1.0 ? -1.0 : ang);
        return acos(ang);
    }
    // euclidean_distance, evaluate_covariance.cpp:28-37 (z = 0 for planar points)
    double dx = b.c0 - a.c0, dy = b.c1 - a.c1, dz = b.c2 - a.c2;
    return sqrt(dx * dx + dy * dy + dz * dz);
}

__device__ __forceinline__ double matern(int nu_x2, double h) {
    if (nu_x2 == 3) {
        double s = 1.7320508075688772 * h;
        return (1.0 + s) * exp(-s);
    }
    return exp(-h);
}

// C(s1, s2) with per-point sigma^2 (s) and beta (b): evaluate_covariance.cpp:218-225
// (nonstationary) and :82 (stationary: s1 = sill, b1 = range).
__device__ __forceinline__ double cov_entry(const Geom& g, const Pt& p1, double s1, double b1, const Pt& p2,
                                            double s2, double b2) {
    double D = g.dist_scale * point_distance(g, p1, p2);
    if (!g.nonstat) return s1 * matern(g.nu_x2, D / b1);
    double bms = (b1 * b1 + b2 * b2) / 2;
    double x = (b1 * b2) / bms;
    double pre = g.pref_kind == 0 ? x * sqrt(x) : (g.pref_kind == 1 ? x : pow(x, g.pref_exp));
    double c = sqrt(s1 * s2) * pre;
    return c * matern(g.nu_x2, D / sqrt(bms));
}

// A point set laid out SoA: coordinates c0/c1/c2 and fields s2 (sigma^2),
// beta, t2 (tau^2), all indexed by the same global point index.
struct PointSet {
    const double* c0;
    const double* c1;
    const double* c2;
    const double* s2;
    const double* beta;
    const double* t2;
    __device__ __forceinline__ Pt pt(long i) const { return Pt{c0[i], c1[i], c2[i]}; }
};

// out[t + q*ld] = C(A_{a0+t}, B_{b0+q}), t < na, q < nb.  When `self` the
// diagonal (t == q) is sigma^2 + tau^2 (evaluate_covariance.cpp:103,307).
__device__ inline void fill_cov(const Geom& g, const PointSet& P, long a0, int na, long b0, int nb, bool self,
                                double* out, long ld) {
    for (int e = threadIdx.x; e < na * nb; e += blockDim.x) {
        int t = e % na, q = e / na;
        long ia = a0 + t, ib = b0 + q;
        double v;
        if (self && t == q) {
            v = P.s2[ia] + P.t2[ia];
        } else {
            v = cov_entry(g, P.pt(ia), P.s2[ia], P.beta[ia], P.pt(ib), P.s2[ib], P.beta[ib]);
        }
        out[t + (long)q * ld] = v;
    }
}

// ----------------------------------------------------------------------------
// CTA-cooperative FP64 dense linear algebra (column-major)
// ----------------------------------------------------------------------------
constexpr int TM = 64, TN = 64, TK = 16, NB = 32;

struct LaSmem {
    double A[TK][TM + 1];
    double B[TK][TN + 1];
    double D[NB][NB + 1];  // staged diagonal block for the triangular kernels
    double red[kThreads / 32];
    int flag;
};

// C = alpha * op(A) * op(B) + beta * C; op(A): M x K, op(B): K x N.
// beta == 0 never reads C.  Ends with a barrier.
template <bool TA, bool TB>
__device__ inline void gemm(int M, int N, int K, double alpha, const double* A, long lda, const double* B, long ldb,
                     double beta, double* C, long ldc, LaSmem& sm) {
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    for (int m0 = 0; m0 < M; m0 += TM) {
        for (int n0 = 0; n0 < N; n0 += TN) {
            double acc[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
            for (int k0 = 0; k0 < K; k0 += TK) {
#pragma unroll
                for (int e = tid; e < TK * TM; e += kThreads) {
                    int i, k;
                    if (!TA) { i = e % TM; k = e / TM; } else { k = e % TK; i = e / TK; }
                    int gi = m0 + i, gk = k0 + k;
                    double v = 0.0;
                    if (gi < M && gk < K) v = TA ? A[gk + (long)gi * lda] : A[gi + (long)gk * lda];
                    sm.A[k][i] = v;
                }
#pragma unroll
                for (int e = tid; e < TK * TN; e += kThreads) {
                    int j, k;
                    if (!TB) { k = e % TK; j = e / TK; } else { j = e % TN; k = e / TN; }
                    int gj = n0 + j, gk = k0 + k;
                    double v = 0.0;
                    if (gj < N && gk < K) v = TB ? B[gj + (long)gk * ldb] : B[gk + (long)gj * ldb];
                    sm.B[k][j] = v;
                }
                __syncthreads();
#pragma unroll
                for (int kk = 0; kk < TK; ++kk) {
                    double a[4], b[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) a[q] = sm.A[kk][tx + 16 * q];
#pragma unroll
                    for (int q = 0; q < 4; ++q) b[q] = sm.B[kk][ty + 16 * q];
#pragma unroll
                    for (int x = 0; x < 4; ++x)
#pragma unroll
                        for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
                }
                __syncthreads();
            }
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                int gi = m0 + tx + 16 * x;
                if (gi >= M) continue;
#pragma unroll
                for (int y = 0; y < 4; ++y) {
                    int gj = n0 + ty + 16 * y;
                    if (gj >= N) continue;
                    double* c = C + gi + (long)gj * ldc;
                    *c = beta == 0.0 ? alpha * acc[x][y] : fma(alpha, acc[x][y], beta * *c);
                }
            }
        }
    }
    __syncthreads();
}

// B <- L^{-1} B  (L: n x n lower, non-unit; B: n x nrhs).  dtrtrs('L','N','N').
__device__ inline void trsm_left_lower(int n, int nrhs, const double* L, long ldl, double* B, long ldb, LaSmem& sm) {
    const int tid = threadIdx.x;
    for (int b0 = 0; b0 < n; b0 += NB) {
        int nb = min(NB, n - b0);
        for (int e = tid; e < nb * nb; e += kThreads) {
            int i = e % nb, j = e / nb;
            sm.D[i][j] = L[(b0 + i) + (long)(b0 + j) * ldl];
        }
        __syncthreads();
        for (int c = tid; c < nrhs; c += kThreads) {
            double x[NB];
            double* col = B + b0 + (long)c * ldb;
#pragma unroll
            for (int i = 0; i < NB; ++i) x[i] = i < nb ? col[i] : 0.0;
#pragma unroll
            for (int i = 0; i < NB; ++i) {
                if (i < nb) {
                    double s = x[i];
#pragma unroll
                    for (int k = 0; k < i; ++k) s -= sm.D[i][k] * x[k];
                    x[i] = s / sm.D[i][i];
                }
            }
#pragma unroll
            for (int i = 0; i < NB; ++i)
                if (i < nb) col[i] = x[i];
        }
        __syncthreads();
        if (b0 + nb < n)
            gemm<false, false>(n - b0 - nb, nrhs, nb, -1.0, L + (b0 + nb) + (long)b0 * ldl, ldl, B + b0, ldb, 1.0,
                               B + b0 + nb, ldb, sm);
    }
}

// B <- B L^{-T}  (L: n x n lower; B: rows x n).  Row-wise forward substitution.
__device__ inline void trsm_right_lower_trans(int rows, int n, const double* L, long ldl, double* B, long ldb,
                                       LaSmem& sm) {
    const int tid = threadIdx.x;
    for (int b0 = 0; b0 < n; b0 += NB) {
        int nb = min(NB, n - b0);
        for (int e = tid; e < nb * nb; e += kThreads) {
            int i = e % nb, j = e / nb;
            sm.D[i][j] = L[(b0 + i) + (long)(b0 + j) * ldl];
        }
        __syncthreads();
        for (int row = tid; row < rows; row += kThreads) {
            double x[NB];
            double* p = B + row + (long)b0 * ldb;
#pragma unroll
            for (int i = 0; i < NB; ++i) x[i] = i < nb ? p[(long)i * ldb] : 0.0;
#pragma unroll
            for (int i = 0; i < NB; ++i) {
                if (i < nb) {
                    double s = x[i];
#pragma unroll
                    for (int k = 0; k < i; ++k) s -= sm.D[i][k] * x[k];
                    x[i] = s / sm.D[i][i];
                }
            }
#pragma unroll
            for (int i = 0; i < NB; ++i)
                if (i < nb) p[(long)i * ldb] = x[i];
        }
        __syncthreads();
        if (b0 + nb < n)
            gemm<false, true>(rows, n - b0 - nb, nb, -1.0, B + (long)b0 * ldb, ldb, L + (b0 + nb) + (long)b0 * ldl,
                              ldl, 1.0, B + (long)(b0 + nb) * ldb, ldb, sm);
    }
}

// In-place lower Cholesky A = L L^T (strict upper part zeroed, like
// Armadillo's chol(X, "lower")).  Returns 0, or the 1-based index of the
// first non-positive pivot (LAPACK dpotrf's info); the factorization then
// continues on NaNs and the caller reports the region.
__device__ inline int potrf_lower(int n, double* A, long lda, LaSmem& sm) {
    const int tid = threadIdx.x;
    if (tid == 0) sm.flag = 0;
    for (int b0 = 0; b0 < n; b0 += NB) {
        int nb = min(NB, n - b0);
        for (int e = tid; e < nb * nb; e += kThreads) {
            int i = e % nb, j = e / nb;
            sm.D[i][j] = A[(b0 + i) + (long)(b0 + j) * lda];
        }
        __syncthreads();
        for (int k = 0; k < nb; ++k) {
            if (tid == 0) {
                double d = sm.D[k][k];
                if (!(d > 0.0) && sm.flag == 0) sm.flag = b0 + k + 1;
                sm.D[k][k] = sqrt(d);
            }
            __syncthreads();
            double dk = sm.D[k][k];
            for (int i = k + 1 + tid; i < nb; i += kThreads) sm.D[i][k] /= dk;
            __syncthreads();
            int rem = nb - k - 1;
            for (int e = tid; e < rem * rem; e += kThreads) {
                int i = k + 1 + e % rem, j = k + 1 + e / rem;
                if (j <= i) sm.D[i][j] -= sm.D[i][k] * sm.D[j][k];
            }
            __syncthreads();
        }
        for (int e = tid; e < nb * nb; e += kThreads) {
            int i = e % nb, j = e / nb;
            A[(b0 + i) + (long)(b0 + j) * lda] = j <= i ? sm.D[i][j] : 0.0;
        }
        __syncthreads();
        int rest = n - b0 - nb;
        if (rest > 0) {
            // panel: A[b0+nb:, b0:b0+nb] <- A[...] * D^{-T}
            for (int row = tid; row < rest; row += kThreads) {
                double x[NB];
                double* p = A + (b0 + nb + row) + (long)b0 * lda;
#pragma unroll
                for (int i = 0; i < NB; ++i) x[i] = i < nb ? p[(long)i * lda] : 0.0;
#pragma unroll
                for (int i = 0; i < NB; ++i) {
                    if (i < nb) {
                        double s = x[i];
#pragma unroll
                        for (int k = 0; k < i; ++k) s -= sm.D[i][k] * x[k];
                        x[i] = s / sm.D[i][i];
                    }
                }
#pragma unroll
                for (int i = 0; i < NB; ++i)
                    if (i < nb) p[(long)i * lda] = x[i];
            }
            __syncthreads();
            const double* P = A + (b0 + nb) + (long)b0 * lda;
            gemm<false, true>(rest, rest, nb, -1.0, P, lda, P, lda, 1.0, A + (b0 + nb) + (long)(b0 + nb) * lda, lda,
                              sm);
            // the strict upper part of the trailing block is scratch; zero it
            for (int e = tid; e < nb * rest; e += kThreads) {
                int i = e % nb, j = e / nb;
                A[(b0 + i) + (long)(b0 + nb + j) * lda] = 0.0;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    return sm.flag;
}

// Deterministic CTA sum (fixed thread -> element mapping and tree order).
__device__ inline double cta_sum(double v, LaSmem& sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm.red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w) s += sm.red[w];
    __syncthreads();
    return s;  // valid in thread 0
}

}  // namespace mra
