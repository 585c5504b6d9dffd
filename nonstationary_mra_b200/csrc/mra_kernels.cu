// Region kernels of the MRA hot path, templated on the storage type T
// (double: plain FP64 path; float: mixed path, FP32 storage and 3xTF32 tensor
// products, FP64 diagonal blocks and log-likelihood accumulation).
//
// Schedule of one log-likelihood (one launch per stage and tree level):
//   k_fields            sigma^2/beta/tau^2 at every knot, observation and
//                       prediction point (class_nonstationary_covariance.cpp:479-573)
//   k_prior_level(m)    levels 0..M-2, one CTA per region: U_{i,j} = L_{a_j}^{-1} V_j,
//                       L_i = chol(K_i)   (class_approximation.cpp:46-50,84-169)
//   k_finest_group      one CTA per level M-3 region: conditioning of all its
//                       observations on the shared ancestors (levels 0..M-3),
//                       then per level M-2 child (a sibling group of finest
//                       regions) the level M-2 step and per finest region
//                       Sigma, L_Sigma, y~,
//                       B^ and the log-lik terms
//                       (...-loop-regions-at-finest-level-in-prior.cpp:90-269),
//                       then the level M-2 posterior of the parent
//   k_posterior_level(m) levels M-3..0 (...-posterior-inference.cpp:14-265,
//                       class_approximation.cpp:186-306)
//   k_reduce            deterministic sum of the per-region terms
//   k_predict           prediction, one CTA per level M-2 region (its finest
//                       children's predictions together)
//                       (...-prior.cpp:271-392, class_approximation-predict.cpp:105-189)
//
// Posterior representation.  A region's contribution to its parent is the pair
// (A~, w~) of the reference (class_approximation.cpp:266-306).  Below a size
// threshold it is carried in factored observation-space form instead: a matrix
// F (n x m r, one row per observation of the subtree) and a vector f with
// A~_(j,k) = F_j^T F_k and w~_j = F_j^T f.  The finest level starts in this
// form (F = B^, f = y~).  For a region i at level m with factored input (F, f):
//   Y = L_i^{-1} F_m^T,  R R^T = I + Y^T Y,
//   output F' = R^{-1} F_{0..m-1},  f' = R^{-1} f,
//   log-lik term 2 log|R| - (f^T f - f'^T f'),
// which equals the reference's -2 log|L_i| + 2 log|L~_i| - v^T v with
// L~ L~^T = L L^T + F_m^T F_m (Sylvester's determinant identity and Woodbury),
// and F'^T F' / F'^T f' equal the reference's A~ / w~ of the region.  Larger
// regions use the reference's dense r x r slices.  Prediction mode also forms
// L~, v and G of factored regions from (F, f).
#include "mra_kernels.cuh"

namespace mra {

__device__ inline void report_error(int* err, long region) {
    if (atomicCAS(&err[0], 0, 4 /* MRA_ERR_NOT_SPD */) == 0) {
        err[1] = (int)(region & 0x7fffffff);
        err[2] = (int)(region >> 31);
    }
}

// ---------------------------------------------------------------------------
// a1: fields
// ---------------------------------------------------------------------------
__global__ void k_fields(Geom g, FieldParams fp, const double* __restrict__ c0, const double* __restrict__ c1,
                         const double* __restrict__ c2, long n, double* __restrict__ s2, double* __restrict__ beta,
                         double* __restrict__ t2) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* th = fp.theta;
    if (!g.nonstat) {
        s2[i] = th[6];
        beta[i] = th[7];
        t2[i] = th[8];
        return;
    }
    Pt p{c0[i], c1[i], c2[i]};
    double out[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        double v = th[3 + f];
        const long nb = fp.nb[f];
        const double* c = fp.centers[f];
        const double* w = fp.weights[f];
        for (long b = 0; b < nb; ++b) {
            Pt q{c[b], c[nb + b], c[2 * nb + b]};
            double d = point_distance(g, p, q) / fp.basis_len;
            if (fp.basis == 0) {
                if (d >= 1) continue;
                double u = 1 - d, u2 = u * u;
                v += u2 * u2 * u2 * (35 * d * d + 18 * d + 3) * w[b] / 3;
            } else {
                v += exp(-0.5 * d * d) * w[b];
            }
        }
        out[f] = th[f] * exp(v);
    }
    s2[i] = out[0];
    beta[i] = out[1];
    t2[i] = out[2];
}

// ---------------------------------------------------------------------------
// a2/a3 for the prior: the covariance blocks of one level, in their own launch
// ---------------------------------------------------------------------------
// Regions loc0 .. loc0+nloc-1 (local indices) of level m: block j < m of region
// i is C(Q_{a_j}, Q_i) (rows: the knots of ancestor a_j, columns: the region's
// own knots; evaluate_nonstationary_cross_covariance, evaluate_covariance.cpp:
// 155-234), block m is C(Q_i, Q_i) with sigma^2 + tau^2 on its diagonal
// (:248-313).  Block j of the q-th region goes to out + (q (m+1) + j) r^2,
// column-major with ld r.  One CTA per block at a time; with no barrier-bound
// products beside it the launch keeps every SM full of independent entry
// chains, which the per-region kernel, two CTAs per SM between its products,
// cannot.
constexpr int kCovThreads = 256;
constexpr int kCovChunk = 64;  // column points staged per chunk (7 x 64 doubles of shared memory)

// The straight-line nonstationary FP64 block: one row point per thread with its
// parameters in registers, the column points staged in chunks, entries of
// cov_fast_entry (the same arithmetic as fill_row_fast).
template <typename T, int NU, int PREF>
__device__ __forceinline__ void cov_block_fast(const PointSet& P, long a0, int nr, long b0, int nc, bool self,
                                               T* __restrict__ out, long ld, double ih2, double ihs2,
                                               double* stage) {
    double* sx = stage;
    double* sy = sx + kCovChunk;
    double* sz = sy + kCovChunk;
    double* sg = sz + kCovChunk;
    double* s4 = sg + kCovChunk;  // sqrt(s2) b (PREF 1) or sqrt(s2) (PREF 0)
    double* s5 = s4 + kCovChunk;  // b (PREF 0)
    const int tid = threadIdx.x, nt = blockDim.x;
    const int rows = nr < nt ? nr : nt;
    const int cols = nt / rows;
    const bool worker = tid < rows * cols;
    const int tr = tid % rows, tc = tid / rows;
    for (int q0 = 0; q0 < nc; q0 += kCovChunk) {
        const int qn = nc - q0 < kCovChunk ? nc - q0 : kCovChunk;
        __syncthreads();
        for (int e = tid; e < qn; e += nt) {
            const long ib = b0 + q0 + e;
            const double bb = P.beta[ib], ssq = sqrt(P.s2[ib]);
            sx[e] = P.c0[ib];
            sy[e] = P.c1[ib];
            sz[e] = P.c2[ib];
            sg[e] = bb * bb * ih2;
            s4[e] = PREF == 1 ? ssq * bb : ssq;
            s5[e] = bb;
        }
        __syncthreads();
        if (!worker) continue;
        for (int t = tr; t < nr; t += rows) {
            const long ia = a0 + t;
            const double pc0 = P.c0[ia], pc1 = P.c1[ia], pc2 = P.c2[ia], sa = P.s2[ia], ba = P.beta[ia];
            const double ssa = sqrt(sa), ga = ba * ba * ih2, ca = ssa * ba * ihs2, ba_h = ba * ihs2;
            const double diag = self ? sa + P.t2[ia] : 0.0;
            T* ob = out + t;
#pragma unroll 4
            for (int q = tc; q < qn; q += cols) {
                const int qq = q0 + q;
                double v = cov_fast_entry<NU, PREF, true>(pc0, pc1, pc2, ga, ca, ssa, ba_h, sx[q], sy[q], sz[q], sg[q],
                                                    PREF == 1 ? s4[q] : 0.0, PREF == 1 ? 0.0 : s4[q],
                                                    PREF == 1 ? 0.0 : s5[q]);
                if (self && t == qq) v = diag;  // sigma^2 + tau^2 (evaluate_covariance.cpp:103,307)
                ob[(long)qq * ld] = (T)v;
            }
        }
    }
    __syncthreads();
}

// Block out[t + q ld] = C(A_{a0+t}, B_{b0+q}), t < nr, q < nc (with the
// sigma^2 + tau^2 diagonal when `self`), by the whole CTA.  KIND (cov_kind on the
// host): 1..4 the straight-line nonstationary FP64 forms (Matern 3/2 or 1/2 x
// prefactor exponent 1 or 3/2), 0 every other model.
template <typename T, int KIND>
__device__ __forceinline__ void cov_block(const Geom& g, const PointSet& P, long a0, int nr, long b0, int nc, bool self,
                                          T* out, long ld, double* stage) {
    if constexpr (KIND == 0) {
        fill_cov_staged<T, kCovChunk>(g, P, &a0, 1, nr, b0, nc, self, out, ld, 0, stage);
    } else {
        const double hs = g.dist_scale * (KIND <= 2 ? 1.7320508075688772 : 1.0);
        const double ihs2 = 1.0 / (hs * hs), ih2 = 0.5 * ihs2;
        constexpr int NU = KIND <= 2 ? 3 : 1, PREF = (KIND & 1) ? 1 : 0;
        cov_block_fast<T, NU, PREF>(P, a0, nr, b0, nc, self, out, ld, ih2, ihs2, stage);
    }
}

inline int cov_kind(const Geom& g, bool fp64) {
    if (!(fp64 && g.nonstat && g.distance != 1 && g.pref_kind != 2)) return 0;
    return g.nu_x2 == 3 ? (g.pref_kind == 1 ? 1 : 2) : (g.pref_kind == 1 ? 3 : 4);
}

template <typename T, int KIND>
__global__ void __launch_bounds__(kCovThreads, 4) k_cov_level(Geom g, DevTree<T> t, int m, long loc0, long nloc,
                                                               T* __restrict__ out) {
    __shared__ double stage[7 * kCovChunk];
    const int r = t.r;
    const long rr = (long)r * r;
    const long s0 = level_start(t.J, m);
    const long nblocks = nloc * (m + 1);
    for (long b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const long q = b / (m + 1);
        const int j = (int)(b - q * (m + 1));
        const long i = s0 + loc0 + q;
        if (skipped(t, i)) continue;
        long a = i;  // the ancestor of level j (the region itself for j == m)
        for (int l = m; l > j; --l) a = (a - 1) / t.J;
        cov_block<T, KIND>(g, t.pts, a * r, r, i * r, r, j == m, out + b * rr, r, stage);
    }
}

// Host-side dispatch of the covariance-block launches on the model's form.
template <typename T>
void launch_cov_level(const Geom& g, const DevTree<T>& t, int m, long loc0, long n, unsigned grid, cudaStream_t st) {
    switch (cov_kind(g, sizeof(T) == 8)) {
        case 1: k_cov_level<T, 1><<<grid, kCovThreads, 0, st>>>(g, t, m, loc0, n, t.cbuf); break;
        case 2: k_cov_level<T, 2><<<grid, kCovThreads, 0, st>>>(g, t, m, loc0, n, t.cbuf); break;
        case 3: k_cov_level<T, 3><<<grid, kCovThreads, 0, st>>>(g, t, m, loc0, n, t.cbuf); break;
        case 4: k_cov_level<T, 4><<<grid, kCovThreads, 0, st>>>(g, t, m, loc0, n, t.cbuf); break;
        default: k_cov_level<T, 0><<<grid, kCovThreads, 0, st>>>(g, t, m, loc0, n, t.cbuf); break;
    }
}

// ---------------------------------------------------------------------------
// a5/a6: prior, one level of interior regions
// ---------------------------------------------------------------------------
// One CTA per region.  The inverse L_a^{-1} of every prior factor is formed
// once, right after its Cholesky, so that the m triangular solves of each
// descendant become tensor-pipe products.  The covariance blocks come from
// k_cov_level (C: the q-th region's m+1 blocks at C + q (m+1) r^2); each
// conditioning product takes its block as the added term, so nothing is
// copied: V_j = C_j - U_{a_j}^T U_{i,0..j-1}, U_{i,j} = L_{a_j}^{-1} V_j and
// K_i = C_i - U_i^T U_i straight into the factor's storage.
template <typename T>
__global__ void __launch_bounds__(kThreads, 2) k_prior_level(Geom g, DevTree<T> t, int m, long loc0, long nloc,
                                                            const T* __restrict__ C) {
    LaSmem<T>& sm = la_smem<T>();
    const int r = t.r;
    const long rr = (long)r * r;
    const long s0 = level_start(t.J, m);
    const long mr = (long)m * r;
    for (long q = blockIdx.x; q < nloc; q += gridDim.x) {
        const long loc = loc0 + q;
        const long i = s0 + loc;
        if (skipped(t, i)) continue;
        long anc[kMaxLevels];
        {
            long c = i;
            for (int a = m - 1; a >= 0; --a) {
                c = (c - 1) / t.J;
                anc[a] = c;
            }
        }
        const T* Cq = C + q * (long)(m + 1) * rr;
        T* Ui = t.U + t.u_off[m] + loc * mr * r;  // (m r) x r, ld = m r
        // one r x r scratch per CTA (stays in L2)
        T* V = t.ws + blockIdx.x * t.ws_stride;
        for (int j = 0; j < m; ++j) {
            const long a = anc[j];
            const T* Cj = Cq + j * rr;
            const T* Vj = Cj;  // level 0 has nothing to condition on
            // the next covariance block (or the self block) into L2 while this step's products run
            if (threadIdx.x == 0) prefetch_l2(Cj + rr, rr * sizeof(T));
            if (j > 0) {
                const T* Ua = t.U + t.u_off[j] + (a - level_start(t.J, j)) * (long)j * rr;
                gemm_wide<T, true, false>(r, r, j * r, (T)-1, Ua, (long)j * r, Ui, mr, (T)1, V, r, sm, Cj, r);
                Vj = V;
            }
            // U_{i,j} = L_a^{-1} V as a product with the stored inverse
            gemm<T, false, false>(r, r, r, (T)1, t.Pinv + a * rr, r, Vj, r, (T)0, Ui + (long)j * r, mr, sm);
        }
        T* Li = t.Lprior + i * rr;
        // K_i = C_i - U_i^T U_i (for m == 0 a product with K = 0: the copy of C_i)
        gemm<T, true, false>(r, r, (int)mr, (T)-1, Ui, mr, Ui, mr, (T)1, Li, r, sm, Cq + (long)m * rr, r);
        double ld = 0.0;
        int info = potrf_lower<T>(r, Li, r, sm, &ld, t.Pinv + i * rr, r);
        if (threadIdx.x == 0) {
            t.ldprior[i] = ld;
            if (info) report_error(t.err, i);
        }
    }
}

// ---------------------------------------------------------------------------
// posterior steps of one region (level m): factored and dense forms
// ---------------------------------------------------------------------------
// The products of the posterior steps go through a separate function: the
// steps keep many values live across their products, and inlined there the
// product loops would share (and spill) their registers.  (The finest-level
// kernel measured faster with its products inlined.)
template <typename T, bool TA, bool TB, bool ONE_TILE = false>
__device__ __noinline__ void gemm_call(int M, int N, int K, T alpha, const T* A, long lda, const T* B, long ldb,
                                       T beta, T* C, long ldc, LaSmem<T>& sm, const T* Cin = nullptr,
                                       long ldcin = 0) {
    gemm<T, TA, TB, ONE_TILE>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, sm, Cin, ldcin);
}

// Factored input (F: n rows of width (m+1) r, row stride ldF; f: n doubles).
// Writes F' (n rows of width m r) to Fo and f' to fo when m > 0.
template <typename T>
__device__ __noinline__ void factored_step(const DevTree<T>& t, int m, long i, int n, const T* F, long ldF, const double* f, T* Fo,
                              double* fo, bool keep, T* ws, double* wsd, LaSmem<T>& sm, double& dterm) {
    const int r = t.r;
    const long rr = (long)r * r, mr = (long)m * r;
    const T* Li = t.Lprior + i * rr;
    T* Y = ws;                  // r x n
    T* S = ws + (long)r * n;    // n x n
    T* Rinv = S + (long)n * n;  // n x n (n <= 128)
    // Y = L_i^{-1} F_m^T as a product with the stored inverse of the prior factor
    gemm_call<T, false, false>(r, n, r, (T)1, t.Pinv + i * rr, r, F + mr, ldF, (T)0, Y, r, sm);
    gemm_call<T, true, false>(n, n, r, (T)1, Y, r, Y, r, (T)0, S, n, sm);
    for (int q = threadIdx.x; q < n; q += kThreads) S[q + (long)q * n] += (T)1;
    __syncthreads();
    double ld = 0.0;
    const bool small = sizeof(T) == 8 && n <= 128;
    int info = potrf_lower<T>(n, S, n, sm, &ld, small ? Rinv : nullptr, n);
    double* fp = m > 0 ? fo : wsd;
    double part = 0.0;
    for (int q = threadIdx.x; q < n; q += kThreads) {
        fp[q] = f[q];
        part += f[q] * f[q];
    }
    double ff = cta_sum(part, sm);
    if (small) trmv_lower_inv<T>(n, Rinv, n, fp, fp);  // f' = R^{-1} f with the inverse formed above
    else trsv_lower_f64<T>(n, S, n, fp);
    part = 0.0;
    for (int q = threadIdx.x; q < n; q += kThreads) part += fp[q] * fp[q];
    double pp = cta_sum(part, sm);
    if (threadIdx.x == 0) {
        dterm += ld - (ff - pp);
        if (info) report_error(t.err, i);
    }
    if (m > 0) {
        if (small) {
            // F' = F_{0..m-1} R^{-T}
            gemm_call<T, false, true>((int)mr, n, n, (T)1, F, ldF, Rinv, n, (T)0, Fo, mr, sm);
        } else {
            for (long e = threadIdx.x; e < mr * n; e += kThreads) {
                long x = e % mr, q = e / mr;
                Fo[q * mr + x] = F[q * ldF + x];
            }
            __syncthreads();
            trsm_right_lower_trans<T>((int)mr, n, S, n, Fo, mr, sm);
        }
    }
    if (keep) {
        // predictive factors of the region: L~ L~^T = L L^T + F_m^T F_m, v = L~^{-1} F_m^T f,
        // G = L~^{-1} F_m^T F_{0..m-1}
        T* Lt = t.Lpost + i * rr;
        gemm_call<T, false, true>(r, r, r, (T)1, Li, r, Li, r, (T)0, Lt, r, sm);
        gemm_call<T, false, true>(r, r, n, (T)1, F + mr, ldF, F + mr, ldF, (T)1, Lt, r, sm);
        T* Lti = t.Lpinv ? t.Lpinv + i * rr : nullptr;  // L~^{-1}, kept for prediction
        int info2 = potrf_lower<T>(r, Lt, r, sm, nullptr, Lti, r);
        double* v = t.vpost + i * r;
        for (int tt = threadIdx.x; tt < r; tt += kThreads) {
            double s = 0.0;
            for (int q = 0; q < n; ++q) s += (double)F[(long)q * ldF + mr + tt] * f[q];
            v[tt] = s;
        }
        __syncthreads();
        if (Lti) trmv_lower_inv<T>(r, Lti, r, v, v);
        else trsv_lower_f64<T>(r, Lt, r, v);
        if (m > 0) {
            T* Gi = t.G + t.u_off[m] + (i - level_start(t.J, m)) * mr * r;
            gemm_call<T, false, true>(r, (int)mr, n, (T)1, F + mr, ldF, F, ldF, (T)0, Gi, r, sm);
            // G = L~^{-1} G in place: one row tile (r <= 64) reads all of its
            // column block before writing it
            if (Lti) gemm_call<T, false, false>(r, (int)mr, r, (T)1, Lti, r, Gi, r, (T)0, Gi, r, sm);
            else trsm_left_lower<T>(r, (int)mr, Lt, r, Gi, r, sm);
        }
        if (info2 && threadIdx.x == 0) report_error(t.err, i);
    }
}

// Dense input: Aagg holds the slices (j,k), j <= k <= m, of the summed children
// contributions, wagg the (m+1) x r summed w.
template <typename T>
__device__ __noinline__ void dense_step(const DevTree<T>& t, int m, long i, const T* Aagg, const double* wagg, bool keep, T* Gw,
                           LaSmem<T>& sm, double& dterm) {
    const int r = t.r;
    const long rr = (long)r * r, mr = (long)m * r;
    const long loc = i - level_start(t.J, m);
    const T* Lp = t.Lprior + i * rr;
    T* Lt = t.Lpost + i * rr;
    gemm_call<T, false, true>(r, r, r, (T)1, Lp, r, Lp, r, (T)0, Lt, r, sm);
    const T* Amm = Aagg + slice_index(m + 1, m, m) * rr;
    for (long e = threadIdx.x; e < rr; e += kThreads) Lt[e] += Amm[e];
    __syncthreads();
    double ld = 0.0;
    // L~^{-1}: kept for prediction when that is on, else an r x r scratch after the G scratch
    const bool kept = keep && t.Lpinv;
    T* Ltinv = kept ? t.Lpinv + i * rr : Gw + mr * r;
    const bool small = sizeof(T) == 8 && r <= 64 && (m > 0 || kept);
    int info = potrf_lower<T>(r, Lt, r, sm, &ld, small ? Ltinv : nullptr, r);
    double* v = t.vpost + i * r;
    for (int e = threadIdx.x; e < r; e += kThreads) v[e] = wagg[mr + e];
    __syncthreads();
    if (small) trmv_lower_inv<T>(r, Ltinv, r, v, v);  // v = L~^{-1} w_m with the inverse formed above
    else trsv_lower_f64<T>(r, Lt, r, v);
    double part = 0.0;
    for (int e = threadIdx.x; e < r; e += kThreads) part += v[e] * v[e];
    double vv = cta_sum(part, sm);
    if (threadIdx.x == 0) {
        dterm += ld - t.ldprior[i] - vv;
        if (info) report_error(t.err, i);
    }
    if (m == 0) return;
    T* Gi = keep ? t.G + t.u_off[m] + loc * mr * r : Gw;  // r x (m r), ld = r
    if (small) {
        // G_j = L~^{-1} A_(j,m)^T
        for (int j = 0; j < m; ++j)
            gemm_call<T, false, true>(r, r, r, (T)1, Ltinv, r, Aagg + slice_index(m + 1, j, m) * rr, r, (T)0,
                                 Gi + (long)j * rr, r, sm);
    } else {
        for (long e = threadIdx.x; e < mr * r; e += kThreads) {
            int j = (int)(e / rr);
            long w = e % rr;
            int p = (int)(w % r), q = (int)(w / r);
            Gi[e] = Aagg[slice_index(m + 1, j, m) * rr + q + (long)p * r];  // G_j = A_(j,m)^T
        }
        __syncthreads();
        trsm_left_lower<T>(r, (int)mr, Lt, r, Gi, r, sm);
    }
    const long slot = t.dslot[i];  // compact index among the level's dense regions
    double* wo = t.wout[m & 1] + slot * mr;
    for (long x = threadIdx.x; x < mr; x += kThreads) {
        double s = 0.0;
        for (int tt = 0; tt < r; ++tt) s += (double)Gi[tt + x * r] * v[tt];
        wo[x] = wagg[x] - s;
    }
    // A_out(j, j..m-1) = A(j, j..m-1) - G_j^T G_{j..m-1}: both slice rows are
    // contiguous r x r blocks, one product per j reading A from Aagg
    T* ao = t.aout[m & 1] + slot * n_slices(m) * rr;
    for (int j = 0; j < m; ++j) {
        T* dst = ao + slice_index(m, j, j) * rr;
        const T* src = Aagg + slice_index(m + 1, j, j) * rr;
        gemm_call<T, true, false>(r, (m - j) * r, r, (T)-1, Gi + (long)j * rr, r, Gi + (long)j * rr, r, (T)1, dst, r,
                                  sm, src, r);
    }
}

// Aagg/wagg += the (A~, w~) of factored rows F (n x (m+1) r, row stride ldF), f;
// with `init` they are set instead (the first contribution: no zeroing pass).
// The slices (j, j..m) of A~ are contiguous r x r blocks, so block row j is
// one product F_j^T F_{j..m} (r x (m+1-j) r).
template <typename T>
__device__ __noinline__ void accumulate_factored(const DevTree<T>& t, int m, int n, const T* F, long ldF, const double* f, T* Aagg,
                                    double* wagg, bool init, LaSmem<T>& sm) {
    const int r = t.r;
    const long rr = (long)r * r, mr1 = (long)(m + 1) * r;
    if (n == 0) {
        if (init) {
            for (long e = threadIdx.x; e < n_slices(m + 1) * rr; e += kThreads) Aagg[e] = (T)0;
            for (long e = threadIdx.x; e < mr1; e += kThreads) wagg[e] = 0.0;
            __syncthreads();
        }
        return;
    }
    for (int j = 0; j <= m; ++j)
        gemm_call<T, false, true>(r, (m + 1 - j) * r, n, (T)1, F + (long)j * r, ldF, F + (long)j * r, ldF,
                                  init ? (T)0 : (T)1, Aagg + slice_index(m + 1, j, j) * rr, r, sm);
    for (long x = threadIdx.x; x < mr1; x += kThreads) {
        double s = 0.0;
        for (int q = 0; q < n; ++q) s += (double)F[(long)q * ldF + x] * f[q];
        wagg[x] = init ? s : wagg[x] + s;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// a7/a8: the finest children of one level M-2 region, all at once
// ---------------------------------------------------------------------------
// Used when every child has at most 32 observations and the group at most 64
// (T = double): one covariance block and one product form the whole group's
// conditional covariance, one warp per child factors its diagonal block,
// solves y~ and inverts its factor into a block-diagonal matrix, and one
// product forms the whole group's B^ (in place: each 64-row tile of the
// product reads exactly the rows it then writes, and the group fits one
// column tile).  Returns the group's log-likelihood terms (thread 0).
constexpr int kGroupMax = 64;
constexpr int kChildMax = 32;

template <typename T>
__device__ __noinline__ double finest_children_grouped(const Geom& g, const DevTree<T>& t, long clo, long chi,
                                                       long lo, int np, T* ws, LaSmem<T>& sm) {
    if constexpr (sizeof(T) != 8) {
        return 0.0;
    } else {
        const long Lr = (long)t.L * t.r;
        const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
        T* Sg = ws;                      // np x np conditional covariance of the group
        T* Binv = ws + (long)np * np;    // np x np block-diagonal L_Sigma^{-1}
        fill_cov<T>(g, t.pts, t.obs0 + lo, np, t.obs0 + lo, np, true, Sg, np, sm);
        for (int e = tid; e < np * np; e += kThreads) Binv[e] = 0.0;
        __syncthreads();
        gemm<T, true, false>(np, np, (int)Lr, (T)-1, t.Ufin + lo * Lr, Lr, t.Ufin + lo * Lr, Lr, (T)1, Sg, np, sm);
        constexpr int LD = kChildMax + 1;
        double* Sw = &sm.A[0][0] + w * (kChildMax * LD);  // per-warp 32 x 33 (A and B tiles are contiguous)
        double part = 0.0;
        const long c = clo + w;
        if (c < chi) {
            const long o0 = t.obs_off[c];
            const int n = (int)(t.obs_off[c + 1] - o0), q0 = (int)(o0 - lo);
            if (n > 0) {
                for (int e = lane; e < n * n; e += 32) {
                    const int i = e % n, j = e / n;
                    Sw[i + j * LD] = Sg[(q0 + i) + (long)(q0 + j) * np];
                }
                __syncwarp();
                int bad = 0;
                for (int k = 0; k < n; ++k) {  // lane i owns row i
                    const double d = Sw[k + k * LD];
                    __syncwarp();
                    if (!(d > 0.0)) bad = 1;
                    const double sq = sqrt(d);
                    if (lane == k) Sw[k + k * LD] = sq;
                    if (lane > k && lane < n) Sw[lane + k * LD] *= 1.0 / sq;
                    __syncwarp();
                    const double lik = lane < n ? Sw[lane + k * LD] : 0.0;
                    for (int j = k + 1; j < n; ++j)  // uniform trip count across the warp
                        if (lane >= j && lane < n) Sw[lane + j * LD] -= lik * Sw[j + k * LD];
                    __syncwarp();
                }
                T* Lc = t.Lsig + t.lsig_off[c];
                for (int e = lane; e < n * n; e += 32) {
                    const int i = e % n, j = e / n;
                    Lc[i + (long)j * n] = i >= j ? Sw[i + j * LD] : 0.0;
                }
                double ldp = lane < n ? log(Sw[lane + lane * LD]) : 0.0;
                for (int o = 16; o > 0; o >>= 1) ldp += __shfl_xor_sync(0xffffffffu, ldp, o);
                // y~ = L_Sigma^{-1} y: lane i ends holding x_i
                double xl = 0.0;
                for (int i = 0; i < n; ++i) {
                    double sp = lane < i ? Sw[i + lane * LD] * xl : 0.0;
                    for (int o = 16; o > 0; o >>= 1) sp += __shfl_xor_sync(0xffffffffu, sp, o);
                    if (lane == i) xl = (t.y[o0 + i] - sp) / Sw[i + i * LD];
                }
                if (lane < n) t.yt[o0 + lane] = xl;
                double yy = lane < n ? xl * xl : 0.0;
                for (int o = 16; o > 0; o >>= 1) yy += __shfl_xor_sync(0xffffffffu, yy, o);
                // column j of L_Sigma^{-1} by lane j, into the child's diagonal block
                {
                    // lanes walk the same rows and terms (X[k] = 0 above the
                    // diagonal): no divergence, broadcast reads of L
                    const int j = lane;
                    double xs[kChildMax];  // column j of the inverse, in registers
#pragma unroll
                    for (int i = 0; i < kChildMax; ++i) xs[i] = 0.0;
                    double* col = Binv + q0 + (long)(q0 + (j < n ? j : 0)) * np;
                    for (int i = 0; i < n; ++i) {
                        double v = 0.0;
#pragma unroll
                        for (int k = 0; k < kChildMax; ++k)
                            if (k < i) v += Sw[i + k * LD] * xs[k];
                        const double xi = i == j ? 1.0 / Sw[i + i * LD] : (i > j ? -v / Sw[i + i * LD] : 0.0);
#pragma unroll
                        for (int k = 0; k < kChildMax; ++k)
                            if (k == i) xs[k] = xi;
                        if (j < n && i >= j) col[i] = xi;
                    }
                }
                part = yy + 2.0 * ldp;
                if (bad && lane == 0) report_error(t.err, t.n_int + c);
            }
        }
        __syncthreads();
        if (lane == 0) sm.red[w] = part;
        __syncthreads();
        double tot = 0.0;
        if (tid == 0)
            for (int k = 0; k < kThreads / 32; ++k) tot += sm.red[k];
        __syncthreads();
        gemm<T, false, true, true>((int)Lr, np, np, (T)1, t.Bhat + lo * Lr, Lr, Binv, np, (T)0, t.Bhat + lo * Lr, Lr,
                                   sm);
        return tot;
    }
}

// ---------------------------------------------------------------------------
// a7/a8 (+ a9 at level M-2): finest level, one CTA per level M-3 region
// ---------------------------------------------------------------------------
// A work item is either a unit -- a level M-3 region with its J level M-2
// children (sibling groups), taken together when it holds few observations --
// or a single level M-2 group (large units are split for load balance; for
// M = 2 the single level-0 group).  The observations of an item are
// contiguous and all of them share the ancestors at levels 0..M-3: their
// conditioning on those levels runs once per item (for a unit: products J
// times wider, the ancestors' U read once).  The level M-2 step, the finest
// children and the level M-2 posterior then run per group.
template <typename T>
__global__ void __launch_bounds__(kThreads, 2) k_finest_group(Geom g, DevTree<T> t, int keep) {
    LaSmem<T>& sm = la_smem<T>();
    __shared__ long s_u;
    const int r = t.r, L = t.L, m = t.M - 2;
    const long rr = (long)r * r, Lr = (long)L * r;
    const long s2 = level_start(t.J, m);
    const long n_units = t.M >= 3 ? level_count(t.J, m - 1) : 0;
    T* ws = t.ws + blockIdx.x * t.ws_stride;
    double* wsd = t.wsd + blockIdx.x * t.wsd_stride;
    for (;;) {
        if (threadIdx.x == 0) {
            int q = atomicAdd(&t.queue[0], 1);
            s_u = q < t.n_fin_items ? t.par_order[q] : -1;
        }
        __syncthreads();
        const long item = s_u;
        __syncthreads();
        if (item < 0) break;
        // item < n_units: unit (level M-3 local index); else group item - n_units (level M-2 local index)
        const bool unit = item < n_units;
        const long g_lo = unit ? item * t.J : item - n_units, g_hi = unit ? g_lo + t.J : g_lo + 1;
        const long ui = unit ? level_start(t.J, m - 1) + item : s2 + g_lo;  // region whose subtree is the item
        if (skipped(t, ui)) continue;  // uniform: the item is the same for the whole CTA
        long anc[kMaxLevels];
        if (m > 0) {
            long c = unit ? ui : (ui - 1) / t.J;
            anc[m - 1] = c;
            for (int a = m - 2; a >= 0; --a) {
                c = (c - 1) / t.J;
                anc[a] = c;
            }
        }
        const long ulo = t.sub_lo[ui];
        const int nu = (int)(t.sub_hi[ui] - ulo);
        if (m > 0 && nu > 0) {
            // C(Q_{a_j}, S) of levels 0..M-3 for all observations of the unit, into B^
            T* Uf = t.Ufin + ulo * Lr;  // (L r) x nu, ld = L r
            T* Bh = t.Bhat + ulo * Lr;
            long aoff[kMaxLevels];
            for (int j = 0; j < m; ++j) aoff[j] = anc[j] * r;
            fill_cov_blocks<T>(g, t.pts, aoff, m, r, t.obs0 + ulo, nu, false, Bh, Lr, r, sm);
            for (int j = 0; j < m; ++j) {
                const long a = anc[j];
                T* V = Bh + (long)j * r;  // V_j (kept: B^ is L_Sigma^{-1} V^T)
                if (j > 0) {
                    const T* Ua = t.U + t.u_off[j] + (a - level_start(t.J, j)) * (long)j * rr;
                    gemm<T, true, false>(r, nu, j * r, (T)-1, Ua, (long)j * r, Uf, Lr, (T)1, V, Lr, sm);
                }
                gemm<T, false, false>(r, nu, r, (T)1, t.Pinv + a * rr, r, V, Lr, (T)0, Uf + (long)j * r, Lr, sm);
            }
        }
        for (long ploc = g_lo; ploc < g_hi; ++ploc) {
            const long p = s2 + ploc;
            const long clo = t.child_lo[ploc], chi = t.child_hi[ploc];
            const long lo = t.obs_off[clo];
            const int np = (int)(t.obs_off[chi] - lo);
            double dterm = 0.0;
            if (np > 0) {
                // level M-2: the group's own parent p
                T* Uf = t.Ufin + lo * Lr;
                T* V = t.Bhat + lo * Lr + (long)m * r;
                const long ap = p * r;
                fill_cov_blocks<T>(g, t.pts, &ap, 1, r, t.obs0 + lo, np, false, V, Lr, 0, sm);
                if (m > 0) {
                    const T* Ua = t.U + t.u_off[m] + ploc * (long)m * rr;
                    gemm<T, true, false>(r, np, m * r, (T)-1, Ua, (long)m * r, Uf, Lr, (T)1, V, Lr, sm);
                }
                gemm<T, false, false>(r, np, r, (T)1, t.Pinv + p * rr, r, V, Lr, (T)0, Uf + (long)m * r, Lr, sm);
                int nmax = 0;
                for (long c = clo; c < chi; ++c) nmax = max(nmax, (int)(t.obs_off[c + 1] - t.obs_off[c]));
                const bool grouped = sizeof(T) == 8 && nmax <= kChildMax && np <= kGroupMax &&
                                     chi - clo <= kThreads / 32;
                if (grouped) dterm += finest_children_grouped<T>(g, t, clo, chi, lo, np, ws, sm);
                for (long c = clo; c < chi && !grouped; ++c) {
                    const long o0 = t.obs_off[c];
                    const int n = (int)(t.obs_off[c + 1] - o0);
                    if (n == 0) continue;
                    T* S = t.Lsig + t.lsig_off[c];
                    fill_cov<T>(g, t.pts, t.obs0 + o0, n, t.obs0 + o0, n, true, S, n, sm);
                    __syncthreads();
                    gemm<T, true, false>(n, n, (int)Lr, (T)-1, t.Ufin + o0 * Lr, Lr, t.Ufin + o0 * Lr, Lr, (T)1, S,
                                         n, sm);
                    double ld = 0.0;
                    const bool small = sizeof(T) == 8 && n <= 64;
                    T* Sinv = ws;  // n x n
                    int info = potrf_lower<T>(n, S, n, sm, &ld, small ? Sinv : nullptr, n);
                    double* ytc = t.yt + o0;
                    for (int e = threadIdx.x; e < n; e += kThreads) ytc[e] = t.y[o0 + e];
                    __syncthreads();
                    if (small) trmv_lower_inv<T>(n, Sinv, n, ytc, ytc);  // y~ = L_Sigma^{-1} y
                    else trsv_lower_f64<T>(n, S, n, ytc);
                    if (small) {
                        // B^ = V L_Sigma^{-T}, in place: each 64-row tile of the product
                        // reads exactly the rows it then writes
                        gemm<T, false, true, true>((int)Lr, n, n, (T)1, t.Bhat + o0 * Lr, Lr, Sinv, n, (T)0,
                                                   t.Bhat + o0 * Lr, Lr, sm);
                    } else {
                        trsm_right_lower_trans<T>((int)Lr, n, S, n, t.Bhat + o0 * Lr, Lr, sm);
                    }
                    double part = 0.0;
                    for (int e = threadIdx.x; e < n; e += kThreads) part += ytc[e] * ytc[e];
                    double yy = cta_sum(part, sm);
                    if (threadIdx.x == 0) {
                        dterm += yy + ld;
                        if (info) report_error(t.err, t.n_int + c);
                    }
                }
            }
            if (threadIdx.x == 0) t.dfin[ploc] = dterm;
            if (!t.fuse_post) continue;
            dterm = 0.0;
            // posterior of the parent at level m = M-2 from F = B^ rows, f = y~
            const T* F = t.Bhat + lo * Lr;
            const double* f = t.yt + lo;
            if (t.factored[p]) {
                T* Fo = m > 0 ? t.Fbuf[m & 1] + lo * (long)m * r : nullptr;
                double* fo = m > 0 ? t.fbuf[m & 1] + lo : nullptr;
                factored_step<T>(t, m, p, np, F, Lr, f, Fo, fo, keep != 0, ws, wsd, sm, dterm);
            } else {
                T* Aagg = ws;
                double* wagg = wsd;
                accumulate_factored<T>(t, m, np, F, Lr, f, Aagg, wagg, true, sm);
                dense_step<T>(t, m, p, Aagg, wagg, keep != 0, Aagg + n_slices(m + 1) * rr, sm, dterm);
            }
            if (threadIdx.x == 0) t.dpost[p] = dterm;
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// a9/a10/a11: posterior, one level (m = M-3 .. 0)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads, 2) k_posterior_level(Geom g, DevTree<T> t, int m, int keep) {
    LaSmem<T>& sm = la_smem<T>();
    const int r = t.r;
    const long rr = (long)r * r, mr1 = (long)(m + 1) * r;
    const long s0 = level_start(t.J, m), cnt = level_count(t.J, m);
    const long ns_in = n_slices(m + 1);
    T* ws = t.ws + blockIdx.x * t.ws_stride;
    double* wsd = t.wsd + blockIdx.x * t.wsd_stride;
    const T* Fin = t.Fbuf[(m + 1) & 1];
    const double* fin = t.fbuf[(m + 1) & 1];
    const T* ain = t.aout[(m + 1) & 1];
    const double* win = t.wout[(m + 1) & 1];
    const bool from_finest = m == t.M - 2;  // children are finest regions: rows of B^, y~
    // regions taken from a shared counter, most expensive first (the clustered
    // regions' dense steps cost tens of factored ones)
    __shared__ long s_loc;
    for (;;) {
        __syncthreads();  // every thread has read the previous s_loc
        if (threadIdx.x == 0) {
            const int q = atomicAdd(&t.queue[kQueuePost + m], 1);
            s_loc = q < cnt ? t.post_order[s0 + q] : -1;
        }
        __syncthreads();
        const long loc = s_loc;
        if (loc < 0) break;
        const long i = s0 + loc;
        if (skipped(t, i)) continue;
        double dterm = 0.0;
        if (from_finest) {
            const long lo = t.sub_lo[i];
            const int n = (int)(t.sub_hi[i] - lo);
            const T* F = t.Bhat + lo * mr1;
            const double* f = t.yt + lo;
            if (t.factored[i]) {
                T* Fo = m > 0 ? t.Fbuf[m & 1] + lo * (long)m * r : nullptr;
                double* fo = m > 0 ? t.fbuf[m & 1] + lo : nullptr;
                factored_step<T>(t, m, i, n, F, mr1, f, Fo, fo, keep != 0, ws, wsd, sm, dterm);
            } else {
                T* Aagg = ws;
                double* wagg = wsd;
                accumulate_factored<T>(t, m, n, F, mr1, f, Aagg, wagg, true, sm);
                dense_step<T>(t, m, i, Aagg, wagg, keep != 0, Aagg + ns_in * rr, sm, dterm);
            }
        } else if (t.factored[i]) {
            const long lo = t.sub_lo[i];
            const int n = (int)(t.sub_hi[i] - lo);
            T* Fo = m > 0 ? t.Fbuf[m & 1] + lo * (long)m * r : nullptr;
            double* fo = m > 0 ? t.fbuf[m & 1] + lo : nullptr;
            factored_step<T>(t, m, i, n, Fin + lo * mr1, mr1, fin + lo, Fo, fo, keep != 0, ws, wsd, sm, dterm);
        } else {
            T* Aagg = ws;
            double* wagg = wsd;
            bool first = true;  // the first contribution sets Aagg / wagg
            for (int cc = 1; cc <= t.J; ++cc) {
                const long c = i * t.J + cc;
                if (t.factored[c]) {
                    // factored children with adjacent rows are accumulated together
                    const long lo = t.sub_lo[c];
                    long hi = t.sub_hi[c], cl = c;
                    while (cc < t.J && t.factored[cl + 1] && t.sub_lo[cl + 1] == hi) {
                        ++cc;
                        ++cl;
                        hi = t.sub_hi[cl];
                    }
                    accumulate_factored<T>(t, m, (int)(hi - lo), Fin + lo * mr1, mr1, fin + lo, Aagg, wagg, first, sm);
                } else {
                    const long cl = t.dslot[c];
                    const T* as = ain + cl * ns_in * rr;
                    const double* wsrc = win + cl * mr1;
                    for (long e = threadIdx.x; e < ns_in * rr; e += kThreads) Aagg[e] = first ? as[e] : Aagg[e] + as[e];
                    for (long e = threadIdx.x; e < mr1; e += kThreads) wagg[e] = first ? wsrc[e] : wagg[e] + wsrc[e];
                    __syncthreads();
                }
                first = false;
            }
            dense_step<T>(t, m, i, Aagg, wagg, keep != 0, Aagg + ns_in * rr, sm, dterm);
        }
        if (threadIdx.x == 0) t.dpost[i] = dterm;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// a12: prediction
// ---------------------------------------------------------------------------
// For every prediction q < np, one warp forms ss = sum_x c_x^2 and
// mm = sum_x c_x v_x over the column c = C + q ldc (len entries; v may be
// null) with a fixed lane -> entry mapping and shuffle tree, and lane 0 applies
// var[q] += sgn * ss, mean[q] = (add_mean ? mean[q] : 0) + mm.  Ends with a barrier.
template <typename T>
__device__ inline void predict_column_sums(int np, const T* C, long ldc, int len, const double* v, double sgn,
                                           bool add_mean, double* var, double* mean) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = w; q < np; q += kThreads / 32) {
        const T* col = C + (long)q * ldc;
        double ss = 0.0, mm = 0.0;
        for (int x = lane; x < len; x += 32) {
            const double c = (double)col[x];
            ss += c * c;
            if (v) mm += c * v[x];
        }
        for (int o = 16; o > 0; o >>= 1) {
            ss += __shfl_xor_sync(0xffffffffu, ss, o);
            mm += __shfl_xor_sync(0xffffffffu, mm, o);
        }
        if (lane == 0) {
            var[q] += sgn * ss;
            if (v) mean[q] = (add_mean ? mean[q] : 0.0) + mm;
        }
    }
    __syncthreads();
}

// One CTA per level M-2 region: the finest children of a region share all of
// their ancestors, so the conditioning of the group's predictions on the
// ancestors (prior part) and the posterior pass back over the ancestors run
// once for all of them; only the part of each finest region's own
// observations runs per child.
template <typename T>
__global__ void __launch_bounds__(kThreads, 2) k_predict(Geom g, DevTree<T> t) {
    LaSmem<T>& sm = la_smem<T>();
    __shared__ long s_k;
    const int r = t.r, L = t.L;
    const long rr = (long)r * r, Lr = (long)L * r;
    const long cnt2 = level_count(t.J, t.M - 2);
    for (;;) {
        if (threadIdx.x == 0) {
            int q = atomicAdd(&t.queue[1], 1);
            s_k = q < cnt2 ? t.pred_order[q] : -1;
        }
        __syncthreads();
        const long gl = s_k;
        __syncthreads();
        if (gl < 0) break;
        const long clo = t.child_lo[gl], chi = t.child_hi[gl];
        if (chi <= clo) continue;
        const long p0 = t.pred_off[clo];
        const int np = (int)(t.pred_off[chi] - p0);
        if (np == 0) continue;
        const int64_t* anc = t.fin_anc + clo * L;  // shared by every finest child of the region
        T* P = t.P + p0 * Lr;
        T* Bt = t.Bt + p0 * Lr;
        for (int j = 0; j < L; ++j) {
            const long a = anc[j];
            T* Cj = Bt + (long)j * r;
            fill_cov<T>(g, t.pts, a * r, r, t.pred0 + p0, np, false, Cj, Lr, sm);
            __syncthreads();
            if (j > 0) {
                const T* Ua = t.U + t.u_off[j] + (a - level_start(t.J, j)) * (long)j * rr;
                gemm<T, true, false>(r, np, j * r, (T)-1, Ua, (long)j * r, P, Lr, (T)1, Cj, Lr, sm);
            }
            // P_j = L_a^{-1} C_j as a product with the stored inverse of the prior factor
            gemm<T, false, false>(r, np, r, (T)1, t.Pinv + a * rr, r, Cj, Lr, (T)0, P + (long)j * r, Lr, sm);
        }
        double* mean = t.mean + p0;
        double* var = t.var + p0;
        for (int q = threadIdx.x; q < np; q += kThreads) {
            const long ip = t.pred0 + p0 + q;
            var[q] = t.pts.s2[ip] + t.pts.t2[ip];
            mean[q] = 0.0;
        }
        __syncthreads();
        predict_column_sums<T>(np, P, Lr, (int)Lr, nullptr, -1.0, false, var, mean);
        for (long k = clo; k < chi; ++k) {
            const long pk = t.pred_off[k];
            const int npk = (int)(t.pred_off[k + 1] - pk);
            const long o0 = t.obs_off[k];
            const int n = (int)(t.obs_off[k + 1] - o0);
            if (npk == 0 || n == 0) continue;
            T* Pk = t.P + pk * Lr;
            T* Pc = t.Pc + t.pc_off[k];  // n x npk, ld = n
            fill_cov<T>(g, t.pts, t.obs0 + o0, n, t.pred0 + pk, npk, false, Pc, n, sm);
            __syncthreads();
            gemm<T, true, false>(n, npk, (int)Lr, (T)-1, t.Ufin + o0 * Lr, Lr, Pk, Lr, (T)1, Pc, n, sm);
            trsm_left_lower<T>(n, npk, t.Lsig + t.lsig_off[k], n, Pc, n, sm);
            predict_column_sums<T>(npk, Pc, n, n, t.yt + o0, -1.0, false, var + (pk - p0), mean + (pk - p0));
            gemm<T, false, false>((int)Lr, npk, n, (T)-1, t.Bhat + o0 * Lr, Lr, Pc, n, (T)1, t.Bt + pk * Lr, Lr, sm);
        }
        for (int j = L - 1; j >= 0; --j) {
            const long a = anc[j];
            T* KcB = Bt + (long)j * r;
            if (t.Lpinv) {
                // L~_a^{-1} KcB in place (one row tile, r <= 64)
                gemm<T, false, false>(r, np, r, (T)1, t.Lpinv + a * rr, r, KcB, Lr, (T)0, KcB, Lr, sm);
            } else {
                trsm_left_lower<T>(r, np, t.Lpost + a * rr, r, KcB, Lr, sm);
            }
            if (j > 0) {
                const T* Ga = t.G + t.u_off[j] + (a - level_start(t.J, j)) * (long)j * rr;
                gemm<T, true, false>(j * r, np, r, (T)-1, Ga, r, KcB, Lr, (T)1, Bt, Lr, sm);
            }
            predict_column_sums<T>(np, KcB, Lr, r, t.vpost + a * r, 1.0, true, var, mean);
        }
    }
}

// ---------------------------------------------------------------------------
// deterministic final sum: d = sum(dpost) + sum(dfin)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_reduce(DevTree<T> t, double* out) {
    LaSmem<T>& sm = la_smem<T>();
    double s = 0.0;
    for (long i = threadIdx.x; i < t.n_int; i += kThreads) s += t.dpost[i];
    const long cnt2 = level_count(t.J, t.M - 2);
    for (long i = threadIdx.x; i < cnt2; i += kThreads) s += t.dfin[i];
    double tot = cta_sum(s, sm);
    if (threadIdx.x == 0) out[0] = tot;
}

// ---------------------------------------------------------------------------
// prior sample y = sum_j U_{obs,j}^T z_{a_j} + L_Sigma z_obs
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads, 2) k_sample(DevTree<T> t, const double* z_int, const double* z_obs,
                                                    double* y_out) {
    const int r = t.r, L = t.L;
    const long Lr = (long)L * r;
    for (long k = blockIdx.x; k < t.n_fin; k += gridDim.x) {
        const long o0 = t.obs_off[k];
        const int n = (int)(t.obs_off[k + 1] - o0);
        const int64_t* anc = t.fin_anc + k * L;
        const T* S = t.Lsig + t.lsig_off[k];
        for (int q = threadIdx.x; q < n; q += kThreads) {
            const T* col = t.Ufin + (o0 + q) * Lr;
            double y = 0.0;
            for (int j = 0; j < L; ++j) {
                const double* z = z_int + anc[j] * r;
                for (int x = 0; x < r; ++x) y += (double)col[(long)j * r + x] * z[x];
            }
            for (int x = 0; x <= q; ++x) y += (double)S[q + (long)x * n] * z_obs[o0 + x];
            y_out[o0 + q] = y;
        }
    }
}

// ---------------------------------------------------------------------------
// evaluate_*covariance blocks (layout out[i1*n2 + i2])
// ---------------------------------------------------------------------------
__global__ void k_cov_block(Geom g, PointSet P, long a0, int na, long b0, int nb, int self, double* out) {
    long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)na * nb) return;
    int tt = (int)(e % na), q = (int)(e / na);
    long ia = a0 + tt, ib = b0 + q;
    double v;
    if (self && tt == q)
        v = P.s2[ia] + P.t2[ia];
    else
        v = cov_entry(g, P.pt(ia), P.s2[ia], P.beta[ia], P.pt(ib), P.s2[ib], P.beta[ib]);
    out[e] = v;
}

template <typename Ti, typename To>
__global__ void k_convert(const Ti* __restrict__ in, To* __restrict__ out, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = (To)in[i];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_fields(const Geom& g, const FieldParams& fp, const double* c0, const double* c1, const double* c2,
                   long n, double* s2, double* beta, double* t2, cudaStream_t st) {
    if (n <= 0) return;
    k_fields<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, fp, c0, c1, c2, n, s2, beta, t2);
}
template <typename T>
int launch_prior_level(const Geom& g, const DevTree<T>& t, int m, int grid, cudaStream_t st, CovTiming* tm) {
    auto mark = [&](cudaEvent_t e) {
        if (tm->capturing) cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
        else cudaEventRecord(e, st);
    };
    const long cnt = level_count(t.J, m);
    const long per_region = (long)(m + 1) * t.r * t.r;
    long per = t.cbuf_elems / per_region;  // regions whose blocks fit the buffer at once
    if (per < 1) per = 1;
    int launches = 0;
    for (long loc0 = 0; loc0 < cnt; loc0 += per) {
        const long n = cnt - loc0 < per ? cnt - loc0 : per;
        const long nb = n * (m + 1);
        const long cov_grid = (long)grid * 16;  // 16 per region-kernel slot: 32 CTAs per SM
        const bool timed = tm && tm->used < tm->cap;
        if (tm && !timed) tm->overflow = true;
        if (timed) mark(tm->ev[2 * tm->used]);
        launch_cov_level<T>(g, t, m, loc0, n, (unsigned)(nb < cov_grid ? nb : cov_grid), st);
        if (timed) mark(tm->ev[2 * tm->used++ + 1]);
        k_prior_level<T><<<(unsigned)(n < grid ? n : grid), kThreads, sizeof(LaSmem<T>), st>>>(g, t, m, loc0, n,
                                                                                                t.cbuf);
        launches += 2;
    }
    return launches;
}
template <typename T>
int launch_finest_group(const Geom& g, const DevTree<T>& t, int grid, bool keep, cudaStream_t st) {
    long cnt = t.n_fin_items;
    k_finest_group<T><<<(unsigned)(cnt < grid ? cnt : grid), kThreads, sizeof(LaSmem<T>), st>>>(g, t, keep ? 1 : 0);
    return 1;
}
template <typename T>
void launch_posterior_level(const Geom& g, const DevTree<T>& t, int m, int grid, bool keep, cudaStream_t st) {
    long cnt = level_count(t.J, m);
    k_posterior_level<T><<<(unsigned)(cnt < grid ? cnt : grid), kThreads, sizeof(LaSmem<T>), st>>>(g, t, m, keep ? 1 : 0);
}
template <typename T>
void launch_predict(const Geom& g, const DevTree<T>& t, int grid, cudaStream_t st) {
    const long cnt2 = level_count(t.J, t.M - 2);
    k_predict<T><<<(unsigned)(cnt2 < grid ? cnt2 : grid), kThreads, sizeof(LaSmem<T>), st>>>(g, t);
}
template <typename T>
void launch_reduce(const DevTree<T>& t, double* out, cudaStream_t st) {
    k_reduce<T><<<1, kThreads, sizeof(LaSmem<T>), st>>>(t, out);
}
template <typename T>
void launch_sample(const DevTree<T>& t, const double* z_int, const double* z_obs, double* y_out, int grid,
                   cudaStream_t st) {
    k_sample<T><<<(unsigned)(t.n_fin < grid ? t.n_fin : grid), kThreads, sizeof(LaSmem<T>), st>>>(t, z_int, z_obs, y_out);
}
void launch_cov_block(const Geom& g, const PointSet& P, long a0, int na, long b0, int nb, bool self, double* out,
                      cudaStream_t st) {
    long n = (long)na * nb;
    if (n <= 0) return;
    k_cov_block<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, P, a0, na, b0, nb, self ? 1 : 0, out);
}

template <typename Ti, typename To>
void launch_convert(const Ti* in, To* out, long n, cudaStream_t st) {
    if (n <= 0) return;
    long blocks = (n + 255) / 256;
    k_convert<Ti, To><<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(in, out, n);
}
template void launch_convert<float, double>(const float*, double*, long, cudaStream_t);
template void launch_convert<double, float>(const double*, float*, long, cudaStream_t);

template <typename T>
static cudaError_t prepare_type() {
    const int bytes = (int)sizeof(LaSmem<T>);
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* fn) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    };
    set((const void*)k_prior_level<T>);
    set((const void*)k_finest_group<T>);
    set((const void*)k_posterior_level<T>);
    set((const void*)k_predict<T>);
    set((const void*)k_reduce<T>);
    set((const void*)k_sample<T>);
    return e;
}

cudaError_t set_gemm_tiles(const int nw[3]) { return cudaMemcpyToSymbol(c_gemm_nw, nw, 3 * sizeof(int)); }

cudaError_t prepare_kernels() {
    cudaError_t e = prepare_type<double>();
    return e == cudaSuccess ? prepare_type<float>() : e;
}

#define MRA_INSTANTIATE(T)                                                                                   \
    template int launch_prior_level<T>(const Geom&, const DevTree<T>&, int, int, cudaStream_t, CovTiming*); \
    template int launch_finest_group<T>(const Geom&, const DevTree<T>&, int, bool, cudaStream_t);           \
    template void launch_posterior_level<T>(const Geom&, const DevTree<T>&, int, int, bool, cudaStream_t);  \
    template void launch_predict<T>(const Geom&, const DevTree<T>&, int, cudaStream_t);                     \
    template void launch_reduce<T>(const DevTree<T>&, double*, cudaStream_t);                               \
    template void launch_sample<T>(const DevTree<T>&, const double*, const double*, double*, int, cudaStream_t);
MRA_INSTANTIATE(double)
MRA_INSTANTIATE(float)

}  // namespace mra
