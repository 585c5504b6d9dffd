// FP64 region kernels of the MRA hot path.
//
// Level-synchronous schedule (one launch per tree level and stage):
//   k_fields          sigma^2/beta/tau^2 at every knot, observation and
//                     prediction point (class_nonstationary_covariance.cpp:479-573)
//   k_prior_level(m)  one CTA per level-m region: U_{i,j} = L_{a_j}^{-1} V_j and
//                     L_i = chol(K_i)   (class_approximation.cpp:84-169)
//   k_finest          one CTA per finest region, largest first from a work
//                     queue: U, Sigma_i, L_Sigma, y~, B^, log-lik terms
//                     (...-loop-regions-at-finest-level-in-prior.cpp:90-269)
//   k_posterior(m)    levels M-2..0: child sums, L~ = chol(L L^T + A), v, G,
//                     w~, A~   (...-posterior-inference.cpp:14-265,
//                     class_approximation.cpp:186-306)
//   k_predict         one CTA per finest region with predictions: prior half
//                     (...-prior.cpp:271-392) then the top-down pass
//                     (class_approximation-predict.cpp:105-189)
//   k_reduce          deterministic sum of the per-region log-lik terms
//
// Finest-level A~ slices are never materialised: the level M-2 posterior forms
// the children's sum sum_c B^_{c,j}^T B^_{c,k} directly as one product over the
// stacked observation rows of its children.
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
// a5/a6: prior, one level of interior regions
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 2) k_prior_level(Geom g, DevTree t, int m) {
    __shared__ LaSmem sm;
    const int r = t.r;
    const long rr = (long)r * r;
    const long s0 = level_start(t.J, m), cnt = level_count(t.J, m);
    const long mr = (long)m * r;
    for (long loc = blockIdx.x; loc < cnt; loc += gridDim.x) {
        const long i = s0 + loc;
        long anc[kMaxLevels];
        {
            long c = i;
            for (int a = m - 1; a >= 0; --a) {
                c = (c - 1) / t.J;
                anc[a] = c;
            }
        }
        double* Ui = t.U + t.u_off[m] + loc * mr * r;  // (m r) x r, ld = m r
        for (int j = 0; j < m; ++j) {
            const long a = anc[j];
            double* V = Ui + (long)j * r;
            fill_cov(g, t.pts, a * r, r, i * r, r, false, V, mr);
            __syncthreads();
            if (j > 0) {
                const double* Ua = t.U + t.u_off[j] + (a - level_start(t.J, j)) * (long)j * rr;
                gemm<true, false>(r, r, j * r, -1.0, Ua, (long)j * r, Ui, mr, 1.0, V, mr, sm);
            }
            trsm_left_lower(r, r, t.Lprior + a * rr, r, V, mr, sm);
        }
        double* Li = t.Lprior + i * rr;
        fill_cov(g, t.pts, i * r, r, i * r, r, true, Li, r);
        __syncthreads();
        if (m > 0) gemm<true, false>(r, r, (int)mr, -1.0, Ui, mr, Ui, mr, 1.0, Li, r, sm);
        int info = potrf_lower(r, Li, r, sm);
        if (info && threadIdx.x == 0) report_error(t.err, i);
    }
}

// ---------------------------------------------------------------------------
// a7/a8: prior at the finest level
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 2) k_finest(Geom g, DevTree t) {
    __shared__ LaSmem sm;
    __shared__ long s_k;
    const int r = t.r, L = t.L;
    const long rr = (long)r * r, Lr = (long)L * r;
    for (;;) {
        if (threadIdx.x == 0) {
            int q = atomicAdd(&t.queue[0], 1);
            s_k = q < t.n_fin ? t.fin_order[q] : -1;
        }
        __syncthreads();
        const long k = s_k;
        __syncthreads();
        if (k < 0) break;
        const long o0 = t.obs_off[k];
        const int n = (int)(t.obs_off[k + 1] - o0);
        if (n == 0) {
            if (threadIdx.x == 0) t.dfin[k] = 0.0;
            continue;
        }
        const int64_t* anc = t.fin_anc + k * L;
        double* Uf = t.Ufin + o0 * Lr;  // (L r) x n, ld = L r
        double* Bh = t.Bhat + o0 * Lr;  // (L r) x n, ld = L r  (= B^ transposed)
        for (int j = 0; j < L; ++j) {
            const long a = anc[j];
            double* V = Uf + (long)j * r;
            fill_cov(g, t.pts, a * r, r, t.obs0 + o0, n, false, V, Lr);
            __syncthreads();
            if (j > 0) {
                const double* Ua = t.U + t.u_off[j] + (a - level_start(t.J, j)) * (long)j * rr;
                gemm<true, false>(r, n, j * r, -1.0, Ua, (long)j * r, Uf, Lr, 1.0, V, Lr, sm);
            }
            for (int e = threadIdx.x; e < r * n; e += kThreads) {
                int tt = e % r, q = e / r;
                Bh[(long)j * r + tt + (long)q * Lr] = V[tt + (long)q * Lr];
            }
            __syncthreads();
            trsm_left_lower(r, n, t.Lprior + a * rr, r, V, Lr, sm);
        }
        double* S = t.Lsig + t.lsig_off[k];
        fill_cov(g, t.pts, t.obs0 + o0, n, t.obs0 + o0, n, true, S, n);
        __syncthreads();
        gemm<true, false>(n, n, (int)Lr, -1.0, Uf, Lr, Uf, Lr, 1.0, S, n, sm);
        int info = potrf_lower(n, S, n, sm);
        double* yt = t.yt + o0;
        for (int e = threadIdx.x; e < n; e += kThreads) yt[e] = t.y[o0 + e];
        __syncthreads();
        trsm_left_lower(n, 1, S, n, yt, n, sm);
        trsm_right_lower_trans((int)Lr, n, S, n, Bh, Lr, sm);
        double part = 0.0;
        for (int e = threadIdx.x; e < n; e += kThreads) part += yt[e] * yt[e] + 2 * log(S[e + (long)e * n]);
        double tot = cta_sum(part, sm);
        if (threadIdx.x == 0) {
            t.dfin[k] = tot;
            if (info) report_error(t.err, t.n_int + k);
        }
    }
}

// ---------------------------------------------------------------------------
// a9/a10/a11/a14: posterior, one level (m = M-2 .. 0)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 2) k_posterior_level(Geom g, DevTree t, int m, int keep_g) {
    __shared__ LaSmem sm;
    const int r = t.r;
    const long rr = (long)r * r;
    const long s0 = level_start(t.J, m), cnt = level_count(t.J, m);
    const long ns_in = n_slices(m + 1), ns_out = n_slices(m);
    const long mr1 = (long)(m + 1) * r;
    double* ws = t.ws + blockIdx.x * t.ws_stride;
    double* Aagg = ws;               // ns_in slices of r x r
    double* wagg = Aagg + ns_in * rr;  // (m+1) x r
    double* Gw = wagg + mr1;         // m slices, when G is not kept
    const double* ain = t.aout[(m + 1) & 1];
    const double* win = t.wout[(m + 1) & 1];
    double* aout = t.aout[m & 1];
    double* wout = t.wout[m & 1];
    for (long loc = blockIdx.x; loc < cnt; loc += gridDim.x) {
        const long i = s0 + loc;
        if (m == t.M - 2) {
            // children are finest regions: A_(j,k) = X_j X_k^T over their stacked rows
            const long cl = t.child_lo[loc], ch = t.child_hi[loc];
            const long o0 = t.obs_off[cl];
            const int np = (int)(t.obs_off[ch] - o0);
            const double* X = t.Bhat + o0 * mr1;  // (L r) x np, ld = L r, L = m+1
            for (int j = 0; j <= m; ++j)
                for (int k = j; k <= m; ++k)
                    gemm<false, true>(r, r, np, 1.0, X + (long)j * r, mr1, X + (long)k * r, mr1, 0.0,
                                      Aagg + slice_index(m + 1, j, k) * rr, r, sm);
            gemm<false, false>((int)mr1, 1, np, 1.0, X, mr1, t.yt + o0, np > 0 ? np : 1, 0.0, wagg, mr1, sm);
        } else {
            const long c0 = i * t.J + 1 - level_start(t.J, m + 1);
            for (long e = threadIdx.x; e < ns_in * rr; e += kThreads) {
                double s = 0.0;
                for (int c = 0; c < t.J; ++c) s += ain[(c0 + c) * ns_in * rr + e];
                Aagg[e] = s;
            }
            for (long e = threadIdx.x; e < mr1; e += kThreads) {
                double s = 0.0;
                for (int c = 0; c < t.J; ++c) s += win[(c0 + c) * mr1 + e];
                wagg[e] = s;
            }
            __syncthreads();
        }
        const double* Lp = t.Lprior + i * rr;
        double* Lt = t.Lpost + i * rr;
        double part = 0.0;
        for (int e = threadIdx.x; e < r; e += kThreads) part -= 2 * log(Lp[e + (long)e * r]);
        gemm<false, true>(r, r, r, 1.0, Lp, r, Lp, r, 0.0, Lt, r, sm);
        const double* Amm = Aagg + slice_index(m + 1, m, m) * rr;
        for (long e = threadIdx.x; e < rr; e += kThreads) Lt[e] += Amm[e];
        __syncthreads();
        int info = potrf_lower(r, Lt, r, sm);
        double* v = t.vpost + i * r;
        for (int e = threadIdx.x; e < r; e += kThreads) v[e] = wagg[(long)m * r + e];
        __syncthreads();
        trsm_left_lower(r, 1, Lt, r, v, r, sm);
        for (int e = threadIdx.x; e < r; e += kThreads) part += 2 * log(Lt[e + (long)e * r]) - v[e] * v[e];
        double tot = cta_sum(part, sm);
        if (threadIdx.x == 0) {
            t.dpost[i] = tot;
            if (info) report_error(t.err, i);
        }
        if (m > 0) {
            double* Gi = keep_g ? t.G + t.u_off[m] + loc * (long)m * rr : Gw;  // r x (m r), ld = r
            for (long e = threadIdx.x; e < (long)m * rr; e += kThreads) {
                int j = (int)(e / rr);
                long w = e % rr;
                int p = (int)(w % r), q = (int)(w / r);
                Gi[e] = Aagg[slice_index(m + 1, j, m) * rr + q + (long)p * r];  // G_j = A_(j,m)^T
            }
            __syncthreads();
            trsm_left_lower(r, m * r, Lt, r, Gi, r, sm);
            double* wo = wout + loc * (long)m * r;
            for (long e = threadIdx.x; e < (long)m * r; e += kThreads) wo[e] = wagg[e];
            __syncthreads();
            gemm<true, false>(m * r, 1, r, -1.0, Gi, r, v, r, 1.0, wo, (long)m * r, sm);
            double* ao = aout + loc * ns_out * rr;
            for (int j = 0; j < m; ++j) {
                for (int k = j; k < m; ++k) {
                    double* dst = ao + slice_index(m, j, k) * rr;
                    const double* src = Aagg + slice_index(m + 1, j, k) * rr;
                    for (long e = threadIdx.x; e < rr; e += kThreads) dst[e] = src[e];
                    __syncthreads();
                    gemm<true, false>(r, r, r, -1.0, Gi + (long)j * rr, r, Gi + (long)k * rr, r, 1.0, dst, r, sm);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// a12: prediction
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 2) k_predict(Geom g, DevTree t) {
    __shared__ LaSmem sm;
    __shared__ long s_k;
    const int r = t.r, L = t.L;
    const long rr = (long)r * r, Lr = (long)L * r;
    for (;;) {
        if (threadIdx.x == 0) {
            int q = atomicAdd(&t.queue[1], 1);
            s_k = q < t.n_fin ? t.fin_order[q] : -1;
        }
        __syncthreads();
        const long k = s_k;
        __syncthreads();
        if (k < 0) break;
        const long p0 = t.pred_off[k];
        const int np = (int)(t.pred_off[k + 1] - p0);
        if (np == 0) continue;
        const long o0 = t.obs_off[k];
        const int n = (int)(t.obs_off[k + 1] - o0);
        const int64_t* anc = t.fin_anc + k * L;
        double* P = t.P + p0 * Lr;
        double* Bt = t.Bt + p0 * Lr;
        for (int j = 0; j < L; ++j) {
            const long a = anc[j];
            double* Cj = Bt + (long)j * r;
            fill_cov(g, t.pts, a * r, r, t.pred0 + p0, np, false, Cj, Lr);
            __syncthreads();
            if (j > 0) {
                const double* Ua = t.U + t.u_off[j] + (a - level_start(t.J, j)) * (long)j * rr;
                gemm<true, false>(r, np, j * r, -1.0, Ua, (long)j * r, P, Lr, 1.0, Cj, Lr, sm);
            }
            for (int e = threadIdx.x; e < r * np; e += kThreads) {
                int tt = e % r, q = e / r;
                P[(long)j * r + tt + (long)q * Lr] = Cj[tt + (long)q * Lr];
            }
            __syncthreads();
            trsm_left_lower(r, np, t.Lprior + a * rr, r, P + (long)j * r, Lr, sm);
        }
        double* mean = t.mean + p0;
        double* var = t.var + p0;
        for (int q = threadIdx.x; q < np; q += kThreads) {
            long ip = t.pred0 + p0 + q;
            double s = t.pts.s2[ip] + t.pts.t2[ip];
            const double* col = P + (long)q * Lr;
            double ss = 0.0;
            for (long x = 0; x < Lr; ++x) ss += col[x] * col[x];
            var[q] = s - ss;
            mean[q] = 0.0;
        }
        __syncthreads();
        if (n > 0) {
            double* Pc = t.Pc + t.pc_off[k];  // n x np, ld = n
            fill_cov(g, t.pts, t.obs0 + o0, n, t.pred0 + p0, np, false, Pc, n);
            __syncthreads();
            gemm<true, false>(n, np, (int)Lr, -1.0, t.Ufin + o0 * Lr, Lr, P, Lr, 1.0, Pc, n, sm);
            trsm_left_lower(n, np, t.Lsig + t.lsig_off[k], n, Pc, n, sm);
            const double* yt = t.yt + o0;
            for (int q = threadIdx.x; q < np; q += kThreads) {
                const double* col = Pc + (long)q * n;
                double ss = 0.0, mm = 0.0;
                for (int x = 0; x < n; ++x) {
                    ss += col[x] * col[x];
                    mm += col[x] * yt[x];
                }
                var[q] -= ss;
                mean[q] = mm;
            }
            __syncthreads();
            gemm<false, false>((int)Lr, np, n, -1.0, t.Bhat + o0 * Lr, Lr, Pc, n, 1.0, Bt, Lr, sm);
        }
        for (int j = L - 1; j >= 0; --j) {
            const long a = anc[j];
            double* KcB = Bt + (long)j * r;
            trsm_left_lower(r, np, t.Lpost + a * rr, r, KcB, Lr, sm);
            if (j > 0) {
                const double* Ga = t.G + t.u_off[j] + (a - level_start(t.J, j)) * (long)j * rr;
                gemm<true, false>(j * r, np, r, -1.0, Ga, r, KcB, Lr, 1.0, Bt, Lr, sm);
            }
            const double* va = t.vpost + a * r;
            for (int q = threadIdx.x; q < np; q += kThreads) {
                const double* col = KcB + (long)q * Lr;
                double ss = 0.0, mm = 0.0;
                for (int x = 0; x < r; ++x) {
                    ss += col[x] * col[x];
                    mm += col[x] * va[x];
                }
                var[q] += ss;
                mean[q] += mm;
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// deterministic final sum: d = sum(dfin) + sum(dpost)
// ---------------------------------------------------------------------------
__global__ void k_reduce(DevTree t, double* out) {
    __shared__ LaSmem sm;
    double s = 0.0;
    for (long i = threadIdx.x; i < t.n_fin; i += kThreads) s += t.dfin[i];
    for (long i = threadIdx.x; i < t.n_int; i += kThreads) s += t.dpost[i];
    double tot = cta_sum(s, sm);
    if (threadIdx.x == 0) out[0] = tot;
}

// ---------------------------------------------------------------------------
// prior sample y = sum_j U_{obs,j}^T z_{a_j} + L_Sigma z_obs
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_sample(DevTree t, const double* z_int, const double* z_obs,
                                                    double* y_out) {
    const int r = t.r, L = t.L;
    const long Lr = (long)L * r;
    for (long k = blockIdx.x; k < t.n_fin; k += gridDim.x) {
        const long o0 = t.obs_off[k];
        const int n = (int)(t.obs_off[k + 1] - o0);
        const int64_t* anc = t.fin_anc + k * L;
        const double* S = t.Lsig + t.lsig_off[k];
        for (int q = threadIdx.x; q < n; q += kThreads) {
            const double* col = t.Ufin + (o0 + q) * Lr;
            double y = 0.0;
            for (int j = 0; j < L; ++j) {
                const double* z = z_int + anc[j] * r;
                for (int x = 0; x < r; ++x) y += col[(long)j * r + x] * z[x];
            }
            for (int x = 0; x <= q; ++x) y += S[q + (long)x * n] * z_obs[o0 + x];
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

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_fields(const Geom& g, const FieldParams& fp, const double* c0, const double* c1, const double* c2,
                   long n, double* s2, double* beta, double* t2, cudaStream_t st) {
    if (n <= 0) return;
    k_fields<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, fp, c0, c1, c2, n, s2, beta, t2);
}
void launch_prior_level(const Geom& g, const DevTree& t, int m, int grid, cudaStream_t st) {
    long cnt = level_count(t.J, m);
    k_prior_level<<<(unsigned)(cnt < grid ? cnt : grid), kThreads, 0, st>>>(g, t, m);
}
void launch_finest(const Geom& g, const DevTree& t, int grid, bool, cudaStream_t st) {
    k_finest<<<(unsigned)(t.n_fin < grid ? t.n_fin : grid), kThreads, 0, st>>>(g, t);
}
void launch_posterior_level(const Geom& g, const DevTree& t, int m, int grid, bool keep_g, cudaStream_t st) {
    long cnt = level_count(t.J, m);
    k_posterior_level<<<(unsigned)(cnt < grid ? cnt : grid), kThreads, 0, st>>>(g, t, m, keep_g ? 1 : 0);
}
void launch_predict(const Geom& g, const DevTree& t, int grid, cudaStream_t st) {
    k_predict<<<(unsigned)(t.n_fin < grid ? t.n_fin : grid), kThreads, 0, st>>>(g, t);
}
void launch_reduce(const DevTree& t, double* out, cudaStream_t st) { k_reduce<<<1, kThreads, 0, st>>>(t, out); }
void launch_sample(const DevTree& t, const double* z_int, const double* z_obs, double* y_out, int grid,
                   cudaStream_t st) {
    k_sample<<<(unsigned)(t.n_fin < grid ? t.n_fin : grid), kThreads, 0, st>>>(t, z_int, z_obs, y_out);
}
void launch_cov_block(const Geom& g, const PointSet& P, long a0, int na, long b0, int nb, bool self, double* out,
                      cudaStream_t st) {
    long n = (long)na * nb;
    if (n <= 0) return;
    k_cov_block<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, P, a0, na, b0, nb, self ? 1 : 0, out);
}

}  // namespace mra
