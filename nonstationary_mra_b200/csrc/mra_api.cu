// C ABI of the MRA hot path (include/mra_b200.h): context lifetime, device
// residency of the partition, the per-evaluation launch sequence, CUDA-graph
// capture and statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mra_b200.h"
#include "mra_kernels.cuh"

using namespace mra;

namespace {

thread_local std::string g_last_error;

mra_status fail(mra_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

#define CU(call)                                                                                \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            if (e_ == cudaErrorMemoryAllocation)                                                \
                return fail(MRA_ERR_OOM, std::string(#call ": ") + cudaGetErrorString(e_));     \
            return fail(MRA_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_));        \
        }                                                                                       \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

void mra::set_last_error(const char* msg) { g_last_error = msg; }

struct mra_ctx {
    int device = 0;
    int precision = 0;
    int sms = 0;
    int grid = 0;  // CTAs per region-kernel launch
    int J = 0, M = 0, r = 0, L = 0, tf = 0;
    long n_int = 0, n_fin = 0, n_obs = 0, n_pred = 0;
    Geom geom{};
    FieldParams fp{};
    DevTree<double> td{};
    DevTree<float> tf32{};
    std::vector<DevBuf> bufs;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8]{};
    cudaEvent_t tev[2 * MRA_MAX_TIMED]{};  // start/stop of every launch
    // start/stop of each covariance-block launch of the prior levels, and the
    // timed launch (index into tev pairs) that each belongs to
    static constexpr int kMaxCovTimed = 64;
    cudaEvent_t cev[2 * kMaxCovTimed]{};
    int cov_owner[kMaxCovTimed]{};
    int n_cov = 0;
    bool cov_overflow = false;
    struct Launch {
        int kind, level;
        double flop;
    };
    std::vector<Launch> plan;  // launches of one log-likelihood, in order
    double flop_predict_launch = 0;
    int n_timed = 0;
    std::vector<int> timed_plan;  // plan index of each timed launch of the last evaluation (-1: prediction)
    // sub-tree sharding: split level (0 = off), the device mask of computed
    // regions, and the evaluation phase (0 whole, 1 own sub-trees, 2 top levels)
    int shard_split = 0;
    int8_t* d_active = nullptr;
    int eval_phase = 0;
    std::vector<int8_t> h_factored;          // [n_int] posterior output kept as F, f
    std::vector<int64_t> h_sub_lo, h_sub_hi;  // [n_int] observation range of each sub-tree
    std::vector<int64_t> h_dslot;            // [n_int] slot among the level's dense regions
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    // prior -> posterior (predictive factors kept) -> prediction, when the
    // structure has prediction locations
    cudaGraph_t graph_pred = nullptr;
    cudaGraphExec_t graph_pred_exec = nullptr;
    int graph_timed[2] = {0, 0};     // timed stages of the log-likelihood / prediction graph
    int graph_launches[2] = {0, 0};  // kernels launched by each
    int graph_cov[2] = {0, 0};       // timed covariance-block launches of each
    double* d_theta = nullptr;  // 16 doubles
    double* d_weights[3]{};
    long nb[3]{};
    std::vector<double> model_weights[3];
    double model_intercept[3]{};
    double* d_result = nullptr;  // [0] d
    double flop_loglik = 0, flop_reference = 0;
    int64_t u_total = 0;
    mra_stats stats{};
    int last_launches = 0;
    bool have_pred = false;
    // mixed path stages kept in FP32 (a diagnostic switch, MRA_MIXED_FP32):
    // the prior levels and the finest level; the posterior is always FP64
    bool mixed_prior32 = true, mixed_finest32 = true;

    void* alloc_bytes(size_t bytes_, cudaError_t* err) {
        DevBuf b;
        b.bytes = std::max<size_t>(bytes_, 16);
        *err = cudaMalloc(&b.p, b.bytes);
        if (*err != cudaSuccess) return nullptr;
        bufs.push_back(b);
        bytes += b.bytes;
        return b.p;
    }
    template <typename T>
    T* alloc(size_t count, cudaError_t* err) {
        return static_cast<T*>(alloc_bytes(count * sizeof(T), err));
    }
    ~mra_ctx() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        if (graph_pred_exec) cudaGraphExecDestroy(graph_pred_exec);
        if (graph_pred) cudaGraphDestroy(graph_pred);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : tev)
            if (e) cudaEventDestroy(e);
        for (auto& e : cev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
        for (auto& b : bufs) cudaFree(b.p);
    }
};

namespace {

Geom make_geom(const mra_model* m) {
    Geom g{};
    g.nonstat = m->nonstationary ? 1 : 0;
    g.distance = m->distance;
    g.nu_x2 = m->nu_x2;
    g.pref_exp = m->prefactor_exp;
    g.pref_kind = m->prefactor_exp == 1.5 ? 0 : (m->prefactor_exp == 1.0 ? 1 : 2);
    g.dist_scale = m->dist_scale;
    return g;
}

}  // namespace

mra_status mra::check_model(const mra_model* m) {
    if (!m) return fail(MRA_ERR_ARG, "model is NULL");
    if (m->distance < 0 || m->distance > 2) return fail(MRA_ERR_ARG, "unknown distance kind");
    if (m->nu_x2 != 1 && m->nu_x2 != 3) return fail(MRA_ERR_ARG, "nu must be 1/2 or 3/2");
    if (m->basis != 0 && m->basis != 1) return fail(MRA_ERR_ARG, "unknown basis kind");
    if (m->nonstationary) {
        if (!(m->basis_len > 0)) return fail(MRA_ERR_ARG, "basis length must be positive");
        for (int f = 0; f < 3; ++f)
            if (m->field[f].n_basis && (!m->field[f].centers || !m->field[f].weights))
                return fail(MRA_ERR_ARG, "field basis arrays are NULL");
    }
    return MRA_OK;
}

namespace {

mra_status upload(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return MRA_OK;
    CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return MRA_OK;
}

// Host-side description of the tree used for sizing, scheduling and FLOP counts.
struct HostTree {
    std::vector<int64_t> nfin, npred, obs_off, pred_off, fin_anc, pred_order, lsig_off, pc_off;
    std::vector<int64_t> child_lo, child_hi, par_order, sub_lo, sub_hi, dslot, post_order;
    std::vector<int8_t> factored;
};

// Algorithmic multiply-adds of the region kernels as run here (symmetric
// products counted once), per launch, from the realised region sizes; and the
// reference algorithm's canonical count for the same tree:
//   prior, level m:     r^3 [m(m-1)/2 + m/2 + m/2 + 1/6]
//   posterior, level m: r^3 [1/3 + m/2 + m/2 + m(m-1)/2] + r^2 (1/2 + m)
//   finest region (n observations, L = M-1): r^2 n L(L-1)/2 + L r^2 n/2 + L r n^2/2
//     + n^3/6 + n^2/2 + L n^2 r/2 + L r n + L r^2 n/2 + L(L-1)/2 r^2 n
// Factored posterior step of a region with n rows at level m:
//   r^2 n/2 + r n^2/2 + n^3/6 + n^2/2 + m r n^2/2.
void make_plan(mra_ctx* c, const HostTree& h) {
    const int J = c->J, M = c->M;
    const double R = c->r, Lv = M - 1;
    double fields = 0;
    for (int f = 0; f < 3; ++f) fields += (double)c->nb[f];
    c->plan.clear();
    c->plan.push_back({MRA_KERNEL_FIELDS, -1, (double)(c->n_int * c->r + c->n_obs + c->n_pred) * (fields * 12 + 8)});
    double ref = 0;
    for (int m = 0; m <= M - 2; ++m) {
        double cnt = std::pow((double)J, m), mm = m;
        double f = cnt * R * R * R * (mm * (mm - 1) / 2 + mm / 2 + mm / 2 + 1.0 / 6);
        c->plan.push_back({MRA_KERNEL_PRIOR_LEVEL, m, 2 * f});
        ref += f + cnt * (R * R * R * (1.0 / 3 + mm / 2 + mm / 2 + mm * (mm - 1) / 2) + R * R * (0.5 + mm));
    }
    auto dense_post = [&](double mm) {
        return R * R * R * (1.0 / 3 + mm / 2 + mm / 2 + mm * (mm - 1) / 2) + R * R * (0.5 + mm);
    };
    auto fact_post = [&](double n, double mm) {
        return R * R * n / 2 + R * n * n / 2 + n * n * n / 6 + n * n / 2 + mm * R * n * n / 2;
    };
    auto agg = [&](double n, double mm) { return (mm + 1) * (mm + 2) / 2 * R * R * n + (mm + 1) * R * n; };
    // finest groups (+ level M-2 posterior)
    double fin = 0;
    const long s2 = level_start(J, M - 2), cnt2 = level_count(J, M - 2);
    for (long q = 0; q < cnt2; ++q) {
        double np = (double)(h.sub_hi[s2 + q] - h.sub_lo[s2 + q]);
        fin += R * R * np * Lv * (Lv - 1) / 2 + Lv * R * R * np / 2;
        for (long k = h.child_lo[q]; k < h.child_hi[q]; ++k) {
            double n = (double)h.nfin[k];
            if (n == 0) continue;
            fin += Lv * R * n * n / 2 + n * n * n / 6 + n * n / 2 + Lv * n * n * R / 2;
            ref += R * R * n * Lv * (Lv - 1) / 2 + Lv * R * R * n / 2 + Lv * R * n * n / 2 + n * n * n / 6 + n * n / 2 +
                   Lv * n * n * R / 2 + Lv * R * n + Lv * R * R * n / 2 + Lv * (Lv - 1) / 2 * R * R * n;
        }
        fin += h.factored[s2 + q] ? fact_post(np, M - 2) : agg(np, M - 2) + dense_post(M - 2);
    }
    c->plan.push_back({MRA_KERNEL_FINEST, M - 1, 2 * fin});
    const bool split = c->precision == MRA_PRECISION_MIXED;
    if (split) {
        // the posterior runs in FP64: FP32 prior factors and B^ are widened first,
        // and the level M-2 posterior moves out of the finest-group kernel
        c->plan.push_back({MRA_KERNEL_CONVERT, -1, 0.0});
        double f2 = 0;
        for (long q = 0; q < cnt2; ++q) {
            double np = (double)(h.sub_hi[s2 + q] - h.sub_lo[s2 + q]);
            f2 += h.factored[s2 + q] ? fact_post(np, M - 2) : agg(np, M - 2) + dense_post(M - 2);
        }
        fin -= f2;
        c->plan.back().flop = 0;
        c->plan[c->plan.size() - 2].flop = 2 * fin;
        c->plan.push_back({MRA_KERNEL_POSTERIOR_LEVEL, M - 2, 2 * f2});
    }
    for (int m = M - 3; m >= 0; --m) {
        const long s0 = level_start(J, m), cnt = level_count(J, m);
        double f = 0;
        for (long q = 0; q < cnt; ++q) {
            const long i = s0 + q;
            double n = (double)(h.sub_hi[i] - h.sub_lo[i]);
            if (h.factored[i]) {
                f += fact_post(n, m);
            } else {
                for (int cc = 1; cc <= J; ++cc) {
                    long ch = i * J + cc;
                    if (h.factored[ch]) f += agg((double)(h.sub_hi[ch] - h.sub_lo[ch]), m);
                }
                f += dense_post(m);
            }
        }
        c->plan.push_back({MRA_KERNEL_POSTERIOR_LEVEL, m, 2 * f});
    }
    c->plan.push_back({MRA_KERNEL_REDUCE, -1, (double)c->n_int});
    c->flop_loglik = 0;
    for (auto& l : c->plan) c->flop_loglik += l.flop;
    c->flop_reference = 2 * ref;
}

cudaError_t record(cudaEvent_t e, cudaStream_t st, bool capturing) {
    return capturing ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal) : cudaEventRecord(e, st);
}

// Issues one evaluation on the context's stream: every launch of the plan
// (plus prediction) bracketed by its own pair of timing events.  The events are
// recorded as external nodes so that they still time each launch when the
// sequence is replayed from a captured CUDA graph.
// FP64 path: every stage on the double tree.  Mixed path: fields, prior and
// finest level on the FP32 tree, conversion, posterior and reduction on the
// FP64 tree, prediction on the FP32 tree with the widened-back posterior factors.
mra_status run_eval(mra_ctx* c, bool predict) {
    cudaStream_t st = c->stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CU(cudaStreamIsCapturing(st, &cap));
    const bool capturing = cap == cudaStreamCaptureStatusActive;
    const bool mixed = c->precision == MRA_PRECISION_MIXED;
    DevTree<double>& td = c->td;
    DevTree<float>& tf = c->tf32;
    CU(cudaMemsetAsync(td.queue, 0, kQueueCounters * sizeof(int), st));
    CU(cudaMemsetAsync(td.err, 0, 4 * sizeof(int), st));
    const long np_all = c->n_int * c->r + c->n_obs + c->n_pred;
    const long rr = (long)c->r * c->r;
    int i = 0, launched = 0;
    c->timed_plan.clear();
    CovTiming cov{c->cev, mra_ctx::kMaxCovTimed, 0, capturing, false};
    for (size_t pi = 0; pi < c->plan.size(); ++pi) {
        const auto& l = c->plan[pi];
        if (c->eval_phase != 0) {
            // phase 1: everything of the own sub-trees (levels >= split); phase 2: the levels above + the sum
            const bool top = (l.kind == MRA_KERNEL_POSTERIOR_LEVEL && l.level < c->shard_split) ||
                             l.kind == MRA_KERNEL_REDUCE;
            if (top != (c->eval_phase == 2)) continue;
        }
        c->timed_plan.push_back((int)pi);
        CU(record(c->tev[2 * i], st, capturing));
        switch (l.kind) {
            case MRA_KERNEL_FIELDS:
                launch_fields(c->geom, c->fp, td.pts.c0, td.pts.c1, td.pts.c2, np_all, const_cast<double*>(td.pts.s2),
                              const_cast<double*>(td.pts.beta), const_cast<double*>(td.pts.t2), st);
                launched += 1;
                break;
            case MRA_KERNEL_PRIOR_LEVEL: {
                const int u0 = cov.used;
                if (mixed && c->mixed_prior32)
                    launched += launch_prior_level<float>(c->geom, tf, l.level, c->grid, st, &cov);
                else launched += launch_prior_level<double>(c->geom, td, l.level, c->grid, st, &cov);
                for (int k = u0; k < cov.used; ++k) c->cov_owner[k] = i;
                break;
            }
            case MRA_KERNEL_FINEST:
                if (mixed && c->mixed_prior32 != c->mixed_finest32) {
                    // the finest level runs in the other precision: its ancestors' factors follow it
                    if (c->mixed_prior32) {
                        launch_convert<float, double>(tf.U, td.U, c->u_total, st);
                        launch_convert<float, double>(tf.Lprior, td.Lprior, c->n_int * rr, st);
                        launch_convert<float, double>(tf.Pinv, td.Pinv, c->n_int * rr, st);
                    } else {
                        launch_convert<double, float>(td.U, tf.U, c->u_total, st);
                        launch_convert<double, float>(td.Lprior, tf.Lprior, c->n_int * rr, st);
                        launch_convert<double, float>(td.Pinv, tf.Pinv, c->n_int * rr, st);
                    }
                    launched += 3;
                }
                if (mixed && c->mixed_finest32) launched += launch_finest_group<float>(c->geom, tf, c->grid, predict, st);
                else launched += launch_finest_group<double>(c->geom, td, c->grid, predict, st);
                break;
            case MRA_KERNEL_CONVERT:
                if (c->mixed_prior32 && c->mixed_finest32) {
                    launch_convert<float, double>(tf.Lprior, td.Lprior, c->n_int * rr, st);
                    launch_convert<float, double>(tf.Pinv, td.Pinv, c->n_int * rr, st);
                    launched += 2;
                }
                if (c->mixed_finest32) {
                    launch_convert<float, double>(tf.Bhat, td.Bhat, c->n_obs * (long)c->L * c->r, st);
                    launched += 1;
                }
                break;
            case MRA_KERNEL_POSTERIOR_LEVEL:
                launch_posterior_level<double>(c->geom, td, l.level, c->grid, predict, st);
                launched += 1;
                break;
            case MRA_KERNEL_REDUCE:
                launch_reduce<double>(td, c->d_result, st);
                launched += 1;
                break;
        }
        CU(record(c->tev[2 * i + 1], st, capturing));
        ++i;
    }
    if (predict) {
        c->timed_plan.push_back(-1);
        CU(record(c->tev[2 * i], st, capturing));
        if (mixed) {
            launch_convert<double, float>(td.Lpost, tf.Lpost, c->n_int * rr, st);
            launch_convert<double, float>(td.G, tf.G, c->u_total, st);
            launch_predict<float>(c->geom, tf, c->grid, st);
            launched += 3;
        } else {
            launch_predict<double>(c->geom, td, c->grid, st);
            launched += 1;
        }
        CU(record(c->tev[2 * i + 1], st, capturing));
        ++i;
    }
    CU(cudaGetLastError());
    c->n_timed = i;
    c->n_cov = cov.used;
    c->cov_overflow = cov.overflow;
    c->last_launches = launched;
    return MRA_OK;
}

int* err_ptr(mra_ctx* c) { return c->td.err; }

mra_status finish_eval(mra_ctx* c) {
    CU(cudaStreamSynchronize(c->stream));
    int err[4];
    double d;
    CU(cudaMemcpy(err, err_ptr(c), sizeof(err), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&d, c->d_result, sizeof(double), cudaMemcpyDeviceToHost));
    mra_stats& s = c->stats;
    s.ms_fields = s.ms_prior = s.ms_finest = s.ms_posterior = s.ms_predict = s.ms_total = 0;
    s.n_timed = c->n_timed;
    for (int i = 0; i < c->n_timed; ++i) {
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, c->tev[2 * i], c->tev[2 * i + 1]));
        const int pi = i < (int)c->timed_plan.size() ? c->timed_plan[i] : -1;
        const bool in_plan = pi >= 0;
        int kind = in_plan ? c->plan[pi].kind : MRA_KERNEL_PREDICT;
        s.timed_kind[i] = kind;
        s.timed_level[i] = in_plan ? c->plan[pi].level : -1;
        s.timed_flop[i] = in_plan ? c->plan[pi].flop : c->flop_predict_launch;
        s.timed_ms[i] = ms;
        s.timed_ms_cov[i] = 0;
        s.ms_total += ms;
        if (kind == MRA_KERNEL_FIELDS) s.ms_fields += ms;
        else if (kind == MRA_KERNEL_PRIOR_LEVEL) s.ms_prior += ms;
        else if (kind == MRA_KERNEL_FINEST) s.ms_finest += ms;
        else if (kind == MRA_KERNEL_PREDICT) s.ms_predict += ms;
        else s.ms_posterior += ms;
    }
    for (int k = 0; k < c->n_cov; ++k) {
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, c->cev[2 * k], c->cev[2 * k + 1]));
        if (c->cov_owner[k] < c->n_timed) s.timed_ms_cov[c->cov_owner[k]] += ms;
    }
    if (c->cov_overflow)  // some covariance launches went untimed: the split is unknown
        for (int i = 0; i < c->n_timed; ++i)
            if (s.timed_kind[i] == MRA_KERNEL_PRIOR_LEVEL) s.timed_ms_cov[i] = -1;
    s.d = d;
    s.loglik = -0.5 * (d + (double)c->n_obs * std::log(2 * 3.14159265359));
    s.flop_last = c->flop_loglik;
    s.flop_reference = c->flop_reference;
    s.bytes_device = c->bytes;
    s.kernel_launches = c->last_launches;
    s.bad_region = -1;
    if (err[0] == MRA_ERR_TIMEOUT)
        return fail(MRA_ERR_TIMEOUT, "a bounded device-side wait gave up");
    if (err[0] != 0) {
        s.bad_region = (int64_t)(unsigned)err[1] | ((int64_t)err[2] << 31);
        char buf[128];
        std::snprintf(buf, sizeof(buf), "Cholesky pivot not positive in region %lld", (long long)s.bad_region);
        return fail(MRA_ERR_NOT_SPD, buf);
    }
    return MRA_OK;
}

// Allocates the typed buffers of one precision and fills its DevTree.
// Shared FP64 vectors and bookkeeping used by both trees.
struct Shared {
    double *yt, *ldprior, *vpost, *dpost, *dfin, *mean, *var;
    int *queue, *err;
    int8_t* factored;
};

template <typename T>
mra_status setup_tree(mra_ctx* c, DevTree<T>& t, const HostTree& h, const PointSet& pts, const double* y,
                      int64_t* const* idx, int64_t u_total, const Shared& sh, bool prior_part, bool post_part,
                      bool pred_part) {
    const int J = c->J, M = c->M, r = c->r, L = c->L;
    const long rr = (long)r * r;
    cudaError_t ce = cudaSuccess;
    t.J = J; t.M = M; t.r = r; t.L = L; t.tf = c->tf;
    t.n_int = c->n_int; t.n_fin = c->n_fin; t.n_obs = c->n_obs; t.n_pred = c->n_pred;
    t.obs0 = c->n_int * r;
    t.pred0 = c->n_int * r + c->n_obs;
    t.pts = pts;
    t.y = y;
    t.obs_off = idx[0]; t.pred_off = idx[1]; t.fin_anc = idx[2]; t.pred_order = idx[3]; t.lsig_off = idx[4];
    t.pc_off = idx[5]; t.child_lo = idx[6]; t.child_hi = idx[7]; t.par_order = idx[8]; t.sub_lo = idx[9];
    t.sub_hi = idx[10];
    t.dslot = idx[11];
    t.post_order = idx[12];
    t.n_fin_items = (long)h.par_order.size();
    // sizes of the level-parity buffers
    size_t aout_sz[2] = {1, 1}, wout_sz[2] = {1, 1}, F_sz[2] = {1, 1}, f_sz[2] = {1, 1};
    for (int m = 1; m <= M - 2; ++m) {
        const long s0 = level_start(J, m), cnt = level_count(J, m);
        long n_dense = 0;
        bool any_fact = false;
        for (long q = 0; q < cnt; ++q) {
            if (h.factored[s0 + q]) any_fact = true;
            else ++n_dense;
        }
        if (n_dense > 0) {
            aout_sz[m & 1] = std::max(aout_sz[m & 1], (size_t)(n_dense * n_slices(m) * rr));
            wout_sz[m & 1] = std::max(wout_sz[m & 1], (size_t)(n_dense * m * r));
        }
        if (any_fact) {
            F_sz[m & 1] = std::max(F_sz[m & 1], (size_t)(c->n_obs * (long)m * r));
            f_sz[m & 1] = std::max(f_sz[m & 1], (size_t)c->n_obs);
        }
    }
    t.ws_stride = post_part ? std::max((long)r * c->tf + 2L * c->tf * c->tf, n_slices(M - 1) * rr + (long)(M - 2) * rr + rr) + 64
                            : 64;
    // prior: V of one conditioning step (r x r); finest: the inverse of a
    // child's L_Sigma (n x n, n <= 64), or a whole sibling group's conditional
    // covariance and block-diagonal inverse (2 x 64 x 64)
    if (prior_part) t.ws_stride = std::max(t.ws_stride, std::max(rr, 2L * 64 * 64) + 64);
    t.wsd_stride = post_part ? (long)(M - 1) * r + c->tf + 64 : 64;
    if (!post_part) {
        for (int p = 0; p < 2; ++p) aout_sz[p] = wout_sz[p] = F_sz[p] = f_sz[p] = 1;
    }
    const bool need_lpost_g = post_part || pred_part;
#define TALLOC(ptr, TYPE, n)                                                                          \
    do {                                                                                              \
        ptr = c->alloc<TYPE>((size_t)(n), &ce);                                                       \
        if (ce) return fail(MRA_ERR_OOM, std::string("device allocation failed: ") + #ptr);           \
    } while (0)
    TALLOC(t.Lprior, T, c->n_int * rr);
    TALLOC(t.Pinv, T, (prior_part || post_part) ? c->n_int * rr : 1);
    TALLOC(t.Bhat, T, c->n_obs * (long)L * r);
    TALLOC(t.U, T, prior_part ? u_total : 1);
    TALLOC(t.Ufin, T, prior_part ? c->n_obs * (long)L * r : 1);
    TALLOC(t.Lsig, T, prior_part ? h.lsig_off[c->n_fin] : 1);
    TALLOC(t.Lpost, T, need_lpost_g ? c->n_int * rr : 1);
    TALLOC(t.G, T, need_lpost_g && c->have_pred ? u_total : 1);
    // inverses of the posterior factors, so that prediction multiplies instead of solving
    t.Lpinv = nullptr;
    if (sizeof(T) == 8 && post_part && c->have_pred && r <= 64) TALLOC(t.Lpinv, T, c->n_int * rr);
    for (int p = 0; p < 2; ++p) {
        TALLOC(t.aout[p], T, aout_sz[p]);
        TALLOC(t.wout[p], double, wout_sz[p]);
        TALLOC(t.Fbuf[p], T, F_sz[p]);
        TALLOC(t.fbuf[p], double, f_sz[p]);
    }
    TALLOC(t.ws, T, (long)c->grid * t.ws_stride);
    // covariance blocks of the prior levels: all of a level's blocks when they
    // fit MRA_COV_BUF_MB (default 2048 MB; 8192 MB for the FP64 path when more
    // than 24 GB stay free: fewer chunks, fewer drained launches), else the
    // level runs in chunks of regions (a smaller buffer is tried when the first
    // allocation fails)
    t.cbuf = nullptr;
    t.cbuf_elems = 0;
    if (prior_part) {
        long need = 0;
        for (int m = 0; m <= M - 2; ++m) need = std::max(need, level_count(J, m) * (long)(m + 1) * rr);
        long cap_mb = 2048;
        size_t free_b = 0, total_b = 0;
        if (sizeof(T) == 8 && c->precision == MRA_PRECISION_FP64 && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
            free_b > (size_t)24 << 30)
            cap_mb = 8192;
        if (const char* e = std::getenv("MRA_COV_BUF_MB")) cap_mb = std::max(1L, std::atol(e));
        long elems = std::min(need, cap_mb * (1L << 20) / (long)sizeof(T));
        const long floor_elems = std::min(need, (long)(M - 1) * rr * c->grid);  // one region per CTA slot
        elems = std::max(elems, floor_elems);
        for (;;) {
            cudaError_t e2 = cudaSuccess;
            t.cbuf = c->alloc<T>((size_t)elems, &e2);
            if (!e2) break;
            cudaGetLastError();
            if (elems <= floor_elems) return fail(MRA_ERR_OOM, "device allocation failed: t.cbuf");
            elems = std::max(floor_elems, elems / 4);
        }
        t.cbuf_elems = elems;
    }
    TALLOC(t.wsd, double, (long)c->grid * t.wsd_stride);
    TALLOC(t.P, T, pred_part ? c->n_pred * (long)L * r : 1);
    TALLOC(t.Bt, T, pred_part ? c->n_pred * (long)L * r : 1);
    TALLOC(t.Pc, T, pred_part ? h.pc_off[c->n_fin] : 1);
#undef TALLOC
    t.yt = sh.yt;
    t.ldprior = sh.ldprior;
    t.vpost = sh.vpost;
    t.dpost = sh.dpost;
    t.dfin = sh.dfin;
    t.mean = sh.mean;
    t.var = sh.var;
    t.queue = sh.queue;
    t.err = sh.err;
    t.factored = sh.factored;
    t.active = nullptr;
    t.fuse_post = (prior_part && post_part) ? 1 : 0;
    int64_t uo = 0;
    for (int m = 0; m < kMaxLevels; ++m) t.u_off[m] = 0;
    for (int m = 0; m <= M - 2; ++m) {
        t.u_off[m] = uo;
        uo += level_count(J, m) * (int64_t)m * r * r;
    }
    (void)u_total;
    return MRA_OK;
}

}  // namespace

extern "C" {

const char* mra_last_error(void) { return g_last_error.c_str(); }

mra_status mra_set_device(int32_t device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
        return fail(MRA_ERR_NO_DEVICE, "no such CUDA device");
    CU(cudaSetDevice(device));
    return MRA_OK;
}

mra_status mra_create(const mra_structure* s, const mra_model* m, int32_t precision, mra_ctx** out) {
    if (!out) return fail(MRA_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!s) return fail(MRA_ERR_ARG, "structure is NULL");
    mra_status ms = check_model(m);
    if (ms != MRA_OK) return ms;
    if (s->J != 2 && s->J != 4) return fail(MRA_ERR_ARG, "J must be 2 or 4");
    if (s->M < 2 || s->M > kMaxLevels) return fail(MRA_ERR_ARG, "M must be in [2, 16]");
    if (s->r < 1 || s->r > 256) return fail(MRA_ERR_ARG, "r must be in [1, 256]");
    if (precision != MRA_PRECISION_FP64 && precision != MRA_PRECISION_MIXED)
        return fail(MRA_ERR_ARG, "unknown precision");
    const int J = s->J, M = s->M, r = s->r, L = M - 1;
    const long n_int = level_start(J, M - 1);
    if ((long)s->n_interior != n_int) return fail(MRA_ERR_ARG, "n_interior must equal (J^(M-1)-1)/(J-1)");
    const long n_fin = (long)s->n_finest;
    if (n_fin < 1 || !s->finest_parent || !s->knots || !s->obs_offset)
        return fail(MRA_ERR_ARG, "structure arrays are NULL or empty");
    if (s->obs_offset[0] != 0) return fail(MRA_ERR_ARG, "obs_offset[0] must be 0");
    const long n_obs = (long)s->obs_offset[n_fin];
    if (n_obs > 0 && (!s->obs || !s->obs_value)) return fail(MRA_ERR_ARG, "observation arrays are NULL");
    const long lvl2 = level_start(J, M - 2), cnt2 = level_count(J, M - 2);
    HostTree h;
    h.nfin.assign(n_fin, 0);
    h.npred.assign(n_fin, 0);
    h.child_lo.assign(cnt2, -1);
    h.child_hi.assign(cnt2, -1);
    long prev_parent = -1;
    for (long k = 0; k < n_fin; ++k) {
        if (s->obs_offset[k + 1] < s->obs_offset[k]) return fail(MRA_ERR_ARG, "obs_offset must be non-decreasing");
        h.nfin[k] = (int64_t)(s->obs_offset[k + 1] - s->obs_offset[k]);
        long p = (long)s->finest_parent[k];
        if (p < lvl2 || p >= lvl2 + cnt2) return fail(MRA_ERR_ARG, "finest_parent must be a level M-2 region");
        if (p < prev_parent)
            return fail(MRA_ERR_ARG, "finest regions must be ordered by parent (children of a region contiguous)");
        prev_parent = p;
        long q = p - lvl2;
        if (h.child_lo[q] < 0) h.child_lo[q] = k;
        h.child_hi[q] = k + 1;
    }
    for (long q = 0; q < cnt2; ++q)
        if (h.child_lo[q] < 0) h.child_lo[q] = h.child_hi[q] = 0;
    long n_pred = 0;
    const bool have_pred_arr = s->pred_offset != nullptr;
    if (have_pred_arr) {
        if (s->pred_offset[0] != 0) return fail(MRA_ERR_ARG, "pred_offset[0] must be 0");
        n_pred = (long)s->pred_offset[n_fin];
        if (n_pred > 0 && !s->pred) return fail(MRA_ERR_ARG, "prediction coordinates are NULL");
        for (long k = 0; k < n_fin; ++k) {
            if (s->pred_offset[k + 1] < s->pred_offset[k])
                return fail(MRA_ERR_ARG, "pred_offset must be non-decreasing");
            h.npred[k] = (int64_t)(s->pred_offset[k + 1] - s->pred_offset[k]);
        }
    }

    int dev = 0, count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(MRA_ERR_NO_DEVICE, "no CUDA device");
    CU(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) return fail(MRA_ERR_NO_DEVICE, "an sm_100 (B200) device is required");

    mra_ctx* c = new mra_ctx();
    auto bail = [&](mra_status st) {
        delete c;
        return st;
    };
    c->device = dev;
    c->precision = precision;
    c->sms = prop.multiProcessorCount;
    c->grid = 2 * c->sms;
    c->J = J; c->M = M; c->r = r; c->L = L;
    c->n_int = n_int; c->n_fin = n_fin; c->n_obs = n_obs; c->n_pred = n_pred;
    c->have_pred = have_pred_arr && n_pred > 0;
    c->tf = 2 * r;
    if (const char* e = std::getenv("MRA_FACTORED_MAX")) c->tf = std::max(0, std::atoi(e));
    c->geom = make_geom(m);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(MRA_ERR_CUDA, "stream creation failed"));
    if (cudaError_t pe = prepare_kernels(); pe != cudaSuccess)
        return bail(fail(MRA_ERR_CUDA, std::string("kernel attributes: ") + cudaGetErrorString(pe)));
    for (auto& e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return bail(fail(MRA_ERR_CUDA, "event creation failed"));
    for (auto& e : c->tev)
        if (cudaEventCreate(&e) != cudaSuccess) return bail(fail(MRA_ERR_CUDA, "event creation failed"));
    for (auto& e : c->cev)
        if (cudaEventCreate(&e) != cudaSuccess) return bail(fail(MRA_ERR_CUDA, "event creation failed"));

    // host-side tables
    h.obs_off.assign(n_fin + 1, 0);
    h.pred_off.assign(n_fin + 1, 0);
    h.fin_anc.assign(n_fin * L, 0);
    h.lsig_off.assign(n_fin + 1, 0);
    h.pc_off.assign(n_fin + 1, 0);
    for (long k = 0; k <= n_fin; ++k) {
        h.obs_off[k] = (int64_t)s->obs_offset[k];
        if (have_pred_arr) h.pred_off[k] = (int64_t)s->pred_offset[k];
    }
    for (long k = 0; k < n_fin; ++k) {
        long a = (long)s->finest_parent[k];
        h.fin_anc[k * L + L - 1] = a;
        for (int j = L - 2; j >= 0; --j) {
            a = (a - 1) / J;
            h.fin_anc[k * L + j] = a;
        }
        h.lsig_off[k + 1] = h.lsig_off[k] + h.nfin[k] * h.nfin[k];
        h.pc_off[k + 1] = h.pc_off[k] + h.nfin[k] * h.npred[k];
    }
    // prediction work items: level M-2 regions (their finest children together),
    // most expensive first
    {
        std::vector<double> cost(cnt2, 0.0);
        for (long k = 0; k < n_fin; ++k) {
            const long q = (long)s->finest_parent[k] - lvl2;
            cost[q] += (double)h.npred[k] * (double)(64L * L + h.nfin[k] + 1);
        }
        h.pred_order.resize(cnt2);
        for (long q = 0; q < cnt2; ++q) h.pred_order[q] = q;
        std::stable_sort(h.pred_order.begin(), h.pred_order.end(),
                         [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
    }
    // subtree observation ranges and the factored / dense decision per interior region
    h.sub_lo.assign(n_int, 0);
    h.sub_hi.assign(n_int, 0);
    h.factored.assign(n_int, 0);
    for (long q = 0; q < cnt2; ++q) {
        h.sub_lo[lvl2 + q] = h.obs_off[h.child_lo[q]];
        h.sub_hi[lvl2 + q] = h.child_hi[q] > h.child_lo[q] ? h.obs_off[h.child_hi[q]] : h.sub_lo[lvl2 + q];
    }
    for (int mm = M - 3; mm >= 0; --mm) {
        const long s0 = level_start(J, mm), cnt = level_count(J, mm);
        for (long q = 0; q < cnt; ++q) {
            long i = s0 + q, lo = -1, hi = -1;
            for (int cc = 1; cc <= J; ++cc) {
                long ch = i * J + cc;
                if (h.sub_hi[ch] > h.sub_lo[ch]) {
                    if (lo < 0) lo = h.sub_lo[ch];
                    hi = h.sub_hi[ch];
                }
            }
            h.sub_lo[i] = lo < 0 ? 0 : lo;
            h.sub_hi[i] = lo < 0 ? 0 : hi;
        }
    }
    for (long i = 0; i < n_int; ++i) h.factored[i] = (h.sub_hi[i] - h.sub_lo[i]) <= c->tf ? 1 : 0;
    c->h_factored = h.factored;
    c->h_sub_lo = h.sub_lo;
    c->h_sub_hi = h.sub_hi;
    // slot of each dense region among the dense regions of its level: the dense
    // outputs (A~ slices, w~) of a level are stored compactly
    h.dslot.assign(n_int, -1);
    for (int mm = 0; mm <= M - 2; ++mm) {
        const long s0 = level_start(J, mm), cnt = level_count(J, mm);
        long k = 0;
        for (long q = 0; q < cnt; ++q)
            if (!h.factored[s0 + q]) h.dslot[s0 + q] = k++;
    }
    c->h_dslot = h.dslot;
    // posterior work items of each level, most expensive first: a factored
    // region costs about n^2 (m r) for its n observations, a dense one the
    // accumulation of its factored children ((m+1) r)^2 per row plus its
    // r^3-sized step
    h.post_order.assign(n_int, 0);
    for (int mm = 0; mm <= M - 2; ++mm) {
        const long s0 = level_start(J, mm), cnt = level_count(J, mm);
        std::vector<double> cost(cnt);
        const double w = (double)(mm + 1) * r;
        for (long q = 0; q < cnt; ++q) {
            const long i = s0 + q;
            const double n = (double)(h.sub_hi[i] - h.sub_lo[i]);
            if (h.factored[i]) {
                cost[q] = n * n * (double)(mm * r) + n * (double)r * r;
            } else {
                double rows = 0.0;
                if (mm == M - 2) rows = n;
                else
                    for (int cc = 1; cc <= J; ++cc) {
                        const long ch = i * J + cc;
                        if (h.factored[ch]) rows += (double)(h.sub_hi[ch] - h.sub_lo[ch]);
                    }
                cost[q] = rows * w * w / 2 + (double)r * r * r * (0.5 * mm * mm + mm + 1.0);
            }
        }
        for (long q = 0; q < cnt; ++q) h.post_order[s0 + q] = q;
        std::stable_sort(h.post_order.begin() + s0, h.post_order.begin() + s0 + cnt,
                         [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
    }
    // work items of the finest kernel: a level M-3 region with its J sibling
    // groups when it holds at most 64 J observations (conditioning shared by
    // the groups), else each of its groups alone (load balance); for M = 2 the
    // single level-0 group.  Most expensive first.
    {
        const long n_units = M >= 3 ? level_count(J, M - 3) : 0;
        const long lvl3 = M >= 3 ? level_start(J, M - 3) : 0;
        long unit_max = 64L * J;  // observations of a unit processed as one item
        if (const char* e = std::getenv("MRA_UNIT_OBS_MAX")) unit_max = std::max(0L, std::atol(e));
        auto group_cost = [&](long gl) {
            const double n = (double)(h.sub_hi[lvl2 + gl] - h.sub_lo[lvl2 + gl]);
            return n * (n + 64.0 * L);
        };
        std::vector<std::pair<double, int64_t>> items;
        if (M >= 3) {
            for (long u = 0; u < n_units; ++u) {
                const long nu = h.sub_hi[lvl3 + u] - h.sub_lo[lvl3 + u];
                if (nu <= unit_max) {
                    double c = 0.0;
                    for (long gl = u * J; gl < u * J + J; ++gl) c += group_cost(gl);
                    items.push_back({c, (int64_t)u});
                } else {
                    for (long gl = u * J; gl < u * J + J; ++gl)
                        items.push_back({group_cost(gl), (int64_t)(n_units + gl)});
                }
            }
        } else {
            items.push_back({group_cost(0), 0});
        }
        std::stable_sort(items.begin(), items.end(),
                         [](const std::pair<double, int64_t>& x, const std::pair<double, int64_t>& y) {
                             return x.first > y.first;
                         });
        h.par_order.resize(items.size());
        for (size_t q = 0; q < items.size(); ++q) h.par_order[q] = items[q].second;
    }
    int64_t u_total = 0;
    for (int mm = 0; mm <= M - 2; ++mm) u_total += level_count(J, mm) * (int64_t)mm * r * r;

    // shared device arrays: coordinates, fields, observations, index tables
    cudaError_t ce = cudaSuccess;
    const long np_all = n_int * r + n_obs + n_pred;
    double* pc[3];
    double* fields[3];
    for (int d = 0; d < 3; ++d) {
        pc[d] = c->alloc<double>(np_all, &ce);
        if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed: coordinates"));
        fields[d] = c->alloc<double>(np_all, &ce);
        if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed: fields"));
    }
    double* y = c->alloc<double>(n_obs, &ce);
    if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed: y"));
    const std::vector<int64_t>* tabs[13] = {&h.obs_off, &h.pred_off, &h.fin_anc, &h.pred_order, &h.lsig_off,
                                            &h.pc_off, &h.child_lo, &h.child_hi, &h.par_order, &h.sub_lo, &h.sub_hi,
                                            &h.dslot, &h.post_order};
    int64_t* idx[13];
    for (int q = 0; q < 13; ++q) {
        idx[q] = c->alloc<int64_t>(tabs[q]->size(), &ce);
        if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed: index tables"));
        mra_status u = upload(idx[q], tabs[q]->data(), tabs[q]->size() * sizeof(int64_t), c->stream);
        if (u) return bail(u);
    }
    c->d_theta = c->alloc<double>(16, &ce);
    if (!ce) c->d_result = c->alloc<double>(4, &ce);
    if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed"));
    for (int f = 0; f < 3; ++f) {
        c->nb[f] = m->nonstationary ? (long)m->field[f].n_basis : 0;
        double* centers = c->alloc<double>(3 * c->nb[f], &ce);
        if (!ce) c->d_weights[f] = c->alloc<double>(c->nb[f], &ce);
        if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed: basis"));
        c->model_weights[f].assign(m->nonstationary && c->nb[f] ? m->field[f].weights : nullptr,
                                   m->nonstationary && c->nb[f] ? m->field[f].weights + c->nb[f] : nullptr);
        c->model_intercept[f] = m->nonstationary ? m->field[f].intercept : 0.0;
        if (c->nb[f]) {
            mra_status u = upload(centers, m->field[f].centers, 3 * c->nb[f] * sizeof(double), c->stream);
            if (!u) u = upload(c->d_weights[f], m->field[f].weights, c->nb[f] * sizeof(double), c->stream);
            if (u) return bail(u);
        }
        c->fp.nb[f] = c->nb[f];
        c->fp.centers[f] = centers;
        c->fp.weights[f] = c->d_weights[f];
    }
    c->fp.basis = m->basis;
    c->fp.basis_len = m->basis_len;
    c->fp.theta = c->d_theta;
    PointSet pts{pc[0], pc[1], pc[2], fields[0], fields[1], fields[2]};
    Shared sh{};
    sh.yt = c->alloc<double>(n_obs, &ce);
    if (!ce) sh.ldprior = c->alloc<double>(n_int, &ce);
    if (!ce) sh.vpost = c->alloc<double>(n_int * r, &ce);
    if (!ce) sh.dpost = c->alloc<double>(n_int, &ce);
    if (!ce) sh.dfin = c->alloc<double>(cnt2, &ce);
    if (!ce) sh.mean = c->alloc<double>(n_pred, &ce);
    if (!ce) sh.var = c->alloc<double>(n_pred, &ce);
    if (!ce) sh.queue = c->alloc<int>(kQueueCounters, &ce);
    if (!ce) sh.err = c->alloc<int>(4, &ce);
    if (!ce) sh.factored = c->alloc<int8_t>(n_int, &ce);
    if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed: shared vectors"));
    {
        mra_status u = upload(sh.factored, h.factored.data(), n_int * sizeof(int8_t), c->stream);
        if (u) return bail(u);
        CU(cudaMemsetAsync(sh.dpost, 0, n_int * sizeof(double), c->stream));
    }
    c->u_total = u_total;
    mra_status st;
    if (precision == MRA_PRECISION_MIXED) {
        if (const char* e = std::getenv("MRA_MIXED_FP32")) {
            const std::string v(e);
            c->mixed_prior32 = v.find("prior") != std::string::npos;
            c->mixed_finest32 = v.find("finest") != std::string::npos;
        }
        const bool both = c->mixed_prior32 && c->mixed_finest32;
        st = setup_tree<float>(c, c->tf32, h, pts, y, idx, u_total, sh, true, false, c->have_pred);
        if (!st) st = setup_tree<double>(c, c->td, h, pts, y, idx, u_total, sh, !both, true, false);
        c->td.fuse_post = 0;  // the plan runs the level M-2 posterior on its own
    } else {
        st = setup_tree<double>(c, c->td, h, pts, y, idx, u_total, sh, true, true, c->have_pred);
    }
    if (st) return bail(st);
    make_plan(c, h);
    {
        double R = r, fl = 0;
        for (long k = 0; k < n_fin; ++k) {
            double np = (double)h.npred[k], n = (double)h.nfin[k];
            fl += np * (L * R * R * (L - 1) / 2 + L * R * R / 2 + n * L * R + n * n / 2 + L * R * n + L * R * R / 2 +
                        L * (L - 1) / 2 * R * R);
        }
        c->flop_predict_launch = 2 * fl;
    }
    // upload the structure (coordinates: knots | obs | preds per coordinate)
    for (int d = 0; d < 3; ++d) {
        mra_status u = upload(pc[d], s->knots + (size_t)d * n_int * r, n_int * r * sizeof(double), c->stream);
        if (!u && n_obs) u = upload(pc[d] + n_int * r, s->obs + (size_t)d * n_obs, n_obs * sizeof(double), c->stream);
        if (!u && n_pred)
            u = upload(pc[d] + n_int * r + n_obs, s->pred + (size_t)d * n_pred, n_pred * sizeof(double), c->stream);
        if (u) return bail(u);
    }
    {
        mra_status u = upload(y, s->obs_value, n_obs * sizeof(double), c->stream);
        if (u) return bail(u);
    }
    double th0[16] = {1, 1, 1, c->model_intercept[0], c->model_intercept[1], c->model_intercept[2], 1, 1, 0};
    {
        mra_status u = upload(c->d_theta, th0, sizeof(th0), c->stream);
        if (u) return bail(u);
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(MRA_ERR_CUDA, "upload failed"));
    *out = c;
    return MRA_OK;
}

mra_status mra_destroy(mra_ctx* ctx) {
    delete ctx;
    return MRA_OK;
}

mra_status mra_set_theta(mra_ctx* c, const mra_theta* th) {
    if (!c || !th) return fail(MRA_ERR_ARG, "NULL argument");
    double v[16] = {0};
    if (c->geom.nonstat) {
        v[0] = th->sill_scale; v[1] = th->range_scale; v[2] = th->nugget_scale;
        if (!(v[0] > 0 && v[1] > 0 && v[2] > 0)) return fail(MRA_ERR_ARG, "scales must be positive");
    }
    for (int f = 0; f < 3; ++f) v[3 + f] = th->intercepts ? th->intercepts[f] : c->model_intercept[f];
    v[6] = th->sill; v[7] = th->range; v[8] = th->nugget;
    if (!c->geom.nonstat && !(v[6] > 0 && v[7] > 0 && v[8] >= 0))
        return fail(MRA_ERR_ARG, "sill and range must be positive, nugget non-negative");
    for (int f = 3; f < 6; ++f)
        if (!std::isfinite(v[f])) return fail(MRA_ERR_ARG, "intercepts must be finite");
    CU(cudaMemcpyAsync(c->d_theta, v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
    for (int f = 0; f < 3; ++f) {
        if (!c->nb[f]) continue;
        const double* w = th->weights[f] ? th->weights[f] : c->model_weights[f].data();
        CU(cudaMemcpyAsync(c->d_weights[f], w, c->nb[f] * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    return MRA_OK;
}

mra_status mra_set_obs_values(mra_ctx* c, const double* y) {
    if (!c || (!y && c->n_obs)) return fail(MRA_ERR_ARG, "NULL argument");
    const double* dy = c->td.y;
    CU(cudaMemcpyAsync(const_cast<double*>(dy), y, c->n_obs * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    return MRA_OK;
}

mra_status mra_loglik(mra_ctx* c, double* d_out, double* ll_out) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    if (c->shard_split) return fail(MRA_ERR_STATE, "the context is sharded: use mra_shard_* (or clear the sharding)");
    if (c->graph_exec) {
        CU(cudaGraphLaunch(c->graph_exec, c->stream));
        c->stats.graph_replays++;
        c->n_timed = c->graph_timed[0];
        c->n_cov = c->graph_cov[0];
        c->last_launches = c->graph_launches[0];
    } else {
        mra_status s = run_eval(c, false);
        if (s) return s;
    }
    mra_status s = finish_eval(c);
    if (d_out) *d_out = c->stats.d;
    if (ll_out) *ll_out = c->stats.loglik;
    return s;
}

mra_status mra_predict(mra_ctx* c, double* mean, double* var) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    if (!c->have_pred) return fail(MRA_ERR_STATE, "the structure has no prediction locations");
    if (c->shard_split) return fail(MRA_ERR_STATE, "prediction is not sharded: clear the sharding first");
    if (!(c->mixed_prior32 && c->mixed_finest32))
        return fail(MRA_ERR_STATE, "prediction needs the mixed path with both FP32 stages (MRA_MIXED_FP32)");
    if (c->graph_pred_exec) {
        CU(cudaGraphLaunch(c->graph_pred_exec, c->stream));
        c->stats.graph_replays++;
        c->n_timed = c->graph_timed[1];
        c->n_cov = c->graph_cov[1];
        c->last_launches = c->graph_launches[1];
    } else {
        mra_status s = run_eval(c, true);
        if (s) return s;
    }
    mra_status s = finish_eval(c);
    if (s) return s;
    const double* dm = c->td.mean;
    const double* dv = c->td.var;
    if (mean) CU(cudaMemcpy(mean, dm, c->n_pred * sizeof(double), cudaMemcpyDeviceToHost));
    if (var) CU(cudaMemcpy(var, dv, c->n_pred * sizeof(double), cudaMemcpyDeviceToHost));
    return MRA_OK;
}

namespace {

// Captures one evaluation sequence (log-likelihood, or log-likelihood with the
// predictive factors kept followed by prediction) from the context's stream.
mra_status capture_one(mra_ctx* c, bool predict, cudaGraph_t* graph, cudaGraphExec_t* exec) {
    CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    mra_status s = run_eval(c, predict);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (s) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return fail(MRA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    cudaError_t ie = cudaGraphInstantiate(exec, g, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(g);
        *exec = nullptr;
        return fail(MRA_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    *graph = g;
    c->graph_timed[predict ? 1 : 0] = c->n_timed;
    c->graph_launches[predict ? 1 : 0] = c->last_launches;
    c->graph_cov[predict ? 1 : 0] = c->n_cov;
    return MRA_OK;
}

}  // namespace

mra_status mra_capture_graph(mra_ctx* c) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    if (c->shard_split) return fail(MRA_ERR_STATE, "sharded evaluations are not captured");
    if (!c->graph_exec) {
        mra_status s = capture_one(c, false, &c->graph, &c->graph_exec);
        if (s) return s;
    }
    if (c->have_pred && !c->graph_pred_exec) {
        mra_status s = capture_one(c, true, &c->graph_pred, &c->graph_pred_exec);
        if (s) return s;
    }
    return MRA_OK;
}

// ---------------------------------------------------------------------------
// sub-tree sharding
// ---------------------------------------------------------------------------
namespace {

long shard_pow(int J, int e) { return level_count(J, e); }

// doubles of the export record of one split-level region (see mra_b200.h)
long shard_record_doubles(const mra_ctx* c, long q) {
    const int s = c->shard_split, r = c->r;
    const long i = level_start(c->J, s) + q;
    const long rr = (long)r * r;
    long n = 2;
    if (c->h_factored[i]) {
        const long rows = c->h_sub_hi[i] - c->h_sub_lo[i];
        n += rows * (long)s * r + rows;
    } else {
        n += n_slices(s) * rr + (long)s * r;
    }
    for (int m = s; m <= c->M - 2; ++m) n += shard_pow(c->J, m - s);  // posterior terms of the sub-tree
    n += shard_pow(c->J, c->M - 2 - s);                                 // finest terms of its groups
    return n;
}

// copies between a record and the device buffers (to_device: import)
mra_status shard_copy(mra_ctx* c, long q, double* rec, bool to_device) {
    const int s = c->shard_split, r = c->r, J = c->J;
    const long i = level_start(J, s) + q;
    const long rr = (long)r * r;
    DevTree<double>& t = c->td;
    const cudaMemcpyKind k = to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    auto cp = [&](double* dev, double* host, long n) -> cudaError_t {
        if (n <= 0) return cudaSuccess;
        return to_device ? cudaMemcpy(dev, host, n * sizeof(double), k) : cudaMemcpy(host, dev, n * sizeof(double), k);
    };
    const double kind = c->h_factored[i] ? 1.0 : 0.0;
    const long rows = c->h_sub_hi[i] - c->h_sub_lo[i];
    if (to_device) {
        if (rec[0] != kind || (kind == 1.0 && rec[1] != (double)rows))
            return fail(MRA_ERR_ARG, "mra_shard_import: the record does not match this structure");
    } else {
        rec[0] = kind;
        rec[1] = kind == 1.0 ? (double)rows : 0.0;
    }
    double* p = rec + 2;
    if (kind == 1.0) {
        const long lo = c->h_sub_lo[i];
        CU(cp(t.Fbuf[s & 1] + lo * (long)s * r, p, rows * (long)s * r));
        p += rows * (long)s * r;
        CU(cp(t.fbuf[s & 1] + lo, p, rows));
        p += rows;
    } else {
        const long slot = c->h_dslot[i];
        CU(cp(t.aout[s & 1] + slot * n_slices(s) * rr, p, n_slices(s) * rr));
        p += n_slices(s) * rr;
        CU(cp(t.wout[s & 1] + slot * (long)s * r, p, (long)s * r));
        p += (long)s * r;
    }
    for (int m = s; m <= c->M - 2; ++m) {
        const long w = shard_pow(J, m - s);
        CU(cp(t.dpost + level_start(J, m) + q * w, p, w));
        p += w;
    }
    const long wg = shard_pow(J, c->M - 2 - s);
    CU(cp(t.dfin + q * wg, p, wg));
    return MRA_OK;
}

mra_status shard_run(mra_ctx* c, int phase) {
    c->eval_phase = phase;
    mra_status s = run_eval(c, false);
    c->eval_phase = 0;
    if (s) return s;
    return finish_eval(c);
}

}  // namespace

mra_status mra_shard_set(mra_ctx* c, int32_t split_level, const uint8_t* owned) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    if (!owned) {
        c->shard_split = 0;
        c->td.active = nullptr;
        return MRA_OK;
    }
    if (c->precision != MRA_PRECISION_FP64) return fail(MRA_ERR_ARG, "sharding runs the FP64 path only");
    if (c->M < 4 || split_level < 1 || split_level > c->M - 3)
        return fail(MRA_ERR_ARG, "the split level must be in [1, M-3] (M >= 4)");
    const int J = c->J, s = split_level;
    std::vector<int8_t> act(c->n_int, 1);
    for (int m = s; m <= c->M - 2; ++m) {
        const long s0 = level_start(J, m), cnt = level_count(J, m), w = shard_pow(J, m - s);
        for (long q = 0; q < cnt; ++q) act[s0 + q] = owned[q / w] ? 1 : 0;
    }
    if (!c->d_active) {
        cudaError_t e = cudaSuccess;
        c->d_active = c->alloc<int8_t>(c->n_int, &e);
        if (e) return fail(MRA_ERR_OOM, "device allocation failed: sharding mask");
    }
    CU(cudaMemcpy(c->d_active, act.data(), c->n_int, cudaMemcpyHostToDevice));
    c->shard_split = s;
    c->td.active = c->d_active;
    return MRA_OK;
}

mra_status mra_shard_loglik_subtrees(mra_ctx* c) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    if (!c->shard_split) return fail(MRA_ERR_STATE, "mra_shard_set first");
    return shard_run(c, 1);
}

mra_status mra_shard_record_size(const mra_ctx* c, uint64_t region, uint64_t* n_doubles) {
    if (!c || !n_doubles) return fail(MRA_ERR_ARG, "NULL argument");
    if (!c->shard_split) return fail(MRA_ERR_STATE, "mra_shard_set first");
    if ((long)region >= level_count(c->J, c->shard_split)) return fail(MRA_ERR_ARG, "region out of range");
    *n_doubles = (uint64_t)shard_record_doubles(c, (long)region);
    return MRA_OK;
}

mra_status mra_shard_export(mra_ctx* c, uint64_t region, double* record, uint64_t n_doubles) {
    if (!c || !record) return fail(MRA_ERR_ARG, "NULL argument");
    if (!c->shard_split) return fail(MRA_ERR_STATE, "mra_shard_set first");
    if ((long)region >= level_count(c->J, c->shard_split)) return fail(MRA_ERR_ARG, "region out of range");
    if ((long)n_doubles != shard_record_doubles(c, (long)region)) return fail(MRA_ERR_ARG, "record size mismatch");
    CU(cudaStreamSynchronize(c->stream));
    return shard_copy(c, (long)region, record, false);
}

mra_status mra_shard_import(mra_ctx* c, uint64_t region, const double* record, uint64_t n_doubles) {
    if (!c || !record) return fail(MRA_ERR_ARG, "NULL argument");
    if (!c->shard_split) return fail(MRA_ERR_STATE, "mra_shard_set first");
    if ((long)region >= level_count(c->J, c->shard_split)) return fail(MRA_ERR_ARG, "region out of range");
    if ((long)n_doubles != shard_record_doubles(c, (long)region)) return fail(MRA_ERR_ARG, "record size mismatch");
    CU(cudaStreamSynchronize(c->stream));
    return shard_copy(c, (long)region, const_cast<double*>(record), true);
}

mra_status mra_shard_loglik_top(mra_ctx* c, double* d_out, double* ll_out) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    if (!c->shard_split) return fail(MRA_ERR_STATE, "mra_shard_set first");
    mra_status s = shard_run(c, 2);
    if (d_out) *d_out = c->stats.d;
    if (ll_out) *ll_out = c->stats.loglik;
    return s;
}

mra_status mra_get_terms(mra_ctx* c, double* out, int32_t n_out) {
    if (!c || !out) return fail(MRA_ERR_ARG, "NULL argument");
    if (n_out < c->M) return fail(MRA_ERR_ARG, "mra_get_terms: n_out must be at least M");
    CU(cudaStreamSynchronize(c->stream));
    std::vector<double> dpost(c->n_int), dfin(level_count(c->J, c->M - 2));
    CU(cudaMemcpy(dpost.data(), c->td.dpost, dpost.size() * sizeof(double), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(dfin.data(), c->td.dfin, dfin.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int m = 0; m < c->M; ++m) out[m] = 0.0;
    for (int m = 0; m <= c->M - 2; ++m) {
        const long s0 = level_start(c->J, m), cnt = level_count(c->J, m);
        for (long q = 0; q < cnt; ++q) out[m] += dpost[s0 + q];
    }
    for (double v : dfin) out[c->M - 1] += v;
    return MRA_OK;
}

mra_status mra_get_stats(const mra_ctx* c, mra_stats* out) {
    if (!c || !out) return fail(MRA_ERR_ARG, "NULL argument");
    *out = c->stats;
    out->bytes_device = c->bytes;
    out->flop_last = c->flop_loglik;
    out->flop_reference = c->flop_reference;
    return MRA_OK;
}

mra_status mra_timer_start(mra_ctx* c) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    CU(cudaEventRecord(c->ev[6], c->stream));
    return MRA_OK;
}

mra_status mra_timer_stop(mra_ctx* c, double* ms) {
    if (!c || !ms) return fail(MRA_ERR_ARG, "NULL argument");
    CU(cudaEventRecord(c->ev[7], c->stream));
    CU(cudaEventSynchronize(c->ev[7]));
    float f = 0;
    CU(cudaEventElapsedTime(&f, c->ev[6], c->ev[7]));
    *ms = f;
    return MRA_OK;
}

mra_status mra_autotune(mra_ctx* c, int32_t evals, int32_t* choice_out, double* ms_out) {
    if (!c || evals < 1) return fail(MRA_ERR_ARG, "mra_autotune: NULL context or evals < 1");
    // candidate FP64 tile widths per product-width bucket (N <= 16, <= 32, wider)
    static const int cand[][3] = {{1, 2, 4}, {1, 2, 2}, {1, 4, 4}, {2, 2, 4}, {1, 1, 4}, {2, 4, 4}};
    const int nc = (int)(sizeof(cand) / sizeof(cand[0]));
    double best = 1e300;
    int ib = 0;
    for (int k = 0; k < nc; ++k) {
        CU(set_gemm_tiles(cand[k]));
        double d, ll, ms = 0.0;
        mra_status st = mra_loglik(c, &d, &ll);  // warm-up with this choice
        if (st != MRA_OK) return st;
        st = mra_timer_start(c);
        if (st != MRA_OK) return st;
        for (int e = 0; e < evals; ++e) {
            st = mra_loglik(c, &d, &ll);
            if (st != MRA_OK) return st;
        }
        st = mra_timer_stop(c, &ms);
        if (st != MRA_OK) return st;
        if (ms < best) best = ms, ib = k;
    }
    CU(set_gemm_tiles(cand[ib]));
    if (choice_out)
        for (int b = 0; b < 3; ++b) choice_out[b] = cand[ib][b];
    if (ms_out) *ms_out = best / evals;
    return MRA_OK;
}

mra_status mra_sample_prior(mra_ctx* c, const double* z_int, const double* z_obs, double* y_out) {
    if (!c || !z_int || (!z_obs && c->n_obs) || (!y_out && c->n_obs)) return fail(MRA_ERR_ARG, "NULL argument");
    if (!(c->mixed_prior32 && c->mixed_finest32))
        return fail(MRA_ERR_STATE, "sampling needs the mixed path with both FP32 stages (MRA_MIXED_FP32)");
    if (c->shard_split) return fail(MRA_ERR_STATE, "sampling is not sharded: clear the sharding first");
    // the prior factors (U of the finest level, L_Sigma) come from one evaluation
    mra_status s = run_eval(c, false);
    if (s) return s;
    s = finish_eval(c);
    if (s) return s;
    double *dz = nullptr, *dzo = nullptr, *dy = nullptr;
    size_t nzi = (size_t)c->n_int * c->r;
    cudaError_t e = cudaMalloc(&dz, nzi * sizeof(double));
    if (!e) e = cudaMalloc(&dzo, std::max<size_t>(c->n_obs, 1) * sizeof(double));
    if (!e) e = cudaMalloc(&dy, std::max<size_t>(c->n_obs, 1) * sizeof(double));
    if (!e) e = cudaMemcpy(dz, z_int, nzi * sizeof(double), cudaMemcpyHostToDevice);
    if (!e && c->n_obs) e = cudaMemcpy(dzo, z_obs, c->n_obs * sizeof(double), cudaMemcpyHostToDevice);
    if (!e) {
        if (c->precision == MRA_PRECISION_MIXED) launch_sample<float>(c->tf32, dz, dzo, dy, c->grid, c->stream);
        else launch_sample<double>(c->td, dz, dzo, dy, c->grid, c->stream);
        e = cudaGetLastError();
    }
    if (!e) e = cudaStreamSynchronize(c->stream);
    if (!e && c->n_obs) e = cudaMemcpy(y_out, dy, c->n_obs * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dz);
    cudaFree(dzo);
    cudaFree(dy);
    if (e) return fail(e == cudaErrorMemoryAllocation ? MRA_ERR_OOM : MRA_ERR_CUDA, cudaGetErrorString(e));
    return MRA_OK;
}

// Standalone covariance / field evaluation (unit-level parity with the
// reference's evaluate_* and Nonstationary_covariance::get_*).
static mra_status eval_points(const mra_model* m, const mra_theta* th, const double* p, uint64_t n,
                              std::vector<void*>& frees, PointSet* ps, cudaStream_t st) {
    Geom g = make_geom(m);
    double *c[3], *f[3];
    for (int d = 0; d < 3; ++d) {
        CU(cudaMalloc(&c[d], std::max<uint64_t>(n, 1) * sizeof(double)));
        frees.push_back(c[d]);
        CU(cudaMalloc(&f[d], std::max<uint64_t>(n, 1) * sizeof(double)));
        frees.push_back(f[d]);
        if (n) CU(cudaMemcpyAsync(c[d], p + d * n, n * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    FieldParams fp{};
    fp.basis = m->basis;
    fp.basis_len = m->basis_len;
    double v[16] = {0};
    v[0] = th->sill_scale; v[1] = th->range_scale; v[2] = th->nugget_scale;
    v[6] = th->sill; v[7] = th->range; v[8] = th->nugget;
    double* dth;
    CU(cudaMalloc(&dth, sizeof(v)));
    frees.push_back(dth);
    for (int k = 0; k < 3; ++k) {
        long nb = m->nonstationary ? (long)m->field[k].n_basis : 0;
        v[3 + k] = th->intercepts ? th->intercepts[k] : (m->nonstationary ? m->field[k].intercept : 0.0);
        fp.nb[k] = nb;
        double *dc, *dw;
        CU(cudaMalloc(&dc, std::max<long>(3 * nb, 1) * sizeof(double)));
        frees.push_back(dc);
        CU(cudaMalloc(&dw, std::max<long>(nb, 1) * sizeof(double)));
        frees.push_back(dw);
        if (nb) {
            CU(cudaMemcpyAsync(dc, m->field[k].centers, 3 * nb * sizeof(double), cudaMemcpyHostToDevice, st));
            const double* w = th->weights[k] ? th->weights[k] : m->field[k].weights;
            CU(cudaMemcpyAsync(dw, w, nb * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        fp.centers[k] = dc;
        fp.weights[k] = dw;
    }
    CU(cudaMemcpyAsync(dth, v, sizeof(v), cudaMemcpyHostToDevice, st));
    fp.theta = dth;
    launch_fields(g, fp, c[0], c[1], c[2], (long)n, f[0], f[1], f[2], st);
    *ps = PointSet{c[0], c[1], c[2], f[0], f[1], f[2]};
    return MRA_OK;
}

mra_status mra_eval_fields(const mra_model* m, const mra_theta* th, const double* p, uint64_t n, double* out) {
    mra_status s = check_model(m);
    if (s) return s;
    if (!th || (!p && n) || (!out && n)) return fail(MRA_ERR_ARG, "NULL argument");
    std::vector<void*> frees;
    PointSet ps{};
    s = eval_points(m, th, p, n, frees, &ps, 0);
    if (!s) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e == cudaSuccess && n) {
            cudaMemcpy(out, ps.s2, n * sizeof(double), cudaMemcpyDeviceToHost);
            cudaMemcpy(out + n, ps.beta, n * sizeof(double), cudaMemcpyDeviceToHost);
            e = cudaMemcpy(out + 2 * n, ps.t2, n * sizeof(double), cudaMemcpyDeviceToHost);
        }
        if (e != cudaSuccess) s = fail(MRA_ERR_CUDA, cudaGetErrorString(e));
    }
    for (void* q : frees) cudaFree(q);
    return s;
}

mra_status mra_eval_covariance(const mra_model* m, const mra_theta* th, const double* p1, uint64_t n1,
                               const double* p2, uint64_t n2, int32_t self, double* out) {
    mra_status s = check_model(m);
    if (s) return s;
    if (!th || !p1 || (!self && !p2) || !out) return fail(MRA_ERR_ARG, "NULL argument");
    if (self) n2 = n1;
    std::vector<void*> frees;
    PointSet a{}, b{};
    s = eval_points(m, th, p1, n1, frees, &a, 0);
    if (!s && !self) s = eval_points(m, th, p2, n2, frees, &b, 0);
    if (!s) {
        double* d;
        cudaError_t e = cudaMalloc(&d, std::max<uint64_t>(n1 * n2, 1) * sizeof(double));
        if (e == cudaSuccess) {
            frees.push_back(d);
            if (self) {
                launch_cov_block(make_geom(m), a, 0, (int)n1, 0, (int)n1, true, d, 0);
            } else {
                // one point set with both: set 2 rows, set 1 columns (out[i1*n2 + i2])
                double* cc[6];
                for (int q = 0; q < 6 && e == cudaSuccess; ++q) {
                    e = cudaMalloc(&cc[q], std::max<uint64_t>(n1 + n2, 1) * sizeof(double));
                    if (e == cudaSuccess) frees.push_back(cc[q]);
                }
                const double* srcA[6] = {a.c0, a.c1, a.c2, a.s2, a.beta, a.t2};
                const double* srcB[6] = {b.c0, b.c1, b.c2, b.s2, b.beta, b.t2};
                for (int q = 0; q < 6 && e == cudaSuccess; ++q) {
                    if (n2) e = cudaMemcpy(cc[q], srcB[q], n2 * sizeof(double), cudaMemcpyDeviceToDevice);
                    if (e == cudaSuccess && n1)
                        e = cudaMemcpy(cc[q] + n2, srcA[q], n1 * sizeof(double), cudaMemcpyDeviceToDevice);
                }
                if (e == cudaSuccess) {
                    PointSet both{cc[0], cc[1], cc[2], cc[3], cc[4], cc[5]};
                    launch_cov_block(make_geom(m), both, 0, (int)n2, (long)n2, (int)n1, false, d, 0);
                }
            }
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaDeviceSynchronize();
            if (e == cudaSuccess && n1 > 0 && n2 > 0)
                e = cudaMemcpy(out, d, n1 * n2 * sizeof(double), cudaMemcpyDeviceToHost);
        }
        if (e != cudaSuccess) s = fail(MRA_ERR_CUDA, cudaGetErrorString(e));
    }
    for (void* q : frees) cudaFree(q);
    return s;
}

}  // extern "C"
