// C ABI of the MRA hot path (include/mra_b200.h): context lifetime, device
// residency of the partition, the per-evaluation launch sequence, CUDA-graph
// capture and statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
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
    int J = 0, M = 0, r = 0, L = 0;
    long n_int = 0, n_fin = 0, n_obs = 0, n_pred = 0;
    Geom geom{};
    FieldParams fp{};
    DevTree t{};
    std::vector<DevBuf> bufs;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8]{};
    cudaEvent_t tev[2 * MRA_MAX_TIMED]{};   // start/stop of every launch
    struct Launch {
        int kind, level;
        double flop;
    };
    std::vector<Launch> plan;               // launches of one log-likelihood, in order
    double flop_predict_launch = 0;
    int n_timed = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    double* d_theta = nullptr;  // 9 doubles
    double* d_weights[3]{};
    long nb[3]{};
    std::vector<double> model_weights[3];
    double model_intercept[3]{};
    double* d_result = nullptr;  // [0] d
    double flop_loglik = 0, flop_predict = 0;
    mra_stats stats{};
    int last_launches = 0;
    bool have_pred = false;

    template <typename T>
    T* alloc(size_t count, cudaError_t* err) {
        DevBuf b;
        b.bytes = std::max<size_t>(count * sizeof(T), 16);
        *err = cudaMalloc(&b.p, b.bytes);
        if (*err != cudaSuccess) return nullptr;
        bufs.push_back(b);
        bytes += b.bytes;
        return static_cast<T*>(b.p);
    }
    ~mra_ctx() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : tev)
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

mra_status check_model(const mra_model* m) {
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

// Algorithmic FLOPs (2 per multiply-add; symmetric products counted once) of
// every launch of one log-likelihood, from the realised region sizes.  The
// per-region multiply-add counts are the canonical ones of the MRA:
//   prior, level m:     r^3 [m(m-1)/2 + m/2 + m/2 + 1/6]
//   posterior, level m: r^3 [1/3 + m/2 + m/2 + m(m-1)/2] + r^2 (1/2 + m)
//   finest region, n observations, L = M-1 ancestors:
//     r^2 n L(L-1)/2 + L r^2 n/2 + L r n^2/2 + n^3/6 + n^2/2 + L n^2 r/2   (finest kernel)
//     L r n + L r^2 n/2 + L(L-1)/2 r^2 n     (w~ and A~ products; formed by the
//                                              level M-2 posterior kernel here)
void make_plan(mra_ctx* c, const std::vector<int64_t>& nfin) {
    const int J = c->J, M = c->M;
    const double R = c->r, Lv = M - 1;
    double fields = 0;
    for (int f = 0; f < 3; ++f) fields += (double)c->nb[f];
    c->plan.clear();
    c->plan.push_back({MRA_KERNEL_FIELDS, -1,
                       (double)(c->n_int * c->r + c->n_obs + c->n_pred) * (fields * 12 + 8)});
    for (int m = 0; m <= M - 2; ++m) {
        double cnt = std::pow((double)J, m), mm = m;
        c->plan.push_back({MRA_KERNEL_PRIOR_LEVEL, m,
                           2 * cnt * R * R * R * (mm * (mm - 1) / 2 + mm / 2 + mm / 2 + 1.0 / 6)});
    }
    double fin = 0, agg = 0;
    for (int64_t n64 : nfin) {
        double n = (double)n64;
        if (n == 0) continue;
        fin += R * R * n * Lv * (Lv - 1) / 2 + Lv * R * R * n / 2 + Lv * R * n * n / 2 + n * n * n / 6 + n * n / 2 +
               Lv * n * n * R / 2;
        agg += Lv * R * n + Lv * R * R * n / 2 + Lv * (Lv - 1) / 2 * R * R * n;
    }
    c->plan.push_back({MRA_KERNEL_FINEST, M - 1, 2 * fin});
    for (int m = M - 2; m >= 0; --m) {
        double cnt = std::pow((double)J, m), mm = m;
        double f = cnt * (R * R * R * (1.0 / 3 + mm / 2 + mm / 2 + mm * (mm - 1) / 2) + R * R * (0.5 + mm));
        if (m == M - 2) f += agg;
        c->plan.push_back({MRA_KERNEL_POSTERIOR_LEVEL, m, 2 * f});
    }
    c->plan.push_back({MRA_KERNEL_REDUCE, -1, (double)(c->n_int + c->n_fin)});
    c->flop_loglik = 0;
    for (auto& l : c->plan) c->flop_loglik += l.flop;
}

mra_status upload(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return MRA_OK;
    CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return MRA_OK;
}

// Issues one evaluation on the context's stream: every launch of the plan
// (plus prediction) bracketed by its own pair of timing events.  The events are
// recorded as external nodes so that they still time each launch when the
// sequence is replayed from a captured CUDA graph.
cudaError_t record(cudaEvent_t e, cudaStream_t st, bool capturing) {
    return capturing ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal) : cudaEventRecord(e, st);
}

mra_status run_eval(mra_ctx* c, bool predict) {
    cudaStream_t st = c->stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CU(cudaStreamIsCapturing(st, &cap));
    const bool capturing = cap == cudaStreamCaptureStatusActive;
    CU(cudaMemsetAsync(c->t.queue, 0, 4 * sizeof(int), st));
    CU(cudaMemsetAsync(c->t.err, 0, 4 * sizeof(int), st));
    const long np_all = c->n_int * c->r + c->n_obs + c->n_pred;
    int i = 0;
    for (const auto& l : c->plan) {
        CU(record(c->tev[2 * i], st, capturing));
        switch (l.kind) {
            case MRA_KERNEL_FIELDS:
                launch_fields(c->geom, c->fp, c->t.pts.c0, c->t.pts.c1, c->t.pts.c2, np_all,
                              const_cast<double*>(c->t.pts.s2), const_cast<double*>(c->t.pts.beta),
                              const_cast<double*>(c->t.pts.t2), st);
                break;
            case MRA_KERNEL_PRIOR_LEVEL: launch_prior_level(c->geom, c->t, l.level, c->grid, st); break;
            case MRA_KERNEL_FINEST: launch_finest(c->geom, c->t, c->grid, predict, st); break;
            case MRA_KERNEL_POSTERIOR_LEVEL:
                launch_posterior_level(c->geom, c->t, l.level, c->grid, predict, st);
                break;
            case MRA_KERNEL_REDUCE: launch_reduce(c->t, c->d_result, st); break;
        }
        CU(record(c->tev[2 * i + 1], st, capturing));
        ++i;
    }
    if (predict) {
        CU(record(c->tev[2 * i], st, capturing));
        launch_predict(c->geom, c->t, c->grid, st);
        CU(record(c->tev[2 * i + 1], st, capturing));
        ++i;
    }
    CU(cudaGetLastError());
    c->n_timed = i;
    c->last_launches = i;
    return MRA_OK;
}

mra_status finish_eval(mra_ctx* c, bool predict) {
    CU(cudaStreamSynchronize(c->stream));
    int err[4];
    double d;
    CU(cudaMemcpy(err, c->t.err, sizeof(err), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&d, c->d_result, sizeof(double), cudaMemcpyDeviceToHost));
    mra_stats& s = c->stats;
    s.ms_fields = s.ms_prior = s.ms_finest = s.ms_posterior = s.ms_predict = s.ms_total = 0;
    s.n_timed = c->n_timed;
    for (int i = 0; i < c->n_timed; ++i) {
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, c->tev[2 * i], c->tev[2 * i + 1]));
        int kind = i < (int)c->plan.size() ? c->plan[i].kind : MRA_KERNEL_PREDICT;
        s.timed_kind[i] = kind;
        s.timed_level[i] = i < (int)c->plan.size() ? c->plan[i].level : -1;
        s.timed_flop[i] = i < (int)c->plan.size() ? c->plan[i].flop : c->flop_predict_launch;
        s.timed_ms[i] = ms;
        s.ms_total += ms;
        if (kind == MRA_KERNEL_FIELDS) s.ms_fields += ms;
        else if (kind == MRA_KERNEL_PRIOR_LEVEL) s.ms_prior += ms;
        else if (kind == MRA_KERNEL_FINEST) s.ms_finest += ms;
        else if (kind == MRA_KERNEL_PREDICT) s.ms_predict += ms;
        else s.ms_posterior += ms;
    }
    s.d = d;
    s.loglik = -0.5 * (d + (double)c->n_obs * std::log(2 * 3.14159265359));
    s.flop_last = c->flop_loglik;
    s.bytes_device = c->bytes;
    s.kernel_launches = c->last_launches;
    s.bad_region = -1;
    if (err[0] != 0) {
        s.bad_region = (int64_t)(unsigned)err[1] | ((int64_t)err[2] << 31);
        char buf[128];
        std::snprintf(buf, sizeof(buf), "Cholesky pivot not positive in region %lld", (long long)s.bad_region);
        return fail(MRA_ERR_NOT_SPD, buf);
    }
    (void)predict;
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
    const long n_obs = (long)s->obs_offset[n_fin];
    if (s->obs_offset[0] != 0) return fail(MRA_ERR_ARG, "obs_offset[0] must be 0");
    if (n_obs > 0 && (!s->obs || !s->obs_value)) return fail(MRA_ERR_ARG, "observation arrays are NULL");
    const long lvl2 = level_start(J, M - 2), cnt2 = level_count(J, M - 2);
    std::vector<int64_t> nfin(n_fin), child_lo(cnt2, -1), child_hi(cnt2, -1);
    for (long k = 0; k < n_fin; ++k) {
        if (s->obs_offset[k + 1] < s->obs_offset[k]) return fail(MRA_ERR_ARG, "obs_offset must be non-decreasing");
        nfin[k] = (int64_t)(s->obs_offset[k + 1] - s->obs_offset[k]);
        long p = (long)s->finest_parent[k];
        if (p < lvl2 || p >= lvl2 + cnt2) return fail(MRA_ERR_ARG, "finest_parent must be a level M-2 region");
        long q = p - lvl2;
        if (child_lo[q] < 0) child_lo[q] = k;
        else if (child_hi[q] != k) return fail(MRA_ERR_ARG, "finest children of a region must be contiguous");
        child_hi[q] = k + 1;
    }
    for (long q = 0; q < cnt2; ++q)
        if (child_lo[q] < 0) child_lo[q] = child_hi[q] = 0;
    long n_pred = 0;
    bool have_pred = s->pred_offset != nullptr;
    std::vector<int64_t> npred(n_fin, 0);
    if (have_pred) {
        if (s->pred_offset[0] != 0) return fail(MRA_ERR_ARG, "pred_offset[0] must be 0");
        n_pred = (long)s->pred_offset[n_fin];
        if (n_pred > 0 && !s->pred) return fail(MRA_ERR_ARG, "prediction coordinates are NULL");
        for (long k = 0; k < n_fin; ++k) {
            if (s->pred_offset[k + 1] < s->pred_offset[k]) return fail(MRA_ERR_ARG, "pred_offset must be non-decreasing");
            npred[k] = (int64_t)(s->pred_offset[k + 1] - s->pred_offset[k]);
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
    c->have_pred = have_pred && n_pred > 0;
    c->geom = make_geom(m);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(MRA_ERR_CUDA, "stream creation failed"));
    for (auto& e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return bail(fail(MRA_ERR_CUDA, "event creation failed"));
    for (auto& e : c->tev)
        if (cudaEventCreate(&e) != cudaSuccess) return bail(fail(MRA_ERR_CUDA, "event creation failed"));

    // host-side tables
    std::vector<int64_t> obs_off(n_fin + 1), pred_off(n_fin + 1, 0), fin_anc(n_fin * L), lsig_off(n_fin + 1),
        pc_off(n_fin + 1), fin_order(n_fin);
    lsig_off[0] = pc_off[0] = 0;
    for (long k = 0; k <= n_fin; ++k) {
        obs_off[k] = (int64_t)s->obs_offset[k];
        if (have_pred) pred_off[k] = (int64_t)s->pred_offset[k];
    }
    for (long k = 0; k < n_fin; ++k) {
        long a = (long)s->finest_parent[k];
        fin_anc[k * L + L - 1] = a;
        for (int j = L - 2; j >= 0; --j) {
            a = (a - 1) / J;
            fin_anc[k * L + j] = a;
        }
        lsig_off[k + 1] = lsig_off[k] + nfin[k] * nfin[k];
        pc_off[k + 1] = pc_off[k] + nfin[k] * npred[k];
        fin_order[k] = k;
    }
    std::stable_sort(fin_order.begin(), fin_order.end(),
                     [&](int64_t a, int64_t b) { return nfin[a] + npred[a] > nfin[b] + npred[b]; });
    int64_t u_total = 0;
    for (int mm = 0; mm < kMaxLevels; ++mm) c->t.u_off[mm] = 0;
    for (int mm = 0; mm <= M - 2; ++mm) {
        c->t.u_off[mm] = u_total;
        u_total += level_count(J, mm) * (int64_t)mm * r * r;
    }
    // posterior outputs: ping-pong by level parity
    size_t aout_sz[2] = {16, 16}, wout_sz[2] = {16, 16};
    for (int mm = 1; mm <= M - 2; ++mm) {
        aout_sz[mm & 1] = std::max(aout_sz[mm & 1], (size_t)(level_count(J, mm) * n_slices(mm) * r * r));
        wout_sz[mm & 1] = std::max(wout_sz[mm & 1], (size_t)(level_count(J, mm) * mm * r));
    }
    const long rr = (long)r * r;
    c->t.ws_stride = n_slices(M - 1) * rr + (long)(M - 1) * r + (long)(M - 2 > 0 ? M - 2 : 0) * rr;

    cudaError_t ce = cudaSuccess;
    const long np_all = n_int * r + n_obs + n_pred;
    double* pc[3];
    for (int d = 0; d < 3; ++d) {
        pc[d] = c->alloc<double>(np_all, &ce);
        if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed"));
    }
    double* fields[3];
    for (int d = 0; d < 3; ++d) {
        fields[d] = c->alloc<double>(np_all, &ce);
        if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed"));
    }
    DevTree& t = c->t;
    t.J = J; t.M = M; t.r = r; t.L = L;
    t.n_int = n_int; t.n_fin = n_fin; t.n_obs = n_obs; t.n_pred = n_pred;
    t.obs0 = n_int * r;
    t.pred0 = n_int * r + n_obs;
    t.pts = PointSet{pc[0], pc[1], pc[2], fields[0], fields[1], fields[2]};
#define ALLOC(ptr, T, n)                                                   \
    do {                                                                   \
        ptr = c->alloc<T>((size_t)(n), &ce);                               \
        if (ce) return bail(fail(MRA_ERR_OOM, "device allocation failed: " #ptr)); \
    } while (0)
    double* y;
    ALLOC(y, double, n_obs);
    t.y = y;
    int64_t *d_obs_off, *d_pred_off, *d_fin_anc, *d_fin_order, *d_lsig_off, *d_pc_off, *d_clo, *d_chi;
    ALLOC(d_obs_off, int64_t, n_fin + 1);
    ALLOC(d_pred_off, int64_t, n_fin + 1);
    ALLOC(d_fin_anc, int64_t, n_fin * L);
    ALLOC(d_fin_order, int64_t, n_fin);
    ALLOC(d_lsig_off, int64_t, n_fin + 1);
    ALLOC(d_pc_off, int64_t, n_fin + 1);
    ALLOC(d_clo, int64_t, cnt2);
    ALLOC(d_chi, int64_t, cnt2);
    t.obs_off = d_obs_off; t.pred_off = d_pred_off; t.fin_anc = d_fin_anc; t.fin_order = d_fin_order;
    t.lsig_off = d_lsig_off; t.pc_off = d_pc_off; t.child_lo = d_clo; t.child_hi = d_chi;
    ALLOC(t.Lprior, double, n_int * rr);
    ALLOC(t.Lpost, double, n_int * rr);
    ALLOC(t.U, double, u_total);
    ALLOC(t.Ufin, double, n_obs * (long)L * r);
    ALLOC(t.Bhat, double, n_obs * (long)L * r);
    ALLOC(t.yt, double, n_obs);
    ALLOC(t.Lsig, double, lsig_off[n_fin]);
    ALLOC(t.dfin, double, n_fin);
    ALLOC(t.vpost, double, n_int * r);
    ALLOC(t.G, double, c->have_pred ? u_total : 1);
    ALLOC(t.dpost, double, n_int);
    ALLOC(t.aout[0], double, aout_sz[0]);
    ALLOC(t.aout[1], double, aout_sz[1]);
    ALLOC(t.wout[0], double, wout_sz[0]);
    ALLOC(t.wout[1], double, wout_sz[1]);
    ALLOC(t.ws, double, (long)c->grid * t.ws_stride);
    ALLOC(t.P, double, n_pred * (long)L * r);
    ALLOC(t.Bt, double, n_pred * (long)L * r);
    ALLOC(t.Pc, double, pc_off[n_fin]);
    ALLOC(t.mean, double, n_pred);
    ALLOC(t.var, double, n_pred);
    ALLOC(t.queue, int, 4);
    ALLOC(t.err, int, 4);
    ALLOC(c->d_theta, double, 16);
    ALLOC(c->d_result, double, 4);
    for (int f = 0; f < 3; ++f) {
        c->nb[f] = m->nonstationary ? (long)m->field[f].n_basis : 0;
        double* centers;
        ALLOC(centers, double, 3 * c->nb[f]);
        ALLOC(c->d_weights[f], double, c->nb[f]);
        c->model_weights[f].assign(m->nonstationary && c->nb[f] ? m->field[f].weights : nullptr,
                                   m->nonstationary && c->nb[f] ? m->field[f].weights + c->nb[f] : nullptr);
        c->model_intercept[f] = m->nonstationary ? m->field[f].intercept : 0.0;
        if (c->nb[f]) {
            mra_status u = upload(centers, m->field[f].centers, 3 * c->nb[f] * sizeof(double), c->stream);
            if (u) return bail(u);
            u = upload(c->d_weights[f], m->field[f].weights, c->nb[f] * sizeof(double), c->stream);
            if (u) return bail(u);
        }
        c->fp.nb[f] = c->nb[f];
        c->fp.centers[f] = centers;
        c->fp.weights[f] = c->d_weights[f];
    }
#undef ALLOC
    make_plan(c, nfin);
    {
        double R = r, fl = 0;
        for (long k = 0; k < n_fin; ++k) {
            double np = (double)npred[k], n = (double)nfin[k];
            fl += np * (L * R * R * (L - 1) / 2 + L * R * R / 2 + n * L * R + n * n / 2 + L * R * n + L * R * R / 2 +
                        L * (L - 1) / 2 * R * R);
        }
        c->flop_predict_launch = 2 * fl;
    }
    c->fp.basis = m->basis;
    c->fp.basis_len = m->basis_len;
    c->fp.theta = c->d_theta;

    // upload the structure (coordinates: knots | obs | preds per coordinate)
    for (int d = 0; d < 3; ++d) {
        mra_status u = upload(pc[d], s->knots + (size_t)d * n_int * r, n_int * r * sizeof(double), c->stream);
        if (!u && n_obs) u = upload(pc[d] + n_int * r, s->obs + (size_t)d * n_obs, n_obs * sizeof(double), c->stream);
        if (!u && n_pred)
            u = upload(pc[d] + n_int * r + n_obs, s->pred + (size_t)d * n_pred, n_pred * sizeof(double), c->stream);
        if (u) return bail(u);
    }
    struct {
        void* dst;
        const void* src;
        size_t bytes;
    } ups[] = {
        {y, s->obs_value, n_obs * sizeof(double)},
        {d_obs_off, obs_off.data(), (n_fin + 1) * sizeof(int64_t)},
        {d_pred_off, pred_off.data(), (n_fin + 1) * sizeof(int64_t)},
        {d_fin_anc, fin_anc.data(), n_fin * L * sizeof(int64_t)},
        {d_fin_order, fin_order.data(), n_fin * sizeof(int64_t)},
        {d_lsig_off, lsig_off.data(), (n_fin + 1) * sizeof(int64_t)},
        {d_pc_off, pc_off.data(), (n_fin + 1) * sizeof(int64_t)},
        {d_clo, child_lo.data(), cnt2 * sizeof(int64_t)},
        {d_chi, child_hi.data(), cnt2 * sizeof(int64_t)},
    };
    for (auto& u : ups) {
        mra_status e = upload(u.dst, u.src, u.bytes, c->stream);
        if (e) return bail(e);
    }
    double th0[16] = {1, 1, 1, c->model_intercept[0], c->model_intercept[1], c->model_intercept[2], 1, 1, 0};
    {
        mra_status e = upload(c->d_theta, th0, sizeof(th0), c->stream);
        if (e) return bail(e);
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
    CU(cudaMemcpyAsync(const_cast<double*>(c->t.y), y, c->n_obs * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    return MRA_OK;
}

mra_status mra_loglik(mra_ctx* c, double* d_out, double* ll_out) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    if (c->graph_exec) {
        CU(cudaGraphLaunch(c->graph_exec, c->stream));
        c->stats.graph_replays++;
    } else {
        mra_status s = run_eval(c, false);
        if (s) return s;
    }
    mra_status s = finish_eval(c, false);
    if (d_out) *d_out = c->stats.d;
    if (ll_out) *ll_out = c->stats.loglik;
    return s;
}

mra_status mra_predict(mra_ctx* c, double* mean, double* var) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    if (!c->have_pred) return fail(MRA_ERR_STATE, "the structure has no prediction locations");
    mra_status s = run_eval(c, true);
    if (s) return s;
    s = finish_eval(c, true);
    if (s) return s;
    if (mean) CU(cudaMemcpy(mean, c->t.mean, c->n_pred * sizeof(double), cudaMemcpyDeviceToHost));
    if (var) CU(cudaMemcpy(var, c->t.var, c->n_pred * sizeof(double), cudaMemcpyDeviceToHost));
    return MRA_OK;
}

mra_status mra_capture_graph(mra_ctx* c) {
    if (!c) return fail(MRA_ERR_ARG, "NULL context");
    if (c->graph_exec) return MRA_OK;
    CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    mra_status s = run_eval(c, false);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (s) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return fail(MRA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    c->graph = g;
    CU(cudaGraphInstantiate(&c->graph_exec, g, 0));
    return MRA_OK;
}

mra_status mra_get_stats(const mra_ctx* c, mra_stats* out) {
    if (!c || !out) return fail(MRA_ERR_ARG, "NULL argument");
    *out = c->stats;
    out->bytes_device = c->bytes;
    out->flop_last = c->flop_loglik;
    return MRA_OK;
}

mra_status mra_sample_prior(mra_ctx* c, const double* z_int, const double* z_obs, double* y_out) {
    if (!c || !z_int || (!z_obs && c->n_obs) || (!y_out && c->n_obs)) return fail(MRA_ERR_ARG, "NULL argument");
    // the prior factors come from one evaluation in prediction layout (keeps U_fin, L_Sigma)
    mra_status s = run_eval(c, false);
    if (s) return s;
    s = finish_eval(c, false);
    if (s) return s;
    double *dz, *dzo, *dy;
    size_t nzi = (size_t)c->n_int * c->r;
    CU(cudaMalloc(&dz, nzi * sizeof(double)));
    CU(cudaMalloc(&dzo, std::max<size_t>(c->n_obs, 1) * sizeof(double)));
    CU(cudaMalloc(&dy, std::max<size_t>(c->n_obs, 1) * sizeof(double)));
    CU(cudaMemcpy(dz, z_int, nzi * sizeof(double), cudaMemcpyHostToDevice));
    if (c->n_obs) CU(cudaMemcpy(dzo, z_obs, c->n_obs * sizeof(double), cudaMemcpyHostToDevice));
    launch_sample(c->t, dz, dzo, dy, c->grid, c->stream);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(c->stream));
    if (c->n_obs) CU(cudaMemcpy(y_out, dy, c->n_obs * sizeof(double), cudaMemcpyDeviceToHost));
    cudaFree(dz);
    cudaFree(dzo);
    cudaFree(dy);
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
            if (e == cudaSuccess && n1 * n2) e = cudaMemcpy(out, d, n1 * n2 * sizeof(double), cudaMemcpyDeviceToHost);
        }
        if (e != cudaSuccess) s = fail(MRA_ERR_CUDA, cudaGetErrorString(e));
    }
    for (void* q : frees) cudaFree(q);
    return s;
}

}  // extern "C"
