// mra_eval_covariance_static: the covariance-block evaluation of
// mra_eval_covariance without any device allocation.
//
// mra_eval_covariance allocates its temporaries (coordinates, per-point
// sigma^2 / beta / tau^2, basis tables) with cudaMalloc and frees them on every
// call.  Some callers cannot do that: applications that hand all device memory
// to their own pool or arena and do not allow the CUDA runtime allocator next to
// it, and tight host loops (an optimizer evaluating many small blocks) that
// cannot afford the device-wide synchronisation cudaMalloc / cudaFree imply.
// This variant takes the caller's device buffers for inputs and output and keeps
// its scratch in one fixed array in device global memory, sized for
// MRA_STATIC_MAX_POINTS points and MRA_STATIC_MAX_BASIS basis functions per
// field; every GPU that loads the library holds that array until the process
// exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/mra_b200.h"
#include "mra_kernels.cuh"

using namespace mra;

namespace {

// scratch layout (doubles): theta [16] | centers [3 fields][3][MAX_BASIS] |
// weights [3][MAX_BASIS] | coordinates [3][MAX_POINTS] | fields [3][MAX_POINTS]
constexpr long kTheta = 0;
constexpr long kCenters = 16;
constexpr long kWeights = kCenters + 3L * 3 * MRA_STATIC_MAX_BASIS;
constexpr long kCoords = kWeights + 3L * MRA_STATIC_MAX_BASIS;
constexpr long kFields = kCoords + 3L * MRA_STATIC_MAX_POINTS;
constexpr long kScratchDoubles = kFields + 3L * MRA_STATIC_MAX_POINTS;

}  // namespace

// The scratch itself.  In host code this name is only a stand-in for the
// device symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_mra_static_scratch[kScratchDoubles];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};
mra_status static_fail(mra_status s, const char* msg) {
    set_last_error(msg);
    return s;
}

// Device address of the scratch on the current device, looked up once per
// device with that device current.
mra_status scratch_on_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return static_fail(MRA_ERR_NO_DEVICE, "no current CUDA device");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_mra_static_scratch);
        if (e != cudaSuccess || !p) return static_fail(MRA_ERR_CUDA, cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return MRA_OK;
}

}  // namespace

extern "C" mra_status mra_eval_covariance_static(const mra_model* m, const mra_theta* th, const double* p1_dev,
                                                 uint64_t n1, const double* p2_dev, uint64_t n2, int32_t self,
                                                 double* out_dev, void* stream) {
    if (!m || !th || !p1_dev || !out_dev || (!self && !p2_dev))
        return static_fail(MRA_ERR_ARG, "mra_eval_covariance_static: NULL argument");
    if (mra_status ms = check_model(m)) return ms;
    if (self) n2 = 0;
    // each count on its own first, so that the sum below cannot wrap around
    if (n1 > (uint64_t)MRA_STATIC_MAX_POINTS || n2 > (uint64_t)MRA_STATIC_MAX_POINTS ||
        n1 + n2 > (uint64_t)MRA_STATIC_MAX_POINTS)
        return static_fail(MRA_ERR_ARG,
                           "mra_eval_covariance_static: n1 + n2 exceeds MRA_STATIC_MAX_POINTS (32768 points)");
    for (int f = 0; f < 3; ++f)
        if (m->nonstationary && m->field[f].n_basis > (uint64_t)MRA_STATIC_MAX_BASIS)
            return static_fail(MRA_ERR_ARG,
                               "mra_eval_covariance_static: a field has more than MRA_STATIC_MAX_BASIS (1024) "
                               "basis functions");
    double* scr = nullptr;
    mra_status s = scratch_on_current_device(&scr);
    if (s) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long np = (long)(n1 + n2);
#define SCU(call)                                                                       \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) return static_fail(MRA_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)
    // parameters: every word the kernels read is rewritten on each call
    double v[16] = {0};
    v[0] = th->sill_scale; v[1] = th->range_scale; v[2] = th->nugget_scale;
    v[6] = th->sill; v[7] = th->range; v[8] = th->nugget;
    FieldParams fp{};
    fp.basis = m->basis;
    fp.basis_len = m->basis_len;
    for (int f = 0; f < 3; ++f) {
        long nb = m->nonstationary ? (long)m->field[f].n_basis : 0;
        v[3 + f] = th->intercepts ? th->intercepts[f] : (m->nonstationary ? m->field[f].intercept : 0.0);
        double* cen = scr + kCenters + (long)f * 3 * MRA_STATIC_MAX_BASIS;
        double* w = scr + kWeights + (long)f * MRA_STATIC_MAX_BASIS;
        if (nb) {
            for (int c = 0; c < 3; ++c)
                SCU(cudaMemcpyAsync(cen + (long)c * nb, m->field[f].centers + (long)c * nb, nb * sizeof(double),
                                    cudaMemcpyHostToDevice, st));
            const double* wsrc = th->weights[f] ? th->weights[f] : m->field[f].weights;
            SCU(cudaMemcpyAsync(w, wsrc, nb * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        fp.nb[f] = nb;
        fp.centers[f] = cen;
        fp.weights[f] = w;
    }
    SCU(cudaMemcpyAsync(scr + kTheta, v, sizeof(v), cudaMemcpyHostToDevice, st));
    fp.theta = scr + kTheta;
    // coordinates: set 2 first, then set 1 (rows of the output are set-2 points)
    double* cc[3];
    for (int c = 0; c < 3; ++c) {
        cc[c] = scr + kCoords + (long)c * MRA_STATIC_MAX_POINTS;
        if (n2) SCU(cudaMemcpyAsync(cc[c], p2_dev + (long)c * n2, n2 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        SCU(cudaMemcpyAsync(cc[c] + n2, p1_dev + (long)c * n1, n1 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    double* fl[3];
    for (int f = 0; f < 3; ++f) fl[f] = scr + kFields + (long)f * MRA_STATIC_MAX_POINTS;
    Geom g{};
    g.nonstat = m->nonstationary ? 1 : 0;
    g.distance = m->distance;
    g.nu_x2 = m->nu_x2;
    g.pref_exp = m->prefactor_exp;
    g.pref_kind = m->prefactor_exp == 1.5 ? 0 : (m->prefactor_exp == 1.0 ? 1 : 2);
    g.dist_scale = m->dist_scale;
    launch_fields(g, fp, cc[0], cc[1], cc[2], np, fl[0], fl[1], fl[2], st);
    PointSet P{cc[0], cc[1], cc[2], fl[0], fl[1], fl[2]};
    if (self)
        launch_cov_block(g, P, 0, (int)n1, 0, (int)n1, true, out_dev, st);
    else
        launch_cov_block(g, P, 0, (int)n2, (long)n2, (int)n1, false, out_dev, st);
    SCU(cudaGetLastError());
#undef SCU
    return MRA_OK;
}
