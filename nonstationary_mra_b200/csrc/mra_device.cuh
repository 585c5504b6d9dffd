// Device-side building blocks of the MRA hot path (sm_100a).
//
//  * covariance entries, following src/evaluate_covariance.cpp:155-313 and the
//    fields of src/class_nonstationary_covariance.cpp:479-573;
//  * CTA-cooperative dense primitives on column-major operands that may live
//    in global or shared memory, templated on the storage type T:
//      T = double  the plain FP64 path: products on the FP64 tensor pipe
//                  (mma.sync m8n8k4 f64);
//      T = float   the mixed path: operands stored in FP32, products on the
//                  tensor cores as three TF32 products (hi*hi + hi*lo + lo*hi,
//                  FP32-accurate) with FP32 accumulation.
//    Diagonal blocks of every Cholesky factorization and triangular solve are
//    computed in FP64 whatever T is, and log-determinants are accumulated in
//    FP64.  One CTA owns one region's problem; the region kernels in
//    mra_kernels.cu are sequences of these calls.
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

__device__ __forceinline__ float matern_f(int nu_x2, float h) {
    if (nu_x2 == 3) {
        float s = 1.7320508f * h;
        return (1.0f + s) * expf(-s);
    }
    return expf(-h);
}

// C(s1, s2) with per-point sigma^2 (s) and beta (b): evaluate_covariance.cpp:218-225
// (nonstationary) and :82 (stationary: s1 = sill, b1 = range).
// For the straight-line distances the scaled distance over sqrt(bbar^2) is
// taken as sqrt(d^2 / bbar^2) with one reciprocal of bbar^2 shared with the
// prefactor (one division and one square root fewer than the literal form;
// the results agree to a few units in the last place).
__device__ __forceinline__ double cov_entry(const Geom& g, const Pt& p1, double s1, double b1, const Pt& p2,
                                            double s2, double b2) {
    if (g.distance == 1 || !g.nonstat) {
        double D = g.dist_scale * point_distance(g, p1, p2);
        if (!g.nonstat) return s1 * matern(g.nu_x2, D / b1);
        double bms = (b1 * b1 + b2 * b2) / 2;
        double x = (b1 * b2) / bms;
        double pre = g.pref_kind == 0 ? x * sqrt(x) : (g.pref_kind == 1 ? x : pow(x, g.pref_exp));
        return sqrt(s1 * s2) * pre * matern(g.nu_x2, D / sqrt(bms));
    }
    double dx = p2.c0 - p1.c0, dy = p2.c1 - p1.c1, dz = p2.c2 - p1.c2;
    double d2 = dx * dx + dy * dy + dz * dz;
    double ibms = 2.0 / (b1 * b1 + b2 * b2);
    double x = (b1 * b2) * ibms;
    double pre = g.pref_kind == 0 ? x * sqrt(x) : (g.pref_kind == 1 ? x : pow(x, g.pref_exp));
    double h = g.dist_scale * sqrt(d2 * ibms);
    return sqrt(s1 * s2) * pre * matern(g.nu_x2, h);
}

// The same entry evaluated in FP32 (the mixed path's covariance evaluation).
__device__ __forceinline__ float cov_entry_f(const Geom& g, const Pt& p1, float s1, float b1, const Pt& p2, float s2,
                                             float b2) {
    float D;
    if (g.distance == 1) {
        D = (float)(g.dist_scale * point_distance(g, p1, p2));
    } else {
        float dx = (float)(p2.c0 - p1.c0), dy = (float)(p2.c1 - p1.c1), dz = (float)(p2.c2 - p1.c2);
        D = (float)g.dist_scale * sqrtf(dx * dx + dy * dy + dz * dz);
    }
    if (!g.nonstat) return s1 * matern_f(g.nu_x2, D / b1);
    float bms = (b1 * b1 + b2 * b2) * 0.5f;
    float x = (b1 * b2) / bms;
    float pre = g.pref_kind == 0 ? x * sqrtf(x) : (g.pref_kind == 1 ? x : powf(x, (float)g.pref_exp));
    return sqrtf(s1 * s2) * pre * matern_f(g.nu_x2, D / sqrtf(bms));
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


// ----------------------------------------------------------------------------
// tensor-pipe fragments
// ----------------------------------------------------------------------------
__device__ __forceinline__ void mma_f64(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ----------------------------------------------------------------------------
// CTA-cooperative dense linear algebra (column-major)
// ----------------------------------------------------------------------------
constexpr int TM = 64, TN = 64, TK = 16, NB = 16;

// FP64 products (T = double): CTA tile 64 x (16 NW), NW in {1, 2, 4} picked by
// the width of the product, K slabs of 32.  Each operand tile is staged in
// shared memory in the layout of its global storage -- K-contiguous operands
// as [row][k] (stride 36), the others as [k][row] (stride 68) -- so that the
// coalesced global reads, the staging stores and the m8n8k4 fragment loads
// are all free of bank conflicts (both strides are 4 mod 16 doubles).
constexpr int TK64 = 32;
constexpr int KS64 = TK64 + 4;
constexpr int RS64 = 64 + 4;
constexpr int TILE64 = 64 * KS64;  // >= TK64 * RS64

template <typename T>
struct TilePad;
template <>
struct TilePad<double> {
    static constexpr int v = 4;
};
template <>
struct TilePad<float> {
    static constexpr int v = 8;  // row stride 72 floats: conflict-free m16n8k8 fragment loads
};

template <typename T>
struct LaSmem;
template <>
struct LaSmem<double> {
    double A[2][TILE64];   // two pipeline stages of each operand tile
    double B[2][TILE64];
    double D[NB][NB + 1];  // staged diagonal block
    double inv[NB];        // reciprocals of its diagonal
    double red[kThreads / 32];
    int flag;
};
template <>
struct LaSmem<float> {
    float A[TK][TM + TilePad<float>::v];
    float B[TK][TN + TilePad<float>::v];
    double D[NB][NB + 1];  // staged diagonal block (always FP64)
    double inv[NB];
    double red[kThreads / 32];
    int flag;
};

// The region kernels keep their LaSmem in dynamic shared memory (the FP64
// version is larger than the 48 KB static limit).
template <typename T>
__device__ __forceinline__ LaSmem<T>& la_smem() {
    extern __shared__ __align__(16) unsigned char la_dyn_smem[];
    return *reinterpret_cast<LaSmem<T>*>(la_dyn_smem);
}

// ---- branch-free FP64 elementary functions for the covariance entries ----
// e^{-s} for s >= 0 (s clamped at 700, where the result is below 1e-304):
// Cody-Waite reduction s = n ln2 + r, |r| <= ln2/2, with ln2 split in a
// 32-bit head (n * head exact) and a tail; e^{-r} from its Taylor polynomial
// of degree 13 in Horner form (truncation below 5e-18 relative); 2^{-n} built
// in the exponent field.  Within 1 ulp of exp(-s) on this range (checked on
// 4M arguments against the CUDA library).
__device__ __forceinline__ double exp_neg(double s) {
    s = fmin(s, 700.0);
    const double kShift = 6755399441055744.0;  // 1.5 * 2^52: rounds s/ln2 to an integer in the low word
    const double t = fma(s, 1.4426950408889634, kShift);
    const double n = t - kShift;
    double r = fma(-n, 0.6931471803691238, s);
    r = fma(-n, 1.9082149292705877e-10, r);
    const double u = -r;
    double p = 1.6059043836821613e-10;  // 1/13!
    p = fma(p, u, 2.08767569878681e-09);
    p = fma(p, u, 2.505210838544172e-08);
    p = fma(p, u, 2.755731922398589e-07);
    p = fma(p, u, 2.7557319223985893e-06);
    p = fma(p, u, 2.48015873015873e-05);
    p = fma(p, u, 0.0001984126984126984);
    p = fma(p, u, 0.001388888888888889);
    p = fma(p, u, 0.008333333333333333);
    p = fma(p, u, 0.041666666666666664);
    p = fma(p, u, 0.16666666666666666);
    p = fma(p, u, 0.5);
    p = fma(p, u, 1.0);
    p = fma(p, u, 1.0);
    return p * __hiloint2double((1023 - __double2loint(t)) << 20, 0);
}

// 1/s from the PTX approximation refined by one third-order Newton step
// (y <- y (1 + e + e^2), e = 1 - s y); s positive and normal.
__device__ __forceinline__ double rcp_nr(double s) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(s));
    const double e = fma(-s, y, 1.0);
    return fma(y, fma(e, e, e), y);
}

// 1/sqrt(x) from the PTX approximation refined by one third-order Newton step
// (y <- y (1 + e/2 + 3e^2/8), e = 1 - x y^2); x positive and normal.
__device__ __forceinline__ double rsqrt_nr(double x) {
    double y;
    asm("rsqrt.approx.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x * y, y, 1.0);
    return fma(y * e, fma(0.375, e, 0.5), y);
}

// The same two quantities seeded by the single-precision approximations
// (rcp.approx.ftz.f32 / rsqrt.approx.ftz.f32 of the argument rounded to FP32,
// relative error near 2^-23) and refined by the same third-order Newton step,
// whose cubic convergence takes the seed error below 2^-66: the result is within
// an ulp or two of the FP64-seeded form.  The FP32 units issue these far faster
// than the FP64 approximations; arguments outside [1e-30, 1e30], where the FP32
// seed would underflow or overflow, take the FP64-seeded path.
__device__ __forceinline__ double rcp_fast(double s) {
    if (!(s > 1e-30 && s < 1e30)) return rcp_nr(s);
    float yf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(__double2float_rn(s)));
    const double y = (double)yf;
    const double e = fma(-s, y, 1.0);
    return fma(y, fma(e, e, e), y);
}

__device__ __forceinline__ double rsqrt_fast(double x) {
    if (!(x > 1e-30 && x < 1e30)) return rsqrt_nr(x);
    float yf;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(__double2float_rn(x)));
    const double y = (double)yf;
    const double e = fma(-x * y, y, 1.0);
    return fma(y * e, fma(0.375, e, 0.5), y);
}

// One nonstationary straight-line entry from per-point quantities (see
// fill_row_fast): row point (pc, ga, ca = sqrt(s1) b1 / scale^2 for PREF 1;
// ssa, ba_h = b1 / scale^2 for PREF 0), column point (q, gq, ssbq = sqrt(s2) b2;
// ssq, bq).  F32SEED: reciprocal and inverse square root seeded in FP32
// (rcp_fast / rsqrt_fast; more independent work per issue slot, for launches
// that are issue-bound) or in FP64 (rcp_nr / rsqrt_nr; shorter dependent
// chains, for fills that are latency-bound inside the region kernels).
template <int NU, int PREF, bool F32SEED = false>
__device__ __forceinline__ double cov_fast_entry(double pc0, double pc1, double pc2, double ga, double ca,
                                                 double ssa, double ba_h, double qx, double qy, double qz, double gq,
                                                 double ssbq, double ssq, double bq) {
    const double dx = qx - pc0, dy = qy - pc1, dz = qz - pc2;
    const double d2 = fma(dx, dx, fma(dy, dy, dz * dz));
    const double w = F32SEED ? rcp_fast(ga + gq) : rcp_nr(ga + gq);  // 2 scale^2 / (b1^2 + b2^2)
    const double u = d2 * w;                                            // h^2
    const double h = u > 1e-300 ? u * (F32SEED ? rsqrt_fast(u) : rsqrt_nr(u)) : 0.0;
    const double em = exp_neg(h);
    const double m = NU == 3 ? (1.0 + h) * em : em;
    if (PREF == 1) return (ca * ssbq) * w * m;
    const double x = ba_h * bq * w;
    return (ssa * ssq) * (x * sqrt(x)) * m;
}

// One row point against the staged column points q_begin, q_begin + q_step,
// ... < q_end (straight-line distance, nonstationary): writes ob[(qoff + q) ld].
// NU: 1 exponential, 3 Matern 3/2; PREF: 0 prefactor x^1.5, 1 prefactor x.
// Entry: sqrt(s1 s2) pre(x) matern(h), x = 2 b1 b2 / (b1^2 + b2^2),
// h = scale sqrt(2 d^2 / (b1^2 + b2^2)).  With g = b^2 / (2 scale^2) staged per
// point, w = 1 / (g1 + g2) gives h = sqrt(d^2 w) and x = b1 b2 w / scale^2,
// so the entry is (sqrt(s1) b1 / scale^2) (sqrt(s2) b2) w matern(h) for
// PREF 1.  Every parameter is in registers so the loop carries no reloads;
// one reciprocal, one inverse square root and one exponential per entry,
// none with a branch.
template <typename T, int NU, int PREF>
__device__ __noinline__ void fill_row_fast(const double* __restrict__ sx, const double* __restrict__ sy,
                                           const double* __restrict__ sz, const double* __restrict__ ss,
                                           const double* __restrict__ sb, const double* __restrict__ sg,
                                           const double* __restrict__ ssb, double pc0, double pc1, double pc2,
                                           double ssa, double ba, double ga, double ihs2, int q_begin, int q_end,
                                           int q_step, int qoff, T* __restrict__ ob, long ld) {
    const double ca = ssa * ba * ihs2, ba_h = ba * ihs2;
#pragma unroll 4
    for (int q = q_begin; q < q_end; q += q_step) {
        const double v = cov_fast_entry<NU, PREF>(pc0, pc1, pc2, ga, ca, ssa, ba_h, sx[q], sy[q], sz[q], sg[q],
                                                  PREF == 1 ? ssb[q] : 0.0, PREF == 1 ? 0.0 : ss[q],
                                                  PREF == 1 ? 0.0 : sb[q]);
        ob[(long)(qoff + q) * ld] = (T)v;
    }
}

// out[t + q*ld] = C(A_{a0+t}, B_{b0+q}), t < na, q < nb.  When `self` the
// diagonal (t == q) is sigma^2 + tau^2 (evaluate_covariance.cpp:103,307).
// The column points (coordinates, sqrt(sigma^2), beta and two products) are staged in
// shared memory in chunks, each thread keeps one row point in registers and
// walks columns strided by the number of row groups (consecutive threads
// write consecutive rows).  The straight-line nonstationary FP64 case with
// the prefactor exponents 1.5 or 1 goes through fill_row_fast; the others
// evaluate cov_entry / cov_entry_f per entry.  Ends with a barrier; uses the
// tile buffers of sm.
// fill_cov_blocks: nblk blocks of na rows each, block k from the row points
// starting at a0[k], written to out + k * blk (same columns for every block);
// `self` applies to block 0 only.
// fill_cov_staged: the same with the staging area given explicitly (7 CH
// doubles) and CH columns staged per chunk; every entry is computed by the same
// per-entry code whatever CH is.
template <typename T, int CH>
__device__ __noinline__ void fill_cov_staged(const Geom& g, const PointSet& P, const long* a0, int nblk, int na,
                                             long b0, int nb, bool self, T* out, long ld, long blk,
                                             double* stage) {
    double* sx = stage;
    double* sy = sx + CH;
    double* sz = sy + CH;
    double* ss = sz + CH;
    double* sb = ss + CH;
    double* sg = sb + CH;   // FP64 fast path only: beta^2 / (2 scale^2) and sqrt(sigma^2) beta
    double* ssb = sg + CH;  // (7 CH doubles fit the FP64 tile buffers)
    const int tid = threadIdx.x, nt = blockDim.x;
    const int R = nblk * na;  // all rows of all blocks
    const int rows = R < nt ? R : nt;
    const int cols = nt / rows;
    const bool worker = tid < rows * cols;
    const int tr = tid % rows, tq = tid / rows;
    const int nu = g.nu_x2, pk = g.pref_kind;
    const bool fast = sizeof(T) == 8 && g.nonstat && g.distance != 1 && pk != 2;
    const double hs = g.dist_scale * (nu == 3 ? 1.7320508075688772 : 1.0);
    const double ihs2 = 1.0 / (hs * hs), ih2 = 0.5 * ihs2;
    for (int q0 = 0; q0 < nb; q0 += CH) {
        const int qn = nb - q0 < CH ? nb - q0 : CH;
        __syncthreads();
        for (int e = tid; e < qn; e += nt) {
            const long ib = b0 + q0 + e;
            sx[e] = P.c0[ib];
            sy[e] = P.c1[ib];
            sz[e] = P.c2[ib];
            ss[e] = fast ? sqrt(P.s2[ib]) : P.s2[ib];
            const double bb = P.beta[ib];
            sb[e] = bb;
            if (fast) {
                sg[e] = bb * bb * ih2;
                ssb[e] = ss[e] * bb;
            }
        }
        __syncthreads();
        if (!worker) continue;
        for (int tt = tr; tt < R; tt += rows) {
            const int kb = tt / na, t = tt - kb * na;
            const long ia = a0[kb] + t;
            if (fast) {
                T* ob = out + kb * blk + t;
                const double pc0 = P.c0[ia], pc1 = P.c1[ia], pc2 = P.c2[ia];
                const double sa = P.s2[ia], ba = P.beta[ia];
                const double ssa = sqrt(sa), ga = ba * ba * ih2;
                if (nu == 3 && pk == 1)
                    fill_row_fast<T, 3, 1>(sx, sy, sz, ss, sb, sg, ssb, pc0, pc1, pc2, ssa, ba, ga, ihs2, tq, qn, cols,
                                           q0, ob, ld);
                else if (nu == 3)
                    fill_row_fast<T, 3, 0>(sx, sy, sz, ss, sb, sg, ssb, pc0, pc1, pc2, ssa, ba, ga, ihs2, tq, qn, cols,
                                           q0, ob, ld);
                else if (pk == 1)
                    fill_row_fast<T, 1, 1>(sx, sy, sz, ss, sb, sg, ssb, pc0, pc1, pc2, ssa, ba, ga, ihs2, tq, qn, cols,
                                           q0, ob, ld);
                else
                    fill_row_fast<T, 1, 0>(sx, sy, sz, ss, sb, sg, ssb, pc0, pc1, pc2, ssa, ba, ga, ihs2, tq, qn, cols,
                                           q0, ob, ld);
                // the diagonal of a self block, whose entry this thread has just written
                if (self && kb == 0) {
                    const int qd = t - q0;
                    if (qd >= tq && qd < qn && (qd - tq) % cols == 0) ob[(long)t * ld] = (T)(sa + P.t2[ia]);
                }
                continue;
            }
            T* ob = out + kb * blk;
            const Pt pa = P.pt(ia);
            const double sa = P.s2[ia], ba = P.beta[ia];
#pragma unroll 4
            for (int q = tq; q < qn; q += cols) {
                const int qq = q0 + q;
                T v;
                if (self && kb == 0 && t == qq) {
                    v = (T)(sa + P.t2[ia]);
                } else if (sizeof(T) == 8) {
                    v = (T)cov_entry(g, pa, sa, ba, Pt{sx[q], sy[q], sz[q]}, ss[q], sb[q]);
                } else {
                    v = (T)cov_entry_f(g, pa, (float)sa, (float)ba, Pt{sx[q], sy[q], sz[q]}, (float)ss[q],
                                       (float)sb[q]);
                }
                ob[t + (long)qq * ld] = v;
            }
        }
    }
    __syncthreads();
}

template <typename T>
__device__ inline void fill_cov_blocks(const Geom& g, const PointSet& P, const long* a0, int nblk, int na, long b0,
                                       int nb, bool self, T* out, long ld, long blk, LaSmem<T>& sm) {
    // the staging area is the tile buffers of sm: 7 CH doubles
    fill_cov_staged<T, sizeof(T) == 8 ? 512 : 96>(g, P, a0, nblk, na, b0, nb, self, out, ld, blk,
                                                   reinterpret_cast<double*>(&sm.A[0][0]));
}

template <typename T>
__device__ inline void fill_cov(const Geom& g, const PointSet& P, long a0, int na, long b0, int nb, bool self,
                                T* out, long ld, LaSmem<T>& sm) {
    fill_cov_blocks<T>(g, P, &a0, 1, na, b0, nb, self, out, ld, 0, sm);
}

// ---- FP64: warp tile (8 NW) rows x 16 columns --------------------------------
template <int NW>
struct AccD {
    double v[NW][2][2];  // NW (m8) x 2 (n8) fragments of m8n8
};

// 8-byte asynchronous global -> shared copy; pred == false writes zeros.
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool pred) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
// Bulk prefetch into L2 of the 16-byte aligned part of [p, p + bytes) (the
// instruction takes a 16-byte aligned address and a multiple of 16 bytes).
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned long bytes) {
    const unsigned long a = ((unsigned long)p + 15) & ~15ul, b = ((unsigned long)p + bytes) & ~15ul;
    if (b <= a || b - a > 0xffffffffull) return;
    asm volatile(
        "{\n\t.reg .u64 ga;\n\tcvta.to.global.u64 ga, %0;\n\tcp.async.bulk.prefetch.L2.global [ga], %1;\n\t}\n" ::"l"(a),
        "r"((unsigned)(b - a))
        : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <bool TA, bool TB, int NW>
__device__ __forceinline__ void warp_step_f64(AccD<NW>& acc, const double* sA, const double* sB, int wm, int wn,
                                              int lane) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int k4 = 0; k4 < TK64; k4 += 4) {
        double a[NW], b[2];
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            const int row = wm + 8 * i + g, k = k4 + t;
            a[i] = TA ? sA[row * KS64 + k] : sA[k * RS64 + row];
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int col = wn + 8 * j + g, k = k4 + t;
            b[j] = TB ? sB[k * RS64 + col] : sB[col * KS64 + k];
        }
#pragma unroll
        for (int i = 0; i < NW; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) mma_f64(acc.v[i][j], a[i], b[j]);
    }
}

// Operands must be in global memory (they are copied with cp.async): a
// two-stage pipeline keeps the next K slab in flight while the tensor pipe
// works on the current one.
template <bool TA, bool TB, int NW>
__device__ inline void gemm_f64(int M, int N, int K, double alpha, const double* A, long lda, const double* B,
                                long ldb, double beta, double* C, long ldc, LaSmem<double>& sm,
                                const double* Cin = nullptr, long ldcin = 0) {
    constexpr int W = 16 * NW;                // CTA tile width
    constexpr int WM = 8 / NW;                // warps along M
    constexpr int PA = 64 * TK64 / kThreads;  // A elements per thread per slab (8)
    constexpr int PB = W * TK64 / kThreads;   // B elements per thread per slab (2 NW)
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int wm = (w % WM) * 8 * NW, wn = (w / WM) * 16;
    for (int m0 = 0; m0 < M; m0 += 64) {
        for (int n0 = 0; n0 < N; n0 += W) {
            AccD<NW> acc;
#pragma unroll
            for (int i = 0; i < NW; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) acc.v[i][j][0] = acc.v[i][j][1] = 0.0;
            auto issue = [&](int k0, int stage) {
                double* sA = sm.A[stage];
                double* sB = sm.B[stage];
#pragma unroll
                for (int q = 0; q < PA; ++q) {
                    const int e = tid + q * kThreads;
                    // TA: op(A)[i][k] = A[k + i lda] (K-contiguous), else A[i + k lda]
                    const int i = TA ? e / TK64 : e % 64, k = TA ? e % TK64 : e / 64;
                    const int gi = m0 + i, gk = k0 + k;
                    const bool ok = gi < M && gk < K;
                    const double* src = ok ? (TA ? A + gk + (long)gi * lda : A + gi + (long)gk * lda) : A;
                    cp_async8(sA + (TA ? i * KS64 + k : k * RS64 + i), src, ok);
                }
#pragma unroll
                for (int q = 0; q < PB; ++q) {
                    const int e = tid + q * kThreads;
                    // TB: op(B)[k][j] = B[j + k ldb], else B[k + j ldb] (K-contiguous)
                    const int j = TB ? e % W : e / TK64, k = TB ? e / W : e % TK64;
                    const int gj = n0 + j, gk = k0 + k;
                    const bool ok = gj < N && gk < K;
                    const double* src = ok ? (TB ? B + gj + (long)gk * ldb : B + gk + (long)gj * ldb) : B;
                    cp_async8(sB + (TB ? k * RS64 + j : j * KS64 + k), src, ok);
                }
                cp_async_commit();
            };
            // warps whose tile lies outside the product skip the tensor work
            const bool active = m0 + wm < M && n0 + wn < N;
            if (K > 0) issue(0, 0);
            int stage = 0;
            for (int k0 = 0; k0 < K; k0 += TK64, stage ^= 1) {
                if (k0 + TK64 < K) {
                    issue(k0 + TK64, stage ^ 1);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncthreads();
                if (active) warp_step_f64<TA, TB, NW>(acc, sm.A[stage], sm.B[stage], wm, wn, lane);
                __syncthreads();
            }
            if (active) {
                const int g = lane >> 2, t = lane & 3;
#pragma unroll
                for (int i = 0; i < NW; ++i)
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const int r = m0 + wm + 8 * i + g, c = n0 + wn + 8 * j + 2 * t;
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            if (r < M && c + h < N) {
                                double* p = C + r + (long)(c + h) * ldc;
                                const double* q = Cin ? Cin + r + (long)(c + h) * ldcin : p;
                                *p = beta == 0.0 ? alpha * acc.v[i][j][h] : alpha * acc.v[i][j][h] + beta * *q;
                            }
                        }
                    }
            }
        }
    }
    __syncthreads();
}

// 16-byte asynchronous global -> shared copy through L2 only (not L1); both
// addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(double* dst, const double* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// gemm_f64 for whole tiles (M % 64 == 0, N % (16 NW) == 0, K % 32 == 0) with
// 16-byte aligned operand rows (aligned A and B, even lda and ldb): the same
// tiles, the same shared-memory layout and the same per-element K order, hence
// bitwise the same results, with the operands staged in pairs of elements by
// 16-byte copies through L2 only -- half the copy instructions and no L1
// allocation.
template <bool TA, bool TB, int NW>
__device__ inline void gemm_f64_wide(int M, int N, int K, double alpha, const double* A, long lda, const double* B,
                                     long ldb, double beta, double* C, long ldc, LaSmem<double>& sm,
                                     const double* Cin, long ldcin) {
    constexpr int W = 16 * NW;
    constexpr int WM = 8 / NW;
    constexpr int QA = 64 * TK64 / 2 / kThreads;  // A pairs per thread per slab (4)
    constexpr int QB = W * TK64 / 2 / kThreads;   // B pairs per thread per slab (NW)
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int wm = (w % WM) * 8 * NW, wn = (w / WM) * 16;
    for (int m0 = 0; m0 < M; m0 += 64) {
        for (int n0 = 0; n0 < N; n0 += W) {
            AccD<NW> acc;
#pragma unroll
            for (int i = 0; i < NW; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) acc.v[i][j][0] = acc.v[i][j][1] = 0.0;
            auto issue = [&](int k0, int stage) {
                double* sA = sm.A[stage];
                double* sB = sm.B[stage];
#pragma unroll
                for (int q = 0; q < QA; ++q) {
                    const int e = tid + q * kThreads;
                    // TA: pair (i, k..k+1) of A[k + i lda]; else pair (i..i+1, k) of A[i + k lda]
                    const int i = TA ? e / (TK64 / 2) : 2 * (e % 32), k = TA ? 2 * (e % (TK64 / 2)) : e / 32;
                    const double* src = TA ? A + (k0 + k) + (long)(m0 + i) * lda : A + (m0 + i) + (long)(k0 + k) * lda;
                    cp_async16(sA + (TA ? i * KS64 + k : k * RS64 + i), src);
                }
#pragma unroll
                for (int q = 0; q < QB; ++q) {
                    const int e = tid + q * kThreads;
                    // TB: pair (k, j..j+1) of B[j + k ldb]; else pair (k..k+1, j) of B[k + j ldb]
                    const int j = TB ? 2 * (e % (W / 2)) : e / (TK64 / 2), k = TB ? e / (W / 2) : 2 * (e % (TK64 / 2));
                    const double* src = TB ? B + (n0 + j) + (long)(k0 + k) * ldb : B + (k0 + k) + (long)(n0 + j) * ldb;
                    cp_async16(sB + (TB ? k * RS64 + j : j * KS64 + k), src);
                }
                cp_async_commit();
            };
            issue(0, 0);
            int stage = 0;
            for (int k0 = 0; k0 < K; k0 += TK64, stage ^= 1) {
                if (k0 + TK64 < K) {
                    issue(k0 + TK64, stage ^ 1);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncthreads();
                warp_step_f64<TA, TB, NW>(acc, sm.A[stage], sm.B[stage], wm, wn, lane);
                __syncthreads();
            }
            const int g = lane >> 2, t = lane & 3;
#pragma unroll
            for (int i = 0; i < NW; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int r = m0 + wm + 8 * i + g, c = n0 + wn + 8 * j + 2 * t;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        double* p = C + r + (long)(c + h) * ldc;
                        const double* q = Cin ? Cin + r + (long)(c + h) * ldcin : p;
                        *p = beta == 0.0 ? alpha * acc.v[i][j][h] : alpha * acc.v[i][j][h] + beta * *q;
                    }
                }
        }
    }
    __syncthreads();
}

// ---- FP32 storage (mixed path): 3xTF32 products, 64 x 64 tiles, K slabs of 16
struct AccF {
    float v[2][2][4];  // 2 (m16) x 2 (n8) fragments of m16n8
};

__device__ __forceinline__ void warp_step_tf32x3(AccF& acc, const LaSmem<float>& sm, int wm, int wn, int lane) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int k8 = 0; k8 < TK; k8 += 8) {
        uint32_t ah[2][4], al[2][4], bh[2][2], bl[2][2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r0 = wm + 16 * i + g;
            float x[4] = {sm.A[k8 + t][r0], sm.A[k8 + t][r0 + 8], sm.A[k8 + t + 4][r0], sm.A[k8 + t + 4][r0 + 8]};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                ah[i][q] = to_tf32(x[q]);
                al[i][q] = to_tf32(x[q] - __uint_as_float(ah[i][q]));
            }
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int c0 = wn + 8 * j + g;
            float y[2] = {sm.B[k8 + t][c0], sm.B[k8 + t + 4][c0]};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                bh[j][q] = to_tf32(y[q]);
                bl[j][q] = to_tf32(y[q] - __uint_as_float(bh[j][q]));
            }
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                mma_tf32(acc.v[i][j], al[i], bh[j]);
                mma_tf32(acc.v[i][j], ah[i], bl[j]);
                mma_tf32(acc.v[i][j], ah[i], bh[j]);
            }
    }
}

template <bool TA, bool TB>
__device__ inline void gemm_f32(int M, int N, int K, float alpha, const float* A, long lda, const float* B, long ldb,
                                float beta, float* C, long ldc, LaSmem<float>& sm, const float* Cin = nullptr,
                                long ldcin = 0) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int wm = (w & 1) * 32, wn = (w >> 1) * 16;
    constexpr int PER = TK * TM / kThreads;  // elements of each operand per thread per slab (4)
    for (int m0 = 0; m0 < M; m0 += TM) {
        for (int n0 = 0; n0 < N; n0 += TN) {
            AccF acc;
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j)
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc.v[i][j][q] = 0.f;
            float ra[PER], rb[PER];
            auto fetch = [&](int k0) {
#pragma unroll
                for (int q = 0; q < PER; ++q) {
                    const int e = tid + q * kThreads;
                    int i, k;
                    if (!TA) { i = e % TM; k = e / TM; } else { k = e % TK; i = e / TK; }
                    const int gi = m0 + i, gk = k0 + k;
                    ra[q] = (gi < M && gk < K) ? (TA ? A[gk + (long)gi * lda] : A[gi + (long)gk * lda]) : 0.f;
                    int j, kb;
                    if (!TB) { kb = e % TK; j = e / TK; } else { j = e % TN; kb = e / TN; }
                    const int gj = n0 + j, gkb = k0 + kb;
                    rb[q] = (gj < N && gkb < K) ? (TB ? B[gj + (long)gkb * ldb] : B[gkb + (long)gj * ldb]) : 0.f;
                }
            };
            auto stash = [&]() {
#pragma unroll
                for (int q = 0; q < PER; ++q) {
                    const int e = tid + q * kThreads;
                    int i, k;
                    if (!TA) { i = e % TM; k = e / TM; } else { k = e % TK; i = e / TK; }
                    sm.A[k][i] = ra[q];
                    int j, kb;
                    if (!TB) { kb = e % TK; j = e / TK; } else { j = e % TN; kb = e / TN; }
                    sm.B[kb][j] = rb[q];
                }
            };
            if (K > 0) {
                fetch(0);
                stash();
            }
            __syncthreads();
            for (int k0 = 0; k0 < K; k0 += TK) {
                const bool more = k0 + TK < K;
                if (more) fetch(k0 + TK);
                warp_step_tf32x3(acc, sm, wm, wn, lane);
                __syncthreads();
                if (more) {
                    stash();
                    __syncthreads();
                }
            }
            const int g = lane >> 2, t = lane & 3;
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int r = m0 + wm + 16 * i + g, c = n0 + wn + 8 * j + 2 * t;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int rr = r + (q >> 1) * 8, cc = c + (q & 1);
                        if (rr < M && cc < N) {
                            float* p = C + rr + (long)cc * ldc;
                            const float* qi = Cin ? Cin + rr + (long)cc * ldcin : p;
                            *p = beta == 0.f ? alpha * acc.v[i][j][q] : alpha * acc.v[i][j][q] + beta * *qi;
                        }
                    }
                }
        }
    }
    __syncthreads();
}

// C = alpha * op(A) * op(B) + beta * Cin (Cin = C unless given, ld ldcin);
// op(A): M x K, op(B): K x N, column-major,
// any leading dimensions; A and B in global memory.  beta == 0 never reads C.
// Ends with a barrier.
// FP64 tile width (NW) per product-width bucket (N <= 16, N <= 32, wider),
// chosen per device by the autotuner (mra_autotune); {1, 2, 4} by default.
// The choice changes only how output tiles are spread over warps: every
// element is accumulated by one thread in the same K order, so results are
// bitwise the same whatever the choice.
__constant__ int c_gemm_nw[3] = {1, 2, 4};

// ONE_TILE: the product must be computed as one column tile (N <= 64) --
// required when C aliases A (an in-place product C = C X): each row tile then
// reads all of its rows before writing them, whereas a second column tile
// would read columns the first one has already overwritten.
template <typename T, bool TA, bool TB, bool ONE_TILE = false>
__device__ inline void gemm(int M, int N, int K, T alpha, const T* A, long lda, const T* B, long ldb, T beta, T* C,
                            long ldc, LaSmem<T>& sm, const T* Cin = nullptr, long ldcin = 0) {
    if constexpr (sizeof(T) == 8) {
        const int nw = ONE_TILE ? (N <= 16 ? 1 : (N <= 32 ? 2 : 4)) : c_gemm_nw[N <= 16 ? 0 : (N <= 32 ? 1 : 2)];
        if (nw == 1) gemm_f64<TA, TB, 1>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, sm, Cin, ldcin);
        else if (nw == 2) gemm_f64<TA, TB, 2>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, sm, Cin, ldcin);
        else gemm_f64<TA, TB, 4>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, sm, Cin, ldcin);
    } else {
        gemm_f32<TA, TB>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, sm, Cin, ldcin);
    }
}

// Stages the nb x nb diagonal block of L at b0 in FP64 with the reciprocals of
// its diagonal.  Ends with a barrier.
template <typename T>
__device__ inline void stage_diag_block(const T* L, long ldl, int b0, int nb, LaSmem<T>& sm) {
    for (int e = threadIdx.x; e < nb * nb; e += kThreads) {
        int i = e % nb, j = e / nb;
        sm.D[i][j] = (double)L[(b0 + i) + (long)(b0 + j) * ldl];
    }
    __syncthreads();
    if (threadIdx.x < nb) sm.inv[threadIdx.x] = 1.0 / sm.D[threadIdx.x][threadIdx.x];
    __syncthreads();
}

// B <- L^{-1} B  (L: n x n lower, non-unit; B: n x nrhs).  dtrtrs('L','N','N').
// Diagonal blocks are solved in FP64; trailing updates go through gemm<T>.
template <typename T>
__device__ inline void trsm_left_lower(int n, int nrhs, const T* L, long ldl, T* B, long ldb, LaSmem<T>& sm) {
    const int tid = threadIdx.x;
    for (int b0 = 0; b0 < n; b0 += NB) {
        int nb = min(NB, n - b0);
        stage_diag_block(L, ldl, b0, nb, sm);
        for (int c = tid; c < nrhs; c += kThreads) {
            double x[NB];
            T* col = B + b0 + (long)c * ldb;
#pragma unroll
            for (int i = 0; i < NB; ++i) x[i] = i < nb ? (double)col[i] : 0.0;
#pragma unroll
            for (int i = 0; i < NB; ++i) {
                if (i < nb) {
                    double s = x[i];
#pragma unroll
                    for (int k = 0; k < i; ++k) s -= sm.D[i][k] * x[k];
                    x[i] = s * sm.inv[i];
                }
            }
#pragma unroll
            for (int i = 0; i < NB; ++i)
                if (i < nb) col[i] = (T)x[i];
        }
        __syncthreads();
        if (b0 + nb < n)
            gemm<T, false, false>(n - b0 - nb, nrhs, nb, (T)-1, L + (b0 + nb) + (long)b0 * ldl, ldl, B + b0, ldb,
                                  (T)1, B + b0 + nb, ldb, sm);
    }
}

// B <- B L^{-T}  (L: n x n lower; B: rows x n).  Row-wise forward substitution.
template <typename T>
__device__ inline void trsm_right_lower_trans(int rows, int n, const T* L, long ldl, T* B, long ldb, LaSmem<T>& sm) {
    const int tid = threadIdx.x;
    for (int b0 = 0; b0 < n; b0 += NB) {
        int nb = min(NB, n - b0);
        stage_diag_block(L, ldl, b0, nb, sm);
        for (int row = tid; row < rows; row += kThreads) {
            double x[NB];
            T* p = B + row + (long)b0 * ldb;
#pragma unroll
            for (int i = 0; i < NB; ++i) x[i] = i < nb ? (double)p[(long)i * ldb] : 0.0;
#pragma unroll
            for (int i = 0; i < NB; ++i) {
                if (i < nb) {
                    double s = x[i];
#pragma unroll
                    for (int k = 0; k < i; ++k) s -= sm.D[i][k] * x[k];
                    x[i] = s * sm.inv[i];
                }
            }
#pragma unroll
            for (int i = 0; i < NB; ++i)
                if (i < nb) p[(long)i * ldb] = (T)x[i];
        }
        __syncthreads();
        if (b0 + nb < n)
            gemm<T, false, true>(rows, n - b0 - nb, nb, (T)-1, B + (long)b0 * ldb, ldb, L + (b0 + nb) + (long)b0 * ldl,
                                 ldl, (T)1, B + (long)(b0 + nb) * ldb, ldb, sm);
    }
}

// gemm with the operand staging of gemm_f64_wide where the product qualifies
// (FP64, whole tiles, 16-byte aligned rows), else gemm; the results are bitwise
// the same either way.
template <typename T, bool TA, bool TB>
__device__ inline void gemm_wide(int M, int N, int K, T alpha, const T* A, long lda, const T* B, long ldb, T beta,
                                 T* C, long ldc, LaSmem<T>& sm, const T* Cin = nullptr, long ldcin = 0) {
    if constexpr (sizeof(T) == 8) {
        const int nw = c_gemm_nw[N <= 16 ? 0 : (N <= 32 ? 1 : 2)];
        if (M > 0 && K > 0 && M % 64 == 0 && N % (16 * nw) == 0 && K % TK64 == 0 && lda % 2 == 0 && ldb % 2 == 0 &&
            (((unsigned long)A | (unsigned long)B) & 15ul) == 0) {
            if (nw == 1) gemm_f64_wide<TA, TB, 1>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, sm, Cin, ldcin);
            else if (nw == 2) gemm_f64_wide<TA, TB, 2>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, sm, Cin, ldcin);
            else gemm_f64_wide<TA, TB, 4>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, sm, Cin, ldcin);
            return;
        }
    }
    gemm<T, TA, TB>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, sm, Cin, ldcin);
}

// Solves L x = b for one right-hand side entirely in FP64 (the vectors that feed
// quadratic forms), x overwrites b.  Single warp does the work; ends with a barrier.
template <typename T>
__device__ inline void trsv_lower_f64(int n, const T* L, long ldl, double* b) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int k = lane; k < i; k += 32) s += (double)L[i + (long)k * ldl] * b[k];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) b[i] = (b[i] - s) / (double)L[i + (long)i * ldl];
            __syncwarp();
        }
    }
    __syncthreads();
}

// x = Linv b for a lower-triangular Linv (n x n, ld ldl) that is the inverse
// of a factor, stored with exact zeros above its diagonal: the triangular
// solve as a product, one row per thread, every row over all n columns (a
// uniform trip count, unrolled, so the loads of a row are in flight
// together).  x may alias b.  Ends with a barrier.
template <typename T>
__device__ inline void trmv_lower_inv(int n, const T* Linv, long ldl, double* x, const double* b) {
    double v[2] = {0.0, 0.0};
    for (int h = 0; h < 2; ++h) {
        const int q = threadIdx.x + h * kThreads;
        if (q < n) {
            double s[4] = {0.0, 0.0, 0.0, 0.0};
            int k = 0;
            for (; k + 8 <= n; k += 8) {
#pragma unroll
                for (int u = 0; u < 8; ++u) s[u & 3] += (double)Linv[q + (long)(k + u) * ldl] * b[k + u];
            }
            for (; k < n; ++k) s[0] += (double)Linv[q + (long)k * ldl] * b[k];
            v[h] = (s[0] + s[1]) + (s[2] + s[3]);
        }
    }
    __syncthreads();
    for (int h = 0; h < 2; ++h) {
        const int q = threadIdx.x + h * kThreads;
        if (q < n) x[q] = v[h];
    }
    __syncthreads();
}

// Deterministic CTA sum (fixed thread -> element mapping and tree order).
template <typename T>
__device__ inline double cta_sum(double v, LaSmem<T>& sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm.red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w) s += sm.red[w];
    __syncthreads();
    return s;  // valid in thread 0
}

// In-place lower Cholesky A = L L^T (strict upper part zeroed, like
// Armadillo's chol(X, "lower")).  Diagonal blocks and panels in FP64, trailing
// updates through gemm<T>.  Returns 0, or the 1-based index of the first
// non-positive (or NaN) pivot (LAPACK's info); the factorization then goes on
// with NaNs and the caller reports the region.  *logdet (thread 0) receives
// 2 * sum(log(diag L)) accumulated in FP64.
template <typename T>
__device__ inline int potrf_blocked(int n, T* A, long lda, LaSmem<T>& sm, double* logdet) {
    const int tid = threadIdx.x;
    double ld = 0.0;
    if (tid == 0) sm.flag = 0;
    for (int b0 = 0; b0 < n; b0 += NB) {
        int nb = min(NB, n - b0);
        for (int e = tid; e < nb * nb; e += kThreads) {
            int i = e % nb, j = e / nb;
            sm.D[i][j] = (double)A[(b0 + i) + (long)(b0 + j) * lda];
        }
        __syncthreads();
        // the diagonal block by warp 0, lane i owning row i (right-looking)
        if (tid < 32) {
            const int lane = tid;
            for (int k = 0; k < nb; ++k) {
                if (lane == 0) {
                    double d = sm.D[k][k];
                    if (!(d > 0.0) && sm.flag == 0) sm.flag = b0 + k + 1;
                    double sq = sqrt(d);
                    sm.D[k][k] = sq;
                    sm.inv[k] = 1.0 / sq;
                    ld += 2.0 * log(sq);
                }
                __syncwarp();
                if (lane > k && lane < nb) sm.D[lane][k] *= sm.inv[k];
                __syncwarp();
                // lane i reads column k (final) and writes row i beyond column k
                if (lane > k && lane < nb) {
                    const double lik = sm.D[lane][k];
                    for (int j = k + 1; j <= lane; ++j) sm.D[lane][j] -= lik * sm.D[j][k];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (int e = tid; e < nb * nb; e += kThreads) {
            int i = e % nb, j = e / nb;
            A[(b0 + i) + (long)(b0 + j) * lda] = j <= i ? (T)sm.D[i][j] : (T)0;
        }
        __syncthreads();
        int rest = n - b0 - nb;
        if (rest > 0) {
            // panel: A[b0+nb:, b0:b0+nb] <- A[...] * D^{-T}, in FP64
            for (int row = tid; row < rest; row += kThreads) {
                double x[NB];
                T* p = A + (b0 + nb + row) + (long)b0 * lda;
#pragma unroll
                for (int i = 0; i < NB; ++i) x[i] = i < nb ? (double)p[(long)i * lda] : 0.0;
#pragma unroll
                for (int i = 0; i < NB; ++i) {
                    if (i < nb) {
                        double s = x[i];
#pragma unroll
                        for (int k = 0; k < i; ++k) s -= sm.D[i][k] * x[k];
                        x[i] = s * sm.inv[i];
                    }
                }
#pragma unroll
                for (int i = 0; i < NB; ++i)
                    if (i < nb) p[(long)i * lda] = (T)x[i];
            }
            __syncthreads();
            const T* P = A + (b0 + nb) + (long)b0 * lda;
            gemm<T, false, true>(rest, rest, nb, (T)-1, P, lda, P, lda, (T)1, A + (b0 + nb) + (long)(b0 + nb) * lda,
                                 lda, sm);
            for (int e = tid; e < nb * rest; e += kThreads) {
                int i = e % nb, j = e / nb;
                A[(b0 + i) + (long)(b0 + nb + j) * lda] = (T)0;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    if (tid == 0 && logdet) *logdet = ld;
    return sm.flag;
}


// FP64 Cholesky (and optionally the inverse of the factor) of an n x n
// matrix, n <= 64, staged whole in shared memory (column-major, ld 65),
// right-looking in 16-wide block columns:
//  * each 16 x 16 diagonal block is factored by one warp with lane l holding
//    row l in registers (pivots broadcast by shuffles, 1/sqrt(pivot) by
//    rsqrt), and the same warp inverts the block (lane l: column l);
//  * the panel below it is the product of the panel with the block's inverse
//    (transposed), and the trailing update a rank-16 product, each thread
//    owning rows tx + 16a / columns ty + 16c of the 16 x 16 thread grid;
//  * X = L^{-1} is completed block by block away from the diagonal:
//    X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj.
// n that is not a multiple of 16 is padded with an identity block.  A
// non-positive or NaN pivot sets sm.flag (1-based index, first wins) and the
// factorization goes on with NaNs.  logdet (thread 0) = 2 sum log L_ii.
constexpr int SLD = 65;
constexpr unsigned kFullMask = 0xffffffffu;

// One warp: factors the 16 x 16 block of S at (b0, b0) in place and writes its
// inverse to the same block of X (both with zeros above the diagonal).
static __device__ __noinline__ void potrf_diag16(double* S, double* X, int b0, LaSmem<double>& sm) {
    const int l = threadIdx.x & 31;
    double x[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) x[c] = (l < 16 && c <= l) ? S[(b0 + l) + (b0 + c) * SLD] : 0.0;
    int bad = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const double d = __shfl_sync(kFullMask, x[k], k);
        if (!(d > 0.0) && bad == 0) bad = b0 + k + 1;
        const double r = rsqrt(d);
        if (l == 0) sm.inv[k] = r;
        x[k] = l == k ? d * r : (l > k ? x[k] * r : x[k]);
#pragma unroll
        for (int j = k + 1; j < 16; ++j) {
            const double ljk = __shfl_sync(kFullMask, x[k], j);
            if (l >= j) x[j] = fma(-x[k], ljk, x[j]);
        }
    }
    if (l < 16) {
#pragma unroll
        for (int c = 0; c < 16; ++c) S[(b0 + l) + (b0 + c) * SLD] = c <= l ? x[c] : 0.0;
    }
    if (l == 0 && bad && sm.flag == 0) sm.flag = bad;
    __syncwarp();
    double y[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) y[i] = i == l ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        y[k] *= sm.inv[k];
#pragma unroll
        for (int i = k + 1; i < 16; ++i) y[i] = fma(-S[(b0 + i) + (b0 + k) * SLD], y[k], y[i]);
    }
    if (l < 16) {
#pragma unroll
        for (int i = 0; i < 16; ++i) X[(b0 + i) + (b0 + l) * SLD] = y[i];
    }
}

__device__ inline int potrf_small(int n, double* A, long lda, LaSmem<double>& sm, double* logdet, double* inv,
                                  long ldinv) {
    const int tid = threadIdx.x;
    double* S = &sm.A[0][0];  // 64 x 65 (fits in the operand tile buffers)
    double* X = &sm.B[0][0];
    const int nbk = (n + 15) >> 4, N = nbk << 4;
    {
        // every load issued before the first store (16 columns per thread)
        const int i = tid & 63, j0 = tid >> 6;
        double v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int j = j0 + 4 * q;
            v[q] = (i < n && j < n) ? A[i + (long)j * lda] : (i == j ? 1.0 : 0.0);
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int j = j0 + 4 * q;
            if (i < N && j < N) S[i + j * SLD] = v[q];
        }
    }
    if (tid == 0) sm.flag = 0;
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;
    for (int b = 0; b < nbk; ++b) {
        const int b0 = b << 4;
        if (tid < 32) potrf_diag16(S, X, b0, sm);
        __syncthreads();
        const int rest = N - b0 - 16;
        if (rest > 0) {
            const int r0 = b0 + 16, na = rest >> 4;
            // panel: L[i][b0+k] = sum_{c<=k} A[i][b0+c] Y[k][c], Y the block's inverse
            double v[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                if (c <= ty) {
                    const double yk = X[(b0 + ty) + (b0 + c) * SLD];
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        if (a < na) v[a] = fma(S[(r0 + tx + 16 * a) + (b0 + c) * SLD], yk, v[a]);
                }
            }
            __syncthreads();
#pragma unroll
            for (int a = 0; a < 3; ++a)
                if (a < na) S[(r0 + tx + 16 * a) + (b0 + ty) * SLD] = v[a];
            __syncthreads();
            // trailing update of the lower triangle
            double acc[3][3];
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int e = 0; e < 3; ++e) acc[a][e] = 0.0;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                double li[3], lj[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    li[a] = a < na ? S[(r0 + tx + 16 * a) + (b0 + k) * SLD] : 0.0;
                    lj[a] = a < na ? S[(r0 + ty + 16 * a) + (b0 + k) * SLD] : 0.0;
                }
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int e = 0; e <= a; ++e) acc[a][e] = fma(li[a], lj[e], acc[a][e]);
            }
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int e = 0; e <= a; ++e)
                    if (a < na && (a > e || tx >= ty)) S[(r0 + tx + 16 * a) + (r0 + ty + 16 * e) * SLD] -= acc[a][e];
            __syncthreads();
        }
    }
    double part = 0.0;
    for (int i = tid; i < n; i += kThreads) part += log(S[i + i * SLD]);
    const double sum = cta_sum(part, sm);
    if (tid == 0 && logdet) *logdet = 2.0 * sum;
    {
        const int i = tid & 63;
        for (int j = tid >> 6; j < n; j += kThreads / 64)
            if (i < n) A[i + (long)j * lda] = i >= j ? S[i + j * SLD] : 0.0;
    }
    if (inv) {
        // off-diagonal blocks of X by distance dd from the diagonal; thread
        // (tx, ty) forms element (tx, ty) of each block
        for (int dd = 1; dd < nbk; ++dd) {
            const int np = nbk - dd;
            double v[3];
#pragma unroll
            for (int u = 0; u < 3; ++u) {
                v[u] = 0.0;
                if (u < np) {
                    const int row = 16 * (u + dd) + tx, col = 16 * u + ty;
                    double s[4] = {0.0, 0.0, 0.0, 0.0};
                    for (int kb = u; kb < u + dd; ++kb) {
#pragma unroll
                        for (int c = 0; c < 16; ++c)
                            s[c & 3] = fma(S[row + (16 * kb + c) * SLD], X[(16 * kb + c) + col * SLD], s[c & 3]);
                    }
                    v[u] = (s[0] + s[1]) + (s[2] + s[3]);
                }
            }
#pragma unroll
            for (int u = 0; u < 3; ++u)
                if (u < np) X[(16 * (u + dd) + tx) + (16 * u + ty) * SLD] = v[u];
            __syncthreads();
#pragma unroll
            for (int u = 0; u < 3; ++u) {
                if (u < np) {
                    const int ib = u + dd, row = 16 * ib + tx, col = 16 * u + ty;
                    double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
                    for (int c = 0; c < 16; ++c)
                        if (c <= tx) s[c & 3] = fma(X[row + (16 * ib + c) * SLD], X[(16 * ib + c) + col * SLD], s[c & 3]);
                    v[u] = -((s[0] + s[1]) + (s[2] + s[3]));
                }
            }
            __syncthreads();
#pragma unroll
            for (int u = 0; u < 3; ++u)
                if (u < np) X[(16 * (u + dd) + tx) + (16 * u + ty) * SLD] = v[u];
            __syncthreads();
        }
        const int i = tid & 63;
        for (int j = tid >> 6; j < n; j += kThreads / 64)
            if (i < n) inv[i + (long)j * ldinv] = i >= j ? X[i + j * SLD] : 0.0;
    }
    __syncthreads();
    return sm.flag;
}

// FP64 Cholesky with the inverse of the factor for 64 < n <= 128, as a 2 x 2
// block factorization around potrf_small (64 + n2 with n2 = n - 64):
//   L11 = chol(A11), X11 = L11^{-1};  L21 = A21 X11^T;  A22 -= L21 L21^T;
//   L22 = chol(A22), X22 = L22^{-1};  X21 = -X22 (L21 X11)
// so that everything but the two diagonal factorizations runs as products on
// the tensor pipe.  A and inv get zeros above the diagonal.  Returns 0 or the
// 1-based index of the first bad pivot; logdet (thread 0) = 2 sum log L_ii.
__device__ inline int potrf_mid(int n, double* A, long lda, LaSmem<double>& sm, double* logdet, double* inv,
                                long ldinv) {
    const int n2 = n - 64;
    double ld1 = 0.0, ld2 = 0.0;
    const int info1 = potrf_small(64, A, lda, sm, &ld1, inv, ldinv);
    double* A21 = A + 64;
    double* A22 = A + 64 + 64 * lda;
    double* X21 = inv + 64;
    double* X22 = inv + 64 + 64 * ldinv;
    // L21 = A21 X11^T in place (a single output tile reads all of A21 first)
    gemm<double, false, true, true>(n2, 64, 64, 1.0, A21, lda, inv, ldinv, 0.0, A21, lda, sm);
    gemm<double, false, true>(n2, n2, 64, -1.0, A21, lda, A21, lda, 1.0, A22, lda, sm);
    const int info2 = potrf_small(n2, A22, lda, sm, &ld2, X22, ldinv);
    gemm<double, false, false>(n2, 64, 64, 1.0, A21, lda, inv, ldinv, 0.0, X21, ldinv, sm);
    gemm<double, false, false, true>(n2, 64, n2, -1.0, X22, ldinv, X21, ldinv, 0.0, X21, ldinv, sm);
    for (int e = threadIdx.x; e < 64 * n2; e += kThreads) {
        const int i = e & 63, j = 64 + (e >> 6);
        A[i + (long)j * lda] = 0.0;
        inv[i + (long)j * ldinv] = 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0 && logdet) *logdet = ld1 + ld2;
    return info1 ? info1 : (info2 ? info2 + 64 : 0);
}

// In-place lower Cholesky (see potrf_blocked); FP64 matrices up to 64 go
// through potrf_small, and up to 128 through potrf_mid when the inverse is
// asked for.  With `inv`, L^{-1} is also written there (ld ldinv).
template <typename T>
__device__ inline int potrf_lower(int n, T* A, long lda, LaSmem<T>& sm, double* logdet, T* inv = nullptr,
                                  long ldinv = 0) {
    if constexpr (sizeof(T) == 8) {
        if (n <= 64) return potrf_small(n, A, lda, sm, logdet, inv, ldinv);
        if (n <= 128 && inv) return potrf_mid(n, A, lda, sm, logdet, inv, ldinv);
    }
    const int info = potrf_blocked(n, A, lda, sm, logdet);
    if (inv) {
        for (long e = threadIdx.x; e < (long)n * n; e += kThreads) {
            const int i = (int)(e % n), j = (int)(e / n);
            inv[i + (long)j * ldinv] = i == j ? (T)1 : (T)0;
        }
        __syncthreads();
        trsm_left_lower<T>(n, n, A, lda, inv, ldinv, sm);
    }
    return info;
}

}  // namespace mra
