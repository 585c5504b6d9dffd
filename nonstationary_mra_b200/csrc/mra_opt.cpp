// Bound-constrained derivative-free minimiser (include/mra_surrogate.h,
// mra_opt_minimize): the trust-region method with quadratic interpolation
// models that Powell published as BOBYQA (M.J.D. Powell, "The BOBYQA
// algorithm for bound constrained optimization without derivatives",
// DAMTP 2009/NA06), which the reference calls through
// dlib::find_min_bobyqa (src/optimization.cpp:158-192).
//
// Written from the published description, in a plain form:
//   * the interpolation set starts at x0 and x0 +- rho_begin e_i (stepping
//     inwards at a bound), so that for npt = 2n+1 the first model has the
//     exact gradient and diagonal second derivatives of those points;
//   * every model is the one of least Frobenius-norm change of the second
//     derivative matrix that interpolates all npt points, obtained by solving
//     the (npt+n+1) KKT system afresh (dense LU), not by Powell's updating of
//     its inverse -- n is small here and the direct solve is the simpler,
//     well-conditioned choice;
//   * the step minimises the model in the trust region intersected with the
//     bounds by truncated conjugate gradients with an active set of bounds;
//   * the point to drop is chosen by the Lagrange function values weighted by
//     distance; far points are replaced by model-improvement steps before the
//     radius bound rho is reduced (rho_begin -> rho_end as in BOBYQA).
#include <algorithm>
#include <cmath>
#include <limits>
#include <string>
#include <vector>

#include "../../include/mra_surrogate.h"

namespace mra {
void set_last_error(const char* msg);
}

namespace {

// Dense LU with partial pivoting of a k x k row-major matrix.
struct Lu {
    int k = 0;
    std::vector<double> a;
    std::vector<int> piv;
    bool factor(int k_, const std::vector<double>& m) {
        k = k_;
        a = m;
        piv.resize(k);
        for (int c = 0; c < k; ++c) {
            int p = c;
            double best = std::fabs(a[(long)c * k + c]);
            for (int r = c + 1; r < k; ++r)
                if (std::fabs(a[(long)r * k + c]) > best) best = std::fabs(a[(long)r * k + c]), p = r;
            if (!(best > 0)) return false;
            piv[c] = p;
            if (p != c)
                for (int j = 0; j < k; ++j) std::swap(a[(long)c * k + j], a[(long)p * k + j]);
            double d = a[(long)c * k + c];
            for (int r = c + 1; r < k; ++r) {
                double f = a[(long)r * k + c] / d;
                a[(long)r * k + c] = f;
                if (f != 0)
                    for (int j = c + 1; j < k; ++j) a[(long)r * k + j] -= f * a[(long)c * k + j];
            }
        }
        return true;
    }
    // Solves A x = b in place: the row interchanges first, then L, then U.
    void solve(std::vector<double>& b) const {
        for (int c = 0; c < k; ++c)
            if (piv[c] != c) std::swap(b[c], b[piv[c]]);
        for (int c = 0; c < k; ++c)
            for (int r = c + 1; r < k; ++r) b[r] -= a[(long)r * k + c] * b[c];
        for (int r = k - 1; r >= 0; --r) {
            double s = b[r];
            for (int j = r + 1; j < k; ++j) s -= a[(long)r * k + j] * b[j];
            b[r] = s / a[(long)r * k + r];
        }
    }
};

double dot(const double* a, const double* b, int n) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

class Bobyqa {
  public:
    Bobyqa(int n, const double* lo, const double* hi, const mra_opt_config& cfg, mra_objective_fn f, void* user)
        : n_(n), lo_(lo, lo + n), hi_(hi, hi + n), f_(f), user_(user) {
        npt_ = cfg.npt > 0 ? cfg.npt : 2 * n + 1;
        rho_beg_ = cfg.rho_begin;
        rho_end_ = cfg.rho_end;
        max_evals_ = cfg.max_evals;
    }

    // Returns the status code of mra_opt_result.
    int run(double* x, mra_opt_result* res) {
        const int n = n_;
        std::vector<double> x0(x, x + n);
        for (int i = 0; i < n; ++i) x0[i] = std::min(std::max(x0[i], lo_[i]), hi_[i]);
        rho_ = rho_beg_;
        delta_ = rho_;
        Y_.assign((long)npt_ * n, 0.0);
        F_.assign(npt_, 0.0);
        H_.assign((long)n * n, 0.0);
        int st = initial_points(x0);
        if (st < 0) {
            int ntr = 0;
            while (true) {
                st = iterate(ntr);
                if (st >= 0) break;
            }
        }
        const double* xb = &Y_[(long)kopt_ * n];
        std::copy(xb, xb + n, x);
        if (res) {
            res->f_best = F_.empty() ? std::numeric_limits<double>::quiet_NaN() : F_[kopt_];
            res->evals = evals_;
            res->status = st;
            res->rho_final = rho_;
        }
        return st;
    }

  private:
    int n_, npt_;
    std::vector<double> lo_, hi_;
    mra_objective_fn f_;
    void* user_;
    double rho_beg_, rho_end_, rho_ = 0, delta_ = 0;
    int max_evals_ = 0, evals_ = 0, kopt_ = 0, filled_ = 0;
    std::vector<double> Y_, F_, H_, g_;
    Lu lu_;
    bool lu_ok_ = false;

    // -1: keep going; else a final status
    int evaluate(const std::vector<double>& x, double* fx) {
        if (evals_ >= max_evals_) return 1;
        int32_t stop = 0;
        double v = f_(x.data(), user_, &stop);
        ++evals_;
        *fx = v;
        if (stop || !std::isfinite(v)) return 2;
        return -1;
    }

    int initial_points(const std::vector<double>& x0) {
        const int n = n_;
        auto put = [&](int k, const std::vector<double>& x) -> int {
            double fx;
            int s = evaluate(x, &fx);
            if (s == 1) return 1;
            std::copy(x.begin(), x.end(), &Y_[(long)k * n]);
            F_[k] = fx;
            filled_ = k + 1;
            if (!std::isfinite(fx)) return 2;
            if (fx < F_[kopt_]) kopt_ = k;
            return s;
        };
        kopt_ = 0;
        int s = put(0, x0);
        if (s >= 0) return s;
        // +- rho along each axis, stepping inwards at a bound
        int k = 1;
        for (int i = 0; i < n && k < npt_; ++i) {
            std::vector<double> x = x0;
            double up = hi_[i] - x0[i], dn = x0[i] - lo_[i];
            double step = up >= rho_ ? rho_ : (dn >= rho_ ? -rho_ : (up >= dn ? up : -dn));
            x[i] = x0[i] + step;
            s = put(k++, x);
            if (s >= 0) return s;
        }
        for (int i = 0; i < n && k < npt_; ++i) {
            std::vector<double> x = x0;
            double first = Y_[(long)(i + 1) * n + i] - x0[i];
            double step = -first;
            if (x0[i] + step < lo_[i] || x0[i] + step > hi_[i]) step = 2 * first;
            step = std::min(std::max(x0[i] + step, lo_[i]), hi_[i]) - x0[i];
            if (step == 0) step = first / 2;
            x[i] = x0[i] + step;
            s = put(k++, x);
            if (s >= 0) return s;
        }
        // further points (npt > 2n+1): pairs of axes
        for (int i = 0; i < n && k < npt_; ++i)
            for (int j = i + 1; j < n && k < npt_; ++j) {
                std::vector<double> x = x0;
                x[i] = Y_[(long)(i + 1) * n + i];
                x[j] = Y_[(long)(j + 1) * n + j];
                s = put(k++, x);
                if (s >= 0) return s;
            }
        if (k < npt_) npt_ = k;
        return -1;
    }

    const double* xopt() const { return &Y_[(long)kopt_ * n_]; }

    // Least-Frobenius-change model around x_opt: fills g_, updates H_.
    bool build_model() {
        const int n = n_, m = npt_, K = m + n + 1;
        std::vector<double> W((long)K * K, 0.0), z((long)m * n);
        const double* xo = xopt();
        for (int k = 0; k < m; ++k)
            for (int i = 0; i < n; ++i) z[(long)k * n + i] = Y_[(long)k * n + i] - xo[i];
        for (int k = 0; k < m; ++k) {
            for (int l = 0; l < m; ++l) {
                double d = dot(&z[(long)k * n], &z[(long)l * n], n);
                W[(long)k * K + l] = 0.5 * d * d;
            }
            W[(long)k * K + m] = W[(long)m * K + k] = 1.0;
            for (int i = 0; i < n; ++i) W[(long)k * K + m + 1 + i] = W[(long)(m + 1 + i) * K + k] = z[(long)k * n + i];
        }
        lu_ok_ = lu_.factor(K, W);
        if (!lu_ok_) return false;
        std::vector<double> b(K, 0.0);
        std::vector<double> Hz(n);
        for (int k = 0; k < m; ++k) {
            const double* zk = &z[(long)k * n];
            for (int i = 0; i < n; ++i) Hz[i] = dot(&H_[(long)i * n], zk, n);
            b[k] = F_[k] - F_[kopt_] - 0.5 * dot(zk, Hz.data(), n);
        }
        lu_.solve(b);
        g_.assign(b.begin() + m + 1, b.begin() + m + 1 + n);
        for (int k = 0; k < m; ++k) {
            const double lam = b[k];
            if (lam == 0) continue;
            const double* zk = &z[(long)k * n];
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) H_[(long)i * n + j] += lam * zk[i] * zk[j];
        }
        return true;
    }

    // Lagrange function values of every point at x_opt + s.
    std::vector<double> lagrange(const std::vector<double>& s) const {
        const int n = n_, m = npt_, K = m + n + 1;
        std::vector<double> w(K, 0.0);
        for (int k = 0; k < m; ++k) {
            double d = 0;
            for (int i = 0; i < n; ++i) d += (Y_[(long)k * n + i] - xopt()[i]) * s[i];
            w[k] = 0.5 * d * d;
        }
        w[m] = 1.0;
        for (int i = 0; i < n; ++i) w[m + 1 + i] = s[i];
        lu_.solve(w);
        w.resize(m);
        return w;
    }

    double model_change(const std::vector<double>& s) const {
        const int n = n_;
        double q = dot(g_.data(), s.data(), n);
        for (int i = 0; i < n; ++i) q += 0.5 * s[i] * dot(&H_[(long)i * n], s.data(), n);
        return q;  // Q(x_opt + s) - Q(x_opt)
    }

    // min g.s + s.H.s/2, |s| <= delta, lo <= x_opt + s <= hi (truncated CG, active bounds)
    std::vector<double> tr_step(double delta) const {
        const int n = n_;
        const double* xo = xopt();
        std::vector<double> s(n, 0.0), r(n), p(n), Hp(n);
        std::vector<char> fixed(n, 0);
        auto grad_at = [&](std::vector<double>& gr) {
            for (int i = 0; i < n; ++i) gr[i] = g_[i] + dot(&H_[(long)i * n], s.data(), n);
        };
        std::vector<double> gr(n);
        grad_at(gr);
        for (int i = 0; i < n; ++i) {
            if ((xo[i] <= lo_[i] && gr[i] >= 0) || (xo[i] >= hi_[i] && gr[i] <= 0)) fixed[i] = 1;
        }
        for (int restart = 0; restart <= n; ++restart) {
            grad_at(gr);
            for (int i = 0; i < n; ++i) r[i] = fixed[i] ? 0.0 : -gr[i];
            double rr = dot(r.data(), r.data(), n);
            const double rr0 = rr;
            if (rr <= 1e-30) break;
            p = r;
            bool hit_bound = false, done = false;
            for (int it = 0; it < 2 * n + 2; ++it) {
                for (int i = 0; i < n; ++i) Hp[i] = fixed[i] ? 0.0 : dot(&H_[(long)i * n], p.data(), n);
                for (int i = 0; i < n; ++i)
                    if (fixed[i]) Hp[i] = 0;
                double kappa = dot(p.data(), Hp.data(), n);
                // step to the trust-region boundary
                double ss = dot(s.data(), s.data(), n), sp = dot(s.data(), p.data(), n), pp = dot(p.data(), p.data(), n);
                double disc = sp * sp + pp * (delta * delta - ss);
                double a_tr = pp > 0 ? (-sp + std::sqrt(std::max(disc, 0.0))) / pp : 0.0;
                // step to the nearest bound
                double a_bd = std::numeric_limits<double>::infinity();
                int ibd = -1;
                for (int i = 0; i < n; ++i) {
                    if (fixed[i] || p[i] == 0) continue;
                    double lim = p[i] > 0 ? (hi_[i] - xo[i] - s[i]) / p[i] : (lo_[i] - xo[i] - s[i]) / p[i];
                    lim = std::max(lim, 0.0);
                    if (lim < a_bd) a_bd = lim, ibd = i;
                }
                double a = kappa > 0 ? rr / kappa : std::numeric_limits<double>::infinity();
                int why = 0;  // 0 interior, 1 trust region, 2 bound
                if (a_tr <= a) a = a_tr, why = 1;
                if (a_bd < a) a = a_bd, why = 2;
                for (int i = 0; i < n; ++i) s[i] += a * p[i];
                if (why == 1) {
                    done = true;
                    break;
                }
                if (why == 2) {
                    const double* xb = xo;
                    s[ibd] = (p[ibd] > 0 ? hi_[ibd] : lo_[ibd]) - xb[ibd];
                    fixed[ibd] = 1;
                    hit_bound = true;
                    break;
                }
                for (int i = 0; i < n; ++i) r[i] -= a * Hp[i];
                double rr_new = dot(r.data(), r.data(), n);
                if (rr_new <= 1e-4 * rr0) {
                    done = true;
                    break;
                }
                double beta = rr_new / rr;
                rr = rr_new;
                for (int i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
            }
            if (done || !hit_bound) break;
        }
        for (int i = 0; i < n; ++i) s[i] = std::min(std::max(xo[i] + s[i], lo_[i]), hi_[i]) - xo[i];
        return s;
    }

    // Replaces point k by x (value fx).
    void replace(int k, const std::vector<double>& x, double fx) {
        std::copy(x.begin(), x.end(), &Y_[(long)k * n_]);
        F_[k] = fx;
        if (fx < F_[kopt_]) kopt_ = k;
    }

    double dist_to_opt(int k) const {
        double d = 0;
        for (int i = 0; i < n_; ++i) {
            double t = Y_[(long)k * n_ + i] - xopt()[i];
            d += t * t;
        }
        return std::sqrt(d);
    }

    // Model-improvement step for the point k: the candidate step of length
    // delta (axes, towards point k, along the gradient of its Lagrange
    // function) with the largest |l_k|.
    std::vector<double> geometry_step(int k, double delta) const {
        const int n = n_;
        const double* xo = xopt();
        std::vector<std::vector<double>> cand;
        auto add = [&](std::vector<double> d) {
            double nd = std::sqrt(dot(d.data(), d.data(), n));
            if (!(nd > 0)) return;
            for (int sgn = -1; sgn <= 1; sgn += 2) {
                std::vector<double> s(n);
                for (int i = 0; i < n; ++i)
                    s[i] = std::min(std::max(xo[i] + sgn * delta * d[i] / nd, lo_[i]), hi_[i]) - xo[i];
                cand.push_back(s);
            }
        };
        std::vector<double> d(n);
        for (int i = 0; i < n; ++i) d[i] = Y_[(long)k * n + i] - xo[i];
        add(d);
        // gradient of l_k at x_opt: coefficient block of W^{-1} e_k
        {
            std::vector<double> e(npt_ + n + 1, 0.0);
            e[k] = 1.0;
            lu_.solve(e);
            std::vector<double> gk(e.begin() + npt_ + 1, e.end());
            add(gk);
        }
        for (int i = 0; i < n; ++i) {
            std::vector<double> a(n, 0.0);
            a[i] = 1.0;
            add(a);
        }
        double best = -1;
        std::vector<double> sbest(n, 0.0);
        for (auto& s : cand) {
            // skip steps that land on (or next to) a point of the set
            bool dup = false;
            for (int j = 0; j < npt_ && !dup; ++j) {
                if (j == k) continue;
                double dd = 0;
                for (int i = 0; i < n; ++i) {
                    double t = xo[i] + s[i] - Y_[(long)j * n + i];
                    dd += t * t;
                }
                dup = std::sqrt(dd) < 1e-3 * delta;
            }
            if (dup) continue;
            double v = std::fabs(lagrange(s)[k]);
            if (v > best) best = v, sbest = s;
        }
        return sbest;
    }

    int far_point(double thresh) const {
        int kf = -1;
        double dmax = thresh;
        for (int k = 0; k < npt_; ++k) {
            if (k == kopt_) continue;
            double d = dist_to_opt(k);
            if (d > dmax) dmax = d, kf = k;
        }
        return kf;
    }

    // Reduces rho (BOBYQA's schedule); returns 0 when rho_end was reached.
    bool reduce_rho() {
        if (rho_ <= rho_end_) return false;
        double ratio = rho_ / rho_end_;
        double rnew = ratio <= 16 ? rho_end_ : (ratio <= 250 ? std::sqrt(ratio) * rho_end_ : 0.1 * rho_);
        delta_ = std::max(0.5 * rho_, rnew);
        rho_ = rnew;
        return true;
    }

    int iterate(int& ntr) {
        const int n = n_;
        if (!build_model()) return 3;
        std::vector<double> s = tr_step(delta_);
        double snorm = std::sqrt(dot(s.data(), s.data(), n));
        if (snorm < 0.5 * rho_) {
            // short step: fix the geometry first, else lower rho
            int kf = far_point(2.0 * rho_);
            if (kf >= 0) return improve_geometry(kf);
            delta_ = std::max(0.1 * delta_, rho_);
            if (!reduce_rho()) return 0;
            return -1;
        }
        double pred = -model_change(s);
        std::vector<double> x(n);
        for (int i = 0; i < n; ++i) x[i] = std::min(std::max(xopt()[i] + s[i], lo_[i]), hi_[i]);
        double fx;
        int st = evaluate(x, &fx);
        if (st >= 0) return st;
        ++ntr;
        const double fopt = F_[kopt_];
        double ratio = pred > 0 ? (fopt - fx) / pred : -1.0;
        if (ratio <= 0.1) delta_ = std::min(0.5 * delta_, snorm);
        else if (ratio <= 0.7) delta_ = std::max(0.5 * delta_, snorm);
        else delta_ = std::max(0.5 * delta_, 2.0 * snorm);
        if (delta_ <= 1.5 * rho_) delta_ = rho_;
        // point to drop: largest distance-weighted |Lagrange value| at x
        std::vector<double> lag = lagrange(s);
        int kdrop = -1;
        double best = -1;
        for (int k = 0; k < npt_; ++k) {
            if (k == kopt_ && fx >= fopt) continue;
            double d = dist_to_opt(k) / std::max(delta_, rho_);
            double w = std::max(1.0, d * d);
            double v = std::fabs(lag[k]) * w * w;
            if (v > best) best = v, kdrop = k;
        }
        if (kdrop >= 0) replace(kdrop, x, fx);
        if (ratio < 0.1) {
            int kf = far_point(2.0 * delta_);
            if (kf >= 0) return improve_geometry(kf);
            if (delta_ <= rho_ && fx >= fopt) {
                if (!reduce_rho()) return 0;
            }
        }
        return -1;
    }

    int improve_geometry(int kf) {
        if (!build_model()) return 3;
        double dg = std::max(std::min(0.1 * dist_to_opt(kf), delta_), rho_);
        std::vector<double> s = geometry_step(kf, dg);
        std::vector<double> x(n_);
        for (int i = 0; i < n_; ++i) x[i] = xopt()[i] + s[i];
        double fx;
        int st = evaluate(x, &fx);
        if (st >= 0) return st;
        replace(kf, x, fx);
        return -1;
    }
};

}  // namespace

extern "C" mra_status mra_opt_minimize(int32_t n, double* x, const double* lower, const double* upper,
                                       const mra_opt_config* cfg, mra_objective_fn f, void* user,
                                       mra_opt_result* out) {
    if (n < 1 || !x || !lower || !upper || !cfg || !f) {
        mra::set_last_error("mra_opt_minimize: bad argument");
        return MRA_ERR_ARG;
    }
    const int npt = cfg->npt > 0 ? cfg->npt : 2 * n + 1;
    if (npt < n + 2 || npt > (n + 1) * (n + 2) / 2) {
        mra::set_last_error("mra_opt_minimize: npt must be in [n+2, (n+1)(n+2)/2]");
        return MRA_ERR_ARG;
    }
    if (!(cfg->rho_begin > 0) || !(cfg->rho_end > 0) || cfg->rho_end > cfg->rho_begin || cfg->max_evals < npt + 1) {
        mra::set_last_error("mra_opt_minimize: need 0 < rho_end <= rho_begin and max_evals > npt");
        return MRA_ERR_ARG;
    }
    for (int i = 0; i < n; ++i) {
        if (!(upper[i] - lower[i] >= 2 * cfg->rho_begin)) {
            mra::set_last_error("mra_opt_minimize: every bound range must be at least 2 rho_begin (as in BOBYQA)");
            return MRA_ERR_ARG;
        }
    }
    Bobyqa b(n, lower, upper, *cfg, f, user);
    b.run(x, out);
    return MRA_OK;
}
