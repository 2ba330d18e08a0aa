/*
 * Bound-constrained derivative-free maximisation for the MLE driver.
 *
 * The reference maximises MLE_alg with NLopt's BOBYQA (nlopt 2.7.0,
 * examples/synthetic_dmle_test.c:140-142,283-284; bounds and ftol_abs from
 * init_optimizer, misc/compute/MLE_misc.c:1352-1366).  NLopt is a third-party
 * library that is not part of the reference tree, so this file provides the
 * same kind of method, written from the published description of BOBYQA
 * (M. J. D. Powell, "The BOBYQA algorithm for bound constrained optimization
 * without derivatives", Cambridge report DAMTP 2009/NA06):
 *
 *   - a quadratic model interpolating m = 2n+1 points, initialised along the
 *     coordinate axes and afterwards updated so that the change of its
 *     Hessian has least Frobenius norm (solved here directly from the
 *     (m + n + 1) KKT system, which is tiny for the 3-4 Matern parameters);
 *   - a trust-region step that minimises the model inside the box and the
 *     ball (truncated conjugate gradients with active-bound fixing);
 *   - the new point replaces the interpolation point whose Lagrange function,
 *     weighted by its distance, is largest; geometry-improving steps when the
 *     model is poor; a resolution rho decreasing from rhobeg to rhoend.
 *
 * It is not a transcription of NLopt's code, so its iterate sequence differs;
 * agreement with the reference is measured on the maximiser and the value.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/exageostat_b200.h"

namespace {

typedef double (*Objective)(unsigned, const double *, double *, void *);

struct Problem {
    int n;
    Objective f;
    void *data;
    const double *lb, *ub;
    int evals = 0, maxeval;
    double best_f = INFINITY; /* minimisation of -f */
    std::vector<double> best_x;
    double eval(const double *x)
    {
        ++evals;
        double v = -f((unsigned)n, x, nullptr, data);
        if (!(v == v)) v = INFINITY; /* NaN -> worst */
        if (v < best_f) {
            best_f = v;
            best_x.assign(x, x + n);
        }
        return v;
    }
};

/* Solves A x = b in place (Gaussian elimination, partial pivoting);
 * returns false if A is numerically singular. */
bool solve_dense(std::vector<double> A, std::vector<double> &b, int n)
{
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (fabs(A[r * n + c]) > fabs(A[p * n + c])) p = r;
        if (fabs(A[p * n + c]) < 1e-300) return false;
        if (p != c) {
            for (int k = 0; k < n; ++k) std::swap(A[c * n + k], A[p * n + k]);
            std::swap(b[c], b[p]);
        }
        for (int r = c + 1; r < n; ++r) {
            const double m = A[r * n + c] / A[c * n + c];
            if (m == 0) continue;
            for (int k = c; k < n; ++k) A[r * n + k] -= m * A[c * n + k];
            b[r] -= m * b[c];
        }
    }
    for (int c = n - 1; c >= 0; --c) {
        double s = b[c];
        for (int k = c + 1; k < n; ++k) s -= A[c * n + k] * b[k];
        b[c] = s / A[c * n + c];
    }
    return true;
}

struct Model {
    int n, m;
    std::vector<double> xb;          /* base point */
    std::vector<double> Y;           /* m x n interpolation points */
    std::vector<double> F;           /* values */
    double c = 0;
    std::vector<double> g, H;        /* gradient at xb, n x n Hessian */

    double value(const double *x) const
    {
        double q = c;
        for (int i = 0; i < n; ++i) {
            const double di = x[i] - xb[i];
            q += g[i] * di;
            double hd = 0;
            for (int j = 0; j < n; ++j) hd += H[i * n + j] * (x[j] - xb[j]);
            q += 0.5 * di * hd;
        }
        return q;
    }
    /* gradient of the model at x */
    void grad(const double *x, double *out) const
    {
        for (int i = 0; i < n; ++i) {
            double s = g[i];
            for (int j = 0; j < n; ++j) s += H[i * n + j] * (x[j] - xb[j]);
            out[i] = s;
        }
    }
    /* KKT matrix of least-Frobenius-norm interpolation on the current points */
    std::vector<double> kkt() const
    {
        const int K = m + n + 1;
        std::vector<double> W((size_t)K * K, 0.0);
        for (int a = 0; a < m; ++a) {
            for (int b = 0; b < m; ++b) {
                double dot = 0;
                for (int i = 0; i < n; ++i) dot += (Y[a * n + i] - xb[i]) * (Y[b * n + i] - xb[i]);
                W[a * K + b] = 0.5 * dot * dot;
            }
            W[a * K + m] = W[m * K + a] = 1.0;
            for (int i = 0; i < n; ++i) W[a * K + m + 1 + i] = W[(m + 1 + i) * K + a] = Y[a * n + i] - xb[i];
        }
        return W;
    }
    /* Least-Frobenius-norm change of the model so it interpolates F. */
    bool update()
    {
        const int K = m + n + 1;
        std::vector<double> rhs((size_t)K, 0.0);
        for (int a = 0; a < m; ++a) rhs[a] = F[a] - value(&Y[a * n]);
        if (!solve_dense(kkt(), rhs, K)) return false;
        c += rhs[m];
        for (int i = 0; i < n; ++i) g[i] += rhs[m + 1 + i];
        for (int a = 0; a < m; ++a)
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j)
                    H[i * n + j] += rhs[a] * (Y[a * n + i] - xb[i]) * (Y[a * n + j] - xb[j]);
        return true;
    }
    /* moves the base point to x (the model itself is unchanged): keeps the
     * KKT system well scaled as the points cluster around the optimum */
    void rebase(const double *x)
    {
        std::vector<double> gx((size_t)n);
        grad(x, gx.data());
        c = value(x);
        g = gx;
        xb.assign(x, x + n);
    }
    /* values of all m Lagrange functions at x */
    bool lagrange(const double *x, std::vector<double> &out) const
    {
        const int K = m + n + 1;
        std::vector<double> W = kkt();
        out.assign((size_t)m, 0.0);
        /* column t of W^-1 gives the coefficients of Lagrange function t; by
         * symmetry l(x) = W^-1 v(x) with v = [w(x); 1; x - xb] */
        std::vector<double> v((size_t)K, 0.0);
        for (int a = 0; a < m; ++a) {
            double dot = 0;
            for (int i = 0; i < n; ++i) dot += (Y[a * n + i] - xb[i]) * (x[i] - xb[i]);
            v[a] = 0.5 * dot * dot;
        }
        v[m] = 1.0;
        for (int i = 0; i < n; ++i) v[m + 1 + i] = x[i] - xb[i];
        if (!solve_dense(W, v, K)) return false;
        for (int a = 0; a < m; ++a) out[a] = v[a];
        return true;
    }
};

/* Approximately minimises the model within the box and ||s|| <= delta from
 * xo: truncated conjugate gradients on the free variables; a variable that
 * reaches a bound is fixed there and CG restarts. */
void trust_region_step(const Model &M, const double *xo, const double *lb, const double *ub, double delta,
                       std::vector<double> &s)
{
    const int n = M.n;
    s.assign((size_t)n, 0.0);
    std::vector<double> x(xo, xo + n), gq((size_t)n), d((size_t)n), hd((size_t)n);
    std::vector<char> fixed((size_t)n, 0);
    for (int restart = 0; restart <= n; ++restart) {
        M.grad(x.data(), gq.data());
        for (int i = 0; i < n; ++i)
            if ((x[i] <= lb[i] && gq[i] > 0) || (x[i] >= ub[i] && gq[i] < 0)) fixed[i] = 1;
        for (int i = 0; i < n; ++i) d[i] = fixed[i] ? 0.0 : -gq[i];
        double gg = 0;
        for (int i = 0; i < n; ++i) gg += d[i] * d[i];
        if (gg < 1e-30) return;
        bool hit_bound = false;
        for (int it = 0; it < n && !hit_bound; ++it) {
            for (int i = 0; i < n; ++i) {
                double t = 0;
                for (int j = 0; j < n; ++j) t += M.H[i * n + j] * d[j];
                hd[i] = t;
            }
            double dhd = 0, gd = 0, ss = 0, sd = 0, dd = 0;
            for (int i = 0; i < n; ++i) {
                dhd += d[i] * hd[i];
                gd += gq[i] * d[i];
                ss += s[i] * s[i];
                sd += s[i] * d[i];
                dd += d[i] * d[i];
            }
            /* largest step along d inside the ball */
            const double disc = sd * sd + dd * (delta * delta - ss);
            double amax = disc > 0 ? (-sd + sqrt(disc)) / dd : 0.0;
            /* and inside the box */
            int blocking = -1;
            for (int i = 0; i < n; ++i) {
                if (d[i] > 0 && (ub[i] - x[i]) / d[i] < amax) {
                    amax = (ub[i] - x[i]) / d[i];
                    blocking = i;
                } else if (d[i] < 0 && (lb[i] - x[i]) / d[i] < amax) {
                    amax = (lb[i] - x[i]) / d[i];
                    blocking = i;
                }
            }
            double alpha = amax;
            bool interior = false;
            if (dhd > 0 && -gd / dhd < amax) {
                alpha = -gd / dhd;
                interior = true;
            }
            if (alpha < 0) alpha = 0;
            for (int i = 0; i < n; ++i) {
                s[i] += alpha * d[i];
                x[i] = std::min(ub[i], std::max(lb[i], xo[i] + s[i]));
                gq[i] += alpha * hd[i];
            }
            if (!interior) {
                if (blocking < 0) return; /* reached the trust-region boundary */
                fixed[blocking] = 1;
                hit_bound = true;
                break;
            }
            double gnew = 0;
            for (int i = 0; i < n; ++i)
                if (!fixed[i]) gnew += gq[i] * gq[i];
            if (gnew < 1e-24 * (1 + gg)) return;
            const double beta = gnew / gg;
            gg = gnew;
            for (int i = 0; i < n; ++i) d[i] = fixed[i] ? 0.0 : -gq[i] + beta * d[i];
        }
        if (!hit_bound) return;
    }
}

double norm2(const double *a, const double *b, int n)
{
    double s = 0;
    for (int i = 0; i < n; ++i) s += (a[i] - b[i]) * (a[i] - b[i]);
    return sqrt(s);
}

} /* namespace */

/* Maximises f over lb <= x <= ub starting from x (overwritten with the
 * maximiser).  f has NLopt's nlopt_func signature (MLE_alg fits).  Stops when
 * the trust-region resolution reaches rhoend, when an accepted step changes
 * the value by less than ftol_abs (> 0), or after maxeval evaluations
 * (<= 0: no limit).  The ftol test needs two accepted steps in a row below
 * the threshold, so one lucky tiny step on a flat stretch does not end the
 * search.  Returns the number of evaluations, or a negative
 * XG_ERR_* code; *fmax receives the best value found. */
extern "C" int exageostat_b200_bobyqa(int n, double *x, const double *lb, const double *ub, double rhobeg,
                                      double rhoend, double ftol_abs, int maxeval,
                                      double (*f)(unsigned, const double *, double *, void *), void *data,
                                      double *fmax)
{
    if (n <= 0 || n > 64 || !x || !lb || !ub || !f) return -XG_ERR_BAD_ARGUMENT;
    for (int i = 0; i < n; ++i)
        if (!(lb[i] < ub[i])) return -XG_ERR_BAD_ARGUMENT;
    double minrange = INFINITY;
    for (int i = 0; i < n; ++i) minrange = std::min(minrange, ub[i] - lb[i]);
    if (!(rhobeg > 0)) rhobeg = 0.25 * minrange;
    rhobeg = std::min(rhobeg, 0.5 * minrange);
    if (!(rhoend > 0) || rhoend > rhobeg) rhoend = 1e-6 * rhobeg;
    Problem P;
    P.n = n;
    P.f = f;
    P.data = data;
    P.lb = lb;
    P.ub = ub;
    P.maxeval = maxeval > 0 ? maxeval : 1 << 30;

    const int m = 2 * n + 1;
    Model M;
    M.n = n;
    M.m = m;
    M.xb.assign(x, x + n);
    for (int i = 0; i < n; ++i) M.xb[i] = std::min(ub[i], std::max(lb[i], M.xb[i]));
    M.Y.assign((size_t)m * n, 0.0);
    M.F.assign((size_t)m, 0.0);
    M.g.assign((size_t)n, 0.0);
    M.H.assign((size_t)n * n, 0.0);
    /* initial points: xb, then two points per axis, +-rhobeg, or +rhobeg and
     * +2 rhobeg (-rhobeg, -2 rhobeg) when xb sits on a lower (upper) bound */
    for (int a = 0; a < m; ++a)
        for (int i = 0; i < n; ++i) M.Y[a * n + i] = M.xb[i];
    std::vector<double> step1((size_t)n), step2((size_t)n);
    for (int i = 0; i < n; ++i) {
        double s1 = rhobeg, s2 = -rhobeg;
        if (M.xb[i] - rhobeg < lb[i]) {
            M.xb[i] = lb[i];
            s1 = rhobeg;
            s2 = 2 * rhobeg;
        } else if (M.xb[i] + rhobeg > ub[i]) {
            M.xb[i] = ub[i];
            s1 = -rhobeg;
            s2 = -2 * rhobeg;
        }
        step1[i] = s1;
        step2[i] = s2;
    }
    for (int a = 0; a < m; ++a)
        for (int i = 0; i < n; ++i) M.Y[a * n + i] = M.xb[i];
    for (int i = 0; i < n; ++i) {
        M.Y[(1 + i) * n + i] += step1[i];
        M.Y[(1 + n + i) * n + i] += step2[i];
    }
    for (int a = 0; a < m && P.evals < P.maxeval; ++a) M.F[a] = P.eval(&M.Y[a * n]);
    if (P.evals < m) {
        memcpy(x, P.best_x.data(), sizeof(double) * n);
        if (fmax) *fmax = -P.best_f;
        return P.evals;
    }
    /* separable quadratic through the three points of every axis */
    M.c = M.F[0];
    for (int i = 0; i < n; ++i) {
        const double a1 = step1[i], a2 = step2[i];
        const double f0 = M.F[0], f1 = M.F[1 + i], f2 = M.F[1 + n + i];
        /* q(t) = f0 + g t + h t^2 / 2 through (a1, f1), (a2, f2) */
        const double h = 2.0 * ((f1 - f0) / a1 - (f2 - f0) / a2) / (a1 - a2);
        M.g[i] = (f1 - f0) / a1 - 0.5 * h * a1;
        M.H[i * n + i] = h;
    }

    double rho = rhobeg, delta = rhobeg;
    int kopt = 0;
    for (int a = 1; a < m; ++a)
        if (M.F[a] < M.F[kopt]) kopt = a;
    std::vector<double> s, xnew((size_t)n), lag;
    bool stop_ftol = false;
    int small_steps = 0;
    while (P.evals < P.maxeval && !stop_ftol) {
        M.rebase(&M.Y[kopt * n]);
        const double *xo = &M.Y[kopt * n];
        trust_region_step(M, xo, lb, ub, delta, s);
        double snorm = 0;
        for (int i = 0; i < n; ++i) snorm += s[i] * s[i];
        snorm = sqrt(snorm);
        if (snorm < 0.5 * rho) {
            /* the model's step is too short to be worth a function value */
            delta = std::max(0.1 * delta, rho);
            if (delta <= 1.5 * rho) delta = rho;
        } else {
            for (int i = 0; i < n; ++i) xnew[i] = std::min(ub[i], std::max(lb[i], xo[i] + s[i]));
            const double qred = M.value(xo) - M.value(xnew.data());
            const double fnew = P.eval(xnew.data());
            const double fold = M.F[kopt];
            const double ratio = qred > 0 ? (fold - fnew) / qred : -1.0;
            if (ratio <= 0.1)
                delta = std::min(0.5 * delta, snorm);
            else if (ratio <= 0.7)
                delta = std::max(0.5 * delta, snorm);
            else
                delta = std::max(0.5 * delta, 2.0 * snorm);
            if (delta <= 1.5 * rho) delta = rho;
            /* point to replace: largest |Lagrange value| weighted by distance */
            int t = -1;
            if (M.lagrange(xnew.data(), lag)) {
                double best = -1;
                for (int a = 0; a < m; ++a) {
                    if (a == kopt) continue;
                    const double d = norm2(&M.Y[a * n], fnew < fold ? xnew.data() : xo, n);
                    const double w = std::max(1.0, (d / delta) * (d / delta));
                    const double sc = fabs(lag[a]) * w * w;
                    if (sc > best) {
                        best = sc;
                        t = a;
                    }
                }
            }
            if (t < 0) t = (kopt + 1) % m;
            memcpy(&M.Y[t * n], xnew.data(), sizeof(double) * n);
            M.F[t] = fnew;
            M.update();
            if (fnew < fold) {
                kopt = t;
                /* two accepted steps in a row that change f by < ftol_abs */
                small_steps = (ftol_abs > 0 && fold - fnew < ftol_abs) ? small_steps + 1 : 0;
                if (small_steps >= 2) stop_ftol = true;
            }
            if (ratio > 0.1) continue;
        }
        /* failure at this radius: improve the geometry if a point is far */
        int far = -1;
        double dmax = 0;
        for (int a = 0; a < m; ++a) {
            const double d = norm2(&M.Y[a * n], &M.Y[kopt * n], n);
            if (d > dmax) {
                dmax = d;
                far = a;
            }
        }
        if (far >= 0 && dmax > 2.0 * delta && P.evals < P.maxeval) {
            /* candidates on the box-clipped ball of radius max(rho, delta/10)
             * around x_opt: the coordinate directions and the direction to the
             * far point; keep the one where the far point's Lagrange function
             * is largest */
            const double rad = std::max(rho, 0.1 * delta);
            const double *xo2 = &M.Y[kopt * n];
            std::vector<double> cand((size_t)n), bestc((size_t)n);
            double bestv = -1;
            for (int dir = 0; dir <= 2 * n; ++dir) {
                for (int i = 0; i < n; ++i) cand[i] = xo2[i];
                if (dir < 2 * n) {
                    cand[dir / 2] += (dir & 1) ? -rad : rad;
                } else {
                    for (int i = 0; i < n; ++i) cand[i] += rad * (M.Y[far * n + i] - xo2[i]) / dmax;
                }
                for (int i = 0; i < n; ++i) cand[i] = std::min(ub[i], std::max(lb[i], cand[i]));
                if (norm2(cand.data(), xo2, n) < 1e-3 * rad) continue;
                if (!M.lagrange(cand.data(), lag)) continue;
                if (fabs(lag[far]) > bestv) {
                    bestv = fabs(lag[far]);
                    bestc = cand;
                }
            }
            if (bestv > 0) {
                const double fg = P.eval(bestc.data());
                memcpy(&M.Y[far * n], bestc.data(), sizeof(double) * n);
                M.F[far] = fg;
                M.update();
                if (fg < M.F[kopt]) kopt = far;
                continue;
            }
        }
        /* retry with the reduced radius before refining the resolution */
        if (std::max(delta, snorm) > rho) continue;
        if (rho <= rhoend) break;
        const double ratio = rho / rhoend;
        const double rho_old = rho;
        if (ratio <= 16.0)
            rho = rhoend;
        else if (ratio <= 250.0)
            rho = sqrt(ratio) * rhoend;
        else
            rho *= 0.1;
        delta = std::max(0.5 * rho_old, rho);
    }
    memcpy(x, P.best_x.data(), sizeof(double) * n);
    if (fmax) *fmax = -P.best_f;
    return P.evals;
}
