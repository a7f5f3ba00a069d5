// Projected limited-memory BFGS for fit jobs (the host side of a fit: one
// device likelihood evaluation per function call).
//
// The reference fits with torch.optim.LBFGS over parameters that it clamps
// into their bounds before every evaluation, with the gradient components that
// point out of an active bound set to zero (example/fit.py:113-200). Here the
// same scheme is one routine: the search direction comes from the two-loop
// recursion of limited-memory BFGS (Nocedal, Math. Comp. 35 (1980) 773) over
// the variables not held at a bound, the line search backtracks along the
// projection of the step onto the box (projected Armijo rule, Bertsekas,
// SIAM J. Control Optim. 20 (1982) 221), with a quadratic-interpolation step
// cut, and correction pairs with s.y <= 0 are skipped.
#include "fit.hpp"

#include <algorithm>
#include <cmath>
#include <deque>
#include <vector>

namespace ctpwa {

int boxLbfgs(const FgFn& fg, int n, double* x, const unsigned char* fr, const double* lo, const double* hi,
             const BoxLbfgsOptions& opt, BoxLbfgsResult* res)
{
    BoxLbfgsResult r;
    auto box = [&](int i, double v) { return std::min(std::max(v, lo[i]), hi[i]); };
    for (int i = 0; i < n; ++i)
        if (fr[i]) x[i] = box(i, x[i]);
    std::vector<double> g(n), xn(n), gn(n), d(n), q(n);
    std::vector<char> act(n);
    struct Pair {
        std::vector<double> s, y;
    };
    std::deque<Pair> mem;
    double f = 0.0;
    if (int rc = fg(x, &f, g.data())) return rc;
    r.evals = 1;
    if (!std::isfinite(f)) {
        r.f = f;
        r.status = 3;
        *res = r;
        return 0;
    }
    // products over the free variables not held at a bound
    auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) {
        double s = 0.0;
        for (int i = 0; i < n; ++i)
            if (!act[i]) s += a[i] * b[i];
        return s;
    };
    bool steepest = true;  // no curvature information yet: scaled gradient step
    for (;;) {
        // projected-gradient test; a variable is held when it sits on a bound
        // and its gradient points out of the box
        double pg = 0.0;
        for (int i = 0; i < n; ++i) {
            act[i] = !fr[i] || (x[i] <= lo[i] && g[i] > 0.0) || (x[i] >= hi[i] && g[i] < 0.0);
            if (fr[i]) pg = std::max(pg, std::fabs(box(i, x[i] - g[i]) - x[i]));
        }
        if (pg <= opt.gtol) {
            r.status = 0;
            break;
        }
        if (r.evals >= opt.max_evals) {
            r.status = 2;
            break;
        }
        // d = -H g by the two-loop recursion (pairs whose restricted s.y is
        // not positive are left out)
        for (int i = 0; i < n; ++i) q[i] = act[i] ? 0.0 : g[i];
        const int k = (int)mem.size();
        std::vector<double> al(k, 0.0), rho(k, 0.0);
        double gamma = 1.0;
        bool scaled = false;
        for (int j = k - 1; j >= 0; --j) {
            const double sy = dot(mem[j].s, mem[j].y);
            if (!(sy > 0.0)) continue;
            rho[j] = 1.0 / sy;
            if (!scaled) {
                const double yy = dot(mem[j].y, mem[j].y);
                if (yy > 0.0) gamma = sy / yy;
                scaled = true;
            }
            al[j] = rho[j] * dot(mem[j].s, q);
            for (int i = 0; i < n; ++i)
                if (!act[i]) q[i] -= al[j] * mem[j].y[i];
        }
        for (int i = 0; i < n; ++i) q[i] *= gamma;
        for (int j = 0; j < k; ++j) {
            if (rho[j] == 0.0) continue;
            const double b = rho[j] * dot(mem[j].y, q);
            for (int i = 0; i < n; ++i)
                if (!act[i]) q[i] += (al[j] - b) * mem[j].s[i];
        }
        double gd = 0.0;
        for (int i = 0; i < n; ++i) {
            d[i] = act[i] ? 0.0 : -q[i];
            gd += g[i] * d[i];
        }
        if (!(gd < 0.0) || !std::isfinite(gd)) {
            mem.clear();
            steepest = true;
            gd = 0.0;
            for (int i = 0; i < n; ++i) {
                d[i] = act[i] ? 0.0 : -g[i];
                gd += g[i] * d[i];
            }
        }
        // first trial: the full step, or after a reset a step of unit
        // 1-norm in the gradient (as torch.optim.LBFGS starts)
        double alpha = 1.0;
        if (steepest) {
            double g1 = 0.0;
            for (int i = 0; i < n; ++i)
                if (!act[i]) g1 += std::fabs(g[i]);
            alpha = std::min(1.0, 1.0 / std::max(g1, 1e-300));
        }
        bool ok = false;
        double fn = f;
        for (int t = 0; t < 30 && r.evals < opt.max_evals; ++t) {
            bool moved = false;
            for (int i = 0; i < n; ++i) {
                xn[i] = act[i] ? x[i] : box(i, x[i] + alpha * d[i]);
                moved = moved || xn[i] != x[i];
            }
            if (!moved) break;
            if (int rc = fg(xn.data(), &fn, gn.data())) return rc;
            ++r.evals;
            double dphi = 0.0;  // first-order change along the projected step
            for (int i = 0; i < n; ++i) dphi += g[i] * (xn[i] - x[i]);
            if (std::isfinite(fn) && fn <= f + 1e-4 * std::min(dphi, 0.0)) {
                ok = true;
                break;
            }
            // minimum of the quadratic through f, the slope dphi / alpha and
            // fn, kept within [0.1, 0.5] of the current step
            double an = 0.1 * alpha;
            if (std::isfinite(fn)) {
                const double den = 2.0 * (fn - f - dphi);
                if (den > 0.0 && dphi < 0.0) an = -dphi * alpha / den;
            }
            alpha = std::min(0.5 * alpha, std::max(0.1 * alpha, an));
        }
        if (!ok) {
            if (!steepest) {  // retry from the gradient alone
                mem.clear();
                steepest = true;
                continue;
            }
            r.status = r.evals >= opt.max_evals ? 2 : 3;
            break;
        }
        Pair p{std::vector<double>(n), std::vector<double>(n)};
        double sy = 0.0, ss = 0.0, yy = 0.0;
        for (int i = 0; i < n; ++i) {
            p.s[i] = xn[i] - x[i];
            p.y[i] = gn[i] - g[i];
            if (!fr[i]) continue;
            sy += p.s[i] * p.y[i];
            ss += p.s[i] * p.s[i];
            yy += p.y[i] * p.y[i];
        }
        if (sy > 1e-10 * std::sqrt(ss * yy)) {
            mem.push_back(std::move(p));
            if ((int)mem.size() > std::max(1, opt.m)) mem.pop_front();
            steepest = false;
        }
        const double fold = f;
        std::copy(xn.begin(), xn.end(), x);
        g.swap(gn);
        f = fn;
        ++r.iters;
        if (fold - f <= opt.ftol * std::max({std::fabs(fold), std::fabs(f), 1.0})) {
            r.status = 1;
            break;
        }
    }
    r.f = f;
    *res = r;
    return 0;
}

namespace {

// Cholesky factor of the m x m row-major SPD matrix A in place (lower
// triangle); false when a pivot is not positive
bool cholesky(std::vector<double>& A, int m)
{
    for (int j = 0; j < m; ++j) {
        double d = A[j * m + j];
        for (int k = 0; k < j; ++k) d -= A[j * m + k] * A[j * m + k];
        if (!(d > 0.0) || !std::isfinite(d)) return false;
        d = std::sqrt(d);
        A[j * m + j] = d;
        for (int i = j + 1; i < m; ++i) {
            double v = A[i * m + j];
            for (int k = 0; k < j; ++k) v -= A[i * m + k] * A[j * m + k];
            A[i * m + j] = v / d;
        }
    }
    return true;
}

// solves L L^T y = b in place
void cholSolve(const std::vector<double>& L, int m, std::vector<double>& b)
{
    for (int i = 0; i < m; ++i) {
        double v = b[i];
        for (int k = 0; k < i; ++k) v -= L[i * m + k] * b[k];
        b[i] = v / L[i * m + i];
    }
    for (int i = m - 1; i >= 0; --i) {
        double v = b[i];
        for (int k = i + 1; k < m; ++k) v -= L[k * m + i] * b[k];
        b[i] = v / L[i * m + i];
    }
}

}  // namespace

int boxNewton(const FgFn& fg, const HessFn& hf, int n, double* x, const unsigned char* fr, const double* lo,
              const double* hi, const NewtonOptions& opt, BoxLbfgsResult* res)
{
    BoxLbfgsResult r;
    auto box = [&](int i, double v) { return std::min(std::max(v, lo[i]), hi[i]); };
    for (int i = 0; i < n; ++i)
        if (fr[i]) x[i] = box(i, x[i]);
    std::vector<double> g(n), gn(n), xn(n), H((size_t)n * n), s(n);
    double f = 0.0;
    if (int rc = fg(x, &f, g.data())) return rc;
    r.evals = 1;
    if (!std::isfinite(f)) {
        r.f = f;
        r.status = 3;
        *res = r;
        return 0;
    }
    if (int rc = hf(x, H.data())) return rc;
    r.iters = 1;
    double lambda = 0.0;
    for (;;) {
        // variables held at a bound (gradient pointing out of the box)
        std::vector<int> idx;
        double pg = 0.0;
        for (int i = 0; i < n; ++i) {
            if (!fr[i]) continue;
            pg = std::max(pg, std::fabs(box(i, x[i] - g[i]) - x[i]));
            if (!((x[i] <= lo[i] && g[i] > 0.0) || (x[i] >= hi[i] && g[i] < 0.0))) idx.push_back(i);
        }
        if (pg <= opt.gtol || idx.empty()) {
            r.status = 0;
            break;
        }
        const int m = (int)idx.size();
        double dmax = 0.0;
        for (int i : idx) dmax = std::max(dmax, std::fabs(H[(size_t)i * n + i]));
        std::vector<double> D(m);
        for (int a = 0; a < m; ++a) D[a] = std::max(std::fabs(H[(size_t)idx[a] * n + idx[a]]), 1e-12 * dmax + 1e-300);
        bool accepted = false, converged = false;
        for (int trial = 0; trial < 60; ++trial) {
            std::vector<double> A((size_t)m * m), b(m);
            for (int a = 0; a < m; ++a) {
                for (int c = 0; c < m; ++c) A[(size_t)a * m + c] = H[(size_t)idx[a] * n + idx[c]];
                A[(size_t)a * m + a] += lambda * D[a];
                b[a] = -g[idx[a]];
            }
            if (!cholesky(A, m)) {
                lambda = lambda == 0.0 ? 1e-6 : lambda * 10.0;
                if (lambda > 1e12) break;
                continue;
            }
            cholSolve(A, m, b);
            std::fill(s.begin(), s.end(), 0.0);
            for (int i = 0; i < n; ++i) xn[i] = x[i];
            for (int a = 0; a < m; ++a) {
                const int i = idx[a];
                xn[i] = box(i, x[i] + b[a]);
                s[i] = xn[i] - x[i];
            }
            // decrease predicted by the quadratic model along the projected step
            double gs = 0.0, sHs = 0.0;
            for (int a = 0; a < m; ++a) {
                const int i = idx[a];
                gs += g[i] * s[i];
                double hs = 0.0;
                for (int c = 0; c < m; ++c) hs += H[(size_t)i * n + idx[c]] * s[idx[c]];
                sHs += s[i] * hs;
            }
            const double pred = -(gs + 0.5 * sHs);
            double step = 0.0;
            for (int a = 0; a < m; ++a) step = std::max(step, std::fabs(s[idx[a]]) * std::sqrt(D[a]));
            if (step == 0.0) {
                converged = true;
                break;
            }
            if (!(pred > 0.0)) {
                lambda = std::max(lambda * 4.0, 1e-4);
                if (lambda > 1e12) break;
                continue;
            }
            double fn = 0.0;
            if (int rc = fg(xn.data(), &fn, gn.data())) return rc;
            ++r.evals;
            const bool noise = pred <= opt.fnoise && fn <= f + opt.fnoise;
            if (std::isfinite(fn) && (f - fn >= 1e-4 * pred || noise)) {
                const double rho = (f - fn) / pred;
                std::copy(xn.begin(), xn.end(), x);
                g.swap(gn);
                f = fn;
                if (rho > 0.75 || noise) lambda *= 0.25;
                else if (rho < 0.25) lambda = std::max(lambda * 2.0, 1e-6);
                if (lambda < 1e-10) lambda = 0.0;
                accepted = true;
                // a step within xtol, or one whose predicted decrease is below
                // a hundredth of f's rounding level: what is left to gain is
                // rounding (its H-norm sqrt(2 pred) bounds every parameter's
                // move in units of its error)
                converged = step <= opt.xtol || (opt.fnoise > 0.0 && pred <= 1e-2 * opt.fnoise);
                break;
            }
            lambda = std::max(lambda * 4.0, 1e-4);
            if (lambda > 1e12) break;
        }
        if (converged) {
            r.status = 1;
            break;
        }
        if (!accepted) {
            r.status = 3;
            break;
        }
        if (r.iters >= opt.max_iter) {
            r.status = 2;
            break;
        }
        if (int rc = hf(x, H.data())) return rc;
        ++r.iters;
    }
    r.f = f;
    *res = r;
    return 0;
}

}  // namespace ctpwa
