// Box-constrained limited-memory BFGS on the host, for fit jobs that run one
// likelihood evaluation per function call on the device.
#pragma once

#include <functional>

namespace ctpwa {

struct BoxLbfgsOptions {
    int max_evals = 100;  // function evaluations, line-search trials included
    int m = 20;           // correction pairs kept
    double ftol = 1e-13;  // stop when (f_k - f_{k+1}) <= ftol * max(|f_k|, |f_{k+1}|, 1)
    double gtol = 1e-9;   // stop when max |P(x - g) - x| <= gtol over the free variables
};

// status: 0 projected gradient below gtol, 1 relative decrease below ftol,
// 2 evaluation budget spent, 3 no decrease found along the search direction
struct BoxLbfgsResult {
    double f = 0.0;
    int evals = 0;
    int iters = 0;
    int status = 0;
};

// f(x) and its gradient; a nonzero return aborts the minimisation with that
// code (a non-finite f is a failed trial point, not an error)
using FgFn = std::function<int(const double* x, double* f, double* g)>;

// Minimises over the variables with free[i] != 0 (the others stay at x[i])
// within lo[i] <= x[i] <= hi[i] (+-infinity for none). x is projected onto the
// box first and holds the best point found on return. Returns 0 or the first
// nonzero code of fg.
int boxLbfgs(const FgFn& fg, int n, double* x, const unsigned char* free, const double* lo, const double* hi,
             const BoxLbfgsOptions& opt, BoxLbfgsResult* res);

struct NewtonOptions {
    int max_iter = 50;     // Hessian evaluations
    double xtol = 1e-4;    // stop after a step with max_i |s_i| sqrt(H_ii) <= xtol (free variables),
                           // or one whose predicted decrease is <= 1e-2 fnoise
    double gtol = 1e-9;    // stop when max |P(x - g) - x| <= gtol over the free variables
    double fnoise = 0.0;   // steps whose predicted decrease is at most this are accepted when f
                           // rises by at most this (the rounding level of f)
};

// the Hessian at x, row-major n x n; a nonzero return aborts with that code
using HessFn = std::function<int(const double* x, double* H)>;

// Levenberg-Marquardt Newton iteration with the exact Hessian over the same
// box and free variables as boxLbfgs: steps solve (H + lambda diag|H|) s =
// -g over the variables not held at a bound, are projected onto the box and
// kept when f falls by at least 1e-4 of the quadratic model's prediction;
// lambda shrinks after good steps (to 0: Newton steps) and grows after
// rejected ones or an indefinite matrix. It converges to the stationary point
// of the start's basin, where the Hessian is positive definite. Result:
// evals counts f evaluations, iters Hessian evaluations; status 0 projected
// gradient <= gtol, 1 step <= xtol (or predicted decrease <= 1e-2 fnoise),
// 2 max_iter Hessians spent, 3 no acceptable step found.
int boxNewton(const FgFn& fg, const HessFn& hf, int n, double* x, const unsigned char* free, const double* lo,
              const double* hi, const NewtonOptions& opt, BoxLbfgsResult* res);

}  // namespace ctpwa
