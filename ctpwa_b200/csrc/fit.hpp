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

}  // namespace ctpwa
