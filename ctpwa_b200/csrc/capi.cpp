// C ABI (include/ctpwa_b200.h) over the C++ engine: status codes instead of
// exceptions, host-buffer convenience entry point, model introspection.
#include "../../include/ctpwa_b200.h"

#include "engine.hpp"
#include "fit.hpp"

#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>
#include <stdexcept>
#include <string>

struct ctpwa_handle {
    std::unique_ptr<ctpwa::Engine> eng;
    std::string err;
    double* d_params = nullptr;  // host-entry staging
    double* d_out = nullptr;     // [1 + n_params]
    double* h_pin = nullptr;     // pinned [1 + 2 n_params]
    double* d_hess = nullptr;    // [n_params^2], allocated by the first Newton fit
};

namespace {
std::mutex g_err_mu;
std::string g_create_err;

int setErr(ctpwa_handle* h, int code, const std::string& m)
{
    if (h) h->err = m;
    else {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_create_err = m;
    }
    return code;
}

// A fit none of whose resonance parameters can move (free[i] == 0 or
// lo[i] == hi[i] for each): its evaluations can all use one normalisation cache.
bool thetaFixed(const ctpwa_handle* h, const unsigned char* free_mask, const double* lo, const double* hi)
{
    const int np = h->eng->nParams(), off = 2 * h->eng->model().nVector();
    for (int i = off; i < np; ++i)
        if (free_mask[i] && lo[i] != hi[i]) return false;
    return true;
}

// the normalisation cache at the resonance parameters of the host array x
// (built unless it already matches them)
void ensureNormCache(ctpwa_handle* h, const double* x, void* stream)
{
    if (h->eng->normCacheMatches(x)) return;
    const int np = h->eng->nParams();
    cudaStream_t s = (cudaStream_t)stream;
    std::memcpy(h->h_pin, x, sizeof(double) * np);
    if (cudaMemcpyAsync(h->d_params, h->h_pin, sizeof(double) * np, cudaMemcpyHostToDevice, s) != cudaSuccess)
        throw std::runtime_error("CUDA error: host-to-device copy failed");
    h->eng->normCacheBuild(h->d_params, s);
}

int copyOut(const std::string& s, char* buf, size_t cap)
{
    if (buf && cap > 0) {
        size_t n = std::min(cap - 1, s.size());
        std::memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return (int)s.size() + 1;
}
}  // namespace

extern "C" {

ctpwa_handle* ctpwa_create(const char* config_path, int device, int* status, char* err, size_t errlen)
{
    return ctpwa_create_shard(config_path, device, 0, 1, status, err, errlen);
}

namespace {
ctpwa_handle* createWith(const char* config_path, const ctpwa::EngineOptions& opt, int* status, char* err,
                         size_t errlen)
{
    auto h = std::make_unique<ctpwa_handle>();
    int code = CTPWA_OK;
    std::string msg;
    try {
        h->eng = std::make_unique<ctpwa::Engine>(config_path ? config_path : "config.yml", opt);
        int np = h->eng->nParams();
        if (cudaMalloc(&h->d_params, sizeof(double) * std::max(1, np)) != cudaSuccess ||
            cudaMalloc(&h->d_out, sizeof(double) * (1 + np)) != cudaSuccess ||
            cudaMallocHost(&h->h_pin, sizeof(double) * (1 + 2 * np)) != cudaSuccess)
            throw std::runtime_error("CUDA allocation of evaluation buffers failed");
    } catch (const std::exception& e) {
        msg = e.what();
        code = (msg.rfind("CUDA", 0) == 0 || msg.find("NVRTC") != std::string::npos) ? CTPWA_ERR_CUDA : CTPWA_ERR_CONFIG;
    }
    if (status) *status = code;
    if (code != CTPWA_OK) {
        setErr(nullptr, code, msg);
        if (err && errlen) copyOut(msg, err, errlen);
        return nullptr;
    }
    return h.release();
}
}  // namespace

ctpwa_handle* ctpwa_create_shard(const char* config_path, int device, int rank, int world, int* status, char* err,
                                 size_t errlen)
{
    if (world < 1 || rank < 0 || rank >= world) {
        const std::string msg = "shard: need 0 <= rank < world";
        if (status) *status = CTPWA_ERR_ARG;
        setErr(nullptr, CTPWA_ERR_ARG, msg);
        if (err && errlen) copyOut(msg, err, errlen);
        return nullptr;
    }
    ctpwa::EngineOptions opt;
    opt.device = device;
    opt.shard_rank = rank;
    opt.shard_world = world;
    return createWith(config_path, opt, status, err, errlen);
}

ctpwa_handle* ctpwa_create_from_device(const char* config_path, int device, const double* const* p4,
                                       const long long* n, const double* const* w, int* status, char* err,
                                       size_t errlen)
{
    return ctpwa_create_from_device_flags(config_path, device, p4, n, w, 0, status, err, errlen);
}

ctpwa_handle* ctpwa_create_from_device_flags(const char* config_path, int device, const double* const* p4,
                                             const long long* n, const double* const* w, int flags, int* status,
                                             char* err, size_t errlen)
{
    if (!p4 || !n || (flags & ~CTPWA_CREATE_FP64_ONLY)) {
        const std::string msg = (!p4 || !n) ? "null argument" : "unknown creation flags";
        if (status) *status = CTPWA_ERR_ARG;
        setErr(nullptr, CTPWA_ERR_ARG, msg);
        if (err && errlen) copyOut(msg, err, errlen);
        return nullptr;
    }
    ctpwa::EngineOptions opt;
    opt.device = device;
    opt.device_samples = true;
    if (flags & CTPWA_CREATE_FP64_ONLY) {
        opt.mixed_tables = false;
        opt.pair_polarisations = false;
    }
    for (int k = 0; k < 3; ++k) {
        opt.dev_p4[k] = p4[k];
        opt.dev_n[k] = n[k];
        opt.dev_w[k] = w ? w[k] : nullptr;
    }
    return createWith(config_path, opt, status, err, errlen);
}

void ctpwa_destroy(ctpwa_handle* h)
{
    if (!h) return;
    cudaFree(h->d_params);
    cudaFree(h->d_out);
    cudaFree(h->d_hess);
    cudaFreeHost(h->h_pin);
    delete h;
}

int ctpwa_n_vector(const ctpwa_handle* h) { return h ? h->eng->model().nVector() : CTPWA_ERR_ARG; }
int ctpwa_n_free_theta(const ctpwa_handle* h) { return h ? h->eng->model().nTheta() : CTPWA_ERR_ARG; }
int ctpwa_n_params(const ctpwa_handle* h) { return h ? h->eng->nParams() : CTPWA_ERR_ARG; }

int ctpwa_param_names(const ctpwa_handle* h, char* buf, size_t cap)
{
    if (!h) return CTPWA_ERR_ARG;
    std::string s;
    for (const auto& n : h->eng->model().param_names) {
        if (!s.empty()) s += "\n";
        s += n;
    }
    return copyOut(s, buf, cap);
}

int ctpwa_free_res_params(const ctpwa_handle* h, double* out)
{
    if (!h || !out) return CTPWA_ERR_ARG;
    const auto& sl = h->eng->model().slots;
    int n = (int)sl.size();
    for (int i = 0; i < n; ++i) {
        out[i] = sl[i].init;
        out[n + i] = sl[i].lower;
        out[2 * n + i] = sl[i].upper;
    }
    return CTPWA_OK;
}

int ctpwa_nll_grad(ctpwa_handle* h, const double* d_params, double* d_nll, double* d_grad, int precision, void* stream)
{
    if (!h || !d_params || !d_nll || !d_grad) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (precision != CTPWA_FP64 && precision != CTPWA_MIXED) return setErr(h, CTPWA_ERR_ARG, "precision must be 0 or 1");
    try {
        h->eng->nllGrad(d_params, d_nll, d_grad, precision, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_nll_grad_static(ctpwa_handle* h, const double* d_params, double* d_nll, double* d_grad, int precision,
                          void* stream)
{
    if (!h || !d_params || !d_nll || !d_grad) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (precision != CTPWA_FP64 && precision != CTPWA_MIXED) return setErr(h, CTPWA_ERR_ARG, "precision must be 0 or 1");
    try {
        h->eng->nllGradStatic(d_params, d_nll, d_grad, precision, (cudaStream_t)stream);
    } catch (const std::length_error& e) {
        return setErr(h, CTPWA_ERR_ARG, e.what());
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_hessian(ctpwa_handle* h, const double* d_params, double* d_hess, double rel_step, void* stream)
{
    if (!h || !d_params || !d_hess) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (!(rel_step > 0.0) || rel_step > 1e-2) return setErr(h, CTPWA_ERR_ARG, "rel_step must be in (0, 1e-2]");
    try {
        h->eng->hessian(d_params, d_hess, rel_step, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_hessian_exact(ctpwa_handle* h, const double* d_params, double* d_hess, void* stream)
{
    if (!h || !d_params || !d_hess) return setErr(h, CTPWA_ERR_ARG, "null argument");
    try {
        h->eng->hessianExact(d_params, d_hess, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_hessian_gram(ctpwa_handle* h, const double* d_params, double* d_hess, void* stream)
{
    if (!h || !d_params || !d_hess) return setErr(h, CTPWA_ERR_ARG, "null argument");
    try {
        h->eng->hessianGram(d_params, d_hess, (cudaStream_t)stream);
    } catch (const std::length_error& e) {
        return setErr(h, CTPWA_ERR_ARG, e.what());
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_gram_shape(ctpwa_handle* h, int* out4)
{
    if (!h || !out4) return setErr(h, CTPWA_ERR_ARG, "null argument");
    try {
        h->eng->gramShape(out4);
    } catch (const std::length_error& e) {
        return setErr(h, CTPWA_ERR_ARG, e.what());
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_gram(ctpwa_handle* h, const double* d_params, double* d_out, void* stream)
{
    if (!h || !d_params || !d_out) return setErr(h, CTPWA_ERR_ARG, "null argument");
    try {
        h->eng->gram(d_params, d_out, (cudaStream_t)stream);
    } catch (const std::length_error& e) {
        return setErr(h, CTPWA_ERR_ARG, e.what());
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_norm_cache_build(ctpwa_handle* h, const double* d_params, double* ms, void* stream)
{
    if (!h || !d_params) return setErr(h, CTPWA_ERR_ARG, "null argument");
    try {
        const double t = h->eng->normCacheBuild(d_params, (cudaStream_t)stream);
        if (ms) *ms = t;
    } catch (const std::length_error& e) {
        return setErr(h, CTPWA_ERR_ARG, e.what());
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_norm_cache_clear(ctpwa_handle* h)
{
    if (!h) return setErr(h, CTPWA_ERR_ARG, "null argument");
    h->eng->normCacheClear();
    return CTPWA_OK;
}

int ctpwa_norm_cache_valid(const ctpwa_handle* h)
{
    return h && h->eng->normCacheValid() ? 1 : 0;
}

int ctpwa_nll_grad_cached(ctpwa_handle* h, const double* d_params, double* d_nll, double* d_grad, int precision,
                          void* stream)
{
    if (!h || !d_params || !d_nll || !d_grad) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (precision != CTPWA_FP64 && precision != CTPWA_MIXED) return setErr(h, CTPWA_ERR_ARG, "precision must be 0 or 1");
    if (!h->eng->normCacheValid()) return setErr(h, CTPWA_ERR_ARG, "no normalisation cache: build it first");
    try {
        h->eng->nllGradCached(d_params, d_nll, d_grad, precision, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_hvp(ctpwa_handle* h, const double* d_params, const double* d_dirs, int ndir, double* d_out, void* stream)
{
    if (!h || !d_params || !d_dirs || !d_out) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (ndir < 0) return setErr(h, CTPWA_ERR_ARG, "ndir must be >= 0");
    try {
        h->eng->hessianVectorProducts(d_params, d_dirs, ndir, d_out, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_hvp_sums_size(const ctpwa_handle* h, int ndir)
{
    if (!h || ndir < 0) return CTPWA_ERR_ARG;
    return h->eng->hvpSumsSize(ndir);
}

int ctpwa_shard_hvp_sums(ctpwa_handle* h, const double* d_params, const double* d_dirs, int ndir, double* d_tsums,
                         void* stream)
{
    if (!h || !d_params || !d_dirs || !d_tsums) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (ndir < 0) return setErr(h, CTPWA_ERR_ARG, "ndir must be >= 0");
    try {
        h->eng->hvpSums(d_params, d_dirs, ndir, d_tsums, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_finalize_hvp(ctpwa_handle* h, const double* d_params, const double* d_dirs, int ndir, const double* d_vsums,
                       const double* d_tsums, double* d_out, void* stream)
{
    if (!h || !d_params || !d_dirs || !d_vsums || !d_tsums || !d_out) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (ndir < 0) return setErr(h, CTPWA_ERR_ARG, "ndir must be >= 0");
    try {
        h->eng->finalizeHvp(d_params, d_dirs, ndir, d_vsums, d_tsums, d_out, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_n_blocks(const ctpwa_handle* h) { return h ? h->eng->nBlocks() : CTPWA_ERR_ARG; }

int ctpwa_partial_integrals(ctpwa_handle* h, const double* d_params, int kind, double* d_out, void* stream)
{
    if (!h || !d_params || !d_out) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (kind < 0 || kind > 3) return setErr(h, CTPWA_ERR_ARG, "sample kind must be 0 (phsp), 1, 2 or 3 (phsp_truth)");
    try {
        h->eng->partialIntegrals(d_params, kind, d_out, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        std::string m = e.what();
        return setErr(h, m.rfind("No phsp_truth", 0) == 0 ? CTPWA_ERR_CONFIG : CTPWA_ERR_CUDA, m);
    }
    return CTPWA_OK;
}

long long ctpwa_table_stride(const ctpwa_handle* h, int kind)
{
    if (!h || kind < 0 || kind > 2) return CTPWA_ERR_ARG;
    return h->eng->tableStride(kind);
}

int ctpwa_export_weights(ctpwa_handle* h, const double* d_params, const int* wave_mask, double* d_total,
                         double* d_partial, double* d_interf_ev, double* d_interf, void* stream)
{
    if (!h || !d_params || !d_total || !d_partial || !d_interf) return setErr(h, CTPWA_ERR_ARG, "null argument");
    try {
        std::vector<int> mask;
        if (wave_mask) mask.assign(wave_mask, wave_mask + h->eng->nBlocks());
        h->eng->exportWeights(d_params, mask, d_total, d_partial, d_interf_ev, d_interf, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_sums_size(const ctpwa_handle* h) { return h ? h->eng->sumsSize() : CTPWA_ERR_ARG; }

int ctpwa_shard_sums(ctpwa_handle* h, const double* d_params, int precision, double* d_sums, void* stream)
{
    if (!h || !d_params || !d_sums) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (precision != CTPWA_FP64 && precision != CTPWA_MIXED) return setErr(h, CTPWA_ERR_ARG, "precision must be 0 or 1");
    try {
        h->eng->shardSums(d_params, precision, d_sums, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_finalize_sums(ctpwa_handle* h, const double* d_params, const double* d_sums, double* d_nll, double* d_grad,
                        void* stream)
{
    if (!h || !d_params || !d_sums || !d_nll || !d_grad) return setErr(h, CTPWA_ERR_ARG, "null argument");
    try {
        h->eng->finalizeSums(d_params, d_sums, d_nll, d_grad, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_nll_grad_host(ctpwa_handle* h, const double* params, double* nll, double* grad, int precision, void* stream)
{
    if (!h || !params || !nll || !grad) return setErr(h, CTPWA_ERR_ARG, "null argument");
    int np = h->eng->nParams();
    cudaStream_t s = (cudaStream_t)stream;
    try {
        std::memcpy(h->h_pin, params, sizeof(double) * np);
        if (cudaMemcpyAsync(h->d_params, h->h_pin, sizeof(double) * np, cudaMemcpyHostToDevice, s) != cudaSuccess)
            throw std::runtime_error("CUDA error: host-to-device copy failed");
        // points at the cached resonance parameters: from the normalisation cache
        int rc = h->eng->normCacheMatches(params) ? ctpwa_nll_grad_cached(h, h->d_params, h->d_out, h->d_out + 1, precision, stream)
                                                  : ctpwa_nll_grad(h, h->d_params, h->d_out, h->d_out + 1, precision, stream);
        if (rc != CTPWA_OK) return rc;
        if (cudaMemcpyAsync(h->h_pin + np, h->d_out, sizeof(double) * (1 + np), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError()));
        *nll = h->h_pin[np];
        std::memcpy(grad, h->h_pin + np + 1, sizeof(double) * np);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Evaluation batches: several handles of one model evaluated in one launch.
// A batch also gathers blocking host-buffer evaluations from the fit threads
// of a serving loop: each request waits until every fit that has joined the
// batch has a request pending (or a short window has passed), and one of
// the waiting threads then runs all pending requests, one multi-job launch
// per model and precision, on the batch's stream.
// ---------------------------------------------------------------------------
struct ctpwa_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    ctpwa::MultiScratch scratch;
    std::string err;
    // request gathering
    struct Request {
        ctpwa_handle* h;
        const double* params;
        double* nll;
        double* grad;
        int precision;
        int rc = CTPWA_OK;
        bool done = false;
    };
    std::mutex mu;
    std::condition_variable cv;
    int members = 0;
    bool running = false;
    std::vector<Request*> pending;
    int window_us = 200;
    long long rounds = 0, requests = 0;
};

namespace {

int batchErr(ctpwa_batch* b, int code, const std::string& m)
{
    if (b) b->err = m;
    return setErr(nullptr, code, m);
}

// Runs requests (handles' host staging buffers, one multi-job launch per
// model and precision); called by the leading thread with the lock released.
void runRound(ctpwa_batch* b, std::vector<ctpwa_batch::Request*>& reqs)
{
    std::map<std::pair<const void*, int>, std::vector<ctpwa_batch::Request*>> groups;
    for (auto* r : reqs) groups[{r->h->eng->kernelImageKey(), r->precision}].push_back(r);
    for (auto& g : groups) {
        auto& rs = g.second;
        try {
            std::vector<ctpwa::Engine*> es;
            std::vector<const double*> dp;
            std::vector<double*> dn, dg;
            for (auto* r : rs) {
                const int np = r->h->eng->nParams();
                std::memcpy(r->h->h_pin, r->params, sizeof(double) * np);
                if (cudaMemcpyAsync(r->h->d_params, r->h->h_pin, sizeof(double) * np, cudaMemcpyHostToDevice,
                                    b->stream) != cudaSuccess)
                    throw std::runtime_error("CUDA error: host-to-device copy failed");
                es.push_back(r->h->eng.get());
                dp.push_back(r->h->d_params);
                dn.push_back(r->h->d_out);
                dg.push_back(r->h->d_out + 1);
            }
            ctpwa::Engine::nllGradMulti(es, dp, dn, dg, g.first.second, b->scratch, b->stream);
            for (auto* r : rs) {
                const int np = r->h->eng->nParams();
                if (cudaMemcpyAsync(r->h->h_pin + np, r->h->d_out, sizeof(double) * (1 + np), cudaMemcpyDeviceToHost,
                                    b->stream) != cudaSuccess)
                    throw std::runtime_error("CUDA error: device-to-host copy failed");
            }
            if (cudaStreamSynchronize(b->stream) != cudaSuccess)
                throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError()));
            for (auto* r : rs) {
                const int np = r->h->eng->nParams();
                *r->nll = r->h->h_pin[np];
                std::memcpy(r->grad, r->h->h_pin + np + 1, sizeof(double) * np);
            }
        } catch (const std::exception& e) {
            for (auto* r : rs) r->rc = setErr(r->h, CTPWA_ERR_CUDA, e.what());
        }
    }
}

}  // namespace

extern "C" {

ctpwa_batch* ctpwa_batch_create(int device)
{
    auto b = std::make_unique<ctpwa_batch>();
    b->device = device;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        batchErr(nullptr, CTPWA_ERR_CUDA, "batch: stream creation failed");
        cudaSetDevice(prev);
        return nullptr;
    }
    cudaSetDevice(prev);
    return b.release();
}

void ctpwa_batch_destroy(ctpwa_batch* b)
{
    if (!b) return;
    if (b->stream) {
        cudaStreamSynchronize(b->stream);
        cudaStreamDestroy(b->stream);
    }
    delete b;
}

int ctpwa_nll_grad_multi(ctpwa_batch* b, ctpwa_handle* const* hs, int n, const double* const* d_params,
                         double* const* d_nll, double* const* d_grad, int precision, void* stream)
{
    if (!b || !hs || !d_params || !d_nll || !d_grad || n < 0) return batchErr(b, CTPWA_ERR_ARG, "null argument");
    if (precision != CTPWA_FP64 && precision != CTPWA_MIXED) return batchErr(b, CTPWA_ERR_ARG, "precision must be 0 or 1");
    try {
        std::vector<ctpwa::Engine*> es;
        std::vector<const double*> dp(d_params, d_params + n);
        std::vector<double*> dn(d_nll, d_nll + n), dg(d_grad, d_grad + n);
        for (int i = 0; i < n; ++i) {
            if (!hs[i] || !d_params[i] || !d_nll[i] || !d_grad[i]) return batchErr(b, CTPWA_ERR_ARG, "null argument");
            es.push_back(hs[i]->eng.get());
        }
        ctpwa::Engine::nllGradMulti(es, dp, dn, dg, precision, b->scratch, (cudaStream_t)stream);
    } catch (const std::invalid_argument& e) {
        return batchErr(b, CTPWA_ERR_ARG, e.what());
    } catch (const std::exception& e) {
        return batchErr(b, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_batch_join(ctpwa_batch* b)
{
    if (!b) return batchErr(nullptr, CTPWA_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(b->mu);
    ++b->members;
    return CTPWA_OK;
}

int ctpwa_batch_leave(ctpwa_batch* b)
{
    if (!b) return batchErr(nullptr, CTPWA_ERR_ARG, "null argument");
    {
        std::lock_guard<std::mutex> lk(b->mu);
        if (b->members > 0) --b->members;
    }
    b->cv.notify_all();
    return CTPWA_OK;
}

int ctpwa_batch_eval_host(ctpwa_batch* b, ctpwa_handle* h, const double* params, double* nll, double* grad,
                          int precision)
{
    if (!b || !h || !params || !nll || !grad) return batchErr(b, CTPWA_ERR_ARG, "null argument");
    if (precision != CTPWA_FP64 && precision != CTPWA_MIXED) return setErr(h, CTPWA_ERR_ARG, "precision must be 0 or 1");
    ctpwa_batch::Request req{h, params, nll, grad, precision};
    std::unique_lock<std::mutex> lk(b->mu);
    b->pending.push_back(&req);
    ++b->requests;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds(b->window_us);
    while (!req.done) {
        const bool full = (int)b->pending.size() >= std::max(1, b->members);
        if (!b->running && !b->pending.empty() && (full || std::chrono::steady_clock::now() >= deadline)) {
            // this thread runs the round for everything pending
            std::vector<ctpwa_batch::Request*> reqs;
            reqs.swap(b->pending);
            b->running = true;
            ++b->rounds;
            lk.unlock();
            runRound(b, reqs);
            lk.lock();
            for (auto* r : reqs) r->done = true;
            b->running = false;
            b->cv.notify_all();
            continue;
        }
        if (b->running || full) b->cv.wait(lk);
        else b->cv.wait_until(lk, deadline);
    }
    return req.rc;
}

int ctpwa_batch_stats(const ctpwa_batch* b, long long* rounds, long long* requests)
{
    if (!b) return CTPWA_ERR_ARG;
    if (rounds) *rounds = b->rounds;
    if (requests) *requests = b->requests;
    return CTPWA_OK;
}

int ctpwa_fit_batched(ctpwa_batch* b, ctpwa_handle* h, double* params, const unsigned char* free_mask, const double* lo,
                      const double* hi, int precision, int max_evals, int history, double ftol, double gtol,
                      double* out4, float* eval_ms)
{
    if (!b || !h || !params || !free_mask || !lo || !hi || !out4) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (max_evals < 1 || history < 1) return setErr(h, CTPWA_ERR_ARG, "max_evals and history must be >= 1");
    const int np = h->eng->nParams();
    for (int i = 0; i < np; ++i)
        if (!(lo[i] <= hi[i])) return setErr(h, CTPWA_ERR_ARG, "lower bound above upper bound");
    ctpwa::BoxLbfgsOptions opt;
    opt.max_evals = max_evals;
    opt.m = history;
    opt.ftol = ftol;
    opt.gtol = gtol;
    int ne = 0;
    auto fg = [&](const double* x, double* f, double* g) -> int {
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = ctpwa_batch_eval_host(b, h, x, f, g, precision);
        if (eval_ms && ne < max_evals)
            eval_ms[ne] = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        ++ne;
        return rc;
    };
    ctpwa_batch_join(b);
    ctpwa::BoxLbfgsResult r;
    const int rc = ctpwa::boxLbfgs(fg, np, params, free_mask, lo, hi, opt, &r);
    ctpwa_batch_leave(b);
    if (rc != 0) return rc;
    out4[0] = r.f;
    out4[1] = r.evals;
    out4[2] = r.iters;
    out4[3] = r.status;
    return CTPWA_OK;
}

int ctpwa_fit(ctpwa_handle* h, double* params, const unsigned char* free_mask, const double* lo, const double* hi,
              int precision, int max_evals, int history, double ftol, double gtol, double* out4, float* eval_ms,
              void* stream)
{
    if (!h || !params || !free_mask || !lo || !hi || !out4) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (max_evals < 1 || history < 1) return setErr(h, CTPWA_ERR_ARG, "max_evals and history must be >= 1");
    const int np = h->eng->nParams();
    for (int i = 0; i < np; ++i)
        if (!(lo[i] <= hi[i])) return setErr(h, CTPWA_ERR_ARG, "lower bound above upper bound");
    ctpwa::BoxLbfgsOptions opt;
    opt.max_evals = max_evals;
    opt.m = history;
    opt.ftol = ftol;
    opt.gtol = gtol;
    int ne = 0;
    bool fixed = thetaFixed(h, free_mask, lo, hi);
    auto fg = [&](const double* x, double* f, double* g) -> int {
        const auto t0 = std::chrono::steady_clock::now();
        if (fixed) {
            try {
                ensureNormCache(h, x, stream);
            } catch (const std::length_error&) {
                fixed = false;  // a model the cache does not support: full passes
            } catch (const std::exception& e) {
                return setErr(h, CTPWA_ERR_CUDA, e.what());
            }
        }
        const int rc = ctpwa_nll_grad_host(h, x, f, g, precision, stream);
        if (eval_ms && ne < max_evals)
            eval_ms[ne] = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        ++ne;
        return rc;
    };
    ctpwa::BoxLbfgsResult r;
    const int rc = ctpwa::boxLbfgs(fg, np, params, free_mask, lo, hi, opt, &r);
    if (rc != 0) return rc;
    out4[0] = r.f;
    out4[1] = r.evals;
    out4[2] = r.iters;
    out4[3] = r.status;
    return CTPWA_OK;
}

int ctpwa_fit_newton(ctpwa_handle* h, double* params, const unsigned char* free_mask, const double* lo,
                     const double* hi, int precision, int max_iter, double xtol, double gtol, double fnoise, double* out4,
                     void* stream)
{
    if (!h || !params || !free_mask || !lo || !hi || !out4) return setErr(h, CTPWA_ERR_ARG, "null argument");
    if (max_iter < 1 || !(xtol >= 0.0) || !(gtol >= 0.0) || !(fnoise >= 0.0))
        return setErr(h, CTPWA_ERR_ARG, "max_iter must be >= 1 and xtol, gtol, fnoise >= 0");
    const int np = h->eng->nParams();
    for (int i = 0; i < np; ++i)
        if (!(lo[i] <= hi[i])) return setErr(h, CTPWA_ERR_ARG, "lower bound above upper bound");
    cudaStream_t s = (cudaStream_t)stream;
    try {
        if (!h->d_hess && cudaMalloc(&h->d_hess, sizeof(double) * np * np) != cudaSuccess)
            throw std::runtime_error("CUDA error: Hessian buffer allocation failed");
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    bool fixed = thetaFixed(h, free_mask, lo, hi);
    auto fg = [&](const double* x, double* f, double* g) -> int {
        if (fixed) {
            try {
                ensureNormCache(h, x, stream);
            } catch (const std::length_error&) {
                fixed = false;  // a model the cache does not support: full passes
            } catch (const std::exception& e) {
                return setErr(h, CTPWA_ERR_CUDA, e.what());
            }
        }
        return ctpwa_nll_grad_host(h, x, f, g, precision, stream);
    };
    // the exact FP64 Hessian at x (both precisions: the mixed form keeps its
    // Hessian in FP64)
    auto hf = [&](const double* x, double* H) -> int {
        try {
            std::memcpy(h->h_pin, x, sizeof(double) * np);
            if (cudaMemcpyAsync(h->d_params, h->h_pin, sizeof(double) * np, cudaMemcpyHostToDevice, s) != cudaSuccess)
                throw std::runtime_error("CUDA error: host-to-device copy failed");
            h->eng->hessianExact(h->d_params, h->d_hess, s);
            if (cudaMemcpyAsync(H, h->d_hess, sizeof(double) * np * np, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError()));
        } catch (const std::exception& e) {
            return setErr(h, CTPWA_ERR_CUDA, e.what());
        }
        return CTPWA_OK;
    };
    ctpwa::NewtonOptions opt;
    opt.max_iter = max_iter;
    opt.xtol = xtol;
    opt.gtol = gtol;
    opt.fnoise = fnoise;
    ctpwa::BoxLbfgsResult r;
    const int rc = ctpwa::boxNewton(fg, hf, np, params, free_mask, lo, hi, opt, &r);
    if (rc != 0) return rc;
    out4[0] = r.f;
    out4[1] = r.evals;
    out4[2] = r.iters;
    out4[3] = r.status;
    return CTPWA_OK;
}

int ctpwa_minimize_box(ctpwa_fg_fn fn, void* user, int n, double* x, const unsigned char* free_mask, const double* lo,
                       const double* hi, int max_evals, int history, double ftol, double gtol, double* out4)
{
    if (!fn || !x || !free_mask || !lo || !hi || !out4 || n < 1) return setErr(nullptr, CTPWA_ERR_ARG, "bad argument");
    if (max_evals < 1 || history < 1) return setErr(nullptr, CTPWA_ERR_ARG, "max_evals and history must be >= 1");
    for (int i = 0; i < n; ++i)
        if (!(lo[i] <= hi[i])) return setErr(nullptr, CTPWA_ERR_ARG, "lower bound above upper bound");
    ctpwa::BoxLbfgsOptions opt;
    opt.max_evals = max_evals;
    opt.m = history;
    opt.ftol = ftol;
    opt.gtol = gtol;
    ctpwa::BoxLbfgsResult r;
    const int rc = ctpwa::boxLbfgs([&](const double* xx, double* f, double* g) { return fn(xx, f, g, user); }, n, x,
                                   free_mask, lo, hi, opt, &r);
    if (rc != 0) return rc;
    out4[0] = r.f;
    out4[1] = r.evals;
    out4[2] = r.iters;
    out4[3] = r.status;
    return CTPWA_OK;
}

int ctpwa_minimize_box_newton(ctpwa_fg_fn fn, ctpwa_hess_fn hfn, void* user, int n, double* x,
                              const unsigned char* free_mask, const double* lo, const double* hi, int max_iter,
                              double xtol, double gtol, double fnoise, double* out4)
{
    if (!fn || !hfn || !x || !free_mask || !lo || !hi || !out4 || n < 1)
        return setErr(nullptr, CTPWA_ERR_ARG, "bad argument");
    if (max_iter < 1 || !(xtol >= 0.0) || !(gtol >= 0.0) || !(fnoise >= 0.0))
        return setErr(nullptr, CTPWA_ERR_ARG, "max_iter must be >= 1 and xtol, gtol, fnoise >= 0");
    for (int i = 0; i < n; ++i)
        if (!(lo[i] <= hi[i])) return setErr(nullptr, CTPWA_ERR_ARG, "lower bound above upper bound");
    ctpwa::NewtonOptions opt;
    opt.max_iter = max_iter;
    opt.xtol = xtol;
    opt.gtol = gtol;
    opt.fnoise = fnoise;
    ctpwa::BoxLbfgsResult r;
    const int rc = ctpwa::boxNewton([&](const double* xx, double* f, double* g) { return fn(xx, f, g, user); },
                                    [&](const double* xx, double* H) { return hfn(xx, H, user); }, n, x, free_mask, lo,
                                    hi, opt, &r);
    if (rc != 0) return rc;
    out4[0] = r.f;
    out4[1] = r.evals;
    out4[2] = r.iters;
    out4[3] = r.status;
    return CTPWA_OK;
}

int ctpwa_intensity(ctpwa_handle* h, const double* d_params, int kind, double* d_out, void* stream)
{
    if (!h || !d_params || !d_out) return setErr(h, CTPWA_ERR_ARG, "null argument");
    try {
        h->eng->intensity(d_params, kind, d_out, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_last_parts(ctpwa_handle* h, double* out6, void* stream)
{
    if (!h || !out6) return CTPWA_ERR_ARG;
    try {
        h->eng->lastParts(out6, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_event_layout(const ctpwa_handle* h, int* out4)
{
    if (!h || !out4) return CTPWA_ERR_ARG;
    const ctpwa::GeneratedModel& g = h->eng->generated();
    int nmass = 0;
    for (const auto& s : g.slots) nmass += s.type == 0 ? 1 : 0;  // AG_K_MASS
    out4[0] = g.nplane;
    out4[1] = h->eng->model().npol;
    out4[2] = (int)g.slots.size();
    out4[3] = nmass;
    return CTPWA_OK;
}

int ctpwa_spd_inverse(const double* d_a, int n, double* d_out, int* d_info, void* stream)
{
    if (!d_a || !d_out || !d_info) return setErr(nullptr, CTPWA_ERR_ARG, "null argument");
    if (n <= 0 || n > 4096) return setErr(nullptr, CTPWA_ERR_ARG, "n must be in 1..4096");
    try {
        ctpwa::spdInverse(d_a, n, d_out, d_info, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        return setErr(nullptr, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_phase_space(double M, const double* masses3, long long n, unsigned long long seed, double* d_out,
                      void* stream)
{
    if (!masses3 || (n > 0 && !d_out)) return setErr(nullptr, CTPWA_ERR_ARG, "null argument");
    try {
        ctpwa::phaseSpace(M, masses3, n, seed, d_out, (cudaStream_t)stream);
    } catch (const std::exception& e) {
        const std::string m = e.what();
        return setErr(nullptr, m.rfind("CUDA", 0) == 0 ? CTPWA_ERR_CUDA : CTPWA_ERR_ARG, m);
    }
    return CTPWA_OK;
}

int ctpwa_event_cache_layout(const ctpwa_handle* h, int* out3)
{
    if (!h || !out3) return CTPWA_ERR_ARG;
    const ctpwa::GeneratedModel& g = h->eng->generated();
    out3[0] = g.nev64;
    out3[1] = g.nevf;
    out3[2] = g.nevd;
    return CTPWA_OK;
}

int ctpwa_launch_shape(const ctpwa_handle* h, int* out14)
{
    if (!h || !out14) return CTPWA_ERR_ARG;
    const ctpwa::FusedShape& sh = h->eng->shape();
    for (int pr = 0; pr < 2; ++pr) {
        int* o = out14 + 7 * pr;
        o[0] = sh.block[pr];
        o[1] = sh.minb[pr];
        o[2] = sh.stage[pr];
        o[3] = sh.acc[pr];
        o[4] = sh.dsmem[pr];
        o[5] = h->eng->fusedGrid(pr);
        o[6] = h->eng->polPaired(pr) ? 1 : 0;
    }
    return CTPWA_OK;
}

int ctpwa_kernel_timing(ctpwa_handle* h, int slots)
{
    if (!h) return CTPWA_ERR_ARG;
    try {
        h->eng->setKernelTiming(slots);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
    return CTPWA_OK;
}

int ctpwa_kernel_times(ctpwa_handle* h, float* ms, int cap)
{
    if (!h || (!ms && cap > 0) || cap < 0) return setErr(h, CTPWA_ERR_ARG, "bad argument");
    try {
        return h->eng->kernelTimes(ms, cap);
    } catch (const std::exception& e) {
        return setErr(h, CTPWA_ERR_CUDA, e.what());
    }
}

long long ctpwa_n_events(const ctpwa_handle* h, int kind)
{
    if (!h || kind < 0 || kind > 2) return CTPWA_ERR_ARG;
    return h->eng->nEvents(kind);
}

int ctpwa_model_json(const ctpwa_handle* h, char* buf, size_t cap)
{
    if (!h) return CTPWA_ERR_ARG;
    return copyOut(ctpwa::modelToJson(h->eng->model()), buf, cap);
}

size_t ctpwa_device_bytes(const ctpwa_handle* h) { return h ? h->eng->deviceBytes() : 0; }

double ctpwa_jit_seconds(const ctpwa_handle* h) { return h ? h->eng->jitSeconds() : -1.0; }

int ctpwa_setup_times(const ctpwa_handle* h, char* buf, size_t cap)
{
    if (!h) return CTPWA_ERR_ARG;
    std::string t;
    for (const auto& p : h->eng->setupTimes()) {
        char v[64];
        std::snprintf(v, sizeof v, "%.4f", p.second);
        t += (t.empty() ? "" : ";") + p.first + "=" + v;
    }
    return copyOut(t, buf, cap);
}

const char* ctpwa_last_error(const ctpwa_handle* h)
{
    if (h) return h->err.c_str();
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_create_err.c_str();
}

int ctpwa_describe(const char* config_path, char* buf, size_t cap, char* err, size_t errlen)
{
    try {
        ctpwa::Config cfg = ctpwa::loadConfig(config_path ? config_path : "config.yml");
        if (!cfg.valid())
            throw std::runtime_error("analysis not initialized: invalid or missing config file \"" +
                                     std::string(config_path ? config_path : "config.yml") + "\"");
        ctpwa::Model m = ctpwa::buildModel(cfg, 1);
        for (const auto& b : m.blocks)
            for (const auto& r : b.res)
                if (r.type == ctpwa::ModelType::Custom) ctpwa::checkCustomExpr(r.options.at("expr"), r.param_names);
        return copyOut(ctpwa::modelToJson(m), buf, cap);
    } catch (const std::exception& e) {
        std::string m = e.what();
        setErr(nullptr, CTPWA_ERR_CONFIG, m);
        if (err && errlen) copyOut(m, err, errlen);
        return CTPWA_ERR_CONFIG;
    }
}

int ctpwa_precompile(const char* config_path, double* seconds, char* err, size_t errlen)
{
    try {
        double s = ctpwa::precompileConfig(config_path ? config_path : "config.yml");
        if (seconds) *seconds = s;
    } catch (const std::exception& e) {
        std::string m = e.what();
        setErr(nullptr, CTPWA_ERR_CONFIG, m);
        if (err && errlen) copyOut(m, err, errlen);
        return m.find("NVRTC") != std::string::npos ? CTPWA_ERR_CUDA : CTPWA_ERR_CONFIG;
    }
    return CTPWA_OK;
}

const char* ctpwa_version(void) { return "ctpwa_b200 0.1.0"; }

}  // extern "C"
