/*
 * ctpwa_b200 C ABI — the drop-in boundary of the B200 likelihood engine.
 *
 * Each entry point replaces one member of the reference's pybind11 class
 * `ctpwa.analysis` (src/main.cu:91-131), whose methods a Python, ctypes,
 * cffi or C/C++ host binds; the Python module ctpwa_b200 binds these with
 * ctypes and keeps the reference method names and tensor contracts.
 *
 * Conventions
 *  - Parameter vectors use the reference layout [Re p (nV), Im p (nV), theta (nT)]
 *    (src/Analysis.cu:629-681, src/Parameters.cu:263-300), nV = ctpwa_n_vector,
 *    nT = ctpwa_n_free_theta.
 *  - Functions return 0 on success and a negative status on failure; the
 *    message is available from ctpwa_last_error (no exit(), no exceptions
 *    across the ABI).
 *  - Evaluation entry points taking device pointers are stream ordered on the
 *    given cudaStream_t (passed as void*, 0 = legacy default stream), perform
 *    no host synchronisation and no allocation, and may be captured in a CUDA
 *    graph. Each handle owns its scratch; different handles are independent.
 */
#ifndef CTPWA_B200_H
#define CTPWA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ctpwa_handle ctpwa_handle;

#define CTPWA_OK 0
#define CTPWA_ERR_CONFIG (-1)   /* invalid config / model (reference: isValid()=False, runtime_error) */
#define CTPWA_ERR_CUDA (-2)     /* CUDA runtime / NVRTC failure */
#define CTPWA_ERR_ARG (-3)      /* bad argument (reference: TORCH_CHECK -> RuntimeError) */

#define CTPWA_FP64 0            /* plain FP64 path (reference built with CTPWA_DOUBLE_COMPLEX) */
#define CTPWA_MIXED 1           /* FP32 amplitudes, FP64 reductions */

/* Replaces: analysis(config_file) — src/Analysis.cu:1271-1281 (initialize :3849-4208).
 * Builds the model, reads the samples, computes the angular/kinematic caches on
 * `device` and JIT-compiles the model's fused kernel. Returns NULL on failure
 * with *status set and the message copied to err (if non-NULL). */
ctpwa_handle* ctpwa_create(const char* config_path, int device, int* status, char* err, size_t errlen);

/* Event-sharded variant of ctpwa_create for multi-GPU evaluation: keeps the
 * contiguous event block `rank` of `world` of every sample, as the
 * reference's multi-device split does (src/Analysis.cu:4210-4238). */
ctpwa_handle* ctpwa_create_shard(const char* config_path, int device, int rank, int world, int* status, char* err,
                                 size_t errlen);

/* In-memory samples (no counterpart in the reference, which reads every
 * sample from the files of its config): the model from config_path, the
 * events from device arrays instead of the config's Data files. For k = 0
 * phase space, 1 data, 2 background: p4[k] device pointer to AoS
 * [n[k]][n_final][4] (E, px, py, pz in the config's Data.order; n[2] = 0 for
 * no background), w[k] device per-event weights or nullptr (unit weights).
 * The arrays are copied during the call; the caller keeps them. For toy-MC
 * jobs whose events are generated on the device (no file round trip). */
ctpwa_handle* ctpwa_create_from_device(const char* config_path, int device, const double* const* p4,
                                       const long long* n, const double* const* w, int* status, char* err,
                                       size_t errlen);

/* The same with creation flags. CTPWA_CREATE_FP64_ONLY: no mixed-form
 * tables and no polarisation pairing (nor its compact tables): a handle
 * for FP64 evaluations and intensities only, cheaper to build (a toy
 * generator's accept-reject candidates); a mixed-form evaluation on it fails
 * with CTPWA_ERR_CUDA ("mixed-precision tables were not built"). Unknown
 * flags: CTPWA_ERR_ARG. No counterpart in the reference. */
#define CTPWA_CREATE_FP64_ONLY 1
ctpwa_handle* ctpwa_create_from_device_flags(const char* config_path, int device, const double* const* p4,
                                             const long long* n, const double* const* w, int flags, int* status,
                                             char* err, size_t errlen);

/* Releases device memory of the handle (the reference never frees;
 * src/Analysis.cu:1284-1290) into this library's per-device memory pool,
 * where later handles reuse it. It does not wait for work on the caller's
 * streams: work queued on the handle must be complete. */
void ctpwa_destroy(ctpwa_handle* h);

/* Replaces: analysis::getNVector — src/Analysis.cu:1311-1315 (vspace fit mode). */
int ctpwa_n_vector(const ctpwa_handle* h);

/* Replaces: analysis::getNFreeTheta — src/Analysis.cu:1316. */
int ctpwa_n_free_theta(const ctpwa_handle* h);

/* Replaces: analysis::getNParams — src/Analysis.cu:1344 (= 2 nV + nT). */
int ctpwa_n_params(const ctpwa_handle* h);

/* Replaces: analysis::getParamNames — src/Analysis.cu:1318-1342.
 * Writes the names separated by '\n' (NUL-terminated); returns the number of
 * bytes needed including the terminator (call with cap = 0 to size). */
int ctpwa_param_names(const ctpwa_handle* h, char* buf, size_t cap);

/* Replaces: analysis::getFreeResParams — src/Analysis.cu:3779-3792.
 * out: host array [3][nT] = (initial value, lower bound, upper bound). */
int ctpwa_free_res_params(const ctpwa_handle* h, double* out);

/* Replaces: analysis::getNLL forward + NLLFunction::backward — src/Analysis.cu:625-1261.
 * d_params [n_params], d_nll [1], d_grad [n_params]: device pointers.
 * precision: CTPWA_FP64 or CTPWA_MIXED. */
int ctpwa_nll_grad(ctpwa_handle* h, const double* d_params, double* d_nll, double* d_grad, int precision, void* stream);

/* Allocation-free variant of ctpwa_nll_grad. No counterpart in the reference.
 *
 * For callers that cannot let a library allocate device memory for them: a
 * host program that hands all device memory to its own pool allocator after
 * start-up, or one that counts every device byte against a fixed budget (a
 * serving loop that admits jobs by memory). The evaluation scratch (coupling
 * vector, parameter-only constants, one partial-sum row per CTA) lives in one
 * fixed 2 MiB array compiled into libctpwa_b200.so, present on every GPU that
 * loads the library until the process exits; the call allocates nothing.
 * Besides that array it writes one per-handle buffer that the regular entry
 * point writes too: the handle's kernel-module constant block (the per-call
 * constants and couplings the fused kernel reads), so a static call must be
 * ordered (same stream, or an event) against the same handle's other
 * evaluations. Same arguments, results (bit for bit) and stream ordering as
 * ctpwa_nll_grad.
 *  - A model whose scratch does not fit (about 4 + 2 nA + nT doubles per CTA
 *    row, up to 8 rows per SM) is rejected with CTPWA_ERR_ARG and a message;
 *    use ctpwa_nll_grad for it.
 *  - The first call on a device looks the array's address up (once per
 *    device, with the handle's device current); make that first call before
 *    beginning any stream capture on the device.
 *  - Every call writes all the scratch it reads (its error flag is cleared
 *    by the call's first kernel), so nothing needs clearing beforehand, but
 *    all handles on a device share the one array: calls whose GPU work can
 *    overlap (other streams, threads or handles without ordering between
 *    them) race and give wrong results. ctpwa_last_parts does not see these
 *    calls. */
int ctpwa_nll_grad_static(ctpwa_handle* h, const double* d_params, double* d_nll, double* d_grad, int precision,
                          void* stream);

/* Replaces: analysis::getHessian — src/Analysis.cu:2689-3378.
 * d_hess: device [n_params][n_params] row-major, grouped [Re p, Im p, theta]
 * like the reference. Central differences of the exact FP64 device gradient
 * with steps h_i = rel_step * max(|p_i|, 1e-2) (rel_step in (0, 1e-2];
 * 1e-5 is the library default), symmetrised; 2 n_params gradient evaluations
 * queued on the stream, no host synchronisation, no allocation. */
int ctpwa_hessian(ctpwa_handle* h, const double* d_params, double* d_hess, double rel_step, void* stream);

/* Replaces: analysis::getHessian — src/Analysis.cu:2689-3378 (with
 * computeDataHessianContribFast, computePhspHessian, computeUnifiedHessian and
 * transformExtendedHessian, src/ComputeHessian.cu:149-1556,
 * src/AmpGen.cu:3020-3540, src/Parameters.cu:348-584).
 * The exact FP64 Hessian, same layout as ctpwa_hessian: forward-mode
 * (dual-number) derivatives of the device gradient pass along the n_params
 * unit directions, symmetrised. The first call on a handle compiles the
 * kernels (or loads them from the kernel cache) and allocates their buffers;
 * later calls are queued on the stream without host synchronisation. */
int ctpwa_hessian_exact(ctpwa_handle* h, const double* d_params, double* d_hess, void* stream);

/* The Hessian (same layout as ctpwa_hessian_exact) with its coupling block
 * formed from tensor-core Gram sums: over data and background the sums
 * sum (w/f) A_a conj(A_b) and sum (w/f^2) c_a conj(c_b) (c_a = sum_pol
 * A_a conj(S)), over phase space the normalisation matrix, in FP32
 * amplitudes with split-BF16 products and FP64 assembly (~1e-6 relative to
 * the exact Hessian); the resonance-parameter rows from the exact FP64
 * Hessian-vector products along their unit directions. The reference builds
 * its Hessian from Gram products of the stored amplitudes
 * (src/ComputeHessian.cu:149-1556). Host-synchronising; needs
 * (npol + 1) * 2 * nA <= 128 (CTPWA_ERR_ARG otherwise). */
int ctpwa_hessian_gram(ctpwa_handle* h, const double* d_params, double* d_hess, void* stream);

/* Launch shape of the tensor-core Gram kernel (compiled on first use):
 * out4 = {grid, dynamic shared memory bytes, resident CTAs per SM from the
 * occupancy query, threads per CTA}. No counterpart in the reference. */
int ctpwa_gram_shape(ctpwa_handle* h, int* out4);

/* Replaces: the phase-space normalisation matrix of the reference, built by
 * scalePhspAmpsKernel + CGEMM over its amplitude table
 * (src/ComputeHessian.cu:1181-1197, src/Analysis.cu:729-805; used by its
 * quadratic form, src/ComputeNLL.cu:414-597, and its Hessian).
 * d_out [nA][nA] complex (re, im interleaved), FP64, device pointer:
 *   M_ab = (1/W) sum_e w_e sum_pol A_a conj(A_b)
 * over the phase-space sample at d_params, amplitudes in the mixed form
 * (FP32), products on the tensor cores (BF16 hi + lo split operands, FP32
 * accumulation in tensor memory, FP64 across chunks of 1024 events).
 * Models with npol * 2 * nA > 128 are rejected with CTPWA_ERR_ARG. The first
 * call compiles the kernels (or loads them from the kernel cache) and
 * allocates their per-CTA partial buffer; later calls are stream-ordered
 * without host synchronisation. */
int ctpwa_gram(ctpwa_handle* h, const double* d_params, double* d_out, void* stream);

/* Normalisation cache. Replaces: the reference's phase-space matrix
 * d_phsp_matrix_ = A^H diag(w/W) A, kept between its evaluations when no
 * resonance parameter is free and used through its quadratic form
 * (src/Analysis.cu:748-829, src/ComputeNLL.cu:575-597). Here the matrices
 * are FP64 and carry the lineshape derivatives as well, so that the
 * normalisation term, the coupling gradient and the resonance-parameter
 * gradient at fixed resonance parameters all come from them:
 * ctpwa_norm_cache_build sums them over the phase-space sample at the
 * resonance parameters of d_params (FP64, one pass; host-synchronising;
 * *ms, if not null, receives the pass's device time). While the cache is
 * set, ctpwa_nll_grad_host, ctpwa_fit and ctpwa_fit_newton evaluate every
 * point whose resonance parameters equal the cached ones bitwise from the
 * data and background samples and the matrices alone (the phase-space
 * sample is not read); other points take the full pass. ctpwa_fit and
 * ctpwa_fit_newton build the cache themselves when no resonance parameter
 * is free (free[i] == 0 or lo[i] == hi[i] for all of them).
 * ctpwa_nll_grad_cached is the device-buffer evaluation from the cache; its
 * resonance parameters must equal the cached ones, otherwise the result is
 * flagged invalid (NLL 1e30, zero gradient). ctpwa_norm_cache_valid returns
 * 1 while a cache is set, 0 otherwise. */
int ctpwa_norm_cache_build(ctpwa_handle* h, const double* d_params, double* ms, void* stream);
int ctpwa_norm_cache_clear(ctpwa_handle* h);
int ctpwa_norm_cache_valid(const ctpwa_handle* h);
int ctpwa_nll_grad_cached(ctpwa_handle* h, const double* d_params, double* d_nll, double* d_grad, int precision,
                          void* stream);

/* Exact Hessian-vector products (no counterpart in the reference, which only
 * forms the full matrix): d_out[d] = H(d_params) d_dirs[d] for ndir directions
 * (device [ndir][n_params] in, [ndir][n_params] out). */
int ctpwa_hvp(ctpwa_handle* h, const double* d_params, const double* d_dirs, int ndir, double* d_out, void* stream);

/* Event-sharded Hessian-vector products (the multi-GPU form of
 * ctpwa_hessian_exact; the reference sums per-GPU Hessian contributions with
 * peer copies, src/Analysis.cu:2689-3378): this handle's per-sample tangent
 * sums, ctpwa_hvp_sums_size(h, ndir) doubles, to be summed over shards; then
 * the rows H u_d from the summed value sums (ctpwa_shard_sums, FP64) and the
 * summed tangent sums. */
int ctpwa_hvp_sums_size(const ctpwa_handle* h, int ndir);
int ctpwa_shard_hvp_sums(ctpwa_handle* h, const double* d_params, const double* d_dirs, int ndir, double* d_tsums,
                         void* stream);
int ctpwa_finalize_hvp(ctpwa_handle* h, const double* d_params, const double* d_dirs, int ndir, const double* d_vsums,
                       const double* d_tsums, double* d_out, void* stream);

/* Number of resonance blocks (the partial waves of the fit fractions; the
 * reference's nSLvectors_, src/Analysis.cu:1350). */
int ctpwa_n_blocks(const ctpwa_handle* h);

/* Replaces the partial integrals of analysis::getFitFractions —
 * src/Analysis.cu:3431-3526 (computeTruthBatchIntegrals), src/ComputeBF.cu:9-60.
 * d_out[i] = sum_e w_e sum_pol |sum_{a in block i} v_a A_a|^2 over sample kind
 * 0 (phase space), 1 (data), 2 (background) or 3 (Data.phsp_truth, read and
 * prepared on the first call), at d_params; device pointers, FP64. */
int ctpwa_partial_integrals(ctpwa_handle* h, const double* d_params, int kind, double* d_out, void* stream);

/* Row stride (events, padded to a multiple of 256) of the per-event export
 * arrays of sample kind (0 phase space, 1 data, 2 background). */
long long ctpwa_table_stride(const ctpwa_handle* h, int kind);

/* Replaces the device part of analysis::writeResult — src/Analysis.cu:1355-1700
 * (computeResults, src/ComputeResults.cu) — over the phase-space sample, FP64:
 *   d_total[e]          intensity of event e (of the blocks with wave_mask[i] != 0
 *                       when wave_mask, a host array of ctpwa_n_blocks ints, is given)
 *   d_partial[i*ld + e] intensity of block i alone
 *   d_interf_ev[k*ld + e] (optional, may be NULL) 2 Re(P_i conj(P_j)) of pair k (i < j)
 *   d_interf[k]         the same summed over events for pairs i <= j (diagonal 2|P_i|^2),
 *                       packed k = i*n - i*(i-1)/2 + (j - i)
 * with ld = ctpwa_table_stride(h, 0); device pointers. Normalisation to the
 * data yield is left to the caller (ctpwa_b200.analysis.writeResult). */
int ctpwa_export_weights(ctpwa_handle* h, const double* d_params, const int* wave_mask, double* d_total,
                         double* d_partial, double* d_interf_ev, double* d_interf, void* stream);

/* Event-sharded evaluation, the exchange step of the reference's multi-device
 * NLL (src/Analysis.cu:4210-4238, which gathers per-device partial results
 * with peer copies). ctpwa_shard_sums writes this shard's per-sample sums
 * (ctpwa_sums_size doubles: [phase space, data, background] x [sum -w log f,
 * sum f, coupling-gradient terms (re, im) x nA, theta-gradient terms x nT],
 * then [n_phsp, W_phsp, W_data, W_bkg]); the caller sums these buffers over
 * the shards (one all-reduce) and ctpwa_finalize_sums turns the total into
 * the NLL and gradient of the union of the shards. Device pointers,
 * stream-ordered, no host synchronisation. ctpwa_finalize_sums takes the sums
 * to be of the precision of this handle's last ctpwa_shard_sums call: sums
 * of the mixed form, which is evaluated at the couplings rounded to FP32,
 * get the first-order term of the rounding added to the NLL. */
int ctpwa_sums_size(const ctpwa_handle* h);
int ctpwa_shard_sums(ctpwa_handle* h, const double* d_params, int precision, double* d_sums, void* stream);
int ctpwa_finalize_sums(ctpwa_handle* h, const double* d_params, const double* d_sums, double* d_nll, double* d_grad,
                        void* stream);

/* Same evaluation from host buffers: copies params host->device, evaluates,
 * copies NLL and gradient back, and synchronises the stream. */
int ctpwa_nll_grad_host(ctpwa_handle* h, const double* params, double* nll, double* grad, int precision, void* stream);

/* Fit driver: minimises the NLL over the parameters with free[i] != 0 within
 * lo[i] <= p[i] <= hi[i] (host arrays of n_params; +-INFINITY for none) by
 * projected limited-memory BFGS (history correction pairs), one evaluation
 * through ctpwa_nll_grad_host per function call, on the calling thread and
 * stream. Replaces the reference's fit loop, torch.optim.LBFGS over
 * parameters clamped into their bounds with the gradient components that
 * point out of an active bound zeroed (example/fit.py:113-200). params (host)
 * holds the start and receives the best point found; out4 receives {nll at
 * that point, evaluations, iterations, status}: status 0 projected gradient
 * <= gtol, 1 relative decrease <= ftol, 2 max_evals spent, 3 no decrease
 * along the search direction. eval_ms (optional, capacity max_evals)
 * receives each evaluation's host latency in ms. */
int ctpwa_fit(ctpwa_handle* h, double* params, const unsigned char* free_mask, const double* lo, const double* hi,
              int precision, int max_evals, int history, double ftol, double gtol, double* out4, float* eval_ms,
              void* stream);

/* Newton fit with the exact FP64 Hessian (ctpwa_hessian_exact) over the same
 * box and free variables as ctpwa_fit: Levenberg-Marquardt steps (H + lambda
 * diag|H|) s = -g, projected onto the box, kept when the NLL (in `precision`)
 * falls by 1e-4 of the quadratic model's prediction or, for a predicted
 * decrease <= fnoise, rises by at most fnoise (the NLL's rounding level). It
 * converges to the stationary point of the start's basin. The reference
 * checks the Hessian at its L-BFGS result for positive definiteness
 * (example/fit.py:202-230); this routine polishes a start to such a point,
 * quadratically. out4: {nll, evaluations, Hessians, status}: status 0
 * projected gradient <= gtol, 1 a step of max_i |s_i| sqrt(H_ii) <= xtol or
 * with a predicted decrease <= 1e-2 fnoise, 2 max_iter Hessians spent, 3 no
 * acceptable step. */
int ctpwa_fit_newton(ctpwa_handle* h, double* params, const unsigned char* free_mask, const double* lo,
                     const double* hi, int precision, int max_iter, double xtol, double gtol, double fnoise, double* out4,
                     void* stream);

/* Evaluation batches (no counterpart in the reference, which serves one
 * analysis per process): several handles of one model (equal configuration,
 * hence one generated kernel) evaluated in one prepare, one prologue, one
 * fused and one finalize launch. Each job keeps its own CTAs, partial rows
 * and finalize, so its NLL and gradient equal those of ctpwa_nll_grad bit
 * for bit. A batch owns a CUDA stream and a small argument table on `device`
 * (grown on demand by the first calls); jobs of another model or device are
 * rejected with CTPWA_ERR_ARG. */
typedef struct ctpwa_batch ctpwa_batch;
ctpwa_batch* ctpwa_batch_create(int device);
void ctpwa_batch_destroy(ctpwa_batch* b);

/* Device pointers per job; stream-ordered on `stream` (not the batch's own),
 * no host synchronisation beyond the reuse of the batch's argument table. */
int ctpwa_nll_grad_multi(ctpwa_batch* b, ctpwa_handle* const* hs, int n, const double* const* d_params,
                         double* const* d_nll, double* const* d_grad, int precision, void* stream);

/* Serving: blocking host-buffer evaluation gathered across threads. A fit
 * that joined the batch (ctpwa_batch_join) submits each evaluation with
 * ctpwa_batch_eval_host; the call returns when its result is in nll / grad.
 * Requests wait until every joined fit has one pending, or at most 200
 * microseconds, and one waiting thread then runs all pending requests (one
 * multi-job launch per model and precision) on the batch's stream.
 * ctpwa_batch_leave ends a fit's membership. */
int ctpwa_batch_join(ctpwa_batch* b);
int ctpwa_batch_leave(ctpwa_batch* b);
int ctpwa_batch_eval_host(ctpwa_batch* b, ctpwa_handle* h, const double* params, double* nll, double* grad,
                          int precision);
/* rounds run and requests served so far (either pointer may be NULL) */
int ctpwa_batch_stats(const ctpwa_batch* b, long long* rounds, long long* requests);

/* ctpwa_fit with every evaluation gathered into the batch (joins the batch
 * for the duration of the minimisation). Same arguments and results. */
int ctpwa_fit_batched(ctpwa_batch* b, ctpwa_handle* h, double* params, const unsigned char* free_mask, const double* lo,
                      const double* hi, int precision, int max_evals, int history, double ftol, double gtol,
                      double* out4, float* eval_ms);

/* The same minimiser over a host function (no GPU): fn(x, &f, g, user)
 * returns 0, or a nonzero code that ends the minimisation and is returned. */
typedef int (*ctpwa_fg_fn)(const double* x, double* f, double* g, void* user);
int ctpwa_minimize_box(ctpwa_fg_fn fn, void* user, int n, double* x, const unsigned char* free_mask, const double* lo,
                       const double* hi, int max_evals, int history, double ftol, double gtol, double* out4);

/* The Newton fit of ctpwa_fit_newton over host functions (no GPU): hfn(x, H,
 * user) writes the row-major n x n Hessian at x and returns 0 or a nonzero
 * code that ends the minimisation and is returned. */
typedef int (*ctpwa_hess_fn)(const double* x, double* H, void* user);
int ctpwa_minimize_box_newton(ctpwa_fg_fn fn, ctpwa_hess_fn hfn, void* user, int n, double* x,
                              const unsigned char* free_mask, const double* lo, const double* hi, int max_iter,
                              double xtol, double gtol, double fnoise, double* out4);

/* Per-sample parts of the last evaluation (host, synchronising):
 * [data_nll, bkg_nll, sum_phsp_intensity, W_data, W_bkg, n_phsp]. */
int ctpwa_last_parts(ctpwa_handle* h, double* out6, void* stream);

/* Per-event intensity f_e = sum_pol |sum_a v_a A_a|^2 of sample kind (0 phase
 * space, 1 data, 2 background) at d_params; d_out: device array [n_events].
 * The reference computes the same quantity inside computeFactorNLL
 * (src/ComputeNLL.cu:21-84) and for its result export (ComputeResults.cu:22). */
int ctpwa_intensity(ctpwa_handle* h, const double* d_params, int kind, double* d_out, void* stream);

/* Replaces: the covariance step of the reference's fit driver, the inverse
 * of the Hessian over the free parameters (example/fit.py:213,333,
 * torch.linalg.inv on the Hessian). d_a [n][n] symmetric positive definite,
 * row-major FP64 (device), d_out [n][n] its inverse (device, symmetrised),
 * *d_info (device int) 0 or k + 1 when the k-th pivot of the elimination is
 * not positive (not positive definite; d_out is then not an inverse).
 * Gauss-Jordan elimination in FP64 in one CTA, n <= 4096; stream-ordered,
 * no host synchronisation, no allocation. */
int ctpwa_spd_inverse(const double* d_a, int n, double* d_out, int* d_info, void* stream);

/* Toy-MC events on the device (no counterpart in the reference, whose toys
 * are generated outside the library): n events of uniform three-body phase
 * space for a parent of mass M at rest decaying to masses[0..2], written to
 * d_out [n][3][4] (E, px, py, pz per particle) on the current device; event i
 * depends only on (seed, i) (counter-based Philox-4x32-10 random numbers). */
int ctpwa_phase_space(double M, const double* masses3, long long n, unsigned long long seed, double* d_out,
                      void* stream);

/* Per-event layout of the device event caches (no counterpart in the
 * reference): out[0] angular planes, out[1] polarisation states, out[2]
 * kinematic values the lineshapes are built from, out[3] of which invariant
 * masses. */
int ctpwa_event_layout(const ctpwa_handle* h, int* out4);

/* Per-event frontier tables (no counterpart in the reference): the
 * parameter-independent lineshape subexpressions each evaluation reads,
 * computed once per event when the samples are loaded. out[0] FP64 values of
 * the plain path, out[1] FP32 and out[2] FP64 values of the mixed form. */
int ctpwa_event_cache_layout(const ctpwa_handle* h, int* out3);

/* Launch shape of the fused kernels (no counterpart in the reference): for
 * the plain [0..6] and mixed [7..13] kernels: threads per CTA, minimum
 * resident CTAs per SM, table staging mode (0 off, 1 frontier rows, 2
 * frontier and angular rows, 3 frontier values by asynchronous copies),
 * gradient sums in shared memory (0/1), dynamic shared memory bytes per CTA,
 * CTAs per launch, polarisation pairing of the angular tables (1: only the
 * first (npol+1)/2 polarisations stored, the others their conjugates). */
int ctpwa_launch_shape(const ctpwa_handle* h, int* out14);

/* Per-launch timing of the fused likelihood kernel (no counterpart in the
 * reference, which times nothing on the device). slots > 0 records a CUDA
 * event pair on the launching stream around every fused launch, in a ring of
 * `slots` pairs; slots = 0 switches timing off. */
int ctpwa_kernel_timing(ctpwa_handle* h, int slots);

/* Durations in milliseconds of the most recent fused launches (at most cap,
 * oldest first); waits for their end events. Returns the number written. */
int ctpwa_kernel_times(ctpwa_handle* h, float* ms, int cap);

/* Event counts of phase space (kind 0), data (1), background (2). */
long long ctpwa_n_events(const ctpwa_handle* h, int kind);

/* Lowered model as JSON (columns, groups, theta slots, coupling map); same
 * sizing convention as ctpwa_param_names. */
int ctpwa_model_json(const ctpwa_handle* h, char* buf, size_t cap);

/* Device bytes held by the handle's event caches. */
size_t ctpwa_device_bytes(const ctpwa_handle* h);

/* Seconds spent compiling (or loading from the disk cache) the fused kernel. */
double ctpwa_jit_seconds(const ctpwa_handle* h);

/* Host milliseconds of the handle's set-up phases (model, context, kernels,
 * samples, angular_tables, angular, pairing, buffers; each phase's device
 * work finished), as "name=ms;name=ms" into buf (cap bytes, NUL-terminated).
 * Returns the length the full text needs, including the NUL. */
int ctpwa_setup_times(const ctpwa_handle* h, char* buf, size_t cap);

/* Message of the last failure on this handle (or of the last failed create when h is NULL). */
const char* ctpwa_last_error(const ctpwa_handle* h);

/* Host-only model description (no GPU): the lowered model of a config as
 * JSON, as ctpwa_model_json. Replaces the reference's DecayInfo class
 * (src/main.cu:41-51, src/Info.cu:43-357) for inspection of amplitude and
 * parameter names. Returns the bytes needed (>0) or a negative status. */
int ctpwa_describe(const char* config_path, char* buf, size_t cap, char* err, size_t errlen);

/* Ahead-of-time compile of a config's fused kernel into the kernel cache
 * (NVRTC only; no GPU needed). The reference compiles its lineshape JIT on the
 * first getNLL call (src/JITCustom.cu:894-1003); this moves that cost out of
 * the first evaluation. seconds (optional) receives the time spent. */
int ctpwa_precompile(const char* config_path, double* seconds, char* err, size_t errlen);

/* Library version string. */
const char* ctpwa_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CTPWA_B200_H */
