// Likelihood engine: device-resident samples, angular/kinematic caches,
// the JIT-compiled fused NLL + adjoint kernel and its finalize step.
#pragma once

#include "codegen.hpp"
#include "dataio.hpp"
#include "model.hpp"

#include <cuda_runtime.h>

#include <string>
#include <cstdint>
#include <vector>

namespace ctpwa {

enum Precision : int { kFP64 = 0, kMixed = 1 };

// Launch shape of the plain [0] and mixed [1] fused kernels: block size,
// minimum resident CTAs per SM, the staging of the event tables through
// shared memory (0 off; 1, 2 per-warp bulk copies; 3 per-thread
// asynchronous copies of the frontier values), gradient sums in shared
// memory, and the dynamic shared memory bytes per CTA (fusedShape decides
// them per model).
struct FusedShape {
    int block[2] = {192, 256};
    int minb[2] = {2, 2};
    int stage[2] = {0, 0};
    int acc[2] = {1, 0};  // per-thread gradient sums in shared memory
    int dsmem[2] = {0, 0};
};
FusedShape fusedShape(const GeneratedModel& gen);

struct DeviceSample {
    long long n = 0;
    long long ld = 0;          // row stride of the tables below (n padded to 256)
    double* p4 = nullptr;      // SoA [n_final * 4][n]
    double2* slamp64 = nullptr;  // [nplane * npol][ld]
    float2* slamp32 = nullptr;   // mixed-precision copy (polarisation-paired when the engine pairs them)
    double2* slamp64p = nullptr; // polarisation-paired FP64 copy for the plain fused kernel
    double* kin = nullptr;     // [nkin][ld] kinematic cache (initialisation only)
    double* ev64 = nullptr;    // [nev64][ld] frontier values, FP64
    float* evf = nullptr;      // [nevf][ld] mixed form, FP32 frontier values
    double* evd = nullptr;     // [nevd][ld] mixed form, FP64 frontier values
    double* w = nullptr;       // weights or nullptr
    double wsum = 0.0;         // sum of weights (or n)
};

// Host staging and device copy of the argument tables of a multi-job
// evaluation (Engine::nllGradMulti); reused across calls, grown on demand.
struct MultiScratch {
    void* host = nullptr;  // pinned
    void* dev = nullptr;
    size_t cap = 0;
    cudaEvent_t copied = nullptr;  // the last host -> device copy of the tables
    MultiScratch() = default;
    MultiScratch(const MultiScratch&) = delete;
    MultiScratch& operator=(const MultiScratch&) = delete;
    ~MultiScratch();
};

struct EngineOptions {
    int device = 0;
    bool keep_momenta = false;
    bool mixed_tables = true;  // build the FP32 angular table for the mixed path
    bool pair_polarisations = true;  // check the conjugate pairing and build the compact tables
    int shard_rank = 0;        // keep event block shard_rank of shard_world of every sample
    int shard_world = 1;
    // In-memory samples: when set, the events come from these device arrays
    // (AoS [n][n_final][4], the config's Data.order; weights or nullptr)
    // instead of the config's Data files; the arrays are copied.
    bool device_samples = false;
    const double* dev_p4[3] = {nullptr, nullptr, nullptr};
    long long dev_n[3] = {0, 0, 0};
    const double* dev_w[3] = {nullptr, nullptr, nullptr};
};

// Compile (or find in the disk cache) the fused kernel of a config's model
// without touching a GPU; returns seconds spent.
double precompileConfig(const std::string& config_path);

// Seeded three-body phase space for a parent of mass M at rest on the current
// device: d_out [n][3][4] (E, px, py, pz), event i a function of (seed, i)
// only (csrc/toymc.cu).
void phaseSpace(double M, const double* masses, long long n, unsigned long long seed, double* d_out,
                cudaStream_t stream);

// Inverse of the symmetric positive definite FP64 matrix a [n][n] (row-major,
// device) into out (device), on the device in one CTA; *d_info (device) = 0,
// or k + 1 when the k-th pivot is not positive (a not positive definite).
// Stream-ordered, no host synchronisation (csrc/linalg.cu).
void spdInverse(const double* d_a, int n, double* d_out, int* d_info, cudaStream_t stream);

class Engine {
public:
    Engine(const std::string& config_path, const EngineOptions& opt);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    const Model& model() const { return model_; }
    int nParams() const { return model_.nParams(); }

    // NLL and gradient in the reference layout [Re p, Im p, theta]; all
    // pointers are device pointers; stream-ordered, no host synchronisation.
    void nllGrad(const double* d_params, double* d_nll, double* d_grad, int precision, cudaStream_t stream);
    // The same evaluation with its scratch (couplings, parameter-only
    // constants, per-CTA partial rows, per-sample parts) in one fixed array
    // compiled into the library instead of the handle's buffers; allocates
    // nothing. Throws std::length_error when this model's scratch exceeds the
    // array (kStaticScratchBytes). All handles on a device share the array;
    // the handle's module constant block (k_sym_) is written as by nllGrad,
    // so calls on one handle must be ordered against its other evaluations.
    void nllGradStatic(const double* d_params, double* d_nll, double* d_grad, int precision, cudaStream_t stream);
    // The evaluations of several handles of one model (same generated kernel)
    // in one prepare, prologue, fused and finalize launch on `stream`; each
    // job's NLL and gradient equal its own nllGrad's. Device pointers per job.
    // Identity of the compiled fused kernel image (generated model and
    // launch layout): handles with equal keys can share a multi-job launch.
    const void* kernelImageKey() const
    {
        return (const void*)((uintptr_t)image_key_ ^ (paired_[0] ? 1u : 0u) ^ (paired_[1] ? 2u : 0u));
    }
    static void nllGradMulti(const std::vector<Engine*>& es, const std::vector<const double*>& d_params,
                             const std::vector<double*>& d_nll, const std::vector<double*>& d_grad, int precision,
                             MultiScratch& sc, cudaStream_t stream);
    // Phase-space Gram matrix M_ab = (1/W) sum_e w_e sum_p A_a conj(A_b) of the
    // mixed-form amplitudes at d_params, on the tensor cores; d_out [nA][nA]
    // complex (re, im) FP64. The first call compiles the kernels.
    void gram(const double* d_params, double* d_out, cudaStream_t stream);
    // Gram launch: grid, dynamic shared memory, resident CTAs per SM, block (compiles it if needed)
    void gramShape(int* out4);
    // Hessian with its coupling block from tensor-core Gram sums (host-synchronising)
    void hessianGram(const double* d_params, double* d_hess, cudaStream_t stream);
    // Normalisation cache (kernels/norm.cuh): the phase-space sums as FP64
    // quadratic forms in the couplings at the resonance parameters of
    // d_params. normCacheBuild computes them (one pass over the phase-space
    // sample; host-synchronising; returns the pass's device time in ms);
    // nllGradCached then evaluates at any couplings with those resonance
    // parameters from the data and background samples and the matrices
    // alone. Its resonance parameters must equal the cached ones bitwise; if
    // not, the evaluation is flagged invalid (NLL 1e30, zero gradient).
    double normCacheBuild(const double* d_params, cudaStream_t stream);
    void normCacheClear() { norm_valid_ = false; }
    bool normCacheValid() const { return norm_valid_; }
    // true when the cache is valid for the resonance parameters of the host array params
    bool normCacheMatches(const double* params) const;
    void nllGradCached(const double* d_params, double* d_nll, double* d_grad, int precision, cudaStream_t stream);
    static constexpr size_t kStaticScratchBytes = size_t(2) << 20;
    // Event-sharded evaluation: the per-sample sums of this handle's events,
    // [3][nacc] + [n_phsp, W_phsp, W_data, W_bkg] (sumsSize() doubles), ready
    // to be summed over shards; then loss and gradient from summed sums.
    int sumsSize() const { return 3 * (2 + 2 * model_.nAmp() + model_.nTheta()) + 4; }
    void shardSums(const double* d_params, int precision, double* d_sums, cudaStream_t stream);
    void finalizeSums(const double* d_params, const double* d_sums, double* d_nll, double* d_grad, cudaStream_t stream);
    // Hessian [nP][nP] (row-major, symmetric) of the FP64 NLL at d_params:
    // central differences of the exact device gradient, step
    // h_i = rel_step * max(|p_i|, 1e-2), 2 nP gradient evaluations queued on
    // the stream with no host synchronisation.
    void hessian(const double* d_params, double* d_hess, double rel_step, cudaStream_t stream);
    // Exact FP64 Hessian-vector products, forward mode over the adjoint pass:
    // for directions u_d (device [ndir][nP], parameter layout) the rows H u_d
    // (device [ndir][nP]). Every evaluation recomputes the lineshapes and
    // amplitudes in dual numbers; no per-parameter table is stored. The
    // kernels are compiled on the first call.
    void hessianVectorProducts(const double* d_params, const double* d_dirs, int ndir, double* d_out,
                               cudaStream_t stream);
    // The full Hessian from the nP unit directions, symmetrised.
    void hessianExact(const double* d_params, double* d_hess, cudaStream_t stream);
    // Event-sharded form: this handle's per-sample tangent sums
    // [ndir][3][nacc] (ready to be summed over shards like shardSums), and the
    // rows H u_d from summed value sums (shardSums, FP64) and tangent sums.
    void hvpSums(const double* d_params, const double* d_dirs, int ndir, double* d_tsums, cudaStream_t stream);
    void finalizeHvp(const double* d_params, const double* d_dirs, int ndir, const double* d_vsums,
                     const double* d_tsums, double* d_out, cudaStream_t stream);
    int hvpSumsSize(int ndir) const { return ndir * 3 * (2 + 2 * model_.nAmp() + model_.nTheta()); }
    // Partial-wave integrals sum_e w_e sum_p |sum_{a in block i} v_a A_{a,p}|^2
    // per resonance block i over sample `kind` (0 phase space, 1 data,
    // 2 background, 3 phase-space truth from the config's Data.phsp_truth,
    // loaded on first use); d_out: device [nBlocks()]. Fit fractions are
    // ratios of these (FP64).
    int nBlocks() const { return (int)model_.blocks.size(); }
    void partialIntegrals(const double* d_params, int kind, double* d_out, cudaStream_t stream);
    // Result export over the phase-space sample (FP64): per event the total
    // intensity (of the masked blocks, all when mask is empty), per block the
    // partial intensities [nBlocks()][ld], optionally the per-event block
    // interferences [npair][ld] (i < j pairs), and the summed interference
    // matrix (packed i <= j, nBlocks()(nBlocks()+1)/2) into d_interf.
    void exportWeights(const double* d_params, const std::vector<int>& mask, double* d_total, double* d_partial,
                       double* d_interf_ev, double* d_interf, cudaStream_t stream);
    long long tableStride(int kind) const { return samples_[kind].ld; }
    // Per-event intensities of sample `kind` at d_params (device output [n]).
    void intensity(const double* d_params, int kind, double* d_out, cudaStream_t stream);
    // Per-sample partial sums of the last evaluation (diagnostics):
    // [data_nll, bkg_nll, phsp_sum, W_data, W_bkg, n_phsp]
    void lastParts(double* out6, cudaStream_t stream);

    // Optional per-launch timing of the fused kernel: CUDA events recorded on
    // the launching stream around each fused launch into a ring of `slots`
    // pairs (0 switches timing off). kernelTimes synchronises on the recorded
    // events and returns the durations (ms) of the most recent launches.
    void setKernelTiming(int slots);
    int kernelTimes(float* ms, int cap);

    long long nEvents(int kind) const { return samples_[kind].n; }
    size_t deviceBytes() const { return device_bytes_; }
    const GeneratedModel& generated() const { return gen_; }
    const FusedShape& shape() const { return shape_; }
    int fusedGrid(int precision) const { return lay_[precision == kMixed ? 1 : 0].grid; }
    bool polPaired(int precision) const { return paired_[precision == kMixed ? 1 : 0]; }
    double jitSeconds() const { return jit_seconds_; }
    const std::vector<std::pair<std::string, double>>& setupTimes() const { return setup_ms_; }
    bool jitCacheHit() const { return jit_cache_hit_; }

private:
    void loadSamples();
    void buildTables();
    void computeAngular(int kind);
    void buildEventCache(int kind);
    void pairPolarisations();
    void eventMajorMixedAngular();
    // SL_{npol-1-q} = conj(SL_q) on every event of every sample: the fused
    // kernels' tables keep the first (npol + 1) / 2 polarisations
    bool paired_[2] = {false, false};  // plain, mixed fused kernels use the paired tables
    void* k_pc_[2] = {nullptr, nullptr};  // ct_fused_f64_pc, ct_fused_mixed_pc
    void compileKernel();
    void compileHvp();

    Model model_;
    EngineOptions opt_;
    GeneratedModel gen_;
    DeviceSample samples_[4];  // phsp, data, bkg, phase-space truth (loaded on first use)
    bool truth_loaded_ = false;
    void loadTruth();
    bool has_bkg_ = false;
    size_t device_bytes_ = 0;

    // angular tables (device)
    void* d_ag_tables_ = nullptr;  // single allocation holding all host-built tables
    std::vector<char> ag_host_;     // host image of group descriptors
    struct GroupDev;
    std::vector<std::vector<char>> group_desc_;  // AgGroup images per group

    // JIT
    void* lib_ = nullptr;  // cudaLibrary_t
    void* k_f64_ = nullptr;
    void* k_mixed_ = nullptr;
    void* k_int_ = nullptr;
    void* k_part_ = nullptr;
    void* k_exp_ = nullptr;
    int* d_mask_ = nullptr;  // [nBlocks] export wave mask
    void* k_pro_ = nullptr;
    void* k_multi_[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [plain, mixed][paired]
    void* k_pro_multi_ = nullptr;
    const void* image_key_ = nullptr;
    // tensor-core Gram (compiled on the first request)
    void compileGram();
    void compileGramHess();
    void* gram_hess_lib_ = nullptr;
    void* k_gramh_ = nullptr;
    void* k_gramh_fin_ = nullptr;
    int gramh_grid_ = 0;
    int gramh_dsmem_ = 0;
    double* d_ghpart_ = nullptr;
    double* d_ghout_ = nullptr;
    void* gram_lib_ = nullptr;
    void* k_gram_ = nullptr;
    void* k_gram_fin_ = nullptr;
    int gram_grid_ = 0;
    int gram_dsmem_ = 0;
    int gram_resident_ = 0;  // CTAs per SM from the occupancy query
    double* d_gpart_ = nullptr;
    // normalisation cache (compiled and allocated on the first build)
    void compileNorm();
    void* norm_lib_ = nullptr;
    void* k_norm_build_ = nullptr;
    void* k_norm_red_ = nullptr;
    void* k_norm_row_ = nullptr;
    int norm_grid_ = 0;
    int norm_dsmem_ = 0;
    int norm_rows_ = 0;                 // rows of Mu, D (and Mw for a weighted sample), each of nterm entries
    int norm_ne_ = 0;                   // complex entries: norm_rows_ x nterm
    double* d_npart_ = nullptr;         // [norm_grid_][norm_ne_][2]
    double* d_nmat_ = nullptr;          // [norm_ne_][2]
    double* d_ntheta_ = nullptr;        // [nT] resonance parameters of the matrices
    double* d_nrow_ = nullptr;          // [nacc] phase-space row of one cached evaluation
    std::vector<double> norm_theta_;    // host copy of d_ntheta_
    bool norm_valid_ = false;
    void* k_evc_ = nullptr;  // ct_event_cache
    std::vector<std::pair<std::string, double>> setup_ms_;  // set-up phases (host ms)
    // generated angular kernels, one per angular group (empty: the
    // interpreter ag_group_kernel runs instead); their module is shared
    // process-wide
    std::vector<void*> k_ang_;
    // polarisation-pairing maxima accumulated by the generated angular
    // kernels over the three samples (layout of ct_pair_check_kernel's output)
    unsigned long long* d_pairmax_ = nullptr;
    double jit_seconds_ = 0.0;
    bool jit_cache_hit_ = false;

    // evaluation buffers
    double* d_v_ = nullptr;         // [2 nA]
    double* d_consts_ = nullptr;    // [nconst] parameter-only subexpressions
    void* d_kblock_ = nullptr;      // constant-bank image of the last call (CtConsts)
    void* k_sym_ = nullptr;         // address of the fused kernels' constant-bank block (ct_k)
    size_t k_sym_bytes_ = 0;
    double* d_partials_ = nullptr;  // [grid][nacc]
    double* d_parts_ = nullptr;     // [8]
    double* d_hscratch_ = nullptr;  // finite-difference Hessian: perturbed params, two gradients, nll [3 nP + 1]
    int* d_err_ = nullptr;          // set by a fused kernel whose staged copy did not arrive
    // the precision of the last shardSums: finalizeSums applies the mixed
    // form's first-order coupling term to sums of the mixed form
    bool sums_mixed_ = false;
    int* d_amp_chain_ = nullptr;
    double* d_ratio_ = nullptr;
    int* d_gauss_idx_ = nullptr;
    double* d_gauss_ms_ = nullptr;  // [mu, sigma] pairs
    struct CtaLayout {
        int cta[3][2] = {};  // per sample: begin, count
        int grid = 0;
    };
    CtaLayout lay_[2];   // fused-kernel grid of the plain [0] and mixed [1] forms
    CtaLayout lay_data_[2];  // the same over the data and background samples only (cached normalisation)
    int grid_max_ = 0;   // rows of the partials table
    FusedShape shape_;
    int residentCtas(void* kernel, int block, int dsmem) const;
    void layoutCtas(int target, long long tot, int block, CtaLayout& lay, bool no_phsp = false) const;

    // Hessian-vector products (compiled and allocated on first use)
    void* hvp_lib_ = nullptr;  // cudaLibrary_t
    void* k_hvp_pro_ = nullptr;
    void* k_hvp_ = nullptr;
    int hvp_block_ = 128;
    int hvp_dsmem_ = 0;
    int hvp_cap_ = 0;            // directions per launch
    CtaLayout hlay_;             // CTAs of one direction over the samples
    double* d_hdirs_ = nullptr;  // [nP][nP] unit directions
    double* d_hconsts_ = nullptr;  // [cap][nconst][2]
    double* d_hrows_ = nullptr;    // [cap][ctas][nacc]
    double* d_hvsums_ = nullptr;   // value sums
    double* d_htsums_ = nullptr;   // [cap][3][nacc] tangent sums

    cudaStream_t init_stream_ = nullptr;  // initialisation only

    // Device memory of the handle: stream-ordered allocations from a
    // per-device pool of this library that keeps freed memory for the next
    // handle (no device-wide synchronisation, no page mapping on reuse).
    // Frees do not wait for work on other streams: the caller's work on a
    // handle must be complete before it is destroyed.
    cudaStream_t mem_stream_ = nullptr;
    void* devAlloc(size_t bytes);
    void devFree(void* p);
    template <typename T>
    void alloc(T*& p, size_t bytes)
    {
        p = static_cast<T*>(devAlloc(bytes));
    }

    // fused-kernel timing ring
    std::vector<cudaEvent_t> ev_begin_, ev_end_;
    long long ev_count_ = 0;
};

}  // namespace ctpwa
