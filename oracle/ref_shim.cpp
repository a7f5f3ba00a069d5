// Builds the reference's own per-event math as host C++ so tests can pin the
// oracle's restatement against it. This file contains no reference code: it
// #includes the reference sources where they lie (REF_ROOT, passed by the
// Makefile) and exposes a few entry points with plain C types.
//   pwa_amp            src/Amplitude.cu:500-644
//   Bf / BWR / Flatte  include/ResModel.cuh:184-223, 419-451
//   compileCustomExpr + evalCustomAll   src/CustomExpr.cu:1223-1306
//   buildModelAST (builtin models, per-call path)   src/ResModel.cu:376-588
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
using std::max;
using std::min;
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __shfl_down_sync(m, v, o, w) (v)
#define REF_STR2(x) #x
#define REF_STR(x) REF_STR2(x)
#include REF_STR(REF_ROOT/src/Amplitude.cu)
#include REF_STR(REF_ROOT/include/ResModel.cuh)
#include REF_STR(REF_ROOT/src/CustomExpr.cu)
#include REF_STR(REF_ROOT/src/ResModel.cu)

extern "C" {

void ref_pwa_amp(const double* p1, int dj1, const double* p2, int dj2, int dj, int S, int L, double* out)
{
    std::vector<thrust::complex<double>> amp(dj * dj1 * dj2);
    std::vector<thrust::complex<double>> buf(4096);
    LorentzVector a(p1[0], p1[1], p1[2], p1[3]), b(p2[0], p2[1], p2[2], p2[3]);
    pwa_amp(amp.data(), a, dj1, b, dj2, dj, S, L, buf.data());
    for (size_t i = 0; i < amp.size(); ++i) {
        out[2 * i] = amp[i].real();
        out[2 * i + 1] = amp[i].imag();
    }
}

double ref_clebsch(int dj1, int m1, int dj2, int m2, int dJ, int M) { return ClebschGordan(dj1, m1, dj2, m2, dJ, M); }

double ref_bf(int L, double q, double q0, double d) { return Bf<double>(L, q, q0, d); }

void ref_bwr(double m, double m0, double g0, int L, double q, double q0, double d, double* out)
{
    auto z = BWR<double>(m, m0, g0, L, q, q0, d);
    out[0] = z.real();
    out[1] = z.imag();
}

void ref_flatte(double m, double m0, int n, const double* g, const double* ch, double* out)
{
    auto z = Flatte<double>(m, m0, n, g, ch);
    out[0] = z.real();
    out[1] = z.imag();
}

static int evalAux(const std::vector<double>& aux, const double* params, int P, double m, double q, double q0, int L,
                   double d, double md1, double md2, const double* pk, double* out)
{
    double Fr, Fi, dFr[16], dFi[16], d2r[256], d2i[256];
    evalCustomAll(aux.data(), 0, m, q, q0, L, d, md1, md2, pk[0], pk[1], pk[2], pk[3], pk[4], pk[5], pk[6], pk[7], params,
                  P, Fr, Fi, dFr, dFi, d2r, d2i, true);
    out[0] = Fr;
    out[1] = Fi;
    for (int j = 0; j < P; ++j) {
        out[2 + 2 * j] = dFr[j];
        out[3 + 2 * j] = dFi[j];
    }
    for (int j = 0; j < P * P; ++j) {
        out[2 + 2 * P + 2 * j] = d2r[j];
        out[3 + 2 * P + 2 * j] = d2i[j];
    }
    return 0;
}

// Custom DSL: out = [F, dF_0..P-1, d2F (P*P)] as (re, im) pairs; returns -1 on a parse error.
int ref_custom_eval(const char* expr, const char* pnames_csv, const double* params, int P, double m, double q,
                    double q0, int L, double d, double md1, double md2, const double* pk, double* out)
{
    std::vector<std::string> names;
    std::string s(pnames_csv);
    size_t pos = 0;
    while (!s.empty() && pos <= s.size()) {
        size_t c = s.find(',', pos);
        names.push_back(s.substr(pos, c == std::string::npos ? std::string::npos : c - pos));
        if (c == std::string::npos) break;
        pos = c + 1;
    }
    try {
        std::vector<double> aux = compileCustomExpr(expr, names);
        return evalAux(aux, params, P, m, q, q0, L, d, md1, md2, pk, out);
    } catch (...) {
        return -1;
    }
}

// Builtin model (type id as ResModelType) through the symbolic per-call path.
// mdep: Q0MassDep for the two daughters; mfix: their fixed masses.
int ref_model_eval(int type, int L_blk, int Lmin, double d, int P, int n_ch, const double* ch, const int* mdep,
                   const double* mfix, int has_bf, const double* params, double m, double q, int L, double bf_d,
                   double md1, double md2, double* out)
{
    std::vector<double> chm(ch, ch + 2 * n_ch);
    std::vector<double> aux = buildModelAST((ResModelType)type, L_blk, Lmin, d, P, n_ch, chm, (Q0MassDep)mdep[0],
                                            mfix[0], (Q0MassDep)mdep[1], mfix[1], has_bf != 0);
    double pk[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    return evalAux(aux, params, P, m, q, 0.0, L, bf_d, md1, md2, pk, out);
}


// Compile once, evaluate many times (the symbolic second-derivative compile
// of the reference is slow). Returns an opaque handle or nullptr.
void* ref_model_build(int type, int L_blk, int Lmin, double d, int P, int n_ch, const double* ch, const int* mdep,
                      const double* mfix, int has_bf)
{
    std::vector<double> chm(ch, ch + 2 * n_ch);
    return new std::vector<double>(buildModelAST((ResModelType)type, L_blk, Lmin, d, P, n_ch, chm, (Q0MassDep)mdep[0],
                                                 mfix[0], (Q0MassDep)mdep[1], mfix[1], has_bf != 0));
}

void* ref_custom_build(const char* expr, const char* pnames_csv)
{
    std::vector<std::string> names;
    std::string s(pnames_csv);
    size_t pos = 0;
    while (!s.empty() && pos <= s.size()) {
        size_t c = s.find(',', pos);
        names.push_back(s.substr(pos, c == std::string::npos ? std::string::npos : c - pos));
        if (c == std::string::npos) break;
        pos = c + 1;
    }
    try {
        return new std::vector<double>(compileCustomExpr(expr, names));
    } catch (...) {
        return nullptr;
    }
}

int ref_aux_eval(void* h, const double* params, int P, double m, double q, int L, double d, double md1, double md2,
                 const double* pk, double* out)
{
    return evalAux(*static_cast<std::vector<double>*>(h), params, P, m, q, 0.0, L, d, md1, md2, pk, out);
}

void ref_aux_free(void* h) { delete static_cast<std::vector<double>*>(h); }

}  // extern "C"
