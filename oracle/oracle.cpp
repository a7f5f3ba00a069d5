// ORACLE — test infrastructure, not product code.
//
// A plain FP64 CPU (OpenMP) restatement of the reference likelihood path,
// used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg. The product (ctpwa_b200) never links or calls it.
//
// It takes the lowered model from the product's host layer (config.cpp,
// model.cpp, dataio.cpp; pinned separately by tests/test_config_model.py) and
// restates the per-event numerics:
//   angular tensors and chain contraction  src/AmpGen.cu:1034-1219 (+ Amplitude.cu)
//   lineshape assembly, per-call blocks    src/AmpGen.cu:1593-1932 (computeCustomAmpsKernelT)
//   lineshape assembly, fixed blocks       src/AmpGen.cu:1396-1585 (computeAmpsKernelT)
//   per-event NLL terms and weights        src/ComputeNLL.cu:21-84, 312-407
//   phase-space mean                       src/ComputeNLL.cu:244-307, src/Analysis.cu:826-840
//   loss / gradient assembly               src/Analysis.cu:1134-1183
//   resonance-parameter gradient           src/AmpGen.cu:2762-2822, src/Analysis.cu:996-1108
//   coupling-gradient transform            src/AmpGen.cu:3581-3637
// Derivatives with respect to resonance parameters use dual numbers.
#include "../ctpwa_b200/csrc/dataio.hpp"
#include "../ctpwa_b200/csrc/model.hpp"
#include "oracle_angular.hpp"
#include "oracle_lineshape.hpp"

#include <omp.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace oracle;
using ctpwa::Block;
using ctpwa::Group;
using ctpwa::MassSource;
using ctpwa::Model;
using ctpwa::ModelNode;
using ctpwa::ModelType;
using ctpwa::ResInstance;

namespace {

struct OSample {
    ctpwa::Sample s;
    std::vector<std::vector<cplx>> slamp;  // [group][ev][sl][pol]
    std::vector<std::vector<LV>> mom;      // [group][ev * np + particle]
};

struct Oracle {
    Model m;
    OSample smp[3];  // phsp, data, bkg
    bool has_bkg = false;
    double W_data = 0, W_bkg = 0;
    std::vector<std::vector<ExprP>> expr;  // [block][res] custom expressions
    std::string err;
};

// Momenta of every particle of a group for one event (src/AmpGen.cu:514-640;
// the initial state is the running sum of the finals, src/Analysis.cu:146-156).
void groupMomenta(const Group& g, const double* p4, int nfin, std::vector<LV>& out)
{
    out.assign(g.particle_names.size(), LV());
    LV parent(0, 0, 0, 0);
    for (int f = 0; f < nfin; ++f) parent = parent + LV(p4[4 * f], p4[4 * f + 1], p4[4 * f + 2], p4[4 * f + 3]);
    for (int idx : g.build_order) {
        int s = g.input_slot[idx];
        if (s >= 0) out[idx] = LV(p4[4 * s], p4[4 * s + 1], p4[4 * s + 2], p4[4 * s + 3]);
        else if (s == -1) out[idx] = parent;
        else out[idx] = out[g.sum_of[idx].first] + out[g.sum_of[idx].second];
    }
}

// Contracted SL-amplitude tensor for every SL combination of a group.
void groupSlamp(const Model& m, const Group& g, const std::vector<LV>& p, cplx* out /*[nSL][npol]*/)
{
    for (int s = 0; s < g.nSL(); ++s) {
        std::vector<cplx> cur, node;
        std::vector<int> shape, labels;
        for (size_t ni = 0; ni < g.nodes.size(); ++ni) {
            const ModelNode& n = g.nodes[ni];
            const ctpwa::SLPair& sl = n.sls[g.sl_combs[s][ni]];
            pwaAmp(node, p[n.d1], n.dj1, p[n.d2], n.dj2, n.dj, sl.S, sl.L);
            if (ni == 0) {
                cur = node;
                shape = {n.dj, n.dj1, n.dj2};
                labels = {n.mother, n.d1, n.d2};
                continue;
            }
            int c = -1;
            for (size_t j = 0; j < labels.size(); ++j)
                if (labels[j] == n.mother) {
                    c = (int)j;
                    break;
                }
            // out[(A dims without c) , dj1, dj2] = sum_sigma cur[.., sigma@c, ..] * node[sigma][e1][e2]
            std::vector<int> oshape;
            for (size_t j = 0; j < shape.size(); ++j)
                if ((int)j != c) oshape.push_back(shape[j]);
            oshape.push_back(n.dj1);
            oshape.push_back(n.dj2);
            int rankA = (int)shape.size();
            std::vector<int> sA(rankA);
            sA[rankA - 1] = 1;
            for (int j = rankA - 2; j >= 0; --j) sA[j] = sA[j + 1] * shape[j + 1];
            int total = 1;
            for (int d : oshape) total *= d;
            std::vector<cplx> o(total);
            int ro = (int)oshape.size();
            for (int idx = 0; idx < total; ++idx) {
                std::vector<int> ic(ro);
                int t = idx;
                for (int j = ro - 1; j >= 0; --j) {
                    ic[j] = t % oshape[j];
                    t /= oshape[j];
                }
                int baseA = 0, pos = 0;
                for (int j = 0; j < rankA; ++j)
                    if (j != c) baseA += ic[pos++] * sA[j];
                int e1 = ic[ro - 2], e2 = ic[ro - 1];
                cplx sum = 0.0;
                for (int sg = 0; sg < shape[c]; ++sg)
                    sum += cur[baseA + sg * sA[c]] * node[(sg * n.dj1 + e1) * n.dj2 + e2];
                o[idx] = sum;
            }
            cur = o;
            shape = oshape;
            labels.erase(labels.begin() + c);
            labels.push_back(n.d1);
            labels.push_back(n.d2);
        }
        for (int i = 0; i < m.npol; ++i) out[s * m.npol + i] = m.pol_map.empty() ? cur[i] : cur[m.pol_map[i]];
    }
}

// Value of resonance parameter p of block resonance r for theta vector th,
// seeded as a dual variable when it is a fitted parameter.
struct BlockParams {
    std::vector<std::vector<D>> par;    // [res][param]
    std::vector<int> local_to_theta;    // local dual slot -> global theta index
};

BlockParams blockParams(const Block& b, const double* theta)
{
    BlockParams bp;
    bp.par.resize(b.res.size());
    for (size_t r = 0; r < b.res.size(); ++r) {
        const ResInstance& R = b.res[r];
        for (size_t p = 0; p < R.params.size(); ++p) {
            int t = R.theta[p];
            if (t >= 0 && theta) {
                int k = (int)bp.local_to_theta.size();
                if (k >= NDUAL) throw std::runtime_error("oracle: too many fitted parameters in one block");
                bp.local_to_theta.push_back(t);
                bp.par[r].push_back(D::var(theta[t], k));
            } else {
                bp.par[r].push_back(D(R.params[p]));
            }
        }
    }
    return bp;
}

D massDep(MassSource src, double fixed, const D& m0, const D& runtime)
{
    if (src == MassSource::Fixed) return D(fixed);
    if (src == MassSource::M0Param) return m0;
    return runtime;
}

// Per-call ("free") lineshape of one resonance on its decay node
// (buildModelAST semantics, src/ResModel.cu:376-588; custom: compileCustomExpr).
CD resonanceFactor(const ResInstance& R, const std::vector<D>& par, const ExprP& ex, const D& mm, const D& qq, int L,
                   double bf_d, const D& md1q, const D& md2q, const LV& pD1, const LV& pD2)
{
    int P = (int)par.size();
    D m0 = P > 0 ? par[0] : D(1.0);
    D q0r = q0AD(m0, massDep(R.md_src[0], R.md_fixed[0], m0, md1q), massDep(R.md_src[1], R.md_fixed[1], m0, md2q));
    switch (R.type) {
    case ModelType::BWR: {
        CD bw = BWR(mm, par[0], par[1], R.Lmin, qq, q0r, R.has_bf ? R.d : 0.0);
        if (R.has_bf) {
            D bf = Bf(L, qq, q0r, R.d);
            return CD(bw.re * bf, bw.im * bf);
        }
        return bw;
    }
    case ModelType::BW: return BW(mm, par[0], par[1]);
    case ModelType::ONE: return R.has_bf ? CD(Bf(L, qq, q0r, R.d)) : CD(D(1.0));
    case ModelType::Flatte: {
        std::vector<D> g(par.begin() + 1, par.end());
        std::vector<double> ch;
        for (const auto& c : R.channels) {
            ch.push_back(c.first);
            ch.push_back(c.second);
        }
        g.resize(R.channels.size(), D(0.0));
        CD f = flatte(mm, par[0], g, ch);
        if (R.has_bf) {
            D bf = Bf(L, qq, q0r, R.d);
            return CD(f.re * bf, f.im * bf);
        }
        return f;
    }
    case ModelType::GS: {
        double mpi = R.channels.empty() ? 0.1396 : R.channels[0].first;
        CD f = gs(mm, qq, par[0], par[1], q0r, mpi);
        if (R.has_bf) {
            D bf = Bf(L, qq, q0r, R.d);
            return CD(f.re * bf, f.im * bf);
        }
        return f;
    }
    case ModelType::Custom: {
        EvalVars v;
        v.v[V_M] = mm;
        v.v[V_Q] = qq;
        v.v[V_Q0] = D(0.0);
        v.L = L;
        v.v[V_D] = D(bf_d);
        v.v[V_MD1] = md1q;
        v.v[V_MD2] = md2q;
        double p1P = pD1.P(), p2P = pD2.P();
        v.v[V_P1P] = D(p1P);
        v.v[V_P1E] = D(pD1.E);
        v.v[V_P1CT] = D(p1P > 0 ? pD1.Pz / p1P : 0.0);
        v.v[V_P1PHI] = D(std::atan2(pD1.Py, pD1.Px));
        v.v[V_P2P] = D(p2P);
        v.v[V_P2E] = D(pD2.E);
        v.v[V_P2CT] = D(p2P > 0 ? pD2.Pz / p2P : 0.0);
        v.v[V_P2PHI] = D(std::atan2(pD2.Py, pD2.Px));
        return evalExpr(*ex, v, par);
    }
    case ModelType::Interp: {
        double fr, fi;
        interpLookup(R.aux, mm.v, fr, fi);
        return CD(D(fr), D(fi));
    }
    case ModelType::Hist: return CD(D(histLookup(mm.v, R.aux)));
    }
    return CD(D(1.0));
}

// Fixed-parameter node factor (computeNodeFactor, include/ResModel.cuh:103-181).
CD fixedNodeFactor(const ResInstance& R, const std::vector<D>& par, const ExprP& ex, int L, int Lmin, double mm,
                   double qq, double q0, double bf_d, bool has_bf)
{
    D M(mm), Q(qq), Q0(q0);
    switch (R.type) {
    case ModelType::BWR: {
        CD bw = BWR(M, par[0], par[1], Lmin, Q, Q0, has_bf ? bf_d : 0.0);
        if (has_bf) {
            D bf = Bf(L, Q, Q0, bf_d);
            return CD(bw.re * bf, bw.im * bf);
        }
        return bw;
    }
    case ModelType::BW: return BW(M, par[0], par[1]);
    case ModelType::ONE: return has_bf ? CD(Bf(L, Q, Q0, bf_d)) : CD(D(1.0));
    case ModelType::Flatte: {
        // ResModel.cuh Flatte<T>: D = m0^2 - s - i m0/2 sum g_i rho_i
        std::vector<D> g(par.begin() + 1, par.end());
        g.resize(R.channels.size(), D(0.0));
        D s = M * M, tr(0.0), ti(0.0);
        for (size_t i = 0; i < R.channels.size(); ++i) {
            double rr, ri;
            flatteRho(s.v, R.channels[i].first, R.channels[i].second, rr, ri);
            D gw = (par[0] / D(2.0)) * g[i];
            tr = tr + gw * D(rr);
            ti = ti + gw * D(ri);
        }
        D dre = par[0] * par[0] - s + ti, dim = D(0.0) - tr;
        D dsq = dre * dre + dim * dim;
        CD f(dre / dsq, (D(0.0) - dim) / dsq);
        if (has_bf) {
            D bf = Bf(L, Q, Q0, bf_d);
            return CD(f.re * bf, f.im * bf);
        }
        return f;
    }
    case ModelType::Hist: return CD(D(histLookup(mm, R.aux)));
    case ModelType::Custom: {
        // segment 0 with md1 = md2 = 0 and no daughter kinematics, at most 3 params
        EvalVars v;
        v.v[V_M] = M;
        v.v[V_Q] = Q;
        v.v[V_Q0] = Q0;
        v.L = L;
        v.v[V_D] = D(bf_d);
        std::vector<D> p3(par.begin(), par.begin() + std::min<size_t>(3, par.size()));
        return evalExpr(*ex, v, p3);
    }
    default: return CD(D(1.0));  // GS / Interp have no fixed-parameter branch
    }
}

double breakupRaw(double m, double m1, double m2)  // no clamp (src/AmpGen.cu:1486-1500)
{
    return std::sqrt((m * m - std::pow(m1 + m2, 2)) * (m * m - std::pow(m1 - m2, 2))) / 2 / m;
}

// Lineshape product F_s (complex dual) for SL combination s of block b.
CD blockFactor(const Model& m, const Block& b, const BlockParams& bp, const std::vector<ExprP>& ex, int s,
               const std::vector<LV>& p)
{
    const Group& g = m.groups[b.group];
    CD F(D(1.0));
    if (b.free_path) {
        for (size_t ni = 0; ni < g.nodes.size(); ++ni) {
            const ModelNode& n = g.nodes[ni];
            int L = n.sls[g.sl_combs[s][ni]].L;
            const LV &pM = p[n.mother], &p1 = p[n.d1], &p2 = p[n.d2];
            double mm = pM.M(), md1 = p1.M(), md2 = p2.M();
            D qq = breakup(D(mm), D(md1), D(md2));
            int match = -1;
            for (size_t r = 0; r < b.res.size(); ++r)
                if (b.res[r].particle_idx == n.mother && n.mass[0] <= 0) {
                    match = (int)r;
                    break;
                }
            D m0q = match >= 0 ? (bp.par[match].empty() ? D(1.0) : bp.par[match][0]) : D(n.mass[0] > 0 ? n.mass[0] : 1.0);
            auto dq = [&](int k, double evm) {
                if (n.mass[k + 1] > 0) return D(n.mass[k + 1]);
                int di = k == 0 ? n.d1 : n.d2;
                for (size_t r = 0; r < b.res.size(); ++r)
                    if (b.res[r].particle_idx == di && !bp.par[r].empty()) return bp.par[r][0];
                return D(evm);
            };
            D md1q = dq(0, md1), md2q = dq(1, md2);
            if (match >= 0) {
                CD f = resonanceFactor(b.res[match], bp.par[match], ex[match], D(mm), qq, L, n.bf_d, md1q, md2q, p1, p2);
                F = F * f;
            } else if (n.has_bf) {
                D q0 = breakup(m0q, md1q, md2q);
                D bf = Bf(L, qq, q0, n.bf_d);
                F = CD(F.re * bf, F.im * bf);
            }
        }
        return F;
    }
    // fixed-parameter block (computeAmpsKernelT)
    for (size_t ni = 0; ni < g.nodes.size(); ++ni) {
        const ModelNode& n = g.nodes[ni];
        int L = n.sls[g.sl_combs[s][ni]].L;
        const LV &pM = p[n.mother], &p1 = p[n.d1], &p2 = p[n.d2];
        double mm = pM.M();
        double qq = breakupRaw(mm, p1.M(), p2.M());
        int match = -1;
        for (size_t r = 0; r < b.res.size(); ++r)
            if (b.res[r].particle_idx == n.mother) {
                match = (int)r;
                break;
            }
        double mo = n.mass[0], ma = n.mass[1], mb = n.mass[2];
        if (mo == -1 && match >= 0) mo = b.res[match].params.empty() ? 1.0 : b.res[match].params[0];
        auto sub = [&](double ms, int di) {
            if (ms != -1) return ms;
            for (const auto& r : b.res)
                if (r.particle_idx == di) return r.params.empty() ? 1.0 : r.params[0];
            return ms;
        };
        ma = sub(ma, n.d1);
        mb = sub(mb, n.d2);
        double q0 = breakupRaw(mo, ma, mb);
        if (ni == 0) {
            if (n.has_bf) {
                D bf = Bf(L, D(qq), D(q0), n.bf_d);
                F = CD(F.re * bf, F.im * bf);
            }
            continue;
        }
        if (match >= 0) F = F * fixedNodeFactor(b.res[match], bp.par[match], ex[match], L, n.l_min, mm, qq, q0, n.bf_d, n.has_bf);
    }
    return F;
}

struct Accum {
    double nll = 0;       // sum -w log f
    double fsum = 0;      // phsp: sum f
    std::vector<cplx> gv;       // data/bkg: sum -conj(A) u   | phsp: sum (w/W) conj(A) S
    std::vector<double> gt;     // data/bkg: sum -2Re(conj(u) dS) | phsp: sum 2Re(conj(S) dS)
};

// Per-event evaluation over one sample; kind 0 = phsp, 1 = data, 2 = bkg.
void evalSample(const Oracle& o, int kind, const std::vector<cplx>& v, const double* theta, double W_phsp, Accum& acc,
                int nthreads)
{
    const Model& m = o.m;
    const OSample& S = o.smp[kind];
    int nA = m.nAmp(), nT = m.nTheta(), npol = m.npol;
    long n = S.s.n;
    std::vector<BlockParams> bps;
    for (const auto& b : m.blocks) bps.push_back(blockParams(b, theta));
    int nth = nthreads > 0 ? nthreads : omp_get_max_threads();
    std::vector<Accum> part(nth);
    for (auto& a : part) {
        a.gv.assign(nA, 0.0);
        a.gt.assign(nT, 0.0);
    }
#pragma omp parallel num_threads(nth)
    {
        Accum& a = part[omp_get_thread_num()];
        std::vector<cplx> A(npol * nA);
        std::vector<cplx> dS(npol * nT);
#pragma omp for schedule(static)
        for (long e = 0; e < n; ++e) {
            std::fill(A.begin(), A.end(), cplx(0.0));
            std::fill(dS.begin(), dS.end(), cplx(0.0));
            for (size_t bi = 0; bi < m.blocks.size(); ++bi) {
                const Block& b = m.blocks[bi];
                const Group& g = m.groups[b.group];
                // base group and its identical-particle permutations (src/AmpGen.cu:194-405)
                std::vector<int> vars = {b.group};
                for (int vg : g.variants) vars.push_back(vg);
                for (int gv : vars) {
                    const LV* pm = &S.mom[gv][(size_t)e * g.particle_names.size()];
                    std::vector<LV> pv(pm, pm + g.particle_names.size());
                    const cplx* sl = &S.slamp[gv][(size_t)e * g.nSL() * npol];
                    const double sign = m.groups[gv].sign;
                    for (int s = 0; s < g.nSL(); ++s) {
                        CD F = blockFactor(m, b, bps[bi], o.expr[bi], s, pv);
                        int a_idx = b.site + s;
                        cplx Fv(sign * F.re.v, sign * F.im.v);
                        for (int pp = 0; pp < npol; ++pp) {
                            cplx amp = Fv * sl[s * npol + pp];
                            A[pp * nA + a_idx] += amp;
                            for (size_t k = 0; k < bps[bi].local_to_theta.size(); ++k) {
                                cplx dF(sign * F.re.g[k], sign * F.im.g[k]);
                                dS[pp * nT + bps[bi].local_to_theta[k]] += v[a_idx] * dF * sl[s * npol + pp];
                            }
                        }
                    }
                }
            }
            std::vector<cplx> Sv(npol, 0.0);
            double f = 0.0;
            for (int pp = 0; pp < npol; ++pp) {
                cplx s = 0.0;
                for (int a2 = 0; a2 < nA; ++a2) s += A[pp * nA + a2] * v[a2];
                Sv[pp] = s;
                f += s.real() * s.real() + s.imag() * s.imag();
            }
            if (kind == 0) {
                double we = S.s.weights.empty() ? 1.0 : S.s.weights[e];
                a.fsum += f;
                for (int a2 = 0; a2 < nA; ++a2) {
                    cplx t = 0.0;
                    for (int pp = 0; pp < npol; ++pp) t += std::conj(A[pp * nA + a2]) * Sv[pp];
                    a.gv[a2] += (we / W_phsp) * t;
                }
                for (int j = 0; j < nT; ++j) {
                    double t = 0.0;
                    for (int pp = 0; pp < npol; ++pp) t += 2.0 * (std::conj(Sv[pp]) * dS[pp * nT + j]).real();
                    a.gt[j] += t;
                }
            } else {
                double w = S.s.weights.empty() ? 1.0 : S.s.weights[e];
                if (f == 0.0) {
                    a.nll += -std::log(1e-10) * w;
                    continue;
                }
                a.nll += -std::log(f) * w;
                std::vector<cplx> u(npol);
                for (int pp = 0; pp < npol; ++pp) {
                    double ur = Sv[pp].real() * (w / f), ui = Sv[pp].imag() * (w / f);
                    ur = std::fmin(std::fmax(ur, -1e10), 1e10);
                    ui = std::fmin(std::fmax(ui, -1e10), 1e10);
                    u[pp] = cplx(ur, ui);
                }
                for (int a2 = 0; a2 < nA; ++a2) {
                    cplx t = 0.0;
                    for (int pp = 0; pp < npol; ++pp) t += std::conj(A[pp * nA + a2]) * u[pp];
                    a.gv[a2] -= t;
                }
                for (int j = 0; j < nT; ++j) {
                    double t = 0.0;
                    for (int pp = 0; pp < npol; ++pp) t += (std::conj(u[pp]) * dS[pp * nT + j]).real();
                    a.gt[j] += -2.0 * t;
                }
            }
        }
    }
    acc.gv.assign(nA, 0.0);
    acc.gt.assign(nT, 0.0);
    for (const auto& a : part) {
        acc.nll += a.nll;
        acc.fsum += a.fsum;
        for (int i = 0; i < nA; ++i) acc.gv[i] += a.gv[i];
        for (int j = 0; j < nT; ++j) acc.gt[j] += a.gt[j];
    }
}

int fail(char* err, int len, const std::string& msg)
{
    if (err && len > 0) {
        std::strncpy(err, msg.c_str(), (size_t)len - 1);
        err[len - 1] = 0;
    }
    return -1;
}

}  // namespace

extern "C" {

void* orc_open_shard(const char* config_path, int rank, int world, char* err, int errlen);

void* orc_open(const char* config_path, char* err, int errlen) { return orc_open_shard(config_path, 0, 1, err, errlen); }

// Oracle over event block `rank` of `world` of every sample (the same blocks
// as the engine's shards).
void* orc_open_shard(const char* config_path, int rank, int world, char* err, int errlen)
{
    try {
        auto o = std::make_unique<Oracle>();
        ctpwa::Config cfg = ctpwa::loadConfig(config_path);
        o->m = ctpwa::buildModel(cfg, 1);
        const Model& m = o->m;
        int nfin = (int)m.final_order.size();
        const char* kinds[3] = {"phsp", "data", "bkg"};
        for (int k = 0; k < 3; ++k) {
            auto it = m.cfg.data_files.find(kinds[k]);
            if (it == m.cfg.data_files.end()) {
                if (k < 2) throw std::runtime_error(std::string("config has no Data.") + kinds[k]);
                continue;
            }
            if (k == 2) o->has_bkg = true;
            o->smp[k].s = ctpwa::readSample(it->second, nfin);
        }
        auto wt = [&](const char* key, int k) {
            auto it = m.cfg.data_files.find(key);
            if (it != m.cfg.data_files.end()) o->smp[k].s.weights = ctpwa::readWeights(it->second, o->smp[k].s.n);
        };
        wt("phsp_weights", 0);
        wt("data_weights", 1);
        if (o->has_bkg) wt("bkg_weights", 2);
        for (int k = 0; k < 3; ++k) {
            std::vector<double> none;
            ctpwa::shardSample(o->smp[k].s, none, rank, world);
        }
        for (int k = 0; k < 3; ++k) {
            auto& S = o->smp[k];
            S.slamp.resize(m.groups.size());
            S.mom.resize(m.groups.size());
            for (size_t gi = 0; gi < m.groups.size(); ++gi) {
                const Group& g = m.groups[gi];
                size_t np = g.particle_names.size();
                S.mom[gi].resize((size_t)S.s.n * np);
                S.slamp[gi].resize((size_t)S.s.n * g.nSL() * m.npol);
#pragma omp parallel for schedule(static)
                for (long e = 0; e < S.s.n; ++e) {
                    std::vector<LV> p;
                    groupMomenta(g, &S.s.p4[(size_t)e * nfin * 4], nfin, p);
                    std::copy(p.begin(), p.end(), S.mom[gi].begin() + (size_t)e * np);
                    groupSlamp(m, g, p, &S.slamp[gi][(size_t)e * g.nSL() * m.npol]);
                }
            }
        }
        o->W_data = 0;
        for (long e = 0; e < o->smp[1].s.n; ++e) o->W_data += o->smp[1].s.weights.empty() ? 1.0 : o->smp[1].s.weights[e];
        o->W_bkg = 0;
        for (long e = 0; e < o->smp[2].s.n; ++e) o->W_bkg += o->smp[2].s.weights.empty() ? 1.0 : o->smp[2].s.weights[e];
        o->expr.resize(m.blocks.size());
        for (size_t b = 0; b < m.blocks.size(); ++b) {
            for (const auto& r : m.blocks[b].res) {
                if (r.type == ModelType::Custom) {
                    ExprParser ps(r.options.at("expr"), r.param_names);
                    o->expr[b].push_back(ps.parse());
                } else {
                    o->expr[b].push_back(nullptr);
                }
            }
        }
        return o.release();
    } catch (const std::exception& e) {
        fail(err, errlen, e.what());
        return nullptr;
    }
}

void orc_close(void* h) { delete static_cast<Oracle*>(h); }

// Rebuilds sample k from its events idx[0..n) (repeats allowed), keeping the
// angular tensors already computed: accept-reject selection of a candidate
// sample, or a resample of it, without recomputing its events.
int orc_take(void* h, int k, const long* idx, long n)
{
    auto* o = static_cast<Oracle*>(h);
    try {
        if (k < 0 || k > 2 || n < 0) throw std::runtime_error("orc_take: bad arguments");
        OSample& S = o->smp[k];
        const int nfin = S.s.n_final;
        for (long i = 0; i < n; ++i)
            if (idx[i] < 0 || idx[i] >= S.s.n) throw std::runtime_error("orc_take: index out of range");
        OSample T;
        T.s.n = n;
        T.s.n_final = nfin;
        T.s.p4.resize((size_t)n * nfin * 4);
        if (!S.s.weights.empty()) T.s.weights.resize(n);
        T.slamp.resize(S.slamp.size());
        T.mom.resize(S.mom.size());
        for (size_t gi = 0; gi < S.slamp.size(); ++gi) {
            const size_t ps = S.s.n ? S.slamp[gi].size() / S.s.n : 0, pm = S.s.n ? S.mom[gi].size() / S.s.n : 0;
            T.slamp[gi].resize((size_t)n * ps);
            T.mom[gi].resize((size_t)n * pm);
#pragma omp parallel for schedule(static)
            for (long i = 0; i < n; ++i) {
                std::copy_n(S.slamp[gi].begin() + (size_t)idx[i] * ps, ps, T.slamp[gi].begin() + (size_t)i * ps);
                std::copy_n(S.mom[gi].begin() + (size_t)idx[i] * pm, pm, T.mom[gi].begin() + (size_t)i * pm);
            }
        }
        for (long i = 0; i < n; ++i) {
            std::copy_n(S.s.p4.begin() + (size_t)idx[i] * nfin * 4, nfin * 4, T.s.p4.begin() + (size_t)i * nfin * 4);
            if (!S.s.weights.empty()) T.s.weights[i] = S.s.weights[idx[i]];
        }
        S = std::move(T);
        double W = 0;
        for (long e = 0; e < S.s.n; ++e) W += S.s.weights.empty() ? 1.0 : S.s.weights[e];
        if (k == 1) o->W_data = W;
        if (k == 2) o->W_bkg = W;
        return 0;
    } catch (const std::exception& e) {
        o->err = e.what();
        return -1;
    }
}

// sizes: [nA, nTheta, nVector, npol, nGroups, n_phsp, n_data, n_bkg]
int orc_sizes(void* h, long* out)
{
    auto* o = static_cast<Oracle*>(h);
    out[0] = o->m.nAmp();
    out[1] = o->m.nTheta();
    out[2] = o->m.nVector();
    out[3] = o->m.npol;
    out[4] = (long)o->m.groups.size();
    for (int k = 0; k < 3; ++k) out[5 + k] = o->smp[k].s.n;
    return 0;
}

// Free resonance parameters: out[3][nTheta] = (initial value, lower, upper)
int orc_theta_init(void* h, double* out)
{
    auto* o = static_cast<Oracle*>(h);
    const int nT = o->m.nTheta();
    for (int j = 0; j < nT; ++j) {
        out[j] = o->m.slots[j].init;
        out[nT + j] = o->m.slots[j].lower;
        out[2 * nT + j] = o->m.slots[j].upper;
    }
    return 0;
}

int orc_group_nsl(void* h, int g)
{
    auto* o = static_cast<Oracle*>(h);
    return o->m.groups[g].nSL();
}

// Angular table of group g for sample k: [ev][sl][pol] complex (re, im pairs).
int orc_slamp(void* h, int k, int g, double* out)
{
    auto* o = static_cast<Oracle*>(h);
    const auto& t = o->smp[k].slamp[g];
    std::memcpy(out, t.data(), t.size() * sizeof(cplx));
    return 0;
}

// Amplitude columns A[ev][pol][nA] for sample k at theta (nullptr = templates).
int orc_columns(void* h, int k, const double* theta, double* out)
{
    auto* o = static_cast<Oracle*>(h);
    const Model& m = o->m;
    const OSample& S = o->smp[k];
    int nA = m.nAmp(), npol = m.npol;
    std::vector<BlockParams> bps;
    for (const auto& b : m.blocks) bps.push_back(blockParams(b, theta));
    cplx* A = reinterpret_cast<cplx*>(out);
#pragma omp parallel for schedule(static)
    for (long e = 0; e < S.s.n; ++e) {
        for (size_t bi = 0; bi < m.blocks.size(); ++bi) {
            const Block& b = m.blocks[bi];
            const Group& g = m.groups[b.group];
            for (int s = 0; s < g.nSL(); ++s)
                for (int pp = 0; pp < npol; ++pp) A[((size_t)e * npol + pp) * nA + b.site + s] = 0.0;
            // base group and its identical-particle permutations (src/AmpGen.cu:194-405)
            std::vector<int> vars = {b.group};
            for (int v : g.variants) vars.push_back(v);
            for (int gv : vars) {
                const LV* pm = &S.mom[gv][(size_t)e * g.particle_names.size()];
                std::vector<LV> pv(pm, pm + g.particle_names.size());
                const cplx* sl = &S.slamp[gv][(size_t)e * g.nSL() * npol];
                const double sign = m.groups[gv].sign;
                for (int s = 0; s < g.nSL(); ++s) {
                    CD F = blockFactor(m, b, bps[bi], o->expr[bi], s, pv);
                    for (int pp = 0; pp < npol; ++pp)
                        A[((size_t)e * npol + pp) * nA + b.site + s] += sign * cplx(F.re.v, F.im.v) * sl[s * npol + pp];
                }
            }
        }
    }
    return 0;
}

// NLL and gradient in the reference parameter layout [Re p, Im p, theta].
// parts (optional, 6 doubles): data_nll, bkg_nll, phsp_factor, W_data, W_bkg, n_phsp
namespace {

std::vector<cplx> couplings(const Model& m, const double* params)
{
    int nA = m.nAmp(), nc = m.nVector();
    std::vector<cplx> v(nA);
    for (int a = 0; a < nA; ++a) {
        int c = m.coupling.amp_chain[a];
        v[a] = m.coupling.ratio[a] * cplx(params[c], params[nc + c]);
    }
    return v;
}

// Loss and gradient from the three samples' sums (src/Analysis.cu:1134-1183)
// and the coupling transform (src/AmpGen.cu:3581-3637). ap.gv is already
// divided by the phase-space weight total.
void assemble(const Model& m, const double* params, const std::vector<cplx>& v, const Accum& ap, const Accum& ad,
              const Accum& ab, double Np, double W_data, double W_bkg, double* nll, double* grad, double* parts)
{
    int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta();
    const double* theta = params + 2 * nc;
    double pf = Np > 0 ? ap.fsum / Np : 0.0;
    if (pf <= 1e-30 || std::isnan(pf) || std::isinf(pf)) pf = 1e-30;
    double Weff = W_data - W_bkg;
    double loss = ad.nll - ab.nll + Weff * std::log(pf);
    for (const auto& g : m.gauss) {
        double dlt = theta[g.first] - g.second.first;
        loss += dlt * dlt / (2.0 * g.second.second * g.second.second);
    }
    std::vector<cplx> gv(nA);
    std::vector<double> gt(nT);
    bool reset = std::isnan(loss) || std::isinf(loss);
    if (reset) loss = 1e30;
    for (int a = 0; a < nA; ++a) gv[a] = reset ? 0.0 : ad.gv[a] - ab.gv[a] + (Weff / pf) * ap.gv[a];
    for (int j = 0; j < nT; ++j) gt[j] = reset ? 0.0 : ad.gt[j] - ab.gt[j] + (Weff / (pf * Np)) * ap.gt[j];
    if (!reset)
        for (const auto& g : m.gauss)
            gt[g.first] += (theta[g.first] - g.second.first) / (g.second.second * g.second.second);
    // coupling transform (src/AmpGen.cu:3581-3637): dL = (1/p) sum conj(g_a) v_a
    for (int c = 0; c < nc; ++c) {
        cplx sum = 0.0;
        for (int a = 0; a < nA; ++a)
            if (m.coupling.amp_chain[a] == c) sum += std::conj(gv[a]) * v[a];
        double pr = params[c], pi = params[nc + c];
        double ps = pr * pr + pi * pi;
        if (ps < 1e-30) ps = 1e-30;
        double dr = (sum.real() * pr + sum.imag() * pi) / ps;
        double di = (sum.imag() * pr - sum.real() * pi) / ps;
        grad[c] = 2.0 * dr;
        grad[nc + c] = -2.0 * di;
    }
    for (int j = 0; j < nT; ++j) grad[2 * nc + j] = gt[j];
    *nll = loss;
    if (parts) {
        parts[0] = ad.nll;
        parts[1] = ab.nll;
        parts[2] = pf;
        parts[3] = W_data;
        parts[4] = W_bkg;
        parts[5] = Np;
    }
}

double phspWeight(const Oracle& o)
{
    const auto& ph = o.smp[0].s;
    double Wp = 0;
    if (ph.weights.empty()) Wp = (double)ph.n;
    else
        for (double w : ph.weights) Wp += w;
    return Wp;
}

void evalAll(Oracle& o, const std::vector<cplx>& v, const double* theta, double Wp, Accum& ap, Accum& ad, Accum& ab,
             int nthreads)
{
    int nA = o.m.nAmp(), nT = o.m.nTheta();
    evalSample(o, 0, v, theta, Wp, ap, nthreads);
    evalSample(o, 1, v, theta, Wp, ad, nthreads);
    if (o.has_bkg) evalSample(o, 2, v, theta, Wp, ab, nthreads);
    else {
        ab.gv.assign(nA, 0.0);
        ab.gt.assign(nT, 0.0);
    }
}

}  // namespace

int orc_nll_grad(void* h, const double* params, double* nll, double* grad, double* parts, int nthreads)
{
    auto* o = static_cast<Oracle*>(h);
    try {
        const Model& m = o->m;
        std::vector<cplx> v = couplings(m, params);
        double Wp = phspWeight(*o);
        if (Wp <= 0) Wp = 1.0;
        Accum ap, ad, ab;
        evalAll(*o, v, params + 2 * m.nVector(), Wp, ap, ad, ab, nthreads);
        assemble(m, params, v, ap, ad, ab, (double)o->smp[0].s.n, o->W_data, o->W_bkg, nll, grad, parts);
        return 0;
    } catch (const std::exception& e) {
        o->err = e.what();
        return -1;
    }
}

// Partial sums of this oracle's samples (one shard of an event-sharded
// evaluation), in the device layout: per sample (phase space, data,
// background) [nll, fsum, gv (re, im) x nA, gt x nT], the phase-space gv not
// yet divided by the phase-space weight total; then [n_phsp, W_phsp, W_data,
// W_bkg]. Summing these over shards and calling orc_finalize_sums gives the
// evaluation of the union of the shards.
int orc_shard_sums(void* h, const double* params, double* out, int nthreads)
{
    auto* o = static_cast<Oracle*>(h);
    try {
        const Model& m = o->m;
        int nA = m.nAmp(), nT = m.nTheta(), nacc = 2 + 2 * nA + nT;
        std::vector<cplx> v = couplings(m, params);
        Accum acc[3];
        evalAll(*o, v, params + 2 * m.nVector(), 1.0, acc[0], acc[1], acc[2], nthreads);
        for (int k = 0; k < 3; ++k) {
            double* r = out + k * nacc;
            r[0] = acc[k].nll;
            r[1] = acc[k].fsum;
            for (int a = 0; a < nA; ++a) {
                r[2 + 2 * a] = acc[k].gv[a].real();
                r[3 + 2 * a] = acc[k].gv[a].imag();
            }
            for (int j = 0; j < nT; ++j) r[2 + 2 * nA + j] = acc[k].gt[j];
        }
        out[3 * nacc + 0] = (double)o->smp[0].s.n;
        out[3 * nacc + 1] = phspWeight(*o);
        out[3 * nacc + 2] = o->W_data;
        out[3 * nacc + 3] = o->W_bkg;
        return 0;
    } catch (const std::exception& e) {
        o->err = e.what();
        return -1;
    }
}

// Loss and gradient from summed shard sums (layout of orc_shard_sums).
int orc_finalize_sums(void* h, const double* params, const double* sums, double* nll, double* grad)
{
    auto* o = static_cast<Oracle*>(h);
    try {
        const Model& m = o->m;
        int nA = m.nAmp(), nT = m.nTheta(), nacc = 2 + 2 * nA + nT;
        std::vector<cplx> v = couplings(m, params);
        Accum acc[3];
        double Wp = sums[3 * nacc + 1];
        if (Wp <= 0) Wp = 1.0;
        for (int k = 0; k < 3; ++k) {
            const double* r = sums + k * nacc;
            acc[k].nll = r[0];
            acc[k].fsum = r[1];
            acc[k].gv.resize(nA);
            acc[k].gt.resize(nT);
            for (int a = 0; a < nA; ++a) acc[k].gv[a] = cplx(r[2 + 2 * a], r[3 + 2 * a]) / (k == 0 ? Wp : 1.0);
            for (int j = 0; j < nT; ++j) acc[k].gt[j] = r[2 + 2 * nA + j];
        }
        assemble(m, params, v, acc[0], acc[1], acc[2], sums[3 * nacc + 0], sums[3 * nacc + 2], sums[3 * nacc + 3], nll,
                 grad, nullptr);
        return 0;
    } catch (const std::exception& e) {
        o->err = e.what();
        return -1;
    }
}

// One two-body amplitude tensor (for pinning against the reference's pwa_amp):
// p1, p2 = (E, px, py, pz); out = dj*dj1*dj2 complex.
void orc_pwa_amp(const double* p1, int dj1, const double* p2, int dj2, int dj, int S, int L, double* out)
{
    std::vector<cplx> a;
    pwaAmp(a, LV(p1[0], p1[1], p1[2], p1[3]), dj1, LV(p2[0], p2[1], p2[2], p2[3]), dj2, dj, S, L);
    std::memcpy(out, a.data(), a.size() * sizeof(cplx));
}

double orc_clebsch(int dj1, int m1, int dj2, int m2, int dJ, int M) { return clebsch(dj1, m1, dj2, m2, dJ, M); }

// Wigner small-d d^j_{m1 m2}(beta) (dim = 2j + 1, m doubled) and the
// spherical harmonic Y_l^m(theta, phi) as (re, im) (pinning aids)
double orc_small_d(int dim, int m1x2, int m2x2, double beta) { return smallD(dim, m1x2, m2x2, beta); }
void orc_ylm(int l, int m, double theta, double phi, double* out2)
{
    const cplx y = sphericalY(l, m, theta, phi);
    out2[0] = y.real();
    out2[1] = y.imag();
}

// Custom expression: value and parameter derivatives (out = [Fr, Fi, dF0r, dF0i, ...]).
int orc_custom_eval(const char* expr, const char* pnames_csv, const double* params, int P, double m, double q, int L,
                    double d, double md1, double md2, double* out, char* err, int errlen)
{
    try {
        std::vector<std::string> names;
        std::string s(pnames_csv);
        size_t pos = 0;
        while (pos <= s.size() && !s.empty()) {
            size_t c = s.find(',', pos);
            names.push_back(s.substr(pos, c == std::string::npos ? std::string::npos : c - pos));
            if (c == std::string::npos) break;
            pos = c + 1;
        }
        ExprParser ps(expr, names);
        ExprP e = ps.parse();
        std::vector<D> par;
        for (int i = 0; i < P; ++i) par.push_back(D::var(params[i], i));
        EvalVars v;
        v.v[V_M] = D(m);
        v.v[V_Q] = D(q);
        v.L = L;
        v.v[V_D] = D(d);
        v.v[V_MD1] = D(md1);
        v.v[V_MD2] = D(md2);
        CD f = evalExpr(*e, v, par);
        out[0] = f.re.v;
        out[1] = f.im.v;
        for (int i = 0; i < P; ++i) {
            out[2 + 2 * i] = f.re.g[i];
            out[3 + 2 * i] = f.im.g[i];
        }
        return 0;
    } catch (const std::exception& ex) {
        return fail(err, errlen, ex.what());
    }
}

const char* orc_error(void* h) { return static_cast<Oracle*>(h)->err.c_str(); }

}  // extern "C"

extern "C" {
// Per-call lineshape of a builtin model with explicit settings (pinning aid):
// out = [F, dF/dparam_0 .. dF/dparam_{P-1}] as (re, im) pairs.
int orc_model_eval(int type, int Lmin, double d, int P, int n_ch, const double* ch, const int* mdep,
                   const double* mfix, int has_bf, const double* params, double m, double q, int L, double bf_d,
                   double md1, double md2, double* out)
{
    ResInstance R;
    R.type = (ModelType)type;
    R.Lmin = Lmin;
    R.d = d;
    R.has_bf = has_bf != 0;
    for (int i = 0; i < n_ch; ++i) R.channels.emplace_back(ch[2 * i], ch[2 * i + 1]);
    for (int k = 0; k < 2; ++k) {
        R.md_src[k] = (MassSource)mdep[k];
        R.md_fixed[k] = mfix[k];
    }
    std::vector<D> par;
    for (int i = 0; i < P; ++i) par.push_back(D::var(params[i], i));
    LV z;
    CD f = resonanceFactor(R, par, nullptr, D(m), D(q), L, bf_d, D(md1), D(md2), z, z);
    out[0] = f.re.v;
    out[1] = f.im.v;
    for (int i = 0; i < P; ++i) {
        out[2 + 2 * i] = f.re.g[i];
        out[3 + 2 * i] = f.im.g[i];
    }
    return 0;
}
}

extern "C" {
// Per-event intensity f_e = sum_p |sum_a v_a A_{a,p}|^2 of sample k at params.
int orc_intensity(void* h, int k, const double* params, double* out)
{
    auto* o = static_cast<Oracle*>(h);
    const Model& m = o->m;
    int nA = m.nAmp(), nc = m.nVector(), npol = m.npol;
    long n = o->smp[k].s.n;
    std::vector<double> A((size_t)n * npol * nA * 2);
    orc_columns(h, k, params + 2 * nc, A.data());
    const cplx* Ac = reinterpret_cast<const cplx*>(A.data());
    std::vector<cplx> v(nA);
    for (int a = 0; a < nA; ++a) {
        int c = m.coupling.amp_chain[a];
        v[a] = m.coupling.ratio[a] * cplx(params[c], params[nc + c]);
    }
#pragma omp parallel for schedule(static)
    for (long e = 0; e < n; ++e) {
        double f = 0.0;
        for (int p = 0; p < npol; ++p) {
            cplx s = 0.0;
            for (int a = 0; a < nA; ++a) s += Ac[((size_t)e * npol + p) * nA + a] * v[a];
            f += s.real() * s.real() + s.imag() * s.imag();
        }
        out[e] = f;
    }
    return 0;
}
}
