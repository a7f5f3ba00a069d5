// Model-specific code generation for the fused likelihood kernel (see codegen.hpp).
//
// Lineshape assembly follows the reference kernels:
//   per-call blocks  src/AmpGen.cu:1593-1932 (computeCustomAmpsKernelT), with the
//                    builtin lineshapes as built by buildModelAST (src/ResModel.cu:376-588)
//                    and custom expressions in the language of src/CustomExpr.cu:236-528
//                    (front end: lineshape_lang.cpp)
//   fixed blocks     src/AmpGen.cu:1396-1585 (computeAmpsKernelT) with
//                    computeNodeFactor (include/ResModel.cuh:103-181)
#include "codegen.hpp"

#include "exprdag.hpp"
#include "lineshape_lang.hpp"

#include <algorithm>

#include <cctype>
#include <cmath>
#include <cstdio>
#include <functional>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <tuple>

namespace ctpwa {

namespace {

std::string num(double v)
{
    if (std::isnan(v)) return "ct_nan()";
    if (std::isinf(v)) return v > 0 ? "ct_inf()" : "(-ct_inf())";
    char b[40];
    std::snprintf(b, sizeof b, "%.17g", v);
    std::string s(b);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return s;
}

// ------------------------------------------------------------- generator
// kinematic slot types (angular.cuh AG_K_*)
constexpr int AG_K_MASS_ = 0, AG_K_Q_ = 1, AG_K_QRAW_ = 2, AG_K_P_ = 3, AG_K_E_ = 4, AG_K_CT_ = 5, AG_K_PHI_ = 6;

using dag::Cx;
using dag::Graph;

// DAG builders of the lineshapes, written so that parameter-only factors and
// event-only factors multiply separately (both hoist / share cleanly).
struct Shapes {
    Graph& g;
    explicit Shapes(Graph& gg) : g(gg) {}
    int sq(int a) { return g.mul(a, a); }
    // per-call q0: sqrt((m0^2-(m1+m2)^2)(m0^2-(m1-m2)^2)/(4 m0^2)), 0 below threshold
    int q0(int m0, int m1, int m2)
    {
        int s = g.add(m1, m2), d = g.sub(m1, m2), m0s = sq(m0);
        int q2 = g.mul(g.mul(g.sub(m0s, sq(s)), g.sub(m0s, sq(d))), g.recip(g.mul(g.cnst(4.0), m0s)));
        return g.sel(dag::LT0, q2, g.zero(), g.sqrt(q2));
    }
    // breakup momentum sqrt((m^2-(m1+m2)^2)(m^2-(m1-m2)^2))/(2m), 0 at or below threshold
    int breakup(int m, int m1, int m2)
    {
        int s = g.add(m1, m2), d = g.sub(m1, m2), ms = sq(m);
        int q2 = g.mul(g.sub(ms, sq(s)), g.sub(ms, sq(d)));
        return g.sel(dag::LE0, q2, g.zero(), g.mul(g.sqrt(q2), g.recip(g.mul(g.cnst(2.0), m))));
    }
    int poly(int L, int z)
    {
        static const double C[7][7] = {{1}, {1, 1}, {9, 3, 1}, {225, 45, 6, 1}, {11025, 1575, 135, 10, 1},
                                       {893025, 99225, 6300, 315, 15, 1},
                                       {540326025, 6185025, 363825, 17325, 630, 21, 1}};
        int z2 = sq(z);
        int r = g.cnst(1.0);
        for (int k = L - 1; k >= 0; --k) r = g.add(g.mul(r, z2), g.cnst(C[L][k]));
        return r;
    }
    // Bf(L, q, q0, d) = sqrt(N(q0 d)) * sqrt(1 / N(q d))
    int bf(int L, int q, int q0v, double d)
    {
        if (L <= 0 || L > 6) return g.one();
        int dn = g.cnst(d);
        return g.mul(g.sqrt(poly(L, g.mul(q0v, dn))), g.sqrt(g.recip(poly(L, g.mul(q, dn)))));
    }
    int bf2(int L, int q, int q0v, double d)
    {
        if (L <= 0 || L > 6) return g.one();
        int dn = g.cnst(d);
        return g.mul(poly(L, g.mul(q0v, dn)), g.recip(poly(L, g.mul(q, dn))));
    }
    // 1 / (m0^2 - m^2 - i m0 G(m)), G = G0 (q/q0)^(2L+1) (m0/m) Bf^2
    Cx bwr(int m, int m0, int g0, int L, int q, int q0v, double d)
    {
        int x = g.sub(sq(m0), sq(m));
        int thp = g.mul(g.mul(g0, sq(m0)), g.powi(g.recip(q0v), 2 * L + 1));
        int evp = g.mul(g.powi(q, 2 * L + 1), g.recip(m));
        int y;
        if (L > 0 && L <= 6 && d != 0.0) {
            int dn = g.cnst(d);
            thp = g.mul(thp, poly(L, g.mul(q0v, dn)));
            evp = g.mul(evp, g.recip(poly(L, g.mul(q, dn))));
        }
        y = g.mul(thp, evp);
        int is = g.recip(g.add(sq(x), sq(y)));
        return {g.mul(x, is), g.mul(y, is)};
    }
    Cx bw(int m, int m0, int g0)
    {
        int x = g.sub(sq(m0), sq(m)), y = g.mul(m0, g0);
        int is = g.recip(g.add(sq(x), sq(y)));
        return {g.mul(x, is), g.mul(y, is)};
    }
    // Flatte (FlatteC), per-call form: (A - iB) / (A^2 + B^2)
    Cx flatte(int m, int m0, const std::vector<int>& gs, const std::vector<int>& ch)
    {
        int s = sq(m);
        // m0^2 - s first: the cancelling pair stays one subtraction
        int A = g.sub(sq(m0), s), B = g.zero(), half = g.mul(m0, g.cnst(0.5));
        for (size_t i = 0; i < gs.size(); ++i) {
            int gw = g.mul(gs[i], half);
            A = g.add(A, g.mul(gw, g.rho(true, s, ch[2 * i], ch[2 * i + 1])));
            B = g.sub(B, g.mul(gw, g.rho(false, s, ch[2 * i], ch[2 * i + 1])));
        }
        int iD = g.recip(g.add(sq(A), sq(B)));
        return {g.mul(A, iD), g.neg(g.mul(B, iD))};
    }
    // Flatte, fixed-parameter form (same value, reference arrangement)
    Cx flatteFixed(int m, int m0, const std::vector<int>& gs, const std::vector<int>& ch)
    {
        int s = sq(m), tr = g.zero(), ti = g.zero();
        for (size_t i = 0; i < gs.size(); ++i) {
            int gw = g.mul(g.mul(m0, g.cnst(0.5)), gs[i]);
            tr = g.add(tr, g.mul(gw, g.rho(false, s, ch[2 * i], ch[2 * i + 1])));
            ti = g.add(ti, g.mul(gw, g.rho(true, s, ch[2 * i], ch[2 * i + 1])));
        }
        int dre = g.add(g.sub(sq(m0), s), ti), dim = g.neg(tr);
        int is = g.recip(g.add(sq(dre), sq(dim)));
        return {g.mul(dre, is), g.neg(g.mul(dim, is))};
    }
    // Gounaris-Sakurai (rho -> pi pi), per-call form
    Cx gs(int m, int q, int m0, int g0, int q0v, double mpi)
    {
        const double pi = 3.14159265358979323846;
        auto C = [&](double v) { return g.cnst(v); };
        int hm = g.mul(C(2.0 / pi), g.mul(g.div(q, m), g.log(g.mul(g.add(m, g.mul(C(2.0), q)), C(1.0 / (2.0 * mpi))))));
        int q02 = sq(q0v), q03 = g.mul(q02, q0v);
        int mpi2 = C(mpi * mpi);
        int la = g.log(g.mul(g.add(m0, g.mul(C(2.0), q0v)), C(1.0 / (2.0 * mpi))));
        int dv = g.sub(g.add(g.mul(g.mul(C(3.0 / pi), g.div(mpi2, q02)), la), g.div(m0, g.mul(C(2.0 * pi), q0v))),
                       g.div(g.mul(mpi2, m0), g.mul(C(pi), q03)));
        int h0 = g.mul(C(2.0 / pi), g.mul(g.div(q0v, m0), la));
        int m0s = sq(m0);
        int dh0 = g.add(g.mul(h0, g.sub(g.recip(g.mul(C(8.0), q02)), g.recip(g.mul(C(2.0), m0s)))),
                        g.recip(g.mul(C(2.0 * pi), m0s)));
        int qr = g.div(q, q0v);
        int gam = g.mul(g.mul(g0, g.mul(g.mul(qr, qr), qr)), g.div(m0, m));
        int f = g.mul(g.mul(g0, g.div(m0s, q03)),
                      g.add(g.mul(sq(q), g.sub(hm, h0)), g.mul(g.mul(g.sub(m0s, sq(m)), q02), dh0)));
        int num = g.add(C(1.0), g.div(g.mul(dv, g0), m0));
        int dre = g.add(g.sub(m0s, sq(m)), f);
        int dim = g.neg(g.mul(m0, gam));
        int is = g.recip(g.add(sq(dre), sq(dim)));
        return {g.mul(g.mul(num, dre), is), g.neg(g.mul(g.mul(num, dim), is))};
    }
};

struct Gen {
    const Model& m;
    GeneratedModel out;
    Graph G;
    Shapes S{G};
    std::map<std::tuple<int, unsigned, unsigned, unsigned>, int> slot_of;
    std::vector<std::vector<double>> tables;  // Hist / Interp tables
    // One term of an amplitude column: the lineshape product of one group
    // variant (the base group, or a permutation of identical particles) and
    // the angular plane it multiplies. Without identical particles every
    // column has exactly one term.
    struct TermOut {
        int col = 0, plane = 0;
        int re = 0, im = 0;
        std::vector<std::pair<int, std::pair<int, int>>> der;  // theta -> (d re, d im)
    };
    std::vector<TermOut> cols;  // terms, in block / SL / variant order
    std::vector<int> blk_term0, blk_nterm;
    std::vector<std::pair<int, int>> extra;  // opaque per-event values: (table id, mass node) placeholders

    explicit Gen(const Model& mm) : m(mm) {}

    unsigned mask(const Group& g, int i) const
    {
        int s = g.input_slot[i];
        if (s >= 0) return 1u << s;
        if (s == -1) return (1u << m.final_order.size()) - 1u;
        return mask(g, g.sum_of[i].first) | mask(g, g.sum_of[i].second);
    }
    int slot(int type, int g, int a, int b = -1, int c = -1)
    {
        const Group& Gr = m.groups[g];
        auto key = std::make_tuple(type, mask(Gr, a), b >= 0 ? mask(Gr, b) : 0u, c >= 0 ? mask(Gr, c) : 0u);
        auto it = slot_of.find(key);
        if (it != slot_of.end()) return it->second;
        int id = (int)out.slots.size();
        out.slots.push_back({type, g, a, b, c});
        slot_of[key] = id;
        return id;
    }
    int kin(int type, int g, int a, int b = -1, int c = -1) { return G.kin(slot(type, g, a, b, c)); }

    // custom expression -> DAG (complex)
    struct XCtx {
        int mm, qq, md1, md2, d;
        int L;
        std::vector<int> par;
        int gi = -1, d1 = -1, d2 = -1;
    };
    Cx emitX(const XP& x, const XCtx& c)
    {
        switch (x->k) {
        case XNode::Num: return G.c(x->v);
        case XNode::Param: return G.cr(c.par[x->idx]);
        case XNode::Var: {
            const std::string& v = x->id;
            if (v == "m") return G.cr(c.mm);
            if (v == "q") return G.cr(c.qq);
            if (v == "L") return G.c((double)c.L);
            if (v == "d") return G.cr(c.d);
            if (v == "md1") return G.cr(c.md1);
            if (v == "md2") return G.cr(c.md2);
            static const char* pv[] = {"p1p", "p1e", "p1costheta", "p1phi", "p2p", "p2e", "p2costheta", "p2phi"};
            static const int pt[] = {AG_K_P_, AG_K_E_, AG_K_CT_, AG_K_PHI_};
            for (int i = 0; i < 8; ++i)
                if (v == pv[i]) return c.gi < 0 ? G.c(0.0) : G.cr(kin(pt[i % 4], c.gi, i < 4 ? c.d1 : c.d2));
            return G.c(0.0);
        }
        case XNode::Add: return G.cadd(emitX(x->kids[0], c), emitX(x->kids[1], c));
        case XNode::Sub: return G.csub(emitX(x->kids[0], c), emitX(x->kids[1], c));
        case XNode::Mul: return G.cmul(emitX(x->kids[0], c), emitX(x->kids[1], c));
        case XNode::Div: return G.cdivRef(emitX(x->kids[0], c), emitX(x->kids[1], c));
        case XNode::Pow: return G.cpow(emitX(x->kids[0], c), emitX(x->kids[1], c));
        case XNode::Neg: return G.cneg(emitX(x->kids[0], c));
        case XNode::Func: {
            Cx a = emitX(x->kids[0], c);
            const std::string& f = x->id;
            if (f == "exp") return G.cexp(a);
            if (f == "log") return G.clogRef(a);
            if (f == "sin") return G.csin(a);
            if (f == "cos") return G.ccos(a);
            if (f == "sqrt") return G.csqrt(a);
            if (f == "abs") return G.cr(G.sqrt(G.add(G.mul(a.re, a.re), G.mul(a.im, a.im))));
            if (f == "re") return G.cr(a.re);
            if (f == "im") return G.cr(a.im);
            if (f == "conj") return G.cconj(a);
            return a;
        }
        case XNode::Model: {
            const std::string& id = x->id;
            if (id == "i") return G.c(0.0, 1.0);
            if (id == "q0") {
                Cx a = emitX(x->kids[0], c), b = emitX(x->kids[1], c), d = emitX(x->kids[2], c);
                return G.cr(S.q0(a.re, b.re, d.re));
            }
            if (id == "bf") {
                Cx q = emitX(x->kids[1], c), q0 = emitX(x->kids[2], c), d = emitX(x->kids[3], c);
                if (!G.isConst(d.re)) throw std::runtime_error("custom lineshape: the barrier radius d of Bf must be a constant");
                return G.cr(S.bf((int)x->kids[0]->v, q.re, q0.re, G.val(d.re)));
            }
            if (id == "bw") {
                Cx mm = emitX(x->kids[0], c), m0 = emitX(x->kids[1], c), g0 = emitX(x->kids[2], c);
                return S.bw(mm.re, m0.re, g0.re);
            }
            if (id == "bwr") {
                Cx mm = emitX(x->kids[0], c), m0 = emitX(x->kids[1], c), g0 = emitX(x->kids[2], c);
                Cx q = emitX(x->kids[4], c), q0 = emitX(x->kids[5], c);
                return S.bwr(mm.re, m0.re, g0.re, (int)x->kids[3]->v, q.re, q0.re, x->kids[6]->v);
            }
            if (id == "rho_re" || id == "rho_im") {
                Cx s = emitX(x->kids[0], c), a = emitX(x->kids[1], c), b = emitX(x->kids[2], c);
                return G.cr(G.rho(id == "rho_im", s.re, a.re, b.re));
            }
            return G.c(1.0);
        }
        }
        return G.c(0.0);
    }

    // parameter value nodes of block b: theta leaves (per-call blocks) or constants
    std::vector<std::vector<int>> params(const Block& b)
    {
        std::vector<std::vector<int>> par(b.res.size());
        for (size_t r = 0; r < b.res.size(); ++r)
            for (size_t p = 0; p < b.res[r].params.size(); ++p) {
                int th = b.free_path ? b.res[r].theta[p] : -1;
                par[r].push_back(th >= 0 ? G.theta(th) : G.cnst(b.res[r].params[p]));
            }
        return par;
    }

    // gi: the group (base or permutation variant) whose kinematics are read
    Cx nodeFactor(const Block& b, int gi, int ni, int s, const std::vector<std::vector<int>>& par)
    {
        const Group& g = m.groups[gi];
        const ModelNode& n = g.nodes[ni];
        int L = n.sls[g.sl_combs[s][ni]].L;
        if (b.free_path) {
            int match = -1;
            for (size_t r = 0; r < b.res.size(); ++r)
                if (b.res[r].particle_idx == n.mother && n.mass[0] <= 0) {
                    match = (int)r;
                    break;
                }
            int qq = kin(AG_K_Q_, gi, n.mother, n.d1, n.d2);
            auto mdq = [&](int k) -> int {
                if (n.mass[k + 1] > 0) return G.cnst(n.mass[k + 1]);
                int di = k == 0 ? n.d1 : n.d2;
                for (size_t r = 0; r < b.res.size(); ++r)
                    if (b.res[r].particle_idx == di && !par[r].empty()) return par[r][0];
                return kin(AG_K_MASS_, gi, di);
            };
            int md1 = mdq(0), md2 = mdq(1);
            if (match < 0) {
                if (!n.has_bf) return G.c(1.0);
                int q0 = S.breakup(G.cnst(n.mass[0] > 0 ? n.mass[0] : 1.0), md1, md2);
                return G.cr(S.bf(L, qq, q0, n.bf_d));
            }
            const ResInstance& R = b.res[match];
            const auto& P = par[match];
            int mm = kin(AG_K_MASS_, gi, n.mother);
            int m0 = P.empty() ? G.one() : P[0];
            auto dep = [&](int k) -> int {
                if (R.md_src[k] == MassSource::Fixed) return G.cnst(R.md_fixed[k]);
                if (R.md_src[k] == MassSource::M0Param) return m0;
                return k == 0 ? md1 : md2;
            };
            int q0r = S.q0(m0, dep(0), dep(1));
            Cx bfx = R.has_bf ? G.cr(S.bf(L, qq, q0r, R.d)) : G.c(1.0);
            switch (R.type) {
            case ModelType::BWR: return G.cmul(S.bwr(mm, P[0], P[1], R.Lmin, qq, q0r, R.has_bf ? R.d : 0.0), bfx);
            case ModelType::BW: return S.bw(mm, P[0], P[1]);
            case ModelType::ONE: return bfx;
            case ModelType::Flatte: {
                std::vector<int> gs, ch;
                for (size_t i = 0; i < R.channels.size(); ++i) {
                    gs.push_back(1 + i < P.size() ? P[1 + i] : G.zero());
                    ch.push_back(G.cnst(R.channels[i].first));
                    ch.push_back(G.cnst(R.channels[i].second));
                }
                return G.cmul(S.flatte(mm, P[0], gs, ch), bfx);
            }
            case ModelType::GS: {
                double mpi = R.channels.empty() ? 0.1396 : R.channels[0].first;
                return G.cmul(S.gs(mm, qq, P[0], P[1], q0r, mpi), bfx);
            }
            case ModelType::Custom: {
                XP expr = parseLineshapeExpr(R.options.at("expr"), R.param_names);
                XCtx c;
                c.mm = mm;
                c.qq = qq;
                c.md1 = md1;
                c.md2 = md2;
                c.d = G.cnst(n.bf_d);
                c.L = L;
                c.par = P;
                c.gi = gi;
                c.d1 = n.d1;
                c.d2 = n.d2;
                return emitX(expr, c);
            }
            case ModelType::Interp: return table(R.aux, mm, true);
            case ModelType::Hist: return table(R.aux, mm, false);
            }
            return G.c(1.0);
        }
        // ---- fixed-parameter block (values only) ----
        int mm = kin(AG_K_MASS_, gi, n.mother);
        int qq = kin(AG_K_QRAW_, gi, n.mother, n.d1, n.d2);
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
        int q0 = G.cnst(std::sqrt((mo * mo - std::pow(ma + mb, 2)) * (mo * mo - std::pow(ma - mb, 2))) / 2 / mo);
        if (ni == 0) return n.has_bf ? G.cr(S.bf(L, qq, q0, n.bf_d)) : G.c(1.0);
        if (match < 0) return G.c(1.0);
        const ResInstance& R = b.res[match];
        const auto& P = par[match];
        Cx bfx = n.has_bf ? G.cr(S.bf(L, qq, q0, n.bf_d)) : G.c(1.0);
        switch (R.type) {
        case ModelType::BWR: return G.cmul(S.bwr(mm, P[0], P[1], n.l_min, qq, q0, n.has_bf ? n.bf_d : 0.0), bfx);
        case ModelType::BW: return S.bw(mm, P[0], P[1]);
        case ModelType::ONE: return bfx;
        case ModelType::Flatte: {
            std::vector<int> gs, ch;
            for (size_t i = 0; i < R.channels.size(); ++i) {
                gs.push_back(1 + i < P.size() ? P[1 + i] : G.zero());
                ch.push_back(G.cnst(R.channels[i].first));
                ch.push_back(G.cnst(R.channels[i].second));
            }
            return G.cmul(S.flatteFixed(mm, P[0], gs, ch), bfx);
        }
        case ModelType::Hist: return table(R.aux, mm, false);
        case ModelType::Custom: {
            // value segment with md1 = md2 = 0, no daughter kinematics, at most 3 params
            XP expr = parseLineshapeExpr(R.options.at("expr"), R.param_names);
            XCtx c;
            c.mm = mm;
            c.qq = qq;
            c.md1 = G.zero();
            c.md2 = G.zero();
            c.d = G.cnst(n.bf_d);
            c.L = L;
            for (size_t i = 0; i < P.size(); ++i) c.par.push_back(i < 3 ? P[i] : G.zero());
            return emitX(expr, c);
        }
        default: return G.c(1.0);  // GS / Interp have no fixed-parameter factor in the reference
        }
    }

    // table lookups become opaque per-event values computed by generated helper calls
    struct TabUse {
        int table, mnode;
        bool interp;
        int re_kin, im_kin;  // pseudo kin slots holding the looked-up values
    };
    std::vector<TabUse> tab_uses;
    Cx table(const std::vector<double>& aux, int mnode, bool interp)
    {
        int t = (int)tables.size();
        tables.push_back(aux);
        // represent the looked-up value as pseudo "kin" leaves with negative ids resolved at emission
        int re = G.kin(-1000 - 2 * (int)tab_uses.size()), im = G.kin(-1001 - 2 * (int)tab_uses.size());
        tab_uses.push_back({t, mnode, interp, re, im});
        return {re, interp ? im : G.zero()};
    }

    std::string emit();
};

std::string numf(double v)
{
    if (std::isnan(v)) return "ct_nanf()";
    if (std::isinf(v)) return v > 0 ? "ct_inff()" : "(-ct_inff())";
    char b[40];
    std::snprintf(b, sizeof b, "%.9g", v);
    std::string s(b);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return s + "f";
}

std::string Gen::emit()
{
    const auto& N = G.nodes;
    // roots
    std::vector<int> roots;
    for (const auto& c : cols) {
        roots.push_back(c.re);
        roots.push_back(c.im);
        for (const auto& d : c.der) {
            roots.push_back(d.second.first);
            roots.push_back(d.second.second);
        }
    }
    for (const auto& t : tab_uses) roots.push_back(t.mnode);
    std::vector<char> live(N.size(), 0);
    std::vector<int> stack(roots.begin(), roots.end());
    while (!stack.empty()) {
        int x = stack.back();
        stack.pop_back();
        if (x < 0 || live[x]) continue;
        live[x] = 1;
        for (int k : {N[x].a, N[x].b, N[x].c})
            if (k >= 0) stack.push_back(k);
    }
    // constant slots: parameter-only nodes (theta leaves included) used by
    // event nodes or taken directly as an output
    std::vector<int> cslot(N.size(), -1);
    int ncon = 0;
    auto isTheta = [&](int x) { return N[x].dep == dag::DEP_THETA; };
    std::vector<char> needC(N.size(), 0);
    for (size_t x = 0; x < N.size(); ++x) {
        if (!live[x] || !(N[x].dep & dag::DEP_EVENT)) continue;
        for (int k : {N[x].a, N[x].b, N[x].c})
            if (k >= 0 && isTheta(k)) needC[k] = 1;
    }
    for (int r : roots)
        if (r >= 0 && isTheta(r)) needC[r] = 1;
    for (size_t x = 0; x < N.size(); ++x)
        if (needC[x]) cslot[x] = ncon++;

    // ---------------- parameter-only prologue (FP64) ----------------
    std::ostringstream pro;
    auto proRef = [&](int x) -> std::string {
        const auto& nd = N[x];
        if (nd.op == dag::Const) return num(nd.v);
        if (nd.op == dag::Theta) return "th[" + std::to_string(nd.idx) + "]";
        return "t" + std::to_string(x);
    };
    auto opExpr = [&](const dag::Node& nd, const std::string& A, const std::string& B, const std::string& Cc,
                      bool f32) -> std::string {
        switch (nd.op) {
        case dag::Add: return A + " + " + B;
        case dag::Sub: return A + " - " + B;
        case dag::Mul: return A + " * " + B;
        case dag::Recip: return f32 ? "ct_rcpf(" + A + ")" : "1.0 / " + A;
        case dag::Neg: return "-" + A;
        case dag::Sqrt: return f32 ? "ct_sqrtf(" + A + ")" : "sqrt(" + A + ")";
        case dag::Log: return "log(" + A + ")";
        case dag::Exp: return "exp(" + A + ")";
        case dag::Sin: return "sin(" + A + ")";
        case dag::Cos: return "cos(" + A + ")";
        case dag::Atan2: return "atan2(" + A + ", " + B + ")";
        case dag::Sel: {
            static const char* ops[] = {">=", ">", "<=", "<", "=="};
            return "(" + Cc + " " + ops[nd.cmp] + (f32 ? " 0.0f ? " : " 0.0 ? ") + A + " : " + B + ")";
        }
        case dag::RhoRe: return std::string(f32 ? "(float)" : "") + "ct_rho(" + A + ", " + B + ", " + Cc + ", 0)";
        case dag::RhoIm: return std::string(f32 ? "(float)" : "") + "ct_rho(" + A + ", " + B + ", " + Cc + ", 1)";
        default: return num(nd.v);
        }
    };
    for (size_t x = 0; x < N.size(); ++x) {
        if (!live[x] || N[x].op == dag::Const) continue;
        if (N[x].dep != dag::DEP_THETA) continue;
        if (N[x].op != dag::Theta) {
            const auto& nd = N[x];
            pro << "  const double t" << x << " = "
                << opExpr(nd, nd.a >= 0 ? proRef(nd.a) : "", nd.b >= 0 ? proRef(nd.b) : "", nd.c >= 0 ? proRef(nd.c) : "",
                          false)
                << ";\n";
        }
        if (cslot[x] >= 0) pro << "  C[" << cslot[x] << "] = " << proRef((int)x) << ";\n";
    }

    // ---------------- per-event code ----------------
    // Event nodes come in two kinds. Event-only nodes (kinematic values,
    // table lookups and everything built from them and constants) do not
    // change between likelihood calls: model_event / model_event_mx evaluate
    // them once per event when a sample is loaded and keep, as per-event
    // tables, the ones that parameter-dependent nodes or the outputs consume
    // (the frontier). The per-call code (model_columns*) evaluates only the
    // parameter-dependent nodes, reading frontier values from those tables.
    //
    // Precision of the mixed form (f32): event nodes built from kinematic
    // values and constants by + - * only, that feed a subtraction (or an
    // addition of terms of unknown sign), stay FP64, so the cancellation in
    // m0^2 - m^2 and the like happens in full precision; transcendental
    // functions are FP64 too (their FP32 versions are not correctly rounded,
    // and a bias would not average out over a sample); everything else is
    // FP32 with correctly rounded reciprocals and square roots. This applies
    // to the per-call code: event-only nodes are evaluated once per event in
    // FP64, and the mixed form stores each frontier value either as FP64
    // (the ones marked here, and kinematic values) or rounded once to FP32.
    std::vector<char> cap(N.size(), 0), dbl(N.size(), 0);
    {
        for (size_t x = 0; x < N.size(); ++x) {
            const auto& nd = N[x];
            if (!live[x] || !(nd.dep & dag::DEP_EVENT)) continue;
            if (nd.op == dag::Kin) {
                cap[x] = nd.idx >= 0;
                continue;
            }
            if (nd.op != dag::Add && nd.op != dag::Sub && nd.op != dag::Mul && nd.op != dag::Neg) continue;
            bool ok = true;
            for (int k : {nd.a, nd.b})
                if (k >= 0 && (N[k].dep & dag::DEP_EVENT) && !cap[k]) ok = false;
            cap[x] = ok;
        }
        // nodes known to be >= 0 (an addition of two of them cannot cancel)
        std::vector<char> nonneg(N.size(), 0);
        for (size_t x = 0; x < N.size(); ++x) {
            const auto& nd = N[x];
            switch (nd.op) {
            case dag::Const: nonneg[x] = nd.v >= 0.0; break;
            case dag::Kin:
                nonneg[x] = nd.idx >= 0 && out.slots[nd.idx].type != AG_K_CT_ && out.slots[nd.idx].type != AG_K_PHI_;
                break;
            case dag::Mul: nonneg[x] = nd.a == nd.b || (nonneg[nd.a] && nonneg[nd.b]); break;
            case dag::Add: nonneg[x] = nonneg[nd.a] && nonneg[nd.b]; break;
            case dag::Recip:
            case dag::Sqrt: nonneg[x] = nonneg[nd.a]; break;
            case dag::Exp: nonneg[x] = 1; break;
            default: break;
            }
        }
        for (size_t x = 0; x < N.size(); ++x) {
            const auto& nd = N[x];
            if (live[x] && (nd.dep & dag::DEP_EVENT) &&
                (nd.op == dag::Log || nd.op == dag::Exp || nd.op == dag::Sin || nd.op == dag::Cos || nd.op == dag::Atan2))
                dbl[x] = 1;
        }
        for (size_t x = N.size(); x-- > 0;) {
            const auto& nd = N[x];
            if (!cap[x]) continue;
            if (nd.op == dag::Sub) dbl[x] = 1;
            if (nd.op == dag::Add && nd.a != nd.b && !(nonneg[nd.a] && nonneg[nd.b])) dbl[x] = 1;
            if (!dbl[x]) continue;
            for (int k : {nd.a, nd.b})
                if (k >= 0 && cap[k]) dbl[k] = 1;
        }
    }
    auto evOnly = [&](int x) { return N[x].dep == dag::DEP_EVENT && N[x].op != dag::Const; };
    auto mixedDep = [&](int x) { return (N[x].dep & dag::DEP_EVENT) && (N[x].dep & dag::DEP_THETA); };
    // frontier slots: FP64 table (all), mixed tables (FP32 / FP64 values)
    std::vector<int> fs64(N.size(), -1), fsF(N.size(), -1), fsD(N.size(), -1);
    std::vector<char> shifted(N.size(), 0), shiftUser(N.size(), 0);
    std::vector<double> shiftR(N.size(), 0.0);
    // value of a parameter-only node at the initial parameters
    std::vector<double> tval(N.size(), std::nan(""));
    std::vector<char> tdone(N.size(), 0);
    std::function<double(int)> thetaValue = [&](int x) -> double {
        if (tdone[x]) return tval[x];
        const auto& nd = N[x];
        auto v = [&](int k) { return k >= 0 ? thetaValue(k) : 0.0; };
        double r = std::nan("");
        switch (nd.op) {
        case dag::Const: r = nd.v; break;
        case dag::Theta: r = nd.idx < (int)m.slots.size() ? m.slots[nd.idx].init : std::nan(""); break;
        case dag::Add: r = v(nd.a) + v(nd.b); break;
        case dag::Sub: r = v(nd.a) - v(nd.b); break;
        case dag::Mul: r = v(nd.a) * v(nd.b); break;
        case dag::Recip: r = 1.0 / v(nd.a); break;
        case dag::Neg: r = -v(nd.a); break;
        case dag::Sqrt: r = std::sqrt(v(nd.a)); break;
        case dag::Log: r = std::log(v(nd.a)); break;
        case dag::Exp: r = std::exp(v(nd.a)); break;
        case dag::Sin: r = std::sin(v(nd.a)); break;
        case dag::Cos: r = std::cos(v(nd.a)); break;
        case dag::Atan2: r = std::atan2(v(nd.a), v(nd.b)); break;
        case dag::Sel: {
            const double c = v(nd.c);
            bool t = false;
            switch ((dag::Cmp)nd.cmp) {
            case dag::GE0: t = c >= 0.0; break;
            case dag::GT0: t = c > 0.0; break;
            case dag::LE0: t = c <= 0.0; break;
            case dag::LT0: t = c < 0.0; break;
            case dag::EQ0: t = c == 0.0; break;
            }
            r = t ? v(nd.a) : v(nd.b);
            break;
        }
        default: break;  // channel factors: not needed for a reference value
        }
        tdone[x] = 1;
        tval[x] = r;
        return r;
    };
    {
        std::vector<char> front(N.size(), 0);
        for (size_t x = 0; x < N.size(); ++x) {
            if (!live[x] || !mixedDep((int)x)) continue;
            for (int k : {N[x].a, N[x].b, N[x].c})
                if (k >= 0 && evOnly(k)) front[k] = 1;
        }
        for (const auto& c : cols) {
            for (int r : {c.re, c.im})
                if (r >= 0 && evOnly(r)) front[r] = 1;
            for (const auto& d : c.der)
                for (int r : {d.second.first, d.second.second})
                    if (r >= 0 && evOnly(r)) front[r] = 1;
        }
        // Shifted FP32 storage for the mixed form: a cancellation-prone FP64
        // event value X (such as m^2) whose every use is T - X, X - T or
        // T + X with a parameter-only T, and whose results are used in FP32
        // only, is stored as the FP32 value X - R (R: T at the initial
        // parameters); the per-call code forms (T - R) - X' in FP32. The
        // difference keeps the relative precision of an FP32 rounding of
        // T - X (|X - R| stays of the order of |T - X| while the fit moves T
        // near its start), as the FP64 subtraction rounded to FP32 did, from
        // 4 bytes instead of 8.
        std::vector<std::vector<int>> users(N.size());
        for (size_t y = 0; y < N.size(); ++y) {
            if (!live[y] || !(N[y].dep & dag::DEP_EVENT)) continue;
            for (int k : {N[y].a, N[y].b, N[y].c})
                if (k >= 0) users[k].push_back((int)y);
        }
        std::vector<char> isRoot(N.size(), 0);
        for (const auto& c : cols) {
            for (int r : {c.re, c.im})
                if (r >= 0) isRoot[r] = 1;
            for (const auto& d : c.der)
                for (int r : {d.second.first, d.second.second})
                    if (r >= 0) isRoot[r] = 1;
        }
        for (size_t x = 0; x < N.size(); ++x) {
            if (!front[x] || !dbl[x] || N[x].op == dag::Kin || isRoot[x] || users[x].empty()) continue;
            bool ok = true;
            int tfirst = -1;
            for (int y : users[x]) {
                // event-only users are evaluated once per event, at load, from
                // the FP64 value itself: only the per-call users read X'
                if (evOnly(y)) continue;
                const auto& yn = N[y];
                const int other = yn.a == (int)x ? yn.b : yn.a;
                if (!mixedDep(y) || (yn.op != dag::Sub && yn.op != dag::Add) || yn.a == yn.b || other < 0 ||
                    N[other].dep != dag::DEP_THETA || isRoot[y]) {
                    ok = false;
                    break;
                }
                for (int z : users[y])
                    if (dbl[z] || N[z].op == dag::RhoRe || N[z].op == dag::RhoIm) ok = false;
                for (const auto& t : tab_uses)
                    if (t.mnode == y) ok = false;
                if (tfirst < 0) tfirst = other;
            }
            if (!ok || tfirst < 0) continue;
            const double R = thetaValue(tfirst);
            if (!std::isfinite(R)) continue;
            shiftR[x] = R;
            shifted[x] = 1;
            for (int y : users[x]) {
                if (evOnly(y)) continue;
                shiftUser[y] = 1;
                dbl[y] = 0;
            }
        }
        for (size_t x = 0; x < N.size(); ++x) {
            if (!front[x]) continue;
            fs64[x] = out.nev64++;
            if ((!dbl[x] && N[x].op != dag::Kin) || shifted[x]) fsF[x] = out.nevf++;
            else fsD[x] = out.nevd++;
        }
    }
    // The parameter-only part of every shifted use, T - R (T + R for an
    // addition), becomes a constant of its own, set at the end of the
    // prologue: its FP32 hi + lo then come with the constant bank, and the
    // per-event code adds no FP64 arithmetic or conversion for it.
    std::vector<int> shiftSlot(N.size(), -1);
    std::string shiftPro;
    {
        std::map<std::tuple<int, bool, double>, int> seen;
        for (size_t y = 0; y < N.size(); ++y) {
            if (!shiftUser[y]) continue;
            const auto& nd = N[y];
            const bool xa = shifted[nd.a] != 0;
            const int xs = xa ? nd.a : nd.b, t = xa ? nd.b : nd.a;
            const bool add = nd.op == dag::Add;
            if (cslot[t] < 0) throw std::logic_error("codegen: shifted use without a constant slot");
            const auto key = std::make_tuple(cslot[t], add, shiftR[xs]);
            auto it = seen.find(key);
            if (it == seen.end()) {
                it = seen.emplace(key, ncon++).first;
                shiftPro += "  C[" + std::to_string(it->second) + "] = C[" + std::to_string(cslot[t]) + "]" +
                            (add ? " + " : " - ") + num(shiftR[xs]) + ";\n";
            }
            shiftSlot[y] = it->second;
        }
    }
    pro << shiftPro;
    using RefFn = std::function<std::string(int, bool)>;
    // reference to a kinematic leaf, a table lookup or an event node from the
    // once-per-event code, for a consumer evaluated in FP32 (wantF) or FP64
    auto preRef = [&](bool f32) -> RefFn {
        return [&, f32](int x, bool wantF) -> std::string {
            const auto& nd = N[x];
            if (nd.op == dag::Const) return wantF ? numf(nd.v) : num(nd.v);
            if (nd.op == dag::Kin && nd.idx >= 0)
                return (wantF ? "kf" : "kv[") + std::to_string(nd.idx) + (wantF ? "" : "]");
            if (nd.op == dag::Kin) {
                int u = (-nd.idx - 1000) / 2;
                std::string v = ((-nd.idx - 1000) % 2 == 0 ? "tre" : "tim") + std::to_string(u);
                return wantF ? "(float)" + v : v;
            }
            bool isF = f32 && !dbl[x];
            std::string v = "e" + std::to_string(x);
            if (wantF && !isF) return "(float)" + v;
            if (!wantF && isF) return "(double)" + v;
            return v;
        };
    };
    // the same from the per-call code: event-only operands are frontier values
    auto colRef = [&](bool f32) -> RefFn {
        return [&, f32](int x, bool wantF) -> std::string {
            const auto& nd = N[x];
            if (nd.op == dag::Const) return wantF ? numf(nd.v) : num(nd.v);
            if (nd.dep == dag::DEP_THETA) return (wantF ? "Cfh[" : "C[") + std::to_string(cslot[x]) + "]";
            if (evOnly(x)) {
                if (fs64[x] < 0) throw std::logic_error("codegen: event value outside the frontier");
                if (!f32) return "ev[" + std::to_string(fs64[x]) + "]";
                if (fsF[x] >= 0) return (wantF ? "evf[" : "(double)evf[") + std::to_string(fsF[x]) + "]";
                return (wantF ? "(float)evd[" : "evd[") + std::to_string(fsD[x]) + "]";
            }
            bool isF = f32 && !dbl[x];
            std::string v = "e" + std::to_string(x);
            if (wantF && !isF) return "(float)" + v;
            if (!wantF && isF) return "(double)" + v;
            return v;
        };
    };
    // nodes the lineshape values depend on (the others feed only the
    // derivatives, i.e. the gradient, where a common FP32 rounding of a
    // parameter-only factor is a relative error of 6e-8 and no bias of the
    // likelihood)
    std::vector<char> valueNode(N.size(), 0);
    {
        std::vector<int> st;
        for (const auto& c : cols) {
            st.push_back(c.re);
            st.push_back(c.im);
        }
        while (!st.empty()) {
            int x = st.back();
            st.pop_back();
            if (x < 0 || valueNode[x]) continue;
            valueNode[x] = 1;
            for (int k : {N[x].a, N[x].b, N[x].c})
                if (k >= 0) st.push_back(k);
        }
    }
    // FP32 value nodes kept as an unevaluated sum hi + lo (names e<x>_h,
    // e<x>_l; e<x> is their rounded sum for the other consumers). A sum of a
    // per-event value and a parameter-only constant, or its shifted form, is
    // formed by an exact two-sum: its rounding would otherwise be the same
    // for every event of a binade (below the event value's ulp the bits are
    // the constant's), and so would be that of adding the constant's lo
    // part, which moves every event's value by the same fraction of an ulp:
    // a bias of ~1e-9 of the sample mean that the data weight sum multiplies.
    // The products and sums that consume such a value take its lo part in,
    // where the other factor's bits make the rounding independent per event.
    std::vector<char> hasLo(N.size(), 0);
    auto twoSum = [](size_t x, const std::string& a, const std::string& b, const std::string& c) {
        const std::string X = "e" + std::to_string(x), H = X + "_h", L = X + "_l", BB = X + "_b";
        return "  const float " + H + " = " + a + " + " + b + ";\n  const float " + BB + " = " + H + " - " + a +
               ";\n  const float " + L + " = ((" + a + " - (" + H + " - " + BB + ")) + (" + b + " - " + BB + "))" +
               (c.empty() ? std::string() : " + " + c) + ";\n  const float " + X + " = " + H + " + " + L + ";\n";
    };
    auto neg = [](const std::string& v) { return v.empty() ? v : "-(" + v + ")"; };
    auto addLo = [](const std::string& a, const std::string& b) {
        if (a.empty()) return b;
        if (b.empty()) return a;
        return "(" + a + " + " + b + ")";
    };
    // definition of event node x
    auto nodeLine = [&](size_t x, bool f32, const RefFn& ref) -> std::string {
        const auto& nd = N[x];
        if (f32 && shiftUser[x]) {
            // T - X, X - T or T + X from the shifted FP32 value X' = X - R
            const bool xa = shifted[nd.a] != 0;
            const int xs = xa ? nd.a : nd.b, t = xa ? nd.b : nd.a;
            (void)t;
            const std::string Xs = "evf[" + std::to_string(fsF[xs]) + "]", ks = std::to_string(shiftSlot[x]),
                              Dh = "Cfh[" + ks + "]", Dl = "Cfl[" + ks + "]";
            // the parameter-only part D = T -+ R enters as hi + lo (a single
            // FP32 rounding of it would shift every event alike)
            if (valueNode[x]) {
                hasLo[x] = 1;
                if (nd.op == dag::Add) return twoSum(x, Dh, Xs, Dl);  // (T + R) + X'
                if (xa) return twoSum(x, Xs, neg(Dh), neg(Dl));         // X - T = X' - D
                return twoSum(x, Dh, neg(Xs), Dl);                     // T - X = D - X'
            }
            std::string rhs;
            if (nd.op == dag::Add) rhs = "(" + Dh + " + " + Xs + ") + " + Dl;     // (T + R) + X'
            else if (xa) rhs = "-((" + Dh + " - " + Xs + ") + " + Dl + ")";      // X - T
            else rhs = "(" + Dh + " - " + Xs + ") + " + Dl;                      // (T - R) - X'
            return "  const float e" + std::to_string(x) + " = " + rhs + ";\n";
        }
        bool isF = f32 && !dbl[x];
        std::string A, B, Cc;
        if (nd.op == dag::RhoRe || nd.op == dag::RhoIm) {
            // channel factors are evaluated by an FP64 helper
            A = ref(nd.a, false);
            B = ref(nd.b, false);
            Cc = ref(nd.c, false);
        } else {
            A = nd.a >= 0 ? ref(nd.a, isF) : "";
            B = nd.b >= 0 ? ref(nd.b, isF) : "";
            if (nd.c >= 0) {
                // the condition is tested in the precision it was computed in
                const auto& cn = N[nd.c];
                bool cF = f32 && (cn.dep & dag::DEP_EVENT) && cn.op != dag::Kin && !dbl[nd.c];
                Cc = ref(nd.c, cF);
            }
        }
        std::string rhs = opExpr(nd, A, B, Cc, isF);
        if (isF && valueNode[x] && (nd.op == dag::Add || nd.op == dag::Sub || nd.op == dag::Mul || nd.op == dag::Neg)) {
            // An event-independent operand of a value node enters as hi + lo,
            // and so does an operand kept as hi + lo; a product is rounded
            // once (fmaf): rounding it to FP32 first would bias every event
            // alike, and so would rounding the product of two FP32-grid
            // factors (structured low bits).
            struct Part {
                std::string hi, lo;
                bool cst = false;
            };
            auto part = [&](int y, const std::string& plain) -> Part {
                const auto& yn = N[y];
                if (yn.op == dag::Const) {
                    float h = (float)yn.v;
                    double l = yn.v - (double)h;
                    if (l == 0.0 || !std::isfinite(yn.v)) return {plain, "", true};
                    return {numf((double)h), numf(l), true};
                }
                if (yn.dep == dag::DEP_THETA)
                    return {"Cfh[" + std::to_string(cslot[y]) + "]", "Cfl[" + std::to_string(cslot[y]) + "]", true};
                if (hasLo[y]) return {"e" + std::to_string(y) + "_h", "e" + std::to_string(y) + "_l", false};
                return {plain, "", false};
            };
            const std::string X = "e" + std::to_string(x);
            if (nd.op == dag::Neg) {
                if (hasLo[nd.a]) {
                    hasLo[x] = 1;
                    return "  const float " + X + "_h = -e" + std::to_string(nd.a) + "_h;\n  const float " + X +
                           "_l = -e" + std::to_string(nd.a) + "_l;\n  const float " + X + " = -e" + std::to_string(nd.a) +
                           ";\n";
                }
            } else {
                const Part pa = part(nd.a, A), pb = part(nd.b, B);
                const bool event_a = (N[nd.a].dep & dag::DEP_EVENT) != 0, event_b = (N[nd.b].dep & dag::DEP_EVENT) != 0;
                if (nd.op == dag::Mul) {
                    if (nd.a == nd.b && !pa.lo.empty()) {
                        rhs = "fmaf(" + pa.hi + ", " + pa.hi + ", (" + pa.hi + " + " + pa.hi + ") * " + pa.lo + ")";
                    } else if (!pa.lo.empty() || !pb.lo.empty()) {
                        std::string corr;
                        if (!pa.lo.empty() && !pb.lo.empty())
                            corr = "fmaf(" + pa.hi + ", " + pb.lo + ", " + pa.lo + " * " + pb.hi + ")";
                        else if (!pb.lo.empty()) corr = pa.hi + " * " + pb.lo;
                        else corr = pa.lo + " * " + pb.hi;
                        rhs = "fmaf(" + pa.hi + ", " + pb.hi + ", " + corr + ")";
                    }
                } else if ((event_a && event_b && (!pa.lo.empty() || !pb.lo.empty())) ||
                           (event_a != event_b && (!pa.lo.empty() || !pb.lo.empty()))) {
                    // a sum with a constant or with a hi + lo operand: two-sum of the
                    // hi parts, the lo parts added to its error
                    const bool sub = nd.op == dag::Sub;
                    hasLo[x] = 1;
                    return twoSum(x, pa.hi, sub ? neg(pb.hi) : pb.hi, addLo(pa.lo, sub ? neg(pb.lo) : pb.lo));
                }
            }
        }
        return std::string("  const ") + (isF ? "float" : "double") + " e" + std::to_string(x) + " = " + rhs + ";\n";
    };
    // once per event (FP64): event-only nodes, then the frontier values
    auto eventPart = [&]() -> std::string {
        std::ostringstream evs;
        const RefFn ref = preRef(false);
        for (size_t u = 0; u < tab_uses.size(); ++u) {
            const auto& t = tab_uses[u];
            if (t.interp)
                evs << "  double tre" << u << ", tim" << u << "; ls_interp(ct_tab" << t.table << ", " << ref(t.mnode, false)
                    << ", tre" << u << ", tim" << u << ");\n";
            else
                evs << "  const double tre" << u << " = ls_hist(" << ref(t.mnode, false) << ", ct_tab" << t.table
                    << "), tim" << u << " = 0.0;\n";
        }
        for (size_t x = 0; x < N.size(); ++x)
            if (live[x] && evOnly((int)x) && N[x].op != dag::Kin) evs << nodeLine(x, false, ref);
        for (size_t x = 0; x < N.size(); ++x)
            if (fs64[x] >= 0) evs << "  o[" << fs64[x] << "] = " << ref((int)x, false) << ";\n";
        return evs.str();
    };
    // per call: parameter-dependent event nodes and the outputs
    auto callPart = [&](bool f32) -> std::string {
        std::ostringstream evs;
        const RefFn ref = colRef(f32);
        for (size_t x = 0; x < N.size(); ++x)
            if (live[x] && mixedDep((int)x) && N[x].op != dag::Const && N[x].op != dag::Theta && N[x].op != dag::Kin)
                evs << nodeLine(x, f32, ref);
        int k = 0;
        for (size_t a = 0; a < cols.size(); ++a) {
            evs << "  Fr[" << a << "] = " << ref(cols[a].re, f32) << "; Fi[" << a << "] = " << ref(cols[a].im, f32) << ";\n";
            for (const auto& d : cols[a].der) {
                evs << "  dFr[" << k << "] = " << ref(d.second.first, f32) << "; dFi[" << k << "] = "
                    << ref(d.second.second, f32) << ";\n";
                ++k;
            }
        }
        return evs.str();
    };

    // ---------------- dual-number form (Hessian-vector products) ----------------
    // The per-call FP64 code in which every parameter-dependent value is a
    // CtDual (value, directional derivative): the prologue runs on dual theta
    // leaves, parameter-dependent event nodes become dual, frontier values
    // stay plain doubles. Channel factors take plain values (their parameter
    // derivative is zero, as in the symbolic derivatives above).
    {
        auto dualRef = [&](int x) -> std::string {
            const auto& nd = N[x];
            if (nd.op == dag::Const) return num(nd.v);
            if (nd.dep == dag::DEP_THETA) return "C[" + std::to_string(cslot[x]) + "]";
            if (evOnly(x)) return "ev[" + std::to_string(fs64[x]) + "]";
            return "e" + std::to_string(x);
        };
        auto plain = [](const std::string& s) { return "ct_value(" + s + ")"; };
        auto rhs = [&](const dag::Node& nd, const std::function<std::string(int)>& r) {
            const bool rho = nd.op == dag::RhoRe || nd.op == dag::RhoIm;
            std::string A = nd.a >= 0 ? r(nd.a) : "", B = nd.b >= 0 ? r(nd.b) : "", Cc = nd.c >= 0 ? r(nd.c) : "";
            if (rho) {
                A = plain(A);
                B = plain(B);
                Cc = plain(Cc);
            }
            return opExpr(nd, A, B, Cc, false);
        };
        std::ostringstream dpro, dev;
        for (size_t x = 0; x < N.size(); ++x) {
            if (!live[x] || N[x].op == dag::Const || N[x].dep != dag::DEP_THETA) continue;
            if (N[x].op != dag::Theta) dpro << "  const CtDual t" << x << " = " << rhs(N[x], proRef) << ";\n";
            if (cslot[x] >= 0) dpro << "  C[" << cslot[x] << "] = " << proRef((int)x) << ";\n";
        }
        dpro << shiftPro;
        for (size_t x = 0; x < N.size(); ++x) {
            const auto& nd = N[x];
            if (!live[x] || !mixedDep((int)x) || nd.op == dag::Const || nd.op == dag::Theta || nd.op == dag::Kin) continue;
            dev << "  const CtDual e" << x << " = " << rhs(nd, dualRef) << ";\n";
        }
        int q = 0;
        for (size_t a = 0; a < cols.size(); ++a) {
            dev << "  Fr[" << a << "] = " << dualRef(cols[a].re) << "; Fi[" << a << "] = " << dualRef(cols[a].im) << ";\n";
            for (const auto& d : cols[a].der) {
                dev << "  dFr[" << q << "] = " << dualRef(d.second.first) << "; dFi[" << q << "] = "
                    << dualRef(d.second.second) << ";\n";
                ++q;
            }
        }
        std::ostringstream dh;
        dh << "// generated by ctpwa_b200 codegen: the lineshape products in dual numbers\n#pragma once\n";
        dh << "// parameter-only subexpressions with their directional derivatives\n";
        dh << "__device__ __forceinline__ void model_prologue_dual(const CtDual* __restrict__ th, CtDual* __restrict__ C)\n{\n"
              "  (void)th; (void)C;\n"
           << dpro.str() << "}\n";
        dh << "// per-event lineshape products, their theta derivatives, and the directional\n"
              "// derivatives of both (FP64), from the event's frontier values\n";
        dh << "__device__ __forceinline__ void model_columns_dual(const double* __restrict__ ev, const CtDual* __restrict__ C,\n"
              "    CtDual* Fr, CtDual* Fi, CtDual* dFr, CtDual* dFi)\n{\n  (void)ev; (void)C; (void)dFr; (void)dFi;\n"
           << dev.str() << "}\n";
        out.dual_header = dh.str();
    }

    std::vector<std::pair<int, int>> der_entries;  // (term, theta)
    for (size_t a = 0; a < cols.size(); ++a)
        for (const auto& d : cols[a].der) der_entries.push_back({(int)a, d.first});
    const int k = (int)der_entries.size();
    out.nder = k;
    out.nterm = (int)cols.size();
    out.nconst = ncon;
    std::ostringstream h;
    auto table = [&](const char* name, const std::vector<int>& v) {
        h << "__device__ __forceinline__ int " << name << "(int i) {\n  switch (i) {\n";
        for (size_t i = 0; i < v.size(); ++i) h << "  case " << i << ": return " << v[i] << ";\n";
        h << "  default: return 0;\n  }\n}\n";
    };
    h << "// generated by ctpwa_b200 codegen: model-specific lineshape products\n#pragma once\n";
    h << "#define M_NA " << m.nAmp() << "\n#define M_NTERM " << cols.size() << "\n#define M_NPOL " << m.npol
      << "\n#define M_NPLANE " << out.nplane << "\n#define M_NKIN " << out.slots.size() << "\n#define M_NTH "
      << m.nTheta() << "\n#define M_NDER " << k << "\n#define M_NCONST " << ncon << "\n";
    h << "#define M_NEV " << out.nev64 << "\n#define M_NEVF " << out.nevf << "\n#define M_NEVD " << out.nevd << "\n";
    // terms: amplitude column and angular plane of each
    std::vector<int> tcol, tplane;
    for (const auto& t : cols) {
        tcol.push_back(t.col);
        tplane.push_back(t.plane);
    }
    table("term_col", tcol);
    table("term_plane", tplane);
    // resonance blocks (partial waves of the fit fractions): their terms
    h << "#define M_NBLK " << m.blocks.size() << "\n";
    table("blk_term0", blk_term0);
    table("blk_nterm", blk_nterm);
    std::vector<int> dterm;
    for (const auto& d : der_entries) dterm.push_back(d.first);
    table("der_term", dterm);
    h << "__device__ __forceinline__ int der_th(int k) {\n  switch (k) {\n";
    for (size_t q = 0; q < der_entries.size(); ++q) h << "  case " << q << ": return " << der_entries[q].second << ";\n";
    h << "  default: return 0;\n  }\n}\n";
    for (size_t t = 0; t < tables.size(); ++t) {
        h << "__device__ const double ct_tab" << t << "[" << std::max<size_t>(1, tables[t].size()) << "] = {";
        for (size_t i = 0; i < tables[t].size(); ++i) h << (i ? ", " : "") << num(tables[t][i]);
        if (tables[t].empty()) h << "0.0";
        h << "};\n";
    }
    h << "// parameter-only subexpressions, evaluated once per likelihood call\n";
    h << "__device__ __forceinline__ void model_prologue(const double* __restrict__ th, double* __restrict__ C)\n{\n"
         "  (void)th; (void)C;\n"
      << pro.str() << "}\n";
    h << "// once per event (sample loading): the parameter-independent values the\n"
         "// per-call code reads (frontier), FP64\n";
    h << "__device__ __forceinline__ void model_event(const double* __restrict__ kv, double* __restrict__ o)\n{\n"
         "  (void)kv; (void)o;\n"
      << eventPart() << "}\n";
    // The mixed form's frontier is the FP64 frontier rounded once per value
    // (shifted values X - R formed in FP64 first): the once-per-event work
    // costs nothing per call, so its FP64 result is kept rather than an FP32
    // evaluation whose error of a few ulps would add to every event's
    // intensity.
    std::ostringstream mx;
    for (size_t x = 0; x < N.size(); ++x) {
        if (fs64[x] < 0) continue;
        const std::string o = "o[" + std::to_string(fs64[x]) + "]";
        if (shifted[x]) mx << "  of[" << fsF[x] << "] = (float)(" << o << " - " << num(shiftR[x]) << ");\n";
        else if (fsF[x] >= 0) mx << "  of[" << fsF[x] << "] = (float)" << o << ";\n";
        else mx << "  od[" << fsD[x] << "] = " << o << ";\n";
    }
    h << "// the same for the mixed form from the FP64 frontier o: FP32 values (of)\n"
         "// and FP64 values (od)\n";
    h << "__device__ __forceinline__ void model_event_mx(const double* __restrict__ o, float* __restrict__ of,\n"
         "    double* __restrict__ od)\n{\n  (void)o; (void)of; (void)od;\n"
      << mx.str() << "}\n";
    h << "// per-event lineshape products and their parameter derivatives (FP64) from the\n"
         "// event's frontier values\n";
    h << "__device__ __forceinline__ void model_columns(const double* __restrict__ ev, const double* __restrict__ C,\n"
         "    double* Fr, double* Fi, double* dFr, double* dFi)\n{\n  (void)ev; (void)C; (void)dFr; (void)dFi;\n"
      << callPart(false) << "}\n";
    h << "// the same in the mixed form (FP32 except cancellation-prone polynomial parts and\n"
         "// transcendental functions; parameter-only constants enter as hi + lo FP32 pairs)\n";
    h << "__device__ __forceinline__ void model_columns_f32(const float* __restrict__ evf, const double* __restrict__ evd,\n"
         "    const double* __restrict__ C, const float* __restrict__ Cfh, const float* __restrict__ Cfl, float* Fr, float* Fi,\n"
         "    float* dFr, float* dFi)\n{\n"
         "  (void)evf; (void)evd; (void)C; (void)Cfh; (void)Cfl; (void)dFr; (void)dFi;\n"
      << callPart(true) << "}\n";
    return h.str();
}

}  // namespace

GeneratedModel generateModel(const Model& m)
{
    Gen g(m);
    int pl = 0;
    for (const auto& gr : m.groups) {
        g.out.group_plane0.push_back(pl);
        pl += gr.nSL();
    }
    g.out.nplane = pl;
    g.out.npol = m.npol;
    g.out.ngrad = 2 * m.nAmp() + m.nTheta();
    for (const auto& b : m.blocks) {
        const Group& gr = m.groups[b.group];
        auto par = g.params(b);
        std::vector<int> ths;
        if (b.free_path)
            for (const auto& r : b.res)
                for (int t : r.theta)
                    if (t >= 0 && std::find(ths.begin(), ths.end(), t) == ths.end()) ths.push_back(t);
        std::vector<int> vars = {b.group};
        for (int v : gr.variants) vars.push_back(v);
        g.blk_term0.push_back((int)g.cols.size());
        for (int s = 0; s < gr.nSL(); ++s)
            for (int v : vars) {
                Cx F = g.G.c(m.groups[v].sign);
                for (size_t ni = 0; ni < gr.nodes.size(); ++ni) F = g.G.cmul(F, g.nodeFactor(b, v, (int)ni, s, par));
                Gen::TermOut t;
                t.col = b.site + s;
                t.plane = g.out.group_plane0[v] + s;
                t.re = F.re;
                t.im = F.im;
                for (int th : ths) {
                    int dr = g.G.deriv(F.re, th), di = g.G.deriv(F.im, th);
                    if (g.G.isConst(dr) && g.G.val(dr) == 0.0 && g.G.isConst(di) && g.G.val(di) == 0.0) continue;
                    t.der.push_back({th, {dr, di}});
                }
                g.cols.push_back(t);
            }
        g.blk_nterm.push_back((int)g.cols.size() - g.blk_term0.back());
    }
    g.out.header = g.emit();
    return g.out;
}

void checkCustomExpr(const std::string& expr, const std::vector<std::string>& params)
{
    parseLineshapeExpr(expr, params);
}

}  // namespace ctpwa
