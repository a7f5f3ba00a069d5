// Model-specific code generation for the fused likelihood kernel (see codegen.hpp).
//
// Lineshape assembly follows the reference kernels:
//   per-call blocks  src/AmpGen.cu:1593-1932 (computeCustomAmpsKernelT), with the
//                    builtin lineshapes as built by buildModelAST (src/ResModel.cu:376-588)
//                    and custom expressions as parsed by src/CustomExpr.cu:236-528
//   fixed blocks     src/AmpGen.cu:1396-1585 (computeAmpsKernelT) with
//                    computeNodeFactor (include/ResModel.cuh:103-181)
#include "codegen.hpp"

#include <cctype>
#include <cmath>
#include <cstdio>
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

// ------------------------------------------------------------- expressions
struct XNode {
    enum K { Num, Var, Param, Add, Sub, Mul, Div, Pow, Neg, Func, Model } k = Num;
    double v = 0;
    std::string id;  // var / func / model name
    int idx = 0;     // param index
    std::vector<std::shared_ptr<XNode>> kids;
};
using XP = std::shared_ptr<XNode>;

XP xn(XNode::K k, std::vector<XP> kids = {}, double v = 0, std::string id = "", int idx = 0)
{
    auto n = std::make_shared<XNode>();
    n->k = k;
    n->kids = std::move(kids);
    n->v = v;
    n->id = std::move(id);
    n->idx = idx;
    return n;
}

// Recursive-descent parser of the custom-lineshape language
// (grammar of src/CustomExpr.cu:236-528).
class XParser {
public:
    XParser(const std::string& s, const std::vector<std::string>& params) : params_(params) { lex(s); }
    XP parse()
    {
        XP e = expr();
        if (t_[p_].k != T::End) throw std::runtime_error("CustomExpr: trailing tokens");
        return e;
    }

private:
    struct T {
        enum Kind { Num, Id, Op, LP, RP, Comma, End } k;
        double v = 0;
        std::string s;
    };
    std::vector<T> t_;
    size_t p_ = 0;
    const std::vector<std::string>& params_;

    void lex(const std::string& s)
    {
        size_t i = 0;
        while (i < s.size()) {
            char c = s[i];
            if (std::isspace((unsigned char)c)) { ++i; continue; }
            if (std::isdigit((unsigned char)c) || c == '.') {
                if (c == '1' && i + 1 < s.size() && (s[i + 1] == 'j' || s[i + 1] == 'i')) {
                    t_.push_back({T::Id, 0, "1j"});
                    i += 2;
                    continue;
                }
                size_t j = i;
                while (j < s.size() && (std::isdigit((unsigned char)s[j]) || s[j] == '.' || s[j] == 'e' || s[j] == 'E' ||
                                        ((s[j] == '+' || s[j] == '-') && j > i && (s[j - 1] == 'e' || s[j - 1] == 'E'))))
                    ++j;
                t_.push_back({T::Num, std::stod(s.substr(i, j - i)), ""});
                i = j;
                continue;
            }
            if (std::isalpha((unsigned char)c) || c == '_') {
                size_t j = i;
                while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
                t_.push_back({T::Id, 0, s.substr(i, j - i)});
                i = j;
                continue;
            }
            if (std::string("+-*/^").find(c) != std::string::npos) { t_.push_back({T::Op, 0, std::string(1, c)}); ++i; continue; }
            if (c == '(') { t_.push_back({T::LP, 0, ""}); ++i; continue; }
            if (c == ')') { t_.push_back({T::RP, 0, ""}); ++i; continue; }
            if (c == ',') { t_.push_back({T::Comma, 0, ""}); ++i; continue; }
            throw std::runtime_error(std::string("CustomExpr: unexpected char '") + c + "'");
        }
        t_.push_back({T::End, 0, ""});
    }
    bool op(const char* o) const { return t_[p_].k == T::Op && t_[p_].s == o; }
    XP expr()
    {
        XP l = term();
        while (op("+") || op("-")) {
            bool a = t_[p_++].s == "+";
            l = xn(a ? XNode::Add : XNode::Sub, {l, term()});
        }
        return l;
    }
    XP term()
    {
        XP l = factor();
        while (op("*") || op("/")) {
            bool m = t_[p_++].s == "*";
            l = xn(m ? XNode::Mul : XNode::Div, {l, factor()});
        }
        return l;
    }
    XP factor()
    {
        XP b = unary();
        if (op("^")) {
            ++p_;
            return xn(XNode::Pow, {b, factor()});
        }
        return b;
    }
    XP unary()
    {
        if (op("-")) {
            ++p_;
            return xn(XNode::Neg, {unary()});
        }
        if (op("+")) {
            ++p_;
            return unary();
        }
        return primary();
    }
    std::vector<XP> args()
    {
        if (t_[p_].k != T::LP) throw std::runtime_error("CustomExpr: function needs (");
        ++p_;
        std::vector<XP> a;
        if (t_[p_].k == T::RP) {
            ++p_;
            return a;
        }
        while (true) {
            a.push_back(expr());
            if (t_[p_].k == T::Comma) { ++p_; continue; }
            break;
        }
        if (t_[p_].k != T::RP) throw std::runtime_error("CustomExpr: missing )");
        ++p_;
        return a;
    }
    XP q0node()
    {
        return xn(XNode::Model, {params_.empty() ? xn(XNode::Num, {}, 1.0) : xn(XNode::Param, {}, 0, "", 0),
                                 xn(XNode::Var, {}, 0, "md1"), xn(XNode::Var, {}, 0, "md2")},
                  0, "q0");
    }
    XP primary()
    {
        T t = t_[p_];
        if (t.k == T::Num) {
            ++p_;
            return xn(XNode::Num, {}, t.v);
        }
        if (t.k == T::LP) {
            ++p_;
            XP e = expr();
            if (t_[p_].k != T::RP) throw std::runtime_error("CustomExpr: missing )");
            ++p_;
            return e;
        }
        if (t.k != T::Id) throw std::runtime_error("CustomExpr: unexpected token");
        ++p_;
        const std::string& s = t.s;
        if (s == "1j") return xn(XNode::Model, {}, 0, "i");
        if (s == "pi") return xn(XNode::Num, {}, 3.14159265358979323846);
        if (s == "q0" && t_[p_].k != T::LP) return q0node();
        static const char* vars[] = {"m", "q", "L", "d", "p1p", "p1e", "p1costheta", "p1phi",
                                     "p2p", "p2e", "p2costheta", "p2phi"};
        for (const char* v : vars)
            if (s == v) return xn(XNode::Var, {}, 0, s);
        static const std::map<std::string, std::string> funcs = {
            {"exp", "exp"}, {"log", "log"}, {"ln", "log"}, {"sin", "sin"}, {"cos", "cos"}, {"sqrt", "sqrt"},
            {"abs", "abs"}, {"Re", "re"}, {"real", "re"}, {"Im", "im"}, {"imag", "im"}, {"conj", "conj"}, {"csqrt", "sqrt"}};
        auto fi = funcs.find(s);
        if (fi != funcs.end()) {
            if (t_[p_].k != T::LP) throw std::runtime_error("CustomExpr: function '" + s + "' needs (");
            ++p_;
            XP a = expr();
            if (t_[p_].k != T::RP) throw std::runtime_error("CustomExpr: missing )");
            ++p_;
            return xn(XNode::Func, {a}, 0, fi->second);
        }
        if (s == "BW" || s == "BWR" || s == "Bf" || s == "Flatte" || (s == "q0" && t_[p_].k == T::LP)) {
            auto a = args();
            XP m = xn(XNode::Var, {}, 0, "m");
            if (s == "BW") {
                if (a.size() != 2) throw std::runtime_error("CustomExpr: BW(m0, w0) needs exactly 2 args");
                return xn(XNode::Model, {m, a[0], a[1]}, 0, "bw");
            }
            if (s == "BWR") {
                if (a.size() < 2 || a.size() > 4) throw std::runtime_error("CustomExpr: BWR(m0, g0[, L, d]) needs 2~4 args");
                if (a.size() >= 3 && a[2]->k != XNode::Num) throw std::runtime_error("CustomExpr: BWR L must be a literal (e.g. 1)");
                if (a.size() >= 4 && a[3]->k != XNode::Num) throw std::runtime_error("CustomExpr: BWR d must be a literal (e.g. 3.0)");
                double Lv = a.size() >= 3 ? a[2]->v : 1.0, dv = a.size() >= 4 ? a[3]->v : 3.0;
                return xn(XNode::Model, {m, a[0], a[1], xn(XNode::Num, {}, Lv), xn(XNode::Var, {}, 0, "q"), q0node(), xn(XNode::Num, {}, dv)}, 0, "bwr");
            }
            if (s == "Bf") {
                if (a.size() != 4) throw std::runtime_error("CustomExpr: Bf(L, q, q0, d) needs exactly 4 args");
                if (a[0]->k != XNode::Num) throw std::runtime_error("CustomExpr: Bf L must be a literal (e.g. 1)");
                return xn(XNode::Model, a, 0, "bf");
            }
            if (s == "q0") {
                if (a.size() == 1) return xn(XNode::Model, {a[0], xn(XNode::Var, {}, 0, "md1"), xn(XNode::Var, {}, 0, "md2")}, 0, "q0");
                if (a.size() == 3) return xn(XNode::Model, a, 0, "q0");
                throw std::runtime_error("CustomExpr: q0(x) or q0(x, md1, md2) expected");
            }
            if (a.size() < 4 || (a.size() - 1) % 3 != 0)
                throw std::runtime_error("CustomExpr: Flatte(m0, g..., (ma,mb)...) needs 1+3n args (n>=1)");
            // Flatte expanded to (A - iB)/(A^2 + B^2) (src/CustomExpr.cu:844-872)
            int n = (int)(a.size() - 1) / 3;
            XP sq = xn(XNode::Mul, {m, m});
            XP A = xn(XNode::Mul, {a[0], a[0]}), B = xn(XNode::Num, {}, 0.0);
            XP half = xn(XNode::Mul, {a[0], xn(XNode::Num, {}, 0.5)});
            for (int i = 0; i < n; ++i) {
                XP R = xn(XNode::Model, {sq, a[1 + n + 2 * i], a[2 + n + 2 * i]}, 0, "rho_re");
                XP I = xn(XNode::Model, {sq, a[1 + n + 2 * i], a[2 + n + 2 * i]}, 0, "rho_im");
                XP gw = xn(XNode::Mul, {a[1 + i], half});
                A = xn(XNode::Add, {A, xn(XNode::Mul, {gw, I})});
                B = xn(XNode::Sub, {B, xn(XNode::Mul, {gw, R})});
            }
            A = xn(XNode::Sub, {A, sq});
            XP Dn = xn(XNode::Add, {xn(XNode::Mul, {A, A}), xn(XNode::Mul, {B, B})});
            return xn(XNode::Add, {xn(XNode::Div, {A, Dn}), xn(XNode::Mul, {xn(XNode::Neg, {xn(XNode::Div, {B, Dn})}), xn(XNode::Model, {}, 0, "i")})});
        }
        for (size_t i = 0; i < params_.size(); ++i)
            if (params_[i] == s) return xn(XNode::Param, {}, 0, "", (int)i);
        throw std::runtime_error("CustomExpr: unknown identifier '" + s + "'");
    }
};

// ------------------------------------------------------------- generator
struct Gen {
    const Model& m;
    GeneratedModel out;
    std::map<std::tuple<int, unsigned, unsigned, unsigned>, int> slot_of;
    std::ostringstream body;
    std::ostringstream globals;
    int tmp = 0;
    int ntab = 0;

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
        const Group& G = m.groups[g];
        auto key = std::make_tuple(type, mask(G, a), b >= 0 ? mask(G, b) : 0u, c >= 0 ? mask(G, c) : 0u);
        auto it = slot_of.find(key);
        if (it != slot_of.end()) return it->second;
        int id = (int)out.slots.size();
        out.slots.push_back({type, g, a, b, c});
        slot_of[key] = id;
        return id;
    }
    std::string kv(int s) { return "kv[" + std::to_string(s) + "]"; }
    std::string t() { return "t" + std::to_string(tmp++); }

    // custom expression -> CJet<N> temporaries; returns variable name
    struct XCtx {
        int N;
        std::string mm, qq, md1, md2, L, d;
        std::vector<std::string> par;  // Jet<N> parameter names
        int gi = -1, d1 = -1, d2 = -1; // daughters for p1*/p2* variables (-1: zero)
    };
    std::string emitX(const XP& x, const XCtx& c)
    {
        std::string N = std::to_string(c.N);
        auto J = [&](const std::string& e) { return "cjr(" + e + ")"; };
        auto K = [&](const std::string& e) { return "cjr(jc<" + N + ">(" + e + "))"; };
        std::string r = t(), e;
        switch (x->k) {
        case XNode::Num: e = "cjc<" + N + ">(" + num(x->v) + ", 0.0)"; break;
        case XNode::Param: e = J(c.par[x->idx]); break;
        case XNode::Var: {
            const std::string& v = x->id;
            if (v == "m") e = K(c.mm);
            else if (v == "q") e = K(c.qq);
            else if (v == "L") e = K("(double)" + c.L);
            else if (v == "d") e = K(c.d);
            else if (v == "md1") e = J(c.md1);
            else if (v == "md2") e = J(c.md2);
            else {
                static const char* pv[] = {"p1p", "p1e", "p1costheta", "p1phi", "p2p", "p2e", "p2costheta", "p2phi"};
                static const int pt[] = {AG_K_P_, AG_K_E_, AG_K_CT_, AG_K_PHI_};
                for (int i = 0; i < 8; ++i)
                    if (v == pv[i]) e = K(c.gi < 0 ? std::string("0.0") : kv(slot(pt[i % 4], c.gi, i < 4 ? c.d1 : c.d2)));
            }
            break;
        }
        case XNode::Add: e = emitX(x->kids[0], c) + " + " + emitX(x->kids[1], c); break;
        case XNode::Sub: e = emitX(x->kids[0], c) + " - " + emitX(x->kids[1], c); break;
        case XNode::Mul: e = emitX(x->kids[0], c) + " * " + emitX(x->kids[1], c); break;
        case XNode::Div: { auto a = emitX(x->kids[0], c), b = emitX(x->kids[1], c); e = "c_div(" + a + ", " + b + ")"; break; }
        case XNode::Pow: { auto a = emitX(x->kids[0], c), b = emitX(x->kids[1], c); e = "c_pow(" + a + ", " + b + ")"; break; }
        case XNode::Neg: e = "-" + emitX(x->kids[0], c); break;
        case XNode::Func: e = "c_" + x->id + "(" + emitX(x->kids[0], c) + ")"; break;
        case XNode::Model: {
            const std::string& id = x->id;
            if (id == "i") e = "cjc<" + N + ">(0.0, 1.0)";
            else if (id == "q0") {
                auto a = emitX(x->kids[0], c), b = emitX(x->kids[1], c), d = emitX(x->kids[2], c);
                e = "c_q0(" + a + ", " + b + ", " + d + ")";
            } else if (id == "bf") {
                auto q = emitX(x->kids[1], c), q0 = emitX(x->kids[2], c), d = emitX(x->kids[3], c);
                e = "c_bf(" + std::to_string((int)x->kids[0]->v) + ", " + q + ", " + q0 + ", " + d + ".re.v)";
            } else if (id == "bw") {
                auto a = emitX(x->kids[0], c), b = emitX(x->kids[1], c), d = emitX(x->kids[2], c);
                e = "c_bw(" + a + ", " + b + ", " + d + ")";
            } else if (id == "bwr") {
                auto mm = emitX(x->kids[0], c), m0 = emitX(x->kids[1], c), g0 = emitX(x->kids[2], c);
                auto q = emitX(x->kids[4], c), q0 = emitX(x->kids[5], c);
                e = "c_bwr(" + mm + ", " + m0 + ", " + g0 + ", " + std::to_string((int)x->kids[3]->v) + ", " + q + ", " + q0 +
                    ", " + num(x->kids[6]->v) + ")";
            } else if (id == "rho_re" || id == "rho_im") {
                auto s = emitX(x->kids[0], c), a = emitX(x->kids[1], c), b = emitX(x->kids[2], c);
                e = "c_" + id + "(" + s + ", " + a + ", " + b + ")";
            }
            break;
        }
        }
        body << "      const CJet<" << N << "> " << r << " = " << e << ";\n";
        return r;
    }

    std::string table(const std::vector<double>& v)
    {
        std::string name = "ct_tab" + std::to_string(ntab++);
        globals << "__device__ const double " << name << "[" << std::max<size_t>(1, v.size()) << "] = {";
        for (size_t i = 0; i < v.size(); ++i) globals << (i ? ", " : "") << num(v[i]);
        if (v.empty()) globals << "0.0";
        globals << "};\n";
        return name;
    }

    void block(int bi, int& der)
    {
        const Block& b = m.blocks[bi];
        const Group& g = m.groups[b.group];
        // local fitted parameters
        std::vector<std::vector<std::string>> par(b.res.size());
        std::vector<int> loc_theta;
        for (size_t r = 0; r < b.res.size(); ++r)
            for (size_t p = 0; p < b.res[r].params.size(); ++p)
                if (b.res[r].theta[p] >= 0 && b.free_path) loc_theta.push_back(b.res[r].theta[p]);
        int N = (int)loc_theta.size();
        if (N > 16) throw std::runtime_error("more than 16 fitted parameters in one amplitude block");
        std::string NS = std::to_string(N);
        body << "  { // block " << bi << ":";
        for (const auto& r : b.res) body << " " << r.name;
        body << (b.free_path ? " (per-call)" : " (fixed)") << "\n";
        int k = 0;
        for (size_t r = 0; r < b.res.size(); ++r)
            for (size_t p = 0; p < b.res[r].params.size(); ++p) {
                std::string nm = "r" + std::to_string(r) + "p" + std::to_string(p);
                par[r].push_back(nm);
                int th = b.free_path ? b.res[r].theta[p] : -1;
                if (th >= 0) body << "    const Jet<" << NS << "> " << nm << " = jvar<" << NS << ">(th[" << th << "], " << k++ << ");\n";
                else body << "    const Jet<" << NS << "> " << nm << " = jc<" << NS << ">(" << num(b.res[r].params[p]) << ");\n";
            }
        for (int s = 0; s < g.nSL(); ++s) {
            int a = b.site + s;
            body << "    { // column " << a << "\n";
            body << "      CJet<" << NS << "> F = cjc<" << NS << ">(1.0, 0.0);\n";
            for (size_t ni = 0; ni < g.nodes.size(); ++ni) nodeFactor(b, g, (int)ni, s, N, par);
            body << "      Fr[" << a << "] = F.re.v; Fi[" << a << "] = F.im.v;\n";
            for (int q = 0; q < N; ++q)
                body << "      dFr[" << der + q << "] = F.re.d[" << q << "]; dFi[" << der + q << "] = F.im.d[" << q << "];\n";
            body << "    }\n";
            for (int q = 0; q < N; ++q) der_entries.push_back({a, loc_theta[q]});
            der += N;
        }
        body << "  }\n";
    }
    std::vector<std::pair<int, int>> der_entries;

    void nodeFactor(const Block& b, const Group& g, int ni, int s, int N, const std::vector<std::vector<std::string>>& par)
    {
        const ModelNode& n = g.nodes[ni];
        int gi = b.group;
        int L = n.sls[g.sl_combs[s][ni]].L;
        std::string NS = std::to_string(N);
        auto jcs = [&](const std::string& e) { return "jc<" + NS + ">(" + e + ")"; };
        if (b.free_path) {
            int match = -1;
            for (size_t r = 0; r < b.res.size(); ++r)
                if (b.res[r].particle_idx == n.mother && n.mass[0] <= 0) {
                    match = (int)r;
                    break;
                }
            std::string qq = kv(slot(AG_K_Q_, gi, n.mother, n.d1, n.d2));
            auto mdq = [&](int k) -> std::string {
                if (n.mass[k + 1] > 0) return jcs(num(n.mass[k + 1]));
                int di = k == 0 ? n.d1 : n.d2;
                for (size_t r = 0; r < b.res.size(); ++r)
                    if (b.res[r].particle_idx == di && !par[r].empty()) return par[r][0];
                return jcs(kv(slot(AG_K_MASS_, gi, di)));
            };
            std::string md1 = mdq(0), md2 = mdq(1);
            if (match < 0) {
                if (!n.has_bf) return;
                std::string m0q;
                m0q = jcs(num(n.mass[0] > 0 ? n.mass[0] : 1.0));
                body << "      F = F * cjr(ls_bf<" << NS << ">(" << L << ", " << jcs(qq) << ", ls_breakup<" << NS << ">(" << m0q
                     << ", " << md1 << ", " << md2 << "), " << num(n.bf_d) << "));\n";
                return;
            }
            const ResInstance& R = b.res[match];
            const auto& P = par[match];
            std::string mm = kv(slot(AG_K_MASS_, gi, n.mother));
            std::string m0 = P.empty() ? jcs("1.0") : P[0];
            auto dep = [&](int k) -> std::string {
                if (R.md_src[k] == MassSource::Fixed) return jcs(num(R.md_fixed[k]));
                if (R.md_src[k] == MassSource::M0Param) return m0;
                return k == 0 ? md1 : md2;
            };
            std::string q0r = "ls_q0<" + NS + ">(" + m0 + ", " + dep(0) + ", " + dep(1) + ")";
            std::string bfx = R.has_bf ? " * cjr(ls_bf<" + NS + ">(" + std::to_string(L) + ", " + jcs(qq) + ", q0r, " + num(R.d) + "))" : "";
            body << "      {\n        const Jet<" << NS << "> q0r = " << q0r << ";\n";
            switch (R.type) {
            case ModelType::BWR:
                body << "        F = F * (ls_bwr<" << NS << ">(" << jcs(mm) << ", " << P[0] << ", " << P[1] << ", " << R.Lmin << ", "
                     << jcs(qq) << ", q0r, " << num(R.has_bf ? R.d : 0.0) << ")" << bfx << ");\n";
                break;
            case ModelType::BW:
                body << "        F = F * ls_bw<" << NS << ">(" << jcs(mm) << ", " << P[0] << ", " << P[1] << ");\n";
                break;
            case ModelType::ONE:
                if (R.has_bf) body << "        F = F * cjr(ls_bf<" << NS << ">(" << L << ", " << jcs(qq) << ", q0r, " << num(R.d) << "));\n";
                break;
            case ModelType::Flatte: {
                int nch = (int)R.channels.size();
                std::vector<double> ch;
                for (auto& c : R.channels) {
                    ch.push_back(c.first);
                    ch.push_back(c.second);
                }
                body << "        const Jet<" << NS << "> gg[" << std::max(1, nch) << "] = {";
                for (int i = 0; i < std::max(1, nch); ++i)
                    body << (i ? ", " : "") << ((size_t)(1 + i) < P.size() ? P[1 + i] : jcs("0.0"));
                body << "};\n        F = F * (ls_flatte<" << NS << ", " << nch << ">(" << jcs(mm) << ", " << P[0] << ", gg, "
                     << table(ch) << ")" << bfx << ");\n";
                break;
            }
            case ModelType::GS: {
                double mpi = R.channels.empty() ? 0.1396 : R.channels[0].first;
                body << "        F = F * (ls_gs<" << NS << ">(" << jcs(mm) << ", " << jcs(qq) << ", " << P[0] << ", " << P[1]
                     << ", q0r, " << num(mpi) << ")" << bfx << ");\n";
                break;
            }
            case ModelType::Custom: {
                XParser ps(R.options.at("expr"), R.param_names);
                XP x = ps.parse();
                XCtx c;
                c.N = N;
                c.mm = mm;
                c.qq = qq;
                c.md1 = md1;
                c.md2 = md2;
                c.L = std::to_string(L);
                c.d = num(n.bf_d);
                c.par = P;
                c.gi = gi;
                c.d1 = n.d1;
                c.d2 = n.d2;
                std::string r = emitX(x, c);
                body << "        F = F * " << r << ";\n";
                break;
            }
            case ModelType::Interp: {
                std::string tb = table(R.aux);
                body << "        { double fr, fi; ls_interp(" << tb << ", " << mm << ", fr, fi); F = F * cjc<" << NS << ">(fr, fi); }\n";
                break;
            }
            case ModelType::Hist: {
                std::string tb = table(R.aux);
                body << "        F = F * cjc<" << NS << ">(ls_hist(" << mm << ", " << tb << "), 0.0);\n";
                break;
            }
            }
            body << "      }\n";
            return;
        }
        // ---- fixed-parameter block ----
        std::string mm = kv(slot(AG_K_MASS_, gi, n.mother));
        std::string qq = kv(slot(AG_K_QRAW_, gi, n.mother, n.d1, n.d2));
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
        double q0 = std::sqrt((mo * mo - std::pow(ma + mb, 2)) * (mo * mo - std::pow(ma - mb, 2))) / 2 / mo;
        std::string Q = jcs(qq), Q0 = jcs(num(q0));
        if (ni == 0) {
            if (n.has_bf) body << "      F = F * cjr(ls_bf<" << NS << ">(" << L << ", " << Q << ", " << Q0 << ", " << num(n.bf_d) << "));\n";
            return;
        }
        if (match < 0) return;
        const ResInstance& R = b.res[match];
        const auto& P = par[match];
        std::string bfx = n.has_bf ? " * cjr(ls_bf<" + NS + ">(" + std::to_string(L) + ", " + Q + ", " + Q0 + ", " + num(n.bf_d) + "))" : "";
        switch (R.type) {
        case ModelType::BWR:
            body << "      F = F * (ls_bwr<" << NS << ">(" << jcs(mm) << ", " << P[0] << ", " << P[1] << ", " << n.l_min << ", " << Q
                 << ", " << Q0 << ", " << num(n.has_bf ? n.bf_d : 0.0) << ")" << bfx << ");\n";
            break;
        case ModelType::BW: body << "      F = F * ls_bw<" << NS << ">(" << jcs(mm) << ", " << P[0] << ", " << P[1] << ");\n"; break;
        case ModelType::ONE: if (n.has_bf) body << "      F = F * cjr(ls_bf<" << NS << ">(" << L << ", " << Q << ", " << Q0 << ", " << num(n.bf_d) << "));\n"; break;
        case ModelType::Flatte: {
            int nch = (int)R.channels.size();
            std::vector<double> ch;
            for (auto& c : R.channels) {
                ch.push_back(c.first);
                ch.push_back(c.second);
            }
            body << "      { const Jet<" << NS << "> gg[" << std::max(1, nch) << "] = {";
            for (int i = 0; i < std::max(1, nch); ++i) body << (i ? ", " : "") << ((size_t)(1 + i) < P.size() ? P[1 + i] : jcs("0.0"));
            body << "};\n        F = F * (ls_flatte_fixed<" << NS << ", " << nch << ">(" << jcs(mm) << ", " << P[0] << ", gg, "
                 << table(ch) << ")" << bfx << "); }\n";
            break;
        }
        case ModelType::Hist: body << "      F = F * cjc<" << NS << ">(ls_hist(" << mm << ", " << table(R.aux) << "), 0.0);\n"; break;
        case ModelType::Custom: {
            // value segment with md1 = md2 = 0, no daughter kinematics, at most 3 params
            XParser ps(R.options.at("expr"), R.param_names);
            XP x = ps.parse();
            XCtx c;
            c.N = N;
            c.mm = mm;
            c.qq = qq;
            c.md1 = jcs("0.0");
            c.md2 = jcs("0.0");
            c.L = std::to_string(L);
            c.d = num(n.bf_d);
            for (size_t i = 0; i < P.size(); ++i) c.par.push_back(i < 3 ? P[i] : jcs("0.0"));
            body << "      {\n";
            std::string r = emitX(x, c);
            body << "      F = F * " << r << ";\n      }\n";
            break;
        }
        default: break;  // GS / Interp: no fixed-parameter factor in the reference
        }
    }

    // slot type ids mirrored from angular.cuh
    static constexpr int AG_K_MASS_ = 0, AG_K_Q_ = 1, AG_K_QRAW_ = 2, AG_K_P_ = 3, AG_K_E_ = 4, AG_K_CT_ = 5, AG_K_PHI_ = 6;

    void run()
    {
        out.group_plane0.clear();
        int pl = 0;
        for (const auto& g : m.groups) {
            out.group_plane0.push_back(pl);
            pl += g.nSL();
        }
        out.nplane = pl;
        int der = 0;
        for (size_t b = 0; b < m.blocks.size(); ++b) block((int)b, der);
        out.nder = der;
        std::ostringstream h;
        h << "// generated by ctpwa_b200 codegen: model-specific lineshape products\n#pragma once\n";
        h << "#define M_NA " << m.nAmp() << "\n#define M_NPOL " << m.npol << "\n#define M_NPLANE " << out.nplane
          << "\n#define M_NKIN " << out.slots.size() << "\n#define M_NTH " << m.nTheta() << "\n#define M_NDER " << der << "\n";
        h << "__device__ __forceinline__ double ct_nan() { return __longlong_as_double(0x7ff8000000000000LL); }\n";
        h << "__device__ __forceinline__ double ct_inf() { return __longlong_as_double(0x7ff0000000000000LL); }\n";
        h << "__device__ __forceinline__ int col_plane(int a) {\n  switch (a) {\n";
        for (const auto& b : m.blocks)
            for (int s = 0; s < m.groups[b.group].nSL(); ++s)
                h << "  case " << b.site + s << ": return " << out.group_plane0[b.group] + s << ";\n";
        h << "  default: return 0;\n  }\n}\n";
        h << "__device__ __forceinline__ int der_col(int k) {\n  switch (k) {\n";
        for (size_t k = 0; k < der_entries.size(); ++k) h << "  case " << k << ": return " << der_entries[k].first << ";\n";
        h << "  default: return 0;\n  }\n}\n";
        h << "__device__ __forceinline__ int der_th(int k) {\n  switch (k) {\n";
        for (size_t k = 0; k < der_entries.size(); ++k) h << "  case " << k << ": return " << der_entries[k].second << ";\n";
        h << "  default: return 0;\n  }\n}\n";
        h << globals.str();
        h << "__device__ __forceinline__ void model_columns(const double* __restrict__ kv, const double* __restrict__ th,\n"
             "    double* Fr, double* Fi, double* dFr, double* dFi)\n{\n  (void)kv; (void)th; (void)dFr; (void)dFi;\n";
        h << body.str() << "}\n";
        out.header = h.str();
    }
};

}  // namespace

GeneratedModel generateModel(const Model& m)
{
    Gen g(m);
    g.run();
    return g.out;
}

void checkCustomExpr(const std::string& expr, const std::vector<std::string>& params)
{
    XParser p(expr, params);
    p.parse();
}

}  // namespace ctpwa
