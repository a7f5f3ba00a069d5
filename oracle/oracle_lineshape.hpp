// Oracle test infrastructure (not product code): FP64 restatement of the
// reference lineshapes and of its custom-lineshape expression language,
// evaluated on dual numbers so that parameter derivatives come out exactly.
//
// Lineshapes follow include/ResModel.cuh (Bf :184-211, BWR :214-223,
// BW :398-405, Flatte :419-451, computeQ0AD :85-95, computeNodeFactor
// :103-181, lookupHistTable :66-82, interpEval :248-293) and
// src/ResModel.cu:376-588 (buildModelAST: BWR x Bf, Flatte x Bf, GS x Bf, ONE).
// The expression language follows src/CustomExpr.cu (tokenizer :236-278,
// recursive-descent parser :280-528, buildFlatteAST :844-872, device
// interpreter semantics :999-1221) and include/CustomExpr.cuh:6-27.
#pragma once

#include "oracle_dual.hpp"

#include <cctype>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- lineshapes
inline D bfPoly(int L, const D& z)
{
    D z2 = z * z;
    switch (L) {
    case 0: return D(1.0);
    case 1: return D(1.0) + z2;
    case 2: return D(9.0) + D(3.0) * z2 + z2 * z2;
    case 3: return powi(z, 6) + D(6.0) * powi(z, 4) + D(45.0) * z2 + D(225.0);
    case 4: return powi(z, 8) + D(10.0) * powi(z, 6) + D(135.0) * powi(z, 4) + D(1575.0) * z2 + D(11025.0);
    case 5:
        return powi(z, 10) + D(15.0) * powi(z, 8) + D(315.0) * powi(z, 6) + D(6300.0) * powi(z, 4) + D(99225.0) * z2 +
               D(893025.0);
    case 6:
        return powi(z, 12) + D(21.0) * powi(z, 10) + D(630.0) * powi(z, 8) + D(17325.0) * powi(z, 6) +
               D(363825.0) * powi(z, 4) + D(6185025.0) * z2 + D(540326025.0);
    default: return D(1.0);
    }
}

// Blatt-Weisskopf barrier ratio Bf(L, q, q0, d) = sqrt(N_L(q0 d) / N_L(q d)).
inline D Bf(int L, const D& q, const D& q0, double d)
{
    if (L <= 0 || L > 6) return D(1.0);
    return sqrt(bfPoly(L, q0 * D(d)) / bfPoly(L, q * D(d)));
}

inline D breakup(const D& m, const D& m1, const D& m2)  // AmpGen breakup_momentum
{
    D qs = (m * m - (m1 + m2) * (m1 + m2)) * (m * m - (m1 - m2) * (m1 - m2));
    if (qs.v <= 0.0) return D(0.0);
    return sqrt(qs) / (D(2.0) * m);
}

inline D q0AD(const D& m0, const D& m1, const D& m2)  // computeQ0AD
{
    D s = m1 + m2, dd = m1 - m2, m0s = m0 * m0;
    D q0s = (m0s - s * s) * (m0s - dd * dd) / (D(4.0) * m0s);
    if (q0s.v < 0.0) return D(0.0);
    return sqrt(q0s);
}

inline CD BWR(const D& m, const D& m0, const D& g0, int L, const D& q, const D& q0, double d)
{
    D bf = Bf(L, q, q0, d);
    D gam = g0 * powi(q / q0, 2 * L + 1) * (m0 / m) * (bf * bf);
    D x = m0 * m0 - m * m, y = m0 * gam, s = x * x + y * y;
    return CD(x / s, y / s);
}

inline CD BW(const D& m, const D& m0, const D& g0)
{
    D x = m0 * m0 - m * m, y = m0 * g0, s = x * x + y * y;
    return CD(x / s, y / s);
}

// rho_i = csqrt(1 - (ma+mb)^2/s) * sqrt(max(0, 1 - (ma-mb)^2/s)); value only
inline void flatteRho(double s, double ma, double mb, double& re, double& im)
{
    double S = (ma + mb) * (ma + mb), Dd = (ma - mb) * (ma - mb);
    double f1 = 1.0 - S / s, f1r, f1i;
    if (f1 >= 0.0) {
        f1r = std::sqrt(f1);
        f1i = 0.0;
    } else {
        f1r = 0.0;
        f1i = std::sqrt(-f1);
    }
    double f2s = 1.0 - Dd / s;
    double f2 = f2s > 0.0 ? std::sqrt(f2s) : 0.0;
    re = f1r * f2;
    im = f1i * f2;
}

// Flatte (FlatteC convention) expanded as in buildFlatteAST: F = (A - iB)/D.
inline CD flatte(const D& m, const D& m0, const std::vector<D>& g, const std::vector<double>& ch)
{
    D s = m * m, A = m0 * m0, B(0.0), half = m0 * D(0.5);
    for (size_t i = 0; i < g.size(); ++i) {
        double rr, ri;
        flatteRho(s.v, ch[2 * i], ch[2 * i + 1], rr, ri);
        D gw = g[i] * half;
        A = A + gw * D(ri);
        B = B - gw * D(rr);
    }
    A = A - s;
    D den = A * A + B * B;
    return CD(A / den, -(B / den));
}

// Gounaris-Sakurai as built by buildModelAST (src/ResModel.cu:484-555).
inline CD gs(const D& m, const D& q, const D& m0, const D& g0, const D& q0, double mpi)
{
    const double pi = 3.14159265358979323846;
    D hm = D(2.0 / pi) * ((q / m) * log((m + D(2.0) * q) / D(2.0 * mpi)));
    D q02 = q0 * q0, q03 = q02 * q0;
    D mpi2(mpi * mpi);
    D la = log((m0 + D(2.0) * q0) / D(2.0 * mpi));
    D dv = (D(3.0 / pi) * (mpi2 / q02)) * la + m0 / (D(2.0 * pi) * q0) - (mpi2 * m0) / (D(pi) * q03);
    D h0 = D(2.0 / pi) * ((q0 / m0) * la);
    D dh0 = h0 * (D(1.0) / (D(8.0) * q02) - D(1.0) / (D(2.0) * (m0 * m0))) + D(1.0) / (D(2.0 * pi) * (m0 * m0));
    D qr = q / q0;
    D gam = (g0 * (qr * qr * qr)) * (m0 / m);
    D f = (g0 * ((m0 * m0) / q03)) * ((q * q) * (hm - h0) + ((m0 * m0 - m * m) * q02) * dh0);
    D num = D(1.0) + (dv * g0) / m0;
    D dre = (m0 * m0 - m * m) + f;
    D dim = -(m0 * gam);
    D dsq = dre * dre + dim * dim;
    return CD((num * dre) / dsq, -((num * dim) / dsq));
}

inline double histLookup(double m, const std::vector<double>& aux)
{
    if (aux.size() < 3 || !(m >= 0.0)) return 0.0;
    double lo = aux[0], hi = aux[1];
    int n = (int)aux[2];
    const double* v = aux.data() + 3;
    if (n < 2 || hi <= lo) return 0.0;
    if (m <= lo) return v[0];
    if (m >= hi) return v[n - 1];
    double x = (m - lo) / (hi - lo) * n;
    if (x < 0.0) x = 0.0;
    if (x >= (double)(n - 1)) x = (double)(n - 2);
    int i = (int)x;
    double fr = x - i;
    return v[i] * (1.0 - fr) + v[i + 1] * fr;
}

inline double interp1(const double* y, int i, double fr, int method, int N)
{
    switch (method) {
    case 1: return y[i] + (y[i + 1] - y[i]) * fr;
    case 2: {
        double y0 = (i > 0) ? y[i - 1] : y[i] - (y[i + 1] - y[i]);
        double y1 = y[i], y2 = y[i + 1];
        double y3 = (i + 2 < N) ? y[i + 2] : y[i + 1] + (y[i + 1] - y[i]);
        double f2 = fr * fr, f3 = f2 * fr;
        return 0.5 * ((2 * y1) + (-y0 + y2) * fr + (2 * y0 - 5 * y1 + 4 * y2 - y3) * f2 + (-y0 + 3 * y1 - 3 * y2 + y3) * f3);
    }
    default: return y[i];
    }
}

inline void interpLookup(const std::vector<double>& t, double x, double& Fr, double& Fi)
{
    Fr = Fi = 0.0;
    if (t.size() < 2) return;
    int hdr = (int)t[0];
    int method = hdr >= 0 ? hdr : -(hdr + 1);
    int N = (int)t[1];
    int i;
    double fr;
    const double *re, *im;
    if (hdr >= 0) {
        double xmin = t[2], dx = t[3];
        re = t.data() + 4;
        im = t.data() + 4 + N;
        double pos = (x - xmin) / dx;
        i = (int)pos;
        if (i < 0) { i = 0; fr = 0.0; }
        else if (i >= N - 1) { i = N - 2; fr = 1.0; }
        else fr = pos - (double)i;
    } else {
        const double* xv = t.data() + 2;
        re = t.data() + 2 + N;
        im = t.data() + 2 + 2 * N;
        int lo = 0, hi = N - 1;
        while (lo < hi - 1) {
            int mid = (lo + hi) / 2;
            if (x < xv[mid]) hi = mid;
            else lo = mid;
        }
        i = lo;
        if (i < 0) { i = 0; fr = 0.0; }
        else if (i >= N - 1) { i = N - 2; fr = 1.0; }
        else fr = (x - xv[i]) / (xv[i + 1] - xv[i]);
        if (method == 2) method = 0;
    }
    Fr = interp1(re, i, fr, method, N);
    Fi = interp1(im, i, fr, method, N);
}

// ------------------------------------------------------- expression language
enum VarId { V_M = 0, V_Q, V_Q0, V_L, V_D, V_MD1, V_MD2, V_P1P, V_P1E, V_P1CT, V_P1PHI, V_P2P, V_P2E, V_P2CT, V_P2PHI, V_N };
enum FuncId { F_EXP, F_LOG, F_SIN, F_COS, F_SQRT, F_ABS, F_RE, F_IM, F_CONJ, F_CSQRT };
enum ModelId { M_Q0, M_BF, M_BW, M_BWR, M_RHO_RE, M_RHO_IM, M_I };

struct Expr {
    enum Kind { Num, Var, Param, Add, Sub, Mul, Div, Pow, Neg, Func, Model } kind = Num;
    double num = 0.0;
    int id = 0;
    std::vector<std::shared_ptr<Expr>> kids;
};
using ExprP = std::shared_ptr<Expr>;

inline ExprP mk(Expr::Kind k, std::vector<ExprP> kids = {}, double num = 0.0, int id = 0)
{
    auto e = std::make_shared<Expr>();
    e->kind = k;
    e->kids = std::move(kids);
    e->num = num;
    e->id = id;
    return e;
}

// The reference simplifies every parsed expression before it compiles or
// evaluates it (simplify, src/CustomExpr.cu:785-835; called at :1281 and
// src/ResModel.cu:569): bottom-up, 0+x / x+0 -> x, x-0 -> x, 0*x / x*0 -> 0,
// 1*x / x*1 -> x, 0/x -> 0, x/1 -> x, x^1 -> x, 1^x -> 1, 0^x -> 0,
// -(-x) -> x, -c -> (-c), and two numbers fold (a power by real std::pow).
inline bool exprNum(const ExprP& e) { return e->kind == Expr::Num; }
inline bool exprIs(const ExprP& e, double v) { return e->kind == Expr::Num && e->num == v; }
inline ExprP simplifyRef(const ExprP& e)
{
    auto out = std::make_shared<Expr>(*e);
    for (auto& k : out->kids) k = simplifyRef(k);
    const auto& k = out->kids;
    switch (out->kind) {
    case Expr::Add:
        if (exprIs(k[0], 0.0)) return k[1];
        if (exprIs(k[1], 0.0)) return k[0];
        if (exprNum(k[0]) && exprNum(k[1])) return mk(Expr::Num, {}, k[0]->num + k[1]->num);
        break;
    case Expr::Sub:
        if (exprIs(k[1], 0.0)) return k[0];
        if (exprNum(k[0]) && exprNum(k[1])) return mk(Expr::Num, {}, k[0]->num - k[1]->num);
        break;
    case Expr::Mul:
        if (exprIs(k[0], 0.0) || exprIs(k[1], 0.0)) return mk(Expr::Num, {}, 0.0);
        if (exprIs(k[0], 1.0)) return k[1];
        if (exprIs(k[1], 1.0)) return k[0];
        if (exprNum(k[0]) && exprNum(k[1])) return mk(Expr::Num, {}, k[0]->num * k[1]->num);
        break;
    case Expr::Div:
        if (exprIs(k[0], 0.0)) return mk(Expr::Num, {}, 0.0);
        if (exprIs(k[1], 1.0)) return k[0];
        if (exprNum(k[0]) && exprNum(k[1]) && k[1]->num != 0.0) return mk(Expr::Num, {}, k[0]->num / k[1]->num);
        break;
    case Expr::Pow:
        if (exprIs(k[1], 1.0)) return k[0];
        if (exprIs(k[0], 1.0)) return mk(Expr::Num, {}, 1.0);
        if (exprIs(k[0], 0.0)) return mk(Expr::Num, {}, 0.0);
        if (exprNum(k[0]) && exprNum(k[1])) return mk(Expr::Num, {}, std::pow(k[0]->num, k[1]->num));
        break;
    case Expr::Neg:
        if (k[0]->kind == Expr::Neg) return k[0]->kids[0];
        if (exprNum(k[0])) return mk(Expr::Num, {}, -k[0]->num);
        break;
    default: break;
    }
    return out;
}

class ExprParser {
public:
    ExprParser(const std::string& s, const std::vector<std::string>& params) : params_(params)
    {
        tokenize(s);
    }
    ExprP parse()
    {
        ExprP e = expr();
        if (toks_[pos_].t != Tok::End) throw std::runtime_error("CustomExpr: trailing tokens");
        return simplifyRef(e);
    }

private:
    struct Tok {
        enum T { Num, Ident, Op, LP, RP, Comma, End } t;
        double v = 0;
        std::string s;
    };
    std::vector<Tok> toks_;
    size_t pos_ = 0;
    const std::vector<std::string>& params_;

    void tokenize(const std::string& s)
    {
        size_t i = 0;
        while (i < s.size()) {
            char c = s[i];
            if (std::isspace((unsigned char)c)) { ++i; continue; }
            if (std::isdigit((unsigned char)c) || c == '.') {
                if (c == '1' && i + 1 < s.size() && (s[i + 1] == 'j' || s[i + 1] == 'i')) {
                    toks_.push_back({Tok::Ident, 0, "1j"});
                    i += 2;
                    continue;
                }
                size_t j = i;
                while (j < s.size() && (std::isdigit((unsigned char)s[j]) || s[j] == '.' || s[j] == 'e' || s[j] == 'E' ||
                                        ((s[j] == '+' || s[j] == '-') && j > i && (s[j - 1] == 'e' || s[j - 1] == 'E'))))
                    ++j;
                toks_.push_back({Tok::Num, std::stod(s.substr(i, j - i)), ""});
                i = j;
                continue;
            }
            if (std::isalpha((unsigned char)c) || c == '_') {
                size_t j = i;
                while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
                toks_.push_back({Tok::Ident, 0, s.substr(i, j - i)});
                i = j;
                continue;
            }
            if (c == '+' || c == '-' || c == '*' || c == '/' || c == '^') { toks_.push_back({Tok::Op, 0, std::string(1, c)}); ++i; continue; }
            if (c == '(') { toks_.push_back({Tok::LP, 0, ""}); ++i; continue; }
            if (c == ')') { toks_.push_back({Tok::RP, 0, ""}); ++i; continue; }
            if (c == ',') { toks_.push_back({Tok::Comma, 0, ""}); ++i; continue; }
            throw std::runtime_error(std::string("CustomExpr: unexpected char '") + c + "'");
        }
        toks_.push_back({Tok::End, 0, ""});
    }
    const Tok& peek() const { return toks_[pos_]; }
    const Tok& next() { return toks_[pos_++]; }
    bool isOp(const char* o) const { return peek().t == Tok::Op && peek().s == o; }

    ExprP expr()
    {
        ExprP l = term();
        while (isOp("+") || isOp("-")) {
            bool add = next().s == "+";
            ExprP r = term();
            l = mk(add ? Expr::Add : Expr::Sub, {l, r});
        }
        return l;
    }
    ExprP term()
    {
        ExprP l = factor();
        while (isOp("*") || isOp("/")) {
            bool mul = next().s == "*";
            ExprP r = factor();
            l = mk(mul ? Expr::Mul : Expr::Div, {l, r});
        }
        return l;
    }
    ExprP factor()
    {
        ExprP b = unary();
        if (isOp("^")) {
            next();
            return mk(Expr::Pow, {b, factor()});
        }
        return b;
    }
    ExprP unary()
    {
        if (isOp("-")) {
            next();
            return mk(Expr::Neg, {unary()});
        }
        if (isOp("+")) {
            next();
            return unary();
        }
        return primary();
    }
    std::vector<ExprP> args()
    {
        if (peek().t != Tok::LP) throw std::runtime_error("CustomExpr: function needs (");
        next();
        std::vector<ExprP> a;
        if (peek().t == Tok::RP) {
            next();
            return a;
        }
        while (true) {
            a.push_back(expr());
            if (peek().t == Tok::Comma) { next(); continue; }
            break;
        }
        if (peek().t != Tok::RP) throw std::runtime_error("CustomExpr: missing )");
        next();
        return a;
    }
    ExprP q0node()
    {
        return mk(Expr::Model, {params_.empty() ? mk(Expr::Num, {}, 1.0) : mk(Expr::Param, {}, 0, 0), mk(Expr::Var, {}, 0, V_MD1),
                                mk(Expr::Var, {}, 0, V_MD2)},
                  0, M_Q0);
    }
    ExprP primary()
    {
        Tok t = peek();
        if (t.t == Tok::Num) {
            next();
            return mk(Expr::Num, {}, t.v);
        }
        if (t.t == Tok::LP) {
            next();
            ExprP e = expr();
            if (peek().t != Tok::RP) throw std::runtime_error("CustomExpr: missing )");
            next();
            return e;
        }
        if (t.t != Tok::Ident) throw std::runtime_error("CustomExpr: unexpected token");
        next();
        const std::string& s = t.s;
        if (s == "1j") return mk(Expr::Model, {}, 0, M_I);
        if (s == "pi") return mk(Expr::Num, {}, 3.14159265358979323846);
        static const std::map<std::string, int> vars = {
            {"m", V_M},     {"q", V_Q},       {"L", V_L},        {"d", V_D},      {"p1p", V_P1P},
            {"p1e", V_P1E}, {"p1costheta", V_P1CT}, {"p1phi", V_P1PHI}, {"p2p", V_P2P}, {"p2e", V_P2E},
            {"p2costheta", V_P2CT}, {"p2phi", V_P2PHI}};
        if (s == "q0" && peek().t != Tok::LP) return q0node();
        auto vi = vars.find(s);
        if (vi != vars.end()) return mk(Expr::Var, {}, 0, vi->second);
        static const std::map<std::string, int> funcs = {
            {"exp", F_EXP},   {"log", F_LOG},   {"ln", F_LOG},     {"sin", F_SIN},  {"cos", F_COS},
            {"sqrt", F_SQRT}, {"abs", F_ABS},   {"Re", F_RE},      {"real", F_RE},  {"Im", F_IM},
            {"imag", F_IM},   {"conj", F_CONJ}, {"csqrt", F_CSQRT}};
        auto fi = funcs.find(s);
        if (fi != funcs.end()) {
            if (peek().t != Tok::LP) throw std::runtime_error("CustomExpr: function '" + s + "' needs (");
            next();
            ExprP a = expr();
            if (peek().t != Tok::RP) throw std::runtime_error("CustomExpr: missing )");
            next();
            return mk(Expr::Func, {a}, 0, fi->second);
        }
        if (s == "BW" || s == "BWR" || s == "Bf" || s == "Flatte" || (s == "q0" && peek().t == Tok::LP)) {
            auto a = args();
            if (s == "BW") {
                if (a.size() != 2) throw std::runtime_error("CustomExpr: BW(m0, w0) needs exactly 2 args");
                return mk(Expr::Model, {mk(Expr::Var, {}, 0, V_M), a[0], a[1]}, 0, M_BW);
            }
            if (s == "BWR") {
                if (a.size() < 2 || a.size() > 4) throw std::runtime_error("CustomExpr: BWR(m0, g0[, L, d]) needs 2~4 args");
                if (a.size() >= 3 && a[2]->kind != Expr::Num) throw std::runtime_error("CustomExpr: BWR L must be a literal");
                if (a.size() >= 4 && a[3]->kind != Expr::Num) throw std::runtime_error("CustomExpr: BWR d must be a literal");
                double Lv = a.size() >= 3 ? a[2]->num : 1.0, dv = a.size() >= 4 ? a[3]->num : 3.0;
                return mk(Expr::Model, {mk(Expr::Var, {}, 0, V_M), a[0], a[1], mk(Expr::Num, {}, Lv), mk(Expr::Var, {}, 0, V_Q), q0node(), mk(Expr::Num, {}, dv)}, 0, M_BWR);
            }
            if (s == "Bf") {
                if (a.size() != 4) throw std::runtime_error("CustomExpr: Bf(L, q, q0, d) needs exactly 4 args");
                if (a[0]->kind != Expr::Num) throw std::runtime_error("CustomExpr: Bf L must be a literal");
                return mk(Expr::Model, a, 0, M_BF);
            }
            if (s == "q0") {
                if (a.size() == 1) return mk(Expr::Model, {a[0], mk(Expr::Var, {}, 0, V_MD1), mk(Expr::Var, {}, 0, V_MD2)}, 0, M_Q0);
                if (a.size() == 3) return mk(Expr::Model, a, 0, M_Q0);
                throw std::runtime_error("CustomExpr: q0(x) or q0(x, md1, md2) expected");
            }
            // Flatte(m0, g_0..g_{n-1}, (ma, mb)_0..) expanded (src/CustomExpr.cu:844-872)
            if (a.size() < 4 || (a.size() - 1) % 3 != 0)
                throw std::runtime_error("CustomExpr: Flatte(m0, g..., (ma,mb)...) needs 1+3n args (n>=1)");
            int n = (int)(a.size() - 1) / 3;
            ExprP m = mk(Expr::Var, {}, 0, V_M);
            ExprP sq = mk(Expr::Mul, {m, m});
            ExprP A = mk(Expr::Mul, {a[0], a[0]});
            ExprP B = mk(Expr::Num, {}, 0.0);
            ExprP half = mk(Expr::Mul, {a[0], mk(Expr::Num, {}, 0.5)});
            for (int i = 0; i < n; ++i) {
                ExprP R = mk(Expr::Model, {sq, a[1 + n + 2 * i], a[2 + n + 2 * i]}, 0, M_RHO_RE);
                ExprP I = mk(Expr::Model, {sq, a[1 + n + 2 * i], a[2 + n + 2 * i]}, 0, M_RHO_IM);
                ExprP gw = mk(Expr::Mul, {a[1 + i], half});
                A = mk(Expr::Add, {A, mk(Expr::Mul, {gw, I})});
                B = mk(Expr::Sub, {B, mk(Expr::Mul, {gw, R})});
            }
            A = mk(Expr::Sub, {A, sq});
            ExprP Dn = mk(Expr::Add, {mk(Expr::Mul, {A, A}), mk(Expr::Mul, {B, B})});
            return mk(Expr::Add, {mk(Expr::Div, {A, Dn}), mk(Expr::Mul, {mk(Expr::Neg, {mk(Expr::Div, {B, Dn})}), mk(Expr::Model, {}, 0, M_I)})});
        }
        for (size_t i = 0; i < params_.size(); ++i)
            if (params_[i] == s) return mk(Expr::Param, {}, 0, (int)i);
        throw std::runtime_error("CustomExpr: unknown identifier '" + s + "'");
    }
};

// Evaluation on complex duals with the reference interpreter's conventions
// (division by |b|^2 = 0 uses 1e-30, log|0| uses 1e-30, pow = exp(e log b),
// sqrt = principal complex square root).
inline CD cdiv(const CD& a, const CD& b)
{
    D s = b.re * b.re + b.im * b.im;
    if (s.v == 0.0) s = D(1e-30);
    return CD((a.re * b.re + a.im * b.im) / s, (a.im * b.re - a.re * b.im) / s);
}
inline CD cexp(const CD& a)
{
    D e = exp(a.re);
    return CD(e * cos(a.im), e * sin(a.im));
}
inline CD clog(const CD& a)
{
    D r = sqrt(a.re * a.re + a.im * a.im);
    if (r.v == 0.0) r = D(1e-30);
    return CD(log(r), atan2(a.im, a.re));
}
inline CD csqrtD(const CD& a)
{
    D r = sqrt(a.re * a.re + a.im * a.im);
    D re = sqrt((r + a.re) * D(0.5));
    D im = sqrt((r - a.re) * D(0.5));
    if (a.im.v < 0) im = -im;
    return CD(re, im);
}

struct EvalVars {
    D v[V_N];
    int L = 0;
};

inline CD evalExpr(const Expr& e, const EvalVars& vars, const std::vector<D>& params)
{
    switch (e.kind) {
    case Expr::Num: return CD(D(e.num));
    case Expr::Var: return CD(e.id == V_L ? D((double)vars.L) : vars.v[e.id]);
    case Expr::Param: return CD(params[e.id]);
    case Expr::Add: return evalExpr(*e.kids[0], vars, params) + evalExpr(*e.kids[1], vars, params);
    case Expr::Sub: return evalExpr(*e.kids[0], vars, params) - evalExpr(*e.kids[1], vars, params);
    case Expr::Mul: return evalExpr(*e.kids[0], vars, params) * evalExpr(*e.kids[1], vars, params);
    case Expr::Div: return cdiv(evalExpr(*e.kids[0], vars, params), evalExpr(*e.kids[1], vars, params));
    case Expr::Pow: {
        CD b = evalExpr(*e.kids[0], vars, params), x = evalExpr(*e.kids[1], vars, params);
        return cexp(x * clog(b));
    }
    case Expr::Neg: return -evalExpr(*e.kids[0], vars, params);
    case Expr::Func: {
        CD a = evalExpr(*e.kids[0], vars, params);
        switch (e.id) {
        case F_EXP: return cexp(a);
        case F_LOG: return clog(a);
        case F_SIN: {
            D ep = exp(a.im), em = exp(-a.im);
            return CD(sin(a.re) * (ep + em) * D(0.5), cos(a.re) * (ep - em) * D(0.5));
        }
        case F_COS: {
            D ep = exp(a.im), em = exp(-a.im);
            return CD(cos(a.re) * (ep + em) * D(0.5), -(sin(a.re) * (ep - em) * D(0.5)));
        }
        case F_SQRT:
        case F_CSQRT: return csqrtD(a);
        case F_ABS: return CD(sqrt(a.re * a.re + a.im * a.im));
        case F_RE: return CD(a.re);
        case F_IM: return CD(a.im);
        case F_CONJ: return CD(a.re, -a.im);
        }
        return CD();
    }
    case Expr::Model: {
        auto ev = [&](int k) { return evalExpr(*e.kids[k], vars, params); };
        switch (e.id) {
        case M_I: return CD(D(0.0), D(1.0));
        case M_Q0: return CD(q0AD(ev(0).re, ev(1).re, ev(2).re));
        case M_BF: return CD(Bf((int)ev(0).re.v, ev(1).re, ev(2).re, ev(3).re.v));
        case M_BW: return BW(ev(0).re, ev(1).re, ev(2).re);
        case M_BWR: return BWR(ev(0).re, ev(1).re, ev(2).re, (int)e.kids[3]->num, ev(4).re, ev(5).re, ev(6).re.v);
        case M_RHO_RE:
        case M_RHO_IM: {
            double rr, ri;
            flatteRho(ev(0).re.v, ev(1).re.v, ev(2).re.v, rr, ri);
            return CD(D(e.id == M_RHO_RE ? rr : ri));
        }
        }
        return CD();
    }
    }
    return CD();
}

}  // namespace oracle
