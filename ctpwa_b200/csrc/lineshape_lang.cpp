// Custom-lineshape language: scanner, precedence-climbing parser and name
// resolution (grammar in lineshape_lang.hpp).
//
// Parsing and resolution are separate steps: the parser builds a plain syntax
// tree (numbers, names, calls, signs, binary operators) without knowing any
// name; `Resolver` then turns names and calls into lineshape nodes and checks
// the argument rules of the builtin functions.
#include "lineshape_lang.hpp"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <stdexcept>

namespace ctpwa {

namespace {

[[noreturn]] void fail(const std::string& text, size_t col, const std::string& what)
{
    throw std::runtime_error("custom lineshape '" + text + "': " + what + " (column " + std::to_string(col + 1) + ")");
}

// ---------------------------------------------------------------- scanner
struct Tok {
    enum Kind { Number, Imag, Name, Sym, End } kind = End;
    char sym = 0;       // + - * / ^ ( ) ,
    double value = 0;   // Number
    std::string name;   // Name
    size_t col = 0;
};

bool nameStart(char c) { return std::isalpha((unsigned char)c) || c == '_'; }
bool nameChar(char c) { return std::isalnum((unsigned char)c) || c == '_'; }
bool digit(char c) { return c >= '0' && c <= '9'; }

std::vector<Tok> scan(const std::string& s)
{
    std::vector<Tok> out;
    size_t i = 0;
    const size_t n = s.size();
    while (i < n) {
        const char c = s[i];
        if (std::isspace((unsigned char)c)) {
            ++i;
            continue;
        }
        Tok t;
        t.col = i;
        if (c == '1' && i + 1 < n && (s[i + 1] == 'j' || s[i + 1] == 'i') && !(i + 2 < n && nameChar(s[i + 2]))) {
            t.kind = Tok::Imag;
            i += 2;
        } else if (digit(c) || (c == '.' && i + 1 < n && digit(s[i + 1]))) {
            size_t j = i;
            while (j < n && digit(s[j])) ++j;
            if (j < n && s[j] == '.') {
                ++j;
                while (j < n && digit(s[j])) ++j;
            }
            if (j < n && (s[j] == 'e' || s[j] == 'E')) {
                size_t k = j + 1;
                if (k < n && (s[k] == '+' || s[k] == '-')) ++k;
                if (k >= n || !digit(s[k])) fail(s, j, "exponent without digits");
                while (k < n && digit(s[k])) ++k;
                j = k;
            }
            if (j < n && (nameChar(s[j]) || s[j] == '.')) fail(s, j, "malformed number");
            t.kind = Tok::Number;
            t.value = std::strtod(s.substr(i, j - i).c_str(), nullptr);
            i = j;
        } else if (nameStart(c)) {
            size_t j = i;
            while (j < n && nameChar(s[j])) ++j;
            t.kind = Tok::Name;
            t.name = s.substr(i, j - i);
            i = j;
        } else if (c == '+' || c == '-' || c == '*' || c == '/' || c == '^' || c == '(' || c == ')' || c == ',') {
            t.kind = Tok::Sym;
            t.sym = c;
            ++i;
        } else {
            fail(s, i, std::string("character '") + c + "' is not part of the language");
        }
        out.push_back(t);
    }
    Tok end;
    end.col = n;
    out.push_back(end);
    return out;
}

// ----------------------------------------------------------- syntax tree
struct Syn {
    enum Kind { Number, Imag, Name, Call, Sign, Binary } kind = Number;
    char op = 0;  // Sign: '-' ; Binary: + - * / ^
    double value = 0;
    std::string name;
    size_t col = 0;
    std::vector<std::unique_ptr<Syn>> sub;  // operands or call arguments
};
using SynP = std::unique_ptr<Syn>;

SynP syn(Syn::Kind k, size_t col)
{
    SynP p(new Syn);
    p->kind = k;
    p->col = col;
    return p;
}

class Parser {
public:
    Parser(const std::string& text) : text_(text), toks_(scan(text)) {}

    SynP parseAll()
    {
        SynP e = expression(0);
        if (toks_[at_].kind != Tok::End) fail(text_, toks_[at_].col, "unexpected token after a complete expression");
        return e;
    }

private:
    static constexpr int kSignOperand = 40;  // a sign's operand takes no infix operator
    const std::string& text_;
    std::vector<Tok> toks_;
    size_t at_ = 0;

    const Tok& peek() const { return toks_[at_]; }
    bool isSym(char c) const { return peek().kind == Tok::Sym && peek().sym == c; }

    // left binding power of an infix operator, 0 if the token is none
    static int leftPower(const Tok& t)
    {
        if (t.kind != Tok::Sym) return 0;
        switch (t.sym) {
        case '+': case '-': return 10;
        case '*': case '/': return 20;
        case '^': return 30;
        default: return 0;
        }
    }

    SynP expression(int min_power)
    {
        SynP lhs = operand();
        for (;;) {
            const Tok& t = peek();
            const int lp = leftPower(t);
            if (lp == 0 || lp <= min_power) break;
            ++at_;
            // '^' is right associative: its right side may contain another '^'
            SynP rhs = expression(t.sym == '^' ? lp - 1 : lp);
            SynP b = syn(Syn::Binary, t.col);
            b->op = t.sym;
            b->sub.push_back(std::move(lhs));
            b->sub.push_back(std::move(rhs));
            lhs = std::move(b);
        }
        return lhs;
    }

    SynP operand()
    {
        const Tok t = peek();
        switch (t.kind) {
        case Tok::End: fail(text_, t.col, "expression ends where an operand is expected");
        case Tok::Number: {
            ++at_;
            SynP p = syn(Syn::Number, t.col);
            p->value = t.value;
            return p;
        }
        case Tok::Imag: ++at_; return syn(Syn::Imag, t.col);
        case Tok::Name: {
            ++at_;
            if (!isSym('(')) {
                SynP p = syn(Syn::Name, t.col);
                p->name = t.name;
                return p;
            }
            ++at_;
            SynP call = syn(Syn::Call, t.col);
            call->name = t.name;
            if (isSym(')')) {
                ++at_;
                return call;
            }
            for (;;) {
                call->sub.push_back(expression(0));
                if (isSym(',')) {
                    ++at_;
                    continue;
                }
                if (isSym(')')) {
                    ++at_;
                    return call;
                }
                fail(text_, peek().col, "expected ',' or ')' in the argument list of " + t.name);
            }
        }
        case Tok::Sym:
            if (t.sym == '-' || t.sym == '+') {
                ++at_;
                SynP inner = expression(kSignOperand);
                if (t.sym == '+') return inner;
                SynP p = syn(Syn::Sign, t.col);
                p->op = '-';
                p->sub.push_back(std::move(inner));
                return p;
            }
            if (t.sym == '(') {
                ++at_;
                SynP inner = expression(0);
                if (!isSym(')')) fail(text_, peek().col, "expected ')'");
                ++at_;
                return inner;
            }
            fail(text_, t.col, std::string("'") + t.sym + "' where an operand is expected");
        }
        fail(text_, t.col, "unexpected token");
    }
};

// ------------------------------------------------------------ resolution
XP node(XNode::K k, std::vector<XP> kids = {}, double v = 0, const std::string& id = "", int idx = 0)
{
    XP n = std::make_shared<XNode>();
    n->k = k;
    n->kids = std::move(kids);
    n->v = v;
    n->id = id;
    n->idx = idx;
    return n;
}
XP number(double v) { return node(XNode::Num, {}, v); }
XP variable(const char* name) { return node(XNode::Var, {}, 0, name); }

class Resolver {
public:
    Resolver(const std::string& text, const std::vector<std::string>& params) : text_(text), params_(params) {}

    XP resolve(const Syn& s)
    {
        switch (s.kind) {
        case Syn::Number: return number(s.value);
        case Syn::Imag: return node(XNode::Model, {}, 0, "i");
        case Syn::Sign: return node(XNode::Neg, {resolve(*s.sub[0])});
        case Syn::Binary: {
            XP a = resolve(*s.sub[0]), b = resolve(*s.sub[1]);
            const XNode::K k = s.op == '+' ? XNode::Add : s.op == '-' ? XNode::Sub : s.op == '*' ? XNode::Mul
                             : s.op == '/' ? XNode::Div : XNode::Pow;
            return node(k, {a, b});
        }
        case Syn::Name: return name(s);
        case Syn::Call: return call(s);
        }
        fail(text_, s.col, "unexpected syntax node");
    }

private:
    const std::string& text_;
    const std::vector<std::string>& params_;

    static bool eventVariable(const std::string& n)
    {
        static const char* const vars[] = {"m", "q", "L", "d", "p1p", "p1e", "p1costheta", "p1phi",
                                           "p2p", "p2e", "p2costheta", "p2phi"};
        for (const char* v : vars)
            if (n == v) return true;
        return false;
    }
    // one-argument functions: language name -> generator name
    static const char* unaryFunction(const std::string& n)
    {
        static const char* const table[][2] = {{"exp", "exp"}, {"log", "log"}, {"ln", "log"},   {"sin", "sin"},
                                               {"cos", "cos"}, {"sqrt", "sqrt"}, {"csqrt", "sqrt"}, {"abs", "abs"},
                                               {"Re", "re"},   {"real", "re"},  {"Im", "im"},     {"imag", "im"},
                                               {"conj", "conj"}};
        for (const auto& e : table)
            if (n == e[0]) return e[1];
        return nullptr;
    }
    static bool lineshapeFunction(const std::string& n)
    {
        return n == "BW" || n == "BWR" || n == "Bf" || n == "Flatte" || n == "q0";
    }

    // q0 of the first parameter (1 without parameters) and the daughter masses
    XP defaultQ0() const
    {
        XP m0 = params_.empty() ? number(1.0) : node(XNode::Param, {}, 0, "", 0);
        return node(XNode::Model, {m0, variable("md1"), variable("md2")}, 0, "q0");
    }

    XP name(const Syn& s)
    {
        const std::string& n = s.name;
        if (n == "pi") return number(3.14159265358979323846);
        if (n == "q0") return defaultQ0();
        if (eventVariable(n)) return node(XNode::Var, {}, 0, n);
        if (unaryFunction(n) || lineshapeFunction(n)) fail(text_, s.col, "function " + n + " is used without an argument list");
        for (size_t i = 0; i < params_.size(); ++i)
            if (params_[i] == n) return node(XNode::Param, {}, 0, "", (int)i);
        fail(text_, s.col, "'" + n + "' is neither a parameter of this resonance nor a known name");
    }

    [[noreturn]] void arity(const Syn& s, const std::string& form) const
    {
        fail(text_, s.col, s.name + " takes " + form + ", got " + std::to_string(s.sub.size()) + " argument(s)");
    }
    void requireLiteral(const Syn& s, const XP& a, const char* what) const
    {
        if (a->k != XNode::Num) fail(text_, s.col, std::string("the ") + what + " of " + s.name + " must be a number");
    }

    XP call(const Syn& s)
    {
        const std::string& n = s.name;
        std::vector<XP> a;
        for (const auto& x : s.sub) a.push_back(resolve(*x));
        const size_t na = a.size();
        if (const char* f = unaryFunction(n)) {
            if (na != 1) arity(s, "one argument");
            return node(XNode::Func, {a[0]}, 0, f);
        }
        if (!lineshapeFunction(n)) fail(text_, s.col, "'" + n + "' is not a function");
        const XP m = variable("m");
        if (n == "BW") {
            if (na != 2) arity(s, "(m0, w0)");
            return node(XNode::Model, {m, a[0], a[1]}, 0, "bw");
        }
        if (n == "BWR") {
            if (na < 2 || na > 4) arity(s, "(m0, g0[, L[, d]])");
            if (na >= 3) requireLiteral(s, a[2], "orbital angular momentum L");
            if (na >= 4) requireLiteral(s, a[3], "barrier radius d");
            const double L = na >= 3 ? a[2]->v : 1.0, d = na >= 4 ? a[3]->v : 3.0;
            return node(XNode::Model, {m, a[0], a[1], number(L), variable("q"), defaultQ0(), number(d)}, 0, "bwr");
        }
        if (n == "Bf") {
            if (na != 4) arity(s, "(L, q, q0, d)");
            requireLiteral(s, a[0], "orbital angular momentum L");
            return node(XNode::Model, a, 0, "bf");
        }
        if (n == "q0") {
            if (na == 1) return node(XNode::Model, {a[0], variable("md1"), variable("md2")}, 0, "q0");
            if (na == 3) return node(XNode::Model, a, 0, "q0");
            arity(s, "(m0) or (m0, md1, md2)");
        }
        // Flatte(m0, g_1..g_n, (ma_i, mb_i)_i): the language defines it as
        // 1 / (m0^2 - m^2 - i m0/2 sum_i g_i rho_i(m^2)) with the complex
        // two-body phase-space factor rho_i; it is expanded here into
        // (A - iB) / (A^2 + B^2), A + iB = the denominator.
        if (na < 4 || (na - 1) % 3 != 0) arity(s, "(m0, g_1..g_n, ma_1, mb_1, .., ma_n, mb_n) with n >= 1");
        const int nch = (int)(na - 1) / 3;
        const XP m2 = node(XNode::Mul, {m, m});
        const XP half_m0 = node(XNode::Mul, {a[0], number(0.5)});
        // m0^2 - m^2 first, so that the cancelling pair is one subtraction
        XP re = node(XNode::Sub, {node(XNode::Mul, {a[0], a[0]}), m2});
        XP im = number(0.0);
        for (int c = 0; c < nch; ++c) {
            const XP& ma = a[1 + nch + 2 * c];
            const XP& mb = a[2 + nch + 2 * c];
            const XP rho_re = node(XNode::Model, {m2, ma, mb}, 0, "rho_re");
            const XP rho_im = node(XNode::Model, {m2, ma, mb}, 0, "rho_im");
            const XP w = node(XNode::Mul, {a[1 + c], half_m0});
            re = node(XNode::Add, {re, node(XNode::Mul, {w, rho_im})});
            im = node(XNode::Sub, {im, node(XNode::Mul, {w, rho_re})});
        }
        const XP norm = node(XNode::Add, {node(XNode::Mul, {re, re}), node(XNode::Mul, {im, im})});
        const XP unit = node(XNode::Model, {}, 0, "i");
        return node(XNode::Add, {node(XNode::Div, {re, norm}),
                                 node(XNode::Mul, {node(XNode::Neg, {node(XNode::Div, {im, norm})}), unit})});
    }
};

// ------------------------------------------------------------ folding
// The language folds a resolved expression bottom-up before it is evaluated
// (reference: simplify, src/CustomExpr.cu:785-835), and the folding is
// observable: a constant power is the real pow ((-2)^0.5 is NaN), 0^x is 0,
// a negated number literal is a negative number (imaginary part +0, not -0).
// Rules, with "number" a Num node and 0 / 1 its value:
//   0 + x, x + 0 -> x        x - 0 -> x          number op number -> number
//   0 * x, x * 0 -> 0        1 * x, x * 1 -> x   0 / x -> 0, x / 1 -> x
//   x ^ 1 -> x, 1 ^ x -> 1, 0 ^ x -> 0           -(-x) -> x, -number -> number
bool isNum(const XP& x) { return x->k == XNode::Num; }
bool isNum(const XP& x, double v) { return x->k == XNode::Num && x->v == v; }

XP fold(const XP& x)
{
    if (x->kids.empty()) return x;
    std::vector<XP> k;
    for (const XP& c : x->kids) k.push_back(fold(c));
    switch (x->k) {
    case XNode::Add:
        if (isNum(k[0], 0.0)) return k[1];
        if (isNum(k[1], 0.0)) return k[0];
        if (isNum(k[0]) && isNum(k[1])) return number(k[0]->v + k[1]->v);
        break;
    case XNode::Sub:
        if (isNum(k[1], 0.0)) return k[0];
        if (isNum(k[0]) && isNum(k[1])) return number(k[0]->v - k[1]->v);
        break;
    case XNode::Mul:
        if (isNum(k[0], 0.0) || isNum(k[1], 0.0)) return number(0.0);
        if (isNum(k[0], 1.0)) return k[1];
        if (isNum(k[1], 1.0)) return k[0];
        if (isNum(k[0]) && isNum(k[1])) return number(k[0]->v * k[1]->v);
        break;
    case XNode::Div:
        if (isNum(k[0], 0.0)) return number(0.0);
        if (isNum(k[1], 1.0)) return k[0];
        if (isNum(k[0]) && isNum(k[1]) && k[1]->v != 0.0) return number(k[0]->v / k[1]->v);
        break;
    case XNode::Pow:
        if (isNum(k[1], 1.0)) return k[0];
        if (isNum(k[0], 1.0)) return number(1.0);
        if (isNum(k[0], 0.0)) return number(0.0);
        if (isNum(k[0]) && isNum(k[1])) return number(std::pow(k[0]->v, k[1]->v));
        break;
    case XNode::Neg:
        if (k[0]->k == XNode::Neg) return k[0]->kids[0];
        if (isNum(k[0])) return number(-k[0]->v);
        break;
    default: break;
    }
    XP n = std::make_shared<XNode>(*x);
    n->kids = std::move(k);
    return n;
}

}  // namespace

XP parseLineshapeExpr(const std::string& text, const std::vector<std::string>& params)
{
    Parser p(text);
    SynP tree = p.parseAll();
    Resolver r(text, params);
    return fold(r.resolve(*tree));
}

}  // namespace ctpwa
