// Expression DAG (see exprdag.hpp).
#include "exprdag.hpp"

#include <cmath>
#include <stdexcept>

namespace ctpwa {
namespace dag {

namespace {
double foldUnary(Op op, double x)
{
    switch (op) {
    case Neg: return -x;
    case Sqrt: return std::sqrt(x);
    case Log: return std::log(x);
    case Exp: return std::exp(x);
    case Sin: return std::sin(x);
    case Cos: return std::cos(x);
    default: return x;
    }
}
bool cmpTrue(Cmp c, double x)
{
    switch (c) {
    case GE0: return x >= 0.0;
    case GT0: return x > 0.0;
    case LE0: return x <= 0.0;
    case LT0: return x < 0.0;
    case EQ0: return x == 0.0;
    }
    return false;
}
}  // namespace

Graph::Graph()
{
    zero_ = cnst(0.0);
    one_ = cnst(1.0);
}

int Graph::make(Node n)
{
    auto key = std::make_tuple((int)n.op, (int)n.cmp, n.a, n.b, n.c, n.v, n.idx);
    auto it = memo_.find(key);
    if (it != memo_.end()) return it->second;
    uint8_t dep = 0;
    if (n.op == Theta) dep = DEP_THETA;
    else if (n.op == Kin) dep = DEP_EVENT;
    for (int k : {n.a, n.b, n.c})
        if (k >= 0) dep |= nodes[k].dep;
    n.dep = dep;
    int id = (int)nodes.size();
    nodes.push_back(n);
    memo_[key] = id;
    return id;
}

int Graph::cnst(double v)
{
    Node n;
    n.op = Const;
    n.v = v == 0.0 ? 0.0 : v;  // fold -0.0
    return make(n);
}
int Graph::theta(int j)
{
    Node n;
    n.op = Theta;
    n.idx = j;
    return make(n);
}
int Graph::kin(int k)
{
    Node n;
    n.op = Kin;
    n.idx = k;
    return make(n);
}

int Graph::add(int a, int b)
{
    if (isConst(a) && isConst(b)) return cnst(val(a) + val(b));
    if (isConst(a) && val(a) == 0.0) return b;
    if (isConst(b) && val(b) == 0.0) return a;
    // x + x for a product x with a parameter-only factor: the 2 joins that
    // factor (2 c is a per-call constant; doubling is exact either way)
    if (a == b && nodes[a].op == Mul && nodes[a].dep == (DEP_THETA | DEP_EVENT)) {
        auto pOnly = [&](int x) { return nodes[x].dep == DEP_THETA || nodes[x].dep == DEP_NONE; };
        if (pOnly(nodes[a].a) || pOnly(nodes[a].b)) return mul(cnst(2.0), a);
    }
    if (a > b) std::swap(a, b);
    Node n;
    n.op = Add;
    n.a = a;
    n.b = b;
    return make(n);
}
int Graph::sub(int a, int b)
{
    if (isConst(a) && isConst(b)) return cnst(val(a) - val(b));
    if (isConst(b) && val(b) == 0.0) return a;
    if (isConst(a) && val(a) == 0.0) return neg(b);
    if (a == b) return zero_;
    Node n;
    n.op = Sub;
    n.a = a;
    n.b = b;
    return make(n);
}
int Graph::mul(int a, int b)
{
    if (isConst(a) && isConst(b)) return cnst(val(a) * val(b));
    if ((isConst(a) && val(a) == 0.0) || (isConst(b) && val(b) == 0.0)) return zero_;
    if (isConst(a) && val(a) == 1.0) return b;
    if (isConst(b) && val(b) == 1.0) return a;
    if (isConst(a) && val(a) == -1.0) return neg(b);
    if (isConst(b) && val(b) == -1.0) return neg(a);
    // A product that depends on both the parameters and the event is
    // regrouped by dependence: its event-only factors are multiplied together
    // (one per-event value, evaluated once per event) and its parameter-only
    // factors together (one per-call value), so e.g. the Blatt-Weisskopf
    // factors of q at both vertices of a chain become one per-event value.
    auto cls = [&](int x) { return nodes[x].dep == DEP_NONE ? (int)DEP_THETA : (int)nodes[x].dep; };
    if ((cls(a) | cls(b)) == (DEP_THETA | DEP_EVENT)) {
        std::vector<int> f;
        std::vector<std::pair<int, int>> st = {{a, 0}, {b, 0}};
        while (!st.empty()) {
            auto [x, depth] = st.back();
            st.pop_back();
            if (nodes[x].op == Mul && cls(x) == (DEP_THETA | DEP_EVENT) && depth < 3) {
                st.push_back({nodes[x].a, depth + 1});
                st.push_back({nodes[x].b, depth + 1});
            } else {
                f.push_back(x);
            }
        }
        if (f.size() > 2) {
            int e = -1, t = -1, m = -1;
            for (int x : f) {
                int& acc = cls(x) == DEP_EVENT ? e : cls(x) == DEP_THETA ? t : m;
                acc = acc < 0 ? x : (cls(x) == (DEP_THETA | DEP_EVENT) ? mulRaw(acc, x) : mul(acc, x));
            }
            int r = m;
            for (int x : {t, e})
                if (x >= 0) r = r < 0 ? x : mulRaw(r, x);
            return r;
        }
    }
    return mulRaw(a, b);
}

int Graph::mulRaw(int a, int b)
{
    if (a > b) std::swap(a, b);
    Node n;
    n.op = Mul;
    n.a = a;
    n.b = b;
    return make(n);
}
int Graph::recip(int a)
{
    if (isConst(a)) return cnst(1.0 / val(a));
    if (nodes[a].op == Recip) return nodes[a].a;
    Node n;
    n.op = Recip;
    n.a = a;
    return make(n);
}

// a / b as a * (1/b): one reciprocal per denominator, shared by every use and
// by every derivative (d(1/b) = -(1/b)^2 db needs no further division)
int Graph::div(int a, int b)
{
    if (isConst(a) && isConst(b)) return cnst(val(a) / val(b));
    if (isConst(b) && val(b) == 1.0) return a;
    if (isConst(a) && val(a) == 0.0) return zero_;
    return mul(a, recip(b));
}

int Graph::neg(int a)
{
    if (isConst(a)) return cnst(-val(a));
    if (nodes[a].op == Neg) return nodes[a].a;
    Node n;
    n.op = Neg;
    n.a = a;
    return make(n);
}

#define CT_UNARY(name, OP)             \
    int Graph::name(int a)             \
    {                                  \
        if (isConst(a)) return cnst(foldUnary(OP, val(a))); \
        Node n;                        \
        n.op = OP;                     \
        n.a = a;                       \
        return make(n);                \
    }
CT_UNARY(sqrt, Sqrt)
CT_UNARY(log, Log)
CT_UNARY(exp, Exp)
CT_UNARY(sin, Sin)
CT_UNARY(cos, Cos)
#undef CT_UNARY

int Graph::atan2(int y, int x)
{
    if (isConst(y) && isConst(x)) return cnst(std::atan2(val(y), val(x)));
    Node n;
    n.op = Atan2;
    n.a = y;
    n.b = x;
    return make(n);
}

int Graph::sel(Cmp cmp, int c, int a, int b)
{
    if (isConst(c)) return cmpTrue(cmp, val(c)) ? a : b;
    if (a == b) return a;
    Node n;
    n.op = Sel;
    n.cmp = cmp;
    n.a = a;
    n.b = b;
    n.c = c;
    return make(n);
}

int Graph::rho(bool im, int s, int ma, int mb)
{
    Node n;
    n.op = im ? RhoIm : RhoRe;
    n.a = s;
    n.b = ma;
    n.c = mb;
    if (isConst(s) && isConst(ma) && isConst(mb)) {
        double S = (val(ma) + val(mb)) * (val(ma) + val(mb)), D = (val(ma) - val(mb)) * (val(ma) - val(mb));
        double f1 = 1.0 - S / val(s), f2s = 1.0 - D / val(s), f2 = f2s > 0 ? std::sqrt(f2s) : 0.0;
        double re = f1 >= 0 ? std::sqrt(f1) * f2 : 0.0, imv = f1 >= 0 ? 0.0 : std::sqrt(-f1) * f2;
        return cnst(im ? imv : re);
    }
    return make(n);
}

int Graph::powi(int a, int n)
{
    if (n < 0) return recip(powi(a, -n));
    if (n == 0) return one_;
    if (n == 1) return a;
    int h = powi(a, n / 2);
    int h2 = mul(h, h);
    return (n % 2) ? mul(h2, a) : h2;
}

int Graph::deriv(int n, int j)
{
    const Node nd = nodes[n];
    if (!(nd.dep & DEP_THETA)) return zero_;
    auto key = std::make_pair(n, j);
    auto it = dmemo_.find(key);
    if (it != dmemo_.end()) return it->second;
    int r = zero_;
    switch (nd.op) {
    case Const:
    case Kin:
    case RhoRe:
    case RhoIm: r = zero_; break;
    case Theta: r = nd.idx == j ? one_ : zero_; break;
    case Add: r = add(deriv(nd.a, j), deriv(nd.b, j)); break;
    case Sub: r = sub(deriv(nd.a, j), deriv(nd.b, j)); break;
    case Mul: r = add(mul(deriv(nd.a, j), nd.b), mul(nd.a, deriv(nd.b, j))); break;
    case Recip: r = neg(mul(mul(n, n), deriv(nd.a, j))); break;
    case Neg: r = neg(deriv(nd.a, j)); break;
    case Sqrt: r = mul(mul(cnst(0.5), deriv(nd.a, j)), recip(n)); break;
    case Log: r = div(deriv(nd.a, j), nd.a); break;
    case Exp: r = mul(n, deriv(nd.a, j)); break;
    case Sin: r = mul(cos(nd.a), deriv(nd.a, j)); break;
    case Cos: r = neg(mul(sin(nd.a), deriv(nd.a, j))); break;
    case Atan2: {
        int y = nd.a, x = nd.b;
        int den = add(mul(x, x), mul(y, y));
        r = div(sub(mul(x, deriv(y, j)), mul(y, deriv(x, j))), den);
        break;
    }
    case Sel: r = sel((Cmp)nd.cmp, nd.c, deriv(nd.a, j), deriv(nd.b, j)); break;
    }
    dmemo_[key] = r;
    return r;
}

int Graph::negZero()
{
    Node n;
    n.op = Const;
    n.v = -0.0;
    n.idx = 1;  // keeps it apart from +0.0 in the node memo
    return make(n);
}

ZS Graph::zconst(bool negative) const
{
    auto z = std::make_shared<ZSign>();
    z->k = negative ? ZSign::Neg : ZSign::Pos;
    return z;
}

ZS Graph::zsign(const Cx& a) const
{
    if (a.zs) return a.zs;
    return zconst(isConst(a.im) && std::signbit(val(a.im)));
}

ZS Graph::sgn(int x) const
{
    if (isConst(x)) return zconst(std::signbit(val(x)));
    auto z = std::make_shared<ZSign>();
    z->k = ZSign::SignOf;
    z->node = x;
    return z;
}

ZS Graph::zprod(const ZS& a, const ZS& b) const
{
    if (zisConst(a) && zisConst(b)) return zconst(zneg(a) != zneg(b));
    auto z = std::make_shared<ZSign>();
    z->k = ZSign::Prod;
    z->a = a;
    z->b = b;
    return z;
}

ZS Graph::zflip(const ZS& a) const
{
    if (zisConst(a)) return zconst(!zneg(a));
    auto z = std::make_shared<ZSign>();
    z->k = ZSign::Flip;
    z->a = a;
    return z;
}

ZS Graph::zsum(const ZS& a, const ZS& b) const
{
    if (zisConst(a) && zisConst(b)) return zconst(zneg(a) && zneg(b));
    if (zisConst(a) && !zneg(a)) return zconst(false);
    if (zisConst(b) && !zneg(b)) return zconst(false);
    auto z = std::make_shared<ZSign>();
    z->k = ZSign::Both;
    z->a = a;
    z->b = b;
    return z;
}

int Graph::zmaterialize(const ZS& a)
{
    if (!a || a->k == ZSign::Pos) return one_;
    switch (a->k) {
    case ZSign::Neg: return cnst(-1.0);
    case ZSign::SignOf: return sel(LT0, a->node, cnst(-1.0), one_);
    case ZSign::Prod: return mul(zmaterialize(a->a), zmaterialize(a->b));
    case ZSign::Flip: return neg(zmaterialize(a->a));
    case ZSign::Both: return sel(LT0, zmaterialize(a->a), zmaterialize(a->b), one_);
    default: return one_;
    }
}

Cx Graph::cadd(Cx a, Cx b)
{
    Cx r{add(a.re, b.re), add(a.im, b.im)};
    if (zeroIm(a) && zeroIm(b)) r.zs = zsum(zsign(a), zsign(b));
    return r;
}

Cx Graph::csub(Cx a, Cx b)
{
    Cx r{sub(a.re, b.re), sub(a.im, b.im)};
    if (zeroIm(a) && zeroIm(b)) r.zs = zsum(zsign(a), zflip(zsign(b)));
    return r;
}

Cx Graph::cneg(Cx a)
{
    Cx r{neg(a.re), neg(a.im)};
    if (zeroIm(a)) r.zs = zflip(zsign(a));
    return r;
}

Cx Graph::cconj(Cx a)
{
    Cx r{a.re, neg(a.im)};
    if (zeroIm(a)) r.zs = zflip(zsign(a));
    return r;
}

// im = a.re b.im + a.im b.re: for real a and b the two zero terms have the
// signs sgn(a.re) zs(b) and zs(a) sgn(b.re)
Cx Graph::cmul(Cx a, Cx b)
{
    Cx r{sub(mul(a.re, b.re), mul(a.im, b.im)), add(mul(a.re, b.im), mul(a.im, b.re))};
    if (zeroIm(a) && zeroIm(b)) r.zs = zsum(zprod(sgn(a.re), zsign(b)), zprod(zsign(a), sgn(b.re)));
    return r;
}

// im = (a.im b.re - a.re b.im) / |b|^2
Cx Graph::cdivRef(Cx a, Cx b)
{
    int s = add(mul(b.re, b.re), mul(b.im, b.im));
    s = sel(EQ0, s, cnst(1e-30), s);
    int is = recip(s);
    Cx r{mul(add(mul(a.re, b.re), mul(a.im, b.im)), is), mul(sub(mul(a.im, b.re), mul(a.re, b.im)), is)};
    if (zeroIm(a) && zeroIm(b)) r.zs = zsum(zprod(zsign(a), sgn(b.re)), zflip(zprod(sgn(a.re), zsign(b))));
    return r;
}

// im = e^re sin(im): sin(+-0) = +-0
Cx Graph::cexp(Cx a)
{
    int e = exp(a.re);
    Cx r{mul(e, cos(a.im)), mul(e, sin(a.im))};
    if (zeroIm(a)) r.zs = zsign(a);
    return r;
}

// im = atan2(a.im, a.re): +-pi on the negative real axis by the sign of a's
// zero imaginary part
Cx Graph::clogRef(Cx a)
{
    int r = sqrt(add(mul(a.re, a.re), mul(a.im, a.im)));
    r = sel(EQ0, r, cnst(1e-30), r);
    int y = a.im;
    if (zeroIm(a)) {
        ZS z = zsign(a);
        y = zisConst(z) ? (zneg(z) ? negZero() : zero_) : sel(LT0, zmaterialize(z), negZero(), zero_);
    }
    Cx out{log(r), atan2(y, a.re)};
    if (zeroIm(out))  // folded: y and a.re are constants
        out.zs = zconst(std::signbit(std::atan2(val(y), val(a.re))));
    return out;
}

Cx Graph::csqrt(Cx a)
{
    int r = sqrt(add(mul(a.re, a.re), mul(a.im, a.im)));
    int re = sqrt(mul(add(r, a.re), cnst(0.5)));
    int im = sqrt(mul(sub(r, a.re), cnst(0.5)));
    return {re, sel(LT0, a.im, neg(im), im)};
}

// im = cos(re) (e^im - e^-im) / 2: for real a, sgn(cos(re)) times +0
Cx Graph::csin(Cx a)
{
    int ep = exp(a.im), em = exp(neg(a.im));
    Cx r{mul(mul(sin(a.re), add(ep, em)), cnst(0.5)), mul(mul(cos(a.re), sub(ep, em)), cnst(0.5))};
    if (zeroIm(a)) r.zs = sgn(cos(a.re));  // the cos node exists already (memo)
    return r;
}

// im = -sin(re) (e^im - e^-im) / 2: for real a, -sgn(sin(re)) times +0
Cx Graph::ccos(Cx a)
{
    int ep = exp(a.im), em = exp(neg(a.im));
    Cx r{mul(mul(cos(a.re), add(ep, em)), cnst(0.5)), neg(mul(mul(sin(a.re), sub(ep, em)), cnst(0.5)))};
    if (zeroIm(a)) r.zs = zflip(sgn(sin(a.re)));  // the sin node exists already (memo)
    return r;
}

}  // namespace dag
}  // namespace ctpwa
