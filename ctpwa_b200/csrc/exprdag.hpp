// Expression DAG for the generated lineshape code.
//
// Every amplitude column's lineshape product and its derivatives with
// respect to the fitted resonance parameters are built as nodes of one
// hash-consed DAG over three kinds of leaves: constants, fitted parameters
// (theta) and per-event kinematic values. Each node is classified by what it
// depends on:
//   theta-only nodes are evaluated once per likelihood call (prologue),
//   nodes that depend on the event are evaluated per event,
//   event-only subexpressions are shared by all columns that use them.
// Derivatives are symbolic (chain rule on the DAG, memoised), so the per-event
// code contains only the arithmetic that genuinely varies per event.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace ctpwa {
namespace dag {

enum Op : uint8_t {
    Const,
    Theta,
    Kin,
    Add,
    Sub,
    Mul,
    Recip,   // 1 / a
    Neg,
    Sqrt,
    Log,
    Exp,
    Sin,
    Cos,
    Atan2,
    Sel,     // cmp(c) ? a : b
    RhoRe,   // Flatte channel factor, value only (args s, ma, mb)
    RhoIm,
};

enum Cmp : uint8_t { GE0 = 0, GT0, LE0, LT0, EQ0 };

enum Dep : uint8_t { DEP_NONE = 0, DEP_THETA = 1, DEP_EVENT = 2 };

struct Node {
    Op op;
    uint8_t cmp = 0;
    uint8_t dep = 0;
    int a = -1, b = -1, c = -1;
    double v = 0.0;  // Const value
    int idx = 0;     // Theta / Kin index
};

// Sign (+1 / -1) of a zero imaginary part, kept as a small expression
// outside the DAG and turned into nodes only where it is read.
struct ZSign;
using ZS = std::shared_ptr<const ZSign>;
struct ZSign {
    enum K { Pos, Neg, SignOf, Prod, Flip, Both } k = Pos;
    int node = -1;  // SignOf: the real node whose sign is taken
    ZS a, b;
};

// A complex value. When the imaginary part is a constant zero, `zs` carries
// the sign that zero has under IEEE arithmetic with the formulas of the
// custom-expression language (-x of a real x has imaginary part -0; null:
// +0). The sign matters only where the value reaches the branch cut of
// log / pow (atan2(+-0, re < 0) = +-pi), the one place it is read.
struct Cx {
    int re, im;
    ZS zs;
};

class Graph {
public:
    Graph();
    int cnst(double v);
    int theta(int j);
    int kin(int k);
    int add(int a, int b);
    int sub(int a, int b);
    int mul(int a, int b);
    int div(int a, int b);
    int neg(int a);
    int sqrt(int a);
    int log(int a);
    int exp(int a);
    int sin(int a);
    int cos(int a);
    int atan2(int y, int x);
    int sel(Cmp cmp, int c, int a, int b);
    int rho(bool im, int s, int ma, int mb);
    int powi(int a, int n);
    int recip(int a);
    int zero() { return zero_; }
    int one() { return one_; }

    // d(node)/d(theta_j)
    int deriv(int n, int j);

    bool isConst(int n) const { return nodes[n].op == Const; }
    double val(int n) const { return nodes[n].v; }

    // complex helpers (formulas of the custom-expression language)
    Cx c(double re, double im = 0.0) { return {cnst(re), cnst(im)}; }
    Cx cr(int re) { return {re, zero_}; }
    Cx cadd(Cx a, Cx b);
    Cx csub(Cx a, Cx b);
    Cx cneg(Cx a);
    Cx cconj(Cx a);
    Cx cmul(Cx a, Cx b);
    Cx cscale(Cx a, int s) { return {mul(a.re, s), mul(a.im, s)}; }
    Cx cdivRef(Cx a, Cx b);  // |b|^2 == 0 uses 1e-30 (custom-expression convention)
    Cx cexp(Cx a);
    Cx clogRef(Cx a);        // log|0| uses 1e-30
    Cx cpow(Cx b, Cx e) { return cexp(cmul(e, clogRef(b))); }
    Cx csqrt(Cx a);
    Cx csin(Cx a);
    Cx ccos(Cx a);

    std::vector<Node> nodes;

private:
    // signed zeros of imaginary parts (see Cx)
    int negZero();                                     // the constant -0.0 (distinct from zero())
    bool zeroIm(const Cx& a) const { return isConst(a.im) && val(a.im) == 0.0; }
    ZS zsign(const Cx& a) const;                       // sign of a's zero imaginary part
    ZS zconst(bool negative) const;
    ZS sgn(int x) const;                               // sign of a real node
    ZS zprod(const ZS& a, const ZS& b) const;
    ZS zflip(const ZS& a) const;
    ZS zsum(const ZS& a, const ZS& b) const;           // (+-0) + (+-0): negative iff both are
    static bool zisConst(const ZS& a) { return !a || a->k == ZSign::Pos || a->k == ZSign::Neg; }
    static bool zneg(const ZS& a) { return a && a->k == ZSign::Neg; }
    int zmaterialize(const ZS& a);                     // +-1 as a node
    int make(Node n);
    int mulRaw(int a, int b);  // a * b as one node, no regrouping
    int zero_, one_;
    std::map<std::tuple<int, int, int, int, int, double, int>, int> memo_;
    std::map<std::pair<int, int>, int> dmemo_;
};

}  // namespace dag
}  // namespace ctpwa
