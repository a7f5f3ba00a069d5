// Front end of the custom-lineshape language: the `expr:` of a resonance of
// type custom in config.yml (reference language: src/CustomExpr.cu:236-528,
// include/CustomExpr.cuh:6-27). The language (operators, precedence,
// identifiers, builtin functions and their argument rules) is part of the
// drop-in contract; this front end is written from the grammar below.
//
//   expression := operand { infix operand }
//   infix      := '+' | '-'          binding 10, left associative
//               | '*' | '/'          binding 20, left associative
//               | '^'                binding 30, right associative
//   operand    := ('-' | '+') operand-tight        (sign binds tighter than '^':
//                                                   -a^b is (-a)^b, a^-b is a^(-b))
//               | number | imaginary | '(' expression ')'
//               | name | name '(' [ expression { ',' expression } ] ')'
//   number     := digits ['.' digits] [('e'|'E') ['+'|'-'] digits], or '.' digits ...
//   imaginary  := the two characters "1j" or "1i"
//
// Names: pi; the event variables m, q, L, d, p1p, p1e, p1costheta, p1phi,
// p2p, p2e, p2costheta, p2phi; q0 (alone: q0 of the first parameter and the
// daughter masses md1, md2); the resonance's parameter names. Functions of one
// argument: exp, log (ln), sin, cos, sqrt (csqrt), abs, Re (real), Im (imag),
// conj. Builtin lineshapes: BW(m0, w0), BWR(m0, g0[, L[, d]]) with L and d
// literals, Bf(L, q, q0, d) with L a literal, q0(x) or q0(x, md1, md2),
// Flatte(m0, g_1..g_n, ma_1, mb_1, .., ma_n, mb_n).
#pragma once

#include <memory>
#include <string>
#include <vector>

namespace ctpwa {

// Lineshape tree consumed by the code generator.
struct XNode {
    enum K { Num, Var, Param, Add, Sub, Mul, Div, Pow, Neg, Func, Model } k = Num;
    double v = 0;
    std::string id;  // var / func / model name
    int idx = 0;     // param index
    std::vector<std::shared_ptr<XNode>> kids;
};
using XP = std::shared_ptr<XNode>;

// Parses and resolves one expression against the resonance's parameter names,
// then folds it by the language's constant rules (lineshape_lang.cpp, fold).
// Throws std::runtime_error("custom lineshape: ...") with the column of the
// offending token on any syntax or name error.
XP parseLineshapeExpr(const std::string& text, const std::vector<std::string>& params);

}  // namespace ctpwa
