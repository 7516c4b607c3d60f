// Reverse mode on the IR: the adjoint law of a term.
//
// One step of a term is U' = U + dt R(U, s, p) for the fields U it writes, the fields s it only reads (static inputs,
// model numbers) and the params p. Given the cotangent A of U' (one field F__adj per written field), its
// vector-Jacobian product is
//
//   U_bar = A + dt (dR/dU)^T A,      s_bar += dt (dR/ds)^T A,      p_bar += dt (dR/dp)^T A (a field; its total over the
//                                                                   lattice is the param's gradient)
//
// built by one reverse sweep over the term's SSA instructions (highest id first: every user before what it uses), each
// instruction adding its local derivative times its own adjoint to its arguments'. The result is a law, as text: the
// primal values as `let`s, the adjoints as `let`s, and one equation `d X__adj = ...` a field or param, so the engine's
// own Euler store X__adj + dt * (...) is the product above and the reverse kernels are the ones the backend generates for
// any law. The reference builds adjoints the same way (src/field/ir/Adjoint.hpp:8-22, Adjoint.cpp:27-223); this one is
// written afresh over this backend's IR and adds what the reference refuses: the tridiagonal solves. For X = T^-1 d
// (T = tridiag(a, b, c) with the edge repeat), with Y = T^-T X_bar (tridiag_*_t):
//
//   d_bar += Y,    a_bar -= Y * X(i-1),    b_bar -= Y * X,    c_bar -= Y * X(i+1)     (the edge repeat: X clamped)
//
// Stencils go to their transposes (shift -> shift_t, gx -> gx_t, lap symmetric, diffuse with one k symmetric in its
// field). Refused, with the reason: reductions, the matter-moving ops, distance, poisson, nets, adv, and diffuse whose k
// is a field.
#pragma once

#include "law.hpp"

#include <string>

namespace fe::adjoint {

// The adjoint law of `term` (the law's first term when empty): empty text and `error` set when it cannot be built.
std::string adjoint_law(const law::Law& law, const std::string& term, std::string& error);

} // namespace fe::adjoint
