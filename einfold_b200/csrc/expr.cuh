// The row-expression interpreter shared by the tile kernels and the
// evaluation entry point.
#pragma once

#include <cmath>

#include "fold.h"

namespace ef {

// A postfix expression (expression.rs:61-120) over slots; column nodes
// carry their slot in `a`. Every operation rounds once, as Rust's f64 does;
// power(a, 2) is the product a·a, rounded once (the correctly rounded
// square, which a power function returns up to its own rounding error; the
// same NaN, infinities and signed zeros).
// DEPTH bounds the stack (the host passes the expressions' deepest);
// slot(i) reads slot i.
template <int DEPTH, class Slot>
__device__ __forceinline__ double eval(const ExprNode* __restrict__ nodes, int n, Slot slot) {
  double st[DEPTH];
  int sp = 0;
  for (int i = 0; i < n; i++) {
    const ExprNode e = nodes[i];
    if (e.kind == 0) {
      st[sp++] = slot(e.a);
    } else if (e.kind == 1) {
      st[sp++] = e.value;
    } else if (e.kind == 2) {
      const double x = st[sp - 1];
      st[sp - 1] = e.a == 0 ? -x : e.a == 1 ? fabs(x) : e.a == 2 ? exp(x) : log(x);
    } else {
      const double b = st[--sp], a = st[sp - 1];
      double r;
      switch (e.a) {
        case 0: r = __dadd_rn(a, b); break;
        case 1: r = __dsub_rn(a, b); break;
        case 2: r = __dmul_rn(a, b); break;
        case 3: r = __ddiv_rn(a, b); break;
        default: r = b == 2.0 ? __dmul_rn(a, a) : pow(a, b); break;
      }
      st[sp - 1] = r;
    }
  }
  return st[0];
}

}  // namespace ef
