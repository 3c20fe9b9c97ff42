// A dense backend over the C ABI: the two calls of einfold's DenseBackend
// trait (crates/einfold-kernels/src/backend.rs:124-143), may_run and run,
// for the work kinds it offers (DenseWork::Product, DenseWork::Attention,
// backend.rs:46-96), with operands either packed in host memory, as the
// trait hands them, or already in HBM (the device-resident operands that a
// replacement of the trait passes, docs/design.md:495).
#include "attention.cuh"

namespace ef {

// An attention's allowed ranges as conditions between x and j: every row's
// range [lo, hi) must be [x + a, x + b) clamped to [0, keys), for constants
// a and b (either side may be unbounded), as einfold's own conditions give.
// False if the ranges have another form.
bool ranges_as_mask(const int64_t* ranges, int64_t queries, int64_t keys, Mask& m) {
  bool have_a = false, have_b = false;
  int64_t a = 0, b = 0;
  for (int64_t x = 0; x < queries; x++) {
    const int64_t lo = ranges[2 * x], hi = ranges[2 * x + 1];
    if (lo < 0 || hi > keys) return false;
    if (lo >= hi) continue;  // an empty range constrains nothing here; checked below
    if (lo > 0) {
      if (have_a && lo - x != a) return false;
      a = lo - x;
      have_a = true;
    }
    if (hi < keys) {
      if (have_b && hi - x != b) return false;
      b = hi - x;
      have_b = true;
    }
  }
  m = Mask{};
  if (have_a) {  // j >= x + a: x <= j - a
    m.cmp[m.n] = 1;
    m.off[m.n] = -a;
    m.n++;
  }
  if (have_b) {  // j < x + b: x > j - b
    m.cmp[m.n] = 2;
    m.off[m.n] = -b;
    m.n++;
  }
  m.lnx = queries > 0 ? queries : 1;
  m.lnj = keys;
  // Every row, the empty ones included, must be what the conditions give.
  for (int64_t x = 0; x < queries; x++) {
    int64_t lo = 0, hi = 0;
    allowed(m, x, lo, hi);
    const int64_t wlo = ranges[2 * x], whi = ranges[2 * x + 1];
    const bool empty = lo >= hi, wempty = wlo >= whi;
    if (empty != wempty || (!empty && (lo != wlo || hi != whi))) return false;
  }
  return true;
}

}  // namespace ef
