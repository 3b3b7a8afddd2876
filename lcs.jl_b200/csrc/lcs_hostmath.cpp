// lcs_hostmath.cpp -- host-side tables of the particle statistics, in
// extended precision where the reference computes in extended precision.
//
// lcs_logrange: the bin edges of rdf_assume_ci (src/particles/rdf.jl:21-23),
// `logrange(rmin, rmax, len)` (Julia's Base.LogRange): the endpoints exactly,
// every other edge exp of the interpolated logarithm, which Julia evaluates in
// double-double arithmetic; here in IEEE binary128 (libquadmath) and rounded
// once to double.
#include <quadmath.h>

extern "C" __attribute__((visibility("hidden"))) void lcs_logrange(double a, double b, int len, double* out) {
  if (len <= 0) return;
  out[0] = a;
  if (len == 1) return;
  const __float128 la = logq((__float128)a), lb = logq((__float128)b);
  for (int i = 2; i < len; i++) {
    const __float128 x = ((__float128)(len - i) * la + (__float128)(i - 1) * lb) / (__float128)(len - 1);
    out[i - 1] = (double)expq(x);
  }
  out[len - 1] = b;
}
