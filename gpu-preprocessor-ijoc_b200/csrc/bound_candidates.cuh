// Bound-strengthening candidates of one stored entry, shared by the fused
// activity + candidate sweep (live.cu) and the support-row pass
// (rules_bound.cu).  Reference: rules/rule_bound_strengthening.cu:349-430.
#pragma once

#include "common.cuh"

namespace gpp {

// Implied bounds of the column of entry a from its row (reference :349-430).
__device__ __forceinline__ void implied_bounds(double a, double lj, double uj, double al, double au, double mn,
                                               double mx, int ni, int pi, double& il, double& iu) {
  double tmin, tmax;
  if (a >= 0.0) { tmin = a * lj; tmax = a * uj; } else { tmin = a * uj; tmax = a * lj; }
  double rmin, rmax;
  if (isfinite(tmin)) rmin = ni == 0 ? mn - tmin : -INFINITY;
  else if (tmin < 0.0) rmin = ni > 1 ? -INFINITY : mn;
  else rmin = mn;
  if (isfinite(tmax)) rmax = pi == 0 ? mx - tmax : INFINITY;
  else if (tmax > 0.0) rmax = pi > 1 ? INFINITY : mx;
  else rmax = mx;
  il = -INFINITY;
  iu = INFINITY;
  if (a > 0.0) {
    if (isfinite(al) && isfinite(rmax)) il = (al - rmax) / a;
    if (isfinite(au) && isfinite(rmin)) iu = (au - rmin) / a;
  } else {
    if (isfinite(au) && isfinite(rmin)) il = (au - rmin) / a;
    if (isfinite(al) && isfinite(rmax)) iu = (al - rmax) / a;
  }
}

// Where the candidates of a row's entries go: the row's sides, the live
// degrees (rows of one live entry are left to the singleton-row rule), and
// the per-column candidate bounds combined by order-free RED max / min.
struct CandSink {
  const double* AL;
  const double* AU;
  const int32_t* row_nnz;
  double* cand_l;
  double* cand_u;
  // Candidate bounds of column j from entry a (|a| above the zero
  // tolerance, column kept) of a row with sides al, au and activity summary
  // mn, mx, ni, pi; b holds the column's current bounds.
  __device__ __forceinline__ void entry(int j, double a, double2 b, double al, double au, double mn, double mx,
                                        int ni, int pi) const {
    const double ol = b.x, ou = b.y;
    double il, iu;
    implied_bounds(a, ol, ou, al, au, mn, mx, ni, pi, il, iu);
    double nl = ol, nu = ou;
    if (isfinite(il)) nl = fmax(nl, il);
    if (isfinite(iu)) nu = fmin(nu, iu);
    if (nl > ol) red_max_f64(&cand_l[j], nl);
    if (nu < ou) red_min_f64(&cand_u[j], nu);
  }
};

}  // namespace gpp
