// physics.cuh -- device-side physics of the ECHO-QGP step: equation of
// state, reconstruction, fluxes, sources, primitive<->conserved maps.
//
// Every routine restates a reference Fortran routine (file:line given on
// each) with the same operation order and parenthesisation, so that a build
// with -fmad=false reproduces the CPU restatement bit for bit (IEEE division
// and square root are correctly rounded on both sides).  The `KIND`
// template parameter selects the equation set at compile time:
//   KIND_HD      ideal hydro, nv = 5
//   KIND_VISC    Israel-Stewart viscous hydro, nv = 12
//   KIND_MHD     ideal MHD, nv = 8
//   KIND_MHDGLM  ideal MHD with GLM divergence cleaning, nv = 9
//   KIND_RES     resistive MHD (E a primitive) with GLM, nv = 12
#pragma once

#include <cstdint>
#include <math.h>

#include "../../include/echo_gpu.h"

namespace echo {

enum { KIND_HD = 0, KIND_VISC = 1, KIND_MHD = 2, KIND_MHDGLM = 3, KIND_RES = 4 };

template <int KIND>
struct Traits;
template <>
struct Traits<KIND_HD> {
  static constexpr int NV = 5, KG = -1;
  static constexpr bool MHD = false, VISC = false, GLM = false, RES = false;
};
template <>
struct Traits<KIND_VISC> {
  static constexpr int NV = 12, KG = -1;
  static constexpr bool MHD = false, VISC = true, GLM = false, RES = false;
};
template <>
struct Traits<KIND_MHD> {
  static constexpr int NV = 8, KG = -1;
  static constexpr bool MHD = true, VISC = false, GLM = false, RES = false;
};
template <>
struct Traits<KIND_MHDGLM> {
  static constexpr int NV = 9, KG = 8;
  static constexpr bool MHD = true, VISC = false, GLM = true, RES = false;
};
// resistive runs (MHD = 2): B, E, psi (system.f90:92-105, 113-116)
template <>
struct Traits<KIND_RES> {
  static constexpr int NV = 12, KG = 11;
  static constexpr bool MHD = true, VISC = false, GLM = true, RES = true;
};

// variable indices (common.f90:63), 0-based
enum { KRH = 0, KVX = 1, KVY = 2, KVZ = 3, KPR = 4, KPIBU = 5, KPIXY = 6, KPIXZ = 7,
       KPIYZ = 8, KPIXX = 9, KPIYY = 10, KPIZZ = 11 };
enum { KBX = 5, KBY = 6, KBZ = 7, KGLM = 8 };  // KGLM: ideal MHD; Traits<K>::KG in general
enum { KEX = 8, KEY = 9, KEZ = 10 };              // resistive E^i
// derivative indices (common.f90:70-71), 0-based
enum { DTX = 0, DTY, DTZ, DXX, DXY, DXZ, DYX, DYY, DYZ, DZX, DZY, DZZ, DTT, DXT, DYT, DZT, NDER = 16 };

// Parameters and per-step metric, passed by value to every kernel.
struct DevPhys {
  int eqstate, coordinates, recal, obtained_zz, init_type, bulkvis;
  int nt;
  const double* __restrict__ tT;
  const double* __restrict__ te;
  const double* __restrict__ tp;
  const double* __restrict__ tc;
  // bracket accelerators for te and tp (see tab_bracket); null = plain search
  const int* __restrict__ bke;
  const int* __restrict__ bkp;
  long long bke0, bkp0;
  int nbke, nbkp;
  // product build: slopes of every table interval, de/dp, d(c_s^2)/de and
  // dp/de (null: interpolate with divisions, as the reference does)
  const double* __restrict__ sl_ep;
  const double* __restrict__ sl_ce;
  const double* __restrict__ sl_pe;
  double maxspeed, eta_over_s, tau_pi_coeff, enezero, przero, glm_alpha;
  double sigma_el, sigma_chiral;  // resistive runs: conductivities (code units)
};

// metric (system_metric_*, system.f90:132-160), derived from t on device.
// g_11 = g_22 = 1 in both coordinate systems of the reference (Minkowski
// and Bjorken), so they are compile-time ones: x * 1.0 is exactly x, and
// the multiplications the reference writes with them drop out.
struct Metric {
  static constexpr double g1 = 1.0, g2 = 1.0;
  double g3, gp, gm, g0, t, t3, ig3;
};

__device__ __forceinline__ Metric make_metric(int coordinates, double t, double t3) {
  Metric m;
  m.g0 = -1.;
  m.t = t;
  m.t3 = t3;
  if (coordinates == ECHO_BJORKEN) {
    m.g3 = t * t;
    m.gp = t;
    m.gm = 1. / m.gp;
  } else {
    m.g3 = 1.;
    m.gp = 1.;
    m.gm = 1.;
  }
  m.ig3 = 1. / m.g3;
  return m;
}

// x / g3 and x / gp as the reference writes them; the product build
// multiplies by the reciprocals, computed once per thread
__device__ __forceinline__ double over_g3(const Metric& M, double x) {
#ifdef ECHO_EXACT
  return x / M.g3;
#else
  return x * M.ig3;
#endif
}
__device__ __forceinline__ double over_gp(const Metric& M, double x) {
#ifdef ECHO_EXACT
  return x / M.gp;
#else
  return x * M.gm;
#endif
}

// ---------------------------------------------------------------------------
// equation of state (eos.f90)
// ---------------------------------------------------------------------------

// the bracket search of eos.f90:430-442; returns indxh (1-based)
__device__ __forceinline__ int tab_search(const double* __restrict__ arr, int n, double val) {
  int lo = 1, hi = n, mid = (lo + hi) / 2;
  while (lo + 1 != hi) {
    if (val > __ldg(arr + mid - 1)) {
      lo = mid;
    } else {
      hi = mid;
    }
    mid = (lo + hi) / 2;
  }
  return hi;
}

// The bracket of the search above in O(1): the index of a positive double's
// bit pattern >> BK_SHIFT is monotonic in its value (128 buckets per binade);
// bk[b] holds, for bucket b, a lower bound of the bracket of every value in
// the bucket, built on the host from the table itself.  A short forward scan
// then lands on exactly the index the binary search returns:
// max(2, smallest i with arr(i) >= val) for arr(1) <= val <= arr(n).
#define BK_SHIFT 45
__device__ __forceinline__ int tab_bracket(const double* __restrict__ arr, const int* __restrict__ bk,
                                           long long k0, int nb, int n, double val) {
  if (bk == nullptr) return tab_search(arr, n, val);
  long long key = (__double_as_longlong(val) >> BK_SHIFT) - k0;
  key = key < 0 ? 0 : (key >= nb ? nb - 1 : key);
  int h = __ldg(bk + key);
  while (h < n && __ldg(arr + h - 1) < val) h++;
  return h;
}
#define SEARCH_E(P, val) tab_bracket((P).te, (P).bke, (P).bke0, (P).nbke, (P).nt, (val))
#define SEARCH_P(P, val) tab_bracket((P).tp, (P).bkp, (P).bkp0, (P).nbkp, (P).nt, (val))

// eos_energy: get_energy (eos.f90:468-523) / eos_energy_ana (eos.f90:1104-1185)
__device__ __forceinline__ int eos_energy(const DevPhys& P, double rh, double* en, double pr) {
  if (P.eqstate == ECHO_EOS_TABLE) {
    if (pr < __ldg(P.tp)) return 125;
    if (pr > __ldg(P.tp + P.nt - 1)) return 126;
    int h = SEARCH_P(P, pr);
#ifndef ECHO_EXACT
    if (P.sl_ep) {
      *en = __ldg(P.te + h - 2) + (pr - __ldg(P.tp + h - 2)) * __ldg(P.sl_ep + h - 2);
      return 0;
    }
#endif
    double p2 = __ldg(P.tp + h - 1), p1 = __ldg(P.tp + h - 2);
    double e2 = __ldg(P.te + h - 1), e1 = __ldg(P.te + h - 2);
    *en = e1 + (e2 - e1) * (pr - p1) / (p2 - p1);
    return 0;
  }
  if (pr <= P.przero) {
    *en = P.enezero * pr / P.przero;
    return 0;
  }
  if (P.eqstate == ECHO_EOS_CONFORMAL)
    *en = 3. * pr;
  else
    *en = rh + pr / (4.0 / 3.0 - 1.);
  return 0;
}

// eos_pressure: get_pressure (eos.f90:399-464) / eos_pressure_ana (eos.f90:886-922)
__device__ __forceinline__ int eos_pressure(const DevPhys& P, double rh, double en, double* pr,
                                            double* dprdrh, double* dprden) {
  if (P.eqstate == ECHO_EOS_TABLE) {
    if (en < __ldg(P.te)) return 123;
    if (en > __ldg(P.te + P.nt - 1)) return 124;
    int h = SEARCH_E(P, en);
#ifndef ECHO_EXACT
    if (P.sl_pe) {  // dp/de = (dp/dT)/(de/dT) of the interval, precomputed
      double sl = __ldg(P.sl_pe + h - 2);
      *pr = __ldg(P.tp + h - 2) + (en - __ldg(P.te + h - 2)) * sl;
      *dprdrh = 0;
      *dprden = sl;
      return 0;
    }
#endif
    double p2 = __ldg(P.tp + h - 1), p1 = __ldg(P.tp + h - 2);
    double e2 = __ldg(P.te + h - 1), e1 = __ldg(P.te + h - 2);
    double t2 = __ldg(P.tT + h - 1), t1 = __ldg(P.tT + h - 2);
    *pr = p1 + (p2 - p1) * (en - e1) / (e2 - e1);
    double dpt = (p2 - p1) / (t2 - t1);
    double det = (e2 - e1) / (t2 - t1);
    *dprdrh = 0;
    *dprden = dpt / det;
    return 0;
  }
  if (P.eqstate == ECHO_EOS_CONFORMAL) {
    double a = 3.0;
    *pr = en / a;
    *dprdrh = 0.;
    *dprden = 1. / 3.;
  } else {
    double gam = 4.0 / 3.0;
    *pr = (gam - 1.) * (en - rh);
    *dprdrh = -gam + 1.;
    *dprden = gam - 1.;
  }
  return 0;
}

#ifndef ECHO_EXACT
// Product build, the face states of system_flux: e(p) interpolated in the p
// interval of the bracket h (returned for eos_sound_at), with the interval's
// precomputed slope instead of a division.  h = 0 when the EoS is not a
// table with slopes (then eos_energy / eos_sound are used).
__device__ __forceinline__ int eos_energy_h(const DevPhys& P, double rh, double* en, double pr, int* h) {
  if (P.eqstate == ECHO_EOS_TABLE && P.sl_ep) {
    if (pr < __ldg(P.tp)) return 125;
    if (pr > __ldg(P.tp + P.nt - 1)) return 126;
    int hh = SEARCH_P(P, pr);
    *en = __ldg(P.te + hh - 2) + (pr - __ldg(P.tp + hh - 2)) * __ldg(P.sl_ep + hh - 2);
    *h = hh;
    return 0;
  }
  *h = 0;
  return eos_energy(P, rh, en, pr);
}
// c_s^2(e) for the e just interpolated in bracket h: e lies in the same
// interval of the e column (e(p) is monotonic; at a node both neighbouring
// intervals give the node value), so get_sound's search is skipped
__device__ __forceinline__ double eos_sound_at(const DevPhys& P, int h, double en) {
  return __ldg(P.tc + h - 2) + (en - __ldg(P.te + h - 2)) * __ldg(P.sl_ce + h - 2);
}
#endif

// eos_sound: get_sound (eos.f90:590-641) / eos_sound_ana (eos.f90:926-952)
__device__ __forceinline__ int eos_sound(const DevPhys& P, double rh, double en, double pr, double* cs2) {
  if (P.eqstate == ECHO_EOS_TABLE) {
    if (en < __ldg(P.te)) return 131;
    if (en > __ldg(P.te + P.nt - 1)) return 132;
    int h = SEARCH_E(P, en);
#ifndef ECHO_EXACT
    if (P.sl_ce) {
      *cs2 = __ldg(P.tc + h - 2) + (en - __ldg(P.te + h - 2)) * __ldg(P.sl_ce + h - 2);
      return 0;
    }
#endif
    double s2 = __ldg(P.tc + h - 1), s1 = __ldg(P.tc + h - 2);
    double e2 = __ldg(P.te + h - 1), e1 = __ldg(P.te + h - 2);
    *cs2 = s1 + (s2 - s1) * (en - e1) / (e2 - e1);
    return 0;
  }
  double dprden, dprdrh;
  if (P.eqstate == ECHO_EOS_CONFORMAL) {
    dprden = 1. / 3.;
    dprdrh = 0.;
  } else {
    double gam = 4.0 / 3.0;
    dprden = gam - 1.;
    dprdrh = -gam + 1.;
  }
  double c;
  if (en + pr == 0)
    c = dprden;
  else
    c = dprden + (rh / (en + pr)) * dprdrh;
  *cs2 = c > 0.0 ? c : 0.0;
  return 0;
}

// get_derived_data: get_derived_data_tab (eos.f90:645-701) / _ana (eos.f90:956-968)
__device__ __forceinline__ int get_derived_data(const DevPhys& P, double rh, double pr, double* en,
                                                double* temp, double* s) {
  if (P.eqstate == ECHO_EOS_TABLE) {
    if (pr < __ldg(P.tp)) return 135;
    if (pr > __ldg(P.tp + P.nt - 1)) return 136;
    int h = SEARCH_P(P, pr);
    double p2 = __ldg(P.tp + h - 1), p1 = __ldg(P.tp + h - 2);
    double e2 = __ldg(P.te + h - 1), e1 = __ldg(P.te + h - 2);
    double t2 = __ldg(P.tT + h - 1), t1 = __ldg(P.tT + h - 2);
    double fac = (pr - p1) / (p2 - p1);
    *temp = t1 + (t2 - t1) * fac;
    *en = e1 + (e2 - e1) * fac;
    *s = (*en + pr) / *temp;
    return 0;
  }
  int err = eos_energy(P, rh, en, pr);
  *temp = 0.148909 * pow(*en, 0.25);
  if (*temp == 0)
    *s = 0.;
  else
    *s = (*en + pr) / *temp;
  return err;
}

// ---------------------------------------------------------------------------
// reconstruction (holib.f90)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double fsign1(double d) { return copysign(1.0, d); }

__device__ __forceinline__ double mm2(double d1, double d2) {  // holib.f90:440-452
  double s1 = fsign1(d1), s2 = fsign1(d2);
  double a1 = fabs(d1), a2 = fabs(d2);
  return .5 * (s1 + s2) * (a1 < a2 ? a1 : a2);
}
__device__ __forceinline__ double fmin3(double a, double b, double c) {
  double r = a;
  if (b < r) r = b;
  if (c < r) r = c;
  return r;
}
__device__ __forceinline__ double fmax3(double a, double b, double c) {
  double r = a;
  if (b > r) r = b;
  if (c > r) r = c;
  return r;
}
__device__ __forceinline__ double mm4(double d1, double d2, double d3, double d4) {  // :472-486
  double s1 = fsign1(d1), s2 = fsign1(d2), s3 = fsign1(d3), s4 = fsign1(d4);
  double m = fabs(d1);
  if (fabs(d2) < m) m = fabs(d2);
  if (fabs(d3) < m) m = fabs(d3);
  if (fabs(d4) < m) m = fabs(d4);
  return .125 * (s1 + s2) * fabs((s1 + s3) * (s1 + s4)) * m;
}
__device__ __forceinline__ double ceno3(double d0, double d1, double d2) {  // :490-510
  const double alpha = 0.7;
  double r = 0.;
  int s = (int)fsign1(d0) + (int)fsign1(d1) + (int)fsign1(d2);
  if (abs(s) == 3) {
    double w0 = fabs(d0), w1 = alpha * fabs(d1), w2 = fabs(d2);
    double wm = w0;
    r = d0;
    if (w1 < wm) {
      wm = w1;
      r = d1;
    }
    if (w2 < wm) {
      wm = w2;
      r = d2;
    }
  }
  return r;
}
__device__ __forceinline__ double mp5(double f, double f1, double f2, double f3, double f4, double f5) {
  double r = f;  // holib.f90:514-536
  double ful = f3 + 2 * (f3 - f2);
  double fmp = f3 + mm2(f4 - f3, ful - f3);
  if ((f - f3) * (f - fmp) > 0.) {
    double dm = f1 - 2 * f2 + f3;
    double d0 = f2 - 2 * f3 + f4;
    double dp = f3 - 2 * f4 + f5;
    double fmd = .5 * (f3 + f4) - .5 * mm4(4 * d0 - dp, 4 * dp - d0, d0, dp);
    double flc = f3 + .5 * (f3 - f2) + (4. / 3.) * mm4(4 * d0 - dm, 4 * dm - d0, d0, dm);
    double lo1 = fmin3(f3, f4, fmd), lo2 = fmin3(f3, ful, flc);
    double hi1 = fmax3(f3, f4, fmd), hi2 = fmax3(f3, ful, flc);
    double fmin = lo1 > lo2 ? lo1 : lo2;
    double fmax = hi1 < hi2 ? hi1 : hi2;
    r = f + mm2(fmin - f, fmax - f);
  }
  return r;
}

// WENO5 one side: f1..f5 in the reference's naming (holib.f90:198-212)
#ifndef ECHO_EXACT
// Product build: the same weights with the common denominator multiplied
// through, sum_k d_k p_k / q_k^2 / sum_k d_k / q_k^2 =
// sum_k d_k p_k Q_j Q_l / sum_k d_k Q_j Q_l with Q = q^2 (Q >= 1e-12, so
// the products cannot underflow), and the two sides of a face sharing one
// division: gl = nl/dl, gr = nr/dr = (nl dr, nr dl) / (dl dr), where
// dl, dr >= 3e-24 and stay far below 1e150 for the values a run holds.
__device__ __forceinline__ void weno5_nd(double f1, double f2, double f3, double f4, double f5, double& num,
                                         double& den) {
  // The smoothness indicators beta_k / 12 + eps = 13/12 t1^2 + 1/4 t2^2 + eps
  // as two fused multiply-adds each, the sub-stencil polynomials with the
  // factor 1/8 and the linear weights 10 and 5 of p2 and p3 folded into their
  // (exactly representable) coefficients, and the denominator sum_k d_k Q_j Q_l
  // with d = (1, 10, 5): the same weights with fewer FP64 instructions.
  const double eps = 1.e-6, c13 = 13. / 12.;
  double t1, t2, q1, q2, q3;
  t1 = f3 - 2 * f2 + f1;
  t2 = fma(3., f3, fma(-4., f2, f1));
  q1 = fma(c13 * t1, t1, fma(0.25 * t2, t2, eps));
  t1 = f4 - 2 * f3 + f2;
  t2 = f4 - f2;
  q2 = fma(c13 * t1, t1, fma(0.25 * t2, t2, eps));
  t1 = f5 - 2 * f4 + f3;
  t2 = fma(3., f3, fma(-4., f4, f5));
  q3 = fma(c13 * t1, t1, fma(0.25 * t2, t2, eps));
  double Q1 = q1 * q1, Q2 = q2 * q2, Q3 = q3 * q3;
  double w1 = Q2 * Q3, w2 = Q1 * Q3, w3 = Q1 * Q2;
  double p1 = fma(1.875, f3, fma(-1.25, f2, 0.375 * f1));       // (3 f1 - 10 f2 + 15 f3) / 8
  double p2 = fma(3.75, f4, fma(7.5, f3, -1.25 * f2));          // 10 (-f2 + 6 f3 + 3 f4) / 8
  double p3 = fma(-0.625, f5, fma(3.75, f4, 1.875 * f3));       // 5 (3 f3 + 6 f4 - f5) / 8
  num = fma(w3, p3, fma(w2, p2, w1 * p1));
  den = fma(5., w3, fma(10., w2, w1));
}
// Cell-centred WENO5 (product build): both face states of one cell from its
// five-point stencil f1..f5 = v(c-2..c+2).  plus = the state at c+1/2 (the
// left state of the face above, holib.f90:198-212 on f1..f5), minus = the
// state at c-1/2 (the right state of the face below, the same formula on
// f5..f1).  The two orientations share their three smoothness indicators
// (the reversed stencil's first is the forward stencil's third) and the
// three products of the weights, and one division serves both.
__device__ __forceinline__ void weno5_cell(double f1, double f2, double f3, double f4, double f5, double& plus,
                                           double& minus) {
  const double eps = 1.e-6, c13 = 13. / 12.;
  double t1, t2;
  t1 = f3 - 2 * f2 + f1;
  t2 = fma(3., f3, fma(-4., f2, f1));
  const double qa = fma(c13 * t1, t1, fma(0.25 * t2, t2, eps));
  t1 = f4 - 2 * f3 + f2;
  t2 = f4 - f2;
  const double qb = fma(c13 * t1, t1, fma(0.25 * t2, t2, eps));
  t1 = f5 - 2 * f4 + f3;
  t2 = fma(3., f3, fma(-4., f4, f5));
  const double qc = fma(c13 * t1, t1, fma(0.25 * t2, t2, eps));
  const double Qa = qa * qa, Qb = qb * qb, Qc = qc * qc;
  const double wbc = Qb * Qc, wac = Qa * Qc, wab = Qa * Qb;
  // forward: weights (wbc, 10 wac, 5 wab); reversed: (wab, 10 wac, 5 wbc)
  const double p1 = fma(1.875, f3, fma(-1.25, f2, 0.375 * f1));
  const double p2 = fma(3.75, f4, fma(7.5, f3, -1.25 * f2));
  const double p3 = fma(-0.625, f5, fma(3.75, f4, 1.875 * f3));
  const double r1 = fma(1.875, f3, fma(-1.25, f4, 0.375 * f5));
  const double r2 = fma(3.75, f2, fma(7.5, f3, -1.25 * f4));
  const double r3 = fma(-0.625, f1, fma(3.75, f2, 1.875 * f3));
  const double np = fma(wab, p3, fma(wac, p2, wbc * p1));
  const double dp = fma(5., wab, fma(10., wac, wbc));
  const double nm = fma(wbc, r3, fma(wac, r2, wab * r1));
  const double dm = fma(5., wbc, fma(10., wac, wab));
  const double inv = 1. / (dp * dm);
  plus = np * dm * inv;
  minus = nm * dp * inv;
}
__device__ __forceinline__ void weno5_face(const double s[6], double& gl, double& gr) {
  double nl, dl, nr, dr;
  weno5_nd(s[0], s[1], s[2], s[3], s[4], nl, dl);
  weno5_nd(s[5], s[4], s[3], s[2], s[1], nr, dr);
  double inv = 1. / (dl * dr);
  gl = nl * dr * inv;
  gr = nr * dl * inv;
}
#else
__device__ __forceinline__ double weno5_side(double f1, double f2, double f3, double f4, double f5) {
  const double d1 = 1 / 16., d2 = 10 / 16., d3 = 5 / 16., eps = 1.e-6;
  const double c11 = 3 / 8., c21 = -10 / 8., c31 = 15 / 8.;
  const double c12 = -1 / 8., c22 = 6 / 8., c32 = 3 / 8.;
  const double c13 = 3 / 8., c23 = 6 / 8., c33 = -1 / 8.;
  double t1, t2, b1, b2, b3, q, a1, a2, a3;
  t1 = f3 - 2 * f2 + f1;
  t2 = 3. * f3 - 4. * f2 + f1;
  b1 = 13. * (t1 * t1) + 3. * (t2 * t2);
  t1 = f4 - 2 * f3 + f2;
  t2 = f4 - f2;
  b2 = 13. * (t1 * t1) + 3. * (t2 * t2);
  t1 = f5 - 2 * f4 + f3;
  t2 = f5 - 4. * f4 + 3. * f3;
  b3 = 13. * (t1 * t1) + 3. * (t2 * t2);
  q = b1 / 12. + eps;
  a1 = d1 / (q * q);
  q = b2 / 12. + eps;
  a2 = d2 / (q * q);
  q = b3 / 12. + eps;
  a3 = d3 / (q * q);
  double p1 = c11 * f1 + c21 * f2 + c31 * f3;
  double p2 = c12 * f2 + c22 * f3 + c32 * f4;
  double p3 = c13 * f3 + c23 * f4 + c33 * f5;
  return (a1 * p1 + a2 * p2 + a3 * p3) / (a1 + a2 + a3);
}
#endif

__device__ __forceinline__ double weno3_side(double f1, double f2, double f3) {  // :149-158
  const double d1 = 1 / 3., d2 = 2 / 3., eps = 1.e-6;
  const double c11 = -1 / 2., c21 = 3 / 2., c12 = 1 / 2., c22 = 1 / 2.;
  double b1 = (f2 - f1) * (f2 - f1);
  double b2 = (f3 - f2) * (f3 - f2);
  double a1 = d1 / ((b1 + eps) * (b1 + eps));
  double a2 = d2 / ((b2 + eps) * (b2 + eps));
  double p1 = c11 * f1 + c21 * f2;
  double p2 = c12 * f2 + c22 * f3;
  return (a1 * p1 + a2 * p2) / (a1 + a2);
}

__device__ __forceinline__ double ceno3_side(double f1, double f2, double f3, double f4, double f5) {
  const double c11 = 3 / 8., c21 = -10 / 8., c31 = 15 / 8.;  // holib.f90:98-109
  const double c12 = -1 / 8., c22 = 6 / 8., c32 = 3 / 8.;
  const double c13 = 3 / 8., c23 = 6 / 8., c33 = -1 / 8.;
  double p = f3 + .5 * mm2(f3 - f2, f4 - f3);
  double d0 = c11 * f1 + c21 * f2 + c31 * f3 - p;
  double d1 = c12 * f2 + c22 * f3 + c32 * f4 - p;
  double d2 = c13 * f3 + c23 * f4 + c33 * f5 - p;
  return p + ceno3(d0, d1, d2);
}

__device__ __forceinline__ double ppm4_side(double f1, double f2, double f3, double f4) {  // :250-255
  return f2 + .5 * (f3 - f2) - .125 * (mm2(f4 - f3, f3 - f2) - mm2(f3 - f2, f2 - f1));
}

// Left and right states at face i+1/2 from the 6-point stencil
// s[0..5] = f(i-2..i+3) (work_rec, work.f90:420-525).
__device__ __forceinline__ void recon_any(int recal, const double s[6], double& gl, double& gr) {
  switch (recal) {
    case ECHO_REC_TVD2: {  // holib.f90:47-77, rewritten per face
      gl = s[2] + .5 * mm2(s[2] - s[1], s[3] - s[2]);
      gr = s[3] - .5 * mm2(s[3] - s[2], s[4] - s[3]);
      break;
    }
    case ECHO_REC_CENO3:
      gl = ceno3_side(s[0], s[1], s[2], s[3], s[4]);
      gr = ceno3_side(s[5], s[4], s[3], s[2], s[1]);
      break;
    case ECHO_REC_WENO3:
      gl = weno3_side(s[1], s[2], s[3]);
      gr = weno3_side(s[4], s[3], s[2]);
      break;
    case ECHO_REC_WENO5:
#ifdef ECHO_EXACT
      gl = weno5_side(s[0], s[1], s[2], s[3], s[4]);
      gr = weno5_side(s[5], s[4], s[3], s[2], s[1]);
#else
      weno5_face(s, gl, gr);
#endif
      break;
    case ECHO_REC_PPM4:
      gl = ppm4_side(s[1], s[2], s[3], s[4]);
      gr = ppm4_side(s[4], s[3], s[2], s[1]);
      break;
    case ECHO_REC_MPE3: {  // holib.f90:272-294
      const double d1 = -1 / 8., d2 = 6 / 8., d3 = 3 / 8.;
      double l = d1 * s[1] + d2 * s[2] + d3 * s[3];
      double r = d1 * s[4] + d2 * s[3] + d3 * s[2];
      gl = mp5(l, s[0], s[1], s[2], s[3], s[4]);
      gr = mp5(r, s[5], s[4], s[3], s[2], s[1]);
      break;
    }
    default: {  // MPE5, holib.f90:298-320
      const double d1 = 3 / 128., d2 = -20 / 128., d3 = 90 / 128., d4 = 60 / 128., d5 = -5 / 128.;
      double l = d1 * s[0] + d2 * s[1] + d3 * s[2] + d4 * s[3] + d5 * s[4];
      double r = d1 * s[5] + d2 * s[4] + d3 * s[3] + d4 * s[2] + d5 * s[1];
      gl = mp5(l, s[0], s[1], s[2], s[3], s[4]);
      gr = mp5(r, s[5], s[4], s[3], s[2], s[1]);
      break;
    }
  }
}

// The reconstruction fixed at compile time (REC = ECHO_REC_*) or chosen at
// run time (REC = REC_RUNTIME).  The face kernels reconstruct every
// variable with an unrolled loop; a run-time switch inside it puts all seven
// schemes into the kernel once per variable, so the common scheme gets a
// kernel of its own.
enum { REC_RUNTIME = -1 };
template <int REC>
__device__ __forceinline__ void recon_face(int recal, const double s[6], double& gl, double& gr) {
  recon_any(REC >= 0 ? REC : recal, s, gl, gr);
}

// ---------------------------------------------------------------------------
// viscous helpers (viscous.f90)
// ---------------------------------------------------------------------------
struct Pit {
  double tt, tx, ty, tz, zz;
};

// get_derived_pi (viscous.f90:244-255)
__device__ __forceinline__ void derived_pi(const Metric& M, const double* p, Pit& o) {
  double g1 = M.g1, g2 = M.g2, g3 = M.g3;
  o.tx = p[KPIXX] * p[KVX] * g1 + p[KPIXY] * p[KVY] * g2 + p[KPIXZ] * p[KVZ] * g3;
  o.ty = p[KPIXY] * p[KVX] * g1 + p[KPIYY] * p[KVY] * g2 + p[KPIYZ] * p[KVZ] * g3;
  o.tz = p[KPIXZ] * p[KVX] * g1 + p[KPIYZ] * p[KVY] * g2 + p[KPIZZ] * p[KVZ] * g3;
  o.tt = o.tx * p[KVX] * g1 + o.ty * p[KVY] * g2 + o.tz * p[KVZ] * g3;
  o.zz = p[KPIZZ];
}

// get_derived_pi_zz (viscous.f90:259-279)
__device__ __forceinline__ void derived_pi_zz(const Metric& M, const double* p, Pit& o) {
  double g1 = M.g1, g2 = M.g2, g3 = M.g3;
  double vx = p[KVX], vy = p[KVY], vz = p[KVZ];
  double pixy = p[KPIXY], pixx = p[KPIXX], piyy = p[KPIYY], piyz = p[KPIYZ], pixz = p[KPIXZ];
  if (vz == 0.) {
    // v^eta = 0 (every cell of a boost-invariant run): the terms below with
    // a factor vz are exact zeros and 1 - vz^2 g3 is exactly 1, so these are
    // the same sums in the same order, with the same bits
    o.tt = vx * g1 * pixy * vy * g2 + vx * vx * g1 * g1 * pixx + vy * g1 * g1 * pixy * vx + vy * vy * g1 * piyy * g2;
    o.tx = pixx * vx * g1 + pixy * vy * g2;
    o.ty = pixy * vx * g1 + piyy * vy * g2;
    o.tz = pixz * vx * g1 + piyz * vy * g2;
    o.zz = 1. / g3 *
           (vx * g1 * pixy * vy * g2 - pixx * g1 - piyy * g2 + vx * vx * g1 * g1 * pixx + vy * g1 * g1 * pixy * vx +
            vy * vy * g1 * piyy * g2);
    return;
  }
  o.tt = 1. / (1. - vz * vz * g3) *
         (vx * g1 * pixy * vy * g2 + vx * vx * g1 * g1 * pixx + vy * g1 * piyz * vz * g3 +
          2. * vx * g1 * pixz * vz * g3 + vy * g1 * g1 * pixy * vx + vy * vy * g1 * piyy * g2 +
          vz * g3 * piyz * vy * g2 - pixx * g1 * vz * vz * g3 - piyy * g2 * vz * vz * g3);
  o.tx = pixx * vx * g1 + pixy * vy * g2 + pixz * vz * g3;
  o.ty = pixy * vx * g1 + piyy * vy * g2 + piyz * vz * g3;
  o.tz = 1. / (1. - vz * vz * g3) *
         (pixz * vx * g1 + pixz * vx * g1 * vz * vz * g3 + piyz * vy * g2 +
          vz * vx * g1 * pixy * vy * g2 - vz * pixx * g1 - vz * piyy * g2 +
          vz * vx * vx * g1 * g1 * pixx + vy * g1 * piyz * vz * vz * g3 +
          vz * vy * g1 * g1 * pixy * vx + vz * vy * vy * g1 * piyy * g2);
  o.zz = 1. / (g3 * (1. - vz * vz * g3)) *
         (vx * g1 * pixy * vy * g2 - pixx * g1 - piyy * g2 + vx * vx * g1 * g1 * pixx +
          vy * g1 * piyz * vz * g3 + 2. * vx * g1 * pixz * vz * g3 + vy * g1 * g1 * pixy * vx +
          vy * vy * g1 * piyy * g2 + vz * g3 * piyz * vy * g2);
}

__device__ __forceinline__ void derived_pi_any(const DevPhys& P, const Metric& M, double* p, Pit& o) {
  if (P.obtained_zz) {
    derived_pi_zz(M, p, o);
    p[KPIZZ] = o.zz;
  } else {
    derived_pi(M, p, o);
  }
}

// get_viscous_parameters (viscous.f90:172-199)
__device__ __forceinline__ int viscous_parameters(const DevPhys& P, double dens, double press,
                                                  double* eta, double* zeta, double* tau_pi,
                                                  double* tau_pi_big) {
  double en = 0, temp = 0, s = 0, cs2 = 0;
  (void)get_derived_data(P, dens, press, &en, &temp, &s);
  int err = eos_sound(P, dens, en, press, &cs2);
  const double hbar = 0.197326;
  *eta = hbar * P.eta_over_s * s;
  if (P.init_type == 2) *eta = P.eta_over_s;
  if (P.bulkvis)
    *zeta = 2. * *eta * (1. / 3. - cs2);
  else
    *zeta = 0.;
  if (temp == 0 || s == 0)
    *tau_pi = 0.;
  else
    *tau_pi = P.tau_pi_coeff * *eta / (temp * s);
  if (P.init_type == 5) *tau_pi = 5. * *eta / (temp * s);
  *tau_pi_big = *tau_pi;
  return err;
}

// ---------------------------------------------------------------------------
// electromagnetic helpers (system.f90:1846-1897)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void e_ideal(const Metric& M, double vx, double vy, double vz, double bx,
                                        double by, double bz, double E[3]) {
  double gp = M.gp;
  E[0] = -gp * (vy * bz - vz * by);
  E[1] = -gp * (vz * bx - vx * bz);
  E[2] = -gp * (vx * by - vy * bx);
}
__device__ __forceinline__ void exb(const Metric& M, const double E[3], double bx, double by, double bz,
                                    double o[3]) {
  double e0 = E[0], e1 = E[1], e2 = over_g3(M, E[2]), gp = M.gp;
  o[0] = gp * (e1 * bz - e2 * by);
  o[1] = gp * (e2 * bx - e0 * bz);
  o[2] = gp * (e0 * by - e1 * bx);
}
// covariant E_i of a cell: the resistive primitive E^i lowered
// (system.f90:203-205; the reference's system_flux omits g_33 for E_3,
// system.f90:1365, which only Minkowski coordinates forgive), or -v x B
template <int KIND>
__device__ __forceinline__ void e_field(const Metric& M, const double* v, double E[3]) {
  if (Traits<KIND>::RES) {
    E[0] = v[KEX];
    E[1] = v[KEY];
    E[2] = v[KEZ] * M.g3;
  } else {
    e_ideal(M, v[KVX], v[KVY], v[KVZ], v[KBX], v[KBY], v[KBZ], E);
  }
}

// ---------------------------------------------------------------------------
// system_prim2cons (system.f90:164-263)
// ---------------------------------------------------------------------------
template <int KIND>
__device__ __forceinline__ int prim2cons(const DevPhys& P, const Metric& M, double* v, double* u) {
  typedef Traits<KIND> T;
  double g1 = M.g1, g2 = M.g2, g3 = M.g3, gp = M.gp;
  double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR];
  double en = 0;
  int err = eos_energy(P, rh, &en, pr);
  if (err) return err;
  double v2 = g1 * vx * vx + g2 * vy * vy + g3 * vz * vz;
  double glf = 1. / sqrt(1. - v2);
  double w = en + pr;
  double ww = w * (glf * glf);
  u[KRH] = rh * glf;
  if (T::VISC) {
    w = w + v[KPIBU];
    ww = w * (glf * glf);
    Pit pi;
    derived_pi_any(P, M, v, pi);
    u[KVX] = (ww * vx + pi.tx);
    u[KVY] = (ww * vy + pi.ty);
    u[KVZ] = (ww * vz + pi.tz) * g3;
    u[KPR] = ww - pr - v[KPIBU] - pi.tt * M.g0;
    u[KPIBU] = v[KPIBU] * u[KRH];
    u[KPIZZ] = v[KPIZZ] * u[KRH];
    u[KPIXZ] = v[KPIXZ] * u[KRH];
    u[KPIXY] = v[KPIXY] * u[KRH];
    u[KPIYZ] = v[KPIYZ] * u[KRH];
    u[KPIXX] = v[KPIXX] * u[KRH];
    u[KPIYY] = v[KPIYY] * u[KRH];
  } else if (T::MHD) {
    double E[3], EXB[3];
    e_field<KIND>(M, v, E);
    double E2 = E[0] * E[0] + E[1] * E[1] + (E[2] * E[2]) / g3;
    exb(M, E, v[KBX], v[KBY], v[KBZ], EXB);
    double bx = v[KBX], by = v[KBY], bz = v[KBZ];
    double B2 = bx * bx + by * by + (bz * bz) * g3;
    double EEM = 0.5 * (E2 + B2);
    u[KVX] = ww * vx + EXB[0];
    u[KVY] = ww * vy + EXB[1];
    u[KVZ] = ww * vz * g3 + EXB[2];
    u[KPR] = ww - pr + EEM;
    u[KBX] = v[KBX];
    u[KBY] = v[KBY];
    u[KBZ] = v[KBZ];
    if (T::RES) {
      u[KEX] = v[KEX];
      u[KEY] = v[KEY];
      u[KEZ] = v[KEZ];
    }
    if (T::GLM) u[T::KG] = v[T::KG] / gp;
  } else {
    u[KVX] = ww * vx;
    u[KVY] = ww * vy;
    u[KVZ] = ww * vz * g3;
    u[KPR] = ww - pr;
  }
#pragma unroll
  for (int k = 0; k < T::NV; k++) u[k] = u[k] * gp;
  return 0;
}

// ---------------------------------------------------------------------------
// system_flux (system.f90:1316-1583); DIR 1..3
// ---------------------------------------------------------------------------
template <int KIND, int DIR>
__device__ __forceinline__ int system_flux(const DevPhys& P, const Metric& M, double* v, double* u,
                                           double* f, double& vfp, double& vfm) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  double g1 = M.g1, g2 = M.g2, g3 = M.g3, gp = M.gp, gm = M.gm;
  double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR];
  double en = 0;
#ifdef ECHO_EXACT
  int err = eos_energy(P, rh, &en, pr);
#else
  int hb = 0;
  int err = eos_energy_h(P, rh, &en, pr, &hb);
#endif
  if (err) return err;
  double v2 = g1 * vx * vx + g2 * vy * vy + g3 * vz * vz;
  if (v2 > 1) return 333;
#ifdef ECHO_EXACT
  double glf = 1. / sqrt(1. - v2);
#else
  double glf = rsqrt(1. - v2);
#endif
  double w, E[3] = {0, 0, 0}, EXB[3] = {0, 0, 0}, E2 = 0, B2 = 0, EEM = 0;
  Pit pi = {0, 0, 0, 0, 0};
  if (!T::VISC) {
    w = en + pr;
    if (T::MHD) {
      e_field<KIND>(M, v, E);
      E2 = E[0] * E[0] + E[1] * E[1] + over_g3(M, E[2] * E[2]);
      exb(M, E, v[KBX], v[KBY], v[KBZ], EXB);
      B2 = v[KBX] * v[KBX] + v[KBY] * v[KBY] + (v[KBZ] * v[KBZ]) * g3;
      EEM = 0.5 * (E2 + B2);
    }
  } else {
    w = en + pr + v[KPIBU];
  }
  double ww = w * (glf * glf);
  u[KRH] = rh * glf;
  if (T::VISC) {
    derived_pi_any(P, M, v, pi);
#pragma unroll
    for (int k = KPIBU; k < NV; k++) u[k] = v[k] * u[KRH];
    u[KVX] = ww * vx + pi.tx;
    u[KVY] = ww * vy + pi.ty;
    u[KVZ] = (ww * vz + pi.tz) * g3;
    u[KPR] = ww - pr - v[KPIBU] - pi.tt * M.g0;
  } else if (T::MHD) {
    u[KVX] = ww * vx + EXB[0];
    u[KVY] = ww * vy + EXB[1];
    u[KVZ] = ww * vz * g3 + EXB[2];
    u[KPR] = ww - pr + EEM;
    u[KBX] = v[KBX];
    u[KBY] = v[KBY];
    u[KBZ] = v[KBZ];
    if (T::RES) {
      u[KEX] = v[KEX];
      u[KEY] = v[KEY];
      u[KEZ] = v[KEZ];
    }
    if (T::GLM) u[T::KG] = over_gp(M, v[T::KG]);
  } else {
    u[KVX] = ww * vx;
    u[KVY] = ww * vy;
    u[KVZ] = ww * vz * g3;
    u[KPR] = ww - pr;
  }
  double wwdir, vdir, gcov_dir;
  if (DIR == 1) {
    wwdir = ww * vx;
    vdir = vx;
    gcov_dir = g1;
    f[KRH] = rh * glf * vx;
    if (T::VISC) {
      f[KVX] = wwdir * vx * g1 + pr + v[KPIBU] + v[KPIXX] * g1;
      f[KVY] = wwdir * vy * g2 + v[KPIXY] * g2;
      f[KVZ] = wwdir * vz * g3 + v[KPIXZ] * g3;
      f[KPR] = wwdir + pi.tx;
#pragma unroll
      for (int k = 5; k < NV; k++) f[k] = u[k] * vx;
    } else if (T::MHD) {
      f[KVX] = wwdir * vx - E[0] * E[0] - v[KBX] * v[KBX] + pr + EEM;
      f[KVY] = wwdir * vy - E[0] * E[1] - v[KBX] * v[KBY];
      f[KVZ] = wwdir * vz * g3 - E[0] * E[2] - v[KBX] * v[KBZ] * g3;
      f[KPR] = wwdir + EXB[0];
      f[KBX] = 0.;
      f[KBY] = -E[2] * gm;
      f[KBZ] = +E[1] * gm;
      if (T::RES) {  // E fluxes (system.f90:1450-1452)
        f[KEX] = 0.;
        f[KEY] = +v[KBZ] * g3 * gm;
        f[KEZ] = -v[KBY] * g2 * gm;
      }
      if (T::GLM) {
        f[KBX] = v[T::KG];
        f[T::KG] = over_gp(M, v[KBX]);
      }
    } else {
      f[KVX] = wwdir * vx * g1 + pr;
      f[KVY] = wwdir * vy * g2;
      f[KVZ] = wwdir * vz * g3;
      f[KPR] = wwdir;
    }
  } else if (DIR == 2) {
    wwdir = ww * vy;
    vdir = vy;
    gcov_dir = g2;
    f[KRH] = rh * glf * vy;
    if (T::VISC) {
      f[KVX] = wwdir * vx * g1 + v[KPIXY] * g1;
      f[KVY] = wwdir * vy * g2 + pr + v[KPIBU] + v[KPIYY] * g2;
      f[KVZ] = wwdir * vz * g3 + v[KPIYZ] * g3;
      f[KPR] = wwdir + pi.ty;
#pragma unroll
      for (int k = 5; k < NV; k++) f[k] = u[k] * vy;
    } else if (T::MHD) {
      f[KVX] = wwdir * vx - E[1] * E[0] - v[KBY] * v[KBX];
      f[KVY] = wwdir * vy - E[1] * E[1] - v[KBY] * v[KBY] + pr + EEM;
      f[KVZ] = wwdir * vz * g3 - E[1] * E[2] - v[KBY] * v[KBZ] * g3;
      f[KPR] = wwdir + EXB[1];
      f[KBX] = E[2] * gm;
      f[KBY] = 0.;
      f[KBZ] = -E[0] * gm;
      if (T::RES) {  // system.f90:1491-1493
        f[KEX] = -v[KBZ] * g3 * gm;
        f[KEY] = 0.;
        f[KEZ] = +v[KBX] * g1 * gm;
      }
      if (T::GLM) {
        f[KBY] = v[T::KG];
        f[T::KG] = over_gp(M, v[KBY]);
      }
    } else {
      f[KVX] = wwdir * vx * g1;
      f[KVY] = wwdir * vy * g2 + pr;
      f[KVZ] = wwdir * vz * g3;
      f[KPR] = wwdir;
    }
  } else {
    wwdir = ww * vz;
    vdir = vz;
    gcov_dir = g3;
    f[KRH] = rh * glf * vz;
    if (T::VISC) {
      f[KVX] = wwdir * vx * g1 + v[KPIXZ] * g1;
      f[KVY] = wwdir * vy * g2 + v[KPIYZ] * g2;
      f[KVZ] = wwdir * vz * g3 + pr + v[KPIBU] + v[KPIZZ] * g3;
      f[KPR] = wwdir + pi.tz;
#pragma unroll
      for (int k = 5; k < NV; k++) f[k] = u[k] * vz;
    } else if (T::MHD) {
      f[KVX] = wwdir * vx - over_g3(M, E[2]) * E[0] - v[KBZ] * v[KBX];
      f[KVY] = wwdir * vy - over_g3(M, E[2]) * E[1] - v[KBZ] * v[KBY];
      f[KVZ] = wwdir * vz * g3 - over_g3(M, E[2] * E[2]) - (v[KBZ] * v[KBZ]) * g3 + pr + EEM;
      f[KPR] = wwdir + over_g3(M, EXB[2]);
      f[KBX] = -E[1] * gm;
      f[KBY] = E[0] * gm;
      f[KBZ] = 0.;
      if (T::RES) {  // system.f90:1532-1534
        f[KEX] = +v[KBY] * g2 * gm;
        f[KEY] = -v[KBX] * g1 * gm;
        f[KEZ] = 0.;
      }
      if (T::GLM) {
        f[KBZ] = over_g3(M, v[T::KG]);
        f[T::KG] = over_gp(M, v[KBZ]);
      }
    } else {
      f[KVX] = wwdir * vx * g1;
      f[KVY] = wwdir * vy * g2;
      f[KVZ] = wwdir * vz * g3 + pr;
      f[KPR] = wwdir;
    }
  }
#pragma unroll
  for (int k = 0; k < NV; k++) u[k] = u[k] * gp;
#pragma unroll
  for (int k = 0; k < NV; k++) f[k] = f[k] * gp;
  double ca2;
  if (T::MHD) {
    double bb2 = B2 - E2;
    ca2 = bb2 / (bb2 + (en + pr));
  } else {
    ca2 = 0.;
  }
  double cs2 = 0;
#ifdef ECHO_EXACT
  err = eos_sound(P, rh, en, pr, &cs2);
#else
  if (hb)
    cs2 = eos_sound_at(P, hb, en);
  else
    err = eos_sound(P, rh, en, pr, &cs2);
#endif
  if (err) return err;
  double a2 = cs2 + ca2 - cs2 * ca2;
  double den = 1. / (1. - v2 * a2);
  double vf1 = den * (1. - a2) * vdir;
  // g_11 = g_22 = 1 in both metrics, so only the eta direction divides
  double hdir = DIR == 3 ? over_g3(M, 1. - v2 * a2) : (1. - v2 * a2);
  (void)gcov_dir;
  double vf2 = den * sqrt(a2 * (1. - v2) * (hdir - (1. - a2) * (vdir * vdir)));
  vfp = vf1 + vf2;
  vfm = vf1 - vf2;
  if (T::RES) {
    // resistive: the light cone bounds the Riemann fan of the E, B waves (the
    // reference keeps the ideal fast speed here, system.f90:1557-1580)
    vfp = 1. / sqrt(DIR == 3 ? g3 : 1.);
    vfm = -vfp;
  }
  return 0;
}

}  // namespace echo
