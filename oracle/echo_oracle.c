/*
 * echo_oracle.c -- CPU oracle (test infrastructure only) for ECHO-QGP's
 * per-step right-hand side and update.
 *
 * A restatement, routine by routine, of the reference Fortran:
 *   holib.f90    reconstructions and limiters
 *   work.f90     work_rec, work_glm[xyz], work_fup[xyz] (HLL)
 *   system.f90   system_metric, prim2cons, cons2prim (HD Newton, viscous
 *                nested Newton, MHD algo 1 = BRENTM), system_flux,
 *                system_source, E x B helpers, sist3
 *   viscous.f90  dts, get_viscous_parameters, get_derived_pi(_zz), get_sigma
 *   eos.f90      analytic (.def) and tabulated EoS lookups
 *   libacm554.f90 BRENTM (ACM TOMS 554)
 *   evolve.f90   evolve_main, evolve_df[xyz], evolve_src, evolve_dt,
 *                evolve_u2v, evolve_bc[xyz], evolve_glm_source,
 *                evolve_smooth_viscosity
 *   echo.f90     one iteration of the time loop
 *
 * Floating point follows gfortran -fdefault-real-8 semantics: every literal
 * is a double, expressions keep the reference's left-to-right grouping and
 * parentheses, integer powers x**2 and the real power x**2. are x*x (gcc
 * folds pow(x,2.0) exactly), other real powers call pow().  The file is
 * compiled with -ffp-contract=off so no multiply-add is fused: that is the
 * canonical arithmetic the CUDA parity build reproduces bit for bit.
 *
 * Where the reference reads memory it never wrote (uninitialised locals,
 * out-of-bounds neighbours in the con2prim repair at the domain edge), the
 * behaviour is undefined in Fortran; this restatement pins one definition
 * and the CUDA code uses the same one:
 *   - EoS table lookups out of range leave their outputs unchanged (locals
 *     start at 0) and return the reference error code;
 *   - the repair reads neighbours through the flat Fortran address
 *     (column-major, no bounds check) and reads 0 outside the allocation.
 *
 * Resistive RMHD (MHD=2) has no runnable reference path: the reference
 * forces algo_solver 7 and IMEX-SSP (common.f90:2109-2118) and then exits in
 * system_cons2prim, which has no algo-7 branch (system.f90:1160-1162).  Its
 * prim2cons, fluxes and sources for resistive runs exist and are restated
 * here (system.f90:199-212, 1360-1545, 1645-1661, 1747-1756, 1901-1919),
 * with E_3 = g_33 E^3 and metric-consistent cross products throughout (the
 * reference mixes co- and contravariant components in Bjorken coordinates;
 * the two agree in Minkowski coordinates).  The implicit Ohm's-law
 * con2prim and the implicit stage solves of IMEX-SSP3(4,3,3) are written
 * from their definitions (cons2prim_res, stage1_implicit).
 */
#include "echo_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NGC 3
#define PADP 4 /* pencil index offset: f(i) stored at [i + PADP] */

/* variable indices, 0-based (common.f90:63) */
enum {
  KRH = 0, KVX = 1, KVY = 2, KVZ = 3, KPR = 4,
  KPIBU = 5, KPIXY = 6, KPIXZ = 7, KPIYZ = 8, KPIXX = 9, KPIYY = 10, KPIZZ = 11
};
/* derivative indices (common.f90:70-72), 0-based */
enum {
  DTX = 0, DTY, DTZ, DXX, DXY, DXZ, DYX, DYY, DYZ, DZX, DZY, DZZ,
  DTT, DXT, DYT, DZT, NDERIV = 20
};
/* sigma indices (viscous.f90:47), 0-based */
enum { SXX = 0, SYY = 1, SZZ = 2, SXY = 3, SXZ = 4, SYZ = 5 };

/* ------------------------------------------------------------------------ */
/* physics context shared by the pointwise routines                         */
/* ------------------------------------------------------------------------ */
typedef struct Phys {
  const EchoParams* p;
  int nv, nu;
  int kbx, kby, kbz, kglm;
  int kex, key, kez; /* resistive E^i (system.f90:92-105) */
  double ohm_h;      /* a_ii dt of the implicit stage being solved, else 0 */
  /* metric (system_metric_*, system.f90:132-160) */
  double g1, g2, g3, gp, gm, g0;
  double t;
  /* EoS table (eos.f90:265-334) */
  int nt;
  const double *tT, *te, *tp, *tc;
} Phys;

static void phys_setup(Phys* ph, const EchoParams* p) {
  memset(ph, 0, sizeof(*ph));
  ph->p = p;
  int nv = p->viscosity ? 12 : 5; /* system_setup, system.f90:80-88 */
  ph->kbx = ph->kby = ph->kbz = ph->kglm = -1;
  ph->kex = ph->key = ph->kez = -1;
  if (p->mhd == 2) {
    nv += 6;
    ph->kbx = nv - 6;
    ph->kby = nv - 5;
    ph->kbz = nv - 4;
    ph->kex = nv - 3;
    ph->key = nv - 2;
    ph->kez = nv - 1;
    if (p->divclean) {
      nv += 1;
      ph->kglm = nv - 1;
    }
  } else if (p->mhd) {
    nv += 3;
    ph->kbx = nv - 3;
    ph->kby = nv - 2;
    ph->kbz = nv - 1;
    if (p->divclean) {
      nv += 1;
      ph->kglm = nv - 1;
    }
  }
  ph->nv = nv;
  ph->nu = nv;
  ph->g0 = -1.;
}

static void phys_metric(Phys* ph, double t) {
  ph->t = t;
  if (ph->p->coordinates == ECHO_BJORKEN) {
    ph->g1 = 1.;
    ph->g2 = 1.;
    ph->g3 = t * t;
    ph->gp = t;
    ph->gm = 1. / ph->gp;
  } else {
    ph->g1 = ph->g2 = ph->g3 = 1.;
    ph->gp = 1.;
    ph->gm = 1.;
  }
  ph->g0 = -1.;
}

/* ------------------------------------------------------------------------ */
/* EoS                                                                      */
/* ------------------------------------------------------------------------ */

/* binary search of eos.f90:430-442 (identical in every table routine):
 * returns indxh (1-based); indxl = indxh - 1 */
static int tab_search(const double* arr, int n, double val) {
  int lo = 1, hi = n, mid = (lo + hi) / 2;
  while (lo + 1 != hi) {
    if (val > arr[mid - 1]) {
      lo = mid;
      mid = (lo + hi) / 2;
    } else {
      hi = mid;
      mid = (lo + hi) / 2;
    }
  }
  return hi;
}

/* eos_energy: tabulated get_energy (eos.f90:468-523) or analytic
 * eos_energy_ana with NUM_DER=0 (eos.f90:1104-1185 + energy_den*.def) */
static int eos_energy(const Phys* ph, double rh, double* en, double pr) {
  const EchoParams* p = ph->p;
  if (p->eqstate == ECHO_EOS_TABLE) {
    if (pr < ph->tp[0]) return 125;
    if (pr > ph->tp[ph->nt - 1]) return 126;
    int h = tab_search(ph->tp, ph->nt, pr);
    double p2 = ph->tp[h - 1], p1 = ph->tp[h - 2];
    double e2 = ph->te[h - 1], e1 = ph->te[h - 2];
    *en = e1 + (e2 - e1) * (pr - p1) / (p2 - p1);
    return 0;
  }
  if (pr <= p->przero) { /* check_on_pressure branch, eos.f90:1118-1123 */
    *en = p->enezero * pr / p->przero;
    return 0;
  }
  if (p->eqstate == ECHO_EOS_CONFORMAL)
    *en = 3. * pr;
  else
    *en = rh + pr / (4.0 / 3.0 - 1.);
  return 0;
}

/* eos_pressure: get_pressure (eos.f90:399-464) or eos_pressure_ana
 * (eos.f90:886-922, pressure_vs_rh_en*.def, part_der_pr_vs_rh_en*.def) */
static int eos_pressure(const Phys* ph, double rh, double en, double* pr,
                        double* dprdrh, double* dprden) {
  const EchoParams* p = ph->p;
  if (p->eqstate == ECHO_EOS_TABLE) {
    if (en < ph->te[0]) return 123;
    if (en > ph->te[ph->nt - 1]) return 124;
    int h = tab_search(ph->te, ph->nt, en);
    double p2 = ph->tp[h - 1], p1 = ph->tp[h - 2];
    double e2 = ph->te[h - 1], e1 = ph->te[h - 2];
    double t2 = ph->tT[h - 1], t1 = ph->tT[h - 2];
    *pr = p1 + (p2 - p1) * (en - e1) / (e2 - e1);
    double dpt = (p2 - p1) / (t2 - t1);
    double det = (e2 - e1) / (t2 - t1);
    *dprdrh = 0;
    *dprden = dpt / det;
    return 0;
  }
  if (p->eqstate == ECHO_EOS_CONFORMAL) {
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

/* eos_sound: get_sound (eos.f90:590-641) or eos_sound_ana (eos.f90:926-952) */
static int eos_sound(const Phys* ph, double rh, double en, double pr,
                     double* cs2) {
  const EchoParams* p = ph->p;
  if (p->eqstate == ECHO_EOS_TABLE) {
    if (en < ph->te[0]) return 131;
    if (en > ph->te[ph->nt - 1]) return 132;
    int h = tab_search(ph->te, ph->nt, en);
    double s2 = ph->tc[h - 1], s1 = ph->tc[h - 2];
    double e2 = ph->te[h - 1], e1 = ph->te[h - 2];
    *cs2 = s1 + (s2 - s1) * (en - e1) / (e2 - e1);
    return 0;
  }
  double dprden, dprdrh;
  if (p->eqstate == ECHO_EOS_CONFORMAL) {
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

/* get_derived_data: get_derived_data_tab (eos.f90:645-701) or
 * get_derived_data_ana (eos.f90:956-968 with temperature.def) */
static int get_derived_data(const Phys* ph, double rh, double pr, double* en,
                            double* temp, double* s) {
  const EchoParams* p = ph->p;
  if (p->eqstate == ECHO_EOS_TABLE) {
    if (pr < ph->tp[0]) return 135;
    if (pr > ph->tp[ph->nt - 1]) return 136;
    int h = tab_search(ph->tp, ph->nt, pr);
    double p2 = ph->tp[h - 1], p1 = ph->tp[h - 2];
    double e2 = ph->te[h - 1], e1 = ph->te[h - 2];
    double t2 = ph->tT[h - 1], t1 = ph->tT[h - 2];
    double fac = (pr - p1) / (p2 - p1);
    *temp = t1 + (t2 - t1) * fac;
    *en = e1 + (e2 - e1) * fac;
    *s = (*en + pr) / *temp;
    return 0;
  }
  int err = eos_energy(ph, rh, en, pr);
  *temp = 0.148909 * pow(*en, 0.25);
  if (*temp == 0)
    *s = 0.;
  else
    *s = (*en + pr) / *temp;
  return err;
}

/* ------------------------------------------------------------------------ */
/* reconstruction (holib.f90)                                               */
/* ------------------------------------------------------------------------ */

static double fsign1(double d) { return copysign(1.0, d); }

static double mm2(double d1, double d2) { /* holib.f90:440-452 */
  double s1 = fsign1(d1), s2 = fsign1(d2);
  double a1 = fabs(d1), a2 = fabs(d2);
  return .5 * (s1 + s2) * (a1 < a2 ? a1 : a2);
}

static double fmin3(double a, double b, double c) {
  double r = a;
  if (b < r) r = b;
  if (c < r) r = c;
  return r;
}
static double fmax3(double a, double b, double c) {
  double r = a;
  if (b > r) r = b;
  if (c > r) r = c;
  return r;
}

static double mm4(double d1, double d2, double d3, double d4) { /* :472-486 */
  double s1 = fsign1(d1), s2 = fsign1(d2), s3 = fsign1(d3), s4 = fsign1(d4);
  double m = fabs(d1);
  if (fabs(d2) < m) m = fabs(d2);
  if (fabs(d3) < m) m = fabs(d3);
  if (fabs(d4) < m) m = fabs(d4);
  return .125 * (s1 + s2) * fabs((s1 + s3) * (s1 + s4)) * m;
}

static double ceno3(const double d[3]) { /* holib.f90:490-510 */
  const double alpha = 0.7;
  double r = 0.;
  int is0 = (int)fsign1(d[0]), is1 = (int)fsign1(d[1]), is2 = (int)fsign1(d[2]);
  int s = is0 + is1 + is2;
  if (abs(s) == 3) {
    double w0 = fabs(d[0]), w1 = alpha * fabs(d[1]), w2 = fabs(d[2]);
    int m = 0;
    double wm = w0;
    if (w1 < wm) {
      wm = w1;
      m = 1;
    }
    if (w2 < wm) {
      wm = w2;
      m = 2;
    }
    r = d[m];
  }
  return r;
}

static double mp5(double f, double f1, double f2, double f3, double f4,
                  double f5) { /* holib.f90:514-536 */
  double r = f;
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

/* f points at f(0); valid f(-3)..f(n+4).  gl/gr are faces 0..n. */
static void rec_pencil(int recal, const double* f, double* gl, double* gr,
                       int n) {
  int i;
  switch (recal) {
    case ECHO_REC_TVD2: /* holib.f90:47-77 */
      for (i = 1; i <= n; i++) {
        double dp = .5 * mm2(f[i] - f[i - 1], f[i + 1] - f[i]);
        gl[i] = f[i] + dp;
        gr[i - 1] = f[i] - dp;
      }
      gl[0] = f[0] + .5 * mm2(f[0] - f[-1], f[1] - f[0]);
      gr[n] = f[n + 1] - .5 * mm2(f[n + 1] - f[n], f[n + 2] - f[n + 1]);
      break;
    case ECHO_REC_CENO3: { /* holib.f90:81-126 */
      const double c11 = 3 / 8., c21 = -10 / 8., c31 = 15 / 8.;
      const double c12 = -1 / 8., c22 = 6 / 8., c32 = 3 / 8.;
      const double c13 = 3 / 8., c23 = 6 / 8., c33 = -1 / 8.;
      for (i = 0; i <= n; i++) {
        double d[3], f1, f2, f3, f4, f5, p;
        f1 = f[i - 2]; f2 = f[i - 1]; f3 = f[i]; f4 = f[i + 1]; f5 = f[i + 2];
        p = f3 + .5 * mm2(f3 - f2, f4 - f3);
        d[0] = c11 * f1 + c21 * f2 + c31 * f3 - p;
        d[1] = c12 * f2 + c22 * f3 + c32 * f4 - p;
        d[2] = c13 * f3 + c23 * f4 + c33 * f5 - p;
        gl[i] = p + ceno3(d);
        f1 = f[i + 3]; f2 = f[i + 2]; f3 = f[i + 1]; f4 = f[i]; f5 = f[i - 1];
        p = f3 + .5 * mm2(f3 - f2, f4 - f3);
        d[0] = c11 * f1 + c21 * f2 + c31 * f3 - p;
        d[1] = c12 * f2 + c22 * f3 + c32 * f4 - p;
        d[2] = c13 * f3 + c23 * f4 + c33 * f5 - p;
        gr[i] = p + ceno3(d);
      }
      break;
    }
    case ECHO_REC_WENO3: { /* holib.f90:130-173 */
      const double d1 = 1 / 3., d2 = 2 / 3., eps = 1.e-6;
      const double c11 = -1 / 2., c21 = 3 / 2., c12 = 1 / 2., c22 = 1 / 2.;
      for (i = 0; i <= n; i++) {
        double f1, f2, f3, b1, b2, a1, a2, p1, p2;
        f1 = f[i - 1]; f2 = f[i]; f3 = f[i + 1];
        b1 = (f2 - f1) * (f2 - f1);
        b2 = (f3 - f2) * (f3 - f2);
        a1 = d1 / ((b1 + eps) * (b1 + eps));
        a2 = d2 / ((b2 + eps) * (b2 + eps));
        p1 = c11 * f1 + c21 * f2;
        p2 = c12 * f2 + c22 * f3;
        gl[i] = (a1 * p1 + a2 * p2) / (a1 + a2);
        f1 = f[i + 2]; f2 = f[i + 1]; f3 = f[i];
        b1 = (f2 - f1) * (f2 - f1);
        b2 = (f3 - f2) * (f3 - f2);
        a1 = d1 / ((b1 + eps) * (b1 + eps));
        a2 = d2 / ((b2 + eps) * (b2 + eps));
        p1 = c11 * f1 + c21 * f2;
        p2 = c12 * f2 + c22 * f3;
        gr[i] = (a1 * p1 + a2 * p2) / (a1 + a2);
      }
      break;
    }
    case ECHO_REC_WENO5: { /* holib.f90:177-232 */
      const double d1 = 1 / 16., d2 = 10 / 16., d3 = 5 / 16., eps = 1.e-6;
      const double c11 = 3 / 8., c21 = -10 / 8., c31 = 15 / 8.;
      const double c12 = -1 / 8., c22 = 6 / 8., c32 = 3 / 8.;
      const double c13 = 3 / 8., c23 = 6 / 8., c33 = -1 / 8.;
      for (i = 0; i <= n; i++) {
        double f1, f2, f3, f4, f5, t1, t2, b1, b2, b3, a1, a2, a3, p1, p2, p3, q;
        f1 = f[i - 2]; f2 = f[i - 1]; f3 = f[i]; f4 = f[i + 1]; f5 = f[i + 2];
        t1 = f3 - 2 * f2 + f1; t2 = 3. * f3 - 4. * f2 + f1;
        b1 = 13. * (t1 * t1) + 3. * (t2 * t2);
        t1 = f4 - 2 * f3 + f2; t2 = f4 - f2;
        b2 = 13. * (t1 * t1) + 3. * (t2 * t2);
        t1 = f5 - 2 * f4 + f3; t2 = f5 - 4. * f4 + 3. * f3;
        b3 = 13. * (t1 * t1) + 3. * (t2 * t2);
        q = b1 / 12. + eps; a1 = d1 / (q * q);
        q = b2 / 12. + eps; a2 = d2 / (q * q);
        q = b3 / 12. + eps; a3 = d3 / (q * q);
        p1 = c11 * f1 + c21 * f2 + c31 * f3;
        p2 = c12 * f2 + c22 * f3 + c32 * f4;
        p3 = c13 * f3 + c23 * f4 + c33 * f5;
        gl[i] = (a1 * p1 + a2 * p2 + a3 * p3) / (a1 + a2 + a3);
        f1 = f[i + 3]; f2 = f[i + 2]; f3 = f[i + 1]; f4 = f[i]; f5 = f[i - 1];
        t1 = f3 - 2 * f2 + f1; t2 = 3. * f3 - 4. * f2 + f1;
        b1 = 13. * (t1 * t1) + 3. * (t2 * t2);
        t1 = f4 - 2 * f3 + f2; t2 = f4 - f2;
        b2 = 13. * (t1 * t1) + 3. * (t2 * t2);
        t1 = f5 - 2 * f4 + f3; t2 = f5 - 4. * f4 + 3. * f3;
        b3 = 13. * (t1 * t1) + 3. * (t2 * t2);
        q = b1 / 12. + eps; a1 = d1 / (q * q);
        q = b2 / 12. + eps; a2 = d2 / (q * q);
        q = b3 / 12. + eps; a3 = d3 / (q * q);
        p1 = c11 * f1 + c21 * f2 + c31 * f3;
        p2 = c12 * f2 + c22 * f3 + c32 * f4;
        p3 = c13 * f3 + c23 * f4 + c33 * f5;
        gr[i] = (a1 * p1 + a2 * p2 + a3 * p3) / (a1 + a2 + a3);
      }
      break;
    }
    case ECHO_REC_PPM4: /* holib.f90:236-268 */
      for (i = 0; i <= n; i++) {
        double f1, f2, f3, f4;
        f1 = f[i - 1]; f2 = f[i]; f3 = f[i + 1]; f4 = f[i + 2];
        gl[i] = f2 + .5 * (f3 - f2) - .125 * (mm2(f4 - f3, f3 - f2) - mm2(f3 - f2, f2 - f1));
        f1 = f[i + 2]; f2 = f[i + 1]; f3 = f[i]; f4 = f[i - 1];
        gr[i] = f2 + .5 * (f3 - f2) - .125 * (mm2(f4 - f3, f3 - f2) - mm2(f3 - f2, f2 - f1));
      }
      break;
    case ECHO_REC_MPE3: { /* holib.f90:272-294 */
      const double d1 = -1 / 8., d2 = 6 / 8., d3 = 3 / 8.;
      for (i = 0; i <= n; i++) {
        gl[i] = d1 * f[i - 1] + d2 * f[i] + d3 * f[i + 1];
        gr[i] = d1 * f[i + 2] + d2 * f[i + 1] + d3 * f[i];
      }
      for (i = 0; i <= n; i++) {
        gl[i] = mp5(gl[i], f[i - 2], f[i - 1], f[i], f[i + 1], f[i + 2]);
        gr[i] = mp5(gr[i], f[i + 3], f[i + 2], f[i + 1], f[i], f[i - 1]);
      }
      break;
    }
    case ECHO_REC_MPE5: { /* holib.f90:298-320 */
      const double d1 = 3 / 128., d2 = -20 / 128., d3 = 90 / 128.,
                   d4 = 60 / 128., d5 = -5 / 128.;
      for (i = 0; i <= n; i++) {
        gl[i] = d1 * f[i - 2] + d2 * f[i - 1] + d3 * f[i] + d4 * f[i + 1] + d5 * f[i + 2];
        gr[i] = d1 * f[i + 3] + d2 * f[i + 2] + d3 * f[i + 1] + d4 * f[i] + d5 * f[i - 1];
      }
      for (i = 0; i <= n; i++) {
        gl[i] = mp5(gl[i], f[i - 2], f[i - 1], f[i], f[i + 1], f[i + 2]);
        gr[i] = mp5(gr[i], f[i + 3], f[i + 2], f[i + 1], f[i], f[i - 1]);
      }
      break;
    }
    default:
      break;
  }
}

void orc_recon(int recal, int m, int n, const double* f, double* gl,
               double* gr) {
  for (int r = 0; r < m; r++)
    rec_pencil(recal, f + (size_t)r * (n + 8) + 4, gl + (size_t)r * (n + 1),
               gr + (size_t)r * (n + 1), n);
}

/* ------------------------------------------------------------------------ */
/* viscous helpers (viscous.f90)                                            */
/* ------------------------------------------------------------------------ */

typedef struct Pit {
  double tt, tx, ty, tz, zz;
} Pit;

/* get_derived_pi (viscous.f90:244-255) */
static void derived_pi(const Phys* ph, const double* p, Pit* o) {
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3;
  o->tx = p[KPIXX] * p[KVX] * g1 + p[KPIXY] * p[KVY] * g2 + p[KPIXZ] * p[KVZ] * g3;
  o->ty = p[KPIXY] * p[KVX] * g1 + p[KPIYY] * p[KVY] * g2 + p[KPIYZ] * p[KVZ] * g3;
  o->tz = p[KPIXZ] * p[KVX] * g1 + p[KPIYZ] * p[KVY] * g2 + p[KPIZZ] * p[KVZ] * g3;
  o->tt = o->tx * p[KVX] * g1 + o->ty * p[KVY] * g2 + o->tz * p[KVZ] * g3;
  o->zz = p[KPIZZ];
}

/* get_derived_pi_zz (viscous.f90:259-279) */
static void derived_pi_zz(const Phys* ph, const double* p, Pit* o) {
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3;
  double vx = p[KVX], vy = p[KVY], vz = p[KVZ];
  double pixy = p[KPIXY], pixx = p[KPIXX], piyy = p[KPIYY], piyz = p[KPIYZ],
         pixz = p[KPIXZ];
  o->tt = 1. / (1. - vz * vz * g3) *
          (vx * g1 * pixy * vy * g2 + vx * vx * g1 * g1 * pixx + vy * g1 * piyz * vz * g3 +
           2. * vx * g1 * pixz * vz * g3 + vy * g1 * g1 * pixy * vx + vy * vy * g1 * piyy * g2 +
           vz * g3 * piyz * vy * g2 - pixx * g1 * vz * vz * g3 - piyy * g2 * vz * vz * g3);
  o->tx = pixx * vx * g1 + pixy * vy * g2 + pixz * vz * g3;
  o->ty = pixy * vx * g1 + piyy * vy * g2 + piyz * vz * g3;
  o->tz = 1. / (1. - vz * vz * g3) *
          (pixz * vx * g1 + pixz * vx * g1 * vz * vz * g3 + piyz * vy * g2 +
           vz * vx * g1 * pixy * vy * g2 - vz * pixx * g1 - vz * piyy * g2 +
           vz * vx * vx * g1 * g1 * pixx + vy * g1 * piyz * vz * vz * g3 +
           vz * vy * g1 * g1 * pixy * vx + vz * vy * vy * g1 * piyy * g2);
  o->zz = 1. / (g3 * (1. - vz * vz * g3)) *
          (vx * g1 * pixy * vy * g2 - pixx * g1 - piyy * g2 + vx * vx * g1 * g1 * pixx +
           vy * g1 * piyz * vz * g3 + 2. * vx * g1 * pixz * vz * g3 + vy * g1 * g1 * pixy * vx +
           vy * vy * g1 * piyy * g2 + vz * g3 * piyz * vy * g2);
}

/* the `obtained` switch used at every call site */
static void derived_pi_any(const Phys* ph, double* p, Pit* o) {
  if (ph->p->obtained_zz) {
    derived_pi_zz(ph, p, o);
    p[KPIZZ] = o->zz;
  } else {
    derived_pi(ph, p, o);
  }
}

/* get_viscous_parameters (viscous.f90:172-199) */
static int viscous_parameters(const Phys* ph, double dens, double press,
                              double* eta, double* zeta, double* tau_pi,
                              double* tau_pi_big) {
  const EchoParams* p = ph->p;
  double en = 0, temp = 0, s = 0, cs2 = 0;
  /* errcode is overwritten by the eos_sound call (viscous.f90:180-181) */
  (void)get_derived_data(ph, dens, press, &en, &temp, &s);
  int err = eos_sound(ph, dens, en, press, &cs2);
  const double hbar = 0.197326;
  *eta = hbar * p->eta_over_s * s;
  if (p->init_type == 2) *eta = p->eta_over_s;
  if (p->bulkvis)
    *zeta = 2. * *eta * (1. / 3. - cs2);
  else
    *zeta = 0.;
  if (temp == 0 || s == 0)
    *tau_pi = 0.;
  else
    *tau_pi = p->tau_pi_coeff * *eta / (temp * s);
  if (p->init_type == 5) *tau_pi = 5. * *eta / (temp * s);
  *tau_pi_big = *tau_pi;
  return err;
}

/* get_sigma (viscous.f90:283-393); d = deriv of the cell, v = primitives */
static void get_sigma(const Phys* ph, const double* v, const double* d,
                      double sigma[6]) {
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3, t = ph->t;
  double ux = v[KVX], uy = v[KVY], uz = v[KVZ];
  double ut = 1. / sqrt(1. - g1 * ux * ux - g2 * uy * uy - g3 * uz * uz);
  ux = ux * ut;
  uy = uy * ut;
  uz = uz * ut;
  double dutdt = d[DTT], dutdx = d[DTX], dutdy = d[DTY], dutdz = d[DTZ];
  double duxdx = d[DXX], duydy = d[DYY], duzdz = d[DZZ], duzdt = d[DZT];
  double duzdx = d[DZX], duzdy = d[DZY], duxdt = d[DXT], duxdy = d[DXY];
  double duxdz = d[DXZ], duydt = d[DYT], duydx = d[DYX], duydz = d[DYZ];
  (void)dutdx; (void)dutdy; (void)dutdz;
  if (ph->p->coordinates == ECHO_MINKOWSKI) {
    sigma[SZZ] = ut * uz * duzdt + uz * ux * duzdx + uz * uy * duzdy + (2. / 3.) * duzdz +
                 (2. / 3.) * duzdz * (uz * uz) - dutdt / 3. - duxdx / 3. - duydy / 3. -
                 (uz * uz) * dutdt / 3. - (uz * uz) * duxdx / 3. - (uz * uz) * duydy / 3.;
    sigma[SXZ] = 0.5 * ut * ux * duzdt + 0.5 * duzdx + 0.5 * (ux * ux) * duzdx +
                 0.5 * ux * uy * duzdy + ux * uz * duzdz / 6. + 0.5 * ut * uz * duxdt +
                 ux * uz * duxdx / 6. + 0.5 * uy * uz * duxdy + 0.5 * duxdz +
                 0.5 * duxdz * (uz * uz) - ux * uz * dutdt / 3. - ux * uz * duydy / 3.;
    sigma[SXY] = 0.5 * ut * ux * duydt + 0.5 * duydx + 0.5 * (ux * ux) * duydx +
                 ux * uy * duydy / 6. + ux * uz * duydz / 2. + 0.5 * ut * uy * duxdt +
                 ux * uy * duxdx / 6. + 0.5 * duxdy + 0.5 * duxdy * (uy * uy) +
                 uy * uz * duxdz / 2. - ux * uy * dutdt / 3. - ux * uy * duzdz / 3.;
    sigma[SYZ] = 0.5 * ut * uy * duzdt + ux * uy * duzdx / 2. + duzdy / 2. +
                 duzdy * (uy * uy) / 2. + uy * uz * duzdz / 6. + ut * uz * duydt / 2. +
                 ux * uz * duydx / 2. + uy * uz * duydy / 6. + duydz / 2. +
                 duydz / 2. * (uz * uz) - uy * uz * dutdt / 3. - uy * uz * duxdx / 3.;
    sigma[SXX] = ut * ux * duxdt + (2. / 3.) * duxdx + (2. / 3.) * duxdx * (ux * ux) +
                 ux * uy * duxdy + ux * uz * duxdz - dutdt / 3. - duydy / 3. - duzdz / 3. -
                 (ux * ux) * dutdt / 3. - (ux * ux) * duydy / 3. - (ux * ux) * duzdz / 3.;
    sigma[SYY] = ut * uy * duydt + ux * uy * duydx + (2. / 3.) * duydy +
                 (2. / 3.) * duydy * (uy * uy) + uy * uz * duydz - dutdt / 3. - duxdx / 3. -
                 duzdz / 3. - (uy * uy) * dutdt / 3. - (uy * uy) * duxdx / 3. -
                 (uy * uy) * duzdz / 3.;
  } else {
    double t2 = t * t, t3 = pow(t, 3.);
    sigma[SZZ] = ut * uz * duzdt + uz * ux * duzdx + uz * uy * duzdy + (2. * duzdz) / (3. * t2) +
                 (2. / 3.) * duzdz * (uz * uz) - dutdt / (3. * t2) - duxdx / (3. * t2) -
                 duydy / (3. * t2) - (uz * uz) * dutdt / 3. - (uz * uz) * duxdx / 3. -
                 (uz * uz) * duydy / 3. + 2. / 3. * ut / t3 + 5. / 3. * (ut / t) * (uz * uz);
    sigma[SXZ] = 0.5 * ut * ux * duzdt + 0.5 * duzdx + 0.5 * (ux * ux) * duzdx +
                 0.5 * ux * uy * duzdy + ux * uz * duzdz / 6. + 0.5 * ut * uz * duxdt +
                 ux * uz * duxdx / 6. + 0.5 * uy * uz * duxdy + duxdz / (2. * t2) +
                 0.5 * duxdz * (uz * uz) - ux * uz * dutdt / 3. - ux * uz * duydy / 3. +
                 (2. / 3.) * ut * uz * ux / t;
    sigma[SXY] = 0.5 * ut * ux * duydt + 0.5 * duydx + 0.5 * (ux * ux) * duydx +
                 ux * uy * duydy / 6. + ux * uz * duydz / 2. + 0.5 * ut * uy * duxdt +
                 ux * uy * duxdx / 6. + 0.5 * duxdy + 0.5 * duxdy * (uy * uy) +
                 uy * uz * duxdz / 2. - ux * uy * dutdt / 3. - ux * uy * duzdz / 3. -
                 ut * ux * uy / (3. * t);
    sigma[SYZ] = 0.5 * ut * uy * duzdt + ux * uy * duzdx / 2. + duzdy / 2. +
                 duzdy * (uy * uy) / 2. + uy * uz * duzdz / 6. + ut * uz * duydt / 2. +
                 ux * uz * duydx / 2. + uy * uz * duydy / 6. + duydz / (2. * t2) +
                 duydz / 2. * (uz * uz) - uy * uz * dutdt / 3. - uy * uz * duxdx / 3. +
                 (2. / 3.) * ut * uz * uy / t;
    sigma[SXX] = ut * ux * duxdt + (2. / 3.) * duxdx + (2. / 3.) * duxdx * (ux * ux) +
                 ux * uy * duxdy + ux * uz * duxdz - dutdt / 3. - duydy / 3. - duzdz / 3. -
                 ut / (3. * t) - (ux * ux) * dutdt / 3. - (ux * ux) * duydy / 3. -
                 (ux * ux) * duzdz / 3. - (ux * ux) * ut / (3. * t);
    sigma[SYY] = ut * uy * duydt + ux * uy * duydx + (2. / 3.) * duydy +
                 (2. / 3.) * duydy * (uy * uy) + uy * uz * duydz - dutdt / 3. - duxdx / 3. -
                 duzdz / 3. - ut / (3. * t) - (uy * uy) * dutdt / 3. - (uy * uy) * duxdx / 3. -
                 (uy * uy) * duzdz / 3. - (uy * uy) * ut / (3. * t);
  }
}

/* ------------------------------------------------------------------------ */
/* E x B helpers (system.f90:1846-1897)                                     */
/* ------------------------------------------------------------------------ */
static void e_ideal(const Phys* ph, const double* vv, const double* b,
                    double* E) {
  double gp = ph->gp;
  E[0] = -gp * (vv[1] * b[2] - vv[2] * b[1]);
  E[1] = -gp * (vv[2] * b[0] - vv[0] * b[2]);
  E[2] = -gp * (vv[0] * b[1] - vv[1] * b[0]);
}
static void exb(const Phys* ph, const double* E, const double* b, double* o) {
  double e0 = E[0], e1 = E[1], e2 = E[2] / ph->g3, gp = ph->gp;
  o[0] = gp * (e1 * b[2] - e2 * b[1]);
  o[1] = gp * (e2 * b[0] - e0 * b[2]);
  o[2] = gp * (e0 * b[1] - e1 * b[0]);
}

/* covariant E_i of a cell: the resistive primitive E^i lowered
   (system.f90:203-205), or the ideal -v x B */
static void e_field(const Phys* ph, const double* v, double* E) {
  if (ph->p->mhd == 2) {
    E[0] = v[ph->kex];
    E[1] = v[ph->key];
    E[2] = v[ph->kez] * ph->g3;
  } else {
    e_ideal(ph, v + KVX, v + ph->kbx, E);
  }
}

/* contravariant (a x b)^i = sqrt(gamma)/g_ii [ijk] a^j b^k of contravariant
   a, b (system_crossprod, system.f90:1867-1880, in Minkowski coordinates) */
static void cross_contra(const Phys* ph, const double* a, const double* b, double* o) {
  double gp = ph->gp;
  o[0] = gp * (a[1] * b[2] - a[2] * b[1]);
  o[1] = gp * (a[2] * b[0] - a[0] * b[2]);
  o[2] = gp / ph->g3 * (a[0] * b[1] - a[1] * b[0]);
}

/* stiff part of the E source, Ohm's law with chiral term (system.f90:
   1656-1660), contravariant, before the sqrt(-g) factor:
   S = -gamma [sigma (E - (E.v) v + v x B) + sigma_chi (B - (B.v) v - v x E)].
   (The reference's Minkowski branch assigns E.v twice and leaves B.v unset,
   system.f90:1750-1751; B.v is used here.) */
static void ohm_stiff(const Phys* ph, const double* vel, const double* B, const double* E, double glf,
                      double* S) {
  double g3 = ph->g3, sig = ph->p->sigma_el, chi = ph->p->sigma_chiral;
  double vxb[3], vxe[3];
  cross_contra(ph, vel, B, vxb);
  cross_contra(ph, vel, E, vxe);
  double vdotb = vel[0] * B[0] + vel[1] * B[1] + vel[2] * B[2] * g3;
  double vdote = vel[0] * E[0] + vel[1] * E[1] + vel[2] * E[2] * g3;
  for (int i = 0; i < 3; i++)
    S[i] = -glf * (sig * (E[i] - vdote * vel[i] + vxb[i]) + chi * (B[i] - vdotb * vel[i] - vxe[i]));
}

/* E = Es + h S(E) for fixed v and B: linear in E,
   [(1 + lam) I - lam v v_cov - mu (v x .)] E = Es - lam v x B - mu (B - (B.v) v)
   with lam = h gamma sigma, mu = h gamma sigma_chi; solved by cofactors. */
static void ohm_solve(const Phys* ph, const double* Es, const double* vel, const double* B, double h,
                      double* E) {
  double g3 = ph->g3, gp = ph->gp, gq = ph->gp / ph->g3;
  double v2 = vel[0] * vel[0] + vel[1] * vel[1] + g3 * (vel[2] * vel[2]);
  double glf = 1. / sqrt(1. - v2);
  double lam = h * glf * ph->p->sigma_el, mu = h * glf * ph->p->sigma_chiral;
  double vxb[3];
  cross_contra(ph, vel, B, vxb);
  double vdotb = vel[0] * B[0] + vel[1] * B[1] + vel[2] * B[2] * g3;
  double vc[3] = {vel[0], vel[1], g3 * vel[2]};
  double C[3][3] = {{0., -gp * vel[2], gp * vel[1]}, {gp * vel[2], 0., -gp * vel[0]}, {-gq * vel[1], gq * vel[0], 0.}};
  double r[3], M[3][3];
  for (int i = 0; i < 3; i++) {
    r[i] = Es[i] - lam * vxb[i] - mu * (B[i] - vdotb * vel[i]);
    for (int j = 0; j < 3; j++) M[i][j] = (i == j ? 1. + lam : 0.) - lam * vel[i] * vc[j] - mu * C[i][j];
  }
  double c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
  double c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
  double c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
  double c10 = M[0][2] * M[2][1] - M[0][1] * M[2][2];
  double c11 = M[0][0] * M[2][2] - M[0][2] * M[2][0];
  double c12 = M[0][1] * M[2][0] - M[0][0] * M[2][1];
  double c20 = M[0][1] * M[1][2] - M[0][2] * M[1][1];
  double c21 = M[0][2] * M[1][0] - M[0][0] * M[1][2];
  double c22 = M[0][0] * M[1][1] - M[0][1] * M[1][0];
  double det = M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02;
  E[0] = (c00 * r[0] + c10 * r[1] + c20 * r[2]) / det;
  E[1] = (c01 * r[0] + c11 * r[1] + c21 * r[2]) / det;
  E[2] = (c02 * r[0] + c12 * r[1] + c22 * r[2]) / det;
}

/* ------------------------------------------------------------------------ */
/* prim2cons (system.f90:164-263)                                           */
/* ------------------------------------------------------------------------ */
static int prim2cons(const Phys* ph, double* v, double* u) {
  const EchoParams* p = ph->p;
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3, gp = ph->gp;
  double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR];
  double en = 0;
  int err = eos_energy(ph, rh, &en, pr);
  if (err) return err;
  double v2 = g1 * vx * vx + g2 * vy * vy + g3 * vz * vz;
  double glf = 1. / sqrt(1. - v2);
  double w = en + pr;
  double ww = w * (glf * glf);
  u[KRH] = rh * glf;
  double E[3], EXB[3], EEM = 0;
  if (p->mhd) {
    e_field(ph, v, E);
    double E2 = E[0] * E[0] + E[1] * E[1] + (E[2] * E[2]) / g3;
    exb(ph, E, v + ph->kbx, EXB);
    double bx = v[ph->kbx], by = v[ph->kby], bz = v[ph->kbz];
    double B2 = bx * bx + by * by + (bz * bz) * g3;
    EEM = 0.5 * (E2 + B2);
  }
  if (p->viscosity) {
    w = w + v[KPIBU];
    ww = w * (glf * glf);
    Pit pi;
    derived_pi_any(ph, v, &pi);
    u[KVX] = (ww * vx + pi.tx);
    u[KVY] = (ww * vy + pi.ty);
    u[KVZ] = (ww * vz + pi.tz) * g3;
    u[KPR] = ww - pr - v[KPIBU] - pi.tt * ph->g0;
    u[KPIBU] = v[KPIBU] * u[KRH];
    u[KPIZZ] = v[KPIZZ] * u[KRH];
    u[KPIXZ] = v[KPIXZ] * u[KRH];
    u[KPIXY] = v[KPIXY] * u[KRH];
    u[KPIYZ] = v[KPIYZ] * u[KRH];
    u[KPIXX] = v[KPIXX] * u[KRH];
    u[KPIYY] = v[KPIYY] * u[KRH];
  } else if (p->mhd) {
    u[KVX] = ww * vx + EXB[0];
    u[KVY] = ww * vy + EXB[1];
    u[KVZ] = ww * vz * g3 + EXB[2];
    u[KPR] = ww - pr + EEM;
    u[ph->kbx] = v[ph->kbx];
    u[ph->kby] = v[ph->kby];
    u[ph->kbz] = v[ph->kbz];
    if (p->mhd == 2) {
      u[ph->kex] = v[ph->kex];
      u[ph->key] = v[ph->key];
      u[ph->kez] = v[ph->kez];
    }
    if (p->divclean) u[ph->kglm] = v[ph->kglm] / gp;
  } else {
    u[KVX] = ww * vx;
    u[KVY] = ww * vy;
    u[KVZ] = ww * vz * g3;
    u[KPR] = ww - pr;
  }
  for (int k = 0; k < ph->nu; k++) u[k] = u[k] * gp;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* BRENTM (libacm554.f90:8-362) applied to sist3 (system.f90:1199-1231)     */
/* ------------------------------------------------------------------------ */
typedef struct Sist3 {
  const Phys* ph;
  double B2, SB2, S2, U, D;
} Sist3;

static void sist3(const Sist3* s, const double* X, double* F, int K) {
  double xx = X[0], yy = X[1], pp = X[2];
  double B2 = s->B2, SB2 = s->SB2, S2 = s->S2, U = s->U, D = s->D;
  if (K == 1) F[0] = (yy + B2) * (yy + B2) * xx - SB2 / (yy * yy) * (2 * yy + B2) - S2;
  if (K == 2) F[1] = yy - pp + 0.5 * (1. + xx) * B2 - 0.5 * SB2 / (yy * yy) - U;
  if (K == 3) {
    double rh = D * sqrt(1 - xx), en = 0;
    (void)eos_energy(s->ph, rh, &en, pp); /* errcode ignored, system.f90:1227 */
    F[2] = yy - (pp + en) / (1 - xx);
  }
}

static double dmax1(double a, double b) { return b > a ? b : a; }
static double dsign(double a, double b) { return copysign(fabs(a), b); }

/* returns INFO; *nfev_out = NFEV */
/* the system a BRENTM call solves: F(K) of X, as sist3 / sist4 */
typedef void (*SysFn)(void* ctx, const double* X, double* F, int K);

static int brentm(int N, SysFn fn, void* ctx, double* X, double* FVEC, double FTOL,
                  double XTOL, int MAXFEV, int MOPT, int* nfev_out) {
  const int LDQ = N;
  double Q[9], SIGMA[3], WA1[3], WA2[3];
#define QQ(i, j) Q[((j)-1) * LDQ + ((i)-1)]
  int I, J, K, M, NFCALL, NIER6, NIER7, NIER8, NSING, INFO, NFEV, IFLAG;
  int CONV;
  double DELTA, DIFIT, DIFIT1, EPS, EPSMCH, ETA, FKY, FKZ, FNORM, FNORM1, H,
      SKNORM, TEMP, XNORM;
  const double ZERO = 0.0, P05 = 5.0e-2, SCALE = 1.0e1;
  EPSMCH = 2.220446049250313080847e-16; /* EPSILON(1.d0) */
  INFO = 0;
  IFLAG = 0;
  NFEV = 0;
  NFCALL = 0;
  NIER6 = -1;
  NIER7 = -1;
  NIER8 = 0;
  FNORM = ZERO;
  DIFIT = ZERO;
  XNORM = ZERO;
  for (I = 1; I <= N; I++) XNORM = dmax1(XNORM, fabs(X[I - 1]));
  EPS = sqrt(EPSMCH);
  DELTA = SCALE * XNORM;
  if (XNORM == ZERO) DELTA = SCALE;
  for (;;) { /* label 20 */
    NSING = N;
    FNORM1 = FNORM;
    DIFIT1 = DIFIT;
    FNORM = ZERO;
    H = EPS * XNORM;
    if (H == ZERO) H = EPS;
    for (J = 1; J <= N; J++) {
      for (I = 1; I <= N; I++) QQ(I, J) = ZERO;
      QQ(J, J) = H;
      WA1[J - 1] = X[J - 1];
    }
    for (K = 1; K <= N; K++) {
      IFLAG = K;
      fn(ctx, WA1, FVEC, IFLAG);
      FKY = FVEC[K - 1];
      NFCALL = NFCALL + 1;
      NFEV = NFCALL / N;
      FNORM = dmax1(FNORM, fabs(FKY));
      for (J = K; J <= N; J++) {
        for (I = 1; I <= N; I++) WA2[I - 1] = WA1[I - 1] + QQ(I, J);
        fn(ctx, WA2, FVEC, IFLAG);
        FKZ = FVEC[K - 1];
        NFCALL = NFCALL + 1;
        NFEV = NFCALL / N;
        SIGMA[J - 1] = FKZ - FKY;
      }
      FVEC[K - 1] = FKY;
      ETA = ZERO;
      for (I = K; I <= N; I++) ETA = dmax1(ETA, fabs(SIGMA[I - 1]));
      if (ETA == ZERO) continue; /* GO TO 150 */
      NSING = NSING - 1;
      SKNORM = ZERO;
      for (I = K; I <= N; I++) {
        SIGMA[I - 1] = SIGMA[I - 1] / ETA;
        SKNORM = SKNORM + SIGMA[I - 1] * SIGMA[I - 1];
      }
      SKNORM = sqrt(SKNORM);
      if (SIGMA[K - 1] < ZERO) SKNORM = -SKNORM;
      SIGMA[K - 1] = SIGMA[K - 1] + SKNORM;
      for (I = 1; I <= N; I++) WA2[I - 1] = ZERO;
      for (J = K; J <= N; J++) {
        TEMP = SIGMA[J - 1];
        for (I = 1; I <= N; I++) WA2[I - 1] = WA2[I - 1] + TEMP * QQ(I, J);
      }
      for (J = K; J <= N; J++) {
        TEMP = SIGMA[J - 1] / (SKNORM * SIGMA[K - 1]);
        for (I = 1; I <= N; I++) QQ(I, J) = QQ(I, J) - TEMP * WA2[I - 1];
      }
      SIGMA[K - 1] = SKNORM * ETA;
      TEMP = FKY / SIGMA[K - 1];
      if (H * fabs(TEMP) > DELTA) TEMP = dsign(DELTA / H, TEMP);
      for (I = 1; I <= N; I++) WA1[I - 1] = WA1[I - 1] + TEMP * QQ(I, K);
    }
    XNORM = ZERO;
    DIFIT = ZERO;
    for (I = 1; I <= N; I++) {
      XNORM = dmax1(XNORM, fabs(WA1[I - 1]));
      DIFIT = dmax1(DIFIT, fabs(X[I - 1] - WA1[I - 1]));
      X[I - 1] = WA1[I - 1];
    }
    DELTA = dmax1(DELTA, SCALE * XNORM);
    CONV = (FNORM < FNORM1 && DIFIT < DIFIT1 && NSING == 0);
    NIER6 = NIER6 + 1;
    NIER7 = NIER7 + 1;
    NIER8 = NIER8 + 1;
    if (CONV) NIER6 = 0;
    if (FNORM < FNORM1 || DIFIT < DIFIT1) NIER7 = 0;
    if (DIFIT > EPS * XNORM) NIER8 = 0;
    if (FNORM <= FTOL) INFO = 1;
    if (DIFIT <= XTOL * XNORM && CONV) INFO = 2;
    if (FNORM <= FTOL && INFO == 2) INFO = 3;
    if (INFO != 0) break;
    if (NFEV >= MAXFEV) INFO = 4;
    if (NSING == N) INFO = 5;
    if (NIER6 == 5) INFO = 6;
    if (NIER7 == 3) INFO = 7;
    if (NIER8 == 4) INFO = 8;
    if (INFO != 0) break;
    if (!CONV || DIFIT > P05 * XNORM || MOPT == 1) continue; /* GO TO 220 */
    int done = 0;
    for (M = 2; M <= MOPT; M++) {
      int stop_refine = 0;
      FNORM1 = FNORM;
      FNORM = ZERO;
      for (K = 1; K <= N; K++) {
        IFLAG = K;
        fn(ctx, WA1, FVEC, IFLAG);
        FKY = FVEC[K - 1];
        NFCALL = NFCALL + 1;
        NFEV = NFCALL / N;
        FNORM = dmax1(FNORM, fabs(FKY));
        if (!(FNORM < FNORM1)) {
          FNORM = FNORM1;
          stop_refine = 1; /* GO TO 220 */
          break;
        }
        TEMP = FKY / SIGMA[K - 1];
        for (I = 1; I <= N; I++) WA1[I - 1] = WA1[I - 1] + TEMP * QQ(I, K);
      }
      if (stop_refine) break;
      XNORM = ZERO;
      DIFIT = ZERO;
      for (I = 1; I <= N; I++) {
        XNORM = dmax1(XNORM, fabs(WA1[I - 1]));
        DIFIT = dmax1(DIFIT, fabs(X[I - 1] - WA1[I - 1]));
        X[I - 1] = WA1[I - 1];
      }
      if (FNORM <= FTOL) INFO = 1;
      if (DIFIT <= XTOL * XNORM) INFO = 2;
      if (FNORM <= FTOL && INFO == 2) INFO = 3;
      if (NFEV >= MAXFEV && INFO == 0) INFO = 4;
      if (INFO != 0) {
        done = 1;
        break;
      }
    }
    if (done) break;
  }
#undef QQ
  *nfev_out = NFEV;
  return INFO;
}

static void sist3_fn(void* ctx, const double* X, double* F, int K) { sist3((const Sist3*)ctx, X, F, K); }

static int brentm3(const Sist3* s, double* X, double* FVEC, double FTOL, double XTOL, int MAXFEV, int MOPT,
                   int* nfev_out) {
  return brentm(3, sist3_fn, (void*)s, X, FVEC, FTOL, XTOL, MAXFEV, MOPT, nfev_out);
}

/* ------------------------------------------------------------------------ */
/* cons2prim (system.f90:423-1166)                                          */
/* u, v have nv entries; v holds the guess.  Returns errcode, *iters the    */
/* number of solver iterations (Newton steps, or BRENTM function evals).    */
/* ------------------------------------------------------------------------ */
/* Resistive con2prim with the implicit Ohm's law of an IMEX stage: the
   algo_solver 7 the reference names (common.f90:292-293, 2109-2113) but
   does not contain.  Unknowns v, p, E.  Given the stage's explicit part E*
   and h = a_ii dt (ph->ohm_h; 0 outside an implicit solve), E solves
   E = E* + h S(E; v, B), linear in E for fixed v (ohm_solve).  Fixed-point
   iteration on v: E(v); the fluid's share S - E x B, U - (E^2 + B^2)/2; the
   ideal-HD Newton on p (system.f90:511-561) for p and the new v; until
   max |dv| <= 1e-14 (one pass when h = 0).  Code 779 when 200 passes do
   not converge.  With h > 0, u[kex..kez] receives sqrt(-g) E. */
static int cons2prim_res(const Phys* ph, double* u, double* v, int* iters) {
  const double tol = 1.e-12, vtol = 1.e-14;
  const int iter_max = 100, outer_max = 200;
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3, gm = ph->gm, gp = ph->gp, h = ph->ohm_h;
  int kbx = ph->kbx, kex = ph->kex;
  double d = gm * u[KRH], U = gm * u[KPR];
  double S[3] = {gm * u[KVX], gm * u[KVY], gm * u[KVZ]};
  double B[3] = {gm * u[kbx], gm * u[kbx + 1], gm * u[kbx + 2]};
  double Es[3] = {gm * u[kex], gm * u[kex + 1], gm * u[kex + 2]};
  double vel[3] = {v[KVX], v[KVY], v[KVZ]}, E[3];
  double pr = v[KPR], rh = v[KRH];
  double B2 = B[0] * B[0] + B[1] * B[1] + (B[2] * B[2]) * g3;
  int errcode = 0, outer, total = 0;
  for (outer = 1; outer <= outer_max; outer++) {
    if (h > 0.) {
      ohm_solve(ph, Es, vel, B, h, E);
    } else {
      E[0] = Es[0];
      E[1] = Es[1];
      E[2] = Es[2];
    }
    double Ec[3] = {E[0], E[1], E[2] * g3}, EXB[3];
    exb(ph, Ec, B, EXB);
    double E2 = Ec[0] * Ec[0] + Ec[1] * Ec[1] + (Ec[2] * Ec[2]) / g3;
    double sx = S[0] - EXB[0], sy = S[1] - EXB[1], sz = (S[2] - EXB[2]) / g3;
    double et = U - 0.5 * (E2 + B2);
    double s2 = g1 * sx * sx + g2 * sy * sy + g3 * sz * sz;
    double w = 0, v2, glf, en, drhdpr, dendpr, pr_eos = 0, dprdrh = 0, dprden = 0, f, df, dpr;
    int iter;
    for (iter = 1; iter <= iter_max; iter++) {
      w = et + pr;
      v2 = s2 / (w * w);
      if (v2 >= 1.) {
        *iters = total + iter;
        return 777;
      }
      glf = 1. / sqrt(1. - v2);
      rh = d / glf;
      en = w * (1. - v2) - pr;
      drhdpr = rh * v2 * glf / (en + pr);
      dendpr = v2;
      errcode = eos_pressure(ph, rh, en, &pr_eos, &dprdrh, &dprden);
      f = pr_eos - pr;
      df = dprdrh * drhdpr + dprden * dendpr - 1.;
      dpr = -f / df;
      if (fabs(dpr) < tol * pr) break;
      pr = pr + dpr;
    }
    total += iter;
    double vn0 = sx / w, vn1 = sy / w, vn2 = sz / w;
    double dv = fmax3(fabs(vn0 - vel[0]), fabs(vn1 - vel[1]), fabs(vn2 - vel[2]) * gp);
    vel[0] = vn0;
    vel[1] = vn1;
    vel[2] = vn2;
    if (!(h > 0.) || dv <= vtol) break;
  }
  *iters = total;
  if (outer > outer_max) return 779;
  v[KRH] = rh;
  v[KVX] = vel[0];
  v[KVY] = vel[1];
  v[KVZ] = vel[2];
  v[KPR] = pr;
  for (int i = 0; i < 3; i++) {
    v[kbx + i] = B[i];
    v[kex + i] = E[i];
    if (h > 0.) u[kex + i] = E[i] * gp;
  }
  if (ph->p->divclean) v[ph->kglm] = u[ph->kglm];
  if (pr <= 0) errcode = 777;
  return errcode;
}


/* ------------------------------------------------------------------------ */
/* the other MHD inversions, algo_solver 2..6 (system.f90:732-1158)          */
/* ------------------------------------------------------------------------ */
/* sist4 (system.f90:1235-1266): the 2x2 system in (y, p) with x = v^2 from
   y; every call leaves its x in xinner, which algo 2 reads after BRENTM */
typedef struct Sist4 {
  const Phys* ph;
  double B2, SB2, S2, U, D, xinner;
} Sist4;

static void sist4_fn(void* ctx, const double* X, double* F, int K) {
  Sist4* s = (Sist4*)ctx;
  double yy = X[0], pp = X[1];
  double xx = (s->S2 + s->SB2 * (2. * yy + s->B2) / (yy * yy)) / ((yy + s->B2) * (yy + s->B2));
  s->xinner = xx;
  if (K == 2) {
    double rh = s->D * sqrt(1 - xx), en = 0;
    (void)eos_energy(s->ph, rh, &en, pp);
    F[1] = yy - (pp + en) / (1 - xx);
  }
  if (K == 1) F[0] = yy - pp + 0.5 * (1. + xx) * s->B2 - 0.5 * s->SB2 / (yy * yy) - s->U;
}

/* eos_energy_with_ders (eos.f90:236-246, 527-584, 1189-1215): e and its
   derivatives.  The tabulated routine sets de/dp = 0 and leaves de/drho
   unset, as does the analytic one below p(ENEZERO): both are 0 here. */
static int eos_energy_ders(const Phys* ph, double rh, double* en, double pr, double* dendrh, double* dendpr) {
  const EchoParams* p = ph->p;
  *dendrh = 0.;
  *dendpr = 0.;
  if (p->eqstate == ECHO_EOS_TABLE) return eos_energy(ph, rh, en, pr);
  if (pr <= p->przero) {
    *en = p->enezero * pr / p->przero;
    return 0;
  }
  if (p->eqstate == ECHO_EOS_CONFORMAL) {
    *en = 3. * pr;
    *dendpr = 3.;
  } else {
    *en = rh + pr / (4.0 / 3.0 - 1.);
    *dendrh = 1.;
    *dendpr = 1. / (4.0 / 3.0 - 1.);
  }
  return 0;
}

/* getfun (system.f90:2060-2097): F(X) of sist3 and, for sw = 1, the
   reference's Jacobian.  The reference never assigns Fnorm (an intent(out)
   it reads back); it is the Euclidean norm of F here. */
static void getfun(const Sist3* s, const double* X, double* F, double J[3][3], double* Fnorm, int sw) {
  double xx = X[0], yy = X[1], pp = X[2];
  double B2 = s->B2, SB2 = s->SB2, S2 = s->S2, U = s->U, D = s->D;
  F[0] = (yy + B2) * (yy + B2) * xx - SB2 / (yy * yy) * (2 * yy + B2) - S2;
  F[1] = yy - pp + 0.5 * (1. + xx) * B2 - 0.5 * SB2 / (yy * yy) - U;
  double rh = D * sqrt(1 - xx), en = 0, dendrh = 0, dendpr = 0;
  (void)eos_energy_ders(s->ph, rh, &en, pp, &dendrh, &dendpr);
  F[2] = yy - (pp + en) / (1 - xx);
  *Fnorm = sqrt(F[0] * F[0] + F[1] * F[1] + F[2] * F[2]);
  if (sw == 0) return;
  J[0][0] = (yy + B2) * (yy + B2);
  J[0][1] = 2 * (yy + B2) * xx + (2 * SB2 * (2 * yy + B2)) / (yy * yy * yy) - 2 * SB2 / (yy * yy);
  J[0][2] = dendrh * (-D / (2. * sqrt(1. - xx)));
  J[1][0] = B2 / 2.;
  J[1][1] = 1. + SB2 / (yy * yy * yy);
  J[1][2] = -1.;
  J[2][0] = -(pp + en) / ((1 - xx) * (1 - xx));
  J[2][1] = 1.;
  J[2][2] = -(1 + dendpr) / (1 - xx);
}

/* ludecompose (system.f90:1924-1986), its pivot test included: the pivot
   starts as A(i,i) itself, not its modulus.  A becomes U. */
static void ludecompose(double A[3][3], double L[3][3], int P[3], double smallvalue) {
  const int n = 3;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) L[i][j] = 0.;
  for (int i = 0; i < n; i++) P[i] = i;
  for (int i = 0; i < n; i++) L[i][i] = 1.;
  for (int i = 0; i < n - 1; i++) {
    double piv = A[i][i];
    int indP = -1;
    for (int j = i; j < n; j++)
      if (fabs(A[j][i]) > piv) {
        piv = A[j][i];
        indP = j;
      }
    if (indP >= 0) {
      int t = P[i];
      P[i] = P[indP];
      P[indP] = t;
      for (int k = i; k < n; k++) {
        double x = A[i][k];
        A[i][k] = A[indP][k];
        A[indP][k] = x;
      }
      for (int k = 0; k < i; k++) {
        double x = L[i][k];
        L[i][k] = L[indP][k];
        L[indP][k] = x;
      }
    }
    for (int j = i + 1; j < n; j++) {
      double m = A[j][i] / piv;
      L[j][i] = m;
      for (int k = i; k < n; k++) {
        A[j][k] = A[j][k] - m * A[i][k];
        if (fabs(A[j][k]) <= smallvalue) A[j][k] = 0.;
      }
    }
  }
}

/* solve (system.f90:2026-2058): L Z = P B, U X = Z */
static void lusolve(double L[3][3], double U[3][3], const int P[3], double* X, const double* B) {
  const int n = 3;
  double Z[3];
  Z[0] = B[P[0]];
  for (int i = 1; i < n; i++) {
    double rowsum = B[P[i]];
    for (int k = 0; k < i; k++) rowsum = rowsum - L[i][k] * Z[k];
    Z[i] = rowsum;
  }
  X[n - 1] = Z[n - 1] / U[n - 1][n - 1];
  for (int j = 1; j <= n - 1; j++) {
    int i = n - 1 - j;
    double rowsum = Z[i];
    for (int k = i + 1; k < n; k++) rowsum = rowsum - U[i][k] * X[k];
    X[i] = rowsum / U[i][i];
  }
}

/* solver7 / solver8 (system.f90:2102-2201): for x = v^2 the cubic in W
   (Newton from the larger root bound), then the residual in v^2 and its
   derivative; *w the W of this x (the reference's w_algo_solver7/8 global) */
typedef struct RtCtx {
  double B2, SB2, S2, UU, D, gam, w;
  int which; /* 7: ideal gas, 8: p = e/3 */
} RtCtx;

static void rt_func(RtCtx* c, double x, double* f, double* df) {
  const double third = 1.0 / 3.0;
  double B2 = c->B2, SB2 = c->SB2, S2 = c->S2, UU = c->UU, D = c->D;
  double v2 = x, rho = 0, c0, c2, c3, dw, dlogw, dc2, dc3, wb, vb2, w, gam = c->gam;
  c3 = 1.0 - gam * (1.0 - v2);
  if (c->which == 7) {
    rho = D * sqrt(1.0 - v2);
    c2 = gam * rho + .5 * B2 * (1.0 + v2) - UU;
  } else {
    c2 = .5 * B2 * (1.0 + v2) - UU;
  }
  c0 = -0.5 * SB2;
  if (c->which == 8 && c0 == 0.0) {
    w = -c2 / c3;
  } else {
    w = fmax(-c2 / c3, pow(-c0 / c3, third));
    int maxit = c->which == 7 ? 50 : 100;
    double wtol = c->which == 7 ? 1.e-10 : 1.e-12;
    for (int iter = 1; iter <= maxit; iter++) {
      dw = -((c3 * w + c2) * (w * w) + c0) / ((3 * c3 * w + 2 * c2) * w);
      if (fabs(dw / w) < wtol) break;
      w = w + dw;
    }
  }
  dc3 = gam;
  if (c->which == 7)
    dc2 = .5 * (B2 - gam * rho / (1. - v2));
  else
    dc2 = .5 * B2;
  dlogw = -(dc3 * w + dc2) / (3 * c3 * w + 2 * c2);
  wb = w + B2;
  vb2 = SB2 / (w * w);
  *f = wb * wb * v2 - (2 * w + B2) * vb2 - S2;
  *df = wb * (wb + 2 * dlogw * (w * v2 + vb2));
  c->w = w;
}

/* rtsafe (system.f90:2227-2286): safeguarded Newton on [x1, x2] from x0 */
static double rtsafe(RtCtx* c, double x0, double x1, double x2, double xacc, int* ierr) {
  const int maxit = 100;
  double f, df, xl = x1, xh = x2, dx, dxold, temp, r = x0;
  *ierr = 0;
  dxold = fabs(x2 - x1);
  dx = dxold;
  rt_func(c, r, &f, &df);
  for (int j = 1; j <= maxit; j++) {
    if (((r - xh) * df - f) * ((r - xl) * df - f) > 0. || fabs(2. * f) > fabs(dxold * df)) {
      dxold = dx;
      dx = 0.5 * (xh - xl);
      r = xl + dx;
      if (xl == r) {
        rt_func(c, r, &f, &df);
        return r;
      }
    } else {
      dxold = dx;
      dx = f / df;
      temp = r;
      r = r - dx;
      if (temp == r) {
        rt_func(c, r, &f, &df);
        return r;
      }
    }
    if (fabs(dx) < xacc) return r;
    rt_func(c, r, &f, &df);
    if (f < 0.)
      xl = r;
    else
      xh = r;
  }
  *ierr = 1;
  return r;
}

/* solver10_approximate (system.f90:2205-2223): Newton-like iteration on the
   depressed quartic; 12 (the reference's exit code) only when the exit test
   is met on the last allowed iteration, as the reference's test reads */
static int solver10_approximate(double b, double c, double d, double oldsol, double* x) {
  const int maxiterations = 100;
  int iter;
  *x = oldsol;
  for (iter = 1; iter <= maxiterations; iter++) {
    double xx = *x;
    double dx = -(12 * (xx * xx * xx) + 3 * b * (xx * xx) + 2 * c * xx + d);
    if (fabs(dx / xx) < 1.e-12) break;
    *x = xx + dx;
  }
  return iter == maxiterations ? 12 : 0;
}

static double get_x9(double y, double s2, double b2, double sb2) { /* system.f90:2290-2297 */
  return (s2 * (y * y) + b2 * sb2 + 2 * sb2 * y) / ((y * y) * ((b2 * b2) + 2 * b2 * y + (y * y)));
}

/* algo_solver 2..6 of the ideal-MHD inversion (system.f90:732-1158); the
   reference's exit() calls become error codes: 8 (algo 3 out of
   iterations), 12 (algo 6 without a solution), 11 (no such solver) */
static int cons2prim_mhd_algo(const Phys* ph, double* u, double* v, int* iters) {
  const EchoParams* p = ph->p;
  const double eps = 1.e-12;
  int algo = p->algo_solver, nu = ph->nu, nv = ph->nv, kbx = ph->kbx, kby = ph->kby, kbz = ph->kbz;
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3, gm = ph->gm;
  double uin[ECHO_MAX_NV];
  for (int k = 0; k < nu; k++) uin[k] = gm * u[k];
  double DD = uin[KRH], sx = uin[KVX], sy = uin[KVY], sz = uin[KVZ], UU = uin[KPR];
  double bx = uin[kbx], by = uin[kby], bz = uin[kbz];
  int errcode = 0;
  *iters = 0;
  if (algo == 2 || algo == 3) {
    v[kbx] = uin[kbx];
    v[kby] = uin[kby];
    v[kbz] = uin[kbz];
    double B2 = bx * bx + by * by + bz * bz * g3;
    double SB = sx * bx + sy * by + sz * bz;
    double SB2 = SB * SB;
    double SS2 = sx * sx + sy * sy + sz * sz / g3;
    double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR], en = 0;
    errcode = eos_energy(ph, rh, &en, pr);
    double xs, ys;
    if (algo == 2) {
      double v2old = g1 * (vx * vx) + g2 * (vy * vy) + g3 * (vz * vz);
      double X[2] = {(en + pr) / (1 - v2old), pr}, F[2] = {0, 0};
      Sist4 s4 = {ph, B2, SB2, SS2, UU, DD, 0.};
      int nfev = 0;
      (void)brentm(2, sist4_fn, &s4, X, F, 1.e-14, 1.e-14, 300, 3, &nfev);
      *iters = nfev;
      ys = X[0];
      pr = X[1];
      xs = s4.xinner;
    } else {
      double v2 = g1 * (vx * vx) + g2 * (vy * vy) + g3 * (vz * vz);
      double X[3] = {v2, (en + pr) / (1 - v2), pr}, F[3], J[3][3], L[3][3], DX[3], mF[3], Xt[3];
      double Fnorm = 0, Fnl = 0;
      int P[3], it = 0;
      Sist3 s3 = {ph, B2, SB2, SS2, UU, DD};
      getfun(&s3, X, F, J, &Fnorm, 1);
      while (Fnorm >= 1.e-14) {
        ludecompose(J, L, P, 4.e-16);
        for (int i = 0; i < 3; i++) mF[i] = -F[i];
        lusolve(L, J, P, DX, mF);
        double lambda = 1.;
        for (int i = 0; i < 3; i++) Xt[i] = X[i] + lambda * DX[i];
        getfun(&s3, Xt, F, J, &Fnl, 1);
        if ((Fnl > (1 - lambda / 2) * Fnorm) && (lambda > 1. / 64)) {
          for (;;) {
            lambda = lambda / 2.;
            for (int i = 0; i < 3; i++) Xt[i] = X[i] + lambda * DX[i];
            getfun(&s3, Xt, F, J, &Fnl, 0);
            if (!((Fnl > (1 - lambda / 2) * Fnorm) && (lambda > 1. / 64))) {
              for (int i = 0; i < 3; i++) X[i] = X[i] + lambda * DX[i];
              Fnorm = Fnl;
              break;
            }
          }
        } else {
          for (int i = 0; i < 3; i++) X[i] = X[i] + lambda * DX[i];
          Fnorm = Fnl;
        }
        it = it + 1;
        if (it > 300) {
          *iters = it;
          return 8;
        }
      }
      *iters = it;
      xs = X[0];
      ys = X[1];
      pr = X[2];
    }
    rh = DD * sqrt(1 - xs);
    v[KRH] = rh;
    v[KVX] = (sx + SB * bx / ys) / (ys + B2);
    v[KVY] = (sy + SB * by / ys) / (ys + B2);
    v[KVZ] = (sz / g3 + SB * bz / ys) / (ys + B2);
    v[KPR] = pr;
    if (p->divclean) v[ph->kglm] = u[ph->kglm];
    return errcode;
  }
  if (algo == 4 || algo == 5) {
    double S2 = sx * sx + sy * sy + sz * sz / g3;
    double B2 = bx * bx + by * by + bz * bz * g3;
    double SB = (sx * bx + sy * by + sz * bz);
    double SB2 = SB * SB;
    RtCtx c = {B2, SB2, S2, UU, DD, algo == 4 ? (4.0 / 3.0 - 1) / (4.0 / 3.0) : 0.25, 0., algo == 4 ? 7 : 8};
    double v2_old = algo == 4 ? v[KVX] * v[KVX] + v[KVY] * v[KVY] + v[KVZ] * v[KVZ]
                              : v[KVX] * v[KVX] + v[KVY] * v[KVY] + v[KVZ] * v[KVZ] * g3;
    int ierr = 0;
    double v2 = rtsafe(&c, v2_old, 0., 1. - 1.e-11, 1.e-12, &ierr);
    if (algo == 4 && ierr > 0) return 0; /* system.f90:926: returns, v untouched */
    if (algo == 5 && ((v2 >= 1) || (ierr > 0))) return 778;
    for (int k = 0; k < nv; k++) v[k] = uin[k];
    if (p->divclean) v[ph->kglm] = u[ph->kglm];
    double w = c.w, rh = DD * sqrt(1. - v2);
    v[KRH] = rh;
    if (algo == 4) {
      double pg = c.gam * (w * (1. - v2) - rh);
      v[KPR] = fmax(pg, eps);
    } else {
      v[KPR] = 0.25 * (1 - v2) * w;
    }
    double vb = SB / w;
    v[KVX] = (sx + vb * bx) / (w + B2);
    v[KVY] = (sy + vb * by) / (w + B2);
    v[KVZ] = (sz / g3 + vb * bz) / (w + B2);
    return 0;
  }
  if (algo == 6) {
    int exact9 = 1;
    double v2_old = v[KVX] * v[KVX] + v[KVY] * v[KVY] + v[KVZ] * v[KVZ];
    double oldsol9 = 4 * v[KPR] / (1 - v2_old);
    double S2 = sx * sx + sy * sy + sz * sz;
    double B2 = bx * bx + by * by + bz * bz;
    double SB = (sx * bx + sy * by + sz * bz);
    double SB2 = SB * SB;
    double b9 = 8 * B2 - 4 * UU;
    double c9 = 7 * (B2 * B2) - 8 * B2 * UU + S2;
    double d9 = 2 * (B2 * B2 * B2) - 4 * (B2 * B2) * UU + 2 * B2 * S2;
    double e9 = SB2 * B2;
    double p9 = (24 * c9 - 3 * (b9 * b9)) / 72;
    double q9 = ((b9 * b9 * b9) - 12 * b9 * c9 + 72 * d9) / 216;
    double dnull9 = (c9 * c9) - 3 * b9 * d9 + 36 * e9;
    double deinz9 = 2 * (c9 * c9 * c9) - 9 * b9 * c9 * d9 + 27 * (b9 * b9) * e9 + 81 * (d9 * d9) - 216 * c9 * e9;
    double discr9 = (deinz9 * deinz9) - 4 * (dnull9 * dnull9 * dnull9);
    double sbig9 = 0., sol9 = -1., v2 = 0.;
    if (discr9 > 0) {
      double droot9 = sqrt(discr9);
      double qbig9 = pow(0.5 * (deinz9 + droot9), 1. / 3.);
      double drad9 = -2 * p9 / 3 + (qbig9 + dnull9 / qbig9) / 9;
      if (drad9 <= 0) return 12;
      sbig9 = 0.5 * sqrt(drad9);
    } else if (dnull9 > 0) {
      double phi9 = acos(deinz9 / (2 * sqrt(dnull9 * dnull9 * dnull9)));
      sbig9 = 0.5 * sqrt(-2. * p9 / 3 + 2. / 9. * sqrt(dnull9) * cos(phi9 / 3.));
    } else {
      if (solver10_approximate(b9, c9, d9, oldsol9, &sol9)) return 12;
      exact9 = 0;
      v2 = get_x9(sol9, S2, B2, SB2);
      if ((v2 < 0) || (v2 > 1) || (sol9 < 0)) return 12;
    }
    if (exact9) {
      /* sol1..sol4 start at -1 each call (the reference leaves the ones of
         a negative radicand unset) */
      double sol1 = -1., sol2 = -1., sol3 = -1., sol4 = -1.;
      double rad129 = -4 * (sbig9 * sbig9) - 2 * p9 + q9 / sbig9;
      double rad349 = -4 * (sbig9 * sbig9) - 2 * p9 - q9 / sbig9;
      double rapp9 = -b9 / 12;
      if (rad129 >= 0) {
        double root129 = 0.5 * sqrt(rad129);
        sol1 = rapp9 - sbig9 - root129;
        sol2 = rapp9 - sbig9 + root129;
      }
      if (rad349 >= 0) {
        double root349 = 0.5 * sqrt(rad349);
        sol3 = rapp9 + sbig9 - root349;
        sol4 = rapp9 + sbig9 + root349;
      }
      double dist9 = 1.e100, v9;
      sol9 = -1.;
      if (sol2 > 0) {
        v9 = get_x9(sol2, S2, B2, SB2);
        if ((v9 >= 0) && (v9 < 1)) {
          sol9 = sol2;
          v2 = v9;
          dist9 = fabs(oldsol9 - sol9);
          if (sol1 > 0) {
            v9 = get_x9(sol1, S2, B2, SB2);
            if ((v9 >= 0) && (v9 < 1)) {
              double d19 = fabs(oldsol9 - sol1);
              if (d19 <= dist9) {
                sol9 = sol1;
                dist9 = d19;
                v2 = v9;
              }
            }
          }
        }
      }
      if (sol4 > 0) {
        v9 = get_x9(sol4, S2, B2, SB2);
        if ((v9 >= 0) && (v9 < 1)) {
          double d49 = fabs(oldsol9 - sol4);
          if (d49 <= dist9) {
            sol9 = sol4;
            dist9 = d49;
            v2 = v9;
          }
        }
        if (sol3 > 0) {
          v9 = get_x9(sol3, S2, B2, SB2);
          if ((v9 >= 0) && (v9 < 1)) {
            double d39 = fabs(oldsol9 - sol3);
            if (d39 <= dist9) {
              sol9 = sol3;
              dist9 = d39;
              v2 = v9;
            }
          }
        }
      }
      if (sol9 < 0) return 12;
    }
    for (int k = 0; k < nv; k++) v[k] = uin[k];
    v[KRH] = DD * sqrt(1. - v2);
    v[KPR] = sol9 / 4 * (1 - v2);
    double vb = SB / sol9;
    v[KVX] = (sx + vb * bx) / (sol9 + B2);
    v[KVY] = (sy + vb * by) / (sol9 + B2);
    v[KVZ] = (sz + vb * bz) / (sol9 + B2);
    if (p->divclean) v[ph->kglm] = u[ph->kglm];
    return 0;
  }
  return 11;
}

static int cons2prim(const Phys* ph, double* u, double* v, int* iters) {
  const EchoParams* p = ph->p;
  if (p->mhd == 2) return cons2prim_res(ph, u, v, iters);
  if (p->mhd == 1 && !p->viscosity && p->algo_solver != ECHO_C2P_BRENT && p->algo_solver != ECHO_C2P_NEWTON &&
      p->algo_solver != ECHO_C2P_MLP)
    return cons2prim_mhd_algo(ph, u, v, iters); /* 2..6, else 11 */
  const double tol = 1.e-12, eps = 1.e-12;
  const int iter_max = 100, ivmax = 100, ipmax = 100;
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3, gm = ph->gm;
  int errcode = 0;
  *iters = 0;
  double d = gm * u[KRH];
  double sx = gm * u[KVX];
  double sy = gm * u[KVY];
  double sz = gm * u[KVZ] / g3;
  double et = gm * u[KPR];
  double s2 = g1 * sx * sx + g2 * sy * sy + g3 * sz * sz;

  if (!p->viscosity && !p->mhd) {
    /* ideal HD Newton-Raphson on p (system.f90:511-561) */
    double pr = v[KPR], w = 0, v2, glf, rh = 0, en, drhdpr, dendpr;
    double pr_eos = 0, dprdrh = 0, dprden = 0, f, df, dpr;
    int iter;
    for (iter = 1; iter <= iter_max; iter++) {
      w = et + pr;
      v2 = s2 / (w * w);
      if (v2 >= 1.) {
        *iters = iter;
        return 777;
      }
      glf = 1. / sqrt(1. - v2);
      rh = d / glf;
      en = w * (1. - v2) - pr;
      drhdpr = rh * v2 * glf / (en + pr);
      dendpr = v2;
      errcode = eos_pressure(ph, rh, en, &pr_eos, &dprdrh, &dprden);
      f = pr_eos - pr;
      df = dprdrh * drhdpr + dprden * dendpr - 1.;
      dpr = -f / df;
      if (fabs(dpr) < tol * pr) break;
      pr = pr + dpr;
    }
    *iters = iter;
    v[KRH] = rh;
    v[KVX] = sx / w;
    v[KVY] = sy / w;
    v[KVZ] = sz / w;
    v[KPR] = pr;
    if (pr <= 0) errcode = 777;
    return errcode;
  }

  if (p->viscosity) {
    /* nested iteration (system.f90:564-666).  The reference's outer loop
     * ends after one pass (its test compares v^2 of the new velocities with
     * the Newton's own v^2, the same number).  algo_solver ECHO_C2P_NEWTON
     * and ECHO_C2P_MLP iterate the passes to the fixed point (max |dv| <=
     * 1e-14, each pass's Newton from the last pass's p), the learned
     * seed's equal-residual comparison; the oracle runs them from the warm
     * start. */
    const int conv = p->algo_solver == ECHO_C2P_NEWTON || p->algo_solver == ECHO_C2P_MLP;
    double uin[ECHO_MAX_NV], vprim[ECHO_MAX_NV];
    for (int k = 0; k < ph->nu; k++) uin[k] = gm * u[k];
    d = uin[KRH];
    for (int k = KPIBU; k <= KPIZZ; k++) v[k] = uin[k] / uin[KRH];
    double vx = v[KVX], vy = v[KVY], vz = v[KVZ];
    double v2 = g1 * (vx * vx) + g2 * (vy * vy) + g3 * (vz * vz);
    for (int k = 0; k < ph->nv; k++) vprim[k] = v[k];
    double rh = 0, pr = 0, glf, en, drhdpr, dendpr, pr_eos = 0, dprdrh = 0,
           dprden = 0, f, df, dpr;
    double p0 = v[KPR];
    int iv, ip, tot = 0;
    for (iv = 1; iv <= ivmax; iv++) {
      vprim[KVX] = vx;
      vprim[KVY] = vy;
      vprim[KVZ] = vz;
      Pit pi;
      derived_pi_any(ph, vprim, &pi);
      double en1 = et + v[KPIBU] + pi.tt * ph->g0;
      double sx_cov = uin[KVX] - pi.tx;
      double sy_cov = uin[KVY] - pi.ty;
      double sz_cov = uin[KVZ] - pi.tz * g3;
      sx = sx_cov;
      sy = sy_cov;
      sz = sz_cov / g3;
      s2 = sx * sx_cov + sy * sy_cov + sz * sz_cov;
      pr = p0;
      for (ip = 1; ip <= ipmax; ip++) {
        tot++;
        v2 = s2 / ((en1 + pr) * (en1 + pr));
        if (v2 >= 1.) {
          *iters = tot;
          return 107;
        }
        glf = 1. / sqrt(1. - v2);
        rh = d / glf;
        en = (en1 + pr) * (1. - v2) - pr - vprim[KPIBU];
        drhdpr = rh * v2 * glf / (en + pr);
        dendpr = v2;
        errcode = eos_pressure(ph, rh, en, &pr_eos, &dprdrh, &dprden);
        f = pr_eos - pr;
        df = dprdrh * drhdpr + dprden * dendpr - 1.;
        dpr = -f / df;
        if (fabs(dpr) < tol * pr) break;
        pr = pr + dpr;
      }
      double nvx = sx / (en1 + pr);
      if (fabs(nvx) < eps) nvx = 0.;
      double nvy = sy / (en1 + pr);
      if (fabs(nvy) < eps) nvy = 0.;
      double nvz = sz / (en1 + pr);
      if (fabs(nvz) < eps) nvz = 0.;
      /* the converged passes' test, as the library states it: a component whose
       * old and new values are both below 2 eps (where the zeroing above can
       * make the passes alternate) counts as settled */
      double dvs = fmax(fmax(fabs(nvx) < 2. * eps && fabs(vx) < 2. * eps ? 0. : fabs(nvx - vx),
                             fabs(nvy) < 2. * eps && fabs(vy) < 2. * eps ? 0. : fabs(nvy - vy)),
                        fabs(nvz) < 2. * eps && fabs(vz) < 2. * eps ? 0. : fabs(nvz - vz) * ph->gp);
      vx = nvx;
      vy = nvy;
      vz = nvz;
      vprim[KVX] = vx;
      vprim[KVY] = vy;
      vprim[KVZ] = vz;
      if (conv) {
        p0 = pr;
        if (dvs <= 1.e-14) break;
      } else if (fabs(g1 * (vx * vx) + g2 * (vy * vy) + g3 * (vz * vz) - v2) < eps) {
        break;
      }
    }
    *iters = tot;
    v[KRH] = rh;
    v[KVX] = vx;
    v[KVY] = vy;
    v[KVZ] = vz;
    v[KPR] = pr;
    if (p->obtained_zz) {
      Pit pi;
      derived_pi_zz(ph, v, &pi);
      v[KPIZZ] = pi.zz;
    }
    return errcode;
  }

  /* ideal MHD, algo_solver 1: BRENTM on sist3 (system.f90:668-730) */
  {
    double uin[ECHO_MAX_NV];
    for (int k = 0; k < ph->nu; k++) uin[k] = gm * u[k];
    double DD = uin[KRH];
    sx = uin[KVX];
    sy = uin[KVY];
    sz = uin[KVZ];
    double UU = uin[KPR];
    double bx = uin[ph->kbx], by = uin[ph->kby], bz = uin[ph->kbz];
    v[ph->kbx] = uin[ph->kbx];
    v[ph->kby] = uin[ph->kby];
    v[ph->kbz] = uin[ph->kbz];
    double B2 = bx * bx + by * by + bz * bz * g3;
    double SB = sx * bx + sy * by + sz * bz;
    double SB2 = SB * SB;
    double SS2 = sx * sx + sy * sy + sz * sz / g3;
    double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR];
    double en = 0;
    errcode = eos_energy(ph, rh, &en, pr);
    double v2 = g1 * (vx * vx) + g2 * (vy * vy) + g3 * (vz * vz);
    double X[3], F[3] = {0, 0, 0};
    X[0] = v2;
    X[1] = (en + pr) / (1 - v2);
    X[2] = pr;
    Sist3 s = {ph, B2, SB2, SS2, UU, DD};
    int nfev = 0;
    (void)brentm3(&s, X, F, 1.e-14, 1.e-14, 300, 3, &nfev);
    *iters = nfev;
    double xs = X[0], ys = X[1];
    pr = X[2];
    rh = DD * sqrt(1 - xs);
    vx = (sx + SB * bx / ys) / (ys + B2);
    vy = (sy + SB * by / ys) / (ys + B2);
    vz = (sz / g3 + SB * bz / ys) / (ys + B2);
    v[KRH] = rh;
    v[KVX] = vx;
    v[KVY] = vy;
    v[KVZ] = vz;
    v[KPR] = pr;
    if (p->divclean) v[ph->kglm] = u[ph->kglm];
    return errcode;
  }
}

/* ------------------------------------------------------------------------ */
/* system_flux (system.f90:1316-1583)                                       */
/* ------------------------------------------------------------------------ */
static int system_flux(const Phys* ph, double* v, double* u, double* f,
                       double* vf, int dir) {
  const EchoParams* p = ph->p;
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3, gp = ph->gp, gm = ph->gm;
  double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR];
  double en = 0;
  int err = eos_energy(ph, rh, &en, pr);
  if (err) return err;
  double v2 = g1 * vx * vx + g2 * vy * vy + g3 * vz * vz;
  if (v2 > 1) return 333;
  double glf = 1. / sqrt(1. - v2);
  double w, E[3] = {0, 0, 0}, EXB[3] = {0, 0, 0}, E2 = 0, B2 = 0, EEM = 0;
  int kbx = ph->kbx, kby = ph->kby, kbz = ph->kbz, kglm = ph->kglm;
  Pit pi = {0, 0, 0, 0, 0};
  if (!p->viscosity) {
    w = en + pr;
    if (p->mhd) {
      e_field(ph, v, E);
      E2 = E[0] * E[0] + E[1] * E[1] + (E[2] * E[2]) / g3;
      exb(ph, E, v + kbx, EXB);
      B2 = v[kbx] * v[kbx] + v[kby] * v[kby] + (v[kbz] * v[kbz]) * g3;
      EEM = 0.5 * (E2 + B2);
    }
  } else {
    w = en + pr + v[KPIBU];
  }
  double ww = w * (glf * glf);
  u[KRH] = rh * glf;
  int nou = 5, nv = ph->nv, nu = ph->nu;
  if (p->viscosity) {
    derived_pi_any(ph, v, &pi);
    for (int k = KPIBU; k < nv; k++) u[k] = v[k] * u[KRH];
    u[KVX] = ww * vx + pi.tx;
    u[KVY] = ww * vy + pi.ty;
    u[KVZ] = (ww * vz + pi.tz) * g3;
    u[KPR] = ww - pr - v[KPIBU] - pi.tt * ph->g0;
  } else if (p->mhd) {
    u[KVX] = ww * vx + EXB[0];
    u[KVY] = ww * vy + EXB[1];
    u[KVZ] = ww * vz * g3 + EXB[2];
    u[KPR] = ww - pr + EEM;
    u[kbx] = v[kbx];
    u[kby] = v[kby];
    u[kbz] = v[kbz];
    if (p->mhd == 2) {
      u[ph->kex] = v[ph->kex];
      u[ph->key] = v[ph->key];
      u[ph->kez] = v[ph->kez];
    }
    if (p->divclean) u[kglm] = v[kglm] / gp;
  } else {
    u[KVX] = ww * vx;
    u[KVY] = ww * vy;
    u[KVZ] = ww * vz * g3;
    u[KPR] = ww - pr;
  }
  double wwdir, vdir, gcov_dir;
  if (dir == 1) {
    wwdir = ww * vx;
    vdir = vx;
    gcov_dir = g1;
    f[KRH] = rh * glf * vx;
    if (p->viscosity) {
      f[KVX] = wwdir * vx * g1 + pr + v[KPIBU] + v[KPIXX] * g1;
      f[KVY] = wwdir * vy * g2 + v[KPIXY] * g2;
      f[KVZ] = wwdir * vz * g3 + v[KPIXZ] * g3;
      f[KPR] = wwdir + pi.tx;
      for (int k = nou; k < nv; k++) f[k] = u[k] * vx;
    } else if (p->mhd) {
      f[KVX] = wwdir * vx - E[0] * E[0] - v[kbx] * v[kbx] + pr + EEM;
      f[KVY] = wwdir * vy - E[0] * E[1] - v[kbx] * v[kby];
      f[KVZ] = wwdir * vz * g3 - E[0] * E[2] - v[kbx] * v[kbz] * g3;
      f[KPR] = wwdir + EXB[0];
      f[kbx] = 0.;
      f[kby] = -E[2] * gm;
      f[kbz] = +E[1] * gm;
      if (p->mhd == 2) {
        f[ph->kex] = 0.;
        f[ph->key] = +v[kbz] * g3 * gm;
        f[ph->kez] = -v[kby] * g2 * gm;
      }
      if (p->divclean) {
        f[kbx] = v[kglm];
        f[kglm] = v[kbx] / gp;
      }
    } else {
      f[KVX] = wwdir * vx * g1 + pr;
      f[KVY] = wwdir * vy * g2;
      f[KVZ] = wwdir * vz * g3;
      f[KPR] = wwdir;
    }
  } else if (dir == 2) {
    wwdir = ww * vy;
    vdir = vy;
    gcov_dir = g2;
    f[KRH] = rh * glf * vy;
    if (p->viscosity) {
      f[KVX] = wwdir * vx * g1 + v[KPIXY] * g1;
      f[KVY] = wwdir * vy * g2 + pr + v[KPIBU] + v[KPIYY] * g2;
      f[KVZ] = wwdir * vz * g3 + v[KPIYZ] * g3;
      f[KPR] = wwdir + pi.ty;
      for (int k = nou; k < nv; k++) f[k] = u[k] * vy;
    } else if (p->mhd) {
      f[KVX] = wwdir * vx - E[1] * E[0] - v[kby] * v[kbx];
      f[KVY] = wwdir * vy - E[1] * E[1] - v[kby] * v[kby] + pr + EEM;
      f[KVZ] = wwdir * vz * g3 - E[1] * E[2] - v[kby] * v[kbz] * g3;
      f[KPR] = wwdir + EXB[1];
      f[kbx] = E[2] * gm;
      f[kby] = 0.;
      f[kbz] = -E[0] * gm;
      if (p->mhd == 2) {
        f[ph->kex] = -v[kbz] * g3 * gm;
        f[ph->key] = 0.;
        f[ph->kez] = +v[kbx] * g1 * gm;
      }
      if (p->divclean) {
        f[kby] = v[kglm];
        f[kglm] = v[kby] / gp;
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
    if (p->viscosity) {
      f[KVX] = wwdir * vx * g1 + v[KPIXZ] * g1;
      f[KVY] = wwdir * vy * g2 + v[KPIYZ] * g2;
      f[KVZ] = wwdir * vz * g3 + pr + v[KPIBU] + v[KPIZZ] * g3;
      f[KPR] = wwdir + pi.tz;
      for (int k = nou; k < nv; k++) f[k] = u[k] * vz;
    } else if (p->mhd) {
      f[KVX] = wwdir * vx - E[2] / g3 * E[0] - v[kbz] * v[kbx];
      f[KVY] = wwdir * vy - E[2] / g3 * E[1] - v[kbz] * v[kby];
      f[KVZ] = wwdir * vz * g3 - (E[2] * E[2]) / g3 - (v[kbz] * v[kbz]) * g3 + pr + EEM;
      f[KPR] = wwdir + EXB[2] / g3;
      f[kbx] = -E[1] * gm;
      f[kby] = E[0] * gm;
      f[kbz] = 0.;
      if (p->mhd == 2) {
        f[ph->kex] = +v[kby] * g2 * gm;
        f[ph->key] = -v[kbx] * g1 * gm;
        f[ph->kez] = 0.;
      }
      if (p->divclean) {
        f[kbz] = v[kglm] / g3;
        f[kglm] = v[kbz] / gp;
      }
    } else {
      f[KVX] = wwdir * vx * g1;
      f[KVY] = wwdir * vy * g2;
      f[KVZ] = wwdir * vz * g3 + pr;
      f[KPR] = wwdir;
    }
  }
  for (int k = 0; k < nu; k++) u[k] = u[k] * gp;
  for (int k = 0; k < nu; k++) f[k] = f[k] * gp;
  double ca2;
  if (p->mhd) {
    double bb2 = B2 - E2;
    ca2 = bb2 / (bb2 + (en + pr));
  } else {
    ca2 = 0.;
  }
  double cs2 = 0;
  err = eos_sound(ph, rh, en, pr, &cs2);
  if (err) return err;
  double a2 = cs2 + ca2 - cs2 * ca2;
  double den = 1. / (1. - v2 * a2);
  double vf1 = den * (1. - a2) * vdir;
  double vf2 = den * sqrt(a2 * (1. - v2) * ((1. - v2 * a2) / gcov_dir - (1. - a2) * (vdir * vdir)));
  vf[0] = vf1 + vf2;
  vf[1] = vf1 - vf2;
  if (p->mhd == 2) {
    /* resistive: the light cone bounds the Riemann fan (the E, B waves); the
       reference keeps the ideal fast speed here (system.f90:1557-1580) */
    vf[0] = 1. / sqrt(gcov_dir);
    vf[1] = -vf[0];
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* system_source (system.f90:1587-1842), non-resistive                      */
/* v: cell primitives (copy), d: deriv of the cell                          */
/* ------------------------------------------------------------------------ */
/* kap, when not NULL and the run is viscous, receives the relaxation rates
   of the Israel-Stewart equations on the conserved stresses: the source of
   u[k] = sqrt(-g) rho gamma v[k] holds -kap u[k] with kap[0] = 1/(gamma tau_Pi)
   for the bulk pressure and kap[1] = 1/(gamma tau_pi) for the shear
   components (the -1/tau (v[k] + ...) terms times rho sqrt(-g)). */
static int system_source(const Phys* ph, double* v, const double* dv, double rhoC,
                         double* src, double* stiff, double* kap) {
  const EchoParams* p = ph->p;
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3, gp = ph->gp, g0 = ph->g0;
  double t = ph->t;
  for (int k = 0; k < ph->nv; k++) src[k] = 0.;
  if (stiff)
    for (int k = 0; k < ph->nv; k++) stiff[k] = 0.;
  double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR];
  double en = 0;
  int err = eos_energy(ph, rh, &en, pr);
  if (err) return err;
  double v2 = g1 * vx * vx + g2 * vy * vy + g3 * vz * vz;
  double glf = 1. / sqrt(1. - v2);
  double ut = glf;
  const double lambda0 = 1., lambda1 = 1., lambda2 = 0.;
  if (p->coordinates == ECHO_BJORKEN) {
    if (!p->viscosity) {
      double w = en + pr;
      double ww = w * (glf * glf);
      if (p->mhd) {
        double E[3];
        e_field(ph, v, E); /* the reference takes the ideal E here also for
                              resistive runs (system.f90:1641) */
        double bx = v[ph->kbx], by = v[ph->kby], bz = v[ph->kbz];
        double B2 = bx * bx + by * by + (bz * bz) * g3;
        double E2 = E[0] * E[0] + E[1] * E[1] + (E[2] * E[2]) / g3;
        double EEM = 0.5 * (E2 + B2);
        double e3g = E[2] / g3;
        src[KPR] = -t * (ww * vz * vz - e3g * e3g - bz * bz + (EEM + pr) / g3);
      } else {
        src[KPR] = -t * (ww * vz * vz + pr / g3);
      }
    } else {
      double sigma[6], eta, zeta, tau_pi, tau_pi_big;
      get_sigma(ph, v, dv, sigma);
      err = viscous_parameters(ph, v[KRH], v[KPR], &eta, &zeta, &tau_pi, &tau_pi_big);
      if (err) return err;
      Pit pi;
      derived_pi_any(ph, v, &pi);
      double pitt = pi.tt, pitx = pi.tx, pity = pi.ty, pitz = pi.tz;
      double dutdt = dv[DTT], dutdx = dv[DTX], dutdy = dv[DTY], dutdz = dv[DTZ];
      double duxdx = dv[DXX], duydy = dv[DYY], duzdz = dv[DZZ], duzdt = dv[DZT];
      double duzdx = dv[DZX], duzdy = dv[DZY], duxdt = dv[DXT], duxdy = dv[DXY];
      double duxdz = dv[DXZ], duydt = dv[DYT], duydx = dv[DYX], duydz = dv[DYZ];
      double sum_der = dutdt + duxdx + duydy + duzdz;
      double sum_der_t = sum_der + ut / t;
      double sum_der_0 = g0 * (glf * dutdt + glf * v[KVX] * dutdx + glf * v[KVY] * dutdy + glf * v[KVZ] * dutdz);
      double sum_der_x = g1 * (glf * duxdt + glf * v[KVX] * duxdx + glf * v[KVY] * duxdy + glf * v[KVZ] * duxdz);
      double sum_der_y = g2 * (glf * duydt + glf * v[KVX] * duydx + glf * v[KVY] * duydy + glf * v[KVZ] * duydz);
      double sum_der_z = glf * ((t * t) * duzdt + 2. * t * v[KVZ]) +
                         (t * t) * (glf * v[KVX] * duzdx + glf * v[KVY] * duzdy + glf * v[KVZ] * duzdz);
      double w = en + pr + v[KPIBU];
      double ww = w * (glf * glf);
      src[KPR] = -t * (ww * vz * vz + (pr + v[KPIBU]) / g3 + v[KPIZZ]);
      src[KPIBU] = -1. / tau_pi_big * (v[KPIBU] + zeta * sum_der_t) - lambda0 * 4. / 3. * v[KPIBU] * sum_der_t;
      double w0x = -0.5 * (dutdx + duxdt) + 0.5 * glf * (sum_der_x - v[KVX] * g1 * sum_der_0);
      double w0y = -0.5 * (dutdy + duydt) + 0.5 * glf * (sum_der_y - v[KVY] * g2 * sum_der_0);
      double w0z = -0.5 * (dutdz + duzdt) + 0.5 * glf * (sum_der_z - v[KVZ] * g3 * sum_der_0);
      double wxy = 0.5 * (g2 * duydx - duxdy) + 0.5 * glf * (g1 * v[KVX] * sum_der_y - g2 * v[KVY] * sum_der_x);
      double wxz = 0.5 * (g3 * duzdx - duxdz) + 0.5 * glf * (g1 * v[KVX] * sum_der_z - g3 * v[KVZ] * sum_der_x);
      double wyz = 0.5 * (g3 * duzdy - duydz) + 0.5 * glf * (g2 * v[KVY] * sum_der_z - g3 * v[KVZ] * sum_der_y);
      double wx0 = w0x, wy0 = w0y, wz0 = w0z, wyx = -wxy, wzx = -wxz, wzy = -wyz;
      double IVzz = 2. * (pitz * wz0 + v[KPIXZ] * wzx + v[KPIYZ] * wzy);
      double IVxx = 2. * (pitx * wx0 + v[KPIXY] * wxy + v[KPIXZ] * wxz);
      double IVyy = 2. * (pity * wy0 + v[KPIXY] * wyx + v[KPIYZ] * wyz);
      double IVxy = v[KPIXX] * wyx + v[KPIYY] * wxy + v[KPIXZ] * wyz + v[KPIYZ] * wxz + pitx * wy0 + pity * wx0;
      double IVxz = v[KPIXX] * wzx + v[KPIZZ] * wxz + v[KPIXY] * wzy + v[KPIYZ] * wxy + pitx * wz0 + pitz * wx0;
      double IVyz = v[KPIYY] * wzy + v[KPIZZ] * wyz + v[KPIXY] * wzx + v[KPIXZ] * wyx + pity * wz0 + pitz * wy0;
      (void)pitt;
      if (kap) {
        kap[0] = 1. / (glf * tau_pi_big);
        kap[1] = 1. / (glf * tau_pi);
      }
      src[KPIZZ] = -1. / tau_pi * (v[KPIZZ] + 2. * eta * sigma[SZZ]) - 2. * glf * v[KPIZZ] / t -
                   2. * (glf * vz) * pitz / t - lambda0 * 4. / 3. * v[KPIZZ] * sum_der_t +
                   lambda1 * glf * (2. * v[KVZ] * (pitz * sum_der_0 + v[KPIXZ] * sum_der_x + v[KPIYZ] * sum_der_y + v[KPIZZ] * sum_der_z)) -
                   lambda2 * IVzz;
      src[KPIXZ] = -1. / tau_pi * (v[KPIXZ] + 2. * eta * sigma[SXZ]) + lambda0 * (-4. / 3. * v[KPIXZ] * sum_der_t) -
                   glf / t * v[KPIXZ] - glf * vz * pitx / t +
                   lambda1 * glf * ((pitx * v[KVZ] + pitz * v[KVX]) * sum_der_0 + (v[KPIXX] * v[KVZ] + v[KPIXZ] * v[KVX]) * sum_der_x +
                                    (v[KPIXY] * v[KVZ] + v[KPIYZ] * v[KVX]) * sum_der_y + (v[KPIXZ] * v[KVZ] + v[KPIZZ] * v[KVX]) * sum_der_z) -
                   lambda2 * IVxz;
      src[KPIYZ] = -1. / tau_pi * (v[KPIYZ] + 2. * eta * sigma[SYZ]) + lambda0 * (-4. / 3. * v[KPIYZ] * sum_der_t) -
                   glf / t * v[KPIYZ] - glf * vz * pity / t +
                   lambda1 * glf * ((pity * v[KVZ] + pitz * v[KVY]) * sum_der_0 + (v[KPIXY] * v[KVZ] + v[KPIXZ] * v[KVY]) * sum_der_x +
                                    (v[KPIYY] * v[KVZ] + v[KPIYZ] * v[KVY]) * sum_der_y + (v[KPIYZ] * v[KVZ] + v[KPIZZ] * v[KVY]) * sum_der_z) -
                   lambda2 * IVyz;
      src[KPIXY] = -1. / tau_pi * (v[KPIXY] + 2. * eta * sigma[SXY]) + lambda0 * (-4. / 3. * v[KPIXY] * sum_der_t) +
                   lambda1 * glf * ((pitx * v[KVY] + pity * v[KVX]) * sum_der_0 + (v[KPIXX] * v[KVY] + v[KPIXY] * v[KVX]) * sum_der_x +
                                    (v[KPIXY] * v[KVY] + v[KPIYY] * v[KVX]) * sum_der_y + (v[KPIXZ] * v[KVY] + v[KPIYZ] * v[KVX]) * sum_der_z) -
                   lambda2 * IVxy;
      src[KPIXX] = -1. / tau_pi * (v[KPIXX] + 2. * eta * sigma[SXX]) + lambda0 * (-4. / 3. * v[KPIXX] * sum_der_t) +
                   lambda1 * glf * (2. * v[KVX] * (pitx * sum_der_0 + v[KPIXX] * sum_der_x + v[KPIXY] * sum_der_y + v[KPIXZ] * sum_der_z)) -
                   lambda2 * IVxx;
      src[KPIYY] = -1. / tau_pi * (v[KPIYY] + 2. * eta * sigma[SYY]) + lambda0 * (-4. / 3. * v[KPIYY] * sum_der_t) +
                   lambda1 * glf * (2. * v[KVY] * (pity * sum_der_0 + v[KPIXY] * sum_der_x + v[KPIYY] * sum_der_y + v[KPIYZ] * sum_der_z)) -
                   lambda2 * IVyy;
    }
  } else {
    if (p->viscosity) {
      double sigma[6], eta, zeta, tau_pi, tau_pi_big;
      get_sigma(ph, v, dv, sigma);
      err = viscous_parameters(ph, v[KRH], v[KPR], &eta, &zeta, &tau_pi, &tau_pi_big);
      if (err) return err;
      Pit pi;
      derived_pi_any(ph, v, &pi);
      double pitx = pi.tx, pity = pi.ty, pitz = pi.tz;
      double dutdt = dv[DTT], dutdx = dv[DTX], dutdy = dv[DTY], dutdz = dv[DTZ];
      double duxdx = dv[DXX], duydy = dv[DYY], duzdz = dv[DZZ], duzdt = dv[DZT];
      double duzdx = dv[DZX], duzdy = dv[DZY], duxdt = dv[DXT], duxdy = dv[DXY];
      double duxdz = dv[DXZ], duydt = dv[DYT], duydx = dv[DYX], duydz = dv[DYZ];
      double sum_der = dutdt + duxdx + duydy + duzdz;
      double sum_der_0 = g0 * (glf * dutdt + v[KVX] * dutdx + v[KVY] * dutdy + v[KVZ] * dutdz);
      double sum_der_x = g1 * (glf * duxdt + v[KVX] * duxdx + v[KVY] * duxdy + v[KVZ] * duxdz);
      double sum_der_y = g2 * (glf * duydt + v[KVX] * duydx + v[KVY] * duydy + v[KVZ] * duydz);
      double sum_der_z = g3 * (glf * duzdt + v[KVX] * duzdx + v[KVY] * duzdy + v[KVZ] * duzdz);
      src[KPIBU] = -1. / tau_pi_big * (v[KPIBU] + zeta * sum_der) + lambda0 * (-1. / 3. * v[KPIBU] * sum_der);
      if (kap) {
        kap[0] = 1. / (glf * tau_pi_big);
        kap[1] = 1. / (glf * tau_pi);
      }
      double w0x = -0.5 * (dutdx + duxdt) + 0.5 * glf * (sum_der_x - v[KVX] * g1 * sum_der_0);
      double w0y = -0.5 * (dutdy + duydt) + 0.5 * glf * (sum_der_y - v[KVY] * g2 * sum_der_0);
      double w0z = -0.5 * (dutdz + duzdt) + 0.5 * glf * (sum_der_z - v[KVZ] * g3 * sum_der_0);
      double wxy = 0.5 * (g2 * duydx - duxdy) + 0.5 * glf * (g1 * v[KVX] * sum_der_y - g2 * v[KVY] * sum_der_x);
      double wxz = 0.5 * (g3 * duzdx - duxdz) + 0.5 * glf * (g1 * v[KVX] * sum_der_z - g3 * v[KVZ] * sum_der_x);
      double wyz = 0.5 * (g3 * duzdy - duydz) + 0.5 * glf * (g2 * v[KVY] * sum_der_z - g3 * v[KVZ] * sum_der_y);
      double wx0 = w0x, wy0 = w0y, wz0 = w0z, wyx = -wxy, wzx = -wxz, wzy = -wyz;
      double IVzz = 2. * (pitz * wz0 + v[KPIXZ] * wzx + v[KPIYZ] * wzy);
      double IVxx = 2. * (pitx * wx0 + v[KPIXY] * wxy + v[KPIXZ] * wxz);
      double IVyy = 2. * (pity * wy0 + v[KPIXY] * wyx + v[KPIYZ] * wyz);
      double IVxy = v[KPIXX] * wyx + v[KPIYY] * wxy + v[KPIXZ] * wyz + v[KPIYZ] * wxz + pitx * wy0 + pity * wx0;
      double IVxz = v[KPIXX] * wzx + v[KPIZZ] * wxz + v[KPIXY] * wzy + v[KPIYZ] * wxy + pitx * wz0 + pitz * wx0;
      double IVyz = v[KPIYY] * wzy + v[KPIZZ] * wyz + v[KPIXY] * wzx + v[KPIXZ] * wyx + pity * wz0 + pitz * wy0;
      src[KPIZZ] = -1. / tau_pi * (v[KPIZZ] + 2. * eta * sigma[SZZ]) + lambda0 * (-4. / 3. * v[KPIZZ] * sum_der) +
                   lambda1 * (2. * v[KVZ] * (pitz * sum_der_0 + v[KPIXZ] * sum_der_x + v[KPIYZ] * sum_der_y + v[KPIZZ] * sum_der_z)) -
                   lambda2 * IVzz;
      src[KPIXZ] = -1. / tau_pi * (v[KPIXZ] + 2. * eta * sigma[SXZ]) + lambda0 * (-4. / 3. * v[KPIXZ] * sum_der) +
                   lambda1 * ((pitx * v[KVZ] + pitz * v[KVX]) * sum_der_0 + (v[KPIXX] * v[KVZ] + v[KPIXZ] * v[KVX]) * sum_der_x +
                              (v[KPIXY] * v[KVZ] + v[KPIYZ] * v[KVX]) * sum_der_y + (v[KPIXZ] * v[KVZ] + v[KPIZZ] * v[KVX]) * sum_der_z) -
                   lambda2 * IVxz;
      src[KPIXY] = -1. / tau_pi * (v[KPIXY] + 2. * eta * sigma[SXY]) + lambda0 * (-4. / 3. * v[KPIXY] * sum_der) +
                   lambda1 * ((pitx * v[KVY] + pity * v[KVX]) * sum_der_0 + (v[KPIXX] * v[KVY] + v[KPIXY] * v[KVX]) * sum_der_x +
                              (v[KPIXY] * v[KVY] + v[KPIYY] * v[KVX]) * sum_der_y + (v[KPIXZ] * v[KVY] + v[KPIYZ] * v[KVX]) * sum_der_z) -
                   lambda2 * IVxy;
      src[KPIYZ] = -1. / tau_pi * (v[KPIYZ] + 2. * eta * sigma[SYZ]) + lambda0 * (-4. / 3. * v[KPIYZ] * sum_der) +
                   lambda1 * ((pity * v[KVZ] + pitz * v[KVY]) * sum_der_0 + (v[KPIXY] * v[KVZ] + v[KPIXZ] * v[KVY]) * sum_der_x +
                              (v[KPIYY] * v[KVZ] + v[KPIYZ] * v[KVY]) * sum_der_y + (v[KPIYZ] * v[KVZ] + v[KPIZZ] * v[KVY]) * sum_der_z) -
                   lambda2 * IVyz;
      src[KPIXX] = -1. / tau_pi * (v[KPIXX] + 2. * eta * sigma[SXX]) + lambda0 * (-4. / 3. * v[KPIXX] * sum_der) +
                   lambda1 * (2. * v[KVX] * (pitx * sum_der_0 + v[KPIXX] * sum_der_x + v[KPIXY] * sum_der_y + v[KPIXZ] * sum_der_z)) -
                   lambda2 * IVxx;
      src[KPIYY] = -1. / tau_pi * (v[KPIYY] + 2. * eta * sigma[SYY]) + lambda0 * (-4. / 3. * v[KPIYY] * sum_der) +
                   lambda1 * (2. * v[KVY] * (pity * sum_der_0 + v[KPIXY] * sum_der_x + v[KPIYY] * sum_der_y + v[KPIYZ] * sum_der_z)) -
                   lambda2 * IVyy;
    }
  }
  if (p->mhd == 2) {
    /* charge current and Ohm's law (system.f90:1650-1661, 1747-1756) */
    double vel[3] = {vx, vy, vz}, S[3];
    ohm_stiff(ph, vel, v + ph->kbx, v + ph->kex, glf, S);
    for (int i = 0; i < 3; i++) {
      src[ph->kex + i] = -rhoC * vel[i];
      if (stiff) stiff[ph->kex + i] = S[i];
    }
  }
  if (p->viscosity)
    for (int k = KPIBU; k < ph->nv; k++) src[k] = src[k] * v[KRH];
  for (int k = 0; k < ph->nv; k++) src[k] = src[k] * gp;
  if (stiff)
    for (int k = 0; k < ph->nv; k++) stiff[k] = stiff[k] * gp;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* the grid context                                                         */
/* ------------------------------------------------------------------------ */
struct Orc {
  EchoParams p;
  Phys ph;
  int nx, ny, nz, nv, nu, nvold;
  size_t ncell;
  double dx, dy, dz, ddx, ddy, ddz;
  int nt;
  double *tT, *te, *tp, *tc;
  double *v, *u, *u0, *du[4], *dus[4], *w, *ax, *ay, *az, *deriv;
  double *vold, *vnewstep, *vtmp;
  double* kap; /* imex: 2 relaxation rates per cell, from the last RHS */
  unsigned char* fail;
  double t, tout, dtout, tmax, timeold, timeinterval, dt, g3old;
  double glm_ch, glm_ch_old, aflux[3];
  int run_crashed, errcode, nthreads;
  long long repairs, c2p_iters;
  /* freeze-out hypersurface (hypersurface.f90, out_hyp out.f90:1569-1650) */
  int hyp_on, hyp_first, hyp_type, hyp_n;
  double hyp_value, hyp_time[2];
  double *hyp_field1, *hyp_field2, *hyp_prim, *hyp_back, *hyp_out;
};

#define IDX(e, k, ix, iy, iz) \
  ((((size_t)(k) * (e)->nz + ((iz)-1)) * (e)->ny + ((iy)-1)) * (e)->nx + ((ix)-1))
#define WIDX(e, k, ix, iy, iz)                                            \
  ((((size_t)(k) * ((e)->nz + 2 * NGC) + ((iz) + NGC - 1)) * ((e)->ny + 2 * NGC) + \
    ((iy) + NGC - 1)) * ((e)->nx + 2 * NGC) + ((ix) + NGC - 1))

int orc_nv(const Orc* e) { return e->nv; }
void orc_set_threads(Orc* e, int n) { e->nthreads = n > 0 ? n : 1; }
double orc_time(const Orc* e) { return e->t; }
double orc_dt(const Orc* e) { return e->dt; }
double orc_glm_ch(const Orc* e) { return e->glm_ch; }
long long orc_repairs(const Orc* e) { return e->repairs; }
long long orc_c2p_iters(const Orc* e) { return e->c2p_iters; }

/* check_temp (out.f90:1487-1557): the maximum over the grid, in the
 * Fortran loop order, of the temperature (freeze_type 0) or the energy
 * density (1) that get_derived_temp_for_check (eos.f90:706-759, 972-983)
 * gives from rho and p -- the interpolation of get_derived_data.  Where the
 * call fails (p outside the table) the reference keeps the previous cell's
 * value, which leaves the maximum unchanged: the cell is skipped. */
double orc_check_temp(const Orc* e, int freeze_type) {
  const Phys* ph = &e->ph;
  size_t nc = e->ncell;
  double mx = 0.;
  for (size_t c = 0; c < nc; c++) {
    double en = 0., temp = 0., s = 0.;
    if (get_derived_data(ph, e->v[(size_t)KRH * nc + c], e->v[(size_t)KPR * nc + c], &en, &temp, &s)) continue;
    double x = freeze_type == 0 ? temp : en;
    if (x > mx) mx = x;
  }
  return mx;
}

/* out_vars (out.f90:232-591): field k of the output is bit k of sel, in the
   order the reference writes them; viscous fields need a viscous run, B, E
   and psi an MHD run (psi with divclean) */
static int out_field_on(const EchoParams* p, unsigned sel, int k) {
  if (!(sel >> k & 1u)) return 0;
  if (k >= 8 && k <= 18) return p->viscosity != 0;
  if (k >= 20 && k <= 25) return p->mhd != 0;
  if (k == 26) return p->mhd != 0 && p->divclean != 0;
  return k <= 26;
}

size_t orc_out_vars(const Orc* e, unsigned sel, int precision, void* buf, int* errcode) {
  const Phys* ph = &e->ph;
  size_t nc = e->ncell;
  int nf = 0, fields[32];
  for (int k = 0; k <= 26; k++)
    if (out_field_on(&e->p, sel, k)) fields[nf++] = k;
  size_t prec = precision == 4 ? 4 : 8;
  size_t bytes = prec + (size_t)nf * nc * prec;
  if (errcode) *errcode = 0;
  if (!buf) return bytes;
  unsigned char* out = (unsigned char*)buf;
  if (prec == 8) {
    double t = e->t;
    memcpy(out, &t, 8);
  } else {
    float t = (float)e->t;
    memcpy(out, &t, 4);
  }
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3;
  int first_err = 0;
  for (size_t c = 0; c < nc; c++) {
    double p[ECHO_MAX_NV];
    for (int k = 0; k < e->nv; k++) p[k] = e->v[(size_t)k * nc + c];
    double en = 0., temp = 0., sd = 0.;
    if ((sel & (ECHO_OUT_ENERGY_DENSITY | ECHO_OUT_TEMPERATURE | ECHO_OUT_ENTROPY_DENSITY)) != 0) {
      int err = get_derived_data(ph, p[KRH], p[KPR], &en, &temp, &sd);
      if (err && !first_err) first_err = err;
    }
    Pit pi = {0, 0, 0, 0, 0};
    if (e->p.viscosity) {
      if (e->p.obtained_zz)
        derived_pi_zz(ph, p, &pi);
      else
        derived_pi(ph, p, &pi);
    }
    double E[3] = {0, 0, 0};
    if (e->p.mhd == 1) e_ideal(ph, p + KVX, p + ph->kbx, E);
    for (int f = 0; f < nf; f++) {
      double x = 0.;
      switch (fields[f]) {
        case 0: x = p[KRH]; break;
        case 1: x = p[KVX]; break;
        case 2: x = p[KVY]; break;
        case 3: x = p[KVZ]; break;
        case 4: x = p[KPR]; break;
        case 5: x = en; break;
        case 6: x = temp; break;
        case 7: x = sd; break;
        case 8: x = p[KPIBU]; break;
        case 9: x = pi.tt; break;
        case 10: x = pi.tx; break;
        case 11: x = pi.ty; break;
        case 12: x = pi.tz; break;
        case 13: x = p[KPIXY]; break;
        case 14: x = p[KPIXZ]; break;
        case 15: x = p[KPIYZ]; break;
        case 16: x = p[KPIXX]; break;
        case 17: x = p[KPIYY]; break;
        case 18: x = e->p.obtained_zz ? pi.zz : p[KPIZZ]; break;
        case 19:
          x = 1. / sqrt(1. - p[KVX] * p[KVX] * g1 - p[KVY] * p[KVY] * g2 - p[KVZ] * p[KVZ] * g3);
          break;
        case 20: x = p[ph->kbx]; break;
        case 21: x = p[ph->kby]; break;
        case 22: x = p[ph->kbz]; break;
        case 23: x = e->p.mhd == 2 ? p[ph->kex] : E[0]; break;
        case 24: x = e->p.mhd == 2 ? p[ph->key] : E[1]; break;
        case 25: x = e->p.mhd == 2 ? p[ph->kez] : E[2] / g3; break;
        default: x = p[ph->kglm]; break;
      }
      size_t at = prec + ((size_t)f * nc + c) * prec;
      if (prec == 8) {
        memcpy(out + at, &x, 8);
      } else {
        float y = (float)x;
        memcpy(out + at, &y, 4);
      }
    }
  }
  if (errcode) *errcode = first_err;
  return bytes;
}

static void table_attach(Phys* ph, double** tT, double** te, double** tp,
                         double** tc, int* nt, const double* tab, int n) {
  *nt = n;
  if (n > 0 && tab) {
    *tT = (double*)malloc(sizeof(double) * n);
    *te = (double*)malloc(sizeof(double) * n);
    *tp = (double*)malloc(sizeof(double) * n);
    *tc = (double*)malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++) {
      (*tT)[i] = tab[4 * i + 0];
      (*te)[i] = tab[4 * i + 1];
      (*tp)[i] = tab[4 * i + 2];
      (*tc)[i] = tab[4 * i + 3];
    }
  }
  ph->nt = n;
  ph->tT = *tT;
  ph->te = *te;
  ph->tp = *tp;
  ph->tc = *tc;
}

Orc* orc_create(const EchoParams* p, const double* eos_table, int n_eos) {
  if (p->mhd && p->viscosity) return NULL;
  if (p->mhd > 2) return NULL;
  if (p->mhd == 2 && p->nrk != ECHO_SSP) return NULL; /* common.f90:2114-2118 */
  if (p->imex && p->nrk == ECHO_SSP) return NULL;
  Orc* e = (Orc*)calloc(1, sizeof(Orc));
  e->p = *p;
  phys_setup(&e->ph, &e->p);
  e->nx = p->nx;
  e->ny = p->ny;
  e->nz = p->nz;
  e->nv = e->ph.nv;
  e->nu = e->ph.nu;
  e->nvold = p->mhd ? e->ph.kbz + 1 : KPR + 1;
  e->ncell = (size_t)e->nx * e->ny * e->nz;
  e->nthreads = 1;
  /* common_grid (common.f90:441-481) */
  e->dx = (p->x2 - p->x1) / e->nx;
  e->dy = (p->y2 - p->y1) / e->ny;
  e->dz = (p->z2 - p->z1) / e->nz;
  e->ddx = e->nx > 1 ? 1. / e->dx : 0.;
  e->ddy = e->ny > 1 ? 1. / e->dy : 0.;
  e->ddz = e->nz > 1 ? 1. / e->dz : 0.;
  table_attach(&e->ph, &e->tT, &e->te, &e->tp, &e->tc, &e->nt, eos_table, n_eos);
  size_t nc = e->ncell, nv = e->nv;
  e->v = (double*)calloc(nc * nv, sizeof(double));
  e->u = (double*)calloc(nc * nv, sizeof(double));
  e->u0 = (double*)calloc(nc * nv, sizeof(double));
  int nstage = p->nrk == ECHO_SSP ? 4 : 1;
  for (int s = 0; s < nstage; s++) {
    e->du[s] = (double*)calloc(nc * nv, sizeof(double));
    e->dus[s] = (double*)calloc(nc * nv, sizeof(double));
  }
  e->w = (double*)calloc((size_t)(e->nx + 2 * NGC) * (e->ny + 2 * NGC) * (e->nz + 2 * NGC) * nv,
                         sizeof(double));
  e->ax = (double*)calloc((size_t)2 * (e->nx + 1) * e->ny * e->nz, sizeof(double));
  e->ay = (double*)calloc((size_t)2 * e->nx * (e->ny + 1) * e->nz, sizeof(double));
  e->az = (double*)calloc((size_t)2 * e->nx * e->ny * (e->nz + 1), sizeof(double));
  e->deriv = (double*)calloc(nc * NDERIV, sizeof(double));
  e->vold = (double*)calloc(nc * e->nvold, sizeof(double));
  e->vnewstep = (double*)calloc(nc * e->nvold, sizeof(double));
  e->vtmp = (double*)calloc(nc * nv, sizeof(double));
  e->fail = (unsigned char*)calloc(nc, 1);
  if (p->viscosity && p->imex) e->kap = (double*)calloc(nc * 2, sizeof(double));
  e->glm_ch_old = 0.5; /* common.f90:283 */
  e->tout = 1e300;
  e->dtout = 1e300;
  e->tmax = 1e300;
  return e;
}

void orc_free(Orc* e) {
  if (!e) return;
  free(e->v); free(e->u); free(e->u0);
  for (int s = 0; s < 4; s++) { free(e->du[s]); free(e->dus[s]); }
  free(e->w); free(e->ax); free(e->ay); free(e->az); free(e->deriv);
  free(e->vold); free(e->vnewstep); free(e->vtmp); free(e->fail); free(e->kap);
  free(e->tT); free(e->te); free(e->tp); free(e->tc);
  free(e->hyp_field1); free(e->hyp_field2); free(e->hyp_prim); free(e->hyp_back); free(e->hyp_out);
  free(e);
}

/* ------------------------------------------------------------------------ */
/* freeze-out hypersurface                                                  */
/* ------------------------------------------------------------------------ */
/* Record of one surface element, HYP_REC(nv) doubles: tau, x, y, eta; the nv
 * primitives interpolated to the crossing; dV_tau, dV_x, dV_y, dV_eta with
 * the crossing's sign.  For ideal and viscous runs these are the columns of
 * hy_ide (tau..prex, dV) and hy_vis (Pi, pi^xy..pi^zz) of the reference. */
#define HYP_REC(nv) (8 + (nv))

int orc_hyp_init(Orc* e, int freeze_type, double freeze_value) {
  size_t nc = e->ncell;
  if (freeze_type != 0 && freeze_type != 1) return -1;
  if (!e->hyp_on) {
    e->hyp_field1 = (double*)calloc(nc, sizeof(double));
    e->hyp_field2 = (double*)calloc(nc, sizeof(double));
    e->hyp_prim = (double*)calloc(nc * e->nv, sizeof(double));
    e->hyp_back = (double*)calloc(nc * e->nv, sizeof(double));
    e->hyp_out = (double*)calloc(4 * nc * HYP_REC(e->nv), sizeof(double));
  }
  e->hyp_on = 1;
  e->hyp_first = 1;
  e->hyp_type = freeze_type;
  e->hyp_value = freeze_value;
  e->hyp_n = 0;
  e->hyp_time[0] = e->hyp_time[1] = 0.;
  return 0;
}

/* one crossing between cell (it; ix,iy,iz) and (iit; iix,iiy,iiz):
 * set_fo_ide / set_fo_vis (hypersurface.f90:354-460, 984-1117) and the
 * sign of save_hypersurface_* (:280-350) */
static int hyp_element(Orc* e, int it, int ix, int iy, int iz, int iit, int iix, int iiy, int iiz, int tau_dir,
                       double* rec) {
  int nv = e->nv;
  const double* f_it = it == 1 ? e->hyp_field1 : e->hyp_field2;
  const double* f_iit = iit == 1 ? e->hyp_field1 : e->hyp_field2;
  size_t c = IDX(e, 0, ix, iy, iz), cc = IDX(e, 0, iix, iiy, iiz);
  double fv = e->hyp_value;
  double weight = (f_it[c] - fv) / (f_it[c] - f_iit[cc]);
  double sign_ = f_it[c] - f_iit[cc] >= 0. ? 1.0 : -1.0; /* sign(1.0d0, .) */
  double xc = e->p.x1 + ((double)ix - 0.5) * e->dx, xcc = e->p.x1 + ((double)iix - 0.5) * e->dx;
  double yc = e->p.y1 + ((double)iy - 0.5) * e->dy, ycc = e->p.y1 + ((double)iiy - 0.5) * e->dy;
  double zc = e->p.z1 + ((double)iz - 0.5) * e->dz, zcc = e->p.z1 + ((double)iiz - 0.5) * e->dz;
  rec[0] = e->hyp_time[it - 1] + weight * (e->hyp_time[iit - 1] - e->hyp_time[it - 1]);
  rec[1] = xc + weight * (xcc - xc);
  rec[2] = yc + weight * (ycc - yc);
  rec[3] = zc + weight * (zcc - zc);
  const double* far = tau_dir ? e->hyp_prim : e->hyp_back;
  for (int k = 0; k < nv; k++) {
    double a = e->hyp_back[(size_t)k * e->ncell + c];
    rec[4 + k] = a + weight * (far[(size_t)k * e->ncell + cc] - a);
  }
  double g3 = e->p.coordinates == ECHO_BJORKEN ? e->hyp_time[1] * e->hyp_time[1] : 1.;
  double betasq = rec[4 + KVX] * rec[4 + KVX] + rec[4 + KVY] * rec[4 + KVY] + rec[4 + KVZ] * rec[4 + KVZ] * g3;
  if (betasq > 1.0) return 1; /* the reference stops here ("you have to fix this") */
  double dt = fabs(e->hyp_time[1] - e->hyp_time[0]);
  double dx = e->dx, dy = e->dy, dz = e->nz > 1 ? e->dz : 1.0; /* d_val, common.f90:472-478 */
  rec[4 + nv] = sign_ * ((double)(iit - it) * dx * dy * dz * rec[0]);
  rec[5 + nv] = sign_ * ((double)(iix - ix) * dt * dy * dz * rec[0]);
  rec[6 + nv] = sign_ * ((double)(iiy - iy) * dx * dt * dz * rec[0]);
  rec[7 + nv] = sign_ * ((double)(iiz - iz) * dx * dy * dt * rec[0]);
  return 0;
}

/* out_hyp (out.f90:1569-1650) with find_hypersurface_* (hypersurface.f90:
 * 172-229 and its viscous and MHD twins): the freeze field of the current
 * primitives becomes slice 2, and from the second call on the crossings
 * between the slices (tau) and inside slice 1 (x, y, eta) are collected in
 * the reference's loop order: ix outer, iz inner; per cell tau, x, y, eta */
int orc_hyp_step(Orc* e, int* nout) {
  size_t nc = e->ncell;
  int nv = e->nv;
  if (!e->hyp_on) return -1;
  *nout = 0;
  if (e->hyp_first) e->hyp_time[1] = e->t;
  for (size_t c = 0; c < nc; c++) {
    double en = 0., temp = 0., s = 0.;
    int err = get_derived_data(&e->ph, e->v[(size_t)KRH * nc + c], e->v[(size_t)KPR * nc + c], &en, &temp, &s);
    if (err > 0) return err; /* out_hyp sets run_crashed */
    e->hyp_field1[c] = e->hyp_field2[c];
    e->hyp_field2[c] = e->hyp_type == 0 ? temp : en;
  }
  if (e->hyp_first) {
    e->hyp_first = 0;
    memcpy(e->hyp_prim, e->v, sizeof(double) * nc * nv);
    e->hyp_n = 0;
    return 0;
  }
  memcpy(e->hyp_back, e->hyp_prim, sizeof(double) * nc * nv);
  memcpy(e->hyp_prim, e->v, sizeof(double) * nc * nv);
  e->hyp_time[0] = e->hyp_time[1];
  e->hyp_time[1] = e->t;
  const double fv = e->hyp_value;
  const double *f1 = e->hyp_field1, *f2 = e->hyp_field2;
  int n = 0;
  for (int ix = 1; ix <= e->nx; ix++)
    for (int iy = 1; iy <= e->ny; iy++)
      for (int iz = 1; iz <= e->nz; iz++) {
        size_t c = IDX(e, 0, ix, iy, iz);
        double* rec;
        if ((f2[c] - fv) * (fv - f1[c]) > 0.0) {
          rec = e->hyp_out + (size_t)n * HYP_REC(nv);
          if (hyp_element(e, 1, ix, iy, iz, 2, ix, iy, iz, 1, rec)) return 1;
          n++;
        }
        if (ix < e->nx && (f1[IDX(e, 0, ix + 1, iy, iz)] - fv) * (fv - f1[c]) > 0.0) {
          rec = e->hyp_out + (size_t)n * HYP_REC(nv);
          if (hyp_element(e, 1, ix, iy, iz, 1, ix + 1, iy, iz, 0, rec)) return 1;
          n++;
        }
        if (iy < e->ny && (f1[IDX(e, 0, ix, iy + 1, iz)] - fv) * (fv - f1[c]) > 0.0) {
          rec = e->hyp_out + (size_t)n * HYP_REC(nv);
          if (hyp_element(e, 1, ix, iy, iz, 1, ix, iy + 1, iz, 0, rec)) return 1;
          n++;
        }
        if (iz < e->nz && (f1[IDX(e, 0, ix, iy, iz + 1)] - fv) * (fv - f1[c]) > 0.0) {
          rec = e->hyp_out + (size_t)n * HYP_REC(nv);
          if (hyp_element(e, 1, ix, iy, iz, 1, ix, iy, iz + 1, 0, rec)) return 1;
          n++;
        }
      }
  e->hyp_n = n;
  *nout = n;
  return 0;
}

void orc_hyp_get(const Orc* e, double* out) {
  memcpy(out, e->hyp_out, sizeof(double) * (size_t)e->hyp_n * HYP_REC(e->nv));
}

int orc_set_state(Orc* e, const double* v, const double* u, double t) {
  size_t nc = e->ncell;
  int nv = e->nv;
  memcpy(e->v, v, sizeof(double) * nc * nv);
  e->t = t;
  e->timeold = t;
  e->timeinterval = 0;
  e->dt = 0;
  phys_metric(&e->ph, t);
  e->g3old = e->ph.g3;
  memset(e->vold, 0, sizeof(double) * nc * e->nvold);
  memset(e->vnewstep, 0, sizeof(double) * nc * e->nvold);
  memset(e->deriv, 0, sizeof(double) * nc * NDERIV);
  e->run_crashed = 0;
  e->errcode = 0;
  if (u) {
    memcpy(e->u, u, sizeof(double) * nc * nv);
    return 0;
  }
  double vv[ECHO_MAX_NV], uu[ECHO_MAX_NV];
  for (size_t c = 0; c < nc; c++) {
    for (int k = 0; k < nv; k++) vv[k] = e->v[(size_t)k * nc + c];
    int err = prim2cons(&e->ph, vv, uu);
    if (err) return err;
    for (int k = 0; k < nv; k++) {
      e->u[(size_t)k * nc + c] = uu[k];
      e->v[(size_t)k * nc + c] = vv[k];
    }
  }
  return 0;
}

void orc_get_state(const Orc* e, double* v, double* u) {
  size_t n = e->ncell * e->nv;
  if (v) memcpy(v, e->v, sizeof(double) * n);
  if (u) memcpy(u, e->u, sizeof(double) * n);
}

void orc_set_tout(Orc* e, double tout, double dtout, double tmax) {
  e->tout = tout;
  e->dtout = dtout;
  e->tmax = tmax;
}

/* ------------------------------------------------------------------------ */
/* boundary conditions (evolve.f90:872-1127) for one direction, on w        */
/* ------------------------------------------------------------------------ */
static void evolve_bc(Orc* e, int dir) {
  int n = dir == 0 ? e->nx : dir == 1 ? e->ny : e->nz;
  const int i0 = 1, l0 = NGC;
  int na = dir == 0 ? e->ny : e->nx; /* the two transverse ranges */
  int nb = dir == 2 ? e->ny : e->nz;
  for (int k = 0; k < e->nv; k++) {
    for (int b = 1; b <= nb; b++)
      for (int a = 1; a <= na; a++) {
#define WP(i)                                                          \
  e->w[dir == 0 ? WIDX(e, k, (i), a, b)                                \
                : dir == 1 ? WIDX(e, k, a, (i), b) : WIDX(e, k, a, b, (i))]
        int l;
        switch (e->p.ibc[k][0][dir]) {
          case 0:
            for (l = 1; l <= l0; l++) WP(-NGC + l) = WP(n - NGC + l);
            break;
          case 1:
            for (l = 1; l <= l0; l++) WP(-NGC + l) = WP(NGC + i0 - l);
            break;
          case -1:
            for (l = 1; l <= l0; l++) WP(-NGC + l) = -WP(NGC + i0 - l);
            break;
          case 2:
            for (l = 1; l <= l0; l++) WP(-NGC + l) = WP(i0);
            break;
          case 3:
            for (l = 1; l <= l0; l++)
              WP(i0 - l) = WP(i0 - l + 3) - 3. * (WP(i0 - l + 2) - WP(i0 - l + 1));
            break;
          default:
            break;
        }
        switch (e->p.ibc[k][1][dir]) {
          case 0:
            for (l = 1; l <= l0; l++) WP(n + l) = WP(l);
            break;
          case 1:
            for (l = 1; l <= l0; l++) WP(n + l) = WP(n + i0 - l);
            break;
          case -1:
            for (l = 1; l <= l0; l++) WP(n + l) = -WP(n + i0 - l);
            break;
          case 2:
            for (l = 1; l <= l0; l++) WP(n + l) = WP(n);
            break;
          case 3:
            for (l = 1; l <= l0; l++)
              WP(n + l) = WP(n + l - 3) - 3. * (WP(n + l - 2) - WP(n + l - 1));
            break;
          default:
            break;
        }
#undef WP
      }
  }
}

/* ------------------------------------------------------------------------ */
/* evolve_dfx/dfy/dfz (evolve.f90:302-685) with work_rec, work_glm,         */
/* work_fup (work.f90)                                                      */
/* ------------------------------------------------------------------------ */
typedef struct Pencil {
  double *w0, *wl, *wr, *w1, *wd, *wdl, *wdr;
  int len;
} Pencil;

static void pencil_alloc(Pencil* pc, int nmax, int nv) {
  pc->len = nmax + 2 * PADP + 2;
  size_t L = (size_t)pc->len;
  pc->w0 = (double*)calloc(L * nv, sizeof(double));
  pc->wl = (double*)calloc(L * nv, sizeof(double));
  pc->wr = (double*)calloc(L * nv, sizeof(double));
  pc->w1 = (double*)calloc(L * (nv + 2), sizeof(double));
  pc->wd = (double*)calloc(L * 4, sizeof(double));
  pc->wdl = (double*)calloc(L * 4, sizeof(double));
  pc->wdr = (double*)calloc(L * 4, sizeof(double));
}
static void pencil_free(Pencil* pc) {
  free(pc->w0); free(pc->wl); free(pc->wr); free(pc->w1);
  free(pc->wd); free(pc->wdl); free(pc->wdr);
}
#define PIX(pc, k, i) ((size_t)(k) * (pc)->len + (size_t)((i) + PADP))

/* one pencil: returns the work_fup error code, writes aflux_last */
static int do_pencil(Orc* e, Pencil* pc, int dir, int a, int b, int iteration,
                     double* aflux_last) {
  const Phys* ph = &e->ph;
  const EchoParams* p = &e->p;
  int n = dir == 0 ? e->nx : dir == 1 ? e->ny : e->nz;
  int nv = e->nv;
  double dd = dir == 0 ? e->ddx : dir == 1 ? e->ddy : e->ddz;
  double g1 = ph->g1, g2 = ph->g2, g3 = ph->g3;
  int i, k;
#define WG(k, i)                                                        \
  e->w[dir == 0 ? WIDX(e, k, (i), a, b)                                 \
                : dir == 1 ? WIDX(e, k, a, (i), b) : WIDX(e, k, a, b, (i))]
#define CELL(i) (dir == 0 ? IDX(e, 0, (i), a, b) : dir == 1 ? IDX(e, 0, a, (i), b) : IDX(e, 0, a, b, (i)))
  for (k = 0; k < nv; k++)
    for (i = 1 - NGC; i <= n + NGC; i++) pc->w0[PIX(pc, k, i)] = WG(k, i);
  if (p->viscosity) {
    for (i = 1 - NGC; i <= n + NGC; i++) {
      double vx = WG(KVX, i), vy = WG(KVY, i), vz = WG(KVZ, i);
      double g = 1. / sqrt(1. - vx * vx - vy * vy - g3 * (vz * vz));
      pc->wd[PIX(pc, 0, i)] = g;
      pc->wd[PIX(pc, 1, i)] = g * vx;
      pc->wd[PIX(pc, 2, i)] = g * vy;
      pc->wd[PIX(pc, 3, i)] = g * vz;
    }
  }
  /* work_rec(n,1,nv,0) and work_rec(n,1,4,1) */
  for (k = 0; k < nv; k++)
    rec_pencil(p->recal, pc->w0 + PIX(pc, k, 0), pc->wl + PIX(pc, k, 0),
               pc->wr + PIX(pc, k, 0), n);
  if (p->viscosity)
    for (k = 0; k < 4; k++)
      rec_pencil(p->recal, pc->wd + PIX(pc, k, 0), pc->wdl + PIX(pc, k, 0),
                 pc->wdr + PIX(pc, k, 0), n);
  /* fix-ups of evolve.f90:334-369 */
  for (i = 0; i <= n; i++) {
    double v2;
    if (pc->wr[PIX(pc, KPR, i)] <= 0) pc->wr[PIX(pc, KPR, i)] = pc->w0[PIX(pc, KPR, i)];
    v2 = 0;
    v2 = v2 + pc->wr[PIX(pc, KVX, i)] * pc->wr[PIX(pc, KVX, i)] * g1;
    v2 = v2 + pc->wr[PIX(pc, KVY, i)] * pc->wr[PIX(pc, KVY, i)] * g2;
    v2 = v2 + pc->wr[PIX(pc, KVZ, i)] * pc->wr[PIX(pc, KVZ, i)] * g3;
    if (v2 >= 1.) {
      for (k = KVX; k <= KVZ; k++) pc->wr[PIX(pc, k, i)] = pc->w0[PIX(pc, k, i)];
      v2 = 0;
      v2 = v2 + pc->wr[PIX(pc, KVX, i)] * pc->wr[PIX(pc, KVX, i)] * g1;
      v2 = v2 + pc->wr[PIX(pc, KVY, i)] * pc->wr[PIX(pc, KVY, i)] * g2;
      v2 = v2 + pc->wr[PIX(pc, KVZ, i)] * pc->wr[PIX(pc, KVZ, i)] * g3;
      if (v2 >= 1) {
        for (k = KVX; k <= KVZ; k++) {
          pc->w0[PIX(pc, k, i)] = pc->w0[PIX(pc, k, i)] * p->maxspeed / (sqrt(v2));
          pc->wr[PIX(pc, k, i)] = pc->w0[PIX(pc, k, i)];
        }
      }
    }
    if (pc->wl[PIX(pc, KPR, i)] <= 0) pc->wl[PIX(pc, KPR, i)] = pc->w0[PIX(pc, KPR, i)];
    v2 = 0;
    v2 = v2 + pc->wl[PIX(pc, KVX, i)] * pc->wl[PIX(pc, KVX, i)] * g1;
    v2 = v2 + pc->wl[PIX(pc, KVY, i)] * pc->wl[PIX(pc, KVY, i)] * g2;
    v2 = v2 + pc->wl[PIX(pc, KVZ, i)] * pc->wl[PIX(pc, KVZ, i)] * g3;
    if (v2 >= 1.) {
      for (k = KVX; k <= KVZ; k++) pc->wl[PIX(pc, k, i)] = pc->w0[PIX(pc, k, i)];
      v2 = 0;
      v2 = v2 + pc->wl[PIX(pc, KVX, i)] * pc->wl[PIX(pc, KVX, i)] * g1;
      v2 = v2 + pc->wl[PIX(pc, KVY, i)] * pc->wl[PIX(pc, KVY, i)] * g2;
      v2 = v2 + pc->wl[PIX(pc, KVZ, i)] * pc->wl[PIX(pc, KVZ, i)] * g3;
      if (v2 >= 1) {
        for (k = KVX; k <= KVZ; k++) {
          pc->w0[PIX(pc, k, i)] = pc->w0[PIX(pc, k, i)] * p->maxspeed / (sqrt(v2));
          pc->wl[PIX(pc, k, i)] = pc->w0[PIX(pc, k, i)];
        }
      }
    }
  }
  /* derivatives of u^mu (evolve.f90:371-374) */
  if (p->viscosity) {
    int dt_ = dir == 0 ? DTX : dir == 1 ? DTY : DTZ;
    int dxk = dir == 0 ? DXX : dir == 1 ? DXY : DXZ;
    int dyk = dir == 0 ? DYX : dir == 1 ? DYY : DYZ;
    int dzk = dir == 0 ? DZX : dir == 1 ? DZY : DZZ;
    int dk[4] = {dt_, dxk, dyk, dzk};
    for (int c = 0; c < 4; c++)
      for (i = 1; i <= n; i++)
        e->deriv[(size_t)dk[c] * e->ncell + CELL(i)] =
            dd * 0.5 * (pc->wdl[PIX(pc, c, i)] + pc->wdr[PIX(pc, c, i)] - pc->wdl[PIX(pc, c, i - 1)] - pc->wdr[PIX(pc, c, i - 1)]);
  }
  /* work_glm[xyz] (work.f90:67-139) */
  if (p->divclean) {
    int kb = dir == 0 ? ph->kbx : dir == 1 ? ph->kby : ph->kbz, kg = ph->kglm;
    double ch = e->glm_ch;
    for (i = 0; i <= n; i++) {
      pc->wl[PIX(pc, kg, i)] = 0.5 * (pc->wl[PIX(pc, kg, i)] + pc->wr[PIX(pc, kg, i)]) -
                               (pc->wr[PIX(pc, kb, i)] - pc->wl[PIX(pc, kb, i)]) * ch / 2;
      pc->wr[PIX(pc, kg, i)] = pc->wl[PIX(pc, kg, i)];
      pc->wl[PIX(pc, kb, i)] = 0.5 * (pc->wl[PIX(pc, kb, i)] + pc->wr[PIX(pc, kb, i)]) -
                               (pc->wr[PIX(pc, kg, i)] - pc->wl[PIX(pc, kg, i)]) / (2 * ch);
      pc->wr[PIX(pc, kb, i)] = pc->wl[PIX(pc, kb, i)];
    }
  }
  /* work_fup[xyz], HLL (work.f90:195-229) */
  int errc = 0;
  for (i = 0; i <= n; i++) {
    double vl[ECHO_MAX_NV], vr[ECHO_MAX_NV], ul[ECHO_MAX_NV], ur[ECHO_MAX_NV],
        fl[ECHO_MAX_NV], fr[ECHO_MAX_NV], vfl[2], vfr[2];
    for (k = 0; k < nv; k++) {
      vl[k] = pc->wl[PIX(pc, k, i)];
      vr[k] = pc->wr[PIX(pc, k, i)];
    }
    errc = system_flux(ph, vl, ul, fl, vfl, dir + 1);
    if (errc) break;
    errc = system_flux(ph, vr, ur, fr, vfr, dir + 1);
    if (errc) break;
    double ap = 0., am = 0.;
    if (vfl[0] > ap) ap = vfl[0];
    if (vfr[0] > ap) ap = vfr[0];
    if (-vfl[1] > am) am = -vfl[1];
    if (-vfr[1] > am) am = -vfr[1];
    *aflux_last = ap > am ? ap : am;
    double a1 = (ap == 0.0 && am == 0.0) ? 1. : 1. / (ap + am);
    for (k = 0; k < nv; k++)
      pc->w1[PIX(pc, k, i)] = a1 * (ap * fl[k] + am * fr[k] - ap * am * (ur[k] - ul[k]));
    pc->w1[PIX(pc, nv, i)] = ap;
    pc->w1[PIX(pc, nv + 1, i)] = am;
  }
  /* du += dd*(w1(i)-w1(i-1)) (evolve.f90:382-384) and ax/ay/az */
  double* du = e->du[iteration - 1];
  for (k = 0; k < e->nu; k++)
    for (i = 1; i <= n; i++) {
      size_t c = CELL(i) + (size_t)k * e->ncell;
      du[c] = du[c] + dd * (pc->w1[PIX(pc, k, i)] - pc->w1[PIX(pc, k, i - 1)]);
    }
  for (i = 0; i <= n; i++)
    for (int s = 0; s < 2; s++) {
      double a_ = pc->w1[PIX(pc, nv + s, i)];
      if (dir == 0)
        e->ax[(((size_t)s * e->nz + (b - 1)) * e->ny + (a - 1)) * (e->nx + 1) + i] = a_;
      else if (dir == 1)
        e->ay[(((size_t)s * e->nz + (b - 1)) * (e->ny + 1) + i) * e->nx + (a - 1)] = a_;
      else
        e->az[(((size_t)s * (e->nz + 1) + i) * e->ny + (b - 1)) * e->nx + (a - 1)] = a_;
    }
#undef WG
#undef CELL
  return errc;
}

static int evolve_df(Orc* e, int dir, int iteration) {
  int n = dir == 0 ? e->nx : dir == 1 ? e->ny : e->nz;
  if (n <= 1) return 0;
  int nv = e->nv;
  /* w(interior) = v */
  for (int k = 0; k < nv; k++)
    for (int iz = 1; iz <= e->nz; iz++)
      for (int iy = 1; iy <= e->ny; iy++)
        for (int ix = 1; ix <= e->nx; ix++)
          e->w[WIDX(e, k, ix, iy, iz)] = e->v[IDX(e, k, ix, iy, iz)];
  evolve_bc(e, dir);
  int na = dir == 0 ? e->ny : e->nx;
  int nb = dir == 2 ? e->ny : e->nz;
  int nmax = e->nx > e->ny ? e->nx : e->ny;
  if (e->nz > nmax) nmax = e->nz;
  int err = 0;
  double af_last = e->aflux[dir];
  int nth = e->nthreads;
#ifdef _OPENMP
#pragma omp parallel num_threads(nth)
#endif
  {
    Pencil pc;
    pencil_alloc(&pc, nmax, nv);
#ifdef _OPENMP
#pragma omp for schedule(static) collapse(2)
#endif
    for (int b = 1; b <= nb; b++)
      for (int a = 1; a <= na; a++) {
        double af = 0;
        int ec = do_pencil(e, &pc, dir, a, b, iteration, &af);
        if (a == na && b == nb) {
          af_last = af;
          err = ec;
        } else if (ec) {
#ifdef _OPENMP
#pragma omp critical
#endif
          { if (!e->run_crashed) e->run_crashed = ec; }
        }
      }
    pencil_free(&pc);
  }
  (void)nth;
  e->aflux[dir] = af_last;
  if (err) {
    e->errcode = err;
    e->run_crashed = 1;
  } else if (e->run_crashed) {
    /* system_flux sets run_crashed itself on any face (system.f90:1346,1355) */
    e->errcode = e->run_crashed;
    e->run_crashed = 1;
  }
  return e->run_crashed ? e->errcode : 0;
}

/* dts (viscous.f90:56-97) */
static void evolve_dts(Orc* e) {
  size_t nc = e->ncell;
  if (e->timeinterval == 0) {
    for (int d = DTT; d <= DZT; d++)
      for (size_t c = 0; c < nc; c++) e->deriv[(size_t)d * nc + c] = 0.;
    return;
  }
  double g1 = e->ph.g1, g2 = e->ph.g2, g3 = e->ph.g3, ti = e->timeinterval;
  for (size_t c = 0; c < nc; c++) {
    double vxo = e->vold[1 * nc + c], vyo = e->vold[2 * nc + c], vzo = e->vold[3 * nc + c];
    double vx = e->vnewstep[1 * nc + c], vy = e->vnewstep[2 * nc + c], vz = e->vnewstep[3 * nc + c];
    double gamma1 = 1. / sqrt(1. - g1 * (vxo * vxo) - g2 * (vyo * vyo) - e->g3old * (vzo * vzo));
    double gamma2 = 1. / sqrt(1. - g1 * (vx * vx) - g2 * (vy * vy) - g3 * (vz * vz));
    e->deriv[(size_t)DTT * nc + c] = (gamma2 - gamma1) / (ti);
    e->deriv[(size_t)DXT * nc + c] = (gamma2 * vx - gamma1 * vxo) / ti;
    e->deriv[(size_t)DYT * nc + c] = (gamma2 * vy - gamma1 * vyo) / ti;
    e->deriv[(size_t)DZT * nc + c] = (gamma2 * vz - gamma1 * vzo) / ti;
  }
}

/* charge density rho_C = d_i E^i by central differences of the ghosted
   primitives w (system_compute_divE, system.f90:1901-1919); directions of
   one cell contribute nothing */
static double div_e(const Orc* e, int ix, int iy, int iz) {
  const Phys* ph = &e->ph;
  double r = 0.;
  if (e->nx > 1) {
    double dx = 2. / e->ddx;
    r = r + (e->w[WIDX(e, ph->kex, ix + 1, iy, iz)] - e->w[WIDX(e, ph->kex, ix - 1, iy, iz)]) / dx;
  }
  if (e->ny > 1) {
    double dy = 2. / e->ddy;
    r = r + (e->w[WIDX(e, ph->key, ix, iy + 1, iz)] - e->w[WIDX(e, ph->key, ix, iy - 1, iz)]) / dy;
  }
  if (e->nz > 1) {
    double dz = 2. / e->ddz;
    r = r + (e->w[WIDX(e, ph->kez, ix, iy, iz + 1)] - e->w[WIDX(e, ph->kez, ix, iy, iz - 1)]) / dz;
  }
  return r;
}

/* evolve_src (evolve.f90:689-718): du -= src, du_stiff -= src_stiff */
static int evolve_src(Orc* e, int iteration) {
  size_t nc = e->ncell;
  int nv = e->nv;
  if (e->p.viscosity) evolve_dts(e);
  int err = 0;
  double* du = e->du[iteration - 1];
  double* dus = e->dus[iteration - 1];
  for (size_t c = 0; c < nc && !err; c++) {
    double vv[ECHO_MAX_NV], src[ECHO_MAX_NV], stiff[ECHO_MAX_NV], dv[NDERIV];
    for (int k = 0; k < nv; k++) vv[k] = e->v[(size_t)k * nc + c];
    if (e->p.viscosity)
      for (int d = 0; d < NDERIV; d++) dv[d] = e->deriv[(size_t)d * nc + c];
    double rhoC = 0.;
    if (e->p.mhd == 2) {
      int ix = (int)(c % (size_t)e->nx) + 1, iy = (int)((c / (size_t)e->nx) % (size_t)e->ny) + 1;
      int iz = (int)(c / ((size_t)e->nx * e->ny)) + 1;
      rhoC = div_e(e, ix, iy, iz);
    }
    double* kap = e->kap ? e->kap + 2 * c : NULL;
    int ec = system_source(&e->ph, vv, dv, rhoC, src, stiff, kap);
    if (ec) {
      err = ec;
      break;
    }
    for (int k = 0; k < e->nu; k++) du[(size_t)k * nc + c] = du[(size_t)k * nc + c] - src[k];
    if (dus)
      for (int k = 0; k < e->nu; k++) dus[(size_t)k * nc + c] = dus[(size_t)k * nc + c] - stiff[k];
  }
  if (err) {
    e->errcode = err;
    e->run_crashed = 1;
  }
  return err;
}

/* evolve_dt (evolve.f90:723-764) */
static double evolve_dt(Orc* e) {
  double amax;
  if (e->p.divclean) {
    amax = 1;
  } else {
    amax = 0.;
    int nx = e->nx, ny = e->ny, nz = e->nz;
    for (int iz = 1; iz <= nz; iz++)
      for (int iy = 1; iy <= ny; iy++)
        for (int ix = 1; ix <= nx; ix++) {
          double m, c;
          if (nx > 1) {
            m = -INFINITY;
            for (int s = 0; s < 2; s++)
              for (int i = ix - 1; i <= ix; i++) {
                c = e->ax[(((size_t)s * nz + (iz - 1)) * ny + (iy - 1)) * (nx + 1) + i];
                if (c > m) m = c;
              }
            c = e->ddx * m;
            if (c > amax) amax = c;
          }
          if (ny > 1) {
            m = -INFINITY;
            for (int s = 0; s < 2; s++)
              for (int i = iy - 1; i <= iy; i++) {
                c = e->ay[(((size_t)s * nz + (iz - 1)) * (ny + 1) + i) * nx + (ix - 1)];
                if (c > m) m = c;
              }
            c = e->ddy * m;
            if (c > amax) amax = c;
          }
          if (nz > 1) {
            m = -INFINITY;
            for (int s = 0; s < 2; s++)
              for (int i = iz - 1; i <= iz; i++) {
                c = e->az[(((size_t)s * (nz + 1) + i) * ny + (iy - 1)) * nx + (ix - 1)];
                if (c > m) m = c;
              }
            c = e->ddz * m;
            if (c > amax) amax = c;
          }
        }
    if (amax == 0) {
      if (nx > 1 && e->ddx > amax) amax = e->ddx;
      if (ny > 1 && e->ddy > amax) amax = e->ddy;
      if (nz > 1 && e->ddz > amax) amax = e->ddz;
    }
  }
  return e->p.cfl / amax;
}

/* evolve_u2v (evolve.f90:769-868) with the repair path of :795-842 */
static double flat_get(const double* a, size_t total, long long off) {
  if (off < 0 || (size_t)off >= total) return 0.;
  return a[off];
}

static int evolve_u2v(Orc* e) {
  const Phys* ph = &e->ph;
  size_t nc = e->ncell;
  int nv = e->nv, nu = e->nu;
  int nx = e->nx, ny = e->ny, nz = e->nz;
  long long c2p = 0;
  /* pass 1: every cell independently (vtmp = new v, fail = flag); the
   * Fortran loop gives the same result because a cell's inversion reads
   * only its own u and its own old v */
  memset(e->fail, 0, nc);
  int nth = e->nthreads;
  (void)nth;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nth) schedule(static) reduction(+ : c2p)
#endif
  for (long long c = 0; c < (long long)nc; c++) {
    double uu[ECHO_MAX_NV], vv[ECHO_MAX_NV];
    for (int k = 0; k < nv; k++) vv[k] = e->v[(size_t)k * nc + c];
    for (int k = 0; k < nu; k++) uu[k] = e->u[(size_t)k * nc + c];
    int it = 0;
    int err = cons2prim(ph, uu, vv, &it);
    c2p += it;
    if (err) {
      e->fail[c] = 1;
    } else {
      for (int k = 0; k < nv; k++) e->vtmp[(size_t)k * nc + c] = vv[k];
      /* the implicit Ohm solve of a resistive stage sets E in u */
      if (ph->p->mhd == 2 && ph->ohm_h > 0.)
        for (int k = ph->kex; k <= ph->kez; k++) e->u[(size_t)k * nc + c] = uu[k];
    }
  }
  e->c2p_iters = c2p;
  /* pass 2: the failing cells in Fortran loop order; neighbours earlier in
   * the loop already hold their new v, later ones still the old v */
  for (int iz = 1; iz <= nz; iz++)
    for (int iy = 1; iy <= ny; iy++)
      for (int ix = 1; ix <= nx; ix++) {
        size_t c = IDX(e, 0, ix, iy, iz);
        if (!e->fail[c]) {
          for (int k = 0; k < nv; k++) e->v[(size_t)k * nc + c] = e->vtmp[(size_t)k * nc + c];
          continue;
        }
        double uu[ECHO_MAX_NV], vv[ECHO_MAX_NV], g3 = ph->g3;
        int it;
        e->repairs++;
        for (int k = 0; k < nv; k++) vv[k] = e->v[(size_t)k * nc + c];
        for (int k = 0; k < nu; k++) uu[k] = e->u[(size_t)k * nc + c];
        (void)cons2prim(ph, uu, vv, &it); /* the failed call, for its side effects on vv */
        size_t totu = nc * nu, totv = nc * nv;
        for (int k = 0; k < nu; k++) {
          long long base = (long long)k * nc;
          long long o = (long long)(ix - 1) + (long long)nx * ((iy - 1) + (long long)ny * (iz - 1));
          double s = flat_get(e->u, totu, base + o - 1) + flat_get(e->u, totu, base + o + 1) +
                     flat_get(e->u, totu, base + o - nx) + flat_get(e->u, totu, base + o + nx) +
                     flat_get(e->u, totu, base + o - (long long)nx * ny) +
                     flat_get(e->u, totu, base + o + (long long)nx * ny);
          e->u[(size_t)k * nc + c] = s / 6.;
          uu[k] = e->u[(size_t)k * nc + c];
        }
        (void)cons2prim(ph, uu, vv, &it);
        double v2 = vv[KVX] * vv[KVX] + vv[KVY] * vv[KVY] + vv[KVZ] * vv[KVZ] * g3;
        if (v2 > 1) {
          double fac = e->p.maxspeed / sqrt(v2);
          vv[KVX] = fac * vv[KVX];
          vv[KVY] = fac * vv[KVY];
          vv[KVZ] = fac * vv[KVZ];
        }
        if (vv[KPR] < 0) {
          long long base = (long long)KPR * nc;
          long long o = (long long)(ix - 1) + (long long)nx * ((iy - 1) + (long long)ny * (iz - 1));
          double pxl = flat_get(e->v, totv, base + o - 1), pxr = flat_get(e->v, totv, base + o + 1);
          double pyl = flat_get(e->v, totv, base + o - nx), pyr = flat_get(e->v, totv, base + o + nx);
          double pzl = flat_get(e->v, totv, base + o - (long long)nx * ny);
          double pzr = flat_get(e->v, totv, base + o + (long long)nx * ny);
          vv[KPR] = (pxl + pxr + pyl + pyr + pzl + pzr) / 6.;
        }
        (void)prim2cons(ph, vv, uu);
        int err = cons2prim(ph, uu, vv, &it);
        (void)err;
        v2 = vv[KVX] * vv[KVX] + vv[KVY] * vv[KVY] + vv[KVZ] * vv[KVZ] * g3;
        int ok = (vv[KPR] > 0) && (v2 < 1);
        if (e->p.viscosity && e->p.obtained_zz) e->v[(size_t)KPIZZ * nc + c] = vv[KPIZZ];
        for (int k = 0; k < nu; k++) e->u[(size_t)k * nc + c] = uu[k];
        if (!ok) {
          e->errcode = 1;
          e->run_crashed = 1;
          return 1;
        }
        for (int k = 0; k < nv; k++) e->v[(size_t)k * nc + c] = vv[k];
      }
  return 0;
}

/* evolve_smooth_viscosity (evolve.f90:1159-1207) */
static int evolve_smooth_viscosity(Orc* e) {
  const Phys* ph = &e->ph;
  size_t nc = e->ncell;
  int nv = e->nv;
  double ps = e->p.smooth_pressure;
  for (size_t c = 0; c < nc; c++) {
    double pr = e->v[(size_t)KPR * nc + c];
    if (pr < ps) {
      double vv[ECHO_MAX_NV], uu[ECHO_MAX_NV];
      for (int k = 0; k < nv; k++) vv[k] = e->v[(size_t)k * nc + c];
      double r = vv[KPR] / ps;
      double fac = r * r;
      for (int k = KPIBU; k <= KPIZZ; k++) vv[k] = vv[k] * fac;
      if (e->p.obtained_zz) {
        Pit pi;
        derived_pi_zz(ph, vv, &pi);
        vv[KPIZZ] = pi.zz;
      }
      int err = prim2cons(ph, vv, uu);
      for (int k = 0; k < nv; k++) {
        e->v[(size_t)k * nc + c] = vv[k];
        e->u[(size_t)k * nc + c] = uu[k];
      }
      if (err) {
        e->errcode = err;
        e->run_crashed = 1;
        return err;
      }
    }
  }
  return 0;
}

static void glm_source(Orc* e, double dt_glm) { /* evolve.f90:83-110 */
  double expfact = exp(-e->glm_ch * e->glm_ch * e->p.glm_alpha * dt_glm);
  size_t nc = e->ncell;
  double* ug = e->u + (size_t)e->ph.kglm * nc;
  for (size_t c = 0; c < nc; c++) ug[c] = ug[c] * expfact;
}

static int rhs_all(Orc* e, int iteration) {
  double* du = e->du[iteration - 1];
  memset(du, 0, sizeof(double) * e->ncell * e->nv);
  if (e->dus[iteration - 1]) memset(e->dus[iteration - 1], 0, sizeof(double) * e->ncell * e->nv);
  e->glm_ch = e->glm_ch_old;
  if (evolve_df(e, 0, iteration)) return e->errcode;
  if (evolve_df(e, 1, iteration)) return e->errcode;
  if (evolve_df(e, 2, iteration)) return e->errcode;
  if (evolve_src(e, iteration)) return e->errcode;
  double m = e->aflux[0];
  if (e->aflux[1] > m) m = e->aflux[1];
  if (e->aflux[2] > m) m = e->aflux[2];
  e->glm_ch_old = m;
  return 0;
}

static double dt_clip(Orc* e, double dt_local) { /* evolve.f90:181-188 */
  if (e->p.maxdt < dt_local) dt_local = e->p.maxdt;
  if (e->tout - e->t < dt_local) dt_local = e->tout - e->t;
  if (fabs(e->t + e->dt - e->tout) < 1.e-9) {
    dt_local = e->tout - e->t;
  } else {
    if ((e->t + 2. * dt_local - e->tout) > 1.e-9) dt_local = (e->tout - e->t) / 2.;
  }
  return dt_local;
}

/* Resistive IMEX-SSP3(4,3,3), first stage: U1 = u^n + alpha dt S(U1), the
   implicit solve the reference leaves to its missing algo-7 con2prim.  U1
   is solved from u0 cell by cell and dus[0] = -S(U1) replaces the stiff
   source the stage's right-hand side took at u^n (only S(U1) enters the
   later stages; the explicit F(U1) has weight 0).  v and u stay at step n. */
static int stage1_implicit(Orc* e, double h) {
  Phys* ph = &e->ph;
  size_t nc = e->ncell;
  int nv = e->nv;
  ph->ohm_h = h;
  for (size_t c = 0; c < nc; c++) {
    double uu[ECHO_MAX_NV], vv[ECHO_MAX_NV], S[3];
    for (int k = 0; k < nv; k++) {
      uu[k] = e->u0[(size_t)k * nc + c];
      vv[k] = e->v[(size_t)k * nc + c];
    }
    int it = 0, err = cons2prim(ph, uu, vv, &it);
    if (err) {
      ph->ohm_h = 0.;
      e->errcode = err;
      e->run_crashed = 1;
      return err;
    }
    double v2 = ph->g1 * vv[KVX] * vv[KVX] + ph->g2 * vv[KVY] * vv[KVY] + ph->g3 * vv[KVZ] * vv[KVZ];
    double glf = 1. / sqrt(1. - v2);
    ohm_stiff(ph, vv + KVX, vv + ph->kbx, vv + ph->kex, glf, S);
    for (int i = 0; i < 3; i++) e->dus[0][(size_t)(ph->kex + i) * nc + c] = 0. - S[i] * ph->gp;
  }
  ph->ohm_h = 0.;
  return 0;
}

/* u2v of an implicit IMEX stage: the resistive con2prim solves Ohm's law
   with h = alpha dt (the diagonal of the implicit tableau) */
static int u2v_implicit(Orc* e, double h) {
  if (e->p.mhd == 2) e->ph.ohm_h = h;
  int err = evolve_u2v(e);
  e->ph.ohm_h = 0.;
  return err;
}

/* evolve_main (evolve.f90:114-298) */
int orc_evolve_main(Orc* e, int irk, double* dt_out) {
  size_t n = e->ncell * e->nv;
  int nu = e->nu;
  (void)nu;
  if (e->p.nrk != ECHO_SSP) {
    static const double crk[3][3][2] = {
        {{0., 1.}, {0., 0.}, {0., 0.}},
        {{0., 1.}, {1. / 2., 1. / 2.}, {0., 0.}},
        {{0., 1.}, {3. / 4., 1. / 4.}, {1. / 3., 2. / 3.}}};
    double c1 = crk[e->p.nrk - 1][irk - 1][0], c2 = crk[e->p.nrk - 1][irk - 1][1];
    if (rhs_all(e, 1)) return e->errcode;
    if (irk == 1) {
      double dtl = dt_clip(e, evolve_dt(e));
      e->dt = dtl;
      if (e->p.divclean) glm_source(e, e->dt / 2.);
      memcpy(e->u0, e->u, sizeof(double) * n);
    }
    double dt = e->dt, *du = e->du[0];
    size_t nimex = e->kap ? (size_t)KPIBU * e->ncell : n;
    for (size_t i = 0; i < nimex; i++) e->u[i] = c1 * e->u0[i] + c2 * (e->u[i] - dt * du[i]);
    /* IMEX RK2/RK3 (no reference counterpart): the relaxation -kap u of the
       stresses taken at the new stage value, linearly implicit; the rest of
       du stays explicit.  u_new = u_expl + c2 dt kap (u - u_new), i.e.
       u_new = (c1 u0 + c2 (u - dt du) + c2 dt kap u) / (1 + c2 dt kap). */
    for (size_t i = nimex; i < n; i++) {
      size_t c = (i - nimex) % e->ncell;
      int k = (int)((i - nimex) / e->ncell) + KPIBU;
      double ck = c2 * dt * e->kap[2 * c + (k == KPIBU ? 0 : 1)];
      e->u[i] = (c1 * e->u0[i] + c2 * (e->u[i] - dt * du[i]) + ck * e->u[i]) / (1. + ck);
    }
    if (e->p.divclean && irk == e->p.nrk) glm_source(e, dt / 2.);
    if (evolve_u2v(e)) return e->errcode;
  } else {
    const double alpha_imex = 0.24169426078821, beta_imex = 0.06042356519705,
                 eta_imex = 0.12915286960590;
    const double delta_imex = 0.5 - beta_imex - eta_imex - alpha_imex;
    double dt;
    if (irk == 1) {
      double dtl = dt_clip(e, evolve_dt(e));
      e->dt = dtl;
      memcpy(e->u0, e->u, sizeof(double) * n);
      if (rhs_all(e, 1)) return e->errcode;
      if (e->p.divclean) glm_source(e, e->dt / 2.);
      if (e->p.mhd == 2 && stage1_implicit(e, alpha_imex * e->dt)) return e->errcode;
    } else if (irk == 2) {
      dt = e->dt;
      for (size_t i = 0; i < n; i++) e->u[i] = e->u0[i] + dt * alpha_imex * e->dus[0][i];
      if (u2v_implicit(e, alpha_imex * dt)) return e->errcode;
      if (rhs_all(e, 2)) return e->errcode;
    } else if (irk == 3) {
      dt = e->dt;
      for (size_t i = 0; i < n; i++)
        e->u[i] = e->u0[i] - dt * (e->du[1][i] + (1. - alpha_imex) * e->dus[1][i]);
      if (u2v_implicit(e, alpha_imex * dt)) return e->errcode;
      if (rhs_all(e, 3)) return e->errcode;
    } else {
      dt = e->dt;
      for (size_t i = 0; i < n; i++)
        e->u[i] = e->u0[i] - dt * (e->du[1][i] / 4. + e->du[2][i] / 4. + beta_imex * e->dus[0][i] +
                                   eta_imex * e->dus[1][i] + delta_imex * e->dus[2][i]);
      if (u2v_implicit(e, alpha_imex * dt)) return e->errcode;
      if (rhs_all(e, 4)) return e->errcode;
      for (size_t i = 0; i < n; i++)
        e->u[i] = e->u0[i] - dt * (e->du[1][i] / 6. + e->du[2][i] / 6. + e->du[3][i] * 2. / 3. +
                                   e->dus[1][i] / 6. + e->dus[2][i] / 6. + e->dus[3][i] * 2. / 3.);
      if (e->p.divclean) glm_source(e, dt / 2.);
      if (evolve_u2v(e)) return e->errcode;
    }
  }
  if (e->p.viscosity && e->p.enable_smooth_viscosity)
    if (evolve_smooth_viscosity(e)) return e->errcode;
  if (dt_out) *dt_out = e->dt;
  return 0;
}

/* echo.f90:185-262 without output */
int orc_step(Orc* e, double* dt_out) {
  size_t nc = e->ncell;
  memcpy(e->vnewstep, e->v, sizeof(double) * nc * e->nvold);
  int nstage = e->p.nrk == ECHO_SSP ? 4 : e->p.nrk;
  for (int irk = 1; irk <= nstage; irk++) {
    int err = orc_evolve_main(e, irk, NULL);
    if (err) return err;
  }
  e->timeold = e->t;
  e->t = e->t + e->dt;
  e->g3old = e->ph.g3;
  phys_metric(&e->ph, e->t);
  e->timeinterval = e->dt;
  memcpy(e->vold, e->vnewstep, sizeof(double) * nc * e->nvold);
  if ((e->t > e->tout) || ((e->tout - e->t) < 1.e-10)) {
    e->tout = e->tout + e->dtout;
    if ((fabs(e->tout - e->tmax) < 1.e-10) || (e->tout > e->tmax)) e->tout = e->tmax;
  }
  if (dt_out) *dt_out = e->dt;
  return 0;
}

int orc_rhs(Orc* e, double* du, double* amax3) {
  int err = rhs_all(e, 1);
  if (du) memcpy(du, e->du[0], sizeof(double) * e->ncell * e->nv);
  if (amax3) {
    int nx = e->nx, ny = e->ny, nz = e->nz;
    double m[3] = {0, 0, 0};
    size_t na = (size_t)2 * (nx + 1) * ny * nz, nb = (size_t)2 * nx * (ny + 1) * nz,
           nn = (size_t)2 * nx * ny * (nz + 1);
    for (size_t i = 0; i < na; i++) if (e->ax[i] > m[0]) m[0] = e->ax[i];
    for (size_t i = 0; i < nb; i++) if (e->ay[i] > m[1]) m[1] = e->ay[i];
    for (size_t i = 0; i < nn; i++) if (e->az[i] > m[2]) m[2] = e->az[i];
    amax3[0] = m[0]; amax3[1] = m[1]; amax3[2] = m[2];
  }
  return err;
}

/* ------------------------------------------------------------------------ */
/* pointwise entry points for unit tests                                    */
/* ------------------------------------------------------------------------ */
static void unit_phys(Phys* ph, const EchoParams* p, double g3, double gp,
                      const double* tab, int n, double** bufs) {
  phys_setup(ph, p);
  ph->g1 = 1.;
  ph->g2 = 1.;
  ph->g3 = g3;
  ph->gp = gp;
  ph->gm = 1. / gp;
  ph->t = gp;
  int nt;
  table_attach(ph, &bufs[0], &bufs[1], &bufs[2], &bufs[3], &nt, tab, n);
}

int orc_c2p(const EchoParams* p, const double* tab, int n_eos, int ncells,
            double g3, double gp, const double* u, double* v, int* err,
            int* iters) {
  Phys ph;
  double* bufs[4] = {0, 0, 0, 0};
  unit_phys(&ph, p, g3, gp, tab, n_eos, bufs);
  int nv = ph.nv;
  for (int c = 0; c < ncells; c++) {
    double uu[ECHO_MAX_NV];
    for (int k = 0; k < nv; k++) uu[k] = u[(size_t)c * nv + k];
    int it = 0;
    int e = cons2prim(&ph, uu, v + (size_t)c * nv, &it);
    if (err) err[c] = e;
    if (iters) iters[c] = it;
  }
  for (int i = 0; i < 4; i++) free(bufs[i]);
  return nv;
}

int orc_prim2cons(const EchoParams* p, const double* tab, int n_eos,
                  int ncells, double g3, double gp, double* v, double* u) {
  Phys ph;
  double* bufs[4] = {0, 0, 0, 0};
  unit_phys(&ph, p, g3, gp, tab, n_eos, bufs);
  int nv = ph.nv, bad = 0;
  for (int c = 0; c < ncells; c++)
    if (prim2cons(&ph, v + (size_t)c * nv, u + (size_t)c * nv)) bad++;
  for (int i = 0; i < 4; i++) free(bufs[i]);
  return bad;
}

int orc_flux(const EchoParams* p, const double* tab, int n_eos, double g3,
             double gp, int dir, double* v, double* u, double* f, double* vf) {
  Phys ph;
  double* bufs[4] = {0, 0, 0, 0};
  unit_phys(&ph, p, g3, gp, tab, n_eos, bufs);
  int r = system_flux(&ph, v, u, f, vf, dir);
  for (int i = 0; i < 4; i++) free(bufs[i]);
  return r;
}

/* ------------------------------------------------------------------------ */
/* The learned con2prim seed network in FP64, for the gradient check of the */
/* GPU training kernels: mean-squared loss over n standardised rows and its */
/* gradient w.r.t. the weight vector (layout of ECHO_MLP_NWEIGHTS).         */
/* ------------------------------------------------------------------------ */
void orc_mlp_grad(const float* W, const float* Xs, const float* Ts, int n, double* loss, double* grad) {
  static const int LK[5] = {6, 64, 64, 64, 64}, LN[5] = {64, 64, 64, 64, 2};
  static const int WO[5] = {0, 448, 4608, 8768, 12928}, BO[5] = {384, 4544, 8704, 12864, 13056};
  const int NW = 13058;
  double* g = grad;
  for (int i = 0; i < NW; i++) g[i] = 0.;
  double L = 0.;
  double act[6][64], dz[5][64];
  for (int r = 0; r < n; r++) {
    for (int j = 0; j < 6; j++) act[0][j] = Xs[r * 6 + j];
    for (int l = 0; l < 5; l++)
      for (int o = 0; o < LN[l]; o++) {
        double z = W[BO[l] + o];
        for (int k = 0; k < LK[l]; k++) z += act[l][k] * (double)W[WO[l] + k * LN[l] + o];
        act[l + 1][o] = l < 4 ? tanh(z) : z;
      }
    for (int o = 0; o < 2; o++) {
      double d = act[5][o] - Ts[r * 2 + o];
      L += d * d / (2.0 * n);
      dz[4][o] = 2.0 * d / (2.0 * n);
    }
    for (int l = 4; l >= 0; l--) {
      for (int k = 0; k < LK[l]; k++)
        for (int o = 0; o < LN[l]; o++) g[WO[l] + k * LN[l] + o] += act[l][k] * dz[l][o];
      for (int o = 0; o < LN[l]; o++) g[BO[l] + o] += dz[l][o];
      if (l > 0)
        for (int k = 0; k < LK[l]; k++) {
          double s = 0.;
          for (int o = 0; o < LN[l]; o++) s += dz[l][o] * (double)W[WO[l] + k * LN[l] + o];
          dz[l - 1][k] = s * (1. - act[l][k] * act[l][k]);
        }
    }
  }
  *loss = L;
}

/* FP64 forward pass on raw invariants with normalisation (seed accuracy) */
void orc_mlp_forward(const float* W, const float* norm, const float* X, int n, double* out) {
  static const int LK[5] = {6, 64, 64, 64, 64}, LN[5] = {64, 64, 64, 64, 2};
  static const int WO[5] = {0, 448, 4608, 8768, 12928}, BO[5] = {384, 4544, 8704, 12864, 13056};
  double act[6][64];
  for (int r = 0; r < n; r++) {
    for (int j = 0; j < 6; j++) act[0][j] = ((double)X[r * 6 + j] - norm[j]) / norm[6 + j];
    for (int l = 0; l < 5; l++)
      for (int o = 0; o < LN[l]; o++) {
        double z = W[BO[l] + o];
        for (int k = 0; k < LK[l]; k++) z += act[l][k] * (double)W[WO[l] + k * LN[l] + o];
        act[l + 1][o] = l < 4 ? tanh(z) : z;
      }
    for (int o = 0; o < 2; o++) out[r * 2 + o] = act[5][o] * norm[14 + o] + norm[12 + o];
  }
}

/* ------------------------------------------------------------------------ */
/* tabulated EoS at one point: get_energy (eos.f90:468-523)                  */
/* ------------------------------------------------------------------------ */
int orc_eos_energy(const EchoParams* p, const double* tab, int n_eos, double pr, double* en) {
  Phys ph;
  double* bufs[4] = {0, 0, 0, 0};
  unit_phys(&ph, p, 1., 1., tab, n_eos, bufs);
  int e = eos_energy(&ph, 0., en, pr);
  for (int i = 0; i < 4; i++) free(bufs[i]);
  return e;
}

/* ------------------------------------------------------------------------ */
/* optical Glauber initial state (init.f90:852-1242)                        */
/* ------------------------------------------------------------------------ */

/* Fortran nint: nearest integer, halves away from zero */
static long orc_nint(double x) { return x >= 0. ? (long)floor(x + 0.5) : -(long)floor(-x + 0.5); }

/* thickness (init.f90:1164-1219): the Woods-Saxon thickness at nmax radii
 * r = (nc-1) dr, each the sum over |z| <= 2 radius of the density at
 * z1 = -zmax, -zmax + dz, ... with dz halved from 2 dz1 until the two
 * end-point sums agree to acc (at most ORC_THICK_RUNS halvings; the
 * reference has no limit); thick[nc-1] = sum1 dz.  Returns the reference's
 * "check nucleus mass", check * 2 * 3.1415927 * dr with
 * check = sum_nc r sum1 dz (init.f90:1211-1219), or -1 when a radius did not
 * converge. */
#define ORC_THICK_RUNS 8
double orc_thickness(double radius, double delta, double roze, double dr, double dz1, double acc, int nmax,
                     double* thick) {
  const double delta_inv = 1. / delta;
  const double zmax = 2. * radius;
  double check = 0.;
  int bad = 0;
  /* radii are independent: computed in parallel, summed below in the
   * reference's order */
  double* term = (double*)malloc(sizeof(double) * (size_t)nmax);
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
  for (int nc = 1; nc <= nmax; nc++) {
    double dz = 2. * dz1;
    const double r = (nc - 1) * dr;
    const double r2 = r * r;
    double ratio = 1000., sum1 = 0., sum2 = 0.;
    int nrun = 0;
    while (ratio > acc) {
      if (nrun == ORC_THICK_RUNS) {
        bad = 1;
        break;
      }
      dz = dz * 0.5;
      const long nstep = orc_nint(2. * zmax / dz);
      nrun = nrun + 1;
      double z1 = -zmax, z2 = z1 + dz;
      sum1 = 0.;
      sum2 = 0.;
      for (long n = 1; n <= nstep; n++) {
        double z = z1;
        double erre = sqrt(r2 + z * z);
        double espo = exp((erre - radius) * delta_inv);
        double rho1 = roze / (espo + 1.);
        z = z2;
        erre = sqrt(r2 + z * z);
        espo = exp((erre - radius) * delta_inv);
        double rho2 = roze / (espo + 1.);
        sum1 = sum1 + rho1;
        sum2 = sum2 + rho2;
        z1 = z2;
        z2 = z2 + dz;
      }
      ratio = fabs(2. * (sum2 - sum1) / (sum1 + sum2));
    }
    term[nc - 1] = r * sum1 * dz;
    thick[nc - 1] = sum1 * dz;
  }
  for (int nc = 1; nc <= nmax; nc++) check = check + term[nc - 1];
  free(term);
  return bad ? -1. : check * 2 * 3.1415927 * dr;
}

/* wound (init.f90:1001-1032) and bincoll (:971-997) at (xx, yy) with impact
 * parameter b1: the thickness of each nucleus by the nearest table point
 * nint(r/dr + 1) */
static void orc_wound(const double* thick, int nmax, double dr, double amassa, double sigma_in, double xx, double yy,
                      double b1, double* tA, double* tB, double* thplus, double* thminus, int* bad) {
  double xs = xx + b1 * 0.5;
  double radius = sqrt(xs * xs + yy * yy);
  long ip = orc_nint(radius / dr + 1);
  xs = xx - b1 * 0.5;
  radius = sqrt(xs * xs + yy * yy);
  long im = orc_nint(radius / dr + 1);
  if (ip < 1 || ip > nmax || im < 1 || im > nmax) {
    *bad = 1;
    ip = ip < 1 ? 1 : (ip > nmax ? nmax : ip);
    im = im < 1 ? 1 : (im > nmax ? nmax : im);
  }
  *thplus = thick[ip - 1];
  *thminus = thick[im - 1];
  double a = sigma_in * (*thminus) / amassa;
  a = pow(1. - a, amassa);
  a = 1. - a;
  *tA = a * (*thplus);
  double b = sigma_in * (*thplus) / amassa;
  b = pow(1. - b, amassa);
  b = 1. - b;
  *tB = b * (*thminus);
}

/* H_of_eta (init.f90:933-967) without tilting, centre flag */
static double orc_h_of_eta(double etac, double etaflat, double sigmaetasq_inv, double thplus, double thminus,
                           double gamma_col, double beta_col) {
  double eta0 = 0.5 * log(((thminus + thplus) * gamma_col + (thminus - thplus) * gamma_col * beta_col) /
                          ((thminus + thplus) * gamma_col - (thminus - thplus) * gamma_col * beta_col));
  double d = fabs(etac - eta0);
  if (d > (etaflat * 0.5)) {
    double q = d - (0.5 * etaflat);
    return exp(-1.0 * (q * q) * 0.5 * sigmaetasq_inv);
  }
  return 1.0;
}

/* The energy density of calc_enedens (init.f90:902-929, no tilting) at the
 * cell centres x1 + (i - 1/2) dx of an nx x ny x nz grid (Fortran order),
 * with the weights of a b = 0 collision at the origin (init.f90:1805-1812)
 * and eta from z1 + (k - 1/2) dz when nz > 1.  g: the EchoOpticalGlauber
 * parameters; the thickness table of nmax points is built first.  Returns
 * the check mass, or -1 (a radius that did not converge or a cell beyond
 * the table). */
double orc_optical_glauber(const EchoOpticalGlauber* g, int nx, int ny, int nz, double x1, double x2, double y1,
                           double y2, double z1, double z2, double* e) {
  const double dx = (x2 - x1) / nx, dy = (y2 - y1) / ny, dzz = (z2 - z1) / nz;
  const double largestx = fmax(fabs(x1), fabs(x2)) + g->bimpact;
  const double largesty = fmax(fabs(y1), fabs(y2));
  const double rmax = sqrt(largestx * largestx + largesty * largesty);
  const int nmax = (int)(rmax / g->dr) + 1;
  double* thick = (double*)malloc(sizeof(double) * nmax);
  double check = orc_thickness(g->radius, g->delta, g->roze, g->dr, g->dz1, g->acc, nmax, thick);
  int bad = check < 0.;
  double tt1, tt2, thp, thm;
  orc_wound(thick, nmax, g->dr, g->mass_number, g->sigma_in, 0., 0., 0., &tt1, &tt2, &thp, &thm, &bad);
  const double weightbin = g->sigma_in * thp * thm;
  const double weightwound = tt1 + tt2;
  const double ah = g->ah;
  const double gamma_col = g->sqrt_s / (2. * g->nucleon_mass);
  const double beta_col = sqrt(1. - (1. / (gamma_col * gamma_col)));
  const double sigeta2_inv = 1. / (g->sigeta * g->sigeta);
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const double xx = x1 + (i + 1 - 0.5) * dx, yy = y1 + (j + 1 - 0.5) * dy;
        orc_wound(thick, nmax, g->dr, g->mass_number, g->sigma_in, xx, yy, g->bimpact, &tt1, &tt2, &thp, &thm, &bad);
        const double bc = g->sigma_in * thp * thm;
        double ed = g->ecenter * (ah * bc + (1. - ah) * (tt1 + tt2)) / ((ah * weightbin) + ((1 - ah) * weightwound));
        if (nz > 1) {
          const double eta = z1 + (k + 1 - 0.5) * dzz;
          ed = orc_h_of_eta(eta, g->deta, sigeta2_inv, thp, thm, gamma_col, beta_col) * ed;
        }
        e[((size_t)k * ny + j) * nx + i] = ed;
      }
  free(thick);
  return bad ? -1. : check;
}
