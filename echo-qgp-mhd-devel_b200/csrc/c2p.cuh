// c2p.cuh -- conserved -> primitive inversion on the device
// (system_cons2prim, system.f90:423-1166) and the per-cell source terms
// (system_source, system.f90:1587-1842; get_sigma, viscous.f90:283-393).
#pragma once

#include "mlp.cuh"
#include "physics.cuh"

namespace echo {

// ---------------------------------------------------------------------------
// BRENTM (libacm554.f90:8-362) on the 3x3 system sist3 (system.f90:1199-1231)
// ---------------------------------------------------------------------------
struct Sist3 {
  double B2, SB2, S2, U, D;
  double iUB;  // 1 / (|U| + B2), the scale of the second residual
};

__device__ __forceinline__ double sist3_f(const DevPhys& P, const Sist3& s, const double* X, int K) {
  double xx = X[0], yy = X[1], pp = X[2];
  if (K == 1) return (yy + s.B2) * (yy + s.B2) * xx - s.SB2 / (yy * yy) * (2 * yy + s.B2) - s.S2;
  if (K == 2) return yy - pp + 0.5 * (1. + xx) * s.B2 - 0.5 * s.SB2 / (yy * yy) - s.U;
  double rh = s.D * sqrt(1 - xx), en = 0;
  (void)eos_energy(P, rh, &en, pp);  // errcode ignored (system.f90:1227)
  return yy - (pp + en) / (1 - xx);
}

__device__ __forceinline__ double dmax1(double a, double b) { return b > a ? b : a; }

// BRENTM on N unknowns; sys.f(X, K) is the K-th equation (sist3, sist4).
// Returns INFO; X in/out; *nfev = NFEV.  MAXFEV bounds the iteration count.
template <int N, class Sys>
static __device__ int brentm(Sys& sys, double* X, double FTOL, double XTOL, int MAXFEV, int MOPT, int* nfev_out) {
  double Q[N * N], SIGMA[N], WA1[N], WA2[N];
#define QQ(i, j) Q[((j)-1) * N + ((i)-1)]
  int NFCALL = 0, NIER6 = -1, NIER7 = -1, NIER8 = 0, NSING, INFO = 0, NFEV = 0;
  bool CONV;
  double DELTA, DIFIT = 0., DIFIT1, EPS, FKY, FKZ, FNORM = 0., FNORM1, H, SKNORM, TEMP, XNORM = 0., ETA;
  const double ZERO = 0.0, P05 = 5.0e-2, SCALE = 1.0e1;
  const double EPSMCH = 2.220446049250313080847e-16;
  for (int I = 1; I <= N; I++) XNORM = dmax1(XNORM, fabs(X[I - 1]));
  EPS = sqrt(EPSMCH);
  DELTA = SCALE * XNORM;
  if (XNORM == ZERO) DELTA = SCALE;
  for (;;) {
    NSING = N;
    FNORM1 = FNORM;
    DIFIT1 = DIFIT;
    FNORM = ZERO;
    H = EPS * XNORM;
    if (H == ZERO) H = EPS;
#pragma unroll
    for (int J = 1; J <= N; J++) {
#pragma unroll
      for (int I = 1; I <= N; I++) QQ(I, J) = ZERO;
      QQ(J, J) = H;
      WA1[J - 1] = X[J - 1];
    }
#pragma unroll
    for (int K = 1; K <= N; K++) {
      FKY = sys.f(WA1, K);
      NFCALL = NFCALL + 1;
      NFEV = NFCALL / N;
      FNORM = dmax1(FNORM, fabs(FKY));
#pragma unroll
      for (int J = K; J <= N; J++) {
#pragma unroll
        for (int I = 1; I <= N; I++) WA2[I - 1] = WA1[I - 1] + QQ(I, J);
        FKZ = sys.f(WA2, K);
        NFCALL = NFCALL + 1;
        NFEV = NFCALL / N;
        SIGMA[J - 1] = FKZ - FKY;
      }
      ETA = ZERO;
#pragma unroll
      for (int I = K; I <= N; I++) ETA = dmax1(ETA, fabs(SIGMA[I - 1]));
      if (ETA == ZERO) continue;
      NSING = NSING - 1;
      SKNORM = ZERO;
#pragma unroll
      for (int I = K; I <= N; I++) {
        SIGMA[I - 1] = SIGMA[I - 1] / ETA;
        SKNORM = SKNORM + SIGMA[I - 1] * SIGMA[I - 1];
      }
      SKNORM = sqrt(SKNORM);
      if (SIGMA[K - 1] < ZERO) SKNORM = -SKNORM;
      SIGMA[K - 1] = SIGMA[K - 1] + SKNORM;
#pragma unroll
      for (int I = 1; I <= N; I++) WA2[I - 1] = ZERO;
#pragma unroll
      for (int J = K; J <= N; J++) {
        TEMP = SIGMA[J - 1];
#pragma unroll
        for (int I = 1; I <= N; I++) WA2[I - 1] = WA2[I - 1] + TEMP * QQ(I, J);
      }
#pragma unroll
      for (int J = K; J <= N; J++) {
        TEMP = SIGMA[J - 1] / (SKNORM * SIGMA[K - 1]);
#pragma unroll
        for (int I = 1; I <= N; I++) QQ(I, J) = QQ(I, J) - TEMP * WA2[I - 1];
      }
      SIGMA[K - 1] = SKNORM * ETA;
      TEMP = FKY / SIGMA[K - 1];
      if (H * fabs(TEMP) > DELTA) TEMP = copysign(fabs(DELTA / H), TEMP);
#pragma unroll
      for (int I = 1; I <= N; I++) WA1[I - 1] = WA1[I - 1] + TEMP * QQ(I, K);
    }
    XNORM = ZERO;
    DIFIT = ZERO;
#pragma unroll
    for (int I = 1; I <= N; I++) {
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
    if (!CONV || DIFIT > P05 * XNORM || MOPT == 1) continue;
    bool done = false;
    for (int M = 2; M <= MOPT; M++) {
      bool stop_refine = false;
      FNORM1 = FNORM;
      FNORM = ZERO;
#pragma unroll
      for (int K = 1; K <= N; K++) {
        if (!stop_refine) {
          FKY = sys.f(WA1, K);
          NFCALL = NFCALL + 1;
          NFEV = NFCALL / N;
          FNORM = dmax1(FNORM, fabs(FKY));
          if (!(FNORM < FNORM1)) {
            FNORM = FNORM1;
            stop_refine = true;
          } else {
            TEMP = FKY / SIGMA[K - 1];
#pragma unroll
            for (int I = 1; I <= N; I++) WA1[I - 1] = WA1[I - 1] + TEMP * QQ(I, K);
          }
        }
      }
      if (stop_refine) break;
      XNORM = ZERO;
      DIFIT = ZERO;
#pragma unroll
      for (int I = 1; I <= N; I++) {
        XNORM = dmax1(XNORM, fabs(WA1[I - 1]));
        DIFIT = dmax1(DIFIT, fabs(X[I - 1] - WA1[I - 1]));
        X[I - 1] = WA1[I - 1];
      }
      if (FNORM <= FTOL) INFO = 1;
      if (DIFIT <= XTOL * XNORM) INFO = 2;
      if (FNORM <= FTOL && INFO == 2) INFO = 3;
      if (NFEV >= MAXFEV && INFO == 0) INFO = 4;
      if (INFO != 0) {
        done = true;
        break;
      }
    }
    if (done) break;
  }
#undef QQ
  *nfev_out = NFEV;
  return INFO;
}

struct Sist3F {
  const DevPhys& P;
  const Sist3& s;
  __device__ double f(const double* X, int K) const { return sist3_f(P, s, X, K); }
};
static __device__ int brentm3(const DevPhys& P, const Sist3& s, double* X, double FTOL, double XTOL, int MAXFEV,
                              int MOPT, int* nfev_out) {
  Sist3F sys{P, s};
  return brentm<3>(sys, X, FTOL, XTOL, MAXFEV, MOPT, nfev_out);
}

// ---------------------------------------------------------------------------
// The other ideal-MHD inversions, algo_solver 2..6 (system.f90:732-1158),
// out of line: the kernels that run algo 1 or Newton keep their registers.
// ---------------------------------------------------------------------------
// sist4 (system.f90:1235-1266): 2x2 in (y, p), x = v^2 from y; every call
// leaves its x in xinner, which algo 2 reads after BRENTM
struct Sist4F {
  const DevPhys& P;
  double B2, SB2, S2, U, D, xinner;
  __device__ double f(const double* X, int K) {
    double yy = X[0], pp = X[1];
    double xx = (S2 + SB2 * (2. * yy + B2) / (yy * yy)) / ((yy + B2) * (yy + B2));
    xinner = xx;
    if (K == 2) {
      double rh = D * sqrt(1 - xx), en = 0;
      (void)eos_energy(P, rh, &en, pp);
      return yy - (pp + en) / (1 - xx);
    }
    return yy - pp + 0.5 * (1. + xx) * B2 - 0.5 * SB2 / (yy * yy) - U;
  }
};

// eos_energy_with_ders (eos.f90:236-246, 527-584, 1189-1215); de/drho and
// de/dp are 0 where the reference leaves them unset or zeroes them
__device__ __forceinline__ int eos_energy_ders(const DevPhys& P, double rh, double* en, double pr, double* dendrh,
                                               double* dendpr) {
  *dendrh = 0.;
  *dendpr = 0.;
  if (P.eqstate == ECHO_EOS_TABLE) return eos_energy(P, rh, en, pr);
  if (pr <= P.przero) {
    *en = P.enezero * pr / P.przero;
    return 0;
  }
  if (P.eqstate == ECHO_EOS_CONFORMAL) {
    *en = 3. * pr;
    *dendpr = 3.;
  } else {
    *en = rh + pr / (4.0 / 3.0 - 1.);
    *dendrh = 1.;
    *dendpr = 1. / (4.0 / 3.0 - 1.);
  }
  return 0;
}

// getfun (system.f90:2060-2097); Fnorm, which the reference never assigns,
// is the Euclidean norm of F
__device__ __forceinline__ void getfun(const DevPhys& P, const Sist3& s, const double* X, double* F, double J[3][3],
                                       double* Fnorm, int sw) {
  double xx = X[0], yy = X[1], pp = X[2];
  double B2 = s.B2, SB2 = s.SB2, S2 = s.S2, U = s.U, D = s.D;
  F[0] = (yy + B2) * (yy + B2) * xx - SB2 / (yy * yy) * (2 * yy + B2) - S2;
  F[1] = yy - pp + 0.5 * (1. + xx) * B2 - 0.5 * SB2 / (yy * yy) - U;
  double rh = D * sqrt(1 - xx), en = 0, dendrh = 0, dendpr = 0;
  (void)eos_energy_ders(P, rh, &en, pp, &dendrh, &dendpr);
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

// ludecompose and solve (system.f90:1924-1986, 2026-2058), the pivot test as
// written (the pivot starts as A(i,i), not its modulus); A becomes U
__device__ __forceinline__ void ludecompose(double A[3][3], double L[3][3], int Pm[3], double smallvalue) {
  const int n = 3;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) L[i][j] = 0.;
  for (int i = 0; i < n; i++) Pm[i] = i;
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
      int t = Pm[i];
      Pm[i] = Pm[indP];
      Pm[indP] = t;
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
__device__ __forceinline__ void lusolve(double L[3][3], double U[3][3], const int Pm[3], double* X, const double* B) {
  const int n = 3;
  double Z[3];
  Z[0] = B[Pm[0]];
  for (int i = 1; i < n; i++) {
    double rowsum = B[Pm[i]];
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

// solver7 / solver8 (system.f90:2102-2201) and rtsafe (:2227-2286)
struct RtCtx {
  double B2, SB2, S2, UU, D, gam, w;
  int which;  // 7: ideal gas, 8: p = e/3
};
__device__ __forceinline__ void rt_func(RtCtx& c, double x, double* f, double* df) {
  const double third = 1.0 / 3.0;
  double B2 = c.B2, SB2 = c.SB2, S2 = c.S2, UU = c.UU, D = c.D, gam = c.gam;
  double v2 = x, rho = 0, c0, c2, c3, dw, dlogw, dc2, dc3, wb, vb2, w;
  c3 = 1.0 - gam * (1.0 - v2);
  if (c.which == 7) {
    rho = D * sqrt(1.0 - v2);
    c2 = gam * rho + .5 * B2 * (1.0 + v2) - UU;
  } else {
    c2 = .5 * B2 * (1.0 + v2) - UU;
  }
  c0 = -0.5 * SB2;
  if (c.which == 8 && c0 == 0.0) {
    w = -c2 / c3;
  } else {
    w = fmax(-c2 / c3, pow(-c0 / c3, third));
    int maxit = c.which == 7 ? 50 : 100;
    double wtol = c.which == 7 ? 1.e-10 : 1.e-12;
    for (int iter = 1; iter <= maxit; iter++) {
      dw = -((c3 * w + c2) * (w * w) + c0) / ((3 * c3 * w + 2 * c2) * w);
      if (fabs(dw / w) < wtol) break;
      w = w + dw;
    }
  }
  dc3 = gam;
  if (c.which == 7)
    dc2 = .5 * (B2 - gam * rho / (1. - v2));
  else
    dc2 = .5 * B2;
  dlogw = -(dc3 * w + dc2) / (3 * c3 * w + 2 * c2);
  wb = w + B2;
  vb2 = SB2 / (w * w);
  *f = wb * wb * v2 - (2 * w + B2) * vb2 - S2;
  *df = wb * (wb + 2 * dlogw * (w * v2 + vb2));
  c.w = w;
}
__device__ __forceinline__ double rtsafe(RtCtx& c, double x0, double x1, double x2, double xacc, int* ierr) {
  double f, df, xl = x1, xh = x2, dx, dxold, temp, r = x0;
  *ierr = 0;
  dxold = fabs(x2 - x1);
  dx = dxold;
  rt_func(c, r, &f, &df);
  for (int j = 1; j <= 100; j++) {
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

// solver10_approximate (system.f90:2205-2223) and get_x9 (:2290-2297); 12
// only when the exit test is met on the last allowed iteration, as written
__device__ __forceinline__ int solver10_approximate(double b, double c, double d, double oldsol, double* x) {
  int iter;
  *x = oldsol;
  for (iter = 1; iter <= 100; iter++) {
    double xx = *x;
    double dx = -(12 * (xx * xx * xx) + 3 * b * (xx * xx) + 2 * c * xx + d);
    if (fabs(dx / xx) < 1.e-12) break;
    *x = xx + dx;
  }
  return iter == 100 ? 12 : 0;
}
__device__ __forceinline__ double get_x9(double y, double s2, double b2, double sb2) {
  return (s2 * (y * y) + b2 * sb2 + 2 * sb2 * y) / ((y * y) * ((b2 * b2) + 2 * b2 * y + (y * y)));
}

// algo_solver 2..6; the reference's exit() calls become codes: 8 (algo 3
// out of iterations), 12 (algo 6 without a solution), 11 (no such solver).
// v[0..NV) in/out (guess in), u: conserved of the cell.
template <int KIND>
static __device__ __noinline__ int cons2prim_mhd_algo(const DevPhys& P, const Metric& M, int algo, const double* u,
                                                      double* v, int* iters) {
  typedef Traits<KIND> T;
  const double eps = 1.e-12;
  double g1 = M.g1, g2 = M.g2, g3 = M.g3, gm = M.gm;
  double uin[T::NV];
#pragma unroll
  for (int k = 0; k < T::NV; k++) uin[k] = gm * u[k];
  double DD = uin[KRH], sx = uin[KVX], sy = uin[KVY], sz = uin[KVZ], UU = uin[KPR];
  double bx = uin[KBX], by = uin[KBY], bz = uin[KBZ];
  int errcode = 0;
  *iters = 0;
  if (algo == 2 || algo == 3) {
    v[KBX] = uin[KBX];
    v[KBY] = uin[KBY];
    v[KBZ] = uin[KBZ];
    double B2 = bx * bx + by * by + bz * bz * g3;
    double SB = sx * bx + sy * by + sz * bz;
    double SB2 = SB * SB;
    double SS2 = sx * sx + sy * sy + sz * sz / g3;
    double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR], en = 0;
    errcode = eos_energy(P, rh, &en, pr);
    double xs, ys;
    if (algo == 2) {
      double v2old = g1 * (vx * vx) + g2 * (vy * vy) + g3 * (vz * vz);
      double X[2] = {(en + pr) / (1 - v2old), pr};
      Sist4F sys{P, B2, SB2, SS2, UU, DD, 0.};
      int nfev = 0;
      (void)brentm<2>(sys, X, 1.e-14, 1.e-14, 300, 3, &nfev);
      *iters = nfev;
      ys = X[0];
      pr = X[1];
      xs = sys.xinner;
    } else {
      double v2 = g1 * (vx * vx) + g2 * (vy * vy) + g3 * (vz * vz);
      double X[3] = {v2, (en + pr) / (1 - v2), pr}, F[3], J[3][3], L[3][3], DX[3], mF[3], Xt[3];
      double Fnorm = 0, Fnl = 0;
      int Pm[3], it = 0;
      Sist3 s3 = {B2, SB2, SS2, UU, DD, 0.};
      getfun(P, s3, X, F, J, &Fnorm, 1);
      while (Fnorm >= 1.e-14) {
        ludecompose(J, L, Pm, 4.e-16);
        for (int i = 0; i < 3; i++) mF[i] = -F[i];
        lusolve(L, J, Pm, DX, mF);
        double lambda = 1.;
        for (int i = 0; i < 3; i++) Xt[i] = X[i] + lambda * DX[i];
        getfun(P, s3, Xt, F, J, &Fnl, 1);
        if ((Fnl > (1 - lambda / 2) * Fnorm) && (lambda > 1. / 64)) {
          for (;;) {
            lambda = lambda / 2.;
            for (int i = 0; i < 3; i++) Xt[i] = X[i] + lambda * DX[i];
            getfun(P, s3, Xt, F, J, &Fnl, 0);
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
    if (T::GLM) v[T::KG] = u[T::KG];
    return errcode;
  }
  if (algo == 4 || algo == 5) {
    double S2 = sx * sx + sy * sy + sz * sz / g3;
    double B2 = bx * bx + by * by + bz * bz * g3;
    double SB = (sx * bx + sy * by + sz * bz);
    double SB2 = SB * SB;
    RtCtx c{B2, SB2, S2, UU, DD, algo == 4 ? (4.0 / 3.0 - 1) / (4.0 / 3.0) : 0.25, 0., algo == 4 ? 7 : 8};
    double v2_old = algo == 4 ? v[KVX] * v[KVX] + v[KVY] * v[KVY] + v[KVZ] * v[KVZ]
                              : v[KVX] * v[KVX] + v[KVY] * v[KVY] + v[KVZ] * v[KVZ] * g3;
    int ierr = 0;
    double v2 = rtsafe(c, v2_old, 0., 1. - 1.e-11, 1.e-12, &ierr);
    if (algo == 4 && ierr > 0) return 0;  // system.f90:926: returns, v untouched
    if (algo == 5 && ((v2 >= 1) || (ierr > 0))) return 778;
#pragma unroll
    for (int k = 0; k < T::NV; k++) v[k] = uin[k];
    if (T::GLM) v[T::KG] = u[T::KG];
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
    bool exact9 = true;
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
      exact9 = false;
      v2 = get_x9(sol9, S2, B2, SB2);
      if ((v2 < 0) || (v2 > 1) || (sol9 < 0)) return 12;
    }
    if (exact9) {
      // sol1..sol4 start at -1 (the reference leaves those of a negative
      // radicand unset)
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
#pragma unroll
    for (int k = 0; k < T::NV; k++) v[k] = uin[k];
    v[KRH] = DD * sqrt(1. - v2);
    v[KPR] = sol9 / 4 * (1 - v2);
    double vb = SB / sol9;
    v[KVX] = (sx + vb * bx) / (sol9 + B2);
    v[KVY] = (sy + vb * by) / (sol9 + B2);
    v[KVZ] = (sz + vb * bz) / (sol9 + B2);
    if (T::GLM) v[T::KG] = u[T::KG];
    return 0;
  }
  return 11;
}

// ---------------------------------------------------------------------------
// Newton on the same 3x3 system with the analytic Jacobian (the root BRENTM
// converges to); used by ECHO_C2P_NEWTON.  Residual target `tol` is on the
// relative size of the three equations.  Returns iterations, or -1 when it
// did not converge within `maxit` (the caller then falls back to BRENTM).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int eos_energy_slope(const DevPhys& P, double rh, double pr, double* en,
                                                double* dedp) {
  if (P.eqstate == ECHO_EOS_TABLE) {
    if (pr < __ldg(P.tp)) return 125;
    if (pr > __ldg(P.tp + P.nt - 1)) return 126;
    int h = SEARCH_P(P, pr);
#ifndef ECHO_EXACT
    if (P.sl_ep) {
      double sl = __ldg(P.sl_ep + h - 2);
      *dedp = sl;
      *en = __ldg(P.te + h - 2) + (pr - __ldg(P.tp + h - 2)) * sl;
      return 0;
    }
#endif
    double p2 = __ldg(P.tp + h - 1), p1 = __ldg(P.tp + h - 2);
    double e2 = __ldg(P.te + h - 1), e1 = __ldg(P.te + h - 2);
    *dedp = (e2 - e1) / (p2 - p1);
    *en = e1 + (e2 - e1) * (pr - p1) / (p2 - p1);
    return 0;
  }
  if (pr <= P.przero) {
    *en = P.enezero * pr / P.przero;
    *dedp = P.enezero / P.przero;
    return 0;
  }
  if (P.eqstate == ECHO_EOS_CONFORMAL) {
    *en = 3. * pr;
    *dedp = 3.;
  } else {
    *en = rh + pr / (4.0 / 3.0 - 1.);
    *dedp = 3.;
  }
  return 0;
}

// Newton on sist3 with the analytic Jacobian.  Converged when the relative
// residual max(|F1|/(y+B^2)^2, |F2|/(|U|+B^2), |F3|/y) <= tol; one more
// Newton correction is then applied (the error after it is ~ residual^2).
// Returns the number of corrections made, or -1 (the caller falls back).
static __device__ int newton3(const DevPhys& P, const Sist3& s, double* X, double tol, int maxit) {
  double xx = X[0], yy = X[1], pp = X[2];
  for (int it = 0; it <= maxit; it++) {
    if (!(xx < 1.0) || !(xx >= 0.0) || !(yy > 0.0) || !(pp > 0.0)) return -1;
    double sq = sqrt(1. - xx);
    double rh = s.D * sq, en = 0, dedp = 0;
    if (eos_energy_slope(P, rh, pp, &en, &dedp)) return -1;
    double ib = yy + s.B2, iy2 = 1.0 / (yy * yy), i1x = 1.0 / (1. - xx);
    double F1 = ib * ib * xx - s.SB2 * iy2 * (2 * yy + s.B2) - s.S2;
    double F2 = yy - pp + 0.5 * (1. + xx) * s.B2 - 0.5 * s.SB2 * iy2 - s.U;
    double F3 = yy - (pp + en) * i1x;
#ifdef ECHO_EXACT
    double iy3 = iy2 / yy;
    double r = fmax(fabs(F1) / (ib * ib), fmax(fabs(F2) / (fabs(s.U) + s.B2), fabs(F3) / yy));
#else
    // 1/y = y * (1/y^2); the residual scales as reciprocals (one division)
    double iy1 = yy * iy2, iy3 = iy2 * iy1;
    double r = fmax(fabs(F1) / (ib * ib), fmax(fabs(F2) * s.iUB, fabs(F3) * iy1));
#endif
    // d(en)/dx through rh is zero: the tabulated and conformal e(p) do not depend on rh
    double J11 = ib * ib, J12 = 2 * ib * xx + 2 * s.SB2 * (2 * yy + s.B2) * iy3 - 2 * s.SB2 * iy2, J13 = 0.;
    double J21 = 0.5 * s.B2, J22 = 1. + s.SB2 * iy3, J23 = -1.;
    double J31 = -(pp + en) * i1x * i1x, J32 = 1., J33 = -(1. + dedp) * i1x;
    // Cramer solve of J d = -F
    double c11 = J22 * J33 - J23 * J32, c12 = J23 * J31 - J21 * J33, c13 = J21 * J32 - J22 * J31;
    double det = J11 * c11 + J12 * c12 + J13 * c13;
    if (det == 0.0 || !isfinite(det)) return -1;
    double idet = 1.0 / det;
    double b1 = -F1, b2 = -F2, b3 = -F3;
    double dx = (b1 * c11 + b2 * (J13 * J32 - J12 * J33) + b3 * (J12 * J23 - J13 * J22)) * idet;
    double dy = (b1 * c12 + b2 * (J11 * J33 - J13 * J31) + b3 * (J13 * J21 - J11 * J23)) * idet;
    double dp = (b1 * c13 + b2 * (J12 * J31 - J11 * J32) + b3 * (J11 * J22 - J12 * J21)) * idet;
    if (r <= tol) {  // converged: polish and stop
      xx += dx;
      yy += dy;
      pp += dp;
      if (!(xx < 1.0) || !(yy > 0.0) || !(pp > 0.0)) return -1;
      X[0] = xx;
      X[1] = yy;
      X[2] = pp;
      return it + 1;
    }
    if (it == maxit) return -1;
    // damp steps that would leave the physical domain
    double lam = 1.0;
    for (int k = 0; k < 30 && (xx + lam * dx >= 1.0 || xx + lam * dx < 0.0 || yy + lam * dy <= 0.0 ||
                               pp + lam * dp <= 0.0);
         k++)
      lam *= 0.5;
    xx += lam * dx;
    yy += lam * dy;
    pp += lam * dp;
  }
  return -1;
}

// ---------------------------------------------------------------------------
// Resistive MHD (MHD = 2): Ohm's law and the implicit E solve.
// ---------------------------------------------------------------------------
// contravariant (a x b)^i = sqrt(gamma)/g_ii [ijk] a^j b^k of contravariant a,
// b (system_crossprod, system.f90:1867-1880, as the reference uses it in
// Minkowski coordinates)
__device__ __forceinline__ void cross_contra(const Metric& M, const double* a, const double* b, double* o) {
  double gp = M.gp;
  o[0] = gp * (a[1] * b[2] - a[2] * b[1]);
  o[1] = gp * (a[2] * b[0] - a[0] * b[2]);
  o[2] = gp / M.g3 * (a[0] * b[1] - a[1] * b[0]);
}

// stiff E source before the sqrt(-g) factor (system.f90:1656-1660):
// S = -gamma [sigma (E - (E.v) v + v x B) + sigma_chi (B - (B.v) v - v x E)]
// (B.v where the reference's Minkowski branch leaves it unset, :1750-1751)
__device__ __forceinline__ void ohm_stiff(const DevPhys& P, const Metric& M, const double* vel, const double* B,
                                          const double* E, double glf, double* S) {
  double g3 = M.g3, sig = P.sigma_el, chi = P.sigma_chiral;
  double vxb[3], vxe[3];
  cross_contra(M, vel, B, vxb);
  cross_contra(M, vel, E, vxe);
  double vdotb = vel[0] * B[0] + vel[1] * B[1] + vel[2] * B[2] * g3;
  double vdote = vel[0] * E[0] + vel[1] * E[1] + vel[2] * E[2] * g3;
#pragma unroll
  for (int i = 0; i < 3; i++)
    S[i] = -glf * (sig * (E[i] - vdote * vel[i] + vxb[i]) + chi * (B[i] - vdotb * vel[i] - vxe[i]));
}

// E = Es + h S(E) for fixed v and B, linear in E:
// [(1 + lam) I - lam v v_cov - mu (v x .)] E = Es - lam v x B - mu (B - (B.v) v),
// lam = h gamma sigma, mu = h gamma sigma_chi; solved by cofactors
__device__ __forceinline__ void ohm_solve(const DevPhys& P, const Metric& M, const double* Es, const double* vel,
                                          const double* B, double h, double* E) {
  double g3 = M.g3, gp = M.gp, gq = M.gp / M.g3;
  double v2 = vel[0] * vel[0] + vel[1] * vel[1] + g3 * (vel[2] * vel[2]);
  double glf = 1. / sqrt(1. - v2);
  double lam = h * glf * P.sigma_el, mu = h * glf * P.sigma_chiral;
  double vxb[3];
  cross_contra(M, vel, B, vxb);
  double vdotb = vel[0] * B[0] + vel[1] * B[1] + vel[2] * B[2] * g3;
  double vc[3] = {vel[0], vel[1], g3 * vel[2]};
  double C[3][3] = {{0., -gp * vel[2], gp * vel[1]}, {gp * vel[2], 0., -gp * vel[0]}, {-gq * vel[1], gq * vel[0], 0.}};
  double r[3], Mx[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    r[i] = Es[i] - lam * vxb[i] - mu * (B[i] - vdotb * vel[i]);
#pragma unroll
    for (int j = 0; j < 3; j++) Mx[i][j] = (i == j ? 1. + lam : 0.) - lam * vel[i] * vc[j] - mu * C[i][j];
  }
  double c00 = Mx[1][1] * Mx[2][2] - Mx[1][2] * Mx[2][1];
  double c01 = Mx[1][2] * Mx[2][0] - Mx[1][0] * Mx[2][2];
  double c02 = Mx[1][0] * Mx[2][1] - Mx[1][1] * Mx[2][0];
  double c10 = Mx[0][2] * Mx[2][1] - Mx[0][1] * Mx[2][2];
  double c11 = Mx[0][0] * Mx[2][2] - Mx[0][2] * Mx[2][0];
  double c12 = Mx[0][1] * Mx[2][0] - Mx[0][0] * Mx[2][1];
  double c20 = Mx[0][1] * Mx[1][2] - Mx[0][2] * Mx[1][1];
  double c21 = Mx[0][2] * Mx[1][0] - Mx[0][0] * Mx[1][2];
  double c22 = Mx[0][0] * Mx[1][1] - Mx[0][1] * Mx[1][0];
  double det = Mx[0][0] * c00 + Mx[0][1] * c01 + Mx[0][2] * c02;
  E[0] = (c00 * r[0] + c10 * r[1] + c20 * r[2]) / det;
  E[1] = (c01 * r[0] + c11 * r[1] + c21 * r[2]) / det;
  E[2] = (c02 * r[0] + c12 * r[1] + c22 * r[2]) / det;
}

// Resistive con2prim with the implicit Ohm's law of an IMEX stage (the
// algo_solver 7 the reference names, common.f90:292-293, 2109-2113, but has
// no branch for, system.f90:1160-1162).  h = a_ii dt of the stage (0: plain
// inversion).  Fixed point on v: E(v) from ohm_solve; the fluid's share
// S - E x B, U - (E^2 + B^2)/2; the ideal-HD Newton on p (system.f90:511-561)
// for p and the new v; until max |dv| <= 1e-14 (one pass for h = 0), 779
// after 200 passes.  It starts from the previous primitives in v (the
// reference's warm start) or, given the learned seed (x = v^2, q = p/U of
// the total energy U), from p = q U and v along the fluid momentum S - E x B
// (E of u) with |v|^2 = x; the seeded first pass gets 3 Newton steps, whose
// last must be below 1e-10 of p (the seed's residual bar), and is always
// followed by a pass at the full tolerance; a seed that fails restarts the
// fixed point from the warm start (*seed_failed = 1).  v[KEX..KEZ] receives E and, when h > 0, u[KEX..KEZ]
// sqrt(-g) E: the implicit solve changes the conserved E.
inline __device__ int cons2prim_res(const DevPhys& P, const Metric& M, double* u, double* v, int* iters,
                                    double h, const float* seed = nullptr, int* seed_failed = nullptr) {
  const double ntol = 1.e-12, vtol = 1.e-14;
  double g1 = M.g1, g2 = M.g2, g3 = M.g3, gm = M.gm, gp = M.gp;
  double d = gm * u[KRH], U = gm * u[KPR];
  double S[3] = {gm * u[KVX], gm * u[KVY], gm * u[KVZ]};
  double B[3] = {gm * u[KBX], gm * u[KBY], gm * u[KBZ]};
  double Es[3] = {gm * u[KEX], gm * u[KEY], gm * u[KEZ]};
  double vel[3] = {v[KVX], v[KVY], v[KVZ]}, E[3];
  double pr = v[KPR], rh = v[KRH];
  double B2 = B[0] * B[0] + B[1] * B[1] + (B[2] * B[2]) * g3;
  int cap = 1 << 30;  // Newton steps the current pass may take
  if (seed) {
    const double x = (double)seed[0], q = (double)seed[1];
    if (x >= 0. && x < 1. && q > 0. && U > 0.) {
      double Ec[3] = {Es[0], Es[1], Es[2] * g3}, EXB[3];
      exb(M, Ec, B[0], B[1], B[2], EXB);
      double sx = S[0] - EXB[0], sy = S[1] - EXB[1], sz = (S[2] - EXB[2]) / g3;
      double s2 = g1 * sx * sx + g2 * sy * sy + g3 * sz * sz;
      double a = s2 > 0. ? sqrt(x / s2) : 0.;
      vel[0] = a * sx;
      vel[1] = a * sy;
      vel[2] = a * sz;
      pr = q * U;
      cap = 3;
    } else if (seed_failed) {
      *seed_failed |= 1;
    }
  }
  int errcode = 0, outer, total = 0;
  for (outer = 1; outer <= 200; outer++) {
    if (h > 0.) {
      ohm_solve(P, M, Es, vel, B, h, E);
    } else {
      E[0] = Es[0];
      E[1] = Es[1];
      E[2] = Es[2];
    }
    double Ec[3] = {E[0], E[1], E[2] * g3}, EXB[3];
    exb(M, Ec, B[0], B[1], B[2], EXB);
    double E2 = Ec[0] * Ec[0] + Ec[1] * Ec[1] + (Ec[2] * Ec[2]) / g3;
    double sx = S[0] - EXB[0], sy = S[1] - EXB[1], sz = (S[2] - EXB[2]) / g3;
    double et = U - 0.5 * (E2 + B2);
    double s2 = g1 * sx * sx + g2 * sy * sy + g3 * sz * sz;
    double w = 0, v2 = 0, glf, en, drhdpr, dendpr, pr_eos = 0, dprdrh = 0, dprden = 0, f, df, dpr;
    bool newton_ok = false;
    int iter;
    for (iter = 1; iter <= 100; iter++) {
      w = et + pr;
      v2 = s2 / (w * w);
      if (v2 >= 1.) break;
      glf = 1. / sqrt(1. - v2);
      rh = d / glf;
      en = w * (1. - v2) - pr;
      drhdpr = rh * v2 * glf / (en + pr);
      dendpr = v2;
      errcode = eos_pressure(P, rh, en, &pr_eos, &dprdrh, &dprden);
      f = pr_eos - pr;
      df = dprdrh * drhdpr + dprden * dendpr - 1.;
      dpr = -f / df;
      if (fabs(dpr) < ntol * pr) {
        newton_ok = true;
        break;
      }
      if (iter >= cap) {  // the seed's budget, judged at a 1e-10 step
        newton_ok = fabs(dpr) < 1.e-10 * pr;
        if (newton_ok) pr = pr + dpr;  // the full-tolerance pass starts from the corrected p
        break;
      }
      pr = pr + dpr;
    }
    total += iter;
    if (cap < 100 && (v2 >= 1. || !newton_ok)) {
      // the seed failed: the fixed point from the warm start
      if (seed_failed) *seed_failed |= 1;
      vel[0] = v[KVX];
      vel[1] = v[KVY];
      vel[2] = v[KVZ];
      pr = v[KPR];
      cap = 1 << 30;
      outer = 0;
      continue;
    }
    if (v2 >= 1.) {
      *iters = total;
      return 777;
    }
    const bool seeded_pass = cap < 100;  // another pass at the full tolerance follows
    cap = 1 << 30;
    double vn0 = sx / w, vn1 = sy / w, vn2 = sz / w;
    double dv = fmax3(fabs(vn0 - vel[0]), fabs(vn1 - vel[1]), fabs(vn2 - vel[2]) * gp);
    vel[0] = vn0;
    vel[1] = vn1;
    vel[2] = vn2;
    if (!seeded_pass && (!(h > 0.) || dv <= vtol)) break;
  }
  *iters = total;
  if (outer > 200) return 779;
  v[KRH] = rh;
  v[KVX] = vel[0];
  v[KVY] = vel[1];
  v[KVZ] = vel[2];
  v[KPR] = pr;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    v[KBX + i] = B[i];
    v[KEX + i] = E[i];
    if (h > 0.) u[KEX + i] = E[i] * gp;
  }
  v[Traits<KIND_RES>::KG] = u[Traits<KIND_RES>::KG];
  if (pr <= 0) errcode = 777;
  return errcode;
}

// ---------------------------------------------------------------------------
// system_cons2prim (system.f90:423-1166).  u, v of length NV; v holds the
// initial guess.  Returns the reference errcode; *iters gets the iteration
// count (Newton steps, or BRENTM function evaluations).  h: the implicit
// coefficient of a resistive IMEX stage (cons2prim_res).  ALT: the
// instantiation that also runs ALG_SOLV 2..6 (cons2prim_mhd_algo); the step
// kernels use the other one and leave those algorithms to c2p_alt_kernel, so
// that the out-of-line call does not cost them registers.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ bool c2p_alt_algo(int algo) {
  return algo != ECHO_C2P_BRENT && algo != ECHO_C2P_NEWTON && algo != ECHO_C2P_MLP;
}

template <int KIND, bool ALT = false>
__device__ int cons2prim(const DevPhys& P, const Metric& M, int algo, double tol, const double* u,
                         double* v, int* iters, const float* seed = nullptr, int* seed_failed = nullptr,
                         double h = 0.) {
  typedef Traits<KIND> T;
  // every resistive caller passes its own copy of u, which the implicit
  // solve updates (the reference's con2prim may modify u, evolve.f90:848)
  if (T::RES) return cons2prim_res(P, M, const_cast<double*>(u), v, iters, h, seed, seed_failed);
  const double eps = 1.e-12;
  const double ntol = 1.e-12;
  double g1 = M.g1, g2 = M.g2, g3 = M.g3, gm = M.gm;
  int errcode = 0;
  *iters = 0;
  if (!T::VISC && !T::MHD) {
    // ideal hydro Newton-Raphson (system.f90:511-561)
    double d = gm * u[KRH];
    double sx = gm * u[KVX];
    double sy = gm * u[KVY];
    double sz = gm * u[KVZ] / g3;
    double et = gm * u[KPR];
    double s2 = g1 * sx * sx + g2 * sy * sy + g3 * sz * sz;
    double pr = v[KPR], w = 0, v2, glf, rh = 0, en, drhdpr, dendpr;
    double pr_eos = 0, dprdrh = 0, dprden = 0, f, df, dpr;
    int iter;
    for (iter = 1; iter <= 100; iter++) {
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
      errcode = eos_pressure(P, rh, en, &pr_eos, &dprdrh, &dprden);
      f = pr_eos - pr;
      df = dprdrh * drhdpr + dprden * dendpr - 1.;
      dpr = -f / df;
      if (fabs(dpr) < ntol * pr) break;
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
  } else if (T::VISC) {
    // nested iteration (system.f90:564-666).  The reference's outer loop
    // ends after one pass: its test compares v^2 of the new velocities with
    // the Newton's own v^2, the same number, so pi^{t mu} keep the guess's
    // velocities (a relative residual ~1e-4 in S on the workload).
    // ECHO_C2P_NEWTON and ECHO_C2P_MLP iterate the passes to the fixed
    // point instead (max |dv| <= 1e-14, each pass's Newton from the last
    // pass's p): the inversion's own root, at equal residual whatever the
    // start.  With the learned seed (x = v^2, q = p/U) the first pass starts
    // from v along S with |v|^2 = x and p = q U and its Newton gets 3
    // steps, the last below 1e-10 of p, with a pass at the full tolerance
    // after it; a seed that fails restarts from the warm start
    // (*seed_failed = 1).
    double uin[T::NV], vprim[T::NV];
#pragma unroll
    for (int k = 0; k < T::NV; k++) uin[k] = gm * u[k];
    double d = uin[KRH];
#pragma unroll
    for (int k = KPIBU; k <= KPIZZ; k++) v[k] = uin[k] / uin[KRH];
    double vx = v[KVX], vy = v[KVY], vz = v[KVZ];
    double v2 = g1 * (vx * vx) + g2 * (vy * vy) + g3 * (vz * vz);
#pragma unroll
    for (int k = 0; k < T::NV; k++) vprim[k] = v[k];
    double rh = 0, pr = 0, glf, en, drhdpr, dendpr, pr_eos = 0, dprdrh = 0, dprden = 0, f, df, dpr;
    double et = gm * u[KPR];
    const bool conv = algo == ECHO_C2P_NEWTON || algo == ECHO_C2P_MLP;
    double p0 = v[KPR];  // where each pass's Newton starts
    int cap = 1 << 30;   // Newton steps the current pass may take
    if (seed) {
      const double x = (double)seed[0], q = (double)seed[1];
      if (x >= 0. && x < 1. && q > 0. && et > 0.) {
        double sx = uin[KVX], sy = uin[KVY], sz = uin[KVZ] / g3;
        double s2 = g1 * sx * sx + g2 * sy * sy + g3 * sz * sz;
        double a = s2 > 0. ? sqrt(x / s2) : 0.;
        vx = a * sx;
        vy = a * sy;
        vz = a * sz;
        p0 = q * et;
        cap = 3;
      } else if (seed_failed) {
        *seed_failed |= 1;
      }
    }
    int tot = 0;
    for (int iv = 1; iv <= 100; iv++) {
      vprim[KVX] = vx;
      vprim[KVY] = vy;
      vprim[KVZ] = vz;
      Pit pi;
      derived_pi_any(P, M, vprim, pi);
      double en1 = et + v[KPIBU] + pi.tt * M.g0;
      double sx_cov = uin[KVX] - pi.tx;
      double sy_cov = uin[KVY] - pi.ty;
      double sz_cov = uin[KVZ] - pi.tz * g3;
      double sx = sx_cov, sy = sy_cov, sz = sz_cov / g3;
      double s2 = sx * sx_cov + sy * sy_cov + sz * sz_cov;
      pr = p0;
      bool newton_ok = false;
      for (int ip = 1; ip <= 100; ip++) {
        tot++;
        v2 = s2 / ((en1 + pr) * (en1 + pr));
        if (v2 >= 1.) break;
        glf = 1. / sqrt(1. - v2);
        rh = d / glf;
        en = (en1 + pr) * (1. - v2) - pr - vprim[KPIBU];
        drhdpr = rh * v2 * glf / (en + pr);
        dendpr = v2;
        errcode = eos_pressure(P, rh, en, &pr_eos, &dprdrh, &dprden);
        f = pr_eos - pr;
        df = dprdrh * drhdpr + dprden * dendpr - 1.;
        dpr = -f / df;
        if (fabs(dpr) < ntol * pr) {
          newton_ok = true;
          break;
        }
        if (ip >= cap) {  // the seed's budget, judged at a 1e-10 step
          newton_ok = fabs(dpr) < 1.e-10 * pr;
          if (newton_ok) pr = pr + dpr;  // the full-tolerance pass starts from the corrected p
          break;
        }
        pr = pr + dpr;
      }
      if (cap < 100 && (v2 >= 1. || !newton_ok)) {
        // the seed failed: the iteration from the warm start
        if (seed_failed) *seed_failed |= 1;
        vx = v[KVX];
        vy = v[KVY];
        vz = v[KVZ];
        p0 = v[KPR];
        cap = 1 << 30;
        iv = 0;
        continue;
      }
      if (v2 >= 1.) {
        *iters = tot;
        return 107;
      }
      const bool seeded_pass = cap < 100;  // another pass at the full tolerance follows
      cap = 1 << 30;
      double nvx = sx / (en1 + pr);
      if (fabs(nvx) < eps) nvx = 0.;
      double nvy = sy / (en1 + pr);
      if (fabs(nvy) < eps) nvy = 0.;
      double nvz = sz / (en1 + pr);
      if (fabs(nvz) < eps) nvz = 0.;
      // the converged passes' test: a component below eps is zeroed (above), so
      // one that sits at that threshold can alternate between 0 and just above
      // eps forever; one whose old and new values are both below 2 eps counts
      // as settled
      const double dvs = fmax3(fabs(nvx) < 2. * eps && fabs(vx) < 2. * eps ? 0. : fabs(nvx - vx),
                               fabs(nvy) < 2. * eps && fabs(vy) < 2. * eps ? 0. : fabs(nvy - vy),
                               fabs(nvz) < 2. * eps && fabs(vz) < 2. * eps ? 0. : fabs(nvz - vz) * M.gp);
      vx = nvx;
      vy = nvy;
      vz = nvz;
      vprim[KVX] = vx;
      vprim[KVY] = vy;
      vprim[KVZ] = vz;
      if (conv) {
        p0 = pr;
        if (dvs <= 1.e-14 && !seeded_pass) break;
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
    if (P.obtained_zz) {
      Pit pi;
      derived_pi_zz(M, v, pi);
      v[KPIZZ] = pi.zz;
    }
    return errcode;
  } else {
    // ideal MHD (system.f90:668-730): BRENTM on sist3, or Newton on the same system
    if constexpr (ALT && T::MHD && !T::RES) {
      if (c2p_alt_algo(algo)) return cons2prim_mhd_algo<KIND>(P, M, algo, u, v, iters);
    }
    double uin[T::NV];
#pragma unroll
    for (int k = 0; k < T::NV; k++) uin[k] = gm * u[k];
    double DD = uin[KRH];
    double sx = uin[KVX], sy = uin[KVY], sz = uin[KVZ];
    double UU = uin[KPR];
    double bx = uin[KBX], by = uin[KBY], bz = uin[KBZ];
    v[KBX] = uin[KBX];
    v[KBY] = uin[KBY];
    v[KBZ] = uin[KBZ];
    double B2 = bx * bx + by * by + bz * bz * g3;
    double SB = sx * bx + sy * by + sz * bz;
    double SB2 = SB * SB;
    double SS2 = sx * sx + sy * sy + sz * sz / g3;
    double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR];
    double en = 0;
    errcode = eos_energy(P, rh, &en, pr);
    double v2 = g1 * (vx * vx) + g2 * (vy * vy) + g3 * (vz * vz);
    double X[3];
    X[0] = v2;
    X[1] = (en + pr) / (1 - v2);
    X[2] = pr;
    Sist3 s = {B2, SB2, SS2, UU, DD, 1.0 / (fabs(UU) + B2)};
    int nfev = 0;
    if (algo == ECHO_C2P_NEWTON || algo == ECHO_C2P_MLP) {
      int it = -1, used = 0;
      if (algo == ECHO_C2P_MLP && seed) {
        // learned seed: x = v^2 and p = q U, y from sist3's third equation
        double xs0 = (double)seed[0], ps0 = (double)seed[1] * UU;
        xs0 = xs0 < 0. ? 0. : (xs0 > 0.99 ? 0.99 : xs0);
        double Xs[3] = {xs0, 0., ps0};
        double es = 0;
        if (ps0 > 0. && !eos_energy(P, DD * sqrt(1 - xs0), &es, ps0)) {
          Xs[1] = (ps0 + es) / (1 - xs0);
          it = newton3(P, s, Xs, tol, 3);
          used = it > 0 ? it : 3;
          if (it > 0) {
            X[0] = Xs[0];
            X[1] = Xs[1];
            X[2] = Xs[2];
          }
        }
        if (it <= 0 && seed_failed) *seed_failed |= 1;
      }
      if (it <= 0) {  // plain path: Newton from the previous primitives
        double Xn[3] = {X[0], X[1], X[2]};
        it = newton3(P, s, Xn, tol, 30);
        if (it > 0) {
          X[0] = Xn[0];
          X[1] = Xn[1];
          X[2] = Xn[2];
          it += used;
        }
      }
      if (it > 0) {
        nfev = it;
      } else {
        (void)brentm3(P, s, X, 1.e-14, 1.e-14, 300, 3, &nfev);
        if (seed_failed) *seed_failed |= 2;  // a bracketed fallback, counted on its own
      }
    } else {
      (void)brentm3(P, s, X, 1.e-14, 1.e-14, 300, 3, &nfev);
    }
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
    if (T::GLM) v[T::KG] = u[T::KG];
    return errcode;
  }
}

// ---------------------------------------------------------------------------
// get_sigma (viscous.f90:283-393)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void get_sigma(const DevPhys& P, const Metric& M, const double* v, const double* d,
                                          double sigma[6]) {
  enum { SXX = 0, SYY = 1, SZZ = 2, SXY = 3, SXZ = 4, SYZ = 5 };
  double g1 = M.g1, g2 = M.g2, g3 = M.g3, t = M.t;
  double ux = v[KVX], uy = v[KVY], uz = v[KVZ];
  double ut = 1. / sqrt(1. - g1 * ux * ux - g2 * uy * uy - g3 * uz * uz);
  ux = ux * ut;
  uy = uy * ut;
  uz = uz * ut;
  double dutdt = d[DTT], duxdx = d[DXX], duydy = d[DYY], duzdz = d[DZZ], duzdt = d[DZT];
  double duzdx = d[DZX], duzdy = d[DZY], duxdt = d[DXT], duxdy = d[DXY];
  double duxdz = d[DXZ], duydt = d[DYT], duydx = d[DYX], duydz = d[DYZ];
  if (P.coordinates == ECHO_MINKOWSKI) {
    sigma[SZZ] = ut * uz * duzdt + uz * ux * duzdx + uz * uy * duzdy + (2. / 3.) * duzdz +
                 (2. / 3.) * duzdz * (uz * uz) - dutdt / 3. - duxdx / 3. - duydy / 3. -
                 (uz * uz) * dutdt / 3. - (uz * uz) * duxdx / 3. - (uz * uz) * duydy / 3.;
    sigma[SXZ] = 0.5 * ut * ux * duzdt + 0.5 * duzdx + 0.5 * (ux * ux) * duzdx + 0.5 * ux * uy * duzdy +
                 ux * uz * duzdz / 6. + 0.5 * ut * uz * duxdt + ux * uz * duxdx / 6. + 0.5 * uy * uz * duxdy +
                 0.5 * duxdz + 0.5 * duxdz * (uz * uz) - ux * uz * dutdt / 3. - ux * uz * duydy / 3.;
    sigma[SXY] = 0.5 * ut * ux * duydt + 0.5 * duydx + 0.5 * (ux * ux) * duydx + ux * uy * duydy / 6. +
                 ux * uz * duydz / 2. + 0.5 * ut * uy * duxdt + ux * uy * duxdx / 6. + 0.5 * duxdy +
                 0.5 * duxdy * (uy * uy) + uy * uz * duxdz / 2. - ux * uy * dutdt / 3. - ux * uy * duzdz / 3.;
    sigma[SYZ] = 0.5 * ut * uy * duzdt + ux * uy * duzdx / 2. + duzdy / 2. + duzdy * (uy * uy) / 2. +
                 uy * uz * duzdz / 6. + ut * uz * duydt / 2. + ux * uz * duydx / 2. + uy * uz * duydy / 6. +
                 duydz / 2. + duydz / 2. * (uz * uz) - uy * uz * dutdt / 3. - uy * uz * duxdx / 3.;
    sigma[SXX] = ut * ux * duxdt + (2. / 3.) * duxdx + (2. / 3.) * duxdx * (ux * ux) + ux * uy * duxdy +
                 ux * uz * duxdz - dutdt / 3. - duydy / 3. - duzdz / 3. - (ux * ux) * dutdt / 3. -
                 (ux * ux) * duydy / 3. - (ux * ux) * duzdz / 3.;
    sigma[SYY] = ut * uy * duydt + ux * uy * duydx + (2. / 3.) * duydy + (2. / 3.) * duydy * (uy * uy) +
                 uy * uz * duydz - dutdt / 3. - duxdx / 3. - duzdz / 3. - (uy * uy) * dutdt / 3. -
                 (uy * uy) * duxdx / 3. - (uy * uy) * duzdz / 3.;
  } else {
    double t2 = t * t, t3 = M.t3;
    sigma[SZZ] = ut * uz * duzdt + uz * ux * duzdx + uz * uy * duzdy + (2. * duzdz) / (3. * t2) +
                 (2. / 3.) * duzdz * (uz * uz) - dutdt / (3. * t2) - duxdx / (3. * t2) - duydy / (3. * t2) -
                 (uz * uz) * dutdt / 3. - (uz * uz) * duxdx / 3. - (uz * uz) * duydy / 3. + 2. / 3. * ut / t3 +
                 5. / 3. * (ut / t) * (uz * uz);
    sigma[SXZ] = 0.5 * ut * ux * duzdt + 0.5 * duzdx + 0.5 * (ux * ux) * duzdx + 0.5 * ux * uy * duzdy +
                 ux * uz * duzdz / 6. + 0.5 * ut * uz * duxdt + ux * uz * duxdx / 6. + 0.5 * uy * uz * duxdy +
                 duxdz / (2. * t2) + 0.5 * duxdz * (uz * uz) - ux * uz * dutdt / 3. - ux * uz * duydy / 3. +
                 (2. / 3.) * ut * uz * ux / t;
    sigma[SXY] = 0.5 * ut * ux * duydt + 0.5 * duydx + 0.5 * (ux * ux) * duydx + ux * uy * duydy / 6. +
                 ux * uz * duydz / 2. + 0.5 * ut * uy * duxdt + ux * uy * duxdx / 6. + 0.5 * duxdy +
                 0.5 * duxdy * (uy * uy) + uy * uz * duxdz / 2. - ux * uy * dutdt / 3. - ux * uy * duzdz / 3. -
                 ut * ux * uy / (3. * t);
    sigma[SYZ] = 0.5 * ut * uy * duzdt + ux * uy * duzdx / 2. + duzdy / 2. + duzdy * (uy * uy) / 2. +
                 uy * uz * duzdz / 6. + ut * uz * duydt / 2. + ux * uz * duydx / 2. + uy * uz * duydy / 6. +
                 duydz / (2. * t2) + duydz / 2. * (uz * uz) - uy * uz * dutdt / 3. - uy * uz * duxdx / 3. +
                 (2. / 3.) * ut * uz * uy / t;
    sigma[SXX] = ut * ux * duxdt + (2. / 3.) * duxdx + (2. / 3.) * duxdx * (ux * ux) + ux * uy * duxdy +
                 ux * uz * duxdz - dutdt / 3. - duydy / 3. - duzdz / 3. - ut / (3. * t) - (ux * ux) * dutdt / 3. -
                 (ux * ux) * duydy / 3. - (ux * ux) * duzdz / 3. - (ux * ux) * ut / (3. * t);
    sigma[SYY] = ut * uy * duydt + ux * uy * duydx + (2. / 3.) * duydy + (2. / 3.) * duydy * (uy * uy) +
                 uy * uz * duydz - dutdt / 3. - duxdx / 3. - duzdz / 3. - ut / (3. * t) - (uy * uy) * dutdt / 3. -
                 (uy * uy) * duxdx / 3. - (uy * uy) * duzdz / 3. - (uy * uy) * ut / (3. * t);
  }
}

// ---------------------------------------------------------------------------
// system_source (system.f90:1587-1842) without the resistive terms.
// v: primitives of the cell (modified copy), dv: its 16 derivatives.
// kap, when not null on a viscous run, receives the Israel-Stewart
// relaxation rates on the conserved stresses: the source of
// u[k] = sqrt(-g) rho gamma v[k] holds -kap u[k], with kap[0] = 1/(gamma
// tau_Pi) for the bulk pressure and kap[1] = 1/(gamma tau_pi) for the shear
// components (the -1/tau (v[k] + ...) terms times rho sqrt(-g)).
// ---------------------------------------------------------------------------
template <int KIND>
__device__ int system_source(const DevPhys& P, const Metric& M, double* v, const double* dv, double* src,
                             double* kap = nullptr, double rhoC = 0., double* stiff = nullptr) {
  typedef Traits<KIND> T;
  double g1 = M.g1, g2 = M.g2, g3 = M.g3, gp = M.gp, g0 = M.g0, t = M.t;
#pragma unroll
  for (int k = 0; k < T::NV; k++) src[k] = 0.;
  double rh = v[KRH], vx = v[KVX], vy = v[KVY], vz = v[KVZ], pr = v[KPR];
  double en = 0;
  int err = eos_energy(P, rh, &en, pr);
  if (err) return err;
  double v2 = g1 * vx * vx + g2 * vy * vy + g3 * vz * vz;
  double glf = 1. / sqrt(1. - v2);
  double ut = glf;
  const double lambda0 = 1., lambda1 = 1., lambda2 = 0.;
  if (!T::VISC) {
    if (P.coordinates == ECHO_BJORKEN) {
      double w = en + pr;
      double ww = w * (glf * glf);
      if (T::MHD) {
        double E[3];
        e_field<KIND>(M, v, E);  // the reference takes -v x B here also for
                                 // resistive runs (system.f90:1641)
        double bx = v[KBX], by = v[KBY], bz = v[KBZ];
        double B2 = bx * bx + by * by + (bz * bz) * g3;
        double E2 = E[0] * E[0] + E[1] * E[1] + (E[2] * E[2]) / g3;
        double EEM = 0.5 * (E2 + B2);
        double e3g = E[2] / g3;
        src[KPR] = -t * (ww * vz * vz - e3g * e3g - bz * bz + (EEM + pr) / g3);
      } else {
        src[KPR] = -t * (ww * vz * vz + pr / g3);
      }
    }
  } else {
    double sigma[6], eta, zeta, tau_pi, tau_pi_big;
    enum { SXX = 0, SYY = 1, SZZ = 2, SXY = 3, SXZ = 4, SYZ = 5 };
    get_sigma(P, M, v, dv, sigma);
    err = viscous_parameters(P, v[KRH], v[KPR], &eta, &zeta, &tau_pi, &tau_pi_big);
    if (err) return err;
    Pit pi;
    derived_pi_any(P, M, v, pi);
    double pitx = pi.tx, pity = pi.ty, pitz = pi.tz;
    double dutdt = dv[DTT], dutdx = dv[DTX], dutdy = dv[DTY], dutdz = dv[DTZ];
    double duxdx = dv[DXX], duydy = dv[DYY], duzdz = dv[DZZ], duzdt = dv[DZT];
    double duzdx = dv[DZX], duzdy = dv[DZY], duxdt = dv[DXT], duxdy = dv[DXY];
    double duxdz = dv[DXZ], duydt = dv[DYT], duydx = dv[DYX], duydz = dv[DYZ];
    double sum_der = dutdt + duxdx + duydy + duzdz;
    if (P.coordinates == ECHO_BJORKEN) {
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
    } else {
      double sum_der_0 = g0 * (glf * dutdt + v[KVX] * dutdx + v[KVY] * dutdy + v[KVZ] * dutdz);
      double sum_der_x = g1 * (glf * duxdt + v[KVX] * duxdx + v[KVY] * duxdy + v[KVZ] * duxdz);
      double sum_der_y = g2 * (glf * duydt + v[KVX] * duydx + v[KVY] * duydy + v[KVZ] * duydz);
      double sum_der_z = g3 * (glf * duzdt + v[KVX] * duzdx + v[KVY] * duzdy + v[KVZ] * duzdz);
      src[KPIBU] = -1. / tau_pi_big * (v[KPIBU] + zeta * sum_der) + lambda0 * (-1. / 3. * v[KPIBU] * sum_der);
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
#pragma unroll
    for (int k = KPIBU; k < T::NV; k++) src[k] = src[k] * v[KRH];
    if (kap) {
      kap[0] = 1. / (glf * tau_pi_big);
      kap[1] = 1. / (glf * tau_pi);
    }
  }
  if (T::RES) {
    // charge current and Ohm's law (system.f90:1650-1661, 1747-1756);
    // stiff: the three E components, times sqrt(-g)
    double vel[3] = {vx, vy, vz}, S[3];
    ohm_stiff(P, M, vel, v + KBX, v + KEX, glf, S);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      src[KEX + i] = -rhoC * vel[i];
      if (stiff) stiff[i] = S[i] * gp;
    }
  }
#pragma unroll
  for (int k = 0; k < T::NV; k++) src[k] = src[k] * gp;
  return 0;
}

}  // namespace echo
