// glauber.cu -- the optical Glauber initial state on the device
// (echo_gpu_optical_glauber): the reference's GLAUBER_GEOMETRIC initial
// conditions, init.f90:852-1242.
//
//   thickness_kernel   one thread per table radius r = (nc-1) dr: the
//                      Woods-Saxon density summed over |z| <= 2 radius with
//                      the reference's refinement of dz (init.f90:1164-1216)
//   glauber_kernel     one thread per cell: wounded nucleons and binary
//                      collisions from the nearest table radius (wound,
//                      bincoll, init.f90:971-1032), calc_enedens
//                      (init.f90:902-929) and initio (init.f90:852-893):
//                      rho, v = 0, p = p(e) + przero
//
// The state then goes through echo_gpu_upload_device (prim2cons on the
// device), as an upload of primitives without u.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/echo_gpu.h"
#include "ctx.cuh"

using namespace echo;

namespace {

enum { THICK_RUNS = 8 };  // halvings of dz before a radius counts as not converged

// Fortran nint: nearest integer, halves away from zero
__host__ __device__ inline long nint_f(double x) { return x >= 0. ? (long)floor(x + 0.5) : -(long)floor(-x + 0.5); }

// thick[nc-1] = T((nc-1) dr) and term[nc-1] = r sum1 dz (the summand of the
// check mass); bad = 1 when a radius needed more than THICK_RUNS halvings
__global__ void thickness_kernel(int nmax, double radius, double delta, double roze, double dr, double dz1,
                                 double acc, double* thick, double* term, int* bad) {
  const int nc = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (nc > nmax) return;
  const double delta_inv = 1. / delta;
  const double zmax = 2. * radius;
  double dz = 2. * dz1;
  const double r = (nc - 1) * dr;
  const double r2 = r * r;
  double ratio = 1000., sum1 = 0., sum2 = 0.;
  int nrun = 0;
  while (ratio > acc) {
    if (nrun == THICK_RUNS) {
      *bad = 1;
      break;
    }
    dz = dz * 0.5;
    const long nstep = nint_f(2. * zmax / dz);
    nrun = nrun + 1;
    double z1 = -zmax, z2 = z1 + dz;
    sum1 = 0.;
    sum2 = 0.;
    // rho at z1 of a step is rho at z2 of the previous one (z1 = z2 exactly)
    double rho_prev = roze / (exp((sqrt(r2 + z1 * z1) - radius) * delta_inv) + 1.);
    for (long n = 1; n <= nstep; n++) {
      double rho1 = rho_prev;
      double erre = sqrt(r2 + z2 * z2);
      double espo = exp((erre - radius) * delta_inv);
      double rho2 = roze / (espo + 1.);
      sum1 = sum1 + rho1;
      sum2 = sum2 + rho2;
      rho_prev = rho2;
      z1 = z2;
      z2 = z2 + dz;
    }
    (void)z1;
    ratio = fabs(2. * (sum2 - sum1) / (sum1 + sum2));
  }
  thick[nc - 1] = sum1 * dz;
  term[nc - 1] = r * sum1 * dz;
}

struct GlauberArgs {
  DevPhys P;
  int nx, ny, nz, nv, nmax;
  double x1, y1, z1, dx, dy, dz;
  double dr, amassa, sigma_in, ah, b1, ecenter, rhocenter, weightbin, weightwound;
  double deta, sigeta2_inv, gamma_col, beta_col, przero;
  const double* thick;
  double* v;
  unsigned long long* maxbits;
  int* bad;
};

__device__ __forceinline__ void wound_dev(const GlauberArgs& A, double xx, double yy, double b1, double& tA,
                                          double& tB, double& thplus, double& thminus) {
  double xs = xx + b1 * 0.5;
  double rad = sqrt(xs * xs + yy * yy);
  long ip = nint_f(rad / A.dr + 1);
  xs = xx - b1 * 0.5;
  rad = sqrt(xs * xs + yy * yy);
  long im = nint_f(rad / A.dr + 1);
  if (ip < 1 || ip > A.nmax || im < 1 || im > A.nmax) {
    *A.bad = 2;
    ip = ip < 1 ? 1 : (ip > A.nmax ? A.nmax : ip);
    im = im < 1 ? 1 : (im > A.nmax ? A.nmax : im);
  }
  thplus = A.thick[ip - 1];
  thminus = A.thick[im - 1];
  double a = A.sigma_in * thminus / A.amassa;
  a = pow(1. - a, A.amassa);
  a = 1. - a;
  tA = a * thplus;
  double b = A.sigma_in * thplus / A.amassa;
  b = pow(1. - b, A.amassa);
  b = 1. - b;
  tB = b * thminus;
}

__global__ void __launch_bounds__(256) glauber_kernel(GlauberArgs A) {
  __shared__ double red[8];
  const size_t ncell = (size_t)A.nx * A.ny * A.nz;
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double ed = 0.;
  if (c < ncell) {
    const int i = (int)(c % A.nx);
    const int j = (int)((c / A.nx) % A.ny);
    const int k = (int)(c / ((size_t)A.nx * A.ny));
    const double xx = A.x1 + (i + 1 - 0.5) * A.dx, yy = A.y1 + (j + 1 - 0.5) * A.dy;
    double tt1, tt2, thp, thm;
    wound_dev(A, xx, yy, A.b1, tt1, tt2, thp, thm);
    const double bc = A.sigma_in * thp * thm;
    ed = A.ecenter * (A.ah * bc + (1. - A.ah) * (tt1 + tt2)) /
         ((A.ah * A.weightbin) + ((1 - A.ah) * A.weightwound));
    if (A.nz > 1) {  // H_of_eta, init.f90:933-967 (no tilting)
      const double eta = A.z1 + (k + 1 - 0.5) * A.dz;
      const double eta0 =
          0.5 * log(((thm + thp) * A.gamma_col + (thm - thp) * A.gamma_col * A.beta_col) /
                    ((thm + thp) * A.gamma_col - (thm - thp) * A.gamma_col * A.beta_col));
      const double d = fabs(eta - eta0);
      double H = 1.0;
      if (d > (A.deta * 0.5)) {
        const double q = d - (0.5 * A.deta);
        H = exp(-1.0 * (q * q) * 0.5 * A.sigeta2_inv);
      }
      ed = H * ed;
    }
    // initio (init.f90:852-893): rho, v = 0, p = p(e) + przero
    double pr = 0., d1 = 0., d2 = 0.;
    if (eos_pressure(A.P, A.rhocenter, ed, &pr, &d1, &d2)) *A.bad = 3;
    pr = pr + A.przero;
    for (int q = 0; q < A.nv; q++) A.v[(size_t)q * ncell + c] = 0.;
    A.v[(size_t)KRH * ncell + c] = A.rhocenter;
    A.v[(size_t)KPR * ncell + c] = pr;
  }
  block_max_atomic(ed, A.maxbits, red);
}

}  // namespace

#define GCK(x)                                                                              \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) {                                                                \
      fprintf(stderr, "echo_gpu: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                    \
      cudaFree(buf);                                                                        \
      return ECHO_ERR_CUDA;                                                                 \
    }                                                                                       \
  } while (0)

extern "C" int echo_gpu_optical_glauber(EchoCtx* c, const EchoOpticalGlauber* g, double t, double* check_mass,
                                        double* max_e) {
  (void)cudaGetLastError();
  if (!c || !g || !(g->dr > 0.) || !(g->dz1 > 0.) || !(g->acc > 0.) || !(g->delta > 0.) || !(g->mass_number > 0.))
    return ECHO_ERR_ARG;
  if (c->g.nz > 1 && (!(g->sigeta > 0.) || !(g->sqrt_s > 2. * g->nucleon_mass) || !(g->nucleon_mass > 0.)))
    return ECHO_ERR_ARG;
  const EchoParams& p = c->p;
  const double largestx = fmax(fabs(p.x1), fabs(p.x2)) + g->bimpact;
  const double largesty = fmax(fabs(p.y1), fabs(p.y2));
  const double rmax = sqrt(largestx * largestx + largesty * largesty);
  const int nmax = (int)(rmax / g->dr) + 1;
  if (nmax < 1 || nmax > (1 << 26)) return ECHO_ERR_ARG;
  // one allocation: thick[nmax], term[nmax], max bits, bad flag
  double* buf = nullptr;
  GCK(cudaMalloc(&buf, sizeof(double) * (2 * (size_t)nmax + 2)));
  double* thick = buf;
  double* term = buf + nmax;
  unsigned long long* maxbits = (unsigned long long*)(buf + 2 * (size_t)nmax);
  int* bad = (int*)(buf + 2 * (size_t)nmax + 1);
  GCK(cudaMemsetAsync(buf + 2 * (size_t)nmax, 0, 2 * sizeof(double), c->stream));
  thickness_kernel<<<(unsigned)((nmax + 127) / 128), 128, 0, c->stream>>>(nmax, g->radius, g->delta, g->roze, g->dr,
                                                                          g->dz1, g->acc, thick, term, bad);
  GCK(cudaGetLastError());
  std::vector<double> h_term((size_t)nmax);
  double thick0 = 0.;
  int h_bad = 0;
  GCK(cudaMemcpyAsync(h_term.data(), term, sizeof(double) * nmax, cudaMemcpyDeviceToHost, c->stream));
  GCK(cudaMemcpyAsync(&thick0, thick, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  GCK(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  GCK(cudaStreamSynchronize(c->stream));
  if (h_bad) {
    cudaFree(buf);
    return ECHO_ERR_ARG;
  }
  // the check mass in the reference's order (init.f90:1211-1219)
  double check = 0.;
  for (int i = 0; i < nmax; i++) check = check + h_term[i];
  if (check_mass) *check_mass = check * 2 * 3.1415927 * g->dr;
  // weights of a b = 0 collision at the origin (init.f90:1805-1812): r = 0 is table point 1
  const double a0 = 1. - pow(1. - g->sigma_in * thick0 / g->mass_number, g->mass_number);
  const double weightbin = g->sigma_in * thick0 * thick0;
  const double weightwound = a0 * thick0 + a0 * thick0;
  GlauberArgs A;
  memset(&A, 0, sizeof(A));
  A.P = c->P;
  A.nx = c->g.nx;
  A.ny = c->g.ny;
  A.nz = c->g.nz;
  A.nv = c->nv;
  A.nmax = nmax;
  A.x1 = p.x1;
  A.y1 = p.y1;
  A.z1 = p.z1;
  A.dx = (p.x2 - p.x1) / p.nx;
  A.dy = (p.y2 - p.y1) / p.ny;
  A.dz = (p.z2 - p.z1) / p.nz;
  A.dr = g->dr;
  A.amassa = g->mass_number;
  A.sigma_in = g->sigma_in;
  A.ah = g->ah;
  A.b1 = g->bimpact;
  A.ecenter = g->ecenter;
  A.rhocenter = g->rhocenter;
  A.weightbin = weightbin;
  A.weightwound = weightwound;
  A.deta = g->deta;
  A.sigeta2_inv = c->g.nz > 1 ? 1. / (g->sigeta * g->sigeta) : 0.;
  A.gamma_col = c->g.nz > 1 ? g->sqrt_s / (2. * g->nucleon_mass) : 1.;
  A.beta_col = c->g.nz > 1 ? sqrt(1. - (1. / (A.gamma_col * A.gamma_col))) : 0.;
  A.przero = p.przero;
  A.thick = thick;
  A.v = c->d_v[1];  // staging: the upload below copies it into the current buffer
  A.maxbits = maxbits;
  A.bad = bad;
  glauber_kernel<<<(unsigned)((c->g.ncell + 255) / 256), 256, 0, c->stream>>>(A);
  GCK(cudaGetLastError());
  unsigned long long mb = 0;
  GCK(cudaMemcpyAsync(&mb, maxbits, sizeof(mb), cudaMemcpyDeviceToHost, c->stream));
  GCK(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  GCK(cudaStreamSynchronize(c->stream));
  if (h_bad) {
    cudaFree(buf);
    return ECHO_ERR_ARG;
  }
  if (max_e) memcpy(max_e, &mb, sizeof(double));
  int r = echo_gpu_upload_device(c, c->d_v[1], nullptr, t);
  cudaFree(buf);
  return r;
}
