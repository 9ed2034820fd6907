// output.cu -- output staging in the reference's binary layout: the bytes of
// one outNNNN.dat of out_vars (out.f90:232-591) -- t, then every selected
// field over the grid in Fortran order -- assembled on the device from the
// current primitives and copied once to host memory.
//
// One thread per cell computes every selected field of its cell (derived
// data from the EoS table, pi^{t mu}, the Lorentz factor, the ideal E) and
// stores it at field*ncell + cell in double or single precision; the
// header (t) is written by thread 0.  Coalesced: consecutive threads write
// consecutive cells of each field.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../include/echo_gpu.h"
#include "ctx.cuh"

using namespace echo;

#define CK(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) {                                                                    \
      fprintf(stderr, "echo_out: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                        \
      return ECHO_ERR_CUDA;                                                                     \
    }                                                                                           \
  } while (0)

namespace {

enum { OUT_NFIELD = 27 };

// field k of the output is bit k of sel, in the reference's write order;
// viscous fields need a viscous run, B and E an MHD run, psi also divclean
bool out_field_on(const EchoParams* p, unsigned sel, int k) {
  if (!(sel >> k & 1u)) return false;
  if (k >= 8 && k <= 18) return p->viscosity != 0;
  if (k >= 20 && k <= 25) return p->mhd != 0;
  if (k == 26) return p->mhd != 0 && p->divclean != 0;
  return k < OUT_NFIELD;
}

struct OutArgs {
  DevPhys P;
  Grid g;
  const double* __restrict__ v;
  const DevScalars* sc;
  unsigned char* out;
  unsigned long long* err_key;
  int coordinates, nf, prec, derived, obtained_zz, mhd;
  signed char fields[OUT_NFIELD];
};

template <int KIND>
__global__ void __launch_bounds__(256) out_pack_kernel(OutArgs A) {
  typedef Traits<KIND> T;
  const size_t nc = A.g.ncell;
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c == 0) {
    if (A.prec == 8) {
      double t = A.sc->t;
      memcpy(A.out, &t, 8);
    } else {
      float t = (float)A.sc->t;
      memcpy(A.out, &t, 4);
    }
  }
  if (c >= nc) return;
  const Metric M = make_metric(A.coordinates, A.sc->t, A.sc->t3);
  double p[T::NV];
#pragma unroll
  for (int k = 0; k < T::NV; k++) p[k] = A.v[(size_t)k * nc + c];
  double en = 0., temp = 0., sd = 0.;
  if (A.derived) {
    int err = get_derived_data(A.P, p[KRH], p[KPR], &en, &temp, &sd);
    if (err) atomicMin(A.err_key, ((unsigned long long)c << 20) | (unsigned long long)err);
  }
  Pit pi = {0, 0, 0, 0, 0};
  if (T::VISC) {
    if (A.obtained_zz)
      derived_pi_zz(M, p, pi);
    else
      derived_pi(M, p, pi);
  }
  double E[3] = {0., 0., 0.};
  if (T::MHD && !T::RES) e_ideal(M, p[KVX], p[KVY], p[KVZ], p[KBX], p[KBY], p[KBZ], E);
  for (int f = 0; f < A.nf; f++) {
    double x = 0.;
    switch (A.fields[f]) {
      case 0: x = p[KRH]; break;
      case 1: x = p[KVX]; break;
      case 2: x = p[KVY]; break;
      case 3: x = p[KVZ]; break;
      case 4: x = p[KPR]; break;
      case 5: x = en; break;
      case 6: x = temp; break;
      case 7: x = sd; break;
      case 19: x = 1. / sqrt(1. - p[KVX] * p[KVX] * M.g1 - p[KVY] * p[KVY] * M.g2 - p[KVZ] * p[KVZ] * M.g3); break;
      default:
        if constexpr (T::VISC) {
          switch (A.fields[f]) {
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
            default: x = A.obtained_zz ? pi.zz : p[KPIZZ]; break;
          }
        } else if constexpr (T::MHD) {
          switch (A.fields[f]) {
            case 20: x = p[KBX]; break;
            case 21: x = p[KBY]; break;
            case 22: x = p[KBZ]; break;
            case 23: x = T::RES ? p[T::RES ? KEX : 0] : E[0]; break;
            case 24: x = T::RES ? p[T::RES ? KEY : 0] : E[1]; break;
            case 25: x = T::RES ? p[T::RES ? KEZ : 0] : E[2] / M.g3; break;
            default: x = T::GLM ? p[T::GLM ? T::KG : 0] : 0.; break;
          }
        }
        break;
    }
    const size_t at = (size_t)A.prec + ((size_t)f * nc + c) * (size_t)A.prec;
    if (A.prec == 8)
      *reinterpret_cast<double*>(A.out + at) = x;
    else
      *reinterpret_cast<float*>(A.out + at) = (float)x;
  }
}

int out_layout(const EchoCtx* c, unsigned sel, int precision, signed char* fields, int* nf, size_t* bytes) {
  if (precision != 4 && precision != 8) return ECHO_ERR_ARG;
  if (sel >> OUT_NFIELD) return ECHO_ERR_ARG;
  int n = 0;
  for (int k = 0; k < OUT_NFIELD; k++)
    if (out_field_on(&c->p, sel, k)) fields[n++] = (signed char)k;
  *nf = n;
  *bytes = (size_t)precision + (size_t)n * c->g.ncell * (size_t)precision;
  return ECHO_OK;
}

}  // namespace

extern "C" int echo_gpu_out_vars_size(const EchoCtx* c, unsigned sel, int precision, size_t* bytes) {
  if (!c || !bytes) return ECHO_ERR_ARG;
  signed char fields[OUT_NFIELD];
  int nf = 0;
  return out_layout(c, sel, precision, fields, &nf, bytes);
}

extern "C" int echo_gpu_out_vars(EchoCtx* c, unsigned sel, int precision, void* buf, size_t bytes, int* errcode) {
  if (!c || !buf || !errcode) return ECHO_ERR_ARG;
  OutArgs A;
  size_t need = 0;
  int r = out_layout(c, sel, precision, A.fields, &A.nf, &need);
  if (r) return r;
  if (bytes < need) return ECHO_ERR_ARG;
  if (c->out_bytes < need) {
    cudaFree(c->d_out);
    c->d_out = nullptr;
    c->out_bytes = 0;
    CK(cudaMalloc(&c->d_out, need));
    c->out_bytes = need;
  }
  if (!c->d_out_err) CK(cudaMalloc(&c->d_out_err, sizeof(unsigned long long)));
  CK(cudaMemsetAsync(c->d_out_err, 0xff, sizeof(unsigned long long), c->stream));
  A.P = c->P;
  A.g = c->g;
  A.v = c->d_v[c->vcur];
  A.sc = c->d_sc;
  A.out = (unsigned char*)c->d_out;
  A.err_key = c->d_out_err;
  A.coordinates = c->p.coordinates;
  A.prec = precision;
  A.derived = (sel & (ECHO_OUT_ENERGY_DENSITY | ECHO_OUT_TEMPERATURE | ECHO_OUT_ENTROPY_DENSITY)) != 0;
  A.obtained_zz = c->p.obtained_zz;
  A.mhd = c->p.mhd;
  unsigned blocks = (unsigned)((c->g.ncell + 255) / 256);
  switch (c->kind) {
    case KIND_HD: out_pack_kernel<KIND_HD><<<blocks, 256, 0, c->stream>>>(A); break;
    case KIND_VISC: out_pack_kernel<KIND_VISC><<<blocks, 256, 0, c->stream>>>(A); break;
    case KIND_MHD: out_pack_kernel<KIND_MHD><<<blocks, 256, 0, c->stream>>>(A); break;
    case KIND_RES: out_pack_kernel<KIND_RES><<<blocks, 256, 0, c->stream>>>(A); break;
    default: out_pack_kernel<KIND_MHDGLM><<<blocks, 256, 0, c->stream>>>(A); break;
  }
  CK(cudaGetLastError());
  unsigned long long key = 0;
  CK(cudaMemcpyAsync(buf, c->d_out, need, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&key, c->d_out_err, sizeof(key), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *errcode = key == ~0ull ? 0 : (int)(key & 0xfffffull);
  return ECHO_OK;
}

void echo_out_free(EchoCtx* c) {
  cudaFree(c->d_out);
  cudaFree(c->d_out_err);
  c->d_out = nullptr;
  c->d_out_err = nullptr;
  c->out_bytes = 0;
}
