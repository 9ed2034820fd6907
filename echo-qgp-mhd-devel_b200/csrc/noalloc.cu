// noalloc.cu -- echo_gpu_rhs_noalloc: the right-hand side of one explicit
// stage (what echo_gpu_rhs computes) for callers that cannot allocate device
// memory.
//
// Who they are: a host code coupled to this library inside a larger GPU
// application whose memory is owned by another allocator (a framework's
// caching pool or a coupled solver that reserves HBM up front), where a
// cudaMalloc from here would either fail or fragment that pool; and drivers
// that must not allocate between CUDA-graph captures.  They pass their own
// device buffers for the inputs and the output; the only other memory this
// entry point needs -- the face fluxes of the three sweeps and the run
// scalars -- lives in file-scope __device__ arrays of fixed size that every
// GPU that loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/echo_gpu.h"
#include "ctx.cuh"

using namespace echo;

// Face-flux scratch: nv * (faces_x + faces_y + faces_z) doubles, plus 8 per
// face for the viscous u^mu states.  32 MiB.
static __device__ __align__(256) double g_noalloc_scratch[ECHO_NOALLOC_SCRATCH_DOUBLES];
static __device__ __align__(256) DevScalars g_noalloc_scalars;

// Device addresses of the two arrays, looked up once per device.  In host
// code the symbols above are host-side stand-ins, not device addresses: a
// kernel must be given the address cudaGetSymbolAddress returns.
static double* s_scratch[64];
static DevScalars* s_scalars[64];

static __global__ void noalloc_reset_scalars(DevScalars* sc, double t, double t3, double g3) {
  // every field a kernel of the stage reads starts from the state a fresh
  // upload leaves (echo.f90:141-144; glm_ch_old = 0.5, common.f90:283)
  memset(sc, 0, sizeof(DevScalars));
  sc->t = t;
  sc->t3 = t3;
  sc->tout = 1e300;
  sc->dtout = 1e300;
  sc->tmax = 1e300;
  sc->timeold = t;
  sc->g3old = g3;
  sc->glm_ch_old = 0.5;
  sc->err_key = ~0ull;
}

extern "C" int echo_gpu_rhs_noalloc(const EchoParams* p, const double* d_eos_cols, int n_eos, double t,
                                    const double* d_v, double* d_du, void* stream, int* errcode) {
  if (!p || !d_v || !d_du) return ECHO_ERR_ARG;
  {
    // the checks echo_gpu_init makes (equation set, integrator, grid, table)
    int r = echo_check_params(p, d_eos_cols, n_eos);
    if (r) return r;
  }
  if (p->mhd == 2) return ECHO_ERR_UNSUPPORTED;  // resistive runs: stage right-hand sides need the SSP state
  if (errcode) {
    // reading the error code back synchronises the stream, which a stream
    // being captured into a graph does not allow
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing((cudaStream_t)stream, &cs) != cudaSuccess) return ECHO_ERR_CUDA;
    if (cs != cudaStreamCaptureStatusNone) return ECHO_ERR_ARG;
  }
  int kind = p->viscosity ? KIND_VISC : p->mhd ? (p->divclean ? KIND_MHDGLM : KIND_MHD) : KIND_HD;
  int nv = kind == KIND_VISC ? 12 : kind == KIND_MHD ? 8 : kind == KIND_MHDGLM ? 9 : 5;
  size_t nf[3] = {(size_t)(p->nx + 1) * p->ny * p->nz, (size_t)p->nx * (p->ny + 1) * p->nz,
                  (size_t)p->nx * p->ny * (p->nz + 1)};
  int n[3] = {p->nx, p->ny, p->nz};
  size_t need = 0;
  for (int d = 0; d < 3; d++)
    if (n[d] > 1) need += nf[d] * (size_t)(nv + (kind == KIND_VISC ? 8 : 0));
  if (need > (size_t)ECHO_NOALLOC_SCRATCH_DOUBLES) {
    fprintf(stderr,
            "echo_gpu_rhs_noalloc: grid %dx%dx%d with nv=%d needs %zu doubles of face scratch, "
            "more than the fixed %d\n",
            p->nx, p->ny, p->nz, nv, need, ECHO_NOALLOC_SCRATCH_DOUBLES);
    return ECHO_ERR_ARG;
  }

  // once per device, with that device current: the device addresses of the
  // scratch arrays (documented: make the first call before any stream capture)
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ECHO_ERR_CUDA;
  if (!s_scratch[dev]) {
    void* a = nullptr;
    void* b = nullptr;
    cudaError_t e1 = cudaGetSymbolAddress(&a, g_noalloc_scratch);
    cudaError_t e2 = cudaGetSymbolAddress(&b, g_noalloc_scalars);
    if (e1 != cudaSuccess || e2 != cudaSuccess || !a || !b) {
      fprintf(stderr, "echo_gpu_rhs_noalloc: cudaGetSymbolAddress failed: %s\n",
              cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
      return ECHO_ERR_CUDA;
    }
    s_scratch[dev] = (double*)a;
    s_scalars[dev] = (DevScalars*)b;
  }

  // a context on the host stack that points at the caller's buffers and the
  // static scratch; nothing in it is allocated
  EchoCtx c;
  memset(&c, 0, sizeof(c));
  c.p = *p;
  c.kind = kind;
  c.nv = nv;
  c.g.nx = p->nx;
  c.g.ny = p->ny;
  c.g.nz = p->nz;
  c.g.ncell = (size_t)p->nx * p->ny * p->nz;
  double dx = (p->x2 - p->x1) / p->nx, dy = (p->y2 - p->y1) / p->ny, dz = (p->z2 - p->z1) / p->nz;
  c.g.ddx = p->nx > 1 ? 1. / dx : 0.;
  c.g.ddy = p->ny > 1 ? 1. / dy : 0.;
  c.g.ddz = p->nz > 1 ? 1. / dz : 0.;
  set_grid_div(c.g);
  for (int d = 0; d < 3; d++) {
    int uni = 1, sgn = 0;
    for (int k = 0; k < ECHO_MAX_NV; k++)
      for (int s = 0; s < 2; s++) c.bc[d].c[k][s] = (signed char)p->ibc[k][s][d];
    for (int k = 0; k < nv; k++)
      for (int s = 0; s < 2; s++) {
        int code = p->ibc[k][s][d];
        if (code != p->ibc[0][s][d] || code == 3 || code < -1 || code > 3) uni = 0;
        if (code == -1) sgn = 1;
      }
    c.bc_uniform[d] = uni;
    c.bc_signed[d] = sgn;
    c.nfaces[d] = nf[d];
  }
  double* cur = s_scratch[dev];
  for (int d = 0; d < 3; d++) {
    if (n[d] > 1) {
      c.d_F[d] = cur;
      cur += nf[d] * nv;
      if (kind == KIND_VISC) {
        c.d_WD[d] = cur;
        cur += nf[d] * 8;
      }
    }
  }
  c.d_v[0] = const_cast<double*>(d_v);
  c.vcur = 0;
  c.d_sc = s_scalars[dev];
  c.stream = (cudaStream_t)stream;
  c.P.eqstate = p->eqstate;
  c.P.coordinates = p->coordinates;
  c.P.recal = p->recal;
  c.P.obtained_zz = p->obtained_zz;
  c.P.init_type = p->init_type;
  c.P.bulkvis = p->bulkvis;
  if (p->eqstate == ECHO_EOS_TABLE || (d_eos_cols && n_eos > 0)) {
    c.P.nt = n_eos;
    c.P.tT = d_eos_cols;
    c.P.te = d_eos_cols + n_eos;
    c.P.tp = d_eos_cols + 2 * n_eos;
    c.P.tc = d_eos_cols + 3 * n_eos;
  }
  c.P.bke = c.P.bkp = nullptr;  // plain bracket search: same brackets, no accelerator table
  c.P.sl_ep = c.P.sl_ce = c.P.sl_pe = nullptr;  // interpolation with divisions
  c.P.maxspeed = p->maxspeed;
  c.P.eta_over_s = p->eta_over_s;
  c.P.tau_pi_coeff = p->tau_pi_coeff;
  c.P.enezero = p->enezero;
  c.P.przero = p->przero;
  c.P.glm_alpha = p->glm_alpha;

  (void)cudaGetLastError();
  double g3 = p->coordinates == ECHO_BJORKEN ? t * t : 1.;
  noalloc_reset_scalars<<<1, 1, 0, c.stream>>>(c.d_sc, t, pow(t, 3.), g3);
  for (int d = 0; d < 3; d++) {
    if (n[d] <= 1) continue;
    switch (kind) {
      case KIND_HD: launch_faces<KIND_HD>(&c, d); break;
      case KIND_VISC: launch_faces<KIND_VISC>(&c, d); break;
      case KIND_MHD: launch_faces<KIND_MHD>(&c, d); break;
      default: launch_faces<KIND_MHDGLM>(&c, d); break;
    }
  }
  switch (kind) {
    case KIND_HD: launch_update<KIND_HD>(&c, 1, MODE_RHS, d_du); break;
    case KIND_VISC: launch_update<KIND_VISC>(&c, 1, MODE_RHS, d_du); break;
    case KIND_MHD: launch_update<KIND_MHD>(&c, 1, MODE_RHS, d_du); break;
    default: launch_update<KIND_MHDGLM>(&c, 1, MODE_RHS, d_du); break;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "echo_gpu_rhs_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return ECHO_ERR_CUDA;
  }
  if (errcode) {
    unsigned long long key = ~0ull;
    e = cudaMemcpyAsync(&key, &c.d_sc->err_key, sizeof(key), cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) return ECHO_ERR_CUDA;
    *errcode = key == ~0ull ? 0 : (int)(key & 0xFFFFFull);
  }
  return ECHO_OK;
}
