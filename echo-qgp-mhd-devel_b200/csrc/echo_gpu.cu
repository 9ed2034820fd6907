// echo_gpu.cu -- context management and the C-ABI entry points of
// include/echo_gpu.h.  One CUDA stream per context; every stage is a fixed
// sequence of launches with no host synchronisation, so whole steps are
// captured into a CUDA graph (echo_gpu_run).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/echo_gpu.h"
#include "ctx.cuh"

using namespace echo;

#define CK(x)                                                                               \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) {                                                                \
      fprintf(stderr, "echo_gpu: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                    \
      return ECHO_ERR_CUDA;                                                                 \
    }                                                                                       \
  } while (0)

bool echo_make_buckets(const double* arr, int n, std::vector<int>& bk, long long& k0) {
  if (n < 2 || !(arr[0] > 0.0)) return false;
  for (int i = 1; i < n; i++)
    if (!(arr[i] > arr[i - 1])) return false;
  long long b0, b1;
  memcpy(&b0, &arr[0], 8);
  memcpy(&b1, &arr[n - 1], 8);
  k0 = b0 >> BK_SHIFT;
  long long nb = (b1 >> BK_SHIFT) - k0 + 1;
  if (nb > (1 << 22)) return false;
  bk.resize((size_t)nb);
  int i = 1;  // 1-based
  for (long long b = 0; b < nb; b++) {
    long long bits = (k0 + b) << BK_SHIFT;
    double lo;
    memcpy(&lo, &bits, 8);
    while (i < n && arr[i - 1] < lo) i++;
    bk[(size_t)b] = i < 2 ? 2 : i;
  }
  return true;
}

int echo_kind_of(const EchoParams* p) {
  if (p->viscosity) return KIND_VISC;
  if (p->mhd == 2) return KIND_RES;
  if (p->mhd) return p->divclean ? KIND_MHDGLM : KIND_MHD;
  return KIND_HD;
}
int echo_nv_of(int kind) {
  switch (kind) {
    case KIND_VISC: return 12;
    case KIND_RES: return 12;
    case KIND_MHD: return 8;
    case KIND_MHDGLM: return 9;
    default: return 5;
  }
}

// boundary codes of every variable and direction (ibc, init.f90:137-155)
void echo_setup_bc(const EchoParams* p, int nv, BcDir bc[3], int uniform[3], int sign[3]) {
  for (int d = 0; d < 3; d++)
    for (int k = 0; k < ECHO_MAX_NV; k++)
      for (int s = 0; s < 2; s++) bc[d].c[k][s] = (signed char)p->ibc[k][s][d];
  for (int d = 0; d < 3; d++) {
    int uni = 1, sgn = 0;
    for (int k = 0; k < nv; k++)
      for (int q = 0; q < 2; q++) {
        int code = p->ibc[k][q][d];
        if (code != p->ibc[0][q][d] || code == 3 || code < -1 || code > 3) uni = 0;
        if (code == -1) sgn = 1;
      }
    uniform[d] = uni;
    sign[d] = sgn;
  }
}

// physics constants and the EoS table on the device (eos.f90:265-334)
int echo_setup_phys(const EchoParams* p, const double* eos_table, int n_eos, DevPhys* P, double** d_tab,
                    int** d_bk) {
  *d_tab = nullptr;
  int nt = 0;
  if (eos_table && n_eos > 0) {
    // columns T, e, p, c_s^2, then the interval slopes de/dp, d(c_s^2)/de
    // and dp/de = (dp/dT)/(de/dT) (get_pressure's derivative, eos.f90:458-462)
    nt = n_eos;
    std::vector<double> cols((size_t)7 * n_eos, 0.0);
    for (int i = 0; i < n_eos; i++)
      for (int q = 0; q < 4; q++) cols[(size_t)q * n_eos + i] = eos_table[4 * i + q];
    for (int i = 0; i + 1 < n_eos; i++) {
      const double* a = eos_table + 4 * i;
      const double* b = a + 4;
      cols[(size_t)4 * n_eos + i] = (b[1] - a[1]) / (b[2] - a[2]);
      cols[(size_t)5 * n_eos + i] = (b[3] - a[3]) / (b[1] - a[1]);
      cols[(size_t)6 * n_eos + i] = ((b[2] - a[2]) / (b[0] - a[0])) / ((b[1] - a[1]) / (b[0] - a[0]));
    }
    CK(cudaMalloc(d_tab, sizeof(double) * 7 * n_eos));
    CK(cudaMemcpy(*d_tab, cols.data(), sizeof(double) * 7 * n_eos, cudaMemcpyHostToDevice));
  }
  P->eqstate = p->eqstate;
  P->coordinates = p->coordinates;
  P->recal = p->recal;
  P->obtained_zz = p->obtained_zz;
  P->init_type = p->init_type;
  P->bulkvis = p->bulkvis;
  P->nt = nt;
  P->tT = *d_tab;
  P->te = *d_tab ? *d_tab + nt : nullptr;
  P->tp = *d_tab ? *d_tab + 2 * nt : nullptr;
  P->tc = *d_tab ? *d_tab + 3 * nt : nullptr;
  P->maxspeed = p->maxspeed;
  P->eta_over_s = p->eta_over_s;
  P->tau_pi_coeff = p->tau_pi_coeff;
  P->enezero = p->enezero;
  P->przero = p->przero;
  P->glm_alpha = p->glm_alpha;
  P->sigma_el = p->sigma_el;
  P->sigma_chiral = p->sigma_chiral;
  P->bke = P->bkp = nullptr;
  P->sl_ep = P->sl_ce = P->sl_pe = nullptr;
  *d_bk = nullptr;
  if (nt > 0) {
    std::vector<double> te(nt), tp(nt);
    for (int i = 0; i < nt; i++) {
      te[i] = eos_table[4 * i + 1];
      tp[i] = eos_table[4 * i + 2];
    }
    std::vector<int> be, bp;
    long long ke0 = 0, kp0 = 0;
    if (echo_make_buckets(te.data(), nt, be, ke0) && echo_make_buckets(tp.data(), nt, bp, kp0)) {
      CK(cudaMalloc(d_bk, sizeof(int) * (be.size() + bp.size())));
      CK(cudaMemcpy(*d_bk, be.data(), sizeof(int) * be.size(), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(*d_bk + be.size(), bp.data(), sizeof(int) * bp.size(), cudaMemcpyHostToDevice));
      P->bke = *d_bk;
      P->bkp = *d_bk + be.size();
      P->bke0 = ke0;
      P->bkp0 = kp0;
      P->nbke = (int)be.size();
      P->nbkp = (int)bp.size();
      // strictly increasing e and p: every interval has a finite slope
      P->sl_ep = *d_tab + 4 * nt;
      P->sl_ce = *d_tab + 5 * nt;
      P->sl_pe = *d_tab + 6 * nt;
    }
  }
  return ECHO_OK;
}

// whether the sweeps of a stage run concurrently (launch_sweeps)
#ifndef ECHO_PAR_SWEEPS
#define ECHO_PAR_SWEEPS 1
#endif

// how the product build's face sweeps run (echo_gpu_set_faces)
#ifndef ECHO_FACE_MODE
#define ECHO_FACE_MODE 0
#endif

#define DISPATCH(c, fn, ...)                                      \
  do {                                                            \
    switch ((c)->kind) {                                          \
      case KIND_HD: fn<KIND_HD>(__VA_ARGS__); break;              \
      case KIND_VISC: fn<KIND_VISC>(__VA_ARGS__); break;          \
      case KIND_MHD: fn<KIND_MHD>(__VA_ARGS__); break;            \
      case KIND_RES: fn<KIND_RES>(__VA_ARGS__); break;            \
      default: fn<KIND_MHDGLM>(__VA_ARGS__); break;               \
    }                                                             \
  } while (0)

static void launch_scalars(EchoCtx* c, int irk, int mode = 0) {
  ScalarArgs S;
  S.sc = c->d_sc;
  S.g = c->g;
  S.cfl = c->p.cfl;
  S.maxdt = c->p.maxdt;
  S.glm_alpha = c->p.glm_alpha;
  S.irk = irk;
  S.nrk = c->p.nrk;
  S.divclean = c->p.divclean;
  S.mode = mode;
  stage_scalars_kernel<<<1, 1, 0, c->stream>>>(S);
}

// The flux sweeps of a stage.  They are independent of each other: each
// reads v and writes its own face fluxes and its own signal-speed slots
// (amax_bits[d], aflux[d]).  With par_sweeps the first runs on `stream` and
// the others on the side streams, forked from and joined back into it, so
// that the partial last wave of one overlaps the others (under stream
// capture the fork and join become branches of the step graph).  Per-kernel
// profiling keeps them in order, so that each can be timed.
static void launch_sweeps(EchoCtx* c) {
  int dirs[3], nd = 0;
  for (int d = 0; d < 3; d++) {
    int n = d == 0 ? c->g.nx : d == 1 ? c->g.ny : c->g.nz;
    if (n > 1) dirs[nd++] = d;
  }
  if (!c->par_sweeps || c->marks || nd < 2) {
    for (int j = 0; j < nd; j++) {
      DISPATCH(c, launch_faces, c, dirs[j]);
      mark(c, PK_FACES_X + dirs[j]);
    }
    return;
  }
  cudaEventRecord(c->ev_fork, c->stream);
  const cudaStream_t main = c->stream;
  for (int j = 1; j < nd; j++) {
    cudaStreamWaitEvent(c->side[j - 1], c->ev_fork, 0);
    c->stream = c->side[j - 1];
    DISPATCH(c, launch_faces, c, dirs[j]);
    cudaEventRecord(c->ev_join[j - 1], c->stream);
  }
  c->stream = main;
  DISPATCH(c, launch_faces, c, dirs[0]);
  for (int j = 1; j < nd; j++) cudaStreamWaitEvent(c->stream, c->ev_join[j - 1], 0);
}

// the flux sweeps of a stage; the CFL maxima start from zero
static void enqueue_sweeps(EchoCtx* c) {
  cudaMemsetAsync(c->d_sc->amax_bits, 0, sizeof(unsigned long long) * 3, c->stream);
  launch_sweeps(c);
}

// IMEX-SSP3(4,3,3) stage (evolve.f90:204-267), all asynchronous
static void enqueue_stage_ssp(EchoCtx* c, int irk) {
  if (irk == 1) {
    launch_scalars(c, 1, 1);  // dt from the previous stage's speeds
  } else {
    if (irk == 2) c->ucur = 1 - c->ucur;  // U[ucur] becomes the u built from u0 = U[1-ucur]
    cudaMemsetAsync(&c->d_sc->nfail, 0, sizeof(int), c->stream);
    cudaMemsetAsync(&c->d_sc->c2p_iters, 0, sizeof(unsigned long long), c->stream);
    DISPATCH(c, launch_ssp_combine, c, irk);
    mark(c, PK_UPDATE);
    // smoothing at the end of these stages would act only on values the next
    // combination overwrites, so the reference's smoothing survives only
    // after the final combination
    DISPATCH(c, launch_repair_smooth, c, 1);
    mark(c, PK_REPAIR);
    c->vcur = 1 - c->vcur;
  }
  if (c->st_ok && c->st_on) {
    // sweeps + right-hand side in one kernel; the GLM scalars after it (the
    // right-hand side reads none of them)
    cudaMemsetAsync(c->d_sc->amax_bits, 0, sizeof(unsigned long long) * 3, c->stream);
    DISPATCH(c, launch_stage, c, irk, MODE_RHS, c->d_dussp[irk - 1]);
    mark(c, PK_STAGE);
    launch_scalars(c, irk, 2);
    mark(c, PK_SCALARS);
  } else {
    enqueue_sweeps(c);
    launch_scalars(c, irk, 2);
    mark(c, PK_SCALARS);
    DISPATCH(c, launch_update, c, irk, MODE_RHS, c->d_dussp[irk - 1]);
    mark(c, PK_UPDATE);
  }
  if (irk == 1 && c->kind == KIND_RES) {
    DISPATCH(c, launch_ssp_stage1, c);
    mark(c, PK_UPDATE);
  }
  if (irk == 4) {
    cudaMemsetAsync(&c->d_sc->nfail, 0, sizeof(int), c->stream);
    DISPATCH(c, launch_ssp_combine, c, 5);
    mark(c, PK_UPDATE);
    DISPATCH(c, launch_repair_smooth, c, 3);
    mark(c, PK_REPAIR);
    c->vcur = 1 - c->vcur;
  }
}

// one explicit RK stage, all asynchronous
// the stream waits for the host copy of u of echo_gpu_advance_host
static void join_u(EchoCtx* c) {
  cudaStreamWaitEvent(c->stream, c->ev_u, 0);
  c->wait_u = 0;
}

static void enqueue_stage(EchoCtx* c, int irk) {
  if (c->p.nrk == ECHO_SSP) {
    enqueue_stage_ssp(c, irk);
    return;
  }
  cudaMemsetAsync(c->d_sc->amax_bits, 0, sizeof(unsigned long long) * 3, c->stream);
  // the fused stage needs dt before the faces: every stage but the first,
  // and the first with divergence cleaning (dt = CFL, evolve.f90:734-735)
  if (c->st_ok && c->st_on && (irk > 1 || c->p.divclean)) {
    launch_scalars(c, irk, 3);
    cudaMemsetAsync(&c->d_sc->nfail, 0, sizeof(int), c->stream);
    cudaMemsetAsync(&c->d_sc->c2p_iters, 0, sizeof(unsigned long long), c->stream);
    mark(c, PK_SCALARS);
    DISPATCH(c, launch_stage, c, irk, MODE_RK, (double*)nullptr);
    mark(c, PK_STAGE);
    launch_scalars(c, irk, 4);
    mark(c, PK_SCALARS);
  } else {
    launch_sweeps(c);
    if (c->wait_u) join_u(c);  // the update reads u
    launch_scalars(c, irk);
    cudaMemsetAsync(&c->d_sc->nfail, 0, sizeof(int), c->stream);
    cudaMemsetAsync(&c->d_sc->c2p_iters, 0, sizeof(unsigned long long), c->stream);
    mark(c, PK_SCALARS);
    DISPATCH(c, launch_update, c, irk, MODE_RK, (double*)nullptr);
    mark(c, PK_UPDATE);
  }
  // stage 1 wrote the new u into the other buffer: it becomes current before
  // the repair and the smoothing, which act on the new u
  if (irk == 1) c->ucur = 1 - c->ucur;
  DISPATCH(c, launch_repair_smooth, c, 3);
  mark(c, PK_REPAIR);
  c->vcur = 1 - c->vcur;
}

static void snapshot_vnewstep(EchoCtx* c) {
  // vnewstep = v (echo.f90:193-201); only the viscous time derivatives read it
  if (c->p.viscosity)
    cudaMemcpyAsync(c->d_vh[c->vn], c->d_v[c->vcur], sizeof(double) * c->g.ncell * 4, cudaMemcpyDeviceToDevice,
                    c->stream);
  if (c->keep_old) {  // the full vnewstep / unewstep of the reference, for dump.dat
    size_t b = sizeof(double) * c->g.ncell * c->kold;
    cudaMemcpyAsync(c->d_oldv[c->on], c->d_v[c->vcur], b, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(c->d_oldu[c->on], c->d_u[c->ucur], b, cudaMemcpyDeviceToDevice, c->stream);
  }
}

// end of step: vold = vnewstep, uold = unewstep (echo.f90:240-241) are role swaps
static void end_step(EchoCtx* c) {
  end_step_kernel<<<1, 1, 0, c->stream>>>(c->d_sc, c->p.coordinates);
  mark(c, PK_END);
  if (c->p.viscosity) c->vn = 1 - c->vn;
  if (c->keep_old) c->on = 1 - c->on;
}

static void enqueue_step(EchoCtx* c) {
  // a host copy of u still in flight (echo_gpu_advance_host): the explicit
  // RK stages wait for it after their first sweeps, which read v only; the
  // other paths touch u at once
  if (c->wait_u && (c->keep_old || c->p.nrk == ECHO_SSP || (c->st_ok && c->st_on))) join_u(c);
  snapshot_vnewstep(c);
  for (int irk = 1; irk <= c->p.nrk; irk++) enqueue_stage(c, irk);
  end_step(c);
  if (c->wait_u) join_u(c);
}

// the role changes of enqueue_step without launching anything
static void advance_roles(EchoCtx* c) {
  c->ucur = 1 - c->ucur;
  c->vcur = c->vcur ^ (c->p.nrk & 1);
  if (c->p.viscosity) c->vn = 1 - c->vn;
  if (c->keep_old) c->on = 1 - c->on;
}

// The parameter checks of a run, shared by every entry point that takes an
// EchoParams: equation set, integrator, grid and EoS table.
int echo_check_params(const EchoParams* p, const double* eos_table, int n_eos) {
  if (!p) return ECHO_ERR_ARG;
  if (p->mhd > 2 || (p->mhd && p->viscosity)) return ECHO_ERR_UNSUPPORTED;
  if (p->nrk != ECHO_RK2 && p->nrk != ECHO_RK3 && p->nrk != ECHO_SSP) return ECHO_ERR_UNSUPPORTED;
  // resistive runs: IMEX-SSP (common.f90:2114-2118), with GLM cleaning
  if (p->mhd == 2 && (p->nrk != ECHO_SSP || !p->divclean))
    return ECHO_ERR_UNSUPPORTED;
  if (p->imex != 0 && p->imex != 1) return ECHO_ERR_ARG;
  if (p->imex && p->nrk == ECHO_SSP) return ECHO_ERR_UNSUPPORTED;  // IMEX RK2/RK3 only
  if (p->nx < 1 || p->ny < 1 || p->nz < 1) return ECHO_ERR_ARG;
  if ((p->nx > 1 && p->nx < 3) || (p->ny > 1 && p->ny < 3) || (p->nz > 1 && p->nz < 3)) return ECHO_ERR_ARG;
  if (p->eqstate == ECHO_EOS_TABLE && (!eos_table || n_eos < 2)) return ECHO_ERR_ARG;
  return ECHO_OK;
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

int echo_gpu_nv(const EchoCtx* c) { return c ? c->nv : 0; }

int echo_gpu_init(const EchoParams* p, const double* eos_table, int n_eos, EchoCtx** out) {
  if (!p || !out) return ECHO_ERR_ARG;
  *out = nullptr;
  {
    int r = echo_check_params(p, eos_table, n_eos);
    if (r) return r;
  }
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return ECHO_ERR_CUDA;
  EchoCtx* c = (EchoCtx*)calloc(1, sizeof(EchoCtx));
  c->p = *p;
  c->kind = echo_kind_of(p);
  c->nv = echo_nv_of(c->kind);
  c->g.nx = p->nx;
  c->g.ny = p->ny;
  c->g.nz = p->nz;
  c->g.ncell = (size_t)p->nx * p->ny * p->nz;
  double dx = (p->x2 - p->x1) / p->nx, dy = (p->y2 - p->y1) / p->ny, dz = (p->z2 - p->z1) / p->nz;
  c->g.ddx = p->nx > 1 ? 1. / dx : 0.;
  c->g.ddy = p->ny > 1 ? 1. / dy : 0.;
  c->g.ddz = p->nz > 1 ? 1. / dz : 0.;
  set_grid_div(c->g);
  echo_setup_bc(p, c->nv, c->bc, c->bc_uniform, c->bc_signed);
  c->nfaces[0] = (size_t)(p->nx + 1) * p->ny * p->nz;
  c->nfaces[1] = (size_t)p->nx * (p->ny + 1) * p->nz;
  c->nfaces[2] = (size_t)p->nx * p->ny * (p->nz + 1);
  size_t nvc = (size_t)c->nv * c->g.ncell;
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c->side[0], cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c->side[1], cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&c->ev_join[0], cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&c->ev_join[1], cudaEventDisableTiming));
  CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&c->ev_u, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&c->ev_u_fork, cudaEventDisableTiming));
  c->par_sweeps = ECHO_PAR_SWEEPS;
  for (int i = 0; i < 2; i++) {
    CK(cudaMalloc(&c->d_v[i], sizeof(double) * nvc));
    CK(cudaMalloc(&c->d_u[i], sizeof(double) * nvc));
    CK(cudaMemset(c->d_v[i], 0, sizeof(double) * nvc));
    CK(cudaMemset(c->d_u[i], 0, sizeof(double) * nvc));
  }
  for (int d = 0; d < 3; d++) {
    int n = d == 0 ? p->nx : d == 1 ? p->ny : p->nz;
    c->d_F[d] = nullptr;
    c->d_WD[d] = nullptr;
    if (n > 1) {
      CK(cudaMalloc(&c->d_F[d], sizeof(double) * c->nv * c->nfaces[d]));
      if (p->viscosity) CK(cudaMalloc(&c->d_WD[d], sizeof(double) * 8 * c->nfaces[d]));
    }
  }
  for (int i = 0; i < 2; i++) {
    CK(cudaMalloc(&c->d_vh[i], sizeof(double) * 4 * c->g.ncell));
    CK(cudaMemset(c->d_vh[i], 0, sizeof(double) * 4 * c->g.ncell));
  }
  for (int q = 0; q < 4; q++) {
    c->d_dussp[q] = nullptr;
    c->d_dss[q] = nullptr;
    if (p->nrk == ECHO_SSP) CK(cudaMalloc(&c->d_dussp[q], sizeof(double) * nvc));
    if (c->kind == KIND_RES) {
      CK(cudaMalloc(&c->d_dss[q], sizeof(double) * 3 * c->g.ncell));
      CK(cudaMemset(c->d_dss[q], 0, sizeof(double) * 3 * c->g.ncell));
    }
  }
  CK(cudaMalloc(&c->d_fail, c->g.ncell));
  CK(cudaMemset(c->d_fail, 0, c->g.ncell));
  CK(cudaMalloc(&c->d_sc, sizeof(DevScalars)));
  CK(cudaMallocHost(&c->h_sc, sizeof(DevScalars)));
  memset(c->h_sc, 0, sizeof(DevScalars));
  {
    int r = echo_setup_phys(p, eos_table, n_eos, &c->P, &c->d_tab, &c->d_bk);
    if (r) return r;
  }
  c->d_du = nullptr;
  c->marks = nullptr;
  c->d_mlp_frag = nullptr;
  c->d_mlp_par = nullptr;
  c->hyp = nullptr;
  c->d_out = nullptr;
  c->out_bytes = 0;
  c->d_out_err = nullptr;
  c->kold = p->mhd ? 8 : 5;  // krh..kvold_end: kbz with MHD, kpr without (common.f90:378-386)
#ifdef ECHO_EXACT
  c->face_mode = 0;  // the parity build keeps the reference's face-by-face arithmetic
#else
  c->face_mode = ECHO_FACE_MODE;
#endif
  // the fused stage kernel: tile chosen here, off until echo_gpu_set_stage
  DISPATCH(c, setup_stage, c, 0, 0, 0);
  c->st_on = 0;
  (void)cudaGetLastError();
  *out = c;
  return ECHO_OK;
}

int echo_gpu_free(EchoCtx* c) {
  if (!c) return ECHO_OK;
  cudaStreamSynchronize(c->stream);
  for (int i = 0; i < 16; i++)
    if (c->graph_ok[i]) cudaGraphExecDestroy(c->graph[i]);
  for (int i = 0; i < 2; i++) {
    cudaFree(c->d_v[i]);
    cudaFree(c->d_u[i]);
    cudaFree(c->d_vh[i]);
  }
  for (int d = 0; d < 3; d++) {
    cudaFree(c->d_F[d]);
    cudaFree(c->d_WD[d]);
  }
  for (int q = 0; q < 4; q++) {
    cudaFree(c->d_dussp[q]);
    cudaFree(c->d_dss[q]);
  }
  cudaFree(c->d_fail);
  cudaFree(c->d_sc);
  cudaFree(c->d_tab);
  cudaFree(c->d_bk);
  cudaFree(c->d_du);
  cudaFree(c->d_mlp_frag);
  cudaFree(c->d_mlp_par);
  for (int i = 0; i < 2; i++) {
    cudaFree(c->d_oldv[i]);
    cudaFree(c->d_oldu[i]);
  }
  cudaFreeHost(c->h_sc);
  echo_hyp_free(c->hyp);
  echo_out_free(c);
  cudaStreamDestroy(c->stream);
  cudaStreamDestroy(c->side[0]);
  cudaStreamDestroy(c->side[1]);
  cudaEventDestroy(c->ev_fork);
  cudaEventDestroy(c->ev_join[0]);
  cudaEventDestroy(c->ev_join[1]);
  cudaStreamDestroy(c->copy_stream);
  cudaEventDestroy(c->ev_u);
  cudaEventDestroy(c->ev_u_fork);
  free(c);
  return ECHO_OK;
}

static int reset_scalars(EchoCtx* c, double t) {
  DevScalars s;
  memset(&s, 0, sizeof(s));
  s.t = t;
  s.t3 = pow(t, 3.);
  s.dt = 0.;
  s.tout = 1e300;
  s.dtout = 1e300;
  s.tmax = 1e300;
  s.timeold = t;
  s.timeinterval = 0.;
  s.g3old = c->p.coordinates == ECHO_BJORKEN ? t * t : 1.;
  s.glm_ch_old = 0.5;  // common.f90:283
  s.err_key = ~0ull;
  CK(cudaMemcpyAsync(c->d_sc, &s, sizeof(s), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->d_vh[0], 0, sizeof(double) * 4 * c->g.ncell, c->stream));
  CK(cudaMemsetAsync(c->d_vh[1], 0, sizeof(double) * 4 * c->g.ncell, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ECHO_OK;
}

// vold = v, uold = u of the uploaded state (init.f90:3271-3272)
static int init_old(EchoCtx* c) {
  if (!c->keep_old) return ECHO_OK;
  size_t b = sizeof(double) * c->g.ncell * c->kold;
  CK(cudaMemcpyAsync(c->d_oldv[1 - c->on], c->d_v[c->vcur], b, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_oldu[1 - c->on], c->d_u[c->ucur], b, cudaMemcpyDeviceToDevice, c->stream));
  return ECHO_OK;
}

static int upload_impl(EchoCtx* c, const double* v, const double* u, double t, cudaMemcpyKind kind) {
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!c || !v) return ECHO_ERR_ARG;
  size_t bytes = sizeof(double) * c->nv * c->g.ncell;
  c->vcur = 0;
  c->ucur = 0;
  c->vn = 0;
  c->on = 0;
  int r = reset_scalars(c, t);
  if (r) return r;
  CK(cudaMemcpyAsync(c->d_v[0], v, bytes, kind, c->stream));
  if (u) {
    CK(cudaMemcpyAsync(c->d_u[0], u, bytes, kind, c->stream));
  } else {
    DISPATCH(c, launch_p2c, c);
  }
  r = init_old(c);
  if (r) return r;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  return ECHO_OK;
}

int echo_gpu_upload(EchoCtx* c, const double* v, const double* u, double t) {
  return upload_impl(c, v, u, t, cudaMemcpyHostToDevice);
}
int echo_gpu_upload_device(EchoCtx* c, const double* v, const double* u, double t) {
  return upload_impl(c, v, u, t, cudaMemcpyDeviceToDevice);
}

int echo_gpu_put_state(EchoCtx* c, const double* v, const double* u) {
  if (!c || !v || !u) return ECHO_ERR_ARG;
  size_t bytes = sizeof(double) * c->nv * c->g.ncell;
  CK(cudaMemcpyAsync(c->d_v[c->vcur], v, bytes, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_u[c->ucur], u, bytes, cudaMemcpyHostToDevice, c->stream));
  return ECHO_OK;
}

int echo_gpu_get_state(EchoCtx* c, double* v, double* u) {
  if (!c) return ECHO_ERR_ARG;
  size_t bytes = sizeof(double) * c->nv * c->g.ncell;
  if (v) CK(cudaMemcpyAsync(v, c->d_v[c->vcur], bytes, cudaMemcpyDeviceToHost, c->stream));
  if (u) CK(cudaMemcpyAsync(u, c->d_u[c->ucur], bytes, cudaMemcpyDeviceToHost, c->stream));
  return ECHO_OK;
}

static int download_impl(EchoCtx* c, double* v, double* u, cudaMemcpyKind kind) {
  if (!c) return ECHO_ERR_ARG;
  size_t bytes = sizeof(double) * c->nv * c->g.ncell;
  if (v) CK(cudaMemcpyAsync(v, c->d_v[c->vcur], bytes, kind, c->stream));
  if (u) CK(cudaMemcpyAsync(u, c->d_u[c->ucur], bytes, kind, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ECHO_OK;
}
int echo_gpu_download(EchoCtx* c, double* v, double* u) { return download_impl(c, v, u, cudaMemcpyDeviceToHost); }
int echo_gpu_download_device(EchoCtx* c, double* v, double* u) {
  return download_impl(c, v, u, cudaMemcpyDeviceToDevice);
}

int echo_gpu_set_tout(EchoCtx* c, double tout) {
  if (!c) return ECHO_ERR_ARG;
  CK(cudaMemcpyAsync(&c->d_sc->tout, &tout, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ECHO_OK;
}

static int read_scalars(EchoCtx* c) {
  CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  return ECHO_OK;
}

static int errcode_of(const DevScalars* s, int* cell) {
  if (s->err_key == ~0ull) {
    if (cell) *cell = -1;
    return 0;
  }
  if (cell) *cell = (int)(s->err_key >> 20);
  return (int)(s->err_key & 0xFFFFFull);
}

int echo_gpu_evolve_main(EchoCtx* c, int irk, double* dt, int* errcode) {
  if (c && c->p.algo_solver == ECHO_C2P_MLP && !c->d_mlp_frag) return ECHO_ERR_ARG;  // no network loaded
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!c || irk < 1 || irk > c->p.nrk) return ECHO_ERR_ARG;
  if (irk == 1) snapshot_vnewstep(c);
  enqueue_stage(c, irk);
  CK(cudaGetLastError());
  int r = read_scalars(c);
  if (r) return r;
  if (dt) *dt = c->h_sc->dt;
  if (errcode) *errcode = errcode_of(c->h_sc, nullptr);
  return ECHO_OK;
}

int echo_gpu_end_step(EchoCtx* c) {
  if (!c) return ECHO_ERR_ARG;
  end_step(c);
  CK(cudaGetLastError());
  return ECHO_OK;
}

int echo_gpu_step(EchoCtx* c, double* dt, int* errcode) {
  if (c && c->p.algo_solver == ECHO_C2P_MLP && !c->d_mlp_frag) return ECHO_ERR_ARG;  // no network loaded
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!c) return ECHO_ERR_ARG;
  enqueue_step(c);
  CK(cudaGetLastError());
  int r = read_scalars(c);
  if (r) return r;
  if (dt) *dt = c->h_sc->dt;
  if (errcode) *errcode = errcode_of(c->h_sc, nullptr);
  return ECHO_OK;
}

int echo_gpu_run(EchoCtx* c, int nsteps) {
  if (c && c->p.algo_solver == ECHO_C2P_MLP && !c->d_mlp_frag) return ECHO_ERR_ARG;  // no network loaded
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!c || nsteps < 0) return ECHO_ERR_ARG;
  for (int s = 0; s < nsteps; s++) {
    // buffer roles at step start: which u/v buffer is current and which
    // vnewstep/vold buffer is which; they repeat, so graphs are cached per key
    int key = c->ucur | (c->vcur << 1) | (c->vn << 2) | (c->on << 3);
    if (!c->graph_ok[key]) {
      cudaGraph_t gr;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      enqueue_step(c);  // records the launches and advances the roles
      CK(cudaStreamEndCapture(c->stream, &gr));
      CK(cudaGraphInstantiate(&c->graph[key], gr, 0));
      cudaGraphDestroy(gr);
      c->graph_ok[key] = true;
    } else {
      advance_roles(c);
    }
    CK(cudaGraphLaunch(c->graph[key], c->stream));
  }
  CK(cudaGetLastError());
  return ECHO_OK;
}

int echo_gpu_advance_host(EchoCtx* c, const double* v_in, const double* u_in, double* v_out, double* u_out,
                          int nsteps) {
  if (c && c->p.algo_solver == ECHO_C2P_MLP && !c->d_mlp_frag) return ECHO_ERR_ARG;  // no network loaded
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!c || !v_in || !u_in || nsteps < 0) return ECHO_ERR_ARG;
  const size_t bytes = sizeof(double) * c->nv * c->g.ncell;
  // v first, at the link's full rate: the first sweeps need it
  CK(cudaMemcpyAsync(c->d_v[c->vcur], v_in, bytes, cudaMemcpyHostToDevice, c->stream));
  // u beside the first sweeps, after everything queued so far (which may
  // still read or write u)
  CK(cudaEventRecord(c->ev_u_fork, c->stream));
  CK(cudaStreamWaitEvent(c->copy_stream, c->ev_u_fork, 0));
  CK(cudaMemcpyAsync(c->d_u[c->ucur], u_in, bytes, cudaMemcpyHostToDevice, c->copy_stream));
  CK(cudaEventRecord(c->ev_u, c->copy_stream));
  c->wait_u = 1;
  if (nsteps > 0) {
    enqueue_step(c);  // launched directly: its first stage waits for u after the sweeps
    int r = echo_gpu_run(c, nsteps - 1);
    if (r) return r;
  }
  if (c->wait_u) join_u(c);
  if (v_out) CK(cudaMemcpyAsync(v_out, c->d_v[c->vcur], bytes, cudaMemcpyDeviceToHost, c->stream));
  if (u_out) CK(cudaMemcpyAsync(u_out, c->d_u[c->ucur], bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaGetLastError());
  return ECHO_OK;
}

int echo_gpu_check_temp(EchoCtx* c, int freeze_type, double temp_end, double* max_value, int* stop) {
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!c || (freeze_type != 0 && freeze_type != 1)) return ECHO_ERR_ARG;
  CK(cudaMemsetAsync(&c->d_sc->check_bits, 0, sizeof(unsigned long long), c->stream));
  int dev = 0, nsm = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  size_t blocks = (c->g.ncell + 255) / 256;
  if (blocks > (size_t)(8 * nsm)) blocks = (size_t)(8 * nsm);
  check_temp_kernel<<<(unsigned)blocks, 256, 0, c->stream>>>(c->P, c->g, c->d_v[c->vcur], freeze_type,
                                                              &c->d_sc->check_bits);
  CK(cudaGetLastError());
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, &c->d_sc->check_bits, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double m;
  memcpy(&m, &bits, sizeof(m));
  if (max_value) *max_value = m;
  if (stop) *stop = m < temp_end ? 1 : 0;
  return ECHO_OK;
}

// Checkpoint of the run state at a step boundary (the role of out_dump /
// out_restart, out.f90:1313-1483): the current v and u, vold (the snapshot
// the next step's lagged time derivatives read) and every run scalar.
struct EchoCheckpointHeader {
  char magic[8];
  int kind, nv, nx, ny, nz, nrk;
  int scalars_bytes;
  int pad;
  DevScalars sc;
};
static const char kCkptMagic[8] = {'E', 'C', 'H', 'O', 'C', 'K', 'P', '1'};

int echo_gpu_checkpoint_size(const EchoCtx* c, size_t* bytes) {
  if (!c || !bytes) return ECHO_ERR_ARG;
  *bytes = sizeof(EchoCheckpointHeader) + sizeof(double) * c->g.ncell * (2 * (size_t)c->nv + 4);
  return ECHO_OK;
}

int echo_gpu_checkpoint(EchoCtx* c, void* blob) {
  (void)cudaGetLastError();
  if (!c || !blob) return ECHO_ERR_ARG;
  EchoCheckpointHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, kCkptMagic, 8);
  h.kind = c->kind;
  h.nv = c->nv;
  h.nx = c->g.nx;
  h.ny = c->g.ny;
  h.nz = c->g.nz;
  h.nrk = c->p.nrk;
  h.scalars_bytes = (int)sizeof(DevScalars);
  size_t nvc = (size_t)c->nv * c->g.ncell;
  char* p = (char*)blob + sizeof(h);
  CK(cudaMemcpyAsync(&h.sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(p, c->d_v[c->vcur], sizeof(double) * nvc, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(p + sizeof(double) * nvc, c->d_u[c->ucur], sizeof(double) * nvc, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaMemcpyAsync(p + sizeof(double) * 2 * nvc, c->d_vh[1 - c->vn], sizeof(double) * 4 * c->g.ncell,
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  memcpy(blob, &h, sizeof(h));
  return ECHO_OK;
}

int echo_gpu_restart(EchoCtx* c, const void* blob) {
  (void)cudaGetLastError();
  if (!c || !blob) return ECHO_ERR_ARG;
  EchoCheckpointHeader h;
  memcpy(&h, blob, sizeof(h));
  if (memcmp(h.magic, kCkptMagic, 8) != 0 || h.scalars_bytes != (int)sizeof(DevScalars) || h.kind != c->kind ||
      h.nv != c->nv || h.nx != c->g.nx || h.ny != c->g.ny || h.nz != c->g.nz || h.nrk != c->p.nrk) {
    fprintf(stderr, "echo_gpu_restart: the checkpoint does not belong to a run of this shape\n");
    return ECHO_ERR_ARG;
  }
  size_t nvc = (size_t)c->nv * c->g.ncell;
  const char* p = (const char*)blob + sizeof(h);
  c->vcur = c->ucur = c->vn = c->on = 0;
  CK(cudaMemcpyAsync(c->d_sc, &h.sc, sizeof(DevScalars), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_v[0], p, sizeof(double) * nvc, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_u[0], p + sizeof(double) * nvc, sizeof(double) * nvc, cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaMemcpyAsync(c->d_vh[1], p + sizeof(double) * 2 * nvc, sizeof(double) * 4 * c->g.ncell,
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ECHO_OK;
}

// dump.dat (out_dump / out_restart, out.f90:1313-1483, restart_type /= 0,
// out_freeze off): stream-access records, no markers -- iout (int32), t,
// timeold, timeinterval, vall (nv fields), uall (nv), vallold and uallold
// (krh..kvold_end), g_cov_3_old.
static size_t dump_bytes(const EchoCtx* c) {
  return 4 + 3 * sizeof(double) + sizeof(double) * c->g.ncell * (2 * (size_t)c->nv + 2 * (size_t)c->kold) +
         sizeof(double);
}

int echo_gpu_keep_old(EchoCtx* c, int on) {
  if (!c || (on != 0 && on != 1)) return ECHO_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  if (on && !c->keep_old) {
    size_t b = sizeof(double) * c->g.ncell * c->kold;
    for (int i = 0; i < 2; i++) {
      if (!c->d_oldv[i]) CK(cudaMalloc(&c->d_oldv[i], b));
      if (!c->d_oldu[i]) CK(cudaMalloc(&c->d_oldu[i], b));
    }
    c->keep_old = 1;
    c->on = 0;
    int r = init_old(c);  // from the current state, as init() leaves them
    if (r) return r;
  } else if (!on) {
    c->keep_old = 0;
  }
  for (int i = 0; i < 16; i++)
    if (c->graph_ok[i]) {
      cudaGraphExecDestroy(c->graph[i]);
      c->graph_ok[i] = false;
    }
  CK(cudaStreamSynchronize(c->stream));
  return ECHO_OK;
}

int echo_gpu_dump_size(const EchoCtx* c, size_t* bytes) {
  if (!c || !bytes) return ECHO_ERR_ARG;
  *bytes = dump_bytes(c);
  return ECHO_OK;
}

int echo_gpu_dump(EchoCtx* c, int iout, void* buf, size_t bytes) {
  (void)cudaGetLastError();
  if (!c || !buf || bytes != dump_bytes(c)) return ECHO_ERR_ARG;
  const size_t nc = c->g.ncell, nvc = (size_t)c->nv * nc, nold = (size_t)c->kold * nc;
  DevScalars s;
  CK(cudaMemcpyAsync(&s, c->d_sc, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  char* p = (char*)buf;
  const int32_t io = iout;
  memcpy(p, &io, 4);
  p += 4;
  double* vall = (double*)malloc(sizeof(double) * (2 * nvc + 2 * nold));
  if (!vall) return ECHO_ERR_ARG;
  double* uall = vall + nvc;
  double* vold = uall + nvc;
  double* uold = vold + nold;
  memset(vold, 0, sizeof(double) * 2 * nold);
  cudaError_t e = cudaMemcpyAsync(vall, c->d_v[c->vcur], sizeof(double) * nvc, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(uall, c->d_u[c->ucur], sizeof(double) * nvc, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && c->keep_old) {
    e = cudaMemcpyAsync(vold, c->d_oldv[1 - c->on], sizeof(double) * nold, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(uold, c->d_oldu[1 - c->on], sizeof(double) * nold, cudaMemcpyDeviceToHost, c->stream);
  } else if (e == cudaSuccess && c->p.viscosity) {
    // without keep_old the device holds the viscous vold's rho and velocity
    e = cudaMemcpyAsync(vold, c->d_vh[1 - c->vn], sizeof(double) * 4 * nc, cudaMemcpyDeviceToHost, c->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    free(vall);
    fprintf(stderr, "echo_gpu: CUDA error %s in echo_gpu_dump\n", cudaGetErrorString(e));
    return ECHO_ERR_CUDA;
  }
  const double hdr[3] = {s.t, s.timeold, s.timeinterval};
  memcpy(p, hdr, sizeof(hdr));
  p += sizeof(hdr);
  memcpy(p, vall, sizeof(double) * (2 * nvc + 2 * nold));
  p += sizeof(double) * (2 * nvc + 2 * nold);
  memcpy(p, &s.g3old, sizeof(double));
  free(vall);
  return ECHO_OK;
}

// t^3 as the step's end computes it on the device (end_step_scalars): a
// restarted run must hold the bits the uninterrupted one holds
static __global__ void t3_kernel(DevScalars* sc) { sc->t3 = pow(sc->t, 3.); }

int echo_gpu_restart_dump(EchoCtx* c, const void* buf, size_t bytes, int* iout) {
  (void)cudaGetLastError();
  if (!c || !buf || bytes != dump_bytes(c)) return ECHO_ERR_ARG;
  const size_t nc = c->g.ncell, nvc = (size_t)c->nv * nc, nold = (size_t)c->kold * nc;
  const char* p = (const char*)buf;
  int32_t io;
  memcpy(&io, p, 4);
  p += 4;
  double hdr[3];
  memcpy(hdr, p, sizeof(hdr));
  p += sizeof(hdr);
  const char* arrays = p;
  double g3old;
  memcpy(&g3old, p + sizeof(double) * (2 * nvc + 2 * nold), sizeof(double));
  // the host copy is not necessarily aligned for doubles (iout is 4 bytes)
  double* tmp = (double*)malloc(sizeof(double) * (2 * nvc + 2 * nold));
  if (!tmp) return ECHO_ERR_ARG;
  memcpy(tmp, arrays, sizeof(double) * (2 * nvc + 2 * nold));
  c->vcur = c->ucur = c->vn = c->on = 0;
  int r = reset_scalars(c, hdr[0]);
  if (r) {
    free(tmp);
    return r;
  }
  DevScalars s;
  cudaError_t e = cudaMemcpy(&s, c->d_sc, sizeof(s), cudaMemcpyDeviceToHost);
  s.timeold = hdr[1];
  s.timeinterval = hdr[2];
  s.g3old = g3old;
  if (e == cudaSuccess) e = cudaMemcpy(c->d_sc, &s, sizeof(s), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    t3_kernel<<<1, 1, 0, c->stream>>>(c->d_sc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_v[0], tmp, sizeof(double) * nvc, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_u[0], tmp + nvc, sizeof(double) * nvc, cudaMemcpyHostToDevice);
  // vold: the viscous time derivatives read its velocities (d_vh[1 - vn])
  if (e == cudaSuccess && c->p.viscosity)
    e = cudaMemcpy(c->d_vh[1], tmp + 2 * nvc, sizeof(double) * 4 * nc, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && c->keep_old) {
    e = cudaMemcpy(c->d_oldv[1], tmp + 2 * nvc, sizeof(double) * nold, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_oldu[1], tmp + 2 * nvc + nold, sizeof(double) * nold, cudaMemcpyHostToDevice);
  }
  free(tmp);
  if (e != cudaSuccess) {
    fprintf(stderr, "echo_gpu: CUDA error %s in echo_gpu_restart_dump\n", cudaGetErrorString(e));
    return ECHO_ERR_CUDA;
  }
  if (iout) *iout = io;
  return ECHO_OK;
}

int echo_gpu_stream(EchoCtx* c, void** stream) {
  if (!c || !stream) return ECHO_ERR_ARG;
  *stream = (void*)c->stream;
  return ECHO_OK;
}

int echo_gpu_profile_step(EchoCtx* c, double* ms, int* launches) {
  if (!c || !ms) return ECHO_ERR_ARG;
  (void)cudaGetLastError();
  std::vector<std::pair<int, cudaEvent_t>> marks;
  cudaEvent_t start;
  CK(cudaEventCreate(&start));
  CK(cudaEventRecord(start, c->stream));
  c->marks = &marks;
  enqueue_step(c);
  c->marks = nullptr;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  for (int k = 0; k < PK_N; k++) {
    ms[k] = 0.0;
    if (launches) launches[k] = 0;
  }
  cudaEvent_t prev = start;
  for (auto& m : marks) {
    float t = 0.f;
    cudaEventElapsedTime(&t, prev, m.second);
    ms[m.first] += t;
    if (launches) launches[m.first] += 1;
    prev = m.second;
  }
  for (auto& m : marks) cudaEventDestroy(m.second);
  cudaEventDestroy(start);
  return ECHO_OK;
}

int echo_gpu_set_sweeps(EchoCtx* c, int concurrent) {
  if (!c || (concurrent != 0 && concurrent != 1)) return ECHO_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  c->par_sweeps = concurrent;
  for (int i = 0; i < 16; i++)
    if (c->graph_ok[i]) {
      cudaGraphExecDestroy(c->graph[i]);
      c->graph_ok[i] = false;
    }
  return ECHO_OK;
}

int echo_gpu_set_faces(EchoCtx* c, int mode) {
  if (!c || (mode != 0 && mode != 8 && mode != 16)) return ECHO_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
#ifdef ECHO_EXACT
  c->face_mode = 0;
#else
  c->face_mode = mode;
#endif
  for (int i = 0; i < 16; i++)
    if (c->graph_ok[i]) {
      cudaGraphExecDestroy(c->graph[i]);
      c->graph_ok[i] = false;
    }
  return ECHO_OK;
}

int echo_gpu_set_stage(EchoCtx* c, int fused, int tx, int ty, int zseg, int* info) {
  (void)cudaGetLastError();
  if (!c || (fused != 0 && fused != 1)) return ECHO_ERR_ARG;
  if (fused) {
    if (tx < 0 || ty < 0 || zseg < 0) return ECHO_ERR_ARG;
    DISPATCH(c, setup_stage, c, tx, ty, zseg);
    (void)cudaGetLastError();
    if (!c->st_ok) {
      c->st_on = 0;
      return ECHO_ERR_UNSUPPORTED;
    }
  }
  c->st_on = fused && c->st_ok;
  // the cached step graphs hold the other kernels
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < 16; i++)
    if (c->graph_ok[i]) {
      cudaGraphExecDestroy(c->graph[i]);
      c->graph_ok[i] = false;
    }
  if (info) {
    info[0] = c->st_on;
    info[1] = c->st_tx;
    info[2] = c->st_ty;
    info[3] = c->st_zseg;
    info[4] = c->st_nt;
    info[5] = (int)c->st_grid;
    info[6] = (int)c->st_smem;
  }
  return ECHO_OK;
}

int echo_gpu_sync(EchoCtx* c) {
  if (!c) return ECHO_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  return ECHO_OK;
}

int echo_gpu_stats(EchoCtx* c, EchoStats* st) {
  if (!c || !st) return ECHO_ERR_ARG;
  int r = read_scalars(c);
  if (r) return r;
  const DevScalars* s = c->h_sc;
  st->dt = s->dt;
  st->t = s->t;
  st->glm_ch = s->glm_ch;
  st->c2p_iters = (long long)s->c2p_iters;
  st->c2p_cells = (long long)c->g.ncell;
  st->repairs = (long long)s->repairs;
  st->seed_fallbacks = (long long)s->fallbacks;
  st->errcode = errcode_of(s, &st->err_cell);
  st->bracket_fallbacks = (long long)s->brackets;
  return ECHO_OK;
}

int echo_gpu_rhs(EchoCtx* c, double* du, double* amax3) {
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!c) return ECHO_ERR_ARG;
  size_t nvc = (size_t)c->nv * c->g.ncell;
  if (!c->d_du) CK(cudaMalloc(&c->d_du, sizeof(double) * nvc));
  CK(cudaMemsetAsync(c->d_sc->amax_bits, 0, sizeof(unsigned long long) * 3, c->stream));
  for (int d = 0; d < 3; d++) {
    int n = d == 0 ? c->g.nx : d == 1 ? c->g.ny : c->g.nz;
    if (n > 1) DISPATCH(c, launch_faces, c, d);
  }
  DISPATCH(c, launch_update, c, 1, MODE_RHS, c->d_du);
  CK(cudaGetLastError());
  if (du) CK(cudaMemcpyAsync(du, c->d_du, sizeof(double) * nvc, cudaMemcpyDeviceToHost, c->stream));
  int r = read_scalars(c);
  if (r) return r;
  if (amax3)
    for (int d = 0; d < 3; d++) {
      unsigned long long b = c->h_sc->amax_bits[d];
      double x;
      memcpy(&x, &b, sizeof(x));
      amax3[d] = x;
    }
  return errcode_of(c->h_sc, nullptr) ? 1 : ECHO_OK;
}

}  // extern "C"

