// batch.cu -- the C-ABI of batched event-by-event runs (include/echo_gpu.h,
// echo_batch_*): arena allocation, the per-step launch sequence (captured
// as a CUDA graph), status read-back and the launch-shape autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/echo_gpu.h"
#include "batch.cuh"

using namespace echo;

// the network's BF16 fragments and FP32 parameters (mlp_train.cu)
bool echo_mlp_pack(const float* W, const float* norm, std::vector<unsigned>& frag, std::vector<float>& par);

#define CK(x)                                                                                     \
  do {                                                                                            \
    cudaError_t e_ = (x);                                                                         \
    if (e_ != cudaSuccess) {                                                                      \
      fprintf(stderr, "echo_batch: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                          \
      return ECHO_ERR_CUDA;                                                                       \
    }                                                                                             \
  } while (0)

#define BDISPATCH(b, fn, ...)                                     \
  do {                                                            \
    switch ((b)->kind) {                                          \
      case KIND_HD: fn<KIND_HD>(__VA_ARGS__); break;              \
      case KIND_VISC: fn<KIND_VISC>(__VA_ARGS__); break;          \
      case KIND_MHD: fn<KIND_MHD>(__VA_ARGS__); break;            \
      default: fn<KIND_MHDGLM>(__VA_ARGS__); break;               \
    }                                                             \
  } while (0)

static int batch_roles(const EchoBatch* b) { return b->ucur | (b->vcur << 1); }

static void batch_begin(EchoBatch* b, int irk) {
  batch_stage_begin_kernel<<<1, BEGIN_THREADS, 0, b->stream>>>(batch_dev(b), irk, batch_roles(b));
}

static void batch_scalars(EchoBatch* b, int irk) {
  ScalarArgs S;
  S.sc = nullptr;
  S.g = Grid{};
  S.cfl = b->p.cfl;
  S.maxdt = b->p.maxdt;
  S.glm_alpha = b->p.glm_alpha;
  S.irk = irk;
  S.nrk = b->p.nrk;
  S.divclean = b->p.divclean;
  S.mode = 0;
  batch_scalars_kernel<<<(unsigned)((b->nev + 127) / 128), 128, 0, b->stream>>>(S, batch_dev(b));
}

static void batch_faces_all(EchoBatch* b) {
  for (int d = 0; d < 3; d++)
    if (b->has_dir[d]) {
      BDISPATCH(b, launch_batch_faces, b, d);
      batch_mark(b, PK_FACES_X + d);
    }
}

// one explicit RK stage of every live event (evolve_main, evolve.f90:114-298):
// one launch per phase (mode 0) or one cooperative launch (mode 1)
static void enqueue_batch_stage(EchoBatch* b, int irk) {
  if (b->mode == 1) {
    BDISPATCH(b, launch_batch_stage, b, irk, (unsigned*)nullptr);
    batch_mark(b, PK_STAGE);
    if (irk == 1) b->ucur = 1 - b->ucur;
    b->vcur = 1 - b->vcur;
    return;
  }
  batch_begin(b, irk);
  batch_faces_all(b);
  batch_scalars(b, irk);
  batch_mark(b, PK_SCALARS);
  BDISPATCH(b, launch_batch_update, b, irk);
  batch_mark(b, PK_UPDATE);
  if (irk == 1) b->ucur = 1 - b->ucur;
  BDISPATCH(b, launch_batch_repair_smooth, b);
  batch_mark(b, PK_REPAIR);
  b->vcur = 1 - b->vcur;
}

// one time step of every live event; vnewstep is taken by the first stage's
// update (viscous), vold = vnewstep at the end is the role swap of vn
static void enqueue_batch_step(EchoBatch* b) {
  if (b->temp_end > 0.) {  // check_temp at the top of the time loop (echo.f90:189)
    int g = b->max_tiles[PH_CELL] < 16 * b->nsm ? b->max_tiles[PH_CELL] : 16 * b->nsm;
    batch_check_kernel<<<(unsigned)(g > 0 ? g : 1), 128, 0, b->stream>>>(b->P, batch_dev(b), b->nv,
                                                                        b->d_v[b->vcur]);
  }
  for (int irk = 1; irk <= b->p.nrk; irk++) enqueue_batch_stage(b, irk);
  batch_end_kernel<<<(unsigned)((b->nev + 127) / 128), 128, 0, b->stream>>>(batch_dev(b), b->p.coordinates,
                                                                             batch_roles(b));
  batch_mark(b, PK_END);
  if (b->p.viscosity) b->vn = 1 - b->vn;
}

static void advance_batch_roles(EchoBatch* b) {
  b->ucur = 1 - b->ucur;
  b->vcur = b->vcur ^ (b->p.nrk & 1);
  if (b->p.viscosity) b->vn = 1 - b->vn;
}

static void drop_graphs(EchoBatch* b) {
  for (int i = 0; i < 8; i++)
    if (b->graph_ok[i]) {
      cudaGraphExecDestroy(b->graph[i]);
      b->graph_ok[i] = false;
    }
}

static int host_order_default(EchoBatch* b) {
  std::vector<int> order(b->nev);
  std::iota(order.begin(), order.end(), 0);
  CK(cudaMemcpy(b->d_order, order.data(), sizeof(int) * b->nev, cudaMemcpyHostToDevice));
  return ECHO_OK;
}

extern "C" {

int echo_batch_init(const EchoParams* p, const double* eos_table, int n_eos, int nev, const EchoEventGrid* grids,
                    EchoBatch** out) {
  if (!p || !out || !grids || nev < 1) return ECHO_ERR_ARG;
  *out = nullptr;
  if (p->mhd > 1 || (p->mhd && p->viscosity)) return ECHO_ERR_UNSUPPORTED;
  if (p->nrk != ECHO_RK2 && p->nrk != ECHO_RK3) return ECHO_ERR_UNSUPPORTED;
  if (p->imex != 0 && p->imex != 1) return ECHO_ERR_ARG;
  if (p->mhd && c2p_alt_algo(p->algo_solver)) return ECHO_ERR_UNSUPPORTED;  // ALG_SOLV 2..6: single grid
  if (p->eqstate == ECHO_EOS_TABLE && (!eos_table || n_eos < 2)) return ECHO_ERR_ARG;
  for (int e = 0; e < nev; e++) {
    const EchoEventGrid& q = grids[e];
    if (q.nx < 1 || q.ny < 1 || q.nz < 1) return ECHO_ERR_ARG;
    if ((q.nx > 1 && q.nx < 3) || (q.ny > 1 && q.ny < 3) || (q.nz > 1 && q.nz < 3)) return ECHO_ERR_ARG;
    if (!(q.x2 > q.x1) || !(q.y2 > q.y1) || !(q.z2 > q.z1)) return ECHO_ERR_ARG;
  }
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return ECHO_ERR_CUDA;
  EchoBatch* b = new EchoBatch();
  b->p = *p;
  b->kind = echo_kind_of(p);
  b->nv = echo_nv_of(b->kind);
  b->nev = nev;
  echo_setup_bc(p, b->nv, b->bc, b->bc_uniform, b->bc_signed);
  // arena offsets and tile counts with every event live
  b->h_ev.resize(nev);
  size_t cell = 0, face[3] = {0, 0, 0};
  long long tiles[PH_N] = {0, 0, 0, 0};
  for (int d = 0; d < 3; d++) b->has_dir[d] = false;
  for (int e = 0; e < nev; e++) {
    const EchoEventGrid& q = grids[e];
    EvDesc& d = b->h_ev[e];
    d.g.nx = q.nx;
    d.g.ny = q.ny;
    d.g.nz = q.nz;
    d.g.ncell = (size_t)q.nx * q.ny * q.nz;
    double dx = (q.x2 - q.x1) / q.nx, dy = (q.y2 - q.y1) / q.ny, dz = (q.z2 - q.z1) / q.nz;
    d.g.ddx = q.nx > 1 ? 1. / dx : 0.;
    d.g.ddy = q.ny > 1 ? 1. / dy : 0.;
    d.g.ddz = q.nz > 1 ? 1. / dz : 0.;
    set_grid_div(d.g);
    d.x1 = q.x1;
    d.y1 = q.y1;
    d.dx = dx;
    d.dy = dy;
    d.cell = cell;
    cell += d.g.ncell;
    size_t nf[3] = {faces_of<0>(d.g), faces_of<1>(d.g), faces_of<2>(d.g)};
    int n3[3] = {q.nx, q.ny, q.nz};
    for (int k = 0; k < 3; k++) {
      d.face[k] = face[k];
      if (n3[k] > 1) {
        face[k] += nf[k];
        tiles[k] += tiles_of(nf[k], BATCH_TILE);
        b->has_dir[k] = true;
      }
    }
    tiles[PH_CELL] += tiles_of(d.g.ncell, BATCH_TILE);
  }
  for (int ph = 0; ph < PH_N; ph++) b->tile[ph] = BATCH_TILE;
  for (int ph = 0; ph < PH_N; ph++) {
    if (tiles[ph] >= (1ll << 31)) {
      delete b;
      return ECHO_ERR_ARG;
    }
    b->max_tiles[ph] = (int)tiles[ph];
  }
  b->ncell = cell;
  for (int k = 0; k < 3; k++) b->nfaces[k] = face[k];
  size_t nvc = (size_t)b->nv * cell;
  CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  for (int i = 0; i < 2; i++) {
    CK(cudaMalloc(&b->d_v[i], sizeof(double) * nvc));
    CK(cudaMalloc(&b->d_u[i], sizeof(double) * nvc));
    CK(cudaMemset(b->d_v[i], 0, sizeof(double) * nvc));
    CK(cudaMemset(b->d_u[i], 0, sizeof(double) * nvc));
    CK(cudaMalloc(&b->d_vh[i], sizeof(double) * 4 * cell));
    CK(cudaMemset(b->d_vh[i], 0, sizeof(double) * 4 * cell));
  }
  for (int k = 0; k < 3; k++) {
    b->d_F[k] = nullptr;
    b->d_WD[k] = nullptr;
    if (b->has_dir[k]) {
      CK(cudaMalloc(&b->d_F[k], sizeof(double) * b->nv * face[k]));
      if (p->viscosity) CK(cudaMalloc(&b->d_WD[k], sizeof(double) * 8 * face[k]));
    }
  }
  CK(cudaMalloc(&b->d_fail, cell));
  CK(cudaMemset(b->d_fail, 0, cell));
  CK(cudaMalloc(&b->d_ev, sizeof(EvDesc) * nev));
  CK(cudaMemcpy(b->d_ev, b->h_ev.data(), sizeof(EvDesc) * nev, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&b->d_sc, sizeof(DevScalars) * nev));
  CK(cudaMallocHost(&b->h_sc, sizeof(DevScalars) * nev));
  CK(cudaMalloc(&b->d_state, sizeof(int) * nev));
  CK(cudaMallocHost(&b->h_state, sizeof(int) * nev));
  CK(cudaMalloc(&b->d_steps, sizeof(long long) * nev));
  CK(cudaMallocHost(&b->h_steps, sizeof(long long) * nev));
  CK(cudaMemset(b->d_state, 0xff, sizeof(int) * nev));  // no state before the upload
  CK(cudaMemset(b->d_steps, 0, sizeof(long long) * nev));
  CK(cudaMalloc(&b->d_order, sizeof(int) * nev));
  CK(cudaMalloc(&b->d_prefix, sizeof(int) * PH_N * (nev + 1)));
  CK(cudaMalloc(&b->d_roles, sizeof(int) * nev));
  CK(cudaMallocHost(&b->h_roles, sizeof(int) * nev));
  CK(cudaMemset(b->d_roles, 0xff, sizeof(int) * nev));
  CK(cudaMemset(b->d_prefix, 0, sizeof(int) * PH_N * (nev + 1)));
  {
    int r = host_order_default(b);
    if (r) return r;
    r = echo_setup_phys(p, eos_table, n_eos, &b->P, &b->d_tab, &b->d_bk);
    if (r) return r;
  }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev));
  for (int s = 0; s < SL_N; s++) b->sched[s] = 0;
  b->tmax = 0.;
  b->temp_end = 0.;
  b->freeze_type = 1;
  b->vcur = b->ucur = b->vn = 0;
  b->marks = nullptr;
  b->mode = 0;
  b->coop_grid = 0;
  b->graphs_off = false;
  CK(cudaMalloc(&b->d_bar, 4 * sizeof(unsigned)));
  CK(cudaMemset(b->d_bar, 0, 4 * sizeof(unsigned)));
  *out = b;
  return ECHO_OK;
}

int echo_batch_free(EchoBatch* b) {
  if (!b) return ECHO_OK;
  cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  for (int i = 0; i < 2; i++) {
    cudaFree(b->d_v[i]);
    cudaFree(b->d_u[i]);
    cudaFree(b->d_vh[i]);
  }
  for (int k = 0; k < 3; k++) {
    cudaFree(b->d_F[k]);
    cudaFree(b->d_WD[k]);
  }
  cudaFree(b->d_fail);
  cudaFree(b->d_bar);
  cudaFree(b->d_mlp_frag);
  cudaFree(b->d_mlp_par);
  cudaFree(b->d_ev);
  cudaFree(b->d_sc);
  cudaFree(b->d_state);
  cudaFree(b->d_steps);
  cudaFree(b->d_order);
  cudaFree(b->d_prefix);
  cudaFree(b->d_roles);
  cudaFreeHost(b->h_roles);
  cudaFree(b->d_tab);
  cudaFree(b->d_bk);
  cudaFreeHost(b->h_sc);
  cudaFreeHost(b->h_state);
  cudaFreeHost(b->h_steps);
  cudaStreamDestroy(b->stream);
  delete b;
  return ECHO_OK;
}

int echo_batch_nv(const EchoBatch* b) { return b ? b->nv : 0; }

int echo_batch_offsets(const EchoBatch* b, long long* cell_offset) {
  if (!b || !cell_offset) return ECHO_ERR_ARG;
  for (int e = 0; e < b->nev; e++) cell_offset[e] = (long long)b->h_ev[e].cell;
  cell_offset[b->nev] = (long long)b->ncell;
  return ECHO_OK;
}

// every event live at time t, zero steps, stop at tmax
static int batch_reset(EchoBatch* b, double t, double tmax) {
  b->vcur = b->ucur = b->vn = 0;
  if (tmax != b->tmax) drop_graphs(b);  // the graphs hold tmax
  b->tmax = tmax;
  std::vector<DevScalars> s(b->nev);
  for (int e = 0; e < b->nev; e++) {
    DevScalars& q = s[e];
    memset(&q, 0, sizeof(q));
    q.t = t;
    q.t3 = pow(t, 3.);
    q.tout = tmax;
    q.dtout = tmax - t > 0 ? tmax - t : 1.;
    q.tmax = tmax;
    q.timeold = t;
    q.g3old = b->p.coordinates == ECHO_BJORKEN ? t * t : 1.;
    q.glm_ch_old = 0.5;  // common.f90:283
    q.err_key = ~0ull;
  }
  CK(cudaMemcpyAsync(b->d_sc, s.data(), sizeof(DevScalars) * b->nev, cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemsetAsync(b->d_state, 0, sizeof(int) * b->nev, b->stream));
  CK(cudaMemsetAsync(b->d_steps, 0, sizeof(long long) * b->nev, b->stream));
  CK(cudaMemsetAsync(b->d_roles, 0xff, sizeof(int) * b->nev, b->stream));
  CK(cudaMemsetAsync(b->d_vh[0], 0, sizeof(double) * 4 * b->ncell, b->stream));
  CK(cudaMemsetAsync(b->d_vh[1], 0, sizeof(double) * 4 * b->ncell, b->stream));
  return ECHO_OK;
}

static int batch_upload_impl(EchoBatch* b, const double* v, const double* u, double t, double tmax,
                             cudaMemcpyKind kind) {
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!b || !v) return ECHO_ERR_ARG;
  int r = batch_reset(b, t, tmax);
  if (r) return r;
  size_t bytes = sizeof(double) * b->nv * b->ncell;
  CK(cudaMemcpyAsync(b->d_v[0], v, bytes, kind, b->stream));
  batch_begin(b, 0);  // tile lists of every event (the first check_temp uses them)
  if (u) {
    CK(cudaMemcpyAsync(b->d_u[0], u, bytes, kind, b->stream));
  } else {
    BDISPATCH(b, launch_batch_p2c, b);
  }
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  return ECHO_OK;
}

int echo_batch_upload(EchoBatch* b, const double* v, const double* u, double t, double tmax) {
  return batch_upload_impl(b, v, u, t, tmax, cudaMemcpyHostToDevice);
}
int echo_batch_upload_device(EchoBatch* b, const double* d_v, const double* d_u, double t, double tmax) {
  return batch_upload_impl(b, d_v, d_u, t, tmax, cudaMemcpyDeviceToDevice);
}

// Each event's state is in the buffers that were current when it stopped
// (or the current ones while it runs): one copy per run of events that
// share their buffer roles.
int echo_batch_glauber(EchoBatch* b, const double* src, const long long* src_offset, double sigma, double peak,
                       double t, double tmax) {
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!b || !src_offset || !(sigma > 0.)) return ECHO_ERR_ARG;
  if (src_offset[0] != 0) return ECHO_ERR_ARG;
  for (int e = 0; e < b->nev; e++)
    if (src_offset[e + 1] < src_offset[e]) return ECHO_ERR_ARG;
  const long long nsrc = src_offset[b->nev];
  if (nsrc > 0 && !src) return ECHO_ERR_ARG;
  int r = batch_reset(b, t, tmax);
  if (r) return r;
  double* d_src = nullptr;
  long long* d_off = nullptr;
  CK(cudaMalloc(&d_src, sizeof(double) * 3 * (nsrc > 0 ? nsrc : 1)));
  CK(cudaMalloc(&d_off, sizeof(long long) * (b->nev + 1)));
  if (nsrc > 0) CK(cudaMemcpyAsync(d_src, src, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(d_off, src_offset, sizeof(long long) * (b->nev + 1), cudaMemcpyHostToDevice, b->stream));
  batch_begin(b, 0);  // tile lists of every event; zeroes the maxima
  unsigned grid = (unsigned)(b->max_tiles[PH_CELL] > 0 ? b->max_tiles[PH_CELL] : 1);
  batch_smear_kernel<<<grid, 128, 0, b->stream>>>(batch_dev(b), b->nv, d_src, d_off, sigma, b->d_v[0]);
  batch_glauber_fill_kernel<<<grid, 128, 0, b->stream>>>(b->P, batch_dev(b), b->nv, peak, b->p.enezero,
                                                         b->d_v[0]);
  BDISPATCH(b, launch_batch_p2c, b);
  CK(cudaStreamSynchronize(b->stream));
  cudaFree(d_src);
  cudaFree(d_off);
  CK(cudaGetLastError());
  return ECHO_OK;
}

int echo_batch_download(EchoBatch* b, double* v, double* u) {
  if (!b) return ECHO_ERR_ARG;
  CK(cudaMemcpyAsync(b->h_roles, b->d_roles, sizeof(int) * b->nev, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  const int now = batch_roles(b);
  int e0 = 0;
  while (e0 < b->nev) {
    int r = b->h_roles[e0] >= 0 ? b->h_roles[e0] : now;
    int e1 = e0 + 1;
    while (e1 < b->nev && (b->h_roles[e1] >= 0 ? b->h_roles[e1] : now) == r) e1++;
    size_t off = (size_t)b->nv * b->h_ev[e0].cell;
    size_t end = e1 < b->nev ? (size_t)b->nv * b->h_ev[e1].cell : (size_t)b->nv * b->ncell;
    size_t bytes = sizeof(double) * (end - off);
    if (v) CK(cudaMemcpyAsync(v + off, b->d_v[(r >> 1) & 1] + off, bytes, cudaMemcpyDeviceToHost, b->stream));
    if (u) CK(cudaMemcpyAsync(u + off, b->d_u[r & 1] + off, bytes, cudaMemcpyDeviceToHost, b->stream));
    e0 = e1;
  }
  CK(cudaStreamSynchronize(b->stream));
  return ECHO_OK;
}

int echo_batch_mlp_set(EchoBatch* b, const float* weights, const float* norm) {
  if (!b || !weights || !norm) return ECHO_ERR_ARG;
  std::vector<unsigned> frag;
  std::vector<float> par;
  echo_mlp_pack(weights, norm, frag, par);
  if (!b->d_mlp_frag) {
    CK(cudaMalloc(&b->d_mlp_frag, sizeof(unsigned) * frag.size()));
    CK(cudaMalloc(&b->d_mlp_par, sizeof(float) * par.size()));
  }
  CK(cudaMemcpyAsync(b->d_mlp_frag, frag.data(), sizeof(unsigned) * frag.size(), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->d_mlp_par, par.data(), sizeof(float) * par.size(), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  drop_graphs(b);  // step graphs captured before hold the unseeded update
  return ECHO_OK;
}

int echo_batch_run(EchoBatch* b, int nsteps) {
  (void)cudaGetLastError();  // a failed launch of an earlier call must not be reported here
  if (!b || nsteps < 0) return ECHO_ERR_ARG;
  if (b->p.algo_solver == ECHO_C2P_MLP && !b->d_mlp_frag) return ECHO_ERR_ARG;  // no network loaded
  for (int s = 0; s < nsteps; s++) {
    int key = b->ucur | (b->vcur << 1) | (b->vn << 2);
    if (b->graphs_off) {  // launches straight onto the stream
      enqueue_batch_step(b);
      continue;
    }
    if (!b->graph_ok[key]) {
      cudaGraph_t gr = nullptr;
      const int ucur = b->ucur, vcur = b->vcur, vn = b->vn;
      CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      enqueue_batch_step(b);
      cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
      if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph[key], gr, 0);
      if (gr) cudaGraphDestroy(gr);
      if (e != cudaSuccess) {
        // a launch this stream cannot capture (the cooperative stage
        // kernel on a driver without that support): run without graphs
        (void)cudaGetLastError();
        b->graphs_off = true;
        b->ucur = ucur;
        b->vcur = vcur;
        b->vn = vn;
        enqueue_batch_step(b);
        continue;
      }
      b->graph_ok[key] = true;
    } else {
      advance_batch_roles(b);
    }
    CK(cudaGraphLaunch(b->graph[key], b->stream));
  }
  CK(cudaGetLastError());
  return ECHO_OK;
}

// the timeout flag of the cooperative stage's grid barrier
static int check_barrier(EchoBatch* b) {
  if (b->mode != 1) return ECHO_OK;
  unsigned flag = 0;
  CK(cudaMemcpyAsync(&flag, b->d_bar + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  if (flag) {
    fprintf(stderr, "echo_batch: a grid barrier of the cooperative stage timed out\n");
    return ECHO_ERR_TIMEOUT;
  }
  return ECHO_OK;
}

int echo_batch_live(EchoBatch* b, int* nlive) {
  if (!b || !nlive) return ECHO_ERR_ARG;
  CK(cudaMemcpyAsync(b->h_state, b->d_state, sizeof(int) * b->nev, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  // an event that reached tmax in the last step is marked at the next
  // stage start; count it as finished here already
  CK(cudaMemcpyAsync(b->h_sc, b->d_sc, sizeof(DevScalars) * b->nev, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  int n = 0;
  for (int e = 0; e < b->nev; e++)
    if (b->h_state[e] == EV_LIVE && b->h_sc[e].t < b->tmax && b->h_sc[e].err_key == ~0ull) n++;
  *nlive = n;
  return ECHO_OK;
}

int echo_batch_status(EchoBatch* b, EchoEventStatus* st) {
  if (!b || !st) return ECHO_ERR_ARG;
  CK(cudaMemcpyAsync(b->h_sc, b->d_sc, sizeof(DevScalars) * b->nev, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaMemcpyAsync(b->h_state, b->d_state, sizeof(int) * b->nev, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaMemcpyAsync(b->h_steps, b->d_steps, sizeof(long long) * b->nev, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  for (int e = 0; e < b->nev; e++) {
    const DevScalars& s = b->h_sc[e];
    EchoEventStatus& o = st[e];
    memset(&o, 0, sizeof(o));
    o.t = s.t;
    o.dt = s.dt;
    o.steps = b->h_steps[e];
    int state = b->h_state[e];
    if (state == EV_LIVE && s.err_key != ~0ull) state = EV_CRASHED;
    if (state == EV_LIVE && s.t >= b->tmax) state = EV_DONE;
    o.state = state;
    if (s.err_key != ~0ull) {
      o.errcode = (int)(s.err_key & 0xFFFFFull);
      o.err_cell = (int)(s.err_key >> 20);
    } else {
      o.err_cell = -1;
    }
    o.c2p_iters = (long long)s.c2p_iters;
    o.repairs = (long long)s.repairs;
    o.seed_fallbacks = (long long)s.fallbacks;
  }
  return ECHO_OK;
}

int echo_batch_sync(EchoBatch* b) {
  if (!b) return ECHO_ERR_ARG;
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  return check_barrier(b);
}

int echo_batch_stream(EchoBatch* b, void** stream) {
  if (!b || !stream) return ECHO_ERR_ARG;
  *stream = (void*)b->stream;
  return ECHO_OK;
}

int echo_batch_set_schedule(EchoBatch* b, const int* ctas, const int* order) {
  if (!b) return ECHO_ERR_ARG;
  if (ctas)
    for (int s = 0; s < SL_N; s++)
      if (ctas[s] < 0) return ECHO_ERR_ARG;
  if (order) {
    std::vector<int> seen(b->nev, 0);
    for (int i = 0; i < b->nev; i++) {
      if (order[i] < 0 || order[i] >= b->nev || seen[order[i]]) return ECHO_ERR_ARG;
      seen[order[i]] = 1;
    }
  }
  CK(cudaStreamSynchronize(b->stream));
  if (ctas)
    for (int s = 0; s < SL_N; s++) b->sched[s] = ctas[s];
  if (order) CK(cudaMemcpy(b->d_order, order, sizeof(int) * b->nev, cudaMemcpyHostToDevice));
  drop_graphs(b);
  return ECHO_OK;
}

int echo_batch_set_stop(EchoBatch* b, int freeze_type, double temp_end) {
  if (!b || (freeze_type != 0 && freeze_type != 1)) return ECHO_ERR_ARG;
  CK(cudaStreamSynchronize(b->stream));
  b->freeze_type = freeze_type;
  b->temp_end = temp_end;
  drop_graphs(b);  // the graphs hold both
  return ECHO_OK;
}

int echo_batch_get_schedule(const EchoBatch* b, int* ctas) {
  if (!b || !ctas) return ECHO_ERR_ARG;
  for (int s = 0; s < SL_N; s++) ctas[s] = b->sched[s];
  return ECHO_OK;
}

int echo_batch_profile_step(EchoBatch* b, double* ms, int* launches) {
  if (!b || !ms) return ECHO_ERR_ARG;
  (void)cudaGetLastError();
  std::vector<std::pair<int, cudaEvent_t>> marks;
  cudaEvent_t start;
  CK(cudaEventCreate(&start));
  CK(cudaEventRecord(start, b->stream));
  b->marks = &marks;
  enqueue_batch_step(b);
  b->marks = nullptr;
  CK(cudaStreamSynchronize(b->stream));
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

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------
// The state a tuning run disturbs, saved and put back around it.
struct BatchSave {
  double *v, *u, *vh0, *vh1;
  DevScalars* sc;
  int* state;
  int* roles;
  long long* steps;
};

static int save_batch(EchoBatch* b, BatchSave& s, bool back) {
  size_t nvc = sizeof(double) * b->nv * b->ncell, n4 = sizeof(double) * 4 * b->ncell;
  cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  if (!back) {
    CK(cudaMalloc(&s.v, nvc));
    CK(cudaMalloc(&s.u, nvc));
    CK(cudaMalloc(&s.vh0, n4));
    CK(cudaMalloc(&s.vh1, n4));
    CK(cudaMalloc(&s.sc, sizeof(DevScalars) * b->nev));
    CK(cudaMalloc(&s.state, sizeof(int) * b->nev));
    CK(cudaMalloc(&s.roles, sizeof(int) * b->nev));
    CK(cudaMalloc(&s.steps, sizeof(long long) * b->nev));
    CK(cudaMemcpyAsync(s.v, b->d_v[b->vcur], nvc, k, b->stream));
    CK(cudaMemcpyAsync(s.u, b->d_u[b->ucur], nvc, k, b->stream));
    CK(cudaMemcpyAsync(s.vh0, b->d_vh[0], n4, k, b->stream));
    CK(cudaMemcpyAsync(s.vh1, b->d_vh[1], n4, k, b->stream));
    CK(cudaMemcpyAsync(s.sc, b->d_sc, sizeof(DevScalars) * b->nev, k, b->stream));
    CK(cudaMemcpyAsync(s.state, b->d_state, sizeof(int) * b->nev, k, b->stream));
    CK(cudaMemcpyAsync(s.roles, b->d_roles, sizeof(int) * b->nev, k, b->stream));
    CK(cudaMemcpyAsync(s.steps, b->d_steps, sizeof(long long) * b->nev, k, b->stream));
  } else {
    CK(cudaMemcpyAsync(b->d_v[b->vcur], s.v, nvc, k, b->stream));
    CK(cudaMemcpyAsync(b->d_u[b->ucur], s.u, nvc, k, b->stream));
    CK(cudaMemcpyAsync(b->d_vh[0], s.vh0, n4, k, b->stream));
    CK(cudaMemcpyAsync(b->d_vh[1], s.vh1, n4, k, b->stream));
    CK(cudaMemcpyAsync(b->d_sc, s.sc, sizeof(DevScalars) * b->nev, k, b->stream));
    CK(cudaMemcpyAsync(b->d_state, s.state, sizeof(int) * b->nev, k, b->stream));
    CK(cudaMemcpyAsync(b->d_roles, s.roles, sizeof(int) * b->nev, k, b->stream));
    CK(cudaMemcpyAsync(b->d_steps, s.steps, sizeof(long long) * b->nev, k, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    cudaFree(s.v);
    cudaFree(s.u);
    cudaFree(s.vh0);
    cudaFree(s.vh1);
    cudaFree(s.sc);
    cudaFree(s.state);
    cudaFree(s.roles);
    cudaFree(s.steps);
  }
  return ECHO_OK;
}

// tiles of each list with every event live, for the current tile lengths
static void recompute_max_tiles(EchoBatch* b) {
  for (int ph = 0; ph < PH_N; ph++) {
    long long n = 0;
    for (int e = 0; e < b->nev; e++) n += event_tiles(b->h_ev[e].g, ph, b->tile[ph]);
    b->max_tiles[ph] = (int)n;
  }
}

// device time of `reps` launches of slot sl with its current shape
static int time_slot(EchoBatch* b, int sl, int reps, cudaEvent_t e0, cudaEvent_t e1, double* ms) {
  CK(cudaEventRecord(e0, b->stream));
  for (int r = 0; r < reps; r++) {
    if (sl <= SL_FZ) {
      BDISPATCH(b, launch_batch_faces, b, sl - SL_FX);
    } else if (sl == SL_UPDATE) {
      BDISPATCH(b, launch_batch_update, b, 1);
    } else {
      BDISPATCH(b, launch_batch_repair_smooth, b);
    }
  }
  CK(cudaEventRecord(e1, b->stream));
  CK(cudaEventSynchronize(e1));
  CK(cudaGetLastError());
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, e0, e1));
  *ms = t / reps;
  return ECHO_OK;
}

// device time of `reps` first stages in the current mode; the roles are
// put back after each, so every repetition computes the same stage (it
// writes only the buffers the stage produces)
static int time_stage(EchoBatch* b, int reps, cudaEvent_t e0, cudaEvent_t e1, double* ms) {
  const int u0 = b->ucur, v0 = b->vcur;
  CK(cudaEventRecord(e0, b->stream));
  for (int r = 0; r < reps; r++) {
    enqueue_batch_stage(b, 1);
    b->ucur = u0;
    b->vcur = v0;
  }
  CK(cudaEventRecord(e1, b->stream));
  CK(cudaEventSynchronize(e1));
  CK(cudaGetLastError());
  int r = check_barrier(b);
  if (r) return r;
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, e0, e1));
  *ms = t / reps;
  return ECHO_OK;
}

static void tune_log(EchoBatch* b, double what, double shape, double ctas, double ms) {
  b->tune.push_back(what);
  b->tune.push_back(shape);
  b->tune.push_back(ctas);
  b->tune.push_back(ms);
}

int echo_batch_autotune(EchoBatch* b, int reps, double* ms_out) {
  (void)cudaGetLastError();
  if (!b || reps < 1) return ECHO_ERR_ARG;
  CK(cudaStreamSynchronize(b->stream));
  int occ[SL_N] = {0, 0, 0, 0, 0};
  BDISPATCH(b, batch_occupancy, b, occ);
  CK(cudaGetLastError());
  BatchSave sv;
  int r = save_batch(b, sv, false);
  if (r) return r;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  b->tune.clear();
  const bool smooth = b->kind == KIND_VISC && b->p.enable_smooth_viscosity;
  const int ph_of[SL_N] = {PH_FX, PH_FY, PH_FZ, PH_CELL, PH_CELL};
  const int tiles[3] = {128, 256, 512};
  const int mode0 = b->mode;
  b->mode = 0;
  // one phase at a time: tile length x CTAs (one per tile, or k per SM)
  double best_ms[SL_N];
  int best_tile[SL_N], best_cta[SL_N];
  for (int sl = 0; sl < SL_N; sl++) {
    best_ms[sl] = 1e300;
    best_tile[sl] = b->tile[ph_of[sl]];
    best_cta[sl] = b->sched[sl];
  }
  for (int ti = 0; ti < 3; ti++) {
    for (int ph = 0; ph < PH_N; ph++) b->tile[ph] = tiles[ti];
    recompute_max_tiles(b);
    // the inputs of the first-stage update: tile lists, face fluxes and dt
    batch_begin(b, 1);
    batch_faces_all(b);
    batch_scalars(b, 1);
    for (int sl = 0; sl < SL_N; sl++) {
      if (sl <= SL_FZ && !b->has_dir[sl]) continue;
      if (sl == SL_SMOOTH && !smooth) continue;
      std::vector<int> cand = {0};
      for (int k = 1; k <= occ[sl]; k++)
        if (k * b->nsm < b->max_tiles[ph_of[sl]]) cand.push_back(k * b->nsm);
      for (int c : cand) {
        b->sched[sl] = c;
        double t;
        r = time_slot(b, sl, 1, e0, e1, &t);  // warm-up
        if (!r) r = time_slot(b, sl, reps, e0, e1, &t);
        if (r) return r;
        tune_log(b, sl, tiles[ti], c, t);
        if (t < best_ms[sl]) {
          best_ms[sl] = t;
          best_tile[sl] = tiles[ti];
          best_cta[sl] = c;
        }
      }
      b->sched[sl] = best_cta[sl];
    }
  }
  for (int sl = 0; sl < SL_N; sl++) {
    if (ms_out) ms_out[sl] = best_ms[sl] < 1e299 ? best_ms[sl] : 0.;
    b->sched[sl] = best_cta[sl];
  }
  for (int d = 0; d < 3; d++) b->tile[d] = best_tile[d];
  // the cell list serves the update and the smoothing: the update's choice
  b->tile[PH_CELL] = best_tile[SL_UPDATE];
  recompute_max_tiles(b);
  // the whole first stage: one launch per phase, then one cooperative
  // launch with 1..occupancy CTAs per SM
  double t_phased = 1e300, t_coop = 1e300;
  r = time_stage(b, 1, e0, e1, &t_phased);
  if (!r) r = time_stage(b, reps, e0, e1, &t_phased);
  if (r) return r;
  tune_log(b, SL_N, 0, 0, t_phased);
  unsigned best_grid = 0;
  if (b->p.recal == ECHO_REC_WENO5) {
    b->mode = 1;
    unsigned gmax = 0;
    b->coop_grid = 0;
    BDISPATCH(b, launch_batch_stage, b, 1, &gmax);  // warm-up, and the largest resident grid
    CK(cudaStreamSynchronize(b->stream));
    CK(cudaGetLastError());
    r = check_barrier(b);
    if (r) return r;
    for (unsigned g = (unsigned)b->nsm; g <= gmax && gmax > 0; g += (unsigned)b->nsm) {
      b->coop_grid = g;
      double t;
      r = time_stage(b, reps, e0, e1, &t);
      if (r) return r;
      tune_log(b, SL_N, 1, g, t);
      if (t < t_coop) {
        t_coop = t;
        best_grid = g;
      }
    }
  }
  if (t_coop < t_phased) {
    b->mode = 1;
    b->coop_grid = best_grid;
  } else {
    b->mode = 0;
    b->coop_grid = 0;
  }
  (void)mode0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  drop_graphs(b);
  return save_batch(b, sv, true);
}

int echo_batch_autotune_report(const EchoBatch* b, double* rows, int cap, int* n) {
  if (!b || !n || cap < 0) return ECHO_ERR_ARG;
  int m = (int)(b->tune.size() / 4);
  *n = m;
  if (rows)
    for (int i = 0; i < m && i < cap; i++)
      for (int q = 0; q < 4; q++) rows[4 * i + q] = b->tune[4 * (size_t)i + q];
  return ECHO_OK;
}

int echo_batch_set_tiles(EchoBatch* b, const int* tiles) {
  if (!b || !tiles) return ECHO_ERR_ARG;
  for (int ph = 0; ph < PH_N; ph++)
    if (tiles[ph] < BATCH_NT || tiles[ph] > 8 * BATCH_NT || tiles[ph] % BATCH_NT) return ECHO_ERR_ARG;
  CK(cudaStreamSynchronize(b->stream));
  for (int ph = 0; ph < PH_N; ph++) b->tile[ph] = tiles[ph];
  recompute_max_tiles(b);
  drop_graphs(b);
  return ECHO_OK;
}

int echo_batch_set_mode(EchoBatch* b, int mode, int grid) {
  if (!b || (mode != 0 && mode != 1) || grid < 0) return ECHO_ERR_ARG;
  if (mode == 1 && b->p.recal != ECHO_REC_WENO5) return ECHO_ERR_UNSUPPORTED;
  CK(cudaStreamSynchronize(b->stream));
  b->mode = mode;
  b->coop_grid = (unsigned)grid;
  b->graphs_off = false;
  drop_graphs(b);
  return ECHO_OK;
}

int echo_batch_get_tuning(const EchoBatch* b, int* out) {
  if (!b || !out) return ECHO_ERR_ARG;
  for (int ph = 0; ph < PH_N; ph++) out[ph] = b->tile[ph];
  out[PH_N] = b->mode;
  out[PH_N + 1] = (int)b->coop_grid;
  out[PH_N + 2] = b->graphs_off ? 0 : 1;
  return ECHO_OK;
}

}  // extern "C"
