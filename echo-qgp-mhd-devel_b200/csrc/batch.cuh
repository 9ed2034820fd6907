// batch.cuh -- batched event-by-event execution.
//
// The reference runs Monte Carlo events one after another (the events loop
// of echo.f90:113-308, one grid each).  Here many events, each on its own
// grid size, advance together: all grids live in one arena, and every phase
// of a stage (x faces, y faces, z faces, per-event scalars, cell update,
// repair, smoothing) is ONE launch over the tiles of all live events.  The
// face and update launches are persistent: a grid sized to the GPU walks a
// tile list that the stage-begin kernel rebuilds on the device before every
// stage from the events still running, so events that finished (t >= tmax,
// echo.f90:187) or crashed (echo.f90:206-209) cost nothing and the step
// needs no host round trip (whole steps are CUDA graphs).
//
// Each tile is a run of consecutive faces or cells of one event (its length,
// per tile list, a multiple of the BATCH_NT threads of a block: 128, 256 or
// 512, chosen by the autotuner), so a block's warps never straddle two
// events: the block max of the signal speed and the warp sums of the
// con2prim counters go to that event's own scalars, and each event gets its
// own dt (evolve_dt, evolve.f90:723-764).
#pragma once

#include "ctx.cuh"

namespace echo {

enum { BATCH_NT = 128, BATCH_TILE = 128 };  // threads per block; default tile length
// tile lists: faces along x, y, z and cells
enum { PH_FX = 0, PH_FY = 1, PH_FZ = 2, PH_CELL = 3, PH_N = 4 };
// launch-shape slots of the schedule: the three face sweeps, update, smoothing
enum { SL_FX = 0, SL_FY = 1, SL_FZ = 2, SL_UPDATE = 3, SL_SMOOTH = 4, SL_N = 5 };
// event states
enum { EV_LIVE = 0, EV_DONE = 1, EV_CRASHED = 2, EV_COOLED = 3 };

struct EvDesc {
  Grid g;
  size_t cell;     // first cell of the event in the cell arrays
  size_t face[3];  // first face of the event in each direction's face arrays
  double x1, y1, dx, dy;  // cell centres x1 + (i - 1/2) dx, i = 1..nx (common_grid, common.f90:441-481)
};

struct BatchDev {
  const EvDesc* ev;
  DevScalars* sc;    // one block of run scalars per event
  int* state;        // EV_*
  long long* steps;  // completed steps per event
  const int* order;  // the tile lists visit the events in this order
  int* prefix;       // [PH_N][nev + 1] first tile of each slot of `order`; [nev] = total
  int* roles;        // buffer roles (ucur | vcur << 1) when the event stopped; -1 while live
  int nev;
  double tmax;
  double temp_end;   // check_temp threshold (TEMP_END); <= 0: no check
  int freeze_type;   // 0: temperature, 1: energy density
  int tile[PH_N];    // tile length of each list (a multiple of BATCH_NT)
};

__host__ __device__ __forceinline__ int tiles_of(size_t n, int tile) { return (int)((n + tile - 1) / tile); }

__host__ __device__ __forceinline__ int event_tiles(const Grid& g, int ph, int tile) {
  switch (ph) {
    case PH_FX: return g.nx > 1 ? tiles_of(faces_of<0>(g), tile) : 0;
    case PH_FY: return g.ny > 1 ? tiles_of(faces_of<1>(g), tile) : 0;
    case PH_FZ: return g.nz > 1 ? tiles_of(faces_of<2>(g), tile) : 0;
    default: return tiles_of(g.ncell, tile);
  }
}

// slot of `order` that holds tile t: the largest i with pre[i] <= t (events
// without tiles share their successor's offset and are never chosen)
__device__ __forceinline__ int tile_slot(const int* pre, int nev, int t) {
  int lo = 0, hi = nev;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (pre[mid] <= t)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Start of stage irk for every event: the stop test at the top of the time
// loop (echo.f90:187, irk == 1 only; irk == 0 skips it), the crash test of
// the previous stage (echo.f90:206-209), the per-stage resets, and the tile
// lists of the events that stay live.  An event that stops keeps its state
// in the buffers that are current now (`roles`), which later steps no longer
// touch for it.  One block of BEGIN_THREADS threads; each thread owns a
// contiguous run of `order`.
enum { BEGIN_THREADS = 1024 };
template <int NT>
__device__ __forceinline__ void stage_begin_block(const BatchDev& B, int irk, int roles, int (*s)[NT]) {
  const int tid = threadIdx.x;
  const int per = (B.nev + NT - 1) / NT;
  const int i0 = tid * per;
  const int i1 = min(B.nev, i0 + per);
  int sum[PH_N] = {0, 0, 0, 0};
  for (int i = i0; i < i1; i++) {
    int e = B.order[i];
    DevScalars* sc = B.sc + e;
    int st = B.state[e];
    if (st == EV_LIVE && irk == 1 && sc->t >= B.tmax) st = EV_DONE;
    // check_temp after the tmax test (echo.f90:187-190)
    if (st == EV_LIVE && irk == 1 && B.temp_end > 0. &&
        __longlong_as_double((long long)sc->check_bits) < B.temp_end)
      st = EV_COOLED;
    if (st == EV_LIVE && sc->err_key != ~0ull) st = EV_CRASHED;
    if (st != EV_LIVE && B.state[e] == EV_LIVE) B.roles[e] = roles;
    B.state[e] = st;
    if (st == EV_LIVE) {
      sc->amax_bits[0] = 0;
      sc->amax_bits[1] = 0;
      sc->amax_bits[2] = 0;
      sc->nfail = 0;
      sc->c2p_iters = 0;
#pragma unroll
      for (int ph = 0; ph < PH_N; ph++) sum[ph] += event_tiles(B.ev[e].g, ph, B.tile[ph]);
    }
  }
#pragma unroll
  for (int ph = 0; ph < PH_N; ph++) s[ph][tid] = sum[ph];
  __syncthreads();
  // inclusive scan of the per-thread sums (Hillis-Steele)
  for (int off = 1; off < NT; off <<= 1) {
    int add[PH_N];
#pragma unroll
    for (int ph = 0; ph < PH_N; ph++) add[ph] = tid >= off ? s[ph][tid - off] : 0;
    __syncthreads();
#pragma unroll
    for (int ph = 0; ph < PH_N; ph++) s[ph][tid] += add[ph];
    __syncthreads();
  }
  int run[PH_N];
#pragma unroll
  for (int ph = 0; ph < PH_N; ph++) run[ph] = s[ph][tid] - sum[ph];
  for (int i = i0; i < i1; i++) {
    int e = B.order[i];
    bool live = B.state[e] == EV_LIVE;
#pragma unroll
    for (int ph = 0; ph < PH_N; ph++) {
      B.prefix[ph * (B.nev + 1) + i] = run[ph];
      if (live) run[ph] += event_tiles(B.ev[e].g, ph, B.tile[ph]);
    }
  }
  if (tid == NT - 1) {
#pragma unroll
    for (int ph = 0; ph < PH_N; ph++) B.prefix[ph * (B.nev + 1) + B.nev] = s[ph][tid];
  }
}

static __global__ void __launch_bounds__(BEGIN_THREADS) batch_stage_begin_kernel(BatchDev B, int irk, int roles) {
  __shared__ int s[PH_N][BEGIN_THREADS];
  stage_begin_block<BEGIN_THREADS>(B, irk, roles, s);
}

// face sweep along DIR over the face tiles of all live events
template <int KIND, int DIR, int REC>
__global__ void ECHO_FACE_BOUNDS(KIND) batch_faces_kernel(FaceArgs base, BatchDev B, int nv) {
  __shared__ FaceArgs sA;
  __shared__ double red[4];
  __shared__ int s_tile;
  const int* pre = B.prefix + DIR * (B.nev + 1);
  const int total = pre[B.nev];
  if (threadIdx.x == 0) sA = base;
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    if (threadIdx.x == 0) {
      int i = tile_slot(pre, B.nev, t);
      int e = B.order[i];
      const EvDesc& d = B.ev[e];
      sA.g = d.g;
      sA.v = base.v + (size_t)nv * d.cell;
      sA.F = base.F + (size_t)nv * d.face[DIR];
      sA.WD = base.WD ? base.WD + (size_t)8 * d.face[DIR] : nullptr;
      sA.sc = B.sc + e;
      s_tile = t - pre[i];
    }
    __syncthreads();
    const int T = B.tile[DIR];
    double am = 0.0;
    for (int sub = 0; sub < T; sub += BATCH_NT) {
      size_t fid = (size_t)s_tile * T + sub + threadIdx.x;
      double a = fid < faces_of<DIR>(sA.g) ? face_flux<KIND, DIR, REC>(sA, fid) : 0.0;
      am = a > am ? a : am;
    }
    block_max_atomic(am, &sA.sc->amax_bits[DIR], red);
    __syncthreads();  // sA, red and s_tile are rewritten for the next tile
  }
}

// the scalar logic of evolve_main per live event (dt of each event)
static __global__ void batch_scalars_kernel(ScalarArgs base, BatchDev B) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= B.nev || B.state[e] != EV_LIVE) return;
  ScalarArgs A = base;
  A.sc = B.sc + e;
  A.g = B.ev[e].g;
  stage_scalars(A);
}

// cell update over the cell tiles of all live events
template <int KIND, bool SEED, bool IMEX = false>
__global__ void ECHO_UPDATE_BOUNDS(KIND, SEED) batch_update_kernel(UpdateArgs base, BatchDev B, int nv) {
  __shared__ UpdateArgs sA;
  __shared__ int s_tile;
  const int* pre = B.prefix + PH_CELL * (B.nev + 1);
  const int total = pre[B.nev];
  if (threadIdx.x == 0) sA = base;
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    if (threadIdx.x == 0) {
      int i = tile_slot(pre, B.nev, t);
      int e = B.order[i];
      const EvDesc& d = B.ev[e];
      const size_t cv = (size_t)nv * d.cell, c4 = (size_t)4 * d.cell;
      sA.g = d.g;
      sA.Fx = base.Fx ? base.Fx + (size_t)nv * d.face[0] : nullptr;
      sA.Fy = base.Fy ? base.Fy + (size_t)nv * d.face[1] : nullptr;
      sA.Fz = base.Fz ? base.Fz + (size_t)nv * d.face[2] : nullptr;
      sA.WDx = base.WDx ? base.WDx + (size_t)8 * d.face[0] : nullptr;
      sA.WDy = base.WDy ? base.WDy + (size_t)8 * d.face[1] : nullptr;
      sA.WDz = base.WDz ? base.WDz + (size_t)8 * d.face[2] : nullptr;
      sA.vin = base.vin + cv;
      sA.vout = base.vout + cv;
      sA.uin = base.uin + cv;
      sA.uout = base.uout + cv;
      sA.u0 = base.u0 + cv;
      sA.vnew = base.vnew + c4;
      sA.vold = base.vold + c4;
      sA.vsnap = base.vsnap ? base.vsnap + c4 : nullptr;
      sA.du_out = base.du_out ? base.du_out + cv : nullptr;
      sA.fail = base.fail + d.cell;
      sA.sc = B.sc + e;
      s_tile = t - pre[i];
    }
    __syncthreads();
    const int T = B.tile[PH_CELL];
    for (int sub = 0; sub < T; sub += BATCH_NT) {
      size_t c = (size_t)s_tile * T + sub + threadIdx.x;
      update_cell<KIND, SEED, IMEX>(sA, c, c < sA.g.ncell);
    }
    __syncthreads();
  }
}

// neighbour-average repair: one block per event, which returns at once
// unless the event is live and has failed cells
template <int KIND>
__global__ void __launch_bounds__(256) batch_repair_kernel(RepairArgs base, BatchDev B, int nv) {
  const int e = blockIdx.x;
  if (B.state[e] != EV_LIVE || B.sc[e].nfail == 0) return;
  __shared__ RepairArgs sA;
  __shared__ int s_any, s_stop;
  __shared__ unsigned s_list[ECHO_REPAIR_LIST];
  if (threadIdx.x == 0) {
    const EvDesc& d = B.ev[e];
    const size_t cv = (size_t)nv * d.cell;
    sA = base;
    sA.g = d.g;
    sA.vold = base.vold + cv;
    sA.vnew = base.vnew + cv;
    sA.u = base.u + cv;
    sA.fail = base.fail + d.cell;
    sA.sc = B.sc + e;
  }
  __syncthreads();
  repair_grid<KIND, ECHO_REPAIR_LIST>(sA, s_any, s_stop, s_list);
}

// evolve_smooth_viscosity over the cell tiles of all live events
template <int KIND>
__global__ void __launch_bounds__(128) batch_smooth_kernel(SmoothArgs base, BatchDev B, int nv) {
  __shared__ SmoothArgs sA;
  __shared__ int s_tile;
  const int* pre = B.prefix + PH_CELL * (B.nev + 1);
  const int total = pre[B.nev];
  if (threadIdx.x == 0) sA = base;
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    if (threadIdx.x == 0) {
      int i = tile_slot(pre, B.nev, t);
      int e = B.order[i];
      const EvDesc& d = B.ev[e];
      sA.g = d.g;
      sA.v = base.v + (size_t)nv * d.cell;
      sA.u = base.u + (size_t)nv * d.cell;
      sA.sc = B.sc + e;
      s_tile = t - pre[i];
    }
    __syncthreads();
    const int T = B.tile[PH_CELL];
    for (int sub = 0; sub < T; sub += BATCH_NT) {
      size_t c = (size_t)s_tile * T + sub + threadIdx.x;
      if (c < sA.g.ncell) smooth_cell<KIND>(sA, c);
    }
    __syncthreads();
  }
}

// system_prim2cons over the cell tiles of all live events (upload without u)
template <int KIND>
__global__ void __launch_bounds__(128) batch_p2c_kernel(DevPhys P, BatchDev B, int nv, int coordinates,
                                                        double* v, double* u) {
  const int* pre = B.prefix + PH_CELL * (B.nev + 1);
  const int total = pre[B.nev];
  const int T = B.tile[PH_CELL];
  for (long long tt = blockIdx.x; tt < (long long)total * (T / BATCH_NT); tt += gridDim.x) {
    const int t = (int)(tt / (T / BATCH_NT)), sub = (int)(tt % (T / BATCH_NT)) * BATCH_NT;
    int i = tile_slot(pre, B.nev, t);
    int e = B.order[i];
    const EvDesc& d = B.ev[e];
    size_t c = (size_t)(t - pre[i]) * T + sub + threadIdx.x;
    if (c >= d.g.ncell) continue;
    DevScalars* sc = B.sc + e;
    const Metric M = make_metric(coordinates, sc->t, sc->t3);
    double* ve = v + (size_t)nv * d.cell;
    double* ue = u + (size_t)nv * d.cell;
    double vv[Traits<KIND>::NV], uu[Traits<KIND>::NV];
#pragma unroll
    for (int k = 0; k < Traits<KIND>::NV; k++) vv[k] = ve[(size_t)k * d.g.ncell + c];
    int err = prim2cons<KIND>(P, M, vv, uu);
    if (err) atomicMin(&sc->err_key, ((unsigned long long)c << 20) | (unsigned long long)err);
#pragma unroll
    for (int k = 0; k < Traits<KIND>::NV; k++) {
      ve[(size_t)k * d.g.ncell + c] = vv[k];
      ue[(size_t)k * d.g.ncell + c] = uu[k];
    }
  }
}

// Monte Carlo Glauber initial energy density of every event
// (generate_energy_density_profile, glaubermc.f90:686-873): the sources of
// event e (participants and binary-collision points, src[3*i] = x,
// src[3*i+1] = y, src[3*i+2] = weight, i in [off[e], off[e+1])) smeared by a
// normalised 2D Gaussian of width sigma, summed at every cell centre (the
// same in every eta slice).  The raw sum goes to v[KPR]; the block max goes
// to the event's amax_bits[0] for the normalisation.
enum { SMEAR_CHUNK = 256 };
static __global__ void __launch_bounds__(128) batch_smear_kernel(BatchDev B, int nv, const double* __restrict__ src,
                                                                 const long long* __restrict__ off, double sigma,
                                                                 double* v) {
  __shared__ double sx[SMEAR_CHUNK], sy[SMEAR_CHUNK], sw[SMEAR_CHUNK];
  __shared__ double red[4];
  const int* pre = B.prefix + PH_CELL * (B.nev + 1);
  const int total = pre[B.nev];
  const double norm = 1.0 / (2 * M_PI * sigma * sigma);
  const double two_s2 = 2 * sigma * sigma;
  const int T = B.tile[PH_CELL];
  for (long long tt = blockIdx.x; tt < (long long)total * (T / BATCH_NT); tt += gridDim.x) {
    const int t = (int)(tt / (T / BATCH_NT)), sub = (int)(tt % (T / BATCH_NT)) * BATCH_NT;
    const int i = tile_slot(pre, B.nev, t);
    const int e = B.order[i];
    const EvDesc& d = B.ev[e];
    const size_t c = (size_t)(t - pre[i]) * T + sub + threadIdx.x;
    const bool active = c < d.g.ncell;
    double x = 0., y = 0.;
    if (active) {
      int ix = (int)(c % d.g.nx);
      int iy = (int)((c / d.g.nx) % d.g.ny);
      x = d.x1 + ((double)(ix + 1) - 0.5) * d.dx;
      y = d.y1 + ((double)(iy + 1) - 0.5) * d.dy;
    }
    double sum = 0.;
    for (long long s0 = off[e]; s0 < off[e + 1]; s0 += SMEAR_CHUNK) {
      const int m = (int)min((long long)SMEAR_CHUNK, off[e + 1] - s0);
      __syncthreads();
      for (int q = threadIdx.x; q < m; q += blockDim.x) {
        sx[q] = src[3 * (s0 + q)];
        sy[q] = src[3 * (s0 + q) + 1];
        sw[q] = src[3 * (s0 + q) + 2];
      }
      __syncthreads();
      for (int q = 0; q < m; q++) {
        double ddx = x - sx[q], ddy = y - sy[q];
        sum = sum + sw[q] * norm * exp(-(ddx * ddx + ddy * ddy) / two_s2);
      }
    }
    if (active) v[(size_t)nv * d.cell + (size_t)KPR * d.g.ncell + c] = sum;
    block_max_atomic(active ? sum : 0., &B.sc[e].amax_bits[0], red);
    __syncthreads();
  }
}

// primitives from the smeared density: e = peak * S / max(S) + ENEZERO, p(e)
// from the EoS (get_pressure, eos.f90:399-464), rho = 1, every other
// variable 0
static __global__ void __launch_bounds__(128) batch_glauber_fill_kernel(DevPhys P, BatchDev B, int nv, double peak,
                                                                        double enezero, double* v) {
  const int* pre = B.prefix + PH_CELL * (B.nev + 1);
  const int total = pre[B.nev];
  const int T = B.tile[PH_CELL];
  for (long long tt = blockIdx.x; tt < (long long)total * (T / BATCH_NT); tt += gridDim.x) {
    const int t = (int)(tt / (T / BATCH_NT)), sub = (int)(tt % (T / BATCH_NT)) * BATCH_NT;
    const int i = tile_slot(pre, B.nev, t);
    const int e = B.order[i];
    const EvDesc& d = B.ev[e];
    const size_t c = (size_t)(t - pre[i]) * T + sub + threadIdx.x;
    if (c >= d.g.ncell) continue;
    double* ve = v + (size_t)nv * d.cell;
    const double emax = __longlong_as_double((long long)B.sc[e].amax_bits[0]);
    double en = ve[(size_t)KPR * d.g.ncell + c];
    if (emax > 0.) en = en * (peak / emax);
    en = en + enezero;
    double pr = 0., d1, d2;
    int err = eos_pressure(P, 1.0, en, &pr, &d1, &d2);
    if (err) atomicMin(&B.sc[e].err_key, ((unsigned long long)c << 20) | (unsigned long long)err);
    for (int k = 0; k < nv; k++) ve[(size_t)k * d.g.ncell + c] = 0.;
    ve[(size_t)KRH * d.g.ncell + c] = 1.;
    ve[(size_t)KPR * d.g.ncell + c] = pr;
  }
}

// check_temp of every live event at the top of its time loop (echo.f90:189):
// the event's maximum of check_value over its cells, into its check_bits
static __global__ void __launch_bounds__(128) batch_check_kernel(DevPhys P, BatchDev B, int nv,
                                                                 const double* __restrict__ v) {
  __shared__ double red[4];
  const int* pre = B.prefix + PH_CELL * (B.nev + 1);
  const int total = pre[B.nev];
  const int T = B.tile[PH_CELL];
  for (long long tt = blockIdx.x; tt < (long long)total * (T / BATCH_NT); tt += gridDim.x) {
    const int t = (int)(tt / (T / BATCH_NT)), sub = (int)(tt % (T / BATCH_NT)) * BATCH_NT;
    const int i = tile_slot(pre, B.nev, t);
    const int e = B.order[i];
    const EvDesc& d = B.ev[e];
    const size_t c = (size_t)(t - pre[i]) * T + sub + threadIdx.x;
    double x = 0.;
    if (c < d.g.ncell) {
      const double* ve = v + (size_t)nv * d.cell;
      x = check_value(P, B.freeze_type, ve[(size_t)KRH * d.g.ncell + c], ve[(size_t)KPR * d.g.ncell + c]);
    }
    block_max_atomic(x, &B.sc[e].check_bits, red);
    __syncthreads();
  }
}

// end of step per live event (echo.f90:206-241): a crash ends the event,
// otherwise t advances and the step counts; `roles` are those after the step
static __global__ void batch_end_kernel(BatchDev B, int coordinates, int roles) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= B.nev || B.state[e] != EV_LIVE) return;
  DevScalars* sc = B.sc + e;
  if (sc->err_key != ~0ull) {
    B.state[e] = EV_CRASHED;
    B.roles[e] = roles;
    return;
  }
  end_step_scalars(sc, coordinates);
  B.steps[e] += 1;
  sc->check_bits = 0;  // the next step's check_temp maximum starts from 0
}

// ---------------------------------------------------------------------------
// one launch per stage: every phase of a stage in one cooperative kernel
// ---------------------------------------------------------------------------
// Grid-wide barrier between the phases.  The launch is cooperative, so all
// CTAs are resident and every wait ends; the wait is still bounded (4 s of
// the global timer), after which the CTA sets the timeout flag and every CTA
// leaves the kernel at its next barrier.  bar[0] counts arrivals, bar[1] is
// the generation, bar[2] the timeout flag; the host zeroes them before every
// launch.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool grid_barrier(unsigned* bar) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = bar + 1;
    const unsigned gen = *vgen;
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      while (*vgen == gen) {
        if (global_ns() - t0 > 4000000000ull) {
          atomicExch(bar + 2, 1u);
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile unsigned*)(bar + 2) == 0u;
}

struct BatchStageArgs {
  FaceArgs face;     // per-event pointers and per-direction boundary codes are set per tile
  BcDir bc[3];
  int bc_uniform[3], bc_signed[3];
  double* F[3];      // face-flux arenas
  double* WD[3];     // viscous u^mu face-state arenas (or null)
  UpdateArgs upd;    // as launch_batch_update builds it
  ScalarArgs sca;
  RepairArgs rep;    // with the roles after the update
  SmoothArgs smo;
  BatchDev B;
  int nv, irk, roles, smooth;
  unsigned* bar;
};

// the face and update kernels' register bounds, whichever is lower
#define ECHO_BATCH_STAGE_MINB(KIND, SEED)                                                             \
  ((KIND) == KIND_VISC ? (ECHO_FACE_MINB_VISC > ECHO_UPDATE_MINB_VISC ? ECHO_FACE_MINB_VISC          \
                                                                      : ECHO_UPDATE_MINB_VISC)       \
   : (SEED)          ? (ECHO_FACE_MINB > ECHO_UPDATE_MINB_SEED ? ECHO_FACE_MINB : ECHO_UPDATE_MINB_SEED) \
                     : (ECHO_FACE_MINB > ECHO_UPDATE_MINB ? ECHO_FACE_MINB : ECHO_UPDATE_MINB))

template <int KIND, bool SEED, bool IMEX>
__global__ void __launch_bounds__(BATCH_NT, ECHO_BATCH_STAGE_MINB(KIND, SEED)) batch_stage_kernel(BatchStageArgs S) {
  __shared__ union {
    FaceArgs f;
    UpdateArgs u;
    RepairArgs r;
    SmoothArgs s;
  } sA;
  __shared__ int sbeg[PH_N][BATCH_NT];
  __shared__ double red[BATCH_NT / 32];
  __shared__ int s_tile, s_dir, s_any, s_stop;
  const BatchDev& B = S.B;
  // 0. stop and crash tests, per-stage resets, tile lists (one CTA)
  if (blockIdx.x == 0) stage_begin_block<BATCH_NT>(B, S.irk, S.roles, sbeg);
  if (!grid_barrier(S.bar)) return;
  // 1. face sweeps: the x, y and z tile lists one after the other
  {
    const int* pre[3] = {B.prefix, B.prefix + (B.nev + 1), B.prefix + 2 * (B.nev + 1)};
    const int tot[3] = {pre[0][B.nev], pre[1][B.nev], pre[2][B.nev]};
    for (int t = blockIdx.x; t < tot[0] + tot[1] + tot[2]; t += gridDim.x) {
      if (threadIdx.x == 0) {
        int d = t < tot[0] ? 0 : t < tot[0] + tot[1] ? 1 : 2;
        int tl = t - (d > 0 ? tot[0] : 0) - (d > 1 ? tot[1] : 0);
        int i = tile_slot(pre[d], B.nev, tl);
        int e = B.order[i];
        const EvDesc& ed = B.ev[e];
        sA.f = S.face;
        sA.f.g = ed.g;
        sA.f.v = S.face.v + (size_t)S.nv * ed.cell;
        sA.f.F = S.F[d] + (size_t)S.nv * ed.face[d];
        sA.f.WD = S.WD[d] ? S.WD[d] + (size_t)8 * ed.face[d] : nullptr;
        sA.f.sc = B.sc + e;
        sA.f.bc = S.bc[d];
        sA.f.bc_uniform = S.bc_uniform[d];
        sA.f.bc_signed = S.bc_signed[d];
        s_tile = tl - pre[d][i];
        s_dir = d;
      }
      __syncthreads();
      const int d = s_dir, T = B.tile[d];
      double am = 0.0;
      for (int sub = 0; sub < T; sub += BATCH_NT) {
        size_t fid = (size_t)s_tile * T + sub + threadIdx.x;
        double a = 0.0;
        if (d == 0) {
          if (fid < faces_of<0>(sA.f.g)) a = face_flux<KIND, 0, ECHO_REC_WENO5>(sA.f, fid);
        } else if (d == 1) {
          if (fid < faces_of<1>(sA.f.g)) a = face_flux<KIND, 1, ECHO_REC_WENO5>(sA.f, fid);
        } else {
          if (fid < faces_of<2>(sA.f.g)) a = face_flux<KIND, 2, ECHO_REC_WENO5>(sA.f, fid);
        }
        am = a > am ? a : am;
      }
      block_max_atomic(am, &sA.f.sc->amax_bits[d], red);
      __syncthreads();
    }
  }
  if (!grid_barrier(S.bar)) return;
  // 2. the scalar logic of evolve_main per live event (dt)
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < B.nev; e += gridDim.x * blockDim.x) {
    if (B.state[e] != EV_LIVE) continue;
    ScalarArgs A = S.sca;
    A.sc = B.sc + e;
    A.g = B.ev[e].g;
    stage_scalars(A);
  }
  if (!grid_barrier(S.bar)) return;
  // 3. cell update over the cell tiles
  {
    const int* pre = B.prefix + PH_CELL * (B.nev + 1);
    const int total = pre[B.nev];
    const int T = B.tile[PH_CELL];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
      if (threadIdx.x == 0) {
        int i = tile_slot(pre, B.nev, t);
        int e = B.order[i];
        const EvDesc& d = B.ev[e];
        const size_t cv = (size_t)S.nv * d.cell, c4 = (size_t)4 * d.cell;
        const UpdateArgs& base = S.upd;
        sA.u = base;
        sA.u.g = d.g;
        sA.u.Fx = base.Fx ? base.Fx + (size_t)S.nv * d.face[0] : nullptr;
        sA.u.Fy = base.Fy ? base.Fy + (size_t)S.nv * d.face[1] : nullptr;
        sA.u.Fz = base.Fz ? base.Fz + (size_t)S.nv * d.face[2] : nullptr;
        sA.u.WDx = base.WDx ? base.WDx + (size_t)8 * d.face[0] : nullptr;
        sA.u.WDy = base.WDy ? base.WDy + (size_t)8 * d.face[1] : nullptr;
        sA.u.WDz = base.WDz ? base.WDz + (size_t)8 * d.face[2] : nullptr;
        sA.u.vin = base.vin + cv;
        sA.u.vout = base.vout + cv;
        sA.u.uin = base.uin + cv;
        sA.u.uout = base.uout + cv;
        sA.u.u0 = base.u0 + cv;
        sA.u.vnew = base.vnew + c4;
        sA.u.vold = base.vold + c4;
        sA.u.vsnap = base.vsnap ? base.vsnap + c4 : nullptr;
        sA.u.du_out = base.du_out ? base.du_out + cv : nullptr;
        sA.u.fail = base.fail + d.cell;
        sA.u.sc = B.sc + e;
        s_tile = t - pre[i];
      }
      __syncthreads();
      for (int sub = 0; sub < T; sub += BATCH_NT) {
        size_t c = (size_t)s_tile * T + sub + threadIdx.x;
        update_cell<KIND, SEED, IMEX>(sA.u, c, c < sA.u.g.ncell);
      }
      __syncthreads();
    }
  }
  if (!grid_barrier(S.bar)) return;
  // 4. neighbour-average repair: one CTA per event with failed cells
  for (int e = blockIdx.x; e < B.nev; e += gridDim.x) {
    if (B.state[e] != EV_LIVE || B.sc[e].nfail == 0) continue;
    if (threadIdx.x == 0) {
      const EvDesc& d = B.ev[e];
      const size_t cv = (size_t)S.nv * d.cell;
      sA.r = S.rep;
      sA.r.g = d.g;
      sA.r.vold = S.rep.vold + cv;
      sA.r.vnew = S.rep.vnew + cv;
      sA.r.u = S.rep.u + cv;
      sA.r.fail = S.rep.fail + d.cell;
      sA.r.sc = B.sc + e;
    }
    __syncthreads();
    repair_grid<KIND, 0>(sA.r, s_any, s_stop, nullptr);
    __syncthreads();
  }
  if (!S.smooth) return;
  if (!grid_barrier(S.bar)) return;
  // 5. evolve_smooth_viscosity over the cell tiles
  {
    const int* pre = B.prefix + PH_CELL * (B.nev + 1);
    const int total = pre[B.nev];
    const int T = B.tile[PH_CELL];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
      if (threadIdx.x == 0) {
        int i = tile_slot(pre, B.nev, t);
        int e = B.order[i];
        const EvDesc& d = B.ev[e];
        sA.s = S.smo;
        sA.s.g = d.g;
        sA.s.v = S.smo.v + (size_t)S.nv * d.cell;
        sA.s.u = S.smo.u + (size_t)S.nv * d.cell;
        sA.s.sc = B.sc + e;
        s_tile = t - pre[i];
      }
      __syncthreads();
      for (int sub = 0; sub < T; sub += BATCH_NT) {
        size_t c = (size_t)s_tile * T + sub + threadIdx.x;
        if (c < sA.s.g.ncell) smooth_cell<KIND>(sA.s, c);
      }
      __syncthreads();
    }
  }
}

}  // namespace echo

// The batch context.  Arrays are arenas over all events: event e's block of
// a cell array starts at nv * ev[e].cell (nv variables of ncell_e cells each,
// x fastest: the single-grid layout), of a face array at nv * ev[e].face[d],
// of the u^mu face states at 8 * ev[e].face[d], of vnewstep/vold at
// 4 * ev[e].cell.
struct EchoBatch {
  EchoParams p;
  int kind, nv, nev;
  DevPhys P;
  BcDir bc[3];
  int bc_uniform[3], bc_signed[3];
  cudaStream_t stream;
  std::vector<EvDesc> h_ev;
  EvDesc* d_ev;
  size_t ncell, nfaces[3];
  bool has_dir[3];
  double* d_v[2];
  int vcur;
  double* d_u[2];
  int ucur;
  double *d_F[3], *d_WD[3];
  double* d_vh[2];
  int vn;
  unsigned char* d_fail;
  DevScalars* d_sc;
  DevScalars* h_sc;  // pinned, nev
  int* d_state;
  int* h_state;      // pinned, nev
  long long* d_steps;
  long long* h_steps;  // pinned, nev
  int* d_order;
  int* d_prefix;
  int* d_roles;
  int* h_roles;      // pinned, nev
  double* d_tab;
  int* d_bk;
  double tmax;
  double temp_end;
  int freeze_type;
  int nsm;
  int max_tiles[echo::PH_N];  // tiles with every event live
  int sched[echo::SL_N];      // CTAs per launch of each slot; 0 = one per tile
  int tile[echo::PH_N];       // tile length of each list (128, 256 or 512)
  // how a stage runs: 0 = one launch per phase (faces, scalars, update,
  // repair, smoothing); 1 = one cooperative launch per stage with grid-wide
  // barriers between the phases (coop_grid CTAs, all resident)
  int mode;
  unsigned coop_grid;
  unsigned* d_bar;            // grid barrier: arrival count, generation, timeout flag
  bool graphs_off;            // the stream cannot capture this mode's launches
  std::vector<double> tune;   // the autotuner's candidates: (what, shape, CTAs, ms) rows
  unsigned* d_mlp_frag;  // learned con2prim seed: BF16 weight fragments
  float* d_mlp_par;      //   biases and normalisation
  cudaGraphExec_t graph[8];
  bool graph_ok[8];
  std::vector<std::pair<int, cudaEvent_t>>* marks;
};

namespace echo {

inline BatchDev batch_dev(const EchoBatch* b) {
  BatchDev B;
  B.ev = b->d_ev;
  B.sc = b->d_sc;
  B.state = b->d_state;
  B.steps = b->d_steps;
  B.order = b->d_order;
  B.prefix = b->d_prefix;
  B.roles = b->d_roles;
  B.nev = b->nev;
  B.tmax = b->tmax;
  B.temp_end = b->temp_end;
  B.freeze_type = b->freeze_type;
  for (int ph = 0; ph < PH_N; ph++) B.tile[ph] = b->tile[ph];
  return B;
}

// grid of a launch of slot `sl` over tile list `ph`
inline unsigned batch_grid(const EchoBatch* b, int sl, int ph) {
  int g = b->sched[sl] > 0 ? b->sched[sl] : b->max_tiles[ph];
  if (g > b->max_tiles[ph]) g = b->max_tiles[ph];
  return (unsigned)(g > 0 ? g : 1);
}

inline void batch_mark(EchoBatch* b, int cls) {
  if (!b->marks) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, b->stream);
  b->marks->push_back({cls, e});
}

template <int KIND>
void launch_batch_faces(EchoBatch* b, int dir);
template <int KIND>
void launch_batch_update(EchoBatch* b, int irk);
template <int KIND>
void launch_batch_repair_smooth(EchoBatch* b);
template <int KIND>
void launch_batch_p2c(EchoBatch* b);
// one cooperative launch for stage irk (mode 1); grid = coop_grid, or, when
// coop_grid is 0, the largest co-resident grid (returned in *grid_max)
template <int KIND>
int launch_batch_stage(EchoBatch* b, int irk, unsigned* grid_max);
// occupancy (resident CTAs per SM) of the kernels of each slot
template <int KIND>
void batch_occupancy(const EchoBatch* b, int* per_sm);

}  // namespace echo
