// launchers.cuh -- definitions of the per-equation-set launch functions;
// included only by kind_*.cu, each of which instantiates one equation set.
#pragma once

#include "batch.cuh"
#include "stage.cuh"

namespace echo {

// ---------------------------------------------------------------------------
// kernel dispatch
// ---------------------------------------------------------------------------
template <int KIND>
void launch_faces(EchoCtx* c, int dir) {
  FaceArgs A;
  A.P = c->P;
  A.g = c->g;
  A.bc = c->bc[dir];
  A.bc_uniform = c->bc_uniform[dir];
  A.bc_signed = c->bc_signed[dir];
  A.v = c->d_v[c->vcur];
  A.F = c->d_F[dir];
  A.WD = c->d_WD[dir];
  A.sc = c->d_sc;
  A.coordinates = c->p.coordinates;
  unsigned blocks = (unsigned)((c->nfaces[dir] + 127) / 128);
#ifndef ECHO_EXACT
  // product build: the cell-centred sweep in segments of face_mode cells
  if (c->p.recal == ECHO_REC_WENO5 && c->face_mode > 0) {
    const Grid& g = c->g;
    if (c->face_mode == 8) {
      if (dir == 0) faces_seg_kernel<KIND, 0, 8><<<(unsigned)((seg_warps<0, 8>(g) + 3) / 4), 128, 0, c->stream>>>(A);
      if (dir == 1) faces_seg_kernel<KIND, 1, 8><<<(unsigned)((seg_warps<1, 8>(g) + 3) / 4), 128, 0, c->stream>>>(A);
      if (dir == 2) faces_seg_kernel<KIND, 2, 8><<<(unsigned)((seg_warps<2, 8>(g) + 3) / 4), 128, 0, c->stream>>>(A);
    } else {
      if (dir == 0) faces_seg_kernel<KIND, 0, 16><<<(unsigned)((seg_warps<0, 16>(g) + 3) / 4), 128, 0, c->stream>>>(A);
      if (dir == 1) faces_seg_kernel<KIND, 1, 16><<<(unsigned)((seg_warps<1, 16>(g) + 3) / 4), 128, 0, c->stream>>>(A);
      if (dir == 2) faces_seg_kernel<KIND, 2, 16><<<(unsigned)((seg_warps<2, 16>(g) + 3) / 4), 128, 0, c->stream>>>(A);
    }
    return;
  }
#endif
  if (c->p.recal == ECHO_REC_WENO5) {
    if (dir == 0) faces_kernel<KIND, 0, ECHO_REC_WENO5><<<blocks, 128, 0, c->stream>>>(A);
    if (dir == 1) faces_kernel<KIND, 1, ECHO_REC_WENO5><<<blocks, 128, 0, c->stream>>>(A);
    if (dir == 2) faces_kernel<KIND, 2, ECHO_REC_WENO5><<<blocks, 128, 0, c->stream>>>(A);
  } else {
    if (dir == 0) faces_kernel<KIND, 0, REC_RUNTIME><<<blocks, 128, 0, c->stream>>>(A);
    if (dir == 1) faces_kernel<KIND, 1, REC_RUNTIME><<<blocks, 128, 0, c->stream>>>(A);
    if (dir == 2) faces_kernel<KIND, 2, REC_RUNTIME><<<blocks, 128, 0, c->stream>>>(A);
  }
}

template <int KIND>
void launch_update(EchoCtx* c, int irk, int mode, double* du_out) {
  static const double crk[3][3][2] = {{{0., 1.}, {0., 0.}, {0., 0.}},
                                      {{0., 1.}, {1. / 2., 1. / 2.}, {0., 0.}},
                                      {{0., 1.}, {3. / 4., 1. / 4.}, {1. / 3., 2. / 3.}}};
  UpdateArgs A;
  A.P = c->P;
  A.g = c->g;
  A.Fx = c->d_F[0];
  A.Fy = c->d_F[1];
  A.Fz = c->d_F[2];
  A.WDx = c->d_WD[0];
  A.WDy = c->d_WD[1];
  A.WDz = c->d_WD[2];
  A.vin = c->d_v[c->vcur];
  A.vout = c->d_v[1 - c->vcur];
  A.uin = c->d_u[c->ucur];
  A.uout = irk == 1 ? c->d_u[1 - c->ucur] : c->d_u[c->ucur];
  A.u0 = irk == 1 ? c->d_u[c->ucur] : c->d_u[1 - c->ucur];
  A.vnew = c->d_vh[c->vn];
  A.vold = c->d_vh[1 - c->vn];
  A.du_out = du_out;
  A.fail = c->d_fail;
  A.sc = c->d_sc;
  int nrk = c->p.nrk;
  A.c1 = nrk <= 3 ? crk[nrk - 1][irk - 1][0] : 0.;
  A.c2 = nrk <= 3 ? crk[nrk - 1][irk - 1][1] : 0.;
  A.irk = irk;
  A.nrk = nrk;
  A.divclean = c->p.divclean;
  A.coordinates = c->p.coordinates;
  A.algo = c->p.algo_solver;
  A.mode = mode;
  A.tol = c->p.c2p_tol;
  A.dus_out = nullptr;
  if (Traits<KIND>::RES) {
    if (mode == MODE_RHS) A.dus_out = c->d_dss[irk - 1];
    const int ke[3] = {KEX, KEY, KEZ};
    for (int d = 0; d < 3; d++)
      for (int q = 0; q < 2; q++) A.ebc[d][q] = c->bc[d].c[ke[d]][q];
  }
  A.mlp.frag = c->d_mlp_frag;
  A.mlp.par = c->d_mlp_par;
  A.vsnap = nullptr;
  if (A.algo == ECHO_C2P_MLP && !c->d_mlp_frag) A.algo = ECHO_C2P_NEWTON;  // no network loaded
  unsigned blocks = (unsigned)((c->g.ncell + 127) / 128);
  // the learned seed: RMHD (ideal, resistive) and viscous runs
  constexpr bool CAN_SEED = Traits<KIND>::MHD || Traits<KIND>::VISC;
  if (CAN_SEED && A.algo == ECHO_C2P_MLP && mode == MODE_RK && Traits<KIND>::VISC && c->p.imex)
    update_kernel<KIND, CAN_SEED, Traits<KIND>::VISC><<<blocks, 128, 0, c->stream>>>(A);
  else if (CAN_SEED && A.algo == ECHO_C2P_MLP && mode == MODE_RK)
    update_kernel<KIND, CAN_SEED><<<blocks, 128, 0, c->stream>>>(A);
  else if (Traits<KIND>::VISC && c->p.imex && mode == MODE_RK)
    update_kernel<KIND, false, Traits<KIND>::VISC><<<blocks, 128, 0, c->stream>>>(A);
  else
    update_kernel<KIND, false><<<blocks, 128, 0, c->stream>>>(A);
  if (Traits<KIND>::MHD && !Traits<KIND>::RES && mode == MODE_RK && c2p_alt_algo(A.algo))
    c2p_alt_kernel<KIND><<<blocks, 128, 0, c->stream>>>(c->P, c->g, c->p.coordinates, A.algo, A.tol, c->d_sc, A.uout,
                                                         A.vin, A.vout, c->d_fail);
}

// The fused stage kernel (stage.cuh): the UpdateArgs of launch_update with
// no face arrays, plus the tile decomposition chosen by setup_stage.
template <int KIND>
static UpdateArgs update_args(EchoCtx* c, int irk, int mode, double* du_out) {
  static const double crk[3][3][2] = {{{0., 1.}, {0., 0.}, {0., 0.}},
                                      {{0., 1.}, {1. / 2., 1. / 2.}, {0., 0.}},
                                      {{0., 1.}, {3. / 4., 1. / 4.}, {1. / 3., 2. / 3.}}};
  UpdateArgs A;
  memset(&A, 0, sizeof(A));
  A.P = c->P;
  A.g = c->g;
  A.vin = c->d_v[c->vcur];
  A.vout = c->d_v[1 - c->vcur];
  A.uin = c->d_u[c->ucur];
  A.uout = irk == 1 ? c->d_u[1 - c->ucur] : c->d_u[c->ucur];
  A.u0 = irk == 1 ? c->d_u[c->ucur] : c->d_u[1 - c->ucur];
  A.vnew = c->d_vh[c->vn];
  A.vold = c->d_vh[1 - c->vn];
  A.du_out = du_out;
  A.fail = c->d_fail;
  A.sc = c->d_sc;
  int nrk = c->p.nrk;
  A.c1 = nrk <= 3 ? crk[nrk - 1][irk - 1][0] : 0.;
  A.c2 = nrk <= 3 ? crk[nrk - 1][irk - 1][1] : 0.;
  A.irk = irk;
  A.nrk = nrk;
  A.divclean = c->p.divclean;
  A.coordinates = c->p.coordinates;
  A.algo = c->p.algo_solver;
  A.mode = mode;
  A.tol = c->p.c2p_tol;
  A.dus_out = nullptr;
  if (Traits<KIND>::RES) {
    if (mode == MODE_RHS) A.dus_out = c->d_dss[irk - 1];
    const int ke[3] = {KEX, KEY, KEZ};
    for (int d = 0; d < 3; d++)
      for (int q = 0; q < 2; q++) A.ebc[d][q] = c->bc[d].c[ke[d]][q];
  }
  A.mlp.frag = c->d_mlp_frag;
  A.mlp.par = c->d_mlp_par;
  A.vsnap = nullptr;
  if (A.algo == ECHO_C2P_MLP && !c->d_mlp_frag) A.algo = ECHO_C2P_NEWTON;  // no network loaded
  return A;
}

// the instantiation of stage_kernel a run uses
template <int KIND>
static void* stage_variant(int algo_mlp, int imex) {
  constexpr bool CAN_SEED = Traits<KIND>::MHD || Traits<KIND>::VISC;
  constexpr bool VISC = Traits<KIND>::VISC;
  if (CAN_SEED && algo_mlp && VISC && imex) return (void*)stage_kernel<KIND, CAN_SEED, VISC>;
  if (CAN_SEED && algo_mlp) return (void*)stage_kernel<KIND, CAN_SEED, false>;
  if (VISC && imex) return (void*)stage_kernel<KIND, false, VISC>;
  return (void*)stage_kernel<KIND, false, false>;
}

// Tile, segment and grid of the fused stage for this run: the tile whose
// faces and cells fill a CTA in one pass each and that needs the fewest
// tiles (ties: the fewest CTA threads), then the eta segment length that
// minimises waves x (planes + the extra lower eta face of a segment).
// tx, ty, zseg > 0 force a choice.  Returns 0 and leaves st_ok = 0 when the
// run cannot use the fused stage (the sweep kernels then run).
template <int KIND>
int setup_stage(EchoCtx* c, int tx, int ty, int zseg) {
  typedef Traits<KIND> T;
  const int nw = T::VISC ? 8 : 0;
  c->st_ok = 0;
  const Grid& g = c->g;
  if (c->p.recal != ECHO_REC_WENO5 || g.nx < 3 || g.ny < 3) return 0;
  if (T::MHD && !T::RES && c2p_alt_algo(c->p.algo_solver)) return 0;
  const bool three_d = g.nz > 1;
  int dev = 0, nsm = 148;
  size_t smem_optin = 0;
  {
    int v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    smem_optin = (size_t)v;
  }
  auto threads_of = [](int a, int b) {
    int m = (a + 1) * b;
    if (a * (b + 1) > m) m = a * (b + 1);
    return (m + 31) / 32 * 32;
  };
  if (tx <= 0 || ty <= 0) {
    long long best = -1;
    int bt = 1 << 30;
    for (int a = 6; a <= 32; a++)
      for (int b = 6; b <= 32; b++) {
        int nt = threads_of(a, b);
        if (nt > ECHO_STAGE_NT) continue;
        if (8 * stage_smem_doubles(T::NV, nw, a, b, three_d) > smem_optin / 2) continue;
        long long tiles = (long long)((g.nx + a - 1) / a) * ((g.ny + b - 1) / b);
        if (best < 0 || tiles < best || (tiles == best && nt < bt)) {
          best = tiles;
          bt = nt;
          tx = a;
          ty = b;
        }
      }
    if (best < 0) return 0;
  }
  const int nt = threads_of(tx, ty);
  if (nt > ECHO_STAGE_NT || tx * ty > nt) return 0;
  const size_t smem = 8 * stage_smem_doubles(T::NV, nw, tx, ty, three_d);
  if (smem > smem_optin) return 0;
  int occ = 1 << 30;
  for (int mlp = 0; mlp < 2; mlp++)
    for (int im = 0; im < 2; im++) {
      void* fn = stage_variant<KIND>(mlp, im);
      if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
      int o = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fn, nt, smem) != cudaSuccess) return 0;
      occ = o < occ ? o : occ;
    }
  if (occ < 1) return 0;
  const long long tiles = (long long)((g.nx + tx - 1) / tx) * ((g.ny + ty - 1) / ty);
  const long long slots = (long long)occ * nsm;
  if (zseg <= 0) {
    double best = 1e300;
    zseg = g.nz;
    for (int s = 1; s <= g.nz; s++) {
      int zl = (g.nz + s - 1) / s;
      int nseg = (g.nz + zl - 1) / zl;
      long long waves = (tiles * nseg + slots - 1) / slots;
      double cost = (double)waves * (zl + (three_d ? 0.34 : 0.0));
      if (cost < best - 1e-9) {
        best = cost;
        zseg = zl;
      }
    }
  }
  if (zseg > g.nz) zseg = g.nz;
  const long long nunits = tiles * ((g.nz + zseg - 1) / zseg);
  c->st_tx = tx;
  c->st_ty = ty;
  c->st_zseg = zseg;
  c->st_nt = nt;
  c->st_smem = smem;
  c->st_grid = (unsigned)(nunits < slots ? nunits : slots);
  c->st_ok = 1;
  return 1;
}

template <int KIND>
void launch_stage(EchoCtx* c, int irk, int mode, double* du_out) {
  StageArgs S;
  memset(&S, 0, sizeof(S));
  S.U = update_args<KIND>(c, irk, mode, du_out);
  for (int d = 0; d < 3; d++) S.bc[d] = c->bc[d];
  S.tx = c->st_tx;
  S.ty = c->st_ty;
  S.ntx = (c->g.nx + S.tx - 1) / S.tx;
  S.nty = (c->g.ny + S.ty - 1) / S.ty;
  S.zseg = c->st_zseg;
  S.nunits = (long long)S.ntx * S.nty * ((c->g.nz + S.zseg - 1) / S.zseg);
  void* fn = stage_variant<KIND>(S.U.algo == ECHO_C2P_MLP && mode == MODE_RK, c->p.imex && mode == MODE_RK);
  void* args[] = {&S};
  cudaLaunchKernel(fn, dim3(c->st_grid), dim3(c->st_nt), args, c->st_smem, c->stream);
}

template <int KIND>
void launch_repair_smooth(EchoCtx* c, int what) {
  RepairArgs R;
  R.P = c->P;
  R.g = c->g;
  R.vold = c->d_v[c->vcur];
  R.vnew = c->d_v[1 - c->vcur];
  R.u = c->d_u[c->ucur];
  R.fail = c->d_fail;
  R.sc = c->d_sc;
  R.coordinates = c->p.coordinates;
  R.algo = c->p.algo_solver;
  R.maxspeed = c->p.maxspeed;
  R.tol = c->p.c2p_tol;
  // the con2prim of the implicit stages 2..4 (what == 1) of a resistive run
  // solves Ohm's law, the repair's too
  R.h_alpha = (Traits<KIND>::RES && what == 1) ? 0.24169426078821 : 0.;
  if (what & 1) repair_kernel<KIND><<<1, 256, 0, c->stream>>>(R);
  if ((what & 2) && KIND == KIND_VISC && c->p.enable_smooth_viscosity) {
    SmoothArgs S;
    S.P = c->P;
    S.g = c->g;
    S.v = c->d_v[1 - c->vcur];
    S.u = c->d_u[c->ucur];
    S.sc = c->d_sc;
    S.coordinates = c->p.coordinates;
    S.smooth_pressure = c->p.smooth_pressure;
    unsigned blocks = (unsigned)((c->g.ncell + 255) / 256);
    smooth_kernel<KIND><<<blocks, 256, 0, c->stream>>>(S);
  }
}

template <int KIND>
void launch_p2c(EchoCtx* c) {
  unsigned blocks = (unsigned)((c->g.ncell + 255) / 256);
  prim2cons_kernel<KIND><<<blocks, 256, 0, c->stream>>>(c->P, c->g, c->p.coordinates, c->d_sc,
                                                        c->d_v[c->vcur], c->d_u[c->ucur]);
}


// IMEX-SSP combination of stage `stage` (2..4) or the final one (5); the
// caller has already made U[ucur] the u being built and U[1-ucur] = u0
template <int KIND>
void launch_ssp_combine(EchoCtx* c, int stage) {
  SspArgs A;
  A.P = c->P;
  A.g = c->g;
  A.u0 = c->d_u[1 - c->ucur];
  A.du1 = c->d_dussp[0];
  A.du2 = c->d_dussp[1];
  A.du3 = c->d_dussp[2];
  A.du4 = c->d_dussp[3];
  A.ds1 = c->d_dss[0];
  A.ds2 = c->d_dss[1];
  A.ds3 = c->d_dss[2];
  A.ds4 = c->d_dss[3];
  A.ds_out = nullptr;
  A.uout = c->d_u[c->ucur];
  A.vin = c->d_v[c->vcur];
  A.vout = c->d_v[1 - c->vcur];
  A.fail = c->d_fail;
  A.sc = c->d_sc;
  A.stage = stage;
  A.coordinates = c->p.coordinates;
  A.algo = c->p.algo_solver;
  A.divclean = c->p.divclean;
  A.tol = c->p.c2p_tol;
  A.mlp.frag = c->d_mlp_frag;
  A.mlp.par = c->d_mlp_par;
  if (A.algo == ECHO_C2P_MLP && !c->d_mlp_frag) A.algo = ECHO_C2P_NEWTON;
  unsigned blocks = (unsigned)((c->g.ncell + 127) / 128);
  constexpr bool CAN_SEED = Traits<KIND>::MHD || Traits<KIND>::VISC;
  if (CAN_SEED && A.algo == ECHO_C2P_MLP)
    ssp_combine_kernel<KIND, CAN_SEED><<<blocks, 128, 0, c->stream>>>(A);
  else
    ssp_combine_kernel<KIND, false><<<blocks, 128, 0, c->stream>>>(A);
  if (Traits<KIND>::MHD && !Traits<KIND>::RES && c2p_alt_algo(A.algo))
    c2p_alt_kernel<KIND><<<blocks, 128, 0, c->stream>>>(c->P, c->g, c->p.coordinates, A.algo, A.tol, c->d_sc, A.uout,
                                                         A.vin, A.vout, c->d_fail);
}

// resistive IMEX-SSP first stage: the implicit solve from u^n (U[ucur]) and
// the stiff E right-hand side of stage 1
template <int KIND>
void launch_ssp_stage1(EchoCtx* c) {
  if constexpr (!Traits<KIND>::RES) {
    (void)c;
    return;
  } else {
  SspArgs A;
  A.P = c->P;
  A.g = c->g;
  A.u0 = c->d_u[c->ucur];
  A.du1 = A.du2 = A.du3 = A.du4 = nullptr;
  A.ds1 = A.ds2 = A.ds3 = A.ds4 = nullptr;
  A.ds_out = c->d_dss[0];
  A.uout = nullptr;
  A.vin = c->d_v[c->vcur];
  A.vout = nullptr;
  A.fail = c->d_fail;
  A.sc = c->d_sc;
  A.stage = 1;
  A.coordinates = c->p.coordinates;
  A.algo = c->p.algo_solver;
  A.divclean = c->p.divclean;
  A.tol = c->p.c2p_tol;
  A.mlp.frag = c->d_mlp_frag;
  A.mlp.par = c->d_mlp_par;
  unsigned blocks = (unsigned)((c->g.ncell + 127) / 128);
  if (A.algo == ECHO_C2P_MLP && c->d_mlp_frag)
    ssp_stage1_kernel<KIND, true><<<blocks, 128, 0, c->stream>>>(A);
  else
    ssp_stage1_kernel<KIND, false><<<blocks, 128, 0, c->stream>>>(A);
  }
}

// ---------------------------------------------------------------------------
// batched launches (one launch per phase over all live events)
// ---------------------------------------------------------------------------
template <int KIND>
void launch_batch_faces(EchoBatch* b, int dir) {
  FaceArgs A;
  A.P = b->P;
  A.g = Grid{};
  A.bc = b->bc[dir];
  A.bc_uniform = b->bc_uniform[dir];
  A.bc_signed = b->bc_signed[dir];
  A.v = b->d_v[b->vcur];
  A.F = b->d_F[dir];
  A.WD = b->d_WD[dir];
  A.sc = nullptr;
  A.coordinates = b->p.coordinates;
  BatchDev B = batch_dev(b);
  unsigned grid = batch_grid(b, SL_FX + dir, PH_FX + dir);
  if (b->p.recal == ECHO_REC_WENO5) {
    if (dir == 0) batch_faces_kernel<KIND, 0, ECHO_REC_WENO5><<<grid, 128, 0, b->stream>>>(A, B, b->nv);
    if (dir == 1) batch_faces_kernel<KIND, 1, ECHO_REC_WENO5><<<grid, 128, 0, b->stream>>>(A, B, b->nv);
    if (dir == 2) batch_faces_kernel<KIND, 2, ECHO_REC_WENO5><<<grid, 128, 0, b->stream>>>(A, B, b->nv);
  } else {
    if (dir == 0) batch_faces_kernel<KIND, 0, REC_RUNTIME><<<grid, 128, 0, b->stream>>>(A, B, b->nv);
    if (dir == 1) batch_faces_kernel<KIND, 1, REC_RUNTIME><<<grid, 128, 0, b->stream>>>(A, B, b->nv);
    if (dir == 2) batch_faces_kernel<KIND, 2, REC_RUNTIME><<<grid, 128, 0, b->stream>>>(A, B, b->nv);
  }
}

// the batch runs the learned seed: a network is loaded and the equations have one
template <int KIND>
inline bool batch_seeded(const EchoBatch* b) {
  return (Traits<KIND>::MHD || Traits<KIND>::VISC) && b->p.algo_solver == ECHO_C2P_MLP && b->d_mlp_frag;
}

template <int KIND>
void launch_batch_update(EchoBatch* b, int irk) {
  static const double crk[3][3][2] = {{{0., 1.}, {0., 0.}, {0., 0.}},
                                      {{0., 1.}, {1. / 2., 1. / 2.}, {0., 0.}},
                                      {{0., 1.}, {3. / 4., 1. / 4.}, {1. / 3., 2. / 3.}}};
  UpdateArgs A;
  A.P = b->P;
  A.g = Grid{};
  A.Fx = b->d_F[0];
  A.Fy = b->d_F[1];
  A.Fz = b->d_F[2];
  A.WDx = b->d_WD[0];
  A.WDy = b->d_WD[1];
  A.WDz = b->d_WD[2];
  A.vin = b->d_v[b->vcur];
  A.vout = b->d_v[1 - b->vcur];
  A.uin = b->d_u[b->ucur];
  A.uout = irk == 1 ? b->d_u[1 - b->ucur] : b->d_u[b->ucur];
  A.u0 = irk == 1 ? b->d_u[b->ucur] : b->d_u[1 - b->ucur];
  A.vnew = b->d_vh[b->vn];
  A.vold = b->d_vh[1 - b->vn];
  A.vsnap = (Traits<KIND>::VISC && irk == 1) ? b->d_vh[b->vn] : nullptr;
  A.du_out = nullptr;
  A.fail = b->d_fail;
  A.sc = nullptr;
  int nrk = b->p.nrk;
  A.c1 = crk[nrk - 1][irk - 1][0];
  A.c2 = crk[nrk - 1][irk - 1][1];
  A.irk = irk;
  A.nrk = nrk;
  A.divclean = b->p.divclean;
  A.coordinates = b->p.coordinates;
  A.algo = b->p.algo_solver;
  A.mode = MODE_RK;
  A.tol = b->p.c2p_tol;
  A.mlp.frag = b->d_mlp_frag;
  A.mlp.par = b->d_mlp_par;
  const unsigned grid = batch_grid(b, SL_UPDATE, PH_CELL);
  if (batch_seeded<KIND>(b)) {
    constexpr bool CAN_SEED = Traits<KIND>::MHD || Traits<KIND>::VISC;
    if (Traits<KIND>::VISC && b->p.imex)
      batch_update_kernel<KIND, CAN_SEED, Traits<KIND>::VISC><<<grid, 128, 0, b->stream>>>(A, batch_dev(b), b->nv);
    else
      batch_update_kernel<KIND, CAN_SEED><<<grid, 128, 0, b->stream>>>(A, batch_dev(b), b->nv);
  } else if (Traits<KIND>::VISC && b->p.imex) {
    batch_update_kernel<KIND, false, Traits<KIND>::VISC><<<grid, 128, 0, b->stream>>>(A, batch_dev(b), b->nv);
  } else {
    batch_update_kernel<KIND, false><<<grid, 128, 0, b->stream>>>(A, batch_dev(b), b->nv);
  }
}

template <int KIND>
void launch_batch_repair_smooth(EchoBatch* b) {
  RepairArgs R;
  R.P = b->P;
  R.g = Grid{};
  R.vold = b->d_v[b->vcur];
  R.vnew = b->d_v[1 - b->vcur];
  R.u = b->d_u[b->ucur];
  R.fail = b->d_fail;
  R.sc = nullptr;
  R.coordinates = b->p.coordinates;
  R.algo = b->p.algo_solver;
  R.maxspeed = b->p.maxspeed;
  R.tol = b->p.c2p_tol;
  batch_repair_kernel<KIND><<<(unsigned)b->nev, 256, 0, b->stream>>>(R, batch_dev(b), b->nv);
  if (KIND == KIND_VISC && b->p.enable_smooth_viscosity) {
    SmoothArgs S;
    S.P = b->P;
    S.g = Grid{};
    S.v = b->d_v[1 - b->vcur];
    S.u = b->d_u[b->ucur];
    S.sc = nullptr;
    S.coordinates = b->p.coordinates;
    S.smooth_pressure = b->p.smooth_pressure;
    batch_smooth_kernel<KIND><<<batch_grid(b, SL_SMOOTH, PH_CELL), 128, 0, b->stream>>>(S, batch_dev(b), b->nv);
  }
}

// the instantiation of batch_stage_kernel a batch uses
template <int KIND>
static void* batch_stage_variant(const EchoBatch* b) {
  constexpr bool CAN_SEED = Traits<KIND>::MHD || Traits<KIND>::VISC;
  constexpr bool VISC = Traits<KIND>::VISC;
  if (batch_seeded<KIND>(b) && VISC && b->p.imex) return (void*)batch_stage_kernel<KIND, CAN_SEED, VISC>;
  if (batch_seeded<KIND>(b)) return (void*)batch_stage_kernel<KIND, CAN_SEED, false>;
  if (VISC && b->p.imex) return (void*)batch_stage_kernel<KIND, false, VISC>;
  return (void*)batch_stage_kernel<KIND, false, false>;
}

// Stage irk of every live event as one cooperative launch (mode 1): the
// arguments of the per-phase launches, with the roles of the repair and the
// smoothing those after the update (the update of stage 1 writes the other
// u buffer).
template <int KIND>
int launch_batch_stage(EchoBatch* b, int irk, unsigned* grid_max) {
  static const double crk[3][3][2] = {{{0., 1.}, {0., 0.}, {0., 0.}},
                                      {{0., 1.}, {1. / 2., 1. / 2.}, {0., 0.}},
                                      {{0., 1.}, {3. / 4., 1. / 4.}, {1. / 3., 2. / 3.}}};
  void* fn = batch_stage_variant<KIND>(b);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, BATCH_NT, 0) != cudaSuccess || occ < 1)
    return ECHO_ERR_UNSUPPORTED;
  const unsigned gmax = (unsigned)occ * (unsigned)b->nsm;
  if (grid_max) *grid_max = gmax;
  const unsigned grid = b->coop_grid > 0 && b->coop_grid <= gmax ? b->coop_grid : gmax;
  BatchStageArgs S;
  memset(&S, 0, sizeof(S));
  S.face.P = b->P;
  S.face.g = Grid{};
  S.face.v = b->d_v[b->vcur];
  S.face.sc = nullptr;
  S.face.coordinates = b->p.coordinates;
  for (int d = 0; d < 3; d++) {
    S.bc[d] = b->bc[d];
    S.bc_uniform[d] = b->bc_uniform[d];
    S.bc_signed[d] = b->bc_signed[d];
  }
  for (int d = 0; d < 3; d++) {
    S.F[d] = b->d_F[d];
    S.WD[d] = b->d_WD[d];
  }
  UpdateArgs& A = S.upd;
  A.P = b->P;
  A.g = Grid{};
  A.Fx = b->d_F[0];
  A.Fy = b->d_F[1];
  A.Fz = b->d_F[2];
  A.WDx = b->d_WD[0];
  A.WDy = b->d_WD[1];
  A.WDz = b->d_WD[2];
  A.vin = b->d_v[b->vcur];
  A.vout = b->d_v[1 - b->vcur];
  A.uin = b->d_u[b->ucur];
  A.uout = irk == 1 ? b->d_u[1 - b->ucur] : b->d_u[b->ucur];
  A.u0 = irk == 1 ? b->d_u[b->ucur] : b->d_u[1 - b->ucur];
  A.vnew = b->d_vh[b->vn];
  A.vold = b->d_vh[1 - b->vn];
  A.vsnap = (Traits<KIND>::VISC && irk == 1) ? b->d_vh[b->vn] : nullptr;
  A.du_out = nullptr;
  A.fail = b->d_fail;
  A.sc = nullptr;
  const int nrk = b->p.nrk;
  A.c1 = crk[nrk - 1][irk - 1][0];
  A.c2 = crk[nrk - 1][irk - 1][1];
  A.irk = irk;
  A.nrk = nrk;
  A.divclean = b->p.divclean;
  A.coordinates = b->p.coordinates;
  A.algo = b->p.algo_solver;
  A.mode = MODE_RK;
  A.tol = b->p.c2p_tol;
  A.mlp.frag = b->d_mlp_frag;
  A.mlp.par = b->d_mlp_par;
  ScalarArgs& C = S.sca;
  C.sc = nullptr;
  C.g = Grid{};
  C.cfl = b->p.cfl;
  C.maxdt = b->p.maxdt;
  C.glm_alpha = b->p.glm_alpha;
  C.irk = irk;
  C.nrk = b->p.nrk;
  C.divclean = b->p.divclean;
  C.mode = 0;
  const int ucur_after = irk == 1 ? 1 - b->ucur : b->ucur;
  RepairArgs& R = S.rep;
  R.P = b->P;
  R.g = Grid{};
  R.vold = b->d_v[b->vcur];
  R.vnew = b->d_v[1 - b->vcur];
  R.u = b->d_u[ucur_after];
  R.fail = b->d_fail;
  R.sc = nullptr;
  R.coordinates = b->p.coordinates;
  R.algo = b->p.algo_solver;
  R.maxspeed = b->p.maxspeed;
  R.tol = b->p.c2p_tol;
  R.h_alpha = 0.;
  SmoothArgs& M = S.smo;
  M.P = b->P;
  M.g = Grid{};
  M.v = b->d_v[1 - b->vcur];
  M.u = b->d_u[ucur_after];
  M.sc = nullptr;
  M.coordinates = b->p.coordinates;
  M.smooth_pressure = b->p.smooth_pressure;
  S.B = batch_dev(b);
  S.nv = b->nv;
  S.irk = irk;
  S.roles = b->ucur | (b->vcur << 1);
  S.smooth = (KIND == KIND_VISC && b->p.enable_smooth_viscosity) ? 1 : 0;
  S.bar = b->d_bar;
  void* args[] = {&S};
  cudaMemsetAsync(b->d_bar, 0, 3 * sizeof(unsigned), b->stream);
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(BATCH_NT), args, 0, b->stream) == cudaSuccess
             ? ECHO_OK
             : ECHO_ERR_CUDA;
}

template <int KIND>
void launch_batch_p2c(EchoBatch* b) {
  batch_p2c_kernel<KIND><<<(unsigned)(b->max_tiles[PH_CELL] > 0 ? b->max_tiles[PH_CELL] : 1), 128, 0, b->stream>>>(
      b->P, batch_dev(b), b->nv, b->p.coordinates, b->d_v[b->vcur], b->d_u[b->ucur]);
}

template <int KIND>
void batch_occupancy(const EchoBatch* b, int* per_sm) {
  (void)b;
  if (b->p.recal == ECHO_REC_WENO5) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[SL_FX], batch_faces_kernel<KIND, 0, ECHO_REC_WENO5>, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[SL_FY], batch_faces_kernel<KIND, 1, ECHO_REC_WENO5>, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[SL_FZ], batch_faces_kernel<KIND, 2, ECHO_REC_WENO5>, 128, 0);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[SL_FX], batch_faces_kernel<KIND, 0, REC_RUNTIME>, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[SL_FY], batch_faces_kernel<KIND, 1, REC_RUNTIME>, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[SL_FZ], batch_faces_kernel<KIND, 2, REC_RUNTIME>, 128, 0);
  }
  if (batch_seeded<KIND>(b))
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[SL_UPDATE],
                                                  batch_update_kernel<KIND, Traits<KIND>::MHD || Traits<KIND>::VISC>,
                                                  128, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[SL_UPDATE], batch_update_kernel<KIND, false>, 128, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[SL_SMOOTH], batch_smooth_kernel<KIND>, 128, 0);
}

}  // namespace echo

#define ECHO_INSTANTIATE_GRID(K)                                              \
  template void echo::launch_faces<K>(EchoCtx*, int);                         \
  template int echo::setup_stage<K>(EchoCtx*, int, int, int);                 \
  template void echo::launch_stage<K>(EchoCtx*, int, int, double*);           \
  template void echo::launch_update<K>(EchoCtx*, int, int, double*);          \
  template void echo::launch_repair_smooth<K>(EchoCtx*, int);                 \
  template void echo::launch_p2c<K>(EchoCtx*);                                \
  template void echo::launch_ssp_combine<K>(EchoCtx*, int);                   \
  template void echo::launch_ssp_stage1<K>(EchoCtx*);

#define ECHO_INSTANTIATE(K)                                                   \
  ECHO_INSTANTIATE_GRID(K)                                                    \
  template void echo::launch_batch_faces<K>(EchoBatch*, int);                 \
  template void echo::launch_batch_update<K>(EchoBatch*, int);                \
  template void echo::launch_batch_repair_smooth<K>(EchoBatch*);              \
  template void echo::launch_batch_p2c<K>(EchoBatch*);                        \
  template int echo::launch_batch_stage<K>(EchoBatch*, int, unsigned*);        \
  template void echo::batch_occupancy<K>(const EchoBatch*, int*);
