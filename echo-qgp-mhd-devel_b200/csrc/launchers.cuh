// launchers.cuh -- definitions of the per-equation-set launch functions;
// included only by kind_*.cu, each of which instantiates one equation set.
#pragma once

#include "ctx.cuh"

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
  if (dir == 0) faces_kernel<KIND, 0><<<blocks, 128, 0, c->stream>>>(A);
  if (dir == 1) faces_kernel<KIND, 1><<<blocks, 128, 0, c->stream>>>(A);
  if (dir == 2) faces_kernel<KIND, 2><<<blocks, 128, 0, c->stream>>>(A);
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
  A.mlp.frag = c->d_mlp_frag;
  A.mlp.par = c->d_mlp_par;
  if (A.algo == ECHO_C2P_MLP && !c->d_mlp_frag) A.algo = ECHO_C2P_NEWTON;  // no network loaded
  unsigned blocks = (unsigned)((c->g.ncell + 127) / 128);
  if (Traits<KIND>::MHD && A.algo == ECHO_C2P_MLP && mode == MODE_RK)
    update_kernel<KIND, Traits<KIND>::MHD><<<blocks, 128, 0, c->stream>>>(A);
  else
    update_kernel<KIND, false><<<blocks, 128, 0, c->stream>>>(A);
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
  if (Traits<KIND>::MHD && A.algo == ECHO_C2P_MLP)
    ssp_combine_kernel<KIND, Traits<KIND>::MHD><<<blocks, 128, 0, c->stream>>>(A);
  else
    ssp_combine_kernel<KIND, false><<<blocks, 128, 0, c->stream>>>(A);
}

}  // namespace echo

#define ECHO_INSTANTIATE(K)                                                   \
  template void echo::launch_faces<K>(EchoCtx*, int);                         \
  template void echo::launch_update<K>(EchoCtx*, int, int, double*);          \
  template void echo::launch_repair_smooth<K>(EchoCtx*, int);                      \
  template void echo::launch_p2c<K>(EchoCtx*);                                \
  template void echo::launch_ssp_combine<K>(EchoCtx*, int);
