// stage.cuh -- the fused stage kernel: the three flux sweeps, the flux
// divergence, the sources, the RK combination (or the stage right-hand side
// of an IMEX-SSP stage) and con2prim in one launch, with no face flux in
// global memory.
//
// The reference's stage (evolve_main, evolve.f90:156-203) runs the x, y and
// eta pencil sweeps (evolve_dfx/dfy/dfz, evolve.f90:302-685), each adding
// ddx*(F(i+1/2) - F(i-1/2)) into du, then the sources and the update.  Here
// a CTA owns an x-y tile of TX x TY cells and a segment of eta planes and
// marches through the planes:
//
//   1. the primitives of the plane, tile plus 3 ghost cells in x and in y
//      (the cross of the two stencils; ghosts filled as evolve_bc[xy],
//      evolve.f90:872-1054), are staged in shared memory;
//   2. the (TX+1) x TY x-faces are computed from the staged stencils into
//      shared memory, and every cell forms its x part of du;
//   3. the TX x (TY+1) y-faces likewise (the same buffer), the y part;
//   4. every cell computes its upper eta face from a 6-point stencil read
//      from global memory (L2) and takes its lower eta face from the
//      previous plane (carried in shared memory; the first plane of a
//      segment computes both), the eta part;
//   5. update_finish: lagged time derivatives, sources, RK combination or
//      the MODE_RHS right-hand side, con2prim.
//
// The faces of the tile's edges are computed by both neighbouring tiles
// (the same arithmetic, so the same values); each face is otherwise
// computed once.  The per-face arithmetic is the sweep kernels' (face_tail,
// recon_face), so the fused stage gives the sweep path's results.  The CFL
// speed maxima are reduced per CTA at the end; the GLM speed quirk of the
// reference (the last face of the last pencil, work.f90:217,310,401) is
// recorded by the tile that owns that face.
#pragma once

#include "kernels.cuh"

namespace echo {

#ifndef ECHO_STAGE_NT
#define ECHO_STAGE_NT 256
#endif
#ifndef ECHO_STAGE_MINB
#define ECHO_STAGE_MINB 2
#endif

struct StageArgs {
  UpdateArgs U;       // the update's inputs and outputs (U.Fx.. unused)
  BcDir bc[3];        // boundary codes of every variable along x, y, eta
  int tx, ty;         // tile extent in cells; tx * ty <= blockDim.x
  int ntx, nty;       // tiles along x and y
  int zseg;           // eta planes per segment
  long long nunits;   // tiles x segments
};

// shared-memory doubles of one CTA for a tile (the layout of stage_kernel)
__host__ __device__ inline size_t stage_smem_doubles(int nv, int nw, int tx, int ty, bool three_d) {
  size_t sv = (size_t)nv * (tx + 6) * (ty + 6);
  size_t fst = (size_t)((tx + 1) * ty > tx * (ty + 1) ? (tx + 1) * ty : tx * (ty + 1));
  size_t sf = (size_t)(nv + nw) * fst;
  size_t sz = three_d ? (size_t)(nv + nw) * tx * ty : 0;
  return sv + sf + sz;
}

// the 6-point stencil v(i-3..i+2) (0-based cells, face i between cells i-1
// and i) of variable array a along a pencil: ghosts as evolve_bc fills them
__device__ __forceinline__ void pencil6(const double* __restrict__ a, size_t base, long long stride, int n, int i,
                                        int code_l, int code_r, double s[6]) {
#pragma unroll
  for (int q = 0; q < 6; q++) s[q] = ghost_val(a, base, stride, n, i - 2 + q, code_l, code_r);
}

// The flux of one face from its stencils (sfn(k, q) = variable k at stencil
// point q), with the viscous u^mu face states in WD[8] (l then r).  Returns
// a reference error code; F then holds zeros.
template <int KIND, int DIR, class StencilFn>
__device__ __forceinline__ int stage_face(const DevPhys& P, const Metric& M, double ch, StencilFn sfn, double* F,
                                          double* WD, double& amax) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  double wl[NV], wr[NV], w0[NV];
  double sv[3][6];
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double s[6];
#pragma unroll
    for (int q = 0; q < 6; q++) s[q] = sfn(k, q);
    w0[k] = s[2];
    recon_face<ECHO_REC_WENO5>(P.recal, s, wl[k], wr[k]);
    if (T::VISC && k >= KVX && k <= KVZ) {
#pragma unroll
      for (int q = 0; q < 6; q++) sv[k - KVX][q] = s[q];
    }
  }
  if (T::VISC) {
    double s[4][6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
      double vx = sv[0][q], vy = sv[1][q], vz = sv[2][q];
      double gg = 1. / sqrt(1. - vx * vx - vy * vy - M.g3 * (vz * vz));
      s[0][q] = gg;
      s[1][q] = gg * vx;
      s[2][q] = gg * vy;
      s[3][q] = gg * vz;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) recon_face<ECHO_REC_WENO5>(P.recal, s[c], WD[c], WD[4 + c]);
  }
  int err = face_tail<KIND, DIR>(P, M, ch, wl, wr, w0, F, amax);
  if (err) {
#pragma unroll
    for (int k = 0; k < NV; k++) F[k] = 0.0;
  }
  return err;
}

template <int KIND, bool SEED, bool IMEX>
__global__ void __launch_bounds__(ECHO_STAGE_NT, ECHO_STAGE_MINB) stage_kernel(StageArgs S) {
  typedef Traits<KIND> T;
  constexpr int NV = T::NV;
  constexpr int NW = T::VISC ? 8 : 0;
  constexpr int NF = NV + NW;
  extern __shared__ double sm[];
  __shared__ double red[ECHO_STAGE_NT / 32];
  const UpdateArgs& U = S.U;
  const Grid& g = U.g;
  const int TX = S.tx, TY = S.ty;
  const int SX = TX + 6, SY = TY + 6;
  const int FST = (TX + 1) * TY > TX * (TY + 1) ? (TX + 1) * TY : TX * (TY + 1);
  const bool three_d = g.nz > 1;
  double* sV = sm;                              // [NV][SY][SX]
  double* sF = sV + (size_t)NV * SX * SY;       // [NF][FST]
  double* sZ = sF + (size_t)NF * FST;           // [NF][TX*TY], 3-D only
  const int tid = threadIdx.x;
  const int cx = tid % TX, cy = tid / TX;
  const size_t nxy = (size_t)g.nx * g.ny;
  const double ch = U.sc->glm_ch_old;
  const Metric M = make_metric(U.coordinates, U.sc->t, U.sc->t3);
  double am[3] = {0., 0., 0.};
  const int dk[3][4] = {{DTX, DXX, DYX, DZX}, {DTY, DXY, DYY, DZY}, {DTZ, DXZ, DYZ, DZZ}};

  for (long long unit = blockIdx.x; unit < S.nunits; unit += gridDim.x) {
    const int tile = (int)(unit % ((long long)S.ntx * S.nty));
    const int seg = (int)(unit / ((long long)S.ntx * S.nty));
    const int x0 = (tile % S.ntx) * TX, y0 = (tile / S.ntx) * TY;
    const int z0 = seg * S.zseg;
    const int z1 = z0 + S.zseg < g.nz ? z0 + S.zseg : g.nz;
    const int gx = x0 + cx, gy = y0 + cy;
    const bool own = tid < TX * TY && gx < g.nx && gy < g.ny;
    for (int k = z0; k < z1; k++) {
      __syncthreads();  // the previous plane's readers of sV and sF are done
      // 1. stage the plane: tile + x ghosts in the tile's rows, + y ghosts
      // in its columns (evolve_bcx/bcy fills)
      for (int idx = tid; idx < SX * SY; idx += blockDim.x) {
        const int sy = idx / SX, sx = idx - sy * SX;
        const int px = x0 + sx - 3, py = y0 + sy - 3;
        const bool xrow = sy >= 3 && sy < 3 + TY, ycol = sx >= 3 && sx < 3 + TX;
        const size_t pl = (size_t)k * nxy;
        if (px >= 0 && px < g.nx && py >= 0 && py < g.ny) {
#pragma unroll
          for (int v = 0; v < NV; v++) sV[(size_t)v * SX * SY + idx] = __ldg(U.vin + (size_t)v * g.ncell + pl + (size_t)py * g.nx + px);
        } else if (xrow && py < g.ny && px <= g.nx + 2) {
          const size_t base = pl + (size_t)py * g.nx;
#pragma unroll
          for (int v = 0; v < NV; v++)
            sV[(size_t)v * SX * SY + idx] =
                ghost_val(U.vin + (size_t)v * g.ncell, base, 1, g.nx, px + 1, S.bc[0].c[v][0], S.bc[0].c[v][1]);
        } else if (ycol && px < g.nx && py <= g.ny + 2) {
          const size_t base = pl + (size_t)px;
#pragma unroll
          for (int v = 0; v < NV; v++)
            sV[(size_t)v * SX * SY + idx] = ghost_val(U.vin + (size_t)v * g.ncell, base, g.nx, g.ny, py + 1,
                                                      S.bc[1].c[v][0], S.bc[1].c[v][1]);
        } else {
#pragma unroll
          for (int v = 0; v < NV; v++) sV[(size_t)v * SX * SY + idx] = 0.0;
        }
      }
      __syncthreads();
      double du[NV], dv[NDER];
#pragma unroll
      for (int q = 0; q < NDER; q++) dv[q] = 0.;
      // 2. x faces: face i (0..nx) between cells i-1 and i, stencil cells i-3..i+2
      for (int f = tid; f < (TX + 1) * TY; f += blockDim.x) {
        const int fy = f / (TX + 1), fx = f - fy * (TX + 1);
        const int i = x0 + fx, py = y0 + fy;
        if (i > g.nx || py >= g.ny) continue;
        const double* row = sV + (size_t)(fy + 3) * SX + fx;
        auto sfn = [&](int v, int q) { return row[(size_t)v * SX * SY + q]; };
        double F[NV], WD[8], a;
        int err = stage_face<KIND, 0>(U.P, M, ch, sfn, F, WD, a);
        if (err) {
          size_t cell = (size_t)k * nxy + (size_t)py * g.nx + (size_t)((i >= 1 ? i : 1) - 1);
          atomicMin(&U.sc->err_key, ((unsigned long long)cell << 20) | (unsigned long long)err);
        } else {
          am[0] = a > am[0] ? a : am[0];
          if (i == g.nx && py == g.ny - 1 && k == g.nz - 1) U.sc->aflux[0] = a;
        }
#pragma unroll
        for (int v = 0; v < NV; v++) sF[(size_t)v * FST + f] = F[v];
        if (T::VISC) {
#pragma unroll
          for (int q = 0; q < 8; q++) sF[(size_t)(NV + q) * FST + f] = WD[q];
        }
      }
      __syncthreads();
      if (own) {
        const int f = cy * (TX + 1) + cx;  // face gx-1/2; face gx+1/2 = f + 1
#pragma unroll
        for (int v = 0; v < NV; v++) {
          double d = 0.;
          d = d + g.ddx * (sF[(size_t)v * FST + f + 1] - sF[(size_t)v * FST + f]);
          du[v] = d;
        }
        if (T::VISC) {
#pragma unroll
          for (int q = 0; q < 4; q++)
            dv[dk[0][q]] = g.ddx * 0.5 *
                           (sF[(size_t)(NV + q) * FST + f + 1] + sF[(size_t)(NV + 4 + q) * FST + f + 1] -
                            sF[(size_t)(NV + q) * FST + f] - sF[(size_t)(NV + 4 + q) * FST + f]);
        }
      }
      __syncthreads();
      // 3. y faces: face j (0..ny) between cells j-1 and j, stencil cells j-3..j+2
      for (int f = tid; f < TX * (TY + 1); f += blockDim.x) {
        const int fy = f / TX, fx = f - fy * TX;
        const int j = y0 + fy, px = x0 + fx;
        if (j > g.ny || px >= g.nx) continue;
        const double* col = sV + (size_t)fy * SX + fx + 3;
        auto sfn = [&](int v, int q) { return col[(size_t)v * SX * SY + (size_t)q * SX]; };
        double F[NV], WD[8], a;
        int err = stage_face<KIND, 1>(U.P, M, ch, sfn, F, WD, a);
        if (err) {
          size_t cell = (size_t)k * nxy + (size_t)((j >= 1 ? j : 1) - 1) * g.nx + px;
          atomicMin(&U.sc->err_key, ((unsigned long long)cell << 20) | (unsigned long long)err);
        } else {
          am[1] = a > am[1] ? a : am[1];
          if (j == g.ny && px == g.nx - 1 && k == g.nz - 1) U.sc->aflux[1] = a;
        }
#pragma unroll
        for (int v = 0; v < NV; v++) sF[(size_t)v * FST + f] = F[v];
        if (T::VISC) {
#pragma unroll
          for (int q = 0; q < 8; q++) sF[(size_t)(NV + q) * FST + f] = WD[q];
        }
      }
      __syncthreads();
      if (own) {
        const int f = cy * TX + cx;  // face gy-1/2; face gy+1/2 = f + TX
#pragma unroll
        for (int v = 0; v < NV; v++) du[v] = du[v] + g.ddy * (sF[(size_t)v * FST + f + TX] - sF[(size_t)v * FST + f]);
        if (T::VISC) {
#pragma unroll
          for (int q = 0; q < 4; q++)
            dv[dk[1][q]] = g.ddy * 0.5 *
                           (sF[(size_t)(NV + q) * FST + f + TX] + sF[(size_t)(NV + 4 + q) * FST + f + TX] -
                            sF[(size_t)(NV + q) * FST + f] - sF[(size_t)(NV + 4 + q) * FST + f]);
        }
      }
      // 4. eta faces of the own cell: face kz between planes kz-1 and kz
      if (three_d && own) {
        const size_t base = (size_t)gy * g.nx + gx;
        const int ct = cy * TX + cx;
        auto zface = [&](int kz, double* F, double* WD, double& a) {
          auto sfn = [&](int v, int q) {
            return ghost_val(U.vin + (size_t)v * g.ncell, base, (long long)nxy, g.nz, kz - 2 + q, S.bc[2].c[v][0],
                             S.bc[2].c[v][1]);
          };
          int err = stage_face<KIND, 2>(U.P, M, ch, sfn, F, WD, a);
          if (err) {
            size_t cell = (size_t)((kz >= 1 ? kz : 1) - 1) * nxy + base;
            atomicMin(&U.sc->err_key, ((unsigned long long)cell << 20) | (unsigned long long)err);
          } else {
            am[2] = a > am[2] ? a : am[2];
            if (kz == g.nz && gx == g.nx - 1 && gy == g.ny - 1) U.sc->aflux[2] = a;
          }
        };
        double Flo[NF];
        if (k == z0) {
          double F[NV], WD[8], a;
          zface(k, F, WD, a);
#pragma unroll
          for (int v = 0; v < NV; v++) Flo[v] = F[v];
          if (T::VISC) {
#pragma unroll
            for (int q = 0; q < 8; q++) Flo[NV + q] = WD[q];
          }
        } else {
#pragma unroll
          for (int v = 0; v < NF; v++) Flo[v] = sZ[(size_t)v * TX * TY + ct];
        }
        double F[NV], WD[8], a;
        zface(k + 1, F, WD, a);
#pragma unroll
        for (int v = 0; v < NV; v++) du[v] = du[v] + g.ddz * (F[v] - Flo[v]);
        if (T::VISC) {
#pragma unroll
          for (int q = 0; q < 4; q++)
            dv[dk[2][q]] = g.ddz * 0.5 * (WD[q] + WD[4 + q] - Flo[NV + q] - Flo[NV + 4 + q]);
        }
#pragma unroll
        for (int v = 0; v < NV; v++) sZ[(size_t)v * TX * TY + ct] = F[v];
        if (T::VISC) {
#pragma unroll
          for (int q = 0; q < 8; q++) sZ[(size_t)(NV + q) * TX * TY + ct] = WD[q];
        }
      }
      // 5. sources, RK combination (or the stage right-hand side), con2prim
      const size_t c = (size_t)k * nxy + (size_t)gy * g.nx + gx;
      update_finish<KIND, SEED, IMEX>(U, own ? c : 0, own, gx, gy, k, du, dv);
    }
  }
  block_max_atomic(am[0], &U.sc->amax_bits[0], red);
  __syncthreads();
  block_max_atomic(am[1], &U.sc->amax_bits[1], red);
  __syncthreads();
  block_max_atomic(am[2], &U.sc->amax_bits[2], red);
}

}  // namespace echo
