// kernels.cuh -- the device kernels of one RK stage.
//
//   faces<KIND,DIR>   one thread per cell face along DIR: boundary ghosts,
//                     reconstruction, the p<=0 / v^2>=1 fix-ups, GLM, two
//                     system_flux calls and the HLL flux (evolve_df[xyz],
//                     evolve.f90:302-685; work_fup[xyz], work.f90:143-416);
//                     writes the face flux and the max signal speed.
//   stage_scalars     the scalar logic of evolve_main (dt, CFL reduction
//                     result, GLM speed and damping factor).
//   update<KIND>      one thread per cell: flux divergence + sources + RK
//                     combination + con2prim (evolve.f90:156-203,689-868).
//   repair<KIND>      the neighbour-average repair of failed cells in the
//                     reference's loop order (evolve.f90:795-842).
//   smooth<KIND>      evolve_smooth_viscosity (evolve.f90:1159-1207).
#pragma once

#include <cuda_runtime.h>

#include "c2p.cuh"

namespace echo {

// Device-resident scalars of the run.  Kept on the device so a whole step
// needs no host round trip (and can be captured in a CUDA graph).
struct DevScalars {
  double t, t3, dt, tout, dtout, tmax, timeold, timeinterval, g3old;
  double glm_ch, glm_ch_old, aflux[3], expfact;
  unsigned long long amax_bits[3];
  unsigned long long err_key;  // (cell << 20) | code, min over failures
  int nfail, pad;
  unsigned long long c2p_iters, c2p_cells, repairs, fallbacks;
  unsigned long long check_bits;  // check_temp maximum (bit pattern of a double >= 0)
  unsigned long long brackets;    // con2prim solves that fell back to the bracketed BRENTM
};

// Unsigned 32-bit division by a run-time invariant d >= 1 as a multiply-high,
// a subtraction, an addition and two shifts (T. Granlund and P. L.
// Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994, Fig. 4.1): with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// t = umulhi(m, n) and q = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0) is
// floor(n / d) for every n < 2^32.
struct FastDiv {
  unsigned m;
  unsigned char s1, s2;
};
__host__ __device__ inline FastDiv make_fastdiv(unsigned d) {
  int l = 0;
  while ((1ull << l) < (unsigned long long)d) l++;
  FastDiv f;
  f.m = (unsigned)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
  f.s1 = (unsigned char)(l > 0 ? 1 : 0);
  f.s2 = (unsigned char)(l > 0 ? l - 1 : 0);
  return f;
}
__device__ __forceinline__ unsigned fast_div(unsigned n, const FastDiv& f) {
  const unsigned t = __umulhi(f.m, n);
  return (t + ((n - t) >> f.s1)) >> f.s2;
}

struct Grid {
  int nx, ny, nz;
  size_t ncell;
  double ddx, ddy, ddz;
  // division by nx, ny, nx + 1 and ny + 1 of face and cell indices below
  // 2^32 (set_grid_div)
  FastDiv dnx, dny, dnx1, dny1;
};
__host__ __device__ inline void set_grid_div(Grid& g) {
  g.dnx = make_fastdiv((unsigned)g.nx);
  g.dny = make_fastdiv((unsigned)g.ny);
  g.dnx1 = make_fastdiv((unsigned)g.nx + 1u);
  g.dny1 = make_fastdiv((unsigned)g.ny + 1u);
}

// boundary codes for one sweep direction: bc[k][side]
struct BcDir {
  signed char c[ECHO_MAX_NV][2];
};

// ---------------------------------------------------------------------------
// stencil loads with the ghost fill of evolve_bc[xyz] (evolve.f90:872-1127)
// ---------------------------------------------------------------------------
// Value of variable array `a` (one variable, already offset) at pencil index
// j (1-based, may be a ghost in [-2, n+3]); `base` is the linear index of
// pencil cell 1 and `stride` the step between pencil cells.
__device__ __forceinline__ double ghost_val(const double* __restrict__ a, size_t base, long long stride,
                                            int n, int j, int code_l, int code_r) {
  if (j >= 1 && j <= n) return __ldg(a + base + (long long)(j - 1) * stride);
  auto at = [&](int q) { return __ldg(a + base + (long long)(q - 1) * stride); };
  if (j <= 0) {
    switch (code_l) {
      case 0: return at(j + n);
      case 1: return at(1 - j);
      case -1: return -at(1 - j);
      case 3: {
        double w1 = at(1), w2 = at(2), w3 = at(3);
        double w0 = w3 - 3. * (w2 - w1);
        if (j == 0) return w0;
        double wm1 = w2 - 3. * (w1 - w0);
        if (j == -1) return wm1;
        return w1 - 3. * (w0 - wm1);
      }
      default: return at(1);
    }
  }
  switch (code_r) {
    case 0: return at(j - n);
    case 1: return at(2 * n + 1 - j);
    case -1: return -at(2 * n + 1 - j);
    case 3: {
      double a2 = at(n - 2), a1 = at(n - 1), a0 = at(n);
      double p1 = a2 - 3. * (a1 - a0);
      if (j == n + 1) return p1;
      double p2 = a1 - 3. * (a0 - p1);
      if (j == n + 2) return p2;
      return a0 - 3. * (p1 - p2);
    }
    default: return at(n);
  }
}

// index and sign of the cell that ghost j (1-based pencil index) copies for
// boundary codes 0 (periodic), +-1 (reflecting) and 2 (outflow)
__device__ __forceinline__ void map_ghost(int j, int n, int cl, int cr, int& q, double& sg) {
  q = j;
  sg = 1.0;
  if (j < 1) {
    q = cl == 0 ? j + n : (cl == 1 || cl == -1) ? 1 - j : 1;
    if (cl == -1) sg = -1.0;
  } else if (j > n) {
    q = cr == 0 ? j - n : (cr == 1 || cr == -1) ? 2 * n + 1 - j : n;
    if (cr == -1) sg = -1.0;
  }
}

// The face and update kernels are latency-bound (long-scoreboard and
// dependent FP64 stalls): more resident warps win over the spills a lower
// register cap costs.  Measured on B200 (blocks of 128 per SM): faces 7
// (ideal RMHD; 5 is 10 % slower) and 5 (viscous; 3 is 15 % slower); update
// 7 (ideal RMHD, from 4 uncapped), 5 (viscous, from 2) and 6 with the
// learned seed (from 2: 0.74 vs 1.17 ms per step).
#ifndef ECHO_FACE_MINB
#define ECHO_FACE_MINB 7
#endif
#ifndef ECHO_FACE_MINB_VISC
#define ECHO_FACE_MINB_VISC 5
#endif
// resistive (nv = 12, 193x193x129, per step): faces 7 (6: +3 %, 5: +11 %);
// update 5 (7: +1.9 ms, 6: +2.0, 4: +0.05); the IMEX-SSP combination 8
// (uncapped 118 registers: +3.6 ms; 5: +1.1, 6: +0.5, 7: +0.14)
#ifndef ECHO_FACE_MINB_RES
#define ECHO_FACE_MINB_RES 7
#endif
#define ECHO_FACE_BOUNDS(KIND)                                                      \
  __launch_bounds__(128, (KIND) == KIND_VISC  ? ECHO_FACE_MINB_VISC              \
                         : (KIND) == KIND_RES ? ECHO_FACE_MINB_RES : ECHO_FACE_MINB)
#ifndef ECHO_UPDATE_MINB
#define ECHO_UPDATE_MINB 7
#endif
#ifndef ECHO_UPDATE_MINB_VISC
#define ECHO_UPDATE_MINB_VISC 5
#endif
#ifndef ECHO_UPDATE_MINB_SEED
#define ECHO_UPDATE_MINB_SEED 6
#endif
#ifndef ECHO_UPDATE_MINB_RES
#define ECHO_UPDATE_MINB_RES 5
#endif
// the IMEX-SSP combination (con2prim) kernels
#ifndef ECHO_SSP_MINB
#define ECHO_SSP_MINB 8
#endif
#define ECHO_UPDATE_BOUNDS(KIND, SEED)                                       \
  __launch_bounds__(128, (KIND) == KIND_VISC ? ECHO_UPDATE_MINB_VISC     \
                         : (SEED)             ? ECHO_UPDATE_MINB_SEED     \
                         : (KIND) == KIND_RES ? ECHO_UPDATE_MINB_RES      \
                                              : ECHO_UPDATE_MINB)

struct FaceArgs {
  DevPhys P;
  Grid g;
  BcDir bc;
  int bc_uniform;   // every variable has the same codes, none is 3 (extrapolation)
  int bc_signed;    // some code is -1 (the ghost changes sign)
  const double* __restrict__ v;   // primitives, nv * ncell
  double* __restrict__ F;         // face fluxes, nv * nfaces
  double* __restrict__ WD;        // viscous: wdl(4), wdr(4) per face, or null
  DevScalars* sc;
  int coordinates;
};

// The stencils and the reconstruction of every variable when the boundary
// codes differ between variables or include extrapolation (code 3): a rare
// configuration, kept out of line so that the common kernel body stays
// small in the instruction cache.  Returns w0 (the cell left of the face),
// the face states, and the velocity stencils sv for the viscous u^mu.
template <int NV>
struct ReconOut {
  double w0[NV], wl[NV], wr[NV], sv[3][6];
};
template <int KIND, int REC>
__device__ __noinline__ ReconOut<Traits<KIND>::NV> recon_general(const double* __restrict__ v, size_t ncell,
                                                                  BcDir bc, int recal, size_t base,
                                                                  long long stride, int n, int i) {
  ReconOut<Traits<KIND>::NV> r;
#pragma unroll 1
  for (int k = 0; k < Traits<KIND>::NV; k++) {
    const double* vk = v + (size_t)k * ncell;
    double s[6];
#pragma unroll
    for (int q = 0; q < 6; q++) s[q] = ghost_val(vk, base, stride, n, i - 2 + q, bc.c[k][0], bc.c[k][1]);
    r.w0[k] = s[2];
    recon_face<REC>(recal, s, r.wl[k], r.wr[k]);
    if (k >= KVX && k <= KVZ) {
#pragma unroll
      for (int q = 0; q < 6; q++) r.sv[k - KVX][q] = s[q];
    }
  }
  return r;
}

// face index layout for DIR: (i fastest in x, then the other two)
//   DIR 0: F[k][iz][iy][i],  i = 0..nx
//   DIR 1: F[k][iz][j][ix],  j = 0..ny
//   DIR 2: F[k][kz][iy][ix], kz = 0..nz
template <int DIR>
__host__ __device__ __forceinline__ size_t faces_of(const Grid& g) {
  return DIR == 0 ? (size_t)(g.nx + 1) * g.ny * g.nz
         : DIR == 1 ? (size_t)g.nx * (g.ny + 1) * g.nz
                    : (size_t)g.nx * g.ny * (g.nz + 1);
}

// The face after reconstruction (shared by the sweep kernels and the fused
// stage kernel): the p <= 0 / v^2 >= 1 fix-ups (evolve.f90:334-369, w0 = the
// cell left of the face), GLM upwinding (work_glm[xyz], work.f90:67-139)
// with wave speed ch, the two system_flux calls and the HLL flux
// (work.f90:195-229).  Writes F[NV] and the face's signal speed
// max(a+, a-); returns a reference error code (F undefined then).
template <int KIND, int DIR>
__device__ __forceinline__ int face_tail(const DevPhys& P, const Metric& M, double ch, double* wl, double* wr,
                                         double* w0, double* F, double& amax_local) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  amax_local = 0.0;
  {
    double v2;
    if (wr[KPR] <= 0) wr[KPR] = w0[KPR];
    v2 = 0;
    v2 = v2 + wr[KVX] * wr[KVX] * M.g1;
    v2 = v2 + wr[KVY] * wr[KVY] * M.g2;
    v2 = v2 + wr[KVZ] * wr[KVZ] * M.g3;
    if (v2 >= 1.) {
      wr[KVX] = w0[KVX];
      wr[KVY] = w0[KVY];
      wr[KVZ] = w0[KVZ];
      v2 = 0;
      v2 = v2 + wr[KVX] * wr[KVX] * M.g1;
      v2 = v2 + wr[KVY] * wr[KVY] * M.g2;
      v2 = v2 + wr[KVZ] * wr[KVZ] * M.g3;
      if (v2 >= 1) {
#pragma unroll
        for (int k = KVX; k <= KVZ; k++) {
          w0[k] = w0[k] * P.maxspeed / (sqrt(v2));
          wr[k] = w0[k];
        }
      }
    }
    if (wl[KPR] <= 0) wl[KPR] = w0[KPR];
    v2 = 0;
    v2 = v2 + wl[KVX] * wl[KVX] * M.g1;
    v2 = v2 + wl[KVY] * wl[KVY] * M.g2;
    v2 = v2 + wl[KVZ] * wl[KVZ] * M.g3;
    if (v2 >= 1.) {
      wl[KVX] = w0[KVX];
      wl[KVY] = w0[KVY];
      wl[KVZ] = w0[KVZ];
      v2 = 0;
      v2 = v2 + wl[KVX] * wl[KVX] * M.g1;
      v2 = v2 + wl[KVY] * wl[KVY] * M.g2;
      v2 = v2 + wl[KVZ] * wl[KVZ] * M.g3;
      if (v2 >= 1) {
#pragma unroll
        for (int k = KVX; k <= KVZ; k++) {
          w0[k] = w0[k] * P.maxspeed / (sqrt(v2));
          wl[k] = w0[k];
        }
      }
    }
  }
  if (T::GLM) {
    const int kb = DIR == 0 ? KBX : DIR == 1 ? KBY : KBZ;
    wl[T::KG] = 0.5 * (wl[T::KG] + wr[T::KG]) - (wr[kb] - wl[kb]) * ch / 2;
    wr[T::KG] = wl[T::KG];
    wl[kb] = 0.5 * (wl[kb] + wr[kb]) - (wr[T::KG] - wl[T::KG]) / (2 * ch);
    wr[kb] = wl[kb];
  }
  double ul[NV], ur[NV], fl[NV], fr[NV];
  double vflp, vflm, vfrp, vfrm;
  int err = system_flux<KIND, DIR + 1>(P, M, wl, ul, fl, vflp, vflm);
  if (!err) err = system_flux<KIND, DIR + 1>(P, M, wr, ur, fr, vfrp, vfrm);
  if (err) return err;
  double ap = 0., am = 0.;
  if (vflp > ap) ap = vflp;
  if (vfrp > ap) ap = vfrp;
  if (-vflm > am) am = -vflm;
  if (-vfrm > am) am = -vfrm;
  amax_local = ap > am ? ap : am;
  double a1 = (ap == 0.0 && am == 0.0) ? 1. : 1. / (ap + am);
#pragma unroll
  for (int k = 0; k < NV; k++) F[k] = a1 * (ap * fl[k] + am * fr[k] - ap * am * (ur[k] - ul[k]));
  return 0;
}

// The flux through face `fid` (< faces_of<DIR>(A.g)): writes A.F (and A.WD)
// and returns the face's signal speed max(a+, a-) for the CFL reduction.
template <int KIND, int DIR, int REC>
__device__ __forceinline__ double face_flux(const FaceArgs& A, size_t fid) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  const Grid& g = A.g;
  const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
  const size_t nfaces = faces_of<DIR>(g);
  double amax_local = 0.0;
  {
    int i, a, b;  // face index along DIR, transverse coordinates (1-based)
    size_t base;
    long long stride;
    if (nfaces < (1ull << 32)) {  // multiply-high divisions (FastDiv)
      const unsigned f = (unsigned)fid;
      if (DIR == 0) {
        const unsigned r = fast_div(f, g.dnx1), q = fast_div(r, g.dny);
        i = (int)(f - r * (unsigned)(g.nx + 1));
        a = (int)(r - q * (unsigned)g.ny) + 1;
        b = (int)q + 1;
      } else if (DIR == 1) {
        const unsigned r = fast_div(f, g.dnx), q = fast_div(r, g.dny1);
        a = (int)(f - r * (unsigned)g.nx) + 1;
        i = (int)(r - q * (unsigned)(g.ny + 1));
        b = (int)q + 1;
      } else {
        const unsigned r = fast_div(f, g.dnx), q = fast_div(r, g.dny);
        a = (int)(f - r * (unsigned)g.nx) + 1;
        b = (int)(r - q * (unsigned)g.ny) + 1;
        i = (int)q;
      }
    } else if (DIR == 0) {
      i = (int)(fid % (g.nx + 1));
      size_t r = fid / (g.nx + 1);
      a = (int)(r % g.ny) + 1;
      b = (int)(r / g.ny) + 1;
    } else if (DIR == 1) {
      a = (int)(fid % g.nx) + 1;
      size_t r = fid / g.nx;
      i = (int)(r % (g.ny + 1));
      b = (int)(r / (g.ny + 1)) + 1;
    } else {
      a = (int)(fid % g.nx) + 1;
      size_t r = fid / g.nx;
      b = (int)(r % g.ny) + 1;
      i = (int)(r / g.ny);
    }
    if (DIR == 0) {
      base = ((size_t)(b - 1) * g.ny + (a - 1)) * g.nx;
      stride = 1;
    } else if (DIR == 1) {
      base = (size_t)(b - 1) * g.ny * g.nx + (a - 1);
      stride = g.nx;
    } else {
      base = (size_t)(b - 1) * g.nx + (a - 1);
      stride = (long long)g.nx * g.ny;
    }
    const Metric M = make_metric(A.coordinates, A.sc->t, A.sc->t3);
    double wl[NV], wr[NV], w0[NV];
    double sv[3][6];  // velocity stencils (ghosts filled), for the viscous u^mu
    // reconstruction of every variable (work_rec(n,1,nv,0))
    if (A.bc_uniform) {
      long long off[6];
      double sg[6];
#pragma unroll
      for (int q = 0; q < 6; q++) {
        int qq;
        map_ghost(i - 2 + q, n, A.bc.c[0][0], A.bc.c[0][1], qq, sg[q]);
        off[q] = (long long)base + (long long)(qq - 1) * stride;
      }
#pragma unroll
      for (int k = 0; k < NV; k++) {
        const double* vk = A.v + (size_t)k * g.ncell;
        double s[6];
#pragma unroll
        for (int q = 0; q < 6; q++) s[q] = __ldg(vk + off[q]);
        if (A.bc_signed) {
#pragma unroll
          for (int q = 0; q < 6; q++) s[q] = sg[q] * s[q];
        }
        w0[k] = s[2];
        recon_face<REC>(A.P.recal, s, wl[k], wr[k]);
        if (T::VISC && k >= KVX && k <= KVZ) {
#pragma unroll
          for (int q = 0; q < 6; q++) sv[k - KVX][q] = s[q];
        }
      }
    } else {
      ReconOut<NV> r = recon_general<KIND, REC>(A.v, g.ncell, A.bc, A.P.recal, base, stride, n, i);
#pragma unroll
      for (int k = 0; k < NV; k++) {
        w0[k] = r.w0[k];
        wl[k] = r.wl[k];
        wr[k] = r.wr[k];
      }
      if (T::VISC) {
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int q = 0; q < 6; q++) sv[c][q] = r.sv[c][q];
      }
    }
    // u^mu reconstruction for the viscous derivatives (work_rec(n,1,4,1)),
    // from the same ghost-filled velocity stencils
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
      for (int c = 0; c < 4; c++) {
        double l, r;
        recon_face<REC>(A.P.recal, s[c], l, r);
        A.WD[(size_t)c * nfaces + fid] = l;
        A.WD[(size_t)(4 + c) * nfaces + fid] = r;
      }
    }
    double fl_out[NV];
    int err = face_tail<KIND, DIR>(A.P, M, A.sc->glm_ch_old, wl, wr, w0, fl_out, amax_local);
    if (err) {
      size_t cell = base + (size_t)((i >= 1 ? i : 1) - 1) * stride;
      atomicMin(&A.sc->err_key, ((unsigned long long)cell << 20) | (unsigned long long)err);
#pragma unroll
      for (int k = 0; k < NV; k++) A.F[(size_t)k * nfaces + fid] = 0.0;
    } else {
#pragma unroll
      for (int k = 0; k < NV; k++) A.F[(size_t)k * nfaces + fid] = fl_out[k];
      // GLM speed of the reference: the last face of the last pencil (work.f90:217,310,401)
      int na = DIR == 0 ? g.ny : g.nx;
      int nb = DIR == 2 ? g.ny : g.nz;
      if (i == n && a == na && b == nb) A.sc->aflux[DIR] = amax_local;
    }
  }
  return amax_local;
}

// Block max of the signal speed -> one atomic per block (the CFL reduction of
// evolve_dt, evolve.f90:723-764).  Positive doubles order like their bit
// patterns, so the max is an integer atomicMax.  Called by every thread of
// the block; `red` holds one entry per warp.
__device__ __forceinline__ void block_max_atomic(double m, unsigned long long* dst, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double x = __shfl_xor_sync(0xffffffffu, m, o);
    m = x > m ? x : m;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) mm = red[w] > mm ? red[w] : mm;
    if (mm > 0.0) atomicMax(dst, (unsigned long long)__double_as_longlong(mm));
  }
}

template <int KIND, int DIR, int REC>
__global__ void ECHO_FACE_BOUNDS(KIND) faces_kernel(FaceArgs A) {
  __shared__ double red[4];
  size_t fid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double amax_local = fid < faces_of<DIR>(A.g) ? face_flux<KIND, DIR, REC>(A, fid) : 0.0;
  block_max_atomic(amax_local, &A.sc->amax_bits[DIR], red);
}

#ifndef ECHO_EXACT
// ---------------------------------------------------------------------------
// Face sweep by cell-centred reconstruction (product build, WENO5).  One lane
// per cell: a lane reconstructs both face states of its cell at once
// (weno5_cell: the cell's three smoothness indicators serve the face above
// and the face below), then takes the upper-face state of the cell below it
// from the neighbouring lane (__shfl_up_sync) and computes the flux of the
// face between the two.  The arithmetic after reconstruction is face_tail's,
// as in faces_kernel.
//
// A warp covers segments of L consecutive cells along the sweep; the first
// cell of a segment only feeds the face above it, so a segment yields L - 1
// faces and consecutive segments overlap by one cell.  The 32 / L segments of
// a warp lie side by side across the sweep so that every load touches whole
// sectors: for the x-sweep L lanes run along x (W = 32 / L pencils per warp);
// for the y- and eta-sweeps W = 32 / L consecutive x columns, each L cells
// along the sweep (lane = x-offset + W * position).
// ---------------------------------------------------------------------------
template <int KIND, int DIR, int L>
__global__ void ECHO_FACE_BOUNDS(KIND) faces_seg_kernel(FaceArgs A) {
  typedef Traits<KIND> T;
  constexpr int NV = T::NV;
  constexpr int W = 32 / L;
  constexpr int DELTA = DIR == 0 ? 1 : W;  // lane of the cell below
  __shared__ double red[4];
  const Grid& g = A.g;
  const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
  const int nseg = (n + 1 + L - 2) / (L - 1);  // segments covering faces 0..n
  const int lane = threadIdx.x & 31;
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int s = DIR == 0 ? lane % L : lane / W;  // position in the segment
  int seg, a, b;                                 // segment; transverse indices (0-based)
  bool valid;
  size_t base;
  long long stride;
  if (DIR == 0) {
    const long long ntr = (long long)g.ny * g.nz;
    seg = (int)(wid % nseg);
    const long long p = (wid / nseg) * W + lane / L;
    valid = p < ntr;
    a = (int)(p % g.ny);
    b = (int)(p / g.ny);
    base = ((size_t)b * g.ny + a) * g.nx;
    stride = 1;
  } else {
    const int nxg = (g.nx + W - 1) / W;
    const int nbt = DIR == 1 ? g.nz : g.ny;
    const long long xg = wid % nxg;
    const long long r = wid / nxg;
    seg = (int)(r % nseg);
    b = (int)(r / nseg);
    a = (int)(xg * W + lane % W);
    valid = a < g.nx && b < nbt;
    base = DIR == 1 ? (size_t)b * g.ny * g.nx + a : (size_t)b * g.nx + a;
    stride = DIR == 1 ? (long long)g.nx : (long long)g.nx * g.ny;
  }
  const int c = seg * (L - 1) - 1 + s;  // this lane's cell (0-based, -1..n are used)
  valid = valid && c <= n;
  const Metric M = make_metric(A.coordinates, A.sc->t, A.sc->t3);
  double plus[NV], minus[NV], ctr[4], wplus[4], wminus[4];
#pragma unroll
  for (int k = 0; k < NV; k++) plus[k] = minus[k] = 0.;
#pragma unroll
  for (int q = 0; q < 4; q++) ctr[q] = wplus[q] = wminus[q] = 0.;
  if (valid) {
    // the stencil v(c-2..c+2) of cell c: 1-based pencil positions c-1..c+3
    long long off[5];
    double sg[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
      int qq;
      map_ghost(c - 1 + q, n, A.bc.c[0][0], A.bc.c[0][1], qq, sg[q]);
      off[q] = (long long)base + (long long)(qq - 1) * stride;
    }
    double sv[3][5];
#pragma unroll
    for (int k = 0; k < NV; k++) {
      const double* vk = A.v + (size_t)k * g.ncell;
      double s5[5];
      if (A.bc_uniform) {
#pragma unroll
        for (int q = 0; q < 5; q++) s5[q] = __ldg(vk + off[q]);
        if (A.bc_signed) {
#pragma unroll
          for (int q = 0; q < 5; q++) s5[q] = sg[q] * s5[q];
        }
      } else {
#pragma unroll
        for (int q = 0; q < 5; q++) s5[q] = ghost_val(vk, base, stride, n, c - 1 + q, A.bc.c[k][0], A.bc.c[k][1]);
      }
      weno5_cell(s5[0], s5[1], s5[2], s5[3], s5[4], plus[k], minus[k]);
      if (k >= KVX && k <= KPR) ctr[k - KVX] = s5[2];
      if (T::VISC && k >= KVX && k <= KVZ) {
#pragma unroll
        for (int q = 0; q < 5; q++) sv[k - KVX][q] = s5[q];
      }
    }
    if (T::VISC) {
      double s4[4][5];
#pragma unroll
      for (int q = 0; q < 5; q++) {
        double vx = sv[0][q], vy = sv[1][q], vz = sv[2][q];
        double gg = 1. / sqrt(1. - vx * vx - vy * vy - M.g3 * (vz * vz));
        s4[0][q] = gg;
        s4[1][q] = gg * vx;
        s4[2][q] = gg * vy;
        s4[3][q] = gg * vz;
      }
#pragma unroll
      for (int q = 0; q < 4; q++) weno5_cell(s4[q][0], s4[q][1], s4[q][2], s4[q][3], s4[q][4], wplus[q], wminus[q]);
    }
  }
  // the cell below: its upper-face states and its centre (the fix-ups' w0)
  double wl[NV], w0[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) {
    wl[k] = __shfl_up_sync(0xffffffffu, plus[k], DELTA);
    w0[k] = 0.;
  }
#pragma unroll
  for (int q = 0; q < 4; q++) w0[KVX + q] = __shfl_up_sync(0xffffffffu, ctr[q], DELTA);
  if (T::VISC) {
#pragma unroll
    for (int q = 0; q < 4; q++) wplus[q] = __shfl_up_sync(0xffffffffu, wplus[q], DELTA);
  }
  double amax_local = 0.0;
  if (valid && s >= 1) {
    // face c, between cells c-1 and c
    const size_t nfaces = faces_of<DIR>(g);
    size_t fid;
    if (DIR == 0)
      fid = ((size_t)b * g.ny + a) * (g.nx + 1) + c;
    else if (DIR == 1)
      fid = ((size_t)b * (g.ny + 1) + c) * g.nx + a;
    else
      fid = ((size_t)c * g.ny + b) * g.nx + a;
    if (T::VISC) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        A.WD[(size_t)q * nfaces + fid] = wplus[q];
        A.WD[(size_t)(4 + q) * nfaces + fid] = wminus[q];
      }
    }
    double F[NV];
    int err = face_tail<KIND, DIR>(A.P, M, A.sc->glm_ch_old, wl, minus, w0, F, amax_local);
    if (err) {
      amax_local = 0.0;
      size_t cell = base + (size_t)((c >= 1 ? c : 1) - 1) * stride;
      atomicMin(&A.sc->err_key, ((unsigned long long)cell << 20) | (unsigned long long)err);
#pragma unroll
      for (int k = 0; k < NV; k++) A.F[(size_t)k * nfaces + fid] = 0.0;
    } else {
#pragma unroll
      for (int k = 0; k < NV; k++) A.F[(size_t)k * nfaces + fid] = F[k];
      // GLM speed of the reference: the last face of the last pencil (work.f90:217,310,401)
      const int na = DIR == 0 ? g.ny : g.nx;
      const int nb = DIR == 2 ? g.ny : g.nz;
      if (c == n && a == na - 1 && b == nb - 1) A.sc->aflux[DIR] = amax_local;
    }
  }
  block_max_atomic(amax_local, &A.sc->amax_bits[DIR], red);
}

// warps of faces_seg_kernel<DIR, L> for grid g
template <int DIR, int L>
__host__ __device__ inline long long seg_warps(const Grid& g) {
  constexpr int W = 32 / L;
  const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
  const long long nseg = (n + 1 + L - 2) / (L - 1);
  if (DIR == 0) return nseg * (((long long)g.ny * g.nz + W - 1) / W);
  return (long long)((g.nx + W - 1) / W) * nseg * (DIR == 1 ? g.nz : g.ny);
}
#endif

// ---------------------------------------------------------------------------
// scalar logic of evolve_main (evolve.f90:156-201) and evolve_dt (:723-764)
// ---------------------------------------------------------------------------
struct ScalarArgs {
  DevScalars* sc;
  Grid g;
  double cfl, maxdt, glm_alpha;
  int irk, nrk, divclean;
  int mode;  // 0: explicit RK stage (after the sweeps); 1: IMEX-SSP dt (before the
             // sweeps of stage 1, from the previous stage's speeds); 2: IMEX-SSP GLM;
             // 3, 4: the fused stage kernel's halves of mode 0 -- 3 before it
             // (glm_ch, dt, GLM damping: none of them depends on this stage's
             // faces when the host fuses the stage), 4 after it (glm_ch_old)
};

__device__ __forceinline__ void stage_scalars(const ScalarArgs& A) {
  DevScalars* sc = A.sc;
  if (A.mode == 4) {
    double m = sc->aflux[0];
    if (sc->aflux[1] > m) m = sc->aflux[1];
    if (sc->aflux[2] > m) m = sc->aflux[2];
    sc->glm_ch_old = m;
    return;
  }
  if (A.mode != 1) {
    // glm_ch = glm_ch_old (start of stage); glm_ch_old = maxval(aflux) (end of sweeps)
    sc->glm_ch = sc->glm_ch_old;
    if (A.mode != 3) {
      double m = sc->aflux[0];
      if (sc->aflux[1] > m) m = sc->aflux[1];
      if (sc->aflux[2] > m) m = sc->aflux[2];
      sc->glm_ch_old = m;
    }
  }
  if (A.irk == 1 && A.mode != 2) {
    double amax;
    if (A.divclean) {
      amax = 1;
    } else {
      amax = 0.;
      double c;
      if (A.g.nx > 1) {
        c = A.g.ddx * __longlong_as_double((long long)sc->amax_bits[0]);
        if (c > amax) amax = c;
      }
      if (A.g.ny > 1) {
        c = A.g.ddy * __longlong_as_double((long long)sc->amax_bits[1]);
        if (c > amax) amax = c;
      }
      if (A.g.nz > 1) {
        c = A.g.ddz * __longlong_as_double((long long)sc->amax_bits[2]);
        if (c > amax) amax = c;
      }
      if (amax == 0) {
        if (A.g.nx > 1 && A.g.ddx > amax) amax = A.g.ddx;
        if (A.g.ny > 1 && A.g.ddy > amax) amax = A.g.ddy;
        if (A.g.nz > 1 && A.g.ddz > amax) amax = A.g.ddz;
      }
    }
    double dtl = A.cfl / amax;
    if (A.maxdt < dtl) dtl = A.maxdt;
    if (sc->tout - sc->t < dtl) dtl = sc->tout - sc->t;
    if (fabs(sc->t + sc->dt - sc->tout) < 1.e-9) {
      dtl = sc->tout - sc->t;
    } else {
      if ((sc->t + 2. * dtl - sc->tout) > 1.e-9) dtl = (sc->tout - sc->t) / 2.;
    }
    sc->dt = dtl;
  }
  if (A.divclean && A.mode != 1) sc->expfact = exp(-sc->glm_ch * sc->glm_ch * A.glm_alpha * (sc->dt / 2.));
}

static __global__ void stage_scalars_kernel(ScalarArgs A) { stage_scalars(A); }

// end of step (echo.f90:211-241)
__device__ __forceinline__ void end_step_scalars(DevScalars* sc, int coordinates) {
  sc->timeold = sc->t;
  sc->t = sc->t + sc->dt;
  double g3 = coordinates == ECHO_BJORKEN ? sc->timeold * sc->timeold : 1.;
  sc->g3old = g3;
  sc->t3 = pow(sc->t, 3.);
  sc->timeinterval = sc->dt;
  if ((sc->t > sc->tout) || ((sc->tout - sc->t) < 1.e-10)) {
    sc->tout = sc->tout + sc->dtout;
    if ((fabs(sc->tout - sc->tmax) < 1.e-10) || (sc->tout > sc->tmax)) sc->tout = sc->tmax;
  }
}

static __global__ void end_step_kernel(DevScalars* sc, int coordinates) { end_step_scalars(sc, coordinates); }

// check_temp (out.f90:1487-1557): the quantity the stop criterion compares
// with TEMP_END -- the temperature (freeze_type 0) or the energy density
// (freeze_type 1) of a cell from its rho and p, as
// get_derived_temp_for_check (eos.f90:706-759, 972-983) gives them (the
// interpolation of get_derived_data).  A cell outside the table does not
// count: the reference keeps the previous cell's value there.
__device__ __forceinline__ double check_value(const DevPhys& P, int freeze_type, double rh, double pr) {
  double en = 0., temp = 0., s = 0.;
  if (get_derived_data(P, rh, pr, &en, &temp, &s)) return 0.;
  return freeze_type == 0 ? temp : en;
}

// grid maximum of check_value into *out (zeroed by the caller); the
// reference starts its maximum from 0
static __global__ void __launch_bounds__(256) check_temp_kernel(DevPhys P, Grid g, const double* __restrict__ v,
                                                                int freeze_type, unsigned long long* out) {
  __shared__ double red[8];
  double m = 0.;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.ncell; c += (size_t)gridDim.x * blockDim.x) {
    double x = check_value(P, freeze_type, v[(size_t)KRH * g.ncell + c], v[(size_t)KPR * g.ncell + c]);
    m = x > m ? x : m;
  }
  block_max_atomic(m, out, red);
}

// ---------------------------------------------------------------------------
// per-cell update
// ---------------------------------------------------------------------------
enum { MODE_RK = 0, MODE_RHS = 1 };

struct UpdateArgs {
  DevPhys P;
  Grid g;
  const double* __restrict__ Fx;
  const double* __restrict__ Fy;
  const double* __restrict__ Fz;
  const double* __restrict__ WDx;
  const double* __restrict__ WDy;
  const double* __restrict__ WDz;
  const double* __restrict__ vin;    // stage input primitives (guess for con2prim)
  double* __restrict__ vout;         // new primitives
  double* uin;                       // current conserved (updated in place)
  double* uout;                      // written u (== uin except stage 1)
  double* u0;                        // u at the start of the step
  const double* __restrict__ vnew;   // vnewstep (viscous time derivatives)
  const double* __restrict__ vold;   // vold
  double* du_out;                    // MODE_RHS: du
  unsigned char* fail;
  DevScalars* sc;
  double c1, c2;
  int irk, nrk, divclean, coordinates, algo, mode;
  double tol;
  // resistive runs: stiff right-hand side of E (MODE_RHS, 3 x ncell) and the
  // boundary codes of E^x, E^y, E^eta along x, y, eta for the charge density
  double* dus_out;
  signed char ebc[3][2];
  MlpDev mlp;  // learned seed (algo == ECHO_C2P_MLP)
  // viscous, stage 1 of a batched step: vnewstep = v (echo.f90:192-202) is
  // taken here, per cell, instead of by a separate copy; null otherwise
  double* vsnap;
};

// Learned con2prim seed of the calling lane's cell from its conserved
// variables uu (times sqrt(-g)).  Called by all lanes of the warp together;
// lanes without a cell pass active = false.
template <int KIND>
__device__ __forceinline__ void mlp_seed(const MlpDev& net, const Metric& M, bool active, const double* uu,
                                         float seed[2]) {
  float f[MLP_NIN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (active) {
    double gm = M.gm, g3 = M.g3;
    double D = gm * uu[KRH], sx = gm * uu[KVX], sy = gm * uu[KVY], sz = gm * uu[KVZ], U = gm * uu[KPR];
    double B2 = 0., SB = 0.;
    if (Traits<KIND>::MHD) {
      double bx = gm * uu[KBX], by = gm * uu[KBY], bz = gm * uu[KBZ];
      B2 = bx * bx + by * by + bz * bz * g3;
      SB = sx * bx + sy * by + sz * bz;
    }
    double SS2 = sx * sx + sy * sy + sz * sz / g3;
    double E2 = 0.;
    if (Traits<KIND>::RES) {
      // E contravariant: E^2 = E1^2 + E2^2 + g3 E3^2
      double ex = gm * uu[KEX], ey = gm * uu[KEY], ez = gm * uu[KEZ];
      E2 = ex * ex + ey * ey + ez * ez * g3;
    }
    if (U > 0.) mlp_invariants(D, SS2, U, B2, SB * SB, E2, f);
  }
  mlp_warp(net, f, seed);
}

// The update of cell c (flux divergence, sources, RK combination,
// con2prim).  Called by every thread of a warp together (the learned seed
// and the counters are warp-collective); threads without a cell pass
// active = false.  update_finish takes the flux divergence du[NV] (summed
// in the reference's order: du = 0; += x; += y; += z) and, for viscous
// runs, the spatial derivatives of u^mu in dv[NDER] (the rest zero); it
// adds the lagged time derivatives, the sources, and does the RK
// combination or writes du (MODE_RHS), then con2prim.  update_cell reads
// the face fluxes of the three sweep kernels; the fused stage kernel
// computes them itself (stage.cuh).
template <int KIND, bool SEED, bool IMEX = false>
__device__ __forceinline__ void update_finish(const UpdateArgs& A, size_t c, bool active, int ix, int iy, int iz,
                                              double* du, double* dv) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  const Grid& g = A.g;
  unsigned long long my_iters = 0, my_fallbacks = 0, my_brackets = 0;
  const Metric M = make_metric(A.coordinates, A.sc->t, A.sc->t3);
  double vv[NV], uu[NV];
  if (active) {
    double src[NV], kap[2] = {0., 0.};
#pragma unroll
    for (int k = 0; k < NV; k++) vv[k] = A.vin[(size_t)k * g.ncell + c];
    if (T::VISC) {
      if (A.vsnap) {
#pragma unroll
        for (int k = 0; k < 4; k++) A.vsnap[(size_t)k * g.ncell + c] = vv[k];
      }
      // dts (viscous.f90:56-97)
      double ti = A.sc->timeinterval;
      if (ti != 0) {
        double vxo = A.vold[1 * g.ncell + c], vyo = A.vold[2 * g.ncell + c], vzo = A.vold[3 * g.ncell + c];
        double vx, vy, vz;
        if (A.vsnap) {
          vx = vv[KVX];
          vy = vv[KVY];
          vz = vv[KVZ];
        } else {
          vx = A.vnew[1 * g.ncell + c];
          vy = A.vnew[2 * g.ncell + c];
          vz = A.vnew[3 * g.ncell + c];
        }
        double gamma1 = 1. / sqrt(1. - M.g1 * (vxo * vxo) - M.g2 * (vyo * vyo) - A.sc->g3old * (vzo * vzo));
        double gamma2 = 1. / sqrt(1. - M.g1 * (vx * vx) - M.g2 * (vy * vy) - M.g3 * (vz * vz));
        dv[DTT] = (gamma2 - gamma1) / (ti);
        dv[DXT] = (gamma2 * vx - gamma1 * vxo) / ti;
        dv[DYT] = (gamma2 * vy - gamma1 * vyo) / ti;
        dv[DZT] = (gamma2 * vz - gamma1 * vzo) / ti;
      }
    }
    // resistive: charge density d_i E^i by central differences with the
    // ghost fill (system_compute_divE, system.f90:1901-1919)
    double rhoC = 0., stiff[3] = {0., 0., 0.};
    if (T::RES) {
      if (g.nx > 1) {
        const double* a = A.vin + (size_t)KEX * g.ncell;
        double dx = 2. / g.ddx;
        rhoC = rhoC + (ghost_val(a, c - ix, 1, g.nx, ix + 2, A.ebc[0][0], A.ebc[0][1]) -
                       ghost_val(a, c - ix, 1, g.nx, ix, A.ebc[0][0], A.ebc[0][1])) / dx;
      }
      if (g.ny > 1) {
        const double* a = A.vin + (size_t)KEY * g.ncell;
        size_t base = c - (size_t)iy * g.nx;
        double dy = 2. / g.ddy;
        rhoC = rhoC + (ghost_val(a, base, g.nx, g.ny, iy + 2, A.ebc[1][0], A.ebc[1][1]) -
                       ghost_val(a, base, g.nx, g.ny, iy, A.ebc[1][0], A.ebc[1][1])) / dy;
      }
      if (g.nz > 1) {
        const double* a = A.vin + (size_t)KEZ * g.ncell;
        long long nxy = (long long)g.nx * g.ny;
        size_t base = c - (size_t)iz * (size_t)nxy;
        double dz = 2. / g.ddz;
        rhoC = rhoC + (ghost_val(a, base, nxy, g.nz, iz + 2, A.ebc[2][0], A.ebc[2][1]) -
                       ghost_val(a, base, nxy, g.nz, iz, A.ebc[2][0], A.ebc[2][1])) / dz;
      }
    }
    {
      double vs[NV];
#pragma unroll
      for (int k = 0; k < NV; k++) vs[k] = vv[k];
      int err = system_source<KIND>(A.P, M, vs, dv, src, (T::VISC && IMEX) ? kap : nullptr, rhoC,
                                    T::RES ? stiff : nullptr);
      if (err) atomicMin(&A.sc->err_key, ((unsigned long long)c << 20) | (unsigned long long)err);
    }
#pragma unroll
    for (int k = 0; k < NV; k++) du[k] = du[k] - src[k];
    if (A.mode == MODE_RHS) {
#pragma unroll
      for (int k = 0; k < NV; k++) A.du_out[(size_t)k * g.ncell + c] = du[k];
      if (T::RES && A.dus_out) {
#pragma unroll
        for (int i = 0; i < 3; i++) A.dus_out[(size_t)i * g.ncell + c] = 0. - stiff[i];
      }
    } else {
      // RK combination (evolve.f90:196-201)
      const double dt = A.sc->dt;
#pragma unroll
      for (int k = 0; k < NV; k++) {
        double ui = A.uin[(size_t)k * g.ncell + c];
        if (T::GLM && k == T::KG && A.irk == 1) {
          ui = ui * A.sc->expfact;
          A.uin[(size_t)k * g.ncell + c] = ui;  // u0 = u after the GLM half step
        }
        double u0 = A.irk == 1 ? ui : A.u0[(size_t)k * g.ncell + c];
        if (T::VISC && IMEX && k >= KPIBU) {
          // IMEX RK2/RK3: the relaxation -kap u of the stresses at the new
          // stage value, u_new = u_expl + c2 dt kap (u - u_new)
          double ck = A.c2 * dt * (k == KPIBU ? kap[0] : kap[1]);
          uu[k] = (A.c1 * u0 + A.c2 * (ui - dt * du[k]) + ck * ui) / (1. + ck);
        } else {
          uu[k] = A.c1 * u0 + A.c2 * (ui - dt * du[k]);
        }
      }
      if (T::GLM && A.irk == A.nrk) uu[T::KG] = uu[T::KG] * A.sc->expfact;
#pragma unroll
      for (int k = 0; k < NV; k++) A.uout[(size_t)k * g.ncell + c] = uu[k];
    }
  }
  if (A.mode == MODE_RK) {
    // learned seed, one warp at a time on the tensor cores
    float seed[2] = {0.f, 0.f};
    const float* sp = nullptr;
    if (SEED) {
      mlp_seed<KIND>(A.mlp, M, active, uu, seed);
      sp = seed;
    }
    if (active && !(T::MHD && !T::RES && c2p_alt_algo(A.algo))) {  // ALG_SOLV 2..6: c2p_alt_kernel
      // con2prim (evolve_u2v, evolve.f90:789-866)
      int it = 0, sfail = 0;
      int err = cons2prim<KIND>(A.P, M, A.algo, A.tol, uu, vv, &it, sp, &sfail);
      my_iters = (unsigned long long)it;
      my_fallbacks = (unsigned long long)(sfail & 1);
      my_brackets = (unsigned long long)(sfail >> 1);
      if (err) {
        A.fail[c] = 1;
        atomicAdd(&A.sc->nfail, 1);
      } else {
        A.fail[c] = 0;
#pragma unroll
        for (int k = 0; k < NV; k++) A.vout[(size_t)k * g.ncell + c] = vv[k];
      }
    }
    // per-warp sums of iteration counts, seed and bracketed fallbacks
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      my_iters += __shfl_xor_sync(0xffffffffu, my_iters, o);
      my_fallbacks += __shfl_xor_sync(0xffffffffu, my_fallbacks, o);
      my_brackets += __shfl_xor_sync(0xffffffffu, my_brackets, o);
    }
    if ((threadIdx.x & 31) == 0 && my_iters) atomicAdd(&A.sc->c2p_iters, my_iters);
    if ((threadIdx.x & 31) == 0 && my_fallbacks) atomicAdd(&A.sc->fallbacks, my_fallbacks);
    if ((threadIdx.x & 31) == 0 && my_brackets) atomicAdd(&A.sc->brackets, my_brackets);
  }
}


template <int KIND, bool SEED, bool IMEX = false>
__device__ __forceinline__ void update_cell(const UpdateArgs& A, size_t c, bool active) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  const Grid& g = A.g;
  int ix = 0, iy = 0, iz = 0;
  double du[NV], dv[NDER];
  if (active) {
    if (g.ncell < (1ull << 32)) {  // multiply-high divisions (FastDiv)
      const unsigned cc = (unsigned)c, r = fast_div(cc, g.dnx), q = fast_div(r, g.dny);
      ix = (int)(cc - r * (unsigned)g.nx);
      iy = (int)(r - q * (unsigned)g.ny);
      iz = (int)q;
    } else {
      ix = (int)(c % g.nx);
      size_t r = c / g.nx;
      iy = (int)(r % g.ny);
      iz = (int)(r / g.ny);
    }
    const size_t nfx = (size_t)(g.nx + 1) * g.ny * g.nz;
    const size_t nfy = (size_t)g.nx * (g.ny + 1) * g.nz;
    const size_t nfz = (size_t)g.nx * g.ny * (g.nz + 1);
    const size_t fx = ((size_t)iz * g.ny + iy) * (g.nx + 1) + ix;       // face ix-1/2 -> index ix
    const size_t fy = ((size_t)iz * (g.ny + 1) + iy) * g.nx + ix;
    const size_t fz = ((size_t)iz * g.ny + iy) * g.nx + ix;
    // flux divergence in the reference's order: du = 0; += x; += y; += z
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double d = 0.;
      if (g.nx > 1) d = d + g.ddx * (A.Fx[(size_t)k * nfx + fx + 1] - A.Fx[(size_t)k * nfx + fx]);
      if (g.ny > 1) d = d + g.ddy * (A.Fy[(size_t)k * nfy + fy + g.nx] - A.Fy[(size_t)k * nfy + fy]);
      if (g.nz > 1)
        d = d + g.ddz * (A.Fz[(size_t)k * nfz + fz + (size_t)g.nx * g.ny] - A.Fz[(size_t)k * nfz + fz]);
      du[k] = d;
    }
    if (T::VISC) {
#pragma unroll
      for (int q = 0; q < NDER; q++) dv[q] = 0.;
      const int dk[3][4] = {{DTX, DXX, DYX, DZX}, {DTY, DXY, DYY, DZY}, {DTZ, DXZ, DYZ, DZZ}};
      if (g.nx > 1) {
#pragma unroll
        for (int q = 0; q < 4; q++)
          dv[dk[0][q]] = g.ddx * 0.5 *
                         (A.WDx[(size_t)q * nfx + fx + 1] + A.WDx[(size_t)(4 + q) * nfx + fx + 1] -
                          A.WDx[(size_t)q * nfx + fx] - A.WDx[(size_t)(4 + q) * nfx + fx]);
      }
      if (g.ny > 1) {
#pragma unroll
        for (int q = 0; q < 4; q++)
          dv[dk[1][q]] = g.ddy * 0.5 *
                         (A.WDy[(size_t)q * nfy + fy + g.nx] + A.WDy[(size_t)(4 + q) * nfy + fy + g.nx] -
                          A.WDy[(size_t)q * nfy + fy] - A.WDy[(size_t)(4 + q) * nfy + fy]);
      }
      if (g.nz > 1) {
        size_t s = (size_t)g.nx * g.ny;
#pragma unroll
        for (int q = 0; q < 4; q++)
          dv[dk[2][q]] = g.ddz * 0.5 *
                         (A.WDz[(size_t)q * nfz + fz + s] + A.WDz[(size_t)(4 + q) * nfz + fz + s] -
                          A.WDz[(size_t)q * nfz + fz] - A.WDz[(size_t)(4 + q) * nfz + fz]);
      }
    }
  }
  update_finish<KIND, SEED, IMEX>(A, c, active, ix, iy, iz, du, dv);
}

template <int KIND, bool SEED, bool IMEX = false>
__global__ void ECHO_UPDATE_BOUNDS(KIND, SEED) update_kernel(UpdateArgs A) {
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  update_cell<KIND, SEED, IMEX>(A, c, c < A.g.ncell);
}

// ---------------------------------------------------------------------------
// IMEX-SSP3(4,3,3) stage combinations (evolve.f90:235-266) + con2prim.  The
// stiff right-hand sides du_stiff are exact zeros without resistivity; they
// are kept as explicit 0.0 terms so the arithmetic is the reference's.
// ---------------------------------------------------------------------------
struct SspArgs {
  DevPhys P;
  Grid g;
  const double* __restrict__ u0;
  const double* __restrict__ du1;
  const double* __restrict__ du2;
  const double* __restrict__ du3;
  const double* __restrict__ du4;
  // resistive runs: the stiff right-hand sides of E of stages 1..4 (3 x ncell
  // each; null otherwise); stage 1 (ssp_stage1_kernel) writes ds1
  const double* __restrict__ ds1;
  const double* __restrict__ ds2;
  const double* __restrict__ ds3;
  const double* __restrict__ ds4;
  double* ds_out;
  double* __restrict__ uout;
  const double* __restrict__ vin;
  double* __restrict__ vout;
  unsigned char* fail;
  DevScalars* sc;
  int stage;  // 2, 3, 4: the combination that opens stage irk; 5: the final one
  int coordinates, algo, divclean;
  double tol;
  MlpDev mlp;
};

template <int KIND, bool SEED>
__global__ void __launch_bounds__(128, ECHO_SSP_MINB) ssp_combine_kernel(SspArgs A) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  const double alpha_imex = 0.24169426078821, beta_imex = 0.06042356519705, eta_imex = 0.12915286960590;
  const double delta_imex = 0.5 - beta_imex - eta_imex - alpha_imex;
  const Grid& g = A.g;
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long my_iters = 0;
  const bool active = c < g.ncell;
  const Metric M = make_metric(A.coordinates, A.sc->t, A.sc->t3);
  double uu[NV], vv[NV];
  const double dt = A.sc->dt;
  if (active) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      size_t i = (size_t)k * g.ncell + c;
      double u0 = A.u0[i];
      // stiff right-hand sides: zero but for E of resistive runs
      double s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
      if (T::RES && k >= KEX && k <= KEZ) {
        size_t j = (size_t)(k - KEX) * g.ncell + c;
        if (A.stage == 2 || A.stage == 4) s1 = A.ds1[j];
        if (A.stage >= 3) s2 = A.ds2[j];
        if (A.stage >= 4) s3 = A.ds3[j];
        if (A.stage == 5) s4 = A.ds4[j];
      }
      if (A.stage == 2) {
        uu[k] = u0 + dt * alpha_imex * s1;
      } else if (A.stage == 3) {
        uu[k] = u0 - dt * (A.du2[i] + (1. - alpha_imex) * s2);
      } else if (A.stage == 4) {
        uu[k] = u0 - dt * (A.du2[i] / 4. + A.du3[i] / 4. + beta_imex * s1 + eta_imex * s2 + delta_imex * s3);
      } else {
        uu[k] = u0 - dt * (A.du2[i] / 6. + A.du3[i] / 6. + A.du4[i] * 2. / 3. + s2 / 6. + s3 / 6. + s4 * 2. / 3.);
      }
      vv[k] = A.vin[i];
    }
    if (T::GLM && A.stage == 5) uu[T::KG] = uu[T::KG] * A.sc->expfact;
#pragma unroll
    for (int k = 0; k < NV; k++) A.uout[(size_t)k * g.ncell + c] = uu[k];
  }
  float seed[2] = {0.f, 0.f};
  const float* sp = nullptr;
  if (SEED) {
    mlp_seed<KIND>(A.mlp, M, active, uu, seed);
    sp = seed;
  }
  unsigned long long my_fallbacks = 0;
  if (active && !(T::MHD && !T::RES && c2p_alt_algo(A.algo))) {  // ALG_SOLV 2..6: c2p_alt_kernel
    int it = 0, sfail = 0;
    // the implicit stages of a resistive run solve Ohm's law in con2prim
    const double h = (T::RES && A.stage < 5) ? alpha_imex * dt : 0.;
    int err = cons2prim<KIND>(A.P, M, A.algo, A.tol, uu, vv, &it, sp, &sfail, h);
    my_iters = (unsigned long long)it;
    my_fallbacks = (unsigned long long)(sfail & 1);
    if (err) {
      A.fail[c] = 1;
      atomicAdd(&A.sc->nfail, 1);
    } else {
      A.fail[c] = 0;
#pragma unroll
      for (int k = 0; k < NV; k++) A.vout[(size_t)k * g.ncell + c] = vv[k];
      if (T::RES && h > 0.) {
#pragma unroll
        for (int k = KEX; k <= KEZ; k++) A.uout[(size_t)k * g.ncell + c] = uu[k];
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    my_iters += __shfl_xor_sync(0xffffffffu, my_iters, o);
    if (SEED) my_fallbacks += __shfl_xor_sync(0xffffffffu, my_fallbacks, o);
  }
  if ((threadIdx.x & 31) == 0 && my_iters) atomicAdd(&A.sc->c2p_iters, my_iters);
  if (SEED && (threadIdx.x & 31) == 0 && my_fallbacks) atomicAdd(&A.sc->fallbacks, my_fallbacks);
}

// Resistive IMEX-SSP3(4,3,3), first stage: U1 = u^n + alpha dt S(U1), solved
// from u0 = u^n cell by cell (the implicit stage the reference leaves to its
// missing algo-7 con2prim); ds_out = -S(U1), the stiff E right-hand side the
// later stages combine (only S(U1) enters them: F(U1) has weight 0).  v and
// u stay at step n; a failed solve stops the run with its code.  SEED: the
// solve starts from the learned seed (warp-collective inference, so every
// lane reaches it).
template <int KIND, bool SEED>
__global__ void __launch_bounds__(128, ECHO_SSP_MINB) ssp_stage1_kernel(SspArgs A) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  const double alpha_imex = 0.24169426078821;
  const Grid& g = A.g;
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = c < g.ncell;
  if (!T::RES || (!SEED && !active)) return;
  const Metric M = make_metric(A.coordinates, A.sc->t, A.sc->t3);
  double uu[NV], vv[NV], S[3];
#pragma unroll
  for (int k = 0; k < NV; k++) {
    uu[k] = active ? A.u0[(size_t)k * g.ncell + c] : 1.0;
    vv[k] = active ? A.vin[(size_t)k * g.ncell + c] : 0.0;
  }
  float seed[2] = {0.f, 0.f};
  const float* sp = nullptr;
  if (SEED) {
    mlp_seed<KIND>(A.mlp, M, active, uu, seed);
    sp = seed;
  }
  if (!active) return;
  int it = 0, sfail = 0;
  int err = cons2prim<KIND>(A.P, M, A.algo, A.tol, uu, vv, &it, sp, &sfail, alpha_imex * A.sc->dt);
  if (SEED && (sfail & 1)) atomicAdd(&A.sc->fallbacks, 1ull);
  if (err) {
    atomicMin(&A.sc->err_key, ((unsigned long long)c << 20) | (unsigned long long)err);
    return;
  }
  double v2 = M.g1 * vv[KVX] * vv[KVX] + M.g2 * vv[KVY] * vv[KVY] + M.g3 * vv[KVZ] * vv[KVZ];
  double glf = 1. / sqrt(1. - v2);
  ohm_stiff(A.P, M, vv + KVX, vv + KBX, vv + KEX, glf, S);
#pragma unroll
  for (int i = 0; i < 3; i++) A.ds_out[(size_t)i * g.ncell + c] = 0. - S[i] * M.gp;
}

// ---------------------------------------------------------------------------
// repair of failed cells (evolve.f90:795-842) in Fortran loop order
// ---------------------------------------------------------------------------
// con2prim of every cell with ALG_SOLV 2..6 (the step kernels wrote u and
// skipped the inversion): the same flags, counters and outputs as theirs
template <int KIND>
__global__ void __launch_bounds__(128) c2p_alt_kernel(DevPhys P, Grid g, int coordinates, int algo, double tol,
                                                     DevScalars* sc, const double* __restrict__ u,
                                                     const double* __restrict__ vin, double* __restrict__ vout,
                                                     unsigned char* fail) {
  typedef Traits<KIND> T;
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long my_iters = 0;
  if (c < g.ncell) {
    const Metric M = make_metric(coordinates, sc->t, sc->t3);
    double uu[T::NV], vv[T::NV];
#pragma unroll
    for (int k = 0; k < T::NV; k++) {
      uu[k] = u[(size_t)k * g.ncell + c];
      vv[k] = vin[(size_t)k * g.ncell + c];
    }
    int it = 0;
    int err = cons2prim<KIND, true>(P, M, algo, tol, uu, vv, &it);
    my_iters = (unsigned long long)it;
    if (err) {
      fail[c] = 1;
      atomicAdd(&sc->nfail, 1);
    } else {
      fail[c] = 0;
#pragma unroll
      for (int k = 0; k < T::NV; k++) vout[(size_t)k * g.ncell + c] = vv[k];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_iters += __shfl_xor_sync(0xffffffffu, my_iters, o);
  if ((threadIdx.x & 31) == 0 && my_iters) atomicAdd(&sc->c2p_iters, my_iters);
}

struct RepairArgs {
  DevPhys P;
  Grid g;
  const double* __restrict__ vold;  // stage input primitives (old v)
  double* vnew;                     // new primitives (filled for good cells)
  double* u;                        // conserved after the RK update
  unsigned char* fail;
  DevScalars* sc;
  int coordinates, algo;
  double maxspeed, tol;
  double h_alpha;  // resistive implicit stages: a_ii, the solve uses h = a_ii dt
};

template <int KIND>
__device__ double flat_v(const RepairArgs& A, long long off, size_t cell) {
  // Fortran flat address into v: cells before `cell` hold their new value
  size_t tot = A.g.ncell * Traits<KIND>::NV;
  if (off < 0 || (size_t)off >= tot) return 0.;
  size_t cc = (size_t)off % A.g.ncell;
  return cc < cell ? A.vnew[off] : A.vold[off];
}
__device__ __forceinline__ double flat_u(const double* u, size_t tot, long long off) {
  if (off < 0 || (size_t)off >= tot) return 0.;
  return u[off];
}

// The repair of one failed cell (evolve.f90:795-842): con2prim of the
// failed state, the six-neighbour average of u in the reference's flat
// addressing (flat_u), con2prim, the velocity and pressure fixes, prim2cons
// and con2prim again.  The reference averages in place, so where a flat
// neighbour is the same cell (2-D grids, whose eta offset nx*ny is one
// variable's length) it reads the already averaged variable: un[] holds
// those.  Returns whether the repaired state is valid; uu and vv receive the
// conserved and primitive values to store.
template <int KIND>
__device__ __noinline__ bool repair_cell(const RepairArgs& A, const Metric& M, double h, size_t cell, double* uu,
                                         double* vv) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  const Grid& g = A.g;
  int it;
  for (int k = 0; k < NV; k++) vv[k] = A.vold[(size_t)k * g.ncell + cell];
  for (int k = 0; k < NV; k++) uu[k] = A.u[(size_t)k * g.ncell + cell];
  (void)cons2prim<KIND, true>(A.P, M, A.algo, A.tol, uu, vv, &it, nullptr, nullptr, h);
  const size_t totu = g.ncell * NV;
  const long long nx = g.nx, nxy = (long long)g.nx * g.ny;
  double un[NV];
  for (int k = 0; k < NV; k++) {
    const long long o = (long long)k * g.ncell + (long long)cell;
    const long long q[6] = {o - 1, o + 1, o - nx, o + nx, o - nxy, o + nxy};
    double a[6];
    for (int j = 0; j < 6; j++) {
      a[j] = flat_u(A.u, totu, q[j]);
      if (q[j] >= 0 && (size_t)q[j] < totu && (size_t)q[j] % g.ncell == cell) {
        const int kq = (int)((size_t)q[j] / g.ncell);
        if (kq < k) a[j] = un[kq];
      }
    }
    un[k] = (a[0] + a[1] + a[2] + a[3] + a[4] + a[5]) / 6.;
    uu[k] = un[k];
  }
  (void)cons2prim<KIND, true>(A.P, M, A.algo, A.tol, uu, vv, &it, nullptr, nullptr, h);
  double v2 = vv[KVX] * vv[KVX] + vv[KVY] * vv[KVY] + vv[KVZ] * vv[KVZ] * M.g3;
  if (v2 > 1) {
    double fac = A.maxspeed / sqrt(v2);
    vv[KVX] = fac * vv[KVX];
    vv[KVY] = fac * vv[KVY];
    vv[KVZ] = fac * vv[KVZ];
  }
  if (vv[KPR] < 0) {
    long long o = (long long)KPR * g.ncell + (long long)cell;
    double pxl = flat_v<KIND>(A, o - 1, cell), pxr = flat_v<KIND>(A, o + 1, cell);
    double pyl = flat_v<KIND>(A, o - nx, cell), pyr = flat_v<KIND>(A, o + nx, cell);
    double pzl = flat_v<KIND>(A, o - nxy, cell), pzr = flat_v<KIND>(A, o + nxy, cell);
    vv[KPR] = (pxl + pxr + pyl + pyr + pzl + pzr) / 6.;
  }
  (void)prim2cons<KIND>(A.P, M, vv, uu);
  (void)cons2prim<KIND, true>(A.P, M, A.algo, A.tol, uu, vv, &it, nullptr, nullptr, h);
  v2 = vv[KVX] * vv[KVX] + vv[KVY] * vv[KVY] + vv[KVZ] * vv[KVZ] * M.g3;
  return (vv[KPR] > 0) && (v2 < 1);
}

// Whether failed cell c reads another failed cell: its flat neighbours
// c +- 1, c +- nx, c +- nx*ny of any variable (modulo the cell count).
__device__ __forceinline__ bool repair_touches(const unsigned char* fail, const Grid& g, size_t c) {
  const long long n = (long long)g.ncell;
  const long long d[3] = {1, (long long)g.nx, (long long)g.nx * g.ny};
  for (int j = 0; j < 3; j++) {
    const long long dd = d[j] % n;
    const long long lo = ((long long)c - dd + n) % n, hi = ((long long)c + dd) % n;
    if ((lo != (long long)c && fail[lo]) || (hi != (long long)c && fail[hi])) return true;
  }
  return false;
}

// The repair of every failed cell of a grid.  The reference repairs them
// one after another in cell order, each reading its neighbours' current u
// and v, and stops at the first cell it cannot repair (the run crashes).
// Called by every thread of one block; s_any and s_stop are block-shared.
// s_list (CAP entries, block-shared; CAP may be 0) holds the failed cells in
// order: when they fit and none reads another, their repairs do not depend
// on each other, so the block repairs them in parallel, a round of
// blockDim.x cells at a time in cell order, and stores what the sequential
// loop would: every cell before the first failure in full, the failing cell's
// u, nothing after it.  Otherwise thread 0 repairs them in order.
template <int KIND, int CAP>
__device__ __forceinline__ void repair_grid(const RepairArgs& A, int& s_any, int& s_stop, unsigned* s_list) {
  typedef Traits<KIND> T;
  const int NV = T::NV;
  const Grid& g = A.g;
  const Metric M = make_metric(A.coordinates, A.sc->t, A.sc->t3);
  const double h = A.h_alpha * A.sc->dt;
  __shared__ int s_n, s_conflict;
  __shared__ int s_wc[32];
  __shared__ unsigned s_crash;
  if (threadIdx.x == 0) {
    s_stop = 0;
    s_n = 0;
    s_conflict = CAP == 0 || g.ncell >= 0xffffffffull;
  }
  __syncthreads();
  if (CAP > 0 && !s_conflict) {
    // the failed cells in order, and whether any reads another
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    for (size_t chunk = 0; chunk < g.ncell; chunk += blockDim.x) {
      const size_t c = chunk + threadIdx.x;
      const bool f = c < g.ncell && A.fail[c];
      if (f && repair_touches(A.fail, g, c)) s_conflict = 1;
      const unsigned bal = __ballot_sync(0xffffffffu, f);
      if (lane == 0) s_wc[w] = __popc(bal);
      __syncthreads();
      if (f) {
        int pos = s_n + __popc(bal & ((1u << lane) - 1u));
        for (int i = 0; i < w; i++) pos += s_wc[i];
        if (pos < CAP) s_list[pos] = (unsigned)c;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int tot = 0;
        for (int i = 0; i < nw; i++) tot += s_wc[i];
        s_n += tot;
      }
      __syncthreads();
    }
  }
  if (CAP > 0 && !s_conflict && s_n <= CAP) {
    const int n = s_n;
    for (int r = 0; r < n; r += blockDim.x) {
      const int i = r + (int)threadIdx.x;
      const bool mine = i < n;
      const size_t cell = mine ? s_list[i] : 0;
      double uu[NV], vv[NV];
      bool ok = true;
      if (mine) ok = repair_cell<KIND>(A, M, h, cell, uu, vv);
      if (threadIdx.x == 0) s_crash = 0xffffffffu;
      __syncthreads();
      if (mine && !ok) atomicMin(&s_crash, (unsigned)cell);
      __syncthreads();
      const unsigned crash = s_crash;
      if (mine && cell <= crash) {
        atomicAdd(&A.sc->repairs, 1ull);
        if (T::VISC && A.P.obtained_zz) A.vnew[(size_t)KPIZZ * g.ncell + cell] = vv[KPIZZ];
        for (int k = 0; k < NV; k++) A.u[(size_t)k * g.ncell + cell] = uu[k];
        if (cell < crash) {
          for (int k = 0; k < NV; k++) A.vnew[(size_t)k * g.ncell + cell] = vv[k];
        } else {
          // the run crashes here (evolve.f90:836-858)
          atomicMin(&A.sc->err_key, ((unsigned long long)cell << 20) | 1ull);
        }
      }
      __syncthreads();  // every thread has read s_crash before the next round resets it
      if (crash != 0xffffffffu) {
        if (threadIdx.x == 0) s_stop = 1;
        break;
      }
    }
    return;
  }
  for (size_t chunk = 0; chunk < g.ncell; chunk += blockDim.x) {
    size_t c = chunk + threadIdx.x;
    int f = (c < g.ncell) ? A.fail[c] : 0;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    if (f) atomicOr(&s_any, 1);
    __syncthreads();
    int any = s_any;
    __syncthreads();  // everyone has read s_any before thread 0 resets it
    if (!any) continue;
    if (threadIdx.x == 0) {
      for (unsigned t = 0; t < blockDim.x && chunk + t < g.ncell; t++) {
        size_t cell = chunk + t;
        if (!A.fail[cell]) continue;
        A.sc->repairs++;
        double uu[NV], vv[NV];
        const bool ok = repair_cell<KIND>(A, M, h, cell, uu, vv);
        if (T::VISC && A.P.obtained_zz) A.vnew[(size_t)KPIZZ * g.ncell + cell] = vv[KPIZZ];
        for (int k = 0; k < NV; k++) A.u[(size_t)k * g.ncell + cell] = uu[k];
        if (!ok) {
          // the run crashes here (evolve.f90:836-858): stop repairing
          atomicMin(&A.sc->err_key, ((unsigned long long)cell << 20) | 1ull);
          s_stop = 1;
          break;
        }
        for (int k = 0; k < NV; k++) A.vnew[(size_t)k * g.ncell + cell] = vv[k];
      }
    }
    __syncthreads();
    if (s_stop) break;
  }
}

// failed cells a repair block can list (4 KiB of shared memory)
#define ECHO_REPAIR_LIST 1024

template <int KIND>
__global__ void __launch_bounds__(256) repair_kernel(RepairArgs A) {
  if (A.sc->nfail == 0) return;
  __shared__ int s_any, s_stop;
  __shared__ unsigned s_list[ECHO_REPAIR_LIST];
  repair_grid<KIND, ECHO_REPAIR_LIST>(A, s_any, s_stop, s_list);
}

// evolve_smooth_viscosity (evolve.f90:1159-1207)
struct SmoothArgs {
  DevPhys P;
  Grid g;
  double* v;
  double* u;
  DevScalars* sc;
  int coordinates;
  double smooth_pressure;
};

template <int KIND>
__device__ __forceinline__ void smooth_cell(const SmoothArgs& A, size_t c) {
  typedef Traits<KIND> T;
  double pr = A.v[(size_t)KPR * A.g.ncell + c];
  if (!(pr < A.smooth_pressure)) return;
  const Metric M = make_metric(A.coordinates, A.sc->t, A.sc->t3);
  double vv[T::NV], uu[T::NV];
#pragma unroll
  for (int k = 0; k < T::NV; k++) vv[k] = A.v[(size_t)k * A.g.ncell + c];
  double rr = vv[KPR] / A.smooth_pressure;
  double fac = rr * rr;
#pragma unroll
  for (int k = KPIBU; k <= KPIZZ; k++) vv[k] = vv[k] * fac;
  if (A.P.obtained_zz) {
    Pit pi;
    derived_pi_zz(M, vv, pi);
    vv[KPIZZ] = pi.zz;
  }
  int err = prim2cons<KIND>(A.P, M, vv, uu);
#pragma unroll
  for (int k = 0; k < T::NV; k++) {
    A.v[(size_t)k * A.g.ncell + c] = vv[k];
    A.u[(size_t)k * A.g.ncell + c] = uu[k];
  }
  if (err) atomicMin(&A.sc->err_key, ((unsigned long long)c << 20) | (unsigned long long)err);
}

template <int KIND>
__global__ void smooth_kernel(SmoothArgs A) {
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < A.g.ncell) smooth_cell<KIND>(A, c);
}

// system_prim2cons over the grid (state upload without u)
template <int KIND>
__global__ void prim2cons_kernel(DevPhys P, Grid g, int coordinates, DevScalars* sc, double* v, double* u) {
  typedef Traits<KIND> T;
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.ncell) return;
  const Metric M = make_metric(coordinates, sc->t, sc->t3);
  double vv[T::NV], uu[T::NV];
#pragma unroll
  for (int k = 0; k < T::NV; k++) vv[k] = v[(size_t)k * g.ncell + c];
  int err = prim2cons<KIND>(P, M, vv, uu);
  if (err) atomicMin(&sc->err_key, ((unsigned long long)c << 20) | (unsigned long long)err);
#pragma unroll
  for (int k = 0; k < T::NV; k++) {
    v[(size_t)k * g.ncell + c] = vv[k];
    u[(size_t)k * g.ncell + c] = uu[k];
  }
}

}  // namespace echo
