// hyper.cu -- the freeze-out hypersurface on the device: out_hyp
// (out.f90:1569-1650) with find_hypersurface_ideal / _visco / _mhd
// (hypersurface.f90:172-229 and twins) and set_fo_ide / set_fo_vis
// (:354-460, :984-1117).
//
// Every call turns the freeze field (temperature or energy density from
// get_derived_data) of the current primitives into slice 2, the previous
// slice 2 into slice 1, and from the second call on collects the surface
// elements: per cell, a crossing of the freeze value in tau (between the
// slices) and in x, y, eta (towards the next cell, inside slice 1).  The
// reference fills its output in the loop order ix outer, iz inner, and per
// cell tau, x, y, eta; here each cell counts its crossings, a block scan in
// that order gives every cell its first slot, and the elements are written
// straight to their slots -- the reference's order, with no sort.
//
// Record of one element (8 + nv doubles): tau, x, y, eta; the nv primitives
// interpolated to the crossing; dV_tau, dV_x, dV_y, dV_eta times the
// crossing's sign (for ideal and viscous runs: hy_ide's and hy_vis's
// columns, in their order).
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
      fprintf(stderr, "echo_hyp: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                        \
      return ECHO_ERR_CUDA;                                                                     \
    }                                                                                           \
  } while (0)

namespace {

enum { SCAN_T = 1024 };

struct HypDev {
  const double* f1;    // freeze field of slice 1 (older)
  const double* f2;    // and slice 2
  const double* back;  // primitives of slice 1 (v_backup)
  const double* prim;  // primitives of slice 2 (primitives)
  int nx, ny, nz, nv;
  size_t ncell;
  double x1, y1, z1, dx, dy, dz, dzv;  // dzv = d_val(3): dz, or 1 for one eta cell
  double t1, t2, g3, fv;
};

// bit d set: a crossing in direction d (0 tau, 1 x, 2 y, 3 eta) from the
// cell with reference-order index r
__device__ __forceinline__ unsigned hyp_flags(const HypDev& H, size_t r, int& ix, int& iy, int& iz, size_t& c) {
  iz = (int)(r % H.nz) + 1;
  size_t q = r / H.nz;
  iy = (int)(q % H.ny) + 1;
  ix = (int)(q / H.ny) + 1;
  c = ((size_t)(iz - 1) * H.ny + (iy - 1)) * H.nx + (ix - 1);
  const double fv = H.fv, f1c = H.f1[c];
  unsigned m = 0;
  if ((H.f2[c] - fv) * (fv - f1c) > 0.0) m |= 1u;
  if (ix < H.nx && (H.f1[c + 1] - fv) * (fv - f1c) > 0.0) m |= 2u;
  if (iy < H.ny && (H.f1[c + H.nx] - fv) * (fv - f1c) > 0.0) m |= 4u;
  if (iz < H.nz && (H.f1[c + (size_t)H.nx * H.ny] - fv) * (fv - f1c) > 0.0) m |= 8u;
  return m;
}

__global__ void hyp_field_kernel(DevPhys P, const double* __restrict__ v, size_t ncell, int freeze_type,
                                 double* __restrict__ f, double* __restrict__ prim, int nv, int* err) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (size_t)gridDim.x * blockDim.x) {
    double en = 0., temp = 0., s = 0.;
    int e = get_derived_data(P, v[(size_t)KRH * ncell + c], v[(size_t)KPR * ncell + c], &en, &temp, &s);
    if (e > 0) atomicMin(err, e);
    f[c] = freeze_type == 0 ? temp : en;
    for (int k = 0; k < nv; k++) prim[(size_t)k * ncell + c] = v[(size_t)k * ncell + c];
  }
}

// block-local exclusive scan of the crossing counts in reference order
__global__ void __launch_bounds__(SCAN_T) hyp_count_kernel(HypDev H, int* __restrict__ off, int* __restrict__ bsum) {
  __shared__ int s[SCAN_T];
  const size_t r = (size_t)blockIdx.x * SCAN_T + threadIdx.x;
  int n = 0;
  if (r < H.ncell) {
    int ix, iy, iz;
    size_t c;
    n = __popc(hyp_flags(H, r, ix, iy, iz, c));
  }
  s[threadIdx.x] = n;
  __syncthreads();
  for (int o = 1; o < SCAN_T; o <<= 1) {
    int a = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += a;
    __syncthreads();
  }
  if (r < H.ncell) off[r] = s[threadIdx.x] - n;
  if (threadIdx.x == SCAN_T - 1) bsum[blockIdx.x] = s[SCAN_T - 1];
}

// exclusive scan of the block sums (one block, chunks of SCAN_T); total last
__global__ void __launch_bounds__(SCAN_T) hyp_scan_sums_kernel(int* __restrict__ bsum, int nb, int* __restrict__ total) {
  __shared__ int s[SCAN_T];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nb; b0 += SCAN_T) {
    const int b = b0 + threadIdx.x;
    int n = b < nb ? bsum[b] : 0;
    s[threadIdx.x] = n;
    __syncthreads();
    for (int o = 1; o < SCAN_T; o <<= 1) {
      int a = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
      __syncthreads();
      s[threadIdx.x] += a;
      __syncthreads();
    }
    if (b < nb) bsum[b] = carry + s[threadIdx.x] - n;
    __syncthreads();
    if (threadIdx.x == SCAN_T - 1) carry += s[SCAN_T - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// set_fo_* of one crossing into rec
__device__ __forceinline__ int hyp_element(const HypDev& H, int dir, int ix, int iy, int iz, size_t c, double* rec) {
  const int nv = H.nv;
  const size_t cc = dir == 0 ? c : dir == 1 ? c + 1 : dir == 2 ? c + H.nx : c + (size_t)H.nx * H.ny;
  const int iix = ix + (dir == 1), iiy = iy + (dir == 2), iiz = iz + (dir == 3);
  const double f_it = H.f1[c], f_iit = dir == 0 ? H.f2[c] : H.f1[cc];
  const double fv = H.fv;
  const double weight = (f_it - fv) / (f_it - f_iit);
  const double sign_ = f_it - f_iit >= 0. ? 1.0 : -1.0;
  const double xc = H.x1 + ((double)ix - 0.5) * H.dx, xcc = H.x1 + ((double)iix - 0.5) * H.dx;
  const double yc = H.y1 + ((double)iy - 0.5) * H.dy, ycc = H.y1 + ((double)iiy - 0.5) * H.dy;
  const double zc = H.z1 + ((double)iz - 0.5) * H.dz, zcc = H.z1 + ((double)iiz - 0.5) * H.dz;
  const double tt = dir == 0 ? H.t2 : H.t1;
  rec[0] = H.t1 + weight * (tt - H.t1);
  rec[1] = xc + weight * (xcc - xc);
  rec[2] = yc + weight * (ycc - yc);
  rec[3] = zc + weight * (zcc - zc);
  const double* far = dir == 0 ? H.prim : H.back;
  for (int k = 0; k < nv; k++) {
    double a = H.back[(size_t)k * H.ncell + c];
    rec[4 + k] = a + weight * (far[(size_t)k * H.ncell + cc] - a);
  }
  double betasq = rec[4 + KVX] * rec[4 + KVX] + rec[4 + KVY] * rec[4 + KVY] + rec[4 + KVZ] * rec[4 + KVZ] * H.g3;
  const double dt = fabs(H.t2 - H.t1);
  const double dx = H.dx, dy = H.dy, dz = H.dzv;
  rec[4 + nv] = sign_ * ((double)(dir == 0) * dx * dy * dz * rec[0]);
  rec[5 + nv] = sign_ * ((double)(dir == 1) * dt * dy * dz * rec[0]);
  rec[6 + nv] = sign_ * ((double)(dir == 2) * dx * dt * dz * rec[0]);
  rec[7 + nv] = sign_ * ((double)(dir == 3) * dx * dy * dt * rec[0]);
  return betasq > 1.0;  // the reference stops there (hypersurface.f90:391-395)
}

__global__ void hyp_write_kernel(HypDev H, const int* __restrict__ off, const int* __restrict__ boff,
                                 double* __restrict__ out, int* err) {
  const size_t r = (size_t)blockIdx.x * SCAN_T + threadIdx.x;
  if (r >= H.ncell) return;
  int ix, iy, iz;
  size_t c;
  unsigned m = hyp_flags(H, r, ix, iy, iz, c);
  if (!m) return;
  size_t slot = (size_t)off[r] + (size_t)boff[blockIdx.x];
  const int rl = 8 + H.nv;
  for (int d = 0; d < 4; d++)
    if (m & (1u << d)) {
      if (hyp_element(H, d, ix, iy, iz, c, out + slot * rl)) atomicMin(err, 1);
      slot++;
    }
}

}  // namespace

struct EchoHyp {
  int type;
  double value;
  int first;
  int hs;  // slice 2 is buffer hs
  double t[2];
  double* f[2];
  double* prim[2];
  int *off, *bsum, *total, *err;
  double* out;
  size_t cap;  // records out can hold
  int n;
};

extern "C" {

int echo_gpu_hyp_init(EchoCtx* c, int freeze_type, double freeze_value) {
  (void)cudaGetLastError();
  if (!c || (freeze_type != 0 && freeze_type != 1)) return ECHO_ERR_ARG;
  EchoHyp* h = c->hyp;
  if (!h) {
    h = new EchoHyp();
    size_t nc = c->g.ncell, nb = (nc + SCAN_T - 1) / SCAN_T;
    for (int i = 0; i < 2; i++) {
      CK(cudaMalloc(&h->f[i], sizeof(double) * nc));
      CK(cudaMalloc(&h->prim[i], sizeof(double) * nc * c->nv));
    }
    CK(cudaMalloc(&h->off, sizeof(int) * nc));
    CK(cudaMalloc(&h->bsum, sizeof(int) * (nb > 0 ? nb : 1)));
    CK(cudaMalloc(&h->total, sizeof(int) * 2));
    h->err = h->total + 1;
    h->out = nullptr;
    h->cap = 0;
    c->hyp = h;
  }
  h->type = freeze_type;
  h->value = freeze_value;
  h->first = 1;
  h->hs = 0;
  h->t[0] = h->t[1] = 0.;
  h->n = 0;
  return ECHO_OK;
}

int echo_gpu_hyp_step(EchoCtx* c, int* n_elements, int* errcode) {
  (void)cudaGetLastError();
  if (!c || !c->hyp) return ECHO_ERR_ARG;
  EchoHyp* h = c->hyp;
  const size_t nc = c->g.ncell;
  const unsigned nb = (unsigned)((nc + SCAN_T - 1) / SCAN_T);
  if (n_elements) *n_elements = 0;
  if (errcode) *errcode = 0;
  // t of the call (out.f90:1590,1640)
  DevScalars s;
  CK(cudaMemcpyAsync(&s, c->d_sc, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int init_err = 1 << 30;
  CK(cudaMemcpyAsync(h->err, &init_err, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  h->hs = 1 - h->hs;
  hyp_field_kernel<<<nb > 4096 ? 4096 : nb, SCAN_T, 0, c->stream>>>(c->P, c->d_v[c->vcur], nc, h->type, h->f[h->hs],
                                                                     h->prim[h->hs], c->nv, h->err);
  CK(cudaGetLastError());
  int err = 0;
  CK(cudaMemcpyAsync(&err, h->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (err != init_err) {  // get_derived_data failed: out_hyp sets run_crashed
    if (errcode) *errcode = err;
    return ECHO_OK;
  }
  if (h->first) {
    h->first = 0;
    h->t[1] = s.t;
    h->n = 0;
    return ECHO_OK;
  }
  h->t[0] = h->t[1];
  h->t[1] = s.t;
  HypDev H;
  H.f1 = h->f[1 - h->hs];
  H.f2 = h->f[h->hs];
  H.back = h->prim[1 - h->hs];
  H.prim = h->prim[h->hs];
  H.nx = c->g.nx;
  H.ny = c->g.ny;
  H.nz = c->g.nz;
  H.nv = c->nv;
  H.ncell = nc;
  H.x1 = c->p.x1;
  H.y1 = c->p.y1;
  H.z1 = c->p.z1;
  H.dx = (c->p.x2 - c->p.x1) / c->g.nx;
  H.dy = (c->p.y2 - c->p.y1) / c->g.ny;
  H.dz = (c->p.z2 - c->p.z1) / c->g.nz;
  H.dzv = c->g.nz > 1 ? H.dz : 1.0;  // d_val(3), common.f90:474-478
  H.t1 = h->t[0];
  H.t2 = h->t[1];
  H.g3 = c->p.coordinates == ECHO_BJORKEN ? h->t[1] * h->t[1] : 1.;
  H.fv = h->value;
  hyp_count_kernel<<<nb, SCAN_T, 0, c->stream>>>(H, h->off, h->bsum);
  hyp_scan_sums_kernel<<<1, SCAN_T, 0, c->stream>>>(h->bsum, (int)nb, h->total);
  CK(cudaGetLastError());
  int total = 0;
  CK(cudaMemcpyAsync(&total, h->total, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const size_t rl = 8 + (size_t)c->nv;
  if ((size_t)total > h->cap) {  // grow the output (set-up work, not per step in a steady run)
    cudaFree(h->out);
    h->cap = (size_t)total + total / 2 + 1024;
    CK(cudaMalloc(&h->out, sizeof(double) * rl * h->cap));
  }
  if (total > 0) {
    hyp_write_kernel<<<nb, SCAN_T, 0, c->stream>>>(H, h->off, h->bsum, h->out, h->err);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&err, h->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (err != init_err && errcode) *errcode = err;
  }
  h->n = total;
  if (n_elements) *n_elements = total;
  return ECHO_OK;
}

int echo_gpu_hyp_get(EchoCtx* c, double* out) {
  if (!c || !c->hyp || !out) return ECHO_ERR_ARG;
  EchoHyp* h = c->hyp;
  if (h->n > 0)
    CK(cudaMemcpyAsync(out, h->out, sizeof(double) * (8 + (size_t)c->nv) * h->n, cudaMemcpyDeviceToHost,
                       c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ECHO_OK;
}

}  // extern "C"

void echo_hyp_free(EchoHyp* h) {
  if (!h) return;
  for (int i = 0; i < 2; i++) {
    cudaFree(h->f[i]);
    cudaFree(h->prim[i]);
  }
  cudaFree(h->off);
  cudaFree(h->bsum);
  cudaFree(h->total);
  cudaFree(h->out);
  delete h;
}
