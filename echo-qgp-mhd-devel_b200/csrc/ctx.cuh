// ctx.cuh -- the device context of one run and the per-equation-set launch
// functions.  The launchers are explicitly instantiated once per equation
// set in kind_*.cu so the four instantiations compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include <utility>
#include <vector>

#include "../../include/echo_gpu.h"
#include "kernels.cuh"

using namespace echo;

struct EchoHyp;  // freeze-out hypersurface state (hyper.cu)
void echo_hyp_free(EchoHyp* h);

struct EchoCtx {
  EchoParams p;
  int kind, nv, nvold;
  Grid g;
  DevPhys P;
  BcDir bc[3];
  int bc_uniform[3], bc_signed[3];
  cudaStream_t stream;
  double* d_v[2];
  int vcur;
  double* d_u[2];
  int ucur;
  double *d_F[3], *d_WD[3];
  size_t nfaces[3];
  double* d_vh[2];          // vnewstep / vold history (first 4 components used)
  int vn;                   // d_vh[vn] = vnewstep, d_vh[1-vn] = vold
  double* d_tab;
  int* d_bk;                // EoS bracket accelerators
  double* d_du;             // scratch for echo_gpu_rhs
  double* d_dussp[4];       // IMEX-SSP stage right-hand sides du(:,:,:,:,1..4)
  double* d_dss[4];         // resistive IMEX-SSP: stiff E right-hand sides, 3 x ncell
  unsigned* d_mlp_frag;     // learned con2prim seed: BF16 weight fragments
  float* d_mlp_par;         //   biases and normalisation
  unsigned char* d_fail;
  DevScalars* d_sc;
  DevScalars* h_sc;         // pinned mirror
  cudaGraphExec_t graph[16];  // one per buffer-role key at step start
  bool graph_ok[16];
  // per-kernel timing (echo_gpu_profile_step): events recorded after each launch group
  std::vector<std::pair<int, cudaEvent_t>>* marks;
  EchoHyp* hyp;             // set up by echo_gpu_hyp_init
  void* d_out;              // output staging (echo_gpu_out_vars), grown on demand
  size_t out_bytes;
  unsigned long long* d_out_err;
  // the reference's vnewstep/unewstep -> vold/uold of components
  // krh..kvold_end (echo.f90:192-202, 240-241), kept only for dump.dat
  // (echo_gpu_keep_old): d_oldv[on] / d_oldu[on] = the step-start copies,
  // [1 - on] = vold / uold
  int keep_old, kold, on;
  double *d_oldv[2], *d_oldu[2];
  // product build: how the face sweeps run: 0 one thread per face, 8 or 16
  // the cell-centred kernel in segments of that many cells
  int face_mode;
  // concurrent sweeps: the y and eta sweeps of a stage run on two side
  // streams forked from and joined back into `stream` (par_sweeps = 1)
  int par_sweeps;
  cudaStream_t side[2];
  cudaEvent_t ev_fork, ev_join[2];
  // echo_gpu_advance_host: the host copy of u runs on copy_stream and ev_u
  // marks its end; while wait_u is set, the next step's first u access
  // waits for it (join_u)
  cudaStream_t copy_stream;
  cudaEvent_t ev_u, ev_u_fork;
  int wait_u;
  // the fused stage kernel (stage.cuh): usable, on, tile, segment, launch
  int st_ok, st_on, st_tx, st_ty, st_zseg, st_nt;
  unsigned st_grid;
  size_t st_smem;
};
void echo_out_free(EchoCtx* c);

// kernel classes reported by echo_gpu_profile_step
enum { PK_FACES_X = 0, PK_FACES_Y = 1, PK_FACES_Z = 2, PK_SCALARS = 3, PK_UPDATE = 4, PK_REPAIR = 5, PK_END = 6,
       PK_STAGE = 7, PK_N = 8 };

inline void mark(EchoCtx* c, int cls) {
  if (!c->marks) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, c->stream);
  c->marks->push_back({cls, e});
}

// shared by the single-grid and the batched contexts (echo_gpu.cu)
int echo_check_params(const EchoParams* p, const double* eos_table, int n_eos);
int echo_kind_of(const EchoParams* p);
int echo_nv_of(int kind);
void echo_setup_bc(const EchoParams* p, int nv, BcDir bc[3], int uniform[3], int sign[3]);
int echo_setup_phys(const EchoParams* p, const double* eos_table, int n_eos, DevPhys* P, double** d_tab,
                    int** d_bk);

// Bracket accelerator of tab_bracket: for every bucket of the bit pattern
// (>> BK_SHIFT) between the first and last table value, the smallest
// bracket index max(2, first i with arr(i) >= lowest value of the bucket).

namespace echo {

template <int KIND>
void launch_faces(EchoCtx* c, int dir);
template <int KIND>
void launch_update(EchoCtx* c, int irk, int mode, double* du_out);
// what: 1 = repair only, 2 = smoothing only, 3 = both
template <int KIND>
void launch_repair_smooth(EchoCtx* c, int what = 3);
template <int KIND>
void launch_p2c(EchoCtx* c);
template <int KIND>
void launch_ssp_combine(EchoCtx* c, int stage);
template <int KIND>
void launch_ssp_stage1(EchoCtx* c);
template <int KIND>
int setup_stage(EchoCtx* c, int tx, int ty, int zseg);
template <int KIND>
void launch_stage(EchoCtx* c, int irk, int mode, double* du_out);

}  // namespace echo
