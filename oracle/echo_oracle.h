/*
 * echo_oracle.h -- CPU oracle for the ECHO-QGP step path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a line-by-line C restatement of the
 * reference Fortran (evolve.f90, work.f90, holib.f90, system.f90,
 * viscous.f90, eos.f90, libacm554.f90).  It is the checker for the CUDA
 * library and the CPU baseline of the benchmark; no product code path may
 * call it.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists in
 * this environment or on the GPU hosts (probed), so the restatement cannot
 * be diffed against the reference binary ("parity unpinned" against the
 * Fortran build of the step).  It is pinned instead against the analytic
 * solutions the reference's own test problems use (Bjorken flow, Bjorken
 * MHD flow, Gubser flow), against the two values of the step's
 * neighbourhood that the reference printed in its own run log
 * (doc/images/echo-qgp-output.txt: the optical Glauber thickness check and
 * a tabulated-EoS energy, reproduced digit for digit and bit for bit,
 * tests/test_reference_pins.py), and against committed golden vectors it
 * produced (tests/golden).
 */
#ifndef ECHO_ORACLE_H
#define ECHO_ORACLE_H

#include "../include/echo_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct Orc Orc;

Orc* orc_create(const EchoParams* p, const double* eos_table, int n_eos);
void orc_free(Orc* e);
int orc_nv(const Orc* e);
/* number of OpenMP threads used by the sweeps (1 = serial restatement) */
void orc_set_threads(Orc* e, int nthreads);

/* state in Fortran order v(ix,iy,iz,k); u == NULL -> system_prim2cons */
int orc_set_state(Orc* e, const double* v, const double* u, double t);
void orc_get_state(const Orc* e, double* v, double* u);
void orc_set_tout(Orc* e, double tout, double dtout, double tmax);

/* evolve_main(irk, dt): returns errcode (0 ok) */
int orc_evolve_main(Orc* e, int irk, double* dt);
/* one loop body of echo.f90:185-262 (without output) */
int orc_step(Orc* e, double* dt);
/* du of one explicit stage (dfx+dfy+dfz+src) and the ax/ay/az maxima */
int orc_rhs(Orc* e, double* du, double* amax3);

double orc_time(const Orc* e);
double orc_dt(const Orc* e);
double orc_glm_ch(const Orc* e);
long long orc_repairs(const Orc* e);
long long orc_c2p_iters(const Orc* e);
/* check_temp (out.f90:1487-1557) over the current primitives */
double orc_check_temp(const Orc* e, int freeze_type);
/* out_vars (out.f90:232-591): the bytes of one outNNNN.dat (see
   echo_gpu_out_vars); returns the byte count, *errcode the first derived-data
   error in Fortran loop order; buf may be NULL to get the size only */
size_t orc_out_vars(const Orc* e, unsigned sel, int precision, void* buf, int* errcode);
/* freeze-out hypersurface (out_hyp / find_hypersurface_*): records of
 * 8 + nv doubles (tau, x, y, eta, primitives, dV with sign) */
int orc_hyp_init(Orc* e, int freeze_type, double freeze_value);
int orc_hyp_step(Orc* e, int* n);
void orc_hyp_get(const Orc* e, double* out);

/* kernels on their own, for unit parity tests */
void orc_recon(int recal, int m, int n, const double* f, double* gl,
               double* gr);
int orc_c2p(const EchoParams* p, const double* eos_table, int n_eos,
            int ncells, double g3, double gp, const double* u, double* v,
            int* err, int* iters);
int orc_prim2cons(const EchoParams* p, const double* eos_table, int n_eos,
                  int ncells, double g3, double gp, double* v, double* u);
/* system_flux of one state in direction dir (1..3) */
int orc_flux(const EchoParams* p, const double* eos_table, int n_eos,
             double g3, double gp, int dir, double* v, double* u, double* f,
             double* vf);

/* the learned con2prim seed network (gradient check, FP64) */
/* tabulated EoS e(p) (get_energy, eos.f90:468-523); returns the code */
int orc_eos_energy(const EchoParams* p, const double* eos_table, int n_eos, double pr, double* en);

/* optical Glauber (init.f90:852-1242): the thickness table (returns the
 * reference's printed "check nucleus mass") and the energy density of
 * calc_enedens at the cell centres */
double orc_thickness(double radius, double delta, double roze, double dr, double dz1, double acc, int nmax,
                     double* thick);
double orc_optical_glauber(const EchoOpticalGlauber* g, int nx, int ny, int nz, double x1, double x2, double y1,
                           double y2, double z1, double z2, double* e);

void orc_mlp_grad(const float* W, const float* Xs, const float* Ts, int n, double* loss, double* grad);
void orc_mlp_forward(const float* W, const float* norm, const float* X, int n, double* out);

#ifdef __cplusplus
}
#endif
#endif
