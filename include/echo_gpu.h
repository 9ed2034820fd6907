/*
 * echo_gpu.h -- C-ABI of the B200 (sm_100a) implementation of ECHO-QGP's
 * per-time-step right-hand side and update.
 *
 * The reference keeps all state in Fortran module globals and exposes the
 * step through argument-less module procedures (evolve.f90, work.f90).  This
 * library owns the same state on the device and exposes one entry point per
 * reference procedure.  Every array crosses the boundary in the reference's
 * own Fortran column-major order, v(ix,iy,iz,k) with x fastest and the
 * variable index k slowest, so a Fortran caller passes its arrays unchanged.
 *
 * Conventions
 *   - every function returns an int status: 0 = ok, ECHO_ERR_* < 0 for
 *     API/CUDA errors.  Physics failures (superluminal states, EoS table
 *     range, con2prim failure) are reported through the `errcode`
 *     out-argument with the reference's own codes (333, 777, 107, 121-138).
 *   - one host thread per context; contexts are independent.
 *   - no entry point allocates device memory after echo_gpu_init, except
 *     the batch and MLP set-up calls, which say so.
 *
 * Variable indices (0-based; reference common.f90:63 uses 1-based):
 *   0 rho  1 v^x  2 v^y  3 v^eta  4 p
 *   viscous: 5 Pi  6 pi^xy  7 pi^xeta  8 pi^yeta  9 pi^xx  10 pi^yy  11 pi^etaeta
 *   ideal MHD: 5 B^x  6 B^y  7 B^eta  [8 psi_GLM when divergence cleaning]
 */
#ifndef ECHO_GPU_H
#define ECHO_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ECHO_MAX_NV 16

/* reconstruction algorithms (REC_ALGO, common.f90:595, work.f90:429-523) */
enum {
  ECHO_REC_TVD2 = 0,
  ECHO_REC_CENO3 = 1,
  ECHO_REC_WENO3 = 2,
  ECHO_REC_WENO5 = 3,
  ECHO_REC_PPM4 = 4,
  ECHO_REC_MPE3 = 5,
  ECHO_REC_MPE5 = 6
};

/* time integrators (INT_ALGO, common.f90:186) */
enum { ECHO_RK2 = 2, ECHO_RK3 = 3, ECHO_SSP = 4 };

/* coordinates (COORD, common.f90:83) */
enum { ECHO_MINKOWSKI = 1, ECHO_BJORKEN = 2 };

/* equations of state (EOS, eos.f90:158-188) */
enum { ECHO_EOS_CONFORMAL = 1, ECHO_EOS_IDEALGAS = 2, ECHO_EOS_TABLE = 3 };

/* con2prim solvers (ALG_SOLV, common.f90:289).  Ideal MHD as below.  The
 * viscous inversion (system.f90:564-666) runs the reference's nested loop,
 * which ends after one outer pass, under 1..6, and iterates it to its fixed
 * point (max |dv| <= 1e-14) under ECHO_C2P_NEWTON and ECHO_C2P_MLP.  The
 * resistive inversion (MHD = 2) is its own fixed point under every value;
 * ECHO_C2P_MLP seeds it. */
enum {
  ECHO_C2P_BRENT = 1,   /* reference default: BRENTM on (v^2, w*gamma^2, p);
                           2..6 are the reference's other ideal-MHD solvers
                           (system.f90:732-1158), single grid only */
  ECHO_C2P_NEWTON = 100, /* this library: analytic-Jacobian Newton from the
                            previous primitives, same root; BRENTM fallback */
  ECHO_C2P_MLP = 101     /* Newton from the learned seed (<= 3 steps), then the
                            ECHO_C2P_NEWTON path if it has not converged */
};

/* status codes */
enum {
  ECHO_OK = 0,
  ECHO_ERR_ARG = -1,
  ECHO_ERR_CUDA = -2,
  ECHO_ERR_UNSUPPORTED = -3,
  ECHO_ERR_TIMEOUT = -4,
  ECHO_ERR_NOCTX = -5
};

/* Run-time parameters of the path; the names follow param.dat keys. */
typedef struct EchoParams {
  int nx, ny, nz;                 /* NX NY NZ */
  double x1, x2, y1, y2, z1, z2;  /* XMIN..ZMAX (common_grid, common.f90:441) */
  int coordinates;                /* COORD */
  int mhd;                        /* MHD: 0, 1 ideal, 2 resistive (ECHO_SSP only) */
  int divclean;                   /* DIVCLEAN */
  int viscosity;                  /* VISCOUS */
  int bulkvis;                    /* BULK */
  int recal;                      /* REC_ALGO, ECHO_REC_* */
  int nrk;                        /* INT_ALGO, ECHO_RK2/RK3/SSP */
  int eqstate;                    /* EOS, ECHO_EOS_* */
  int algo_solver;                /* ALG_SOLV, ECHO_C2P_* */
  int obtained_zz;                /* TRACE_IMP: 1 = 'zz', 0 = 'no' */
  int init_type;                  /* INIT_TYPE (2 and 5 change eta, tau_pi) */
  int enable_smooth_viscosity;    /* CUT_TEMP > 0 (common.f90:1849) */
  int ibc[ECHO_MAX_NV][2][3];     /* boundary code per variable, side, dir */
  double cfl;                     /* CFL */
  double maxdt;                   /* MAXDT */
  double maxspeed;                /* MAXSPEED */
  double glm_alpha;               /* GLM_PARAM */
  double eta_over_s;              /* ETA_S */
  double tau_pi_coeff;            /* TAU_PI_C */
  double smooth_pressure;         /* p(T=CUT_TEMP), computed by the host */
  double enezero;                 /* ENEZERO */
  double przero;                  /* p(ENEZERO) (eos.f90:131) */
  double c2p_tol;                 /* Newton residual target (ECHO_C2P_NEWTON) */
  int imex;                       /* this library (no param.dat key): 1 = viscous
                                     runs treat the Israel-Stewart relaxation
                                     linearly implicitly in every RK2/RK3 stage
                                     (the "IMEX RK2" of the batched workload);
                                     0 = explicit, as the reference */
  double sigma_el;                /* EL_COND: electrical conductivity, used in
                                     code units as read (system.f90:1660);
                                     resistive runs (mhd = 2) only */
  double sigma_chiral;            /* CHIR_COND: chiral conductivity (idem) */
} EchoParams;

typedef struct EchoCtx EchoCtx;

/* Per-step diagnostics, counted on the device. */
typedef struct EchoStats {
  double dt;            /* last time step */
  double t;             /* current time */
  double glm_ch;        /* GLM wave speed of the last stage */
  long long c2p_iters;  /* sum of con2prim iterations over cells, last stage */
  long long c2p_cells;  /* cells inverted in the last stage */
  long long repairs;    /* cells that went through the neighbour-average repair */
  long long seed_fallbacks; /* learned seeds that missed (the warm-start solve took over), so far */
  int errcode;          /* first reference error code, 0 if none */
  int err_cell;         /* linear Fortran index of the first failing cell */
  long long bracket_fallbacks; /* Newton solves that fell back to the bracketed BRENTM, so far */
} EchoStats;

/* ---- context ----------------------------------------------------------- */

/* Replaces evolve_alloc (evolve.f90:49-79), work_alloc (work.f90:49-63) and
 * the EoS table load (eos.f90:265-334).  eos_table is n_eos rows of
 * (T, e, p, c_s^2) in GeV and GeV/fm^3, already converted as
 * read_data_from_tabulated_file does; NULL for analytic EoS. */
int echo_gpu_init(const EchoParams* p, const double* eos_table, int n_eos,
                  EchoCtx** out);
int echo_gpu_free(EchoCtx* ctx);
int echo_gpu_nv(const EchoCtx* ctx);

/* State transfer.  v and u are nx*ny*nz*nv doubles, Fortran order.  u may be
 * NULL: the device then runs system_prim2cons (system.f90:164-263).
 * upload also resets the step bookkeeping (echo.f90:141-144: timeold=t,
 * timeinterval=0, vold=0). */
int echo_gpu_upload(EchoCtx* ctx, const double* v, const double* u, double t);
int echo_gpu_download(EchoCtx* ctx, double* v, double* u);
/* Same, with device pointers (no host round trip). */
int echo_gpu_upload_device(EchoCtx* ctx, const double* d_v, const double* d_u,
                           double t);
int echo_gpu_download_device(EchoCtx* ctx, double* d_v, double* d_u);

/* Asynchronous state transfer on the context's stream that keeps the run's
 * bookkeeping (time, dt, GLM speed, vold): what a host driver that owns the
 * arrays between steps calls around each echo_gpu_run.  Host buffers should
 * be page-locked for the copies to overlap nothing else on the stream. */
int echo_gpu_put_state(EchoCtx* ctx, const double* v, const double* u);
int echo_gpu_get_state(EchoCtx* ctx, double* v, double* u);

/* tout of the driver loop (echo.f90:172,243-250); evolve_main clips dt to it */
int echo_gpu_set_tout(EchoCtx* ctx, double tout);

/* ---- the step ------------------------------------------------------------ */

/* evolve_main(irk, dt) (evolve.f90:114-298): one RK/IMEX stage.  dt is
 * computed on irk == 1 and reused afterwards, as in the reference.  On
 * return *errcode is the reference error code (0 = ok) and run_crashed is
 * (*errcode != 0).  Synchronises the stream. */
int echo_gpu_evolve_main(EchoCtx* ctx, int irk, double* dt, int* errcode);

/* The driver's end of step (echo.f90:211-241): timeold=t; t=t+dt;
 * system_metric(); timeinterval=dt; vold=vnewstep.  Asynchronous. */
int echo_gpu_end_step(EchoCtx* ctx);

/* One full time step = snapshot vnewstep + nrk stages + end_step. */
int echo_gpu_step(EchoCtx* ctx, double* dt, int* errcode);

/* nsteps full steps enqueued without host synchronisation (one CUDA graph
 * per step after the first).  Check errors with echo_gpu_stats. */
int echo_gpu_run(EchoCtx* ctx, int nsteps);

/* No counterpart in the reference (the call of a host that owns the state
 * between steps): echo_gpu_put_state(v_in, u_in), echo_gpu_run(nsteps),
 * echo_gpu_get_state(v_out, u_out) in one call, with the same results.  The
 * copy of u runs on a second stream beside the first stage's flux sweeps,
 * which read v only; the first update waits for it.  v_out and u_out may be
 * v_in and u_in, or NULL (not copied).  Asynchronous like
 * echo_gpu_get_state: synchronise before reading the outputs.  Host buffers
 * should be page-locked. */
int echo_gpu_advance_host(EchoCtx* ctx, const double* v_in, const double* u_in, double* v_out,
                          double* u_out, int nsteps);

int echo_gpu_stats(EchoCtx* ctx, EchoStats* st);
int echo_gpu_sync(EchoCtx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events against the library's launches. */
int echo_gpu_stream(EchoCtx* ctx, void** stream);

/* check_temp (out.f90:1487-1557), the stop criterion the driver evaluates at
 * the top of every step when TEMP_END > 0 (echo.f90:189-190): the maximum
 * over the current primitives of the temperature (freeze_type 0) or the
 * energy density (freeze_type 1) that get_derived_temp_for_check
 * (eos.f90:706-759) gives from rho and p, reduced on the device; *stop =
 * (max < temp_end), the reference's temp_check.  Cells outside the table do
 * not count.  Synchronises the stream. */
int echo_gpu_check_temp(EchoCtx* ctx, int freeze_type, double temp_end,
                        double* max_value, int* stop);

/* Output staging in the reference's binary layout (out_vars, out.f90:232-591):
 * the contents of one outNNNN.dat -- t, then every selected field over the
 * whole grid in Fortran order (x fastest), in the reference's field order,
 * in double (precision 8) or single (4) precision -- assembled on the device
 * and copied once into host memory; the caller writes the bytes to the file.
 * Derived fields (energy density, temperature, entropy density: the
 * get_derived_data of eos.f90:645-701; pi^{tmu} from get_derived_pi(_zz),
 * viscous.f90:236-279; the Lorentz factor v0; the ideal E = -v x B,
 * contravariant, for ideal MHD) are computed from the current primitives
 * at the current t.  Viscous fields are written only for viscous runs, B
 * and E only for MHD runs, psi only with divclean, as in the reference; the
 * comoving charge density (out_sel%rc) is not offered.  pi^{eta eta}: the
 * derived value for TRACE_IMP 'zz', else the primitive (the reference writes
 * an array it fills only when one of pi^{t mu} is selected).  `sel` is a
 * mask of ECHO_OUT_* bits (the out_sel flags, common.f90:122-151; their
 * defaults, common.f90:724-805, are ECHO_OUT_DEFAULT).  out_vars_size gives
 * the bytes; out_vars fills `buf` (that many bytes) and sets *errcode to the
 * reference code of the first cell, in Fortran loop order, whose derived
 * data fall outside the EoS table (0: none).  Synchronises the stream. */
enum {
  ECHO_OUT_DENSITY = 1 << 0, ECHO_OUT_VX = 1 << 1, ECHO_OUT_VY = 1 << 2, ECHO_OUT_VZ = 1 << 3,
  ECHO_OUT_PRESSURE = 1 << 4, ECHO_OUT_ENERGY_DENSITY = 1 << 5, ECHO_OUT_TEMPERATURE = 1 << 6,
  ECHO_OUT_ENTROPY_DENSITY = 1 << 7, ECHO_OUT_BULK = 1 << 8, ECHO_OUT_PITT = 1 << 9,
  ECHO_OUT_PITX = 1 << 10, ECHO_OUT_PITY = 1 << 11, ECHO_OUT_PITZ = 1 << 12, ECHO_OUT_PIXY = 1 << 13,
  ECHO_OUT_PIXZ = 1 << 14, ECHO_OUT_PIYZ = 1 << 15, ECHO_OUT_PIXX = 1 << 16, ECHO_OUT_PIYY = 1 << 17,
  ECHO_OUT_PIZZ = 1 << 18, ECHO_OUT_V0 = 1 << 19, ECHO_OUT_BX = 1 << 20, ECHO_OUT_BY = 1 << 21,
  ECHO_OUT_BZ = 1 << 22, ECHO_OUT_EX = 1 << 23, ECHO_OUT_EY = 1 << 24, ECHO_OUT_EZ = 1 << 25,
  ECHO_OUT_GLM = 1 << 26
};
#define ECHO_OUT_DEFAULT                                                                                  \
  (ECHO_OUT_DENSITY | ECHO_OUT_VX | ECHO_OUT_VY | ECHO_OUT_VZ | ECHO_OUT_PRESSURE | ECHO_OUT_ENERGY_DENSITY | \
   ECHO_OUT_BX | ECHO_OUT_BY | ECHO_OUT_BZ | ECHO_OUT_EX | ECHO_OUT_EY | ECHO_OUT_EZ)
int echo_gpu_out_vars_size(const EchoCtx* ctx, unsigned sel, int precision, size_t* bytes);
int echo_gpu_out_vars(EchoCtx* ctx, unsigned sel, int precision, void* buf, size_t bytes, int* errcode);

/* Optical Glauber initial state on the device (init.f90:852-1242, the
 * reference's GLAUBER_GEOMETRIC initial conditions; glaubermc.f90 is the
 * Monte Carlo mode, echo_batch_glauber).  The nucleus' Woods-Saxon
 * thickness is integrated by the reference's own rule (thickness,
 * init.f90:1164-1219: radii r = (nc-1) dr out to the grid's reach plus the
 * impact parameter, |z| <= 2 radius, dz halved from 2 dz1 until the two
 * end-point sums agree to acc), the numbers of binary collisions and wounded
 * nucleons at each cell centre use the nearest radius nint(r/dr + 1) (bincoll,
 * wound, init.f90:971-1032), normalised by those of a b = 0 collision at the
 * origin (init.f90:1805-1812), and calc_enedens (init.f90:902-929, no
 * tilting; with nz > 1 times the plateau-plus-Gaussian H(eta) around the
 * local eta0 of the two thicknesses) gives e; initio (init.f90:852-893)
 * then sets rho = rhocenter, v = 0 and p = p(e) + przero, and the state is
 * uploaded as by echo_gpu_upload(v, NULL, t).  *check_mass = the
 * reference's printed "check nucleus mass" (sum over the table of
 * r T(r) dr times 2 x 3.1415927); *max_e = the largest e of the grid (with
 * ecenter = 1 it is the factor a caller divides a target peak by).
 * Allocates the thickness table (8 bytes per 0.001 fm of reach) on the
 * first call; synchronises.  Returns ECHO_ERR_ARG (nothing uploaded) when
 * the table does not converge within 8 halvings of dz. */
typedef struct EchoOpticalGlauber {
  double mass_number;   /* projmass (nuclear_data.dat) */
  double radius, delta; /* Woods-Saxon radius and width (fm) */
  double roze;          /* normal nuclear density (fm^-3) */
  double sigma_in;      /* inelastic NN cross section in fm^2 (SIGMA_IN/10, common.f90:2259) */
  double ah;            /* hardness: weight of binary collisions (AH) */
  double bimpact;       /* impact parameter (fm) */
  double ecenter;       /* e at the centre of a b = 0 collision (GeV/fm^3) */
  double rhocenter;     /* the density primitive */
  double dr, dz1, acc;  /* thickness table step, first z step, integration accuracy */
  double deta, sigeta;  /* 3+1D: plateau width and Gaussian width of H(eta) */
  double sqrt_s, nucleon_mass; /* gamma_col = sqrt_s / (2 m) (common.f90:2261) for eta0 */
} EchoOpticalGlauber;
int echo_gpu_optical_glauber(EchoCtx* ctx, const EchoOpticalGlauber* g, double t, double* check_mass,
                             double* max_e);

/* Checkpoint / restart of a run at a step boundary (the role of out_dump and
 * out_restart, out.f90:1313-1483, which the reference turns off for MHD and
 * Monte Carlo runs; here every equation set).  The blob (checkpoint_size
 * bytes, host memory) holds the current v and u, vold and every run scalar
 * (t, dt, timeold, timeinterval, tout, GLM speed, ...); a context of the same
 * shape restarted from it continues bit for bit as the original would have.
 * Both synchronise the stream; restart rejects a blob of another shape with
 * ECHO_ERR_ARG. */
int echo_gpu_checkpoint_size(const EchoCtx* ctx, size_t* bytes);
int echo_gpu_checkpoint(EchoCtx* ctx, void* blob);
int echo_gpu_restart(EchoCtx* ctx, const void* blob);

/* dump.dat in the reference's layout (out_dump / out_restart,
 * out.f90:1313-1483, with out_freeze off): stream access, no record
 * markers -- iout (int32), t, timeold, timeinterval (double), vall and uall
 * (nv fields each, Fortran order), vallold and uallold (the fields krh..
 * kvold_end: 5, or 8 with MHD, common.f90:378-386), g_cov_3_old.
 * dump_size gives the bytes; dump fills `buf` with exactly that many (the
 * caller writes them to outrNNNN/dump.dat); restart_dump reads such a file
 * of a run of the same shape into the context at a step boundary and
 * returns its iout, as out_restart does (t, timeold, timeinterval,
 * g_cov_3_old, v, u, vold; dt and the GLM speed start as after an upload, as
 * the reference's restart leaves them).  vold / uold are the reference's
 * step-start copies of the previous step (echo.f90:192-202, 240-241); the
 * device keeps them only after echo_gpu_keep_old(ctx, 1) (two more copies
 * of kvold_end fields per step; set at upload as init() does, init.f90:
 * 3271-3272).  Without it the dump holds the viscous vold's rho and
 * velocities (the only part the evolution reads, dts in viscous.f90:56-97)
 * and zeros elsewhere.  All three synchronise the stream. */
int echo_gpu_keep_old(EchoCtx* ctx, int on);
int echo_gpu_dump_size(const EchoCtx* ctx, size_t* bytes);
int echo_gpu_dump(EchoCtx* ctx, int iout, void* buf, size_t bytes);
int echo_gpu_restart_dump(EchoCtx* ctx, const void* buf, size_t bytes, int* iout);

/* Freeze-out hypersurface (out_hyp, out.f90:1569-1650, with
 * find_hypersurface_ideal/_visco/_mhd and set_fo_ide/_vis,
 * hypersurface.f90:172-460, 775-1117), on the device.  hyp_init sets the
 * freeze criterion -- temperature (freeze_type 0) or energy density (1) equal
 * to freeze_value -- and allocates the two time slices.  Each hyp_step is one
 * out_hyp call at the current t: the field of the current primitives
 * becomes the new slice; from the second call on, the surface elements
 * between the two slices are collected, in the reference's order (ix outer,
 * eta inner; per cell tau, x, y, eta).  Every element is 8 + nv doubles:
 * tau, x, y, eta; the nv primitives interpolated to the crossing; dV_tau,
 * dV_x, dV_y, dV_eta times the crossing's sign (hy_ide's columns, then
 * hy_vis's for viscous runs).  *errcode: a get_derived_data code (the
 * reference crashes the run) or 1 for a superluminal element (the reference
 * exits).  hyp_step synchronises and may grow its output buffer; hyp_get
 * copies the last call's n_elements records to the host. */
int echo_gpu_hyp_init(EchoCtx* ctx, int freeze_type, double freeze_value);
int echo_gpu_hyp_step(EchoCtx* ctx, int* n_elements, int* errcode);
int echo_gpu_hyp_get(EchoCtx* ctx, double* out);

/* Runs one full step with a CUDA event after every launch group and returns
 * the device time per kernel class (ms[8]: faces x, faces y, faces z, stage
 * scalars, update+con2prim, repair(+smoothing), end of step, fused stage)
 * and the number of launches of each class.  The step is a real step of the
 * run. */
int echo_gpu_profile_step(EchoCtx* ctx, double* ms, int* launches);

/* No counterpart in the reference (an execution option).  How the product
 * build (libechogpu.so) computes the WENO5 face sweeps:
 *   mode 0   one thread per face, both face states in one thread (the
 *            default; the reference's arrangement, which the parity build
 *            always runs);
 *   mode 8, 16  one thread per cell, in segments of that many cells along
 *            the sweep: a thread reconstructs both face states of its cell
 *            from one set of WENO5 smoothness indicators and takes the
 *            state of the cell below from its neighbouring lane, so a
 *            segment yields mode - 1 faces.
 * All meet the oracle at the product build's tolerance.  Other
 * reconstructions always run mode 0.  ECHO_ERR_ARG for other modes.
 * Synchronises the stream and drops the step graphs. */
int echo_gpu_set_faces(EchoCtx* ctx, int mode);

/* No counterpart in the reference (an execution option).  concurrent = 1
 * (the default) runs the x, y and eta flux sweeps of a stage side by side
 * on three streams, joined before the update; 0 runs them one after
 * another.  The sweeps are independent, so both give the same bits.
 * Synchronises the stream and drops the step graphs. */
int echo_gpu_set_sweeps(EchoCtx* ctx, int concurrent);

/* No counterpart in the reference (an execution option).  How a stage runs:
 * fused = 1 (where the run allows it) runs the three sweeps,
 * the flux divergence, the sources, the update and con2prim of a stage in
 * one kernel over x-y tiles of tx x ty cells marching through eta segments
 * of zseg planes, with no face flux in global memory; fused = 0 runs the
 * sweep kernels and the update kernel (the default: the sweeps are faster
 * on the benchmarked grids).  The first stage of an explicit RK
 * step without divergence cleaning always runs the sweeps (its dt needs
 * every face's signal speed before any update).  tx, ty, zseg = 0 choose
 * the tile and segment for this grid.  Both give the same results within
 * the parity tolerance.  info (may be NULL) receives 7 ints: fused, tx, ty,
 * zseg, threads per CTA, CTAs, shared-memory bytes per CTA.  Returns
 * ECHO_ERR_UNSUPPORTED (and runs the sweeps) where the run cannot fuse:
 * reconstruction other than WENO5, nx or ny below 3, ALG_SOLV 2-6.
 * Synchronises the stream and drops the cached step graphs. */
int echo_gpu_set_stage(EchoCtx* ctx, int fused, int tx, int ty, int zseg, int* info);

/* ---- pieces of the step, for parity tests against the oracle ----------- */

/* evolve_dfx/dfy/dfz + evolve_src of one stage (evolve.f90:302-718) into
 * du (nx*ny*nz*nv, Fortran order, host memory), with ax/ay/az maxima. */
int echo_gpu_rhs(EchoCtx* ctx, double* du, double* amax3);

/* No counterpart in the reference (measurement).  The FP64 peak of the
 * current GPU: independent DFMA chains on every SM, best of five timed
 * launches; *gflops = FP64 GFLOP/s (a DFMA counts 2), *ms = that launch's
 * time.  The denominator of the FP64 roofline the step kernels report.
 * Allocates 8 bytes and synchronises the device. */
int echo_gpu_fp64_peak(double* gflops, double* ms);

/* No counterpart in the reference (a check of the kernels' index
 * arithmetic): q[i*nn + j] = n[j] / d[i] (unsigned, d[i] >= 1) computed on
 * the device with the multiply-high division the face and cell kernels use
 * to split flat indices into grid coordinates. */
int echo_gpu_test_fastdiv(const unsigned* d, int nd, const unsigned* n, int nn, unsigned* q);

/* Reconstruction of m pencils of length n (+ghosts) with REC_ALGO.
 * f is m rows of (n + 8) values, f[row*(n+8) + (i+4)] = f(i), i=-4..n+3;
 * gl/gr are m rows of n+1 faces (holib.f90:47-348). */
int echo_gpu_test_recon(int recal, int m, int n, const double* f, double* gl,
                        double* gr);

/* system_cons2prim on ncells independent cells (system.f90:423-1166).
 * u and v are ncells*nv, cell-major (u[c*nv+k]); v holds the initial guess
 * on input and the result on output; err gets the per-cell code and iters
 * the per-cell iteration count (may be NULL).  g3 = g_cov(3), gp = sqrt(-g). */
int echo_gpu_test_c2p(const EchoParams* p, const double* eos_table, int n_eos,
                      int ncells, double g3, double gp, const double* u,
                      double* v, int* err, int* iters);

/* system_cons2prim of independent ideal-RMHD cells (u, v cell-major as in
 * echo_gpu_test_c2p) at the residual p->c2p_tol: from the learned seed when
 * weights != NULL (falling back to Newton from v, then BRENTM), else Newton
 * from the guess in v.  seed_failed[c] = 1 where the seed did not converge
 * within 3 Newton steps. */
int echo_gpu_test_c2p_seeded(const EchoParams* p, const double* eos_table,
                             int n_eos, int ncells, double g3, double gp,
                             const float* weights, const float* norm,
                             const double* u, double* v, int* err, int* iters,
                             int* seed_failed);

/* ---- learned con2prim seed (ECHO_C2P_MLP) -------------------------------- */

/* The seed network is a 4x64 tanh MLP from six invariants of the conserved
 * state (log U, D/U, S^2/U^2, B^2/U, (S.B)^2/U^3, E^2/U; E = 0 for ideal
 * RMHD) to (v^2, p/U).  Weight vector: per layer W[K][N] row-major then b[N],
 * (K,N) = (6,64), (64,64) x3, (64,2).  norm: feature mean[6], std[6], target
 * mean[2], std[2]. */
#define ECHO_MLP_NIN 6
#define ECHO_MLP_NWEIGHTS 13058
#define ECHO_MLP_NNORM 16

/* Trains the network with this library's own FP32 forward/backward kernels
 * and Adam on n raw (invariants X[n][6], targets T[n][2]) pairs.  A set-up
 * call: allocates device memory for the data and the optimiser.  loss_out
 * receives one value every report_every steps (may be NULL). */
int echo_gpu_mlp_train(const float* X, const float* T, int n, int steps,
                       int batch, float lr, unsigned seed, float* weights_out,
                       float* norm_out, float* loss_out, int report_every);

/* Mean-squared loss and its gradient w.r.t. the weight vector on n
 * standardised rows (gradient check against the CPU oracle). */
int echo_gpu_mlp_grad(const float* weights, const float* Xs, const float* Ts,
                      int n, float* loss, float* grad);

/* Loads a trained network into a context (BF16 tensor-core fragments);
 * required before stepping with algo_solver = ECHO_C2P_MLP.  Allocates. */
int echo_gpu_mlp_set(EchoCtx* ctx, const float* weights, const float* norm);

/* Tensor-core inference on n raw invariant rows -> out[n][2] = (v^2, p/U). */
int echo_gpu_mlp_infer(const float* weights, const float* norm, const float* X,
                       int n, float* out);

/* ---- allocation-free stage right-hand side ------------------------------ */

/* No counterpart in the reference.  The du of one explicit stage -- what
 * echo_gpu_rhs returns right after echo_gpu_upload of d_v at time t: the
 * three flux sweeps plus the sources -- for callers that cannot allocate
 * device memory:
 * a code coupled to this library inside a GPU application whose memory
 * belongs to another allocator (a framework pool, or a solver that reserves
 * HBM up front), or a driver that must not allocate between graph captures.
 *
 * The caller passes device pointers: d_v and d_du (nx*ny*nz*nv doubles,
 * Fortran order) and, for a tabulated EoS, d_eos_cols = the four columns
 * T, e, p, c_s^2 of the table stored one after the other (4*n_eos doubles).
 * The function calls no cudaMalloc, cudaFree or allocating library routine:
 * the face fluxes go to a fixed file-scope device array of
 * ECHO_NOALLOC_SCRATCH_DOUBLES doubles (32 MiB, held by every GPU that loads
 * the library until the process exits); a grid whose faces need more,
 * nv * (faces in x + y + z) doubles (+8 per face for viscous runs), is
 * rejected with ECHO_ERR_ARG and a message.  The first call on a device
 * looks up that array's device address (cudaGetSymbolAddress) with the
 * device current; make that first call before any stream capture.  All
 * calls share the array, which keeps the last call's contents, so calls
 * that overlap on the GPU (other streams, other host threads) race.
 *
 * The call carries no run state: like a context just uploaded, it takes the
 * GLM wave speed of the face upwinding as 0.5 (common.f90:283) and the
 * viscous lagged time derivatives (dts) as zero (timeinterval = 0).  In the
 * middle of a divergence-cleaning or viscous run its du therefore differs
 * from echo_gpu_rhs on the running context; it equals echo_gpu_rhs on a
 * context that uploads the same primitives at the same t.  Resistive runs
 * (mhd = 2) return ECHO_ERR_UNSUPPORTED; every parameter check of
 * echo_gpu_init applies.
 * Launches go to `stream` (a cudaStream_t, may be NULL).  If errcode is not
 * NULL the call synchronises the stream and returns the first reference
 * error code found (0 = none); a stream being captured cannot be
 * synchronised, so with errcode set on a capturing stream the call returns
 * ECHO_ERR_ARG before any launch: pass errcode = NULL there. */
#define ECHO_NOALLOC_SCRATCH_DOUBLES (4 * 1024 * 1024)
int echo_gpu_rhs_noalloc(const EchoParams* p, const double* d_eos_cols,
                         int n_eos, double t, const double* d_v, double* d_du,
                         void* stream, int* errcode);

/* ---- batched event-by-event runs ----------------------------------------- */

/* No single counterpart in the reference: a batch replaces the events loop
 * of echo.f90:113-308 (Monte Carlo Glauber mode runs its events one after
 * another, each through the whole time loop) by advancing many events at
 * once.  Every event has its own grid size and extent, its own t, dt
 * (evolve_dt per event), stop test (t >= tmax, echo.f90:187) and crash
 * state (a crashed event is abandoned, the others go on: echo.f90:206-209,
 * 283-307); the physics switches (EchoParams other than the grid fields) are
 * shared.  Per event the arithmetic is the single-grid path's.
 *
 * Arrays cross as one arena: event e's primitives v(ix,iy,iz,k) (Fortran
 * order, nv * ncell_e doubles) start at nv * cell_offset[e], where
 * cell_offset is the running sum of the events' cell counts. */
typedef struct EchoBatch EchoBatch;

typedef struct EchoEventGrid {
  int nx, ny, nz;
  double x1, x2, y1, y2, z1, z2;
} EchoEventGrid;

/* event states */
enum { ECHO_EVENT_LIVE = 0, ECHO_EVENT_DONE = 1, ECHO_EVENT_CRASHED = 2,
       ECHO_EVENT_COOLED = 3 /* stopped by check_temp (echo_batch_set_stop) */ };

typedef struct EchoEventStatus {
  double t, dt;
  long long steps;      /* completed time steps */
  int state;            /* ECHO_EVENT_* */
  int errcode;          /* reference code of the crash, 0 = none */
  int err_cell;
  int pad;
  long long c2p_iters;  /* con2prim iterations of the last stage */
  long long repairs;    /* con2prim repairs so far */
  long long seed_fallbacks; /* learned seeds that needed the warm start so far */
} EchoEventStatus;

/* launch-shape slots (echo_batch_set_schedule) */
enum { ECHO_SLOT_FACES_X = 0, ECHO_SLOT_FACES_Y = 1, ECHO_SLOT_FACES_Z = 2,
       ECHO_SLOT_UPDATE = 3, ECHO_SLOT_SMOOTH = 4, ECHO_NSLOTS = 5 };

/* Allocates the batch (RK2 or RK3; the plain con2prim solvers).  The grid
 * fields of p are ignored; grids[e] gives event e's. */
int echo_batch_init(const EchoParams* p, const double* eos_table, int n_eos,
                     int nev, const EchoEventGrid* grids, EchoBatch** out);
int echo_batch_free(EchoBatch* b);
int echo_batch_nv(const EchoBatch* b);
/* cell_offset[0..nev]: first cell of each event, [nev] = total cells */
int echo_batch_offsets(const EchoBatch* b, long long* cell_offset);
/* State of every event at time t (host arrays; u may be NULL: computed by
 * system_prim2cons); events run until t >= tmax.  Resets every event to
 * live, zero steps. */
int echo_batch_upload(EchoBatch* b, const double* v, const double* u, double t,
                      double tmax);
int echo_batch_upload_device(EchoBatch* b, const double* d_v, const double* d_u,
                             double t, double tmax);
/* Monte Carlo Glauber initial state of every event, generated on the device
 * (the energy-density part of generate_energy_density_profile,
 * glaubermc.f90:686-873): the sources of event e -- participants and
 * binary-collision points with their weights, src[3*i..3*i+2] = (x, y, w)
 * for i in [src_offset[e], src_offset[e+1]) -- are smeared by a normalised
 * 2D Gaussian of width sigma (fm) at the cell centres; per event
 * e = peak * S / max(S) + ENEZERO, p = p(e) from the EoS, rho = 1, every
 * other variable 0, u by system_prim2cons.  Then as echo_batch_upload.
 * Sampling the nucleons stays on the host.  Allocates and frees device
 * memory for the sources. */
int echo_batch_glauber(EchoBatch* b, const double* src, const long long* src_offset,
                       double sigma, double peak, double t, double tmax);
int echo_batch_download(EchoBatch* b, double* v, double* u);
/* nsteps time steps of every live event, asynchronous (one CUDA graph per
 * step); finished and crashed events drop out on the device */
int echo_batch_run(EchoBatch* b, int nsteps);
/* Loads a trained con2prim seed network (echo_gpu_mlp_train layout) into
 * the batch; required before running with algo_solver = ECHO_C2P_MLP.
 * Allocates. */
int echo_batch_mlp_set(EchoBatch* b, const float* weights, const float* norm);
/* synchronises; number of live events */
int echo_batch_live(EchoBatch* b, int* nlive);
/* synchronises; status of every event (nev entries) */
int echo_batch_status(EchoBatch* b, EchoEventStatus* st);
int echo_batch_sync(EchoBatch* b);
int echo_batch_stream(EchoBatch* b, void** stream);
/* The per-event check_temp stop criterion (echo_gpu_check_temp): before each
 * step every live event whose maximum temperature (freeze_type 0) or energy
 * density (1) is below temp_end stops (ECHO_EVENT_COOLED), after the
 * t >= tmax test, as the reference's time loop does (echo.f90:187-190).
 * temp_end <= 0 (the default) turns it off. */
int echo_batch_set_stop(EchoBatch* b, int freeze_type, double temp_end);
/* Launch shape of each slot: the number of CTAs of its persistent launch
 * (0 = one CTA per tile); order (nev entries, or NULL = 0..nev-1) is the
 * order in which the tile lists visit the events. */
int echo_batch_set_schedule(EchoBatch* b, const int* ctas, const int* order);
int echo_batch_get_schedule(const EchoBatch* b, int* ctas);
/* The autotuner: on the current state (the state and every event's scalars
 * are restored afterwards) it times, per slot, every tile length (128, 256,
 * 512 faces or cells per tile) with every launch shape (one CTA per tile,
 * or 1..occupancy CTAs per SM persistent), keeps the fastest (the cell
 * list takes the update's tile), and then times whole first stages run
 * both ways -- one launch per phase, and one cooperative launch per stage
 * with 1..occupancy CTAs per SM -- keeping the faster (echo_batch_set_mode).
 * ms[slot] = the chosen per-launch time of each slot.  Synchronises. */
int echo_batch_autotune(EchoBatch* b, int reps, double* ms);
/* Every candidate the last autotune timed, 4 doubles per row: what (slot
 * 0..4, or 5 = a whole stage), shape (the tile length; for a stage 0 =
 * phased, 1 = cooperative), CTAs (0 = one per tile), ms.  *n = rows (the
 * first `cap` are copied). */
int echo_batch_autotune_report(const EchoBatch* b, double* rows, int cap, int* n);
/* Tile lengths of the x, y, z face lists and the cell list (multiples of
 * 128, at most 1024); drops the step graphs. */
int echo_batch_set_tiles(EchoBatch* b, const int* tiles);
/* How a stage runs: mode 0 = one launch per phase (stage begin, face
 * sweeps, per-event scalars, update, repair, smoothing); mode 1 = one
 * cooperative launch per stage running those phases with grid-wide
 * barriers between them (all CTAs resident; every barrier wait is bounded
 * and a timeout ends the launch, reported by echo_batch_sync as
 * ECHO_ERR_TIMEOUT), grid CTAs (0 = the most that are resident; WENO5
 * reconstruction only).  Drops the step graphs. */
int echo_batch_set_mode(EchoBatch* b, int mode, int grid);
/* out[7]: tile lengths (x, y, z faces, cells), mode, cooperative grid
 * (0 = all resident), 1 when steps run as CUDA graphs. */
int echo_batch_get_tuning(const EchoBatch* b, int* out);
/* one step with per-phase CUDA-event timing, like echo_gpu_profile_step */
int echo_batch_profile_step(EchoBatch* b, double* ms, int* launches);

#ifdef __cplusplus
}
#endif
#endif /* ECHO_GPU_H */
