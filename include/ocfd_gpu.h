/*
 * ocfd_gpu.h -- C ABI of the B200 (sm_100a) implementation of the OpenCFD-Comb
 * per-step hot path: flux-split WENO5/WENO7/OMP6/UD7L/HYBRID inviscid flux,
 * CD6/CD8 viscous + heat flux, SSP-RK3 update, species transport and the
 * finite-rate chemistry integrators.
 *
 * The Fortran driver of the reference keeps parsing its control files and
 * keeps its output formats; it replaces the two hot call sites of its time
 * loop with the entry points below (through an iso_c_binding interface module):
 *
 *   code/flow-solver/OCFD_NS_Solver.f90:28,37  call flow_time_advance(dt1)
 *        -> ocfd_gpu_flow_advance(dt1, tt)
 *   code/flow-solver/OCFD_NS_Solver.f90:30-35  Chemical_time_advance x nsub + comput_T_P
 *        -> ocfd_gpu_chem_advance(dt2, nsub)
 *
 * Array conventions (all arrays are Fortran column-major, contiguous):
 *   "halo" arrays    : (1-LAP:nx+LAP, 1-LAP:ny+LAP, 1-LAP:nz+LAP)    H doubles
 *   "interior" arrays: (nx, ny, nz)                                   N doubles
 *   f                : f(nx,ny,nz,5)            (code/head/MODULE_flow.f90:11)
 *   di               : di(halo, N_SPEC)         (code/head/MODULE_flow.f90:12)
 *   prims            : d,u,v,w,T,p,Et stacked, 7 halo arrays
 * All calls return 0 on success or a negative OCFD_ERR_* code; the text of
 * the last error is in ocfd_gpu_last_error().  The library owns all device
 * memory; no host pointer is retained after a call returns.  One host thread,
 * one stream, not re-entrant (the reference's single MPI rank).
 */
#ifndef OCFD_GPU_H
#define OCFD_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OCFD_MAX_SPEC 16
#define OCFD_MAX_REAC 64
#define OCFD_NTCT_MAX 10  /* code/Chemical/CHEM_modules.f90:25 */

/* error codes */
#define OCFD_OK 0
#define OCFD_ERR_PARAM (-1)       /* bad or unsupported parameter (reference: stop in OCFD_readpara.f90) */
#define OCFD_ERR_CUDA (-2)        /* CUDA runtime error / no device / kernel image missing */
#define OCFD_ERR_NAN (-3)         /* NaN in the conserved state (reference: OCFD_debug.f90:20-26) */
#define OCFD_ERR_NEGATIVE_ET (-4) /* more than 10 cells with Et<=0 (OCFD_handle_NegativeT.f90:16-19) */
#define OCFD_ERR_STATE (-5)       /* call order violated (e.g. advance before init) */
#define OCFD_ERR_TIMEOUT (-6)     /* a bounded device wait ran out (persistent chemistry queue) */
#define OCFD_ERR_UNSUPPORTED (-7) /* reference feature outside the built scope */
#define OCFD_ERR_CHEM (-8)        /* chemistry: zero pivot in the implicit step's Gauss elimination
                                     (CHEM_reactions.f90:523-567) or a non-finite reactor result */

/* scheme / option ids: code/head/MODULE_parameter.f90:13-30 */
#define OCFD_SCHEME_WENO5 1
#define OCFD_SCHEME_WENO7 2
#define OCFD_SCHEME_OMP6 3
#define OCFD_SCHEME_UD7L 4
#define OCFD_SCHEME_CD6 5
#define OCFD_SCHEME_CD8 6
#define OCFD_SCHEME_HYBRID 10
#define OCFD_SPLIT_SW 1
#define OCFD_SPLIT_LLF 2
#define OCFD_BC_NONE 0
#define OCFD_BC_BOUNDARYLAYER 2
#define OCFD_BC_JET 4
#define OCFD_CHEM_EULER 1
#define OCFD_CHEM_RK2 2
#define OCFD_CHEM_RK3 3
#define OCFD_CHEM_IMPLICIT (-1)

/* Flat mirror of the reference's Para / Scheme records (code/head/MODULE_parameter.f90:49-96)
 * as they come out of read_control_parameter (code/mpi-io/OCFD_readpara.f90:26-284).
 * Derived quantities of set_parameters (OCFD_readpara.f90:347-431: hx/hy/hz, Bound_index,
 * [Ka,Kb], UD7L coefficients) are computed inside the library from these fields. */
typedef struct ocfd_params {
  int nx, ny, nz;          /* = nx_global.. (single rank) */
  int lap;                 /* halo width, must be 4 */
  int n_spec;
  int iperiodic[3];
  double periodic_span[3][3]; /* [dir][component]: Periodic_ISpan, _JSpan, _KSpan */
  int scheme_invis, scheme_vis;
  int scheme_boundary[6];  /* i-, i+, j-, j+, k-, k+ : 0 WENO5 deleted-stencil, 1 WENO5 full, -1 none */
  int ghost_cell[6];       /* 0 none, 1/2 second-order extrapolation (OCFD_GhostCell.f90:166-364) */
  int if_scheme_character; /* 0 component-wise, 1 characteristic-space flux */
  int if_viscous;
  int flux_splitting;      /* OCFD_SPLIT_SW / OCFD_SPLIT_LLF */
  int if_mass_force;
  double mass_force[3];
  int ibc;                 /* OCFD_BC_NONE / OCFD_BC_BOUNDARYLAYER */
  double bc_para[100];
  double hybrid_para[100];
  double ud7l_diss;
  double aoa;              /* radians (rparameters(20) = AoA*PI/180) */
  int if_realgas;          /* 0 perfect gas (Cv = 2.5 R), 1 NASA-fit thermo */
  int chem_timeadv;        /* 1, 2, 3, -1 */
  int wall_catalysis;      /* must be 0 */
  int istep_show;          /* unused by the library; kept for the mirror */
} ocfd_params;

/* Species thermodynamics: read_Spec (code/Chemical/CHEM_thermdyn.f90:16-51). Ri and the
 * range-continuity offsets Ect are derived inside the library exactly as read_Spec does. */
typedef struct ocfd_thermo {
  int n_spec;
  int n_tct;                         /* number of fit ranges */
  double tct[OCFD_NTCT_MAX];         /* range boundaries Tct(1..n_tct-1) */
  double tct_max;
  double mi[OCFD_MAX_SPEC];          /* molar mass kg/mol */
  int spec_flag[OCFD_MAX_SPEC];      /* 1 monoatomic, 2 diatomic */
  double coef[OCFD_MAX_SPEC][OCFD_NTCT_MAX][7]; /* A,B,C,D,E,F,G per range */
} ocfd_thermo;

/* Reaction mechanism: read_Reac (code/Chemical/CHEM_reactions.f90:15-69). */
typedef struct ocfd_kinetics {
  int n_spec, n_reac;
  int rereac;                         /* 0 Gibbs Kc, 1 Arrhenius reverse, 2 Park fit */
  int af_type[OCFD_MAX_REAC];         /* 0 normal, 1 Troe fall-off, 2 dual Arrhenius */
  int tr_reac[OCFD_MAX_REAC];         /* three-body flag */
  double fc_troe[OCFD_MAX_REAC];
  double af[OCFD_MAX_REAC][2], bf[OCFD_MAX_REAC][2], ef[OCFD_MAX_REAC][2];
  double ar[OCFD_MAX_REAC], br[OCFD_MAX_REAC], er[OCFD_MAX_REAC];
  double park[OCFD_MAX_REAC][5];
  int vf[OCFD_MAX_REAC][OCFD_MAX_SPEC], vr[OCFD_MAX_REAC][OCFD_MAX_SPEC];
  double treff[OCFD_MAX_REAC][OCFD_MAX_SPEC];
} ocfd_kinetics;

/* Transport model: Trans record (code/Chemical/TRANSPORT_modules.f90:16-22). */
typedef struct ocfd_transport {
  int flag_vis, flag_cond, flag_diff;  /* 0 Sutherland/Pr/Sc, 1 Wilke fits */
  double amu0, pr, sc, amk0;
  double mu_an[OCFD_MAX_SPEC][5];
  double k_an[OCFD_MAX_SPEC][5];
  double d_an[OCFD_MAX_SPEC][OCFD_MAX_SPEC][4];
} ocfd_transport;

/* Boundary-layer boundary data (code/boundary-condition/OCFD_BC_Boundarylayers.f90:4-17).
 * Inlet / upper arrays are already re-scaled as init_bcdata_boundary does. The random phases
 * of the wall disturbance (random_number at :523,595) are supplied by the caller. */
typedef struct ocfd_bcdata {
  const double* inlet;        /* BcData_inlet 0: (5+Ns); 1: ny*(5+Ns) as [comp][j]; 2: (5+Ns)*ny*nz as [comp][k][j] */
  const double* upper;        /* BcData_upper 0: (5+Ns); 1: nx*(5+Ns) as [comp][i]; 2: (5+Ns)*nx*nz */
  const double* wall_pertb;   /* nx*nz, BC%wall_pertb(i,k), i fastest; NULL = zero */
  int n_tm;                   /* bc_dis_mt temporal modes */
  const double* tm;           /* TM(1..n_tm) normalised amplitudes */
  const double* fait;         /* fait(1..n_tm) random phases in [0,1) */
} ocfd_bcdata;

/* ---- library lifecycle ---- */

/* Replaces the device-relevant part of NS_solver's setup (OCFD_NS_Solver.f90:12-18, init_mesh
 * OCFD_flow-solver/OCFD_mesh.f90:1-57). coords = Axx,Ayy,Azz (3 halo arrays) as read_mesh* fills
 * them; the library applies the periodic exchange, the periodic coordinate shift, the Jacobian
 * (comput_Jacobian3d, OCFD_mesh.f90:60-107) and Akx1..Asz1 on the device. metrics (optional,
 * NULL = compute) = Akx,Aky,Akz,Aix,Aiy,Aiz,Asx,Asy,Asz,Ajac (10 halo arrays) as for
 * Iflag_Gridtype=31. kin may be NULL when chemistry is off; bc may be NULL for BC_NONE.
 * Differs from a call that would hand over all 19 metric arrays: the library derives the nine
 * Akx1..Asz1 (= A / Ajac) itself, and on a tensor-product grid it keeps the metrics as 1-D
 * derivatives, so the caller passes the coordinates (plus, optionally, the 10 arrays it read). */
int ocfd_gpu_init(const ocfd_params* p, const ocfd_thermo* th, const ocfd_kinetics* kin,
                  const ocfd_transport* tr, const ocfd_bcdata* bc,
                  const double* coords, const double* metrics);

/* Builds the solver state from primitive fields as the reference's start-up does: the tail of
 * init3d (Rescaling_di, conserved f from d,u,v,w,T via comput_E; OCFD_init.f90:8-25) followed by
 * comput_flow_variables and OCFD_bc (OCFD_NS_Solver.f90:17-18). prim5 = d,u,v,w,T (5 interior
 * arrays: the content of the restart file opencfd-comb.dat, OCFD_IO.f90:5-36), di = Ns interior
 * arrays. Halo points take allocate_flow_data's initial values (OCFD_allocate_data.f90:53-67). */
int ocfd_gpu_init_state(const double* prim5, const double* di, double tt);

/* Uploads the Fortran module state: f (N*5), di (H*Ns), prims (7*H: d,u,v,w,T,p,Et). The
 * restart's tt and Istep stay with the caller (tt is an argument of the advancing calls). */
int ocfd_gpu_upload_state(const double* f, const double* di, const double* prims);

/* flow_time_advance(dt1) (code/flow-solver/OCFD_Time_Adv.f90:7-92): 3 RK stages; tt is the
 * solver time at the call (used by the wall disturbance, OCFD_BC_Boundarylayers.f90:147). The
 * reference routine takes dt1 alone and reads tt from the module flow_para; a C library has no
 * such module, so the caller passes its tt. */
int ocfd_gpu_flow_advance(double dt1, double tt);

/* nsub x Chemical_time_advance(dt2) (OCFD_Time_Adv.f90:169-196) followed by comput_T_P
 * (Comput_flow_variables.f90:30-46), as OCFD_NS_Solver.f90:30-35. */
int ocfd_gpu_chem_advance(double dt2, int nsub);

/* One full reference time step (OCFD_NS_Solver.f90:28-37): flow(dt/2), chemistry (if
 * if_reaction), flow(dt/2). Captured as a CUDA graph after the first call with a given dt. */
int ocfd_gpu_step(double dt, double tt, int if_reaction, int nsub);

/* nsteps consecutive ocfd_gpu_step calls (solver time tt0, tt0+dt, ..., accumulated as the
 * reference's tt = tt + dt) replayed back to back on the device with one status check at the end;
 * the reference's time loop without I/O steps. Chunks of 16 steps are one graph launch each (the
 * captured step as a child graph, the step's wall-disturbance time taken on the device). */
int ocfd_gpu_run(double dt, double tt0, int nsteps, int if_reaction, int nsub);

/* Downloads the state; any pointer may be NULL to skip that part. The mixture viscosity Amu is
 * not part of it: the analysis that reads Amu (ana_box) runs on the device
 * (ocfd_gpu_keep_viscosity, ocfd_gpu_ana_box). */
int ocfd_gpu_download_state(double* f, double* di, double* prims);

/* show_flow_msg reductions (OCFD_Time_Adv.f90:210-223): mean total and kinetic energy. */
int ocfd_gpu_diag(double* e_mean, double* k_mean);

/* The same without stalling the time loop: _begin enqueues the sums and their copy to pinned
 * host memory (a copy stream), _end waits for them; steps may run in between (the sums are of
 * the state at _begin). ocfd_gpu_diag = _begin + _end. */
int ocfd_gpu_diag_begin(void);
int ocfd_gpu_diag_end(double* e_mean, double* k_mean);

/* save_flow_data (OCFD_IO.f90:39-64) without a host sync: ocfd_gpu_snapshot packs d, u, v, w, T
 * and every di (interior arrays, the file's field order) on the device and copies them to pinned
 * host memory on a copy stream while the next steps run. ocfd_gpu_snapshot_wait waits for the
 * oldest snapshot in flight and returns its Istep, tt and a pointer to its (5 + N_SPEC) * N doubles;
 * the pointer stays valid until the second-next ocfd_gpu_snapshot (two slots). A third snapshot
 * while two are in flight is OCFD_ERR_STATE. */
int ocfd_gpu_snapshot(int istep, double tt);
int ocfd_gpu_snapshot_wait(int* istep, double* tt, const double** fields);

/* Downloads the hybrid-scheme sensor Rhybrid (halo array) for decision-map comparisons. */
int ocfd_gpu_download_rhybrid(double* rhybrid);

/* Downloads the ten Jacobian arrays (Akx..Asz, Ajac; 10 halo arrays). */
int ocfd_gpu_download_metrics(double* metrics);

/* Batched 0-D chemistry: chemical_timeAdv (CHEM_reactions.f90:374-390) applied nsub[r]
 * times with step dt[r]/nsub[r] to n independent reactors, di (n*Ns, reactor-major) and E
 * (n) updated in place. nsub == NULL means 1 sub-step each. Runs as one persistent
 * work-queue kernel on the device; host buffers in and out. */
int ocfd_gpu_chem_batch(int n, double* di, double* e, const double* dt, const int* nsub);

/* Same as ocfd_gpu_chem_batch with device pointers (no host copies).
 * The batched calls (these two and ocfd_gpu_chem_batch_noalloc) return OCFD_ERR_CHEM when a
 * reactor's implicit step met a zero Gauss pivot or its result is not finite: every reactor's
 * values are still written back as computed (the reference divides by the zero pivot and goes
 * on), the code reports it. n < 0 is OCFD_ERR_PARAM, n = 0 does nothing. */
int ocfd_gpu_chem_batch_device(int n, double* d_di, double* d_e, const double* d_dt,
                               const int* d_nsub);

/* Constant-pressure batched reactors (no counterpart in the reference, whose reactor is the flow
 * solver's constant-volume cell, OCFD_Time_Adv.f90:174-193): on = 1 makes ocfd_gpu_chem_batch*
 * hold each reactor's initial pressure at constant specific total enthalpy after every sub-step
 * (mass fractions fixed, Newton on T, density rescaled to the pressure); on = 0 restores the
 * reference's constant-volume reactor (default); on < 0 returns the setting. The flow solver's
 * cells stay constant-volume either way, and ocfd_gpu_chem_batch_surrogate refuses constant-pressure
 * batches (OCFD_ERR_UNSUPPORTED). */
int ocfd_gpu_chem_constant_pressure(int on);

/* Compiled mechanism kernels (no counterpart in the reference, which interprets its mechanism
 * tables in every reaction loop, CHEM_reactions.f90:130-272): the library carries the 9-species
 * H2-air mechanism of the jet case as straight-line rate and Jacobian code
 * (opencfd-comb_b200/csrc/ocfd_mech_h2air9.cuh, generated from its data file). When the loaded
 * mechanism has exactly that structure (species count, reactions, stoichiometry, rate forms,
 * third-body flags) and CHEM_TimeAdv = -1, the flow step's chemistry and the batched reactors
 * run it; its numbers equal the generic kernels' bit for bit on finite states. on = 0 keeps the
 * generic kernels, on = 1 allows the compiled ones (default), on < 0 changes nothing. Returns 1
 * when the compiled kernels are in use for the current set-up, else 0. */
int ocfd_gpu_chem_compiled_mechanism(int on);

/* The last batched chemistry call's counts: reactors whose Newton T(E) iteration did not converge
 * (comput_T_rgas, CHEM_thermdyn.f90:327-382, at most 31 iterations) and reactors reported by
 * OCFD_ERR_CHEM (zero pivot or non-finite result). Either pointer may be NULL. */
int ocfd_gpu_chem_batch_status(long long* newton_fail, long long* bad);

/* Sets up the chemistry tables alone (no grid) for ocfd_gpu_chem_batch: read_Spec + read_Reac
 * content, IF_RealGas and CHEM_TimeAdv. */
int ocfd_gpu_chem_setup(const ocfd_thermo* th, const ocfd_kinetics* kin, int realgas, int timeadv);

/* filtering (code/others/OCFD_filtering.f90:4-72), the reference's call after every step
 * (OCFD_NS_Solver.f90:48) with Istep already advanced. filter = Para%Filter(100,10) column-major
 * (group m's parameters at filter[100*(m-1) + 0..12]: step interval, filter x/y/z, ib, ie, jb, je,
 * kb, ke (global indices), scheme 1 = 9-point Bogey-Bailly Fo9p, 2 = shock-capturing, amplitude
 * s0, threshold rth), nfiltering = Para%NFiltering (0..10). Each due group filters f in x, then
 * y, then z; the primitives keep their values (the shock filter recomputes them from f first,
 * comput_flow_variables, as the reference does). applied (may be NULL) = 1 when a group ran. */
int ocfd_gpu_filtering(int istep, int nfiltering, const double* filter, int* applied);

/* Keeps the mixture viscosity Amu of every RK stage (comput_Amu_Amk_AMD at the stage start,
 * OCFD_Time_Adv.f90:35) on the device so that ocfd_gpu_ana_box can average it. With N_SPEC > 1
 * it is always kept; a single-species run computes it inline and needs this switch on before
 * the steps whose last stage ana_box reads. */
int ocfd_gpu_keep_viscosity(int on);

/* ana_box (code/others/OCFD_ANA.f90:197-303), isotropic-turbulence statistics of the current
 * state: out[19] = tt, Re_lamda, Re_lamdax, Amt, vv_rms, u_rms, v_rms, w_rms, u_skewness,
 * u_flatness, ux_skewness, ux_flatness, E_kinetic, d_rms, T_aver, Amu_aver, d_aver, Ux_rms,
 * Alamdax (the row the reference appends to statistics.dat). Sums are fixed-order trees. */
int ocfd_gpu_ana_box(double tt, double* out);

/* ana_getQ (OCFD_ANA.f90:143-190): Q, the second invariant of the velocity gradient, into q
 * (N interior doubles, the array the reference writes to Q-<Istep>.dat). */
int ocfd_gpu_ana_q(double* q);

/* ana_time_average (OCFD_ANA.f90:39-140): one accumulation of the running means of d, u, v, w,
 * T and every di on the device; K_average and t_average after it are returned (may be NULL).
 * ocfd_gpu_ana_average downloads (upload = 0) or restores (upload = 1, from a
 * opencfd-comb.dat.average restart) the (5 + N_SPEC) interior arrays with K_average, t_average. */
int ocfd_gpu_ana_time_average(double dt, int* k_average, double* t_average);
int ocfd_gpu_ana_average(int upload, double* fields, int* k_average, double* t_average);

/* Stencil tile autotuner (no counterpart in the reference, whose loops have no tiles). A tile
 * choice is int[9] = {flux tile shape of the x, y, z flow sweeps (0, 1, 2); k planes per block of
 * the viscous-flux kernel and of its divergence kernel; metric form of the flux sweeps, the
 * viscous-flux kernel and the divergence kernel (0 computed from the 1-D grid derivatives of a
 * tensor-product grid, 1 read from the 19 stored arrays, which are then computed once; a general
 * grid always reads them); stream switches, bit 0: the viscous-flux kernel runs beside the flux
 * sweeps on a second stream (a parallel branch of the step's graph) instead of after them, bit 1:
 * the species chain (species sweeps, then divergence and RK update) runs on a third stream beside
 * the species viscous fluxes and the flow part instead of in order}. Shapes (cells along the
 * sweep x pencils): x 56x4, 120x2, 24x8; y / z 24x16, 24x8, 56x8. Every choice gives
 * bit-identical results.
 * ocfd_gpu_autotune times each candidate on the current state (after ocfd_gpu_init_state) over reps
 * launches, applies the fastest and remembers it for this configuration (grid, schemes, species)
 * in the process; reps = 0 applies a remembered choice without timing when there is one. choice
 * (may be NULL) receives the choice; ms (may be NULL, 27 doubles) the mean ms per launch of each
 * candidate: flux x, y, z shapes 0..2, k_visc_ev at 8, 16, 32, 64 planes, k_visc_div at 8, 16,
 * 32, 64 planes and in its per-cell form (k planes 0), then with the stored metric arrays at the
 * best tiles: flux x, y, z, k_visc_ev, k_visc_div, then the flow right-hand side of a stage with
 * the viscous flux after and beside the flux sweeps, then a stage's right-hand sides without the
 * species RK update with the species chain in order and on the third stream (-1 where not timed).
 * The launches write only scratch arrays, so the solution is unchanged. Default choice
 * {0, 0, 0, 16, 16, 0, 0, 0, 3}. */
int ocfd_gpu_autotune(int reps, int* choice, double* ms);
int ocfd_gpu_set_tiles(const int* choice);
int ocfd_gpu_get_tiles(int* choice);

/* Per-kernel-class CUDA-event timing of the non-graph launches (enable resets the totals). */
int ocfd_gpu_profile(int enable);
int ocfd_gpu_profile_read(int cls, double* ms, long long* count);
const char* ocfd_gpu_profile_name(int cls);
int ocfd_gpu_profile_nclass(void);
/* The library's CUDA stream (cudaStream_t), for callers that time or order work around it. */
void* ocfd_gpu_stream(void);
/* CUDA events on the library stream (slots 0..15) and the time between two of them. */
int ocfd_gpu_event_record(int slot);
int ocfd_gpu_event_elapsed(int a, int b, double* ms);
/* Page-locked host buffers for fast host<->device copies of the state. */
int ocfd_gpu_pinned_alloc(size_t bytes, void** ptr);
int ocfd_gpu_pinned_free(void* ptr);
/* Kernels in one captured Strang step. */
int ocfd_gpu_step_launches(void);
/* Kernels launched by the library since init (graph replays count their kernels). */
long long ocfd_gpu_launch_count(void);
/* Bytes of the device arena in use (state, metrics, work arrays). */
long long ocfd_gpu_device_bytes(void);
/* 1 when the grid is a tensor product and metrics are kept as three 1-D arrays. */
int ocfd_gpu_is_separable(void);

/* ocfd_gpu_chem_batch_device for callers that cannot allocate device memory: it allocates
 * nothing and keeps its scratch (reactor ordering, sub-step histogram, work-queue counter) in a
 * fixed array of the library sized for at most 1048576 reactors (about 4 MB, held on every GPU
 * that loads the library until exit). Larger n returns OCFD_ERR_PARAM. The first call on a device
 * looks up the array's device address, so make that first call before any stream capture. All
 * calls share the one array: calls that overlap on the GPU (other threads, other streams) race.
 * No counterpart in the reference (its chemistry loop runs on the CPU and allocates nothing). */
int ocfd_gpu_chem_batch_noalloc(int n, double* d_di, double* d_e, const double* d_dt, const int* d_nsub);

/* Statistics of the last advance: number of Et<=0 repairs, Newton non-converged cells. */
int ocfd_gpu_stats(long long* neg_et, long long* newton_fail);

const char* ocfd_gpu_last_error(void);
int ocfd_gpu_finalize(void);

/* Measures the device's FP64 FMA throughput (GFLOP/s) with a register-resident loop
 * (roofline denominator for the FP64-bound kernels). */
double ocfd_gpu_fp64_peak_gflops(void);

/* ---- learned chemistry surrogate (no counterpart in the reference) ----
 * Tensor-core GEMM of the surrogate's dense layers, exposed for testing: on device pointers,
 * C(M x N) = A(M x K) . B(N x K)^T (+ bias(N)) (+ C when beta = 1), then GELU when act = 1.
 * A and B are BF16 read through element strides (A(m,k) = A[m*sam + k*sak], B(n,k) =
 * B[n*sbn + k*sbk]), C is FP32 with leading dimension ldc. Synchronous. */
int ocfd_gpu_gemm_bf16(int M, int N, int K, const void* A, long long sam, long long sak, const void* B, long long sbn,
                       long long sbk, float* C, long long ldc, const float* bias, int beta, int act);

/* The surrogate: a BF16 MLP (inputs T, log p, Y_1..Y_Ns, log dt; three hidden layers of 256, GELU;
 * outputs dY_1..dY_Ns, dT) for 0-D reactors of the mechanism given to ocfd_gpu_chem_setup (or
 * ocfd_gpu_init), 2 <= N_SPEC <= 9. All reactor arrays are device pointers, di as n x N_SPEC.
 * ocfd_gpu_surrogate_init: seeded initial weights (for ocfd_gpu_surrogate_grad).
 * ocfd_gpu_surrogate_train: trains on n reactors (di0, e0, dt) and their FP64-integrated states
 * (di1, e1) with Adam (cosine-decayed lr), batch a multiple of 128; proj is the N_SPEC x N_SPEC
 * projection onto element-conserving composition changes; loss_history gets one value per epoch.
 * ocfd_gpu_surrogate_predict: ungated network updates (di_out, e_out), T0 + dT_pred (T_pred) and
 * the temperature of the updated state's energy (T_energy).
 * ocfd_gpu_chem_batch_surrogate: gated surrogate chemistry in place; reactors whose |T_energy -
 * T_pred| exceeds tol_T, whose composition goes negative or whose input lies outside the training
 * range are advanced by the FP64 implicit integrator instead; n_fallback gets their number.
 * ocfd_gpu_surrogate_blob: save (set 0) / load (set 1) weights, normalisation and projection as
 * floats; host NULL returns the size. ocfd_gpu_surrogate_grad: loss and parameter gradients of
 * one batch of normalised inputs / targets (B x 16 floats, host), for gradient checks.
 * ocfd_gpu_chem_temperature: T of n reactors from densities and energy (comput_T). */
int ocfd_gpu_surrogate_init(unsigned seed);
int ocfd_gpu_surrogate_train(int n, const double* d_di0, const double* d_e0, const double* d_dt, const double* d_di1,
                             const double* d_e1, const double* proj, int epochs, int batch, double lr, unsigned seed,
                             double* loss_history);
int ocfd_gpu_surrogate_predict(int n, const double* d_di, const double* d_e, const double* d_dt, double* d_di_out,
                               double* d_e_out, double* d_T_pred, double* d_T_energy);
int ocfd_gpu_chem_batch_surrogate(int n, double* d_di, double* d_e, const double* d_dt, const int* d_nsub,
                                  double tol_T, int* n_fallback);
long long ocfd_gpu_surrogate_blob(float* host, long long nfloats, int set);
int ocfd_gpu_surrogate_grad(int B, const float* x, const float* t, float* grads, double* loss);
int ocfd_gpu_chem_temperature(int n, const double* d_di, const double* d_e, double* d_T);

/* Inference form of the network: 1 (default) = one fused tcgen05 kernel for the four layers (the
 * hidden activations stay in shared memory / TMEM), 0 = one GEMM per layer through global memory;
 * both issue the same MMAs and epilogue arithmetic. on < 0 only queries. Returns the previous
 * setting. */
int ocfd_gpu_surrogate_fused(int on);

/* Chemistry of the flow solver's Strang step (ocfd_gpu_step, ocfd_gpu_run, ocfd_gpu_chem_advance).
 * The network is not read from a weights file here: it is trained on the device
 * (ocfd_gpu_surrogate_train) or loaded from floats (ocfd_gpu_surrogate_blob, set = 1), and this
 * call takes the gate tolerance instead of a path:
 * mode 0 the FP64 integrator of Chemical_time_advance (default), mode 1 the gated surrogate, whose
 * rejected cells (|T_energy - T_pred| > tol_T, negative composition, outside the training range)
 * take the FP64 sub-steps; the step stays one CUDA graph. Mode 1 needs a trained or loaded
 * surrogate for this mechanism. ocfd_gpu_chem_surrogate_rejected: cells that took the FP64 path in
 * the last chemistry call; reasons (when not NULL) gets how many failed each test: negative
 * composition, temperature check, T / log p / log dt outside the training range, a mass fraction
 * outside its training range widened by half its normalisation scale. */
int ocfd_gpu_chem_mode(int mode, double tol_T);
long long ocfd_gpu_chem_surrogate_rejected(long long* reasons /* 6 counts or NULL */);

#ifdef __cplusplus
}
#endif
#endif
