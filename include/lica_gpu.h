/*
 * lica_gpu.h -- C ABI of the B200 (sm_100a) hot path of the lica two-phase boiling
 * solver.  Plain pointers and sizes only; every entry point returns a lica_status.
 *
 * Two kinds of entry points:
 *   1. Drop-ins for the reference's Fortran subroutines (1d.f), taking the same arrays
 *      in the same Fortran layout (column-major, the Fortran lower bound of each array
 *      noted per argument).  Arrays are HOST arrays; the call copies them to the GPU,
 *      runs the CUDA kernels and copies the results back, like the subroutine it
 *      replaces.  A Fortran host binds them with ISO_C_BINDING interfaces.
 *   2. Device-resident entry points (suffix _device) taking device pointers and a
 *      cudaStream_t passed as void*, for callers that keep state in HBM.
 *
 * Threading: call a given context from one host thread at a time.  Contexts are
 * independent.  Errors never abort the process: the return value says what happened
 * and lica_last_error() gives a message for LICA_ERR_CUDA / LICA_BAD_ARG.
 */
#ifndef LICA_GPU_H
#define LICA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (the reference has none: it STOPs or prints and continues). */
enum lica_status {
    LICA_OK = 0,
    LICA_NOT_CONVERGED = 1, /* iteration cap reached before the tolerance */
    LICA_BAND_OVERFLOW = 2, /* analogue of the band-size STOP, two_phase.f:1989-1994 */
    LICA_NAN = 3,           /* non-finite value met */
    LICA_BAD_ARG = 4,       /* argument outside what the entry point supports */
    LICA_ERR_CUDA = 5,      /* a CUDA runtime call failed (see lica_last_error) */
    LICA_ERR_NOMEM = 6,
    LICA_ERR_IO = 7,        /* a file could not be opened, read or written, or a record is malformed */
    LICA_STALLED = 8        /* an iterative solve stopped at FP64's attainable accuracy: its true
                               residual rose after falling within 1000x the tolerance, and the
                               iterate before the rise is returned */
};

/* Message for the last LICA_ERR_CUDA / LICA_BAD_ARG on the calling thread. */
const char* lica_last_error(void);

/* Number of kernel launches this library has issued since load (a counter the
 * benchmark reads; graph replays count each kernel node). */
int64_t lica_kernel_launch_count(void);

/* Diagnostic (no counterpart in the reference): fills every SM's shared memory with value
 * (launches on `stream` and returns).  The kernels here must never read shared memory they
 * have not written; running them after this call with a NaN shows any that does, where
 * ordinary runs can hide it behind whatever an earlier kernel left there. */
int lica_debug_poison_shared(double value, void* stream);

/* ------------------------------------------------------------------------------------
 * Tridiagonal solvers
 * ---------------------------------------------------------------------------------- */

/* TRDIAG3 (1d.f:3783-3811): for every line I in [ll1,ll2] solve the tridiagonal
 * system along J in [l1,l2]:  A(I,J) x(J-1) + B(I,J) x(J) + C(I,J) x(J+1) = R(I,J).
 * A,B,C,R,UU are Fortran (ld, *) arrays, 1-based: X(I,J) = x[(I-1) + (J-1)*ld].
 * UU receives the solution, R(I,J) is overwritten with it for J < l2 (as the
 * reference's loop 30 does); R and UU may be the same array (LHSW, 1d.f:1790).
 * Host arrays; one GPU thread per line, Thomas algorithm in the reference's order. */
int lica_gpu_trdiag3(const double* A, const double* B, const double* C, double* R, double* UU,
                     int64_t l1, int64_t l2, int64_t ll1, int64_t ll2, int64_t ld);

/* TRDIAG3P (1d.f:3929-3983): periodic (cyclic) tridiagonal systems; lines K in
 * [l1,l2] (first index), unknowns J in [j1,j2] (second index); the solution
 * overwrites F.  Host arrays, Fortran (ld, *) layout as above. */
int lica_gpu_trdiag3p(const double* A, const double* B, const double* C, double* F,
                      int64_t j1, int64_t j2, int64_t l1, int64_t l2, int64_t ld);

/* Device-resident batched variants: same layout, device pointers. */
int lica_gpu_trdiag3_device(const double* A, const double* B, const double* C, double* R, double* UU,
                            int64_t l1, int64_t l2, int64_t ll1, int64_t ll2, int64_t ld, void* stream);
int lica_gpu_trdiag3p_device(const double* A, const double* B, const double* C, double* F,
                             int64_t j1, int64_t j2, int64_t l1, int64_t l2, int64_t ld, void* stream);

/* TRDIAG3 on device arrays that allocates no memory.  No counterpart in the reference:
 * it is for callers that cannot call cudaMalloc -- e.g. a solver loop whose device
 * memory is owned by a pre-allocated pool, or one that must not hit the device-wide
 * synchronisation of cudaMalloc/cudaFree or an out-of-memory failure mid-run.  Same
 * kernel and bit-identical results as lica_gpu_trdiag3_device; its scratch is a fixed
 * 2 MiB device array inside this library, so ld * l2 must not exceed 262144 (else
 * LICA_BAD_ARG).  The first call on a device sets up the scratch address and should be
 * made before any stream capture; the address is kept for the life of the process, so do
 * not use this entry point on a device after cudaDeviceReset.  Enqueues on `stream` and
 * returns without waiting.
 * Calls that overlap on the GPU share the scratch and race: serialise them (one stream
 * per device). */
int lica_gpu_trdiag3_noalloc_device(const double* A, const double* B, const double* C, double* R, double* UU,
                                    int64_t l1, int64_t l2, int64_t ll1, int64_t ll2, int64_t ld, void* stream);

/* POISSON (1d.f:3492-3578), the 1-D column the reference solves (N1M = N2M = 1):
 * AK = VVDZ(K)*SSDZ(K)*DENF_ZI(1,1,K)*(1-FIXKL(K)), CK = VVDZ(KP1)*SSDZ(K)*DENF_ZI(1,1,KP1),
 * BK = -(AK+CK), Thomas solve, P(1,1,K) = x(K), then P(I,J,0)=P(I,J,1) and
 * P(I,J,N3)=P(I,J,N3M).  Array bounds (Fortran):
 *   P, DENF_ZI: (0:m1, 0:m2, 0:m3)     DIVGSUM: (m1-1, m2-1, m3-1), 1-based
 *   vvdz: VVDZ(1:m3)   ssdz: SSDZ(0:m3)   fixkl: FIXKL(1:m3-1)   kpv: KPV(0:m3+1)
 * Host arrays.  Returns LICA_BAD_ARG unless n1m = n2m = 1 (2-D and 3-D fields use the
 * multigrid entry points below). */
int lica_gpu_poisson(int64_t m1, int64_t m2, int64_t m3, int64_t n1m, int64_t n2m, int64_t n3m,
                     const double* vvdz, const double* ssdz, const double* fixkl, const int64_t* kpv,
                     double* p, const double* divgsum, const double* denf_zi);

/* ------------------------------------------------------------------------------------
 * Multigrid-preconditioned CG pressure Poisson, 2-D (new build; the reference's POISSON
 * is 1-D Thomas).  Operator: the 2-D generalisation of 1d.f:3535-3541 on a uniform
 * nx x ny cell grid, x periodic, y a wall with Neumann bottom (FIXKL) and p = 0 on the
 * top face (VVDZ(N3) = 2/h, FIXKU commented out at 1d.f:3538):
 *   (A u)_ij = sum over the 4 faces of beta_face/h^2 * (u_nb - u_ij),
 *   bx[j*nx+i] = beta on the face left of cell i (periodic), j in [0,ny)
 *   by[j*nx+i] = beta on the face below cell row j, j in [0,ny]  (row 0 unused, row ny
 *                the top wall, weighted 2/h^2).
 * Solves A p = f to ||f - A p||_2 <= rtol ||f||_2 with PCG whose preconditioner is one
 * symmetric V(nu1,nu2) red-black Gauss-Seidel cycle (piecewise-constant prolongation,
 * 2x2 restriction, face-averaged beta), the coarsest outer level solved by ncoarse inner
 * V-cycles ending in a dense elimination.
 * ---------------------------------------------------------------------------------- */
typedef struct lica_mg lica_mg;

typedef struct {
    int32_t nlevels;   /* outer levels, e.g. 6 for 1024^2 (coarsest 32^2) */
    int32_t nu1, nu2;  /* pre/post red-black sweeps, e.g. 2,2 */
    int32_t ncoarse;   /* inner V-cycles at the coarsest outer level */
    int32_t precision; /* 0: FP64 throughout; 1: mixed -- FP32 smoothing, restriction and
                          prolongation; FP64 residual, CG vectors and coarsest solve */
    int32_t use_graph; /* 1: the whole solve is one CUDA graph with a device-side loop */
    int32_t smoother;  /* 0: red-black point Gauss-Seidel (temporal-blocked tiles, the
                          single-CTA coarse kernel); 1: y-line zebra relaxation -- columns of
                          one parity solved exactly along y (Thomas), for cells much finer
                          in y than in x (stretched wall grids, lica_mg_stretched_system);
                          FP64 only, every level as plain grid kernels */
} lica_mg_options;

typedef struct {
    int32_t iterations;  /* PCG iterations taken */
    int32_t status;      /* lica_status of the solve */
    double rel_residual; /* ||f - A p||_2 / ||f||_2 (FP64 true residual) */
} lica_mg_result;

/* Create a solver for an nx x ny grid with spacings hx, hy.  nx and ny must be
 * multiples of 32 and halve evenly nlevels-1 times. */
int lica_mg_create(lica_mg** out, int32_t nx, int32_t ny, double hx, double hy, const lica_mg_options* opt);
int lica_mg_destroy(lica_mg* mg);

/* Device-resident solve: p (initial guess in, solution out), f, bx, by are device
 * arrays of nx*ny, nx*ny, nx*ny, nx*(ny+1) doubles.  Enqueued on stream; the call
 * returns after the solve finished (it reads back the result). */
int lica_mg_solve_device(lica_mg* mg, double* p, const double* f, const double* bx, const double* by,
                         double rtol, int32_t max_iters, lica_mg_result* res, void* stream);

/* Same solve on HOST arrays: copies f, bx, by, p to the GPU, solves, copies p back.
 * stream may be NULL (the context's own stream); the call returns when p is on the host. */
int lica_mg_solve_host(lica_mg* mg, double* p, const double* f, const double* bx, const double* by,
                       double rtol, int32_t max_iters, lica_mg_result* res, void* stream);
/* A sequence of independent solves from host arrays (count systems, each with its own p, f,
 * bx, by): the upload of system k + 1 and the download of system k - 1 overlap the solve of
 * system k (two staging buffers on the device, separate upload and download streams; pinned
 * host arrays are needed for the overlap).  res holds count results; returns the first
 * non-OK solve status, or LICA_OK. */
int lica_mg_solve_host_batch(lica_mg* mg, int32_t count, double* const* p, const double* const* f,
                             const double* const* bx, const double* const* by, double rtol, int32_t max_iters,
                             lica_mg_result* res);

/* One application of the preconditioner, z = M r (device arrays). */
int lica_mg_precond_device(lica_mg* mg, double* z, const double* r, const double* bx, const double* by,
                           void* stream);

/* out = A u (device arrays). */
int lica_mg_apply_device(lica_mg* mg, double* out, const double* u, const double* bx, const double* by,
                         void* stream);

/* Kernel-class timing with CUDA events around each launch.  While enabled, solves run
 * as individual launches (not as a graph) so each kernel can be bracketed; the kernel
 * sequence is the same as the graph's.  lica_mg_profile resets the totals. */
enum lica_mg_kernel_class {
    LICA_MG_DOWN0 = 0,   /* k_down on level 0 */
    LICA_MG_DOWN = 1,    /* k_down on coarser grid levels */
    LICA_MG_UP0 = 2,     /* k_up on level 0 (with the r.z partial) */
    LICA_MG_UP = 3,
    LICA_MG_CTA = 4,     /* single-CTA coarse levels */
    LICA_MG_PUPDATE = 5, /* p = z + beta p, p.Ap */
    LICA_MG_XUPDATE = 6, /* x += alpha p, r = f - A x, ||r|| */
    LICA_MG_SETUP = 7,   /* beta coarsening */
    LICA_MG_NCLASS = 8
};
int lica_mg_profile(lica_mg* mg, int32_t enable);
int lica_mg_profile_read(lica_mg* mg, int32_t kernel_class, double* total_ms, int64_t* launches);

/* ------------------------------------------------------------------------------------
 * Level-set transport of 1-D columns: TRANSPORT (two_phase.f:701-984, called from MAIN,
 * 1d.f:242) followed by GRID_COUPLING(0) (two_phase.f:4863-5118, 1d.f:244), for the
 * 1 x 1 x n flow column with its 2 x 2 x 2n refined level-set grid (the reference's 1-D
 * case; the refined field is the same on the four (I,J) replicas, so one value per
 * refined z-level is stored).  A batch of ncol columns of equal n and length is stored
 * back to back; each column is independent.  Per column (nf = 2n):
 *   phi    [nf+7]  ALPHI(k), k = -2..nf+4 at [k+2]: band values (outside the band any
 *                  value; TRANSPORT zeroes it)                                    in/out
 *   layer  [nf+7]  band layer of refined cell k (0 outside, 1..11), the reference's
 *                  I_B/J_B/K_B lists as a per-cell number                         in/out
 *   psif   [nf+2]  PSIF(k) at [k], k = 1..nf                                      in/out
 *   wo     [n+2]   WO(k), k = 0..n+1: the face velocity of the previous call      in/out
 *   w      [n+2]   W(k), k = 0..n+1                                               in
 *   mflvs  [nf+7]  interfacial mass flux of band cell k (MFLVS), read if iphs = 1 in
 *   vol_tot_ori    VOL_TOT_ORI, the target vapour volume                          in/out
 *   vol_tot_iphs   VOL_TOT_IPHS from VOL_TOT_MFDOT (used if iphs = 1)             in
 *   psi_cn, psi_zn [n+2] PSI_CN(k), PSI_ZN(k), k = 0..n+1                         in/out
 *   status         per-column lica_status (LICA_BAND_OVERFLOW: the band, 11 layers around
 *                  every interface, spans more than 112 refined cells or left its window;
 *                  that column is left unchanged)                                 out
 *   stats  [4]     subcycles (0 if there was nothing to move), |grad phi| max and
 *                  min over layers 1..8, IMASS                                    out
 * n >= 8.  Host arrays for lica_gpu_lvs_transport (returns the last non-OK column
 * status, or LICA_OK); device arrays and a stream for the _device form (enqueues and
 * returns; read status afterwards). */
typedef struct {
    int32_t iphs;    /* IPHS: 1 with phase change (source term, reinit every subcycle) */
    int32_t first;   /* 1 on the first call of a run: WO = W before averaging */
    int32_t m_step;  /* time step number M (the MOD(M,50) mass-correction trigger) */
    int32_t mglobal; /* MGLOBAL: 1 applies GLOBAL_MASS_CORRECTION */
    double denr;     /* DENR, liquid/vapour density ratio used by the source term */
    double dtconst;  /* DTCONST, the flow time step */
} lica_lvs_params;

int lica_gpu_lvs_transport(int32_t ncol, int32_t n, double length, double* phi, int32_t* layer, double* psif,
                           double* wo, const double* w, const double* mflvs, double* vol_tot_ori,
                           const double* vol_tot_iphs, double* psi_cn, double* psi_zn, int32_t* status,
                           double* stats, const lica_lvs_params* prm);
/* ------------------------------------------------------------------------------------
 * Whole RK3 time steps of 1-D boiling columns: MAIN's step (1d.f:190-250) -- DETERMINE_DT,
 * three substeps of RHSNLHS (CAL_CONTINUITY, CAL_CONT_BC, PASSIVE_SCALAR with TEMP_GRAD /
 * TEMP_EXTP / TF_GRAD / VOL_TOT_MFDOT / CAL_CONTINUITY2, RHSZ, LHSW, BC, FSM_CHOI,
 * PRESSURE_CORRECTION), CONVRGE1, TRANSPORT and GRID_COUPLING -- for a batch of independent
 * columns of n flow cells, one persistent kernel for any number of steps.
 * The missing LHSPS2 of the reference (called at 1d.f:3665) is the LHSPS solve.
 * ---------------------------------------------------------------------------------- */
typedef struct {
    double re, visr, denr; /* RE_M, VISR, DENR (lica.in) */
    double weber, fr;      /* WEBER, FR */
    double prm, scr, tcr;  /* PRM, SCR, TCR */
    double t_sat, jakob;   /* T_SAT, JAKOB */
    double cflmax, dt0;    /* CFLFAC, initial DT */
    int32_t iphs, mglobal; /* IPHS (phase change), MGLOBAL (global mass correction) */
} lica_col_props;

/* State of ncol columns stored back to back (nf = 2n):
 *   w, p, t, psi_cn, psi_zn, wo : n+2 doubles per column, index k = 0..n+1
 *   phi, mflvs : nf+7 doubles (k = -2..nf+4 at k+2);  layer : nf+7 int32
 *   psif, sfgas, sfgas2 : nf+2 doubles (k = 1..nf at k);  imask : n+2 int32
 *   scal : 5 doubles  (DT, TIME, M = steps taken, VOL_TOT_ORI, VOL_TOT_IPHS)
 *   stats: 8 doubles  (flow CFL, max |div u - source|, TEMP_EXTP iterations, level-set
 *                      subcycles, mass-correction triggers, interface height, vapour
 *                      volume, DT) of the last step */
typedef struct {
    double *w, *p, *t, *psi_cn, *psi_zn;
    double* phi;
    int32_t* layer;
    double *psif, *wo, *mflvs, *sfgas, *sfgas2;
    int32_t* imask;
    double *scal, *stats;
} lica_col_state;

/* Initial state of one column with a vapour film of thickness z0 at the wall (MAKEFLD
 * 1d.f:821-946 with IPHS = 1, LVSINIT two_phase.f:116-388, GRID_COUPLING(1)); host arrays
 * of one column. */
int lica_gpu_column_init(int32_t n, double length, double z0, const lica_col_props* props, lica_col_state* st);

/* ------------------------------------------------------------------------------------
 * Non-uniform grids (host code, no GPU)
 * ---------------------------------------------------------------------------------- */

/* One section of the grid generator (grid.f:118-128): XYZ(N), N = ngi..ngf, into
 * xyz[N - 1].  iopt 1: UNIFORM (grid.f:326-345); 2: GEOPRO (348-380), fac1 = ER, fac2 =
 * YESEXP (1 expansion, else compression); any other: HYPTAN (383-420), fac1 = GAM, fac2 =
 * XSI (1 clusters at xyzi, 0.5 at both ends, 0 at xyzf).  Double precision. */
int lica_grid_section(int32_t iopt, double xyzi, double xyzf, int32_t ngi, int32_t ngf, double fac1, double fac2,
                      double* xyz);

/* GEOMETRIC (1d.f:4808-4882) for one wall-bounded direction with n faces z[1..n] (z[0]
 * unused): SDZ(0..n), VDZ(1..n), SSDZ(0..n), VVDZ(1..n), ZP(0..n), each array n+1 long
 * and indexed by the Fortran index (entries the reference leaves unset are 0).  The VVDZ
 * and SSDZ of a column are the vvdz / ssdz arguments of lica_gpu_poisson. */
int lica_grid_metrics(int32_t n, const double* z, double* sdz, double* vdz, double* ssdz, double* vvdz, double* zp);

/* GEOM_COUPLING's z tables (1d.f:5037-5370) between flow faces z[1..n3] (any spacing) and
 * the uniform level-set faces zf[1..n3f] (z[0], zf[0] unused); ZP and ZPF as GEOMETRIC and
 * GEOMETRIC_LVS compute them.  KCOU1/KCOU2(K) of flow face K and KCOUMP1/KCOUMP2(K) of flow
 * centre K are the refined faces (KF-1, KF) that it coincides with (within 1e-10), or
 * (KF-1, KF-1) with ZF(KF) the first refined face above it; ghosts extrapolated as the
 * reference does.  Outputs: kcou1, kcou2 [n3+4] for K = -1..n3+2 at [K+1]; kcoump1,
 * kcoump2 [n3+3] for K = -1..n3+1 at [K+1]; kcou_vel, kcoump_vel [n3f+1] for K = 1..n3f
 * at [K] (the flow centre at or below ZF(K), ZPF(K)).  The box of flow cell K runs over
 * refined cells KCOU2(K)..KCOU1(K+1), of face K over KCOUMP2(K-1)..KCOUMP1(K).
 * LICA_BAD_ARG where the reference prints its coupling problem. */
int lica_grid_coupling_z(int32_t n3, const double* z, int32_t n3f, const double* zf, int32_t* kcou1, int32_t* kcou2,
                         int32_t* kcoump1, int32_t* kcoump2, int32_t* kcou_vel, int32_t* kcoump_vel);

/* A pressure system on a wall-normal (y) grid of faces yface[0..ny], stretched, x uniform
 * and periodic: POISSON's operator (1d.f:3535-3541) in 2-D, multiplied by each row's
 * height so that it is symmetric, written as the multigrid's arrays for hy = 1:
 * bx_out = bx dy_j, by_out = by / (centre distance) (top row: by / dy_{ny-1}), f_out =
 * f dy_j.  Solve with lica_mg_create(nx, ny, hx, 1.0, ...); p is the solution of the
 * stretched system. */
int lica_mg_stretched_system(int32_t nx, int32_t ny, const double* yface, const double* bx, const double* by,
                             const double* f, double* bx_out, double* by_out, double* f_out);

/* ------------------------------------------------------------------------------------
 * fld###### restart files of one column (host code, no GPU): the reference's ASCII field
 * file, record for record.  The column is the reference's 1-D case (N1 = N2 = 2, N3 = n+1;
 * N1F = N2F = 3, N3F = 2n+1); each field is written on all its (I, J) replicas and read from
 * I = J = 1.  The band lists are the cells of each layer in ascending K, four replicas each.
 * ---------------------------------------------------------------------------------- */
typedef struct {
    int64_t ihist;                 /* IHIST, the number in the file name */
    int64_t m;                     /* M, the time-step counter (written: scal[2]) */
    double time, dt;               /* TIME, DT (written: scal[1], scal[0]; read: DT_O) */
    double qvol_ori;               /* QVOL_ORI, the flow-rate reference of ICH = 1 runs */
    int32_t ips, ipx, ipy, ipz;    /* IPS (1: PRM, SCR, TCR and T follow), IPX, IPY, IPZ */
    double pra;                    /* PRA = PRM (read only) */
    double denr, visr, fr, surf_j, fk, re_air; /* FORMAT 1012 (written: props, and fk) */
    double prm, scr, tcr;          /* FORMAT 1006 (read only; written from props) */
    int32_t n_max;                 /* N_MAX, band layers listed (read only; written: 11) */
    int32_t contact, contact_old, lvson;           /* the level set's contact state */
    double vol_tot_ori;            /* VOL_TOT_ORI (read only; written: scal[3]) */
    double contact_start, contact_time, t_con;
} lica_fld_info;

/* lica.in switches applied after a read. */
typedef struct {
    int32_t ireset; /* IRESET = 1: TIME starts from 0 in the state (1d.f:175-178); the run's
                       IHIST, the caller's counter, restarts from 0 too (info keeps the file's) */
    int32_t idtold; /* IDTOLD = 1: DT = the file's DT_O, else props->dt0 (1d.f:1080-1085) */
    int32_t ipzero; /* IPZERO = 1: P = 0 after the read (1d.f:1055) */
} lica_fld_options;

/* The reference's file name for IHIST (1d.f:1155-1163): "fld" and six digits; out gets
 * 10 bytes with the terminating NUL.  LICA_BAD_ARG for IHIST outside 0..999999. */
int lica_fld_name(int64_t ihist, char* out, int32_t cap);

/* WRITEFIELD (1d.f:1121-1232) of one column's host state.  From info: ihist, qvol_ori,
 * ips, ipx, ipy, ipz, fk and the contact fields; the rest comes from props and st. */
int lica_col_fld_write(const char* path, int32_t n, const lica_col_props* props, const lica_col_state* st,
                       const lica_fld_info* info);

/* The column size n (= N3 - 1) of a file; LICA_BAD_ARG if it is not a column. */
int lica_col_fld_dims(const char* path, int32_t* n);

/* PREFLD (1d.f:972-1098) into one column's host state, then the start-up that follows a
 * read: LVSINIT's read branch (two_phase.f:148-205: the band from the lists, ALPHI_BC,
 * CAL_PSIF(1, N_MAX)), GRID_COUPLING(1), VOL_TOT_IPHS = VOL_TOT_ORI, the options above and
 * M = 0 (the time loop starts again at M = 1).  info receives the file's header values. */
int lica_col_fld_read(const char* path, int32_t n, double length, const lica_col_props* props,
                      const lica_fld_options* opt, lica_col_state* st, lica_fld_info* info);

/* Device scratch the step kernel needs for ncol columns of n cells. */
size_t lica_gpu_column_scratch_bytes(int32_t ncol, int32_t n);

/* nsteps time steps of every column; device arrays.  threads: CTA width per column, 32,
 * 64, 128 or 256 (0: 256 for up to one column per SM, else 64); wider CTAs finish one
 * column sooner, narrower ones keep more columns per SM; every width gives the same bits.  scratch: NULL (the library keeps
 * one) or lica_gpu_column_scratch_bytes() of device memory.  status[ncol] (device) gets
 * LICA_OK, LICA_NOT_CONVERGED (TEMP_EXTP did not converge), LICA_BAND_OVERFLOW or
 * LICA_BAD_ARG per column; a column stops at its first non-OK step.  Enqueues on stream. */
int lica_gpu_column_steps_device(int32_t ncol, int32_t n, double length, const lica_col_props* props,
                                 const lica_col_state* st, int32_t nsteps, int32_t threads, void* scratch,
                                 int32_t* status, void* stream);

/* Cycle profile of the step kernel: while prof (device, 11 int64 per column) is set,
 * thread 0 of each column adds the SM cycles spent in each phase -- 0 time-step choice and
 * substep entry, 1 CAL_CONTINUITY + CAL_CONT_BC, 2 energy RHS + LHSPS, 3 TEMP_GRAD without
 * TEMP_EXTP, 4 TEMP_EXTP, 5 CAL_CONTINUITY2 + CAL_CONT_BC, 6 RHSZ, 7 LHSW, 8 BC + FSM_CHOI +
 * PRESSURE_CORRECTION, 9 CONVRGE1, 10 TRANSPORT + GRID_COUPLING.  NULL turns it off. */
int lica_gpu_column_profile_device(int64_t* prof);

/* Interface history of the step kernels (the reference's per-step record of 0interface.dat,
 * chphase.f:1419-1438, and VOL_TOT_IPHS, chphase.f:1457): while hist (device, 4 * capacity
 * doubles per column) is set, every launch of lica_gpu_column_steps_device /
 * lica_gpu_column_batch_steps_device writes for step s < capacity of column c, at
 * hist[4 (c capacity + s) ..]: TIME before the step (the value the reference writes), the
 * interface position `place` of VOL_TOT_MFDOT in the third substep (zpf(k) + |phi(k)| at
 * the last sign change of the trial level set; 0 in a step without phase change), the
 * vapour volume VOL_TOT_IPHS and DT.  NULL turns it off. */
int lica_gpu_column_history_device(double* hist, int32_t capacity);

/* Batches of columns of uneven size, length and properties (one opaque handle per batch
 * layout).  Column c has n[c] flow cells over length[c] with props[c]; its arrays are packed
 * back to back: lica_gpu_column_batch_layout gives per column the offsets (in elements) of
 * its flow arrays (w, p, t, psi_cn, psi_zn, wo, imask), its phi-like arrays (phi, layer,
 * mflvs) and its psif-like arrays (psif, sfgas, sfgas2): offsets[3c .. 3c+2]; and the
 * totals: totals[0..2] elements of each kind, totals[3] scratch bytes.  scal and stats
 * stay 5 and 8 per column.  The kernel runs the longest columns first. */
typedef struct lica_col_batch lica_col_batch;
int lica_gpu_column_batch_create(lica_col_batch** out, int32_t ncol, const int32_t* n, const double* length,
                                 const lica_col_props* props);
int lica_gpu_column_batch_destroy(lica_col_batch* batch);
int lica_gpu_column_batch_layout(const lica_col_batch* batch, int64_t* offsets, int64_t* totals);
int lica_gpu_column_batch_steps_device(const lica_col_batch* batch, const lica_col_state* st, int32_t nsteps,
                                       int32_t threads, void* scratch, int32_t* status, void* stream);
/* The same with a limit on the column length whose Thomas arrays live in shared memory
 * (tri_cap < 0: as large as the CTAs per SM allow, the default; 0: all in scratch; the arithmetic
 * and results are the same either way) -- the launch autotuner's second axis. */
int lica_gpu_column_batch_steps_ex_device(const lica_col_batch* batch, const lica_col_state* st, int32_t nsteps,
                                          int32_t threads, int32_t tri_cap, void* scratch, int32_t* status,
                                          void* stream);

/* Same on host arrays (copies in, runs, copies out); returns the last non-OK column status. */
int lica_gpu_column_steps(int32_t ncol, int32_t n, double length, const lica_col_props* props,
                          lica_col_state* st, int32_t nsteps, int32_t* status);

/* Stretched columns: a flow grid of n cells on faces Z(1..n+1) (GEOMETRIC, 1d.f:4808-4882;
 * any spacing whose cells are at least one refined cell, length/(2n), wide) under the
 * uniform level-set grid of 2n cells (GEOMETRIC_LVS, 1d.f:4885), coupled by the z tables of
 * GEOM_COUPLING (1d.f:5037-5370).  Host arrays, Fortran index as offset:
 *   z, zp, sdz, vdz, ssdz, vvdz : n+2 doubles, k = 0..n+1 (z[k] = Z(k), z[0] unused)
 *   kcou1, kcou2               : n+5 int32, K = -1..n+3 at [K+1]
 *   kcoump1, kcoump2           : n+4 int32, K = -1..n+2 at [K+1]
 *   kcou_vel, kcoump_vel       : 2n+2 int32, k = 0..2n+1 at [k]
 * (lica_grid_metrics and lica_grid_coupling_z produce them).  Every routine of the step
 * that the uniform column evaluates in closed form -- CAL_DENVIS's upwind boxes, the
 * GRID_COUPLING boxes, PHINSINTP, VEL_INTP, TEMP_GRAD's flow lookups, the metric factors --
 * reads these instead. */
typedef struct {
    const double *z, *zp, *sdz, *vdz, *ssdz, *vvdz;
    const int32_t *kcou1, *kcou2, *kcoump1, *kcoump2, *kcou_vel, *kcoump_vel;
} lica_col_geometry;

/* lica_gpu_column_init on a stretched column (MAKEFLD's profile at ZP, GRID_COUPLING(1)'s
 * boxes from the tables); LICA_BAD_ARG for a geometry that does not rise from 0 to length,
 * has a cell narrower than a refined cell, or a table entry outside the grid. */
int lica_gpu_column_init_geometry(int32_t n, double length, double z0, const lica_col_props* props,
                                  const lica_col_geometry* geo, lica_col_state* st);

/* A checked device copy of a geometry (the same checks); every column of the steps below
 * is that column. */
typedef struct lica_col_geo lica_col_geo;
int lica_gpu_column_geometry_create(lica_col_geo** out, int32_t n, double length, const lica_col_geometry* geo);
int lica_gpu_column_geometry_destroy(lica_col_geo* geo);

/* lica_gpu_column_steps_device / lica_gpu_column_steps for ncol stretched columns of the
 * geometry's n and length. */
int lica_gpu_column_steps_geometry_device(const lica_col_geo* geo, int32_t ncol, const lica_col_props* props,
                                          const lica_col_state* st, int32_t nsteps, int32_t threads, void* scratch,
                                          int32_t* status, void* stream);
int lica_gpu_column_steps_geometry(const lica_col_geo* geo, int32_t ncol, const lica_col_props* props,
                                   lica_col_state* st, int32_t nsteps, int32_t* status);

/* lica_gpu_lvs_transport[_device] on ncol stretched columns of the geometry's n and length:
 * VEL_INTP's 4-point stencil on the stretched flow faces (KCOU_VEL), GRID_COUPLING(0)'s
 * boxes from the tables. */
int lica_gpu_lvs_transport_geometry_device(const lica_col_geo* geo, int32_t ncol, double* phi, int32_t* layer,
                                           double* psif, double* wo, const double* w, const double* mflvs,
                                           double* vol_tot_ori, const double* vol_tot_iphs, double* psi_cn,
                                           double* psi_zn, int32_t* status, double* stats, const lica_lvs_params* prm,
                                           void* stream);
int lica_gpu_lvs_transport_geometry(const lica_col_geo* geo, int32_t ncol, double* phi, int32_t* layer, double* psif,
                                    double* wo, const double* w, const double* mflvs, double* vol_tot_ori,
                                    const double* vol_tot_iphs, double* psi_cn, double* psi_zn, int32_t* status,
                                    double* stats, const lica_lvs_params* prm);

int lica_gpu_lvs_transport_device(int32_t ncol, int32_t n, double length, double* phi, int32_t* layer,
                                  double* psif, double* wo, const double* w, const double* mflvs,
                                  double* vol_tot_ori, const double* vol_tot_iphs, double* psi_cn,
                                  double* psi_zn, int32_t* status, double* stats, const lica_lvs_params* prm,
                                  void* stream);

/* ------------------------------------------------------------------------------------
 * Single subroutines of the step, for a host that replaces the reference's routines one at
 * a time.  Batches of ncol columns of n flow cells over length, in the column layout of
 * lica_col_state (flow arrays n+2 per column, phi-like nf+7 at k+2, psif-like nf+2 at k).
 * Host arrays (copied in and out) or, with _device, device arrays and a stream (enqueues
 * and returns).  Each runs the same device code as the fused step, so a sequence of them
 * gives the step's results bit for bit.
 * ---------------------------------------------------------------------------------- */

/* REINITIALIZATION(NN1, NN2, ILIMIT, LLVS) (two_phase.f:2033-2474; called from TRANSPORT,
 * two_phase.f:906,928, and VOL_TOT_MFDOT, chphase.f:1415): ILIMIT SSP-RK3 pseudo-time
 * iterations of the Sussman/Peng reinitialisation with dtau = h_f/2 on the band layers
 * 1..NN2 = 1..N_MAX-1 (HJ-WENO5 on 1..NN1 = 1..N_MAX-3, first order beyond).  phi is
 * ALPHI_EXT as the caller holds it (every cell is read; the reference's call sites hold it
 * zero off the band), layer the band (cell k in layer m = 1..N_MAX, 0 off the band); only
 * the band cells of phi are written.  status[ncol]: LICA_OK, LICA_BAND_OVERFLOW (the band
 * spans more than 112 refined cells; phi unchanged) or LICA_BAD_ARG (a band cell outside
 * k = 1..nf). */
int lica_gpu_reinitialization(int32_t ncol, int32_t n, double length, double* phi, const int32_t* layer,
                              int32_t ilimit, int32_t* status);
int lica_gpu_reinitialization_device(int32_t ncol, int32_t n, double length, double* phi, const int32_t* layer,
                                     int32_t ilimit, int32_t* status, void* stream);

/* GRID_COUPLING(INI_PSI, PSI_XN, PSI_YN, PSI_ZN, PSI_CN) (two_phase.f:4863-5118; called from
 * MAIN, 1d.f:244, and LVSINIT): the flow-grid liquid fractions from PSIF by box integrals
 * over the refined cells (INTER_PSI), snapped at 1e-3 / 0.999.  ini_psi = 1: every flow
 * cell; 0: the flow cells of the band cells of layers 1..NN1 (layer may be NULL with
 * ini_psi = 1).  psi_cn, psi_zn are updated in place (cells the mask leaves are only
 * snapped).  PSI_XN and PSI_YN are zero in the 1-D column. */
int lica_gpu_grid_coupling(int32_t ncol, int32_t n, double length, int32_t ini_psi, const double* psif,
                           const int32_t* layer, double* psi_cn, double* psi_zn);
int lica_gpu_grid_coupling_device(int32_t ncol, int32_t n, double length, int32_t ini_psi, const double* psif,
                                  const int32_t* layer, double* psi_cn, double* psi_zn, void* stream);

/* TEMP_GRAD(PSI_CN) (chphase.f:55-368; called from PASSIVE_SCALAR, 1d.f:3667) with the
 * routines it calls -- PHINSINTP, TEMP_EXTP(_RK3), TEMPASSIGN, TF_GRAD, VOL_TOT_MFDOT --
 * and CAL_PSI_TMP(1): reads T, PSI_CN and the band (phi, layer) and the module values
 * DTCONST and the lica.in properties; writes MFLVS (nf+7 per column), SFGAS, SFGAS2
 * (nf+2), IMASK_PH (n+2) and VOL_TOT_IPHS (vol_tot_iphs[ncol], in: the previous value);
 * iterations[ncol] gets the TEMP_EXTP pseudo-time iterations.  status: LICA_OK,
 * LICA_NOT_CONVERGED (TEMP_EXTP's retries ran out) or LICA_BAND_OVERFLOW.  The _device
 * form takes scratch (NULL: the library's) of lica_gpu_column_scratch_bytes(ncol, n). */
int lica_gpu_temp_grad(int32_t ncol, int32_t n, double length, const lica_col_props* props, double dtconst,
                       const double* t, const double* psi_cn, const double* phi, const int32_t* layer, double* mflvs,
                       double* sfgas, double* sfgas2, int32_t* imask, double* vol_tot_iphs, int32_t* iterations,
                       int32_t* status);
int lica_gpu_temp_grad_device(int32_t ncol, int32_t n, double length, const lica_col_props* props, double dtconst,
                              const double* t, const double* psi_cn, const double* phi, const int32_t* layer,
                              double* mflvs, double* sfgas, double* sfgas2, int32_t* imask, double* vol_tot_iphs,
                              int32_t* iterations, int32_t* status, void* scratch, void* stream);

/* PRESSURE_CORRECTION(U, V, W, P, DENF_Y, DENF_C, DENF_XI, DENF_YI, DENF_ZI) (1d.f:3403-3488;
 * called from RHSNLHS, 1d.f:1589) of the 1-D column: DIVGS (3180-3303, with the
 * phase-change source from SFGAS when props->iphs = 1, and DTCONST), POISSON (3492-3578),
 * UCALC (3582-3627) and the shift P -= P(1,1,1) with the ghost copies.  W and P (n+2 per
 * column) in place; DENF_ZI (n+2) and SFGAS (nf+2) read.  U, V, DENF_XI, DENF_YI, DENF_Y
 * and DENF_C play no part in the 1-D column. */
int lica_gpu_pressure_correction(int32_t ncol, int32_t n, double length, const lica_col_props* props, double dtconst,
                                 double* w, double* p, const double* denf_zi, const double* sfgas);
int lica_gpu_pressure_correction_device(int32_t ncol, int32_t n, double length, const lica_col_props* props,
                                        double dtconst, double* w, double* p, const double* denf_zi,
                                        const double* sfgas, int32_t* status, void* scratch, void* stream);

/* ---------------------------------------------------------------- learned guess
 * Convolution primitive of the U-Net that supplies the multigrid initial guess (new; the
 * reference has no learned part): 3x3, stride 1, zero padding 1, NHWC BF16 activations,
 * BF16 weights W[cout][9*(c0+c1)] (k = tap*(c0+c1) + channel, tap = 3*dy + dx) with FP32
 * accumulation on the tcgen05 tensor cores.  x1 (c1 channels, may be null with c1 = 0) is
 * concatenated after x0 (c0 channels) along the channels.  The result (+ bias, ReLU when
 * relu != 0) goes to channels [out_c0, out_c0 + cout) of the NHWC tensor out (BF16, out_c
 * channels) and/or out32 (FP32).  c0, c1, cout: multiples of 16 (cout <= 256); the width
 * a multiple of 8, the height of 16.  *err is set to 1 if a bounded wait inside the kernel
 * ran out. */
int lica_unet_conv3x3_device(const void* x0, int32_t c0, const void* x1, int32_t c1, const void* w,
                             const float* bias, int32_t n, int32_t h, int32_t wd, int32_t cout, int32_t relu,
                             void* out, float* out32, int32_t out_c, int32_t out_c0, int32_t* err, void* stream);

/* The U-Net of the learned initial guess (new; no counterpart in the reference).  Input per
 * image: rho and f (row-major h x w, FP64, device); output: the guess x0 of the pressure
 * solve A p = f (FP64; the network's output times rms(f) h^2 rho, h^2 = hsq), which the
 * caller passes to lica_mg_solve_* as the initial iterate
 * (the solver keeps its own tolerance; a guess whose residual exceeds ||f|| should be
 * replaced by zero).  Network: 3 levels of 32/64/128 channels, two 3x3 convolutions with
 * ReLU per level and per decoder level, 2x2 average pooling, nearest upsampling, skip
 * connections, a 1x1 head; BF16 weights and activations, FP32 accumulation on the tcgen05
 * tensor cores (lica_unet_conv3x3_device).  Parameters: FP32 vector, layer by layer
 * (weights [cout][tap][cin], then bias), then the head (32 weights, 1 bias).
 * lica_unet_create: n images of h x w (multiples of 64, >= 64), deterministic He
 * initialisation from seed.  lica_unet_train_step_device: one Adam step on the loss
 * mean_images ||f - A x0||^2 / ||f||^2 with A the solver's operator (face coefficients bx,
 * by as in lica_mg_solve_*), or, given the solver's solutions p_star (A p* = f), on the
 * relative A-norm error (x0 - p*).(-A)(x0 - p*) / p*.(-A)p*; *loss is the loss before
 * the step.  lica_unet_grad_device:
 * parameter gradient of sum(gx0 * x0) (the gradient check). */
typedef struct lica_unet lica_unet;
int lica_unet_create(lica_unet** out, int32_t n, int32_t h, int32_t w, uint64_t seed);
int lica_unet_destroy(lica_unet* net);
int64_t lica_unet_param_count(const lica_unet* net);
int lica_unet_get_params(lica_unet* net, float* host, int64_t count);
int lica_unet_set_params(lica_unet* net, const float* host, int64_t count);
int lica_unet_guess_device(lica_unet* net, const double* rho, const double* f, double hsq, double* x0, void* stream);
/* The guess with its relative residual ||f - A x0|| / ||f|| per image in rel0 (host
 * array of n); an image whose guess is no better than zero gets x0 = 0 (the fallback). */
int lica_unet_guess_checked_device(lica_unet* net, const double* rho, const double* f, const double* bx,
                                   const double* by, double hx, double hy, double* x0, double* rel0, void* stream);
int lica_unet_grad_device(lica_unet* net, const double* rho, const double* f, double hsq, const double* gx0,
                          float* grad_host, int64_t count, void* stream);
int lica_unet_train_step_device(lica_unet* net, const double* rho, const double* f, const double* bx,
                                const double* by, const double* p_star, double hx, double hy, float lr,
                                double* loss, void* stream);

/* ----------------------------------------------------------------------------------
 * 2-D film boiling: one RK3 time step (three substeps and the level-set
 * reinitialisation) on an nx x ny MAC grid (x periodic, Lx = 1, h = 1/nx; heated no-slip
 * wall at the bottom, outflow top with p = 0 on the face) with the level set on the
 * 2 nx x 2 ny refined grid.  Generalises the reference's 1-D step rows to 2-D: RK3COEF
 * (1d.f:1310-1322), RHSZ/LHSW (1603-1809, explicit), PRESSURE_CORRECTION through the 2-D
 * multigrid (lica_mg_*), TEMP_GRAD/TF_GRAD/VOL_TOT_MFDOT (chphase.f) as a smeared mass
 * flux, PASSIVE_SCALAR/TEMPASSIGN, TRANSPORT_RK3 + HJWENO and REINITIALIZATION + GODUNOV
 * (two_phase.f), surface tension by CAL_CUR's curvature as a continuum surface force.
 * Device arrays (row-major, x fastest): u (ny, nx) on the face west of
 * cell i; v (ny + 1, nx) on the face below cell row j (v[0] = 0, v[ny] the top face);
 * p = the modified pressure p + rho_l g y (ny, nx); th = (T - T_sat) / dT_wall (ny, nx);
 * phi (2 ny, 2 nx), liquid where phi > 0.  nx, ny multiples of 32 that halve evenly
 * nlevels - 1 times (the multigrid's rule); precision 0: FP64 pressure solves, 1: mixed.
 * lica_film2d_step_device enqueues on the stream and waits for each pressure solve;
 * returns the first non-OK solve status (LICA_NOT_CONVERGED) or LICA_OK.
 * ---------------------------------------------------------------------------------- */
typedef struct lica_film2d lica_film2d;

typedef struct {
    double re, visr, denr, prm, scr, tcr, jakob, fr; /* Re; liquid/vapour viscosity, density,
                                                        specific-heat and conductivity ratios;
                                                        Pr; Ja; Fr (gravity 1/Fr^2, 0: off) */
    double we;         /* Weber number (surface tension 1/We, 0: off) */
    double rtol;       /* pressure-solve relative residual */
    int32_t max_iters; /* pressure-solve iteration cap */
    int32_t nreinit;   /* reinitialisation iterations after the step */
} lica_film2d_props;

typedef struct {
    int32_t iterations[3];  /* pressure-solve iterations of each substep */
    int32_t status[3];
    double rel_residual[3];
    double guess_rel[3];    /* ||f - A x0|| / ||f|| of the learned guess each solve started
                               from (1 without a guess, or when the guess fell back to zero) */
} lica_film2d_stats;

int lica_film2d_create(lica_film2d** out, int32_t nx, int32_t ny, const lica_film2d_props* props,
                       int32_t nlevels, int32_t precision);
int lica_film2d_destroy(lica_film2d* film);
int lica_film2d_step_device(lica_film2d* film, double* u, double* v, double* p, double* th, double* phi, double dt,
                            lica_film2d_stats* stats, void* stream);
/* Copies the interfacial mass flux per cell of the last substep into out (device, ny x nx). */
int lica_film2d_mdot_device(lica_film2d* film, double* out, void* stream);
/* The learned initial guess of the three pressure solves (new; no counterpart in the
 * reference): net, a U-Net of one ny x nx image (lica_unet_create(&net, 1, ny, nx, ...)),
 * predicts each increment from the substep's density and right-hand side; a guess no
 * better than zero is replaced by zero, and the solve keeps its own tolerance.  NULL
 * detaches it.  The film step does not own net. */
int lica_film2d_set_guess(lica_film2d* film, lica_unet* net);
/* Warm start of the pressure solves (new; the reference solves from zero): with on = 1,
 * each substep's increment starts from the increment the same RK3 substep solved in the
 * previous step (zero in the first step after the call), which leaves a relative residual of
 * about 0.2-0.5 on a developing film and saves about one MG-PCG iteration in ten; the solve
 * keeps its tolerance.  The learned guess, when attached, takes precedence.  on = 0 turns it
 * off; either call forgets the kept increments. */
int lica_film2d_set_warm_start(lica_film2d* film, int32_t on);
/* Training pairs from the film's own solves: while systems (device) is set, every step
 * writes for substep k = 0..2, at systems + k (4 nx ny + (ny + 1) nx): the density (ny x nx),
 * the right-hand side f, bx (ny x nx), by ((ny + 1) x nx) and the solved increment dp.  NULL
 * turns it off. */
int lica_film2d_capture_device(lica_film2d* film, double* systems);

/* ------------------------------------------------------------------------------------
 * Bubble statistics of several level sets on a 3-D grid: BUBBLE_TRACKING(LLVS, PSI_TMP,
 * U, V, W) (two_phase.f:6321-6555) with BUBBLE_EIGENV (6558-6705) and Jacobi_bub
 * (two_phase.f:19-97), for level sets llvs0 .. llvs0 + nlvs - 1 in one call.  Per level
 * set: the gas volume VOL = sum (1 - PSI_TMP) SDX SDY SDZ over the cells with PSI_TMP != 1,
 * the volume-weighted centroid and cell-centred velocity, the second moment of the gas
 * volume about the centroid, its eigenvalues by cyclic Jacobi rotations (threshold 1e-12),
 * the aspect ratio sqrt(largest / smallest) and the angles (degrees, folded into [0, 90])
 * of the smallest eigenvalue's axis to x and to z.  With ipz = 1 and gas in the top cell
 * plane K = N3M (IZ_PERIODIC), cells in the lower half (ZP <= ZL/2) count at ZP + ZL.
 * The reference runs it in substep MSUB = 3 only; the caller decides when to call.
 *
 * Grid (Fortran index as offset, lower bound 0): sdx, xp n1m+2 doubles (SDX(0:N1),
 * XP(0:N1)), likewise sdy, yp (n2m+2) and sdz, zp (n3m+2); cell I = 1..N1M uses SDX(I),
 * XP(I).  ipx, ipy, ipz: periodic directions (IPV(N1M) = 1 when ipx, else N1).
 * Fields U, V, W, PSI_TMP(0:N1, 0:N2, 0:N3), column-major: (i, j, k) at
 * i + (n1m+2) (j + (n2m+2) k); psi_tmp holds nlvs such fields back to back.
 * icacy 1: the record holds x, y, z and u, v, w; 2: r, theta, z and u_r, u_theta, w.
 *
 * The GPU computes each level set's moments in one pass over the fields (a weighted
 * Welford update per gas cell, merged by Chan's rule in a fixed order), where the
 * reference sums twice; the results agree to rounding.  An empty level set (VOL = 0)
 * gives zero centroid, velocity and moments, ar = NaN (0/0) and angles 90 and 0, which
 * is what the reference's formulas give from a zero moment. */
typedef struct {
    int32_t n1m, n2m, n3m;      /* cells per direction (N1M, N2M, N3M) */
    int32_t ipx, ipy, ipz;      /* periodic directions (IPX, IPY, IPZ) */
    double zl;                  /* ZL, the z period */
    const double *sdx, *sdy, *sdz, *xp, *yp, *zp;
} lica_bub_grid;

typedef struct {
    double time;
    int64_t llvs;
    double col[9];        /* the record of 0bub_tracking.dat after TIME and LLVS (FORMAT
                             1ES15.7, 1I5, 9ES15.7; two_phase.f:6440-6443, 6539-6542) */
    double vel[3];        /* VELVS(LLVS, 1:3) = UU, VV, WW (two_phase.f:6547-6549) */
    double vol;           /* VOL */
    double ami[3];        /* eigenvalues AMI(1,1), AMI(2,2), AMI(3,3) after Jacobi_bub */
    int64_t iz_periodic;  /* IZ_PERIODIC */
} lica_bub_record;

/* A device copy of the grid with room for max_lvs (1..65535) level sets per call;
 * LICA_BAD_ARG for a size below 1, a field of 2^31 or more doubles, or a cell width that
 * is not positive. */
typedef struct lica_bub_geo lica_bub_geo;
int lica_gpu_bubble_grid_create(lica_bub_geo** out, const lica_bub_grid* grid, int32_t max_lvs);
int lica_gpu_bubble_grid_destroy(lica_bub_geo* geo);
/* Device arrays and a stream (enqueues and returns; one call at a time per geo); out is a
 * device array of nlvs lica_bub_record. */
int lica_gpu_bubble_tracking_device(lica_bub_geo* geo, int32_t nlvs, int32_t llvs0, const double* psi_tmp,
                                    const double* u, const double* v, const double* w, double time, int32_t icacy,
                                    void* out, void* stream);
/* Host arrays (copies in, runs, copies out); out[nlvs]. */
int lica_gpu_bubble_tracking(const lica_bub_grid* grid, int32_t nlvs, int32_t llvs0, const double* psi_tmp,
                             const double* u, const double* v, const double* w, double time, int32_t icacy,
                             lica_bub_record* out);

#ifdef __cplusplus
}
#endif

#endif /* LICA_GPU_H */
