/*
 * lag2d.h -- C-ABI of the B200 Lagrangian DG time step (Lag2D, curved P2).
 *
 * The reference has no FFI: its seam is the Fortran subroutine
 *   getsolvdg_lag(intfac, inpoel, iptri, ipqua, bface, cooro, coord, coora,
 *                 geofa, geoel, gesgt0, gesgq0, uchar, unkno, unold, unkaw,
 *                 unkgd, unogd, strnq_devtp, ltelem, estri, esqua, itime,
 *                 amatr, amagd, ustar, coold, esuv1, esuv2)
 * (srccurv-lag/Getrhslag.f90:1553-1555), called once per time step from the
 * driver loop (srccurv-lag/dgflo2d.f90:372-373), with the inner seams
 * getrhsdg_lag_mcnew (Getrhslagmc.f90:6693), getcellvol_lag
 * (Limiterlag.f90:1869) and getdelt_lag (Getrhslag.f90:20600).
 *
 * Every entry point is bind(C)-compatible: plain ints, doubles and pointers.
 * Arrays use the Fortran layouts (column-major, 1-based ids):
 *   unkno(ndegr, nq, nsize), coord(2, npoin), ustar(2, npoin),
 *   geoel(24, nsize), amatr(nmatr, ncell), ipqua(9, nquad), iptri(6, ntria),
 *   bface(5, nbfac), esqua(4, nquad), esuv1(npoin1), esuv2(npoin+1).
 * The caller owns host buffers; the library owns device buffers.  One CUDA
 * stream per handle; calls on one handle are not thread-safe.  Every call
 * returns LAG2D_OK (0) or a status code; lag2d_last_error() gives text.
 */
#ifndef LAG2D_H
#define LAG2D_H

#ifdef __cplusplus
extern "C" {
#endif

#define LAG2D_OK 0
#define LAG2D_EINVAL 1      /* bad argument or array size */
#define LAG2D_ECUDA 2       /* CUDA runtime error (message in lag2d_last_error) */
#define LAG2D_EUNSUP 3      /* configuration outside the built path */
#define LAG2D_ENONPHYS 4    /* non-positive cell volume or NaN in the state */
#define LAG2D_ESTENCIL 5    /* WENO vertex valence the reference rejects (WENO.f90:7699) */
#define LAG2D_ENODEV 6      /* no usable CUDA device */

typedef struct lag2d_handle lag2d_handle;

/* Mesh arrays as preprocess1/preprocess2 leave them (Preprocess.f90:4-1009)
 * and getesuel produces them (dgflo2d.f90:1220-1309). */
typedef struct {
  int ntria, nquad, npoin, nbfac;
  const int *iptri;     /* iptri(6, ntria)   1-based node ids            */
  const int *ipqua;     /* ipqua(9, nquad)   1-based node ids            */
  const int *bface;     /* bface(5, nbfac)   n1, n2, code, sub-code, mid */
  const int *esuv1;     /* esuv1(npoin1)     cells surrounding points    */
  const int *esuv2;     /* esuv2(npoin+1)    CSR offsets, esuv2(1) = 0   */
  const int *esqua;     /* esqua(4, nquad)   face neighbours / ghost ids */
  const double *coold;  /* coold(2, npoin)   initial coordinates         */
} lag2d_mesh;

/* The module-constant knobs the step reads (dgflo2d.f90:4-56). */
typedef struct {
  int npoly, ndegr, mdegr, nq;
  int nstag;            /* 2 or 3 (SSP-RK2/3)                            */
  int ndt;              /* 1: CFL dt (getdelt_lag), 0: fixed dtfix       */
  int ncase;            /* initial-condition / source case               */
  int nlimi, ndens;
  int ngausd, ngausd_geo;
  int precision;        /* 0: FP64; 1: FP32-mixed corner/RHS arithmetic  */
  int order_exact;      /* 1: kernels that keep the reference's loop and
                           summation order (bit-identical to the CPU
                           restatement in the no-FMA build); 0: optimised */
  int nsedov;           /* number of Sedov energy cells (<= 4)           */
  int sedov_cell[4];    /* their 1-based ids                             */
  double gamlg, cfl, cdrho, cimpd, tend, sedov_energy;
  int nrz;              /* 0: Cartesian; 1: RZ (true volume, axis y = 0);
                           2: area-weighted RZ; both built on the P1 path
                           (npoly = 1)                                     */
} lag2d_config;

/* Create a handle: validates the mesh, builds the device connectivity
 * (node-to-corner gather lists, WENO stencils, boundary node masks) and
 * allocates device state.  Replaces the array set-up the Fortran driver does
 * before its time loop (dgflo2d.f90:61-350). */
int lag2d_create(const lag2d_mesh *mesh, const lag2d_config *cfg, lag2d_handle **out);

/* Initial geometry, mass matrix and DOFs computed on the device:
 * getgeoel_initial_lag + getgeoelho_initial_lag (GetInitial.f90:1278,1704),
 * inifield_mcnew (Getrhslagmc.f90:3293) and getunkno_initial_lag
 * (GetInitial.f90:151).  Sets the device state to it (coord = coold,
 * ustar = 0) and copies geoel, amatr, unkno to the host pointers that are
 * not NULL. */
int lag2d_init_fields(lag2d_handle *h, double *geoel, double *amatr, double *unkno);

/* Initial-condition hook: rho0(ncell) multiplies the initial density of each
 * cell (getrhog_initial and the density of getunkin; pressure and velocity
 * unchanged), so it enters the cell and sub-cell masses, the mass matrices
 * and the initial DOFs that lag2d_init_fields computes, and the reference
 * density of the physical mass centres.  Call before lag2d_init_fields;
 * NULL restores the case's own density.  Values must be positive.  No
 * counterpart in the reference, which reads the density from its case
 * tables only. */
int lag2d_set_rho0(lag2d_handle *h, const double *rho0);

/* Upload a state: unkno(ndegr,nq,nsize), coord(2,npoin), ustar(2,npoin),
 * geoel(24,nsize) (fields 1-4 and 19-21 are read), amatr(nmatr,ncell).
 * geoel/amatr may be NULL to keep the device copies. */
int lag2d_set_state(lag2d_handle *h, const double *unkno, const double *coord,
                    const double *ustar, const double *geoel, const double *amatr);

/* One time step: getsolvdg_lag (Getrhslag.f90:1553-2035) followed by the
 * driver's copy of unold into unkno and cooro into coord
 * (dgflo2d.f90:407-423).  dtfix and tacru are the driver's mutable module
 * scalars (in/out).  Synchronises the handle's stream. */
int lag2d_step(lag2d_handle *h, int itime, double *dtfix, double *tacru);

/* nsteps steps of the driver loop (dgflo2d.f90:358-472) with no host
 * synchronisation in between; stops early (on the device) once
 * |tacru - tend| / tend <= 1e-11 as the driver does (dgflo2d.f90:459).
 * *done receives the number of steps taken.  Captured in a CUDA graph. */
int lag2d_run(lag2d_handle *h, int itime0, int nsteps, double *dtfix, double *tacru, int *done);

/* Download the state; any pointer may be NULL. geoel(24,nsize) receives the
 * device geometry (fields 1-4, 19-21 and the current volume centre 5-6). */
int lag2d_get_state(lag2d_handle *h, double *unkno, double *coord, double *ustar, double *geoel);

/* getrhsdg_lag_mcnew (Getrhslagmc.f90:6693-8732, curved branch 7556-7710)
 * on the current device state with ustar as the previous nodal velocity:
 * limits unkno in place on the device, updates ustar, writes
 * rhsel(ndegr,nq,ncell) and the Persson marks flags(ncell) (either may be
 * NULL).  For per-stage parity checks. */
int lag2d_rhs(lag2d_handle *h, int itime, double *rhsel, int *flags);

/* weno_char_quad_orthgl (WENO.f90:5927) on the cells with flags(ie) != 0,
 * applied to the device state.  For limiter parity checks. */
int lag2d_weno(lag2d_handle *h, const int *flags);

/* The WENO reconstruction of the handle's current state, linearised with its
 * active set frozen (Persson marks, stencils, nonlinear weights, velocity
 * frame and characteristic matrices held at their values for that state):
 * the map M with M(v) = v except on the quads WENO replaces, whose moments
 * 2..ndegr become the frozen reconstruction of v's stencil DOFs.  transpose =
 * 0 writes out = M(in), 1 writes out = M^T(in); in and out have the layout
 * of unkno(ndegr,nq,nsize) (ghost entries of out are zeroed).  M(unkno) is
 * the reconstruction itself; M^T is what the adjoint applies per RK stage.
 * No counterpart in the reference (it has no adjoint). */
int lag2d_weno_linear(lag2d_handle *h, int transpose, const double *in, double *out);

/* getcellvol_lag (Limiterlag.f90:1869) on the device coordinates; returns
 * geoel(24,nsize) with fields 3, 5, 6 refreshed if geoel is not NULL. */
int lag2d_cellvol(lag2d_handle *h, double *geoel);

/* geterror_lag_curvhybrid (Postprocess.f90:3587-4143): the L2 errors of the
 * handle's state against the exact solution, 25-point Gauss on the current
 * coordinates, errl2[3] = sqrt of the integrals of the squared errors of
 * (rho, |u|, p) for ncase 1 (Taylor-Green) or (rho, e_int, p) for ncase 2
 * (shockless Noh).  The reference prints these at the end of a run.  P2
 * all-quad meshes; other cases, triangles and the P1 path return
 * LAG2D_EUNSUP.  The sum over cells is a fixed-order reduction. */
int lag2d_error_norms(lag2d_handle *h, double *errl2);

/* End-of-run cell values of the reference's post-processing, from the
 * handle's state (cell averages U^n and the current nodes): cellout(9, ncell)
 * = (radius of the cell centre, rho, p, e_int, x_c, y_c, |u|, u, v) per
 * cell, the values geterror_lag_curvhybrid (Postprocess.f90:3700-3717,
 * :3944-3983) and geterror_lag_hybrid (:3515-3560) write to their radial
 * profile files and getoutput_cellvtk (:1258-1398) writes as cell data; the
 * centre is the map at (0, 0) for quads and at (rc, sc) for triangles.
 * badcell(ncell), if not NULL, receives the troubled-cell marker of a
 * Persson pass on the state (getSIHO_Persson, Limiterlag.f90:12042-12239;
 * 100 or 0, as the driver computes it before the VTK file,
 * dgflo2d.f90:525-528), 0 on triangles and on the P1 path. */
int lag2d_cell_output(lag2d_handle *h, double *cellout, double *badcell);

/* The handle's CUDA stream (a cudaStream_t), for callers that time or
 * order work against the library's launches. */
void *lag2d_stream(const lag2d_handle *h);

/* Number of this library's kernel launches since the handle was created. */
long long lag2d_kernel_launches(const lag2d_handle *h);

/* Average device time (ms) per launch of the named kernel family over the
 * launches timed since lag2d_timing(h, 1); families: "corner", "node",
 * "rhs", "update", "persson", "weno", "nodes", "geom", "dt".  Returns -1
 * when timing is off or the family is unknown. */
int lag2d_timing(lag2d_handle *h, int enable);
double lag2d_kernel_ms(const lag2d_handle *h, const char *family, long long *launches);

/* ---------------------------------------------------------------------------
 * Adjoint of the time step.  No counterpart in the reference (it has no
 * adjoint); both entry points differentiate what lag2d_step computes (quads
 * and triangles) with order_exact 0 (order_exact 1 returns LAG2D_EUNSUP).
 * With precision 1 the forward passes are the FP32-mixed ones and the reverse
 * runs its volume-integral and sub-cell-mass transposes in FP32 (the
 * FP32-mixed adjoint); precision 0 is FP64 throughout.  Reverse mode per RK
 * stage with these held fixed: the time step size of each step (ndt == 1
 * picks it on the forward pass; the gradient treats it as a constant), the
 * Persson marks, the WENO reconstruction's active set (stencils, nonlinear
 * weights, velocity frame and characteristic matrices taken at each stage's
 * input: the reconstruction is differentiated as the linear map
 * lag2d_weno_linear describes, with no sensitivity through the node
 * positions), and the reference-configuration quantities (geoel fields 1-4
 * and 19-21, amatr, the initial sub-cell masses).  Marked cells whose
 * stencil is rejected keep their DOFs and are differentiated as such; a
 * window in which the step reports LAG2D_ESTENCIL (a troubled quad left
 * unlimited) is differentiated all the same and returns LAG2D_ESTENCIL with
 * every output written.  More than 16384 WENO-limited quads in one stage
 * return LAG2D_EUNSUP.  Gradients use the
 * layouts of lag2d_set_state: unkno(ndegr,nq,ncell), coord(2,npoin),
 * ustar(2,npoin).
 * ------------------------------------------------------------------------- */

/* One step with its adjoint: from the handle's state (the step's input) runs
 * lag2d_step(h, itime, dtfix, tacru), leaving the handle at the step's output,
 * and returns the gradients of <seed, output> with respect to the input
 * state.  Any seed pointer may be NULL (zero seed); any grad pointer may be
 * NULL (not returned). */
int lag2d_adjoint_step(lag2d_handle *h, int itime, double *dtfix, double *tacru,
                       const double *seed_unkno, const double *seed_coord,
                       const double *seed_ustar, double *grad_unkno, double *grad_coord,
                       double *grad_ustar);

/* nsteps steps from the handle's state with the gradient of the final kinetic
 * energy J = 1/2 sum_c m_c (u_c^2 + v_c^2) (m_c = geoel field 4, u_c and v_c
 * the cell averages unkno(1,2,c), unkno(1,3,c)) with respect to the initial
 * unkno, coord and ustar.  Checkpoints are taken every checkpoint_every steps;
 * each segment is recomputed once on the reverse sweep, so device memory is
 * (nsteps / checkpoint_every + 1) states plus checkpoint_every steps of RK
 * stage inputs.  dtfix and tacru are in/out as in lag2d_step; the handle ends
 * at the final state.  ms[3] (may be NULL) receives the device time of the
 * forward pass, of the segment recomputes and of the reverse sweep. */
int lag2d_adjoint(lag2d_handle *h, int itime0, int nsteps, int checkpoint_every, double *dtfix,
                  double *tacru, double *J, double *dJ_dunkno, double *dJ_dcoord,
                  double *dJ_dustar, double *ms);

/* ---------------------------------------------------------------------------
 * Allocation-free time-step size.  No counterpart in the reference: it is an
 * addition of this library, computing what getdelt_lag (Getrhslag.f90:
 * 20600-20716) computes, for callers that cannot allocate device memory.
 *
 * Which callers need it: every other entry point works on a handle whose
 * device buffers lag2d_create allocated.  A host code that owns a fixed
 * device arena and forbids the CUDA allocator after start-up, a step loop
 * that must not synchronise the device (cudaMalloc and cudaFree may), or a
 * caller that keeps its state in device memory in the reference's layouts
 * and has no handle, can call this one: it calls no cudaMalloc, cudaFree or
 * other allocating routine.  Its only scratch (per-block minima of the
 * reduction) is a fixed array in the library's own device memory, sized for
 * LAG2D_DELT_NOALLOC_MAX_QUADS quads (256 KiB); larger meshes are rejected
 * with LAG2D_EINVAL.  Nothing in that scratch has to start at zero.
 *
 * Arguments: ntria, nquad, npoin, nvqua, ndegr, nq, ngeel are the
 * reference's dimensions and ncurv its geometry knob: ncurv = 0 takes the
 * edge lengths between the 4 corner nodes (straight quads, nvqua >= 4, e.g.
 * the linear P1 path's ipqua(4,nquad)); ncurv >= 1 takes corner - mid-edge
 * node - corner over nodes 1..8 (curved quads, nvqua >= 8, e.g.
 * ipqua(9,nquad)); other combinations are rejected with LAG2D_EINVAL.  Every
 * array is a DEVICE pointer in the reference's layout: ipqua(nvqua,nquad)
 * 1-based, unkno(ndegr,nq,nsize) (the stage-1 state after
 * limiting), geoel(ngeel,nsize) (geoel(3,:) = cell volume), coord(2,npoin)
 * (positions at the start of the step), dvdt(ncell) = rhsel(1,1,:) of stage
 * 1.  itime == 1 gives dtfix = min(cfl dtcfl, 0.1 dtvol); otherwise the
 * previous *dtfix also bounds it by 1.01 dtfix.  dtfix is a device pointer
 * (in/out); it receives NaN if a node id lies outside 1..npoin.  ndens
 * selects how unkno(1,1,:) is read (1: tau, 2/3: density).  The work is
 * queued on `stream` (a cudaStream_t; NULL = the default stream) and the call
 * returns without synchronising.
 *
 * Set-up: every call looks up the scratch address on the current device
 * (so a device reset between calls is harmless); the first call on each
 * device (with that device current) also loads the kernels, so make one call
 * per device before any stream capture begins.  Concurrency: the scratch is one array per
 * device, so calls that may overlap on the same device (different streams or
 * host threads with no order between them) race and give wrong results:
 * serialise them.
 * ------------------------------------------------------------------------- */
#define LAG2D_DELT_NOALLOC_MAX_QUADS 4194304
int lag2d_delt_noalloc(int ntria, int nquad, int npoin, int nvqua, int ncurv, int ndegr, int nq,
                       int ngeel, const int *ipqua, const double *unkno, const double *geoel,
                       const double *coord, const double *dvdt, int itime, int ndens,
                       double gamlg, double cfl, double *dtfix, void *stream);

void lag2d_destroy(lag2d_handle *h);
const char *lag2d_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
