/*
 * Lag2D CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A single-threaded FP64 C restatement of the reference Fortran time step
 * (cell-centred Lagrangian DG, curved 9-node quads and 6-node triangles, P2 Taylor basis, the
 * ncurv=1 / nriem=1 / nfint=4 branch).  It exists to check the CUDA product
 * path and to serve as the timed CPU baseline; nothing in the product
 * library links or calls it.
 *
 * Parity pin: the reference is Fortran 90 and no Fortran compiler exists in
 * this environment, and the reference ships no tests, inputs or golden
 * outputs.  This restatement is therefore "parity unpinned" against the
 * reference binary; it is pinned instead by quadrature exactness checks,
 * free-stream preservation, exact per-cell mass conservation and total
 * energy conservation (tests/test_oracle.py), and by golden fixtures it
 * generated itself (tests/golden/).
 *
 * Storage follows the Fortran arrays exactly (column-major, flattened),
 * with 0-based offsets and 1-based ids stored in the integer arrays:
 *   unkno(ndegr, nq, nsize)  -> U[id + ndegr*(iq + nq*ie)]
 *   coord(2, npoin)          -> X[d + 2*ip]
 *   geoel(24, nsize)         -> G[k + 24*ie]
 *   amatr(nmatr, ncell)      -> A[k + nmatr*ie]
 *   ipqua(9, nquad)          -> 1-based node ids, node index fastest
 *                               (ipqua(4, nquad) on the straight-quad P1 path)
 *   bface(5, nbfac)          -> (node1, node2, bc code, bc sub-code, mid node)
 *   esuv1 / esuv2            -> cells-surrounding-point CSR (1-based)
 *   esqua(4, nquad)          -> cell across quad face k (ghost = ncell+iface)
 */
#ifndef LAG2D_ORACLE_H
#define LAG2D_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int ntria, nquad, npoin, nbfac;
  const int *iptri;  /* (6, ntria)  */
  const int *ipqua;  /* (9, nquad)  */
  const int *bface;  /* (5, nbfac)  */
  const int *esuv1;  /* (npoin1)    */
  const int *esuv2;  /* (npoin+1)   */
  const int *esqua;  /* (4, nquad)  */
  int nvqua;         /* nodes per quad in ipqua: 9 (curved, ncurv=1) or 4 (straight, ncurv=0) */
} o_mesh;

typedef struct {
  int npoly, ndegr, mdegr, nq;
  int nstag, ndt, ncase, nlimi, ndens;
  int ngausd, ngausd_geo;      /* triangle rules (ctrl file) */
  int sedov_ncell, sedov_cell[4];  /* 1-based ids that receive the Sedov energy */
  double gamlg, cfl, cdrho, cimpd, tend;
  double sedov_energy;         /* 0.244816 in the reference */
  const double *rho0;          /* (ncell) initial-density factor per cell, or NULL (1) */
  int nrz;                     /* 0: Cartesian; 1: RZ, y the radius (P1 path only) */
} o_cfg;

/* Initial geometry, mass matrix and DOFs: getgeoel_initial_lag,
 * getgeoelho_initial_lag, inifield_mcnew, getunkno_initial_lag. */
void o_init(const o_mesh *m, const o_cfg *c, const double *coord,
            double *geoel, double *amatr, double *unkno);

/* getcellvol_lag: geoel(3,5,6) at the given coordinates. */
void o_cellvol(const o_mesh *m, const o_cfg *c, double *geoel, const double *coord);

/* getrhsdg_lag_mcnew (curved P2 branch).  unkno is limited in place,
 * ustar is overwritten with the new nodal velocity, rhsel is written,
 * flags (optional, ncell) receives the Persson troubled-cell marks. */
void o_rhs(const o_mesh *m, const o_cfg *c, double *ustar, double *unkno,
           double *rhsel, double *geoel, const double *coord,
           const double *coold, const double *amatr, int itime, int *flags);

/* Test bookkeeping (no counterpart in the reference): the number of quads
 * Persson marked troubled and of quads whose DOFs WENO replaced since the
 * previous call; resets both. */
void o_counts(long long *marked, long long *replaced);

/* weno_char_quad_orthgl on the cells with flags[ie] != 0. */
void o_weno(const o_mesh *m, const o_cfg *c, double *unkno, double *geoel,
            const double *coord, const double *coold, const int *flags);

/* Status bits since the last call (2: WENO stencil rejected, where the
 * reference stops); reading clears them. */
int o_status(void);

/* getdelt_lag: returns the new dtfix. */
double o_delt(const o_mesh *m, const o_cfg *c, const double *unkno,
              const double *geoel, const double *coord, const double *dvdt,
              int itime, double dtfix);

/* getsolvdg_lag: one full time step.  unkno (U^n, read) and unold (stage
 * state, read/write); cooro (stage coords, read/write); coord (x^n, read);
 * dtfix/tacru are the driver's mutable module scalars. */
void o_step(const o_mesh *m, const o_cfg *c, const double *unkno, double *unold,
            const double *coord, double *cooro, const double *coold,
            double *geoel, const double *amatr, double *ustar, int itime,
            double *dtfix, double *tacru);

/* The driver loop of the main program for nsteps steps (copies unold into
 * unkno and cooro into coord after each step, stops at tend). */
int o_run(const o_mesh *m, const o_cfg *c, double *unkno, double *coord,
          const double *coold, double *geoel, const double *amatr,
          double *ustar, int itime0, int nsteps, double *dtfix, double *tacru);

/* geterror_lag_curvhybrid (Postprocess.f90:3587-4143), quads: L2 errors
 * against the exact solution of ncase 1 (rho, |u|, p) or 2 (rho, e_int, p)
 * on the current coordinates; errl2[3] = sqrt(errlp(1:3)). */
void o_error(const o_mesh *m, const o_cfg *c, const double *unkno, const double *geoel,
             const double *coord, double *errl2);

/* ---- Linear P1 path (ncurv=0, nfint=1, nlimi=6, nrz=0; 4-node quads, no
 * triangles).  o_init, o_cellvol and o_run serve it too (o_mesh.nvqua = 4,
 * o_cfg.npoly = 1); these are its inner seams. ---- */

/* getrhsdg_lag_mcnew, ncurv=0 / nfint=1 branch (Getrhslagmc.f90:6810-6980,
 * 7270-7300): Barth limiting, nodal solver, face and volume integrals, then
 * the limited slopes applied to unkno in place.  ustar is overwritten with
 * the new nodal velocity; aflim (5, ncell) and afvec (4, ncell), if not
 * NULL, receive the limiter coefficients. */
void o1_rhs(const o_mesh *m, const o_cfg *c, double *ustar, double *unkno,
            double *rhsel, const double *geoel, const double *coord,
            double *aflim, double *afvec);

#ifdef __cplusplus
}
#endif
#endif
