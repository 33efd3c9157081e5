// Device-side building blocks of the Lag2D curved-P2 time step.
//
// Layout in HBM (structure of arrays, 0-based, one contiguous slab per field):
//   U[(q*6 + k)*ncell + e]   DOF k of field q (tau, u, v, e) of cell e
//   x[p], y[p]               node coordinates (separate arrays per config)
//   ipq[k*nquad + iq]        node k (0..8) of quad iq
//   cf[(v*32 + slot)*nquad + iq]  corner coefficient v (m, m*u, m*v, s_x, s_y)
//                                  of corner-face slot = f + 2*(ivsg + 4*isg)
//   ipt[k*ntria + it], tcf[(v*24 + slot)*ntria + it]   the same for triangles
//                                  (slot = f + 2*(ivsg + 3*isg))
// Triangles are cells 0..ntria-1, quads ntria..ncell-1 (the reference's order).
#pragma once
#include <cstdint>

namespace lag2d {

constexpr int NDEG = 6;   // P2 Taylor basis
constexpr int NQ = 4;     // tau, u, v, e
constexpr int NU = NDEG * NQ;

// Status bits written by kernels and returned by the C-ABI.
constexpr int ST_NONPHYS = 1;   // non-positive volume or NaN
constexpr int ST_STENCIL = 2;   // WENO valence the reference stops on

struct Scalars {           // device-resident module scalars
  double dtfix, tacru;
  int itime, done, status, pad;
};

struct Dev {
  int ntria, nquad, npoin, nbfac, ncell;
  int ndegr, mdegr, ncase, nlimi;
  double gamlg, cfl, cdrho, cimpd, tend, sedov_energy;
  int nsedov, sedov_cell[4];
  // connectivity
  const int *ipq;          // [9][nquad]
  const int *esq;          // [4][nquad], -1 on boundary faces
  const int *stencil;      // [9][nquad] WENO stencil cells (0-based); row 0 = -1: none, -2: valence error
  const int *node_ptr;     // [npoin+1]
  const int *node_cf;      // corner-face ids iq*32 + slot, reference summation order
  const unsigned char *bcmask;  // [npoin] bit0: u=0, bit1: v=0, bit2: keep (no solve)
  const double *x0, *y0;   // initial coordinates
  const double *rho0;      // [ncell] caller's initial-density factor per cell, or null (1)
  // geometry (time invariant except vol / vcx / vcy)
  double *rc, *sc, *mass, *g19, *g20, *g21;
  double *vol, *vcx, *vcy;
  double *msub;            // [4][nquad] initial sub-cell masses (time invariant)
  // state
  double *Un, *Us;         // U^n and the stage state
  double *xn, *yn, *xs, *ys;   // x^n and stage coordinates
  double *us, *vs;         // nodal velocity ustar
  double *amatr;           // [16][ncell]
  // work
  double *rhs;             // [24][ncell]
  double *cf;              // [5][32][nquad]
  int *flag;               // [ncell] Persson troubled-cell marks
  double *geoph;           // [2][ncell] physical mass centre
  double *mapmt;           // [4][ncell] velocity-aligned frame
  double *Uw;              // [20][nquad] WENO output (high-order moments)
  int *wlist;              // compacted troubled-quad list
  int *wcount;
  double *dtpart;          // [2][nblocks] partial minima for getdelt_lag
  Scalars *sc_dev;
  // optimised path
  const int *node_ptr2;    // [npoin+1]
  const int *node_slot;    // iq*9 + k: quad iq touches the node as its node k, cells ascending
  double *npart;           // [5][9][nquad] per-cell node partial sums (m, m*u, m*v, s_x, s_y)
  double *corr;            // [4][nquad] sub-cell density corrections
  double *src;             // [6][nquad] Taylor-Green source moments of the stage (corner pass -> RHS pass)
  double *us_new, *vs_new; // ustar of the current stage (us, vs hold the previous one)
  double *wmom;            // [9][nquad] time-invariant mass-weighted shape moments
  // triangles (cells 0..ntria-1)
  const int *ipt;          // [6][ntria] node k of triangle it
  double *tmsub;           // [4][ntria] initial sub-cell masses
  double *tcf;             // [5][24][ntria] corner coefficients (m, m u, m v, sigma.n A) per corner face
  double *tpart;           // [5][6][ntria] their per-node sums
};

// Quadrature tables (filled from the host with the reference's literals).
struct QuadTables {
  double g25[25][2], w25[25];   // 5x5 Gauss (ruqope)
  double g36[36][2], w36[36];   // 6x6 Gauss (ruqope)
  double l25[25][2], wl25[25];  // 5x5 Gauss-Lobatto (ruqope_lobatto)
  double t7[7][2], tw7[7];      // 7-point triangle rule (rutope)
};

// Adjoint (reverse-mode) work arrays of one RK stage, shared by the quad and
// triangle reverse kernels.
struct Adj {
  double *lU, *lUn;        // [24][ncell] adjoints of U^(s) and U^n
  double *lx, *ly;         // adjoint of the stage coordinates
  double *lxn, *lyn;       // adjoint of x^n
  double *lus, *lvs;       // adjoint of the stage's previous ustar
  double *luw, *lvw;       // adjoint of the stage's new ustar
  double *lR;              // [24][ncell] adjoint of the stage RHS
  double *lS;              // [5][npoin] adjoint of the node sums (m, m u, m v, sigma.n A)
  double *lP;              // [5][9][nquad] RHS pass's adjoint of each quad's node partial sums
  double *lcorr;           // [4][nquad] adjoint of the sub-cell density corrections (corner faces -> corrections)
  double *pbuf;            // [6][9][nquad] per (quad, node) adjoint contributions
  double *tx, *ty;         // scratch of the centre-node transpose
  double *tbuf;            // [6][6][ntria] per (triangle, node) adjoint contributions
  double *ltcf;            // [5][24][ntria] adjoint of the triangle corner coefficients (RHS pass)
};

}  // namespace lag2d
