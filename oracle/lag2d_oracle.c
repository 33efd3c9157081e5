/*
 * Lag2D CPU oracle -- TEST INFRASTRUCTURE ONLY (see lag2d_oracle.h).
 *
 * Single-threaded FP64 restatement of the reference time step for the
 * curved tri/quad P2 path.  Every routine keeps the reference's loop nests and
 * left-to-right accumulation order so that, compiled with
 * -O2 -ffp-contract=off (no FMA, like gfortran -O on x86-64), it reproduces
 * the reference arithmetic.  Citations are to srccurv-lag/<file>:<line>.
 *
 * Deliberate differences (each is rounding-level or a documented knob):
 *  - small dense inverses (Matinv225, LinearAlgebra.f90:130) are computed by
 *    Gauss-Jordan elimination instead of the expanded cofactor formulas;
 *  - the Sedov energy cells are a parameter instead of the hard-coded ids
 *    of Getrhslagmc.f90:5634;
 *  - barthlimit_lagcurv (Limiterlag.f90:5957) is not called: on the P2
 *    branch its node bounds are never read (Getrhslagmc.f90:7598-7656);
 *  - getbc_lagc_general (GetBClag.f90:628) is not called: its force is
 *    computed but the ustar solve has it commented out
 *    (Getrhslaggauss.f90:4502-4503).
 */
#include "lag2d_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define U_(U, c, id, iq, ie) (U)[(id) + (c)->ndegr * ((iq) + (c)->nq * (ie))]
#define G_(G, k, ie) (G)[(k) + 24 * (ie)]
#define X_(X, d, ip) (X)[(d) + 2 * (ip)]

static const double PI_ = 3.14159265358979311599796346854;  /* 4*atan(1) */

/* Set when a troubled quad has a vertex neighbourhood the reference's WENO
 * stencil search rejects with `stop` (WENO.f90:7699); the cell is skipped. */
static int g_status = 0;
int o_status(void) { int s = g_status; g_status = 0; return s; }
/* test bookkeeping (not part of the reference): Persson marks and WENO
 * replacements counted since the last o_counts call */
static long long g_marked = 0, g_replaced = 0;
void o_counts(long long *marked, long long *replaced) {
  if (marked) *marked = g_marked;
  if (replaced) *replaced = g_replaced;
  g_marked = 0;
  g_replaced = 0;
}

/* ---------------------------------------------------------------------- */
/* Quadrature rules: dgflo2d.f90:2497-2783 (2-D tensor rules).            */
/* ---------------------------------------------------------------------- */
static void gauss_1d(int n, double *p, double *w) {
  /* ruqope, dgflo2d.f90:2700-2753 (points listed in the reference order) */
  if (n == 5) {
    p[2] = 0.0;
    p[3] = 0.5384693101056830910363144;  p[1] = -0.5384693101056830910363144;
    p[4] = 0.9061798459386639927976269;  p[0] = -0.9061798459386639927976269;
    w[2] = 0.5688888888888888888888889;
    w[3] = 0.4786286704993664680412915;  w[1] = 0.4786286704993664680412915;
    w[4] = 0.2369268850561890875142640;  w[0] = 0.2369268850561890875142640;
  } else if (n == 6) {
    p[0] = 0.2386191860831969086305017;  p[1] = -0.2386191860831969086305017;
    p[2] = 0.6612093864662645136613996;  p[3] = -0.6612093864662645136613996;
    p[4] = -0.9324695142031520278123016; p[5] = 0.9324695142031520278123016;
    w[0] = 0.4679139345726910; w[1] = 0.4679139345726910;
    w[2] = 0.3607615730481386; w[3] = 0.3607615730481386;
    w[4] = 0.1713244923791704; w[5] = 0.1713244923791704;
  } else if (n == 3) {
    p[0] = -0.7745966692414833770358531; p[1] = 0.0; p[2] = 0.7745966692414833770358531;
    w[0] = 0.5555555555555555555555556; w[1] = 0.8888888888888888888888889;
    w[2] = 0.5555555555555555555555556;
  } else if (n == 2) {
    p[0] = -0.5773502691896257645091488; p[1] = 0.5773502691896257645091488;
    w[0] = 1.0; w[1] = 1.0;
  } else {
    fprintf(stderr, "oracle: unsupported Gauss rule %d\n", n);
    abort();
  }
}

static void lobatto_1d(int n, double *p, double *w) {
  /* ruqope_lobatto, dgflo2d.f90:2551-2605 */
  if (n == 5) {
    p[0] = -1.0; p[1] = -0.6546536707079771437983; p[2] = 0.0;
    p[3] = 0.6546536707079771437983; p[4] = 1.0;
    w[0] = 0.1; w[1] = 0.544444444444444444444; w[2] = 0.7111111111111111111111;
    w[3] = 0.544444444444444444444; w[4] = 0.1;
  } else {
    fprintf(stderr, "oracle: unsupported Lobatto rule %d\n", n);
    abort();
  }
}

/* 2-D tensor rule: point (i,j) with i the outer loop (dgflo2d.f90:2618-2626). */
static int quad_rule(int ngaus, int lobatto, double (*pos)[2], double *wt) {
  int n = 0;
  while (n * n < ngaus) n++;
  double p[8], w[8];
  if (lobatto) lobatto_1d(n, p, w); else gauss_1d(n, p, w);
  int ig = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      wt[ig] = w[i] * w[j];
      pos[ig][0] = p[i];
      pos[ig][1] = p[j];
      ig++;
    }
  return ig;
}

/* ---------------------------------------------------------------------- */
/* 9-node quad shape functions: GetFE.f90:89-127 (same literal forms).     */
/* ---------------------------------------------------------------------- */
static void shp9(double r, double s, double *shp, double *dr, double *ds) {
  const double c10 = 1.0;
  if (shp) {
    shp[0] = 0.25 * (c10 - r) * r * s * (c10 - s);
    shp[1] = -0.25 * (c10 + r) * (c10 - s) * r * s;
    shp[2] = 0.25 * (c10 + r) * (c10 + s) * r * s;
    shp[3] = -0.25 * (c10 - r) * (c10 + s) * r * s;
    shp[4] = -0.5 * (c10 - r * r) * (c10 - s) * s;
    shp[5] = 0.5 * (c10 + r) * (c10 - s * s) * r;
    shp[6] = 0.5 * (c10 - r * r) * (c10 + s) * s;
    shp[7] = -0.5 * (c10 - r) * (c10 - s * s) * r;
    shp[8] = (c10 - r * r) * (c10 - s * s);
  }
  if (dr) {
    dr[0] = 0.25 * (2.0 * r - c10) * s * (s - 1.0);
    dr[1] = 0.25 * (2.0 * r + c10) * s * (s - 1.0);
    dr[2] = 0.25 * (2.0 * r + c10) * s * (s + 1.0);
    dr[3] = 0.25 * (2.0 * r - c10) * s * (s + 1.0);
    dr[4] = -r * s * (s - c10);
    dr[5] = 0.5 * (2.0 * r + c10) * (c10 - s * s);
    dr[6] = -r * s * (s + c10);
    dr[7] = 0.5 * (2.0 * r - c10) * (1.0 - s * s);
    dr[8] = -2.0 * r * (1.0 - s * s);
  }
  if (ds) {
    ds[0] = 0.25 * (2.0 * s - c10) * r * (r - 1.0);
    ds[1] = 0.25 * (2.0 * s - c10) * r * (r + 1.0);
    ds[2] = 0.25 * (2.0 * s + c10) * r * (r + 1.0);
    ds[3] = 0.25 * (2.0 * s + c10) * r * (r - 1.0);
    ds[4] = 0.5 * (1.0 - r * r) * (2.0 * s - c10);
    ds[5] = -r * s * (r + c10);
    ds[6] = 0.5 * (1.0 - r * r) * (2.0 * s + c10);
    ds[7] = -r * s * (r - c10);
    ds[8] = -2.0 * s * (1.0 - r * r);
  }
}

static void jac9(const double (*xp)[2], const double *dr, const double *ds,
                 double *dxdr, double *dxds, double *dydr, double *dyds) {
  double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
  for (int k = 0; k < 9; k++) {
    a = a + dr[k] * xp[k][0];
    b = b + ds[k] * xp[k][0];
    c = c + dr[k] * xp[k][1];
    d = d + ds[k] * xp[k][1];
  }
  *dxdr = a; *dxds = b; *dydr = c; *dyds = d;
}

static void map9(const double (*xp)[2], const double *shp, double *x, double *y) {
  double a = 0.0, b = 0.0;
  for (int k = 0; k < 9; k++) {
    a = a + shp[k] * xp[k][0];
    b = b + shp[k] * xp[k][1];
  }
  *x = a; *y = b;
}

static void load_quad(const o_mesh *m, const double *X, int ie, double (*xp)[2]) {
  if (m->nvqua == 4) {
    /* ncurv = 0: the straight quad's 9-node image, built from its vertices
     * as every geometry routine does (e.g. Limiterlag.f90:2040-2048,
     * GetInitial.f90:1513-1521) */
    for (int k = 0; k < 4; k++) {
      int ip = m->ipqua[4 * ie + k] - 1;
      xp[k][0] = X_(X, 0, ip);
      xp[k][1] = X_(X, 1, ip);
    }
    for (int d = 0; d < 2; d++) {
      xp[4][d] = 0.5 * (xp[0][d] + xp[1][d]);
      xp[5][d] = 0.5 * (xp[1][d] + xp[2][d]);
      xp[6][d] = 0.5 * (xp[2][d] + xp[3][d]);
      xp[7][d] = 0.5 * (xp[3][d] + xp[0][d]);
      xp[8][d] = 0.5 * (xp[4][d] + xp[6][d]);
    }
    return;
  }
  for (int k = 0; k < 9; k++) {
    int ip = m->ipqua[9 * ie + k] - 1;
    xp[k][0] = X_(X, 0, ip);
    xp[k][1] = X_(X, 1, ip);
  }
}

/* ---------------------------------------------------------------------- */
/* Small dense linear algebra.                                            */
/* ---------------------------------------------------------------------- */
/* Inverse of an n x n matrix (n <= 5), column-major a(i,j) = a[i + n*j].
 * Gauss-Jordan with partial pivoting; replaces Matinv225
 * (LinearAlgebra.f90:130) whose expanded cofactor forms give the same
 * inverse up to rounding. */
static void inv_small(int n, const double *a, double *b) {
  double t[25], e[25];
  memcpy(t, a, sizeof(double) * n * n);
  for (int i = 0; i < n * n; i++) e[i] = 0.0;
  for (int i = 0; i < n; i++) e[i + n * i] = 1.0;
  for (int k = 0; k < n; k++) {
    int piv = k;
    double big = fabs(t[k + n * k]);
    for (int i = k + 1; i < n; i++)
      if (fabs(t[i + n * k]) > big) { big = fabs(t[i + n * k]); piv = i; }
    if (piv != k)
      for (int j = 0; j < n; j++) {
        double s = t[k + n * j]; t[k + n * j] = t[piv + n * j]; t[piv + n * j] = s;
        s = e[k + n * j]; e[k + n * j] = e[piv + n * j]; e[piv + n * j] = s;
      }
    double d = 1.0 / t[k + n * k];
    for (int j = 0; j < n; j++) { t[k + n * j] *= d; e[k + n * j] *= d; }
    for (int i = 0; i < n; i++) {
      if (i == k) continue;
      double f = t[i + n * k];
      if (f == 0.0) continue;
      for (int j = 0; j < n; j++) {
        t[i + n * j] -= f * t[k + n * j];
        e[i + n * j] -= f * e[k + n * j];
      }
    }
  }
  memcpy(b, e, sizeof(double) * n * n);
}

/* getinvmat / ludeco / lureso, dgflo2d.f90:2792-2908: in-place LU without
 * pivoting followed by n triangular solves (column-major). */
static void getinvmat(int n, double *a, double *x) {
  for (int k = 0; k < n; k++) {
    for (int mm = 0; mm < k; mm++) a[k + n * k] = a[k + n * k] - a[k + n * mm] * a[mm + n * k];
    double adicv = 1.0 / a[k + n * k];
    for (int i = k + 1; i < n; i++) {
      for (int mm = 0; mm < k; mm++) {
        a[k + n * i] = a[k + n * i] - a[k + n * mm] * a[mm + n * i];
        a[i + n * k] = a[i + n * k] - a[i + n * mm] * a[mm + n * k];
      }
      a[i + n * k] = a[i + n * k] * adicv;
    }
  }
  for (int col = 0; col < n; col++) {
    double b[8], *xc = x + n * col;
    for (int j = 0; j < n; j++) b[j] = 0.0;
    b[col] = 1.0;
    for (int i = 0; i < n; i++) {
      double c = 0.0;
      for (int j = 0; j < i; j++) c = c + a[i + n * j] * xc[j];
      xc[i] = b[i] - c;
    }
    for (int i = n - 1; i >= 0; i--) {
      double c = 0.0;
      for (int j = i + 1; j < n; j++) c = c + a[i + n * j] * xc[j];
      xc[i] = (xc[i] - c) / a[i + n * i];
    }
  }
}

/* ---------------------------------------------------------------------- */
/* Initial condition tables: getrhog_initial (GetInitial.f90:4-147) and   */
/* getunkin (Getrhslagmc.f90:5527-5844), ideal-gas cases used here.      */
/* ---------------------------------------------------------------------- */
static double rho_initial(const o_cfg *c, int ielem, double xg, double yg, double xc, double yc) {
  (void)xg; (void)yg;
  const double f = c->rho0 ? c->rho0[ielem] : 1.0;  /* caller's per-cell factor (0-based cell) */
  if (c->ncase == 6) return f * ((sqrt(xc * xc + yc * yc) <= 0.5) ? 1.0 : 0.125);
  return f;  /* TGV (1), shockless Noh (2), Noh (3), Sedov (7) */
}

static int is_sedov_cell(const o_cfg *c, int ielem1) {
  for (int i = 0; i < c->sedov_ncell; i++) if (c->sedov_cell[i] == ielem1) return 1;
  return 0;
}

static void getunkin(const o_cfg *c, double *unkin, double xg, double yg,
                     int ielem1, double volel, double xc, double yc) {
  const double g = c->gamlg;
  double rhoini = 1.0, uini = 0.0, vini = 0.0, pini = 1.0, ieini;
  switch (c->ncase) {
    case 1:
      rhoini = 1.0;
      uini = sin(PI_ * xg) * cos(PI_ * yg);
      vini = -cos(PI_ * xg) * sin(PI_ * yg);
      pini = 0.25 * (cos(2.0 * PI_ * xg) + cos(2.0 * PI_ * yg)) + 1.0;
      break;
    case 2:
      rhoini = 1.0; uini = -xg; vini = -yg; pini = (g - 1.0);
      break;
    case 3:
      rhoini = 1.0;
      uini = -xg / sqrt(xg * xg + yg * yg);
      vini = -yg / sqrt(xg * xg + yg * yg);
      pini = 1.0e-6;
      break;
    case 6:
      if (sqrt(xc * xc + (yc - 0.0) * (yc - 0.0)) <= 0.5) {
        rhoini = 1.0; ieini = 2.5; pini = ieini * (g - 1.0) * rhoini;
      } else {
        rhoini = 0.125; ieini = 2.0; pini = ieini * (g - 1.0) * rhoini;
      }
      break;
    case 7:
      rhoini = 1.0;
      if (is_sedov_cell(c, ielem1)) pini = (g - 1.0) * 1.0 * c->sedov_energy / (1.0 * volel);
      else pini = 1.0e-6;
      break;
    default:
      fprintf(stderr, "oracle: unsupported ncase %d\n", c->ncase);
      abort();
  }
  if (c->rho0) rhoini *= c->rho0[ielem1 - 1];  /* per-cell density factor at fixed p, u, v */
  unkin[0] = 1.0;
  unkin[1] = rhoini * uini;
  unkin[2] = rhoini * vini;
  unkin[3] = (pini / rhoini / (g - 1.0) + 0.5 * (uini * uini + vini * vini)) * rhoini;
}

/* GetCellctr_quad_initial, GetInitial.f90:2100-2159 */
static void cellctr_quad(const double (*xpqi)[2], double rc, double sc, double *x, double *y) {
  double shp[9];
  shp9(rc, sc, shp, NULL, NULL);
  map9(xpqi, shp, x, y);
}

/* triangle parts (defined with the triangle routines below) */
static void init_tria(const o_mesh *m, const o_cfg *c, const double *coord, double *geoel,
                      double *amatr, double *unkno);
static void cellvol_tria(const o_mesh *m, const o_cfg *c, double *geoel, const double *coord);

/* ---------------------------------------------------------------------- */
/* Initialisation                                                         */
/* ---------------------------------------------------------------------- */
void o_init(const o_mesh *m, const o_cfg *c, const double *coord,
            double *geoel, double *amatr, double *unkno) {
  const int ntria = m->ntria, nquad = m->nquad;
  const int ncell = ntria + nquad, nsize = ncell + m->nbfac;
  /* alfrz (dgflo2d.f90:150-156): 1 in RZ (nrz = 1 or 2), where the cell
   * integrals carry the radius y as a weight; RZ is dispatched on linear
   * cells only */
  const double alfrz = (c->npoly == 1 && c->nrz >= 1) ? 1.0 : 0.0;
  const int aw = (c->npoly == 1 && c->nrz == 2);
  double pos36[36][2], w36[36], pos25[25][2], w25[25];
  quad_rule(36, 0, pos36, w36);
  quad_rule(25, 0, pos25, w25);
  memset(geoel, 0, sizeof(double) * 24 * nsize);
  memset(unkno, 0, sizeof(double) * c->ndegr * c->nq * nsize);
  if (ntria > 0) init_tria(m, c, coord, geoel, amatr, unkno);

  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + ntria;
    double xp[9][2], shp[9], dr[9], ds[9];
    load_quad(m, coord, ie, xp);

    /* getgeoel_initial_lag, GetInitial.f90:1484-1694 */
    double xc, yc;
    shp9(0.0, 0.0, shp, NULL, NULL);
    map9((const double(*)[2])xp, shp, &xc, &yc);
    double xcent = 0, ycent = 0, xcel = 0, ycel = 0, volel = 0, masel = 0;
    double maselrz = 0, xcerz = 0, ycerz = 0, xceli = 0, yceli = 0, areel = 0;
    for (int ig = 0; ig < 36; ig++) {
      double r = pos36[ig][0], s = pos36[ig][1], wi = w36[ig];
      double a, b, cc, d, xg, yg;
      shp9(r, s, shp, dr, ds);
      jac9((const double(*)[2])xp, dr, ds, &a, &b, &cc, &d);
      double djaco = wi * (a * d - cc * b);
      map9((const double(*)[2])xp, shp, &xg, &yg);
      double rhog = rho_initial(c, ielem, xg, yg, xc, yc);
      double rcoef = 1.0 - alfrz + alfrz * yg;
      masel = masel + rhog * djaco * rcoef;
      volel = volel + djaco * rcoef;
      xcent = xcent + rhog * r * djaco * rcoef;
      ycent = ycent + rhog * s * djaco * rcoef;
      xcel = xcel + djaco * r * rcoef;
      ycel = ycel + djaco * s * rcoef;
      if (aw) {  /* the area (plane) integrals of nrz = 2 (GetInitial.f90:1655-1666) */
        maselrz = maselrz + rhog * djaco;
        xcerz = xcerz + rhog * r * djaco;
        ycerz = ycerz + rhog * s * djaco;
        xceli = xceli + djaco * r;
        yceli = yceli + djaco * s;
        areel = areel + djaco;
      }
    }
    G_(geoel, 0, ielem) = xcent / masel;
    G_(geoel, 1, ielem) = ycent / masel;
    G_(geoel, 2, ielem) = volel;
    G_(geoel, 3, ielem) = masel;
    {
      double mx = xp[0][1], mn = xp[0][1];
      for (int k = 1; k < 4; k++) { if (xp[k][1] > mx) mx = xp[k][1]; if (xp[k][1] < mn) mn = xp[k][1]; }
      G_(geoel, 4, ielem) = mx - mn;
    }
    G_(geoel, 6, ielem) = xcel / volel;
    G_(geoel, 7, ielem) = ycel / volel;
    if (aw) {  /* GetInitial.f90:1682-1691: geoel(11) the cell-averaged radius */
      G_(geoel, 0, ielem) = xcerz / maselrz;
      G_(geoel, 1, ielem) = ycerz / maselrz;
      G_(geoel, 2, ielem) = volel;
      G_(geoel, 3, ielem) = maselrz;
      G_(geoel, 6, ielem) = xceli / areel;
      G_(geoel, 7, ielem) = yceli / areel;
      G_(geoel, 10, ielem) = volel / areel;
      G_(geoel, 11, ielem) = areel;
    }
  }

  if (c->npoly == 2) {
    /* getgeoelho_initial_lag, GetInitial.f90:1891-2094 */
    for (int ie = 0; ie < nquad; ie++) {
      const int ielem = ie + ntria;
      double xp[9][2], shp[9], dr[9], ds[9];
      load_quad(m, coord, ie, xp);
      double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
      double rci = G_(geoel, 6, ielem), sci = G_(geoel, 7, ielem);
      double volel = G_(geoel, 2, ielem), masel = G_(geoel, 3, ielem);
      double xc, yc;
      shp9(rc, sc, shp, NULL, NULL);
      map9((const double(*)[2])xp, shp, &xc, &yc);
      double bq[6] = {0, 0, 0, 0, 0, 0}, bqi[6] = {0, 0, 0, 0, 0, 0};
      for (int ig = 0; ig < 36; ig++) {
        double r = pos36[ig][0], s = pos36[ig][1], wi = w36[ig];
        double a, b, cc, d, xg, yg;
        shp9(r, s, shp, dr, ds);
        jac9((const double(*)[2])xp, dr, ds, &a, &b, &cc, &d);
        double djaco = wi * (a * d - cc * b);
        map9((const double(*)[2])xp, shp, &xg, &yg);
        double rhog = rho_initial(c, ielem, xg, yg, xc, yc);
        double rcoef = 1.0 - alfrz + alfrz * yg;
        bq[0] = 1.0;
        bq[1] = (r - rc) / 1.0;
        bq[2] = (s - sc) / 1.0;
        bq[3] = bq[3] + 0.5 * rhog * bq[1] * bq[1] * djaco * rcoef;
        bq[4] = bq[4] + 0.5 * rhog * bq[2] * bq[2] * djaco * rcoef;
        bq[5] = bq[5] + rhog * bq[1] * bq[2] * djaco * rcoef;
        bqi[0] = 1.0;
        bqi[1] = (r - rci) / 1.0;
        bqi[2] = (s - sci) / 1.0;
        bqi[3] = bqi[3] + 0.5 * bqi[1] * bqi[1] * djaco * rcoef;
        bqi[4] = bqi[4] + 0.5 * bqi[2] * bqi[2] * djaco * rcoef;
        bqi[5] = bqi[5] + bqi[1] * bqi[2] * djaco * rcoef;
      }
      G_(geoel, 18, ielem) = bq[3] / masel;
      G_(geoel, 19, ielem) = bq[4] / masel;
      G_(geoel, 20, ielem) = bq[5] / masel;
      G_(geoel, 21, ielem) = bqi[3] / volel;
      G_(geoel, 22, ielem) = bqi[4] / volel;
      G_(geoel, 23, ielem) = bqi[5] / volel;
    }
  }

  /* inifield_mcnew, Getrhslagmc.f90:3621-3917: cell averages */
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + ntria;
    double xp[9][2], shp[9], dr[9], ds[9], unkin[4];
    load_quad(m, coord, ie, xp);
    double volel = G_(geoel, 2, ielem), masel = G_(geoel, 3, ielem);
    double xcel = xp[8][0], ycel = xp[8][1];
    double rv[4] = {0, 0, 0, 0};
    for (int ig = 0; ig < 25; ig++) {
      double r = pos25[ig][0], s = pos25[ig][1], wi = w25[ig];
      double a, b, cc, d, xg, yg;
      shp9(r, s, shp, dr, ds);
      jac9((const double(*)[2])xp, dr, ds, &a, &b, &cc, &d);
      double djaco = wi * (a * d - cc * b);
      map9((const double(*)[2])xp, shp, &xg, &yg);
      getunkin(c, unkin, xg, yg, ielem + 1, volel, xcel, ycel);
      double rcoef = 1.0 - alfrz + alfrz * yg;
      /* nrz = 2 integrates over the area (Getrhslagmc.f90:3744-3754) */
      if (aw) for (int q = 0; q < 4; q++) rv[q] = rv[q] + unkin[q] * djaco;
      else for (int q = 0; q < 4; q++) rv[q] = rv[q] + unkin[q] * djaco * rcoef;
    }
    for (int q = 0; q < 4; q++) U_(unkno, c, 0, q, ielem) = rv[q] / masel;
  }

  /* getunkno_initial_lag, GetInitial.f90:412-690: M^-1 and L2 projection */
  const int nmatr = (c->npoly == 2) ? 16 : 4;
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + ntria;
    const int nd = c->ndegr, nb = nd - 1;
    double xp[9][2], shp[9], dr[9], ds[9], unkin[4];
    load_quad(m, coord, ie, xp);
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double volel = G_(geoel, 2, ielem);
    double xc, yc;
    shp9(rc, sc, shp, NULL, NULL);
    map9((const double(*)[2])xp, shp, &xc, &yc);
    double rhsini[6][4];
    double mmatr[25], matri[25];
    memset(rhsini, 0, sizeof rhsini);
    memset(mmatr, 0, sizeof mmatr);
    double f0 = 0.0;
    for (int ig = 0; ig < 25; ig++) {
      double r = pos25[ig][0], s = pos25[ig][1], wi = w25[ig];
      double a, b, cc, d, xg, yg, bq[6];
      shp9(r, s, shp, dr, ds);
      jac9((const double(*)[2])xp, dr, ds, &a, &b, &cc, &d);
      double djaco = wi * (a * d - cc * b);
      map9((const double(*)[2])xp, shp, &xg, &yg);
      getunkin(c, unkin, xg, yg, ielem + 1, volel, xc, yc);
      bq[0] = 1.0;
      bq[1] = (r - rc) / 1.0;
      bq[2] = (s - sc) / 1.0;
      if (c->npoly == 2) {
        bq[3] = 0.5 * bq[1] * bq[1] - G_(geoel, 18, ielem);
        bq[4] = 0.5 * bq[2] * bq[2] - G_(geoel, 19, ielem);
        bq[5] = bq[1] * bq[2] - G_(geoel, 20, ielem);
      }
      for (int q = 0; q < 4; q++)
        for (int k = 0; k < nd; k++) rhsini[k][q] = rhsini[k][q] + unkin[q] * bq[k] * djaco;
      double rho0 = rho_initial(c, ielem, xg, yg, xc, yc);
      double rcoef = 1.0 - alfrz + alfrz * yg;
      if (aw) {  /* GetInitial.f90:604-610: the area mass matrix */
        f0 = f0 + rho0 * djaco;
        for (int ix = 0; ix < nb; ix++)
          for (int iy = 0; iy < nb; iy++)
            mmatr[ix + nb * iy] = mmatr[ix + nb * iy] + rho0 * bq[ix + 1] * bq[iy + 1] * djaco;
        continue;
      }
      f0 = f0 + rho0 * djaco * rcoef;
      for (int ix = 0; ix < nb; ix++)
        for (int iy = 0; iy < nb; iy++)
          mmatr[ix + nb * iy] = mmatr[ix + nb * iy] + rho0 * bq[ix + 1] * bq[iy + 1] * djaco * rcoef;
    }
    double *am = amatr + nmatr * ielem;
    if (c->npoly == 1) {
      double det = mmatr[0] * mmatr[3] - mmatr[2] * mmatr[2];
      am[0] = mmatr[3] / det;
      am[1] = -mmatr[2] / det;
      am[2] = mmatr[0] / det;
      am[3] = 1.0 / f0;
      matri[0] = am[0]; matri[2] = am[1]; matri[1] = am[1]; matri[3] = am[2];
    } else {
      getinvmat(5, mmatr, matri);
      int k = 0;
      for (int im = 0; im < 5; im++)
        for (int jm = im; jm < 5; jm++) am[k++] = matri[im + 5 * jm];
      am[15] = 1.0 / f0;
    }
    /* GetInitial.f90:675: nrz = 2 divides M^-1 by the cell-averaged radius
     * (after matri, which projects the initial state, was taken) */
    if (aw) for (int k = 0; k < nmatr; k++) am[k] = am[k] / G_(geoel, 10, ielem);
    for (int q = 0; q < 4; q++)
      for (int k = 1; k < nd; k++) U_(unkno, c, k, q, ielem) = 0.0;
    for (int q = 0; q < 4; q++)
      for (int ix = 0; ix < nb; ix++)
        for (int iy = 0; iy < nb; iy++)
          U_(unkno, c, ix + 1, q, ielem) = U_(unkno, c, ix + 1, q, ielem) + matri[ix + nb * iy] * rhsini[iy + 1][q];
  }
}

/* ---------------------------------------------------------------------- */
/* getcellvol_lag, Limiterlag.f90:1869-2167 (quad loop :2038-2165)        */
/* ---------------------------------------------------------------------- */
void o_cellvol(const o_mesh *m, const o_cfg *c, double *geoel, const double *coord) {
  if (m->ntria > 0) cellvol_tria(m, c, geoel, coord);
  double pos36[36][2], w36[36];
  quad_rule(36, 0, pos36, w36);
  const double alfrz = (c->npoly == 1 && c->nrz >= 1) ? 1.0 : 0.0;
  const int aw = (c->npoly == 1 && c->nrz == 2);
  for (int ie = 0; ie < m->nquad; ie++) {
    const int ielem = ie + m->ntria;
    double xp[9][2], shp[9], dr[9], ds[9];
    load_quad(m, coord, ie, xp);
    double rcv = 0, scv = 0, volel = 0, areel = 0, rcvrz = 0, scvrz = 0;
    for (int ig = 0; ig < 36; ig++) {
      double r = pos36[ig][0], s = pos36[ig][1], wi = w36[ig];
      double a, b, cc, d, xg, yg;
      shp9(r, s, shp, dr, ds);
      jac9((const double(*)[2])xp, dr, ds, &a, &b, &cc, &d);
      map9((const double(*)[2])xp, shp, &xg, &yg);
      double rcoef = 1.0 - alfrz + alfrz * yg;
      double djaco = wi * (a * d - cc * b);
      volel = volel + djaco * rcoef;
      rcv = rcv + r * djaco * rcoef;
      scv = scv + s * djaco * rcoef;
      if (aw) {
        areel = areel + djaco;
        rcvrz = rcvrz + r * djaco;
        scvrz = scvrz + s * djaco;
      }
    }
    G_(geoel, 2, ielem) = volel;
    G_(geoel, 4, ielem) = rcv / volel;
    G_(geoel, 5, ielem) = scv / volel;
    if (aw) {  /* Limiterlag.f90:2149-2156 */
      G_(geoel, 4, ielem) = rcvrz / areel;
      G_(geoel, 5, ielem) = scvrz / areel;
      G_(geoel, 10, ielem) = volel / areel;
      G_(geoel, 11, ielem) = areel;
      G_(geoel, 14, ielem) = rcvrz / areel;
      G_(geoel, 15, ielem) = scvrz / areel;
    }
  }
}

/* ---------------------------------------------------------------------- */
/* Sub-cell normals for quads.                                            */
/* gesgq(3,16,nquad): 1..8 corner points of the 4 outer faces,            */
/* 9..12 inner sub-cell faces at the edge nodes, 13..16 outer faces at    */
/* the edge nodes.                                                        */
/* ---------------------------------------------------------------------- */
static void normals_quad(const double (*xpq)[2], double (*gq)[3]) {
  const double c10 = 1.0;
  /* getfnds_lagsmsif_hybrid, Getrhslaggauss.f90:3537-3599 */
  static const double posqc[4][2] = {{0.0, -0.5}, {0.5, 0.0}, {0.0, 0.5}, {-0.5, 0.0}};
  static const int ipifq[4][3] = {{5, 9, 1}, {6, 9, 2}, {7, 9, 3}, {8, 9, 4}};
  double xpqv[4][2], shp[9];
  for (int isv = 0; isv < 4; isv++) {
    shp9(posqc[isv][0], posqc[isv][1], shp, NULL, NULL);
    map9(xpq, shp, &xpqv[isv][0], &xpqv[isv][1]);
  }
  for (int ifa = 0; ifa < 4; ifa++) {
    double xpf[3][2];
    for (int d = 0; d < 2; d++) {
      xpf[0][d] = xpq[ipifq[ifa][0] - 1][d];
      xpf[1][d] = xpq[ipifq[ifa][1] - 1][d];
      xpf[2][d] = xpqv[ipifq[ifa][2] - 1][d];
    }
    double r = -1.0, dsh[3];
    dsh[0] = -0.5 + r; dsh[1] = 0.5 + r; dsh[2] = -2.0 * r;
    double dxdr = 0.0, dydr = 0.0;
    for (int k = 0; k < 3; k++) { dxdr = dxdr + dsh[k] * xpf[k][0]; dydr = dydr + dsh[k] * xpf[k][1]; }
    double djaco = sqrt(dxdr * dxdr + dydr * dydr);
    double anx = -dydr, any = dxdr;
    gq[8 + ifa][0] = anx / sqrt(anx * anx + any * any);
    gq[8 + ifa][1] = any / sqrt(anx * anx + any * any);
    gq[8 + ifa][2] = djaco * 2.0;
  }
  (void)c10;
  /* getfnds_lagsms_simpsonhybrid, Getrhslaggauss.f90:9908-10010 */
  static const double posiq[12][2] = {{-1, -1}, {1, -1}, {1, -1}, {1, 1}, {1, 1}, {-1, 1},
                                      {-1, 1}, {-1, -1}, {0, -1}, {1, 0}, {0, 1}, {-1, 0}};
  for (int ig = 0; ig < 12; ig++) {
    double dr[9], ds[9], dxdr, dxds, dydr, dyds;
    shp9(posiq[ig][0], posiq[ig][1], NULL, dr, ds);
    jac9(xpq, dr, ds, &dxdr, &dxds, &dydr, &dyds);
    double c11 = dyds, c12 = -dydr, c21 = -dxds, c22 = dxdr;
    double vn0, vn1, larea = 2.0;
    int g1 = ig + 1;
    if (g1 == 1 || g1 == 2 || g1 == 9) { vn0 = 0.0; vn1 = -1.0; }
    else if (g1 == 3 || g1 == 4 || g1 == 10) { vn0 = 1.0; vn1 = 0.0; }
    else if (g1 == 5 || g1 == 6 || g1 == 11) { vn0 = 0.0; vn1 = 1.0; }
    else { vn0 = -1.0; vn1 = 0.0; }
    double anx = c11 * vn0 + c12 * vn1;
    double any = c21 * vn0 + c22 * vn1;
    double v0 = anx * larea, v1 = any * larea;
    double farea = sqrt(v0 * v0 + v1 * v1);
    int slot = (ig < 8) ? ig : ig + 4;  /* gelagq(9..12) -> gesgq(13..16) */
    gq[slot][0] = anx * larea / farea;
    gq[slot][1] = any * larea / farea;
    gq[slot][2] = farea;
  }
}

/* ---------------------------------------------------------------------- */
/* Persson troubled-cell indicator: getSIHO_Persson,                      */
/* Limiterlag.f90:12042-12239.                                            */
/* ---------------------------------------------------------------------- */
static void persson(const o_mesh *m, const o_cfg *c, const double *coord,
                    double *geoel, const double *unkno) {
  double pos[25][2], w[25];
  quad_rule(25, 0, pos, w);
  const double thr = -3.0 * log10(4.0) - 4.0;
  for (int ie = 0; ie < m->nquad; ie++) {
    const int ielem = ie + m->ntria;
    double xp[9][2], dr[9], ds[9];
    load_quad(m, coord, ie, xp);
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double unvar2[4] = {0, 0, 0, 0}, unvar1[4] = {0, 0, 0, 0};
    for (int ig = 0; ig < 25; ig++) {
      double r = pos[ig][0], s = pos[ig][1], wi = w[ig];
      double a, b, cc, d, bq[6];
      shp9(r, s, NULL, dr, ds);
      jac9((const double(*)[2])xp, dr, ds, &a, &b, &cc, &d);
      double djaco = wi * (a * d - cc * b);
      bq[0] = 1.0; bq[1] = (r - rc) / 1.0; bq[2] = (s - sc) / 1.0;
      bq[3] = 0.5 * bq[1] * bq[1] - G_(geoel, 18, ielem);
      bq[4] = 0.5 * bq[2] * bq[2] - G_(geoel, 19, ielem);
      bq[5] = bq[1] * bq[2] - G_(geoel, 20, ielem);
      double un[4] = {0, 0, 0, 0}, up1[4] = {0, 0, 0, 0};
      for (int k = 0; k < c->ndegr; k++)
        for (int q = 0; q < 4; q++) un[q] = un[q] + U_(unkno, c, k, q, ielem) * bq[k];
      for (int k = 0; k < 3; k++)
        for (int q = 0; q < 4; q++) up1[q] = up1[q] + U_(unkno, c, k, q, ielem) * bq[k];
      for (int q = 0; q < 4; q++) {
        unvar2[q] = unvar2[q] + (up1[q] - un[q]) * (up1[q] - un[q]) * djaco;
        unvar1[q] = unvar1[q] + (un[q]) * (un[q]) * djaco;
      }
    }
    G_(geoel, 9, ielem) = (log10(unvar2[0] / unvar1[0]) <= thr) ? 0.0 : 100.0;
    if (G_(geoel, 9, ielem) >= 10) g_marked++;
  }
}

/* ---------------------------------------------------------------------- */
/* WENO (WENO.f90:5927-8101)                                              */
/* ---------------------------------------------------------------------- */
typedef struct {
  const o_mesh *m;
  const o_cfg *c;
  const double *coord, *coold, *geoel, *unknr;
  double *geoph;  /* (2, nsize) */
} weno_ctx;

/* getvector_local, Limiterlag.f90:19009 */
static void vec_local(const double *mp, double *dx, double *dy) {
  double a11 = mp[0], a12 = mp[2], a21 = mp[1], a22 = mp[3];
  double xl = *dx * a11 + *dy * a12;
  double yl = *dx * a21 + *dy * a22;
  *dx = xl; *dy = yl;
}
/* getvector_local2(1, ...), WENO.f90:5889 */
static void vec_local_back(const double *mp, double *dx, double *dy) {
  double a11 = mp[3], a12 = -mp[2], a21 = -mp[1], a22 = mp[0];
  double xl = *dx * a11 + *dy * a12;
  double yl = *dx * a21 + *dy * a22;
  *dx = xl; *dy = yl;
}

/* basis_orthg with nbsis=1, WENO.f90:6683-6746 */
static void basis_orthg1(const double *bt, const double *cf, double *bo) {
  bo[0] = bt[0]; bo[1] = bt[1]; bo[2] = bt[2];
  bo[3] = 0.5 * bt[1] * bt[1] - cf[0];
  bo[4] = 0.5 * bt[2] * bt[2] - cf[1];
  bo[5] = bt[1] * bt[2] - cf[2];
}

/* matrix_sym, LinearAlgebra.f90:89-127 (column-major a(ni,nj), rhs(nq,ni)) */
static void matrix_sym(int ni, int nj, const double *a, const double *rhs,
                       double *ms, double *rs) {
  for (int i = 0; i < nj * nj; i++) ms[i] = 0.0;
  for (int i = 0; i < 4 * nj; i++) rs[i] = 0.0;
  for (int im = 0; im < nj; im++)
    for (int jm = 0; jm < nj; jm++)
      for (int km = 0; km < ni; km++)
        ms[im + nj * jm] = ms[im + nj * jm] + a[km + ni * im] * a[km + ni * jm];
  for (int iq = 0; iq < 4; iq++)
    for (int im = 0; im < nj; im++)
      for (int km = 0; km < ni; km++)
        rs[iq + 4 * im] = rs[iq + 4 * im] + a[km + ni * im] * rhs[iq + 4 * km];
}

/* getmatrix_prj2, Limiterlag.f90:16455-16562 */
static void matrix_prj2(double g, double *qmat, double *qinvm, double dnx, double dny,
                        const double *ul, const double *ur) {
  const double eps = 1.0e-6;
  double rhom1 = ul[0], u1 = ul[1], v1 = ul[2], e1 = ul[3];
  double rhoc1 = 1.0 / rhom1;
  double rhom2 = ur[0], u2 = ur[1], v2 = ur[2], e2 = ur[3];
  double rhoc2 = 1.0 / rhom2;
  double rhof = sqrt(rhoc1 * rhoc2);
  double rhosq = sqrt(rhoc1) + sqrt(rhoc2);
  double uf = (sqrt(rhoc1) * u1 + sqrt(rhoc2) * u2) / rhosq;
  double vf = (sqrt(rhoc1) * v1 + sqrt(rhoc2) * v2) / rhosq;
  double h1 = fmax(eps, g * e1 - (g - 1.0) * 0.5 * (u1 * u1 + v1 * v1));
  double h2 = fmax(eps, g * e2 - (g - 1.0) * 0.5 * (u2 * u2 + v2 * v2));
  double hf = (sqrt(rhoc1) * h1 + sqrt(rhoc2) * h2) / rhosq;
  double sdf = sqrt(fmax(eps, (g - 1.0) * (hf - 0.5 * (uf * uf + vf * vf))));
  double rhosd = rhof * sdf;
  double pf = sdf * sdf * rhof / g;
  double gam1 = (g - 1.0) / g;
  double vnm = vf * dnx - uf * dny;
  /* column-major 4x4: q(i,j) = q[i + 4*j] */
#define Q(a, i, j) a[(i - 1) + 4 * (j - 1)]
  for (int i = 0; i < 16; i++) { qinvm[i] = 0.0; qmat[i] = 0.0; }
  Q(qinvm, 1, 1) = -.5 / g;
  Q(qinvm, 1, 2) = .5 * dnx / rhosd - 0.5 * uf / pf * gam1;
  Q(qinvm, 1, 3) = .5 * dny / rhosd - 0.5 * vf / pf * gam1;
  Q(qinvm, 1, 4) = .5 / pf * gam1;
  Q(qinvm, 2, 1) = 1.0 / g;
  Q(qinvm, 2, 2) = -dny * vnm / pf - uf / pf / g;
  Q(qinvm, 2, 3) = dnx * vnm / pf - vf / pf / g;
  Q(qinvm, 2, 4) = 1.0 / pf / g;
  Q(qinvm, 3, 1) = 0.0;
  Q(qinvm, 3, 2) = dny / pf;
  Q(qinvm, 3, 3) = -dnx / pf;
  Q(qinvm, 3, 4) = 0.0;
  Q(qinvm, 4, 1) = .5 / g;
  Q(qinvm, 4, 2) = .5 * dnx / rhosd + 0.5 * uf / pf * gam1;
  Q(qinvm, 4, 3) = .5 * dny / rhosd + 0.5 * vf / pf * gam1;
  Q(qinvm, 4, 4) = -.5 / pf * gam1;
  double vedn = uf * dnx + vf * dny;
  Q(qmat, 1, 1) = -1.0;
  Q(qmat, 1, 2) = g - 1.0;
  Q(qmat, 1, 3) = (g - 1.0) * vnm;
  Q(qmat, 1, 4) = 1.0;
  Q(qmat, 2, 1) = rhosd * dnx;
  Q(qmat, 2, 2) = 0.0;
  Q(qmat, 2, 3) = pf * dny;
  Q(qmat, 2, 4) = rhosd * dnx;
  Q(qmat, 3, 1) = rhosd * dny;
  Q(qmat, 3, 2) = 0.0;
  Q(qmat, 3, 3) = -pf * dnx;
  Q(qmat, 3, 4) = rhosd * dny;
  Q(qmat, 4, 1) = pf + rhosd * vedn;
  Q(qmat, 4, 2) = pf;
  Q(qmat, 4, 3) = 0.0;
  Q(qmat, 4, 4) = -pf + rhosd * vedn;
#undef Q
}

/* Per-point data of a stencil cell j: initial-config Jacobian weight,
 * density and the local (rotated) physical position of the Gauss point. */
static void weno_cell_points(const weno_ctx *w, int jelem, const double *mapmt,
                             double *rhodj, double *xl, double *yl) {
  const o_mesh *m = w->m;
  double pos[25][2], wt[25];
  quad_rule(25, 0, pos, wt);
  int je = jelem - m->ntria;
  double xpqi[9][2], xpql[9][2], shp[9], dr[9], ds[9];
  load_quad(m, w->coold, je, xpqi);
  load_quad(m, w->coord, je, xpql);
  for (int k = 0; k < 9; k++) vec_local(mapmt, &xpql[k][0], &xpql[k][1]);
  double rcj = G_(w->geoel, 0, jelem), scj = G_(w->geoel, 1, jelem);
  double xcrho, ycrho;
  cellctr_quad((const double(*)[2])xpqi, rcj, scj, &xcrho, &ycrho);
  for (int ig = 0; ig < 25; ig++) {
    double r = pos[ig][0], s = pos[ig][1], wi = wt[ig];
    double a, b, cc, d, xgi, ygi, xg, yg;
    shp9(r, s, shp, dr, ds);
    jac9((const double(*)[2])xpqi, dr, ds, &a, &b, &cc, &d);
    double djacoi = wi * (a * d - cc * b);
    map9((const double(*)[2])xpqi, shp, &xgi, &ygi);
    map9((const double(*)[2])xpql, shp, &xg, &yg);
    double rhogi = rho_initial(w->c, jelem, xgi, ygi, xcrho, ycrho);
    rhodj[ig] = rhogi * djacoi;
    xl[ig] = xg; yl[ig] = yg;
  }
}

/* weno_cell_Taylor (nbsis=1, npoly=2), WENO.f90:7219-7537 */
static void weno_cell(const weno_ctx *w, int isten, int ielem, const double (*xpq)[2],
                      const double *mapmt, const double *unksl /* (6,4,10) */,
                      double *unk_phy /* (6,4) */) {
  const o_mesh *m = w->m;
  const int ncell = m->ntria + m->nquad;
  const int ie = ielem - m->ntria;
  const double epsil = 1.0e-6;
  double volel = G_(w->geoel, 2, ielem);
  double dxc = sqrt(volel), dyc = dxc;
  static const int mapfe[4][2] = {{1, 2}, {2, 3}, {3, 4}, {4, 1}};
  double unkf_phy[4][4][6];
  memset(unkf_phy, 0, sizeof unkf_phy);
  int ifprj = 0;
#define SL(id, iq, is) unksl[(id) + 6 * ((iq) + 4 * (is))]
  for (int ies = 0; ies < 4; ies++) {
    int jelem = m->esqua[4 * ie + ies];
    if (jelem > ncell) continue;
    jelem -= 1;
    double dtx = xpq[mapfe[ies][1] - 1][0] - xpq[mapfe[ies][0] - 1][0];
    double dty = xpq[mapfe[ies][1] - 1][1] - xpq[mapfe[ies][0] - 1][1];
    double dlgt = sqrt(dtx * dtx + dty * dty);
    double dnx = dty / dlgt, dny = -dtx / dlgt;
    vec_local(mapmt, &dnx, &dny);
    double ul[4], ur[4];
    for (int q = 0; q < 4; q++) { ul[q] = U_(w->unknr, w->c, 0, q, ielem); ur[q] = U_(w->unknr, w->c, 0, q, jelem); }
    vec_local(mapmt, &ul[1], &ul[2]);
    vec_local(mapmt, &ur[1], &ur[2]);
    double qmat[16], qinvm[16];
    matrix_prj2(w->c->gamlg, qmat, qinvm, dnx, dny, ul, ur);
    double cha[10][4][6];
    memset(cha, 0, sizeof cha);
    for (int is = 0; is < isten; is++)
      for (int iq = 0; iq < 4; iq++)
        for (int id = 0; id < 6; id++)
          for (int k = 0; k < 4; k++)
            cha[is][k][id] = cha[is][k][id] + qinvm[k + 4 * iq] * SL(id, iq, is);
    double os1[10];
    for (int is = 0; is < isten; is++) {
      double mx = 0.0;
      for (int iq = 0; iq < 4; iq++) {
        double t1 = cha[is][iq][1] / dxc, t2 = cha[is][iq][2] / dyc;
        double os = t1 * t1 + t2 * t2;
        if (iq == 0 || os > mx) mx = os;
      }
      os1[is] = mx;
    }
    double weigl[10];
    weigl[0] = .2;
    for (int is = 1; is < isten; is++) weigl[is] = 0.8 / (isten - 1.0);
    double weigh[10][4], weigt[4] = {0, 0, 0, 0};
    for (int is = 0; is < isten; is++)
      for (int iq = 0; iq < 4; iq++) {
        double t = epsil + os1[is];
        weigh[is][iq] = weigl[is] / (t * t);
      }
    for (int iq = 0; iq < 4; iq++)
      for (int is = 0; is < isten; is++) weigt[iq] = weigt[iq] + weigh[is][iq];
    for (int is = 0; is < isten; is++)
      for (int iq = 0; iq < 4; iq++) weigh[is][iq] = weigh[is][iq] / weigt[iq];
    double fch[4][6];
    memset(fch, 0, sizeof fch);
    for (int is = 0; is < isten; is++)
      for (int iq = 0; iq < 4; iq++)
        for (int id = 0; id < 6; id++) fch[iq][id] = fch[iq][id] + weigh[is][iq] * cha[is][iq][id];
    for (int iq = 0; iq < 4; iq++)
      for (int id = 1; id < 6; id++)
        for (int k = 0; k < 4; k++)
          unkf_phy[ifprj][k][id] = unkf_phy[ifprj][k][id] + qmat[k + 4 * iq] * fch[iq][id];
    ifprj++;
  }
#undef SL
  double weigf = 1.0 / ifprj;
  for (int i = 0; i < 24; i++) unk_phy[i] = 0.0;
  for (int ifa = 0; ifa < ifprj; ifa++)
    for (int iq = 0; iq < 4; iq++)
      for (int id = 1; id < 6; id++)
        unk_phy[id + 6 * iq] = unk_phy[id + 6 * iq] + weigf * unkf_phy[ifa][iq][id];
}

/* weno_stncl_quad_orthol3, WENO.f90:7541-8101 */
static void weno_stencil(const weno_ctx *w, int ielem, const double *mapmt, double *unkno) {
  const o_mesh *m = w->m;
  const o_cfg *c = w->c;
  const int ntria = m->ntria;
  static const int ielst1[4][7] = {{1, 2, 5, 6, 9, 8, 3}, {1, 3, 2, 7, 6, 9, 5},
                                   {1, 4, 3, 8, 7, 6, 5}, {1, 5, 4, 9, 8, 7, 3}};
  static const int ielst2[4][5] = {{1, 2, 6, 9, 6}, {1, 3, 6, 7, 7},
                                   {1, 4, 8, 7, 8}, {1, 5, 8, 9, 9}};
  const int ie = ielem - ntria;
  double xpq[9][2];
  load_quad(m, w->coord, ie, xpq);
  double dxcl = sqrt(G_(w->geoel, 2, ielem)), dycl = dxcl;
  int ielaj[9];
  ielaj[0] = ielem + 1;
  /* the reference indexes esqua by the global id here (WENO.f90:7648); on
   * a mesh with triangles that index leaves the quad range, so the quad's
   * own row is used there */
  for (int k = 0; k < 4; k++) ielaj[1 + k] = m->esqua[4 * (ntria > 0 ? ie : ielem) + k];
  for (int k = 5; k < 9; k++) ielaj[k] = 0;
  int ipq[9];
  for (int k = 0; k < 9; k++) ipq[k] = m->ipqua[9 * ie + k];
  for (int iv = 0; iv < 4; iv++) {
    int jelaj[5] = {0, 0, 0, 0, 0}, nvaj = 0;
    int ip = ipq[iv];
    for (int is = m->esuv2[ip - 1]; is < m->esuv2[ip]; is++) {
      int je = m->esuv1[is];
      if (je != ielem + 1) { if (nvaj < 5) jelaj[nvaj] = je; nvaj++; }
    }
    int idxod = 1, idxiv[3] = {0, 0, 0};
    for (int a = 0; a < 3; a++)
      for (int f = 0; f < 4; f++)
        if (jelaj[a] == ielaj[f + 1]) { idxod *= (f + 1); idxiv[a] = 1; }
    for (int a = 0; a < 3; a++)
      if (idxiv[a] == 0) {
        if (idxod == 2) ielaj[5] = jelaj[a];
        else if (idxod == 6) ielaj[6] = jelaj[a];
        else if (idxod == 12) ielaj[7] = jelaj[a];
        else if (idxod == 4) ielaj[8] = jelaj[a];
        else {
          /* the reference stops here (WENO.f90:7699); next to triangles
           * this is the normal case and the quad is left unlimited */
          if (ntria == 0) g_status |= 2;
          return;
        }
      }
  }
  for (int k = 0; k < 9; k++) if (ielaj[k] == 0) return;  /* boundary cell */
  /* a stencil that reaches a triangle is not a 3x3 quad block: the cell is
   * left unlimited (the reference's quad-only WENO has no such case) */
  for (int k = 0; k < 9; k++) if (ielaj[k] <= ntria) return;
  for (int k = 0; k < 9; k++) ielaj[k] -= 1;               /* 0-based */

  /* local copies of the stencil DOFs in the rotated frame */
  double unkrl[9][4][6];
  for (int s = 0; s < 9; s++)
    for (int q = 0; q < 4; q++)
      for (int d = 0; d < 6; d++) unkrl[s][q][d] = U_(w->unknr, c, d, q, ielaj[s]);
  for (int s = 0; s < 9; s++)
    for (int d = 0; d < 6; d++) vec_local(mapmt, &unkrl[s][1][d], &unkrl[s][2][d]);

  /* per-cell point data (initial-config weights, local positions) */
  double rhodj[9][25], xl[9][25], yl[9][25];
  for (int s = 0; s < 9; s++) weno_cell_points(w, ielaj[s], mapmt, rhodj[s], xl[s], yl[s]);

  /* getgeophy_local_Taylor (nbsis=1), WENO.f90:6750-7001 */
  double geopl[9][16];
  memset(geopl, 0, sizeof geopl);
  for (int s = 0; s < 9; s++) {
    int jelem = ielaj[s];
    double xclj = w->geoph[2 * jelem], yclj = w->geoph[2 * jelem + 1];
    vec_local(mapmt, &xclj, &yclj);
    geopl[s][0] = xclj; geopl[s][1] = yclj;
    double dxclj = sqrt(G_(w->geoel, 2, jelem)), dyclj = dxclj;
    double masel = G_(w->geoel, 3, jelem);
    double v1 = 0, v2 = 0, v3 = 0;
    for (int ig = 0; ig < 25; ig++) {
      double b2 = (xl[s][ig] - xclj) / dxclj, b3 = (yl[s][ig] - yclj) / dyclj;
      v1 = v1 + rhodj[s][ig] * b2 * b2;
      v2 = v2 + rhodj[s][ig] * b3 * b3;
      v3 = v3 + rhodj[s][ig] * b2 * b3;
    }
    v1 = v1 / masel; v2 = v2 / masel; v3 = v3 / masel;
    geopl[s][2] = 0.5 * v1;
    geopl[s][3] = 0.5 * v2;
    geopl[s][4] = v3;
  }

  /* getunknp_local_Taylor, WENO.f90:7005-7215 */
  double pos[25][2], wt[25];
  quad_rule(25, 0, pos, wt);
  double unkpl[9][4][6], mtbbq[25], mtbbi[25];
  for (int s = 0; s < 9; s++) {
    int jelem = ielaj[s];
    double rcj = G_(w->geoel, 0, jelem), scj = G_(w->geoel, 1, jelem);
    double xclj = geopl[s][0], yclj = geopl[s][1];
    double dxclj = sqrt(G_(w->geoel, 2, jelem)), dyclj = dxclj;
    double bb[25], bbq[25], bbi[25], bbqi[25];
    for (int i = 0; i < 25; i++) { bb[i] = 0.0; bbq[i] = 0.0; }
    for (int ig = 0; ig < 25; ig++) {
      double r = pos[ig][0], s_ = pos[ig][1];
      double bq[6], bqpl[3], bqol[6];
      bq[0] = 1.0; bq[1] = (r - rcj) / 1.0; bq[2] = (s_ - scj) / 1.0;
      bq[3] = 0.5 * bq[1] * bq[1] - G_(w->geoel, 18, jelem);
      bq[4] = 0.5 * bq[2] * bq[2] - G_(w->geoel, 19, jelem);
      bq[5] = bq[1] * bq[2] - G_(w->geoel, 20, jelem);
      bqpl[0] = 1.0; bqpl[1] = (xl[s][ig] - xclj) / dxclj; bqpl[2] = (yl[s][ig] - yclj) / dyclj;
      basis_orthg1(bqpl, &geopl[s][2], bqol);
      for (int i = 1; i < 6; i++)
        for (int j = 1; j < 6; j++) {
          bb[(i - 1) + 5 * (j - 1)] = bb[(i - 1) + 5 * (j - 1)] + rhodj[s][ig] * bq[i] * bqol[j];
          bbq[(i - 1) + 5 * (j - 1)] = bbq[(i - 1) + 5 * (j - 1)] + rhodj[s][ig] * bqol[i] * bqol[j];
        }
    }
    double rhs[6][4];
    memset(rhs, 0, sizeof rhs);
    for (int i = 1; i < 6; i++)
      for (int j = 1; j < 6; j++)
        for (int q = 0; q < 4; q++) rhs[i][q] = rhs[i][q] + unkrl[s][q][j] * bb[(j - 1) + 5 * (i - 1)];
    inv_small(5, bbq, bbqi);
    inv_small(5, bb, bbi);
    for (int q = 0; q < 4; q++) for (int d = 0; d < 6; d++) unkpl[s][q][d] = 0.0;
    for (int i = 1; i < 6; i++)
      for (int j = 1; j < 6; j++)
        for (int q = 0; q < 4; q++) unkpl[s][q][i] = unkpl[s][q][i] + rhs[j][q] * bbqi[(j - 1) + 5 * (i - 1)];
    if (s == 0) { memcpy(mtbbq, bbq, sizeof bbq); memcpy(mtbbi, bbi, sizeof bbi); }
    for (int q = 0; q < 4; q++) unkpl[s][q][0] = unkrl[s][q][0];
  }

  /* candidate stencil polynomials unksl(6,4,10) */
  double unksl[10 * 4 * 6];
#define SL(id, iq, is) unksl[(id) + 6 * ((iq) + 4 * (is))]
  memset(unksl, 0, sizeof unksl);
  for (int is = 0; is < 10; is++) for (int q = 0; q < 4; q++) SL(0, q, is) = unkpl[0][q][0];
  for (int d = 0; d < 6; d++) for (int q = 0; q < 4; q++) SL(d, q, 0) = unkpl[0][q][d];
  int isten = 0;
  const double xmcl = geopl[0][0], ymcl = geopl[0][1];
  /* 4 Lagrangian stencils: 5 cell-average equations each (WENO.f90:7740-7838) */
  for (int is = 0; is < 4; is++) {
    isten++;
    double matlg[25], rhslg[20], matin[25];
    for (int i = 0; i < 25; i++) matlg[i] = 0.0;
    for (int i = 0; i < 20; i++) rhslg[i] = 0.0;
    for (int ies = 0; ies < 5; ies++) {
      int sl = ielst1[is][ies + 1] - 1;
      double masej = G_(w->geoel, 3, ielaj[sl]);
      for (int ig = 0; ig < 25; ig++) {
        double bqplj[3], bqolj[6];
        bqplj[0] = 1.0; bqplj[1] = (xl[sl][ig] - xmcl) / dxcl; bqplj[2] = (yl[sl][ig] - ymcl) / dycl;
        basis_orthg1(bqplj, &geopl[0][2], bqolj);
        for (int k = 0; k < 5; k++)
          matlg[ies + 5 * k] = matlg[ies + 5 * k] + rhodj[sl][ig] * bqolj[k + 1] / masej;
      }
      for (int q = 0; q < 4; q++) rhslg[q + 4 * ies] = unkpl[sl][q][0] - unkpl[0][q][0];
    }
    inv_small(5, matlg, matin);
    for (int d = 1; d < 6; d++)
      for (int ies = 0; ies < 5; ies++)
        for (int q = 0; q < 4; q++) SL(d, q, isten) = SL(d, q, isten) + matin[(d - 1) + 5 * ies] * rhslg[q + 4 * ies];
  }
  /* 4 Hermite stencils: 3 averages + 6 derivative equations, least squares
   * (WENO.f90:7843-7990) */
  for (int is = 0; is < 4; is++) {
    isten++;
    double mathm[45], rhshm[36], matls[25], rhsls[20], matin[25];
    for (int i = 0; i < 45; i++) mathm[i] = 0.0;
    for (int i = 0; i < 36; i++) rhshm[i] = 0.0;
    for (int ies = 0; ies < 3; ies++) {
      int sl = ielst2[is][ies + 1] - 1;
      int jelem = ielaj[sl];
      double masej = G_(w->geoel, 3, jelem);
      double dxclj = sqrt(G_(w->geoel, 2, jelem)), dyclj = dxclj;
      double xclj = geopl[sl][0], yclj = geopl[sl][1];
      for (int ig = 0; ig < 25; ig++) {
        double bqplj[3], bqol[6], bqolj[6];
        bqplj[0] = 1.0; bqplj[1] = (xl[sl][ig] - xmcl) / dxcl; bqplj[2] = (yl[sl][ig] - ymcl) / dycl;
        basis_orthg1(bqplj, &geopl[0][2], bqol);
        for (int k = 0; k < 5; k++)
          mathm[ies + 9 * k] = mathm[ies + 9 * k] + rhodj[sl][ig] * bqol[k + 1] / masej;
        bqplj[0] = 1.0; bqplj[1] = (xl[sl][ig] - xclj) / dxclj; bqplj[2] = (yl[sl][ig] - yclj) / dyclj;
        basis_orthg1(bqplj, &geopl[sl][2], bqolj);
        int ieshm = 3 + 2 * (ies + 1) - 1 - 1; /* 0-based row */
        for (int d = 1; d < 6; d++) {
          mathm[ieshm + 9 * (d - 1)] = mathm[ieshm + 9 * (d - 1)] + rhodj[sl][ig] * bqol[d] * bqolj[1] / masej;
          mathm[ieshm + 1 + 9 * (d - 1)] = mathm[ieshm + 1 + 9 * (d - 1)] + rhodj[sl][ig] * bqol[d] * bqolj[2] / masej;
        }
        for (int d = 1; d < 6; d++)
          for (int q = 0; q < 4; q++) {
            rhshm[q + 4 * ieshm] = rhshm[q + 4 * ieshm] + rhodj[sl][ig] * bqolj[d] * bqolj[1] * unkpl[sl][q][d] / masej;
            rhshm[q + 4 * (ieshm + 1)] = rhshm[q + 4 * (ieshm + 1)] + rhodj[sl][ig] * bqolj[d] * bqolj[2] * unkpl[sl][q][d] / masej;
          }
      }
      for (int q = 0; q < 4; q++) rhshm[q + 4 * ies] = unkpl[sl][q][0] - unkpl[0][q][0];
    }
    matrix_sym(9, 5, mathm, rhshm, matls, rhsls);
    inv_small(5, matls, matin);
    for (int d = 1; d < 6; d++)
      for (int ies = 0; ies < 5; ies++)
        for (int q = 0; q < 4; q++) SL(d, q, isten) = SL(d, q, isten) + matin[(d - 1) + 5 * ies] * rhsls[q + 4 * ies];
  }
#undef SL
  isten++;  /* number of stencils = 9 */
  double unk_phy[24];
  weno_cell(w, isten, ielem, (const double(*)[2])xpq, mapmt, unksl, unk_phy);

  /* inverse L2 projection back to the Taylor basis of the target cell */
  double rhsuk[5][4];
  memset(rhsuk, 0, sizeof rhsuk);
  for (int i = 1; i < 6; i++)
    for (int j = 1; j < 6; j++)
      for (int q = 0; q < 4; q++) rhsuk[i - 1][q] = rhsuk[i - 1][q] + unk_phy[j + 6 * q] * mtbbq[(j - 1) + 5 * (i - 1)];
  double out[4][6];
  for (int q = 0; q < 4; q++) for (int d = 1; d < 6; d++) out[q][d] = 0.0;
  for (int i = 1; i < 6; i++)
    for (int j = 1; j < 6; j++)
      for (int q = 0; q < 4; q++) out[q][i] = out[q][i] + rhsuk[j - 1][q] * mtbbi[(j - 1) + 5 * (i - 1)];
  for (int d = 1; d < 6; d++) vec_local_back(mapmt, &out[1][d], &out[2][d]);
  for (int q = 0; q < 4; q++)
    for (int d = 1; d < 6; d++) U_(unkno, c, d, q, ielem) = out[q][d];
  g_replaced++;
}

/* weno_char_quad_orthgl, WENO.f90:5927-6123 */
static void weno(const o_mesh *m, const o_cfg *c, double *unkno, const double *geoel,
                 const double *coord, const double *coold) {
  const int ncell = m->ntria + m->nquad, nsize = ncell + m->nbfac;
  double pos[25][2], wt[25];
  quad_rule(25, 0, pos, wt);
  double *geoph = (double *)calloc(2 * (size_t)nsize, sizeof(double));
  double *mapmt = (double *)calloc(4 * (size_t)nsize, sizeof(double));
  for (int ie = 0; ie < m->nquad; ie++) {
    const int ielem = ie + m->ntria;
    double xp[9][2], xpi[9][2], shp[9], dr[9], ds[9];
    load_quad(m, coord, ie, xp);
    load_quad(m, coold, ie, xpi);
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double xcrho, ycrho;
    cellctr_quad((const double(*)[2])xpi, rc, sc, &xcrho, &ycrho);
    double masel = G_(geoel, 3, ielem);
    double xmc = 0.0, ymc = 0.0;
    for (int ig = 0; ig < 25; ig++) {
      double r = pos[ig][0], s = pos[ig][1], wi = wt[ig];
      double a, b, cc, d, xgi, ygi, xg, yg;
      shp9(r, s, shp, dr, ds);
      jac9((const double(*)[2])xpi, dr, ds, &a, &b, &cc, &d);
      double djacoi = wi * (a * d - cc * b);
      map9((const double(*)[2])xpi, shp, &xgi, &ygi);
      map9((const double(*)[2])xp, shp, &xg, &yg);
      double rhogi = rho_initial(c, ielem, xgi, ygi, xcrho, ycrho);
      xmc = xmc + rhogi * djacoi * xg;
      ymc = ymc + rhogi * djacoi * yg;
    }
    geoph[2 * ielem] = xmc / masel;
    geoph[2 * ielem + 1] = ymc / masel;
    double ma = U_(unkno, c, 0, 1, ielem), mb = U_(unkno, c, 0, 2, ielem);
    double *mp = mapmt + 4 * ielem;  /* column-major 2x2 */
    if (sqrt(ma * ma + mb * mb) > 1.0e-10) {
      mp[0] = ma / sqrt(ma * ma + mb * mb);
      mp[2] = mb / sqrt(ma * ma + mb * mb);
      mp[1] = -mb / sqrt(ma * ma + mb * mb);
      mp[3] = ma / sqrt(ma * ma + mb * mb);
    } else {
      mp[0] = mp[1] = mp[2] = mp[3] = 0.0;
    }
  }
  size_t nu = (size_t)c->ndegr * c->nq * nsize;
  double *unknr = (double *)malloc(nu * sizeof(double));
  memcpy(unknr, unkno, nu * sizeof(double));
  weno_ctx w = {m, c, coord, coold, geoel, unknr, geoph};
  for (int ie = 0; ie < m->nquad; ie++) {
    const int ielem = ie + m->ntria;
    if (G_(geoel, 9, ielem) < 10) continue;
    weno_stencil(&w, ielem, mapmt + 4 * ielem, unkno);
  }
  free(unknr);
  free(geoph);
  free(mapmt);
}

/* ---------------------------------------------------------------------- */
/* Sub-cell densities for the quad corners.                               */
/* ---------------------------------------------------------------------- */
static const int IPQSG[4][4] = {{1, 5, 9, 8}, {5, 2, 6, 9}, {9, 6, 3, 7}, {8, 9, 7, 4}};

/* getrhosubg_averg, Getrhslaggauss.f90:7067-7395: initial sub-cell mass
 * over current sub-cell volume. */
static void rhosubg_averg(const o_cfg *c, int ielem, const double (*xpq)[2], const double (*xpqi)[2],
                          double *unksgq) {
  static const double posqc[12][2] = {{-0.5, -1.0}, {0.5, -1.0}, {1.0, -0.5}, {1.0, 0.5},
                                      {0.5, 1.0}, {-0.5, 1.0}, {-1.0, 0.5}, {-1.0, -0.5},
                                      {0.0, -0.5}, {0.5, 0.0}, {0.0, 0.5}, {-0.5, 0.0}};
  static const int ipqsc[4][4] = {{1, 9, 12, 8}, {2, 3, 10, 9}, {10, 4, 5, 11}, {12, 11, 6, 7}};
  double pos[25][2], wt[25];
  quad_rule(25, 0, pos, wt);
  double xpqc[12][2], xpqic[12][2], shp[9], dr[9], ds[9];
  for (int isc = 0; isc < 12; isc++) {
    shp9(posqc[isc][0], posqc[isc][1], shp, NULL, NULL);
    map9(xpq, shp, &xpqc[isc][0], &xpqc[isc][1]);
    map9(xpqi, shp, &xpqic[isc][0], &xpqic[isc][1]);
  }
  double matin[4];
  for (int isg = 0; isg < 4; isg++) {
    double xs[9][2];
    for (int k = 0; k < 4; k++) {
      xs[k][0] = xpq[IPQSG[isg][k] - 1][0]; xs[k][1] = xpq[IPQSG[isg][k] - 1][1];
      xs[4 + k][0] = xpqc[ipqsc[isg][k] - 1][0]; xs[4 + k][1] = xpqc[ipqsc[isg][k] - 1][1];
    }
    for (int d = 0; d < 2; d++)
      xs[8][d] = -0.25 * (xs[0][d] + xs[1][d] + xs[2][d] + xs[3][d]) + 0.5 * (xs[4][d] + xs[5][d] + xs[6][d] + xs[7][d]);
    double f0 = 0.0;
    for (int ig = 0; ig < 25; ig++) {
      double a, b, cc, d;
      shp9(pos[ig][0], pos[ig][1], NULL, dr, ds);
      jac9((const double(*)[2])xs, dr, ds, &a, &b, &cc, &d);
      f0 = f0 + wt[ig] * (a * d - cc * b);
    }
    matin[isg] = 1.0 / f0;
  }
  for (int isg = 0; isg < 4; isg++) {
    double xs[9][2];
    for (int k = 0; k < 4; k++) {
      xs[k][0] = xpqi[IPQSG[isg][k] - 1][0]; xs[k][1] = xpqi[IPQSG[isg][k] - 1][1];
      xs[4 + k][0] = xpqic[ipqsc[isg][k] - 1][0]; xs[4 + k][1] = xpqic[ipqsc[isg][k] - 1][1];
    }
    for (int d = 0; d < 2; d++)
      xs[8][d] = -0.25 * (xs[0][d] + xs[1][d] + xs[2][d] + xs[3][d]) + 0.5 * (xs[4][d] + xs[5][d] + xs[6][d] + xs[7][d]);
    double rhs = 0.0, xci, yci;
    /* getrhoig_quadcurv2 (Getrhslag.f90:17761) evaluates the density at the
     * parent's initial centre for the piecewise cases */
    shp9(0.0, 0.0, shp, NULL, NULL);
    map9(xpqi, shp, &xci, &yci);
    for (int ig = 0; ig < 25; ig++) {
      double a, b, cc, d;
      shp9(pos[ig][0], pos[ig][1], NULL, dr, ds);
      jac9((const double(*)[2])xs, dr, ds, &a, &b, &cc, &d);
      double djaco = wt[ig] * (a * d - cc * b);
      double rhoi = rho_initial(c, ielem, 0, 0, xci, yci);
      rhs = rhs + rhoi * 1.0 * djaco;
    }
    unksgq[isg] = 0.0 + matin[isg] * rhs;
  }
}

/* getrhosubg_daverg, Getrhslaggauss.f90:10949-11112: harmonic mean of the
 * DG specific volume over each sub-cell (uqsgc = volume / integral of rho). */
static void rhosubg_daverg(const o_cfg *c, double rc, double sc, const double *bqho,
                           const double (*xpq)[2], const double *u1 /* unkno(:,1) */,
                           double aflim1, double *uqsgc) {
  double pos[25][2], wt[25], dr[9], ds[9];
  quad_rule(25, 0, pos, wt);
  double rhomc = u1[0];
  for (int isg = 0; isg < 4; isg++) {
    double masel = 0.0, volel = 0.0;
    for (int ig = 0; ig < 25; ig++) {
      double r, s;
      if (isg == 0) { r = (pos[ig][0] - 1.0) / 2.0; s = (pos[ig][1] - 1.0) / 2.0; }
      else if (isg == 1) { r = (pos[ig][0] + 1.0) / 2.0; s = (pos[ig][1] - 1.0) / 2.0; }
      else if (isg == 2) { r = (pos[ig][0] + 1.0) / 2.0; s = (pos[ig][1] + 1.0) / 2.0; }
      else { r = (pos[ig][0] - 1.0) / 2.0; s = (pos[ig][1] + 1.0) / 2.0; }
      double b[6];
      b[0] = 1.0; b[1] = (r - rc) / 1.0; b[2] = (s - sc) / 1.0;
      b[3] = 0.5 * b[1] * b[1] - bqho[0];
      b[4] = 0.5 * b[2] * b[2] - bqho[1];
      b[5] = b[1] * b[2] - bqho[2];
      double rhomsg = 0.0;
      for (int k = 0; k < c->mdegr; k++) rhomsg = rhomsg + u1[k] * b[k];
      if (c->nlimi == 6) rhomsg = rhomc + aflim1 * (rhomsg - rhomc);
      double a, bb, cc, d;
      shp9(r, s, NULL, dr, ds);
      jac9(xpq, dr, ds, &a, &bb, &cc, &d);
      double djaco = wt[ig] * (a * d - cc * bb) * 0.25;
      masel = masel + 1.0 / rhomsg * djaco;
      volel = volel + djaco;
    }
    uqsgc[isg] = volel / masel;
  }
}

/* ---------------------------------------------------------------------- */
/* Corner tables shared by the Riemann solver and the face integral.      */
/* fnqsg: gesgq slot (sign = orientation) of face ifsg at sub-cell vertex */
/* ivsg of sub-cell isg (Getrhslaggauss.f90:10486-10506).                 */
/* ---------------------------------------------------------------------- */
static const int FNQSG[4][8] = {{8, 1, 13, -9, -9, 12, 12, 16},
                                {9, 13, 2, 3, 14, -10, -10, 9},
                                {-11, 10, 10, 14, 4, 5, 15, -11},
                                {16, -12, -12, 11, 11, 15, 6, 7}};

static void corner_normals(const double (*gq)[3], int isg, double vn[4][2][3]) {
  for (int ivsg = 0; ivsg < 4; ivsg++)
    for (int f = 0; f < 2; f++) {
      int code = FNQSG[isg][2 * ivsg + f];
      int slot = abs(code) - 1;
      double sg = (code >= 0) ? 1.0 : -1.0;
      vn[ivsg][f][0] = sg * gq[slot][0];
      vn[ivsg][f][1] = sg * gq[slot][1];
      vn[ivsg][f][2] = gq[slot][2];
    }
}

/* ---------------------------------------------------------------------- */
/* Riemann input per quad: getriem_quadsubg2, Getrhslaggauss.f90:10409.   */
/* Accumulates node sums and records the per-corner coefficients.         */
/* ---------------------------------------------------------------------- */
typedef struct { double mn[2][2], mu[2], sn[2]; } corner_t;  /* per (ifa,ivsg,isg) */

static void riem_quad(const o_mesh *m, const o_cfg *c, int ie, const double *geoel,
                      const double (*gq)[3], const double *vlave, const double *unkno,
                      const double *coord, const double *coold,
                      double *munacn, double *munacu, double *snsigm, corner_t *cq) {
  const int ielem = ie + m->ntria;
  const double eps = 1.0e-6, g = c->gamlg;
  const double slpdu = (g + 1.0) / 2.0;
  static const double xvq[9] = {-1, 1, 1, -1, 0, 1, 0, -1, 0};
  static const double yvq[9] = {-1, -1, 1, 1, -1, 0, 1, 0, 0};
  double wfgsq[4][4][2];  /* [isg][ivsg][ifsg] */
  {
    /* second table of Getrhslaggauss.f90:10534-10552, then *0.25 */
    const double t[4][4][2] = {
        {{4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}, {1.0, 1.0}, {8.0 / 3.0, 4.0 / 3.0}},
        {{8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}, {1.0, 1.0}},
        {{1.0, 1.0}, {8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}},
        {{4.0 / 3.0, 8.0 / 3.0}, {1.0, 1.0}, {8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}}};
    for (int a = 0; a < 4; a++) for (int b = 0; b < 4; b++) for (int f = 0; f < 2; f++) wfgsq[a][b][f] = 0.25 * t[a][b][f];
  }
  int ipq[9];
  for (int k = 0; k < 9; k++) ipq[k] = m->ipqua[9 * ie + k] - 1;
  double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
  double bq[9][6];
  for (int iv = 0; iv < 9; iv++) {
    bq[iv][0] = 1.0;
    bq[iv][1] = (xvq[iv] - rc) / 1.0;
    bq[iv][2] = (yvq[iv] - sc) / 1.0;
    bq[iv][3] = 0.5 * bq[iv][1] * bq[iv][1] - G_(geoel, 18, ielem);
    bq[iv][4] = 0.5 * bq[iv][2] * bq[iv][2] - G_(geoel, 19, ielem);
    bq[iv][5] = bq[iv][1] * bq[iv][2] - G_(geoel, 20, ielem);
  }
  double rhomc = U_(unkno, c, 0, 0, ielem);
  double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
  double rhoct = 1.0 / rhomc;
  double pctr = fmax(eps, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
  double unknvq[9][4];
  for (int iv = 0; iv < 9; iv++) {
    for (int q = 0; q < 4; q++) unknvq[iv][q] = 0.0;
    for (int k = 0; k < c->mdegr; k++)
      for (int q = 0; q < 4; q++) unknvq[iv][q] = unknvq[iv][q] + U_(unkno, c, k, q, ielem) * bq[iv][k];
  }
  double xpq[9][2], xpqi[9][2];
  load_quad(m, coord, ie, xpq);
  load_quad(m, coold, ie, xpqi);
  double unksgq[4], uqsgc[4];
  rhosubg_averg(c, ielem, (const double(*)[2])xpq, (const double(*)[2])xpqi, unksgq);
  double u1[6];
  for (int k = 0; k < c->ndegr; k++) u1[k] = U_(unkno, c, k, 0, ielem);
  rhosubg_daverg(c, rc, sc, &G_(geoel, 18, ielem), (const double(*)[2])xpq, u1, 1.0, uqsgc);

  for (int isg = 0; isg < 4; isg++) {
    double vn[4][2][3];
    corner_normals(gq, isg, vn);
    for (int ivsg = 0; ivsg < 4; ivsg++)
      for (int f = 0; f < 2; f++) vn[ivsg][f][2] = vn[ivsg][f][2] * wfgsq[isg][ivsg][f];
    double uv[4][2], sig[4], aujmp[4][3];
    for (int ivsg = 0; ivsg < 4; ivsg++) {
      int iv = IPQSG[isg][ivsg] - 1;
      double rhovt = 1.0 / unknvq[iv][0];
      double rhovsg = rhovt + c->cdrho * (unksgq[isg] - 1.0 / uqsgc[isg]);
      double uvtx = unknvq[iv][1], vvtx = unknvq[iv][2], evtx = unknvq[iv][3];
      double pvtx = fmax(eps, (g - 1.0) * rhovsg * (evtx - 0.5 * (uvtx * uvtx + vvtx * vvtx)));
      uv[ivsg][0] = uvtx; uv[ivsg][1] = vvtx;
      sig[ivsg] = -pvtx;
      double ax = X_(vlave, 0, ipq[iv]) - uvtx;
      double ay = X_(vlave, 1, ipq[iv]) - vvtx;
      double acnx = ax, acny = ay;
      if (sqrt(acnx * acnx + acny * acny) < (double)1.e-11f) {
        ax = (double)1.e-11f; ay = (double)1.e-11f;
      } else {
        ax = ax / sqrt(acnx * acnx + acny * acny);
        ay = ay / sqrt(acnx * acnx + acny * acny);
      }
      aujmp[ivsg][0] = ax; aujmp[ivsg][1] = ay;
      aujmp[ivsg][2] = sqrt(acnx * acnx + acny * acny);
    }
    double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
    for (int ivsg = 0; ivsg < 4; ivsg++) aujmp[ivsg][2] = aujmp[ivsg][2] / sdctr;
    double murie[4][2];
    for (int ivsg = 0; ivsg < 4; ivsg++) {
      int iv = IPQSG[isg][ivsg] - 1;
      double dux = X_(vlave, 0, ipq[iv]) - uv[ivsg][0];
      double duy = X_(vlave, 1, ipq[iv]) - uv[ivsg][1];
      for (int f = 0; f < 2; f++) {
        double deltu = fabs(dux * vn[ivsg][f][0] + duy * vn[ivsg][f][1]);
        murie[ivsg][f] = rhoct * sdctr + c->cimpd * rhoct * slpdu * deltu;
      }
    }
    for (int ivsg = 0; ivsg < 4; ivsg++) {
      int iv = IPQSG[isg][ivsg] - 1, ip = ipq[iv];
      for (int f = 0; f < 2; f++) {
        /* getriecoef_matrixnew, Limiterlag.f90:1037-1076 */
        double area = vn[ivsg][f][2], n0 = vn[ivsg][f][0], n1 = vn[ivsg][f][1];
        double vnau = (aujmp[ivsg][2] < 1.0e12) ? 1.0 : n0 * aujmp[ivsg][0] + n1 * aujmp[ivsg][1];
        corner_t k;
        k.mn[0][0] = murie[ivsg][f] * area * fabs(vnau); k.mn[1][0] = 0.0;
        k.mn[0][1] = 0.0; k.mn[1][1] = murie[ivsg][f] * area * fabs(vnau);
        /* k.mn[i][j] holds munacn(i+1, j+1) */
        k.mu[0] = k.mn[0][0] * uv[ivsg][0] + k.mn[1][0] * uv[ivsg][1];
        k.mu[1] = k.mn[1][0] * uv[ivsg][0] + k.mn[1][1] * uv[ivsg][1];
        k.sn[0] = sig[ivsg] * area * n0 + 0.0 * area * n1;
        k.sn[1] = 0.0 * area * n0 + sig[ivsg] * area * n1;
        munacn[0 + 4 * ip] = munacn[0 + 4 * ip] + k.mn[0][0];
        munacn[1 + 4 * ip] = munacn[1 + 4 * ip] + k.mn[1][0];
        munacn[2 + 4 * ip] = munacn[2 + 4 * ip] + k.mn[0][1];
        munacn[3 + 4 * ip] = munacn[3 + 4 * ip] + k.mn[1][1];
        munacu[0 + 2 * ip] = munacu[0 + 2 * ip] + k.mu[0];
        munacu[1 + 2 * ip] = munacu[1 + 2 * ip] + k.mu[1];
        snsigm[0 + 2 * ip] = snsigm[0 + 2 * ip] + k.sn[0];
        snsigm[1 + 2 * ip] = snsigm[1 + 2 * ip] + k.sn[1];
        cq[(f + 2 * (ivsg + 4 * isg))] = k;
      }
    }
  }
}

/* ---------------------------------------------------------------------- */
/* 6-node triangles: P2 map on the reference triangle (0,0), (1,0), (0,1);*/
/* nodes 1-3 vertices, 4 on edge 1-2, 5 on edge 2-3, 6 on edge 3-1.       */
/* Shape functions as in getcellvol_lag (Limiterlag.f90:1935-1962).       */
/* ---------------------------------------------------------------------- */
static void shp6(double r, double s, double *shp, double *dspr, double *dsps) {
  const double c10 = 1.0;
  if (shp) {
    shp[0] = -(c10 - r - s) * (c10 - 2.0 * (c10 - r - s));
    shp[1] = -r * (c10 - 2.0 * r);
    shp[2] = -s * (c10 - 2.0 * s);
    shp[3] = 4.0 * r * (c10 - r - s);
    shp[4] = 4.0 * r * s;
    shp[5] = 4.0 * s * (c10 - r - s);
  }
  if (dspr) {
    dspr[0] = c10 - 4.0 * (c10 - r - s);
    dspr[1] = -1.0 + 4.0 * r;
    dspr[2] = 0.0;
    dspr[3] = 4.0 * (1.0 - 2.0 * r - s);
    dspr[4] = 4.0 * s;
    dspr[5] = -4.0 * s;
  }
  if (dsps) {
    dsps[0] = c10 - 4.0 * (c10 - r - s);
    dsps[1] = 0.0;
    dsps[2] = -1.0 + 4.0 * s;
    dsps[3] = -4.0 * r;
    dsps[4] = 4.0 * r;
    dsps[5] = 4.0 * (1.0 - r - 2.0 * s);
  }
}

/* dx/dr, dx/ds, dy/dr, dy/ds of the 6-node map */
static void jac6(const double (*xp)[2], const double *dspr, const double *dsps,
                 double *dxdr, double *dxds, double *dydr, double *dyds) {
  double a = 0.0, b = 0.0, cc = 0.0, d = 0.0;
  for (int k = 0; k < 6; k++) {
    a = a + dspr[k] * xp[k][0];
    b = b + dsps[k] * xp[k][0];
    cc = cc + dspr[k] * xp[k][1];
    d = d + dsps[k] * xp[k][1];
  }
  *dxdr = a; *dxds = b; *dydr = cc; *dyds = d;
}

static void map6(const double (*xp)[2], const double *shp, double *x, double *y) {
  double a = 0.0, b = 0.0;
  for (int k = 0; k < 6; k++) { a = a + shp[k] * xp[k][0]; b = b + shp[k] * xp[k][1]; }
  *x = a; *y = b;
}

static void load_tria(const o_mesh *m, const double *X, int it, double (*xp)[2]) {
  for (int k = 0; k < 6; k++) {
    int ip = m->iptri[6 * it + k] - 1;
    xp[k][0] = X_(X, 0, ip);
    xp[k][1] = X_(X, 1, ip);
  }
}

/* rutope, 2-D open rules for triangles (dgflo2d.f90:2175-2270); the
 * literals are the reference's.  Returns the number of points. */
static int tri_rule(int ngaus, double (*pos)[2], double *w) {
  if (ngaus == 1) {
    pos[0][0] = 1.0 / 3.0; pos[0][1] = 1.0 / 3.0; w[0] = 1.0;
    return 1;
  }
  if (ngaus == 3) {
    pos[0][0] = 2.0 / 3.0; pos[0][1] = 1.0 / 6.0;
    pos[1][0] = 1.0 / 6.0; pos[1][1] = 2.0 / 3.0;
    pos[2][0] = 1.0 / 6.0; pos[2][1] = 1.0 / 6.0;
    w[0] = w[1] = w[2] = 1.0 / 3.0;
    return 3;
  }
  if (ngaus == 7) {
    const double a = 0.333333333333333, b1 = 0.059715871789770, b2 = 0.470142064105115;
    const double c1 = 0.797426985353087, c2 = 0.101286507323456;
    pos[0][0] = a;  pos[0][1] = a;
    pos[1][0] = b1; pos[1][1] = b2;
    pos[2][0] = b2; pos[2][1] = b1;
    pos[3][0] = b2; pos[3][1] = b2;
    pos[4][0] = c1; pos[4][1] = c2;
    pos[5][0] = c2; pos[5][1] = c1;
    pos[6][0] = c2; pos[6][1] = c2;
    w[0] = 0.225000000000000;
    w[1] = w[2] = w[3] = 0.132394152788506;
    w[4] = w[5] = w[6] = 0.125939180544827;
    return 7;
  }
  fprintf(stderr, "oracle: triangle rule with %d points not restated\n", ngaus);
  abort();
}

/* reference coordinates of the 6 nodes */
static const double XVT[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
static const double YVT[6] = {0.0, 0.0, 1.0, 0.0, 0.5, 0.5};

/* Taylor basis of a triangle at reference point (r, s): scale dr = ds = 1/2
 * (e.g. getriem_triasubg3, Getrhslaggauss.f90:12303-12316) */
static void basis_tria(const double *geoel_e, double r, double s, double *b) {
  const double dr = 0.5, ds = 0.5;
  b[0] = 1.0;
  b[1] = (r - geoel_e[0]) / dr;
  b[2] = (s - geoel_e[1]) / ds;
  b[3] = 0.5 * b[1] * b[1] - geoel_e[18];
  b[4] = 0.5 * b[2] * b[2] - geoel_e[19];
  b[5] = b[1] * b[2] - geoel_e[20];
}

/* Initial geometry and DOFs of the triangles: the ntria loops of
 * getgeoel_initial_lag (GetInitial.f90:1334-1478), getgeoelho_initial_lag
 * (:1754-1905), inifield_mcnew (Getrhslagmc.f90:3344-3480) and
 * getunkno_initial_lag (GetInitial.f90:190-411). */
static void init_tria(const o_mesh *m, const o_cfg *c, const double *coord, double *geoel,
                      double *amatr, double *unkno) {
  const double alfrz = 0.0;
  double posg[13][2], wg[13], posd[13][2], wd[13];
  const int ng = tri_rule(c->ngausd_geo, posg, wg);
  const int nd = tri_rule(c->ngausd, posd, wd);
  const int nmatr = (c->npoly == 2) ? 16 : 4;
  for (int it = 0; it < m->ntria; it++) {
    const int ielem = it;
    double xp[6][2], shp[6], dspr[6], dsps[6], a, b, cc, d;
    load_tria(m, coord, it, xp);
    double xc, yc;
    shp6(1.0 / 3.0, 1.0 / 3.0, shp, NULL, NULL);
    map6((const double(*)[2])xp, shp, &xc, &yc);
    double xcent = 0, ycent = 0, xcel = 0, ycel = 0, volel = 0, masel = 0;
    for (int ig = 0; ig < ng; ig++) {
      double r = posg[ig][0], s = posg[ig][1], wi = wg[ig], xg, yg;
      shp6(r, s, shp, dspr, dsps);
      jac6((const double(*)[2])xp, dspr, dsps, &a, &b, &cc, &d);
      double djaco = 0.5 * wi * (a * d - cc * b);
      map6((const double(*)[2])xp, shp, &xg, &yg);
      double rhog = rho_initial(c, ielem, xg, yg, xc, yc);
      double rcoef = 1.0 - alfrz + alfrz * yg;
      masel = masel + rhog * djaco * rcoef;
      volel = volel + djaco * rcoef;
      xcent = xcent + rhog * r * djaco * rcoef;
      ycent = ycent + rhog * s * djaco * rcoef;
      xcel = xcel + djaco * r * rcoef;
      ycel = ycel + djaco * s * rcoef;
    }
    G_(geoel, 0, ielem) = xcent / masel;
    G_(geoel, 1, ielem) = ycent / masel;
    G_(geoel, 2, ielem) = volel;
    G_(geoel, 3, ielem) = masel;
    G_(geoel, 6, ielem) = xcel / volel;
    G_(geoel, 7, ielem) = ycel / volel;
    {
      double mx = xp[0][1], mn = xp[0][1];
      for (int k = 1; k < 3; k++) { if (xp[k][1] > mx) mx = xp[k][1]; if (xp[k][1] < mn) mn = xp[k][1]; }
      G_(geoel, 4, ielem) = mx - mn;
    }
  }
  if (c->npoly == 2) {
    for (int it = 0; it < m->ntria; it++) {
      const int ielem = it;
      double xp[6][2], shp[6], dspr[6], dsps[6], a, b, cc, d;
      load_tria(m, coord, it, xp);
      const double dr = 0.5, ds = 0.5;
      double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
      double rci = G_(geoel, 6, ielem), sci = G_(geoel, 7, ielem);
      double volel = G_(geoel, 2, ielem), masel = G_(geoel, 3, ielem);
      double xc, yc;
      shp6(rc, sc, shp, NULL, NULL);
      map6((const double(*)[2])xp, shp, &xc, &yc);
      double bt[6] = {0, 0, 0, 0, 0, 0}, bti[6] = {0, 0, 0, 0, 0, 0};
      for (int ig = 0; ig < ng; ig++) {
        double r = posg[ig][0], s = posg[ig][1], wi = wg[ig], xg, yg;
        shp6(r, s, shp, dspr, dsps);
        jac6((const double(*)[2])xp, dspr, dsps, &a, &b, &cc, &d);
        double djaco = 0.5 * wi * (a * d - cc * b);
        map6((const double(*)[2])xp, shp, &xg, &yg);
        double rhog = rho_initial(c, ielem, xg, yg, xc, yc);
        double rcoef = 1.0 - alfrz + alfrz * yg;
        bt[0] = 1.0;
        bt[1] = (r - rc) / dr;
        bt[2] = (s - sc) / ds;
        bt[3] = bt[3] + 0.5 * rhog * bt[1] * bt[1] * djaco * rcoef;
        bt[4] = bt[4] + 0.5 * rhog * bt[2] * bt[2] * djaco * rcoef;
        bt[5] = bt[5] + rhog * bt[1] * bt[2] * djaco * rcoef;
        bti[0] = 1.0;
        bti[1] = (r - rci) / dr;
        bti[2] = (s - sci) / ds;
        bti[3] = bti[3] + 0.5 * bti[1] * bti[1] * djaco * rcoef;
        bti[4] = bti[4] + 0.5 * bti[2] * bti[2] * djaco * rcoef;
        bti[5] = bti[5] + bti[1] * bti[2] * djaco * rcoef;
      }
      G_(geoel, 18, ielem) = bt[3] / masel;
      G_(geoel, 19, ielem) = bt[4] / masel;
      G_(geoel, 20, ielem) = bt[5] / masel;
      G_(geoel, 21, ielem) = bti[3] / volel;
      G_(geoel, 22, ielem) = bti[4] / volel;
      G_(geoel, 23, ielem) = bti[5] / volel;
    }
  }
  /* cell averages */
  for (int it = 0; it < m->ntria; it++) {
    const int ielem = it;
    double xp[6][2], shp[6], dspr[6], dsps[6], a, b, cc, d, unkin[4];
    load_tria(m, coord, it, xp);
    double volel = G_(geoel, 2, ielem), masel = G_(geoel, 3, ielem);
    double xcel = (-xp[0][0] - xp[1][0] - xp[2][0] + 4.0 * xp[3][0] + 4.0 * xp[4][0] + 4.0 * xp[5][0]) / 9.0;
    double ycel = (-xp[0][1] - xp[1][1] - xp[2][1] + 4.0 * xp[3][1] + 4.0 * xp[4][1] + 4.0 * xp[5][1]) / 9.0;
    double rv[4] = {0, 0, 0, 0};
    for (int ig = 0; ig < nd; ig++) {
      double r = posd[ig][0], s = posd[ig][1], wi = wd[ig], xg, yg;
      shp6(r, s, shp, dspr, dsps);
      jac6((const double(*)[2])xp, dspr, dsps, &a, &b, &cc, &d);
      double djaco = 0.5 * wi * (a * d - cc * b);
      map6((const double(*)[2])xp, shp, &xg, &yg);
      getunkin(c, unkin, xg, yg, ielem + 1, volel, xcel, ycel);
      double rcoef = 1.0 - alfrz + alfrz * yg;
      for (int q = 0; q < 4; q++) rv[q] = rv[q] + unkin[q] * djaco * rcoef;
    }
    for (int q = 0; q < 4; q++) U_(unkno, c, 0, q, ielem) = rv[q] / masel;
  }
  /* M^-1 and L2 projection of the higher moments */
  for (int it = 0; it < m->ntria; it++) {
    const int ielem = it;
    const int ndg = c->ndegr, nb = ndg - 1;
    double xp[6][2], shp[6], dspr[6], dsps[6], a, b, cc, d, unkin[4];
    load_tria(m, coord, it, xp);
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double volel = G_(geoel, 2, ielem);
    double xc, yc;
    shp6(rc, sc, shp, NULL, NULL);
    map6((const double(*)[2])xp, shp, &xc, &yc);
    double rhsini[6][4], mmatr[25], matri[25];
    memset(rhsini, 0, sizeof rhsini);
    memset(mmatr, 0, sizeof mmatr);
    double f0 = 0.0;
    for (int ig = 0; ig < nd; ig++) {
      double r = posd[ig][0], s = posd[ig][1], wi = wd[ig], xg, yg, bt[6];
      shp6(r, s, shp, dspr, dsps);
      jac6((const double(*)[2])xp, dspr, dsps, &a, &b, &cc, &d);
      double djaco = 0.5 * wi * (a * d - cc * b);
      map6((const double(*)[2])xp, shp, &xg, &yg);
      bt[0] = 1.0;
      bt[1] = (r - rc) / 0.5;
      bt[2] = (s - sc) / 0.5;
      if (c->npoly == 2) {
        bt[3] = 0.5 * bt[1] * bt[1] - G_(geoel, 18, ielem);
        bt[4] = 0.5 * bt[2] * bt[2] - G_(geoel, 19, ielem);
        bt[5] = bt[1] * bt[2] - G_(geoel, 20, ielem);
      }
      getunkin(c, unkin, xg, yg, ielem + 1, volel, xc, yc);
      for (int q = 0; q < 4; q++)
        for (int k = 0; k < ndg; k++) rhsini[k][q] = rhsini[k][q] + unkin[q] * bt[k] * djaco;
      double rho0 = rho_initial(c, ielem, xg, yg, xc, yc);
      double rcoef = 1.0 - alfrz + alfrz * yg;
      f0 = f0 + rho0 * djaco * rcoef;
      for (int ix = 0; ix < nb; ix++)
        for (int iy = 0; iy < nb; iy++)
          mmatr[ix + nb * iy] = mmatr[ix + nb * iy] + rho0 * bt[ix + 1] * bt[iy + 1] * djaco * rcoef;
    }
    double *am = amatr + nmatr * ielem;
    if (c->npoly == 1) {
      double det = mmatr[0] * mmatr[3] - mmatr[2] * mmatr[2];
      am[0] = mmatr[3] / det; am[1] = -mmatr[2] / det; am[2] = mmatr[0] / det; am[3] = 1.0 / f0;
      matri[0] = am[0]; matri[2] = am[1]; matri[1] = am[1]; matri[3] = am[2];
    } else {
      getinvmat(5, mmatr, matri);
      int k = 0;
      for (int im = 0; im < 5; im++)
        for (int jm = im; jm < 5; jm++) am[k++] = matri[im + 5 * jm];
      am[15] = 1.0 / f0;
    }
    for (int q = 0; q < 4; q++)
      for (int k = 1; k < ndg; k++) U_(unkno, c, k, q, ielem) = 0.0;
    for (int q = 0; q < 4; q++)
      for (int ix = 0; ix < nb; ix++)
        for (int iy = 0; iy < nb; iy++)
          U_(unkno, c, ix + 1, q, ielem) = U_(unkno, c, ix + 1, q, ielem) + matri[ix + nb * iy] * rhsini[iy + 1][q];
  }
}

/* getcellvol_lag, triangle loop (Limiterlag.f90:1908-2036) */
static void cellvol_tria(const o_mesh *m, const o_cfg *c, double *geoel, const double *coord) {
  const double alfrz = 0.0;
  double pos[13][2], w[13];
  const int ng = tri_rule(c->ngausd_geo, pos, w);
  for (int it = 0; it < m->ntria; it++) {
    double xp[6][2], shp[6], dspr[6], dsps[6], a, b, cc, d, xg, yg;
    load_tria(m, coord, it, xp);
    double rcv = 0, scv = 0, volel = 0;
    for (int ig = 0; ig < ng; ig++) {
      double r = pos[ig][0], s = pos[ig][1], wi = w[ig];
      shp6(r, s, shp, dspr, dsps);
      jac6((const double(*)[2])xp, dspr, dsps, &a, &b, &cc, &d);
      map6((const double(*)[2])xp, shp, &xg, &yg);
      double rcoef = 1.0 - alfrz + alfrz * yg;
      double djaco = 0.5 * wi * (a * d - cc * b);
      volel = volel + djaco * rcoef;
      rcv = rcv + r * djaco * rcoef;
      scv = scv + s * djaco * rcoef;
    }
    G_(geoel, 2, it) = volel;
    G_(geoel, 4, it) = rcv / volel;
    G_(geoel, 5, it) = scv / volel;
  }
}

/* Sub-cell face normals of a triangle, gesgt(3,15): slots 1-6 and 10-12
 * from the nine Simpson points of the three edges
 * (getfnds_lagsms_simpsonhybrid, Getrhslaggauss.f90:9735-9853), slots 7-9
 * and 13-15 at the two ends of the three inner sub-cell faces
 * (getfnds_lagsmsif_hybrid, Getrhslaggauss.f90:3432-3520). */
static void normals_tria(const double (*xpt)[2], double (*gt)[3]) {
  static const double postc[3][2] = {{0.25, 0.25}, {0.5, 0.25}, {0.25, 0.5}};
  static const int ipift[3][3] = {{4, 6, 1}, {5, 4, 2}, {6, 5, 3}};  /* [ifa][k] */
  double xptv[3][2], shp[6];
  for (int isv = 0; isv < 3; isv++) {
    shp6(postc[isv][0], postc[isv][1], shp, NULL, NULL);
    map6(xpt, shp, &xptv[isv][0], &xptv[isv][1]);
  }
  for (int ifa = 0; ifa < 3; ifa++) {
    double xpf[3][2];
    for (int d = 0; d < 2; d++) {
      xpf[0][d] = xpt[ipift[ifa][0] - 1][d];
      xpf[1][d] = xpt[ipift[ifa][1] - 1][d];
      xpf[2][d] = xptv[ipift[ifa][2] - 1][d];
    }
    for (int end = 0; end < 2; end++) {
      double r = end == 0 ? -1.0 : 1.0;
      double dshpr[3] = {-0.5 + r, 0.5 + r, -2.0 * r};
      double dxdr = 0.0, dydr = 0.0;
      for (int k = 0; k < 3; k++) {
        dxdr = dxdr + dshpr[k] * xpf[k][0];
        dydr = dydr + dshpr[k] * xpf[k][1];
      }
      double djaco = sqrt(dxdr * dxdr + dydr * dydr);
      double anx = -dydr, any = dxdr;
      int slot = (end == 0 ? 6 : 12) + ifa;
      gt[slot][0] = anx / sqrt(anx * anx + any * any);
      gt[slot][1] = any / sqrt(anx * anx + any * any);
      gt[slot][2] = djaco * 2.0;
    }
  }
  static const double posit[9][2] = {{0, 0}, {1, 0}, {1, 0}, {0, 1}, {0, 1}, {0, 0}, {0.5, 0}, {0.5, 0.5}, {0, 0.5}};
  double gelag[9][3];
  for (int ig = 0; ig < 9; ig++) {
    double dspr[6], dsps[6], dxdr, dxds, dydr, dyds, vn0, vn1, larea;
    shp6(posit[ig][0], posit[ig][1], shp, dspr, dsps);
    jac6(xpt, dspr, dsps, &dxdr, &dxds, &dydr, &dyds);
    double c11 = dyds, c12 = -dydr, c21 = -dxds, c22 = dxdr;
    int g1 = ig + 1;
    if (g1 == 1 || g1 == 2 || g1 == 7) { vn0 = 0.0; vn1 = -1.0; larea = 1.0; }
    else if (g1 == 3 || g1 == 4 || g1 == 8) { vn0 = sqrt(2.0) * 0.5; vn1 = sqrt(2.0) * 0.5; larea = sqrt(2.0); }
    else { vn0 = -1.0; vn1 = 0.0; larea = 1.0; }
    double anx = c11 * vn0 + c12 * vn1;
    double any = c21 * vn0 + c22 * vn1;
    double v0 = anx * larea, v1 = any * larea;
    double farea = sqrt(v0 * v0 + v1 * v1);
    gelag[ig][0] = anx * larea / farea;
    gelag[ig][1] = any * larea / farea;
    gelag[ig][2] = farea;
  }
  for (int k = 0; k < 6; k++) for (int d = 0; d < 3; d++) gt[k][d] = gelag[k][d];
  for (int k = 0; k < 3; k++) for (int d = 0; d < 3; d++) gt[9 + k][d] = gelag[6 + k][d];
}

/* Sub-cell vertices and face slots of a triangle (getriem_triasubg3,
 * Getrhslaggauss.f90:12264-12287): 4 sub-triangles of 3 vertices, 2 faces
 * per vertex; fntsg = gesgt slot, the sign orients it outwards. */
static const int IPTSG[4][3] = {{1, 4, 6}, {4, 5, 6}, {4, 2, 5}, {6, 5, 3}};
static const int FNTSG[4][6] = {{6, 1, 10, -7, -13, 12}, {7, 14, 8, 15, 9, 13},
                                {-14, 10, 2, 3, 11, -8}, {12, -9, -15, 11, 4, 5}};
/* Riemann / mass face weights x 0.25 (Getrhslaggauss.f90:12289-12302), [isg][ivsg][ifa] */
static double wfgst_tria(int isg, int ivsg, int f) {
  static const double t[4][3][2] = {
      {{4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}, {8.0 / 3.0, 4.0 / 3.0}},
      {{8.0 / 3.0, 8.0 / 3.0}, {8.0 / 3.0, 8.0 / 3.0}, {8.0 / 3.0, 8.0 / 3.0}},
      {{8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}},
      {{4.0 / 3.0, 8.0 / 3.0}, {8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}}};
  return 0.25 * t[isg][ivsg][f];
}

/* getrhosubgt_average2 (Getrhslaggauss.f90:12595-12945): sub-cell density
 * (initial sub-cell mass / current sub-cell volume) and the harmonic mean
 * of the DG specific volume over each of the 4 sub-triangles. */
static void rhosubgt_average2(const o_cfg *c, int ielem, double rc, double sc, const double *btho,
                              const double (*xpt)[2], const double (*xpti)[2], const double *u1,
                              double aflim1, double *unksgt, double *utsgc) {
  static const double postc[9][2] = {{0.25, 0.0}, {0.75, 0.0}, {0.75, 0.25}, {0.25, 0.75}, {0.0, 0.75},
                                     {0.0, 0.25}, {0.25, 0.25}, {0.5, 0.25}, {0.25, 0.5}};
  static const int iptsc[4][3] = {{1, 7, 6}, {8, 9, 7}, {2, 3, 8}, {9, 4, 5}};
  const double dr = 0.5, ds = 0.5;
  double pos[13][2], w[13];
  const int ng = tri_rule(c->ngausd, pos, w);
  double xptc[9][2], xptic[9][2], shp[6];
  for (int isc = 0; isc < 9; isc++) {
    shp6(postc[isc][0], postc[isc][1], shp, NULL, NULL);
    map6(xpt, shp, &xptc[isc][0], &xptc[isc][1]);
    map6(xpti, shp, &xptic[isc][0], &xptic[isc][1]);
  }
  const double rhomc = u1[0];
  double matin[4];
  for (int isg = 0; isg < 4; isg++) {
    double xs[6][2];
    for (int k = 0; k < 3; k++)
      for (int d = 0; d < 2; d++) {
        xs[k][d] = xpt[IPTSG[isg][k] - 1][d];
        xs[3 + k][d] = xptc[iptsc[isg][k] - 1][d];
      }
    double f0 = 0.0, masel = 0.0, volel = 0.0;
    for (int ig = 0; ig < ng; ig++) {
      double r = pos[ig][0], s = pos[ig][1], wi = w[ig];
      double shps[3] = {1.0 - r - s, r, s};
      double rg = 0.0, sg = 0.0;
      for (int k = 0; k < 3; k++) {
        rg = rg + shps[k] * XVT[IPTSG[isg][k] - 1];
        sg = sg + shps[k] * YVT[IPTSG[isg][k] - 1];
      }
      double btsg[6];
      btsg[0] = 1.0;
      btsg[1] = (rg - rc) / dr;
      btsg[2] = (sg - sc) / ds;
      btsg[3] = 0.5 * btsg[1] * btsg[1] - btho[0];
      btsg[4] = 0.5 * btsg[2] * btsg[2] - btho[1];
      btsg[5] = btsg[1] * btsg[2] - btho[2];
      double rhomsg = 0.0;
      for (int k = 0; k < c->mdegr; k++) rhomsg = rhomsg + u1[k] * btsg[k];
      if (c->nlimi == 6) rhomsg = rhomc + aflim1 * (rhomsg - rhomc);
      double dspr[6], dsps[6], a, b, cc, d;
      shp6(r, s, NULL, dspr, dsps);
      jac6((const double(*)[2])xs, dspr, dsps, &a, &b, &cc, &d);
      double djaco = 0.5 * wi * (a * d - cc * b);
      f0 = f0 + djaco;
      masel = masel + 1.0 / rhomsg * djaco;
      volel = volel + djaco;
    }
    matin[isg] = 1.0 / f0;
    utsgc[isg] = volel / masel;
  }
  double xci, yci;
  shp6(1.0 / 3.0, 1.0 / 3.0, shp, NULL, NULL);
  map6(xpti, shp, &xci, &yci);
  for (int isg = 0; isg < 4; isg++) {
    double xs[6][2];
    for (int k = 0; k < 3; k++)
      for (int d = 0; d < 2; d++) {
        xs[k][d] = xpti[IPTSG[isg][k] - 1][d];
        xs[3 + k][d] = xptic[iptsc[isg][k] - 1][d];
      }
    double rhs = 0.0;
    for (int ig = 0; ig < ng; ig++) {
      double r = pos[ig][0], s = pos[ig][1], wi = w[ig];
      double dspr[6], dsps[6], a, b, cc, d;
      shp6(r, s, NULL, dspr, dsps);
      jac6((const double(*)[2])xs, dspr, dsps, &a, &b, &cc, &d);
      double djaco = 0.5 * wi * (a * d - cc * b);
      /* getrhoig_triacurv2 (Getrhslag.f90:17622): the cases built here
       * have a density that depends on the parent's initial centroid only */
      double rhoi = rho_initial(c, ielem, 0, 0, xci, yci);
      rhs = rhs + rhoi * 1.0 * djaco;
    }
    unksgt[isg] = 0.0 + matin[isg] * rhs;
  }
}

/* getriem_triasubg3 (Getrhslaggauss.f90:12201-12590): corner coefficients
 * of the 4 sub-triangles (3 vertices x 2 faces each), scattered into the
 * node sums; no impedance jump term and no cdrho factor on triangles. */
static void riem_tria(const o_mesh *m, const o_cfg *c, int it, const double *geoel,
                      const double (*gt)[3], const double *vlave, const double *unkno,
                      const double *coord, const double *coold,
                      double *munacn, double *munacu, double *snsigm, corner_t *ct) {
  const int ielem = it;
  const double eps = 1.0e-15, g = c->gamlg;
  const double slpdu = (g + 1.0) / 2.0;
  int ipt[6];
  for (int k = 0; k < 6; k++) ipt[k] = m->iptri[6 * it + k] - 1;
  const double *ge = &G_(geoel, 0, ielem);
  double bt[6][6];
  for (int iv = 0; iv < 6; iv++) basis_tria(ge, XVT[iv], YVT[iv], bt[iv]);
  double rhomc = U_(unkno, c, 0, 0, ielem);
  double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
  double rhoct = 1.0 / rhomc;
  double pctr = fmax(eps, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
  double unknvt[6][4];
  for (int iv = 0; iv < 6; iv++) {
    for (int q = 0; q < 4; q++) unknvt[iv][q] = 0.0;
    for (int k = 0; k < c->mdegr; k++)
      for (int q = 0; q < 4; q++) unknvt[iv][q] = unknvt[iv][q] + U_(unkno, c, k, q, ielem) * bt[iv][k];
  }
  double xpt[6][2], xpti[6][2];
  load_tria(m, coord, it, xpt);
  load_tria(m, coold, it, xpti);
  double unksgt[4], utsgc[4], u1[6];
  for (int k = 0; k < c->ndegr; k++) u1[k] = U_(unkno, c, k, 0, ielem);
  rhosubgt_average2(c, ielem, ge[0], ge[1], ge + 18, (const double(*)[2])xpt, (const double(*)[2])xpti, u1, 1.0,
                    unksgt, utsgc);
  for (int isg = 0; isg < 4; isg++) {
    double vn[3][2][3];
    for (int ivsg = 0; ivsg < 3; ivsg++)
      for (int f = 0; f < 2; f++) {
        int code = FNTSG[isg][2 * ivsg + f];
        int slot = abs(code) - 1;
        double sg = code >= 0 ? 1.0 : -1.0;
        vn[ivsg][f][0] = sg * gt[slot][0];
        vn[ivsg][f][1] = sg * gt[slot][1];
        vn[ivsg][f][2] = gt[slot][2] * wfgst_tria(isg, ivsg, f);
      }
    double uv[3][2], sig[3], aujmp[3][3];
    for (int ivsg = 0; ivsg < 3; ivsg++) {
      int iv = IPTSG[isg][ivsg] - 1;
      double rhovt = 1.0 / unknvt[iv][0];
      double rhovsg = rhovt + 1.0 * (unksgt[isg] - 1.0 / utsgc[isg]);
      double uvtx = unknvt[iv][1], vvtx = unknvt[iv][2], evtx = unknvt[iv][3];
      double pvtx = fmax(eps, (g - 1.0) * rhovsg * (evtx - 0.5 * (uvtx * uvtx + vvtx * vvtx)));
      uv[ivsg][0] = uvtx; uv[ivsg][1] = vvtx;
      sig[ivsg] = -pvtx;
      double ax = X_(vlave, 0, ipt[iv]) - uvtx, ay = X_(vlave, 1, ipt[iv]) - vvtx;
      double acnx = ax, acny = ay;
      if (sqrt(acnx * acnx + acny * acny) < (double)1.e-11f) {
        ax = (double)1.e-11f; ay = (double)1.e-11f;
      } else {
        ax = ax / sqrt(acnx * acnx + acny * acny);
        ay = ay / sqrt(acnx * acnx + acny * acny);
      }
      aujmp[ivsg][0] = ax; aujmp[ivsg][1] = ay;
      aujmp[ivsg][2] = sqrt(acnx * acnx + acny * acny);
    }
    double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
    for (int ivsg = 0; ivsg < 3; ivsg++) aujmp[ivsg][2] = aujmp[ivsg][2] / sdctr;
    double murie[3][2];
    for (int ivsg = 0; ivsg < 3; ivsg++) {
      int iv = IPTSG[isg][ivsg] - 1;
      double dux = X_(vlave, 0, ipt[iv]) - uv[ivsg][0];
      double duy = X_(vlave, 1, ipt[iv]) - uv[ivsg][1];
      for (int f = 0; f < 2; f++) {
        double deltu = 0.0 * fabs(dux * vn[ivsg][f][0] + duy * vn[ivsg][f][1]);
        murie[ivsg][f] = rhoct * sdctr + rhoct * slpdu * deltu;
      }
    }
    for (int ivsg = 0; ivsg < 3; ivsg++) {
      int iv = IPTSG[isg][ivsg] - 1, ip = ipt[iv];
      for (int f = 0; f < 2; f++) {
        double area = vn[ivsg][f][2], n0 = vn[ivsg][f][0], n1 = vn[ivsg][f][1];
        double vnau = (aujmp[ivsg][2] < 1.0e12) ? 1.0 : n0 * aujmp[ivsg][0] + n1 * aujmp[ivsg][1];
        corner_t k;
        k.mn[0][0] = murie[ivsg][f] * area * fabs(vnau); k.mn[1][0] = 0.0;
        k.mn[0][1] = 0.0; k.mn[1][1] = murie[ivsg][f] * area * fabs(vnau);
        k.mu[0] = k.mn[0][0] * uv[ivsg][0] + k.mn[1][0] * uv[ivsg][1];
        k.mu[1] = k.mn[1][0] * uv[ivsg][0] + k.mn[1][1] * uv[ivsg][1];
        k.sn[0] = sig[ivsg] * area * n0 + 0.0 * area * n1;
        k.sn[1] = 0.0 * area * n0 + sig[ivsg] * area * n1;
        munacn[0 + 4 * ip] = munacn[0 + 4 * ip] + k.mn[0][0];
        munacn[1 + 4 * ip] = munacn[1 + 4 * ip] + k.mn[1][0];
        munacn[2 + 4 * ip] = munacn[2 + 4 * ip] + k.mn[0][1];
        munacn[3 + 4 * ip] = munacn[3 + 4 * ip] + k.mn[1][1];
        munacu[0 + 2 * ip] = munacu[0 + 2 * ip] + k.mu[0];
        munacu[1 + 2 * ip] = munacu[1 + 2 * ip] + k.mu[1];
        snsigm[0 + 2 * ip] = snsigm[0 + 2 * ip] + k.sn[0];
        snsigm[1 + 2 * ip] = snsigm[1 + 2 * ip] + k.sn[1];
        ct[f + 2 * (ivsg + 3 * isg)] = k;
      }
    }
  }
}

/* rhsifacedg_lagsubgt3 (Getrhslaggauss.f90:8297-8496): face integral of a
 * triangle; mass-equation weights wfgstm (= the Riemann weights), unit
 * momentum/energy weights. */
static void iface_tria(const o_mesh *m, const o_cfg *c, int it, const double *geoel,
                       const double (*gt)[3], const double *ustar, const double *fstart,
                       double *rhsel) {
  const int ielem = it;
  const double *ge = &G_(geoel, 0, ielem);
  double bt[6][6];
  for (int iv = 0; iv < 6; iv++) basis_tria(ge, XVT[iv], YVT[iv], bt[iv]);
  const int nd = c->ndegr;
  double ulnpn[6] = {0}, pln0[6] = {0}, pln1[6] = {0}, elnpn[6] = {0};
  for (int isg = 0; isg < 4; isg++) {
    double vn[3][2][3];
    for (int ivsg = 0; ivsg < 3; ivsg++)
      for (int f = 0; f < 2; f++) {
        int code = FNTSG[isg][2 * ivsg + f];
        int slot = abs(code) - 1;
        double sg = code >= 0 ? 1.0 : -1.0;
        vn[ivsg][f][0] = sg * gt[slot][0];
        vn[ivsg][f][1] = sg * gt[slot][1];
        vn[ivsg][f][2] = gt[slot][2] * wfgst_tria(isg, ivsg, f);
      }
    for (int ivsg = 0; ivsg < 3; ivsg++) {
      int iv = IPTSG[isg][ivsg] - 1;
      int ip = m->iptri[6 * it + iv] - 1;
      double us = X_(ustar, 0, ip), vs = X_(ustar, 1, ip);
      const double *f1 = fstart + 2 * (0 + 2 * (ivsg + 3 * (isg + 4 * (size_t)it)));
      const double *f2 = fstart + 2 * (1 + 2 * (ivsg + 3 * (isg + 4 * (size_t)it)));
      for (int k = 0; k < nd; k++) {
        double b = bt[iv][k];
        ulnpn[k] = ulnpn[k] + us * vn[ivsg][0][0] * vn[ivsg][0][2] * b + vs * vn[ivsg][0][1] * vn[ivsg][0][2] * b +
                   us * vn[ivsg][1][0] * vn[ivsg][1][2] * b + vs * vn[ivsg][1][1] * vn[ivsg][1][2] * b;
        pln0[k] = pln0[k] + f1[0] * b * 1.0 + f2[0] * b * 1.0;
        pln1[k] = pln1[k] + f1[1] * b * 1.0 + f2[1] * b * 1.0;
        elnpn[k] = elnpn[k] + us * f1[0] * b * 1.0 + vs * f1[1] * b * 1.0 + us * f2[0] * b * 1.0 +
                   vs * f2[1] * b * 1.0;
      }
    }
  }
  for (int k = 0; k < nd; k++) {
    U_(rhsel, c, k, 0, ielem) = ulnpn[k];
    U_(rhsel, c, k, 1, ielem) = pln0[k];
    U_(rhsel, c, k, 2, ielem) = pln1[k];
    U_(rhsel, c, k, 3, ielem) = elnpn[k];
  }
}

/* rhsdomndg_lagmc_curvtria (Getrhslag.f90:4449-4711): volume integral in
 * cofactor form, rutope(ngausd). */
static void domn_tria(const o_mesh *m, const o_cfg *c, int it, const double *geoel,
                      const double *coord, const double *unkno, double *rhsel) {
  const int ielem = it;
  const double dr = 0.5, ds = 0.5, g = c->gamlg;
  double pos[13][2], w[13];
  const int ng = tri_rule(c->ngausd, pos, w);
  double xp[6][2];
  load_tria(m, coord, it, xp);
  const double *ge = &G_(geoel, 0, ielem);
  double rc = ge[0], sc = ge[1];
  double dbdr[6] = {0.0, 1.0 / dr, 0.0, 0, 0, 0}, dbds[6] = {0.0, 0.0, 1.0 / ds, 0, 0, 0};
  for (int ig = 0; ig < ng; ig++) {
    double r = pos[ig][0], s = pos[ig][1], wi = w[ig];
    double shp[6], dspr[6], dsps[6], dxdr, dxds, dydr, dyds;
    shp6(r, s, shp, dspr, dsps);
    jac6((const double(*)[2])xp, dspr, dsps, &dxdr, &dxds, &dydr, &dyds);
    double djaco = 0.5 * wi;
    if (c->npoly == 2) {
      dbdr[3] = (r - rc) / (dr * dr); dbdr[4] = 0.0; dbdr[5] = (s - sc) / dr / ds;
      dbds[3] = 0.0; dbds[4] = (s - sc) / (ds * ds); dbds[5] = (r - rc) / dr / ds;
    }
    double gd[2][6];
    for (int k = 0; k < c->ndegr; k++) {
      gd[0][k] = dyds * dbdr[k] + (-dydr) * dbds[k];
      gd[1][k] = (-dxds) * dbdr[k] + dxdr * dbds[k];
    }
    double b[6];
    basis_tria(ge, r, s, b);
    double un[4] = {0, 0, 0, 0};
    for (int k = 0; k < c->mdegr; k++)
      for (int q = 0; q < 4; q++) un[q] = un[q] + U_(unkno, c, k, q, ielem) * b[k];
    double rhoad = 1.0 / un[0];
    double uadv = un[1], vadv = un[2], eadv = un[3];
    double pres = (g - 1.0) * rhoad * (eadv - 0.5 * (uadv * uadv + vadv * vadv));
    for (int k = 0; k < c->ndegr; k++) {
      double f0 = gd[0][k] * uadv + gd[1][k] * vadv;
      double f1 = gd[0][k] * (-pres);
      double f2 = gd[1][k] * (-pres);
      double f3 = (gd[0][k] * uadv + gd[1][k] * vadv) * (-pres);
      U_(rhsel, c, k, 0, ielem) = U_(rhsel, c, k, 0, ielem) - f0 * djaco;
      U_(rhsel, c, k, 1, ielem) = U_(rhsel, c, k, 1, ielem) - f1 * djaco;
      U_(rhsel, c, k, 2, ielem) = U_(rhsel, c, k, 2, ielem) - f2 * djaco;
      U_(rhsel, c, k, 3, ielem) = U_(rhsel, c, k, 3, ielem) - f3 * djaco;
    }
  }
}

/* rhsdomnsrcdg_lag_curvtria (Getrhslag.f90:3907-4066): Taylor-Green energy
 * source.  The reference sets only b(1:3) there and leaves b(4:6) of its
 * P2 basis undefined; the full P2 basis is used here (as in the quad
 * routine). */
static void src_tria(const o_mesh *m, const o_cfg *c, int it, const double *geoel,
                     const double *coord, double *rhsel) {
  const int ielem = it;
  const double g = c->gamlg;
  double pos[13][2], w[13];
  const int ng = tri_rule(c->ngausd, pos, w);
  double xp[6][2];
  load_tria(m, coord, it, xp);
  const double *ge = &G_(geoel, 0, ielem);
  for (int ig = 0; ig < ng; ig++) {
    double r = pos[ig][0], s = pos[ig][1], wi = w[ig];
    double shp[6], dspr[6], dsps[6], a, b, cc, d, xg, yg;
    shp6(r, s, shp, dspr, dsps);
    jac6((const double(*)[2])xp, dspr, dsps, &a, &b, &cc, &d);
    double djaco = 0.5 * wi * (a * d - cc * b);
    map6((const double(*)[2])xp, shp, &xg, &yg);
    double bb[6];
    basis_tria(ge, r, s, bb);
    double src = 0.25 * PI_ * (cos(3.0 * PI_ * xg) * cos(PI_ * yg) - cos(3.0 * PI_ * yg) * cos(PI_ * xg)) / (g - 1.0);
    for (int k = 0; k < c->ndegr; k++) U_(rhsel, c, k, 3, ielem) = U_(rhsel, c, k, 3, ielem) + src * bb[k] * djaco;
  }
}

/* ---------------------------------------------------------------------- */
/* getndvelo_lagsubg, Getrhslaggauss.f90:4348-4617                        */
/* ---------------------------------------------------------------------- */
static void ndvelo(const o_mesh *m, const o_cfg *c, const double *geoel, const double *gq,
                   const double *gt, const double *coord, const double *coold, const double *unkno,
                   double *ustar, double *fstarq /* (2,2,4,4,nquad) */, double *fstart /* (2,2,3,4,ntria) */) {
  const int npoin = m->npoin;
  char *indnd = (char *)calloc(npoin, 1);
  for (int f = 0; f < m->nbfac; f++) {
    const int *bf = m->bface + 5 * f;
    if (c->ncase == 2 || bf[2] == 25) { indnd[bf[0] - 1] = 1; indnd[bf[1] - 1] = 1; indnd[bf[4] - 1] = 1; }
  }
  double *vlave = (double *)malloc(sizeof(double) * 2 * npoin);
  memcpy(vlave, ustar, sizeof(double) * 2 * npoin);
  double *munacn = (double *)calloc(4 * (size_t)npoin, sizeof(double));
  double *munacu = (double *)calloc(2 * (size_t)npoin, sizeof(double));
  double *snsigm = (double *)calloc(2 * (size_t)npoin, sizeof(double));
  corner_t *cq = (corner_t *)malloc(sizeof(corner_t) * 32 * (size_t)m->nquad);
  corner_t *ct = (corner_t *)malloc(sizeof(corner_t) * 24 * (size_t)(m->ntria > 0 ? m->ntria : 1));
  for (int it = 0; it < m->ntria; it++)
    riem_tria(m, c, it, geoel, (const double(*)[3])(gt + 45 * (size_t)it), vlave, unkno, coord, coold,
              munacn, munacu, snsigm, ct + 24 * (size_t)it);
  for (int ie = 0; ie < m->nquad; ie++)
    riem_quad(m, c, ie, geoel, (const double(*)[3])(gq + 48 * (size_t)ie), vlave, unkno, coord, coold,
              munacn, munacu, snsigm, cq + 32 * (size_t)ie);
  for (int ip = 0; ip < npoin; ip++) {
    if (indnd[ip]) continue;
    const double *mn = munacn + 4 * ip;  /* (1,1),(2,1),(1,2),(2,2) */
    double detma = mn[0] * mn[3] - mn[1] * mn[2];
    double i11 = mn[3] / detma, i12 = -mn[2] / detma, i21 = -mn[1] / detma, i22 = mn[0] / detma;
    double r1 = munacu[2 * ip] - snsigm[2 * ip];
    double r2 = munacu[2 * ip + 1] - snsigm[2 * ip + 1];
    ustar[2 * ip] = i11 * r1 + i12 * r2;
    ustar[2 * ip + 1] = i21 * r1 + i22 * r2;
  }
  for (int f = 0; f < m->nbfac; f++) {
    const int *bf = m->bface + 5 * f;
    int nodes[3] = {bf[0] - 1, bf[1] - 1, bf[4] - 1};
    if (bf[2] == 22) {
      if (bf[3] == 221) for (int k = 0; k < 3; k++) ustar[2 * nodes[k] + 1] = 0.0;
      else if (bf[3] == 222) for (int k = 0; k < 3; k++) ustar[2 * nodes[k]] = 0.0;
    } else if (bf[2] == 25) {
      for (int k = 0; k < 3; k++) { ustar[2 * nodes[k] + 1] = 0.0; ustar[2 * nodes[k]] = 0.0; }
    }
  }
  for (int it = 0; it < m->ntria; it++)
    for (int isg = 0; isg < 4; isg++)
      for (int ivsg = 0; ivsg < 3; ivsg++) {
        int ip = m->iptri[6 * it + IPTSG[isg][ivsg] - 1] - 1;
        for (int f = 0; f < 2; f++) {
          const corner_t *k = ct + 24 * (size_t)it + (f + 2 * (ivsg + 3 * isg));
          double *fs = fstart + 2 * (f + 2 * (ivsg + 3 * (isg + 4 * (size_t)it)));
          fs[0] = k->sn[0] + k->mn[0][0] * ustar[2 * ip] + k->mn[1][0] * ustar[2 * ip + 1] - k->mu[0];
          fs[1] = k->sn[1] + k->mn[0][1] * ustar[2 * ip] + k->mn[1][1] * ustar[2 * ip + 1] - k->mu[1];
        }
      }
  for (int ie = 0; ie < m->nquad; ie++) {
    for (int isg = 0; isg < 4; isg++)
      for (int ivsg = 0; ivsg < 4; ivsg++) {
        int ip = m->ipqua[9 * ie + IPQSG[isg][ivsg] - 1] - 1;
        for (int f = 0; f < 2; f++) {
          const corner_t *k = cq + 32 * (size_t)ie + (f + 2 * (ivsg + 4 * isg));
          double *fs = fstarq + 2 * (f + 2 * (ivsg + 4 * (isg + 4 * (size_t)ie)));
          fs[0] = k->sn[0] + k->mn[0][0] * ustar[2 * ip] + k->mn[1][0] * ustar[2 * ip + 1] - k->mu[0];
          fs[1] = k->sn[1] + k->mn[0][1] * ustar[2 * ip] + k->mn[1][1] * ustar[2 * ip + 1] - k->mu[1];
        }
      }
  }
  free(indnd); free(vlave); free(munacn); free(munacu); free(snsigm); free(cq); free(ct);
}

/* ---------------------------------------------------------------------- */
/* rhsifacedg_lagsubgq2, Getrhslaggauss.f90:8501-8748                     */
/* ---------------------------------------------------------------------- */
static void iface_quad(const o_mesh *m, const o_cfg *c, int ie, const double *geoel,
                       const double (*gq)[3], const double *ustar, const double *fstarq,
                       double *rhsel) {
  const int ielem = ie + m->ntria;
  static const double xvq[9] = {-1, 1, 1, -1, 0, 1, 0, -1, 0};
  static const double yvq[9] = {-1, -1, 1, 1, -1, 0, 1, 0, 0};
  /* wfgsq (momentum, 0/1) and wfgsqm (mass) of Getrhslaggauss.f90:8580-8637 */
  static const double wq[4][4] = {{1, 1, 0, 1}, {1, 1, 1, 0}, {0, 1, 1, 1}, {1, 0, 1, 1}};
  double wm[4][4][2];
  {
    const double t[4][4][2] = {
        {{4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 0.0}, {0.0, 0.0}, {0.0, 4.0 / 3.0}},
        {{0.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 0.0 / 3.0}, {0.0, 0.0}},
        {{0.0, 0.0}, {0.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 0.0 / 3.0}},
        {{4.0 / 3.0, 0.0 / 3.0}, {0.0, 0.0}, {0.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}}};
    for (int a = 0; a < 4; a++) for (int b = 0; b < 4; b++) for (int f = 0; f < 2; f++) wm[a][b][f] = 0.25 * t[a][b][f];
  }
  double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
  double bq[9][6];
  const int nd = c->ndegr;
  for (int iv = 0; iv < 9; iv++) {
    bq[iv][0] = 1.0;
    bq[iv][1] = (xvq[iv] - rc) / 1.0;
    bq[iv][2] = (yvq[iv] - sc) / 1.0;
    bq[iv][3] = 0.5 * bq[iv][1] * bq[iv][1] - G_(geoel, 18, ielem);
    bq[iv][4] = 0.5 * bq[iv][2] * bq[iv][2] - G_(geoel, 19, ielem);
    bq[iv][5] = bq[iv][1] * bq[iv][2] - G_(geoel, 20, ielem);
  }
  double ul[6] = {0}, p0[6] = {0}, p1[6] = {0}, el[6] = {0};
  for (int isg = 0; isg < 4; isg++) {
    double vn[4][2][3];
    corner_normals(gq, isg, vn);
    for (int ivsg = 0; ivsg < 4; ivsg++)
      for (int f = 0; f < 2; f++) vn[ivsg][f][2] = vn[ivsg][f][2] * wm[isg][ivsg][f];
    for (int ivsg = 0; ivsg < 4; ivsg++) {
      int iv = IPQSG[isg][ivsg] - 1;
      int ip = m->ipqua[9 * ie + iv] - 1;
      double us0 = ustar[2 * ip], us1 = ustar[2 * ip + 1];
      const double *fs = fstarq + 2 * (0 + 2 * (ivsg + 4 * (isg + 4 * (size_t)ie)));
      /* fs[0..1] = fstarq(1:2, 1, ...), fs[2..3] = fstarq(1:2, 2, ...) */
      double w1 = wq[isg][ivsg], w2 = wq[isg][ivsg];
      for (int k = 0; k < nd; k++) {
        double b = bq[iv][k];
        ul[k] = ul[k] + us0 * vn[ivsg][0][0] * vn[ivsg][0][2] * b + us1 * vn[ivsg][0][1] * vn[ivsg][0][2] * b +
                us0 * vn[ivsg][1][0] * vn[ivsg][1][2] * b + us1 * vn[ivsg][1][1] * vn[ivsg][1][2] * b;
        p0[k] = p0[k] + fs[0] * b * w1 + fs[2] * b * w2;
        p1[k] = p1[k] + fs[1] * b * w1 + fs[3] * b * w2;
        el[k] = el[k] + us0 * fs[0] * b * w1 + us1 * fs[1] * b * w1 + us0 * fs[2] * b * w2 + us1 * fs[3] * b * w2;
      }
    }
  }
  for (int k = 0; k < nd; k++) {
    U_(rhsel, c, k, 0, ielem) = ul[k];
    U_(rhsel, c, k, 1, ielem) = p0[k];
    U_(rhsel, c, k, 2, ielem) = p1[k];
    U_(rhsel, c, k, 3, ielem) = el[k];
  }
}

/* ---------------------------------------------------------------------- */
/* rhsdomndg_lagmc_curvquad, Getrhslag.f90:4716-5016 (5x5 Gauss-Lobatto,   */
/* cofactor form, no Jacobian determinant).                               */
/* ---------------------------------------------------------------------- */
static void domn_quad(const o_mesh *m, const o_cfg *c, int ie, const double *geoel,
                      const double *coord, const double *unkno, double *rhsel) {
  const int ielem = ie + m->ntria;
  const double eps = 1.0e-6, g = c->gamlg;
  double pos[25][2], wt[25], dr[9], ds[9];
  quad_rule(25, 1, pos, wt);
  double xp[9][2];
  load_quad(m, coord, ie, xp);
  double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
  double dbdr[6] = {0.0, 1.0 / 1.0, 0.0, 0, 0, 0}, dbds[6] = {0.0, 0.0, 1.0 / 1.0, 0, 0, 0};
  const int nd = c->ndegr;
  for (int ig = 0; ig < 25; ig++) {
    double r = pos[ig][0], s = pos[ig][1], wi = wt[ig];
    double dxdr, dxds, dydr, dyds;
    shp9(r, s, NULL, dr, ds);
    jac9((const double(*)[2])xp, dr, ds, &dxdr, &dxds, &dydr, &dyds);
    double djaco = wi;
    if (c->npoly == 2) {
      dbdr[3] = (r - rc) / (1.0 * 1.0); dbdr[4] = 0.0; dbdr[5] = (s - sc) / 1.0 / 1.0;
      dbds[3] = 0.0; dbds[4] = (s - sc) / (1.0 * 1.0); dbds[5] = (r - rc) / 1.0 / 1.0;
    }
    double j11 = dyds, j12 = -dydr, j21 = -dxds, j22 = dxdr;
    double gd[6][2];
    for (int k = 0; k < nd; k++) {
      gd[k][0] = j11 * dbdr[k] + j12 * dbds[k];
      gd[k][1] = j21 * dbdr[k] + j22 * dbds[k];
    }
    double b[6];
    b[0] = 1.0; b[1] = (r - rc) / 1.0; b[2] = (s - sc) / 1.0;
    if (c->npoly == 2) {
      b[3] = 0.5 * b[1] * b[1] - G_(geoel, 18, ielem);
      b[4] = 0.5 * b[2] * b[2] - G_(geoel, 19, ielem);
      b[5] = b[1] * b[2] - G_(geoel, 20, ielem);
    }
    double un[4] = {0, 0, 0, 0};
    for (int k = 0; k < nd; k++)
      for (int q = 0; q < 4; q++) un[q] = un[q] + U_(unkno, c, k, q, ielem) * b[k];
    double rhoma = un[0], rhoad = 1.0 / rhoma;
    double uadv = un[1], vadv = un[2], eadv = un[3];
    double pres = fmax(eps, (g - 1.0) * rhoad * (eadv - 0.5 * (uadv * uadv + vadv * vadv)));
    for (int k = 0; k < nd; k++) {
      double f0 = gd[k][0] * uadv + gd[k][1] * vadv;
      double f1 = gd[k][0] * (-pres);
      double f2 = gd[k][1] * (-pres);
      double f3 = (gd[k][0] * uadv + gd[k][1] * vadv) * (-pres);
      U_(rhsel, c, k, 0, ielem) = U_(rhsel, c, k, 0, ielem) - f0 * djaco;
      U_(rhsel, c, k, 1, ielem) = U_(rhsel, c, k, 1, ielem) - f1 * djaco;
      U_(rhsel, c, k, 2, ielem) = U_(rhsel, c, k, 2, ielem) - f2 * djaco;
      U_(rhsel, c, k, 3, ielem) = U_(rhsel, c, k, 3, ielem) - f3 * djaco;
    }
  }
}

/* rhsdomnsrcdg_lag_curvquad, Getrhslag.f90:4070-4251 (TGV energy source) */
static void src_quad(const o_mesh *m, const o_cfg *c, int ie, const double *geoel,
                     const double *coord, double *rhsel) {
  const int ielem = ie + m->ntria;
  double pos[25][2], wt[25], shp[9], dr[9], ds[9];
  quad_rule(25, 0, pos, wt);
  double xp[9][2];
  load_quad(m, coord, ie, xp);
  double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
  for (int ig = 0; ig < 25; ig++) {
    double r = pos[ig][0], s = pos[ig][1], wi = wt[ig];
    double a, b_, cc, d, xg, yg;
    shp9(r, s, shp, dr, ds);
    jac9((const double(*)[2])xp, dr, ds, &a, &b_, &cc, &d);
    double djaco = wi * (a * d - cc * b_);
    map9((const double(*)[2])xp, shp, &xg, &yg);
    double b[6];
    b[0] = 1.0; b[1] = (r - rc) / 1.0; b[2] = (s - sc) / 1.0;
    b[3] = 0.5 * b[1] * b[1] - G_(geoel, 18, ielem);
    b[4] = 0.5 * b[2] * b[2] - G_(geoel, 19, ielem);
    b[5] = b[1] * b[2] - G_(geoel, 20, ielem);
    double src = 0.25 * PI_ * (cos(3.0 * PI_ * xg) * cos(PI_ * yg) - cos(3.0 * PI_ * yg) * cos(PI_ * xg)) / (c->gamlg - 1.0);
    for (int k = 0; k < c->ndegr; k++) U_(rhsel, c, k, 3, ielem) = U_(rhsel, c, k, 3, ielem) + src * b[k] * djaco;
  }
}

/* ---------------------------------------------------------------------- */
/* getrhsdg_lag_mcnew, curved branch (Getrhslagmc.f90:7556-7710)          */
/* ---------------------------------------------------------------------- */
void o_rhs(const o_mesh *m, const o_cfg *c, double *ustar, double *unkno,
           double *rhsel, double *geoel, const double *coord,
           const double *coold, const double *amatr, int itime, int *flags) {
  (void)amatr; (void)itime;
  const int ncell = m->ntria + m->nquad, nsize = ncell + m->nbfac;
  memset(rhsel, 0, sizeof(double) * c->ndegr * c->nq * ncell);
  double *gt = (double *)malloc(sizeof(double) * 45 * (size_t)(m->ntria > 0 ? m->ntria : 1));
  for (int it = 0; it < m->ntria; it++) {
    double xp[6][2];
    load_tria(m, coord, it, xp);
    normals_tria((const double(*)[2])xp, (double(*)[3])(gt + 45 * (size_t)it));
  }
  double *gq = (double *)malloc(sizeof(double) * 48 * (size_t)m->nquad);
  for (int ie = 0; ie < m->nquad; ie++) {
    double xp[9][2];
    load_quad(m, coord, ie, xp);
    normals_quad((const double(*)[2])xp, (double(*)[3])(gq + 48 * (size_t)ie));
  }
  if (c->npoly > 1) persson(m, c, coord, geoel, unkno);
  if (flags) for (int ie = 0; ie < ncell; ie++) flags[ie] = G_(geoel, 9, ie) >= 10.0;
  weno(m, c, unkno, geoel, coord, coold);
  for (int ie = 0; ie < nsize; ie++) G_(geoel, 9, ie) = 0.0;
  double *fstarq = (double *)malloc(sizeof(double) * 64 * (size_t)m->nquad);
  double *fstart = (double *)malloc(sizeof(double) * 48 * (size_t)(m->ntria > 0 ? m->ntria : 1));
  ndvelo(m, c, geoel, gq, gt, coord, coold, unkno, ustar, fstarq, fstart);
  for (int it = 0; it < m->ntria; it++)
    iface_tria(m, c, it, geoel, (const double(*)[3])(gt + 45 * (size_t)it), ustar, fstart, rhsel);
  for (int ie = 0; ie < m->nquad; ie++)
    iface_quad(m, c, ie, geoel, (const double(*)[3])(gq + 48 * (size_t)ie), ustar, fstarq, rhsel);
  for (int it = 0; it < m->ntria; it++) domn_tria(m, c, it, geoel, coord, unkno, rhsel);
  for (int ie = 0; ie < m->nquad; ie++) domn_quad(m, c, ie, geoel, coord, unkno, rhsel);
  if (c->ncase == 1) {
    for (int it = 0; it < m->ntria; it++) src_tria(m, c, it, geoel, coord, rhsel);
    for (int ie = 0; ie < m->nquad; ie++) src_quad(m, c, ie, geoel, coord, rhsel);
  }
  if (c->nlimi == 6 && c->npoly >= 1) {
    /* II.4.6 with aflim = 1 and afvec = I (Getrhslagmc.f90:7695-7708) */
    for (int ie = 0; ie < ncell; ie++) {
      U_(unkno, c, 1, 0, ie) = U_(unkno, c, 1, 0, ie) * 1.0;
      U_(unkno, c, 2, 0, ie) = U_(unkno, c, 2, 0, ie) * 1.0;
      double dudr = 1.0 * U_(unkno, c, 1, 1, ie) + 0.0 * U_(unkno, c, 1, 2, ie);
      double duds = 1.0 * U_(unkno, c, 2, 1, ie) + 0.0 * U_(unkno, c, 2, 2, ie);
      double dvdr = 0.0 * U_(unkno, c, 1, 1, ie) + 1.0 * U_(unkno, c, 1, 2, ie);
      double dvds = 0.0 * U_(unkno, c, 2, 1, ie) + 1.0 * U_(unkno, c, 2, 2, ie);
      U_(unkno, c, 1, 1, ie) = dudr; U_(unkno, c, 2, 1, ie) = duds;
      U_(unkno, c, 1, 2, ie) = dvdr; U_(unkno, c, 2, 2, ie) = dvds;
      U_(unkno, c, 1, 3, ie) = U_(unkno, c, 1, 3, ie) * 1.0;
      U_(unkno, c, 2, 3, ie) = U_(unkno, c, 2, 3, ie) * 1.0;
    }
  }
  free(gq);
  free(gt);
  free(fstarq);
  free(fstart);
}

/* ---------------------------------------------------------------------- */
/* getdelt_lag, Getrhslag.f90:20600-20716                                 */
/* ---------------------------------------------------------------------- */
double o_delt(const o_mesh *m, const o_cfg *c, const double *unkno,
              const double *geoel, const double *coord, const double *dvdt,
              int itime, double dtfix) {
  const double eps = 1.0e-6, g = c->gamlg;
  double dtcfl = 1e10, dtvol = 1e10;
  for (int ie = 0; ie < m->nquad; ie++) {
    const int ielem = ie + m->ntria;
    double xp[9][2];
    load_quad(m, coord, ie, xp);
    double dl[4];
    static const int e[4][3] = {{0, 4, 1}, {1, 5, 2}, {2, 6, 3}, {3, 7, 0}};
    for (int k = 0; k < 4; k++) {
      const double *a = xp[e[k][0]], *b = xp[e[k][1]], *cc = xp[e[k][2]];
      if (m->nvqua == 4) {  /* ncurv = 0: straight edges (Getrhslag.f90:20649-20654) */
        dl[k] = sqrt((a[0] - cc[0]) * (a[0] - cc[0]) + (a[1] - cc[1]) * (a[1] - cc[1]));
        continue;
      }
      dl[k] = sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1])) +
              sqrt((b[0] - cc[0]) * (b[0] - cc[0]) + (b[1] - cc[1]) * (b[1] - cc[1]));
    }
    double rhomc = U_(unkno, c, 0, 0, ielem);
    double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
    double rhoct = 1.0 / rhomc;
    double pctr = fmax(eps, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
    double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
    double dlen = dl[0];
    for (int k = 1; k < 4; k++) if (dl[k] < dlen) dlen = dl[k];
    dtcfl = fmin(dtcfl, dlen / sdctr);
  }
  for (int ie = 0; ie < m->nquad; ie++) {
    const int ielem = ie + m->ntria;
    dtvol = fmin(dtvol, G_(geoel, 2, ielem) / fabs(dvdt[ielem]));
  }
  if (itime == 1) return fmin(c->cfl * dtcfl, 0.1 * dtvol);
  return fmin(fmin(c->cfl * dtcfl, 0.1 * dtvol), 1.01 * dtfix);
}

static void o1_rhs_x(const o_mesh *m, const o_cfg *c, double *ustar, double *unkno,
                     double *rhsel, double *geoel, const double *coord, double *amatr, int rev,
                     double *aflim_out, double *afvec_out);

/* ---------------------------------------------------------------------- */
/* getsolvdg_lag, Getrhslag.f90:1553-2035                                 */
/* ---------------------------------------------------------------------- */
void o_step(const o_mesh *m, const o_cfg *c, const double *unkno, double *unold,
            const double *coord, double *cooro, const double *coold,
            double *geoel, const double *amatr, double *ustar, int itime,
            double *dtfix, double *tacru) {
  static const double rklag[2][3] = {{0.0, 0.5, 0.0}, {0.0, 0.75, 0.3333333333333333}};
  const int ncell = m->ntria + m->nquad;
  const int nd = c->ndegr, nq = c->nq;
  const int nmatr = (c->npoly == 2) ? 16 : 4;
  double *rhsel = (double *)malloc(sizeof(double) * nd * nq * (size_t)ncell);
  double *dvdt = (double *)malloc(sizeof(double) * (size_t)ncell);
  o_cellvol(m, c, geoel, coord);
  for (int istag = 1; istag <= c->nstag; istag++) {
    double alfa = rklag[c->nstag - 2][istag - 1];
    /* nrz = 2 rewrites amatr each stage (getamatr_lagmc_rzawrev) */
    if (c->npoly == 1)
      o1_rhs_x(m, c, ustar, unold, rhsel, geoel, cooro, (double *)amatr, itime > 1 || istag > 1, NULL, NULL);
    else o_rhs(m, c, ustar, unold, rhsel, geoel, cooro, coold, amatr, itime, NULL);
    if (c->ndt == 1) {
      if (istag == 1) {
        for (int ie = 0; ie < ncell; ie++) dvdt[ie] = U_(rhsel, c, 0, 0, ie);
        *dtfix = o_delt(m, c, unold, geoel, coord, dvdt, itime, *dtfix);
        if ((*tacru + *dtfix) > c->tend) *dtfix = c->tend - *tacru;
        *tacru = *tacru + *dtfix;
      }
    } else if (istag == 1) {
      *tacru = *tacru + *dtfix;
    }
    for (size_t i = 0; i < (size_t)nd * nq * ncell; i++) rhsel[i] = *dtfix * rhsel[i];
    for (int ie = 0; ie < ncell; ie++) {
      double mm[6][6];
      const double *am = amatr + nmatr * (size_t)ie;
      memset(mm, 0, sizeof mm);
      if (c->npoly == 2) {
        mm[0][0] = am[15];
        int k = 0;
        for (int im = 1; im < nd; im++)
          for (int jm = im; jm < nd; jm++) { mm[im][jm] = am[k]; mm[jm][im] = am[k]; k++; }
      } else {
        mm[0][0] = am[3];
        mm[1][1] = am[0]; mm[1][2] = am[1]; mm[2][1] = am[1]; mm[2][2] = am[2];
      }
      for (int id = 0; id < nd; id++) {
        double unint[4] = {0, 0, 0, 0};
        for (int iu = 0; iu < nd; iu++)
          for (int q = 0; q < nq; q++) unint[q] = unint[q] + mm[id][iu] * U_(rhsel, c, iu, q, ie);
        for (int q = 0; q < nq; q++)
          U_(unold, c, id, q, ie) = alfa * U_(unkno, c, id, q, ie) + (1.0 - alfa) * (U_(unold, c, id, q, ie) + unint[q]);
      }
    }
    for (int ip = 0; ip < m->npoin; ip++)
      for (int d = 0; d < 2; d++)
        X_(cooro, d, ip) = alfa * X_(coord, d, ip) + (1.0 - alfa) * (X_(cooro, d, ip) + *dtfix * X_(ustar, d, ip));
    for (int ie = 0; ie < m->nquad && m->nvqua != 4; ie++) {  /* ncurv = 1 only (:1963-1971) */
      const int *ipq = m->ipqua + 9 * ie;
      for (int d = 0; d < 2; d++) {
        double x[8];
        for (int k = 0; k < 8; k++) x[k] = X_(cooro, d, ipq[k] - 1);
        X_(cooro, d, ipq[8] - 1) = -0.25 * (x[0] + x[1] + x[2] + x[3]) + 0.5 * (x[4] + x[5] + x[6] + x[7]);
      }
    }
    o_cellvol(m, c, geoel, cooro);
  }
  free(rhsel);
  free(dvdt);
}

int o_run(const o_mesh *m, const o_cfg *c, double *unkno, double *coord,
          const double *coold, double *geoel, const double *amatr,
          double *ustar, int itime0, int nsteps, double *dtfix, double *tacru) {
  const int ncell = m->ntria + m->nquad, nsize = ncell + m->nbfac;
  size_t nu = (size_t)c->ndegr * c->nq * nsize;
  double *unold = (double *)malloc(nu * sizeof(double));
  double *cooro = (double *)malloc(sizeof(double) * 2 * (size_t)m->npoin);
  memcpy(unold, unkno, nu * sizeof(double));
  memcpy(cooro, coord, sizeof(double) * 2 * (size_t)m->npoin);
  int done = 0;
  for (int it = itime0; it < itime0 + nsteps; it++) {
    o_step(m, c, unkno, unold, coord, cooro, coold, geoel, amatr, ustar, it, dtfix, tacru);
    done++;
    for (int ie = 0; ie < ncell; ie++)
      for (int q = 0; q < c->nq; q++)
        for (int k = 0; k < c->ndegr; k++) U_(unkno, c, k, q, ie) = U_(unold, c, k, q, ie);
    memcpy(coord, cooro, sizeof(double) * 2 * (size_t)m->npoin);
    if (fabs(*tacru - c->tend) / c->tend <= 1e-11) break;
  }
  free(unold);
  free(cooro);
  return done;
}

/* WENO on the cells whose flag is set (test entry point; the step derives
 * the flags from the Persson indicator). */
void o_weno(const o_mesh *m, const o_cfg *c, double *unkno, double *geoel,
            const double *coord, const double *coold, const int *flags) {
  const int ncell = m->ntria + m->nquad;
  for (int ie = 0; ie < ncell; ie++) G_(geoel, 9, ie) = flags[ie] ? 100.0 : 0.0;
  weno(m, c, unkno, geoel, coord, coold);
  for (int ie = 0; ie < ncell; ie++) G_(geoel, 9, ie) = 0.0;
}

/* ====================================================================== */
/* Linear P1 path: ncurv=0, nriem=1, nfint=1, nlimi=6, nrz=0 on 4-node    */
/* quads (the Sod configuration).  getrhsdg_lag_mcnew's branch at         */
/* Getrhslagmc.f90:6810-6980 and the slope application at :7283-7298.    */
/* Calls that do not change the result are left out: getbc_lagmaire2      */
/* (Getrhslag.f90:11269) only forms the unused boundary force `fpres`;    */
/* getAS_llnl (Limiterlag.f90:15476) ends with `sgmas = 0`; the           */
/* divergence limiter of barthlimit_sympre_quadlb (Limiterlag.f90:        */
/* 8127-8692, the `afdu` loops) only writes geoel(10), which this branch  */
/* never reads, and so does not need the divergence bound unmax(nq+2) of  */
/* barthlimit_lag_vtxunknew either (computed there from `dr`, `ds` that   */
/* are set only in its triangle loop).                                    */
/* ====================================================================== */

/* Literals the Fortran writes in single precision (`eps = 1.e-6`,
 * `1.e-11`), widened to double as gfortran does. */
#define EPS_S ((double)1.0e-6f)
#define TINY_S ((double)1.0e-11f)

/* barthfct, Getrhslagmc.f90:9171-9222 */
static double barthfct(double umax, double umin, double uctr, double dunk) {
  const double coef = 0.7;
  double fiy;
  if (dunk > 1.0e-8) {
    fiy = coef * (umax - uctr) / dunk;
    return fmin((fiy * fiy + 2.0 * fiy) / (fiy * fiy + fiy + 2.0), 1.0);
  } else if (dunk < -1.0e-8) {
    fiy = coef * (umin - uctr) / dunk;
    return fmin((fiy * fiy + 2.0 * fiy) / (fiy * fiy + fiy + 2.0), 1.0);
  }
  return 1.0;
}

static const double XVQ[4] = {-1.0, 1.0, 1.0, -1.0}, YVQ[4] = {-1.0, -1.0, 1.0, 1.0};

/* vertex values of the P1 DOFs: bq = (1, (xv-rc)/dr, (yv-sc)/ds), dr = ds = 1 */
static void p1_vertex(const o_cfg *c, const double *unkno, int ielem, double rc, double sc,
                      double unknvq[4][5]) {
  for (int iv = 0; iv < 4; iv++) {
    double bq[3] = {1.0, (XVQ[iv] - rc) / 1.0, (YVQ[iv] - sc) / 1.0};
    for (int q = 0; q < 4; q++) {
      double a = 0.0;
      for (int k = 0; k < c->mdegr; k++) a = a + U_(unkno, c, k, q, ielem) * bq[k];
      unknvq[iv][q] = a;
    }
  }
}

/* bilinear Jacobian at (r, s) (the 4-node shape derivatives of
 * barthlimit_sympre_quadlb, Limiterlag.f90:8262-8282) */
static void jac4(const double (*xpq)[2], double r, double s, double *dxdr, double *dxds,
                 double *dydr, double *dyds) {
  const double rp = 1.0 + r, rm = 1.0 - r, sp = 1.0 + s, sm = 1.0 - s;
  const double dsprq[4] = {-0.25 * sm, 0.25 * sm, 0.25 * sp, -0.25 * sp};
  const double dspsq[4] = {-0.25 * rm, -0.25 * rp, 0.25 * rp, 0.25 * rm};
  double a = 0, b = 0, cc = 0, d = 0;
  for (int k = 0; k < 4; k++) {
    a = a + dsprq[k] * xpq[k][0];
    b = b + dspsq[k] * xpq[k][0];
    cc = cc + dsprq[k] * xpq[k][1];
    d = d + dspsq[k] * xpq[k][1];
  }
  *dxdr = a; *dxds = b; *dydr = cc; *dyds = d;
}

/* ---------------------------------------------------------------------- */
/* RZ (nrz = 1, alfrz = 1, the radius is y) nodal solve and face integral */
/* of the linear P1 branch: getndvelo_lagmc_rz (Getrhslagmc.f90:          */
/* 17284-17597) with getriem_quadrz (:17963-18336) and getbc_lagmaire2    */
/* (Getrhslag.f90:11269-11491), then rhsifacedg_lagmc_quadrz              */
/* (Getrhslagmc.f90:18534-18734).  Quads only.  Each vertex has 4 corner  */
/* faces: its two edges, each twice, with the radius weights of the two   */
/* halves of the edge's r-weighted length.  aflim (5, nquad), afvec       */
/* (2,2,nquad) and gelq (3,4,nquad) are o1_rhs's arrays; ustar holds the  */
/* previous nodal velocity on entry and the new one on return.            */
/* ---------------------------------------------------------------------- */
static void o1_rz_nodes_faces(const o_mesh *m, const o_cfg *c, double *ustar, const double *unkno,
                              double *rhsel, const double *geoel, const double *coord, const double *aflim,
                              const double *afvec, const double *gelq) {
  const int nquad = m->nquad, npoin = m->npoin;
  const double g = c->gamlg, alfrz = 1.0, eps9 = 1.0e-09;
#define QN(ie, k) (m->ipqua[4 * (ie) + (k)] - 1)
#define GL(f, ie) (gelq + 3 * ((f) + 4 * (ie)))
#define AF(k, ie) aflim[(k) + 5 * (ie)]
#define AV(i, j, ie) afvec[(i) + 2 * (j) + 4 * (ie)]
  int *indnd = (int *)calloc((size_t)npoin, sizeof(int));
  double *vlave = (double *)malloc(sizeof(double) * 2 * (size_t)npoin);
  double *munacn = (double *)calloc((size_t)4 * npoin, sizeof(double));
  double *munacu = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *snsigm = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *mcl = (double *)malloc(sizeof(double) * 4 * 16 * (size_t)nquad);  /* munaclq(2,2,4,4) */
  double *mul = (double *)malloc(sizeof(double) * 2 * 16 * (size_t)nquad);  /* munaulq(2,4,4) */
  double *snl = (double *)malloc(sizeof(double) * 2 * 16 * (size_t)nquad);  /* snsigmlq(2,4,4) */
  double *fst = (double *)malloc(sizeof(double) * 2 * 16 * (size_t)nquad);  /* fsqrz(2,4,4) */
  double *fpres = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *bsnv = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *bsnpf = (double *)calloc((size_t)2 * npoin, sizeof(double));

  for (int ifa = 0; ifa < m->nbfac; ifa++) {
    if (c->ncase == 2) for (int k = 0; k < 2; k++) indnd[m->bface[5 * ifa + k] - 1] = 1;
  }
  for (int ifa = 0; ifa < m->nbfac; ifa++)
    if (m->bface[5 * ifa + 2] == 25) for (int k = 0; k < 2; k++) indnd[m->bface[5 * ifa + k] - 1] = 1;
  /* getvlavenew's average is overwritten by the previous nodal velocity (:17404-17407) */
  memcpy(vlave, ustar, sizeof(double) * 2 * (size_t)npoin);

  /* getriem_quadrz, scattering in cell order */
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double bq[4][3];
    for (int iv = 0; iv < 4; iv++) { bq[iv][0] = 1.0; bq[iv][1] = (XVQ[iv] - rc) / 1.0; bq[iv][2] = (YVQ[iv] - sc) / 1.0; }
    double rcoeq[4];
    for (int iv = 0; iv < 4; iv++) rcoeq[iv] = 1.0 - alfrz + alfrz * fabs(X_(coord, 1, QN(ie, iv)));
    /* faces 1, 3: the edge to the previous vertex; 2, 4: the edge to the next */
    double vn[4][4][3];
    for (int iv = 0; iv < 4; iv++) {
      const int ep = (iv + 3) % 4, en = iv, vp = (iv + 3) % 4, vx = (iv + 1) % 4;
      for (int k = 0; k < 3; k++) {
        vn[iv][0][k] = GL(ep, ie)[k]; vn[iv][1][k] = GL(en, ie)[k];
        vn[iv][2][k] = GL(ep, ie)[k]; vn[iv][3][k] = GL(en, ie)[k];
      }
      vn[iv][0][2] = (3.0 * rcoeq[iv] + rcoeq[vp]) / 3.0 * 0.5 * vn[iv][0][2];
      vn[iv][1][2] = (3.0 * rcoeq[iv] + rcoeq[vx]) / 3.0 * 0.5 * vn[iv][1][2];
      vn[iv][2][2] = (1.0 * rcoeq[iv] + rcoeq[vp]) / 3.0 * 0.5 * vn[iv][2][2];
      vn[iv][3][2] = (1.0 * rcoeq[iv] + rcoeq[vx]) / 3.0 * 0.5 * vn[iv][3][2];
    }
    for (int iv = 0; iv < 4; iv++)
      for (int f = 0; f < 4; f++) vn[iv][f][2] = 0.5 * vn[iv][f][2];
    double rhomc = U_(unkno, c, 0, 0, ielem);
    double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
    double rhoct = 1.0 / rhomc;
    double pctr = fmax(eps9, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
    double unknvq[4][5], sig[4], aujmp[4][3];
    p1_vertex(c, unkno, ielem, rc, sc, unknvq);
    const double a11 = AV(0, 0, ie), a12 = AV(0, 1, ie), a21 = AV(1, 0, ie), a22 = AV(1, 1, ie);
    for (int iv = 0; iv < 4; iv++) {
      double rhovt = 1.0 / unknvq[iv][0];
      double uv = unknvq[iv][1], vv = unknvq[iv][2], ev = unknvq[iv][3];
      double pvtx = fmax(eps9, (g - 1.0) * rhovt * (ev - 0.5 * (uv * uv + vv * vv)));
      double dudr = a11 * U_(unkno, c, 1, 1, ielem) + a12 * U_(unkno, c, 1, 2, ielem);
      double duds = a11 * U_(unkno, c, 2, 1, ielem) + a12 * U_(unkno, c, 2, 2, ielem);
      double dvdr = a21 * U_(unkno, c, 1, 1, ielem) + a22 * U_(unkno, c, 1, 2, ielem);
      double dvds = a21 * U_(unkno, c, 2, 1, ielem) + a22 * U_(unkno, c, 2, 2, ielem);
      uv = U_(unkno, c, 0, 1, ielem) + dudr * bq[iv][1] + duds * bq[iv][2];
      vv = U_(unkno, c, 0, 2, ielem) + dvdr * bq[iv][1] + dvds * bq[iv][2];
      pvtx = pctr + AF(3, ie) * (pvtx - pctr);
      unknvq[iv][1] = uv;
      unknvq[iv][2] = vv;
      sig[iv] = -pvtx;
      int ip = QN(ie, iv);
      double acnx = X_(vlave, 0, ip) - uv, acny = X_(vlave, 1, ip) - vv;
      double nrm = sqrt(acnx * acnx + acny * acny);
      if (nrm < TINY_S) { aujmp[iv][0] = TINY_S; aujmp[iv][1] = TINY_S; }
      else { aujmp[iv][0] = acnx / nrm; aujmp[iv][1] = acny / nrm; }
      aujmp[iv][2] = nrm;
    }
    double sdctr = sqrt(fmax(eps9, g * pctr / rhoct));
    for (int iv = 0; iv < 4; iv++) aujmp[iv][2] = aujmp[iv][2] / sdctr;
    /* the impedance is the acoustic one: the shock term is commented out (:18273) */
    const double murie = rhoct * sdctr;
    for (int iv = 0; iv < 4; iv++) {
      int ip = QN(ie, iv);
      for (int f = 0; f < 4; f++) {
        /* getriecoef_matrixnew, Limiterlag.f90:1037-1076 */
        double area = vn[iv][f][2], n1 = vn[iv][f][0], n2 = vn[iv][f][1];
        double vnau = (aujmp[iv][2] < 1.0e12) ? 1.0 : n1 * aujmp[iv][0] + n2 * aujmp[iv][1];
        double mc11 = murie * area * fabs(vnau), mc21 = 0.0, mc12 = 0.0, mc22 = murie * area * fabs(vnau);
        double mu1 = mc11 * unknvq[iv][1] + mc21 * unknvq[iv][2];
        double mu2 = mc21 * unknvq[iv][1] + mc22 * unknvq[iv][2];
        double s1 = sig[iv] * area * n1 + (0.0 + 0.0) * area * n2;
        double s2 = (0.0 + 0.0) * area * n1 + sig[iv] * area * n2;
        munacn[0 + 4 * ip] = munacn[0 + 4 * ip] + mc11;
        munacn[1 + 4 * ip] = munacn[1 + 4 * ip] + mc21;
        munacn[2 + 4 * ip] = munacn[2 + 4 * ip] + mc12;
        munacn[3 + 4 * ip] = munacn[3 + 4 * ip] + mc22;
        munacu[0 + 2 * ip] = munacu[0 + 2 * ip] + mu1;
        munacu[1 + 2 * ip] = munacu[1 + 2 * ip] + mu2;
        snsigm[0 + 2 * ip] = snsigm[0 + 2 * ip] + s1;
        snsigm[1 + 2 * ip] = snsigm[1 + 2 * ip] + s2;
        const size_t o = (size_t)f + 4 * (iv + 4 * (size_t)ie);
        mcl[4 * o + 0] = mc11; mcl[4 * o + 1] = mc21; mcl[4 * o + 2] = mc12; mcl[4 * o + 3] = mc22;
        mul[2 * o + 0] = mu1; mul[2 * o + 1] = mu2;
        snl[2 * o + 0] = s1; snl[2 * o + 1] = s2;
      }
    }
  }
  /* getbc_lagmaire2 (Getrhslag.f90:11269-11491): boundary area vectors of
   * the velocity walls (code 22, with the radius weights of the face's two
   * ends) and pressure forces of code 21 (ncase 3: p = 1e-6); then at the
   * wall nodes the force fpres that removes the wall-normal velocity from
   * the node solve.  gflag = unit normal and length of the boundary face
   * (getfnds_lag_mc_hybrid, Getrhslagmc.f90:2147-2162). */
  for (int ifa = 0; ifa < m->nbfac; ifa++) {
    const int *bf = m->bface + 5 * ifa;
    const int ipf[2] = {bf[0] - 1, bf[1] - 1};
    double anx = X_(coord, 1, ipf[1]) - X_(coord, 1, ipf[0]);
    double any = -(X_(coord, 0, ipf[1]) - X_(coord, 0, ipf[0]));
    const double gf1 = anx / sqrt(anx * anx + any * any), gf2 = any / sqrt(anx * anx + any * any);
    const double gf3 = sqrt(anx * anx + any * any);
    double rcoef[2];
    rcoef[0] = 1.0 - alfrz + alfrz * X_(coord, 1, ipf[0]);
    rcoef[1] = 1.0 - alfrz + alfrz * X_(coord, 1, ipf[1]);
    double bsnx = 0.0, bsny = 0.0;
    if (bf[2] == 22) {
      if (bf[3] == 221) {
        bsnx = 0.0 * gf3 * 0.5;
        bsny = -1.0 * gf3 * 0.5;
        if (c->ncase == 1 || c->ncase == 2 || c->ncase == 12) {
          if (X_(coord, 1, ipf[0]) < 1.0e-6 && X_(coord, 1, ipf[1]) < 1.0e-6) {
            bsnx = 0.0 * gf3 * 0.5; bsny = -1.0 * gf3 * 0.5;
          } else if (fabs(X_(coord, 1, ipf[0]) - 1.0) < 1.0e-6 && fabs(X_(coord, 1, ipf[1]) - 1.0) < 1.0e-6) {
            bsnx = 0.0 * gf3 * 0.5; bsny = 1.0 * gf3 * 0.5;
          }
        }
      } else if (bf[3] == 222) {
        bsnx = -1.0 * gf3 * 0.5;
        bsny = 0.0 * gf3 * 0.5;
        if (c->ncase == 1) {
          if (X_(coord, 0, ipf[0]) < 1.0e-6 && X_(coord, 0, ipf[1]) < 1.0e-6) {
            bsnx = -1.0 * gf3 * 0.5; bsny = 0.0 * gf3 * 0.5;
          } else if (fabs(X_(coord, 0, ipf[0]) - 1.0) < 1.0e-6 && fabs(X_(coord, 0, ipf[1]) - 1.0) < 1.0e-6) {
            bsnx = 1.0 * gf3 * 0.5; bsny = 0.0 * gf3 * 0.5;
          }
        }
      }
      bsnv[0 + 2 * ipf[0]] = bsnv[0 + 2 * ipf[0]] + bsnx * (2.0 * rcoef[0] + rcoef[1]) / 3.0;
      bsnv[1 + 2 * ipf[0]] = bsnv[1 + 2 * ipf[0]] + bsny * (2.0 * rcoef[0] + rcoef[1]) / 3.0;
      bsnv[0 + 2 * ipf[1]] = bsnv[0 + 2 * ipf[1]] + bsnx * (2.0 * rcoef[1] + rcoef[0]) / 3.0;
      bsnv[1 + 2 * ipf[1]] = bsnv[1 + 2 * ipf[1]] + bsny * (2.0 * rcoef[1] + rcoef[0]) / 3.0;
    } else if (bf[2] == 21) {
      bsnx = gf1 * gf3 * 0.5;
      bsny = gf2 * gf3 * 0.5;
      if (c->ncase == 3) {
        const double pres0 = 1.0e-6;
        bsnpf[0 + 2 * ipf[0]] = bsnpf[0 + 2 * ipf[0]] + pres0 * bsnx * (2.0 * rcoef[0] + rcoef[1]) / 3.0;
        bsnpf[1 + 2 * ipf[0]] = bsnpf[1 + 2 * ipf[0]] + pres0 * bsny * (2.0 * rcoef[0] + rcoef[1]) / 3.0;
        bsnpf[0 + 2 * ipf[1]] = bsnpf[0 + 2 * ipf[1]] + pres0 * bsnx * (2.0 * rcoef[1] + rcoef[0]) / 3.0;
        bsnpf[1 + 2 * ipf[1]] = bsnpf[1 + 2 * ipf[1]] + pres0 * bsny * (2.0 * rcoef[1] + rcoef[0]) / 3.0;
      }
    }
  }
  for (int ifa = 0; ifa < m->nbfac; ifa++) {
    const int *bf = m->bface + 5 * ifa;
    if (bf[2] != 22) continue;
    for (int k = 0; k < 2; k++) {
      const int ip = bf[k] - 1;
      const double *mn = munacn + 4 * ip;  /* (1,1), (2,1), (1,2), (2,2) */
      double detma = mn[0] * mn[3] - mn[1] * mn[2];
      double i11 = mn[3] / detma, i12 = -mn[2] / detma, i21 = -mn[1] / detma, i22 = mn[0] / detma;
      double lnx = bsnv[0 + 2 * ip], lny = bsnv[1 + 2 * ip];
      double coefl = (i11 * lnx + i12 * lny) * lnx + (i21 * lnx + i22 * lny) * lny;
      double rhsx = munacu[0 + 2 * ip] - snsigm[0 + 2 * ip] - bsnpf[0 + 2 * ip];
      double rhsy = munacu[1 + 2 * ip] - snsigm[1 + 2 * ip] - bsnpf[1 + 2 * ip];
      double coefr = (i11 * rhsx + i12 * rhsy) * lnx + (i21 * rhsx + i22 * rhsy) * lny;
      fpres[0 + 2 * ip] = coefr / fmax(1.0e-16, coefl) * lnx;
      fpres[1 + 2 * ip] = coefr / fmax(1.0e-16, coefl) * lny;
    }
  }
  for (int ip = 0; ip < npoin; ip++) {
    fpres[0 + 2 * ip] = fpres[0 + 2 * ip] + bsnpf[0 + 2 * ip];
    fpres[1 + 2 * ip] = fpres[1 + 2 * ip] + bsnpf[1 + 2 * ip];
  }
  /* the node solve with the boundary forces (:17446-17461) */
  for (int ip = 0; ip < npoin; ip++) {
    if (indnd[ip]) continue;
    const double *mn = munacn + 4 * ip;
    double detma = mn[0] * mn[3] - mn[1] * mn[2];
    double i11 = mn[3] / detma, i12 = -mn[2] / detma, i21 = -mn[1] / detma, i22 = mn[0] / detma;
    double r1 = munacu[2 * ip] - snsigm[2 * ip] - fpres[2 * ip];
    double r2 = munacu[2 * ip + 1] - snsigm[2 * ip + 1] - fpres[2 * ip + 1];
    X_(ustar, 0, ip) = i11 * r1 + i12 * r2;
    X_(ustar, 1, ip) = i21 * r1 + i22 * r2;
  }
  /* node 1 held (:17475), then the walls: 222 holds u, code 25 both; the
   * zeroing of v on 221 is commented out in RZ (:17482) */
  X_(ustar, 0, 0) = 0.0;
  X_(ustar, 1, 0) = 0.0;
  for (int ifa = 0; ifa < m->nbfac; ifa++) {
    const int *bf = m->bface + 5 * ifa;
    for (int k = 0; k < 2; k++) {
      int ip = bf[k] - 1;
      if (bf[2] == 22) {
        if (bf[3] == 222) X_(ustar, 0, ip) = 0.0;
      } else if (bf[2] == 25) {
        X_(ustar, 1, ip) = 0.0;
        X_(ustar, 0, ip) = 0.0;
      }
    }
  }
  /* corner forces fsqrz (:17568-17590) */
  for (int ie = 0; ie < nquad; ie++)
    for (int iv = 0; iv < 4; iv++) {
      int ip = QN(ie, iv);
      for (int f = 0; f < 4; f++) {
        const size_t o = (size_t)f + 4 * (iv + 4 * (size_t)ie);
        fst[2 * o + 0] = snl[2 * o + 0] + mcl[4 * o + 0] * X_(ustar, 0, ip) + mcl[4 * o + 1] * X_(ustar, 1, ip) - mul[2 * o + 0];
        fst[2 * o + 1] = snl[2 * o + 1] + mcl[4 * o + 2] * X_(ustar, 0, ip) + mcl[4 * o + 3] * X_(ustar, 1, ip) - mul[2 * o + 1];
      }
    }
  /* rhsifacedg_lagmc_quadrz: per corner face the basis of the face's own
   * vertex (faces 1, 2) or of the edge's other vertex (3, 4), with the
   * radius weights rcapt */
  const double c05 = 0.5;
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double bq[4][3];
    for (int iv = 0; iv < 4; iv++) { bq[iv][0] = 1.0; bq[iv][1] = (XVQ[iv] - rc) / 1.0; bq[iv][2] = (YVQ[iv] - sc) / 1.0; }
    double rcoeq[4];
    for (int iv = 0; iv < 4; iv++) rcoeq[iv] = 1.0 - alfrz + alfrz * fabs(X_(coord, 1, QN(ie, iv)));
    double ul[3] = {0, 0, 0}, p1[3] = {0, 0, 0}, p2[3] = {0, 0, 0}, el[3] = {0, 0, 0};
    for (int iv = 0; iv < 4; iv++) {
      const int ep = (iv + 3) % 4, en = iv, vp = (iv + 3) % 4, vx = (iv + 1) % 4;
      const int edge[4] = {ep, en, ep, en}, bvert[4] = {iv, iv, vp, vx};
      double rcapt[4];
      rcapt[0] = (3.0 * rcoeq[iv] + rcoeq[vp]) / 6.0;
      rcapt[1] = (3.0 * rcoeq[iv] + rcoeq[vx]) / 6.0;
      rcapt[2] = (1.0 * rcoeq[iv] + rcoeq[vp]) / 6.0;
      rcapt[3] = (1.0 * rcoeq[iv] + rcoeq[vx]) / 6.0;
      int ip = QN(ie, iv);
      double us = X_(ustar, 0, ip), vs = X_(ustar, 1, ip);
      for (int f = 0; f < 4; f++) {
        const size_t o = (size_t)f + 4 * (iv + 4 * (size_t)ie);
        const double *gl = GL(edge[f], ie);
        for (int k = 0; k < c->ndegr; k++) {
          double lx = c05 * gl[0] * gl[2] * bq[bvert[f]][k];
          double ly = c05 * gl[1] * gl[2] * bq[bvert[f]][k];
          double bc = bq[bvert[f]][k];
          ul[k] = ul[k] + us * lx * rcapt[f] + vs * ly * rcapt[f];
          p1[k] = p1[k] + fst[2 * o] * bc;
          p2[k] = p2[k] + fst[2 * o + 1] * bc;
          el[k] = el[k] + us * fst[2 * o] * bc + vs * fst[2 * o + 1] * bc;
        }
      }
    }
    for (int k = 0; k < c->ndegr; k++) {
      U_(rhsel, c, k, 0, ielem) = ul[k];
      U_(rhsel, c, k, 1, ielem) = p1[k];
      U_(rhsel, c, k, 2, ielem) = p2[k];
      U_(rhsel, c, k, 3, ielem) = el[k];
    }
  }
#undef QN
#undef GL
#undef AF
#undef AV
  free(indnd); free(vlave); free(munacn); free(munacu); free(snsigm); free(mcl); free(mul); free(snl);
  free(fst); free(fpres); free(bsnv); free(bsnpf);
}

/* ---------------------------------------------------------------------- */
/* Area-weighted RZ (nrz = 2) of the linear P1 branch.  The per-stage     */
/* geometry of getgeoel_lagmc_rzawrev (Getrhslagrz.f90:4590-4998, quads   */
/* :4812-4994): the mass centre (geoel(1:2)) of the limited DG density    */
/* over the cell's area, 5 fixed-point passes from the area centroid;     */
/* then getamatr_lagmc_rzawrev (:3633-4221, quads :3949-4219): M^-1 of    */
/* the area mass matrix about that centre, divided by geoel(11).  Both    */
/* run at the start of every stage but the very first (Getrhslagmc.f90:   */
/* 6883-6886); aflim is this stage's limiter (5, nquad).                  */
/* ---------------------------------------------------------------------- */
static void o1_rzaw_rev(const o_mesh *m, const o_cfg *c, const double *unkno, double *geoel, double *amatr,
                        const double *coord, const double *aflim) {
  double pos36[36][2], w36[36], pos25[25][2], w25[25];
  quad_rule(36, 0, pos36, w36);
  quad_rule(25, 0, pos25, w25);
  for (int ie = 0; ie < m->nquad; ie++) {
    const int ielem = ie + m->ntria;
    double xp[9][2], shp[9], dr[9], ds[9];
    load_quad(m, coord, ie, xp);
    const double af1 = aflim[0 + 5 * ie];
    const double rhomc = U_(unkno, c, 0, 0, ielem);
    for (int iloop = 1; iloop <= 5; iloop++) {
      double xcent = 0.0, ycent = 0.0, masel = 0.0;
      const double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
      for (int ig = 0; ig < 36; ig++) {
        const double r = pos36[ig][0], s = pos36[ig][1], wi = w36[ig];
        double a, b, cc, d;
        shp9(r, s, shp, dr, ds);
        jac9((const double(*)[2])xp, dr, ds, &a, &b, &cc, &d);
        const double djaco = wi * (a * d - cc * b);
        const double bq[3] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
        double rhomg = 0.0;
        for (int k = 0; k < c->mdegr; k++) rhomg = rhomg + U_(unkno, c, k, 0, ielem) * bq[k];
        if (iloop == 1) rhomg = rhomc;
        rhomg = rhomc + af1 * (rhomg - rhomc);
        const double rhog = 1.0 / rhomg;
        masel = masel + 1.0 / rhomc * djaco;
        xcent = xcent + rhog * r * djaco;
        ycent = ycent + rhog * s * djaco;
      }
      G_(geoel, 0, ielem) = xcent / masel;
      G_(geoel, 1, ielem) = ycent / masel;
    }
    const double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
    for (int ig = 0; ig < 25; ig++) {
      const double r = pos25[ig][0], s = pos25[ig][1], wi = w25[ig];
      double a, b, cc, d;
      shp9(r, s, shp, dr, ds);
      jac9((const double(*)[2])xp, dr, ds, &a, &b, &cc, &d);
      const double djaco = wi * (a * d - cc * b);
      const double bq[3] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
      double rhomg = 0.0;
      for (int k = 0; k < c->mdegr; k++) rhomg = rhomg + U_(unkno, c, k, 0, ielem) * bq[k];
      rhomg = rhomc + af1 * (rhomg - rhomc);
      const double rhog = 1.0 / rhomg;
      f0 = f0 + rhog * djaco;
      f1 = f1 + rhog * (r - rc) / 1.0 * (r - rc) / 1.0 * djaco;
      f2 = f2 + rhog * (r - rc) / 1.0 * (s - sc) / 1.0 * djaco;
      f3 = f3 + rhog * (s - sc) / 1.0 * (s - sc) / 1.0 * djaco;
    }
    const double det = f1 * f3 - f2 * f2;
    double *am = amatr + 4 * (size_t)ielem;
    am[0] = f3 / det;
    am[1] = -f2 / det;
    am[2] = f1 / det;
    am[3] = 1.0 / f0;
    for (int k = 0; k < 4; k++) am[k] = am[k] / G_(geoel, 10, ielem);
  }
}

/* ---------------------------------------------------------------------- */
/* Area-weighted RZ (nrz = 2) nodal solve and face integral of the linear */
/* P1 branch: getndvelo_lagmc_rzaw (Getrhslagrz.f90:822-1100) with        */
/* getriem_quadrzaw (:1389-1669) and getbc_lagmaire_rzaw (GetBClag.f90:   */
/* 57-250), then rhsifacedg_lagmc_quadrzaw (Getrhslagrz.f90:1673-1812).   */
/* Quads only.  Each vertex has the two corner faces of the plane solver  */
/* (half of each edge at the vertex, no radius weight), the impedance is  */
/* the acoustic one and the floors are 1e-8; the face integral weighs the */
/* corner forces with the linear basis along the edge, (2 b_v + b_w)/3.   */
/* ---------------------------------------------------------------------- */
static void o1_rzaw_nodes_faces(const o_mesh *m, const o_cfg *c, double *ustar, const double *unkno,
                                double *rhsel, const double *geoel, const double *coord, const double *aflim,
                                const double *afvec, const double *gelq) {
  const int nquad = m->nquad, npoin = m->npoin;
  const double g = c->gamlg, eps8 = 1.0e-08, slpdu = (g + 1.0) / 2.0;
#define QN(ie, k) (m->ipqua[4 * (ie) + (k)] - 1)
#define GL(f, ie) (gelq + 3 * ((f) + 4 * (ie)))
#define AF(k, ie) aflim[(k) + 5 * (ie)]
#define AV(i, j, ie) afvec[(i) + 2 * (j) + 4 * (ie)]
  int *indnd = (int *)calloc((size_t)npoin, sizeof(int));
  double *vlave = (double *)malloc(sizeof(double) * 2 * (size_t)npoin);
  double *munacn = (double *)calloc((size_t)4 * npoin, sizeof(double));
  double *munacu = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *snsigm = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *mcl = (double *)malloc(sizeof(double) * 4 * 8 * (size_t)nquad);  /* munaclq(2,2,2,4) */
  double *mul = (double *)malloc(sizeof(double) * 2 * 8 * (size_t)nquad);  /* munaulq(2,2,4) */
  double *snl = (double *)malloc(sizeof(double) * 2 * 8 * (size_t)nquad);  /* snsigmlq(2,2,4) */
  double *fst = (double *)malloc(sizeof(double) * 2 * 8 * (size_t)nquad);  /* fsqrzaw(2,2,4) */
  double *fpres = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *bsnv = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *bsnpf = (double *)calloc((size_t)2 * npoin, sizeof(double));

  for (int ifa = 0; ifa < m->nbfac; ifa++) {
    if (c->ncase == 2) for (int k = 0; k < 2; k++) indnd[m->bface[5 * ifa + k] - 1] = 1;
  }
  for (int ifa = 0; ifa < m->nbfac; ifa++)
    if (m->bface[5 * ifa + 2] == 25) for (int k = 0; k < 2; k++) indnd[m->bface[5 * ifa + k] - 1] = 1;
  /* getvlavenew's average is overwritten by the previous nodal velocity (`vlave = ustar`) */
  memcpy(vlave, ustar, sizeof(double) * 2 * (size_t)npoin);

  /* getriem_quadrzaw, scattering in cell order */
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double bq[4][3];
    for (int iv = 0; iv < 4; iv++) { bq[iv][0] = 1.0; bq[iv][1] = (XVQ[iv] - rc) / 1.0; bq[iv][2] = (YVQ[iv] - sc) / 1.0; }
    /* face 1 of vertex iv: the edge to the previous vertex; face 2: to the next */
    double vn[4][2][3];
    for (int iv = 0; iv < 4; iv++) {
      const int fa = (iv + 3) % 4, fb = iv;
      for (int k = 0; k < 3; k++) { vn[iv][0][k] = GL(fa, ie)[k]; vn[iv][1][k] = GL(fb, ie)[k]; }
      vn[iv][0][2] = 0.5 * vn[iv][0][2];
      vn[iv][1][2] = 0.5 * vn[iv][1][2];
    }
    double rhomc = U_(unkno, c, 0, 0, ielem);
    double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
    double rhoct = 1.0 / rhomc;
    double pctr = fmax(eps8, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
    double unknvq[4][5], sig[4], aujmp[4][3];
    p1_vertex(c, unkno, ielem, rc, sc, unknvq);
    const double a11 = AV(0, 0, ie), a12 = AV(0, 1, ie), a21 = AV(1, 0, ie), a22 = AV(1, 1, ie);
    for (int iv = 0; iv < 4; iv++) {
      double rhovt = 1.0 / unknvq[iv][0];
      double uv = unknvq[iv][1], vv = unknvq[iv][2], ev = unknvq[iv][3];
      double pvtx = fmax(eps8, (g - 1.0) * rhovt * (ev - 0.5 * (uv * uv + vv * vv)));
      double dudr = a11 * U_(unkno, c, 1, 1, ielem) + a12 * U_(unkno, c, 1, 2, ielem);
      double duds = a11 * U_(unkno, c, 2, 1, ielem) + a12 * U_(unkno, c, 2, 2, ielem);
      double dvdr = a21 * U_(unkno, c, 1, 1, ielem) + a22 * U_(unkno, c, 1, 2, ielem);
      double dvds = a21 * U_(unkno, c, 2, 1, ielem) + a22 * U_(unkno, c, 2, 2, ielem);
      uv = U_(unkno, c, 0, 1, ielem) + dudr * bq[iv][1] + duds * bq[iv][2];
      vv = U_(unkno, c, 0, 2, ielem) + dvdr * bq[iv][1] + dvds * bq[iv][2];
      pvtx = pctr + AF(3, ie) * (pvtx - pctr);
      unknvq[iv][1] = uv;
      unknvq[iv][2] = vv;
      sig[iv] = -pvtx;
      int ip = QN(ie, iv);
      double acnx = X_(vlave, 0, ip) - uv, acny = X_(vlave, 1, ip) - vv;
      double nrm = sqrt(acnx * acnx + acny * acny);
      if (nrm < TINY_S) { aujmp[iv][0] = TINY_S; aujmp[iv][1] = TINY_S; }
      else { aujmp[iv][0] = acnx / nrm; aujmp[iv][1] = acny / nrm; }
      aujmp[iv][2] = nrm;
    }
    double sdctr = sqrt(fmax(eps8, g * pctr / rhoct));
    for (int iv = 0; iv < 4; iv++) aujmp[iv][2] = aujmp[iv][2] / sdctr;
    double murie[4][2];
    for (int iv = 0; iv < 4; iv++) {
      int ip = QN(ie, iv);
      double dux = X_(vlave, 0, ip) - unknvq[iv][1], duy = X_(vlave, 1, ip) - unknvq[iv][2];
      for (int f = 0; f < 2; f++) {
        /* the shock term is switched off: deltu = 0 * |du.n| */
        double deltu = 0.0 * fabs(dux * vn[iv][f][0] + duy * vn[iv][f][1]);
        murie[iv][f] = rhoct * sdctr + rhoct * slpdu * deltu;
      }
    }
    for (int iv = 0; iv < 4; iv++) {
      int ip = QN(ie, iv);
      for (int f = 0; f < 2; f++) {
        /* getriecoef_matrixnew, Limiterlag.f90:1037-1076 */
        double area = vn[iv][f][2], n1 = vn[iv][f][0], n2 = vn[iv][f][1];
        double vnau = (aujmp[iv][2] < 1.0e12) ? 1.0 : n1 * aujmp[iv][0] + n2 * aujmp[iv][1];
        double mc11 = murie[iv][f] * area * fabs(vnau), mc21 = 0.0, mc12 = 0.0, mc22 = murie[iv][f] * area * fabs(vnau);
        double mu1 = mc11 * unknvq[iv][1] + mc21 * unknvq[iv][2];
        double mu2 = mc21 * unknvq[iv][1] + mc22 * unknvq[iv][2];
        double s1 = sig[iv] * area * n1 + 0.0 * area * n2;
        double s2 = 0.0 * area * n1 + sig[iv] * area * n2;
        munacn[0 + 4 * ip] = munacn[0 + 4 * ip] + mc11;
        munacn[1 + 4 * ip] = munacn[1 + 4 * ip] + mc21;
        munacn[2 + 4 * ip] = munacn[2 + 4 * ip] + mc12;
        munacn[3 + 4 * ip] = munacn[3 + 4 * ip] + mc22;
        munacu[0 + 2 * ip] = munacu[0 + 2 * ip] + mu1;
        munacu[1 + 2 * ip] = munacu[1 + 2 * ip] + mu2;
        snsigm[0 + 2 * ip] = snsigm[0 + 2 * ip] + s1;
        snsigm[1 + 2 * ip] = snsigm[1 + 2 * ip] + s2;
        const size_t o = (size_t)f + 2 * (iv + 4 * (size_t)ie);
        mcl[4 * o + 0] = mc11; mcl[4 * o + 1] = mc21; mcl[4 * o + 2] = mc12; mcl[4 * o + 3] = mc22;
        mul[2 * o + 0] = mu1; mul[2 * o + 1] = mu2;
        snl[2 * o + 0] = s1; snl[2 * o + 1] = s2;
      }
    }
  }
  /* getbc_lagmaire_rzaw (GetBClag.f90:57-250): the boundary area vectors of
   * the velocity walls (code 22, half the face at each end, no radius
   * weight) and the pressure forces of code 21 (ncase 3: p = 1e-6); then
   * at the wall nodes the force fpres that removes the wall-normal
   * velocity from the node solve. */
  for (int ifa = 0; ifa < m->nbfac; ifa++) {
    const int *bf = m->bface + 5 * ifa;
    const int ipf[2] = {bf[0] - 1, bf[1] - 1};
    double anx = X_(coord, 1, ipf[1]) - X_(coord, 1, ipf[0]);
    double any = -(X_(coord, 0, ipf[1]) - X_(coord, 0, ipf[0]));
    const double gf1 = anx / sqrt(anx * anx + any * any), gf2 = any / sqrt(anx * anx + any * any);
    const double gf3 = sqrt(anx * anx + any * any);
    double bsnx = 0.0, bsny = 0.0;
    if (bf[2] == 22) {
      if (bf[3] == 221) {
        bsnx = 0.0 * gf3 * 0.5;
        bsny = -1.0 * gf3 * 0.5;
        if (c->ncase == 1 || c->ncase == 2 || c->ncase == 12) {
          if (X_(coord, 1, ipf[0]) < 1.0e-6 && X_(coord, 1, ipf[1]) < 1.0e-6) {
            bsnx = 0.0 * gf3 * 0.5; bsny = -1.0 * gf3 * 0.5;
          } else if (fabs(X_(coord, 1, ipf[0]) - 1.0) < 1.0e-6 && fabs(X_(coord, 1, ipf[1]) - 1.0) < 1.0e-6) {
            bsnx = 0.0 * gf3 * 0.5; bsny = 1.0 * gf3 * 0.5;
          }
        }
      } else if (bf[3] == 222) {
        bsnx = -1.0 * gf3 * 0.5;
        bsny = 0.0 * gf3 * 0.5;
        if (c->ncase == 1) {
          if (X_(coord, 0, ipf[0]) < 1.0e-6 && X_(coord, 0, ipf[1]) < 1.0e-6) {
            bsnx = -1.0 * gf3 * 0.5; bsny = 0.0 * gf3 * 0.5;
          } else if (fabs(X_(coord, 0, ipf[0]) - 1.0) < 1.0e-6 && fabs(X_(coord, 0, ipf[1]) - 1.0) < 1.0e-6) {
            bsnx = 1.0 * gf3 * 0.5; bsny = 0.0 * gf3 * 0.5;
          }
        }
      }
      for (int k = 0; k < 2; k++) {
        bsnv[0 + 2 * ipf[k]] = bsnv[0 + 2 * ipf[k]] + bsnx;
        bsnv[1 + 2 * ipf[k]] = bsnv[1 + 2 * ipf[k]] + bsny;
      }
    } else if (bf[2] == 21) {
      bsnx = gf1 * gf3 * 0.5;
      bsny = gf2 * gf3 * 0.5;
      if (c->ncase == 3) {
        const double pres0 = 1.0e-6;
        for (int k = 0; k < 2; k++) {
          bsnpf[0 + 2 * ipf[k]] = bsnpf[0 + 2 * ipf[k]] + pres0 * bsnx;
          bsnpf[1 + 2 * ipf[k]] = bsnpf[1 + 2 * ipf[k]] + pres0 * bsny;
        }
      }
    }
  }
  for (int ifa = 0; ifa < m->nbfac; ifa++) {
    const int *bf = m->bface + 5 * ifa;
    if (bf[2] != 22) continue;
    for (int k = 0; k < 2; k++) {
      const int ip = bf[k] - 1;
      const double *mn = munacn + 4 * ip;  /* (1,1), (2,1), (1,2), (2,2) */
      double detma = mn[0] * mn[3] - mn[1] * mn[2];
      double i11 = mn[3] / detma, i12 = -mn[2] / detma, i21 = -mn[1] / detma, i22 = mn[0] / detma;
      double lnx = bsnv[0 + 2 * ip], lny = bsnv[1 + 2 * ip];
      double coefl = (i11 * lnx + i12 * lny) * lnx + (i21 * lnx + i22 * lny) * lny;
      double rhsx = munacu[0 + 2 * ip] - snsigm[0 + 2 * ip] - bsnpf[0 + 2 * ip];
      double rhsy = munacu[1 + 2 * ip] - snsigm[1 + 2 * ip] - bsnpf[1 + 2 * ip];
      double coefr = (i11 * rhsx + i12 * rhsy) * lnx + (i21 * rhsx + i22 * rhsy) * lny;
      fpres[0 + 2 * ip] = coefr / fmax(1.0e-16, coefl) * lnx;
      fpres[1 + 2 * ip] = coefr / fmax(1.0e-16, coefl) * lny;
    }
  }
  for (int ip = 0; ip < npoin; ip++) {
    fpres[0 + 2 * ip] = fpres[0 + 2 * ip] + bsnpf[0 + 2 * ip];
    fpres[1 + 2 * ip] = fpres[1 + 2 * ip] + bsnpf[1 + 2 * ip];
  }
  /* the node solve with the boundary forces */
  for (int ip = 0; ip < npoin; ip++) {
    if (indnd[ip]) continue;
    const double *mn = munacn + 4 * ip;
    double detma = mn[0] * mn[3] - mn[1] * mn[2];
    double i11 = mn[3] / detma, i12 = -mn[2] / detma, i21 = -mn[1] / detma, i22 = mn[0] / detma;
    double r1 = munacu[2 * ip] - snsigm[2 * ip] - fpres[2 * ip];
    double r2 = munacu[2 * ip + 1] - snsigm[2 * ip + 1] - fpres[2 * ip + 1];
    X_(ustar, 0, ip) = i11 * r1 + i12 * r2;
    X_(ustar, 1, ip) = i21 * r1 + i22 * r2;
  }
  /* the walls: 221 holds v, 222 holds u, code 25 both */
  for (int ifa = 0; ifa < m->nbfac; ifa++) {
    const int *bf = m->bface + 5 * ifa;
    for (int k = 0; k < 2; k++) {
      int ip = bf[k] - 1;
      if (bf[2] == 22) {
        if (bf[3] == 221) X_(ustar, 1, ip) = 0.0;
        else if (bf[3] == 222) X_(ustar, 0, ip) = 0.0;
      } else if (bf[2] == 25) {
        X_(ustar, 1, ip) = 0.0;
        X_(ustar, 0, ip) = 0.0;
      }
    }
  }
  /* corner forces fsqrzaw */
  for (int ie = 0; ie < nquad; ie++)
    for (int iv = 0; iv < 4; iv++) {
      int ip = QN(ie, iv);
      for (int f = 0; f < 2; f++) {
        const size_t o = (size_t)f + 2 * (iv + 4 * (size_t)ie);
        fst[2 * o + 0] = snl[2 * o + 0] + mcl[4 * o + 0] * X_(ustar, 0, ip) + mcl[4 * o + 1] * X_(ustar, 1, ip) - mul[2 * o + 0];
        fst[2 * o + 1] = snl[2 * o + 1] + mcl[4 * o + 2] * X_(ustar, 0, ip) + mcl[4 * o + 3] * X_(ustar, 1, ip) - mul[2 * o + 1];
      }
    }
  /* rhsifacedg_lagmc_quadrzaw: face 1 of vertex iv is the edge to the
   * previous vertex, face 2 to the next; each weighs (2 b_iv + b_w) */
  const double c16 = 0.1666666666666666, c13 = 0.3333333333333333;
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double bq[4][3];
    for (int iv = 0; iv < 4; iv++) { bq[iv][0] = 1.0; bq[iv][1] = (XVQ[iv] - rc) / 1.0; bq[iv][2] = (YVQ[iv] - sc) / 1.0; }
    double ul[3] = {0, 0, 0}, p1[3] = {0, 0, 0}, p2[3] = {0, 0, 0}, el[3] = {0, 0, 0};
    for (int iv = 0; iv < 4; iv++) {
      const int vp = (iv + 3) % 4, vx = (iv + 1) % 4;
      const double *ga = GL(vp, ie), *gb = GL(iv, ie);
      int ip = QN(ie, iv);
      double us = X_(ustar, 0, ip), vs = X_(ustar, 1, ip);
      const size_t o0 = 2 * (iv + 4 * (size_t)ie), o1 = o0 + 1;
      for (int k = 0; k < c->ndegr; k++) {
        const double wa = 2.0 * bq[iv][k] + bq[vp][k], wb = 2.0 * bq[iv][k] + bq[vx][k];
        const double l1x = c16 * wa * ga[0] * ga[2], l1y = c16 * wa * ga[1] * ga[2];
        const double l2x = c16 * wb * gb[0] * gb[2], l2y = c16 * wb * gb[1] * gb[2];
        ul[k] = ul[k] + us * l1x + vs * l1y + us * l2x + vs * l2y;
        p1[k] = p1[k] + fst[2 * o0] * c13 * wa + fst[2 * o1] * c13 * wb;
        p2[k] = p2[k] + fst[2 * o0 + 1] * c13 * wa + fst[2 * o1 + 1] * c13 * wb;
        el[k] = el[k] + us * fst[2 * o0] * c13 * wa + vs * fst[2 * o0 + 1] * c13 * wa +
                us * fst[2 * o1] * c13 * wb + vs * fst[2 * o1 + 1] * c13 * wb;
      }
    }
    for (int k = 0; k < c->ndegr; k++) {
      U_(rhsel, c, k, 0, ielem) = ul[k];
      U_(rhsel, c, k, 1, ielem) = p1[k];
      U_(rhsel, c, k, 2, ielem) = p2[k];
      U_(rhsel, c, k, 3, ielem) = el[k];
    }
  }
#undef QN
#undef GL
#undef AF
#undef AV
  free(indnd); free(vlave); free(munacn); free(munacu); free(snsigm); free(mcl); free(mul); free(snl);
  free(fst); free(fpres); free(bsnv); free(bsnpf);
}

/* One stage's right-hand side; with nrz = 2, `amatr` (4, ncell) and
 * `rev` = (itime > 1 or the stage > 1) select the per-stage mass centre and
 * mass matrix of getgeoel_lagmc_rzawrev / getamatr_lagmc_rzawrev, which
 * rewrite geoel(1:2) and amatr. */
static void o1_rhs_x(const o_mesh *m, const o_cfg *c, double *ustar, double *unkno,
                     double *rhsel, double *geoel, const double *coord, double *amatr, int rev,
                     double *aflim_out, double *afvec_out) {
  const int nquad = m->nquad, npoin = m->npoin;
  const double g = c->gamlg, epsd = 1.0e-6;
  const double slpdu = (g + 1.0) / 2.0;
  double *gelq = (double *)calloc((size_t)12 * nquad, sizeof(double));   /* (3,4,nquad) */
  double *unmax = (double *)malloc(sizeof(double) * 5 * (size_t)npoin);
  double *unmin = (double *)malloc(sizeof(double) * 5 * (size_t)npoin);
  double *aflim = (double *)calloc((size_t)5 * nquad, sizeof(double));  /* (nq+1, ncell) */
  double *afvec = (double *)calloc((size_t)4 * nquad, sizeof(double));  /* (2,2,ncell) col-major */
  double *mapmt = (double *)calloc((size_t)4 * nquad, sizeof(double));
  int *bnd = (int *)calloc((size_t)npoin, sizeof(int));
  int *indbd = (int *)calloc((size_t)npoin, sizeof(int));
  int *indnd = (int *)calloc((size_t)npoin, sizeof(int));
  double *munacn = (double *)calloc((size_t)4 * npoin, sizeof(double));
  double *munacu = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *snsigm = (double *)calloc((size_t)2 * npoin, sizeof(double));
  double *mcl = (double *)malloc(sizeof(double) * 4 * 8 * (size_t)nquad);  /* munaclq(2,2,2,4) */
  double *mul = (double *)malloc(sizeof(double) * 2 * 8 * (size_t)nquad);  /* munaulq(2,2,4) */
  double *snl = (double *)malloc(sizeof(double) * 2 * 8 * (size_t)nquad);  /* snsigmlq(2,2,4) */
  double *fst = (double *)malloc(sizeof(double) * 2 * 8 * (size_t)nquad);  /* fstarq(2,2,4) */
  double *vlave = (double *)malloc(sizeof(double) * 2 * (size_t)npoin);
#define QN(ie, k) (m->ipqua[4 * (ie) + (k)] - 1)
#define GL(f, ie) (gelq + 3 * ((f) + 4 * (ie)))
#define AF(k, ie) aflim[(k) + 5 * (ie)]
#define AV(i, j, ie) afvec[(i) + 2 * (j) + 4 * (ie)]
#define MP(i, j, ie) mapmt[(i) + 2 * (j) + 4 * (ie)]

  /* I.1.1 getfnds_lag_mc_hybrid, Getrhslagmc.f90:2117-2265 (quad faces) */
  for (int ie = 0; ie < nquad; ie++) {
    for (int f = 0; f < 4; f++) {
      int a = QN(ie, f), b = QN(ie, (f + 1) % 4);
      double anx = X_(coord, 1, b) - X_(coord, 1, a);
      double any = -(X_(coord, 0, b) - X_(coord, 0, a));
      GL(f, ie)[0] = anx / sqrt(anx * anx + any * any);
      GL(f, ie)[1] = any / sqrt(anx * anx + any * any);
      GL(f, ie)[2] = sqrt(anx * anx + any * any);
    }
  }

  /* I.1.2a barthlimit_lag_vtxunknew, Getrhslagmctria.f90:2373-2643:
   * node bounds of (tau, u, v, p, e) over the cells sharing the node */
  for (int ip = 0; ip < npoin; ip++)
    for (int q = 0; q < 5; q++) { unmax[q + 5 * ip] = -1.0e10; unmin[q + 5 * ip] = 1.0e10; }
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double rhom = U_(unkno, c, 0, 0, ielem);
    double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
    double rhoct = 1.0 / rhom;
    double pctr = fmax(EPS_S, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
    double unctr[5] = {U_(unkno, c, 0, 0, ielem), uctr, vctr, pctr, ectr};
    for (int iv = 0; iv < 4; iv++) {
      int ip = QN(ie, iv);
      for (int q = 0; q < 5; q++) {
        if (unctr[q] > unmax[q + 5 * ip]) unmax[q + 5 * ip] = unctr[q];
        if (unctr[q] < unmin[q + 5 * ip]) unmin[q + 5 * ip] = unctr[q];
      }
    }
  }

  /* I.1.2b barthlimit_lagsym_quad, Limiterlag.f90:4-404 */
  for (int ifa = 0; ifa < m->nbfac; ifa++)
    for (int k = 0; k < 2; k++) bnd[m->bface[5 * ifa + k] - 1] = 1;
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double unknvq[4][5];
    p1_vertex(c, unkno, ielem, rc, sc, unknvq);
    for (int iv = 0; iv < 4; iv++) {
      double rhov = 1.0 / unknvq[iv][0];
      double uv = unknvq[iv][1], vv = unknvq[iv][2], ev = unknvq[iv][3];
      double pvtx = fmax(EPS_S, (g - 1.0) * rhov * (ev - 0.5 * (uv * uv + vv * vv)));
      unknvq[iv][0] = 1.0 / rhov;
      unknvq[iv][3] = pvtx;
    }
    double rhom = U_(unkno, c, 0, 0, ielem);
    double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
    double rhoct = 1.0 / rhom;
    double pctr = fmax(EPS_S, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
    double unctr[4] = {1.0 / rhoct, uctr, vctr, pctr};
    double alfa[4][4];
    for (int iv = 0; iv < 4; iv++) {
      int ip = QN(ie, iv);
      double dunk[4];
      for (int q = 0; q < 4; q++) {
        dunk[q] = unknvq[iv][q] - unctr[q];
        alfa[iv][q] = barthfct(unmax[q + 5 * ip], unmin[q + 5 * ip], unctr[q], dunk[q]);
      }
      if (bnd[ip] && c->ncase == 1) {
        if (X_(coord, 0, ip) < 1.0e-6 || fabs(X_(coord, 0, ip) - 1.0) < 1.0e-6)
          alfa[iv][1] = fmin(fmax((-unctr[1]) / (dunk[1]), 0.0), 1.0);
        if (X_(coord, 1, ip) < 1.0e-6 || fabs(X_(coord, 1, ip) - 1.0) < 1.0e-6)
          alfa[iv][2] = fmin(fmax((-unctr[2]) / (dunk[2]), 0.0), 1.0);
      }
    }
    for (int q = 0; q < 4; q++) {
      double a = alfa[0][q];
      for (int iv = 1; iv < 4; iv++) if (alfa[iv][q] < a) a = alfa[iv][q];
      AF(q, ie) = a;
    }
  }

  /* barthlimit_sympre_quadlb, Limiterlag.f90:8127-8692: the velocity
   * limited in the principal frame of the strain rate, as a 2x2 tensor */
  if (c->ncase != 1) {
    for (int ifa = 0; ifa < m->nbfac; ifa++)
      if (m->bface[5 * ifa + 2] == 22 && m->bface[5 * ifa + 3] == 221)
        for (int k = 0; k < 2; k++) indbd[m->bface[5 * ifa + k] - 1] = 3;
    for (int ifa = 0; ifa < m->nbfac; ifa++)
      if (m->bface[5 * ifa + 2] == 22 && m->bface[5 * ifa + 3] == 222)
        for (int k = 0; k < 2; k++) {
          int ip = m->bface[5 * ifa + k] - 1;
          indbd[ip] = (indbd[ip] == 3) ? 10 : 2;
        }
  } else {
    for (int ifa = 0; ifa < m->nbfac; ifa++)
      for (int k = 0; k < 2; k++) indbd[m->bface[5 * ifa + k] - 1] = 1;
  }
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double xpq[4][2];
    for (int k = 0; k < 4; k++) { xpq[k][0] = X_(coord, 0, QN(ie, k)); xpq[k][1] = X_(coord, 1, QN(ie, k)); }
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double dudr = U_(unkno, c, 1, 1, ielem) / 1.0, duds = U_(unkno, c, 2, 1, ielem) / 1.0;
    double dvdr = U_(unkno, c, 1, 2, ielem) / 1.0, dvds = U_(unkno, c, 2, 2, ielem) / 1.0;
    double dxdr, dxds, dydr, dyds;
    jac4((const double(*)[2])xpq, rc, sc, &dxdr, &dxds, &dydr, &dyds);
    double jacom = dxdr * dyds - dydr * dxds;
    double drdx = dyds / jacom, drdy = -dxds / jacom, dsdx = -dydr / jacom, dsdy = dxdr / jacom;
    double dudx = dudr * drdx + duds * dsdx, dudy = dudr * drdy + duds * dsdy;
    double dvdx = dvdr * drdx + dvds * dsdx, dvdy = dvdr * drdy + dvds * dsdy;
    /* the velocity-aligned frame set first (:8290-8301) is always overwritten below */
    double matra = dudx, matrb = 0.5 * (dudy + dvdx), matrc = matrb, matrd = dvdy;
    double mapt = matra + matrd, mapd = matra * matrd - matrb * matrc;
    double lamda1 = 0.5 * mapt + sqrt(0.25 * (mapt * mapt) - mapd);
    double lamda2 = 0.5 * mapt - sqrt(0.25 * (mapt * mapt) - mapd);
    if (fabs(matrc) > 1.0e-8) {
      double lmat1 = sqrt((lamda1 - matrd) * (lamda1 - matrd) + matrc * matrc);
      double lmat2 = sqrt((lamda2 - matrd) * (lamda2 - matrd) + matrc * matrc);
      int r1 = (matrc > 0.0) ? 0 : 1, r2 = 1 - r1;
      MP(r1, 0, ie) = (lamda1 - matrd) / lmat1;
      MP(r1, 1, ie) = matrc / lmat1;
      MP(r2, 0, ie) = (lamda2 - matrd) / lmat2;
      MP(r2, 1, ie) = matrc / lmat2;
    } else {
      MP(0, 0, ie) = 0.0; MP(0, 1, ie) = 0.0; MP(1, 0, ie) = 0.0; MP(1, 1, ie) = 0.0;
    }
  }
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    const double m11 = MP(0, 0, ie), m12 = MP(0, 1, ie), m21 = MP(1, 0, ie), m22 = MP(1, 1, ie);
    double unknvq[4][5];
    p1_vertex(c, unkno, ielem, rc, sc, unknvq);
    for (int iv = 0; iv < 4; iv++) {
      double uv = unknvq[iv][1], vv = unknvq[iv][2];
      unknvq[iv][1] = uv * m11 + vv * m12;
      unknvq[iv][2] = uv * m21 + vv * m22;
    }
    double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem);
    double unctr[3] = {0.0, uctr * m11 + vctr * m12, uctr * m21 + vctr * m22};
    double alfa[4][3];
    for (int iv = 0; iv < 4; iv++) {
      int ip = QN(ie, iv);
      double mx[3] = {0, unctr[1], unctr[2]}, mn[3] = {0, unctr[1], unctr[2]};
      for (int is = m->esuv2[ip]; is < m->esuv2[ip + 1]; is++) {
        int je = m->esuv1[is] - 1;
        double uj = U_(unkno, c, 0, 1, je), vj = U_(unkno, c, 0, 2, je);
        /* the cell's own average, then the images across the walls */
        double img[4][2];
        int nimg = 0;
        img[nimg][0] = uj; img[nimg][1] = vj; nimg++;
        if (c->ncase != 1) {
          if (indbd[ip] == 3) { img[nimg][0] = uj; img[nimg][1] = -vj; nimg++; }
          else if (indbd[ip] == 2) { img[nimg][0] = -uj; img[nimg][1] = vj; nimg++; }
          else if (indbd[ip] == 10) {
            img[nimg][0] = uj; img[nimg][1] = -vj; nimg++;
            img[nimg][0] = -uj; img[nimg][1] = vj; nimg++;
            img[nimg][0] = -uj; img[nimg][1] = -vj; nimg++;
          }
        }
        for (int k = 0; k < nimg; k++) {
          double ul = img[k][0] * m11 + img[k][1] * m12;
          double vl = img[k][0] * m21 + img[k][1] * m22;
          mx[1] = fmax(mx[1], ul); mx[2] = fmax(mx[2], vl);
          mn[1] = fmin(mn[1], ul); mn[2] = fmin(mn[2], vl);
        }
      }
      for (int q = 1; q < 3; q++) {
        double dunk = unknvq[iv][q] - unctr[q];
        alfa[iv][q] = barthfct(mx[q], mn[q], unctr[q], dunk);
      }
      if (indbd[ip] == 1 && c->ncase == 1) {
        if (X_(coord, 0, ip) < 1.0e-6 || fabs(X_(coord, 0, ip) - 1.0) < 1.0e-6) { alfa[iv][1] = 1.0; alfa[iv][2] = 1.0; }
        if (X_(coord, 1, ip) < 1.0e-6 || fabs(X_(coord, 1, ip) - 1.0) < 1.0e-6) { alfa[iv][1] = 1.0; alfa[iv][2] = 1.0; }
      }
    }
    double fl[3];
    for (int q = 1; q < 3; q++) {
      double a = alfa[0][q];
      for (int iv = 1; iv < 4; iv++) if (alfa[iv][q] < a) a = alfa[iv][q];
      fl[q] = a;
    }
    /* afvec = R^T diag(fixi, fiet) R, R = mapmt (:8679-8691) */
    double fixi = fl[1], fiet = fl[2];
    double fi11 = (m11 * m11) * fixi + (m21 * m21) * fiet;
    double fi12 = m11 * m12 * fixi + m21 * m22 * fiet;
    double fi22 = (m12 * m12) * fixi + (m22 * m22) * fiet;
    AV(0, 0, ie) = fi11; AV(0, 1, ie) = fi12; AV(1, 0, ie) = fi12; AV(1, 1, ie) = fi22;
  }
  /* energy limiter on the reconstructed vertex energy (Limiterlag.f90:290-380) */
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    double rhom = U_(unkno, c, 0, 0, ielem);
    double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
    double rhoct = 1.0 / rhom;
    double pctr = fmax(EPS_S, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
    double unknvq[4][5];
    p1_vertex(c, unkno, ielem, rc, sc, unknvq);
    double alfa5[4];
    for (int iv = 0; iv < 4; iv++) {
      double rhov = 1.0 / unknvq[iv][0];
      double uv = unknvq[iv][1], vv = unknvq[iv][2], ev = unknvq[iv][3];
      double pvtx = fmax(EPS_S, (g - 1.0) * rhov * (ev - 0.5 * (uv * uv + vv * vv)));
      double t = rhom + AF(0, ie) * (1.0 / rhov - rhom);
      double pv = pctr + AF(3, ie) * (pvtx - pctr);
      double e5 = pv / (g - 1.0) * t + 0.5 * (uv * uv + vv * vv);
      int ip = QN(ie, iv);
      double dunk = e5 - ectr;
      alfa5[iv] = barthfct(unmax[4 + 5 * ip], unmin[4 + 5 * ip], ectr, dunk);
    }
    double a = alfa5[0];
    for (int iv = 1; iv < 4; iv++) if (alfa5[iv] < a) a = alfa5[iv];
    AF(4, ie) = a;
  }

  if (c->nrz == 2 && rev && amatr) o1_rzaw_rev(m, c, unkno, geoel, amatr, coord, aflim);
  if (c->nrz == 1) {
    /* RZ: getndvelo_lagmc_rz and rhsifacedg_lagmc_quadrz (Getrhslagmc.f90:6884-6887, :6911-6917) */
    o1_rz_nodes_faces(m, c, ustar, unkno, rhsel, geoel, coord, aflim, afvec, gelq);
  } else if (c->nrz == 2) {
    /* area-weighted RZ: getndvelo_lagmc_rzaw and rhsifacedg_lagmc_quadrzaw
     * (Getrhslagmc.f90:6888-6889, :6919-6922) */
    o1_rzaw_nodes_faces(m, c, ustar, unkno, rhsel, geoel, coord, aflim, afvec, gelq);
  } else {
    /* I.1.3 getndvelo_lag_mc_matrixsym, Limiterlag.f90:408-704 */
    for (int ifa = 0; ifa < m->nbfac; ifa++) {
      if (c->ncase == 2) for (int k = 0; k < 2; k++) indnd[m->bface[5 * ifa + k] - 1] = 1;
      if (m->bface[5 * ifa + 2] == 25) for (int k = 0; k < 2; k++) indnd[m->bface[5 * ifa + k] - 1] = 1;
    }
    memcpy(vlave, ustar, sizeof(double) * 2 * (size_t)npoin);
    /* getriem_quad_matrixsym, Limiterlag.f90:708-1033, scattering in cell order */
    for (int ie = 0; ie < nquad; ie++) {
      const int ielem = ie + m->ntria;
      double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
      double bq[4][3];
      for (int iv = 0; iv < 4; iv++) { bq[iv][0] = 1.0; bq[iv][1] = (XVQ[iv] - rc) / 1.0; bq[iv][2] = (YVQ[iv] - sc) / 1.0; }
      /* corner iv touches faces iv-1 and iv; the area weight (2 r_a + r_b)/3 * 0.5 * |f| with r = 1 */
      double vn[4][2][3];
      for (int iv = 0; iv < 4; iv++) {
        int fa = (iv + 3) % 4, fb = iv;
        for (int k = 0; k < 3; k++) { vn[iv][0][k] = GL(fa, ie)[k]; vn[iv][1][k] = GL(fb, ie)[k]; }
        vn[iv][0][2] = (2.0 * 1.0 + 1.0) / 3.0 * 0.5 * vn[iv][0][2];
        vn[iv][1][2] = (2.0 * 1.0 + 1.0) / 3.0 * 0.5 * vn[iv][1][2];
      }
      double rhomc = U_(unkno, c, 0, 0, ielem);
      double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
      double rhoct = 1.0 / rhomc;
      double pctr = fmax(epsd, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
      double unknvq[4][5], sig[4], aujmp[4][3];
      p1_vertex(c, unkno, ielem, rc, sc, unknvq);
      const double a11 = AV(0, 0, ie), a12 = AV(0, 1, ie), a21 = AV(1, 0, ie), a22 = AV(1, 1, ie);
      for (int iv = 0; iv < 4; iv++) {
        double rhovt = 1.0 / unknvq[iv][0];
        double uv = unknvq[iv][1], vv = unknvq[iv][2], ev = unknvq[iv][3];
        double pvtx = fmax(epsd, (g - 1.0) * rhovt * (ev - 0.5 * (uv * uv + vv * vv)));
        double rhomv = rhomc + AF(0, ie) * (unknvq[iv][0] - rhomc);
        rhovt = 1.0 / rhomv;
        (void)rhovt;
        double dudr = a11 * U_(unkno, c, 1, 1, ielem) + a12 * U_(unkno, c, 1, 2, ielem);
        double duds = a11 * U_(unkno, c, 2, 1, ielem) + a12 * U_(unkno, c, 2, 2, ielem);
        double dvdr = a21 * U_(unkno, c, 1, 1, ielem) + a22 * U_(unkno, c, 1, 2, ielem);
        double dvds = a21 * U_(unkno, c, 2, 1, ielem) + a22 * U_(unkno, c, 2, 2, ielem);
        uv = U_(unkno, c, 0, 1, ielem) + dudr * bq[iv][1] + duds * bq[iv][2];
        vv = U_(unkno, c, 0, 2, ielem) + dvdr * bq[iv][1] + dvds * bq[iv][2];
        pvtx = pctr + AF(3, ie) * (pvtx - pctr);
        unknvq[iv][1] = uv;
        unknvq[iv][2] = vv;
        sig[iv] = -pvtx + 0.0;
        int ip = QN(ie, iv);
        double acnx = X_(vlave, 0, ip) - uv, acny = X_(vlave, 1, ip) - vv;
        double nrm = sqrt(acnx * acnx + acny * acny);
        if (nrm < TINY_S) { aujmp[iv][0] = TINY_S; aujmp[iv][1] = TINY_S; }
        else { aujmp[iv][0] = acnx / nrm; aujmp[iv][1] = acny / nrm; }
        aujmp[iv][2] = nrm;
      }
      double sdctr = sqrt(fmax(epsd, g * pctr / rhoct));
      for (int iv = 0; iv < 4; iv++) aujmp[iv][2] = aujmp[iv][2] / sdctr;
      double murie[4][2];
      for (int iv = 0; iv < 4; iv++) {
        int ip = QN(ie, iv);
        double dux = X_(vlave, 0, ip) - unknvq[iv][1], duy = X_(vlave, 1, ip) - unknvq[iv][2];
        for (int f = 0; f < 2; f++) {
          double deltu = fabs(dux * vn[iv][f][0] + duy * vn[iv][f][1]);
          murie[iv][f] = rhoct * sdctr + c->cimpd * rhoct * slpdu * deltu;
        }
      }
      for (int iv = 0; iv < 4; iv++) {
        int ip = QN(ie, iv);
        for (int f = 0; f < 2; f++) {
          /* getriecoef_matrixnew, Limiterlag.f90:1037-1076 */
          double area = vn[iv][f][2], n1 = vn[iv][f][0], n2 = vn[iv][f][1];
          double vnau = (aujmp[iv][2] < 1.0e12) ? 1.0 : n1 * aujmp[iv][0] + n2 * aujmp[iv][1];
          double mc11 = murie[iv][f] * area * fabs(vnau), mc21 = 0.0, mc12 = 0.0, mc22 = murie[iv][f] * area * fabs(vnau);
          double mu1 = mc11 * unknvq[iv][1] + mc21 * unknvq[iv][2];
          double mu2 = mc21 * unknvq[iv][1] + mc22 * unknvq[iv][2];
          double s1 = sig[iv] * area * n1 + (0.0 + 0.0) * area * n2;
          double s2 = (0.0 + 0.0) * area * n1 + sig[iv] * area * n2;
          munacn[0 + 4 * ip] = munacn[0 + 4 * ip] + mc11;
          munacn[1 + 4 * ip] = munacn[1 + 4 * ip] + mc21;
          munacn[2 + 4 * ip] = munacn[2 + 4 * ip] + mc12;
          munacn[3 + 4 * ip] = munacn[3 + 4 * ip] + mc22;
          munacu[0 + 2 * ip] = munacu[0 + 2 * ip] + mu1;
          munacu[1 + 2 * ip] = munacu[1 + 2 * ip] + mu2;
          snsigm[0 + 2 * ip] = snsigm[0 + 2 * ip] + s1;
          snsigm[1 + 2 * ip] = snsigm[1 + 2 * ip] + s2;
          const size_t o = (size_t)f + 2 * (iv + 4 * (size_t)ie);
          mcl[4 * o + 0] = mc11; mcl[4 * o + 1] = mc21; mcl[4 * o + 2] = mc12; mcl[4 * o + 3] = mc22;
          mul[2 * o + 0] = mu1; mul[2 * o + 1] = mu2;
          snl[2 * o + 0] = s1; snl[2 * o + 1] = s2;
        }
      }
    }
    for (int ip = 0; ip < npoin; ip++) {
      if (indnd[ip]) continue;
      const double *mn = munacn + 4 * ip;  /* (1,1), (2,1), (1,2), (2,2) */
      double detma = mn[0] * mn[3] - mn[1] * mn[2];
      double i11 = mn[3] / detma, i12 = -mn[2] / detma, i21 = -mn[1] / detma, i22 = mn[0] / detma;
      double r1 = munacu[2 * ip] - snsigm[2 * ip], r2 = munacu[2 * ip + 1] - snsigm[2 * ip + 1];
      X_(ustar, 0, ip) = i11 * r1 + i12 * r2;
      X_(ustar, 1, ip) = i21 * r1 + i22 * r2;
    }
    for (int ifa = 0; ifa < m->nbfac; ifa++) {
      const int *bf = m->bface + 5 * ifa;
      for (int k = 0; k < 2; k++) {
        int ip = bf[k] - 1;
        if (bf[2] == 22) {
          if (bf[3] == 221) X_(ustar, 1, ip) = 0.0;
          else if (bf[3] == 222) X_(ustar, 0, ip) = 0.0;
        } else if (bf[2] == 25) {
          X_(ustar, 0, ip) = 0.0;
          X_(ustar, 1, ip) = 0.0;
        }
      }
    }
    for (int ie = 0; ie < nquad; ie++)
      for (int iv = 0; iv < 4; iv++) {
        int ip = QN(ie, iv);
        for (int f = 0; f < 2; f++) {
          const size_t o = (size_t)f + 2 * (iv + 4 * (size_t)ie);
          fst[2 * o + 0] = snl[2 * o + 0] + mcl[4 * o + 0] * X_(ustar, 0, ip) + mcl[4 * o + 1] * X_(ustar, 1, ip) - mul[2 * o + 0];
          fst[2 * o + 1] = snl[2 * o + 1] + mcl[4 * o + 2] * X_(ustar, 0, ip) + mcl[4 * o + 3] * X_(ustar, 1, ip) - mul[2 * o + 1];
        }
      }

    /* I.1.4 rhsifacedg_lag_mc_hybridquad2, Getrhslagmc.f90:14468-14618 */
    const double c16 = 0.1666666666666666, c13 = 0.3333333333333333;
    for (int ie = 0; ie < nquad; ie++) {
      const int ielem = ie + m->ntria;
      double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
      double bq[4][3];
      for (int iv = 0; iv < 4; iv++) { bq[iv][0] = 1.0; bq[iv][1] = (XVQ[iv] - rc) / 1.0; bq[iv][2] = (YVQ[iv] - sc) / 1.0; }
      double ul[3] = {0, 0, 0}, p1[3] = {0, 0, 0}, p2[3] = {0, 0, 0}, el[3] = {0, 0, 0};
      for (int iv = 0; iv < 4; iv++) {
        int ip = QN(ie, iv);
        int fa = (iv + 3) % 4, fb = iv;
        double us = X_(ustar, 0, ip), vs = X_(ustar, 1, ip);
        const size_t o0 = 2 * (iv + 4 * (size_t)ie), o1 = o0 + 1;
        for (int k = 0; k < c->ndegr; k++) {
          double b3 = 2.0 * bq[iv][k] + bq[iv][k];
          double l1x = c16 * b3 * GL(fa, ie)[0] * GL(fa, ie)[2], l1y = c16 * b3 * GL(fa, ie)[1] * GL(fa, ie)[2];
          double l2x = c16 * b3 * GL(fb, ie)[0] * GL(fb, ie)[2], l2y = c16 * b3 * GL(fb, ie)[1] * GL(fb, ie)[2];
          ul[k] = ul[k] + us * l1x + vs * l1y + us * l2x + vs * l2y;
          p1[k] = p1[k] + fst[2 * o0] * c13 * b3 + fst[2 * o1] * c13 * b3;
          p2[k] = p2[k] + fst[2 * o0 + 1] * c13 * b3 + fst[2 * o1 + 1] * c13 * b3;
          el[k] = el[k] + us * fst[2 * o0] * c13 * b3 + vs * fst[2 * o0 + 1] * c13 * b3 +
                  us * fst[2 * o1] * c13 * b3 + vs * fst[2 * o1 + 1] * c13 * b3;
        }
      }
      for (int k = 0; k < c->ndegr; k++) {
        U_(rhsel, c, k, 0, ielem) = ul[k];
        U_(rhsel, c, k, 1, ielem) = p1[k];
        U_(rhsel, c, k, 2, ielem) = p2[k];
        U_(rhsel, c, k, 3, ielem) = el[k];
      }
    }
  }

  /* I.1.5 rhsdomndg_lag_mc_quadsym, Limiterlag.f90:1108-1490 (5x5 Gauss) */
  double pos25[25][2], w25[25];
  quad_rule(25, 0, pos25, w25);
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    double xpq[4][2];
    for (int k = 0; k < 4; k++) { xpq[k][0] = X_(coord, 0, QN(ie, k)); xpq[k][1] = X_(coord, 1, QN(ie, k)); }
    double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    const double dbdr[3] = {0.0, 1.0 / 1.0, 0.0}, dbds[3] = {0.0, 0.0, 1.0 / 1.0};
    const double a11 = AV(0, 0, ie), a12 = AV(0, 1, ie), a21 = AV(1, 0, ie), a22 = AV(1, 1, ie);
    for (int ig = 0; ig < 25; ig++) {
      double r = pos25[ig][0], s = pos25[ig][1], wi = w25[ig];
      double dxdr, dxds, dydr, dyds;
      jac4((const double(*)[2])xpq, r, s, &dxdr, &dxds, &dydr, &dyds);
      double djaco = wi;
      /* rcoef = 1 - alfrz + alfrz*ygaus (Limiterlag.f90:1268-1279) */
      double rcoef = 1.0;
      if (c->nrz == 1) {
        const double rp = 1.0 + r, rm = 1.0 - r, sp = 1.0 + s, sm = 1.0 - s;
        const double shpq[4] = {0.25 * rm * sm, 0.25 * rp * sm, 0.25 * rp * sp, 0.25 * rm * sp};
        double ygaus = 0.0;
        for (int k = 0; k < 4; k++) ygaus = ygaus + shpq[k] * xpq[k][1];
        rcoef = 1.0 - 1.0 + 1.0 * ygaus;
      }
      double gd[2][3];
      for (int k = 0; k < 3; k++) {
        gd[0][k] = dyds * dbdr[k] + (-dydr) * dbds[k];
        gd[1][k] = (-dxds) * dbdr[k] + dxdr * dbds[k];
      }
      double b[3] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
      double un[4];
      for (int q = 0; q < 4; q++) {
        double a = 0.0;
        for (int k = 0; k < c->mdegr; k++) a = a + U_(unkno, c, k, q, ielem) * b[k];
        un[q] = a;
      }
      double rhoad = 1.0 / un[0];
      double uadv = un[1], vadv = un[2], eadv = un[3];
      double pres = (g - 1.0) * rhoad * (eadv - 0.5 * (uadv * uadv + vadv * vadv));
      double rhomc = U_(unkno, c, 0, 0, ielem);
      double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
      double rhoct = 1.0 / rhomc;
      double pctr = fmax(epsd, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
      double dudr = a11 * U_(unkno, c, 1, 1, ielem) + a12 * U_(unkno, c, 1, 2, ielem);
      double duds = a11 * U_(unkno, c, 2, 1, ielem) + a12 * U_(unkno, c, 2, 2, ielem);
      double dvdr = a21 * U_(unkno, c, 1, 1, ielem) + a22 * U_(unkno, c, 1, 2, ielem);
      double dvds = a21 * U_(unkno, c, 2, 1, ielem) + a22 * U_(unkno, c, 2, 2, ielem);
      uadv = U_(unkno, c, 0, 1, ielem) + dudr * b[1] + duds * b[2];
      vadv = U_(unkno, c, 0, 2, ielem) + dvdr * b[1] + dvds * b[2];
      pres = pctr + AF(3, ie) * (pres - pctr);
      if (c->nrz == 2) {
        /* rhsdomndg_lagmc_quadrzaw (Getrhslagrz.f90:2243-2555): the plane
         * fluxes written without the stress tensor, no radius weight */
        for (int k = 0; k < c->ndegr; k++) {
          double f1 = gd[0][k] * uadv + gd[1][k] * vadv;
          double f2 = gd[0][k] * (-pres);
          double f3 = gd[1][k] * (-pres);
          double f4 = (gd[0][k] * uadv + gd[1][k] * vadv) * (-pres);
          U_(rhsel, c, k, 0, ielem) = U_(rhsel, c, k, 0, ielem) - f1 * djaco;
          U_(rhsel, c, k, 1, ielem) = U_(rhsel, c, k, 1, ielem) - f2 * djaco;
          U_(rhsel, c, k, 2, ielem) = U_(rhsel, c, k, 2, ielem) - f3 * djaco;
          U_(rhsel, c, k, 3, ielem) = U_(rhsel, c, k, 3, ielem) - f4 * djaco;
        }
        continue;
      }
      double s11 = -pres + 0.0, s12 = 0.0 + 0.0, s21 = 0.0 + 0.0, s22 = -pres + 0.0;
      for (int k = 0; k < c->ndegr; k++) {
        double f1 = gd[0][k] * uadv + gd[1][k] * vadv;
        double f2 = gd[0][k] * s11 + gd[1][k] * s12;
        double f3 = gd[0][k] * s21 + gd[1][k] * s22;
        double f4 = gd[0][k] * (s11 * uadv + s12 * vadv) + gd[1][k] * (s21 * uadv + s22 * vadv);
        U_(rhsel, c, k, 0, ielem) = U_(rhsel, c, k, 0, ielem) - f1 * djaco * rcoef;
        U_(rhsel, c, k, 1, ielem) = U_(rhsel, c, k, 1, ielem) - f2 * djaco * rcoef;
        U_(rhsel, c, k, 2, ielem) = U_(rhsel, c, k, 2, ielem) - f3 * djaco * rcoef;
        U_(rhsel, c, k, 3, ielem) = U_(rhsel, c, k, 3, ielem) - f4 * djaco * rcoef;
      }
    }
  }

  /* I.1.6 rhsdomnsrcdg_lagmc_quadrz (Getrhslagmc.f90:15800-16048): the
   * RZ hoop-stress source of the radial (y) momentum, 5x5 Gauss, the
   * limited pressure of the point, no radius weight */
  if (c->nrz == 1) {
    for (int ie = 0; ie < nquad; ie++) {
      const int ielem = ie + m->ntria;
      double xpq[4][2];
      for (int k = 0; k < 4; k++) { xpq[k][0] = X_(coord, 0, QN(ie, k)); xpq[k][1] = X_(coord, 1, QN(ie, k)); }
      double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
      for (int ig = 0; ig < 25; ig++) {
        double r = pos25[ig][0], s = pos25[ig][1], wi = w25[ig];
        double dxdr, dxds, dydr, dyds;
        jac4((const double(*)[2])xpq, r, s, &dxdr, &dxds, &dydr, &dyds);
        double djaco = wi * (dxdr * dyds - dydr * dxds);
        double b[3] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
        double un[4];
        for (int q = 0; q < 4; q++) {
          double a = 0.0;
          for (int k = 0; k < c->mdegr; k++) a = a + U_(unkno, c, k, q, ielem) * b[k];
          un[q] = a;
        }
        double rhoad = 1.0 / un[0];
        double pres = (g - 1.0) * rhoad * (un[3] - 0.5 * (un[1] * un[1] + un[2] * un[2]));
        double rhomc = U_(unkno, c, 0, 0, ielem);
        double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
        double rhoct = 1.0 / rhomc;
        double pctr = fmax(epsd, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
        pres = pctr + AF(3, ie) * (pres - pctr);
        for (int k = 0; k < c->ndegr; k++) {
          double f3 = 1.0 * (-pres) * b[k];
          U_(rhsel, c, k, 2, ielem) = U_(rhsel, c, k, 2, ielem) - f3 * djaco;
        }
      }
    }
  }

  /* I.1.6 for nrz = 2 (Getrhslagmc.f90:6961-6973): the right-hand side
   * times the cell-averaged radius geoel(11), then the source terms of
   * rhsdomnsrcdg_lagmc_quadrzaw (Getrhslagrz.f90:2818-3096): 5x5 Gauss over
   * the area, v of the cell average times b into the specific volume and
   * -p v b (the limited pressure of the point) into the energy */
  if (c->nrz == 2) {
    for (int ie = 0; ie < nquad; ie++) {
      const int ielem = ie + m->ntria;
      const double rb = G_(geoel, 10, ielem);
      for (int q = 0; q < 4; q++)
        for (int k = 0; k < c->ndegr; k++) U_(rhsel, c, k, q, ielem) = rb * U_(rhsel, c, k, q, ielem);
    }
    for (int ie = 0; ie < nquad; ie++) {
      const int ielem = ie + m->ntria;
      double xpq[4][2];
      for (int k = 0; k < 4; k++) { xpq[k][0] = X_(coord, 0, QN(ie, k)); xpq[k][1] = X_(coord, 1, QN(ie, k)); }
      double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
      for (int ig = 0; ig < 25; ig++) {
        double r = pos25[ig][0], s = pos25[ig][1], wi = w25[ig];
        double dxdr, dxds, dydr, dyds;
        jac4((const double(*)[2])xpq, r, s, &dxdr, &dxds, &dydr, &dyds);
        double djaco = wi * (dxdr * dyds - dxds * dydr);
        double b[3] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
        double un[4];
        for (int q = 0; q < 4; q++) {
          double a = 0.0;
          for (int k = 0; k < c->mdegr; k++) a = a + U_(unkno, c, k, q, ielem) * b[k];
          un[q] = a;
        }
        double rhoad = 1.0 / un[0];
        double pres = (g - 1.0) * rhoad * (un[3] - 0.5 * (un[1] * un[1] + un[2] * un[2]));
        double rhomc = U_(unkno, c, 0, 0, ielem);
        double uctr = U_(unkno, c, 0, 1, ielem), vctr = U_(unkno, c, 0, 2, ielem), ectr = U_(unkno, c, 0, 3, ielem);
        double rhoct = 1.0 / rhomc;
        double pctr = fmax(epsd, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
        double vadv = vctr;
        pres = pctr + AF(3, ie) * (pres - pctr);
        for (int k = 0; k < c->ndegr; k++) {
          U_(rhsel, c, k, 0, ielem) = U_(rhsel, c, k, 0, ielem) + vadv * b[k] * djaco;
          U_(rhsel, c, k, 3, ielem) = U_(rhsel, c, k, 3, ielem) + vadv * (-pres) * b[k] * djaco;
        }
      }
    }
  }

  /* I.x.7 limited slopes into the stage state, Getrhslagmc.f90:7283-7298 */
  for (int ie = 0; ie < nquad; ie++) {
    const int ielem = ie + m->ntria;
    for (int k = 1; k < 3; k++) U_(unkno, c, k, 0, ielem) = U_(unkno, c, k, 0, ielem) * AF(0, ie);
    double u22 = U_(unkno, c, 1, 1, ielem), u32 = U_(unkno, c, 2, 1, ielem);
    double u23 = U_(unkno, c, 1, 2, ielem), u33 = U_(unkno, c, 2, 2, ielem);
    double dudr = AV(0, 0, ie) * u22 + AV(0, 1, ie) * u23;
    double duds = AV(0, 0, ie) * u32 + AV(0, 1, ie) * u33;
    double dvdr = AV(1, 0, ie) * u22 + AV(1, 1, ie) * u23;
    double dvds = AV(1, 0, ie) * u32 + AV(1, 1, ie) * u33;
    U_(unkno, c, 1, 1, ielem) = dudr; U_(unkno, c, 2, 1, ielem) = duds;
    U_(unkno, c, 1, 2, ielem) = dvdr; U_(unkno, c, 2, 2, ielem) = dvds;
    for (int k = 1; k < 3; k++) U_(unkno, c, k, 3, ielem) = U_(unkno, c, k, 3, ielem) * AF(4, ie);
  }
  if (aflim_out) memcpy(aflim_out, aflim, sizeof(double) * 5 * (size_t)nquad);
  if (afvec_out) memcpy(afvec_out, afvec, sizeof(double) * 4 * (size_t)nquad);
#undef QN
#undef GL
#undef AF
#undef AV
#undef MP
  free(gelq); free(unmax); free(unmin); free(aflim); free(afvec); free(mapmt); free(bnd); free(indbd);
  free(indnd); free(munacn); free(munacu); free(snsigm); free(mcl); free(mul); free(snl); free(fst);
  free(vlave);
}

void o1_rhs(const o_mesh *m, const o_cfg *c, double *ustar, double *unkno,
            double *rhsel, const double *geoel, const double *coord,
            double *aflim_out, double *afvec_out) {
  o1_rhs_x(m, c, ustar, unkno, rhsel, (double *)geoel, coord, NULL, 0, aflim_out, afvec_out);
}

/* ---------------------------------------------------------------------- */
/* geterror_lag_curvhybrid, Postprocess.f90:3587-4143 (quad loop          */
/* :3736-3944): L2 errors against the exact solution, 25-point Gauss on    */
/* the current coordinates, returned as sqrt(errlp(1:3)).  ncase 1         */
/* (Taylor-Green: rho, |u|, p) and 2 (shockless Noh: rho, e_int, p).       */
/* ---------------------------------------------------------------------- */
void o_error(const o_mesh *m, const o_cfg *c, const double *unkno, const double *geoel,
             const double *coord, double *errl2) {
  double pos25[25][2], w25[25];
  quad_rule(25, 0, pos25, w25);
  const double g = c->gamlg;
  double errlp[3] = {0.0, 0.0, 0.0};
  for (int ie = 0; ie < m->nquad; ie++) {
    const int ielem = ie + m->ntria;
    double xp[9][2], shp[9], dr[9], ds[9];
    load_quad(m, coord, ie, xp);
    const double rc = G_(geoel, 0, ielem), sc = G_(geoel, 1, ielem);
    for (int ig = 0; ig < 25; ig++) {
      double r = pos25[ig][0], s = pos25[ig][1], wi = w25[ig];
      double a, b, cc, d, xg, yg;
      shp9(r, s, shp, dr, ds);
      jac9((const double(*)[2])xp, dr, ds, &a, &b, &cc, &d);
      double djaco = wi * (a * d - cc * b);
      map9((const double(*)[2])xp, shp, &xg, &yg);
      double bq[6];
      bq[0] = 1.0;
      bq[1] = (r - rc) / 1.0;
      bq[2] = (s - sc) / 1.0;
      if (c->npoly == 2) {
        bq[3] = 0.5 * bq[1] * bq[1] - G_(geoel, 18, ielem);
        bq[4] = 0.5 * bq[2] * bq[2] - G_(geoel, 19, ielem);
        bq[5] = bq[1] * bq[2] - G_(geoel, 20, ielem);
      }
      double un[4] = {0.0, 0.0, 0.0, 0.0};
      for (int k = 0; k < c->mdegr; k++)
        for (int q = 0; q < 4; q++) un[q] = un[q] + U_(unkno, c, k, q, ielem) * bq[k];
      const double rho = 1.0 / un[0], uadv = un[1], vadv = un[2], eadv = un[3];
      const double pres = (g - 1.0) * rho * (eadv - 0.5 * (uadv * uadv + vadv * vadv));
      if (c->ncase == 1) {
        const double pexa = 0.25 * (cos(2.0 * PI_ * xg) + cos(2.0 * PI_ * yg)) + 1.0;
        const double uexa = sin(PI_ * xg) * cos(PI_ * yg);
        const double vexa = -cos(PI_ * xg) * sin(PI_ * yg);
        const double vemag = sqrt(uadv * uadv + vadv * vadv), veexa = sqrt(uexa * uexa + vexa * vexa);
        errlp[0] = errlp[0] + fabs(rho - 1.0) * fabs(rho - 1.0) * djaco;
        errlp[1] = errlp[1] + fabs(vemag - veexa) * fabs(vemag - veexa) * djaco;
        errlp[2] = errlp[2] + fabs(pres - pexa) * fabs(pres - pexa) * djaco;
      } else if (c->ncase == 2) {
        const double eiadv = eadv - 0.5 * (uadv * uadv + vadv * vadv);
        const double eiexa = pow(1.0 - 0.6, -2.0 * (g - 1.0));
        const double rhoexa = pow(1.0 - 0.6, -2.0);
        const double pexa = (g - 1.0) * rhoexa * eiadv;
        errlp[0] = errlp[0] + fabs(rho - rhoexa) * fabs(rho - rhoexa) * djaco;
        errlp[1] = errlp[1] + fabs(eiadv - eiexa) * fabs(eiadv - eiexa) * djaco;
        errlp[2] = errlp[2] + fabs(pres - pexa) * fabs(pres - pexa) * djaco;
      }
    }
  }
  for (int k = 0; k < 3; k++) errl2[k] = sqrt(errlp[k]);
}
