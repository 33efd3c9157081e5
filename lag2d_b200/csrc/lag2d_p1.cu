// The linear P1 time step of Lag2D on straight 4-node quads (sm_100a): the
// branch ncurv = 0, nriem = 1, nfint = 1, nlimi = 6, nrz = 0 of
// getrhsdg_lag_mcnew (srccurv-lag/Getrhslagmc.f90:6810-6980, slope
// application :7283-7298) inside getsolvdg_lag (Getrhslag.f90:1553-2035),
// the configuration of the reference's Sod shock tube.
//
// One RK stage is
//   bounds  (nodes)  Barth node bounds of (tau, u, v, p, e) over the cells
//                    around each node (barthlimit_lag_vtxunknew,
//                    Getrhslagmctria.f90:2373-2643)
//   cell    (quads)  the limiter (barthlimit_lagsym_quad, Limiterlag.f90:
//                    4-404, with barthlimit_sympre_quadlb :8127-8692 and
//                    barthfct, Getrhslagmc.f90:9171-9222) and the corner
//                    Riemann coefficients (getriem_quad_matrixsym,
//                    Limiterlag.f90:708-1033, getriecoef_matrixnew :1037)
//   node    (nodes)  fixed-order gather of the corner coefficients, the 2x2
//                    nodal solve and the wall conditions
//                    (getndvelo_lag_mc_matrixsym, Limiterlag.f90:408-704)
//   rhs     (quads)  corner forces, face integral (rhsifacedg_lag_mc_
//                    hybridquad2, Getrhslagmc.f90:14468-14618), volume
//                    integral (rhsdomndg_lag_mc_quadsym, Limiterlag.f90:
//                    1108-1490), then (stages after the first) the limited
//                    slopes and the M^-1 update fused in
//   dt, update (stage 1), nodes, geom (getcellvol_lag on the 9-node image of
//                    the straight quad, Limiterlag.f90:2038-2165)
//
// Calls of the reference branch that do not change its result are not
// made: getbc_lagmaire2 (Getrhslag.f90:11269) forms a boundary force that the
// nodal solve leaves unused, getAS_llnl (Limiterlag.f90:15476) ends by
// zeroing its stress, and the divergence limiter of
// barthlimit_sympre_quadlb writes only geoel(10), which this branch never
// reads.  With order_exact the kernels keep the reference's expression and
// summation order, so the build with --fmad=false reproduces the CPU
// restatement bit for bit; the optimised form (order_exact 0) sums the two
// faces of each corner before the node gather and the face integral, takes
// the volume of the straight quad in closed form and evaluates the limiter
// function with one division.
//
// Layout in HBM (0-based, structure of arrays):
//   U[(q*3 + k)*ncell + e]        P1 DOF k of field q (tau, u, v, e)
//   ipq[k*nquad + iq]             vertex k (0..3, counter-clockwise) of quad iq
//   cf[(v*8 + f + 2*iv)*nquad+iq] corner-face coefficient v (m, m u, m v,
//                                 sigma.n A x, y) of corner iv, face f
//                                 (optimised kernels: cf[(v*4 + iv)*nquad+iq],
//                                 the two faces of corner iv summed)
//   lim[k*ncell + e]              aflim(1), aflim(4), aflim(5), afvec(1,1),
//                                 afvec(1,2), afvec(2,1), afvec(2,2)
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "lag2d.h"
#include "lag2d_device.cuh"
#include "lag2d_p1.h"
#include "lag2d_shape9.cuh"

namespace lag2d {
void fill_rule(int n, bool lobatto, double (*pos)[2], double *w);
void launch_xy_in(int n, cudaStream_t st, const double *xy, double *x, double *y, double *x2, double *y2);
void launch_xy_out(int n, cudaStream_t st, double *xy, const double *x, const double *y);

namespace p1 {

constexpr int ND = 3;            // P1 Taylor basis
constexpr int NU1 = ND * NQ;     // 12 DOFs per cell

// Literals the Fortran writes in single precision (`eps = 1.e-6`,
// `1.e-11`), widened to double as gfortran does.
#define EPS_S ((double)1.0e-6f)
#define TINY_S ((double)1.0e-11f)

// node flags
constexpr unsigned char BC_V0 = 1;    // bface 22 / 221: v* = 0
constexpr unsigned char BC_U0 = 2;    // bface 22 / 222: u* = 0
constexpr unsigned char BC_UV0 = 4;   // bface 25: u* = v* = 0
constexpr unsigned char BC_KEEP = 8;  // no nodal solve (indnd = 1)

struct Dev1 {
  int nquad, npoin, ncell, mdegr, ncase, nsedov, sedov_cell[4];
  double gamlg, cfl, cimpd, tend, sedov_energy;
  const int *ipq;                     // [4][nquad]
  const int *esuv_ptr, *esuv;         // cells around each node (0-based)
  const int *ncor_ptr, *ncor;         // corners (iq*4 + iv) at each node, cells ascending
  const unsigned char *bc;            // [npoin] BC_* flags
  const unsigned char *wall;          // [npoin] limiter wall class 0, 2, 3, 10
  const double *x0, *y0;              // initial coordinates
  double *rc, *sc, *vol, *vcx, *vcy, *mass, *amatr;  // amatr [4][ncell]
  double *Un, *Us;                    // [12][ncell]
  double *xn, *yn, *xs, *ys, *us, *vs;
  double *bmax, *bmin;                // [5][npoin]
  double *lim;                        // [7][ncell]
  double *cf;                         // [5][8][nquad]
  double *rhs;                        // [12][ncell]
  double *dtpart;
  Scalars *sc_dev;
  // RZ (nrz = 1 true volume, 2 area-weighted; y the radius): alfrz = 1,
  // per node its boundary faces in face order (bf_ptr/bf_list) with the
  // faces' end nodes and codes, and (nrz = 2) the cell-averaged radius
  // geoel(11) = volume / area
  int nrz, nbfac;
  double alfrz;
  double *rbar;                       // [ncell] geoel(11), nrz = 2
  const int *bf_ptr, *bf_list;        // node -> boundary faces, ascending
  const int *bfn;                     // [2][nbfac] end nodes (0-based)
  const int *bfcode;                  // [nbfac] code * 1000 + sub-code
};

struct Rules {
  double g25[25][2], w25[25];
  double g36[36][2], w36[36];
};
__constant__ Rules cR;

__device__ __forceinline__ bool stopped(const Dev1 &d) { return d.sc_dev->done != 0; }
__device__ __forceinline__ double U(const Dev1 &d, const double *A, int k, int q, int e) {
  return A[(q * ND + k) * (size_t)d.ncell + e];
}

__device__ __forceinline__ void load4(const Dev1 &d, const double *X, const double *Y, int iq, double (*xp)[2]) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int p = d.ipq[k * d.nquad + iq];
    xp[k][0] = X[p];
    xp[k][1] = Y[p];
  }
}

// the straight quad's 9-node image (Limiterlag.f90:2040-2048)
__device__ __forceinline__ void image9(const double (*x4)[2], double (*xp)[2]) {
#pragma unroll
  for (int k = 0; k < 4; k++) { xp[k][0] = x4[k][0]; xp[k][1] = x4[k][1]; }
#pragma unroll
  for (int c = 0; c < 2; c++) {
    xp[4][c] = 0.5 * (xp[0][c] + xp[1][c]);
    xp[5][c] = 0.5 * (xp[1][c] + xp[2][c]);
    xp[6][c] = 0.5 * (xp[2][c] + xp[3][c]);
    xp[7][c] = 0.5 * (xp[3][c] + xp[0][c]);
    xp[8][c] = 0.5 * (xp[4][c] + xp[6][c]);
  }
}

// bilinear Jacobian at (r, s) (Limiterlag.f90:8262-8282)
__device__ __forceinline__ void jac4(const double (*x)[2], double r, double s, double &dxdr, double &dxds,
                                     double &dydr, double &dyds) {
  const double rp = 1.0 + r, rm = 1.0 - r, sp = 1.0 + s, sm = 1.0 - s;
  const double dr[4] = {-0.25 * sm, 0.25 * sm, 0.25 * sp, -0.25 * sp};
  const double ds[4] = {-0.25 * rm, -0.25 * rp, 0.25 * rp, 0.25 * rm};
  double a = 0.0, b = 0.0, c = 0.0, e = 0.0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    a = a + dr[k] * x[k][0];
    b = b + ds[k] * x[k][0];
    c = c + dr[k] * x[k][1];
    e = e + ds[k] * x[k][1];
  }
  dxdr = a; dxds = b; dydr = c; dyds = e;
}

__device__ __forceinline__ double barthfct(double umax, double umin, double uctr, double dunk) {
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

// The same limiter function with one division: with fiy = a / b,
// (fiy^2 + 2 fiy) / (fiy^2 + fiy + 2) = (a^2 + 2 a b) / (a^2 + a b + 2 b^2)
// (optimised kernels; equal up to rounding).
__device__ __forceinline__ double barthfct1(double umax, double umin, double uctr, double dunk) {
  if (!(dunk > 1.0e-8) && !(dunk < -1.0e-8)) return 1.0;
  const double a = 0.7 * ((dunk > 1.0e-8 ? umax : umin) - uctr), b = dunk;
  return fmin((a * a + 2.0 * a * b) / (a * a + a * b + 2.0 * b * b), 1.0);
}

template <bool FAST>
__device__ __forceinline__ double limfct(double umax, double umin, double uctr, double dunk) {
  return FAST ? barthfct1(umax, umin, uctr, dunk) : barthfct(umax, umin, uctr, dunk);
}

__device__ __forceinline__ double xv(int iv) { return (iv == 0 || iv == 3) ? -1.0 : 1.0; }
__device__ __forceinline__ double yv(int iv) { return (iv < 2) ? -1.0 : 1.0; }

// ---------------------------------------------------------------------------
// Initial geometry and fields: getgeoel_initial_lag (GetInitial.f90:1484-
// 1694), inifield_mcnew (Getrhslagmc.f90:3621-3917) and getunkno_initial_lag
// (GetInitial.f90:412-690) on the 9-node image, npoly = 1
// ---------------------------------------------------------------------------
__device__ double rho_initial1(const Dev1 &d, double xc, double yc) {
  if (d.ncase == 6) return (sqrt(xc * xc + yc * yc) <= 0.5) ? 1.0 : 0.125;
  return 1.0;
}

__device__ void getunkin1(const Dev1 &d, double *unkin, double xg, double yg, int ielem1, double volel, double xc,
                          double yc) {
  const double g = d.gamlg;
  double rhoini = 1.0, uini = 0.0, vini = 0.0, pini = 1.0;
  if (d.ncase == 3) {
    uini = -xg / sqrt(xg * xg + yg * yg);
    vini = -yg / sqrt(xg * xg + yg * yg);
    pini = 1.0e-6;
  } else if (d.ncase == 6) {
    double ieini;
    if (sqrt(xc * xc + (yc - 0.0) * (yc - 0.0)) <= 0.5) { rhoini = 1.0; ieini = 2.5; }
    else { rhoini = 0.125; ieini = 2.0; }
    pini = ieini * (g - 1.0) * rhoini;
  } else if (d.ncase == 7) {
    bool hit = false;
    for (int i = 0; i < d.nsedov; i++) hit |= (d.sedov_cell[i] == ielem1);
    pini = hit ? (g - 1.0) * 1.0 * d.sedov_energy / (1.0 * volel) : 1.0e-6;
  }
  unkin[0] = 1.0;
  unkin[1] = rhoini * uini;
  unkin[2] = rhoini * vini;
  unkin[3] = (pini / rhoini / (g - 1.0) + 0.5 * (uini * uini + vini * vini)) * rhoini;
}

__global__ void k1_init_geo(Dev1 d) {
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= d.nquad) return;
  const double alfrz = d.alfrz;
  double x4[4][2], xp[9][2], shp[9], dr[9], ds[9];
  load4(d, d.x0, d.y0, iq, x4);
  image9(x4, xp);
  double xc, yc;
  shp9v(0.0, 0.0, shp);
  map9(xp, shp, xc, yc);
  double xcent = 0, ycent = 0, volel = 0, masel = 0;
  double maselrz = 0, xcerz = 0, ycerz = 0, areel = 0;
  for (int ig = 0; ig < 36; ig++) {
    const double r = cR.g36[ig][0], s = cR.g36[ig][1], wi = cR.w36[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    const double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map9(xp, shp, xg, yg);
    const double rhog = rho_initial1(d, xc, yc);
    const double rcoef = 1.0 - alfrz + alfrz * yg;
    masel = masel + rhog * djaco * rcoef;
    volel = volel + djaco * rcoef;
    xcent = xcent + rhog * r * djaco * rcoef;
    ycent = ycent + rhog * s * djaco * rcoef;
    if (d.nrz == 2) {  // the area integrals of nrz = 2 (GetInitial.f90:1655-1666)
      maselrz = maselrz + rhog * djaco;
      xcerz = xcerz + rhog * r * djaco;
      ycerz = ycerz + rhog * s * djaco;
      areel = areel + djaco;
    }
  }
  d.rc[iq] = xcent / masel;
  d.sc[iq] = ycent / masel;
  d.vol[iq] = volel;
  d.mass[iq] = masel;
  if (d.nrz == 2) {  // GetInitial.f90:1682-1691
    d.rc[iq] = xcerz / maselrz;
    d.sc[iq] = ycerz / maselrz;
    d.mass[iq] = maselrz;
    d.rbar[iq] = volel / areel;
  }
}

__global__ void k1_init_fields(Dev1 d) {
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= d.nquad) return;
  const int e = iq;
  const double alfrz = d.alfrz;
  double x4[4][2], xp[9][2], shp[9], dr[9], ds[9];
  load4(d, d.x0, d.y0, iq, x4);
  image9(x4, xp);
  const double volel = d.vol[e], masel = d.mass[e], rc = d.rc[e], sc = d.sc[e];
  double unkin[4], rv[4] = {0, 0, 0, 0};
  const double xcel = xp[8][0], ycel = xp[8][1];
  for (int ig = 0; ig < 25; ig++) {
    const double r = cR.g25[ig][0], s = cR.g25[ig][1], wi = cR.w25[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    const double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map9(xp, shp, xg, yg);
    getunkin1(d, unkin, xg, yg, e + 1, volel, xcel, ycel);
    const double rcoef = 1.0 - alfrz + alfrz * yg;
    // nrz = 2 integrates over the area (Getrhslagmc.f90:3744-3754)
    if (d.nrz == 2) for (int q = 0; q < 4; q++) rv[q] = rv[q] + unkin[q] * djaco;
    else for (int q = 0; q < 4; q++) rv[q] = rv[q] + unkin[q] * djaco * rcoef;
  }
  double xc, yc;
  shp9v(rc, sc, shp);
  map9(xp, shp, xc, yc);
  double rhsini[ND][4], mm[4] = {0.0, 0.0, 0.0, 0.0}, f0 = 0.0;
  for (int k = 0; k < ND; k++)
    for (int q = 0; q < 4; q++) rhsini[k][q] = 0.0;
  for (int ig = 0; ig < 25; ig++) {
    const double r = cR.g25[ig][0], s = cR.g25[ig][1], wi = cR.w25[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    const double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map9(xp, shp, xg, yg);
    getunkin1(d, unkin, xg, yg, e + 1, volel, xc, yc);
    const double bq[ND] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < ND; k++) rhsini[k][q] = rhsini[k][q] + unkin[q] * bq[k] * djaco;
    const double rho0 = rho_initial1(d, xc, yc);
    const double rcoef = 1.0 - alfrz + alfrz * yg;
    if (d.nrz == 2) {  // the area mass matrix (GetInitial.f90:604-610)
      f0 = f0 + rho0 * djaco;
      mm[0] = mm[0] + rho0 * bq[1] * bq[1] * djaco;
      mm[2] = mm[2] + rho0 * bq[1] * bq[2] * djaco;
      mm[3] = mm[3] + rho0 * bq[2] * bq[2] * djaco;
      continue;
    }
    f0 = f0 + rho0 * djaco * rcoef;
    // mmatr(1,1), (2,1), (1,2), (2,2) (GetInitial.f90:622-627); (2,1) is not used
    mm[0] = mm[0] + rho0 * bq[1] * bq[1] * djaco * rcoef;
    mm[2] = mm[2] + rho0 * bq[1] * bq[2] * djaco * rcoef;
    mm[3] = mm[3] + rho0 * bq[2] * bq[2] * djaco * rcoef;
  }
  const double det = mm[0] * mm[3] - mm[2] * mm[2];
  const double a1 = mm[3] / det, a2 = -mm[2] / det, a3 = mm[0] / det;
  // nrz = 2 divides M^-1 by geoel(11) after the projection's copy was taken (GetInitial.f90:675)
  const double rb = (d.nrz == 2) ? d.rbar[e] : 1.0;
  d.amatr[0 * (size_t)d.ncell + e] = (d.nrz == 2) ? a1 / rb : a1;
  d.amatr[1 * (size_t)d.ncell + e] = (d.nrz == 2) ? a2 / rb : a2;
  d.amatr[2 * (size_t)d.ncell + e] = (d.nrz == 2) ? a3 / rb : a3;
  d.amatr[3 * (size_t)d.ncell + e] = (d.nrz == 2) ? 1.0 / f0 / rb : 1.0 / f0;
  const double mi[2][2] = {{a1, a2}, {a2, a3}};
  for (int q = 0; q < 4; q++) {
    d.Un[(q * ND + 0) * (size_t)d.ncell + e] = rv[q] / masel;
    for (int ix = 0; ix < 2; ix++) {
      double acc = 0.0;
      for (int iy = 0; iy < 2; iy++) acc = acc + mi[ix][iy] * rhsini[iy + 1][q];
      d.Un[(q * ND + ix + 1) * (size_t)d.ncell + e] = acc;
    }
  }
}

// ---------------------------------------------------------------------------
// getcellvol_lag on the 9-node image (Limiterlag.f90:2038-2165)
// ---------------------------------------------------------------------------
__global__ void k1_geom(Dev1 d, const double *X, const double *Y) {
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= d.nquad || stopped(d)) return;
  const double alfrz = d.alfrz;
  double x4[4][2], xp[9][2], shp[9], dr[9], ds[9];
  load4(d, X, Y, iq, x4);
  image9(x4, xp);
  double rcv = 0.0, scv = 0.0, volel = 0.0, areel = 0.0, rcvrz = 0.0, scvrz = 0.0;
  for (int ig = 0; ig < 36; ig++) {
    const double r = cR.g36[ig][0], s = cR.g36[ig][1], wi = cR.w36[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    double xg, yg;
    map9(xp, shp, xg, yg);
    const double rcoef = 1.0 - alfrz + alfrz * yg;
    const double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    volel = volel + djaco * rcoef;
    rcv = rcv + r * djaco * rcoef;
    scv = scv + s * djaco * rcoef;
    if (d.nrz == 2) {
      areel = areel + djaco;
      rcvrz = rcvrz + r * djaco;
      scvrz = scvrz + s * djaco;
    }
  }
  d.vol[iq] = volel;
  d.vcx[iq] = rcv / volel;
  d.vcy[iq] = scv / volel;
  if (d.nrz == 2) {  // the area centroid and geoel(11) (Limiterlag.f90:2149-2156)
    d.vcx[iq] = rcvrz / areel;
    d.vcy[iq] = scvrz / areel;
    d.rbar[iq] = volel / areel;
  }
  if (!(volel > 0.0)) atomicOr(&d.sc_dev->status, ST_NONPHYS);
}

// The same volume and volume centre in closed form: the 9-node image of a
// straight quad is its bilinear map, whose Jacobian is J0 + J1 r + J2 s, so
// V = 4 J0 and the centre in reference coordinates is (J1, J2) / (3 J0).
__global__ void k1_geom_fast(Dev1 d, const double *X, const double *Y) {
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= d.nquad || stopped(d)) return;
  double x[4][2];
  load4(d, X, Y, iq, x);
  const double e1 = 0.25 * (-x[0][0] + x[1][0] + x[2][0] - x[3][0]);
  const double e2 = 0.25 * (-x[0][0] - x[1][0] + x[2][0] + x[3][0]);
  const double e3 = 0.25 * (x[0][0] - x[1][0] + x[2][0] - x[3][0]);
  const double f1 = 0.25 * (-x[0][1] + x[1][1] + x[2][1] - x[3][1]);
  const double f2 = 0.25 * (-x[0][1] - x[1][1] + x[2][1] + x[3][1]);
  const double f3 = 0.25 * (x[0][1] - x[1][1] + x[2][1] - x[3][1]);
  const double j0 = e1 * f2 - f1 * e2, j1 = e1 * f3 - f1 * e3, j2 = e3 * f2 - f3 * e2;
  const double volel = 4.0 * j0;
  d.vol[iq] = volel;
  d.vcx[iq] = j1 / (3.0 * j0);
  d.vcy[iq] = j2 / (3.0 * j0);
  if (!(volel > 0.0)) atomicOr(&d.sc_dev->status, ST_NONPHYS);
}

// ---------------------------------------------------------------------------
// Node bounds (barthlimit_lag_vtxunknew, Getrhslagmctria.f90:2548-2641):
// max/min over the cells around the node, so the visiting order is free
// ---------------------------------------------------------------------------
__global__ void k1_bounds(Dev1 d) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.npoin || stopped(d)) return;
  const double g = d.gamlg;
  double mx[5], mn[5];
#pragma unroll
  for (int q = 0; q < 5; q++) { mx[q] = -1.0e10; mn[q] = 1.0e10; }
  for (int i = d.esuv_ptr[p]; i < d.esuv_ptr[p + 1]; i++) {
    const int e = d.esuv[i];
    const double rhom = U(d, d.Us, 0, 0, e);
    const double uctr = U(d, d.Us, 0, 1, e), vctr = U(d, d.Us, 0, 2, e), ectr = U(d, d.Us, 0, 3, e);
    const double rhoct = 1.0 / rhom;
    const double pctr = fmax(EPS_S, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
    const double v[5] = {rhom, uctr, vctr, pctr, ectr};
#pragma unroll
    for (int q = 0; q < 5; q++) {
      if (v[q] > mx[q]) mx[q] = v[q];
      if (v[q] < mn[q]) mn[q] = v[q];
    }
  }
#pragma unroll
  for (int q = 0; q < 5; q++) {
    d.bmax[q * (size_t)d.npoin + p] = mx[q];
    d.bmin[q * (size_t)d.npoin + p] = mn[q];
  }
}

// ---------------------------------------------------------------------------
// Limiter and corner coefficients of one quad
// ---------------------------------------------------------------------------
// RZ corner coefficients (getriem_quadrz, Getrhslagmc.f90:17963-18336):
// 4 corner faces per vertex (its two edges, each twice: faces 1, 3 the edge
// to the previous vertex, 2, 4 to the next) with the radius weights of the
// edge halves, the acoustic impedance rho c only and the 1e-9 floors; stored
// per face in cf[(k*16 + f + 4*iv)*nquad + iq] (k: m, m u, m v, sigma.n A).
template <int MD>
__device__ void rz_corners(const Dev1 &d, int iq, const double (*x4)[2], const int *ip, const double (*u)[ND],
                           const double (*bq)[ND], const double (*uvq)[4], double af4, double fi11, double fi12,
                           double fi22) {
  const double g = d.gamlg, eps9 = 1.0e-09, alfrz = d.alfrz;
  double fn[4][3], rco[4];
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const int b = (f + 1) & 3;
    const double anx = x4[b][1] - x4[f][1];
    const double any = -(x4[b][0] - x4[f][0]);
    fn[f][0] = anx / sqrt(anx * anx + any * any);
    fn[f][1] = any / sqrt(anx * anx + any * any);
    fn[f][2] = sqrt(anx * anx + any * any);
    rco[f] = 1.0 - alfrz + alfrz * fabs(x4[f][1]);
  }
  const double rhomc = u[0][0], uctr = u[1][0], vctr = u[2][0], ectr = u[3][0];
  const double rhoct = 1.0 / rhomc;
  const double pctr = fmax(eps9, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
  const double sdctr = sqrt(fmax(eps9, g * pctr / rhoct));
  const double murie = rhoct * sdctr;
  const double dudr = fi11 * u[1][1] + fi12 * u[2][1];
  const double duds = fi11 * u[1][2] + fi12 * u[2][2];
  const double dvdr = fi12 * u[1][1] + fi22 * u[2][1];
  const double dvds = fi12 * u[1][2] + fi22 * u[2][2];
#pragma unroll
  for (int iv = 0; iv < 4; iv++) {
    const int vp = (iv + 3) & 3, vx = (iv + 1) & 3;
    const double rhovt = 1.0 / uvq[iv][0];
    const double ev = uvq[iv][3];
    double pvtx = fmax(eps9, (g - 1.0) * rhovt * (ev - 0.5 * (uvq[iv][1] * uvq[iv][1] + uvq[iv][2] * uvq[iv][2])));
    const double uvl = u[1][0] + dudr * bq[iv][1] + duds * bq[iv][2];
    const double vvl = u[2][0] + dvdr * bq[iv][1] + dvds * bq[iv][2];
    pvtx = pctr + af4 * (pvtx - pctr);
    const double sig = -pvtx;
    const double acnx = d.us[ip[iv]] - uvl, acny = d.vs[ip[iv]] - vvl;
    const double nrm = sqrt(acnx * acnx + acny * acny);
    double aj0, aj1;
    if (nrm < TINY_S) { aj0 = TINY_S; aj1 = TINY_S; }
    else { aj0 = acnx / nrm; aj1 = acny / nrm; }
    const double aj2 = nrm / sdctr;
#pragma unroll
    for (int f = 0; f < 4; f++) {
      const int edge = (f & 1) ? iv : vp;
      const double rw = (f < 2) ? 3.0 * rco[iv] : 1.0 * rco[iv];
      const double ro = (f & 1) ? rco[vx] : rco[vp];
      const double n1 = fn[edge][0], n2 = fn[edge][1];
      const double area = 0.5 * ((rw + ro) / 3.0 * 0.5 * fn[edge][2]);
      const double vnau = (aj2 < 1.0e12) ? 1.0 : n1 * aj0 + n2 * aj1;
      const double m = murie * area * fabs(vnau);
      const double mu1 = m * uvl + 0.0 * vvl;
      const double mu2 = 0.0 * uvl + m * vvl;
      const double s1 = sig * area * n1 + (0.0 + 0.0) * area * n2;
      const double s2 = (0.0 + 0.0) * area * n1 + sig * area * n2;
      const int slot = f + 4 * iv;
      d.cf[(0 * 16 + slot) * (size_t)d.nquad + iq] = m;
      d.cf[(1 * 16 + slot) * (size_t)d.nquad + iq] = mu1;
      d.cf[(2 * 16 + slot) * (size_t)d.nquad + iq] = mu2;
      d.cf[(3 * 16 + slot) * (size_t)d.nquad + iq] = s1;
      d.cf[(4 * 16 + slot) * (size_t)d.nquad + iq] = s2;
    }
  }
}

// Area-weighted RZ (nrz = 2), at the start of every stage but the very
// first: the mass centre geoel(1:2) of the limited DG density over the
// cell's area, 5 fixed-point passes from the area centroid
// (getgeoel_lagmc_rzawrev, Getrhslagrz.f90:4812-4994), then M^-1 of the
// area mass matrix about it divided by geoel(11) (getamatr_lagmc_rzawrev,
// :3949-4219).  Writes rc, sc and amatr of quad iq.
template <int MD>
__device__ void aw_rev(const Dev1 &d, int iq, const double (*x4)[2], const double (*u)[ND], double af1, double &rc,
                       double &sc) {
  double xp[9][2], dr[9], ds[9];
  image9(x4, xp);
  const double rhomc = u[0][0];
  for (int iloop = 1; iloop <= 5; iloop++) {
    double xcent = 0.0, ycent = 0.0, masel = 0.0;
    for (int ig = 0; ig < 36; ig++) {
      const double r = cR.g36[ig][0], s = cR.g36[ig][1], wi = cR.w36[ig];
      shp9d(r, s, dr, ds);
      Jac j = jac9(xp, dr, ds);
      const double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
      const double bq[ND] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
      double rhomg = 0.0;
#pragma unroll
      for (int k = 0; k < MD; k++) rhomg = rhomg + u[0][k] * bq[k];
      if (iloop == 1) rhomg = rhomc;
      rhomg = rhomc + af1 * (rhomg - rhomc);
      const double rhog = 1.0 / rhomg;
      masel = masel + 1.0 / rhomc * djaco;
      xcent = xcent + rhog * r * djaco;
      ycent = ycent + rhog * s * djaco;
    }
    rc = xcent / masel;
    sc = ycent / masel;
  }
  double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
  for (int ig = 0; ig < 25; ig++) {
    const double r = cR.g25[ig][0], s = cR.g25[ig][1], wi = cR.w25[ig];
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    const double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    const double bq[ND] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
    double rhomg = 0.0;
#pragma unroll
    for (int k = 0; k < MD; k++) rhomg = rhomg + u[0][k] * bq[k];
    rhomg = rhomc + af1 * (rhomg - rhomc);
    const double rhog = 1.0 / rhomg;
    f0 = f0 + rhog * djaco;
    f1 = f1 + rhog * (r - rc) / 1.0 * (r - rc) / 1.0 * djaco;
    f2 = f2 + rhog * (r - rc) / 1.0 * (s - sc) / 1.0 * djaco;
    f3 = f3 + rhog * (s - sc) / 1.0 * (s - sc) / 1.0 * djaco;
  }
  const double det = f1 * f3 - f2 * f2;
  const double rb = d.rbar[iq];
  const size_t nc = d.ncell;
  d.amatr[0 * nc + iq] = f3 / det / rb;
  d.amatr[1 * nc + iq] = -f2 / det / rb;
  d.amatr[2 * nc + iq] = f1 / det / rb;
  d.amatr[3 * nc + iq] = 1.0 / f0 / rb;
  d.rc[iq] = rc;
  d.sc[iq] = sc;
}

// Area-weighted RZ corner coefficients (getriem_quadrzaw, Getrhslagrz.f90:
// 1389-1669): the two corner faces of the plane solver (half of each edge at
// the vertex, no radius weight), the acoustic impedance rho c and the 1e-8
// floors, on the vertex values of the stage's mass centre; stored per face
// in cf[(k*8 + f + 2*iv)*nquad + iq] (k: m, m u, m v, sigma.n A).
template <int MD>
__device__ void aw_corners(const Dev1 &d, int iq, const double (*x4)[2], const int *ip, const double (*u)[ND],
                           double rc, double sc, double af4, double fi11, double fi12, double fi22) {
  const double g = d.gamlg, eps8 = 1.0e-08, slpdu = (g + 1.0) / 2.0;
  double fn[4][3], bq[4][ND], uvq[4][4];
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const int b = (f + 1) & 3;
    const double anx = x4[b][1] - x4[f][1];
    const double any = -(x4[b][0] - x4[f][0]);
    fn[f][0] = anx / sqrt(anx * anx + any * any);
    fn[f][1] = any / sqrt(anx * anx + any * any);
    fn[f][2] = sqrt(anx * anx + any * any);
    bq[f][0] = 1.0; bq[f][1] = (xv(f) - rc) / 1.0; bq[f][2] = (yv(f) - sc) / 1.0;
  }
#pragma unroll
  for (int iv = 0; iv < 4; iv++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      double a = 0.0;
#pragma unroll
      for (int k = 0; k < MD; k++) a = a + u[q][k] * bq[iv][k];
      uvq[iv][q] = a;
    }
  const double rhomc = u[0][0], uctr = u[1][0], vctr = u[2][0], ectr = u[3][0];
  const double rhoct = 1.0 / rhomc;
  const double pctr = fmax(eps8, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
  const double sdctr = sqrt(fmax(eps8, g * pctr / rhoct));
  const double dudr = fi11 * u[1][1] + fi12 * u[2][1];
  const double duds = fi11 * u[1][2] + fi12 * u[2][2];
  const double dvdr = fi12 * u[1][1] + fi22 * u[2][1];
  const double dvds = fi12 * u[1][2] + fi22 * u[2][2];
#pragma unroll
  for (int iv = 0; iv < 4; iv++) {
    const double rhovt = 1.0 / uvq[iv][0];
    const double ev = uvq[iv][3];
    double pvtx = fmax(eps8, (g - 1.0) * rhovt * (ev - 0.5 * (uvq[iv][1] * uvq[iv][1] + uvq[iv][2] * uvq[iv][2])));
    const double uvl = u[1][0] + dudr * bq[iv][1] + duds * bq[iv][2];
    const double vvl = u[2][0] + dvdr * bq[iv][1] + dvds * bq[iv][2];
    pvtx = pctr + af4 * (pvtx - pctr);
    const double sig = -pvtx;
    const double acnx = d.us[ip[iv]] - uvl, acny = d.vs[ip[iv]] - vvl;
    const double nrm = sqrt(acnx * acnx + acny * acny);
    double aj0, aj1;
    if (nrm < TINY_S) { aj0 = TINY_S; aj1 = TINY_S; }
    else { aj0 = acnx / nrm; aj1 = acny / nrm; }
    const double aj2 = nrm / sdctr;
#pragma unroll
    for (int f = 0; f < 2; f++) {
      const int edge = (f == 0) ? ((iv + 3) & 3) : iv;
      const double n1 = fn[edge][0], n2 = fn[edge][1];
      const double area = 0.5 * fn[edge][2];
      // the shock term is switched off in the reference: deltu = 0 |du.n|
      const double deltu = 0.0 * fabs(acnx * n1 + acny * n2);
      const double murie = rhoct * sdctr + rhoct * slpdu * deltu;
      const double vnau = (aj2 < 1.0e12) ? 1.0 : n1 * aj0 + n2 * aj1;
      const double m = murie * area * fabs(vnau);
      const double mu1 = m * uvl + 0.0 * vvl;
      const double mu2 = 0.0 * uvl + m * vvl;
      const double s1 = sig * area * n1 + 0.0 * area * n2;
      const double s2 = 0.0 * area * n1 + sig * area * n2;
      const int slot = f + 2 * iv;
      d.cf[(0 * 8 + slot) * (size_t)d.nquad + iq] = m;
      d.cf[(1 * 8 + slot) * (size_t)d.nquad + iq] = mu1;
      d.cf[(2 * 8 + slot) * (size_t)d.nquad + iq] = mu2;
      d.cf[(3 * 8 + slot) * (size_t)d.nquad + iq] = s1;
      d.cf[(4 * 8 + slot) * (size_t)d.nquad + iq] = s2;
    }
  }
}

template <int MD, bool FAST, int GEO>
__device__ void cell_pass(const Dev1 &d, int iq, int rev) {
  const int e = iq;
  const double g = d.gamlg, epsd = 1.0e-6, slpdu = (g + 1.0) / 2.0;
  double x4[4][2];
  load4(d, d.xs, d.ys, iq, x4);
  int ip[4];
#pragma unroll
  for (int k = 0; k < 4; k++) ip[k] = d.ipq[k * d.nquad + iq];
  const double rc = d.rc[e], sc = d.sc[e];
  double u[4][ND];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int k = 0; k < ND; k++) u[q][k] = U(d, d.Us, k, q, e);
  double bq[4][ND];
#pragma unroll
  for (int iv = 0; iv < 4; iv++) { bq[iv][0] = 1.0; bq[iv][1] = (xv(iv) - rc) / 1.0; bq[iv][2] = (yv(iv) - sc) / 1.0; }
  // vertex values of the unlimited DOFs
  double uvq[4][4];
#pragma unroll
  for (int iv = 0; iv < 4; iv++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      double a = 0.0;
#pragma unroll
      for (int k = 0; k < MD; k++) a = a + u[q][k] * bq[iv][k];
      uvq[iv][q] = a;
    }
  const double rhom = u[0][0], uctr = u[1][0], vctr = u[2][0], ectr = u[3][0];
  const double rhoct = 1.0 / rhom;
  const double pctr_s = fmax(EPS_S, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));

  // (1) aflim(1..4) against the node bounds (Limiterlag.f90:69-188)
  double af[4];
  {
    const double unctr[4] = {1.0 / rhoct, uctr, vctr, pctr_s};
#pragma unroll
    for (int q = 0; q < 4; q++) af[q] = 0.0;
#pragma unroll
    for (int iv = 0; iv < 4; iv++) {
      const double rhov = 1.0 / uvq[iv][0];
      const double uv = uvq[iv][1], vv = uvq[iv][2], ev = uvq[iv][3];
      const double pvtx = fmax(EPS_S, (g - 1.0) * rhov * (ev - 0.5 * (uv * uv + vv * vv)));
      const double w[4] = {1.0 / rhov, uv, vv, pvtx};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const double dunk = w[q] - unctr[q];
        const double a = limfct<FAST>(d.bmax[q * (size_t)d.npoin + ip[iv]], d.bmin[q * (size_t)d.npoin + ip[iv]],
                                      unctr[q], dunk);
        if (iv == 0 || a < af[q]) af[q] = a;
      }
    }
  }

  // (2) the velocity limited in the principal frame of the strain rate
  // (barthlimit_sympre_quadlb, Limiterlag.f90:8242-8692)
  double m11 = 0.0, m12 = 0.0, m21 = 0.0, m22 = 0.0;
  {
    const double dudr = u[1][1] / 1.0, duds = u[1][2] / 1.0, dvdr = u[2][1] / 1.0, dvds = u[2][2] / 1.0;
    double dxdr, dxds, dydr, dyds;
    jac4(x4, rc, sc, dxdr, dxds, dydr, dyds);
    const double jacom = dxdr * dyds - dydr * dxds;
    const double drdx = dyds / jacom, drdy = -dxds / jacom, dsdx = -dydr / jacom, dsdy = dxdr / jacom;
    const double dudx = dudr * drdx + duds * dsdx, dudy = dudr * drdy + duds * dsdy;
    const double dvdx = dvdr * drdx + dvds * dsdx, dvdy = dvdr * drdy + dvds * dsdy;
    const double matra = dudx, matrb = 0.5 * (dudy + dvdx), matrc = matrb, matrd = dvdy;
    const double mapt = matra + matrd, mapd = matra * matrd - matrb * matrc;
    const double lamda1 = 0.5 * mapt + sqrt(0.25 * (mapt * mapt) - mapd);
    const double lamda2 = 0.5 * mapt - sqrt(0.25 * (mapt * mapt) - mapd);
    if (fabs(matrc) > 1.0e-8) {
      const double lmat1 = sqrt((lamda1 - matrd) * (lamda1 - matrd) + matrc * matrc);
      const double lmat2 = sqrt((lamda2 - matrd) * (lamda2 - matrd) + matrc * matrc);
      const double a1 = (lamda1 - matrd) / lmat1, b1 = matrc / lmat1;
      const double a2 = (lamda2 - matrd) / lmat2, b2 = matrc / lmat2;
      if (matrc > 0.0) { m11 = a1; m12 = b1; m21 = a2; m22 = b2; }
      else { m21 = a1; m22 = b1; m11 = a2; m12 = b2; }
    }
  }
  double fl1 = 0.0, fl2 = 0.0;
  {
    const double uc = uctr * m11 + vctr * m12, vc = uctr * m21 + vctr * m22;
#pragma unroll
    for (int iv = 0; iv < 4; iv++) {
      const double ur = uvq[iv][1] * m11 + uvq[iv][2] * m12;
      const double vr = uvq[iv][1] * m21 + uvq[iv][2] * m22;
      double mx1 = uc, mx2 = vc, mn1 = uc, mn2 = vc;
      const int p = ip[iv];
      const int cls = (d.ncase != 1) ? d.wall[p] : 0;
      auto take = [&](double a, double b) {
        const double ul = a * m11 + b * m12;
        const double vl = a * m21 + b * m22;
        mx1 = fmax(mx1, ul); mx2 = fmax(mx2, vl);
        mn1 = fmin(mn1, ul); mn2 = fmin(mn2, vl);
      };
      for (int i = d.esuv_ptr[p]; i < d.esuv_ptr[p + 1]; i++) {
        const int je = d.esuv[i];
        const double uj = U(d, d.Us, 0, 1, je), vj = U(d, d.Us, 0, 2, je);
        // the cell's own average, then its images across the walls at the node
        take(uj, vj);
        if (cls == 3 || cls == 10) take(uj, -vj);
        if (cls == 2 || cls == 10) take(-uj, vj);
        if (cls == 10) take(-uj, -vj);
      }
      const double a1 = limfct<FAST>(mx1, mn1, uc, ur - uc);
      const double a2 = limfct<FAST>(mx2, mn2, vc, vr - vc);
      if (iv == 0 || a1 < fl1) fl1 = a1;
      if (iv == 0 || a2 < fl2) fl2 = a2;
    }
  }
  // afvec = R^T diag(fixi, fiet) R, R = mapmt (Limiterlag.f90:8679-8691)
  const double fi11 = (m11 * m11) * fl1 + (m21 * m21) * fl2;
  const double fi12 = m11 * m12 * fl1 + m21 * m22 * fl2;
  const double fi22 = (m12 * m12) * fl1 + (m22 * m22) * fl2;

  // (3) aflim(5): the energy of the limited vertex state (Limiterlag.f90:290-380)
  double af5 = 0.0;
#pragma unroll
  for (int iv = 0; iv < 4; iv++) {
    const double rhov = 1.0 / uvq[iv][0];
    const double uv = uvq[iv][1], vv = uvq[iv][2], ev = uvq[iv][3];
    const double pvtx = fmax(EPS_S, (g - 1.0) * rhov * (ev - 0.5 * (uv * uv + vv * vv)));
    const double t = rhom + af[0] * (1.0 / rhov - rhom);
    const double pv = pctr_s + af[3] * (pvtx - pctr_s);
    const double e5 = pv / (g - 1.0) * t + 0.5 * (uv * uv + vv * vv);
    const double a = limfct<FAST>(d.bmax[4 * (size_t)d.npoin + ip[iv]], d.bmin[4 * (size_t)d.npoin + ip[iv]],
                                  ectr, e5 - ectr);
    if (iv == 0 || a < af5) af5 = a;
  }
  const size_t nc = d.ncell;
  d.lim[0 * nc + e] = af[0];
  d.lim[1 * nc + e] = af[3];
  d.lim[2 * nc + e] = af5;
  d.lim[3 * nc + e] = fi11;
  d.lim[4 * nc + e] = fi12;
  d.lim[5 * nc + e] = fi12;
  d.lim[6 * nc + e] = fi22;

  if (GEO == 1) {
    rz_corners<MD>(d, iq, x4, ip, u, bq, uvq, af[3], fi11, fi12, fi22);
    return;
  }
  if (GEO == 2) {
    // the stage's mass centre and mass matrix (Getrhslagmc.f90:6883-6886),
    // then the corners on the vertex values about that centre
    double rcn = rc, scn = sc;
    if (rev) aw_rev<MD>(d, iq, x4, u, af[0], rcn, scn);
    aw_corners<MD>(d, iq, x4, ip, u, rcn, scn, af[3], fi11, fi12, fi22);
    return;
  }
  // (4) corner Riemann coefficients (getriem_quad_matrixsym, Limiterlag.f90:
  // 708-1033): face f of quad iq joins vertices f and f+1, its normal is
  // (dy, -dx)/|.| (getfnds_lag_mc_hybrid, Getrhslagmc.f90:2210-2262)
  double fn[4][3];
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const int b = (f + 1) & 3;
    const double anx = x4[b][1] - x4[f][1];
    const double any = -(x4[b][0] - x4[f][0]);
    fn[f][0] = anx / sqrt(anx * anx + any * any);
    fn[f][1] = any / sqrt(anx * anx + any * any);
    fn[f][2] = sqrt(anx * anx + any * any);
  }
  const double pctr = fmax(epsd, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
  const double sdctr = sqrt(fmax(epsd, g * pctr / rhoct));
  double csum[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const double dudr = fi11 * u[1][1] + fi12 * u[2][1];
  const double duds = fi11 * u[1][2] + fi12 * u[2][2];
  const double dvdr = fi12 * u[1][1] + fi22 * u[2][1];
  const double dvds = fi12 * u[1][2] + fi22 * u[2][2];
#pragma unroll
  for (int iv = 0; iv < 4; iv++) {
    const double rhovt = 1.0 / uvq[iv][0];
    const double ev = uvq[iv][3];
    double pvtx = fmax(epsd, (g - 1.0) * rhovt * (ev - 0.5 * (uvq[iv][1] * uvq[iv][1] + uvq[iv][2] * uvq[iv][2])));
    const double uvl = uctr + dudr * bq[iv][1] + duds * bq[iv][2];
    const double vvl = vctr + dvdr * bq[iv][1] + dvds * bq[iv][2];
    pvtx = pctr + af[3] * (pvtx - pctr);
    const double sig = -pvtx + 0.0;
    const int p = ip[iv];
    const double us0 = d.us[p], vs0 = d.vs[p];
    const double acnx = us0 - uvl, acny = vs0 - vvl;
    const double nrm = sqrt(acnx * acnx + acny * acny);
    double aj0, aj1;
    if (nrm < TINY_S) { aj0 = TINY_S; aj1 = TINY_S; }
    else { aj0 = acnx / nrm; aj1 = acny / nrm; }
    const double aj2 = nrm / sdctr;
#pragma unroll
    for (int f = 0; f < 2; f++) {
      const int face = (f == 0) ? ((iv + 3) & 3) : iv;
      const double n1 = fn[face][0], n2 = fn[face][1];
      const double area = (2.0 * 1.0 + 1.0) / 3.0 * 0.5 * fn[face][2];
      const double deltu = fabs(acnx * n1 + acny * n2);
      const double murie = rhoct * sdctr + d.cimpd * rhoct * slpdu * deltu;
      // getriecoef_matrixnew (Limiterlag.f90:1037-1076): a diagonal mu A
      const double vnau = (aj2 < 1.0e12) ? 1.0 : n1 * aj0 + n2 * aj1;
      const double m = murie * area * fabs(vnau);
      const double mu1 = m * uvl + 0.0 * vvl;
      const double mu2 = 0.0 * uvl + m * vvl;
      const double s1 = sig * area * n1 + (0.0 + 0.0) * area * n2;
      const double s2 = (0.0 + 0.0) * area * n1 + sig * area * n2;
      if (FAST) {
        const double v[5] = {m, mu1, mu2, s1, s2};
#pragma unroll
        for (int k = 0; k < 5; k++) csum[k] = (f == 0) ? v[k] : csum[k] + v[k];
      } else {
        const int slot = f + 2 * iv;
        d.cf[(0 * 8 + slot) * (size_t)d.nquad + iq] = m;
        d.cf[(1 * 8 + slot) * (size_t)d.nquad + iq] = mu1;
        d.cf[(2 * 8 + slot) * (size_t)d.nquad + iq] = mu2;
        d.cf[(3 * 8 + slot) * (size_t)d.nquad + iq] = s1;
        d.cf[(4 * 8 + slot) * (size_t)d.nquad + iq] = s2;
      }
    }
    if (FAST) {
#pragma unroll
      for (int k = 0; k < 5; k++) d.cf[(k * 4 + iv) * (size_t)d.nquad + iq] = csum[k];
    }
  }
}
// compiled for 4 resident blocks of 128 per SM (128 registers): on the
// 1024 x 512 Sod mesh 136 us per launch against 161 us at 138 registers
// GEO: 0 plane, 1 RZ (nrz = 1), 2 area-weighted RZ (nrz = 2); `stage` is
// the RK stage (1-based): nrz = 2 renews the mass centre and mass matrix at
// every stage but the first of step 1
template <int MD, bool FAST, int GEO>
__global__ void __launch_bounds__(128, 4) k1_cell(Dev1 d, int stage) {
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= d.nquad || stopped(d)) return;
  const int rev = (GEO == 2) && (stage > 1 || d.sc_dev->itime > 1);
  cell_pass<MD, FAST, GEO>(d, iq, rev);
}

// ---------------------------------------------------------------------------
// Nodal solve (getndvelo_lag_mc_matrixsym, Limiterlag.f90:478-642): the
// corner sums in the order the reference scatters them (cells ascending,
// corner faces 1, 2), the 2x2 solve and the wall conditions
// ---------------------------------------------------------------------------
// RZ nodal solve (getndvelo_lagmc_rz, Getrhslagmc.f90:17284-17597, with
// getbc_lagmaire2, Getrhslag.f90:11269-11491): the node sums of the 4 corner
// faces per corner in the reference's scatter order; at the node's boundary
// faces (in face order) the radius-weighted area vectors of the velocity
// walls (code 22) and the pressure forces of code 21 (ncase 3: p = 1e-6);
// fpres removes the wall-normal velocity from the solve; node 1 is held, 222
// holds u and code 25 both (the 221 zeroing is commented out in RZ).
__device__ void rz_node(const Dev1 &d, int p) {
  double n11 = 0.0, n21 = 0.0, n12 = 0.0, n22 = 0.0, a1 = 0.0, a2 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int i = d.ncor_ptr[p]; i < d.ncor_ptr[p + 1]; i++) {
    const int c = d.ncor[i], iq = c >> 2, iv = c & 3;
    for (int f = 0; f < 4; f++) {
      const int slot = f + 4 * iv;
      const double m = d.cf[(0 * 16 + slot) * (size_t)d.nquad + iq];
      n11 = n11 + m;
      n21 = n21 + 0.0;
      n12 = n12 + 0.0;
      n22 = n22 + m;
      a1 = a1 + d.cf[(1 * 16 + slot) * (size_t)d.nquad + iq];
      a2 = a2 + d.cf[(2 * 16 + slot) * (size_t)d.nquad + iq];
      s1 = s1 + d.cf[(3 * 16 + slot) * (size_t)d.nquad + iq];
      s2 = s2 + d.cf[(4 * 16 + slot) * (size_t)d.nquad + iq];
    }
  }
  const double alfrz = d.alfrz;
  double bvx = 0.0, bvy = 0.0, bpx = 0.0, bpy = 0.0;
  bool wall22 = false;
  for (int i = d.bf_ptr[p]; i < d.bf_ptr[p + 1]; i++) {
    const int ifa = d.bf_list[i];
    const int q0 = d.bfn[ifa], q1 = d.bfn[d.nbfac + ifa], code = d.bfcode[ifa];
    const double anx = d.ys[q1] - d.ys[q0];
    const double any = -(d.xs[q1] - d.xs[q0]);
    const double gf3 = sqrt(anx * anx + any * any);
    const double r0 = 1.0 - alfrz + alfrz * d.ys[q0], r1 = 1.0 - alfrz + alfrz * d.ys[q1];
    // this node's weight (2 r_self + r_other) / 3, divided last as the reference does
    const double wsum = (q0 == p) ? (2.0 * r0 + r1) : (2.0 * r1 + r0);
    if (code / 1000 == 22) {
      wall22 = true;
      double bsnx = 0.0, bsny = 0.0;
      const int sub = code % 1000;
      if (sub == 221) {
        bsnx = 0.0 * gf3 * 0.5;
        bsny = -1.0 * gf3 * 0.5;
        if (d.ncase == 1 || d.ncase == 2 || d.ncase == 12) {
          if (d.ys[q0] < 1.0e-6 && d.ys[q1] < 1.0e-6) { bsnx = 0.0 * gf3 * 0.5; bsny = -1.0 * gf3 * 0.5; }
          else if (fabs(d.ys[q0] - 1.0) < 1.0e-6 && fabs(d.ys[q1] - 1.0) < 1.0e-6) { bsnx = 0.0 * gf3 * 0.5; bsny = 1.0 * gf3 * 0.5; }
        }
      } else if (sub == 222) {
        bsnx = -1.0 * gf3 * 0.5;
        bsny = 0.0 * gf3 * 0.5;
        if (d.ncase == 1) {
          if (d.xs[q0] < 1.0e-6 && d.xs[q1] < 1.0e-6) { bsnx = -1.0 * gf3 * 0.5; bsny = 0.0 * gf3 * 0.5; }
          else if (fabs(d.xs[q0] - 1.0) < 1.0e-6 && fabs(d.xs[q1] - 1.0) < 1.0e-6) { bsnx = 1.0 * gf3 * 0.5; bsny = 0.0 * gf3 * 0.5; }
        }
      }
      bvx = bvx + bsnx * wsum / 3.0;
      bvy = bvy + bsny * wsum / 3.0;
    } else if (code / 1000 == 21 && d.ncase == 3) {
      const double pres0 = 1.0e-6;
      const double bsnx = anx / gf3 * gf3 * 0.5, bsny = any / gf3 * gf3 * 0.5;
      bpx = bpx + pres0 * bsnx * wsum / 3.0;
      bpy = bpy + pres0 * bsny * wsum / 3.0;
    }
  }
  double fpx = 0.0, fpy = 0.0;
  if (wall22) {
    const double detma = n11 * n22 - n21 * n12;
    const double i11 = n22 / detma, i12 = -n12 / detma, i21 = -n21 / detma, i22 = n11 / detma;
    const double coefl = (i11 * bvx + i12 * bvy) * bvx + (i21 * bvx + i22 * bvy) * bvy;
    const double rhsx = a1 - s1 - bpx, rhsy = a2 - s2 - bpy;
    const double coefr = (i11 * rhsx + i12 * rhsy) * bvx + (i21 * rhsx + i22 * rhsy) * bvy;
    fpx = coefr / fmax(1.0e-16, coefl) * bvx;
    fpy = coefr / fmax(1.0e-16, coefl) * bvy;
  }
  fpx = fpx + bpx;
  fpy = fpy + bpy;
  const unsigned char bc = d.bc[p];
  double us = d.us[p], vs = d.vs[p];
  if (!(bc & BC_KEEP)) {
    const double detma = n11 * n22 - n21 * n12;
    const double i11 = n22 / detma, i12 = -n12 / detma, i21 = -n21 / detma, i22 = n11 / detma;
    const double r1 = a1 - s1 - fpx, r2 = a2 - s2 - fpy;
    us = i11 * r1 + i12 * r2;
    vs = i21 * r1 + i22 * r2;
  }
  if (p == 0) { us = 0.0; vs = 0.0; }
  if (bc & BC_UV0) vs = 0.0;
  if (bc & (BC_U0 | BC_UV0)) us = 0.0;
  d.us[p] = us;
  d.vs[p] = vs;
}

// Area-weighted RZ nodal solve (getndvelo_lagmc_rzaw, Getrhslagrz.f90:
// 822-1100, with getbc_lagmaire_rzaw, GetBClag.f90:57-250): the node sums of
// the two corner faces per corner in the reference's scatter order; at the
// node's boundary faces (in face order) the area vectors of the velocity
// walls (code 22, half the face at each end) and the pressure forces of
// code 21 (ncase 3: p = 1e-6); fpres removes the wall-normal velocity from
// the solve; then 221 holds v, 222 holds u and code 25 both.
__device__ void aw_node(const Dev1 &d, int p) {
  double n11 = 0.0, n21 = 0.0, n12 = 0.0, n22 = 0.0, a1 = 0.0, a2 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int i = d.ncor_ptr[p]; i < d.ncor_ptr[p + 1]; i++) {
    const int c = d.ncor[i], iq = c >> 2, iv = c & 3;
    for (int f = 0; f < 2; f++) {
      const int slot = f + 2 * iv;
      const double m = d.cf[(0 * 8 + slot) * (size_t)d.nquad + iq];
      n11 = n11 + m;
      n21 = n21 + 0.0;
      n12 = n12 + 0.0;
      n22 = n22 + m;
      a1 = a1 + d.cf[(1 * 8 + slot) * (size_t)d.nquad + iq];
      a2 = a2 + d.cf[(2 * 8 + slot) * (size_t)d.nquad + iq];
      s1 = s1 + d.cf[(3 * 8 + slot) * (size_t)d.nquad + iq];
      s2 = s2 + d.cf[(4 * 8 + slot) * (size_t)d.nquad + iq];
    }
  }
  double bvx = 0.0, bvy = 0.0, bpx = 0.0, bpy = 0.0;
  bool wall22 = false;
  for (int i = d.bf_ptr[p]; i < d.bf_ptr[p + 1]; i++) {
    const int ifa = d.bf_list[i];
    const int q0 = d.bfn[ifa], q1 = d.bfn[d.nbfac + ifa], code = d.bfcode[ifa];
    const double anx = d.ys[q1] - d.ys[q0];
    const double any = -(d.xs[q1] - d.xs[q0]);
    const double gf3 = sqrt(anx * anx + any * any);
    if (code / 1000 == 22) {
      wall22 = true;
      double bsnx = 0.0, bsny = 0.0;
      const int sub = code % 1000;
      if (sub == 221) {
        bsnx = 0.0 * gf3 * 0.5;
        bsny = -1.0 * gf3 * 0.5;
        if (d.ncase == 1 || d.ncase == 2 || d.ncase == 12) {
          if (d.ys[q0] < 1.0e-6 && d.ys[q1] < 1.0e-6) { bsnx = 0.0 * gf3 * 0.5; bsny = -1.0 * gf3 * 0.5; }
          else if (fabs(d.ys[q0] - 1.0) < 1.0e-6 && fabs(d.ys[q1] - 1.0) < 1.0e-6) { bsnx = 0.0 * gf3 * 0.5; bsny = 1.0 * gf3 * 0.5; }
        }
      } else if (sub == 222) {
        bsnx = -1.0 * gf3 * 0.5;
        bsny = 0.0 * gf3 * 0.5;
        if (d.ncase == 1) {
          if (d.xs[q0] < 1.0e-6 && d.xs[q1] < 1.0e-6) { bsnx = -1.0 * gf3 * 0.5; bsny = 0.0 * gf3 * 0.5; }
          else if (fabs(d.xs[q0] - 1.0) < 1.0e-6 && fabs(d.xs[q1] - 1.0) < 1.0e-6) { bsnx = 1.0 * gf3 * 0.5; bsny = 0.0 * gf3 * 0.5; }
        }
      }
      bvx = bvx + bsnx;
      bvy = bvy + bsny;
    } else if (code / 1000 == 21 && d.ncase == 3) {
      const double pres0 = 1.0e-6;
      const double bsnx = anx / gf3 * gf3 * 0.5, bsny = any / gf3 * gf3 * 0.5;
      bpx = bpx + pres0 * bsnx;
      bpy = bpy + pres0 * bsny;
    }
  }
  double fpx = 0.0, fpy = 0.0;
  if (wall22) {
    const double detma = n11 * n22 - n21 * n12;
    const double i11 = n22 / detma, i12 = -n12 / detma, i21 = -n21 / detma, i22 = n11 / detma;
    const double coefl = (i11 * bvx + i12 * bvy) * bvx + (i21 * bvx + i22 * bvy) * bvy;
    const double rhsx = a1 - s1 - bpx, rhsy = a2 - s2 - bpy;
    const double coefr = (i11 * rhsx + i12 * rhsy) * bvx + (i21 * rhsx + i22 * rhsy) * bvy;
    fpx = coefr / fmax(1.0e-16, coefl) * bvx;
    fpy = coefr / fmax(1.0e-16, coefl) * bvy;
  }
  fpx = fpx + bpx;
  fpy = fpy + bpy;
  const unsigned char bc = d.bc[p];
  double us = d.us[p], vs = d.vs[p];
  if (!(bc & BC_KEEP)) {
    const double detma = n11 * n22 - n21 * n12;
    const double i11 = n22 / detma, i12 = -n12 / detma, i21 = -n21 / detma, i22 = n11 / detma;
    const double r1 = a1 - s1 - fpx, r2 = a2 - s2 - fpy;
    us = i11 * r1 + i12 * r2;
    vs = i21 * r1 + i22 * r2;
  }
  if (bc & (BC_V0 | BC_UV0)) vs = 0.0;
  if (bc & (BC_U0 | BC_UV0)) us = 0.0;
  d.us[p] = us;
  d.vs[p] = vs;
}

template <bool FAST, int GEO>
__global__ void k1_node(Dev1 d) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.npoin || stopped(d)) return;
  if (GEO == 1) {
    rz_node(d, p);
    return;
  }
  if (GEO == 2) {
    aw_node(d, p);
    return;
  }
  double n11 = 0.0, n21 = 0.0, n12 = 0.0, n22 = 0.0, a1 = 0.0, a2 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int i = d.ncor_ptr[p]; i < d.ncor_ptr[p + 1]; i++) {
    const int c = d.ncor[i], iq = c >> 2, iv = c & 3;
    if (FAST) {
      const double m = d.cf[(0 * 4 + iv) * (size_t)d.nquad + iq];
      n11 = n11 + m;
      n22 = n22 + m;
      a1 = a1 + d.cf[(1 * 4 + iv) * (size_t)d.nquad + iq];
      a2 = a2 + d.cf[(2 * 4 + iv) * (size_t)d.nquad + iq];
      s1 = s1 + d.cf[(3 * 4 + iv) * (size_t)d.nquad + iq];
      s2 = s2 + d.cf[(4 * 4 + iv) * (size_t)d.nquad + iq];
      continue;
    }
#pragma unroll
    for (int f = 0; f < 2; f++) {
      const int slot = f + 2 * iv;
      const double m = d.cf[(0 * 8 + slot) * (size_t)d.nquad + iq];
      n11 = n11 + m;
      n21 = n21 + 0.0;
      n12 = n12 + 0.0;
      n22 = n22 + m;
      a1 = a1 + d.cf[(1 * 8 + slot) * (size_t)d.nquad + iq];
      a2 = a2 + d.cf[(2 * 8 + slot) * (size_t)d.nquad + iq];
      s1 = s1 + d.cf[(3 * 8 + slot) * (size_t)d.nquad + iq];
      s2 = s2 + d.cf[(4 * 8 + slot) * (size_t)d.nquad + iq];
    }
  }
  const unsigned char bc = d.bc[p];
  double us = d.us[p], vs = d.vs[p];
  if (!(bc & BC_KEEP)) {
    const double detma = n11 * n22 - n21 * n12;
    const double i11 = n22 / detma, i12 = -n12 / detma, i21 = -n21 / detma, i22 = n11 / detma;
    const double r1 = a1 - s1, r2 = a2 - s2;
    us = i11 * r1 + i12 * r2;
    vs = i21 * r1 + i22 * r2;
  }
  if (bc & (BC_V0 | BC_UV0)) vs = 0.0;
  if (bc & (BC_U0 | BC_UV0)) us = 0.0;
  d.us[p] = us;
  d.vs[p] = vs;
}

// ---------------------------------------------------------------------------
// Limited slopes into the stage state (Getrhslagmc.f90:7283-7298) and the
// stage update (Getrhslag.f90:1789-1904, npoly = 1)
// ---------------------------------------------------------------------------
__device__ void update_cell(const Dev1 &d, int e, double alfa, const double (*R)[4]) {
  const size_t nc = d.ncell;
  const double dt = d.sc_dev->dtfix;
  const double af1 = d.lim[0 * nc + e], af5 = d.lim[2 * nc + e];
  const double v11 = d.lim[3 * nc + e], v12 = d.lim[4 * nc + e], v21 = d.lim[5 * nc + e], v22 = d.lim[6 * nc + e];
  double s[4][ND];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int k = 0; k < ND; k++) s[q][k] = U(d, d.Us, k, q, e);
  s[0][1] = s[0][1] * af1;
  s[0][2] = s[0][2] * af1;
  {
    const double u22 = s[1][1], u32 = s[1][2], u23 = s[2][1], u33 = s[2][2];
    s[1][1] = v11 * u22 + v12 * u23;
    s[1][2] = v11 * u32 + v12 * u33;
    s[2][1] = v21 * u22 + v22 * u23;
    s[2][2] = v21 * u32 + v22 * u33;
  }
  s[3][1] = s[3][1] * af5;
  s[3][2] = s[3][2] * af5;
  double r[ND][4];
#pragma unroll
  for (int k = 0; k < ND; k++)
#pragma unroll
    for (int q = 0; q < 4; q++) r[k][q] = dt * R[k][q];
  const double a1 = d.amatr[0 * nc + e], a2 = d.amatr[1 * nc + e], a3 = d.amatr[2 * nc + e];
  const double a4 = d.amatr[3 * nc + e];
  const double mm[ND][ND] = {{a4, 0.0, 0.0}, {0.0, a1, a2}, {0.0, a2, a3}};
  const double oma = 1.0 - alfa;
#pragma unroll
  for (int id = 0; id < ND; id++) {
    double unint[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int iu = 0; iu < ND; iu++)
#pragma unroll
      for (int q = 0; q < 4; q++) unint[q] = unint[q] + mm[id][iu] * r[iu][q];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const size_t idx = (q * ND + id) * nc + e;
      d.Us[idx] = alfa * d.Un[idx] + oma * (s[q][id] + unint[q]);
    }
  }
}

__global__ void k1_update(Dev1 d, double alfa) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.ncell || stopped(d)) return;
  double R[ND][4];
#pragma unroll
  for (int k = 0; k < ND; k++)
#pragma unroll
    for (int q = 0; q < 4; q++) R[k][q] = d.rhs[(q * ND + k) * (size_t)d.ncell + e];
  update_cell(d, e, alfa, R);
}

// ---------------------------------------------------------------------------
// Corner forces, face and volume integrals of one quad
// ---------------------------------------------------------------------------
// RZ face integral (rhsifacedg_lagmc_quadrz, Getrhslagmc.f90:18534-18734):
// corner forces F = sigma.n A + m (u* - u_v) of the 16 corner faces; face f
// of vertex iv weighs the basis of its own vertex (f = 1, 2) or of the edge's
// other vertex (f = 3, 4), the mass flux with the radius weights rcapt
__device__ void rz_faces(const Dev1 &d, int iq, const double (*x4)[2], double rc, double sc, double (*R)[4]) {
  const double alfrz = d.alfrz, c05 = 0.5;
  double fn[4][3], rco[4], bq[4][ND];
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const int b = (f + 1) & 3;
    const double anx = x4[b][1] - x4[f][1];
    const double any = -(x4[b][0] - x4[f][0]);
    fn[f][0] = anx / sqrt(anx * anx + any * any);
    fn[f][1] = any / sqrt(anx * anx + any * any);
    fn[f][2] = sqrt(anx * anx + any * any);
    rco[f] = 1.0 - alfrz + alfrz * fabs(x4[f][1]);
    bq[f][0] = 1.0; bq[f][1] = (xv(f) - rc) / 1.0; bq[f][2] = (yv(f) - sc) / 1.0;
  }
#pragma unroll
  for (int k = 0; k < ND; k++)
#pragma unroll
    for (int q = 0; q < 4; q++) R[k][q] = 0.0;
#pragma unroll
  for (int iv = 0; iv < 4; iv++) {
    const int vp = (iv + 3) & 3, vx = (iv + 1) & 3;
    const int p = d.ipq[iv * d.nquad + iq];
    const double us = d.us[p], vs = d.vs[p];
#pragma unroll
    for (int f = 0; f < 4; f++) {
      const int edge = (f & 1) ? iv : vp;
      const int bv = (f < 2) ? iv : ((f == 2) ? vp : vx);
      const double rw = (f < 2) ? 3.0 * rco[iv] : 1.0 * rco[iv];
      const double rcapt = (rw + ((f & 1) ? rco[vx] : rco[vp])) / 6.0;
      const int slot = f + 4 * iv;
      const double m = d.cf[(0 * 16 + slot) * (size_t)d.nquad + iq];
      const double mu1 = d.cf[(1 * 16 + slot) * (size_t)d.nquad + iq];
      const double mu2 = d.cf[(2 * 16 + slot) * (size_t)d.nquad + iq];
      const double s1 = d.cf[(3 * 16 + slot) * (size_t)d.nquad + iq];
      const double s2 = d.cf[(4 * 16 + slot) * (size_t)d.nquad + iq];
      const double F0 = s1 + m * us + 0.0 * vs - mu1;
      const double F1 = s2 + 0.0 * us + m * vs - mu2;
#pragma unroll
      for (int k = 0; k < ND; k++) {
        const double lx = c05 * fn[edge][0] * fn[edge][2] * bq[bv][k];
        const double ly = c05 * fn[edge][1] * fn[edge][2] * bq[bv][k];
        const double bc = bq[bv][k];
        R[k][0] = R[k][0] + us * lx * rcapt + vs * ly * rcapt;
        R[k][1] = R[k][1] + F0 * bc;
        R[k][2] = R[k][2] + F1 * bc;
        R[k][3] = R[k][3] + us * F0 * bc + vs * F1 * bc;
      }
    }
  }
}

// Area-weighted RZ face integral (rhsifacedg_lagmc_quadrzaw, Getrhslagrz.f90:
// 1673-1812): corner forces F = sigma.n A + m (u* - u_v) of the two corner
// faces; face 1 of vertex iv (the edge to the previous vertex w) weighs
// (2 b_iv + b_w)/3, face 2 (to the next vertex) likewise
__device__ void aw_faces(const Dev1 &d, int iq, const double (*x4)[2], double rc, double sc, double (*R)[4]) {
  const double c16 = 0.1666666666666666, c13 = 0.3333333333333333;
  double fn[4][3], bq[4][ND];
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const int b = (f + 1) & 3;
    const double anx = x4[b][1] - x4[f][1];
    const double any = -(x4[b][0] - x4[f][0]);
    fn[f][0] = anx / sqrt(anx * anx + any * any);
    fn[f][1] = any / sqrt(anx * anx + any * any);
    fn[f][2] = sqrt(anx * anx + any * any);
    bq[f][0] = 1.0; bq[f][1] = (xv(f) - rc) / 1.0; bq[f][2] = (yv(f) - sc) / 1.0;
  }
#pragma unroll
  for (int k = 0; k < ND; k++)
#pragma unroll
    for (int q = 0; q < 4; q++) R[k][q] = 0.0;
#pragma unroll
  for (int iv = 0; iv < 4; iv++) {
    const int vp = (iv + 3) & 3, vx = (iv + 1) & 3;
    const int p = d.ipq[iv * d.nquad + iq];
    const double us = d.us[p], vs = d.vs[p];
    double F[2][2];
#pragma unroll
    for (int f = 0; f < 2; f++) {
      const int slot = f + 2 * iv;
      const double m = d.cf[(0 * 8 + slot) * (size_t)d.nquad + iq];
      const double mu1 = d.cf[(1 * 8 + slot) * (size_t)d.nquad + iq];
      const double mu2 = d.cf[(2 * 8 + slot) * (size_t)d.nquad + iq];
      const double s1 = d.cf[(3 * 8 + slot) * (size_t)d.nquad + iq];
      const double s2 = d.cf[(4 * 8 + slot) * (size_t)d.nquad + iq];
      F[f][0] = s1 + m * us + 0.0 * vs - mu1;
      F[f][1] = s2 + 0.0 * us + m * vs - mu2;
    }
#pragma unroll
    for (int k = 0; k < ND; k++) {
      const double wa = 2.0 * bq[iv][k] + bq[vp][k], wb = 2.0 * bq[iv][k] + bq[vx][k];
      const double l1x = c16 * wa * fn[vp][0] * fn[vp][2], l1y = c16 * wa * fn[vp][1] * fn[vp][2];
      const double l2x = c16 * wb * fn[iv][0] * fn[iv][2], l2y = c16 * wb * fn[iv][1] * fn[iv][2];
      R[k][0] = R[k][0] + us * l1x + vs * l1y + us * l2x + vs * l2y;
      R[k][1] = R[k][1] + F[0][0] * c13 * wa + F[1][0] * c13 * wb;
      R[k][2] = R[k][2] + F[0][1] * c13 * wa + F[1][1] * c13 * wb;
      R[k][3] = R[k][3] + us * F[0][0] * c13 * wa + vs * F[0][1] * c13 * wa + us * F[1][0] * c13 * wb +
                vs * F[1][1] * c13 * wb;
    }
  }
}

template <int MD, bool FAST, int GEO>
__global__ void __launch_bounds__(128) k1_rhs(Dev1 d, int fuse, double alfa) {
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  if (iq >= d.nquad || stopped(d)) return;
  const int e = iq;
  const double g = d.gamlg, epsd = 1.0e-6;
  const size_t nc = d.ncell;
  double x4[4][2];
  load4(d, d.xs, d.ys, iq, x4);
  const double rc = d.rc[e], sc = d.sc[e];
  double u[4][ND];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int k = 0; k < ND; k++) u[q][k] = U(d, d.Us, k, q, e);
  double fn[4][3];
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const int b = (f + 1) & 3;
    const double anx = x4[b][1] - x4[f][1];
    const double any = -(x4[b][0] - x4[f][0]);
    fn[f][0] = anx / sqrt(anx * anx + any * any);
    fn[f][1] = any / sqrt(anx * anx + any * any);
    fn[f][2] = sqrt(anx * anx + any * any);
  }
  // face integral (rhsifacedg_lag_mc_hybridquad2)
  const double c16 = 0.1666666666666666, c13 = 0.3333333333333333;
  double R[ND][4];
#pragma unroll
  for (int k = 0; k < ND; k++)
#pragma unroll
    for (int q = 0; q < 4; q++) R[k][q] = 0.0;
  if (GEO == 1) {
    rz_faces(d, iq, x4, rc, sc, R);
  } else if (GEO == 2) {
    aw_faces(d, iq, x4, rc, sc, R);
  } else {
#pragma unroll
    for (int iv = 0; iv < 4; iv++) {
      const int p = d.ipq[iv * d.nquad + iq];
      const double us = d.us[p], vs = d.vs[p];
      // fstarq (Limiterlag.f90:686-698): sigma.n A + mu A (u* - u_v)
      double F[2][2];
      if (FAST) {
        // the corner's two faces summed: F = sum sigma.n A + (sum mu A) u* - sum mu A u_v
        const double m = d.cf[(0 * 4 + iv) * (size_t)d.nquad + iq];
        F[0][0] = d.cf[(3 * 4 + iv) * (size_t)d.nquad + iq] + m * us - d.cf[(1 * 4 + iv) * (size_t)d.nquad + iq];
        F[0][1] = d.cf[(4 * 4 + iv) * (size_t)d.nquad + iq] + m * vs - d.cf[(2 * 4 + iv) * (size_t)d.nquad + iq];
        F[1][0] = 0.0;
        F[1][1] = 0.0;
      }
#pragma unroll
      for (int f = 0; f < (FAST ? 0 : 2); f++) {
        const int slot = f + 2 * iv;
        const double m = d.cf[(0 * 8 + slot) * (size_t)d.nquad + iq];
        const double mu1 = d.cf[(1 * 8 + slot) * (size_t)d.nquad + iq];
        const double mu2 = d.cf[(2 * 8 + slot) * (size_t)d.nquad + iq];
        const double s1 = d.cf[(3 * 8 + slot) * (size_t)d.nquad + iq];
        const double s2 = d.cf[(4 * 8 + slot) * (size_t)d.nquad + iq];
        F[f][0] = s1 + m * us + 0.0 * vs - mu1;
        F[f][1] = s2 + 0.0 * us + m * vs - mu2;
      }
      const int fa = (iv + 3) & 3, fb = iv;
      const double bqv[ND] = {1.0, (xv(iv) - rc) / 1.0, (yv(iv) - sc) / 1.0};
#pragma unroll
      for (int k = 0; k < ND; k++) {
        const double b3 = 2.0 * bqv[k] + bqv[k];
        const double l1x = c16 * b3 * fn[fa][0] * fn[fa][2], l1y = c16 * b3 * fn[fa][1] * fn[fa][2];
        const double l2x = c16 * b3 * fn[fb][0] * fn[fb][2], l2y = c16 * b3 * fn[fb][1] * fn[fb][2];
        if (FAST) {
          const double w = c13 * b3;
          R[k][0] = R[k][0] + us * (l1x + l2x) + vs * (l1y + l2y);
          R[k][1] = R[k][1] + F[0][0] * w;
          R[k][2] = R[k][2] + F[0][1] * w;
          R[k][3] = R[k][3] + (us * F[0][0] + vs * F[0][1]) * w;
          continue;
        }
        R[k][0] = R[k][0] + us * l1x + vs * l1y + us * l2x + vs * l2y;
        R[k][1] = R[k][1] + F[0][0] * c13 * b3 + F[1][0] * c13 * b3;
        R[k][2] = R[k][2] + F[0][1] * c13 * b3 + F[1][1] * c13 * b3;
        R[k][3] = R[k][3] + us * F[0][0] * c13 * b3 + vs * F[0][1] * c13 * b3 + us * F[1][0] * c13 * b3 +
                  vs * F[1][1] * c13 * b3;
      }
    }
  }
  // volume integral (rhsdomndg_lag_mc_quadsym, 5x5 Gauss)
  const double af4 = d.lim[1 * nc + e];
  const double v11 = d.lim[3 * nc + e], v12 = d.lim[4 * nc + e], v21 = d.lim[5 * nc + e], v22 = d.lim[6 * nc + e];
  const double rhomc = u[0][0], uctr = u[1][0], vctr = u[2][0], ectr = u[3][0];
  const double rhoct = 1.0 / rhomc;
  const double pctr = fmax(epsd, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
  const double dudr = v11 * u[1][1] + v12 * u[2][1];
  const double duds = v11 * u[1][2] + v12 * u[2][2];
  const double dvdr = v21 * u[1][1] + v22 * u[2][1];
  const double dvds = v21 * u[1][2] + v22 * u[2][2];
  for (int ig = 0; ig < 25; ig++) {
    const double r = cR.g25[ig][0], s = cR.g25[ig][1], wi = cR.w25[ig];
    double dxdr, dxds, dydr, dyds;
    jac4(x4, r, s, dxdr, dxds, dydr, dyds);
    const double djaco = wi;
    // rcoef = 1 - alfrz + alfrz * ygaus (Limiterlag.f90:1268-1279): 1 in plane geometry
    double rcoef = 1.0;
    if (GEO == 1) {
      const double rp = 1.0 + r, rm = 1.0 - r, sp = 1.0 + s, sm = 1.0 - s;
      const double shpq[4] = {0.25 * rm * sm, 0.25 * rp * sm, 0.25 * rp * sp, 0.25 * rm * sp};
      double ygaus = 0.0;
#pragma unroll
      for (int k = 0; k < 4; k++) ygaus = ygaus + shpq[k] * x4[k][1];
      rcoef = 1.0 - d.alfrz + d.alfrz * ygaus;
    }
    // gdshp = adj(J) grad_xi b, b = (1, r - rc, s - sc): the rows for b2, b3
    const double g1[ND] = {dyds * 0.0 + (-dydr) * 0.0, dyds * 1.0 + (-dydr) * 0.0, dyds * 0.0 + (-dydr) * 1.0};
    const double g2[ND] = {(-dxds) * 0.0 + dxdr * 0.0, (-dxds) * 1.0 + dxdr * 0.0, (-dxds) * 0.0 + dxdr * 1.0};
    const double b1 = (r - rc) / 1.0, b2 = (s - sc) / 1.0;
    double un[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const double bb[ND] = {1.0, b1, b2};
      double a = 0.0;
#pragma unroll
      for (int k = 0; k < MD; k++) a = a + u[q][k] * bb[k];
      un[q] = a;
    }
    const double rhoad = 1.0 / un[0];
    double pres = (g - 1.0) * rhoad * (un[3] - 0.5 * (un[1] * un[1] + un[2] * un[2]));
    const double uadv = uctr + dudr * b1 + duds * b2;
    const double vadv = vctr + dvdr * b1 + dvds * b2;
    pres = pctr + af4 * (pres - pctr);
    if (GEO == 2) {
      // rhsdomndg_lagmc_quadrzaw (Getrhslagrz.f90:2243-2555): the plane
      // fluxes written without the stress tensor, no radius weight
#pragma unroll
      for (int k = 0; k < ND; k++) {
        const double f1 = g1[k] * uadv + g2[k] * vadv;
        const double f2 = g1[k] * (-pres);
        const double f3 = g2[k] * (-pres);
        const double f4 = (g1[k] * uadv + g2[k] * vadv) * (-pres);
        R[k][0] = R[k][0] - f1 * djaco;
        R[k][1] = R[k][1] - f2 * djaco;
        R[k][2] = R[k][2] - f3 * djaco;
        R[k][3] = R[k][3] - f4 * djaco;
      }
      continue;
    }
    const double s11 = -pres + 0.0, s12 = 0.0 + 0.0, s21 = 0.0 + 0.0, s22 = -pres + 0.0;
#pragma unroll
    for (int k = 0; k < ND; k++) {
      const double f1 = g1[k] * uadv + g2[k] * vadv;
      const double f2 = g1[k] * s11 + g2[k] * s12;
      const double f3 = g1[k] * s21 + g2[k] * s22;
      const double f4 = g1[k] * (s11 * uadv + s12 * vadv) + g2[k] * (s21 * uadv + s22 * vadv);
      R[k][0] = R[k][0] - f1 * djaco * rcoef;
      R[k][1] = R[k][1] - f2 * djaco * rcoef;
      R[k][2] = R[k][2] - f3 * djaco * rcoef;
      R[k][3] = R[k][3] - f4 * djaco * rcoef;
    }
  }
  if (GEO == 2) {
    // nrz = 2 (Getrhslagmc.f90:6961-6973): the right-hand side times the
    // cell-averaged radius geoel(11), then rhsdomnsrcdg_lagmc_quadrzaw
    // (Getrhslagrz.f90:2818-3096): 5x5 Gauss over the area, v of the cell
    // average times b into the specific volume, -p v b (the limited
    // pressure of the point) into the energy
    const double rb = d.rbar[e];
#pragma unroll
    for (int k = 0; k < ND; k++)
#pragma unroll
      for (int q = 0; q < 4; q++) R[k][q] = rb * R[k][q];
    for (int ig = 0; ig < 25; ig++) {
      const double r = cR.g25[ig][0], s = cR.g25[ig][1], wi = cR.w25[ig];
      double dxdr, dxds, dydr, dyds;
      jac4(x4, r, s, dxdr, dxds, dydr, dyds);
      const double djaco = wi * (dxdr * dyds - dxds * dydr);
      const double bb[ND] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
      double un[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        double a = 0.0;
#pragma unroll
        for (int k = 0; k < MD; k++) a = a + u[q][k] * bb[k];
        un[q] = a;
      }
      const double rhoad = 1.0 / un[0];
      double pres = (g - 1.0) * rhoad * (un[3] - 0.5 * (un[1] * un[1] + un[2] * un[2]));
      pres = pctr + af4 * (pres - pctr);
#pragma unroll
      for (int k = 0; k < ND; k++) {
        R[k][0] = R[k][0] + vctr * bb[k] * djaco;
        R[k][3] = R[k][3] + vctr * (-pres) * bb[k] * djaco;
      }
    }
  }
  if (GEO == 1) {
    // RZ hoop-stress source of the radial (y) momentum
    // (rhsdomnsrcdg_lagmc_quadrz, Getrhslagmc.f90:15800-16048): 5x5 Gauss,
    // the limited pressure of the point, no radius weight
    for (int ig = 0; ig < 25; ig++) {
      const double r = cR.g25[ig][0], s = cR.g25[ig][1], wi = cR.w25[ig];
      double dxdr, dxds, dydr, dyds;
      jac4(x4, r, s, dxdr, dxds, dydr, dyds);
      const double djaco = wi * (dxdr * dyds - dydr * dxds);
      const double bb[ND] = {1.0, (r - rc) / 1.0, (s - sc) / 1.0};
      double un[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        double a = 0.0;
#pragma unroll
        for (int k = 0; k < MD; k++) a = a + u[q][k] * bb[k];
        un[q] = a;
      }
      const double rhoad = 1.0 / un[0];
      double pres = (g - 1.0) * rhoad * (un[3] - 0.5 * (un[1] * un[1] + un[2] * un[2]));
      pres = pctr + af4 * (pres - pctr);
#pragma unroll
      for (int k = 0; k < ND; k++) {
        const double f3 = d.alfrz * (-pres) * bb[k];
        R[k][2] = R[k][2] - f3 * djaco;
      }
    }
  }
  if (!fuse) {
#pragma unroll
    for (int k = 0; k < ND; k++)
#pragma unroll
      for (int q = 0; q < 4; q++) d.rhs[(q * ND + k) * nc + e] = R[k][q];
    return;
  }
  update_cell(d, e, alfa, R);
}

// ---------------------------------------------------------------------------
// getdelt_lag (Getrhslag.f90:20600-20716, straight edges :20649-20654)
// ---------------------------------------------------------------------------
__global__ void k1_dt_partial(Dev1 d) {
  __shared__ double sm_cfl[256], sm_vol[256];
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  double dtcfl = 1e10, dtvol = 1e10;
  if (iq < d.nquad && !stopped(d)) {
    const double eps = 1.0e-6, g = d.gamlg;
    double x4[4][2];
    load4(d, d.xn, d.yn, iq, x4);
    double dlen = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int b = (k + 1) & 3;
      const double dl = sqrt((x4[k][0] - x4[b][0]) * (x4[k][0] - x4[b][0]) + (x4[k][1] - x4[b][1]) * (x4[k][1] - x4[b][1]));
      if (k == 0 || dl < dlen) dlen = dl;
    }
    const double rhomc = U(d, d.Us, 0, 0, iq);
    const double uctr = U(d, d.Us, 0, 1, iq), vctr = U(d, d.Us, 0, 2, iq), ectr = U(d, d.Us, 0, 3, iq);
    const double rhoct = 1.0 / rhomc;
    const double pctr = fmax(eps, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
    const double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
    dtcfl = dlen / sdctr;
    dtvol = d.vol[iq] / fabs(d.rhs[0 * (size_t)d.ncell + iq]);
  }
  sm_cfl[threadIdx.x] = dtcfl;
  sm_vol[threadIdx.x] = dtvol;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sm_cfl[threadIdx.x] = fmin(sm_cfl[threadIdx.x], sm_cfl[threadIdx.x + s]);
      sm_vol[threadIdx.x] = fmin(sm_vol[threadIdx.x], sm_vol[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    d.dtpart[2 * blockIdx.x] = sm_cfl[0];
    d.dtpart[2 * blockIdx.x + 1] = sm_vol[0];
  }
}

__global__ void k1_dt_final(Dev1 d, int nblk, int ndt) {
  __shared__ double sm_cfl[256], sm_vol[256];
  if (stopped(d)) return;
  double a = 1e10, b = 1e10;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    a = fmin(a, d.dtpart[2 * i]);
    b = fmin(b, d.dtpart[2 * i + 1]);
  }
  sm_cfl[threadIdx.x] = a;
  sm_vol[threadIdx.x] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sm_cfl[threadIdx.x] = fmin(sm_cfl[threadIdx.x], sm_cfl[threadIdx.x + s]);
      sm_vol[threadIdx.x] = fmin(sm_vol[threadIdx.x], sm_vol[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    Scalars *S = d.sc_dev;
    double dt = S->dtfix;
    if (ndt == 1) {
      const double dtcfl = fmin(1e10, sm_cfl[0]), dtvol = fmin(1e10, sm_vol[0]);
      if (S->itime == 1) dt = fmin(d.cfl * dtcfl, 0.1 * dtvol);
      else dt = fmin(fmin(d.cfl * dtcfl, 0.1 * dtvol), 1.01 * dt);
      if ((S->tacru + dt) > d.tend) dt = d.tend - S->tacru;
    }
    S->dtfix = dt;
    S->tacru = S->tacru + dt;
  }
}

// node motion (Getrhslag.f90:1948-1957); no centre node on straight quads
__global__ void k1_nodes(Dev1 d, double alfa) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.npoin || stopped(d)) return;
  const double dt = d.sc_dev->dtfix, oma = 1.0 - alfa;
  d.xs[p] = alfa * d.xn[p] + oma * (d.xs[p] + dt * d.us[p]);
  d.ys[p] = alfa * d.yn[p] + oma * (d.ys[p] + dt * d.vs[p]);
}

// driver copy-back (dgflo2d.f90:407-423)
__global__ void k1_copyback(Dev1 d) {
  if (stopped(d)) return;
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < NU1 * d.ncell; t += stride) d.Un[t] = d.Us[t];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < d.npoin; t += stride) {
    d.xn[t] = d.xs[t];
    d.yn[t] = d.ys[t];
  }
}

__global__ void k1_step_begin(Dev1 d, int itime) {
  Scalars *S = d.sc_dev;
  if (S->done) return;
  S->itime = (itime < 0) ? S->itime + 1 : itime;
}

__global__ void k1_step_end(Dev1 d) {
  Scalars *S = d.sc_dev;
  if (S->done) return;
  if (fabs(S->tacru - d.tend) / d.tend <= 1e-11) S->done = 1;
}

// caller layout unkno(3, 4, ncell) <-> device slabs
__global__ void k1_unkno_in(Dev1 d, const double *aos) {
  const int n = NU1 * d.ncell;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int e = t / NU1, qk = t % NU1;
    d.Un[qk * (size_t)d.ncell + e] = aos[t];
    d.Us[qk * (size_t)d.ncell + e] = aos[t];
  }
}
__global__ void k1_unkno_out(Dev1 d, const double *src, double *aos) {
  const int n = NU1 * d.ncell;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int e = t / NU1, qk = t % NU1;
    aos[t] = src[qk * (size_t)d.ncell + e];
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct Family { double ms = 0.0; long long n = 0; };

// Per-cell output values of the end-of-run post-processing of the linear
// path (geterror_lag_hybrid, Postprocess.f90:3515-3560, written to its radial
// profile file): out[k*ncell + e] for k = 0..8 = (radius of the centre, rho,
// p, e_int, x_c, y_c, |u|, u, v) from the cell averages of U^n, the centre
// being the bilinear map at (r, s) = (0, 0).
__global__ void k1_cell_output(Dev1 d, double *out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.nquad) return;
  double x4[4][2];
  load4(d, d.xn, d.yn, e, x4);
  double xc = 0.0, yc = 0.0;
  for (int k = 0; k < 4; k++) {
    xc = xc + 0.25 * x4[k][0];
    yc = yc + 0.25 * x4[k][1];
  }
  const double g = d.gamlg;
  const double rhoc = 1.0 / U(d, d.Un, 0, 0, e);
  const double uctr = U(d, d.Un, 0, 1, e), vctr = U(d, d.Un, 0, 2, e), ectr = U(d, d.Un, 0, 3, e);
  const double pctr = (g - 1.0) * rhoc * (ectr - 0.5 * (uctr * uctr + vctr * vctr));
  const size_t n = d.ncell;
  out[0 * n + e] = sqrt(xc * xc + yc * yc);
  out[1 * n + e] = rhoc;
  out[2 * n + e] = pctr;
  out[3 * n + e] = pctr / rhoc / (g - 1.0);
  out[4 * n + e] = xc;
  out[5 * n + e] = yc;
  out[6 * n + e] = sqrt(uctr * uctr + vctr * vctr);
  out[7 * n + e] = uctr;
  out[8 * n + e] = vctr;
}

struct Solver {
  Dev1 d{};
  lag2d_config cfg{};
  cudaStream_t st = nullptr;
  std::vector<void *> allocs;
  double *stage_u = nullptr, *stage_x = nullptr, *cellout = nullptr;
  cudaGraphExec_t graph = nullptr;
  long long graph_launches = 0, launches = 0;
  bool timing = false;
  std::map<std::string, Family> fam;
  std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
};

static int nb(int n, int t) { return std::max(1, (n + t - 1) / t); }

template <typename T>
static bool dalloc(Solver *s, T **p, size_t n) {
  void *q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return false;
  cudaMemsetAsync(q, 0, std::max<size_t>(n, 1) * sizeof(T), s->st);
  s->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return true;
}

template <typename F>
static void launch(Solver *s, const char *family, F &&f, int n = 1) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (s->timing) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s->st);
  }
  f();
  s->launches += n;
  if (s->timing) {
    cudaEventRecord(b, s->st);
    s->pending.push_back({family, {a, b}});
  }
}

static void flush_timing(Solver *s) {
  for (auto &p : s->pending) {
    cudaEventSynchronize(p.second.second);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.second.first, p.second.second);
    Family &f = s->fam[p.first];
    f.ms += ms;
    f.n += 1;
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  s->pending.clear();
}

#define CK1(call)                                                          \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);            \
      return LAG2D_ECUDA;                                                  \
    }                                                                      \
  } while (0)

static const double kRK[2][3] = {{0.0, 0.5, 0.0}, {0.0, 0.75, 0.3333333333333333}};

static void geom(Solver *s, const double *X, const double *Y) {
  const Dev1 &d = s->d;
  launch(s, "geom", [&] {
    // the closed form is the plane area; RZ volumes carry the radius weight
    if (s->cfg.order_exact || d.nrz) k1_geom<<<nb(d.nquad, 128), 128, 0, s->st>>>(d, X, Y);
    else k1_geom_fast<<<nb(d.nquad, 128), 128, 0, s->st>>>(d, X, Y);
  });
}

// RZ runs its own instantiations (in the reference's order: the RZ branch
// has no optimised variant), so the plane kernels keep their registers
template <int GEO, bool FAST>
static void launch_cell_g(const Dev1 &d, dim3 g, dim3 b, cudaStream_t st, int stage) {
  if (d.mdegr == 3) k1_cell<3, FAST, GEO><<<g, b, 0, st>>>(d, stage);
  else if (d.mdegr == 2) k1_cell<2, FAST, GEO><<<g, b, 0, st>>>(d, stage);
  else k1_cell<1, FAST, GEO><<<g, b, 0, st>>>(d, stage);
}
template <bool FAST>
static void launch_cell(const Dev1 &d, dim3 g, dim3 b, cudaStream_t st, int stage) {
  if (d.nrz == 1) launch_cell_g<1, false>(d, g, b, st, stage);
  else if (d.nrz == 2) launch_cell_g<2, false>(d, g, b, st, stage);
  else launch_cell_g<0, FAST>(d, g, b, st, stage);
}
template <int GEO, bool FAST>
static void launch_rhs_g(const Dev1 &d, dim3 g, dim3 b, cudaStream_t st, int fuse, double alfa) {
  if (d.mdegr == 3) k1_rhs<3, FAST, GEO><<<g, b, 0, st>>>(d, fuse, alfa);
  else if (d.mdegr == 2) k1_rhs<2, FAST, GEO><<<g, b, 0, st>>>(d, fuse, alfa);
  else k1_rhs<1, FAST, GEO><<<g, b, 0, st>>>(d, fuse, alfa);
}
template <bool FAST>
static void launch_rhs(const Dev1 &d, dim3 g, dim3 b, cudaStream_t st, int fuse, double alfa) {
  if (d.nrz == 1) launch_rhs_g<1, false>(d, g, b, st, fuse, alfa);
  else if (d.nrz == 2) launch_rhs_g<2, false>(d, g, b, st, fuse, alfa);
  else launch_rhs_g<0, FAST>(d, g, b, st, fuse, alfa);
}

// the stage sequence of getrhsdg_lag_mcnew's linear branch
static void enqueue_rhs(Solver *s, int fuse, double alfa, int stage) {
  const Dev1 &d = s->d;
  launch(s, "bounds", [&] { k1_bounds<<<nb(d.npoin, 256), 256, 0, s->st>>>(d); });
  const dim3 gq(nb(d.nquad, 128)), bq(128), gp(nb(d.npoin, 256)), bp(256);
  const bool ex = s->cfg.order_exact != 0;
  launch(s, "cell", [&] {
    ex ? launch_cell<false>(d, gq, bq, s->st, stage) : launch_cell<true>(d, gq, bq, s->st, stage);
  });
  launch(s, "node", [&] {
    if (d.nrz == 1) k1_node<false, 1><<<gp, bp, 0, s->st>>>(d);
    else if (d.nrz == 2) k1_node<false, 2><<<gp, bp, 0, s->st>>>(d);
    else if (ex) k1_node<false, 0><<<gp, bp, 0, s->st>>>(d);
    else k1_node<true, 0><<<gp, bp, 0, s->st>>>(d);
  });
  launch(s, "rhs", [&] {
    ex ? launch_rhs<false>(d, gq, bq, s->st, fuse, alfa) : launch_rhs<true>(d, gq, bq, s->st, fuse, alfa);
  });
}

// getsolvdg_lag (Getrhslag.f90:1553-2035) and the driver copy-back.  On
// this branch the cell volume is read only by getdelt_lag in the first stage,
// so of the reference's getcellvol_lag calls (at the start of the step and
// after every stage) only the one after the last stage is made: it is the
// start-of-step volume of the next step (same coordinates, same arithmetic),
// and set_state / init_fields compute it for the first step.  Area-weighted
// RZ (nrz = 2) reads geoel(11) in every stage, so there it follows each
// stage.
static void enqueue_step(Solver *s, int itime) {
  const Dev1 &d = s->d;
  const int ns = s->cfg.nstag;
  launch(s, "copy", [&] { k1_step_begin<<<1, 1, 0, s->st>>>(d, itime); });
  for (int istag = 1; istag <= ns; istag++) {
    const double alfa = kRK[ns - 2][istag - 1];
    if (istag == 1) {
      enqueue_rhs(s, 0, 0.0, 1);
      const int nblk = nb(d.nquad, 256);
      launch(s, "dt", [&] {
        k1_dt_partial<<<nblk, 256, 0, s->st>>>(d);
        k1_dt_final<<<1, 256, 0, s->st>>>(d, nblk, s->cfg.ndt);
      }, 2);
      launch(s, "update", [&] { k1_update<<<nb(d.ncell, 128), 128, 0, s->st>>>(d, alfa); });
    } else {
      enqueue_rhs(s, 1, alfa, istag);
    }
    launch(s, "nodes", [&] { k1_nodes<<<nb(d.npoin, 256), 256, 0, s->st>>>(d, alfa); });
    if (istag == ns || d.nrz == 2) geom(s, d.xs, d.ys);
  }
  launch(s, "copy", [&] {
    k1_copyback<<<nb(std::max(NU1 * d.ncell, d.npoin), 256), 256, 0, s->st>>>(d);
    k1_step_end<<<1, 1, 0, s->st>>>(d);
  }, 2);
}

static int read_status(Solver *s, std::string &err) {
  Scalars sc;
  CK1(cudaMemcpyAsync(&sc, s->d.sc_dev, sizeof(Scalars), cudaMemcpyDeviceToHost, s->st));
  CK1(cudaStreamSynchronize(s->st));
  CK1(cudaGetLastError());
  if (sc.status & ST_NONPHYS) { err = "non-positive cell volume"; return LAG2D_ENONPHYS; }
  return LAG2D_OK;
}

static int put_scalars(Solver *s, int itime, double dtfix, double tacru, std::string &err) {
  Scalars sc{};
  sc.dtfix = dtfix; sc.tacru = tacru; sc.itime = itime;
  CK1(cudaMemcpyAsync(s->d.sc_dev, &sc, sizeof(Scalars), cudaMemcpyHostToDevice, s->st));
  CK1(cudaStreamSynchronize(s->st));
  return LAG2D_OK;
}

int create(const lag2d_mesh *m, const lag2d_config *c, cudaStream_t st, Solver **out, std::string &err) {
  *out = nullptr;
  const int nq = m->nquad, np = m->npoin;
  for (size_t i = 0; i < 4 * (size_t)nq; i++)
    if (m->ipqua[i] < 1 || m->ipqua[i] > np) { err = "ipqua node id out of range"; return LAG2D_EINVAL; }
  for (int i = 0; i < m->nbfac; i++) {
    const int *b = m->bface + 5 * (size_t)i;
    if (b[0] < 1 || b[0] > np || b[1] < 1 || b[1] > np) { err = "bface node id out of range"; return LAG2D_EINVAL; }
  }
  const int nsu = m->esuv2[np];
  for (int i = 0; i < nsu; i++)
    if (m->esuv1[i] < 1 || m->esuv1[i] > nq) { err = "esuv1 cell id out of range"; return LAG2D_EINVAL; }
  if (c->nrz < 0 || c->nrz > 2) { err = "nrz must be 0, 1 or 2"; return LAG2D_EINVAL; }
  if (c->nrz != 0 && c->ncase == 7) {
    err = "RZ Sedov runs a hard-coded dt schedule (Getrhslag.f90:1673-1693) that is not built";
    return LAG2D_EUNSUP;
  }
  Solver *s = new Solver();
  s->cfg = *c;
  s->st = st;
  Dev1 &d = s->d;
  d.nquad = nq; d.npoin = np; d.ncell = nq; d.mdegr = c->mdegr; d.ncase = c->ncase;
  d.nsedov = c->nsedov;
  for (int i = 0; i < 4; i++) d.sedov_cell[i] = c->sedov_cell[i];
  d.gamlg = c->gamlg; d.cfl = c->cfl; d.cimpd = c->cimpd; d.tend = c->tend; d.sedov_energy = c->sedov_energy;
  d.nrz = c->nrz; d.alfrz = c->nrz ? 1.0 : 0.0; d.nbfac = m->nbfac;
  // connectivity
  std::vector<int> ipq(4 * (size_t)nq), eptr(np + 1), esv(nsu), cptr(np + 1, 0), cor(4 * (size_t)nq);
  for (int iq = 0; iq < nq; iq++)
    for (int k = 0; k < 4; k++) ipq[k * (size_t)nq + iq] = m->ipqua[4 * (size_t)iq + k] - 1;
  for (int p = 0; p <= np; p++) eptr[p] = m->esuv2[p];
  for (int i = 0; i < nsu; i++) esv[i] = m->esuv1[i] - 1;
  // corners at each node in the order getriem_quad_matrixsym scatters them
  for (int iq = 0; iq < nq; iq++)
    for (int k = 0; k < 4; k++) cptr[ipq[k * (size_t)nq + iq] + 1]++;
  for (int p = 0; p < np; p++) cptr[p + 1] += cptr[p];
  {
    std::vector<int> fill(cptr.begin(), cptr.end() - 1);
    for (int iq = 0; iq < nq; iq++)
      for (int k = 0; k < 4; k++) cor[fill[ipq[k * (size_t)nq + iq]]++] = iq * 4 + k;
  }
  // wall conditions of the nodal solve (Limiterlag.f90:462-476, 617-642) and
  // the limiter's wall classes (Limiterlag.f90:8197-8234)
  std::vector<unsigned char> bc(np, 0), wall(np, 0);
  for (int i = 0; i < m->nbfac; i++) {
    const int *b = m->bface + 5 * (size_t)i;
    for (int k = 0; k < 2; k++) {
      const int p = b[k] - 1;
      if (b[2] == 22 && b[3] == 221) bc[p] |= BC_V0;
      else if (b[2] == 22 && b[3] == 222) bc[p] |= BC_U0;
      else if (b[2] == 25) bc[p] |= BC_UV0 | BC_KEEP;
      if (c->ncase == 2) bc[p] |= BC_KEEP;
    }
  }
  for (int i = 0; i < m->nbfac; i++) {
    const int *b = m->bface + 5 * (size_t)i;
    if (b[2] == 22 && b[3] == 221)
      for (int k = 0; k < 2; k++) wall[b[k] - 1] = 3;
  }
  for (int i = 0; i < m->nbfac; i++) {
    const int *b = m->bface + 5 * (size_t)i;
    if (b[2] == 22 && b[3] == 222)
      for (int k = 0; k < 2; k++) wall[b[k] - 1] = (wall[b[k] - 1] == 3) ? 10 : 2;
  }
  // RZ: each node's boundary faces in face order, the faces' end nodes and
  // codes (getbc_lagmaire2 loops over the boundary faces)
  const int nbf = m->nbfac;
  std::vector<int> bptr(np + 1, 0), blist, bfn(2 * (size_t)std::max(nbf, 1)), bfcode(std::max(nbf, 1));
  for (int i = 0; i < nbf; i++) {
    const int *b = m->bface + 5 * (size_t)i;
    bfn[i] = b[0] - 1;
    bfn[nbf + i] = b[1] - 1;
    bfcode[i] = b[2] * 1000 + b[3];
    bptr[b[0]]++;
    if (b[1] != b[0]) bptr[b[1]]++;
  }
  for (int p = 0; p < np; p++) bptr[p + 1] += bptr[p];
  blist.resize(std::max(bptr[np], 1));
  {
    std::vector<int> fill(bptr.begin(), bptr.end() - 1);
    for (int i = 0; i < nbf; i++) {
      const int *b = m->bface + 5 * (size_t)i;
      blist[fill[b[0] - 1]++] = i;
      if (b[1] != b[0]) blist[fill[b[1] - 1]++] = i;
    }
  }
  int *ipq_d, *eptr_d, *esv_d, *cptr_d, *cor_d, *bptr_d, *blist_d, *bfn_d, *bfcode_d;
  unsigned char *bc_d, *wall_d;
  double *x0, *y0;
  bool ok = dalloc(s, &ipq_d, ipq.size()) && dalloc(s, &eptr_d, eptr.size()) && dalloc(s, &esv_d, esv.size()) &&
            dalloc(s, &cptr_d, cptr.size()) && dalloc(s, &cor_d, cor.size()) && dalloc(s, &bc_d, bc.size()) &&
            dalloc(s, &wall_d, wall.size()) && dalloc(s, &x0, np) && dalloc(s, &y0, np) &&
            dalloc(s, &bptr_d, bptr.size()) && dalloc(s, &blist_d, blist.size()) && dalloc(s, &bfn_d, bfn.size()) &&
            dalloc(s, &bfcode_d, bfcode.size());
  const size_t ncl = nq;
  ok = ok && dalloc(s, &d.rc, ncl) && dalloc(s, &d.sc, ncl) && dalloc(s, &d.vol, ncl) && dalloc(s, &d.vcx, ncl) &&
       dalloc(s, &d.vcy, ncl) && dalloc(s, &d.mass, ncl) && dalloc(s, &d.amatr, 4 * ncl) &&
       dalloc(s, &d.Un, NU1 * ncl) && dalloc(s, &d.Us, NU1 * ncl) && dalloc(s, &d.xn, np) && dalloc(s, &d.yn, np) &&
       dalloc(s, &d.xs, np) && dalloc(s, &d.ys, np) && dalloc(s, &d.us, np) && dalloc(s, &d.vs, np) &&
       dalloc(s, &d.bmax, 5 * (size_t)np) && dalloc(s, &d.bmin, 5 * (size_t)np) && dalloc(s, &d.lim, 7 * ncl) &&
       dalloc(s, &d.cf, (c->nrz == 1 ? 80 : 40) * ncl) && dalloc(s, &d.rhs, NU1 * ncl) && dalloc(s, &d.rbar, ncl) &&
       dalloc(s, &d.dtpart, 2 * (size_t)nb(nq, 256)) && dalloc(s, &d.sc_dev, 1) &&
       dalloc(s, &s->stage_u, NU1 * ncl) && dalloc(s, &s->stage_x, 2 * (size_t)np);
  if (!ok) {
    destroy(s);
    err = "cudaMalloc failed";
    return LAG2D_ECUDA;
  }
  d.ipq = ipq_d; d.esuv_ptr = eptr_d; d.esuv = esv_d; d.ncor_ptr = cptr_d; d.ncor = cor_d; d.bc = bc_d;
  d.wall = wall_d; d.x0 = x0; d.y0 = y0;
  d.bf_ptr = bptr_d; d.bf_list = blist_d; d.bfn = bfn_d; d.bfcode = bfcode_d;
  std::vector<double> xx(np), yy(np);
  for (int p = 0; p < np; p++) { xx[p] = m->coold[2 * (size_t)p]; yy[p] = m->coold[2 * (size_t)p + 1]; }
#define UP1(dst, src, n) cudaMemcpyAsync((void *)(dst), (src), (n) * sizeof(*(src)), cudaMemcpyHostToDevice, st)
  UP1(ipq_d, ipq.data(), ipq.size()); UP1(eptr_d, eptr.data(), eptr.size()); UP1(esv_d, esv.data(), esv.size());
  UP1(cptr_d, cptr.data(), cptr.size()); UP1(cor_d, cor.data(), cor.size()); UP1(bc_d, bc.data(), bc.size());
  UP1(wall_d, wall.data(), wall.size()); UP1(x0, xx.data(), np); UP1(y0, yy.data(), np);
  UP1(bptr_d, bptr.data(), bptr.size()); UP1(blist_d, blist.data(), blist.size());
  UP1(bfn_d, bfn.data(), bfn.size()); UP1(bfcode_d, bfcode.data(), bfcode.size());
  UP1(d.xn, xx.data(), np); UP1(d.yn, yy.data(), np); UP1(d.xs, xx.data(), np); UP1(d.ys, yy.data(), np);
#undef UP1
  Rules rl;
  fill_rule(5, false, rl.g25, rl.w25);
  fill_rule(6, false, rl.g36, rl.w36);
  cudaMemcpyToSymbolAsync(cR, &rl, sizeof(Rules), 0, cudaMemcpyHostToDevice, st);
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    destroy(s);
    err = "device set-up failed";
    return LAG2D_ECUDA;
  }
  *out = s;
  return LAG2D_OK;
}

static int download_geoel(Solver *s, double *geoel, std::string &err) {
  const Dev1 &d = s->d;
  const int ncell = d.ncell;
  std::vector<double> f(ncell);
  double *src[6] = {d.rc, d.sc, d.vol, d.mass, d.vcx, d.vcy};
  for (int k = 0; k < 6; k++) {
    CK1(cudaMemcpyAsync(f.data(), src[k], ncell * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK1(cudaStreamSynchronize(s->st));
    for (int e = 0; e < ncell; e++) geoel[24 * (size_t)e + k] = f[e];
  }
  if (d.nrz == 2) {  // geoel(11), the cell-averaged radius
    CK1(cudaMemcpyAsync(f.data(), d.rbar, ncell * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK1(cudaStreamSynchronize(s->st));
    for (int e = 0; e < ncell; e++) geoel[24 * (size_t)e + 10] = f[e];
  }
  return LAG2D_OK;
}

static int download_unkno(Solver *s, const double *src, double *unkno, std::string &err) {
  const Dev1 &d = s->d;
  launch(s, "copy", [&] { k1_unkno_out<<<nb(NU1 * d.ncell, 256), 256, 0, s->st>>>(d, src, s->stage_u); });
  CK1(cudaMemcpyAsync(unkno, s->stage_u, NU1 * (size_t)d.ncell * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  CK1(cudaStreamSynchronize(s->st));
  return LAG2D_OK;
}

static int download_xy(Solver *s, const double *X, const double *Y, double *xy, std::string &err) {
  const int np = s->d.npoin;
  launch_xy_out(np, s->st, s->stage_x, X, Y);
  s->launches += 1;
  CK1(cudaMemcpyAsync(xy, s->stage_x, 2 * (size_t)np * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  CK1(cudaStreamSynchronize(s->st));
  return LAG2D_OK;
}

int init_fields(Solver *s, double *geoel, double *amatr, double *unkno, std::string &err) {
  const Dev1 &d = s->d;
  const int np = d.npoin, ncell = d.ncell;
  launch(s, "init", [&] {
    k1_init_geo<<<nb(d.nquad, 128), 128, 0, s->st>>>(d);
    k1_init_fields<<<nb(d.nquad, 128), 128, 0, s->st>>>(d);
  }, 2);
  CK1(cudaMemcpyAsync(d.Us, d.Un, NU1 * (size_t)ncell * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
  CK1(cudaMemcpyAsync(d.xn, d.x0, np * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
  CK1(cudaMemcpyAsync(d.yn, d.y0, np * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
  CK1(cudaMemcpyAsync(d.xs, d.x0, np * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
  CK1(cudaMemcpyAsync(d.ys, d.y0, np * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
  CK1(cudaMemsetAsync(d.us, 0, np * sizeof(double), s->st));
  CK1(cudaMemsetAsync(d.vs, 0, np * sizeof(double), s->st));
  Scalars s0{};
  CK1(cudaMemcpyAsync(d.sc_dev, &s0, sizeof(Scalars), cudaMemcpyHostToDevice, s->st));
  geom(s, d.xn, d.yn);
  int r = read_status(s, err);
  if (r) return r;
  if (geoel) {
    std::fill(geoel, geoel + 24 * (size_t)ncell, 0.0);
    if ((r = download_geoel(s, geoel, err))) return r;
  }
  if (amatr) {
    std::vector<double> f(4 * (size_t)ncell);
    CK1(cudaMemcpyAsync(f.data(), d.amatr, f.size() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK1(cudaStreamSynchronize(s->st));
    for (int e = 0; e < ncell; e++)
      for (int k = 0; k < 4; k++) amatr[4 * (size_t)e + k] = f[k * (size_t)ncell + e];
  }
  if (unkno && (r = download_unkno(s, d.Un, unkno, err))) return r;
  return LAG2D_OK;
}

int set_state(Solver *s, const double *unkno, const double *coord, const double *ustar, const double *geoel,
              const double *amatr, std::string &err) {
  const Dev1 &d = s->d;
  const int ncell = d.ncell, np = d.npoin;
  CK1(cudaMemcpyAsync(s->stage_u, unkno, NU1 * (size_t)ncell * sizeof(double), cudaMemcpyHostToDevice, s->st));
  launch(s, "copy", [&] { k1_unkno_in<<<nb(NU1 * ncell, 256), 256, 0, s->st>>>(d, s->stage_u); });
  CK1(cudaMemcpyAsync(s->stage_x, coord, 2 * (size_t)np * sizeof(double), cudaMemcpyHostToDevice, s->st));
  launch_xy_in(np, s->st, s->stage_x, d.xn, d.yn, d.xs, d.ys);
  CK1(cudaStreamSynchronize(s->st));
  CK1(cudaMemcpyAsync(s->stage_x, ustar, 2 * (size_t)np * sizeof(double), cudaMemcpyHostToDevice, s->st));
  launch_xy_in(np, s->st, s->stage_x, d.us, d.vs, nullptr, nullptr);
  s->launches += 2;
  if (geoel) {
    std::vector<double> g(ncell);
    double *dst[4] = {d.rc, d.sc, d.vol, d.mass};
    for (int k = 0; k < 4; k++) {
      for (int e = 0; e < ncell; e++) g[e] = geoel[24 * (size_t)e + k];
      CK1(cudaMemcpyAsync(dst[k], g.data(), ncell * sizeof(double), cudaMemcpyHostToDevice, s->st));
      CK1(cudaStreamSynchronize(s->st));
    }
  }
  if (amatr) {
    std::vector<double> g(4 * (size_t)ncell);
    for (int e = 0; e < ncell; e++)
      for (int k = 0; k < 4; k++) g[k * (size_t)ncell + e] = amatr[4 * (size_t)e + k];
    CK1(cudaMemcpyAsync(d.amatr, g.data(), g.size() * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK1(cudaStreamSynchronize(s->st));
  }
  Scalars s0{};
  CK1(cudaMemcpyAsync(d.sc_dev, &s0, sizeof(Scalars), cudaMemcpyHostToDevice, s->st));
  geom(s, d.xs, d.ys);
  return read_status(s, err);
}

int step(Solver *s, int itime, double *dtfix, double *tacru, std::string &err) {
  int r = put_scalars(s, itime, *dtfix, *tacru, err);
  if (r) return r;
  enqueue_step(s, itime);
  Scalars sc;
  CK1(cudaMemcpyAsync(&sc, s->d.sc_dev, sizeof(Scalars), cudaMemcpyDeviceToHost, s->st));
  CK1(cudaStreamSynchronize(s->st));
  if (s->timing) flush_timing(s);
  *dtfix = sc.dtfix;
  *tacru = sc.tacru;
  return read_status(s, err);
}

int run(Solver *s, int itime0, int nsteps, double *dtfix, double *tacru, int *done, std::string &err) {
  int r = put_scalars(s, itime0 - 1, *dtfix, *tacru, err);
  if (r) return r;
  int steps = 0;
  if (s->timing) {
    for (int i = 0; i < nsteps; i++) { enqueue_step(s, itime0 + i); steps++; }
    flush_timing(s);
  } else {
    if (!s->graph) {
      cudaGraph_t g;
      CK1(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
      const long long before = s->launches;
      enqueue_step(s, -1);
      CK1(cudaStreamEndCapture(s->st, &g));
      CK1(cudaGraphInstantiate(&s->graph, g, 0));
      cudaGraphDestroy(g);
      s->graph_launches = s->launches - before;
      s->launches = before;
    }
    for (int i = 0; i < nsteps; i++) {
      CK1(cudaGraphLaunch(s->graph, s->st));
      s->launches += s->graph_launches;
      steps++;
    }
  }
  Scalars sc;
  CK1(cudaMemcpyAsync(&sc, s->d.sc_dev, sizeof(Scalars), cudaMemcpyDeviceToHost, s->st));
  CK1(cudaStreamSynchronize(s->st));
  *dtfix = sc.dtfix;
  *tacru = sc.tacru;
  if (done) *done = sc.done ? std::min(steps, std::max(0, sc.itime - itime0 + 1)) : steps;
  return read_status(s, err);
}

int get_state(Solver *s, double *unkno, double *coord, double *ustar, double *geoel, std::string &err) {
  int r;
  if (unkno && (r = download_unkno(s, s->d.Un, unkno, err))) return r;
  if (coord && (r = download_xy(s, s->d.xn, s->d.yn, coord, err))) return r;
  if (ustar && (r = download_xy(s, s->d.us, s->d.vs, ustar, err))) return r;
  if (geoel) {
    std::fill(geoel, geoel + 24 * (size_t)s->d.ncell, 0.0);
    if ((r = download_geoel(s, geoel, err))) return r;
  }
  return LAG2D_OK;
}

// the inner seam getrhsdg_lag_mcnew on the current state: limits the state,
// updates ustar, returns rhsel(3, 4, ncell)
int rhs(Solver *s, double *rhsel, std::string &err) {
  const Dev1 &d = s->d;
  int r = put_scalars(s, 1, 0.0, 0.0, err);
  if (r) return r;
  enqueue_rhs(s, 0, 0.0, 1);
  // the slope application of :7283-7298 alone: the update with alfa = 0 and dt = 0
  launch(s, "update", [&] { k1_update<<<nb(d.ncell, 128), 128, 0, s->st>>>(d, 0.0); });
  if ((r = read_status(s, err))) return r;
  if (s->timing) flush_timing(s);
  CK1(cudaMemcpyAsync(d.Un, d.Us, NU1 * (size_t)d.ncell * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
  if (rhsel) return download_unkno(s, d.rhs, rhsel, err);
  return LAG2D_OK;
}

int cellvol(Solver *s, double *geoel, std::string &err) {
  geom(s, s->d.xs, s->d.ys);
  int r = read_status(s, err);
  if (r) return r;
  if (geoel) {
    std::fill(geoel, geoel + 24 * (size_t)s->d.ncell, 0.0);
    return download_geoel(s, geoel, err);
  }
  return LAG2D_OK;
}

int cell_output(Solver *s, double *out, std::string &err) {
  const Dev1 &d = s->d;
  if (!s->cellout && !dalloc(s, &s->cellout, 9 * (size_t)d.ncell)) { err = "cudaMalloc failed"; return LAG2D_ECUDA; }
  launch(s, "post", [&] { k1_cell_output<<<nb(d.ncell, 256), 256, 0, s->st>>>(d, s->cellout); });
  std::vector<double> h(9 * (size_t)d.ncell);
  CK1(cudaMemcpyAsync(h.data(), s->cellout, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  CK1(cudaStreamSynchronize(s->st));
  CK1(cudaGetLastError());
  for (size_t e = 0; e < (size_t)d.ncell; e++)
    for (int k = 0; k < 9; k++) out[9 * e + k] = h[k * (size_t)d.ncell + e];
  return LAG2D_OK;
}

long long launches(const Solver *s) { return s->launches; }

void set_timing(Solver *s, bool on) {
  s->timing = on;
  s->fam.clear();
}

double kernel_ms(const Solver *s, const char *family, long long *n) {
  auto it = s->fam.find(family);
  if (it == s->fam.end() || it->second.n == 0) return -1.0;
  if (n) *n = it->second.n;
  return it->second.ms / it->second.n;
}

void destroy(Solver *s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  for (auto &p : s->pending) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
  if (s->graph) cudaGraphExecDestroy(s->graph);
  for (void *p : s->allocs) cudaFree(p);
  delete s;
}

}  // namespace p1
}  // namespace lag2d
