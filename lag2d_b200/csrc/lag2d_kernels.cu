// CUDA kernels of the Lag2D curved-P2 Lagrangian DG time step (sm_100a).
//
// One RK stage is the sequence
//   persson   (all quads)  troubled-cell marks, physical mass centre, frame
//   weno      (troubled)   WENO reconstruction into a side buffer, then commit
//   corner    (all quads)  sub-cell normals/densities, corner impedances and
//                          Riemann coefficients per corner face
//   node      (all nodes)  fixed-order gather of the corner coefficients and
//                          the 2x2 nodal solve for ustar (no atomics)
//   rhs       (all quads)  corner forces, face + volume integrals, source
//   dt        (stage 1)    deterministic min-reduction for getdelt_lag
//   update    (all cells)  M^-1 apply and RK combine
//   nodes     (all nodes)  node motion; centre-node re-interpolation and the
//                          cell volumes follow in the geom kernel
// Each kernel cites the reference routine it replaces (srccurv-lag/...).
// Arithmetic keeps the reference's expression order so that a build with
// --fmad=false reproduces the CPU restatement bit for bit.
#include <cuda_runtime.h>
#include <math.h>
#include "lag2d_device.cuh"
#include "lag2d_shape9.cuh"

namespace lag2d {

// Constant tables: one copy in constant memory for the kernels and a host
// mirror so that the same __host__ __device__ bodies can be checked on a CPU.
struct Tables {
  QuadTables q;
  double wrie[4][4][2];   // corner-face weights of the Riemann solver
  double wmas[4][4][2];   // mass-equation face weights of the face integral
  double wmom[4][4];      // momentum/energy face weights of the face integral
  double wtri[4][3][2];   // triangle corner-face weights (Getrhslaggauss.f90:12289-12302) x 0.25
};
__constant__ Tables cT;
static Tables hT;

__host__ __host__ __device__ __forceinline__ const Tables &TB() {
#ifdef __CUDA_ARCH__
  return cT;
#else
  return hT;
#endif
}
#define cQ (TB().q)
#define cPI 3.14159265358979311599796346854

__host__ __host__ __device__ __forceinline__ int atomic_add(int *p, int v) {
#ifdef __CUDA_ARCH__
  return atomicAdd(p, v);
#else
  int o = *p;
  *p = o + v;
  return o;
#endif
}
__host__ __host__ __device__ __forceinline__ void atomic_or(int *p, int v) {
#ifdef __CUDA_ARCH__
  atomicOr(p, v);
#else
  *p |= v;
#endif
}


__host__ __device__ __forceinline__ void load_quad(const Dev &d, const double *X, const double *Y, int iq,
                                          double (*xp)[2]) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    int p = d.ipq[k * d.nquad + iq];
    xp[k][0] = X[p];
    xp[k][1] = Y[p];
  }
}

__host__ __device__ __forceinline__ double Uget(const Dev &d, const double *U, int k, int q, int e) {
  return U[(q * NDEG + k) * d.ncell + e];
}

// initial density of cell e (getrhog_initial, GetInitial.f90:4-147: uniform per
// cell in the cases built here), times the caller's per-cell factor if set
__host__ __device__ __forceinline__ double rho_initial(const Dev &d, int e, double xc, double yc) {
  const double f = d.rho0 ? d.rho0[e] : 1.0;
  if (d.ncase == 6) return f * ((sqrt(xc * xc + yc * yc) <= 0.5) ? 1.0 : 0.125);
  return f;
}

__host__ __device__ __forceinline__ bool stopped(const Dev &d) { return d.sc_dev->done != 0; }

// ---------------------------------------------------------------------------
// getcellvol_lag (Limiterlag.f90:2038-2165): 6x6 Gauss volume and volume
// centre in reference coordinates.
// ---------------------------------------------------------------------------
__host__ __device__ void b_geom(const Dev &d, int iq, const double *X, const double *Y) {
  if (iq >= d.nquad || stopped(d)) return;
  const int e = iq + d.ntria;
  double xp[9][2], shp[9], dr[9], ds[9];
  load_quad(d, X, Y, iq, xp);
  const double alfrz = 0.0;
  double rcv = 0.0, scv = 0.0, volel = 0.0;
  for (int ig = 0; ig < 36; ig++) {
    double r = cQ.g36[ig][0], s = cQ.g36[ig][1], wi = cQ.w36[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    double xg, yg;
    map9(xp, shp, xg, yg);
    double rcoef = 1.0 - alfrz + alfrz * yg;
    double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    volel = volel + djaco * rcoef;
    rcv = rcv + r * djaco * rcoef;
    scv = scv + s * djaco * rcoef;
  }
  d.vol[e] = volel;
  d.vcx[e] = rcv / volel;
  d.vcy[e] = scv / volel;
  if (!(volel > 0.0)) atomic_or(&d.sc_dev->status, ST_NONPHYS);
}
__global__ void k_geom(Dev d, const double *X, const double *Y) { b_geom(d, blockIdx.x * blockDim.x + threadIdx.x, X, Y); }

// Step 9th-node re-interpolation (Getrhslag.f90:1963-1971) fused in front of
// the volume computation: the centre node belongs to one quad only.
__host__ __device__ void b_center_geom(const Dev &d, int iq) {
  if (iq >= d.nquad || stopped(d)) return;
  int p[9];
#pragma unroll
  for (int k = 0; k < 9; k++) p[k] = d.ipq[k * d.nquad + iq];
  double *XY[2] = {d.xs, d.ys};
  for (int c = 0; c < 2; c++) {
    double *X = XY[c];
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = X[p[k]];
    X[p[8]] = -0.25 * (x[0] + x[1] + x[2] + x[3]) + 0.5 * (x[4] + x[5] + x[6] + x[7]);
  }
}
__global__ void k_center_geom(Dev d) { b_center_geom(d, blockIdx.x * blockDim.x + threadIdx.x); }

// ---------------------------------------------------------------------------
// getSIHO_Persson (Limiterlag.f90:12042-12239) + Part I of
// weno_char_quad_orthgl (WENO.f90:5990-6090): troubled-cell marks, physical
// mass centre and the velocity-aligned frame for every quad.
// ---------------------------------------------------------------------------
__host__ __device__ void b_persson(const Dev &d, int iq) {
  if (iq >= d.nquad || stopped(d)) return;
  const int e = iq + d.ntria;
  double xp[9][2], xpi[9][2], shp[9], dr[9], ds[9];
  load_quad(d, d.xs, d.ys, iq, xp);
  load_quad(d, d.x0, d.y0, iq, xpi);
  const double rc = d.rc[e], sc = d.sc[e];
  const double g19 = d.g19[e], g20 = d.g20[e], g21 = d.g21[e];
  double u[NDEG];
#pragma unroll
  for (int k = 0; k < NDEG; k++) u[k] = Uget(d, d.Us, k, 0, e);
  double unvar2 = 0.0, unvar1 = 0.0;
  double xcrho, ycrho;
  shp9v(rc, sc, shp);
  map9(xpi, shp, xcrho, ycrho);
  double xmc = 0.0, ymc = 0.0;
  for (int ig = 0; ig < 25; ig++) {
    double r = cQ.g25[ig][0], s = cQ.g25[ig][1], wi = cQ.w25[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    double b[NDEG];
    b[0] = 1.0; b[1] = (r - rc) / 1.0; b[2] = (s - sc) / 1.0;
    b[3] = 0.5 * b[1] * b[1] - g19;
    b[4] = 0.5 * b[2] * b[2] - g20;
    b[5] = b[1] * b[2] - g21;
    double un = 0.0, up1 = 0.0;
#pragma unroll
    for (int k = 0; k < NDEG; k++) un = un + u[k] * b[k];
#pragma unroll
    for (int k = 0; k < 3; k++) up1 = up1 + u[k] * b[k];
    unvar2 = unvar2 + (up1 - un) * (up1 - un) * djaco;
    unvar1 = unvar1 + (un) * (un)*djaco;
    // physical mass centre (WENO.f90:6040-6082)
    Jac ji = jac9(xpi, dr, ds);
    double djacoi = wi * (ji.xr * ji.ys - ji.yr * ji.xs);
    double xgi, ygi, xg, yg;
    map9(xpi, shp, xgi, ygi);
    map9(xp, shp, xg, yg);
    double rhogi = rho_initial(d, e, xcrho, ycrho);
    xmc = xmc + rhogi * djacoi * xg;
    ymc = ymc + rhogi * djacoi * yg;
  }
  const double thr = -3.0 * log10(4.0) - 4.0;
  int fl = (log10(unvar2 / unvar1) <= thr) ? 0 : 1;
  d.flag[e] = fl;
  const double masel = d.mass[e];
  d.geoph[e] = xmc / masel;
  d.geoph[d.ncell + e] = ymc / masel;
  double ma = Uget(d, d.Us, 0, 1, e), mb = Uget(d, d.Us, 0, 2, e);
  double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
  if (sqrt(ma * ma + mb * mb) > 1.0e-10) {
    m0 = ma / sqrt(ma * ma + mb * mb);
    m2 = mb / sqrt(ma * ma + mb * mb);
    m1 = -mb / sqrt(ma * ma + mb * mb);
    m3 = ma / sqrt(ma * ma + mb * mb);
  }
  d.mapmt[0 * d.ncell + e] = m0;
  d.mapmt[1 * d.ncell + e] = m1;
  d.mapmt[2 * d.ncell + e] = m2;
  d.mapmt[3 * d.ncell + e] = m3;
  if (fl) {
    int slot = atomic_add(d.wcount, 1);
    d.wlist[slot] = iq;
  }
}
__global__ void k_persson(Dev d) { b_persson(d, blockIdx.x * blockDim.x + threadIdx.x); }

// Marks given by the caller instead of the Persson indicator (lag2d_weno).
__host__ __device__ void b_flags_from_host(const Dev &d, int iq, const int *flags) {
  if (iq >= d.nquad) return;
  const int e = iq + d.ntria;
  int fl = flags[e] != 0;
  d.flag[e] = fl;
  if (fl) {
    int slot = atomic_add(d.wcount, 1);
    d.wlist[slot] = iq;
  }
}
__global__ void k_flags_from_host(Dev d, const int *flags) { b_flags_from_host(d, blockIdx.x * blockDim.x + threadIdx.x, flags); }

// ---------------------------------------------------------------------------
// WENO reconstruction of one troubled quad (weno_stncl_quad_orthol3,
// WENO.f90:7541-8101; weno_cell_Taylor :7219; getgeophy_local_Taylor :6750;
// getunknp_local_Taylor :7005; basis_orthg :6683 with nbsis = 1).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ void vec_local(const double *mp, double &dx, double &dy) {
  double xl = dx * mp[0] + dy * mp[2];
  double yl = dx * mp[1] + dy * mp[3];
  dx = xl;
  dy = yl;
}
__host__ __device__ __forceinline__ void vec_local_back(const double *mp, double &dx, double &dy) {
  double xl = dx * mp[3] + dy * (-mp[2]);
  double yl = dx * (-mp[1]) + dy * mp[0];
  dx = xl;
  dy = yl;
}
__host__ __device__ __forceinline__ void basis_orthg1(const double *bt, const double *cf, double *bo) {
  bo[0] = bt[0]; bo[1] = bt[1]; bo[2] = bt[2];
  bo[3] = 0.5 * bt[1] * bt[1] - cf[0];
  bo[4] = 0.5 * bt[2] * bt[2] - cf[1];
  bo[5] = bt[1] * bt[2] - cf[2];
}

// n x n inverse (n <= 5), column-major, Gauss-Jordan with partial pivoting
// (stands in for Matinv225, LinearAlgebra.f90:130; same inverse up to rounding).
__host__ __device__ void inv_small(int n, const double *a, double *b) {
  double t[25];
  for (int i = 0; i < n * n; i++) { t[i] = a[i]; b[i] = 0.0; }
  for (int i = 0; i < n; i++) b[i + n * i] = 1.0;
  for (int k = 0; k < n; k++) {
    int piv = k;
    double big = fabs(t[k + n * k]);
    for (int i = k + 1; i < n; i++)
      if (fabs(t[i + n * k]) > big) { big = fabs(t[i + n * k]); piv = i; }
    if (piv != k)
      for (int j = 0; j < n; j++) {
        double s = t[k + n * j]; t[k + n * j] = t[piv + n * j]; t[piv + n * j] = s;
        s = b[k + n * j]; b[k + n * j] = b[piv + n * j]; b[piv + n * j] = s;
      }
    double dd = 1.0 / t[k + n * k];
    for (int j = 0; j < n; j++) { t[k + n * j] *= dd; b[k + n * j] *= dd; }
    for (int i = 0; i < n; i++) {
      if (i == k) continue;
      double f = t[i + n * k];
      if (f == 0.0) continue;
      for (int j = 0; j < n; j++) {
        t[i + n * j] -= f * t[k + n * j];
        b[i + n * j] -= f * b[k + n * j];
      }
    }
  }
}

// getmatrix_prj2 (Limiterlag.f90:16455-16562), column-major 4x4 outputs
__host__ __device__ void matrix_prj2(double g, double *qmat, double *qinvm, double dnx, double dny,
                            const double *ul, const double *ur) {
  const double eps = 1.0e-6;
  double rhoc1 = 1.0 / ul[0], u1 = ul[1], v1 = ul[2], e1 = ul[3];
  double rhoc2 = 1.0 / ur[0], u2 = ur[1], v2 = ur[2], e2 = ur[3];
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
#define Q(a, i, j) a[(i - 1) + 4 * (j - 1)]
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

// Initial-config density weights and rotated physical positions of the 25
// Gauss points of stencil cell jelem (shared by the WENO sub-steps).
__host__ __device__ void weno_points(const Dev &d, int jelem, const double *mp, double *rhodj, double *xl,
                            double *yl) {
  const int je = jelem - d.ntria;
  double xpqi[9][2], xpql[9][2], shp[9], dr[9], ds[9];
  load_quad(d, d.x0, d.y0, je, xpqi);
  load_quad(d, d.xs, d.ys, je, xpql);
  for (int k = 0; k < 9; k++) vec_local(mp, xpql[k][0], xpql[k][1]);
  double xcrho, ycrho;
  shp9v(d.rc[jelem], d.sc[jelem], shp);
  map9(xpqi, shp, xcrho, ycrho);
  const double rhogi = rho_initial(d, jelem, xcrho, ycrho);
  for (int ig = 0; ig < 25; ig++) {
    double r = cQ.g25[ig][0], s = cQ.g25[ig][1], wi = cQ.w25[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xpqi, dr, ds);
    double djacoi = wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map9(xpql, shp, xg, yg);
    rhodj[ig] = rhogi * djacoi;
    xl[ig] = xg;
    yl[ig] = yg;
  }
}

__host__ __device__ void b_weno(const Dev &d, int t) {
  if (stopped(d) || t >= *d.wcount) return;
  const int iq = d.wlist[t];
  const int ielem = iq + d.ntria;
  int ielaj[9];
  for (int k = 0; k < 9; k++) ielaj[k] = d.stencil[k * d.nquad + iq];
  if (ielaj[0] == -2) { atomic_or(&d.sc_dev->status, ST_STENCIL); }
  if (ielaj[0] < 0) return;  // boundary cell: the reference leaves it (WENO.f90:7704)
  const int ielst1[4][7] = {{1, 2, 5, 6, 9, 8, 3}, {1, 3, 2, 7, 6, 9, 5},
                                   {1, 4, 3, 8, 7, 6, 5}, {1, 5, 4, 9, 8, 7, 3}};
  const int ielst2[4][4] = {{1, 2, 6, 9}, {1, 3, 6, 7}, {1, 4, 8, 7}, {1, 5, 8, 9}};
  double mp[4];
  for (int k = 0; k < 4; k++) mp[k] = d.mapmt[k * d.ncell + ielem];
  double xpq[9][2];
  load_quad(d, d.xs, d.ys, iq, xpq);
  const double dxcl = sqrt(d.vol[ielem]), dycl = dxcl;

  double unkrl[9][4][6];
  for (int s = 0; s < 9; s++)
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < 6; k++) unkrl[s][q][k] = Uget(d, d.Us, k, q, ielaj[s]);
  for (int s = 0; s < 9; s++)
    for (int k = 0; k < 6; k++) vec_local(mp, unkrl[s][1][k], unkrl[s][2][k]);

  double rhodj[9][25], xl[9][25], yl[9][25];
  for (int s = 0; s < 9; s++) weno_points(d, ielaj[s], mp, rhodj[s], xl[s], yl[s]);

  // getgeophy_local_Taylor (nbsis = 1)
  double geopl[9][5];
  for (int s = 0; s < 9; s++) {
    int jelem = ielaj[s];
    double xclj = d.geoph[jelem], yclj = d.geoph[d.ncell + jelem];
    vec_local(mp, xclj, yclj);
    geopl[s][0] = xclj;
    geopl[s][1] = yclj;
    double dxclj = sqrt(d.vol[jelem]), dyclj = dxclj;
    double masel = d.mass[jelem];
    double v1 = 0.0, v2 = 0.0, v3 = 0.0;
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

  // getunknp_local_Taylor: local orthogonal-basis coefficients per stencil cell
  double unkpl[9][4][6], mtbbq[25], mtbbi[25];
  for (int s = 0; s < 9; s++) {
    int jelem = ielaj[s];
    double rcj = d.rc[jelem], scj = d.sc[jelem];
    double xclj = geopl[s][0], yclj = geopl[s][1];
    double dxclj = sqrt(d.vol[jelem]), dyclj = dxclj;
    double bb[25], bbq[25], bbi[25], bbqi[25];
    for (int i = 0; i < 25; i++) { bb[i] = 0.0; bbq[i] = 0.0; }
    for (int ig = 0; ig < 25; ig++) {
      double r = cQ.g25[ig][0], s_ = cQ.g25[ig][1];
      double bq[6], bqpl[3], bqol[6];
      bq[0] = 1.0; bq[1] = (r - rcj) / 1.0; bq[2] = (s_ - scj) / 1.0;
      bq[3] = 0.5 * bq[1] * bq[1] - d.g19[jelem];
      bq[4] = 0.5 * bq[2] * bq[2] - d.g20[jelem];
      bq[5] = bq[1] * bq[2] - d.g21[jelem];
      bqpl[0] = 1.0; bqpl[1] = (xl[s][ig] - xclj) / dxclj; bqpl[2] = (yl[s][ig] - yclj) / dyclj;
      basis_orthg1(bqpl, &geopl[s][2], bqol);
      for (int i = 1; i < 6; i++)
        for (int j = 1; j < 6; j++) {
          bb[(i - 1) + 5 * (j - 1)] = bb[(i - 1) + 5 * (j - 1)] + rhodj[s][ig] * bq[i] * bqol[j];
          bbq[(i - 1) + 5 * (j - 1)] = bbq[(i - 1) + 5 * (j - 1)] + rhodj[s][ig] * bqol[i] * bqol[j];
        }
    }
    double rhs[6][4];
    for (int i = 0; i < 6; i++) for (int q = 0; q < 4; q++) rhs[i][q] = 0.0;
    for (int i = 1; i < 6; i++)
      for (int j = 1; j < 6; j++)
        for (int q = 0; q < 4; q++) rhs[i][q] = rhs[i][q] + unkrl[s][q][j] * bb[(j - 1) + 5 * (i - 1)];
    inv_small(5, bbq, bbqi);
    inv_small(5, bb, bbi);
    for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) unkpl[s][q][k] = 0.0;
    for (int i = 1; i < 6; i++)
      for (int j = 1; j < 6; j++)
        for (int q = 0; q < 4; q++) unkpl[s][q][i] = unkpl[s][q][i] + rhs[j][q] * bbqi[(j - 1) + 5 * (i - 1)];
    if (s == 0)
      for (int i = 0; i < 25; i++) { mtbbq[i] = bbq[i]; mtbbi[i] = bbi[i]; }
    for (int q = 0; q < 4; q++) unkpl[s][q][0] = unkrl[s][q][0];
  }

  // candidate polynomials: 1 central + 4 Lagrangian + 4 Hermite stencils
  double unksl[9][4][6];
  for (int is = 0; is < 9; is++)
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < 6; k++) unksl[is][q][k] = 0.0;
  for (int is = 0; is < 9; is++) for (int q = 0; q < 4; q++) unksl[is][q][0] = unkpl[0][q][0];
  for (int k = 0; k < 6; k++) for (int q = 0; q < 4; q++) unksl[0][q][k] = unkpl[0][q][k];
  int isten = 0;
  const double xmcl = geopl[0][0], ymcl = geopl[0][1];
  for (int is = 0; is < 4; is++) {
    isten++;
    double matlg[25], rhslg[20], matin[25];
    for (int i = 0; i < 25; i++) matlg[i] = 0.0;
    for (int i = 0; i < 20; i++) rhslg[i] = 0.0;
    for (int ies = 0; ies < 5; ies++) {
      int sl = ielst1[is][ies + 1] - 1;
      double masej = d.mass[ielaj[sl]];
      for (int ig = 0; ig < 25; ig++) {
        double bqplj[3], bqolj[6];
        bqplj[0] = 1.0; bqplj[1] = (xl[sl][ig] - xmcl) / dxcl; bqplj[2] = (yl[sl][ig] - ymcl) / dycl;
        basis_orthg1(bqplj, &geopl[0][2], bqolj);
        for (int k = 0; k < 5; k++) matlg[ies + 5 * k] = matlg[ies + 5 * k] + rhodj[sl][ig] * bqolj[k + 1] / masej;
      }
      for (int q = 0; q < 4; q++) rhslg[q + 4 * ies] = unkpl[sl][q][0] - unkpl[0][q][0];
    }
    inv_small(5, matlg, matin);
    for (int k = 1; k < 6; k++)
      for (int ies = 0; ies < 5; ies++)
        for (int q = 0; q < 4; q++)
          unksl[isten][q][k] = unksl[isten][q][k] + matin[(k - 1) + 5 * ies] * rhslg[q + 4 * ies];
  }
  for (int is = 0; is < 4; is++) {
    isten++;
    double mathm[45], rhshm[36], matls[25], rhsls[20], matin[25];
    for (int i = 0; i < 45; i++) mathm[i] = 0.0;
    for (int i = 0; i < 36; i++) rhshm[i] = 0.0;
    for (int ies = 0; ies < 3; ies++) {
      int sl = ielst2[is][ies + 1] - 1;
      int jelem = ielaj[sl];
      double masej = d.mass[jelem];
      double dxclj = sqrt(d.vol[jelem]), dyclj = dxclj;
      double xclj = geopl[sl][0], yclj = geopl[sl][1];
      for (int ig = 0; ig < 25; ig++) {
        double bqplj[3], bqol[6], bqolj[6];
        bqplj[0] = 1.0; bqplj[1] = (xl[sl][ig] - xmcl) / dxcl; bqplj[2] = (yl[sl][ig] - ymcl) / dycl;
        basis_orthg1(bqplj, &geopl[0][2], bqol);
        for (int k = 0; k < 5; k++) mathm[ies + 9 * k] = mathm[ies + 9 * k] + rhodj[sl][ig] * bqol[k + 1] / masej;
        bqplj[0] = 1.0; bqplj[1] = (xl[sl][ig] - xclj) / dxclj; bqplj[2] = (yl[sl][ig] - yclj) / dyclj;
        basis_orthg1(bqplj, &geopl[sl][2], bqolj);
        int ieshm = 3 + 2 * ies;
        for (int k = 1; k < 6; k++) {
          mathm[ieshm + 9 * (k - 1)] = mathm[ieshm + 9 * (k - 1)] + rhodj[sl][ig] * bqol[k] * bqolj[1] / masej;
          mathm[ieshm + 1 + 9 * (k - 1)] = mathm[ieshm + 1 + 9 * (k - 1)] + rhodj[sl][ig] * bqol[k] * bqolj[2] / masej;
        }
        for (int k = 1; k < 6; k++)
          for (int q = 0; q < 4; q++) {
            rhshm[q + 4 * ieshm] = rhshm[q + 4 * ieshm] + rhodj[sl][ig] * bqolj[k] * bqolj[1] * unkpl[sl][q][k] / masej;
            rhshm[q + 4 * (ieshm + 1)] =
                rhshm[q + 4 * (ieshm + 1)] + rhodj[sl][ig] * bqolj[k] * bqolj[2] * unkpl[sl][q][k] / masej;
          }
      }
      for (int q = 0; q < 4; q++) rhshm[q + 4 * ies] = unkpl[sl][q][0] - unkpl[0][q][0];
    }
    // matrix_sym (LinearAlgebra.f90:89): normal equations of the 9x5 system
    for (int i = 0; i < 25; i++) matls[i] = 0.0;
    for (int i = 0; i < 20; i++) rhsls[i] = 0.0;
    for (int im = 0; im < 5; im++)
      for (int jm = 0; jm < 5; jm++)
        for (int km = 0; km < 9; km++) matls[im + 5 * jm] = matls[im + 5 * jm] + mathm[km + 9 * im] * mathm[km + 9 * jm];
    for (int q = 0; q < 4; q++)
      for (int im = 0; im < 5; im++)
        for (int km = 0; km < 9; km++) rhsls[q + 4 * im] = rhsls[q + 4 * im] + mathm[km + 9 * im] * rhshm[q + 4 * km];
    inv_small(5, matls, matin);
    for (int k = 1; k < 6; k++)
      for (int ies = 0; ies < 5; ies++)
        for (int q = 0; q < 4; q++)
          unksl[isten][q][k] = unksl[isten][q][k] + matin[(k - 1) + 5 * ies] * rhsls[q + 4 * ies];
  }
  isten++;  // 9 candidate polynomials

  // weno_cell_Taylor: characteristic WENO per interior face, averaged
  const double epsil = 1.0e-6;
  const double dxc = sqrt(d.vol[ielem]), dyc = dxc;
  const int mapfe[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
  double unk_phy[4][6];
  for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) unk_phy[q][k] = 0.0;
  double unkf_phy[4][4][6];
  for (int a = 0; a < 4; a++) for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) unkf_phy[a][q][k] = 0.0;
  int ifprj = 0;
  for (int ies = 0; ies < 4; ies++) {
    int jelem = d.esq[ies * d.nquad + iq];
    if (jelem < 0) continue;
    double dtx = xpq[mapfe[ies][1]][0] - xpq[mapfe[ies][0]][0];
    double dty = xpq[mapfe[ies][1]][1] - xpq[mapfe[ies][0]][1];
    double dlgt = sqrt(dtx * dtx + dty * dty);
    double dnx = dty / dlgt, dny = -dtx / dlgt;
    vec_local(mp, dnx, dny);
    double ul[4], ur[4];
    for (int q = 0; q < 4; q++) { ul[q] = Uget(d, d.Us, 0, q, ielem); ur[q] = Uget(d, d.Us, 0, q, jelem); }
    vec_local(mp, ul[1], ul[2]);
    vec_local(mp, ur[1], ur[2]);
    double qmat[16], qinvm[16];
    matrix_prj2(d.gamlg, qmat, qinvm, dnx, dny, ul, ur);
    double weigh[9][4], weigt[4] = {0.0, 0.0, 0.0, 0.0}, os1[9];
    for (int is = 0; is < isten; is++) {
      double mx = 0.0;
      for (int k = 0; k < 4; k++) {
        // characteristic coefficient k of moments 2 and 3 (first derivatives)
        double c1 = 0.0, c2 = 0.0;
        for (int q = 0; q < 4; q++) {
          c1 = c1 + qinvm[k + 4 * q] * unksl[is][q][1];
          c2 = c2 + qinvm[k + 4 * q] * unksl[is][q][2];
        }
        double t1 = c1 / dxc, t2 = c2 / dyc;
        double os = t1 * t1 + t2 * t2;
        if (k == 0 || os > mx) mx = os;
      }
      os1[is] = mx;
    }
    double weigl0 = .2, weigl1 = 0.8 / (isten - 1.0);
    for (int is = 0; is < isten; is++)
      for (int q = 0; q < 4; q++) {
        double tt = epsil + os1[is];
        weigh[is][q] = (is == 0 ? weigl0 : weigl1) / (tt * tt);
      }
    for (int q = 0; q < 4; q++)
      for (int is = 0; is < isten; is++) weigt[q] = weigt[q] + weigh[is][q];
    for (int is = 0; is < isten; is++)
      for (int q = 0; q < 4; q++) weigh[is][q] = weigh[is][q] / weigt[q];
    double fch[4][6];
    for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) fch[q][k] = 0.0;
    for (int is = 0; is < isten; is++)
      for (int kq = 0; kq < 4; kq++)
        for (int k = 0; k < 6; k++) {
          double ch = 0.0;
          for (int q = 0; q < 4; q++) ch = ch + qinvm[kq + 4 * q] * unksl[is][q][k];
          fch[kq][k] = fch[kq][k] + weigh[is][kq] * ch;
        }
    for (int kq = 0; kq < 4; kq++)
      for (int k = 1; k < 6; k++)
        for (int q = 0; q < 4; q++) unkf_phy[ifprj][q][k] = unkf_phy[ifprj][q][k] + qmat[q + 4 * kq] * fch[kq][k];
    ifprj++;
  }
  double weigf = 1.0 / ifprj;
  for (int a = 0; a < ifprj; a++)
    for (int q = 0; q < 4; q++)
      for (int k = 1; k < 6; k++) unk_phy[q][k] = unk_phy[q][k] + weigf * unkf_phy[a][q][k];

  // inverse L2 projection back to the target's Taylor basis, un-rotate
  double rhsuk[5][4], out[4][6];
  for (int i = 0; i < 5; i++) for (int q = 0; q < 4; q++) rhsuk[i][q] = 0.0;
  for (int i = 1; i < 6; i++)
    for (int j = 1; j < 6; j++)
      for (int q = 0; q < 4; q++) rhsuk[i - 1][q] = rhsuk[i - 1][q] + unk_phy[q][j] * mtbbq[(j - 1) + 5 * (i - 1)];
  for (int q = 0; q < 4; q++) for (int k = 1; k < 6; k++) out[q][k] = 0.0;
  for (int i = 1; i < 6; i++)
    for (int j = 1; j < 6; j++)
      for (int q = 0; q < 4; q++) out[q][i] = out[q][i] + rhsuk[j - 1][q] * mtbbi[(j - 1) + 5 * (i - 1)];
  for (int k = 1; k < 6; k++) vec_local_back(mp, out[1][k], out[2][k]);
  for (int q = 0; q < 4; q++)
    for (int k = 1; k < 6; k++) d.Uw[(q * 5 + (k - 1)) * d.nquad + iq] = out[q][k];
  d.flag[ielem] = 2;  // reconstructed
}
__global__ void __launch_bounds__(64) k_weno(Dev d) { b_weno(d, blockIdx.x * blockDim.x + threadIdx.x); }

// Copy the reconstructions into the stage state once every read of the
// pre-limit state is done (the reference's unknr copy, WENO.f90:6096).
__host__ __device__ void b_weno_commit(const Dev &d, int t) {
  if (stopped(d) || t >= *d.wcount) return;
  const int iq = d.wlist[t];
  const int e = iq + d.ntria;
  if (d.flag[e] != 2) return;
  for (int q = 0; q < 4; q++)
    for (int k = 1; k < 6; k++) d.Us[(q * NDEG + k) * d.ncell + e] = d.Uw[(q * 5 + (k - 1)) * d.nquad + iq];
}
__global__ void k_weno_commit(Dev d) { b_weno_commit(d, blockIdx.x * blockDim.x + threadIdx.x); }
// Exchange the replaced moments between the state and the reconstruction
// buffer (the adjoint's reverse stage switches the recorded stage input
// between its values before and after WENO this way, in place).
__global__ void k_weno_swap(Dev d) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *d.wcount) return;
  const int iq = d.wlist[t];
  const int e = iq + d.ntria;
  if (d.flag[e] != 2) return;
  for (int q = 0; q < 4; q++)
    for (int k = 1; k < 6; k++) {
      double *a = d.Us + (q * NDEG + k) * (size_t)d.ncell + e, *b = d.Uw + (q * 5 + (k - 1)) * (size_t)d.nquad + iq;
      const double v = *a;
      *a = *b;
      *b = v;
    }
}

// ---------------------------------------------------------------------------
// The same WENO reconstruction with one warp per troubled quad (the optimised
// step's version).  The per-item arithmetic is b_weno's; the independent
// items run on different lanes: the 216 stencil DOFs, the 81 stencil nodes,
// the 225 stencil quadrature points, the 9 stencil cells' local geometry and
// L2 projections, the 8 candidate stencils and the 4 faces, with the data
// between phases in shared memory.  Lane 0 combines the faces in order and
// writes the result.  Blocks of one warp loop over the troubled list.
// ---------------------------------------------------------------------------
struct WenoShared {
  double unkrl[9][4][6];
  double xpqi[9][9][2], xpql[9][9][2], rhogi[9];
  double rhodj[9][25], xl[9][25], yl[9][25];
  double geopl[9][5];
  double unkpl[9][4][6];
  double mtbbq[25], mtbbi[25];
  double unksl[9][4][6];
  double unkf[4][4][6];
  int fvalid[4];
};

// The reconstruction's linear factors at a given state, for its adjoint: with
// the stencil, the frame mapmt, the characteristic matrices and the nonlinear
// weights held at their values for that state (the limiter's active set
// frozen), the new moments 1..5 of the troubled quad are a linear map of its
// 3x3 stencil's DOFs: rotation R, per-cell local projection T_s, candidate
// polynomials (Lagrangian: matL on cell-average differences; Hermite: G on
// the 9 least-squares rows, whose derivative rows are H applied to the
// neighbour's local moments), per face the characteristic projection and
// weighted sum, the face average, the back projection B and the inverse
// rotation.
struct WenoFactors {
  double T[9][25];          // T_s[(m-1)*5 + (i-1)]: local moment i from rotated moment m
  double matL[4][25];       // Lagrangian stencils: moment k from cell-average difference ies
  double G[4][5][9];        // Hermite stencils: moment k from least-squares row km
  double H[4][3][2][5];     // Hermite derivative rows of stencil cell ies: weights of its moments 1..5
  double qinvm[4][16], qmat[4][16], wgt[4][9][4];  // per face
  double B[5][5];           // back projection: out moment i from face-averaged moment j, B[j-1][i-1]
  double mp[4];
  int ifprj;
};

template <bool FACT>
__device__ void weno_warp_cell_t(const Dev &d, int t, WenoShared &S, WenoFactors *F) {
  const int lane = threadIdx.x & 31;
  const int iq = d.wlist[t];
  const int ielem = iq + d.ntria;
  int ielaj[9];
  for (int k = 0; k < 9; k++) ielaj[k] = d.stencil[k * d.nquad + iq];
  if (ielaj[0] == -2 && lane == 0 && !FACT) atomic_or(&d.sc_dev->status, ST_STENCIL);
  if (ielaj[0] < 0) return;  // boundary cell: the reference leaves it (WENO.f90:7704)
  const int ielst1[4][7] = {{1, 2, 5, 6, 9, 8, 3}, {1, 3, 2, 7, 6, 9, 5},
                            {1, 4, 3, 8, 7, 6, 5}, {1, 5, 4, 9, 8, 7, 3}};
  const int ielst2[4][4] = {{1, 2, 6, 9}, {1, 3, 6, 7}, {1, 4, 8, 7}, {1, 5, 8, 9}};
  double mp[4];
  for (int k = 0; k < 4; k++) mp[k] = d.mapmt[k * d.ncell + ielem];
  const double dxcl = sqrt(d.vol[ielem]), dycl = dxcl;

  // stencil DOFs (velocities rotated to the local frame) and stencil nodes
  for (int e = lane; e < 216; e += 32) {
    const int s = e / 24, q = (e / 6) % 4, k = e % 6;
    S.unkrl[s][q][k] = Uget(d, d.Us, k, q, ielaj[s]);
  }
  for (int e = lane; e < 81; e += 32) {
    const int s = e / 9, k = e % 9;
    const int p = d.ipq[k * d.nquad + (ielaj[s] - d.ntria)];
    S.xpqi[s][k][0] = d.x0[p];
    S.xpqi[s][k][1] = d.y0[p];
    double x = d.xs[p], y = d.ys[p];
    vec_local(mp, x, y);
    S.xpql[s][k][0] = x;
    S.xpql[s][k][1] = y;
  }
  __syncwarp();
  for (int e = lane; e < 54; e += 32) {
    const int s = e / 6, k = e % 6;
    vec_local(mp, S.unkrl[s][1][k], S.unkrl[s][2][k]);
  }
  if (lane < 9) {
    const int jelem = ielaj[lane];
    double shp[9], xcrho, ycrho;
    shp9v(d.rc[jelem], d.sc[jelem], shp);
    map9(S.xpqi[lane], shp, xcrho, ycrho);
    S.rhogi[lane] = rho_initial(d, jelem, xcrho, ycrho);
  }
  __syncwarp();
  // quadrature points of the stencil cells (weno_points)
  for (int e = lane; e < 225; e += 32) {
    const int s = e / 25, ig = e % 25;
    const double r = cQ.g25[ig][0], sp = cQ.g25[ig][1], wi = cQ.w25[ig];
    double shp[9], dr[9], ds[9];
    shp9v(r, sp, shp);
    shp9d(r, sp, dr, ds);
    Jac j = jac9(S.xpqi[s], dr, ds);
    const double djacoi = wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map9(S.xpql[s], shp, xg, yg);
    S.rhodj[s][ig] = S.rhogi[s] * djacoi;
    S.xl[s][ig] = xg;
    S.yl[s][ig] = yg;
  }
  __syncwarp();
  // getgeophy_local_Taylor, then getunknp_local_Taylor, one stencil cell per lane
  if (lane < 9) {
    const int s = lane, jelem = ielaj[s];
    double xclj = d.geoph[jelem], yclj = d.geoph[d.ncell + jelem];
    vec_local(mp, xclj, yclj);
    const double dxclj = sqrt(d.vol[jelem]), dyclj = dxclj;
    const double masel = d.mass[jelem];
    double v1 = 0.0, v2 = 0.0, v3 = 0.0;
    for (int ig = 0; ig < 25; ig++) {
      double b2 = (S.xl[s][ig] - xclj) / dxclj, b3 = (S.yl[s][ig] - yclj) / dyclj;
      v1 = v1 + S.rhodj[s][ig] * b2 * b2;
      v2 = v2 + S.rhodj[s][ig] * b3 * b3;
      v3 = v3 + S.rhodj[s][ig] * b2 * b3;
    }
    v1 = v1 / masel; v2 = v2 / masel; v3 = v3 / masel;
    double gp[5] = {xclj, yclj, 0.5 * v1, 0.5 * v2, v3};
    for (int k = 0; k < 5; k++) S.geopl[s][k] = gp[k];
    const double rcj = d.rc[jelem], scj = d.sc[jelem];
    double bb[25], bbq[25], bbi[25], bbqi[25];
    for (int i = 0; i < 25; i++) { bb[i] = 0.0; bbq[i] = 0.0; }
    for (int ig = 0; ig < 25; ig++) {
      double r = cQ.g25[ig][0], s_ = cQ.g25[ig][1];
      double bq[6], bqpl[3], bqol[6];
      bq[0] = 1.0; bq[1] = (r - rcj) / 1.0; bq[2] = (s_ - scj) / 1.0;
      bq[3] = 0.5 * bq[1] * bq[1] - d.g19[jelem];
      bq[4] = 0.5 * bq[2] * bq[2] - d.g20[jelem];
      bq[5] = bq[1] * bq[2] - d.g21[jelem];
      bqpl[0] = 1.0; bqpl[1] = (S.xl[s][ig] - xclj) / dxclj; bqpl[2] = (S.yl[s][ig] - yclj) / dyclj;
      basis_orthg1(bqpl, &gp[2], bqol);
      for (int i = 1; i < 6; i++)
        for (int j = 1; j < 6; j++) {
          bb[(i - 1) + 5 * (j - 1)] = bb[(i - 1) + 5 * (j - 1)] + S.rhodj[s][ig] * bq[i] * bqol[j];
          bbq[(i - 1) + 5 * (j - 1)] = bbq[(i - 1) + 5 * (j - 1)] + S.rhodj[s][ig] * bqol[i] * bqol[j];
        }
    }
    double rhs[6][4];
    for (int i = 0; i < 6; i++) for (int q = 0; q < 4; q++) rhs[i][q] = 0.0;
    for (int i = 1; i < 6; i++)
      for (int j = 1; j < 6; j++)
        for (int q = 0; q < 4; q++) rhs[i][q] = rhs[i][q] + S.unkrl[s][q][j] * bb[(j - 1) + 5 * (i - 1)];
    inv_small(5, bbq, bbqi);
    inv_small(5, bb, bbi);
    double up[4][6];
    for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) up[q][k] = 0.0;
    for (int i = 1; i < 6; i++)
      for (int j = 1; j < 6; j++)
        for (int q = 0; q < 4; q++) up[q][i] = up[q][i] + rhs[j][q] * bbqi[(j - 1) + 5 * (i - 1)];
    for (int q = 0; q < 4; q++) up[q][0] = S.unkrl[s][q][0];
    for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) S.unkpl[s][q][k] = up[q][k];
    if (s == 0)
      for (int i = 0; i < 25; i++) { S.mtbbq[i] = bbq[i]; S.mtbbi[i] = bbi[i]; }
    if (FACT) {
      // up[i] = sum_m unkrl[m] sum_j bb[(m-1)+5(j-1)] bbqi[(j-1)+5(i-1)]
      for (int m = 1; m < 6; m++)
        for (int i = 1; i < 6; i++) {
          double acc = 0.0;
          for (int j = 1; j < 6; j++) acc += bb[(m - 1) + 5 * (j - 1)] * bbqi[(j - 1) + 5 * (i - 1)];
          F->T[s][(m - 1) * 5 + (i - 1)] = acc;
        }
    }
  }
  __syncwarp();
  // candidate polynomials: 1 central (lane 8) + 4 Lagrangian (lanes 0-3) + 4 Hermite (lanes 4-7)
  const double xmcl = S.geopl[0][0], ymcl = S.geopl[0][1];
  if (lane < 9) {
    const int isten = lane < 8 ? lane + 1 : 0;
    double us[4][6];
    for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) us[q][k] = 0.0;
    for (int q = 0; q < 4; q++) us[q][0] = S.unkpl[0][q][0];
    if (isten == 0) {
      for (int k = 0; k < 6; k++) for (int q = 0; q < 4; q++) us[q][k] = S.unkpl[0][q][k];
    } else if (isten <= 4) {
      const int is = isten - 1;
      double matlg[25], rhslg[20], matin[25];
      for (int i = 0; i < 25; i++) matlg[i] = 0.0;
      for (int i = 0; i < 20; i++) rhslg[i] = 0.0;
      for (int ies = 0; ies < 5; ies++) {
        int sl = ielst1[is][ies + 1] - 1;
        double masej = d.mass[ielaj[sl]];
        for (int ig = 0; ig < 25; ig++) {
          double bqplj[3], bqolj[6];
          bqplj[0] = 1.0; bqplj[1] = (S.xl[sl][ig] - xmcl) / dxcl; bqplj[2] = (S.yl[sl][ig] - ymcl) / dycl;
          basis_orthg1(bqplj, &S.geopl[0][2], bqolj);
          for (int k = 0; k < 5; k++) matlg[ies + 5 * k] = matlg[ies + 5 * k] + S.rhodj[sl][ig] * bqolj[k + 1] / masej;
        }
        for (int q = 0; q < 4; q++) rhslg[q + 4 * ies] = S.unkpl[sl][q][0] - S.unkpl[0][q][0];
      }
      inv_small(5, matlg, matin);
      if (FACT)
        for (int i = 0; i < 25; i++) F->matL[is][i] = matin[i];
      for (int k = 1; k < 6; k++)
        for (int ies = 0; ies < 5; ies++)
          for (int q = 0; q < 4; q++) us[q][k] = us[q][k] + matin[(k - 1) + 5 * ies] * rhslg[q + 4 * ies];
    } else {
      const int is = isten - 5;
      double mathm[45], rhshm[36], matls[25], rhsls[20], matin[25];
      for (int i = 0; i < 45; i++) mathm[i] = 0.0;
      for (int i = 0; i < 36; i++) rhshm[i] = 0.0;
      for (int ies = 0; ies < 3; ies++) {
        int sl = ielst2[is][ies + 1] - 1;
        int jelem = ielaj[sl];
        double masej = d.mass[jelem];
        double dxclj = sqrt(d.vol[jelem]), dyclj = dxclj;
        double xclj = S.geopl[sl][0], yclj = S.geopl[sl][1];
        for (int ig = 0; ig < 25; ig++) {
          double bqplj[3], bqol[6], bqolj[6];
          bqplj[0] = 1.0; bqplj[1] = (S.xl[sl][ig] - xmcl) / dxcl; bqplj[2] = (S.yl[sl][ig] - ymcl) / dycl;
          basis_orthg1(bqplj, &S.geopl[0][2], bqol);
          for (int k = 0; k < 5; k++) mathm[ies + 9 * k] = mathm[ies + 9 * k] + S.rhodj[sl][ig] * bqol[k + 1] / masej;
          bqplj[0] = 1.0; bqplj[1] = (S.xl[sl][ig] - xclj) / dxclj; bqplj[2] = (S.yl[sl][ig] - yclj) / dyclj;
          basis_orthg1(bqplj, &S.geopl[sl][2], bqolj);
          int ieshm = 3 + 2 * ies;
          for (int k = 1; k < 6; k++) {
            mathm[ieshm + 9 * (k - 1)] = mathm[ieshm + 9 * (k - 1)] + S.rhodj[sl][ig] * bqol[k] * bqolj[1] / masej;
            mathm[ieshm + 1 + 9 * (k - 1)] =
                mathm[ieshm + 1 + 9 * (k - 1)] + S.rhodj[sl][ig] * bqol[k] * bqolj[2] / masej;
          }
          for (int k = 1; k < 6; k++)
            for (int q = 0; q < 4; q++) {
              rhshm[q + 4 * ieshm] =
                  rhshm[q + 4 * ieshm] + S.rhodj[sl][ig] * bqolj[k] * bqolj[1] * S.unkpl[sl][q][k] / masej;
              rhshm[q + 4 * (ieshm + 1)] =
                  rhshm[q + 4 * (ieshm + 1)] + S.rhodj[sl][ig] * bqolj[k] * bqolj[2] * S.unkpl[sl][q][k] / masej;
            }
          if (FACT)
            for (int k = 1; k < 6; k++) {
              F->H[is][ies][0][k - 1] = (ig == 0 ? 0.0 : F->H[is][ies][0][k - 1]) +
                                        S.rhodj[sl][ig] * bqolj[k] * bqolj[1] / masej;
              F->H[is][ies][1][k - 1] = (ig == 0 ? 0.0 : F->H[is][ies][1][k - 1]) +
                                        S.rhodj[sl][ig] * bqolj[k] * bqolj[2] / masej;
            }
        }
        for (int q = 0; q < 4; q++) rhshm[q + 4 * ies] = S.unkpl[sl][q][0] - S.unkpl[0][q][0];
      }
      for (int i = 0; i < 25; i++) matls[i] = 0.0;
      for (int i = 0; i < 20; i++) rhsls[i] = 0.0;
      for (int im = 0; im < 5; im++)
        for (int jm = 0; jm < 5; jm++)
          for (int km = 0; km < 9; km++) matls[im + 5 * jm] = matls[im + 5 * jm] + mathm[km + 9 * im] * mathm[km + 9 * jm];
      for (int q = 0; q < 4; q++)
        for (int im = 0; im < 5; im++)
          for (int km = 0; km < 9; km++) rhsls[q + 4 * im] = rhsls[q + 4 * im] + mathm[km + 9 * im] * rhshm[q + 4 * km];
      inv_small(5, matls, matin);
      if (FACT)
        for (int k = 1; k < 6; k++)
          for (int km = 0; km < 9; km++) {
            double acc = 0.0;
            for (int im = 0; im < 5; im++) acc += matin[(k - 1) + 5 * im] * mathm[km + 9 * im];
            F->G[is][k - 1][km] = acc;
          }
      for (int k = 1; k < 6; k++)
        for (int ies = 0; ies < 5; ies++)
          for (int q = 0; q < 4; q++) us[q][k] = us[q][k] + matin[(k - 1) + 5 * ies] * rhsls[q + 4 * ies];
    }
    for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) S.unksl[isten][q][k] = us[q][k];
  }
  __syncwarp();
  // weno_cell_Taylor: characteristic WENO per interior face (lanes 0-3)
  const int isten = 9;
  const double epsil = 1.0e-6;
  const double dxc = sqrt(d.vol[ielem]), dyc = dxc;
  if (lane < 4) {
    const int ies = lane;
    const int mapfe[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
    const int jelem = d.esq[ies * d.nquad + iq];
    S.fvalid[ies] = jelem >= 0;
    if (jelem >= 0) {
      const int pa = d.ipq[mapfe[ies][0] * d.nquad + iq], pb = d.ipq[mapfe[ies][1] * d.nquad + iq];
      double dtx = d.xs[pb] - d.xs[pa];
      double dty = d.ys[pb] - d.ys[pa];
      double dlgt = sqrt(dtx * dtx + dty * dty);
      double dnx = dty / dlgt, dny = -dtx / dlgt;
      vec_local(mp, dnx, dny);
      double ul[4], ur[4];
      for (int q = 0; q < 4; q++) { ul[q] = Uget(d, d.Us, 0, q, ielem); ur[q] = Uget(d, d.Us, 0, q, jelem); }
      vec_local(mp, ul[1], ul[2]);
      vec_local(mp, ur[1], ur[2]);
      double qmat[16], qinvm[16];
      matrix_prj2(d.gamlg, qmat, qinvm, dnx, dny, ul, ur);
      double weigh[9][4], weigt[4] = {0.0, 0.0, 0.0, 0.0}, os1[9];
      for (int is = 0; is < isten; is++) {
        double mx = 0.0;
        for (int k = 0; k < 4; k++) {
          double c1 = 0.0, c2 = 0.0;
          for (int q = 0; q < 4; q++) {
            c1 = c1 + qinvm[k + 4 * q] * S.unksl[is][q][1];
            c2 = c2 + qinvm[k + 4 * q] * S.unksl[is][q][2];
          }
          double t1 = c1 / dxc, t2 = c2 / dyc;
          double os = t1 * t1 + t2 * t2;
          if (k == 0 || os > mx) mx = os;
        }
        os1[is] = mx;
      }
      double weigl0 = .2, weigl1 = 0.8 / (isten - 1.0);
      for (int is = 0; is < isten; is++)
        for (int q = 0; q < 4; q++) {
          double tt = epsil + os1[is];
          weigh[is][q] = (is == 0 ? weigl0 : weigl1) / (tt * tt);
        }
      for (int q = 0; q < 4; q++)
        for (int is = 0; is < isten; is++) weigt[q] = weigt[q] + weigh[is][q];
      for (int is = 0; is < isten; is++)
        for (int q = 0; q < 4; q++) weigh[is][q] = weigh[is][q] / weigt[q];
      if (FACT) {
        for (int i = 0; i < 16; i++) { F->qinvm[ies][i] = qinvm[i]; F->qmat[ies][i] = qmat[i]; }
        for (int is = 0; is < isten; is++)
          for (int q = 0; q < 4; q++) F->wgt[ies][is][q] = weigh[is][q];
      }
      double fch[4][6];
      for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) fch[q][k] = 0.0;
      for (int is = 0; is < isten; is++)
        for (int kq = 0; kq < 4; kq++)
          for (int k = 0; k < 6; k++) {
            double ch = 0.0;
            for (int q = 0; q < 4; q++) ch = ch + qinvm[kq + 4 * q] * S.unksl[is][q][k];
            fch[kq][k] = fch[kq][k] + weigh[is][kq] * ch;
          }
      double uf[4][6];
      for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) uf[q][k] = 0.0;
      for (int kq = 0; kq < 4; kq++)
        for (int k = 1; k < 6; k++)
          for (int q = 0; q < 4; q++) uf[q][k] = uf[q][k] + qmat[q + 4 * kq] * fch[kq][k];
      for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) S.unkf[ies][q][k] = uf[q][k];
    }
  }
  __syncwarp();
  if (FACT) {
    if (lane == 0) {
      int ifprj = 0;
      for (int a = 0; a < 4; a++) ifprj += S.fvalid[a];
      F->ifprj = ifprj;
      for (int k = 0; k < 4; k++) F->mp[k] = mp[k];
      for (int j = 1; j < 6; j++)
        for (int i = 1; i < 6; i++) {
          double acc = 0.0;
          for (int m = 1; m < 6; m++) acc += S.mtbbq[(j - 1) + 5 * (m - 1)] * S.mtbbi[(m - 1) + 5 * (i - 1)];
          F->B[j - 1][i - 1] = acc;
        }
    }
    __syncwarp();
    return;
  }
  if (lane == 0) {
    int ifprj = 0;
    for (int a = 0; a < 4; a++) ifprj += S.fvalid[a];
    double unk_phy[4][6];
    for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) unk_phy[q][k] = 0.0;
    const double weigf = 1.0 / ifprj;
    for (int a = 0; a < 4; a++) {
      if (!S.fvalid[a]) continue;
      for (int q = 0; q < 4; q++)
        for (int k = 1; k < 6; k++) unk_phy[q][k] = unk_phy[q][k] + weigf * S.unkf[a][q][k];
    }
    // inverse L2 projection back to the target's Taylor basis, un-rotate
    double rhsuk[5][4], out[4][6];
    for (int i = 0; i < 5; i++) for (int q = 0; q < 4; q++) rhsuk[i][q] = 0.0;
    for (int i = 1; i < 6; i++)
      for (int j = 1; j < 6; j++)
        for (int q = 0; q < 4; q++) rhsuk[i - 1][q] = rhsuk[i - 1][q] + unk_phy[q][j] * S.mtbbq[(j - 1) + 5 * (i - 1)];
    for (int q = 0; q < 4; q++) for (int k = 1; k < 6; k++) out[q][k] = 0.0;
    for (int i = 1; i < 6; i++)
      for (int j = 1; j < 6; j++)
        for (int q = 0; q < 4; q++) out[q][i] = out[q][i] + rhsuk[j - 1][q] * S.mtbbi[(j - 1) + 5 * (i - 1)];
    for (int k = 1; k < 6; k++) vec_local_back(mp, out[1][k], out[2][k]);
    for (int q = 0; q < 4; q++)
      for (int k = 1; k < 6; k++) d.Uw[(q * 5 + (k - 1)) * d.nquad + iq] = out[q][k];
    d.flag[ielem] = 2;  // reconstructed
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// The frozen reconstruction as a linear map, and its transpose (the WENO
// part of the adjoint).  For troubled quad c (list slot t) with a complete
// stencil, out_c = L_c v: the factors of L_c come from weno_warp_cell_t<true>
// at the state d.Us; v is a state-shaped vector.  The transpose kernel
// writes L_c^T lam_c (lam_c: the adjoint of c's replaced moments 1..5) per
// stencil cell into wbuf[(s*24 + q*6 + k) * cap + t]; the gather kernel adds
// these into the adjoint of each cell in a fixed order and zeroes the
// replaced moments' own adjoint (the step overwrote them).
// ---------------------------------------------------------------------------
struct WenoAdjShared {
  double vr[9][4][6];       // tangent: rotated stencil moments; transpose: adjoint of unkpl
  double vp[9][4][6];       // tangent: local projections
  double vus[9][4][6];      // candidate polynomials (tangent) / their adjoints (transpose)
  double vf[4][4][6];       // per face: characteristic sums (tangent) / their adjoints
  double vphy[4][6];        // face-averaged moments / their adjoint
  double vd[8][4][9];       // transpose: adjoints of the Lagrangian differences and Hermite rows
};
__constant__ int cIelst1[4][7] = {{1, 2, 5, 6, 9, 8, 3}, {1, 3, 2, 7, 6, 9, 5}, {1, 4, 3, 8, 7, 6, 5}, {1, 5, 4, 9, 8, 7, 3}};
__constant__ int cIelst2[4][4] = {{1, 2, 6, 9}, {1, 3, 6, 7}, {1, 4, 8, 7}, {1, 5, 8, 9}};

// out moments 1..5 of troubled slot t = L_t v (v and out are state-shaped)
__device__ void weno_tangent_cell(const Dev &d, int t, const WenoFactors &F, WenoAdjShared &A, const double *v,
                                  double *out) {
  const int lane = threadIdx.x & 31;
  const int iq = d.wlist[t], ielem = iq + d.ntria;
  int ielaj[9];
  for (int k = 0; k < 9; k++) ielaj[k] = d.stencil[k * d.nquad + iq];
  const double *mp = F.mp;
  if (lane < 9) {
    const int s = lane;
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < 6; k++) A.vr[s][q][k] = Uget(d, v, k, q, ielaj[s]);
    for (int k = 0; k < 6; k++) vec_local(mp, A.vr[s][1][k], A.vr[s][2][k]);
    for (int q = 0; q < 4; q++) {
      A.vp[s][q][0] = A.vr[s][q][0];
      for (int i = 1; i < 6; i++) {
        double acc = 0.0;
        for (int m = 1; m < 6; m++) acc += A.vr[s][q][m] * F.T[s][(m - 1) * 5 + (i - 1)];
        A.vp[s][q][i] = acc;
      }
    }
  }
  __syncwarp();
  if (lane < 9) {
    const int isten = lane < 8 ? lane + 1 : 0;
    double us[4][6];
    for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) us[q][k] = 0.0;
    for (int q = 0; q < 4; q++) us[q][0] = A.vp[0][q][0];
    if (isten == 0) {
      for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) us[q][k] = A.vp[0][q][k];
    } else if (isten <= 4) {
      const int is = isten - 1;
      for (int ies = 0; ies < 5; ies++) {
        const int sl = cIelst1[is][ies + 1] - 1;
        for (int q = 0; q < 4; q++) {
          const double dv = A.vp[sl][q][0] - A.vp[0][q][0];
          for (int k = 1; k < 6; k++) us[q][k] += F.matL[is][(k - 1) + 5 * ies] * dv;
        }
      }
    } else {
      const int is = isten - 5;
      for (int q = 0; q < 4; q++) {
        double rh[9];
        for (int km = 0; km < 3; km++) rh[km] = A.vp[cIelst2[is][km + 1] - 1][q][0] - A.vp[0][q][0];
        for (int ies = 0; ies < 3; ies++) {
          const int sl = cIelst2[is][ies + 1] - 1;
          for (int row = 0; row < 2; row++) {
            double acc = 0.0;
            for (int k = 1; k < 6; k++) acc += F.H[is][ies][row][k - 1] * A.vp[sl][q][k];
            rh[3 + 2 * ies + row] = acc;
          }
        }
        for (int k = 1; k < 6; k++) {
          double acc = 0.0;
          for (int km = 0; km < 9; km++) acc += F.G[is][k - 1][km] * rh[km];
          us[q][k] = acc;
        }
      }
    }
    for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) A.vus[isten][q][k] = us[q][k];
  }
  __syncwarp();
  if (lane < 4) {
    const int a = lane;
    double fch[4][6];
    for (int kq = 0; kq < 4; kq++)
      for (int k = 1; k < 6; k++) {
        double acc = 0.0;
        for (int is = 0; is < 9; is++) {
          double ch = 0.0;
          for (int q = 0; q < 4; q++) ch += F.qinvm[a][kq + 4 * q] * A.vus[is][q][k];
          acc += F.wgt[a][is][kq] * ch;
        }
        fch[kq][k] = acc;
      }
    for (int q = 0; q < 4; q++)
      for (int k = 1; k < 6; k++) {
        double acc = 0.0;
        for (int kq = 0; kq < 4; kq++) acc += F.qmat[a][q + 4 * kq] * fch[kq][k];
        A.vf[a][q][k] = acc;
      }
  }
  __syncwarp();
  if (lane == 0) {
    const double weigf = 1.0 / F.ifprj;
    double phy[4][6];
    for (int q = 0; q < 4; q++)
      for (int k = 1; k < 6; k++) {
        double acc = 0.0;
        for (int a = 0; a < 4; a++)
          if (d.esq[a * d.nquad + iq] >= 0) acc += weigf * A.vf[a][q][k];
        phy[q][k] = acc;
      }
    double o[4][6];
    for (int q = 0; q < 4; q++)
      for (int i = 1; i < 6; i++) {
        double acc = 0.0;
        for (int j = 1; j < 6; j++) acc += phy[q][j] * F.B[j - 1][i - 1];
        o[q][i] = acc;
      }
    for (int k = 1; k < 6; k++) vec_local_back(mp, o[1][k], o[2][k]);
    for (int q = 0; q < 4; q++)
      for (int k = 1; k < 6; k++) out[(q * 6 + k) * (size_t)d.ncell + ielem] = o[q][k];
  }
  __syncwarp();
}

// wbuf slot t: L_t^T lam, lam = the adjoint of troubled quad t's moments 1..5 in lamU
__device__ void weno_transpose_cell(const Dev &d, int t, const WenoFactors &F, WenoAdjShared &A,
                                    const double *lamU, double *wbuf, int cap) {
  const int lane = threadIdx.x & 31;
  const int iq = d.wlist[t], ielem = iq + d.ntria;
  const double *mp = F.mp;
  // back rotation, back projection and face average, transposed
  if (lane == 0) {
    double lo[4][6];
    for (int q = 0; q < 4; q++)
      for (int k = 1; k < 6; k++) lo[q][k] = lamU[(q * 6 + k) * (size_t)d.ncell + ielem];
    for (int k = 1; k < 6; k++) {
      const double l1 = lo[1][k], l2 = lo[2][k];
      lo[1][k] = mp[3] * l1 - mp[1] * l2;    // vec_local_back: x' = mp3 x - mp2 y, y' = -mp1 x + mp0 y
      lo[2][k] = -mp[2] * l1 + mp[0] * l2;
    }
    const double weigf = 1.0 / F.ifprj;
    for (int q = 0; q < 4; q++) {
      A.vphy[q][0] = 0.0;
      for (int j = 1; j < 6; j++) {
        double acc = 0.0;
        for (int i = 1; i < 6; i++) acc += F.B[j - 1][i - 1] * lo[q][i];
        A.vphy[q][j] = weigf * acc;
      }
    }
  }
  __syncwarp();
  // per face: characteristic back transform, transposed
  if (lane < 4) {
    const int a = lane;
    const bool valid = d.esq[a * d.nquad + iq] >= 0;
    for (int kq = 0; kq < 4; kq++)
      for (int k = 0; k < 6; k++) {
        double acc = 0.0;
        if (valid && k > 0)
          for (int q = 0; q < 4; q++) acc += F.qmat[a][q + 4 * kq] * A.vphy[q][k];
        A.vf[a][kq][k] = acc;
      }
  }
  __syncwarp();
  // candidates: weights and characteristic projection, transposed (faces in order)
  if (lane < 9) {
    const int is = lane;
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < 6; k++) {
        double acc = 0.0;
        if (k > 0)
          for (int a = 0; a < 4; a++)
            for (int kq = 0; kq < 4; kq++) acc += F.qinvm[a][kq + 4 * q] * F.wgt[a][is][kq] * A.vf[a][kq][k];
        A.vus[is][q][k] = acc;
      }
  }
  __syncwarp();
  // adjoints of the candidates' inputs: Lagrangian differences, Hermite rows
  if (lane < 8) {
    if (lane < 4) {
      const int is = lane;
      for (int q = 0; q < 4; q++)
        for (int ies = 0; ies < 5; ies++) {
          double acc = 0.0;
          for (int k = 1; k < 6; k++) acc += F.matL[is][(k - 1) + 5 * ies] * A.vus[1 + is][q][k];
          A.vd[is][q][ies] = acc;
        }
    } else {
      const int is = lane - 4;
      for (int q = 0; q < 4; q++)
        for (int km = 0; km < 9; km++) {
          double acc = 0.0;
          for (int k = 1; k < 6; k++) acc += F.G[is][k - 1][km] * A.vus[5 + is][q][k];
          A.vd[4 + is][q][km] = acc;
        }
    }
  }
  __syncwarp();
  // per stencil cell: adjoint of its local projection, of the projection and rotation
  if (lane < 9) {
    const int s = lane;
    double lp[4][6];
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < 6; k++) lp[q][k] = (s == 0 && k > 0) ? A.vus[0][q][k] : 0.0;
    for (int is = 0; is < 4; is++)
      for (int ies = 0; ies < 5; ies++) {
        const int sl = cIelst1[is][ies + 1] - 1;
        for (int q = 0; q < 4; q++) {
          if (sl == s) lp[q][0] += A.vd[is][q][ies];
          if (s == 0) lp[q][0] -= A.vd[is][q][ies];
        }
      }
    for (int is = 0; is < 4; is++) {
      for (int km = 0; km < 3; km++) {
        const int sl = cIelst2[is][km + 1] - 1;
        for (int q = 0; q < 4; q++) {
          if (sl == s) lp[q][0] += A.vd[4 + is][q][km];
          if (s == 0) lp[q][0] -= A.vd[4 + is][q][km];
        }
      }
      for (int ies = 0; ies < 3; ies++) {
        if (cIelst2[is][ies + 1] - 1 != s) continue;
        for (int row = 0; row < 2; row++)
          for (int q = 0; q < 4; q++)
            for (int k = 1; k < 6; k++) lp[q][k] += F.H[is][ies][row][k - 1] * A.vd[4 + is][q][3 + 2 * ies + row];
      }
    }
    double lr[4][6];
    for (int q = 0; q < 4; q++) {
      lr[q][0] = lp[q][0];
      for (int m = 1; m < 6; m++) {
        double acc = 0.0;
        for (int i = 1; i < 6; i++) acc += F.T[s][(m - 1) * 5 + (i - 1)] * lp[q][i];
        lr[q][m] = acc;
      }
    }
    // vec_local: x' = mp0 x + mp2 y, y' = mp1 x + mp3 y; transposed
    for (int k = 0; k < 6; k++) {
      const double a1 = lr[1][k], a2 = lr[2][k];
      lr[1][k] = mp[0] * a1 + mp[1] * a2;
      lr[2][k] = mp[2] * a1 + mp[3] * a2;
    }
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < 6; k++) wbuf[((size_t)(s * 24 + q * 6 + k)) * cap + t] = lr[q][k];
  }
  __syncwarp();
}

struct WenoAdjBlock {
  WenoShared S;
  WenoFactors F;
  WenoAdjShared A;
};

// mode 0: the tangent out = L v on troubled quads; mode 1: the transpose into wbuf
__global__ void __launch_bounds__(32) k_weno_linear(Dev d, int mode, const double *v, double *out, double *wbuf,
                                                    int *wslot, int cap, int *overflow) {
  extern __shared__ __align__(16) unsigned char wsm[];
  WenoAdjBlock &B = *reinterpret_cast<WenoAdjBlock *>(wsm);
  const int n = *d.wcount;
  const int lane = threadIdx.x & 31;
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    const int iq = d.wlist[t];
    if (d.stencil[iq] < 0 || d.flag[iq + d.ntria] != 2) continue;  // left unlimited by the forward pass
    weno_warp_cell_t<true>(d, t, B.S, &B.F);
    if (mode == 0) {
      weno_tangent_cell(d, t, B.F, B.A, v, out);
    } else {
      if (t >= cap) {
        if (lane == 0) atomicExch(overflow, 1);
        continue;
      }
      if (lane == 0) wslot[iq] = t;
      weno_transpose_cell(d, t, B.F, B.A, v, wbuf, cap);
    }
  }
}

// per cell: the adjoint of the stage state before WENO from the one after it
// (quads), and with fold the adjoint of U^n added in (the end of stage 1's
// reverse, every cell); nothing to do, and no memory touched, when WENO
// replaced no quad and fold is 0
__global__ void k_weno_gather(Dev d, double *lamU, double *lamUn, int fold, const double *wbuf, const int *wslot,
                              int cap, const int *inv_ptr, const int *inv_ent) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.ncell) return;
  const int nw = *d.wcount;
  if (nw == 0 && !fold) return;
  const int jq = e - d.ntria;
  if (!fold) {
    // a cell that is neither replaced nor in a replaced quad's stencil keeps
    // its adjoint: leave it untouched (most cells, when few quads are troubled)
    bool touched = false;
    if (jq >= 0) {
      touched = d.flag[e] == 2 && d.stencil[jq] >= 0;
      for (int i = inv_ptr[jq]; i < inv_ptr[jq + 1] && !touched; i++) {
        const int c = inv_ent[i] / 9;
        touched = d.flag[c + d.ntria] == 2 && d.stencil[c] >= 0 && wslot[c] >= 0 && wslot[c] < cap;
      }
    }
    if (!touched) return;
  }
  const size_t nc = d.ncell;
  double l[24];
  for (int v = 0; v < 24; v++) l[v] = lamU[v * nc + e];
  const int j = e - d.ntria;
  if (nw > 0 && j >= 0) {
    if (d.flag[e] == 2 && d.stencil[j] >= 0)
      for (int q = 0; q < 4; q++)
        for (int k = 1; k < 6; k++) l[q * 6 + k] = 0.0;
    for (int i = inv_ptr[j]; i < inv_ptr[j + 1]; i++) {
      const int c = inv_ent[i] / 9, s = inv_ent[i] - 9 * c;
      if (d.flag[c + d.ntria] != 2 || d.stencil[c] < 0) continue;
      const int t = wslot[c];
      if (t < 0 || t >= cap) continue;
      for (int v = 0; v < 24; v++) l[v] += wbuf[((size_t)(s * 24 + v)) * cap + t];
    }
  }
  if (fold)
    for (int v = 0; v < 24; v++) {
      l[v] += lamUn[v * nc + e];
      lamUn[v * nc + e] = 0.0;
    }
  for (int v = 0; v < 24; v++) lamU[v * nc + e] = l[v];
}

__global__ void __launch_bounds__(32) k_weno_warp(Dev d) {
  __shared__ WenoShared S;
  if (stopped(d)) return;
  const int n = *d.wcount;
  for (int t = blockIdx.x; t < n; t += gridDim.x) weno_warp_cell_t<false>(d, t, S, nullptr);
}


// ---------------------------------------------------------------------------
// Sub-cell normals of a quad (getfnds_lagsmsif_hybrid, Getrhslaggauss.f90:
// 3537-3599; getfnds_lagsms_simpsonhybrid, :9908-10010): gq[16][3].
// ---------------------------------------------------------------------------
__host__ __device__ void normals_quad(const double (*xpq)[2], double (*gq)[3]) {
  const double posqc[4][2] = {{0.0, -0.5}, {0.5, 0.0}, {0.0, 0.5}, {-0.5, 0.0}};
  double shp[9];
#pragma unroll
  for (int ifa = 0; ifa < 4; ifa++) {
    double xv, yv;
    shp9v(posqc[ifa][0], posqc[ifa][1], shp);
    map9(xpq, shp, xv, yv);
    const double r = -1.0;
    double d0 = -0.5 + r, d1 = 0.5 + r, d2 = -2.0 * r;
    double dxdr = 0.0, dydr = 0.0;
    dxdr = dxdr + d0 * xpq[4 + ifa][0];
    dydr = dydr + d0 * xpq[4 + ifa][1];
    dxdr = dxdr + d1 * xpq[8][0];
    dydr = dydr + d1 * xpq[8][1];
    dxdr = dxdr + d2 * xv;
    dydr = dydr + d2 * yv;
    double djaco = sqrt(dxdr * dxdr + dydr * dydr);
    double anx = -dydr, any = dxdr;
    gq[8 + ifa][0] = anx / sqrt(anx * anx + any * any);
    gq[8 + ifa][1] = any / sqrt(anx * anx + any * any);
    gq[8 + ifa][2] = djaco * 2.0;
  }
  const double posiq[12][2] = {{-1, -1}, {1, -1}, {1, -1}, {1, 1}, {1, 1}, {-1, 1},
                               {-1, 1}, {-1, -1}, {0, -1}, {1, 0}, {0, 1}, {-1, 0}};
  const double vnx[4] = {0.0, 1.0, 0.0, -1.0}, vny[4] = {-1.0, 0.0, 1.0, 0.0};
  const int side[12] = {0, 0, 1, 1, 2, 2, 3, 3, 0, 1, 2, 3};
#pragma unroll
  for (int ig = 0; ig < 12; ig++) {
    double dr[9], ds[9];
    shp9d(posiq[ig][0], posiq[ig][1], dr, ds);
    Jac j = jac9(xpq, dr, ds);
    double vn0 = vnx[side[ig]], vn1 = vny[side[ig]], larea = 2.0;
    double anx = j.ys * vn0 + (-j.yr) * vn1;
    double any = (-j.xs) * vn0 + j.xr * vn1;
    double v0 = anx * larea, v1 = any * larea;
    double farea = sqrt(v0 * v0 + v1 * v1);
    int slot = (ig < 8) ? ig : ig + 4;
    gq[slot][0] = anx * larea / farea;
    gq[slot][1] = any * larea / farea;
    gq[slot][2] = farea;
  }
}

// sub-cell vertices (getndvelo_lagsubg ipqsg, Getrhslaggauss.f90:4424-4427), 0-based
// corner-face -> gesgq slot with orientation sign (fnqsg, Getrhslaggauss.f90:10486-10506)
__host__ __host__ __device__ __forceinline__ int ipqsg_(int isg, int ivsg) {
  const int t[16] = {0, 4, 8, 7, 4, 1, 5, 8, 8, 5, 2, 6, 7, 8, 6, 3};
  return t[4 * isg + ivsg];
}
__host__ __host__ __device__ __forceinline__ int fnqsg_(int isg, int k) {
  const int t[32] = {8, 1, 13, -9, -9, 12, 12, 16, 9, 13, 2, 3, 14, -10, -10, 9,
                     -11, 10, 10, 14, 4, 5, 15, -11, 16, -12, -12, 11, 11, 15, 6, 7};
  return t[8 * isg + k];
}
__host__ __host__ __device__ __forceinline__ double xvq_(int iv) {
  const double t[9] = {-1, 1, 1, -1, 0, 1, 0, -1, 0};
  return t[iv];
}
__host__ __host__ __device__ __forceinline__ double yvq_(int iv) {
  const double t[9] = {-1, -1, 1, 1, -1, 0, 1, 0, 0};
  return t[iv];
}
#define cWRIE (TB().wrie)
#define cWMAS (TB().wmas)
#define cWMOM (TB().wmom)

__host__ __device__ __forceinline__ void corner_normal(const double (*gq)[3], int isg, int ivsg, int f, double &n0,
                                              double &n1, double &a) {
  int code = fnqsg_(isg, 2 * ivsg + f);
  int slot = abs(code) - 1;
  double sg = (code >= 0) ? 1.0 : -1.0;
  n0 = sg * gq[slot][0];
  n1 = sg * gq[slot][1];
  a = gq[slot][2];
}

// Taylor basis at the 9 nodes (bq of getriem_quadsubg2 / rhsifacedg_lagsubgq2)
__host__ __device__ __forceinline__ void node_basis(double rc, double sc, double g19, double g20, double g21, int iv,
                                           double *b) {
  b[0] = 1.0;
  b[1] = (xvq_(iv) - rc) / 1.0;
  b[2] = (yvq_(iv) - sc) / 1.0;
  b[3] = 0.5 * b[1] * b[1] - g19;
  b[4] = 0.5 * b[2] * b[2] - g20;
  b[5] = b[1] * b[2] - g21;
}

// ---------------------------------------------------------------------------
// Corner pass: getriem_quadsubg2 (Getrhslaggauss.f90:10409-10867) with
// getrhosubg_averg (:7067, initial sub-cell masses hoisted to set-up) and
// getrhosubg_daverg (:10949).  Writes, per corner face, the Riemann
// coefficients of getriecoef_matrixnew (Limiterlag.f90:1037): m = mu*A,
// m*u_c, m*v_c and sigma.n*A.
// ---------------------------------------------------------------------------
__host__ __device__ void b_corner(const Dev &d, int iq) {
  if (iq >= d.nquad || stopped(d)) return;
  const int e = iq + d.ntria;
  const double eps = 1.0e-6, g = d.gamlg;
  const double slpdu = (g + 1.0) / 2.0;
  double xpq[9][2];
  load_quad(d, d.xs, d.ys, iq, xpq);
  double gq[16][3];
  normals_quad(xpq, gq);
  const double rc = d.rc[e], sc = d.sc[e], g19 = d.g19[e], g20 = d.g20[e], g21 = d.g21[e];
  double u[4][NDEG];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int k = 0; k < NDEG; k++) u[q][k] = Uget(d, d.Us, k, q, e);
  const double rhomc = u[0][0];
  const double uctr = u[1][0], vctr = u[2][0], ectr = u[3][0];
  const double rhoct = 1.0 / rhomc;
  const double pctr = fmax(eps, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
  const double sdctr = sqrt(fmax(eps, g * pctr / rhoct));

  // getrhosubg_averg: initial sub-cell mass / current sub-cell volume
  double unksgq[4];
  {
    const double posqc[12][2] = {{-0.5, -1.0}, {0.5, -1.0}, {1.0, -0.5}, {1.0, 0.5}, {0.5, 1.0}, {-0.5, 1.0},
                                 {-1.0, 0.5}, {-1.0, -0.5}, {0.0, -0.5}, {0.5, 0.0}, {0.0, 0.5}, {-0.5, 0.0}};
    const int ipqsc[4][4] = {{0, 8, 11, 7}, {1, 2, 9, 8}, {9, 3, 4, 10}, {11, 10, 5, 6}};
    double xpqc[12][2], shp[9];
#pragma unroll
    for (int isc = 0; isc < 12; isc++) {
      shp9v(posqc[isc][0], posqc[isc][1], shp);
      map9(xpq, shp, xpqc[isc][0], xpqc[isc][1]);
    }
    for (int isg = 0; isg < 4; isg++) {
      double xs[9][2];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        xs[k][0] = xpq[ipqsg_(isg, k)][0]; xs[k][1] = xpq[ipqsg_(isg, k)][1];
        xs[4 + k][0] = xpqc[ipqsc[isg][k]][0]; xs[4 + k][1] = xpqc[ipqsc[isg][k]][1];
      }
#pragma unroll
      for (int c = 0; c < 2; c++)
        xs[8][c] = -0.25 * (xs[0][c] + xs[1][c] + xs[2][c] + xs[3][c]) + 0.5 * (xs[4][c] + xs[5][c] + xs[6][c] + xs[7][c]);
      double f0 = 0.0;
      for (int ig = 0; ig < 25; ig++) {
        double dr[9], ds[9];
        shp9d(cQ.g25[ig][0], cQ.g25[ig][1], dr, ds);
        Jac j = jac9(xs, dr, ds);
        f0 = f0 + cQ.w25[ig] * (j.xr * j.ys - j.yr * j.xs);
      }
      unksgq[isg] = 0.0 + (1.0 / f0) * d.msub[isg * d.nquad + iq];
    }
  }
  // getrhosubg_daverg: sub-cell harmonic specific volume of the DG tau
  double uqsgc[4];
  for (int isg = 0; isg < 4; isg++) {
    double masel = 0.0, volel = 0.0;
    const double ofr = (isg == 0 || isg == 3) ? -1.0 : 1.0;
    const double ofs = (isg == 0 || isg == 1) ? -1.0 : 1.0;
    for (int ig = 0; ig < 25; ig++) {
      double r = (cQ.g25[ig][0] + ofr) / 2.0;
      double s = (cQ.g25[ig][1] + ofs) / 2.0;
      double b[6];
      b[0] = 1.0; b[1] = (r - rc) / 1.0; b[2] = (s - sc) / 1.0;
      b[3] = 0.5 * b[1] * b[1] - g19;
      b[4] = 0.5 * b[2] * b[2] - g20;
      b[5] = b[1] * b[2] - g21;
      double rhomsg = 0.0;
#pragma unroll
      for (int k = 0; k < NDEG; k++)
        if (k < d.mdegr) rhomsg = rhomsg + u[0][k] * b[k];
      if (d.nlimi == 6) rhomsg = rhomc + 1.0 * (rhomsg - rhomc);
      double dr[9], ds[9];
      shp9d(r, s, dr, ds);
      Jac j = jac9(xpq, dr, ds);
      double djaco = cQ.w25[ig] * (j.xr * j.ys - j.yr * j.xs) * 0.25;
      masel = masel + 1.0 / rhomsg * djaco;
      volel = volel + djaco;
    }
    uqsgc[isg] = volel / masel;
  }
  // states at the 9 nodes
  double unknvq[9][4];
#pragma unroll
  for (int iv = 0; iv < 9; iv++) {
    double b[6];
    node_basis(rc, sc, g19, g20, g21, iv, b);
#pragma unroll
    for (int q = 0; q < 4; q++) unknvq[iv][q] = 0.0;
#pragma unroll
    for (int k = 0; k < NDEG; k++)
      if (k < d.mdegr)
#pragma unroll
        for (int q = 0; q < 4; q++) unknvq[iv][q] = unknvq[iv][q] + u[q][k] * b[k];
  }
  for (int isg = 0; isg < 4; isg++) {
    double uv[4][2], sig[4], aj3[4];
#pragma unroll
    for (int ivsg = 0; ivsg < 4; ivsg++) {
      const int iv = ipqsg_(isg, ivsg);
      double rhovt = 1.0 / unknvq[iv][0];
      double rhovsg = rhovt + d.cdrho * (unksgq[isg] - 1.0 / uqsgc[isg]);
      double uvtx = unknvq[iv][1], vvtx = unknvq[iv][2], evtx = unknvq[iv][3];
      double pvtx = fmax(eps, (g - 1.0) * rhovsg * (evtx - 0.5 * (uvtx * uvtx + vvtx * vvtx)));
      uv[ivsg][0] = uvtx;
      uv[ivsg][1] = vvtx;
      sig[ivsg] = -pvtx;
      const int p = d.ipq[iv * d.nquad + iq];
      double acnx = d.us[p] - uvtx, acny = d.vs[p] - vvtx;
      aj3[ivsg] = sqrt(acnx * acnx + acny * acny) / sdctr;
    }
#pragma unroll
    for (int ivsg = 0; ivsg < 4; ivsg++) {
      const int iv = ipqsg_(isg, ivsg);
      const int p = d.ipq[iv * d.nquad + iq];
      double dux = d.us[p] - uv[ivsg][0];
      double duy = d.vs[p] - uv[ivsg][1];
#pragma unroll
      for (int f = 0; f < 2; f++) {
        double n0, n1, a;
        corner_normal(gq, isg, ivsg, f, n0, n1, a);
        a = a * cWRIE[isg][ivsg][f];
        double deltu = fabs(dux * n0 + duy * n1);
        double murie = rhoct * sdctr + d.cimpd * rhoct * slpdu * deltu;
        double vnau;
        if (aj3[ivsg] < 1.0e12) {
          vnau = 1.0;
        } else {
          // unit jump direction (Getrhslaggauss.f90:10780-10786)
          double acnx = dux, acny = duy;
          double ax, ay;
          if (sqrt(acnx * acnx + acny * acny) < (double)1.e-11f) { ax = (double)1.e-11f; ay = (double)1.e-11f; }
          else { ax = acnx / sqrt(acnx * acnx + acny * acny); ay = acny / sqrt(acnx * acnx + acny * acny); }
          vnau = n0 * ax + n1 * ay;
        }
        double m = murie * a * fabs(vnau);
        double mu0 = m * uv[ivsg][0] + 0.0 * uv[ivsg][1];
        double mu1 = 0.0 * uv[ivsg][0] + m * uv[ivsg][1];
        double sn0 = sig[ivsg] * a * n0 + 0.0 * a * n1;
        double sn1 = 0.0 * a * n0 + sig[ivsg] * a * n1;
        const int slot = f + 2 * (ivsg + 4 * isg);
        d.cf[(0 * 32 + slot) * d.nquad + iq] = m;
        d.cf[(1 * 32 + slot) * d.nquad + iq] = mu0;
        d.cf[(2 * 32 + slot) * d.nquad + iq] = mu1;
        d.cf[(3 * 32 + slot) * d.nquad + iq] = sn0;
        d.cf[(4 * 32 + slot) * d.nquad + iq] = sn1;
      }
    }
  }
}
__global__ void __launch_bounds__(128) k_corner(Dev d) { b_corner(d, blockIdx.x * blockDim.x + threadIdx.x); }

// ---------------------------------------------------------------------------
// Node pass: node sums in the reference's scatter order, 2x2 solve and wall
// conditions (getndvelo_lagsubg, Getrhslaggauss.f90:4465-4545).
// ---------------------------------------------------------------------------
__host__ __device__ void b_node(const Dev &d, int p) {
  if (p >= d.npoin || stopped(d)) return;
  double mn0 = 0.0, mn1 = 0.0, mn2 = 0.0, mn3 = 0.0, mu0 = 0.0, mu1 = 0.0, sn0 = 0.0, sn1 = 0.0;
  const int b = d.node_ptr[p], en = d.node_ptr[p + 1];
  for (int i = b; i < en; i++) {
    const int id = d.node_cf[i];
    double m, a1, a2, a3, a4;
    if (id < 0) {  // triangle corner face: -1 - (it*24 + slot)
      const int t = -1 - id, it = t / 24, slot = t - 24 * it;
      const size_t nt = d.ntria;
      m = d.tcf[(0 * 24 + slot) * nt + it];
      a1 = d.tcf[(1 * 24 + slot) * nt + it];
      a2 = d.tcf[(2 * 24 + slot) * nt + it];
      a3 = d.tcf[(3 * 24 + slot) * nt + it];
      a4 = d.tcf[(4 * 24 + slot) * nt + it];
    } else {
      const int iq = id >> 5, slot = id & 31;
      m = d.cf[(0 * 32 + slot) * d.nquad + iq];
      a1 = d.cf[(1 * 32 + slot) * d.nquad + iq];
      a2 = d.cf[(2 * 32 + slot) * d.nquad + iq];
      a3 = d.cf[(3 * 32 + slot) * d.nquad + iq];
      a4 = d.cf[(4 * 32 + slot) * d.nquad + iq];
    }
    mn0 = mn0 + m;
    mn1 = mn1 + 0.0;
    mn2 = mn2 + 0.0;
    mn3 = mn3 + m;
    mu0 = mu0 + a1;
    mu1 = mu1 + a2;
    sn0 = sn0 + a3;
    sn1 = sn1 + a4;
  }
  const unsigned char mask = d.bcmask[p];
  double us = d.us[p], vs = d.vs[p];
  if (!(mask & 4)) {
    double detma = mn0 * mn3 - mn1 * mn2;
    double i11 = mn3 / detma, i12 = -mn2 / detma, i21 = -mn1 / detma, i22 = mn0 / detma;
    double r1 = mu0 - sn0, r2 = mu1 - sn1;
    us = i11 * r1 + i12 * r2;
    vs = i21 * r1 + i22 * r2;
  }
  if (mask & 1) us = 0.0;
  if (mask & 2) vs = 0.0;
  d.us[p] = us;
  d.vs[p] = vs;
}
__global__ void k_node(Dev d) { b_node(d, blockIdx.x * blockDim.x + threadIdx.x); }

// ---------------------------------------------------------------------------
// RHS pass: corner forces (getndvelo_lagsubg Part III, :4588-4610), face
// integral (rhsifacedg_lagsubgq2, :8501-8748), volume integral
// (rhsdomndg_lagmc_curvquad, Getrhslag.f90:4716-5016, 5x5 Gauss-Lobatto,
// cofactor form) and the Taylor-Green source (rhsdomnsrcdg_lag_curvquad,
// Getrhslag.f90:4070-4251).
// ---------------------------------------------------------------------------
__host__ __device__ void b_rhs(const Dev &d, int iq) {
  if (iq >= d.nquad || stopped(d)) return;
  const int e = iq + d.ntria;
  const double eps = 1.0e-6, g = d.gamlg;
  double xpq[9][2];
  load_quad(d, d.xs, d.ys, iq, xpq);
  double gq[16][3];
  normals_quad(xpq, gq);
  const double rc = d.rc[e], sc = d.sc[e], g19 = d.g19[e], g20 = d.g20[e], g21 = d.g21[e];
  double ul[6] = {0, 0, 0, 0, 0, 0}, p0[6] = {0, 0, 0, 0, 0, 0}, p1[6] = {0, 0, 0, 0, 0, 0},
         el[6] = {0, 0, 0, 0, 0, 0};
  for (int isg = 0; isg < 4; isg++) {
#pragma unroll
    for (int ivsg = 0; ivsg < 4; ivsg++) {
      const int iv = ipqsg_(isg, ivsg);
      const int p = d.ipq[iv * d.nquad + iq];
      const double us0 = d.us[p], us1 = d.vs[p];
      double b[6];
      node_basis(rc, sc, g19, g20, g21, iv, b);
      double n[2][2], a[2], fs[2][2];
#pragma unroll
      for (int f = 0; f < 2; f++) {
        corner_normal(gq, isg, ivsg, f, n[f][0], n[f][1], a[f]);
        a[f] = a[f] * cWMAS[isg][ivsg][f];
        const int slot = f + 2 * (ivsg + 4 * isg);
        const double m = d.cf[(0 * 32 + slot) * d.nquad + iq];
        const double mu0 = d.cf[(1 * 32 + slot) * d.nquad + iq];
        const double mu1 = d.cf[(2 * 32 + slot) * d.nquad + iq];
        const double sn0 = d.cf[(3 * 32 + slot) * d.nquad + iq];
        const double sn1 = d.cf[(4 * 32 + slot) * d.nquad + iq];
        fs[f][0] = sn0 + m * us0 + 0.0 * us1 - mu0;
        fs[f][1] = sn1 + 0.0 * us0 + m * us1 - mu1;
      }
      const double w1 = cWMOM[isg][ivsg], w2 = cWMOM[isg][ivsg];
#pragma unroll
      for (int k = 0; k < NDEG; k++) {
        const double bk = b[k];
        ul[k] = ul[k] + us0 * n[0][0] * a[0] * bk + us1 * n[0][1] * a[0] * bk + us0 * n[1][0] * a[1] * bk +
                us1 * n[1][1] * a[1] * bk;
        p0[k] = p0[k] + fs[0][0] * bk * w1 + fs[1][0] * bk * w2;
        p1[k] = p1[k] + fs[0][1] * bk * w1 + fs[1][1] * bk * w2;
        el[k] = el[k] + us0 * fs[0][0] * bk * w1 + us1 * fs[0][1] * bk * w1 + us0 * fs[1][0] * bk * w2 +
                us1 * fs[1][1] * bk * w2;
      }
    }
  }
  // volume integral
  double u[4][NDEG];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int k = 0; k < NDEG; k++) u[q][k] = Uget(d, d.Us, k, q, e);
  double dbdr[6] = {0.0, 1.0 / 1.0, 0.0, 0.0, 0.0, 0.0}, dbds[6] = {0.0, 0.0, 1.0 / 1.0, 0.0, 0.0, 0.0};
  for (int ig = 0; ig < 25; ig++) {
    const double r = cQ.l25[ig][0], s = cQ.l25[ig][1], wi = cQ.wl25[ig];
    double dr[9], ds[9];
    shp9d(r, s, dr, ds);
    Jac j = jac9(xpq, dr, ds);
    const double djaco = wi;
    dbdr[3] = (r - rc) / (1.0 * 1.0); dbdr[4] = 0.0; dbdr[5] = (s - sc) / 1.0 / 1.0;
    dbds[3] = 0.0; dbds[4] = (s - sc) / (1.0 * 1.0); dbds[5] = (r - rc) / 1.0 / 1.0;
    double b[6];
    b[0] = 1.0; b[1] = (r - rc) / 1.0; b[2] = (s - sc) / 1.0;
    b[3] = 0.5 * b[1] * b[1] - g19;
    b[4] = 0.5 * b[2] * b[2] - g20;
    b[5] = b[1] * b[2] - g21;
    double un[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < NDEG; k++)
#pragma unroll
      for (int q = 0; q < 4; q++) un[q] = un[q] + u[q][k] * b[k];
    const double rhoad = 1.0 / un[0];
    const double uadv = un[1], vadv = un[2], eadv = un[3];
    const double pres = fmax(eps, (g - 1.0) * rhoad * (eadv - 0.5 * (uadv * uadv + vadv * vadv)));
#pragma unroll
    for (int k = 0; k < NDEG; k++) {
      double gd0 = j.ys * dbdr[k] + (-j.yr) * dbds[k];
      double gd1 = (-j.xs) * dbdr[k] + j.xr * dbds[k];
      double f0 = gd0 * uadv + gd1 * vadv;
      double f1 = gd0 * (-pres);
      double f2 = gd1 * (-pres);
      double f3 = (gd0 * uadv + gd1 * vadv) * (-pres);
      ul[k] = ul[k] - f0 * djaco;
      p0[k] = p0[k] - f1 * djaco;
      p1[k] = p1[k] - f2 * djaco;
      el[k] = el[k] - f3 * djaco;
    }
  }
  if (d.ncase == 1) {
    for (int ig = 0; ig < 25; ig++) {
      const double r = cQ.g25[ig][0], s = cQ.g25[ig][1], wi = cQ.w25[ig];
      double shp[9], dr[9], ds[9];
      shp9v(r, s, shp);
      shp9d(r, s, dr, ds);
      Jac j = jac9(xpq, dr, ds);
      double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
      double xg, yg;
      map9(xpq, shp, xg, yg);
      double b[6];
      b[0] = 1.0; b[1] = (r - rc) / 1.0; b[2] = (s - sc) / 1.0;
      b[3] = 0.5 * b[1] * b[1] - g19;
      b[4] = 0.5 * b[2] * b[2] - g20;
      b[5] = b[1] * b[2] - g21;
      double src = 0.25 * cPI * (cos(3.0 * cPI * xg) * cos(cPI * yg) - cos(3.0 * cPI * yg) * cos(cPI * xg)) / (g - 1.0);
#pragma unroll
      for (int k = 0; k < NDEG; k++) el[k] = el[k] + src * b[k] * djaco;
    }
  }
#pragma unroll
  for (int k = 0; k < NDEG; k++) {
    d.rhs[(0 * NDEG + k) * d.ncell + e] = ul[k];
    d.rhs[(1 * NDEG + k) * d.ncell + e] = p0[k];
    d.rhs[(2 * NDEG + k) * d.ncell + e] = p1[k];
    d.rhs[(3 * NDEG + k) * d.ncell + e] = el[k];
  }
}
__global__ void __launch_bounds__(128) k_rhs(Dev d) { b_rhs(d, blockIdx.x * blockDim.x + threadIdx.x); }

// ---------------------------------------------------------------------------
// getdelt_lag (Getrhslag.f90:20600-20716): per-block minima of the CFL and
// volume-change limits; min is exact, so the reduction is order independent.
// ---------------------------------------------------------------------------
// per-quad limits of getdelt_lag: dlen / c (CFL) and V / |dV/dt|
__host__ __device__ void b_dt_values(const Dev &d, int iq, double &dtcfl, double &dtvol) {
  dtcfl = 1e10;
  dtvol = 1e10;
  if (iq >= d.nquad || stopped(d)) return;
  const int e = iq + d.ntria;
  const double eps = 1.0e-6, g = d.gamlg;
  double xp[9][2];
  load_quad(d, d.xn, d.yn, iq, xp);
  const int ed[4][3] = {{0, 4, 1}, {1, 5, 2}, {2, 6, 3}, {3, 7, 0}};
  double dlen = 0.0;
  for (int k = 0; k < 4; k++) {
    const double *a = xp[ed[k][0]], *b = xp[ed[k][1]], *c = xp[ed[k][2]];
    double dl = sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1])) +
                sqrt((b[0] - c[0]) * (b[0] - c[0]) + (b[1] - c[1]) * (b[1] - c[1]));
    if (k == 0 || dl < dlen) dlen = dl;
  }
  const double rhomc = Uget(d, d.Us, 0, 0, e);
  const double uctr = Uget(d, d.Us, 0, 1, e), vctr = Uget(d, d.Us, 0, 2, e), ectr = Uget(d, d.Us, 0, 3, e);
  const double rhoct = 1.0 / rhomc;
  const double pctr = fmax(eps, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
  const double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
  dtcfl = dlen / sdctr;
  dtvol = d.vol[e] / fabs(d.rhs[(0 * NDEG + 0) * d.ncell + e]);
}

// dtfix from the global minima (getdelt_lag :20705-20709, getsolvdg_lag :1766-1773)
__host__ __device__ void b_dt_apply(const Dev &d, double mcfl, double mvol, int ndt) {
  Scalars *S = d.sc_dev;
  double dt = S->dtfix;
  if (ndt == 1) {
    double dtcfl = fmin(1e10, mcfl), dtvol = fmin(1e10, mvol);
    if (S->itime == 1) dt = fmin(d.cfl * dtcfl, 0.1 * dtvol);
    else dt = fmin(fmin(d.cfl * dtcfl, 0.1 * dtvol), 1.01 * dt);
    if ((S->tacru + dt) > d.tend) dt = d.tend - S->tacru;
  }
  S->dtfix = dt;
  S->tacru = S->tacru + dt;
}

// per-block minima; min is exact, so the reduction is order independent
__global__ void k_dt_partial(Dev d) {
  __shared__ double sm_cfl[256], sm_vol[256];
  double dtcfl, dtvol;
  b_dt_values(d, blockIdx.x * blockDim.x + threadIdx.x, dtcfl, dtvol);
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

__global__ void k_dt_final(Dev d, int nblk, int ndt) {
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
  if (threadIdx.x == 0) b_dt_apply(d, sm_cfl[0], sm_vol[0], ndt);
}

// ---------------------------------------------------------------------------
// Stage update (Getrhslag.f90:1789-1904): rhs *= dtfix, M^-1 apply and
// U^(s+1) = alfa U^n + (1 - alfa)(U^(s) + M^-1 rhs).
// ---------------------------------------------------------------------------
__host__ __device__ void b_update(const Dev &d, int e, double alfa) {
  if (e >= d.ncell || stopped(d)) return;
  const double dt = d.sc_dev->dtfix;
  double rhs[NDEG][4];
#pragma unroll
  for (int k = 0; k < NDEG; k++)
#pragma unroll
    for (int q = 0; q < 4; q++) rhs[k][q] = dt * d.rhs[(q * NDEG + k) * d.ncell + e];
  double am[16];
#pragma unroll
  for (int i = 0; i < 16; i++) am[i] = d.amatr[i * d.ncell + e];
  double mm[NDEG][NDEG];
#pragma unroll
  for (int i = 0; i < NDEG; i++)
#pragma unroll
    for (int j = 0; j < NDEG; j++) mm[i][j] = 0.0;
  mm[0][0] = am[15];
  {
    int k = 0;
#pragma unroll
    for (int im = 1; im < NDEG; im++)
#pragma unroll
      for (int jm = im; jm < NDEG; jm++) {
        mm[im][jm] = am[k];
        mm[jm][im] = am[k];
        k++;
      }
  }
  const double oma = 1.0 - alfa;
#pragma unroll
  for (int id = 0; id < NDEG; id++) {
    double unint[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int iu = 0; iu < NDEG; iu++)
#pragma unroll
      for (int q = 0; q < 4; q++) unint[q] = unint[q] + mm[id][iu] * rhs[iu][q];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int idx = (q * NDEG + id) * d.ncell + e;
      d.Us[idx] = alfa * d.Un[idx] + oma * (d.Us[idx] + unint[q]);
    }
  }
}
__global__ void k_update(Dev d, double alfa) { b_update(d, blockIdx.x * blockDim.x + threadIdx.x, alfa); }

// Node motion (Getrhslag.f90:1948-1957)
__host__ __device__ void b_nodes(const Dev &d, int p, double alfa) {
  if (p >= d.npoin || stopped(d)) return;
  const double dt = d.sc_dev->dtfix;
  const double oma = 1.0 - alfa;
  d.xs[p] = alfa * d.xn[p] + oma * (d.xs[p] + dt * d.us[p]);
  d.ys[p] = alfa * d.yn[p] + oma * (d.ys[p] + dt * d.vs[p]);
}
__global__ void k_nodes(Dev d, double alfa) { b_nodes(d, blockIdx.x * blockDim.x + threadIdx.x, alfa); }

// Driver copy-back (dgflo2d.f90:407-423) and exit test (dgflo2d.f90:459)
__host__ __device__ void b_copyback(const Dev &d, int i, int stride) {
  if (stopped(d)) return;
  const int nu = NU * d.ncell;
  for (int t = i; t < nu; t += stride) d.Un[t] = d.Us[t];
  for (int t = i; t < d.npoin; t += stride) {
    d.xn[t] = d.xs[t];
    d.yn[t] = d.ys[t];
  }
}
__global__ void k_copyback(Dev d) { b_copyback(d, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x); }

// itime < 0: advance the device-resident step counter (graph replays)
__host__ __device__ void b_step_begin(const Dev &d, int itime) {
  Scalars *S = d.sc_dev;
  if (S->done) return;
  S->itime = (itime < 0) ? S->itime + 1 : itime;
}
__global__ void k_step_begin(Dev d, int itime) { b_step_begin(d, itime); }

__host__ __device__ void b_step_end(const Dev &d, int check_done) {
  Scalars *S = d.sc_dev;
  if (S->done) return;
  if (check_done && fabs(S->tacru - d.tend) / d.tend <= 1e-11) S->done = 1;
}
__global__ void k_step_end(Dev d, int check_done) { b_step_end(d, check_done); }

__global__ void k_reset_count(Dev d) {
  *d.wcount = 0;
}

// ---------------------------------------------------------------------------
// Initial fields on the device: getgeoel_initial_lag (GetInitial.f90:
// 1484-1694), getgeoelho_initial_lag (:1891-2094), inifield_mcnew
// (Getrhslagmc.f90:3621-3917), getunkno_initial_lag (GetInitial.f90:412-690)
// and the initial sub-cell masses of getrhosubg_averg (Getrhslaggauss.f90:
// 7300-7392), which the corner pass reuses every stage.
// ---------------------------------------------------------------------------
__host__ __device__ void getunkin(const Dev &d, double *unkin, double xg, double yg, int ielem1, double volel,
                         double xc, double yc) {
  const double g = d.gamlg;
  double rhoini = 1.0, uini = 0.0, vini = 0.0, pini = 1.0;
  if (d.ncase == 1) {
    rhoini = 1.0;
    uini = sin(cPI * xg) * cos(cPI * yg);
    vini = -cos(cPI * xg) * sin(cPI * yg);
    pini = 0.25 * (cos(2.0 * cPI * xg) + cos(2.0 * cPI * yg)) + 1.0;
  } else if (d.ncase == 2) {
    uini = -xg; vini = -yg; pini = (g - 1.0);
  } else if (d.ncase == 3) {
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
  if (d.rho0) rhoini *= d.rho0[ielem1 - 1];  // per-cell density factor at fixed p, u, v
  unkin[0] = 1.0;
  unkin[1] = rhoini * uini;
  unkin[2] = rhoini * vini;
  unkin[3] = (pini / rhoini / (g - 1.0) + 0.5 * (uini * uini + vini * vini)) * rhoini;
}

__host__ __device__ void b_init_geo(const Dev &d, int iq) {
  if (iq >= d.nquad) return;
  const int e = iq + d.ntria;
  const double alfrz = 0.0;
  double xp[9][2], shp[9], dr[9], ds[9];
  load_quad(d, d.x0, d.y0, iq, xp);
  double xc, yc;
  shp9v(0.0, 0.0, shp);
  map9(xp, shp, xc, yc);
  double xcent = 0, ycent = 0, xcel = 0, ycel = 0, volel = 0, masel = 0;
  for (int ig = 0; ig < 36; ig++) {
    double r = cQ.g36[ig][0], s = cQ.g36[ig][1], wi = cQ.w36[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map9(xp, shp, xg, yg);
    double rhog = rho_initial(d, e, xc, yc);
    double rcoef = 1.0 - alfrz + alfrz * yg;
    masel = masel + rhog * djaco * rcoef;
    volel = volel + djaco * rcoef;
    xcent = xcent + rhog * r * djaco * rcoef;
    ycent = ycent + rhog * s * djaco * rcoef;
    xcel = xcel + djaco * r * rcoef;
    ycel = ycel + djaco * s * rcoef;
  }
  const double rc = xcent / masel, sc = ycent / masel;
  const double rci = xcel / volel, sci = ycel / volel;
  d.rc[e] = rc;
  d.sc[e] = sc;
  d.vol[e] = volel;
  d.mass[e] = masel;
  // P2 basis offsets
  shp9v(rc, sc, shp);
  map9(xp, shp, xc, yc);
  double bq[6] = {0, 0, 0, 0, 0, 0}, bqi[6] = {0, 0, 0, 0, 0, 0};
  for (int ig = 0; ig < 36; ig++) {
    double r = cQ.g36[ig][0], s = cQ.g36[ig][1], wi = cQ.w36[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map9(xp, shp, xg, yg);
    double rhog = rho_initial(d, e, xc, yc);
    double rcoef = 1.0 - alfrz + alfrz * yg;
    bq[1] = (r - rc) / 1.0;
    bq[2] = (s - sc) / 1.0;
    bq[3] = bq[3] + 0.5 * rhog * bq[1] * bq[1] * djaco * rcoef;
    bq[4] = bq[4] + 0.5 * rhog * bq[2] * bq[2] * djaco * rcoef;
    bq[5] = bq[5] + rhog * bq[1] * bq[2] * djaco * rcoef;
    bqi[1] = (r - rci) / 1.0;
    bqi[2] = (s - sci) / 1.0;
    bqi[3] = bqi[3] + 0.5 * bqi[1] * bqi[1] * djaco * rcoef;
    bqi[4] = bqi[4] + 0.5 * bqi[2] * bqi[2] * djaco * rcoef;
    bqi[5] = bqi[5] + bqi[1] * bqi[2] * djaco * rcoef;
  }
  d.g19[e] = bq[3] / masel;
  d.g20[e] = bq[4] / masel;
  d.g21[e] = bq[5] / masel;
}
__global__ void k_init_geo(Dev d) { b_init_geo(d, blockIdx.x * blockDim.x + threadIdx.x); }

// Initial sub-cell masses (getrhosubg_averg, Getrhslaggauss.f90:7300-7392):
// time invariant, computed once from the initial coordinates.
__host__ __device__ void b_init_msub(const Dev &d, int iq) {
  if (iq >= d.nquad) return;
  double xp[9][2], shp[9], dr[9], ds[9];
  load_quad(d, d.x0, d.y0, iq, xp);
  {
    const double posqc[12][2] = {{-0.5, -1.0}, {0.5, -1.0}, {1.0, -0.5}, {1.0, 0.5}, {0.5, 1.0}, {-0.5, 1.0},
                                 {-1.0, 0.5}, {-1.0, -0.5}, {0.0, -0.5}, {0.5, 0.0}, {0.0, 0.5}, {-0.5, 0.0}};
    const int ipqsc[4][4] = {{0, 8, 11, 7}, {1, 2, 9, 8}, {9, 3, 4, 10}, {11, 10, 5, 6}};
    double xpqc[12][2];
    for (int isc = 0; isc < 12; isc++) {
      shp9v(posqc[isc][0], posqc[isc][1], shp);
      map9(xp, shp, xpqc[isc][0], xpqc[isc][1]);
    }
    double xci, yci;
    shp9v(0.0, 0.0, shp);
    map9(xp, shp, xci, yci);
    for (int isg = 0; isg < 4; isg++) {
      double xs[9][2];
      for (int k = 0; k < 4; k++) {
        xs[k][0] = xp[ipqsg_(isg, k)][0]; xs[k][1] = xp[ipqsg_(isg, k)][1];
        xs[4 + k][0] = xpqc[ipqsc[isg][k]][0]; xs[4 + k][1] = xpqc[ipqsc[isg][k]][1];
      }
      for (int c = 0; c < 2; c++)
        xs[8][c] = -0.25 * (xs[0][c] + xs[1][c] + xs[2][c] + xs[3][c]) + 0.5 * (xs[4][c] + xs[5][c] + xs[6][c] + xs[7][c]);
      double rhs = 0.0;
      for (int ig = 0; ig < 25; ig++) {
        shp9d(cQ.g25[ig][0], cQ.g25[ig][1], dr, ds);
        Jac j = jac9(xs, dr, ds);
        double djaco = cQ.w25[ig] * (j.xr * j.ys - j.yr * j.xs);
        double rhoi = rho_initial(d, iq + d.ntria, xci, yci);
        rhs = rhs + rhoi * 1.0 * djaco;
      }
      d.msub[isg * d.nquad + iq] = rhs;
    }
  }
}
__global__ void k_init_msub(Dev d) { b_init_msub(d, blockIdx.x * blockDim.x + threadIdx.x); }


__host__ __device__ void getinvmat5(double *a, double *x) {
  const int n = 5;
  for (int k = 0; k < n; k++) {
    for (int m = 0; m < k; m++) a[k + n * k] = a[k + n * k] - a[k + n * m] * a[m + n * k];
    double adicv = 1.0 / a[k + n * k];
    for (int i = k + 1; i < n; i++) {
      for (int m = 0; m < k; m++) {
        a[k + n * i] = a[k + n * i] - a[k + n * m] * a[m + n * i];
        a[i + n * k] = a[i + n * k] - a[i + n * m] * a[m + n * k];
      }
      a[i + n * k] = a[i + n * k] * adicv;
    }
  }
  for (int col = 0; col < n; col++) {
    double *xc = x + n * col;
    for (int i = 0; i < n; i++) {
      double c = 0.0;
      for (int j = 0; j < i; j++) c = c + a[i + n * j] * xc[j];
      xc[i] = (i == col ? 1.0 : 0.0) - c;
    }
    for (int i = n - 1; i >= 0; i--) {
      double c = 0.0;
      for (int j = i + 1; j < n; j++) c = c + a[i + n * j] * xc[j];
      xc[i] = (xc[i] - c) / a[i + n * i];
    }
  }
}

__host__ __device__ void b_init_fields(const Dev &d, int iq) {
  if (iq >= d.nquad) return;
  const int e = iq + d.ntria;
  const double alfrz = 0.0;
  double xp[9][2], shp[9], dr[9], ds[9];
  load_quad(d, d.x0, d.y0, iq, xp);
  const double volel = d.vol[e], masel = d.mass[e];
  const double rc = d.rc[e], sc = d.sc[e];
  double unkin[4], rv[4] = {0, 0, 0, 0};
  const double xcel = xp[8][0], ycel = xp[8][1];
  for (int ig = 0; ig < 25; ig++) {
    double r = cQ.g25[ig][0], s = cQ.g25[ig][1], wi = cQ.w25[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map9(xp, shp, xg, yg);
    getunkin(d, unkin, xg, yg, e + 1, volel, xcel, ycel);
    double rcoef = 1.0 - alfrz + alfrz * yg;
    for (int q = 0; q < 4; q++) rv[q] = rv[q] + unkin[q] * djaco * rcoef;
  }
  double u0[4];
  for (int q = 0; q < 4; q++) u0[q] = rv[q] / masel;
  double xc, yc;
  shp9v(rc, sc, shp);
  map9(xp, shp, xc, yc);
  double rhsini[6][4], mmatr[25], matri[25];
  for (int k = 0; k < 6; k++) for (int q = 0; q < 4; q++) rhsini[k][q] = 0.0;
  for (int i = 0; i < 25; i++) mmatr[i] = 0.0;
  double f0 = 0.0;
  for (int ig = 0; ig < 25; ig++) {
    double r = cQ.g25[ig][0], s = cQ.g25[ig][1], wi = cQ.w25[ig];
    shp9v(r, s, shp);
    shp9d(r, s, dr, ds);
    Jac j = jac9(xp, dr, ds);
    double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map9(xp, shp, xg, yg);
    getunkin(d, unkin, xg, yg, e + 1, volel, xc, yc);
    double bq[6];
    bq[0] = 1.0; bq[1] = (r - rc) / 1.0; bq[2] = (s - sc) / 1.0;
    bq[3] = 0.5 * bq[1] * bq[1] - d.g19[e];
    bq[4] = 0.5 * bq[2] * bq[2] - d.g20[e];
    bq[5] = bq[1] * bq[2] - d.g21[e];
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < 6; k++) rhsini[k][q] = rhsini[k][q] + unkin[q] * bq[k] * djaco;
    double rho0 = rho_initial(d, e, xc, yc);
    double rcoef = 1.0 - alfrz + alfrz * yg;
    f0 = f0 + rho0 * djaco * rcoef;
    for (int ix = 0; ix < 5; ix++)
      for (int iy = 0; iy < 5; iy++) mmatr[ix + 5 * iy] = mmatr[ix + 5 * iy] + rho0 * bq[ix + 1] * bq[iy + 1] * djaco * rcoef;
  }
  getinvmat5(mmatr, matri);
  {
    int k = 0;
    for (int im = 0; im < 5; im++)
      for (int jm = im; jm < 5; jm++) d.amatr[(k++) * d.ncell + e] = matri[im + 5 * jm];
    d.amatr[15 * d.ncell + e] = 1.0 / f0;
  }
  for (int q = 0; q < 4; q++) {
    d.Un[(q * NDEG + 0) * d.ncell + e] = u0[q];
    for (int ix = 0; ix < 5; ix++) {
      double acc = 0.0;
      for (int iy = 0; iy < 5; iy++) acc = acc + matri[ix + 5 * iy] * rhsini[iy + 1][q];
      d.Un[(q * NDEG + ix + 1) * d.ncell + e] = acc;
    }
  }
}
__global__ void k_init_fields(Dev d) { b_init_fields(d, blockIdx.x * blockDim.x + threadIdx.x); }

// ---------------------------------------------------------------------------
// Boundary layout conversion: the caller's Fortran arrays unkno(ndegr,nq,nsize)
// and coord/ustar(2,npoin) <-> the device structure of arrays.
// ---------------------------------------------------------------------------
__global__ void k_unkno_in(Dev d, const double *aos, int to_both) {
  const size_t n = (size_t)NU * d.ncell;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const size_t e = t / NU;
    const int qk = (int)(t % NU);  // q*6 + k, coalesced read of the caller's layout
    const double v = aos[t];
    d.Un[qk * (size_t)d.ncell + e] = v;
    if (to_both) d.Us[qk * (size_t)d.ncell + e] = v;
  }
}
__global__ void k_unkno_out(Dev d, double *aos) {
  const size_t n = (size_t)NU * d.ncell;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const size_t e = t / NU;
    const int qk = (int)(t % NU);
    aos[t] = d.Un[qk * (size_t)d.ncell + e];
  }
}
__global__ void k_xy_in(int n, const double *xy, double *x, double *y, double *x2, double *y2) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const double2 v = reinterpret_cast<const double2 *>(xy)[p];
    x[p] = v.x;
    y[p] = v.y;
    if (x2) { x2[p] = v.x; y2[p] = v.y; }
  }
}
__global__ void k_xy_out(int n, double *xy, const double *x, const double *y) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    reinterpret_cast<double2 *>(xy)[p] = make_double2(x[p], y[p]);
}
void launch_unkno_in(const Dev &d, cudaStream_t st, const double *aos, int both) {
  k_unkno_in<<<2368, 256, 0, st>>>(d, aos, both);
}
void launch_unkno_out(const Dev &d, cudaStream_t st, double *aos) { k_unkno_out<<<2368, 256, 0, st>>>(d, aos); }
void launch_xy_in(int n, cudaStream_t st, const double *xy, double *x, double *y, double *x2, double *y2) {
  k_xy_in<<<1184, 256, 0, st>>>(n, xy, x, y, x2, y2);
}
void launch_xy_out(int n, cudaStream_t st, double *xy, const double *x, const double *y) {
  k_xy_out<<<1184, 256, 0, st>>>(n, xy, x, y);
}

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Triangles (6-node, P2 map on the reference triangle (0,0), (1,0), (0,1);
// nodes 1-3 vertices, 4 on edge 1-2, 5 on edge 2-3, 6 on edge 3-1).  The
// same stage as the quads: init (GetInitial.f90 triangle loops), volume
// (getcellvol_lag :1908-2036), corner coefficients (getriem_triasubg3 with
// getrhosubgt_average2, Getrhslaggauss.f90:12201-12945), face integral
// (rhsifacedg_lagsubgt3 :8297-8496), volume integral
// (rhsdomndg_lagmc_curvtria, Getrhslag.f90:4449-4711) and source
// (rhsdomnsrcdg_lag_curvtria :3907-4066).  Triangles are cells 0..ntria-1.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ void shp6v(double r, double s, double *shp) {
  const double c10 = 1.0;
  shp[0] = -(c10 - r - s) * (c10 - 2.0 * (c10 - r - s));
  shp[1] = -r * (c10 - 2.0 * r);
  shp[2] = -s * (c10 - 2.0 * s);
  shp[3] = 4.0 * r * (c10 - r - s);
  shp[4] = 4.0 * r * s;
  shp[5] = 4.0 * s * (c10 - r - s);
}
__host__ __device__ __forceinline__ void shp6d(double r, double s, double *dspr, double *dsps) {
  const double c10 = 1.0;
  dspr[0] = c10 - 4.0 * (c10 - r - s);
  dspr[1] = -1.0 + 4.0 * r;
  dspr[2] = 0.0;
  dspr[3] = 4.0 * (1.0 - 2.0 * r - s);
  dspr[4] = 4.0 * s;
  dspr[5] = -4.0 * s;
  dsps[0] = c10 - 4.0 * (c10 - r - s);
  dsps[1] = 0.0;
  dsps[2] = -1.0 + 4.0 * s;
  dsps[3] = -4.0 * r;
  dsps[4] = 4.0 * r;
  dsps[5] = 4.0 * (1.0 - r - 2.0 * s);
}
__host__ __device__ __forceinline__ Jac jac6(const double (*xp)[2], const double *dspr, const double *dsps) {
  Jac j = {0.0, 0.0, 0.0, 0.0};
  for (int k = 0; k < 6; k++) {
    j.xr = j.xr + dspr[k] * xp[k][0];
    j.xs = j.xs + dsps[k] * xp[k][0];
    j.yr = j.yr + dspr[k] * xp[k][1];
    j.ys = j.ys + dsps[k] * xp[k][1];
  }
  return j;
}
__host__ __device__ __forceinline__ void map6(const double (*xp)[2], const double *shp, double &x, double &y) {
  x = 0.0;
  y = 0.0;
  for (int k = 0; k < 6; k++) {
    x = x + shp[k] * xp[k][0];
    y = y + shp[k] * xp[k][1];
  }
}
__host__ __device__ __forceinline__ void load_tria(const Dev &d, const double *X, const double *Y, int it,
                                                   double (*xp)[2]) {
  for (int k = 0; k < 6; k++) {
    const int p = d.ipt[k * d.ntria + it];
    xp[k][0] = X[p];
    xp[k][1] = Y[p];
  }
}
__host__ __device__ __forceinline__ double xvt(int k) {
  const double v[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
  return v[k];
}
__host__ __device__ __forceinline__ double yvt(int k) {
  const double v[6] = {0.0, 0.0, 1.0, 0.0, 0.5, 0.5};
  return v[k];
}
// sub-triangle vertices (1-based node ids) and face slots (getriem_triasubg3 :12264-12287)
__host__ __device__ __forceinline__ int iptsg(int isg, int ivsg) {
  const int t[12] = {1, 4, 6, 4, 5, 6, 4, 2, 5, 6, 5, 3};
  return t[3 * isg + ivsg];
}
__host__ __device__ __forceinline__ int fntsg(int isg, int k) {
  const int t[24] = {6, 1, 10, -7, -13, 12, 7, 14, 8, 15, 9, 13, -14, 10, 2, 3, 11, -8, 12, -9, -15, 11, 4, 5};
  return t[6 * isg + k];
}
// Taylor basis of a triangle at (r, s), scale 1/2 in r and s
__host__ __device__ __forceinline__ void tri_basis(double rc, double sc, double g19, double g20, double g21,
                                                   double r, double s, double *b) {
  b[0] = 1.0;
  b[1] = (r - rc) / 0.5;
  b[2] = (s - sc) / 0.5;
  b[3] = 0.5 * b[1] * b[1] - g19;
  b[4] = 0.5 * b[2] * b[2] - g20;
  b[5] = b[1] * b[2] - g21;
}

// Initial geometry and DOFs of one triangle (getgeoel_initial_lag :1334-1478,
// getgeoelho_initial_lag :1754-1905, inifield_mcnew Getrhslagmc.f90:3344-3480,
// getunkno_initial_lag GetInitial.f90:190-411) and its initial sub-cell
// masses (getrhosubgt_average2, Getrhslaggauss.f90:12860-12940).
__host__ __device__ void b_tri_init(const Dev &d, int it) {
  if (it >= d.ntria) return;
  const int e = it;
  const double alfrz = 0.0;
  double xp[6][2], shp[6], dspr[6], dsps[6];
  load_tria(d, d.x0, d.y0, it, xp);
  double xc, yc;
  shp6v(1.0 / 3.0, 1.0 / 3.0, shp);
  map6(xp, shp, xc, yc);
  double xcent = 0, ycent = 0, volel = 0, masel = 0;
  for (int ig = 0; ig < 7; ig++) {
    const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
    shp6v(r, s, shp);
    shp6d(r, s, dspr, dsps);
    Jac j = jac6(xp, dspr, dsps);
    const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map6(xp, shp, xg, yg);
    const double rhog = rho_initial(d, e, xc, yc);
    const double rcoef = 1.0 - alfrz + alfrz * yg;
    masel = masel + rhog * djaco * rcoef;
    volel = volel + djaco * rcoef;
    xcent = xcent + rhog * r * djaco * rcoef;
    ycent = ycent + rhog * s * djaco * rcoef;
  }
  const double rc = xcent / masel, sc = ycent / masel;
  d.rc[e] = rc;
  d.sc[e] = sc;
  d.vol[e] = volel;
  d.mass[e] = masel;
  shp6v(rc, sc, shp);
  map6(xp, shp, xc, yc);
  double bt[6] = {0, 0, 0, 0, 0, 0};
  for (int ig = 0; ig < 7; ig++) {
    const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
    shp6v(r, s, shp);
    shp6d(r, s, dspr, dsps);
    Jac j = jac6(xp, dspr, dsps);
    const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map6(xp, shp, xg, yg);
    const double rhog = rho_initial(d, e, xc, yc);
    const double rcoef = 1.0 - alfrz + alfrz * yg;
    bt[1] = (r - rc) / 0.5;
    bt[2] = (s - sc) / 0.5;
    bt[3] = bt[3] + 0.5 * rhog * bt[1] * bt[1] * djaco * rcoef;
    bt[4] = bt[4] + 0.5 * rhog * bt[2] * bt[2] * djaco * rcoef;
    bt[5] = bt[5] + rhog * bt[1] * bt[2] * djaco * rcoef;
  }
  const double g19 = bt[3] / masel, g20 = bt[4] / masel, g21 = bt[5] / masel;
  d.g19[e] = g19;
  d.g20[e] = g20;
  d.g21[e] = g21;
  // cell averages (the centroid of the P2 triangle is the reference's xcel)
  const double xce = (-xp[0][0] - xp[1][0] - xp[2][0] + 4.0 * xp[3][0] + 4.0 * xp[4][0] + 4.0 * xp[5][0]) / 9.0;
  const double yce = (-xp[0][1] - xp[1][1] - xp[2][1] + 4.0 * xp[3][1] + 4.0 * xp[4][1] + 4.0 * xp[5][1]) / 9.0;
  double unkin[4], rv[4] = {0, 0, 0, 0};
  for (int ig = 0; ig < 7; ig++) {
    const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
    shp6v(r, s, shp);
    shp6d(r, s, dspr, dsps);
    Jac j = jac6(xp, dspr, dsps);
    const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map6(xp, shp, xg, yg);
    getunkin(d, unkin, xg, yg, e + 1, volel, xce, yce);
    const double rcoef = 1.0 - alfrz + alfrz * yg;
    for (int q = 0; q < 4; q++) rv[q] = rv[q] + unkin[q] * djaco * rcoef;
  }
  double u0[4];
  for (int q = 0; q < 4; q++) u0[q] = rv[q] / masel;
  // M^-1 and the L2 projection of the higher moments
  double rhsini[6][4], mmatr[25], matri[25];
  for (int k = 0; k < 6; k++) for (int q = 0; q < 4; q++) rhsini[k][q] = 0.0;
  for (int i = 0; i < 25; i++) mmatr[i] = 0.0;
  double f0 = 0.0;
  for (int ig = 0; ig < 7; ig++) {
    const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
    shp6v(r, s, shp);
    shp6d(r, s, dspr, dsps);
    Jac j = jac6(xp, dspr, dsps);
    const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
    double xg, yg;
    map6(xp, shp, xg, yg);
    double b[6];
    tri_basis(rc, sc, g19, g20, g21, r, s, b);
    getunkin(d, unkin, xg, yg, e + 1, volel, xc, yc);
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < 6; k++) rhsini[k][q] = rhsini[k][q] + unkin[q] * b[k] * djaco;
    const double rho0 = rho_initial(d, e, xc, yc);
    const double rcoef = 1.0 - alfrz + alfrz * yg;
    f0 = f0 + rho0 * djaco * rcoef;
    for (int ix = 0; ix < 5; ix++)
      for (int iy = 0; iy < 5; iy++) mmatr[ix + 5 * iy] = mmatr[ix + 5 * iy] + rho0 * b[ix + 1] * b[iy + 1] * djaco * rcoef;
  }
  getinvmat5(mmatr, matri);
  {
    int k = 0;
    for (int im = 0; im < 5; im++)
      for (int jm = im; jm < 5; jm++) d.amatr[(k++) * d.ncell + e] = matri[im + 5 * jm];
    d.amatr[15 * d.ncell + e] = 1.0 / f0;
  }
  for (int q = 0; q < 4; q++) {
    d.Un[(q * NDEG + 0) * d.ncell + e] = u0[q];
    for (int ix = 0; ix < 5; ix++) {
      double acc = 0.0;
      for (int iy = 0; iy < 5; iy++) acc = acc + matri[ix + 5 * iy] * rhsini[iy + 1][q];
      d.Un[(q * NDEG + ix + 1) * d.ncell + e] = acc;
    }
  }
  // initial sub-cell masses: sub-triangles of the initial map, 6-node each
  {
    const double postc[9][2] = {{0.25, 0.0}, {0.75, 0.0}, {0.75, 0.25}, {0.25, 0.75}, {0.0, 0.75},
                                {0.0, 0.25}, {0.25, 0.25}, {0.5, 0.25}, {0.25, 0.5}};
    const int iptsc[4][3] = {{1, 7, 6}, {8, 9, 7}, {2, 3, 8}, {9, 4, 5}};
    double xptic[9][2];
    for (int isc = 0; isc < 9; isc++) {
      shp6v(postc[isc][0], postc[isc][1], shp);
      map6(xp, shp, xptic[isc][0], xptic[isc][1]);
    }
    double xci, yci;
    shp6v(1.0 / 3.0, 1.0 / 3.0, shp);
    map6(xp, shp, xci, yci);
    for (int isg = 0; isg < 4; isg++) {
      double xs[6][2];
      for (int k = 0; k < 3; k++)
        for (int c = 0; c < 2; c++) {
          xs[k][c] = xp[iptsg(isg, k) - 1][c];
          xs[3 + k][c] = xptic[iptsc[isg][k] - 1][c];
        }
      double rhs = 0.0;
      for (int ig = 0; ig < 7; ig++) {
        shp6d(cQ.t7[ig][0], cQ.t7[ig][1], dspr, dsps);
        Jac j = jac6(xs, dspr, dsps);
        const double djaco = 0.5 * cQ.tw7[ig] * (j.xr * j.ys - j.yr * j.xs);
        rhs = rhs + rho_initial(d, e, xci, yci) * 1.0 * djaco;
      }
      d.tmsub[isg * d.ntria + it] = rhs;
    }
  }
}
__global__ void k_tri_init(Dev d) { b_tri_init(d, blockIdx.x * blockDim.x + threadIdx.x); }

// getcellvol_lag triangle loop (Limiterlag.f90:1908-2036): volume and its
// centre in reference coordinates
__host__ __device__ void b_tri_geom(const Dev &d, int it, const double *X, const double *Y) {
  if (it >= d.ntria || stopped(d)) return;
  const double alfrz = 0.0;
  double xp[6][2], shp[6], dspr[6], dsps[6];
  load_tria(d, X, Y, it, xp);
  double rcv = 0, scv = 0, volel = 0;
  for (int ig = 0; ig < 7; ig++) {
    const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
    shp6v(r, s, shp);
    shp6d(r, s, dspr, dsps);
    Jac j = jac6(xp, dspr, dsps);
    double xg, yg;
    map6(xp, shp, xg, yg);
    const double rcoef = 1.0 - alfrz + alfrz * yg;
    const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
    volel = volel + djaco * rcoef;
    rcv = rcv + r * djaco * rcoef;
    scv = scv + s * djaco * rcoef;
  }
  d.vol[it] = volel;
  d.vcx[it] = rcv / volel;
  d.vcy[it] = scv / volel;
  if (!(volel > 0.0)) atomic_or(&d.sc_dev->status, ST_NONPHYS);
}
__global__ void k_tri_geom(Dev d, const double *X, const double *Y) {
  b_tri_geom(d, blockIdx.x * blockDim.x + threadIdx.x, X, Y);
}

// Sub-cell face normals gesgt(3,15) of a triangle (getfnds_lagsms_simpsonhybrid
// :9735-9853 for slots 1-6 and 10-12, getfnds_lagsmsif_hybrid :3432-3520
// for slots 7-9 and 13-15)
__host__ __device__ void normals_tria(const double (*xpt)[2], double (*gt)[3]) {
  const double postc[3][2] = {{0.25, 0.25}, {0.5, 0.25}, {0.25, 0.5}};
  const int ipift[3][3] = {{4, 6, 1}, {5, 4, 2}, {6, 5, 3}};
  double xptv[3][2], shp[6];
  for (int isv = 0; isv < 3; isv++) {
    shp6v(postc[isv][0], postc[isv][1], shp);
    map6(xpt, shp, xptv[isv][0], xptv[isv][1]);
  }
  for (int ifa = 0; ifa < 3; ifa++) {
    double xpf[3][2];
    for (int c = 0; c < 2; c++) {
      xpf[0][c] = xpt[ipift[ifa][0] - 1][c];
      xpf[1][c] = xpt[ipift[ifa][1] - 1][c];
      xpf[2][c] = xptv[ipift[ifa][2] - 1][c];
    }
    for (int end = 0; end < 2; end++) {
      const double r = end == 0 ? -1.0 : 1.0;
      const double dshpr[3] = {-0.5 + r, 0.5 + r, -2.0 * r};
      double dxdr = 0.0, dydr = 0.0;
      for (int k = 0; k < 3; k++) {
        dxdr = dxdr + dshpr[k] * xpf[k][0];
        dydr = dydr + dshpr[k] * xpf[k][1];
      }
      const double djaco = sqrt(dxdr * dxdr + dydr * dydr);
      const double anx = -dydr, any = dxdr;
      const int slot = (end == 0 ? 6 : 12) + ifa;
      gt[slot][0] = anx / sqrt(anx * anx + any * any);
      gt[slot][1] = any / sqrt(anx * anx + any * any);
      gt[slot][2] = djaco * 2.0;
    }
  }
  const double posit[9][2] = {{0, 0}, {1, 0}, {1, 0}, {0, 1}, {0, 1}, {0, 0}, {0.5, 0}, {0.5, 0.5}, {0, 0.5}};
  for (int ig = 0; ig < 9; ig++) {
    double dspr[6], dsps[6];
    shp6d(posit[ig][0], posit[ig][1], dspr, dsps);
    Jac j = jac6(xpt, dspr, dsps);
    const double c11 = j.ys, c12 = -j.yr, c21 = -j.xs, c22 = j.xr;
    const int g1 = ig + 1;
    double vn0, vn1, larea;
    if (g1 == 1 || g1 == 2 || g1 == 7) { vn0 = 0.0; vn1 = -1.0; larea = 1.0; }
    else if (g1 == 3 || g1 == 4 || g1 == 8) { vn0 = sqrt(2.0) * 0.5; vn1 = sqrt(2.0) * 0.5; larea = sqrt(2.0); }
    else { vn0 = -1.0; vn1 = 0.0; larea = 1.0; }
    const double anx = c11 * vn0 + c12 * vn1;
    const double any = c21 * vn0 + c22 * vn1;
    const double v0 = anx * larea, v1 = any * larea;
    const double farea = sqrt(v0 * v0 + v1 * v1);
    const int slot = ig < 6 ? ig : ig + 3;
    gt[slot][0] = anx * larea / farea;
    gt[slot][1] = any * larea / farea;
    gt[slot][2] = farea;
  }
}

// corner-face normal (unit n, weighted area) of face f of vertex ivsg of sub-triangle isg
__host__ __device__ __forceinline__ void tri_corner_normal(const double (*gt)[3], int isg, int ivsg, int f,
                                                           double &n0, double &n1, double &a) {
  const int code = fntsg(isg, 2 * ivsg + f);
  const int slot = (code >= 0 ? code : -code) - 1;
  const double sg = code >= 0 ? 1.0 : -1.0;
  n0 = sg * gt[slot][0];
  n1 = sg * gt[slot][1];
  a = gt[slot][2] * TB().wtri[isg][ivsg][f];
}

// Corner coefficients of one triangle (getriem_triasubg3): per corner face
// (f + 2 (ivsg + 3 isg)) the values m, m u_c, m v_c, sigma.n A (2) into
// tcf, and their per-node sums into tpart (node k of the triangle, in the
// face order above).  Triangles carry no impedance jump term and no cdrho.
__host__ __device__ void b_tri_corner(const Dev &d, int it) {
  if (it >= d.ntria || stopped(d)) return;
  const int e = it;
  const double eps = 1.0e-15, g = d.gamlg, slpdu = (g + 1.0) / 2.0;
  const double rc = d.rc[e], sc = d.sc[e], g19 = d.g19[e], g20 = d.g20[e], g21 = d.g21[e];
  double xpt[6][2];
  load_tria(d, d.xs, d.ys, it, xpt);
  double gt[15][3];
  normals_tria(xpt, gt);
  double u[4][6];
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) u[q][k] = Uget(d, d.Us, k, q, e);
  const double rhomc = u[0][0];
  const double rhoct = 1.0 / rhomc;
  const double pctr = fmax(eps, (g - 1.0) * rhoct * (u[3][0] - 0.5 * (u[1][0] * u[1][0] + u[2][0] * u[2][0])));
  double unknvt[6][4];
  for (int iv = 0; iv < 6; iv++) {
    double b[6];
    tri_basis(rc, sc, g19, g20, g21, xvt(iv), yvt(iv), b);
    for (int q = 0; q < 4; q++) {
      unknvt[iv][q] = 0.0;
      for (int k = 0; k < d.mdegr; k++) unknvt[iv][q] = unknvt[iv][q] + u[q][k] * b[k];
    }
  }
  // sub-cell densities (getrhosubgt_average2): current sub-cell volumes and
  // the harmonic tau mean over each sub-triangle
  double unksgt[4], utsgc[4];
  {
    const double postc[9][2] = {{0.25, 0.0}, {0.75, 0.0}, {0.75, 0.25}, {0.25, 0.75}, {0.0, 0.75},
                                {0.0, 0.25}, {0.25, 0.25}, {0.5, 0.25}, {0.25, 0.5}};
    const int iptsc[4][3] = {{1, 7, 6}, {8, 9, 7}, {2, 3, 8}, {9, 4, 5}};
    double xptc[9][2], shp[6], dspr[6], dsps[6];
    for (int isc = 0; isc < 9; isc++) {
      shp6v(postc[isc][0], postc[isc][1], shp);
      map6(xpt, shp, xptc[isc][0], xptc[isc][1]);
    }
    for (int isg = 0; isg < 4; isg++) {
      double xs[6][2];
      for (int k = 0; k < 3; k++)
        for (int c = 0; c < 2; c++) {
          xs[k][c] = xpt[iptsg(isg, k) - 1][c];
          xs[3 + k][c] = xptc[iptsc[isg][k] - 1][c];
        }
      double f0 = 0.0, masel = 0.0, volel = 0.0;
      for (int ig = 0; ig < 7; ig++) {
        const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
        const double shps[3] = {1.0 - r - s, r, s};
        double rg = 0.0, sg = 0.0;
        for (int k = 0; k < 3; k++) {
          rg = rg + shps[k] * xvt(iptsg(isg, k) - 1);
          sg = sg + shps[k] * yvt(iptsg(isg, k) - 1);
        }
        double b[6];
        tri_basis(rc, sc, g19, g20, g21, rg, sg, b);
        double rhomsg = 0.0;
        for (int k = 0; k < d.mdegr; k++) rhomsg = rhomsg + u[0][k] * b[k];
        if (d.nlimi == 6) rhomsg = rhomc + 1.0 * (rhomsg - rhomc);
        shp6d(r, s, dspr, dsps);
        Jac j = jac6(xs, dspr, dsps);
        const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
        f0 = f0 + djaco;
        masel = masel + 1.0 / rhomsg * djaco;
        volel = volel + djaco;
      }
      unksgt[isg] = 0.0 + (1.0 / f0) * d.tmsub[isg * d.ntria + it];
      utsgc[isg] = volel / masel;
    }
  }
  double part[6][5];
  for (int k = 0; k < 6; k++)
    for (int v = 0; v < 5; v++) part[k][v] = 0.0;
  const double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
  for (int isg = 0; isg < 4; isg++) {
    for (int ivsg = 0; ivsg < 3; ivsg++) {
      const int iv = iptsg(isg, ivsg) - 1;
      const int pn = d.ipt[iv * d.ntria + it];
      const double rhovt = 1.0 / unknvt[iv][0];
      const double rhovsg = rhovt + 1.0 * (unksgt[isg] - 1.0 / utsgc[isg]);
      const double uvtx = unknvt[iv][1], vvtx = unknvt[iv][2], evtx = unknvt[iv][3];
      const double pvtx = fmax(eps, (g - 1.0) * rhovsg * (evtx - 0.5 * (uvtx * uvtx + vvtx * vvtx)));
      double ax = d.us[pn] - uvtx, ay = d.vs[pn] - vvtx;
      const double acnx = ax, acny = ay;
      if (sqrt(acnx * acnx + acny * acny) < (double)1.e-11f) {
        ax = (double)1.e-11f;
        ay = (double)1.e-11f;
      } else {
        ax = ax / sqrt(acnx * acnx + acny * acny);
        ay = ay / sqrt(acnx * acnx + acny * acny);
      }
      const double ajmp = sqrt(acnx * acnx + acny * acny) / sdctr;
      const double dux = d.us[pn] - uvtx, duy = d.vs[pn] - vvtx;
      for (int f = 0; f < 2; f++) {
        double n0, n1, area;
        tri_corner_normal(gt, isg, ivsg, f, n0, n1, area);
        const double deltu = 0.0 * fabs(dux * n0 + duy * n1);
        const double murie = rhoct * sdctr + rhoct * slpdu * deltu;
        const double vnau = (ajmp < 1.0e12) ? 1.0 : n0 * ax + n1 * ay;
        const double m = murie * area * fabs(vnau);
        const double mu0 = m * uvtx + 0.0 * vvtx;
        const double mu1 = 0.0 * uvtx + m * vvtx;
        const double sn0 = -pvtx * area * n0 + 0.0 * area * n1;
        const double sn1 = 0.0 * area * n0 + -pvtx * area * n1;
        const int slot = f + 2 * (ivsg + 3 * isg);
        const size_t nt = d.ntria;
        d.tcf[(0 * 24 + slot) * nt + it] = m;
        d.tcf[(1 * 24 + slot) * nt + it] = mu0;
        d.tcf[(2 * 24 + slot) * nt + it] = mu1;
        d.tcf[(3 * 24 + slot) * nt + it] = sn0;
        d.tcf[(4 * 24 + slot) * nt + it] = sn1;
        part[iv][0] += m;
        part[iv][1] += mu0;
        part[iv][2] += mu1;
        part[iv][3] += sn0;
        part[iv][4] += sn1;
      }
    }
  }
  for (int k = 0; k < 6; k++)
    for (int v = 0; v < 5; v++) d.tpart[(v * 6 + k) * (size_t)d.ntria + it] = part[k][v];
}
__global__ void __launch_bounds__(128) k_tri_corner(Dev d) { b_tri_corner(d, blockIdx.x * blockDim.x + threadIdx.x); }

// RHS of one triangle: corner forces F* = sigma.n A + m (u* - u_c) with the
// new nodal velocity (usn, vsn), face integral, volume integral, source;
// then either the RHS is stored or, with fuse, the M^-1 solve and RK combine.
__host__ __device__ void b_tri_rhs(const Dev &d, int it, const double *usn, const double *vsn, int fuse,
                                   double alfa) {
  if (it >= d.ntria || stopped(d)) return;
  const int e = it;
  const double g = d.gamlg;
  const double rc = d.rc[e], sc = d.sc[e], g19 = d.g19[e], g20 = d.g20[e], g21 = d.g21[e];
  double xpt[6][2];
  load_tria(d, d.xs, d.ys, it, xpt);
  double gt[15][3];
  normals_tria(xpt, gt);
  double bt[6][6];
  for (int iv = 0; iv < 6; iv++) tri_basis(rc, sc, g19, g20, g21, xvt(iv), yvt(iv), bt[iv]);
  double R[4][6];
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) R[q][k] = 0.0;
  const size_t nt = d.ntria;
  // face integral (rhsifacedg_lagsubgt3): mass weights = Riemann weights, unit momentum/energy weights
  for (int isg = 0; isg < 4; isg++) {
    for (int ivsg = 0; ivsg < 3; ivsg++) {
      const int iv = iptsg(isg, ivsg) - 1;
      const int pn = d.ipt[iv * d.ntria + it];
      const double us = usn[pn], vs = vsn[pn];
      double vn[2][3], fs[2][2];
      for (int f = 0; f < 2; f++) {
        tri_corner_normal(gt, isg, ivsg, f, vn[f][0], vn[f][1], vn[f][2]);
        const int slot = f + 2 * (ivsg + 3 * isg);
        const double m = d.tcf[(0 * 24 + slot) * nt + it];
        fs[f][0] = d.tcf[(3 * 24 + slot) * nt + it] + m * us + 0.0 * vs - d.tcf[(1 * 24 + slot) * nt + it];
        fs[f][1] = d.tcf[(4 * 24 + slot) * nt + it] + 0.0 * us + m * vs - d.tcf[(2 * 24 + slot) * nt + it];
      }
      for (int k = 0; k < 6; k++) {
        const double b = bt[iv][k];
        R[0][k] = R[0][k] + us * vn[0][0] * vn[0][2] * b + vs * vn[0][1] * vn[0][2] * b + us * vn[1][0] * vn[1][2] * b +
                  vs * vn[1][1] * vn[1][2] * b;
        R[1][k] = R[1][k] + fs[0][0] * b * 1.0 + fs[1][0] * b * 1.0;
        R[2][k] = R[2][k] + fs[0][1] * b * 1.0 + fs[1][1] * b * 1.0;
        R[3][k] = R[3][k] + us * fs[0][0] * b * 1.0 + vs * fs[0][1] * b * 1.0 + us * fs[1][0] * b * 1.0 +
                  vs * fs[1][1] * b * 1.0;
      }
    }
  }
  // volume integral (cofactor form, 7-point rule, djaco = w/2)
  {
    double dbdr[6] = {0.0, 1.0 / 0.5, 0.0, 0.0, 0.0, 0.0}, dbds[6] = {0.0, 0.0, 1.0 / 0.5, 0.0, 0.0, 0.0};
    for (int ig = 0; ig < 7; ig++) {
      const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
      double dspr[6], dsps[6];
      shp6d(r, s, dspr, dsps);
      Jac j = jac6(xpt, dspr, dsps);
      const double djaco = 0.5 * wi;
      dbdr[3] = (r - rc) / (0.5 * 0.5); dbdr[4] = 0.0; dbdr[5] = (s - sc) / 0.5 / 0.5;
      dbds[3] = 0.0; dbds[4] = (s - sc) / (0.5 * 0.5); dbds[5] = (r - rc) / 0.5 / 0.5;
      double b[6];
      tri_basis(rc, sc, g19, g20, g21, r, s, b);
      double un[4] = {0.0, 0.0, 0.0, 0.0};
      for (int k = 0; k < d.mdegr; k++)
        for (int q = 0; q < 4; q++) un[q] = un[q] + Uget(d, d.Us, k, q, e) * b[k];
      const double rhoad = 1.0 / un[0];
      const double uadv = un[1], vadv = un[2], eadv = un[3];
      const double pres = (g - 1.0) * rhoad * (eadv - 0.5 * (uadv * uadv + vadv * vadv));
      for (int k = 0; k < 6; k++) {
        const double gd0 = j.ys * dbdr[k] + (-j.yr) * dbds[k];
        const double gd1 = (-j.xs) * dbdr[k] + j.xr * dbds[k];
        const double f0 = gd0 * uadv + gd1 * vadv;
        R[0][k] = R[0][k] - f0 * djaco;
        R[1][k] = R[1][k] - gd0 * (-pres) * djaco;
        R[2][k] = R[2][k] - gd1 * (-pres) * djaco;
        R[3][k] = R[3][k] - (gd0 * uadv + gd1 * vadv) * (-pres) * djaco;
      }
    }
  }
  if (d.ncase == 1) {
    // Taylor-Green source with the full P2 basis
    for (int ig = 0; ig < 7; ig++) {
      const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
      double shp[6], dspr[6], dsps[6];
      shp6v(r, s, shp);
      shp6d(r, s, dspr, dsps);
      Jac j = jac6(xpt, dspr, dsps);
      const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
      double xg, yg;
      map6(xpt, shp, xg, yg);
      double b[6];
      tri_basis(rc, sc, g19, g20, g21, r, s, b);
      const double src = 0.25 * cPI * (cos(3.0 * cPI * xg) * cos(cPI * yg) - cos(3.0 * cPI * yg) * cos(cPI * xg)) /
                         (g - 1.0);
      for (int k = 0; k < 6; k++) R[3][k] = R[3][k] + src * b[k] * djaco;
    }
  }
  if (!fuse) {
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < 6; k++) d.rhs[(q * NDEG + k) * d.ncell + e] = R[q][k];
    return;
  }
  // fused stage update (Getrhslag.f90:1789-1904), the arithmetic of b_update
  const double dt = d.sc_dev->dtfix;
  double am[16];
  for (int i = 0; i < 16; i++) am[i] = d.amatr[i * d.ncell + e];
  double mm[NDEG][NDEG];
  for (int i = 0; i < NDEG; i++)
    for (int jj = 0; jj < NDEG; jj++) mm[i][jj] = 0.0;
  mm[0][0] = am[15];
  {
    int k = 0;
    for (int im = 1; im < NDEG; im++)
      for (int jm = im; jm < NDEG; jm++) {
        mm[im][jm] = am[k];
        mm[jm][im] = am[k];
        k++;
      }
  }
  const double oma = 1.0 - alfa;
  for (int id = 0; id < NDEG; id++) {
    double unint[4] = {0.0, 0.0, 0.0, 0.0};
    for (int iu = 0; iu < NDEG; iu++)
      for (int q = 0; q < 4; q++) unint[q] = unint[q] + mm[id][iu] * (dt * R[q][iu]);
    for (int q = 0; q < 4; q++) {
      const int idx = (q * NDEG + id) * d.ncell + e;
      d.Us[idx] = alfa * d.Un[idx] + oma * (d.Us[idx] + unint[q]);
    }
  }
}
__global__ void __launch_bounds__(128) k_tri_rhs(Dev d, const double *usn, const double *vsn, int fuse, double alfa) {
  b_tri_rhs(d, blockIdx.x * blockDim.x + threadIdx.x, usn, vsn, fuse, alfa);
}

void set_tables(const QuadTables &q, cudaStream_t st) {
  Tables t;
  t.q = q;
  const double t1[4][4][2] = {
      {{4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}, {1.0, 1.0}, {8.0 / 3.0, 4.0 / 3.0}},
      {{8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}, {1.0, 1.0}},
      {{1.0, 1.0}, {8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}},
      {{4.0 / 3.0, 8.0 / 3.0}, {1.0, 1.0}, {8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}}};
  const double t2[4][4][2] = {
      {{4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 0.0}, {0.0, 0.0}, {0.0, 4.0 / 3.0}},
      {{0.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 0.0 / 3.0}, {0.0, 0.0}},
      {{0.0, 0.0}, {0.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 0.0 / 3.0}},
      {{4.0 / 3.0, 0.0 / 3.0}, {0.0, 0.0}, {0.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}}};
  const double t3[4][4] = {{1, 1, 0, 1}, {1, 1, 1, 0}, {0, 1, 1, 1}, {1, 0, 1, 1}};
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      t.wmom[a][b] = t3[a][b];
      for (int f = 0; f < 2; f++) {
        t.wrie[a][b][f] = 0.25 * t1[a][b][f];
        t.wmas[a][b][f] = 0.25 * t2[a][b][f];
      }
    }
  const double t4[4][3][2] = {{{4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}, {8.0 / 3.0, 4.0 / 3.0}},
                              {{8.0 / 3.0, 8.0 / 3.0}, {8.0 / 3.0, 8.0 / 3.0}, {8.0 / 3.0, 8.0 / 3.0}},
                              {{8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}, {4.0 / 3.0, 8.0 / 3.0}},
                              {{4.0 / 3.0, 8.0 / 3.0}, {8.0 / 3.0, 4.0 / 3.0}, {4.0 / 6.0, 4.0 / 6.0}}};
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 3; b++)
      for (int f = 0; f < 2; f++) t.wtri[a][b][f] = 0.25 * t4[a][b][f];
  hT = t;
  if (st) cudaMemcpyToSymbolAsync(cT, &t, sizeof(Tables), 0, cudaMemcpyHostToDevice, st);
}

static inline int nblk(int n, int b) { return (n + b - 1) / b; }

#define LAUNCH_FAMILY(name) (name)

void launch_geom(const Dev &d, cudaStream_t st, const double *X, const double *Y) {
  k_geom<<<nblk(d.nquad, 128), 128, 0, st>>>(d, X, Y);
}
void launch_center_geom(const Dev &d, cudaStream_t st) {
  k_center_geom<<<nblk(d.nquad, 256), 256, 0, st>>>(d);
}
void launch_reset_count(const Dev &d, cudaStream_t st) { k_reset_count<<<1, 1, 0, st>>>(d); }
void launch_tri_init(const Dev &d, cudaStream_t st) {
  if (d.ntria) k_tri_init<<<nblk(d.ntria, 128), 128, 0, st>>>(d);
}
void launch_tri_geom(const Dev &d, cudaStream_t st, const double *X, const double *Y) {
  if (d.ntria) k_tri_geom<<<nblk(d.ntria, 128), 128, 0, st>>>(d, X, Y);
}
void launch_tri_corner(const Dev &d, cudaStream_t st) {
  if (d.ntria) k_tri_corner<<<nblk(d.ntria, 128), 128, 0, st>>>(d);
}
// ---------------------------------------------------------------------------
// Adjoint of the triangle passes (reverse mode of b_tri_corner and b_tri_rhs;
// the fused update, node motion and gathers are shared with the quads).
// ---------------------------------------------------------------------------

// transpose of normals_tria: lgt[slot] = (adjoint of n0, n1, A) -> lxpt
__host__ __device__ void normals_tria_T(const double (*xpt)[2], const double (*lgt)[3], double (*lxpt)[2]) {
  const double postc[3][2] = {{0.25, 0.25}, {0.5, 0.25}, {0.25, 0.5}};
  const int ipift[3][3] = {{4, 6, 1}, {5, 4, 2}, {6, 5, 3}};
  double xptv[3][2], shpv[3][6];
  for (int isv = 0; isv < 3; isv++) {
    shp6v(postc[isv][0], postc[isv][1], shpv[isv]);
    map6(xpt, shpv[isv], xptv[isv][0], xptv[isv][1]);
  }
  double lxptv[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  for (int ifa = 0; ifa < 3; ifa++) {
    double xpf[3][2];
    for (int c = 0; c < 2; c++) {
      xpf[0][c] = xpt[ipift[ifa][0] - 1][c];
      xpf[1][c] = xpt[ipift[ifa][1] - 1][c];
      xpf[2][c] = xptv[ipift[ifa][2] - 1][c];
    }
    for (int end = 0; end < 2; end++) {
      const double r = end == 0 ? -1.0 : 1.0;
      const double dshpr[3] = {-0.5 + r, 0.5 + r, -2.0 * r};
      double a = 0.0, b = 0.0;  // dx/dr, dy/dr
      for (int k = 0; k < 3; k++) {
        a += dshpr[k] * xpf[k][0];
        b += dshpr[k] * xpf[k][1];
      }
      // n = (-b, a) / J, A = 2 J, J = |(a, b)|
      const int slot = (end == 0 ? 6 : 12) + ifa;
      const double J = sqrt(a * a + b * b), iJ = 1.0 / J, iJ3 = iJ * iJ * iJ;
      const double t = lgt[slot][0] * a + lgt[slot][1] * b;
      const double la = b * iJ3 * t + 2.0 * lgt[slot][2] * a * iJ;
      const double lb = -a * iJ3 * t + 2.0 * lgt[slot][2] * b * iJ;
      for (int k = 0; k < 3; k++) {
        const double lx = la * dshpr[k], ly = lb * dshpr[k];
        if (k < 2) {
          lxpt[ipift[ifa][k] - 1][0] += lx;
          lxpt[ipift[ifa][k] - 1][1] += ly;
        } else {
          lxptv[ipift[ifa][2] - 1][0] += lx;
          lxptv[ipift[ifa][2] - 1][1] += ly;
        }
      }
    }
  }
  for (int isv = 0; isv < 3; isv++)
    for (int k = 0; k < 6; k++) {
      lxpt[k][0] += lxptv[isv][0] * shpv[isv][k];
      lxpt[k][1] += lxptv[isv][1] * shpv[isv][k];
    }
  const double posit[9][2] = {{0, 0}, {1, 0}, {1, 0}, {0, 1}, {0, 1}, {0, 0}, {0.5, 0}, {0.5, 0.5}, {0, 0.5}};
  for (int ig = 0; ig < 9; ig++) {
    double dspr[6], dsps[6];
    shp6d(posit[ig][0], posit[ig][1], dspr, dsps);
    Jac j = jac6(xpt, dspr, dsps);
    const int g1 = ig + 1;
    double vn0, vn1, larea;
    if (g1 == 1 || g1 == 2 || g1 == 7) { vn0 = 0.0; vn1 = -1.0; larea = 1.0; }
    else if (g1 == 3 || g1 == 4 || g1 == 8) { vn0 = sqrt(2.0) * 0.5; vn1 = sqrt(2.0) * 0.5; larea = sqrt(2.0); }
    else { vn0 = -1.0; vn1 = 0.0; larea = 1.0; }
    // v = larea (ys vn0 - yr vn1, -xs vn0 + xr vn1); n = v / |v|, A = |v|
    const double v0 = larea * (j.ys * vn0 - j.yr * vn1), v1 = larea * (-j.xs * vn0 + j.xr * vn1);
    const double A = sqrt(v0 * v0 + v1 * v1), iA = 1.0 / A;
    const double n0 = v0 * iA, n1 = v1 * iA;
    const int slot = ig < 6 ? ig : ig + 3;
    const double ln0 = lgt[slot][0], ln1 = lgt[slot][1], lA = lgt[slot][2];
    const double dot = ln0 * n0 + ln1 * n1;
    const double lv0 = (ln0 - n0 * dot) * iA + lA * n0, lv1 = (ln1 - n1 * dot) * iA + lA * n1;
    const double lys = larea * lv0 * vn0, lyr = -larea * lv0 * vn1;
    const double lxs = -larea * lv1 * vn0, lxr = larea * lv1 * vn1;
    for (int k = 0; k < 6; k++) {
      lxpt[k][0] += lxr * dspr[k] + lxs * dsps[k];
      lxpt[k][1] += lyr * dspr[k] + lys * dsps[k];
    }
  }
}

// transpose of the cell-average sound speed of the triangle passes (eps 1e-15)
__host__ __device__ __forceinline__ void tri_centre_T(const double u[4][6], double g, double lrho_in, double lsd,
                                                      double lu[4][6]) {
  const double eps = 1.0e-15;
  const double rhoct = 1.0 / u[0][0];
  const double kin = u[3][0] - 0.5 * (u[1][0] * u[1][0] + u[2][0] * u[2][0]);
  const double pe = (g - 1.0) * rhoct * kin;
  const double pctr = fmax(eps, pe);
  const double se = g * pctr / rhoct;
  const double sdctr = sqrt(fmax(eps, se));
  double lrho = lrho_in, lp = 0.0;
  if (se > eps) {
    const double lse = lsd / (2.0 * sdctr);
    lp += lse * g / rhoct;
    lrho += -lse * g * pctr / (rhoct * rhoct);
  }
  if (pe > eps) {
    lrho += lp * (g - 1.0) * kin;
    lu[3][0] += lp * (g - 1.0) * rhoct;
    lu[1][0] -= lp * (g - 1.0) * rhoct * u[1][0];
    lu[2][0] -= lp * (g - 1.0) * rhoct * u[2][0];
  }
  lu[0][0] += -lrho * rhoct * rhoct;
}

// Reverse of b_tri_rhs: lR (RHS adjoint of the cell) -> adjoints of the cell
// DOFs, the node coordinates, the new nodal velocity (tbuf v = 0, 1, 4, 5)
// and the corner coefficients (ltcf).
__host__ __device__ void a_tri_rhs(const Dev &d, const Adj &a, int it) {
  if (it >= d.ntria) return;
  const int e = it;
  const double g = d.gamlg;
  const double rc = d.rc[e], sc = d.sc[e], g19 = d.g19[e], g20 = d.g20[e], g21 = d.g21[e];
  const size_t nt = d.ntria;
  double xpt[6][2];
  load_tria(d, d.xs, d.ys, it, xpt);
  double gt[15][3];
  normals_tria(xpt, gt);
  double u[4][6], lR[4][6], lu[4][6];
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) {
      u[q][k] = Uget(d, d.Us, k, q, e);
      lR[q][k] = a.lR[(q * NDEG + k) * d.ncell + e];
      lu[q][k] = 0.0;
    }
  double lxpt[6][2], lun[6][2];
  for (int k = 0; k < 6; k++) { lxpt[k][0] = lxpt[k][1] = 0.0; lun[k][0] = lun[k][1] = 0.0; }
  double lgt[15][3];
  for (int sl = 0; sl < 15; sl++) lgt[sl][0] = lgt[sl][1] = lgt[sl][2] = 0.0;
  // face integral
  for (int isg = 0; isg < 4; isg++)
    for (int ivsg = 0; ivsg < 3; ivsg++) {
      const int iv = iptsg(isg, ivsg) - 1;
      const int pn = d.ipt[iv * d.ntria + it];
      const double us = d.us_new[pn], vs = d.vs_new[pn];
      double bt[6];
      tri_basis(rc, sc, g19, g20, g21, xvt(iv), yvt(iv), bt);
      double Lq[4];
      for (int q = 0; q < 4; q++) {
        Lq[q] = 0.0;
        for (int k = 0; k < 6; k++) Lq[q] += lR[q][k] * bt[k];
      }
      for (int f = 0; f < 2; f++) {
        const int code = fntsg(isg, 2 * ivsg + f);
        const int slot = (code >= 0 ? code : -code) - 1;
        const double sg = code >= 0 ? 1.0 : -1.0;
        const double w = TB().wtri[isg][ivsg][f];
        const double n0 = sg * gt[slot][0], n1 = sg * gt[slot][1], ar = gt[slot][2] * w;
        const int cs = f + 2 * (ivsg + 3 * isg);
        const double m = d.tcf[(0 * 24 + cs) * nt + it];
        const double fs0 = d.tcf[(3 * 24 + cs) * nt + it] + m * us - d.tcf[(1 * 24 + cs) * nt + it];
        const double fs1 = d.tcf[(4 * 24 + cs) * nt + it] + m * vs - d.tcf[(2 * 24 + cs) * nt + it];
        const double lfs0 = Lq[1] + Lq[3] * us, lfs1 = Lq[2] + Lq[3] * vs;
        lun[iv][0] += Lq[0] * n0 * ar + Lq[3] * fs0 + lfs0 * m;
        lun[iv][1] += Lq[0] * n1 * ar + Lq[3] * fs1 + lfs1 * m;
        a.ltcf[(0 * 24 + cs) * nt + it] = lfs0 * us + lfs1 * vs;
        a.ltcf[(1 * 24 + cs) * nt + it] = -lfs0;
        a.ltcf[(2 * 24 + cs) * nt + it] = -lfs1;
        a.ltcf[(3 * 24 + cs) * nt + it] = lfs0;
        a.ltcf[(4 * 24 + cs) * nt + it] = lfs1;
        lgt[slot][0] += sg * Lq[0] * us * ar;
        lgt[slot][1] += sg * Lq[0] * vs * ar;
        lgt[slot][2] += w * Lq[0] * (us * n0 + vs * n1);
      }
    }
  // volume integral (cofactor form, 7-point rule)
  for (int ig = 0; ig < 7; ig++) {
    const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
    double dspr[6], dsps[6];
    shp6d(r, s, dspr, dsps);
    Jac j = jac6(xpt, dspr, dsps);
    const double djaco = 0.5 * wi;
    double dbdr[6] = {0.0, 1.0 / 0.5, 0.0, 0.0, 0.0, 0.0}, dbds[6] = {0.0, 0.0, 1.0 / 0.5, 0.0, 0.0, 0.0};
    dbdr[3] = (r - rc) / (0.5 * 0.5); dbdr[5] = (s - sc) / 0.5 / 0.5;
    dbds[4] = (s - sc) / (0.5 * 0.5); dbds[5] = (r - rc) / 0.5 / 0.5;
    double b[6];
    tri_basis(rc, sc, g19, g20, g21, r, s, b);
    double un[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < d.mdegr; k++)
      for (int q = 0; q < 4; q++) un[q] += u[q][k] * b[k];
    const double rhoad = 1.0 / un[0];
    const double ke = un[3] - 0.5 * (un[1] * un[1] + un[2] * un[2]);
    const double pres = (g - 1.0) * rhoad * ke;
    double lp = 0.0, lua = 0.0, lva = 0.0, lxr = 0.0, lxs = 0.0, lyr = 0.0, lys = 0.0;
    for (int k = 0; k < 6; k++) {
      const double gd0 = j.ys * dbdr[k] - j.yr * dbds[k];
      const double gd1 = -j.xs * dbdr[k] + j.xr * dbds[k];
      const double f0 = gd0 * un[1] + gd1 * un[2];
      const double lf0 = -lR[0][k] * djaco + lR[3][k] * pres * djaco;
      lp += djaco * (lR[1][k] * gd0 + lR[2][k] * gd1 + lR[3][k] * f0);
      const double lgd0 = lR[1][k] * pres * djaco + lf0 * un[1];
      const double lgd1 = lR[2][k] * pres * djaco + lf0 * un[2];
      lua += lf0 * gd0;
      lva += lf0 * gd1;
      lys += lgd0 * dbdr[k];
      lyr -= lgd0 * dbds[k];
      lxs -= lgd1 * dbdr[k];
      lxr += lgd1 * dbds[k];
    }
    const double lrhoad = lp * (g - 1.0) * ke, lke = lp * (g - 1.0) * rhoad;
    const double lq[4] = {-lrhoad * rhoad * rhoad, lua - lke * un[1], lva - lke * un[2], lke};
    for (int k = 0; k < d.mdegr; k++)
      for (int q = 0; q < 4; q++) lu[q][k] += lq[q] * b[k];
    for (int k = 0; k < 6; k++) {
      lxpt[k][0] += lxr * dspr[k] + lxs * dsps[k];
      lxpt[k][1] += lyr * dspr[k] + lys * dsps[k];
    }
  }
  if (d.ncase == 1) {
    const double C = 0.25 * cPI / (g - 1.0);
    for (int ig = 0; ig < 7; ig++) {
      const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
      double shp[6], dspr[6], dsps[6];
      shp6v(r, s, shp);
      shp6d(r, s, dspr, dsps);
      Jac j = jac6(xpt, dspr, dsps);
      const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
      double xg, yg;
      map6(xpt, shp, xg, yg);
      double b[6];
      tri_basis(rc, sc, g19, g20, g21, r, s, b);
      double Ls = 0.0;
      for (int k = 0; k < 6; k++) Ls += lR[3][k] * b[k];
      const double c1x = cospi(xg), c1y = cospi(yg), s1x = sinpi(xg), s1y = sinpi(yg);
      const double c3x = cospi(3.0 * xg), c3y = cospi(3.0 * yg), s3x = sinpi(3.0 * xg), s3y = sinpi(3.0 * yg);
      const double src = C * (c3x * c1y - c3y * c1x);
      const double dsx = C * cPI * (-3.0 * s3x * c1y + c3y * s1x);
      const double dsy = C * cPI * (-c3x * s1y + 3.0 * s3y * c1x);
      const double ldj = Ls * src * 0.5 * wi;
      const double lxg = Ls * djaco * dsx, lyg = Ls * djaco * dsy;
      const double lxr = ldj * j.ys, lys = ldj * j.xr, lyr = -ldj * j.xs, lxs = -ldj * j.yr;
      for (int k = 0; k < 6; k++) {
        lxpt[k][0] += lxr * dspr[k] + lxs * dsps[k] + lxg * shp[k];
        lxpt[k][1] += lyr * dspr[k] + lys * dsps[k] + lyg * shp[k];
      }
    }
  }
  normals_tria_T(xpt, lgt, lxpt);
  for (int k = 0; k < 6; k++) {
    a.tbuf[(0 * 6 + k) * nt + it] = lxpt[k][0];
    a.tbuf[(1 * 6 + k) * nt + it] = lxpt[k][1];
    a.tbuf[(2 * 6 + k) * nt + it] = 0.0;
    a.tbuf[(3 * 6 + k) * nt + it] = 0.0;
    a.tbuf[(4 * 6 + k) * nt + it] = lun[k][0];
    a.tbuf[(5 * 6 + k) * nt + it] = lun[k][1];
  }
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) a.lU[(q * NDEG + k) * d.ncell + e] += lu[q][k];
}
__global__ void __launch_bounds__(128) k_a_tri_rhs(Dev d, Adj a) { a_tri_rhs(d, a, blockIdx.x * blockDim.x + threadIdx.x); }

// Reverse of b_tri_corner (its normal branch: no impedance jump term, unit
// jump factor): the adjoint of each corner coefficient is the RHS pass's
// (ltcf) plus the node-sum adjoint lS of its node; -> adjoints of the cell
// DOFs and node coordinates (tbuf v = 0, 1; the triangle corners do not read
// the previous nodal velocity).
__host__ __device__ void a_tri_corner(const Dev &d, const Adj &a, int it) {
  if (it >= d.ntria) return;
  const int e = it;
  const double eps = 1.0e-15, g = d.gamlg;
  const double rc = d.rc[e], sc = d.sc[e], g19 = d.g19[e], g20 = d.g20[e], g21 = d.g21[e];
  const size_t nt = d.ntria, np = d.npoin;
  double xpt[6][2];
  load_tria(d, d.xs, d.ys, it, xpt);
  double gt[15][3];
  normals_tria(xpt, gt);
  double u[4][6], lu[4][6];
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) {
      u[q][k] = Uget(d, d.Us, k, q, e);
      lu[q][k] = 0.0;
    }
  const double rhomc = u[0][0], rhoct = 1.0 / rhomc;
  const double pctr = fmax(eps, (g - 1.0) * rhoct * (u[3][0] - 0.5 * (u[1][0] * u[1][0] + u[2][0] * u[2][0])));
  const double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
  double bt[6][6], unknvt[6][4];
  for (int iv = 0; iv < 6; iv++) {
    tri_basis(rc, sc, g19, g20, g21, xvt(iv), yvt(iv), bt[iv]);
    for (int q = 0; q < 4; q++) {
      unknvt[iv][q] = 0.0;
      for (int k = 0; k < d.mdegr; k++) unknvt[iv][q] += u[q][k] * bt[iv][k];
    }
  }
  // sub-cell areas f0 (= volel) and harmonic masses masel, as in the forward pass
  const double postc[9][2] = {{0.25, 0.0}, {0.75, 0.0}, {0.75, 0.25}, {0.25, 0.75}, {0.0, 0.75},
                              {0.0, 0.25}, {0.25, 0.25}, {0.5, 0.25}, {0.25, 0.5}};
  const int iptsc[4][3] = {{1, 7, 6}, {8, 9, 7}, {2, 3, 8}, {9, 4, 5}};
  double shpc[9][6], xptc[9][2];
  for (int isc = 0; isc < 9; isc++) {
    shp6v(postc[isc][0], postc[isc][1], shpc[isc]);
    map6(xpt, shpc[isc], xptc[isc][0], xptc[isc][1]);
  }
  double f0v[4], masv[4];
  for (int isg = 0; isg < 4; isg++) {
    double xs[6][2];
    for (int k = 0; k < 3; k++)
      for (int c = 0; c < 2; c++) {
        xs[k][c] = xpt[iptsg(isg, k) - 1][c];
        xs[3 + k][c] = xptc[iptsc[isg][k] - 1][c];
      }
    double f0 = 0.0, masel = 0.0;
    for (int ig = 0; ig < 7; ig++) {
      const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
      const double shps[3] = {1.0 - r - s, r, s};
      double rg = 0.0, sgp = 0.0;
      for (int k = 0; k < 3; k++) {
        rg += shps[k] * xvt(iptsg(isg, k) - 1);
        sgp += shps[k] * yvt(iptsg(isg, k) - 1);
      }
      double b[6];
      tri_basis(rc, sc, g19, g20, g21, rg, sgp, b);
      double tau = 0.0;
      for (int k = 0; k < d.mdegr; k++) tau += u[0][k] * b[k];
      double dspr[6], dsps[6];
      shp6d(r, s, dspr, dsps);
      Jac j = jac6(xs, dspr, dsps);
      const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
      f0 += djaco;
      masel += djaco / tau;
    }
    f0v[isg] = f0;
    masv[isg] = masel;
  }
  // corner coefficients, reversed
  double lrho = 0.0, lsd = 0.0, lf0[4] = {0, 0, 0, 0}, lmas[4] = {0, 0, 0, 0};
  double lunk[6][4];
  for (int iv = 0; iv < 6; iv++)
    for (int q = 0; q < 4; q++) lunk[iv][q] = 0.0;
  double lgt[15][3];
  for (int sl = 0; sl < 15; sl++) lgt[sl][0] = lgt[sl][1] = lgt[sl][2] = 0.0;
  for (int isg = 0; isg < 4; isg++) {
    const double tms = d.tmsub[isg * d.ntria + it];
    for (int ivsg = 0; ivsg < 3; ivsg++) {
      const int iv = iptsg(isg, ivsg) - 1;
      const int pn = d.ipt[iv * d.ntria + it];
      const double rhovt = 1.0 / unknvt[iv][0];
      const double rhovsg = rhovt + (tms / f0v[isg] - masv[isg] / f0v[isg]);
      const double uv = unknvt[iv][1], vv = unknvt[iv][2], ev = unknvt[iv][3];
      const double kev = ev - 0.5 * (uv * uv + vv * vv);
      const double pe = (g - 1.0) * rhovsg * kev;
      const double pv = fmax(eps, pe);
      double lpv = 0.0;
      for (int f = 0; f < 2; f++) {
        const int code = fntsg(isg, 2 * ivsg + f);
        const int slot = (code >= 0 ? code : -code) - 1;
        const double sg = code >= 0 ? 1.0 : -1.0;
        const double w = TB().wtri[isg][ivsg][f];
        const double n0 = sg * gt[slot][0], n1 = sg * gt[slot][1], ar = gt[slot][2] * w;
        const int cs = f + 2 * (ivsg + 3 * isg);
        double L[5];
        for (int v = 0; v < 5; v++) L[v] = a.ltcf[(v * 24 + cs) * nt + it] + a.lS[v * np + pn];
        const double m = rhoct * sdctr * ar;
        // (m, m u, m v, -p A n0, -p A n1)
        const double lm = L[0] + L[1] * uv + L[2] * vv;
        lunk[iv][1] += L[1] * m;
        lunk[iv][2] += L[2] * m;
        lpv += -ar * (L[3] * n0 + L[4] * n1);
        double lar = -pv * (L[3] * n0 + L[4] * n1) + lm * rhoct * sdctr;
        lrho += lm * sdctr * ar;
        lsd += lm * rhoct * ar;
        lgt[slot][0] += sg * (-L[3] * pv * ar);
        lgt[slot][1] += sg * (-L[4] * pv * ar);
        lgt[slot][2] += w * lar;
      }
      if (pe > eps) {
        const double lrs = lpv * (g - 1.0) * kev, lke = lpv * (g - 1.0) * rhovsg;
        lunk[iv][3] += lke;
        lunk[iv][1] -= lke * uv;
        lunk[iv][2] -= lke * vv;
        // rhovsg = 1/unknvt0 + (tmsub - masel) / f0
        lunk[iv][0] += -lrs * rhovt * rhovt;
        lf0[isg] += -lrs * (tms - masv[isg]) / (f0v[isg] * f0v[isg]);
        lmas[isg] += -lrs / f0v[isg];
      }
    }
  }
  for (int iv = 0; iv < 6; iv++)
    for (int q = 0; q < 4; q++)
      for (int k = 0; k < d.mdegr; k++) lu[q][k] += lunk[iv][q] * bt[iv][k];
  tri_centre_T(u, g, lrho, lsd, lu);
  // sub-cell quadratures, reversed
  double lxpt[6][2], lxptc[9][2];
  for (int k = 0; k < 6; k++) lxpt[k][0] = lxpt[k][1] = 0.0;
  for (int k = 0; k < 9; k++) lxptc[k][0] = lxptc[k][1] = 0.0;
  for (int isg = 0; isg < 4; isg++) {
    double xs[6][2], lxs[6][2];
    for (int k = 0; k < 3; k++)
      for (int c = 0; c < 2; c++) {
        xs[k][c] = xpt[iptsg(isg, k) - 1][c];
        xs[3 + k][c] = xptc[iptsc[isg][k] - 1][c];
      }
    for (int k = 0; k < 6; k++) lxs[k][0] = lxs[k][1] = 0.0;
    for (int ig = 0; ig < 7; ig++) {
      const double r = cQ.t7[ig][0], s = cQ.t7[ig][1], wi = cQ.tw7[ig];
      const double shps[3] = {1.0 - r - s, r, s};
      double rg = 0.0, sgp = 0.0;
      for (int k = 0; k < 3; k++) {
        rg += shps[k] * xvt(iptsg(isg, k) - 1);
        sgp += shps[k] * yvt(iptsg(isg, k) - 1);
      }
      double b[6];
      tri_basis(rc, sc, g19, g20, g21, rg, sgp, b);
      double tau = 0.0;
      for (int k = 0; k < d.mdegr; k++) tau += u[0][k] * b[k];
      double dspr[6], dsps[6];
      shp6d(r, s, dspr, dsps);
      Jac j = jac6(xs, dspr, dsps);
      const double djaco = 0.5 * wi * (j.xr * j.ys - j.yr * j.xs);
      const double ldj = lf0[isg] + lmas[isg] / tau;
      const double ltau = -lmas[isg] * djaco / (tau * tau);
      for (int k = 0; k < d.mdegr; k++) lu[0][k] += ltau * b[k];
      const double h = 0.5 * wi * ldj;
      const double lxr = h * j.ys, lys = h * j.xr, lyr = -h * j.xs, lxs_ = -h * j.yr;
      for (int k = 0; k < 6; k++) {
        lxs[k][0] += lxr * dspr[k] + lxs_ * dsps[k];
        lxs[k][1] += lyr * dspr[k] + lys * dsps[k];
      }
    }
    for (int k = 0; k < 3; k++)
      for (int c = 0; c < 2; c++) {
        lxpt[iptsg(isg, k) - 1][c] += lxs[k][c];
        lxptc[iptsc[isg][k] - 1][c] += lxs[3 + k][c];
      }
  }
  for (int isc = 0; isc < 9; isc++)
    for (int k = 0; k < 6; k++) {
      lxpt[k][0] += lxptc[isc][0] * shpc[isc][k];
      lxpt[k][1] += lxptc[isc][1] * shpc[isc][k];
    }
  normals_tria_T(xpt, lgt, lxpt);
  for (int k = 0; k < 6; k++) {
    a.tbuf[(0 * 6 + k) * nt + it] = lxpt[k][0];
    a.tbuf[(1 * 6 + k) * nt + it] = lxpt[k][1];
    for (int v = 2; v < 6; v++) a.tbuf[(v * 6 + k) * nt + it] = 0.0;
  }
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) a.lU[(q * NDEG + k) * d.ncell + e] += lu[q][k];
}
__global__ void __launch_bounds__(128) k_a_tri_corner(Dev d, Adj a) {
  a_tri_corner(d, a, blockIdx.x * blockDim.x + threadIdx.x);
}

void launch_tri_adjoint_rhs(const Dev &d, const Adj &a, cudaStream_t st) {
  if (d.ntria > 0) k_a_tri_rhs<<<(d.ntria + 127) / 128, 128, 0, st>>>(d, a);
}
void launch_tri_adjoint_corner(const Dev &d, const Adj &a, cudaStream_t st) {
  if (d.ntria > 0) k_a_tri_corner<<<(d.ntria + 127) / 128, 128, 0, st>>>(d, a);
}

void launch_tri_rhs(const Dev &d, cudaStream_t st, const double *usn, const double *vsn, int fuse, double alfa) {
  if (d.ntria) k_tri_rhs<<<nblk(d.ntria, 128), 128, 0, st>>>(d, usn, vsn, fuse, alfa);
}
void launch_persson(const Dev &d, cudaStream_t st) { k_persson<<<nblk(d.nquad, 128), 128, 0, st>>>(d); }
void launch_flags_from_host(const Dev &d, cudaStream_t st, const int *flags) {
  k_flags_from_host<<<nblk(d.nquad, 256), 256, 0, st>>>(d, flags);
}
// geterror_lag_curvhybrid (Postprocess.f90:3587-4143, quad loop :3736-3944):
// per-block partial sums of the squared L2 errors against the exact solution
// of ncase 1 (rho, |u|, p) or 2 (rho, e_int, p), 25-point Gauss on the current
// coordinates; the host adds the block partials in block order.
__global__ void k_error_partial(Dev d, const double *X, const double *Y, double *part) {
  __shared__ double sm[3][256];
  const int iq = blockIdx.x * blockDim.x + threadIdx.x;
  double err[3] = {0.0, 0.0, 0.0};
  if (iq < d.nquad) {
    const int e = iq + d.ntria;
    const double g = d.gamlg;
    double xp[9][2], shp[9], dr[9], ds[9];
    load_quad(d, X, Y, iq, xp);
    const double rc = d.rc[e], sc = d.sc[e];
    for (int ig = 0; ig < 25; ig++) {
      const double r = cQ.g25[ig][0], s = cQ.g25[ig][1], wi = cQ.w25[ig];
      shp9v(r, s, shp);
      shp9d(r, s, dr, ds);
      Jac j = jac9(xp, dr, ds);
      const double djaco = wi * (j.xr * j.ys - j.yr * j.xs);
      double xg, yg;
      map9(xp, shp, xg, yg);
      double bq[6];
      bq[0] = 1.0; bq[1] = (r - rc) / 1.0; bq[2] = (s - sc) / 1.0;
      bq[3] = 0.5 * bq[1] * bq[1] - d.g19[e];
      bq[4] = 0.5 * bq[2] * bq[2] - d.g20[e];
      bq[5] = bq[1] * bq[2] - d.g21[e];
      double un[4] = {0.0, 0.0, 0.0, 0.0};
      for (int k = 0; k < d.mdegr; k++)
        for (int q = 0; q < 4; q++) un[q] = un[q] + Uget(d, d.Us, k, q, e) * bq[k];
      const double rho = 1.0 / un[0], uadv = un[1], vadv = un[2], eadv = un[3];
      const double pres = (g - 1.0) * rho * (eadv - 0.5 * (uadv * uadv + vadv * vadv));
      double e0, e1, e2;
      if (d.ncase == 1) {
        const double pexa = 0.25 * (cos(2.0 * cPI * xg) + cos(2.0 * cPI * yg)) + 1.0;
        const double uexa = sin(cPI * xg) * cos(cPI * yg), vexa = -cos(cPI * xg) * sin(cPI * yg);
        e0 = rho - 1.0;
        e1 = sqrt(uadv * uadv + vadv * vadv) - sqrt(uexa * uexa + vexa * vexa);
        e2 = pres - pexa;
      } else {
        const double eiadv = eadv - 0.5 * (uadv * uadv + vadv * vadv);
        const double eiexa = pow(1.0 - 0.6, -2.0 * (g - 1.0)), rhoexa = pow(1.0 - 0.6, -2.0);
        e0 = rho - rhoexa;
        e1 = eiadv - eiexa;
        e2 = pres - (g - 1.0) * rhoexa * eiadv;
      }
      err[0] = err[0] + fabs(e0) * fabs(e0) * djaco;
      err[1] = err[1] + fabs(e1) * fabs(e1) * djaco;
      err[2] = err[2] + fabs(e2) * fabs(e2) * djaco;
    }
  }
  for (int k = 0; k < 3; k++) sm[k][threadIdx.x] = err[k];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 3; k++) sm[k][threadIdx.x] += sm[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) part[3 * blockIdx.x + k] = sm[k][0];
}
int error_blocks(const Dev &d) { return nblk(d.nquad, 256); }

// Per-cell output values of the end-of-run post-processing: the quantities
// geterror_lag_curvhybrid writes for each cell to its radial profile file
// (Postprocess.f90:3700-3717 triangles, :3944-3983 quads) and
// getoutput_cellvtk writes as cell data (:1324-1391), from the cell averages:
// out[k*ncell + e] for k = 0..8 = (radius of the centre, rho, p, e_int, x_c,
// y_c, |u|, u, v), with rho = 1/tau (ndens = 1), p = (gamma - 1) rho (e -
// (u^2 + v^2)/2), e_int = p / rho / (gamma - 1).  The centre is the map at
// (r, s) = (0, 0) for quads (the 9th node) and at the reference mass centre
// (rc, sc) for triangles (6-node shape functions), from the state U and the
// coordinates X, Y.
__global__ void k_cell_output(Dev d, const double *U, const double *X, const double *Y, double *out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.ncell) return;
  const double g = d.gamlg;
  double xc = 0.0, yc = 0.0;
  if (e < d.ntria) {
    double shp[6];
    shp6v(d.rc[e], d.sc[e], shp);
    for (int k = 0; k < 6; k++) {
      const int p = d.ipt[k * d.ntria + e];
      xc = xc + shp[k] * X[p];
      yc = yc + shp[k] * Y[p];
    }
  } else {
    const int p = d.ipq[8 * d.nquad + (e - d.ntria)];
    xc = X[p];
    yc = Y[p];
  }
  const double rhoc = 1.0 / Uget(d, U, 0, 0, e);
  const double uctr = Uget(d, U, 0, 1, e), vctr = Uget(d, U, 0, 2, e), ectr = Uget(d, U, 0, 3, e);
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
void launch_cell_output(const Dev &d, cudaStream_t st, const double *U, const double *X, const double *Y,
                        double *out) {
  k_cell_output<<<nblk(d.ncell, 256), 256, 0, st>>>(d, U, X, Y, out);
}
void launch_error(const Dev &d, cudaStream_t st, const double *X, const double *Y, double *part) {
  k_error_partial<<<nblk(d.nquad, 256), 256, 0, st>>>(d, X, Y, part);
}
void launch_weno(const Dev &d, cudaStream_t st) { k_weno<<<nblk(d.nquad, 64), 64, 0, st>>>(d); }
// one warp per troubled quad, a grid of at most 8 blocks per SM looping over the list
void launch_weno_warp(const Dev &d, cudaStream_t st) {
  k_weno_warp<<<d.nquad < 1184 ? (d.nquad > 0 ? d.nquad : 1) : 1184, 32, 0, st>>>(d);
}
size_t weno_linear_smem() { return sizeof(WenoAdjBlock); }
void launch_weno_linear(const Dev &d, cudaStream_t st, int mode, const double *v, double *out, double *wbuf,
                        int *wslot, int cap, int *overflow) {
  const int g = d.nquad < 1184 ? (d.nquad > 0 ? d.nquad : 1) : 1184;
  k_weno_linear<<<g, 32, sizeof(WenoAdjBlock), st>>>(d, mode, v, out, wbuf, wslot, cap, overflow);
}
void launch_weno_gather(const Dev &d, cudaStream_t st, double *lamU, double *lamUn, int fold, const double *wbuf,
                        const int *wslot, int cap, const int *inv_ptr, const int *inv_ent) {
  k_weno_gather<<<nblk(d.ncell, 128), 128, 0, st>>>(d, lamU, lamUn, fold, wbuf, wslot, cap, inv_ptr, inv_ent);
}
void launch_weno_swap(const Dev &d, cudaStream_t st) { k_weno_swap<<<nblk(d.nquad, 256), 256, 0, st>>>(d); }
void launch_weno_commit(const Dev &d, cudaStream_t st) { k_weno_commit<<<nblk(d.nquad, 256), 256, 0, st>>>(d); }
void launch_corner(const Dev &d, cudaStream_t st) { k_corner<<<nblk(d.nquad, 128), 128, 0, st>>>(d); }
void launch_node(const Dev &d, cudaStream_t st) { k_node<<<nblk(d.npoin, 256), 256, 0, st>>>(d); }
void launch_rhs(const Dev &d, cudaStream_t st) { k_rhs<<<nblk(d.nquad, 128), 128, 0, st>>>(d); }
int dt_blocks(const Dev &d) { return nblk(d.nquad, 256); }
void launch_dt(const Dev &d, cudaStream_t st, int ndt) {
  int nb = nblk(d.nquad, 256);
  k_dt_partial<<<nb, 256, 0, st>>>(d);
  k_dt_final<<<1, 256, 0, st>>>(d, nb, ndt);
}
void launch_dt_final(const Dev &d, cudaStream_t st, int nb, int ndt) { k_dt_final<<<1, 256, 0, st>>>(d, nb, ndt); }
void launch_update(const Dev &d, cudaStream_t st, double alfa) {
  k_update<<<nblk(d.ncell, 128), 128, 0, st>>>(d, alfa);
}
void launch_nodes(const Dev &d, cudaStream_t st, double alfa) {
  k_nodes<<<nblk(d.npoin, 256), 256, 0, st>>>(d, alfa);
}
void launch_copyback(const Dev &d, cudaStream_t st) { k_copyback<<<1184, 256, 0, st>>>(d); }
void launch_step_begin(const Dev &d, cudaStream_t st, int itime) { k_step_begin<<<1, 1, 0, st>>>(d, itime); }
void launch_step_end(const Dev &d, cudaStream_t st, int check) { k_step_end<<<1, 1, 0, st>>>(d, check); }
void launch_init_msub(const Dev &d, cudaStream_t st) {
  k_init_msub<<<nblk(d.nquad, 128), 128, 0, st>>>(d);
}
void launch_init(const Dev &d, cudaStream_t st) {
  k_init_geo<<<nblk(d.nquad, 128), 128, 0, st>>>(d);
  k_init_fields<<<nblk(d.nquad, 128), 128, 0, st>>>(d);
}

}  // namespace lag2d
