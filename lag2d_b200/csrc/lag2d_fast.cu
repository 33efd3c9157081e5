// Optimised kernels of the curved-P2 Lagrangian DG stage (sm_100a, FP64).
//
// Same arithmetic as the reference-order kernels (lag2d_kernels.cu) up to
// rounding, with far fewer FP64 instructions per cell:
//  * every volume the reference integrates with Gauss rules of a 9-node map
//    (cell: getcellvol_lag 6x6; sub-cells: getrhosubg_averg 5x5) is exact for
//    those polynomial integrands, so it is evaluated in closed form from the
//    36 node cross products x_i y_j - x_j y_i (lag2d_tables.inc);
//  * det J at fixed points (Persson, sub-cell densities, source) comes from its
//    16 bicubic coefficients, a fixed linear map of the same cross products;
//  * Jacobians on the 5x5 Gauss-Lobatto grid are sum-factorised on the 3x3
//    tensor of quad nodes;
//  * the corner pass reduces its 32 corner faces to per-node partial sums
//    (9 nodes x 5 values) that the node pass gathers in cell order, and the
//    RHS pass recomputes the cheap corner data instead of reading it back;
//  * in RK stages 2 and 3 the mass-matrix solve and RK combine are fused into
//    the RHS pass.
#include <cuda_pipeline.h>
#include <cuda_runtime.h>
#ifndef LAG2D_ACC_MINB
#define LAG2D_ACC_MINB 3
#endif
#ifndef LAG2D_ACF_MINB
#define LAG2D_ACF_MINB 2
#endif
// the RHS kernel: 2 resident blocks of kRhsBlock per SM leave it up to 255
// registers and no spills (on the 1024 x 1024 Taylor-Green step 1.11 ms per
// step against 1.49 ms at 3 blocks and 168 registers with 584 bytes of
// spill loads per thread)
#ifndef LAG2D_RHS_MINB
#define LAG2D_RHS_MINB 2
#endif
#ifndef LAG2D_AREVF_MINB
#define LAG2D_AREVF_MINB 3
#endif
#ifndef LAG2D_CCORR_MINB
#define LAG2D_CCORR_MINB 4
#endif
#ifndef LAG2D_CFACES_MINB
#define LAG2D_CFACES_MINB 4
#endif
#include <math.h>

#include "lag2d_device.cuh"
#include "lag2d_fast_tables.h"

namespace lag2d {

namespace fast {

#include "lag2d_tables.inc"

// Small lookup tables indexed by warp-uniform loop counters: constant memory
// for the kernels, a host mirror for CPU checks of the same bodies.
struct FastTables {
  int nc_start[10];   // node k owns corner entries [nc_start[k], nc_start[k+1])
  int nc_entry[16];   // isg * 4 + ivsg, in the reference's (isg, ivsg) order per node
  int fnqsg[32];      // gesgq slot (sign = orientation) of corner face (isg, ivsg, f)
  double wrie[32];    // Riemann corner-face weights (Getrhslaggauss.f90:10534-10552) x 0.25
  double wmas[32];    // mass-equation face weights (Getrhslaggauss.f90:8611-8634) x 0.25
  double wmom[16];    // momentum/energy face weights (Getrhslaggauss.f90:8580-8603)
  int pa[12], pb[12], side[12];  // Simpson points as tensor nodes and their face
  double dl[9];       // L'_c at r = -1, 0, 1: dl[3a + c]
  double xv[9], yv[9];  // reference coordinates of the 9 nodes
};
// compile-time tables: lookups with indices known after unrolling fold to
// constants (no constant-bank loads, no branches on the looked-up values)
__host__ __device__ __forceinline__ const FastTables &FT() {
  static constexpr FastTables t = LAG2D_FAST_TABLES;
  return t;
}

// 1-D quadratic Lagrange basis on {-1, 0, 1} and its derivative
__host__ __device__ __forceinline__ void lag3(double r, double *l) {
  l[0] = 0.5 * r * (r - 1.0);
  l[1] = 1.0 - r * r;
  l[2] = 0.5 * r * (r + 1.0);
}
__host__ __device__ __forceinline__ void dlag3(double r, double *l) {
  l[0] = r - 0.5;
  l[1] = -2.0 * r;
  l[2] = r + 0.5;
}

// cos(pi d) and sin(pi d) for small |d| from their Taylor series in t = pi d
// with N terms each: cos to degree 2N-2, sin to degree 2N-1.  N = 7 covers
// |d| <= 0.15, N = 4 covers |d| <= 0.00625 and N = 3 covers |d| <= 0.0009375,
// each with the first omitted term below 1e-17 relative.  Coefficients are
// (-1)^k / (2k)! and (-1)^k / (2k+1)!, evaluated by Horner's rule in t^2.
template <int N>
__host__ __device__ __forceinline__ void cossin_pi_series(double d, double &c, double &s) {
  constexpr double kc[7] = {1.0, -1.0 / 2.0, 1.0 / 24.0, -1.0 / 720.0, 1.0 / 40320.0, -1.0 / 3628800.0,
                            1.0 / 479001600.0};
  constexpr double ks[7] = {1.0, -1.0 / 6.0, 1.0 / 120.0, -1.0 / 5040.0, 1.0 / 362880.0, -1.0 / 39916800.0,
                            1.0 / 6227020800.0};
  const double t = 3.14159265358979311599796346854 * d, t2 = t * t;
  double pc = kc[N - 1], ps = ks[N - 1];
#pragma unroll
  for (int k = N - 2; k >= 0; k--) {
    pc = kc[k] + t2 * pc;
    ps = ks[k] + t2 * ps;
  }
  c = pc;
  s = t * ps;
}

__host__ __device__ __forceinline__ double deteval(const double *D, double r, double s) {
  double e[4];
#pragma unroll
  for (int n = 0; n < 4; n++) e[n] = D[n] + r * (D[4 + n] + r * (D[8 + n] + r * D[12 + n]));
  return e[0] + s * (e[1] + s * (e[2] + s * e[3]));
}

// integral of det J over the sub-square [r0, r0+1] x [s0, s0+1]
__host__ __device__ __forceinline__ double det_integral(const double *D, double r0, double s0) {
  double mr[4], ms[4];
  const double r1 = r0 + 1.0, s1 = s0 + 1.0;
  double pr0 = r0, pr1 = r1, ps0 = s0, ps1 = s1;
#pragma unroll
  for (int m = 0; m < 4; m++) {
    mr[m] = (pr1 - pr0) / (m + 1);
    ms[m] = (ps1 - ps0) / (m + 1);
    pr0 *= r0; pr1 *= r1; ps0 *= s0; ps1 *= s1;
  }
  double v = 0.0;
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int n = 0; n < 4; n++) v += D[4 * m + n] * mr[m] * ms[n];
  return v;
}

// 1-D Gauss (ruqope) and Gauss-Lobatto (ruqope_lobatto) 5-point rules
__host__ __device__ __forceinline__ double g5p(int i) {
  const double p[5] = {-0.9061798459386639927976269, -0.5384693101056830910363144, 0.0,
                       0.5384693101056830910363144, 0.9061798459386639927976269};
  return p[i];
}
__host__ __device__ __forceinline__ double g5w(int i) {
  const double w[5] = {0.2369268850561890875142640, 0.4786286704993664680412915, 0.5688888888888888888888889,
                       0.4786286704993664680412915, 0.2369268850561890875142640};
  return w[i];
}
__host__ __device__ __forceinline__ double l5p(int i) {
  const double p[5] = {-1.0, -0.6546536707079771437983, 0.0, 0.6546536707079771437983, 1.0};
  return p[i];
}
__host__ __device__ __forceinline__ double l5w(int i) {
  const double w[5] = {0.1, 0.544444444444444444444, 0.7111111111111111111111, 0.544444444444444444444, 0.1};
  return w[i];
}

struct CellGeo {
  double rc, sc, g19, g20, g21;
};

__host__ __device__ __forceinline__ void node_basis2(const CellGeo &g, int iv, double *b) {
  b[0] = 1.0;
  b[1] = FT().xv[iv] - g.rc;
  b[2] = FT().yv[iv] - g.sc;
  b[3] = 0.5 * b[1] * b[1] - g.g19;
  b[4] = 0.5 * b[2] * b[2] - g.g20;
  b[5] = b[1] * b[2] - g.g21;
}


__host__ __device__ __forceinline__ int fnqsg2(int isg, int k) { return FT().fnqsg[8 * isg + k]; }
// corner-face weights (Getrhslaggauss.f90:10534-10552 x 0.25; :8580-8637)
__host__ __device__ __forceinline__ double wrie(int isg, int ivsg, int f) { return FT().wrie[8 * isg + 2 * ivsg + f]; }
__host__ __device__ __forceinline__ double wmas(int isg, int ivsg, int f) { return FT().wmas[8 * isg + 2 * ivsg + f]; }
__host__ __device__ __forceinline__ double wmom(int isg, int ivsg) { return FT().wmom[4 * isg + ivsg]; }

// Impedance-weighted area m = mu * A * w of one corner face
// (getriecoef_matrixnew, Limiterlag.f90:1037) from the unnormalised face
// vector an (unit normal n = an / |an|, face length A = 2 |an|) and the face
// weight w:  m = 2 w (rho c |an| + cimpd rho slpdu |du . an|), which needs no
// division.  The jump-direction branch is taken only when |u* - u_c| / c >=
// 1e12, tested on squares.
__host__ __device__ __forceinline__ double corner_m(double rhoct, double sdctr, double cimpd, double slpdu,
                                                   double dux, double duy, double ax, double ay, double w) {
  const double nn = sqrt(ax * ax + ay * ay);
  const double dun = fabs(dux * ax + duy * ay);
  const double j2 = dux * dux + duy * duy;
  const double lim = 1.0e12 * sdctr;
  if (j2 < lim * lim) return 2.0 * w * (rhoct * sdctr * nn + cimpd * rhoct * slpdu * dun);
  const double murie = rhoct * sdctr + cimpd * rhoct * slpdu * (dun / nn);
  const double nrm = sqrt(j2);
  double jx, jy;
  if (nrm < (double)1.e-11f) { jx = (double)1.e-11f; jy = (double)1.e-11f; }
  else { jx = dux / nrm; jy = duy / nrm; }
  return murie * 2.0 * w * fabs(ax * jx + ay * jy);
}

// Corner faces grouped by the node they belong to, in the reference's
// (isg, ivsg) order: node k is vertex ivsg of sub-cell isg for the entries
// NODE_CORNERS[NC_START[k] .. NC_START[k+1]) encoded as isg * 4 + ivsg.
__host__ __device__ __forceinline__ int nc_start(int k) { return FT().nc_start[k]; }
__host__ __device__ __forceinline__ int nc_entry(int i) { return FT().nc_entry[i]; }

// Unnormalised face vector an of the gesgq slot `slot`: the unit normal is
// an / |an| and the face length 2 |an| (getfnds_lagsms_simpsonhybrid and
// getfnds_lagsmsif_hybrid, Getrhslaggauss.f90:9660-10021, 3356-3602)
__host__ __device__ __forceinline__ void slot_an(const double X[3][3], const double Y[3][3], int slot, double &ax,
                                                 double &ay) {
  if (slot >= 8 && slot < 12) {
    // inner sub-cell face at edge node (5..8) towards the centre
    const int f = slot - 8;
    const double lm0 = 0.375, lm1 = 0.75, lm2 = -0.125, lp0 = -0.125, lp1 = 0.75, lp2 = 0.375;
    double ex, ey, vx, vy;
    if (f == 0) {
      ex = X[1][0]; ey = Y[1][0];
      vx = lm0 * X[1][0] + lm1 * X[1][1] + lm2 * X[1][2];
      vy = lm0 * Y[1][0] + lm1 * Y[1][1] + lm2 * Y[1][2];
    } else if (f == 1) {
      ex = X[2][1]; ey = Y[2][1];
      vx = lp0 * X[0][1] + lp1 * X[1][1] + lp2 * X[2][1];
      vy = lp0 * Y[0][1] + lp1 * Y[1][1] + lp2 * Y[2][1];
    } else if (f == 2) {
      ex = X[1][2]; ey = Y[1][2];
      vx = lp0 * X[1][0] + lp1 * X[1][1] + lp2 * X[1][2];
      vy = lp0 * Y[1][0] + lp1 * Y[1][1] + lp2 * Y[1][2];
    } else {
      ex = X[0][1]; ey = Y[0][1];
      vx = lm0 * X[0][1] + lm1 * X[1][1] + lm2 * X[2][1];
      vy = lm0 * Y[0][1] + lm1 * Y[1][1] + lm2 * Y[2][1];
    }
    const double dxdr = -1.5 * ex - 0.5 * X[1][1] + 2.0 * vx;
    const double dydr = -1.5 * ey - 0.5 * Y[1][1] + 2.0 * vy;
    ax = -dydr;
    ay = dxdr;
    return;
  }
  // Simpson points (getfnds_lagsms_simpsonhybrid order) on the 4 outer faces
  const int ig = slot < 8 ? slot : slot - 4;
  const FastTables &T = FT();
  const int ia = T.pa[ig], ib = T.pb[ig];
  const double *da = T.dl + 3 * ia, *db = T.dl + 3 * ib;
  // the tensor rows/columns are selected with uniform branches to keep X, Y in registers
  double xa0, xa1, xa2, ya0, ya1, ya2, xb0, xb1, xb2, yb0, yb1, yb2;
  if (ib == 0) { xa0 = X[0][0]; xa1 = X[1][0]; xa2 = X[2][0]; ya0 = Y[0][0]; ya1 = Y[1][0]; ya2 = Y[2][0]; }
  else if (ib == 1) { xa0 = X[0][1]; xa1 = X[1][1]; xa2 = X[2][1]; ya0 = Y[0][1]; ya1 = Y[1][1]; ya2 = Y[2][1]; }
  else { xa0 = X[0][2]; xa1 = X[1][2]; xa2 = X[2][2]; ya0 = Y[0][2]; ya1 = Y[1][2]; ya2 = Y[2][2]; }
  if (ia == 0) { xb0 = X[0][0]; xb1 = X[0][1]; xb2 = X[0][2]; yb0 = Y[0][0]; yb1 = Y[0][1]; yb2 = Y[0][2]; }
  else if (ia == 1) { xb0 = X[1][0]; xb1 = X[1][1]; xb2 = X[1][2]; yb0 = Y[1][0]; yb1 = Y[1][1]; yb2 = Y[1][2]; }
  else { xb0 = X[2][0]; xb1 = X[2][1]; xb2 = X[2][2]; yb0 = Y[2][0]; yb1 = Y[2][1]; yb2 = Y[2][2]; }
  const double xr = da[0] * xa0 + da[1] * xa1 + da[2] * xa2;
  const double yr = da[0] * ya0 + da[1] * ya1 + da[2] * ya2;
  const double xs = db[0] * xb0 + db[1] * xb1 + db[2] * xb2;
  const double ys = db[0] * yb0 + db[1] * yb1 + db[2] * yb2;
  switch (T.side[ig]) {
    case 0: ax = yr; ay = -xr; break;     // vnorm (0,-1)
    case 1: ax = ys; ay = -xs; break;     // vnorm (1, 0)
    case 2: ax = -yr; ay = xr; break;     // vnorm (0, 1)
    default: ax = -ys; ay = xs; break;    // vnorm (-1,0)
  }
}

// face vector of corner face f of vertex ivsg of sub-cell isg, oriented outwards
__host__ __device__ __forceinline__ void corner_an(const double X[3][3], const double Y[3][3], int isg, int ivsg,
                                                   int f, double &ax, double &ay) {
  const int code = fnqsg2(isg, 2 * ivsg + f);
  const int slot = (code >= 0 ? code : -code) - 1;
  slot_an(X, Y, slot, ax, ay);
  if (code < 0) { ax = -ax; ay = -ay; }
}

struct Loaded {
  double X[3][3], Y[3][3];  // node coordinates on the 3x3 tensor
};

__host__ __device__ __forceinline__ void load_cell(const Dev &d, const double *XS, const double *YS, int iq, Loaded &L) {
  const int A[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
  const int B[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const int p = d.ipq[k * d.nquad + iq];
    L.X[A[k]][B[k]] = XS[p];
    L.Y[A[k]][B[k]] = YS[p];
  }
}

// node coordinates relative to the centre node, in the reference node order:
// the cross products x_i y_j - x_j y_i of absolute coordinates cancel about
// log10(|x|^2 / V) digits on a small cell far from the origin; every
// quantity built from them here (areas, sub-areas, det J coefficients) is
// invariant under translation, so they are taken relative to the cell
__host__ __device__ __forceinline__ void node_xy_rel(const Loaded &L, double (*xp)[2]) {
  const int A[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
  const int B[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
  const double ox = L.X[1][1], oy = L.Y[1][1];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    xp[k][0] = L.X[A[k]][B[k]] - ox;
    xp[k][1] = L.Y[A[k]][B[k]] - oy;
  }
}

// cross36 of centre-relative coordinates (xp[8] = 0): the 8 products with
// the centre node vanish and are zero constants here, so the tables fold them
__host__ __device__ __forceinline__ void cross36_rel(const double (*xp)[2], double *c) {
  cross36(xp, c);
  c[7] = 0.0; c[14] = 0.0; c[20] = 0.0; c[25] = 0.0; c[29] = 0.0; c[32] = 0.0; c[34] = 0.0; c[35] = 0.0;
}

// node coordinates back in the reference node order
__host__ __device__ __forceinline__ void node_xy(const Loaded &L, double (*xp)[2]) {
  const int A[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
  const int B[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
#pragma unroll
  for (int k = 0; k < 9; k++) {
    xp[k][0] = L.X[A[k]][B[k]];
    xp[k][1] = L.Y[A[k]][B[k]];
  }
}

__host__ __device__ __forceinline__ void load_u(const Dev &d, const double *U, int e, double u[4][6]) {
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int k = 0; k < 6; k++) u[q][k] = U[(q * 6 + k) * (size_t)d.ncell + e];
}

// ---------------------------------------------------------------------------
// Persson indicator + physical mass centre + frame (all quads)
// ---------------------------------------------------------------------------
__host__ __device__ void f_persson(const Dev &d, int iq) {
  if (iq >= d.nquad || d.sc_dev->done) return;
  const int e = iq + d.ntria;
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  double c[36], D[16];
  {
    double xp[9][2];
    node_xy_rel(L, xp);
    cross36_rel(xp, c);
  }
  detpoly(c, D);
  const CellGeo g{d.rc[e], d.sc[e], d.g19[e], d.g20[e], d.g21[e]};
  double t[6];
#pragma unroll
  for (int k = 0; k < 6; k++) t[k] = d.Us[k * (size_t)d.ncell + e];
  double unvar2 = 0.0, unvar1 = 0.0;
#pragma unroll
  for (int i = 0; i < 5; i++) {
    const double r = g5p(i);
    const double dr = r - g.rc;
    // along the row r: det J cubic, P1 part linear and P2 part quadratic in s
    double e[4];
#pragma unroll
    for (int n = 0; n < 4; n++) e[n] = D[n] + r * (D[4 + n] + r * (D[8 + n] + r * D[12 + n]));
    const double a0 = t[0] + t[1] * dr;
    const double h0 = t[3] * (0.5 * dr * dr - g.g19) - t[4] * g.g20 - t[5] * g.g21;
    const double h1 = t[5] * dr, h2 = 0.5 * t[4];
    const double wi = g5w(i);
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const double s = g5p(j);
      const double ds = s - g.sc;
      const double djaco = wi * g5w(j) * (e[0] + s * (e[1] + s * (e[2] + s * e[3])));
      const double p1 = a0 + t[2] * ds;
      const double hi = h0 + ds * (h1 + h2 * ds);
      const double un = p1 + hi;
      unvar2 += hi * hi * djaco;
      unvar1 += un * un * djaco;
    }
  }
  const double thr = -3.0 * log10(4.0) - 4.0;
  const int fl = (log10(unvar2 / unvar1) <= thr) ? 0 : 1;
  d.flag[e] = fl;
  // physical mass centre from the time-invariant mass-weighted shape moments
  double xmc = 0.0, ymc = 0.0;
  {
    double xp[9][2];
    node_xy(L, xp);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const double w = d.wmom[k * (size_t)d.nquad + iq];
      xmc += w * xp[k][0];
      ymc += w * xp[k][1];
    }
  }
  const double masel = d.mass[e];
  d.geoph[e] = xmc / masel;
  d.geoph[d.ncell + e] = ymc / masel;
  const double ma = d.Us[(1 * 6) * (size_t)d.ncell + e], mb = d.Us[(2 * 6) * (size_t)d.ncell + e];
  double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
  const double nrm = sqrt(ma * ma + mb * mb);
  if (nrm > 1.0e-10) {
    m0 = ma / nrm;
    m2 = mb / nrm;
    m1 = -mb / nrm;
    m3 = ma / nrm;
  }
  d.mapmt[0 * (size_t)d.ncell + e] = m0;
  d.mapmt[1 * (size_t)d.ncell + e] = m1;
  d.mapmt[2 * (size_t)d.ncell + e] = m2;
  d.mapmt[3 * (size_t)d.ncell + e] = m3;
  if (fl) {
#ifdef __CUDA_ARCH__
    const int slot = atomicAdd(d.wcount, 1);
#else
    const int slot = (*d.wcount)++;
#endif
    d.wlist[slot] = iq;
  }
}

// Taylor-Green source moments el[k] += sum_g src(x_g) b_k(g) detJ_g w_g over
// the 5x5 Gauss points.  cos(pi x) at the points by angle addition from the
// centre node x_c: cos(pi x) = cos(pi x_c) cos(pi d) - sin(pi x_c) sin(pi d),
// d = x - x_c, with the NSER-term series of cossin_pi_series when every node
// of the cell lies within delta of the centre node in x and y (the quadratic
// map then keeps |d| <= 1.5625 delta at the Gauss points): delta <= 0.09 for
// 7 terms, 0.004 for 4, 0.0006 for 3; otherwise (NSER = 0) cospi at each
// point.  The point loop has no branch.  The basis sums are taken per row:
// b_k along a row is a polynomial in ds of degree <= 2.
template <int NSER>
__host__ __device__ __forceinline__ void tgv_source_rows(const Loaded &L, const CellGeo &G, const double D[16],
                                                         double g, double el[6]) {
  const double coef = 0.25 * 3.14159265358979311599796346854 / (g - 1.0);
  const double xc = L.X[1][1], yc = L.Y[1][1];
  const double cxc = cospi(xc), sxc = sinpi(xc), cyc = cospi(yc), syc = sinpi(yc);
#pragma unroll 1
  for (int i = 0; i < 5; i++) {
    const double r = g5p(i), dr = r - G.rc;
    double lr[3];
    lag3(r, lr);
    double Px[3], Py[3];
#pragma unroll
    for (int bb = 0; bb < 3; bb++) {
      Px[bb] = lr[0] * (L.X[0][bb] - xc) + lr[1] * (L.X[1][bb] - xc) + lr[2] * (L.X[2][bb] - xc);
      Py[bb] = lr[0] * (L.Y[0][bb] - yc) + lr[1] * (L.Y[1][bb] - yc) + lr[2] * (L.Y[2][bb] - yc);
    }
    double e[4];
#pragma unroll
    for (int n = 0; n < 4; n++) e[n] = D[n] + r * (D[4 + n] + r * (D[8 + n] + r * D[12 + n]));
    const double wi = coef * g5w(i);
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const double s = g5p(j), ds = s - G.sc;
      double ls[3];
      lag3(s, ls);
      const double dx = Px[0] * ls[0] + Px[1] * ls[1] + Px[2] * ls[2];
      const double dy = Py[0] * ls[0] + Py[1] * ls[1] + Py[2] * ls[2];
      const double djaco = wi * g5w(j) * (e[0] + s * (e[1] + s * (e[2] + s * e[3])));
      double cx, cy;
      if (NSER > 0) {
        double cdx, sdx, cdy, sdy;
        cossin_pi_series<NSER>(dx, cdx, sdx);
        cossin_pi_series<NSER>(dy, cdy, sdy);
        cx = cxc * cdx - sxc * sdx;
        cy = cyc * cdy - syc * sdy;
      } else {
        cx = cospi(xc + dx);
        cy = cospi(yc + dy);
      }
      const double c3x = cx * (4.0 * cx * cx - 3.0), c3y = cy * (4.0 * cy * cy - 3.0);
      const double src = (c3x * cy - c3y * cx) * djaco;
      m0 += src;
      m1 += src * ds;
      m2 += src * ds * ds;
    }
    // b = (1, dr, ds, dr^2/2 - g19, ds^2/2 - g20, dr ds - g21) along the row
    el[0] += m0;
    el[1] += m0 * dr;
    el[2] += m1;
    el[3] += m0 * (0.5 * dr * dr - G.g19);
    el[4] += 0.5 * m2 - G.g20 * m0;
    el[5] += m1 * dr - G.g21 * m0;
  }
}
__host__ __device__ __forceinline__ void tgv_source(const Loaded &L, const CellGeo &G, const double D[16], double g,
                                                    double el[6]) {
  double mx = 0.0, my = 0.0;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      mx = fmax(mx, fabs(L.X[a][b] - L.X[1][1]));
      my = fmax(my, fabs(L.Y[a][b] - L.Y[1][1]));
    }
  const double delta = fmax(mx, my);
  if (delta <= 0.0006) tgv_source_rows<3>(L, G, D, g, el);
  else if (delta <= 0.004) tgv_source_rows<4>(L, G, D, g, el);
  else if (delta <= 0.09) tgv_source_rows<7>(L, G, D, g, el);
  else tgv_source_rows<0>(L, G, D, g, el);
}

// Taylor-Green energy source of the stage (rhsdomnsrcdg_lag_curvquad,
// Getrhslag.f90:4070-4251), one thread per quad: it depends on the stage's
// nodes and the reference geometry only; the RHS pass adds the 6 moments
// (d.src, [6][nquad]).  A kernel of its own: inside the corner or RHS kernels
// its registers and code cost those kernels more than its own launch.
__host__ __device__ void f_tgv_src(const Dev &d, int iq) {
  if (iq >= d.nquad || d.sc_dev->done) return;
  const int e = iq + d.ntria;
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  double c[36], D[16];
  {
    double xp[9][2];
    node_xy_rel(L, xp);
    cross36_rel(xp, c);
  }
  detpoly(c, D);
  const CellGeo G{d.rc[e], d.sc[e], d.g19[e], d.g20[e], d.g21[e]};
  double el[6] = {0, 0, 0, 0, 0, 0};
  tgv_source(L, G, D, d.gamlg, el);
#pragma unroll
  for (int k = 0; k < 6; k++) d.src[k * (size_t)d.nquad + iq] = el[k];
}

// ---------------------------------------------------------------------------
// Corner pass: node partial sums of the Riemann coefficients + sub-cell
// density corrections (getriem_quadsubg2 with getrhosubg_averg/_daverg)
// ---------------------------------------------------------------------------
// The corner pass runs as two kernels: f_corner_corr, the sub-cell density
// corrections (written to d.corr, which the RHS pass reads anyway), and
// f_corner_faces, the corner faces with the corrections read back.  Each is
// compiled for 4 resident blocks of 128 per SM (128 registers): on the
// 1024x1024 Taylor-Green step the pair takes 1.68 ms against 1.83 ms for a
// single kernel at 168 registers (3 blocks).
__host__ __device__ void f_corner_corr(const Dev &d, int iq) {
  if (iq >= d.nquad || d.sc_dev->done) return;
  const int e = iq + d.ntria;
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  double c[36], D[16];
  {
    double xp[9][2];
    node_xy_rel(L, xp);
    cross36_rel(xp, c);
  }
  detpoly(c, D);
  const CellGeo G{d.rc[e], d.sc[e], d.g19[e], d.g20[e], d.g21[e]};
  // the tau DOFs
  double u[6];
#pragma unroll
  for (int k = 0; k < 6; k++) u[k] = d.Us[k * (size_t)d.ncell + e];
  // sub-cell densities: initial mass / exact sub-cell area, and the DG-implied
  // harmonic mean of tau over each sub-cell (5x5 Gauss per sub-cell)
  double vsub4[4];
  subareas(c, vsub4);
  // The harmonic mean sum masel = sum_g w_g det_g / tau_g is kept as one
  // fraction num / den (a/b + c/d = (a d + c b) / (b d)): three multiply-adds
  // per point and one division per sub-cell instead of one division per point.
  // tau is scaled by the cell-average tau first (rtc), so that the product of
  // the 25 scaled values stays near 1; masel = rtc num / den.
  // Sub-cells 0 and 3 (r in [-1, 0]) share their Gauss rows, and so do 1 and
  // 2 (r in [0, 1]): each row's det J and tau coefficients serve both, whose
  // two fraction chains (s in [-1, 0] and [0, 1]) run side by side.
  const double rtc = 1.0 / u[0];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const double ofr = h == 0 ? -1.0 : 1.0;
    const int ilo = h == 0 ? 0 : 1, ihi = h == 0 ? 3 : 2;  // s in [-1, 0], [0, 1]
    double nlo = 0.0, dlo = 1.0, nhi = 0.0, dhi = 1.0;
#pragma unroll 1
    for (int i = 0; i < 5; i++) {
      const double r = (g5p(i) + ofr) / 2.0;
      // along the row r, det J is a cubic and tau a quadratic in s
      double e[4];
#pragma unroll
      for (int n = 0; n < 4; n++) e[n] = D[n] + r * (D[4 + n] + r * (D[8 + n] + r * D[12 + n]));
      const double dr = r - G.rc;
      const double t0 = rtc * (u[0] + u[1] * dr + u[3] * (0.5 * dr * dr - G.g19) - u[4] * G.g20 - u[5] * G.g21);
      const double t1 = rtc * (u[2] + u[5] * dr), t2 = rtc * (0.5 * u[4]);
      const double wi = 0.25 * g5w(i);
#pragma unroll
      for (int j = 0; j < 5; j++) {
        const double w = wi * g5w(j);
        {
          const double s = (g5p(j) - 1.0) / 2.0;
          const double ds = s - G.sc;
          const double tau = t0 + ds * (t1 + t2 * ds);
          const double det = e[0] + s * (e[1] + s * (e[2] + s * e[3]));
          nlo = nlo * tau + (w * det) * dlo;
          dlo = dlo * tau;
        }
        {
          const double s = (g5p(j) + 1.0) / 2.0;
          const double ds = s - G.sc;
          const double tau = t0 + ds * (t1 + t2 * ds);
          const double det = e[0] + s * (e[1] + s * (e[2] + s * e[3]));
          nhi = nhi * tau + (w * det) * dhi;
          dhi = dhi * tau;
        }
      }
    }
    // 1 / uqsgc = masel / volel with masel = rtc num / den
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const int isg = t == 0 ? ilo : ihi;
      const double num = t == 0 ? nlo : nhi, den = t == 0 ? dlo : dhi;
      const double unksgq = (1.0 / vsub4[isg]) * d.msub[isg * (size_t)d.nquad + iq];
      const double volel = det_integral(D, (isg == 0 || isg == 3) ? -1.0 : 0.0, (isg == 0 || isg == 1) ? -1.0 : 0.0);
      d.corr[isg * (size_t)d.nquad + iq] = d.cdrho * (unksgq - (rtc * num) / (den * volel));
    }
  }
}

// Corner faces of one quad: per node the vertex state, then its corner faces
// in the reference's order, summed into the node's 5 partials.  The cell's
// 24 DOFs and 4 sub-cell corrections are copied asynchronously (cp.async)
// into this thread's column of shared memory (stride kCornerBlock) at entry,
// so their loads overlap the coordinate gathers and they take no registers
// between the vertex states (corner pass 1.404 -> 1.189 ms per step on the
// 1024x1024 Taylor-Green mesh against the same kernel with them in
// registers).
constexpr int kCornerBlock = 128;
constexpr int kCornerStage = 28;
__device__ void f_corner_faces(const Dev &d, int iq_in, double *col) {
  // every thread of the block reaches the barriers below: a thread past the
  // last quad works on the last quad and stores nothing
  if (d.nquad <= 0 || d.sc_dev->done) return;
  const bool live = iq_in < d.nquad;
  const int iq = live ? iq_in : d.nquad - 1;
  const int e = iq + d.ntria;
  {
    const size_t nc = d.ncell;
    for (int v = 0; v < 24; v++) __pipeline_memcpy_async(col + v * kCornerBlock, d.Us + v * nc + e, sizeof(double));
    for (int s = 0; s < 4; s++)
      __pipeline_memcpy_async(col + (24 + s) * kCornerBlock, d.corr + s * (size_t)d.nquad + iq, sizeof(double));
    __pipeline_commit();
  }
#define CF_U(q, k) col[((q) * 6 + (k)) * kCornerBlock]
#define CF_CORR(s) col[(24 + (s)) * kCornerBlock]
  const double eps = 1.0e-6, g = d.gamlg, slpdu = (g + 1.0) / 2.0;
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  const CellGeo G{d.rc[e], d.sc[e], d.g19[e], d.g20[e], d.g21[e]};
  __pipeline_wait_prior(0);
  const double rhoct = 1.0 / CF_U(0, 0);
  const double pctr =
      fmax(eps, (g - 1.0) * rhoct * (CF_U(3, 0) - 0.5 * (CF_U(1, 0) * CF_U(1, 0) + CF_U(2, 0) * CF_U(2, 0))));
  const double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
#pragma unroll
  for (int k = 0; k < 9; k++) {
    double b[6];
    node_basis2(G, k, b);
    double st[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      double acc = 0.0;
#pragma unroll
      for (int kk = 0; kk < 6; kk++)
        if (kk < d.mdegr) acc += CF_U(q, kk) * b[kk];
      st[q] = acc;
    }
    const double rhovt = 1.0 / st[0];
    const double ke = st[3] - 0.5 * (st[1] * st[1] + st[2] * st[2]);
    const int pn = d.ipq[k * d.nquad + iq];
    const double dux = d.us[pn] - st[1];
    const double duy = d.vs[pn] - st[2];
    double P0 = 0.0, P1 = 0.0, P2 = 0.0, P3 = 0.0, P4 = 0.0;
#pragma unroll
    for (int i = nc_start(k); i < nc_start(k + 1); i++) {
      const int isg = nc_entry(i) >> 2, ivsg = nc_entry(i) & 3;
      const double pv = fmax(eps, (g - 1.0) * (rhovt + CF_CORR(isg)) * ke);
#pragma unroll
      for (int f = 0; f < 2; f++) {
        double ax, ay;
        corner_an(L.X, L.Y, isg, ivsg, f, ax, ay);
        const double w = wrie(isg, ivsg, f);
        const double m = corner_m(rhoct, sdctr, d.cimpd, slpdu, dux, duy, ax, ay, w);
        const double pw = -2.0 * pv * w;  // sigma . n A w = -p 2 w an
        P0 += m;
        P1 += m * st[1];
        P2 += m * st[2];
        P3 += pw * ax;
        P4 += pw * ay;
      }
    }
    if (live) {
      d.npart[(0 * 9 + k) * (size_t)d.nquad + iq] = P0;
      d.npart[(1 * 9 + k) * (size_t)d.nquad + iq] = P1;
      d.npart[(2 * 9 + k) * (size_t)d.nquad + iq] = P2;
      d.npart[(3 * 9 + k) * (size_t)d.nquad + iq] = P3;
      d.npart[(4 * 9 + k) * (size_t)d.nquad + iq] = P4;
    }
    // keep the block's warps on the same stretch of this long unrolled code
    // (fewer instruction-fetch stalls: 1.233 -> 1.188 ms per step for the
    // corner pass on the 1024x1024 Taylor-Green mesh)
    __syncthreads();
  }
#undef CF_U
#undef CF_CORR
}

// ---------------------------------------------------------------------------
// Node pass: gather the per-cell partial sums in cell order, 2x2 solve and
// wall conditions (getndvelo_lagsubg, Getrhslaggauss.f90:4465-4545)
// ---------------------------------------------------------------------------
__host__ __device__ void f_node(const Dev &d, int p) {
  if (p >= d.npoin || d.sc_dev->done) return;
  double mn = 0.0, mu0 = 0.0, mu1 = 0.0, sn0 = 0.0, sn1 = 0.0;
  const int b = d.node_ptr2[p], en = d.node_ptr2[p + 1];
  for (int i = b; i < en; i++) {
    const int id = d.node_slot[i];
    if (id < 0) {  // triangle: -1 - (it*6 + k), partials of its node k
      const int t = -1 - id, it = t / 6, k = t - 6 * it;
      const size_t nt = d.ntria;
      mn += d.tpart[(0 * 6 + k) * nt + it];
      mu0 += d.tpart[(1 * 6 + k) * nt + it];
      mu1 += d.tpart[(2 * 6 + k) * nt + it];
      sn0 += d.tpart[(3 * 6 + k) * nt + it];
      sn1 += d.tpart[(4 * 6 + k) * nt + it];
      continue;
    }
    const int iq = id / 9, k = id - 9 * iq;
    mn += d.npart[(0 * 9 + k) * (size_t)d.nquad + iq];
    mu0 += d.npart[(1 * 9 + k) * (size_t)d.nquad + iq];
    mu1 += d.npart[(2 * 9 + k) * (size_t)d.nquad + iq];
    sn0 += d.npart[(3 * 9 + k) * (size_t)d.nquad + iq];
    sn1 += d.npart[(4 * 9 + k) * (size_t)d.nquad + iq];
  }
  const unsigned char mask = d.bcmask[p];
  double us = d.us[p], vs = d.vs[p];
  if (!(mask & 4)) {
    us = (mu0 - sn0) / mn;
    vs = (mu1 - sn1) / mn;
  }
  if (mask & 1) us = 0.0;
  if (mask & 2) vs = 0.0;
  d.us_new[p] = us;
  d.vs_new[p] = vs;
}

// ---------------------------------------------------------------------------
// RHS pass: corner forces + face integral + volume integral (+ source), and
// in stages 2 and 3 the M^-1 solve and RK combine
// ---------------------------------------------------------------------------

// The momentum and energy face weights of rhsifacedg_lagsubgq2 are 1 on every
// corner entry of the 8 boundary nodes of the quad and 0 on the 4 entries of
// the centre node (Getrhslaggauss.f90:8580-8603), and the mass weights vanish
// on the centre node's corner faces; the face integral below relies on both.
constexpr FastTables kFastTablesC = LAG2D_FAST_TABLES;
constexpr int node_wmom(int k) {
  int ones = 0, zeros = 0;
  for (int i = kFastTablesC.nc_start[k]; i < kFastTablesC.nc_start[k + 1]; i++) {
    const double w = kFastTablesC.wmom[kFastTablesC.nc_entry[i]];
    ones += w == 1.0;
    zeros += w == 0.0;
  }
  return zeros == 0 ? 1 : (ones == 0 ? 0 : -1);
}
static_assert(node_wmom(0) == 1 && node_wmom(1) == 1 && node_wmom(2) == 1 && node_wmom(3) == 1 &&
              node_wmom(4) == 1 && node_wmom(5) == 1 && node_wmom(6) == 1 && node_wmom(7) == 1 &&
              node_wmom(8) == 0, "momentum face weights: 1 on the boundary nodes, 0 at the centre");
constexpr bool centre_wmas_zero() {
  for (int i = kFastTablesC.nc_start[8]; i < kFastTablesC.nc_start[9]; i++)
    for (int f = 0; f < 2; f++)
      if (kFastTablesC.wmas[2 * kFastTablesC.nc_entry[i] + f] != 0.0) return false;
  return true;
}
static_assert(centre_wmas_zero(), "mass face weights vanish at the centre node");

// Mass-flux weights of node k (0..7): t = sum over the node's outer corner
// faces of 2 w_mass,f an_f, so that the node's mass flux is u* . t.
__host__ __device__ __forceinline__ void mass_flux_weights(const Loaded &L, int k, double &tx, double &ty) {
  tx = 0.0;
  ty = 0.0;
#pragma unroll
  for (int i = nc_start(k); i < nc_start(k + 1); i++) {
    const int isg = nc_entry(i) >> 2, ivsg = nc_entry(i) & 3;
#pragma unroll
    for (int f = 0; f < 2; f++) {
      if (wmas(isg, ivsg, f) != 0.0) {
        double ax, ay;
        corner_an(L.X, L.Y, isg, ivsg, f, ax, ay);
        tx += ax * (2.0 * wmas(isg, ivsg, f));
        ty += ay * (2.0 * wmas(isg, ivsg, f));
      }
    }
  }
}

// RHS pass, one kernel per quad: face integral, volume integral, Taylor-Green
// source, and either the RHS store or the M^-1 solve and RK combine.
//
// Face integral (rhsifacedg_lagsubgq2, Getrhslaggauss.f90:8501-8748).  At node
// k the corner force of corner face f is F_f = sigma.n A w_f + m_f (u* - u_k),
// with u* the node's new velocity and m_f, sigma.n A w_f, u_k what the corner
// pass used (Getrhslaggauss.f90:10409-10867).  The momentum sum is therefore
// affine in u*: sum_f F_f = (P3, P4) + u* P0 - (P1, P2), where P0..P4 are the
// node partial sums the corner pass wrote (sum m, sum m u_k, sum m v_k, sum
// sigma.n A w); the energy term is u* . sum_f F_f; the mass term is
// u* . sum_f 2 w_mass,f an_f over the 16 outer corner faces.  So the corner
// data are not recomputed here: 40 partials and the 8 boundary nodes'
// velocities replace the 32 corner faces' vertex states, impedances and
// forces (same sums up to rounding and summation order).
//
// Staging: the cell's DOFs U^(s) (24 values) and, for the fused update, M^-1
// (16) and U^n (24) are copied asynchronously (cp.async) into this thread's
// column of shared memory (stride kRhsBlock) when the thread starts, so their
// load latency overlaps the face integral and they are read from shared
// memory where used instead of being held in registers.
constexpr int kRhsBlock = 128;
constexpr int kRhsStage = 64;
__device__ void f_rhs3(const Dev &d, int iq, int fuse_update, double alfa, double *col) {
  if (iq >= d.nquad || d.sc_dev->done) return;
  const int e = iq + d.ntria;
  const double eps = 1.0e-6, g = d.gamlg;
  {
    const size_t nc = d.ncell;
    for (int v = 0; v < 24; v++) __pipeline_memcpy_async(col + v * kRhsBlock, d.Us + v * nc + e, sizeof(double));
    if (fuse_update) {
      for (int i = 0; i < 16; i++)
        __pipeline_memcpy_async(col + (24 + i) * kRhsBlock, d.amatr + i * nc + e, sizeof(double));
      for (int v = 0; v < 24; v++)
        __pipeline_memcpy_async(col + (40 + v) * kRhsBlock, d.Un + v * nc + e, sizeof(double));
    }
    __pipeline_commit();
    // the node partial sums of the 8 boundary nodes (and the source moments)
    // towards L2 while the coordinates are gathered: their loads in the face
    // loop then wait on L2, not HBM (RHS pass 1.635 -> 1.507 ms per step on
    // the 1024x1024 Taylor-Green mesh)
    const size_t nq = d.nquad;
#pragma unroll
    for (int v = 0; v < 5; v++)
#pragma unroll
      for (int k = 0; k < 8; k++) asm volatile("prefetch.global.L2 [%0];" ::"l"(d.npart + (v * 9 + k) * nq + iq));
    if (d.ncase == 1) {
#pragma unroll
      for (int k = 0; k < 6; k++) asm volatile("prefetch.global.L2 [%0];" ::"l"(d.src + k * nq + iq));
    }
  }
#define RHS_U(q, k) col[((q) * 6 + (k)) * kRhsBlock]
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  const CellGeo G{d.rc[e], d.sc[e], d.g19[e], d.g20[e], d.g21[e]};
  double ul[6] = {0, 0, 0, 0, 0, 0}, p0[6] = {0, 0, 0, 0, 0, 0}, p1[6] = {0, 0, 0, 0, 0, 0}, el[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 8; k++) {
    double b[6];
    node_basis2(G, k, b);
    const int pn = d.ipq[k * d.nquad + iq];
    const double un = d.us_new[pn], vn = d.vs_new[pn];
    double tx, ty;
    mass_flux_weights(L, k, tx, ty);
    const double tw = un * tx + vn * ty;
    const size_t nq = d.nquad;
    const double P0 = d.npart[(0 * 9 + k) * nq + iq], P1 = d.npart[(1 * 9 + k) * nq + iq];
    const double P2 = d.npart[(2 * 9 + k) * nq + iq], P3 = d.npart[(3 * 9 + k) * nq + iq];
    const double P4 = d.npart[(4 * 9 + k) * nq + iq];
    const double f0 = P3 + (un * P0 - P1);
    const double f1 = P4 + (vn * P0 - P2);
    const double fe = un * f0 + vn * f1;
#pragma unroll
    for (int kk = 0; kk < 6; kk++) {
      ul[kk] += tw * b[kk];
      p0[kk] += f0 * b[kk];
      p1[kk] += f1 * b[kk];
      el[kk] += fe * b[kk];
    }
  }
  __pipeline_wait_prior(0);
  // volume integral on the 5x5 Gauss-Lobatto grid (cofactor form), sum
  // factorised row by row: for fixed r_i, Q_b = sum_a L'_a(r_i) X[a][b] and
  // P_b = sum_a L_a(r_i) X[a][b] give dx/dr and dx/ds along the row
#pragma unroll 1
  for (int i = 0; i < 5; i++) {
    const double r = l5p(i), dr = r - G.rc;
    double lr[3], dlr[3];
    lag3(r, lr);
    dlag3(r, dlr);
    double Qx[3], Qy[3], Px[3], Py[3];
#pragma unroll
    for (int bb = 0; bb < 3; bb++) {
      Qx[bb] = dlr[0] * L.X[0][bb] + dlr[1] * L.X[1][bb] + dlr[2] * L.X[2][bb];
      Qy[bb] = dlr[0] * L.Y[0][bb] + dlr[1] * L.Y[1][bb] + dlr[2] * L.Y[2][bb];
      Px[bb] = lr[0] * L.X[0][bb] + lr[1] * L.X[1][bb] + lr[2] * L.X[2][bb];
      Py[bb] = lr[0] * L.Y[0][bb] + lr[1] * L.Y[1][bb] + lr[2] * L.Y[2][bb];
    }
    // the DOFs along the row: u_q(s) = a_q + ds (b_q + c_q ds), ds = s - sc
    double ra[4], rb[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      ra[q] = RHS_U(q, 0) + RHS_U(q, 1) * dr + RHS_U(q, 3) * (0.5 * dr * dr - G.g19) - RHS_U(q, 4) * G.g20 -
              RHS_U(q, 5) * G.g21;
      rb[q] = RHS_U(q, 2) + RHS_U(q, 5) * dr;
    }
    const double wi = l5w(i);
    // 1/tau at the row's 5 points with one division (batched reciprocals:
    // prefix products, one reciprocal of the last, then back substitution)
    double rtau[5];
    {
      double tq[5], pre[5];
#pragma unroll
      for (int j = 0; j < 5; j++) {
        const double ds = l5p(j) - G.sc;
        tq[j] = ra[0] + ds * (rb[0] + 0.5 * RHS_U(0, 4) * ds);
        pre[j] = j == 0 ? tq[0] : pre[j - 1] * tq[j];
      }
      double inv = 1.0 / pre[4];
#pragma unroll
      for (int j = 4; j > 0; j--) {
        rtau[j] = inv * pre[j - 1];
        inv = inv * tq[j];
      }
      rtau[0] = inv;
    }
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const double s = l5p(j), ds = s - G.sc;
      double ls[3], dls[3];
      lag3(s, ls);
      dlag3(s, dls);
      const double w = wi * l5w(j);
      const double xr = Qx[0] * ls[0] + Qx[1] * ls[1] + Qx[2] * ls[2];
      const double yr = Qy[0] * ls[0] + Qy[1] * ls[1] + Qy[2] * ls[2];
      const double xs = Px[0] * dls[0] + Px[1] * dls[1] + Px[2] * dls[2];
      const double ys = Py[0] * dls[0] + Py[1] * dls[1] + Py[2] * dls[2];
      double un[4];
#pragma unroll
      for (int q = 1; q < 4; q++) un[q] = ra[q] + ds * (rb[q] + 0.5 * RHS_U(q, 4) * ds);
      const double rhoad = rtau[j];
      const double pres = fmax(eps, (g - 1.0) * rhoad * (un[3] - 0.5 * (un[1] * un[1] + un[2] * un[2])));
      // G . grad_xi b for b = 2..6: dbdr = (1, 0, dr, 0, ds), dbds = (0, 1, 0, ds, dr)
      // (the FP32-mixed kernel sums these per row instead; here the row sums'
      // 16 extra accumulators cost more in spills than the 16 operations a
      // point they save)
      double gd0[5], gd1[5];
      gd0[0] = ys;       gd1[0] = -xs;
      gd0[1] = -yr;      gd1[1] = xr;
      gd0[2] = ys * dr;  gd1[2] = -xs * dr;
      gd0[3] = -yr * ds; gd1[3] = xr * ds;
      gd0[4] = ys * ds - yr * dr;
      gd1[4] = -xs * ds + xr * dr;
      const double wp = w * pres;
#pragma unroll
      for (int kk = 0; kk < 5; kk++) {
        const double fv = gd0[kk] * un[1] + gd1[kk] * un[2];
        ul[kk + 1] -= fv * w;
        p0[kk + 1] += gd0[kk] * wp;
        p1[kk + 1] += gd1[kk] * wp;
        el[kk + 1] += fv * wp;
      }
    }
  }
  if (d.ncase == 1) {
    // Taylor-Green energy source, computed by k_tgv_src2 before the corner pass
#pragma unroll
    for (int k = 0; k < 6; k++) el[k] += d.src[k * (size_t)d.nquad + iq];
  }
  if (!fuse_update) {
#pragma unroll
    for (int k = 0; k < 6; k++) {
      d.rhs[(0 * 6 + k) * (size_t)d.ncell + e] = ul[k];
      d.rhs[(1 * 6 + k) * (size_t)d.ncell + e] = p0[k];
      d.rhs[(2 * 6 + k) * (size_t)d.ncell + e] = p1[k];
      d.rhs[(3 * 6 + k) * (size_t)d.ncell + e] = el[k];
    }
    return;
  }
  // fused stage update (Getrhslag.f90:1789-1904)
  const double dt = d.sc_dev->dtfix;
#define RHS_AM(i) col[(24 + (i)) * kRhsBlock]
#define RHS_UN(v) col[(40 + (v)) * kRhsBlock]
  double R[4][6];
#pragma unroll
  for (int k = 0; k < 6; k++) {
    R[0][k] = dt * ul[k];
    R[1][k] = dt * p0[k];
    R[2][k] = dt * p1[k];
    R[3][k] = dt * el[k];
  }
  const double oma = 1.0 - alfa;
  // symmetric 5x5 block rows from the packed upper triangle, M(1,1) = amatr(16)
  const int IDX[5][5] = {{0, 1, 2, 3, 4}, {1, 5, 6, 7, 8}, {2, 6, 9, 10, 11}, {3, 7, 10, 12, 13}, {4, 8, 11, 13, 14}};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const size_t base = (size_t)(q * 6) * d.ncell + e;
    const double d0 = RHS_AM(15) * R[q][0];
    d.Us[base] = alfa * RHS_UN(q * 6) + oma * (RHS_U(q, 0) + d0);
#pragma unroll
    for (int i = 0; i < 5; i++) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < 5; j++) acc += RHS_AM(IDX[i][j]) * R[q][j + 1];
      const size_t idx = base + (size_t)(i + 1) * d.ncell;
      d.Us[idx] = alfa * RHS_UN(q * 6 + i + 1) + oma * (RHS_U(q, i + 1) + acc);
    }
  }
#undef RHS_U
#undef RHS_AM
#undef RHS_UN
}

// getdelt_lag's per-quad limits (Getrhslag.f90:20641-20700) before the RHS
// pass of stage 1: dvdt = rhsel(1,1,ielem) is the cell-average mass flux,
// which only the face integral contributes to (the volume integral has no
// moment-0 term and the source acts on the energy), i.e. sum_k u*_k . t_k
// with the same per-node sums as f_rhs3.  With dt known before the RHS pass,
// stage 1 fuses its M^-1 solve and update into the RHS kernel like the later
// stages.  Edge lengths use the stage's nodes, which in stage 1 are x^n.
__host__ __device__ void f_dt_quad(const Dev &d, int iq, double &dtcfl, double &dtvol) {
  dtcfl = 1e10;
  dtvol = 1e10;
  if (iq >= d.nquad || d.sc_dev->done) return;
  const int e = iq + d.ntria;
  const double eps = 1.0e-6, g = d.gamlg;
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  double dvdt = 0.0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int pn = d.ipq[k * d.nquad + iq];
    double tx, ty;
    mass_flux_weights(L, k, tx, ty);
    dvdt += d.us_new[pn] * tx + d.vs_new[pn] * ty;
  }
  double xp[9][2];
  node_xy(L, xp);
  // curved edges: corner - mid-edge node - corner
  const int ed[4][3] = {{0, 4, 1}, {1, 5, 2}, {2, 6, 3}, {3, 7, 0}};
  double dlen = 0.0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const double *a = xp[ed[k][0]], *b = xp[ed[k][1]], *c = xp[ed[k][2]];
    const double dl = sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1])) +
                      sqrt((b[0] - c[0]) * (b[0] - c[0]) + (b[1] - c[1]) * (b[1] - c[1]));
    if (k == 0 || dl < dlen) dlen = dl;
  }
  const size_t nc = d.ncell;
  const double rhomc = d.Us[0 * nc + e];
  const double uctr = d.Us[6 * nc + e], vctr = d.Us[12 * nc + e], ectr = d.Us[18 * nc + e];
  const double rhoct = 1.0 / rhomc;
  const double pctr = fmax(eps, (g - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
  const double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
  dtcfl = dlen / sdctr;
  dtvol = d.vol[e] / fabs(dvdt);
}

// Node motion with the new ustar, which becomes the previous ustar of the next stage
__host__ __device__ void f_nodes(const Dev &d, int p, double alfa) {
  if (p >= d.npoin || d.sc_dev->done) return;
  const double dt = d.sc_dev->dtfix;
  const double oma = 1.0 - alfa;
  const double un = d.us_new[p], vn = d.vs_new[p];
  d.xs[p] = alfa * d.xn[p] + oma * (d.xs[p] + dt * un);
  d.ys[p] = alfa * d.yn[p] + oma * (d.ys[p] + dt * vn);
  d.us[p] = un;
  d.vs[p] = vn;
}

// Centre-node re-interpolation and the exact cell volume
__host__ __device__ void f_geom(const Dev &d, int iq, int fix_centre) {
  if (iq >= d.nquad || d.sc_dev->done) return;
  const int e = iq + d.ntria;
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  if (fix_centre) {
    // X[1][1] is node 9; corners X[0|2][0|2], edge nodes X[1][0], X[2][1], X[1][2], X[0][1]
    L.X[1][1] = -0.25 * (L.X[0][0] + L.X[2][0] + L.X[2][2] + L.X[0][2]) + 0.5 * (L.X[1][0] + L.X[2][1] + L.X[1][2] + L.X[0][1]);
    L.Y[1][1] = -0.25 * (L.Y[0][0] + L.Y[2][0] + L.Y[2][2] + L.Y[0][2]) + 0.5 * (L.Y[1][0] + L.Y[2][1] + L.Y[1][2] + L.Y[0][1]);
    const int pc = d.ipq[8 * d.nquad + iq];
    d.xs[pc] = L.X[1][1];
    d.ys[pc] = L.Y[1][1];
  }
  double c[36], D[16];
  {
    double xp[9][2];
    node_xy_rel(L, xp);
    cross36_rel(xp, c);
  }
  detpoly(c, D);
  const double vol = cell_area(D);
  d.vol[e] = vol;
  if (!(vol > 0.0)) {
#ifdef __CUDA_ARCH__
    atomicOr(&d.sc_dev->status, ST_NONPHYS);
#else
    d.sc_dev->status |= ST_NONPHYS;
#endif
  }
}

// Time-invariant mass-weighted shape moments W_k = sum_g rho0 J0_g N_k(g)
// (5x5 Gauss on the initial map) for the physical mass centre
__host__ __device__ void f_init_wmom(const Dev &d, int iq) {
  if (iq >= d.nquad) return;
  Loaded L;
  load_cell(d, d.x0, d.y0, iq, L);
  double c[36], D[16];
  {
    double xp[9][2];
    node_xy_rel(L, xp);
    cross36_rel(xp, c);
  }
  detpoly(c, D);
  // initial density of the reference cases is uniform per cell
  double rho0 = d.rho0 ? d.rho0[iq + d.ntria] : 1.0;
  if (d.ncase == 6) {
    const double xc = L.X[1][1], yc = L.Y[1][1];
    rho0 *= (sqrt(xc * xc + yc * yc) <= 0.5) ? 1.0 : 0.125;
  }
  double W[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) W[a][b] = 0.0;
  for (int i = 0; i < 5; i++) {
    double lr[3];
    lag3(g5p(i), lr);
    for (int j = 0; j < 5; j++) {
      double ls[3];
      lag3(g5p(j), ls);
      const double w = rho0 * g5w(i) * g5w(j) * deteval(D, g5p(i), g5p(j));
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) W[a][b] += w * lr[a] * ls[b];
    }
  }
  const int A[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
  const int B[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
  for (int k = 0; k < 9; k++) d.wmom[k * (size_t)d.nquad + iq] = W[A[k]][B[k]];
}

// ---------------------------------------------------------------------------
// Adjoint (reverse mode) of the optimised FP64 stage on all-quad meshes.
//
// The stage maps (U^(s), x^(s), u*_prev) through the corner pass, the node
// solve, the RHS pass, the RK update and the node motion to the next stage;
// each kernel below is the transpose of one of those maps at a recorded
// forward state (the stage inputs are restored into Dev before the launch).
// The time step size, the Persson marks and the WENO active set are frozen
// from the forward pass (the adjoint is only formed when no cell is troubled,
// so WENO is the identity).  Derivatives of max(eps, .) are taken on the
// active branch; the impedance's jump-direction branch (|u* - u_c| >= 1e12 c)
// is taken as the regular one.
// ---------------------------------------------------------------------------

// transpose of cross36: c[p] = x_i y_j - x_j y_i
__host__ __device__ __forceinline__ void cross36_T(const double (*xp)[2], const double *lc, double (*lxp)[2]) {
  int p = 0;
  for (int i = 0; i < 9; i++)
    for (int j = i + 1; j < 9; j++, p++) {
      lxp[i][0] += lc[p] * xp[j][1];
      lxp[j][1] += lc[p] * xp[i][0];
      lxp[j][0] -= lc[p] * xp[i][1];
      lxp[i][1] -= lc[p] * xp[j][0];
    }
}

// transpose of slot_an (a linear map of the tensor coordinates)
__host__ __device__ __forceinline__ void slot_an_T(int slot, double lax, double lay, double lX[3][3], double lY[3][3]) {
  if (slot >= 8 && slot < 12) {
    // ax = -dydr, ay = dxdr, d.dr = -1.5 e - 0.5 c + 2 v with v = l0 q0 + l1 q1 + l2 q2
    const int f = slot - 8;
    const double ldx = lay, ldy = -lax;
    const double lm[3] = {0.375, 0.75, -0.125}, lp[3] = {-0.125, 0.75, 0.375};
    lX[1][1] += -0.5 * ldx;
    lY[1][1] += -0.5 * ldy;
    if (f == 0) {
      lX[1][0] += -1.5 * ldx; lY[1][0] += -1.5 * ldy;
      for (int t = 0; t < 3; t++) { lX[1][t] += 2.0 * lm[t] * ldx; lY[1][t] += 2.0 * lm[t] * ldy; }
    } else if (f == 1) {
      lX[2][1] += -1.5 * ldx; lY[2][1] += -1.5 * ldy;
      for (int t = 0; t < 3; t++) { lX[t][1] += 2.0 * lp[t] * ldx; lY[t][1] += 2.0 * lp[t] * ldy; }
    } else if (f == 2) {
      lX[1][2] += -1.5 * ldx; lY[1][2] += -1.5 * ldy;
      for (int t = 0; t < 3; t++) { lX[1][t] += 2.0 * lp[t] * ldx; lY[1][t] += 2.0 * lp[t] * ldy; }
    } else {
      lX[0][1] += -1.5 * ldx; lY[0][1] += -1.5 * ldy;
      for (int t = 0; t < 3; t++) { lX[t][1] += 2.0 * lm[t] * ldx; lY[t][1] += 2.0 * lm[t] * ldy; }
    }
    return;
  }
  const int ig = slot < 8 ? slot : slot - 4;
  const FastTables &T = FT();
  const int ia = T.pa[ig], ib = T.pb[ig];
  const double *da = T.dl + 3 * ia, *db = T.dl + 3 * ib;
  double lxr = 0, lyr = 0, lxs = 0, lys = 0;
  switch (T.side[ig]) {
    case 0: lyr += lax; lxr -= lay; break;   // ax = yr, ay = -xr
    case 1: lys += lax; lxs -= lay; break;   // ax = ys, ay = -xs
    case 2: lyr -= lax; lxr += lay; break;   // ax = -yr, ay = xr
    default: lys -= lax; lxs += lay; break;  // ax = -ys, ay = xs
  }
  // xr = sum_t da[t] X[t][ib], xs = sum_t db[t] X[ia][t]; column ib and row
  // ia are selected with (warp-uniform) branches so that lX, lY stay in
  // registers
  const double cx0 = da[0] * lxr, cx1 = da[1] * lxr, cx2 = da[2] * lxr;
  const double cy0 = da[0] * lyr, cy1 = da[1] * lyr, cy2 = da[2] * lyr;
  if (ib == 0) { lX[0][0] += cx0; lX[1][0] += cx1; lX[2][0] += cx2; lY[0][0] += cy0; lY[1][0] += cy1; lY[2][0] += cy2; }
  else if (ib == 1) { lX[0][1] += cx0; lX[1][1] += cx1; lX[2][1] += cx2; lY[0][1] += cy0; lY[1][1] += cy1; lY[2][1] += cy2; }
  else { lX[0][2] += cx0; lX[1][2] += cx1; lX[2][2] += cx2; lY[0][2] += cy0; lY[1][2] += cy1; lY[2][2] += cy2; }
  const double rx0 = db[0] * lxs, rx1 = db[1] * lxs, rx2 = db[2] * lxs;
  const double ry0 = db[0] * lys, ry1 = db[1] * lys, ry2 = db[2] * lys;
  if (ia == 0) { lX[0][0] += rx0; lX[0][1] += rx1; lX[0][2] += rx2; lY[0][0] += ry0; lY[0][1] += ry1; lY[0][2] += ry2; }
  else if (ia == 1) { lX[1][0] += rx0; lX[1][1] += rx1; lX[1][2] += rx2; lY[1][0] += ry0; lY[1][1] += ry1; lY[1][2] += ry2; }
  else { lX[2][0] += rx0; lX[2][1] += rx1; lX[2][2] += rx2; lY[2][0] += ry0; lY[2][1] += ry1; lY[2][2] += ry2; }
}
// entry isg of a 4-vector with a warp-uniform index, without local memory
__host__ __device__ __forceinline__ double pick4(const double v[4], int i) {
  return i == 0 ? v[0] : i == 1 ? v[1] : i == 2 ? v[2] : v[3];
}
__host__ __device__ __forceinline__ void add4(double v[4], int i, double x) {
  if (i == 0) v[0] += x;
  else if (i == 1) v[1] += x;
  else if (i == 2) v[2] += x;
  else v[3] += x;
}

__host__ __device__ __forceinline__ void corner_an_T(int isg, int ivsg, int f, double lax, double lay, double lX[3][3],
                                                     double lY[3][3]) {
  const int code = fnqsg2(isg, 2 * ivsg + f);
  const int slot = (code >= 0 ? code : -code) - 1;
  if (code < 0) { lax = -lax; lay = -lay; }
  slot_an_T(slot, lax, lay, lX, lY);
}

// transpose of corner_m (regular branch): m = 2 w (rho c nn + cimpd rho slpdu |dn|)
__host__ __device__ __forceinline__ void corner_m_T(double rhoct, double sdctr, double cimpd, double slpdu, double dux,
                                                    double duy, double ax, double ay, double w, double lm,
                                                    double &lrho, double &lsd, double &ldux, double &lduy,
                                                    double &lax, double &lay) {
  const double nn2 = ax * ax + ay * ay;
  const double rnn = rsqrt(nn2), nn = nn2 * rnn;
  const double dn = dux * ax + duy * ay;
  const double adn = fabs(dn), sg = dn >= 0.0 ? 1.0 : -1.0;
  lrho += lm * 2.0 * w * (sdctr * nn + cimpd * slpdu * adn);
  lsd += lm * 2.0 * w * rhoct * nn;
  const double lnn = lm * 2.0 * w * rhoct * sdctr * rnn;
  lax += lnn * ax;
  lay += lnn * ay;
  const double ldn = lm * 2.0 * w * cimpd * rhoct * slpdu * sg;
  ldux += ldn * ax;
  lduy += ldn * ay;
  lax += ldn * dux;
  lay += ldn * duy;
}

// transpose of the cell-centre state: rhoct = 1/tau, pctr = max(eps, ...),
// sdctr = sqrt(max(eps, g pctr / rhoct)); adds into lu
__host__ __device__ __forceinline__ void centre_T(const double u[4][6], double g, double lrho_in, double lsd,
                                                  double lu[4][6]) {
  const double eps = 1.0e-6;
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

// vertex state transpose: st[q] = sum_{k<mdegr} u[q][k] b[k], rhovt = 1/st0,
// ke = st3 - (st1^2 + st2^2)/2
__host__ __device__ __forceinline__ void vertex_T(const double *b, int mdegr, const double st[4], double lrhovt,
                                                  double lke, double lst1, double lst2, double lu[4][6]) {
  double lst[4];
  lst[0] = -lrhovt / (st[0] * st[0]);
  lst[1] = lst1 - lke * st[1];
  lst[2] = lst2 - lke * st[2];
  lst[3] = lke;
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++)
      if (k < mdegr) lu[q][k] += lst[q] * b[k];
}

// Reverse of the corner pass of quad iq, in two kernels like the forward
// pass.  First the corner faces: reads the node-sum adjoints lS at its nodes
// plus the RHS pass's adjoints of its partials (lP); adds the cell DOF
// adjoint into lU, writes the node contributions (x, y, u*_prev, v*_prev)
// into pbuf and the adjoints of the 4 sub-cell density corrections into
// lcorr.  Without the det J polynomial, sub-cell areas and masses the
// corrections' transpose needs, it holds far fewer values across its 32
// unrolled faces.
__host__ __device__ void a_corner_faces(const Dev &d, const Adj &a, int iq) {
  if (iq >= d.nquad) return;
  const int e = iq + d.ntria;
  const size_t nq = d.nquad;
  const double eps = 1.0e-6, g = d.gamlg, slpdu = (g + 1.0) / 2.0;
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  const CellGeo G{d.rc[e], d.sc[e], d.g19[e], d.g20[e], d.g21[e]};
  double u[4][6];
  load_u(d, d.Us, e, u);
  const double rhoct = 1.0 / u[0][0];
  const double pctr = fmax(eps, (g - 1.0) * rhoct * (u[3][0] - 0.5 * (u[1][0] * u[1][0] + u[2][0] * u[2][0])));
  const double sdctr = sqrt(fmax(eps, g * pctr / rhoct));
  // the stage's sub-cell density corrections come from the forward pass
  double corr[4];
#pragma unroll
  for (int isg = 0; isg < 4; isg++) corr[isg] = d.corr[isg * nq + iq];
  double lu[4][6];
  for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) lu[q][k] = 0.0;
  double lX[3][3], lY[3][3];
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) { lX[i][j] = 0.0; lY[i][j] = 0.0; }
  double lrho = 0.0, lsd = 0.0, lcr[4] = {0, 0, 0, 0};
  for (int k = 0; k < 9; k++) {
    double b[6];
    node_basis2(G, k, b);
    double st[4];
    for (int q = 0; q < 4; q++) {
      double acc = 0.0;
      for (int kk = 0; kk < 6; kk++)
        if (kk < d.mdegr) acc += u[q][kk] * b[kk];
      st[q] = acc;
    }
    const double rhovt = 1.0 / st[0];
    const double ke = st[3] - 0.5 * (st[1] * st[1] + st[2] * st[2]);
    const int pn = d.ipq[k * d.nquad + iq];
    const double dux = d.us[pn] - st[1], duy = d.vs[pn] - st[2];
    // adjoint of this quad's partials at node k: through the node sums (node
    // solve) and directly through the RHS pass's face integral
    const double lP0 = a.lS[0 * (size_t)d.npoin + pn] + a.lP[(0 * 9 + k) * nq + iq];
    const double lP1 = a.lS[1 * (size_t)d.npoin + pn] + a.lP[(1 * 9 + k) * nq + iq];
    const double lP2 = a.lS[2 * (size_t)d.npoin + pn] + a.lP[(2 * 9 + k) * nq + iq];
    const double lP3 = a.lS[3 * (size_t)d.npoin + pn] + a.lP[(3 * 9 + k) * nq + iq];
    const double lP4 = a.lS[4 * (size_t)d.npoin + pn] + a.lP[(4 * 9 + k) * nq + iq];
    double lst1 = 0, lst2 = 0, lrhovt = 0, lke = 0, ldux = 0, lduy = 0;
    for (int i = nc_start(k); i < nc_start(k + 1); i++) {
      const int isg = nc_entry(i) >> 2, ivsg = nc_entry(i) & 3;
      const double ci = pick4(corr, isg);
      const double pe = (g - 1.0) * (rhovt + ci) * ke;
      const double pv = fmax(eps, pe);
      double lpv = 0.0;
      for (int f = 0; f < 2; f++) {
        double ax, ay;
        corner_an(L.X, L.Y, isg, ivsg, f, ax, ay);
        const double w = wrie(isg, ivsg, f);
        const double m = corner_m(rhoct, sdctr, d.cimpd, slpdu, dux, duy, ax, ay, w);
        const double pw = -2.0 * pv * w;
        const double lm = lP0 + lP1 * st[1] + lP2 * st[2];
        lst1 += lP1 * m;
        lst2 += lP2 * m;
        const double lpw = lP3 * ax + lP4 * ay;
        double lax = lP3 * pw, lay = lP4 * pw;
        lpv += -2.0 * w * lpw;
        corner_m_T(rhoct, sdctr, d.cimpd, slpdu, dux, duy, ax, ay, w, lm, lrho, lsd, ldux, lduy, lax, lay);
        corner_an_T(isg, ivsg, f, lax, lay, lX, lY);
      }
      if (pe > eps) {
        lrhovt += lpv * (g - 1.0) * ke;
        add4(lcr, isg, lpv * (g - 1.0) * ke);
        lke += lpv * (g - 1.0) * (rhovt + ci);
      }
    }
    // dux = us - st1, duy = vs - st2
    double *pb = a.pbuf;
    pb[(2 * 9 + k) * nq + iq] = ldux;
    pb[(3 * 9 + k) * nq + iq] = lduy;
    lst1 -= ldux;
    lst2 -= lduy;
    vertex_T(b, d.mdegr, st, lrhovt, lke, lst1, lst2, lu);
  }
  centre_T(u, g, lrho, lsd, lu);
#pragma unroll
  for (int isg = 0; isg < 4; isg++) a.lcorr[isg * nq + iq] = lcr[isg];
  const int A[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
  const int B[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
  for (int k = 0; k < 9; k++) {
    a.pbuf[(0 * 9 + k) * nq + iq] = lX[A[k]][B[k]];
    a.pbuf[(1 * 9 + k) * nq + iq] = lY[A[k]][B[k]];
    a.pbuf[(4 * 9 + k) * nq + iq] = 0.0;
    a.pbuf[(5 * 9 + k) * nq + iq] = 0.0;
  }
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) a.lU[(q * 6 + k) * (size_t)d.ncell + e] += lu[q][k];
}

// Second part: the transpose of the sub-cell density corrections
// corr = cdrho (msub / vsub - masel / volel) from their adjoints in lcorr;
// adds into the tau DOF adjoints and the node-coordinate contributions.
// The corrections come from the forward pass; the sub-cell masses masel
// are recovered from them and the closed-form volumes volel.
template <typename R>
__host__ __device__ void a_corner_corr(const Dev &d, const Adj &a, int iq) {
  if (iq >= d.nquad) return;
  const int e = iq + d.ntria;
  const size_t nq = d.nquad;
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  double xp[9][2], c[36], D[16];
  node_xy_rel(L, xp);
  cross36_rel(xp, c);
  detpoly(c, D);
  const CellGeo G{d.rc[e], d.sc[e], d.g19[e], d.g20[e], d.g21[e]};
  double u0[6];
#pragma unroll
  for (int k = 0; k < 6; k++) u0[k] = d.Us[k * (size_t)d.ncell + e];
  double vsub4[4], masel4[4], volel4[4], lcr[4];
  subareas(c, vsub4);
#pragma unroll
  for (int isg = 0; isg < 4; isg++) {
    const double corr = d.corr[isg * nq + iq];
    volel4[isg] = det_integral(D, (isg == 0 || isg == 3) ? -1.0 : 0.0, (isg == 0 || isg == 1) ? -1.0 : 0.0);
    const double rho_sub = d.cdrho != 0.0 ? d.msub[isg * nq + iq] / vsub4[isg] - corr / d.cdrho : 0.0;
    masel4[isg] = volel4[isg] * rho_sub;
    lcr[isg] = a.lcorr[isg * nq + iq];
  }
  double lu0[6] = {0, 0, 0, 0, 0, 0};
  // sub-cell density corrections: corr = cdrho (msub / vsub - masel / volel)
  double lD[16], lv4[4] = {0, 0, 0, 0};
  for (int t = 0; t < 16; t++) lD[t] = 0.0;
  for (int isg = 0; isg < 4; isg++) {
    const double lc = lcr[isg];
    const double msub = d.msub[isg * nq + iq];
    lv4[isg] += -d.cdrho * lc * msub / (vsub4[isg] * vsub4[isg]);
    const double lmasel = -d.cdrho * lc / volel4[isg];
    const double lvolel = d.cdrho * lc * masel4[isg] / (volel4[isg] * volel4[isg]);
    // volel = sum_mn D[mn] mr[m] ms[n]
    {
      const double r0 = (isg == 0 || isg == 3) ? -1.0 : 0.0, s0 = (isg == 0 || isg == 1) ? -1.0 : 0.0;
      double mr[4], ms[4];
      const double r1 = r0 + 1.0, s1 = s0 + 1.0;
      double pr0 = r0, pr1 = r1, ps0 = s0, ps1 = s1;
      for (int mm = 0; mm < 4; mm++) {
        mr[mm] = (pr1 - pr0) / (mm + 1);
        ms[mm] = (ps1 - ps0) / (mm + 1);
        pr0 *= r0; pr1 *= r1; ps0 *= s0; ps1 *= s1;
      }
      for (int mm = 0; mm < 4; mm++)
        for (int n = 0; n < 4; n++) lD[4 * mm + n] += lvolel * mr[mm] * ms[n];
    }
    // masel = sum w det / tau, transposed row by row (per-row moments of the
    // det and tau adjoints in s, as in the volume integral)
    const double ofr = (isg == 0 || isg == 3) ? -1.0 : 1.0;
    const double ofs = (isg == 0 || isg == 1) ? -1.0 : 1.0;
#pragma unroll 1
    for (int i = 0; i < 5; i++) {
      const double r = (g5p(i) + ofr) / 2.0, dr = r - G.rc;
      double ee[4];
#pragma unroll
      for (int n = 0; n < 4; n++) ee[n] = D[n] + r * (D[4 + n] + r * (D[8 + n] + r * D[12 + n]));
      const double t0 = u0[0] + u0[1] * dr + u0[3] * (0.5 * dr * dr - G.g19) - u0[4] * G.g20 - u0[5] * G.g21;
      const double t1 = u0[2] + u0[5] * dr, t2 = 0.5 * u0[4];
      // point arithmetic in R (FP32 in the mixed adjoint), rows added in FP64
      const R t0r = R(t0), t1r = R(t1), t2r = R(t2), lm = R(lmasel), wi = R(0.25 * g5w(i));
      const R e0 = R(ee[0]), e1 = R(ee[1]), e2 = R(ee[2]), e3 = R(ee[3]);
      R m0 = 0, m1 = 0, m2 = 0, Ls[4] = {0, 0, 0, 0};
#pragma unroll
      for (int j = 0; j < 5; j++) {
        const double sd = (g5p(j) + ofs) / 2.0;
        const R s = R(sd), ds = R(sd - G.sc);
        const R tau = t0r + ds * (t1r + t2r * ds);
        const R det = e0 + s * (e1 + s * (e2 + s * e3));
        const R itau = R(1) / tau;
        const R ldet = lm * (wi * R(g5w(j))) * itau;
        const R ltau = -ldet * det * itau;
        m0 += ltau;
        m1 += ltau * ds;
        m2 += ltau * ds * ds;
        Ls[0] += ldet;
        Ls[1] += ldet * s;
        Ls[2] += ldet * s * s;
        Ls[3] += ldet * s * s * s;
      }
      const double a0 = m0, a1 = m1, a2 = m2;
      lu0[0] += a0;
      lu0[1] += dr * a0;
      lu0[2] += a1;
      lu0[3] += (0.5 * dr * dr - G.g19) * a0;
      lu0[4] += 0.5 * a2 - G.g20 * a0;
      lu0[5] += dr * a1 - G.g21 * a0;
      double rp = 1.0;
#pragma unroll
      for (int mm = 0; mm < 4; mm++) {
#pragma unroll
        for (int n = 0; n < 4; n++) lD[4 * mm + n] += rp * double(Ls[n]);
        rp *= r;
      }
    }
  }
  double lc36[36];
  for (int p = 0; p < 36; p++) lc36[p] = 0.0;
  detpoly_T(lD, lc36);
  subareas_T(lv4, lc36);
  double lxp[9][2];
  for (int k = 0; k < 9; k++) { lxp[k][0] = 0.0; lxp[k][1] = 0.0; }
  cross36_T(xp, lc36, lxp);
  for (int k = 0; k < 9; k++) {
    a.pbuf[(0 * 9 + k) * nq + iq] += lxp[k][0];
    a.pbuf[(1 * 9 + k) * nq + iq] += lxp[k][1];
  }
#pragma unroll
  for (int k = 0; k < 6; k++) a.lU[k * (size_t)d.ncell + e] += lu0[k];
}

// Reverse of the volume integral of the RHS pass (5x5 Gauss-Lobatto,
// cofactor form), row by row: the DOFs along a row are a_q + ds (b_q + c_q ds),
// and the transposed sums over a row collapse to per-row moments (sum l,
// sum l ds, sum l ds^2 for the DOF adjoints; sum l L_b(s), sum l L_b'(s) for
// the node adjoints).  R = double for the FP64 adjoint; R = float for the
// FP32-mixed one, where the point arithmetic and the per-row moments are FP32
// and the rows are added into the FP64 adjoints.
template <typename R>
__host__ __device__ __forceinline__ void vol_T(const Loaded &L, const CellGeo &G, const double u[4][6],
                                               const double lR[4][6], double g, double eps, double lu[4][6],
                                               double lX[3][3], double lY[3][3]) {
#pragma unroll 1
  for (int i = 0; i < 5; i++) {
    const double r = l5p(i), dr = r - G.rc;
    double lr[3], dlr[3];
    lag3(r, lr);
    dlag3(r, dlr);
    R Qx[3], Qy[3], Px[3], Py[3];
#pragma unroll
    for (int bb = 0; bb < 3; bb++) {
      Qx[bb] = R(dlr[0] * L.X[0][bb] + dlr[1] * L.X[1][bb] + dlr[2] * L.X[2][bb]);
      Qy[bb] = R(dlr[0] * L.Y[0][bb] + dlr[1] * L.Y[1][bb] + dlr[2] * L.Y[2][bb]);
      Px[bb] = R(lr[0] * L.X[0][bb] + lr[1] * L.X[1][bb] + lr[2] * L.X[2][bb]);
      Py[bb] = R(lr[0] * L.Y[0][bb] + lr[1] * L.Y[1][bb] + lr[2] * L.Y[2][bb]);
    }
    R ra[4], rb[4], rc2[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      ra[q] = R(u[q][0] + u[q][1] * dr + u[q][3] * (0.5 * dr * dr - G.g19) - u[q][4] * G.g20 - u[q][5] * G.g21);
      rb[q] = R(u[q][2] + u[q][5] * dr);
      rc2[q] = R(0.5 * u[q][4]);
    }
    R lR1[4][5];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int kk = 0; kk < 5; kk++) lR1[q][kk] = R(lR[q][kk + 1]);
    R m0[4] = {0, 0, 0, 0}, m1[4] = {0, 0, 0, 0}, m2[4] = {0, 0, 0, 0};
    R Mxr[3] = {0, 0, 0}, Mxs[3] = {0, 0, 0}, Myr[3] = {0, 0, 0}, Mys[3] = {0, 0, 0};
    const R wi = R(l5w(i)), drr = R(dr), gm1 = R(g - 1.0), epsr = R(eps), half = R(0.5), one = R(1);
#pragma unroll 1
    for (int j = 0; j < 5; j++) {
      const R ds = R(l5p(j) - G.sc);
      double lsd[3], dlsd[3];
      lag3(l5p(j), lsd);
      dlag3(l5p(j), dlsd);
      const R ls[3] = {R(lsd[0]), R(lsd[1]), R(lsd[2])}, dls[3] = {R(dlsd[0]), R(dlsd[1]), R(dlsd[2])};
      const R w = wi * R(l5w(j));
      const R xr = Qx[0] * ls[0] + Qx[1] * ls[1] + Qx[2] * ls[2];
      const R yr = Qy[0] * ls[0] + Qy[1] * ls[1] + Qy[2] * ls[2];
      const R xs = Px[0] * dls[0] + Px[1] * dls[1] + Px[2] * dls[2];
      const R ys = Py[0] * dls[0] + Py[1] * dls[1] + Py[2] * dls[2];
      R un[4];
#pragma unroll
      for (int q = 0; q < 4; q++) un[q] = ra[q] + ds * (rb[q] + rc2[q] * ds);
      const R rhoad = one / un[0];
      const R kin = un[3] - half * (un[1] * un[1] + un[2] * un[2]);
      const R pe = gm1 * rhoad * kin;
      const R pres = pe > epsr ? pe : epsr;
      R gd0[5], gd1[5];
      gd0[0] = ys;        gd1[0] = -xs;
      gd0[1] = -yr;       gd1[1] = xr;
      gd0[2] = ys * drr;  gd1[2] = -xs * drr;
      gd0[3] = -yr * ds;  gd1[3] = xr * ds;
      gd0[4] = ys * ds - yr * drr;
      gd1[4] = -xs * ds + xr * drr;
      const R wp = w * pres;
      R lgd0[5], lgd1[5], lwp = 0, lun1 = 0, lun2 = 0;
#pragma unroll
      for (int kk = 0; kk < 5; kk++) {
        const R fv = gd0[kk] * un[1] + gd1[kk] * un[2];
        const R lfv = -lR1[0][kk] * w + lR1[3][kk] * wp;
        lwp += lR1[3][kk] * fv + lR1[1][kk] * gd0[kk] + lR1[2][kk] * gd1[kk];
        lgd0[kk] = lR1[1][kk] * wp + lfv * un[1];
        lgd1[kk] = lR1[2][kk] * wp + lfv * un[2];
        lun1 += lfv * gd0[kk];
        lun2 += lfv * gd1[kk];
      }
      const R lpres = lwp * w;
      R lun0 = 0, lun3 = 0;
      if (pe > epsr) {
        const R lrhoad = lpres * gm1 * kin;
        lun3 += lpres * gm1 * rhoad;
        lun1 -= lpres * gm1 * rhoad * un[1];
        lun2 -= lpres * gm1 * rhoad * un[2];
        lun0 += -lrhoad * rhoad * rhoad;
      }
      const R lunq[4] = {lun0, lun1, lun2, lun3};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        m0[q] += lunq[q];
        m1[q] += lunq[q] * ds;
        m2[q] += lunq[q] * ds * ds;
      }
      const R lys = lgd0[0] + lgd0[2] * drr + lgd0[4] * ds;
      const R lyr = -lgd0[1] - lgd0[3] * ds - lgd0[4] * drr;
      const R lxs = -lgd1[0] - lgd1[2] * drr - lgd1[4] * ds;
      const R lxr = lgd1[1] + lgd1[3] * ds + lgd1[4] * drr;
#pragma unroll
      for (int b2 = 0; b2 < 3; b2++) {
        Mxr[b2] += lxr * ls[b2];
        Mxs[b2] += lxs * dls[b2];
        Myr[b2] += lyr * ls[b2];
        Mys[b2] += lys * dls[b2];
      }
    }
    // basis (1, dr, ds, dr^2/2 - g19, ds^2/2 - g20, dr ds - g21) along the row
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const double a0 = m0[q], a1 = m1[q], a2 = m2[q];
      lu[q][0] += a0;
      lu[q][1] += dr * a0;
      lu[q][2] += a1;
      lu[q][3] += (0.5 * dr * dr - G.g19) * a0;
      lu[q][4] += 0.5 * a2 - G.g20 * a0;
      lu[q][5] += dr * a1 - G.g21 * a0;
    }
#pragma unroll
    for (int aa = 0; aa < 3; aa++)
#pragma unroll
      for (int b2 = 0; b2 < 3; b2++) {
        lX[aa][b2] += dlr[aa] * double(Mxr[b2]) + lr[aa] * double(Mxs[b2]);
        lY[aa][b2] += dlr[aa] * double(Myr[b2]) + lr[aa] * double(Mys[b2]);
      }
  }
}

// Transpose of the Taylor-Green source moments (f_tgv_src) of one quad: from
// the energy rows lR3 of the RHS adjoint adds the node-coordinate adjoints
// into lX, lY (tensor nodes) and lxp (through the det J polynomial).  cos and
// sin of pi x at the Gauss points by angle addition from the centre node.
__host__ __device__ __forceinline__ void src_T(const Loaded &L, const CellGeo &G, const double lR3[6], double g,
                                               double lX[3][3], double lY[3][3], double lxp[9][2]) {
    double xp[9][2], c[36], D[16];
    node_xy_rel(L, xp);
    cross36_rel(xp, c);
    detpoly(c, D);
    const double PI = 3.14159265358979311599796346854;
    const double coef = 0.25 * PI / (g - 1.0);
    const double xc = L.X[1][1], yc = L.Y[1][1];
    const double cxc = cospi(xc), sxc = sinpi(xc), cyc = cospi(yc), syc = sinpi(yc);
    double lD[16];
    for (int t = 0; t < 16; t++) lD[t] = 0.0;
#pragma unroll 1
    for (int i = 0; i < 5; i++) {
      const double r = g5p(i), dr = r - G.rc;
      double lr[3];
      lag3(r, lr);
      double Px[3], Py[3];
#pragma unroll
      for (int bb = 0; bb < 3; bb++) {
        Px[bb] = lr[0] * (L.X[0][bb] - xc) + lr[1] * (L.X[1][bb] - xc) + lr[2] * (L.X[2][bb] - xc);
        Py[bb] = lr[0] * (L.Y[0][bb] - yc) + lr[1] * (L.Y[1][bb] - yc) + lr[2] * (L.Y[2][bb] - yc);
      }
      double ee[4];
#pragma unroll
      for (int n = 0; n < 4; n++) ee[n] = D[n] + r * (D[4 + n] + r * (D[8 + n] + r * D[12 + n]));
      // lsrc = sum_k lR3[k] b_k(s) = sa + ds (sb + sc ds) along the row
      const double sa = lR3[0] + lR3[1] * dr + lR3[3] * (0.5 * dr * dr - G.g19) - lR3[4] * G.g20 - lR3[5] * G.g21;
      const double sb = lR3[2] + lR3[5] * dr, sc = 0.5 * lR3[4];
      double Mx[3] = {0, 0, 0}, My[3] = {0, 0, 0}, Ls[4] = {0, 0, 0, 0};
      const double wi = g5w(i);
#pragma unroll 1
      for (int j = 0; j < 5; j++) {
        const double s = g5p(j), ds = s - G.sc;
        double ls[3];
        lag3(s, ls);
        const double dx = Px[0] * ls[0] + Px[1] * ls[1] + Px[2] * ls[2];
        const double dy = Py[0] * ls[0] + Py[1] * ls[1] + Py[2] * ls[2];
        const double wij = wi * g5w(j);
        const double djaco = wij * (ee[0] + s * (ee[1] + s * (ee[2] + s * ee[3])));
        double cx, sx, cy, sy;
        if (fabs(dx) <= 0.15 && fabs(dy) <= 0.15) {
          double cdx, sdx, cdy, sdy;
          cossin_pi_series<7>(dx, cdx, sdx);
          cossin_pi_series<7>(dy, cdy, sdy);
          cx = cxc * cdx - sxc * sdx;
          sx = sxc * cdx + cxc * sdx;
          cy = cyc * cdy - syc * sdy;
          sy = syc * cdy + cyc * sdy;
        } else {
          sincospi(xc + dx, &sx, &cx);
          sincospi(yc + dy, &sy, &cy);
        }
        const double c3x = cx * (4.0 * cx * cx - 3.0), c3y = cy * (4.0 * cy * cy - 3.0);
        const double lsrc = sa + ds * (sb + sc * ds);
        const double ldj = lsrc * coef * (c3x * cy - c3y * cx);
        const double lc3x = lsrc * coef * djaco * cy, lc3y = -lsrc * coef * djaco * cx;
        const double lcx = -lsrc * coef * djaco * c3y + lc3x * (12.0 * cx * cx - 3.0);
        const double lcy = lsrc * coef * djaco * c3x + lc3y * (12.0 * cy * cy - 3.0);
        const double lxg = -lcx * PI * sx, lyg = -lcy * PI * sy;
#pragma unroll
        for (int b2 = 0; b2 < 3; b2++) {
          Mx[b2] += lxg * ls[b2];
          My[b2] += lyg * ls[b2];
        }
        const double lw = ldj * wij;
        Ls[0] += lw;
        Ls[1] += lw * s;
        Ls[2] += lw * s * s;
        Ls[3] += lw * s * s * s;
      }
#pragma unroll
      for (int aa = 0; aa < 3; aa++)
#pragma unroll
        for (int b2 = 0; b2 < 3; b2++) {
          lX[aa][b2] += lr[aa] * Mx[b2];
          lY[aa][b2] += lr[aa] * My[b2];
        }
      double rp = 1.0;
#pragma unroll
      for (int mm = 0; mm < 4; mm++) {
#pragma unroll
        for (int n = 0; n < 4; n++) lD[4 * mm + n] += rp * Ls[n];
        rp *= r;
      }
    }
    double lc36[36];
    for (int p = 0; p < 36; p++) lc36[p] = 0.0;
    detpoly_T(lD, lc36);
    cross36_T(xp, lc36, lxp);
  }

// Reverse of the RHS pass of quad iq (the RHS written, no fused update):
// from lR adds into lU, writes pbuf (x, y, u*_prev = 0, v*_prev = 0, u*_new,
// v*_new) and the adjoints of the node partial sums the face integral reads
// (lP, consumed by a_corner).
template <typename R>
__host__ __device__ void a_rhs(const Dev &d, const Adj &a, int iq) {
  if (iq >= d.nquad) return;
  const int e = iq + d.ntria;
  const size_t nq = d.nquad, nc = d.ncell;
  const double eps = 1.0e-6, g = d.gamlg;
  Loaded L;
  load_cell(d, d.xs, d.ys, iq, L);
  const CellGeo G{d.rc[e], d.sc[e], d.g19[e], d.g20[e], d.g21[e]};
  double u[4][6];
  load_u(d, d.Us, e, u);
  double lR[4][6];
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) lR[q][k] = a.lR[(q * 6 + k) * nc + e];
  double lu[4][6];
  for (int q = 0; q < 4; q++) for (int k = 0; k < 6; k++) lu[q][k] = 0.0;
  double lX[3][3], lY[3][3];
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) { lX[i][j] = 0.0; lY[i][j] = 0.0; }
  // ---- face integral (f_rhs3): transpose of f = (P3, P4) + u* P0 - (P1, P2),
  // fe = u* . f, tw = u* . t per boundary node; the adjoints of the node
  // partial sums P0..P4 go to a.lP for the corner pass's transpose, those of
  // u* to pbuf, those of the mass-flux weights t to the face vectors
  for (int k = 0; k < 9; k++) {
    if (k == 8) {
      for (int v = 2; v < 6; v++) a.pbuf[(v * 9 + k) * nq + iq] = 0.0;
      for (int v = 0; v < 5; v++) a.lP[(v * 9 + k) * nq + iq] = 0.0;
      continue;
    }
    double b[6];
    node_basis2(G, k, b);
    const int pn = d.ipq[k * d.nquad + iq];
    const double un = d.us_new[pn], vn = d.vs_new[pn];
    double tx, ty;
    mass_flux_weights(L, k, tx, ty);
    const double P0 = d.npart[(0 * 9 + k) * nq + iq], P1 = d.npart[(1 * 9 + k) * nq + iq];
    const double P2 = d.npart[(2 * 9 + k) * nq + iq], P3 = d.npart[(3 * 9 + k) * nq + iq];
    const double P4 = d.npart[(4 * 9 + k) * nq + iq];
    const double f0 = P3 + (un * P0 - P1), f1 = P4 + (vn * P0 - P2);
    double ltw = 0, lf0 = 0, lf1 = 0, lfe = 0;
    for (int kk = 0; kk < 6; kk++) {
      ltw += lR[0][kk] * b[kk];
      lf0 += lR[1][kk] * b[kk];
      lf1 += lR[2][kk] * b[kk];
      lfe += lR[3][kk] * b[kk];
    }
    lf0 += lfe * un;
    lf1 += lfe * vn;
    const double lun = lfe * f0 + lf0 * P0 + ltw * tx;
    const double lvn = lfe * f1 + lf1 * P0 + ltw * ty;
    a.lP[(0 * 9 + k) * nq + iq] = lf0 * un + lf1 * vn;
    a.lP[(1 * 9 + k) * nq + iq] = -lf0;
    a.lP[(2 * 9 + k) * nq + iq] = -lf1;
    a.lP[(3 * 9 + k) * nq + iq] = lf0;
    a.lP[(4 * 9 + k) * nq + iq] = lf1;
    a.pbuf[(2 * 9 + k) * nq + iq] = 0.0;
    a.pbuf[(3 * 9 + k) * nq + iq] = 0.0;
    a.pbuf[(4 * 9 + k) * nq + iq] = lun;
    a.pbuf[(5 * 9 + k) * nq + iq] = lvn;
    // t = sum over the node's outer corner faces of 2 w_mass,f an_f
    const double ltx = ltw * un, lty = ltw * vn;
    for (int i = nc_start(k); i < nc_start(k + 1); i++) {
      const int isg = nc_entry(i) >> 2, ivsg = nc_entry(i) & 3;
      for (int f = 0; f < 2; f++)
        if (wmas(isg, ivsg, f) != 0.0)
          corner_an_T(isg, ivsg, f, ltx * (2.0 * wmas(isg, ivsg, f)), lty * (2.0 * wmas(isg, ivsg, f)), lX, lY);
    }
  }
  vol_T<R>(L, G, u, lR, g, eps, lu, lX, lY);
  // the DOF adjoints are complete: out before the source's transpose
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) a.lU[(q * 6 + k) * nc + e] += lu[q][k];
  // ---- Taylor-Green source
  double lxp[9][2];
  for (int k = 0; k < 9; k++) { lxp[k][0] = 0.0; lxp[k][1] = 0.0; }
  if (d.ncase == 1) {
    double lR3[6];
    for (int k = 0; k < 6; k++) lR3[k] = lR[3][k];
    src_T(L, G, lR3, g, lX, lY, lxp);
  }
  const int A[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
  const int B[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
  for (int k = 0; k < 9; k++) {
    a.pbuf[(0 * 9 + k) * nq + iq] = lxp[k][0] + lX[A[k]][B[k]];
    a.pbuf[(1 * 9 + k) * nq + iq] = lxp[k][1] + lY[A[k]][B[k]];
  }
}

// Gather of the per-(quad, node) contributions into the node adjoints:
// nv = 4 (x, y, u*_prev, v*_prev) after the corner pass, 6 after the RHS
// pass (also u*_new, v*_new); quads in cell order.
__host__ __device__ void a_gather(const Dev &d, const Adj &a, int p, int nv) {
  if (p >= d.npoin) return;
  double s[6] = {0, 0, 0, 0, 0, 0};
  const int b = d.node_ptr2[p], en = d.node_slot ? d.node_ptr2[p + 1] : b;
  for (int i = b; i < en; i++) {
    const int id = d.node_slot[i];
    if (id < 0) {  // triangle: -1 - (it*6 + k)
      const int t = -1 - id, it = t / 6, k = t - 6 * it;
      for (int v = 0; v < nv; v++) s[v] += a.tbuf[(v * 6 + k) * (size_t)d.ntria + it];
      continue;
    }
    const int iq = id / 9, k = id - 9 * iq;
    for (int v = 0; v < nv; v++) s[v] += a.pbuf[(v * 9 + k) * (size_t)d.nquad + iq];
  }
  a.lx[p] += s[0];
  a.ly[p] += s[1];
  a.lus[p] += s[2];
  a.lvs[p] += s[3];
  if (nv > 4) {
    a.luw[p] += s[4];
    a.lvw[p] += s[5];
  }
}

// Gather of the RHS pass's per-(cell, node) contributions (x, y, u*_prev,
// u*_new) fused with the reverse of the node solve u* = (S1 - S3) / S0,
// v* = (S2 - S4) / S0 (wall masks; kept nodes take u*_prev).  Only S0 is
// gathered again: u* itself is the forward pass's d.us_new / d.vs_new.
__host__ __device__ void a_gather_solve(const Dev &d, const Adj &a, int p) {
  if (p >= d.npoin) return;
  double s[6] = {0, 0, 0, 0, 0, 0}, S0 = 0.0;
  for (int i = d.node_ptr2[p]; i < d.node_ptr2[p + 1]; i++) {
    const int id = d.node_slot[i];
    if (id < 0) {  // triangle: -1 - (it*6 + k)
      const int t = -1 - id, it = t / 6, k = t - 6 * it;
#pragma unroll
      for (int v = 0; v < 6; v++) s[v] += a.tbuf[(v * 6 + k) * (size_t)d.ntria + it];
      S0 += d.tpart[k * (size_t)d.ntria + it];
      continue;
    }
    const int iq = id / 9, k = id - 9 * iq;
#pragma unroll
    for (int v = 0; v < 6; v++) s[v] += a.pbuf[(v * 9 + k) * (size_t)d.nquad + iq];
    S0 += d.npart[k * (size_t)d.nquad + iq];
  }
  a.lx[p] += s[0];
  a.ly[p] += s[1];
  double lus = a.lus[p] + s[2], lvs = a.lvs[p] + s[3];
  const double luw = a.luw[p] + s[4], lvw = a.lvw[p] + s[5];
  const unsigned char mask = d.bcmask[p];
  const double lu = (mask & 1) ? 0.0 : luw;
  const double lv = (mask & 2) ? 0.0 : lvw;
  const size_t np = d.npoin;
  if (mask & 4) {
    a.lus[p] = lus + lu;
    a.lvs[p] = lvs + lv;
#pragma unroll
    for (int v = 0; v < 5; v++) a.lS[v * np + p] = 0.0;
    return;
  }
  a.lus[p] = lus;
  a.lvs[p] = lvs;
  const double iS0 = 1.0 / S0;
  a.lS[0 * np + p] = -(lu * d.us_new[p] + lv * d.vs_new[p]) * iS0;
  a.lS[1 * np + p] = lu * iS0;
  a.lS[3 * np + p] = -lu * iS0;
  a.lS[2 * np + p] = lv * iS0;
  a.lS[4 * np + p] = -lv * iS0;
}

// fold (stage 1, the last one reversed): U^(1) is U^n itself, so the adjoint
// of U^n gathered from the later stages joins the adjoint of U^(1).
__host__ __device__ void a_update(const Dev &d, const Adj &a, int e, double alfa, double dt, int fold) {
  if (e >= d.ncell) return;
  const size_t nc = d.ncell;
  double am[16];
  for (int i = 0; i < 16; i++) am[i] = d.amatr[i * nc + e];
  const int IDX[5][5] = {{0, 1, 2, 3, 4}, {1, 5, 6, 7, 8}, {2, 6, 9, 10, 11}, {3, 7, 10, 12, 13}, {4, 8, 11, 13, 14}};
  const double oma = 1.0 - alfa;
  for (int q = 0; q < 4; q++) {
    double l[6];
    for (int k = 0; k < 6; k++) l[k] = a.lU[(q * 6 + k) * nc + e];
    for (int k = 0; k < 6; k++) {
      const double ln = a.lUn[(q * 6 + k) * nc + e] + alfa * l[k];
      if (fold) {
        a.lU[(q * 6 + k) * nc + e] = oma * l[k] + ln;
        a.lUn[(q * 6 + k) * nc + e] = 0.0;
      } else {
        a.lU[(q * 6 + k) * nc + e] = oma * l[k];
        a.lUn[(q * 6 + k) * nc + e] = ln;
      }
    }
    a.lR[(q * 6) * nc + e] = oma * dt * am[15] * l[0];
    for (int i = 0; i < 5; i++) {
      double acc = 0.0;
      for (int j = 0; j < 5; j++) acc += am[IDX[i][j]] * l[j + 1];
      a.lR[(q * 6 + i + 1) * nc + e] = oma * dt * acc;
    }
  }
}

// Reverse of the node motion x = alfa x^n + (1 - alfa)(x + dt u*_new), with
// u*_new becoming the next stage's u*_prev.  The adjoint of the stage's
// output coordinates is (tx, ty), after the centre-node transpose; fold as in
// a_update.
__host__ __device__ void a_nodes(const Dev &d, const Adj &a, int p, double alfa, double dt, int fold) {
  if (p >= d.npoin) return;
  const double oma = 1.0 - alfa;
  const double lxo = a.tx[p], lyo = a.ty[p];
  const double lxn = a.lxn[p] + alfa * lxo, lyn = a.lyn[p] + alfa * lyo;
  a.luw[p] = oma * dt * lxo + a.lus[p];
  a.lvw[p] = oma * dt * lyo + a.lvs[p];
  if (fold) {
    a.lx[p] = oma * lxo + lxn;
    a.ly[p] = oma * lyo + lyn;
    a.lxn[p] = 0.0;
    a.lyn[p] = 0.0;
  } else {
    a.lx[p] = oma * lxo;
    a.ly[p] = oma * lyo;
    a.lxn[p] = lxn;
    a.lyn[p] = lyn;
  }
  a.lus[p] = 0.0;
  a.lvs[p] = 0.0;
}

// Reverse of the centre-node re-interpolation x9 = -(x1+..+x4)/4 + (x5+..+x8)/2
// (per node: its own adjoint plus the contributions of the quads whose
// centre it feeds; a centre node's own coordinate is overwritten).
__host__ __device__ void a_centre(const Dev &d, const Adj &a, int p) {
  if (p >= d.npoin) return;
  double sx = a.lx[p], sy = a.ly[p];
  for (int i = d.node_ptr2[p]; i < d.node_ptr2[p + 1]; i++) {
    const int id = d.node_slot[i];
    if (id < 0) continue;
    const int iq = id / 9, k = id - 9 * iq;
    if (k == 8) { sx = 0.0; sy = 0.0; break; }
  }
  for (int i = d.node_ptr2[p]; i < d.node_ptr2[p + 1]; i++) {
    const int id = d.node_slot[i];
    if (id < 0) continue;
    const int iq = id / 9, k = id - 9 * iq;
    if (k == 8) continue;
    const int pc = d.ipq[8 * d.nquad + iq];
    const double cw = k < 4 ? -0.25 : 0.5;
    sx += cw * a.lx[pc];
    sy += cw * a.ly[pc];
  }
  a.tx[p] = sx;
  a.ty[p] = sy;
}

__global__ void __launch_bounds__(128) k_persson2(Dev d) { f_persson(d, blockIdx.x * blockDim.x + threadIdx.x); }
__global__ void __launch_bounds__(128, LAG2D_CCORR_MINB) k_corner2_corr(Dev d) {
  f_corner_corr(d, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void __launch_bounds__(kCornerBlock, LAG2D_CFACES_MINB) k_corner2_faces(Dev d) {
  extern __shared__ double faces_stage[];
  f_corner_faces(d, blockIdx.x * blockDim.x + threadIdx.x, faces_stage + threadIdx.x);
}
__global__ void __launch_bounds__(128) k_tgv_src2(Dev d) { f_tgv_src(d, blockIdx.x * blockDim.x + threadIdx.x); }
__global__ void k_node2(Dev d) { f_node(d, blockIdx.x * blockDim.x + threadIdx.x); }
__global__ void __launch_bounds__(kRhsBlock, LAG2D_RHS_MINB) k_rhs3(Dev d, int fuse, double alfa) {
  extern __shared__ double rhs_stage[];
  f_rhs3(d, blockIdx.x * blockDim.x + threadIdx.x, fuse, alfa, rhs_stage + threadIdx.x);
}
// per-block minima of getdelt_lag's two limits (consumed by k_dt_final)
__global__ void __launch_bounds__(256) k_dt2_partial(Dev d) {
  __shared__ double sm_cfl[256], sm_vol[256];
  double dtcfl, dtvol;
  f_dt_quad(d, blockIdx.x * blockDim.x + threadIdx.x, dtcfl, dtvol);
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
__global__ void k_nodes2(Dev d, double alfa) { f_nodes(d, blockIdx.x * blockDim.x + threadIdx.x, alfa); }
__global__ void k_geom2(Dev d, int fix) { f_geom(d, blockIdx.x * blockDim.x + threadIdx.x, fix); }
__global__ void k_init_wmom(Dev d) { f_init_wmom(d, blockIdx.x * blockDim.x + threadIdx.x); }

// resident blocks of 128 per SM the reverse corner and RHS kernels are
// compiled for: 3 (168 registers) in the FP32-mixed adjoint (reverse sweep
// 15.65 -> 15.08 ms per step on the 1024x1024 Taylor-Green mesh), 1 (255)
// in the FP64 one (3 would cost 12%)
template <typename R>
constexpr int arev_minb() { return sizeof(R) == 4 ? LAG2D_AREVF_MINB : 1; }
__global__ void __launch_bounds__(128, LAG2D_ACF_MINB) k_a_corner_faces(Dev d, Adj a) {
  a_corner_faces(d, a, blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename R>
__global__ void __launch_bounds__(128, LAG2D_ACC_MINB) k_a_corner_corr(Dev d, Adj a) {
  a_corner_corr<R>(d, a, blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename R>
__global__ void __launch_bounds__(128, arev_minb<R>()) k_a_rhs(Dev d, Adj a) { a_rhs<R>(d, a, blockIdx.x * blockDim.x + threadIdx.x); }
__global__ void k_a_gather(Dev d, Adj a, int nv) { a_gather(d, a, blockIdx.x * blockDim.x + threadIdx.x, nv); }
__global__ void k_a_gather_solve(Dev d, Adj a) { a_gather_solve(d, a, blockIdx.x * blockDim.x + threadIdx.x); }
__global__ void k_a_update(Dev d, Adj a, double alfa, const double *dtp, int fold) {
  a_update(d, a, blockIdx.x * blockDim.x + threadIdx.x, alfa, *dtp, fold);
}
__global__ void k_a_nodes(Dev d, Adj a, double alfa, const double *dtp, int fold) {
  a_nodes(d, a, blockIdx.x * blockDim.x + threadIdx.x, alfa, *dtp, fold);
}
__global__ void k_a_centre(Dev d, Adj a) { a_centre(d, a, blockIdx.x * blockDim.x + threadIdx.x); }

static inline int nb(int n, int b) { return (n + b - 1) / b; }

}  // namespace fast

void launch_tri_adjoint_rhs(const Dev &d, const Adj &a, cudaStream_t st);
void launch_tri_adjoint_corner(const Dev &d, const Adj &a, cudaStream_t st);

// Reverse of one RK stage of the optimised step.  Triangles run their own
// reverse corner and RHS kernels next to the quads' ones.  d views
// the stage's inputs (U^(s) in d.Us, x^(s) in d.xs/ys, u*_prev in d.us/vs) and
// the forward corner and node outputs of that stage (d.npart, d.corr,
// d.us_new/vs_new); the transposes run in reverse order.  dtp is the device
// address of the step's time step size; fold = 1 for stage 1, which ends the
// step's reverse (U^(1) and x^(1) are U^n and x^n).  mixed = 1 selects the
// FP32-mixed adjoint: the volume-integral and sub-cell-mass transposes run in
// FP32 with per-row moments added into the FP64 adjoints; geometry, corner
// coefficients, the node solve, the update and node motion stay FP64.
// fold_u = 0 keeps the adjoint of U^n apart from that of the stage state in
// stage 1 too, so that the WENO transpose can act on the latter alone; the
// caller then folds them (the WENO gather does, with its fold flag).
void launch_adjoint_stage(const Dev &d, const void *adj, cudaStream_t st, double alfa, const double *dtp, int fold,
                          int fold_u, int mixed) {
  const Adj &a = *static_cast<const Adj *>(adj);
  const int bq = fast::nb(d.nquad, 128), bp = fast::nb(d.npoin, 256), bc = fast::nb(d.ncell, 256);
  fast::k_a_centre<<<bp, 256, 0, st>>>(d, a);
  fast::k_a_nodes<<<bp, 256, 0, st>>>(d, a, alfa, dtp, fold);
  fast::k_a_update<<<bc, 256, 0, st>>>(d, a, alfa, dtp, fold_u);
  if (mixed) fast::k_a_rhs<float><<<bq, 128, 0, st>>>(d, a);
  else fast::k_a_rhs<double><<<bq, 128, 0, st>>>(d, a);
  launch_tri_adjoint_rhs(d, a, st);
  fast::k_a_gather_solve<<<bp, 256, 0, st>>>(d, a);
  fast::k_a_corner_faces<<<bq, 128, 0, st>>>(d, a);
  if (mixed) fast::k_a_corner_corr<float><<<bq, 128, 0, st>>>(d, a);
  else fast::k_a_corner_corr<double><<<bq, 128, 0, st>>>(d, a);
  launch_tri_adjoint_corner(d, a, st);
  fast::k_a_gather<<<bp, 256, 0, st>>>(d, a, 4);
}
int adjoint_stage_launches(const Dev &d) { return d.ntria > 0 ? 10 : 8; }


void launch_fast_persson(const Dev &d, cudaStream_t st) { fast::k_persson2<<<fast::nb(d.nquad, 128), 128, 0, st>>>(d); }
void launch_fast_corner(const Dev &d, cudaStream_t st) {
  fast::k_corner2_corr<<<fast::nb(d.nquad, 128), 128, 0, st>>>(d);
  constexpr int smem = fast::kCornerStage * fast::kCornerBlock * sizeof(double);
  fast::k_corner2_faces<<<fast::nb(d.nquad, fast::kCornerBlock), fast::kCornerBlock, smem, st>>>(d);
}
void launch_fast_src(const Dev &d, cudaStream_t st) { fast::k_tgv_src2<<<fast::nb(d.nquad, 128), 128, 0, st>>>(d); }
void launch_fast_node(const Dev &d, cudaStream_t st) { fast::k_node2<<<fast::nb(d.npoin, 256), 256, 0, st>>>(d); }
void launch_fast_rhs(const Dev &d, cudaStream_t st, int fuse, double alfa) {
  constexpr int smem = fast::kRhsStage * fast::kRhsBlock * sizeof(double);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(fast::k_rhs3, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(fast::k_rhs3, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    attr = true;
  }
  fast::k_rhs3<<<fast::nb(d.nquad, fast::kRhsBlock), fast::kRhsBlock, smem, st>>>(d, fuse, alfa);
}
void launch_dt_final(const Dev &d, cudaStream_t st, int nblk, int ndt);  // lag2d_kernels.cu
void launch_fast_dt(const Dev &d, cudaStream_t st, int ndt) {
  const int nb = fast::nb(d.nquad, 256);
  fast::k_dt2_partial<<<nb, 256, 0, st>>>(d);
  launch_dt_final(d, st, nb, ndt);
}
void launch_fast_nodes(const Dev &d, cudaStream_t st, double alfa) {
  fast::k_nodes2<<<fast::nb(d.npoin, 256), 256, 0, st>>>(d, alfa);
}
void launch_fast_geom(const Dev &d, cudaStream_t st, int fix) { fast::k_geom2<<<fast::nb(d.nquad, 256), 256, 0, st>>>(d, fix); }
void launch_init_wmom(const Dev &d, cudaStream_t st) { fast::k_init_wmom<<<fast::nb(d.nquad, 128), 128, 0, st>>>(d); }

}  // namespace lag2d
