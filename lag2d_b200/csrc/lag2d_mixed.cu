// FP32-mixed corner and RHS passes of the curved-P2 Lagrangian DG stage.
//
// The same scheme as the FP64 passes of lag2d_fast.cu, with the precision
// split of the mixed form:
//   FP32  the bulk flux and quadrature arithmetic of the momentum and energy
//         equations: vertex states, impedances and corner coefficients, the
//         100-point harmonic tau mean of the sub-cell densities, pressure and
//         the momentum/energy terms of the 5x5 Gauss-Lobatto volume integral,
//         the source quadrature, all accumulated in FP32;
//   FP64  everything that decides mesh validity and conservation: node
//         positions (geometry works on FP64 offsets from the cell's centre
//         node), sub-cell face normals and Jacobians, the det J polynomial,
//         cell and sub-cell volumes, the sub-cell density correction, the node
//         partial sums and the nodal 2x2 solve (node pass of lag2d_fast.cu),
//         the corner forces F* = sigma.n A + m (u* - u_c), every cell-average
//         (moment 0) contribution, the whole specific-volume (tau) equation,
//         the mass-matrix solve and the RK combine.  The tau equation is the
//         discrete volume change: its face and volume terms cancel to
//         O(h^2) of each other, so FP32 there would be amplified by 1/h^2
//         (and would trip the Persson indicator, which reads tau).
// Both passes compute each corner's FP32 coefficients m, sigma.n A and the
// vertex state with the same inline code from the same inputs, and the
// corner forces are formed from them in FP64, so at every interior node the
// corner forces of the surrounding cells cancel to FP64 rounding: momentum
// and total energy are conserved to FP64 round-off, as in the FP64 step.
// Storage (DOFs, M^-1, geometry, nodes) stays FP64.
#include <cuda_pipeline.h>
#include <cuda_runtime.h>
#include <math.h>

#include "lag2d_device.cuh"
#include "lag2d_fast_tables.h"

#ifndef LAG2D_MXF_MINB
#define LAG2D_MXF_MINB 3
#endif
// the mixed RHS kernel at 2 resident blocks per SM: 255 registers, 60 bytes
// of spill loads (500 at 3 blocks); 1.22 against 1.38 ms per 1024 x 1024 step
#ifndef LAG2D_RHSMX_MINB
#define LAG2D_RHSMX_MINB 2
#endif

namespace lag2d {

namespace mixed {

#include "lag2d_tables.inc"

struct MixTables {
  int nc_start[10];
  int nc_entry[16];
  int fnqsg[32];
  float wrie[32];
  float wmas[32];
  float wmom[16];
  int pa[12], pb[12], side[12];
  float dl[9];
  float xv[9], yv[9];
};
// compile-time tables (lookups fold to constants once the loops are unrolled)
__device__ __forceinline__ const MixTables &MT() {
  static constexpr MixTables t = LAG2D_FAST_TABLES;
  return t;
}

__device__ __forceinline__ void lag3f(float r, float *l) {
  l[0] = 0.5f * r * (r - 1.0f);
  l[1] = 1.0f - r * r;
  l[2] = 0.5f * r * (r + 1.0f);
}
__device__ __forceinline__ void dlag3f(float r, float *l) {
  l[0] = r - 0.5f;
  l[1] = -2.0f * r;
  l[2] = r + 0.5f;
}

__device__ __forceinline__ float detevalf(const float *D, float r, float s) {
  float e[4];
#pragma unroll
  for (int n = 0; n < 4; n++) e[n] = D[n] + r * (D[4 + n] + r * (D[8 + n] + r * D[12 + n]));
  return e[0] + s * (e[1] + s * (e[2] + s * e[3]));
}

// integral of det J over the sub-square [r0, r0+1] x [s0, s0+1] (FP64)
__device__ __forceinline__ double det_integral(const double *D, double r0, double s0) {
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

// 5-point Gauss (ruqope, FP32) and Gauss-Lobatto (ruqope_lobatto, FP64) rules
__device__ __forceinline__ float g5p(int i) {
  const float p[5] = {-0.9061798459386640f, -0.5384693101056831f, 0.0f, 0.5384693101056831f, 0.9061798459386640f};
  return p[i];
}
__device__ __forceinline__ float g5w(int i) {
  const float w[5] = {0.2369268850561891f, 0.4786286704993665f, 0.5688888888888889f, 0.4786286704993665f,
                      0.2369268850561891f};
  return w[i];
}
__device__ __forceinline__ double l5pd(int i) {
  const double p[5] = {-1.0, -0.6546536707079771437983, 0.0, 0.6546536707079771437983, 1.0};
  return p[i];
}
__device__ __forceinline__ double l5wd(int i) {
  const double w[5] = {0.1, 0.544444444444444444444, 0.7111111111111111111111, 0.544444444444444444444, 0.1};
  return w[i];
}

struct GeoF {
  float rc, sc, g19, g20, g21;
};

__device__ __forceinline__ void node_basis(const GeoF &g, int iv, float *b) {
  b[0] = 1.0f;
  b[1] = MT().xv[iv] - g.rc;
  b[2] = MT().yv[iv] - g.sc;
  b[3] = __fmaf_rn(__fmul_rn(0.5f, b[1]), b[1], -g.g19);
  b[4] = __fmaf_rn(__fmul_rn(0.5f, b[2]), b[2], -g.g20);
  b[5] = __fmaf_rn(b[1], b[2], -g.g21);
}


// FP64 copies of the weights and node tables (same initialiser)
struct MixTablesD {
  int nc_start[10];
  int nc_entry[16];
  int fnqsg[32];
  double wrie[32];
  double wmas[32];
  double wmom[16];
  int pa[12], pb[12], side[12];
  double dl[9];
  double xv[9], yv[9];
};
__device__ __forceinline__ const MixTablesD &MD() {
  static constexpr MixTablesD t = LAG2D_FAST_TABLES;
  return t;
}

// Unnormalised face vector an of gesgq slot `slot` in FP64 (unit normal
// an / |an|, face length 2 |an|; getfnds_lagsms_simpsonhybrid and
// getfnds_lagsmsif_hybrid)
// a0 x0 + a1 x1 + a2 x2 with a fixed rounding sequence (see vertex_state)
__device__ __forceinline__ double dot3(double a0, double x0, double a1, double x1, double a2, double x2) {
  return __fma_rn(a2, x2, __fma_rn(a1, x1, __dmul_rn(a0, x0)));
}
__device__ __forceinline__ void slot_an(const double X[3][3], const double Y[3][3], int slot, double &ax,
                                        double &ay) {
  if (slot >= 8 && slot < 12) {
    // inner sub-cell face from edge node (5..8) towards the centre
    const int f = slot - 8;
    const double lm0 = 0.375, lm1 = 0.75, lm2 = -0.125, lp0 = -0.125, lp1 = 0.75, lp2 = 0.375;
    double ex, ey, vx, vy;
    if (f == 0) {
      ex = X[1][0]; ey = Y[1][0];
      vx = dot3(lm0, X[1][0], lm1, X[1][1], lm2, X[1][2]);
      vy = dot3(lm0, Y[1][0], lm1, Y[1][1], lm2, Y[1][2]);
    } else if (f == 1) {
      ex = X[2][1]; ey = Y[2][1];
      vx = dot3(lp0, X[0][1], lp1, X[1][1], lp2, X[2][1]);
      vy = dot3(lp0, Y[0][1], lp1, Y[1][1], lp2, Y[2][1]);
    } else if (f == 2) {
      ex = X[1][2]; ey = Y[1][2];
      vx = dot3(lp0, X[1][0], lp1, X[1][1], lp2, X[1][2]);
      vy = dot3(lp0, Y[1][0], lp1, Y[1][1], lp2, Y[1][2]);
    } else {
      ex = X[0][1]; ey = Y[0][1];
      vx = dot3(lm0, X[0][1], lm1, X[1][1], lm2, X[2][1]);
      vy = dot3(lm0, Y[0][1], lm1, Y[1][1], lm2, Y[2][1]);
    }
    ax = -dot3(-1.5, ey, -0.5, Y[1][1], 2.0, vy);
    ay = dot3(-1.5, ex, -0.5, X[1][1], 2.0, vx);
    return;
  }
  const int ig = slot < 8 ? slot : slot - 4;
  const int ia = MD().pa[ig], ib = MD().pb[ig];
  const double *da = MD().dl + 3 * ia, *db = MD().dl + 3 * ib;
  double xa0, xa1, xa2, ya0, ya1, ya2, xb0, xb1, xb2, yb0, yb1, yb2;
  if (ib == 0) { xa0 = X[0][0]; xa1 = X[1][0]; xa2 = X[2][0]; ya0 = Y[0][0]; ya1 = Y[1][0]; ya2 = Y[2][0]; }
  else if (ib == 1) { xa0 = X[0][1]; xa1 = X[1][1]; xa2 = X[2][1]; ya0 = Y[0][1]; ya1 = Y[1][1]; ya2 = Y[2][1]; }
  else { xa0 = X[0][2]; xa1 = X[1][2]; xa2 = X[2][2]; ya0 = Y[0][2]; ya1 = Y[1][2]; ya2 = Y[2][2]; }
  if (ia == 0) { xb0 = X[0][0]; xb1 = X[0][1]; xb2 = X[0][2]; yb0 = Y[0][0]; yb1 = Y[0][1]; yb2 = Y[0][2]; }
  else if (ia == 1) { xb0 = X[1][0]; xb1 = X[1][1]; xb2 = X[1][2]; yb0 = Y[1][0]; yb1 = Y[1][1]; yb2 = Y[1][2]; }
  else { xb0 = X[2][0]; xb1 = X[2][1]; xb2 = X[2][2]; yb0 = Y[2][0]; yb1 = Y[2][1]; yb2 = Y[2][2]; }
  const double xr = dot3(da[0], xa0, da[1], xa1, da[2], xa2);
  const double yr = dot3(da[0], ya0, da[1], ya1, da[2], ya2);
  const double xs = dot3(db[0], xb0, db[1], xb1, db[2], xb2);
  const double ys = dot3(db[0], yb0, db[1], yb1, db[2], yb2);
  switch (MD().side[ig]) {
    case 0: ax = yr; ay = -xr; break;
    case 1: ax = ys; ay = -xs; break;
    case 2: ax = -yr; ay = xr; break;
    default: ax = -ys; ay = xs; break;
  }
}

__device__ __forceinline__ void corner_an(const double X[3][3], const double Y[3][3], int isg, int ivsg, int f,
                                          double &ax, double &ay) {
  const int code = MD().fnqsg[8 * isg + 2 * ivsg + f];
  const int slot = (code >= 0 ? code : -code) - 1;
  slot_an(X, Y, slot, ax, ay);
  if (code < 0) { ax = -ax; ay = -ay; }
}

// m = mu * A * w of one corner face (getriecoef_matrixnew, Limiterlag.f90:1037)
// from the face vector an: m = 2 w (rho c |an| + cimpd rho slpdu |du . an|);
// the jump-direction branch needs |u* - u_c| >= 1e12 c
__device__ __forceinline__ float corner_m(float rhoct, float sdctr, float cimpd, float slpdu, float dux, float duy,
                                          float ax, float ay, float w) {
  const float nn = __fsqrt_rn(__fmaf_rn(ax, ax, __fmul_rn(ay, ay)));
  const float dn = __fmaf_rn(dux, ax, __fmul_rn(duy, ay));
  const float dun = fabsf(dn);
  const float j2 = __fmaf_rn(dux, dux, __fmul_rn(duy, duy));
  const float rs = __fmul_rn(rhoct, sdctr), cr = __fmul_rn(__fmul_rn(cimpd, rhoct), slpdu);
  const float w2 = __fmul_rn(2.0f, w);
  if (__fmul_rn(j2, 1.0e-24f) < __fmul_rn(sdctr, sdctr)) return __fmul_rn(w2, __fmaf_rn(rs, nn, __fmul_rn(cr, dun)));
  const float murie = __fmaf_rn(cr, __fdiv_rn(dun, nn), rs);
  return __fmul_rn(__fmul_rn(murie, w2), fabsf(__fmul_rn(dn, rsqrtf(j2))));
}

// node coordinates of quad iq as FP64 offsets from its centre node on the 3x3 tensor
struct CellXY {
  double ox, oy;
  double X[3][3], Y[3][3];
};

__device__ __forceinline__ void load_cell(const Dev &d, int iq, CellXY &L, double *c) {
  const int A[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
  const int B[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
  double xp[9][2];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const int p = d.ipq[k * d.nquad + iq];
    xp[k][0] = d.xs[p];
    xp[k][1] = d.ys[p];
  }
  L.ox = xp[8][0];
  L.oy = xp[8][1];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    xp[k][0] -= L.ox;
    xp[k][1] -= L.oy;
    L.X[A[k]][B[k]] = xp[k][0];
    L.Y[A[k]][B[k]] = xp[k][1];
  }
  if (c) cross36(xp, c);
}

// cell-centre sound speed and 1/tau (getriem_quadsubg2), FP32
__device__ __forceinline__ void centre_state(const float u[4][6], float g, float &rhoct, float &sdctr) {
  const float eps = 1.0e-6f;
  rhoct = __fdiv_rn(1.0f, u[0][0]);
  const float kc = __fmaf_rn(-0.5f, __fmaf_rn(u[1][0], u[1][0], __fmul_rn(u[2][0], u[2][0])), u[3][0]);
  const float pctr = fmaxf(eps, __fmul_rn(__fmul_rn(g - 1.0f, rhoct), kc));
  sdctr = __fsqrt_rn(fmaxf(eps, __fdiv_rn(__fmul_rn(g, pctr), rhoct)));
}

// vertex state of node k: (tau, u, v, e) from the first mdegr Taylor modes
// The quantities that both the corner pass and the RHS pass compute (vertex
// states, pressures, corner coefficients, face vectors) use explicitly rounded
// operations: the two kernels must produce them bit for bit alike, or the
// corner forces of the RHS no longer balance the node solve and total energy
// drifts (the compiler may otherwise fuse multiply-adds differently in each).
__device__ __forceinline__ void vertex_state(const float u[4][6], const float *b, int mdegr, float st[4]) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    float acc = 0.0f;
#pragma unroll
    for (int kk = 0; kk < 6; kk++)
      if (kk < mdegr) acc = __fmaf_rn(u[q][kk], b[kk], acc);
    st[q] = acc;
  }
}
__device__ __forceinline__ float kinetic_f(const float st[4]) {
  return __fmaf_rn(-0.5f, __fmaf_rn(st[1], st[1], __fmul_rn(st[2], st[2])), st[3]);
}

// FP32 coefficients of one corner face from its FP64 face vector: m and
// sigma.n A w = -p 2 w an (sx, sy)
__device__ __forceinline__ void corner_coeffs(double axd, double ayd, float w, float pv, float rhoct, float sdctr,
                                              float cimpd, float slpdu, float dux, float duy, float &m, float &sx,
                                              float &sy) {
  const float ax = (float)axd, ay = (float)ayd;
  m = corner_m(rhoct, sdctr, cimpd, slpdu, dux, duy, ax, ay, w);
  const float pw = __fmul_rn(__fmul_rn(-2.0f, pv), w);
  sx = __fmul_rn(pw, ax);
  sy = __fmul_rn(pw, ay);
}

// ---------------------------------------------------------------------------
// Taylor-Green energy source (rhsdomnsrcdg_lag_curvquad, Getrhslag.f90:4070-4251)
// in FP32, one thread per quad, for the RHS pass (it depends on the stage's
// nodes only); the cell-average moment is accumulated in FP64
// ---------------------------------------------------------------------------
__device__ void m_tgv_src(const Dev &d, int iq) {
  if (iq >= d.nquad || d.sc_dev->done) return;
  const int e = iq + d.ntria;
  CellXY L;
  double c[36], D[16];
  load_cell(d, iq, L, c);
  detpoly(c, D);
  float Df[16];
#pragma unroll
  for (int t = 0; t < 16; t++) Df[t] = (float)D[t];
  const GeoF G{(float)d.rc[e], (float)d.sc[e], (float)d.g19[e], (float)d.g20[e], (float)d.g21[e]};
  double el0 = 0.0;
  float el[6] = {0, 0, 0, 0, 0, 0};
  float Xf[3][3], Yf[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int bb = 0; bb < 3; bb++) {
      Xf[a][bb] = (float)L.X[a][bb];
      Yf[a][bb] = (float)L.Y[a][bb];
    }
  const float coef = (float)(0.25 * 3.14159265358979311599796346854 / (d.gamlg - 1.0));
  const float oxf = (float)L.ox, oyf = (float)L.oy;
#pragma unroll 1
  for (int i = 0; i < 5; i++) {
    const float r = g5p(i), dr = r - G.rc;
    float lr[3];
    lag3f(r, lr);
    float Px[3], Py[3];
#pragma unroll
    for (int bb = 0; bb < 3; bb++) {
      Px[bb] = lr[0] * Xf[0][bb] + lr[1] * Xf[1][bb] + lr[2] * Xf[2][bb];
      Py[bb] = lr[0] * Yf[0][bb] + lr[1] * Yf[1][bb] + lr[2] * Yf[2][bb];
    }
    const float wi = g5w(i);
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const float s = g5p(j), ds = s - G.sc;
      float ls[3];
      lag3f(s, ls);
      const float xg = oxf + (Px[0] * ls[0] + Px[1] * ls[1] + Px[2] * ls[2]);
      const float yg = oyf + (Py[0] * ls[0] + Py[1] * ls[1] + Py[2] * ls[2]);
      const float djaco = wi * g5w(j) * detevalf(Df, r, s);
      const float cx = cospif(xg), cy = cospif(yg);
      const float c3x = cx * (4.0f * cx * cx - 3.0f), c3y = cy * (4.0f * cy * cy - 3.0f);
      const float src = coef * (c3x * cy - c3y * cx) * djaco;
      el0 += (double)src;
      el[1] += src * dr;
      el[2] += src * ds;
      el[3] += src * (0.5f * dr * dr - G.g19);
      el[4] += src * (0.5f * ds * ds - G.g20);
      el[5] += src * (dr * ds - G.g21);
    }
  }
  d.src[(size_t)iq] = el0;
#pragma unroll
  for (int k = 1; k < 6; k++) d.src[k * (size_t)d.nquad + iq] = (double)el[k];
}

// ---------------------------------------------------------------------------
// Corner pass (getriem_quadsubg2 with getrhosubg_averg/_daverg)
// ---------------------------------------------------------------------------
// The corner pass runs as two kernels, as in the FP64 form: the sub-cell
// density corrections (m_corner_corr, written to d.corr in FP64), then the
// corner faces (m_corner_faces) with the corrections read back.
__device__ void m_corner_corr(const Dev &d, int iq) {
  if (iq >= d.nquad || d.sc_dev->done) return;
  const int e = iq + d.ntria;
  CellXY L;
  double c[36], D[16];
  load_cell(d, iq, L, c);
  detpoly(c, D);
  float Df[16];
#pragma unroll
  for (int t = 0; t < 16; t++) Df[t] = (float)D[t];
  const GeoF G{(float)d.rc[e], (float)d.sc[e], (float)d.g19[e], (float)d.g20[e], (float)d.g21[e]};
  float u0[6];
#pragma unroll
  for (int k = 0; k < 6; k++) u0[k] = (float)d.Us[k * (size_t)d.ncell + e];
  // sub-cell densities: initial mass / exact sub-cell area (FP64) against the
  // DG-implied harmonic tau mean (FP32 5x5 Gauss per sub-cell).  Sub-cells 0
  // and 3 (r in [-1, 0]) share their Gauss rows, and so do 1 and 2: each
  // row's det J and tau coefficients serve both.
  double vsub4[4];
  subareas(c, vsub4);
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const float ofr = h == 0 ? -1.0f : 1.0f;
    const int ilo = h == 0 ? 0 : 1, ihi = h == 0 ? 3 : 2;  // s in [-1, 0], [0, 1]
    float mlo = 0.0f, mhi = 0.0f;
#pragma unroll 1
    for (int i = 0; i < 5; i++) {
      const float r = (g5p(i) + ofr) * 0.5f;
      // along the row r, det J is a cubic and tau a quadratic in s
      float e[4];
#pragma unroll
      for (int n = 0; n < 4; n++) e[n] = Df[n] + r * (Df[4 + n] + r * (Df[8 + n] + r * Df[12 + n]));
      const float dr = r - G.rc;
      const float t0 = u0[0] + u0[1] * dr + u0[3] * (0.5f * dr * dr - G.g19) - u0[4] * G.g20 - u0[5] * G.g21;
      const float t1 = u0[2] + u0[5] * dr, t2 = 0.5f * u0[4];
      const float wi = 0.25f * g5w(i);
#pragma unroll
      for (int j = 0; j < 5; j++) {
        const float w = wi * g5w(j);
        {
          const float s = (g5p(j) - 1.0f) * 0.5f;
          const float ds = s - G.sc;
          const float tau = t0 + ds * (t1 + t2 * ds);
          const float det = e[0] + s * (e[1] + s * (e[2] + s * e[3]));
          mlo += w * __fdividef(det, tau);
        }
        {
          const float s = (g5p(j) + 1.0f) * 0.5f;
          const float ds = s - G.sc;
          const float tau = t0 + ds * (t1 + t2 * ds);
          const float det = e[0] + s * (e[1] + s * (e[2] + s * e[3]));
          mhi += w * __fdividef(det, tau);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const int isg = t == 0 ? ilo : ihi;
      const float masel = t == 0 ? mlo : mhi;
      const double unksgq = d.msub[isg * (size_t)d.nquad + iq] / vsub4[isg];
      const double volel = det_integral(D, (isg == 0 || isg == 3) ? -1.0 : 0.0, (isg == 0 || isg == 1) ? -1.0 : 0.0);
      d.corr[isg * (size_t)d.nquad + iq] = d.cdrho * (unksgq - (double)masel / volel);
    }
  }
}

__device__ void m_corner_faces(const Dev &d, int iq_in) {
  // every thread of the block reaches the barriers below: a thread past the
  // last quad works on the last quad and stores nothing
  if (d.nquad <= 0 || d.sc_dev->done) return;
  const bool live = iq_in < d.nquad;
  const int iq = live ? iq_in : d.nquad - 1;
  const int e = iq + d.ntria;
  const float eps = 1.0e-6f, g = (float)d.gamlg, slpdu = (g + 1.0f) / 2.0f, cimpd = (float)d.cimpd;
  CellXY L;
  load_cell(d, iq, L, nullptr);
  const GeoF G{(float)d.rc[e], (float)d.sc[e], (float)d.g19[e], (float)d.g20[e], (float)d.g21[e]};
  float u[4][6];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int k = 0; k < 6; k++) u[q][k] = (float)d.Us[(q * 6 + k) * (size_t)d.ncell + e];
  // the velocity DOFs in FP64 as well: the node sums sum m u_vertex take the
  // vertex velocities in FP64 (an FP32 vertex velocity's rounding, carried
  // into u* tangentially, is amplified by the long faces of stretched cells)
  double uvd[2][6];
#pragma unroll
  for (int q = 0; q < 2; q++)
#pragma unroll
    for (int k = 0; k < 6; k++) uvd[q][k] = d.Us[((q + 1) * 6 + k) * (size_t)d.ncell + e];
  const double rcd = d.rc[e], scd = d.sc[e], g19d = d.g19[e], g20d = d.g20[e], g21d = d.g21[e];
  float rhoct, sdctr;
  centre_state(u, g, rhoct, sdctr);
  float corr[4];
#pragma unroll
  for (int isg = 0; isg < 4; isg++) corr[isg] = (float)d.corr[isg * (size_t)d.nquad + iq];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    float b[6], st[4];
    node_basis(G, k, b);
    vertex_state(u, b, d.mdegr, st);
    const float rhovt = __fdiv_rn(1.0f, st[0]);
    const float ke = kinetic_f(st);
    const int pn = d.ipq[k * d.nquad + iq];
    const float dux = (float)d.us[pn] - st[1];
    const float duy = (float)d.vs[pn] - st[2];
    double st1d, st2d;
    {
      const double b1 = MD().xv[k] - rcd, b2 = MD().yv[k] - scd;
      const double bd[6] = {1.0, b1, b2, 0.5 * b1 * b1 - g19d, 0.5 * b2 * b2 - g20d, b1 * b2 - g21d};
      st1d = 0.0;
      st2d = 0.0;
#pragma unroll
      for (int kk = 0; kk < 6; kk++)
        if (kk < d.mdegr) {
          st1d += uvd[0][kk] * bd[kk];
          st2d += uvd[1][kk] * bd[kk];
        }
    }
    double P0 = 0.0, P1 = 0.0, P2 = 0.0, P3 = 0.0, P4 = 0.0;
#pragma unroll
    for (int i = MT().nc_start[k]; i < MT().nc_start[k + 1]; i++) {
      const int isg = MT().nc_entry[i] >> 2, ivsg = MT().nc_entry[i] & 3;
      const float ci = isg == 0 ? corr[0] : isg == 1 ? corr[1] : isg == 2 ? corr[2] : corr[3];
      const float pv = fmaxf(eps, __fmul_rn(__fmul_rn(g - 1.0f, __fadd_rn(rhovt, ci)), ke));
#pragma unroll
      for (int f = 0; f < 2; f++) {
        double ax, ay;
        corner_an(L.X, L.Y, isg, ivsg, f, ax, ay);
        float m, sx, sy;
        corner_coeffs(ax, ay, MT().wrie[8 * isg + 2 * ivsg + f], pv, rhoct, sdctr, cimpd, slpdu, dux, duy, m, sx, sy);
        P0 += (double)m;
        P1 += (double)m * st1d;
        P2 += (double)m * st2d;
        P3 += (double)sx;
        P4 += (double)sy;
      }
    }
    if (live) {
      d.npart[(0 * 9 + k) * (size_t)d.nquad + iq] = P0;
      d.npart[(1 * 9 + k) * (size_t)d.nquad + iq] = P1;
      d.npart[(2 * 9 + k) * (size_t)d.nquad + iq] = P2;
      d.npart[(3 * 9 + k) * (size_t)d.nquad + iq] = P3;
      d.npart[(4 * 9 + k) * (size_t)d.nquad + iq] = P4;
    }
    // keep the block's warps on the same stretch of the unrolled code
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// RHS pass: face integral from the corner pass's FP64 node partial sums, the
// tau equation in FP64, FP32 momentum/energy volume terms and source, FP64
// moment 0; the FP64 M^-1 solve and RK combine when fused
// ---------------------------------------------------------------------------
// Face integral (rhsifacedg_lagsubgq2, Getrhslaggauss.f90:8501-8748): at node
// k the corner forces sum to (P3, P4) + u* P0 - (P1, P2) with P0..P4 the
// FP64 partial sums of the FP32 corner coefficients that the corner pass
// wrote (the momentum weights are 1 on the 8 boundary nodes and 0 at the
// centre node), the energy term is u* . that sum and the mass term u* . sum_f
// 2 w_mass,f an_f over the outer corner faces; see f_rhs3 in lag2d_fast.cu.
// The cell's U^(s), M^-1 and U^n are staged in shared memory by cp.async at
// entry, as in the FP64 RHS kernel (thread column, stride kMxBlock).
constexpr int kMxBlock = 128;
constexpr int kMxStage = 64;
__device__ void m_rhs(const Dev &d, int iq, int fuse_update, double alfa, double *col) {
  if (iq >= d.nquad || d.sc_dev->done) return;
  const int e = iq + d.ntria;
  const float eps = 1.0e-6f, g = (float)d.gamlg;
  {
    const size_t nc = d.ncell;
    for (int v = 0; v < 24; v++) __pipeline_memcpy_async(col + v * kMxBlock, d.Us + v * nc + e, sizeof(double));
    if (fuse_update) {
      for (int i = 0; i < 16; i++)
        __pipeline_memcpy_async(col + (24 + i) * kMxBlock, d.amatr + i * nc + e, sizeof(double));
      for (int v = 0; v < 24; v++)
        __pipeline_memcpy_async(col + (40 + v) * kMxBlock, d.Un + v * nc + e, sizeof(double));
    }
    __pipeline_commit();
    // the node partial sums of the 8 boundary nodes (and the source moments)
    // towards L2 while the coordinates are gathered
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
#define MX_U(q, k) col[((q) * 6 + (k)) * kMxBlock]
  CellXY L;
  load_cell(d, iq, L, nullptr);
  const double rc = d.rc[e], sc = d.sc[e], g19 = d.g19[e], g20 = d.g20[e], g21 = d.g21[e];
  const GeoF G{(float)rc, (float)sc, (float)g19, (float)g20, (float)g21};
  const float g19f = G.g19, g20f = G.g20, g21f = G.g21;
  double tr[6] = {0, 0, 0, 0, 0, 0};          // tau equation, all moments
  double pa0 = 0.0, pb0 = 0.0, el0 = 0.0;     // cell averages of momentum and energy
  float p0[6] = {0, 0, 0, 0, 0, 0}, p1[6] = {0, 0, 0, 0, 0, 0}, el[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 8; k++) {
    float b[6];
    node_basis(G, k, b);
    const int pn = d.ipq[k * d.nquad + iq];
    const double un = d.us_new[pn], vn = d.vs_new[pn];
    double tx = 0.0, ty = 0.0;
#pragma unroll
    for (int i = MT().nc_start[k]; i < MT().nc_start[k + 1]; i++) {
      const int isg = MT().nc_entry[i] >> 2, ivsg = MT().nc_entry[i] & 3;
#pragma unroll
      for (int f = 0; f < 2; f++) {
        if (MD().wmas[8 * isg + 2 * ivsg + f] != 0.0) {
          double ax, ay;
          corner_an(L.X, L.Y, isg, ivsg, f, ax, ay);
          tx += ax * (2.0 * MD().wmas[8 * isg + 2 * ivsg + f]);
          ty += ay * (2.0 * MD().wmas[8 * isg + 2 * ivsg + f]);
        }
      }
    }
    const double tw = un * tx + vn * ty;
    const size_t nq = d.nquad;
    const double P0 = d.npart[(0 * 9 + k) * nq + iq], P1 = d.npart[(1 * 9 + k) * nq + iq];
    const double P2 = d.npart[(2 * 9 + k) * nq + iq], P3 = d.npart[(3 * 9 + k) * nq + iq];
    const double P4 = d.npart[(4 * 9 + k) * nq + iq];
    const double f0 = P3 + (un * P0 - P1);
    const double f1 = P4 + (vn * P0 - P2);
    const double fe = un * f0 + vn * f1;
    // tau: all moments in FP64 with the FP64 node basis
    {
      const double b1 = MD().xv[k] - rc, b2 = MD().yv[k] - sc;
      tr[0] += tw;
      tr[1] += tw * b1;
      tr[2] += tw * b2;
      tr[3] += tw * (0.5 * b1 * b1 - g19);
      tr[4] += tw * (0.5 * b2 * b2 - g20);
      tr[5] += tw * (b1 * b2 - g21);
    }
    pa0 += f0;
    pb0 += f1;
    el0 += fe;
    const float f0f = (float)f0, f1f = (float)f1, fef = (float)fe;
#pragma unroll
    for (int kk = 1; kk < 6; kk++) {
      p0[kk] += f0f * b[kk];
      p1[kk] += f1f * b[kk];
      el[kk] += fef * b[kk];
    }
  }
  __pipeline_wait_prior(0);
  float u[4][6];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int k = 0; k < 6; k++) u[q][k] = (float)MX_U(q, k);
  // volume integral, 5x5 Gauss-Lobatto, cofactor form, sum-factorised rows:
  // Jacobian and velocity in FP64 (tau equation), pressure work in FP32
#pragma unroll 1
  for (int i = 0; i < 5; i++) {
    const double r = l5pd(i);
    const double dr = r - rc;
    const double lr0 = 0.5 * r * (r - 1.0), lr1 = 1.0 - r * r, lr2 = 0.5 * r * (r + 1.0);
    const double dl0 = r - 0.5, dl1 = -2.0 * r, dl2 = r + 0.5;
    double Qx[3], Qy[3], Px[3], Py[3];
#pragma unroll
    for (int bb = 0; bb < 3; bb++) {
      Qx[bb] = dl0 * L.X[0][bb] + dl1 * L.X[1][bb] + dl2 * L.X[2][bb];
      Qy[bb] = dl0 * L.Y[0][bb] + dl1 * L.Y[1][bb] + dl2 * L.Y[2][bb];
      Px[bb] = lr0 * L.X[0][bb] + lr1 * L.X[1][bb] + lr2 * L.X[2][bb];
      Py[bb] = lr0 * L.Y[0][bb] + lr1 * L.Y[1][bb] + lr2 * L.Y[2][bb];
    }
    const float drf = (float)dr;
    // FP64 velocities along the row: a + ds (b + c ds)
    const double rau = MX_U(1, 0) + MX_U(1, 1) * dr + MX_U(1, 3) * (0.5 * dr * dr - g19) - MX_U(1, 4) * g20 -
                       MX_U(1, 5) * g21;
    const double rbu = MX_U(1, 2) + MX_U(1, 5) * dr, rcu = 0.5 * MX_U(1, 4);
    const double rav = MX_U(2, 0) + MX_U(2, 1) * dr + MX_U(2, 3) * (0.5 * dr * dr - g19) - MX_U(2, 4) * g20 -
                       MX_U(2, 5) * g21;
    const double rbv = MX_U(2, 2) + MX_U(2, 5) * dr, rcv = 0.5 * MX_U(2, 4);
    // FP32 tau and total energy along the row: a + ds (b + c ds)
    const float b3r = 0.5f * drf * drf - g19f;
    const float rat = u[0][0] + u[0][1] * drf + u[0][3] * b3r - u[0][4] * g20f - u[0][5] * g21f;
    const float rbt = u[0][2] + u[0][5] * drf, rct = 0.5f * u[0][4];
    const float rae = u[3][0] + u[3][1] * drf + u[3][3] * b3r - u[3][4] * g20f - u[3][5] * g21f;
    const float rbe = u[3][2] + u[3][5] * drf, rce = 0.5f * u[3][4];
    // G . grad_xi b for b = 2..6 with dbdr = (1, 0, dr, 0, ds), dbds = (0,
    // 1, 0, ds, dr): G0 = (ys, -yr, ys dr, -yr ds, ys ds - yr dr), G1 =
    // (-xs, xr, -xs dr, xr ds, -xs ds + xr dr), and the mass flux
    // G0 u + G1 v = (A, B, dr A, ds B, ds A + dr B).  dr is fixed along the
    // row, so each equation needs only 4 sums over the row: of A, B (or ys,
    // yr, xs, xr) weighted by w_j and by w_j ds; those of the tau equation
    // in FP64, the pressure work in FP32.
    double SA = 0, SB = 0, TA = 0, TB = 0;
    float X1 = 0, X2 = 0, X3 = 0, X4 = 0, Y1 = 0, Y2 = 0, Y3 = 0, Y4 = 0, E1 = 0, E2 = 0, E3 = 0, E4 = 0;
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const double s = l5pd(j);
      const double ds = s - sc;
      const double ls0 = 0.5 * s * (s - 1.0), ls1 = 1.0 - s * s, ls2 = 0.5 * s * (s + 1.0);
      const double dls0 = s - 0.5, dls1 = -2.0 * s, dls2 = s + 0.5;
      const double wj = l5wd(j);
      const double xr = Qx[0] * ls0 + Qx[1] * ls1 + Qx[2] * ls2;
      const double yr = Qy[0] * ls0 + Qy[1] * ls1 + Qy[2] * ls2;
      const double xs = Px[0] * dls0 + Px[1] * dls1 + Px[2] * dls2;
      const double ys = Py[0] * dls0 + Py[1] * dls1 + Py[2] * dls2;
      const double uq = rau + ds * (rbu + rcu * ds);
      const double vq = rav + ds * (rbv + rcv * ds);
      const double A = ys * uq - xs * vq, B = xr * vq - yr * uq;
      const double wd = wj * ds;
      SA += wj * A; SB += wj * B; TA += wd * A; TB += wd * B;
      // FP32 pressure work
      const float dsf = (float)ds;
      const float tq = rat + dsf * (rbt + rct * dsf);
      const float eq = rae + dsf * (rbe + rce * dsf);
      const float uqf = (float)uq, vqf = (float)vq;
      const float pres = fmaxf(eps, (g - 1.0f) * (1.0f / tq) * (eq - 0.5f * (uqf * uqf + vqf * vqf)));
      const float pw = (float)wj * pres, pwd = (float)wd * pres;
      const float ysf = (float)ys, yrf = (float)yr, xsf = (float)xs, xrf = (float)xr, Af = (float)A, Bf = (float)B;
      X1 += pw * ysf; X2 += pw * yrf; X3 += pwd * yrf; X4 += pwd * ysf;
      Y1 += pw * xsf; Y2 += pw * xrf; Y3 += pwd * xrf; Y4 += pwd * xsf;
      E1 += pw * Af; E2 += pw * Bf; E3 += pwd * Bf; E4 += pwd * Af;
    }
    const double wi = l5wd(i);
    tr[1] -= wi * SA;
    tr[2] -= wi * SB;
    tr[3] -= wi * (dr * SA);
    tr[4] -= wi * TB;
    tr[5] -= wi * (TA + dr * SB);
    const float wif = (float)wi;
    p0[1] += wif * X1;
    p0[2] -= wif * X2;
    p0[3] += wif * (drf * X1);
    p0[4] -= wif * X3;
    p0[5] += wif * (X4 - drf * X2);
    p1[1] -= wif * Y1;
    p1[2] += wif * Y2;
    p1[3] -= wif * (drf * Y1);
    p1[4] += wif * Y3;
    p1[5] += wif * (drf * Y2 - Y4);
    el[1] += wif * E1;
    el[2] += wif * E2;
    el[3] += wif * (drf * E1);
    el[4] += wif * E3;
    el[5] += wif * (E4 + drf * E2);
  }
  if (d.ncase == 1) {
    // Taylor-Green energy source (FP32), computed by k_tgv_src_mx before the corner pass
    el0 += d.src[(size_t)iq];
#pragma unroll
    for (int k = 1; k < 6; k++) el[k] += (float)d.src[k * (size_t)d.nquad + iq];
  }
  double R[4][6];
  R[1][0] = pa0;
  R[2][0] = pb0;
  R[3][0] = el0;
#pragma unroll
  for (int k = 0; k < 6; k++) R[0][k] = tr[k];
#pragma unroll
  for (int k = 1; k < 6; k++) {
    R[1][k] = (double)p0[k];
    R[2][k] = (double)p1[k];
    R[3][k] = (double)el[k];
  }
  if (!fuse_update) {
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int k = 0; k < 6; k++) d.rhs[(q * 6 + k) * (size_t)d.ncell + e] = R[q][k];
    return;
  }
  // fused stage update in FP64 (Getrhslag.f90:1789-1904)
  const double dt = d.sc_dev->dtfix;
#define MX_AM(i) col[(24 + (i)) * kMxBlock]
#define MX_UN(v) col[(40 + (v)) * kMxBlock]
  const double oma = 1.0 - alfa;
  const int IDX[5][5] = {{0, 1, 2, 3, 4}, {1, 5, 6, 7, 8}, {2, 6, 9, 10, 11}, {3, 7, 10, 12, 13}, {4, 8, 11, 13, 14}};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const size_t base = (size_t)(q * 6) * d.ncell + e;
    d.Us[base] = alfa * MX_UN(q * 6) + oma * (MX_U(q, 0) + MX_AM(15) * (dt * R[q][0]));
#pragma unroll
    for (int i = 0; i < 5; i++) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < 5; j++) acc += MX_AM(IDX[i][j]) * (dt * R[q][j + 1]);
      const size_t idx = base + (size_t)(i + 1) * d.ncell;
      d.Us[idx] = alfa * MX_UN(q * 6 + i + 1) + oma * (MX_U(q, i + 1) + acc);
    }
  }
#undef MX_U
#undef MX_AM
#undef MX_UN
}

__global__ void __launch_bounds__(128, 4) k_corner_mx_corr(Dev d) {
  m_corner_corr(d, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void __launch_bounds__(128, LAG2D_MXF_MINB) k_corner_mx_faces(Dev d) {
  m_corner_faces(d, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void __launch_bounds__(128) k_tgv_src_mx(Dev d) { m_tgv_src(d, blockIdx.x * blockDim.x + threadIdx.x); }
__global__ void __launch_bounds__(kMxBlock, LAG2D_RHSMX_MINB) k_rhs_mx(Dev d, int fuse, double alfa) {
  extern __shared__ double mx_stage[];
  m_rhs(d, blockIdx.x * blockDim.x + threadIdx.x, fuse, alfa, mx_stage + threadIdx.x);
}

static inline int nb(int n, int b) { return (n + b - 1) / b; }

}  // namespace mixed

void launch_mixed_corner(const Dev &d, cudaStream_t st) {
  mixed::k_corner_mx_corr<<<mixed::nb(d.nquad, 128), 128, 0, st>>>(d);
  mixed::k_corner_mx_faces<<<mixed::nb(d.nquad, 128), 128, 0, st>>>(d);
}
void launch_mixed_src(const Dev &d, cudaStream_t st) {
  mixed::k_tgv_src_mx<<<mixed::nb(d.nquad, 128), 128, 0, st>>>(d);
}
void launch_mixed_rhs(const Dev &d, cudaStream_t st, int fuse, double alfa) {
  constexpr int smem = mixed::kMxStage * mixed::kMxBlock * sizeof(double);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(mixed::k_rhs_mx, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(mixed::k_rhs_mx, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    attr = true;
  }
  mixed::k_rhs_mx<<<mixed::nb(d.nquad, mixed::kMxBlock), mixed::kMxBlock, smem, st>>>(d, fuse, alfa);
}

}  // namespace lag2d
