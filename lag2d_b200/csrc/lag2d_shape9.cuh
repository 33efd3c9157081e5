// Shapes of the 9-node quad (GetFE.f90:89-127), in the reference's literal
// forms, shared by the curved P2 kernels and the straight-quad P1 kernels
// (whose geometry routines use the 9-node image of the straight quad).
#pragma once

namespace lag2d {

__host__ __device__ __forceinline__ void shp9v(double r, double s, double *shp) {
  const double c10 = 1.0;
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

__host__ __device__ __forceinline__ void shp9d(double r, double s, double *dr, double *ds) {
  const double c10 = 1.0;
  dr[0] = 0.25 * (2.0 * r - c10) * s * (s - 1.0);
  dr[1] = 0.25 * (2.0 * r + c10) * s * (s - 1.0);
  dr[2] = 0.25 * (2.0 * r + c10) * s * (s + 1.0);
  dr[3] = 0.25 * (2.0 * r - c10) * s * (s + 1.0);
  dr[4] = -r * s * (s - c10);
  dr[5] = 0.5 * (2.0 * r + c10) * (c10 - s * s);
  dr[6] = -r * s * (s + c10);
  dr[7] = 0.5 * (2.0 * r - c10) * (1.0 - s * s);
  dr[8] = -2.0 * r * (1.0 - s * s);
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

struct Jac { double xr, xs, yr, ys; };

__host__ __device__ __forceinline__ Jac jac9(const double (*xp)[2], const double *dr, const double *ds) {
  Jac j = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int k = 0; k < 9; k++) {
    j.xr = j.xr + dr[k] * xp[k][0];
    j.xs = j.xs + ds[k] * xp[k][0];
    j.yr = j.yr + dr[k] * xp[k][1];
    j.ys = j.ys + ds[k] * xp[k][1];
  }
  return j;
}

__host__ __device__ __forceinline__ void map9(const double (*xp)[2], const double *shp, double &x, double &y) {
  double a = 0.0, b = 0.0;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    a = a + shp[k] * xp[k][0];
    b = b + shp[k] * xp[k][1];
  }
  x = a;
  y = b;
}

}  // namespace lag2d
