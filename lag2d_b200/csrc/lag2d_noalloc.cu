// getdelt_lag without allocation: lag2d_delt_noalloc (include/lag2d.h).
//
// Who needs this entry point.  Every other entry point works on a handle whose
// device buffers lag2d_create allocated.  Some callers cannot allocate device
// memory at the point where they need a time-step size: a host code that
// owns a fixed device arena and forbids the CUDA allocator after start-up, a
// step loop that must not synchronise the device (cudaMalloc and cudaFree may
// synchronise it), or a caller that keeps its own state in device memory in
// the reference's array layouts and has no handle at all.  This entry point
// takes the caller's device arrays and uses, for its only scratch (the
// per-block minima of the reduction), a fixed array in the library's own
// device memory.  It calls no cudaMalloc, cudaFree or other allocating
// routine; on success it allocates no host memory either.
//
// Scratch: g_delt_scratch, 2 doubles per block of kThreads quads, sized for
// LAG2D_DELT_NOALLOC_MAX_QUADS quads (256 KiB).  Larger meshes are rejected
// with LAG2D_EINVAL.  Nothing in it has to start at zero: the final kernel
// reads only the slots the first kernel of the same call has written.
//
// Set-up.  Every call looks up the scratch address on the current device with
// cudaGetSymbolAddress; the first call on each device (with that device
// current) also loads both kernels, which may make the CUDA runtime load the
// library's module onto the device.  Make one call on each device before any
// stream capture is begun.
//
// Concurrency.  There is one scratch array per device.  Two calls whose work
// may overlap on the same device (different streams, or different host
// threads, without an order between them) race on it and give wrong results:
// serialise them (one stream, or an event between them).
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "lag2d.h"

namespace lag2d {
int set_error(int code, const std::string &msg);  // lag2d_capi.cu
}

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = LAG2D_DELT_NOALLOC_MAX_QUADS / kThreads;
static_assert(LAG2D_DELT_NOALLOC_MAX_QUADS % kThreads == 0, "whole blocks");
constexpr int kMaxDevices = 64;

// per-block minima of one call: [2 * block] = CFL limit, [2 * block + 1] = volume limit
static __device__ __align__(256) double g_delt_scratch[2 * kMaxBlocks];

std::mutex g_setup_mu;
bool g_loaded[kMaxDevices];  // per device: kernels loaded by the first call on it

// Per-quad limits of getdelt_lag (Getrhslag.f90:20641-20700) on the
// reference's layouts; block minima go to part.  ipqua has nvqua entries per
// quad; ncurv selects the edge length as the reference does (0: straight
// edges between the 4 corners; >= 1: corner - mid-edge node - corner, nodes
// 1..8).  A node id outside 1..npoin is not read: the block reports NaN, and
// the final kernel turns it into dtfix = NaN.
__global__ void __launch_bounds__(kThreads)
k_delt_noalloc_blocks(int ntria, int nquad, int npoin, int nvqua, int ncurv, int ndegr, int nq, int ngeel, int ndens,
                      double gamlg, const int *__restrict__ ipqua, const double *__restrict__ unkno,
                      const double *__restrict__ geoel, const double *__restrict__ coord,
                      const double *__restrict__ dvdt, double *__restrict__ part) {
  __shared__ double s_cfl[kThreads], s_vol[kThreads];
  const int ie = blockIdx.x * kThreads + threadIdx.x;
  double dtcfl = 1e10, dtvol = 1e10;
  int bad = 0;
  if (ie < nquad) {
    const long long ielem = (long long)ie + ntria;
    const int *ipq = ipqua + (long long)nvqua * ie;
    const int nread = ncurv == 0 ? 4 : 8;   // nvqua >= nread is checked on the host
    double xp[8][2];
    for (int k = 0; k < 8; k++) {
      xp[k][0] = xp[k][1] = 0.0;
      if (k >= nread) continue;
      const int p = ipq[k] - 1;
      if (p < 0 || p >= npoin) {
        bad = 1;
      } else {
        xp[k][0] = coord[2ll * p];
        xp[k][1] = coord[2ll * p + 1];
      }
    }
    double dlen = 0.0;
    if (ncurv == 0) {
      // straight edges 1-2, 2-3, 3-4, 4-1 (Getrhslag.f90:20647-20651)
      for (int k = 0; k < 4; k++) {
        const double *a = xp[k], *b = xp[(k + 1) & 3];
        const double dl = sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]));
        if (k == 0 || dl < dlen) dlen = dl;
      }
    } else {
      // curved edges: corner - mid-edge node - corner (Getrhslag.f90:20652-20660)
      const int ed[4][3] = {{0, 4, 1}, {1, 5, 2}, {2, 6, 3}, {3, 7, 0}};
      for (int k = 0; k < 4; k++) {
        const double *a = xp[ed[k][0]], *b = xp[ed[k][1]], *c = xp[ed[k][2]];
        const double dl = sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1])) +
                          sqrt((b[0] - c[0]) * (b[0] - c[0]) + (b[1] - c[1]) * (b[1] - c[1]));
        if (k == 0 || dl < dlen) dlen = dl;
      }
    }
    const double *u = unkno + ielem * ndegr * nq;  // unkno(1, q, ielem) = u[(q-1)*ndegr]
    const double rhomc = ndens == 1 ? u[0] : 1.0 / u[0];
    const double uctr = u[ndegr], vctr = u[2 * ndegr], ectr = u[3 * ndegr];
    const double eps = 1.0e-6;
    const double rhoct = 1.0 / rhomc;
    const double pctr = fmax(eps, (gamlg - 1.0) * rhoct * (ectr - 0.5 * (uctr * uctr + vctr * vctr)));
    const double sdctr = sqrt(fmax(eps, gamlg * pctr / rhoct));
    dtcfl = dlen / sdctr;
    dtvol = geoel[ielem * ngeel + 2] / fabs(dvdt[ielem]);
  }
  const int any_bad = __syncthreads_or(bad);
  s_cfl[threadIdx.x] = dtcfl;
  s_vol[threadIdx.x] = dtvol;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s_cfl[threadIdx.x] = fmin(s_cfl[threadIdx.x], s_cfl[threadIdx.x + s]);
      s_vol[threadIdx.x] = fmin(s_vol[threadIdx.x], s_vol[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = any_bad ? nan("") : s_cfl[0];
    part[2 * blockIdx.x + 1] = s_vol[0];
  }
}

// Global minima and dtfix (Getrhslag.f90:20705-20709).
__global__ void __launch_bounds__(kThreads)
k_delt_noalloc_final(int nblk, int itime, double cfl, const double *__restrict__ part, double *dtfix) {
  __shared__ double s_cfl[kThreads], s_vol[kThreads];
  double a = 1e10, b = 1e10;
  int bad = 0;
  for (int i = threadIdx.x; i < nblk; i += kThreads) {
    const double pc = part[2 * i];
    if (isnan(pc)) bad = 1;
    a = fmin(a, pc);
    b = fmin(b, part[2 * i + 1]);
  }
  const int any_bad = __syncthreads_or(bad);
  s_cfl[threadIdx.x] = a;
  s_vol[threadIdx.x] = b;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s_cfl[threadIdx.x] = fmin(s_cfl[threadIdx.x], s_cfl[threadIdx.x + s]);
      s_vol[threadIdx.x] = fmin(s_vol[threadIdx.x], s_vol[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double dt;
    if (itime == 1) dt = fmin(cfl * s_cfl[0], 0.1 * s_vol[0]);
    else dt = fmin(fmin(cfl * s_cfl[0], 0.1 * s_vol[0]), 1.01 * (*dtfix));
    *dtfix = any_bad ? nan("") : dt;
  }
}

// Scratch address on the current device.  The address is looked up on every
// call (cudaGetSymbolAddress allocates nothing), so it stays valid if the
// caller resets the device and the module is loaded again; the first call per
// device also loads both kernels (cudaFuncGetAttributes).
int scratch_for_current_device(double **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return lag2d::set_error(LAG2D_ENODEV, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return lag2d::set_error(LAG2D_EUNSUP, "device ordinal beyond 63");
  void *p = nullptr;
  e = cudaGetSymbolAddress(&p, g_delt_scratch);
  if (e != cudaSuccess || !p)
    return lag2d::set_error(LAG2D_ECUDA, std::string("cudaGetSymbolAddress(g_delt_scratch): ") +
                                             cudaGetErrorString(e));
  {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_loaded[dev]) {
      cudaFuncAttributes fa;
      e = cudaFuncGetAttributes(&fa, k_delt_noalloc_blocks);
      if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_delt_noalloc_final);
      if (e != cudaSuccess)
        return lag2d::set_error(LAG2D_ECUDA, std::string("cudaFuncGetAttributes: ") + cudaGetErrorString(e));
      g_loaded[dev] = true;
    }
  }
  *out = static_cast<double *>(p);
  return LAG2D_OK;
}

}  // namespace

extern "C" int lag2d_delt_noalloc(int ntria, int nquad, int npoin, int nvqua, int ncurv, int ndegr, int nq,
                                  int ngeel, const int *ipqua, const double *unkno, const double *geoel,
                                  const double *coord, const double *dvdt, int itime, int ndens,
                                  double gamlg, double cfl, double *dtfix, void *stream) {
  if (ntria < 0 || nquad < 0 || npoin < 0) return lag2d::set_error(LAG2D_EINVAL, "negative mesh size");
  if (nquad > LAG2D_DELT_NOALLOC_MAX_QUADS)
    return lag2d::set_error(LAG2D_EINVAL, "lag2d_delt_noalloc: nquad = " + std::to_string(nquad) +
                                              " exceeds LAG2D_DELT_NOALLOC_MAX_QUADS = " +
                                              std::to_string(LAG2D_DELT_NOALLOC_MAX_QUADS));
  if (ncurv < 0) return lag2d::set_error(LAG2D_EINVAL, "lag2d_delt_noalloc: ncurv must be >= 0");
  if (ncurv == 0 && nvqua < 4)
    return lag2d::set_error(LAG2D_EINVAL, "lag2d_delt_noalloc: ncurv = 0 needs nvqua >= 4 (ipqua(nvqua,nquad))");
  if (ncurv >= 1 && nvqua < 8)
    return lag2d::set_error(LAG2D_EINVAL, "lag2d_delt_noalloc: ncurv >= 1 needs nvqua >= 8 (ipqua(nvqua,nquad))");
  if (ndegr < 1 || nq < 4 || ngeel < 3) return lag2d::set_error(LAG2D_EINVAL, "need ndegr >= 1, nq >= 4, ngeel >= 3");
  if (ndens < 1 || ndens > 3) return lag2d::set_error(LAG2D_EINVAL, "ndens must be 1, 2 or 3");
  if (!dtfix || (nquad > 0 && (!ipqua || !unkno || !geoel || !coord || !dvdt)))
    return lag2d::set_error(LAG2D_EINVAL, "null device pointer");
  double *part = nullptr;
  int r = scratch_for_current_device(&part);
  if (r) return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nblk = (nquad + kThreads - 1) / kThreads;
  if (nblk > 0)
    k_delt_noalloc_blocks<<<nblk, kThreads, 0, st>>>(ntria, nquad, npoin, nvqua, ncurv, ndegr, nq, ngeel, ndens,
                                                     gamlg, ipqua, unkno, geoel, coord, dvdt, part);
  k_delt_noalloc_final<<<1, kThreads, 0, st>>>(nblk, itime, cfl, part, dtfix);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lag2d::set_error(LAG2D_ECUDA, std::string("lag2d_delt_noalloc launch: ") + cudaGetErrorString(e));
  return LAG2D_OK;
}
