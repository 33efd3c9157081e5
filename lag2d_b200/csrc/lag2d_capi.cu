// Host side of the Lag2D C-ABI (include/lag2d.h): handle, device memory,
// connectivity set-up and the per-step launch sequence of getsolvdg_lag.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <type_traits>
#include <string>
#include <vector>

#include "lag2d.h"
#include "lag2d_device.cuh"
#include "lag2d_p1.h"

namespace lag2d {
void set_tables(const QuadTables &q, cudaStream_t st);
void launch_geom(const Dev &d, cudaStream_t st, const double *X, const double *Y);
void launch_center_geom(const Dev &d, cudaStream_t st);
void launch_reset_count(const Dev &d, cudaStream_t st);
void launch_persson(const Dev &d, cudaStream_t st);
void launch_flags_from_host(const Dev &d, cudaStream_t st, const int *flags);
void launch_weno(const Dev &d, cudaStream_t st);
void launch_weno_warp(const Dev &d, cudaStream_t st);
void launch_weno_commit(const Dev &d, cudaStream_t st);
void launch_corner(const Dev &d, cudaStream_t st);
void launch_node(const Dev &d, cudaStream_t st);
void launch_rhs(const Dev &d, cudaStream_t st);
int dt_blocks(const Dev &d);
void launch_dt(const Dev &d, cudaStream_t st, int ndt);
void launch_update(const Dev &d, cudaStream_t st, double alfa);
void launch_nodes(const Dev &d, cudaStream_t st, double alfa);
void launch_copyback(const Dev &d, cudaStream_t st);
void launch_step_begin(const Dev &d, cudaStream_t st, int itime);
void launch_step_end(const Dev &d, cudaStream_t st, int check);
void launch_init(const Dev &d, cudaStream_t st);
void launch_init_msub(const Dev &d, cudaStream_t st);
void launch_unkno_in(const Dev &d, cudaStream_t st, const double *aos, int both);
void launch_unkno_out(const Dev &d, cudaStream_t st, double *aos);
void launch_xy_in(int n, cudaStream_t st, const double *xy, double *x, double *y, double *x2, double *y2);
void launch_xy_out(int n, cudaStream_t st, double *xy, const double *x, const double *y);
void launch_fast_persson(const Dev &d, cudaStream_t st);
void launch_fast_corner(const Dev &d, cudaStream_t st);
void launch_fast_node(const Dev &d, cudaStream_t st);
void launch_fast_rhs(const Dev &d, cudaStream_t st, int fuse, double alfa);
void launch_fast_dt(const Dev &d, cudaStream_t st, int ndt);
void launch_mixed_corner(const Dev &d, cudaStream_t st);
void launch_fast_src(const Dev &d, cudaStream_t st);
void launch_mixed_src(const Dev &d, cudaStream_t st);
void launch_mixed_rhs(const Dev &d, cudaStream_t st, int fuse, double alfa);
void launch_fast_nodes(const Dev &d, cudaStream_t st, double alfa);
void launch_fast_geom(const Dev &d, cudaStream_t st, int fix);
void launch_init_wmom(const Dev &d, cudaStream_t st);
void launch_tri_init(const Dev &d, cudaStream_t st);
void launch_tri_geom(const Dev &d, cudaStream_t st, const double *X, const double *Y);
void launch_tri_corner(const Dev &d, cudaStream_t st);
void launch_tri_rhs(const Dev &d, cudaStream_t st, const double *usn, const double *vsn, int fuse, double alfa);
void launch_adjoint_stage(const Dev &d, const void *adj, cudaStream_t st, double alfa, const double *dtp, int fold,
                          int fold_u, int mixed);
void launch_weno_linear(const Dev &d, cudaStream_t st, int mode, const double *v, double *out, double *wbuf,
                        int *wslot, int cap, int *overflow);
void launch_weno_gather(const Dev &d, cudaStream_t st, double *lamU, double *lamUn, int fold, const double *wbuf,
                        const int *wslot, int cap, const int *inv_ptr, const int *inv_ent);
void launch_weno_swap(const Dev &d, cudaStream_t st);
int adjoint_stage_launches(const Dev &d);
int error_blocks(const Dev &d);
void launch_error(const Dev &d, cudaStream_t st, const double *X, const double *Y, double *part);
void launch_cell_output(const Dev &d, cudaStream_t st, const double *U, const double *X, const double *Y,
                        double *out);
}  // namespace lag2d

using namespace lag2d;

static thread_local std::string g_err;

static int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

namespace lag2d {
// error text for lag2d_last_error from entry points in other translation units
int set_error(int code, const std::string &msg) { return fail(code, msg); }
}  // namespace lag2d

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(LAG2D_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
  } while (0)

struct Family {
  double ms = 0.0;
  long long n = 0;
};

struct lag2d_handle {
  Dev d{};
  lag2d_config cfg{};
  cudaStream_t st = nullptr;
  std::vector<void *> allocs;
  int *flags_dev = nullptr;
  double *rho0_dev = nullptr;  // per-cell initial-density factors (lag2d_set_rho0)
  double *stage_u = nullptr;   // staging for unkno(ndegr,nq,ncell) in the caller's layout
  double *stage_x = nullptr;   // staging for coord(2,npoin)
  double *stage_v = nullptr;   // staging for ustar(2,npoin) (its own, so no copy waits for another)
  cudaGraphExec_t graph = nullptr;
  long long graph_launches = 0;
  long long launches = 0;
  bool timing = false;
  std::map<std::string, Family> fam;
  std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  p1::Solver *p1 = nullptr;    // the linear P1 path (npoly = 1) when set; Dev d is then unused
  double *errpart = nullptr;   // per-block partial sums of lag2d_error_norms
  double *cellout = nullptr;   // [9][ncell] values of lag2d_cell_output
  // inverse of the WENO stencil table: for quad j, the entries c*9 + s of the
  // quads c whose stencil position s is j, c ascending (the WENO transpose's
  // fixed summation order)
  int *sinv_ptr = nullptr, *sinv_ent = nullptr;
};

template <typename T>
static int dalloc(lag2d_handle *h, T **p, size_t n) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return fail(LAG2D_ECUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  cudaMemset(q, 0, std::max<size_t>(n, 1) * sizeof(T));
  h->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return LAG2D_OK;
}

// Quadrature literals of ruqope / ruqope_lobatto (dgflo2d.f90:2497-2783),
// points ordered as the reference's 2-D loops produce them.
namespace lag2d {
void fill_rule(int n, bool lobatto, double (*pos)[2], double *w) {
  double p[6], q[6];
  if (lobatto) {
    p[0] = -1.0; p[1] = -0.6546536707079771437983; p[2] = 0.0; p[3] = 0.6546536707079771437983; p[4] = 1.0;
    q[0] = 0.1; q[1] = 0.544444444444444444444; q[2] = 0.7111111111111111111111; q[3] = 0.544444444444444444444;
    q[4] = 0.1;
  } else if (n == 5) {
    p[2] = 0.0;
    p[3] = 0.5384693101056830910363144; p[1] = -0.5384693101056830910363144;
    p[4] = 0.9061798459386639927976269; p[0] = -0.9061798459386639927976269;
    q[2] = 0.5688888888888888888888889;
    q[3] = 0.4786286704993664680412915; q[1] = 0.4786286704993664680412915;
    q[4] = 0.2369268850561890875142640; q[0] = 0.2369268850561890875142640;
  } else {
    p[0] = 0.2386191860831969086305017; p[1] = -0.2386191860831969086305017;
    p[2] = 0.6612093864662645136613996; p[3] = -0.6612093864662645136613996;
    p[4] = -0.9324695142031520278123016; p[5] = 0.9324695142031520278123016;
    q[0] = 0.4679139345726910; q[1] = 0.4679139345726910;
    q[2] = 0.3607615730481386; q[3] = 0.3607615730481386;
    q[4] = 0.1713244923791704; q[5] = 0.1713244923791704;
  }
  int ig = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      w[ig] = q[i] * q[j];
      pos[ig][0] = p[i];
      pos[ig][1] = p[j];
      ig++;
    }
}

}  // namespace lag2d
static const int kIPQSG[4][4] = {{0, 4, 8, 7}, {4, 1, 5, 8}, {8, 5, 2, 6}, {7, 8, 6, 3}};

// 7-point triangle rule of rutope (dgflo2d.f90:2232-2254), the reference's literals
static void fill_tri_rule7(double (*pos)[2], double *w) {
  const double a = 0.333333333333333, b1 = 0.059715871789770, b2 = 0.470142064105115;
  const double c1 = 0.797426985353087, c2 = 0.101286507323456;
  const double p[7][2] = {{a, a}, {b1, b2}, {b2, b1}, {b2, b2}, {c1, c2}, {c2, c1}, {c2, c2}};
  for (int i = 0; i < 7; i++) { pos[i][0] = p[i][0]; pos[i][1] = p[i][1]; }
  w[0] = 0.225000000000000;
  w[1] = w[2] = w[3] = 0.132394152788506;
  w[4] = w[5] = w[6] = 0.125939180544827;
}

// WENO stencil of every quad from esqua and the cells-surrounding-point
// lists, ordered as weno_stncl_quad_orthol3 orders it (WENO.f90:7646-7704).
static void build_stencils(const lag2d_mesh *m, std::vector<int> &sten) {
  const int nquad = m->nquad, ntria = m->ntria;
  sten.assign(9 * (size_t)nquad, -1);
  for (int iq = 0; iq < nquad; iq++) {
    const int ielem = iq + ntria;  // 0-based
    int ielaj[9];
    ielaj[0] = ielem + 1;
    // the reference reads esqua at the global cell id here (WENO.f90:7648);
    // on a mesh with triangles that id leaves the quad range and the quad's
    // own row is read instead
    const int row = ntria > 0 ? iq : ielem;
    const bool inrange = row < nquad;
    for (int k = 0; k < 4; k++) ielaj[1 + k] = inrange ? m->esqua[4 * (size_t)row + k] : 0;
    for (int k = 5; k < 9; k++) ielaj[k] = 0;
    bool bad = false;
    for (int iv = 0; iv < 4 && !bad; iv++) {
      const int ip = m->ipqua[9 * (size_t)iq + iv];
      int jelaj[5] = {0, 0, 0, 0, 0}, nvaj = 0;
      for (int s = m->esuv2[ip - 1]; s < m->esuv2[ip]; s++) {
        int je = m->esuv1[s];
        if (je != ielem + 1) {
          if (nvaj < 5) jelaj[nvaj] = je;
          nvaj++;
        }
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
          else bad = true;
        }
    }
    // the reference stops on this valence (WENO.f90:7699); on a mesh with
    // triangles it is the normal case next to them and the quad is skipped
    if (bad) { sten[iq] = ntria > 0 ? -1 : -2; continue; }
    bool complete = true;
    for (int k = 0; k < 9; k++) complete &= ielaj[k] != 0;
    // a stencil reaching a triangle is not a 3x3 quad block: left unlimited
    for (int k = 0; k < 9; k++) complete &= ielaj[k] > ntria;
    if (!complete) continue;
    for (int k = 0; k < 9; k++) sten[k * (size_t)nquad + iq] = ielaj[k] - 1;
  }
}

static double now_ms_event(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// Launch helper: counts launches and, when timing is on, brackets the
// launch with events on the handle's stream.
template <typename F>
static void run(lag2d_handle *h, const char *family, F &&f, int nlaunch = 1) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (h->timing) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, h->st);
  }
  f();
  h->launches += nlaunch;
  if (h->timing) {
    cudaEventRecord(b, h->st);
    h->pending.push_back({family, {a, b}});
  }
}

static void flush_timing(lag2d_handle *h) {
  for (auto &p : h->pending) {
    cudaEventSynchronize(p.second.second);
    Family &f = h->fam[p.first];
    f.ms += now_ms_event(p.second.first, p.second.second);
    f.n += 1;
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  h->pending.clear();
}

static const double kRK[2][3] = {{0.0, 0.5, 0.0}, {0.0, 0.75, 0.3333333333333333}};

// getrhsdg_lag_mcnew, curved P2 branch (Getrhslagmc.f90:7556-7710),
// reference-order kernels
static void enqueue_rhs(lag2d_handle *h) {
  const Dev &d = h->d;
  run(h, "persson", [&] { launch_reset_count(d, h->st); launch_persson(d, h->st); }, 2);
  run(h, "weno", [&] { launch_weno(d, h->st); launch_weno_commit(d, h->st); }, 2);
  const int T = d.ntria > 0;
  run(h, "corner", [&] { launch_tri_corner(d, h->st); launch_corner(d, h->st); }, 1 + T);
  run(h, "node", [&] { launch_node(d, h->st); });
  run(h, "rhs", [&] { launch_tri_rhs(d, h->st, d.us, d.vs, 0, 0.0); launch_rhs(d, h->st); }, 1 + T);
}

// volumes of all cells at the coordinates (X, Y): triangles, then quads
static void geom_all(lag2d_handle *h, const double *X, const double *Y) {
  launch_tri_geom(h->d, h->st, X, Y);
  launch_geom(h->d, h->st, X, Y);
}

// getsolvdg_lag (Getrhslag.f90:1553-2035) + the driver copy-back
static void enqueue_step_reference_order(lag2d_handle *h, int itime) {
  const Dev &d = h->d;
  const int nstag = h->cfg.nstag;
  const int T = d.ntria > 0;
  run(h, "geom", [&] { launch_step_begin(d, h->st, itime); geom_all(h, d.xn, d.yn); }, 2 + T);
  for (int istag = 1; istag <= nstag; istag++) {
    const double alfa = kRK[nstag - 2][istag - 1];
    enqueue_rhs(h);
    if (istag == 1) run(h, "dt", [&] { launch_dt(d, h->st, h->cfg.ndt); }, 2);
    run(h, "update", [&] { launch_update(d, h->st, alfa); });
    run(h, "nodes", [&] { launch_nodes(d, h->st, alfa); });
    run(h, "geom", [&] { launch_center_geom(d, h->st); geom_all(h, d.xs, d.ys); }, 2 + T);
  }
  run(h, "copy", [&] { launch_copyback(d, h->st); launch_step_end(d, h->st, 1); }, 2);
}

// Corner and RHS passes of the optimised step: FP64, or the FP32-mixed form
// (config precision = 1) with the same node pass, update and geometry.
// Triangles run their FP64 kernels in both forms.
// launches of corner_pass: the triangles' kernel, then two quad kernels
// (sub-cell corrections, corner faces)
static int corner_launches(const lag2d_handle *h, const Dev &d) {
  (void)h;
  return (d.ntria > 0) + 2;
}

// Taylor-Green energy source of the stage (quads; ncase 1 only), read by the
// RHS pass
static int src_launches(const Dev &d) { return d.ncase == 1 && d.nquad > 0; }
static void src_pass(lag2d_handle *h, const Dev &d) {
  if (!src_launches(d)) return;
  if (h->cfg.precision == 1) launch_mixed_src(d, h->st);
  else launch_fast_src(d, h->st);
}

static void corner_pass(lag2d_handle *h, const Dev &d) {
  launch_tri_corner(d, h->st);
  if (h->cfg.precision == 1) launch_mixed_corner(d, h->st);
  else launch_fast_corner(d, h->st);
}
// launches of rhs_pass: the triangles' kernel, then one quad kernel
static int rhs_launches(const lag2d_handle *h, const Dev &d) {
  (void)h;
  return (d.ntria > 0) + 1;
}

static void rhs_pass(lag2d_handle *h, const Dev &d, int fuse, double alfa) {
  launch_tri_rhs(d, h->st, d.us_new, d.vs_new, fuse, alfa);
  if (h->cfg.precision == 1) launch_mixed_rhs(d, h->st, fuse, alfa);
  else launch_fast_rhs(d, h->st, fuse, alfa);
}

// Stage recorder of the adjoint's recompute pass.  Before each stage the
// stage state (U^(s), x^(s), u*_prev) is copied into slot (step, stage); the
// stage's corner and node outputs (node partial sums, sub-cell density
// corrections, u*_new) are written straight into the slot instead of the
// handle's buffers; the step's time step size is kept after stage 1, and the
// number of cells WENO replaced in each stage is accumulated (the adjoint
// needs it to stay zero).
struct StageRec {
  double *U, *x, *y, *us, *vs, *dt;
  double *npart, *corr, *usn, *vsn, *tcf, *tpart;
  int step, nstag;
  size_t nu, np, nq, nt;
  // the handle's device view with the corner/node outputs of a slot
  Dev outputs(const Dev &d0, size_t slot) const {
    Dev d = d0;
    d.npart = npart + slot * 45 * nq;
    d.corr = corr + slot * 4 * nq;
    d.us_new = usn + slot * np;
    d.vs_new = vsn + slot * np;
    if (nt > 0) {
      d.tcf = tcf + slot * 120 * nt;
      d.tpart = tpart + slot * 30 * nt;
    }
    return d;
  }
  // ... and with the recorded stage inputs as well
  Dev inputs(const Dev &d0, size_t slot) const {
    Dev d = outputs(d0, slot);
    d.Us = U + slot * nu;
    d.xs = x + slot * np;
    d.ys = y + slot * np;
    d.us = us + slot * np;
    d.vs = vs + slot * np;
    return d;
  }
};
// The same step with the optimised kernels: node partial sums, recomputed
// corner data, closed-form volumes and the stage update fused into the RHS
// pass in stages 2 and 3.
static void enqueue_step_fast(lag2d_handle *h, int itime, const StageRec *rec = nullptr) {
  Dev d = h->d;
  const int nstag = h->cfg.nstag;
  const int T = d.ntria > 0;
  run(h, "begin", [&] { launch_step_begin(d, h->st, itime); });
  for (int istag = 1; istag <= nstag; istag++) {
    const double alfa = kRK[nstag - 2][istag - 1];
    if (rec) {
      const size_t slot = (size_t)rec->step * rec->nstag + (istag - 1);
      d = rec->outputs(h->d, slot);
      cudaMemcpyAsync(rec->U + slot * rec->nu, d.Us, rec->nu * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
      cudaMemcpyAsync(rec->x + slot * rec->np, d.xs, rec->np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
      cudaMemcpyAsync(rec->y + slot * rec->np, d.ys, rec->np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
      cudaMemcpyAsync(rec->us + slot * rec->np, d.us, rec->np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
      cudaMemcpyAsync(rec->vs + slot * rec->np, d.vs, rec->np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    }
    run(h, "persson", [&] { launch_reset_count(d, h->st); launch_fast_persson(d, h->st); }, 2);
    run(h, "weno", [&] { launch_weno_warp(d, h->st); launch_weno_commit(d, h->st); }, 2);
    if (src_launches(d)) run(h, "src", [&] { src_pass(h, d); });
    run(h, "corner", [&] { corner_pass(h, d); }, corner_launches(h, d));
    run(h, "node", [&] { launch_fast_node(d, h->st); });
    if (istag == 1) {
      // getdelt_lag needs only the cell-average mass flux of this stage's
      // RHS, which the node velocities give: dt first, then every stage's
      // RHS pass carries its own update
      run(h, "dt", [&] { launch_fast_dt(d, h->st, h->cfg.ndt); }, 2);
      if (rec)
        cudaMemcpyAsync(rec->dt + rec->step, &d.sc_dev->dtfix, sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    }
    run(h, "rhs", [&] { rhs_pass(h, d, 1, alfa); }, rhs_launches(h, d));
    run(h, "nodes", [&] { launch_fast_nodes(d, h->st, alfa); });
    run(h, "geom", [&] { launch_tri_geom(d, h->st, d.xs, d.ys); launch_fast_geom(d, h->st, 1); }, 1 + T);
  }
  run(h, "copy", [&] { launch_copyback(d, h->st); launch_step_end(d, h->st, 1); }, 2);
}

static void enqueue_step(lag2d_handle *h, int itime) {
  if (h->cfg.order_exact) enqueue_step_reference_order(h, itime);
  else enqueue_step_fast(h, itime);
}

static int read_status(lag2d_handle *h) {
  Scalars s;
  CK(cudaMemcpyAsync(&s, h->d.sc_dev, sizeof(Scalars), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  // a broken state outranks the stencil notice (which leaves the step complete)
  if (s.status & ST_NONPHYS) return fail(LAG2D_ENONPHYS, "non-positive cell volume");
  if (s.status & ST_STENCIL)
    return fail(LAG2D_ESTENCIL, "WENO: a troubled quad has a vertex valence the reference rejects");
  return LAG2D_OK;
}

// npoly = 1: the linear branch on straight 4-node quads (ipqua(4, nquad)),
// quads only, ndens = 1, the cases without a source term
static int create_p1(const lag2d_mesh *m, const lag2d_config *c, lag2d_handle **out) {
  if (m->ntria > 0) return fail(LAG2D_EUNSUP, "the P1 path is built for quads only (ntria = 0)");
  if (c->ndegr != 3 || c->nq != 4 || c->ndens != 1 || c->nlimi != 6)
    return fail(LAG2D_EUNSUP, "the P1 path needs ndegr=3, nq=4, ndens=1, nlimi=6");
  if (c->mdegr < 1 || c->mdegr > 3) return fail(LAG2D_EINVAL, "mdegr out of range");
  if (c->nstag != 2 && c->nstag != 3) return fail(LAG2D_EINVAL, "nstag must be 2 or 3");
  if (c->precision != 0) return fail(LAG2D_EUNSUP, "the P1 path is FP64 only (precision = 0)");
  if (c->nsedov < 0 || c->nsedov > 4) return fail(LAG2D_EINVAL, "nsedov must be 0..4");
  if (c->ncase != 3 && c->ncase != 6 && c->ncase != 7)
    return fail(LAG2D_EUNSUP, "the P1 path is built for the cases 3, 6 and 7");
  if (c->nrz < 0 || c->nrz > 2) return fail(LAG2D_EINVAL, "nrz must be 0, 1 or 2");
  if (c->nrz != 0 && c->ncase == 7)
    return fail(LAG2D_EUNSUP, "RZ Sedov runs a hard-coded dt schedule (Getrhslag.f90:1673-1693) that is not built");
  if (m->esuv2[0] != 0) return fail(LAG2D_EINVAL, "esuv2(1) must be 0");
  for (int p = 0; p < m->npoin; p++)
    if (m->esuv2[p + 1] < m->esuv2[p]) return fail(LAG2D_EINVAL, "esuv2 not monotone");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LAG2D_ENODEV, "no CUDA device");
  lag2d_handle *h = new lag2d_handle();
  h->cfg = *c;
  h->d.nquad = m->nquad; h->d.npoin = m->npoin; h->d.ncell = m->nquad; h->d.nbfac = m->nbfac;
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return fail(LAG2D_ECUDA, "cudaStreamCreate failed");
  }
  std::string err;
  int r = p1::create(m, c, h->st, &h->p1, err);
  if (r) {
    cudaStreamDestroy(h->st);
    delete h;
    return fail(r, err);
  }
  *out = h;
  return LAG2D_OK;
}

// forwards a P1 call, turning its message into the thread's last error
#define P1_CALL(expr)              \
  do {                             \
    std::string err_;              \
    int r_ = (expr);               \
    if (r_) return fail(r_, err_); \
    return LAG2D_OK;               \
  } while (0)

extern "C" {

const char *lag2d_last_error(void) { return g_err.c_str(); }

int lag2d_create(const lag2d_mesh *m, const lag2d_config *c, lag2d_handle **out) {
  if (!m || !c || !out) return fail(LAG2D_EINVAL, "null argument");
  (void)cudaGetLastError();  // an earlier call's launch error is not this handle's
  *out = nullptr;
  if (m->nquad <= 0 || m->npoin <= 0 || m->nbfac < 0 || m->ntria < 0)
    return fail(LAG2D_EINVAL, "mesh sizes must be positive");
  if (!m->ipqua || !m->bface || !m->esuv1 || !m->esuv2 || !m->esqua || !m->coold)
    return fail(LAG2D_EINVAL, "missing mesh array");
  if (m->ntria > 0 && !m->iptri) return fail(LAG2D_EINVAL, "missing iptri");
  if (c->npoly == 1) return create_p1(m, c, out);
  // the reference dispatches RZ on linear cells only (Getrhslagmc.f90:6876-6975)
  if (c->nrz != 0) return fail(LAG2D_EUNSUP, "RZ (nrz = 1, 2) is built for the linear P1 path only");
  if (m->ntria > 0 && (c->ngausd != 7 || c->ngausd_geo != 7))
    return fail(LAG2D_EUNSUP, "triangles need the 7-point rule (ngausd = ngausd_geo = 7)");
  if (c->npoly != 2 || c->ndegr != 6 || c->nq != 4 || c->ndens != 1)
    return fail(LAG2D_EUNSUP, "only P2 (npoly=2, ndegr=6, nq=4, ndens=1) is built");
  if (c->mdegr < 1 || c->mdegr > 6) return fail(LAG2D_EINVAL, "mdegr out of range");
  if (c->nstag != 2 && c->nstag != 3) return fail(LAG2D_EINVAL, "nstag must be 2 or 3");
  if (c->precision != 0 && c->precision != 1) return fail(LAG2D_EINVAL, "precision must be 0 (FP64) or 1 (FP32-mixed)");
  if (c->precision == 1 && c->order_exact) return fail(LAG2D_EINVAL, "order_exact needs precision = 0");
  if (c->nsedov < 0 || c->nsedov > 4) return fail(LAG2D_EINVAL, "nsedov must be 0..4");
  if (c->ncase != 1 && c->ncase != 2 && c->ncase != 3 && c->ncase != 6 && c->ncase != 7)
    return fail(LAG2D_EUNSUP, "initial-condition case not built");
  const int ncell = m->ntria + m->nquad;
  for (size_t i = 0; i < 9 * (size_t)m->nquad; i++)
    if (m->ipqua[i] < 1 || m->ipqua[i] > m->npoin) return fail(LAG2D_EINVAL, "ipqua node id out of range");
  for (size_t i = 0; i < 6 * (size_t)m->ntria; i++)
    if (m->iptri[i] < 1 || m->iptri[i] > m->npoin) return fail(LAG2D_EINVAL, "iptri node id out of range");
  for (size_t i = 0; i < (size_t)m->nbfac; i++) {
    const int *b = m->bface + 5 * i;
    if (b[0] < 1 || b[0] > m->npoin || b[1] < 1 || b[1] > m->npoin || b[4] < 1 || b[4] > m->npoin)
      return fail(LAG2D_EINVAL, "bface node id out of range");
  }
  if (m->esuv2[0] != 0) return fail(LAG2D_EINVAL, "esuv2(1) must be 0");
  for (int p = 0; p < m->npoin; p++)
    if (m->esuv2[p + 1] < m->esuv2[p]) return fail(LAG2D_EINVAL, "esuv2 not monotone");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LAG2D_ENODEV, "no CUDA device");

  lag2d_handle *h = new lag2d_handle();
  h->cfg = *c;
  Dev &d = h->d;
  d.ntria = m->ntria; d.nquad = m->nquad; d.npoin = m->npoin; d.nbfac = m->nbfac; d.ncell = ncell;
  d.ndegr = c->ndegr; d.mdegr = c->mdegr; d.ncase = c->ncase; d.nlimi = c->nlimi;
  d.gamlg = c->gamlg; d.cfl = c->cfl; d.cdrho = c->cdrho; d.cimpd = c->cimpd; d.tend = c->tend;
  d.sedov_energy = c->sedov_energy; d.nsedov = c->nsedov;
  for (int i = 0; i < 4; i++) d.sedov_cell[i] = c->sedov_cell[i];
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return fail(LAG2D_ECUDA, "cudaStreamCreate failed");
  }
  const int nq = m->nquad, np = m->npoin;
  // ---- connectivity
  std::vector<int> ipq(9 * (size_t)nq), esq(4 * (size_t)nq), sten;
  for (int iq = 0; iq < nq; iq++)
    for (int k = 0; k < 9; k++) ipq[k * (size_t)nq + iq] = m->ipqua[9 * (size_t)iq + k] - 1;
  for (int iq = 0; iq < nq; iq++)
    for (int k = 0; k < 4; k++) {
      int v = m->esqua[4 * (size_t)iq + k];
      esq[k * (size_t)nq + iq] = (v >= 1 && v <= ncell) ? v - 1 : -1;
    }
  build_stencils(m, sten);
  const int nt = m->ntria;
  std::vector<int> ipt(6 * (size_t)nt);
  for (int it = 0; it < nt; it++)
    for (int k = 0; k < 6; k++) ipt[k * (size_t)nt + it] = m->iptri[6 * (size_t)it + k] - 1;
  // node -> corner-face lists in the order getndvelo_lagsubg scatters them:
  // getriem_triasubg3 (triangles, entries -1 - (it*24 + slot)), then
  // getriem_quadsubg2 (quads, entries iq*32 + slot)
  static const int kIPTSG[4][3] = {{0, 3, 5}, {3, 4, 5}, {3, 1, 4}, {5, 4, 2}};
  std::vector<int> cnt(np + 1, 0), nodecf(24 * (size_t)nt + 32 * (size_t)nq);
  for (int it = 0; it < nt; it++)
    for (int isg = 0; isg < 4; isg++)
      for (int ivsg = 0; ivsg < 3; ivsg++) cnt[ipt[kIPTSG[isg][ivsg] * (size_t)nt + it] + 1] += 2;
  for (int iq = 0; iq < nq; iq++)
    for (int isg = 0; isg < 4; isg++)
      for (int ivsg = 0; ivsg < 4; ivsg++) cnt[ipq[kIPQSG[isg][ivsg] * (size_t)nq + iq] + 1] += 2;
  for (int p = 0; p < np; p++) cnt[p + 1] += cnt[p];
  std::vector<int> fillp(cnt.begin(), cnt.end() - 1);
  for (int it = 0; it < nt; it++)
    for (int isg = 0; isg < 4; isg++)
      for (int ivsg = 0; ivsg < 3; ivsg++) {
        int p = ipt[kIPTSG[isg][ivsg] * (size_t)nt + it];
        for (int f = 0; f < 2; f++) nodecf[fillp[p]++] = -1 - (it * 24 + (f + 2 * (ivsg + 3 * isg)));
      }
  for (int iq = 0; iq < nq; iq++)
    for (int isg = 0; isg < 4; isg++)
      for (int ivsg = 0; ivsg < 4; ivsg++) {
        int p = ipq[kIPQSG[isg][ivsg] * (size_t)nq + iq];
        for (int f = 0; f < 2; f++) nodecf[fillp[p]++] = iq * 32 + (f + 2 * (ivsg + 4 * isg));
      }
  // node -> (cell, local node) lists in cell order for the optimised gather:
  // triangles -1 - (it*6 + k), then quads iq*9 + k
  std::vector<int> cnt2(np + 1, 0), slots(6 * (size_t)nt + 9 * (size_t)nq);
  for (int it = 0; it < nt; it++)
    for (int k = 0; k < 6; k++) cnt2[ipt[k * (size_t)nt + it] + 1]++;
  for (int iq = 0; iq < nq; iq++)
    for (int k = 0; k < 9; k++) cnt2[ipq[k * (size_t)nq + iq] + 1]++;
  for (int p = 0; p < np; p++) cnt2[p + 1] += cnt2[p];
  {
    std::vector<int> fp(cnt2.begin(), cnt2.end() - 1);
    for (int it = 0; it < nt; it++)
      for (int k = 0; k < 6; k++) slots[fp[ipt[k * (size_t)nt + it]]++] = -1 - (it * 6 + k);
    for (int iq = 0; iq < nq; iq++)
      for (int k = 0; k < 9; k++) slots[fp[ipq[k * (size_t)nq + iq]]++] = iq * 9 + k;
  }
  // wall masks (getndvelo_lagsubg, Getrhslaggauss.f90:4420-4545)
  std::vector<unsigned char> mask(np, 0);
  for (int f = 0; f < m->nbfac; f++) {
    const int *b = m->bface + 5 * (size_t)f;
    const int nodes[3] = {b[0] - 1, b[1] - 1, b[4] - 1};
    for (int k = 0; k < 3; k++) {
      if (c->ncase == 2 || b[2] == 25) mask[nodes[k]] |= 4;
      if (b[2] == 22 && b[3] == 221) mask[nodes[k]] |= 2;
      if (b[2] == 22 && b[3] == 222) mask[nodes[k]] |= 1;
      if (b[2] == 25) mask[nodes[k]] |= 3;
    }
  }
  int rc = LAG2D_OK;
  auto A = [&](auto **p, size_t n) { if (rc == LAG2D_OK) rc = dalloc(h, p, n); };
  int *ipq_d, *esq_d, *sten_d, *ptr_d, *ncf_d;
  unsigned char *mask_d;
  double *x0, *y0;
  A(&ipq_d, ipq.size()); A(&esq_d, esq.size()); A(&sten_d, sten.size());
  A(&ptr_d, cnt.size()); A(&ncf_d, nodecf.size()); A(&mask_d, mask.size());
  A(&x0, np); A(&y0, np);
  A(&d.rc, ncell); A(&d.sc, ncell); A(&d.mass, ncell); A(&d.g19, ncell); A(&d.g20, ncell); A(&d.g21, ncell);
  A(&d.vol, ncell); A(&d.vcx, ncell); A(&d.vcy, ncell); A(&d.msub, 4 * (size_t)nq);
  A(&d.Un, NU * (size_t)ncell); A(&d.Us, NU * (size_t)ncell);
  A(&d.xn, np); A(&d.yn, np); A(&d.xs, np); A(&d.ys, np); A(&d.us, np); A(&d.vs, np);
  A(&d.amatr, 16 * (size_t)ncell); A(&d.rhs, NU * (size_t)ncell); A(&d.cf, 5 * 32 * (size_t)nq);
  A(&d.flag, ncell); A(&d.geoph, 2 * (size_t)ncell); A(&d.mapmt, 4 * (size_t)ncell);
  A(&d.Uw, 20 * (size_t)nq); A(&d.wlist, nq); A(&d.wcount, 1);
  A(&d.dtpart, 2 * (size_t)dt_blocks(d) + 2); A(&d.sc_dev, 1); A(&h->flags_dev, ncell);
  A(&h->stage_u, NU * (size_t)ncell); A(&h->stage_x, 2 * (size_t)np); A(&h->stage_v, 2 * (size_t)np);
  int *ptr2_d, *slot_d;
  A(&ptr2_d, cnt2.size()); A(&slot_d, slots.size());
  A(&d.npart, 45 * (size_t)nq); A(&d.corr, 4 * (size_t)nq); A(&d.src, 6 * (size_t)nq); A(&d.us_new, np); A(&d.vs_new, np);
  A(&d.wmom, 9 * (size_t)nq);
  int *ipt_d;
  A(&ipt_d, ipt.size()); A(&d.tmsub, 4 * (size_t)nt); A(&d.tcf, 5 * 24 * (size_t)nt); A(&d.tpart, 5 * 6 * (size_t)nt);
  if (rc != LAG2D_OK) { lag2d_destroy(h); return rc; }
  d.ipt = ipt_d;
  d.ipq = ipq_d; d.esq = esq_d; d.stencil = sten_d; d.node_ptr = ptr_d; d.node_cf = ncf_d;
  d.bcmask = mask_d; d.x0 = x0; d.y0 = y0;
  d.node_ptr2 = ptr2_d; d.node_slot = slot_d;
  std::vector<double> xx(np), yy(np);
  for (int p = 0; p < np; p++) { xx[p] = m->coold[2 * (size_t)p]; yy[p] = m->coold[2 * (size_t)p + 1]; }
#define UP(dst, src, n) cudaMemcpyAsync((void *)(dst), (src), (n) * sizeof(*(src)), cudaMemcpyHostToDevice, h->st)
  UP(ipq_d, ipq.data(), ipq.size()); UP(esq_d, esq.data(), esq.size()); UP(sten_d, sten.data(), sten.size());
  {
    std::vector<int> iptr(nq + 1, 0), ient;
    for (int c = 0; c < nq; c++)
      if (sten[c] >= 0)
        for (int k = 0; k < 9; k++) iptr[sten[k * (size_t)nq + c] - m->ntria + 1]++;
    for (int j = 0; j < nq; j++) iptr[j + 1] += iptr[j];
    ient.assign(std::max(iptr[nq], 1), 0);
    std::vector<int> fill(iptr.begin(), iptr.end() - 1);
    for (int c = 0; c < nq; c++)
      if (sten[c] >= 0)
        for (int k = 0; k < 9; k++) ient[fill[sten[k * (size_t)nq + c] - m->ntria]++] = c * 9 + k;
    if (dalloc(h, &h->sinv_ptr, iptr.size()) || dalloc(h, &h->sinv_ent, ient.size())) {
      lag2d_destroy(h);
      return LAG2D_ECUDA;
    }
    CK(cudaMemcpyAsync(h->sinv_ptr, iptr.data(), iptr.size() * sizeof(int), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->sinv_ent, ient.data(), ient.size() * sizeof(int), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
  }
  UP(ptr_d, cnt.data(), cnt.size()); UP(ncf_d, nodecf.data(), nodecf.size()); UP(mask_d, mask.data(), mask.size());
  UP(x0, xx.data(), np); UP(y0, yy.data(), np);
  UP(ptr2_d, cnt2.data(), cnt2.size()); UP(slot_d, slots.data(), slots.size());
  if (nt) UP(ipt_d, ipt.data(), ipt.size());
  UP(d.xn, xx.data(), np); UP(d.yn, yy.data(), np); UP(d.xs, xx.data(), np); UP(d.ys, yy.data(), np);
#undef UP
  QuadTables qt;
  fill_rule(5, false, qt.g25, qt.w25);
  fill_rule(6, false, qt.g36, qt.w36);
  fill_rule(5, true, qt.l25, qt.wl25);
  fill_tri_rule7(qt.t7, qt.tw7);
  set_tables(qt, h->st);
  Scalars s0{};
  cudaMemcpyAsync(d.sc_dev, &s0, sizeof(Scalars), cudaMemcpyHostToDevice, h->st);
  run(h, "init", [&] { launch_init_msub(d, h->st); launch_init_wmom(d, h->st); launch_tri_init(d, h->st); },
      2 + (nt > 0));
  if (cudaStreamSynchronize(h->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    lag2d_destroy(h);
    return fail(LAG2D_ECUDA, "device set-up failed");
  }
  *out = h;
  return LAG2D_OK;
}

static int download_geoel(lag2d_handle *h, double *geoel) {
  const Dev &d = h->d;
  const int ncell = d.ncell, nsize = ncell + d.nbfac;
  std::vector<double> f(ncell);
  std::fill(geoel, geoel + 24 * (size_t)nsize, 0.0);
  double *src[9] = {d.rc, d.sc, d.vol, d.mass, d.vcx, d.vcy, d.g19, d.g20, d.g21};
  const int slot[9] = {0, 1, 2, 3, 4, 5, 18, 19, 20};
  for (int k = 0; k < 9; k++) {
    CK(cudaMemcpyAsync(f.data(), src[k], ncell * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int e = 0; e < ncell; e++) geoel[24 * (size_t)e + slot[k]] = f[e];
  }
  return LAG2D_OK;
}

// unkno(ndegr,nq,nsize): the ncell real cells are copied, ghosts are zeroed
static int download_unkno(lag2d_handle *h, double *unkno) {
  const Dev &d = h->d;
  const size_t nu = NU * (size_t)d.ncell;
  launch_unkno_out(d, h->st, h->stage_u);
  h->launches += 1;
  CK(cudaMemcpyAsync(unkno, h->stage_u, nu * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  std::fill(unkno + nu, unkno + NU * (size_t)(d.ncell + d.nbfac), 0.0);
  return LAG2D_OK;
}


int lag2d_set_rho0(lag2d_handle *h, const double *rho0) {
  if (!h) return fail(LAG2D_EINVAL, "null handle");
  if (h->p1) return fail(LAG2D_EUNSUP, "the initial-density hook is built for the P2 path");
  Dev &d = h->d;
  if (rho0) {
    for (int e = 0; e < d.ncell; e++)
      if (!(rho0[e] > 0.0)) return fail(LAG2D_EINVAL, "rho0 must be positive");
    if (!h->rho0_dev) {
      int r = dalloc(h, &h->rho0_dev, (size_t)d.ncell);
      if (r) return r;
    }
    CK(cudaMemcpyAsync(h->rho0_dev, rho0, d.ncell * sizeof(double), cudaMemcpyHostToDevice, h->st));
    d.rho0 = h->rho0_dev;
  } else {
    d.rho0 = nullptr;
  }
  // the time-invariant reference-configuration masses lag2d_create computed
  // (sub-cell masses, mass-weighted shape moments) follow the new density
  run(h, "init", [&] { launch_init_msub(d, h->st); launch_init_wmom(d, h->st); launch_tri_init(d, h->st); },
      2 + (d.ntria > 0));
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  return LAG2D_OK;
}

int lag2d_init_fields(lag2d_handle *h, double *geoel, double *amatr, double *unkno) {
  if (!h) return fail(LAG2D_EINVAL, "null handle");
  if (h->p1) P1_CALL(p1::init_fields(h->p1, geoel, amatr, unkno, err_));
  Dev &d = h->d;
  const int ncell = d.ncell, np = d.npoin;
  run(h, "init", [&] { launch_tri_init(d, h->st); launch_init(d, h->st); }, 2 + (d.ntria > 0));
  CK(cudaMemcpyAsync(d.Us, d.Un, NU * (size_t)ncell * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync(d.xn, d.x0, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync(d.yn, d.y0, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync(d.xs, d.x0, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync(d.ys, d.y0, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemsetAsync(d.us, 0, np * sizeof(double), h->st));
  CK(cudaMemsetAsync(d.vs, 0, np * sizeof(double), h->st));
  run(h, "geom", [&] { geom_all(h, d.xn, d.yn); }, 1 + (d.ntria > 0));
  int st = read_status(h);
  if (st != LAG2D_OK) return st;
  if (geoel) { int r = download_geoel(h, geoel); if (r) return r; }
  if (amatr) {
    std::vector<double> f(16 * (size_t)ncell);
    CK(cudaMemcpyAsync(f.data(), d.amatr, f.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int e = 0; e < ncell; e++)
      for (int k = 0; k < 16; k++) amatr[16 * (size_t)e + k] = f[k * (size_t)ncell + e];
  }
  if (unkno) { int r = download_unkno(h, unkno); if (r) return r; }
  return LAG2D_OK;
}

int lag2d_set_state(lag2d_handle *h, const double *unkno, const double *coord, const double *ustar,
                    const double *geoel, const double *amatr) {
  if (!h || !unkno || !coord || !ustar) return fail(LAG2D_EINVAL, "null argument");
  if (h->p1) P1_CALL(p1::set_state(h->p1, unkno, coord, ustar, geoel, amatr, err_));
  Dev &d = h->d;
  const int ncell = d.ncell, np = d.npoin;
  // straight copies of the caller's buffers (pinned buffers go at full link
  // speed), then layout conversion on the device
  // the three copies go back to back (each into its own staging buffer), the
  // layout conversions queue behind them on the same stream
  CK(cudaMemcpyAsync(h->stage_u, unkno, NU * (size_t)ncell * sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->stage_x, coord, 2 * (size_t)np * sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->stage_v, ustar, 2 * (size_t)np * sizeof(double), cudaMemcpyHostToDevice, h->st));
  launch_unkno_in(d, h->st, h->stage_u, 1);
  launch_xy_in(np, h->st, h->stage_x, d.xn, d.yn, d.xs, d.ys);
  launch_xy_in(np, h->st, h->stage_v, d.us, d.vs, nullptr, nullptr);
  h->launches += 3;
  // host-side repacks of geoel / amatr live until the stream sync below
  std::vector<double> gslab, aslab;
  if (geoel) {
    double *dst[7] = {d.rc, d.sc, d.vol, d.mass, d.g19, d.g20, d.g21};
    const int slot[7] = {0, 1, 2, 3, 18, 19, 20};
    gslab.resize(7 * (size_t)ncell);
    for (int k = 0; k < 7; k++) {
      double *g = gslab.data() + k * (size_t)ncell;
      for (int e = 0; e < ncell; e++) g[e] = geoel[24 * (size_t)e + slot[k]];
      CK(cudaMemcpyAsync(dst[k], g, ncell * sizeof(double), cudaMemcpyHostToDevice, h->st));
    }
  }
  if (amatr) {
    aslab.resize(16 * (size_t)ncell);
    for (int e = 0; e < ncell; e++)
      for (int k = 0; k < 16; k++) aslab[k * (size_t)ncell + e] = amatr[16 * (size_t)e + k];
    CK(cudaMemcpyAsync(d.amatr, aslab.data(), aslab.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
  }
  Scalars s0{};
  CK(cudaMemcpyAsync(d.sc_dev, &s0, sizeof(Scalars), cudaMemcpyHostToDevice, h->st));
  run(h, "geom", [&] { geom_all(h, d.xs, d.ys); }, 1 + (d.ntria > 0));
  return read_status(h);
}

static int put_scalars(lag2d_handle *h, int itime, double dtfix, double tacru) {
  Scalars s{};
  CK(cudaMemcpyAsync(&s, h->d.sc_dev, sizeof(Scalars), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  s.dtfix = dtfix; s.tacru = tacru; s.itime = itime; s.done = 0; s.status = 0;
  CK(cudaMemcpyAsync(h->d.sc_dev, &s, sizeof(Scalars), cudaMemcpyHostToDevice, h->st));
  return LAG2D_OK;
}

static int get_scalars(lag2d_handle *h, Scalars *s) {
  CK(cudaMemcpyAsync(s, h->d.sc_dev, sizeof(Scalars), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return LAG2D_OK;
}

int lag2d_step(lag2d_handle *h, int itime, double *dtfix, double *tacru) {
  if (!h || !dtfix || !tacru) return fail(LAG2D_EINVAL, "null argument");
  if (h->p1) P1_CALL(p1::step(h->p1, itime, dtfix, tacru, err_));
  int r = put_scalars(h, itime, *dtfix, *tacru);
  if (r) return r;
  enqueue_step(h, itime);
  Scalars s;
  r = get_scalars(h, &s);
  if (r) return r;
  if (h->timing) flush_timing(h);
  *dtfix = s.dtfix;
  *tacru = s.tacru;
  return read_status(h);
}

int lag2d_run(lag2d_handle *h, int itime0, int nsteps, double *dtfix, double *tacru, int *done) {
  if (!h || !dtfix || !tacru || nsteps < 0) return fail(LAG2D_EINVAL, "bad argument");
  if (h->p1) P1_CALL(p1::run(h->p1, itime0, nsteps, dtfix, tacru, done, err_));
  int r = put_scalars(h, itime0 - 1, *dtfix, *tacru);
  if (r) return r;
  int steps = 0;
  if (h->timing) {
    // timed path: no graph, events around every kernel family
    for (int i = 0; i < nsteps; i++) { enqueue_step(h, itime0 + i); steps++; }
    flush_timing(h);
  } else {
    if (!h->graph) {
      // one step with itime incremented on the device, captured once
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
      long long before = h->launches;
      enqueue_step(h, -1);
      CK(cudaStreamEndCapture(h->st, &g));
      CK(cudaGraphInstantiate(&h->graph, g, 0));
      cudaGraphDestroy(g);
      h->graph_launches = h->launches - before;
      h->launches = before;  // counted per replay below
    }
    const long long per_step = h->graph_launches;
    for (int i = 0; i < nsteps; i++) {
      CK(cudaGraphLaunch(h->graph, h->st));
      h->launches += per_step;
      steps++;
    }
  }
  Scalars s;
  r = get_scalars(h, &s);
  if (r) return r;
  *dtfix = s.dtfix;
  *tacru = s.tacru;
  if (done) *done = s.done ? std::min(steps, std::max(0, s.itime - itime0 + 1)) : steps;
  return read_status(h);
}

int lag2d_get_state(lag2d_handle *h, double *unkno, double *coord, double *ustar, double *geoel) {
  if (!h) return fail(LAG2D_EINVAL, "null handle");
  if (h->p1) P1_CALL(p1::get_state(h->p1, unkno, coord, ustar, geoel, err_));
  // layout conversions into the staging buffers first, then the copies back to
  // back, then one synchronisation
  const Dev &d = h->d;
  const int np = d.npoin;
  const size_t nu = NU * (size_t)d.ncell;
  if (unkno) launch_unkno_out(d, h->st, h->stage_u);
  if (coord) launch_xy_out(np, h->st, h->stage_x, d.xn, d.yn);
  if (ustar) launch_xy_out(np, h->st, h->stage_v, d.us, d.vs);
  h->launches += (unkno != nullptr) + (coord != nullptr) + (ustar != nullptr);
  if (unkno) CK(cudaMemcpyAsync(unkno, h->stage_u, nu * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  if (coord) CK(cudaMemcpyAsync(coord, h->stage_x, 2 * (size_t)np * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  if (ustar) CK(cudaMemcpyAsync(ustar, h->stage_v, 2 * (size_t)np * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  if (unkno) std::fill(unkno + nu, unkno + NU * (size_t)(d.ncell + d.nbfac), 0.0);
  int r;
  if (geoel && (r = download_geoel(h, geoel))) return r;
  return LAG2D_OK;
}

int lag2d_rhs(lag2d_handle *h, int itime, double *rhsel, int *flags) {
  if (!h) return fail(LAG2D_EINVAL, "null handle");
  if (h->p1) {
    // no troubled-cell marking on the P1 branch
    if (flags) std::fill(flags, flags + h->d.ncell, 0);
    P1_CALL(p1::rhs(h->p1, rhsel, err_));
  }
  Dev &d = h->d;
  int r = put_scalars(h, itime, 0.0, 0.0);
  if (r) return r;
  const bool ex = h->cfg.order_exact != 0;
  run(h, "persson", [&] {
    launch_reset_count(d, h->st);
    if (ex) launch_persson(d, h->st); else launch_fast_persson(d, h->st);
  }, 2);
  if (flags) {
    CK(cudaMemcpyAsync(h->flags_dev, d.flag, d.ncell * sizeof(int), cudaMemcpyDeviceToDevice, h->st));
  }
  run(h, "weno", [&] { launch_weno(d, h->st); launch_weno_commit(d, h->st); }, 2);
  if (ex) {
    run(h, "corner", [&] { launch_tri_corner(d, h->st); launch_corner(d, h->st); }, 1 + (d.ntria > 0));
    run(h, "node", [&] { launch_node(d, h->st); });
    run(h, "rhs", [&] { launch_tri_rhs(d, h->st, d.us, d.vs, 0, 0.0); launch_rhs(d, h->st); }, 1 + (d.ntria > 0));
  } else {
    if (src_launches(d)) run(h, "src", [&] { src_pass(h, d); });
    run(h, "corner", [&] { corner_pass(h, d); }, corner_launches(h, d));
    run(h, "node", [&] { launch_fast_node(d, h->st); });
    run(h, "rhs", [&] { rhs_pass(h, d, 0, 0.0); }, rhs_launches(h, d));
    // the RHS keeps ustar of the previous stage for the impedances; expose the new one
    CK(cudaMemcpyAsync(d.us, d.us_new, d.npoin * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(d.vs, d.vs_new, d.npoin * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  }
  r = read_status(h);
  if (h->timing) flush_timing(h);
  if (r) return r;
  // the stage state is the limited one after the RHS, as in the reference
  CK(cudaMemcpyAsync(d.Un, d.Us, NU * (size_t)d.ncell * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  if (rhsel) {
    std::vector<double> f(NU * (size_t)d.ncell);
    CK(cudaMemcpyAsync(f.data(), d.rhs, f.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int e = 0; e < d.ncell; e++)
      for (int q = 0; q < NQ; q++)
        for (int k = 0; k < NDEG; k++) rhsel[(size_t)e * NU + q * NDEG + k] = f[(q * NDEG + k) * (size_t)d.ncell + e];
  }
  if (flags) {
    std::vector<int> fl(d.ncell);
    CK(cudaMemcpyAsync(fl.data(), h->flags_dev, d.ncell * sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int e = 0; e < d.ncell; e++) flags[e] = fl[e] != 0;
  }
  return LAG2D_OK;
}

int lag2d_weno(lag2d_handle *h, const int *flags) {
  if (!h || !flags) return fail(LAG2D_EINVAL, "null argument");
  if (h->p1) return fail(LAG2D_EUNSUP, "WENO is not on the P1 branch");
  Dev &d = h->d;
  int r = put_scalars(h, 1, 0.0, 0.0);
  if (r) return r;
  CK(cudaMemcpyAsync(h->flags_dev, flags, d.ncell * sizeof(int), cudaMemcpyHostToDevice, h->st));
  run(h, "persson", [&] { launch_reset_count(d, h->st); launch_persson(d, h->st); }, 2);
  run(h, "persson", [&] { launch_reset_count(d, h->st); launch_flags_from_host(d, h->st, h->flags_dev); }, 2);
  run(h, "weno", [&] { launch_weno(d, h->st); launch_weno_commit(d, h->st); }, 2);
  CK(cudaMemcpyAsync(d.Un, d.Us, NU * (size_t)d.ncell * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  r = read_status(h);
  if (h->timing) flush_timing(h);
  return r;
}

int lag2d_weno_linear(lag2d_handle *h, int transpose, const double *in, double *out) {
  if (!h || !in || !out) return fail(LAG2D_EINVAL, "null argument");
  if (h->p1) return fail(LAG2D_EUNSUP, "WENO is not on the P1 branch");
  if (h->cfg.order_exact) return fail(LAG2D_EUNSUP, "the linearised WENO follows the optimised step (order_exact 0)");
  Dev &d = h->d;
  const size_t nu = (size_t)NU * d.ncell;
  int r = put_scalars(h, 1, 0.0, 0.0);
  if (r) return r;
  // Persson marks and the reconstruction at the handle's state (not committed)
  run(h, "persson", [&] { launch_reset_count(d, h->st); launch_fast_persson(d, h->st); }, 2);
  run(h, "weno", [&] { launch_weno_warp(d, h->st); });
  const int cap = std::max(1, std::min(d.nquad, 16384));
  double *vbuf = nullptr, *obuf = nullptr, *wbuf = nullptr;
  int *wslot = nullptr, *overflow = nullptr;
  struct Free {
    std::vector<void *> p;
    ~Free() { for (void *q : p) cudaFree(q); }
  } fr;
  auto alloc = [&](void **q, size_t bytes) {
    cudaError_t e = cudaMalloc(q, std::max<size_t>(bytes, 8));
    if (e == cudaSuccess) { fr.p.push_back(*q); cudaMemsetAsync(*q, 0, std::max<size_t>(bytes, 8), h->st); }
    return e;
  };
  if (alloc((void **)&vbuf, nu * 8) || alloc((void **)&obuf, nu * 8) || alloc((void **)&wbuf, 216 * (size_t)cap * 8) ||
      alloc((void **)&wslot, (size_t)d.nquad * 4) || alloc((void **)&overflow, 4))
    return fail(LAG2D_ECUDA, "cudaMalloc (lag2d_weno_linear)");
  // the layout conversions read and write the view's U^n slab
  Dev dv = d, dout = d;
  dv.Un = vbuf;
  dout.Un = obuf;
  CK(cudaMemcpyAsync(h->stage_u, in, nu * sizeof(double), cudaMemcpyHostToDevice, h->st));
  launch_unkno_in(dv, h->st, h->stage_u, 0);
  CK(cudaMemcpyAsync(obuf, vbuf, nu * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  if (transpose) {
    launch_weno_linear(d, h->st, 1, vbuf, nullptr, wbuf, wslot, cap, overflow);
    launch_weno_gather(d, h->st, obuf, nullptr, 0, wbuf, wslot, cap, h->sinv_ptr, h->sinv_ent);
  } else {
    launch_weno_linear(d, h->st, 0, vbuf, obuf, nullptr, nullptr, cap, overflow);
  }
  launch_unkno_out(dout, h->st, h->stage_u);
  h->launches += 4;
  CK(cudaMemcpyAsync(out, h->stage_u, nu * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  int o = 0;
  CK(cudaMemcpyAsync(&o, overflow, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  if (o) return fail(LAG2D_EUNSUP, "more WENO-limited quads than the buffer holds");
  std::fill(out + nu, out + NU * (size_t)(d.ncell + d.nbfac), 0.0);
  return read_status(h);
}

int lag2d_cellvol(lag2d_handle *h, double *geoel) {
  if (!h) return fail(LAG2D_EINVAL, "null handle");
  if (h->p1) P1_CALL(p1::cellvol(h->p1, geoel, err_));
  run(h, "geom", [&] { geom_all(h, h->d.xs, h->d.ys); }, 1 + (h->d.ntria > 0));
  int r = read_status(h);
  if (r) return r;
  if (geoel) return download_geoel(h, geoel);
  return LAG2D_OK;
}

int lag2d_error_norms(lag2d_handle *h, double *errl2) {
  if (!h || !errl2) return fail(LAG2D_EINVAL, "null argument");
  if (h->p1) return fail(LAG2D_EUNSUP, "the error norms are built for the P2 path");
  Dev &d = h->d;
  if (d.ntria > 0) return fail(LAG2D_EUNSUP, "the error norms are built for all-quad meshes");
  if (d.ncase != 1 && d.ncase != 2)
    return fail(LAG2D_EUNSUP, "geterror_lag_curvhybrid has an exact solution for the cases 1 and 2 only");
  const int nb = error_blocks(d);
  if (!h->errpart) {
    int r = dalloc(h, &h->errpart, 3 * (size_t)nb);
    if (r) return r;
  }
  run(h, "error", [&] { launch_error(d, h->st, d.xs, d.ys, h->errpart); });
  std::vector<double> part(3 * (size_t)nb);
  CK(cudaMemcpyAsync(part.data(), h->errpart, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  double e[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < nb; b++)
    for (int k = 0; k < 3; k++) e[k] += part[3 * (size_t)b + k];
  for (int k = 0; k < 3; k++) errl2[k] = std::sqrt(e[k]);
  return LAG2D_OK;
}

int lag2d_cell_output(lag2d_handle *h, double *cellout, double *badcell) {
  if (!h || !cellout) return fail(LAG2D_EINVAL, "null argument");
  if (h->p1) {
    if (badcell) std::fill(badcell, badcell + h->d.ncell, 0.0);
    P1_CALL(p1::cell_output(h->p1, cellout, err_));
  }
  Dev &d = h->d;
  if (!h->cellout) {
    int r = dalloc(h, &h->cellout, 9 * (size_t)d.ncell);
    if (r) return r;
  }
  run(h, "post", [&] { launch_cell_output(d, h->st, d.Un, d.xn, d.yn, h->cellout); });
  std::vector<double> v(9 * (size_t)d.ncell);
  CK(cudaMemcpyAsync(v.data(), h->cellout, v.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  if (badcell) {
    // getSIHO_Persson on the state, as the reference's driver runs it before
    // writing the cell file: 100 on troubled quads, 0 elsewhere
    run(h, "persson", [&] {
      launch_reset_count(d, h->st);
      if (h->cfg.order_exact) launch_persson(d, h->st); else launch_fast_persson(d, h->st);
    }, 2);
    std::vector<int> f(d.ncell);
    CK(cudaMemcpyAsync(f.data(), d.flag, d.ncell * sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int e = 0; e < d.ncell; e++) badcell[e] = (e >= d.ntria && f[e] != 0) ? 100.0 : 0.0;
  }
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  for (size_t e = 0; e < (size_t)d.ncell; e++)
    for (int k = 0; k < 9; k++) cellout[9 * e + k] = v[k * (size_t)d.ncell + e];
  return LAG2D_OK;
}

long long lag2d_kernel_launches(const lag2d_handle *h) {
  if (!h) return -1;
  return h->p1 ? p1::launches(h->p1) : h->launches;
}

void *lag2d_stream(const lag2d_handle *h) { return h ? (void *)h->st : nullptr; }

int lag2d_timing(lag2d_handle *h, int enable) {
  if (!h) return fail(LAG2D_EINVAL, "null handle");
  if (h->p1) p1::set_timing(h->p1, enable != 0);
  h->timing = enable != 0;
  h->fam.clear();
  return LAG2D_OK;
}

double lag2d_kernel_ms(const lag2d_handle *h, const char *family, long long *launches) {
  if (!h || !family) return -1.0;
  if (h->p1) return p1::kernel_ms(h->p1, family, launches);
  auto it = h->fam.find(family);
  if (it == h->fam.end() || it->second.n == 0) return -1.0;
  if (launches) *launches = it->second.n;
  return it->second.ms / it->second.n;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint of the optimised step (quads and triangles; FP64, or FP32-mixed when
// the handle's precision is 1: the recompute runs the mixed forward passes and the
// reverse the mixed transposes).
//
// Reverse mode per RK stage with the time step size, the Persson marks and
// the WENO active set (chosen stencil, nonlinear weights, characteristic
// frame) frozen from the forward pass: the reconstruction is differentiated
// as the linear map it is for those choices.  Marked cells whose stencil is
// rejected keep their DOFs and are differentiated as unlimited cells; more
// than 16384 replaced quads in a stage return LAG2D_EUNSUP.
// Reference-configuration quantities (cell masses, mass matrices,
// initial-mesh moments) are constants.
// The stage inputs are recorded by recomputing each checkpoint segment, so the
// device memory of a window is (segments + 1) checkpoints plus K steps of
// stage records.
struct AdjWork {
  lag2d_handle *h;
  std::vector<void *> mem;
  Adj a{};
  StageRec rec{};
  int rc = LAG2D_OK;
  // WENO transpose: per-slot stencil adjoints, slot of each troubled quad,
  // overflow flag; cap = slots per stage
  double *wbuf = nullptr;
  int *wslot = nullptr, *overflow = nullptr;
  int cap = 0;
  explicit AdjWork(lag2d_handle *hh) : h(hh) {}
  ~AdjWork() {
    cudaStreamSynchronize(h->st);
    for (void *q : mem) cudaFree(q);
  }
  template <typename T> void alloc(T **p, size_t n) {
    if (rc != LAG2D_OK) return;
    void *q = nullptr;
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      rc = fail(LAG2D_ECUDA, std::string("cudaMalloc (adjoint): ") + cudaGetErrorString(e));
      return;
    }
    cudaMemsetAsync(q, 0, bytes, h->st);
    mem.push_back(q);
    *p = static_cast<T *>(q);
  }
  // adjoint buffers plus the stage records of K steps
  void setup(int K) {
    const Dev &d = h->d;
    const size_t nu = (size_t)NU * d.ncell, np = d.npoin;
    const int nstag = h->cfg.nstag;
    alloc(&a.lU, nu); alloc(&a.lUn, nu); alloc(&a.lR, nu);
    alloc(&a.lx, np); alloc(&a.ly, np); alloc(&a.lxn, np); alloc(&a.lyn, np); alloc(&a.lus, np); alloc(&a.lvs, np);
    alloc(&a.luw, np); alloc(&a.lvw, np); alloc(&a.tx, np); alloc(&a.ty, np);
    alloc(&a.lS, 5 * np); alloc(&a.lP, 45 * (size_t)d.nquad); alloc(&a.pbuf, 54 * (size_t)d.nquad);
    alloc(&a.lcorr, 4 * (size_t)d.nquad);
    alloc(&a.tbuf, 36 * (size_t)d.ntria); alloc(&a.ltcf, 120 * (size_t)d.ntria);
    const size_t ns = (size_t)K * nstag;
    alloc(&rec.U, ns * nu); alloc(&rec.x, ns * np); alloc(&rec.y, ns * np);
    alloc(&rec.us, ns * np); alloc(&rec.vs, ns * np); alloc(&rec.dt, K);
    alloc(&rec.npart, ns * 45 * (size_t)d.nquad); alloc(&rec.corr, ns * 4 * (size_t)d.nquad);
    alloc(&rec.usn, ns * np); alloc(&rec.vsn, ns * np);
    alloc(&rec.tcf, ns * 120 * (size_t)d.ntria); alloc(&rec.tpart, ns * 30 * (size_t)d.ntria);
    rec.nstag = nstag; rec.nu = nu; rec.np = np; rec.nq = d.nquad; rec.nt = d.ntria;
    cap = std::max(1, std::min(d.nquad, 16384));
    alloc(&wbuf, 216 * (size_t)cap); alloc(&wslot, (size_t)d.nquad); alloc(&overflow, 1);
  }
  // forward of nk steps from the handle's state, recording every stage input
  int record(int itime, int nk) {
    for (int k = 0; k < nk; k++) {
      rec.step = k;
      enqueue_step_fast(h, itime + k, &rec);
    }
    return LAG2D_OK;
  }
  int check_overflow() {
    int o = 0;
    CK(cudaMemcpyAsync(&o, overflow, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (o)
      return fail(LAG2D_EUNSUP, "more WENO-limited quads in one stage than the adjoint's WENO buffer holds (" +
                                    std::to_string(cap) + ")");
    return LAG2D_OK;
  }
  // reverse of the nk recorded steps; a.lU / a.lx / a.lus hold the adjoints of
  // the last step's outputs on entry and of the first step's inputs on return
  // Each stage's reverse linearises at the state after WENO: Persson and
  // WENO run again on the recorded stage input (same marks, same
  // reconstruction) and the replaced moments are swapped into the record in
  // place; the reverse kernels run on it; the swap back restores the input;
  // then the WENO transpose, with its stencils, weights, frame and
  // characteristic matrices taken at the input (the limiter's active set
  // frozen), maps the adjoint of the post-WENO state to that of the input.
  void reverse(int nk) {
    const int nstag = h->cfg.nstag;
    // the recompute must not see the end-of-run flag a window ending at tend leaves
    cudaMemsetAsync(&h->d.sc_dev->done, 0, sizeof(int), h->st);
    for (int k = nk - 1; k >= 0; k--) {
      for (int istag = nstag; istag >= 1; istag--) {
        const Dev ds = rec.inputs(h->d, (size_t)k * nstag + (istag - 1));
        // the stage's cell volumes (WENO scales its stencil bases by them) from
        // the recorded nodes, as the forward pass had them
        launch_tri_geom(ds, h->st, ds.xs, ds.ys);
        launch_fast_geom(ds, h->st, 0);
        launch_reset_count(ds, h->st);
        launch_fast_persson(ds, h->st);
        launch_weno_warp(ds, h->st);
        launch_weno_swap(ds, h->st);
        // stage 1 reads x^n directly: its reverse folds the coordinate adjoints
        // in; the U^n fold waits for the WENO transpose (in the gather)
        launch_adjoint_stage(ds, &a, h->st, kRK[nstag - 2][istag - 1], rec.dt + k, istag == 1, 0,
                             h->cfg.precision == 1);
        launch_weno_swap(ds, h->st);
        launch_weno_linear(ds, h->st, 1, a.lU, nullptr, wbuf, wslot, cap, overflow);
        launch_weno_gather(ds, h->st, a.lU, a.lUn, istag == 1, wbuf, wslot, cap, h->sinv_ptr, h->sinv_ent);
        h->launches += adjoint_stage_launches(h->d) + 8 + (h->d.ntria > 0);
      }
    }
  }
};

// whole-state snapshot of the handle (U^n, x^n, ustar, scalars)
struct Snapshot {
  double *U = nullptr, *x = nullptr, *y = nullptr, *us = nullptr, *vs = nullptr;
  Scalars *sc = nullptr;
  void alloc(AdjWork &w, int n) {
    const size_t nu = (size_t)NU * w.h->d.ncell, np = w.h->d.npoin;
    w.alloc(&U, n * nu); w.alloc(&x, n * np); w.alloc(&y, n * np); w.alloc(&us, n * np); w.alloc(&vs, n * np);
    w.alloc(&sc, n);
  }
  void save(lag2d_handle *h, int c) const {
    const Dev &d = h->d;
    const size_t nu = (size_t)NU * d.ncell, np = d.npoin;
    cudaMemcpyAsync(U + c * nu, d.Un, nu * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(x + c * np, d.xn, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(y + c * np, d.yn, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(us + c * np, d.us, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(vs + c * np, d.vs, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(sc + c, d.sc_dev, sizeof(Scalars), cudaMemcpyDeviceToDevice, h->st);
  }
  void restore(lag2d_handle *h, int c) const {
    const Dev &d = h->d;
    const size_t nu = (size_t)NU * d.ncell, np = d.npoin;
    cudaMemcpyAsync(d.Un, U + c * nu, nu * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(d.Us, U + c * nu, nu * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(d.xn, x + c * np, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(d.xs, x + c * np, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(d.yn, y + c * np, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(d.ys, y + c * np, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(d.us, us + c * np, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(d.vs, vs + c * np, np * sizeof(double), cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(d.sc_dev, sc + c, sizeof(Scalars), cudaMemcpyDeviceToDevice, h->st);
    // cell volumes (and triangle centres) of the restored nodes: the next
    // stage 1 reads them in WENO and the time step
    launch_tri_geom(d, h->st, d.xs, d.ys);
    launch_fast_geom(d, h->st, 0);
    h->launches += 1 + (d.ntria > 0);
  }
};

static int adjoint_supported(lag2d_handle *h) {
  if (h->p1) return fail(LAG2D_EUNSUP, "the adjoint is built for the P2 path");
  if (h->cfg.order_exact)
    return fail(LAG2D_EUNSUP, "the adjoint follows the optimised step (order_exact 0)");
  return LAG2D_OK;
}

// caller layouts <-> device SoA for the adjoint fields
static int put_adjoint(lag2d_handle *h, const Adj &a, const double *unkno, const double *coord,
                       const double *ustar) {
  const Dev &d = h->d;
  const size_t nc = d.ncell, np = d.npoin, nu = (size_t)NU * nc;
  std::vector<double> g(nu, 0.0);
  if (unkno)
    for (size_t e = 0; e < nc; e++)
      for (int t = 0; t < NU; t++) g[(size_t)t * nc + e] = unkno[e * NU + t];
  CK(cudaMemcpyAsync(a.lU, g.data(), nu * sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  const double *src[2] = {coord, ustar};
  double *dst[2][2] = {{a.lx, a.ly}, {a.lus, a.lvs}};
  std::vector<double> gx(np), gy(np);
  for (int f = 0; f < 2; f++) {
    for (size_t p = 0; p < np; p++) {
      gx[p] = src[f] ? src[f][2 * p] : 0.0;
      gy[p] = src[f] ? src[f][2 * p + 1] : 0.0;
    }
    CK(cudaMemcpyAsync(dst[f][0], gx.data(), np * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(dst[f][1], gy.data(), np * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
  }
  return LAG2D_OK;
}
static int get_adjoint(lag2d_handle *h, const Adj &a, double *unkno, double *coord, double *ustar) {
  const Dev &d = h->d;
  const size_t nc = d.ncell, np = d.npoin, nu = (size_t)NU * nc;
  if (unkno) {
    std::vector<double> g(nu);
    CK(cudaMemcpyAsync(g.data(), a.lU, nu * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (size_t e = 0; e < nc; e++)
      for (int t = 0; t < NU; t++) unkno[e * NU + t] = g[(size_t)t * nc + e];
  }
  const double *src[2][2] = {{a.lx, a.ly}, {a.lus, a.lvs}};
  double *dst[2] = {coord, ustar};
  std::vector<double> gx(np), gy(np);
  for (int f = 0; f < 2; f++) {
    if (!dst[f]) continue;
    CK(cudaMemcpyAsync(gx.data(), src[f][0], np * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(gy.data(), src[f][1], np * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (size_t p = 0; p < np; p++) {
      dst[f][2 * p] = gx[p];
      dst[f][2 * p + 1] = gy[p];
    }
  }
  return LAG2D_OK;
}

extern "C" {

int lag2d_adjoint_step(lag2d_handle *h, int itime, double *dtfix, double *tacru, const double *seed_unkno,
                       const double *seed_coord, const double *seed_ustar, double *grad_unkno, double *grad_coord,
                       double *grad_ustar) {
  if (!h || !dtfix || !tacru) return fail(LAG2D_EINVAL, "null argument");
  int r = adjoint_supported(h);
  if (r) return r;
  AdjWork w(h);
  w.setup(1);
  if (w.rc) return w.rc;
  r = put_scalars(h, itime, *dtfix, *tacru);
  if (r) return r;
  w.record(itime, 1);
  Scalars fin;
  r = get_scalars(h, &fin);
  if (r) return r;
  // a broken state ends here; the stencil notice (a troubled quad left
  // unlimited, the step complete) lets the reverse run and is returned last
  if (fin.status & ST_NONPHYS) return read_status(h);
  r = put_adjoint(h, w.a, seed_unkno, seed_coord, seed_ustar);
  if (r) return r;
  // keep the step's outputs: the reverse pass overwrites the stage buffers
  Snapshot out;
  out.alloc(w, 1);
  if (w.rc) return w.rc;
  out.save(h, 0);
  w.reverse(1);
  out.restore(h, 0);
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  if ((r = w.check_overflow())) return r;
  r = get_adjoint(h, w.a, grad_unkno, grad_coord, grad_ustar);
  if (r) return r;
  *dtfix = fin.dtfix;
  *tacru = fin.tacru;
  if (fin.status & ST_STENCIL)
    return fail(LAG2D_ESTENCIL, "WENO left a troubled quad unlimited (vertex valence); step and gradients complete");
  return LAG2D_OK;
}

int lag2d_adjoint(lag2d_handle *h, int itime0, int nsteps, int checkpoint_every, double *dtfix, double *tacru,
                  double *J, double *dJ_dunkno, double *dJ_dcoord, double *dJ_dustar, double *ms) {
  if (!h || !dtfix || !tacru || !J) return fail(LAG2D_EINVAL, "null argument");
  if (nsteps < 1 || checkpoint_every < 1) return fail(LAG2D_EINVAL, "nsteps and checkpoint_every must be >= 1");
  int r = adjoint_supported(h);
  if (r) return r;
  Dev &d = h->d;
  const int K = std::min(checkpoint_every, nsteps);
  const int nseg = (nsteps + K - 1) / K;
  const size_t nc = d.ncell, nu = (size_t)NU * nc;
  AdjWork w(h);
  w.setup(K);
  Snapshot ck;
  ck.alloc(w, nseg + 1);
  if (w.rc) return w.rc;
  cudaEvent_t ev[2];
  CK(cudaEventCreate(&ev[0]));
  CK(cudaEventCreate(&ev[1]));
  struct EvGuard {
    cudaEvent_t *e;
    ~EvGuard() { cudaEventDestroy(e[0]); cudaEventDestroy(e[1]); }
  } evg{ev};
  auto elapsed = [&] {
    float t = 0.f;
    cudaEventSynchronize(ev[1]);
    cudaEventElapsedTime(&t, ev[0], ev[1]);
    return (double)t;
  };
  double t_fwd = 0, t_rec = 0, t_rev = 0;
  // forward with a checkpoint at every segment start and at the end
  r = put_scalars(h, itime0, *dtfix, *tacru);
  if (r) return r;
  cudaEventRecord(ev[0], h->st);
  for (int n = 0; n < nsteps; n++) {
    if (n % K == 0) ck.save(h, n / K);
    enqueue_step_fast(h, itime0 + n);
  }
  ck.save(h, nseg);
  cudaEventRecord(ev[1], h->st);
  t_fwd = elapsed();
  Scalars fin;
  r = get_scalars(h, &fin);
  if (r) return r;
  if (fin.status & ST_NONPHYS) return read_status(h);
  if (fin.done && fin.itime != itime0 + nsteps - 1)
    return fail(LAG2D_EINVAL, "the window runs past tend (the steps after it are skipped)");
  // J and its seed dJ/dU = m (0, u, v, 0) in the cell-average modes
  {
    std::vector<double> u(nc), v(nc), m(nc);
    CK(cudaMemcpyAsync(u.data(), d.Un + 6 * nc, nc * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(v.data(), d.Un + 12 * nc, nc * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(m.data(), d.mass, nc * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    double s = 0.0;
    std::vector<double> seed(nu, 0.0);
    for (size_t e = 0; e < nc; e++) {
      s += 0.5 * m[e] * (u[e] * u[e] + v[e] * v[e]);
      seed[6 * nc + e] = m[e] * u[e];
      seed[12 * nc + e] = m[e] * v[e];
    }
    *J = s;
    CK(cudaMemcpyAsync(w.a.lU, seed.data(), nu * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
  }
  // reverse sweep, one segment at a time: recompute it from its checkpoint
  // with the stage inputs recorded, then run its steps backwards
  for (int sg = nseg - 1; sg >= 0; sg--) {
    const int n0 = sg * K, nk = std::min(K, nsteps - n0);
    ck.restore(h, sg);
    cudaEventRecord(ev[0], h->st);
    w.record(itime0 + n0, nk);
    cudaEventRecord(ev[1], h->st);
    t_rec += elapsed();
    cudaEventRecord(ev[0], h->st);
    w.reverse(nk);
    cudaEventRecord(ev[1], h->st);
    t_rev += elapsed();
  }
  // the handle returns to the final forward state
  ck.restore(h, nseg);
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  if ((r = w.check_overflow())) return r;
  r = get_adjoint(h, w.a, dJ_dunkno, dJ_dcoord, dJ_dustar);
  if (r) return r;
  *dtfix = fin.dtfix;
  *tacru = fin.tacru;
  if (ms) {
    ms[0] = t_fwd;
    ms[1] = t_rec;
    ms[2] = t_rev;
  }
  if (fin.status & ST_STENCIL)
    return fail(LAG2D_ESTENCIL, "WENO left a troubled quad unlimited (vertex valence); window and gradients complete");
  return LAG2D_OK;
}

void lag2d_destroy(lag2d_handle *h) {
  if (!h) return;
  if (h->p1) p1::destroy(h->p1);
  if (h->st) cudaStreamSynchronize(h->st);
  for (auto &p : h->pending) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (void *p : h->allocs) cudaFree(p);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

}  // extern "C"
