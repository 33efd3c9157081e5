// The linear P1 time step on straight 4-node quads (ncurv = 0, nfint = 1,
// nlimi = 6, nrz = 0): the host side of lag2d_p1.cu, called by the C-ABI
// entry points of lag2d_capi.cu when lag2d_create sees npoly = 1.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "lag2d.h"

namespace lag2d {
namespace p1 {

struct Solver;

// Every call returns a LAG2D_* status; on failure err receives the text.
int create(const lag2d_mesh *m, const lag2d_config *c, cudaStream_t st, Solver **out, std::string &err);
int init_fields(Solver *s, double *geoel, double *amatr, double *unkno, std::string &err);
int set_state(Solver *s, const double *unkno, const double *coord, const double *ustar, const double *geoel,
              const double *amatr, std::string &err);
int step(Solver *s, int itime, double *dtfix, double *tacru, std::string &err);
int run(Solver *s, int itime0, int nsteps, double *dtfix, double *tacru, int *done, std::string &err);
int get_state(Solver *s, double *unkno, double *coord, double *ustar, double *geoel, std::string &err);
int rhs(Solver *s, double *rhsel, std::string &err);
int cellvol(Solver *s, double *geoel, std::string &err);
int cell_output(Solver *s, double *out, std::string &err);
long long launches(const Solver *s);
void set_timing(Solver *s, bool on);
double kernel_ms(const Solver *s, const char *family, long long *n);
void destroy(Solver *s);

}  // namespace p1
}  // namespace lag2d
