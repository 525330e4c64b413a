// Monolithic conjugate-heat-transfer energy solve with a frozen flow field and
// its adjoint (implemented in hs_cht.cu).
#pragma once
#include <cstdint>

namespace hs {

struct ChtSetup {
  int device;
  void *stream;                   // cudaStream_t of the owning solver
  int Nx, Ny, Nz, nreg;
  const double *xs, *ys, *zs;     // host grid points
  const uint8_t *ctype;           // host, Nx*Ny*Nz, 1 = solid
  const int *region;              // host, solid region per cell
  double t_boundary, tol;
  int maxiter;
};

// where the face velocities come from: the fluid box's padded u*, v*, w*
struct ChtVelSrc {
  int Nx, Ny, Nz, cx, cy, cz, fx, fy, fz, ox, oy, oz;
  const double *u, *v, *w;        // device
  const uint8_t *ctype;           // device, Nx*Ny*Nz (filled by cht_set_velocities)
};

struct ChtState;
ChtState *cht_create(const ChtSetup &s);
void cht_destroy(ChtState *c);
void cht_set_solid(ChtState *c, double k_fluid, const double *k_region, const double *q_cell);
void cht_set_velocities(ChtState *c, const ChtVelSrc &src);
void cht_get_velocities(ChtState *c, double *ug, double *vg, double *wg);
void cht_forward(ChtState *c, double *T_host, double *J, int *iters, double *relres);
void cht_adjoint(ChtState *c, double *dJdq_host, double *dJdk_host, int *iters, double *relres);

}  // namespace hs
