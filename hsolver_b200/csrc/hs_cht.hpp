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
  int bc;                         // 0 Dirichlet t_boundary on every boundary face; 1 channel (Dirichlet at
                                  // x = 0, upwind outflow at x = Nx, adiabatic y / z walls)
  int precond;                    // BiCGStab preconditioner: 0 Jacobi, 1 multigrid V-cycle in FP32, 2 in FP64
  int step_fp32 = 0;              // cht_energy_step solves for the correction to T with FP32 Krylov vectors
                                  // (residual, dot products and T in FP64)
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
// device_done: a cudaEvent_t recorded on the solver's stream once the
// gradients are on the device, before their copies to the host (or null)
void cht_adjoint(ChtState *c, double *dJdq_host, double *dJdk_host, int *iters, double *relres,
                 void *device_done = nullptr);
// channel use: the owner's device face velocities, T = v everywhere, one relaxed
// energy step (BiCGStab from the current T to tol * ||r0||, T += alpha (T~ - T);
// with step_fp32, BiCGStab for the correction d = T~ - T from 0 in FP32 vectors,
// T += alpha d), its results (iterations, ||r|| / ||r0||, ||r0||) after a stream sync
void cht_bind_velocities(ChtState *c, const double *ug, const double *vg, const double *wg);
void cht_fill_T(ChtState *c, double v);
double *cht_T_device(ChtState *c);
void cht_energy_step(ChtState *c, double alpha_t, double tol, int maxiter);
void cht_step_results(ChtState *c, int *iters, double *relres, double *r0);
// the same results copied on the owner's stream, without waiting, into
// (pinned) host memory: iterations, then ||r|| / ||r0|| and ||r0||
void cht_step_results_async(ChtState *c, int *iters, double *relres_r0);
void cht_set_tolerance(ChtState *c, double tol, int maxiter);
// channel form: FP64 global balances {volume flux in at x = 0, out at
// x = Nx, sum of q V, heat leaving through the boundary faces}, blocking
void cht_balance(ChtState *c, double out4[4]);

}  // namespace hs
