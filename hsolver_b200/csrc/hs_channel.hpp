// Channel conjugate-heat-transfer SIMPLE solver (implemented in
// hs_channel.cu): inlet plug flow at x = 0, zero-gradient outlet at x = Nx,
// no-slip walls, solid blocks with a volumetric heat source and a
// conductivity ratio, energy in fluid and solid as one operator.
#pragma once
#include <cstdint>

#include "hs_case.hpp"

namespace hs {

struct ChParams {
  double re, pr, u_in, t_in;        // Reynolds number on the channel height, Prandtl number, inlet values
  double alpha_u, alpha_p, alpha_t; // relaxation of momentum, pressure, temperature
  int mom_sweeps;                   // red-black Gauss-Seidel sweeps per momentum solve
  double p_tol;                     // pressure-correction CG: ||r|| / ||b|| stop
  int p_maxiter;
  double t_tol;                     // energy BiCGStab: ||r|| / ||r0|| stop
  int t_maxiter;
  int precision;                    // 0 FP64, 1 mixed (FP32 fields, sweeps and V-cycle)
  int p_precond;                    // 0 plain CG, 1 multigrid V-cycle
  int p_mg_sweeps;                  // V-cycle sweeps on the finest level (0: 2); coarser levels one more
  int p_level0;                     // finest level of the p' solve: 0 the default form, 1 grid-wide, 2 z-marching
  int conv;                         // momentum convection: 0 first-order upwind, 1 hybrid, 2 QUICK (deferred correction)
  int g_axis;                       // buoyancy along + this axis (gravity along -g_axis)
  double ri;                        // Richardson number Gr / Re^2 of the Boussinesq term (0: none)
};

struct ChStats {
  double res[5];      // momentum u v w, continuity, energy (absolute)
  double norm[5];     // maximum of each over the first five outer steps
  double global;      // max_x res[x] / norm[x]
  int iter, pcg_iters, t_iters;
  double pcg_relres, t_relres;
};

struct ChannelState;
ChannelState *ch_create(const Case &c, const ChParams &p, int device);
void ch_destroy(ChannelState *s);
int ch_nreg(const ChannelState *s);
void ch_set_solid(ChannelState *s, const double *k_ratio_region, const double *q_cell);
void ch_init(ChannelState *s);
// flags: bit 0 skip the pressure correction solve (p' = 0), bit 1 skip the energy solve
void ch_step(ChannelState *s, int n, int flags, ChStats *out);
// outer steps until the global residual <= tol or max_outer steps; returns steps taken
int ch_solve_to(ChannelState *s, double tol, int max_outer, ChStats *out);
long ch_field_size(const ChannelState *s, int f);
void ch_get_field(ChannelState *s, int f, double *host, long n);
void ch_set_field(ChannelState *s, int f, const double *host, long n);
void *ch_stream(ChannelState *s);
// per-phase CUDA-event times (momentum, p' assembly, p' solve, correction,
// energy), summed over the steps since profiling was switched on
void ch_profile(ChannelState *s, bool on);
int ch_profile_read(const ChannelState *s, double *ms5);
void ch_sync(ChannelState *s);
// FP64 global balances of the current state (blocking): volume flux in and
// out, heat source, heat leaving through the boundary
void ch_balance(ChannelState *s, double out4[4]);
long long ch_device_bytes(const ChannelState *s);
// energy adjoint on the current (frozen) flow: forward solve of the energy
// equation from T = t_in to tol, then the adjoint; J = (sum_solid T^8 V)^(1/8)
void ch_adjoint(ChannelState *s, double tol, int maxiter, double *J, double *dJdq, double *dJdk, int *fwd_iters,
                int *adj_iters, double *fwd_ms, double *adj_ms);

}  // namespace hs
