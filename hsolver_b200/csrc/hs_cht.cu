// Conjugate-heat-transfer energy equation on the whole grid (fluid and solid
// cells as one operator) with the flow frozen at the solver's current face
// velocities, and its adjoint for J = (sum_solid T^8 dV)^(1/8).
//
// The reference couples fluid and solid temperatures only through a ghost
// value swap (solver.h:62-148) and has no heat source, conductivity ratio or
// adjoint; this module is the monolithic form: per face between cells P, N
//   G = A / (dP/(2 kP) + dN/(2 kN))     (harmonic-mean interface conductance)
//   F = u A (outward from P)            (first-order upwind convection)
// boundary faces carry Dirichlet Tb through G_b = 2 kP A / dP (bc = 0), or,
// for the channel (bc = 1), only the inlet face x = 0 does and the others are
// adiabatic, with upwind outflow at x = Nx; row P is
//   (sum G + max(F,0)) T_P - sum (G + max(-F,0)) T_N = q_P V_P + boundary terms.
// The transposed operator has the same stencil with the upwind side swapped:
// A^T_{P,N} = A_{N,P}, read from the neighbour's stored coefficient.
// Both solves use the same cooperative BiCGStab, preconditioned by the
// geometric multigrid V-cycle of hs_mg.cuh on the same operator (or by
// Jacobi).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "hs_cht.hpp"
#include "hs_mg.cuh"

namespace cg = cooperative_groups;

namespace hs {

#define HC_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_) + \
                                                    " at " #call);                                 \
  } while (0)

namespace {

constexpr int kB = 256;
// the cooperative BiCGStab: one block per SM (few arrivals at each grid
// barrier) of 1024 threads, the fastest of 512 / 768 / 1024 on a 256x128x128
// channel (energy step 1.85 / 1.60 / 1.57 ms in FP64, 1.29 / 1.16 / 1.13 mixed)
constexpr int kBiT = 1024;

struct ChtDev {
  int Nx, Ny, Nz;
  const double *dx, *dy, *dz;      // cell widths
  const uint8_t *solid;            // padded
  const double *k;                 // padded conductivity
  const double *q;                 // padded source
  const double *ug, *vg, *wg;      // global face velocities
  double *d, *aw, *ae, *as, *an, *ab, *af, *b, *dinv;  // padded coefficients
  int bc;                          // 0 Dirichlet everywhere, 1 channel
};

__device__ __forceinline__ int pidx(const ChtDev &H, int i, int j, int k) {  // 0-based cell -> padded
  return (i + 1) + (H.Nx + 2) * ((j + 1) + (H.Ny + 2) * (k + 1));
}

__device__ double blk_sum(double v, double *sh) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (wid == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;
}

// several sums at once over the grid, identical in every thread
template <int M>
__device__ void grid_sums(double (&v)[M], double *partials, int &buf, double *sh, cg::grid_group &grid) {
  double *pp = partials + (size_t)buf * gridDim.x * M;
  buf ^= 1;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double b = blk_sum(v[m], sh);
    if (threadIdx.x == 0) pp[(size_t)blockIdx.x * M + m] = b;
  }
  grid.sync();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int m = 0; m < M; ++m) {
      double a = 0.0;
      for (int q = threadIdx.x; q < (int)gridDim.x; q += 32) a += __ldcg(pp + (size_t)q * M + m);
      for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (threadIdx.x == 0) sh[40 + m] = a;
    }
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < M; ++m) v[m] = sh[40 + m];
  __syncthreads();
}

// face (direction d: W E S N B F) of cell (i,j,k): conductance, outward flux, neighbour exists
__device__ __forceinline__ void face(const ChtDev &H, int i, int j, int k, int d, double &G, double &F, bool &has) {
  const double dxi = H.dx[i], dyj = H.dy[j], dzk = H.dz[k];
  const double kp = H.k[pidx(H, i, j, k)];
  const int ax = d >> 1, hi = d & 1;
  double A, dP, dN = 0, u;
  int ii = i, jj = j, kk = k;
  if (ax == 0) {
    A = dyj * dzk; dP = dxi; ii = hi ? i + 1 : i - 1;
    u = H.ug[(hi ? i + 1 : i) + (H.Nx + 1) * (j + H.Ny * k)];
    has = ii >= 0 && ii < H.Nx; if (has) dN = H.dx[ii];
  } else if (ax == 1) {
    A = dxi * dzk; dP = dyj; jj = hi ? j + 1 : j - 1;
    u = H.vg[i + H.Nx * ((hi ? j + 1 : j) + (H.Ny + 1) * k)];
    has = jj >= 0 && jj < H.Ny; if (has) dN = H.dy[jj];
  } else {
    A = dxi * dyj; dP = dzk; kk = hi ? k + 1 : k - 1;
    u = H.wg[i + H.Nx * (j + H.Ny * (hi ? k + 1 : k))];
    has = kk >= 0 && kk < H.Nz; if (has) dN = H.dz[kk];
  }
  if (has) G = A / (dP / (2 * kp) + dN / (2 * H.k[pidx(H, ii, jj, kk)]));
  else if (H.bc == 0 || (ax == 0 && !hi)) G = 2 * kp * A / dP;
  else G = 0.0;
  F = (hi ? u : -u) * A;
}

// The operator rows, and (L0.gx non-null) level 0 of the multigrid
// hierarchy in its precision from the same face values: each cell's low-face
// conductance and + direction flux, the ghost past each high end carrying
// that boundary face (every other entry of the level-0 face arrays stays 0
// from the allocation).
template <class MT>
__global__ void __launch_bounds__(kB, 4) k_cht_assemble(ChtDev H, double Tb, mg::Level<MT> L0) {  // 64 registers
  const int PX = H.Nx + 2, PXY = (H.Nx + 2) * (H.Ny + 2);
  for (mg::Walk w(H.Nx, H.Ny, H.Nz, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x); w.ok(); w.next()) {
    const int i = w.m, j = w.j, k = w.k;
    const int q = pidx(H, i, j, k);
    double diag = 0.0, a[6], rhs = H.q[q] * H.dx[i] * H.dy[j] * H.dz[k];
    for (int d = 0; d < 6; ++d) {
      double G, F;
      bool has;
      face(H, i, j, k, d, G, F, has);
      diag += G + fmax(F, 0.0);
      a[d] = has ? G + fmax(-F, 0.0) : 0.0;
      if (!has) rhs += (G + fmax(-F, 0.0)) * Tb;
      if (L0.gx) {
        MT *g = d < 2 ? L0.gx : d < 4 ? L0.gy : L0.gz, *f = d < 2 ? L0.fx : d < 4 ? L0.fy : L0.fz;
        const int st = d < 2 ? 1 : d < 4 ? PX : PXY;
        const bool last = d == 1 ? i == H.Nx - 1 : d == 3 ? j == H.Ny - 1 : k == H.Nz - 1;
        if (!(d & 1)) { g[q] = (MT)G; f[q] = (MT)(-F); }
        else if (last) { g[q + st] = (MT)G; f[q + st] = (MT)F; }
      }
    }
    H.d[q] = diag; H.dinv[q] = 1.0 / diag;
    H.aw[q] = a[0]; H.ae[q] = a[1]; H.as[q] = a[2]; H.an[q] = a[3]; H.ab[q] = a[4]; H.af[q] = a[5];
    H.b[q] = rhs;
  }
}

// Krylov vectors (padded cells) in storage precision VT
template <class VT>
struct VecT {
  VT *x, *r, *rh, *p, *v, *ph, *s, *sh, *t;
};
using Vec = VecT<double>;

// Jacobi-preconditioned BiCGStab (van der Vorst, SIAM J. Sci. Stat. Comput.
// 13(2), 1992) for A x = rhs or A^T x = rhs; x holds the start.

// y = A x (transpose = 0) or A^T x at padded q, x in any precision
template <class XT>
__device__ __forceinline__ double apply_any(const ChtDev &H, const XT *x, int q, int PX, int PXY, bool tr) {
  const double off = tr ? H.ae[q - 1] * (double)__ldcg(x + q - 1) + H.aw[q + 1] * (double)__ldcg(x + q + 1) +
                              H.an[q - PX] * (double)__ldcg(x + q - PX) + H.as[q + PX] * (double)__ldcg(x + q + PX) +
                              H.af[q - PXY] * (double)__ldcg(x + q - PXY) + H.ab[q + PXY] * (double)__ldcg(x + q + PXY)
                        : H.aw[q] * (double)__ldcg(x + q - 1) + H.ae[q] * (double)__ldcg(x + q + 1) +
                              H.as[q] * (double)__ldcg(x + q - PX) + H.an[q] * (double)__ldcg(x + q + PX) +
                              H.ab[q] * (double)__ldcg(x + q - PXY) + H.af[q] * (double)__ldcg(x + q + PXY);
  return H.d[q] * (double)__ldcg(x + q) - off;
}

// Right-preconditioned BiCGStab (van der Vorst, SIAM J. Sci. Stat. Comput.
// 13(2), 1992) for A x = rhs or A^T x = rhs; x holds the start.  The
// preconditioner is the V-cycle of hs_mg.cuh on the same operator (Gm.L > 0)
// or Jacobi.  With the V-cycle, the products A p^ and A s^ read the cycle's
// output directly and store p^, s^ on the way; <r^, r> of the next iteration
// is summed with <r, r>.
// rel0: stop on ||r|| / ||r0|| instead of ||r|| / ||rhs||; out_r0 = ||r0||.
// Vectors stored in VT, arithmetic and dot products in FP64.  x0 (FP64,
// optional, FP32 vectors only): solve for the correction to x0 instead, from
// x = 0, with the first residual rhs - A x0 (and ||r0||) evaluated in FP64.
template <class MT, class VT>
__global__ void __launch_bounds__(kBiT, 1) k_cht_bicgstab(ChtDev H, VecT<VT> V, mg::Hier<MT> Gm, const double *rhs,
                                                        int transpose, double tol, int maxiter, double *partials,
                                                        int *out_it, double *out_rel, int rel0, double *out_r0,
                                                        const double *x0) {
  constexpr bool kFp64 = std::is_same<VT, double>::value;
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[48];
  const int Nx = H.Nx, Ny = H.Ny;
  const int PX = Nx + 2, PXY = (Nx + 2) * (Ny + 2);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  const bool tr = transpose != 0, mgp = Gm.L > 0;
  const MT *z = mgp ? Gm.lv[0].x : nullptr;
  int buf = 0;
  if (mgp) mg::build(Gm, tr, grid, tid, T);  // level 0 written by k_cht_assemble
  double red[2] = {0.0, 0.0};
  for (mg::Walk w(Nx, Ny, H.Nz, tid, T); w.ok(); w.next()) {
    const int q = (w.m + 1) + PX * ((w.j + 1) + (Ny + 2) * (w.k + 1));
    const double bq = rhs[q];
    double ax;
    if constexpr (kFp64) {
      ax = apply_any(H, V.x, q, PX, PXY, tr);
    } else {
      ax = x0 ? apply_any(H, x0, q, PX, PXY, tr) : apply_any(H, V.x, q, PX, PXY, tr);
      if (x0) V.x[q] = VT(0);
    }
    const double rv = bq - ax;
    V.r[q] = (VT)rv; V.rh[q] = (VT)rv; V.p[q] = VT(0); V.v[q] = VT(0);
    red[0] += bq * bq;
    red[1] += rv * rv;
  }
  grid_sums<2>(red, partials, buf, sh, grid);
  double bb = rel0 ? red[1] : red[0], rr = red[1];
  if (bb == 0) bb = 1.0;
  if (tid == 0 && out_r0) *out_r0 = sqrt(rr);
  const double eps = tol * tol;
  double rho = 1.0, alpha = 1.0, omega = 1.0, rho1 = red[1];
  int it = 0;
  while (it < maxiter && !(rr / bb < eps)) {
    it++;
    const double beta = (rho1 / rho) * (alpha / omega);
    // each pass issues every load of a cell before its first store
    for (mg::Walk w(Nx, Ny, H.Nz, tid, T); w.ok(); w.next()) {
      const int q = (w.m + 1) + PX * ((w.j + 1) + (Ny + 2) * (w.k + 1));
      const double r_ = (double)V.r[q], p_ = (double)V.p[q], v_ = (double)V.v[q];
      const mg::Seed<MT> sd = mgp ? mg::seed_at(Gm.lv[0], w.m, w.j, w.k, q, tr) : mg::Seed<MT>{};
      const double di = mgp ? 0.0 : H.dinv[q];
      const VT pv = (VT)(r_ + beta * (p_ - omega * v_));
      V.p[q] = pv;
      if (mgp) sd.store(Gm.lv[0], q, pv);
      else V.ph[q] = (VT)((double)pv * di);
    }
    grid.sync();
    if (mgp) mg::vcycle(Gm, tr, grid, tid, T);
    double s2[1] = {0.0};
    for (mg::Walk w(Nx, Ny, H.Nz, tid, T); w.ok(); w.next()) {
      const int q = (w.m + 1) + PX * ((w.j + 1) + (Ny + 2) * (w.k + 1));
      const double rh = (double)V.rh[q];
      const VT vv = (VT)(mgp ? apply_any(H, z, q, PX, PXY, tr) : apply_any(H, V.ph, q, PX, PXY, tr));
      if (mgp) V.ph[q] = (VT)__ldcg(z + q);
      V.v[q] = vv;
      s2[0] += rh * (double)vv;
    }
    grid_sums<1>(s2, partials, buf, sh, grid);
    alpha = rho1 / s2[0];
    double s3[1] = {0.0};
    for (mg::Walk w(Nx, Ny, H.Nz, tid, T); w.ok(); w.next()) {
      const int q = (w.m + 1) + PX * ((w.j + 1) + (Ny + 2) * (w.k + 1));
      const double r_ = (double)V.r[q], v_ = (double)V.v[q];
      const mg::Seed<MT> sd = mgp ? mg::seed_at(Gm.lv[0], w.m, w.j, w.k, q, tr) : mg::Seed<MT>{};
      const double di = mgp ? 0.0 : H.dinv[q];
      const VT sv = (VT)(r_ - alpha * v_);
      V.s[q] = sv;
      if (mgp) sd.store(Gm.lv[0], q, sv);
      else V.sh[q] = (VT)((double)sv * di);
      s3[0] += (double)sv * (double)sv;
    }
    grid_sums<1>(s3, partials, buf, sh, grid);
    if (s3[0] / bb < eps) {
      for (mg::Walk w(Nx, Ny, H.Nz, tid, T); w.ok(); w.next()) {
        const int q = (w.m + 1) + PX * ((w.j + 1) + (Ny + 2) * (w.k + 1));
        V.x[q] = (VT)((double)V.x[q] + alpha * (double)V.ph[q]);
      }
      rr = s3[0];
      break;
    }
    if (mgp) mg::vcycle(Gm, tr, grid, tid, T);
    double s4[2] = {0.0, 0.0};
    for (mg::Walk w(Nx, Ny, H.Nz, tid, T); w.ok(); w.next()) {
      const int q = (w.m + 1) + PX * ((w.j + 1) + (Ny + 2) * (w.k + 1));
      const double sq = (double)V.s[q];
      const VT tv = (VT)(mgp ? apply_any(H, z, q, PX, PXY, tr) : apply_any(H, V.sh, q, PX, PXY, tr));
      if (mgp) V.sh[q] = (VT)__ldcg(z + q);
      V.t[q] = tv;
      s4[0] += (double)tv * sq;
      s4[1] += (double)tv * (double)tv;
    }
    grid_sums<2>(s4, partials, buf, sh, grid);
    omega = s4[0] / s4[1];
    double s5[2] = {0.0, 0.0};
    for (mg::Walk w(Nx, Ny, H.Nz, tid, T); w.ok(); w.next()) {
      const int q = (w.m + 1) + PX * ((w.j + 1) + (Ny + 2) * (w.k + 1));
      const double x_ = (double)V.x[q], ph = (double)V.ph[q], sh_ = (double)V.sh[q], s_ = (double)V.s[q],
                   t_ = (double)V.t[q], rh = (double)V.rh[q];
      V.x[q] = (VT)(x_ + (alpha * ph + omega * sh_));
      const VT rv = (VT)(s_ - omega * t_);
      V.r[q] = rv;
      s5[0] += (double)rv * (double)rv;
      s5[1] += rh * (double)rv;
    }
    grid_sums<2>(s5, partials, buf, sh, grid);
    rr = s5[0];
    rho = rho1;
    rho1 = s5[1];
  }
  if (tid == 0) { *out_it = it; *out_rel = sqrt(rr / bb); }
}

// dJ/dT (into g) and the per-block sum of T^8 dV for J
__global__ void k_cht_objective(ChtDev H, const double *T, double *g, double *partial_sum8) {
  __shared__ double sh[48];
  const int n = H.Nx * H.Ny * H.Nz;
  double acc = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % H.Nx, j = (c / H.Nx) % H.Ny, k = c / (H.Nx * H.Ny);
    const int q = pidx(H, i, j, k);
    if (!H.solid[q]) continue;
    const double t = T[q], t2 = t * t, t4 = t2 * t2;
    acc += t4 * t4 * H.dx[i] * H.dy[j] * H.dz[k];
  }
  double b = blk_sum(acc, sh);
  if (threadIdx.x == 0) partial_sum8[blockIdx.x] = b;
  (void)g;
}

__global__ void k_cht_djdt(ChtDev H, const double *T, double f, double *g) {
  const int n = H.Nx * H.Ny * H.Nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % H.Nx, j = (c / H.Nx) % H.Ny, k = c / (H.Nx * H.Ny);
    const int q = pidx(H, i, j, k);
    if (!H.solid[q]) { g[q] = 0.0; continue; }
    const double t = T[q], t2 = t * t, t3 = t2 * t, t7 = t3 * t3 * t;
    g[q] = f * t7 * H.dx[i] * H.dy[j] * H.dz[k];
  }
}

// per-cell pieces of the gradients: dJ/dq_P = lam_P V_P and the cell's share
// of dJ/dk (sum over its faces of -dG/dk_P (lam_P - lam_N)(T_P - T_N))
__global__ void k_cht_grad(ChtDev H, const double *T, const double *lam, double Tb, double *dJdq, double *dk_cell) {
  const int n = H.Nx * H.Ny * H.Nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % H.Nx, j = (c / H.Nx) % H.Ny, k = c / (H.Nx * H.Ny);
    const int q = pidx(H, i, j, k);
    if (!H.solid[q]) { dJdq[c] = 0.0; dk_cell[c] = 0.0; continue; }
    const double dx = H.dx[i], dy = H.dy[j], dz = H.dz[k], kp = H.k[q];
    dJdq[c] = lam[q] * dx * dy * dz;
    double acc = 0.0;
    for (int d = 0; d < 6; ++d) {
      double G, F;
      bool has;
      face(H, i, j, k, d, G, F, has);
      const int ax = d >> 1;
      const double A = ax == 0 ? dy * dz : ax == 1 ? dx * dz : dx * dy, dP = ax == 0 ? dx : ax == 1 ? dy : dz;
      const double dG = has ? G * G * dP / (2 * A * kp * kp) : G / kp;
      int qn = q;
      if (d == 0) qn = q - 1; else if (d == 1) qn = q + 1;
      else if (d == 2) qn = q - (H.Nx + 2); else if (d == 3) qn = q + (H.Nx + 2);
      else if (d == 4) qn = q - (H.Nx + 2) * (H.Ny + 2); else qn = q + (H.Nx + 2) * (H.Ny + 2);
      const double tn = has ? T[qn] : Tb, ln = has ? lam[qn] : 0.0;
      acc -= dG * (lam[q] - ln) * (T[q] - tn);
    }
    dk_cell[c] = acc;
  }
}

// face velocities of the global grid from the fluid box's u*, v*, w*; faces
// outside the fluid box or touching a solid cell carry no flow
__global__ void k_cht_velocities(ChtVelSrc S, double *ug, double *vg, double *wg) {
  const int Nx = S.Nx, Ny = S.Ny, Nz = S.Nz;
  const long long nu = (long long)(Nx + 1) * Ny * Nz, nv = (long long)Nx * (Ny + 1) * Nz, nw = (long long)Nx * Ny * (Nz + 1);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nu + nv + nw; e += (long long)gridDim.x * blockDim.x) {
    int dir, i, j, k;
    if (e < nu) { dir = 0; i = e % (Nx + 1); j = (e / (Nx + 1)) % Ny; k = e / ((long long)(Nx + 1) * Ny); }
    else if (e < nu + nv) { long long f = e - nu; dir = 1; i = f % Nx; j = (f / Nx) % (Ny + 1); k = f / ((long long)Nx * (Ny + 1)); }
    else { long long f = e - nu - nv; dir = 2; i = f % Nx; j = (f / Nx) % Ny; k = f / ((long long)Nx * Ny); }
    // the two cells the face separates (0-based global); -1 outside
    int ia = i, ja = j, ka = k;
    if (dir == 0) ia = i - 1; else if (dir == 1) ja = j - 1; else ka = k - 1;
    auto is_solid = [&](int a, int b, int c) {
      if (a < 0 || b < 0 || c < 0 || a >= Nx || b >= Ny || c >= Nz) return false;
      return S.ctype[a + Nx * (b + Ny * c)] != 0;
    };
    double val = 0.0;
    if (!is_solid(ia, ja, ka) && !is_solid(i, j, k)) {
      // local face index in the fluid box (1-based offsets)
      const int li = i - (S.ox - 1), lj = j - (S.oy - 1), lk = k - (S.oz - 1);
      if (dir == 0 && li >= 0 && li < S.fx && lj >= 0 && lj < S.cy && lk >= 0 && lk < S.cz)
        val = S.u[(li + 1) + (S.fx + 2) * ((lj + 1) + (S.cy + 2) * (lk + 1))];
      else if (dir == 1 && li >= 0 && li < S.cx && lj >= 0 && lj < S.fy && lk >= 0 && lk < S.cz)
        val = S.v[(li + 1) + (S.cx + 2) * ((lj + 1) + (S.fy + 2) * (lk + 1))];
      else if (dir == 2 && li >= 0 && li < S.cx && lj >= 0 && lj < S.cy && lk >= 0 && lk < S.fz)
        val = S.w[(li + 1) + (S.cx + 2) * ((lj + 1) + (S.cy + 2) * (lk + 1))];
    }
    if (dir == 0) ug[e] = val; else if (dir == 1) vg[e - nu] = val; else wg[e - nu - nv] = val;
  }
}

// T = T + a (x - T) on the interior of padded arrays
__global__ void k_cht_relax(int n, int Nx, int Ny, double a, const double *x, double *T) {
  for (mg::Walk w(Nx, Ny, n / (Nx * Ny), blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x); w.ok(); w.next()) {
    const int q = (w.m + 1) + (Nx + 2) * ((w.j + 1) + (Ny + 2) * (w.k + 1));
    T[q] = T[q] + a * (x[q] - T[q]);
  }
}

// T = T + a d on the interior of padded arrays
__global__ void k_cht_relax_correction(int n, int Nx, int Ny, double a, const float *d, double *T) {
  for (mg::Walk w(Nx, Ny, n / (Nx * Ny), blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x); w.ok(); w.next()) {
    const int q = (w.m + 1) + (Nx + 2) * ((w.j + 1) + (Ny + 2) * (w.k + 1));
    T[q] = T[q] + a * (double)d[q];
  }
}

// T = v on the interior
__global__ void k_cht_fill(int n, int Nx, int Ny, double v, double *T) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int q = (c % Nx + 1) + (Nx + 2) * ((c / Nx) % Ny + 1 + (Ny + 2) * (c / (Nx * Ny) + 1));
    T[q] = v;
  }
}
int coop_grid(const void *kernel, int device) {
  int nsm = 0, per = 0;
  HC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  // the V-cycle's staging of block 0's levels: up to kMgStageTotal bytes per launch
  HC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mg::kMgStageTotal));
  HC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kBiT, mg::kMgStageTotal));
  if (per < 1) throw std::runtime_error("cooperative kernel cannot be resident");
  return per * nsm;
}

int gfor(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + kB - 1) / kB, 148LL * 16)); }

}  // namespace

struct ChtState {
  int device;
  cudaStream_t stream;
  ChtDev H{};
  Vec V{};
  double Tb, tol;
  int maxiter, grid, nreg;
  int asm_grid = 1;  // k_cht_assemble's blocks
  std::vector<void *> allocs;
  double *T = nullptr, *lam = nullptr, *g = nullptr, *partials = nullptr, *res = nullptr;
  double *ug = nullptr, *vg = nullptr, *wg = nullptr, *dJdq = nullptr, *dkc = nullptr;
  double *kp = nullptr, *qp = nullptr;
  uint8_t *solid = nullptr, *ctype_dev = nullptr;
  int *it = nullptr;
  std::vector<int> region;      // per global cell (-1 fluid)
  std::vector<uint8_t> ctype;
  double J = 0;
  bool have_T = false;
  int precond = 0;              // 0 Jacobi, 1 V-cycle FP32, 2 V-cycle FP64
  bool step_fp32 = false;       // energy steps in correction form with FP32 vectors (Vf)
  VecT<float> Vf{};             // laid over the storage of V (not used at the same time)
  mg::Hier<float> Gf{};
  mg::Hier<double> Gd{};
  template <class T_>
  T_ *alloc(size_t n) {
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T_));
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA alloc: ") + cudaGetErrorString(e));
    allocs.push_back(p);
    HC_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T_), stream));
    return (T_ *)p;
  }
  ~ChtState() {
    for (void *p : allocs) cudaFree(p);
  }
};

namespace {
template <class MT>
void setup_levels(ChtState &C, mg::Hier<MT> &G) {
  int nx = C.H.Nx, ny = C.H.Ny, nz = C.H.Nz, L = 0;
  while (true) {
    if (L >= mg::kMgMaxLv) throw std::runtime_error("multigrid: too many levels");
    mg::Level<MT> &l = G.lv[L];
    l.nx = nx; l.ny = ny; l.nz = nz; l.px = nx + 2;
    const size_t np = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    l.x = C.alloc<MT>(np); l.rhs = C.alloc<MT>(np);
    l.gx = C.alloc<MT>(np); l.gy = C.alloc<MT>(np); l.gz = C.alloc<MT>(np);
    l.fx = C.alloc<MT>(np); l.fy = C.alloc<MT>(np); l.fz = C.alloc<MT>(np);
    l.m = nullptr;
    ++L;
    if ((long long)nx * ny * nz <= mg::kMgCoarse) break;
    nx = (nx + 1) / 2; ny = (ny + 1) / 2; nz = (nz + 1) / 2;
  }
  G.L = L;
  G.lu = C.alloc<double>((size_t)mg::kMgCoarse * mg::kMgCoarse);
  mg::plan_stage(G, false);  // the V-cycles of the energy solves keep their read-only arrays in global memory
}
}  // namespace

ChtState *cht_create(const ChtSetup &S) {
  HC_CUDA(cudaSetDevice(S.device));
  std::unique_ptr<ChtState> C(new ChtState());
  C->device = S.device;
  C->stream = (cudaStream_t)S.stream;
  C->Tb = S.t_boundary; C->tol = S.tol; C->maxiter = S.maxiter; C->nreg = S.nreg;
  ChtDev &H = C->H;
  H.bc = S.bc;
  H.Nx = S.Nx; H.Ny = S.Ny; H.Nz = S.Nz;
  const size_t np = (size_t)(S.Nx + 2) * (S.Ny + 2) * (S.Nz + 2), n = (size_t)S.Nx * S.Ny * S.Nz;
  auto up = [&](const std::vector<double> &v) {
    double *p = C->alloc<double>(v.size());
    HC_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * 8, cudaMemcpyHostToDevice, C->stream));
    return p;
  };
  std::vector<double> dx(S.Nx), dy(S.Ny), dz(S.Nz);
  for (int i = 0; i < S.Nx; ++i) dx[i] = S.xs[i + 1] - S.xs[i];
  for (int j = 0; j < S.Ny; ++j) dy[j] = S.ys[j + 1] - S.ys[j];
  for (int k = 0; k < S.Nz; ++k) dz[k] = S.zs[k + 1] - S.zs[k];
  H.dx = up(dx); H.dy = up(dy); H.dz = up(dz);
  C->ctype.assign(S.ctype, S.ctype + n);
  C->region.assign(S.region, S.region + n);
  std::vector<uint8_t> solid(np, 0);
  for (int k = 0; k < S.Nz; ++k)
    for (int j = 0; j < S.Ny; ++j)
      for (int i = 0; i < S.Nx; ++i)
        solid[(i + 1) + (S.Nx + 2) * ((j + 1) + (S.Ny + 2) * (k + 1))] = S.ctype[i + S.Nx * (j + S.Ny * k)];
  C->ctype_dev = C->alloc<uint8_t>(n);
  HC_CUDA(cudaMemcpyAsync(C->ctype_dev, S.ctype, n, cudaMemcpyHostToDevice, C->stream));
  C->solid = C->alloc<uint8_t>(np);
  HC_CUDA(cudaMemcpyAsync(C->solid, solid.data(), np, cudaMemcpyHostToDevice, C->stream));
  H.solid = C->solid;
  C->kp = C->alloc<double>(np); C->qp = C->alloc<double>(np);
  H.k = C->kp; H.q = C->qp;
  C->ug = C->alloc<double>((size_t)(S.Nx + 1) * S.Ny * S.Nz);
  C->vg = C->alloc<double>((size_t)S.Nx * (S.Ny + 1) * S.Nz);
  C->wg = C->alloc<double>((size_t)S.Nx * S.Ny * (S.Nz + 1));
  H.ug = C->ug; H.vg = C->vg; H.wg = C->wg;
  double **coef[] = {&H.d, &H.aw, &H.ae, &H.as, &H.an, &H.ab, &H.af, &H.b, &H.dinv};
  for (double **c : coef) *c = C->alloc<double>(np);
  double **vec[] = {&C->V.x, &C->V.r, &C->V.rh, &C->V.p, &C->V.v, &C->V.ph, &C->V.s, &C->V.sh, &C->V.t};
  for (double **v : vec) *v = C->alloc<double>(np);
  C->T = C->alloc<double>(np); C->lam = C->alloc<double>(np); C->g = C->alloc<double>(np);
  C->dJdq = C->alloc<double>(n); C->dkc = C->alloc<double>(n);
  C->precond = S.precond;
  if (S.precond == 1) setup_levels(*C, C->Gf);
  if (S.precond == 2) setup_levels(*C, C->Gd);
  C->step_fp32 = S.step_fp32 != 0;
  if (C->step_fp32) {
    // nine FP32 vectors in the first five FP64 ones (2 x np floats each)
    float *base[] = {(float *)C->V.x, (float *)C->V.r, (float *)C->V.rh, (float *)C->V.p, (float *)C->V.v};
    float **vf[] = {&C->Vf.x, &C->Vf.r, &C->Vf.rh, &C->Vf.p, &C->Vf.v, &C->Vf.ph, &C->Vf.s, &C->Vf.sh, &C->Vf.t};
    for (int a = 0; a < 9; ++a) *vf[a] = base[a / 2] + (a % 2) * np;
  }
  C->grid = std::min({coop_grid((const void *)k_cht_bicgstab<float, double>, S.device),
                      coop_grid((const void *)k_cht_bicgstab<double, double>, S.device),
                      coop_grid((const void *)k_cht_bicgstab<float, float>, S.device)});
  {
    // the assembly: a grid resident at once (every instantiation holds four
    // blocks per SM by its launch bounds; against 148 x 16 blocks the energy
    // step took 1.500 -> 1.487 ms FP64, 1.075 -> 1.063 ms mixed at 256x128x128)
    int nsm = 0, per = 0;
    HC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, S.device));
    HC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_cht_assemble<double>, kB, 0));
    C->asm_grid = std::min(gfor((long long)S.Nx * S.Ny * S.Nz), std::max(1, per * nsm));
  }
  C->partials = C->alloc<double>((size_t)2 * C->grid * 2 + 4096);
  C->res = C->alloc<double>(2); C->it = C->alloc<int>(1);
  HC_CUDA(cudaStreamSynchronize(C->stream));
  return C.release();
}

void cht_destroy(ChtState *C) {
  if (!C) return;
  cudaSetDevice(C->device);
  cudaStreamSynchronize(C->stream);
  delete C;
}

void cht_set_solid(ChtState *C, double k_fluid, const double *k_region, const double *q_cell) {
  HC_CUDA(cudaSetDevice(C->device));
  const ChtDev &H = C->H;
  const size_t np = (size_t)(H.Nx + 2) * (H.Ny + 2) * (H.Nz + 2);
  std::vector<double> k(np, 0.0), q(np, 0.0);
  for (int kk = 0; kk < H.Nz; ++kk)
    for (int j = 0; j < H.Ny; ++j)
      for (int i = 0; i < H.Nx; ++i) {
        const size_t c = i + (size_t)H.Nx * (j + (size_t)H.Ny * kk);
        const size_t p = (i + 1) + (H.Nx + 2) * ((j + 1) + (size_t)(H.Ny + 2) * (kk + 1));
        if (C->ctype[c]) {
          const int r = C->region[c];
          if (r < 0 || r >= C->nreg) throw std::invalid_argument("solid cell without a region");
          if (!(k_region[r] > 0)) throw std::invalid_argument("solid conductivity must be positive");
          k[p] = k_region[r];
          q[p] = q_cell ? q_cell[c] : 0.0;
        } else {
          k[p] = k_fluid;
        }
      }
  HC_CUDA(cudaMemcpyAsync(C->kp, k.data(), np * 8, cudaMemcpyHostToDevice, C->stream));
  HC_CUDA(cudaMemcpyAsync(C->qp, q.data(), np * 8, cudaMemcpyHostToDevice, C->stream));
  HC_CUDA(cudaStreamSynchronize(C->stream));
}

void cht_set_velocities(ChtState *C, const ChtVelSrc &src) {
  HC_CUDA(cudaSetDevice(C->device));
  const ChtDev &H = C->H;
  long long nf = (long long)(H.Nx + 1) * H.Ny * H.Nz + (long long)H.Nx * (H.Ny + 1) * H.Nz + (long long)H.Nx * H.Ny * (H.Nz + 1);
  ChtVelSrc S = src;
  S.ctype = C->ctype_dev;
  k_cht_velocities<<<gfor(nf), kB, 0, C->stream>>>(S, C->ug, C->vg, C->wg);
  HC_CUDA(cudaGetLastError());
}

void cht_get_velocities(ChtState *C, double *ug, double *vg, double *wg) {
  const ChtDev &H = C->H;
  HC_CUDA(cudaMemcpyAsync(ug, C->ug, (size_t)(H.Nx + 1) * H.Ny * H.Nz * 8, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaMemcpyAsync(vg, C->vg, (size_t)H.Nx * (H.Ny + 1) * H.Nz * 8, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaMemcpyAsync(wg, C->wg, (size_t)H.Nx * H.Ny * (H.Nz + 1) * 8, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaStreamSynchronize(C->stream));
}

namespace {
template <class K, class... A>
void launch_coop(K kernel, int blocks, size_t smem, cudaStream_t s, A... args) {
  void *argv[] = {(void *)&args...};
  HC_CUDA(cudaLaunchCooperativeKernel((void *)kernel, dim3(blocks), dim3(kBiT), argv, smem, s));
}

// operator rows and the fine level of the hierarchy in use (every solve is
// preceded by this, on the same stream)
void assemble(ChtState *C) {
  const int nb = C->asm_grid;
  if (C->precond == 2) k_cht_assemble<double><<<nb, kB, 0, C->stream>>>(C->H, C->Tb, C->Gd.lv[0]);
  else if (C->precond == 1) k_cht_assemble<float><<<nb, kB, 0, C->stream>>>(C->H, C->Tb, C->Gf.lv[0]);
  else k_cht_assemble<float><<<nb, kB, 0, C->stream>>>(C->H, C->Tb, mg::Level<float>{});
  HC_CUDA(cudaGetLastError());
}

void solve(ChtState *C, const double *rhs, int transpose, double tol, int maxiter, int rel0, double *out_r0) {
  const double *nox = nullptr;
  if (C->precond == 2)
    launch_coop(k_cht_bicgstab<double, double>, C->grid, C->Gd.stage, C->stream, C->H, C->V, C->Gd, rhs, transpose, tol, maxiter,
                C->partials, C->it, C->res, rel0, out_r0, nox);
  else {
    mg::Hier<float> G = C->Gf;
    if (C->precond == 0) G.L = 0;
    launch_coop(k_cht_bicgstab<float, double>, C->grid, G.stage, C->stream, C->H, C->V, G, rhs, transpose, tol, maxiter,
                C->partials, C->it, C->res, rel0, out_r0, nox);
  }
}

// A d = b - A T with d from 0 in FP32 vectors (V-cycle in FP32), stopping on
// ||r|| <= tol ||r0||; ||r0|| (FP64) into out_r0
void solve_correction(ChtState *C, double tol, int maxiter, double *out_r0) {
  mg::Hier<float> G = C->Gf;
  if (C->precond != 1) G.L = 0;
  const double *x0 = C->T;
  launch_coop(k_cht_bicgstab<float, float>, C->grid, G.stage, C->stream, C->H, C->Vf, G, (const double *)C->H.b, 0, tol,
              maxiter, C->partials, C->it, C->res, 1, out_r0, x0);
}

void unpad(const ChtDev &H, const double *dev, double *host, cudaStream_t s) {
  const size_t np = (size_t)(H.Nx + 2) * (H.Ny + 2) * (H.Nz + 2);
  std::vector<double> tmp(np);
  HC_CUDA(cudaMemcpyAsync(tmp.data(), dev, np * 8, cudaMemcpyDeviceToHost, s));
  HC_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k < H.Nz; ++k)
    for (int j = 0; j < H.Ny; ++j)
      for (int i = 0; i < H.Nx; ++i)
        host[i + (size_t)H.Nx * (j + (size_t)H.Ny * k)] = tmp[(i + 1) + (H.Nx + 2) * ((j + 1) + (size_t)(H.Ny + 2) * (k + 1))];
}

double objective(ChtState *C, bool grad) {
  const ChtDev &H = C->H;
  const int nb = gfor((long long)H.Nx * H.Ny * H.Nz);
  k_cht_objective<<<nb, kB, 0, C->stream>>>(H, C->T, C->g, C->partials);
  std::vector<double> part(nb);
  HC_CUDA(cudaMemcpyAsync(part.data(), C->partials, nb * 8, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaStreamSynchronize(C->stream));
  double s = 0;
  for (double v : part) s += v;
  const double J = std::pow(s, 1.0 / 8.0);
  if (grad) k_cht_djdt<<<nb, kB, 0, C->stream>>>(H, C->T, std::pow(J, -7.0), C->g);
  return J;
}
}  // namespace

void cht_forward(ChtState *C, double *T_host, double *J, int *iters, double *relres) {
  HC_CUDA(cudaSetDevice(C->device));
  const ChtDev &H = C->H;
  const size_t np = (size_t)(H.Nx + 2) * (H.Ny + 2) * (H.Nz + 2);
  assemble(C);
  k_cht_fill<<<gfor((long long)H.Nx * H.Ny * H.Nz), kB, 0, C->stream>>>(H.Nx * H.Ny * H.Nz, H.Nx, H.Ny, C->Tb, C->V.x);
  solve(C, H.b, 0, C->tol, C->maxiter, 0, nullptr);
  HC_CUDA(cudaMemcpyAsync(C->T, C->V.x, np * 8, cudaMemcpyDeviceToDevice, C->stream));
  int it = 0;
  double rr = 0;
  HC_CUDA(cudaMemcpyAsync(&it, C->it, 4, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaMemcpyAsync(&rr, C->res, 8, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaStreamSynchronize(C->stream));
  C->J = objective(C, false);
  C->have_T = true;
  if (T_host) unpad(H, C->T, T_host, C->stream);
  if (J) *J = C->J;
  if (iters) *iters = it;
  if (relres) *relres = rr;
}

void cht_adjoint(ChtState *C, double *dJdq_host, double *dJdk_host, int *iters, double *relres, void *device_done) {
  HC_CUDA(cudaSetDevice(C->device));
  if (!C->have_T) throw std::logic_error("adjoint before forward solve");
  const ChtDev &H = C->H;
  const size_t np = (size_t)(H.Nx + 2) * (H.Ny + 2) * (H.Nz + 2);
  const long long n = (long long)H.Nx * H.Ny * H.Nz;
  objective(C, true);
  HC_CUDA(cudaMemsetAsync(C->V.x, 0, np * 8, C->stream));
  solve(C, C->g, 1, C->tol, C->maxiter, 0, nullptr);
  HC_CUDA(cudaMemcpyAsync(C->lam, C->V.x, np * 8, cudaMemcpyDeviceToDevice, C->stream));
  k_cht_grad<<<gfor(n), kB, 0, C->stream>>>(H, C->T, C->lam, C->Tb, C->dJdq, C->dkc);
  if (device_done) HC_CUDA(cudaEventRecord((cudaEvent_t)device_done, C->stream));
  std::vector<double> dq(n), dk(n);
  int it = 0;
  double rr = 0;
  HC_CUDA(cudaMemcpyAsync(dq.data(), C->dJdq, n * 8, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaMemcpyAsync(dk.data(), C->dkc, n * 8, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaMemcpyAsync(&it, C->it, 4, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaMemcpyAsync(&rr, C->res, 8, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaStreamSynchronize(C->stream));
  if (dJdq_host) std::copy(dq.begin(), dq.end(), dJdq_host);
  if (dJdk_host) {
    for (int r = 0; r < C->nreg; ++r) dJdk_host[r] = 0.0;
    for (long long c = 0; c < n; ++c)
      if (C->ctype[c]) dJdk_host[C->region[c]] += dk[c];
  }
  if (iters) *iters = it;
  if (relres) *relres = rr;
}

void cht_bind_velocities(ChtState *C, const double *ug, const double *vg, const double *wg) {
  C->H.ug = ug; C->H.vg = vg; C->H.wg = wg;
}

void cht_fill_T(ChtState *C, double v) {
  HC_CUDA(cudaSetDevice(C->device));
  const ChtDev &H = C->H;
  const int n = H.Nx * H.Ny * H.Nz;
  k_cht_fill<<<gfor(n), kB, 0, C->stream>>>(n, H.Nx, H.Ny, v, C->T);
  HC_CUDA(cudaGetLastError());
  C->have_T = false;
}

double *cht_T_device(ChtState *C) { return C->T; }

namespace {
// Global balances of the channel form (bc = 1) in FP64, by one block in a
// fixed order: out = {volume flux in through x = 0, out through x = Nx,
// sum of q V, heat leaving through the boundary}.  A boundary face with
// outward flux F and conductance G_b carries G_b (T_P - Tb) + max(F, 0) T_P
// - max(-F, 0) Tb out of the domain (the energy operator's boundary terms):
// at x = 0, G_b = 2 k_P A / dx_P and F = -u A; at x = Nx, G_b = 0 and
// F = u A; the walls carry nothing.
__global__ void k_cht_balance(ChtDev H, const double *T, double Tb, double *out) {
  __shared__ double sh[32];
  const int Nx = H.Nx, Ny = H.Ny, Nz = H.Nz;
  double in = 0.0, outf = 0.0, src = 0.0, heat = 0.0;
  for (int e = threadIdx.x; e < Ny * Nz; e += blockDim.x) {
    const int j = e % Ny, k = e / Ny;
    const double A = H.dy[j] * H.dz[k];
    const double u0 = H.ug[0 + (Nx + 1) * (j + Ny * k)], u1 = H.ug[Nx + (Nx + 1) * (j + Ny * k)];
    in += u0 * A;
    outf += u1 * A;
    const int p0 = pidx(H, 0, j, k), p1 = pidx(H, Nx - 1, j, k);
    const double T0 = T[p0], T1 = T[p1];
    const double G0 = 2.0 * H.k[p0] * A / H.dx[0], F0 = -u0 * A, F1 = u1 * A;
    heat += G0 * (T0 - Tb) + (F0 > 0.0 ? F0 * T0 : F0 * Tb);
    heat += F1 > 0.0 ? F1 * T1 : F1 * Tb;
  }
  for (int e = threadIdx.x; e < Nx * Ny * Nz; e += blockDim.x) {
    const int i = e % Nx, j = (e / Nx) % Ny, k = e / (Nx * Ny);
    src += H.q[pidx(H, i, j, k)] * (H.dx[i] * H.dy[j] * H.dz[k]);
  }
  in = blk_sum(in, sh);
  outf = blk_sum(outf, sh);
  src = blk_sum(src, sh);
  heat = blk_sum(heat, sh);
  if (threadIdx.x == 0) { out[0] = in; out[1] = outf; out[2] = src; out[3] = heat; }
}
}  // namespace

void cht_balance(ChtState *C, double out4[4]) {
  HC_CUDA(cudaSetDevice(C->device));
  double *d = nullptr;
  HC_CUDA(cudaMallocAsync((void **)&d, 4 * sizeof(double), C->stream));
  k_cht_balance<<<1, 1024, 0, C->stream>>>(C->H, C->T, C->Tb, d);
  HC_CUDA(cudaGetLastError());
  HC_CUDA(cudaMemcpyAsync(out4, d, 4 * sizeof(double), cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaFreeAsync(d, C->stream));
  HC_CUDA(cudaStreamSynchronize(C->stream));
}

void cht_energy_step(ChtState *C, double alpha_t, double tol, int maxiter) {
  const ChtDev &H = C->H;
  const int n = H.Nx * H.Ny * H.Nz;
  const size_t np = (size_t)(H.Nx + 2) * (H.Ny + 2) * (H.Nz + 2);
  assemble(C);
  if (C->step_fp32) {
    solve_correction(C, tol, maxiter, C->res + 1);
    k_cht_relax_correction<<<gfor(n), kB, 0, C->stream>>>(n, H.Nx, H.Ny, alpha_t, (const float *)C->Vf.x, C->T);
  } else {
    HC_CUDA(cudaMemcpyAsync(C->V.x, C->T, np * 8, cudaMemcpyDeviceToDevice, C->stream));
    solve(C, H.b, 0, tol, maxiter, 1, C->res + 1);
    k_cht_relax<<<gfor(n), kB, 0, C->stream>>>(n, H.Nx, H.Ny, alpha_t, (const double *)C->V.x, C->T);
  }
  HC_CUDA(cudaGetLastError());
  C->have_T = false;
}

void cht_step_results(ChtState *C, int *iters, double *relres, double *r0) {
  double rr[2];
  int it = 0;
  HC_CUDA(cudaMemcpyAsync(&it, C->it, 4, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaMemcpyAsync(rr, C->res, 16, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaStreamSynchronize(C->stream));
  if (iters) *iters = it;
  if (relres) *relres = rr[0];
  if (r0) *r0 = rr[1];
}

void cht_step_results_async(ChtState *C, int *iters, double *relres_r0) {
  HC_CUDA(cudaMemcpyAsync(iters, C->it, 4, cudaMemcpyDeviceToHost, C->stream));
  HC_CUDA(cudaMemcpyAsync(relres_r0, C->res, 16, cudaMemcpyDeviceToHost, C->stream));
}

void cht_set_tolerance(ChtState *C, double tol, int maxiter) { C->tol = tol; C->maxiter = maxiter; }

}  // namespace hs
