// sm_100a kernels and host orchestration of one SIMPLE-CHT outer step.
//
// Gauss-Seidel sweeps.  The reference sweeps every equation in place in
// lexicographic order (k outer, j, i inner; fluid_solver.h:419-421,
// 505-507, 588-590, 807-809; mobs_solver.h:477-479).  With a 7-point
// dependency, cell (i,j,k) reads new values at (i-1,j,k), (i,j-1,k),
// (i,j,k-1) and old values at (i+1,j,k), (i,j+1,k), (i,j,k+1).  Cells on
// the hyperplane i+j+k = s therefore depend only on hyperplane s-1, so the
// sweep runs as a wavefront: one cooperative kernel per solve, one grid-wide
// barrier per hyperplane, one thread per (j,k) row.  Every point update uses
// the reference's arithmetic in the reference's operation order (the build
// disables FMA contraction), so the sweep is the reference's sweep, not an
// approximation of it.
//
// Pressure correction.  Matrix-free CG over the fluid cells with HYPRE
// PCG's recurrences and stopping rule (identity preconditioner, two-norm,
// tol 1e-5, maxiter 1000, zero start; fluid_solver.h:1871-1875), run as one
// cooperative kernel with two grid reductions per iteration.  The direction
// update p = r + beta p is fused into the next SpMV (double-buffered p), and
// x += alpha p is deferred into the same pass, so an iteration streams
// r, p, x, 3 coefficients and writes p, s, x, then streams r, s and writes r.
//
// Reductions are deterministic: per-block partials, then every block sums
// the partials in the same fixed order.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "hs_engine.hpp"

namespace cg = cooperative_groups;

namespace hs {

#define HS_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_) + \
                                                    " at " #call);                                 \
  } while (0)

constexpr int kBlock = 256;

// ---------------------------------------------------------------- views
struct Prm {
  double nu, rho, alpha, u_lid, relax, relax_solid, mom_tol, energy_tol, solid_tol, t_wall, t_solid0, pcg_tol;
  int gs_max, pcg_maxiter;
};

struct FluidDev {
  int cx, cy, cz, fx, fy, fz, ox, oy, oz;
  int Nx, Ny, Nz;
  double *u, *v, *w, *up, *vp, *wp, *pt, *tt;  // padded
  double *pc, *tc, *ux, *uy, *uz;              // LocalCell / LocalFace values
  const uint8_t *empty;                        // cx*cy*cz
  const double *xp, *xw, *xe, *yp, *ys, *yn, *zp, *zf, *zb;
  // 1/s/s per axis index with s = (p + m)/2 (fluid_solver.h:831-842), so the
  // energy denominator 2*alpha*(1/sx/sx + 1/sy/sy + 1/sz/sz) costs no division
  const double *ix2, *iy2, *iz2;
  // RN(1/s) of the energy spacings s = (p + m)/2 per axis index
  const double *rsx, *rsy, *rsz;
  // RN(1/(p+m)) and RN(1/(p+q)) of the momentum diffusion distances per axis
  // index: xp+xw, xp+xe | ys+yp, yn+yp | zb+zp, zf+zp (fluid_solver.h:1266-1268)
  const double *rxw, *rxe, *rys, *ryn, *rzb, *rzf;
  // parity-split copies used inside the energy solve: cell (i,j,k) of the
  // padded grid at (i&1)*hs + (i>>1) + hx*(j + (cy+2)*k), so the cells of one
  // parity that a time step updates are contiguous
  double *ts, *us, *vs, *ws;
  int hx;
  long long hs;
  double *acx, *acy, *acz;                     // padded, frozen pressure-correction coefficients
  double *x, *r, *pa, *pb, *s;                 // padded CG vectors; x is p'
  double *pscr;                                // cx*cy*cz scratch for the cell BC
};

struct SolidReg {
  int cx, cy, cz, rows, blk0, nblk;
  long long tt_off, tc_off, em_off;
};

struct DevStats {
  int sweeps[4];      // u v w t
  double res[4];
  int pcg_iters;
  double pcg_relres;
  int solid_sweeps_max;
  int pad;
  // running totals since creation (bench byte accounting)
  long long cum_sweeps[4];
  long long cum_solid_cell_sweeps;
  long long cum_pcg_iters;
  long long cum_pcg_solves;
};

__device__ __forceinline__ int IU(const FluidDev &F, int i, int j, int k) { return i + (F.fx + 2) * (j + (F.cy + 2) * k); }
__device__ __forceinline__ int IV(const FluidDev &F, int i, int j, int k) { return i + (F.cx + 2) * (j + (F.fy + 2) * k); }
__device__ __forceinline__ int IW(const FluidDev &F, int i, int j, int k) { return i + (F.cx + 2) * (j + (F.cy + 2) * k); }
__device__ __forceinline__ int IP(const FluidDev &F, int i, int j, int k) { return i + (F.cx + 2) * (j + (F.cy + 2) * k); }
__device__ __forceinline__ int GC(const FluidDev &F, int i, int j, int k) { return i + F.cx * (j + F.cy * k); }
__device__ __forceinline__ int GX(const FluidDev &F, int i, int j, int k) { return i + F.fx * (j + F.cy * k); }
__device__ __forceinline__ int GY(const FluidDev &F, int i, int j, int k) { return i + F.cx * (j + F.fy * k); }
__device__ __forceinline__ int GZ(const FluidDev &F, int i, int j, int k) { return i + F.cx * (j + F.cy * k); }

__device__ __forceinline__ double dmax0(double a) { return a < 0.0 ? 0.0 : a; }  // std::max(a, 0.0)

// a / b for a divisor known ahead of time, from its correctly rounded
// reciprocal y = RN(1/b) (Markstein, IBM J. Res. Dev. 34(1), 1990): q = RN(a*y)
// is within one ulp of a/b, the remainder a - q*b is exact in one FMA, and
// RN(q + r*y) is the correctly rounded quotient RN(a/b) -- the same value the
// IEEE division gives, for finite, normal operands and a nonzero a.
__device__ __forceinline__ double div_pre(double a, double b, double y) {
  const double q = a * y;
  const double r = __fma_rn(-q, b, a);
  return __fma_rn(r, y, q);
}
__device__ __forceinline__ double ld(const double *p) { return __ldcg(p); }   // L2-coherent load

// ---------------------------------------------------------------- reductions
__device__ double block_sum(double v, double *sh) {
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
  return t;  // valid in warp 0
}

// Sum over the whole grid; identical value in every thread of every block.
// `buf` alternates between two partial arrays so that consecutive reductions
// never overwrite partials another block may still be reading.
__device__ double grid_sum(double v, double *partials, int &buf, double *sh, cg::grid_group &grid) {
  double *pp = partials + buf * gridDim.x;
  buf ^= 1;
  double b = block_sum(v, sh);
  if (threadIdx.x == 0) pp[blockIdx.x] = b;
  grid.sync();
  if (threadIdx.x < 32) {
    double a = 0.0;
    for (int q = threadIdx.x; q < (int)gridDim.x; q += 32) a += __ldcg(pp + q);
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (threadIdx.x == 0) sh[32] = a;
  }
  __syncthreads();
  double r = sh[32];
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------- boundary conditions
// applyXBoundaryCondition (fluid_solver.h:209-254)
__device__ void bc_x(const FluidDev &F, int tid, int T) {
  const int cx = F.cx, cy = F.cy, cz = F.cz, fx = F.fx;
  if (F.ox == 1) {
    for (int e = tid; e < (cz + 2) * (cy + 2); e += T) {
      int j = e % (cy + 2), k = e / (cy + 2);
      F.u[IU(F, 0, j, k)] = 0; F.v[IV(F, 0, j, k)] = 0; F.w[IW(F, 0, j, k)] = 0;
    }
  } else if (F.ox - 1 + fx == F.Nx + 1) {
    for (int e = tid; e < (cz + 2) * (cy + 2); e += T) {
      int j = e % (cy + 2), k = e / (cy + 2);
      F.u[IU(F, fx + 1, j, k)] = 0; F.v[IV(F, cx + 1, j, k)] = 0; F.w[IW(F, cx + 1, j, k)] = 0;
    }
  }
  if (F.ox - 1 + fx - 1 == F.Nx)
    for (int e = tid; e < cz * cy; e += T) {
      int j = e % cy, k = e / cy;
      F.ux[GX(F, fx - 1, j, k)] = 0; F.u[IU(F, fx, j + 1, k + 1)] = 0;
    }
}
// applyYBoundaryCondition (fluid_solver.h:289-323)
__device__ void bc_y(const FluidDev &F, const Prm &P, int tid, int T) {
  const int cx = F.cx, cy = F.cy, cz = F.cz, fy = F.fy;
  if (F.oy == 1) {
    for (int e = tid; e < (cz + 2) * (cx + 2); e += T) {
      int i = e % (cx + 2), k = e / (cx + 2);
      F.u[IU(F, i, 0, k)] = 0; F.v[IV(F, i, 0, k)] = 0; F.w[IW(F, i, 0, k)] = 0;
    }
  } else if (F.oy - 1 + fy == F.Ny + 1) {
    for (int e = tid; e < (cz + 2) * (cx + 2); e += T) {
      int i = e % (cx + 2), k = e / (cx + 2);
      F.u[IU(F, i, cy + 1, k)] = P.u_lid; F.v[IV(F, i, fy + 1, k)] = 0; F.w[IW(F, i, cy + 1, k)] = 0;
    }
  }
  if (F.oy - 1 + fy - 1 == F.Ny)
    for (int e = tid; e < cz * cx; e += T) {
      int i = e % cx, k = e / cx;
      F.uy[GY(F, i, fy - 1, k)] = 0; F.v[IV(F, i + 1, fy, k + 1)] = 0;
      F.ux[GX(F, i, cy - 1, k)] = P.u_lid; F.u[IU(F, i + 1, cy, k + 1)] = P.u_lid;
    }
}
// applyZBoundaryCondition (fluid_solver.h:256-287)
__device__ void bc_z(const FluidDev &F, int tid, int T) {
  const int cx = F.cx, cy = F.cy, cz = F.cz, fz = F.fz;
  if (F.oz == 1) {
    for (int e = tid; e < (cy + 2) * (cx + 2); e += T) {
      int i = e % (cx + 2), j = e / (cx + 2);
      F.u[IU(F, i, j, 0)] = 0; F.v[IV(F, i, j, 0)] = 0; F.w[IW(F, i, j, 0)] = 0;
    }
  } else if (F.oz - 1 + fz == F.Nz + 1) {
    for (int e = tid; e < (cy + 2) * (cx + 2); e += T) {
      int i = e % (cx + 2), j = e / (cx + 2);
      F.u[IU(F, i, j, cz + 1)] = 0; F.v[IV(F, i, j, cz + 1)] = 0; F.w[IW(F, i, j, fz + 1)] = 0;
    }
  }
  if (F.oz - 1 + fz - 1 == F.Nz)
    for (int e = tid; e < cy * cx; e += T) {
      int i = e % cx, j = e / cx;
      F.uz[GZ(F, i, j, fz - 1)] = 0; F.w[IW(F, i + 1, j + 1, fz)] = 0;
    }
}

__global__ void k_bc(FluidDev F, Prm P, int which) {
  int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  if (which == 0) bc_x(F, tid, T);
  else if (which == 1) bc_y(F, P, tid, T);
  else bc_z(F, tid, T);
}

// ---------------------------------------------------------------- momentum point updates
// solveXmomentum body (fluid_solver.h:591-624)
__device__ __forceinline__ double upd_u(const FluidDev &F, const Prm &P, int i, int j, int k, double &ap, double &old) {
  const double *u = F.u, *v = F.v, *w = F.w;
  double xp = F.xp[i], xw = F.xw[i], xe = F.xe[i], yp = F.yp[j], ys = F.ys[j], yn = F.yn[j];
  double zp = F.zp[k], zf = F.zf[k], zb = F.zb[k];
  double facexy = xp * yp, facexz = xp * zp, faceyz = yp * zp;
  double Dw = div_pre(2 * P.nu * faceyz, xp + xw, F.rxw[i]), De = div_pre(2 * P.nu * faceyz, xp + xe, F.rxe[i]);
  double Ds = div_pre(2 * P.nu * facexz, ys + yp, F.rys[j]), Dn = div_pre(2 * P.nu * facexz, yn + yp, F.ryn[j]);
  double Db = div_pre(2 * P.nu * facexy, zb + zp, F.rzb[k]), Df = div_pre(2 * P.nu * facexy, zf + zp, F.rzf[k]);
  double uc = ld(u + IU(F, i, j, k));
  double fw = 0.5 * P.rho * faceyz * (uc + ld(u + IU(F, i - 1, j, k)));
  double fe = 0.5 * P.rho * faceyz * (uc + ld(u + IU(F, i + 1, j, k)));
  double fs = 0.5 * P.rho * facexz * (ld(v + IV(F, i, j, k)) + ld(v + IV(F, i - 1, j, k)));
  double fn = 0.5 * P.rho * facexz * (ld(v + IV(F, i, j + 1, k)) + ld(v + IV(F, i - 1, j + 1, k)));
  double fb = 0.5 * P.rho * facexy * (ld(w + IW(F, i, j, k + 1)) + ld(w + IW(F, i - 1, j, k + 1)));
  double ff = 0.5 * P.rho * facexy * (ld(w + IW(F, i, j, k)) + ld(w + IW(F, i - 1, j, k)));
  double ae = De + dmax0(-fe), aw = Dw + dmax0(fw), an = Dn + dmax0(-fn);
  double as = Ds + dmax0(fs), ab = Db + dmax0(-fb), af = Df + dmax0(ff);
  ap = ae + aw + an + as + ab + af;
  double b = faceyz * (__ldg(F.pt + IP(F, i - 1, j, k)) - __ldg(F.pt + IP(F, i, j, k)));
  old = uc;
  double nv = (ae * ld(u + IU(F, i + 1, j, k)) + aw * ld(u + IU(F, i - 1, j, k)) + an * ld(u + IU(F, i, j + 1, k)) +
               as * ld(u + IU(F, i, j - 1, k)) + af * ld(u + IU(F, i, j, k - 1)) + ab * ld(u + IU(F, i, j, k + 1)) + b) / ap;
  return P.relax * nv + (1 - P.relax) * old;
}
// solveYmomentum body (fluid_solver.h:508-541)
__device__ __forceinline__ double upd_v(const FluidDev &F, const Prm &P, int i, int j, int k, double &ap, double &old,
                                        bool lid) {
  const double *u = F.u, *v = F.v, *w = F.w;
  double xp = F.xp[i], xw = F.xw[i], xe = F.xe[i], yp = F.yp[j], ys = F.ys[j], yn = F.yn[j];
  double zp = F.zp[k], zf = F.zf[k], zb = F.zb[k];
  double facexy = xp * yp, facexz = xp * zp, faceyz = yp * zp;
  double Dw = div_pre(2 * P.nu * faceyz, xp + xw, F.rxw[i]), De = div_pre(2 * P.nu * faceyz, xp + xe, F.rxe[i]);
  double Ds = div_pre(2 * P.nu * facexz, ys + yp, F.rys[j]), Dn = div_pre(2 * P.nu * facexz, yn + yp, F.ryn[j]);
  double Db = div_pre(2 * P.nu * facexy, zb + zp, F.rzb[k]), Df = div_pre(2 * P.nu * facexy, zf + zp, F.rzf[k]);
  double vc = ld(v + IV(F, i, j, k));
  double fn = 0.5 * P.rho * facexz * (vc + ld(v + IV(F, i, j - 1, k)));
  double fs = 0.5 * P.rho * facexz * (vc + ld(v + IV(F, i, j + 1, k)));
  // lid row of u (j == cy, 1 <= i <= cx) reads U0 once applyY has run (after v sweep 1)
  const bool at_lid = lid && j == F.cy;
  double u_c = at_lid ? P.u_lid : ld(u + IU(F, i, j, k));
  double u_e = (at_lid && i + 1 <= F.cx) ? P.u_lid : ld(u + IU(F, i + 1, j, k));
  double fe = 0.5 * P.rho * faceyz * (u_c + ld(u + IU(F, i, j - 1, k)));
  double fw = 0.5 * P.rho * faceyz * (u_e + ld(u + IU(F, i + 1, j - 1, k)));
  double fb = 0.5 * P.rho * facexy * (ld(w + IW(F, i, j, k + 1)) + ld(w + IW(F, i, j - 1, k + 1)));
  double ff = 0.5 * P.rho * facexy * (ld(w + IW(F, i, j, k)) + ld(w + IW(F, i, j - 1, k)));
  double ae = De + dmax0(-fe), aw = Dw + dmax0(fw), an = Dn + dmax0(-fn);
  double as = Ds + dmax0(fs), ab = Db + dmax0(-fb), af = Df + dmax0(ff);
  ap = ae + aw + an + as + ab + af;
  double b = facexz * (__ldg(F.pt + IP(F, i, j - 1, k)) - __ldg(F.pt + IP(F, i, j, k)));
  old = vc;
  double nv = (ae * ld(v + IV(F, i + 1, j, k)) + aw * ld(v + IV(F, i - 1, j, k)) + an * ld(v + IV(F, i, j + 1, k)) +
               as * ld(v + IV(F, i, j - 1, k)) + af * ld(v + IV(F, i, j, k - 1)) + ab * ld(v + IV(F, i, j, k + 1)) + b) / ap;
  return P.relax * nv + (1 - P.relax) * old;
}
// solveZmomentum body (fluid_solver.h:422-455)
__device__ __forceinline__ double upd_w(const FluidDev &F, const Prm &P, int i, int j, int k, double &ap, double &old) {
  const double *u = F.u, *v = F.v, *w = F.w;
  double xp = F.xp[i], xw = F.xw[i], xe = F.xe[i], yp = F.yp[j], ys = F.ys[j], yn = F.yn[j];
  double zp = F.zp[k], zf = F.zf[k], zb = F.zb[k];
  double facexy = xp * yp, facexz = xp * zp, faceyz = yp * zp;
  double Dw = div_pre(2 * P.nu * faceyz, xp + xw, F.rxw[i]), De = div_pre(2 * P.nu * faceyz, xp + xe, F.rxe[i]);
  double Ds = div_pre(2 * P.nu * facexz, ys + yp, F.rys[j]), Dn = div_pre(2 * P.nu * facexz, yn + yp, F.ryn[j]);
  double Db = div_pre(2 * P.nu * facexy, zb + zp, F.rzb[k]), Df = div_pre(2 * P.nu * facexy, zf + zp, F.rzf[k]);
  double wc = ld(w + IW(F, i, j, k));
  double fb = 0.5 * P.rho * facexy * (wc + ld(w + IW(F, i, j, k - 1)));
  double ff = 0.5 * P.rho * facexy * (wc + ld(w + IW(F, i, j, k + 1)));
  double fw = 0.5 * P.rho * faceyz * (ld(u + IU(F, i, j, k)) + ld(u + IU(F, i, j, k - 1)));
  double fe = 0.5 * P.rho * faceyz * (ld(u + IU(F, i + 1, j, k)) + ld(u + IU(F, i + 1, j, k - 1)));
  double fs = 0.5 * P.rho * facexz * (ld(v + IV(F, i, j, k)) + ld(v + IV(F, i, j, k - 1)));
  double fn = 0.5 * P.rho * facexz * (ld(v + IV(F, i, j + 1, k)) + ld(v + IV(F, i, j + 1, k - 1)));
  double ae = De + dmax0(-fe), aw = Dw + dmax0(fw), an = Dn + dmax0(-fn);
  double as = Ds + dmax0(fs), ab = Db + dmax0(-fb), af = Df + dmax0(ff);
  ap = ae + aw + an + as + ab + af;
  double b = facexy * (__ldg(F.pt + IP(F, i, j, k - 1)) - __ldg(F.pt + IP(F, i, j, k)));
  old = wc;
  double nv = (ae * ld(w + IW(F, i + 1, j, k)) + aw * ld(w + IW(F, i - 1, j, k)) + an * ld(w + IW(F, i, j + 1, k)) +
               as * ld(w + IW(F, i, j - 1, k)) + af * ld(w + IW(F, i, j, k - 1)) + ab * ld(w + IW(F, i, j, k + 1)) + b) / ap;
  return P.relax * nv + (1 - P.relax) * old;
}

// ---------------------------------------------------------------- pipelined exact Gauss-Seidel
// Consecutive lexicographic sweeps overlap: sweep n+1 may update hyperplane
// s once sweep n has finished hyperplane s+1 (it needs sweep n's values at
// i+1, j+1, k+1 and its own new values at i-1, j-1, k-1).  At time t sweep
// n therefore works on hyperplane t - 2n; every read is of a value written at
// an earlier time step, so one grid barrier per time step suffices and W
// sweeps take S + 2(W-1) steps instead of W*S.
//
// The reference decides after each sweep whether to sweep again (residual
// test, fluid_solver.h:414-416).  A window of W sweeps is therefore
// speculative: the per-sweep residual sums are kept separately, the stop
// test is replayed sweep by sweep, and if the reference would have stopped
// inside the window the field is restored from a snapshot and exactly that
// many sweeps are rerun (bit-identical, the arithmetic is deterministic).
// The window size is the previous outer step's sweep count.
//
// Boundary conditions applied after every sweep (fluid_solver.h:487, 573,
// 656) only rewrite values the sweeps never change, except that applyY sets
// the lid row of u to U0 after the first v sweep; later v sweeps read U0
// there directly (`lid`), and each BC is applied once after the solve.

__device__ __forceinline__ int pow2_at_least(int w) { int a = 1; while (a < w) a <<= 1; return a; }

// Per-window-slot residual totals after a pipelined pass; identical in every
// block.  `acc` is the thread's sum for its slot (tid % walloc).
__device__ void slot_totals(double acc, int walloc, int w, double *partials, int &buf, double *red, double *tot,
                            cg::grid_group &grid) {
  red[threadIdx.x] = acc;
  __syncthreads();
  double *pp = partials + (size_t)buf * gridDim.x * kBlock;
  buf ^= 1;
  if ((int)threadIdx.x < walloc) {
    double a = 0.0;
    for (int q = threadIdx.x; q < kBlock; q += walloc) a += red[q];
    pp[(size_t)blockIdx.x * walloc + threadIdx.x] = a;
  }
  grid.sync();
  if ((int)threadIdx.x < w) {
    double a = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) a += __ldcg(pp + (size_t)b * walloc + threadIdx.x);
    tot[threadIdx.x] = a;
  }
  __syncthreads();
}

template <int EQ>
__device__ __forceinline__ void gs_point(const FluidDev &F, const Prm &P, int i, int j, int k, bool lid, double &acc) {
  // the face is updated only when the cell on its plus side is fluid; the
  // mask load is issued with the others and only gates the stores
  const bool fl = !F.empty[GC(F, i - 1, j - 1, k - 1)];
  double ap, old, nv;
  int idx;
  if (EQ == 0) { nv = upd_u(F, P, i, j, k, ap, old); idx = IU(F, i, j, k); if (fl) { F.u[idx] = nv; F.up[idx] = ap; } }
  else if (EQ == 1) { nv = upd_v(F, P, i, j, k, ap, old, lid); idx = IV(F, i, j, k); if (fl) { F.v[idx] = nv; F.vp[idx] = ap; } }
  else if (EQ == 2) { nv = upd_w(F, P, i, j, k, ap, old); idx = IW(F, i, j, k); if (fl) { F.w[idx] = nv; F.wp[idx] = ap; } }
  else {
    nv = 0; old = 0; idx = 0;  // the energy equation runs through energy_apply
  }
  (void)idx;
  if (fl) acc += (nv - old) * (nv - old);
}

// solveTemp body (fluid_solver.h:810-846) for up to four independent cells of
// one time step: every load of the four is issued before any arithmetic.
struct EnergyIn {
  double te, tw, tn, ts, tf, tb, tc, u, v, w;
  int q, i, j, k;
  bool ok;
};
__device__ __forceinline__ void energy_gather(const FluidDev &F, int i, int j, int k, EnergyIn &e) {
  const double *Ts = F.ts;
  const long long row = (long long)F.hx * (j + (long long)(F.cy + 2) * k);
  const long long q = (i & 1) * F.hs + (i >> 1) + row, qo = ((i & 1) ^ 1) * F.hs + row;
  e.q = (int)q; e.i = i; e.j = j; e.k = k;
  const int PY = F.hx, PZ = F.hx * (F.cy + 2);
  e.te = ld(Ts + qo + ((i + 1) >> 1)); e.tw = ld(Ts + qo + ((i - 1) >> 1));
  e.tn = ld(Ts + q + PY); e.ts = ld(Ts + q - PY); e.tf = ld(Ts + q + PZ); e.tb = ld(Ts + q - PZ);
  e.tc = ld(Ts + q);
  e.u = __ldg(F.us + q); e.v = __ldg(F.vs + q); e.w = __ldg(F.ws + q);
  e.ok = e.ok && !F.empty[GC(F, i - 1, j - 1, k - 1)];
}
__device__ __forceinline__ void energy_apply(const FluidDev &F, const Prm &P, const EnergyIn &e, double &acc) {
  double xp = F.xp[e.i], xw = F.xw[e.i], yp = F.yp[e.j], ys = F.ys[e.j], zp = F.zp[e.k], zf = F.zf[e.k];
  double sx = (xp + xw) / 2.0, sy = (yp + ys) / 2.0, sz = (zp + zf) / 2.0;
  double conv = -e.u * (e.te - e.tw) - e.v * (e.tn - e.ts) - e.w * (e.tf - e.tb);
  const double rx = F.rsx[e.i], ry = F.rsy[e.j], rz = F.rsz[e.k];
  // alpha*(te+tw)/sx/sx etc. (fluid_solver.h:838-840) with exact divisions
  double diff = div_pre(div_pre(P.alpha * (e.te + e.tw), sx, rx), sx, rx) +
                div_pre(div_pre(P.alpha * (e.tn + e.ts), sy, ry), sy, ry) +
                div_pre(div_pre(P.alpha * (e.tf + e.tb), sz, rz), sz, rz);
  double denom = 2 * P.alpha * (F.ix2[e.i] + F.iy2[e.j] + F.iz2[e.k]);
  double nv = (conv + diff) / denom * (P.relax) + (1 - P.relax) * e.tc;
  F.ts[e.q] = nv;
  acc += (nv - e.tc) * (nv - e.tc);
}

// One GS solve of equation EQ (0 u, 1 v, 2 w momentum; 3 fluid energy).
template <int EQ>
__global__ void __launch_bounds__(kBlock, 2) k_gs(FluidDev F, Prm P, double *partials, DevStats *st, double *snap) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double red[kBlock];
  __shared__ double tot[kBlock];
  const int NI = EQ == 0 ? F.fx - 1 : F.cx, NJ = EQ == 1 ? F.fy - 1 : F.cy, NK = EQ == 2 ? F.fz - 1 : F.cz;
  const double d1 = EQ == 2 ? F.fz : F.cz, d2 = EQ == 1 ? F.fy : F.cy, d3 = EQ == 0 ? F.fx : F.cx;
  const double tol = EQ == 3 ? P.energy_tol : P.mom_tol;
  const int nrows = NJ * NK, S = NI + NJ + NK - 2;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  double *own = EQ == 0 ? F.u : EQ == 1 ? F.v : EQ == 2 ? F.w : F.ts;
  const long long nown = EQ == 0 ? (long long)(F.fx + 2) * (F.cy + 2) * (F.cz + 2)
                       : EQ == 1 ? (long long)(F.cx + 2) * (F.fy + 2) * (F.cz + 2)
                       : EQ == 2 ? (long long)(F.cx + 2) * (F.cy + 2) * (F.fz + 2)
                                 : 2 * F.hs;
  const long long npadT = (long long)(F.cx + 2) * (F.cy + 2) * (F.cz + 2);
  if (EQ == 3) {
    // parity-split copies of T, u, v, w for this solve
    for (long long q = tid; q < npadT; q += T) {
      const int i = (int)(q % (F.cx + 2)), j = (int)((q / (F.cx + 2)) % (F.cy + 2)), k = (int)(q / ((long long)(F.cx + 2) * (F.cy + 2)));
      const long long sq = (i & 1) * F.hs + (i >> 1) + (long long)F.hx * (j + (long long)(F.cy + 2) * k);
      F.ts[sq] = F.tt[q];
      F.us[sq] = F.u[IU(F, i, j, k)];
      F.vs[sq] = F.v[IV(F, i, j, k)];
      F.ws[sq] = F.w[IW(F, i, j, k)];
    }
  }
  const bool lid_row = (F.oy - 1 + F.fy - 1 == F.Ny);
  int buf = 0;
  const int pred = st->sweeps[EQ] > 0 ? st->sweeps[EQ] : 2;
  grid.sync();  // every block has read the prediction before thread 0 rewrites it
  double residual = 1.0, gres = 1.0;
  int done = 0;
  while (done < P.gs_max && !(gres < tol)) {
    int W = done < pred ? pred - done : max(1, done);
    W = min(W, min(P.gs_max - done, kBlock));
    const bool spec = W > 1;
    if (spec) {
      for (long long q = tid; q < nown; q += T) snap[q] = ld(own + q);
      grid.sync();
    }
    int runs = 0, stop = W;
    double r_new = residual, g_new = gres;
    for (;;) {
      const int walloc = pow2_at_least(W);
      const int n = tid % walloc;
      double acc = 0.0;
      const int steps = S + 2 * (W - 1);
      // this thread's rows: row0 + m*R, stepped incrementally in (j, k)
      const int R = T / walloc, row0 = tid / walloc;
      const int dj = R % NJ, dk = R / NJ;
      const int j0 = row0 % NJ + 1, k0 = row0 / NJ + 1;
      for (int t = 0; t < steps; ++t) {
        if (n < W) {
          const bool lid = EQ == 1 && lid_row && (done + n) >= 1;
          const int base = t - 2 * n + 1;  // i = base - (j - 1) - (k - 1)
          int j = j0, k = k0;
          if (EQ == 3) {
            // groups of four of this thread's rows; loads of the active ones
            // are issued together (static indices keep them in registers)
            for (int row = row0; row < nrows; row += 4 * R) {
              EnergyIn e[4];
#pragma unroll
              for (int b = 0; b < 4; ++b) {
                const int i = base - (j - 1) - (k - 1);
                e[b].ok = row + b * R < nrows && (unsigned)(i - 1) < (unsigned)NI;
                if (e[b].ok) energy_gather(F, i, j, k, e[b]);
                j += dj; k += dk;
                if (j > NJ) { j -= NJ; ++k; }
              }
#pragma unroll
              for (int b = 0; b < 4; ++b)
                if (e[b].ok) energy_apply(F, P, e[b], acc);
            }
          } else {
            for (int row = row0; row < nrows; row += R) {
              const int i = base - (j - 1) - (k - 1);
              if ((unsigned)(i - 1) < (unsigned)NI) gs_point<EQ>(F, P, i, j, k, lid, acc);
              j += dj; k += dk;
              if (j > NJ) { j -= NJ; ++k; }
            }
          }
        }
        grid.sync();
      }
      slot_totals(acc, walloc, W, partials, buf, red, tot, grid);
      if (runs == 1) break;  // the rerun reproduces the first pass exactly
      // replay the reference's stop test sweep by sweep
      double r = residual, g = gres;
      stop = W;
      for (int c = 1; c <= W; ++c) {
        r = (r + tot[c - 1]) / d1 / d2 / d3;
        g = sqrt(r);
        if (g < tol || done + c >= P.gs_max) { stop = c; break; }
      }
      r_new = r; g_new = g;
      runs = 1;
      if (stop == W) break;
      for (long long q = tid; q < nown; q += T) own[q] = snap[q];
      grid.sync();
      W = stop;
    }
    done += stop;
    residual = r_new;
    gres = g_new;
  }
  const int T2 = T;
  if (EQ == 3)
    for (long long q = tid; q < npadT; q += T) {
      const int i = (int)(q % (F.cx + 2)), j = (int)((q / (F.cx + 2)) % (F.cy + 2)), k = (int)(q / ((long long)(F.cx + 2) * (F.cy + 2)));
      F.tt[q] = ld(F.ts + (i & 1) * F.hs + (i >> 1) + (long long)F.hx * (j + (long long)(F.cy + 2) * k));
    }
  if (EQ == 0) bc_x(F, tid, T2);
  else if (EQ == 1) bc_y(F, P, tid, T2);
  else if (EQ == 2) bc_z(F, tid, T2);
  if (tid == 0) { st->sweeps[EQ] = done; st->res[EQ] = gres; st->cum_sweeps[EQ] += done; }
}

// ---------------------------------------------------------------- solid energy
// MobSolver::solve (mobs_solver.h:303-319) with solveTemperature
// (mobs_solver.h:467-500) for every solid region at once, pipelined and
// speculated like k_gs; each region keeps its own residual, stop test and
// sweep count.
constexpr int kMaxRegions = 256;
__global__ void __launch_bounds__(kBlock, 2) k_solid(const SolidReg *regs, int nreg, const int *blk_reg, double *tt_all,
                                                  double *tc_all, const uint8_t *em_all, Prm P, double *partials,
                                                  DevStats *st, double *snap, int *pred_all) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double red[kBlock];
  __shared__ double r2[kMaxRegions];
  __shared__ int done[kMaxRegions], W[kMaxRegions], stopc[kMaxRegions];
  __shared__ double rnew[kMaxRegions];
  __shared__ int ctl[3];  // any-active, max-steps, any-rollback
  const int r = blk_reg[blockIdx.x];
  const SolidReg R = regs[r];
  double *Tr = tt_all + R.tt_off;
  const uint8_t *em = em_all + R.em_off;
  const int ltid = (blockIdx.x - R.blk0) * blockDim.x + threadIdx.x, LT = R.nblk * blockDim.x;
  const int PX = R.cx + 2, PXY = (R.cx + 2) * (R.cy + 2);
  const long long npad_r = (long long)PXY * (R.cz + 2);
  // applyOuterBoundaryCondition: every cell of the box to T1 (mobs_solver.h:105-115)
  for (int c = ltid; c < R.cx * R.cy * R.cz; c += LT) tc_all[R.tc_off + c] = P.t_solid0;
  for (int q = threadIdx.x; q < nreg; q += blockDim.x) { r2[q] = 1.0; done[q] = 0; }
  __syncthreads();
  int buf = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      int any = 0, steps = 0;
      for (int q = 0; q < nreg; ++q) {
        const bool act = done[q] < P.gs_max && !(r2[q] < P.solid_tol);
        int w = 0;
        if (act) {
          const int pr = pred_all[q] > 0 ? pred_all[q] : 2;
          w = done[q] < pr ? pr - done[q] : max(1, done[q]);
          w = min(w, min(P.gs_max - done[q], kBlock));
          any = 1;
          steps = max(steps, regs[q].cx + regs[q].cy + regs[q].cz - 2 + 2 * (w - 1));
        }
        W[q] = w;
      }
      ctl[0] = any; ctl[1] = steps;
    }
    __syncthreads();
    if (!ctl[0]) break;
    // snapshot this block's share of its region
    if (W[r] > 1)
      for (long long q = ltid; q < npad_r; q += LT) snap[R.tt_off + q] = ld(Tr + q);
    grid.sync();
    for (int run = 0; run < 2; ++run) {
      const int w = W[r], walloc = pow2_at_least(max(w, 1));
      const int n = ltid % walloc;
      double acc = 0.0;
      const int steps = ctl[1];
      const int Rr = LT / walloc, row0 = ltid / walloc;
      const int dj = Rr % R.cy, dk = Rr / R.cy;
      const int j0 = row0 % R.cy + 1, k0 = row0 / R.cy + 1;
      for (int t = 0; t < steps; ++t) {
        if (n < w) {
          const int base = t - 2 * n + 1;
          int j = j0, k = k0;
          for (int row = row0; row < R.rows; row += 4 * Rr) {
            double v[4][7];
            int qq[4];
            bool ok[4];
#pragma unroll
            for (int b = 0; b < 4; ++b) {
              const int i = base - (j - 1) - (k - 1);
              ok[b] = row + b * Rr < R.rows && (unsigned)(i - 1) < (unsigned)R.cx;
              if (ok[b]) {
                const int q = i + PX * j + PXY * k;
                qq[b] = q;
                ok[b] = !em[(i - 1) + R.cx * ((j - 1) + R.cy * (k - 1))];
                v[b][0] = ld(Tr + q); v[b][1] = ld(Tr + q + 1); v[b][2] = ld(Tr + q - 1); v[b][3] = ld(Tr + q - PX);
                v[b][4] = ld(Tr + q + PX); v[b][5] = ld(Tr + q - PXY); v[b][6] = ld(Tr + q + PXY);
              }
              j += dj; k += dk;
              if (j > R.cy) { j -= R.cy; ++k; }
            }
#pragma unroll
            for (int b = 0; b < 4; ++b)
              if (ok[b]) {
                const double old = v[b][0];
                double nv = 1.0 / 6.0 * (v[b][1] + v[b][2] + v[b][3] + v[b][4] + v[b][5] + v[b][6]);
                nv = nv * P.relax_solid + (1 - P.relax_solid) * old;
                Tr[qq[b]] = nv;
                acc += (nv - old) * (nv - old);
              }
          }
        }
        grid.sync();
      }
      // per-(region, slot) totals: block partial per slot, region sum in block order
      red[threadIdx.x] = acc;
      __syncthreads();
      double *pp = partials + (size_t)buf * gridDim.x * kBlock;
      buf ^= 1;
      if ((int)threadIdx.x < kBlock) {
        double a = 0.0;
        if ((int)threadIdx.x < walloc)
          for (int q = threadIdx.x; q < kBlock; q += walloc) a += red[q];
        pp[(size_t)blockIdx.x * kBlock + threadIdx.x] = a;
      }
      grid.sync();
      if (run == 1) break;
      // replay every region's stop test (all blocks compute the same)
      for (int q = threadIdx.x; q < nreg; q += blockDim.x) {
        stopc[q] = W[q];
        rnew[q] = r2[q];
        if (W[q] == 0) continue;
        const SolidReg Q = regs[q];
        double rr = r2[q];
        for (int c = 1; c <= W[q]; ++c) {
          double a = 0.0;
          for (int b = Q.blk0; b < Q.blk0 + Q.nblk; ++b) a += __ldcg(pp + (size_t)b * kBlock + (c - 1));
          rr = sqrt((rr + a) / (double)Q.cz / (double)Q.cy / (double)Q.cx);
          if (rr < P.solid_tol || done[q] + c >= P.gs_max) { stopc[q] = c; break; }
        }
        rnew[q] = rr;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int rb = 0, steps = 0;
        for (int q = 0; q < nreg; ++q) {
          if (stopc[q] < W[q]) { rb = 1; steps = max(steps, regs[q].cx + regs[q].cy + regs[q].cz - 2 + 2 * (stopc[q] - 1)); }
        }
        ctl[2] = rb; ctl[1] = steps;
      }
      __syncthreads();
      if (!ctl[2]) break;
      // regions that overran: restore and rerun exactly stopc sweeps; others idle
      const bool mine_rb = stopc[r] < W[r];
      if (mine_rb)
        for (long long q = ltid; q < npad_r; q += LT) Tr[q] = snap[R.tt_off + q];
      __syncthreads();
      if (threadIdx.x == 0)
        for (int q = 0; q < nreg; ++q) W[q] = stopc[q] < W[q] ? stopc[q] : 0;
      __syncthreads();
      grid.sync();
    }
    // stopc holds the sweeps each region executed in this window
    for (int q = threadIdx.x; q < nreg; q += blockDim.x)
      if (stopc[q] > 0) { done[q] += stopc[q]; r2[q] = rnew[q]; }
    __syncthreads();
  }
  grid.sync();  // every block has read pred_all before it is rewritten
  if (blockIdx.x == 0) {
    for (int q = threadIdx.x; q < nreg; q += blockDim.x) pred_all[q] = done[q];
    if (threadIdx.x == 0) {
      int m = 0;
      long long cells = 0;
      for (int q = 0; q < nreg; ++q) {
        m = max(m, done[q]);
        cells += (long long)done[q] * regs[q].cx * regs[q].cy * regs[q].cz;
      }
      st->solid_sweeps_max = m;
      st->cum_solid_cell_sweeps += cells;
    }
  }
}

// MobSolver::setForNext (mobs_solver.h:290-301)
__global__ void k_solid_setfornext(const SolidReg *regs, int nreg, double *tt_all, double *tc_all, const uint8_t *em_all) {
  for (int r = blockIdx.y; r < nreg; r += gridDim.y) {
    const SolidReg R = regs[r];
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < R.cx * R.cy * R.cz; c += gridDim.x * blockDim.x) {
      if (em_all[R.em_off + c]) continue;
      int i = c % R.cx, j = (c / R.cx) % R.cy, k = c / (R.cx * R.cy);
      tc_all[R.tc_off + c] = tt_all[R.tt_off + (i + 1) + (R.cx + 2) * ((j + 1) + (R.cy + 2) * (k + 1))];
    }
  }
}

// ---------------------------------------------------------------- interface swap (solver.h:83-148)
__global__ void k_swap_gather(const long long *f_send, const long long *s_send, int n, const double *ft, const double *st_,
                              double *fbuf, double *sbuf) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    fbuf[e] = ft[f_send[e]];
    sbuf[e] = st_[s_send[e]];
  }
}
__global__ void k_swap_scatter(const long long *f_recv, const long long *s_recv, int n, double *ft, double *st_,
                               const double *fbuf, const double *sbuf) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    ft[f_recv[e]] = sbuf[e];
    st_[s_recv[e]] = fbuf[e];
  }
}

// ---------------------------------------------------------------- pressure correction
// Assembly (fluid_solver.h:1969-2002 / 2123-2162) + HYPRE PCG restated.
//
// Pass A of an iteration (p = r + beta p, s = A p, x += alpha_prev p_old,
// <s,p>) runs over 32 x 8 x TZ tiles: each block marches a tile column in
// z, keeping three planes of the new direction (with a one-cell halo) in
// shared memory, so every neighbour comes from shared memory and each cell's
// r and p are read once.  Coefficients are zero off the fluid cells, where
// r, p, x, s stay zero, so no mask test is needed.  Pass B (r -= alpha s,
// <r,r>) streams the padded arrays as double2.
constexpr int kTX = 32, kTY = 16;  // CG tiles of 32 x 16 columns; a thread owns rows ty and ty + 8

// The CG iterations of hypre_PCGSolve restated (identity preconditioner,
// two-norm test <r,r>/<b,b> < tol^2, maxiter): on entry r = p_a = b, x = 0 on
// the padded grid and bb = <b,b>.  Coefficients are zero off the unknowns.
struct CgView {
  int cx, cy, cz;
  const double *acx, *acy, *acz;
  double *x, *r, *pa, *pb, *s;
};

__device__ void cg_core(const CgView &V, double bb, double tol, int maxiter, double *partials, int &buf, double *sh,
                        cg::grid_group &grid, int TZ, int *out_iters, double *out_relres) {
  __shared__ double pl[4][kTY + 2][kTX + 2];  // four plane slots: the plane written at kk never aliases those read at kk - 1
  const int cx = V.cx, cy = V.cy, cz = V.cz;
  const int PX = cx + 2, PXY = (cx + 2) * (cy + 2);
  const long long npad = (long long)PXY * (cz + 2);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  const double eps = tol * tol;
  double gamma = bb, iprod = bb, beta = 0.0, alpha_prev = 0.0, acc;
  double *pold = V.pa, *pnew = V.pb;
  const int ntx = (cx + kTX - 1) / kTX, nty = (cy + kTY - 1) / kTY, ntz = (cz + TZ - 1) / TZ;
  const int ntiles = ntx * nty * ntz;
  const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;  // ty in [0, 8)
  // halo role (96 cells: y-1 row, y+16 row, x-1 column, x+32 column)
  const int h = threadIdx.x;
  int hx = -1, hy = -1;
  if (h < kTX) { hx = h + 1; hy = 0; }
  else if (h < 2 * kTX) { hx = h - kTX + 1; hy = kTY + 1; }
  else if (h < 2 * kTX + kTY) { hx = 0; hy = h - 2 * kTX + 1; }
  else if (h < 2 * kTX + 2 * kTY) { hx = kTX + 1; hy = h - 2 * kTX - kTY + 1; }
  int it = 0;
  bool pending = false;
  while (it + 1 <= maxiter) {
    it++;
    acc = 0.0;
    const double *r = V.r;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      const int tz = tile / (ntx * nty), rem = tile % (ntx * nty);
      const int i0 = 1 + (rem % ntx) * kTX, j0 = 1 + (rem / ntx) * kTY, k0 = 1 + tz * TZ;
      const int kend = min(k0 + TZ - 1, cz);
      const int i = i0 + tx, ja = j0 + ty, jb = ja + 8;
      const bool inA = i <= cx && ja <= cy, inB = i <= cx && jb <= cy;
      const bool padA = i <= cx + 1 && ja <= cy + 1, padB = i <= cx + 1 && jb <= cy + 1;
      const int hi = i0 - 1 + hx, hj = j0 - 1 + hy;
      const bool hin = hx >= 0 && hi <= cx + 1 && hj <= cy + 1;
      double poA = 0.0, poB = 0.0;  // p_old of the plane being computed (kk - 1)
      double nA = 0.0, nB = 0.0;    // p_old of plane kk
      for (int kk = k0 - 1; kk <= kend + 1; ++kk) {
        const int slot = (kk - k0 + 1) & 3;
        const bool comp = kk >= k0 + 1;
        // issue every load of this plane step before using any of them
        const int qA = i + PX * ja + PXY * kk, qB = qA + 8 * PX;
        double rA = 0.0, rB = 0.0, hr = 0.0, hp = 0.0;
        poA = nA; poB = nB;
        nA = 0.0; nB = 0.0;
        if (padA) { nA = ld(pold + qA); if (it > 1) rA = ld(r + qA); }
        if (padB) { nB = ld(pold + qB); if (it > 1) rB = ld(r + qB); }
        if (hin) {
          const int qh = hi + PX * hj + PXY * kk;
          hp = ld(pold + qh);
          if (it > 1) hr = ld(r + qh);
        }
        const int cA = qA - PXY, cB = qB - PXY;
        double axA = 0, ayA = 0, azA = 0, xA = 0, axB = 0, ayB = 0, azB = 0, xB = 0;
        if (comp && inA) { axA = V.acx[cA]; ayA = V.acy[cA]; azA = V.acz[cA]; if (it > 1) xA = ld(V.x + cA); }
        if (comp && inB) { axB = V.acx[cB]; ayB = V.acy[cB]; azB = V.acz[cB]; if (it > 1) xB = ld(V.x + cB); }
        pl[slot][ty + 1][tx + 1] = it == 1 ? nA : rA + beta * nA;
        pl[slot][ty + 9][tx + 1] = it == 1 ? nB : rB + beta * nB;
        if (hx >= 0) pl[slot][hy][hx] = it == 1 ? hp : hr + beta * hp;
        __syncthreads();
        if (comp) {
          const int sc = (slot + 3) & 3, sb = (slot + 2) & 3;
          if (inA) {
            const int y = ty + 1;
            const double c0 = pl[sc][y][tx + 1];
            const double d = axA + axA + ayA + ayA + azA + azA;
            const double sv = d * c0 - azA * pl[sb][y][tx + 1] - ayA * pl[sc][y - 1][tx + 1] - axA * pl[sc][y][tx] -
                              axA * pl[sc][y][tx + 2] - ayA * pl[sc][y + 1][tx + 1] - azA * pl[slot][y][tx + 1];
            if (it > 1) V.x[cA] = xA + alpha_prev * poA;
            pnew[cA] = c0;
            V.s[cA] = sv;
            acc += sv * c0;
          }
          if (inB) {
            const int y = ty + 9;
            const double c0 = pl[sc][y][tx + 1];
            const double d = axB + axB + ayB + ayB + azB + azB;
            const double sv = d * c0 - azB * pl[sb][y][tx + 1] - ayB * pl[sc][y - 1][tx + 1] - axB * pl[sc][y][tx] -
                              axB * pl[sc][y][tx + 2] - ayB * pl[sc][y + 1][tx + 1] - azB * pl[slot][y][tx + 1];
            if (it > 1) V.x[cB] = xB + alpha_prev * poB;
            pnew[cB] = c0;
            V.s[cB] = sv;
            acc += sv * c0;
          }
        }
      }
      __syncthreads();  // the next tile reuses the slots
    }
    const double sdotp = grid_sum(acc, partials, buf, sh, grid);
    if (sdotp == 0.0) { pending = false; break; }
    const double alpha = gamma / sdotp, gamma_old = gamma;
    acc = 0.0;
    {
      double2 *r2 = reinterpret_cast<double2 *>(V.r);
      const double2 *s2 = reinterpret_cast<const double2 *>(V.s);
      const long long nh = npad / 2;
      for (long long e = tid; e < nh; e += T) {
        double2 rv = __ldcg(r2 + e), sv = __ldcg(s2 + e);
        rv.x = rv.x - alpha * sv.x;
        rv.y = rv.y - alpha * sv.y;
        r2[e] = rv;
        acc += rv.x * rv.x;
        acc += rv.y * rv.y;
      }
      if ((npad & 1) && tid == 0) {
        const long long e = npad - 1;
        double rv = ld(V.r + e) - alpha * ld(V.s + e);
        V.r[e] = rv;
        acc += rv * rv;
      }
    }
    gamma = grid_sum(acc, partials, buf, sh, grid);
    iprod = gamma;
    alpha_prev = alpha;
    pending = true;
    double *t = pold; pold = pnew; pnew = t;
    if (iprod / bb < eps) break;
    beta = gamma / gamma_old;
  }
  if (pending)
    for (long long e = tid; e < npad; e += T) V.x[e] = ld(V.x + e) + alpha_prev * ld(pold + e);
  if (tid == 0) { *out_iters = it; *out_relres = sqrt(iprod / bb); }
}

__global__ void __launch_bounds__(kBlock) k_pcorr(FluidDev F, Prm P, double *partials, DevStats *st, int assemble,
                                                  int TZ) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[33];
  const int cx = F.cx, cy = F.cy, cz = F.cz, n = cx * cy * cz;
  const int PX = cx + 2, PXY = (cx + 2) * (cy + 2);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  int buf = 0;
  double acc = 0.0;
  for (int c = tid; c < n; c += T) {
    if (F.empty[c]) continue;
    const int i = c % cx, j = (c / cx) % cy, k = c / (cx * cy);
    const int q = (i + 1) + PX * (j + 1) + PXY * (k + 1);
    if (assemble) {
      double xp = F.xp[i + 1], yp = F.yp[j + 1], zp = F.zp[k + 1];
      double facexy = xp * yp, facexz = xp * zp, faceyz = yp * zp;
      F.acx[q] = faceyz / F.up[IU(F, i + 1, j + 1, k + 1)];
      F.acy[q] = facexz / F.vp[IV(F, i + 1, j + 1, k + 1)];
      F.acz[q] = facexy / F.wp[IW(F, i + 1, j + 1, k + 1)];
    }
    double b = -(F.u[IU(F, i + 2, j + 1, k + 1)] - F.u[IU(F, i + 1, j + 1, k + 1)]) -
               (F.v[IV(F, i + 1, j + 2, k + 1)] - F.v[IV(F, i + 1, j + 1, k + 1)]) -
               (F.w[IW(F, i + 1, j + 1, k + 2)] - F.w[IW(F, i + 1, j + 1, k + 1)]);
    F.r[q] = b;
    F.pa[q] = b;
    F.x[q] = 0.0;
    acc += b * b;
  }
  const double bb = grid_sum(acc, partials, buf, sh, grid);
  if (bb == 0.0) {
    if (tid == 0) { st->pcg_iters = 0; st->pcg_relres = 0.0; st->cum_pcg_solves += 1; }
    return;
  }
  CgView V{cx, cy, cz, F.acx, F.acy, F.acz, F.x, F.r, F.pa, F.pb, F.s};
  int iters = 0;
  double relres = 0.0;
  cg_core(V, bb, P.pcg_tol, P.pcg_maxiter, partials, buf, sh, grid, TZ, &iters, &relres);
  if (tid == 0) {
    st->pcg_iters = iters; st->pcg_relres = relres; st->cum_pcg_iters += iters; st->cum_pcg_solves += 1;
  }
}

// Standalone HYPRE-rule CG on caller-provided padded arrays: r = p_a = b,
// x = 0, then cg_core (hs_pcg_solve).
__global__ void __launch_bounds__(kBlock) k_pcg(CgView V, const double *b, double tol, int maxiter, double *partials,
                                                int TZ, int *out_iters, double *out_relres) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[33];
  const long long npad = (long long)(V.cx + 2) * (V.cy + 2) * (V.cz + 2);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  int buf = 0;
  double acc = 0.0;
  for (long long e = tid; e < npad; e += T) {
    const double bv = b[e];
    V.r[e] = bv;
    V.pa[e] = bv;
    V.pb[e] = 0.0;
    V.s[e] = 0.0;
    V.x[e] = 0.0;
    acc += bv * bv;
  }
  const double bb = grid_sum(acc, partials, buf, sh, grid);
  if (bb == 0.0) {
    if (tid == 0) { *out_iters = 0; *out_relres = 0.0; }
    return;
  }
  cg_core(V, bb, tol, maxiter, partials, buf, sh, grid, TZ, out_iters, out_relres);
}

// ---------------------------------------------------------------- multigrid-preconditioned CG
// HS_PSOLVE_MGCG: the same pressure-correction system, solved by CG with a
// geometric multigrid V-cycle as preconditioner.  The V-cycle runs in FP32
// (fields, coefficients, smoother, transfers); the CG recurrences, residual,
// dot products and the coarsest-grid direct solve are FP64.
//   coarsening   2x per axis (ceil), masked: a coarse cell is an unknown when
//                any child is; per-cell coefficients c_C = (sum of children)/4
//                (a 2x2 face patch summed, halved for the doubled spacing)
//   smoother     red-black Gauss-Seidel, one pre (red, black) and one post
//                (black, red) sweep, x = 0 start
//   transfers    sum restriction of the residual, constant prolongation
//   coarsest     <= 64 cells, LU with partial pivoting factored on the host
constexpr int kMaxLevels = 14;
constexpr int kMaxCoarse = 64;

struct MgLevel {
  int nx, ny, nz;
  float *x, *rhs, *ax, *ay, *az;
  uint8_t *m;  // 1 = unknown
};
struct MgView {
  int L;
  MgLevel lv[kMaxLevels];
  int nc;             // unknowns of the coarsest level (all its padded-interior cells)
  const double *lu;   // nc x nc, row-major, L (unit) and U packed
  const int *piv;
  double *yc;         // nc scratch
};

__device__ __forceinline__ int mgidx(const MgLevel &L, int i, int j, int k) { return i + (L.nx + 2) * (j + (L.ny + 2) * k); }

// level 0 coefficients and mask from the FP64 frozen coefficients
__global__ void k_mg_fine(FluidDev F, MgLevel L0) {
  const int cx = F.cx, cy = F.cy, n = cx * cy * F.cz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % cx, j = (c / cx) % cy, k = c / (cx * cy);
    const int q = (i + 1) + (cx + 2) * ((j + 1) + (cy + 2) * (k + 1));
    const bool u = !F.empty[c];
    L0.m[q] = u;
    L0.ax[q] = u ? (float)F.acx[q] : 0.f;
    L0.ay[q] = u ? (float)F.acy[q] : 0.f;
    L0.az[q] = u ? (float)F.acz[q] : 0.f;
  }
}

__global__ void k_mg_coarsen(MgLevel Fl, MgLevel C) {
  const int n = C.nx * C.ny * C.nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int I = c % C.nx, J = (c / C.nx) % C.ny, K = c / (C.nx * C.ny);
    float sx = 0.f, sy = 0.f, sz = 0.f;
    int any = 0;
    for (int dk = 0; dk < 2; ++dk)
      for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
          const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
          if (i >= Fl.nx || j >= Fl.ny || k >= Fl.nz) continue;
          const int q = mgidx(Fl, i + 1, j + 1, k + 1);
          if (!Fl.m[q]) continue;
          any = 1;
          sx += Fl.ax[q]; sy += Fl.ay[q]; sz += Fl.az[q];
        }
    const int qc = mgidx(C, I + 1, J + 1, K + 1);
    C.m[qc] = any;
    C.ax[qc] = 0.25f * sx; C.ay[qc] = 0.25f * sy; C.az[qc] = 0.25f * sz;
  }
}

// one red-black half sweep on level L; zero_nb: neighbours read as zero (first pass of a cycle)
__device__ void mg_smooth(const MgLevel &L, int color, bool zero_nb, int tid, int T) {
  const int n = L.nx * L.ny * L.nz, PX = L.nx + 2, PXY = (L.nx + 2) * (L.ny + 2);
  for (int c = tid; c < n; c += T) {
    const int i = c % L.nx, j = (c / L.nx) % L.ny, k = c / (L.nx * L.ny);
    if (((i + j + k) & 1) != color) continue;
    const int q = (i + 1) + PX * (j + 1) + PXY * (k + 1);
    if (!L.m[q]) continue;
    const float ax = L.ax[q], ay = L.ay[q], az = L.az[q];
    const float d = 2.f * (ax + ay + az);
    float sum = L.rhs[q];
    if (!zero_nb) {
      const float *x = L.x;
      sum += ax * (__ldcg(x + q - 1) + __ldcg(x + q + 1)) + ay * (__ldcg(x + q - PX) + __ldcg(x + q + PX)) +
             az * (__ldcg(x + q - PXY) + __ldcg(x + q + PXY));
    }
    L.x[q] = sum / d;
  }
}

// coarse rhs = sum over the children of (rhs - A x)
__device__ void mg_restrict(const MgLevel &Fl, const MgLevel &C, int tid, int T) {
  const int n = C.nx * C.ny * C.nz, PX = Fl.nx + 2, PXY = (Fl.nx + 2) * (Fl.ny + 2);
  for (int c = tid; c < n; c += T) {
    const int I = c % C.nx, J = (c / C.nx) % C.ny, K = c / (C.nx * C.ny);
    float acc = 0.f;
    for (int dk = 0; dk < 2; ++dk)
      for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
          const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
          if (i >= Fl.nx || j >= Fl.ny || k >= Fl.nz) continue;
          const int q = (i + 1) + PX * (j + 1) + PXY * (k + 1);
          if (!Fl.m[q]) continue;
          const float *x = Fl.x;
          const float ax = Fl.ax[q], ay = Fl.ay[q], az = Fl.az[q];
          const float r = Fl.rhs[q] - (2.f * (ax + ay + az) * __ldcg(x + q) -
                                       ax * (__ldcg(x + q - 1) + __ldcg(x + q + 1)) -
                                       ay * (__ldcg(x + q - PX) + __ldcg(x + q + PX)) -
                                       az * (__ldcg(x + q - PXY) + __ldcg(x + q + PXY)));
          acc += r;
        }
    const int qc = mgidx(C, I + 1, J + 1, K + 1);
    C.rhs[qc] = C.m[qc] ? acc : 0.f;
  }
}

__device__ void mg_prolong(const MgLevel &Fl, const MgLevel &C, int tid, int T) {
  const int n = Fl.nx * Fl.ny * Fl.nz;
  for (int c = tid; c < n; c += T) {
    const int i = c % Fl.nx, j = (c / Fl.nx) % Fl.ny, k = c / (Fl.nx * Fl.ny);
    const int q = mgidx(Fl, i + 1, j + 1, k + 1);
    if (!Fl.m[q]) continue;
    Fl.x[q] = __ldcg(Fl.x + q) + __ldcg(C.x + mgidx(C, i / 2 + 1, j / 2 + 1, k / 2 + 1));
  }
}

// z = V-cycle(rhs of level 0), result in lv[0].x
__device__ void mg_vcycle(const MgView &M, cg::grid_group &grid, int tid, int T) {
  for (int l = 0; l < M.L - 1; ++l) {
    mg_smooth(M.lv[l], 0, true, tid, T);
    grid.sync();
    mg_smooth(M.lv[l], 1, false, tid, T);
    grid.sync();
    mg_restrict(M.lv[l], M.lv[l + 1], tid, T);
    grid.sync();
  }
  {
    // coarsest: FP64 LU solve by one warp of block 0
    const MgLevel &C = M.lv[M.L - 1];
    if (blockIdx.x == 0 && threadIdx.x < 32) {
      const int nc = M.nc, lane = threadIdx.x;
      double *y = M.yc;
      // permuted rhs
      if (lane == 0)
        for (int r = 0; r < nc; ++r) {
          const int s = M.piv[r];
          y[r] = (double)C.rhs[mgidx(C, s % C.nx + 1, (s / C.nx) % C.ny + 1, s / (C.nx * C.ny) + 1)];
        }
      __syncwarp();
      for (int r = 0; r < nc; ++r) {  // forward (unit lower)
        double a = 0.0;
        for (int c2 = lane; c2 < r; c2 += 32) a += M.lu[r * nc + c2] * y[c2];
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) y[r] -= a;
        __syncwarp();
      }
      for (int r = nc - 1; r >= 0; --r) {  // backward
        double a = 0.0;
        for (int c2 = r + 1 + lane; c2 < nc; c2 += 32) a += M.lu[r * nc + c2] * y[c2];
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) y[r] = (y[r] - a) / M.lu[r * nc + r];
        __syncwarp();
      }
      for (int r = lane; r < nc; r += 32) {
        const int q = mgidx(C, r % C.nx + 1, (r / C.nx) % C.ny + 1, r / (C.nx * C.ny) + 1);
        C.x[q] = C.m[q] ? (float)y[r] : 0.f;
      }
    }
    grid.sync();
  }
  for (int l = M.L - 2; l >= 0; --l) {
    mg_prolong(M.lv[l], M.lv[l + 1], tid, T);
    grid.sync();
    mg_smooth(M.lv[l], 1, false, tid, T);
    grid.sync();
    mg_smooth(M.lv[l], 0, false, tid, T);
    grid.sync();
  }
}

// Pressure correction by MG-preconditioned CG (HYPRE PCG with a
// preconditioner: r = b, z = M r, p = z, gamma = <r,z>; s = A p,
// alpha = gamma/<s,p>, x += alpha p, r -= alpha s, z = M r, gamma' = <r,z>,
// stop on <r,r>/<b,b> < tol^2, p = z + beta p).  Assembly (coefficients, b)
// has been done by k_pcorr_setup.
__global__ void __launch_bounds__(kBlock) k_mgcg(FluidDev F, Prm P, MgView M, double *partials, DevStats *st) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[33];
  const int cx = F.cx, cy = F.cy, n = cx * cy * F.cz;
  const int PX = cx + 2, PXY = (cx + 2) * (cy + 2);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  int buf = 0;
  const MgLevel &L0 = M.lv[0];
  // r = b is in F.r, x = 0; bb
  double acc = 0.0;
  for (int c = tid; c < n; c += T) {
    if (F.empty[c]) continue;
    const int q = (c % cx + 1) + PX * ((c / cx) % cy + 1) + PXY * (c / (cx * cy) + 1);
    const double rv = F.r[q];
    acc += rv * rv;
    L0.rhs[q] = (float)rv;
  }
  const double bb = grid_sum(acc, partials, buf, sh, grid);
  if (bb == 0.0) {
    if (tid == 0) { st->pcg_iters = 0; st->pcg_relres = 0.0; st->cum_pcg_solves += 1; }
    return;
  }
  const double eps = P.pcg_tol * P.pcg_tol;
  mg_vcycle(M, grid, tid, T);
  acc = 0.0;
  for (int c = tid; c < n; c += T) {
    if (F.empty[c]) continue;
    const int q = (c % cx + 1) + PX * ((c / cx) % cy + 1) + PXY * (c / (cx * cy) + 1);
    const double z = (double)__ldcg(L0.x + q);
    F.pa[q] = z;
    acc += F.r[q] * z;
  }
  double gamma = grid_sum(acc, partials, buf, sh, grid), iprod = bb;
  int it = 0;
  while (it + 1 <= P.pcg_maxiter) {
    it++;
    acc = 0.0;
    for (int c = tid; c < n; c += T) {
      if (F.empty[c]) continue;
      const int q = (c % cx + 1) + PX * ((c / cx) % cy + 1) + PXY * (c / (cx * cy) + 1);
      const double *p = F.pa;
      const double ax = F.acx[q], ay = F.acy[q], az = F.acz[q], d = ax + ax + ay + ay + az + az;
      const double sv = d * ld(p + q) - az * ld(p + q - PXY) - ay * ld(p + q - PX) - ax * ld(p + q - 1) -
                        ax * ld(p + q + 1) - ay * ld(p + q + PX) - az * ld(p + q + PXY);
      F.s[q] = sv;
      acc += sv * ld(p + q);
    }
    const double sdotp = grid_sum(acc, partials, buf, sh, grid);
    if (sdotp == 0.0) break;
    const double alpha = gamma / sdotp, gamma_old = gamma;
    acc = 0.0;
    for (int c = tid; c < n; c += T) {
      if (F.empty[c]) continue;
      const int q = (c % cx + 1) + PX * ((c / cx) % cy + 1) + PXY * (c / (cx * cy) + 1);
      F.x[q] = F.x[q] + alpha * F.pa[q];
      const double rv = F.r[q] - alpha * F.s[q];
      F.r[q] = rv;
      acc += rv * rv;
      L0.rhs[q] = (float)rv;
    }
    iprod = grid_sum(acc, partials, buf, sh, grid);
    if (iprod / bb < eps) break;
    mg_vcycle(M, grid, tid, T);
    acc = 0.0;
    for (int c = tid; c < n; c += T) {
      if (F.empty[c]) continue;
      const int q = (c % cx + 1) + PX * ((c / cx) % cy + 1) + PXY * (c / (cx * cy) + 1);
      acc += F.r[q] * (double)__ldcg(L0.x + q);
    }
    gamma = grid_sum(acc, partials, buf, sh, grid);
    const double beta = gamma / gamma_old;
    for (int c = tid; c < n; c += T) {
      if (F.empty[c]) continue;
      const int q = (c % cx + 1) + PX * ((c / cx) % cy + 1) + PXY * (c / (cx * cy) + 1);
      F.pa[q] = (double)__ldcg(L0.x + q) + beta * F.pa[q];
    }
    grid.sync();
  }
  if (tid == 0) { st->pcg_iters = it; st->pcg_relres = sqrt(iprod / bb); st->cum_pcg_iters += it; st->cum_pcg_solves += 1; }
}

// Assembly of the pressure-correction system for the MG path: coefficients
// (when `assemble`), r = b, x = 0 (fluid_solver.h:1969-2002 / 2123-2162).
__global__ void k_pcorr_setup(FluidDev F, int assemble) {
  const int cx = F.cx, cy = F.cy, n = cx * cy * F.cz;
  const int PX = cx + 2, PXY = (cx + 2) * (cy + 2);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    if (F.empty[c]) continue;
    const int i = c % cx, j = (c / cx) % cy, k = c / (cx * cy);
    const int q = (i + 1) + PX * (j + 1) + PXY * (k + 1);
    if (assemble) {
      double xp = F.xp[i + 1], yp = F.yp[j + 1], zp = F.zp[k + 1];
      double facexy = xp * yp, facexz = xp * zp, faceyz = yp * zp;
      F.acx[q] = faceyz / F.up[IU(F, i + 1, j + 1, k + 1)];
      F.acy[q] = facexz / F.vp[IV(F, i + 1, j + 1, k + 1)];
      F.acz[q] = facexy / F.wp[IW(F, i + 1, j + 1, k + 1)];
    }
    F.r[q] = -(F.u[IU(F, i + 2, j + 1, k + 1)] - F.u[IU(F, i + 1, j + 1, k + 1)]) -
             (F.v[IV(F, i + 1, j + 2, k + 1)] - F.v[IV(F, i + 1, j + 1, k + 1)]) -
             (F.w[IW(F, i + 1, j + 1, k + 2)] - F.w[IW(F, i + 1, j + 1, k + 1)]);
    F.x[q] = 0.0;
  }
}

// Velocity correction, pressure update and p_temp refresh
// (fluid_solver.h:1460-1597); p' is the CG solution x.
__global__ void k_correct(FluidDev F, Prm P) {
  const int cx = F.cx, cy = F.cy, n = cx * cy * F.cz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    if (F.empty[c]) continue;
    const int i = c % cx, j = (c / cx) % cy, k = c / (cx * cy);
    const int I = i + 1, J = j + 1, K = k + 1;
    const double *pp = F.x;
    const double pc = pp[IP(F, I, J, K)];
    {
      double faceyz = F.yp[J] * F.zp[K];
      double ap = F.up[IU(F, I, J, K)];
      if (ap == 0) ap = 1e-10;
      double corr = (pp[IP(F, I - 1, J, K)] - pc) * faceyz / ap;
      double nv = F.u[IU(F, I, J, K)] + corr;
      F.ux[GX(F, i, j, k)] = nv; F.u[IU(F, I, J, K)] = nv;
    }
    {
      double facexz = F.xp[I] * F.zp[K];
      double ap = F.vp[IV(F, I, J, K)];
      if (ap == 0) ap = 1e-10;
      double corr = (pp[IP(F, I, J - 1, K)] - pc) * facexz / ap;
      double nv = F.v[IV(F, I, J, K)] + corr;
      F.uy[GY(F, i, j, k)] = nv; F.v[IV(F, I, J, K)] = nv;
    }
    {
      double facexy = F.xp[I] * F.yp[J];
      double ap = F.wp[IW(F, I, J, K)];
      if (ap == 0) ap = 1e-10;
      double corr = (pp[IP(F, I, J, K - 1)] - pc) * facexy / ap;
      double nv = F.w[IW(F, I, J, K)] + corr;
      F.uz[GZ(F, i, j, k)] = nv; F.w[IW(F, I, J, K)] = nv;
    }
    double np_ = F.pc[c] + P.relax * pc;
    F.pc[c] = np_;
    F.pt[IP(F, I, J, K)] = np_;
  }
}

// ---------------------------------------------------------------- cell boundary condition
// applyCellBoundaryCondition (fluid_solver.h:324-405) runs in place in k-j-i
// order: a boundary cell copies its inward neighbour, which is itself a
// boundary cell already updated in this pass when it comes earlier in that
// order.  Each thread follows that chain on the pre-pass values.
__device__ __forceinline__ int cell_src(const FluidDev &F, int i, int j, int k, int c) {
  const int gx = i + F.ox - 1, gy = j + F.oy - 1, gz = k + F.oz - 1;
  if (gx == 0) return c + 1;
  if (gx == F.Nx - 1) return c - 1;
  if (gy == 0) return c + F.cx;
  if (gy == F.Ny - 1) return c - F.cx;
  if (gz == 0) return c + F.cx * F.cy;
  if (gz == F.Nz - 1) return c - F.cx * F.cy;
  return -1;
}
__global__ void k_cellbc_resolve(FluidDev F) {
  const int cx = F.cx, cy = F.cy, n = cx * cy * F.cz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    int cur = c;
    int s = cell_src(F, c % cx, (c / cx) % cy, c / (cx * cy), c);
    if (s < 0) continue;
    for (int hop = 0; hop < 64; ++hop) {
      const int t = cell_src(F, s % cx, (s / cx) % cy, s / (cx * cy), s);
      if (s < cur && t >= 0) { cur = s; s = t; continue; }
      break;
    }
    F.pscr[c] = F.pc[s];
  }
}
// Commit the resolved values, write the ghost layers of p_temp, p(0,0,0) = 0,
// boundary t = 293.  With `after_step` (setForNext, fluid_solver.h:1638-1657)
// t is first refreshed from t_temp and p_temp's interior from p.
__global__ void k_cellbc_commit(FluidDev F, Prm P, int after_step) {
  const int cx = F.cx, cy = F.cy, cz = F.cz, n = cx * cy * cz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % cx, j = (c / cx) % cy, k = c / (cx * cy);
    const int gx = i + F.ox - 1, gy = j + F.oy - 1, gz = k + F.oz - 1;
    const bool bnd = cell_src(F, i, j, k, c) >= 0;
    const double v = bnd ? F.pscr[c] : F.pc[c];
    double *pt = F.pt;
    if (bnd) {
      pt[IP(F, i + 1, j + 1, k + 1)] = v;
      if (gx == 0) pt[IP(F, i, j + 1, k + 1)] = v;
      else if (gx == F.Nx - 1) pt[IP(F, i + 2, j + 1, k + 1)] = v;
      else if (gy == 0) pt[IP(F, i + 1, j, k + 1)] = v;
      else if (gy == F.Ny - 1) {
        pt[IP(F, i + 1, j + 2, k + 1)] = v;
        if (i + 1 == cx) pt[IP(F, i + 2, j + 2, k + 1)] = v;
        if (k + 1 == cz) pt[IP(F, i + 1, j + 2, k + 2)] = v;
        if (i + 1 == 1) pt[IP(F, i, j + 2, k + 1)] = v;
        if (k + 1 == 1) pt[IP(F, i + 1, j + 2, k)] = v;
        if (i + 1 == cx && k + 1 == cz) pt[IP(F, i + 2, j + 2, k + 2)] = v;
        if (i + 1 == 1 && k + 1 == 1) pt[IP(F, i, j + 2, k)] = v;
      } else if (gz == 0) pt[IP(F, i + 1, j + 1, k)] = v;
      else if (gz == F.Nz - 1) pt[IP(F, i + 1, j + 1, k + 2)] = v;
    }
    const double pfinal = (c == 0) ? 0.0 : v;
    F.pc[c] = pfinal;
    if (after_step) {
      pt[IP(F, i + 1, j + 1, k + 1)] = pfinal;
      F.tc[c] = bnd ? P.t_wall : F.tt[IP(F, i + 1, j + 1, k + 1)];
    } else if (bnd) {
      F.tc[c] = P.t_wall;
    }
  }
}

// Interface faces get u = u* = 0 in FluidSolver::init (fluid_solver.h:1005,1116,1225).
__global__ void k_zero_faces(const long long *pad_idx, const long long *face_idx, int n, double *star, double *out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    out[face_idx[e]] = 0.0;
    star[pad_idx[e]] = 0.0;
  }
}

// ---------------------------------------------------------------- host side
struct DeviceState {
  cudaStream_t stream = nullptr;
  int nsm = 0;
  FluidDev F{};
  Prm P{};
  std::vector<void *> allocs;
  double *partials = nullptr;
  DevStats *stats = nullptr;
  DevStats *stats_host = nullptr;
  // solids
  int nreg = 0, solid_blocks = 0, maxS = 0;
  SolidReg *regs = nullptr;
  int *blk_reg = nullptr;
  std::vector<SolidReg> regs_h;
  double *stt = nullptr, *stc = nullptr;
  uint8_t *sem = nullptr;
  long long ntt = 0, ntc = 0;
  // swap
  int nswap = 0;
  long long *f_send = nullptr, *f_recv = nullptr, *s_send = nullptr, *s_recv = nullptr;
  double *fbuf = nullptr, *sbuf = nullptr;
  // interface-face zeroing lists
  long long *ibu_pad = nullptr, *ibu_face = nullptr, *ibv_pad = nullptr, *ibv_face = nullptr, *ibw_pad = nullptr,
            *ibw_face = nullptr;
  int nibu = 0, nibv = 0, nibw = 0;
  // cooperative grid sizes
  int g_gs[4] = {0, 0, 0, 0}, g_pcorr = 0, tz = 16;
  // optional per-phase CUDA-event timing on the engine stream
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_used;
  cudaEvent_t ev_get() {
    if (ev_pool.empty()) {
      cudaEvent_t e;
      HS_CUDA(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = ev_pool.back();
    ev_pool.pop_back();
    return e;
  }
  double *snap = nullptr, *ssnap = nullptr;
  int *spred = nullptr;
  bool have_matrix = false;
  // multigrid hierarchy (HS_PSOLVE_MGCG)
  MgView mg{};
  int g_mgcg = 0;
  bool mg_ready = false;

  template <class T>
  T *alloc(size_t n) {
    void *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA alloc: ") + cudaGetErrorString(e));
    allocs.push_back(p);
    HS_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), stream));
    return (T *)p;
  }
  template <class T>
  T *upload(const std::vector<T> &h) {
    T *p = alloc<T>(h.size());
    if (!h.empty()) HS_CUDA(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return p;
  }
  ~DeviceState() {
    for (auto &u : ev_used) { cudaEventDestroy(u.second.first); cudaEventDestroy(u.second.second); }
    for (auto e : ev_pool) cudaEventDestroy(e);
    for (void *p : allocs) cudaFree(p);
    if (stats_host) cudaFreeHost(stats_host);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

template <class K>
int coop_blocks(K kernel, int nsm, int want) {
  int per = 0;
  HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kBlock, 0));
  int cap = per * nsm;
  if (cap < 1) throw std::runtime_error("cooperative kernel cannot be resident");
  return std::max(1, std::min(cap, want));
}

// z-depth of the CG tiles: balance tiles over the resident blocks and keep
// the two halo planes a small share of each tile
int choose_tz(long cx, long cy, long cz, int grid) {
  long ntxy = ((cx + kTX - 1) / kTX) * ((cy + kTY - 1) / kTY);
  double best = -1;
  int tz_best = 16;
  for (int tz = 4; tz <= 64; ++tz) {
    long nt = ntxy * ((cz + tz - 1) / tz);
    long rounds = (nt + grid - 1) / grid;
    double eff = (double)cz / ((double)rounds * grid / ntxy * tz) * (double)tz / (tz + 2);
    if (eff > best) { best = eff; tz_best = tz; }
  }
  return tz_best;
}

template <class K, class... A>
void coop_launch(K kernel, int blocks, cudaStream_t s, A... args) {
  void *argv[] = {(void *)&args...};
  HS_CUDA(cudaLaunchCooperativeKernel((void *)kernel, dim3(blocks), dim3(kBlock), argv, 0, s));
}

int grid_for(long n) { return (int)std::max<long>(1, std::min<long>((n + kBlock - 1) / kBlock, 148L * 16)); }

}  // namespace

Engine::Engine(const Case &c, const hs_params &p, int device) : case_(c), prm_(p), device_(device) {
  HS_CUDA(cudaSetDevice(device));
  d_.reset(new DeviceState());
  DeviceState &D = *d_;
  HS_CUDA(cudaStreamCreateWithFlags(&D.stream, cudaStreamNonBlocking));
  HS_CUDA(cudaDeviceGetAttribute(&D.nsm, cudaDevAttrMultiProcessorCount, device));
  int coop = 0;
  HS_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  if (!coop) throw std::runtime_error("device does not support cooperative launch");
  const Meta &M = c.fluid;
  if (M.nu() > (1L << 31) - 1 || M.npad() > (1L << 31) - 1) throw std::runtime_error("fluid box too large for 32-bit indexing");

  Prm &P = D.P;
  P.nu = p.nu; P.rho = p.rho; P.alpha = p.alpha; P.u_lid = p.u_lid; P.relax = p.relax; P.relax_solid = p.relax_solid;
  P.mom_tol = p.mom_tol; P.energy_tol = p.energy_tol; P.solid_tol = p.solid_tol; P.t_wall = p.t_wall;
  P.t_solid0 = p.t_solid0; P.pcg_tol = p.pcg_tol; P.gs_max = p.gs_max; P.pcg_maxiter = p.pcg_maxiter;

  FluidDev &F = D.F;
  F.cx = (int)M.cx; F.cy = (int)M.cy; F.cz = (int)M.cz; F.fx = (int)M.fx; F.fy = (int)M.fy; F.fz = (int)M.fz;
  F.ox = (int)M.ox; F.oy = (int)M.oy; F.oz = (int)M.oz;
  F.Nx = (int)c.Nx; F.Ny = (int)c.Ny; F.Nz = (int)c.Nz;
  F.u = D.alloc<double>(M.nu()); F.up = D.alloc<double>(M.nu());
  F.v = D.alloc<double>(M.nv()); F.vp = D.alloc<double>(M.nv());
  F.w = D.alloc<double>(M.nw()); F.wp = D.alloc<double>(M.nw());
  F.pt = D.alloc<double>(M.npad());
  F.tt = D.upload(std::vector<double>(M.npad(), p.t_fluid0));
  F.pc = D.alloc<double>(M.ncell()); F.tc = D.alloc<double>(M.ncell());
  F.ux = D.alloc<double>(M.fx * M.cy * M.cz); F.uy = D.alloc<double>(M.cx * M.fy * M.cz);
  F.uz = D.alloc<double>(M.cx * M.cy * M.fz);
  F.empty = D.upload(c.fluid_empty);
  F.xp = D.upload(c.xp); F.xw = D.upload(c.xw); F.xe = D.upload(c.xe);
  F.yp = D.upload(c.yp); F.ys = D.upload(c.ys); F.yn = D.upload(c.yn);
  F.zp = D.upload(c.zp); F.zf = D.upload(c.zf); F.zb = D.upload(c.zb);
  {
    auto inv2 = [](const std::vector<double> &p, const std::vector<double> &m) {
      std::vector<double> o(p.size(), 0.0);
      for (size_t i = 1; i + 1 < p.size(); ++i) {
        double sp = (p[i] + m[i]) / 2.0;
        o[i] = 1 / sp / sp;
      }
      return o;
    };
    F.ix2 = D.upload(inv2(c.xp, c.xw)); F.iy2 = D.upload(inv2(c.yp, c.ys)); F.iz2 = D.upload(inv2(c.zp, c.zf));
    auto rcp = [](const std::vector<double> &p, const std::vector<double> &m) {
      std::vector<double> o(p.size(), 0.0);
      for (size_t i = 1; i + 1 < p.size(); ++i) o[i] = 1.0 / ((p[i] + m[i]) / 2.0);
      return o;
    };
    F.rsx = D.upload(rcp(c.xp, c.xw)); F.rsy = D.upload(rcp(c.yp, c.ys)); F.rsz = D.upload(rcp(c.zp, c.zf));
    auto rsum = [](const std::vector<double> &p, const std::vector<double> &m) {
      std::vector<double> o(p.size(), 0.0);
      for (size_t i = 1; i + 1 < p.size(); ++i) o[i] = 1.0 / (p[i] + m[i]);
      return o;
    };
    F.rxw = D.upload(rsum(c.xp, c.xw)); F.rxe = D.upload(rsum(c.xp, c.xe));
    F.rys = D.upload(rsum(c.ys, c.yp)); F.ryn = D.upload(rsum(c.yn, c.yp));
    F.rzb = D.upload(rsum(c.zb, c.zp)); F.rzf = D.upload(rsum(c.zf, c.zp));
  }
  F.acx = D.alloc<double>(M.npad()); F.acy = D.alloc<double>(M.npad()); F.acz = D.alloc<double>(M.npad());
  F.x = D.alloc<double>(M.npad()); F.r = D.alloc<double>(M.npad()); F.pa = D.alloc<double>(M.npad());
  F.pb = D.alloc<double>(M.npad()); F.s = D.alloc<double>(M.npad());
  F.pscr = D.alloc<double>(M.ncell());
  F.hx = (int)((M.cx + 3) / 2);
  F.hs = (long long)F.hx * (M.cy + 2) * (M.cz + 2);
  F.ts = D.alloc<double>(2 * F.hs); F.us = D.alloc<double>(2 * F.hs);
  F.vs = D.alloc<double>(2 * F.hs); F.ws = D.alloc<double>(2 * F.hs);

  // solids: one contiguous buffer per quantity, per-region offsets
  D.nreg = (int)c.solids.size();
  if (D.nreg > kMaxRegions) throw std::runtime_error("more than 256 solid regions");
  std::vector<double> tt_h, tc_h;
  std::vector<uint8_t> em_h;
  D.regs_h.resize(D.nreg);
  long long want_blocks = 0;
  for (int r = 0; r < D.nreg; ++r) {
    const Meta &S = c.solids[r];
    SolidReg &R = D.regs_h[r];
    R.cx = (int)S.cx; R.cy = (int)S.cy; R.cz = (int)S.cz; R.rows = (int)(S.cy * S.cz);
    R.tt_off = (long long)tt_h.size(); R.tc_off = (long long)tc_h.size(); R.em_off = (long long)em_h.size();
    tt_h.insert(tt_h.end(), S.npad(), p.t_solid0);
    tc_h.insert(tc_h.end(), S.ncell(), 0.0);
    em_h.insert(em_h.end(), c.solid_empty[r].begin(), c.solid_empty[r].end());
    D.maxS = std::max<int>(D.maxS, (int)(S.cx + S.cy + S.cz - 2));
    want_blocks += (R.rows + 1) / 2;
  }
  D.ntt = (long long)tt_h.size(); D.ntc = (long long)tc_h.size();
  D.stt = D.upload(tt_h); D.stc = D.upload(tc_h); D.sem = D.upload(em_h);
  if (D.nreg) {
    int per = 0;
    HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_solid, kBlock, 0));
    long long cap = (long long)per * D.nsm;
    if (cap < D.nreg) throw std::runtime_error("too many solid regions for one cooperative launch");
    std::vector<int> blk_reg;
    int b0 = 0;
    for (int r = 0; r < D.nreg; ++r) {
      SolidReg &R = D.regs_h[r];
      long long wantr = (R.rows + 1) / 2;  // room for a 128-sweep window at 2 slots per thread
      long long nb = want_blocks <= cap ? wantr : std::max<long long>(1, wantr * (cap - D.nreg) / want_blocks);
      if (b0 + nb > cap) nb = 1;
      R.blk0 = b0; R.nblk = (int)nb;
      for (int q = 0; q < nb; ++q) blk_reg.push_back(r);
      b0 += (int)nb;
    }
    D.solid_blocks = b0;
    D.regs = D.upload(D.regs_h);
    D.blk_reg = D.upload(blk_reg);
  }
  // interface swap lists (solid indices made absolute into the joined buffer)
  D.nswap = (int)c.swap.size();
  {
    std::vector<long long> fs, fr, ss, sr;
    for (auto &sp : c.swap) {
      fs.push_back(sp.f_send); fr.push_back(sp.f_recv);
      ss.push_back(sp.s_send + D.regs_h[sp.region].tt_off); sr.push_back(sp.s_recv + D.regs_h[sp.region].tt_off);
    }
    D.f_send = D.upload(fs); D.f_recv = D.upload(fr); D.s_send = D.upload(ss); D.s_recv = D.upload(sr);
    D.fbuf = D.alloc<double>(D.nswap); D.sbuf = D.alloc<double>(D.nswap);
  }
  // interface faces to zero at init
  {
    std::vector<long long> up_, uf, vp_, vf, wp_, wf;
    for (long k = 0; k < M.cz; ++k)
      for (long j = 0; j < M.cy; ++j)
        for (long i = 0; i < M.fx; ++i)
          if (c.ib_x[i + j * M.fx + k * M.fx * M.cy]) {
            uf.push_back(i + j * M.fx + k * M.fx * M.cy);
            up_.push_back((i + 1) + (j + 1) * (M.fx + 2) + (k + 1) * (M.fx + 2) * (M.cy + 2));
          }
    for (long k = 0; k < M.cz; ++k)
      for (long j = 0; j < M.fy; ++j)
        for (long i = 0; i < M.cx; ++i)
          if (c.ib_y[i + j * M.cx + k * M.cx * M.fy]) {
            vf.push_back(i + j * M.cx + k * M.cx * M.fy);
            vp_.push_back((i + 1) + (j + 1) * (M.cx + 2) + (k + 1) * (M.cx + 2) * (M.fy + 2));
          }
    for (long k = 0; k < M.fz; ++k)
      for (long j = 0; j < M.cy; ++j)
        for (long i = 0; i < M.cx; ++i)
          if (c.ib_z[i + j * M.cx + k * M.cx * M.cy]) {
            wf.push_back(i + j * M.cx + k * M.cx * M.cy);
            wp_.push_back((i + 1) + (j + 1) * (M.cx + 2) + (k + 1) * (M.cx + 2) * (M.cy + 2));
          }
    D.nibu = (int)uf.size(); D.nibv = (int)vf.size(); D.nibw = (int)wf.size();
    D.ibu_pad = D.upload(up_); D.ibu_face = D.upload(uf); D.ibv_pad = D.upload(vp_); D.ibv_face = D.upload(vf);
    D.ibw_pad = D.upload(wp_); D.ibw_face = D.upload(wf);
  }
  // cooperative grid sizes
  {
    long rows[4] = {M.cy * M.cz, (M.fy - 1) * M.cz, M.cy * (M.fz - 1), M.cy * M.cz};
    D.g_gs[0] = coop_blocks(k_gs<0>, D.nsm, (int)std::min<long>((rows[0] + 1) / 2, 1 << 20));
    D.g_gs[1] = coop_blocks(k_gs<1>, D.nsm, (int)std::min<long>((rows[1] + 1) / 2, 1 << 20));
    D.g_gs[2] = coop_blocks(k_gs<2>, D.nsm, (int)std::min<long>((rows[2] + 1) / 2, 1 << 20));
    D.g_gs[3] = coop_blocks(k_gs<3>, D.nsm, (int)std::min<long>((rows[3] + 1) / 2, 1 << 20));
  }
  D.g_pcorr = coop_blocks(k_pcorr, D.nsm, 1 << 30);
  D.tz = choose_tz(M.cx, M.cy, M.cz, D.g_pcorr);
  D.snap = D.alloc<double>(std::max({M.nu(), M.nv(), M.nw(), M.npad(), 2 * (long)F.hs}));
  D.ssnap = D.alloc<double>(std::max<long long>(D.ntt, 1));
  D.spred = D.alloc<int>(std::max(D.nreg, 1));
  int gmax = std::max({D.g_gs[0], D.g_gs[1], D.g_gs[2], D.g_gs[3], D.g_pcorr, D.solid_blocks, 1});
  if (p.pressure_solver == HS_PSOLVE_MGCG) {
    MgView &G = D.mg;
    int nx = (int)M.cx, ny = (int)M.cy, nz = (int)M.cz;
    int L = 0;
    for (;;) {
      MgLevel &lv = G.lv[L];
      lv.nx = nx; lv.ny = ny; lv.nz = nz;
      size_t np = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
      lv.x = D.alloc<float>(np); lv.rhs = D.alloc<float>(np);
      lv.ax = D.alloc<float>(np); lv.ay = D.alloc<float>(np); lv.az = D.alloc<float>(np);
      lv.m = D.alloc<uint8_t>(np);
      ++L;
      if ((long)nx * ny * nz <= kMaxCoarse || L == kMaxLevels) break;
      nx = (nx + 1) / 2; ny = (ny + 1) / 2; nz = (nz + 1) / 2;
    }
    if ((long)G.lv[L - 1].nx * G.lv[L - 1].ny * G.lv[L - 1].nz > kMaxCoarse)
      throw std::runtime_error("multigrid hierarchy too deep for this grid");
    G.L = L;
    G.nc = G.lv[L - 1].nx * G.lv[L - 1].ny * G.lv[L - 1].nz;
    G.lu = D.alloc<double>((size_t)G.nc * G.nc);
    G.piv = D.alloc<int>(G.nc);
    G.yc = D.alloc<double>(G.nc);
    D.g_mgcg = coop_blocks(k_mgcg, D.nsm, 1 << 30);
    gmax = std::max(gmax, D.g_mgcg);
  }
  D.partials = D.alloc<double>(2 * (size_t)gmax * kBlock);
  D.stats = D.alloc<DevStats>(1);
  HS_CUDA(cudaMallocHost(&D.stats_host, sizeof(DevStats)));
  std::memset(D.stats_host, 0, sizeof(DevStats));
  HS_CUDA(cudaStreamSynchronize(D.stream));
}

Engine::~Engine() {
  if (d_) {
    cudaSetDevice(device_);
    cudaStreamSynchronize(d_->stream);
  }
}

void Engine::init() {
  HS_CUDA(cudaSetDevice(device_));
  DeviceState &D = *d_;
  cudaStream_t s = D.stream;
  long nplane = std::max({(D.F.cz + 2) * (D.F.cy + 2), (D.F.cz + 2) * (D.F.cx + 2), (D.F.cy + 2) * (D.F.cx + 2)});
  for (int which = 0; which < 3; ++which) k_bc<<<grid_for(nplane), kBlock, 0, s>>>(D.F, D.P, which);
  long n = (long)D.F.cx * D.F.cy * D.F.cz;
  k_cellbc_resolve<<<grid_for(n), kBlock, 0, s>>>(D.F);
  k_cellbc_commit<<<grid_for(n), kBlock, 0, s>>>(D.F, D.P, 0);
  if (D.nibu) k_zero_faces<<<grid_for(D.nibu), kBlock, 0, s>>>(D.ibu_pad, D.ibu_face, D.nibu, D.F.u, D.F.ux);
  if (D.nibv) k_zero_faces<<<grid_for(D.nibv), kBlock, 0, s>>>(D.ibv_pad, D.ibv_face, D.nibv, D.F.v, D.F.uy);
  if (D.nibw) k_zero_faces<<<grid_for(D.nibw), kBlock, 0, s>>>(D.ibw_pad, D.ibw_face, D.nibw, D.F.w, D.F.uz);
  // MobSolver::init: t = T1 (mobs_solver.h:118)
  if (D.ntc) {
    std::vector<double> t333(D.ntc, prm_.t_solid0);
    HS_CUDA(cudaMemcpyAsync(D.stc, t333.data(), D.ntc * sizeof(double), cudaMemcpyHostToDevice, s));
    HS_CUDA(cudaStreamSynchronize(s));
  }
  HS_CUDA(cudaGetLastError());
  inited_ = true;
}

void Engine::step(int nsteps) {
  HS_CUDA(cudaSetDevice(device_));
  if (!inited_) throw std::logic_error("hs_step before hs_init");
  DeviceState &D = *d_;
  cudaStream_t s = D.stream;
  const long n = (long)D.F.cx * D.F.cy * D.F.cz;
  const long nplane = std::max({(D.F.cz + 2) * (D.F.cy + 2), (D.F.cz + 2) * (D.F.cx + 2), (D.F.cy + 2) * (D.F.cx + 2)});
  struct Mark {
    DeviceState &D;
    int phase;
    cudaEvent_t a = nullptr;
    Mark(DeviceState &d, int ph) : D(d), phase(ph) {
      if (D.profiling) { a = D.ev_get(); HS_CUDA(cudaEventRecord(a, D.stream)); }
    }
    ~Mark() {
      if (a) {
        cudaEvent_t b = D.ev_get();
        cudaEventRecord(b, D.stream);
        D.ev_used.push_back({phase, {a, b}});
      }
    }
  };
  for (int it = 0; it < nsteps; ++it) {
    // FluidSolver::solve (fluid_solver.h:1401-1633)
    { Mark m(D, 0); coop_launch(k_gs<0>, D.g_gs[0], s, D.F, D.P, D.partials, D.stats, D.snap); }
    { Mark m(D, 1); coop_launch(k_gs<1>, D.g_gs[1], s, D.F, D.P, D.partials, D.stats, D.snap); }
    { Mark m(D, 2); coop_launch(k_gs<2>, D.g_gs[2], s, D.F, D.P, D.partials, D.stats, D.snap); }
    int assemble = (!D.have_matrix || !prm_.frozen_matrix) ? 1 : 0;
    if (prm_.pressure_solver == HS_PSOLVE_MGCG) {
      Mark m(D, 3);
      k_pcorr_setup<<<grid_for(n), kBlock, 0, s>>>(D.F, assemble);
      if (assemble) build_multigrid();
      coop_launch(k_mgcg, D.g_mgcg, s, D.F, D.P, D.mg, D.partials, D.stats);
    } else {
      Mark m(D, 3);
      coop_launch(k_pcorr, D.g_pcorr, s, D.F, D.P, D.partials, D.stats, assemble, D.tz);
    }
    D.have_matrix = true;
    {
      Mark m(D, 4);
      k_correct<<<grid_for(n), kBlock, 0, s>>>(D.F, D.P);
      HS_CUDA(cudaMemsetAsync(D.F.x, 0, sizeof(double) * (size_t)case_.fluid.npad(), s));
    }
    { Mark m(D, 5); coop_launch(k_gs<3>, D.g_gs[3], s, D.F, D.P, D.partials, D.stats, D.snap); }
    // MobSolver::solve for every region
    if (D.nreg) {
      Mark m(D, 6);
      coop_launch(k_solid, D.solid_blocks, s, (const SolidReg *)D.regs, D.nreg, (const int *)D.blk_reg, D.stt, D.stc,
                  (const uint8_t *)D.sem, D.P, D.partials, D.stats, D.ssnap, D.spred);
    }
    {
      Mark m(D, 7);
      // interface swap (solver.h:83-148)
      if (D.nswap) {
        k_swap_gather<<<grid_for(D.nswap), kBlock, 0, s>>>(D.f_send, D.s_send, D.nswap, D.F.tt, D.stt, D.fbuf, D.sbuf);
        k_swap_scatter<<<grid_for(D.nswap), kBlock, 0, s>>>(D.f_recv, D.s_recv, D.nswap, D.F.tt, D.stt, D.fbuf, D.sbuf);
      }
      // FluidSolver::setForNext (fluid_solver.h:1634-1682)
      for (int which = 0; which < 3; ++which) k_bc<<<grid_for(nplane), kBlock, 0, s>>>(D.F, D.P, which);
      k_cellbc_resolve<<<grid_for(n), kBlock, 0, s>>>(D.F);
      k_cellbc_commit<<<grid_for(n), kBlock, 0, s>>>(D.F, D.P, 1);
      // MobSolver::setForNext
      if (D.nreg) k_solid_setfornext<<<dim3(64, std::min(D.nreg, 64)), kBlock, 0, s>>>(D.regs, D.nreg, D.stt, D.stc, D.sem);
    }
    HS_CUDA(cudaGetLastError());
    steps_++;
  }
}

void Engine::profile(bool on) {
  HS_CUDA(cudaSetDevice(device_));
  d_->profiling = on;
}

int Engine::profile_read(double *ms, int nphase) {
  HS_CUDA(cudaSetDevice(device_));
  DeviceState &D = *d_;
  HS_CUDA(cudaStreamSynchronize(D.stream));
  for (int q = 0; q < nphase; ++q) ms[q] = 0.0;
  int count = 0;
  for (auto &u : D.ev_used) {
    float t = 0.f;
    HS_CUDA(cudaEventElapsedTime(&t, u.second.first, u.second.second));
    if (u.first < nphase) ms[u.first] += t;
    if (u.first == 0) ++count;
    D.ev_pool.push_back(u.second.first);
    D.ev_pool.push_back(u.second.second);
  }
  D.ev_used.clear();
  return count;
}

void Engine::counters(long long *out8) {
  DeviceState &D = *d_;
  HS_CUDA(cudaMemcpyAsync(D.stats_host, D.stats, sizeof(DevStats), cudaMemcpyDeviceToHost, D.stream));
  HS_CUDA(cudaStreamSynchronize(D.stream));
  const DevStats &h = *D.stats_host;
  out8[0] = h.cum_sweeps[0]; out8[1] = h.cum_sweeps[1]; out8[2] = h.cum_sweeps[2]; out8[3] = h.cum_sweeps[3];
  out8[4] = h.cum_solid_cell_sweeps; out8[5] = h.cum_pcg_iters; out8[6] = h.cum_pcg_solves; out8[7] = steps_;
}

void *Engine::stream_handle() { return (void *)d_->stream; }

// Coefficients of every level from the frozen FP64 matrix, then the dense
// FP64 LU (partial pivoting) of the coarsest level on the host.
void Engine::build_multigrid() {
  DeviceState &D = *d_;
  MgView &G = D.mg;
  cudaStream_t s = D.stream;
  const long n = (long)D.F.cx * D.F.cy * D.F.cz;
  k_mg_fine<<<grid_for(n), kBlock, 0, s>>>(D.F, G.lv[0]);
  for (int l = 0; l + 1 < G.L; ++l) {
    long nc = (long)G.lv[l + 1].nx * G.lv[l + 1].ny * G.lv[l + 1].nz;
    k_mg_coarsen<<<grid_for(nc), kBlock, 0, s>>>(G.lv[l], G.lv[l + 1]);
  }
  const MgLevel &C = G.lv[G.L - 1];
  const size_t np = (size_t)(C.nx + 2) * (C.ny + 2) * (C.nz + 2);
  std::vector<float> ax(np), ay(np), az(np);
  std::vector<uint8_t> m(np);
  HS_CUDA(cudaMemcpyAsync(ax.data(), C.ax, np * 4, cudaMemcpyDeviceToHost, s));
  HS_CUDA(cudaMemcpyAsync(ay.data(), C.ay, np * 4, cudaMemcpyDeviceToHost, s));
  HS_CUDA(cudaMemcpyAsync(az.data(), C.az, np * 4, cudaMemcpyDeviceToHost, s));
  HS_CUDA(cudaMemcpyAsync(m.data(), C.m, np, cudaMemcpyDeviceToHost, s));
  HS_CUDA(cudaStreamSynchronize(s));
  const int nc = G.nc;
  std::vector<double> A((size_t)nc * nc, 0.0);
  auto pid = [&](int i, int j, int k) { return (size_t)(i + 1) + (C.nx + 2) * ((j + 1) + (size_t)(C.ny + 2) * (k + 1)); };
  for (int r = 0; r < nc; ++r) {
    const int i = r % C.nx, j = (r / C.nx) % C.ny, k = r / (C.nx * C.ny);
    const size_t q = pid(i, j, k);
    if (!m[q]) { A[(size_t)r * nc + r] = 1.0; continue; }
    const double cxv = ax[q], cyv = ay[q], czv = az[q];
    A[(size_t)r * nc + r] = 2.0 * (cxv + cyv + czv);
    auto nb = [&](int ii, int jj, int kk, double cval) {
      if (ii < 0 || jj < 0 || kk < 0 || ii >= C.nx || jj >= C.ny || kk >= C.nz) return;
      if (!m[pid(ii, jj, kk)]) return;
      A[(size_t)r * nc + (ii + C.nx * (jj + C.ny * kk))] -= cval;
    };
    nb(i - 1, j, k, cxv); nb(i + 1, j, k, cxv); nb(i, j - 1, k, cyv); nb(i, j + 1, k, cyv);
    nb(i, j, k - 1, czv); nb(i, j, k + 1, czv);
  }
  std::vector<int> piv(nc);
  for (int r = 0; r < nc; ++r) piv[r] = r;
  for (int c = 0; c < nc; ++c) {  // Doolittle LU with row pivoting; piv maps row -> original row
    int best = c;
    for (int r = c + 1; r < nc; ++r)
      if (std::fabs(A[(size_t)r * nc + c]) > std::fabs(A[(size_t)best * nc + c])) best = r;
    if (A[(size_t)best * nc + c] == 0.0) throw std::runtime_error("singular coarsest multigrid matrix");
    if (best != c) {
      for (int k2 = 0; k2 < nc; ++k2) std::swap(A[(size_t)c * nc + k2], A[(size_t)best * nc + k2]);
      std::swap(piv[c], piv[best]);
    }
    for (int r = c + 1; r < nc; ++r) {
      const double f = A[(size_t)r * nc + c] / A[(size_t)c * nc + c];
      A[(size_t)r * nc + c] = f;
      for (int k2 = c + 1; k2 < nc; ++k2) A[(size_t)r * nc + k2] -= f * A[(size_t)c * nc + k2];
    }
  }
  HS_CUDA(cudaMemcpyAsync((void *)G.lu, A.data(), A.size() * 8, cudaMemcpyHostToDevice, s));
  HS_CUDA(cudaMemcpyAsync((void *)G.piv, piv.data(), piv.size() * 4, cudaMemcpyHostToDevice, s));
  HS_CUDA(cudaStreamSynchronize(s));
  D.mg_ready = true;
}

void Engine::sync() {
  HS_CUDA(cudaSetDevice(device_));
  HS_CUDA(cudaStreamSynchronize(d_->stream));
}

void Engine::stats(hs_stats *out) {
  DeviceState &D = *d_;
  HS_CUDA(cudaMemcpyAsync(D.stats_host, D.stats, sizeof(DevStats), cudaMemcpyDeviceToHost, D.stream));
  HS_CUDA(cudaStreamSynchronize(D.stream));
  const DevStats &h = *D.stats_host;
  out->sweeps_u = h.sweeps[0]; out->sweeps_v = h.sweeps[1]; out->sweeps_w = h.sweeps[2]; out->sweeps_t = h.sweeps[3];
  out->sweeps_solid_max = h.solid_sweeps_max; out->pcg_iters = h.pcg_iters;
  out->res_u = h.res[0]; out->res_v = h.res[1]; out->res_w = h.res[2]; out->res_t = h.res[3];
  out->pcg_relres = h.pcg_relres; out->steps = steps_;
}

namespace {
double *field_ptr(DeviceState &D, const Meta &M, int f, long *n) {
  FluidDev &F = D.F;
  switch (f) {
    case HS_F_U_STAR: *n = M.nu(); return F.u;
    case HS_F_V_STAR: *n = M.nv(); return F.v;
    case HS_F_W_STAR: *n = M.nw(); return F.w;
    case HS_F_P_TEMP: *n = M.npad(); return F.pt;
    case HS_F_T_TEMP: *n = M.npad(); return F.tt;
    case HS_F_UP: *n = M.nu(); return F.up;
    case HS_F_VP: *n = M.nv(); return F.vp;
    case HS_F_WP: *n = M.nw(); return F.wp;
    case HS_F_UX: *n = M.fx * M.cy * M.cz; return F.ux;
    case HS_F_UY: *n = M.cx * M.fy * M.cz; return F.uy;
    case HS_F_UZ: *n = M.cx * M.cy * M.fz; return F.uz;
    case HS_F_P: *n = M.ncell(); return F.pc;
    case HS_F_T: *n = M.ncell(); return F.tc;
    case HS_F_P_PRIME: *n = M.npad(); return F.x;
  }
  *n = -1;
  return nullptr;
}
}  // namespace

long Engine::field_size(int f) const {
  long n;
  field_ptr(*d_, case_.fluid, f, &n);
  return n;
}

double *Engine::field_device_ptr(int f, long *n) { return field_ptr(*d_, case_.fluid, f, n); }

void Engine::get_field(int f, double *host, long n) {
  HS_CUDA(cudaSetDevice(device_));
  long m;
  double *p = field_ptr(*d_, case_.fluid, f, &m);
  if (!p || m != n) throw std::invalid_argument("field id or size mismatch");
  HS_CUDA(cudaMemcpyAsync(host, p, sizeof(double) * n, cudaMemcpyDeviceToHost, d_->stream));
  HS_CUDA(cudaStreamSynchronize(d_->stream));
}

void Engine::set_field(int f, const double *host, long n) {
  HS_CUDA(cudaSetDevice(device_));
  long m;
  double *p = field_ptr(*d_, case_.fluid, f, &m);
  if (!p || m != n) throw std::invalid_argument("field id or size mismatch");
  HS_CUDA(cudaMemcpyAsync(p, host, sizeof(double) * n, cudaMemcpyHostToDevice, d_->stream));
  HS_CUDA(cudaStreamSynchronize(d_->stream));
}

void Engine::get_solid(int r, int which, double *host, long n) {
  HS_CUDA(cudaSetDevice(device_));
  DeviceState &D = *d_;
  if (r < 0 || r >= D.nreg) throw std::invalid_argument("solid region out of range");
  const Meta &S = case_.solids[r];
  const SolidReg &R = D.regs_h[r];
  long m = which == 0 ? S.npad() : S.ncell();
  if (n != m) throw std::invalid_argument("solid field size mismatch");
  const double *src = which == 0 ? D.stt + R.tt_off : D.stc + R.tc_off;
  HS_CUDA(cudaMemcpyAsync(host, src, sizeof(double) * n, cudaMemcpyDeviceToHost, D.stream));
  HS_CUDA(cudaStreamSynchronize(D.stream));
}

// ---------------------------------------------------------------- standalone CG
struct PcgWork {
  int device = 0, cx = 0, cy = 0, cz = 0, grid = 0, tz = 16;
  double *r = nullptr, *pa = nullptr, *pb = nullptr, *s = nullptr, *partials = nullptr, *relres = nullptr;
  int *iters = nullptr;
};

PcgWork *pcg_create(int nx, int ny, int nz, int device) {
  if (nx < 1 || ny < 1 || nz < 1) throw std::invalid_argument("grid dimensions must be positive");
  long long npad = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  if (npad > (1LL << 31) - 1) throw std::invalid_argument("grid too large for 32-bit indexing");
  HS_CUDA(cudaSetDevice(device));
  int nsm = 0;
  HS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  std::unique_ptr<PcgWork> w(new PcgWork());
  w->device = device; w->cx = nx; w->cy = ny; w->cz = nz;
  w->grid = coop_blocks(k_pcg, nsm, 1 << 30);
  w->tz = choose_tz(nx, ny, nz, w->grid);
  auto get = [](void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA alloc: ") + cudaGetErrorString(e));
  };
  try {
    get((void **)&w->r, npad * 8); get((void **)&w->pa, npad * 8); get((void **)&w->pb, npad * 8);
    get((void **)&w->s, npad * 8); get((void **)&w->partials, 2 * (size_t)w->grid * kBlock * 8);
    get((void **)&w->relres, 8); get((void **)&w->iters, 4);
  } catch (...) {
    pcg_destroy(w.release());
    throw;
  }
  return w.release();
}

void pcg_destroy(PcgWork *w) {
  if (!w) return;
  cudaSetDevice(w->device);
  for (void *p : {(void *)w->r, (void *)w->pa, (void *)w->pb, (void *)w->s, (void *)w->partials, (void *)w->relres,
                  (void *)w->iters})
    if (p) cudaFree(p);
  delete w;
}

void pcg_solve(PcgWork *w, const double *acx, const double *acy, const double *acz, const double *b, double *x,
               double tol, int maxiter, void *stream, int *iters, double *relres) {
  if (!acx || !acy || !acz || !b || !x) throw std::invalid_argument("null device pointer");
  if (maxiter < 0 || !(tol >= 0)) throw std::invalid_argument("invalid tolerance or iteration limit");
  HS_CUDA(cudaSetDevice(w->device));
  cudaStream_t st = (cudaStream_t)stream;
  CgView V{w->cx, w->cy, w->cz, acx, acy, acz, x, w->r, w->pa, w->pb, w->s};
  coop_launch(k_pcg, w->grid, st, V, b, tol, maxiter, w->partials, w->tz, w->iters, w->relres);
  int it = 0;
  double rr = 0;
  HS_CUDA(cudaMemcpyAsync(&it, w->iters, sizeof(int), cudaMemcpyDeviceToHost, st));
  HS_CUDA(cudaMemcpyAsync(&rr, w->relres, sizeof(double), cudaMemcpyDeviceToHost, st));
  HS_CUDA(cudaStreamSynchronize(st));
  if (iters) *iters = it;
  if (relres) *relres = rr;
}

// ---------------------------------------------------------------- allocation-free CG
// Some callers cannot allocate device memory while they run: hosts whose whole
// GPU memory is owned by their own arena (a coupled multiphysics code that
// reserves HBM at start-up and hands each component a fixed budget), and
// loops that must not call cudaMalloc/cudaFree after set-up because those
// calls may synchronise the device and stall work queued on other streams.
// pcg_solve_noalloc serves them: the same CG kernel as pcg_solve, with its
// scratch (four padded vectors, the reduction partials and the two result
// words) in this file-scope array.  It is part of the library's device code,
// which the runtime loads on a device at the library's first use there (lazy
// loading: the first call of this function does it when no other kernel of
// the library has run on that device), and every GPU that loaded it holds it
// until the process exits (8.06 MiB per device).  The address looked up below
// is kept per device for the life of the process, so a cudaDeviceReset in
// between is not supported.  Every call shares the array: calls that overlap
// on the GPU race, so a caller issuing from several streams or threads must
// serialise them.
constexpr long long kNoAllocMaxPad = 1LL << 18;  // padded cells (nx+2)(ny+2)(nz+2)
constexpr int kNoAllocMaxBlocks = 4096;           // cooperative grid limit for the partials
constexpr long long kNoAllocDoubles = 4 * kNoAllocMaxPad + 2 * kNoAllocMaxBlocks + 2;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

namespace {
// Device address of g_noalloc_scratch and the cooperative grid, resolved once
// per device with that device current (the host-side name of a __device__
// array is not a device address).
struct NoAllocSetup {
  double *base = nullptr;
  int grid = 0, nsm = 0;
};
std::mutex g_noalloc_mu;
NoAllocSetup g_noalloc_dev[64];

NoAllocSetup noalloc_setup(int device) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (device < 0 || device >= 64) throw std::invalid_argument("device ordinal out of range");
  NoAllocSetup &S = g_noalloc_dev[device];
  if (!S.base) {
    void *ptr = nullptr;
    HS_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    HS_CUDA(cudaDeviceGetAttribute(&S.nsm, cudaDevAttrMultiProcessorCount, device));
    S.grid = coop_blocks(k_pcg, S.nsm, kNoAllocMaxBlocks);
    S.base = (double *)ptr;
  }
  return S;
}
}  // namespace

long long noalloc_max_padded_cells() { return kNoAllocMaxPad; }

void pcg_solve_noalloc(int nx, int ny, int nz, const double *acx, const double *acy, const double *acz, const double *b,
                       double *x, double tol, int maxiter, void *stream, int *iters, double *relres) {
  if (nx < 1 || ny < 1 || nz < 1) throw std::invalid_argument("grid dimensions must be positive");
  const long long npad = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  if (npad > kNoAllocMaxPad)
    throw std::invalid_argument("grid too large for the allocation-free solve: (nx+2)(ny+2)(nz+2) = " +
                                std::to_string(npad) + " padded cells, the static scratch holds " +
                                std::to_string(kNoAllocMaxPad));
  if (!acx || !acy || !acz || !b || !x) throw std::invalid_argument("null device pointer");
  if (maxiter < 0 || !(tol >= 0)) throw std::invalid_argument("invalid tolerance or iteration limit");
  int device = 0;
  HS_CUDA(cudaGetDevice(&device));
  const NoAllocSetup S = noalloc_setup(device);
  double *base = S.base;
  double *r = base, *pa = base + kNoAllocMaxPad, *pb = base + 2 * kNoAllocMaxPad, *sv = base + 3 * kNoAllocMaxPad;
  double *partials = base + 4 * kNoAllocMaxPad;
  double *out_rel = partials + 2 * kNoAllocMaxBlocks;
  int *out_it = reinterpret_cast<int *>(out_rel + 1);
  cudaStream_t st = (cudaStream_t)stream;
  CgView V{nx, ny, nz, acx, acy, acz, x, r, pa, pb, sv};
  // k_pcg writes every scratch word it later reads (r, p, s over the padded
  // grid, each partial before its reduction, both results), so the previous
  // call's contents never leak into this one
  coop_launch(k_pcg, S.grid, st, V, b, tol, maxiter, partials, choose_tz(nx, ny, nz, S.grid), out_it, out_rel);
  int it = 0;
  double rr = 0;
  HS_CUDA(cudaMemcpyAsync(&it, out_it, sizeof(int), cudaMemcpyDeviceToHost, st));
  HS_CUDA(cudaMemcpyAsync(&rr, out_rel, sizeof(double), cudaMemcpyDeviceToHost, st));
  HS_CUDA(cudaStreamSynchronize(st));
  if (iters) *iters = it;
  if (relres) *relres = rr;
}

// Check of div_pre against the IEEE quotient over caller arrays: out[i] = 1
// where div_pre(a[i], b[i], RN(1/b[i])) differs from a[i]/b[i] in any bit.
__global__ void k_div_check(const double *a, const double *b, long long n, unsigned char *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double y = 1.0 / b[i];
    const double q1 = div_pre(a[i], b[i], y), q2 = a[i] / b[i];
    out[i] = __double_as_longlong(q1) != __double_as_longlong(q2);
  }
}

long long div_check(const double *a, const double *b, long long n) {
  unsigned char *out = nullptr;
  double *da = nullptr, *db = nullptr;
  HS_CUDA(cudaMalloc(&da, n * 8));
  HS_CUDA(cudaMalloc(&db, n * 8));
  HS_CUDA(cudaMalloc(&out, n));
  HS_CUDA(cudaMemcpy(da, a, n * 8, cudaMemcpyHostToDevice));
  HS_CUDA(cudaMemcpy(db, b, n * 8, cudaMemcpyHostToDevice));
  k_div_check<<<1024, 256>>>(da, db, n, out);
  std::vector<unsigned char> h(n);
  HS_CUDA(cudaMemcpy(h.data(), out, n, cudaMemcpyDeviceToHost));
  cudaFree(da); cudaFree(db); cudaFree(out);
  long long bad = 0;
  for (auto v : h) bad += v;
  return bad;
}

}  // namespace hs
