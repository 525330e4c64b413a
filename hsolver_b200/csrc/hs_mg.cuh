// Geometric multigrid V-cycle for 7-point finite-volume operators on padded
// cell grids, used as the preconditioner of the pressure-correction CG
// (hs_channel.cu) and of the energy BiCGStab (hs_cht.cu).  Device code only;
// every function runs inside a cooperative kernel.
//
// Operator.  Each cell q stores the data of its low face on every axis:
// conductance g and flux f through it in the + direction (no convection when
// the flux arrays are null).  The ghost cell past the high end of an axis
// carries that boundary face; ghost values of x are 0, which is the
// homogeneous form of every boundary condition the solvers use.  Row P:
//   A:   sum_faces (g + max(f_out, 0)) x_P - (g + max(-f_out, 0)) x_N
//   A^T: same diagonal, off-diagonals with the upwind side swapped.
// Cells with m = 0 (masked) are not unknowns: x stays 0 there.
//
// Hierarchy: 2x coarsening per axis (ceil); a coarse cell is an unknown when
// any child is; coarse face g = (sum of the 2x2 fine g) / 2 (the patch area is
// 4x, the spacing 2x), coarse flux = sum of the fine fluxes (conservative);
// down to <= kMgCoarse cells, where an LU with partial pivoting (FP64, on the
// GPU) solves exactly.  Smoother: red-black Gauss-Seidel, one sweep before
// (red, black) and one after (black, red); the first red half-sweep (from
// x = 0) is applied by whoever writes the level's rhs, the prolongation is
// fused into the first post-smoothing half-sweep.  Levels below kMgSmall cells run inside
// block 0 alone, separated by __syncthreads instead of grid barriers.
#pragma once
#include <cooperative_groups.h>
#include <cstdint>

namespace hs {
namespace mg {

namespace cg = cooperative_groups;

constexpr int kMgMaxLv = 16;
constexpr int kMgCoarse = 64;
constexpr long long kMgSmall = 2048;

template <class M>
struct Level {
  int nx, ny, nz;
  M *x, *rhs;
  M *gx, *gy, *gz;
  M *fx, *fy, *fz;  // null: pure diffusion
  uint8_t *m;       // null: every interior cell is an unknown
};

template <class M>
struct Hier {
  int L;
  Level<M> lv[kMgMaxLv];
  double *lu;  // kMgCoarse^2
  int *piv;    // kMgCoarse
  double *y;   // kMgCoarse
};

template <class M>
__device__ __forceinline__ int idx(const Level<M> &L, int i, int j, int k) {
  return i + (L.nx + 2) * (j + (L.ny + 2) * k);
}

template <class M>
__device__ __forceinline__ M pos(M a) { return a > M(0) ? a : M(0); }

// diagonal and the six off-diagonal magnitudes of row q (order W E S N B F)
template <class M>
__device__ __forceinline__ void row(const Level<M> &L, int q, bool tr, M &d, M (&o)[6]) {
  const int PX = L.nx + 2, PXY = (L.nx + 2) * (L.ny + 2);
  const int st[3] = {1, PX, PXY};
  const M *g[3] = {L.gx, L.gy, L.gz};
  const M *f[3] = {L.fx, L.fy, L.fz};
  d = M(0);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const M gl = g[a][q], gh = g[a][q + st[a]];
    if (f[a]) {
      const M fl = f[a][q], fh = f[a][q + st[a]];  // + direction fluxes of the low and high face
      d += gl + pos(-fl) + gh + pos(fh);
      o[2 * a] = gl + (tr ? pos(-fl) : pos(fl));
      o[2 * a + 1] = gh + (tr ? pos(fh) : pos(-fh));
    } else {
      d += gl + gh;
      o[2 * a] = gl;
      o[2 * a + 1] = gh;
    }
  }
}

template <class M>
__device__ __forceinline__ M offsum(const Level<M> &L, const M (&o)[6], const M *x, int q) {
  const int PX = L.nx + 2, PXY = (L.nx + 2) * (L.ny + 2);
  return o[0] * __ldcg(x + q - 1) + o[1] * __ldcg(x + q + 1) + o[2] * __ldcg(x + q - PX) + o[3] * __ldcg(x + q + PX) +
         o[4] * __ldcg(x + q - PXY) + o[5] * __ldcg(x + q + PXY);
}

template <class M>
__device__ __forceinline__ bool unknown(const Level<M> &L, int q) { return L.m ? L.m[q] != 0 : true; }

// coarse level C from fine level F (every padded cell of C that holds a face)
template <class M>
__device__ void coarsen(const Level<M> &F, const Level<M> &C, int tid, int T) {
  const int n = (C.nx + 1) * (C.ny + 1) * (C.nz + 1);
  const bool conv = F.fx != nullptr;
  for (int e = tid; e < n; e += T) {
    const int row_ = e / (C.nx + 1), I = e - row_ * (C.nx + 1);
    const int K = row_ / (C.ny + 1), J = row_ - K * (C.ny + 1);
    const int qc = idx(C, I + 1, J + 1, K + 1);
    if (J < C.ny && K < C.nz) {
      const int fi = min(2 * I, F.nx);
      M sg = M(0), sf = M(0);
      for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj) {
          const int j = 2 * J + dj, k = 2 * K + dk;
          if (j < F.ny && k < F.nz) {
            const int q = idx(F, fi + 1, j + 1, k + 1);
            sg += F.gx[q];
            if (conv) sf += F.fx[q];
          }
        }
      C.gx[qc] = M(0.5) * sg;
      if (conv) C.fx[qc] = sf;
    }
    if (I < C.nx && K < C.nz) {
      const int fj = min(2 * J, F.ny);
      M sg = M(0), sf = M(0);
      for (int dk = 0; dk < 2; ++dk)
        for (int di = 0; di < 2; ++di) {
          const int i = 2 * I + di, k = 2 * K + dk;
          if (i < F.nx && k < F.nz) {
            const int q = idx(F, i + 1, fj + 1, k + 1);
            sg += F.gy[q];
            if (conv) sf += F.fy[q];
          }
        }
      C.gy[qc] = M(0.5) * sg;
      if (conv) C.fy[qc] = sf;
    }
    if (I < C.nx && J < C.ny) {
      const int fk = min(2 * K, F.nz);
      M sg = M(0), sf = M(0);
      for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
          const int i = 2 * I + di, j = 2 * J + dj;
          if (i < F.nx && j < F.ny) {
            const int q = idx(F, i + 1, j + 1, fk + 1);
            sg += F.gz[q];
            if (conv) sf += F.fz[q];
          }
        }
      C.gz[qc] = M(0.5) * sg;
      if (conv) C.fz[qc] = sf;
    }
    if (C.m && I < C.nx && J < C.ny && K < C.nz) {
      uint8_t any = 0;
      for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
          for (int di = 0; di < 2; ++di) {
            const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
            if (i < F.nx && j < F.ny && k < F.nz && F.m[idx(F, i + 1, j + 1, k + 1)]) any = 1;
          }
      C.m[qc] = any;
    }
  }
}

// a masked cell has zero couplings on every face (its faces touch a
// non-unknown), so d == 0 identifies it without reading the mask
template <class M>
__device__ void smooth(const Level<M> &L, int color, bool tr, int tid, int T) {
  const int half = (L.nx + 1) / 2;
  const int n = half * L.ny * L.nz;
  for (int e = tid; e < n; e += T) {
    const int row_ = e / half, m = e - row_ * half;
    const int k = row_ / L.ny, j = row_ - k * L.ny;
    const int i = 2 * m + ((j + k + color) & 1);
    if (i >= L.nx) continue;
    const int q = idx(L, i + 1, j + 1, k + 1);
    M d, o[6];
    row(L, q, tr, d, o);
    if (d == M(0)) { L.x[q] = M(0); continue; }
    M s = L.rhs[q];
    s += offsum(L, o, L.x, q);
    L.x[q] = s / d;
  }
}

// The last colour-0 half-sweep of level 0, also accumulating sum r x over
// every cell (colour 0 as it is computed, colour 1 as left by the previous
// half-sweep): the V-cycle's output dotted with the caller's residual r
// (padded, any precision; FP64 sums) without a pass of its own.
template <class M, class RT>
__device__ void smooth_dot(const Level<M> &L, bool tr, const RT *r, double &acc, int tid, int T) {
  const int half = (L.nx + 1) / 2;
  const int n = half * L.ny * L.nz;
  for (int e = tid; e < n; e += T) {
    const int row_ = e / half, m = e - row_ * half;
    const int k = row_ / L.ny, j = row_ - k * L.ny;
    const int i = 2 * m + ((j + k) & 1), ib = 2 * m + ((j + k + 1) & 1);
    if (i < L.nx) {
      const int q = idx(L, i + 1, j + 1, k + 1);
      M d, o[6];
      row(L, q, tr, d, o);
      M xv = M(0);
      if (d != M(0)) {
        M s = L.rhs[q];
        s += offsum(L, o, L.x, q);
        xv = s / d;
      }
      L.x[q] = xv;
      acc += (double)r[q] * (double)xv;
    }
    if (ib < L.nx) {
      const int q = idx(L, ib + 1, j + 1, k + 1);
      acc += (double)r[q] * (double)__ldcg(L.x + q);
    }
  }
}

// The first pre-smoothing half-sweep starts from x = 0, so on the colour-0
// cells it is local, x = rhs / d: whoever writes a level's rhs applies it to
// the cell in the same pass (the restriction for the coarse levels, the
// Krylov solver for level 0), which saves that half-sweep and its barrier.
template <class M>
__device__ __forceinline__ void seed(const Level<M> &L, int q, int i, int j, int k, M rhs, bool tr) {
  if ((i + j + k) & 1) return;
  M d, o[6];
  row(L, q, tr, d, o);
  L.x[q] = d == M(0) ? M(0) : rhs / d;
}

// coarse rhs = sum over the children of (rhs - A x), and the coarse seed.  It follows the
// colour-1 half-sweep, after which a colour-1 cell's residual is zero up to
// rounding (its update solved its own row), so only the colour-0 children
// are evaluated.
template <class M>
__device__ void restrict_res(const Level<M> &F, const Level<M> &C, bool tr, int tid, int T) {
  const int n = C.nx * C.ny * C.nz;
  for (int e = tid; e < n; e += T) {
    const int row_ = e / C.nx, I = e - row_ * C.nx;
    const int K = row_ / C.ny, J = row_ - K * C.ny;
    M acc = M(0);
    for (int dk = 0; dk < 2; ++dk)
      for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
          const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
          if (i >= F.nx || j >= F.ny || k >= F.nz || ((i + j + k) & 1)) continue;
          const int q = idx(F, i + 1, j + 1, k + 1);
          M d, o[6];
          row(F, q, tr, d, o);
          acc += F.rhs[q] - (d * __ldcg(F.x + q) - offsum(F, o, F.x, q));
        }
    const int qc = idx(C, I + 1, J + 1, K + 1);
    const M v = unknown(C, qc) ? acc : M(0);
    C.rhs[qc] = v;
    seed(C, qc, I, J, K, v, tr);
  }
}

// Prolongation fused into the first post-smoothing half-sweep (colour 1):
// every neighbour (colour 0) is read as x + x_coarse(parent).  A Gauss-Seidel
// update never reads its own cell, so the colour-0 cells' prolonged values
// are needed only as these neighbour values (the colour-0 half-sweep that
// follows recomputes them) and the colour-1 cells' not at all.  Ghost
// neighbours are 0, as they are never prolonged; a masked neighbour has a
// zero coupling.  The arithmetic is that of prolongation followed by smooth().
template <class M>
__device__ void prolong_smooth(const Level<M> &F, const Level<M> &C, bool tr, int tid, int T) {
  const int half = (F.nx + 1) / 2;
  const int n = half * F.ny * F.nz;
  const int PX = F.nx + 2, PXY = (F.nx + 2) * (F.ny + 2);
  for (int e = tid; e < n; e += T) {
    const int row_ = e / half, m = e - row_ * half;
    const int k = row_ / F.ny, j = row_ - k * F.ny;
    const int i = 2 * m + ((j + k + 1) & 1);
    if (i >= F.nx) continue;
    const int q = idx(F, i + 1, j + 1, k + 1);
    M d, o[6];
    row(F, q, tr, d, o);
    if (d == M(0)) { F.x[q] = M(0); continue; }
    auto xp = [&](int ii, int jj, int kk, int qq) -> M {
      if (ii < 0 || jj < 0 || kk < 0 || ii >= F.nx || jj >= F.ny || kk >= F.nz) return M(0);
      return __ldcg(F.x + qq) + __ldcg(C.x + idx(C, ii / 2 + 1, jj / 2 + 1, kk / 2 + 1));
    };
    const M off = o[0] * xp(i - 1, j, k, q - 1) + o[1] * xp(i + 1, j, k, q + 1) + o[2] * xp(i, j - 1, k, q - PX) +
                  o[3] * xp(i, j + 1, k, q + PX) + o[4] * xp(i, j, k - 1, q - PXY) + o[5] * xp(i, j, k + 1, q + PXY);
    M s = F.rhs[q];
    s += off;
    F.x[q] = s / d;
  }
}

// LU with partial pivoting of the coarsest operator (A or A^T), by block 0,
// in shared memory; the pivot is the largest |a| in the column, the lowest
// row among equals; the factors are copied to G.lu for coarse_solve
template <class M>
__device__ void factor(const Hier<M> &G, bool tr) {
  if (blockIdx.x != 0) return;
  __shared__ double a[kMgCoarse * kMgCoarse];
  __shared__ int spiv;
  const Level<M> &C = G.lv[G.L - 1];
  const int nc = C.nx * C.ny * C.nz, PX = C.nx + 2, PXY = (C.nx + 2) * (C.ny + 2);
  for (int e = threadIdx.x; e < nc * nc; e += blockDim.x) {
    const int r = e / nc, c2 = e % nc;
    const int q = idx(C, r % C.nx + 1, (r / C.nx) % C.ny + 1, r / (C.nx * C.ny) + 1);
    double v = 0.0;
    if (!unknown(C, q)) {
      v = r == c2 ? 1.0 : 0.0;
    } else {
      M d, o[6];
      row(C, q, tr, d, o);
      if (r == c2) {
        v = (double)d;
        if (v == 0.0) v = 1.0;
      } else {
        const int qc = idx(C, c2 % C.nx + 1, (c2 / C.nx) % C.ny + 1, c2 / (C.nx * C.ny) + 1);
        if (unknown(C, qc)) {
          const int off[6] = {-1, 1, -PX, PX, -PXY, PXY};
          for (int s = 0; s < 6; ++s)
            if (qc == q + off[s]) v = -(double)o[s];
        }
      }
    }
    a[e] = v;
  }
  __syncthreads();
  for (int col = 0; col < nc; ++col) {
    if (threadIdx.x < 32) {
      double bv = -1.0;
      int br = nc;
      for (int r = col + threadIdx.x; r < nc; r += 32) {
        const double v = fabs(a[r * nc + col]);
        if (v > bv || (v == bv && r < br)) { bv = v; br = r; }
      }
      for (int o = 16; o; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int orow = __shfl_xor_sync(0xffffffffu, br, o);
        if (ov > bv || (ov == bv && orow < br)) { bv = ov; br = orow; }
      }
      if (threadIdx.x == 0) { spiv = br; G.piv[col] = br; }
    }
    __syncthreads();
    const int pr = spiv;
    if (pr != col)
      for (int c2 = threadIdx.x; c2 < nc; c2 += blockDim.x) {
        const double t = a[col * nc + c2];
        a[col * nc + c2] = a[pr * nc + c2];
        a[pr * nc + c2] = t;
      }
    __syncthreads();
    const double piv = a[col * nc + col];
    for (int r = col + 1 + threadIdx.x; r < nc; r += blockDim.x) a[r * nc + col] /= piv;
    __syncthreads();
    const int rem = nc - col - 1;
    for (int e = threadIdx.x; e < rem * rem; e += blockDim.x) {
      const int r = col + 1 + e / rem, c2 = col + 1 + e % rem;
      a[r * nc + c2] -= a[r * nc + col] * a[col * nc + c2];
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nc * nc; e += blockDim.x) G.lu[e] = a[e];
}

// exact solve on the coarsest level, by warp 0 of block 0 (the permuted
// right-hand side in shared memory, triangular solves with warp dot products)
template <class M>
__device__ void coarse_solve(const Hier<M> &G) {
  if (threadIdx.x >= 32) return;
  __shared__ double y[kMgCoarse];
  const Level<M> &C = G.lv[G.L - 1];
  const int nc = C.nx * C.ny * C.nz, lane = threadIdx.x;
  if (lane == 0) {
    for (int r = 0; r < nc; ++r) y[r] = (double)C.rhs[idx(C, r % C.nx + 1, (r / C.nx) % C.ny + 1, r / (C.nx * C.ny) + 1)];
    for (int c2 = 0; c2 < nc; ++c2) {
      const int pr = G.piv[c2];
      if (pr != c2) { const double t = y[c2]; y[c2] = y[pr]; y[pr] = t; }
    }
  }
  __syncwarp();
  for (int r = 0; r < nc; ++r) {
    double a = 0.0;
    for (int c2 = lane; c2 < r; c2 += 32) a += G.lu[r * nc + c2] * y[c2];
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) y[r] -= a;
    __syncwarp();
  }
  for (int r = nc - 1; r >= 0; --r) {
    double a = 0.0;
    for (int c2 = r + 1 + lane; c2 < nc; c2 += 32) a += G.lu[r * nc + c2] * y[c2];
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) y[r] = (y[r] - a) / G.lu[r * nc + r];
    __syncwarp();
  }
  for (int r = lane; r < nc; r += 32) {
    const int q = idx(C, r % C.nx + 1, (r / C.nx) % C.ny + 1, r / (C.nx * C.ny) + 1);
    C.x[q] = unknown(C, q) ? (M)y[r] : M(0);
  }
}

template <class M>
__device__ __forceinline__ bool small(const Level<M> &L) { return (long long)L.nx * L.ny * L.nz <= kMgSmall; }

// build levels 1.. from level 0 and factor the coarsest (the caller filled level 0)
template <class M>
__device__ void build(const Hier<M> &G, bool tr, cg::grid_group &grid, int tid, int T) {
  for (int l = 0; l + 1 < G.L; ++l) {
    if (small(G.lv[l + 1]) && blockIdx.x != 0) break;
    if (small(G.lv[l + 1])) {
      coarsen(G.lv[l], G.lv[l + 1], threadIdx.x, blockDim.x);
      __syncthreads();
    } else {
      coarsen(G.lv[l], G.lv[l + 1], tid, T);
      grid.sync();
    }
  }
  factor(G, tr);
  grid.sync();
}

// lv[0].x = V-cycle applied to lv[0].rhs; the caller has written lv[0].rhs
// and seeded lv[0] (seed() on every interior cell) before the barrier that
// precedes this call.  With dot_r, the last level-0 pass also adds this
// thread's share of sum dot_r x to *dot_acc and the final barrier is left to
// the caller's reduction (returns true); it returns false, with the barrier
// done and nothing added, when level 0 is handled by block 0 alone.
template <class M, class RT = double>
__device__ bool vcycle(const Hier<M> &G, bool tr, cg::grid_group &grid, int tid, int T,
                       const RT *dot_r = nullptr, double *dot_acc = nullptr) {
  int ls = 0;  // first level handled by block 0 alone
  while (ls < G.L - 1 && !small(G.lv[ls])) ++ls;
  for (int l = 0; l < ls; ++l) {
    smooth(G.lv[l], 1, tr, tid, T);
    grid.sync();
    restrict_res(G.lv[l], G.lv[l + 1], tr, tid, T);
    grid.sync();
  }
  if (blockIdx.x == 0) {
    const int t = threadIdx.x, B = blockDim.x;
    for (int l = ls; l < G.L - 1; ++l) {
      smooth(G.lv[l], 1, tr, t, B);
      __syncthreads();
      restrict_res(G.lv[l], G.lv[l + 1], tr, t, B);
      __syncthreads();
    }
    coarse_solve(G);
    __syncthreads();
    for (int l = G.L - 2; l >= ls; --l) {
      prolong_smooth(G.lv[l], G.lv[l + 1], tr, t, B);
      __syncthreads();
      smooth(G.lv[l], 0, tr, t, B);
      __syncthreads();
    }
  }
  grid.sync();
  for (int l = ls - 1; l >= 0; --l) {
    prolong_smooth(G.lv[l], G.lv[l + 1], tr, tid, T);
    grid.sync();
    if (l == 0 && dot_r) {
      smooth_dot(G.lv[0], tr, dot_r, *dot_acc, tid, T);
      return true;
    }
    smooth(G.lv[l], 0, tr, tid, T);
    grid.sync();
  }
  return false;
}

}  // namespace mg
}  // namespace hs
