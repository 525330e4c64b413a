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
// (red, black) and one after (black, red).  Levels below kMgSmall cells run
// inside block 0 alone, separated by __syncthreads instead of grid barriers.
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
__device__ void smooth(const Level<M> &L, int color, bool zero_nb, bool tr, int tid, int T) {
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
    if (!zero_nb) s += offsum(L, o, L.x, q);
    L.x[q] = s / d;
  }
}

// coarse rhs = sum over the children of (rhs - A x)
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
          if (i >= F.nx || j >= F.ny || k >= F.nz) continue;
          const int q = idx(F, i + 1, j + 1, k + 1);
          M d, o[6];
          row(F, q, tr, d, o);
          acc += F.rhs[q] - (d * __ldcg(F.x + q) - offsum(F, o, F.x, q));
        }
    const int qc = idx(C, I + 1, J + 1, K + 1);
    C.rhs[qc] = unknown(C, qc) ? acc : M(0);
  }
}

template <class M>
__device__ void prolong(const Level<M> &F, const Level<M> &C, int tid, int T) {
  const int n = F.nx * F.ny * F.nz;
  for (int e = tid; e < n; e += T) {
    const int row_ = e / F.nx, i = e - row_ * F.nx;
    const int k = row_ / F.ny, j = row_ - k * F.ny;
    const int q = idx(F, i + 1, j + 1, k + 1);
    if (!unknown(F, q)) continue;
    F.x[q] = __ldcg(F.x + q) + __ldcg(C.x + idx(C, i / 2 + 1, j / 2 + 1, k / 2 + 1));
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

// lv[0].x = V-cycle applied to lv[0].rhs
template <class M>
__device__ void vcycle(const Hier<M> &G, bool tr, cg::grid_group &grid, int tid, int T) {
  int ls = 0;  // first level handled by block 0 alone
  while (ls < G.L - 1 && !small(G.lv[ls])) ++ls;
  for (int l = 0; l < ls; ++l) {
    smooth(G.lv[l], 0, true, tr, tid, T);
    grid.sync();
    smooth(G.lv[l], 1, false, tr, tid, T);
    grid.sync();
    restrict_res(G.lv[l], G.lv[l + 1], tr, tid, T);
    grid.sync();
  }
  if (blockIdx.x == 0) {
    const int t = threadIdx.x, B = blockDim.x;
    for (int l = ls; l < G.L - 1; ++l) {
      smooth(G.lv[l], 0, true, tr, t, B);
      __syncthreads();
      smooth(G.lv[l], 1, false, tr, t, B);
      __syncthreads();
      restrict_res(G.lv[l], G.lv[l + 1], tr, t, B);
      __syncthreads();
    }
    coarse_solve(G);
    __syncthreads();
    for (int l = G.L - 2; l >= ls; --l) {
      prolong(G.lv[l], G.lv[l + 1], t, B);
      __syncthreads();
      smooth(G.lv[l], 1, false, tr, t, B);
      __syncthreads();
      smooth(G.lv[l], 0, false, tr, t, B);
      __syncthreads();
    }
  }
  grid.sync();
  for (int l = ls - 1; l >= 0; --l) {
    prolong(G.lv[l], G.lv[l + 1], tid, T);
    grid.sync();
    smooth(G.lv[l], 1, false, tr, tid, T);
    grid.sync();
    smooth(G.lv[l], 0, false, tr, tid, T);
    grid.sync();
  }
}

}  // namespace mg
}  // namespace hs
