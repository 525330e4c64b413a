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
// GPU) solves exactly.  Smoother: red-black Gauss-Seidel, G.nsw sweeps on
// level 0 and G.nswc on the coarser levels before (red, black, ...) and after
// (black, red, ...) each coarse correction, mirrored so that the cycle stays
// symmetric for CG; the first red half-sweep (from
// x = 0) is applied by whoever writes the level's rhs, the prolongation is
// fused into the first post-smoothing half-sweep.  The coarse levels (at most kMgSmall
// cells each, with x and rhs together at most kMgStageMax bytes) run inside block 0
// alone, separated by __syncthreads instead of grid barriers, with their x and rhs
// staged in the launch's dynamic shared memory (plan_stage); the couplings, fluxes
// and masks of as many of them as fit (coarsest first, up to kMgStageTotal bytes
// in all) are copied there once per solve, after the hierarchy is built.
#pragma once
#include <cooperative_groups.h>
#include <cstdint>
#include <stdexcept>

namespace hs {
namespace mg {

namespace cg = cooperative_groups;

constexpr int kMgMaxLv = 16;
constexpr int kMgCoarse = 64;
constexpr long long kMgSmall = 2048;
constexpr int kMgStageMax = 64 * 1024;     // bytes of x and rhs of the levels block 0 runs alone
constexpr int kMgStageTotal = 160 * 1024;  // with their read-only arrays: the dynamic shared memory the kernels accept

template <class M>
struct Level {
  int nx, ny, nz;
  int px;           // row pitch of the padded arrays (>= nx + 2; the cells past nx + 1 are zero)
  M *x, *rhs;
  M *gx, *gy, *gz;
  M *fx, *fy, *fz;  // null: pure diffusion
  uint8_t *m;       // null: every interior cell is an unknown
  M *d;             // null, or the diagonal of every row (read by seed_diag)
};

template <class M>
struct Hier {
  int L;
  int nsw;   // red-black sweeps before and after the coarse correction on level 0 (0 or 1: one)
  int nswc;  // the same on the coarser levels (0 or 1: one)
  Level<M> lv[kMgMaxLv];
  double *lu;  // kMgCoarse^2: the factors, read back while the inverse is formed
  int ls;      // first level that block 0 handles alone (plan_stage)
  int stage;   // bytes of dynamic shared memory holding x and rhs of levels ls..L-1 and the read-only arrays
  int sx[kMgMaxLv], sr[kMgMaxLv];  // byte offsets of a staged level's x and rhs in it
  int sro;     // first level whose couplings, fluxes and mask are staged too (L: none)
  int sg[kMgMaxLv][3], sf[kMgMaxLv][3], sm[kMgMaxLv];  // their byte offsets (-1: the array is null)
};

// Grid-stride walk over an mx x ny x nz box in flat order (m fastest): the
// cell sequence of `for (e = tid; e < mx*ny*nz; e += T)` without a division
// per cell.  The start and the stride T are split into (m, j, k) once; each
// step adds the stride and carries (dm < mx and dj < ny, so one carry per
// axis suffices).  Needs mx, ny >= 1 and mx*ny*nz + T < 2^31.
struct Walk {
  int m, j, k, dm, dj, dk, mx, ny, nz;
  __host__ __device__ __forceinline__ Walk(int mx_, int ny_, int nz_, int tid, int T) : mx(mx_), ny(ny_), nz(nz_) {
    const int row = tid / mx, srow = T / mx;
    m = tid - row * mx;
    j = row % ny;
    k = row / ny;
    dm = T - srow * mx;
    dj = srow % ny;
    dk = srow / ny;
  }
  __host__ __device__ __forceinline__ bool ok() const { return k < nz; }
  __host__ __device__ __forceinline__ void next() {
    m += dm;
    int c = 0;
    if (m >= mx) { m -= mx; c = 1; }
    j += dj + c;
    c = 0;
    if (j >= ny) { j -= ny; c = 1; }
    k += dk + c;
  }
  __host__ __device__ __forceinline__ int flat() const { return m + mx * (j + ny * k); }
};

// values in each padded array of level L (row pitch px)
template <class M>
__host__ __device__ __forceinline__ long long padded(const Level<M> &L) { return (long long)L.px * (L.ny + 2) * (L.nz + 2); }

template <class M>
__host__ __device__ __forceinline__ bool small(const Level<M> &L) { return (long long)L.nx * L.ny * L.nz <= kMgSmall; }

// Host: the levels that block 0 handles alone, ls..L-1: every level from the
// first of at most kMgSmall cells on, less the finest of them while their x
// and rhs (padded layout as in global memory, each array 16-byte aligned)
// exceed kMgStageMax bytes; the coarsest (<= kMgCoarse cells) always fits.
// Places those arrays in the launch's dynamic shared memory (G.stage bytes),
// followed, when ro is set, by the couplings, fluxes and mask of the coarsest
// of those levels, as many as fit in kMgStageTotal bytes in all (levels
// G.sro..L-1): they do not change during a solve and are copied in once
// (stage_ro).  A kernel that reuses the staging area between the V-cycles
// (the z-marching p' solve) plans with ro = false.
template <class M>
inline void plan_stage(Hier<M> &G, bool ro = true) {
  G.ls = 0;
  G.stage = 0;
  G.sro = G.L;
  if (G.L < 1) return;
  auto bytes = [&](int l) {
    const Level<M> &L = G.lv[l];
    return (padded(L) * (long long)sizeof(M) + 15) / 16 * 16;
  };
  int ls = 0;
  while (ls < G.L - 1 && !small(G.lv[ls])) ++ls;
  long long tot = 0;
  for (int l = ls; l < G.L; ++l) tot += 2 * bytes(l);
  while (tot > kMgStageMax && ls < G.L - 1) tot -= 2 * bytes(ls++);
  if (tot > kMgStageMax) throw std::runtime_error("multigrid: coarsest level exceeds the shared-memory staging");
  long long off = 0;
  for (int l = ls; l < G.L; ++l) {
    G.sx[l] = (int)off;
    G.sr[l] = (int)(off + bytes(l));
    off += 2 * bytes(l);
  }
  G.ls = ls;
  for (int l = G.L - 1; ro && l >= ls; --l) {
    const Level<M> &L = G.lv[l];
    const long long mb = L.m ? (padded(L) + 15) / 16 * 16 : 0;
    if (off + (L.fx ? 6 : 3) * bytes(l) + mb > kMgStageTotal) break;
    for (int a = 0; a < 3; ++a) {
      G.sg[l][a] = (int)off;
      off += bytes(l);
    }
    for (int a = 0; a < 3; ++a) {
      G.sf[l][a] = L.fx ? (int)off : -1;
      if (L.fx) off += bytes(l);
    }
    G.sm[l] = L.m ? (int)off : -1;
    off += mb;
    G.sro = l;
  }
  G.stage = (int)off;
}

template <class M>
__device__ __forceinline__ int idx(const Level<M> &L, int i, int j, int k) {
  return i + L.px * (j + (L.ny + 2) * k);
}

template <class M>
__device__ __forceinline__ M pos(M a) { return a > M(0) ? a : M(0); }

// diagonal and the six off-diagonal magnitudes of row q (order W E S N B F)
template <class M>
__device__ __forceinline__ void row(const Level<M> &L, int q, bool tr, M &d, M (&o)[6]) {
  const int PX = L.px, PXY = L.px * (L.ny + 2);
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

// a value of x: from L2 in the grid-wide passes (other blocks wrote it), by a
// plain load when x is staged in block 0's shared memory (S)
template <bool S, class M>
__device__ __forceinline__ M ldx(const M *p) {
  if constexpr (S) return *p;
  else return __ldcg(p);
}

template <class M, bool S = false>
__device__ __forceinline__ M offsum(const Level<M> &L, const M (&o)[6], const M *x, int q) {
  const int PX = L.px, PXY = L.px * (L.ny + 2);
  return o[0] * ldx<S>(x + q - 1) + o[1] * ldx<S>(x + q + 1) + o[2] * ldx<S>(x + q - PX) + o[3] * ldx<S>(x + q + PX) +
         o[4] * ldx<S>(x + q - PXY) + o[5] * ldx<S>(x + q + PXY);
}

template <class M>
__device__ __forceinline__ bool unknown(const Level<M> &L, int q) { return L.m ? L.m[q] != 0 : true; }

// coarse level C from fine level F (every padded cell of C that holds a face)
template <class M>
__device__ __forceinline__ void coarsen(const Level<M> &F, const Level<M> &C, int tid, int T) {
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
template <class M, bool S = false>
__device__ __forceinline__ void smooth(const Level<M> &L, int color, bool tr, int tid, int T) {
  for (Walk w((L.nx + 1) / 2, L.ny, L.nz, tid, T); w.ok(); w.next()) {
    const int j = w.j, k = w.k, i = 2 * w.m + ((j + k + color) & 1);
    if (i >= L.nx) continue;
    const int q = idx(L, i + 1, j + 1, k + 1);
    M d, o[6];
    row(L, q, tr, d, o);
    const M s = L.rhs[q] + offsum<M, S>(L, o, L.x, q);
    L.x[q] = d == M(0) ? M(0) : s / d;
  }
}

// The last colour-0 half-sweep of level 0, also accumulating sum r x over
// every cell (colour 0 as it is computed, colour 1 as left by the previous
// half-sweep): the V-cycle's output dotted with the caller's residual r
// (padded, any precision; FP64 sums) without a pass of its own.
template <class M, class RT>
__device__ __forceinline__ void smooth_dot(const Level<M> &L, bool tr, const RT *r, double &acc, int tid, int T) {
  for (Walk w((L.nx + 1) / 2, L.ny, L.nz, tid, T); w.ok(); w.next()) {
    const int j = w.j, k = w.k;
    const int i = 2 * w.m + ((j + k) & 1), ib = 2 * w.m + ((j + k + 1) & 1);
    const int q = idx(L, i + 1, j + 1, k + 1), qb = idx(L, ib + 1, j + 1, k + 1);
    const bool ha = i < L.nx, hb = ib < L.nx;
    const double rb = hb ? (double)r[qb] : 0.0, xb = hb ? (double)__ldcg(L.x + qb) : 0.0;
    if (ha) {
      const double ra = (double)r[q];
      M d, o[6];
      row(L, q, tr, d, o);
      const M s = L.rhs[q] + offsum(L, o, L.x, q);
      const M xv = d == M(0) ? M(0) : s / d;
      L.x[q] = xv;
      acc += ra * (double)xv;
    }
    if (hb) acc += rb * xb;
  }
}

// The first pre-smoothing half-sweep starts from x = 0, so on the colour-0
// cells it is local, x = rhs / d: whoever writes a level's rhs applies it to
// the cell in the same pass (the restriction for the coarse levels, the
// Krylov solver for level 0), which saves that half-sweep and its barrier.
// In two halves, so that a pass can issue every load before its first store
// (a load after a store to another array waits for it: the compiler cannot
// prove that they do not alias): seed_diag() loads the diagonal of a colour-0
// cell (0 for colour 1, which is not seeded), seed_store() writes rhs and the
// seed.
template <class M>
__device__ __forceinline__ M seed_diag(const Level<M> &L, int q, int i, int j, int k, bool tr) {
  if ((i + j + k) & 1) return M(0);
  if (L.d) return L.d[q];
  M d, o[6];
  row(L, q, tr, d, o);
  return d;
}

template <class M>
__device__ __forceinline__ void seed_store(const Level<M> &L, int q, int i, int j, int k, M rhs, M d) {
  L.rhs[q] = rhs;
  if (!((i + j + k) & 1)) L.x[q] = d == M(0) ? M(0) : rhs / d;
}

// both halves for cell (i, j, k) of level L (padded index q):
// Seed s = seed_at(L, i, j, k, q, tr) with the pass's loads, s.store(L, q, v) last
template <class M>
struct Seed {
  int i, j, k;
  M d;
  template <class V>
  __device__ __forceinline__ void store(const Level<M> &L, int q, V v) const { seed_store(L, q, i, j, k, (M)v, d); }
};

template <class M>
__device__ __forceinline__ Seed<M> seed_at(const Level<M> &L, int i, int j, int k, int q, bool tr) {
  Seed<M> s;
  s.i = i;
  s.j = j;
  s.k = k;
  s.d = seed_diag(L, q, i, j, k, tr);
  return s;
}

// coarse rhs = sum over the children of (rhs - A x), and the coarse seed.  It follows the
// colour-1 half-sweep, after which a colour-1 cell's residual is zero up to
// rounding (its update solved its own row), so only the colour-0 children
// are evaluated, in (dk, dj) order.  Large levels: a thread per coarse cell.
// Levels whose children all fit in one pass of the threads: four lanes per
// coarse cell, lane c of a group evaluating the colour-0 child of (dj, dk) =
// (c & 1, c >> 1) (di = (dj + dk) & 1) and the group's first lane summing
// them in the same order, so that one memory round trip replaces four
// (every lane of a warp runs the same number of iterations: the shuffles
// need the full warp).
template <class M, bool S = false>
__device__ __forceinline__ void restrict_res(const Level<M> &F, const Level<M> &C, bool tr, int tid, int T) {
  if (4LL * C.nx * C.ny * C.nz > T) {
    for (Walk w(C.nx, C.ny, C.nz, tid, T); w.ok(); w.next()) {
      const int I = w.m, J = w.j, K = w.k;
      M acc = M(0);
      for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
          for (int di = 0; di < 2; ++di) {
            const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
            if (i >= F.nx || j >= F.ny || k >= F.nz || ((i + j + k) & 1)) continue;
            const int q = idx(F, i + 1, j + 1, k + 1);
            M d, o[6];
            row(F, q, tr, d, o);
            acc += F.rhs[q] - (d * ldx<S>(F.x + q) - offsum<M, S>(F, o, F.x, q));
          }
      const int qc = idx(C, I + 1, J + 1, K + 1);
      const M v = unknown(C, qc) ? acc : M(0);
      seed_store(C, qc, I, J, K, v, seed_diag(C, qc, I, J, K, tr));
    }
    return;
  }
  const int c = tid & 3, dj = c & 1, dk = c >> 1, di = (dj + dk) & 1;
  const int g0 = (threadIdx.x & 31) & ~3;
  for (Walk w(C.nx, C.ny, C.nz, tid >> 2, T >> 2); __any_sync(0xffffffffu, w.ok()); w.next()) {
    const bool live = w.ok();
    const int I = w.m, J = w.j, K = w.k;
    const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
    const bool has = live && i < F.nx && j < F.ny && k < F.nz;
    const bool lead = live && c == 0;
    const int qc = lead ? idx(C, I + 1, J + 1, K + 1) : 0;
    const M dc = lead ? seed_diag(C, qc, I, J, K, tr) : M(0);
    const bool uc = lead && unknown(C, qc);
    M v = M(0);
    if (has) {
      const int q = idx(F, i + 1, j + 1, k + 1);
      M d, o[6];
      row(F, q, tr, d, o);
      v = F.rhs[q] - (d * ldx<S>(F.x + q) - offsum<M, S>(F, o, F.x, q));
    }
    const M v1 = __shfl_sync(0xffffffffu, v, g0 + 1), v2 = __shfl_sync(0xffffffffu, v, g0 + 2),
            v3 = __shfl_sync(0xffffffffu, v, g0 + 3);
    const unsigned hm = __ballot_sync(0xffffffffu, has) >> g0;
    if (lead) {
      M acc = M(0);
      if (hm & 1u) acc += v;
      if (hm & 2u) acc += v1;
      if (hm & 4u) acc += v2;
      if (hm & 8u) acc += v3;
      seed_store(C, qc, I, J, K, uc ? acc : M(0), dc);
    }
  }
}

// Prolongation fused into the first post-smoothing half-sweep (colour 1):
// every neighbour (colour 0) is read as x + x_coarse(parent).  A Gauss-Seidel
// update never reads its own cell, so the colour-0 cells' prolonged values
// are needed only as these neighbour values (the colour-0 half-sweep that
// follows recomputes them) and the colour-1 cells' not at all.  Ghost
// neighbours are 0, as they are never prolonged; a masked neighbour has a
// zero coupling.  The arithmetic is that of prolongation followed by smooth().
template <class M, bool S = false>
__device__ __forceinline__ void prolong_smooth(const Level<M> &F, const Level<M> &C, bool tr, int tid, int T) {
  const int PX = F.px, PXY = F.px * (F.ny + 2);
  const int CPX = C.px, CPXY = C.px * (C.ny + 2);
  for (Walk w((F.nx + 1) / 2, F.ny, F.nz, tid, T); w.ok(); w.next()) {
    const int j = w.j, k = w.k, i = 2 * w.m + ((j + k + 1) & 1);
    if (i >= F.nx) continue;
    const int q = idx(F, i + 1, j + 1, k + 1);
    M d, o[6];
    row(F, q, tr, d, o);
    // the parent P of this cell is the parent of three of its neighbours; on
    // each axis the other neighbour's parent is P's neighbour on the side of
    // this cell's parity (P -+ 1 for an even / odd index)
    const int qc = idx(C, (i >> 1) + 1, (j >> 1) + 1, (k >> 1) + 1);
    const M cp = ldx<S>(C.x + qc);
    const M cx = ldx<S>(C.x + ((i & 1) ? qc + 1 : qc - 1));
    const M cy = ldx<S>(C.x + ((j & 1) ? qc + CPX : qc - CPX));
    const M cz = ldx<S>(C.x + ((k & 1) ? qc + CPXY : qc - CPXY));
    // neighbour values x + x_coarse(parent); ghosts stay 0 (never prolonged)
    const M xw = i > 0 ? ldx<S>(F.x + q - 1) + ((i & 1) ? cp : cx) : M(0);
    const M xe = i + 1 < F.nx ? ldx<S>(F.x + q + 1) + ((i & 1) ? cx : cp) : M(0);
    const M xs = j > 0 ? ldx<S>(F.x + q - PX) + ((j & 1) ? cp : cy) : M(0);
    const M xn = j + 1 < F.ny ? ldx<S>(F.x + q + PX) + ((j & 1) ? cy : cp) : M(0);
    const M xb = k > 0 ? ldx<S>(F.x + q - PXY) + ((k & 1) ? cp : cz) : M(0);
    const M xf = k + 1 < F.nz ? ldx<S>(F.x + q + PXY) + ((k & 1) ? cz : cp) : M(0);
    const M off = o[0] * xw + o[1] * xe + o[2] * xs + o[3] * xn + o[4] * xb + o[5] * xf;
    const M s = F.rhs[q] + off;
    F.x[q] = d == M(0) ? M(0) : s / d;
  }
}

// Block 0's shared memory for the coarsest operator: the LU factors during
// factor(), then the explicit inverse read by every coarse_solve() of the
// same launch; and the pivots (one instance per block: function-scope
// __shared__ storage is static).
__device__ __forceinline__ double *lu_smem() {
  __shared__ double a[kMgCoarse * kMgCoarse];
  return a;
}
__device__ __forceinline__ int *piv_smem() {
  __shared__ int p[kMgCoarse];
  return p;
}

// LU with partial pivoting of the coarsest operator (A or A^T), by block 0,
// in shared memory; the pivot is the largest |a| in the column, the lowest
// row among equals; the factors are copied to G.lu and the explicit
// inverse is left in shared memory for coarse_solve
template <class M>
__device__ __forceinline__ void factor(const Hier<M> &G, bool tr) {
  if (blockIdx.x != 0) return;
  double *a = lu_smem();
  int *sp = piv_smem();
  __shared__ int spiv;
  const Level<M> &C = G.lv[G.L - 1];
  const int nc = C.nx * C.ny * C.nz, PX = C.px, PXY = C.px * (C.ny + 2);
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
      // br starts at the diagonal: a column with no comparable |a| (every
      // entry NaN) keeps its own row, so the swap below stays in the matrix
      double bv = -1.0;
      int br = col;
      for (int r = col + threadIdx.x; r < nc; r += 32) {
        const double v = fabs(a[r * nc + col]);
        if (v > bv || (v == bv && r < br)) { bv = v; br = r; }
      }
      for (int o = 16; o; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int orow = __shfl_xor_sync(0xffffffffu, br, o);
        if (ov > bv || (ov == bv && orow < br)) { bv = ov; br = orow; }
      }
      if (threadIdx.x == 0) { spiv = br; sp[col] = br; }
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
  __syncthreads();
  // explicit inverse from the factors (A = P^T L U): thread j solves
  // A x = e_j and stores x as column j, at a[j * nc + r], over the factors
  // (read back from G.lu)
  if (threadIdx.x < nc) {
    const int j = threadIdx.x;
    double *x = a + j * nc;
    int pos = j;  // where the swaps move the 1 of e_j
    for (int c2 = 0; c2 < nc; ++c2) {
      const int pr = sp[c2];
      if (pos == c2) pos = pr;
      else if (pos == pr) pos = c2;
    }
    for (int r = 0; r < nc; ++r) {
      double v = r == pos ? 1.0 : 0.0;
      for (int c2 = 0; c2 < r; ++c2) v -= G.lu[r * nc + c2] * x[c2];
      x[r] = v;
    }
    for (int r = nc - 1; r >= 0; --r) {
      double v = x[r];
      for (int c2 = r + 1; c2 < nc; ++c2) v -= G.lu[r * nc + c2] * x[c2];
      x[r] = v / G.lu[r * nc + r];
    }
  }
}

// exact solve on the coarsest level C (G.lv[G.L - 1], or its staged copy) by
// block 0 (every thread of the block calls it): x = A^-1 rhs with the inverse
// that factor() left in shared memory, thread r summing row r in column order
template <class M>
__device__ __forceinline__ void coarse_solve(const Level<M> &C) {
  __shared__ double y[kMgCoarse];
  const double *ainv = lu_smem();
  const int nc = C.nx * C.ny * C.nz, r = threadIdx.x;
  const int q = r < nc ? idx(C, r % C.nx + 1, (r / C.nx) % C.ny + 1, r / (C.nx * C.ny) + 1) : 0;
  if (r < nc) y[r] = (double)C.rhs[q];
  __syncthreads();
  if (r < nc) {
    double v = 0.0;
    for (int c2 = 0; c2 < nc; ++c2) v += ainv[c2 * nc + r] * y[c2];
    C.x[q] = unknown(C, q) ? (M)v : M(0);
  }
}

// the launch's dynamic shared memory (Hier::stage bytes)
__device__ __forceinline__ unsigned char *stage_smem() {
  extern __shared__ __align__(16) unsigned char mg_stage[];
  return mg_stage;
}

// level l (>= G.ls) with x and rhs in the staging area, and its read-only
// arrays when RO is set and they are staged (l >= G.sro)
template <bool RO = false, class M>
__device__ __forceinline__ Level<M> staged(const Hier<M> &G, int l) {
  Level<M> L = G.lv[l];
  unsigned char *b = stage_smem();
  L.x = reinterpret_cast<M *>(b + G.sx[l]);
  L.rhs = reinterpret_cast<M *>(b + G.sr[l]);
  if (RO && l >= G.sro) {
    L.gx = reinterpret_cast<M *>(b + G.sg[l][0]);
    L.gy = reinterpret_cast<M *>(b + G.sg[l][1]);
    L.gz = reinterpret_cast<M *>(b + G.sg[l][2]);
    if (L.fx) {
      L.fx = reinterpret_cast<M *>(b + G.sf[l][0]);
      L.fy = reinterpret_cast<M *>(b + G.sf[l][1]);
      L.fz = reinterpret_cast<M *>(b + G.sf[l][2]);
    }
    if (L.m) L.m = b + G.sm[l];
  }
  return L;
}

// Block 0 copies the read-only arrays of levels G.sro.. into the staging
// area (every thread of the block calls it; the hierarchy is built and
// visible to block 0).  They stay there for the rest of the launch.
template <class M>
__device__ __forceinline__ void stage_ro(const Hier<M> &G) {
  for (int l = G.sro; l < G.L; ++l) {
    const Level<M> &Lg = G.lv[l];
    const Level<M> Ls = staged<true>(G, l);
    const int n = (int)padded(Lg);
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      Ls.gx[e] = __ldcg(Lg.gx + e);
      Ls.gy[e] = __ldcg(Lg.gy + e);
      Ls.gz[e] = __ldcg(Lg.gz + e);
      if (Lg.fx) {
        Ls.fx[e] = __ldcg(Lg.fx + e);
        Ls.fy[e] = __ldcg(Lg.fy + e);
        Ls.fz[e] = __ldcg(Lg.fz + e);
      }
      if (Lg.m) Ls.m[e] = __ldcg(Lg.m + e);
    }
  }
  __syncthreads();
}

// build levels 1.. from level 0 and factor the coarsest (the caller filled level 0)
template <class M>
__device__ __forceinline__ void build(const Hier<M> &G, bool tr, cg::grid_group &grid, int tid, int T) {
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
  if (blockIdx.x == 0) stage_ro(G);
  grid.sync();
}

// Levels G.ls.. of the V-cycle, by block 0 alone (every thread of the block
// calls it), with x and rhs in shared memory: level ls's are copied in (as
// the grid-wide passes left them: rhs and the seeded x) and its x is copied
// back at the end; the coarser levels' x start from 0, so that their ghosts
// are 0 as in global memory.  The arithmetic is that of the grid-wide passes.
template <bool RO, class M>
__device__ __forceinline__ void small_levels(const Hier<M> &G, bool tr) {
  const int t = threadIdx.x, B = blockDim.x, ls = G.ls;
  {
    const Level<M> &Lg = G.lv[ls];
    const Level<M> Ls = staged<RO>(G, ls);
    const int n = (int)padded(Lg);
    for (int e = t; e < n; e += B) {
      const M xv = __ldcg(Lg.x + e), rv = __ldcg(Lg.rhs + e);
      Ls.x[e] = xv;
      Ls.rhs[e] = rv;
    }
    for (int l = ls + 1; l < G.L; ++l) {
      const Level<M> C = staged<RO>(G, l);
      const int nc = (int)padded(C);
      for (int e = t; e < nc; e += B) C.x[e] = M(0);
    }
    __syncthreads();
  }
  for (int l = ls; l < G.L - 1; ++l) {
    const Level<M> F = staged<RO>(G, l), C = staged<RO>(G, l + 1);
    const int ns = l == 0 ? G.nsw : G.nswc;
    smooth<M, true>(F, 1, tr, t, B);
    __syncthreads();
    for (int s = 1; s < ns; ++s) {
      smooth<M, true>(F, 0, tr, t, B);
      __syncthreads();
      smooth<M, true>(F, 1, tr, t, B);
      __syncthreads();
    }
    restrict_res<M, true>(F, C, tr, t, B);
    __syncthreads();
  }
  coarse_solve(staged<RO>(G, G.L - 1));
  __syncthreads();
  for (int l = G.L - 2; l >= ls; --l) {
    const Level<M> F = staged<RO>(G, l), C = staged<RO>(G, l + 1);
    const int ns = l == 0 ? G.nsw : G.nswc;
    prolong_smooth<M, true>(F, C, tr, t, B);
    __syncthreads();
    smooth<M, true>(F, 0, tr, t, B);
    __syncthreads();
    for (int s = 1; s < ns; ++s) {
      smooth<M, true>(F, 1, tr, t, B);
      __syncthreads();
      smooth<M, true>(F, 0, tr, t, B);
      __syncthreads();
    }
  }
  {
    const Level<M> &Lg = G.lv[ls];
    const Level<M> Ls = staged<RO>(G, ls);
    const int n = (int)padded(Lg);
    for (int e = t; e < n; e += B) Lg.x[e] = Ls.x[e];
  }
}

// lv[first].x = V-cycle applied to lv[first].rhs (first = 0: the whole
// cycle; first = 1: the part below a level 0 that the caller smooths itself,
// with first < ls); the caller has written lv[first].rhs
// and seeded lv[first] (seed_diag / seed_store on every interior cell) before the barrier that
// precedes this call.  With dot_r, the last level-0 pass also adds this
// thread's share of sum dot_r x to *dot_acc and the final barrier is left to
// the caller's reduction (returns true); it returns false, with the barrier
// done and nothing added, when level 0 is handled by block 0 alone or is not
// part of the call.  RO: block 0's levels read the couplings, fluxes and
// masks that stage_ro copied into shared memory (levels G.sro..).
template <class M, class RT = double, bool RO = false>
__device__ __forceinline__ bool vcycle(const Hier<M> &G, bool tr, cg::grid_group &grid, int tid, int T,
                       const RT *dot_r = nullptr, double *dot_acc = nullptr, int first = 0) {
  const int ls = G.ls;  // first level handled by block 0 alone
  // the barrier after the last write of lv[first].x: with first > 0 the
  // caller's next pass reads it through the TMA unit (async proxy), so each
  // writing thread orders its writes for that proxy first
  auto last_sync = [&]() {
    if (first > 0) asm volatile("fence.proxy.async.global;" ::: "memory");
    grid.sync();
  };
  for (int l = first; l < ls; ++l) {
    smooth(G.lv[l], 1, tr, tid, T);
    grid.sync();
    for (int s = 1; s < (l == 0 ? G.nsw : G.nswc); ++s) {
      smooth(G.lv[l], 0, tr, tid, T);
      grid.sync();
      smooth(G.lv[l], 1, tr, tid, T);
      grid.sync();
    }
    restrict_res(G.lv[l], G.lv[l + 1], tr, tid, T);
    grid.sync();
  }
  if (blockIdx.x == 0) small_levels<RO>(G, tr);
  if (ls == first) last_sync();
  else grid.sync();
  for (int l = ls - 1; l >= first; --l) {
    prolong_smooth(G.lv[l], G.lv[l + 1], tr, tid, T);
    grid.sync();
    for (int s = 1; s < (l == 0 ? G.nsw : G.nswc); ++s) {
      smooth(G.lv[l], 0, tr, tid, T);
      grid.sync();
      smooth(G.lv[l], 1, tr, tid, T);
      grid.sync();
    }
    if (l == 0 && dot_r) {
      smooth_dot(G.lv[0], tr, dot_r, *dot_acc, tid, T);
      return true;
    }
    smooth(G.lv[l], 0, tr, tid, T);
    if (l == first) last_sync();
    else grid.sync();
  }
  return false;
}

}  // namespace mg
}  // namespace hs
