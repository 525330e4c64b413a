// One rank's z-slab of the channel pressure-correction system, for meshes
// sharded over GPUs (the reference's domain decomposition: Scotch parts,
// mesh/mesh.cpp:735-1122, and a HYPRE PCG over MPI ranks,
// fluid_solver.h:1713-2194).  The slab holds its interior planes plus one
// ghost plane below and above; the host drives the CG recurrences, all-reduces
// the per-slab partial dot products in FP64 and exchanges the search
// direction's boundary planes into the neighbours' ghost planes before each
// product (hsolver_b200/slabs.py: over NCCL, or between slabs of one process).
// Preconditioner: the multigrid V-cycle of hs_mg.cuh on the slab's own rows
// (block Jacobi: the couplings across the slab faces stay in the diagonal,
// the neighbour values are zero), so the preconditioner is symmetric positive
// definite and block-diagonal, and CG with all-reduced dots is the global CG.
//
// Layout: padded cells (px = nx + 2 rounded up to 4, ny + 2, nz + 2), the
// coupling of each cell's low face stored at the cell, the high boundary face
// of the last cell on each axis in the ghost cell (so the coupling across the
// slab's top face sits in the upper ghost plane), FP64.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "hs_mg.cuh"
#include "hs_slab.hpp"

namespace cg = cooperative_groups;

namespace hs {

#define SL_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_) + \
                                                    " at " #call);                                 \
  } while (0)

namespace {

constexpr int kSlT = 256;      // threads of the vector kernels
constexpr int kSlVT = 512;     // threads of the V-cycle kernel (one block per SM)
constexpr int kSlBlocks = 592; // blocks of the vector kernels (4 per SM)

struct SlabDev {
  int nx, ny, nz, px;
  const double *gx, *gy, *gz;  // couplings (level 0 of the hierarchy)
  double *x, *r, *p, *s;       // CG vectors (p with its ghost planes filled by the host)
};

__device__ __forceinline__ int sq(const SlabDev &D, int i, int j, int k) {
  return (i + 1) + D.px * ((j + 1) + (D.ny + 2) * (k + 1));
}

__device__ double sl_block_sum(double v) {
  __shared__ double sh[32];
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;
}

// x = 0, r = b; partial sums of <b, b> per block
__global__ void k_sl_begin(SlabDev D, const double *b, double *part) {
  double acc = 0.0;
  const int T = gridDim.x * blockDim.x;
  for (mg::Walk w(D.nx, D.ny, D.nz, blockIdx.x * blockDim.x + threadIdx.x, T); w.ok(); w.next()) {
    const int q = sq(D, w.m, w.j, w.k);
    const double bv = b[q];
    D.x[q] = 0.0;
    D.r[q] = bv;
    acc += bv * bv;
  }
  const double t = sl_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// z = V-cycle(r) on the slab's rows (level 0's x), with the hierarchy built
// first when `build` is set; partial sums of <r, z> per block.  Shared memory
// does not outlive a launch, so every launch factors the coarsest level again
// (at most 64 cells, in block 0) and stages block 0's read-only arrays.
__global__ void __launch_bounds__(kSlVT, 1) k_sl_vcycle(SlabDev D, mg::Hier<double> G, int build, double *part) {
  cg::grid_group grid = cg::this_grid();
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  const mg::Level<double> &L0 = G.lv[0];
  if (build) {
    mg::build(G, false, grid, tid, T);
  } else {
    mg::factor(G, false);
    if (blockIdx.x == 0) mg::stage_ro(G);
    grid.sync();
  }
  for (mg::Walk w(D.nx, D.ny, D.nz, tid, T); w.ok(); w.next()) {
    const int q = sq(D, w.m, w.j, w.k);
    const mg::Seed<double> sd = mg::seed_at(L0, w.m, w.j, w.k, q, false);
    sd.store(L0, q, D.r[q]);
  }
  grid.sync();
  double acc = 0.0;
  if (!mg::vcycle<double, double, true>(G, false, grid, tid, T, D.r, &acc))
    for (mg::Walk w(D.nx, D.ny, D.nz, tid, T); w.ok(); w.next()) {
      const int q = sq(D, w.m, w.j, w.k);
      acc += D.r[q] * __ldcg(L0.x + q);
    }
  const double t = sl_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// p = z + beta p (beta = 0: p = z) on the interior
__global__ void k_sl_direction(SlabDev D, const double *z, double beta, int first) {
  const int T = gridDim.x * blockDim.x;
  for (mg::Walk w(D.nx, D.ny, D.nz, blockIdx.x * blockDim.x + threadIdx.x, T); w.ok(); w.next()) {
    const int q = sq(D, w.m, w.j, w.k);
    const double zq = z[q];
    D.p[q] = first ? zq : zq + beta * D.p[q];
  }
}

// s = A p (p's ghost planes hold the neighbours' planes, or zero at the
// domain's ends); partial sums of <s, p> per block
__global__ void k_sl_apply(SlabDev D, double *part) {
  const int PX = D.px, PXY = D.px * (D.ny + 2), T = gridDim.x * blockDim.x;
  double acc = 0.0;
  for (mg::Walk w(D.nx, D.ny, D.nz, blockIdx.x * blockDim.x + threadIdx.x, T); w.ok(); w.next()) {
    const int q = sq(D, w.m, w.j, w.k);
    const double cw = D.gx[q], ce = D.gx[q + 1], cs = D.gy[q], cn = D.gy[q + PX], cb = D.gz[q], cf = D.gz[q + PXY];
    const double p0 = D.p[q];
    const double pw = D.p[q - 1], pe = D.p[q + 1], ps = D.p[q - PX], pn = D.p[q + PX], pb = D.p[q - PXY],
                 pf = D.p[q + PXY];
    const double d = cw + ce + cs + cn + cb + cf;
    const double sv = d * p0 - (cw * pw + ce * pe + cs * ps + cn * pn + cb * pb + cf * pf);
    D.s[q] = sv;
    acc += sv * p0;
  }
  const double t = sl_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// x += alpha p, r -= alpha s; partial sums of <r, r> per block
__global__ void k_sl_update(SlabDev D, double alpha, double *part) {
  const int T = gridDim.x * blockDim.x;
  double acc = 0.0;
  for (mg::Walk w(D.nx, D.ny, D.nz, blockIdx.x * blockDim.x + threadIdx.x, T); w.ok(); w.next()) {
    const int q = sq(D, w.m, w.j, w.k);
    const double xv = D.x[q], pv = D.p[q], rv = D.r[q], sv = D.s[q];
    D.x[q] = xv + alpha * pv;
    const double rn = rv - alpha * sv;
    D.r[q] = rn;
    acc += rn * rn;
  }
  const double t = sl_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// level 0's mask and diagonal from the couplings: a cell with no coupling on
// any face is not an unknown
__global__ void k_sl_mask(SlabDev D, uint8_t *m, double *d) {
  const int PX = D.px, PXY = D.px * (D.ny + 2), T = gridDim.x * blockDim.x;
  for (mg::Walk w(D.nx, D.ny, D.nz, blockIdx.x * blockDim.x + threadIdx.x, T); w.ok(); w.next()) {
    const int q = sq(D, w.m, w.j, w.k);
    const double dv = D.gx[q] + D.gx[q + 1] + D.gy[q] + D.gy[q + PX] + D.gz[q] + D.gz[q + PXY];
    d[q] = dv;
    m[q] = dv > 0.0;
  }
}

int pitch4(int n) { return (n + 3) / 4 * 4; }

// The two-level preconditioner's global coarse grid: aggregates of agg^3 fine
// cells (fine (i, j, kg) with kg the global plane, in coarse cell
// (i / agg, j / agg, kg / agg)), piecewise-constant prolongation P, the
// restriction P^T (sums over an aggregate) and A_c = P^T A P, whose face
// couplings are the sums of the fine couplings on the aggregates' faces.
struct CoarseMap {
  int agg, kg0, ncx, ncy, ncz;
};

// partial P^T r of this slab: one thread per coarse cell sums its fine cells
// in this slab's planes (k, j, i ascending), 0 where it has none
__global__ void k_sl_restrict(SlabDev D, CoarseMap M, double *rc) {
  const int nc = M.ncx * M.ncy * M.ncz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const int I = c % M.ncx, J = (c / M.ncx) % M.ncy, K = c / (M.ncx * M.ncy);
    const int i0 = I * M.agg, i1 = min(i0 + M.agg, D.nx), j0 = J * M.agg, j1 = min(j0 + M.agg, D.ny);
    const int k0 = max(K * M.agg - M.kg0, 0), k1 = min((K + 1) * M.agg - M.kg0, D.nz);
    double acc = 0.0;
    for (int k = k0; k < k1; ++k)
      for (int j = j0; j < j1; ++j)
        for (int i = i0; i < i1; ++i) acc += D.r[sq(D, i, j, k)];
    rc[c] = acc;
  }
}

// coarse correction: the coarse grid's V-cycle on rc (the coarse hierarchy
// built first when `build` is set), then z += P zc on this slab's unknowns
// (level 0's x of the slab's hierarchy holds z from slab_precond) and the
// partial sums of <r, z> per block
__global__ void __launch_bounds__(kSlVT, 1) k_sl_coarse(SlabDev D, mg::Hier<double> G, mg::Hier<double> C,
                                                       CoarseMap M, const double *rc, int build, double *part) {
  cg::grid_group grid = cg::this_grid();
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  const mg::Level<double> &C0 = C.lv[0];
  if (build) {
    mg::build(C, false, grid, tid, T);
  } else {
    mg::factor(C, false);
    if (blockIdx.x == 0) mg::stage_ro(C);
    grid.sync();
  }
  for (mg::Walk w(C0.nx, C0.ny, C0.nz, tid, T); w.ok(); w.next()) {
    const int q = mg::idx(C0, w.m + 1, w.j + 1, w.k + 1);
    const mg::Seed<double> sd = mg::seed_at(C0, w.m, w.j, w.k, q, false);
    sd.store(C0, q, rc[w.flat()]);
  }
  grid.sync();
  mg::vcycle<double, double, true>(C, false, grid, tid, T);
  const mg::Level<double> &L0 = G.lv[0];
  double acc = 0.0;
  for (mg::Walk w(D.nx, D.ny, D.nz, tid, T); w.ok(); w.next()) {
    const int q = sq(D, w.m, w.j, w.k);
    const int qc = mg::idx(C0, w.m / M.agg + 1, w.j / M.agg + 1, (w.k + M.kg0) / M.agg + 1);
    const double zc = __ldcg(C0.x + qc);
    const double z = __ldcg(L0.x + q) + (L0.m[q] ? zc : 0.0);
    L0.x[q] = z;
    acc += D.r[q] * z;
  }
  const double t = sl_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

}  // namespace

struct SlabState {
  int device = 0, nx = 0, ny = 0, nz = 0, px = 0;
  size_t np = 0;
  cudaStream_t stream = nullptr;
  std::vector<void *> allocs;
  SlabDev D{};
  double *b = nullptr, *part = nullptr;
  std::vector<double> host_part;
  mg::Hier<double> G{};
  int vgrid = 0;
  bool built = false;
  // the global coarse grid of the two-level preconditioner (aggregates of
  // agg^3 cells; every slab holds the whole coarse grid and its hierarchy)
  int agg = 0, kg0 = 0, nzg = 0, ncx = 0, ncy = 0, ncz = 0;
  mg::Hier<double> C{};
  double *crhs = nullptr;  // coarse rhs (nc values, x fastest), uploaded each application
  double *crc = nullptr;   // this slab's partial coarse rhs
  bool cbuilt = false;
  std::vector<double> cpart[3];  // this slab's partial coarse face couplings (set_system)

  template <class T_>
  T_ *alloc(size_t n) {
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T_));
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA alloc: ") + cudaGetErrorString(e));
    allocs.push_back(p);
    SL_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T_), stream));
    return (T_ *)p;
  }
  ~SlabState() {
    for (void *p : allocs) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

template <class K, class... A>
void sl_coop(K kernel, int blocks, int threads, size_t smem, cudaStream_t s, A... args) {
  void *argv[] = {(void *)&args...};
  SL_CUDA(cudaLaunchCooperativeKernel((void *)kernel, dim3(blocks), dim3(threads), argv, smem, s));
}

// the sum of the first n block partials, in block order (deterministic)
double sl_sum(SlabState &S, int n) {
  S.host_part.resize(n);
  SL_CUDA(cudaMemcpyAsync(S.host_part.data(), S.part, n * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
  SL_CUDA(cudaStreamSynchronize(S.stream));
  double t = 0.0;
  for (int i = 0; i < n; ++i) t += S.host_part[i];
  return t;
}

}  // namespace

SlabState *slab_create(int nx, int ny, int nz, int device) {
  if (nx < 1 || ny < 1 || nz < 1) throw std::invalid_argument("slab dimensions must be positive");
  if ((long long)pitch4(nx + 2) * (ny + 2) * (nz + 2) >= (1LL << 31)) throw std::invalid_argument("slab too large");
  SL_CUDA(cudaSetDevice(device));
  std::unique_ptr<SlabState> S(new SlabState());
  S->device = device;
  S->nx = nx; S->ny = ny; S->nz = nz; S->px = pitch4(nx + 2);
  S->np = (size_t)S->px * (ny + 2) * (nz + 2);
  SL_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
  SlabDev &D = S->D;
  D.nx = nx; D.ny = ny; D.nz = nz; D.px = S->px;
  double *g[3];
  for (double *&a : g) a = S->alloc<double>(S->np);
  D.gx = g[0]; D.gy = g[1]; D.gz = g[2];
  D.x = S->alloc<double>(S->np); D.r = S->alloc<double>(S->np);
  D.p = S->alloc<double>(S->np); D.s = S->alloc<double>(S->np);
  S->b = S->alloc<double>(S->np);
  // the hierarchy: level 0 on the slab's couplings, 2x coarser levels below
  mg::Hier<double> &G = S->G;
  int lx = nx, ly = ny, lz = nz, L = 0;
  while (true) {
    if (L >= mg::kMgMaxLv) throw std::runtime_error("multigrid: too many levels");
    mg::Level<double> &l = G.lv[L];
    l.nx = lx; l.ny = ly; l.nz = lz; l.px = pitch4(lx + 2);
    const size_t n = (size_t)l.px * (ly + 2) * (lz + 2);
    l.x = S->alloc<double>(n); l.rhs = S->alloc<double>(n);
    if (L == 0) {
      l.gx = g[0]; l.gy = g[1]; l.gz = g[2];
      l.d = S->alloc<double>(n);
    } else {
      l.gx = S->alloc<double>(n); l.gy = S->alloc<double>(n); l.gz = S->alloc<double>(n);
      l.d = nullptr;
    }
    l.fx = l.fy = l.fz = nullptr;
    l.m = S->alloc<uint8_t>(n);
    ++L;
    if ((long long)lx * ly * lz <= mg::kMgCoarse) break;
    lx = (lx + 1) / 2; ly = (ly + 1) / 2; lz = (lz + 1) / 2;
  }
  G.L = L;
  G.nsw = 2;   // the channel p' solve's sweeps (k_ch_pcg)
  G.nswc = 3;
  G.lu = S->alloc<double>((size_t)mg::kMgCoarse * mg::kMgCoarse);
  mg::plan_stage(G);
  int nsm = 0, per = 0;
  SL_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  SL_CUDA(cudaFuncSetAttribute((const void *)k_sl_vcycle, cudaFuncAttributeMaxDynamicSharedMemorySize, mg::kMgStageTotal));
  SL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_sl_vcycle, kSlVT, G.stage));
  if (per < 1) throw std::runtime_error("slab V-cycle kernel cannot be resident");
  S->vgrid = per * nsm;
  S->part = S->alloc<double>((size_t)std::max(kSlBlocks, S->vgrid));
  SL_CUDA(cudaStreamSynchronize(S->stream));
  return S.release();
}

void slab_destroy(SlabState *S) { delete S; }

namespace {
// a hierarchy for an nx x ny x nz level 0 whose couplings are allocated here
void alloc_hier(SlabState &S, mg::Hier<double> &G, int lx, int ly, int lz, const double *g0x, const double *g0y,
                const double *g0z) {
  int L = 0;
  while (true) {
    if (L >= mg::kMgMaxLv) throw std::runtime_error("multigrid: too many levels");
    mg::Level<double> &l = G.lv[L];
    l.nx = lx; l.ny = ly; l.nz = lz; l.px = pitch4(lx + 2);
    const size_t n = (size_t)l.px * (ly + 2) * (lz + 2);
    l.x = S.alloc<double>(n); l.rhs = S.alloc<double>(n);
    if (L == 0 && g0x) {
      l.gx = const_cast<double *>(g0x); l.gy = const_cast<double *>(g0y); l.gz = const_cast<double *>(g0z);
    } else {
      l.gx = S.alloc<double>(n); l.gy = S.alloc<double>(n); l.gz = S.alloc<double>(n);
    }
    l.d = L == 0 ? S.alloc<double>(n) : nullptr;
    l.fx = l.fy = l.fz = nullptr;
    l.m = S.alloc<uint8_t>(n);
    ++L;
    if ((long long)lx * ly * lz <= mg::kMgCoarse) break;
    lx = (lx + 1) / 2; ly = (ly + 1) / 2; lz = (lz + 1) / 2;
  }
  G.L = L;
  G.nsw = 2;
  G.nswc = 3;
  G.lu = S.alloc<double>((size_t)mg::kMgCoarse * mg::kMgCoarse);
  mg::plan_stage(G);
}

// the padded level-0 couplings, mask and diagonal of hierarchy G from host
// face arrays (as slab_set_system takes them)
void upload_level0(SlabState &S, const mg::Level<double> &L, const double *gx, const double *gy, const double *gz) {
  const int nx = L.nx, ny = L.ny, nz = L.nz, px = L.px;
  const size_t np = (size_t)px * (ny + 2) * (nz + 2);
  auto pq = [&](int i, int j, int k) { return (size_t)i + px * ((size_t)j + (ny + 2) * (size_t)k); };
  std::vector<double> a(np), d(np, 0.0);
  std::vector<uint8_t> m(np, 0);
  const double *src[3] = {gx, gy, gz};
  double *dst[3] = {L.gx, L.gy, L.gz};
  std::vector<double> g[3];
  for (int ax = 0; ax < 3; ++ax) {
    std::fill(a.begin(), a.end(), 0.0);
    const int fx = nx + (ax == 0), fy = ny + (ax == 1), fz = nz + (ax == 2);
    for (int k = 0; k < fz; ++k)
      for (int j = 0; j < fy; ++j)
        for (int i = 0; i < fx; ++i) a[pq(i + 1, j + 1, k + 1)] = src[ax][i + (size_t)fx * (j + (size_t)fy * k)];
    g[ax] = a;
    SL_CUDA(cudaMemcpyAsync(dst[ax], a.data(), np * 8, cudaMemcpyHostToDevice, S.stream));
    SL_CUDA(cudaStreamSynchronize(S.stream));
  }
  const size_t PX = px, PXY = (size_t)px * (ny + 2);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const size_t q = pq(i + 1, j + 1, k + 1);
        const double dv = g[0][q] + g[0][q + 1] + g[1][q] + g[1][q + PX] + g[2][q] + g[2][q + PXY];
        d[q] = dv;
        m[q] = dv > 0.0;
      }
  SL_CUDA(cudaMemcpyAsync(L.d, d.data(), np * 8, cudaMemcpyHostToDevice, S.stream));
  SL_CUDA(cudaMemcpyAsync(L.m, m.data(), np, cudaMemcpyHostToDevice, S.stream));
  SL_CUDA(cudaStreamSynchronize(S.stream));
}
}  // namespace

void slab_set_coarse(SlabState *S, int agg, int kg0, int nzg) {
  if (agg < 2 || kg0 < 0 || kg0 + S->nz > nzg) throw std::invalid_argument("invalid coarse grid");
  if (S->agg) throw std::invalid_argument("the coarse grid is set already");
  S->agg = agg;
  S->kg0 = kg0;
  S->nzg = nzg;
  S->ncx = (S->nx + agg - 1) / agg;
  S->ncy = (S->ny + agg - 1) / agg;
  S->ncz = (nzg + agg - 1) / agg;
  alloc_hier(*S, S->C, S->ncx, S->ncy, S->ncz, nullptr, nullptr, nullptr);
  const size_t nc = (size_t)S->ncx * S->ncy * S->ncz;
  S->crhs = S->alloc<double>(nc);
  S->crc = S->alloc<double>(nc);
  SL_CUDA(cudaFuncSetAttribute((const void *)k_sl_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, mg::kMgStageTotal));
  int nsm = 0, per = 0;
  SL_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, S->device));
  SL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_sl_coarse, kSlVT,
                                                        (size_t)std::max(S->C.stage, S->G.stage)));
  if (per < 1) throw std::runtime_error("slab coarse-correction kernel cannot be resident");
  S->vgrid = std::min(S->vgrid, per * nsm);
  SL_CUDA(cudaStreamSynchronize(S->stream));
}

// the partial coarse face couplings of this slab (sums of its fine faces on
// aggregate faces; a z-face between two slabs counted by the upper one)
void slab_coarse_partial_compute(SlabState *S, const double *gx, const double *gy, const double *gz) {
  if (!S->agg) return;
  const int nx = S->nx, ny = S->ny, nz = S->nz, a = S->agg, kg0 = S->kg0;
  const int ncx = S->ncx, ncy = S->ncy, ncz = S->ncz;
  std::vector<double> &cx = S->cpart[0], &cy = S->cpart[1], &cz = S->cpart[2];
  cx.assign((size_t)(ncx + 1) * ncy * ncz, 0.0);
  cy.assign((size_t)ncx * (ncy + 1) * ncz, 0.0);
  cz.assign((size_t)ncx * ncy * (ncz + 1), 0.0);
  for (int k = 0; k < nz; ++k) {
    const int K = (k + kg0) / a;
    for (int j = 0; j < ny; ++j)
      for (int f = 0; f <= nx; ++f)
        if (f % a == 0 || f == nx) {
          const int I = (f == nx) ? ncx : f / a;
          cx[I + (size_t)(ncx + 1) * (j / a + (size_t)ncy * K)] += gx[f + (size_t)(nx + 1) * (j + (size_t)ny * k)];
        }
    for (int f = 0; f <= ny; ++f)
      if (f % a == 0 || f == ny) {
        const int J = (f == ny) ? ncy : f / a;
        for (int i = 0; i < nx; ++i)
          cy[i / a + (size_t)ncx * (J + (size_t)(ncy + 1) * K)] += gy[i + (size_t)nx * (f + (size_t)(ny + 1) * k)];
      }
  }
  // z faces: local face f (global f + kg0) for f in [0, nz), and the top face
  // nz only when it is the domain's top face (else the slab above owns it)
  for (int f = 0; f <= nz; ++f) {
    const int fg = f + kg0;
    if (f == nz && fg != S->nzg) continue;
    if (!(fg % a == 0 || fg == S->nzg)) continue;  // inside an aggregate
    const int Kf = fg == S->nzg ? ncz : fg / a;
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        cz[i / a + (size_t)ncx * (j / a + (size_t)ncy * Kf)] += gz[i + (size_t)nx * (j + (size_t)ny * f)];
  }
}

void slab_set_system(SlabState *S, const double *gx, const double *gy, const double *gz, const double *b) {
  const int nx = S->nx, ny = S->ny, nz = S->nz, px = S->px;
  const size_t np = S->np;
  auto pq = [&](int i, int j, int k) { return (size_t)i + px * ((size_t)j + (ny + 2) * (size_t)k); };
  std::vector<double> a(np);
  // face f of axis x (0 .. nx) is the low face of cell f: padded (f + 1, j + 1, k + 1)
  std::fill(a.begin(), a.end(), 0.0);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int f = 0; f <= nx; ++f) a[pq(f + 1, j + 1, k + 1)] = gx[f + (size_t)(nx + 1) * (j + (size_t)ny * k)];
  SL_CUDA(cudaMemcpyAsync((void *)S->D.gx, a.data(), np * 8, cudaMemcpyHostToDevice, S->stream));
  SL_CUDA(cudaStreamSynchronize(S->stream));
  std::fill(a.begin(), a.end(), 0.0);
  for (int k = 0; k < nz; ++k)
    for (int f = 0; f <= ny; ++f)
      for (int i = 0; i < nx; ++i) a[pq(i + 1, f + 1, k + 1)] = gy[i + (size_t)nx * (f + (size_t)(ny + 1) * k)];
  SL_CUDA(cudaMemcpyAsync((void *)S->D.gy, a.data(), np * 8, cudaMemcpyHostToDevice, S->stream));
  SL_CUDA(cudaStreamSynchronize(S->stream));
  std::fill(a.begin(), a.end(), 0.0);
  for (int f = 0; f <= nz; ++f)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) a[pq(i + 1, j + 1, f + 1)] = gz[i + (size_t)nx * (j + (size_t)ny * f)];
  SL_CUDA(cudaMemcpyAsync((void *)S->D.gz, a.data(), np * 8, cudaMemcpyHostToDevice, S->stream));
  SL_CUDA(cudaStreamSynchronize(S->stream));
  std::fill(a.begin(), a.end(), 0.0);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) a[pq(i + 1, j + 1, k + 1)] = b[i + (size_t)nx * (j + (size_t)ny * k)];
  SL_CUDA(cudaMemcpyAsync(S->b, a.data(), np * 8, cudaMemcpyHostToDevice, S->stream));
  k_sl_mask<<<kSlBlocks, kSlT, 0, S->stream>>>(S->D, S->G.lv[0].m, S->G.lv[0].d);
  SL_CUDA(cudaGetLastError());
  SL_CUDA(cudaStreamSynchronize(S->stream));
  S->built = false;
  slab_coarse_partial_compute(S, gx, gy, gz);
  S->cbuilt = false;
}

void slab_coarse_sizes(const SlabState *S, long long *n4) {
  n4[0] = (long long)(S->ncx + 1) * S->ncy * S->ncz;
  n4[1] = (long long)S->ncx * (S->ncy + 1) * S->ncz;
  n4[2] = (long long)S->ncx * S->ncy * (S->ncz + 1);
  n4[3] = (long long)S->ncx * S->ncy * S->ncz;
}

void slab_coarse_partial(const SlabState *S, double *cgx, double *cgy, double *cgz) {
  if (!S->agg) throw std::invalid_argument("no coarse grid set (hs_slab_set_coarse)");
  if (S->cpart[0].empty()) throw std::invalid_argument("no system set (hs_slab_set_system)");
  std::copy(S->cpart[0].begin(), S->cpart[0].end(), cgx);
  std::copy(S->cpart[1].begin(), S->cpart[1].end(), cgy);
  std::copy(S->cpart[2].begin(), S->cpart[2].end(), cgz);
}

void slab_coarse_build(SlabState *S, const double *cgx, const double *cgy, const double *cgz) {
  if (!S->agg) throw std::invalid_argument("no coarse grid set (hs_slab_set_coarse)");
  upload_level0(*S, S->C.lv[0], cgx, cgy, cgz);
  S->cbuilt = false;
}

void slab_restrict(SlabState *S, double *rc_host) {
  if (!S->agg) throw std::invalid_argument("no coarse grid set (hs_slab_set_coarse)");
  const CoarseMap M{S->agg, S->kg0, S->ncx, S->ncy, S->ncz};
  const int nc = S->ncx * S->ncy * S->ncz;
  k_sl_restrict<<<std::max(1, std::min((nc + kSlT - 1) / kSlT, kSlBlocks)), kSlT, 0, S->stream>>>(S->D, M, S->crc);
  SL_CUDA(cudaGetLastError());
  SL_CUDA(cudaMemcpyAsync(rc_host, S->crc, (size_t)nc * 8, cudaMemcpyDeviceToHost, S->stream));
  SL_CUDA(cudaStreamSynchronize(S->stream));
}

double slab_coarse_correct(SlabState *S, const double *rc_host) {
  if (!S->agg) throw std::invalid_argument("no coarse grid set (hs_slab_set_coarse)");
  const CoarseMap M{S->agg, S->kg0, S->ncx, S->ncy, S->ncz};
  const size_t nc = (size_t)S->ncx * S->ncy * S->ncz;
  SL_CUDA(cudaMemcpyAsync(S->crhs, rc_host, nc * 8, cudaMemcpyHostToDevice, S->stream));
  const int build = S->cbuilt ? 0 : 1;
  sl_coop(k_sl_coarse, S->vgrid, kSlVT, (size_t)S->C.stage, S->stream, S->D, S->G, S->C, M, (const double *)S->crhs,
          build, S->part);
  S->cbuilt = true;
  return sl_sum(*S, S->vgrid);
}

double slab_begin(SlabState *S) {
  k_sl_begin<<<kSlBlocks, kSlT, 0, S->stream>>>(S->D, S->b, S->part);
  SL_CUDA(cudaGetLastError());
  return sl_sum(*S, kSlBlocks);
}

double slab_precond(SlabState *S) {
  const int build = S->built ? 0 : 1;
  sl_coop(k_sl_vcycle, S->vgrid, kSlVT, (size_t)S->G.stage, S->stream, S->D, S->G, build, S->part);
  S->built = true;
  return sl_sum(*S, S->vgrid);
}

void slab_direction(SlabState *S, double beta, int first) {
  k_sl_direction<<<kSlBlocks, kSlT, 0, S->stream>>>(S->D, (const double *)S->G.lv[0].x, beta, first);
  SL_CUDA(cudaGetLastError());
  SL_CUDA(cudaStreamSynchronize(S->stream));
}

double slab_apply(SlabState *S) {
  k_sl_apply<<<kSlBlocks, kSlT, 0, S->stream>>>(S->D, S->part);
  SL_CUDA(cudaGetLastError());
  return sl_sum(*S, kSlBlocks);
}

double slab_update(SlabState *S, double alpha) {
  k_sl_update<<<kSlBlocks, kSlT, 0, S->stream>>>(S->D, alpha, S->part);
  SL_CUDA(cudaGetLastError());
  return sl_sum(*S, kSlBlocks);
}

long long slab_plane_size(const SlabState *S) { return (long long)S->px * (S->ny + 2); }

void slab_halo_get(SlabState *S, double *lo, double *hi) {
  const size_t pl = (size_t)S->px * (S->ny + 2);
  if (lo) SL_CUDA(cudaMemcpyAsync(lo, S->D.p + pl, pl * 8, cudaMemcpyDeviceToDevice, S->stream));
  if (hi) SL_CUDA(cudaMemcpyAsync(hi, S->D.p + pl * S->nz, pl * 8, cudaMemcpyDeviceToDevice, S->stream));
  SL_CUDA(cudaStreamSynchronize(S->stream));
}

void slab_halo_put(SlabState *S, const double *lo, const double *hi) {
  const size_t pl = (size_t)S->px * (S->ny + 2);
  if (lo) SL_CUDA(cudaMemcpyAsync(S->D.p, lo, pl * 8, cudaMemcpyDeviceToDevice, S->stream));
  if (hi) SL_CUDA(cudaMemcpyAsync(S->D.p + pl * (S->nz + 1), hi, pl * 8, cudaMemcpyDeviceToDevice, S->stream));
  SL_CUDA(cudaStreamSynchronize(S->stream));
}

void slab_get(SlabState *S, int which, double *host) {
  const double *src = which == 0 ? S->D.x : which == 1 ? S->D.r : which == 2 ? S->D.p : S->D.s;
  std::vector<double> a(S->np);
  SL_CUDA(cudaMemcpyAsync(a.data(), src, S->np * 8, cudaMemcpyDeviceToHost, S->stream));
  SL_CUDA(cudaStreamSynchronize(S->stream));
  const int nx = S->nx, ny = S->ny, px = S->px;
  for (int k = 0; k < S->nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        host[i + (size_t)nx * (j + (size_t)ny * k)] = a[(i + 1) + px * ((size_t)(j + 1) + (ny + 2) * (size_t)(k + 1))];
}

}  // namespace hs
