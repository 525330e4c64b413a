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
