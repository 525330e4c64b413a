// z-marching passes over level 0 of the pressure-correction V-cycle and its
// CG, with the planes staged in shared memory by the Tensor Memory
// Accelerator (TMA).  Device code only; every pass runs inside the
// cooperative kernel of the p' solve (hs_channel.cu).
//
// Work split.  The level's interior is cut into kTX x kTY tiles in (x, y)
// and its planes into nch z-chunks; a unit is one tile over one chunk (a
// segment of consecutive planes).  The units, in chunk-major order, are dealt
// round-robin over the blocks, so the blocks of one round march over
// neighbouring tiles of the same chunk at the same time and each halo row a
// block stages is, most of the time, a row its neighbour staged moments
// before (in L2).  The host picks nch to balance the rounds against the two
// extra planes each segment stages at either end.  Every pass has two stages
// per z step t:
//   stage 1: a value v1 on the tile and a one-cell ring around it (T+1) at
//            plane t, kept in a three-plane shared-memory ring;
//   stage 2: the pass's outputs on the tile (T) at plane t - 1, from the v1
//            ring (planes t - 2 .. t) and the staged inputs.
// The ring cells of T+1 belong to the neighbouring tiles: they are computed
// again here from the same inputs, so no block waits for another within a
// pass and every output is a pure function of the pass's inputs (the passes
// read one buffer and write another).
//   Red-black Gauss-Seidel sweep: v1 = the first colour's update on T+1 (from
//     the input x), stage 2 = the second colour's update on T (from v1); the
//     sweep of both colours costs one pass over the level instead of two.
//   A p: v1 = p = z + beta p_old on T+1, stage 2 = s = A p on T.
//   The CG update: v1 = the seed of the V-cycle (red cells, x = r / d with
//     r = r_old - alpha s) on T+1, stage 2 = the black half-sweep, and on T
//     x += alpha p, r written.
// Every point update is the expression of the grid-wide passes of hs_mg.cuh
// in the same operation order, so the V-cycle gives the same values bit for
// bit; only the dot products are summed in another order.
//
// Staging.  Each input array is a 3-D tensor map over its padded layout (row
// pitch a multiple of 16 bytes); one plane of a box of BX x BY values around
// the tile (T plus two cells each side, x widened to 16-byte boundaries) is
// one cp.async.bulk.tensor load into shared memory; loads outside the array
// (below plane 0 of the padded grid, left of its column 0) are zero-filled by
// the TMA unit.  A ring of SLOTS planes (5 in FP64, 7 in FP32), each holding
// the pass's five boxes (and a coarse-level box for the prolongation), is
// filled SLOTS - 3 planes ahead of the last plane stage 1 reads; one
// mbarrier per slot counts the bytes.  No multicast: every load is this
// block's own.
//
// Waits.  Every wait on an mbarrier polls with a limit of kWaitNs of wall
// time (%globaltimer); a wait that runs out marks the block failed, after
// which it issues no loads and waits no more, but still takes every barrier
// of the kernel, and the failure reaches the host through the next grid-wide
// reduction (the solve reports -1 iterations).
#pragma once
#include <cuda.h>

#include <cstdint>

#include "hs_mg.cuh"

namespace hs {
namespace zm {

constexpr int kTX = 32, kTY = 16;  // tile interior (x, y)
constexpr int kBoxes = 5;          // fine-level boxes per plane
constexpr int kThreads = 512;      // threads per block: one per tile cell in stage 2
constexpr unsigned long long kWaitNs = 200ull * 1000 * 1000;  // one wait: 0.2 s of wall time

// geometry of a box of precision M: A values per 16 bytes; the box starts A
// values left of the tile's first padded column (a 16-byte boundary when the
// tile origin is) and spans the tile, two cells each side and the
// alignment; rows: two each side
template <class M>
struct Box {
  static constexpr int A = 16 / (int)sizeof(M);
  static constexpr int BX = (kTX + 3 + A + A - 1) / A * A;
  static constexpr int BY = kTY + 4;
  static constexpr int N = BX * BY;
  static constexpr int BYTES = N * (int)sizeof(M);
  static constexpr int STRIDE = (BYTES + 127) / 128 * 128;
  // the coarse level's box for the prolongation: parents of the fine box's
  // cells (x from the tile origin / 2, a 16-byte boundary)
  static constexpr int CBX = (kTX / 2 + 2 + A - 1) / A * A;
  static constexpr int CBY = kTY / 2 + 2;
  static constexpr int CBYTES = CBX * CBY * (int)sizeof(M);
  static constexpr int CSTRIDE = (CBYTES + 127) / 128 * 128;
  static constexpr int SLOT = kBoxes * STRIDE + CSTRIDE;
  // planes in the staging ring: three resident, the rest in flight (two
  // planes of FP64 boxes, four of FP32, per block)
  static constexpr int SLOTS = sizeof(M) == 8 ? 5 : 7;
  // shared memory of the passes: the ring, the v1 ring, the mbarriers
  static constexpr int SMEM = SLOTS * SLOT + 3 * STRIDE + SLOTS * 8;
};

// ---------------------------------------------------------------- PTX
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t gtime() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// the mbarrier initialisations visible to the async proxy (the TMA unit)
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// waits (suspended in hardware, up to a system-dependent time) for the phase
// with the given parity to complete; true when it has
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// one box of a 3-D tiled tensor map into shared memory, completing bytes on bar
__device__ __forceinline__ void tma_load3(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// generic-proxy writes to global memory ordered before later async-proxy
// (TMA) reads of it, on either side of a grid barrier
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// ---------------------------------------------------------------- the staging ring
// Per block, uniform over its threads: loads issued and waited (the n-th load
// goes to slot n % SLOTS; its mbarrier phase parity is (n / SLOTS) & 1; after
// a failure the counts go on, so that the slots stay in step, but nothing is
// loaded or waited for), loads seen complete (ok) and really issued (live),
// and the failure flag.
struct Pipe {
  uint32_t issued, waited, ok, live;
  int fail;
};

// the maps a pass stages: five fine boxes (order: x-like, r-like, gx, gy, gz)
// and, for the prolongation, the coarse level's x
struct PassMaps {
  const CUtensorMap *m[kBoxes];
  const CUtensorMap *coarse;
};

template <class M>
struct Smem {
  unsigned char *base;
  __device__ __forceinline__ M *box(int slot, int b) const {
    return reinterpret_cast<M *>(base + slot * Box<M>::SLOT + b * Box<M>::STRIDE);
  }
  __device__ __forceinline__ M *cbox(int slot) const {
    return reinterpret_cast<M *>(base + slot * Box<M>::SLOT + kBoxes * Box<M>::STRIDE);
  }
  __device__ __forceinline__ M *ring(int r) const {
    return reinterpret_cast<M *>(base + Box<M>::SLOTS * Box<M>::SLOT + r * Box<M>::STRIDE);
  }
  __device__ __forceinline__ uint64_t *bars() const {
    return reinterpret_cast<uint64_t *>(base + Box<M>::SLOTS * Box<M>::SLOT + 3 * Box<M>::STRIDE);
  }
};

// thread 0: the boxes of interior plane k of the tile at (i0, j0) into the
// next slot (the slot's previous contents are consumed: every thread passed
// the barrier that follows its last read)
template <class M>
__device__ __forceinline__ void issue(const Smem<M> &S, Pipe &P, const PassMaps &pm, int i0, int j0, int k) {
  const int slot = (int)(P.issued % Box<M>::SLOTS);
  P.issued++;
  if (P.fail) return;
  P.live = P.issued;
  if (threadIdx.x != 0) return;
  uint64_t *bar = S.bars() + slot;
  const uint32_t bytes = kBoxes * Box<M>::BYTES + (pm.coarse ? Box<M>::CBYTES : 0);
  mbar_expect_tx(bar, bytes);
  const int x = i0 - Box<M>::A, y = j0 - 1, z = k + 1;  // padded coordinates of the box origin
  for (int b = 0; b < kBoxes; ++b) tma_load3(S.box(slot, b), pm.m[b], bar, x, y, z);
  if (pm.coarse) tma_load3(S.cbox(slot), pm.coarse, bar, i0 / 2, j0 / 2, (k >> 1) + 1);
}

// every thread: wait for the next load in order (bounded)
template <int SLOTS>
__device__ __forceinline__ void wait_next(uint64_t *bars, Pipe &P) {
  const uint32_t n = P.waited++;
  if (P.fail) return;
  uint64_t *bar = bars + n % SLOTS;
  const uint32_t par = (n / SLOTS) & 1u;
  if (!mbar_try(bar, par)) {
    const uint64_t t0 = gtime();
    while (!mbar_try(bar, par))
      if (gtime() - t0 > kWaitNs) {
        P.fail = 1;
        return;
      }
  }
  P.ok = n + 1;
}

// after a failure: wait (bounded, briefly) for the loads issued and not seen
// complete, so that no TMA write lands in shared memory after the block has
// moved on
template <int SLOTS>
__device__ __forceinline__ void drain(uint64_t *bars, Pipe &P) {
  for (uint32_t n = P.ok; n < P.live; ++n) {
    uint64_t *bar = bars + n % SLOTS;
    const uint32_t par = (n / SLOTS) & 1u;
    const uint64_t t0 = gtime();
    while (!mbar_test(bar, par))
      if (gtime() - t0 > kWaitNs / 4) break;
  }
  P.ok = P.live;
}

// ---------------------------------------------------------------- work split
struct Tiles {
  int nx, ny, nz, px;  // level interior and row pitch
  int ntx, nty;        // tiles per axis
  int nch;             // z-chunks
};

// the z-chunk count for `ntiles` tiles of nz planes over `blocks` blocks:
// the fewest rounds of units weighed against the two planes each segment
// stages beyond either end, i.e. minimal ceil(ntiles nch / blocks) * (nz /
// nch + 4), the first such nch
inline int pick_chunks(int ntiles, int nz, int blocks) {
  int best = 1;
  double cost = 1e300;
  for (int c = 1; c <= (nz + 3) / 4; ++c) {
    const long long rounds = ((long long)ntiles * c + blocks - 1) / blocks;
    const double v = (double)rounds * ((double)(nz + c - 1) / c + 4.0);
    if (v < cost) { cost = v; best = c; }
  }
  return best;
}

// local (box) coordinates of interior cell (i, j) of the tile at (i0, j0)
template <class M>
__device__ __forceinline__ int lq(int i, int j, int i0, int j0) {
  return (j - j0 + 2) * Box<M>::BX + (i - i0 + 1 + Box<M>::A);
}

// ---------------------------------------------------------------- pass kinds
enum Kind { kSeed = 0, kSweep = 1, kProlong = 2, kAp = 3 };

// one pass's inputs and outputs (device pointers of the padded arrays, row pitch px)
template <class M>
struct PassArgs {
  int kind;
  int c1;            // sweeps: colour of stage 1 ((i + j + k) & 1); stage 2 takes the other
  int dot;           // sweeps: add sum r x_out over T to the block's dot (kSweep, kProlong)
  int upd;           // kSeed: the CG update (x += alpha p, r = r_old - alpha s) before the seed
  double alpha;      // kSeed with upd
  M beta;            // kAp: p = z + beta p_old (first: p = z)
  int first;         // kAp
  M *out;            // sweeps and kSeed: the level's new x; kAp: the new p
  M *out2;           // kSeed with upd: the new r; kAp: s
  M *xcg;            // kSeed with upd: the CG's x (read and written on T)
  const M *pcg;      // kSeed with upd: the CG's p (read on T)
};

// the staged value of box b at local index q of the plane in slot s
#define ZM_AT(b, s, q) (S.box((s), (b))[(q)])

// One pass over this block's tile-planes.  acc: this thread's share of the
// pass's dot product (kSeed with upd: sum r^2; kAp: sum s p; sweeps with dot:
// sum r x).
template <class M>
__device__ void run_pass(const Smem<M> &S, Pipe &P, const PassMaps &pm, const Tiles &Tl, const PassArgs<M> &a,
                         double &acc) {
  constexpr int BX = Box<M>::BX, NS = Box<M>::SLOTS;
  const int nx = Tl.nx, ny = Tl.ny, nz = Tl.nz, PX = Tl.px;
  uint64_t *bars = S.bars();
  const int ntiles = Tl.ntx * Tl.nty, units = ntiles * Tl.nch;
  const int t_id = threadIdx.x, NT = kThreads;
  for (int u = blockIdx.x; u < units; u += gridDim.x) {
    const int chunk = u / ntiles, tile = u - chunk * ntiles;
    const int k0 = (int)((long long)nz * chunk / Tl.nch), k1 = (int)((long long)nz * (chunk + 1) / Tl.nch);
    if (k1 <= k0) continue;
    const int i0 = (tile % Tl.ntx) * kTX, j0 = (tile / Tl.ntx) * kTY;
    // planes k0 - 2 .. k1 + 1 are staged, in order; slot of plane k
    const uint32_t base = P.issued;
    const int kfirst = k0 - 2, klast = k1 + 1;
    auto slot_of = [&](int k) { return (int)((base + (uint32_t)(k - kfirst)) % NS); };
    for (int k = kfirst; k <= klast && k < kfirst + NS; ++k) issue(S, P, pm, i0, j0, k);
    int next = kfirst + NS;  // next plane to issue
    // this thread's stage-2 cell at plane k: for A p the tile in row order;
    // for the colour passes threads 0..255 take the second colour's cells and
    // 256..511 the first colour's (row j0 + m / 16, its m % 16-th cell of the
    // colour), so that no warp splits between updating and copying
    auto cell = [&](int k, int &ci, int &cj) {
      if (a.kind == kAp) {
        ci = i0 + (t_id % kTX);
        cj = j0 + (t_id / kTX);
      } else {
        const int m = t_id & (kTX * kTY / 2 - 1);
        const int colour = t_id < kTX * kTY / 2 ? 1 - a.c1 : a.c1;
        cj = j0 + m / (kTX / 2);
        ci = i0 + 2 * (m % (kTX / 2)) + ((colour - cj - k) & 1);
      }
    };
    // the CG's x and p of this thread's stage-2 cell, one plane ahead
    M xpre = M(0), ppre = M(0);
    if (a.kind == kSeed && a.upd) {
      int ci, cj;
      cell(k0, ci, cj);
      if (ci < nx && cj < ny) {
        const int g = (ci + 1) + PX * ((cj + 1) + (ny + 2) * (k0 + 1));
        xpre = a.xcg[g];
        ppre = a.pcg[g];
      }
    }
    for (int t = k0 - 1; t <= k1; ++t) {
      // planes t - 1 .. t + 1 resident
      if (t == k0 - 1) {
        wait_next<NS>(bars, P);
        wait_next<NS>(bars, P);
      }
      wait_next<NS>(bars, P);
      const int s0 = slot_of(t), sp = slot_of(t + 1), sm = slot_of(t - 1);
      M *v1 = S.ring((t + 3) % 3);
      // ---- stage 1 on T+1 at plane t
      const bool tin = t >= 0 && t < nz;
      if (a.kind == kAp) {
        for (int e = t_id; e < (kTX + 2) * (kTY + 2); e += NT) {
          const int i = i0 - 1 + e % (kTX + 2), j = j0 - 1 + e / (kTX + 2);
          const int q = lq<M>(i, j, i0, j0);
          const M z = ZM_AT(0, s0, q);
          const M p = a.first ? z : z + a.beta * ZM_AT(1, s0, q);
          v1[q] = (tin && i >= 0 && i < nx && j >= 0 && j < ny) ? p : M(0);
        }
      } else {
        constexpr int HR = (kTX + 2) / 2;  // cells of one colour per ring row
        for (int e = t_id; e < HR * (kTY + 2); e += NT) {
          const int j = j0 - 1 + e / HR;
          const int ib = i0 - 1;
          const int i = ib + ((a.c1 - ib - j - t) & 1) + 2 * (e % HR);
          const int q = lq<M>(i, j, i0, j0);
          M v = M(0);
          if (tin && i >= 0 && i < nx && j >= 0 && j < ny) {
            const M gxl = ZM_AT(2, s0, q), gxh = ZM_AT(2, s0, q + 1), gyl = ZM_AT(3, s0, q), gyh = ZM_AT(3, s0, q + BX);
            const M gzl = ZM_AT(4, s0, q), gzh = ZM_AT(4, sp, q);
            const M d = ((gxl + gxh) + (gyl + gyh)) + (gzl + gzh);
            if (a.kind == kSeed) {
              const M rn = a.upd ? (M)((double)ZM_AT(0, s0, q) - a.alpha * (double)ZM_AT(1, s0, q)) : ZM_AT(0, s0, q);
              v = d == M(0) ? M(0) : rn / d;
            } else {
              M xw, xe, xs, xn, xb, xf;
              if (a.kind == kProlong) {
                // neighbour values x + x_coarse(parent), 0 at a ghost (never prolonged)
                const M *cb = S.cbox(s0), *cbm = S.cbox(sm), *cbp = S.cbox(sp);
                auto cq = [&](int ii, int jj) { return ((jj >> 1) + 1 - j0 / 2) * Box<M>::CBX + ((ii >> 1) + 1 - i0 / 2); };
                xw = i > 0 ? ZM_AT(0, s0, q - 1) + cb[cq(i - 1, j)] : M(0);
                xe = i + 1 < nx ? ZM_AT(0, s0, q + 1) + cb[cq(i + 1, j)] : M(0);
                xs = j > 0 ? ZM_AT(0, s0, q - BX) + cb[cq(i, j - 1)] : M(0);
                xn = j + 1 < ny ? ZM_AT(0, s0, q + BX) + cb[cq(i, j + 1)] : M(0);
                xb = t > 0 ? ZM_AT(0, sm, q) + cbm[cq(i, j)] : M(0);
                xf = t + 1 < nz ? ZM_AT(0, sp, q) + cbp[cq(i, j)] : M(0);
              } else {
                xw = ZM_AT(0, s0, q - 1);
                xe = ZM_AT(0, s0, q + 1);
                xs = ZM_AT(0, s0, q - BX);
                xn = ZM_AT(0, s0, q + BX);
                xb = ZM_AT(0, sm, q);
                xf = ZM_AT(0, sp, q);
              }
              const M off = gxl * xw + gxh * xe + gyl * xs + gyh * xn + gzl * xb + gzh * xf;
              const M s = ZM_AT(1, s0, q) + off;
              v = d == M(0) ? M(0) : s / d;
            }
          }
          v1[q] = v;
        }
      }
      __syncthreads();
      // ---- stage 2 on T at plane t - 1
      const int k = t - 1;
      if (k >= k0) {
        const M *vm = S.ring((k + 2) % 3), *vc = S.ring((k + 3) % 3), *vp = v1;  // planes k - 1, k, k + 1
        int i, j;
        cell(k, i, j);
        if (i < nx && j < ny) {
          const int q = lq<M>(i, j, i0, j0);
          const int g = (i + 1) + PX * ((j + 1) + (ny + 2) * (k + 1));
          const M gxl = ZM_AT(2, sm, q), gxh = ZM_AT(2, sm, q + 1), gyl = ZM_AT(3, sm, q), gyh = ZM_AT(3, sm, q + BX);
          const M gzl = ZM_AT(4, sm, q), gzh = ZM_AT(4, s0, q);
          if (a.kind == kAp) {
            const double cw = gxl, ce = gxh, cs = gyl, cn = gyh, cb = gzl, cf = gzh;
            const double d = cw + ce + cs + cn + cb + cf;
            const M p0 = vc[q];
            const double sv = d * (double)p0 - (cw * (double)vc[q - 1] + ce * (double)vc[q + 1] + cs * (double)vc[q - BX] +
                                                cn * (double)vc[q + BX] + cb * (double)vm[q] + cf * (double)vp[q]);
            a.out[g] = p0;
            a.out2[g] = (M)sv;
            acc += (double)(M)sv * (double)p0;
          } else {
            const bool second = t_id < kTX * kTY / 2;  // ((i + j + k) & 1) != c1
            M rhs;
            if (a.kind == kSeed && a.upd) rhs = (M)((double)ZM_AT(0, sm, q) - a.alpha * (double)ZM_AT(1, sm, q));
            else rhs = ZM_AT(a.kind == kSeed ? 0 : 1, sm, q);
            M v = vc[q];
            if (second) {
              const M d = ((gxl + gxh) + (gyl + gyh)) + (gzl + gzh);
              const M off = gxl * vc[q - 1] + gxh * vc[q + 1] + gyl * vc[q - BX] + gyh * vc[q + BX] + gzl * vm[q] + gzh * vp[q];
              const M s = rhs + off;
              v = d == M(0) ? M(0) : s / d;
            }
            a.out[g] = v;
            if (a.kind == kSeed && a.upd) {
              a.out2[g] = rhs;
              a.xcg[g] = (M)((double)xpre + a.alpha * (double)ppre);
              acc += (double)rhs * (double)rhs;
            } else if (a.dot) {
              acc += (double)rhs * (double)v;
            }
          }
        }
        if (a.kind == kSeed && a.upd && k + 1 < k1) {  // the next plane's x and p
          int ci, cj;
          cell(k + 1, ci, cj);
          if (ci < nx && cj < ny) {
            const int g = (ci + 1) + PX * ((cj + 1) + (ny + 2) * (k + 2));
            xpre = a.xcg[g];
            ppre = a.pcg[g];
          }
        }
      }
      // every read of plane t - 1's slot is done: refill it with plane `next`
      P.fail = __syncthreads_or(P.fail);
      if (next <= klast) issue(S, P, pm, i0, j0, next++);
    }
    if (P.fail) drain<NS>(bars, P);
  }
}

#undef ZM_AT

}  // namespace zm
}  // namespace hs
