// Channel conjugate-heat-transfer SIMPLE solver on the GPU.
//
// The reference solves a lid-driven cavity only; this is the extended
// physics of the build (inlet, outlet, heat source, conductivity ratio,
// global residual), with the reference's differencing scheme (first-order
// upwind a_nb = D + max(-+F, 0), a_P = sum a_nb, fluid_solver.h:577-659) kept.
//
//   faces of axis a, index c = (i,j,k), c_a in [0, N_a] (x-fastest, unpadded):
//     c_a = 0      x: inlet (u = u_in over fluid cells); y, z: wall (0)
//     c_a = N_a    x: outlet, u = u*(N_x - 1) + d p'(N_x - 1); y, z: wall (0)
//     otherwise    unknown when both cells are fluid, else 0
//   momentum at an unknown face, coefficients frozen at u^n, Patankar relaxation:
//     (a_P/alpha_u) u_P = sum a_nb u_nb + (p_lo - p_hi) A + (1 - alpha_u)(a_P/alpha_u) u^n_P
//     stencil order E W N S T B; the outlet neighbour is zero-gradient (dropped),
//     a wall or inlet neighbour is 0 at half a cell; d = A / (a_P/alpha_u)
//   convection scheme: first-order upwind (above; the reference's), hybrid
//     a_nb = max(-+F, D -+ F/2, 0), or QUICK by deferred correction: the upwind
//     operator implicit and b += sum over the control-volume faces of
//     -+F (u_f^QUICK - u_f^upwind) at u^n, the QUICK value from per-axis weight
//     tables (quick_weights; upwind where the far-upwind node is off the grid)
//   buoyancy (Boussinesq): b += ri (T_f - t_in) A h on the faces of axis
//     g_axis, T_f the mean of the two cells' T^n
//   red-black Gauss-Seidel on the face colour (i+j+k)&1: one pass per colour,
//   all three components in one launch (they only read each other's u^n)
//   p': couplings A d per face (A d(N_x - 1) at the outlet, p' = 0 outside),
//     b = mass imbalance of u* (u*(N_x) := u*(N_x - 1)); SPD, CG preconditioned
//     by a geometric multigrid V-cycle
//   correction u = u* + d (p'_lo - p'_hi), p += alpha_p p'
//   energy: the conjugate-heat-transfer operator of hs_cht.cu (bc = 1) with a
//     warm-started BiCGStab and relaxation alpha_t
// Every point update is written in the operation order of the CPU oracle, with
// FMA contraction off, so the FP64 form reproduces it bit for bit; sums of
// residuals and dot products are per-block partials reduced in a fixed order.
//
// Precision: R = double (plain form) or float (mixed form: the momentum and
// energy steps in correction form, with FP64 residuals and FP32 sweeps,
// Krylov vectors and V-cycles; dot products, mass imbalance, the p and T
// updates and the coarsest-grid solve in FP64).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "hs_channel.hpp"
#include "hs_cht.hpp"
#include "hs_mg.cuh"
#include "hs_zm.cuh"

namespace cg = cooperative_groups;

namespace hs {

#define CH_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_) + \
                                                    " at " #call);                                 \
  } while (0)

namespace {

constexpr int kT = 256;

// Device view.  U and p are the FP64 iterate in both forms.  In the FP64 form
// C aliases U and S holds u*; in the mixed form C is an FP32 copy of U (the
// coefficient arithmetic reads it), S holds the correction delta = u* - u^n
// swept in FP32, and Q the FP64 residual of the relaxed equation at u^n
// rounded to FP32 (the right-hand side of the delta equation): iterative
// refinement, so the FP32 rounding scales with delta, which vanishes at the
// fixed point.
template <class R>
struct ChDev {
  int N0, N1, N2;
  int PX;                     // row pitch of the padded p' arrays (a multiple of 4 values, >= N0 + 2)
  const R *d0, *d1, *d2;      // cell widths
  const R *h0, *h1, *h2;      // centre distances, [0] and [N] half widths
  const uint8_t *solid;       // N0 N1 N2
  double *U0, *U1, *U2;       // u^n (after correction: the new iterate)
  R *C0, *C1, *C2;            // coefficient copy of U
  R *S0, *S1, *S2;            // u* (FP64) or delta (mixed)
  R *Q0, *Q1, *Q2;            // mixed: right-hand side of the delta sweeps
  R *D0, *D1, *D2;            // d = A / (a_P / alpha_u)
  double *p;                  // pressure, cells
  R nu, au, u_in;
  double ap;                  // alpha_p
  const double *xd0, *xd1, *xd2, *xh0, *xh1, *xh2;  // FP64 geometry (the residual of the mixed form)
  double nu_d, au_d, u_in_d;
  // correctly rounded reciprocals of the divisors known ahead (FP64 arithmetic only)
  const double *rd0, *rd1, *rd2, *rh0, *rh1, *rh2;  // 1 / cell width, 1 / centre distance
  double rau;                                       // 1 / alpha_u
  int conv;           // 0 upwind, 1 hybrid, 2 QUICK (deferred correction)
  int g_axis;         // buoyancy along + this axis
  double ri, t_in;    // Richardson number (0: no buoyancy), reference temperature
  const double *T;    // T^n, padded cells (row pitch N0 + 2), the energy solver's array
  const double *qw[3][2];  // QUICK weights per axis: [0] cell nodes, [1] face nodes (6 per control-volume face)
};

__host__ __device__ constexpr bool is_mixed(float) { return true; }
__host__ __device__ constexpr bool is_mixed(double) { return false; }

template <int A, class R> __device__ __forceinline__ double *Uarr(const ChDev<R> &H) { return A == 0 ? H.U0 : A == 1 ? H.U1 : H.U2; }
template <int A, class R> __device__ __forceinline__ R *Carr(const ChDev<R> &H) { return A == 0 ? H.C0 : A == 1 ? H.C1 : H.C2; }
template <int A, class R> __device__ __forceinline__ R *Sarr(const ChDev<R> &H) { return A == 0 ? H.S0 : A == 1 ? H.S1 : H.S2; }
template <int A, class R> __device__ __forceinline__ R *Qarr(const ChDev<R> &H) { return A == 0 ? H.Q0 : A == 1 ? H.Q1 : H.Q2; }
template <int A, class R> __device__ __forceinline__ R *Darr(const ChDev<R> &H) { return A == 0 ? H.D0 : A == 1 ? H.D1 : H.D2; }
template <int A, class R> __device__ __forceinline__ R wid(const ChDev<R> &H, int i) { return A == 0 ? H.d0[i] : A == 1 ? H.d1[i] : H.d2[i]; }
template <int A, class R> __device__ __forceinline__ R ctr(const ChDev<R> &H, int i) { return A == 0 ? H.h0[i] : A == 1 ? H.h1[i] : H.h2[i]; }
template <int A, class R> __device__ __forceinline__ int ncell(const ChDev<R> &H) { return A == 0 ? H.N0 : A == 1 ? H.N1 : H.N2; }
template <int A, class R> __device__ __forceinline__ double rwid(const ChDev<R> &H, int i) { return A == 0 ? H.rd0[i] : A == 1 ? H.rd1[i] : H.rd2[i]; }
template <int A, class R> __device__ __forceinline__ double rctr(const ChDev<R> &H, int i) { return A == 0 ? H.rh0[i] : A == 1 ? H.rh1[i] : H.rh2[i]; }

// a / b.  In FP64, for a divisor known ahead of time, from its correctly
// rounded reciprocal y = RN(1/b) (Markstein, IBM J. Res. Dev. 34(1), 1990):
// q = RN(a y) is within one ulp of a/b, the remainder a - q b is exact in one
// FMA, and RN(q + r y) is the correctly rounded quotient -- the IEEE value,
// for finite normal operands and a nonzero a (as tests/test_gpu_division.py
// checks for the same construction on the reference path).  FP32 (the mixed
// form's correction sweeps, whose operator only approximates the FP64 one:
// the fixed point is set by the FP64 residual) takes the fast approximate
// quotient (2 ulp), 0.68 -> 0.58 ms per mixed momentum solve at 256x128x128.
__device__ __forceinline__ double div_known(double a, double b, double y) {
  const double q = a * y;
  const double r = __fma_rn(-q, b, a);
  return __fma_rn(r, y, q);
}
__device__ __forceinline__ float div_known(float a, float b, double) { return __fdividef(a, b); }

template <int A, class R>
__device__ __forceinline__ int fidx(const ChDev<R> &H, int i, int j, int k) {
  return i + (H.N0 + (A == 0)) * (j + (H.N1 + (A == 1)) * k);
}
template <class R>
__device__ __forceinline__ int cidx(const ChDev<R> &H, int i, int j, int k) { return i + H.N0 * (j + H.N1 * k); }

template <class R> __device__ __forceinline__ R rmax0(R a) { return a < R(0) ? R(0) : a; }  // maxd(a, 0)

// 0 unknown, 1 fixed, 2 outlet
template <int A, class R>
__device__ __forceinline__ int face_kind(const ChDev<R> &H, const int (&c)[3]) {
  const int f = c[A];
  if (f == 0 || f == ncell<A>(H)) return (A == 0 && f == H.N0) ? 2 : 1;
  int lo[3] = {c[0], c[1], c[2]};
  lo[A] -= 1;
  return (!H.solid[cidx(H, lo[0], lo[1], lo[2])] && !H.solid[cidx(H, c[0], c[1], c[2])]) ? 0 : 1;
}

template <int A, class R>
__device__ __forceinline__ R face_fixed(const ChDev<R> &H, const int (&c)[3]) {
  if (A == 0 && c[0] == 0 && !H.solid[cidx(H, 0, c[1], c[2])]) return H.u_in;
  return R(0);
}

template <int A, class R>
__device__ __forceinline__ R face_area(const ChDev<R> &H, const int (&c)[3]) {
  if (A == 0) return H.d1[c[1]] * H.d2[c[2]];
  if (A == 1) return H.d0[c[0]] * H.d2[c[2]];
  return H.d0[c[0]] * H.d1[c[1]];
}

template <int A, class R>
__device__ __forceinline__ int fidx3(const ChDev<R> &H, const int (&c)[3]) { return fidx<A>(H, c[0], c[1], c[2]); }

template <class R> __device__ __forceinline__ R rmaxd(R a, R b) { return a < b ? b : a; }  // maxd(a, b)

// coefficient of the neighbour across a control-volume face of conductance D
// and flux F (+ direction) on its high (HI) or low side: upwind D + max(-+F, 0),
// or hybrid max(-+F, D -+ F/2, 0)
template <int HI, class R>
__device__ __forceinline__ R anb(int conv, R D, R F) {
  if (conv == 1) return HI ? rmaxd(rmaxd(-F, D - R(0.5) * F), R(0)) : rmaxd(rmaxd(F, D + R(0.5) * F), R(0));
  return HI ? D + rmax0(-F) : D + rmax0(F);
}

// QUICK deferred-correction term F (u_f^QUICK - u_f^upwind) of the control-
// volume face e along axis B of component A, from u^n (FP64): the nodes are
// A's faces with the index along B replaced (faces of axis B itself when
// B == A, kind 1: e between nodes e and e + 1; cell centres otherwise, kind
// 0: e between nodes e - 1 and e); weights (far upwind, upwind, downwind)
// for the flux direction, (0, 1, 0) where a node is off the grid
template <int A, int B, class R>
__device__ __forceinline__ double quick_term(const ChDev<R> &H, const int (&c)[3], int e, double F) {
  constexpr int kind = B == A;
  const double *w = H.qw[B][kind] + 6 * e + (F > 0.0 ? 0 : 3);
  const int lo = kind ? e : e - 1;
  int iuu = F > 0.0 ? lo - 1 : lo + 2, iu = F > 0.0 ? lo : lo + 1, id = F > 0.0 ? lo + 1 : lo;
  const double w0 = w[0], w1 = w[1], w2 = w[2];
  if (w0 == 0.0 && w2 == 0.0) iuu = id = iu;
  const double *UA = Uarr<A>(H);
  int q[3] = {c[0], c[1], c[2]};
  q[B] = iuu;
  const double uuu = UA[fidx3<A>(H, q)];
  q[B] = iu;
  const double uu = UA[fidx3<A>(H, q)];
  q[B] = id;
  const double ud = UA[fidx3<A>(H, q)];
  const double uq = (w0 * uuu + w1 * uu) + w2 * ud;
  return F * (uq - uu);
}

// one stencil term (neighbour across axis B, high side when HI) of the unknown
// face (A, c): coefficient at the frozen iterate and the neighbour's face
// index (-1: the neighbour value is 0 or the term is dropped)
template <int A, int B, int HI, int X, class R>
__device__ __forceinline__ void term(const ChDev<R> &H, const int (&c)[3], R Ar, R da, R &coef, int &nb, R &Fo, int &eo) {
  const int conv = X == 0 ? 0 : X == 1 ? 1 : H.conv;
  coef = R(0);
  nb = -1;
  Fo = R(0);
  eo = 0;
  const R *CA = Carr<A>(H);
  if constexpr (B == A) {
    int q[3] = {c[0], c[1], c[2]};
    if (HI) {
      q[A] += 1;
      if (!(A == 0 && q[0] == H.N0)) {
        const R F = R(0.5) * (CA[fidx3<A>(H, c)] + CA[fidx3<A>(H, q)]) * Ar;
        const R Dd = div_known(H.nu * Ar, wid<A>(H, c[A]), rwid<A>(H, c[A]));
        coef = anb<1>(conv, Dd, F);
        nb = fidx3<A>(H, q);
        Fo = F;
        eo = c[A];
      }
    } else {
      q[A] -= 1;
      const R F = R(0.5) * (CA[fidx3<A>(H, q)] + CA[fidx3<A>(H, c)]) * Ar;
      const R Dd = div_known(H.nu * Ar, wid<A>(H, c[A] - 1), rwid<A>(H, c[A] - 1));
      coef = anb<0>(conv, Dd, F);
      nb = fidx3<A>(H, q);
      Fo = F;
      eo = c[A] - 1;
    }
  } else {
    constexpr int O = 3 - A - B;
    const R *CB = Carr<B>(H);
    const R wo = wid<O>(H, c[O]);
    const R ar = da * wo;
    int flo[3] = {c[0], c[1], c[2]}, fhi[3] = {c[0], c[1], c[2]};
    flo[A] -= 1;
    if (HI) { flo[B] += 1; fhi[B] += 1; }
    const R F = R(0.5) * (CB[fidx3<B>(H, flo)] * wid<A>(H, c[A] - 1) + CB[fidx3<B>(H, fhi)] * wid<A>(H, c[A])) * wo;
    int q[3] = {c[0], c[1], c[2]};
    Fo = F;
    if (HI) {
      if (c[B] + 1 == ncell<B>(H)) {
        if (B != 0) coef = anb<1>(conv, div_known(H.nu * ar, ctr<B>(H, ncell<B>(H)), rctr<B>(H, ncell<B>(H))), F);
      } else {
        coef = anb<1>(conv, div_known(H.nu * ar, ctr<B>(H, c[B] + 1), rctr<B>(H, c[B] + 1)), F);
        q[B] += 1;
        nb = fidx3<A>(H, q);
        eo = c[B] + 1;
      }
    } else {
      if (c[B] == 0) {
        coef = anb<0>(conv, div_known(H.nu * ar, ctr<B>(H, 0), rctr<B>(H, 0)), F);
      } else {
        coef = anb<0>(conv, div_known(H.nu * ar, ctr<B>(H, c[B]), rctr<B>(H, c[B])), F);
        q[B] -= 1;
        nb = fidx3<A>(H, q);
        eo = c[B];
      }
    }
  }
}

// The source terms beyond the pressure term of the unknown face (A, c), in
// FP64 from u^n and T^n: bs (the pressure term) plus the QUICK deferred
// correction (stencil order, - on the high faces, + on the low ones) and the
// Boussinesq term, in the oracle's order
template <int A>
__device__ __forceinline__ double add_sources(const ChDev<double> &H, const int (&c)[3], const int (&nb)[6],
                                              const double (&F)[6], const int (&e)[6], double A_, double da, double bs) {
  if (H.conv == 2) {
    double dc = 0.0;
    if (nb[0] >= 0) dc -= quick_term<A, 0>(H, c, e[0], F[0]);
    if (nb[1] >= 0) dc += quick_term<A, 0>(H, c, e[1], F[1]);
    if (nb[2] >= 0) dc -= quick_term<A, 1>(H, c, e[2], F[2]);
    if (nb[3] >= 0) dc += quick_term<A, 1>(H, c, e[3], F[3]);
    if (nb[4] >= 0) dc -= quick_term<A, 2>(H, c, e[4], F[4]);
    if (nb[5] >= 0) dc += quick_term<A, 2>(H, c, e[5], F[5]);
    bs = bs + dc;
  }
  if (H.ri != 0.0 && A == H.g_axis) {
    int lo[3] = {c[0], c[1], c[2]};
    lo[A] -= 1;
    const int P0 = H.N0 + 2, P1 = H.N1 + 2;
    const double tl = H.T[(lo[0] + 1) + P0 * ((lo[1] + 1) + P1 * (lo[2] + 1))];
    const double th = H.T[(c[0] + 1) + P0 * ((c[1] + 1) + P1 * (c[2] + 1))];
    bs = bs + H.ri * (0.5 * (tl + th) - H.t_in) * A_ * da;
  }
  return bs;
}

// Mixed form, first pass: the FP64 form's residual of the relaxed equation
// at u^n (FP64 coefficients from the FP64 iterate), stored rounded to FP32
// as the right-hand side of the correction sweeps, and the first half-sweep
// of the correction (neighbour corrections are still 0).  The sweeps that
// follow use FP32 coefficients from the FP32 copy, which only approximates
// the correction operator: the fixed point solves the FP64 equations (defect
// correction).
template <int A, int X>
__device__ __forceinline__ void mom_face_mixed_first(const ChDev<float> &H, const int (&c)[3], int f, bool upd,
                                                     bool last, double &racc, bool keep) {
  ChDev<double> H64;
  H64.N0 = H.N0; H64.N1 = H.N1; H64.N2 = H.N2;
  H64.d0 = H.xd0; H64.d1 = H.xd1; H64.d2 = H.xd2; H64.h0 = H.xh0; H64.h1 = H.xh1; H64.h2 = H.xh2;
  H64.solid = H.solid;
  H64.U0 = H.U0; H64.U1 = H.U1; H64.U2 = H.U2;
  H64.C0 = H.U0; H64.C1 = H.U1; H64.C2 = H.U2;
  H64.p = H.p; H64.nu = H.nu_d; H64.au = H.au_d; H64.u_in = H.u_in_d;
  H64.rd0 = H.rd0; H64.rd1 = H.rd1; H64.rd2 = H.rd2; H64.rh0 = H.rh0; H64.rh1 = H.rh1; H64.rh2 = H.rh2;
  H64.rau = H.rau;
  H64.conv = H.conv; H64.g_axis = H.g_axis; H64.ri = H.ri; H64.t_in = H.t_in; H64.T = H.T;
  for (int a = 0; a < 3; ++a) { H64.qw[a][0] = H.qw[a][0]; H64.qw[a][1] = H.qw[a][1]; }
  const double Ad = face_area<A>(H64, c);
  const double dad = ctr<A>(H64, c[A]);
  double ad[6], Fd[6];
  int nd[6], ed[6];
  term<A, 0, 1, X>(H64, c, Ad, dad, ad[0], nd[0], Fd[0], ed[0]);
  term<A, 0, 0, X>(H64, c, Ad, dad, ad[1], nd[1], Fd[1], ed[1]);
  term<A, 1, 1, X>(H64, c, Ad, dad, ad[2], nd[2], Fd[2], ed[2]);
  term<A, 1, 0, X>(H64, c, Ad, dad, ad[3], nd[3], Fd[3], ed[3]);
  term<A, 2, 1, X>(H64, c, Ad, dad, ad[4], nd[4], Fd[4], ed[4]);
  term<A, 2, 0, X>(H64, c, Ad, dad, ad[5], nd[5], Fd[5], ed[5]);
  const double aPd = ad[0] + ad[1] + ad[2] + ad[3] + ad[4] + ad[5];
  const double *UA = Uarr<A>(H);
  int lo[3] = {c[0], c[1], c[2]};
  lo[A] -= 1;
  double bs = (H.p[cidx(H, lo[0], lo[1], lo[2])] - H.p[cidx(H, c[0], c[1], c[2])]) * Ad;
  if constexpr (X == 2) bs = add_sources<A>(H64, c, nd, Fd, ed, Ad, dad, bs);
  double s = 0.0;
#pragma unroll
  for (int n = 0; n < 6; ++n) s += ad[n] * (nd[n] >= 0 ? UA[nd[n]] : 0.0);
  const double r = (s + bs) - aPd * UA[f];
  if (!keep) return;
  racc += r * r;
  const float rhs = (float)r;
  Qarr<A>(H)[f] = rhs;
  if (upd) {
    const float apr = (float)div_known(aPd, H.au_d, H.rau);
    Sarr<A>(H)[f] = rhs / apr;
    if (last) Darr<A>(H)[f] = face_area<A>(H, c) / apr;
  }
}

// momentum work on the unknown face (A, c): residual at u^n (first pass),
// relaxed Gauss-Seidel update (upd), d (last sweep)
template <int A, int X, class R>
__device__ __forceinline__ void mom_face(const ChDev<R> &H, const int (&c)[3], bool first, bool upd, bool last,
                                         double &racc, bool keep) {
  const int f = fidx3<A>(H, c);
  if constexpr (is_mixed(R())) {
    if (first) {
      mom_face_mixed_first<A, X>(H, c, f, upd, last, racc, keep);
      return;
    }
  }
  const R Ar = face_area<A>(H, c);
  const R da = ctr<A>(H, c[A]);
  R an[6], Fn[6];
  int nb[6], en[6];
  term<A, 0, 1, X>(H, c, Ar, da, an[0], nb[0], Fn[0], en[0]);
  term<A, 0, 0, X>(H, c, Ar, da, an[1], nb[1], Fn[1], en[1]);
  term<A, 1, 1, X>(H, c, Ar, da, an[2], nb[2], Fn[2], en[2]);
  term<A, 1, 0, X>(H, c, Ar, da, an[3], nb[3], Fn[3], en[3]);
  term<A, 2, 1, X>(H, c, Ar, da, an[4], nb[4], Fn[4], en[4]);
  term<A, 2, 0, X>(H, c, Ar, da, an[5], nb[5], Fn[5], en[5]);
  const R aP = an[0] + an[1] + an[2] + an[3] + an[4] + an[5];
  const R apr = div_known(aP, H.au, H.rau);
  const double *UA = Uarr<A>(H);
  R *SA = Sarr<A>(H);
  if constexpr (!is_mixed(R())) {
    // u* in place: a_P/alpha u_P = sum a_nb u_nb + b + (1 - alpha) a_P/alpha u^n_P
    int lo[3] = {c[0], c[1], c[2]};
    lo[A] -= 1;
    R bs = (H.p[cidx(H, lo[0], lo[1], lo[2])] - H.p[cidx(H, c[0], c[1], c[2])]) * Ar;
    if constexpr (X == 2) bs = add_sources<A>(H, c, nb, Fn, en, Ar, da, bs);
    const R un = UA[f];
    const R *src = first ? (const R *)UA : (const R *)SA;
    if (first) {
      double s = 0.0;
#pragma unroll
      for (int n = 0; n < 6; ++n) s += (double)an[n] * (nb[n] >= 0 ? UA[nb[n]] : 0.0);
      const double r = (double)aP * (double)un - (s + (double)bs);
      if (keep) racc += r * r;
    }
    if (upd) {
      R s = R(0);
#pragma unroll
      for (int n = 0; n < 6; ++n) s += an[n] * (nb[n] >= 0 ? src[nb[n]] : R(0));
      const R rhs = s + bs + (R(1) - H.au) * apr * un;
      if (keep) {
        SA[f] = rhs / apr;
        if (last) Darr<A>(H)[f] = Ar / apr;
      }
    }
  } else {
    // correction sweeps after the first pass (FP32 operator, FP32 right-hand side from the first pass)
    const R rhs = Qarr<A>(H)[f];
    if (upd && keep) {
      R s = R(0);
#pragma unroll
      for (int n = 0; n < 6; ++n) s += an[n] * (nb[n] >= 0 ? SA[nb[n]] : R(0));
      SA[f] = __fdividef(rhs + s, apr);
      if (last) Darr<A>(H)[f] = Ar / apr;
    }
  }
}

__device__ double block_sum(double v, double *sh) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid_ = threadIdx.x >> 5;
  if (lane == 0) sh[wid_] = v;
  __syncthreads();
  double t = 0.0;
  if (wid_ == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;
}

// One red-black pass of all three momentum components (component A).
// first: the pass of colour 0 in sweep 0, which also evaluates the residual of
// every unknown face at u^n and writes the fixed faces of u* (delta = 0).
template <int A, int X, class R>
__device__ void mom_pass_axis(const ChDev<R> &H, int color, bool first, bool last, double &racc) {
  const int nf0 = H.N0 + (A == 0), nf1 = H.N1 + (A == 1), nf2 = H.N2 + (A == 2);
  // blocks 3b, 3b + 1, 3b + 2 take chunk b of the three components (k_ch_mom)
  const int T = (gridDim.x / 3) * blockDim.x, tid = (blockIdx.x / 3) * blockDim.x + threadIdx.x;
  if (first) {
    for (mg::Walk w(nf0, nf1, nf2, tid, T); w.ok(); w.next()) {
      const int c[3] = {w.m, w.j, w.k};
      const int f = fidx3<A>(H, c);
      if (c[A] == 0 || c[A] == ncell<A>(H)) {  // boundary faces: fixed or outlet (an index test)
        Sarr<A>(H)[f] = is_mixed(R()) ? R(0) : face_fixed<A>(H, c);
        Darr<A>(H)[f] = R(0);
        continue;
      }
      // an interior face: its update is evaluated whatever the solid mask
      // says (every index it reads is valid) and kept only for an unknown
      // face, so that no branch on the mask waits ahead of the stencil loads
      const bool keep = face_kind<A>(H, c) == 0;
      const bool mine = ((c[0] + c[1] + c[2]) & 1) == color;
      mom_face<A, X>(H, c, true, mine, last && mine, racc, keep);
      if (!keep) {
        Sarr<A>(H)[f] = R(0);
        Darr<A>(H)[f] = R(0);
      }
    }
  } else {
    for (mg::Walk w((nf0 + 1) / 2, nf1, nf2, tid, T); w.ok(); w.next()) {
      const int j = w.j, k = w.k, i = 2 * w.m + ((j + k + color) & 1);
      if (i >= nf0) continue;
      const int c[3] = {i, j, k};
      if (c[A] == 0 || c[A] == ncell<A>(H)) continue;
      mom_face<A, X>(H, c, false, true, last, racc, face_kind<A>(H, c) == 0);
    }
  }
}

// four 256-thread blocks per SM (64 registers: above that the SM holds three).
// X: 0 first-order upwind, 1 hybrid, 2 any scheme with the source terms
// (QUICK deferred correction, buoyancy): separate instantiations, so that the
// upwind and hybrid forms keep their registers (the source-term one spills
// 360 B at 64 registers, and is still faster than at 80 registers without
// spills and three blocks per SM: 1.42 against 1.58 ms per momentum solve).
// The grid is 3 x (chunks): the three components of one chunk of faces are
// consecutive blocks, so they run at the same time and share the u^n they
// all read in L2 (component-major order read the three velocity arrays once
// per component from DRAM: 0.80 -> 0.71 ms per FP64 momentum solve at
// 256x128x128).
template <class R, int X>
__global__ void __launch_bounds__(kT, 4) k_ch_mom(ChDev<R> H, int color, int first, int last, double *partials) {
  __shared__ double sh[32];
  double racc = 0.0;
  const int comp = blockIdx.x % 3;
  if (comp == 0) mom_pass_axis<0, X>(H, color, first, last, racc);
  else if (comp == 1) mom_pass_axis<1, X>(H, color, first, last, racc);
  else mom_pass_axis<2, X>(H, color, first, last, racc);
  if (first) {
    const double b = block_sum(racc, sh);
    if (threadIdx.x == 0) partials[comp * (gridDim.x / 3) + blockIdx.x / 3] = b;
  }
}

// padded cell index of the CG arrays
__device__ __forceinline__ int pq(int PX, int N1, int i, int j, int k) { return (i + 1) + PX * ((j + 1) + (N1 + 2) * (k + 1)); }

// u* of a face in FP64
template <int A, class R>
__device__ __forceinline__ double ustar(const ChDev<R> &H, int f) {
  if constexpr (is_mixed(R())) return Uarr<A>(H)[f] + (double)Sarr<A>(H)[f];
  else return Sarr<A>(H)[f];
}

// p' couplings per face into padded cell arrays (the coupling of the face on a
// cell's low side; the outlet face sits in the ghost cell i = N0) and the mass
// imbalance b per cell (r = b, x = 0)
template <class R>
__global__ void k_ch_passemble(ChDev<R> H, R *acx, R *acy, R *acz, R *r, R *x, double *partials) {
  __shared__ double sh[32];
  const int T = gridDim.x * blockDim.x, tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int N0 = H.N0, N1 = H.N1, N2 = H.N2;
  double acc = 0.0;
  if (blockIdx.y == 0) {
    // every value a face may need is loaded before its kind (from the solid
    // mask) is known, so no branch on the mask waits ahead of the loads
    for (mg::Walk w(N0 + 1, N1, N2, tid, T); w.ok(); w.next()) {
      const int c[3] = {w.m, w.j, w.k};
      const double dn = c[0] < N0 ? (double)H.D0[fidx3<0>(H, c)] : 0.0;
      const double dl = c[0] > 0 ? (double)H.D0[fidx<0>(H, c[0] - 1, c[1], c[2])] : 0.0;
      const bool lo_fluid = c[0] > 0 && !H.solid[cidx(H, c[0] - 1, c[1], c[2])];
      const int kind = face_kind<0>(H, c);
      double v = 0.0;
      if (kind == 0) v = (double)face_area<0>(H, c) * dn;
      else if (kind == 2 && lo_fluid) v = (double)face_area<0>(H, c) * dl;
      acx[pq(H.PX, N1, c[0], c[1], c[2])] = (R)v;
    }
  } else if (blockIdx.y == 1) {
    for (mg::Walk w(N0, N1 + 1, N2, tid, T); w.ok(); w.next()) {
      const int c[3] = {w.m, w.j, w.k};
      const double dn = (double)H.D1[fidx3<1>(H, c)];
      acy[pq(H.PX, N1, c[0], c[1], c[2])] = (R)(face_kind<1>(H, c) == 0 ? (double)face_area<1>(H, c) * dn : 0.0);
    }
  } else if (blockIdx.y == 2) {
    for (mg::Walk w(N0, N1, N2 + 1, tid, T); w.ok(); w.next()) {
      const int c[3] = {w.m, w.j, w.k};
      const double dn = (double)H.D2[fidx3<2>(H, c)];
      acz[pq(H.PX, N1, c[0], c[1], c[2])] = (R)(face_kind<2>(H, c) == 0 ? (double)face_area<2>(H, c) * dn : 0.0);
    }
  } else {
    for (mg::Walk w(N0, N1, N2, tid, T); w.ok(); w.next()) {
      const int i = w.m, j = w.j, k = w.k, e = w.flat();
      const int q = pq(H.PX, N1, i, j, k);
      const bool sol = H.solid[e] != 0;
      const double uw = ustar<0>(H, fidx<0>(H, i, j, k));
      const double ue = (i + 1 == N0) ? uw : ustar<0>(H, fidx<0>(H, i + 1, j, k));
      const double b = (uw - ue) * ((double)H.d1[j] * (double)H.d2[k]) +
                       (ustar<1>(H, fidx<1>(H, i, j, k)) - ustar<1>(H, fidx<1>(H, i, j + 1, k))) * ((double)H.d0[i] * (double)H.d2[k]) +
                       (ustar<2>(H, fidx<2>(H, i, j, k)) - ustar<2>(H, fidx<2>(H, i, j, k + 1))) * ((double)H.d0[i] * (double)H.d1[j]);
      x[q] = R(0);
      r[q] = sol ? R(0) : (R)b;
      if (!sol) acc += b * b;
    }
  }
  const double bsum = block_sum(acc, sh);
  if (threadIdx.x == 0 && blockIdx.y == 3) partials[blockIdx.x] = bsum;
}

// The four-part correction pass (k_ch_correct): block b does part b % 4 (u,
// v, w, p) on chunk b / 4 of that part's elements in flat order, kT * per of
// them (thread t: chunk * kT * per + t + kT m, m < per).  The resident blocks
// of the four parts then cover the same z-planes at a time, so p', which
// every part reads, comes from DRAM once (with the parts one after another it
// came four times), and the block scheduler balances parts of unequal cost:
// 0.102 -> 0.094 ms FP64, 0.126 -> 0.114 ms mixed at 256x128x128.  The
// p' assembly's parts share only the solid mask and are slower dealt this
// way (0.101 -> 0.114 ms: more arrays streaming at once).
struct ChunkWalk : mg::Walk {
  int left;
  __device__ __forceinline__ ChunkWalk(int mx, int ny, int nz, int per)
      : mg::Walk(mx, ny, nz, (int)(blockIdx.x >> 2) * kT * per + (int)threadIdx.x, kT), left(per) {}
  __device__ __forceinline__ bool ok() const { return left > 0 && mg::Walk::ok(); }
  __device__ __forceinline__ void next() {
    --left;
    mg::Walk::next();
  }
};

template <int A, class R>
__device__ void correct_axis(const ChDev<R> &H, const R *pp, int per) {
  const int nf0 = H.N0 + (A == 0), nf1 = H.N1 + (A == 1), nf2 = H.N2 + (A == 2);
  for (ChunkWalk w(nf0, nf1, nf2, per); w.ok(); w.next()) {
    const int c[3] = {w.m, w.j, w.k};
    const int e = w.flat();
    // mixed form: u* = u^n + delta is read from u^n, which this pass
    // replaces, so the outlet face (from its upstream face's u*) is written
    // by the thread of that upstream face, after its own loads (below)
    if (is_mixed(R()) && A == 0 && c[0] == H.N0) continue;
    // the values of every case are loaded before the face kind (from the
    // solid mask) selects one; p' is padded, so its ghost cells are readable
    int lo[3] = {c[0], c[1], c[2]};
    lo[A] -= 1;
    const double plo = (double)pp[pq(H.PX, H.N1, lo[0], lo[1], lo[2])];
    const double phi = (double)pp[pq(H.PX, H.N1, c[0], c[1], c[2])];
    const double sf = is_mixed(R()) ? ustar<A>(H, e) : (double)Sarr<A>(H)[e];
    const double df = (double)Darr<A>(H)[e];
    double so = 0.0, dso = 0.0;  // the outlet's upstream face (x faces)
    bool lo_solid = true;
    if (A == 0 && c[0] == H.N0) {
      so = is_mixed(R()) ? ustar<0>(H, e - 1) : (double)H.S0[e - 1];
      dso = (double)H.D0[e - 1];
      lo_solid = H.solid[cidx(H, c[0] - 1, c[1], c[2])] != 0;
    }
    const bool feeds_outlet = is_mixed(R()) && A == 0 && c[0] == H.N0 - 1;
    const bool up_solid = feeds_outlet && H.solid[cidx(H, c[0], c[1], c[2])] != 0;
    const int kind = face_kind<A>(H, c);
    double val;
    if (kind == 1) val = (double)face_fixed<A>(H, c);
    else if (kind == 2) val = lo_solid ? 0.0 : so + dso * plo;
    else val = sf + df * (plo - phi);
    Uarr<A>(H)[e] = val;
    if constexpr (is_mixed(R())) {
      Carr<A>(H)[e] = (R)val;
      if (feeds_outlet) {  // the outlet face e + 1, as the FP64 form computes it
        const double vo = up_solid ? 0.0 : sf + df * phi;
        Uarr<0>(H)[e + 1] = vo;
        Carr<0>(H)[e + 1] = (R)vo;
      }
    }
  }
}

// a four-part pass (ChunkWalk): u, v, w and p, every part reading p'
template <class R>
__global__ void __launch_bounds__(kT) k_ch_correct(ChDev<R> H, const R *pp, int per) {
  const int part = blockIdx.x & 3;
  if (part == 0) correct_axis<0>(H, pp, per);
  else if (part == 1) correct_axis<1>(H, pp, per);
  else if (part == 2) correct_axis<2>(H, pp, per);
  else {
    for (ChunkWalk w(H.N0, H.N1, H.N2, per); w.ok(); w.next()) {
      const int e = w.flat();
      if (H.solid[e]) continue;
      H.p[e] = H.p[e] + H.ap * pp[pq(H.PX, H.N1, w.m, w.j, w.k)];
    }
  }
}

// initial state: u = u_in on the inlet, unknown and outlet faces over fluid, 0 elsewhere; v = w = 0; p = 0
template <class R>
__global__ void k_ch_init(ChDev<R> H) {
  const long long n0 = (long long)(H.N0 + 1) * H.N1 * H.N2;
  const long long n1 = (long long)H.N0 * (H.N1 + 1) * H.N2, n2 = (long long)H.N0 * H.N1 * (H.N2 + 1);
  const long long nc = (long long)H.N0 * H.N1 * H.N2;
  const R s0 = is_mixed(R()) ? R(0) : R(1);  // u* starts at u (FP64 form), delta at 0 (mixed)
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n0 + n1 + n2 + nc; e += gridDim.x * blockDim.x) {
    if (e < n0) {
      const int c[3] = {(int)(e % (H.N0 + 1)), (int)((e / (H.N0 + 1)) % H.N1), (int)(e / ((long long)(H.N0 + 1) * H.N1))};
      const int kind = face_kind<0>(H, c);
      R v = R(0);
      if (kind == 0) v = H.u_in;
      else if (kind == 1) v = face_fixed<0>(H, c);
      else v = H.solid[cidx(H, c[0] - 1, c[1], c[2])] ? R(0) : H.u_in;
      H.U0[e] = (double)v; H.S0[e] = s0 * v; H.D0[e] = R(0);
      if constexpr (is_mixed(R())) { H.C0[e] = v; H.Q0[e] = R(0); }
    } else if (e < n0 + n1) {
      const long long f = e - n0;
      H.U1[f] = 0.0; H.S1[f] = R(0); H.D1[f] = R(0);
      if constexpr (is_mixed(R())) { H.C1[f] = R(0); H.Q1[f] = R(0); }
    } else if (e < n0 + n1 + n2) {
      const long long f = e - n0 - n1;
      H.U2[f] = 0.0; H.S2[f] = R(0); H.D2[f] = R(0);
      if constexpr (is_mixed(R())) { H.C2[f] = R(0); H.Q2[f] = R(0); }
    } else {
      H.p[e - n0 - n1 - n2] = 0.0;
    }
  }
}

// ---------------------------------------------------------------- multigrid-preconditioned CG
// Symmetric operator on padded cells: (A x)_q = sum_f c_f (x_q - x_nb), with
// c stored on each cell's low face (acx[q] couples q-1 and q; acx of the
// ghost cell N0 + 1 is the outlet face, neighbour value 0).  Preconditioner:
// the V-cycle of hs_mg.cuh in precision M on the same couplings (no
// convection), solid cells masked.
// p' system and CG vectors, stored in V (FP64 form: double; mixed form:
// float, with the search-direction update in FP32 and the product, the x and r
// updates and the dot products in FP64: p' is a correction that vanishes at
// the fixed point, whose residuals are all FP64)
template <class V>
struct CgVec {
  int N0, N1, N2;
  int px;  // row pitch of every padded array (ChDev::PX)
  int nch;  // the z-marching form's z-chunks (zm::pick_chunks)
  const V *acx, *acy, *acz;
  const uint8_t *solid;
  V *x, *r, *p, *p2, *s;  // p, p2: search direction, double-buffered
  V *r2;                  // the z-marching form's second residual buffer
};

__device__ double grid_sum(double v, double *partials, int &buf, double *sh, cg::grid_group &grid) {
  double *pp = partials + (size_t)buf * gridDim.x;
  buf ^= 1;
  const double b = block_sum(v, sh);
  if (threadIdx.x == 0) pp[blockIdx.x] = b;
  grid.sync();
  double a = 0.0;
  if (threadIdx.x < 32) {
    for (int q = threadIdx.x; q < (int)gridDim.x; q += 32) a += __ldcg(pp + q);
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (threadIdx.x == 0) sh[32] = a;
  }
  __syncthreads();
  a = sh[32];
  __syncthreads();
  return a;
}

// padded index (row pitch PX) of the cell with flat index e (x fastest)
__device__ __forceinline__ int cell_q(int e, int N0, int N1, int PX) {
  const int row_ = e / N0, i = e - row_ * N0;
  const int k = row_ / N1, j = row_ - k * N1;
  return (i + 1) + PX * ((j + 1) + (N1 + 2) * (k + 1));
}

// one block per SM (few arrivals at every grid barrier), its size by
// precision: 512 threads for FP64 (128 registers, no spills) and 640 for FP32,
// the fastest of 512 / 640 / 768 / 1024 for each on a 256x128x128 channel
// (FP64 5.32 / 5.56 / 5.85 / 5.49 ms per solve, FP32 3.99 / 3.62 / 3.65 /
// 3.81)
template <class M>
struct PcgT {
  static constexpr int v = 640;
};
template <>
struct PcgT<double> {
  static constexpr int v = 512;
};

// One pass over the padded cells: level 0 of the V-cycle (its couplings are
// the CG's own arrays, the same pointers; the mask and the diagonal of every
// row) and, on the interior, the V-cycle's right-hand side r with its seed
// (which needs only the cell's own diagonal) and this thread's share of <r, r>
template <class M>
__device__ void mg_fine_and_rhs(const CgVec<M> &V, const mg::Level<M> &L0, double &acc, int tid, int T) {
  for (mg::Walk w(V.px, V.N1 + 2, V.N2 + 2, tid, T); w.ok(); w.next()) {
    const int q = w.flat(), i = w.m - 1, j = w.j - 1, k = w.k - 1;
    const bool in = i >= 0 && j >= 0 && k >= 0 && i < V.N0 && j < V.N1 && k < V.N2;
    M d = M(0), o[6];
    double rv = 0.0;
    bool solid = true;
    if (in) {
      mg::row(L0, q, false, d, o);
      rv = (double)V.r[q];
      solid = V.solid[i + V.N0 * (j + V.N1 * k)] != 0;
    }
    L0.m[q] = in && !solid;
    L0.d[q] = d;
    if (in) {
      acc += rv * rv;
      mg::seed_store(L0, q, i, j, k, (M)rv, d);
    }
  }
}

// The mixed form's two CG passes by runs of W consecutive padded cells of
// an interior row per thread step (W = 2 or 4; aligned: the row pitch is a
// multiple of four values), with 8- or 16-byte loads and stores: a fraction
// 1/W of the load and store instructions of the per-cell passes, whose FP32
// form was bound by them rather than by DRAM bytes.  Lanes outside the
// interior (the ghost cells and the row's padding) compute from in-bounds
// loads and store the zeros those cells hold.  Every interior cell's
// arithmetic is the per-cell pass's, term for term; only the order of this
// thread's dot-product terms differs.  Mixed p' solve per outer step at
// 256x128x128: 3.39 ms per cell, 3.15 ms with W = 2, 3.11 ms with W = 4
// (which spills 64 bytes at the kernel's 96 registers, and is still faster).
constexpr int kCgRun = 4;

template <int W>
__device__ __forceinline__ void ldv(float (&v)[W], const float *p, bool cg_) {
  if constexpr (W == 4) {
    const float4 t = cg_ ? __ldcg(reinterpret_cast<const float4 *>(p)) : *reinterpret_cast<const float4 *>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else {
    const float2 t = cg_ ? __ldcg(reinterpret_cast<const float2 *>(p)) : *reinterpret_cast<const float2 *>(p);
    v[0] = t.x; v[1] = t.y;
  }
}
template <int W>
__device__ __forceinline__ void stv(float *p, const float (&v)[W]) {
  if constexpr (W == 4) *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  else *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
}
// p = z + beta p_old (or z in the first iteration) at the run q0
template <int W>
__device__ __forceinline__ void p_run(float (&v)[W], const float *zs, const float *po, int q0, bool first, float bm) {
  ldv<W>(v, zs + q0, true);
  if (!first) {
    float o[W];
    ldv<W>(o, po + q0, true);
#pragma unroll
    for (int c = 0; c < W; ++c) v[c] = v[c] + bm * o[c];
  }
}
__device__ __forceinline__ float p_one(const float *zs, const float *po, int q, bool first, float bm) {
  const float z = __ldcg(zs + q);
  return first ? z : z + bm * __ldcg(po + q);
}

// s = A p with the new p formed on the way (k_ch_pcg's first pass); returns
// this thread's share of <s, p>
template <int W>
__device__ double cg_ap_runs(const CgVec<float> &V, const float *zs, const float *po, float *pn, bool first, float bm,
                             int tid, int T) {
  const int N0 = V.N0, PX = V.px, PY = V.N1 + 2, PXY = V.px * (V.N1 + 2);
  double acc = 0.0;
  for (mg::Walk w(PX / W, V.N1, V.N2, tid, T); w.ok(); w.next()) {
    const int q0 = W * w.m + PX * ((w.j + 1) + PY * (w.k + 1));
    // the sums d = cw + ce + cs + cn + cb + cf and o = cw pW + ce pE + cs pS
    // + cn pN + cb pB + cf pF built up in that order, one neighbour run at a
    // time (fewer values live at once)
    float pc[W + 2], g[W + 1], v[W], h[W];
    double d[W], o[W];
    p_run<W>(v, zs, po, q0, first, bm);
    pc[0] = p_one(zs, po, q0 - 1, first, bm);
#pragma unroll
    for (int c = 0; c < W; ++c) pc[c + 1] = v[c];
    pc[W + 1] = p_one(zs, po, q0 + W, first, bm);
    ldv<W>(v, V.acx + q0, false);
#pragma unroll
    for (int c = 0; c < W; ++c) g[c] = v[c];
    g[W] = V.acx[q0 + W];
#pragma unroll
    for (int c = 0; c < W; ++c) {
      d[c] = (double)g[c] + (double)g[c + 1];
      o[c] = (double)g[c] * (double)pc[c] + (double)g[c + 1] * (double)pc[c + 2];
    }
    p_run<W>(v, zs, po, q0 - PX, first, bm);
    ldv<W>(h, V.acy + q0, false);
#pragma unroll
    for (int c = 0; c < W; ++c) { d[c] = d[c] + (double)h[c]; o[c] = o[c] + (double)h[c] * (double)v[c]; }
    p_run<W>(v, zs, po, q0 + PX, first, bm);
    ldv<W>(h, V.acy + q0 + PX, false);
#pragma unroll
    for (int c = 0; c < W; ++c) { d[c] = d[c] + (double)h[c]; o[c] = o[c] + (double)h[c] * (double)v[c]; }
    p_run<W>(v, zs, po, q0 - PXY, first, bm);
    ldv<W>(h, V.acz + q0, false);
#pragma unroll
    for (int c = 0; c < W; ++c) { d[c] = d[c] + (double)h[c]; o[c] = o[c] + (double)h[c] * (double)v[c]; }
    p_run<W>(v, zs, po, q0 + PXY, first, bm);
    ldv<W>(h, V.acz + q0 + PXY, false);
    float pv[W], sv[W];
#pragma unroll
    for (int c = 0; c < W; ++c) {
      d[c] = d[c] + (double)h[c];
      o[c] = o[c] + (double)h[c] * (double)v[c];
      const int i = W * w.m + c;  // padded x
      const bool in = i >= 1 && i <= N0;
      const float p0 = pc[c + 1];
      const double s_ = d[c] * (double)p0 - o[c];
      pv[c] = in ? p0 : 0.0f;
      sv[c] = in ? (float)s_ : 0.0f;
      if (in) acc += (double)(float)s_ * (double)p0;
    }
    stv<W>(pn + q0, pv);
    stv<W>(V.s + q0, sv);
  }
  return acc;
}

// x += alpha p, r -= alpha s and, with the V-cycle, its level-0 right-hand
// side r and the seed of the first half-sweep (x = r / d on colour 0; colour
// 1, which the next half-sweep writes before any pass reads it, gets 0);
// returns this thread's share of <r, r>
template <int W>
__device__ double cg_update_runs(const CgVec<float> &V, const mg::Level<float> &L0, bool pre, const float *pn,
                                 double alpha, int tid, int T) {
  const int N0 = V.N0, PX = V.px, PY = V.N1 + 2;
  double acc = 0.0;
  for (mg::Walk w(PX / W, V.N1, V.N2, tid, T); w.ok(); w.next()) {
    const int q0 = W * w.m + PX * ((w.j + 1) + PY * (w.k + 1));
    float xv[W], pv[W], rv[W], sv[W], dv[W];
    ldv<W>(xv, V.x + q0, false);
    ldv<W>(pv, pn + q0, false);
    ldv<W>(rv, V.r + q0, false);
    ldv<W>(sv, V.s + q0, false);
    if (pre) ldv<W>(dv, L0.d + q0, false);
    else
#pragma unroll
      for (int c = 0; c < W; ++c) dv[c] = 0.0f;
    float xo[W], ro[W], sx[W];
#pragma unroll
    for (int c = 0; c < W; ++c) {
      const int i = W * w.m + c;
      const bool in = i >= 1 && i <= N0;
      const float xn = (float)((double)xv[c] + alpha * (double)pv[c]);
      const float rn = (float)((double)rv[c] - alpha * (double)sv[c]);
      xo[c] = in ? xn : xv[c];
      ro[c] = in ? rn : rv[c];
      if (in) acc += (double)rn * (double)rn;
      const bool red = in && !(((i - 1) + w.j + w.k) & 1);
      sx[c] = red ? (dv[c] == 0.0f ? 0.0f : rn / dv[c]) : 0.0f;
      rv[c] = in ? rn : 0.0f;
    }
    stv<W>(V.x + q0, xo);
    stv<W>(V.r + q0, ro);
    if (pre) {
      stv<W>(L0.rhs + q0, rv);
      stv<W>(L0.x + q0, sx);
    }
  }
  return acc;
}

// PCG: r = b (assembled), x = 0; z = M r (V-cycle, or z = r when precond = 0);
// s = A p, alpha = <r,z>/<s,p>, x += alpha p, r -= alpha s, stop on ||r||/||b|| < tol.
// The update p = z + beta p is done inside the product A p (each thread
// forms the new p of its cell and of the six neighbours from z and the old
// p; p is double-buffered), and <r, z> inside the V-cycle's last pass.
template <class M>
__global__ void __launch_bounds__(PcgT<M>::v, 1) k_ch_pcg(CgVec<M> V, mg::Hier<M> G, int precond, double tol, int maxiter, double *partials,
                                               int *out_it, double *out_rel) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[40];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  const int N0 = V.N0, N1 = V.N1, PX = V.px, PY = N1 + 2, PXY = V.px * (N1 + 2);
  int buf = 0;
  const mg::Level<M> &L0 = G.lv[0];
  double acc = 0.0;
  if (precond) {
    mg_fine_and_rhs(V, L0, acc, tid, T);
  } else {
    for (mg::Walk w(N0, N1, V.N2, tid, T); w.ok(); w.next()) {
      const double rv = (double)V.r[(w.m + 1) + PX * ((w.j + 1) + PY * (w.k + 1))];
      acc += rv * rv;
    }
  }
  const double bb = grid_sum(acc, partials, buf, sh, grid);
  if (bb == 0.0) {
    if (tid == 0) { *out_it = 0; *out_rel = 0.0; }
    return;
  }
  if (precond) mg::build(G, false, grid, tid, T);
  const double eps = tol * tol;
  // gamma = <r, z>
  auto rz = [&]() {
    double a = 0.0;
    if (!precond) return bb;
    if (!mg::vcycle<M, M, true>(G, false, grid, tid, T, V.r, &a))
      for (mg::Walk w(N0, N1, V.N2, tid, T); w.ok(); w.next()) {
        const int q = (w.m + 1) + PX * ((w.j + 1) + PY * (w.k + 1));
        a += (double)V.r[q] * (double)__ldcg(L0.x + q);
      }
    return grid_sum(a, partials, buf, sh, grid);
  };
  double gamma = rz(), rr = bb, beta = 0.0;
  M *po = V.p, *pn = V.p2;
  int it = 0;
  while (it < maxiter && !(rr / bb < eps)) {
    const bool first = it == 0;
    it++;
    acc = 0.0;
    const M bm = (M)beta;
    auto pval = [&](int qq) -> M {
      const M z = precond ? __ldcg(L0.x + qq) : __ldcg(V.r + qq);
      return first ? z : z + bm * __ldcg(po + qq);
    };
    // p in storage precision; the product in FP64 (in FP32 its cancellation
    // error for smooth p would reach the near-null modes of the p' system)
    if constexpr (is_mixed(M())) acc = cg_ap_runs<kCgRun>(V, precond ? L0.x : V.r, po, pn, first, bm, tid, T);
    else for (mg::Walk w(N0, N1, V.N2, tid, T); w.ok(); w.next()) {
      const int q = (w.m + 1) + PX * ((w.j + 1) + PY * (w.k + 1));
      const M p0 = pval(q);
      const double cw = V.acx[q], ce = V.acx[q + 1], cs = V.acy[q], cn = V.acy[q + PX], cb = V.acz[q], cf = V.acz[q + PXY];
      const double d = cw + ce + cs + cn + cb + cf;
      const double sv = d * (double)p0 - (cw * (double)pval(q - 1) + ce * (double)pval(q + 1) + cs * (double)pval(q - PX) +
                                          cn * (double)pval(q + PX) + cb * (double)pval(q - PXY) + cf * (double)pval(q + PXY));
      pn[q] = p0;
      V.s[q] = (M)sv;
      acc += (double)(M)sv * (double)p0;
    }
    const double sp = grid_sum(acc, partials, buf, sh, grid);
    if (sp == 0.0) break;
    const double alpha = gamma / sp;
    acc = 0.0;
    if constexpr (is_mixed(M())) acc = cg_update_runs<kCgRun>(V, L0, precond != 0, pn, alpha, tid, T);
    else for (mg::Walk w(N0, N1, V.N2, tid, T); w.ok(); w.next()) {
      const int q = (w.m + 1) + PX * ((w.j + 1) + PY * (w.k + 1));
      const double xv = (double)V.x[q], pv = (double)pn[q], r0 = (double)V.r[q], sv = (double)V.s[q];
      const mg::Seed<M> sd = precond ? mg::seed_at(L0, w.m, w.j, w.k, q, false) : mg::Seed<M>{};
      V.x[q] = (M)(xv + alpha * pv);
      const M rv = (M)(r0 - alpha * sv);
      V.r[q] = rv;
      acc += (double)rv * (double)rv;
      if (precond) sd.store(L0, q, rv);
    }
    rr = grid_sum(acc, partials, buf, sh, grid);
    if (rr / bb < eps || it >= maxiter) break;  // no V-cycle for an iteration that will not run
    const double gnew = precond ? rz() : rr;
    beta = gnew / gamma;
    gamma = gnew;
    M *t = po; po = pn; pn = t;
  }
  if (tid == 0) { *out_it = it; *out_rel = sqrt(rr / bb); }
}

// ---------------------------------------------------------------- p' solve with z-marching level-0 passes
// The tensor maps of the arrays the z-marching passes stage (hs_zm.cuh):
// level 0's couplings, both residual buffers, both V-cycle buffers (level 0's
// x and rhs arrays, which this form uses as two x buffers: the residual is
// the V-cycle's right-hand side), both search-direction buffers, A p, and
// level 1's x for the prolongation.
struct PcgMaps {
  CUtensorMap acx, acy, acz, r[2], xm[2], p[2], s, x1;
};

// grid_sum with a per-block failure flag: every block reads the same flags
// after the barrier, so the decision to stop is the same in every block
__device__ double grid_sum_f(double v, int fail, double *partials, int &buf, double *sh, cg::grid_group &grid,
                             int &any_fail) {
  double *pf = partials + (size_t)(2 + buf) * gridDim.x;
  if (threadIdx.x == 0) pf[blockIdx.x] = fail ? 1.0 : 0.0;
  const double s = grid_sum(v, partials, buf, sh, grid);  // flips buf; its barrier orders the flags
  const double *pr = partials + (size_t)(2 + (buf ^ 1)) * gridDim.x;
  if (threadIdx.x < 32) {
    int f = 0;
    for (int q = threadIdx.x; q < (int)gridDim.x; q += 32) f |= __ldcg(pr + q) != 0.0;
    f = __any_sync(0xffffffffu, f);
    if (threadIdx.x == 0) sh[33] = f ? 1.0 : 0.0;
  }
  __syncthreads();
  any_fail = sh[33] != 0.0;
  __syncthreads();
  return s;
}

// The multigrid-preconditioned CG of k_ch_pcg with level 0 of the V-cycle,
// the product A p and the CG update as z-marching passes (hs_zm.cuh), each
// one pass over level 0 between two grid barriers:
//   setup:    the level-0 mask and <b, b>; the hierarchy; V0 = the seed and
//             first black half-sweep from r;
//   V-cycle:  nsw - 1 red-black sweeps, the restriction (grid-wide), the
//             levels below (vcycle from level 1), nsw black-red sweeps, the
//             first with the prolongation fused, the last with <r, z>;
//   per CG iteration: p = z + beta p and s = A p with <s, p>; x += alpha p,
//             r -= alpha s with <r, r> and the next V-cycle's seed and first
//             black half-sweep; the V-cycle.
// The residual and search direction are double-buffered (a pass reads one
// buffer, writes the other), z is level 0's second x buffer.  Needs G.ls >= 1
// (level 0 grid-wide) and precond; one block of zm::kThreads per SM.
template <class M>
__global__ void __launch_bounds__(zm::kThreads, 1)
    k_ch_pcg_zm(const __grid_constant__ CgVec<M> V, const __grid_constant__ mg::Hier<M> G,
                const __grid_constant__ PcgMaps TM, double tol, int maxiter, double *partials, int *out_it,
                double *out_rel) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[40];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  const int N0 = V.N0, N1 = V.N1, N2 = V.N2, PX = V.px;
  zm::Smem<M> S{reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(mg::stage_smem()) + 127) & ~uintptr_t(127))};
  if (threadIdx.x == 0) {
    for (int s = 0; s < zm::Box<M>::SLOTS; ++s) zm::mbar_init(S.bars() + s, 1);
    zm::fence_mbar_init();
  }
  __syncthreads();
  zm::Pipe P{0u, 0u, 0u, 0u, 0};
  const zm::Tiles Tl{N0, N1, N2, PX, (N0 + zm::kTX - 1) / zm::kTX, (N1 + zm::kTY - 1) / zm::kTY, V.nch};
  // the two buffers of each double-buffered vector
  auto xm = [&](int i) { return i ? G.lv[0].rhs : G.lv[0].x; };
  auto rb = [&](int i) { return i ? V.r2 : V.r; };
  auto pb = [&](int i) { return i ? V.p2 : V.p; };
  int buf = 0, fail = 0;
  // set-up: level 0's mask (read by the coarsening) and <b, b>
  double acc = 0.0;
  for (mg::Walk w(PX, N1 + 2, N2 + 2, tid, T); w.ok(); w.next()) {
    const int q = w.flat(), i = w.m - 1, j = w.j - 1, k = w.k - 1;
    const bool in = i >= 0 && j >= 0 && k >= 0 && i < N0 && j < N1 && k < N2;
    const bool solid = !in || V.solid[i + N0 * (j + N1 * k)] != 0;
    G.lv[0].m[q] = !solid;
    if (in) {
      const double rv = (double)V.r[q];
      acc += rv * rv;
    }
  }
  const double bb = grid_sum(acc, partials, buf, sh, grid);
  if (bb == 0.0) {
    if (tid == 0) { *out_it = 0; *out_rel = 0.0; }
    return;
  }
  mg::build(G, false, grid, tid, T);
  zm::fence_async_global();

  auto maps = [&](const CUtensorMap *b0, const CUtensorMap *b1, const CUtensorMap *coarse) {
    zm::PassMaps pm;
    pm.m[0] = b0; pm.m[1] = b1; pm.m[2] = &TM.acx; pm.m[3] = &TM.acy; pm.m[4] = &TM.acz;
    pm.coarse = coarse;
    return pm;
  };
  auto pass_end = [&]() {
    zm::fence_async_global();
    grid.sync();
    zm::fence_async_global();
  };
  int cur = 0;  // the current residual buffer
  // z = V(r[cur]) after the seed pass wrote xm(0); returns <r, z> (z in xm(1))
  auto vtail = [&]() -> double {
    int in = 0;
    for (int s = 1; s < G.nsw; ++s) {
      zm::PassArgs<M> a{};
      a.kind = zm::kSweep; a.c1 = 0; a.out = xm(in ^ 1);
      double dummy = 0.0;
      zm::run_pass(S, P, maps(&TM.xm[in], &TM.r[cur], nullptr), Tl, a, dummy);
      pass_end();
      in ^= 1;
    }
    mg::Level<M> F = G.lv[0];
    F.x = xm(in);
    F.rhs = rb(cur);
    mg::restrict_res(F, G.lv[1], false, tid, T);
    grid.sync();
    mg::vcycle<M, double>(G, false, grid, tid, T, nullptr, nullptr, 1);
    zm::fence_async_global();  // level 1's x, written before vcycle's last barrier, is read by the TMA unit next
    double d = 0.0;
    for (int s = 0; s < G.nsw; ++s) {
      zm::PassArgs<M> a{};
      a.kind = s == 0 ? zm::kProlong : zm::kSweep;
      a.c1 = 1;
      a.dot = s == G.nsw - 1;
      a.out = xm(in ^ 1);
      zm::run_pass(S, P, maps(&TM.xm[in], &TM.r[cur], s == 0 ? &TM.x1 : nullptr), Tl, a, d);
      in ^= 1;
      if (s < G.nsw - 1) pass_end();
    }
    zm::fence_async_global();
    const double g = grid_sum_f(d, P.fail, partials, buf, sh, grid, fail);
    zm::fence_async_global();
    return g;
  };
  {
    zm::PassArgs<M> a{};
    a.kind = zm::kSeed; a.c1 = 0; a.out = xm(0);
    double dummy = 0.0;
    zm::run_pass(S, P, maps(&TM.r[cur], &TM.r[cur], nullptr), Tl, a, dummy);
    pass_end();
  }
  const double eps = tol * tol;
  double gamma = vtail(), rr = bb, beta = 0.0;
  int po = 0, it = 0;
  while (!fail && it < maxiter && !(rr / bb < eps)) {
    const bool first = it == 0;
    it++;
    // p = z + beta p_old, s = A p, <s, p>
    double sp;
    {
      zm::PassArgs<M> a{};
      a.kind = zm::kAp; a.first = first; a.beta = (M)beta; a.out = pb(po ^ 1); a.out2 = V.s;
      acc = 0.0;
      zm::run_pass(S, P, maps(&TM.xm[1], &TM.p[po], nullptr), Tl, a, acc);
      zm::fence_async_global();
      sp = grid_sum_f(acc, P.fail, partials, buf, sh, grid, fail);
      zm::fence_async_global();
    }
    po ^= 1;
    if (fail || sp == 0.0) break;
    const double alpha = gamma / sp;
    // x += alpha p, r -= alpha s, <r, r>, the next V-cycle's seed and first black half-sweep
    {
      zm::PassArgs<M> a{};
      a.kind = zm::kSeed; a.c1 = 0; a.upd = 1; a.alpha = alpha; a.out = xm(0); a.out2 = rb(cur ^ 1);
      a.xcg = V.x; a.pcg = pb(po);
      acc = 0.0;
      zm::run_pass(S, P, maps(&TM.r[cur], &TM.s, nullptr), Tl, a, acc);
      zm::fence_async_global();
      rr = grid_sum_f(acc, P.fail, partials, buf, sh, grid, fail);
      zm::fence_async_global();
      cur ^= 1;
    }
    if (fail || rr / bb < eps || it >= maxiter) break;  // no V-cycle for an iteration that will not run
    const double gnew = vtail();
    beta = gnew / gamma;
    gamma = gnew;
  }
  if (tid == 0) {
    *out_it = fail ? -1 : it;
    *out_rel = sqrt(rr / bb);
  }
}

// residual sums of the momentum pass (3 x nbm partials) and continuity (nbc) -> res[0..3]
// (launched with 4 warps: warp a sums array a, each lane over four
// interleaved strides so that four loads are in flight)
__global__ void k_ch_finalize(const double *mom, int nbm, const double *cont, int nbc, double *res) {
  const int a = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (a >= 4) return;
  const double *src = a < 3 ? mom + a * nbm : cont;
  const int nb = a < 3 ? nbm : nbc;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int q = lane;
  for (; q + 96 < nb; q += 128) {
    s0 += src[q];
    s1 += src[q + 32];
    s2 += src[q + 64];
    s3 += src[q + 96];
  }
  for (; q < nb; q += 32) s0 += src[q];
  double s = (s0 + s1) + (s2 + s3);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) res[a] = sqrt(s);
}

// n rounded up to a multiple of 4: a row pitch of 16-byte rows in FP32 and FP64
int pitch4(int n) { return (n + 3) / 4 * 4; }

int blocks_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + kT - 1) / kT, 148LL * 8)); }

template <class K, class... A>
void launch_coop(K kernel, int blocks, int threads, size_t smem, cudaStream_t s, A... args) {
  void *argv[] = {(void *)&args...};
  CH_CUDA(cudaLaunchCooperativeKernel((void *)kernel, dim3(blocks), dim3(threads), argv, smem, s));
}

}  // namespace

// ---------------------------------------------------------------- host state
struct ChannelState {
  Case kase;
  ChParams prm;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool mixed = false;
  int N0 = 0, N1 = 0, N2 = 0, nreg = 0;
  int PX = 0;  // row pitch of the padded p' arrays and levels: N0 + 2 rounded up to 4 values (16-byte rows)
  double nu = 0, kf = 0;
  std::vector<int> region;
  std::vector<void *> allocs;
  long long bytes = 0;
  ChDev<double> Hd{};
  ChDev<float> Hf{};
  CgVec<double> Vd{};
  CgVec<float> Vf{};
  double *scratch = nullptr;  // FP64 staging of field copies (padded cells)
  mg::Hier<double> Gd{};
  mg::Hier<float> Gf{};
  int mom_blocks = 0, pcg_grid = 0;
  int asm_blocks = 0;             // k_ch_passemble: blocks per part
  int chunks = 0, chunk_per = 0;  // k_ch_correct: chunks per part, elements per thread
  // the z-marching form of the p' solve (k_ch_pcg_zm): its tensor maps, grid and shared memory
  PcgMaps TMd{}, TMf{};
  bool use_zm = false;
  int zm_grid = 0;
  size_t zm_smem = 0;
  double *mom_part = nullptr, *cont_part = nullptr, *pcg_part = nullptr, *res = nullptr, *pcg_rel = nullptr;
  int *pcg_it = nullptr;
  ChtState *cht = nullptr;
  std::vector<double> kratio, qcell;
  ChStats st{};
  int iter = 0;
  bool prof = false;
  // statistics of the steps of one ch_step call, copied without waiting
  // (pinned), applied in order after one stream synchronisation per kRing steps
  struct StepRec {
    double res[4], prel, trr[2];
    int pit, tit;
  };
  static constexpr int kRing = 64;
  StepRec *ring = nullptr;
  cudaEvent_t ev[6] = {};
  double prof_ms[5] = {0, 0, 0, 0, 0};
  int prof_steps = 0;

  template <class T_>
  T_ *alloc(size_t n) {
    void *p = nullptr;
    const size_t b = std::max<size_t>(n, 1) * sizeof(T_);
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA alloc: ") + cudaGetErrorString(e));
    allocs.push_back(p);
    bytes += (long long)b;
    CH_CUDA(cudaMemsetAsync(p, 0, b, stream));
    return (T_ *)p;
  }
  ~ChannelState() {
    if (ring) cudaFreeHost(ring);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    if (cht) cht_destroy(cht);
    for (void *p : allocs) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// QUICK weights along one axis (n cells, grid points pts[0..n]): for node kind
// 1 (faces of this axis: control-volume faces at the cell centres, e = 0 ..
// n - 1 between nodes e and e + 1) or 0 (cell centres: control-volume faces at
// the grid points, e = 0 .. n between cells e - 1 and e), per e six weights,
// (far upwind, upwind, downwind) for a flux in the + direction, then against
// it: the quadratic through the three nodes at their positions evaluated at
// the face (Leonard 1979), or (0, 1, 0) where a node is off the grid
std::vector<double> quick_weights(const std::vector<double> &pts, int n, int kind) {
  std::vector<double> W(6 * (size_t)(n + 1));
  const int nn = kind ? n + 1 : n;  // nodes 0 .. nn - 1
  auto xnode = [&](int m) { return kind ? pts[m] : 0.5 * (pts[m] + pts[m + 1]); };
  for (int e = 0; e <= n; ++e) {
    double *w = W.data() + 6 * (size_t)e;
    if (kind && e == n) {  // no control-volume face there
      w[0] = w[3] = 0.0; w[1] = w[4] = 1.0; w[2] = w[5] = 0.0;
      continue;
    }
    const double xf = kind ? 0.5 * (pts[e] + pts[e + 1]) : pts[e];
    const int lo = kind ? e : e - 1;
    for (int dir = 0; dir < 2; ++dir) {
      const int iuu = dir == 0 ? lo - 1 : lo + 2, iu = dir == 0 ? lo : lo + 1, id = dir == 0 ? lo + 1 : lo;
      double *o = w + 3 * dir;
      if (iuu < 0 || iuu >= nn || iu < 0 || iu >= nn || id < 0 || id >= nn) {
        o[0] = 0.0; o[1] = 1.0; o[2] = 0.0;
        continue;
      }
      const double xuu = xnode(iuu), xu = xnode(iu), xd = xnode(id);
      o[0] = ((xf - xu) * (xf - xd)) / ((xuu - xu) * (xuu - xd));
      o[1] = ((xf - xuu) * (xf - xd)) / ((xu - xuu) * (xu - xd));
      o[2] = ((xf - xuu) * (xf - xu)) / ((xd - xuu) * (xd - xu));
    }
  }
  return W;
}

template <class R>
void setup_fields(ChannelState &S, ChDev<R> &H, const std::vector<double> (&d)[3], const std::vector<double> (&h)[3],
                  const uint8_t *solid) {
  H.N0 = S.N0; H.N1 = S.N1; H.N2 = S.N2; H.PX = S.PX;
  const R **dd[3] = {&H.d0, &H.d1, &H.d2}, **hh[3] = {&H.h0, &H.h1, &H.h2};
  for (int a = 0; a < 3; ++a) {
    std::vector<R> dv(d[a].begin(), d[a].end()), hv(h[a].begin(), h[a].end());
    R *pd = S.alloc<R>(dv.size()), *ph = S.alloc<R>(hv.size());
    CH_CUDA(cudaMemcpyAsync(pd, dv.data(), dv.size() * sizeof(R), cudaMemcpyHostToDevice, S.stream));
    CH_CUDA(cudaMemcpyAsync(ph, hv.data(), hv.size() * sizeof(R), cudaMemcpyHostToDevice, S.stream));
    *dd[a] = pd; *hh[a] = ph;
  }
  H.solid = solid;
  const size_t nf[3] = {(size_t)(S.N0 + 1) * S.N1 * S.N2, (size_t)S.N0 * (S.N1 + 1) * S.N2, (size_t)S.N0 * S.N1 * (S.N2 + 1)};
  double **U[3] = {&H.U0, &H.U1, &H.U2};
  R **C[3] = {&H.C0, &H.C1, &H.C2}, **Sx[3] = {&H.S0, &H.S1, &H.S2}, **Q[3] = {&H.Q0, &H.Q1, &H.Q2};
  R **D[3] = {&H.D0, &H.D1, &H.D2};
  for (int a = 0; a < 3; ++a) {
    *U[a] = S.alloc<double>(nf[a]);
    *Sx[a] = S.alloc<R>(nf[a]);
    *D[a] = S.alloc<R>(nf[a]);
    if (is_mixed(R())) {
      *C[a] = S.alloc<R>(nf[a]);
      *Q[a] = S.alloc<R>(nf[a]);
    } else {
      *C[a] = (R *)*U[a];  // the FP64 form reads its coefficients from U itself
      *Q[a] = nullptr;
    }
  }
  H.p = S.alloc<double>((size_t)S.N0 * S.N1 * S.N2);
  H.nu = (R)S.nu; H.au = (R)S.prm.alpha_u; H.u_in = (R)S.prm.u_in; H.ap = S.prm.alpha_p;
  H.nu_d = S.nu; H.au_d = S.prm.alpha_u; H.u_in_d = S.prm.u_in;
  const double **xd[3] = {&H.xd0, &H.xd1, &H.xd2}, **xh[3] = {&H.xh0, &H.xh1, &H.xh2};
  for (int a = 0; a < 3; ++a) {
    if (!is_mixed(R())) { *xd[a] = (const double *)*dd[a]; *xh[a] = (const double *)*hh[a]; continue; }
    double *pd = S.alloc<double>(d[a].size()), *ph = S.alloc<double>(h[a].size());
    CH_CUDA(cudaMemcpyAsync(pd, d[a].data(), d[a].size() * sizeof(double), cudaMemcpyHostToDevice, S.stream));
    CH_CUDA(cudaMemcpyAsync(ph, h[a].data(), h[a].size() * sizeof(double), cudaMemcpyHostToDevice, S.stream));
    *xd[a] = pd; *xh[a] = ph;
  }
  // RN(1/x) of the FP64 widths and centre distances (IEEE division on the host)
  const double **rd[3] = {&H.rd0, &H.rd1, &H.rd2}, **rh[3] = {&H.rh0, &H.rh1, &H.rh2};
  for (int a = 0; a < 3; ++a) {
    std::vector<double> rdv(d[a].size()), rhv(h[a].size());
    for (size_t i = 0; i < rdv.size(); ++i) rdv[i] = 1.0 / d[a][i];
    for (size_t i = 0; i < rhv.size(); ++i) rhv[i] = 1.0 / h[a][i];
    double *pd = S.alloc<double>(rdv.size()), *ph = S.alloc<double>(rhv.size());
    CH_CUDA(cudaMemcpyAsync(pd, rdv.data(), rdv.size() * sizeof(double), cudaMemcpyHostToDevice, S.stream));
    CH_CUDA(cudaMemcpyAsync(ph, rhv.data(), rhv.size() * sizeof(double), cudaMemcpyHostToDevice, S.stream));
    *rd[a] = pd; *rh[a] = ph;
  }
  H.rau = 1.0 / S.prm.alpha_u;
  H.conv = S.prm.conv;
  H.g_axis = S.prm.g_axis;
  H.ri = S.prm.ri;
  H.t_in = S.prm.t_in;
  H.T = nullptr;  // the energy solver's T, bound once it exists
  const std::vector<double> *pts[3] = {&S.kase.deck.xs, &S.kase.deck.ys, &S.kase.deck.zs};
  const int N[3] = {S.N0, S.N1, S.N2};
  for (int a = 0; a < 3; ++a)
    for (int kind = 0; kind < 2; ++kind) {
      H.qw[a][kind] = nullptr;
      if (S.prm.conv != 2) continue;
      const std::vector<double> W = quick_weights(*pts[a], N[a], kind);
      double *pw = S.alloc<double>(W.size());
      CH_CUDA(cudaMemcpyAsync(pw, W.data(), W.size() * sizeof(double), cudaMemcpyHostToDevice, S.stream));
      H.qw[a][kind] = pw;
    }
}

template <class R> CgVec<R> &cg_vec(ChannelState &S);
template <> CgVec<double> &cg_vec<double>(ChannelState &S) { return S.Vd; }
template <> CgVec<float> &cg_vec<float>(ChannelState &S) { return S.Vf; }

template <class R>
void setup_cg(ChannelState &S, CgVec<R> &V, const uint8_t *solid, size_t np) {
  V.N0 = S.N0; V.N1 = S.N1; V.N2 = S.N2; V.px = S.PX; V.solid = solid;
  V.acx = S.alloc<R>(np); V.acy = S.alloc<R>(np); V.acz = S.alloc<R>(np);
  V.x = S.alloc<R>(np); V.r = S.alloc<R>(np); V.p = S.alloc<R>(np); V.s = S.alloc<R>(np);
  V.p2 = S.alloc<R>(np);
  V.r2 = S.alloc<R>(np);
}

template <class M>
void setup_mg(ChannelState &S, mg::Hier<M> &G, const CgVec<M> &V) {
  int nx = S.N0, ny = S.N1, nz = S.N2, L = 0;
  while (true) {
    if (L >= mg::kMgMaxLv) throw std::runtime_error("multigrid: too many levels");
    mg::Level<M> &l = G.lv[L];
    l.nx = nx; l.ny = ny; l.nz = nz; l.px = pitch4(nx + 2);
    const size_t np = (size_t)l.px * (ny + 2) * (nz + 2);
    l.x = S.alloc<M>(np); l.rhs = S.alloc<M>(np);
    if (L == 0) {  // the p' couplings themselves (written by the assembly, read-only in the solve)
      l.gx = const_cast<M *>(V.acx); l.gy = const_cast<M *>(V.acy); l.gz = const_cast<M *>(V.acz);
      l.d = S.alloc<M>(np);
    } else {
      l.gx = S.alloc<M>(np); l.gy = S.alloc<M>(np); l.gz = S.alloc<M>(np);
      l.d = nullptr;
    }
    l.fx = l.fy = l.fz = nullptr;
    l.m = S.alloc<uint8_t>(np);
    ++L;
    if ((long long)nx * ny * nz <= mg::kMgCoarse) break;
    nx = (nx + 1) / 2; ny = (ny + 1) / 2; nz = (nz + 1) / 2;
  }
  G.L = L;
  // two sweeps on level 0 halve the CG iterations (17 -> 8 on a 256x128x128
  // channel) for less than twice the cost of a cycle; one more on the
  // coarser levels, whose passes are short and barrier-bound, improves the
  // coarse correction (8 -> 7 iterations, 5% less time)
  G.nsw = S.prm.p_mg_sweeps > 0 ? S.prm.p_mg_sweeps : 2;
  G.nswc = G.nsw + 1;
  G.lu = S.alloc<double>((size_t)mg::kMgCoarse * mg::kMgCoarse);
  mg::plan_stage(G);
}

// ---- TMA tensor maps (the driver's encoder, reached through the runtime)
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled tensor_map_encoder() {
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q{};
  CH_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (q != cudaDriverEntryPointSuccess || !fn) throw std::runtime_error("CUDA: cuTensorMapEncodeTiled is not available");
  return reinterpret_cast<EncodeTiled>(fn);
}

// a 3-D tiled map over a padded array (px x py x pz values of M, x fastest)
// with a bx x by x 1 box; reads outside the array are zero-filled
template <class M>
CUtensorMap padded_map(EncodeTiled enc, const M *base, int px, int py, int pz, int bx, int by) {
  CUtensorMap m;
  const cuuint64_t dims[3] = {(cuuint64_t)px, (cuuint64_t)py, (cuuint64_t)pz};
  const cuuint64_t strides[2] = {(cuuint64_t)px * sizeof(M), (cuuint64_t)px * py * sizeof(M)};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1u};
  const cuuint32_t es[3] = {1u, 1u, 1u};
  const CUresult r = enc(&m, sizeof(M) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                         const_cast<M *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error("CUDA: tensor map encoding failed (" + std::to_string((int)r) + ")");
  return m;
}

// The z-marching form of the p' solve when the case allows it: the V-cycle
// preconditioner on, a coarser level below the finest and level 0 handled
// grid-wide (not by block 0 alone), p_level0 = 0, and one block of
// zm::kThreads resident per SM with the ring in shared memory.
template <class M>
void setup_zm(ChannelState &S, CgVec<M> &V, mg::Hier<M> &G, PcgMaps &TM, int nsm) {
  S.use_zm = false;
  // p_level0: 0 the faster form on this pool (the grid-wide passes until the
  // z-marching ones beat them), 1 grid-wide, 2 z-marching
  if (!S.prm.p_precond || S.prm.p_level0 != 2 || G.L < 2 || G.ls < 1) return;
  const EncodeTiled enc = tensor_map_encoder();
  const int py = S.N1 + 2, pz = S.N2 + 2;
  auto fine = [&](const M *a) { return padded_map<M>(enc, a, S.PX, py, pz, zm::Box<M>::BX, zm::Box<M>::BY); };
  TM.acx = fine(V.acx); TM.acy = fine(V.acy); TM.acz = fine(V.acz);
  TM.r[0] = fine(V.r); TM.r[1] = fine(V.r2);
  TM.xm[0] = fine(G.lv[0].x); TM.xm[1] = fine(G.lv[0].rhs);
  TM.p[0] = fine(V.p); TM.p[1] = fine(V.p2);
  TM.s = fine(V.s);
  const mg::Level<M> &L1 = G.lv[1];
  TM.x1 = padded_map<M>(enc, L1.x, L1.px, L1.ny + 2, L1.nz + 2, zm::Box<M>::CBX, zm::Box<M>::CBY);
  // the ring shares the launch's dynamic shared memory with block 0's staging
  // of the small levels, which therefore holds their x and rhs only (the
  // read-only arrays would not survive the ring between V-cycles)
  mg::plan_stage(G, false);
  const size_t smem = std::max<size_t>((size_t)zm::Box<M>::SMEM + 128, (size_t)G.stage);
  CH_CUDA(cudaFuncSetAttribute((const void *)k_ch_pcg_zm<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per = 0;
  CH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_ch_pcg_zm<M>, zm::kThreads, smem));
  if (per < 1) return;
  S.zm_grid = per * nsm;
  S.zm_smem = smem;
  V.nch = zm::pick_chunks(((S.N0 + zm::kTX - 1) / zm::kTX) * ((S.N1 + zm::kTY - 1) / zm::kTY), S.N2, S.zm_grid);
  S.use_zm = true;
}

template <class R>
void mom_solve(ChannelState &S, ChDev<R> &H) {
  const int sw = std::max(1, S.prm.mom_sweeps);
  for (int s = 0; s < sw; ++s)
    for (int color = 0; color < 2; ++color)
      if (H.conv == 2 || H.ri != 0.0)
        k_ch_mom<R, 2><<<dim3(3 * S.mom_blocks), kT, 0, S.stream>>>(H, color, s == 0 && color == 0, s == sw - 1,
                                                                  S.mom_part);
      else if (H.conv == 1)
        k_ch_mom<R, 1><<<dim3(3 * S.mom_blocks), kT, 0, S.stream>>>(H, color, s == 0 && color == 0, s == sw - 1,
                                                                  S.mom_part);
      else
        k_ch_mom<R, 0><<<dim3(3 * S.mom_blocks), kT, 0, S.stream>>>(H, color, s == 0 && color == 0, s == sw - 1,
                                                                  S.mom_part);
  CH_CUDA(cudaGetLastError());
}

template <class R>
void step_once(ChannelState &S, ChDev<R> &H, int flags) {
  if (S.prof) CH_CUDA(cudaEventRecord(S.ev[0], S.stream));
  mom_solve(S, H);
  if (S.prof) CH_CUDA(cudaEventRecord(S.ev[1], S.stream));
  CgVec<R> &V = cg_vec<R>(S);
  k_ch_passemble<R><<<dim3(S.asm_blocks, 4), kT, 0, S.stream>>>(H, (R *)V.acx, (R *)V.acy, (R *)V.acz, V.r, V.x,
                                                                S.cont_part);
  k_ch_finalize<<<1, 128, 0, S.stream>>>(S.mom_part, S.mom_blocks, S.cont_part, S.asm_blocks, S.res);
  CH_CUDA(cudaGetLastError());
  if (S.prof) CH_CUDA(cudaEventRecord(S.ev[2], S.stream));
  if (!(flags & 1)) {
    const int pre = S.prm.p_precond ? 1 : 0;
    if (S.use_zm && S.mixed)
      launch_coop(k_ch_pcg_zm<float>, S.zm_grid, zm::kThreads, S.zm_smem, S.stream, S.Vf, S.Gf, S.TMf, S.prm.p_tol,
                  S.prm.p_maxiter, S.pcg_part, S.pcg_it, S.pcg_rel);
    else if (S.use_zm)
      launch_coop(k_ch_pcg_zm<double>, S.zm_grid, zm::kThreads, S.zm_smem, S.stream, S.Vd, S.Gd, S.TMd, S.prm.p_tol,
                  S.prm.p_maxiter, S.pcg_part, S.pcg_it, S.pcg_rel);
    else if (S.mixed)
      launch_coop(k_ch_pcg<float>, S.pcg_grid, PcgT<float>::v, S.Gf.stage, S.stream, S.Vf, S.Gf, pre, S.prm.p_tol, S.prm.p_maxiter, S.pcg_part, S.pcg_it,
                  S.pcg_rel);
    else
      launch_coop(k_ch_pcg<double>, S.pcg_grid, PcgT<double>::v, S.Gd.stage, S.stream, S.Vd, S.Gd, pre, S.prm.p_tol, S.prm.p_maxiter, S.pcg_part, S.pcg_it,
                  S.pcg_rel);
  } else {
    const long long np = (long long)S.PX * (S.N1 + 2) * (S.N2 + 2);
    CH_CUDA(cudaMemsetAsync(V.x, 0, np * sizeof(R), S.stream));
    CH_CUDA(cudaMemsetAsync(S.pcg_it, 0, sizeof(int), S.stream));
  }
  if (S.prof) CH_CUDA(cudaEventRecord(S.ev[3], S.stream));
  k_ch_correct<R><<<dim3(4 * S.chunks), kT, 0, S.stream>>>(H, (const R *)V.x, S.chunk_per);
  CH_CUDA(cudaGetLastError());
  if (S.prof) CH_CUDA(cudaEventRecord(S.ev[4], S.stream));
  if (!(flags & 2)) cht_energy_step(S.cht, S.prm.alpha_t, S.prm.t_tol, S.prm.t_maxiter);
  if (S.prof) CH_CUDA(cudaEventRecord(S.ev[5], S.stream));
}

// the step's statistics into rec, on the stream (rec in pinned memory: the
// copies do not wait; read rec after the stream has passed them)
void enqueue_stats(ChannelState &S, ChannelState::StepRec &rec, int flags) {
  CH_CUDA(cudaMemcpyAsync(rec.res, S.res, 32, cudaMemcpyDeviceToHost, S.stream));
  CH_CUDA(cudaMemcpyAsync(&rec.pit, S.pcg_it, 4, cudaMemcpyDeviceToHost, S.stream));
  CH_CUDA(cudaMemcpyAsync(&rec.prel, S.pcg_rel, 8, cudaMemcpyDeviceToHost, S.stream));
  if (!(flags & 2)) cht_step_results_async(S.cht, &rec.tit, rec.trr);
}

// the step's bookkeeping from its statistics: residuals, the normalisers
// (maxima over the first five steps) and the global residual
void apply_stats(ChannelState &S, const ChannelState::StepRec &rec, int flags) {
  if (!(flags & 1) && rec.pit < 0)
    throw std::runtime_error("pressure-correction solve: a wait for staged planes ran out (the solve was abandoned)");
  for (int a = 0; a < 4; ++a) S.st.res[a] = rec.res[a];
  S.st.pcg_iters = (flags & 1) ? 0 : rec.pit;
  S.st.pcg_relres = (flags & 1) ? 0.0 : rec.prel;
  if (!(flags & 2)) {
    S.st.res[4] = rec.trr[1]; S.st.t_iters = rec.tit; S.st.t_relres = rec.trr[0];
  } else {
    S.st.res[4] = 0.0; S.st.t_iters = 0; S.st.t_relres = 0.0;
  }
  S.iter++;
  S.st.iter = S.iter;
  double g = 0.0;
  for (int x = 0; x < 5; ++x) {
    if (S.iter <= 5 && S.st.res[x] > S.st.norm[x]) S.st.norm[x] = S.st.res[x];
    const double q = S.st.res[x] / (S.st.norm[x] > 1e-300 ? S.st.norm[x] : 1e-300);
    if (q > g) g = q;
  }
  S.st.global = g;
}

void read_stats(ChannelState &S, int flags) {
  ChannelState::StepRec &rec = S.ring[0];
  enqueue_stats(S, rec, flags);
  CH_CUDA(cudaStreamSynchronize(S.stream));
  if (S.prof) {
    for (int ph = 0; ph < 5; ++ph) {
      float ms = 0;
      CH_CUDA(cudaEventElapsedTime(&ms, S.ev[ph], S.ev[ph + 1]));
      S.prof_ms[ph] += ms;
    }
    S.prof_steps++;
  }
  apply_stats(S, rec, flags);
}

}  // namespace

namespace {
double *uarr(ChannelState *S, int a) {
  double *u[3] = {S->Hd.U0, S->Hd.U1, S->Hd.U2}, *m[3] = {S->Hf.U0, S->Hf.U1, S->Hf.U2};
  return S->mixed ? m[a] : u[a];
}
}  // namespace

ChannelState *ch_create(const Case &c, const ChParams &p, int device) {
  if (!(p.re > 0) || !(p.pr > 0) || !(p.alpha_u > 0 && p.alpha_u <= 1) || !(p.alpha_p > 0 && p.alpha_p <= 1) ||
      !(p.alpha_t > 0 && p.alpha_t <= 1) || p.mom_sweeps < 1 || !(p.p_tol > 0) || p.p_maxiter < 0 || !(p.t_tol > 0) ||
      p.t_maxiter < 0 || (p.precision != 0 && p.precision != 1) || p.p_mg_sweeps < 0 || p.p_mg_sweeps > 8 ||
      p.p_level0 < 0 || p.p_level0 > 2 || p.conv < 0 || p.conv > 2 || p.g_axis < 0 || p.g_axis > 2 ||
      !std::isfinite(p.ri))
    throw std::invalid_argument("invalid channel parameters");
  if ((long long)pitch4((int)c.Nx + 2) * (c.Ny + 2) * (c.Nz + 2) >= (1LL << 31))
    throw std::invalid_argument("grid too large for 32-bit indices");
  CH_CUDA(cudaSetDevice(device));
  std::unique_ptr<ChannelState> S(new ChannelState());
  S->kase = c;
  S->prm = p;
  S->device = device;
  S->mixed = p.precision == 1;
  CH_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
  S->N0 = (int)c.Nx; S->N1 = (int)c.Ny; S->N2 = (int)c.Nz;
  S->PX = pitch4(S->N0 + 2);
  S->nreg = c.nsolid_regions;
  const std::vector<double> *pts[3] = {&c.deck.xs, &c.deck.ys, &c.deck.zs};
  std::vector<double> d[3], h[3];
  const int N[3] = {S->N0, S->N1, S->N2};
  for (int a = 0; a < 3; ++a) {
    const std::vector<double> &x = *pts[a];
    d[a].resize(N[a]); h[a].resize(N[a] + 1);
    for (int i = 0; i < N[a]; ++i) d[a][i] = x[i + 1] - x[i];
    h[a][0] = 0.5 * d[a][0];
    h[a][N[a]] = 0.5 * d[a][N[a] - 1];
    for (int i = 1; i < N[a]; ++i) h[a][i] = 0.5 * (x[i] + x[i + 1]) - 0.5 * (x[i - 1] + x[i]);
  }
  const double ly = c.deck.ys[S->N1] - c.deck.ys[0];
  S->nu = p.u_in * ly / p.re;
  S->kf = S->nu / p.pr;
  const size_t n = (size_t)S->N0 * S->N1 * S->N2;
  uint8_t *solid = S->alloc<uint8_t>(n);
  CH_CUDA(cudaMemcpyAsync(solid, c.ctype.data(), n, cudaMemcpyHostToDevice, S->stream));
  if (S->mixed) setup_fields(*S, S->Hf, d, h, solid);
  else setup_fields(*S, S->Hd, d, h, solid);
  // CG vectors and couplings (padded, row pitch PX)
  const size_t np = (size_t)S->PX * (S->N1 + 2) * (S->N2 + 2);
  if (S->mixed) setup_cg(*S, S->Vf, solid, np);
  else setup_cg(*S, S->Vd, solid, np);
  S->scratch = S->alloc<double>(np);
  if (S->mixed) setup_mg(*S, S->Gf, S->Vf);
  else setup_mg(*S, S->Gd, S->Vd);
  int per = 0, nsm = 0;
  CH_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  // momentum: a grid resident at once (its three components of a chunk of
  // faces in consecutive blocks then march through the z-planes together:
  // 0.71 -> 0.66 ms per FP64 momentum solve at 256x128x128 against 3 x 1184
  // blocks); every instantiation holds four blocks per SM (launch bounds)
  const long long nmax = (long long)(S->N0 + 1) * (S->N1 + 1) * (S->N2 + 1);  // >= any part's element count
  CH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per, S->mixed ? (const void *)k_ch_mom<float, 0> : (const void *)k_ch_mom<double, 0>, kT, 0));
  S->mom_blocks = std::min(blocks_for(nmax), std::max(1, per * nsm / 3));
  S->mom_part = S->alloc<double>((size_t)3 * S->mom_blocks);
  S->res = S->alloc<double>(4);
  S->asm_blocks = blocks_for(nmax);
  S->cont_part = S->alloc<double>((size_t)S->asm_blocks);
  // the four-part correction: at least 148 x 8 chunks per part (fewer on a
  // small grid), each thread taking at most 32 elements, so that the last
  // wave of blocks is short on large grids too
  const long long span = (long long)kT * blocks_for(nmax);
  S->chunk_per = (int)std::min<long long>(32, (nmax + span - 1) / span);
  S->chunks = (int)((nmax + (long long)kT * S->chunk_per - 1) / ((long long)kT * S->chunk_per));
  // the V-cycle's staging of block 0's levels: up to kMgStageTotal bytes per launch
  const void *pk = S->mixed ? (const void *)k_ch_pcg<float> : (const void *)k_ch_pcg<double>;
  CH_CUDA(cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, mg::kMgStageTotal));
  CH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, pk, S->mixed ? PcgT<float>::v : PcgT<double>::v,
                                                        S->mixed ? S->Gf.stage : S->Gd.stage));
  if (per < 1) throw std::runtime_error("pressure-correction kernel cannot be resident");
  S->pcg_grid = per * nsm;
  if (S->mixed) setup_zm(*S, S->Vf, S->Gf, S->TMf, nsm);
  else setup_zm(*S, S->Vd, S->Gd, S->TMd, nsm);
  S->pcg_part = S->alloc<double>((size_t)4 * std::max(S->pcg_grid, S->zm_grid) + 64);
  S->pcg_it = S->alloc<int>(1);
  S->pcg_rel = S->alloc<double>(1);
  // energy: the conjugate-heat-transfer operator in channel mode, on this stream
  S->region.resize(n);
  for (size_t i = 0; i < n; ++i) S->region[i] = c.ctype[i] ? c.region[i] : -1;
  ChtSetup cs;
  cs.device = device; cs.stream = S->stream;
  cs.Nx = S->N0; cs.Ny = S->N1; cs.Nz = S->N2; cs.nreg = S->nreg;
  cs.xs = c.deck.xs.data(); cs.ys = c.deck.ys.data(); cs.zs = c.deck.zs.data();
  cs.ctype = c.ctype.data(); cs.region = S->region.data();
  cs.t_boundary = p.t_in; cs.tol = 1e-10; cs.maxiter = 5000; cs.bc = 1;
  cs.precond = p.precision == 1 ? 1 : 2;
  cs.step_fp32 = p.precision == 1;
  S->cht = cht_create(cs);
  CH_CUDA(cudaHostAlloc((void **)&S->ring, ChannelState::kRing * sizeof(ChannelState::StepRec), cudaHostAllocDefault));
  cht_bind_velocities(S->cht, uarr(S.get(), 0), uarr(S.get(), 1), uarr(S.get(), 2));
  if (S->mixed) S->Hf.T = cht_T_device(S->cht);
  else S->Hd.T = cht_T_device(S->cht);
  S->kratio.assign(S->nreg, 100.0);
  S->qcell.assign(n, 0.0);
  std::vector<double> kabs(S->nreg);
  for (int r = 0; r < S->nreg; ++r) kabs[r] = S->kratio[r] * S->kf;
  cht_set_solid(S->cht, S->kf, kabs.data(), S->qcell.data());
  CH_CUDA(cudaStreamSynchronize(S->stream));
  return S.release();
}

void ch_destroy(ChannelState *S) {
  if (!S) return;
  cudaSetDevice(S->device);
  if (S->stream) cudaStreamSynchronize(S->stream);
  delete S;
}

int ch_nreg(const ChannelState *S) { return S->nreg; }

void ch_set_solid(ChannelState *S, const double *k_ratio, const double *q_cell) {
  CH_CUDA(cudaSetDevice(S->device));
  const size_t n = (size_t)S->N0 * S->N1 * S->N2;
  for (int r = 0; r < S->nreg; ++r)
    if (!(k_ratio[r] > 0)) throw std::invalid_argument("conductivity ratio must be positive");
  S->kratio.assign(k_ratio, k_ratio + S->nreg);
  for (size_t c = 0; c < n; ++c) S->qcell[c] = S->kase.ctype[c] ? q_cell[c] : 0.0;
  std::vector<double> kabs(S->nreg);
  for (int r = 0; r < S->nreg; ++r) kabs[r] = S->kratio[r] * S->kf;
  cht_set_solid(S->cht, S->kf, kabs.data(), S->qcell.data());
}

void ch_init(ChannelState *S) {
  CH_CUDA(cudaSetDevice(S->device));
  const long long tot = (long long)(S->N0 + 1) * (S->N1 + 1) * (S->N2 + 1) * 4;
  if (S->mixed) k_ch_init<float><<<blocks_for(tot), kT, 0, S->stream>>>(S->Hf);
  else k_ch_init<double><<<blocks_for(tot), kT, 0, S->stream>>>(S->Hd);
  CH_CUDA(cudaGetLastError());
  cht_fill_T(S->cht, S->prm.t_in);
  S->iter = 0;
  S->st = ChStats{};
  S->st.global = 1.0;
  CH_CUDA(cudaStreamSynchronize(S->stream));
}

void ch_step(ChannelState *S, int n, int flags, ChStats *out) {
  CH_CUDA(cudaSetDevice(S->device));
  if (S->prof) {  // per-phase events of every step: one step at a time
    for (int s = 0; s < n; ++s) {
      if (S->mixed) step_once(*S, S->Hf, flags);
      else step_once(*S, S->Hd, flags);
      read_stats(*S, flags);
    }
  } else {
    // steps queued back to back, their statistics applied afterwards in order
    for (int done = 0; done < n;) {
      const int b = std::min(n - done, ChannelState::kRing);
      for (int s = 0; s < b; ++s) {
        if (S->mixed) step_once(*S, S->Hf, flags);
        else step_once(*S, S->Hd, flags);
        enqueue_stats(*S, S->ring[s], flags);
      }
      CH_CUDA(cudaStreamSynchronize(S->stream));
      for (int s = 0; s < b; ++s) apply_stats(*S, S->ring[s], flags);
      done += b;
    }
  }
  if (out) *out = S->st;
}

int ch_solve_to(ChannelState *S, double tol, int max_outer, ChStats *out) {
  CH_CUDA(cudaSetDevice(S->device));
  int s = 0;
  while (s < max_outer) {
    if (S->mixed) step_once(*S, S->Hf, 0);
    else step_once(*S, S->Hd, 0);
    read_stats(*S, 0);
    ++s;
    if (S->iter > 5 && S->st.global <= tol) break;
  }
  if (out) *out = S->st;
  return s;
}

// fields: 0..2 u v w, 3 p, 4 T, 5..7 u* v* w*, 8..10 d, 11 p'
long ch_field_size(const ChannelState *S, int f) {
  const long n = (long)S->N0 * S->N1 * S->N2;
  if (f == 3 || f == 4 || f == 11) return n;
  if (f < 0 || f > 11) return -1;
  const int a = f < 3 ? f : (f - 5) % 3;
  return (long)(S->N0 + (a == 0)) * (S->N1 + (a == 1)) * (S->N2 + (a == 2));
}

namespace {
// device-side conversions for the field copies (the caller's host buffer is
// copied to or from directly; pinned buffers go by DMA)
template <class T>
__global__ void k_unpad(const T *src, double *dst, int N0, int N1, int N2, int PX) {
  const int n = N0 * N1 * N2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    dst[e] = src[cell_q(e, N0, N1, PX)];
}
__global__ void k_pad(const double *src, double *dst, int N0, int N1, int N2, int PX) {
  const int n = N0 * N1 * N2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    dst[cell_q(e, N0, N1, PX)] = src[e];
}
template <class R>
__global__ void k_widen(const R *src, const double *add, double *dst, long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    dst[e] = (double)src[e] + (add ? add[e] : 0.0);
}
__global__ void k_narrow(const double *src, float *dst, long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    dst[e] = (float)src[e];
}

void d2h(ChannelState *S, const double *dev, double *host, long n) {
  CH_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, S->stream));
  CH_CUDA(cudaStreamSynchronize(S->stream));
}
void h2d(ChannelState *S, double *dev, const double *host, long n) {
  CH_CUDA(cudaMemcpyAsync(dev, host, n * sizeof(double), cudaMemcpyHostToDevice, S->stream));
  CH_CUDA(cudaStreamSynchronize(S->stream));
}
}  // namespace

// Field copies between steps stage through `scratch` (padded FP64).
void ch_get_field(ChannelState *S, int f, double *host, long n) {
  CH_CUDA(cudaSetDevice(S->device));
  if (ch_field_size(S, f) != n) throw std::invalid_argument("field size mismatch");
  double *scr = S->scratch;
  const int g = blocks_for(n);
  if (f == 4 || f == 11) {
    if (f == 4) k_unpad<double><<<g, kT, 0, S->stream>>>(cht_T_device(S->cht), scr, S->N0, S->N1, S->N2, S->N0 + 2);
    else if (S->mixed) k_unpad<float><<<g, kT, 0, S->stream>>>(S->Vf.x, scr, S->N0, S->N1, S->N2, S->PX);
    else k_unpad<double><<<g, kT, 0, S->stream>>>(S->Vd.x, scr, S->N0, S->N1, S->N2, S->PX);
    CH_CUDA(cudaGetLastError());
    d2h(S, scr, host, n);
    return;
  }
  if (f < 3) { d2h(S, uarr(S, f), host, n); return; }
  if (f == 3) { d2h(S, S->mixed ? S->Hf.p : S->Hd.p, host, n); return; }
  const int a = (f - 5) % 3;
  if (!S->mixed) {
    const double *src = f >= 8 ? (a == 0 ? S->Hd.D0 : a == 1 ? S->Hd.D1 : S->Hd.D2)
                               : (a == 0 ? S->Hd.S0 : a == 1 ? S->Hd.S1 : S->Hd.S2);
    d2h(S, src, host, n);
    return;
  }
  const float *src = f >= 8 ? (a == 0 ? S->Hf.D0 : a == 1 ? S->Hf.D1 : S->Hf.D2)
                            : (a == 0 ? S->Hf.S0 : a == 1 ? S->Hf.S1 : S->Hf.S2);
  k_widen<float><<<g, kT, 0, S->stream>>>(src, f >= 8 ? nullptr : uarr(S, a), scr, n);  // u* = u^n + delta
  CH_CUDA(cudaGetLastError());
  d2h(S, scr, host, n);
}

void ch_set_field(ChannelState *S, int f, const double *host, long n) {
  CH_CUDA(cudaSetDevice(S->device));
  if (ch_field_size(S, f) != n || f > 4) throw std::invalid_argument("field size mismatch or read-only field");
  const int g = blocks_for(n);
  if (f == 4) {
    h2d(S, S->scratch, host, n);
    k_pad<<<g, kT, 0, S->stream>>>(S->scratch, cht_T_device(S->cht), S->N0, S->N1, S->N2, S->N0 + 2);
    CH_CUDA(cudaGetLastError());
    return;
  }
  if (f == 3) { h2d(S, S->mixed ? S->Hf.p : S->Hd.p, host, n); return; }
  h2d(S, uarr(S, f), host, n);
  if (S->mixed) {
    k_narrow<<<g, kT, 0, S->stream>>>(uarr(S, f), f == 0 ? S->Hf.C0 : f == 1 ? S->Hf.C1 : S->Hf.C2, n);
    CH_CUDA(cudaGetLastError());
  }
}

void ch_profile(ChannelState *S, bool on) {
  CH_CUDA(cudaSetDevice(S->device));
  if (on && !S->ev[0])
    for (cudaEvent_t &e : S->ev) CH_CUDA(cudaEventCreate(&e));
  S->prof = on;
  for (double &m : S->prof_ms) m = 0.0;
  S->prof_steps = 0;
}

int ch_profile_read(const ChannelState *S, double *ms5) {
  for (int ph = 0; ph < 5; ++ph) ms5[ph] = S->prof_ms[ph];
  return S->prof_steps;
}

void *ch_stream(ChannelState *S) { return S->stream; }
void ch_balance(ChannelState *S, double out4[4]) {
  CH_CUDA(cudaSetDevice(S->device));
  cht_balance(S->cht, out4);
}
void ch_sync(ChannelState *S) { CH_CUDA(cudaSetDevice(S->device)); CH_CUDA(cudaStreamSynchronize(S->stream)); }
long long ch_device_bytes(const ChannelState *S) { return S->bytes; }

void ch_adjoint(ChannelState *S, double tol, int maxiter, double *J, double *dJdq, double *dJdk, int *fwd_iters,
                int *adj_iters, double *fwd_ms, double *adj_ms) {
  CH_CUDA(cudaSetDevice(S->device));
  // the relaxed outer-loop temperature is kept; the adjoint works on a full solve
  const size_t np = (size_t)(S->N0 + 2) * (S->N1 + 2) * (S->N2 + 2);
  double *keep = nullptr;
  CH_CUDA(cudaMalloc(&keep, np * 8));
  CH_CUDA(cudaMemcpyAsync(keep, cht_T_device(S->cht), np * 8, cudaMemcpyDeviceToDevice, S->stream));
  cudaEvent_t e0, e1, e2;
  CH_CUDA(cudaEventCreate(&e0)); CH_CUDA(cudaEventCreate(&e1)); CH_CUDA(cudaEventCreate(&e2));
  cht_set_tolerance(S->cht, tol, maxiter);
  double rel = 0;
  CH_CUDA(cudaEventRecord(e0, S->stream));
  cht_forward(S->cht, nullptr, J, fwd_iters, &rel);
  CH_CUDA(cudaEventRecord(e1, S->stream));
  // the adjoint's time ends with the gradients on the device: their copies
  // to the host are left out, as the forward's T stays on the device
  cht_adjoint(S->cht, dJdq, dJdk, adj_iters, &rel, e2);
  CH_CUDA(cudaEventSynchronize(e2));
  float a = 0, b = 0;
  CH_CUDA(cudaEventElapsedTime(&a, e0, e1));
  CH_CUDA(cudaEventElapsedTime(&b, e1, e2));
  if (fwd_ms) *fwd_ms = a;
  if (adj_ms) *adj_ms = b;
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
  CH_CUDA(cudaMemcpyAsync(cht_T_device(S->cht), keep, np * 8, cudaMemcpyDeviceToDevice, S->stream));
  CH_CUDA(cudaStreamSynchronize(S->stream));
  cudaFree(keep);
}

}  // namespace hs
