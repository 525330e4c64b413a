// Implementations behind the single-rank MPI / HYPRE / Scotch shim headers.
// Test infrastructure: only oracle/ref/ref_driver links this.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>
#include "HYPRE.h"
#include "mpi.h"
#include "scotch.h"

// ---------------------------------------------------------------- MPI
static size_t type_size(MPI_Datatype t) {
  switch (t) { case MPI_DOUBLE: return 8; case MPI_INT: return 4; case MPI_LONG: return 8; }
  return 72;  // derived struct type (OutputData in main.cpp:72-90)
}
struct PendingMsg { const void *buf; size_t bytes; int tag; bool send; void *rbuf; };
static std::vector<PendingMsg> g_pending;

int MPI_Init(int *, char ***) { return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
int MPI_Sendrecv(const void *sb, int sc, MPI_Datatype st, int, int, void *rb, int rc, MPI_Datatype rt, int, int, MPI_Comm,
                 MPI_Status *) {
  size_t n = std::min((size_t)sc * type_size(st), (size_t)rc * type_size(rt));
  if (n) std::memmove(rb, sb, n);
  return 0;
}
int MPI_Isend(const void *b, int c, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request *r) {
  *r = (int)g_pending.size(); g_pending.push_back({b, (size_t)c * type_size(t), tag, true, nullptr}); return 0;
}
int MPI_Irecv(void *b, int c, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request *r) {
  *r = (int)g_pending.size(); g_pending.push_back({nullptr, (size_t)c * type_size(t), tag, false, b}); return 0;
}
int MPI_Waitall(int, MPI_Request *, MPI_Status *) {
  // match every receive with the earliest unmatched send of the same tag
  std::vector<bool> used(g_pending.size(), false);
  for (size_t i = 0; i < g_pending.size(); ++i) {
    if (g_pending[i].send) continue;
    for (size_t j = 0; j < g_pending.size(); ++j) {
      if (!g_pending[j].send || used[j] || g_pending[j].tag != g_pending[i].tag) continue;
      used[j] = true;
      size_t n = std::min(g_pending[i].bytes, g_pending[j].bytes);
      if (n != g_pending[i].bytes || n != g_pending[j].bytes) { std::fprintf(stderr, "shim MPI: message size mismatch\n"); std::abort(); }
      if (n) std::memcpy(g_pending[i].rbuf, g_pending[j].buf, n);
      break;
    }
  }
  g_pending.clear();
  return 0;
}
int MPI_Allreduce(const void *s, void *r, int c, MPI_Datatype t, MPI_Op, MPI_Comm) { std::memmove(r, s, (size_t)c * type_size(t)); return 0; }
int MPI_Exscan(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }  // undefined on rank 0
int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) { std::memmove(r, s, (size_t)sc * type_size(st)); return 0; }
int MPI_Allgatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *, const int *d, MPI_Datatype, MPI_Comm) {
  std::memmove((char *)r + (size_t)d[0] * type_size(st), s, (size_t)sc * type_size(st)); return 0;
}
int MPI_Gather(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, int, MPI_Comm) { std::memmove(r, s, (size_t)sc * type_size(st)); return 0; }
int MPI_Gatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *, const int *d, MPI_Datatype, int, MPI_Comm) {
  if (sc) std::memmove((char *)r + (size_t)d[0] * type_size(st), s, (size_t)sc * type_size(st)); return 0;
}
int MPI_Get_address(const void *p, MPI_Aint *a) { *a = (MPI_Aint)p; return 0; }
int MPI_Type_create_struct(int, const int *, const MPI_Aint *, const MPI_Datatype *, MPI_Datatype *t) { *t = 100; return 0; }
int MPI_Type_commit(MPI_Datatype *) { return 0; }
int MPI_Type_free(MPI_Datatype *) { return 0; }

// ---------------------------------------------------------------- HYPRE
struct hs_ij_matrix { int ilower, iupper; std::vector<std::vector<std::pair<int, double>>> rows; };
struct hs_ij_vector { int ilower, iupper; std::vector<double> v; };
struct hs_pcg { int maxiter = 1000; double tol = 1e-6; int two_norm = 0; int iters = 0; double relres = 0; };
static int g_last_pcg_iters = 0;
static double g_last_pcg_relres = 0;
extern "C" int hs_shim_last_pcg_iters(void) { return g_last_pcg_iters; }
extern "C" double hs_shim_last_pcg_relres(void) { return g_last_pcg_relres; }

HYPRE_Int HYPRE_Initialize(void) { return 0; }
HYPRE_Int HYPRE_Finalize(void) { return 0; }
HYPRE_Int HYPRE_IJMatrixCreate(MPI_Comm, HYPRE_Int il, HYPRE_Int iu, HYPRE_Int, HYPRE_Int, HYPRE_IJMatrix *A) {
  *A = new hs_ij_matrix{il, iu, {}}; (*A)->rows.resize((size_t)(iu - il + 1)); return 0;
}
HYPRE_Int HYPRE_IJMatrixSetObjectType(HYPRE_IJMatrix, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_IJMatrixInitialize(HYPRE_IJMatrix) { return 0; }
HYPRE_Int HYPRE_IJMatrixSetValues(HYPRE_IJMatrix A, HYPRE_Int nrows, HYPRE_Int *ncols, const HYPRE_Int *rows,
                                  const HYPRE_Int *cols, const HYPRE_Complex *vals) {
  size_t k = 0;
  for (int r = 0; r < nrows; ++r) {
    auto &row = A->rows[(size_t)(rows[r] - A->ilower)];
    for (int e = 0; e < ncols[r]; ++e, ++k) {
      bool found = false;
      for (auto &pr : row) if (pr.first == cols[k]) { pr.second = vals[k]; found = true; break; }
      if (!found) row.push_back({cols[k], vals[k]});
    }
  }
  return 0;
}
HYPRE_Int HYPRE_IJMatrixAssemble(HYPRE_IJMatrix) { return 0; }
HYPRE_Int HYPRE_IJMatrixGetObject(HYPRE_IJMatrix A, void **o) { *o = A; return 0; }
HYPRE_Int HYPRE_IJMatrixDestroy(HYPRE_IJMatrix A) { delete A; return 0; }
HYPRE_Int HYPRE_IJVectorCreate(MPI_Comm, HYPRE_Int il, HYPRE_Int iu, HYPRE_IJVector *v) {
  *v = new hs_ij_vector{il, iu, std::vector<double>((size_t)(iu - il + 1), 0.0)}; return 0;
}
HYPRE_Int HYPRE_IJVectorSetObjectType(HYPRE_IJVector, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_IJVectorInitialize(HYPRE_IJVector) { return 0; }
HYPRE_Int HYPRE_IJVectorSetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_Int *idx, const HYPRE_Complex *val) {
  for (int i = 0; i < n; ++i) v->v[(size_t)(idx[i] - v->ilower)] = val[i]; return 0;
}
HYPRE_Int HYPRE_IJVectorAssemble(HYPRE_IJVector) { return 0; }
HYPRE_Int HYPRE_IJVectorGetObject(HYPRE_IJVector v, void **o) { *o = v; return 0; }
HYPRE_Int HYPRE_IJVectorGetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_Int *idx, HYPRE_Complex *out) {
  for (int i = 0; i < n; ++i) out[i] = v->v[(size_t)(idx[i] - v->ilower)]; return 0;
}
HYPRE_Int HYPRE_IJVectorDestroy(HYPRE_IJVector v) { delete v; return 0; }
HYPRE_Int HYPRE_ParCSRPCGCreate(MPI_Comm, HYPRE_Solver *s) { *s = new hs_pcg(); return 0; }
HYPRE_Int HYPRE_ParCSRPCGDestroy(HYPRE_Solver s) { delete s; return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { return 0; }
HYPRE_Int HYPRE_PCGSetMaxIter(HYPRE_Solver s, HYPRE_Int m) { s->maxiter = m; return 0; }
HYPRE_Int HYPRE_PCGSetTol(HYPRE_Solver s, HYPRE_Real t) { s->tol = t; return 0; }
HYPRE_Int HYPRE_PCGSetTwoNorm(HYPRE_Solver s, HYPRE_Int t) { s->two_norm = t; return 0; }
HYPRE_Int HYPRE_PCGGetNumIterations(HYPRE_Solver s, HYPRE_Int *n) { *n = s->iters; return 0; }
HYPRE_Int HYPRE_PCGGetFinalRelativeResidualNorm(HYPRE_Solver s, HYPRE_Real *r) { *r = s->relres; return 0; }

// y = A x with the diagonal first, then the row's other entries in the
// order they were first set.
static void csr_matvec(const hs_ij_matrix *A, const std::vector<double> &x, std::vector<double> &y) {
  for (size_t r = 0; r < A->rows.size(); ++r) {
    int grow = (int)r + A->ilower; double acc = 0; bool first = true;
    for (auto &pr : A->rows[r]) if (pr.first == grow) { acc = pr.second * x[r]; first = false; break; }
    for (auto &pr : A->rows[r]) {
      if (pr.first == grow) continue;
      double t = pr.second * x[(size_t)(pr.first - A->ilower)];
      if (first) { acc = t; first = false; } else acc = acc + t;
    }
    y[r] = acc;
  }
}
static double dotv(const std::vector<double> &a, const std::vector<double> &b) {
  double s = 0; for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i]; return s;
}
// hypre_PCGSolve (HYPRE 2.27.0, pcg.c) with the identity preconditioner.
HYPRE_Int HYPRE_ParCSRPCGSolve(HYPRE_Solver S, HYPRE_ParCSRMatrix A, HYPRE_ParVector bv, HYPRE_ParVector xv) {
  std::vector<double> &b = bv->v, &x = xv->v; size_t n = b.size();
  double bb = dotv(b, b);
  S->iters = 0; S->relres = 0;
  if (bb == 0.0) { x = b; g_last_pcg_iters = 0; g_last_pcg_relres = 0; return 0; }
  double eps = S->tol * S->tol;
  std::vector<double> r(b), s(n), p(n);
  std::vector<double> ax(n); csr_matvec(A, x, ax);
  for (size_t i = 0; i < n; ++i) r[i] = r[i] + (-1.0) * ax[i];
  p = r;
  double gamma = dotv(r, p), iprod = gamma; int i = 0;
  while (i + 1 <= S->maxiter) {
    i++;
    csr_matvec(A, p, s);
    double sdotp = dotv(s, p);
    if (sdotp == 0.0) break;
    double alpha = gamma / sdotp, gamma_old = gamma;
    for (size_t q = 0; q < n; ++q) { x[q] = x[q] + alpha * p[q]; r[q] = r[q] - alpha * s[q]; }
    gamma = dotv(r, r); iprod = gamma;
    if (iprod / bb < eps) break;
    double beta = gamma / gamma_old;
    for (size_t q = 0; q < n; ++q) p[q] = r[q] + beta * p[q];
  }
  S->iters = i; S->relres = std::sqrt(iprod / bb);
  g_last_pcg_iters = i; g_last_pcg_relres = S->relres;
  return 0;
}

// ---------------------------------------------------------------- Scotch
static int scotch_unreachable() { std::fprintf(stderr, "scotch shim reached: nParts must be 1\n"); std::abort(); }
int SCOTCH_graphInit(SCOTCH_Graph *) { return scotch_unreachable(); }
int SCOTCH_graphBuild(SCOTCH_Graph *, SCOTCH_Num, SCOTCH_Num, const SCOTCH_Num *, const SCOTCH_Num *, const SCOTCH_Num *,
                      const SCOTCH_Num *, SCOTCH_Num, const SCOTCH_Num *, const SCOTCH_Num *) { return scotch_unreachable(); }
int SCOTCH_archInit(SCOTCH_Arch *) { return scotch_unreachable(); }
int SCOTCH_archCmplt(SCOTCH_Arch *, SCOTCH_Num) { return scotch_unreachable(); }
int SCOTCH_stratInit(SCOTCH_Strat *) { return scotch_unreachable(); }
int SCOTCH_stratGraphMapBuild(SCOTCH_Strat *, SCOTCH_Num, SCOTCH_Num, double) { return scotch_unreachable(); }
int SCOTCH_graphMap(SCOTCH_Graph *, const SCOTCH_Arch *, SCOTCH_Strat *, SCOTCH_Num *) { return scotch_unreachable(); }
