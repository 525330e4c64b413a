// Runs the reference's own FluidSolver / MobSolver sources single-rank and
// dumps their state, to pin the oracle restatement (test infrastructure).
//
//   ref_driver <deck.in> <workdir> <out_prefix> <step,step,...>   per-step dumps
//   ref_driver <deck.in> <workdir> <out_prefix> solver            Solver::solve() (100 steps)
//   ref_driver <deck.in> <workdir> - time:N                       N outer steps, timed
//
// The deck is decomposed with nParts = 1 (decompose.cpp:8 uses 4), the
// processor0/ files are written into <workdir> and read back exactly like
// main.cpp:18-45.  Dumps are records of [name[32] | kind i32 | count i64 |
// data] with kind 0 = f64, 1 = i32.
#include <unistd.h>
#include <sys/stat.h>
#include <cstdio>
#include <chrono>
#include <cstring>
#include <ctime>
#include <set>
#include <string>
#include <vector>
#include "mpi.h"
#include "mesh/mesh.h"
#include "distributed_mesh.h"
#include "fluid_solver.h"
#include "mobs_solver.h"
#include "solver.h"

extern "C" int hs_shim_last_pcg_iters(void);

static void rec(FILE *f, const char *name, int kind, const void *data, long long n) {
  char nm[32] = {0}; std::strncpy(nm, name, 31);
  std::fwrite(nm, 1, 32, f); std::fwrite(&kind, 4, 1, f); std::fwrite(&n, 8, 1, f);
  std::fwrite(data, kind == 0 ? 8 : 4, (size_t)n, f);
}
static std::vector<double> face_u(const std::vector<LocalFace> &v) { std::vector<double> o; for (auto &e : v) o.push_back(e.u); return o; }
static std::vector<double> cell_d(const std::vector<LocalCell> &v) { std::vector<double> o; for (auto &e : v) o.push_back(e.data); return o; }
static std::vector<int> cell_e(const std::vector<LocalCell> &v) { std::vector<int> o; for (auto &e : v) o.push_back(e.isEmpty ? 1 : 0); return o; }

static void dump(const std::string &path, Solver &s, int pcg_iters) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) { std::perror(path.c_str()); std::exit(2); }
  for (size_t n = 0; n < s.fluids.size(); ++n) {
    FluidSolver *e = s.fluids[n];
    std::vector<double> meta(e->metadata.begin(), e->metadata.end());
    rec(f, "fluid.meta", 0, meta.data(), (long long)meta.size());
    rec(f, "u_star", 0, e->u_star.data(), (long long)e->u_star.size());
    rec(f, "v_star", 0, e->v_star.data(), (long long)e->v_star.size());
    rec(f, "w_star", 0, e->w_star.data(), (long long)e->w_star.size());
    rec(f, "up", 0, e->up.data(), (long long)e->up.size());
    rec(f, "vp", 0, e->vp.data(), (long long)e->vp.size());
    rec(f, "wp", 0, e->wp.data(), (long long)e->wp.size());
    rec(f, "p_temp", 0, e->p_temp.data(), (long long)e->p_temp.size());
    rec(f, "t_temp", 0, e->t_temp.data(), (long long)e->t_temp.size());
    auto ux = face_u(e->ux), uy = face_u(e->uy), uz = face_u(e->uz), p = cell_d(e->p), t = cell_d(e->t);
    rec(f, "ux", 0, ux.data(), (long long)ux.size());
    rec(f, "uy", 0, uy.data(), (long long)uy.size());
    rec(f, "uz", 0, uz.data(), (long long)uz.size());
    rec(f, "p", 0, p.data(), (long long)p.size());
    rec(f, "t", 0, t.data(), (long long)t.size());
    auto em = cell_e(e->p);
    rec(f, "fluid.empty", 1, em.data(), (long long)em.size());
    rec(f, "id", 1, e->id.data(), (long long)e->id.size());
    std::vector<int> tb, th;
    for (auto &kv : e->t_boundary) for (auto a : kv.second) tb.push_back((int)a);
    for (auto &kv : e->t_halo) for (auto a : kv.second) th.push_back((int)a);
    rec(f, "fluid.t_boundary", 1, tb.data(), (long long)tb.size());
    rec(f, "fluid.t_halo", 1, th.data(), (long long)th.size());
  }
  for (size_t n = 0; n < s.mobs.size(); ++n) {
    MobSolver *m = s.mobs[n];
    std::vector<double> meta(m->metadata.begin(), m->metadata.end());
    rec(f, "solid.meta", 0, meta.data(), (long long)meta.size());
    rec(f, "solid.t_temp", 0, m->t_temp.data(), (long long)m->t_temp.size());
    auto t = cell_d(m->t); auto em = cell_e(m->t);
    rec(f, "solid.t", 0, t.data(), (long long)t.size());
    rec(f, "solid.empty", 1, em.data(), (long long)em.size());
    std::vector<int> tb, th;
    for (auto &kv : m->t_boundary) for (auto a : kv.second) tb.push_back((int)a);
    for (auto &kv : m->t_halo) for (auto a : kv.second) th.push_back((int)a);
    rec(f, "solid.t_boundary", 1, tb.data(), (long long)tb.size());
    rec(f, "solid.t_halo", 1, th.data(), (long long)th.size());
  }
  rec(f, "pcg_iters", 1, &pcg_iters, 1);
  std::fclose(f);
}

// one pass of the loop body of Solver::solve (solver.h:55-154), single rank:
// the fluid's and the solids' interface messages are self-messages.
static void one_step(Solver &solver) {
  for (auto *e : solver.fluids) e->solve();
  for (auto *e : solver.mobs) e->solve();
  std::vector<double> fsend, ssend;
  for (auto *e : solver.fluids) for (auto &kv : e->t_boundary) for (auto a : kv.second) fsend.push_back(e->t_temp[a]);
  for (auto *e : solver.mobs) for (auto &kv : e->t_boundary) for (auto a : kv.second) ssend.push_back(e->t_temp[a]);
  size_t n = 0;
  for (auto *e : solver.fluids) for (auto &kv : e->t_halo) for (auto a : kv.second) e->t_temp[a] = ssend.at(n++);
  n = 0;
  for (auto *e : solver.mobs) for (auto &kv : e->t_halo) for (auto a : kv.second) e->t_temp[a] = fsend.at(n++);
  for (auto *e : solver.fluids) e->setForNext();
  for (auto *e : solver.mobs) e->setForNext();
}

int main(int argc, char **argv) {
  if (argc < 5) { std::fprintf(stderr, "usage: %s deck workdir out_prefix steps|solver\n", argv[0]); return 2; }
  char deck[4096];
  if (!realpath(argv[1], deck)) { std::perror(argv[1]); return 2; }
  std::string outp = argv[3];
  if (outp[0] != '/') { char cwd[4096]; if (getcwd(cwd, sizeof cwd)) outp = std::string(cwd) + "/" + outp; }
  mkdir(argv[2], 0755);
  if (chdir(argv[2])) { std::perror(argv[2]); return 2; }
  MPI_Init(&argc, &argv);
  const auto s0 = std::chrono::steady_clock::now();
  {
    StructuredMesh mesh(deck);
    std::vector<std::vector<I64>> fR, mR;
    mesh.getConnectedRegions(fR, mR);
    mesh.decomposeMesh(fR, mR, 1);
    mesh.writeProcFile("test", 1);
  }
  CYCASMesh cm(deck, 0);
  cm.readCells(0); cm.readFaces(0); cm.readBoundaries(0);
  DistributedMesh dm(cm);
  dm.generateLocalDomain();
  Solver solver(0);
  for (auto &kv : dm.fluidMetadata)
    solver.addFluids(new FluidSolver(dm, dm.fluidMetadata[kv.first], dm.p[kv.first], dm.ux[kv.first], dm.uy[kv.first], dm.uz[kv.first]));
  for (auto &kv : dm.solidMetadata)
    solver.addMobs(new MobSolver(dm, dm.solidMetadata[kv.first], dm.mt[kv.first], dm.mx[kv.first], dm.my[kv.first], dm.mz[kv.first]));
  const double setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
  if (std::string(argv[4]) == "solver") {
    solver.solve();
    dump(outp + ".solver.bin", solver, hs_shim_last_pcg_iters());
    return 0;
  }
  if (std::string(argv[4]).rfind("time:", 0) == 0) {
    // the loop body of Solver::solve (solver.h:55-154) timed per step, by
    // clock() as solver.h:51-58 does and by the wall clock; one JSON line
    const int n = std::stoi(std::string(argv[4]).substr(5));
    const auto w0 = std::chrono::steady_clock::now();
    for (auto *e : solver.fluids) e->init();
    for (auto *e : solver.mobs) e->init();
    const double init_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    std::printf("{\"setup_s\": %.6f, \"init_s\": %.6f, \"steps\": [", setup_s, init_s);
    for (int step = 1; step <= n; ++step) {
      const clock_t c0 = clock();
      const auto t0 = std::chrono::steady_clock::now();
      one_step(solver);
      const double cpu = double(clock() - c0) / CLOCKS_PER_SEC;
      const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      std::printf("%s{\"clock_s\": %.6f, \"wall_s\": %.6f, \"pcg_iters\": %d}", step > 1 ? ", " : "", cpu, wall,
                  hs_shim_last_pcg_iters());
    }
    std::printf("]}\n");
    return 0;
  }
  std::set<int> want;
  { std::string s = argv[4]; size_t p = 0; while (p < s.size()) { size_t q = s.find(',', p); if (q == std::string::npos) q = s.size(); want.insert(std::stoi(s.substr(p, q - p))); p = q + 1; } }
  int last = want.empty() ? 0 : *want.rbegin();
  for (auto *e : solver.fluids) e->init();
  for (auto *e : solver.mobs) e->init();
  if (want.count(0)) dump(outp + ".step0.bin", solver, 0);
  for (int step = 1; step <= last; ++step) {
    one_step(solver);
    if (want.count(step)) dump(outp + ".step" + std::to_string(step) + ".bin", solver, hs_shim_last_pcg_iters());
  }
  return 0;
}
