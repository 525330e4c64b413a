// Drop-in Solver (replaces solver.h's struct of the same name, solver.h:18-44):
// addFluids / addMobs / solve with the reference's semantics: init every
// solver, 100 outer steps (fluid, solids, interface swap, setForNext), the
// average step time over steps 10..99 printed, then the per-cell results.
// One hs_ctx (include/hsolver_b200.h) runs all regions on one GPU; the rank
// picks the device.  Link with -lhsolver_b200 -lcudart.
#pragma once
#include <chrono>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "mobs_solver.h"

struct Solver {
  std::vector<FluidSolver *> fluids;
  std::vector<MobSolver *> mobs;
  int rank;
  int steps = 100;           // solver.h:55 runs 100 outer steps
  hs_params params;          // the reference's constants (hs_params_default)
  hs_ctx *engine = nullptr;

  explicit Solver(int r) : rank(r) { hs_params_default(&params); }
  ~Solver() {
    if (engine) hs_destroy(engine);
  }
  Solver(const Solver &) = delete;
  Solver &operator=(const Solver &) = delete;

  void addFluids(FluidSolver *f) { fluids.push_back(f); }
  void addMobs(MobSolver *m) { mobs.push_back(m); }

  void solve() {
    const DistributedMesh *m = !fluids.empty() ? &fluids[0]->mesh : !mobs.empty() ? &mobs[0]->mesh : nullptr;
    if (!m) throw std::logic_error("Solver::solve without solvers");
    if (engine) hs_destroy(engine);
    engine = nullptr;
    if (hs_create(m->cycasMesh.deck.c_str(), &params, rank, &engine) != HS_OK)
      throw std::runtime_error(hs_last_error(nullptr));
    for (auto *f : fluids) f->engine = engine;
    for (auto *s : mobs) s->engine = engine;
    check(hs_init(engine));
    const int warm = steps < 10 ? steps : 10;
    check(hs_step(engine, warm, nullptr));
    check(hs_sync(engine));
    auto t0 = std::chrono::steady_clock::now();
    check(hs_step(engine, steps - warm, nullptr));
    check(hs_sync(engine));
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (steps > warm) std::printf("time: %g s  average: %g s per outer step\n", dt, dt / (steps - warm));
    getResult();
  }

  void getResult() {
    for (auto *f : fluids) { f->pull(); f->collect(); }
    for (auto *s : mobs) { s->pull(); s->collect(); }
  }

 private:
  void check(int rc) {
    if (rc != HS_OK) throw std::runtime_error(hs_last_error(engine));
  }
};
