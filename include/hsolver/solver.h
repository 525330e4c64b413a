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

#include "channel_case.h"
#include "mobs_solver.h"

struct Solver {
  std::vector<FluidSolver *> fluids;
  std::vector<MobSolver *> mobs;
  int rank;
  int steps = 100;           // solver.h:55 runs 100 outer steps
  hs_params params;          // the reference's constants (hs_params_default)
  hs_ctx *engine = nullptr;
  hs_channel *channel = nullptr;  // the channel case, when the deck has a ".channel" sidecar
  hs_channel_stats channel_stats{};
  int channel_steps = 0;

  explicit Solver(int r) : rank(r) { hs_params_default(&params); }
  ~Solver() {
    if (engine) hs_destroy(engine);
    if (channel) hs_channel_destroy(channel);
  }
  Solver(const Solver &) = delete;
  Solver &operator=(const Solver &) = delete;

  void addFluids(FluidSolver *f) { fluids.push_back(f); }
  void addMobs(MobSolver *m) { mobs.push_back(m); }

  void solve() {
    const DistributedMesh *m = !fluids.empty() ? &fluids[0]->mesh : !mobs.empty() ? &mobs[0]->mesh : nullptr;
    if (!m) throw std::logic_error("Solver::solve without solvers");
    if (!m->cycasMesh.channel.empty()) {
      solve_channel(*m);
      return;
    }
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

  // The channel physics of the deck's sidecar (channel_case.h) on this
  // rank's GPU: create, the blocks' k ratio and heat source, init, then
  // `steps` outer steps, or steps until the sidecar's global-residual tol
  // (at most max_outer, default `steps`; not reaching it throws); the
  // fields then fill every solver's public state and result.
  void solve_channel(const DistributedMesh &m) {
    const ChannelSpec spec = parse_channel_spec(m.cycasMesh.channel);
    if (channel) hs_channel_destroy(channel);
    channel = nullptr;
    const std::string &deck = m.cycasMesh.deck;
    if (hs_channel_create(deck.c_str(), &spec.prm, rank, &channel) != HS_OK)
      throw std::runtime_error(hs_last_error(nullptr));
    int nb = 0;
    check_ch(hs_channel_num_blocks(channel, &nb));
    ChannelFields F;
    F.Nx = m.cycasMesh.Nx; F.Ny = m.cycasMesh.Ny; F.Nz = m.cycasMesh.Nz;
    const long long n = F.Nx * F.Ny * F.Nz;
    F.type.resize((size_t)n);
    F.region.resize((size_t)n);
    hs_case *c = nullptr;
    if (hs_case_create(deck.c_str(), &c) != HS_OK) throw std::runtime_error(hs_last_error(nullptr));
    const int rc = hs_case_cell_types(c, F.type.data(), F.region.data(), n);
    std::vector<std::vector<long long>> solid_meta((size_t)hs_case_num_solids(c), std::vector<long long>(9));
    for (size_t r = 0; r < solid_meta.size(); ++r) hs_case_solid_meta(c, (int)r, solid_meta[r].data());
    hs_case_destroy(c);
    check_ch(rc);
    auto per_block = [&](const std::vector<double> &v, const char *what, double dflt) {
      if (v.empty()) return std::vector<double>((size_t)nb, dflt);
      if (v.size() == 1) return std::vector<double>((size_t)nb, v[0]);
      if ((int)v.size() != nb)
        throw std::runtime_error(std::string("channel sidecar: ") + what + " needs one value or one per block (" +
                                 std::to_string(nb) + ")");
      return v;
    };
    const std::vector<double> k = per_block(spec.k_ratio, "k_ratio", 100.0), qb = per_block(spec.q, "q", 0.0);
    std::vector<double> q((size_t)n, 0.0);
    for (long long e = 0; e < n; ++e)
      if (F.type[e] == 1) q[e] = qb[F.region[e]];
    check_ch(hs_channel_set_solid(channel, k.data(), nb, q.data(), n));
    check_ch(hs_channel_init(channel));
    if (spec.tol > 0) {
      const int rc2 = hs_channel_solve_to(channel, spec.tol, spec.max_outer > 0 ? spec.max_outer : steps,
                                          &channel_steps, &channel_stats);
      check_ch(rc2);
    } else {
      check_ch(hs_channel_step(channel, steps, 0, &channel_stats));
      channel_steps = steps;
    }
    std::vector<double> *dst[5] = {&F.u, &F.v, &F.w, &F.p, &F.T};
    for (int f = 0; f < 5; ++f) {
      long long sz = 0;
      check_ch(hs_channel_field_size(channel, f, &sz));
      dst[f]->resize((size_t)sz);
      check_ch(hs_channel_get_field(channel, f, dst[f]->data(), sz));
    }
    for (auto *f : fluids) {
      f->pull_channel(F);
      f->collect();
    }
    for (auto *s : mobs) {
      int r = -1;
      for (size_t q2 = 0; q2 < solid_meta.size() && r < 0; ++q2) {
        bool same = true;
        for (int e = 0; e < 9; ++e) same = same && solid_meta[q2][e] == s->metadata[e];
        if (same) r = (int)q2;
      }
      if (r < 0) throw std::runtime_error("MobSolver: no solid region with this metadata");
      s->pull_channel(F, r);
      s->collect();
    }
  }

 private:
  void check(int rc) {
    if (rc != HS_OK) throw std::runtime_error(hs_last_error(engine));
  }
  static void check_ch(int rc) {
    if (rc != HS_OK) throw std::runtime_error(hs_last_error(nullptr));
  }
};
