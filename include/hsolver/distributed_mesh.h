// Drop-in DistributedMesh (replaces distributed_mesh.h's struct of the same
// name, distributed_mesh.h:30-62): the local box metadata of every region
// and the per-region output arrays the solvers write, built from the deck
// by the C ABI's case model.  Region keys follow the reference: fluid and
// solid regions are numbered separately from 0.
#pragma once
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "mesh.h"

struct LocalCell {
  double data = 0.0;
  bool isEmpty = true;
};

struct LocalFace {
  bool isBoundary = false;
  double u = 0.0;
  void *info = nullptr;
  double location = 0.0;
};

struct DistributedMesh {
  explicit DistributedMesh(const CYCASMesh &mesh) : cycasMesh(mesh) {}
  CYCASMesh cycasMesh;

  std::map<int, std::vector<LocalCell>> p;          // fluid cells of each fluid box
  std::map<int, std::vector<LocalFace>> ux, uy, uz;
  std::map<int, std::vector<I64>> fluidMetadata;    // {cx, cy, cz, fx, fy, fz, ox, oy, oz}
  std::map<int, std::vector<LocalCell>> mt;         // solid cells of each solid box
  std::map<int, std::vector<LocalFace>> mx, my, mz;
  std::map<int, std::vector<I64>> solidMetadata;

  // every region's local box and output arrays (sizes as the reference's);
  // cells read from processor files must be the deck's
  void generateLocalDomain() {
    hs_case *c = nullptr;
    if (hs_case_create(cycasMesh.deck.c_str(), &c) != HS_OK) throw std::runtime_error(hs_last_error(nullptr));
    try {
      check_processor_cells(c);
    } catch (...) {
      hs_case_destroy(c);
      throw;
    }
    long long m[9];
    hs_case_fluid_meta(c, m);
    fluidMetadata[0] = std::vector<I64>(m, m + 9);
    p[0].assign((size_t)(m[0] * m[1] * m[2]), LocalCell());
    ux[0].assign((size_t)(m[3] * m[1] * m[2]), LocalFace());
    uy[0].assign((size_t)(m[0] * m[4] * m[2]), LocalFace());
    uz[0].assign((size_t)(m[0] * m[1] * m[5]), LocalFace());
    const int ns = hs_case_num_solids(c);
    for (int r = 0; r < ns; ++r) {
      hs_case_solid_meta(c, r, m);
      solidMetadata[r] = std::vector<I64>(m, m + 9);
      mt[r].assign((size_t)(m[0] * m[1] * m[2]), LocalCell());
      mx[r].assign((size_t)(m[3] * m[1] * m[2]), LocalFace());
      my[r].assign((size_t)(m[0] * m[4] * m[2]), LocalFace());
      mz[r].assign((size_t)(m[0] * m[1] * m[5]), LocalFace());
    }
    hs_case_destroy(c);
  }

 private:
  // the cells of each region in the processor files (1-based global indices,
  // mesh/mesh.cpp:2300-2330) against the deck's cell types and regions: one
  // rank holds every region whole (nParts = 1)
  void check_processor_cells(hs_case *c) const {
    const CYCASMesh &g = cycasMesh;
    if (g.fluidRegions.empty() && g.mobsRegions.empty()) return;
    const long long n = g.Nx * g.Ny * g.Nz;
    std::vector<unsigned char> type((size_t)n);
    std::vector<int> region((size_t)n);
    if (hs_case_cell_types(c, type.data(), region.data(), n) != HS_OK) throw std::runtime_error(hs_last_error(nullptr));
    auto expect = [&](bool solid, int r) {
      std::vector<I64> v;
      for (long long e = 0; e < n; ++e)
        if ((type[e] != 0) == solid && (!solid || region[e] == r)) v.push_back(e + 1);
      return v;
    };
    if (g.fluidRegions.size() != 1 || g.fluidRegions.count(0) != 1 || g.fluidRegions.at(0) != expect(false, 0))
      throw std::runtime_error("processor files: the fluid cells are not the deck's (files of another deck or rank?)");
    if ((int)g.mobsRegions.size() != hs_case_num_solids(c))
      throw std::runtime_error("processor files: the number of solid regions is not the deck's");
    for (auto &kv : g.mobsRegions)
      if (kv.second != expect(true, kv.first))
        throw std::runtime_error("processor files: the cells of solid region " + std::to_string(kv.first) +
                                 " are not the deck's");
  }
};
