// Drop-in DistributedMesh (replaces distributed_mesh.h's struct of the same
// name, distributed_mesh.h:30-62): the local box metadata of every region
// and the per-region output arrays the solvers write, built from the deck
// by the C ABI's case model.  Region keys follow the reference: fluid and
// solid regions are numbered separately from 0.
#pragma once
#include <map>
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

  // every region's local box and output arrays (sizes as the reference's)
  void generateLocalDomain() {
    hs_case *c = nullptr;
    if (hs_case_create(cycasMesh.deck.c_str(), &c) != HS_OK) throw std::runtime_error(hs_last_error(nullptr));
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
};
