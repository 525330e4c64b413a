// Drop-in MobSolver (replaces mobs_solver.h's struct of the same name,
// mobs_solver.h:30-56): constructor signature and public state.  The solid
// region is identified by its local box metadata; the solve itself is part of
// the coupled GPU step driven by Solver::solve.
#pragma once
#include <map>
#include <stdexcept>
#include <vector>

#include "fluid_solver.h"

struct MobSolver {
  DistributedMesh &mesh;
  std::vector<I64> &metadata;
  std::vector<LocalCell> &t;
  std::vector<LocalFace> &mx;
  std::vector<LocalFace> &my;
  std::vector<LocalFace> &mz;
  std::vector<OutputData> result;
  std::vector<I64> idArray;
  std::map<int, OutputData> idToData;
  std::vector<double> t_temp;
  hs_ctx *engine = nullptr;  // set by Solver::solve
  int region = -1;           // solid region of the engine, matched by metadata

  MobSolver(DistributedMesh &m1, std::vector<I64> &m2, std::vector<LocalCell> &c, std::vector<LocalFace> &f1,
            std::vector<LocalFace> &f2, std::vector<LocalFace> &f3)
      : mesh(m1), metadata(m2), t(c), mx(f1), my(f2), mz(f3) {
    const I64 cx = metadata[0], cy = metadata[1], cz = metadata[2];
    t_temp.assign((size_t)((cx + 2) * (cy + 2) * (cz + 2)), 0.0);
  }

  void init() { need(); }
  void solve() { need(); }
  void setForNext() { need(); }

  // find the engine's region with this box and copy its temperatures
  void pull() {
    hs_ctx *e = need();
    const int ns = hs_num_solids(e);
    region = -1;
    for (int r = 0; r < ns && region < 0; ++r) {
      long long m[9];
      if (hs_solid_meta(e, r, m) != HS_OK) continue;
      bool same = true;
      for (int q = 0; q < 9; ++q) same = same && m[q] == metadata[q];
      if (same) region = r;
    }
    if (region < 0) throw std::runtime_error("MobSolver: no solid region with this metadata");
    const I64 cx = metadata[0], cy = metadata[1], cz = metadata[2];
    const long long np = (cx + 2) * (cy + 2) * (cz + 2), nc = cx * cy * cz;
    t_temp.resize((size_t)np);
    if (hs_get_solid(e, region, 0, t_temp.data(), np) != HS_OK) throw std::runtime_error(hs_last_error(nullptr));
    std::vector<double> tc((size_t)nc);
    if (hs_get_solid(e, region, 1, tc.data(), nc) != HS_OK) throw std::runtime_error(hs_last_error(nullptr));
    // a cell of the box belongs to the region when the case model says so
    long long d[3];
    hs_grid_dims(e, d);
    std::vector<unsigned char> ty((size_t)(d[0] * d[1] * d[2]));
    std::vector<int> rg(ty.size());
    hs_get_cell_types(e, ty.data(), rg.data(), (long long)ty.size());
    const I64 ox = metadata[6], oy = metadata[7], oz = metadata[8];
    t.resize((size_t)nc);
    for (I64 k = 0; k < cz; ++k)
      for (I64 j = 0; j < cy; ++j)
        for (I64 i = 0; i < cx; ++i) {
          const I64 c = i + cx * (j + cy * k);
          const I64 g = (ox - 1 + i) + d[0] * ((oy - 1 + j) + d[1] * (oz - 1 + k));
          t[c].data = tc[c];
          t[c].isEmpty = !(ty[g] == 1 && rg[g] == region);
        }
  }

  // the public state from a channel run: the temperatures of this box's
  // cells of solid region r (the deck's region order), padded t_temp with
  // the neighbouring cells' temperatures in its ghost layer
  void pull_channel(const ChannelFields &F, int r) {
    region = r;
    const I64 cx = metadata[0], cy = metadata[1], cz = metadata[2];
    const I64 ox = metadata[6] - 1, oy = metadata[7] - 1, oz = metadata[8] - 1;
    auto gidx = [&](I64 i, I64 j, I64 k) { return i + F.Nx * (j + F.Ny * k); };
    t.resize((size_t)(cx * cy * cz));
    for (I64 k = 0; k < cz; ++k)
      for (I64 j = 0; j < cy; ++j)
        for (I64 i = 0; i < cx; ++i) {
          const I64 g = gidx(ox + i, oy + j, oz + k);
          t[i + cx * (j + cy * k)].data = F.T[g];
          t[i + cx * (j + cy * k)].isEmpty = !(F.type[g] == 1 && F.region[g] == r);
        }
    t_temp.assign((size_t)((cx + 2) * (cy + 2) * (cz + 2)), 0.0);
    for (I64 k = -1; k <= cz; ++k)
      for (I64 j = -1; j <= cy; ++j)
        for (I64 i = -1; i <= cx; ++i) {
          const I64 gi = ox + i, gj = oy + j, gk = oz + k;
          if (gi < 0 || gj < 0 || gk < 0 || gi >= F.Nx || gj >= F.Ny || gk >= F.Nz) continue;
          t_temp[(i + 1) + (cx + 2) * ((j + 1) + (cy + 2) * (k + 1))] = F.T[gidx(gi, gj, gk)];
        }
  }

  // Solver::getResult for this solid (solver.h:189-211): temperature and location per cell
  void collect() {
    const I64 cx = metadata[0], cy = metadata[1], cz = metadata[2];
    const I64 ox = metadata[6], oy = metadata[7], oz = metadata[8];
    const CYCASMesh &g = mesh.cycasMesh;
    idToData.clear();
    for (I64 k = 0; k < cz; ++k)
      for (I64 j = 0; j < cy; ++j)
        for (I64 i = 0; i < cx; ++i) {
          const I64 c = i + cx * (j + cy * k);
          if (t[c].isEmpty) continue;
          const I64 gi = ox + i, gj = oy + j, gk = oz + k;
          OutputData d;
          d.t = t[c].data;
          d.locationx = g.xPoints[gi - 1];
          d.locationy = g.yPoints[gj - 1];
          d.locationz = g.zPoints[gk - 1];
          idToData[(int)((gi - 1) + (gj - 1) * g.Nx + (gk - 1) * g.Nx * g.Ny + 1)] = d;
        }
    idArray.clear();
    result.clear();
    for (auto &v : idToData) {
      idArray.push_back(v.first);
      result.push_back(v.second);
    }
  }

 private:
  hs_ctx *need() {
    if (!engine) throw std::logic_error("MobSolver runs inside Solver::solve (the GPU engine couples all regions)");
    return engine;
  }
};
