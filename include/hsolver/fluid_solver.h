// Drop-in FluidSolver (replaces fluid_solver.h's struct of the same name,
// fluid_solver.h:46-109): the constructor signature and the public state a
// driver reads (result, idArray, t_temp, u_star, ...).  The GPU engine steps
// the fluid, every solid region and the interface swap together, so the
// numerical work is driven by Solver::solve (solver.h below); init / solve /
// setForNext act on that shared engine once Solver has created it.
#pragma once
#include <map>
#include <stdexcept>
#include <vector>

#include "distributed_mesh.h"

struct OutputData {
  double ux = 0, uy = 0, uz = 0, p = 0;
  double t = 0;
  double locationx = 0.0;
  double locationy = 0.0;
  double locationz = 0.0;
  int globalid = -1;
};

// the fields of a channel run (Solver::solve with a ".channel" sidecar) on
// the global grid: face velocities (Nx+1)NyNz, Nx(Ny+1)Nz, NxNy(Nz+1), cell
// pressure and temperature, cell type (0 fluid, 1 solid) and solid region
struct ChannelFields {
  I64 Nx = 0, Ny = 0, Nz = 0;
  std::vector<double> u, v, w, p, T;
  std::vector<unsigned char> type;
  std::vector<int> region;
};

struct FluidSolver {
  DistributedMesh &mesh;
  std::vector<I64> &metadata;
  std::vector<LocalCell> &p;
  std::vector<LocalFace> &ux;
  std::vector<LocalFace> &uy;
  std::vector<LocalFace> &uz;
  std::vector<LocalCell> t;
  std::vector<int> id;
  std::vector<double> u_star, v_star, w_star, up, vp, wp, p_temp, p_prime, t_temp;
  std::vector<OutputData> result;
  std::vector<I64> idArray;
  std::map<int, OutputData> idToData;
  hs_ctx *engine = nullptr;  // set by Solver::solve

  FluidSolver(DistributedMesh &m, std::vector<I64> &md, std::vector<LocalCell> &pc, std::vector<LocalFace> &fx,
              std::vector<LocalFace> &fy, std::vector<LocalFace> &fz)
      : mesh(m), metadata(md), p(pc), ux(fx), uy(fy), uz(fz) {
    const I64 cx = metadata[0], cy = metadata[1], cz = metadata[2];
    t.assign((size_t)(cx * cy * cz), LocalCell());
  }

  // FluidSolver::init / solve (fluid_solver.h:882, 1401): the coupled
  // engine's init and one full outer step; setForNext is part of the step
  void init() { check(hs_init(need())); }
  void solve() { check(hs_step(need(), 1, nullptr)); }
  void setForNext() { need(); }

  // copy the engine's fields into the public state (after Solver::solve)
  void pull() {
    hs_ctx *e = need();
    struct F { int id; std::vector<double> *v; } f[] = {{HS_F_U_STAR, &u_star}, {HS_F_V_STAR, &v_star},
        {HS_F_W_STAR, &w_star}, {HS_F_UP, &up}, {HS_F_VP, &vp}, {HS_F_WP, &wp}, {HS_F_P_TEMP, &p_temp},
        {HS_F_P_PRIME, &p_prime}, {HS_F_T_TEMP, &t_temp}};
    for (auto &x : f) {
      long long n = 0;
      check(hs_field_size(e, x.id, &n));
      x.v->resize((size_t)n);
      check(hs_get_field(e, x.id, x.v->data(), n));
    }
    std::vector<double> a;
    auto faces = [&](int fid, std::vector<LocalFace> &out) {
      long long n = 0;
      check(hs_field_size(e, fid, &n));
      a.resize((size_t)n);
      check(hs_get_field(e, fid, a.data(), n));
      out.resize((size_t)n);
      for (long long i = 0; i < n; ++i) out[i].u = a[i];
    };
    faces(HS_F_UX, ux); faces(HS_F_UY, uy); faces(HS_F_UZ, uz);
    const long long nc = metadata[0] * metadata[1] * metadata[2];
    std::vector<unsigned char> empty((size_t)nc);
    check(hs_get_fluid_mask(e, empty.data(), nc));
    std::vector<double> pc((size_t)nc), tc((size_t)nc);
    check(hs_get_field(e, HS_F_P, pc.data(), nc));
    check(hs_get_field(e, HS_F_T, tc.data(), nc));
    id.resize((size_t)nc);
    check(hs_get_row_ids(e, id.data(), nc));
    p.resize((size_t)nc);
    t.resize((size_t)nc);
    for (long long i = 0; i < nc; ++i) {
      p[i].data = pc[i]; p[i].isEmpty = empty[i] != 0;
      t[i].data = tc[i]; t[i].isEmpty = empty[i] != 0;
    }
  }

  // the public state from a channel run: the fluid box's faces and cells
  // (metadata {cx,cy,cz,fx,fy,fz,ox,oy,oz}, 1-based origin), row ids
  // numbering the fluid cells in k-j-i order as the reference's rows do
  // (fluid_solver.h:1894-1906)
  void pull_channel(const ChannelFields &F) {
    const I64 cx = metadata[0], cy = metadata[1], cz = metadata[2], fx = metadata[3], fy = metadata[4],
              fz = metadata[5];
    const I64 ox = metadata[6] - 1, oy = metadata[7] - 1, oz = metadata[8] - 1;
    const I64 Nx = F.Nx, Ny = F.Ny;
    ux.resize((size_t)(fx * cy * cz));
    uy.resize((size_t)(cx * fy * cz));
    uz.resize((size_t)(cx * cy * fz));
    for (I64 k = 0; k < cz; ++k)
      for (I64 j = 0; j < cy; ++j)
        for (I64 i = 0; i < fx; ++i) ux[i + fx * (j + cy * k)].u = F.u[(ox + i) + (Nx + 1) * ((oy + j) + Ny * (oz + k))];
    for (I64 k = 0; k < cz; ++k)
      for (I64 j = 0; j < fy; ++j)
        for (I64 i = 0; i < cx; ++i) uy[i + cx * (j + fy * k)].u = F.v[(ox + i) + Nx * ((oy + j) + (Ny + 1) * (oz + k))];
    for (I64 k = 0; k < fz; ++k)
      for (I64 j = 0; j < cy; ++j)
        for (I64 i = 0; i < cx; ++i) uz[i + cx * (j + cy * k)].u = F.w[(ox + i) + Nx * ((oy + j) + Ny * (oz + k))];
    const I64 nc = cx * cy * cz;
    p.resize((size_t)nc);
    t.resize((size_t)nc);
    id.assign((size_t)nc, -1);
    int row = 0;
    for (I64 k = 0; k < cz; ++k)
      for (I64 j = 0; j < cy; ++j)
        for (I64 i = 0; i < cx; ++i) {
          const I64 c = i + cx * (j + cy * k), g = (ox + i) + Nx * ((oy + j) + Ny * (oz + k));
          const bool empty = F.type[g] != 0;
          p[c].data = F.p[g]; p[c].isEmpty = empty;
          t[c].data = F.T[g]; t[c].isEmpty = empty;
          if (!empty) id[c] = row++;
        }
  }

  // Solver::getResult for this fluid (solver.h:160-188): one OutputData per
  // fluid cell, keyed and ordered by the 1-based global cell index
  void collect() {
    const I64 cx = metadata[0], cy = metadata[1], cz = metadata[2], fx = metadata[3], fy = metadata[4];
    const I64 ox = metadata[6], oy = metadata[7], oz = metadata[8];
    const CYCASMesh &g = mesh.cycasMesh;
    idToData.clear();
    for (I64 k = 0; k < cz; ++k)
      for (I64 j = 0; j < cy; ++j)
        for (I64 i = 0; i < cx; ++i) {
          const I64 c = i + cx * (j + cy * k);
          if (p[c].isEmpty) continue;
          const I64 gi = ox + i, gj = oy + j, gk = oz + k;  // 1-based global
          OutputData d;
          d.ux = ux[i + fx * (j + cy * k)].u;
          d.uy = uy[i + cx * (j + fy * k)].u;
          d.uz = uz[i + cx * (j + cy * k)].u;
          d.p = p[c].data;
          d.t = t[c].data;
          d.globalid = id[c];
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
    if (!engine) throw std::logic_error("FluidSolver runs inside Solver::solve (the GPU engine couples all regions)");
    return engine;
  }
  static void check(int rc) {
    if (rc != HS_OK) throw std::runtime_error(hs_last_error(nullptr));
  }
};
