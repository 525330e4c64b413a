// The reference's main.cpp sequence (main.cpp:18-156) on one process with the
// drop-in headers: deck -> CYCASMesh -> DistributedMesh -> one FluidSolver per
// fluid region and one MobSolver per solid region -> Solver::solve ->
// results keyed by global cell id -> result.vtk.  MPI_Init / MPI_Gather of a
// single rank reduce to the local vectors.
//   driver <deck.in> <outer steps> <result.vtk>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>

#include "hsolver/distributed_mesh.h"
#include "hsolver/fluid_solver.h"
#include "hsolver/mesh.h"
#include "hsolver/mobs_solver.h"
#include "hsolver/result_vtk.h"
#include "hsolver/solver.h"

int main(int argc, char **argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s deck.in steps result.vtk\n", argv[0]);
    return 2;
  }
  int rank = 0;
  std::string filename = argv[1];
  CYCASMesh mesh(filename, rank);
  mesh.readCells(rank);
  mesh.readFaces(rank);
  mesh.readBoundaries(rank);
  DistributedMesh newMesh(mesh);
  newMesh.generateLocalDomain();

  std::vector<OutputData> local_result;
  std::vector<I64> local_id;
  Solver solver(rank);
  solver.steps = std::atoi(argv[2]);
  for (auto iter = newMesh.fluidMetadata.begin(); iter != newMesh.fluidMetadata.end(); ++iter) {
    auto id = iter->first;
    FluidSolver *fluidSolver = new FluidSolver(newMesh, newMesh.fluidMetadata[id], newMesh.p[id], newMesh.ux[id],
                                               newMesh.uy[id], newMesh.uz[id]);
    solver.addFluids(fluidSolver);
  }
  for (auto iter = newMesh.solidMetadata.begin(); iter != newMesh.solidMetadata.end(); ++iter) {
    auto id = iter->first;
    MobSolver *mobSolver = new MobSolver(newMesh, newMesh.solidMetadata[id], newMesh.mt[id], newMesh.mx[id],
                                         newMesh.my[id], newMesh.mz[id]);
    solver.addMobs(mobSolver);
  }
  try {
    solver.solve();
  } catch (const std::exception &e) {
    std::fprintf(stderr, "solve failed: %s\n", e.what());
    return 1;
  }
  for (auto &e : solver.fluids) {
    local_result.insert(local_result.end(), e->result.begin(), e->result.end());
    local_id.insert(local_id.end(), e->idArray.begin(), e->idArray.end());
  }
  for (auto &e : solver.mobs) {
    local_result.insert(local_result.end(), e->result.begin(), e->result.end());
    local_id.insert(local_id.end(), e->idArray.begin(), e->idArray.end());
  }
  std::map<I64, OutputData> resultMap;
  for (size_t i = 0; i < local_id.size(); ++i) resultMap[local_id[i]] = local_result[i];
  write_result_vtk(argv[3], resultMap, mesh.Nx, mesh.Ny, mesh.Nz);
  std::printf("VTK file written: %s (%zu points)\n", argv[3], resultMap.size());
  for (auto *f : solver.fluids) delete f;
  for (auto *m : solver.mobs) delete m;
  return 0;
}
