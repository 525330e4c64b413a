// Reads a deck's processor files with the drop-in CYCASMesh (run from the
// directory that holds processor0/) and checks them against the deck in
// DistributedMesh::generateLocalDomain; prints what was read.
//   proc_check <deck.in>
#include <cstdio>
#include <exception>

#include "hsolver/distributed_mesh.h"
#include "hsolver/mesh.h"

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  try {
    CYCASMesh mesh(argv[1], 0);
    mesh.readCells(0);
    mesh.readFaces(0);
    mesh.readBoundaries(0);
    DistributedMesh dm(mesh);
    dm.generateLocalDomain();
    for (auto &kv : mesh.fluidRegions) std::printf("fluid %d cells %zu\n", kv.first, kv.second.size());
    for (auto &kv : mesh.mobsRegions) std::printf("mobs %d cells %zu\n", kv.first, kv.second.size());
    for (auto &kv : mesh.fluidFaces) std::printf("fluid %d faces %zu\n", kv.first, kv.second.size());
    for (auto &kv : mesh.mobsFaces) std::printf("mobs %d faces %zu\n", kv.first, kv.second.size());
    for (auto &kv : mesh.fluidBoundaries)
      for (auto &b : kv.second) std::printf("fluid %d boundary %s %d %d\n", kv.first, b.first.c_str(), b.second.startFace, b.second.nFaces);
    for (auto &kv : mesh.mobsBoundaries)
      for (auto &b : kv.second) std::printf("mobs %d boundary %s %d %d\n", kv.first, b.first.c_str(), b.second.startFace, b.second.nFaces);
  } catch (const std::exception &e) {
    std::printf("error: %s\n", e.what());
    return 1;
  }
  return 0;
}
