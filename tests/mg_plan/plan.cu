// Host-side check of mg::plan_stage (hsolver_b200/csrc/hs_mg.cuh): builds the
// level dimensions of a hierarchy the way the solvers' set-up does (2x
// coarsening, ceil, down to <= kMgCoarse cells) and prints, per precision,
// the first level block 0 handles alone, the staging bytes and each staged
// level's x / rhs offsets, then the first level whose couplings are staged too
// and their offsets.  No device code runs.
#include <cstdio>
#include <cstdlib>

#include "../../hsolver_b200/csrc/hs_mg.cuh"

template <class M>
void plan(int nx, int ny, int nz) {
  hs::mg::Hier<M> G{};
  int L = 0;
  while (true) {
    G.lv[L].nx = nx; G.lv[L].ny = ny; G.lv[L].nz = nz; G.lv[L].px = nx + 2;
    ++L;
    if ((long long)nx * ny * nz <= hs::mg::kMgCoarse) break;
    nx = (nx + 1) / 2; ny = (ny + 1) / 2; nz = (nz + 1) / 2;
  }
  G.L = L;
  hs::mg::plan_stage(G);
  std::printf("%d %d %d %d", (int)sizeof(M), G.L, G.ls, G.stage);
  for (int l = G.ls; l < G.L; ++l) std::printf(" %d:%d", G.sx[l], G.sr[l]);
  std::printf(" | %d", G.sro);
  for (int l = G.sro; l < G.L; ++l) std::printf(" %d:%d:%d", G.sg[l][0], G.sg[l][1], G.sg[l][2]);
  std::printf("\n");
}

int main(int argc, char **argv) {
  if (argc != 4) return 2;
  const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), nz = std::atoi(argv[3]);
  plan<double>(nx, ny, nz);
  plan<float>(nx, ny, nz);
  return 0;
}
