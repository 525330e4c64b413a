// Host-side case model: deck parsing, cell / face classification, connected
// regions, the per-region local boxes and the fluid<->solid interface pairs.
// This is the reference's decompose + CYCASMesh + DistributedMesh front end
// for a single rank (nParts = 1), rebuilt as flat arrays for the GPU path.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace hs {

// Local box of one region: cell sizes, face sizes and 1-based global offsets
// of its first cell (the 9-entry metadata of distributed_mesh.h:152-154).
struct Meta {
  long cx = 0, cy = 0, cz = 0, fx = 0, fy = 0, fz = 0, ox = 0, oy = 0, oz = 0;
  long ncell() const { return cx * cy * cz; }
  long npad() const { return (cx + 2) * (cy + 2) * (cz + 2); }
  long nu() const { return (fx + 2) * (cy + 2) * (cz + 2); }
  long nv() const { return (cx + 2) * (fy + 2) * (cz + 2); }
  long nw() const { return (cx + 2) * (cy + 2) * (fz + 2); }
};

struct Deck {
  std::vector<double> xs, ys, zs;
  std::vector<std::array<int, 6>> mobs;
  std::vector<std::array<int, 8>> walls;
  std::vector<std::array<int, 13>> holes;
};

// One fluid<->solid interface face, as padded indices: the fluid sends
// T[f_send] into the solid's s_recv, the solid sends T[s_send] into the
// fluid's f_recv (solver.h:83-148 with the lists of fluid_solver.h:983-1006
// and mobs_solver.h:147-167).
struct SwapPair {
  long f_send, f_recv, s_send, s_recv;
  int region;
};

struct Case {
  Deck deck;
  long Nx = 0, Ny = 0, Nz = 0;
  std::vector<uint8_t> ctype;          // Nx*Ny*Nz, 0 fluid, 1 obstacle
  std::vector<int> region;             // region id within its type
  std::vector<uint8_t> wx, wy, wz;     // wall flags of x / y / z faces
  int nfluid_regions = 0, nsolid_regions = 0;

  Meta fluid;
  std::vector<uint8_t> fluid_empty;    // cx*cy*cz, LocalCell::isEmpty
  std::vector<uint8_t> ib_x, ib_y, ib_z;  // fluid-box faces that are "ib_" faces
  std::vector<int> row_id;             // HYPRE row per fluid-box cell (-1 empty)
  long nfluid = 0;
  // per padded index geometry (fluid_solver.h:1248-1261), size n+2
  std::vector<double> xp, xw, xe, yp, ys, yn, zp, zf, zb;

  std::vector<Meta> solids;
  std::vector<std::vector<uint8_t>> solid_empty;
  std::vector<SwapPair> swap;
};

// Parse the `.in` text; returns false with `err` set on failure.
bool parse_deck(const std::string &text, Deck &deck, std::string &err);
// Classify cells and faces and build every region's local box.
bool build_case(const Deck &deck, Case &c, std::string &err);

}  // namespace hs
