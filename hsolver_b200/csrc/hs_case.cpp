// Deck reader and mesh classification for the single-GPU path.
//
// Deck rules follow StructuredMesh::readMesh (mesh/mesh.cpp:1616-1796): each
// section runs from the '=' after its key up to the next key; comments run
// from ';' to the end of the line; values are read as `value separator`
// pairs, so a value without a following separator is dropped
// (mesh/mesh.cpp:1677).  The per-rank reader CYCASMesh::readMesh
// (mesh/mesh.cpp:2419-2420) only agrees with it when the deck starts with
// `xgrid` and the grid keys come in x, y, z, mobs order; decks that break
// this are rejected here instead of being misread.
#include "hs_case.hpp"

#include <algorithm>
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <deque>

namespace hs {
namespace {

bool is_space(char ch) { return ch == ' ' || ch == '\t' || ch == '\r' || ch == '\v' || ch == '\f'; }

// Numbers on one line, `value sep value sep ...`; comment-stripped first.
template <class T, class Conv>
std::vector<T> line_values(const std::string &line, Conv conv, bool allow_point) {
  std::string s = line.substr(0, line.find(';'));
  std::vector<T> out;
  const char *p = s.c_str();
  for (;;) {
    while (is_space(*p)) ++p;
    if (!*p) break;
    bool start = (*p >= '0' && *p <= '9') || *p == '-' || *p == '+' || (allow_point && *p == '.');
    if (!start) break;
    char *end = nullptr;
    T v = conv(p, &end);
    if (end == p) break;
    p = end;
    while (is_space(*p)) ++p;
    if (!*p) break;  // no separator: the reference drops this value
    ++p;             // one separator character, whatever it is
    out.push_back(v);
  }
  return out;
}

std::vector<std::string> section_lines(const std::string &c, size_t key_pos, const std::vector<size_t> &sorted) {
  size_t eq = c.find('=', key_pos);
  size_t xstart = eq == std::string::npos ? 0 : eq - key_pos;
  size_t length;
  auto it = std::find(sorted.begin(), sorted.end(), key_pos);
  if (it + 1 == sorted.end()) length = c.size() - xstart - 2;
  else length = *(it + 1) - key_pos;
  size_t b = std::min(key_pos + xstart + 1, c.size());
  std::string sub = c.substr(b, length);
  std::vector<std::string> lines;
  size_t i = 0;
  while (i <= sub.size()) {
    size_t j = sub.find('\n', i);
    if (j == std::string::npos) j = sub.size();
    lines.push_back(sub.substr(i, j - i));
    i = j + 1;
  }
  return lines;
}

double to_double(const char *p, char **e) { return std::strtod(p, e); }
long to_long(const char *p, char **e) { return std::strtol(p, e, 10); }

}  // namespace

bool parse_deck(const std::string &text, Deck &deck, std::string &err) {
  deck = Deck();
  const char *keys[6] = {"xgrid", "ygrid", "zgrid", "mobs", "walls", "holes"};
  std::vector<size_t> pos(6);
  for (int i = 0; i < 6; ++i) {
    pos[i] = text.find(keys[i]);
    if (pos[i] == std::string::npos) {
      err = std::string("deck: section '") + keys[i] + "' missing";
      return false;
    }
  }
  if (pos[0] != 0) { err = "deck: must start with 'xgrid' (the per-rank reader reads x from byte 0)"; return false; }
  if (!(pos[0] < pos[1] && pos[1] < pos[2] && pos[2] < pos[3])) {
    err = "deck: grid sections must appear in xgrid, ygrid, zgrid, mobs order";
    return false;
  }
  std::vector<size_t> sorted = pos;
  std::sort(sorted.begin(), sorted.end());
  std::vector<double> *axes[3] = {&deck.xs, &deck.ys, &deck.zs};
  for (int a = 0; a < 3; ++a)
    for (auto &ln : section_lines(text, pos[a], sorted)) {
      auto v = line_values<double>(ln, to_double, true);
      axes[a]->insert(axes[a]->end(), v.begin(), v.end());
    }
  for (auto &ln : section_lines(text, pos[3], sorted)) {
    auto v = line_values<long>(ln, to_long, false);
    if (v.empty()) continue;
    if (v.size() < 6) { err = "deck: mobs line with fewer than 6 values"; return false; }
    deck.mobs.push_back({(int)v[0], (int)v[1], (int)v[2], (int)v[3], (int)v[4], (int)v[5]});
  }
  for (auto &ln : section_lines(text, pos[4], sorted)) {
    auto v = line_values<long>(ln, to_long, false);
    if (v.size() != 8) continue;
    std::array<int, 8> w;
    for (int i = 0; i < 8; ++i) w[i] = (int)v[i];
    deck.walls.push_back(w);
  }
  for (auto &ln : section_lines(text, pos[5], sorted)) {
    auto v = line_values<long>(ln, to_long, false);
    if (v.size() != 13) continue;
    std::array<int, 13> h;
    for (int i = 0; i < 13; ++i) h[i] = (int)v[i];
    deck.holes.push_back(h);
  }
  if (deck.xs.size() < 3 || deck.ys.size() < 3 || deck.zs.size() < 3) {
    err = "deck: every axis needs at least 3 points";
    return false;
  }
  return true;
}

namespace {

void axis_geometry(const std::vector<double> &pts, long off, long n, std::vector<double> &p, std::vector<double> &m,
                   std::vector<double> &q) {
  // padded index i in [1, n] is global point index g = i + off - 2
  long np = (long)pts.size();
  p.assign(n + 2, 0.0); m.assign(n + 2, 0.0); q.assign(n + 2, 0.0);
  for (long i = 1; i <= n; ++i) {
    long g = i + off - 2;
    double xp = (g + 1) < np ? (pts[g + 1] - pts[g]) : (pts[g] - pts[g - 1]);
    double xw = (g - 1) >= 0 ? (pts[g] - pts[g - 1]) : xp;
    double xe = (g + 2) < np ? (pts[g + 2] - pts[g + 1]) : xp;
    p[i] = xp; m[i] = xw; q[i] = xe;
  }
}

}  // namespace

bool build_case(const Deck &deck, Case &c, std::string &err) {
  c.deck = deck;
  c.Nx = (long)deck.xs.size() - 1; c.Ny = (long)deck.ys.size() - 1; c.Nz = (long)deck.zs.size() - 1;
  const long Nx = c.Nx, Ny = c.Ny, Nz = c.Nz, N = Nx * Ny * Nz;
  auto cid = [&](long i, long j, long k) { return i + j * Nx + k * Nx * Ny; };
  auto fxid = [&](long i, long j, long k) { return i + j * (Nx + 1) + k * (Nx + 1) * Ny; };
  auto fyid = [&](long i, long j, long k) { return i + j * Nx + k * Nx * (Ny + 1); };
  auto fzid = [&](long i, long j, long k) { return i + j * Nx + k * Nx * Ny; };

  // cell type: first mobs box containing the cell (mesh/mesh.cpp:84-114)
  c.ctype.assign(N, 0);
  for (auto &b : deck.mobs) {
    long i0 = std::max<long>(b[0], 1), i1 = std::min<long>(b[1], Nx);
    long j0 = std::max<long>(b[2], 1), j1 = std::min<long>(b[3], Ny);
    long k0 = std::max<long>(b[4], 1), k1 = std::min<long>(b[5], Nz);
    for (long k = k0; k <= k1; ++k)
      for (long j = j0; j <= j1; ++j)
        for (long i = i0; i <= i1; ++i) c.ctype[cid(i - 1, j - 1, k - 1)] = 1;
  }
  // wall faces: domain boundary + internal wall patches (mesh/mesh.cpp:133-237)
  c.wx.assign((Nx + 1) * Ny * Nz, 0); c.wy.assign(Nx * (Ny + 1) * Nz, 0); c.wz.assign(Nx * Ny * (Nz + 1), 0);
  for (long k = 0; k < Nz; ++k)
    for (long j = 0; j < Ny; ++j) c.wx[fxid(0, j, k)] = c.wx[fxid(Nx, j, k)] = 1;
  for (long k = 0; k < Nz; ++k)
    for (long i = 0; i < Nx; ++i) c.wy[fyid(i, 0, k)] = c.wy[fyid(i, Ny, k)] = 1;
  for (long j = 0; j < Ny; ++j)
    for (long i = 0; i < Nx; ++i) c.wz[fzid(i, j, 0)] = c.wz[fzid(i, j, Nz)] = 1;
  for (auto &w : deck.walls) {
    int i0 = w[0], i1 = w[1], j0 = w[2], j1 = w[3], k0 = w[4], k1 = w[5];
    if (i0 == i1 && i0 >= 1 && i0 <= Nx + 1)
      for (long k = std::max(k0, 1); k <= std::min<long>(k1, Nz); ++k)
        for (long j = std::max(j0, 1); j <= std::min<long>(j1, Ny); ++j) c.wx[fxid(i0 - 1, j - 1, k - 1)] = 1;
    if (j0 == j1 && j0 >= 1 && j0 <= Ny + 1)
      for (long k = std::max(k0, 1); k <= std::min<long>(k1, Nz); ++k)
        for (long i = std::max(i0, 1); i <= std::min<long>(i1, Nx); ++i) c.wy[fyid(i - 1, j0 - 1, k - 1)] = 1;
    if (k0 == k1 && k0 >= 1 && k0 <= Nz + 1)
      for (long j = std::max(j0, 1); j <= std::min<long>(j1, Ny); ++j)
        for (long i = std::max(i0, 1); i <= std::min<long>(i1, Nx); ++i) c.wz[fzid(i - 1, j - 1, k0 - 1)] = 1;
  }
  // regions: same-type components through non-wall faces, numbered by their
  // lowest cell index (mesh/mesh.cpp:298-454)
  c.region.assign(N, -1);
  int nreg[2] = {0, 0};
  std::vector<long> queue;
  queue.reserve(N);
  for (long s = 0; s < N; ++s) {
    if (c.region[s] >= 0) continue;
    int t = c.ctype[s], id = nreg[t]++;
    queue.clear(); queue.push_back(s); c.region[s] = id;
    for (size_t h = 0; h < queue.size(); ++h) {
      long q = queue[h];
      long i = q % Nx, j = (q / Nx) % Ny, k = q / (Nx * Ny);
      auto visit = [&](bool ok, long n) {
        if (ok && c.region[n] < 0 && c.ctype[n] == t) { c.region[n] = id; queue.push_back(n); }
      };
      visit(i > 0 && !c.wx[fxid(i, j, k)], q - 1);
      visit(i < Nx - 1 && !c.wx[fxid(i + 1, j, k)], q + 1);
      visit(j > 0 && !c.wy[fyid(i, j, k)], q - Nx);
      visit(j < Ny - 1 && !c.wy[fyid(i, j + 1, k)], q + Nx);
      visit(k > 0 && !c.wz[fzid(i, j, k)], q - Nx * Ny);
      visit(k < Nz - 1 && !c.wz[fzid(i, j, k + 1)], q + Nx * Ny);
    }
  }
  c.nfluid_regions = nreg[0]; c.nsolid_regions = nreg[1];
  if (c.nfluid_regions != 1) {
    err = "exactly one connected fluid region is supported (found " + std::to_string(c.nfluid_regions) + ")";
    return false;
  }
  auto bbox = [&](int type, int reg, Meta &m) {
    long mn[3] = {1L << 40, 1L << 40, 1L << 40}, mx[3] = {-1, -1, -1};
    for (long k = 0; k < Nz; ++k)
      for (long j = 0; j < Ny; ++j)
        for (long i = 0; i < Nx; ++i) {
          long q = cid(i, j, k);
          if (c.ctype[q] != type || c.region[q] != reg) continue;
          long g[3] = {i + 1, j + 1, k + 1};
          for (int a = 0; a < 3; ++a) { mn[a] = std::min(mn[a], g[a]); mx[a] = std::max(mx[a], g[a]); }
        }
    m.cx = mx[0] - mn[0] + 1; m.cy = mx[1] - mn[1] + 1; m.cz = mx[2] - mn[2] + 1;
    m.fx = m.cx + 1; m.fy = m.cy + 1; m.fz = m.cz + 1;
    m.ox = mn[0]; m.oy = mn[1]; m.oz = mn[2];
  };
  // fluid box (distributed_mesh.h:117-168)
  Meta &F = c.fluid;
  bbox(0, 0, F);
  if (F.cx < 2 || F.cy < 2 || F.cz < 2) { err = "fluid box thinner than 2 cells"; return false; }
  c.fluid_empty.assign(F.ncell(), 1);
  c.row_id.assign(F.ncell(), -1);
  c.nfluid = 0;
  for (long k = 0; k < F.cz; ++k)
    for (long j = 0; j < F.cy; ++j)
      for (long i = 0; i < F.cx; ++i) {
        long g = cid(i + F.ox - 1, j + F.oy - 1, k + F.oz - 1);
        long l = i + j * F.cx + k * F.cx * F.cy;
        if (c.ctype[g] == 0 && c.region[g] == 0) { c.fluid_empty[l] = 0; c.row_id[l] = (int)c.nfluid++; }
      }
  axis_geometry(deck.xs, F.ox, F.cx, c.xp, c.xw, c.xe);
  axis_geometry(deck.ys, F.oy, F.cy, c.yp, c.ys, c.yn);
  axis_geometry(deck.zs, F.oz, F.cz, c.zp, c.zf, c.zb);
  // solid boxes (distributed_mesh.h:228-317)
  c.solids.assign(c.nsolid_regions, Meta());
  c.solid_empty.assign(c.nsolid_regions, {});
  for (int r = 0; r < c.nsolid_regions; ++r) {
    Meta &S = c.solids[r];
    bbox(1, r, S);
    c.solid_empty[r].assign(S.ncell(), 1);
    for (long k = 0; k < S.cz; ++k)
      for (long j = 0; j < S.cy; ++j)
        for (long i = 0; i < S.cx; ++i) {
          long g = cid(i + S.ox - 1, j + S.oy - 1, k + S.oz - 1);
          if (c.ctype[g] == 1 && c.region[g] == r) c.solid_empty[r][i + j * S.cx + k * S.cx * S.cy] = 0;
        }
  }
  // interface faces of the fluid box, x then y then z, each k-j-i
  // (fluid_solver.h:900-1229): non-wall faces between a fluid cell and an
  // obstacle cell
  c.ib_x.assign(F.fx * F.cy * F.cz, 0); c.ib_y.assign(F.cx * F.fy * F.cz, 0); c.ib_z.assign(F.cx * F.cy * F.fz, 0);
  c.swap.clear();
  auto fpad = [&](const long g[3]) { return (g[0] - F.ox + 2) + (g[1] - F.oy + 2) * (F.cx + 2) + (g[2] - F.oz + 2) * (F.cx + 2) * (F.cy + 2); };
  for (int dir = 0; dir < 3; ++dir) {
    long ni = dir == 0 ? F.fx : F.cx, nj = dir == 1 ? F.fy : F.cy, nk = dir == 2 ? F.fz : F.cz;
    long Nd = dir == 0 ? Nx : dir == 1 ? Ny : Nz;
    std::vector<uint8_t> &ib = dir == 0 ? c.ib_x : dir == 1 ? c.ib_y : c.ib_z;
    for (long k = 0; k < nk; ++k)
      for (long j = 0; j < nj; ++j)
        for (long i = 0; i < ni; ++i) {
          long gb[3] = {i + F.ox - 1, j + F.oy - 1, k + F.oz - 1};  // plus-side cell (0-based)
          long ga[3] = {gb[0], gb[1], gb[2]};
          ga[dir] -= 1;
          if (ga[dir] < 0 || gb[dir] >= Nd) continue;
          bool wall = dir == 0 ? c.wx[fxid(gb[0], gb[1], gb[2])] : dir == 1 ? c.wy[fyid(gb[0], gb[1], gb[2])] : c.wz[fzid(gb[0], gb[1], gb[2])];
          if (wall) continue;
          long qa = cid(ga[0], ga[1], ga[2]), qb = cid(gb[0], gb[1], gb[2]);
          bool fa = c.ctype[qa] == 0 && c.region[qa] == 0, fb = c.ctype[qb] == 0 && c.region[qb] == 0;
          const long *gf, *gs;
          int reg;
          if (fa && c.ctype[qb] == 1) { gf = ga; gs = gb; reg = c.region[qb]; }
          else if (fb && c.ctype[qa] == 1) { gf = gb; gs = ga; reg = c.region[qa]; }
          else continue;
          long nfi = dir == 0 ? F.fx : F.cx, nfj = dir == 1 ? F.fy : F.cy;
          ib[i + j * nfi + k * nfi * nfj] = 1;
          const Meta &S = c.solids[reg];
          auto spad = [&](const long g[3]) { return (g[0] - S.ox + 2) + (g[1] - S.oy + 2) * (S.cx + 2) + (g[2] - S.oz + 2) * (S.cx + 2) * (S.cy + 2); };
          c.swap.push_back({fpad(gf), fpad(gs), spad(gs), spad(gf), reg});
        }
  }
  return true;
}

}  // namespace hs
