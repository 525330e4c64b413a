// Drop-in CYCASMesh for single-GPU drivers (replaces mesh/mesh.h's class of
// the same name, mesh/mesh.h:335).  The deck is the input the GPU case model
// is built from (hs_case_*).  readCells / readFaces / readBoundaries read the
// per-rank processor files the reference's decompose step writes
// (processor<iProc>/{cells,faces,boundary}.txt, mesh/mesh.cpp:2277-2366) into
// the reference's public members, as mesh/mesh.cpp:2507-2642 does; a missing
// file leaves its members empty (the deck alone is enough here), and
// DistributedMesh::generateLocalDomain checks the cells read against the
// deck's case model.  A file named like the deck plus ".channel", when
// present, selects the channel physics for Solver::solve (channel_case.h).
#pragma once
#include <cstdint>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../hsolver_b200.h"

typedef int64_t I64;

// a face of a region as the processor files list it (mesh/mesh.h:47-54)
struct StFace {
  I64 owner = 0;      // cell on the face's low side
  I64 neighbour = 0;  // cell on its high side, -1 when none
  I64 globalId = 0;   // global face id, from 0
};

// a named run of a region's boundary faces (mesh/mesh.h:89-97)
struct BoundaryFaces {
  std::string name;
  int nFaces = 0;
  int startFace = 0;
};

class CYCASMesh {
 public:
  CYCASMesh(std::string filename, int iProc) : iProc_(iProc) {
    std::ifstream f(filename);
    if (!f) throw std::runtime_error("cannot open deck " + filename);
    std::stringstream ss;
    ss << f.rdbuf();
    deck = ss.str();
    std::ifstream side(filename + ".channel");
    if (side) {
      std::stringstream cs;
      cs << side.rdbuf();
      channel = cs.str();
    }
    hs_case *c = nullptr;
    if (hs_case_create(deck.c_str(), &c) != HS_OK) throw std::runtime_error(hs_last_error(nullptr));
    long long d[3];
    hs_case_dims(c, d);
    Nx = d[0]; Ny = d[1]; Nz = d[2];
    std::vector<double> *pts[3] = {&xPoints, &yPoints, &zPoints};
    for (int a = 0; a < 3; ++a) {
      pts[a]->resize(d[a] + 1);
      hs_case_points(c, a, pts[a]->data(), d[a] + 1);
    }
    hs_case_destroy(c);
  }

  // processor<iProc>/cells.txt: "meta <fluid|mobs> <n> <region> <group>"
  // followed by a line of n global cell indices
  void readCells(int iProc) {
    std::ifstream file(proc_file(iProc, "cells.txt"));
    if (!file) return;
    std::string line;
    while (std::getline(file, line)) {
      if (line.compare(0, 4, "meta") != 0) continue;
      std::string type;
      int n = 0, region = 0;
      meta(line, type, n, region);
      std::string cells;
      std::getline(file, cells);
      std::istringstream is(cells);
      std::vector<I64> v((size_t)n);
      for (int q = 0; q < n; ++q)
        if (!(is >> v[q])) throw std::runtime_error("processor cells file: short cell list");
      (type == "fluid" ? fluidRegions : mobsRegions)[region] = v;
    }
  }

  // processor<iProc>/faces.txt: a meta line, then n lines "globalId owner neighbour"
  void readFaces(int iProc) {
    std::ifstream file(proc_file(iProc, "faces.txt"));
    if (!file) return;
    std::string line;
    while (std::getline(file, line)) {
      if (line.compare(0, 4, "meta") != 0) continue;
      std::string type;
      int n = 0, region = 0;
      meta(line, type, n, region);
      std::vector<StFace> v((size_t)n);
      for (int q = 0; q < n; ++q) {
        if (!std::getline(file, line)) throw std::runtime_error("processor faces file: short face list");
        std::istringstream is(line);
        is >> v[q].globalId >> v[q].owner >> v[q].neighbour;
      }
      (type == "fluid" ? fluidFaces : mobsFaces)[region] = v;
    }
  }

  // processor<iProc>/boundary.txt: a meta line, then n lines "name startFace nFaces"
  void readBoundaries(int iProc) {
    std::ifstream file(proc_file(iProc, "boundary.txt"));
    if (!file) return;
    std::string line;
    while (std::getline(file, line)) {
      if (line.compare(0, 4, "meta") != 0) continue;
      std::string type;
      int n = 0, region = 0;
      meta(line, type, n, region);
      auto &m = (type == "fluid" ? fluidBoundaries : mobsBoundaries)[region];
      for (int q = 0; q < n; ++q) {
        if (!std::getline(file, line)) throw std::runtime_error("processor boundary file: short list");
        std::istringstream is(line);
        BoundaryFaces b;
        is >> b.name >> b.startFace >> b.nFaces;
        m[b.name] = b;
      }
    }
  }

  I64 Nx = 0, Ny = 0, Nz = 0;
  std::vector<double> xPoints, yPoints, zPoints;
  std::string deck;     // the .in text the GPU engine is built from
  std::string channel;  // the ".channel" sidecar's text, empty without one
  // what the processor files hold (empty when they were not read)
  std::map<int, std::vector<I64>> fluidRegions, mobsRegions;
  std::map<int, std::vector<StFace>> fluidFaces, mobsFaces;
  std::map<int, std::map<std::string, BoundaryFaces>> fluidBoundaries, mobsBoundaries;

 private:
  static std::string proc_file(int iProc, const char *name) {
    return "processor" + std::to_string(iProc) + "/" + name;
  }
  static void meta(const std::string &line, std::string &type, int &n, int &region) {
    std::istringstream is(line);
    std::string tag;
    int group = 0;
    if (!(is >> tag >> type >> n >> region >> group) || (type != "fluid" && type != "mobs") || n < 0)
      throw std::runtime_error("processor file: bad meta line '" + line + "'");
  }
  int iProc_;
};
