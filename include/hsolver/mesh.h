// Drop-in CYCASMesh for single-GPU drivers (replaces mesh/mesh.h's class of
// the same name, mesh/mesh.h:335).  The reference reads the deck and then
// per-rank processor files written by its decompose step; here the deck is
// the only input and the case model is built from it by the C ABI
// (hs_case_*), so readCells / readFaces / readBoundaries have nothing left to
// read and only check that the deck parsed.
#pragma once
#include <cstdint>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../hsolver_b200.h"

typedef int64_t I64;

class CYCASMesh {
 public:
  CYCASMesh(std::string filename, int iProc) : iProc_(iProc) {
    std::ifstream f(filename);
    if (!f) throw std::runtime_error("cannot open deck " + filename);
    std::stringstream ss;
    ss << f.rdbuf();
    deck = ss.str();
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
  void readCells(int) {}
  void readFaces(int) {}
  void readBoundaries(int) {}

  I64 Nx = 0, Ny = 0, Nz = 0;
  std::vector<double> xPoints, yPoints, zPoints;
  std::string deck;  // the .in text the GPU engine is built from

 private:
  int iProc_;
};
