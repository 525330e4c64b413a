// result.vtk in the layout main.cpp:109-156 writes (legacy ASCII structured
// grid: points, then pressure, velocity, temperature and id per point, in
// the order of the global cell index), with the grid's own dimensions where
// the reference prints a fixed "DIMENSIONS 50 50 50".
#pragma once
#include <fstream>
#include <iomanip>
#include <map>
#include <string>

#include "fluid_solver.h"

inline void write_result_vtk(const std::string &path, const std::map<I64, OutputData> &points, I64 nx, I64 ny,
                             I64 nz) {
  std::ofstream f(path);
  f << "# vtk DataFile Version 3.0\n";
  f << "MPI gathered data with scalar p\n";
  f << "ASCII\n";
  f << "DATASET STRUCTURED_GRID\n";
  f << "DIMENSIONS " << nx << " " << ny << " " << nz << "\n";
  f << "POINTS " << points.size() << " double\n";
  f << std::fixed << std::setprecision(12);
  for (auto &e : points) f << e.second.locationx << " " << e.second.locationy << " " << e.second.locationz << "\n";
  f << "POINT_DATA " << points.size() << "\n";
  f << "SCALARS pressure double 1\nLOOKUP_TABLE default\n";
  for (auto &e : points) f << e.second.p << "\n";
  f << "VECTORS velocity double\n";
  for (auto &e : points) f << e.second.ux << " " << e.second.uy << " " << e.second.uz << "\n";
  f << "SCALARS temperature double 1\nLOOKUP_TABLE default\n";
  for (auto &e : points) f << e.second.t << "\n";
  f << "SCALARS id int 1\nLOOKUP_TABLE default\n";
  for (auto &e : points) f << e.second.globalid << "\n";
}
