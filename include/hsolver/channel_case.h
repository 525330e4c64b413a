// Optional channel-physics sidecar of a deck for the drop-in classes.  The
// reference's drivers run its lid-driven cavity; a file named like the deck
// plus ".channel" (example.in -> example.in.channel) next to it makes
// Solver::solve run the channel conjugate-heat-transfer case of the C ABI
// (hs_channel_*: inlet plug flow, zero-gradient outlet, the deck's mobs boxes
// as heated blocks with a conductivity ratio) on the same deck, with the
// results in the same result / idArray / result.vtk form.  Format: one
// `key = value` per line, `#` starts a comment, lists separated by commas:
//   physics   = channel                 (required)
//   re, pr, u_in, t_in                  Reynolds number on the channel height, Prandtl number, inlet values
//   alpha_u, alpha_p, alpha_t           relaxation
//   mom_sweeps, p_tol, p_maxiter, t_tol, t_maxiter, p_mg_sweeps   inner solvers
//   precision = fp64 | mixed
//   convection = upwind | hybrid | quick  momentum convection (upwind: the reference's)
//   richardson = Ri, gravity_axis = x | y | z   Boussinesq buoyancy along + that axis
//   k_ratio   = k1, k2, ...             k_solid / k_fluid per block (one value: every block)
//   q         = q1, q2, ...             volumetric heat source per block (one value: every block)
//   tol       = 1e-6                    optional: outer steps until the global residual <= tol
//   max_outer = 5000                    the step limit with tol (default: Solver::steps)
// Unset keys keep hs_channel_params_default.
#pragma once
#include <cstdlib>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../hsolver_b200.h"

struct ChannelSpec {
  hs_channel_params prm;
  std::vector<double> k_ratio, q;
  double tol = 0.0;
  int max_outer = 0;
};

inline ChannelSpec parse_channel_spec(const std::string &text) {
  ChannelSpec s;
  hs_channel_params_default(&s.prm);
  bool channel = false;
  std::istringstream in(text);
  std::string line;
  int ln = 0;
  auto trim = [](std::string v) {
    const size_t a = v.find_first_not_of(" \t\r"), b = v.find_last_not_of(" \t\r");
    return a == std::string::npos ? std::string() : v.substr(a, b - a + 1);
  };
  while (std::getline(in, line)) {
    ++ln;
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    line = trim(line);
    if (line.empty()) continue;
    const size_t eq = line.find('=');
    if (eq == std::string::npos) throw std::runtime_error("channel sidecar line " + std::to_string(ln) + ": no '='");
    const std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
    auto num = [&](const std::string &v) {
      char *end = nullptr;
      const double d = std::strtod(v.c_str(), &end);
      if (v.empty() || trim(end) != "") throw std::runtime_error("channel sidecar line " + std::to_string(ln) + ": bad number");
      return d;
    };
    auto list = [&]() {
      std::vector<double> out;
      std::istringstream ls(val);
      std::string item;
      while (std::getline(ls, item, ',')) {
        item = trim(item);
        if (!item.empty()) out.push_back(num(item));
      }
      return out;
    };
    if (key == "physics") {
      if (val != "channel") throw std::runtime_error("channel sidecar: physics must be 'channel'");
      channel = true;
    } else if (key == "re") s.prm.re = num(val);
    else if (key == "pr") s.prm.pr = num(val);
    else if (key == "u_in") s.prm.u_in = num(val);
    else if (key == "t_in") s.prm.t_in = num(val);
    else if (key == "alpha_u") s.prm.alpha_u = num(val);
    else if (key == "alpha_p") s.prm.alpha_p = num(val);
    else if (key == "alpha_t") s.prm.alpha_t = num(val);
    else if (key == "mom_sweeps") s.prm.mom_sweeps = (int)num(val);
    else if (key == "p_tol") s.prm.p_tol = num(val);
    else if (key == "p_maxiter") s.prm.p_maxiter = (int)num(val);
    else if (key == "t_tol") s.prm.t_tol = num(val);
    else if (key == "t_maxiter") s.prm.t_maxiter = (int)num(val);
    else if (key == "p_mg_sweeps") s.prm.p_mg_sweeps = (int)num(val);
    else if (key == "precision") {
      if (val == "fp64") s.prm.precision = HS_PREC_FP64;
      else if (val == "mixed") s.prm.precision = HS_PREC_MIXED;
      else throw std::runtime_error("channel sidecar: precision must be fp64 or mixed");
    } else if (key == "convection") {
      if (val == "upwind") s.prm.conv = HS_CONV_UPWIND;
      else if (val == "hybrid") s.prm.conv = HS_CONV_HYBRID;
      else if (val == "quick") s.prm.conv = HS_CONV_QUICK;
      else throw std::runtime_error("channel sidecar: convection must be upwind, hybrid or quick");
    } else if (key == "richardson") s.prm.ri = num(val);
    else if (key == "gravity_axis") {
      if (val == "x") s.prm.g_axis = 0;
      else if (val == "y") s.prm.g_axis = 1;
      else if (val == "z") s.prm.g_axis = 2;
      else throw std::runtime_error("channel sidecar: gravity_axis must be x, y or z");
    } else if (key == "k_ratio") s.k_ratio = list();
    else if (key == "q") s.q = list();
    else if (key == "tol") s.tol = num(val);
    else if (key == "max_outer") s.max_outer = (int)num(val);
    else throw std::runtime_error("channel sidecar: unknown key '" + key + "'");
  }
  if (!channel) throw std::runtime_error("channel sidecar: 'physics = channel' missing");
  return s;
}
