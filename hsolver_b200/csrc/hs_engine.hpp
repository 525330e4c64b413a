// Single-GPU engine for the SIMPLE conjugate-heat-transfer step: owns the
// case, all device state and the stream; runs FluidSolver::init/solve/
// setForNext, MobSolver::init/solve/setForNext and the interface swap as
// sm_100a kernels.
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/hsolver_b200.h"
#include "hs_case.hpp"

namespace hs {

struct DeviceState;  // defined in hs_engine.cu

class Engine {
 public:
  Engine(const Case &c, const hs_params &p, int device);
  ~Engine();
  Engine(const Engine &) = delete;
  Engine &operator=(const Engine &) = delete;

  void init();
  void step(int n);
  void sync();
  void stats(hs_stats *out);
  void profile(bool on);
  int profile_read(double *ms, int nphase);
  void counters(long long *out8);
  void *stream_handle();

  long field_size(int f) const;
  void get_field(int f, double *host, long n);
  void set_field(int f, const double *host, long n);
  double *field_device_ptr(int f, long *n);
  void get_solid(int r, int which, double *host, long n);

  const Case &kase() const { return case_; }
  int device() const { return device_; }
  bool inited() const { return inited_; }

 private:
  void build_multigrid();
  Case case_;
  hs_params prm_;
  int device_;
  bool inited_ = false;
  long long steps_ = 0;
  std::unique_ptr<DeviceState> d_;
};

// Standalone pressure-correction CG with its own device workspace.
struct PcgWork;
PcgWork *pcg_create(int nx, int ny, int nz, int device);
void pcg_destroy(PcgWork *w);
void pcg_solve(PcgWork *w, const double *acx, const double *acy, const double *acz, const double *b, double *x,
               double tol, int maxiter, void *stream, int *iters, double *relres);

// Same solve with no allocation: scratch in a static device array.
long long noalloc_max_padded_cells();
void pcg_solve_noalloc(int nx, int ny, int nz, const double *acx, const double *acy, const double *acz, const double *b,
                       double *x, double tol, int maxiter, void *stream, int *iters, double *relres);

// Number of (a, b) pairs where the precomputed-reciprocal division used by the
// sweeps differs from IEEE a/b (validation helper).
long long div_check(const double *a, const double *b, long long n);

}  // namespace hs
