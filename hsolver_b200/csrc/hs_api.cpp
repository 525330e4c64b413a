// extern "C" boundary of hsolver_b200 (declared in include/hsolver_b200.h).
// Every entry point catches C++ exceptions and maps them to an int status;
// the message is kept per context (and per thread for context-less errors).
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/hsolver_b200.h"
#include "hs_case.hpp"
#include "hs_channel.hpp"
#include "hs_cht.hpp"
#include "hs_engine.hpp"
#include "hs_slab.hpp"

struct hs_ctx {
  hs::Engine *engine = nullptr;
  std::string err;
};

struct hs_case {
  hs::Case c;
};

struct hs_pcg {
  hs::PcgWork *w = nullptr;
};

struct hs_channel {
  hs::ChannelState *st = nullptr;
  int nreg = 0;
  long long ncell = 0;
};

struct hs_cht {
  hs_ctx *ctx = nullptr;
  hs::ChtState *st = nullptr;
  double k_fluid = 1.0;
  std::string err;
};

namespace {
thread_local std::string g_err;

int fail(hs_ctx *ctx, int code, const std::string &msg) {
  g_err = msg;
  if (ctx) ctx->err = msg;
  return code;
}

int classify(const std::exception &e) {
  std::string m = e.what();
  if (m.rfind("CUDA alloc", 0) == 0) return HS_ERR_NOMEM;
  if (m.rfind("CUDA", 0) == 0) return HS_ERR_CUDA;
  if (dynamic_cast<const std::invalid_argument *>(&e)) return HS_ERR_ARG;
  if (dynamic_cast<const std::logic_error *>(&e)) return HS_ERR_STATE;
  return HS_ERR_INTERNAL;
}

template <class Fn>
int guarded(hs_ctx *ctx, Fn fn) {
  if (!ctx || !ctx->engine) return fail(ctx, HS_ERR_ARG, "null context");
  try {
    return fn(*ctx->engine);
  } catch (const std::bad_alloc &) {
    return fail(ctx, HS_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(ctx, classify(e), e.what());
  }
}
}  // namespace

namespace {
template <class Fn>
int ch_guarded(hs_channel *h, Fn fn) {
  if (!h || !h->st) return fail(nullptr, HS_ERR_ARG, "null channel handle");
  try {
    return fn(*h);
  } catch (const std::bad_alloc &) {
    return fail(nullptr, HS_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(nullptr, classify(e), e.what());
  }
}

void ch_copy_stats(const hs::ChStats &a, hs_channel_stats *b) {
  if (!b) return;
  for (int x = 0; x < 5; ++x) { b->res[x] = a.res[x]; b->norm[x] = a.norm[x]; }
  b->global = a.global; b->iter = a.iter; b->pcg_iters = a.pcg_iters; b->t_iters = a.t_iters;
  b->pcg_relres = a.pcg_relres; b->t_relres = a.t_relres;
}

bool ch_finite(const hs::ChStats &a) {
  for (int x = 0; x < 5; ++x)
    if (!(a.res[x] == a.res[x]) || a.res[x] > 1e300) return false;
  return true;
}
}  // namespace

extern "C" {

void hs_params_default(hs_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->nu = 0.001; p->rho = 1; p->alpha = 0.001; p->u_lid = 0.1;
  p->relax = 0.3; p->relax_solid = 0.3;
  p->mom_tol = 2e-3; p->energy_tol = 2e-3; p->solid_tol = 1e-3;
  p->gs_max = 100; p->t_fluid0 = 293; p->t_wall = 293; p->t_solid0 = 333;
  p->pcg_tol = 1e-5; p->pcg_maxiter = 1000; p->frozen_matrix = 1;
  p->pressure_solver = HS_PSOLVE_CG;
}

int hs_create(const char *deck, const hs_params *prm, int device, hs_ctx **out) {
  if (!deck || !out) return fail(nullptr, HS_ERR_ARG, "null deck or output pointer");
  *out = nullptr;
  hs_params p;
  if (prm) p = *prm; else hs_params_default(&p);
  if (p.gs_max < 0 || p.pcg_maxiter < 0 || !(p.pcg_tol >= 0)) return fail(nullptr, HS_ERR_ARG, "invalid parameters");
  if (p.pressure_solver != HS_PSOLVE_CG && p.pressure_solver != HS_PSOLVE_MGCG)
    return fail(nullptr, HS_ERR_ARG, "unknown pressure solver");
  std::string err;
  hs::Deck d;
  if (!hs::parse_deck(deck, d, err)) return fail(nullptr, HS_ERR_DECK, err);
  hs::Case c;
  if (!hs::build_case(d, c, err)) return fail(nullptr, err.rfind("deck", 0) == 0 ? HS_ERR_DECK : HS_ERR_UNSUPPORTED, err);
  hs_ctx *ctx = new (std::nothrow) hs_ctx();
  if (!ctx) return fail(nullptr, HS_ERR_NOMEM, "host allocation failed");
  try {
    ctx->engine = new hs::Engine(c, p, device);
  } catch (const std::exception &e) {
    int code = classify(e);
    std::string m = e.what();
    delete ctx;
    return fail(nullptr, code, m);
  }
  *out = ctx;
  return HS_OK;
}

int hs_init(hs_ctx *ctx) {
  return guarded(ctx, [](hs::Engine &e) { e.init(); return HS_OK; });
}

int hs_step(hs_ctx *ctx, int n, hs_stats *stats) {
  if (n < 0) return fail(ctx, HS_ERR_ARG, "negative step count");
  return guarded(ctx, [&](hs::Engine &e) {
    if (!e.inited()) throw std::logic_error("hs_step before hs_init");
    e.step(n);
    if (stats) {
      e.stats(stats);
      double r[5] = {stats->res_u, stats->res_v, stats->res_w, stats->res_t, stats->pcg_relres};
      for (double v : r)
        if (!(v == v) || v > 1e300 || v < -1e300) {
          ctx->err = g_err = "non-finite residual";
          return HS_ERR_DIVERGED;
        }
    }
    return HS_OK;
  });
}

int hs_sync(hs_ctx *ctx) {
  return guarded(ctx, [](hs::Engine &e) { e.sync(); return HS_OK; });
}

int hs_stream(hs_ctx *ctx, void **stream) {
  if (!stream) return fail(ctx, HS_ERR_ARG, "null output pointer");
  return guarded(ctx, [&](hs::Engine &e) { *stream = e.stream_handle(); return HS_OK; });
}

int hs_profile(hs_ctx *ctx, int on) {
  return guarded(ctx, [&](hs::Engine &e) { e.profile(on != 0); return HS_OK; });
}

int hs_profile_read(hs_ctx *ctx, double ms[HS_NPHASE], int *steps) {
  if (!ms) return fail(ctx, HS_ERR_ARG, "null buffer");
  return guarded(ctx, [&](hs::Engine &e) {
    int c = e.profile_read(ms, HS_NPHASE);
    if (steps) *steps = c;
    return HS_OK;
  });
}

int hs_counters(hs_ctx *ctx, long long out8[8]) {
  if (!out8) return fail(ctx, HS_ERR_ARG, "null buffer");
  return guarded(ctx, [&](hs::Engine &e) { e.counters(out8); return HS_OK; });
}

int hs_field_size(hs_ctx *ctx, int field, long long *n) {
  return guarded(ctx, [&](hs::Engine &e) {
    long m = e.field_size(field);
    if (m < 0 || !n) throw std::invalid_argument("unknown field id");
    *n = m;
    return HS_OK;
  });
}

int hs_get_field(hs_ctx *ctx, int field, double *host, long long n) {
  if (!host) return fail(ctx, HS_ERR_ARG, "null buffer");
  return guarded(ctx, [&](hs::Engine &e) { e.get_field(field, host, (long)n); return HS_OK; });
}

int hs_set_field(hs_ctx *ctx, int field, const double *host, long long n) {
  if (!host) return fail(ctx, HS_ERR_ARG, "null buffer");
  return guarded(ctx, [&](hs::Engine &e) { e.set_field(field, host, (long)n); return HS_OK; });
}

int hs_field_device_ptr(hs_ctx *ctx, int field, double **dptr, long long *n) {
  if (!dptr || !n) return fail(ctx, HS_ERR_ARG, "null output pointer");
  return guarded(ctx, [&](hs::Engine &e) {
    long m;
    double *p = e.field_device_ptr(field, &m);
    if (!p) throw std::invalid_argument("unknown field id");
    *dptr = p;
    *n = m;
    return HS_OK;
  });
}

int hs_fluid_meta(hs_ctx *ctx, long long out9[9]) {
  return guarded(ctx, [&](hs::Engine &e) {
    const hs::Meta &m = e.kase().fluid;
    long long v[9] = {m.cx, m.cy, m.cz, m.fx, m.fy, m.fz, m.ox, m.oy, m.oz};
    std::memcpy(out9, v, sizeof v);
    return HS_OK;
  });
}

int hs_grid_dims(hs_ctx *ctx, long long out3[3]) {
  return guarded(ctx, [&](hs::Engine &e) {
    out3[0] = e.kase().Nx; out3[1] = e.kase().Ny; out3[2] = e.kase().Nz;
    return HS_OK;
  });
}

int hs_num_solids(hs_ctx *ctx) {
  return guarded(ctx, [](hs::Engine &e) { return (int)e.kase().solids.size(); });
}

int hs_solid_meta(hs_ctx *ctx, int region, long long out9[9]) {
  return guarded(ctx, [&](hs::Engine &e) {
    if (region < 0 || region >= (int)e.kase().solids.size()) throw std::invalid_argument("solid region out of range");
    const hs::Meta &m = e.kase().solids[region];
    long long v[9] = {m.cx, m.cy, m.cz, m.fx, m.fy, m.fz, m.ox, m.oy, m.oz};
    std::memcpy(out9, v, sizeof v);
    return HS_OK;
  });
}

int hs_get_solid(hs_ctx *ctx, int region, int which, double *host, long long n) {
  if (!host) return fail(ctx, HS_ERR_ARG, "null buffer");
  return guarded(ctx, [&](hs::Engine &e) { e.get_solid(region, which, host, (long)n); return HS_OK; });
}

int hs_get_fluid_mask(hs_ctx *ctx, unsigned char *host, long long n) {
  if (!host) return fail(ctx, HS_ERR_ARG, "null buffer");
  return guarded(ctx, [&](hs::Engine &e) {
    const auto &m = e.kase().fluid_empty;
    if ((long long)m.size() != n) throw std::invalid_argument("mask size mismatch");
    std::memcpy(host, m.data(), m.size());
    return HS_OK;
  });
}

int hs_get_cell_types(hs_ctx *ctx, unsigned char *type, int *region, long long n) {
  if (!type || !region) return fail(ctx, HS_ERR_ARG, "null buffer");
  return guarded(ctx, [&](hs::Engine &e) {
    const auto &c = e.kase();
    if ((long long)c.ctype.size() != n) throw std::invalid_argument("cell-type size mismatch");
    std::memcpy(type, c.ctype.data(), c.ctype.size());
    std::memcpy(region, c.region.data(), c.region.size() * sizeof(int));
    return HS_OK;
  });
}

int hs_get_row_ids(hs_ctx *ctx, int *host, long long n) {
  if (!host) return fail(ctx, HS_ERR_ARG, "null buffer");
  return guarded(ctx, [&](hs::Engine &e) {
    const auto &r = e.kase().row_id;
    if ((long long)r.size() != n) throw std::invalid_argument("row-id size mismatch");
    std::memcpy(host, r.data(), r.size() * sizeof(int));
    return HS_OK;
  });
}

int hs_case_create(const char *deck, hs_case **out) {
  if (!deck || !out) return fail(nullptr, HS_ERR_ARG, "null deck or output pointer");
  *out = nullptr;
  try {
    std::string err;
    hs::Deck d;
    if (!hs::parse_deck(deck, d, err)) return fail(nullptr, HS_ERR_DECK, err);
    hs_case *c = new hs_case();
    if (!hs::build_case(d, c->c, err)) {
      delete c;
      return fail(nullptr, err.rfind("deck", 0) == 0 ? HS_ERR_DECK : HS_ERR_UNSUPPORTED, err);
    }
    *out = c;
    return HS_OK;
  } catch (const std::exception &e) {
    return fail(nullptr, HS_ERR_INTERNAL, e.what());
  }
}

int hs_case_dims(const hs_case *c, long long out3[3]) {
  if (!c || !out3) return fail(nullptr, HS_ERR_ARG, "null argument");
  out3[0] = c->c.Nx; out3[1] = c->c.Ny; out3[2] = c->c.Nz;
  return HS_OK;
}

static void meta9(const hs::Meta &m, long long *o) {
  long long v[9] = {m.cx, m.cy, m.cz, m.fx, m.fy, m.fz, m.ox, m.oy, m.oz};
  std::memcpy(o, v, sizeof v);
}

int hs_case_fluid_meta(const hs_case *c, long long out9[9]) {
  if (!c || !out9) return fail(nullptr, HS_ERR_ARG, "null argument");
  meta9(c->c.fluid, out9);
  return HS_OK;
}

int hs_case_num_solids(const hs_case *c) {
  if (!c) return fail(nullptr, HS_ERR_ARG, "null argument");
  return (int)c->c.solids.size();
}

int hs_case_solid_meta(const hs_case *c, int region, long long out9[9]) {
  if (!c || !out9 || region < 0 || region >= (int)c->c.solids.size()) return fail(nullptr, HS_ERR_ARG, "bad region");
  meta9(c->c.solids[region], out9);
  return HS_OK;
}

int hs_case_cell_types(const hs_case *c, unsigned char *type, int *region, long long n) {
  if (!c || !type || !region || n != (long long)c->c.ctype.size()) return fail(nullptr, HS_ERR_ARG, "bad buffer");
  std::memcpy(type, c->c.ctype.data(), c->c.ctype.size());
  std::memcpy(region, c->c.region.data(), c->c.region.size() * sizeof(int));
  return HS_OK;
}

int hs_case_fluid_mask(const hs_case *c, unsigned char *empty, long long n) {
  if (!c || !empty || n != (long long)c->c.fluid_empty.size()) return fail(nullptr, HS_ERR_ARG, "bad buffer");
  std::memcpy(empty, c->c.fluid_empty.data(), c->c.fluid_empty.size());
  return HS_OK;
}

long long hs_case_num_interface(const hs_case *c) { return c ? (long long)c->c.swap.size() : -1; }

int hs_case_interface(const hs_case *c, long long *out5, long long n) {
  if (!c || !out5 || n != (long long)c->c.swap.size()) return fail(nullptr, HS_ERR_ARG, "bad buffer");
  for (long long i = 0; i < n; ++i) {
    const hs::SwapPair &s = c->c.swap[i];
    out5[5 * i] = s.f_send; out5[5 * i + 1] = s.f_recv; out5[5 * i + 2] = s.s_send;
    out5[5 * i + 3] = s.s_recv; out5[5 * i + 4] = s.region;
  }
  return HS_OK;
}

int hs_case_geometry(const hs_case *c, int axis, double *out, long long n) {
  if (!c || !out || axis < 0 || axis > 2) return fail(nullptr, HS_ERR_ARG, "bad argument");
  const hs::Case &k = c->c;
  const std::vector<double> *a[3][3] = {{&k.xp, &k.xw, &k.xe}, {&k.yp, &k.ys, &k.yn}, {&k.zp, &k.zf, &k.zb}};
  long long m = (long long)a[axis][0]->size();
  if (n != 3 * m) return fail(nullptr, HS_ERR_ARG, "geometry size mismatch");
  for (int q = 0; q < 3; ++q) std::memcpy(out + q * m, a[axis][q]->data(), m * sizeof(double));
  return HS_OK;
}

int hs_case_points(const hs_case *c, int axis, double *out, long long n) {
  if (!c || !out || axis < 0 || axis > 2) return fail(nullptr, HS_ERR_ARG, "bad argument");
  const std::vector<double> &v = axis == 0 ? c->c.deck.xs : axis == 1 ? c->c.deck.ys : c->c.deck.zs;
  if (n != (long long)v.size()) return fail(nullptr, HS_ERR_ARG, "points size mismatch");
  std::memcpy(out, v.data(), v.size() * sizeof(double));
  return HS_OK;
}

void hs_case_destroy(hs_case *c) { delete c; }

int hs_pcg_create(int nx, int ny, int nz, int device, hs_pcg **out) {
  if (!out) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  *out = nullptr;
  try {
    hs_pcg *h = new hs_pcg();
    try {
      h->w = hs::pcg_create(nx, ny, nz, device);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return HS_OK;
  } catch (const std::bad_alloc &) {
    return fail(nullptr, HS_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(nullptr, classify(e), e.what());
  }
}

int hs_pcg_solve(hs_pcg *h, const double *acx, const double *acy, const double *acz, const double *b, double *x,
                 double tol, int maxiter, void *stream, int *iters, double *relres) {
  if (!h || !h->w) return fail(nullptr, HS_ERR_ARG, "null solver handle");
  try {
    hs::pcg_solve(h->w, acx, acy, acz, b, x, tol, maxiter, stream, iters, relres);
    return HS_OK;
  } catch (const std::exception &e) {
    return fail(nullptr, classify(e), e.what());
  }
}

int hs_pcg_solve_noalloc(int nx, int ny, int nz, const double *acx, const double *acy, const double *acz,
                         const double *b, double *x, double tol, int maxiter, void *stream, int *iters, double *relres) {
  try {
    hs::pcg_solve_noalloc(nx, ny, nz, acx, acy, acz, b, x, tol, maxiter, stream, iters, relres);
    return HS_OK;
  } catch (const std::exception &e) {
    return fail(nullptr, classify(e), e.what());
  }
}

void hs_pcg_destroy(hs_pcg *h) {
  if (!h) return;
  hs::pcg_destroy(h->w);
  delete h;
}

void hs_cht_params_default(hs_cht_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->k_fluid = 1.0;
  p->t_boundary = 293.0;
  p->tol = 1e-10;
  p->maxiter = 5000;
}

int hs_cht_create(hs_ctx *ctx, const hs_cht_params *prm, hs_cht **out) {
  if (!out) return fail(ctx, HS_ERR_ARG, "null output pointer");
  *out = nullptr;
  return guarded(ctx, [&](hs::Engine &e) {
    hs_cht_params p;
    if (prm) p = *prm; else hs_cht_params_default(&p);
    if (!(p.k_fluid > 0) || !(p.tol > 0) || p.maxiter < 1) throw std::invalid_argument("invalid CHT parameters");
    const hs::Case &c = e.kase();
    hs::ChtSetup S;
    S.device = e.device(); S.stream = e.stream_handle();
    S.Nx = (int)c.Nx; S.Ny = (int)c.Ny; S.Nz = (int)c.Nz; S.nreg = (int)c.solids.size();
    S.xs = c.deck.xs.data(); S.ys = c.deck.ys.data(); S.zs = c.deck.zs.data();
    S.ctype = c.ctype.data();
    std::vector<int> reg(c.region.size());
    for (size_t i = 0; i < reg.size(); ++i) reg[i] = c.ctype[i] ? c.region[i] : -1;
    S.region = reg.data();
    S.t_boundary = p.t_boundary; S.tol = p.tol; S.maxiter = p.maxiter; S.bc = 0; S.precond = 1;
    hs_cht *h = new hs_cht();
    h->ctx = ctx;
    h->k_fluid = p.k_fluid;
    try {
      h->st = hs::cht_create(S);
      std::vector<double> kr(S.nreg, p.k_fluid);
      hs::cht_set_solid(h->st, p.k_fluid, kr.data(), nullptr);
    } catch (...) {
      if (h->st) hs::cht_destroy(h->st);
      delete h;
      throw;
    }
    *out = h;
    return HS_OK;
  });
}

int hs_cht_set_solid(hs_cht *h, const double *k_region, const double *q_cell) {
  if (!h || !k_region) return fail(nullptr, HS_ERR_ARG, "null argument");
  return guarded(h->ctx, [&](hs::Engine &) {
    hs::cht_set_solid(h->st, h->k_fluid, k_region, q_cell);
    return HS_OK;
  });
}

int hs_cht_forward(hs_cht *h, double *T, double *J, int *iters, double *relres) {
  if (!h) return fail(nullptr, HS_ERR_ARG, "null handle");
  return guarded(h->ctx, [&](hs::Engine &e) {
    const hs::Case &c = e.kase();
    hs::ChtVelSrc V;
    V.Nx = (int)c.Nx; V.Ny = (int)c.Ny; V.Nz = (int)c.Nz;
    V.cx = (int)c.fluid.cx; V.cy = (int)c.fluid.cy; V.cz = (int)c.fluid.cz;
    V.fx = (int)c.fluid.fx; V.fy = (int)c.fluid.fy; V.fz = (int)c.fluid.fz;
    V.ox = (int)c.fluid.ox; V.oy = (int)c.fluid.oy; V.oz = (int)c.fluid.oz;
    long n;
    V.u = e.field_device_ptr(HS_F_U_STAR, &n); V.v = e.field_device_ptr(HS_F_V_STAR, &n);
    V.w = e.field_device_ptr(HS_F_W_STAR, &n);
    V.ctype = nullptr;
    hs::cht_set_velocities(h->st, V);
    hs::cht_forward(h->st, T, J, iters, relres);
    return HS_OK;
  });
}

int hs_cht_adjoint(hs_cht *h, double *dJdq, double *dJdk, int *iters, double *relres) {
  if (!h) return fail(nullptr, HS_ERR_ARG, "null handle");
  return guarded(h->ctx, [&](hs::Engine &) {
    hs::cht_adjoint(h->st, dJdq, dJdk, iters, relres);
    return HS_OK;
  });
}

int hs_cht_velocities(hs_cht *h, double *ug, double *vg, double *wg) {
  if (!h || !ug || !vg || !wg) return fail(nullptr, HS_ERR_ARG, "null argument");
  return guarded(h->ctx, [&](hs::Engine &) {
    hs::cht_get_velocities(h->st, ug, vg, wg);
    return HS_OK;
  });
}

void hs_cht_destroy(hs_cht *h) {
  if (!h) return;
  hs::cht_destroy(h->st);
  delete h;
}

void hs_channel_params_default(hs_channel_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->re = 100; p->pr = 0.71; p->u_in = 1.0; p->t_in = 0.0;
  p->alpha_u = 0.7; p->alpha_p = 0.3; p->alpha_t = 0.9;
  p->mom_sweeps = 2; p->p_tol = 1e-8; p->p_maxiter = 1000; p->t_tol = 1e-2; p->t_maxiter = 200;
  p->precision = HS_PREC_FP64; p->p_precond = 1;
  p->conv = HS_CONV_UPWIND; p->g_axis = 2; p->ri = 0.0;
}


int hs_channel_create(const char *deck, const hs_channel_params *prm, int device, hs_channel **out) {
  if (!deck || !out) return fail(nullptr, HS_ERR_ARG, "null deck or output pointer");
  *out = nullptr;
  hs_channel_params p;
  if (prm) p = *prm; else hs_channel_params_default(&p);
  std::string err;
  hs::Deck d;
  if (!hs::parse_deck(deck, d, err)) return fail(nullptr, HS_ERR_DECK, err);
  hs::Case c;
  if (!hs::build_case(d, c, err)) return fail(nullptr, err.rfind("deck", 0) == 0 ? HS_ERR_DECK : HS_ERR_UNSUPPORTED, err);
  hs::ChParams q;
  q.re = p.re; q.pr = p.pr; q.u_in = p.u_in; q.t_in = p.t_in;
  q.alpha_u = p.alpha_u; q.alpha_p = p.alpha_p; q.alpha_t = p.alpha_t;
  q.mom_sweeps = p.mom_sweeps; q.p_tol = p.p_tol; q.p_maxiter = p.p_maxiter; q.t_tol = p.t_tol; q.t_maxiter = p.t_maxiter;
  q.precision = p.precision; q.p_precond = p.p_precond; q.p_mg_sweeps = p.p_mg_sweeps; q.p_level0 = p.p_level0;
  q.conv = p.conv; q.g_axis = p.g_axis; q.ri = p.ri;
  hs_channel *h = new (std::nothrow) hs_channel();
  if (!h) return fail(nullptr, HS_ERR_NOMEM, "host allocation failed");
  try {
    h->st = hs::ch_create(c, q, device);
  } catch (const std::exception &e) {
    int code = classify(e);
    std::string m = e.what();
    delete h;
    return fail(nullptr, code, m);
  }
  h->nreg = hs::ch_nreg(h->st);
  h->ncell = (long long)c.Nx * c.Ny * c.Nz;
  *out = h;
  return HS_OK;
}

int hs_channel_num_blocks(hs_channel *h, int *n) {
  if (!n) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  return ch_guarded(h, [&](hs_channel &c) { *n = c.nreg; return HS_OK; });
}

int hs_channel_set_solid(hs_channel *h, const double *k_ratio, int n_blocks, const double *q_cell, long long n) {
  return ch_guarded(h, [&](hs_channel &c) {
    if (!k_ratio || !q_cell || n_blocks != c.nreg || n != c.ncell) throw std::invalid_argument("set_solid: sizes");
    hs::ch_set_solid(c.st, k_ratio, q_cell);
    return HS_OK;
  });
}

int hs_channel_init(hs_channel *h) {
  return ch_guarded(h, [&](hs_channel &c) { hs::ch_init(c.st); return HS_OK; });
}

int hs_channel_step(hs_channel *h, int n, int flags, hs_channel_stats *stats) {
  if (n < 0 || (flags & ~3)) return fail(nullptr, HS_ERR_ARG, "bad step count or flags");
  return ch_guarded(h, [&](hs_channel &c) {
    hs::ChStats st{};
    hs::ch_step(c.st, n, flags, &st);
    ch_copy_stats(st, stats);
    if (n > 0 && !ch_finite(st)) return fail(nullptr, HS_ERR_DIVERGED, "non-finite residual");
    return HS_OK;
  });
}

int hs_channel_solve_to(hs_channel *h, double tol, int max_outer, int *steps, hs_channel_stats *stats) {
  if (!(tol > 0) || max_outer < 0) return fail(nullptr, HS_ERR_ARG, "bad tolerance or step limit");
  return ch_guarded(h, [&](hs_channel &c) {
    hs::ChStats st{};
    const int s = hs::ch_solve_to(c.st, tol, max_outer, &st);
    if (steps) *steps = s;
    ch_copy_stats(st, stats);
    if (s > 0 && !ch_finite(st)) return fail(nullptr, HS_ERR_DIVERGED, "non-finite residual");
    if (!(st.iter > 5 && st.global <= tol)) return fail(nullptr, HS_ERR_MAXITER, "global residual above tolerance");
    return HS_OK;
  });
}

int hs_channel_field_size(hs_channel *h, int field, long long *n) {
  if (!n) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  return ch_guarded(h, [&](hs_channel &c) {
    const long v = hs::ch_field_size(c.st, field);
    if (v < 0) throw std::invalid_argument("unknown field");
    *n = v;
    return HS_OK;
  });
}

int hs_channel_get_field(hs_channel *h, int field, double *host, long long n) {
  if (!host) return fail(nullptr, HS_ERR_ARG, "null buffer");
  return ch_guarded(h, [&](hs_channel &c) { hs::ch_get_field(c.st, field, host, (long)n); return HS_OK; });
}

int hs_channel_set_field(hs_channel *h, int field, const double *host, long long n) {
  if (!host) return fail(nullptr, HS_ERR_ARG, "null buffer");
  return ch_guarded(h, [&](hs_channel &c) { hs::ch_set_field(c.st, field, host, (long)n); return HS_OK; });
}

int hs_channel_stream(hs_channel *h, void **stream) {
  if (!stream) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  return ch_guarded(h, [&](hs_channel &c) { *stream = hs::ch_stream(c.st); return HS_OK; });
}

int hs_channel_profile(hs_channel *h, int on) {
  return ch_guarded(h, [&](hs_channel &c) { hs::ch_profile(c.st, on != 0); return HS_OK; });
}

int hs_channel_profile_read(hs_channel *h, double ms[HS_CH_NPHASE], int *steps) {
  if (!ms) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  return ch_guarded(h, [&](hs_channel &c) {
    const int n = hs::ch_profile_read(c.st, ms);
    if (steps) *steps = n;
    return HS_OK;
  });
}

int hs_channel_sync(hs_channel *h) {
  return ch_guarded(h, [&](hs_channel &c) { hs::ch_sync(c.st); return HS_OK; });
}

int hs_channel_balance(hs_channel *h, double out[HS_CH_NBAL]) {
  if (!out) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  return ch_guarded(h, [&](hs_channel &c) {
    hs::ch_balance(c.st, out);
    return HS_OK;
  });
}

int hs_channel_device_bytes(hs_channel *h, long long *bytes) {
  if (!bytes) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  return ch_guarded(h, [&](hs_channel &c) { *bytes = hs::ch_device_bytes(c.st); return HS_OK; });
}

int hs_channel_adjoint(hs_channel *h, double tol, int maxiter, double *J, double *dJdq, long long n, double *dJdk,
                       int n_blocks, hs_adjoint_info *info) {
  if (!(tol > 0) || maxiter < 1) return fail(nullptr, HS_ERR_ARG, "bad tolerance or iteration limit");
  return ch_guarded(h, [&](hs_channel &c) {
    if ((dJdq && n != c.ncell) || (dJdk && n_blocks != c.nreg)) throw std::invalid_argument("adjoint: sizes");
    int fi = 0, ai = 0;
    double fm = 0, am = 0;
    hs::ch_adjoint(c.st, tol, maxiter, J, dJdq, dJdk, &fi, &ai, &fm, &am);
    if (info) { info->fwd_iters = fi; info->adj_iters = ai; info->fwd_ms = fm; info->adj_ms = am; }
    return HS_OK;
  });
}

void hs_channel_destroy(hs_channel *h) {
  if (!h) return;
  try {
    hs::ch_destroy(h->st);
  } catch (...) {
  }
  delete h;
}

long long hs_check_division(const double *a, const double *b, long long n) {
  try {
    return hs::div_check(a, b, n);
  } catch (const std::exception &e) {
    return fail(nullptr, classify(e), e.what());
  }
}

void hs_destroy(hs_ctx *ctx) {
  if (!ctx) return;
  delete ctx->engine;
  delete ctx;
}

const char *hs_last_error(const hs_ctx *ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

}  // extern "C"

// ---------------------------------------------------------------- z-slab p' solve
struct hs_slab {
  hs::SlabState *st = nullptr;
};

namespace {
template <class Fn>
int slab_guarded(hs_slab *h, Fn fn) {
  if (!h || !h->st) return fail(nullptr, HS_ERR_ARG, "null slab handle");
  try {
    return fn(h->st);
  } catch (const std::exception &e) {
    return fail(nullptr, classify(e), e.what());
  }
}
}  // namespace

int hs_slab_create(int nx, int ny, int nz, int device, hs_slab **out) {
  if (!out) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  *out = nullptr;
  hs_slab *h = new (std::nothrow) hs_slab();
  if (!h) return fail(nullptr, HS_ERR_NOMEM, "host allocation failed");
  try {
    h->st = hs::slab_create(nx, ny, nz, device);
  } catch (const std::exception &e) {
    delete h;
    return fail(nullptr, classify(e), e.what());
  }
  *out = h;
  return HS_OK;
}

int hs_slab_set_system(hs_slab *h, const double *gx, const double *gy, const double *gz, const double *b) {
  if (!gx || !gy || !gz || !b) return fail(nullptr, HS_ERR_ARG, "null array");
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_set_system(s, gx, gy, gz, b); return HS_OK; });
}

int hs_slab_begin(hs_slab *h, double *bb) {
  return slab_guarded(h, [&](hs::SlabState *s) { const double v = hs::slab_begin(s); if (bb) *bb = v; return HS_OK; });
}

int hs_slab_precond(hs_slab *h, double *rz) {
  return slab_guarded(h, [&](hs::SlabState *s) { const double v = hs::slab_precond(s); if (rz) *rz = v; return HS_OK; });
}

int hs_slab_direction(hs_slab *h, double beta, int first) {
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_direction(s, beta, first); return HS_OK; });
}

int hs_slab_apply(hs_slab *h, double *sp) {
  return slab_guarded(h, [&](hs::SlabState *s) { const double v = hs::slab_apply(s); if (sp) *sp = v; return HS_OK; });
}

int hs_slab_update(hs_slab *h, double alpha, double *rr) {
  return slab_guarded(h, [&](hs::SlabState *s) { const double v = hs::slab_update(s, alpha); if (rr) *rr = v; return HS_OK; });
}

int hs_slab_plane_size(hs_slab *h, long long *n) {
  if (!n) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  return slab_guarded(h, [&](hs::SlabState *s) { *n = hs::slab_plane_size(s); return HS_OK; });
}

int hs_slab_halo_get(hs_slab *h, double *lo, double *hi) {
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_halo_get(s, lo, hi); return HS_OK; });
}

int hs_slab_halo_put(hs_slab *h, const double *lo, const double *hi) {
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_halo_put(s, lo, hi); return HS_OK; });
}

int hs_slab_get(hs_slab *h, int which, double *host) {
  if (!host || which < 0 || which > 3) return fail(nullptr, HS_ERR_ARG, "bad field or null output");
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_get(s, which, host); return HS_OK; });
}

int hs_slab_set_coarse(hs_slab *h, int agg, int kg0, int nzg) {
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_set_coarse(s, agg, kg0, nzg); return HS_OK; });
}

int hs_slab_coarse_sizes(hs_slab *h, long long *n4) {
  if (!n4) return fail(nullptr, HS_ERR_ARG, "null output pointer");
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_coarse_sizes(s, n4); return HS_OK; });
}

int hs_slab_coarse_partial(hs_slab *h, double *cgx, double *cgy, double *cgz) {
  if (!cgx || !cgy || !cgz) return fail(nullptr, HS_ERR_ARG, "null array");
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_coarse_partial(s, cgx, cgy, cgz); return HS_OK; });
}

int hs_slab_coarse_build(hs_slab *h, const double *cgx, const double *cgy, const double *cgz) {
  if (!cgx || !cgy || !cgz) return fail(nullptr, HS_ERR_ARG, "null array");
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_coarse_build(s, cgx, cgy, cgz); return HS_OK; });
}

int hs_slab_restrict(hs_slab *h, double *rc) {
  if (!rc) return fail(nullptr, HS_ERR_ARG, "null array");
  return slab_guarded(h, [&](hs::SlabState *s) { hs::slab_restrict(s, rc); return HS_OK; });
}

int hs_slab_coarse_correct(hs_slab *h, const double *rc, double *rz) {
  if (!rc) return fail(nullptr, HS_ERR_ARG, "null array");
  return slab_guarded(h, [&](hs::SlabState *s) { const double v = hs::slab_coarse_correct(s, rc); if (rz) *rz = v; return HS_OK; });
}

void hs_slab_destroy(hs_slab *h) {
  if (!h) return;
  hs::slab_destroy(h->st);
  delete h;
}
