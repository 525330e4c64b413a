/*
 * hsolver_b200.h -- C ABI of the B200-native SIMPLE conjugate-heat-transfer
 * step (one process, one GPU, the whole mesh resident in HBM).
 *
 * The reference (bolyme/hsolver) exposes this path as C++ classes driven by
 * main.cpp; there is no FFI.  Each entry point below replaces the reference
 * call named beside it, with plain pointers and sizes and an int status
 * (0 = HS_OK, negative = error; hs_last_error() gives the text).  No C++
 * exception crosses this boundary.  Calls on one context are serialised by
 * the caller; several contexts may share a GPU.
 */
#ifndef HSOLVER_B200_H
#define HSOLVER_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define HS_OK 0
#define HS_ERR_ARG (-1)         /* bad argument or size */
#define HS_ERR_DECK (-2)        /* deck parse / classification error */
#define HS_ERR_UNSUPPORTED (-3) /* case outside what the path supports */
#define HS_ERR_CUDA (-4)        /* CUDA runtime error */
#define HS_ERR_NOMEM (-5)       /* device allocation failed */
#define HS_ERR_STATE (-6)       /* call out of order */
#define HS_ERR_DIVERGED (-7)    /* non-finite residual */
#define HS_ERR_INTERNAL (-8)    /* a bounded device wait gave up */
#define HS_ERR_MAXITER (-9)     /* iteration limit reached before the tolerance */

/* Pressure-correction solver choice. */
#define HS_PSOLVE_CG 0   /* HYPRE PCG restated: identity preconditioner (fluid_solver.h:1871-1875) */
#define HS_PSOLVE_MGCG 1 /* CG preconditioned by the structured-grid multigrid V-cycle */

/* Field ids (the FluidSolver members of fluid_solver.h:60-67, 93-108). */
enum hs_field {
  HS_F_U_STAR = 0, /* u*  padded (fx+2)(cy+2)(cz+2) */
  HS_F_V_STAR = 1, /* v*  padded (cx+2)(fy+2)(cz+2) */
  HS_F_W_STAR = 2, /* w*  padded (cx+2)(cy+2)(fz+2) */
  HS_F_P_TEMP = 3, /* p   padded (cx+2)(cy+2)(cz+2) */
  HS_F_T_TEMP = 4, /* T   padded (cx+2)(cy+2)(cz+2) */
  HS_F_UP = 5,     /* a_P of the u faces, padded like u* */
  HS_F_VP = 6,
  HS_F_WP = 7,
  HS_F_UX = 8,     /* LocalFace u of x faces, fx*cy*cz */
  HS_F_UY = 9,     /* cx*fy*cz */
  HS_F_UZ = 10,    /* cx*cy*fz */
  HS_F_P = 11,     /* LocalCell p, cx*cy*cz */
  HS_F_T = 12,     /* LocalCell t, cx*cy*cz */
  HS_F_P_PRIME = 13 /* p' padded (zero between steps, fluid_solver.h:1598) */
};

/* Runtime form of the reference's compile-time macros
 * (fluid_solver.h:21-37, mobs_solver.h:15-29). */
typedef struct hs_params {
  double nu;          /* NU 0.001 */
  double rho;         /* RHO 1 */
  double alpha;       /* ALPHA 0.001 */
  double u_lid;       /* U0 0.1 */
  double relax;       /* UNDER_RELAX 0.3 (fluid) */
  double relax_solid; /* UNDER_RELAX 0.3 (solid) */
  double mom_tol;     /* CONVERGENCE 2e-3 */
  double energy_tol;  /* CONVERGENCE 2e-3 */
  double solid_tol;   /* CONVERGENCE2 1e-3 (mobs_solver.h) */
  int gs_max;         /* GS_STEP 100 */
  double t_fluid0;    /* 293 */
  double t_wall;      /* 293 */
  double t_solid0;    /* 333 */
  double pcg_tol;     /* 1e-5 */
  int pcg_maxiter;    /* 1000 */
  int frozen_matrix;  /* 1 = the reference's first-assembly matrix (fluid_solver.h:2188-2193) */
  int pressure_solver;/* HS_PSOLVE_* */
  int reserved[7];
} hs_params;

typedef struct hs_stats {
  int sweeps_u, sweeps_v, sweeps_w, sweeps_t, sweeps_solid_max, pcg_iters;
  double res_u, res_v, res_w, res_t, pcg_relres;
  long long steps;
} hs_stats;

typedef struct hs_ctx hs_ctx;

/* Defaults equal to the reference's macros. */
void hs_params_default(hs_params *p);

/* StructuredMesh(deck) + getConnectedRegions + decomposeMesh(nParts=1) +
 * CYCASMesh/DistributedMesh::generateLocalDomain + FluidSolver/MobSolver
 * constructors (mesh/mesh.cpp:42-58, 298-454; distributed_mesh.h:97-318;
 * fluid_solver.h:93-109; mobs_solver.h:50-56).  `deck` is the `.in` text.
 * Allocates all device state on `device`. */
int hs_create(const char *deck, const hs_params *prm, int device, hs_ctx **out);

/* FluidSolver::init + MobSolver::init (fluid_solver.h:882-1237,
 * mobs_solver.h:116-288). */
int hs_init(hs_ctx *ctx);

/* n passes of the Solver::solve loop body (solver.h:55-154): fluid solve,
 * solid solves, interface temperature swap, setForNext.  Asynchronous on the
 * context's stream unless `stats` is non-NULL (then it synchronises and
 * fills the last step's statistics). */
int hs_step(hs_ctx *ctx, int n, hs_stats *stats);

/* Wait for the context's stream. */
int hs_sync(hs_ctx *ctx);
/* The context's cudaStream_t (as void*), for callers that order their own
 * work after hs_step. */
int hs_stream(hs_ctx *ctx, void **stream);

/* Per-phase timing with CUDA events on the context's stream.  Phases:
 * 0-2 u/v/w momentum, 3 pressure-correction solve, 4 velocity/pressure
 * correction, 5 fluid energy, 6 solid energy, 7 swap + setForNext.
 * hs_profile_read returns the summed milliseconds per phase since the last
 * read and the number of steps they cover. */
#define HS_NPHASE 8
int hs_profile(hs_ctx *ctx, int on);
int hs_profile_read(hs_ctx *ctx, double ms[HS_NPHASE], int *steps);
/* Running counters since creation: sweeps of u, v, w, fluid T; solid
 * cell-sweeps; CG iterations; CG solves; outer steps. */
int hs_counters(hs_ctx *ctx, long long out8[8]);

/* Field access (host buffers; blocking). */
int hs_field_size(hs_ctx *ctx, int field, long long *n);
int hs_get_field(hs_ctx *ctx, int field, double *host, long long n);
int hs_set_field(hs_ctx *ctx, int field, const double *host, long long n);
/* Device address of a field (for callers that keep data in HBM). */
int hs_field_device_ptr(hs_ctx *ctx, int field, double **dptr, long long *n);

/* Case description: fluid metadata {cx,cy,cz,fx,fy,fz,ox,oy,oz}
 * (distributed_mesh.h:152-154), grid dims, solid regions. */
int hs_fluid_meta(hs_ctx *ctx, long long out9[9]);
int hs_grid_dims(hs_ctx *ctx, long long out3[3]);
int hs_num_solids(hs_ctx *ctx);
int hs_solid_meta(hs_ctx *ctx, int region, long long out9[9]);
/* which = 0: padded t_temp, 1: LocalCell t. */
int hs_get_solid(hs_ctx *ctx, int region, int which, double *host, long long n);
/* 1 where the fluid box cell is not fluid (LocalCell::isEmpty). */
int hs_get_fluid_mask(hs_ctx *ctx, unsigned char *host, long long n);
/* Global cell type (0 fluid, 1 obstacle) and region id, Nx*Ny*Nz. */
int hs_get_cell_types(hs_ctx *ctx, unsigned char *type, int *region, long long n);
/* HYPRE row id per fluid-box cell (-1 for empty), fluid_solver.h:1966. */
int hs_get_row_ids(hs_ctx *ctx, int *host, long long n);

/* Host-only case model (no GPU needed): the reference's decompose step for
 * one rank -- deck parse, cell types, connected regions, local boxes and the
 * fluid<->solid interface pairs (mesh/mesh.cpp:42-58, 84-454, 1124-1581;
 * distributed_mesh.h:97-318; fluid_solver.h:900-1229). */
typedef struct hs_case hs_case;
int hs_case_create(const char *deck, hs_case **out);
int hs_case_dims(const hs_case *c, long long out3[3]);
int hs_case_fluid_meta(const hs_case *c, long long out9[9]);
int hs_case_num_solids(const hs_case *c);
int hs_case_solid_meta(const hs_case *c, int region, long long out9[9]);
int hs_case_cell_types(const hs_case *c, unsigned char *type, int *region, long long n);
int hs_case_fluid_mask(const hs_case *c, unsigned char *empty, long long n);
/* Interface pairs as rows {fluid send, fluid recv, solid send, solid recv,
 * solid region}; padded indices into the fluid / solid t_temp arrays. */
long long hs_case_num_interface(const hs_case *c);
int hs_case_interface(const hs_case *c, long long *out5, long long n);
/* Per padded index geometry {xp,xw,xe | yp,ys,yn | zp,zf,zb} of the fluid
 * box (fluid_solver.h:1248-1261); axis 0..2, out3 = 3 arrays of n+2. */
int hs_case_geometry(const hs_case *c, int axis, double *out, long long n);
/* The deck's grid points of one axis (N+1 values; CYCASMesh::xPoints etc.). */
int hs_case_points(const hs_case *c, int axis, double *out, long long n);
void hs_case_destroy(hs_case *c);

/* Standalone pressure-correction solve, the counterpart of the reference's
 * HYPRE IJ/ParCSR PCG call (fluid_solver.h:1758-1799 with the settings of
 * fluid_solver.h:1871-1875): CG with the identity preconditioner, stopping
 * when <r,r>/<b,b> < tol^2 or after maxiter iterations, zero initial guess.
 * The system lives on a padded (nx+2)(ny+2)(nz+2) x-fastest grid; row P is
 *   (2cx+2cy+2cz) x_P - cz x_B - cy x_S - cx x_W - cx x_E - cy x_N - cz x_F
 * with cx, cy, cz = acx[P], acy[P], acz[P] (the coefficient construction of
 * fluid_solver.h:1990-1996).  Coefficients and b must be zero at every
 * padded index that is not an unknown; x is written everywhere (zero there).
 * All arrays are device pointers.  hs_pcg_create allocates the workspace
 * (four padded vectors and the reduction buffers). */
typedef struct hs_pcg hs_pcg;
int hs_pcg_create(int nx, int ny, int nz, int device, hs_pcg **out);
int hs_pcg_solve(hs_pcg *h, const double *acx, const double *acy, const double *acz, const double *b, double *x,
                 double tol, int maxiter, void *stream, int *iters, double *relres);
void hs_pcg_destroy(hs_pcg *h);

/* Allocation-free form of hs_pcg_solve; no counterpart in the reference.
 * For callers that cannot allocate device memory while they run -- hosts
 * whose GPU memory is all owned by their own arena, or loops that must not
 * call cudaMalloc/cudaFree after set-up because those calls can synchronise
 * the device -- it solves the same system with the same kernel on the
 * calling thread's current device, keeping its scratch in a static device
 * array of 8.06 MiB that every GPU loading the library holds until exit.
 * Limit: (nx+2)(ny+2)(nz+2) <= 262144 padded cells; larger grids return
 * HS_ERR_ARG.  The first call on a device looks up the array's device
 * address; make that first call before any stream capture.  The array
 * belongs to the library's device code, which the CUDA runtime loads on a
 * device when the library is first used there (lazy module loading): if no
 * other solve of this library has run on the device, that first call is
 * what loads it, so make one call (or any other solve of this library)
 * before the region that must not allocate.  The looked-up address is kept
 * for the life of the process: a cudaDeviceReset in between is not
 * supported.  Each call returns after its iteration count and residual have
 * reached the host.  All calls share the array, so calls that overlap on the
 * GPU race: serialise them.  It allocates nothing: no cudaMalloc, no
 * cudaFree. */
int hs_pcg_solve_noalloc(int nx, int ny, int nz, const double *acx, const double *acy, const double *acz,
                         const double *b, double *x, double tol, int maxiter, void *stream, int *iters, double *relres);

/* Conjugate-heat-transfer energy equation and its adjoint (no counterpart in
 * the reference, whose fluid and solid temperatures meet only through a
 * ghost-value swap, solver.h:62-148).  One operator over all cells of the
 * grid: harmonic-mean face conductance G = A/(dP/(2kP) + dN/(2kN)) (so a
 * fluid-solid face gets the series conductance of its two halves), upwind
 * convection with the face velocities of the owning solver at the time of
 * hs_cht_forward (faces touching a solid carry none), volumetric sources q in
 * solid cells, Dirichlet t_boundary on the domain boundary.  The objective is
 * J = (sum over solid cells of T^8 dV)^(1/8); hs_cht_adjoint solves the
 * transposed operator with the same BiCGStab and returns dJ/dq per cell
 * (zero in fluid) and dJ/dk per solid region. */
typedef struct hs_cht hs_cht;
typedef struct hs_cht_params {
  double k_fluid;     /* fluid conductivity (rho c = 1) */
  double t_boundary;  /* Dirichlet temperature on the domain boundary */
  double tol;         /* BiCGStab relative residual */
  int maxiter;
  int reserved[5];
} hs_cht_params;
void hs_cht_params_default(hs_cht_params *p);
int hs_cht_create(hs_ctx *ctx, const hs_cht_params *prm, hs_cht **out);
/* k per solid region (hs_num_solids values) and q per cell (Nx*Ny*Nz, host;
 * read in solid cells only, NULL = no source). */
int hs_cht_set_solid(hs_cht *h, const double *k_region, const double *q_cell);
/* Freeze the solver's current face velocities, solve; T (Nx*Ny*Nz host) and
 * J optional. */
int hs_cht_forward(hs_cht *h, double *T, double *J, int *iters, double *relres);
int hs_cht_adjoint(hs_cht *h, double *dJdq, double *dJdk, int *iters, double *relres);
/* The frozen face velocities ((Nx+1)NyNz, Nx(Ny+1)Nz, NxNy(Nz+1), host). */
int hs_cht_velocities(hs_cht *h, double *ug, double *vg, double *wg);
void hs_cht_destroy(hs_cht *h);

/* Channel conjugate heat transfer: the SIMPLE outer step with the physics the
 * reference lacks (its FluidSolver::solve, fluid_solver.h:1401-1633, drives a
 * lid cavity with no inlet, heat source or conductivity ratio).  Inlet plug
 * flow u_in at x = 0, zero-gradient outlet at x = Nx (p' = 0 there), no-slip
 * walls, the deck's mobs boxes as solid blocks with a conductivity ratio per
 * block and a volumetric source per cell, nu = u_in H / Re on the channel
 * height H, fluid conductivity nu / Pr.  Momentum keeps the reference's
 * first-order upwind coefficients (fluid_solver.h:577-659) with Patankar
 * relaxation alpha_u, solved by red-black Gauss-Seidel; the pressure
 * correction is SIMPLE's symmetric p' system, solved by CG preconditioned by
 * a geometric multigrid V-cycle; the energy equation is the conjugate-heat-
 * transfer operator of hs_cht_* over fluid and solid (inlet Dirichlet t_in,
 * adiabatic walls, upwind outflow), warm-started BiCGStab, relaxation alpha_t.
 * Global residual: the largest of the momentum (u, v, w), continuity and
 * energy residuals, each the L2 norm of its unrelaxed equation residual
 * divided by its largest value over the first five outer steps. */
#define HS_PREC_FP64 0
#define HS_PREC_MIXED 1   /* FP32 fields, sweeps and V-cycle; FP64 residuals, CG recurrences, dots, coarsest solve */
#define HS_CONV_UPWIND 0  /* a_nb = D + max(-+F, 0) (the reference's scheme) */
#define HS_CONV_HYBRID 1  /* a_nb = max(-+F, D -+ F/2, 0) (Spalding) */
#define HS_CONV_QUICK 2   /* upwind implicit, QUICK (Leonard) face values by deferred correction at u^n */
#define HS_CH_SKIP_PRESSURE 1
#define HS_CH_SKIP_ENERGY 2
typedef struct hs_channel hs_channel;
typedef struct hs_channel_params {
  double re, pr, u_in, t_in;
  double alpha_u, alpha_p, alpha_t;
  int mom_sweeps;      /* red-black sweeps per momentum solve */
  double p_tol;        /* pressure-correction CG: ||r|| / ||b|| */
  int p_maxiter;
  double t_tol;        /* energy BiCGStab per outer step: ||r|| / ||r0|| */
  int t_maxiter;
  int precision;       /* HS_PREC_* */
  int p_precond;       /* 0 plain CG, 1 multigrid V-cycle */
  int p_mg_sweeps;     /* red-black sweeps before and after the coarse
                          correction on the finest level of the p' V-cycle
                          (0: the default, 2); the coarser levels take one
                          more */
  int p_level0;        /* form of the finest level of the p' solve: 0 (the
                          default) the faster of the two on B200 (today the
                          grid-wide passes), 1 grid-wide passes (one per
                          colour), 2 z-marching passes with TMA-staged planes
                          (both colours of a red-black sweep in one pass)
                          wherever the grid has a coarser level below it */
  int conv;            /* momentum convection, HS_CONV_*: the reference's
                          first-order upwind (fluid_solver.h:441-447, 526-532,
                          609-615), hybrid, or QUICK by deferred correction */
  int g_axis;          /* Boussinesq buoyancy acts along + this axis (0..2) */
  double ri;           /* Richardson number Gr/Re^2: b += ri (T_f - t_in) V on
                          the faces of axis g_axis, T_f the mean T of the two
                          cells at the start of the step (0: no buoyancy) */
  double reserved[3];
} hs_channel_params;
typedef struct hs_channel_stats {
  double res[5];       /* u, v, w momentum, continuity, energy (absolute L2) */
  double norm[5];      /* normalisers: maximum over the first five outer steps */
  double global;       /* max_x res[x] / norm[x] */
  int iter;            /* outer steps since hs_channel_init */
  int pcg_iters, t_iters;
  double pcg_relres, t_relres;
} hs_channel_stats;
/* Channel fields for hs_channel_get_field / set_field (set: 0..4 only):
 * 0..2 u, v, w on faces ((Nx+1)NyNz, Nx(Ny+1)Nz, NxNy(Nz+1), x fastest),
 * 3 p, 4 T (Nx*Ny*Nz), 5..7 u*, v*, w*, 8..10 d = A alpha_u / a_P, 11 p'. */
void hs_channel_params_default(hs_channel_params *p);
int hs_channel_create(const char *deck, const hs_channel_params *prm, int device, hs_channel **out);
int hs_channel_num_blocks(hs_channel *h, int *n);
/* k_solid / k_fluid per block (n_blocks values, blocks numbered as the solid
 * regions of hs_get_cell_types), q per cell (Nx*Ny*Nz, read in solid cells). */
int hs_channel_set_solid(hs_channel *h, const double *k_ratio, int n_blocks, const double *q_cell, long long n);
int hs_channel_init(hs_channel *h);
/* n outer steps; flags HS_CH_SKIP_* leave out the pressure or energy solve. */
int hs_channel_step(hs_channel *h, int n, int flags, hs_channel_stats *stats);
/* Outer steps until the global residual <= tol (HS_OK) or max_outer steps
 * (HS_ERR_MAXITER); *steps = steps taken. */
int hs_channel_solve_to(hs_channel *h, double tol, int max_outer, int *steps, hs_channel_stats *stats);
int hs_channel_field_size(hs_channel *h, int field, long long *n);
int hs_channel_get_field(hs_channel *h, int field, double *host, long long n);
int hs_channel_set_field(hs_channel *h, int field, const double *host, long long n);
int hs_channel_stream(hs_channel *h, void **stream);
/* Per-phase CUDA-event times of the outer step (HS_CH_NPHASE: momentum, p'
 * assembly, p' solve, velocity/pressure correction, energy), summed over the
 * steps since profiling was switched on (which resets them). */
#define HS_CH_NPHASE 5
int hs_channel_profile(hs_channel *h, int on);
/* Global balances of the current state, summed in FP64 on the GPU (no
 * counterpart in the reference, whose only global sums are the per-sweep
 * residual allreduces, fluid_solver.h:485,571,654,878): out[0] volume flux
 * in through the inlet x = 0, out[1] out through the outlet x = Nx (mass
 * balance: equal at convergence), out[2] the heat source sum q V, out[3]
 * the heat leaving through the boundary faces (convection at inlet and
 * outlet relative to t_in, conduction through the inlet; heat balance: equal
 * to out[2] at convergence).  Blocking. */
#define HS_CH_NBAL 4
int hs_channel_balance(hs_channel *h, double out[HS_CH_NBAL]);
int hs_channel_profile_read(hs_channel *h, double ms[HS_CH_NPHASE], int *steps);
int hs_channel_sync(hs_channel *h);
/* Device memory the solver holds (bytes). */
int hs_channel_device_bytes(hs_channel *h, long long *bytes);
/* Energy adjoint on the current flow, frozen: a forward energy solve from
 * T = t_in to ||r|| / ||b|| < tol, then the adjoint.  J = (sum over solid
 * cells of T^8 dV)^(1/8); dJdq per cell (n = Nx*Ny*Nz), dJdk per block
 * (derivative with respect to the block's conductivity k_solid).  Both
 * timings are CUDA-event times on the solver's stream: fwd_ms the forward
 * solve with J, adj_ms from there until dJ/dT, the transposed solve and the
 * per-cell gradients are done on the device (the copies of dJdq and dJdk to
 * the host excluded, as the forward's T is not copied).  The outer loop's
 * temperature is left as it was. */
typedef struct hs_adjoint_info {
  int fwd_iters, adj_iters;
  double fwd_ms, adj_ms;
} hs_adjoint_info;
int hs_channel_adjoint(hs_channel *h, double tol, int maxiter, double *J, double *dJdq, long long n, double *dJdk,
                       int n_blocks, hs_adjoint_info *info);
void hs_channel_destroy(hs_channel *h);

/* One rank's z-slab of the channel pressure-correction system, for meshes
 * sharded over GPUs; the reference's counterpart is its domain decomposition
 * (Scotch parts, mesh/mesh.cpp:735-1122) with the HYPRE PCG over MPI ranks
 * (fluid_solver.h:1713-2194, setup 1840-1889).  The slab holds its nz
 * interior planes of an nx x ny grid and a ghost plane below and above.  The
 * host runs the CG recurrences: it all-reduces the local partial sums these
 * calls return (FP64) and, before each hs_slab_apply, moves the search
 * direction's first and last interior planes (hs_slab_halo_get) into the
 * neighbouring slabs' ghost planes (hs_slab_halo_put); the end slabs' outer
 * ghost planes stay zero.  Preconditioner: a multigrid V-cycle on the slab's
 * own rows (block Jacobi), symmetric positive definite.  hsolver_b200/slabs.py
 * drives it over NCCL or for several slabs of one process.  Every call is
 * synchronous. */
typedef struct hs_slab hs_slab;
int hs_slab_create(int nx, int ny, int nz, int device, hs_slab **out);
/* Host face couplings: gx ((nx+1) ny nz), gy (nx (ny+1) nz), gz (nx ny (nz+1):
 * faces 0 and nz are the slab's bottom and top faces), x fastest; b (nx ny nz). */
int hs_slab_set_system(hs_slab *h, const double *gx, const double *gy, const double *gz, const double *b);
int hs_slab_begin(hs_slab *h, double *bb);               /* x = 0, r = b; local <b, b> */
int hs_slab_precond(hs_slab *h, double *rz);             /* z = V-cycle(r); local <r, z> */
int hs_slab_direction(hs_slab *h, double beta, int first); /* p = z + beta p (first: p = z) */
int hs_slab_apply(hs_slab *h, double *sp);               /* s = A p; local <s, p> */
int hs_slab_update(hs_slab *h, double alpha, double *rr); /* x += alpha p, r -= alpha s; local <r, r> */
int hs_slab_plane_size(hs_slab *h, long long *n);        /* FP64 values per padded plane */
/* p's first / last interior plane into device buffers of hs_slab_plane_size
 * values (NULL: skipped); and device buffers into p's ghost planes below /
 * above (NULL: left as they are). */
int hs_slab_halo_get(hs_slab *h, double *lo, double *hi);
int hs_slab_halo_put(hs_slab *h, const double *lo, const double *hi);
int hs_slab_get(hs_slab *h, int which, double *host);    /* 0 x, 1 r, 2 p, 3 s: nx ny nz values */
/* Two-level preconditioner (additive): z = V-cycle(r) on the slab + P A_c^-1
 * P^T r on a global coarse grid of agg^3-cell aggregates held by every slab
 * (P piecewise constant, A_c = P^T A P, solved by its own V-cycle), which
 * restores the global coarse correction that block Jacobi lacks.  Set once
 * after hs_slab_create (this slab's first plane is global plane kg0 of nzg);
 * after each hs_slab_set_system, sum every slab's hs_slab_coarse_partial
 * couplings (sizes from hs_slab_coarse_sizes: coarse gx, gy, gz faces and
 * cells) and pass the sums to hs_slab_coarse_build on every slab.  Per
 * application: hs_slab_precond, then sum every slab's hs_slab_restrict and
 * pass the sum to hs_slab_coarse_correct, whose local <r, z> replaces the
 * one hs_slab_precond returned. */
int hs_slab_set_coarse(hs_slab *h, int agg, int kg0, int nzg);
int hs_slab_coarse_sizes(hs_slab *h, long long n4[4]);
int hs_slab_coarse_partial(hs_slab *h, double *cgx, double *cgy, double *cgz);
int hs_slab_coarse_build(hs_slab *h, const double *cgx, const double *cgy, const double *cgz);
int hs_slab_restrict(hs_slab *h, double *rc);
int hs_slab_coarse_correct(hs_slab *h, const double *rc, double *rz);
void hs_slab_destroy(hs_slab *h);

/* Validation of the divisions the sweeps perform with precomputed
 * reciprocals: returns how many of the n host pairs (a[i], b[i]) give a
 * quotient that differs in any bit from IEEE a/b on the current device
 * (negative HS_ERR_* on failure). */
long long hs_check_division(const double *a, const double *b, long long n);

/* Release all device and host state. */
void hs_destroy(hs_ctx *ctx);

/* Text of the last error on `ctx` (or of the calling thread when ctx is NULL). */
const char *hs_last_error(const hs_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* HSOLVER_B200_H */
