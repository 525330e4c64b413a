// One rank's z-slab of the channel pressure-correction system (implemented in
// hs_slab.cu): the CG's vector passes and a block-Jacobi multigrid V-cycle on
// the slab, for a host that all-reduces the partial dot products and
// exchanges the search direction's boundary planes between slabs.
#pragma once

namespace hs {

struct SlabState;
SlabState *slab_create(int nx, int ny, int nz, int device);
void slab_destroy(SlabState *s);
// host face couplings gx ((nx+1) ny nz), gy (nx (ny+1) nz), gz (nx ny (nz+1):
// faces 0 and nz couple to the neighbouring slabs or to zero), b (nx ny nz)
void slab_set_system(SlabState *s, const double *gx, const double *gy, const double *gz, const double *b);
double slab_begin(SlabState *s);                      // x = 0, r = b; local <b, b>
double slab_precond(SlabState *s);                    // z = V-cycle(r); local <r, z>
void slab_direction(SlabState *s, double beta, int first);  // p = z + beta p (first: p = z)
double slab_apply(SlabState *s);                      // s = A p; local <s, p>
double slab_update(SlabState *s, double alpha);       // x += alpha p, r -= alpha s; local <r, r>
long long slab_plane_size(const SlabState *s);        // values per padded plane
void slab_halo_get(SlabState *s, double *lo, double *hi);        // p's first / last interior plane -> device buffers
void slab_halo_put(SlabState *s, const double *lo, const double *hi);  // device buffers -> p's ghost planes
void slab_get(SlabState *s, int which, double *host);  // 0 x, 1 r, 2 p, 3 s: nx ny nz values
// the two-level preconditioner's global coarse grid (aggregates of agg^3
// cells; this slab's first plane is global plane kg0 of nzg): set once, before
// slab_set_system, which then computes this slab's partial coarse couplings
void slab_set_coarse(SlabState *s, int agg, int kg0, int nzg);
void slab_coarse_sizes(const SlabState *s, long long *n4);  // coarse gx, gy, gz, cells
void slab_coarse_partial(const SlabState *s, double *cgx, double *cgy, double *cgz);
void slab_coarse_build(SlabState *s, const double *cgx, const double *cgy, const double *cgz);  // the sums over slabs
void slab_restrict(SlabState *s, double *rc_host);           // this slab's part of P^T r
double slab_coarse_correct(SlabState *s, const double *rc);  // z += P A_c^-1 rc (summed rc); local <r, z>

}  // namespace hs
