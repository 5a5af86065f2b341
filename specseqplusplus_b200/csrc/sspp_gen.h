// Synthetic filtered complexes (Vietoris-Rips of seeded point clouds,
// Freudenthal lower-star of smoothed noise) as PHAT boundary matrices.
// Input-side helpers for tests and benchmarks; not part of the reduction.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sspp_gen_matrix sspp_gen_matrix;

/* Rips complex of npts points i.i.d. uniform in [0,1]^space_dim (1..3; the
 * points of sspp_gen_points), edges of float32 Euclidean length <= radius,
 * simplices up to maxdim (<= 3).  Returns NULL on invalid arguments. */
sspp_gen_matrix* sspp_gen_rips(int64_t npts, int32_t space_dim, uint64_t seed, float radius, int32_t maxdim);
/* Same for the caller's points (npts x space_dim, row-major, finite). */
sspp_gen_matrix* sspp_gen_rips_points(int64_t npts, int32_t space_dim, const float* points, float radius,
                                      int32_t maxdim);
/* The seeded points of sspp_gen_rips: out[npts * space_dim]. */
int32_t sspp_gen_points(int64_t npts, int32_t space_dim, uint64_t seed, float* out);

/* Lower-star filtration of the Freudenthal triangulation of a grid^3 lattice
 * (all vertices, edges, triangles, tetrahedra); vertex values are N(0,1)
 * white noise smoothed by a Gaussian of width sigma voxels (sspp_gen_field). */
sspp_gen_matrix* sspp_gen_lowerstar(int32_t grid, float sigma, uint64_t seed);
/* Same for the caller's gx x gy x gz field (x fastest, no NaN; -0 read as +0),
 * simplices up to maxdim. */
sspp_gen_matrix* sspp_gen_lowerstar_field(int32_t gx, int32_t gy, int32_t gz, const float* values, int32_t maxdim);
/* The smoothed field of sspp_gen_lowerstar: out[grid^3]. */
int32_t sspp_gen_field(int32_t grid, float sigma, uint64_t seed, float* out);

int64_t sspp_gen_ncols(const sspp_gen_matrix* m);
int64_t sspp_gen_nnz(const sspp_gen_matrix* m);
/* Copies dims[ncols], col_ptr[ncols+1], rows[nnz], values[ncols]; any may be NULL. */
int32_t sspp_gen_copy(const sspp_gen_matrix* m, int32_t* dims, int64_t* col_ptr, int32_t* rows, float* values);
void sspp_gen_free(sspp_gen_matrix* m);

#ifdef __cplusplus
}
#endif
