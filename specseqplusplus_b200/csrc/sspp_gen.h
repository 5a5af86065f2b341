// Synthetic filtered complexes (Vietoris-Rips of seeded point clouds,
// Freudenthal lower-star of smoothed noise) as PHAT boundary matrices.
// Input-side helpers for tests and benchmarks; not part of the reduction.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sspp_gen_matrix sspp_gen_matrix;

/* Rips complex of npts points i.i.d. uniform in [0,1]^space_dim (2 or 3),
 * edges of float32 Euclidean length <= radius, simplices up to maxdim (<= 3).
 * Returns NULL on invalid arguments. */
sspp_gen_matrix* sspp_gen_rips(int64_t npts, int32_t space_dim, uint64_t seed, float radius, int32_t maxdim);

/* Lower-star filtration of the Freudenthal triangulation of a grid^3 lattice
 * (all vertices, edges, triangles, tetrahedra); vertex values are N(0,1)
 * white noise smoothed by a Gaussian of width sigma voxels. */
sspp_gen_matrix* sspp_gen_lowerstar(int32_t grid, float sigma, uint64_t seed);

int64_t sspp_gen_ncols(const sspp_gen_matrix* m);
int64_t sspp_gen_nnz(const sspp_gen_matrix* m);
/* Copies dims[ncols], col_ptr[ncols+1], rows[nnz], values[ncols]; any may be NULL. */
int32_t sspp_gen_copy(const sspp_gen_matrix* m, int32_t* dims, int64_t* col_ptr, int32_t* rows, float* values);
void sspp_gen_free(sspp_gen_matrix* m);

#ifdef __cplusplus
}
#endif
