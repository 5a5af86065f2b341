// Device builders of filtered flag complexes (Vietoris-Rips of a point cloud,
// lower-star filtration of the Freudenthal triangulation of a 3-D grid) that
// write the boundary matrix straight into device memory, in the column order
// of the reference's input files: (filtration value, dimension, lexicographic
// vertex tuple).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace sspp {

// Stream-ordered device buffers, grown on demand and reused across builds.
struct BuildScratch {
    enum {
        UP_OFF, UP_V, UP_W, UP_V2, UP_W2, E_SRC,      // upper adjacency (edges in lexicographic order)
        TRI_OFF, TRI_K, TRI_F, TRI_W,                 // triangles: third vertex, facet edges, value
        TET_OFF, TET_F, TET_W,                        // tetrahedra: facet triangles, value
        VVAL, IN, CELL_A, CELL_B, PT_A, PT_B,         // vertex values, copied input, Rips cell sort
        KEY_A, KEY_B, IDX_A, IDX_B, RANK,             // global order
        DIMS, COLPTR, ROWS, VALUES,                   // the boundary matrix
        BLK, MISC, TMP, NUM
    };
    void* p[NUM] = {};
    size_t cap[NUM] = {};
    int64_t* h_misc = nullptr;  // pinned, 8 entries
};

struct Built {
    int64_t ncols = 0, nnz = 0;
    int32_t* dims = nullptr;
    int64_t* col_ptr = nullptr;
    int32_t* rows = nullptr;
    float* values = nullptr;
};

// points: device array npts x space_dim (row-major), space_dim in 1..3.
// Returns 0, or -1 (bad input: non-finite coordinate, size limit) / -2 (CUDA
// error) with a message in *err.
int build_rips(BuildScratch& S, const float* d_points, int64_t npts, int space_dim, float radius, int maxdim,
               cudaStream_t s, Built* out, std::string* err);

// values: device array gx*gy*gz, x fastest.  All simplices of the Freudenthal
// triangulation up to maxdim (<= 3).
int build_lowerstar(BuildScratch& S, const float* d_values, int64_t gx, int64_t gy, int64_t gz, int maxdim,
                    cudaStream_t s, Built* out, std::string* err);

// Device buffer of at least `bytes` for a copy of the caller's input (the IN slot).
cudaError_t build_stage(BuildScratch& S, size_t bytes, cudaStream_t s, void** out);

void build_free(BuildScratch& S);

}  // namespace sspp
