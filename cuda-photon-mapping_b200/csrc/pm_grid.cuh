// pm_grid.cuh -- photon grid build (count, scan, stable scatter into cell-sorted SoA).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pm {

// The reference's grid sizing (CudaPhotonMapping/PhotonGrid.cu:41-56), evaluated
// on the host with the same float operations.
void grid_dims(const float aabb[6], int64_t n, int desired, int dims[3], float* cell);

struct GridBuffers {
    // inputs: unsorted photon list, 3 floats per photon each
    const float* pos;
    const float* dir;
    const float* pow;
    int64_t n;
    // outputs (sized by grid_build_sizes)
    uint32_t* cell_starts;
    uint32_t* cell_sizes;
    float4* gpos;         // sorted: xyz + source index bits in w
    float* gdir;          // sorted: 3 floats per photon
    float* gpow;          // sorted: 3 floats per photon
    // scratch
    uint32_t* cid;        // n
    uint32_t* keys[2];    // n each
    uint32_t* vals[2];    // n each
    uint32_t* hist;       // 256 * tiles
    void* scan_ws;
    uint32_t* small;      // 16 u32 of device scratch (max count, totals)
    unsigned* status;
};

// Build the grid of one photon map.  desired: photons per cell (1000 in the
// reference); the grid is rebuilt at desired / regrid_div when a cell holds more
// than regrid_mult * desired (5 and 5 in the reference).  Writes dims / cell /
// cells.  Requires buffers sized for the larger of the two candidate grids.
cudaError_t grid_build(GridBuffers& B, const float aabb[6], int desired, int regrid_mult, int regrid_div,
                       int dims[3], float* cell, int64_t* cells, cudaStream_t st);

// scratch sizes for n photons and at most max_cells cells
void grid_scratch_sizes(int64_t n, int64_t max_cells, size_t* hist_elems, size_t* scan_ws_bytes);

}  // namespace pm
