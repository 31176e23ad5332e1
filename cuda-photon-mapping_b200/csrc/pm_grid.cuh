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
    const float4* rec = nullptr;   // when set: (position, 0), (direction, 0) per photon, gathered as one record
    bool uniform_pow = false;   // every photon has power pow_value: the sorted power is written, not gathered
    bool defer_pow = false;     // with uniform_pow: the sorted power is not written at all (the caller fills
                                // it with pow_value when it is asked for)
    float pow_value[3] = {0.f, 0.f, 0.f};
    int64_t n;
    // outputs (sized by grid_build_sizes)
    uint32_t* cell_starts;
    uint32_t* cell_sizes;
    float4* gpos;         // sorted: xyz + source index bits in w
    float* gdir;          // sorted: 3 floats per photon
    float* gpow;          // sorted: 3 floats per photon
    uint32_t* key_counts; // cells * S^3 (sub-cell counts)
    uint32_t* key_starts; // cells * S^3 + 1 (exclusive scan, total last)
    // scratch
    uint32_t* cid;        // n
    uint32_t* keys[2];    // n each
    uint32_t* vals[2];    // n each
    uint32_t* counts2;    // cells of the re-grid resolution (count scratch)
    uint32_t* hist;       // 512 * tiles
    void* scan_ws;
    uint32_t* small;      // 16 u32 of device scratch (max count, totals)
    uint32_t* host_words = nullptr;   // 2 pinned host words the count maxima are read into (else the stack)
    unsigned* status;
};

struct GridPlan {
    int dims[3];
    float cell;
    int64_t cells;
    uint32_t max_count;   // photons in the fullest cell of the chosen grid
    int launches;         // kernels launched by grid_count + grid_sort
};

// Phase 1: the reference's grid, including its re-grid rule (desired photons
// per cell, 1000 in the reference; rebuilt at desired / regrid_div when a cell
// holds more than regrid_mult * desired, 5 and 5).  One pass counts the photons
// of both candidate grids (scratch: cell_sizes, counts2) and their fullest
// cells; the plan is the chosen grid.  Synchronises the stream once (the
// re-grid decision is taken on the host, as in the reference).
cudaError_t grid_count(GridBuffers& B, const float aabb[6], int desired, int regrid_mult, int regrid_div,
                       GridPlan* plan, cudaStream_t st);

// Phase 2: order the photons by (cell, sub-cell, trace index), where each cell
// is split into S^3 sub-cells (S = 1, 2, 4 or 8), and write cell_starts /
// cell_sizes (exactly the reference's), key_starts (sub-cell ranges) and the
// sorted arrays.  Buffers: key arrays sized for cells * S^3 (+1).
cudaError_t grid_sort(GridBuffers& B, const float aabb[6], GridPlan& plan, int S, cudaStream_t st);

// ---- several instances in one key space ----
struct GridInstDev {
    float mn[3];
    int gx, gy, gz;
    float cell;
    int S;
    int64_t key0;             // first key of the instance
    int64_t cell0;            // first global cell of the instance
    int64_t ph0, cap;         // the instance's photon slots [ph0, ph0 + cap)
};
struct GridMulti {
    int ninst;
    const GridInstDev* tab;   // device, ninst
    const int64_t* ph_off;    // device, ninst + 1: slot offsets (ph0 of each instance, then the total)
    const int64_t* cell_off;  // device, ninst + 1
    const int64_t* filled;    // device, ninst: photons each instance produced (slots past min(cap, filled) are empty)
    int64_t total_keys, total_cells;
};
// B.n = all slots; B.key_counts >= total_keys + 1, B.key_starts >= total_keys + 2,
// cell arrays >= total_cells; cell_starts are instance-relative.
cudaError_t grid_multi(GridBuffers& B, const GridMulti& M, int* launches, cudaStream_t st);
cudaError_t radix_and_gather(GridBuffers& B, int64_t n, int64_t key_space, int* launches, cudaStream_t st);

// Scratch of a stand-alone radix sort: keys / vals ping-pong buffers (n each),
// hist (radix_hist_elems(n)), scan workspace (scan_workspace_bytes(hist elems)).
struct RadixBuffers {
    uint32_t* keys[2];
    uint32_t* vals[2];
    uint32_t* hist;
    void* scan_ws;
    unsigned* status;
};
size_t radix_hist_elems(int64_t n);
// Stable LSD radix sort of n keys below 2^key_bits carrying values (vals_in
// null: the input index).  *vals_sorted (and *keys_sorted when want_keys)
// point into B's buffers.
cudaError_t radix_sort_u32(const RadixBuffers& B, const uint32_t* keys_in, const uint32_t* vals_in, int64_t n,
                           int key_bits, bool want_keys, const uint32_t** keys_sorted, const uint32_t** vals_sorted,
                           int* launches, cudaStream_t st);

// sub-cell division for a grid whose fullest cell holds max_count photons:
// about 2k photons per sub-cell slab of a surface crossing the cell
int grid_auto_subdiv(uint32_t max_count, int k_hint);

// scratch sizes for n photons and at most max_keys sub-cells
void grid_scratch_sizes(int64_t n, int64_t max_keys, size_t* hist_elems, size_t* scan_ws_bytes);

}  // namespace pm
