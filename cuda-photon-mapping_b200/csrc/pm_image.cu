// pm_image.cu -- headless frame output (host code).
//
// The reference shows each frame through an OpenGL pixel buffer
// (CudaPhotonMapping/Drawer.cu:22-41, Window.cuh:88-126); this library renders
// into device buffers instead, and these two writers put such a frame in a
// file: the 8-bit canvas as a binary PPM, the float radiance as a PFM.  The
// canvas's row 0 is the bottom row (Camera.cuh:67-81: v = (y + 0.5) / H runs
// upwards), so the PPM writer flips the rows; a PFM stores its rows bottom to
// top already.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/pm_api.h"

namespace {

// the frame's bytes in host memory: copied from the device when ptr is a
// device (or managed) pointer, else read in place.  A host without a usable
// CUDA driver has no device pointers, so its buffers are host memory.
int host_bytes(const void* ptr, size_t bytes, std::vector<uint8_t>& copy, const uint8_t** out) {
    cudaPointerAttributes attr;
    std::memset(&attr, 0, sizeof(attr));
    const cudaError_t e = cudaPointerGetAttributes(&attr, ptr);
    const bool device = e == cudaSuccess && (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
    if (e != cudaSuccess) (void)cudaGetLastError();   // not a CUDA pointer (or no driver): plain host memory
    if (!device) {
        *out = static_cast<const uint8_t*>(ptr);
        return PM_OK;
    }
    copy.resize(bytes);
    if (cudaMemcpy(copy.data(), ptr, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
        (void)cudaGetLastError();
        return PM_ERR_CUDA;
    }
    *out = copy.data();
    return PM_OK;
}

bool valid_size(int32_t w, int32_t h) {
    return w > 0 && h > 0 && (int64_t)w * (int64_t)h <= ((int64_t)1 << 31);
}

int write_file(const char* path, const std::string& header, const uint8_t* rows, size_t row_bytes, int32_t h,
               bool flip) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return PM_ERR_IO;
    bool ok = std::fwrite(header.data(), 1, header.size(), f) == header.size();
    for (int32_t r = 0; ok && r < h; r++) {
        const int32_t src = flip ? h - 1 - r : r;
        ok = std::fwrite(rows + (size_t)src * row_bytes, 1, row_bytes, f) == row_bytes;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PM_OK : PM_ERR_IO;
}

bool little_endian() {
    const uint32_t one = 1u;
    uint8_t b;
    std::memcpy(&b, &one, 1);
    return b == 1;
}

}  // namespace

extern "C" int pm_write_ppm(const char* path, const uint8_t* rgb8, int32_t width, int32_t height) {
    if (!path || !rgb8 || !valid_size(width, height)) return PM_ERR_INVALID;
    const size_t row = (size_t)width * 3;
    std::vector<uint8_t> copy;
    const uint8_t* px = nullptr;
    if (int rc = host_bytes(rgb8, row * (size_t)height, copy, &px)) return rc;
    const std::string header = "P6\n" + std::to_string(width) + " " + std::to_string(height) + "\n255\n";
    return write_file(path, header, px, row, height, true);
}

extern "C" int pm_write_pfm(const char* path, const float* radiance, int32_t width, int32_t height) {
    if (!path || !radiance || !valid_size(width, height)) return PM_ERR_INVALID;
    if (!little_endian()) return PM_ERR_INVALID;   // the header's scale -1.0 declares little-endian floats
    const size_t row = (size_t)width * 3 * sizeof(float);
    std::vector<uint8_t> copy;
    const uint8_t* px = nullptr;
    if (int rc = host_bytes(radiance, row * (size_t)height, copy, &px)) return rc;
    const std::string header = "PF\n" + std::to_string(width) + " " + std::to_string(height) + "\n-1.0\n";
    return write_file(path, header, px, row, height, false);
}
