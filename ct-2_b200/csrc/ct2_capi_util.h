// Helpers shared by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "ct2_common.cuh"
#include "ct2_status.h"

namespace ct2 {

// Per-thread, per-device non-blocking stream used by the host entry points.
cudaStream_t lib_stream();

int check_grid(float dx, float dy, float dz, float x0, float y0, float z0, int nx, int ny, int nz);
int check_view(int ns, int nu, int nv, float du, float dv, float u0, float v0);
// Volume dimensions of the TV / regulariser entry points: non-negative, fewer
// than 2^40 voxels.
int check_vol(int nx, int ny, int nz);
Grid make_grid(float dx, float dy, float dz, float x0, float y0, float z0, int nx, int ny, int nz);

// Host entry points: stage host arrays through stream-ordered device
// allocations; everything is freed (and the stream synchronised) on exit.
struct HostCall {
    cudaStream_t st;
    std::vector<void*> bufs;
    HostCall();
    ~HostCall();
    int alloc(void** d, size_t bytes, bool zero);
    int upload(void** d, const void* h, size_t bytes);
    int download(void* h, const void* d, size_t bytes);
    int finish();
};

// Scratch for the device entry points: stream-ordered allocations released
// (stream-ordered) when the scope ends.
struct Scratch {
    cudaStream_t st;
    std::vector<void*> bufs;
    explicit Scratch(cudaStream_t s);
    ~Scratch();
    int get(void** d, size_t bytes, bool zero);
};

}  // namespace ct2
