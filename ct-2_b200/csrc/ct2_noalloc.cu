// TV gradient entry point that allocates no device memory.
//
// Some callers of this library cannot let it call cudaMalloc: a reconstruction
// service that reserves its whole device-memory budget when it starts and
// forbids allocation while frames are in flight (an allocation there can fail
// or stall behind the driver at the worst moment), and host applications
// whose own allocator owns the device's memory, where a library's private
// cudaMalloc either fails or fragments that pool.  For them this variant of
// ct2_dev_totalvar_total_var_grad3d keeps its only scratch -- the per-block
// FP64 partial sums of the squared gradient -- in a fixed array in the
// library's own device memory instead of a per-call allocation.
#include <cuda_runtime.h>

#include <mutex>

#include "ct2_capi_util.h"
#include "ct2_exact.h"

namespace {

// Capacity of the scratch array: one double per reduction block.  The TV
// reduction uses min(ceil(voxels / 256), 8 * SMs) blocks, i.e. at most 1184 on
// a 148-SM B200, so 4096 entries (32 KiB) cover any volume on any GPU with up
// to 512 SMs.  Every GPU that loads the library holds this array until exit.
constexpr int kMaxPartials = 4096;
static __device__ __align__(256) double g_tv_partials[kMaxPartials];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_partials_ptr[kMaxDevices] = {};

// The array's device address for the current device, looked up once per
// device with that device current.  Host code must not pass g_tv_partials
// itself to a kernel: in host code that name is a host-side stand-in.
int partials_for_current_device(double** out)
{
    int dev = 0;
    CT2_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return ct2::set_error(CT2_EINVAL, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_partials_ptr[dev] == nullptr) {
        void* p = nullptr;
        CT2_CUDA(cudaGetSymbolAddress(&p, g_tv_partials));
        g_partials_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_partials_ptr[dev];
    return CT2_OK;
}

}  // namespace

extern "C" int ct2_dev_totalvar_total_var_grad3d_noalloc(float ambdala, float* tvgmat,
                                                         const float* smat, int nx, int ny,
                                                         int nz, int normalizeq, float* bobo,
                                                         void* stream)
{
    ct2::clear_error();
    int rc = ct2::check_vol(nx, ny, nz);  // the allocating entry point's own checks
    if (rc) return rc;
    if (bobo == nullptr) return ct2::set_error(CT2_EINVAL, "null bobo");
    const long long n = (long long)nx * ny * nz;
    if (n > 0 && (tvgmat == nullptr || smat == nullptr))
        return ct2::set_error(CT2_EINVAL, "null tvgmat/smat");
    const int parts = ct2::tv_parts(n);
    if (parts > kMaxPartials)
        return ct2::set_error(CT2_EINVAL,
                              "total_var_grad3d_noalloc: %d reduction blocks needed, the "
                              "preallocated scratch holds %d",
                              parts, kMaxPartials);
    double* partials = nullptr;
    rc = partials_for_current_device(&partials);
    if (rc) return rc;
    // Each block writes its partial sum before the finishing kernel reads
    // it, so nothing in the shared array has to be cleared between calls.
    return ct2::tv_grad(smat, tvgmat, nx, ny, nz, ambdala, normalizeq, bobo, partials,
                        (cudaStream_t)stream);
}
