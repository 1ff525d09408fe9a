// solweig_step_static_scratch: the hourly step with its scratch planes in a
// file-scope device array instead of a caller-provided buffer.
//
// Who needs it: a host that drives the step through the C ABI but owns no
// device allocator of its own for temporaries -- e.g. a Fortran / C urban
// climate model that hands over pointers to arrays it allocated once at start
// up and must not call cudaMalloc/cudaFree inside its time loop (cudaFree
// synchronises the whole device, which stalls the host's other streams, and
// a per-call allocation can fail part way through a long run).  Such a caller
// would otherwise have to reserve and manage 20 scratch planes itself.
//
// The array is reserved on a device when the library's device code is loaded
// there.  Under CUDA's default lazy module loading that happens at the first
// call of this entry point on the device, so other processes do not pay the
// 20 MiB; with CUDA_MODULE_LOADING=EAGER every process that creates a context
// after loading libsolweig_b200.so reserves it on that device.
#include <mutex>

#include "common.cuh"

namespace {

constexpr long long kMaxPixels = SOLWEIG_STATIC_SCRATCH_MAX_PIXELS;
constexpr long long kPlanes = SOLWEIG_STEP_SCRATCH_PLANES;
constexpr int kMaxDevices = 64;

// [20][kMaxPixels] float32 scratch planes, reused by every call on a device.
// Nothing in it has to start at zero: within one call every plane is written
// before it is read (night hours read none of it).
__device__ __align__(256) float g_step_scratch[kPlanes * kMaxPixels];

std::mutex g_lock;
float* g_address[kMaxDevices] = {};

// Address of this device's copy of the array, looked up once per device with
// that device current (the first call on a device does the lookup, which may
// load the module; later calls only read the cached pointer).
int scratch_address(float** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        solweig::set_error("solweig_step_static_scratch: cudaGetDevice: %s", cudaGetErrorString(e));
        return SOLWEIG_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        solweig::set_error("solweig_step_static_scratch: device %d beyond the %d devices supported",
                           dev, kMaxDevices);
        return SOLWEIG_ERR_INVALID;
    }
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_address[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_step_scratch);
        if (e != cudaSuccess || !p) {
            solweig::set_error("solweig_step_static_scratch: cudaGetSymbolAddress on device %d: %s",
                               dev, cudaGetErrorString(e));
            return SOLWEIG_ERR_CUDA;
        }
        g_address[dev] = static_cast<float*>(p);
    }
    *out = g_address[dev];
    return SOLWEIG_OK;
}

}  // namespace

extern "C" int solweig_step_static_scratch(const SolweigScene* scene, const SolweigSkyLayout* layout,
                                           const SolweigHour* hours, int hour,
                                           const SolweigState* state, const SolweigOutputs* out,
                                           const int32_t* gvf_dxdy, int first_steps,
                                           int second_steps, void* stream) {
    SOLWEIG_CHECK_ARG(scene, "solweig_step_static_scratch: null scene");
    const long long pixels = (long long)scene->rows * scene->cols;
    SOLWEIG_CHECK_ARG(scene->rows > 0 && scene->cols > 0 && pixels <= kMaxPixels,
                      "solweig_step_static_scratch: a %d x %d tile (%lld pixels) exceeds the static "
                      "scratch capacity of %lld pixels; use solweig_step with a caller scratch buffer",
                      scene->rows, scene->cols, pixels, kMaxPixels);
    float* scratch = nullptr;
    const int rc = scratch_address(&scratch);
    if (rc) return rc;
    // The planes are laid out for this tile's pixel count ([20][pixels]),
    // packed at the start of the array.
    return solweig_step(scene, layout, hours, hour, state, out, gvf_dxdy, first_steps, second_steps,
                        scratch, stream);
}
