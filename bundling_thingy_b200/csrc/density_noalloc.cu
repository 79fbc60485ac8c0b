// density_noalloc.cu — the density blur and normalisation without allocating.
//
// For callers that may not allocate device memory: a renderer or plugin that
// receives its device buffers from a host application which owns all GPU
// memory, or a frame loop that cannot afford cudaMalloc's implicit device
// synchronisation or an allocation failure mid-frame. The caller passes the
// splat counts and the output image; the one intermediate image lives in a
// file-scope static device array of a fixed size (held by every GPU that
// loads this library until the process exits).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "bt.h"
#include "kernels.cuh"

namespace bt {
bool make_blur_taps(double sigma, Taps* taps);
void set_thread_error(const char* message);
}  // namespace bt

namespace {

constexpr size_t kHeadWords = 64;   // 256-byte head: word 0 is the running maximum
constexpr size_t kMaxTexels = BT_NOALLOC_MAX_TEXELS;
constexpr int kMaxDevices = 64;

// The shared scratch: the peak word, then one f32 image of up to kMaxTexels.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kHeadWords + kMaxTexels];

struct DeviceSetup {
    bool done = false;
    uint32_t* base = nullptr;
};

std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

// Once per device, with that device current: the device address of the static
// array (its name in host code is only a host-side stand-in) and the blur
// kernels' shared-memory attribute. Only a successful set-up is remembered: a
// failed one (a transient error) is tried again by the next call.
cudaError_t device_setup(int device, uint32_t** base) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& s = g_setup[device];
    if (!s.done) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e == cudaSuccess) e = bt::prepare_density_kernels();
        if (e != cudaSuccess) return e;
        s.base = static_cast<uint32_t*>(p);
        s.done = true;
    }
    *base = s.base;
    return cudaSuccess;
}

bt_status reject(bt_status code, const std::string& message) {
    bt::set_thread_error(message.c_str());
    return code;
}

}  // namespace

extern "C" bt_status bt_density_noalloc(const uint32_t* counts, float* density, uint32_t width, uint32_t height,
                                        float blur_sigma, void* stream) {
    if (!counts || !density) return reject(BT_ERR_INVALID, "null device buffer");
    // The normalisation stores four texels at a time and the horizontal pass
    // reads whole words: a misaligned buffer would fault on the device.
    if (reinterpret_cast<uintptr_t>(density) % 16 != 0)
        return reject(BT_ERR_INVALID, "density output must be 16-byte aligned");
    if (reinterpret_cast<uintptr_t>(counts) % 4 != 0)
        return reject(BT_ERR_INVALID, "splat counts must be 4-byte aligned");
    if (width == 0 || height == 0) return reject(BT_ERR_INVALID, "density map dimensions must be nonzero");
    const unsigned long long texels = static_cast<unsigned long long>(width) * height;
    if (texels > kMaxTexels)
        return reject(BT_ERR_INVALID, "width*height = " + std::to_string(texels) +
                                          " exceeds the static scratch of " + std::to_string(kMaxTexels) +
                                          " texels (BT_NOALLOC_MAX_TEXELS)");
    bt::Taps taps;
    if (!bt::make_blur_taps(blur_sigma, &taps)) return reject(BT_ERR_INVALID, "invalid blur sigma");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return reject(BT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices) return reject(BT_ERR_INVALID, "device ordinal out of range");
    uint32_t* base = nullptr;
    if ((e = device_setup(device, &base)) != cudaSuccess)
        return reject(BT_ERR_CUDA, std::string("static scratch set-up: ") + cudaGetErrorString(e));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* peak = base;
    float* vertical = reinterpret_cast<float*>(base + kHeadWords);
    // The maximum must start at zero; the array keeps the previous call's values.
    if ((e = cudaMemsetAsync(peak, 0, sizeof(uint32_t), s)) != cudaSuccess)
        return reject(BT_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    // Horizontal pass into the caller's output, vertical pass (and maximum)
    // into the static image, normalisation back into the output.
    bt::launch_blur_horizontal(counts, density, width, height, taps, s);
    bt::launch_blur_vertical(density, vertical, width, height, taps, peak, s);
    bt::launch_normalize(vertical, peak, density, texels, s);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return reject(BT_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return BT_OK;
}
