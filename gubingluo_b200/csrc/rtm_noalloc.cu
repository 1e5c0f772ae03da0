// rtm_noalloc.cu — GPU Laplacian image filter that makes no device allocation.
//
// rtm_laplace_image (laplacefd1d, image_function.cpp:44-79) filters an image on the host.
// This entry runs the same filter on the device for callers that cannot allocate device
// memory per call:
//   * code running next to a framework whose caching allocator already holds nearly all of
//     the device's memory, where a fresh cudaMalloc of two image-sized buffers can fail or
//     force that allocator to give back its cache;
//   * multi-stream pipelines that cannot afford the device-wide synchronisation that the
//     matching cudaFree performs.  The copies and the kernel run on the calling thread's
//     per-thread default stream (cudaStreamPerThread), which does not wait for the caller's
//     other streams; the call returns once that stream has finished.
// The image travels through one fixed scratch area that is part of this translation unit's
// device image: a file-scope __device__ array of kScratchCells cells for the input copy and as
// many for the filtered result (48 MiB per device in all, kept by every GPU on which this
// library's device code is loaded until the process exits).  Images above kScratchCells cells
// are refused.  Nothing in the scratch has to start at zero: every call copies the whole image
// in, and the kernel writes every output cell (the border included).  There is one scratch
// area per device, so calls on the same device must not overlap in time: two concurrent calls
// would read and write the same cells.
// The scratch address is looked up per device context: after cudaDeviceReset (or under another
// context of the same device) the module is loaded again, and the next call looks the address
// up again instead of using the old one.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "rtm_internal.h"

namespace {

constexpr long kScratchCells = 6L * 1024 * 1024;   // largest image, nx * nz
constexpr int kMaxDevices = 64;

// [0, kScratchCells): input copy; [kScratchCells, 2*kScratchCells): filtered image.
static __device__ __align__(256) float g_scratch[2 * kScratchCells];

// Same arithmetic as the host filter: sums of float neighbours, the centre term and the
// division in double, each axis rounded to float before the two are added; border cells 0.
// `scratch` is the device address of g_scratch (the host looks it up; in host code the
// array's name stands for a host-side shadow, not for device memory).
__global__ void k_laplace_scratch(float *scratch, int nx, int nz, int dx, int dz)
{
    const float *in = scratch;
    float *out = scratch + kScratchCells;
    const long n = (long)nx * nz;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int iz = (int)(i / nx), ix = (int)(i - (long)iz * nx);
        if (ix == 0 || iz == 0 || ix == nx - 1 || iz == nz - 1) {
            out[i] = 0.0f;
            continue;
        }
        const float *r = &in[i];
        const float t1 = (float)((r[1] + r[-1] - 2.0 * r[0]) / (dx * dx));
        const float t2 = (float)((r[nx] + r[-nx] - 2.0 * r[0]) / (dz * dz));
        out[i] = t1 + t2;
    }
}

std::mutex g_mu;
// device address of g_scratch and the context it was looked up in, per device
float *g_base[kMaxDevices];
CUcontext g_ctx[kMaxDevices];

// cuCtxGetCurrent from the driver (through the runtime, so the library needs no -lcuda).
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
CtxGetCurrentFn ctx_get_current()
{
    static CtxGetCurrentFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (CtxGetCurrentFn)p;
    });
    return fn;
}

}  // namespace

extern "C" int rtm_laplace_image_noalloc(float *image, int nx, int nz, int dx, int dz)
{
    rtm::clear_error();
    if (!image) return rtm::fail(RTM_ERR_ARG, "null image");
    if (nx < 1 || nz < 1) return rtm::fail(RTM_ERR_ARG, "image sizes must be positive");
    const long n = (long)nx * nz;
    if (n > kScratchCells) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "image of %ld cells exceeds the %ld-cell scratch of rtm_laplace_image_noalloc",
                      n, kScratchCells);
        return rtm::fail(RTM_ERR_ARG, msg);
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return rtm::fail(RTM_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return rtm::fail(RTM_ERR_ARG, "device index out of range");
    // cudaFree(0) makes the device's primary context current if no context is yet
    e = cudaFree(nullptr);
    if (e != cudaSuccess) return rtm::fail(RTM_ERR_CUDA, cudaGetErrorString(e));
    CtxGetCurrentFn get_ctx = ctx_get_current();
    CUcontext ctx = nullptr;
    if (!get_ctx || get_ctx(&ctx) != CUDA_SUCCESS || !ctx)
        return rtm::fail(RTM_ERR_CUDA, "no current CUDA context");
    float *base = nullptr;
    {
        // the first call in a device context (that device current) looks the scratch address up
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_base[dev] || g_ctx[dev] != ctx) {
            float *addr = nullptr;
            e = cudaGetSymbolAddress((void **)&addr, g_scratch);
            if (e != cudaSuccess) {
                g_base[dev] = nullptr;
                g_ctx[dev] = nullptr;
                return rtm::fail(RTM_ERR_CUDA, cudaGetErrorString(e));
            }
            g_base[dev] = addr;
            g_ctx[dev] = ctx;
        }
        base = g_base[dev];
    }
    const size_t bytes = (size_t)n * sizeof(float);
    cudaStream_t st = cudaStreamPerThread;
    if ((e = cudaMemcpyAsync(base, image, bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return rtm::fail(RTM_ERR_CUDA, cudaGetErrorString(e));
    const int blocks = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
    k_laplace_scratch<<<blocks, 256, 0, st>>>(base, nx, nz, dx, dz);
    if ((e = cudaGetLastError()) != cudaSuccess) return rtm::fail(RTM_ERR_CUDA, cudaGetErrorString(e));
    if ((e = cudaMemcpyAsync(image, base + kScratchCells, bytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return rtm::fail(RTM_ERR_CUDA, cudaGetErrorString(e));
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return rtm::fail(RTM_ERR_CUDA, cudaGetErrorString(e));
    return RTM_OK;
}
