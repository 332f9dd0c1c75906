// fx_static.cu -- the producer schedule with no device allocation.
//
// Some callers cannot allocate device memory at the moment they need the
// producer records: a scanning service whose HBM is already claimed by its
// own memory pool (a cudaMalloc there fails, or forces the pool to give
// memory back), and real-time acquisition loops, where the cudaFree that
// grows a context's frame buffers synchronizes the whole device and stalls
// every other stream.  fx_producer_rows_static serves them: its scratch is
// one file-scope __device__ array, reserved when the library's module for
// this file is loaded, and the call itself makes no cudaMalloc, cudaFree or
// other allocating call.
//
// When the array is reserved depends on how the CUDA runtime loads modules.
// Under lazy loading (CUDA_MODULE_LOADING=LAZY, the default since CUDA 12.2)
// the module is loaded, and the 24 MiB reserved, by the first
// cudaGetSymbolAddress of this entry point, so only processes that call it
// pay for it.  Under CUDA_MODULE_LOADING=EAGER every context of the process
// reserves it when the context is created.
#include <cstring>
#include <mutex>

#include "fx_internal.cuh"

namespace fx {

// Producer scratch for frames up to a full 5782x3946 4000-dpi scan (that
// frame needs 23.8 MB), plus the error word.
constexpr size_t kStaticScratchBytes = (size_t)24 << 20;
constexpr size_t kStaticErrBytes = 256;
constexpr int kStaticMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch, looked up once per device with that
// device current.  The first lookup loads the module (reserving the array),
// so a caller should make its first call before it starts any stream
// capture.
static void *g_static_ptr[kStaticMaxDevices];
static std::mutex g_static_mu[kStaticMaxDevices];

// Holds the context's call lock for the whole call, so fx_set_tables cannot
// rewrite the LUT while this call's kernels read it and no other call on the
// context overwrites its error text; restores the caller's current device.
class StaticCallScope {
  public:
    explicit StaticCallScope(fx_context *ctx) : ctx_(ctx) {
        context_lock(ctx_);
        restore_ = cudaGetDevice(&saved_) == cudaSuccess;
    }
    ~StaticCallScope() {
        if (restore_) cudaSetDevice(saved_);
        context_unlock(ctx_);
    }
    StaticCallScope(const StaticCallScope &) = delete;
    StaticCallScope &operator=(const StaticCallScope &) = delete;

  private:
    fx_context *ctx_;
    int saved_ = 0;
    bool restore_ = false;
};

}  // namespace fx

using namespace fx;

FX_API int fx_producer_rows_static(fx_context *ctx, const uint16_t *d_main_rgbi, int32_t h,
                                   int32_t w, float *d_rows, fx_stage *d_stages, void *stream) {
    if (!ctx || !d_main_rgbi || !d_rows || !d_stages || h < 1 || w < 8)
        return FX_ERR_INVALID_ARGUMENT;
    // lock order: the context's lock, then the device's scratch lock
    StaticCallScope scope(ctx);
    const int device = context_device(ctx);
    if (device < 0 || device >= kStaticMaxDevices)
        return context_fail(ctx, FX_ERR_INVALID_ARGUMENT, "device index outside the static table");
    const float *lut = context_lut(ctx);
    if (!lut) return context_fail(ctx, FX_ERR_TABLES, "fx_set_tables has not been called");
    const size_t need = producer_bytes(h, w);
    if (need > kStaticScratchBytes - kStaticErrBytes)
        return context_fail(ctx, FX_ERR_INVALID_ARGUMENT,
                            "a %dx%d frame needs %zu bytes of producer scratch; the static "
                            "scratch holds %zu",
                            h, w, need, kStaticScratchBytes - kStaticErrBytes);

    // One scratch array per device: two calls in flight at once would race
    // on it.  The lock is held until this call's work on `stream` is done,
    // so calls through this entry point are serialized.
    std::lock_guard<std::mutex> lock(g_static_mu[device]);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess)
        return context_fail(ctx, FX_ERR_CUDA, "cudaSetDevice failed: %s", cudaGetErrorString(e));
    if (!g_static_ptr[device]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            if (e == cudaErrorMemoryAllocation)
                return context_fail(ctx, FX_ERR_OUT_OF_MEMORY,
                                    "the device has no room for the %zu MiB static producer "
                                    "scratch (reserved when the module loads)",
                                    kStaticScratchBytes >> 20);
            return context_fail(ctx, FX_ERR_CUDA, "cudaGetSymbolAddress failed: %s",
                                cudaGetErrorString(e));
        }
        g_static_ptr[device] = p;
    }
    char *base = reinterpret_cast<char *>(g_static_ptr[device]);
    uint32_t *err = reinterpret_cast<uint32_t *>(base);
    void *scratch = base + kStaticErrBytes;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

    // Only the error word must start at zero: the producer kernels write
    // every scratch element before they read it.
    e = cudaMemsetAsync(err, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess)
        e = launch_producer(d_main_rgbi, h, w, lut, scratch, d_stages, d_rows, err, st);
    uint32_t status = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&status, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return context_fail(ctx, FX_ERR_CUDA, "producer launch failed: %s", cudaGetErrorString(e));
    }
    // A stage whose setter fails is written as zeros and reported with the
    // setter's message; the rows are complete either way.
    if (status) return context_device_error(ctx, status);
    return FX_OK;
}
