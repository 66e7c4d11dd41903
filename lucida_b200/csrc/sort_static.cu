// Radix sort for callers that cannot allocate device memory.
//
// luc_sort_u32_dev sorts through scratch buffers its context grows with
// cudaMalloc. Some callers cannot allow that: a host that reserves all of a
// GPU's memory when it starts (an engine running under a fixed device-memory
// budget, or a process sharing the GPU under a strict allocation policy) gets
// no memory later, and a cudaMalloc/cudaFree inside a latency-critical frame
// loop can synchronise the whole device. luc_sort_u32_static serves them: it
// takes the caller's device arrays and stream, keeps its scratch in the
// file-scope device arrays below (allocated once, with the module, on every
// GPU that loads this library, and held until the process exits) and calls no
// allocating routine.
#include <cstdio>
#include <cstring>
#include "ctx.cuh"
#include "sort_kernels.cuh"

namespace {

using namespace luc;

// The largest sort this entry point accepts: 2^20 (key, value) pairs.
constexpr uint32_t kStaticMaxKeys = 1u << 20;
constexpr uint32_t kStaticMaxTiles = (kStaticMaxKeys + kTile - 1) / kTile;
constexpr uint32_t kHistWords = 4 * 256 + 4 * 256 + 8;  // histograms, offsets, 4 tile counters, error flag

// Scratch: ping-pong keys/values (8 MiB), look-back status words (256 KiB)
// and histograms. Every call reuses it and it keeps the last call's contents.
static __device__ __align__(256) uint32_t g_scratch_keys[kStaticMaxKeys];
static __device__ __align__(256) uint32_t g_scratch_vals[kStaticMaxKeys];
static __device__ __align__(256) uint32_t g_scratch_status[kStaticMaxTiles * 256];
static __device__ __align__(256) uint32_t g_scratch_hist[kHistWords];

// Device addresses of the arrays in the current context. In host code the
// array names are host-side stand-ins, never device addresses, so kernels
// only ever get the addresses cudaGetSymbolAddress returns. They are looked
// up on every call (cheap once the module is loaded), so no address outlives
// the context it was taken in.
struct ScratchAddr {
    uint32_t *keys = nullptr, *vals = nullptr, *status = nullptr, *hist = nullptr;
};

void set_err(char* msg, uint32_t len, const char* text) {
    if (msg && len) {
        std::strncpy(msg, text, len - 1);
        msg[len - 1] = '\0';
    }
}

int32_t scratch_addresses(ScratchAddr& a, char* msg, uint32_t len) {
    cudaError_t e;
    if ((e = cudaGetSymbolAddress((void**)&a.keys, g_scratch_keys)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&a.vals, g_scratch_vals)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&a.status, g_scratch_status)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&a.hist, g_scratch_hist)) != cudaSuccess) {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "luc_sort_u32_static: cudaGetSymbolAddress failed: %s",
                      cudaGetErrorString(e));
        set_err(msg, len, buf);
        return LUC_ERR_LAUNCH;
    }
    return LUC_OK;
}

// Launch with the launch's own status as the result (not the thread's
// last-error word, which may hold an earlier, unrelated failure).
template <typename... Params, typename... Args>
cudaError_t launch(void (*kernel)(Params...), unsigned grid, unsigned block, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = s;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

}  // namespace

extern "C" uint32_t luc_sort_u32_static_max(void) { return kStaticMaxKeys; }

extern "C" int32_t luc_sort_u32_static(void* keys_dev, void* vals_dev, uint32_t n, void* stream, char* err_msg,
                                       uint32_t err_len) {
    set_err(err_msg, err_len, "");
    if (n > kStaticMaxKeys) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "luc_sort_u32_static: %u keys exceeds the static scratch maximum of %u",
                      n, kStaticMaxKeys);
        set_err(err_msg, err_len, buf);
        return LUC_ERR_VALIDATION;
    }
    if (n <= 1) return LUC_OK;
    if (!keys_dev || !vals_dev) {
        set_err(err_msg, err_len, "luc_sort_u32_static: null device array");
        return LUC_ERR_VALIDATION;
    }
    ScratchAddr sa;
    int32_t rc = scratch_addresses(sa, err_msg, err_len);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    uint32_t* hist = sa.hist;
    uint32_t* offs = hist + 1024;
    uint32_t* tcount = hist + 2048;
    const unsigned grid = std::min<uint32_t>((n + 255) / 256, 148 * 32);
    uint32_t *ka = (uint32_t*)keys_dev, *va = (uint32_t*)vals_dev, *kb = sa.keys, *vb = sa.vals;
    int dev = 0, sms = 0;
    cudaError_t ae = cudaGetDevice(&dev);
    if (ae == cudaSuccess) ae = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (ae != cudaSuccess || sms <= 0) {
        set_err(err_msg, err_len, "luc_sort_u32_static: cannot query the device");
        return LUC_ERR_LAUNCH;
    }
    // The scratch keeps the previous call's contents: clear what must start at zero.
    cudaError_t e = cudaMemsetAsync(hist, 0, kHistWords * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = launch(k_hist4, grid, 256, s, (const uint32_t*)keys_dev, n, hist);
    if (e == cudaSuccess) e = launch(k_hist_scan, 1, 256, s, (const uint32_t*)hist, offs);
    for (int p = 0; p < 4 && e == cudaSuccess; ++p) {
        e = cudaMemsetAsync(sa.status, 0, (size_t)tiles * 256 * sizeof(uint32_t), s);
        if (e == cudaSuccess)
            e = launch(k_onesweep, onesweep_grid(tiles, sms), kSortThreads, s, (const uint32_t*)ka, (const uint32_t*)va, kb, vb, n,
                       8 * p, (const uint32_t*)(offs + 256 * p), sa.status, tcount + p, tcount + 4, kSpinLimit);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    // After four passes the sorted pairs are back in the caller's arrays.
    uint32_t flag = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, tcount + 4, sizeof(flag), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "luc_sort_u32_static: %s", cudaGetErrorString(e));
        set_err(err_msg, err_len, buf);
        return LUC_ERR_LAUNCH;
    }
    if (flag) {
        set_err(err_msg, err_len, "luc_sort_u32_static: look-back wait gave up");
        return LUC_ERR_VALIDATION;
    }
    return LUC_OK;
}
