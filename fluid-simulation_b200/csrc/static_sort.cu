// static_sort.cu — stable sort permutation of caller-owned device keys that
// allocates no device memory (wcsph_sort_keys_static in include/wcsph.h).
//
// Who needs it: callers that must not call cudaMalloc/cudaFree while they
// run — a render or control loop that cannot take the device-wide
// synchronisation cudaFree implies, or a host that runs under a fixed device
// memory budget reserved up front. The regular path (CUDASPHSimulator)
// allocates its sort buffers per context; this variant runs the same onesweep
// kernels on one scratch block that is part of the library image instead.
//
// The scratch is a file-scope device array sized for WCSPH_STATIC_SORT_MAX_KEYS
// keys (about 1.8 MiB). Every GPU that loads the library holds it until the
// process exits, and every call on that GPU shares it.
#include <mutex>
#include <string>

#include <cuda.h>   // CUcontext (the driver entry point is fetched through the runtime)

#include "simulator.cuh"
#include "static_sort.cuh"

namespace wcsph {

namespace {

constexpr u32 kStaticTiles = (WCSPH_STATIC_SORT_MAX_KEYS + SORT_TILE - 1) / SORT_TILE;

struct StaticSortScratch {
    u64 keys[2][WCSPH_STATIC_SORT_MAX_KEYS];   // ping-pong keys of the digit passes
    u32 vals[2][WCSPH_STATIC_SORT_MAX_KEYS];   // ping-pong particle indices
    u32 hist[SORT_DIGITS * 256];               // digit histograms (must start at zero)
    u32 offsets[SORT_DIGITS * 256];
    u32 lookback[SORT_DIGITS * kStaticTiles * 256];  // zeroed by enqueue_sort_passes
    DevState st;                                // pass plan, tile counters, error flags (zeroed per call)
};

static __device__ __align__(256) StaticSortScratch g_static_sort_scratch;

// perm[i] = index of the key of rank i (identity when no digit pass was
// active). When a look-back wait of the sort ran out, the passes did not
// produce a permutation: every entry then reads WCSPH_STATIC_SORT_FAILED, an
// index no key has (n <= WCSPH_STATIC_SORT_MAX_KEYS), so that the failure is
// visible in the caller's own output without a host round trip.
__global__ void write_perm_kernel(const StaticSortScratch* s, u32 n, u32* __restrict__ perm) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s->st.error_flags) {
        perm[i] = WCSPH_STATIC_SORT_FAILED;
        return;
    }
    const u32 sel = s->st.sort_sel[SORT_DIGITS];
    perm[i] = sel == 0u ? i : s->vals[sel - 1u][i];
}

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
struct ScratchSlot {
    CUcontext ctx = nullptr;   // context the address was looked up in
    StaticSortScratch* addr = nullptr;
};
ScratchSlot g_scratch[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);

// The calling thread's current context, through the driver entry point the
// runtime hands out (the library does not link the driver library itself).
CUcontext current_context() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

// Device address of the scratch on the current device. On the host the name
// g_static_sort_scratch is only a stand-in for the device symbol, never an
// address a kernel may use, so the address is looked up with that device
// current: once per device, and again whenever the device's current context
// is not the one the address was found in (after cudaDeviceReset, or under a
// caller's own driver-API context).
StaticSortScratch* scratch_on_current_device() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) throw Error(WCSPH_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        throw Error(WCSPH_ERR_NOT_SUPPORTED, "wcsph_sort_keys_static supports devices 0..63");
    // binds the device's primary context to this thread (CUDA 12 initialises
    // it here) before the current context is read
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) throw Error(WCSPH_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    const CUcontext ctx = current_context();
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    ScratchSlot& slot = g_scratch[dev];
    if (!slot.addr || slot.ctx != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_sort_scratch);
        if (e != cudaSuccess)
            throw Error(WCSPH_ERR_CUDA, std::string("cudaGetSymbolAddress(static sort scratch): ") +
                                            cudaGetErrorString(e));
        slot.addr = static_cast<StaticSortScratch*>(p);
        slot.ctx = ctx;
    }
    return slot.addr;
}

}  // namespace

void static_sort_permutation(const uint64_t* keys, uint32_t n, uint32_t* perm, cudaStream_t stream) {
    if (n > WCSPH_STATIC_SORT_MAX_KEYS)
        throw Error(WCSPH_ERR_INVALID_ARGUMENT,
                    "wcsph_sort_keys_static: n = " + std::to_string(n) + " exceeds the maximum of " +
                        std::to_string(WCSPH_STATIC_SORT_MAX_KEYS) + " keys");
    if (n == 0) return;
    if (!keys || !perm) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "wcsph_sort_keys_static: null keys or perm");
    StaticSortScratch* s = scratch_on_current_device();
    // The scratch keeps the previous call's contents: clear what the passes
    // expect to start at zero.
    WCSPH_CUDA(cudaMemsetAsync(s->hist, 0, sizeof(s->hist), stream));
    WCSPH_CUDA(cudaMemsetAsync(&s->st, 0, sizeof(DevState), stream));
    SortBuffers b{};
    b.keys[0] = const_cast<u64*>(reinterpret_cast<const u64*>(keys));  // read only
    b.keys[1] = s->keys[0];
    b.keys[2] = s->keys[1];
    b.vals[1] = s->vals[0];
    b.vals[2] = s->vals[1];
    b.hist = s->hist;
    b.offsets = s->offsets;
    b.lookback = s->lookback;
    b.capacity = WCSPH_STATIC_SORT_MAX_KEYS;
    const u32 blocks = (n + 255u) / 256u;
    hist_only_kernel<<<blocks, 256, 0, stream>>>(b.keys[0], n, s->hist);
    WCSPH_CUDA(cudaGetLastError());
    WCSPH_CUDA(enqueue_sort_passes(b, n, &s->st, stream));
    write_perm_kernel<<<blocks, 256, 0, stream>>>(s, n, perm);
    WCSPH_CUDA(cudaGetLastError());
}

}  // namespace wcsph
