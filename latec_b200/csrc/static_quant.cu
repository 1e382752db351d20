// latec_quantize_static: the flat quantizer (latec_quantize) for callers that
// cannot allocate device memory.
//
// Who needs it: code that must not call cudaMalloc/cudaFree -- for example an
// application whose device memory is entirely owned by another allocator (a
// framework's caching allocator that has reserved the GPU), or a
// latency-critical loop where cudaMalloc/cudaFree would implicitly
// synchronise the device. latec_quantize asks the caller for a workspace;
// this variant needs none: its scratch (outlier staging, per-tile outlier
// counts and offsets, per-CTA statistics) lives in one file-scope device
// array of fixed size that every GPU loading the library holds until the
// process exits. The caller still passes every input and output buffer.
//
// Limits and sharing: at most LATEC_STATIC_MAX_ITEMS values per call. All
// calls on a device share the same scratch array and it keeps the contents of
// the previous call, so this function clears what must start at zero, and
// calls whose GPU work overlaps (on different streams, or from different host
// threads without ordering) race on the scratch and must not be issued.
// Set-up: the first call on each device looks the array's device address up
// with cudaGetSymbolAddress (with that device current); make that first call
// before any stream capture. The address is looked up again in a new context
// of the device (after cudaDeviceReset, for example), so such a call is a
// set-up call too.
#include <cuda_runtime.h>
#include <mutex>

#include "host_util.h"
#include "interp_kernels.cuh"

namespace latec {

namespace {

constexpr uint64_t kItems = LATEC_STATIC_MAX_ITEMS;
constexpr uint64_t kAlign = 256;
constexpr uint64_t round_up(uint64_t v) { return (v + kAlign - 1) / kAlign * kAlign; }
// scratch layout: staging (float64 worst case) | tile counts | tile offsets | CTA partials
constexpr uint64_t kTiles = (kItems + TILE - 1) / TILE + 1;
constexpr uint64_t kStagingOff = 0;
constexpr uint64_t kTileCntOff = round_up(kStagingOff + kItems * 8);
constexpr uint64_t kTileOffOff = round_up(kTileCntOff + kTiles * 4);
constexpr uint64_t kPartialsOff = round_up(kTileOffOff + kTiles * 4);
constexpr uint64_t kBytes = round_up(kPartialsOff + ((uint64_t)MAX_BLOCKS * 5 + 5) * 8);

// The shared scratch array (one copy per device that loads this library).
static __device__ __align__(256) unsigned char g_quant_scratch[kBytes];

constexpr int kMaxDevices = 64;

// Per device: the context the address was looked up in, and the address. A
// device reset (cudaDeviceReset) or a new primary context reloads the module,
// which may move the array, so the address is looked up again whenever the
// current context differs from the one it was found in.
struct ScratchSlot {
    std::mutex mu;
    unsigned long long ctx = 0;
    void* addr = nullptr;
};
ScratchSlot g_scratch[kMaxDevices];

// Device address of g_quant_scratch in the current device's context.
int scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return LATEC_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return LATEC_ERR_UNSUPPORTED;
    const unsigned long long ctx = current_context_id();
    ScratchSlot& slot = g_scratch[dev];
    std::lock_guard<std::mutex> lk(slot.mu);
    // ctx 0: no context was current yet; the lookup below makes the primary
    // context current, and the next call records its id
    if (!slot.addr || ctx == 0 || ctx != slot.ctx) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_quant_scratch) != cudaSuccess || !p) return LATEC_ERR_CUDA;
        slot.addr = p;
        slot.ctx = ctx;
    }
    *out = slot.addr;
    return LATEC_OK;
}

}  // namespace
}  // namespace latec

using namespace latec;

extern "C" {

int latec_quantize_static(const latec_quant_params* prm, double eb, uint64_t items, const void* x,
                          const void* pred, uint16_t* codes, void* recon_out, void* outliers,
                          latec_stage_stats* stats, uint32_t* hist_seg, uint32_t* hist_total,
                          void* stream) {
    // the same parameter checks as latec_quantize, in the same order
    if (!valid_params(prm) || (items && (!x || !pred || !codes || !recon_out || !outliers)) ||
        !stats || !hist_seg || !hist_total)
        return LATEC_ERR_ARG;
    QParams q;
    if (!make_q(prm, eb, items, q)) return LATEC_ERR_ARG;
    if (items > kItems) return LATEC_ERR_TOO_LARGE;
    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char* s = (unsigned char*)base;
    void* staging = s + kStagingOff;
    uint32_t* tile_cnt = (uint32_t*)(s + kTileCntOff);
    uint32_t* tile_off = (uint32_t*)(s + kTileOffOff);
    double* partials = (double*)(s + kPartialsOff);
    cudaStream_t st = (cudaStream_t)stream;
    // outputs that accumulate start at zero; tile counts are zeroed by the launcher
    if (cudaMemsetAsync(stats, 0, sizeof(latec_stage_stats), st) != cudaSuccess ||
        cudaMemsetAsync(hist_seg, 0, sizeof(uint32_t) * HBINS * n_segments(items), st) !=
            cudaSuccess ||
        cudaMemsetAsync(hist_total, 0, sizeof(uint32_t) * 65536ull, st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    StageAcc* acc = (StageAcc*)stats;
    const int elem = prm->dtype == LATEC_F64 ? 8 : 4;
    rc = launch_quantize_flat(q, prm->dtype, items, x, pred, codes, staging, tile_cnt, tile_off,
                              hist_total, hist_seg, acc, partials, recon_out, st);
    if (!rc) rc = launch_compact(codes, items, staging, elem, tile_cnt, tile_off, outliers, st);
    return rc;
}

}  // extern "C"
