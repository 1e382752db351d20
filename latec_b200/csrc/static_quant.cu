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
// before any stream capture.
#include <atomic>
#include <cmath>
#include <cuda_runtime.h>

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
std::atomic<void*> g_scratch_addr[kMaxDevices];

// Device address of g_quant_scratch for the current device, looked up once.
int scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return LATEC_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return LATEC_ERR_UNSUPPORTED;
    void* p = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!p) {
        if (cudaGetSymbolAddress(&p, g_quant_scratch) != cudaSuccess || !p) return LATEC_ERR_CUDA;
        g_scratch_addr[dev].store(p, std::memory_order_release);
    }
    *out = p;
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
    if (!prm || (prm->dtype != LATEC_F32 && prm->dtype != LATEC_F64) || prm->channels < 1 ||
        prm->radius < 1 || prm->radius > 32768 || prm->order < 0 || prm->order > 1 ||
        prm->center < 0 || prm->center > 2 || prm->end_mode < 0 || prm->end_mode > 3)
        return LATEC_ERR_ARG;
    if (items > kItems) return LATEC_ERR_TOO_LARGE;
    if ((items && (!x || !pred || !codes || !recon_out || !outliers)) || !stats || !hist_seg ||
        !hist_total)
        return LATEC_ERR_ARG;
    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char* s = (unsigned char*)base;
    void* staging = s + kStagingOff;
    uint32_t* tile_cnt = (uint32_t*)(s + kTileCntOff);
    uint32_t* tile_off = (uint32_t*)(s + kTileOffOff);
    double* partials = (double*)(s + kPartialsOff);
    QParams q;
    if (!(eb > 0.0)) return LATEC_ERR_ARG;
    q.w = 2.0 * eb;
    const double inv = 1.0 / q.w;
    q.inv_w = (std::isfinite(inv) && q.w > 0x1p-1000 && std::isfinite(q.w)) ? inv : 0.0;
    q.eb = eb;
    q.eb_f = (float)eb;
    q.radius = prm->radius;
    q.order = prm->order;
    q.center = prm->center;
    q.end_mode = prm->end_mode;
    q.round_output = prm->round_output;
    if (q.round_output < 0 || q.round_output > 2 ||
        (q.round_output == 2 && !(prm->round_span > 0.0 && std::isfinite(prm->round_span) &&
                                  std::isfinite(prm->round_offset))))
        return LATEC_ERR_ARG;
    q.rspan = q.round_output == 2 ? prm->round_span : 1.0;
    q.roff = q.round_output == 2 ? prm->round_offset : 0.0;
    q.channels = prm->channels;
    q.points = items;
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
