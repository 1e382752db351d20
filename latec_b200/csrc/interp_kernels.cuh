// Kernel launch helpers of the fused interpolation / quantizer stage.
#pragma once

#include <atomic>

#include "latec_common.cuh"

namespace latec {

constexpr int TILE = 2048;            // outlier-count granularity (points)
constexpr int THREADS = 256;
constexpr int GROUP = 2 * THREADS;    // encode: points per CTA iteration (two per thread)
constexpr int MAX_BLOCKS = 148 * 8;   // encode grid cap (8 CTAs per SM)
constexpr int HWIN = 256;             // histogram window |q| < HWIN kept in SMEM
constexpr int HBINS = 2 * HWIN;       // bin 0: outliers, q + HWIN otherwise
constexpr int SEG_SHIFT = 22;         // float32 histogram accumulation segment

struct QParams {
    double w;        // 2 * eb, float64
    double inv_w;    // 1 / w, or 0 when the reciprocal is not finite
    double eb;       // float64 bound (float64 path)
    float eb_f;      // float32(eb) (float32 path)
    int radius;
    int order;       // 0 linear, 1 cubic
    int center;      // 0 average, 1 first odd axis, 2 last odd axis
    int end_mode;    // bit 0 quadratic ends, bit 1 extrapolation
    int round_output;  // 0 none, 1 rint, 2 via the raw integer (rspan / roff)
    int channels;
    uint64_t points;  // grid points per channel
    double rspan, roff;  // round_output 2: the data range and its minimum
};

// Per-stage device accumulators (one struct per stage).
struct StageAcc {
    uint32_t n_out;
    uint32_t maxq;
    uint32_t done;   // CTAs of the stage pass that have finished
    uint32_t nout;   // running outlier total (CTA atomics)
    double stats[5];  // pred_sae, pred_sse, recon_sae, recon_sse, recon_max
};

inline uint32_t n_tiles(uint64_t items) { return (uint32_t)((items + TILE - 1) / TILE); }
__host__ __device__ inline uint32_t n_tiles_of(uint64_t items) {
    return (uint32_t)((items + TILE - 1) / TILE);
}

// Decode: one stage of the all-stage tile passes (the stages of one tensor,
// or of many: each stage names its own codes and error word).
struct DecStage {
    const uint16_t* codes;  // the stage's codes
    uint32_t* err;          // bit 1: outlier count mismatch
    uint64_t items;         // codes of the stage
    uint32_t tile0;         // first global tile of the stage
    uint32_t n_out;         // outliers stored for the stage
};
// Level kernels: all sub-stages of one level of the schedule in one launch,
// as work items (sub-stage, band along axis 0, tile range) claimed in a fixed
// order; an item waits only for lower-weight items that precede it.
struct LvlStage {
    StageDesc d;
    QParams q;
    const uint16_t* codes;     // the stage's codes
    const uint8_t* outliers;   // the stage's outliers (decode)
    const uint32_t* tile_cnt;  // the stage's outlier counts / offsets per tile
    const uint32_t* tile_off;
    uint32_t n_out;
    uint32_t pad;
};
struct LvlBand {
    uint32_t stage;    // index into the level's LvlStage array
    uint32_t counter;  // finished items of this band
    uint32_t dep_off;  // dependencies: LvlDep[dep_off, dep_off + dep_cnt)
    uint32_t dep_cnt;
};
struct LvlDep {
    uint32_t counter;
    uint32_t need;     // items of that band
};
struct LvlItem {
    uint32_t band;
    uint32_t tile0, tile1;  // stage-local tiles
    uint32_t pad;
};
constexpr uint32_t LEVEL_WAIT_LIMIT = 1u << 22;  // polls of one dependency (x ~100 ns)
constexpr uint32_t ERR_LEVEL_WAIT = 0x200u;

// Many tensors per launch: one stage of one tensor is a job of a launch whose
// CTAs are dealt to its jobs in order (first[j]: the first CTA of job j).
struct ManyJob {
    const StageDesc* d;   // device copy of the stage's descriptor
    QParams q;
    const void* x;        // encode: the field
    void* recon;
    const uint16_t* codes_in;  // decode: the stage's codes
    uint16_t* codes;      // encode: the stage's codes
    void* staging;        // encode: the tensor's outlier staging buffer
    uint32_t* tile_cnt;   // the stage's per-tile outlier counts / offsets
    uint32_t* tile_off;
    uint32_t* hist_total;  // encode: the stage's full-code histogram
    uint32_t* hist_seg;    // encode: the stage's first histogram segment
    StageAcc* acc;         // encode: the stage's statistics
    double* partials;      // encode: per-CTA partial statistics
    uint8_t* out;          // encode: where the stage's outliers are compacted
    const uint8_t* outliers;  // decode: the stage's stored outliers
    uint32_t* err;         // decode: the tensor's error word
    uint64_t items;
    uint32_t gpb;          // encode: 512-point groups per CTA
    uint32_t blocks;       // CTAs of the stage pass (encode) / tiles (decode)
    uint32_t is_anchor;
    uint32_t elem;         // bytes per value
    uint32_t n_out;        // decode: stored outliers
    uint32_t cblocks;      // encode: compaction CTAs
};
struct ZeroRange {
    uint32_t* p;
    uint64_t words;
};
constexpr uint64_t ZERO_CHUNK = 1u << 16;  // words cleared by one CTA of k_zero_many

// Launch kinds of the many-tensor passes: rank class (2, 3, 4, or 0 for the
// runtime rank), fused stage layout, interpolation order.
int launch_quant_many(int dtype, int nd, int kind, int cubic, const ManyJob* jobs,
                      const uint32_t* first, uint32_t n_jobs, uint32_t ctas, cudaStream_t st);
int launch_dequant_many(int dtype, int nd, int kind, int cubic, const ManyJob* jobs,
                        const uint32_t* first, uint32_t n_jobs, uint32_t ctas, cudaStream_t st);
int launch_compact_many(const ManyJob* jobs, const uint32_t* first, uint32_t n_jobs,
                        uint32_t ctas, cudaStream_t st);
int launch_zero_many(const ZeroRange* r, const uint32_t* first, uint32_t n, uint32_t ctas,
                     cudaStream_t st);
// The encode grid of a stage of `items` points: CTAs (at most `cap`, 0 = the
// single-stage cap) and 512-point groups per CTA.
uint32_t encode_grid(uint64_t items, uint32_t cap, uint32_t* blocks);

// CTAs of the encode kernels for a stage of `items` points (partials rows).
uint32_t encode_blocks(uint64_t items);
inline uint32_t n_blocks(uint64_t items) { return encode_blocks(items); }
inline uint32_t n_segments(uint64_t items) {
    return (uint32_t)((items + (1ull << SEG_SHIFT) - 1) >> SEG_SHIFT);
}

// Row-segment stage kernels on (1, default) or off (0): process-wide.
extern std::atomic<int> g_row_mode;

// Launchers (interp_kernels.cu). items = channels * stage points.
int launch_interp_quant(const StageDesc& d, const QParams& q, int dtype, int is_anchor,
                        const void* x, void* recon, uint16_t* codes, void* staging,
                        uint32_t* tile_cnt, uint32_t* tile_off, uint32_t* hist_total,
                        uint32_t* hist_seg, StageAcc* acc, double* partials, cudaStream_t st);
int launch_interp_predict(const StageDesc& d, const QParams& q, int dtype, const void* recon,
                          void* pred, cudaStream_t st);
int launch_count_zeros_all(const DecStage* ds, int n_stages, uint32_t total_tiles,
                           uint32_t* tile_cnt, cudaStream_t st);
int launch_tile_offsets_all(const DecStage* ds, int n_stages, const uint32_t* tile_cnt,
                            uint32_t* tile_off, cudaStream_t st);
int launch_compact(const uint16_t* codes, uint64_t items, const void* staging, int elem,
                   const uint32_t* tile_cnt, const uint32_t* tile_off, void* out,
                   cudaStream_t st);
int launch_interp_dequant(const StageDesc& d, const QParams& q, int dtype, int is_anchor,
                          const uint16_t* codes, const void* outliers, const uint32_t* tile_cnt,
                          const uint32_t* tile_off, uint32_t n_out, void* recon, uint32_t* err,
                          cudaStream_t st);
int launch_dequant_flat(const QParams& q, int dtype, uint64_t items, const void* pred,
                        const uint16_t* codes, const void* outliers, const uint32_t* tile_cnt,
                        const uint32_t* tile_off, uint32_t n_out, void* recon, uint32_t* err,
                        cudaStream_t st);
int launch_level_dequant(int dtype, int nd, int cubic, const LvlStage* stages,
                         const LvlBand* bands, const LvlDep* deps, const LvlItem* items,
                         uint32_t n_items, uint32_t* ctr, void* recon, uint32_t* err,
                         cudaStream_t st);
int launch_quantize_flat(const QParams& q, int dtype, uint64_t items, const void* x,
                         const void* pred, uint16_t* codes, void* staging, uint32_t* tile_cnt,
                         uint32_t* tile_off, uint32_t* hist_total, uint32_t* hist_seg,
                         StageAcc* acc, double* partials, void* recon_out, cudaStream_t st);

}  // namespace latec
