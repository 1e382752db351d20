// Device-side descriptors and launchers of the rANS entropy stage.
#pragma once

#include "interp_kernels.cuh"
#include "latec_common.cuh"

namespace latec {

constexpr int BUCKET_BITS = 10;
constexpr int NBUCKET = 1 << BUCKET_BITS;
constexpr int MODE_LANES = 0;
constexpr int MODE_COMPAT = 1;

// Encoder entry of one symbol (32 bytes). The lane coder divides by the
// frequency with rcp / shift (exact below 2^63); the single-stack coder, whose
// state spans all 64 bits, with the Granlund-Montgomery multiplier gm and the
// shifts gsh1 / gsh2 (exact for every 64-bit state).
// The lane coder's fields come first (24 bytes, the loads it issues), the
// stack coder's multiplier last.
struct EncSym {
    uint64_t rcp;
    uint32_t bias;
    uint32_t cmpl;
    uint32_t freq;
    uint8_t shift;
    uint8_t gsh1;
    uint8_t gsh2;
    uint8_t pad;
    uint64_t gm;
};

// One stage of the entropy stage, shared layout with the host (see capi.cu;
// the Python host fills the same fields through latec_rans_stage).
struct RansStageDesc {
    uint64_t codes_off;   // first code of the stage in the codes buffer
    uint64_t out_off;     // first outlier of the stage in the outlier buffer
    uint64_t enc;         // EncSym table (rows of alphabet + 1)
    uint64_t cdf;         // CDF rows (alphabet + 1 entries each)
    uint64_t bucket;      // bucket rows (NBUCKET entries each)
    uint64_t scratch_off; // word offset of the stage's scratch region
    uint64_t blob_off;    // decode: word offset of the blob in the words buffer
    uint64_t rec_off;     // encode: byte offset of the stage record in the payload
    uint64_t framed_hi;   // frame word without the length (kexp/shape/level/owx/lit)
    uint32_t n;           // symbols (channels * points)
    uint32_t K;           // lane coder: symbols per lane per chunk
    uint32_t n_chunks;
    uint32_t chunk0;      // first global chunk of the stage
    uint32_t alphabet;
    int32_t kexp;
    int32_t radius;
    int32_t mode;         // MODE_LANES or MODE_COMPAT
    int32_t per_point;    // 1: per-symbol table row from the levels array
    uint32_t blob_words;  // encode: computed; decode: given
    uint32_t n_out;
    uint32_t block0;      // decode: first CTA of the stage (filled by the library)
};

constexpr int DEC_WARPS = 4;             // warps (chunks) per decoder CTA
constexpr int SMEM_ALPHA = 8192;         // largest alphabet decoded from shared memory
constexpr int RING = 256;                // decoder word window per warp (power of two)

int launch_build_tables(const uint32_t* cdf, int alphabet, int rows, EncSym* enc, uint16_t* bucket,
                        cudaStream_t st);
int launch_lanes_encode(const RansStageDesc* st, int n_stages, uint32_t total_chunks,
                        const uint16_t* codes, const uint8_t* levels, uint32_t* scratch,
                        uint32_t* chunk_words, uint32_t* err, cudaStream_t s);
int launch_lanes_decode(const RansStageDesc* st, int n_stages, uint32_t total_blocks,
                        int max_alphabet,
                        const uint32_t* words, const uint64_t* chunk_range, const uint8_t* levels,
                        uint16_t* codes, uint32_t* err, cudaStream_t s);
int launch_stack_encode(const RansStageDesc* st, int n_stages, const uint16_t* codes,
                        const uint8_t* levels, uint32_t* scratch, uint32_t* stage_words,
                        uint32_t* err, cudaStream_t s);
int launch_stack_decode(const RansStageDesc* st, int n_stages, const uint32_t* words,
                        const uint8_t* levels, uint16_t* codes, uint32_t* err, cudaStream_t s);
int launch_assemble(RansStageDesc* st, int n_stages, uint32_t total_chunks,
                    const uint32_t* lane_scratch, const uint32_t* chunk_words, uint32_t* chunk_off,
                    const uint32_t* stack_scratch, const uint32_t* stage_words,
                    const StageAcc* acc, const uint8_t* outliers, int elem, uint8_t* payload,
                    uint64_t cap, uint64_t* total, uint32_t* err, cudaStream_t s);

}  // namespace latec
