// Fused level kernels for 3-D grids: all five sub-stages of one level of the
// dyadic schedule (weight 1 along axes 0, 1, 2, then the fused weight-2 and
// weight-3 stages) in one launch each way, column by column of the level's
// lattice, with the planes of a column in shared memory.
#pragma once

#include "interp_kernels.cuh"

namespace latec {

constexpr int TILE_STAGES = 5;  // w1 axis 0, w1 axis 1, w1 axis 2, w2, w3

// One sub-stage of the fused level (its slot in TileLevel::st is its order in
// the schedule).
struct TileStage {
    QParams q;             // the stage's quantizer (per-stage error bound)
    uint16_t* codes;       // the stage's codes, channel-major (encode writes, decode reads)
    void* staging;         // encode: outlier values at their code index
    uint32_t* tile_cnt;    // encode: outliers per 2048-code tile (zeroed by the caller)
    uint32_t* hist_total;  // encode: 65536-bin histogram of codes outside the window
    uint32_t* hist_seg;    // encode: HBINS bins per 2^22-code segment of the stage
    double* partials;      // encode: 5 statistics per CTA
    StageAcc* acc;         // encode: maxq / outlier totals
    uint32_t n;            // points of the stage per channel
    uint32_t pad;
};

// A level of stride s seen as its lattice: lattice point u (per axis) is the
// grid point s * u. Level points are the lattice points with an odd
// coordinate; the even-even-even points are the coarser levels.
struct TileLevel {
    int32_t N[3];          // lattice points per axis
    int32_t pad0;
    int64_t ls[3];         // grid element stride of one lattice step per axis
    uint64_t points;       // grid points per channel
    int32_t channels;
    int32_t tiles_x, tiles_y;  // column tiles along the lattice's axes 2 and 1
    int32_t chunks, zc;        // axis-0 chunks of zc planes (zc even)
    uint32_t items;            // channels * chunks * tiles_y * tiles_x work items
    int32_t tma;               // planes arrive by TMA (else per-element async copies)
    int32_t pad1;
    TileStage st[TILE_STAGES];
};

// Column tile (lattice points) along axis 2 and axis 1 for an element size.
inline int tile_tx(int) { return 64; }
inline int tile_ty(int elem) { return elem == 8 ? 16 : 32; }

// The TMA path applies: unit lattice step along axis 2, rows of whole 16-byte
// groups, every 16-byte aligned base pointer.
inline bool tile_tma_ok(const TileLevel& L, int elem, const void* a, const void* b) {
    const int64_t v = 16 / elem;
    return L.ls[2] == 1 && L.ls[1] % v == 0 && L.ls[0] % v == 0 && (int64_t)L.points % v == 0 &&
           ((uintptr_t)a % 16) == 0 && ((uintptr_t)b % 16) == 0;
}

// Work decomposition of a level: tiles, axis-0 chunk length, items. grid is
// the persistent CTA count (one wave of resident CTAs).
void tile_level_geometry(TileLevel& L, int elem, int n_sm, uint32_t* grid);

// Fused encode / decode of one level. Encode reports a failed load wait by
// setting bit 31 of `done` in the stages' statistics; decode through err.
int launch_tile_level_encode(const TileLevel& L, int dtype, int cubic, uint32_t grid,
                             const void* x, void* recon, cudaStream_t st);
int launch_tile_level_decode(const TileLevel& L, int dtype, int cubic, uint32_t grid, void* recon,
                             uint32_t* err, cudaStream_t st);
constexpr uint32_t TILE_WAIT_FAILED = 0x80000000u;  // StageAcc::done bit (encode)
constexpr uint32_t ERR_TILE_WAIT = 0x400u;          // err bit (decode)

// Stage tails of a fused encode: per stage (one CTA each) the fixed-order
// reduction of the per-CTA statistics and the exclusive scan of the tile
// outlier counts.
struct TailStage {
    const double* partials;
    uint32_t blocks;
    uint32_t tiles;
    const uint32_t* tile_cnt;
    uint32_t* tile_off;
    StageAcc* acc;
};
struct TailArgs {
    TailStage s[TILE_STAGES];
};
int launch_stage_tails(const TailArgs& a, int n, cudaStream_t st);

// Decode: write every outlier of the given stages into the canvas at its grid
// position (the fused decode then takes code-0 points from the canvas).
struct ScatterStage {
    StageDesc d;
    const uint16_t* codes;
    const uint8_t* outliers;
    const uint32_t* tile_cnt;
    const uint32_t* tile_off;
    uint64_t items;
    uint32_t n_out;
    uint32_t tile0;  // first block of the stage in the launch
};
struct ScatterArgs {
    ScatterStage s[TILE_STAGES];
    int n;
    int channels;
    uint64_t points;
};
int launch_scatter_outliers(const ScatterArgs& a, int dtype, uint32_t total_tiles, void* recon,
                            uint32_t* err, cudaStream_t st);

}  // namespace latec
