// Shared definitions of the LATEC B200 library: stage descriptors, fast
// integer division, rank -> grid-coordinate decoding, error plumbing.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/latec_b200.h"

namespace latec {

constexpr int MAXD = LATEC_MAX_NDIM;

// Process-wide count of kernel launches issued by this library (capi.cu).
void count_launches(unsigned n);

// Unsigned 32-bit division by a runtime constant (round-up multiplier method,
// Granlund & Montgomery 1994): q = (t + ((n - t) >> 1)) >> sh with
// t = mulhi(n, mul), exact for every n < 2^32 and d >= 1 (d == 1: mul = 0,
// sh = 0 gives (n >> 1) + ... so d == 1 is flagged and returns n).
struct FastDiv {
    uint32_t d, mul, sh, one;
};

inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f{d, 0u, 0u, d == 1u ? 1u : 0u};
    if (d > 1) {
        uint32_t l = 0;
        while ((1ull << l) < d) l++;  // l = ceil(log2 d) >= 1
        // mul = floor(2^32 * (2^l - d) / d) + 1
        uint64_t m = ((uint64_t)((1ull << l) - d) << 32) / d + 1;
        f.mul = (uint32_t)m;
        f.sh = l - 1;
    }
    return f;
}

__host__ __device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
#ifdef __CUDA_ARCH__
    uint32_t t = __umulhi(n, f.mul);
#else
    uint32_t t = (uint32_t)(((uint64_t)n * f.mul) >> 32);
#endif
    uint32_t q = (t + ((n - t) >> 1)) >> f.sh;
    return f.one ? n : q;
}

// One sub-stage of the dyadic schedule, in the form the kernels consume.
//
// kind 0 -- a single parity class laid out row-major (the anchor stage and the
//           weight-1 sub-stages): coord_j = start_j + step * m_j with
//           m = unravel(rank, size).
// kind 1 -- a fused weight-w sub-stage: the union of all weight-w parity
//           classes in flat grid order, decoded axis by axis with the
//           per-lattice-index block sizes G[j][r] and the even-parity
//           completion counts F[j+1][r] (r = odd axes still to place).
struct StageDesc {
    int32_t ndim;
    int32_t kind;
    int32_t axis;     // weight-1 axis; -1 for the anchor stage; -2 for fused
    int32_t weight;   // number of odd axes (0 anchors)
    uint32_t n;       // points of the stage per channel
    int32_t s;        // level stride (tap distance unit)
    int32_t step;     // kind 0: lattice step of the class
    int32_t shape[MAXD];
    int64_t gstride[MAXD];
    int32_t start[MAXD];      // kind 0
    FastDiv size_div[MAXD];   // kind 0 / 2: class extent per axis
    FastDiv g_div[MAXD][MAXD + 1];  // kind 1: G[j][r]
    uint32_t f_even[MAXD][MAXD + 1];  // kind 1: F[j+1][r]
    // Blocked anchors (anchor_block > 1): the anchor stage is kind 2, every
    // anchor_block^ndim block of the anchor lattice in C order; a later stage
    // whose point set meets those blocks skips them ("holes"). Its points are
    // then the full set above minus the holes, in the same C order.
    int32_t astride;          // anchor stride (a power of two)
    int32_t ablock;           // anchor block edge (1: no blocked anchors)
    int32_t holes;            // the stage's full set contains anchor-block points
    int32_t lg2s;             // log2(2 s): lattice positions of one parity are 2 s apart
    uint32_t n_full;          // points of the full set (n + holes)
    FastDiv blk_div;          // kind 2: divide by ablock
    // per axis and parity (0: even, 1: odd multiple of s): positions of the
    // progression parity * s + 2 s m per anchor period (log2), how many of
    // them start inside a block, and how many of the axis's positions do
    uint32_t h_lgp[MAXD][2];
    uint32_t h_k[MAXD][2];
    uint32_t h_tot[MAXD][2];
    uint32_t h_c[MAXD + 1][MAXD + 1];  // kind 1: block completions of axes j.., r odd left
    uint32_t h_suf[MAXD + 1];          // kind 0: product of h_tot over axes j..
};

// The anchor stage of a blocked plan (kind 2): every anchor_block^ndim block
// of the anchor lattice in C order; rank -> coordinates, flat grid index.
__host__ __device__ __forceinline__ int64_t block_anchor_coords(const StageDesc& d, uint32_t rank,
                                                                int32_t* coord) {
    int64_t flat = 0;
    uint32_t rem = rank;
    for (int j = MAXD - 1; j >= 0; j--) {
        if (j < d.ndim) {
            const uint32_t q = fdiv(rem, d.size_div[j]);
            const uint32_t m = rem - q * d.size_div[j].d;
            rem = q;
            const uint32_t b = fdiv(m, d.blk_div);  // block m / ablock, offset m % ablock
            coord[j] = (int32_t)(b * (uint32_t)d.astride + (m - b * d.blk_div.d));
            flat += (int64_t)coord[j] * d.gstride[j];
        }
    }
    return flat;
}

// Decode a stage-local rank into grid coordinates; returns the flat grid index.
__host__ __device__ __forceinline__ int64_t stage_coords(const StageDesc& d, uint32_t rank,
                                                int32_t* coord) {
    if (d.kind == 2) return block_anchor_coords(d, rank, coord);
    int64_t flat = 0;
    if (d.kind == 0) {
        uint32_t rem = rank;
#pragma unroll
        for (int j = MAXD - 1; j >= 0; j--) {
            if (j < d.ndim) {
                uint32_t q = fdiv(rem, d.size_div[j]);
                uint32_t m = rem - q * d.size_div[j].d;
                rem = q;
                coord[j] = d.start[j] + d.step * (int32_t)m;
                flat += (int64_t)coord[j] * d.gstride[j];
            }
        }
    } else {
        uint32_t rem = rank;
        int r = d.weight;
        const int32_t s2 = 2 * d.s;
#pragma unroll
        for (int j = 0; j < MAXD; j++) {
            if (j < d.ndim) {
                const FastDiv& g = d.g_div[j][r];
                uint32_t m = fdiv(rem, g);
                rem -= m * g.d;
                uint32_t f0 = d.f_even[j][r];
                int p = rem >= f0;
                if (p) {
                    rem -= f0;
                    r -= 1;
                }
                coord[j] = s2 * (int32_t)m + (p ? d.s : 0);
                flat += (int64_t)coord[j] * d.gstride[j];
            }
        }
    }
    return flat;
}

// Compile-time specialised decode: ND > 0 fixes the rank (loops unroll, the
// coordinates stay in registers), KIND fixes the stage layout (0 single
// class, 1 fused); ND == 0 falls back to the runtime rank. Blocked-anchor
// stages (kind 2) go through stage_point_t.
template <int ND, int KIND>
__host__ __device__ __forceinline__ int64_t stage_coords_t(const StageDesc& d, uint32_t rank,
                                                           int32_t* coord) {
    constexpr int NDV = ND > 0 ? ND : MAXD;
    int64_t flat = 0;
    uint32_t rem = rank;
    if (KIND == 0) {
#pragma unroll
        for (int j = NDV - 1; j >= 0; j--) {
            if (ND > 0 || j < d.ndim) {
                const uint32_t q = fdiv(rem, d.size_div[j]);
                const uint32_t m = rem - q * d.size_div[j].d;
                rem = q;
                coord[j] = d.start[j] + d.step * (int32_t)m;
                flat += (int64_t)coord[j] * d.gstride[j];
            }
        }
    } else {
        int r = d.weight;
        const int32_t s2 = 2 * d.s;
#pragma unroll
        for (int j = 0; j < NDV; j++) {
            if (ND > 0 || j < d.ndim) {
                const FastDiv& g = d.g_div[j][r];
                const uint32_t m = fdiv(rem, g);
                rem -= m * g.d;
                const uint32_t f0 = d.f_even[j][r];
                const int p = rem >= f0;
                if (p) {
                    rem -= f0;
                    r -= 1;
                }
                coord[j] = s2 * (int32_t)m + (p ? d.s : 0);
                flat += (int64_t)coord[j] * d.gstride[j];
            }
        }
    }
    return flat;
}

// ---- stages with holes (blocked anchors)

// In-block positions among the first m positions of a progression with
// 2^lgp positions per anchor period, k of them inside a block (the first k).
__host__ __device__ __forceinline__ uint32_t block_count(uint32_t m, uint32_t lgp, uint32_t k) {
    const uint32_t r = m & ((1u << lgp) - 1u);
    return (m >> lgp) * k + (r < k ? r : k);
}

// The point lies in an anchor block: every coordinate's offset in its anchor
// period is below the block edge.
template <int ND>
__host__ __device__ __forceinline__ bool in_blocks(const StageDesc& d, const int32_t* coord) {
    constexpr int NDV = ND > 0 ? ND : MAXD;
    bool in = true;
#pragma unroll
    for (int j = 0; j < NDV; j++)
        if (ND > 0 || j < d.ndim) in = in && (coord[j] & (d.astride - 1)) < d.ablock;
    return in;
}

// Holes (anchor-block points of the stage's full set) before the point in C
// order. A hole precedes the point iff it agrees on axes < j, is smaller on
// axis j and the agreeing prefix is itself inside the blocks: a sum over j of
// (in-block positions before coord[j]) x (in-block completions of the later
// axes), with the stage's parity constraint carried along for the fused kind.
template <int ND, int KIND>
__host__ __device__ __forceinline__ uint32_t holes_before(const StageDesc& d,
                                                          const int32_t* coord) {
    constexpr int NDV = ND > 0 ? ND : MAXD;
    uint32_t h = 0;
    bool in = true;
    int r = d.weight;
    const int32_t s = d.s;
#pragma unroll
    for (int j = 0; j < NDV; j++) {
        if (ND > 0 || j < d.ndim) {
            const uint32_t c = (uint32_t)coord[j];
            if (KIND == 0) {
                const uint32_t par = d.start[j] == s ? 1u : 0u;
                const uint32_t m = (c - (uint32_t)d.start[j]) >> d.lg2s;  // position index
                if (in) h += block_count(m, d.h_lgp[j][par], d.h_k[j][par]) * d.h_suf[j + 1];
            } else {
                // positions of each parity strictly before c
                const uint32_t m0 = (c + (1u << d.lg2s) - 1u) >> d.lg2s;
                const uint32_t m1 = (c + (uint32_t)s - 1u) >> d.lg2s;
                if (in) {
                    h += block_count(m0, d.h_lgp[j][0], d.h_k[j][0]) * d.h_c[j + 1][r];
                    if (r > 0) h += block_count(m1, d.h_lgp[j][1], d.h_k[j][1]) * d.h_c[j + 1][r - 1];
                }
                r -= (c & (uint32_t)s) ? 1 : 0;
            }
            in = in && (c & (uint32_t)(d.astride - 1)) < (uint32_t)d.ablock;
        }
    }
    return h;
}

// Rank -> grid point of a stage, holes skipped. Without holes this is the
// closed-form decode; with holes, the rank-r point is the least full-set index
// i with i - holes_before(i) = r that is not a hole: i = r + holes_before(i)
// is reached by fixed-point iteration from i = r (the right side never
// decreases and never passes the least solution), then holes are stepped over.
template <int ND, int KIND>
__host__ __device__ __forceinline__ int64_t stage_point_holes(const StageDesc& d, uint32_t rank,
                                                              int32_t* coord) {
    uint32_t i = rank;
    int64_t f = stage_coords_t<ND, KIND>(d, i, coord);
    for (int it = 0; it < 256; it++) {
        const uint32_t ni = rank + holes_before<ND, KIND>(d, coord);
        if (ni == i || ni >= d.n_full) break;
        i = ni;
        f = stage_coords_t<ND, KIND>(d, i, coord);
    }
    while (in_blocks<ND>(d, coord) && i + 1 < d.n_full) f = stage_coords_t<ND, KIND>(d, ++i, coord);
    return f;
}

template <int ND, int KIND>
__host__ __device__ __forceinline__ int64_t stage_point_t(const StageDesc& d, uint32_t rank,
                                                          int32_t* coord) {
    // blocked-anchor stages (kind 2, or with holes) run only on the runtime-
    // rank instances (ND == 0): the rank-specialised ones keep the plain
    // decode, with no blocked-anchor code beside it
    if constexpr (ND == 0) {
        if (KIND == 0 && d.kind == 2) return block_anchor_coords(d, rank, coord);
        if (d.holes) return stage_point_holes<ND, KIND>(d, rank, coord);
    }
    return stage_coords_t<ND, KIND>(d, rank, coord);
}

// Runtime-rank form of stage_point_t (host code and rank-generic kernels).
__host__ __device__ __forceinline__ int64_t stage_point(const StageDesc& d, uint32_t rank,
                                                        int32_t* coord) {
    return d.kind == 1 ? stage_point_t<0, 1>(d, rank, coord) : stage_point_t<0, 0>(d, rank, coord);
}

// Message rows of the GNN's embedding pass assembled in the MLP's operand
// staging (latec/gnn_predictor.py:843-871 message layout, d = 64, ds = 16):
// two-sided rows [e_neg | state_neg | e_pos | state_pos | logd_neg |
// logd_pos] (162 features), one-sided [e_side | state_side | sign |
// logd_side] (82). Row w of the launch is (pair pairs[w / K], axis w % K).
struct RowGather {
    const float* E;         // (B, N, K, 64) embedding field
    int64_t N;
    int K, b, M;
    const float* table;     // direction-state rows of 16
    const int32_t* pairs;   // pair ids l * M + m of the launch's rows
    const int32_t* nbr_p;   // (L, M) neighbours, -1 = none
    const int32_t* nbr_n;
    const float* logd_p;    // (L, M)
    const float* logd_n;
    const int32_t* sidx_p;  // (L, K) state rows
    const int32_t* sidx_n;
};

}  // namespace latec
