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
    FastDiv size_div[MAXD];   // kind 0: class extent per axis
    FastDiv g_div[MAXD][MAXD + 1];  // kind 1: G[j][r]
    uint32_t f_even[MAXD][MAXD + 1];  // kind 1: F[j+1][r]
};

// Decode a stage-local rank into grid coordinates; returns the flat grid index.
__host__ __device__ __forceinline__ int64_t stage_coords(const StageDesc& d, uint32_t rank,
                                                int32_t* coord) {
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
// coordinates stay in registers), KIND fixes the stage layout; ND == 0 falls
// back to the runtime rank.
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

}  // namespace latec
