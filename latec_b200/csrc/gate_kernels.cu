// Scale-gated interpolation fallback of the learned codec
// (latec/gnn_codec.py:386-462, 776-1000): per stage the encoder scores the GNN
// prediction against three classical candidates (cubic axis-average,
// first-odd-axis linear, last-odd-axis linear) with an rANS-aligned Laplace
// rate, per bucket of the model's scale b relative to eb * 2^T, T = 2..13,
// and for scale shifts 0 / 2 / 4 / 6; the host then picks the
// (candidate, side, T, shift) that codes fewest bits, or none. Applying a
// choice replaces the prediction by the candidate and the scale by
// b * 2^-shift on one side of the threshold, identically in the decoder.
//
// The per-bucket sums are kept in fixed point (2^-20 bit units; lanes of a
// warp with the same bucket are summed by one integer warp reduction, then
// 64-bit integer atomics), so the choice does not depend on the order in
// which threads add: encoder runs are deterministic.
#include <cuda_runtime.h>

#include <cstdint>

#include "latec_common.cuh"

namespace latec {
namespace {

constexpr int GT = 256;
constexpr int GATE_NT = 12;              // thresholds eb * 2^T, T = 2 .. 13
constexpr int GATE_NB = GATE_NT + 1;     // scale buckets
constexpr int GATE_NS = 4;               // shifts 0, 2, 4, 6
constexpr int GATE_NK = 3;               // classical candidates
constexpr int GATE_R = 1 + GATE_NK * GATE_NS;
constexpr double FIX = 1048576.0;        // 2^20 fixed-point units per bit (56 bits x 32 lanes < 2^32)

// Scale snapped to the gate's 64-level log grid: the number of float32
// boundaries <= s picks the grid value.
__device__ __forceinline__ double snap(float s, const float* __restrict__ thr,
                                       const double* __restrict__ grid) {
    int lo = 0, hi = 63;  // count of thr[j] <= s, thr ascending
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (thr[mid] <= s) lo = mid + 1; else hi = mid;
    }
    return grid[lo];
}

// Code length in bits of a residual of magnitude absr under Laplace(bq) with
// the 2 eb cell: capped at the 24-bit table precision; a code at or past the
// radius is an outlier (marker + raw float32: 56 bits).
__device__ __forceinline__ double cell_bits(double absr, double bq, double eb, int radius) {
    const double k = rint(absr / (2.0 * eb));
    double p;
    if (k == 0.0) p = -expm1(-eb / bq);
    else p = 0.5 * exp(-((2.0 * k - 1.0) * eb / bq)) * -expm1(-2.0 * eb / bq);
    const double bits = fmin(-log2(p), 24.0);
    return k >= (double)radius ? 56.0 : bits;
}

__global__ void __launch_bounds__(GT)
    k_gate_costs(int64_t n, const float* __restrict__ x, const float* __restrict__ mu,
                 const float* __restrict__ ip0, const float* __restrict__ ip1,
                 const float* __restrict__ ip2, const float* __restrict__ b, double eb,
                 int radius, const float* __restrict__ thr, const double* __restrict__ grid,
                 unsigned long long* __restrict__ sums) {
    __shared__ unsigned long long acc[GATE_R * GATE_NB];
    __shared__ float s_thr[63];
    __shared__ double s_grid[64];
    for (int i = threadIdx.x; i < GATE_R * GATE_NB; i += GT) acc[i] = 0ull;
    for (int i = threadIdx.x; i < 63; i += GT) s_thr[i] = thr[i];
    for (int i = threadIdx.x; i < 64; i += GT) s_grid[i] = grid[i];
    __syncthreads();
    const float* ips[GATE_NK] = {ip0, ip1, ip2};
    const int lane = threadIdx.x & 31;
    // uniform trip count so every lane reaches the warp collectives
    for (int64_t base = (int64_t)blockIdx.x * GT; base < n; base += (int64_t)gridDim.x * GT) {
        const int64_t i = base + threadIdx.x;
        const bool act = i < n;
        const float bi = act ? b[i] : 1.0f;
        const double bd = (double)bi;
        int bucket = GATE_NB;  // inactive lanes form their own group
        if (act) {
            bucket = 0;
#pragma unroll
            for (int t = 0; t < GATE_NT; t++) bucket += (eb * (double)(1 << (t + 2)) < bd) ? 1 : 0;
        }
        const unsigned grp = __match_any_sync(0xffffffffu, bucket);
        const bool leader = act && lane == __ffs(grp) - 1;
        const double xv = act ? (double)x[i] : 0.0;
        auto add = [&](int row, double bits) {
            const unsigned v = act ? (unsigned)llrint(bits * FIX) : 0u;
            const unsigned s = __reduce_add_sync(grp, v);
            if (leader) atomicAdd(&acc[row * GATE_NB + bucket], (unsigned long long)s);
        };
        add(0, act ? cell_bits(fabs(xv - (double)mu[i]), snap(bi, s_thr, s_grid), eb, radius) : 0.0);
        double bq[GATE_NS];
#pragma unroll
        for (int s = 0; s < GATE_NS; s++) bq[s] = snap(bi * exp2f(-2.0f * s), s_thr, s_grid);
#pragma unroll
        for (int k = 0; k < GATE_NK; k++) {
            if (!ips[k]) continue;  // uniform: a kernel argument
            const double r = act ? fabs(xv - (double)ips[k][i]) : 0.0;
#pragma unroll
            for (int s = 0; s < GATE_NS; s++)
                add(1 + k * GATE_NS + s, act ? cell_bits(r, bq[s], eb, radius) : 0.0);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < GATE_R * GATE_NB; i += GT)
        if (acc[i]) atomicAdd(&sums[i], acc[i]);
}

__global__ void __launch_bounds__(GT)
    k_gate_apply(int64_t n, float* __restrict__ mu, float* __restrict__ b,
                 const float* __restrict__ ip, double thr, float mult, int high) {
    const int64_t i = (int64_t)blockIdx.x * GT + threadIdx.x;
    if (i >= n) return;
    const float bi = b[i];
    const bool below = (double)bi < thr;
    if (high ? !below : below) {
        mu[i] = ip[i];
        b[i] = bi * mult;
    }
}

// The gate's choice on the device (one thread, the 13 x 13 sums table): per
// row the cumulative sums over the scale buckets; a low-side split at column
// c costs tot - gnn[c] + cand[c], a high-side split gnn[c] + cand[last] -
// cand[c]; the first least cost over (side, row, column) in that order wins
// when it is below the GNN's total, else the word is 0. Integer arithmetic,
// the same values as the host rule's exact float64 sums.
__global__ void k_gate_choose(const unsigned long long* __restrict__ sums,
                              uint32_t* __restrict__ word) {
    if (threadIdx.x || blockIdx.x) return;
    long long cum[GATE_R][GATE_NB];
    for (int r = 0; r < GATE_R; r++) {
        long long run = 0;
        for (int c = 0; c < GATE_NB; c++) {
            run += (long long)sums[r * GATE_NB + c];
            cum[r][c] = run;
        }
    }
    const long long tot = cum[0][GATE_NB - 1];
    const int rows = GATE_NK * GATE_NS;
    long long best = 0;
    int fi = -1;
    for (int side = 0; side < 2; side++)
        for (int r = 0; r < rows; r++)
            for (int c = 0; c < GATE_NT; c++) {
                const long long cost = side == 0
                                           ? tot - cum[0][c] + cum[1 + r][c]
                                           : cum[0][c] + (cum[1 + r][GATE_NB - 1] - cum[1 + r][c]);
                if (fi < 0 || cost < best) {
                    best = cost;
                    fi = (side * rows + r) * GATE_NT + c;
                }
            }
    uint32_t w = 0;
    if (fi >= 0 && best < tot) {
        const int row = fi / GATE_NT, side_row = row % rows;
        const uint32_t kind = (uint32_t)(side_row / GATE_NS + 1), high = row >= rows ? 1u : 0u;
        const uint32_t T = (uint32_t)(2 + fi % GATE_NT), shift = (uint32_t)(2 * (side_row % GATE_NS));
        w = (high << 10) | (kind << 8) | (T << 4) | shift;
    }
    *word = w;
}

// k_gate_apply with its parameters from a gate word in device memory.
__global__ void __launch_bounds__(GT)
    k_gate_apply_word(int64_t n, float* __restrict__ mu, float* __restrict__ b,
                      const float* __restrict__ ip0, const float* __restrict__ ip1,
                      const float* __restrict__ ip2, double eb, const uint32_t* __restrict__ word) {
    const uint32_t w = *word;
    const uint32_t kind = (w >> 8) & 3u, T = (w >> 4) & 15u, shift = w & 15u;
    if (!kind || !T) return;
    const int64_t i = (int64_t)blockIdx.x * GT + threadIdx.x;
    if (i >= n) return;
    const float* ip = kind == 1 ? ip0 : (kind == 2 ? ip1 : ip2);
    const double thr = eb * (double)(1u << T);
    const float mult = ldexpf(1.0f, -(int)shift);
    const float bi = b[i];
    const bool below = (double)bi < thr;
    if ((w >> 10) & 1u ? !below : below) {
        mu[i] = ip[i];
        b[i] = bi * mult;
    }
}

}  // namespace
}  // namespace latec

using namespace latec;

extern "C" {

// sums: GATE_R x GATE_NB unsigned 64-bit fixed-point bit counts (2^-20 bit
// units), zeroed by the caller; row 0 the GNN, row 1 + 4 k + s candidate k
// (0 cubic, 1 first-axis linear, 2 last-axis linear; NULL = not scored) with
// scale shift 2 s; column = the number of thresholds eb * 2^T (T = 2..13)
// below b. thr (63 float32) / grid (64 float64): the gate's scale grid.
int latec_gate_costs(int64_t n, const float* x, const float* mu, const float* ip0,
                     const float* ip1, const float* ip2, const float* b, double eb, int32_t radius,
                     const float* thr, const double* grid, uint64_t* sums, void* stream) {
    if (n < 0 || !(eb > 0.0) || radius < 1 || !thr || !grid || !sums ||
        (n && (!x || !mu || !b)))
        return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    int64_t blocks = (n + GT - 1) / GT;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_gate_costs<<<(unsigned)blocks, GT, 0, (cudaStream_t)stream>>>(
        n, x, mu, ip0, ip1, ip2, b, eb, radius, thr, grid, (unsigned long long*)sums);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

// Apply a gate word: where b < eb * 2^T (high = 0) or b >= eb * 2^T
// (high = 1), mu = ip and b *= 2^-shift. T <= 0 leaves everything unchanged.
int latec_gate_apply(int64_t n, float* mu, float* b, const float* ip, double eb, int32_t T,
                     int32_t shift, int32_t high, void* stream) {
    if (n < 0 || shift < 0 || shift > 30 || T > 30) return LATEC_ERR_ARG;
    if (!n || T <= 0) return LATEC_OK;
    if (!mu || !b || !ip || !(eb > 0.0)) return LATEC_ERR_ARG;
    k_gate_apply<<<(unsigned)((n + GT - 1) / GT), GT, 0, (cudaStream_t)stream>>>(
        n, mu, b, ip, eb * (double)(1 << T), exp2f(-(float)shift), high ? 1 : 0);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

// latec_gate_costs' sums -> the gate word (the host rule of gate_choose in
// latec_b200/gnn_codec.py) written to *word, then that gate applied; ip0..2
// the three candidates (cubic, first-axis linear, last-axis linear). Nothing
// returns to the host: the word stays on the device.
int latec_gate_choose_apply(int64_t n, const uint64_t* sums, float* mu, float* b, const float* ip0,
                            const float* ip1, const float* ip2, double eb, uint32_t* word,
                            void* stream) {
    if (n < 0 || !sums || !word || !(eb > 0.0) ||
        (n && (!mu || !b || !ip0 || !ip1 || !ip2)))
        return LATEC_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    k_gate_choose<<<1, 32, 0, st>>>((const unsigned long long*)sums, word);
    if (n)
        k_gate_apply_word<<<(unsigned)((n + GT - 1) / GT), GT, 0, st>>>(n, mu, b, ip0, ip1, ip2,
                                                                       eb, word);
    count_launches(n ? 2 : 1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

// The gate of a word already on the device (a finest-level word reused).
int latec_gate_apply_word(int64_t n, float* mu, float* b, const float* ip0, const float* ip1,
                          const float* ip2, double eb, const uint32_t* word, void* stream) {
    if (n < 0 || !word || !(eb > 0.0) || (n && (!mu || !b || !ip0 || !ip1 || !ip2)))
        return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    k_gate_apply_word<<<(unsigned)((n + GT - 1) / GT), GT, 0, (cudaStream_t)stream>>>(
        n, mu, b, ip0, ip1, ip2, eb, word);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // extern "C"
