// Per-point rANS support (the learned path's entropy stage): Laplacian scale
// to table level, the level-grouped symbol order of the single-stack stream,
// and the per-point model cost used to pick a dictionary shape.
//
// latec/rans.py:270-278 scale_to_level quantises float32 scales to 64 levels
// with float32 logs; on the device the same assignment is made by comparing
// against the 63 float32 thresholds where the level changes (found on the
// host by bisection over float32 bit patterns with the authoritative NumPy
// formula), so the result is identical without any device logarithm.
//
// latec/rans.py:546-616 codes the symbols of level 0 first, then level 1, ...,
// each group in index order. latec_level_order returns that order as a
// permutation (a stable counting sort on the 8-bit level), latec_permute
// applies it or its inverse.
#include <cuda_runtime.h>

#include "latec_common.cuh"

namespace latec {

namespace {

constexpr int PT_THREADS = 256;
constexpr int SORT_BLOCK = 4096;  // levels per counting-sort CTA
constexpr int SORT_WARPS = PT_THREADS / 32;
constexpr int SORT_PER_WARP = SORT_BLOCK / SORT_WARPS;  // 512
constexpr int NLEV = 256;                               // u8 level range

struct Thresholds {
    float t[64];  // t[0..n-2] ascending; level = #{k : t[k] <= v}
    int n;        // number of thresholds (levels - 1)
};

__global__ void __launch_bounds__(PT_THREADS)
    k_scale_levels(const float* __restrict__ scale, uint64_t n, const Thresholds th,
                   uint8_t* __restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * PT_THREADS + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * PT_THREADS) {
        const float v = scale[i];
        int lo = 0;  // thresholds below or at v (NaN compares false: level 0)
#pragma unroll
        for (int step = 32; step; step >>= 1)
            if (lo + step <= th.n && th.t[lo + step - 1] <= v) lo += step;
        out[i] = (uint8_t)lo;
    }
}

// Pass 1: per-CTA level counts (CTA-major: counts[b * NLEV + level]).
__global__ void __launch_bounds__(PT_THREADS)
    k_level_counts(const uint8_t* __restrict__ lv, uint64_t n, uint32_t* __restrict__ counts) {
    __shared__ uint32_t h[NLEV];
    for (int k = threadIdx.x; k < NLEV; k += PT_THREADS) h[k] = 0;
    __syncthreads();
    const uint64_t b0 = (uint64_t)blockIdx.x * SORT_BLOCK;
    for (int k = threadIdx.x; k < SORT_BLOCK; k += PT_THREADS) {
        const uint64_t i = b0 + k;
        if (i < n) atomicAdd(&h[lv[i]], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < NLEV; k += PT_THREADS)
        counts[(uint64_t)blockIdx.x * NLEV + k] = h[k];
}

// Pass 2 (one CTA): level-major exclusive offsets, offs[b * NLEV + level] =
// #{symbols of lower levels} + #{symbols of this level in earlier CTAs}.
// Thread t owns level t (NLEV == PT_THREADS): a serial walk over the CTAs per
// level, then a scan of the level totals.
__global__ void __launch_bounds__(PT_THREADS)
    k_level_offsets(const uint32_t* __restrict__ counts, uint32_t n_blocks,
                    uint32_t* __restrict__ offs) {
    __shared__ uint32_t tot[NLEV];
    const int l = threadIdx.x;
    uint32_t run = 0;
    for (uint32_t b = 0; b < n_blocks; b++) {
        const uint32_t c = counts[(uint64_t)b * NLEV + l];
        offs[(uint64_t)b * NLEV + l] = run;
        run += c;
    }
    tot[l] = run;
    __syncthreads();
    for (int o = 1; o < NLEV; o <<= 1) {
        const uint32_t v = l >= o ? tot[l - o] : 0u;
        __syncthreads();
        tot[l] += v;
        __syncthreads();
    }
    const uint32_t base = tot[l] - run;
    for (uint32_t b = 0; b < n_blocks; b++) offs[(uint64_t)b * NLEV + l] += base;
}

// Pass 3: stable scatter. Each warp owns 512 consecutive symbols of the CTA;
// per-warp level counts are scanned across the warps, then each warp walks its
// run 32 symbols at a time, ranking equal levels with a match mask.
__global__ void __launch_bounds__(PT_THREADS)
    k_level_scatter(const uint8_t* __restrict__ lv, uint64_t n, const uint32_t* __restrict__ offs,
                    uint32_t* __restrict__ order) {
    __shared__ uint32_t wc[SORT_WARPS][NLEV];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = lane; k < NLEV; k += 32) wc[w][k] = 0;
    __syncwarp();
    const uint64_t w0 = (uint64_t)blockIdx.x * SORT_BLOCK + (uint64_t)w * SORT_PER_WARP;
    for (int k = 0; k < SORT_PER_WARP; k += 32) {
        const uint64_t i = w0 + k + lane;
        const int l = i < n ? (int)lv[i] : -1;
        const unsigned same = __match_any_sync(0xffffffffu, l);
        if (l >= 0 && lane == __ffs(same) - 1) wc[w][l] += __popc(same);
        __syncwarp();
    }
    __syncthreads();
    // exclusive scan over warps, per level, plus the CTA's offset
    for (int l = threadIdx.x; l < NLEV; l += PT_THREADS) {
        uint32_t run = offs[(uint64_t)blockIdx.x * NLEV + l];
        for (int ww = 0; ww < SORT_WARPS; ww++) {
            const uint32_t c = wc[ww][l];
            wc[ww][l] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int k = 0; k < SORT_PER_WARP; k += 32) {
        const uint64_t i = w0 + k + lane;
        const int l = i < n ? (int)lv[i] : -1;
        const unsigned same = __match_any_sync(0xffffffffu, l);
        if (l >= 0) {
            const uint32_t pos = wc[w][l] + __popc(same & ((1u << lane) - 1u));
            order[pos] = (uint32_t)i;
        }
        __syncwarp();
        if (l >= 0 && lane == __ffs(same) - 1) wc[w][l] += __popc(same);
        __syncwarp();
    }
}

template <typename E>
__global__ void __launch_bounds__(PT_THREADS)
    k_permute(const E* __restrict__ src, const uint32_t* __restrict__ order, uint64_t n,
              E* __restrict__ dst, int inverse) {
    for (uint64_t j = (uint64_t)blockIdx.x * PT_THREADS + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * PT_THREADS) {
        const uint32_t i = order[j];
        if (inverse) dst[i] = src[j];
        else dst[j] = src[i];
    }
}

// Per-point model cost: bits = sum of (24 - log2 p), p the integer frequency
// of the symbol in its level's CDF row (latec/rans.py:332-357). Per-CTA
// partial sums in a fixed order; the host adds the partials in CTA order.
__global__ void __launch_bounds__(PT_THREADS)
    k_point_bits(const uint16_t* __restrict__ codes, const uint8_t* __restrict__ lv, uint64_t n,
                 const uint32_t* __restrict__ cdf, uint32_t alphabet, int radius, int kexp,
                 double* __restrict__ partial, uint32_t* __restrict__ err) {
    __shared__ double red[PT_THREADS];
    double s = 0.0;
    const uint64_t per = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t a = (uint64_t)blockIdx.x * per, e = a + per < n ? a + per : n;
    for (uint64_t i = a + threadIdx.x; i < e; i += PT_THREADS) {
        const uint32_t c = codes[i];
        const uint32_t sym = c ? (uint32_t)((int)c - radius + (1 << kexp)) : 0u;
        if (sym >= alphabet) {
            atomicOr(err, 1u);
            continue;
        }
        const uint32_t* row = cdf + (uint64_t)lv[i] * (alphabet + 1);
        const uint32_t p = row[sym + 1] - row[sym];
        s = __dadd_rn(s, __dsub_rn(24.0, log2((double)p)));
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = PT_THREADS / 2; o; o >>= 1) {
        if (threadIdx.x < (unsigned)o) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Dictionary-shape cost over sampled points (every `step`-th symbol) for one
// shape per blockIdx.y: p = weights[level][sym], mixed with the level `d`
// steps broader by weight `w` (latec/rans.py:204-243), cost = sum -log2(max(p,
// floor)). weights: (n_levels, alphabet) float64.
struct ShapeSpec {
    int d[24];
    double w[24];
    int n_shapes;
};

__global__ void __launch_bounds__(PT_THREADS)
    k_shape_costs(const uint16_t* __restrict__ codes, const uint8_t* __restrict__ lv, uint64_t n,
                  uint64_t step, const double* __restrict__ weights, uint32_t alphabet,
                  int n_levels, int radius, int kexp, double floor_p, const ShapeSpec sp,
                  double* __restrict__ partial) {
    __shared__ double red[PT_THREADS];
    const int sh = blockIdx.y;
    const int d = sp.d[sh];
    const double w = sp.w[sh], w1 = __dsub_rn(1.0, sp.w[sh]);
    const uint64_t m = (n + step - 1) / step;  // sampled symbols
    const uint64_t per = (m + gridDim.x - 1) / gridDim.x;
    const uint64_t a = (uint64_t)blockIdx.x * per, e = a + per < m ? a + per : m;
    double s = 0.0;
    for (uint64_t j = a + threadIdx.x; j < e; j += PT_THREADS) {
        const uint64_t i = j * step;
        const uint32_t c = codes[i];
        uint32_t sym = c ? (uint32_t)((int)c - radius + (1 << kexp)) : 0u;
        if (sym >= alphabet) sym = 0;
        const int l = lv[i];
        double p = weights[(uint64_t)l * alphabet + sym];
        if (w != 0.0) {
            const int lb = l + d < n_levels - 1 ? l + d : n_levels - 1;
            const double broad = weights[(uint64_t)lb * alphabet + sym];
            p = __dadd_rn(__dmul_rn(w1, p), __dmul_rn(w, broad));
        }
        s = __dadd_rn(s, -log2(fmax(p, floor_p)));
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = PT_THREADS / 2; o; o >>= 1) {
        if (threadIdx.x < (unsigned)o) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[(uint64_t)sh * gridDim.x + blockIdx.x] = red[0];
}

uint32_t grid_for(uint64_t n) {
    uint64_t b = (n + PT_THREADS - 1) / PT_THREADS;
    if (b > 148ull * 16) b = 148ull * 16;
    return (uint32_t)(b ? b : 1);
}

}  // namespace
}  // namespace latec

using namespace latec;

extern "C" {

int latec_scale_levels(const float* scale, uint64_t n, const float* thresholds, int32_t n_levels,
                       uint8_t* levels, void* stream) {
    if (n_levels < 1 || n_levels > 64 || !thresholds || (n && (!scale || !levels)))
        return LATEC_ERR_ARG;
    Thresholds th;
    th.n = n_levels - 1;
    for (int k = 0; k < 64; k++) th.t[k] = k < th.n ? thresholds[k] : 0.0f;
    for (int k = 1; k < th.n; k++)
        if (!(th.t[k - 1] <= th.t[k])) return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    k_scale_levels<<<grid_for(n), PT_THREADS, 0, (cudaStream_t)stream>>>(scale, n, th, levels);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

uint64_t latec_level_order_workspace_bytes(uint64_t n) {
    const uint64_t nb = (n + SORT_BLOCK - 1) / SORT_BLOCK;
    return 2 * sizeof(uint32_t) * NLEV * (nb ? nb : 1);
}

int latec_level_order(const uint8_t* levels, uint64_t n, uint32_t* order, void* workspace,
                      uint64_t workspace_bytes, void* stream) {
    if (n > 0xffffffffull || (n && (!levels || !order))) return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    if (!workspace || workspace_bytes < latec_level_order_workspace_bytes(n))
        return LATEC_ERR_WORKSPACE;
    const uint32_t nb = (uint32_t)((n + SORT_BLOCK - 1) / SORT_BLOCK);
    uint32_t* counts = (uint32_t*)workspace;
    uint32_t* offs = counts + (uint64_t)NLEV * nb;
    cudaStream_t st = (cudaStream_t)stream;
    k_level_counts<<<nb, PT_THREADS, 0, st>>>(levels, n, counts);
    k_level_offsets<<<1, PT_THREADS, 0, st>>>(counts, nb, offs);
    k_level_scatter<<<nb, PT_THREADS, 0, st>>>(levels, n, offs, order);
    count_launches(3);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

int latec_permute(const void* src, int32_t elem, const uint32_t* order, uint64_t n, void* dst,
                  int32_t inverse, void* stream) {
    if (n && (!src || !order || !dst)) return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t g = grid_for(n);
    switch (elem) {
        case 1: k_permute<uint8_t><<<g, PT_THREADS, 0, st>>>((const uint8_t*)src, order, n, (uint8_t*)dst, inverse); break;
        case 2: k_permute<uint16_t><<<g, PT_THREADS, 0, st>>>((const uint16_t*)src, order, n, (uint16_t*)dst, inverse); break;
        case 4: k_permute<uint32_t><<<g, PT_THREADS, 0, st>>>((const uint32_t*)src, order, n, (uint32_t*)dst, inverse); break;
        default: return LATEC_ERR_ARG;
    }
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

int latec_point_bits(const uint16_t* codes, const uint8_t* levels, uint64_t n, const uint32_t* cdf,
                     uint32_t alphabet, int32_t radius, int32_t kexp, double* partial,
                     int32_t n_partial, uint32_t* err, void* stream) {
    if (n && (!codes || !levels || !cdf || !partial || !err)) return LATEC_ERR_ARG;
    if (n_partial < 1 || alphabet < 2 || kexp < 0 || kexp > 15) return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    k_point_bits<<<n_partial, PT_THREADS, 0, (cudaStream_t)stream>>>(codes, levels, n, cdf, alphabet,
                                                                   radius, kexp, partial, err);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

int latec_shape_costs(const uint16_t* codes, const uint8_t* levels, uint64_t n, uint64_t step,
                      const double* weights, uint32_t alphabet, int32_t n_levels, int32_t radius,
                      int32_t kexp, double floor_p, const int32_t* shape_d, const double* shape_w,
                      int32_t n_shapes, double* partial, int32_t n_partial, void* stream) {
    if (n && (!codes || !levels || !weights || !partial)) return LATEC_ERR_ARG;
    if (n_shapes < 1 || n_shapes > 24 || !shape_d || !shape_w || n_partial < 1 || step < 1 ||
        n_levels < 1 || n_levels > 256 || kexp < 0 || kexp > 15)
        return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    ShapeSpec sp;
    sp.n_shapes = n_shapes;
    for (int k = 0; k < 24; k++) {
        sp.d[k] = k < n_shapes ? shape_d[k] : 0;
        sp.w[k] = k < n_shapes ? shape_w[k] : 0.0;
    }
    k_shape_costs<<<dim3(n_partial, n_shapes), PT_THREADS, 0, (cudaStream_t)stream>>>(
        codes, levels, n, step, weights, alphabet, n_levels, radius, kexp, floor_p, sp, partial);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // extern "C"
