// Stage-constant rANS model fit on the device (native entropy mode).
//
// The reference fits one (scale level, mixture shape) per stage by a float32
// matrix-vector product of -log2 model weights with the stage histogram and
// an argmin (latec/rans.py:395-430). The native mode keeps that model space
// and selection rule but evaluates every cost deterministically in float64:
//   cost(shape, level) = pairwise sum over the power-of-two alphabet of
//                        f64(W[shape][level][sym]) * f64(count[sym]),
// products correctly rounded, partial sums combined over a perfect binary
// tree of adjacent terms. The first minimum over levels, then the first
// strictly smaller cost over shapes in dictionary order, wins.
#include <cuda_runtime.h>

#include "interp_kernels.cuh"
#include "latec_common.cuh"

namespace latec {

struct FitStage {
    uint64_t counts_off;  // stage counts in the counts buffer (alphabet entries)
    uint64_t w_table;     // device address: (n_shapes, 64, alphabet) float32 weights
    uint64_t seg_off;     // first histogram segment of the stage
    uint32_t n_segs;
    uint32_t alphabet;
    int32_t kexp;
    int32_t radius;
    uint32_t n_shapes;
    uint32_t stage;       // index into hist_total / results
    uint32_t shape_ids[24];
};

// count[sym] for the reduced alphabet: window bins summed over segments,
// bins outside the window from the per-code totals.
__global__ void k_fit_counts(const FitStage* __restrict__ fs, const uint32_t* __restrict__ hist_seg,
                             const uint32_t* __restrict__ hist_total, uint32_t* __restrict__ counts) {
    const FitStage& f = fs[blockIdx.y];
    const uint32_t sym = blockIdx.x * blockDim.x + threadIdx.x;
    if (sym >= f.alphabet) return;
    const int span = (1 << f.kexp) - 1;
    uint32_t v = 0;
    if (sym == 0) {
        for (uint32_t s = 0; s < f.n_segs; s++) v += hist_seg[(f.seg_off + s) * HBINS];
    } else {
        const int q = (int)sym - span - 1;
        if (q >= -span && q <= span) {
            if (q > -HWIN && q < HWIN) {
                for (uint32_t s = 0; s < f.n_segs; s++)
                    v += hist_seg[(f.seg_off + s) * HBINS + (q + HWIN)];
            } else {
                v = hist_total[(uint64_t)f.stage * 65536 + (uint32_t)(q + f.radius)];
            }
        }
    }
    counts[f.counts_off + sym] = v;
}

// One CTA per (stage, shape, level). The alphabet is split into 8 (or fewer)
// power-of-two spans of adjacent terms, one per warp; a warp walks its span 32
// terms at a time (coalesced loads), sums each 32 with a shuffle tree over
// adjacent lanes and folds the 32-term subtree sums in lane 0 with a
// binary-counter stack; the warp totals are then paired adjacently. Every
// partial sum is a node of the perfect binary tree over the alphabet.
__global__ void __launch_bounds__(256)
    k_fit_costs(const FitStage* __restrict__ fs, const uint32_t* __restrict__ counts,
                double* __restrict__ costs) {
    const uint32_t level = blockIdx.x, sh = blockIdx.y;
    const FitStage& f = fs[blockIdx.z];
    if (sh >= f.n_shapes) return;
    const uint32_t A = f.alphabet;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t span = A >= 256 ? A / 8 : (A >= 32 ? 32 : A);  // terms per warp
    const uint32_t n_warps = A / span;
    const uint32_t width = span < 32 ? span : 32;
    __shared__ double wsum[8];
    if (warp < (int)n_warps) {
        const float* W = (const float*)f.w_table + ((uint64_t)sh * 64 + level) * A;
        const uint32_t* cnt = counts + f.counts_off;
        double stack[12];
        int depth[12];
        int top = 0;
        const uint32_t a0 = warp * span;
        for (uint32_t base = a0; base < a0 + span; base += 32) {
            const uint32_t i = base + lane;
            // every term is >= +0 (weights are -log2 p, counts are counts): a
            // run of zero counts sums to exactly +0.0, so its weights need no
            // load (the histogram is narrow; the weight tables are not)
            const uint32_t c = (lane < (int)width) ? cnt[i] : 0u;
            double v = 0.0;
            if (__any_sync(0xffffffffu, c != 0u))
                v = (lane < (int)width) ? __dmul_rn((double)W[i], (double)c) : 0.0;
            for (uint32_t st = 1; st < width; st <<= 1) {
                const double o = __shfl_down_sync(0xffffffffu, v, st);
                if ((lane & (2 * st - 1)) == 0) v = __dadd_rn(v, o);
            }
            if (lane == 0) {
                int dd = 0;
                while (top > 0 && depth[top - 1] == dd) {
                    v = __dadd_rn(stack[--top], v);
                    dd++;
                }
                stack[top] = v;
                depth[top] = dd;
                top++;
            }
        }
        if (lane == 0) wsum[warp] = stack[0];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t st = 1; st < n_warps; st <<= 1)
            for (uint32_t w = 0; w + st < n_warps; w += 2 * st) wsum[w] = __dadd_rn(wsum[w], wsum[w + st]);
        costs[((uint64_t)blockIdx.z * 24 + sh) * 64 + level] = wsum[0];
    }
}

// One warp per stage: first argmin over levels (lower level wins ties), then
// the first strictly smaller cost over shapes in dictionary order.
__global__ void k_fit_pick(const FitStage* __restrict__ fs, int n, const double* __restrict__ costs,
                           double* __restrict__ out) {
    const int t = blockIdx.x;
    if (t >= n) return;
    const int lane = threadIdx.x;
    const FitStage& f = fs[t];
    double best = __longlong_as_double(0x7ff0000000000000ll);  // +inf
    int bl = 0, bs = 0;
    for (uint32_t sh = 0; sh < f.n_shapes; sh++) {
        const double* c = costs + ((uint64_t)t * 24 + sh) * 64;
        double v = c[lane];
        int l = lane;
        const double v2 = c[lane + 32];
        if (v2 < v) {
            v = v2;
            l = lane + 32;
        }
        for (int o = 16; o; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, v, o);
            const int ol = __shfl_xor_sync(0xffffffffu, l, o);
            if (ov < v || (ov == v && ol < l)) {
                v = ov;
                l = ol;
            }
        }
        if (v < best) {
            best = v;
            bl = l;
            bs = (int)f.shape_ids[sh];
        }
    }
    if (lane == 0) {
        out[3 * t] = best;
        out[3 * t + 1] = (double)bl;
        out[3 * t + 2] = (double)bs;
    }
}

}  // namespace latec

using namespace latec;

extern "C" {

uint64_t latec_fit_stage_size(void) { return sizeof(FitStage); }

int latec_fit_const(const void* stages_host, int32_t n, const uint32_t* hist_seg,
                    const uint32_t* hist_total, uint32_t* counts, double* costs, double* out,
                    void* workspace, uint64_t workspace_bytes, void* stream) {
    if (n < 1 || !stages_host || !hist_seg || !hist_total || !counts || !costs || !out)
        return LATEC_ERR_ARG;
    if (!workspace || workspace_bytes < sizeof(FitStage) * (uint64_t)n) return LATEC_ERR_WORKSPACE;
    const FitStage* h = (const FitStage*)stages_host;
    uint32_t max_a = 0, max_s = 0;
    for (int t = 0; t < n; t++) {
        if (h[t].alphabet < 4 || h[t].alphabet > 65536 || (h[t].alphabet & (h[t].alphabet - 1)) ||
            h[t].n_shapes < 1 || h[t].n_shapes > 24 || !h[t].w_table)
            return LATEC_ERR_ARG;
        max_a = h[t].alphabet > max_a ? h[t].alphabet : max_a;
        max_s = h[t].n_shapes > max_s ? h[t].n_shapes : max_s;
    }
    cudaStream_t st = (cudaStream_t)stream;
    FitStage* d = (FitStage*)workspace;
    if (cudaMemcpyAsync(d, h, sizeof(FitStage) * n, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    k_fit_counts<<<dim3((max_a + 255) / 256, n), 256, 0, st>>>(d, hist_seg, hist_total, counts);
    k_fit_costs<<<dim3(64, max_s, n), 256, 0, st>>>(d, counts, costs);
    k_fit_pick<<<n, 32, 0, st>>>(d, n, costs, out);
    count_launches(3);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // extern "C"
