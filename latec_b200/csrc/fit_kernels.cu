// Stage-constant rANS model fit on the device (native entropy mode).
//
// The reference fits one (scale level, mixture shape) per stage by a float32
// matrix-vector product of -log2 model weights with the stage histogram and
// an argmin (latec/rans.py:395-430). The native mode keeps that model space
// and selection rule but evaluates every cost exactly, in fixed point:
//   cost(shape, level) = sum over the power-of-two alphabet of
//                        rint(W[shape][level][sym] * 2^20) * count[sym]
// in 64-bit integers, so the result does not depend on the summation order.
// The first minimum over levels, then the first strictly smaller cost over
// shapes in dictionary order, wins.
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

// One warp per (stage, shape, level), eight levels per CTA: the cost is the
// exact integer sum over the alphabet of Wq[sym] * count[sym], Wq the
// float32 weight (-log2 p) in fixed point with FIT_FRAC_BITS fraction bits,
// rounded to nearest even (W * 2^20 is exact in float32, so the rounding is
// that of the conversion alone). Integer sums do not depend on their order:
// lanes take every 32nd term and the warp adds its lanes' sums. Every partial
// sum stays below 2^56 (Wq < 2^25, counts sum to at most 2^31). A run of 32
// zero counts is skipped by the whole warp, a zero count by its lane. The
// stage's counts sit in shared memory when they fit.
constexpr uint32_t FIT_SMEM_A = 8192;
constexpr int FIT_FRAC_BITS = 20;

__global__ void __launch_bounds__(256)
    k_fit_costs(const FitStage* __restrict__ fs, const uint32_t* __restrict__ counts,
                unsigned long long* __restrict__ costs) {
    const uint32_t sh = blockIdx.y;
    const FitStage& f = fs[blockIdx.z];
    if (sh >= f.n_shapes) return;
    const uint32_t A = f.alphabet;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ uint32_t sc[FIT_SMEM_A];
    const uint32_t* gcnt = counts + f.counts_off;
    const bool in_smem = A <= FIT_SMEM_A;
    if (in_smem) {
        for (uint32_t i = threadIdx.x; i < A; i += 256) sc[i] = gcnt[i];
        __syncthreads();
    }
    const uint32_t* cnt = in_smem ? sc : gcnt;
    const uint32_t level = blockIdx.x * 8 + warp;
    const float* W = (const float*)f.w_table + ((uint64_t)sh * 64 + level) * A;
    unsigned long long acc = 0;
    for (uint32_t base = 0; base < A; base += 32) {
        const uint32_t i = base + lane;
        const uint32_t c = i < A ? cnt[i] : 0u;
        if (!__any_sync(0xffffffffu, c != 0u)) continue;
        if (c) {
            const float scaled = W[i] * (float)(1 << FIT_FRAC_BITS);
            acc += (unsigned long long)(uint32_t)__float2ll_rn(scaled) * c;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) costs[((uint64_t)blockIdx.z * 24 + sh) * 64 + level] = acc;
}

// One warp per stage: first argmin over levels (lower level wins ties), then
// the first strictly smaller cost over shapes in dictionary order.
__global__ void k_fit_pick(const FitStage* __restrict__ fs, int n,
                           const unsigned long long* __restrict__ costs,
                           double* __restrict__ out) {
    const int t = blockIdx.x;
    if (t >= n) return;
    const int lane = threadIdx.x;
    const FitStage& f = fs[t];
    unsigned long long best = ~0ull;
    int bl = 0, bs = 0;
    bool any = false;
    for (uint32_t sh = 0; sh < f.n_shapes; sh++) {
        const unsigned long long* c = costs + ((uint64_t)t * 24 + sh) * 64;
        unsigned long long v = c[lane];
        int l = lane;
        const unsigned long long v2 = c[lane + 32];
        if (v2 < v) {
            v = v2;
            l = lane + 32;
        }
        for (int o = 16; o; o >>= 1) {
            const unsigned long long ov = __shfl_xor_sync(0xffffffffu, v, o);
            const int ol = __shfl_xor_sync(0xffffffffu, l, o);
            if (ov < v || (ov == v && ol < l)) {
                v = ov;
                l = ol;
            }
        }
        if (!any || v < best) {
            best = v;
            bl = l;
            bs = (int)f.shape_ids[sh];
            any = true;
        }
    }
    if (lane == 0) {
        // the cost in bits: the sum converted to float64 (nearest even), then
        // scaled by 2^-FIT_FRAC_BITS (exact)
        out[3 * t] = __ull2double_rn(best) * (1.0 / (double)(1 << FIT_FRAC_BITS));
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
    unsigned long long* icosts = reinterpret_cast<unsigned long long*>(costs);
    k_fit_costs<<<dim3(8, max_s, n), 256, 0, st>>>(d, counts, icosts);
    k_fit_pick<<<n, 32, 0, st>>>(d, n, icosts, out);
    count_launches(3);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // extern "C"
