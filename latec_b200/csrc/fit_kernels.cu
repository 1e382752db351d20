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

// One warp per (stage, shape, level), eight levels per CTA. Every cost is the
// sum over the perfect binary tree of the alphabet's terms (its size is a
// power of two; a term is >= +0: weights are -log2 p, counts are counts):
// * alphabets of 256 or more: lane l sums its contiguous run of A / 32
//   terms, visiting only the terms with a nonzero count (a shared bitmap of
//   the stage's counts): an all-zero subtree sums to +0, which leaves any
//   partial sum unchanged, so the run's tree is the tree of its nonzero terms
//   joined at their lowest common ancestors; the 32 run sums are then paired
//   adjacently by a shuffle tree. Lanes work independently.
// * smaller alphabets: 32 terms at a time, one per lane, summed by the
//   shuffle tree, the 32-term sums folded in order by a binary counter (a
//   subtree completes when its right half does).
// A zero count contributes +0 without its weight being loaded. The stage's
// counts sit in shared memory when they fit.
constexpr uint32_t FIT_SMEM_A = 4096;

__device__ __forceinline__ double fit_term(const float* __restrict__ W,
                                           const uint32_t* __restrict__ cnt, uint32_t i) {
    const uint32_t c = cnt[i];
    return c ? __dmul_rn((double)W[i], (double)c) : 0.0;
}

__global__ void __launch_bounds__(256)
    k_fit_costs(const FitStage* __restrict__ fs, const uint32_t* __restrict__ counts,
                double* __restrict__ costs) {
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
    // one bit per term with a nonzero count
    __shared__ uint32_t nzb[65536 / 32];
    if (A >= 256) {
        for (uint32_t wd = threadIdx.x; wd < A / 32; wd += 256) {
            uint32_t bits = 0;
            for (int k = 0; k < 32; k++) bits |= (cnt[wd * 32 + k] != 0u ? 1u : 0u) << k;
            nzb[wd] = bits;
        }
        __syncthreads();
    }
    const uint32_t level = blockIdx.x * 8 + warp;
    const float* W = (const float*)f.w_table + ((uint64_t)sh * 64 + level) * A;
    double stack[12];
    double v;
    if (A >= 256) {
        // lane l: the run [l R, (l + 1) R) of R = A / 32 terms, walked over
        // its nonzero counts only. A subtree whose terms are all +0 sums to
        // +0 and x + (+0) = x for every x >= +0, so the tree sum equals the
        // tree over the nonzero terms with the all-zero subtrees pruned: two
        // partial sums join at the lowest common ancestor of their positions
        // (level = bit length of pos_a ^ pos_b), left operand first.
        const uint32_t R = A / 32, a0 = lane * R;
        uint32_t spos[12];
        int top = 0;
        for (uint32_t w = a0 / 32; w < (a0 + R + 31) / 32; w++) {
            uint32_t bits = nzb[w];
            if (R < 32) bits = (bits >> (a0 & 31)) & ((1u << R) - 1u);
            while (bits) {
                const uint32_t p = (R < 32 ? a0 : w * 32) + (uint32_t)(__ffs(bits) - 1);
                bits &= bits - 1u;
                const double t = __dmul_rn((double)W[p], (double)cnt[p]);
                while (top >= 2 &&
                       (spos[top - 2] ^ spos[top - 1]) < (spos[top - 1] ^ p)) {
                    stack[top - 2] = __dadd_rn(stack[top - 2], stack[top - 1]);
                    spos[top - 2] = spos[top - 1];
                    top--;
                }
                stack[top] = t;
                spos[top] = p;
                top++;
            }
        }
        while (top >= 2) {
            stack[top - 2] = __dadd_rn(stack[top - 2], stack[top - 1]);
            top--;
        }
        v = top ? stack[0] : 0.0;
        for (uint32_t st = 1; st < 32; st <<= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v, st);
            if ((lane & (2 * st - 1)) == 0) v = __dadd_rn(v, o);
        }
    } else {
        const uint32_t width = A < 32 ? A : 32, chunks = (A + 31) / 32;
        for (uint32_t ch = 0; ch < chunks; ch++) {
            double x = lane < (int)width ? fit_term(W, cnt, ch * 32 + lane) : 0.0;
            for (uint32_t st = 1; st < width; st <<= 1) {
                const double o = __shfl_down_sync(0xffffffffu, x, st);
                if ((lane & (2 * st - 1)) == 0) x = __dadd_rn(x, o);
            }
            uint32_t d = 0;
            for (uint32_t cc = ch; cc & 1u; cc >>= 1) x = __dadd_rn(stack[d++], x);
            stack[d] = x;
        }
        v = stack[31 - __clz(chunks)];
    }
    if (lane == 0) costs[((uint64_t)blockIdx.z * 24 + sh) * 64 + level] = v;
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
    k_fit_costs<<<dim3(8, max_s, n), 256, 0, st>>>(d, counts, costs);
    k_fit_pick<<<n, 32, 0, st>>>(d, n, costs, out);
    count_launches(3);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // extern "C"
