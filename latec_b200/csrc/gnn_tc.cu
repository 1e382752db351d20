// Fused two-layer MLP of the GNN message pass on the 5th-generation tensor
// cores: Y = W2 * gelu(W1 * X + b1) + b2 for rows of X, with BF16 operands in
// shared memory and FP32 accumulators in tensor memory (tcgen05).
//
// One persistent CTA of 8 warps per SM. W1 (N1 x K1) and W2 (N2 x N1) are
// staged once per CTA in shared memory; then for every 128-row tile:
//   1. the 128 rows of X (float32, any row stride) are rounded to BF16 into
//      shared memory (zero-padded to K1p, a multiple of 16);
//   2. one elected thread issues K1p / 16 tcgen05.mma (M 128, N N1, K 16)
//      into TMEM columns [0, N1) and commits them to an mbarrier;
//   3. each warp reads its 32 TMEM lanes (rows) back with tcgen05.ld, adds b1,
//      applies GELU and writes the BF16 hidden row to shared memory: the A
//      operand of layer 2;
//   4. N1 / 16 tcgen05.mma into TMEM columns [N1, N1 + N2), commit, wait;
//   5. the epilogue adds b2 and stores the first ny columns of the float32
//      row of Y.
// Instances: N1 x N2 = 128 x 64 (the message and mix MLPs) and 64 x 32 (the
// line pool's key MLP, 64 -> 64 -> 1 with the output layer zero-padded to 32
// rows; ny = 1 stores the key alone). With NV > 0 layer 1 carries NV more
// output columns that skip the activation and layer 2: they are stored, with
// their bias, as a second float32 output (the line pool's value projection
// rides on its key MLP's first layer: 64 + 64 columns from one A operand).
// Operands use the no-swizzle K-major canonical layout: 8 x 16-byte core
// matrices, row groups 128 bytes apart (SBO) and 8-element K chunks R * 16
// bytes apart (LBO), R the operand's rows. Weights arrive pre-packed in that
// layout (latec_gnn_pack_bf16). Every mbarrier wait has an iteration limit;
// on expiry the kernel records an error, stops issuing and frees its TMEM.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "latec_common.cuh"
#include "tc_sm100.cuh"

namespace latec {
namespace {

constexpr int TC_THREADS = 256;
constexpr int TC_M = 128;

__device__ __forceinline__ float gelu_tc(float x) {
    return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}

struct GatherRow {
    const float* e0;  // first embedding row (negative side / the side)
    const float* s0;  // its state row
    const float* e1;  // positive side's embedding row (two-sided)
    const float* s1;
    float t0, t1;     // the trailing scalars
    bool live;
};

template <int GATHER>
__device__ __forceinline__ void gather_row(const RowGather& rg, int w, GatherRow& g) {
    g.live = w >= 0;
    g.e0 = g.s0 = g.e1 = g.s1 = nullptr;
    g.t0 = g.t1 = 0.0f;
    if (!g.live) return;
    const int p = w / rg.K, k = w - (w / rg.K) * rg.K;
    const int pair = rg.pairs[p];
    const int l = pair / rg.M;
    const int64_t rowbase = (int64_t)rg.b * rg.N;
    if (GATHER == 2) {
        const int64_t in_ = rg.nbr_n[pair], ip = rg.nbr_p[pair];
        g.e0 = rg.E + ((rowbase + in_) * rg.K + k) * 64;
        g.s0 = rg.table + (int64_t)rg.sidx_n[l * rg.K + k] * 16;
        g.e1 = rg.E + ((rowbase + ip) * rg.K + k) * 64;
        g.s1 = rg.table + (int64_t)rg.sidx_p[l * rg.K + k] * 16;
        g.t0 = rg.logd_n[pair];
        g.t1 = rg.logd_p[pair];
    } else {
        const bool pos = rg.nbr_p[pair] >= 0;
        const int64_t nb = pos ? rg.nbr_p[pair] : rg.nbr_n[pair];
        g.e0 = rg.E + ((rowbase + nb) * rg.K + k) * 64;
        g.s0 = rg.table + (int64_t)(pos ? rg.sidx_p[l * rg.K + k] : rg.sidx_n[l * rg.K + k]) * 16;
        g.t0 = pos ? 1.0f : -1.0f;
        g.t1 = pos ? rg.logd_p[pair] : rg.logd_n[pair];
    }
}

// Features [8c, 8c + 8) of a gathered row (zero past the row or the width).
// Embedding rows are 256-byte aligned (float4 loads); state rows are read
// element by element (the table sits at any float offset of the parameters).
template <int GATHER>
__device__ __forceinline__ void gather_chunk(const GatherRow& g, int c, int chunks, float* v) {
#pragma unroll
    for (int e = 0; e < 8; e++) v[e] = 0.0f;
    if (!g.live || c >= chunks) return;
    const float* src = nullptr;
    bool state = false;
    if (c < 8) {
        src = g.e0 + 8 * c;
    } else if (c < 10) {
        src = g.s0 + 8 * (c - 8);
        state = true;
    } else if (GATHER == 2 && c < 18) {
        src = g.e1 + 8 * (c - 10);
    } else if (GATHER == 2 && c < 20) {
        src = g.s1 + 8 * (c - 18);
        state = true;
    } else if (c == (GATHER == 2 ? 20 : 10)) {
        v[0] = g.t0;
        v[1] = g.t1;
        return;
    } else {
        return;
    }
    if (state) {
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] = src[e];
    } else {
        const float4 a = *(const float4*)src, b = *(const float4*)(src + 4);
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
        v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
    }
}

// N1 = hidden width, N2 = output width (multiples of 32). 256 threads: thread t
// converts K chunks of row t % 128 (rows of a warp are 16 bytes apart in the
// canonical layout: conflict-free stores); warp w reads TMEM lanes
// 32 (w % 4) .. + 31, warpgroup w / 4 half of the columns.
template <int N1, int N2, int NV, int GATHER>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_mlp2_tc(const float* __restrict__ X, int ldx, int rows, int k1, int k1p,
              const __nv_bfloat16* __restrict__ w1p, const float* __restrict__ b1,
              const __nv_bfloat16* __restrict__ w2p, const float* __restrict__ b2,
              float* __restrict__ Y, int ldy, int ny, const float* __restrict__ bv,
              float* __restrict__ V, int ldv, const RowGather rg, uint32_t* __restrict__ err) {
    constexpr int NL1 = N1 + NV;  // layer 1 outputs: hidden, then the side output
    static_assert(N1 % 32 == 0 && NV % 32 == 0 && N2 % 32 == 0 && NL1 + N2 <= 512,
                  "MLP widths");
    extern __shared__ __align__(128) uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __nv_bfloat16* sw1 = (__nv_bfloat16*)smem_raw;             // NL1 x k1p
    __nv_bfloat16* sw2 = sw1 + (size_t)NL1 * k1p;               // N2 x N1
    __nv_bfloat16* sa = sw2 + (size_t)N2 * N1;                  // 128 x k1p (then Y staging)
    __nv_bfloat16* sh = sa + (size_t)TC_M * k1p;                // 128 x N1
    float* sy = (float*)sa;                                     // 128 x (N2 + 1) float32
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quarter = warp & 3, half = warp >> 2;

    {  // stage the packed weights (16-byte copies)
        const int4* s1 = (const int4*)w1p;
        int4* d1 = (int4*)sw1;
        for (int i = tid; i < NL1 * k1p / 8; i += TC_THREADS) d1[i] = s1[i];
        const int4* s2 = (const int4*)w2p;
        int4* d2 = (int4*)sw2;
        for (int i = tid; i < N2 * N1 / 8; i += TC_THREADS) d2[i] = s2[i];
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    constexpr uint32_t TMEM_COLS = (NL1 + N2) <= 128 ? 128 : ((NL1 + N2) <= 256 ? 256 : 512);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    const uint32_t mb = smem_u32(&mbar);
    uint32_t phase = 0;
    bool ok = true;
    const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
    const int trow = quarter * 32 + lane;  // TMEM lane (tile row) of this thread
    const int n_tiles = (rows + TC_M - 1) / TC_M;
    const int chunks = k1p / 8;
    // rows start on 16-byte boundaries and ldx >= round_up(k1, 4): a float4
    // starting below k1 stays inside its row
    const bool vec4 = (ldx % 4) == 0 && ((uintptr_t)X % 16) == 0 && ldx >= ((k1 + 3) & ~3);

    for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        const int r0 = t * TC_M;
        // 1. rows of X -> BF16 A operand: thread handles row tid % 128,
        //    K chunks tid / 128, + 2, + 4, ...; four chunks' loads in flight.
        //    GATHER: the row is assembled here from the embedding field, the
        //    direction-state table and the log distances (the message-row
        //    layout of k_rows_two / k_rows_one), with no X buffer in between.
        if (GATHER) {
            const int r = tid & (TC_M - 1);
            const int gr = r0 + r;
            GatherRow row;
            gather_row<GATHER>(rg, gr < rows ? gr : -1, row);
            for (int c0 = tid >> 7; c0 < chunks; c0 += 8) {
                float v[4][8];
#pragma unroll
                for (int u = 0; u < 4; u++) gather_chunk<GATHER>(row, c0 + 2 * u, chunks, v[u]);
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int c = c0 + 2 * u;
                    if (c < chunks) st_bf16x8(sa + canon(r, c * 8, TC_M), v[u]);
                }
            }
        } else {
            {
                const int r = tid & (TC_M - 1);
                const int gr = r0 + r;
                const float* xr = X + (int64_t)gr * ldx;
                for (int c0 = tid >> 7; c0 < chunks; c0 += 8) {
                    float v[4][8];
    #pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int c = c0 + 2 * u;
                        if (vec4) {  // 16-byte rows: two float4 per chunk, masked past k1
    #pragma unroll
                            for (int h2 = 0; h2 < 2; h2++) {
                                const int k = c * 8 + 4 * h2;
                                float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
                                if (c < chunks && gr < rows && k < k1) f = *(const float4*)(xr + k);
                                v[u][4 * h2 + 0] = k + 0 < k1 ? f.x : 0.0f;
                                v[u][4 * h2 + 1] = k + 1 < k1 ? f.y : 0.0f;
                                v[u][4 * h2 + 2] = k + 2 < k1 ? f.z : 0.0f;
                                v[u][4 * h2 + 3] = k + 3 < k1 ? f.w : 0.0f;
                            }
                        } else {
    #pragma unroll
                            for (int e = 0; e < 8; e++) {
                                const int k = c * 8 + e;
                                v[u][e] = (c < chunks && gr < rows && k < k1) ? xr[k] : 0.0f;
                            }
                        }
                    }
    #pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int c = c0 + 2 * u;
                        if (c < chunks) st_bf16x8(sa + canon(r, c * 8, TC_M), v[u]);
                    }
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        // 2. layer 1
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(sa), bb = smem_u32(sw1);
            for (int kk = 0; kk < k1p / 16; kk++) {
                const uint64_t ad = smem_desc(a0 + kk * 2 * TC_M * 16, TC_M * 16, 128);
                const uint64_t bd = smem_desc(bb + kk * 2 * NL1 * 16, NL1 * 16, 128);
                mma_bf16(tmem, ad, bd, idesc_bf16(TC_M, NL1), kk > 0);
            }
            mma_commit(mb);
        }
        ok = __syncthreads_and(mbar_wait(mb, phase)) != 0;  // one decision for the CTA
        if (!ok) {
            if (tid == 0) atomicOr(err, 1u);
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        // 3. epilogue 1: bias + GELU -> BF16 hidden (the side columns: bias,
        //    then float32 rows of V); each warpgroup half the columns
        for (int c = half * (NL1 / 2); c < (half + 1) * (NL1 / 2); c += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + c, v);
            if (NV == 0 || c < N1) {
#pragma unroll
                for (int i = 0; i < 16; i++) v[i] = gelu_tc(__fadd_rn(v[i], b1[c + i]));
                st_bf16x8(sh + canon(trow, c, TC_M), v);
                st_bf16x8(sh + canon(trow, c + 8, TC_M), v + 8);
            } else if (r0 + trow < rows) {
                float* vr = V + (int64_t)(r0 + trow) * ldv + (c - N1);
#pragma unroll
                for (int i = 0; i < 16; i++) vr[i] = __fadd_rn(v[i], bv[c - N1 + i]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        // 4. layer 2
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(sh), bb = smem_u32(sw2);
            for (int kk = 0; kk < N1 / 16; kk++) {
                const uint64_t ad = smem_desc(a0 + kk * 2 * TC_M * 16, TC_M * 16, 128);
                const uint64_t bd = smem_desc(bb + kk * 2 * N2 * 16, N2 * 16, 128);
                mma_bf16(tmem + NL1, ad, bd, idesc_bf16(TC_M, N2), kk > 0);
            }
            mma_commit(mb);
        }
        ok = __syncthreads_and(mbar_wait(mb, phase)) != 0;
        if (!ok) {
            if (tid == 0) atomicOr(err, 1u);
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        // 5. epilogue 2: bias -> float32 tile in shared memory (A is no longer
        //    read), then coalesced row stores
        for (int c = half * (N2 / 2); c < (half + 1) * (N2 / 2); c += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + NL1 + c, v);
#pragma unroll
            for (int i = 0; i < 16; i++) sy[trow * (N2 + 1) + c + i] = __fadd_rn(v[i], b2[c + i]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        for (int e = tid; e < TC_M * ny; e += TC_THREADS) {
            const int r = e / ny, c = e % ny;
            if (r0 + r < rows) Y[(int64_t)(r0 + r) * ldy + c] = sy[r * (N2 + 1) + c];
        }
        __syncthreads();
    }
    if (!ok) {
        // an MMA may still be in flight: wait for it (bounded) before freeing
        // the tensor memory it writes
        mbar_wait(mb, phase);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS));
    }
}


// ---------------------------------------------------------------- FP8 variant
// E4M3 operands, FP32 accumulators. Weights carry one scale per output
// channel (max |w| / 448, applied in the epilogues); activations one scale per
// row, for the input rows and again for the hidden layer before layer 2. The
// canonical layout is the BF16 one in bytes: 8 x 16-byte core matrices of 16
// elements, one K = 32 MMA spanning two of them.
constexpr float FP8_MAX = 448.0f;

__host__ __device__ __forceinline__ uint32_t canon8(uint32_t r, uint32_t k, uint32_t R) {
    return ((k >> 4) * (R >> 3) + (r >> 3)) * 128u + (r & 7u) * 16u + (k & 15u);
}

// kind::f8f6f4 instruction descriptor: E4M3 A and B (K-major), FP32 D, M x N.
__host__ __device__ constexpr uint32_t idesc_e4m3(uint32_t M, uint32_t N) {
    return (1u << 4) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_e4m3(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ uint32_t fp8x4(float a, float b, float c, float d) {
    const uint32_t lo = __nv_cvt_float2_to_fp8x2(make_float2(a, b), __NV_SATFINITE, __NV_E4M3);
    const uint32_t hi = __nv_cvt_float2_to_fp8x2(make_float2(c, d), __NV_SATFINITE, __NV_E4M3);
    return lo | (hi << 16);
}

// 16-byte shared store of 16 E4M3 values (v scaled by inv first).
__device__ __forceinline__ void st_fp8x16(uint8_t* dst, const float* v, float inv) {
    uint4 u;
    u.x = fp8x4(v[0] * inv, v[1] * inv, v[2] * inv, v[3] * inv);
    u.y = fp8x4(v[4] * inv, v[5] * inv, v[6] * inv, v[7] * inv);
    u.z = fp8x4(v[8] * inv, v[9] * inv, v[10] * inv, v[11] * inv);
    u.w = fp8x4(v[12] * inv, v[13] * inv, v[14] * inv, v[15] * inv);
    *(uint4*)dst = u;
}

template <int N1, int N2>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_mlp2_tc8(const float* __restrict__ X, int ldx, int rows, int k1, int k1p,
               const uint8_t* __restrict__ w1p, const float* __restrict__ s1,
               const float* __restrict__ b1, const uint8_t* __restrict__ w2p,
               const float* __restrict__ s2, const float* __restrict__ b2, float* __restrict__ Y,
               int ldy, uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ float red[2][TC_M];
    __shared__ float scale_a[TC_M], scale_h[TC_M];
    uint8_t* sw1 = smem_raw;                        // N1 x k1p
    uint8_t* sw2 = sw1 + (size_t)N1 * k1p;          // N2 x N1
    uint8_t* sa = sw2 + (size_t)N2 * N1;            // 128 x k1p
    uint8_t* sh = sa + (size_t)TC_M * k1p;          // 128 x N1
    float* hbuf = (float*)(sh + (size_t)TC_M * N1); // 128 x (N1 + 1) hidden values
    float* sy = hbuf;                               // 128 x (N2 + 1), after the hidden layer
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quarter = warp & 3, half = warp >> 2;
    {
        const int4* s1p = (const int4*)w1p;
        int4* d1 = (int4*)sw1;
        for (int i = tid; i < N1 * k1p / 16; i += TC_THREADS) d1[i] = s1p[i];
        const int4* s2p = (const int4*)w2p;
        int4* d2 = (int4*)sw2;
        for (int i = tid; i < N2 * N1 / 16; i += TC_THREADS) d2[i] = s2p[i];
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    constexpr uint32_t TMEM_COLS = (N1 + N2) <= 128 ? 128 : ((N1 + N2) <= 256 ? 256 : 512);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    const uint32_t mb = smem_u32(&mbar);
    uint32_t phase = 0;
    bool ok = true;
    const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
    const int trow = quarter * 32 + lane;
    const int n_tiles = (rows + TC_M - 1) / TC_M;
    const int chunks = k1p / 16;
    const int kh = ((k1 + 1) / 2 + 3) & ~3;  // a multiple of 4: float4 steps
    // rows start on 16-byte boundaries and ldx >= round_up(k1, 4): a float4
    // starting below k1 stays inside its row
    const bool vec4 = (ldx % 4) == 0 && ((uintptr_t)X % 16) == 0 && ldx >= ((k1 + 3) & ~3);

    for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        const int r0 = t * TC_M;
        const int r = tid & (TC_M - 1), hf = tid >> 7;
        const int gr = r0 + r;
        const float* xr = X + (int64_t)gr * ldx;
        {  // 1a. per-row scale of X: two threads per row, one half of K each
            float m = 0.0f;
            if (gr < rows) {
                const int ka = hf * kh, kb = min(k1, (hf + 1) * kh);
                if (vec4) {
                    for (int k = ka; k < kb; k += 4) {
                        const float4 f = *(const float4*)(xr + k);
                        m = fmaxf(m, fmaxf(fmaxf(fabsf(f.x), k + 1 < kb ? fabsf(f.y) : 0.0f),
                                           fmaxf(k + 2 < kb ? fabsf(f.z) : 0.0f,
                                                 k + 3 < kb ? fabsf(f.w) : 0.0f)));
                    }
                } else {
                    for (int k = ka; k < kb; k++) m = fmaxf(m, fabsf(xr[k]));
                }
            }
            red[hf][r] = m;
        }
        __syncthreads();
        if (tid < TC_M) {
            const float m = fmaxf(red[0][tid], red[1][tid]);
            scale_a[tid] = m > 0.0f ? m / FP8_MAX : 1.0f;
        }
        __syncthreads();
        {  // 1b. rows of X -> E4M3 A operand, 16-element chunks
            const float inv = 1.0f / scale_a[r];
            for (int c = hf; c < chunks; c += 2) {
                float v[16];
                if (vec4) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int k = c * 16 + 4 * q;
                        float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (gr < rows && k < k1) f = *(const float4*)(xr + k);
                        v[4 * q + 0] = k + 0 < k1 ? f.x : 0.0f;
                        v[4 * q + 1] = k + 1 < k1 ? f.y : 0.0f;
                        v[4 * q + 2] = k + 2 < k1 ? f.z : 0.0f;
                        v[4 * q + 3] = k + 3 < k1 ? f.w : 0.0f;
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 16; e++) {
                        const int k = c * 16 + e;
                        v[e] = (gr < rows && k < k1) ? xr[k] : 0.0f;
                    }
                }
                st_fp8x16(sa + canon8(r, c * 16, TC_M), v, inv);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        // 2. layer 1
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(sa), bb = smem_u32(sw1);
            for (int kk = 0; kk < k1p / 32; kk++) {
                const uint64_t ad = smem_desc(a0 + kk * 2 * TC_M * 16, TC_M * 16, 128);
                const uint64_t bd = smem_desc(bb + kk * 2 * N1 * 16, N1 * 16, 128);
                mma_e4m3(tmem, ad, bd, idesc_e4m3(TC_M, N1), kk > 0);
            }
            mma_commit(mb);
        }
        ok = __syncthreads_and(mbar_wait(mb, phase)) != 0;
        if (!ok) {
            if (tid == 0) atomicOr(err, 1u);
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        // 3. epilogue 1: bias + GELU, per-row hidden scale, E4M3 hidden operand
        const float sa_r = scale_a[trow];
        {  // hidden values into shared memory and their row maximum
            float m = 0.0f;
            for (int c = half * (N1 / 2); c < (half + 1) * (N1 / 2); c += 16) {
                float v[16];
                tmem_ld16(tmem + lane_base + c, v);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const float hv = gelu_tc(__fadd_rn(v[i] * sa_r * s1[c + i], b1[c + i]));
                    hbuf[trow * (N1 + 1) + c + i] = hv;
                    m = fmaxf(m, fabsf(hv));
                }
            }
            red[half][trow] = m;
        }
        __syncthreads();
        if (tid < TC_M) {
            const float m = fmaxf(red[0][tid], red[1][tid]);
            scale_h[tid] = m > 0.0f ? m / FP8_MAX : 1.0f;
        }
        __syncthreads();
        {
            const float inv = 1.0f / scale_h[trow];
            for (int c = half * (N1 / 2); c < (half + 1) * (N1 / 2); c += 16) {
                float v[16];
#pragma unroll
                for (int i = 0; i < 16; i++) v[i] = hbuf[trow * (N1 + 1) + c + i];
                st_fp8x16(sh + canon8(trow, c, TC_M), v, inv);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        // 4. layer 2
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(sh), bb = smem_u32(sw2);
            for (int kk = 0; kk < N1 / 32; kk++) {
                const uint64_t ad = smem_desc(a0 + kk * 2 * TC_M * 16, TC_M * 16, 128);
                const uint64_t bd = smem_desc(bb + kk * 2 * N2 * 16, N2 * 16, 128);
                mma_e4m3(tmem + N1, ad, bd, idesc_e4m3(TC_M, N2), kk > 0);
            }
            mma_commit(mb);
        }
        ok = __syncthreads_and(mbar_wait(mb, phase)) != 0;
        if (!ok) {
            if (tid == 0) atomicOr(err, 1u);
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        // 5. epilogue 2: scales + bias -> float32 staging, coalesced rows
        const float sh_r = scale_h[trow];
        for (int c = half * (N2 / 2); c < (half + 1) * (N2 / 2); c += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + N1 + c, v);
#pragma unroll
            for (int i = 0; i < 16; i++)
                sy[trow * (N2 + 1) + c + i] = __fadd_rn(v[i] * sh_r * s2[c + i], b2[c + i]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        for (int e = tid; e < TC_M * N2; e += TC_THREADS) {
            const int rr = e / N2, c = e % N2;
            if (r0 + rr < rows) Y[(int64_t)(r0 + rr) * ldy + c] = sy[rr * (N2 + 1) + c];
        }
        __syncthreads();
    }
    if (!ok) mbar_wait(mb, phase);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS));
    }
}
}  // namespace

// Shared memory of the fused kernel for an input width padded to k1p.
uint64_t mlp2_tc_smem(int k1p, int n1, int n2, int nv = 0) {
    return 2ull * ((uint64_t)(n1 + nv) * k1p + (uint64_t)n2 * n1 + (uint64_t)TC_M * k1p +
                   (uint64_t)TC_M * n1);
}

int mlp2_tc(const float* X, int ldx, int64_t rows, int k1, int k1p, const void* w1p,
            const float* b1, const void* w2p, const float* b2, int n1, int n2, float* Y, int ldy,
            int ny, uint32_t* err, int n_sm, cudaStream_t st) {
    if (rows <= 0) return LATEC_OK;
    const bool big = n1 == 128 && n2 == 64, key = n1 == 64 && n2 == 32;
    if ((!big && !key) || ny < 1 || ny > n2 || ldy < ny || k1p % 16 || k1p < k1 ||
        rows > 0x7fffffffLL)
        return LATEC_ERR_UNSUPPORTED;
    // the float32 output tile (128 x (n2 + 1)) is staged over the A and hidden buffers
    const uint64_t smem = mlp2_tc_smem(k1p, n1, n2);
    if (smem > 220 * 1024 || 4ull * TC_M * (n2 + 1) > 2ull * TC_M * (k1p + n1))
        return LATEC_ERR_UNSUPPORTED;
    auto kern = big ? k_mlp2_tc<128, 64, 0, 0> : k_mlp2_tc<64, 32, 0, 0>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return LATEC_ERR_CUDA;
    const int64_t tiles = (rows + TC_M - 1) / TC_M;
    const int grid = (int)(tiles < n_sm ? tiles : n_sm);
    kern<<<grid, TC_THREADS, smem, st>>>(X, ldx, (int)rows, k1, k1p, (const __nv_bfloat16*)w1p, b1,
                                         (const __nv_bfloat16*)w2p, b2, Y, ldy, ny, nullptr,
                                         nullptr, 0, RowGather{}, err);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

// The line pool's key MLP with its value projection on layer 1's side columns:
// w1p packs [Wk0; Wv] (128 x 64), KEY gets the key (one float per row), V the
// 64 values of each row (row stride ldv).
int kv_tc(const float* X, int ldx, int64_t rows, const void* w1p, const float* b1,
          const float* bv, const void* w2p, const float* b2, float* KEY, float* V, int ldv,
          uint32_t* err, int n_sm, cudaStream_t st) {
    if (rows <= 0) return LATEC_OK;
    if (rows > 0x7fffffffLL || ldv < 64) return LATEC_ERR_UNSUPPORTED;
    const uint64_t smem = mlp2_tc_smem(64, 64, 32, 64);
    auto kern = k_mlp2_tc<64, 32, 64, 0>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return LATEC_ERR_CUDA;
    const int64_t tiles = (rows + TC_M - 1) / TC_M;
    const int grid = (int)(tiles < n_sm ? tiles : n_sm);
    kern<<<grid, TC_THREADS, smem, st>>>(X, ldx, (int)rows, 64, 64, (const __nv_bfloat16*)w1p, b1,
                                         (const __nv_bfloat16*)w2p, b2, KEY, 1, 1, bv, V, ldv,
                                         RowGather{}, err);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

// The message MLP (hidden 128, output 64) over message rows gathered in the
// operand staging: two_sided 1 = BiDirEmbed rows (k1 162), 0 = DirEmbed rows
// (k1 82). rows = pairs x K; Y gets 64 floats per row (row stride ldy).
int mlp2_tc_gather(const RowGather& rg, int two_sided, int64_t rows, int k1, int k1p,
                   const void* w1p, const float* b1, const void* w2p, const float* b2, float* Y,
                   int ldy, uint32_t* err, int n_sm, cudaStream_t st) {
    if (rows <= 0) return LATEC_OK;
    if (rows > 0x7fffffffLL || k1 != (two_sided ? 162 : 82) || k1p % 16 || k1p < k1 ||
        ((uintptr_t)rg.E % 16) != 0)
        return LATEC_ERR_UNSUPPORTED;
    const uint64_t smem = mlp2_tc_smem(k1p, 128, 64);
    if (smem > 220 * 1024 || 4ull * TC_M * 65 > 2ull * TC_M * (k1p + 128))
        return LATEC_ERR_UNSUPPORTED;
    auto kern = two_sided ? k_mlp2_tc<128, 64, 0, 2> : k_mlp2_tc<128, 64, 0, 1>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return LATEC_ERR_CUDA;
    const int64_t tiles = (rows + TC_M - 1) / TC_M;
    const int grid = (int)(tiles < n_sm ? tiles : n_sm);
    kern<<<grid, TC_THREADS, smem, st>>>(nullptr, 0, (int)rows, k1, k1p, (const __nv_bfloat16*)w1p,
                                         b1, (const __nv_bfloat16*)w2p, b2, Y, ldy, 64, nullptr,
                                         nullptr, 0, rg, err);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}


uint64_t mlp2_tc8_smem(int k1p, int n1, int n2) {
    const uint64_t stage = 4ull * TC_M * ((n1 > n2 ? n1 : n2) + 1);  // hidden, then Y
    return (uint64_t)n1 * k1p + (uint64_t)n2 * n1 + (uint64_t)TC_M * k1p + (uint64_t)TC_M * n1 +
           stage;
}

int mlp2_tc8(const float* X, int ldx, int64_t rows, int k1, int k1p, const void* w1p,
             const float* s1, const float* b1, const void* w2p, const float* s2, const float* b2,
             int n1, int n2, float* Y, int ldy, uint32_t* err, int n_sm, cudaStream_t st) {
    if (rows <= 0) return LATEC_OK;
    if (n1 != 128 || n2 != 64 || k1p % 32 || k1p < k1 || rows > 0x7fffffffLL)
        return LATEC_ERR_UNSUPPORTED;
    const uint64_t smem = mlp2_tc8_smem(k1p, n1, n2);
    if (smem > 200 * 1024) return LATEC_ERR_UNSUPPORTED;
    auto kern = k_mlp2_tc8<128, 64>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return LATEC_ERR_CUDA;
    const int64_t tiles = (rows + TC_M - 1) / TC_M;
    const int grid = (int)(tiles < n_sm ? tiles : n_sm);
    kern<<<grid, TC_THREADS, smem, st>>>(X, ldx, (int)rows, k1, k1p, (const uint8_t*)w1p, s1, b1,
                                         (const uint8_t*)w2p, s2, b2, Y, ldy, err);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // namespace latec

using namespace latec;

extern "C" {

// Pack a float32 (n x k) weight matrix, row-major, into the BF16 no-swizzle
// K-major canonical layout the tensor-core MLP reads (k zero-padded to kp,
// a multiple of 16; n a multiple of 8). Host arrays; out has n * kp entries.
int latec_gnn_pack_bf16(const float* w, int32_t n, int32_t k, int32_t kp, uint16_t* out) {
    if (!w || !out || n < 8 || n % 8 || k < 1 || kp < k || kp % 16) return LATEC_ERR_ARG;
    for (int r = 0; r < n; r++)
        for (int c = 0; c < kp; c++) {
            const float v = c < k ? w[(int64_t)r * k + c] : 0.0f;
            const __nv_bfloat16 b = __float2bfloat16_rn(v);
            out[canon((uint32_t)r, (uint32_t)c, (uint32_t)n)] = *(const uint16_t*)&b;
        }
    return LATEC_OK;
}

// Y = W2 * gelu(W1 * X + b1) + b2 on the tensor cores (hidden 128, output 64).
// w1p / w2p: device, packed by latec_gnn_pack_bf16 (w1: 128 x k1p,
// w2: 64 x 128). err bit 1: a tensor-core wait ran out (results invalid).
int latec_gnn_mlp2_bf16(const float* X, int32_t ldx, int64_t rows, int32_t k1, int32_t k1p,
                        const void* w1p, const float* b1, const void* w2p, const float* b2,
                        float* Y, int32_t ldy, uint32_t* err, void* stream) {
    if ((rows && (!X || !Y)) || !w1p || !b1 || !w2p || !b2 || !err || ldx < k1 || ldy < 64)
        return LATEC_ERR_ARG;
    int dev = 0, n_sm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    return mlp2_tc(X, ldx, rows, k1, k1p, w1p, b1, w2p, b2, 128, 64, Y, ldy, 64, err, n_sm,
                   (cudaStream_t)stream);
}


// Pack a float32 (n x k) weight matrix into E4M3 with one scale per output
// row (max |w| / 448, 1 for a zero row), in the canonical no-swizzle
// K-major layout of the FP8 MLP (k zero-padded to kp, a multiple of 32; n a
// multiple of 8). Host arrays; out has n * kp bytes, scales n floats.
int latec_gnn_pack_fp8(const float* w, int32_t n, int32_t k, int32_t kp, uint8_t* out,
                       float* scales) {
    if (!w || !out || !scales || n < 8 || n % 8 || k < 1 || kp < k || kp % 32) return LATEC_ERR_ARG;
    for (int r = 0; r < n; r++) {
        float m = 0.0f;
        for (int c = 0; c < k; c++) m = fmaxf(m, fabsf(w[(int64_t)r * k + c]));
        const float sc = m > 0.0f ? m / FP8_MAX : 1.0f;
        scales[r] = sc;
        for (int c = 0; c < kp; c++) {
            const float v = c < k ? w[(int64_t)r * k + c] / sc : 0.0f;
            out[canon8((uint32_t)r, (uint32_t)c, (uint32_t)n)] =
                (uint8_t)__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
        }
    }
    return LATEC_OK;
}

// Y = W2 * gelu(W1 * X + b1) + b2 with E4M3 operands (hidden 128, output 64):
// w1p / w2p and s1 / s2 from latec_gnn_pack_fp8 (device). err bit 1: a
// tensor-core wait ran out (results invalid).
int latec_gnn_mlp2_fp8(const float* X, int32_t ldx, int64_t rows, int32_t k1, int32_t k1p,
                       const void* w1p, const float* s1, const float* b1, const void* w2p,
                       const float* s2, const float* b2, float* Y, int32_t ldy, uint32_t* err,
                       void* stream) {
    if ((rows && (!X || !Y)) || !w1p || !s1 || !b1 || !w2p || !s2 || !b2 || !err || ldx < k1 ||
        ldy < 64)
        return LATEC_ERR_ARG;
    int dev = 0, n_sm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    return mlp2_tc8(X, ldx, rows, k1, k1p, w1p, s1, b1, w2p, s2, b2, 128, 64, Y, ldy, err, n_sm,
                    (cudaStream_t)stream);
}

}  // extern "C"
