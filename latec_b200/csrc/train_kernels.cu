// Training kernels of the learned predictor (scripts/train_gnn.py): the
// forward ops of the axial GNN with the activations the backward pass needs,
// their backward ops, the discretised-Laplace rate loss and the AdamW / EMA
// updates. Activations, weights, gradients and optimiser state are float32;
// gradient reductions over rows use atomics (training needs no run-to-run bit
// identity; the codec's inference path is gnn_kernels.cu, whose order is
// fixed). The linear layers' GEMMs run in one of two precisions:
//   - float32: SIMT tiles (k_gemm);
//   - BF16 (the reference's mixed-precision training, with float32 master
//     weights): both operands rounded to BF16 as they are staged, float32
//     accumulation; tcgen05 tensor-core tiles (k_gemm_tc, accumulators in
//     tensor memory) where the output tile is at least 32 wide, the SIMT tile
//     with the same operand rounding for the narrow 1- and 2-wide layers.
//
// Layouts: X (rows, ldx) row-major; weights W (out, in) row-major as in the
// reference's nn.Linear; E (B, N, K, d); contexts (B, M, K, d).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "latec_common.cuh"
#include "tc_sm100.cuh"

namespace latec {
namespace {

constexpr int TT = 256;
constexpr int GM = 64, GN = 64, GK = 16;

inline unsigned tblocks(int64_t n) { return (unsigned)((n + TT - 1) / TT); }

__device__ __forceinline__ float gelu_f(float z) {
    return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_d(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// C (M x N, ldc) = sum_k A(m, k) * B(k, n), 64 x 64 tiles, 4 x 4 per thread.
//   TA = 0: A(m, k) = A[m * lda + k]; TA = 1: A(m, k) = A[k * lda + m]
//   TB = 0: B(k, n) = B[k * ldb + n]; TB = 1: B(k, n) = B[n * ldb + k]
//   GA: A is dY and is multiplied by gelu'(Z) on load (Z laid out like A)
//   split-K over gridDim.z; ACC: add into C with atomics, else store
//   bias (optional; only without split-K)
//   bf: operands rounded to BF16 (round to nearest even) as they are staged
template <int TA, int TB, int GA, int ACC>
__global__ void __launch_bounds__(TT)
    k_gemm(int M, int N, int Kd, const float* __restrict__ A, int64_t lda,
           const float* __restrict__ Bm, int64_t ldb, const float* __restrict__ Z, float* C,
           int64_t ldc, const float* __restrict__ bias, int act, float* Zout, int64_t ldz,
           int bf) {
    __shared__ float as[GK][GM + 4];
    __shared__ float bs[GK][GN + 4];
    const int m0 = blockIdx.x * GM, n0 = blockIdx.y * GN;
    const int64_t per = ((int64_t)Kd + gridDim.z - 1) / gridDim.z;
    const int64_t kb = per * blockIdx.z, ke = kb + per < Kd ? kb + per : Kd;
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    float acc[4][4] = {};
    for (int64_t k0 = kb; k0 < ke; k0 += GK) {
        for (int e = threadIdx.x; e < GM * GK; e += TT) {
            int mm, kk;
            if (TA) { kk = e / GM; mm = e % GM; } else { mm = e / GK; kk = e % GK; }
            const int m = m0 + mm;
            const int64_t k = k0 + kk;
            float v = 0.0f;
            if (m < M && k < ke) {
                const int64_t o = TA ? k * lda + m : (int64_t)m * lda + k;
                v = A[o];
                if (GA) v *= gelu_d(Z[o]);
                if (bf) v = __bfloat162float(__float2bfloat16_rn(v));
            }
            as[kk][mm] = v;
        }
        for (int e = threadIdx.x; e < GN * GK; e += TT) {
            int nn, kk;
            if (TB) { nn = e / GK; kk = e % GK; } else { kk = e / GN; nn = e % GN; }
            const int n = n0 + nn;
            const int64_t k = k0 + kk;
            float v = (n < N && k < ke) ? Bm[TB ? (int64_t)n * ldb + k : k * ldb + n] : 0.0f;
            if (bf) v = __bfloat162float(__float2bfloat16_rn(v));
            bs[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk++) {
            float av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; a++) av[a] = as[kk][tr * 4 + a];
#pragma unroll
            for (int c = 0; c < 4; c++) bv[c] = bs[kk][tc * 4 + c];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[a][c] += av[a] * bv[c];
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; a++) {
        const int m = m0 + tr * 4 + a;
        if (m >= M) continue;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int n = n0 + tc * 4 + c;
            if (n >= N) continue;
            float v = acc[a][c];
            if (ACC) {
                atomicAdd(&C[(int64_t)m * ldc + n], v);
            } else {
                if (bias) v += bias[n];
                if (Zout) Zout[(int64_t)m * ldz + n] = v;
                C[(int64_t)m * ldc + n] = act ? gelu_f(v) : v;
            }
        }
    }
}

// ------------------------------------------------- BF16 tensor-core GEMM
// The contract of k_gemm (same TA / TB / GA / ACC meaning, bias, act, Zout,
// split-K over gridDim.z) on tcgen05: a CTA computes a 128 x NT tile of C
// with FP32 accumulators in tensor memory (NT columns). K is staged GT_KC
// elements at a time into a two-buffer ring: all 256 threads load the chunk of
// A (128 rows) and of B (NT rows of B^T) as float32, apply gelu' to A when GA,
// round both to BF16 and store them in the no-swizzle K-major canonical
// layout; one thread then issues GT_KC / 16 MMAs (M 128, N NT, K 16) and
// commits them to the buffer's mbarrier, which the threads wait on before
// they refill that buffer two chunks later, so the staging of a chunk
// overlaps the MMAs of the previous one. The epilogue reads each thread's
// TMEM lane (one row of the tile) 16 columns at a time. Waits are bounded: on
// expiry the kernel sets bit 0 of g_gemm_tc_err, waits (bounded) for the MMAs
// it issued and frees its tensor memory.
constexpr int GT_THREADS = 256;
constexpr int GT_M = 128;
constexpr int GT_KC = 64;

__device__ uint32_t g_gemm_tc_err;

// One GT_KC-wide K chunk of an R-row operand: element (r, k) is
// src[r * rs + k * ks], zero at r >= r_valid or k >= k_end; times gelu'(Z) at
// the same offset when GA. Each item is 8 consecutive k of one row (one 16-byte
// canonical store); the canonical stores of 8 consecutive rows fill 128
// contiguous bytes.
//   rs == 1 (k strided): consecutive threads take consecutive rows, so each of
//     the 8 loads of a warp reads 128 contiguous bytes.
//   ks == 1 (rows contiguous): a warp takes 8 rows x 4 chunks, so the 4
//     chunks of a row are 128 contiguous bytes, read as float4 (or float2)
//     when vw says the rows allow it (vw = 4, 2 or 1 elements per load).
template <int R, int GA>
__device__ __forceinline__ void stage_chunk(__nv_bfloat16* dst, const float* __restrict__ src,
                                            const float* __restrict__ Z, int64_t rs, int64_t ks,
                                            int vw, int r_valid, int64_t k0, int64_t k_end,
                                            int tid) {
    constexpr int ITEMS = R * (GT_KC / 8);
    for (int it = tid; it < ITEMS; it += GT_THREADS) {
        int r, c;
        if (ks == 1) {
            const int g = it >> 5, l = it & 31;
            r = (g >> 1) * 8 + (l & 7);
            c = (g & 1) * 4 + (l >> 3);
        } else {
            r = it % R;
            c = it / R;
        }
        float v[8];
        const int64_t kc = k0 + c * 8;
        if (ks == 1 && r < r_valid && kc + 8 <= k_end && vw > 1) {
            const int64_t o = (int64_t)r * rs + kc;
            if (vw == 4) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const float4 f = *(const float4*)(src + o + 4 * h);
                    v[4 * h] = f.x, v[4 * h + 1] = f.y, v[4 * h + 2] = f.z, v[4 * h + 3] = f.w;
                    if (GA) {
                        const float4 zz = *(const float4*)(Z + o + 4 * h);
                        v[4 * h] *= gelu_d(zz.x), v[4 * h + 1] *= gelu_d(zz.y);
                        v[4 * h + 2] *= gelu_d(zz.z), v[4 * h + 3] *= gelu_d(zz.w);
                    }
                }
            } else {
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    const float2 f = *(const float2*)(src + o + 2 * h);
                    v[2 * h] = f.x, v[2 * h + 1] = f.y;
                    if (GA) {
                        const float2 zz = *(const float2*)(Z + o + 2 * h);
                        v[2 * h] *= gelu_d(zz.x), v[2 * h + 1] *= gelu_d(zz.y);
                    }
                }
            }
        } else {
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const int64_t k = kc + e;
                float x = 0.0f;
                if (r < r_valid && k < k_end) {
                    const int64_t o = (int64_t)r * rs + k * ks;
                    x = src[o];
                    if (GA) x *= gelu_d(Z[o]);
                }
                v[e] = x;
            }
        }
        st_bf16x8(dst + canon((uint32_t)r, (uint32_t)(c * 8), R), v);
    }
}

// Widest vector (4, 2 or 1 floats) that every row start of a row-contiguous
// operand allows.
__device__ __forceinline__ int row_vec(const float* p, int64_t rs, const float* z) {
    const uintptr_t a = (uintptr_t)p | (z ? (uintptr_t)z : 0);
    if (rs % 4 == 0 && a % 16 == 0) return 4;
    if (rs % 2 == 0 && a % 8 == 0) return 2;
    return 1;
}

template <int TA, int TB, int GA, int ACC, int NT>
__global__ void __launch_bounds__(GT_THREADS)
    k_gemm_tc(int M, int N, int Kd, const float* __restrict__ A, int64_t lda,
              const float* __restrict__ Bm, int64_t ldb, const float* __restrict__ Z, float* C,
              int64_t ldc, const float* __restrict__ bias, int act, float* Zout, int64_t ldz) {
    static_assert(NT == 64 || NT == 128, "tile width");
    constexpr int A_ELEMS = GT_M * GT_KC, B_ELEMS = NT * GT_KC;
    constexpr uint32_t TMEM_COLS = NT;
    extern __shared__ __align__(128) uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base;
    __nv_bfloat16* sbuf = (__nv_bfloat16*)smem_raw;  // [A0 | B0 | A1 | B1]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * GT_M, n0 = blockIdx.y * NT;
    // split-K slices start on GT_KC boundaries (aligned vector loads)
    const int64_t per =
        (((int64_t)Kd + gridDim.z - 1) / gridDim.z + GT_KC - 1) / GT_KC * GT_KC;
    const int64_t kb = per * blockIdx.z;
    const int64_t ke = kb + per < Kd ? kb + per : Kd;
    // A(m, k) = TA ? A[k lda + m] : A[m lda + k]; B^T(n, k) = B(k, n)
    const int64_t a_rs = TA ? 1 : lda, a_ks = TA ? lda : 1;
    const int64_t a_off = TA ? (int64_t)m0 : (int64_t)m0 * lda;
    const int64_t b_rs = TB ? ldb : 1, b_ks = TB ? 1 : ldb;
    const int64_t b_off = TB ? (int64_t)n0 * ldb : (int64_t)n0;
    const int m_valid = M - m0 < GT_M ? M - m0 : GT_M;
    const int n_valid = N - n0 < NT ? N - n0 : NT;
    const int a_vw = TA ? 1 : row_vec(A + a_off, a_rs, GA ? Z + a_off : nullptr);
    const int b_vw = TB ? row_vec(Bm + b_off, b_rs, nullptr) : 1;

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar[0])), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar[1])), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
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

    const int nk = ke > kb ? (int)((ke - kb + GT_KC - 1) / GT_KC) : 0;
    bool ok = true;
    int issued = 0;  // chunks whose MMAs were committed
    for (int i = 0; i < nk; i++) {
        const int s = i & 1;
        if (i >= 2) {  // the MMAs of chunk i - 2 have read buffer s
            ok = __syncthreads_and(mbar_wait(smem_u32(&mbar[s]), (uint32_t)((i - 2) >> 1) & 1u)) != 0;
            if (!ok) break;
        }
        __nv_bfloat16* sa = sbuf + s * (A_ELEMS + B_ELEMS);
        __nv_bfloat16* sb = sa + A_ELEMS;
        const int64_t k0 = kb + (int64_t)i * GT_KC;
        stage_chunk<GT_M, GA>(sa, A + a_off, GA ? Z + a_off : nullptr, a_rs, a_ks, a_vw, m_valid,
                              k0, ke, tid);
        stage_chunk<NT, 0>(sb, Bm + b_off, nullptr, b_rs, b_ks, b_vw, n_valid, k0, ke, tid);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
            for (int kk = 0; kk < GT_KC / 16; kk++) {
                const uint64_t ad = smem_desc(a0 + kk * 2 * GT_M * 16, GT_M * 16, 128);
                const uint64_t bd = smem_desc(b0 + kk * 2 * NT * 16, NT * 16, 128);
                mma_bf16(tmem, ad, bd, idesc_bf16(GT_M, NT), (i > 0 || kk > 0) ? 1u : 0u);
            }
            mma_commit(smem_u32(&mbar[s]));
        }
        issued = i + 1;
    }
    if (issued) {  // the last commit covers every MMA issued before it
        const int l = issued - 1;
        const bool got = __syncthreads_and(
                             mbar_wait(smem_u32(&mbar[l & 1]), (uint32_t)(l >> 1) & 1u)) != 0;
        ok = ok && got;
    }
    if (!ok && tid == 0) atomicOr(&g_gemm_tc_err, 1u);
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok && issued) {
        const int quarter = warp & 3, half = warp >> 2;
        const int m = m0 + quarter * 32 + lane;  // this thread's TMEM lane
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        for (int c = half * (NT / 2); c < (half + 1) * (NT / 2); c += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + c, v);
            if (m >= M) continue;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int n = n0 + c + i;
                if (n >= N) continue;
                float x = v[i];
                if (ACC) {
                    atomicAdd(&C[(int64_t)m * ldc + n], x);
                } else {
                    if (bias) x += bias[n];
                    if (Zout) Zout[(int64_t)m * ldz + n] = x;
                    C[(int64_t)m * ldc + n] = act ? gelu_f(x) : x;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS));
    }
}

template <int NT>
constexpr int gemm_tc_smem() {
    return 2 * (GT_M + NT) * GT_KC * (int)sizeof(__nv_bfloat16);
}

// C = A B (see k_gemm) in float32 (prec 0) or BF16 operands with float32
// accumulation (prec 1: tensor cores when M and N are at least 32, the SIMT
// tile with rounded operands otherwise). Returns the launches.
template <int TA, int TB, int GA, int ACC>
int gemm(int prec, int M, int N, int Kd, unsigned splits, const float* A, int64_t lda,
         const float* Bm, int64_t ldb, const float* Z, float* C, int64_t ldc, const float* bias,
         int act, float* Zout, int64_t ldz, cudaStream_t st) {
    if (prec == 1 && M >= 32 && N >= 32) {
        if (N > 64) {
            constexpr int NT = 128;
            cudaFuncSetAttribute(k_gemm_tc<TA, TB, GA, ACC, NT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_tc_smem<NT>());
            dim3 grid((unsigned)((M + GT_M - 1) / GT_M), (unsigned)((N + NT - 1) / NT), splits);
            k_gemm_tc<TA, TB, GA, ACC, NT><<<grid, GT_THREADS, gemm_tc_smem<NT>(), st>>>(
                M, N, Kd, A, lda, Bm, ldb, Z, C, ldc, bias, act, Zout, ldz);
        } else {
            constexpr int NT = 64;
            cudaFuncSetAttribute(k_gemm_tc<TA, TB, GA, ACC, NT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_tc_smem<NT>());
            dim3 grid((unsigned)((M + GT_M - 1) / GT_M), (unsigned)((N + NT - 1) / NT), splits);
            k_gemm_tc<TA, TB, GA, ACC, NT><<<grid, GT_THREADS, gemm_tc_smem<NT>(), st>>>(
                M, N, Kd, A, lda, Bm, ldb, Z, C, ldc, bias, act, Zout, ldz);
        }
        return 1;
    }
    dim3 grid((unsigned)((M + GM - 1) / GM), (unsigned)((N + GN - 1) / GN), splits);
    k_gemm<TA, TB, GA, ACC><<<grid, TT, 0, st>>>(M, N, Kd, A, lda, Bm, ldb, Z, C, ldc, bias, act,
                                                 Zout, ldz, prec == 1 ? 1 : 0);
    return 1;
}

// db[j] += sum_r dY[r, j] (* gelu'(Z[r, j])): one warp per column slice.
__global__ void __launch_bounds__(TT)
    k_colsum(int64_t rows, int n, const float* __restrict__ dY, int64_t ldy,
             const float* __restrict__ Z, float* __restrict__ db) {
    const int j = blockIdx.y;
    float s = 0.0f;
    for (int64_t r = (int64_t)blockIdx.x * TT + threadIdx.x; r < rows; r += (int64_t)gridDim.x * TT) {
        float v = dY[r * ldy + j];
        if (Z) v *= gelu_d(Z[r * ldy + j]);
        s += v;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&db[j], s);
}

// ---- message rows (all batches at once): row w = (b * np + p) * K + k ----
// two-sided: [E(nbr_n) | table(sidx_n) | E(nbr_p) | table(sidx_p) | logd_n | logd_p]
// one-sided: [E(side) | table(side) | +-1 | logd_side]
__global__ void __launch_bounds__(TT)
    k_tr_rows(const float* __restrict__ E, int64_t N, int K, int d, int ds,
              const float* __restrict__ table, const latec_gnn_geom g,
              const int32_t* __restrict__ pairs, int64_t np, int B, int two, float* __restrict__ X,
              int ldx) {
    const int64_t w = ((int64_t)blockIdx.x * TT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (int64_t)B * np * K) return;
    const int k = (int)(w % K);
    const int64_t bp = w / K;
    const int64_t p = bp % np;
    const int b = (int)(bp / np);
    const int pair = pairs[p];
    const int l = pair / g.M;
    const int de = d + ds;
    float* row = X + w * ldx;
    if (two) {
        const float* en = E + (((int64_t)b * N + g.nbr_n[pair]) * K + k) * d;
        const float* ep = E + (((int64_t)b * N + g.nbr_p[pair]) * K + k) * d;
        const float* sn = table + (int64_t)g.sidx_n[l * K + k] * ds;
        const float* sp = table + (int64_t)g.sidx_p[l * K + k] * ds;
        for (int f = lane; f < 2 * de + 2; f += 32) {
            float v;
            if (f < d) v = en[f];
            else if (f < de) v = sn[f - d];
            else if (f < de + d) v = ep[f - de];
            else if (f < 2 * de) v = sp[f - de - d];
            else if (f == 2 * de) v = g.logd_n[pair];
            else v = g.logd_p[pair];
            row[f] = v;
        }
    } else {
        const bool pos = g.nbr_p[pair] >= 0;
        const int64_t nb = pos ? g.nbr_p[pair] : g.nbr_n[pair];
        const float* e = E + (((int64_t)b * N + nb) * K + k) * d;
        const float* s = table + (int64_t)(pos ? g.sidx_p[l * K + k] : g.sidx_n[l * K + k]) * ds;
        for (int f = lane; f < de + 2; f += 32) {
            float v;
            if (f < d) v = e[f];
            else if (f < de) v = s[f - d];
            else if (f == de) v = pos ? 1.0f : -1.0f;
            else v = pos ? g.logd_p[pair] : g.logd_n[pair];
            row[f] = v;
        }
    }
}

// Backward of k_tr_rows: dE and dtable by atomics (the geometry features are
// constants).
__global__ void __launch_bounds__(TT)
    k_tr_rows_bwd(const float* __restrict__ dX, int ldx, int64_t N, int K, int d, int ds,
                  const latec_gnn_geom g, const int32_t* __restrict__ pairs, int64_t np, int B,
                  int two, float* __restrict__ dE, float* __restrict__ dtable) {
    const int64_t w = ((int64_t)blockIdx.x * TT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (int64_t)B * np * K) return;
    const int k = (int)(w % K);
    const int64_t bp = w / K;
    const int64_t p = bp % np;
    const int b = (int)(bp / np);
    const int pair = pairs[p];
    const int l = pair / g.M;
    const int de = d + ds;
    const float* row = dX + w * ldx;
    if (two) {
        float* en = dE + (((int64_t)b * N + g.nbr_n[pair]) * K + k) * d;
        float* ep = dE + (((int64_t)b * N + g.nbr_p[pair]) * K + k) * d;
        float* sn = dtable + (int64_t)g.sidx_n[l * K + k] * ds;
        float* sp = dtable + (int64_t)g.sidx_p[l * K + k] * ds;
        for (int f = lane; f < 2 * de; f += 32) {
            const float v = row[f];
            if (f < d) atomicAdd(en + f, v);
            else if (f < de) atomicAdd(sn + (f - d), v);
            else if (f < de + d) atomicAdd(ep + (f - de), v);
            else atomicAdd(sp + (f - de - d), v);
        }
    } else {
        const bool pos = g.nbr_p[pair] >= 0;
        const int64_t nb = pos ? g.nbr_p[pair] : g.nbr_n[pair];
        float* e = dE + (((int64_t)b * N + nb) * K + k) * d;
        float* s = dtable + (int64_t)(pos ? g.sidx_p[l * K + k] : g.sidx_n[l * K + k]) * ds;
        for (int f = lane; f < de; f += 32) {
            const float v = row[f];
            if (f < d) atomicAdd(e + f, v);
            else atomicAdd(s + (f - d), v);
        }
    }
}

// Candidate rows of the line pool for every (b, m, k). Message rows are laid
// out as all two-sided rows ((b * np2 + r) * K + k), then all one-sided rows
// (B * np2 * K + (b * np1 + r - np2) * K + k); r = row_of[l, m] (two-sided
// rows first) or -1 (masked).
__global__ void __launch_bounds__(TT)
    k_tr_line_rows(const int32_t* __restrict__ row_of, int M, int L, int K, int B, int64_t np2,
                   int64_t np1, int32_t* __restrict__ rows) {
    const int64_t t = (int64_t)blockIdx.x * TT + threadIdx.x;
    if (t >= (int64_t)B * M * K) return;
    const int k = (int)(t % K);
    const int64_t bm = t / K;
    const int m = (int)(bm % M), b = (int)(bm / M);
    for (int l = 0; l < L; l++) {
        const int64_t r = row_of[(int64_t)l * M + m];
        int64_t v = -1;
        if (r >= 0 && r < np2) v = ((int64_t)b * np2 + r) * K + k;
        else if (r >= np2) v = (int64_t)B * np2 * K + ((int64_t)b * np1 + (r - np2)) * K + k;
        rows[t * L + l] = (int32_t)v;
    }
}

// AttnPool forward with the probabilities kept: P[o, c] (c < n; 0 when
// masked) and P[o, n] (null token). One warp per output; d <= 128.
__global__ void __launch_bounds__(TT)
    k_tr_attn(const float* __restrict__ key, const float* __restrict__ V, int d,
              const int32_t* __restrict__ rows, int n, int64_t n_out, float scale,
              const float* __restrict__ null_k, const float* __restrict__ null_v,
              float* __restrict__ out, float* __restrict__ P) {
    const int64_t o = ((int64_t)blockIdx.x * TT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (o >= n_out) return;
    const float sn = null_k[0] * scale;
    float mx = sn;
    for (int c = 0; c < n; c++) {
        const int64_t r = rows ? rows[o * n + c] : o * n + c;
        if (r >= 0) mx = fmaxf(mx, key[r] * scale);
    }
    float den = expf(sn - mx);
    for (int c = 0; c < n; c++) {
        const int64_t r = rows ? rows[o * n + c] : o * n + c;
        if (r >= 0) den += expf(key[r] * scale - mx);
    }
    const float inv = 1.0f / den;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int c = 0; c < n; c++) {
        const int64_t r = rows ? rows[o * n + c] : o * n + c;
        const float p = r >= 0 ? expf(key[r] * scale - mx) * inv : 0.0f;
        if (lane == 0) P[o * (n + 1) + c] = p;
        if (r < 0) continue;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int f = lane + 32 * q;
            if (f < d) acc[q] += p * V[r * d + f];
        }
    }
    const float pn = expf(sn - mx) * inv;
    if (lane == 0) P[o * (n + 1) + n] = pn;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int f = lane + 32 * q;
        if (f < d) out[o * d + f] = acc[q] + pn * null_v[f];
    }
}

// AttnPool backward: dkey[r] = p (dot(dout, v) - sum) * scale, dV[r] = p dout
// (each candidate row belongs to one output), null key / value by atomics.
__global__ void __launch_bounds__(TT)
    k_tr_attn_bwd(const float* __restrict__ V, int d, const int32_t* __restrict__ rows, int n,
                  int64_t n_out, float scale, const float* __restrict__ null_v,
                  const float* __restrict__ P, const float* __restrict__ dout,
                  float* __restrict__ dkey, float* __restrict__ dV, float* __restrict__ dnull_k,
                  float* __restrict__ dnull_v) {
    const int64_t o = ((int64_t)blockIdx.x * TT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (o >= n_out) return;
    float go[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int f = lane + 32 * q;
        go[q] = f < d ? dout[o * d + f] : 0.0f;
    }
    auto dot = [&](const float* v) {
        float s = 0.0f;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int f = lane + 32 * q;
            if (f < d) s += go[q] * v[f];
        }
#pragma unroll
        for (int m = 16; m; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
        return s;
    };
    const float pn = P[o * (n + 1) + n];
    const float dpn = dot(null_v);
    float sum = pn * dpn;
    for (int c = 0; c < n; c++) {
        const int64_t r = rows ? rows[o * n + c] : o * n + c;
        if (r < 0) continue;
        sum += P[o * (n + 1) + c] * dot(V + r * d);
    }
    for (int c = 0; c < n; c++) {
        const int64_t r = rows ? rows[o * n + c] : o * n + c;
        if (r < 0) continue;
        const float p = P[o * (n + 1) + c];
        const float dp = dot(V + r * d);
        if (lane == 0) dkey[r] = p * (dp - sum) * scale;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int f = lane + 32 * q;
            if (f < d) dV[r * d + f] = p * go[q];
        }
    }
    if (lane == 0) atomicAdd(dnull_k, pn * (dpn - sum) * scale);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int f = lane + 32 * q;
        if (f < d) atomicAdd(&dnull_v[f], pn * go[q]);
    }
}

// Head rows [pooled | log2 eb_b] (per-sample bound) and the readout
// mu = sigmoid(o0), log2 b = log2 eb_b + clamp(o1, -4, 12), with its backward.
__global__ void __launch_bounds__(TT)
    k_tr_head_rows(const float* __restrict__ pooled, int64_t n, int per_b, int d,
                   const float* __restrict__ log_eb, float* __restrict__ X) {
    const int64_t t = (int64_t)blockIdx.x * TT + threadIdx.x;
    if (t >= n * (d + 1)) return;
    const int64_t r = t / (d + 1);
    const int f = (int)(t % (d + 1));
    X[t] = f < d ? pooled[r * d + f] : log_eb[r / per_b];
}

__global__ void __launch_bounds__(TT)
    k_tr_head_out(const float* __restrict__ O, int64_t n, int per_b, const float* __restrict__ log_eb,
                  float* __restrict__ mu, float* __restrict__ log_b) {
    const int64_t r = (int64_t)blockIdx.x * TT + threadIdx.x;
    if (r >= n) return;
    mu[r] = 1.0f / (1.0f + expf(-O[2 * r]));
    log_b[r] = log_eb[r / per_b] + fminf(fmaxf(O[2 * r + 1], -4.0f), 12.0f);
}

__global__ void __launch_bounds__(TT)
    k_tr_head_out_bwd(const float* __restrict__ O, const float* __restrict__ mu, int64_t n,
                      const float* __restrict__ dmu, const float* __restrict__ dlog_b,
                      float* __restrict__ dO) {
    const int64_t r = (int64_t)blockIdx.x * TT + threadIdx.x;
    if (r >= n) return;
    const float m = mu[r], z = O[2 * r + 1];
    dO[2 * r] = dmu[r] * m * (1.0f - m);
    dO[2 * r + 1] = (z >= -4.0f && z <= 12.0f) ? dlog_b[r] : 0.0f;
}

// Discretised-Laplace code length in bits of target under (mu, 2^log_b) with
// the +-eb cell (train_gnn.py discretized_laplace_nll) plus mse_weight x the
// squared prediction error; sums into acc[0] (bits), acc[1] (squared error),
// acc[2] (|error|) and the gradients scaled by `scale` into dmu / dlog_b.
__global__ void __launch_bounds__(TT)
    k_tr_loss(const float* __restrict__ mu, const float* __restrict__ log_b,
              const float* __restrict__ tgt, int64_t n, int per_b, const float* __restrict__ eb,
              float mse_weight, float scale, float* __restrict__ dmu, float* __restrict__ dlog_b,
              double* __restrict__ acc) {
    const int64_t i = (int64_t)blockIdx.x * TT + threadIdx.x;
    float bits = 0.0f, sq = 0.0f, ab = 0.0f;
    if (i < n) {
        const float LN2 = 0.69314718055994531f, LOG2E = 1.4426950408889634f;
        const float e_b = eb[i / per_b];
        const float b = fmaxf(exp2f(log_b[i]), 1.17549435e-38f);
        const float r = tgt[i] - mu[i];
        const float ar = fabsf(r);
        const float rho = ar / b, e = e_b / b;
        float dl_drho, dl_de, logp;
        if (ar >= e_b) {
            const float em2 = -2.0f * e;
            const float eps = 1.1920929e-07f;
            const bool clamped = em2 > -eps;
            const float x2 = clamped ? -eps : em2;
            const float tail = log1pf(-expf(x2));
            const float dtail = clamped ? 0.0f : 2.0f * expf(x2) / (1.0f - expf(x2));
            float t = rho - e, dt = 1.0f;
            const float tmax = 32.0f * LN2;
            if (t > tmax) {
                dt = 1.0f / (1.0f + (t - tmax));
                t = tmax + log1pf(t - tmax);
            }
            logp = -LN2 - t + tail;
            dl_drho = -dt;
            dl_de = dt + dtail;
        } else {
            const float a = expf(-(e - rho)), c = expf(-(e + rho));
            const float cp = 1.0f - 0.5f * a - 0.5f * c;
            const float ok = cp > 1e-30f ? 1.0f / cp : 0.0f;
            logp = logf(fmaxf(cp, 1e-30f));
            dl_drho = (-0.5f * a + 0.5f * c) * ok;
            dl_de = (0.5f * a + 0.5f * c) * ok;
        }
        bits = -logp * LOG2E;
        sq = r * r;
        ab = ar;
        // d(bits)/d mu: rho depends on |t - mu|; d/d log_b through rho and e
        const float sgn = r > 0.0f ? 1.0f : (r < 0.0f ? -1.0f : 0.0f);
        const float dbits_dmu = -LOG2E * dl_drho * (-sgn / b);
        const float dbits_dlb = -LOG2E * (dl_drho * (-rho * LN2) + dl_de * (-e * LN2));
        dmu[i] = scale * (dbits_dmu + mse_weight * 2.0f * (mu[i] - tgt[i]));
        dlog_b[i] = scale * dbits_dlb;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        bits += __shfl_xor_sync(0xffffffffu, bits, o);
        sq += __shfl_xor_sync(0xffffffffu, sq, o);
        ab += __shfl_xor_sync(0xffffffffu, ab, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[0], (double)bits);
        atomicAdd(&acc[1], (double)sq);
        atomicAdd(&acc[2], (double)ab);
    }
}

// MixEmbed rows [ctx(b, m, k) | value_emb(b, m)] and backward (dctx added,
// dvemb summed over k by atomics).
__global__ void __launch_bounds__(TT)
    k_tr_mix_rows(const float* __restrict__ ctx, const float* __restrict__ vemb, int64_t bmk, int K,
                  int d, float* __restrict__ X) {
    const int64_t t = (int64_t)blockIdx.x * TT + threadIdx.x;
    if (t >= bmk * 2 * d) return;
    const int64_t row = t / (2 * d);
    const int f = (int)(t % (2 * d));
    X[t] = f < d ? ctx[row * d + f] : vemb[(row / K) * d + (f - d)];
}

__global__ void __launch_bounds__(TT)
    k_tr_mix_rows_bwd(const float* __restrict__ dX, int64_t bmk, int K, int d,
                      float* __restrict__ dctx, float* __restrict__ dvemb) {
    const int64_t t = (int64_t)blockIdx.x * TT + threadIdx.x;
    if (t >= bmk * 2 * d) return;
    const int64_t row = t / (2 * d);
    const int f = (int)(t % (2 * d));
    if (f < d) dctx[row * d + f] += dX[t];
    else atomicAdd(&dvemb[(row / K) * d + (f - d)], dX[t]);
}

// E[b, query[m], k, :] = Y[(b M + m) K + k, :] and its backward dY = dE[...].
__global__ void __launch_bounds__(TT)
    k_tr_scatter_e(const float* __restrict__ Y, const int32_t* __restrict__ query, int B, int M,
                   int K, int d, int64_t N, float* __restrict__ E, int backward) {
    const int64_t t = (int64_t)blockIdx.x * TT + threadIdx.x;
    if (t >= (int64_t)B * M * K * d) return;
    const int f = (int)(t % d);
    const int64_t row = t / d;
    const int k = (int)(row % K);
    const int64_t bm = row / K;
    const int m = (int)(bm % M), b = (int)(bm / M);
    const int64_t e = (((int64_t)b * N + query[m]) * K + k) * d + f;
    if (backward) ((float*)Y)[t] = E[e];
    else E[e] = Y[t];
}

// AdamW (decoupled weight decay) and the EMA of the weights.
__global__ void __launch_bounds__(TT)
    k_adamw(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float wd,
            float c1, float c2) {
    const int64_t i = (int64_t)blockIdx.x * TT + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] * (1.0f - lr * wd);
    pi -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
}

__global__ void __launch_bounds__(TT)
    k_ema(float* __restrict__ shadow, const float* __restrict__ p, int64_t n, float decay) {
    const int64_t i = (int64_t)blockIdx.x * TT + threadIdx.x;
    if (i < n) shadow[i] = shadow[i] * decay + p[i] * (1.0f - decay);
}

int done(int n) {
    count_launches((unsigned)n);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

int linear_fwd(int prec, const float* X, int64_t ldx, int64_t rows, int32_t in, const float* W,
               const float* b, int32_t out, float* Y, int64_t ldy, int32_t act, float* Z,
               void* stream) {
    if (rows < 0 || in < 1 || out < 1 || !W || (rows && (!X || !Y)) || rows > 0x7fffffff)
        return LATEC_ERR_ARG;
    if (!rows) return LATEC_OK;
    return done(gemm<0, 1, 0, 0>(prec, (int)rows, out, in, 1, X, ldx, W, in, nullptr, Y, ldy, b,
                                 act, Z, ldy, (cudaStream_t)stream));
}

int linear_bwd(int prec, const float* X, int64_t ldx, int64_t rows, int32_t in, const float* W,
               int32_t out, const float* dY, int64_t ldy, const float* Z, int32_t act, float* dX,
               int64_t lddx, int32_t accum_dx, float* dW, float* db, void* stream) {
    if (rows < 0 || in < 1 || out < 1 || !W || !dW || !db || (act && !Z) ||
        (rows && (!X || !dY)) || rows > 0x7fffffff)
        return LATEC_ERR_ARG;
    if (!rows) return LATEC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const float* Zg = act ? Z : nullptr;
    const int r = (int)rows;
    int n = 0;
    if (dX) {  // dX (rows, in) = dZ (rows, out) W (out, in)
        if (act)
            n += accum_dx ? gemm<0, 0, 1, 1>(prec, r, in, out, 1, dY, ldy, W, in, Zg, dX, lddx,
                                             nullptr, 0, nullptr, 0, st)
                          : gemm<0, 0, 1, 0>(prec, r, in, out, 1, dY, ldy, W, in, Zg, dX, lddx,
                                             nullptr, 0, nullptr, 0, st);
        else
            n += accum_dx ? gemm<0, 0, 0, 1>(prec, r, in, out, 1, dY, ldy, W, in, nullptr, dX,
                                             lddx, nullptr, 0, nullptr, 0, st)
                          : gemm<0, 0, 0, 0>(prec, r, in, out, 1, dY, ldy, W, in, nullptr, dX,
                                             lddx, nullptr, 0, nullptr, 0, st);
    }
    // dW[j, i] += sum_r dZ[r, j] X[r, i]: split over rows
    const unsigned splits = (unsigned)std::min<int64_t>(256, (rows + 4095) / 4096);
    if (act)
        n += gemm<1, 0, 1, 1>(prec, out, in, r, splits ? splits : 1, dY, ldy, X, ldx, Zg, dW, in,
                              nullptr, 0, nullptr, 0, st);
    else
        n += gemm<1, 0, 0, 1>(prec, out, in, r, splits ? splits : 1, dY, ldy, X, ldx, nullptr, dW,
                              in, nullptr, 0, nullptr, 0, st);
    dim3 gb((unsigned)std::min<int64_t>(1024, (rows + TT - 1) / TT), (unsigned)out, 1);
    k_colsum<<<gb, TT, 0, st>>>(rows, out, dY, ldy, Zg, db);
    return done(n + 1);
}

}  // namespace
}  // namespace latec

using namespace latec;

extern "C" {

// Y = act(X W^T + b) (act 1 = GELU); Z (optional) keeps the pre-activation.
int latec_tr_linear(const float* X, int64_t ldx, int64_t rows, int32_t in, const float* W,
                    const float* b, int32_t out, float* Y, int64_t ldy, int32_t act, float* Z,
                    void* stream) {
    return linear_fwd(0, X, ldx, rows, in, W, b, out, Y, ldy, act, Z, stream);
}

int latec_tr_linear_bf16(const float* X, int64_t ldx, int64_t rows, int32_t in, const float* W,
                         const float* b, int32_t out, float* Y, int64_t ldy, int32_t act, float* Z,
                         void* stream) {
    return linear_fwd(1, X, ldx, rows, in, W, b, out, Y, ldy, act, Z, stream);
}

// Backward of latec_tr_linear. dY (rows, ldy); Z = the saved pre-activation
// when act (same ld as dY). dX (optional) = dZ W is stored, or added when
// accum_dx; dW (out, in) and db (out) are accumulated.
int latec_tr_linear_bwd(const float* X, int64_t ldx, int64_t rows, int32_t in, const float* W,
                        int32_t out, const float* dY, int64_t ldy, const float* Z, int32_t act,
                        float* dX, int64_t lddx, int32_t accum_dx, float* dW, float* db,
                        void* stream) {
    return linear_bwd(0, X, ldx, rows, in, W, out, dY, ldy, Z, act, dX, lddx, accum_dx, dW, db,
                      stream);
}

int latec_tr_linear_bwd_bf16(const float* X, int64_t ldx, int64_t rows, int32_t in,
                             const float* W, int32_t out, const float* dY, int64_t ldy,
                             const float* Z, int32_t act, float* dX, int64_t lddx,
                             int32_t accum_dx, float* dW, float* db, void* stream) {
    return linear_bwd(1, X, ldx, rows, in, W, out, dY, ldy, Z, act, dX, lddx, accum_dx, dW, db,
                      stream);
}

// Reads and clears the tensor-core GEMMs' error word (bit 0: an MMA wait ran
// out). Synchronises the stream.
int latec_tr_gemm_status(void* stream) {
    uint32_t e = 0;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemcpyFromSymbolAsync(&e, g_gemm_tc_err, sizeof e, 0, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    if (!e) return LATEC_OK;
    const uint32_t zero = 0;
    if (cudaMemcpyToSymbolAsync(g_gemm_tc_err, &zero, sizeof zero, 0, cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    return LATEC_ERR_INTERNAL;
}

int latec_tr_rows(const float* E, int64_t N, int32_t K, int32_t d, int32_t ds, const float* table,
                  const latec_gnn_geom* geom, const int32_t* pairs, int64_t np, int32_t B,
                  int32_t two, float* X, int32_t ldx, void* stream) {
    if (!E || !table || !geom || np < 0 || B < 1 || (np && (!pairs || !X)) || d > 128)
        return LATEC_ERR_ARG;
    if (!np) return LATEC_OK;
    k_tr_rows<<<tblocks((int64_t)B * np * K * 32), TT, 0, (cudaStream_t)stream>>>(
        E, N, K, d, ds, table, *geom, pairs, np, B, two, X, ldx);
    return done(1);
}

int latec_tr_rows_bwd(const float* dX, int32_t ldx, int64_t N, int32_t K, int32_t d, int32_t ds,
                      const latec_gnn_geom* geom, const int32_t* pairs, int64_t np, int32_t B,
                      int32_t two, float* dE, float* dtable, void* stream) {
    if (!geom || np < 0 || B < 1 || (np && (!pairs || !dX || !dE || !dtable)))
        return LATEC_ERR_ARG;
    if (!np) return LATEC_OK;
    k_tr_rows_bwd<<<tblocks((int64_t)B * np * K * 32), TT, 0, (cudaStream_t)stream>>>(
        dX, ldx, N, K, d, ds, *geom, pairs, np, B, two, dE, dtable);
    return done(1);
}

int latec_tr_line_rows(const int32_t* row_of, int32_t M, int32_t L, int32_t K, int32_t B,
                       int64_t np2, int64_t np1, int32_t* rows, void* stream) {
    if (!row_of || !rows || M < 0 || L < 1 || K < 1 || B < 1 || np2 < 0 || np1 < 0 ||
        (int64_t)B * (np2 + np1) * K > 0x7fffffffLL)
        return LATEC_ERR_ARG;
    if (!M) return LATEC_OK;
    k_tr_line_rows<<<tblocks((int64_t)B * M * K), TT, 0, (cudaStream_t)stream>>>(row_of, M, L, K, B,
                                                                                 np2, np1, rows);
    return done(1);
}

int latec_tr_attn(const float* key, const float* V, int32_t d, const int32_t* rows, int32_t n,
                  int64_t n_out, float scale, const float* null_k, const float* null_v, float* out,
                  float* P, void* stream) {
    if (!key || !V || !null_k || !null_v || !out || !P || d < 1 || d > 128 || n < 1 || n_out < 0)
        return LATEC_ERR_ARG;
    if (!n_out) return LATEC_OK;
    k_tr_attn<<<tblocks(n_out * 32), TT, 0, (cudaStream_t)stream>>>(key, V, d, rows, n, n_out, scale,
                                                                   null_k, null_v, out, P);
    return done(1);
}

int latec_tr_attn_bwd(const float* V, int32_t d, const int32_t* rows, int32_t n, int64_t n_out,
                      float scale, const float* null_v, const float* P, const float* dout,
                      float* dkey, float* dV, float* dnull_k, float* dnull_v, void* stream) {
    if (!V || !null_v || !P || !dout || !dkey || !dV || !dnull_k || !dnull_v || d < 1 || d > 128 ||
        n < 1 || n_out < 0)
        return LATEC_ERR_ARG;
    if (!n_out) return LATEC_OK;
    k_tr_attn_bwd<<<tblocks(n_out * 32), TT, 0, (cudaStream_t)stream>>>(
        V, d, rows, n, n_out, scale, null_v, P, dout, dkey, dV, dnull_k, dnull_v);
    return done(1);
}

int latec_tr_head_rows(const float* pooled, int64_t n, int32_t per_b, int32_t d,
                       const float* log_eb, float* X, void* stream) {
    if (!pooled || !log_eb || !X || n < 0 || per_b < 1) return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    k_tr_head_rows<<<tblocks(n * (d + 1)), TT, 0, (cudaStream_t)stream>>>(pooled, n, per_b, d,
                                                                         log_eb, X);
    return done(1);
}

int latec_tr_head_out(const float* O, int64_t n, int32_t per_b, const float* log_eb, float* mu,
                      float* log_b, void* stream) {
    if (!O || !log_eb || !mu || !log_b || n < 0 || per_b < 1) return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    k_tr_head_out<<<tblocks(n), TT, 0, (cudaStream_t)stream>>>(O, n, per_b, log_eb, mu, log_b);
    return done(1);
}

int latec_tr_head_out_bwd(const float* O, const float* mu, int64_t n, const float* dmu,
                          const float* dlog_b, float* dO, void* stream) {
    if (!O || !mu || !dmu || !dlog_b || !dO || n < 0) return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    k_tr_head_out_bwd<<<tblocks(n), TT, 0, (cudaStream_t)stream>>>(O, mu, n, dmu, dlog_b, dO);
    return done(1);
}

int latec_tr_loss(const float* mu, const float* log_b, const float* tgt, int64_t n, int32_t per_b,
                  const float* eb, float mse_weight, float scale, float* dmu, float* dlog_b,
                  double* acc, void* stream) {
    if (!mu || !log_b || !tgt || !eb || !dmu || !dlog_b || !acc || n < 0 || per_b < 1)
        return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    k_tr_loss<<<tblocks(n), TT, 0, (cudaStream_t)stream>>>(mu, log_b, tgt, n, per_b, eb, mse_weight,
                                                          scale, dmu, dlog_b, acc);
    return done(1);
}

int latec_tr_mix_rows(const float* ctx, const float* vemb, int64_t bmk, int32_t K, int32_t d,
                      float* X, void* stream) {
    if (!ctx || !vemb || !X || bmk < 0 || K < 1) return LATEC_ERR_ARG;
    if (!bmk) return LATEC_OK;
    k_tr_mix_rows<<<tblocks(bmk * 2 * d), TT, 0, (cudaStream_t)stream>>>(ctx, vemb, bmk, K, d, X);
    return done(1);
}

int latec_tr_mix_rows_bwd(const float* dX, int64_t bmk, int32_t K, int32_t d, float* dctx,
                          float* dvemb, void* stream) {
    if (!dX || !dctx || !dvemb || bmk < 0 || K < 1) return LATEC_ERR_ARG;
    if (!bmk) return LATEC_OK;
    k_tr_mix_rows_bwd<<<tblocks(bmk * 2 * d), TT, 0, (cudaStream_t)stream>>>(dX, bmk, K, d, dctx,
                                                                            dvemb);
    return done(1);
}

// backward = 0: E[query] = Y; backward = 1: Y = dE[query] (Y is then written).
int latec_tr_scatter_e(float* Y, const int32_t* query, int32_t B, int32_t M, int32_t K, int32_t d,
                       int64_t N, float* E, int32_t backward, void* stream) {
    if (!Y || !query || !E || B < 1 || M < 0 || K < 1) return LATEC_ERR_ARG;
    if (!M) return LATEC_OK;
    k_tr_scatter_e<<<tblocks((int64_t)B * M * K * d), TT, 0, (cudaStream_t)stream>>>(
        Y, query, B, M, K, d, N, E, backward);
    return done(1);
}

int latec_tr_adamw(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1,
                   float b2, float eps, float wd, int64_t step, void* stream) {
    if (!p || !g || !m || !v || n < 0 || step < 1) return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adamw<<<tblocks(n), TT, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, wd, c1, c2);
    return done(1);
}

int latec_tr_ema(float* shadow, const float* p, int64_t n, float decay, void* stream) {
    if (!shadow || !p || n < 0) return LATEC_ERR_ARG;
    if (!n) return LATEC_OK;
    k_ema<<<tblocks(n), TT, 0, (cudaStream_t)stream>>>(shadow, p, n, decay);
    return done(1);
}

}  // extern "C"
