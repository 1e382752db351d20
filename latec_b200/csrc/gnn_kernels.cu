// Axial GNN predictor of the learned path (latec/gnn_predictor.py:593-1000):
// the per-axis message pass with attention pooling (GNN.embed), the axis pool
// and Laplace head (GNN.head_of / PredHead) and the finalisation of revealed
// points (GNN.finalize: InitEmbed + MixEmbed).
//
// float32 storage and arithmetic with float32 accumulation in a fixed order:
// every output element is one thread's sum over the input features in
// ascending order, so a stage evaluates identically on every run, in the
// encoder and in the decoder.
//
// Parameters are one packed float32 buffer in the reference state_dict order
// (see carve()); E is the (B, N, K, d) embedding field; contexts are
// (B, M, K, d).
#include <cuda_runtime.h>

#include <cstdint>

#include "latec_common.cuh"


namespace latec {

int mlp2_tc(const float* X, int ldx, int64_t rows, int k1, int k1p, const void* w1p,
            const float* b1, const void* w2p, const float* b2, int n1, int n2, float* Y, int ldy,
            int ny, uint32_t* err, int n_sm, cudaStream_t st);
int mlp2_tc_gather(const RowGather& rg, int two_sided, int64_t rows, int k1, int k1p,
                   const void* w1p, const float* b1, const void* w2p, const float* b2, float* Y,
                   int ldy, uint32_t* err, int n_sm, cudaStream_t st);
int kv_tc(const float* X, int ldx, int64_t rows, const void* w1p, const float* b1,
          const float* bv, const void* w2p, const float* b2, float* KEY, float* V, int ldv,
          uint32_t* err, int n_sm, cudaStream_t st);
int mlp2_tc8(const float* X, int ldx, int64_t rows, int k1, int k1p, const void* w1p,
             const float* s1, const float* b1, const void* w2p, const float* s2, const float* b2,
             int n1, int n2, float* Y, int ldy, uint32_t* err, int n_sm, cudaStream_t st);

namespace {

constexpr int LT = 256;  // threads of every kernel here
constexpr int BN = 64, BK = 16;

__device__ __forceinline__ float gelu(float x) {
    return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}

// Y[r, j] = act(b[j] + sum_i X[r, i] * W[j, i]); X row stride ldx, Y row
// stride ldy. 128 x 64 output tile per CTA, 8 x 4 per thread (operands read
// as 128-bit shared-memory vectors), k ascending over the zero-padded range
// [0, in rounded up to BK), accumulated with fused multiply-adds.
constexpr int BMR = 128;  // rows of a k_linear tile

template <int ACT>
__global__ void __launch_bounds__(LT)
    k_linear(const float* __restrict__ X, int ldx, int rows, int in, const float* __restrict__ W,
             const float* __restrict__ b, int out, float* __restrict__ Y, int ldy) {
    __shared__ __align__(16) float xs[BK][BMR + 4];
    __shared__ __align__(16) float ws[BK][BN + 4];
    const int r0 = blockIdx.x * BMR, j0 = blockIdx.y * BN;
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    float acc[8][4];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[a][c] = 0.0f;
    for (int k0 = 0; k0 < in; k0 += BK) {
        for (int e = threadIdx.x; e < BMR * BK; e += LT) {
            const int rr = e / BK, kk = e % BK;
            const int r = r0 + rr, k = k0 + kk;
            xs[kk][rr] = (r < rows && k < in) ? X[(int64_t)r * ldx + k] : 0.0f;
        }
        for (int e = threadIdx.x; e < BN * BK; e += LT) {
            const int jj = e / BK, kk = e % BK;
            const int j = j0 + jj, k = k0 + kk;
            ws[kk][jj] = (j < out && k < in) ? W[(int64_t)j * in + k] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            const float4 xa = *reinterpret_cast<const float4*>(&xs[kk][tr * 8]);
            const float4 xb = *reinterpret_cast<const float4*>(&xs[kk][tr * 8 + 4]);
            const float4 w4 = *reinterpret_cast<const float4*>(&ws[kk][tc * 4]);
            const float xv[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
            const float wv[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int a = 0; a < 8; a++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[a][c] = __fadd_rn(acc[a][c], __fmul_rn(xv[a], wv[c]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 8; a++) {
        const int r = r0 + tr * 8 + a;
        if (r >= rows) continue;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int j = j0 + tc * 4 + c;
            if (j >= out) continue;
            float v = __fadd_rn(acc[a][c], b[j]);
            if (ACT) v = gelu(v);
            Y[(int64_t)r * ldy + j] = v;
        }
    }
}

// Y[r, j] = b[j] + sum_i X[r, i] * W[j, i] for OUT <= 2 outputs (the pools'
// key layers, the head's output layer), which k_linear's 64-wide output tile
// would compute 32 to 64 times over: one thread per row, the CTA's rows
// staged through shared memory NK columns at a time. The sum runs over the
// same zero-padded k range as k_linear (in rounded up to BK) in the same
// order, with the products and sums rounded separately: the same bits.
constexpr int NK = 32;

template <int OUT>
__global__ void __launch_bounds__(LT)
    k_linear_narrow(const float* __restrict__ X, int ldx, int rows, int in,
                    const float* __restrict__ W, const float* __restrict__ b,
                    float* __restrict__ Y, int ldy) {
    __shared__ float xs[LT][NK + 1];
    __shared__ float ws[OUT][NK];
    const int64_t r0 = (int64_t)blockIdx.x * LT;
    const int inp = (in + BK - 1) / BK * BK;
    float acc[OUT];
#pragma unroll
    for (int j = 0; j < OUT; j++) acc[j] = 0.0f;
    for (int k0 = 0; k0 < inp; k0 += NK) {
        for (int e = threadIdx.x; e < LT * NK; e += LT) {  // a warp reads 32 columns of a row
            const int rr = e / NK, kk = e % NK;
            const int64_t r = r0 + rr;
            const int k = k0 + kk;
            xs[rr][kk] = (r < rows && k < in) ? X[r * ldx + k] : 0.0f;
        }
        if (threadIdx.x < OUT * NK) {
            const int j = threadIdx.x / NK, k = k0 + threadIdx.x % NK;
            ws[j][threadIdx.x % NK] = k < in ? W[(int64_t)j * in + k] : 0.0f;
        }
        __syncthreads();
        const int kn = inp - k0 < NK ? inp - k0 : NK;
        for (int kk = 0; kk < kn; kk++) {
            const float xv = xs[threadIdx.x][kk];
#pragma unroll
            for (int j = 0; j < OUT; j++) acc[j] = __fadd_rn(acc[j], __fmul_rn(xv, ws[j][kk]));
        }
        __syncthreads();
    }
    const int64_t r = r0 + threadIdx.x;
    if (r < rows) {
#pragma unroll
        for (int j = 0; j < OUT; j++) Y[r * ldy + j] = __fadd_rn(acc[j], b[j]);
    }
}

// Two-sided message rows [e_neg | state_neg | e_pos | state_pos | logd_neg | logd_pos]
// (BiDirEmbed input order), one warp per (pair, axis) row.
__global__ void __launch_bounds__(LT)
    k_rows_two(const float* __restrict__ E, int64_t N, int K, int d, int ds,
               const float* __restrict__ table, const latec_gnn_geom g, int b,
               const int32_t* __restrict__ pairs, int64_t np, float* __restrict__ X, int ldx) {
    const int64_t w = ((int64_t)blockIdx.x * LT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= np * K) return;
    const int64_t p = w / K;
    const int k = (int)(w % K);
    const int pair = pairs[p];
    const int l = pair / g.M;
    const int64_t in_ = g.nbr_n[pair], ip = g.nbr_p[pair];
    const float* en = E + (((int64_t)b * N + in_) * K + k) * d;
    const float* ep = E + (((int64_t)b * N + ip) * K + k) * d;
    const float* sn = table + (int64_t)g.sidx_n[l * K + k] * ds;
    const float* sp = table + (int64_t)g.sidx_p[l * K + k] * ds;
    const int de = d + ds, width = 2 * de + 2;
    float* row = X + w * ldx;
    for (int f = lane; f < width; f += 32) {
        float v;
        if (f < d) v = en[f];
        else if (f < de) v = sn[f - d];
        else if (f < de + d) v = ep[f - de];
        else if (f < 2 * de) v = sp[f - de - d];
        else if (f == 2 * de) v = g.logd_n[pair];
        else v = g.logd_p[pair];
        row[f] = v;
    }
}

// One-sided message rows [e_side | state_side | sign | logd_side] (DirEmbed).
__global__ void __launch_bounds__(LT)
    k_rows_one(const float* __restrict__ E, int64_t N, int K, int d, int ds,
               const float* __restrict__ table, const latec_gnn_geom g, int b,
               const int32_t* __restrict__ pairs, int64_t np, float* __restrict__ X, int ldx) {
    const int64_t w = ((int64_t)blockIdx.x * LT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= np * K) return;
    const int64_t p = w / K;
    const int k = (int)(w % K);
    const int pair = pairs[p];
    const int l = pair / g.M;
    const bool pos = g.nbr_p[pair] >= 0;
    const int64_t nb = pos ? g.nbr_p[pair] : g.nbr_n[pair];
    const float* e = E + (((int64_t)b * N + nb) * K + k) * d;
    const float* s = table + (int64_t)(pos ? g.sidx_p[l * K + k] : g.sidx_n[l * K + k]) * ds;
    const int de = d + ds, width = de + 2;
    float* row = X + w * ldx;
    for (int f = lane; f < width; f += 32) {
        float v;
        if (f < d) v = e[f];
        else if (f < de) v = s[f - d];
        else if (f == de) v = pos ? 1.0f : -1.0f;
        else v = pos ? g.logd_p[pair] : g.logd_n[pair];
        row[f] = v;
    }
}

// Candidate rows of the line pool for outputs (m, k), m in [m0, m0 + mt), of
// batch b: line l's live row ((b * n_live + r) * K + k), or -1 (masked).
__global__ void __launch_bounds__(LT)
    k_line_rows(const int32_t* __restrict__ row_of, int M, int L, int K, int b, int m0, int mt,
                int64_t n_live, int32_t* __restrict__ rows) {
    const int64_t t = (int64_t)blockIdx.x * LT + threadIdx.x;
    if (t >= (int64_t)mt * K) return;
    const int k = (int)(t % K);
    const int m = m0 + (int)(t / K);
    for (int l = 0; l < L; l++) {
        const int32_t r = row_of[(int64_t)l * M + m];
        rows[t * L + l] = r >= 0 ? (int32_t)(((int64_t)b * n_live + r) * K + k) : -1;
    }
}

// AttnPool (latec/gnn_predictor.py:724-749) for n_out outputs of n candidates:
// scores s_c = key_c * scale (masked candidates excluded), the null token's
// score null_k * scale, softmax, and the weighted sum of the values. rows ==
// nullptr means candidate c of output o is row o * n + c. One warp per
// output; d <= 128.
__global__ void __launch_bounds__(LT)
    k_attn(const float* __restrict__ key, const float* __restrict__ V, int d,
           const int32_t* __restrict__ rows, int n, int64_t n_out, float scale,
           const float* __restrict__ null_k, const float* __restrict__ null_v,
           float* __restrict__ out) {
    const int64_t o = ((int64_t)blockIdx.x * LT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (o >= n_out) return;
    const float sn = __fmul_rn(null_k[0], scale);
    float mx = sn;
    for (int c = 0; c < n; c++) {
        const int64_t r = rows ? rows[o * n + c] : o * n + c;
        if (r >= 0) mx = fmaxf(mx, __fmul_rn(key[r], scale));
    }
    float den = 0.0f;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int c = 0; c < n; c++) {
        const int64_t r = rows ? rows[o * n + c] : o * n + c;
        if (r < 0) continue;
        const float p = expf(__fsub_rn(__fmul_rn(key[r], scale), mx));
        den = __fadd_rn(den, p);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int f = lane + 32 * q;
            if (f < d) acc[q] = __fadd_rn(acc[q], __fmul_rn(p, V[r * d + f]));
        }
    }
    const float pn = expf(__fsub_rn(sn, mx));
    den = __fadd_rn(den, pn);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int f = lane + 32 * q;
        if (f < d) out[o * d + f] = __fdiv_rn(__fadd_rn(acc[q], __fmul_rn(pn, null_v[f])), den);
    }
}

// Head input rows [pooled (d) | log2 eb].
__global__ void __launch_bounds__(LT)
    k_head_rows(const float* __restrict__ pooled, int64_t n, int d, float log_eb,
                float* __restrict__ X) {
    const int64_t t = (int64_t)blockIdx.x * LT + threadIdx.x;
    if (t >= n * (d + 1)) return;
    const int64_t r = t / (d + 1);
    const int f = (int)(t % (d + 1));
    X[t] = f < d ? pooled[r * d + f] : log_eb;
}

// mu = sigmoid(o0), log2 b = log2 eb + clamp(o1, -4, 12) (PredHead.forward).
__global__ void __launch_bounds__(LT)
    k_head_out(const float* __restrict__ O, int64_t n, float log_eb, float* __restrict__ mu,
               float* __restrict__ log_b) {
    const int64_t r = (int64_t)blockIdx.x * LT + threadIdx.x;
    if (r >= n) return;
    const float a = O[2 * r], z = O[2 * r + 1];
    mu[r] = __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-a)));
    log_b[r] = __fadd_rn(log_eb, fminf(fmaxf(z, -4.0f), 12.0f));
}

// MixEmbed input rows [ctx(b, m, k) | value_emb(b, m)].
__global__ void __launch_bounds__(LT)
    k_mix_rows(const float* __restrict__ ctx, const float* __restrict__ vemb, int64_t bmk, int K,
               int d, float* __restrict__ X) {
    const int64_t t = (int64_t)blockIdx.x * LT + threadIdx.x;
    if (t >= bmk * 2 * d) return;
    const int64_t row = t / (2 * d);
    const int f = (int)(t % (2 * d));
    X[t] = f < d ? ctx[row * d + f] : vemb[(row / K) * d + (f - d)];
}

// E[b, query[m], k, :] = Y[(b * M + m) * K + k, :].
__global__ void __launch_bounds__(LT)
    k_scatter_e(const float* __restrict__ Y, const int32_t* __restrict__ query, int B, int M, int K,
                int d, int64_t N, float* __restrict__ E) {
    const int64_t t = (int64_t)blockIdx.x * LT + threadIdx.x;
    if (t >= (int64_t)B * M * K * d) return;
    const int f = (int)(t % d);
    const int64_t row = t / d;
    const int k = (int)(row % K);
    const int64_t bm = row / K;
    const int m = (int)(bm % M), b = (int)(bm / M);
    E[(((int64_t)b * N + query[m]) * K + k) * d + f] = Y[t];
}

// ---- parameter layout: the reference state_dict order ----
struct Params {
    const float *init0w, *init0b, *init2w, *init2b, *table;
    const float *dir0w, *dir0b, *dir2w, *dir2b, *bi0w, *bi0b, *bi2w, *bi2b;
    const float *lp_k0w, *lp_k0b, *lp_k2w, *lp_k2b, *lp_vw, *lp_vb, *lp_nk, *lp_nv;
    const float *ap_k0w, *ap_k0b, *ap_k2w, *ap_k2b, *ap_vw, *ap_vb, *ap_nk, *ap_nv;
    const float *hd0w, *hd0b, *hd2w, *hd2b, *mx0w, *mx0b, *mx2w, *mx2b;
    int d, ds, h, de, states;
    uint64_t count;
};

Params carve(const float* p0, int d, int agg) {
    Params q;
    q.d = d;
    q.h = 2 * d;
    q.ds = d / 4 > 1 ? d / 4 : 1;
    q.de = d + q.ds;
    q.states = 2 * agg + 1;
    const uint64_t h = q.h, ds = q.ds, de = q.de, D = d;
    const float* p = p0;
    auto take = [&](uint64_t n) {
        const float* r = p;
        p += n;
        return r;
    };
    q.init0w = take(D); q.init0b = take(D); q.init2w = take(D * D); q.init2b = take(D);
    q.table = take((uint64_t)q.states * ds);
    q.dir0w = take(h * (de + 2)); q.dir0b = take(h); q.dir2w = take(D * h); q.dir2b = take(D);
    q.bi0w = take(h * (2 * de + 2)); q.bi0b = take(h); q.bi2w = take(D * h); q.bi2b = take(D);
    q.lp_k0w = take(D * D); q.lp_k0b = take(D); q.lp_k2w = take(D); q.lp_k2b = take(1);
    q.lp_vw = take(D * D); q.lp_vb = take(D); q.lp_nk = take(1); q.lp_nv = take(D);
    q.ap_k0w = take(D * D); q.ap_k0b = take(D); q.ap_k2w = take(D); q.ap_k2b = take(1);
    q.ap_vw = take(D * D); q.ap_vb = take(D); q.ap_nk = take(1); q.ap_nv = take(D);
    q.hd0w = take(h * (D + 1)); q.hd0b = take(h); q.hd2w = take(2 * h); q.hd2b = take(2);
    q.mx0w = take(h * 2 * D); q.mx0b = take(h); q.mx2w = take(D * h); q.mx2b = take(D);
    q.count = (uint64_t)(p - p0);
    return q;
}

// Tensor-core copies of the BiDir / Dir / Mix MLP weights (d = 64): each
// layer in the layout of latec_gnn_pack_bf16 (input width padded to 16) or of
// latec_gnn_pack_fp8 (E4M3, padded to 32, one scale per output channel).
struct TcMlp {
    const void* w1 = nullptr;
    const void* w2 = nullptr;
    const float* s1 = nullptr;
    const float* s2 = nullptr;
    int k1p = 0;
    int fp8 = 0;
};
struct Packed {
    TcMlp bi, dir, mix;
    // the line pool's key MLP (64 -> 64 -> 1) in BF16 with the value
    // projection's weights stacked under its first layer (128 x 64), its
    // output layer and bias zero-padded to 32 rows; null when the model
    // carries none
    TcMlp key;
    const float* key_b2 = nullptr;
};

inline int pad16(int k) { return (k + 15) / 16 * 16; }
constexpr int KEY_ROWS = 32;  // rows of the padded key output layer
inline int pad32(int k) { return (k + 31) / 32 * 32; }

Packed packed_of(const latec_gnn_model* m, const Params& P) {
    Packed k;
    const int ins[3] = {2 * P.de + 2, P.de + 2, 2 * P.d};
    TcMlp* mlps[3] = {&k.bi, &k.dir, &k.mix};
    if (m->packed_fp8) {
        const uint8_t* p = (const uint8_t*)m->packed_fp8;
        const float* sc = m->fp8_scales;
        for (int i = 0; i < 3; i++) {
            TcMlp& t = *mlps[i];
            t.fp8 = 1;
            t.k1p = pad32(ins[i]);
            t.w1 = p;
            p += (size_t)P.h * t.k1p;
            t.s1 = sc;
            sc += P.h;
            t.w2 = p;
            p += (size_t)P.d * P.h;
            t.s2 = sc;
            sc += P.d;
        }
    } else if (m->packed_bf16) {
        const uint16_t* p = (const uint16_t*)m->packed_bf16;
        for (int i = 0; i < 3; i++) {
            TcMlp& t = *mlps[i];
            t.k1p = pad16(ins[i]);
            t.w1 = p;
            p += (size_t)P.h * t.k1p;
            t.w2 = p;
            p += (size_t)P.d * P.h;
        }
        // then the line pool's key MLP: [W1; Wv] 2d x d, W2 32 x d, b2 as 32 floats
        k.key.k1p = P.d;
        k.key.w1 = p;
        p += (size_t)2 * P.d * P.d;
        k.key.w2 = p;
        p += (size_t)KEY_ROWS * P.d;
        k.key_b2 = (const float*)p;
    }
    return k;
}

int n_sms() {
    static int n = 0;
    if (!n) {
        int dev = 0, v = 148;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
            n = v;
        else
            n = 148;
    }
    return n;
}

// Two-layer MLP over rows of X: on the tensor cores when the model carries
// packed BF16 or E4M3 weights, else the float32 path.
int mlp2(const latec_gnn_model* m, const float* X, int ldx, int64_t rows, int k1, const float* w1,
         const float* b1, const float* w2, const float* b2, const TcMlp& tc, int h, int d,
         float* H, float* Y, int ldy, cudaStream_t st);

int linear(const float* X, int ldx, int64_t rows, int in, const float* W, const float* b, int out,
           float* Y, int ldy, int act, cudaStream_t st) {
    if (rows <= 0) return LATEC_OK;
    if (rows > 0x7fffffffLL) return LATEC_ERR_UNSUPPORTED;
    if (!act && out <= 2) {
        const unsigned g = (unsigned)((rows + LT - 1) / LT);
        if (out == 1) k_linear_narrow<1><<<g, LT, 0, st>>>(X, ldx, (int)rows, in, W, b, Y, ldy);
        else k_linear_narrow<2><<<g, LT, 0, st>>>(X, ldx, (int)rows, in, W, b, Y, ldy);
        count_launches(1);
        return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
    }
    const dim3 grid((unsigned)((rows + BMR - 1) / BMR), (unsigned)((out + BN - 1) / BN));
    if (act) k_linear<1><<<grid, LT, 0, st>>>(X, ldx, (int)rows, in, W, b, out, Y, ldy);
    else k_linear<0><<<grid, LT, 0, st>>>(X, ldx, (int)rows, in, W, b, out, Y, ldy);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

int mlp2(const latec_gnn_model* m, const float* X, int ldx, int64_t rows, int k1, const float* w1,
         const float* b1, const float* w2, const float* b2, const TcMlp& tc, int h, int d,
         float* H, float* Y, int ldy, cudaStream_t st) {
    if (tc.w1 && tc.fp8)
        return mlp2_tc8(X, ldx, rows, k1, tc.k1p, tc.w1, tc.s1, b1, tc.w2, tc.s2, b2, h, d, Y, ldy,
                        m->tc_err, n_sms(), st);
    if (tc.w1)
        return mlp2_tc(X, ldx, rows, k1, tc.k1p, tc.w1, b1, tc.w2, b2, h, d, Y, ldy, d, m->tc_err,
                       n_sms(), st);
    int rc = linear(X, ldx, rows, k1, w1, b1, h, H, h, 1, st);
    if (!rc) rc = linear(H, h, rows, h, w2, b2, d, Y, ldy, 0, st);
    return rc;
}

unsigned blocks_for(int64_t threads) { return (unsigned)((threads + LT - 1) / LT); }

int launched(int n) {
    count_launches(n);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

bool valid_model(const latec_gnn_model* m) {
    return m && m->params && m->d >= 4 && m->d <= 128 && m->d % 2 == 0 && m->agg_level >= 1 &&
           m->agg_level <= 8 && (!m->packed_bf16 || (m->d == 64 && m->tc_err)) &&
           (!m->packed_fp8 || (m->d == 64 && m->tc_err && m->fp8_scales));
}

}  // namespace
}  // namespace latec

using namespace latec;

extern "C" {

uint64_t latec_gnn_param_count(int32_t d, int32_t agg_level) {
    latec_gnn_model m{d, agg_level, (const float*)16, nullptr, nullptr, nullptr, nullptr};
    if (!valid_model(&m)) return 0;
    return carve(nullptr, d, agg_level).count;
}

// Floats of workspace for one embed tile / one head or finalize call.
uint64_t latec_gnn_workspace_bytes(int32_t d, int32_t B, int32_t M, int32_t L, int32_t K,
                                   int32_t m_tile) {
    if (d < 4 || B < 1 || M < 0 || L < 1 || K < 1 || m_tile < 1) return 0;
    const int64_t mt = M < m_tile ? M : m_tile;
    const int64_t h = 2 * d, de = d + (d / 4 > 1 ? d / 4 : 1);
    const int64_t rows = (int64_t)B * mt * L * K;  // live rows of one tile, at most
    const int64_t embed = rows * ((2 * de + 2 + 3) / 4 * 4 + h + d + d + 1 + d) + (int64_t)mt * K * L;
    const int64_t bm = (int64_t)B * M, bmk = bm * K;
    const int64_t head = bmk * (d + 1 + d) + bm * (d + d + 1 + h + 2);
    const int64_t fin = bm * (h + d) + bmk * (2 * d + h + d);
    int64_t f = embed > head ? embed : head;
    f = f > fin ? f : fin;
    return (uint64_t)(f + 256) * 4;
}

// GNN.embed (latec/gnn_predictor.py:843-871): per-axis contexts of the
// stage's queries, ctx (B, M, K, d), from E (B, N, K, d).
int latec_gnn_embed(const latec_gnn_model* model, int32_t B, int64_t N, const float* E,
                    const latec_gnn_geom* geom, float* ctx, void* workspace,
                    uint64_t workspace_bytes, void* stream) {
    if (!valid_model(model) || !geom || !E || !ctx || B < 1 || N < 1) return LATEC_ERR_ARG;
    const latec_gnn_geom& g = *geom;
    const int d = model->d, K = g.K, L = g.L;
    if (g.M < 0 || L < 1 || K < 1 || g.m_tile < 1 || g.n_tiles < 0) return LATEC_ERR_ARG;
    if (!g.M) return LATEC_OK;
    if (!g.query || !g.nbr_p || !g.nbr_n || !g.logd_p || !g.logd_n || !g.row_of || !g.two_off ||
        !g.one_off || !g.sidx_p || !g.sidx_n || g.n_tiles != (g.M + g.m_tile - 1) / g.m_tile)
        return LATEC_ERR_ARG;
    if (!workspace || workspace_bytes < latec_gnn_workspace_bytes(d, B, g.M, L, K, g.m_tile))
        return LATEC_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    const Params P = carve(model->params, d, model->agg_level);
    const Packed pk = packed_of(model, P);
    const float scale = 1.0f / sqrtf((float)d);
    const int64_t w2 = 2 * P.de + 2, w1 = P.de + 2;
    const int64_t l2 = (w2 + 3) / 4 * 4, l1 = (w1 + 3) / 4 * 4;  // 16-byte row strides
    int rc = LATEC_OK;
    for (int t = 0; t < g.n_tiles && !rc; t++) {
        const int m0 = t * g.m_tile;
        const int mt = (g.M - m0) < g.m_tile ? (g.M - m0) : g.m_tile;
        const int64_t n2 = g.two_off[t + 1] - g.two_off[t], n1 = g.one_off[t + 1] - g.one_off[t];
        const int64_t n_live = n2 + n1;
        if (n2 < 0 || n1 < 0 || n_live > (int64_t)mt * L) return LATEC_ERR_ARG;
        const int64_t rows = (int64_t)B * n_live * K;
        float* X = (float*)workspace;
        float* H = X + rows * l2;
        float* MS = H + rows * P.h;
        float* S1 = MS + rows * d;
        float* KEY = S1 + rows * d;
        float* V = KEY + rows;
        int32_t* cand = (int32_t*)(V + rows * d);
        // BF16 message MLPs gather their rows in the operand staging
        const bool gather = pk.bi.w1 && !pk.bi.fp8 && d == 64 && P.ds == 16;
        for (int b = 0; b < B && !rc; b++) {
            float* msb = MS + (int64_t)b * n_live * K * d;
            RowGather rg{E, N, K, b, g.M, P.table, nullptr, g.nbr_p, g.nbr_n, g.logd_p, g.logd_n,
                         g.sidx_p, g.sidx_n};
            if (n2 && gather) {
                rg.pairs = g.two + g.two_off[t];
                rc = mlp2_tc_gather(rg, 1, n2 * K, (int)w2, pk.bi.k1p, pk.bi.w1, P.bi0b, pk.bi.w2,
                                    P.bi2b, msb, d, model->tc_err, n_sms(), st);
            } else if (n2) {
                k_rows_two<<<blocks_for(n2 * K * 32), LT, 0, st>>>(E, N, K, d, P.ds, P.table, g, b,
                                                                  g.two + g.two_off[t], n2, X,
                                                                  (int)l2);
                rc = launched(1);
                if (!rc)
                    rc = mlp2(model, X, (int)l2, n2 * K, (int)w2, P.bi0w, P.bi0b, P.bi2w, P.bi2b,
                              pk.bi, P.h, d, H, msb, d, st);
            }
            if (n1 && !rc && gather) {
                rg.pairs = g.one + g.one_off[t];
                rc = mlp2_tc_gather(rg, 0, n1 * K, (int)w1, pk.dir.k1p, pk.dir.w1, P.dir0b,
                                    pk.dir.w2, P.dir2b, msb + n2 * K * d, d, model->tc_err,
                                    n_sms(), st);
            } else if (n1 && !rc) {
                k_rows_one<<<blocks_for(n1 * K * 32), LT, 0, st>>>(E, N, K, d, P.ds, P.table, g, b,
                                                                  g.one + g.one_off[t], n1, X,
                                                                  (int)l1);
                rc = launched(1);
                if (!rc)
                    rc = mlp2(model, X, (int)l1, n1 * K, (int)w1, P.dir0w, P.dir0b, P.dir2w,
                              P.dir2b, pk.dir, P.h, d, H, msb + n2 * K * d, d, st);
            }
        }
        // line pool keys and values of every live row: on the tensor cores
        // in one pass over MS when the model carries them in BF16
        if (!rc && pk.key.w1) {
            rc = kv_tc(MS, d, rows, pk.key.w1, P.lp_k0b, P.lp_vb, pk.key.w2, pk.key_b2, KEY, V, d,
                       model->tc_err, n_sms(), st);
        } else {
            if (!rc) rc = linear(MS, d, rows, d, P.lp_k0w, P.lp_k0b, d, S1, d, 1, st);
            if (!rc) rc = linear(S1, d, rows, d, P.lp_k2w, P.lp_k2b, 1, KEY, 1, 0, st);
            if (!rc) rc = linear(MS, d, rows, d, P.lp_vw, P.lp_vb, d, V, d, 0, st);
        }
        for (int b = 0; b < B && !rc; b++) {
            k_line_rows<<<blocks_for((int64_t)mt * K), LT, 0, st>>>(g.row_of, g.M, L, K, b, m0, mt,
                                                                    n_live, cand);
            k_attn<<<blocks_for((int64_t)mt * K * 32), LT, 0, st>>>(
                KEY, V, d, cand, L, (int64_t)mt * K, scale, P.lp_nk, P.lp_nv,
                ctx + ((int64_t)b * g.M + m0) * K * d);
            rc = launched(2);
        }
    }
    return rc;
}

// GNN.head_of + PredHead (latec/gnn_predictor.py:760-790, 922-931): axis
// pool of ctx (B, M, K, d) and the Laplace readout: mu, log_b (B, M).
int latec_gnn_head(const latec_gnn_model* model, int32_t B, int32_t M, int32_t K, const float* ctx,
                   float eb, float* mu, float* log_b, void* workspace, uint64_t workspace_bytes,
                   void* stream) {
    if (!valid_model(model) || B < 1 || M < 0 || K < 1 || !ctx || !mu || !log_b) return LATEC_ERR_ARG;
    if (!M) return LATEC_OK;
    const int d = model->d;
    if (!workspace || workspace_bytes < latec_gnn_workspace_bytes(d, B, M, 1, K, 1))
        return LATEC_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    const Params P = carve(model->params, d, model->agg_level);
    const int64_t bm = (int64_t)B * M, bmk = bm * K;
    float* S1 = (float*)workspace;
    float* KEY = S1 + bmk * d;
    float* V = KEY + bmk;
    float* pooled = V + bmk * d;
    float* X = pooled + bm * d;
    float* H = X + bm * (d + 1);
    float* O = H + bm * P.h;
    int rc = linear(ctx, d, bmk, d, P.ap_k0w, P.ap_k0b, d, S1, d, 1, st);
    if (!rc) rc = linear(S1, d, bmk, d, P.ap_k2w, P.ap_k2b, 1, KEY, 1, 0, st);
    if (!rc) rc = linear(ctx, d, bmk, d, P.ap_vw, P.ap_vb, d, V, d, 0, st);
    if (rc) return rc;
    k_attn<<<blocks_for(bm * 32), LT, 0, st>>>(KEY, V, d, nullptr, K, bm, 1.0f / sqrtf((float)d),
                                                P.ap_nk, P.ap_nv, pooled);
    const float tiny = 1.17549435e-38f;
    const float log_eb = log2f(eb > tiny ? eb : tiny);
    k_head_rows<<<blocks_for(bm * (d + 1)), LT, 0, st>>>(pooled, bm, d, log_eb, X);
    rc = launched(2);
    if (!rc) rc = linear(X, d + 1, bm, d + 1, P.hd0w, P.hd0b, P.h, H, P.h, 1, st);
    if (!rc) rc = linear(H, P.h, bm, P.h, P.hd2w, P.hd2b, 2, O, 2, 0, st);
    if (rc) return rc;
    k_head_out<<<blocks_for(bm), LT, 0, st>>>(O, bm, log_eb, mu, log_b);
    return launched(1);
}

// GNN.finalize (latec/gnn_predictor.py:901-920) for the stage's revealed
// points: E[b, query[m], k] = MixEmbed(ctx[b, m, k], InitEmbed(vals[b, m])).
int latec_gnn_finalize(const latec_gnn_model* model, int32_t B, int64_t N, int32_t M, int32_t K,
                       const int32_t* query, const float* ctx, const float* vals, float* E,
                       void* workspace, uint64_t workspace_bytes, void* stream) {
    if (!valid_model(model) || B < 1 || N < 1 || M < 0 || K < 1) return LATEC_ERR_ARG;
    if (!M) return LATEC_OK;
    if (!query || !ctx || !vals || !E) return LATEC_ERR_ARG;
    const int d = model->d;
    if (!workspace || workspace_bytes < latec_gnn_workspace_bytes(d, B, M, 1, K, 1))
        return LATEC_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    const Params P = carve(model->params, d, model->agg_level);
    const int64_t bm = (int64_t)B * M, bmk = bm * K;
    float* H1 = (float*)workspace;
    float* VE = H1 + bm * P.h;
    float* X = VE + bm * d;
    float* H = X + bmk * 2 * d;
    float* Y = H + bmk * P.h;
    int rc = linear(vals, 1, bm, 1, P.init0w, P.init0b, d, H1, d, 1, st);
    if (!rc) rc = linear(H1, d, bm, d, P.init2w, P.init2b, d, VE, d, 0, st);
    if (rc) return rc;
    k_mix_rows<<<blocks_for(bmk * 2 * d), LT, 0, st>>>(ctx, VE, bmk, K, d, X);
    rc = launched(1);
    const Packed pk = packed_of(model, P);
    if (!rc)
        rc = mlp2(model, X, 2 * d, bmk, 2 * d, P.mx0w, P.mx0b, P.mx2w, P.mx2b, pk.mix, P.h, d, H,
                  Y, d, st);
    if (rc) return rc;
    k_scatter_e<<<blocks_for(bmk * d), LT, 0, st>>>(Y, query, B, M, K, d, N, E);
    return launched(1);
}

}  // extern "C"
