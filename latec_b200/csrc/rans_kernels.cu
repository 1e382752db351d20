// rANS entropy stage on the GPU: the native 32-lane interleaved coder, the
// single-stack compatibility coder, the per-symbol tables they use, and the
// on-device assembly of the stage records into one payload.
//
// Native lane coder (one warp per chunk of 32*K symbols; lane l codes symbols
// 32k + l): 64-bit states in [2^31, 2^63), 24-bit precision, 32-bit words.
// Each step the lanes that renormalise are found with a warp ballot and their
// words land at consecutive positions (ascending lanes within a step, steps in
// decode order), so the decoder reads them back with the same ballot.
//
// Compatibility coder (one thread per stage): the single-stack ANS whose byte
// stream is the reference's (constriction AnsCoder, u32 words, u64 state
// starting at 0, encode in reverse).
#include <cuda_runtime.h>

#include "rans_kernels.cuh"

namespace latec {

constexpr uint32_t PREC = 24;
constexpr uint32_t PMASK = (1u << PREC) - 1u;
constexpr uint64_t LANE_L = 1ull << 31;

// --------------------------------------------------------------- tables
// Encoder symbol: x' = x + bias + mulhi(x, rcp) >> shift * cmpl  (Alverson
// reciprocal division, exact for x < 2^63; freq == 1 uses rcp = 2^64 - 1,
// shift 0, bias = start + M - 1). The single-stack coder divides by
// Granlund-Montgomery (PLDI 1994, fig. 4.1, N = 64): with l = ceil(log2 freq)
// and m' = floor(2^64 (2^l - freq) / freq) + 1, t = mulhi(m', x) and
// x / freq = (t + ((x - t) >> min(l, 1))) >> max(l - 1, 0) for every 64-bit x.
__global__ void k_build_enc(const uint32_t* __restrict__ cdf, int alphabet,
                            EncSym* __restrict__ enc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= alphabet) return;
    const uint32_t start = cdf[s], freq = cdf[s + 1] - cdf[s];
    EncSym e;
    e.freq = freq;
    e.cmpl = (1u << PREC) - freq;
    e.pad = 0;
    uint32_t l = 0;
    while (freq > (1u << l)) l++;
    if (freq < 2) {
        e.rcp = ~0ull;
        e.shift = 0;
        e.bias = start + (1u << PREC) - 1u;
    } else {
        const unsigned __int128 num = ((unsigned __int128)1 << (l + 63)) + (freq - 1);
        e.rcp = (uint64_t)(num / freq);
        e.shift = (uint8_t)(l - 1);
        e.bias = start;
    }
    const unsigned __int128 gnum = (unsigned __int128)((1ull << l) - (freq ? freq : 1)) << 64;
    e.gm = (uint64_t)(gnum / (freq ? freq : 1)) + 1ull;
    e.gsh1 = (uint8_t)(l < 1 ? l : 1);
    e.gsh2 = (uint8_t)(l > 1 ? l - 1 : 0);
    enc[s] = e;
}

// Decoder bucket table: bucket[b] = symbol whose interval holds slot b << 12.
__global__ void k_build_bucket(const uint32_t* __restrict__ cdf, int alphabet,
                               uint16_t* __restrict__ bucket) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= NBUCKET) return;
    const uint32_t slot = (uint32_t)b << (PREC - BUCKET_BITS);
    int lo = 0, hi = alphabet;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (cdf[mid] <= slot) lo = mid; else hi = mid;
    }
    bucket[b] = (uint16_t)lo;
}

__device__ __forceinline__ int find_stage(const RansStageDesc* st, int n_stages, uint32_t chunk) {
    int lo = 0, hi = n_stages;  // last stage with chunk0 <= chunk
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (st[mid].chunk0 <= chunk) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t narrow(uint32_t code, int radius, int kexp) {
    return code ? (uint32_t)((int)code - radius + (1 << kexp)) : 0u;
}
__device__ __forceinline__ uint32_t widen(uint32_t sym, int radius, int kexp) {
    return sym ? (uint32_t)((int)sym - (1 << kexp) + radius) : 0u;
}

// --------------------------------------------------------------- lanes
// Steps an encoder warp runs per batch. A step's code, level row and table
// entry do not depend on the coder state, so a batch loads all of them before
// its serial state updates, and the next batch's codes are in flight
// meanwhile: one memory latency per batch instead of one per step (a lane's
// chain of K steps is the kernel's critical path).
constexpr int ENC_U = 8;

__global__ void __launch_bounds__(128)
    k_lanes_encode(const RansStageDesc* __restrict__ st, int n_stages, uint32_t total_chunks,
                   const uint16_t* __restrict__ codes, const uint8_t* __restrict__ levels,
                   uint32_t* __restrict__ scratch, uint32_t* __restrict__ chunk_words,
                   uint32_t* __restrict__ err) {
    const uint32_t chunk = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (chunk >= total_chunks) return;
    const int lane = threadIdx.x & 31;
    const RansStageDesc& d = st[find_stage(st, n_stages, chunk)];
    const uint32_t K = d.K;
    const uint64_t base = (uint64_t)(chunk - d.chunk0) * 32u * K;
    const EncSym* enc = (const EncSym*)d.enc;
    const uint32_t alpha1 = d.alphabet + 1;
    uint32_t* region = scratch + d.scratch_off + (uint64_t)(chunk - d.chunk0) * (64u + 32u * K);
    uint32_t* refill_end = region + 64 + 32u * K;
    const uint16_t* c = codes + d.codes_off;
    const uint8_t* lv = d.per_point ? levels + d.codes_off : nullptr;
    uint64_t x = LANE_L;
    uint32_t tail = 0;
    const unsigned lt = (1u << lane) - 1u;
    // steps k0, k0 - 1, ..., k0 - ENC_U + 1 of this lane (the encode order)
    uint16_t nc[ENC_U];
    uint8_t nr[ENC_U];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int u = 0; u < ENC_U; u++) {
            const int kk = k0 - u;
            const uint64_t i = base + (uint64_t)(kk < 0 ? 0 : kk) * 32u + lane;
            const bool ok = kk >= 0 && i < d.n;
            nc[u] = ok ? c[i] : (uint16_t)0;
            nr[u] = (ok && lv) ? lv[i] : (uint8_t)0;
        }
    };
    fetch((int)K - 1);
    for (int k = (int)K - 1; k >= 0; k -= ENC_U) {  // k is uniform across the warp
        uint16_t cc[ENC_U];
        uint8_t rr[ENC_U];
#pragma unroll
        for (int u = 0; u < ENC_U; u++) {
            cc[u] = nc[u];
            rr[u] = nr[u];
        }
        if (k - ENC_U >= 0) fetch(k - ENC_U);
        EncSym e[ENC_U];
#pragma unroll
        for (int u = 0; u < ENC_U; u++) {
            const int kk = k - u;
            const uint64_t i = base + (uint64_t)(kk < 0 ? 0 : kk) * 32u + lane;
            e[u] = EncSym{};
            if (kk >= 0 && i < d.n) {
                const uint32_t sym = narrow(cc[u], d.radius, d.kexp);
                if (sym >= d.alphabet) {
                    atomicOr(err, 2u);
                    e[u] = enc[rr[u] * alpha1];
                } else {
                    e[u] = enc[rr[u] * alpha1 + sym];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < ENC_U; u++) {
            const int kk = k - u;
            if (kk < 0) break;
            const bool valid = base + (uint64_t)kk * 32u + lane < d.n;
            const bool flush = valid && x >= ((uint64_t)e[u].freq << 39);
            const unsigned bal = __ballot_sync(0xffffffffu, flush);
            const uint32_t ne = __popc(bal);
            if (flush) {
                refill_end[-(int64_t)tail - (int64_t)ne + __popc(bal & lt)] = (uint32_t)x;
                x >>= 32;
            }
            tail += ne;
            if (valid) {
                const uint64_t q = __umul64hi(x, e[u].rcp) >> e[u].shift;
                x = x + e[u].bias + q * e[u].cmpl;
            }
        }
    }
    const bool active = base + lane < d.n;
    const unsigned abal = __ballot_sync(0xffffffffu, active);
    if (active) {
        const uint32_t p = 2u * __popc(abal & lt);
        region[p] = (uint32_t)(x >> 32);
        region[p + 1] = (uint32_t)x;
    }
    if (lane == 0) chunk_words[chunk] = 2u * __popc(abal) + tail;
}

// Symbol whose CDF interval holds `slot`: the bucket of the slot's top bits
// brackets it between bucket[b] and bucket[b + 1]; a binary search finishes.
__device__ __forceinline__ uint32_t lookup_sym(const uint32_t* cdf, const uint16_t* bucket,
                                               uint32_t slot, uint32_t alphabet) {
    const uint32_t b = slot >> (PREC - BUCKET_BITS);
    uint32_t lo = bucket[b];
    uint32_t hi = (b + 1 < (uint32_t)NBUCKET) ? bucket[b + 1] : alphabet - 1;
    while (lo < hi) {  // largest s in [lo, hi] with cdf[s] <= slot
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (cdf[mid] <= slot) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_block_stage(const RansStageDesc* st, int n_stages,
                                                uint32_t block) {
    int lo = 0, hi = n_stages;  // last stage with block0 <= block
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (st[mid].block0 <= block) lo = mid; else hi = mid;
    }
    return lo;
}

// One CTA per DEC_WARPS chunks of a single stage; stage-constant tables are
// staged in shared memory.
__global__ void __launch_bounds__(32 * DEC_WARPS)
    k_lanes_decode(const RansStageDesc* __restrict__ st, int n_stages, const uint32_t smem_alpha,
                   const uint32_t* __restrict__ words, const uint64_t* __restrict__ chunk_range,
                   const uint8_t* __restrict__ levels, uint16_t* __restrict__ codes,
                   uint32_t* __restrict__ err) {
    extern __shared__ uint32_t smem[];
    __shared__ uint32_t ring_all[DEC_WARPS][RING];
    const RansStageDesc& d = st[find_block_stage(st, n_stages, blockIdx.x)];
    const uint32_t local = (blockIdx.x - d.block0) * DEC_WARPS + (threadIdx.x >> 5);
    uint32_t* ring = ring_all[threadIdx.x >> 5];
    // smem_alpha: the largest alphabet the dynamic shared memory was sized for
    const bool smem_tables = !d.per_point && d.alphabet <= smem_alpha;
    const uint32_t alpha1 = d.alphabet + 1;
    const uint32_t* cdfs = (const uint32_t*)d.cdf;
    const uint16_t* buckets = (const uint16_t*)d.bucket;
    if (smem_tables) {
        uint32_t* sc = smem;
        uint16_t* sb = (uint16_t*)(smem + alpha1);
        for (uint32_t i = threadIdx.x; i < alpha1; i += blockDim.x) sc[i] = cdfs[i];
        for (uint32_t i = threadIdx.x; i < (uint32_t)NBUCKET; i += blockDim.x) sb[i] = buckets[i];
        __syncthreads();
        cdfs = sc;
        buckets = sb;
    }
    if (local >= d.n_chunks) return;
    const uint32_t chunk = d.chunk0 + local;
    const int lane = threadIdx.x & 31;
    const uint32_t K = d.K;
    const uint64_t base = (uint64_t)local * 32u * K;
    const uint8_t* lv = d.per_point ? levels + d.codes_off : nullptr;
    uint16_t* out = codes + d.codes_off;
    uint64_t pos = chunk_range[2 * (uint64_t)chunk];
    const uint64_t end = chunk_range[2 * (uint64_t)chunk + 1];
    const unsigned lt = (1u << lane) - 1u;
    const bool active = base + lane < d.n;
    const unsigned abal = __ballot_sync(0xffffffffu, active);
    uint64_t x = 0;
    if (active) {
        const uint64_t p = pos + 2u * __popc(abal & lt);
        if (p + 2 <= end) x = ((uint64_t)words[p] << 32) | words[p + 1];
        else atomicOr(err, 4u);
    }
    pos += 2u * __popc(abal);
    // refill words are consumed in order: keep [pos, hi) in a per-warp ring,
    // topped up RING/2 words at a time with coalesced loads
    uint64_t hi = pos;
    for (uint32_t k = 0; k < K; k++) {
        if (hi < pos + 32 && hi < end) {  // uniform across the warp
            const uint64_t top = hi + RING / 2 < end ? hi + RING / 2 : end;
            for (uint64_t w = hi + lane; w < top; w += 32) ring[w & (RING - 1)] = words[w];
            hi = top;
            __syncwarp();
        }
        const uint64_t i = base + (uint64_t)k * 32u + lane;
        const bool valid = i < d.n;
        bool need = false;
        if (valid) {
            const uint32_t row = lv ? lv[i] : 0u;
            const uint32_t* cdf = cdfs + (uint64_t)row * alpha1;
            const uint32_t slot = (uint32_t)(x & PMASK);
            const uint32_t s = lookup_sym(cdf, buckets + (uint64_t)row * NBUCKET, slot, d.alphabet);
            const uint32_t left = cdf[s], f = cdf[s + 1] - left;
            x = (uint64_t)f * (x >> PREC) + (slot - left);
            out[i] = (uint16_t)widen(s, d.radius, d.kexp);
            need = x < LANE_L;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, need);
        if (need) {
            const uint64_t p = pos + __popc(bal & lt);
            if (p < hi) x = (x << 32) | ring[p & (RING - 1)];
            else atomicOr(err, 4u);
        }
        pos += __popc(bal);
        __syncwarp();
    }
    if ((active && x != LANE_L) || (lane == 0 && pos != end)) atomicOr(err, 8u);
}

// --------------------------------------------------------------- compat
// The single-stack coder: one serial state chain per stage, every stage on
// its own CTA.
//   Encode (reverse symbol order): a CTA of 256 threads per stage. Thread 0
//   carries the chain; warps 1-7 turn the next block of SB codes (and scale
//   levels) into 16-byte records {gm, left, freq | gsh2 << 25 | gsh1 << 30}
//   in shared memory while thread 0 codes the current block (two buffers, one
//   __syncthreads per block), so the chain never waits on a global load.
constexpr int SB = 1024;
constexpr int ST_THREADS = 256;
constexpr int SG = 8;  // decoder: scale levels loaded this many symbols ahead

__global__ void __launch_bounds__(ST_THREADS)
    k_stack_encode(const RansStageDesc* __restrict__ st, int n_stages,
                   const uint16_t* __restrict__ codes, const uint8_t* __restrict__ levels,
                   uint32_t* __restrict__ scratch, uint32_t* __restrict__ stage_words,
                   uint32_t* __restrict__ err) {
    const int t = blockIdx.x;
    if (t >= n_stages) return;
    const RansStageDesc& d = st[t];
    if (d.mode != MODE_COMPAT) return;
    __shared__ uint4 ring[2][SB];
    __shared__ int s_bad;
    const int tid = threadIdx.x;
    const EncSym* enc = (const EncSym*)d.enc;
    const uint32_t alpha1 = d.alphabet + 1;
    const uint16_t* c = codes + d.codes_off;
    const uint8_t* lv = d.per_point ? levels + d.codes_off : nullptr;
    uint32_t* out = scratch + d.scratch_off;
    const int64_t n = d.n;
    const int64_t nb = (n + SB - 1) / SB;
    if (tid == 0) s_bad = 0;
    __syncthreads();
    // block b: slot j holds symbol n - 1 - b SB - j
    auto fill = [&](int64_t b, int buf, int t0, int nt) {
        const int64_t top = n - 1 - b * SB;
        for (int j = t0; j < SB; j += nt) {
            const int64_t i = top - j;
            uint4 r = make_uint4(0u, 0u, 0u, 0u);
            if (i >= 0) {
                const uint32_t sym = narrow(c[i], d.radius, d.kexp);
                const uint32_t row = lv ? lv[i] : 0u;
                if (sym >= d.alphabet) s_bad = 1;
                const EncSym e = enc[(uint64_t)row * alpha1 + (sym < d.alphabet ? sym : 0u)];
                const uint32_t left = e.freq == 1u ? e.bias - ((1u << PREC) - 1u) : e.bias;
                r = make_uint4((uint32_t)e.gm, (uint32_t)(e.gm >> 32), left,
                               e.freq | ((uint32_t)e.gsh2 << 25) | ((uint32_t)e.gsh1 << 30));
            }
            ring[buf][j] = r;
        }
    };
    if (nb > 0) fill(0, 0, tid, ST_THREADS);
    __syncthreads();
    uint64_t x = 0, w = 0;
    for (int64_t b = 0; b < nb; b++) {
        if (tid >= 32) {
            if (b + 1 < nb) fill(b + 1, (int)((b + 1) & 1), tid - 32, ST_THREADS - 32);
        } else if (tid == 0) {
            const int cnt = (int)(n - b * SB < SB ? n - b * SB : SB);
            const uint4* rb = ring[b & 1];
            uint4 nx = rb[0];
            for (int j = 0; j < cnt; j++) {
                const uint4 r = nx;
                if (j + 1 < cnt) nx = rb[j + 1];
                const uint64_t gm = ((uint64_t)r.y << 32) | r.x;
                const uint32_t p = r.w & 0x1FFFFFFu;
                const uint32_t g2 = (r.w >> 25) & 31u, g1 = r.w >> 30;
                if ((x >> (64 - PREC)) >= p) {
                    out[w++] = (uint32_t)x;
                    x >>= 32;
                }
                const uint64_t t1 = __umul64hi(x, gm);
                const uint64_t q = (t1 + ((x - t1) >> g1)) >> g2;
                x = (q << PREC) | (uint64_t)((uint32_t)(x - q * p) + r.z);
            }
        }
        __syncthreads();
    }
    if (tid != 0) return;
    if (s_bad) {
        atomicOr(err, 2u);
        return;
    }
    if (x >> 32) {
        out[w++] = (uint32_t)x;
        out[w++] = (uint32_t)(x >> 32);
    } else if (x) {
        out[w++] = (uint32_t)x;
    }
    stage_words[t] = (uint32_t)w;
}

// One thread per stage (lane 0 of the stage's own CTA). The next blob word
// and the scale levels are loaded ahead of their use; the state chain is the
// bucket and CDF lookups of the slot.
__global__ void k_stack_decode(const RansStageDesc* __restrict__ st, int n_stages,
                               const uint32_t* __restrict__ words, const uint8_t* __restrict__ levels,
                               uint16_t* __restrict__ codes, uint32_t* __restrict__ err) {
    const int t = blockIdx.x;
    if (t >= n_stages || threadIdx.x != 0) return;
    const RansStageDesc& d = st[t];
    if (d.mode != MODE_COMPAT || d.n == 0) return;
    const uint32_t* cdfs = (const uint32_t*)d.cdf;
    const uint16_t* buckets = (const uint16_t*)d.bucket;
    const uint32_t alpha1 = d.alphabet + 1;
    const uint32_t* wd = words + d.blob_off;
    int64_t top = d.blob_words;
    if (top > 0 && wd[top - 1] == 0) {
        atomicOr(err, 16u);
        return;
    }
    uint64_t x = 0;
    for (int k = 0; k < 2 && top > 0; k++) {
        x = (x << 32) | wd[--top];
        if (x >> 32) break;
    }
    uint32_t nw = top > 0 ? wd[top - 1] : 0u;  // the next word, loaded ahead
    const uint8_t* lv = d.per_point ? levels + d.codes_off : nullptr;
    uint16_t* out = codes + d.codes_off;
    const uint64_t n = d.n;
    uint8_t rows[SG];
#pragma unroll
    for (int u = 0; u < SG; u++) rows[u] = (lv && (uint64_t)u < n) ? lv[u] : (uint8_t)0;
    for (uint64_t i0 = 0; i0 < n; i0 += SG) {
        uint8_t cur[SG];
#pragma unroll
        for (int u = 0; u < SG; u++) {
            cur[u] = rows[u];
            rows[u] = (lv && i0 + SG + u < n) ? lv[i0 + SG + u] : (uint8_t)0;
        }
#pragma unroll
        for (int u = 0; u < SG; u++) {
            const uint64_t i = i0 + u;
            if (i >= n) break;
            const uint32_t row = cur[u];
            const uint32_t* cdf = cdfs + (uint64_t)row * alpha1;
            const uint32_t q = (uint32_t)(x & PMASK);
            const uint32_t s = lookup_sym(cdf, buckets + (uint64_t)row * NBUCKET, q, d.alphabet);
            const uint32_t left = cdf[s], p = cdf[s + 1] - left;
            x = (x >> PREC) * p + (q - left);
            if (x < (1ull << 32) && top > 0) {
                x = (x << 32) | nw;
                --top;
                nw = top > 0 ? wd[top - 1] : 0u;
            }
            out[i] = (uint16_t)widen(s, d.radius, d.kexp);
        }
    }
    if (top != 0 || x != 0) atomicOr(err, 16u);
}

// --------------------------------------------------------------- assembly
// Per stage: blob length in words and each chunk's offset inside the blob.
__global__ void __launch_bounds__(256)
    k_stage_sums(RansStageDesc* __restrict__ st, const uint32_t* __restrict__ chunk_words,
                 const uint32_t* __restrict__ stage_words, uint32_t* __restrict__ chunk_off) {
    RansStageDesc& d = st[blockIdx.x];
    __shared__ uint64_t sh[256];
    if (d.mode == MODE_COMPAT) {
        if (threadIdx.x == 0) d.blob_words = stage_words[blockIdx.x];
        return;
    }
    if (d.n == 0) {
        if (threadIdx.x == 0) d.blob_words = 0;
        return;
    }
    const uint32_t nc = d.n_chunks;
    const uint32_t per = (nc + 255) / 256;
    const uint32_t a = threadIdx.x * per, b = min(nc, a + per);
    uint64_t s = 0;
    for (uint32_t i = a; i < b; i++) s += chunk_words[d.chunk0 + i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        uint64_t v = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += v;
        __syncthreads();
    }
    uint64_t run = sh[threadIdx.x] - s + 1 + nc;  // after K and the chunk table
    for (uint32_t i = a; i < b; i++) {
        chunk_off[d.chunk0 + i] = (uint32_t)run;
        run += chunk_words[d.chunk0 + i];
    }
    if (threadIdx.x == 255) d.blob_words = (uint32_t)(1 + nc + sh[255]);
}

// Stage record offsets (bytes) in the payload; one thread, fixed order.
__global__ void k_record_layout(RansStageDesc* __restrict__ st, int n_stages,
                                const StageAcc* __restrict__ acc, int elem,
                                uint64_t* __restrict__ total, uint64_t cap, uint32_t* __restrict__ err) {
    if (threadIdx.x) return;
    uint64_t off = 0;
    for (int t = 0; t < n_stages; t++) {
        RansStageDesc& d = st[t];
        d.rec_off = off;
        d.n_out = acc[t].n_out;
        off += 16 + 4ull * d.blob_words + (uint64_t)elem * d.n_out;
    }
    *total = off;
    if (off > cap) atomicOr(err, 32u);
}

__global__ void __launch_bounds__(128)
    k_copy_chunks(const RansStageDesc* __restrict__ st, int n_stages, uint32_t total_chunks,
                  const uint32_t* __restrict__ scratch, const uint32_t* __restrict__ chunk_words,
                  const uint32_t* __restrict__ chunk_off, uint8_t* __restrict__ payload,
                  uint64_t cap) {
    const uint32_t chunk = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (chunk >= total_chunks) return;
    const int lane = threadIdx.x & 31;
    const RansStageDesc& d = st[find_stage(st, n_stages, chunk)];
    const uint32_t K = d.K;
    const uint32_t* region = scratch + d.scratch_off + (uint64_t)(chunk - d.chunk0) * (64u + 32u * K);
    const uint64_t base_active = (uint64_t)(chunk - d.chunk0) * 32u * K;
    const uint64_t left = (uint64_t)d.n - base_active;
    const uint32_t n_active = left < 32 ? (uint32_t)left : 32u;
    const uint32_t nw = chunk_words[chunk];
    const uint32_t ns = 2 * n_active, nr = nw - ns;
    const uint64_t dst = d.rec_off + 12 + 4ull * chunk_off[chunk];
    if (dst + 4ull * nw > cap) return;
    uint32_t* out = (uint32_t*)(payload + dst);  // 4-byte aligned: records are multiples of 4
    for (uint32_t w = lane; w < ns; w += 32) out[w] = region[w];
    const uint32_t* rf = region + 64 + 32u * K - nr;
    for (uint32_t w = lane; w < nr; w += 32) out[ns + w] = rf[w];
}

__global__ void __launch_bounds__(256)
    k_write_records(const RansStageDesc* __restrict__ st, const uint32_t* __restrict__ chunk_words,
                    const uint32_t* __restrict__ stack_scratch, const uint8_t* __restrict__ outliers,
                    int elem, uint8_t* __restrict__ payload, uint64_t cap) {
    const RansStageDesc& d = st[blockIdx.x];
    const uint64_t r = d.rec_off;
    const uint64_t len = 16 + 4ull * d.blob_words + (uint64_t)elem * d.n_out;
    if (r + len > cap) return;
    uint32_t* w32 = (uint32_t*)(payload + r);
    if (threadIdx.x == 0) {
        const uint64_t framed = (4ull * d.blob_words) | d.framed_hi;
        w32[0] = d.n;
        w32[1] = (uint32_t)framed;
        w32[2] = (uint32_t)(framed >> 32);
        if (d.mode == MODE_LANES && d.n) w32[3] = d.K;
        w32[3 + d.blob_words] = d.n_out;
    }
    if (d.mode == MODE_LANES) {
        for (uint32_t i = threadIdx.x; i < d.n_chunks && d.n; i += blockDim.x)
            w32[4 + i] = chunk_words[d.chunk0 + i];
    } else {
        const uint32_t* src = stack_scratch + d.scratch_off;
        for (uint32_t i = threadIdx.x; i < d.blob_words; i += blockDim.x) w32[3 + i] = src[i];
    }
    const uint8_t* src = outliers + (uint64_t)d.out_off * elem;
    uint8_t* dst = payload + r + 16 + 4ull * d.blob_words;
    const uint64_t nb = (uint64_t)elem * d.n_out;
    for (uint64_t b = threadIdx.x; b < nb; b += blockDim.x) dst[b] = src[b];
}

// --------------------------------------------------------------- launchers
static int last_err() {
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

int launch_build_tables(const uint32_t* cdf, int alphabet, int rows, EncSym* enc, uint16_t* bucket,
                        cudaStream_t st) {
    for (int r = 0; r < rows; r++) {
        const uint32_t* c = cdf + (size_t)r * (alphabet + 1);
        if (enc) k_build_enc<<<(alphabet + 255) / 256, 256, 0, st>>>(c, alphabet, enc + (size_t)r * (alphabet + 1));
        if (bucket) k_build_bucket<<<NBUCKET / 256, 256, 0, st>>>(c, alphabet, bucket + (size_t)r * NBUCKET);
    }
    count_launches((unsigned)rows * ((enc ? 1 : 0) + (bucket ? 1 : 0)) - 1);
    return last_err();
}

int launch_lanes_encode(const RansStageDesc* st, int n_stages, uint32_t total_chunks,
                        const uint16_t* codes, const uint8_t* levels, uint32_t* scratch,
                        uint32_t* chunk_words, uint32_t* err, cudaStream_t s) {
    if (!total_chunks) return LATEC_OK;
    k_lanes_encode<<<(total_chunks + 3) / 4, 128, 0, s>>>(st, n_stages, total_chunks, codes, levels,
                                                          scratch, chunk_words, err);
    return last_err();
}

int launch_lanes_decode(const RansStageDesc* st, int n_stages, uint32_t total_blocks,
                        int max_alphabet, const uint32_t* words, const uint64_t* chunk_range,
                        const uint8_t* levels, uint16_t* codes, uint32_t* err, cudaStream_t s) {
    if (!total_blocks) return LATEC_OK;
    const int a = max_alphabet <= SMEM_ALPHA ? max_alphabet : 0;
    const size_t smem = a ? (size_t)(a + 1) * 4 + NBUCKET * 2 : 0;
    // the static word rings plus the dynamic tables may pass the 48 KB default
    if (smem + sizeof(uint32_t) * DEC_WARPS * RING > 48 * 1024 &&
        cudaFuncSetAttribute(k_lanes_decode, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return LATEC_ERR_CUDA;
    k_lanes_decode<<<total_blocks, 32 * DEC_WARPS, smem, s>>>(st, n_stages, (uint32_t)a, words,
                                                               chunk_range, levels, codes, err);
    return last_err();
}

int launch_stack_encode(const RansStageDesc* st, int n_stages, const uint16_t* codes,
                        const uint8_t* levels, uint32_t* scratch, uint32_t* stage_words,
                        uint32_t* err, cudaStream_t s) {
    if (!n_stages) return LATEC_OK;
    k_stack_encode<<<n_stages, ST_THREADS, 0, s>>>(st, n_stages, codes, levels, scratch,
                                                   stage_words, err);
    return last_err();
}

int launch_stack_decode(const RansStageDesc* st, int n_stages, const uint32_t* words,
                        const uint8_t* levels, uint16_t* codes, uint32_t* err, cudaStream_t s) {
    if (!n_stages) return LATEC_OK;
    k_stack_decode<<<n_stages, 32, 0, s>>>(st, n_stages, words, levels, codes, err);
    return last_err();
}

int launch_assemble(RansStageDesc* st, int n_stages, uint32_t total_chunks,
                    const uint32_t* lane_scratch, const uint32_t* chunk_words, uint32_t* chunk_off,
                    const uint32_t* stack_scratch, const uint32_t* stage_words,
                    const StageAcc* acc, const uint8_t* outliers, int elem, uint8_t* payload,
                    uint64_t cap, uint64_t* total, uint32_t* err, cudaStream_t s) {
    if (!n_stages) return LATEC_OK;
    k_stage_sums<<<n_stages, 256, 0, s>>>(st, chunk_words, stage_words, chunk_off);
    k_record_layout<<<1, 32, 0, s>>>(st, n_stages, acc, elem, total, cap, err);
    if (total_chunks)
        k_copy_chunks<<<(total_chunks + 3) / 4, 128, 0, s>>>(st, n_stages, total_chunks,
                                                             lane_scratch, chunk_words, chunk_off,
                                                             payload, cap);
    k_write_records<<<n_stages, 256, 0, s>>>(st, chunk_words, stack_scratch, outliers, elem,
                                            payload, cap);
    count_launches(total_chunks ? 3 : 2);
    return last_err();
}

}  // namespace latec
