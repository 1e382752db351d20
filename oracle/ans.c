/* CPU oracle for the rANS entropy stage -- TEST INFRASTRUCTURE ONLY.
 *
 * Two coders over the same 24-bit Laplace-mixture tables (reference
 * latec/rans.py:304-329, 466-616):
 *
 * 1. The compatibility coder: a single-stack ANS restated from the published
 *    algorithm of the `constriction` 0.4 crate's `stream::stack::AnsCoder`
 *    (u32 words, u64 state, 24-bit precision), which the reference calls at
 *    latec/rans.py:476-498 and 512-535 but which is not installed here:
 *      - state starts at 0;
 *      - encode(left, p): if (x >> 40) >= p, push low 32 bits and x >>= 32;
 *        then x = (x / p) << 24 | (x % p + left);
 *      - symbols are encoded last-first (encode_reverse), so they decode in
 *        order;
 *      - get_compressed appends the state's significant words, least
 *        significant first (0, 1 or 2 words);
 *      - decode: quantile = x & (2^24-1); x = (x >> 24) * p + quantile - left;
 *        if x < 2^32 and words remain, x = x << 32 | pop();
 *      - the stream is fully consumed iff no words remain and x == 0.
 *    The model is constriction's `Categorical(probs, perfect=False)`, i.e. the
 *    "fast" float32 quantisation of the reference's own integer PMF (see
 *    oracle_fast_quantize). No reference test pins these bytes: parity of the
 *    compatibility stream is unpinned.
 *
 * 2. The native interleaved coder this project defines (its byte layout is
 *    specified here and the CUDA coder must match it bit for bit):
 *      stage blob = u32 K | u32 chunk_words[n_chunks] | chunk streams
 *      n_chunks = ceil(n / (32 K)); chunk c holds symbols [32Kc, 32K(c+1)),
 *      lane l of the chunk codes symbols 32Kc + 32k + l, k = 0..K-1.
 *      Each lane is a 64-bit rANS state in [2^31, 2^63), initial 2^31,
 *      24-bit precision, 32-bit renormalisation words (the range keeps every
 *      state below 2^63, where a 64-bit reciprocal division is exact):
 *        encode (reverse k order): if x >= p << 39 emit low word, x >>= 32;
 *                                  x = (x / p) << 24 | (x % p + left)
 *        decode (forward k order): s = x & (2^24-1) -> symbol;
 *                                  x = p * (x >> 24) + s - left;
 *                                  if x < 2^31: x = x << 32 | next word
 *      Chunk stream, in decoder read order: for every active lane ascending,
 *      the final encoder state as (high word, low word); then the refill words
 *      by decode step k ascending, lanes ascending within a step.
 *    A lane is active iff it holds at least one symbol.
 *
 * Symbols are "narrowed" symbols (0 = outlier marker, q + 2^kexp otherwise),
 * tables are CDF rows of length alphabet + 1 with cdf[0] = 0 and
 * cdf[alphabet] = 2^24. All functions return >= 0 on success, < 0 on error.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PREC 24
#define PMASK ((1u << PREC) - 1u)

/* ---- symbol lookup for the decoders: largest s with cdf[s] <= q ---- */
static int find_sym(const uint32_t* cdf, int alphabet, uint32_t q) {
    int lo = 0, hi = alphabet; /* cdf[lo] <= q < cdf[hi] */
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (cdf[mid] <= q) lo = mid; else hi = mid;
    }
    return lo;
}

/* constriction's fast float32 quantisation of a probability vector to a
 * 24-bit CDF: each symbol keeps one count of slack and the remaining
 * 2^24 - n counts follow the float32 running sum scaled by (2^24 - n) / sum.
 * out_cdf has n + 1 entries. */
int oracle_fast_quantize(const float* probs, int n, uint32_t* out_cdf) {
    if (n < 2 || n >= (1 << PREC)) return -1;
    float norm = 0.0f;
    for (int i = 0; i < n; i++) norm += probs[i];
    if (!(norm > 0.0f)) return -2;
    float scale = (float)((1u << PREC) - (uint32_t)n) / norm;
    float cum = 0.0f;
    for (int i = 0; i < n; i++) {
        float v = cum * scale;
        out_cdf[i] = (uint32_t)v + (uint32_t)i;
        cum += probs[i];
    }
    out_cdf[n] = 1u << PREC;
    for (int i = 0; i < n; i++)
        if (out_cdf[i + 1] <= out_cdf[i]) return -3;
    return 0;
}

/* ---------------------------------------------------------------- stack */

/* Encode syms (length n, each < alphabet) with per-symbol table rows:
 * row(i) = cdfs + level[i] * (alphabet + 1) (level may be NULL -> row 0).
 * Encoding order is i = n-1 .. 0 (constriction encode_reverse over the whole
 * stage). Returns the number of u32 words written to out (<= cap). */
long oracle_stack_encode(const int32_t* syms, const uint8_t* levels, long n,
                         const uint32_t* cdfs, int alphabet, uint32_t* out, long cap) {
    uint64_t x = 0;
    long w = 0;
    for (long i = n - 1; i >= 0; i--) {
        int s = syms[i];
        if (s < 0 || s >= alphabet) return -1;
        const uint32_t* cdf = cdfs + (size_t)(levels ? levels[i] : 0) * (alphabet + 1);
        uint32_t left = cdf[s], p = cdf[s + 1] - cdf[s];
        if (p == 0) return -2;
        if ((x >> (64 - PREC)) >= p) {
            if (w >= cap) return -3;
            out[w++] = (uint32_t)x;
            x >>= 32;
        }
        x = ((x / p) << PREC) | (uint64_t)((uint32_t)(x % p) + left);
    }
    if (x >> 32) {
        if (w + 2 > cap) return -3;
        out[w++] = (uint32_t)x;
        out[w++] = (uint32_t)(x >> 32);
    } else if (x) {
        if (w + 1 > cap) return -3;
        out[w++] = (uint32_t)x;
    }
    return w;
}

/* Inverse of oracle_stack_encode. Returns 0, or < 0 for a malformed stream
 * (-4: ends in a zero word, -5: trailing data). */
int oracle_stack_decode(const uint32_t* words, long n_words, const uint8_t* levels, long n,
                        const uint32_t* cdfs, int alphabet, int32_t* out) {
    long top = n_words;
    if (top > 0 && words[top - 1] == 0) return -4;
    uint64_t x = 0;
    for (int k = 0; k < 2 && top > 0; k++) {
        x = (x << 32) | words[--top];
        if (x >> 32) break;
    }
    for (long i = 0; i < n; i++) {
        const uint32_t* cdf = cdfs + (size_t)(levels ? levels[i] : 0) * (alphabet + 1);
        uint32_t q = (uint32_t)(x & PMASK);
        int s = find_sym(cdf, alphabet, q);
        uint32_t left = cdf[s], p = cdf[s + 1] - cdf[s];
        x = (x >> PREC) * p + (q - left);
        if (x < (1ull << 32) && top > 0) x = (x << 32) | words[--top];
        out[i] = s;
    }
    if (top != 0 || x != 0) return -5;
    return 0;
}

/* ---------------------------------------------------------------- lanes */

long oracle_lanes_encode(const int32_t* syms, const uint8_t* levels, long n, int K,
                         const uint32_t* cdfs, int alphabet, uint32_t* out, long cap) {
    if (K < 1) return -1;
    if (n == 0) return 0; /* an empty stage has an empty blob */
    long per = 32L * K;
    long n_chunks = (n + per - 1) / per;
    long head = 1 + n_chunks;
    if (cap < head) return -3;
    out[0] = (uint32_t)K;
    long w = head;
    uint32_t* scratch = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(per > 0 ? per : 1));
    if (!scratch) return -6;
    for (long c = 0; c < n_chunks; c++) {
        long base = c * per;
        uint64_t x[32];
        int active[32];
        for (int l = 0; l < 32; l++) {
            x[l] = 1ull << 31;
            active[l] = base + l < n;
        }
        long tail = 0; /* refill words, filled from the end of scratch */
        for (int k = K - 1; k >= 0; k--) {
            uint32_t emit[32];
            int ne = 0;
            for (int l = 0; l < 32; l++) {
                long i = base + 32L * k + l;
                if (i >= n) continue;
                int s = syms[i];
                if (s < 0 || s >= alphabet) { free(scratch); return -1; }
                const uint32_t* cdf = cdfs + (size_t)(levels ? levels[i] : 0) * (alphabet + 1);
                uint32_t left = cdf[s], p = cdf[s + 1] - cdf[s];
                if (p == 0) { free(scratch); return -2; }
                if (x[l] >= ((uint64_t)p << 39)) {
                    emit[ne++] = (uint32_t)x[l];
                    x[l] >>= 32;
                }
                x[l] = ((x[l] / p) << PREC) | (uint64_t)((uint32_t)(x[l] % p) + left);
            }
            /* decode order within a step is lanes ascending */
            for (int e = ne - 1; e >= 0; e--) scratch[per - 1 - tail - (ne - 1 - e)] = emit[e];
            tail += ne;
        }
        long start = w;
        for (int l = 0; l < 32; l++) {
            if (!active[l]) continue;
            if (w + 2 > cap) { free(scratch); return -3; }
            out[w++] = (uint32_t)(x[l] >> 32);
            out[w++] = (uint32_t)x[l];
        }
        if (w + tail > cap) { free(scratch); return -3; }
        memcpy(out + w, scratch + (per - tail), sizeof(uint32_t) * (size_t)tail);
        w += tail;
        out[1 + c] = (uint32_t)(w - start);
    }
    free(scratch);
    return w;
}

int oracle_lanes_decode(const uint32_t* words, long n_words, const uint8_t* levels, long n,
                        const uint32_t* cdfs, int alphabet, int32_t* out) {
    if (n == 0) return n_words == 0 ? 0 : -5;
    if (n_words < 1) return -5;
    long K = words[0];
    if (K < 1) return -5;
    long per = 32L * K;
    long n_chunks = (n + per - 1) / per;
    if (n_words < 1 + n_chunks) return -5;
    long pos = 1 + n_chunks;
    for (long c = 0; c < n_chunks; c++) {
        long base = c * per;
        long end = pos + words[1 + c];
        if (end > n_words) return -5;
        uint64_t x[32];
        for (int l = 0; l < 32; l++) {
            x[l] = 0;
            if (base + l < n) {
                if (pos + 2 > end) return -5;
                x[l] = ((uint64_t)words[pos] << 32) | words[pos + 1];
                pos += 2;
            }
        }
        for (long k = 0; k < K; k++) {
            for (int l = 0; l < 32; l++) {
                long i = base + 32L * k + l;
                if (i >= n) continue;
                const uint32_t* cdf = cdfs + (size_t)(levels ? levels[i] : 0) * (alphabet + 1);
                uint32_t q = (uint32_t)(x[l] & PMASK);
                int s = find_sym(cdf, alphabet, q);
                uint32_t left = cdf[s], p = cdf[s + 1] - cdf[s];
                x[l] = (uint64_t)p * (x[l] >> PREC) + (q - left);
                if (x[l] < (1ull << 31)) {
                    if (pos >= end) return -5;
                    x[l] = (x[l] << 32) | words[pos++];
                }
                out[i] = s;
            }
        }
        for (int l = 0; l < 32; l++)
            if (base + l < n && x[l] != (1ull << 31)) return -5;
        if (pos != end) return -5;
    }
    return pos == n_words ? 0 : -5;
}
