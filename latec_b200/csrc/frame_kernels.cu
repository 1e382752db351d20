// Container framing on the device: the LATEC header followed by a zstd frame
// of raw (stored) blocks around the stage payload, and the inverse. The frame
// layout is the zstd format's: magic 0xFD2FB528, descriptor 0xE0 (8-byte
// content size, single segment), then blocks of at most 128 KiB, each with a
// 3-byte little-endian header last | (type 0 << 1) | (size << 3).
#include <cuda_runtime.h>

#include "latec_common.cuh"

namespace latec {

constexpr uint64_t RAW_BLOCK = 1ull << 17;

__host__ __device__ inline uint64_t raw_blocks(uint64_t n) {
    return n ? (n + RAW_BLOCK - 1) / RAW_BLOCK : 1;
}

// One thread per output word-ish unit: every byte of the payload moves to
// 13 + 3 * (block + 1) + p past the header; headers are written by the
// thread that owns the block's first byte.
__global__ void k_frame_raw(const uint8_t* __restrict__ payload, uint64_t n,
                            const uint8_t* __restrict__ header, uint32_t hlen,
                            uint8_t* __restrict__ out) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nb = raw_blocks(n);
    if (tid < hlen) out[tid] = header[tid];
    uint8_t* f = out + hlen;
    if (tid < 13) {
        uint8_t h[13];
        const uint32_t magic = 0xFD2FB528u;
        for (int k = 0; k < 4; k++) h[k] = (uint8_t)(magic >> (8 * k));
        h[4] = 0xE0;
        for (int k = 0; k < 8; k++) h[5 + k] = (uint8_t)(n >> (8 * k));
        f[tid] = h[tid];
    }
    if (tid < nb) {
        const uint64_t size = (tid + 1 < nb) ? RAW_BLOCK : (n - tid * RAW_BLOCK);
        const uint32_t w = (uint32_t)((tid + 1 == nb ? 1u : 0u) | (size << 3));
        uint8_t* hb = f + 13 + tid * (RAW_BLOCK + 3);
        hb[0] = (uint8_t)w;
        hb[1] = (uint8_t)(w >> 8);
        hb[2] = (uint8_t)(w >> 16);
    }
    for (uint64_t p = tid; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = p / RAW_BLOCK;
        f[13 + 3 * (b + 1) + p] = payload[p];
    }
}

__global__ void k_unframe_raw(const uint8_t* __restrict__ frame, uint64_t n,
                              uint8_t* __restrict__ payload, uint32_t* __restrict__ err) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nb = raw_blocks(n);
    if (tid < nb) {  // every block header must be the one the writer emits
        const uint64_t size = (tid + 1 < nb) ? RAW_BLOCK : (n - tid * RAW_BLOCK);
        const uint32_t want = (uint32_t)((tid + 1 == nb ? 1u : 0u) | (size << 3));
        const uint8_t* hb = frame + 13 + tid * (RAW_BLOCK + 3);
        const uint32_t got = hb[0] | ((uint32_t)hb[1] << 8) | ((uint32_t)hb[2] << 16);
        if (got != want && err) atomicOr(err, 64u);
    }
    for (uint64_t p = tid; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = p / RAW_BLOCK;
        payload[p] = frame[13 + 3 * (b + 1) + p];
    }
}

// Parsed stage record (latec/bitstream.py:288-344 framing), one per stage.
struct Record {
    uint64_t blob;      // byte offset of the blob in the payload
    uint64_t out_at;    // byte offset of the outliers
    uint64_t frame;     // the 64-bit frame word
    uint32_t n;         // codes
    uint32_t n_out;
    uint32_t K;         // lane coder symbols per lane (0 otherwise)
    uint32_t n_chunks;
    uint32_t chunk0;
    uint32_t status;    // 0 ok, else the first failed check
};

__device__ __forceinline__ uint64_t rd(const uint8_t* p, int k) {
    uint64_t v = 0;
    for (int i = 0; i < k; i++) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

// One thread walks the records in order (their offsets depend on the previous
// lengths); bounds are checked before every read.
__global__ void k_parse_records(const uint8_t* __restrict__ pay, uint64_t n_bytes, int ns,
                                int elem, int lanes, Record* __restrict__ rec,
                                uint64_t* __restrict__ total_chunks) {
    if (threadIdx.x || blockIdx.x) return;
    uint64_t off = 0, chunks = 0;
    uint32_t bad = 0;
    for (int t = 0; t < ns; t++) {
        Record r = {};
        if (!bad) {
            if (off + 12 > n_bytes) bad = 1;
            else {
                r.n = (uint32_t)rd(pay + off, 4);
                r.frame = rd(pay + off + 4, 8);
                const uint64_t hlen = r.frame & ((1ull << 45) - 1);
                const bool literal = (r.frame >> 63) & 1;
                r.blob = off + 12;
                if (r.blob + hlen + 4 > n_bytes) bad = 2;
                else {
                    r.n_out = (uint32_t)rd(pay + r.blob + hlen, 4);
                    r.out_at = r.blob + hlen + 4;
                    const uint64_t end = r.out_at + (uint64_t)elem * r.n_out;
                    if (end > n_bytes) bad = 3;
                    else {
                        if (lanes && r.n && !literal) {
                            if (hlen < 4 || (r.blob & 3) || (hlen & 3)) bad = 4;
                            else {
                                r.K = (uint32_t)rd(pay + r.blob, 4);
                                if (!r.K) bad = 5;
                                else {
                                    const uint64_t nc = ((uint64_t)r.n + 32ull * r.K - 1) / (32ull * r.K);
                                    if (4 * (1 + nc) > hlen) bad = 6;
                                    r.n_chunks = (uint32_t)nc;
                                    r.chunk0 = (uint32_t)chunks;
                                    chunks += nc;
                                }
                            }
                        }
                        off = end;
                    }
                }
            }
        }
        r.status = bad;
        rec[t] = r;
    }
    if (!bad && off != n_bytes) rec[ns - 1].status = 7;  // trailing data
    *total_chunks = chunks;
}

// Per lane-coded stage: absolute word ranges of every chunk stream.
__global__ void __launch_bounds__(256)
    k_chunk_ranges(const uint32_t* __restrict__ words, const Record* __restrict__ rec,
                   uint64_t* __restrict__ ranges, uint32_t* __restrict__ err) {
    const Record& r = rec[blockIdx.x];
    if (!r.n_chunks || r.status) return;
    __shared__ uint64_t sh[256];
    const uint64_t w0 = r.blob / 4, nc = r.n_chunks;
    const uint64_t hw = (r.frame & ((1ull << 45) - 1)) / 4;
    const uint32_t* cw = words + w0 + 1;
    const uint64_t per = (nc + 255) / 256;
    const uint64_t a = threadIdx.x * per, b = a + per < nc ? a + per : nc;
    uint64_t s = 0;
    for (uint64_t i = a; i < b; i++) s += cw[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        const uint64_t v = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += v;
        __syncthreads();
    }
    uint64_t run = w0 + 1 + nc + sh[threadIdx.x] - s;
    for (uint64_t i = a; i < b; i++) {
        ranges[2 * (r.chunk0 + i)] = run;
        run += cw[i];
        ranges[2 * (r.chunk0 + i) + 1] = run;
    }
    if (threadIdx.x == 255 && w0 + 1 + nc + sh[255] != w0 + hw) atomicOr(err, 128u);
}

}  // namespace latec

using namespace latec;

extern "C" {

uint64_t latec_raw_frame_bytes(uint64_t payload_bytes) {
    return 13 + 3 * raw_blocks(payload_bytes) + payload_bytes;
}

int latec_frame_raw(const uint8_t* payload, uint64_t n, const uint8_t* header, uint32_t hlen,
                    uint8_t* out, uint64_t out_cap, void* stream) {
    if ((n && !payload) || (hlen && !header) || !out) return LATEC_ERR_ARG;
    if (out_cap < hlen + latec_raw_frame_bytes(n)) return LATEC_ERR_WORKSPACE;
    const uint64_t work = n > raw_blocks(n) + 13 + hlen ? n : raw_blocks(n) + 13 + hlen;
    uint64_t blocks = (work + 255) / 256;
    if (blocks > 148ull * 64) blocks = 148ull * 64;
    if (blocks < 1) blocks = 1;
    // the header and block-header writers need one thread each
    const uint64_t need = (raw_blocks(n) + 13 + hlen + 255) / 256;
    if (blocks < need) blocks = need;
    k_frame_raw<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(payload, n, header, hlen, out);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

int latec_unframe_raw(const uint8_t* frame, uint64_t n, uint8_t* payload, uint32_t* err,
                      void* stream) {
    if (!frame || (n && !payload)) return LATEC_ERR_ARG;
    uint64_t blocks = (n > raw_blocks(n) ? n : raw_blocks(n)) / 256 + 1;
    if (blocks > 148ull * 64 && 148ull * 64 * 256 >= raw_blocks(n)) blocks = 148ull * 64;
    k_unframe_raw<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(frame, n, payload, err);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

uint64_t latec_record_size(void) { return sizeof(Record); }

int latec_parse_records(const uint8_t* payload, uint64_t n_bytes, int32_t n_stages, int32_t elem,
                        int32_t lanes, void* records, uint64_t* total_chunks, void* stream) {
    if (!payload || n_stages < 1 || !records || !total_chunks || (elem != 4 && elem != 8))
        return LATEC_ERR_ARG;
    k_parse_records<<<1, 32, 0, (cudaStream_t)stream>>>(payload, n_bytes, n_stages, elem, lanes,
                                                        (Record*)records, total_chunks);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

int latec_chunk_ranges(const uint32_t* words, const void* records, int32_t n_stages,
                       uint64_t* ranges, uint32_t* err, void* stream) {
    if (!words || !records || n_stages < 1 || !err) return LATEC_ERR_ARG;
    k_chunk_ranges<<<n_stages, 256, 0, (cudaStream_t)stream>>>(words, (const Record*)records,
                                                               ranges, err);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // extern "C"
