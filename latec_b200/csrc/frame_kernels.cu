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
                              uint8_t* __restrict__ payload) {
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = p / RAW_BLOCK;
        payload[p] = frame[13 + 3 * (b + 1) + p];
    }
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

int latec_unframe_raw(const uint8_t* frame, uint64_t n, uint8_t* payload, void* stream) {
    if (!n) return LATEC_OK;
    if (!frame || !payload) return LATEC_ERR_ARG;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > 148ull * 64) blocks = 148ull * 64;
    k_unframe_raw<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(frame, n, payload);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // extern "C"
