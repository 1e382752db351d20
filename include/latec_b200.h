/* latec_b200.h -- C ABI of the B200 (sm_100a) LATEC hot path.
 *
 * The reference LATEC is a Python package whose hot path sits behind a
 * duck-typed plugin boundary: the codec driver calls
 * predictor.predict(recon, known, pos) and then quantize / pack_stage on the
 * result (reference latec/codec.py:384-510). This library replaces the work
 * behind that boundary with CUDA kernels; each entry point below names the
 * reference function(s) it replaces. Plain pointers and sizes only: device
 * pointers are raw CUDA device addresses, `stream` is a cudaStream_t (NULL =
 * legacy default stream). Every function returns LATEC_OK (0) or a negative
 * LATEC_ERR_* code; kernels that detect malformed input set bits in a
 * caller-provided device error word instead of faulting.
 */
#ifndef LATEC_B200_H
#define LATEC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LATEC_MAX_NDIM 6

#define LATEC_OK 0
#define LATEC_ERR_ARG (-1)         /* invalid argument (ValueError in the reference) */
#define LATEC_ERR_CUDA (-2)        /* CUDA launch / runtime failure */
#define LATEC_ERR_UNSUPPORTED (-3) /* valid in the reference, not supported here */
#define LATEC_ERR_STREAM (-4)      /* malformed stream */
#define LATEC_ERR_WORKSPACE (-5)   /* workspace too small */
#define LATEC_ERR_INTERNAL (-6)

#define LATEC_F32 1
#define LATEC_F64 2

#define LATEC_RANS_LANES 0  /* native 32-lane interleaved coder */
#define LATEC_RANS_COMPAT 1 /* single-stack coder, reference byte stream */

typedef struct latec_plan latec_plan;

/* Quantizer / predictor parameters shared by all stages of one pass. */
typedef struct latec_quant_params {
    int32_t dtype;        /* LATEC_F32 or LATEC_F64 (value/reconstruction type) */
    int32_t channels;     /* C of the (C, *spatial) field */
    int32_t radius;       /* quantizer radius, <= 32768 */
    int32_t order;        /* 0 linear, 1 cubic */
    int32_t center;       /* 0 average odd axes, 1 first odd axis, 2 last odd axis */
    int32_t end_mode;     /* bit 0 quadratic ends, bit 1 extrapolation */
    int32_t round_output; /* verify against the rounded reconstruction (integer sources):
                           * 0 no, 1 rint(recon), 2 the normalised value of the
                           * nearest raw integer, (rint(recon * round_span +
                           * round_offset) - round_offset) / round_span */
    int32_t reserved;
    double round_span;    /* round_output 2: the data range and its minimum */
    double round_offset;
} latec_quant_params;

/* Per-stage results written on the device. */
typedef struct latec_stage_stats {
    uint32_t n_out;    /* outliers of the stage */
    uint32_t maxq;     /* max |q| over in-range codes */
    uint32_t pad0, pad1;
    double stats[5];   /* pred SAE, pred SSE, recon SAE, recon SSE, recon max */
} latec_stage_stats;

/* One stage of the entropy stage (host array; copied to the device). */
typedef struct latec_rans_stage {
    uint64_t codes_off;   /* first code of the stage in the codes buffer */
    uint64_t out_off;     /* first outlier of the stage in the outlier buffer */
    uint64_t enc;         /* device address: encoder symbol table (32 B/entry) */
    uint64_t cdf;         /* device address: CDF rows (alphabet + 1 u32 each) */
    uint64_t bucket;      /* device address: decoder bucket rows (1024 u16 each) */
    uint64_t scratch_off; /* filled by the library */
    uint64_t blob_off;    /* decode: word offset of the stage blob */
    uint64_t rec_off;     /* filled by the library */
    uint64_t framed_hi;   /* stage frame word without its 45-bit length */
    uint32_t n;           /* symbols */
    uint32_t K;           /* lane coder: symbols per lane per chunk */
    uint32_t n_chunks;    /* filled by the library (encode) / given (decode) */
    uint32_t chunk0;      /* filled by the library */
    uint32_t alphabet;    /* 2^(kexp+1) */
    int32_t kexp;
    int32_t radius;
    int32_t mode;         /* LATEC_RANS_LANES or LATEC_RANS_COMPAT */
    int32_t per_point;    /* 1: per-symbol table row from the levels array */
    uint32_t blob_words;  /* decode: blob length in words */
    uint32_t n_out;
    uint32_t block0;      /* filled by the library (decode) */
} latec_rans_stage;

/* ---- schedule: replaces latec/levels.py:100-147 (iter_stage_plan),
 *      221-282 (stage_counts), 297-326 (stage_strides), 469-574
 *      (stage_layouts). anchor_block in [1, anchor_stride]: blocks of
 *      anchor_block consecutive lattice points per axis every anchor_stride
 *      points form the anchor stage (latec/levels.py:100-147). */
int latec_plan_create(const uint32_t* shape, int32_t ndim, int32_t levels,
                      int32_t anchor_stride, int32_t anchor_block, latec_plan** out);
int latec_plan_destroy(latec_plan* plan);
int latec_plan_num_stages(const latec_plan* plan);
int latec_plan_stage_info(const latec_plan* plan, int32_t stage, uint64_t* n_points,
                          int32_t* stride, int32_t* weight, int32_t* axis);

/* Host-side (no GPU) decode of stage ranks [first, first + count) into flat
 * grid indices, the exact mapping the kernels use; equals the reference's
 * np.flatnonzero(stage mask) order (latec/levels.py:184-208 mask_tiles). */
int latec_plan_stage_flat(const latec_plan* plan, int32_t stage, uint64_t first, uint64_t count,
                          int64_t* out_flat);

/* Bytes of device workspace latec_encode_stages / latec_decode_stages /
 * latec_quantize need for this plan. */
uint64_t latec_stage_workspace_bytes(const latec_plan* plan, int32_t channels, int32_t dtype);
uint64_t latec_flat_workspace_bytes(uint64_t items, int32_t dtype);

/* ---- fused predict + quantize + reconstruct over every stage of the plan:
 *      replaces latec/codec.py:384-459 (_compress_region) with
 *      latec/predictor.py:255-317 (InterpPredictor.predict) and
 *      latec/quantizer.py:28-120 (quantize / dequantize).
 * x, recon: (C, *spatial) device arrays of dtype; every point of recon is
 *   written (the call clears it first when a fused level mode is on).
 * stage_eb: host array, one absolute bound per stage.
 * codes: u16, C*n_t per stage, stage t at offset C*sum(n_<t).
 * outliers: dtype elements, stage t's compacted outliers at the same offset.
 * stats: device array of num_stages latec_stage_stats (zeroed by the call).
 * hist_seg: device, per stage and per 2^22-code segment, 512 u32 bins
 *   (bin 0 outliers, bin q+256 for |q| < 256), stage t at offset
 *   512*sum(segments_<t); zeroed by the call.
 * hist_total: device, num_stages * 65536 u32 code bins for |q| >= 256,
 *   zeroed by the call. */
int latec_encode_stages(const latec_plan* plan, const latec_quant_params* prm,
                        const double* stage_eb, const void* x, void* recon, uint16_t* codes,
                        void* outliers, latec_stage_stats* stats, uint32_t* hist_seg,
                        uint32_t* hist_total, void* workspace, uint64_t workspace_bytes,
                        void* stream);

/* ---- predict one stage from recon (InterpPredictor.predict,
 *      latec/predictor.py:255-317): pred gets C*n_t values, channel-major. */
int latec_interp_predict_stage(const latec_plan* plan, int32_t stage,
                               const latec_quant_params* prm, const void* recon, void* pred,
                               void* stream);

/* ---- quantize a compact array against a given prediction
 *      (latec/quantizer.py:28-87 + dequantize 90-111): the GNN path.
 *      recon_out gets the decoder's reconstruction; hist_seg/hist_total as
 *      above for one stage; stats one element. */
int latec_quantize(const latec_quant_params* prm, double eb, uint64_t items, const void* x,
                   const void* pred, uint16_t* codes, void* recon_out, void* outliers,
                   latec_stage_stats* stats, uint32_t* hist_seg, uint32_t* hist_total,
                   void* workspace, uint64_t workspace_bytes, void* stream);

/* ---- predictor-agnostic dequantize (latec/quantizer.py:82-120, and the
 *      learned codec's device twin latec/gnn_codec.py:1038-1044): recon_out[i]
 *      = the next outlier (scan order) where codes[i] == 0, else the
 *      quantizer's reconstruction of pred[i]; bit-identical to the recon_out
 *      of latec_quantize. err bit 1: the zero codes do not match n_out. */
uint64_t latec_dequantize_workspace_bytes(uint64_t items);
int latec_dequantize(const latec_quant_params* prm, double eb, uint64_t items, const void* pred,
                     const uint16_t* codes, const void* outliers, uint32_t n_out, void* recon_out,
                     uint32_t* err, void* workspace, uint64_t workspace_bytes, void* stream);

/* ---- scheduling of the decode stage kernels (no counterpart in the
 *      reference): 0 (default) = one launch per stage; 1 = levels of >= 4 Mi
 *      points run as one level kernel (work items per sub-stage and slab along
 *      axis 0, claimed in an order where every item's dependencies come
 *      first, so that slabs stay in L2); 2 = every level that qualifies.
 *      Results are bit-identical in all modes. Process-wide. */
int latec_set_level_mode(int32_t mode);

/* ---- fused levels of 3-D plans (no counterpart in the reference): the
 *      five sub-stages of a level (weight 1 along axes 0, 1, 2, weight 2,
 *      weight 3) in one launch each way, over column tiles of the level's
 *      lattice whose planes are staged in shared memory (TMA loads) with a
 *      3-point halo. 0 (default) = off (one launch per stage), 1 = the
 *      finest level, 2 = every level of at least 2^18 points, 3 = every
 *      level. Results are bit-identical in all modes. Process-wide. */
int latec_set_tile_mode(int32_t mode);

/* ---- row segments (no counterpart in the reference): 1 (default) = the
 *      per-stage encode and decode walk each single-class stage (anchors,
 *      weight-1 sub-stages) of a rank 2..4 single-channel plan in warp
 *      segments of 256 consecutive ranks along the grid rows (one rank
 *      decode and one set of tap offsets per segment, rows of at least 128
 *      stage points; decode tiles with outliers keep the per-point path);
 *      0 = one rank decode per point everywhere. Results are bit-identical.
 *      Process-wide. */
int latec_set_row_mode(int32_t on);

/* ---- kernel timing (a measurement aid, no counterpart in the reference):
 *      with timing on, a CUDA event pair is recorded on the launching stream
 *      around every fused level launch and every native lane-coder launch.
 *      latec_kernel_time sums the recorded pairs of one kind (0 = fused encode
 *      of a finest level, 1 = its decode, 2 = lane encode, 3 = lane decode,
 *      4 / 5 = fused encode / decode of a coarser level; it waits for their
 *      end events), returns the milliseconds and the launch count, and clears
 *      them. Process-wide. */
int latec_set_kernel_timing(int32_t on);
int latec_kernel_time(int32_t kind, double* ms, uint32_t* launches);

/* ---- decode: predict + dequantize over every stage
 *      (latec/codec.py:462-510 _decompress_region). codes as produced by
 *      latec_rans_decode; outliers: device byte array holding every stage's
 *      outliers (dtype elements, no alignment required), stage t starting at
 *      byte out_off[t] with n_out[t] entries (host arrays). err: device word,
 *      bit 1 = outlier count mismatch. Every point of recon is written (the
 *      call clears it first when a fused level or level-scheduling mode is
 *      on). */
int latec_decode_stages(const latec_plan* plan, const latec_quant_params* prm,
                        const double* stage_eb, const uint16_t* codes, const void* outliers,
                        const uint64_t* out_off, const uint32_t* n_out, void* recon,
                        uint32_t* err, void* workspace, uint64_t workspace_bytes, void* stream);

/* ---- many tensors per call (no counterpart in the reference, whose batch
 *      form is a serial loop of latec/codec.py:45-285 compress and
 *      :288-381 decompress). One job per tensor holds the arguments
 *      latec_encode_stages / latec_decode_stages take for it (stage_eb,
 *      out_off and n_out are host arrays, the rest device memory as there).
 *      The jobs' stage passes run stage index by stage index: per stage index
 *      one launch per kernel class (value type, rank, stage layout) covers
 *      that stage of every tensor that has it, with one zeroing launch and
 *      (encode) one outlier-compaction launch beside it. Results equal one
 *      latec_encode_stages / latec_decode_stages call per job, bit for bit
 *      (codes, outliers, reconstructions, histograms, counts; the float64
 *      statistic sums may differ in their last bits when max_ctas changes the
 *      CTA split); the fused levels of latec_set_tile_mode and the level
 *      scheduling of latec_set_level_mode are not used. max_ctas: the encode
 *      CTAs of one stage of the job (0 = the single-tensor default).
 *      table: device scratch of latec_*_many_table_bytes bytes; the call
 *      uploads its launch tables there (the host copy is taken before the
 *      call returns). The stage descriptors of each plan are uploaded to the
 *      device once, on the plan's first many-tensor call. */
typedef struct latec_encode_job {
    const latec_plan* plan;
    latec_quant_params prm;
    const double* stage_eb;
    const void* x;
    void* recon;
    uint16_t* codes;
    void* outliers;
    latec_stage_stats* stats;
    uint32_t* hist_seg;
    uint32_t* hist_total;
    void* workspace;
    uint64_t workspace_bytes;
    uint32_t max_ctas;
    uint32_t reserved;
} latec_encode_job;

typedef struct latec_decode_job {
    const latec_plan* plan;
    latec_quant_params prm;
    const double* stage_eb;
    const uint16_t* codes;
    const void* outliers;
    const uint64_t* out_off;
    const uint32_t* n_out;
    void* recon;
    uint32_t* err;
} latec_decode_job;

uint64_t latec_encode_many_table_bytes(const latec_encode_job* jobs, int32_t n_jobs);
int latec_encode_stages_many(const latec_encode_job* jobs, int32_t n_jobs, void* table,
                             uint64_t table_bytes, void* stream);
uint64_t latec_decode_many_table_bytes(const latec_decode_job* jobs, int32_t n_jobs);
int latec_decode_stages_many(const latec_decode_job* jobs, int32_t n_jobs, void* table,
                             uint64_t table_bytes, void* stream);

/* ---- rANS tables: encoder symbols and decoder buckets for `rows` CDF rows
 *      of alphabet + 1 entries (latec/rans.py:304-329 tables, compiled the
 *      way latec/rans.py:629-657 compiles constriction models). enc: device,
 *      32 bytes per entry, rows * (alphabet + 1) entries; bucket: device,
 *      1024 entries per row. Either may be NULL to skip it. */
int latec_rans_build_tables(const uint32_t* cdf_rows, int32_t alphabet, int32_t rows, void* enc,
                            uint16_t* bucket, void* stream);

/* Bytes of device workspace latec_rans_encode needs for these stages
 * (fills scratch_off / n_chunks / chunk0 of the host array). */
uint64_t latec_rans_encode_workspace_bytes(latec_rans_stage* stages, int32_t n_stages);

/* ---- entropy-code every stage and assemble the stage records.
 *      On return the workspace starts with the n_stages stage descriptors
 *      (device copy) with blob_words, n_out and rec_off filled in
 *      (latec/bitstream.py:178-243 pack_stage with latec/rans.py:466-498
 *      rans_encode_const / 546-578 rans_encode) into `payload` on the
 *      device: per stage u32 n | u64 frame | blob | u32 n_out | outliers.
 *      payload_len: device u64; err: device u32 (bit 2: symbol outside the
 *      alphabet, bit 32: payload capacity exceeded). */
int latec_rans_encode(latec_rans_stage* stages, int32_t n_stages, const uint16_t* codes,
                      const uint8_t* levels, const latec_stage_stats* stats,
                      const void* outliers, int32_t elem, uint8_t* payload, uint64_t payload_cap,
                      uint64_t* payload_len, uint32_t* err, void* workspace,
                      uint64_t workspace_bytes, void* stream);

/* ---- decode every stage's rANS blob (latec/bitstream.py:288-344
 *      unpack_stage with latec/rans.py:501-535 / 581-616) into codes.
 *      words: device u32 array holding the blobs (stage t at blob_off);
 *      chunk_range: device u64 pairs (start, end) of every lane-coder chunk
 *      stream, as absolute word offsets in `words`, global chunk order.
 *      err bits: 4 read past a chunk, 8 bad final state, 16 compat stream. */
uint64_t latec_rans_decode_workspace_bytes(int32_t n_stages);
int latec_rans_decode(latec_rans_stage* stages, int32_t n_stages, uint32_t total_chunks,
                      const uint32_t* words, const uint64_t* chunk_range, const uint8_t* levels,
                      uint16_t* codes, uint32_t* err, void* workspace, uint64_t workspace_bytes,
                      void* stream);

/* ---- native-mode stage model fit on the device: the reference's
 *      (level, shape) argmin (latec/rans.py:395-430) over exact costs, the
 *      64-bit sum of rint(W * 2^20) * count with W the float32 -log2 p
 *      weights. stages_host: n latec_fit_stage_size()-byte descriptors (see
 *      fit_kernels.cu); hist_seg / hist_total as written by
 *      latec_encode_stages; counts: device u32 scratch (sum of alphabets);
 *      costs: device 8-byte scratch (n * 24 * 64; holds the integer sums);
 *      out: device f64 (3 per stage: cost in bits = sum * 2^-20, level,
 *      shape id). */
uint64_t latec_fit_stage_size(void);
int latec_fit_const(const void* stages_host, int32_t n, const uint32_t* hist_seg,
                    const uint32_t* hist_total, uint32_t* counts, double* costs, double* out,
                    void* workspace, uint64_t workspace_bytes, void* stream);

/* ---- container framing on the device (latec/bitstream.py:155-164
 *      write_stream / read_stream): out = header[hlen] followed by a zstd
 *      frame of raw blocks holding the n payload bytes, and the inverse
 *      (frame = the zstd frame after the header). */
uint64_t latec_raw_frame_bytes(uint64_t payload_bytes);
int latec_frame_raw(const uint8_t* payload, uint64_t n, const uint8_t* header, uint32_t hlen,
                    uint8_t* out, uint64_t out_cap, void* stream);
/* err (device, may be NULL): bit 64 = a raw block header differs from the
 * layout latec_frame_raw writes. */
int latec_unframe_raw(const uint8_t* frame, uint64_t n, uint8_t* payload, uint32_t* err,
                      void* stream);

/* ---- stage-record walk on the device (latec/bitstream.py:288-344):
 *      records gets n_stages entries of latec_record_size() bytes
 *      {u64 blob, u64 out_at, u64 frame, u32 n, u32 n_out, u32 K,
 *       u32 n_chunks, u32 chunk0, u32 status}; total_chunks (device u64) the
 *      lane-coder chunk count. latec_chunk_ranges then writes each chunk's
 *      (start, end) word offsets for latec_rans_decode (err bit 128: a chunk
 *      table that does not fill its blob). */
uint64_t latec_record_size(void);
int latec_parse_records(const uint8_t* payload, uint64_t n_bytes, int32_t n_stages, int32_t elem,
                        int32_t lanes, void* records, uint64_t* total_chunks, void* stream);
int latec_chunk_ranges(const uint32_t* words, const void* records, int32_t n_stages,
                       uint64_t* ranges, uint32_t* err, void* stream);

/* ---- per-point rANS support (the learned path's entropy stage).
 *      latec_scale_levels: latec/rans.py:270-278 scale_to_level -- level of
 *      each float32 scale = number of the n_levels - 1 ascending float32
 *      thresholds (host array) not above it; NaN gives level 0.
 *      latec_level_order: the symbol order of latec/rans.py:546-578 (level 0
 *      first, each level in index order) as a permutation order[j] = index of
 *      the j-th coded symbol (stable counting sort; n < 2^32).
 *      latec_permute: dst[j] = src[order[j]] (inverse = 0) or
 *      dst[order[j]] = src[j] (inverse = 1), elem 1, 2 or 4 bytes.
 *      latec_point_bits: latec/rans.py:332-357 model_bits, n_partial float64
 *      partial sums (one per CTA, summed by the caller); err bit 1 = a code
 *      outside the window.
 *      latec_shape_costs: latec/rans.py:204-243 choose_shape costs over every
 *      step-th symbol, n_partial partials per shape (shape-major). */
int latec_scale_levels(const float* scale, uint64_t n, const float* thresholds, int32_t n_levels,
                       uint8_t* levels, void* stream);
uint64_t latec_level_order_workspace_bytes(uint64_t n);
int latec_level_order(const uint8_t* levels, uint64_t n, uint32_t* order, void* workspace,
                      uint64_t workspace_bytes, void* stream);
int latec_permute(const void* src, int32_t elem, const uint32_t* order, uint64_t n, void* dst,
                  int32_t inverse, void* stream);
int latec_point_bits(const uint16_t* codes, const uint8_t* levels, uint64_t n, const uint32_t* cdf,
                     uint32_t alphabet, int32_t radius, int32_t kexp, double* partial,
                     int32_t n_partial, uint32_t* err, void* stream);
int latec_shape_costs(const uint16_t* codes, const uint8_t* levels, uint64_t n, uint64_t step,
                      const double* weights, uint32_t alphabet, int32_t n_levels, int32_t radius,
                      int32_t kexp, double floor_p, const int32_t* shape_d, const double* shape_w,
                      int32_t n_shapes, double* partial, int32_t n_partial, void* stream);

/* ---- the axial GNN predictor of the learned path (latec/gnn_predictor.py).
 *      Parameters: one packed float32 device buffer of
 *      latec_gnn_param_count(d, agg_level) floats, the reference state_dict
 *      tensors (build_model, :593-933) concatenated in this order: init.net.0,
 *      init.net.2, dir_state.table, dir.net.0, dir.net.2, bidir.net.0,
 *      bidir.net.2, line_pool {wk.0, wk.2, wv, null_k, null_v}, axis_pool
 *      {same}, head.net.0, head.net.2, mix.net.0, mix.net.2 (weight before
 *      bias). E: the (B, N, K, d) float32 embedding field; contexts
 *      (B, M, K, d). Geometry: one stage's queries and, per line, the nearest
 *      known neighbour on each side (:245-443 _StageGeom), with the live pairs
 *      listed per query tile (two-sided first, then one-sided).
 *      float32 arithmetic in a fixed order: identical on every run. */
typedef struct {
    int32_t d, agg_level;
    const float* params;
    /* optional: BiDirEmbed, DirEmbed and MixEmbed weights packed by
     * latec_gnn_pack_bf16 (in that order, first then second layer each), then
     * the line pool's key MLP with its value projection: line_pool.wk.0 and
     * line_pool.wv stacked (128 x 64, packed as one 128-row operand),
     * line_pool.wk.2 zero-padded to 32 x 64 rows, and its bias as 32 float32
     * (the first the real one, the rest 0); runs those layers in BF16 on the
     * tensor cores (d = 64 only); NULL = float32 */
    const void* packed_bf16;
    uint32_t* tc_err;  /* device word, bit 1: a tensor-core wait ran out */
    /* optional, instead of packed_bf16: the same six layers packed by
     * latec_gnn_pack_fp8 (E4M3) with their per-output-channel scales in the
     * same order (128, 64, 128, 64, 128, 64 floats); NULL = not used */
    const void* packed_fp8;
    const float* fp8_scales;
} latec_gnn_model;

typedef struct {
    int32_t M, L, K, m_tile, n_tiles;
    const int32_t* query;   /* device (M) flat indices */
    const int32_t* nbr_p;   /* device (L, M), -1 = no neighbour */
    const int32_t* nbr_n;
    const float* logd_p;    /* device (L, M) log2 distance + line term */
    const float* logd_n;
    const int32_t* two;     /* device: two-sided pair ids l * M + m, per tile */
    const int32_t* one;     /* device: one-sided pair ids, per tile */
    const int32_t* row_of;  /* device (L, M): tile-local live row, -1 = dead */
    const int64_t* two_off; /* host (n_tiles + 1) */
    const int64_t* one_off; /* host (n_tiles + 1) */
    const int32_t* sidx_p;  /* device (L, K) direction-state rows */
    const int32_t* sidx_n;
} latec_gnn_geom;

uint64_t latec_gnn_param_count(int32_t d, int32_t agg_level);
uint64_t latec_gnn_workspace_bytes(int32_t d, int32_t B, int32_t M, int32_t L, int32_t K,
                                   int32_t m_tile);
/* GNN.embed (:843-871): per-axis contexts of the stage's queries. */
int latec_gnn_embed(const latec_gnn_model* model, int32_t B, int64_t N, const float* E,
                    const latec_gnn_geom* geom, float* ctx, void* workspace,
                    uint64_t workspace_bytes, void* stream);
/* GNN.head_of + PredHead (:760-790, 922-931): mu, log2 b per query. */
int latec_gnn_head(const latec_gnn_model* model, int32_t B, int32_t M, int32_t K, const float* ctx,
                   float eb, float* mu, float* log_b, void* workspace, uint64_t workspace_bytes,
                   void* stream);
/* GNN.finalize (:901-920): E[b, query[m], k] = Mix(ctx, Init(vals[b, m])). */
int latec_gnn_finalize(const latec_gnn_model* model, int32_t B, int64_t N, int32_t M, int32_t K,
                       const int32_t* query, const float* ctx, const float* vals, float* E,
                       void* workspace, uint64_t workspace_bytes, void* stream);

/* ---- tensor-core MLP of the GNN message pass (BiDirEmbed / DirEmbed /
 *      MixEmbed, latec/gnn_predictor.py:624-661,792-806): Y = W2 * gelu(W1 * X
 *      + b1) + b2 with hidden width 128 and output width 64, BF16 operands
 *      and FP32 accumulation on tcgen05. Weights are packed on the host into
 *      the tensor cores' BF16 layout by latec_gnn_pack_bf16 (n x k float32,
 *      k zero-padded to kp, a multiple of 16; out: n * kp uint16). err bit 1:
 *      a tensor-core completion wait ran out (the output is invalid). */
int latec_gnn_pack_bf16(const float* w, int32_t n, int32_t k, int32_t kp, uint16_t* out);
/* FP8 variant: E4M3 operands with one scale per weight output channel
 * (max |w| / 448) and per row of the activations (input rows and the hidden
 * layer), FP32 accumulation; kp a multiple of 32; out n * kp bytes, scales n
 * floats (host). */
int latec_gnn_pack_fp8(const float* w, int32_t n, int32_t k, int32_t kp, uint8_t* out,
                       float* scales);
int latec_gnn_mlp2_fp8(const float* X, int32_t ldx, int64_t rows, int32_t k1, int32_t k1p,
                       const void* w1p, const float* s1, const float* b1, const void* w2p,
                       const float* s2, const float* b2, float* Y, int32_t ldy, uint32_t* err,
                       void* stream);
int latec_gnn_mlp2_bf16(const float* X, int32_t ldx, int64_t rows, int32_t k1, int32_t k1p,
                        const void* w1p, const float* b1, const void* w2p, const float* b2,
                        float* Y, int32_t ldy, uint32_t* err, void* stream);

/* ---- flat quantizer without any device allocation (no counterpart in the
 *      reference). For callers that cannot call cudaMalloc -- e.g. an
 *      application whose GPU memory is owned by another allocator, or a
 *      latency-critical loop where cudaMalloc/cudaFree would synchronise the
 *      device. Same inputs, outputs and results as latec_quantize, but its
 *      scratch is a file-scope device array (about 4 MiB, held by every GPU
 *      that loads the library until exit) instead of a caller workspace.
 *      items must not exceed LATEC_STATIC_MAX_ITEMS (else
 *      LATEC_ERR_TOO_LARGE). All calls on a device share that array: calls
 *      whose GPU work overlaps race and must not be issued. The first call on
 *      each device looks the array up (cudaGetSymbolAddress); make it before
 *      any stream capture. The lookup is repeated in a new context of the
 *      device (after cudaDeviceReset, say), so the first call after a reset
 *      should likewise come before any capture. */
#define LATEC_ERR_TOO_LARGE (-7)
#define LATEC_STATIC_MAX_ITEMS (1u << 19)
int latec_quantize_static(const latec_quant_params* prm, double eb, uint64_t items, const void* x,
                          const void* pred, uint16_t* codes, void* recon_out, void* outliers,
                          latec_stage_stats* stats, uint32_t* hist_seg, uint32_t* hist_total,
                          void* stream);

/* Library version string. */
const char* latec_version(void);

/* Number of CUDA kernel launches this library has issued in this process. */
uint64_t latec_launch_count(void);

/* ---- scale-gated interpolation fallback of the learned codec
 *      (latec/gnn_codec.py:386-462, 776-1000). latec_gate_costs adds, per
 *      scale bucket (the number of thresholds eb * 2^T, T = 2..13, below the
 *      model scale b), the rANS-aligned Laplace bits of the GNN residual
 *      (row 0) and of each candidate ip0..ip2 (cubic, first-axis linear,
 *      last-axis linear; NULL = skipped) at scale b * 2^-2s, s = 0..3 (row
 *      1 + 4 k + s), into sums (13 x 13, 2^-20-bit fixed point, zeroed by the
 *      caller). thr / grid: the 64-level scale grid (63 float32 boundaries,
 *      64 float64 values). latec_gate_apply replaces mu by ip and b by
 *      b * 2^-shift where b < eb * 2^T (high = 0) or b >= eb * 2^T (high = 1). */
int latec_gate_costs(int64_t n, const float* x, const float* mu, const float* ip0,
                     const float* ip1, const float* ip2, const float* b, double eb, int32_t radius,
                     const float* thr, const double* grid, uint64_t* sums, void* stream);
int latec_gate_apply(int64_t n, float* mu, float* b, const float* ip, double eb, int32_t T,
                     int32_t shift, int32_t high, void* stream);
/* The same choice and application without a host round trip (no counterpart
 * in the reference): latec_gate_choose_apply reduces the sums to the gate word
 * on the device (the split rule of _gate_select_t, latec/gnn_codec.py:920-971:
 * the least-cost low- or high-side split over candidates, shifts and
 * thresholds, kept only when it codes fewer bits than the GNN), writes it to
 * *word (layout dir << 10 | kind << 8 | T << 4 | shift; 0 = the GNN
 * everywhere) and applies it with ip0..ip2; latec_gate_apply_word applies a
 * word already on the device. */
int latec_gate_choose_apply(int64_t n, const uint64_t* sums, float* mu, float* b, const float* ip0,
                            const float* ip1, const float* ip2, double eb, uint32_t* word,
                            void* stream);
int latec_gate_apply_word(int64_t n, float* mu, float* b, const float* ip0, const float* ip1,
                          const float* ip2, double eb, const uint32_t* word, void* stream);

/* ---- training of the learned predictor (scripts/train_gnn.py): forward
 *      ops that keep what their backward needs, the backward ops, the
 *      discretised-Laplace rate loss and the AdamW / EMA updates. float32;
 *      weights (out, in) row-major as nn.Linear; device pointers; stream may
 *      be NULL. Gradient buffers accumulate (zero them per step). */
/* Y = act(X W^T + b), act 1 = GELU; Z (optional) keeps the pre-activation. */
int latec_tr_linear(const float* X, int64_t ldx, int64_t rows, int32_t in, const float* W,
                    const float* b, int32_t out, float* Y, int64_t ldy, int32_t act, float* Z,
                    void* stream);
/* dX = dZ W (stored, or added when accum_dx; dX may be NULL), dW += dZ^T X,
 * db += sum dZ, dZ = dY * gelu'(Z) when act. */
int latec_tr_linear_bwd(const float* X, int64_t ldx, int64_t rows, int32_t in, const float* W,
                        int32_t out, const float* dY, int64_t ldy, const float* Z, int32_t act,
                        float* dX, int64_t lddx, int32_t accum_dx, float* dW, float* db,
                        void* stream);
/* The same two ops with BF16 GEMM operands and float32 accumulation: mixed-
 * precision training with float32 master weights, as the reference's
 * optional FP16 autocast (scripts/train_gnn.py:147-150, GradScaler at 938);
 * BF16 keeps float32's exponent range, so no loss scale is needed. Both
 * operands of each GEMM are rounded to BF16 (nearest even) as they are
 * staged; tcgen05 tensor cores with tensor-memory accumulators where both
 * output dimensions are at least 32, SIMT tiles for the narrow layers. Bias,
 * activation, saved pre-activation and gradients stay float32. */
int latec_tr_linear_bf16(const float* X, int64_t ldx, int64_t rows, int32_t in, const float* W,
                         const float* b, int32_t out, float* Y, int64_t ldy, int32_t act, float* Z,
                         void* stream);
int latec_tr_linear_bwd_bf16(const float* X, int64_t ldx, int64_t rows, int32_t in,
                             const float* W, int32_t out, const float* dY, int64_t ldy,
                             const float* Z, int32_t act, float* dX, int64_t lddx,
                             int32_t accum_dx, float* dW, float* db, void* stream);
/* Reads and clears the tensor-core GEMMs' error word; LATEC_ERR_INTERNAL if
 * an MMA completion wait ran out since the last call (its tile is then not
 * written). Synchronises the stream. */
int latec_tr_gemm_status(void* stream);
/* Message rows of all batches (two-sided when two, else one-sided) for the
 * pairs of a stage (latec/gnn_predictor.py:618-660 BiDirEmbed / DirEmbed
 * inputs) and their backward into dE and the direction-state table. */
int latec_tr_rows(const float* E, int64_t N, int32_t K, int32_t d, int32_t ds, const float* table,
                  const latec_gnn_geom* geom, const int32_t* pairs, int64_t np, int32_t B,
                  int32_t two, float* X, int32_t ldx, void* stream);
int latec_tr_rows_bwd(const float* dX, int32_t ldx, int64_t N, int32_t K, int32_t d, int32_t ds,
                      const latec_gnn_geom* geom, const int32_t* pairs, int64_t np, int32_t B,
                      int32_t two, float* dE, float* dtable, void* stream);
int latec_tr_line_rows(const int32_t* row_of, int32_t M, int32_t L, int32_t K, int32_t B,
                       int64_t np2, int64_t np1, int32_t* rows, void* stream);
/* AttnPool (latec/gnn_predictor.py:724-749) keeping the probabilities P
 * (n_out x (n + 1), null token last), and its backward. */
int latec_tr_attn(const float* key, const float* V, int32_t d, const int32_t* rows, int32_t n,
                  int64_t n_out, float scale, const float* null_k, const float* null_v, float* out,
                  float* P, void* stream);
int latec_tr_attn_bwd(const float* V, int32_t d, const int32_t* rows, int32_t n, int64_t n_out,
                      float scale, const float* null_v, const float* P, const float* dout,
                      float* dkey, float* dV, float* dnull_k, float* dnull_v, void* stream);
/* PredHead rows / readout with a per-sample log2 eb, and the readout's
 * backward. */
int latec_tr_head_rows(const float* pooled, int64_t n, int32_t per_b, int32_t d,
                       const float* log_eb, float* X, void* stream);
int latec_tr_head_out(const float* O, int64_t n, int32_t per_b, const float* log_eb, float* mu,
                      float* log_b, void* stream);
int latec_tr_head_out_bwd(const float* O, const float* mu, int64_t n, const float* dmu,
                          const float* dlog_b, float* dO, void* stream);
/* discretized_laplace_nll (bits) + mse_weight * squared error of n points
 * (sample = i / per_b, bound eb[sample]); acc[0..2] += bits, squared error,
 * |error| (double); dmu / dlog_b = scale * d(bits + mse_weight * sq). */
int latec_tr_loss(const float* mu, const float* log_b, const float* tgt, int64_t n, int32_t per_b,
                  const float* eb, float mse_weight, float scale, float* dmu, float* dlog_b,
                  double* acc, void* stream);
/* MixEmbed rows [ctx | value embedding] and backward; E scatter of the
 * finalised rows (backward = 1 gathers dE into Y). */
int latec_tr_mix_rows(const float* ctx, const float* vemb, int64_t bmk, int32_t K, int32_t d,
                      float* X, void* stream);
int latec_tr_mix_rows_bwd(const float* dX, int64_t bmk, int32_t K, int32_t d, float* dctx,
                          float* dvemb, void* stream);
int latec_tr_scatter_e(float* Y, const int32_t* query, int32_t B, int32_t M, int32_t K, int32_t d,
                       int64_t N, float* E, int32_t backward, void* stream);
/* torch.optim.AdamW step (decoupled decay, bias-corrected) and the EMA
 * shadow update. */
int latec_tr_adamw(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1,
                   float b2, float eps, float wd, int64_t step, void* stream);
int latec_tr_ema(float* shadow, const float* p, int64_t n, float decay, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LATEC_B200_H */
