// Fused dyadic interpolation + error-bounded quantizer (encode) and
// interpolation + dequantizer (decode) for one sub-stage of the schedule.
//
// Bit-exactness contract with the reference (latec/predictor.py:97-156,
// 255-317; latec/quantizer.py:28-120): every prediction is evaluated in
// float64 on the float32 (or float64) reconstruction, in the reference's
// operation order, with explicitly rounded intrinsics so that nothing is
// contracted into an FMA; the quotient (x - p) / 2eb is the correctly rounded
// float64 division (a reciprocal product is used only when it provably rounds
// to the same integer); the reconstruction is f32(p + 2eb * q) and the bound is
// verified in float32 exactly as the reference decoder computes it.
#include <atomic>

#include <cuda_runtime.h>

#include "interp_device.cuh"
#include "tile_kernels.cuh"

namespace latec {

template <typename T>
__device__ __forceinline__ double ldv(const T* p) {
    return (double)__ldg(p);
}

// 1-D line rule along one odd axis (c >= s always holds there, so the -s tap
// is valid): cubic / quadratic ends / linear, else the one-sided rule.
// latec/predictor.py:121-156.
template <typename T>
__device__ __forceinline__ double axis_interp(const T* __restrict__ rc, int64_t flat, int c,
                                              int n, int64_t gs, int s, int cubic, int em) {
    const int64_t o1 = (int64_t)s * gs;
    const double Lm1 = ldv(rc + flat - o1);
    const bool vp1 = c + s < n;
    const bool vm3 = c - 3 * s >= 0;
    if (vp1) {
        const double Lp1 = ldv(rc + flat + o1);
        const double lin = 0.5 * __dadd_rn(Lm1, Lp1);
        if (!cubic) return lin;
        const bool vp3 = c + 3 * s < n;
        if (vm3 && vp3) {
            const double Lm3 = ldv(rc + flat - 3 * o1);
            const double Lp3 = ldv(rc + flat + 3 * o1);
            double t = __dadd_rn(-Lm3, __dmul_rn(9.0, Lm1));
            t = __dadd_rn(t, __dmul_rn(9.0, Lp1));
            t = __dsub_rn(t, Lp3);
            return t * 0.0625;
        }
        if (em & 1) {
            if (vp3) {  // interp_quad_1: leading end
                const double Lp3 = ldv(rc + flat + 3 * o1);
                double t = __dadd_rn(__dmul_rn(3.0, Lm1), __dmul_rn(6.0, Lp1));
                t = __dsub_rn(t, Lp3);
                return t * 0.125;
            }
            if (vm3) {  // interp_quad_2: trailing end
                const double Lm3 = ldv(rc + flat - 3 * o1);
                double t = __dadd_rn(-Lm3, __dmul_rn(6.0, Lm1));
                t = __dadd_rn(t, __dmul_rn(3.0, Lp1));
                return t * 0.125;
            }
        }
        return lin;
    }
    if ((em & 2) && vm3) {  // interp_linear1 extrapolation past the line end
        const double Lm3 = ldv(rc + flat - 3 * o1);
        return __dsub_rn(__dmul_rn(1.5, Lm1), __dmul_rn(0.5, Lm3));
    }
    return Lm1;
}

// Prediction of one stage point from its own odd axes (center combine of
// latec/predictor.py:286-314; terms of even axes are exact zeros there).
// ND/KIND/CUBIC specialise the rank, the stage layout and the interpolation
// order at compile time (ND == 0: runtime rank).
template <typename T, int ND, int KIND, int CUBIC>
__device__ __forceinline__ double predict_point(const StageDesc& d, const QParams& q,
                                                const T* __restrict__ rc, int64_t flat,
                                                const int32_t* coord) {
    constexpr int NDV = ND > 0 ? ND : MAXD;
    if (KIND == 0) {
        int ca = 0, na = 1;
        int64_t gs = 0;
#pragma unroll
        for (int j = 0; j < NDV; j++) {
            if (j == d.axis) {
                ca = coord[j];
                na = d.shape[j];
                gs = d.gstride[j];
            }
        }
        return axis_interp(rc, flat, ca, na, gs, d.s, CUBIC, q.end_mode);
    }
    if (q.center == 0) {
        double total = 0.0;
        int cnt = 0;
#pragma unroll
        for (int j = 0; j < NDV; j++) {
            if ((ND > 0 || j < d.ndim) && (coord[j] & d.s)) {
                const double v = axis_interp(rc, flat, coord[j], d.shape[j], d.gstride[j], d.s,
                                             CUBIC, q.end_mode);
                total = cnt ? __dadd_rn(total, v) : v;
                cnt++;
            }
        }
        if (cnt == 1) return total;
        if (cnt == 2) return total * 0.5;
        if (cnt == 4) return total * 0.25;
        return __ddiv_rn(total, (double)cnt);
    }
    int ca = 0, na = 1;
    int64_t gs = 0;
    bool found = false;
#pragma unroll
    for (int j = 0; j < NDV; j++) {
        if ((ND > 0 || j < d.ndim) && (coord[j] & d.s) && (q.center == 2 || !found)) {
            ca = coord[j];
            na = d.shape[j];
            gs = d.gstride[j];
            found = true;
        }
    }
    return axis_interp(rc, flat, ca, na, gs, d.s, CUBIC, q.end_mode);
}

// Per-block statistics: warp shuffles, then one partial row per CTA.
__device__ __forceinline__ void block_finish(BlockAcc& a, double* partials, StageAcc* acc,
                                             uint32_t bid) {
    __shared__ double sh_red[5][THREADS / 32];
    __shared__ uint32_t sh_mq[THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; k++) a.s[k] = warp_sum(a.s[k]);
    a.s[4] = warp_max(a.s[4]);
    a.maxq = warp_umax(a.maxq);
    uint32_t no = a.nout;
#pragma unroll
    for (int o = 16; o; o >>= 1) no += __shfl_xor_sync(0xffffffffu, no, o);
    __shared__ uint32_t sh_no[THREADS / 32];
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 5; k++) sh_red[k][wid] = a.s[k];
        sh_mq[wid] = a.maxq;
        sh_no[wid] = no;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s[5] = {0, 0, 0, 0, 0};
        uint32_t mq = 0, nt = 0;
        for (int w = 0; w < THREADS / 32; w++) {
            for (int k = 0; k < 4; k++) s[k] += sh_red[k][w];
            s[4] = fmax(s[4], sh_red[4][w]);
            mq = max(mq, sh_mq[w]);
            nt += sh_no[w];
        }
        for (int k = 0; k < 5; k++) partials[(size_t)bid * 5 + k] = s[k];
        if (mq) atomicMax(&acc->maxq, mq);
        if (nt) atomicAdd(&acc->nout, nt);
    }
}

// ---------------------------------------------------------------- stage tail
// Run by the last CTA of a stage pass (the one whose arrival completes the
// per-stage counter): the fixed-order reduction of the per-CTA statistics and
// the exclusive scan of the per-tile outlier counts. Both are deterministic:
// neither depends on which CTA happens to arrive last.
__device__ void stage_tail(const double* __restrict__ partials, uint32_t blocks,
                           const uint32_t* __restrict__ tile_cnt, uint32_t tiles,
                           uint32_t* __restrict__ tile_off, StageAcc* __restrict__ acc) {
    __shared__ double red[5][THREADS];
    __shared__ uint32_t sc[THREADS];
    double s[5] = {0, 0, 0, 0, 0};
    for (uint32_t b = threadIdx.x; b < blocks; b += THREADS) {
        for (int k = 0; k < 4; k++) s[k] += partials[(size_t)b * 5 + k];
        s[4] = fmax(s[4], partials[(size_t)b * 5 + 4]);
    }
    for (int k = 0; k < 5; k++) red[k][threadIdx.x] = s[k];
    // tile scan (only when the stage has outliers): thread t sums a contiguous
    // run of tiles, then a block scan of the runs
    const bool any = *(volatile uint32_t*)&acc->nout != 0;
    const uint32_t per = any ? (tiles + THREADS - 1) / THREADS : 0;
    const uint32_t a = threadIdx.x * per, e = min(tiles, a + per);
    uint32_t run = 0;
    for (uint32_t i = a; i < e; i++) run += tile_cnt[i];
    sc[threadIdx.x] = run;
    __syncthreads();
    for (int o = THREADS / 2; o; o >>= 1) {
        if (threadIdx.x < (unsigned)o) {
            for (int k = 0; k < 4; k++) red[k][threadIdx.x] += red[k][threadIdx.x + o];
            red[4][threadIdx.x] = fmax(red[4][threadIdx.x], red[4][threadIdx.x + o]);
        }
        __syncthreads();
    }
    for (int o = 1; o < THREADS; o <<= 1) {
        const uint32_t v = threadIdx.x >= (unsigned)o ? sc[threadIdx.x - o] : 0u;
        __syncthreads();
        sc[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t off = sc[threadIdx.x] - run;
    for (uint32_t i = a; i < e; i++) {
        tile_off[i] = off;
        off += tile_cnt[i];
    }
    if (threadIdx.x == THREADS - 1) acc->n_out = any ? sc[THREADS - 1] : 0u;
    if (threadIdx.x == 0)
        for (int k = 0; k < 5; k++) acc->stats[k] = red[k][0];
}

// Arrival counter: true in the CTA that finishes the stage (nblk CTAs).
__device__ __forceinline__ bool last_block(StageAcc* acc, uint32_t nblk) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(&acc->done, 1u) == nblk - 1;
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// ---------------------------------------------------------------- encode
// A CTA owns a contiguous run of 512-point groups of the stage's ranks; each
// thread takes two points of a group (ranks g + tid and g + 256 + tid, so
// codes are written coalesced) and keeps both in flight: both predictions
// are issued before either result is stored. Outliers are counted into their
// 2048-point tile with global atomics (tile_cnt is zeroed by the caller); the
// shared histogram is flushed whenever the run crosses a 2^22-code segment.
template <typename T, int ND, int KIND, int CUBIC>
__device__ __forceinline__ double locate_predict(const StageDesc& d, const QParams& q,
                                                 const int is_anchor, uint64_t i,
                                                 const T* __restrict__ recon, int64_t& flat,
                                                 uint32_t& c) {
    c = 0;
    uint32_t rank = (uint32_t)i;
    if (q.channels > 1) {
        c = (uint32_t)(i / d.n);
        rank = (uint32_t)(i - (uint64_t)c * d.n);
    }
    int32_t coord[ND > 0 ? ND : MAXD];
    flat = stage_point_t<ND, KIND>(d, rank, coord);
    return is_anchor ? 0.0
                     : predict_point<T, ND, KIND, CUBIC>(d, q, recon + (uint64_t)c * q.points, flat,
                                                         coord);
}

// Locate one stage point and load its taps (prediction deferred to combine).
template <typename T, int ND, int KIND, int CUBIC, int COH = 0>
__device__ __forceinline__ void locate_gather(const StageDesc& d, const QParams& q,
                                              const int is_anchor, uint64_t i,
                                              const T* __restrict__ recon, int64_t& flat,
                                              uint32_t& c, PointTaps<T, ND, KIND>& pt) {
    c = 0;
    uint32_t rank = (uint32_t)i;
    if (q.channels > 1) {
        c = (uint32_t)(i / d.n);
        rank = (uint32_t)(i - (uint64_t)c * d.n);
    }
    int32_t coord[ND > 0 ? ND : MAXD];
    flat = stage_point_t<ND, KIND>(d, rank, coord);
    if (!is_anchor)
        gather_point<T, ND, KIND, CUBIC, COH>(d, q, recon + (uint64_t)c * q.points, flat, coord,
                                              pt);
}

template <typename T>
__device__ __forceinline__ void encode_value(const QParams& q, uint64_t i, T xv, double pd,
                                             T* __restrict__ dst, T* __restrict__ staging,
                                             uint32_t* __restrict__ tile_cnt,
                                             uint16_t* __restrict__ codes, BlockAcc& a, int& key,
                                             uint32_t& code) {
    T rv;
    const QOut o = Quant<T>::run(xv, pd, q, rv);
    *dst = rv;
    code = o.code;
    codes[i] = (uint16_t)o.code;
    if (!o.code) {
        staging[i] = xv;
        atomicAdd(&tile_cnt[i / TILE], 1u);
        a.nout++;
        key = 0;
    } else {
        const uint32_t aq = (uint32_t)abs(o.qv);
        a.maxq = max(a.maxq, aq);
        key = aq < HWIN ? o.qv + HWIN : -2;
    }
    const double e = Quant<T>::err(xv, pd);
    a.s[0] += fabs(e);
    a.s[1] += e * e;
    const double re = Quant<T>::rerr(xv, rv);
    a.s[2] += re;
    a.s[3] += re * re;
    a.s[4] = fmax(a.s[4], re);
}

// One CTA's share of an encode stage pass: CTA bid of nblk takes groups
// [bid * gpb, (bid + 1) * gpb); the last CTA to finish runs the stage tail.
template <typename T, int ND, int KIND, int CUBIC>
__device__ __forceinline__ void quant_cta(const StageDesc& d, const QParams& q,
                                          const int is_anchor, const uint32_t gpb,
                                          const uint32_t bid, const uint32_t nblk,
                                          const T* __restrict__ x, T* __restrict__ recon,
                                          uint16_t* __restrict__ codes, T* __restrict__ staging,
                                          uint32_t* __restrict__ tile_cnt,
                                          uint32_t* __restrict__ tile_off,
                                          uint32_t* __restrict__ hist_total,
                                          uint32_t* __restrict__ hist_seg,
                                          StageAcc* __restrict__ acc,
                                          double* __restrict__ partials) {
    __shared__ uint32_t sh_hist[HBINS];
    for (int b = threadIdx.x; b < HBINS; b += THREADS) sh_hist[b] = 0;
    __syncthreads();
    const uint64_t items = (uint64_t)q.channels * d.n;
    const uint64_t groups = (items + GROUP - 1) / GROUP;
    const uint64_t g0 = (uint64_t)bid * gpb;
    const uint64_t g1 = g0 + gpb < groups ? g0 + gpb : groups;
    const int lane = threadIdx.x & 31;
    BlockAcc a{{0, 0, 0, 0, 0}, 0, 0};
    uint32_t cur_seg = (uint32_t)((g0 * GROUP) >> SEG_SHIFT);
    for (uint64_t g = g0; g < g1; g++) {
        const uint64_t base = g * GROUP;
        const uint32_t seg = (uint32_t)(base >> SEG_SHIFT);
        if (seg != cur_seg) {  // uniform across the CTA
            __syncthreads();
            flush_hist(sh_hist, hist_seg, cur_seg);
            __syncthreads();
            cur_seg = seg;
        }
        const uint64_t i0 = base + threadIdx.x, i1 = i0 + THREADS;
        const bool v0 = i0 < items, v1 = i1 < items;
        int64_t f0 = 0, f1 = 0;
        uint32_t c0 = 0, c1 = 0;
        T x0 = (T)0, x1 = (T)0;
        PointTaps<T, ND, KIND> t0, t1;
        if (v0) {
            locate_gather<T, ND, KIND, CUBIC>(d, q, is_anchor, i0, recon, f0, c0, t0);
            x0 = x[(uint64_t)c0 * q.points + f0];
        }
        if (v1) {
            locate_gather<T, ND, KIND, CUBIC>(d, q, is_anchor, i1, recon, f1, c1, t1);
            x1 = x[(uint64_t)c1 * q.points + f1];
        }
        const double p0 = (v0 && !is_anchor) ? combine_point<T, ND, KIND, CUBIC>(q, t0) : 0.0;
        const double p1 = (v1 && !is_anchor) ? combine_point<T, ND, KIND, CUBIC>(q, t1) : 0.0;
        int k0 = -1, k1 = -1;
        uint32_t cd0 = 0, cd1 = 0;
        if (v0)
            encode_value<T>(q, i0, x0, p0, recon + (uint64_t)c0 * q.points + f0, staging, tile_cnt,
                            codes, a, k0, cd0);
        if (v1)
            encode_value<T>(q, i1, x1, p1, recon + (uint64_t)c1 * q.points + f1, staging, tile_cnt,
                            codes, a, k1, cd1);
        hist_warp(sh_hist, hist_total, k0, cd0, lane);
        hist_warp(sh_hist, hist_total, k1, cd1, lane);
    }
    __syncthreads();
    flush_hist(sh_hist, hist_seg, cur_seg);
    block_finish(a, partials, acc, bid);
    if (last_block(acc, nblk)) stage_tail(partials, nblk, tile_cnt, n_tiles_of(items), tile_off, acc);
}

// ---------------------------------------------------------------- row segments
// Consecutive ranks of a stage (single class or fused weight) run along the
// last axis of one grid row: xstep apart, the other coordinates fixed. A
// warp takes a segment of ROW_SEG consecutive ranks, decodes its first rank
// once and places the rest by offset along the row; the tap offsets of the
// fixed axes (and of the last axis, away from the row's ends) are set once
// per segment. Points past the row's end fall back to the per-point decode.
// The prediction, quantizer and bookkeeping are those of the per-point
// kernels, operation for operation.
constexpr int ROW_SEG = 256;                   // ranks per warp segment
constexpr int ROW_GROUP = ROW_SEG * THREADS / 32;  // ranks per CTA iteration

// Tap offsets of one axis from a point (elements): an out-of-line tap reads
// the -s tap, exactly as load_axis does.
struct SegTaps {
    int32_t m1, p1, m3, p3;
    uint32_t ok;
};

__device__ __forceinline__ SegTaps seg_taps(int c, int n, int32_t gs, int s) {
    const int32_t o1 = s * gs;
    const bool vp1 = c + s < n, vm3 = c - 3 * s >= 0, vp3 = c + 3 * s < n;
    return SegTaps{-o1, vp1 ? o1 : -o1, vm3 ? -3 * o1 : -o1, vp3 ? 3 * o1 : -o1,
                   (vp1 ? 1u : 0u) | (vm3 ? 2u : 0u) | (vp3 ? 4u : 0u)};
}

template <typename T, int CUBIC>
__device__ __forceinline__ void load_seg(const T* __restrict__ b, const SegTaps& o,
                                         AxisTaps<T>& t) {
    t.m1 = __ldg(b + o.m1);
    t.p1 = __ldg(b + o.p1);
    t.m3 = __ldg(b + o.m3);
    t.p3 = CUBIC ? __ldg(b + o.p3) : (T)0;
    t.ok = o.ok;
}

// A row segment: the decoded first point, the points left in its row, the
// axes its points interpolate along (in the order gather_point uses) and the
// tap offsets of the fixed axes.
template <int ND, int KIND>
struct RowSeg {
    int32_t coord[ND];
    int64_t flat;
    uint32_t rem;        // points of the row from the first one on
    int32_t xstep;
    uint32_t axes;       // bit j: taps along axis j (KIND 1, center 0: the odd axes)
    int32_t single;      // the one axis of KIND 0 / centers 1 and 2
    bool interior;       // last-axis taps of every point in line
    // taps of the fixed axes: t[0] for the single axis, t[j] for odd axis j
    // (the last axis's taps are +-s, +-3s when interior, else per point)
    SegTaps t[KIND ? ND - 1 : 1];
};

template <int ND, int KIND>
__device__ __forceinline__ void row_seg(const StageDesc& d, const QParams& q, uint32_t r,
                                        RowSeg<ND, KIND>& g) {
    constexpr int X = ND - 1;
    g.flat = stage_coords_t<ND, KIND>(d, r, g.coord);
    const int s = d.s, nx = d.shape[X];
    uint32_t m, len;
    if (KIND == 0) {
        g.xstep = d.step;
        m = (uint32_t)(g.coord[X] - d.start[X]) / (uint32_t)d.step;
        len = d.size_div[X].d;
    } else {
        g.xstep = 2 * s;
        m = (uint32_t)g.coord[X] >> d.lg2s;
        len = (g.coord[X] & s) ? (uint32_t)(nx + s - 1) >> d.lg2s
                               : (uint32_t)(nx + 2 * s - 1) >> d.lg2s;
    }
    g.rem = len - m;
    g.axes = 0;
    g.single = -1;
    if (KIND == 0) {
        g.single = d.axis;
    } else {
#pragma unroll
        for (int j = 0; j < ND; j++)
            if (g.coord[j] & s) {
                g.axes |= 1u << j;
                if (q.center == 2 || (q.center == 1 && g.single < 0)) g.single = j;
            }
        if (q.center == 0) g.single = -1;
    }
    const int64_t span = (int64_t)(ROW_SEG - 1) * g.xstep;
    g.interior = g.coord[X] - 3 * s >= 0 && g.coord[X] + span + 3 * s < nx;
#pragma unroll
    for (int j = 0; j < X; j++) {
        const SegTaps tj = seg_taps(g.coord[j], d.shape[j], (int32_t)d.gstride[j], s);
        if (g.single == j) g.t[0] = tj;
        if (KIND && g.single < 0 && ((g.axes >> j) & 1u)) g.t[KIND ? j : 0] = tj;
    }
}

// Taps of the segment point at offset k along the row (k < rem).
template <typename T, int ND, int KIND, int CUBIC>
__device__ __forceinline__ void row_gather(const StageDesc& d, const RowSeg<ND, KIND>& g,
                                           uint32_t k, const T* __restrict__ rc, int64_t& flat,
                                           PointTaps<T, ND, KIND>& pt) {
    constexpr int X = ND - 1;
    const int32_t off = (int32_t)k * g.xstep;
    flat = g.flat + off;
    const T* b = rc + flat;
    const int x = g.coord[X] + off, s = d.s;
    const SegTaps tx = g.interior ? SegTaps{-s, s, -3 * s, 3 * s, 7u}
                                  : seg_taps(x, d.shape[X], 1, s);
    pt.odd = 0;
    if (g.single >= 0) {
        load_seg<T, CUBIC>(b, g.single == X ? tx : g.t[0], pt.ax[0]);
        return;
    }
    pt.odd = g.axes;
#pragma unroll
    for (int j = 0; j < ND; j++) {
        if (!((g.axes >> j) & 1u)) continue;
        load_seg<T, CUBIC>(b, j == X ? tx : g.t[KIND && j < X ? j : 0], pt.ax[KIND ? j : 0]);
    }
}

// One point of a row segment: taps by segment offset when the point lies in
// the segment's row, else by the per-point decode.
template <typename T, int ND, int KIND, int CUBIC>
__device__ __forceinline__ void row_point(const StageDesc& d, const QParams& q,
                                          const int is_anchor, const RowSeg<ND, KIND>& g,
                                          uint32_t k,
                                          uint64_t i, const T* __restrict__ recon, int64_t& flat,
                                          PointTaps<T, ND, KIND>& pt) {
    if (k < g.rem) {
        if (is_anchor) {
            flat = g.flat + (int64_t)k * g.xstep;
            pt.odd = 0;
        } else {
            row_gather<T, ND, KIND, CUBIC>(d, g, k, recon, flat, pt);
        }
    } else {
        uint32_t c;
        locate_gather<T, ND, KIND, CUBIC>(d, q, is_anchor, i, recon, flat, c, pt);
    }
}

// The encode stage pass over row segments (single channel): CTA bid of nblk
// takes groups [bid * gpb, (bid + 1) * gpb) of ROW_GROUP ranks; warp w of the
// CTA the w-th segment of each group; lane l its points l, l + 32, ...
// (coalesced codes), two in flight.
template <typename T, int ND, int KIND, int CUBIC>
__device__ __forceinline__ void quant_rows_cta(const StageDesc& d, const QParams& q,
                                               const int is_anchor, const uint32_t gpb,
                                               const uint32_t bid, const uint32_t nblk,
                                               const T* __restrict__ x, T* __restrict__ recon,
                                               uint16_t* __restrict__ codes,
                                               T* __restrict__ staging,
                                               uint32_t* __restrict__ tile_cnt,
                                               uint32_t* __restrict__ tile_off,
                                               uint32_t* __restrict__ hist_total,
                                               uint32_t* __restrict__ hist_seg,
                                               StageAcc* __restrict__ acc,
                                               double* __restrict__ partials) {
    __shared__ uint32_t sh_hist[HBINS];
    for (int b = threadIdx.x; b < HBINS; b += THREADS) sh_hist[b] = 0;
    __syncthreads();
    const uint64_t items = d.n;
    const uint64_t groups = (items + ROW_GROUP - 1) / ROW_GROUP;
    const uint64_t g0 = (uint64_t)bid * gpb;
    const uint64_t g1 = g0 + gpb < groups ? g0 + gpb : groups;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    BlockAcc a{{0, 0, 0, 0, 0}, 0, 0};
    uint32_t cur_seg = (uint32_t)((g0 * ROW_GROUP) >> SEG_SHIFT);
    for (uint64_t g = g0; g < g1; g++) {
        const uint64_t base = g * ROW_GROUP;
        const uint32_t seg = (uint32_t)(base >> SEG_SHIFT);
        if (seg != cur_seg) {  // uniform across the CTA
            __syncthreads();
            flush_hist(sh_hist, hist_seg, cur_seg);
            __syncthreads();
            cur_seg = seg;
        }
        const uint64_t r0 = base + (uint64_t)warp * ROW_SEG;
        if (r0 >= items) continue;  // uniform across the warp
        RowSeg<ND, KIND> gs;
        uint32_t kb = 0;  // segment offset of the decoded point
        row_seg<ND, KIND>(d, q, (uint32_t)r0, gs);
#pragma unroll 1
        for (int j = 0; j < ROW_SEG / 32; j += 2) {
            if (32u * j - kb >= gs.rem && r0 + 32u * j < items) {  // the next row
                kb = 32u * j;
                row_seg<ND, KIND>(d, q, (uint32_t)(r0 + kb), gs);
            }
            const uint32_t k0 = 32 * j + lane, k1 = k0 + 32;
            const uint64_t i0 = r0 + k0, i1 = r0 + k1;
            const bool v0 = i0 < items, v1 = i1 < items;
            int64_t f0 = 0, f1 = 0;
            T x0 = (T)0, x1 = (T)0;
            PointTaps<T, ND, KIND> t0, t1;
            if (v0) {
                row_point<T, ND, KIND, CUBIC>(d, q, is_anchor, gs, k0 - kb, i0, recon, f0, t0);
                x0 = x[f0];
            }
            if (v1) {
                row_point<T, ND, KIND, CUBIC>(d, q, is_anchor, gs, k1 - kb, i1, recon, f1, t1);
                x1 = x[f1];
            }
            const double p0 = (v0 && !is_anchor) ? combine_point<T, ND, KIND, CUBIC>(q, t0) : 0.0;
            const double p1 = (v1 && !is_anchor) ? combine_point<T, ND, KIND, CUBIC>(q, t1) : 0.0;
            int k0h = -1, k1h = -1;
            uint32_t cd0 = 0, cd1 = 0;
            if (v0)
                encode_value<T>(q, i0, x0, p0, recon + f0, staging, tile_cnt, codes, a, k0h, cd0);
            if (v1)
                encode_value<T>(q, i1, x1, p1, recon + f1, staging, tile_cnt, codes, a, k1h, cd1);
            hist_warp(sh_hist, hist_total, k0h, cd0, lane);
            hist_warp(sh_hist, hist_total, k1h, cd1, lane);
        }
    }
    __syncthreads();
    flush_hist(sh_hist, hist_seg, cur_seg);
    block_finish(a, partials, acc, bid);
    if (last_block(acc, nblk)) stage_tail(partials, nblk, tile_cnt, n_tiles_of(items), tile_off, acc);
}

template <typename T, int ND, int KIND, int CUBIC>
__global__ void __launch_bounds__(THREADS, KIND ? 3 : 4)
    k_interp_quant_rows(const StageDesc d, const QParams q, const int is_anchor,
                        const uint32_t gpb, const T* __restrict__ x, T* __restrict__ recon,
                        uint16_t* __restrict__ codes, T* __restrict__ staging,
                        uint32_t* __restrict__ tile_cnt, uint32_t* __restrict__ tile_off,
                        uint32_t* __restrict__ hist_total, uint32_t* __restrict__ hist_seg,
                        StageAcc* __restrict__ acc, double* __restrict__ partials) {
    quant_rows_cta<T, ND, KIND, CUBIC>(d, q, is_anchor, gpb, blockIdx.x, gridDim.x, x, recon,
                                       codes, staging, tile_cnt, tile_off, hist_total, hist_seg,
                                       acc, partials);
}

template <typename T, int ND, int KIND, int CUBIC>
__global__ void __launch_bounds__(THREADS, KIND ? 3 : 4)
    k_interp_quant(const StageDesc d, const QParams q, const int is_anchor, const uint32_t gpb,
                   const T* __restrict__ x, T* __restrict__ recon, uint16_t* __restrict__ codes,
                   T* __restrict__ staging, uint32_t* __restrict__ tile_cnt,
                   uint32_t* __restrict__ tile_off, uint32_t* __restrict__ hist_total,
                   uint32_t* __restrict__ hist_seg, StageAcc* __restrict__ acc,
                   double* __restrict__ partials) {
    quant_cta<T, ND, KIND, CUBIC>(d, q, is_anchor, gpb, blockIdx.x, gridDim.x, x, recon, codes,
                                  staging, tile_cnt, tile_off, hist_total, hist_seg, acc,
                                  partials);
}

// Quantize a compact array against a given prediction (predictor-agnostic
// path: GNN and caller-supplied predictors). recon_out gets the decoder's
// reconstruction in the same compact order.
template <typename T>
__global__ void __launch_bounds__(THREADS)
    k_quantize_flat(const QParams q, const uint64_t items, const uint32_t gpb,
                    const T* __restrict__ x, const T* __restrict__ pred,
                    uint16_t* __restrict__ codes, T* __restrict__ staging,
                    uint32_t* __restrict__ tile_cnt, uint32_t* __restrict__ tile_off,
                    uint32_t* __restrict__ hist_total, uint32_t* __restrict__ hist_seg,
                    StageAcc* __restrict__ acc, double* __restrict__ partials,
                    T* __restrict__ recon_out) {
    __shared__ uint32_t sh_hist[HBINS];
    for (int b = threadIdx.x; b < HBINS; b += THREADS) sh_hist[b] = 0;
    __syncthreads();
    const uint64_t groups = (items + GROUP - 1) / GROUP;
    const uint64_t g0 = (uint64_t)blockIdx.x * gpb;
    const uint64_t g1 = g0 + gpb < groups ? g0 + gpb : groups;
    const int lane = threadIdx.x & 31;
    BlockAcc a{{0, 0, 0, 0, 0}, 0, 0};
    uint32_t cur_seg = (uint32_t)((g0 * GROUP) >> SEG_SHIFT);
    for (uint64_t g = g0; g < g1; g++) {
        const uint64_t base = g * GROUP;
        const uint32_t seg = (uint32_t)(base >> SEG_SHIFT);
        if (seg != cur_seg) {
            __syncthreads();
            flush_hist(sh_hist, hist_seg, cur_seg);
            __syncthreads();
            cur_seg = seg;
        }
        for (int h = 0; h < GROUP / THREADS; h++) {
            const uint64_t i = base + (uint64_t)h * THREADS + threadIdx.x;
            int key = -1;
            uint32_t code = 0;
            if (i < items)
                encode_value<T>(q, i, x[i], (double)pred[i], recon_out + i, staging, tile_cnt,
                                codes, a, key, code);
            hist_warp(sh_hist, hist_total, key, code, lane);
        }
    }
    __syncthreads();
    flush_hist(sh_hist, hist_seg, cur_seg);
    block_finish(a, partials, acc, blockIdx.x);
    if (last_block(acc, gridDim.x))
        stage_tail(partials, gridDim.x, tile_cnt, n_tiles_of(items), tile_off, acc);
}

// Prediction only (the predictor plugin's ``predict``): compact output.
template <typename T, int ND, int KIND, int CUBIC>
__global__ void __launch_bounds__(THREADS)
    k_interp_predict(const StageDesc d, const QParams q, const T* __restrict__ recon,
                     T* __restrict__ pred) {
    const uint64_t items = (uint64_t)q.channels * d.n;
    const uint64_t i = (uint64_t)blockIdx.x * THREADS + threadIdx.x;
    if (i >= items) return;
    uint32_t c = 0, rank = (uint32_t)i;
    if (q.channels > 1) {
        c = (uint32_t)(i / d.n);
        rank = (uint32_t)(i - (uint64_t)c * d.n);
    }
    int32_t coord[ND > 0 ? ND : MAXD];
    const int64_t flat = stage_point_t<ND, KIND>(d, rank, coord);
    pred[i] = (T)predict_point<T, ND, KIND, CUBIC>(d, q, recon + (uint64_t)c * q.points, flat,
                                                    coord);
}

// ---------------------------------------------------------------- scans
// Decode: zero codes (outliers) per 2048-code tile of every stage in one pass.
__global__ void __launch_bounds__(THREADS)
    k_count_zeros_all(const DecStage* __restrict__ ds, int n_stages,
                      uint32_t* __restrict__ tile_cnt) {
    const uint32_t gt = blockIdx.x;
    int lo = 0, hi = n_stages;  // last stage with tile0 <= gt
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (ds[mid].tile0 <= gt) lo = mid; else hi = mid;
    }
    const DecStage& d = ds[lo];
    const uint64_t base = (uint64_t)(gt - d.tile0) * TILE;
    int cnt = 0;
    for (int k = 0; k < TILE / THREADS; k++) {
        const uint64_t i = base + (uint64_t)k * THREADS + threadIdx.x;
        cnt += (i < d.items && d.codes[i] == 0) ? 1 : 0;
    }
    __shared__ int sh[THREADS / 32];
    int v = cnt;
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < THREADS / 32; w++) t += sh[w];
        tile_cnt[gt] = (uint32_t)t;
    }
}

// Decode: per stage (one CTA each) the exclusive tile offsets and the check
// that the stage's zero codes match its stored outlier count.
__global__ void __launch_bounds__(THREADS)
    k_tile_offsets_all(const DecStage* __restrict__ ds, const uint32_t* __restrict__ tile_cnt,
                       uint32_t* __restrict__ tile_off) {
    const DecStage& d = ds[blockIdx.x];
    const uint32_t tiles = n_tiles_of(d.items);
    if (!tiles) return;
    __shared__ uint32_t sc[THREADS];
    const uint32_t* cnt = tile_cnt + d.tile0;
    const uint32_t per = (tiles + THREADS - 1) / THREADS;
    const uint32_t a = threadIdx.x * per, e = min(tiles, a + per);
    uint32_t run = 0;
    for (uint32_t i = a; i < e; i++) run += cnt[i];
    sc[threadIdx.x] = run;
    __syncthreads();
    for (int o = 1; o < THREADS; o <<= 1) {
        const uint32_t v = threadIdx.x >= (unsigned)o ? sc[threadIdx.x - o] : 0u;
        __syncthreads();
        sc[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t off = sc[threadIdx.x] - run;
    for (uint32_t i = a; i < e; i++) {
        tile_off[d.tile0 + i] = off;
        off += cnt[i];
    }
    if (threadIdx.x == THREADS - 1 && sc[THREADS - 1] != d.n_out) atomicOr(d.err, 1u);
}

// Block-local exclusive scan of a per-thread flag in item order (k-major).
__device__ __forceinline__ uint32_t block_excl_flag(bool f, uint32_t& block_total) {
    __shared__ uint32_t sh_w[THREADS / 32];
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh_w[wid] = __popc(bal);
    __syncthreads();
    uint32_t before = 0, tot = 0;
    for (int w = 0; w < THREADS / 32; w++) {
        if (w < wid) before += sh_w[w];
        tot += sh_w[w];
    }
    __syncthreads();
    block_total = tot;
    return before + __popc(bal & ((1u << lane) - 1u));
}

// Outliers of a stage into scan order: tiles bid, bid + nblk, ... of the
// stage, each only if it counted an outlier.
__device__ __forceinline__ void compact_cta(const uint16_t* __restrict__ codes,
                                            const uint64_t items,
                                            const uint8_t* __restrict__ staging, const int elem,
                                            const uint32_t* __restrict__ tile_cnt,
                                            const uint32_t* __restrict__ tile_off,
                                            uint8_t* __restrict__ out, const uint32_t bid,
                                            const uint32_t nblk) {
    const uint32_t tiles = n_tiles_of(items);
    for (uint32_t tile = bid; tile < tiles; tile += nblk) {
        if (tile_cnt[tile] == 0) continue;  // uniform across the CTA
        const uint64_t tile_base = (uint64_t)tile * TILE;
        uint32_t run = tile_off[tile];
        for (int k = 0; k < TILE / THREADS; k++) {
            const uint64_t i = tile_base + (uint64_t)k * THREADS + threadIdx.x;
            const bool z = i < items && codes[i] == 0;
            uint32_t tot;
            const uint32_t pos = run + block_excl_flag(z, tot);
            if (z)
                for (int b = 0; b < elem; b++) out[(uint64_t)pos * elem + b] = staging[i * elem + b];
            run += tot;
        }
    }
}

__global__ void __launch_bounds__(THREADS)
    k_compact(const uint16_t* __restrict__ codes, const uint64_t items,
              const uint8_t* __restrict__ staging, const int elem,
              const uint32_t* __restrict__ tile_cnt, const uint32_t* __restrict__ tile_off,
              uint8_t* __restrict__ out) {
    compact_cta(codes, items, staging, elem, tile_cnt, tile_off, out, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- decode
template <typename T, int ND, int KIND, int CUBIC>
__device__ __forceinline__ void dequant_point(const StageDesc& d, const QParams& q,
                                              const int is_anchor, uint64_t i, uint32_t code,
                                              const uint8_t* __restrict__ outliers, uint32_t pos,
                                              uint32_t n_out, T* __restrict__ recon,
                                              uint32_t* __restrict__ err) {
    uint32_t c = 0, rank = (uint32_t)i;
    if (q.channels > 1) {
        c = (uint32_t)(i / d.n);
        rank = (uint32_t)(i - (uint64_t)c * d.n);
    }
    int32_t coord[ND > 0 ? ND : MAXD];
    const int64_t flat = stage_point_t<ND, KIND>(d, rank, coord);
    T* rc = recon + (uint64_t)c * q.points;
    T rv;
    if (code == 0) {
        if (pos < n_out) {
            rv = load_unaligned<T>(outliers + (uint64_t)pos * sizeof(T));
        } else {
            rv = (T)0;
            atomicOr(err, 1u);
        }
    } else {
        const double pd0 = is_anchor ? 0.0 : predict_point<T, ND, KIND, CUBIC>(d, q, rc, flat, coord);
        const double qv = (double)((int)code - q.radius);
        if (sizeof(T) == 4) {
            const double pd = (double)__double2float_rn(pd0);
            rv = (T)__double2float_rn(__dadd_rn(pd, __dmul_rn(q.w, qv)));
        } else {
            rv = (T)__dadd_rn(pd0, __dmul_rn(q.w, qv));
        }
    }
    rc[flat] = rv;
}

// Tiles without outliers (the common case) take a barrier-free path; others
// rank their outliers with a block scan in item order.
template <typename T, int ND, int KIND, int CUBIC>
__device__ __forceinline__ void dequant_cta(const StageDesc& d, const QParams& q,
                                            const int is_anchor, const uint32_t tile,
                                            const uint16_t* __restrict__ codes,
                                            const uint8_t* __restrict__ outliers,
                                            const uint32_t* __restrict__ tile_cnt,
                                            const uint32_t* __restrict__ tile_off,
                                            const uint32_t n_out, T* __restrict__ recon,
                                            uint32_t* __restrict__ err) {
    const uint64_t items = (uint64_t)q.channels * d.n;
    const uint64_t tile_base = (uint64_t)tile * TILE;
    if (tile_cnt[tile] == 0) {  // no outliers: two points in flight per thread
        for (int k = 0; k < TILE / THREADS; k += 2) {
            const uint64_t i0 = tile_base + (uint64_t)k * THREADS + threadIdx.x;
            const uint64_t i1 = i0 + THREADS;
            int64_t f0 = 0, f1 = 0;
            uint32_t c0 = 0, c1 = 0;
            uint32_t q0 = 1, q1 = 1;
            PointTaps<T, ND, KIND> t0, t1;
            if (i0 < items) {
                q0 = codes[i0];
                locate_gather<T, ND, KIND, CUBIC>(d, q, is_anchor, i0, recon, f0, c0, t0);
            }
            if (i1 < items) {
                q1 = codes[i1];
                locate_gather<T, ND, KIND, CUBIC>(d, q, is_anchor, i1, recon, f1, c1, t1);
            }
            const double p0 =
                (i0 < items && !is_anchor) ? combine_point<T, ND, KIND, CUBIC>(q, t0) : 0.0;
            const double p1 =
                (i1 < items && !is_anchor) ? combine_point<T, ND, KIND, CUBIC>(q, t1) : 0.0;
            if (i0 < items) recon[(uint64_t)c0 * q.points + f0] = dequant_value<T>(q, p0, q0);
            if (i1 < items) recon[(uint64_t)c1 * q.points + f1] = dequant_value<T>(q, p1, q1);
        }
        return;
    }
    uint32_t run = tile_off[tile];
    for (int k = 0; k < TILE / THREADS; k++) {
        const uint64_t i = tile_base + (uint64_t)k * THREADS + threadIdx.x;
        const bool valid = i < items;
        const uint32_t code = valid ? codes[i] : 1u;
        uint32_t tot;
        const uint32_t pos = run + block_excl_flag(code == 0, tot);
        run += tot;
        if (valid)
            dequant_point<T, ND, KIND, CUBIC>(d, q, is_anchor, i, code, outliers, pos, n_out, recon,
                                              err);
    }
}

template <typename T, int ND, int KIND, int CUBIC>
__global__ void __launch_bounds__(THREADS, KIND ? 4 : 5)
    k_interp_dequant(const StageDesc d, const QParams q, const int is_anchor,
                     const uint16_t* __restrict__ codes, const uint8_t* __restrict__ outliers,
                     const uint32_t* __restrict__ tile_cnt, const uint32_t* __restrict__ tile_off,
                     const uint32_t n_out, T* __restrict__ recon, uint32_t* __restrict__ err) {
    dequant_cta<T, ND, KIND, CUBIC>(d, q, is_anchor, blockIdx.x, codes, outliers, tile_cnt,
                                    tile_off, n_out, recon, err);
}

// Decode over row segments (single channel): a tile without outliers is
// eight warp segments of ROW_SEG consecutive ranks, each placed by one rank
// decode (see quant_rows_cta); a tile with outliers takes dequant_cta's path.
template <typename T, int ND, int KIND, int CUBIC>
__global__ void __launch_bounds__(THREADS, KIND ? 4 : 5)
    k_interp_dequant_rows(const StageDesc d, const QParams q, const int is_anchor,
                          const uint16_t* __restrict__ codes,
                          const uint8_t* __restrict__ outliers,
                          const uint32_t* __restrict__ tile_cnt,
                          const uint32_t* __restrict__ tile_off, const uint32_t n_out,
                          T* __restrict__ recon, uint32_t* __restrict__ err) {
    static_assert(TILE == ROW_SEG * THREADS / 32, "a tile is one segment per warp");
    if (tile_cnt[blockIdx.x] != 0) {
        dequant_cta<T, ND, KIND, CUBIC>(d, q, is_anchor, blockIdx.x, codes, outliers, tile_cnt,
                                        tile_off, n_out, recon, err);
        return;
    }
    const uint64_t items = d.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t r0 = (uint64_t)blockIdx.x * TILE + (uint64_t)warp * ROW_SEG;
    if (r0 >= items) return;
    RowSeg<ND, KIND> gs;
    uint32_t kb = 0;
    row_seg<ND, KIND>(d, q, (uint32_t)r0, gs);
#pragma unroll 1
    for (int j = 0; j < ROW_SEG / 32; j += 2) {
        if (32u * j - kb >= gs.rem && r0 + 32u * j < items) {
            kb = 32u * j;
            row_seg<ND, KIND>(d, q, (uint32_t)(r0 + kb), gs);
        }
        const uint32_t k0 = 32 * j + lane, k1 = k0 + 32;
        const uint64_t i0 = r0 + k0, i1 = r0 + k1;
        const bool v0 = i0 < items, v1 = i1 < items;
        int64_t f0 = 0, f1 = 0;
        uint32_t c0 = 1, c1 = 1;
        PointTaps<T, ND, KIND> t0, t1;
        if (v0) {
            c0 = codes[i0];
            row_point<T, ND, KIND, CUBIC>(d, q, is_anchor, gs, k0 - kb, i0, recon, f0, t0);
        }
        if (v1) {
            c1 = codes[i1];
            row_point<T, ND, KIND, CUBIC>(d, q, is_anchor, gs, k1 - kb, i1, recon, f1, t1);
        }
        const double p0 = (v0 && !is_anchor) ? combine_point<T, ND, KIND, CUBIC>(q, t0) : 0.0;
        const double p1 = (v1 && !is_anchor) ? combine_point<T, ND, KIND, CUBIC>(q, t1) : 0.0;
        if (v0) recon[f0] = dequant_value<T>(q, p0, c0);
        if (v1) recon[f1] = dequant_value<T>(q, p1, c1);
    }
}

// Predictor-agnostic decode of a compact array (the decode twin of
// k_quantize_flat): recon = outlier (scan order) where code == 0, else the
// quantizer's reconstruction of pred. One CTA per 2048-code tile.
template <typename T>
__global__ void __launch_bounds__(THREADS)
    k_dequant_flat(const QParams q, const uint64_t items, const T* __restrict__ pred,
                   const uint16_t* __restrict__ codes, const uint8_t* __restrict__ outliers,
                   const uint32_t* __restrict__ tile_cnt, const uint32_t* __restrict__ tile_off,
                   const uint32_t n_out, T* __restrict__ recon, uint32_t* __restrict__ err) {
    const uint64_t tile_base = (uint64_t)blockIdx.x * TILE;
    const bool any = tile_cnt[blockIdx.x] != 0;  // uniform across the CTA
    uint32_t run = any ? tile_off[blockIdx.x] : 0u;
    for (int k = 0; k < TILE / THREADS; k++) {
        const uint64_t i = tile_base + (uint64_t)k * THREADS + threadIdx.x;
        const bool valid = i < items;
        const uint32_t code = valid ? codes[i] : 1u;
        uint32_t pos = 0;
        if (any) {
            uint32_t tot;
            pos = run + block_excl_flag(code == 0, tot);
            run += tot;
        }
        if (!valid) continue;
        if (code == 0) {
            if (pos < n_out) {
                recon[i] = load_unaligned<T>(outliers + (uint64_t)pos * sizeof(T));
            } else {
                recon[i] = (T)0;
                atomicOr(err, 1u);
            }
        } else {
            recon[i] = dequant_value<T>(q, (double)pred[i], code);
        }
    }
}

// ---------------------------------------------------------------- many tensors
// A CTA of a many-tensor launch finds its job (the last one whose first CTA
// is not after it) and copies the job's stage descriptor into shared memory.
__device__ __forceinline__ uint32_t find_job(const uint32_t* __restrict__ first, uint32_t n,
                                             uint32_t b) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (first[mid] <= b) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t job_of_block(const uint32_t* __restrict__ first, uint32_t n) {
    __shared__ uint32_t sj;
    if (threadIdx.x == 0) sj = find_job(first, n, blockIdx.x);
    __syncthreads();
    return sj;
}

__device__ __forceinline__ void load_desc(StageDesc& sd, const StageDesc* __restrict__ g) {
    static_assert(sizeof(StageDesc) % 4 == 0, "descriptor copied as words");
    const uint32_t* src = reinterpret_cast<const uint32_t*>(g);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
    for (uint32_t k = threadIdx.x; k < sizeof(StageDesc) / 4; k += THREADS) dst[k] = src[k];
    __syncthreads();
}

template <typename T, int ND, int KIND, int CUBIC>
__global__ void __launch_bounds__(THREADS, KIND ? 3 : 4)
    k_interp_quant_many(const ManyJob* __restrict__ jobs, const uint32_t* __restrict__ first,
                        const uint32_t n) {
    __shared__ __align__(16) StageDesc sd;
    const uint32_t j = job_of_block(first, n);
    const ManyJob& J = jobs[j];
    load_desc(sd, J.d);
    quant_cta<T, ND, KIND, CUBIC>(sd, J.q, (int)J.is_anchor, J.gpb, blockIdx.x - first[j],
                                  J.blocks, (const T*)J.x, (T*)J.recon, J.codes, (T*)J.staging,
                                  J.tile_cnt, J.tile_off, J.hist_total, J.hist_seg, J.acc,
                                  J.partials);
}

template <typename T, int ND, int KIND, int CUBIC>
__global__ void __launch_bounds__(THREADS, KIND ? 4 : 5)
    k_interp_dequant_many(const ManyJob* __restrict__ jobs, const uint32_t* __restrict__ first,
                          const uint32_t n) {
    __shared__ __align__(16) StageDesc sd;
    const uint32_t j = job_of_block(first, n);
    const ManyJob& J = jobs[j];
    load_desc(sd, J.d);
    dequant_cta<T, ND, KIND, CUBIC>(sd, J.q, (int)J.is_anchor, blockIdx.x - first[j],
                                    J.codes_in, J.outliers, J.tile_cnt, J.tile_off, J.n_out,
                                    (T*)J.recon, J.err);
}

__global__ void __launch_bounds__(THREADS)
    k_compact_many(const ManyJob* __restrict__ jobs, const uint32_t* __restrict__ first,
                   const uint32_t n) {
    const uint32_t j = job_of_block(first, n);
    const ManyJob& J = jobs[j];
    compact_cta(J.codes, J.items, (const uint8_t*)J.staging, (int)J.elem, J.tile_cnt,
                J.tile_off, J.out, blockIdx.x - first[j], J.cblocks);
}

// Zero word ranges: range r takes CTAs first[r] .. first[r + 1] - 1, each
// clearing ZERO_CHUNK words of it.
__global__ void __launch_bounds__(THREADS)
    k_zero_many(const ZeroRange* __restrict__ r, const uint32_t* __restrict__ first,
                const uint32_t n) {
    const uint32_t j = job_of_block(first, n);
    const uint64_t a = (uint64_t)(blockIdx.x - first[j]) * ZERO_CHUNK;
    const uint64_t e = a + ZERO_CHUNK < r[j].words ? a + ZERO_CHUNK : r[j].words;
    uint32_t* p = r[j].p;
    for (uint64_t i = a + threadIdx.x; i < e; i += THREADS) p[i] = 0u;
}

// ---------------------------------------------------------------- fused levels
// Stage tails of a fused level encode: block s runs stage_tail for stage s.
__global__ void __launch_bounds__(THREADS) k_stage_tails(const TailArgs a) {
    const TailStage& t = a.s[blockIdx.x];
    stage_tail(t.partials, t.blocks, t.tile_cnt, t.tiles, t.tile_off, t.acc);
}

__device__ __forceinline__ int scatter_stage_of(const ScatterArgs& a, uint32_t g) {
    int s = 0;
    while (s + 1 < a.n && g >= a.s[s + 1].tile0) s++;
    return s;
}

// Outliers of the given stages into the canvas at their grid positions. A CTA
// takes 256 tiles at a time, lists those with outliers, then ranks each listed
// tile's outliers with a block scan in code order (their stored order).
template <typename T>
__global__ void __launch_bounds__(THREADS)
    k_scatter_outliers(const ScatterArgs a, const uint32_t total_tiles, T* __restrict__ recon,
                       uint32_t* __restrict__ err) {
    __shared__ uint32_t list[THREADS];
    for (uint32_t g0 = blockIdx.x * THREADS; g0 < total_tiles; g0 += gridDim.x * THREADS) {
        const uint32_t g = g0 + threadIdx.x;
        bool has = false;
        if (g < total_tiles) {
            const ScatterStage& S = a.s[scatter_stage_of(a, g)];
            has = S.tile_cnt[g - S.tile0] != 0;
        }
        uint32_t n_list;
        const uint32_t p = block_excl_flag(has, n_list);
        if (has) list[p] = g;
        __syncthreads();
        for (uint32_t k = 0; k < n_list; k++) {
            const uint32_t gt = list[k];
            const ScatterStage& S = a.s[scatter_stage_of(a, gt)];
            const uint32_t tile = gt - S.tile0;
            const uint64_t base = (uint64_t)tile * TILE;
            uint32_t run = S.tile_off[tile];
            for (int j = 0; j < TILE / THREADS; j++) {
                const uint64_t i = base + (uint64_t)j * THREADS + threadIdx.x;
                const bool z = i < S.items && S.codes[i] == 0;
                uint32_t tot;
                const uint32_t pos = run + block_excl_flag(z, tot);
                run += tot;
                if (!z) continue;
                uint32_t c = 0, rank = (uint32_t)i;
                if (a.channels > 1) {
                    c = (uint32_t)(i / S.d.n);
                    rank = (uint32_t)(i - (uint64_t)c * S.d.n);
                }
                int32_t coord[MAXD];
                const int64_t flat = stage_point(S.d, rank, coord);
                T v = (T)0;
                if (pos < S.n_out) {
                    v = load_unaligned<T>(S.outliers + (uint64_t)pos * sizeof(T));
                } else {
                    atomicOr(err, 1u);
                }
                recon[(uint64_t)c * a.points + flat] = v;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- level decode
// One 2048-code tile of a stage, as k_interp_dequant, with taps read through
// L2 (they may have been written by other CTAs of the same launch).
template <typename T, int ND, int KIND, int CUBIC, int COH>
__device__ __forceinline__ void dequant_tile_l2(const StageDesc& d, const QParams& q,
                                                uint32_t tile, const uint16_t* __restrict__ codes,
                                                const uint8_t* __restrict__ outliers,
                                                const uint32_t* __restrict__ tile_cnt,
                                                const uint32_t* __restrict__ tile_off,
                                                uint32_t n_out, T* __restrict__ recon,
                                                uint32_t* __restrict__ err) {
    const uint64_t items = (uint64_t)q.channels * d.n;
    const uint64_t tile_base = (uint64_t)tile * TILE;
    const bool any = tile_cnt[tile] != 0;  // uniform across the CTA
    uint32_t run = any ? tile_off[tile] : 0u;
    for (int k = 0; k < TILE / THREADS; k += 2) {
        const uint64_t i0 = tile_base + (uint64_t)k * THREADS + threadIdx.x;
        const uint64_t i1 = i0 + THREADS;
        const bool v0 = i0 < items, v1 = i1 < items;
        const uint32_t q0 = v0 ? codes[i0] : 1u, q1 = v1 ? codes[i1] : 1u;
        int64_t f0 = 0, f1 = 0;
        uint32_t c0 = 0, c1 = 0;
        PointTaps<T, ND, KIND> t0, t1;
        if (v0 && q0) locate_gather<T, ND, KIND, CUBIC, COH>(d, q, 0, i0, recon, f0, c0, t0);
        if (v1 && q1) locate_gather<T, ND, KIND, CUBIC, COH>(d, q, 0, i1, recon, f1, c1, t1);
        uint32_t p0 = 0, p1 = 0;
        if (any) {  // outlier positions in item order (k, then thread)
            uint32_t tot;
            p0 = run + block_excl_flag(v0 && q0 == 0, tot);
            run += tot;
            p1 = run + block_excl_flag(v1 && q1 == 0, tot);
            run += tot;
        }
        if (v0) {
            T v;
            if (q0) {
                v = dequant_value<T>(q, combine_point<T, ND, KIND, CUBIC>(q, t0), q0);
            } else {
                int32_t coord[ND > 0 ? ND : MAXD];
                uint32_t c = 0, rank = (uint32_t)i0;
                if (q.channels > 1) {
                    c = (uint32_t)(i0 / d.n);
                    rank = (uint32_t)(i0 - (uint64_t)c * d.n);
                }
                f0 = stage_point_t<ND, KIND>(d, rank, coord);
                c0 = c;
                if (p0 < n_out) {
                    v = load_unaligned<T>(outliers + (uint64_t)p0 * sizeof(T));
                } else {
                    v = (T)0;
                    atomicOr(err, 1u);
                }
            }
            recon[(uint64_t)c0 * q.points + f0] = v;
        }
        if (v1) {
            T v;
            if (q1) {
                v = dequant_value<T>(q, combine_point<T, ND, KIND, CUBIC>(q, t1), q1);
            } else {
                int32_t coord[ND > 0 ? ND : MAXD];
                uint32_t c = 0, rank = (uint32_t)i1;
                if (q.channels > 1) {
                    c = (uint32_t)(i1 / d.n);
                    rank = (uint32_t)(i1 - (uint64_t)c * d.n);
                }
                f1 = stage_point_t<ND, KIND>(d, rank, coord);
                c1 = c;
                if (p1 < n_out) {
                    v = load_unaligned<T>(outliers + (uint64_t)p1 * sizeof(T));
                } else {
                    v = (T)0;
                    atomicOr(err, 1u);
                }
            }
            recon[(uint64_t)c1 * q.points + f1] = v;
        }
    }
}

// Bounded wait of thread 0 for an item's dependencies; every later wait is
// skipped once one has run out (the error bit is set, results are invalid).
__device__ __forceinline__ void level_wait(const LvlBand& band, const LvlDep* __restrict__ deps,
                                           uint32_t* __restrict__ ctr, uint32_t* __restrict__ err) {
    for (uint32_t e = 0; e < band.dep_cnt; e++) {
        const LvlDep dp = deps[band.dep_off + e];
        const volatile uint32_t* c = ctr + 1 + dp.counter;
        uint32_t spins = 0;
        while (*c < dp.need) {
            if ((*(volatile uint32_t*)err & ERR_LEVEL_WAIT) || ++spins > LEVEL_WAIT_LIMIT) {
                atomicOr(err, ERR_LEVEL_WAIT);
                return;
            }
            __nanosleep(100);
        }
    }
    __threadfence();
}

template <typename T, int ND, int CUBIC>
__global__ void __launch_bounds__(THREADS, 3)
    k_level_dequant(const LvlStage* __restrict__ stages, const LvlBand* __restrict__ bands,
                    const LvlDep* __restrict__ deps, const LvlItem* __restrict__ items,
                    uint32_t n_items, uint32_t* __restrict__ ctr, T* __restrict__ recon,
                    uint32_t* __restrict__ err) {
    __shared__ StageDesc sd;
    __shared__ QParams sq;
    __shared__ uint32_t s_item;
    uint32_t cur = 0xffffffffu;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(&ctr[0], 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= n_items) break;
        const LvlItem item = items[it];
        const LvlBand band = bands[item.band];
        if (threadIdx.x == 0) level_wait(band, deps, ctr, err);
        if (band.stage != cur) {  // uniform: every thread saw the same item
            const uint32_t* src = (const uint32_t*)&stages[band.stage].d;
            uint32_t* dst = (uint32_t*)&sd;
            for (uint32_t w = threadIdx.x; w < sizeof(StageDesc) / 4; w += THREADS) dst[w] = src[w];
            if (threadIdx.x == 0) sq = stages[band.stage].q;
            cur = band.stage;
        }
        __syncthreads();
        const LvlStage& ls = stages[band.stage];
        for (uint32_t tile = item.tile0; tile < item.tile1; tile++) {
            // weight-1 sub-stages read only coarser levels (finished by earlier
            // launches): their taps may go through L1; the fused sub-stages
            // read this level's other sub-stages and must read through L2
            if (sd.kind == 1)
                dequant_tile_l2<T, ND, 1, CUBIC, 1>(sd, sq, tile, ls.codes, ls.outliers,
                                                    ls.tile_cnt, ls.tile_off, ls.n_out, recon, err);
            else if (sd.weight > 1)
                dequant_tile_l2<T, ND, 0, CUBIC, 1>(sd, sq, tile, ls.codes, ls.outliers,
                                                    ls.tile_cnt, ls.tile_off, ls.n_out, recon, err);
            else
                dequant_tile_l2<T, ND, 0, CUBIC, 0>(sd, sq, tile, ls.codes, ls.outliers,
                                                    ls.tile_cnt, ls.tile_off, ls.n_out, recon, err);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&ctr[1 + band.counter], 1u);
        }
    }
}

// ---------------------------------------------------------------- launchers
static int last_err() {
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

// Compile-time dispatch over (dtype, rank 2/3/4 or runtime, layout, order).
#define LATEC_DISPATCH(KERNEL_CALL)                                                      \
    do {                                                                                 \
        const int nd_ = (d.ndim >= 2 && d.ndim <= 4 && !d.holes && d.kind != 2) ? d.ndim : 0; \
        const int kd_ = d.kind == 1 ? 1 : 0, cu_ = q.order ? 1 : 0;                      \
        if (dtype == LATEC_F64) {                                                        \
            using T = double;                                                            \
            DISPATCH_ND(KERNEL_CALL);                                                    \
        } else {                                                                         \
            using T = float;                                                             \
            DISPATCH_ND(KERNEL_CALL);                                                    \
        }                                                                                \
    } while (0)
#define DISPATCH_ND(KERNEL_CALL)                                                         \
    switch (nd_) {                                                                       \
        case 2: DISPATCH_KC(2, KERNEL_CALL); break;                                      \
        case 3: DISPATCH_KC(3, KERNEL_CALL); break;                                      \
        case 4: DISPATCH_KC(4, KERNEL_CALL); break;                                      \
        default: DISPATCH_KC(0, KERNEL_CALL); break;                                     \
    }
#define DISPATCH_KC(NDC, KERNEL_CALL)                                                    \
    do {                                                                                 \
        if (kd_) {                                                                       \
            if (cu_) { constexpr int ND = NDC, KIND = 1, CUBIC = 1; KERNEL_CALL; }       \
            else { constexpr int ND = NDC, KIND = 1, CUBIC = 0; KERNEL_CALL; }           \
        } else {                                                                         \
            if (cu_) { constexpr int ND = NDC, KIND = 0, CUBIC = 1; KERNEL_CALL; }       \
            else { constexpr int ND = NDC, KIND = 0, CUBIC = 0; KERNEL_CALL; }           \
        }                                                                                \
    } while (0)

static uint32_t groups_per_block(uint64_t items, uint32_t* blocks) {
    const uint64_t groups = (items + GROUP - 1) / GROUP;
    if (groups == 0) {  // empty stage: no CTAs
        *blocks = 0;
        return 1;
    }
    uint64_t b = groups < (uint64_t)MAX_BLOCKS ? groups : (uint64_t)MAX_BLOCKS;
    if (b < 1) b = 1;
    const uint64_t gpb = (groups + b - 1) / b;
    *blocks = (uint32_t)((groups + gpb - 1) / gpb);
    return (uint32_t)gpb;
}

uint32_t encode_grid(uint64_t items, uint32_t cap, uint32_t* blocks) {
    const uint64_t groups = (items + GROUP - 1) / GROUP;
    if (groups == 0) {
        *blocks = 0;
        return 1;
    }
    const uint64_t c = cap ? cap : (uint64_t)MAX_BLOCKS;
    const uint64_t b = groups < c ? groups : c;
    const uint64_t gpb = (groups + b - 1) / b;
    *blocks = (uint32_t)((groups + gpb - 1) / gpb);
    return (uint32_t)gpb;
}

uint32_t encode_blocks(uint64_t items) {
    uint32_t b;
    groups_per_block(items, &b);
    return b;
}

std::atomic<int> g_row_mode{1};

// Row-segment kernels: one channel, rank 2..4 without blocked anchors, 32-bit
// tap offsets, and rows long enough that a warp segment stays in one row.
bool rows_ok(const StageDesc& d, const QParams& q) {
    if (!g_row_mode.load() || q.channels != 1 || d.holes || d.kind != 0 || d.ndim < 2 ||
        d.ndim > 4 || q.points >= (1ull << 30) || d.gstride[d.ndim - 1] != 1)
        return false;
    const int X = d.ndim - 1;
    const uint32_t len = d.kind == 0 ? d.size_div[X].d
                                     : (uint32_t)((d.shape[X] + 2 * d.s - 1) / (2 * d.s));
    return len >= (uint32_t)ROW_SEG / 2;
}

#define ROWS_DISPATCH(KERNEL_CALL)                                                      \
    do {                                                                                \
        const int kd_ = d.kind == 1 ? 1 : 0, cu_ = q.order ? 1 : 0;                     \
        if (dtype == LATEC_F64) {                                                       \
            using T = double;                                                           \
            ROWS_ND(KERNEL_CALL);                                                       \
        } else {                                                                        \
            using T = float;                                                            \
            ROWS_ND(KERNEL_CALL);                                                       \
        }                                                                               \
    } while (0)
#define ROWS_ND(KERNEL_CALL)                                                            \
    switch (d.ndim) {                                                                   \
        case 2: DISPATCH_KC(2, KERNEL_CALL); break;                                     \
        case 3: DISPATCH_KC(3, KERNEL_CALL); break;                                     \
        default: DISPATCH_KC(4, KERNEL_CALL); break;                                    \
    }

int launch_interp_quant(const StageDesc& d, const QParams& q, int dtype, int is_anchor,
                        const void* x, void* recon, uint16_t* codes, void* staging,
                        uint32_t* tile_cnt, uint32_t* tile_off, uint32_t* hist_total,
                        uint32_t* hist_seg, StageAcc* acc, double* partials, cudaStream_t st) {
    const uint64_t items = (uint64_t)q.channels * d.n;
    if (!items) return LATEC_OK;
    if (cudaMemsetAsync(tile_cnt, 0, sizeof(uint32_t) * n_tiles(items), st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    if (rows_ok(d, q)) {
        const uint64_t groups = (items + ROW_GROUP - 1) / ROW_GROUP;
        const uint64_t b = groups < (uint64_t)MAX_BLOCKS ? groups : (uint64_t)MAX_BLOCKS;
        const uint32_t gpb = (uint32_t)((groups + b - 1) / b);
        const uint32_t blocks = (uint32_t)((groups + gpb - 1) / gpb);
        ROWS_DISPATCH((k_interp_quant_rows<T, ND, KIND, CUBIC><<<blocks, THREADS, 0, st>>>(
            d, q, is_anchor, gpb, (const T*)x, (T*)recon, codes, (T*)staging, tile_cnt,
            tile_off, hist_total, hist_seg, acc, partials)));
        return last_err();
    }
    uint32_t blocks;
    const uint32_t gpb = groups_per_block(items, &blocks);
    LATEC_DISPATCH((k_interp_quant<T, ND, KIND, CUBIC><<<blocks, THREADS, 0, st>>>(
        d, q, is_anchor, gpb, (const T*)x, (T*)recon, codes, (T*)staging, tile_cnt, tile_off,
        hist_total, hist_seg, acc, partials)));
    return last_err();
}

int launch_quantize_flat(const QParams& q, int dtype, uint64_t items, const void* x,
                         const void* pred, uint16_t* codes, void* staging, uint32_t* tile_cnt,
                         uint32_t* tile_off, uint32_t* hist_total, uint32_t* hist_seg,
                         StageAcc* acc, double* partials, void* recon_out, cudaStream_t st) {
    if (!items) return LATEC_OK;
    uint32_t blocks;
    const uint32_t gpb = groups_per_block(items, &blocks);
    if (cudaMemsetAsync(tile_cnt, 0, sizeof(uint32_t) * n_tiles(items), st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    if (dtype == LATEC_F64)
        k_quantize_flat<double><<<blocks, THREADS, 0, st>>>(
            q, items, gpb, (const double*)x, (const double*)pred, codes, (double*)staging,
            tile_cnt, tile_off, hist_total, hist_seg, acc, partials, (double*)recon_out);
    else
        k_quantize_flat<float><<<blocks, THREADS, 0, st>>>(
            q, items, gpb, (const float*)x, (const float*)pred, codes, (float*)staging, tile_cnt,
            tile_off, hist_total, hist_seg, acc, partials, (float*)recon_out);
    return last_err();
}

int launch_interp_predict(const StageDesc& d, const QParams& q, int dtype, const void* recon,
                          void* pred, cudaStream_t st) {
    const uint64_t items = (uint64_t)q.channels * d.n;
    if (!items) return LATEC_OK;
    const uint32_t blocks = (uint32_t)((items + THREADS - 1) / THREADS);
    LATEC_DISPATCH((k_interp_predict<T, ND, KIND, CUBIC><<<blocks, THREADS, 0, st>>>(
        d, q, (const T*)recon, (T*)pred)));
    return last_err();
}

int launch_count_zeros_all(const DecStage* ds, int n_stages, uint32_t total_tiles,
                           uint32_t* tile_cnt, cudaStream_t st) {
    if (!total_tiles) return LATEC_OK;
    k_count_zeros_all<<<total_tiles, THREADS, 0, st>>>(ds, n_stages, tile_cnt);
    return last_err();
}

int launch_tile_offsets_all(const DecStage* ds, int n_stages, const uint32_t* tile_cnt,
                            uint32_t* tile_off, cudaStream_t st) {
    if (!n_stages) return LATEC_OK;
    k_tile_offsets_all<<<n_stages, THREADS, 0, st>>>(ds, tile_cnt, tile_off);
    return last_err();
}

int launch_dequant_flat(const QParams& q, int dtype, uint64_t items, const void* pred,
                        const uint16_t* codes, const void* outliers, const uint32_t* tile_cnt,
                        const uint32_t* tile_off, uint32_t n_out, void* recon, uint32_t* err,
                        cudaStream_t st) {
    if (!items) return LATEC_OK;
    if (dtype == LATEC_F64)
        k_dequant_flat<double><<<n_tiles(items), THREADS, 0, st>>>(
            q, items, (const double*)pred, codes, (const uint8_t*)outliers, tile_cnt, tile_off,
            n_out, (double*)recon, err);
    else
        k_dequant_flat<float><<<n_tiles(items), THREADS, 0, st>>>(
            q, items, (const float*)pred, codes, (const uint8_t*)outliers, tile_cnt, tile_off,
            n_out, (float*)recon, err);
    return last_err();
}

int launch_level_dequant(int dtype, int nd, int cubic, const LvlStage* stages,
                         const LvlBand* bands, const LvlDep* deps, const LvlItem* items,
                         uint32_t n_items, uint32_t* ctr, void* recon, uint32_t* err,
                         cudaStream_t st) {
    if (!n_items) return LATEC_OK;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t want = (uint32_t)sms * 3;  // resident CTAs (launch bounds)
    const uint32_t grid = n_items < want ? n_items : want;
#define LVL_DQ(TT, NDC, CU)                                                                     \
    k_level_dequant<TT, NDC, CU><<<grid, THREADS, 0, st>>>(stages, bands, deps, items, n_items, \
                                                           ctr, (TT*)recon, err)
#define LVL_DQ_ND(TT)                                                                           \
    do {                                                                                        \
        if (nd == 2) { if (cubic) LVL_DQ(TT, 2, 1); else LVL_DQ(TT, 2, 0); }                    \
        else if (nd == 3) { if (cubic) LVL_DQ(TT, 3, 1); else LVL_DQ(TT, 3, 0); }               \
        else if (nd == 4) { if (cubic) LVL_DQ(TT, 4, 1); else LVL_DQ(TT, 4, 0); }               \
        else { if (cubic) LVL_DQ(TT, 0, 1); else LVL_DQ(TT, 0, 0); }                            \
    } while (0)
    if (dtype == LATEC_F64) LVL_DQ_ND(double);
    else LVL_DQ_ND(float);
#undef LVL_DQ_ND
#undef LVL_DQ
    return last_err();
}

int launch_compact(const uint16_t* codes, uint64_t items, const void* staging, int elem,
                   const uint32_t* tile_cnt, const uint32_t* tile_off, void* out,
                   cudaStream_t st) {
    if (!items) return LATEC_OK;
    const uint32_t tiles = n_tiles(items);
    k_compact<<<tiles < 592u ? tiles : 592u, THREADS, 0, st>>>(
        codes, items, (const uint8_t*)staging, elem, tile_cnt, tile_off, (uint8_t*)out);
    return last_err();
}

int launch_interp_dequant(const StageDesc& d, const QParams& q, int dtype, int is_anchor,
                          const uint16_t* codes, const void* outliers, const uint32_t* tile_cnt,
                          const uint32_t* tile_off, uint32_t n_out, void* recon, uint32_t* err,
                          cudaStream_t st) {
    const uint64_t items = (uint64_t)q.channels * d.n;
    if (!items) return LATEC_OK;
    if (rows_ok(d, q)) {
        ROWS_DISPATCH((k_interp_dequant_rows<T, ND, KIND, CUBIC><<<n_tiles(items), THREADS, 0,
                                                                   st>>>(
            d, q, is_anchor, codes, (const uint8_t*)outliers, tile_cnt, tile_off, n_out,
            (T*)recon, err)));
        return last_err();
    }
    LATEC_DISPATCH((k_interp_dequant<T, ND, KIND, CUBIC><<<n_tiles(items), THREADS, 0, st>>>(
        d, q, is_anchor, codes, (const uint8_t*)outliers, tile_cnt, tile_off, n_out, (T*)recon,
        err)));
    return last_err();
}


#define MANY_DISPATCH(KERNEL_CALL)                                                      \
    do {                                                                                \
        const int nd_ = nd, kd_ = kind, cu_ = cubic;                                    \
        if (dtype == LATEC_F64) {                                                       \
            using T = double;                                                           \
            DISPATCH_ND(KERNEL_CALL);                                                   \
        } else {                                                                        \
            using T = float;                                                            \
            DISPATCH_ND(KERNEL_CALL);                                                   \
        }                                                                               \
    } while (0)

int launch_quant_many(int dtype, int nd, int kind, int cubic, const ManyJob* jobs,
                      const uint32_t* first, uint32_t n_jobs, uint32_t ctas, cudaStream_t st) {
    if (!n_jobs || !ctas) return LATEC_OK;
    MANY_DISPATCH((k_interp_quant_many<T, ND, KIND, CUBIC><<<ctas, THREADS, 0, st>>>(
        jobs, first, n_jobs)));
    return last_err();
}

int launch_dequant_many(int dtype, int nd, int kind, int cubic, const ManyJob* jobs,
                        const uint32_t* first, uint32_t n_jobs, uint32_t ctas, cudaStream_t st) {
    if (!n_jobs || !ctas) return LATEC_OK;
    MANY_DISPATCH((k_interp_dequant_many<T, ND, KIND, CUBIC><<<ctas, THREADS, 0, st>>>(
        jobs, first, n_jobs)));
    return last_err();
}

int launch_compact_many(const ManyJob* jobs, const uint32_t* first, uint32_t n_jobs,
                        uint32_t ctas, cudaStream_t st) {
    if (!n_jobs || !ctas) return LATEC_OK;
    k_compact_many<<<ctas, THREADS, 0, st>>>(jobs, first, n_jobs);
    return last_err();
}

int launch_zero_many(const ZeroRange* r, const uint32_t* first, uint32_t n, uint32_t ctas,
                     cudaStream_t st) {
    if (!n || !ctas) return LATEC_OK;
    k_zero_many<<<ctas, THREADS, 0, st>>>(r, first, n);
    return last_err();
}

int launch_stage_tails(const TailArgs& a, int n, cudaStream_t st) {
    if (n <= 0) return LATEC_OK;
    k_stage_tails<<<n, THREADS, 0, st>>>(a);
    return last_err();
}

int launch_scatter_outliers(const ScatterArgs& a, int dtype, uint32_t total_tiles, void* recon,
                            uint32_t* err, cudaStream_t st) {
    if (!total_tiles || a.n <= 0) return LATEC_OK;
    uint32_t blocks = (total_tiles + THREADS - 1) / THREADS;
    if (blocks > 148 * 4) blocks = 148 * 4;
    if (dtype == LATEC_F64)
        k_scatter_outliers<double><<<blocks, THREADS, 0, st>>>(a, total_tiles, (double*)recon, err);
    else
        k_scatter_outliers<float><<<blocks, THREADS, 0, st>>>(a, total_tiles, (float*)recon, err);
    return last_err();
}

}  // namespace latec
