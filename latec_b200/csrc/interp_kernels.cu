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
#include <cuda_runtime.h>

#include "interp_kernels.cuh"

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

// ---- gather / combine form of predict_point, used by the stage kernels ----
// All taps a point needs are loaded first, without branches (a tap outside
// the line reads the -s tap, which always exists, and is then ignored), so a
// thread has every load of its points in flight before any arithmetic; the
// combine step is axis_interp's arithmetic, operation for operation.
template <typename T>
struct AxisTaps {
    T m1, p1, m3, p3;
    uint32_t ok;  // bit 0: +s valid, bit 1: -3s valid, bit 2: +3s valid
};

// Tap load: the read-only cache path, or (COH) L2 only, for taps that other
// CTAs of the same launch may have written (the level kernels).
template <typename T, int COH>
__device__ __forceinline__ T ldtap(const T* p) {
    if (COH) return __ldcg(p);
    return __ldg(p);
}

template <typename T, int CUBIC, int COH = 0>
__device__ __forceinline__ void load_axis(const T* __restrict__ rc, int64_t flat, int c, int n,
                                          int64_t gs, int s, AxisTaps<T>& t) {
    const int64_t o1 = (int64_t)s * gs;
    const bool vp1 = c + s < n, vm3 = c - 3 * s >= 0, vp3 = c + 3 * s < n;
    const T* b = rc + flat;
    t.m1 = ldtap<T, COH>(b - o1);
    t.p1 = ldtap<T, COH>(b + (vp1 ? o1 : -o1));
    t.m3 = ldtap<T, COH>(b + (vm3 ? -3 * o1 : -o1));
    t.p3 = CUBIC ? ldtap<T, COH>(b + (vp3 ? 3 * o1 : -o1)) : (T)0;
    t.ok = (vp1 ? 1u : 0u) | (vm3 ? 2u : 0u) | (vp3 ? 4u : 0u);
}

template <typename T, int CUBIC>
__device__ __forceinline__ double axis_combine(const AxisTaps<T>& t, int em) {
    const double Lm1 = (double)t.m1;
    const bool vp1 = t.ok & 1u, vm3 = t.ok & 2u, vp3 = t.ok & 4u;
    if (vp1) {
        const double Lp1 = (double)t.p1;
        const double lin = 0.5 * __dadd_rn(Lm1, Lp1);
        if (!CUBIC) return lin;
        if (vm3 && vp3) {
            const double Lm3 = (double)t.m3, Lp3 = (double)t.p3;
            double u = __dadd_rn(-Lm3, __dmul_rn(9.0, Lm1));
            u = __dadd_rn(u, __dmul_rn(9.0, Lp1));
            u = __dsub_rn(u, Lp3);
            return u * 0.0625;
        }
        if (em & 1) {
            if (vp3) {
                const double Lp3 = (double)t.p3;
                double u = __dadd_rn(__dmul_rn(3.0, Lm1), __dmul_rn(6.0, Lp1));
                u = __dsub_rn(u, Lp3);
                return u * 0.125;
            }
            if (vm3) {
                const double Lm3 = (double)t.m3;
                double u = __dadd_rn(-Lm3, __dmul_rn(6.0, Lm1));
                u = __dadd_rn(u, __dmul_rn(3.0, Lp1));
                return u * 0.125;
            }
        }
        return lin;
    }
    if ((em & 2) && vm3) return __dsub_rn(__dmul_rn(1.5, Lm1), __dmul_rn(0.5, (double)t.m3));
    return Lm1;
}

// Taps of one point: one axis for KIND 0 and for centers 1/2, every odd axis
// for KIND 1 with center 0 (in axis order).
template <typename T, int ND, int KIND>
struct PointTaps {
    static constexpr int NA = KIND ? (ND > 0 ? ND : MAXD) : 1;
    AxisTaps<T> ax[NA];
    uint32_t odd;  // center 0, KIND 1: mask of the odd axes
};

template <typename T, int ND, int KIND, int CUBIC, int COH = 0>
__device__ __forceinline__ void gather_point(const StageDesc& d, const QParams& q,
                                             const T* __restrict__ rc, int64_t flat,
                                             const int32_t* coord, PointTaps<T, ND, KIND>& pt) {
    constexpr int NDV = ND > 0 ? ND : MAXD;
    pt.odd = 0;
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
        load_axis<T, CUBIC, COH>(rc, flat, ca, na, gs, d.s, pt.ax[0]);
        return;
    }
    if (q.center == 0) {
#pragma unroll
        for (int j = 0; j < NDV; j++) {
            if ((ND > 0 || j < d.ndim) && (coord[j] & d.s)) {
                pt.odd |= 1u << j;
                load_axis<T, CUBIC, COH>(rc, flat, coord[j], d.shape[j], d.gstride[j], d.s,
                                    pt.ax[KIND ? j : 0]);
            }
        }
        return;
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
    load_axis<T, CUBIC, COH>(rc, flat, ca, na, gs, d.s, pt.ax[0]);
}

template <typename T, int ND, int KIND, int CUBIC>
__device__ __forceinline__ double combine_point(const QParams& q, const PointTaps<T, ND, KIND>& pt) {
    constexpr int NDV = ND > 0 ? ND : MAXD;
    if (KIND == 0 || q.center != 0) return axis_combine<T, CUBIC>(pt.ax[0], q.end_mode);
    double total = 0.0;
    int cnt = 0;
#pragma unroll
    for (int j = 0; j < NDV; j++) {
        if (pt.odd & (1u << j)) {
            const double v = axis_combine<T, CUBIC>(pt.ax[KIND ? j : 0], q.end_mode);
            total = cnt ? __dadd_rn(total, v) : v;
            cnt++;
        }
    }
    if (cnt == 1) return total;
    if (cnt == 2) return total * 0.5;
    if (cnt == 4) return total * 0.25;
    return __ddiv_rn(total, (double)cnt);
}

// rint((x - p) / w) with the division's exact rounding: the reciprocal
// product is used unless it lies within a few ulps of a half-integer.
__device__ __forceinline__ double quotient_rint(double diff, const QParams& q) {
    if (q.inv_w != 0.0) {
        const double a = __dmul_rn(diff, q.inv_w);
        const double r = rint(a);
        const double frac = fabs(__dsub_rn(a, r));
        const double tol = fabs(a) * 0x1p-48 + 0x1p-1000;
        if (!(fabs(frac - 0.5) <= tol)) return r;  // NaN/inf fall through unchanged
    }
    return rint(__ddiv_rn(diff, q.w));
}

struct QOut {
    uint32_t code;  // 0 = outlier
    int32_t qv;     // bin index when in range
};

// Quantize one value (float32 source). Returns the code and writes the
// reconstruction the decoder will produce.
__device__ __forceinline__ QOut quant_f32(float x, double pd, const QParams& q, float& rv) {
    const double qd = quotient_rint(__dsub_rn((double)x, pd), q);
    QOut o{0u, 0};
    rv = x;
    if (fabs(qd) < (double)q.radius) {
        const int qi = (int)qd;
        const float rf = __double2float_rn(__dadd_rn(pd, __dmul_rn(q.w, (double)qi)));
        const float chk = q.round_output ? rintf(rf) : rf;
        if (fabsf(__fsub_rn(x, chk)) <= q.eb_f) {
            o.code = (uint32_t)(qi + q.radius);
            o.qv = qi;
            rv = rf;
        }
    }
    return o;
}

// float64 source: prediction, reconstruction and bound check stay float64.
__device__ __forceinline__ QOut quant_f64(double x, double pd, const QParams& q, double& rv) {
    const double qd = quotient_rint(__dsub_rn(x, pd), q);
    QOut o{0u, 0};
    rv = x;
    if (fabs(qd) < (double)q.radius) {
        const int qi = (int)qd;
        double rd = __dadd_rn(pd, __dmul_rn(q.w, (double)qi));
        const double chk = q.round_output ? rint(rd) : rd;
        if (fabs(__dsub_rn(x, chk)) <= q.eb) {
            o.code = (uint32_t)(qi + q.radius);
            o.qv = qi;
            rv = rd;
        }
    }
    return o;
}

template <typename T>
struct Quant;
template <>
struct Quant<float> {
    __device__ static QOut run(float x, double pd, const QParams& q, float& rv) {
        return quant_f32(x, (double)__double2float_rn(pd), q, rv);
    }
    __device__ static double err(float x, double pd) {  // f32 residual, like the reference stats
        return (double)__fsub_rn(x, __double2float_rn(pd));
    }
    __device__ static double rerr(float x, float rv) { return (double)fabsf(__fsub_rn(x, rv)); }
};
template <>
struct Quant<double> {
    __device__ static QOut run(double x, double pd, const QParams& q, double& rv) {
        return quant_f64(x, pd, q, rv);
    }
    __device__ static double err(double x, double pd) { return __dsub_rn(x, pd); }
    __device__ static double rerr(double x, double rv) { return fabs(__dsub_rn(x, rv)); }
};

// Block-wide reduction helpers -------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ uint32_t warp_umax(uint32_t v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

struct BlockAcc {
    double s[5];
    uint32_t maxq;
    uint32_t nout;
};

// Per-block statistics: warp shuffles, then one partial row per CTA.
__device__ __forceinline__ void block_finish(BlockAcc& a, double* partials, StageAcc* acc) {
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
        for (int k = 0; k < 5; k++) partials[(size_t)blockIdx.x * 5 + k] = s[k];
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

// Arrival counter: true in the CTA that finishes the stage.
__device__ __forceinline__ bool last_block(StageAcc* acc) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(&acc->done, 1u) == gridDim.x - 1;
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
    flat = stage_coords_t<ND, KIND>(d, rank, coord);
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
    flat = stage_coords_t<ND, KIND>(d, rank, coord);
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

__device__ __forceinline__ void hist_warp(uint32_t* sh_hist, uint32_t* hist_total, int key,
                                          uint32_t code, int lane) {
    const unsigned same = __match_any_sync(0xffffffffu, key);
    if (key >= 0 && lane == __ffs(same) - 1) atomicAdd(&sh_hist[key], (uint32_t)__popc(same));
    if (key == -2) atomicAdd(&hist_total[code], 1u);
}

__device__ __forceinline__ void flush_hist(uint32_t* sh_hist, uint32_t* hist_seg, uint32_t seg) {
    for (int b = threadIdx.x; b < HBINS; b += THREADS) {
        const uint32_t v = sh_hist[b];
        if (v) {
            atomicAdd(&hist_seg[(size_t)seg * HBINS + b], v);
            sh_hist[b] = 0;
        }
    }
}

template <typename T, int ND, int KIND, int CUBIC>
__global__ void __launch_bounds__(THREADS, KIND ? 3 : 4)
    k_interp_quant(const StageDesc d, const QParams q, const int is_anchor, const uint32_t gpb,
                   const T* __restrict__ x, T* __restrict__ recon, uint16_t* __restrict__ codes,
                   T* __restrict__ staging, uint32_t* __restrict__ tile_cnt,
                   uint32_t* __restrict__ tile_off, uint32_t* __restrict__ hist_total,
                   uint32_t* __restrict__ hist_seg, StageAcc* __restrict__ acc,
                   double* __restrict__ partials) {
    __shared__ uint32_t sh_hist[HBINS];
    for (int b = threadIdx.x; b < HBINS; b += THREADS) sh_hist[b] = 0;
    __syncthreads();
    const uint64_t items = (uint64_t)q.channels * d.n;
    const uint64_t groups = (items + GROUP - 1) / GROUP;
    const uint64_t g0 = (uint64_t)blockIdx.x * gpb;
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
    block_finish(a, partials, acc);
    if (last_block(acc)) stage_tail(partials, gridDim.x, tile_cnt, n_tiles_of(items), tile_off, acc);
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
    block_finish(a, partials, acc);
    if (last_block(acc)) stage_tail(partials, gridDim.x, tile_cnt, n_tiles_of(items), tile_off, acc);
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
    const int64_t flat = stage_coords_t<ND, KIND>(d, rank, coord);
    pred[i] = (T)predict_point<T, ND, KIND, CUBIC>(d, q, recon + (uint64_t)c * q.points, flat,
                                                    coord);
}

// ---------------------------------------------------------------- scans
// Decode: zero codes (outliers) per 2048-code tile of every stage in one pass.
__global__ void __launch_bounds__(THREADS)
    k_count_zeros_all(const DecStage* __restrict__ ds, int n_stages, const uint16_t* __restrict__ codes,
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
        cnt += (i < d.items && codes[d.codes_off + i] == 0) ? 1 : 0;
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
                       uint32_t* __restrict__ tile_off, uint32_t* __restrict__ err) {
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
    if (threadIdx.x == THREADS - 1 && sc[THREADS - 1] != d.n_out) atomicOr(err, 1u);
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

__global__ void __launch_bounds__(THREADS)
    k_compact(const uint16_t* __restrict__ codes, const uint64_t items,
              const uint8_t* __restrict__ staging, const int elem,
              const uint32_t* __restrict__ tile_cnt, const uint32_t* __restrict__ tile_off,
              uint8_t* __restrict__ out) {
    const uint32_t tiles = n_tiles_of(items);
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
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

// ---------------------------------------------------------------- decode
template <typename T>
__device__ __forceinline__ T load_unaligned(const uint8_t* p) {
    uint8_t b[sizeof(T)];
#pragma unroll
    for (int k = 0; k < (int)sizeof(T); k++) b[k] = p[k];
    T v;
    memcpy(&v, b, sizeof(T));
    return v;
}

template <typename T>
__device__ __forceinline__ T dequant_value(const QParams& q, double pd0, uint32_t code) {
    const double qv = (double)((int)code - q.radius);
    if (sizeof(T) == 4) {
        const double pd = (double)__double2float_rn(pd0);
        return (T)__double2float_rn(__dadd_rn(pd, __dmul_rn(q.w, qv)));
    }
    return (T)__dadd_rn(pd0, __dmul_rn(q.w, qv));
}

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
    const int64_t flat = stage_coords_t<ND, KIND>(d, rank, coord);
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
__global__ void __launch_bounds__(THREADS, KIND ? 4 : 5)
    k_interp_dequant(const StageDesc d, const QParams q, const int is_anchor,
                     const uint16_t* __restrict__ codes, const uint8_t* __restrict__ outliers,
                     const uint32_t* __restrict__ tile_cnt, const uint32_t* __restrict__ tile_off,
                     const uint32_t n_out, T* __restrict__ recon, uint32_t* __restrict__ err) {
    const uint64_t items = (uint64_t)q.channels * d.n;
    const uint64_t tile_base = (uint64_t)blockIdx.x * TILE;
    if (tile_cnt[blockIdx.x] == 0) {  // no outliers: two points in flight per thread
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
    uint32_t run = tile_off[blockIdx.x];
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
                f0 = stage_coords_t<ND, KIND>(d, rank, coord);
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
                f1 = stage_coords_t<ND, KIND>(d, rank, coord);
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
            if (sd.kind)
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
        const int nd_ = (d.ndim >= 2 && d.ndim <= 4) ? d.ndim : 0;                      \
        const int kd_ = d.kind ? 1 : 0, cu_ = q.order ? 1 : 0;                           \
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

uint32_t encode_blocks(uint64_t items) {
    uint32_t b;
    groups_per_block(items, &b);
    return b;
}

int launch_interp_quant(const StageDesc& d, const QParams& q, int dtype, int is_anchor,
                        const void* x, void* recon, uint16_t* codes, void* staging,
                        uint32_t* tile_cnt, uint32_t* tile_off, uint32_t* hist_total,
                        uint32_t* hist_seg, StageAcc* acc, double* partials, cudaStream_t st) {
    const uint64_t items = (uint64_t)q.channels * d.n;
    if (!items) return LATEC_OK;
    uint32_t blocks;
    const uint32_t gpb = groups_per_block(items, &blocks);
    if (cudaMemsetAsync(tile_cnt, 0, sizeof(uint32_t) * n_tiles(items), st) != cudaSuccess)
        return LATEC_ERR_CUDA;
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
                           const uint16_t* codes, uint32_t* tile_cnt, cudaStream_t st) {
    if (!total_tiles) return LATEC_OK;
    k_count_zeros_all<<<total_tiles, THREADS, 0, st>>>(ds, n_stages, codes, tile_cnt);
    return last_err();
}

int launch_tile_offsets_all(const DecStage* ds, int n_stages, const uint32_t* tile_cnt,
                            uint32_t* tile_off, uint32_t* err, cudaStream_t st) {
    if (!n_stages) return LATEC_OK;
    k_tile_offsets_all<<<n_stages, THREADS, 0, st>>>(ds, tile_cnt, tile_off, err);
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
    LATEC_DISPATCH((k_interp_dequant<T, ND, KIND, CUBIC><<<n_tiles(items), THREADS, 0, st>>>(
        d, q, is_anchor, codes, (const uint8_t*)outliers, tile_cnt, tile_off, n_out, (T*)recon,
        err)));
    return last_err();
}

}  // namespace latec
