// Device helpers shared by the stage kernels (interp_kernels.cu) and the
// fused finest-level tile kernels (tile_kernels.cu): tap gather / combine of
// the interpolation rules, the error-bounded quantizer, warp reductions and
// the shared-memory code histogram.
#pragma once

#include <cuda_runtime.h>

#include "interp_kernels.cuh"

namespace latec {

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

// round_output 2 (integer sources coded in normalised units): the value the
// decoder's caller finally sees is the nearest raw integer, so the bound is
// checked on it, mapped back: (rint(r * span + offset) - offset) / span.
__device__ __forceinline__ float round_raw_f(float r, const QParams& q) {
    const double raw = rint(__dadd_rn(__dmul_rn((double)r, q.rspan), q.roff));
    return __double2float_rn(__ddiv_rn(__dsub_rn(raw, q.roff), q.rspan));
}
__device__ __forceinline__ double round_raw_d(double r, const QParams& q) {
    const double raw = rint(__dadd_rn(__dmul_rn(r, q.rspan), q.roff));
    return __ddiv_rn(__dsub_rn(raw, q.roff), q.rspan);
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
        const float chk = q.round_output == 2 ? round_raw_f(rf, q)
                          : (q.round_output ? rintf(rf) : rf);
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
        const double chk = q.round_output == 2 ? round_raw_d(rd, q)
                           : (q.round_output ? rint(rd) : rd);
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

// ---- decode helpers
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

}  // namespace latec
