// Host-side helpers shared by the entry points: validation of the quantizer
// parameters and their translation into the kernels' QParams (one copy, so
// that every entry point accepts and rejects the same inputs), and access to
// CUDA driver functions through the runtime's entry-point query (the library
// links only the CUDA runtime).
#pragma once

#include <cmath>
#include <cuda.h>
#include <cuda_runtime.h>

#include "interp_kernels.cuh"

namespace latec {

// The checks of latec_quant_params shared by every quantizing entry point
// (the reference's own argument checks are in latec/quantizer.py:28-60).
inline bool valid_params(const latec_quant_params* p) {
    if (!p) return false;
    if (p->dtype != LATEC_F32 && p->dtype != LATEC_F64) return false;
    if (p->channels < 1 || p->radius < 1 || p->radius > 32768) return false;
    if (p->order < 0 || p->order > 1 || p->center < 0 || p->center > 2) return false;
    if (p->end_mode < 0 || p->end_mode > 3) return false;
    if (p->round_output < 0 || p->round_output > 2) return false;
    if (p->round_output == 2 &&
        !(p->round_span > 0.0 && std::isfinite(p->round_span) && std::isfinite(p->round_offset)))
        return false;
    return true;
}

// Kernel parameters of one stage (bound eb) over `points` grid points per
// channel; false for a bound that is not positive. The reciprocal fast path of
// the quantizer is disabled (inv_w = 0) when 1 / (2 eb) is not finite.
inline bool make_q(const latec_quant_params* p, double eb, uint64_t points, QParams& q) {
    if (!(eb > 0.0)) return false;
    q.w = 2.0 * eb;
    const double inv = 1.0 / q.w;
    q.inv_w = (std::isfinite(inv) && q.w > 0x1p-1000 && std::isfinite(q.w)) ? inv : 0.0;
    q.eb = eb;
    q.eb_f = (float)eb;
    q.radius = p->radius;
    q.order = p->order;
    q.center = p->center;
    q.end_mode = p->end_mode;
    q.round_output = p->round_output;
    q.rspan = p->round_output == 2 ? p->round_span : 1.0;
    q.roff = p->round_output == 2 ? p->round_offset : 0.0;
    q.channels = p->channels;
    q.points = points;
    return true;
}

// A driver API function by name (nullptr when the driver does not have it).
template <typename F>
inline F driver_fn(const char* name) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint(name, &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
        return nullptr;
    return (F)fn;
}

// Unique id of the calling thread's current CUDA context (0 if none or the
// query is unavailable). Ids are never reused within a process, unlike the
// context handles themselves.
inline unsigned long long current_context_id() {
    using GetCur = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCur get_cur = driver_fn<GetCur>("cuCtxGetCurrent");
    static GetId get_id = driver_fn<GetId>("cuCtxGetId");
    if (!get_cur || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_cur(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

}  // namespace latec
