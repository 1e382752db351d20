// Fused level kernels for 3-D grids: the five sub-stages of one level of the
// dyadic schedule in one launch each way.
//
// The level is seen as its lattice (lattice point u <-> grid point s * u).
// The level's points are the lattice points with an odd coordinate; their
// predictions read only lattice points one and three steps away along their
// own odd axes, and a point reached by a step along axis j is even along j, so
// no dependency is more than three lattice steps away on any axis. With
// (z, y, x) the lattice axes 0, 1, 2 and the parities written e/o:
//   - an even plane z holds the coarse points (e,e,e), weight 1 along y
//     (e,o,e) and along x (e,e,o), both from the coarse points of the plane,
//     and weight 2 (e,o,o) from those two;
//   - an odd plane z holds weight 1 along z (o,e,e) from the coarse points of
//     the even planes z-3 .. z+3, weight 2 (o,o,e) and (o,e,o) from the even
//     planes' weight-1 points and the plane's own (o,e,e), and weight 3
//     (o,o,o) from the even planes' (e,o,o) and the plane's weight-2 points.
//
// A CTA owns a column of TY x TX lattice points (axes 1, 2) over a chunk of
// axis-0 planes and marches along axis 0: E(zs-2), E(zs), E(zs+2), then the
// pair (E(z+3), O(z)) for every odd z of the chunk. A plane lives in shared
// memory split by (y, x) parity into four dense sub-arrays (EE, EO, OE, OO),
// so that every tap read of a warp touches consecutive words: no bank
// conflicts. The box covers the tile plus the halo the tile's points depend
// on (3 points along each of y and x); halo points are computed from the same
// inputs with the same arithmetic as by the CTA that owns them, so every copy
// of a point holds the same reconstruction, and only owned points write codes,
// outliers, statistics and the canvas.
//
// Planes arrive in a staging buffer in natural layout, by TMA
// (cp.async.bulk.tensor, no multicast: the tensor maps cover this GPU's own
// field and canvas) when rows are whole 16-byte groups, else by per-element
// async copies; the next unit's planes load while the current unit computes.
// A unit runs in three phases separated by barriers, each a flat list of warp
// tasks of 32 points of one class:
//   P1: E.(e,o,e), E.(e,e,o), O.(o,e,e)
//   P2: E.(e,o,o), O.(o,o,e), O.(o,e,o)
//   P3: O.(o,o,o)
// Every prediction and quantization is the per-stage kernels' arithmetic
// (axis_combine / Quant / dequant_value), so codes, outliers and the
// reconstruction are bit-identical to the stage-by-stage path. Codes go to
// each stage's rank order (closed form below), i.e. the reference's per-stage
// flat order (latec/levels.py:469-574).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>

#include "host_util.h"
#include "interp_device.cuh"
#include "tile_kernels.cuh"

namespace latec {
namespace {

// Threads per CTA of the encode and decode kernels (two CTAs per SM each):
// 20 and 24 warps per SM, the most each kernel's registers allow (measured:
// more resident warps hide more of the per-point dependency chains).
constexpr int LT_ENC = 320;
constexpr int LT_DEC = 384;
template <bool ENC>
struct Thr {
    static constexpr int T = ENC ? LT_ENC : LT_DEC;  // threads
    static constexpr int W = T / 32;                 // warps
};
constexpr int LW_ENC = Thr<true>::W, LW_DEC = Thr<false>::W;
constexpr int MAXT = 8;       // warp tasks of one phase at most (decode code prefetch)
constexpr uint32_t LOAD_WAIT_LIMIT = 1u << 24;  // polls of a plane load before giving up

template <typename T>
struct G {
    static constexpr int TX = 64;
    static constexpr int TY = sizeof(T) == 4 ? 32 : 16;
    static constexpr int NER = TY / 2 + 3;  // even rows: y0 - 2 .. y0 + TY + 2
    static constexpr int NOR = TY / 2;      // odd rows: y0 + 1 .. y0 + TY - 1
    static constexpr int P = TX / 2 + 4;    // row pitch: E-cols x0-4 .. x0+TX+2, O-cols x0-3 ..
    static constexpr int EE = 0, EO = NER * P, OE = 2 * NER * P, OO = 2 * NER * P + NOR * P;
    static constexpr int SLOT = 2 * (NER + NOR) * P;  // elements of one plane
    static constexpr int SLOTS = 6;                   // 4 even planes, 2 odd planes
    static constexpr int BX = TX + 8;                 // staging columns x0 - 4 .. x0 + TX + 3
    static constexpr int XR = TY + 5;                 // staging rows y0 - 2 .. y0 + TY + 2
    static constexpr int RR = TY / 2 + 3;             // coarse staging: even rows only
    static constexpr int VEC = 16 / (int)sizeof(T);   // elements per 16-byte group
    static constexpr int GPR = BX / VEC;              // 16-byte groups per staging row
    static_assert(2 * P == BX, "a staging row maps onto one E row and one O row");
};

constexpr uint32_t al128(uint32_t v) { return (v + 127u) & ~127u; }

// Shared-memory layout (byte offsets).
template <typename T, bool ENC>
struct Lay {
    using Gm = G<T>;
    static constexpr uint32_t SLOTS = 0;
    static constexpr uint32_t XE = al128(SLOTS + Gm::SLOTS * Gm::SLOT * sizeof(T));
    static constexpr uint32_t XO = al128(XE + Gm::XR * Gm::BX * sizeof(T));
    static constexpr uint32_t RS = al128(XO + Gm::XR * Gm::BX * sizeof(T));
    static constexpr uint32_t HIST = al128(RS + (ENC ? Gm::RR * Gm::BX * sizeof(T) : 0));
    static constexpr uint32_t WACC =
        al128(HIST + (ENC ? sizeof(uint32_t) * TILE_STAGES * HBINS : 0));
    static constexpr int LW = Thr<ENC>::W;
    static constexpr uint32_t WMQ = WACC + (ENC ? sizeof(double) * LW * TILE_STAGES * 5 : 0);
    static constexpr uint32_t WNO = WMQ + (ENC ? sizeof(uint32_t) * LW * TILE_STAGES : 0);
    // decode: per warp, two buffers of MAXT tasks x 32 lanes of 16-bit codes
    static constexpr uint32_t CODE_ENTRIES = 2u * LW * MAXT * 32;
    static constexpr uint32_t CODES =
        al128(WNO + (ENC ? sizeof(uint32_t) * LW * TILE_STAGES : 0));
    static constexpr uint32_t MBAR = al128(CODES + (ENC ? 0 : sizeof(uint16_t) * CODE_ENTRIES));
    static constexpr uint32_t BYTES = MBAR + 16;
    // two resident CTAs per SM (228 KB of shared memory, 1 KB reserved per CTA)
    static_assert(2 * (BYTES + 1024) <= 228 * 1024, "fused level CTA exceeds half an SM");
};

// ------------------------------------------------------------ async copies
__device__ __forceinline__ uint32_t su32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for a phase of the load barrier: false when it did not
// complete within the limit.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < LOAD_WAIT_LIMIT; i++)
        if (mbar_try(bar, parity)) return true;
    return false;
}
// One box of a 4-D tensor map into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load4(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                          int c2, int c3, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}
template <int BYTES>
__device__ __forceinline__ void cp_el(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(su32(dst)), "l"(src),
                 "n"(BYTES), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// ------------------------------------------------------------ classes
enum { C_W1Y, C_W1X, C_W2E, C_W1Z, C_W2ZY, C_W2ZX, C_W3, C_NONE };

// A class of level points: its plane (even / odd z), its sub-array, the region
// it is computed over (rows x columns of the sub-array) and its stage.
template <typename T, int CL>
struct Cl {
    using Gm = G<T>;
    static constexpr int ZO = CL >= C_W1Z ? 1 : 0;
    static constexpr int YO = (CL == C_W1Y || CL == C_W2E || CL == C_W2ZY || CL == C_W3) ? 1 : 0;
    static constexpr int XO = (CL == C_W1X || CL == C_W2E || CL == C_W2ZX || CL == C_W3) ? 1 : 0;
    static constexpr int SUB = YO ? (XO ? Gm::OO : Gm::OE) : (XO ? Gm::EO : Gm::EE);
    // odd rows: the tile's; even rows: the tile's plus the 3-point halo
    static constexpr int NR = YO ? Gm::NOR : Gm::NER;
    // O-cols: the tile's (2 .. TX/2 + 1); E-cols: plus the halo (1 .. TX/2 + 3)
    static constexpr int C0 = XO ? 2 : 1;
    static constexpr int NC = XO ? Gm::TX / 2 : Gm::TX / 2 + 3;
    static constexpr int STAGE = CL == C_W1Z ? 0 : CL == C_W1Y ? 1 : CL == C_W1X ? 2
                                 : CL == C_W3 ? 4 : 3;
    static constexpr int NPTS = NR * NC;
    static constexpr int NT = (NPTS + 31) / 32;
};

template <typename T, int CL>
constexpr int ntasks() {
    if constexpr (CL == C_NONE) return 0;
    else return Cl<T, CL>::NT;
}

// Closed-form stage ranks of lattice point (z, y, x) (per channel): C order
// over the class lattice for the single-class stages; for the fused weight-2
// stage, the count of weight-2 points before it in C order.
struct LvRanks {
    uint32_t cye, cyo, cxe, cxo, a1, a2;
    __device__ void init(const int32_t* N) {
        cye = (uint32_t)(N[1] + 1) >> 1;
        cyo = (uint32_t)N[1] >> 1;
        cxe = (uint32_t)(N[2] + 1) >> 1;
        cxo = (uint32_t)N[2] >> 1;
        a1 = cyo * cxe + cye * cxo;  // weight-2 points of an odd plane
        a2 = cyo * cxo;              // weight-2 points of an even plane
    }
    template <int CL>
    __device__ __forceinline__ uint32_t of(int z, int y, int x) const {
        const uint32_t zh = (uint32_t)z >> 1, yh = (uint32_t)y >> 1, xh = (uint32_t)x >> 1;
        if (CL == C_W1Z) return (zh * cye + yh) * cxe + xh;
        if (CL == C_W1Y) return (zh * cyo + yh) * cxe + xh;
        if (CL == C_W1X) return (zh * cye + yh) * cxo + xh;
        if (CL == C_W3) return (zh * cyo + yh) * cxo + xh;
        if (CL == C_W2E) return zh * (a2 + a1) + yh * cxo + xh;
        return (zh + 1) * a2 + zh * a1 + (((uint32_t)y + 1) >> 1) * cxo + yh * cxe + xh;
    }
};

struct Item {
    int c, x0, y0, zs, ze;  // ze: end of the owned planes (clipped to the lattice)
    int64_t cbase;          // channel offset in the grid
};

__device__ __forceinline__ Item item_of(const TileLevel& L, uint32_t w, int tx, int ty) {
    Item it;
    const uint32_t ix = w % (uint32_t)L.tiles_x;
    w /= (uint32_t)L.tiles_x;
    const uint32_t iy = w % (uint32_t)L.tiles_y;
    w /= (uint32_t)L.tiles_y;
    const uint32_t ch = w % (uint32_t)L.chunks;
    it.c = (int)(w / (uint32_t)L.chunks);
    it.x0 = (int)ix * tx;
    it.y0 = (int)iy * ty;
    it.zs = (int)ch * L.zc;
    it.ze = min(it.zs + L.zc, L.N[0]);
    it.cbase = (int64_t)it.c * (int64_t)L.points;
    return it;
}

// Units of an item: E(zs-2), E(zs), E(zs+2), then (E(z+3), O(z)) per odd z.
__device__ __forceinline__ int n_units(const Item& it) { return 3 + (it.ze - it.zs) / 2; }
__device__ __forceinline__ void unit_planes(const Item& it, int u, int& ez, int& oz) {
    if (u < 3) {
        ez = it.zs - 2 + 2 * u;
        oz = -1;
    } else {
        ez = it.zs + 4 + 2 * (u - 3);
        oz = it.zs + 1 + 2 * (u - 3);
    }
}

// Slots: even plane z in slot (z/2) mod 4, odd plane z in 4 + (z/2) mod 2.
template <typename T>
__device__ __forceinline__ T* slot_of(T* slots, int z) {
    const int k = (z & 1) ? 4 + ((z >> 1) & 1) : ((z >> 1) & 3);
    return slots + k * G<T>::SLOT;
}

template <typename T>
struct Unit {
    T* E;             // slot of the even plane (valid when ev)
    T* O;             // slot of the odd plane (valid when ov)
    const T* zt[4];   // odd plane's axis-0 taps: even planes z-1, z+1, z-3, z+3
    uint32_t zok;     // bit 0: z+1 valid, bit 1: z-3 valid, bit 2: z+3 valid
    int ez, oz;
    bool ev, ov;      // planes inside the lattice (computed)
    bool eown, oown;  // planes owned by the item
};

template <typename T>
__device__ __forceinline__ Unit<T> make_unit(T* slots, const Item& it, int u, int nz) {
    Unit<T> U;
    unit_planes(it, u, U.ez, U.oz);
    U.ev = U.ez >= 0 && U.ez < nz;
    U.ov = U.oz >= 0 && U.oz < nz;
    U.eown = U.ev && U.ez >= it.zs && U.ez < it.ze;
    U.oown = U.ov && U.oz >= it.zs && U.oz < it.ze;
    U.E = slot_of(slots, U.ez < 0 ? 0 : U.ez);
    U.O = slot_of(slots, U.oz < 0 ? 1 : U.oz);
    const int z = U.oz < 0 ? 1 : U.oz;
    const T* m1 = slot_of(slots, z - 1);
    U.zt[0] = m1;
    U.zt[1] = z + 1 < nz ? slot_of(slots, z + 1) : m1;
    U.zt[2] = z - 3 >= 0 ? slot_of(slots, z - 3) : m1;
    U.zt[3] = z + 3 < nz ? slot_of(slots, z + 3) : m1;
    U.zok = (z + 1 < nz ? 1u : 0u) | (z - 3 >= 0 ? 2u : 0u) | (z + 3 < nz ? 4u : 0u);
    return U;
}

// Tap validity of an odd lattice coordinate c on an axis of n points.
__device__ __forceinline__ uint32_t tap_ok(int c, int n) {
    return (c + 1 < n ? 1u : 0u) | (c >= 3 ? 2u : 0u) | (c + 3 < n ? 4u : 0u);
}

template <typename T>
__device__ __forceinline__ AxisTaps<T> taps4(T m1, T p1, T m3, T p3, uint32_t ok) {
    AxisTaps<T> t;
    t.m1 = m1;
    t.p1 = p1;
    t.m3 = m3;
    t.p3 = p3;
    t.ok = ok;
    return t;
}

// A point of a class region: its sub-array position and lattice coordinates.
// Lanes past the region take its last point and must not store anything.
struct Pt {
    int row, col, y, x, idx;
    bool valid;
};

template <typename T, int CL>
__device__ __forceinline__ Pt point_of(int task, const Item& it) {
    using C = Cl<T, CL>;
    Pt p;
    int e = task * 32 + (int)(threadIdx.x & 31);
    p.valid = e < C::NPTS;
    if (!p.valid) e = C::NPTS - 1;
    const int r = e / C::NC;
    p.row = r;
    p.col = C::C0 + (e - r * C::NC);
    p.y = C::YO ? it.y0 + 1 + 2 * p.row : it.y0 - 2 + 2 * p.row;
    p.x = C::XO ? it.x0 - 3 + 2 * p.col : it.x0 - 4 + 2 * p.col;
    p.idx = p.row * G<T>::P + p.col;
    return p;
}

// Prediction of a point of class CL: predict_point's rule (center 0 averages
// the odd axes in axis order; 1 / 2 take the first / last odd axis).
template <typename T, int CUBIC, int CL>
__device__ __forceinline__ double predict(const QParams& q, const Unit<T>& u, const Pt& p,
                                          const int32_t* N) {
    using C = Cl<T, CL>;
    using Gm = G<T>;
    constexpr int CNT = C::ZO + C::YO + C::XO;
    const int em = q.end_mode;
    const T* plane = C::ZO ? u.O : u.E;
    auto vz = [&]() {
        const int o = C::SUB + p.idx;
        return axis_combine<T, CUBIC>(taps4(u.zt[0][o], u.zt[1][o], u.zt[2][o], u.zt[3][o], u.zok),
                                      em);
    };
    auto vy = [&]() {  // even rows row .. row + 3 are y - 3, y - 1, y + 1, y + 3
        const T* s = plane + (C::XO ? Gm::EO : Gm::EE) + p.idx;
        return axis_combine<T, CUBIC>(
            taps4(s[Gm::P], s[2 * Gm::P], s[0], s[3 * Gm::P], tap_ok(p.y, N[1])), em);
    };
    auto vx = [&]() {  // E-cols col - 1 .. col + 2 are x - 3, x - 1, x + 1, x + 3
        const T* s = plane + (C::YO ? Gm::OE : Gm::EE) + p.idx;
        return axis_combine<T, CUBIC>(taps4(s[0], s[1], s[-1], s[2], tap_ok(p.x, N[2])), em);
    };
    if constexpr (CNT == 1) {
        if constexpr (C::ZO == 1) return vz();
        else if constexpr (C::YO == 1) return vy();
        else return vx();
    } else {
        if (q.center == 1) {  // the first odd axis
            if constexpr (C::ZO == 1) return vz();
            else return vy();
        }
        if (q.center == 2) {  // the last odd axis
            if constexpr (C::XO == 1) return vx();
            else return vy();
        }
        if constexpr (CNT == 2) {
            double a, b;
            if constexpr (C::ZO == 1) a = vz();
            else a = vy();
            if constexpr (C::XO == 1) b = vx();
            else b = vy();
            return __dadd_rn(a, b) * 0.5;
        } else {
            const double t = __dadd_rn(__dadd_rn(vz(), vy()), vx());
            return __ddiv_rn(t, 3.0);
        }
    }
}

template <typename T, int CL>
__device__ __forceinline__ bool owned_pos(const Pt& p) {
    using C = Cl<T, CL>;
    using Gm = G<T>;
    return (C::YO || (p.row >= 1 && p.row <= Gm::TY / 2)) &&
           (C::XO || (p.col >= 2 && p.col <= Gm::TX / 2 + 1));
}

// The shared bins of one stage added to its segment's global bins (and
// cleared), by all threads of an encode CTA.
__device__ __forceinline__ void lvl_flush_hist(uint32_t* sh_hist, uint32_t* hist_seg, uint32_t seg) {
    for (int b = threadIdx.x; b < HBINS; b += LT_ENC) {
        const uint32_t v = sh_hist[b];
        if (v) {
            atomicAdd(&hist_seg[(size_t)seg * HBINS + b], v);
            sh_hist[b] = 0;
        }
    }
}

// ------------------------------------------------------------ encode state
template <typename T>
struct TAcc {
    double s[4];  // pred |e|, pred e^2, recon |e|, recon e^2
    T mx;         // recon max |e|
    uint32_t maxq, nout;
    int stage;    // stage these sums belong to (-1: none)
    __device__ void zero() {
        s[0] = s[1] = s[2] = s[3] = 0.0;
        mx = (T)0;
        maxq = nout = 0;
    }
};

struct EncSm {
    uint32_t* hist;  // TILE_STAGES x HBINS
    double* wacc;    // [warp][stage][5]
    uint32_t* wmq;   // [warp][stage]
    uint32_t* wno;   // [warp][stage]
};

__device__ __forceinline__ double wmax_val(float v) {
    return (double)__uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(v)));
}
__device__ __forceinline__ double wmax_val(double v) { return warp_max(v); }

// Add the warp's sums to its statistics slot of stage a.stage, as a
// reduce-scatter butterfly (lane 8k ends with sum k). Fixed order of the
// additions: deterministic.
template <typename T>
__device__ __forceinline__ void warp_flush(TAcc<T>& a, const EncSm& sm) {
    if (a.stage < 0) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool h16 = lane & 16, h8 = lane & 8;
    double k0 = h16 ? a.s[2] : a.s[0], k1 = h16 ? a.s[3] : a.s[1];
    const double s0 = h16 ? a.s[0] : a.s[2], s1 = h16 ? a.s[1] : a.s[3];
    k0 = __dadd_rn(k0, __shfl_xor_sync(0xffffffffu, s0, 16));
    k1 = __dadd_rn(k1, __shfl_xor_sync(0xffffffffu, s1, 16));
    double k = h8 ? k1 : k0;
    k = __dadd_rn(k, __shfl_xor_sync(0xffffffffu, h8 ? k0 : k1, 8));
#pragma unroll
    for (int o = 4; o; o >>= 1) k = __dadd_rn(k, __shfl_xor_sync(0xffffffffu, k, o));
    const double mx = wmax_val(a.mx);
    const uint32_t mq = __reduce_max_sync(0xffffffffu, a.maxq);
    const uint32_t no = __reduce_add_sync(0xffffffffu, a.nout);
    double* slot = sm.wacc + (w * TILE_STAGES + a.stage) * 5;
    if ((lane & 7) == 0) slot[(h16 ? 2 : 0) + (h8 ? 1 : 0)] += k;
    if (lane == 1) {
        slot[4] = fmax(slot[4], mx);
        uint32_t& m = sm.wmq[w * TILE_STAGES + a.stage];
        m = max(m, mq);
        sm.wno[w * TILE_STAGES + a.stage] += no;
    }
    a.zero();
}

template <typename T, int CUBIC, int CL>
__device__ __forceinline__ void enc_task(const TileLevel& L, const LvRanks& rk, const Item& it,
                                         const Unit<T>& u, int task, const EncSm& sm,
                                         const uint32_t* cseg, TAcc<T>& a) {
    using C = Cl<T, CL>;
    if (a.stage != C::STAGE) {  // uniform across the warp
        warp_flush(a, sm);
        a.stage = C::STAGE;
    }
    const Pt p = point_of<T, CL>(task, it);
    T* P = (C::ZO ? u.O : u.E) + C::SUB;
    const TileStage& S = L.st[C::STAGE];
    const QParams& q = S.q;
    const T xv = P[p.idx];
    const double pd = predict<T, CUBIC, CL>(q, u, p, L.N);
    T rv;
    const QOut o = Quant<T>::run(xv, pd, q, rv);
    if (p.valid) P[p.idx] = rv;
    const bool owned = p.valid && (C::ZO ? u.oown : u.eown) && p.y < L.N[1] && p.x < L.N[2] &&
                       owned_pos<T, CL>(p);
    int key = -1;
    if (owned) {
        const int z = C::ZO ? u.oz : u.ez;
        const uint64_t gi = (uint64_t)it.c * S.n + rk.template of<CL>(z, p.y, p.x);
        S.codes[gi] = (uint16_t)o.code;
        if (!o.code) {
            ((T*)S.staging)[gi] = xv;
            atomicAdd(&S.tile_cnt[gi / TILE], 1u);
            a.nout++;
            key = 0;
        } else {
            const uint32_t aq = (uint32_t)abs(o.qv);
            a.maxq = max(a.maxq, aq);
            key = aq < HWIN ? o.qv + HWIN : -2;
        }
        const uint32_t seg = (uint32_t)(gi >> SEG_SHIFT);
        if (key >= 0 && seg != cseg[C::STAGE]) {  // another segment: straight to global
            atomicAdd(&S.hist_seg[(size_t)seg * HBINS + key], 1u);
            key = -1;
        }
        const double er = Quant<T>::err(xv, pd);
        a.s[0] += fabs(er);
        a.s[1] = __fma_rn(er, er, a.s[1]);
        const double re = Quant<T>::rerr(xv, rv);
        a.s[2] += re;
        a.s[3] = __fma_rn(re, re, a.s[3]);
        a.mx = max(a.mx, (T)re);
    }
    hist_warp(sm.hist + C::STAGE * HBINS, S.hist_total, key, o.code, threadIdx.x & 31);
}

// One phase of up to three classes: warp w takes a contiguous range of the
// phase's tasks (static: the statistics' summation order is fixed).
template <typename T, int CUBIC, int CA, int CB, int CC>
__device__ __forceinline__ void enc_phase(const TileLevel& L, const LvRanks& rk, const Item& it,
                                          const Unit<T>& u, bool ea, bool eb, bool ec,
                                          const EncSm& sm, const uint32_t* cseg, TAcc<T>& a) {
    const int na = ea ? ntasks<T, CA>() : 0, nb = eb ? ntasks<T, CB>() : 0;
    const int nc = ec ? ntasks<T, CC>() : 0;
    const int tot = na + nb + nc, w = threadIdx.x >> 5;
    const int tb = w * tot / LW_ENC, te = (w + 1) * tot / LW_ENC;
    for (int t = tb; t < te; t++) {
        if (t < na) {
            if constexpr (CA != C_NONE) enc_task<T, CUBIC, CA>(L, rk, it, u, t, sm, cseg, a);
        } else if (t < na + nb) {
            if constexpr (CB != C_NONE) enc_task<T, CUBIC, CB>(L, rk, it, u, t - na, sm, cseg, a);
        } else {
            if constexpr (CC != C_NONE)
                enc_task<T, CUBIC, CC>(L, rk, it, u, t - na - nb, sm, cseg, a);
        }
    }
}

// ------------------------------------------------------------ decode tasks
template <typename T, int CL>
__device__ __forceinline__ uint32_t code_of(const TileLevel& L, const LvRanks& rk, const Item& it,
                                            const Unit<T>& u, int task) {
    using C = Cl<T, CL>;
    const Pt p = point_of<T, CL>(task, it);
    if (!p.valid || p.y < 0 || p.x < 0 || p.y >= L.N[1] || p.x >= L.N[2]) return 0u;
    const TileStage& S = L.st[C::STAGE];
    const int z = C::ZO ? u.oz : u.ez;
    return __ldg(S.codes + (uint64_t)it.c * S.n + rk.template of<CL>(z, p.y, p.x));
}

template <typename T, int CUBIC, int CL>
__device__ __forceinline__ void dec_task(const TileLevel& L, const Item& it, const Unit<T>& u,
                                         int task, uint32_t code) {
    using C = Cl<T, CL>;
    if (code == 0) return;  // outlier (already in the canvas box) or outside the lattice
    const Pt p = point_of<T, CL>(task, it);
    T* P = (C::ZO ? u.O : u.E) + C::SUB;
    const QParams& q = L.st[C::STAGE].q;
    const double pd = predict<T, CUBIC, CL>(q, u, p, L.N);
    P[p.idx] = dequant_value<T>(q, pd, code);
}

// The task counts of phase ph (0, 1, 2) of a unit, per class.
template <typename T>
__device__ __forceinline__ void phase_counts(int ph, bool ev, bool ov, int& na, int& nb, int& nc) {
    if (ph == 0) {
        na = ev ? ntasks<T, C_W1Y>() : 0;
        nb = ev ? ntasks<T, C_W1X>() : 0;
        nc = ov ? ntasks<T, C_W1Z>() : 0;
    } else if (ph == 1) {
        na = ev ? ntasks<T, C_W2E>() : 0;
        nb = ov ? ntasks<T, C_W2ZY>() : 0;
        nc = ov ? ntasks<T, C_W2ZX>() : 0;
    } else {
        na = ov ? ntasks<T, C_W3>() : 0;
        nb = nc = 0;
    }
}

// Codes of the warp's tasks of phase ph of unit u into registers.
template <typename T>
__device__ __forceinline__ void fetch_phase(const TileLevel& L, const LvRanks& rk, const Item& it,
                                            const Unit<T>& u, int ph, uint32_t* pf) {
    int na, nb, nc;
    phase_counts<T>(ph, u.ev, u.ov, na, nb, nc);
    const int tot = na + nb + nc, w = threadIdx.x >> 5;
    const int tb = w * tot / LW_DEC, te = (w + 1) * tot / LW_DEC;
#pragma unroll
    for (int k = 0; k < MAXT; k++) {
        const int t = tb + k;
        uint32_t c = 0;
        if (t < te) {
            if (ph == 0) {
                c = t < na ? code_of<T, C_W1Y>(L, rk, it, u, t)
                    : t < na + nb ? code_of<T, C_W1X>(L, rk, it, u, t - na)
                                  : code_of<T, C_W1Z>(L, rk, it, u, t - na - nb);
            } else if (ph == 1) {
                c = t < na ? code_of<T, C_W2E>(L, rk, it, u, t)
                    : t < na + nb ? code_of<T, C_W2ZY>(L, rk, it, u, t - na)
                                  : code_of<T, C_W2ZX>(L, rk, it, u, t - na - nb);
            } else {
                c = code_of<T, C_W3>(L, rk, it, u, t);
            }
        }
        pf[k] = c;
    }
}

template <typename T, int CUBIC, int CA, int CB, int CC>
__device__ __forceinline__ void dec_phase(const TileLevel& L, const Item& it, const Unit<T>& u,
                                          bool ea, bool eb, bool ec, const uint16_t* wcodes) {
    const int na = ea ? ntasks<T, CA>() : 0, nb = eb ? ntasks<T, CB>() : 0;
    const int nc = ec ? ntasks<T, CC>() : 0;
    const int tot = na + nb + nc, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tb = w * tot / LW_DEC, te = (w + 1) * tot / LW_DEC;
    for (int t = tb; t < te; t++) {
        const uint32_t code = wcodes[(t - tb) * 32 + lane];
        if (t < na) {
            if constexpr (CA != C_NONE) dec_task<T, CUBIC, CA>(L, it, u, t, code);
        } else if (t < na + nb) {
            if constexpr (CB != C_NONE) dec_task<T, CUBIC, CB>(L, it, u, t - na, code);
        } else {
            if constexpr (CC != C_NONE) dec_task<T, CUBIC, CC>(L, it, u, t - na - nb, code);
        }
    }
}

// ------------------------------------------------------------ plane movement
// Issue the loads of a unit's planes into the staging buffers: the even
// plane's box (x, or the canvas when decoding) and, when encoding, its coarse
// even rows from the canvas; the odd plane's box. Returns whether anything was
// issued (uniform).
template <typename T, bool ENC, int TMA>
__device__ __forceinline__ bool issue_loads(const CUtensorMap* tmx, const CUtensorMap* tmr,
                                            const TileLevel& L, const Item& it, const Unit<T>& u,
                                            T* XE, T* XO, T* RS, uint32_t bar, const T* src,
                                            const T* canvas) {
    using Gm = G<T>;
    if (!u.ev && !u.ov) return false;
    if (TMA) {
        if (threadIdx.x == 0) {
            constexpr uint32_t XB = Gm::XR * Gm::BX * sizeof(T), RB = Gm::RR * Gm::BX * sizeof(T);
            const uint32_t bytes = (u.ev ? XB + (ENC ? RB : 0u) : 0u) + (u.ov ? XB : 0u);
            mbar_expect(bar, bytes);
            const int cx = it.x0 - 4, cy = it.y0 - 2;
            if (u.ev) {
                tma_load4(su32(XE), tmx, cx, cy, u.ez, it.c, bar);
                if (ENC) tma_load4(su32(RS), tmr, cx, it.y0 / 2 - 1, u.ez, it.c, bar);
            }
            if (u.ov) tma_load4(su32(XO), tmx, cx, cy, u.oz, it.c, bar);
        }
        return true;
    }
    auto box = [&](T* dst, const T* base, int z, int ystep, int rows) {
        const int64_t zo = it.cbase + (int64_t)z * L.ls[0];
        for (int e = threadIdx.x; e < rows * Gm::BX; e += Thr<ENC>::T) {
            const int r = e / Gm::BX, b = e - (e / Gm::BX) * Gm::BX;
            const int Y = it.y0 - 2 + r * ystep, X = it.x0 - 4 + b;
            const bool in = Y >= 0 && Y < L.N[1] && X >= 0 && X < L.N[2];
            const T* s = in ? base + zo + (int64_t)Y * L.ls[1] + (int64_t)X * L.ls[2] : base;
            cp_el<sizeof(T)>(dst + e, s, in ? (uint32_t)sizeof(T) : 0u);
        }
    };
    if (u.ev) {
        box(XE, src, u.ez, 1, Gm::XR);
        if (ENC) box(RS, canvas, u.ez, 2, Gm::RR);
    }
    if (u.ov) box(XO, src, u.oz, 1, Gm::XR);
    cp_commit();
    return true;
}

// Staging (natural layout) -> slot (parity-split layout). For an encoded even
// plane the coarse points (even y, even x) come from the canvas rows in RS.
template <typename T, int NT>
__device__ __forceinline__ void transpose_plane(T* slot, const T* SX, const T* SR) {
    using Gm = G<T>;
    constexpr int ROWS = Gm::NER + Gm::NOR;
    for (int e = threadIdx.x; e < ROWS * Gm::GPR; e += NT) {
        const int i = e / Gm::GPR, g = e - (e / Gm::GPR) * Gm::GPR;
        const bool even = i < Gm::NER;
        const int ri = even ? i : i - Gm::NER;
        const int srow = even ? 2 * ri : 3 + 2 * ri;
        T* Er = slot + (even ? Gm::EE : Gm::OE) + ri * Gm::P;
        T* Or = slot + (even ? Gm::EO : Gm::OO) + ri * Gm::P;
        if constexpr (sizeof(T) == 4) {
            const float4 v = *(const float4*)(SX + srow * Gm::BX + 4 * g);
            float2 ev = make_float2(v.x, v.z);
            if (even && SR) {
                const float4 r = *(const float4*)(SR + ri * Gm::BX + 4 * g);
                ev = make_float2(r.x, r.z);
            }
            *(float2*)(Er + 2 * g) = ev;
            *(float2*)(Or + 2 * g) = make_float2(v.y, v.w);
        } else {
            const double2 v = *(const double2*)(SX + srow * Gm::BX + 2 * g);
            Er[g] = (even && SR) ? SR[ri * Gm::BX + 2 * g] : v.x;
            Or[g] = v.y;
        }
    }
}

// Write the tile of an owned plane from its slot to the canvas (16-byte
// groups on the TMA path, whose rows are whole groups; else element by
// element, skipping the coarse points of even planes).
template <typename T, int TMA, int NT>
__device__ __forceinline__ void store_plane(const TileLevel& L, const Item& it, int z,
                                            const T* slot, T* __restrict__ canvas) {
    using Gm = G<T>;
    const int64_t zo = it.cbase + (int64_t)z * L.ls[0];
    if (TMA) {
        constexpr int GT = Gm::TX / Gm::VEC;
        for (int e = threadIdx.x; e < Gm::TY * GT; e += NT) {
            const int r = e / GT, g = e - (e / GT) * GT;
            const int y = it.y0 + r, x = it.x0 + g * Gm::VEC;
            if (y >= L.N[1] || x >= L.N[2]) continue;
            const bool ey = !(r & 1);
            const int ri = ey ? r / 2 + 1 : r / 2;
            const T* E = slot + (ey ? Gm::EE : Gm::OE) + ri * Gm::P;
            const T* O = slot + (ey ? Gm::EO : Gm::OO) + ri * Gm::P;
            T* d = canvas + zo + (int64_t)y * L.ls[1] + x;
            if constexpr (sizeof(T) == 4) {
                const float2 a = *(const float2*)(E + 2 + 2 * g), b = *(const float2*)(O + 2 + 2 * g);
                *(float4*)d = make_float4(a.x, b.x, a.y, b.y);
            } else {
                *(double2*)d = make_double2(E[2 + g], O[2 + g]);
            }
        }
        return;
    }
    const bool evenz = !(z & 1);
    for (int e = threadIdx.x; e < Gm::TY * Gm::TX; e += NT) {
        const int r = e / Gm::TX, b = e - (e / Gm::TX) * Gm::TX;
        const int y = it.y0 + r, x = it.x0 + b;
        if (y >= L.N[1] || x >= L.N[2]) continue;
        const bool ey = !(r & 1), ex = !(b & 1);
        if (evenz && ey && ex) continue;  // coarse point: unchanged
        const int ri = ey ? r / 2 + 1 : r / 2;
        const int sub = ey ? (ex ? Gm::EE : Gm::EO) : (ex ? Gm::OE : Gm::OO);
        canvas[zo + (int64_t)y * L.ls[1] + (int64_t)x * L.ls[2]] =
            slot[sub + ri * Gm::P + 2 + b / 2];
    }
}

// The histogram segment of stage s's first owned point in unit u (for
// flushing the shared bins when the segment changes). 0xffffffff: the stage
// has no owned point in the unit.
template <typename T>
__device__ __forceinline__ uint32_t unit_seg(const TileLevel& L, const LvRanks& rk,
                                             const Item& it, const Unit<T>& u, int s) {
    uint32_t r;
    const int y0 = it.y0, x0 = it.x0;
    // the stage's first point in the tile must lie in the lattice
    const int fy = y0 + ((s == 1 || s == 4 || (s == 3 && u.eown)) ? 1 : 0);
    const int fx = x0 + ((s == 2 || s == 3 || s == 4) ? 1 : 0);
    if (fy >= L.N[1] || fx >= L.N[2]) return 0xffffffffu;
    switch (s) {
        case 0:
            if (!u.oown) return 0xffffffffu;
            r = rk.of<C_W1Z>(u.oz, y0, x0);
            break;
        case 1:
            if (!u.eown) return 0xffffffffu;
            r = rk.of<C_W1Y>(u.ez, y0 + 1, x0);
            break;
        case 2:
            if (!u.eown) return 0xffffffffu;
            r = rk.of<C_W1X>(u.ez, y0, x0 + 1);
            break;
        case 3:
            if (u.eown) r = rk.of<C_W2E>(u.ez, y0 + 1, x0 + 1);
            else if (u.oown) r = rk.of<C_W2ZX>(u.oz, y0, x0 + 1);
            else return 0xffffffffu;
            break;
        default:
            if (!u.oown) return 0xffffffffu;
            r = rk.of<C_W3>(u.oz, y0 + 1, x0 + 1);
            break;
    }
    return (uint32_t)(((uint64_t)it.c * L.st[s].n + r) >> SEG_SHIFT);
}

// ------------------------------------------------------------ kernels
// The CTA's units, across its items (item blockIdx.x + k gridDim.x).
struct Cursor {
    uint32_t item;
    int u;
};

// Phase 0 of a unit: the previous unit's finished planes out to the canvas,
// then (once its loads landed) this unit's planes from staging into their
// slots. Within an item the two touch different slots; the first unit of an
// item may reuse the slot of the previous item's last plane, so those stores
// finish first.
template <typename T, int TMA, int NT>
__device__ __forceinline__ void phase0(const TileLevel& L, const Item& prev, int st_e, int st_o,
                                       const Unit<T>& u, bool first, bool pending, uint32_t bar,
                                       uint32_t& parity, bool& wait_failed, T* slots, const T* XE,
                                       const T* XO, const T* RS, T* canvas) {
    const bool out = st_e >= 0 || st_o >= 0;
    if (out && first) {
        if (st_e >= 0) store_plane<T, TMA, NT>(L, prev, st_e, slot_of(slots, st_e), canvas);
        if (st_o >= 0) store_plane<T, TMA, NT>(L, prev, st_o, slot_of(slots, st_o), canvas);
        __syncthreads();
    }
    if (pending) {
        if (TMA) {
            if (!mbar_wait(bar, parity)) wait_failed = true;
            parity ^= 1u;
        } else {
            cp_wait_all();
            __syncthreads();
        }
    }
    if (u.ev) transpose_plane<T, NT>(u.E, XE, RS);
    if (u.ov) transpose_plane<T, NT>(u.O, XO, nullptr);
    if (out && !first) {
        if (st_e >= 0) store_plane<T, TMA, NT>(L, prev, st_e, slot_of(slots, st_e), canvas);
        if (st_o >= 0) store_plane<T, TMA, NT>(L, prev, st_o, slot_of(slots, st_o), canvas);
    }
}

template <typename T, int CUBIC, int TMA>
__global__ void __launch_bounds__(LT_ENC, 2)
    k_lvl_enc(const __grid_constant__ CUtensorMap tmx, const __grid_constant__ CUtensorMap tmr,
              const TileLevel L, const T* __restrict__ x, T* __restrict__ recon) {
    using Gm = G<T>;
    using Ly = Lay<T, true>;
    extern __shared__ __align__(128) uint8_t smem[];
    T* slots = (T*)(smem + Ly::SLOTS);
    T* XE = (T*)(smem + Ly::XE);
    T* XO = (T*)(smem + Ly::XO);
    T* RS = (T*)(smem + Ly::RS);
    EncSm sm;
    sm.hist = (uint32_t*)(smem + Ly::HIST);
    sm.wacc = (double*)(smem + Ly::WACC);
    sm.wmq = (uint32_t*)(smem + Ly::WMQ);
    sm.wno = (uint32_t*)(smem + Ly::WNO);
    const uint32_t bar = su32(smem + Ly::MBAR);
    for (int i = threadIdx.x; i < TILE_STAGES * HBINS; i += LT_ENC) sm.hist[i] = 0;
    for (int i = threadIdx.x; i < LW_ENC * TILE_STAGES * 5; i += LT_ENC) sm.wacc[i] = 0.0;
    for (int i = threadIdx.x; i < LW_ENC * TILE_STAGES; i += LT_ENC) sm.wmq[i] = sm.wno[i] = 0u;
    if (threadIdx.x == 0) mbar_init(bar);
    __syncthreads();
    LvRanks rk;
    rk.init(L.N);
    uint32_t cseg[TILE_STAGES];
#pragma unroll
    for (int s = 0; s < TILE_STAGES; s++) cseg[s] = 0xffffffffu;
    TAcc<T> a;
    a.zero();
    a.stage = -1;
    uint32_t parity = 0;
    bool wait_failed = false;

    const int nz = L.N[0];
    Cursor cur{blockIdx.x, 0};
    Item it{}, prev{};
    int st_e = -1, st_o = -1;  // planes of the previous unit still to store
    bool pending = false;
    if (cur.item < L.items) {
        it = item_of(L, cur.item, Gm::TX, Gm::TY);
        pending = issue_loads<T, true, TMA>(&tmx, &tmr, L, it, make_unit(slots, it, 0, nz), XE, XO,
                                            RS, bar, x, recon);
    }
    while (cur.item < L.items) {
        const Unit<T> u = make_unit(slots, it, cur.u, nz);
        phase0<T, TMA, LT_ENC>(L, prev, st_e, st_o, u, cur.u == 0, pending, bar, parity, wait_failed,
                       slots, XE, XO, RS, recon);
        // histogram segments of this unit's stages (uniform decisions)
#pragma unroll
        for (int s = 0; s < TILE_STAGES; s++) {
            const uint32_t ns = unit_seg(L, rk, it, u, s);
            if (ns != 0xffffffffu && ns != cseg[s]) {
                if (cseg[s] != 0xffffffffu)
                    lvl_flush_hist(sm.hist + s * HBINS, L.st[s].hist_seg, cseg[s]);
                cseg[s] = ns;
            }
        }
        __syncthreads();
        // the next unit's loads (the staging buffers are free again)
        Cursor nxt = cur;
        if (++nxt.u >= n_units(it)) {
            nxt.item += gridDim.x;
            nxt.u = 0;
        }
        Item nit = it;
        pending = false;
        if (nxt.item < L.items) {
            if (nxt.item != cur.item) nit = item_of(L, nxt.item, Gm::TX, Gm::TY);
            pending = issue_loads<T, true, TMA>(&tmx, &tmr, L, nit, make_unit(slots, nit, nxt.u, nz),
                                                XE, XO, RS, bar, x, recon);
        }
        enc_phase<T, CUBIC, C_W1Y, C_W1X, C_W1Z>(L, rk, it, u, u.ev, u.ev, u.ov, sm, cseg, a);
        __syncthreads();
        enc_phase<T, CUBIC, C_W2E, C_W2ZY, C_W2ZX>(L, rk, it, u, u.ev, u.ov, u.ov, sm, cseg, a);
        __syncthreads();
        if (u.ov)
            enc_phase<T, CUBIC, C_W3, C_NONE, C_NONE>(L, rk, it, u, true, false, false, sm, cseg,
                                                      a);
        __syncthreads();
        prev = it;
        st_e = u.eown ? u.ez : -1;
        st_o = u.oown ? u.oz : -1;
        cur = nxt;
        it = nit;
    }
    if (st_e >= 0) store_plane<T, TMA, LT_ENC>(L, prev, st_e, slot_of(slots, st_e), recon);
    if (st_o >= 0) store_plane<T, TMA, LT_ENC>(L, prev, st_o, slot_of(slots, st_o), recon);
    warp_flush(a, sm);
    if (TMA && wait_failed) {  // let a late load land before the CTA exits
        mbar_wait(bar, parity ^ 1u);
        if (threadIdx.x == 0) atomicOr(&L.st[0].acc->done, TILE_WAIT_FAILED);
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < TILE_STAGES; s++)
        if (cseg[s] != 0xffffffffu) lvl_flush_hist(sm.hist + s * HBINS, L.st[s].hist_seg, cseg[s]);
    // per stage: the warps' sums in warp order (deterministic), one partial row per CTA
    if (threadIdx.x < TILE_STAGES) {
        const int s = threadIdx.x;
        double t[5] = {0, 0, 0, 0, 0};
        uint32_t mq = 0, no = 0;
        for (int w = 0; w < LW_ENC; w++) {
            const double* sl = sm.wacc + (w * TILE_STAGES + s) * 5;
            for (int k = 0; k < 4; k++) t[k] += sl[k];
            t[4] = fmax(t[4], sl[4]);
            mq = max(mq, sm.wmq[w * TILE_STAGES + s]);
            no += sm.wno[w * TILE_STAGES + s];
        }
        for (int k = 0; k < 5; k++) L.st[s].partials[(size_t)blockIdx.x * 5 + k] = t[k];
        if (mq) atomicMax(&L.st[s].acc->maxq, mq);
        if (no) atomicAdd(&L.st[s].acc->nout, no);
    }
}

template <typename T, int CUBIC, int TMA>
__global__ void __launch_bounds__(LT_DEC, 2)
    k_lvl_dec(const __grid_constant__ CUtensorMap tmx, const TileLevel L, T* __restrict__ recon,
              uint32_t* __restrict__ err) {
    using Gm = G<T>;
    using Ly = Lay<T, false>;
    extern __shared__ __align__(128) uint8_t smem[];
    T* slots = (T*)(smem + Ly::SLOTS);
    T* XE = (T*)(smem + Ly::XE);
    T* XO = (T*)(smem + Ly::XO);
    // this warp's two buffers of MAXT tasks x 32 codes (Ly::CODE_ENTRIES in all)
    static_assert(Ly::CODE_ENTRIES == LW_DEC * 2 * MAXT * 32, "code buffer layout");
    uint16_t* wc = (uint16_t*)(smem + Ly::CODES) + (threadIdx.x >> 5) * 2 * MAXT * 32;
    const uint32_t bar = su32(smem + Ly::MBAR);
    if (threadIdx.x == 0) mbar_init(bar);
    __syncthreads();
    LvRanks rk;
    rk.init(L.N);
    uint32_t parity = 0;
    bool wait_failed = false;
    const int nz = L.N[0], lane = threadIdx.x & 31;

    Cursor cur{blockIdx.x, 0};
    Item it{}, prev{};
    int st_e = -1, st_o = -1;
    bool pending = false;
    uint32_t pf[MAXT];
    int buf = 0;
    if (cur.item < L.items) {
        it = item_of(L, cur.item, Gm::TX, Gm::TY);
        const Unit<T> u0 = make_unit(slots, it, 0, nz);
        pending = issue_loads<T, false, TMA>(&tmx, &tmx, L, it, u0, XE, XO, nullptr, bar, recon,
                                             recon);
        fetch_phase<T>(L, rk, it, u0, 0, pf);
#pragma unroll
        for (int k = 0; k < MAXT; k++) wc[k * 32 + lane] = (uint16_t)pf[k];
        __syncwarp();
    }
    while (cur.item < L.items) {
        const Unit<T> u = make_unit(slots, it, cur.u, nz);
        phase0<T, TMA, LT_DEC>(L, prev, st_e, st_o, u, cur.u == 0, pending, bar, parity, wait_failed,
                       slots, XE, XO, nullptr, recon);
        __syncthreads();
        Cursor nxt = cur;
        if (++nxt.u >= n_units(it)) {
            nxt.item += gridDim.x;
            nxt.u = 0;
        }
        Item nit = it;
        pending = false;
        const bool more = nxt.item < L.items;
        if (more) {
            if (nxt.item != cur.item) nit = item_of(L, nxt.item, Gm::TX, Gm::TY);
            pending = issue_loads<T, false, TMA>(&tmx, &tmx, L, nit,
                                                 make_unit(slots, nit, nxt.u, nz), XE, XO, nullptr,
                                                 bar, recon, recon);
        }
        // each phase: fetch the next phase's codes, decode this one, then
        // store the fetched codes (the loads had the whole phase to land)
        fetch_phase<T>(L, rk, it, u, 1, pf);
        dec_phase<T, CUBIC, C_W1Y, C_W1X, C_W1Z>(L, it, u, u.ev, u.ev, u.ov, wc + buf * MAXT * 32);
        buf ^= 1;
#pragma unroll
        for (int k = 0; k < MAXT; k++) wc[buf * MAXT * 32 + k * 32 + lane] = (uint16_t)pf[k];
        __syncthreads();
        fetch_phase<T>(L, rk, it, u, 2, pf);
        dec_phase<T, CUBIC, C_W2E, C_W2ZY, C_W2ZX>(L, it, u, u.ev, u.ov, u.ov,
                                                   wc + buf * MAXT * 32);
        buf ^= 1;
#pragma unroll
        for (int k = 0; k < MAXT; k++) wc[buf * MAXT * 32 + k * 32 + lane] = (uint16_t)pf[k];
        __syncthreads();
        if (more) fetch_phase<T>(L, rk, nit, make_unit(slots, nit, nxt.u, nz), 0, pf);
        if (u.ov)
            dec_phase<T, CUBIC, C_W3, C_NONE, C_NONE>(L, it, u, true, false, false,
                                                      wc + buf * MAXT * 32);
        buf ^= 1;
#pragma unroll
        for (int k = 0; k < MAXT; k++) wc[buf * MAXT * 32 + k * 32 + lane] = (uint16_t)pf[k];
        __syncthreads();
        prev = it;
        st_e = u.eown ? u.ez : -1;
        st_o = u.oown ? u.oz : -1;
        cur = nxt;
        it = nit;
    }
    if (st_e >= 0) store_plane<T, TMA, LT_DEC>(L, prev, st_e, slot_of(slots, st_e), recon);
    if (st_o >= 0) store_plane<T, TMA, LT_DEC>(L, prev, st_o, slot_of(slots, st_o), recon);
    if (TMA && wait_failed) {
        mbar_wait(bar, parity ^ 1u);
        if (threadIdx.x == 0) atomicOr(err, ERR_TILE_WAIT);
    }
}

template <typename K>
static int set_smem(K kern, uint32_t bytes) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
                   cudaSuccess
               ? LATEC_OK
               : LATEC_ERR_CUDA;
}

// Tensor map of a 4-D (x, y, z, channel) box over the level's lattice (unit
// step along x). row_step 2 maps the even rows only.
template <typename T>
static bool make_map(CUtensorMap* m, const TileLevel& L, const void* base, int row_step,
                     uint32_t box_rows) {
    using Enc = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                             const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                             const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                             CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Enc enc = driver_fn<Enc>("cuTensorMapEncodeTiled");
    if (!enc) return false;
    const uint64_t e = sizeof(T);
    const cuuint64_t dims[4] = {(cuuint64_t)L.N[2],
                                (cuuint64_t)((L.N[1] + row_step - 1) / row_step),
                                (cuuint64_t)L.N[0], (cuuint64_t)L.channels};
    const cuuint64_t strides[3] = {(cuuint64_t)(L.ls[1] * row_step) * e, (cuuint64_t)L.ls[0] * e,
                                   (cuuint64_t)L.points * e};
    const cuuint32_t box[4] = {(cuuint32_t)G<T>::BX, box_rows, 1, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return enc(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
               4, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T, int CUBIC>
static int launch_enc(const TileLevel& L, uint32_t grid, const void* x, void* recon,
                      cudaStream_t st) {
    CUtensorMap mx, mr;
    std::memset(&mx, 0, sizeof(mx));
    std::memset(&mr, 0, sizeof(mr));
    constexpr uint32_t bytes = Lay<T, true>::BYTES;
    int rc;
    if (L.tma) {
        if (!make_map<T>(&mx, L, x, 1, G<T>::XR) || !make_map<T>(&mr, L, recon, 2, G<T>::RR))
            return LATEC_ERR_CUDA;
        if ((rc = set_smem(k_lvl_enc<T, CUBIC, 1>, bytes))) return rc;
        k_lvl_enc<T, CUBIC, 1><<<grid, LT_ENC, bytes, st>>>(mx, mr, L, (const T*)x, (T*)recon);
    } else {
        if ((rc = set_smem(k_lvl_enc<T, CUBIC, 0>, bytes))) return rc;
        k_lvl_enc<T, CUBIC, 0><<<grid, LT_ENC, bytes, st>>>(mx, mr, L, (const T*)x, (T*)recon);
    }
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

template <typename T, int CUBIC>
static int launch_dec(const TileLevel& L, uint32_t grid, void* recon, uint32_t* err,
                      cudaStream_t st) {
    CUtensorMap mx;
    std::memset(&mx, 0, sizeof(mx));
    constexpr uint32_t bytes = Lay<T, false>::BYTES;
    int rc;
    if (L.tma) {
        if (!make_map<T>(&mx, L, recon, 1, G<T>::XR)) return LATEC_ERR_CUDA;
        if ((rc = set_smem(k_lvl_dec<T, CUBIC, 1>, bytes))) return rc;
        k_lvl_dec<T, CUBIC, 1><<<grid, LT_DEC, bytes, st>>>(mx, L, (T*)recon, err);
    } else {
        if ((rc = set_smem(k_lvl_dec<T, CUBIC, 0>, bytes))) return rc;
        k_lvl_dec<T, CUBIC, 0><<<grid, LT_DEC, bytes, st>>>(mx, L, (T*)recon, err);
    }
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // namespace

void tile_level_geometry(TileLevel& L, int elem, int n_sm, uint32_t* grid) {
    const int tx = tile_tx(elem), ty = tile_ty(elem);
    L.tiles_x = (L.N[2] + tx - 1) / tx;
    L.tiles_y = (L.N[1] + ty - 1) / ty;
    const uint64_t cols = (uint64_t)L.tiles_x * L.tiles_y * L.channels;
    const uint64_t slots = 2ull * (uint64_t)n_sm;  // resident CTAs (2 per SM)
    // chunk length: the cost of a CTA is the items it runs (the busiest CTA
    // runs ceil(items / slots) of them) times the planes an item computes
    // (its chunk plus about three halo planes)
    int best = 16;
    double best_cost = 1e300;
    for (int zc = 8; zc <= 128; zc *= 2) {
        const uint64_t chunks = (uint64_t)(L.N[0] + zc - 1) / zc;
        const uint64_t items = cols * chunks;
        const uint64_t per = (items + slots - 1) / slots;
        const double cost = (double)per * (double)(zc + 3);
        if (cost < best_cost * 0.999) {
            best_cost = cost;
            best = zc;
        }
        if ((uint64_t)zc >= (uint64_t)L.N[0]) break;
    }
    L.zc = best;
    L.chunks = (L.N[0] + best - 1) / best;
    const uint64_t items = cols * (uint64_t)L.chunks;
    L.items = (uint32_t)items;
    *grid = (uint32_t)(items < slots ? items : slots);
}

int launch_tile_level_encode(const TileLevel& L, int dtype, int cubic, uint32_t grid,
                             const void* x, void* recon, cudaStream_t st) {
    if (!grid) return LATEC_OK;
    if (dtype == LATEC_F64)
        return cubic ? launch_enc<double, 1>(L, grid, x, recon, st)
                     : launch_enc<double, 0>(L, grid, x, recon, st);
    return cubic ? launch_enc<float, 1>(L, grid, x, recon, st)
                 : launch_enc<float, 0>(L, grid, x, recon, st);
}

int launch_tile_level_decode(const TileLevel& L, int dtype, int cubic, uint32_t grid, void* recon,
                             uint32_t* err, cudaStream_t st) {
    if (!grid) return LATEC_OK;
    if (dtype == LATEC_F64)
        return cubic ? launch_dec<double, 1>(L, grid, recon, err, st)
                     : launch_dec<double, 0>(L, grid, recon, err, st);
    return cubic ? launch_dec<float, 1>(L, grid, recon, err, st)
                 : launch_dec<float, 0>(L, grid, recon, err, st);
}

}  // namespace latec
