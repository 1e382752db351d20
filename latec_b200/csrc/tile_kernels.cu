// Fused level kernels for 3-D grids: the five sub-stages of one level of the
// dyadic schedule in one launch, tile by tile in shared memory.
//
// The level is seen as its lattice (lattice point u <-> grid point s * u).
// The level's points are the lattice points with an odd coordinate; their
// predictions read only lattice points one and three steps away along their
// own odd axes, and a point reached by a step along axis j is even along j,
// so it never steps along j again. A point therefore depends on nothing more
// than three lattice steps away on any axis. A CTA owns a TX x TY column of the
// lattice (axes 2 and 1) over a chunk of axis-0 planes and keeps a box with a
// 3-point halo (4 along axis 2, so rows start on 16-byte boundaries) of each
// plane in shared memory:
//   - a plane with even axis-0 coordinate depends only on itself: its
//     weight-1 points along axes 2 and 1 come from the coarse points, then its
//     weight-2 points from those;
//   - a plane with odd coordinate z needs the even planes z - 3 .. z + 3: its
//     weight-1 points along axis 0, then the weight-2 points, then weight 3.
// The CTA walks its chunk as E(zs - 2), E(zs), E(zs + 2), then E(z + 3), O(z)
// for every odd z of the chunk, with the next plane's box loaded by cp.async
// (16-byte copies when rows are 16-byte aligned) while the current one is
// computed (five even planes in a ring, one odd). Only the classes a neighbour
// needs are computed in the halo, from the same inputs with the same
// arithmetic, so every CTA that holds a point holds the same reconstruction;
// only owned points write codes, outliers, statistics and the canvas.
//
// Every prediction and quantization is the per-stage kernels' arithmetic
// (axis_combine / Quant), so codes, outliers and the reconstruction are
// bit-identical to the stage-by-stage path. Codes go to each stage's rank
// order (closed form below), i.e. the reference's per-stage flat order
// (latec/levels.py:469-574).
#include <cuda_runtime.h>

#include "interp_device.cuh"
#include "tile_kernels.cuh"

namespace latec {
namespace {

template <typename T>
struct TileShape;
template <>
struct TileShape<float> {
    static constexpr int TX = 64, TY = 32;
};
template <>
struct TileShape<double> {
    static constexpr int TX = 64, TY = 16;
};

template <typename T>
struct Box {
    static constexpr int TX = TileShape<T>::TX, TY = TileShape<T>::TY;
    static constexpr int BX = TX + 8;  // lattice columns x0 - 4 .. x0 + TX + 3
    static constexpr int BY = TY + 6;  // lattice rows y0 - 3 .. y0 + TY + 2
    static constexpr int ELEMS = BX * BY;
    static constexpr int SLOTS = 6;  // even planes in a ring of 5, one odd plane
    static constexpr int VEC = 16 / (int)sizeof(T);  // elements per 16-byte group
    static constexpr int GROW = BX / VEC;            // 16-byte groups per box row
    // Class regions (box row r holds lattice row y0 - 3 + r: y is even on odd
    // r; box column b holds lattice column x0 - 4 + b):
    static constexpr int HR_R0 = 1, HR_N = TY / 2 + 3;  // even y over the halo
    static constexpr int TR_R0 = 4, TR_N = TY / 2;      // odd y inside the tile
    static constexpr int HC_B0 = 2, HC_N = TX / 2 + 3;  // even x over the halo
    static constexpr int TC_B0 = 5, TC_N = TX / 2;      // odd x inside the tile
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_addr(dst)), "l"(src),
                 "n"(BYTES));
}
// 16-byte copy; src_bytes 0 writes zeros and reads nothing
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(dst)), "l"(src),
                 "r"(src_bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Even / odd lattice counts along axes 1 and 2 and per-plane class counts:
// the closed-form stage ranks.
struct Ranks {
    uint32_t cye, cyo, cxe, cxo;
    uint32_t a1, a2;  // points of weight 1 / 2 in one axis-0 plane
    __device__ void init(const int32_t* N) {
        cye = (uint32_t)(N[1] + 1) >> 1;
        cyo = (uint32_t)N[1] >> 1;
        cxe = (uint32_t)(N[2] + 1) >> 1;
        cxo = (uint32_t)N[2] >> 1;
        a1 = cyo * cxe + cye * cxo;
        a2 = cyo * cxo;
    }
    // Rank of lattice point (z, y, x) in its stage: C-order over the class
    // lattice for the weight-1 stages; for the fused stages, the count of
    // same-weight points before it in C order.
    template <int STAGE>
    __device__ __forceinline__ uint32_t of(int z, int y, int x) const {
        const uint32_t zh = (uint32_t)z >> 1, yh = (uint32_t)y >> 1, xh = (uint32_t)x >> 1;
        if (STAGE == 0) return (zh * cye + yh) * cxe + xh;
        if (STAGE == 1) return (zh * cyo + yh) * cxe + xh;
        if (STAGE == 2) return (zh * cye + yh) * cxo + xh;
        if (STAGE == 4) return (zh * cyo + yh) * cxo + xh;
        // weight 2
        if (!(z & 1)) return zh * (a2 + a1) + yh * cxo + xh;
        return (zh + 1) * a2 + zh * a1 + (((uint32_t)y + 1) >> 1) * cxo + yh * cxe + xh;
    }
};

// A unit being coded: its plane and its axis-0 neighbours (odd planes only;
// a neighbour outside the lattice aliases the z - 1 plane and is never used).
template <typename T>
struct Unit {
    T* P;
    const T* zm3;
    const T* zm1;
    const T* zp1;
    const T* zp3;
    int z;
    bool owned;
};

struct Item {
    int c, x0, y0, zs, ze;
    int64_t cbase;  // channel offset in the grid
};

template <typename T>
__device__ __forceinline__ AxisTaps<T> mk_taps(T m1, T p1, T m3, T p3, int c, int n) {
    AxisTaps<T> t;
    t.m1 = m1;
    t.p1 = p1;
    t.m3 = m3;
    t.p3 = p3;
    t.ok = (c + 1 < n ? 1u : 0u) | (c >= 3 ? 2u : 0u) | (c + 3 < n ? 4u : 0u);
    return t;
}

// Prediction of a point whose odd axes are (ZO, YO, XO): predict_point's rule
// (center 0 averages the odd axes in axis order; 1 / 2 take the first / last).
template <typename T, int CUBIC, int ZO, int YO, int XO>
__device__ __forceinline__ double predict_tile(const QParams& q, const Unit<T>& u, int pos, int y,
                                               int x, const int32_t* N) {
    using B = Box<T>;
    constexpr int CNT = ZO + YO + XO;
    const int em = q.end_mode;
    auto vz = [&]() {
        return axis_combine<T, CUBIC>(mk_taps(u.zm1[pos], u.zp1[pos], u.zm3[pos], u.zp3[pos], u.z,
                                              N[0]),
                                      em);
    };
    auto vy = [&]() {
        const T* p = u.P + pos;
        return axis_combine<T, CUBIC>(mk_taps(p[-B::BX], p[B::BX], p[-3 * B::BX], p[3 * B::BX], y,
                                              N[1]),
                                      em);
    };
    auto vx = [&]() {
        const T* p = u.P + pos;
        return axis_combine<T, CUBIC>(mk_taps(p[-1], p[1], p[-3], p[3], x, N[2]), em);
    };
    if (CNT == 1) return ZO ? vz() : (YO ? vy() : vx());
    if (q.center == 1) return ZO ? vz() : vy();
    if (q.center == 2) return XO ? vx() : vy();
    if (CNT == 2) {
        const double a = ZO ? vz() : vy();
        const double b = XO ? vx() : vy();
        return __dadd_rn(a, b) * 0.5;
    }
    const double t = __dadd_rn(__dadd_rn(vz(), vy()), vx());
    return __ddiv_rn(t, 3.0);
}

// Point e of a region (rows R0 + 2i, columns B0 + 2j): box position and
// lattice coordinates; inactive points (past the region or outside the
// lattice) take the region's first position, whose taps are in the box.
template <typename T, int R0, int NR, int B0, int NC>
struct RegionPoint {
    int pos, y, x, r, b;
    bool act;
    __device__ __forceinline__ RegionPoint(int e, const Item& it, const int32_t* N) {
        const int i = e / NC, j = e - (e / NC) * NC;
        r = R0 + 2 * i;
        b = B0 + 2 * j;
        y = it.y0 - 3 + r;
        x = it.x0 - 4 + b;
        act = e < NR * NC && y >= 0 && y < N[1] && x >= 0 && x < N[2];
        if (!act) {
            r = R0;
            b = B0;
        }
        pos = r * Box<T>::BX + b;
    }
};

// ------------------------------------------------------------------ encode
template <typename T>
struct TAcc {
    double s[4];  // pred |e|, pred e^2, recon |e|, recon e^2
    T mx;         // recon max |e|
    uint32_t maxq, nout;
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

// Warp maximum of a non-negative value (its bit pattern orders like it).
__device__ __forceinline__ double warp_max_val(float v) {
    return (double)__uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(v)));
}
__device__ __forceinline__ double warp_max_val(double v) { return warp_max(v); }

// Warp sums of the four statistics as a reduce-scatter butterfly (12 shuffles
// instead of 40): lane 8k ends with sum k. The order of the additions is
// fixed, so the sums are deterministic.
template <typename T>
__device__ __forceinline__ void warp_flush(TAcc<T>& a, const EncSm& sm, int stage) {
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
    const double mx = warp_max_val(a.mx);
    const uint32_t mq = __reduce_max_sync(0xffffffffu, a.maxq);
    const uint32_t no = __reduce_add_sync(0xffffffffu, a.nout);
    double* slot = sm.wacc + (w * TILE_STAGES + stage) * 5;
    if ((lane & 7) == 0) slot[(h16 ? 2 : 0) + (h8 ? 1 : 0)] += k;
    if (lane == 1) {
        slot[4] = fmax(slot[4], mx);
        uint32_t& m = sm.wmq[w * TILE_STAGES + stage];
        m = max(m, mq);
        sm.wno[w * TILE_STAGES + stage] += no;
    }
    a.zero();
}

// One class region of a unit, two points in flight per thread.
template <typename T, int CUBIC, int ZO, int YO, int XO, int STAGE, int R0, int NR, int B0, int NC>
__device__ __forceinline__ void enc_region(const TileLevel& L, const Ranks& rk, const Unit<T>& u,
                                           const Item& it, const EncSm& sm, uint32_t cur_seg,
                                           TAcc<T>& a) {
    using B = Box<T>;
    using RP = RegionPoint<T, R0, NR, B0, NC>;
    const TileStage& S = L.st[STAGE];
    const QParams& q = S.q;
    constexpr int NPTS = NR * NC;
    const int lane = threadIdx.x & 31;
    T* staging = (T*)S.staging;
    for (int e0 = 0; e0 < NPTS; e0 += 2 * THREADS) {
        const RP p0(e0 + threadIdx.x, it, L.N), p1(e0 + THREADS + threadIdx.x, it, L.N);
        const T x0 = u.P[p0.pos], x1 = u.P[p1.pos];
        const double d0 = predict_tile<T, CUBIC, ZO, YO, XO>(q, u, p0.pos, p0.y, p0.x, L.N);
        const double d1 = predict_tile<T, CUBIC, ZO, YO, XO>(q, u, p1.pos, p1.y, p1.x, L.N);
        T r0, r1;
        const QOut o0 = Quant<T>::run(x0, d0, q, r0);
        const QOut o1 = Quant<T>::run(x1, d1, q, r1);
        if (p0.act) u.P[p0.pos] = r0;
        if (p1.act) u.P[p1.pos] = r1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const RP& p = h ? p1 : p0;
            const QOut& o = h ? o1 : o0;
            const T xv = h ? x1 : x0, rv = h ? r1 : r0;
            const double pd = h ? d1 : d0;
            int key = -1;
            if (u.owned && p.act && p.r >= 3 && p.r < 3 + B::TY && p.b >= 4 && p.b < 4 + B::TX) {
                const uint64_t gi = (uint64_t)it.c * S.n + rk.of<STAGE>(u.z, p.y, p.x);
                S.codes[gi] = (uint16_t)o.code;
                if (!o.code) {
                    staging[gi] = xv;
                    atomicAdd(&S.tile_cnt[gi / TILE], 1u);
                    a.nout++;
                    key = 0;
                } else {
                    const uint32_t aq = (uint32_t)abs(o.qv);
                    a.maxq = max(a.maxq, aq);
                    key = aq < HWIN ? o.qv + HWIN : -2;
                }
                const uint32_t seg = (uint32_t)(gi >> SEG_SHIFT);
                if (key >= 0 && seg != cur_seg) {  // another segment: straight to global
                    atomicAdd(&S.hist_seg[(size_t)seg * HBINS + key], 1u);
                    key = -1;
                }
                const double er = Quant<T>::err(xv, pd);
                a.s[0] += fabs(er);
                a.s[1] += er * er;
                const double re = Quant<T>::rerr(xv, rv);
                a.s[2] += re;
                a.s[3] += re * re;
                a.mx = max(a.mx, (T)re);
            }
            if (u.owned) hist_warp(sm.hist + STAGE * HBINS, S.hist_total, key, o.code, lane);
        }
    }
}

__device__ __forceinline__ int even_slot(int z) { return (z >> 1) % 5; }

// Issue the cp.async loads of unit plane z (even planes take their coarse
// points from the canvas, every other point from src). vec: 16-byte groups
// (rows 16-byte aligned, unit lattice step along axis 2); even planes then
// stage the canvas rows of even y in `stage` for even_fixup.
template <typename T>
__device__ __forceinline__ void load_plane(const TileLevel& L, const Item& it, int z, bool even,
                                           T* dst, T* stage, const T* __restrict__ src,
                                           const T* __restrict__ canvas, bool vec) {
    using B = Box<T>;
    const int64_t zoff = it.cbase + (int64_t)z * L.ls[0];
    if (vec) {
        for (int e = threadIdx.x; e < B::BY * B::GROW; e += THREADS) {
            const int r = e / B::GROW, g = e - (e / B::GROW) * B::GROW;
            const int y = it.y0 - 3 + r, x = it.x0 - 4 + g * B::VEC;
            const bool in = y >= 0 && y < L.N[1] && x >= 0 && x < L.N[2];
            const int64_t off = in ? zoff + (int64_t)y * L.ls[1] + x : 0;
            cp_async16(dst + r * B::BX + g * B::VEC, src + off, in ? 16u : 0u);
            if (even && !(y & 1))
                cp_async16(stage + r * B::BX + g * B::VEC, canvas + off, in ? 16u : 0u);
        }
        return;
    }
    for (int e = threadIdx.x; e < B::ELEMS; e += THREADS) {
        const int r = e / B::BX, b = e - (e / B::BX) * B::BX;
        const int y = it.y0 - 3 + r, x = it.x0 - 4 + b;
        T* d = dst + r * B::BX + b;
        if (y >= 0 && y < L.N[1] && x >= 0 && x < L.N[2]) {
            const bool coarse = even && !(y & 1) && !(x & 1);
            const int64_t g = zoff + (int64_t)y * L.ls[1] + (int64_t)x * L.ls[2];
            cp_async<sizeof(T)>(d, (coarse ? canvas : src) + g);
        } else {
            *d = (T)0;
        }
    }
}

// Even plane, 16-byte path: the coarse points (even y, even x) from the staged
// canvas rows. Even x sits at offsets 0 and 2 of each 16-byte group of floats
// (offset 0 of doubles).
template <typename T>
__device__ __forceinline__ void even_fixup(T* dst, const T* stage) {
    using B = Box<T>;
    for (int e = threadIdx.x; e < (B::BY / 2) * B::GROW; e += THREADS) {
        const int r = 1 + 2 * (e / B::GROW), g = e - (e / B::GROW) * B::GROW;
        T* d = dst + r * B::BX + g * B::VEC;
        const T* s = stage + r * B::BX + g * B::VEC;
        d[0] = s[0];
        if (B::VEC == 4) d[2] = s[2];
    }
}

// Write an owned plane's tile to the canvas (16-byte groups on the vec path;
// the coarse points of even planes are written back unchanged there).
template <typename T>
__device__ __forceinline__ void store_plane(const TileLevel& L, const Item& it, int z, bool even,
                                            const T* P, T* __restrict__ canvas, bool vec) {
    using B = Box<T>;
    const int64_t zoff = it.cbase + (int64_t)z * L.ls[0];
    if (vec) {
        constexpr int G = B::TX / B::VEC;
        for (int e = threadIdx.x; e < B::TY * G; e += THREADS) {
            const int rr = e / G, g = e - (e / G) * G;
            const int y = it.y0 + rr, x = it.x0 + g * B::VEC;
            if (y < L.N[1] && x < L.N[2])
                *(int4*)(canvas + zoff + (int64_t)y * L.ls[1] + x) =
                    *(const int4*)(P + (rr + 3) * B::BX + 4 + g * B::VEC);
        }
        return;
    }
    for (int e = threadIdx.x; e < B::TX * B::TY; e += THREADS) {
        const int rr = e / B::TX, bb = e - (e / B::TX) * B::TX;
        const int y = it.y0 + rr, x = it.x0 + bb;
        if (y < L.N[1] && x < L.N[2] && !(even && !(y & 1) && !(x & 1)))
            canvas[zoff + (int64_t)y * L.ls[1] + (int64_t)x * L.ls[2]] =
                P[(rr + 3) * B::BX + bb + 4];
    }
}

// Unit k of a chunk: E(zs - 2), E(zs), E(zs + 2), then E(z + 3), O(z) for
// z = zs + 1, zs + 3, ...
__device__ __forceinline__ int unit_z(int k, int zs, bool& even) {
    if (k < 3) {
        even = true;
        return zs - 2 + 2 * k;
    }
    const int j = (k - 3) >> 1;
    even = ((k - 3) & 1) == 0;
    return even ? zs + 4 + 2 * j : zs + 1 + 2 * j;
}

// Work item w: tiles along axis 2 fastest, then axis 1, chunk, channel.
template <typename T>
__device__ __forceinline__ Item item_of(const TileLevel& L, uint32_t w) {
    Item it;
    const uint32_t tx = w % (uint32_t)L.tiles_x;
    w /= (uint32_t)L.tiles_x;
    const uint32_t ty = w % (uint32_t)L.tiles_y;
    w /= (uint32_t)L.tiles_y;
    const uint32_t ch = w % (uint32_t)L.chunks;
    it.c = (int)(w / (uint32_t)L.chunks);
    it.x0 = (int)tx * Box<T>::TX;
    it.y0 = (int)ty * Box<T>::TY;
    it.zs = (int)ch * L.zc;
    it.ze = min(it.zs + L.zc, L.N[0]);
    it.cbase = (int64_t)it.c * (int64_t)L.points;
    return it;
}

template <typename T>
__device__ __forceinline__ Unit<T> make_unit(T* planes, int z, bool even, const Item& it,
                                             int n0) {
    using B = Box<T>;
    Unit<T> u;
    u.z = z;
    u.owned = z >= it.zs && z < it.ze;
    u.P = planes + (even ? even_slot(z) : 5) * B::ELEMS;
    const T* m1 = planes + even_slot(z - 1 >= 0 ? z - 1 : 0) * B::ELEMS;
    u.zm1 = m1;
    u.zp1 = z + 1 < n0 ? planes + even_slot(z + 1) * B::ELEMS : m1;
    u.zm3 = z - 3 >= 0 ? planes + even_slot(z - 3) * B::ELEMS : m1;
    u.zp3 = z + 3 < n0 ? planes + even_slot(z + 3) * B::ELEMS : m1;
    return u;
}

// Units of an item: 3 + 2 x (odd planes in [zs, ze)), zs even.
__device__ __forceinline__ int n_units_of(const Item& it) {
    return 3 + 2 * (it.ze > it.zs ? (it.ze - it.zs) / 2 : 0);
}

// Segment of the histogram that a unit's stage starts in (a hint: points in
// another segment go straight to global memory).
template <int STAGE>
__device__ __forceinline__ uint32_t seg_hint(const TileLevel& L, const Ranks& rk, const Item& it,
                                             int z, int y, int x) {
    return (uint32_t)(((uint64_t)it.c * L.st[STAGE].n + rk.of<STAGE>(z, y, x)) >> SEG_SHIFT);
}

template <typename T, int CUBIC>
__global__ void __launch_bounds__(THREADS, 2)
    k_tile_level_enc(const TileLevel L, const T* __restrict__ x, T* __restrict__ recon) {
    using B = Box<T>;
    extern __shared__ __align__(16) uint8_t smem[];
    T* planes = (T*)smem;
    T* stage = planes + B::SLOTS * B::ELEMS;
    EncSm sm;
    sm.hist = (uint32_t*)(stage + B::ELEMS);
    sm.wacc = (double*)(sm.hist + TILE_STAGES * HBINS);
    sm.wmq = (uint32_t*)(sm.wacc + (THREADS / 32) * TILE_STAGES * 5);
    sm.wno = sm.wmq + (THREADS / 32) * TILE_STAGES;
    for (int i = threadIdx.x; i < TILE_STAGES * HBINS; i += THREADS) sm.hist[i] = 0;
    for (int i = threadIdx.x; i < (THREADS / 32) * TILE_STAGES * 5; i += THREADS) sm.wacc[i] = 0.0;
    for (int i = threadIdx.x; i < (THREADS / 32) * TILE_STAGES; i += THREADS)
        sm.wmq[i] = sm.wno[i] = 0u;
    __syncthreads();
    const bool vec = L.vec != 0;
    Ranks rk;
    rk.init(L.N);
    uint32_t cur_seg[TILE_STAGES];
#pragma unroll
    for (int s = 0; s < TILE_STAGES; s++) cur_seg[s] = 0xffffffffu;
    TAcc<T> a;
    a.zero();

    for (uint32_t w = blockIdx.x; w < L.items; w += gridDim.x) {
        const Item it = item_of<T>(L, w);
        const int n_units = n_units_of(it);
        {
            bool ev;
            const int z = unit_z(0, it.zs, ev);
            if (z >= 0 && z < L.N[0])
                load_plane<T>(L, it, z, ev, planes + even_slot(z) * B::ELEMS, stage, x, recon,
                              vec);
            cp_commit();
        }
        for (int k = 0; k < n_units; k++) {
            bool even;
            const int z = unit_z(k, it.zs, even);
            const bool live = z >= 0 && z < L.N[0];
            cp_wait_all();
            __syncthreads();
            if (live && even && vec) {
                even_fixup<T>(planes + even_slot(z) * B::ELEMS, stage);
                __syncthreads();
            }
            if (k + 1 < n_units) {  // the next unit's plane, while this one is computed
                bool ev;
                const int zn = unit_z(k + 1, it.zs, ev);
                if (zn >= 0 && zn < L.N[0])
                    load_plane<T>(L, it, zn, ev, planes + (ev ? even_slot(zn) : 5) * B::ELEMS,
                                  stage, x, recon, vec);
            }
            cp_commit();
            if (!live) continue;
            const Unit<T> u = make_unit<T>(planes, z, even, it, L.N[0]);
            if (u.owned) {  // histogram segments of this plane's stages (uniform)
                uint32_t ns[3];
                int st[3];
                if (even) {
                    st[0] = 1, st[1] = 2, st[2] = 3;
                    ns[0] = seg_hint<1>(L, rk, it, z, it.y0 + 1, it.x0);
                    ns[1] = seg_hint<2>(L, rk, it, z, it.y0, it.x0 + 1);
                    ns[2] = seg_hint<3>(L, rk, it, z, it.y0 + 1, it.x0 + 1);
                } else {
                    st[0] = 0, st[1] = 3, st[2] = 4;
                    ns[0] = seg_hint<0>(L, rk, it, z, it.y0, it.x0);
                    ns[1] = seg_hint<3>(L, rk, it, z, it.y0, it.x0 + 1);
                    ns[2] = seg_hint<4>(L, rk, it, z, it.y0 + 1, it.x0 + 1);
                }
                bool flushed = false;
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    uint32_t& cs = cur_seg[st[j]];
                    if (ns[j] != cs) {
                        if (cs != 0xffffffffu)
                            flush_hist(sm.hist + st[j] * HBINS, L.st[st[j]].hist_seg, cs);
                        cs = ns[j];
                        flushed = true;
                    }
                }
                if (flushed) __syncthreads();
            }
            if (even) {
                // weight 1 along axis 2 (even y over the halo rows, odd x) and
                // along axis 1 (odd y, even x over the halo columns)
                enc_region<T, CUBIC, 0, 0, 1, 2, B::HR_R0, B::HR_N, B::TC_B0, B::TC_N>(
                    L, rk, u, it, sm, cur_seg[2], a);
                if (u.owned) warp_flush(a, sm, 2);
                enc_region<T, CUBIC, 0, 1, 0, 1, B::TR_R0, B::TR_N, B::HC_B0, B::HC_N>(
                    L, rk, u, it, sm, cur_seg[1], a);
                if (u.owned) warp_flush(a, sm, 1);
                __syncthreads();
                enc_region<T, CUBIC, 0, 1, 1, 3, B::TR_R0, B::TR_N, B::TC_B0, B::TC_N>(
                    L, rk, u, it, sm, cur_seg[3], a);
                if (u.owned) warp_flush(a, sm, 3);
            } else {
                enc_region<T, CUBIC, 1, 0, 0, 0, B::HR_R0, B::HR_N, B::HC_B0, B::HC_N>(
                    L, rk, u, it, sm, cur_seg[0], a);
                if (u.owned) warp_flush(a, sm, 0);
                __syncthreads();
                enc_region<T, CUBIC, 1, 0, 1, 3, B::HR_R0, B::HR_N, B::TC_B0, B::TC_N>(
                    L, rk, u, it, sm, cur_seg[3], a);
                enc_region<T, CUBIC, 1, 1, 0, 3, B::TR_R0, B::TR_N, B::HC_B0, B::HC_N>(
                    L, rk, u, it, sm, cur_seg[3], a);
                if (u.owned) warp_flush(a, sm, 3);
                __syncthreads();
                enc_region<T, CUBIC, 1, 1, 1, 4, B::TR_R0, B::TR_N, B::TC_B0, B::TC_N>(
                    L, rk, u, it, sm, cur_seg[4], a);
                if (u.owned) warp_flush(a, sm, 4);
            }
            __syncthreads();
            if (u.owned) store_plane<T>(L, it, z, even, u.P, recon, vec);
        }
        cp_wait_all();
        __syncthreads();
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < TILE_STAGES; s++)
        if (cur_seg[s] != 0xffffffffu) flush_hist(sm.hist + s * HBINS, L.st[s].hist_seg, cur_seg[s]);
    // per stage: the warps' sums in warp order (deterministic), one partial row per CTA
    if (threadIdx.x < TILE_STAGES) {
        const int s = threadIdx.x;
        double t[5] = {0, 0, 0, 0, 0};
        uint32_t mq = 0, no = 0;
        for (int w = 0; w < THREADS / 32; w++) {
            const double* slot = sm.wacc + (w * TILE_STAGES + s) * 5;
            for (int k = 0; k < 4; k++) t[k] += slot[k];
            t[4] = fmax(t[4], slot[4]);
            mq = max(mq, sm.wmq[w * TILE_STAGES + s]);
            no += sm.wno[w * TILE_STAGES + s];
        }
        for (int k = 0; k < 5; k++) L.st[s].partials[(size_t)blockIdx.x * 5 + k] = t[k];
        if (mq) atomicMax(&L.st[s].acc->maxq, mq);
        if (no) atomicAdd(&L.st[s].acc->nout, no);
    }
}

// ------------------------------------------------------------------ decode
// Codes of a unit's computed points into registers (issued early; stored to
// shared memory once the current unit is done). One compile-time loop per
// class region: fixed register slots, constant divisors, the stage known.
template <typename T, int STAGE, int R0, int NR, int B0, int NC>
__device__ __forceinline__ void fetch_region(const TileLevel& L, const Ranks& rk, const Item& it,
                                             int z, uint16_t* pf) {
    constexpr int K = (NR * NC + THREADS - 1) / THREADS;
    const uint16_t* codes = L.st[STAGE].codes + (uint64_t)it.c * L.st[STAGE].n;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int e = threadIdx.x + k * THREADS;
        const int i = e / NC;
        const int y = it.y0 - 3 + R0 + 2 * i, x = it.x0 - 4 + B0 + 2 * (e - i * NC);
        pf[k] = (e < NR * NC && y >= 0 && y < L.N[1] && x >= 0 && x < L.N[2])
                    ? __ldg(codes + rk.of<STAGE>(z, y, x))
                    : (uint16_t)1;
    }
}

template <typename T, int R0, int NR, int B0, int NC>
__device__ __forceinline__ void put_region(const uint16_t* pf, uint16_t* dst) {
    constexpr int K = (NR * NC + THREADS - 1) / THREADS;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int e = threadIdx.x + k * THREADS;
        const int i = e / NC;
        if (e < NR * NC) dst[(R0 + 2 * i) * Box<T>::BX + B0 + 2 * (e - i * NC)] = pf[k];
    }
}

template <typename T>
struct DecSlots {  // register slots per region: even A, B, C; odd D, E, F, G
    using B = Box<T>;
    static constexpr int k(int n) { return (n + THREADS - 1) / THREADS; }
    static constexpr int A = k(B::HR_N * B::TC_N), Bn = k(B::TR_N * B::HC_N),
                         C = k(B::TR_N * B::TC_N), D = k(B::HR_N * B::HC_N);
    static constexpr int EVEN = A + Bn + C, ODD = D + A + Bn + C;
    static constexpr int PF = EVEN > ODD ? EVEN : ODD;
};

template <typename T>
__device__ __forceinline__ void fetch_codes(const TileLevel& L, const Ranks& rk, const Item& it,
                                            int z, bool even, uint16_t* pf) {
    using B = Box<T>;
    using S = DecSlots<T>;
    if (z < 0 || z >= L.N[0]) return;
    if (even) {
        fetch_region<T, 2, B::HR_R0, B::HR_N, B::TC_B0, B::TC_N>(L, rk, it, z, pf);
        fetch_region<T, 1, B::TR_R0, B::TR_N, B::HC_B0, B::HC_N>(L, rk, it, z, pf + S::A);
        fetch_region<T, 3, B::TR_R0, B::TR_N, B::TC_B0, B::TC_N>(L, rk, it, z, pf + S::A + S::Bn);
    } else {
        fetch_region<T, 0, B::HR_R0, B::HR_N, B::HC_B0, B::HC_N>(L, rk, it, z, pf);
        fetch_region<T, 3, B::HR_R0, B::HR_N, B::TC_B0, B::TC_N>(L, rk, it, z, pf + S::D);
        fetch_region<T, 3, B::TR_R0, B::TR_N, B::HC_B0, B::HC_N>(L, rk, it, z, pf + S::D + S::A);
        fetch_region<T, 4, B::TR_R0, B::TR_N, B::TC_B0, B::TC_N>(L, rk, it, z,
                                                                  pf + S::D + S::A + S::Bn);
    }
}

template <typename T>
__device__ __forceinline__ void put_codes(int z, int n0, bool even, const uint16_t* pf,
                                          uint16_t* dst) {
    using B = Box<T>;
    using S = DecSlots<T>;
    if (z < 0 || z >= n0) return;
    if (even) {
        put_region<T, B::HR_R0, B::HR_N, B::TC_B0, B::TC_N>(pf, dst);
        put_region<T, B::TR_R0, B::TR_N, B::HC_B0, B::HC_N>(pf + S::A, dst);
        put_region<T, B::TR_R0, B::TR_N, B::TC_B0, B::TC_N>(pf + S::A + S::Bn, dst);
    } else {
        put_region<T, B::HR_R0, B::HR_N, B::HC_B0, B::HC_N>(pf, dst);
        put_region<T, B::HR_R0, B::HR_N, B::TC_B0, B::TC_N>(pf + S::D, dst);
        put_region<T, B::TR_R0, B::TR_N, B::HC_B0, B::HC_N>(pf + S::D + S::A, dst);
        put_region<T, B::TR_R0, B::TR_N, B::TC_B0, B::TC_N>(pf + S::D + S::A + S::Bn, dst);
    }
}

template <typename T, int CUBIC, int ZO, int YO, int XO, int STAGE, int R0, int NR, int B0, int NC>
__device__ __forceinline__ void dec_region(const TileLevel& L, const Unit<T>& u, const Item& it,
                                           const uint16_t* codes) {
    using RP = RegionPoint<T, R0, NR, B0, NC>;
    const QParams& q = L.st[STAGE].q;
    constexpr int NPTS = NR * NC;
    for (int e0 = 0; e0 < NPTS; e0 += 2 * THREADS) {
        const RP p0(e0 + threadIdx.x, it, L.N), p1(e0 + THREADS + threadIdx.x, it, L.N);
        const uint32_t c0 = codes[p0.pos], c1 = codes[p1.pos];
        const double d0 = predict_tile<T, CUBIC, ZO, YO, XO>(q, u, p0.pos, p0.y, p0.x, L.N);
        const double d1 = predict_tile<T, CUBIC, ZO, YO, XO>(q, u, p1.pos, p1.y, p1.x, L.N);
        // code 0 (outlier): the canvas value, already in the box
        if (p0.act && c0) u.P[p0.pos] = dequant_value<T>(q, d0, c0);
        if (p1.act && c1) u.P[p1.pos] = dequant_value<T>(q, d1, c1);
    }
}

template <typename T, int CUBIC>
__global__ void __launch_bounds__(THREADS, 2)
    k_tile_level_dec(const TileLevel L, T* __restrict__ recon) {
    using B = Box<T>;
    extern __shared__ __align__(16) uint8_t smem[];
    T* planes = (T*)smem;
    uint16_t* csm = (uint16_t*)(planes + B::SLOTS * B::ELEMS);  // 2 x ELEMS codes
    const bool vec = L.vec != 0;
    Ranks rk;
    rk.init(L.N);
    uint16_t pf[DecSlots<T>::PF];
    for (uint32_t w = blockIdx.x; w < L.items; w += gridDim.x) {
        const Item it = item_of<T>(L, w);
        const int n_units = n_units_of(it);
        {
            bool ev;
            const int z = unit_z(0, it.zs, ev);
            if (z >= 0 && z < L.N[0])
                load_plane<T>(L, it, z, false, planes + even_slot(z) * B::ELEMS, nullptr, recon,
                              recon, vec);
            cp_commit();
            fetch_codes<T>(L, rk, it, z, ev, pf);
            put_codes<T>(z, L.N[0], ev, pf, csm);
        }
        for (int k = 0; k < n_units; k++) {
            bool nev = true;
            int nz = -1;
            if (k + 1 < n_units) nz = unit_z(k + 1, it.zs, nev);
            fetch_codes<T>(L, rk, it, nz, nev, pf);
            cp_wait_all();
            __syncthreads();
            if (nz >= 0 && nz < L.N[0])
                load_plane<T>(L, it, nz, false, planes + (nev ? even_slot(nz) : 5) * B::ELEMS,
                              nullptr, recon, recon, vec);
            cp_commit();
            bool even;
            const int z = unit_z(k, it.zs, even);
            const uint16_t* codes = csm + (k & 1) * B::ELEMS;
            if (z >= 0 && z < L.N[0]) {
                const Unit<T> u = make_unit<T>(planes, z, even, it, L.N[0]);
                if (even) {
                    dec_region<T, CUBIC, 0, 0, 1, 2, B::HR_R0, B::HR_N, B::TC_B0, B::TC_N>(L, u, it,
                                                                                           codes);
                    dec_region<T, CUBIC, 0, 1, 0, 1, B::TR_R0, B::TR_N, B::HC_B0, B::HC_N>(L, u, it,
                                                                                           codes);
                    __syncthreads();
                    dec_region<T, CUBIC, 0, 1, 1, 3, B::TR_R0, B::TR_N, B::TC_B0, B::TC_N>(L, u, it,
                                                                                           codes);
                } else {
                    dec_region<T, CUBIC, 1, 0, 0, 0, B::HR_R0, B::HR_N, B::HC_B0, B::HC_N>(L, u, it,
                                                                                           codes);
                    __syncthreads();
                    dec_region<T, CUBIC, 1, 0, 1, 3, B::HR_R0, B::HR_N, B::TC_B0, B::TC_N>(L, u, it,
                                                                                           codes);
                    dec_region<T, CUBIC, 1, 1, 0, 3, B::TR_R0, B::TR_N, B::HC_B0, B::HC_N>(L, u, it,
                                                                                           codes);
                    __syncthreads();
                    dec_region<T, CUBIC, 1, 1, 1, 4, B::TR_R0, B::TR_N, B::TC_B0, B::TC_N>(L, u, it,
                                                                                           codes);
                }
                __syncthreads();
                if (u.owned) store_plane<T>(L, it, z, even, u.P, recon, vec);
            }
            put_codes<T>(nz, L.N[0], nev, pf, csm + ((k + 1) & 1) * B::ELEMS);
            __syncthreads();
        }
        cp_wait_all();
        __syncthreads();
    }
}

template <typename T>
constexpr uint64_t enc_smem() {
    using B = Box<T>;
    return sizeof(T) * (B::SLOTS + 1) * B::ELEMS + 4ull * TILE_STAGES * HBINS +
           8ull * (THREADS / 32) * TILE_STAGES * 5 + 8ull * (THREADS / 32) * TILE_STAGES;
}
template <typename T>
constexpr uint64_t dec_smem() {
    using B = Box<T>;
    return sizeof(T) * B::SLOTS * B::ELEMS + 2ull * 2 * B::ELEMS;
}

template <typename K>
static int set_smem(K kern, uint64_t bytes) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
                   cudaSuccess
               ? LATEC_OK
               : LATEC_ERR_CUDA;
}

}  // namespace

void tile_level_geometry(TileLevel& L, int elem, int n_sm, uint32_t* grid) {
    const int tx = 64, ty = elem == 8 ? 16 : 32;
    L.tiles_x = (L.N[2] + tx - 1) / tx;
    L.tiles_y = (L.N[1] + ty - 1) / ty;
    // about 6 items per CTA of one wave (2 per SM) and chunks of >= 16 planes
    const uint64_t cols = (uint64_t)L.tiles_x * L.tiles_y * L.channels;
    const uint64_t slots = 2ull * (uint64_t)n_sm;
    uint64_t want = (6 * slots + cols - 1) / cols;
    if (want < 1) want = 1;
    int zc = (int)((L.N[0] + want - 1) / want);
    zc = (zc + 1) & ~1;
    if (zc < 16) zc = 16;
    L.zc = zc;
    L.chunks = (L.N[0] + zc - 1) / zc;
    const uint64_t items = cols * (uint64_t)L.chunks;
    L.items = (uint32_t)items;
    *grid = (uint32_t)(items < slots ? items : slots);
}

int launch_tile_level_encode(const TileLevel& L, int dtype, int cubic, uint32_t grid,
                             const void* x, void* recon, cudaStream_t st) {
    if (!grid) return LATEC_OK;
    int rc;
    if (dtype == LATEC_F64) {
        auto k = cubic ? k_tile_level_enc<double, 1> : k_tile_level_enc<double, 0>;
        if ((rc = set_smem(k, enc_smem<double>()))) return rc;
        k<<<grid, THREADS, enc_smem<double>(), st>>>(L, (const double*)x, (double*)recon);
    } else {
        auto k = cubic ? k_tile_level_enc<float, 1> : k_tile_level_enc<float, 0>;
        if ((rc = set_smem(k, enc_smem<float>()))) return rc;
        k<<<grid, THREADS, enc_smem<float>(), st>>>(L, (const float*)x, (float*)recon);
    }
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

int launch_tile_level_decode(const TileLevel& L, int dtype, int cubic, uint32_t grid, void* recon,
                             cudaStream_t st) {
    if (!grid) return LATEC_OK;
    int rc;
    if (dtype == LATEC_F64) {
        auto k = cubic ? k_tile_level_dec<double, 1> : k_tile_level_dec<double, 0>;
        if ((rc = set_smem(k, dec_smem<double>()))) return rc;
        k<<<grid, THREADS, dec_smem<double>(), st>>>(L, (double*)recon);
    } else {
        auto k = cubic ? k_tile_level_dec<float, 1> : k_tile_level_dec<float, 0>;
        if ((rc = set_smem(k, dec_smem<float>()))) return rc;
        k<<<grid, THREADS, dec_smem<float>(), st>>>(L, (float*)recon);
    }
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? LATEC_OK : LATEC_ERR_CUDA;
}

}  // namespace latec
