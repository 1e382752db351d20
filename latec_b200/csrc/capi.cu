// extern "C" entry points of liblatec_b200 (declared in include/latec_b200.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "host_util.h"
#include "interp_kernels.cuh"
#include "plan.h"
#include "rans_kernels.cuh"
#include "tile_kernels.cuh"

#include <atomic>
#include <mutex>

using namespace latec;

static std::atomic<unsigned long long> g_launches{0};
namespace latec {
void count_launches(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace latec

static_assert(sizeof(latec_stage_stats) == sizeof(StageAcc), "stats layout");
static_assert(sizeof(latec_rans_stage) == sizeof(RansStageDesc), "rans stage layout");
static_assert(sizeof(EncSym) == 32, "encoder symbol layout");
static_assert(sizeof(latec_encode_job) == 144 && sizeof(latec_decode_job) == 112,
              "many-tensor job layouts (the Python binding mirrors them)");

namespace {

constexpr uint64_t ALIGN = 256;
inline uint64_t align_up(uint64_t v) { return (v + ALIGN - 1) & ~(ALIGN - 1); }

struct Carve {
    uint8_t* base;
    uint64_t off = 0;
    template <typename T>
    T* take(uint64_t count) {
        T* p = base ? (T*)(base + off) : nullptr;
        off = align_up(off + count * sizeof(T));
        return p;
    }
};

inline int elem_of(int dtype) { return dtype == LATEC_F64 ? 8 : 4; }

// Level-kernel bounds (per level): bands per sub-stage, sub-stages per level.
constexpr uint32_t LVL_MAX_BANDS = 1024;
constexpr uint32_t LVL_MAX_STAGES = 2 * MAXD - 1;
constexpr uint32_t LVL_MAX_DEPS = LVL_MAX_STAGES * LVL_MAX_BANDS * LVL_MAX_STAGES * 4;
constexpr uint32_t LVL_CHUNK_TILES = 4;  // tiles per decode work item
// slabs between a sub-stage and the next weight in the claim order: a whole
// slab step separates an item from the items it depends on
constexpr int LVL_LAG = 2;

struct StageWs {
    void* staging;
    uint32_t* tile_cnt;   // per tile of the largest stage (encode) / of all stages (decode)
    uint32_t* tile_off;
    uint32_t* total;
    double* partials;
    DecStage* dec;        // decode: per-stage descriptors of the all-stage tile passes
    LvlStage* lvl_stages; // level kernels: descriptors, bands, dependencies, items, counters
    LvlBand* lvl_bands;
    LvlDep* lvl_deps;
    LvlItem* lvl_items;
    uint32_t* lvl_ctr;
    uint64_t lvl_items_cap;
};

// Workspace carve-up: `max_items` sizes the per-stage encode scratch;
// `all_tiles` / `n_stages` the decode's all-stage tile arrays.
uint64_t stage_ws(uint64_t max_items, uint64_t all_tiles, int n_stages, int elem, StageWs* out,
                  void* base) {
    Carve c{(uint8_t*)base};
    StageWs w;
    const uint64_t tiles = (n_tiles(max_items) > all_tiles ? n_tiles(max_items) : all_tiles) + 1;
    w.staging = c.take<uint8_t>(max_items * elem);
    w.tile_cnt = c.take<uint32_t>(tiles);
    w.tile_off = c.take<uint32_t>(tiles);
    w.total = c.take<uint32_t>(4);
    w.partials = c.take<double>((uint64_t)TILE_STAGES * MAX_BLOCKS * 5 + 5);
    w.dec = c.take<DecStage>(n_stages > 0 ? n_stages : 1);
    w.lvl_items_cap = all_tiles + (uint64_t)LVL_MAX_STAGES * LVL_MAX_BANDS;
    w.lvl_stages = c.take<LvlStage>(LVL_MAX_STAGES);
    w.lvl_bands = c.take<LvlBand>((uint64_t)LVL_MAX_STAGES * LVL_MAX_BANDS);
    w.lvl_deps = c.take<LvlDep>(LVL_MAX_DEPS);
    w.lvl_items = c.take<LvlItem>(w.lvl_items_cap);
    w.lvl_ctr = c.take<uint32_t>((uint64_t)LVL_MAX_STAGES * LVL_MAX_BANDS + 1);
    if (out) *out = w;
    return c.off;
}

// Stages [t, t + 5) form a standard level of a 3-D plan: weight 1 along axes
// 0, 1 and 2, then the fused weight-2 and weight-3 stages, all of one stride.
bool tile_level_shape(const latec_plan* plan, int t) {
    // blocked anchors leave holes in the finer stages: per-stage launches only
    if (plan->ndim != 3 || plan->anchor_block != 1 || t < 1 ||
        t + TILE_STAGES > (int)plan->stages.size())
        return false;
    const StageDesc* d = &plan->stages[t];
    const int s = d[0].s;
    for (int j = 0; j < 3; j++)
        if (d[j].kind != 0 || d[j].axis != j || d[j].weight != 1 || d[j].s != s) return false;
    return d[3].kind == 1 && d[3].weight == 2 && d[3].s == s && d[4].kind == 1 &&
           d[4].weight == 3 && d[4].s == s;
}

void plan_sizes(const latec_plan* plan, int C, uint64_t* max_items, uint64_t* all_tiles) {
    uint64_t m = 0, t = 0;
    for (auto& d : plan->stages) {
        const uint64_t items = (uint64_t)d.n * C;
        m = items > m ? items : m;
        t += n_tiles(items);
    }
    // a fused level stages the outliers of its five stages at once
    for (int k = 1; k < (int)plan->stages.size(); k++) {
        if (!tile_level_shape(plan, k)) continue;
        uint64_t sum = 0;
        for (int j = 0; j < TILE_STAGES; j++) sum += (uint64_t)plan->stages[k + j].n * C;
        m = sum > m ? sum : m;
    }
    *max_items = m;
    *all_tiles = t;
}

// Fused levels of 3-D plans: 0 off (per-stage launches, the default: the
// 512^3 round trip measured 9.4 ms against 9.6 ms with the finest level fused
// and 10.0 ms with every large level fused), 1 the finest level (stride 1)
// only, 2 every level of at least TILE_MIN_POINTS points, 3 every level
// whatever its size. Results are bit-identical in every mode.
std::atomic<int> g_tile_mode{0};
// Below this many points a level keeps its per-stage launches: a small
// lattice has too few column tiles to fill the GPU with fused work items.
constexpr uint64_t TILE_MIN_POINTS = 1ull << 18;

// Kernel timing (a measurement aid): when on, a CUDA event pair is recorded
// on the launching stream around every fused-level launch (kind 0 = encode,
// 1 = decode) and every lane-coder launch (2 = encode, 3 = decode).
std::atomic<bool> g_kt_on{false};
std::mutex g_kt_mu;
struct KtPair {
    cudaEvent_t a, b;
    int kind;
};
std::vector<KtPair> g_kt_pairs, g_kt_free;

int kt_start(int kind, cudaStream_t st) {
    if (!g_kt_on.load()) return -1;
    std::lock_guard<std::mutex> lk(g_kt_mu);
    KtPair p;
    if (!g_kt_free.empty()) {
        p = g_kt_free.back();
        g_kt_free.pop_back();
    } else if (cudaEventCreate(&p.a) != cudaSuccess || cudaEventCreate(&p.b) != cudaSuccess) {
        return -1;
    }
    p.kind = kind;
    if (cudaEventRecord(p.a, st) != cudaSuccess) {
        g_kt_free.push_back(p);
        return -1;
    }
    g_kt_pairs.push_back(p);
    return (int)g_kt_pairs.size() - 1;
}

void kt_stop(int idx, cudaStream_t st) {
    if (idx < 0) return;
    std::lock_guard<std::mutex> lk(g_kt_mu);
    if (idx < (int)g_kt_pairs.size()) cudaEventRecord(g_kt_pairs[idx].b, st);
}

bool tile_level_at(const latec_plan* plan, int t, int mode) {
    if (mode == 0 || !tile_level_shape(plan, t)) return false;
    if (mode == 1 && plan->stages[t].s != 1) return false;
    uint64_t n = 0;
    for (int j = 0; j < TILE_STAGES; j++) n += plan->stages[t + j].n;
    return mode == 2 ? n >= TILE_MIN_POINTS : n > 0;
}

int n_sms() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

// The lattice of the level starting at stage t, its work split and the
// per-stage quantizers and code arrays (codes_off: first code of stage t).
bool tile_level_init(const latec_plan* plan, const latec_quant_params* prm,
                     const double* stage_eb, int t, int C, uint16_t* codes, uint64_t codes_off,
                     TileLevel& L, uint32_t* grid) {
    std::memset(&L, 0, sizeof(L));
    const StageDesc& d = plan->stages[t];
    for (int j = 0; j < 3; j++) {
        L.N[j] = (int32_t)((d.shape[j] + d.s - 1) / d.s);
        L.ls[j] = (int64_t)d.s * d.gstride[j];
    }
    L.points = plan->points;
    L.channels = C;
    tile_level_geometry(L, elem_of(prm->dtype), n_sms(), grid);
    if (*grid > (uint32_t)MAX_BLOCKS) *grid = MAX_BLOCKS;
    uint64_t o = codes_off;
    for (int j = 0; j < TILE_STAGES; j++) {
        TileStage& S = L.st[j];
        if (!make_q(prm, stage_eb[t + j], plan->points, S.q)) return false;
        S.n = plan->stages[t + j].n;
        S.codes = codes + o;
        o += (uint64_t)S.n * C;
    }
    return true;
}

// 0 per-stage launches (default: measured faster on B200, see the design
// notes), 1 level kernels for levels of >= 4 Mi points, 2 every level that
// qualifies
std::atomic<int> g_level_mode{0};

// First rank of stage d whose axis-0 coordinate is >= z (ranks follow the flat
// grid order, so the axis-0 coordinate never decreases with the rank).
uint64_t rank_at_z(const StageDesc& d, int32_t z) {
    uint64_t lo = 0, hi = d.n;
    int32_t coord[MAXD];
    while (lo < hi) {
        const uint64_t mid = (lo + hi) / 2;
        stage_coords(d, (uint32_t)mid, coord);
        if (coord[0] < z) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

int32_t z_of(const StageDesc& d, uint64_t r) {
    int32_t coord[MAXD];
    stage_coords(d, (uint32_t)r, coord);
    return coord[0];
}

struct LevelBuild {
    std::vector<LvlStage> st;
    std::vector<LvlBand> bands;
    std::vector<LvlDep> deps;
    std::vector<LvlItem> items;
};

// Work items of one level [t0, t1) for the level decode kernel, or false when
// the level does not qualify (one channel, 2+ axes, enough bands) or when some
// dependency would not precede the item that needs it in the claim order.
// Bands are slabs of T planes along axis 0, T >= 5 s (taps reach 3 s; one
// slab of slack covers the rounding of band starts down to a tile).
bool build_level(const latec_plan* plan, int t0, int t1, int C, int elem, int mode,
                 uint64_t items_cap, LevelBuild& L, uint32_t* tiles_per_stage) {
    if (mode == 0 || C != 1 || plan->ndim < 2 || plan->anchor_block != 1 || t0 < 1 || t1 - t0 < 2 ||
        t1 - t0 > (int)LVL_MAX_STAGES)
        return false;
    const int s = plan->stages[t0].s;
    const int32_t nz = (int32_t)plan->shape[0];
    uint64_t level_points = 0;
    for (int t = t0; t < t1; t++) level_points += plan->stages[t].n;
    if (mode == 1 && level_points < (4ull << 20)) return false;
    const uint64_t plane_bytes = plan->points / (uint64_t)nz * (uint64_t)(elem + 2);
    const int32_t unit = 2 * s;
    // ~12 MB slabs keep a few of them in L2; mode 2 takes the thinnest legal
    // slab so that small grids get several bands too
    int32_t T = mode == 2 ? 5 * s : (int32_t)((12ull << 20) / (plane_bytes ? plane_bytes : 1));
    if (T < 5 * s) T = 5 * s;
    // at least two tiles of every sub-stage per slab, so that rounding slab
    // starts down to a tile moves them by less than half a slab
    for (int t = t0; t < t1; t++) {
        const uint64_t per_plane = plan->stages[t].n / (uint64_t)nz + 1;
        const uint64_t need = (2ull * TILE + per_plane - 1) / per_plane;
        if ((uint64_t)T < need) T = (int32_t)std::min<uint64_t>(need, (uint64_t)nz);
    }
    T = (T + unit - 1) / unit * unit;
    int32_t B = (nz + T - 1) / T;
    if (B > (int32_t)LVL_MAX_BANDS) {
        T = (nz + LVL_MAX_BANDS - 1) / LVL_MAX_BANDS;
        T = (T + unit - 1) / unit * unit;
        B = (nz + T - 1) / T;
    }
    if (B < 2) return false;
    const int ns = t1 - t0;
    std::vector<std::vector<uint64_t>> R(ns, std::vector<uint64_t>(B + 1));
    std::vector<std::vector<int32_t>> zs(ns, std::vector<int32_t>(B)), ze(ns, std::vector<int32_t>(B));
    int maxlag = 0;
    for (int j = 0; j < ns; j++) {
        const StageDesc& d = plan->stages[t0 + j];
        maxlag = std::max(maxlag, LVL_LAG * (d.weight - 1));
        R[j][0] = 0;
        for (int k = 1; k < B; k++) {
            uint64_t r = rank_at_z(d, k * T) / TILE * TILE;
            R[j][k] = r < R[j][k - 1] ? R[j][k - 1] : r;
        }
        R[j][B] = d.n;
        for (int k = 0; k < B; k++)
            if (R[j][k] < R[j][k + 1]) {
                zs[j][k] = z_of(d, R[j][k]);
                ze[j][k] = z_of(d, R[j][k + 1] - 1);
            }
        tiles_per_stage[j] = n_tiles(d.n);
    }
    // claim order: step b runs band b - lag of every sub-stage, lower weights first
    std::vector<int64_t> first(ns * B, -1), last(ns * B, -1), cnt(ns * B, 0);
    for (int b = 0; b < B + maxlag; b++)
        for (int j = 0; j < ns; j++) {
            const int k = b - LVL_LAG * (plan->stages[t0 + j].weight - 1);
            if (k < 0 || k >= B || R[j][k] >= R[j][k + 1]) continue;
            const uint32_t ta = (uint32_t)(R[j][k] / TILE);
            const uint32_t tb = k + 1 == B ? tiles_per_stage[j] : (uint32_t)(R[j][k + 1] / TILE);
            for (uint32_t a = ta; a < tb; a += LVL_CHUNK_TILES) {
                if (first[j * B + k] < 0) first[j * B + k] = (int64_t)L.items.size();
                last[j * B + k] = (int64_t)L.items.size();
                cnt[j * B + k]++;
                L.items.push_back(LvlItem{(uint32_t)(j * B + k), a,
                                          std::min(tb, a + LVL_CHUNK_TILES), 0u});
            }
        }
    if (L.items.size() > items_cap) return false;
    L.bands.resize((size_t)ns * B);
    for (int j = 0; j < ns; j++) {
        const StageDesc& d = plan->stages[t0 + j];
        for (int k = 0; k < B; k++) {
            LvlBand& bd = L.bands[(size_t)j * B + k];
            bd.stage = (uint32_t)j;
            bd.counter = (uint32_t)(j * B + k);
            bd.dep_off = (uint32_t)L.deps.size();
            bd.dep_cnt = 0;
            if (R[j][k] >= R[j][k + 1]) continue;
            const int32_t lo = zs[j][k] - 3 * s, hi = ze[j][k] + 3 * s;
            for (int jp = 0; jp < ns; jp++) {
                if (plan->stages[t0 + jp].weight >= d.weight) continue;
                for (int kp = 0; kp < B; kp++) {
                    if (R[jp][kp] >= R[jp][kp + 1]) continue;
                    if (ze[jp][kp] < lo || zs[jp][kp] > hi) continue;
                    if (last[jp * B + kp] >= first[j * B + k]) return false;
                    L.deps.push_back(LvlDep{(uint32_t)(jp * B + kp), (uint32_t)cnt[jp * B + kp]});
                    bd.dep_cnt++;
                    if (L.deps.size() > LVL_MAX_DEPS) return false;
                }
            }
        }
    }
    return true;
}

// ---- many tensors per call

// The plan's stage descriptors on the current device, uploaded on first use.
const StageDesc* plan_dev_stages(const latec_plan* cp) {
    latec_plan* p = const_cast<latec_plan*>(cp);  // the device copy is a cache
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(p->dev_mu);
    if (p->dev_stages && p->dev_id == dev) return p->dev_stages;
    if (p->dev_stages) {
        cudaFree(p->dev_stages);
        p->dev_stages = nullptr;
    }
    const size_t n = p->stages.size() ? p->stages.size() : 1;
    StageDesc* d = nullptr;
    if (cudaMalloc(&d, sizeof(StageDesc) * n) != cudaSuccess) return nullptr;
    if (!p->stages.empty() &&
        cudaMemcpy(d, p->stages.data(), sizeof(StageDesc) * p->stages.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return nullptr;
    }
    p->dev_stages = d;
    p->dev_id = dev;
    return d;
}

// Kernel class of a stage: value type, rank (runtime rank for blocked
// anchors and ranks outside 2..4), layout, order.
inline int many_nd(const StageDesc& d) {
    return (d.ndim >= 2 && d.ndim <= 4 && !d.holes && d.kind != 2) ? d.ndim : 0;
}
inline int many_key(int dtype, const StageDesc& d, int order) {
    return (((dtype == LATEC_F64 ? 1 : 0) * 8 + many_nd(d)) * 2 + (d.kind == 1 ? 1 : 0)) * 2 +
           (order ? 1 : 0);
}

// Launch tables of a many-tensor call, built on the host and uploaded in one
// copy: 16-byte aligned records appended in launch order.
struct HostTable {
    std::vector<uint8_t> buf;
    template <typename T>
    uint64_t put(const T* p, size_t n) {
        const uint64_t off = (buf.size() + 15) & ~uint64_t(15);
        buf.resize(off + sizeof(T) * n);
        if (n) std::memcpy(buf.data() + off, p, sizeof(T) * n);
        return off;
    }
    uint64_t size() const { return (buf.size() + 15) & ~uint64_t(15); }
};

struct ManyLaunch {
    int op;         // 0 zero ranges, 1 quantize, 2 compact, 3 dequantize
    int key;        // kernel class (op 1)
    uint64_t recs;  // table offset of the ZeroRange / ManyJob / DecStage records
    uint64_t first; // table offset of the first-CTA array
    uint32_t n;     // records
    uint32_t ctas;  // grid
};

// Zero ranges in chunks of ZERO_CHUNK words per CTA.
void add_zero_launch(HostTable& T, std::vector<ManyLaunch>& L, const std::vector<ZeroRange>& r) {
    std::vector<ZeroRange> keep;
    std::vector<uint32_t> first;
    uint64_t ctas = 0;
    for (const ZeroRange& z : r) {
        if (!z.words) continue;
        keep.push_back(z);
        first.push_back((uint32_t)ctas);
        ctas += (z.words + ZERO_CHUNK - 1) / ZERO_CHUNK;
    }
    if (keep.empty()) return;
    ManyLaunch l{0, 0, T.put(keep.data(), keep.size()), T.put(first.data(), first.size()),
                 (uint32_t)keep.size(), (uint32_t)ctas};
    L.push_back(l);
}

// One step's jobs laid out by kernel class; a launch per class (op 1
// quantize, 3 dequantize) and, for the encoder, one compaction launch over
// all of them (op 2).
void add_step_launches(HostTable& T, std::vector<ManyLaunch>& L, std::vector<ManyJob>& jobs,
                       const std::vector<int>& keys, int op, bool compact) {
    if (jobs.empty()) return;
    std::vector<size_t> order(jobs.size());
    for (size_t k = 0; k < order.size(); k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return keys[a] < keys[b]; });
    std::vector<ManyJob> sorted;
    sorted.reserve(jobs.size());
    for (size_t k : order) sorted.push_back(jobs[k]);
    const uint64_t recs = T.put(sorted.data(), sorted.size());
    size_t a = 0;
    while (a < order.size()) {
        size_t e = a;
        std::vector<uint32_t> first;
        uint64_t ctas = 0;
        while (e < order.size() && keys[order[e]] == keys[order[a]]) {
            first.push_back((uint32_t)ctas);
            ctas += sorted[e].blocks;
            e++;
        }
        ManyLaunch l{op, keys[order[a]], recs + sizeof(ManyJob) * a,
                     T.put(first.data(), first.size()), (uint32_t)(e - a), (uint32_t)ctas};
        L.push_back(l);
        a = e;
    }
    if (compact) {
        std::vector<uint32_t> first;
        uint64_t ctas = 0;
        for (const ManyJob& j : sorted) {
            first.push_back((uint32_t)ctas);
            ctas += j.cblocks;
        }
        ManyLaunch l{2, 0, recs, T.put(first.data(), first.size()), (uint32_t)sorted.size(),
                     (uint32_t)ctas};
        L.push_back(l);
    }
}

}  // namespace

extern "C" {

int latec_set_level_mode(int32_t mode) {
    if (mode < 0 || mode > 2) return LATEC_ERR_ARG;
    g_level_mode.store(mode);
    return LATEC_OK;
}

int latec_set_tile_mode(int32_t mode) {
    if (mode < 0 || mode > 3) return LATEC_ERR_ARG;
    g_tile_mode.store(mode);
    return LATEC_OK;
}

int latec_set_row_mode(int32_t on) {
    if (on < 0 || on > 1) return LATEC_ERR_ARG;
    g_row_mode.store(on);
    return LATEC_OK;
}

int latec_set_kernel_timing(int32_t on) {
    g_kt_on.store(on != 0);
    return LATEC_OK;
}

int latec_kernel_time(int32_t kind, double* ms, uint32_t* launches) {
    if (!ms || !launches || kind < 0 || kind > 5) return LATEC_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_kt_mu);
    double sum = 0.0;
    uint32_t n = 0;
    int rc = LATEC_OK;
    std::vector<KtPair> keep;
    for (auto& p : g_kt_pairs) {
        if (p.kind != kind) {
            keep.push_back(p);
            continue;
        }
        float f = 0.0f;
        if (cudaEventSynchronize(p.b) != cudaSuccess || cudaEventElapsedTime(&f, p.a, p.b) != cudaSuccess)
            rc = LATEC_ERR_CUDA;
        sum += f;
        n++;
        g_kt_free.push_back(p);
    }
    g_kt_pairs.swap(keep);
    *ms = sum;
    *launches = n;
    return rc;
}

const char* latec_version(void) { return "latec_b200 0.1 (sm_100a)"; }

uint64_t latec_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int latec_plan_create(const uint32_t* shape, int32_t ndim, int32_t levels, int32_t anchor_stride,
                      int32_t anchor_block, latec_plan** out) {
    if (!shape || !out) return LATEC_ERR_ARG;
    latec_plan* p = new (std::nothrow) latec_plan();
    if (!p) return LATEC_ERR_INTERNAL;
    const int rc = build_plan(*p, shape, ndim, levels, anchor_stride, anchor_block);
    if (rc) {
        delete p;
        return rc;
    }
    *out = p;
    return LATEC_OK;
}

int latec_plan_destroy(latec_plan* plan) {
    delete plan;
    return LATEC_OK;
}

int latec_plan_num_stages(const latec_plan* plan) {
    return plan ? (int)plan->stages.size() : LATEC_ERR_ARG;
}

int latec_plan_stage_info(const latec_plan* plan, int32_t stage, uint64_t* n_points,
                          int32_t* stride, int32_t* weight, int32_t* axis) {
    if (!plan || stage < 0 || stage >= (int)plan->stages.size()) return LATEC_ERR_ARG;
    const StageDesc& d = plan->stages[stage];
    if (n_points) *n_points = d.n;
    if (stride) *stride = d.s;
    if (weight) *weight = d.weight;
    if (axis) *axis = d.axis;
    return LATEC_OK;
}

int latec_plan_stage_flat(const latec_plan* plan, int32_t stage, uint64_t first, uint64_t count,
                          int64_t* out_flat) {
    if (!plan || stage < 0 || stage >= (int)plan->stages.size() || (count && !out_flat))
        return LATEC_ERR_ARG;
    const StageDesc& d = plan->stages[stage];
    if (first + count > d.n) return LATEC_ERR_ARG;
    int32_t coord[MAXD];
    for (uint64_t i = 0; i < count; i++) out_flat[i] = stage_point(d, (uint32_t)(first + i), coord);
    return LATEC_OK;
}

uint64_t latec_stage_workspace_bytes(const latec_plan* plan, int32_t channels, int32_t dtype) {
    if (!plan || channels < 1) return 0;
    uint64_t m, t;
    plan_sizes(plan, channels, &m, &t);
    return stage_ws(m, t, (int)plan->stages.size(), elem_of(dtype), nullptr, nullptr);
}

uint64_t latec_flat_workspace_bytes(uint64_t items, int32_t dtype) {
    return stage_ws(items, 0, 1, elem_of(dtype), nullptr, nullptr);
}

int latec_encode_stages(const latec_plan* plan, const latec_quant_params* prm,
                        const double* stage_eb, const void* x, void* recon, uint16_t* codes,
                        void* outliers, latec_stage_stats* stats, uint32_t* hist_seg,
                        uint32_t* hist_total, void* workspace, uint64_t workspace_bytes,
                        void* stream) {
    if (!plan || !valid_params(prm) || !stage_eb || !x || !recon || !codes || !outliers ||
        !stats || !hist_seg || !hist_total)
        return LATEC_ERR_ARG;
    const int C = prm->channels, elem = elem_of(prm->dtype);
    const uint64_t need = latec_stage_workspace_bytes(plan, C, prm->dtype);
    if (!workspace || workspace_bytes < need) return LATEC_ERR_WORKSPACE;
    uint64_t m, tiles_all;
    plan_sizes(plan, C, &m, &tiles_all);
    StageWs w;
    stage_ws(m, tiles_all, (int)plan->stages.size(), elem, &w, workspace);
    cudaStream_t st = (cudaStream_t)stream;
    const int ns = (int)plan->stages.size();
    uint64_t total_segs = 0;
    for (auto& d : plan->stages) total_segs += n_segments((uint64_t)d.n * C);
    if (cudaMemsetAsync(stats, 0, sizeof(latec_stage_stats) * ns, st) != cudaSuccess ||
        cudaMemsetAsync(hist_seg, 0, sizeof(uint32_t) * HBINS * total_segs, st) != cudaSuccess ||
        cudaMemsetAsync(hist_total, 0, sizeof(uint32_t) * 65536ull * ns, st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    uint64_t off = 0, seg = 0;
    const int tmode = g_tile_mode.load();
    // per-stage launches read only points of earlier stages and write every
    // point; the fused levels stage whole planes of the canvas
    if (tmode && cudaMemsetAsync(recon, 0, plan->points * C * elem, st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    for (int t = 0; t < ns; t++) {
        if (tile_level_at(plan, t, tmode)) {
            // the level's five stages in one fused launch, then per stage the
            // statistics / tile-offset tail and the outlier compaction
            TileLevel L;
            uint32_t grid;
            if (!tile_level_init(plan, prm, stage_eb, t, C, codes, off, L, &grid))
                return LATEC_ERR_ARG;
            L.tma = tile_tma_ok(L, elem, x, recon) ? 1 : 0;
            TailArgs ta;
            std::memset(&ta, 0, sizeof(ta));
            uint64_t stg = 0, o = off, sg = seg;
            uint32_t tl = 0;
            for (int j = 0; j < TILE_STAGES; j++) {
                TileStage& S = L.st[j];
                const uint64_t items = (uint64_t)S.n * C;
                S.staging = (uint8_t*)w.staging + stg * elem;
                S.tile_cnt = w.tile_cnt + tl;
                S.hist_total = hist_total + 65536ull * (t + j);
                S.hist_seg = hist_seg + (uint64_t)HBINS * sg;
                S.partials = w.partials + (uint64_t)j * grid * 5;
                S.acc = (StageAcc*)(stats + t + j);
                ta.s[j] = TailStage{S.partials, grid, n_tiles(items), S.tile_cnt, w.tile_off + tl,
                                    S.acc};
                stg += items;
                o += items;
                sg += n_segments(items);
                tl += n_tiles(items);
            }
            if (tl && cudaMemsetAsync(w.tile_cnt, 0, sizeof(uint32_t) * tl, st) != cudaSuccess)
                return LATEC_ERR_CUDA;
            const int ki = kt_start(plan->stages[t].s == 1 ? 0 : 4, st);
            int rc = launch_tile_level_encode(L, prm->dtype, prm->order ? 1 : 0, grid, x, recon, st);
            kt_stop(ki, st);
            if (!rc) rc = launch_stage_tails(ta, TILE_STAGES, st);
            for (int j = 0; j < TILE_STAGES && !rc; j++) {
                const uint64_t items = (uint64_t)L.st[j].n * C;
                rc = launch_compact(L.st[j].codes, items, L.st[j].staging, elem, ta.s[j].tile_cnt,
                                    ta.s[j].tile_off, (uint8_t*)outliers + off * elem, st);
                off += items;
                seg += n_segments(items);
            }
            if (rc) return rc;
            t += TILE_STAGES - 1;
            continue;
        }
        const StageDesc& d = plan->stages[t];
        const uint64_t items = (uint64_t)d.n * C;
        QParams q;
        if (!make_q(prm, stage_eb[t], plan->points, q)) return LATEC_ERR_ARG;
        StageAcc* acc = (StageAcc*)(stats + t);
        // the pass's last CTA reduces the statistics and scans the tile counts
        int rc = launch_interp_quant(d, q, prm->dtype, t == 0, x, recon, codes + off, w.staging,
                                     w.tile_cnt, w.tile_off, hist_total + 65536ull * t,
                                     hist_seg + (uint64_t)HBINS * seg, acc, w.partials, st);
        if (!rc)
            rc = launch_compact(codes + off, items, w.staging, elem, w.tile_cnt, w.tile_off,
                                (uint8_t*)outliers + off * elem, st);
        if (rc) return rc;
        off += items;
        seg += n_segments(items);
    }
    return LATEC_OK;
}

int latec_interp_predict_stage(const latec_plan* plan, int32_t stage,
                               const latec_quant_params* prm, const void* recon, void* pred,
                               void* stream) {
    if (!plan || !valid_params(prm) || stage < 1 || stage >= (int)plan->stages.size() || !recon ||
        !pred)
        return LATEC_ERR_ARG;
    QParams q;
    make_q(prm, 1.0, plan->points, q);
    return launch_interp_predict(plan->stages[stage], q, prm->dtype, recon, pred,
                                 (cudaStream_t)stream);
}

int latec_quantize(const latec_quant_params* prm, double eb, uint64_t items, const void* x,
                   const void* pred, uint16_t* codes, void* recon_out, void* outliers,
                   latec_stage_stats* stats, uint32_t* hist_seg, uint32_t* hist_total,
                   void* workspace, uint64_t workspace_bytes, void* stream) {
    if (!valid_params(prm) || (items && (!x || !pred || !codes || !recon_out || !outliers)) ||
        !stats || !hist_seg || !hist_total)
        return LATEC_ERR_ARG;
    const int elem = elem_of(prm->dtype);
    if (!workspace || workspace_bytes < latec_flat_workspace_bytes(items, prm->dtype))
        return LATEC_ERR_WORKSPACE;
    StageWs w;
    stage_ws(items, 0, 1, elem, &w, workspace);
    QParams q;
    if (!make_q(prm, eb, items, q)) return LATEC_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(stats, 0, sizeof(latec_stage_stats), st) != cudaSuccess ||
        cudaMemsetAsync(hist_seg, 0, sizeof(uint32_t) * HBINS * n_segments(items), st) !=
            cudaSuccess ||
        cudaMemsetAsync(hist_total, 0, sizeof(uint32_t) * 65536ull, st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    StageAcc* acc = (StageAcc*)stats;
    int rc = launch_quantize_flat(q, prm->dtype, items, x, pred, codes, w.staging, w.tile_cnt,
                                  w.tile_off, hist_total, hist_seg, acc, w.partials, recon_out, st);
    if (!rc)
        rc = launch_compact(codes, items, w.staging, elem, w.tile_cnt, w.tile_off, outliers, st);
    return rc;
}

uint64_t latec_dequantize_workspace_bytes(uint64_t items) {
    Carve c{nullptr};  // the layout latec_dequantize carves
    c.take<DecStage>(1);
    c.take<uint32_t>((uint64_t)n_tiles(items) + 1);
    c.take<uint32_t>((uint64_t)n_tiles(items) + 1);
    return c.off;
}

int latec_dequantize(const latec_quant_params* prm, double eb, uint64_t items, const void* pred,
                     const uint16_t* codes, const void* outliers, uint32_t n_out, void* recon_out,
                     uint32_t* err, void* workspace, uint64_t workspace_bytes, void* stream) {
    if (!valid_params(prm) || !err || (items && (!pred || !codes || !recon_out)) ||
        (n_out && !outliers))
        return LATEC_ERR_ARG;
    if (!items) return LATEC_OK;
    if (!workspace || workspace_bytes < latec_dequantize_workspace_bytes(items))
        return LATEC_ERR_WORKSPACE;
    QParams q;
    if (!make_q(prm, eb, items, q)) return LATEC_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    Carve c{(uint8_t*)workspace};
    DecStage* ds = c.take<DecStage>(1);
    const uint32_t tiles = n_tiles(items);
    uint32_t* tile_cnt = c.take<uint32_t>(tiles + 1);
    uint32_t* tile_off = c.take<uint32_t>(tiles + 1);
    DecStage h{codes, err, items, 0, n_out};
    if (cudaMemcpyAsync(ds, &h, sizeof(h), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(tile_cnt, 0, sizeof(uint32_t) * tiles, st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    int rc = launch_count_zeros_all(ds, 1, tiles, tile_cnt, st);
    if (!rc) rc = launch_tile_offsets_all(ds, 1, tile_cnt, tile_off, st);
    if (!rc)
        rc = launch_dequant_flat(q, prm->dtype, items, pred, codes, outliers, tile_cnt, tile_off,
                                 n_out, recon_out, err, st);
    return rc;
}

int latec_decode_stages(const latec_plan* plan, const latec_quant_params* prm,
                        const double* stage_eb, const uint16_t* codes, const void* outliers,
                        const uint64_t* out_off, const uint32_t* n_out, void* recon,
                        uint32_t* err, void* workspace, uint64_t workspace_bytes, void* stream) {
    if (!plan || !valid_params(prm) || !stage_eb || !codes || !out_off || !n_out || !recon || !err)
        return LATEC_ERR_ARG;
    const int C = prm->channels;
    if (!workspace || workspace_bytes < latec_stage_workspace_bytes(plan, C, prm->dtype))
        return LATEC_ERR_WORKSPACE;
    uint64_t m, tiles_all;
    plan_sizes(plan, C, &m, &tiles_all);
    const int ns = (int)plan->stages.size();
    StageWs w;
    stage_ws(m, tiles_all, ns, elem_of(prm->dtype), &w, workspace);
    cudaStream_t st = (cudaStream_t)stream;
    // all stages' outlier tiles in two launches
    std::vector<DecStage> ds(ns);
    std::vector<uint64_t> coff(ns);  // first code of each stage
    uint64_t off = 0;
    uint32_t tile0 = 0;
    for (int t = 0; t < ns; t++) {
        const uint64_t items = (uint64_t)plan->stages[t].n * C;
        ds[t] = DecStage{codes + off, err, items, tile0, n_out[t]};
        coff[t] = off;
        off += items;
        tile0 += n_tiles(items);
    }
    if (cudaMemcpyAsync(w.dec, ds.data(), sizeof(DecStage) * ns, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
        return LATEC_ERR_CUDA;
    int rc = launch_count_zeros_all(w.dec, ns, tile0, w.tile_cnt, st);
    if (!rc) rc = launch_tile_offsets_all(w.dec, ns, w.tile_cnt, w.tile_off, st);
    if (rc) return rc;
    const int mode = g_level_mode.load();
    const int tmode = g_tile_mode.load();
    if ((mode || tmode) &&
        cudaMemsetAsync(recon, 0, plan->points * C * elem_of(prm->dtype), st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    int t = 0;
    while (t < ns) {
        if (tile_level_at(plan, t, tmode)) {
            // outliers of the level into the canvas, then the fused decode
            ScatterArgs sa;
            std::memset(&sa, 0, sizeof(sa));
            uint32_t tiles = 0;
            for (int j = 0; j < TILE_STAGES; j++) {
                const DecStage& dj = ds[t + j];
                if (!n_out[t + j] || !dj.items || !outliers) continue;
                ScatterStage& S = sa.s[sa.n++];
                S.d = plan->stages[t + j];
                S.codes = codes + coff[t + j];
                S.outliers = (const uint8_t*)outliers + out_off[t + j];
                S.tile_cnt = w.tile_cnt + dj.tile0;
                S.tile_off = w.tile_off + dj.tile0;
                S.items = dj.items;
                S.n_out = n_out[t + j];
                S.tile0 = tiles;
                tiles += n_tiles(dj.items);
            }
            sa.channels = C;
            sa.points = plan->points;
            rc = launch_scatter_outliers(sa, prm->dtype, tiles, recon, err, st);
            if (rc) return rc;
            TileLevel L;
            uint32_t grid;
            if (!tile_level_init(plan, prm, stage_eb, t, C, const_cast<uint16_t*>(codes),
                                 coff[t], L, &grid))
                return LATEC_ERR_ARG;
            L.tma = tile_tma_ok(L, elem_of(prm->dtype), recon, recon) ? 1 : 0;
            const int ki = kt_start(plan->stages[t].s == 1 ? 1 : 5, st);
            rc = launch_tile_level_decode(L, prm->dtype, prm->order ? 1 : 0, grid, recon, err, st);
            kt_stop(ki, st);
            if (rc) return rc;
            t += TILE_STAGES;
            continue;
        }
        // a level: consecutive stages of one stride (the anchors stand alone)
        int t1 = t + 1;
        if (t > 0)
            while (t1 < ns && plan->stages[t1].s == plan->stages[t].s) t1++;
        LevelBuild L;
        uint32_t tps[LVL_MAX_STAGES];
        if (build_level(plan, t, t1, C, elem_of(prm->dtype), mode, w.lvl_items_cap, L, tps)) {
            const int nl = t1 - t;
            L.st.resize(nl);
            for (int j = 0; j < nl; j++) {
                LvlStage& ls = L.st[j];
                memset(&ls, 0, sizeof(ls));
                ls.d = plan->stages[t + j];
                if (!make_q(prm, stage_eb[t + j], plan->points, ls.q)) return LATEC_ERR_ARG;
                ls.codes = codes + coff[t + j];
                ls.outliers = outliers ? (const uint8_t*)outliers + out_off[t + j] : nullptr;
                ls.tile_cnt = w.tile_cnt + ds[t + j].tile0;
                ls.tile_off = w.tile_off + ds[t + j].tile0;
                ls.n_out = n_out[t + j];
            }
            if (cudaMemcpyAsync(w.lvl_stages, L.st.data(), sizeof(LvlStage) * nl,
                                cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaMemcpyAsync(w.lvl_bands, L.bands.data(), sizeof(LvlBand) * L.bands.size(),
                                cudaMemcpyHostToDevice, st) != cudaSuccess ||
                (L.deps.size() &&
                 cudaMemcpyAsync(w.lvl_deps, L.deps.data(), sizeof(LvlDep) * L.deps.size(),
                                 cudaMemcpyHostToDevice, st) != cudaSuccess) ||
                cudaMemcpyAsync(w.lvl_items, L.items.data(), sizeof(LvlItem) * L.items.size(),
                                cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaMemsetAsync(w.lvl_ctr, 0, sizeof(uint32_t) * (L.bands.size() + 1), st) !=
                    cudaSuccess)
                return LATEC_ERR_CUDA;
            rc = launch_level_dequant(prm->dtype, plan->ndim, prm->order ? 1 : 0, w.lvl_stages,
                                      w.lvl_bands, w.lvl_deps, w.lvl_items,
                                      (uint32_t)L.items.size(), w.lvl_ctr, recon, err, st);
            if (rc) return rc;
            t = t1;
            continue;
        }
        for (; t < t1; t++) {
            const StageDesc& d = plan->stages[t];
            if (!ds[t].items) continue;
            QParams q;
            if (!make_q(prm, stage_eb[t], plan->points, q)) return LATEC_ERR_ARG;
            rc = launch_interp_dequant(d, q, prm->dtype, t == 0, codes + coff[t],
                                       outliers ? (const uint8_t*)outliers + out_off[t] : nullptr,
                                       w.tile_cnt + ds[t].tile0, w.tile_off + ds[t].tile0,
                                       n_out[t], recon, err, st);
            if (rc) return rc;
        }
    }
    return LATEC_OK;
}

// Launch tables of latec_encode_stages_many (see the header).
static int encode_many_build(const latec_encode_job* jobs, int n, HostTable& T,
                             std::vector<ManyLaunch>& L) {
    if (n < 0 || (n && !jobs)) return LATEC_ERR_ARG;
    std::vector<StageWs> ws(n);
    std::vector<const StageDesc*> dev(n);
    std::vector<uint64_t> off(n, 0), seg(n, 0);
    std::vector<ZeroRange> zr;
    int max_ns = 0;
    for (int j = 0; j < n; j++) {
        const latec_encode_job& J = jobs[j];
        const latec_plan* plan = J.plan;
        if (!plan || !valid_params(&J.prm) || !J.stage_eb || !J.x || !J.recon || !J.codes ||
            !J.outliers || !J.stats || !J.hist_seg || !J.hist_total)
            return LATEC_ERR_ARG;
        const int C = J.prm.channels, ns = (int)plan->stages.size();
        if (!J.workspace ||
            J.workspace_bytes < latec_stage_workspace_bytes(plan, C, J.prm.dtype))
            return LATEC_ERR_WORKSPACE;
        uint64_t m, tiles_all;
        plan_sizes(plan, C, &m, &tiles_all);
        stage_ws(m, tiles_all, ns, elem_of(J.prm.dtype), &ws[j], J.workspace);
        if (!(dev[j] = plan_dev_stages(plan))) return LATEC_ERR_CUDA;
        uint64_t total_segs = 0;
        for (auto& d : plan->stages) total_segs += n_segments((uint64_t)d.n * C);
        zr.push_back(ZeroRange{(uint32_t*)J.stats, sizeof(latec_stage_stats) * ns / 4});
        zr.push_back(ZeroRange{J.hist_seg, (uint64_t)HBINS * total_segs});
        zr.push_back(ZeroRange{J.hist_total, 65536ull * ns});
        max_ns = ns > max_ns ? ns : max_ns;
    }
    add_zero_launch(T, L, zr);
    for (int t = 0; t < max_ns; t++) {
        std::vector<ManyJob> step;
        std::vector<int> keys;
        zr.clear();
        for (int j = 0; j < n; j++) {
            const latec_encode_job& J = jobs[j];
            if (t >= (int)J.plan->stages.size()) continue;
            const StageDesc& d = J.plan->stages[t];
            const int elem = elem_of(J.prm.dtype);
            const uint64_t items = (uint64_t)d.n * J.prm.channels;
            const uint64_t o = off[j], sg = seg[j];
            off[j] += items;
            seg[j] += n_segments(items);
            if (!items) continue;
            ManyJob mj;
            std::memset(&mj, 0, sizeof(mj));
            if (!make_q(&J.prm, J.stage_eb[t], J.plan->points, mj.q)) return LATEC_ERR_ARG;
            const uint32_t cap = J.max_ctas && J.max_ctas < (uint32_t)MAX_BLOCKS
                                     ? J.max_ctas : (uint32_t)MAX_BLOCKS;
            const StageWs& w = ws[j];
            mj.d = dev[j] + t;
            mj.x = J.x;
            mj.recon = J.recon;
            mj.codes = J.codes + o;
            mj.staging = w.staging;
            mj.tile_cnt = w.tile_cnt;
            mj.tile_off = w.tile_off;
            mj.hist_total = J.hist_total + 65536ull * t;
            mj.hist_seg = J.hist_seg + (uint64_t)HBINS * sg;
            mj.acc = (StageAcc*)(J.stats + t);
            mj.partials = w.partials;
            mj.out = (uint8_t*)J.outliers + o * elem;
            mj.items = items;
            mj.gpb = encode_grid(items, cap, &mj.blocks);
            mj.is_anchor = t == 0 ? 1u : 0u;
            mj.elem = (uint32_t)elem;
            const uint32_t tiles = n_tiles(items);
            mj.cblocks = tiles < 592u ? tiles : 592u;
            zr.push_back(ZeroRange{w.tile_cnt, tiles});
            step.push_back(mj);
            keys.push_back(many_key(J.prm.dtype, d, J.prm.order));
        }
        add_zero_launch(T, L, zr);
        add_step_launches(T, L, step, keys, 1, true);
    }
    return LATEC_OK;
}

static int run_many(const std::vector<ManyLaunch>& L, const HostTable& T, uint64_t upload,
                    void* table, cudaStream_t st) {
    if (upload && cudaMemcpyAsync(table, T.buf.data(), upload, cudaMemcpyHostToDevice, st) !=
                      cudaSuccess)
        return LATEC_ERR_CUDA;
    uint8_t* tb = (uint8_t*)table;
    for (const ManyLaunch& l : L) {
        const uint32_t* first = (const uint32_t*)(tb + l.first);
        int rc = LATEC_OK;
        const int k = l.key, dtype = ((k >> 5) & 1) ? LATEC_F64 : LATEC_F32;
        const int nd = (k >> 2) & 7, kind = (k >> 1) & 1, cubic = k & 1;
        switch (l.op) {
            case 0:
                rc = launch_zero_many((const ZeroRange*)(tb + l.recs), first, l.n, l.ctas, st);
                break;
            case 1:
                rc = launch_quant_many(dtype, nd, kind, cubic, (const ManyJob*)(tb + l.recs),
                                       first, l.n, l.ctas, st);
                break;
            case 2:
                rc = launch_compact_many((const ManyJob*)(tb + l.recs), first, l.n, l.ctas, st);
                break;
            case 3:
                rc = launch_dequant_many(dtype, nd, kind, cubic, (const ManyJob*)(tb + l.recs),
                                         first, l.n, l.ctas, st);
                break;
            default:
                rc = LATEC_ERR_INTERNAL;
        }
        if (rc) return rc;
    }
    return LATEC_OK;
}

uint64_t latec_encode_many_table_bytes(const latec_encode_job* jobs, int32_t n_jobs) {
    HostTable T;
    std::vector<ManyLaunch> L;
    if (encode_many_build(jobs, n_jobs, T, L)) return 0;
    return T.size() ? T.size() : 16;
}

int latec_encode_stages_many(const latec_encode_job* jobs, int32_t n_jobs, void* table,
                             uint64_t table_bytes, void* stream) {
    HostTable T;
    std::vector<ManyLaunch> L;
    const int rc = encode_many_build(jobs, n_jobs, T, L);
    if (rc) return rc;
    if (T.size() && (!table || table_bytes < T.size())) return LATEC_ERR_WORKSPACE;
    return run_many(L, T, T.buf.size(), table, (cudaStream_t)stream);
}

// Launch tables of latec_decode_stages_many: the all-stage outlier tile
// passes over every stage of every job (records at offset `dec`, the tile
// counts and offsets after the uploaded part), then the dequantize steps.
struct DecodeMany {
    uint64_t dec = 0;         // DecStage records
    uint32_t n_dec = 0;
    uint64_t tiles = 0;       // tiles of all stages
    uint64_t tile_cnt = 0;    // table offsets of the two tile arrays
    uint64_t tile_off = 0;
    uint64_t upload = 0;      // bytes uploaded (the records)
    uint64_t total = 0;       // table bytes
};

static int decode_many_build(const latec_decode_job* jobs, int n, HostTable& T,
                             std::vector<ManyLaunch>& L, DecodeMany& D) {
    if (n < 0 || (n && !jobs)) return LATEC_ERR_ARG;
    std::vector<DecStage> ds;
    std::vector<std::vector<uint64_t>> coff(n);
    std::vector<std::vector<uint32_t>> tile0(n);
    std::vector<const StageDesc*> dev(n);
    int max_ns = 0;
    uint64_t tiles = 0;
    for (int j = 0; j < n; j++) {
        const latec_decode_job& J = jobs[j];
        const latec_plan* plan = J.plan;
        if (!plan || !valid_params(&J.prm) || !J.stage_eb || !J.codes || !J.out_off ||
            !J.n_out || !J.recon || !J.err)
            return LATEC_ERR_ARG;
        if (!(dev[j] = plan_dev_stages(plan))) return LATEC_ERR_CUDA;
        const int ns = (int)plan->stages.size();
        max_ns = ns > max_ns ? ns : max_ns;
        uint64_t off = 0;
        for (int t = 0; t < ns; t++) {
            const uint64_t items = (uint64_t)plan->stages[t].n * J.prm.channels;
            if (J.n_out[t] && !J.outliers) return LATEC_ERR_ARG;
            coff[j].push_back(off);
            tile0[j].push_back((uint32_t)tiles);
            ds.push_back(DecStage{J.codes + off, J.err, items, (uint32_t)tiles, J.n_out[t]});
            off += items;
            tiles += n_tiles(items);
            if (tiles >= (1ull << 32)) return LATEC_ERR_TOO_LARGE;
        }
    }
    D.dec = T.put(ds.data(), ds.size());
    D.n_dec = (uint32_t)ds.size();
    D.tiles = tiles;
    for (int t = 0; t < max_ns; t++) {
        std::vector<ManyJob> step;
        std::vector<int> keys;
        for (int j = 0; j < n; j++) {
            const latec_decode_job& J = jobs[j];
            if (t >= (int)J.plan->stages.size()) continue;
            const StageDesc& d = J.plan->stages[t];
            const uint64_t items = (uint64_t)d.n * J.prm.channels;
            if (!items) continue;
            ManyJob mj;
            std::memset(&mj, 0, sizeof(mj));
            if (!make_q(&J.prm, J.stage_eb[t], J.plan->points, mj.q)) return LATEC_ERR_ARG;
            mj.d = dev[j] + t;
            mj.recon = J.recon;
            mj.codes_in = J.codes + coff[j][t];
            mj.outliers = J.outliers ? (const uint8_t*)J.outliers + J.out_off[t] : nullptr;
            mj.err = J.err;
            mj.items = items;
            mj.blocks = n_tiles(items);
            mj.is_anchor = t == 0 ? 1u : 0u;
            mj.elem = (uint32_t)elem_of(J.prm.dtype);
            mj.n_out = J.n_out[t];
            // tile arrays: patched to device addresses once the table is placed
            mj.tile_cnt = (uint32_t*)(uintptr_t)tile0[j][t];
            step.push_back(mj);
            keys.push_back(many_key(J.prm.dtype, d, J.prm.order));
        }
        add_step_launches(T, L, step, keys, 3, false);
    }
    D.upload = T.buf.size();
    D.tile_cnt = T.size();
    D.tile_off = D.tile_cnt + ((tiles + 1) * 4 + 15) / 16 * 16;
    D.total = D.tile_off + ((tiles + 1) * 4 + 15) / 16 * 16;
    return LATEC_OK;
}

uint64_t latec_decode_many_table_bytes(const latec_decode_job* jobs, int32_t n_jobs) {
    HostTable T;
    std::vector<ManyLaunch> L;
    DecodeMany D;
    if (decode_many_build(jobs, n_jobs, T, L, D)) return 0;
    return D.total ? D.total : 16;
}

int latec_decode_stages_many(const latec_decode_job* jobs, int32_t n_jobs, void* table,
                             uint64_t table_bytes, void* stream) {
    HostTable T;
    std::vector<ManyLaunch> L;
    DecodeMany D;
    const int rc = decode_many_build(jobs, n_jobs, T, L, D);
    if (rc) return rc;
    if (!n_jobs || !D.n_dec) return LATEC_OK;
    if (!table || table_bytes < D.total) return LATEC_ERR_WORKSPACE;
    uint8_t* tb = (uint8_t*)table;
    uint32_t* tile_cnt = (uint32_t*)(tb + D.tile_cnt);
    uint32_t* tile_off = (uint32_t*)(tb + D.tile_off);
    // the dequantize records point at their stage's slice of the tile arrays
    for (const ManyLaunch& l : L) {
        ManyJob* mj = (ManyJob*)(T.buf.data() + l.recs);
        for (uint32_t k = 0; k < l.n; k++) {
            const uint64_t t0 = (uint64_t)(uintptr_t)mj[k].tile_cnt;
            mj[k].tile_cnt = tile_cnt + t0;
            mj[k].tile_off = tile_off + t0;
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemcpyAsync(tb, T.buf.data(), D.upload, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    const DecStage* dec = (const DecStage*)(tb + D.dec);
    int r = launch_count_zeros_all(dec, (int)D.n_dec, (uint32_t)D.tiles, tile_cnt, st);
    if (!r) r = launch_tile_offsets_all(dec, (int)D.n_dec, tile_cnt, tile_off, st);
    if (!r) r = run_many(L, T, 0, table, st);
    return r;
}

int latec_rans_build_tables(const uint32_t* cdf_rows, int32_t alphabet, int32_t rows, void* enc,
                            uint16_t* bucket, void* stream) {
    if (!cdf_rows || alphabet < 2 || alphabet > 65536 || rows < 1) return LATEC_ERR_ARG;
    return launch_build_tables(cdf_rows, alphabet, rows, (EncSym*)enc, bucket,
                               (cudaStream_t)stream);
}

static uint64_t rans_layout(latec_rans_stage* s, int n, uint64_t* scratch_words,
                            uint32_t* total_chunks) {
    uint64_t sw = 0;
    uint32_t chunks = 0;
    for (int t = 0; t < n; t++) {
        latec_rans_stage& d = s[t];
        d.scratch_off = sw;
        d.chunk0 = chunks;
        if (d.mode == LATEC_RANS_LANES) {
            const uint64_t per = 32ull * (d.K ? d.K : 1);
            d.n_chunks = d.n ? (uint32_t)((d.n + per - 1) / per) : 0;
            chunks += d.n_chunks;
            sw += (uint64_t)d.n_chunks * (64 + per);
        } else {
            d.n_chunks = 0;
            sw += (uint64_t)d.n + 2;
        }
        sw = (sw + 63) & ~63ull;
    }
    *scratch_words = sw;
    *total_chunks = chunks;
    Carve c{nullptr};
    c.take<RansStageDesc>(n);
    c.take<uint32_t>(sw);
    c.take<uint32_t>(chunks + 1);
    c.take<uint32_t>(chunks + 1);
    c.take<uint32_t>(n + 1);
    return c.off;
}

uint64_t latec_rans_encode_workspace_bytes(latec_rans_stage* stages, int32_t n_stages) {
    if (!stages || n_stages < 1) return 0;
    uint64_t sw;
    uint32_t tc;
    return rans_layout(stages, n_stages, &sw, &tc);
}

int latec_rans_encode(latec_rans_stage* stages, int32_t n_stages, const uint16_t* codes,
                      const uint8_t* levels, const latec_stage_stats* stats,
                      const void* outliers, int32_t elem, uint8_t* payload, uint64_t payload_cap,
                      uint64_t* payload_len, uint32_t* err, void* workspace,
                      uint64_t workspace_bytes, void* stream) {
    if (!stages || n_stages < 1 || !codes || !stats || !payload || !payload_len || !err ||
        (elem != 4 && elem != 8))
        return LATEC_ERR_ARG;
    for (int t = 0; t < n_stages; t++) {
        const latec_rans_stage& d = stages[t];
        if (d.n && (!d.cdf || d.alphabet < 2 || d.alphabet > 65536 || d.kexp < 1 || d.kexp > 15))
            return LATEC_ERR_ARG;
        if (d.n && d.mode == LATEC_RANS_LANES && (!d.enc || d.K < 1)) return LATEC_ERR_ARG;
        if (d.per_point && !levels) return LATEC_ERR_ARG;
    }
    uint64_t sw;
    uint32_t tc;
    const uint64_t need = rans_layout(stages, n_stages, &sw, &tc);
    if (!workspace || workspace_bytes < need) return LATEC_ERR_WORKSPACE;
    Carve c{(uint8_t*)workspace};
    RansStageDesc* dst = c.take<RansStageDesc>(n_stages);
    uint32_t* scratch = c.take<uint32_t>(sw);
    uint32_t* chunk_words = c.take<uint32_t>(tc + 1);
    uint32_t* chunk_off = c.take<uint32_t>(tc + 1);
    uint32_t* stage_words = c.take<uint32_t>(n_stages + 1);
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemcpyAsync(dst, stages, sizeof(RansStageDesc) * n_stages, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
        return LATEC_ERR_CUDA;
    if (cudaMemsetAsync(stage_words, 0, sizeof(uint32_t) * (n_stages + 1), st) != cudaSuccess)
        return LATEC_ERR_CUDA;
    bool any_compat = false;
    for (int t = 0; t < n_stages; t++) any_compat |= stages[t].mode == LATEC_RANS_COMPAT;
    const int ki = kt_start(2, st);
    int rc = launch_lanes_encode(dst, n_stages, tc, codes, levels, scratch, chunk_words, err, st);
    kt_stop(ki, st);
    if (!rc && any_compat)
        rc = launch_stack_encode(dst, n_stages, codes, levels, scratch, stage_words, err, st);
    if (!rc)
        rc = launch_assemble(dst, n_stages, tc, scratch, chunk_words, chunk_off, scratch,
                             stage_words, (const StageAcc*)stats, (const uint8_t*)outliers, elem,
                             payload, payload_cap, payload_len, err, st);
    return rc;
}

uint64_t latec_rans_decode_workspace_bytes(int32_t n_stages) {
    Carve c{nullptr};
    c.take<RansStageDesc>(n_stages > 0 ? n_stages : 1);
    return c.off;
}

int latec_rans_decode(latec_rans_stage* stages, int32_t n_stages, uint32_t total_chunks,
                      const uint32_t* words, const uint64_t* chunk_range, const uint8_t* levels,
                      uint16_t* codes, uint32_t* err, void* workspace, uint64_t workspace_bytes,
                      void* stream) {
    if (!stages || n_stages < 1 || !codes || !err) return LATEC_ERR_ARG;
    if (!workspace || workspace_bytes < latec_rans_decode_workspace_bytes(n_stages))
        return LATEC_ERR_WORKSPACE;
    bool any_compat = false;
    for (int t = 0; t < n_stages; t++) {
        const latec_rans_stage& d = stages[t];
        if (d.n && (!d.cdf || !d.bucket || d.alphabet < 2 || d.alphabet > 65536)) return LATEC_ERR_ARG;
        if (d.per_point && !levels) return LATEC_ERR_ARG;
        any_compat |= d.mode == LATEC_RANS_COMPAT && d.n;
    }
    if (total_chunks && (!words || !chunk_range)) return LATEC_ERR_ARG;
    // One decoder CTA covers DEC_WARPS chunks of one stage: number the CTAs.
    RansStageDesc* host = (RansStageDesc*)stages;  // only block0 is written
    uint32_t blocks = 0, max_alpha = 0;
    for (int t = 0; t < n_stages; t++) {
        host[t].block0 = blocks;
        if (host[t].mode == LATEC_RANS_LANES && host[t].n) {
            blocks += (host[t].n_chunks + DEC_WARPS - 1) / DEC_WARPS;
            // only alphabets the kernel stages in shared memory size the allocation
            if (!host[t].per_point && host[t].alphabet <= (uint32_t)SMEM_ALPHA &&
                host[t].alphabet > max_alpha)
                max_alpha = host[t].alphabet;
        }
    }
    Carve c{(uint8_t*)workspace};
    RansStageDesc* dst = c.take<RansStageDesc>(n_stages);
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemcpyAsync(dst, stages, sizeof(RansStageDesc) * n_stages, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
        return LATEC_ERR_CUDA;
    const int ki = kt_start(3, st);
    int rc = launch_lanes_decode(dst, n_stages, total_chunks ? blocks : 0, (int)max_alpha, words,
                                 chunk_range, levels, codes, err, st);
    kt_stop(ki, st);
    if (!rc && any_compat) rc = launch_stack_decode(dst, n_stages, words, levels, codes, err, st);
    return rc;
}

}  // extern "C"
