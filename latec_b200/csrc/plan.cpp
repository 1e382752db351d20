// Host side of the dyadic stage schedule: closed-form stage sizes and the
// per-stage decode descriptors the kernels use. Follows the reference
// schedule (latec/levels.py:100-147 iter_stage_plan, 221-282 stage_counts,
// 469-574 stage_layouts / _fused_classes) without building any mask.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "latec_common.cuh"
#include "plan.h"

namespace latec {

static uint32_t slice_count(int64_t n, int64_t start, int64_t step) {
    return n <= start ? 0u : (uint32_t)((n - start + step - 1) / step);
}

int check_plan(const uint32_t* shape, int ndim, int levels, int anchor_stride,
               int anchor_block) {
    if (ndim < 1) return LATEC_ERR_ARG;
    if (ndim > MAXD) return LATEC_ERR_UNSUPPORTED;
    if (levels < 1 || levels > 30) return LATEC_ERR_ARG;
    if (anchor_stride < 2 || (anchor_stride & (anchor_stride - 1))) return LATEC_ERR_ARG;
    if (anchor_block < 1 || anchor_block > anchor_stride) return LATEC_ERR_ARG;
    if ((1ll << levels) < anchor_stride) return LATEC_ERR_ARG;
    for (int j = 0; j < ndim; j++)
        if (shape[j] == 0 || shape[j] > (1u << 30)) return LATEC_ERR_ARG;
    return LATEC_OK;
}

static void base_desc(StageDesc& d, const uint32_t* shape, int ndim, int astride, int ablock) {
    std::memset(&d, 0, sizeof(d));
    d.ndim = ndim;
    d.astride = astride;
    d.ablock = ablock;
    d.blk_div = make_fastdiv(1);
    int64_t g = 1;
    for (int j = ndim - 1; j >= 0; j--) {
        d.shape[j] = (int32_t)shape[j];
        d.gstride[j] = g;
        g *= shape[j];
    }
    for (int j = 0; j < MAXD; j++) {
        d.size_div[j] = make_fastdiv(1);
        for (int r = 0; r <= MAXD; r++) d.g_div[j][r] = make_fastdiv(1);
    }
}

static int log2u(uint64_t v) {
    int l = 0;
    while ((1ull << l) < v) l++;
    return l;
}

// Blocked anchors: the anchor stage is every anchor_block^ndim block of the
// anchor lattice, in C order (latec/levels.py:114-120).
static int blocked_anchors(StageDesc& d, int astride, int ablock) {
    uint64_t n = 1;
    d.kind = 2;
    d.step = astride;
    d.blk_div = make_fastdiv((uint32_t)ablock);
    for (int j = 0; j < d.ndim; j++) {
        const uint32_t nj = (uint32_t)d.shape[j];
        const uint32_t c = nj / astride * ablock + std::min<uint32_t>(nj % astride, ablock);
        d.size_div[j] = make_fastdiv(c ? c : 1);
        n *= c;
    }
    if (n > 0xFFFFFFFFull) return LATEC_ERR_UNSUPPORTED;
    d.n = d.n_full = (uint32_t)n;
    return LATEC_OK;
}

// The holes of a stage at level s (anchor-block points of its full set, which
// the anchor stage already coded): per axis and parity, the in-block positions
// of the progression parity * s + 2 s m, then their products over the axes.
static int stage_holes(StageDesc& d) {
    const int s = d.s, nd = d.ndim;
    d.lg2s = log2u(2ull * s);
    if (d.ablock <= 1 || d.n == 0) return LATEC_OK;
    const uint32_t per = d.astride / (2 * s) ? (uint32_t)(d.astride / (2 * s)) : 1u;
    for (int j = 0; j < nd; j++)
        for (int par = 0; par < 2; par++) {
            const int64_t first = (int64_t)par * s;
            uint32_t k = 0;
            if (d.ablock > first) k = (uint32_t)std::min<int64_t>(per, (d.ablock - first + 2 * s - 1) / (2 * s));
            d.h_lgp[j][par] = (uint32_t)log2u(per);
            d.h_k[j][par] = k;
            const uint64_t m_tot = slice_count(d.shape[j], first, 2 * s);
            d.h_tot[j][par] = block_count((uint32_t)m_tot, d.h_lgp[j][par], k);
        }
    uint64_t holes = 0;
    if (d.kind == 0) {
        d.h_suf[nd] = 1;
        for (int j = nd - 1; j >= 0; j--) {
            const int par = d.start[j] == s ? 1 : 0;
            d.h_suf[j] = d.h_suf[j + 1] * d.h_tot[j][par];
        }
        holes = d.h_suf[0];
    } else {
        for (int r = 0; r <= MAXD; r++) d.h_c[nd][r] = r == 0 ? 1u : 0u;
        for (int j = nd - 1; j >= 0; j--)
            for (int r = 0; r <= MAXD; r++)
                d.h_c[j][r] = d.h_tot[j][0] * d.h_c[j + 1][r] +
                              (r ? d.h_tot[j][1] * d.h_c[j + 1][r - 1] : 0u);
        holes = d.h_c[0][d.weight];
    }
    if (holes > d.n) return LATEC_ERR_INTERNAL;
    d.n_full = d.n;
    d.n = (uint32_t)(d.n - holes);
    d.holes = holes ? 1 : 0;
    return LATEC_OK;
}

static int single_class(StageDesc& d, const int32_t* starts, int step) {
    uint64_t n = 1;
    d.kind = 0;
    d.step = step;
    for (int j = 0; j < d.ndim; j++) {
        d.start[j] = starts[j];
        uint32_t c = slice_count(d.shape[j], starts[j], step);
        d.size_div[j] = make_fastdiv(c ? c : 1);
        n *= c;
    }
    if (n > 0xFFFFFFFFull) return LATEC_ERR_UNSUPPORTED;
    d.n = d.n_full = (uint32_t)n;
    return LATEC_OK;
}

static int fused(StageDesc& d, int s, int w) {
    const int nd = d.ndim;
    uint64_t cnt[MAXD][2];
    for (int j = 0; j < nd; j++) {
        cnt[j][0] = slice_count(d.shape[j], 0, 2 * s);
        cnt[j][1] = slice_count(d.shape[j], s, 2 * s);
    }
    // F[j][r]: stage points over axes j.. with r odd axes still to place.
    uint64_t F[MAXD + 1][MAXD + 2];
    std::memset(F, 0, sizeof(F));
    F[nd][0] = 1;
    for (int j = nd - 1; j >= 0; j--)
        for (int r = 0; r <= w; r++) {
            uint64_t odd = r ? F[j + 1][r - 1] : 0;
            F[j][r] = cnt[j][0] * F[j + 1][r] + cnt[j][1] * odd;
        }
    if (F[0][w] > 0xFFFFFFFFull) return LATEC_ERR_UNSUPPORTED;
    d.kind = 1;
    d.weight = w;
    d.n = d.n_full = (uint32_t)F[0][w];
    for (int j = 0; j < nd; j++)
        for (int r = 0; r <= w; r++) {
            uint64_t odd = r ? F[j + 1][r - 1] : 0;
            uint64_t g = F[j + 1][r] + odd;
            d.g_div[j][r] = make_fastdiv(g ? (uint32_t)g : 1u);
            d.f_even[j][r] = (uint32_t)F[j + 1][r];
        }
    return LATEC_OK;
}

int build_plan(Plan& p, const uint32_t* shape, int ndim, int levels, int anchor_stride,
               int anchor_block) {
    int rc = check_plan(shape, ndim, levels, anchor_stride, anchor_block);
    if (rc) return rc;
    p.ndim = ndim;
    p.levels = levels;
    p.anchor_stride = anchor_stride;
    p.anchor_block = anchor_block;
    p.points = 1;
    for (int j = 0; j < ndim; j++) {
        p.shape[j] = shape[j];
        p.points *= shape[j];
    }
    p.stages.clear();
    StageDesc d;
    int32_t starts[MAXD] = {0};
    base_desc(d, shape, ndim, anchor_stride, anchor_block);
    d.axis = -1;
    d.s = anchor_stride;
    if (anchor_block > 1) {
        if ((rc = blocked_anchors(d, anchor_stride, anchor_block))) return rc;
    } else if ((rc = single_class(d, starts, anchor_stride))) {
        return rc;
    }
    p.stages.push_back(d);
    int prev = -1;
    for (int k = 1; k <= levels; k++) {
        int s = anchor_stride >> k;
        if (s < 1) s = 1;
        bool repeat = s == prev;
        prev = s;
        for (int axis = 0; axis < ndim; axis++) {
            base_desc(d, shape, ndim, anchor_stride, anchor_block);
            d.axis = axis;
            d.weight = 1;
            d.s = s;
            for (int j = 0; j < ndim; j++) starts[j] = j == axis ? s : 0;
            if ((rc = single_class(d, starts, 2 * s))) return rc;
            if (repeat) d.n = d.n_full = 0;
            if ((rc = stage_holes(d))) return rc;
            p.stages.push_back(d);
        }
        for (int w = 2; w <= ndim; w++) {
            base_desc(d, shape, ndim, anchor_stride, anchor_block);
            d.axis = -2;
            d.s = s;
            if ((rc = fused(d, s, w))) return rc;
            if (repeat) d.n = d.n_full = 0;
            if ((rc = stage_holes(d))) return rc;
            p.stages.push_back(d);
        }
    }
    uint64_t total = 0;
    for (auto& st : p.stages) total += st.n;
    if (total != p.points) return LATEC_ERR_INTERNAL;  // schedule must partition the grid
    return LATEC_OK;
}

}  // namespace latec
