"""Oracle restatement of the dyadic stage schedule (reference ``latec/levels.py``).

Test infrastructure only (see ``oracle/__init__.py``).
"""

from __future__ import annotations

import itertools

import numpy as np


def check_plan(shape, levels, anchor_stride, anchor_block):
    """Parameter validation; ``latec/levels.py:54-76``."""
    shape = tuple(int(n) for n in shape)
    if len(shape) < 1:
        raise ValueError("shape must have at least one axis")
    if levels < 1:
        raise ValueError("levels must be >= 1")
    if anchor_stride < 2 or anchor_stride & (anchor_stride - 1):
        raise ValueError("anchor_stride must be a power of two >= 2")
    if not 1 <= anchor_block <= anchor_stride:
        raise ValueError("anchor_block must be in [1, anchor_stride]")
    if (1 << levels) < anchor_stride:
        raise ValueError("levels too small to densify to stride 1")
    return shape


def iter_plan(shape, levels, anchor_stride, anchor_block=1):
    """Yield ``(mask, stride, axes)`` per sub-stage; ``latec/levels.py:100-147``.

    Anchors first (every offset in ``[0, anchor_block)^ndim`` of the anchor
    lattice), then per level ``k`` (``s = max(stride >> k, 1)``): one weight-1
    sub-stage per axis, then one fused sub-stage per weight 2..ndim; the last
    sub-stage of the last level absorbs whatever is still uncovered.
    """
    shape = check_plan(shape, levels, anchor_stride, anchor_block)
    nd = len(shape)
    covered = np.zeros(shape, bool)
    anchor = np.zeros(shape, bool)
    for offs in itertools.product(range(anchor_block), repeat=nd):
        anchor[tuple(slice(o, None, anchor_stride) for o in offs)] = True
    covered |= anchor
    yield anchor, anchor_stride, ()
    for k in range(1, levels + 1):
        s = max(anchor_stride >> k, 1)

        def sl(odd_axes):
            return tuple(slice(s, None, 2 * s) if j in odd_axes else slice(0, None, 2 * s)
                         for j in range(nd))

        for axis in range(nd):
            m = np.zeros(shape, bool)
            m[sl((axis,))] = True
            m &= ~covered
            if k == levels and nd == 1:
                m |= ~covered
            covered |= m
            yield m, s, (axis,)
        for w in range(2, nd + 1):
            m = np.zeros(shape, bool)
            for axes in itertools.combinations(range(nd), w):
                m[sl(axes)] = True
            m &= ~covered
            if k == levels and w == nd:
                m |= ~covered
            covered |= m
            yield m, s, tuple(range(nd))


def stage_masks(shape, levels, anchor_stride, anchor_block=1):
    return [m for m, _, _ in iter_plan(shape, levels, anchor_stride, anchor_block)]


def n_stages(ndim, levels):
    """``latec/levels.py:211-213``."""
    return 1 + levels * (2 * ndim - 1)


def _cnt(n, start, step):
    """``latec/levels.py:216-218``."""
    return 0 if n <= start else (n - start + step - 1) // step


def stage_counts(shape, levels, anchor_stride, anchor_block=1):
    """Closed-form stage sizes; ``latec/levels.py:221-282``."""
    shape = check_plan(shape, levels, anchor_stride, anchor_block)
    nd = len(shape)
    if anchor_block != 1:
        return [int(m.sum()) for m in stage_masks(shape, levels, anchor_stride, anchor_block)]
    counts = [int(np.prod([_cnt(n, 0, anchor_stride) for n in shape]))]
    prev = None
    for k in range(1, levels + 1):
        s = max(anchor_stride >> k, 1)
        if s == prev:
            counts += [0] * (2 * nd - 1)
            continue
        prev = s
        for axis in range(nd):
            counts.append(int(np.prod([_cnt(n, s if j == axis else 0, 2 * s)
                                       for j, n in enumerate(shape)])))
        for w in range(2, nd + 1):
            counts.append(sum(int(np.prod([_cnt(n, s if j in ax else 0, 2 * s)
                                           for j, n in enumerate(shape)]))
                              for ax in itertools.combinations(range(nd), w)))
    counts[-1] += int(np.prod(shape)) - sum(counts)
    return counts


def stage_strides(ndim, levels, anchor_stride):
    """``latec/levels.py:297-326``."""
    out = [anchor_stride]
    for k in range(1, levels + 1):
        out += [max(anchor_stride >> k, 1)] * (2 * ndim - 1)
    return out


def stage_ebs(shape, levels, anchor_stride, anchor_block, eb, eb_ratio):
    """Per-stage bound ``eb * ratio ** log2(stride / finest)``; ``latec/levels.py:360-386``."""
    strides = stage_strides(len(shape), levels, anchor_stride)
    finest = min(strides)
    return [eb * eb_ratio ** np.log2(s / finest) for s in strides]


def point_levels(coords, levels, anchor_stride, anchor_block=1):
    """Level that reveals each point; ``latec/levels.py:329-357``."""
    coords = [np.asarray(c, np.int64) for c in coords]
    out = np.full(coords[0].shape, levels, np.int8)
    anchor = np.ones(coords[0].shape, bool)
    for c in coords:
        anchor &= (c % anchor_stride) < anchor_block
    for k in range(levels - 1, 0, -1):
        s = max(anchor_stride >> k, 1)
        on = np.ones(coords[0].shape, bool)
        for c in coords:
            on &= (c % s) == 0
        out[on] = k
    out[anchor] = 0
    return out


def fused_classes(shape, s, weight, low_axes=()):
    """Parity-class layouts of one fused sub-stage with the affine rank formula
    ``rank = offset + sum_j m_j * G_j``; ``latec/levels.py:469-512``."""
    nd = len(shape)
    lo, cnt = [], []
    for j, n in enumerate(shape):
        base = 2 * s if j in low_axes else 0
        lo.append((1 if j in low_axes else 0, 0))
        cnt.append((_cnt(n, base, 2 * s), _cnt(n, s, 2 * s)))
    F = [[0] * (weight + 1) for _ in range(nd + 1)]
    F[nd][0] = 1
    G = [[0] * (weight + 1) for _ in range(nd + 1)]
    for j in range(nd - 1, -1, -1):
        for r in range(weight + 1):
            odd = F[j + 1][r - 1] if r else 0
            F[j][r] = cnt[j][0] * F[j + 1][r] + cnt[j][1] * odd
            G[j][r] = F[j + 1][r] + odd
    out = []
    for combo in itertools.combinations(range(nd), weight):
        parity = tuple(1 if j in combo else 0 for j in range(nd))
        starts, sizes, strides = [], [], []
        offset, r = 0, weight
        for j, p in enumerate(parity):
            strides.append(G[j][r])
            starts.append(s if p else (2 * s if j in low_axes else 0))
            sizes.append(cnt[j][p])
            offset += lo[j][p] * G[j][r]
            if j in low_axes:
                if not p:
                    offset -= F[j + 1][r]
            elif p:
                offset += F[j + 1][r]
            r -= p
        out.append(dict(parity=parity, starts=tuple(starts), step=2 * s, sizes=tuple(sizes),
                        strides=tuple(strides), offset=offset))
    return out, F[0][weight]
