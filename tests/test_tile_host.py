"""Host-side checks of the fused tile-level kernels' index arithmetic
(latec_b200/csrc/tile_kernels.cu), restated in Python:

* the closed-form stage ranks (``Ranks::of``) equal the position of every
  point in its stage's C-order enumeration, i.e. the schedule's flat order
  (latec/levels.py:469-574);
* the unit order of a CTA (E(zs-2), E(zs), E(zs+2), then E(z+3), O(z)) with
  the class regions of the box computes every tap a point reads before the
  point, from coarse points or points of the same CTA, and owns every level
  point exactly once across the grid of tiles and axis-0 chunks (the halo
  argument: each dependency lies within three lattice steps on each axis).
"""

import itertools


def rank(stage, z, y, x, N):
    cye, cyo = (N[1] + 1) >> 1, N[1] >> 1
    cxe, cxo = (N[2] + 1) >> 1, N[2] >> 1
    a1, a2 = cyo * cxe + cye * cxo, cyo * cxo
    zh, yh, xh = z >> 1, y >> 1, x >> 1
    if stage == 0:
        return (zh * cye + yh) * cxe + xh
    if stage == 1:
        return (zh * cyo + yh) * cxe + xh
    if stage == 2:
        return (zh * cye + yh) * cxo + xh
    if stage == 4:
        return (zh * cyo + yh) * cxo + xh
    if not (z & 1):
        return zh * (a2 + a1) + yh * cxo + xh
    return (zh + 1) * a2 + zh * a1 + ((y + 1) >> 1) * cxo + yh * cxe + xh


def stage_of(z, y, x):
    w = (z & 1) + (y & 1) + (x & 1)
    if w == 0:
        return None
    if w == 1:
        return 0 if z & 1 else (1 if y & 1 else 2)
    return 3 if w == 2 else 4


def test_closed_form_ranks_follow_the_stage_order():
    for N in [(1, 1, 1), (2, 3, 5), (5, 4, 7), (9, 8, 6), (16, 17, 33), (3, 35, 67)]:
        count = [0] * 5
        for z, y, x in itertools.product(range(N[0]), range(N[1]), range(N[2])):
            s = stage_of(z, y, x)
            if s is None:
                continue
            assert rank(s, z, y, x, N) == count[s], (N, z, y, x, s)
            count[s] += 1


def _walk(N, TX, TY, zc, cubic):
    BX, BY = TX + 8, TY + 6
    HR, TR, HC, TC = (1, TY // 2 + 3), (4, TY // 2), (2, TX // 2 + 3), (5, TX // 2)
    owned = set()

    def taps(p, a):
        c, n = p[a], N[a]
        ds = [-1] + ([1] if c + 1 < n else []) + ([-3] if c >= 3 else []) + \
             ([3] if cubic and c + 3 < n else [])
        out = []
        for d in ds:
            q = list(p)
            q[a] += d
            out.append(tuple(q))
        return out

    for ch in range(-(-N[0] // zc)):
        zs, ze = ch * zc, min(ch * zc + zc, N[0])
        n_odd = len(range(zs + 1, ze, 2))
        for ty in range(-(-N[1] // TY)):
            for tx in range(-(-N[2] // TX)):
                x0, y0 = tx * TX, ty * TY
                have = set()
                for k in range(3 + 2 * n_odd):
                    if k < 3:
                        z, even = zs - 2 + 2 * k, True
                    else:
                        j, even = (k - 3) >> 1, ((k - 3) & 1) == 0
                        z = zs + 4 + 2 * j if even else zs + 1 + 2 * j
                    if not 0 <= z < N[0]:
                        continue
                    if even:  # coarse points of the box come from the canvas
                        for r in range(BY):
                            for b in range(BX):
                                y, x = y0 - 3 + r, x0 - 4 + b
                                if 0 <= y < N[1] and 0 <= x < N[2] and not (y | x) & 1:
                                    have.add((z, y, x))
                        phases = [[(HR, TC, (2,)), (TR, HC, (1,))], [(TR, TC, (1, 2))]]
                    else:
                        phases = [[(HR, HC, (0,))], [(HR, TC, (0, 2)), (TR, HC, (0, 1))],
                                  [(TR, TC, (0, 1, 2))]]
                    for phase in phases:
                        new = []
                        for (r0, nr), (b0, nc), axes in phase:
                            for i in range(nr):
                                for jj in range(nc):
                                    r, b = r0 + 2 * i, b0 + 2 * jj
                                    y, x = y0 - 3 + r, x0 - 4 + b
                                    if not (0 <= y < N[1] and 0 <= x < N[2]):
                                        continue
                                    p = (z, y, x)
                                    assert tuple(a for a in range(3) if p[a] & 1) == axes
                                    for a in axes:
                                        for q in taps(p, a):
                                            assert q in have, (p, q)
                                            if a:  # in-plane taps stay inside the box
                                                assert 0 <= q[1] - (y0 - 3) < BY
                                                assert 0 <= q[2] - (x0 - 4) < BX
                                    new.append(p)
                                    if zs <= z < ze and 3 <= r < 3 + TY and 4 <= b < 4 + TX:
                                        assert p not in owned
                                        owned.add(p)
                        have.update(new)
    for p in itertools.product(range(N[0]), range(N[1]), range(N[2])):
        if (p[0] | p[1] | p[2]) & 1:
            assert p in owned, p


def test_tile_walk_covers_and_respects_dependencies():
    for N, zc in [((9, 8, 6), 16), ((21, 40, 70), 16), ((35, 70, 66), 18), ((6, 33, 65), 4)]:
        for TX, TY in [(64, 32), (64, 16), (8, 4)]:
            for cubic in (True, False):
                _walk(N, TX, TY, zc, cubic)
