"""Host-side checks of the fused level kernels' index plan
(latec_b200/csrc/tile_kernels.cu), restated in Python and run on the CPU.

The emulation walks a kernel's work exactly as a CTA does -- items (column
tile x axis-0 chunk x channel), units (E(zs-2), E(zs), E(zs+2), then
(E(z+3), O(z)) per odd z), phase 0 (staging -> parity-split slots, stores of
the previous unit's planes), phases P1-P3 of warp tasks of 32 points of one
class -- with the same constants (tile 32 x 64 lattice points for float32,
16 x 64 for float64) and formulas. Every shared-memory position holds a label
of what is in it (an input value, a final reconstruction of a given lattice
point, or garbage), so it checks that

* every slot index and tap index stays inside its sub-array;
* every tap a point reads (for the taps its validity flags allow) holds the
  final reconstruction of exactly the lattice point the interpolation rule
  names, written in an earlier phase (never a same-phase write: no race);
* every point reads its own input value (x, or the canvas when decoding);
* the points marked owned cover every level point of the lattice exactly
  once, and their closed-form stage ranks equal their position in the
  stage's C-order enumeration, i.e. the schedule's flat order
  (latec/levels.py:469-574);
* every plane store writes only final values of owned planes, and a store
  never reads a slot the same phase overwrites;
* no warp gets more tasks in a phase than the decoder's code buffers hold.
"""

import numpy as np
import pytest

W1Y, W1X, W2E, W1Z, W2ZY, W2ZX, W3 = range(7)
# (plane odd, y odd, x odd, stage)
CLS = {W1Y: (0, 1, 0, 1), W1X: (0, 0, 1, 2), W2E: (0, 1, 1, 3), W1Z: (1, 0, 0, 0),
       W2ZY: (1, 1, 0, 3), W2ZX: (1, 0, 1, 3), W3: (1, 1, 1, 4)}
PHASES = [(W1Y, W1X, W1Z), (W2E, W2ZY, W2ZX), (W3,)]
LW, MAXT = 12, 8


class Geo:
    def __init__(self, elem):
        self.TX = 64
        self.TY = 32 if elem == 4 else 16
        self.NER = self.TY // 2 + 3
        self.NOR = self.TY // 2
        self.P = self.TX // 2 + 4
        self.EE, self.EO = 0, self.NER * self.P
        self.OE = 2 * self.NER * self.P
        self.OO = self.OE + self.NOR * self.P
        self.SLOT = 2 * (self.NER + self.NOR) * self.P

    def cls(self, c):
        zo, yo, xo, st = CLS[c]
        sub = (self.OO if xo else self.OE) if yo else (self.EO if xo else self.EE)
        nr = self.NOR if yo else self.NER
        c0, nc = (2, self.TX // 2) if xo else (1, self.TX // 2 + 3)
        return zo, yo, xo, st, sub, nr, c0, nc

    def sub_rows(self, sub):
        return self.NOR if sub in (self.OE, self.OO) else self.NER


def geometry(N, C, elem, n_sm=148):
    """tile_level_geometry (host side of the kernels)."""
    tx, ty = 64, (32 if elem == 4 else 16)
    tiles_x, tiles_y = -(-N[2] // tx), -(-N[1] // ty)
    cols = tiles_x * tiles_y * C
    slots = 2 * n_sm
    best, best_cost = 16, 1e300
    zc = 8
    while zc <= 128:
        items = cols * (-(-N[0] // zc))
        cost = -(-items // slots) * (zc + 3)
        if cost < best_cost * 0.999:
            best, best_cost = zc, cost
        if zc >= N[0]:
            break
        zc *= 2
    return tiles_x, tiles_y, best, -(-N[0] // best)


def rank(cl, z, y, x, N):
    """LvRanks::of."""
    cye, cyo, cxe, cxo = (N[1] + 1) >> 1, N[1] >> 1, (N[2] + 1) >> 1, N[2] >> 1
    a1, a2 = cyo * cxe + cye * cxo, cyo * cxo
    zh, yh, xh = z >> 1, y >> 1, x >> 1
    if cl == W1Z:
        return (zh * cye + yh) * cxe + xh
    if cl == W1Y:
        return (zh * cyo + yh) * cxe + xh
    if cl == W1X:
        return (zh * cye + yh) * cxo + xh
    if cl == W3:
        return (zh * cyo + yh) * cxo + xh
    if cl == W2E:
        return zh * (a2 + a1) + yh * cxo + xh
    return (zh + 1) * a2 + zh * a1 + ((y + 1) >> 1) * cxo + yh * cxe + xh


def stage_order(N):
    """Per stage: flat lattice index -> position in the stage's C order."""
    z, y, x = np.meshgrid(*[np.arange(n) for n in N], indexing="ij")
    w = (z & 1) + (y & 1) + (x & 1)
    st = np.full(N, -1)
    st[(w == 1) & (z & 1 == 1)] = 0
    st[(w == 1) & (y & 1 == 1)] = 1
    st[(w == 1) & (x & 1 == 1)] = 2
    st[w == 2] = 3
    st[w == 3] = 4
    out = []
    for s in range(5):
        flat = np.flatnonzero(st.reshape(-1) == s)
        m = np.full(int(np.prod(N)), -1, np.int64)
        m[flat] = np.arange(len(flat))
        out.append(m)
    return out, st


def tap_ok(c, n):
    return (1 if c + 1 < n else 0) | (2 if c >= 3 else 0) | (4 if c + 3 < n else 0)


def slot_of(z):
    return 4 + ((z >> 1) & 1) if z & 1 else ((z >> 1) & 3)


def emulate(N, C, elem):
    g = Geo(elem)
    tiles_x, tiles_y, zc, chunks = geometry(N, C, elem)
    order, stg = stage_order(N)
    nst = [int((order[s] >= 0).sum()) for s in range(5)]
    seen = [np.zeros(C * nst[s], np.int64) for s in range(5)]
    stored = np.zeros((C,) + tuple(N), np.int64)
    n_items = tiles_x * tiles_y * chunks * C
    for item in range(n_items):
        w = item
        ix = w % tiles_x
        w //= tiles_x
        iy = w % tiles_y
        w //= tiles_y
        ch = w % chunks
        c = w // chunks
        x0, y0, zs = ix * g.TX, iy * g.TY, ch * zc
        ze = min(zs + zc, N[0])
        # label of every slot position: None = garbage, ("x", z, y, x) input,
        # ("r", z, y, x) final reconstruction
        slots = [[None] * g.SLOT for _ in range(6)]

        def coords(sub, row, col):
            ey = sub in (g.EE, g.EO)
            ex = sub in (g.EE, g.OE)
            yy = y0 - 2 + 2 * row if ey else y0 + 1 + 2 * row
            xx = x0 - 4 + 2 * col if ex else x0 - 3 + 2 * col
            return yy, xx

        def inside(yy, xx):
            return 0 <= yy < N[1] and 0 <= xx < N[2]

        def transpose(z, even):
            s = slots[slot_of(z)]
            for sub in (g.EE, g.EO, g.OE, g.OO):
                for row in range(g.sub_rows(sub)):
                    for col in range(g.P):
                        yy, xx = coords(sub, row, col)
                        if not inside(yy, xx):
                            lab = ("zero",)
                        elif even and sub == g.EE:
                            lab = ("r", z, yy, xx)  # coarse point (canvas)
                        else:
                            lab = ("x", z, yy, xx)
                        s[sub + row * g.P + col] = lab

        def store(z):
            s = slots[slot_of(z)]
            for r in range(g.TY):
                for b in range(g.TX):
                    yy, xx = y0 + r, x0 + b
                    if not inside(yy, xx):
                        continue
                    ey, ex = r % 2 == 0, b % 2 == 0
                    ri = r // 2 + 1 if ey else r // 2
                    sub = (g.EE if ex else g.EO) if ey else (g.OE if ex else g.OO)
                    lab = s[sub + ri * g.P + 2 + b // 2]
                    assert lab == ("r", z, yy, xx), (N, item, z, yy, xx, lab)
                    if stg[z, yy, xx] >= 0:
                        stored[c, z, yy, xx] += 1

        n_units = 3 + (ze - zs) // 2
        pend = []  # planes of the previous unit to store
        for u in range(n_units):
            if u < 3:
                ez, oz = zs - 2 + 2 * u, -1
            else:
                ez, oz = zs + 4 + 2 * (u - 3), zs + 1 + 2 * (u - 3)
            ev, ov = 0 <= ez < N[0], 0 <= oz < N[0]
            eown, oown = ev and zs <= ez < ze, ov and zs <= oz < ze
            # phase 0: stores read slots the transposition does not write
            # (the kernel stores first, behind a barrier, at an item's first unit)
            written = set()
            if ev:
                written.add(slot_of(ez))
            if ov:
                written.add(slot_of(oz))
            for z in pend:
                assert u == 0 or slot_of(z) not in written, "store / transpose slot conflict"
                store(z)
            if ev:
                transpose(ez, True)
            if ov:
                transpose(oz, False)
            zz = oz if oz >= 0 else 1
            zt = [slot_of(zz - 1), slot_of(zz + 1) if zz + 1 < N[0] else slot_of(zz - 1),
                  slot_of(zz - 3) if zz - 3 >= 0 else slot_of(zz - 1),
                  slot_of(zz + 3) if zz + 3 < N[0] else slot_of(zz - 1)]
            zok = tap_ok(zz, N[0])
            for phase in PHASES:
                present = [(cl, (ov if CLS[cl][0] else ev)) for cl in phase]
                counts = [(-(-g.cls(cl)[5] * g.cls(cl)[7] // 32) if on else 0)
                          for cl, on in present]
                tot = sum(counts)
                writes, reads = {}, set()
                for wi in range(LW):
                    tb, te = wi * tot // LW, (wi + 1) * tot // LW
                    assert te - tb <= MAXT, "more warp tasks than the code buffers hold"
                    for t in range(tb, te):
                        k, tt = 0, t
                        while tt >= counts[k]:
                            tt -= counts[k]
                            k += 1
                        cl = phase[k]
                        zo, yo, xo, st, sub, nr, c0, nc = g.cls(cl)
                        z = oz if zo else ez
                        plane = slots[slot_of(z)]
                        own_plane = oown if zo else eown
                        for lane in range(32):
                            e = tt * 32 + lane
                            if e >= nr * nc:
                                continue
                            row, col = e // nc, c0 + e % nc
                            idx = row * g.P + col
                            assert 0 <= row < g.sub_rows(sub) and 0 <= col < g.P
                            yy, xx = coords(sub, row, col)
                            pos = sub + idx
                            if inside(yy, xx):
                                assert plane[pos] == ("x", z, yy, xx), (cl, z, yy, xx, plane[pos])
                                # taps of every odd axis, for the flags' valid taps
                                if zo:
                                    for sl, dz, bit in ((zt[0], -1, 0), (zt[1], 1, 1),
                                                        (zt[2], -3, 2), (zt[3], 3, 4)):
                                        if bit and not (zok & bit):
                                            continue
                                        lab = slots[sl][pos]
                                        assert lab == ("r", z + dz, yy, xx), ("z", cl, z, lab)
                                        reads.add((sl, pos))
                                if yo:
                                    ysub = g.EO if xo else g.EE
                                    ok = tap_ok(yy, N[1])
                                    for dr, dy, bit in ((1, -1, 0), (2, 1, 1), (0, -3, 2),
                                                        (3, 3, 4)):
                                        if bit and not (ok & bit):
                                            continue
                                        assert row + dr < g.NER
                                        q = ysub + (row + dr) * g.P + col
                                        assert plane[q] == ("r", z, yy + dy, xx), ("y", cl, plane[q])
                                        reads.add((slot_of(z), q))
                                if xo:
                                    xsub = g.OE if yo else g.EE
                                    ok = tap_ok(xx, N[2])
                                    for dc, dx, bit in ((0, -1, 0), (1, 1, 1), (-1, -3, 2),
                                                        (2, 3, 4)):
                                        if bit and not (ok & bit):
                                            continue
                                        assert 0 <= col + dc < g.P
                                        q = xsub + row * g.P + col + dc
                                        assert plane[q] == ("r", z, yy, xx + dx), ("x", cl, plane[q])
                                        reads.add((slot_of(z), q))
                                writes[(slot_of(z), pos)] = ("r", z, yy, xx)
                                # the decoder reads the code of every computed
                                # point inside the lattice: a valid rank
                                r = rank(cl, z, yy, xx, N)
                                assert 0 <= r < nst[st]
                            else:
                                writes[(slot_of(z), pos)] = ("garbage",)
                            owned = (own_plane and inside(yy, xx) and
                                     (yo or 1 <= row <= g.TY // 2) and
                                     (xo or 2 <= col <= g.TX // 2 + 1))
                            if owned:
                                r = rank(cl, z, yy, xx, N)
                                flat = (z * N[1] + yy) * N[2] + xx
                                assert stg.reshape(-1)[flat] == st
                                assert r == order[st][flat], (cl, z, yy, xx, r, order[st][flat])
                                seen[st][c * nst[st] + r] += 1
                assert not (reads & set(writes)), "a tap reads a same-phase write"
                for (sl, pos), lab in writes.items():
                    slots[sl][pos] = lab
            pend = ([ez] if eown else []) + ([oz] if oown else [])
        for z in pend:
            store(z)
    for s in range(5):
        assert (seen[s] == 1).all(), ("stage", s, np.unique(seen[s]))
    level = np.broadcast_to(stg >= 0, stored.shape)
    assert (stored[level] == 1).all()


@pytest.mark.parametrize("N,C,elem", [
    ((9, 40, 70), 1, 4),     # two column tiles each way, ragged, odd extents
    ((20, 35, 66), 1, 4),    # edges on every axis
    ((7, 33, 130), 2, 4),    # two channels, three x tiles
    ((11, 19, 68), 1, 8),    # float64 tiles (16 rows)
    ((4, 64, 128), 1, 4),    # whole tiles, thin z
])
def test_level_kernel_index_plan(N, C, elem):
    emulate(N, C, elem)


def test_level_kernel_chunks():
    # several axis-0 chunks: few columns make the chunk rule pick short chunks
    N = (70, 12, 20)
    assert geometry(N, 1, 4)[3] > 1
    emulate(N, 1, 4)


def test_closed_form_ranks_follow_the_stage_order():
    for N in [(1, 1, 1), (2, 3, 5), (5, 4, 7), (9, 8, 6), (16, 17, 33), (3, 35, 67)]:
        order, stg = stage_order(N)
        cl_of = {0: W1Z, 1: W1Y, 2: W1X, 4: W3}
        for z in range(N[0]):
            for y in range(N[1]):
                for x in range(N[2]):
                    s = stg[z, y, x]
                    if s < 0:
                        continue
                    cl = cl_of.get(s, W2E if z % 2 == 0 else W2ZY)
                    assert rank(cl, z, y, x, N) == order[s][(z * N[1] + y) * N[2] + x]
