"""Host side of the learned codec's interpolation gate: the split rule picks
the cheapest (candidate, side, T, shift) of a brute-force enumeration, gate
words round-trip, and the gate's scale grid assigns every float32 scale the
level of the reference formula."""

import numpy as np


def _brute(W):
    """Exhaustive costs over every gate setting; W: (13, 13) per-bucket bits."""
    from latec_b200.gnn_codec import GATE_SHIFTS, GATE_T

    nb = len(GATE_T) + 1
    base = W[0]
    best = (base.sum(), (0, 0, 0, 0))
    for k in range(3):
        for si, sh in enumerate(GATE_SHIFTS):
            c = W[1 + 4 * k + si]
            for split in range(nb - 1):  # boundary after bucket `split`
                low = c[:split + 1].sum() + base[split + 1:].sum()
                high = base[:split + 1].sum() + c[split + 1:].sum()
                for cost, d in ((low, 0), (high, 1)):
                    if cost < best[0] - 1e-9:
                        best = (cost, (k + 1, d, GATE_T[split], sh))
    return best


def test_gate_choose_matches_brute_force():
    from latec_b200.gnn_codec import gate_choose

    rng = np.random.default_rng(0)
    for trial in range(200):
        W = rng.uniform(0, 100, (13, 13))
        if trial % 3 == 0:  # a candidate clearly better on the high buckets
            W[1 + 4 * rng.integers(3) + rng.integers(4), 6:] *= 0.1
        if trial % 5 == 0:  # the GNN best everywhere
            W[1:] = W[0] * 1.5
        cost, want = _brute(W)
        got = gate_choose(W.reshape(-1))
        assert got == want, (trial, got, want)


def test_gate_words_round_trip():
    from latec_b200.gnn_codec import gate_fields, gate_word, pack_gates, unpack_gates

    words = [gate_word(k, d, T, s) for k in (0, 1, 2, 3) for d in (0, 1) for T in (2, 9, 13)
             for s in (0, 2, 4, 6)]
    assert unpack_gates(pack_gates(words)) == words
    for w in words:
        assert gate_word(*gate_fields(w)) == w


def test_gate_scale_grid_levels():
    from latec_b200.gnn_codec import gate_scale_grid
    from latec_b200.rans_model import SCALE_HI_MULT, SCALE_LO_DIV

    for eb in (1e-4, 3e-3, 0.05):
        thr, grid = gate_scale_grid(eb, "cpu")
        thr, grid = thr.numpy(), grid.numpy()
        lo, hi = eb / SCALE_LO_DIV, eb * SCALE_HI_MULT
        log_lo = np.log(lo)
        step = (np.log(hi) - log_lo) / 63.0
        v = np.exp(np.random.default_rng(1).uniform(np.log(lo) - 2, np.log(hi) + 2, 20000))
        v = np.concatenate([v, thr, np.nextafter(thr, 0)]).astype(np.float32)
        want = np.rint((np.log(np.clip(v.astype(np.float64), lo, hi)) - log_lo) / step)
        got = np.searchsorted(thr, v, side="right")
        np.testing.assert_array_equal(got, want)
        np.testing.assert_allclose(grid, np.exp(log_lo + step * np.arange(64)), rtol=1e-15)
