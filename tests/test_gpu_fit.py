"""The native stage-model fit on the device (fit_kernels.cu: every
(shape, level) cost the exact 64-bit sum of rint(W * 2^20) * count over the
power-of-two alphabet, first argmin over levels, first strictly smaller shape)
against the oracle's restatement (oracle/rans_model.py fit_const_native), bit
for bit, for coder windows from 4 symbols to 16,384: counts in shared memory
and in global memory, dense, sparse and single-bin histograms, in one
launch."""

import ctypes

import numpy as np
import pytest

from oracle import rans_model as orm

pytestmark = pytest.mark.gpu

RADIUS = 1 << 15
HWIN = 256


def _counts(kexp, kind, rs):
    """A histogram over the narrowed alphabet (sym 0 = outliers, sym s >= 1 =
    q = s - 2^kexp)."""
    A = 2 << kexp
    span = (1 << kexp) - 1
    c = np.zeros(A, np.int64)
    q = np.arange(-span, span + 1)
    if kind == "dense":
        c[1:] = rs.poisson(2000 * np.exp(-np.abs(q) / max(1.0, span / 6)))
    elif kind == "sparse":
        pick = rs.choice(np.arange(1, A), size=min(A - 1, 7), replace=False)
        c[pick] = rs.randint(1, 50, len(pick))
    else:  # one bin
        c[1 + span] = 12345
    c[0] = rs.randint(0, 40)
    return c


def test_device_fit_matches_oracle():
    import torch

    import latec_b200 as lb  # noqa: F401  (loads the library)
    from latec_b200 import _lib, rans_model
    from latec_b200.codec import _FIT_DTYPE

    lib = _lib.load()
    dev = torch.device("cuda")
    rs = np.random.RandomState(3)
    cases = [(k, kind) for k in (1, 3, 4, 6, 7, 8, 11, 12, 13)
             for kind in ("dense", "sparse", "one")]
    n = len(cases)
    hist_seg = np.zeros((n, 2 * HWIN), np.uint32)
    hist_total = np.zeros((n, 65536), np.uint32)
    all_counts = []
    for t, (kexp, kind) in enumerate(cases):
        c = _counts(kexp, kind, rs)
        all_counts.append(c)
        span = (1 << kexp) - 1
        hist_seg[t, 0] = c[0]
        for s in np.flatnonzero(c[1:]) + 1:
            q = int(s) - span - 1
            if -HWIN < q < HWIN:
                hist_seg[t, q + HWIN] = c[s]
            else:
                hist_total[t, q + RADIUS] = c[s]
    fs = np.zeros(n, _FIT_DTYPE)
    alph = np.asarray([2 << k for k, _ in cases], np.int64)
    kexps = np.asarray([k for k, _ in cases], np.int64)
    items = np.asarray([int(c.sum()) for c in all_counts], np.int64)
    owxs = rans_model.choose_outlier_weights(np.asarray([int(c[0]) for c in all_counts]), items)
    fs["counts_off"] = np.concatenate([[0], np.cumsum(alph)[:-1]])
    fs["seg_off"] = np.arange(n, dtype=np.uint64)
    fs["n_segs"] = 1
    fs["alphabet"], fs["kexp"], fs["radius"] = alph, kexps, RADIUS
    fs["stage"] = np.arange(n, dtype=np.uint32)
    keep = []
    for j, (kexp, owx) in enumerate(zip(kexps.tolist(), owxs.tolist())):
        w, ids = rans_model.device_weights.get(kexp, owx, dev)
        keep.append(w)
        row = np.zeros(24, np.uint32)
        row[:len(ids)] = ids
        fs["w_table"][j], fs["n_shapes"][j], fs["shape_ids"][j] = w.data_ptr(), len(ids), row
    seg_d = torch.from_numpy(hist_seg.view(np.int32).reshape(-1)).to(dev)
    tot_d = torch.from_numpy(hist_total.view(np.int32).reshape(-1)).to(dev)
    counts = torch.empty(int(alph.sum()), dtype=torch.int32, device=dev)
    costs = torch.empty(n * 24 * 64, dtype=torch.float64, device=dev)
    out = torch.empty(n * 3, dtype=torch.float64, device=dev)
    ws = torch.empty(n * ctypes.sizeof(_lib.FitStage) + 256, dtype=torch.uint8, device=dev)
    _lib.check(lib.latec_fit_const(fs.ctypes.data, n, seg_d.data_ptr(), tot_d.data_ptr(),
                                   counts.data_ptr(), costs.data_ptr(), out.data_ptr(),
                                   ws.data_ptr(), ws.numel(), _lib.stream_ptr()),
               "latec_fit_const")
    got = out.cpu().numpy().reshape(n, 3)
    dc = counts.cpu().numpy()
    for t, (kexp, kind) in enumerate(cases):
        a = int(fs["counts_off"][t])
        assert np.array_equal(dc[a:a + alph[t]], all_counts[t]), (kexp, kind)
        level, sid, owx, cost = orm.fit_const_native(all_counts[t], int(items[t]), kexp)
        assert owx == int(owxs[t]), (kexp, kind)
        assert (int(got[t, 1]), int(got[t, 2])) == (level, sid), (kexp, kind)
        assert got[t, 0] == cost, (kexp, kind, got[t, 0], cost)
    del keep
