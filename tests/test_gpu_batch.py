"""Many tensors per call (latec_b200.batch): every stream of compress_many is
byte-identical to compress()'s for the same tensor and settings, and
decompress_many returns what decompress() returns, for mixed shapes, ranks,
dtypes (float32, float64, uint8 images), bounds and entropy modes."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _population():
    import torch

    from latec_b200 import fields

    out = [fields.grf_se((96, 80), 6.0, seed=1, device="cuda"),
           fields.grf_se((33, 40, 29), 4.0, seed=2, device="cuda"),
           fields.grf_se((40, 36, 30), 9.0, seed=3, device="cuda").double(),
           fields.turbulence_jumps((48, 50, 44), seed=4, device="cuda"),
           fields.grf_se((12, 10, 14, 9), 3.0, seed=5, device="cuda"),
           fields.grf_se((2, 2), 1.0, seed=6, device="cuda"),
           fields.grf_se((300, 257), 20.0, seed=7, device="cuda")]
    rs = np.random.RandomState(8)
    img = (np.clip(rs.rand(40, 36, 3) * 60 + np.linspace(0, 180, 36)[None, :, None], 0, 255)
           .astype(np.uint8))
    out.append(torch.from_numpy(img).cuda())
    return out


@pytest.mark.parametrize("eb_ratio", [None, 0.8])
def test_streams_equal_one_call_per_tensor(eb_ratio):
    import latec_b200 as lb
    from latec_b200.batch import compress_many, decompress_many

    xs = _population()
    ebs = [1e-3, 5e-3, 1e-4, 2e-3, 1e-2, 1e-3, 1e-3, 2.0]
    pred = lambda: lb.InterpPredictor("cubic", 3, 8, 1)  # noqa: E731
    got = compress_many(xs, ebs, pred(), levels=3, anchor_stride=8, eb_ratio=eb_ratio)
    want = [lb.compress(x, e, pred(), levels=3, anchor_stride=8, eb_ratio=eb_ratio,
                        recon="none")[0] for x, e in zip(xs, ebs)]
    assert len(got) == len(want)
    for j, (g, w) in enumerate(zip(got, want)):
        assert isinstance(g, bytes) and g == w, j
    outs = decompress_many(got, out="device")
    for j, (s, o) in enumerate(zip(got, outs)):
        ref = lb.decompress(s, out="device")
        assert o.dtype == ref.dtype and o.shape == ref.shape
        assert bool((o == ref).all()), j


def test_device_streams_and_a_compat_stream_in_one_batch():
    import torch

    import latec_b200 as lb
    from latec_b200.batch import compress_many, decompress_many

    xs = _population()[:5]
    pred = lb.InterpPredictor("linear", 2, 4, 1)
    dev = compress_many(xs, 3e-3, pred, levels=2, anchor_stride=4, stream_out="device")
    assert all(torch.is_tensor(s) and s.is_cuda and s.dtype == torch.uint8 for s in dev)
    host = compress_many(xs, 3e-3, pred, levels=2, anchor_stride=4)
    assert [bytes(s.cpu().numpy()) for s in dev] == host
    compat, _ = lb.compress(xs[0], 3e-3, lb.InterpPredictor("linear", 2, 4, 1), levels=2,
                            anchor_stride=4, entropy="compat", recon="none")
    mixed = [dev[1], host[2], compat, dev[3], host[4]]
    outs = decompress_many(mixed, out="numpy")
    for s, o in zip(mixed, outs):
        ref = lb.decompress(s)
        assert isinstance(o, np.ndarray) and np.array_equal(o, ref)
    # the bound holds on every element
    for x, o in zip(xs, decompress_many(host)):
        err = np.abs(o.astype(np.float64) - x.double().cpu().numpy()).max()
        assert err <= 3e-3 * (1 + 1e-9)


def test_bad_streams_raise():
    import latec_b200 as lb
    from latec_b200.batch import compress_many, decompress_many

    xs = _population()[:3]
    streams = compress_many(xs, 1e-3, lb.InterpPredictor("cubic", 3, 8, 1), levels=3,
                            anchor_stride=8)
    with pytest.raises(ValueError):
        decompress_many([streams[0], streams[1][:-1], streams[2]])  # truncated frame
    with pytest.raises(ValueError):
        decompress_many([b"NOTLATEC" + streams[0][8:]])
    with pytest.raises(ValueError):
        compress_many(xs, [1e-3, 1e-3], lb.InterpPredictor("cubic", 3, 8, 1), levels=3,
                      anchor_stride=8)
    assert compress_many([], 1e-3, lb.InterpPredictor("cubic", 3, 8, 1), levels=3,
                         anchor_stride=8) == []
    # flipped bits in one stream of a batch: an error or a field, never a fault
    rs = np.random.RandomState(0)
    for _ in range(20):
        bad = bytearray(streams[1])
        pos = rs.randint(100, len(bad))
        bad[pos] ^= 1 << rs.randint(0, 8)
        try:
            outs = decompress_many([streams[0], bytes(bad), streams[2]])
            assert outs[1].shape == tuple(xs[1].shape)
        except (ValueError, KeyError, NotImplementedError):
            pass


def test_runtime_rank_and_blocked_anchor_classes():
    """5-D and 6-D tensors and blocked anchors (runtime-rank launch classes)
    in one batch: streams equal compress()'s, fields equal decompress()'s."""
    import latec_b200 as lb
    from latec_b200 import fields
    from latec_b200.batch import compress_many, decompress_many

    xs = [fields.grf_se((5, 4, 6, 5, 4, 5), 2.0, seed=11, device="cuda"),
          fields.grf_se((6, 5, 7, 6, 5), 2.0, seed=12, device="cuda"),
          fields.grf_se((40, 44), 5.0, seed=13, device="cuda").double(),
          fields.grf_se((20, 18, 22), 4.0, seed=14, device="cuda")]
    for block in (1, 2):
        pred = lambda: lb.InterpPredictor("cubic", 2, 4, block)  # noqa: E731
        got = compress_many(xs, 2e-3, pred(), levels=2, anchor_stride=4, anchor_block=block)
        want = [lb.compress(x, 2e-3, pred(), levels=2, anchor_stride=4, anchor_block=block,
                            recon="none")[0] for x in xs]
        for j, (g, w) in enumerate(zip(got, want)):
            assert g == w, (block, j)
        for j, (s, o) in enumerate(zip(got, decompress_many(got, out="device"))):
            assert bool((o == lb.decompress(s, out="device")).all()), (block, j)


def test_cta_caps_leave_streams_unchanged():
    """Every encode CTA cap (one CTA per stage up to the single-tensor grid),
    and the autotuned table, code the same streams."""
    import latec_b200 as lb
    from latec_b200 import batch

    xs = _population()[:5]
    pred = lambda: lb.InterpPredictor("cubic", 3, 8, 1)  # noqa: E731
    want = [lb.compress(x, 1e-3, pred(), levels=3, anchor_stride=8, recon="none")[0]
            for x in xs]
    saved = batch.cta_caps()
    try:
        for cap in (1, 3, 148, 5000):
            batch._cta_caps.clear()
            for nd in (2, 3, 4):
                for elem in (4, 8):
                    for sc in range(4):
                        batch._cta_caps[(nd, elem, sc)] = cap
            assert batch.compress_many(xs, 1e-3, pred(), levels=3, anchor_stride=8) == want, cap
        batch._cta_caps.clear()
        tuned = batch.autotune_many(xs, 1e-3, pred(), levels=3, anchor_stride=8, repeats=1,
                                    candidates=(2, 148))
        assert set(tuned) and all(c in (2, 148) and ms > 0 for c, ms in tuned.values())
        assert batch.compress_many(xs, 1e-3, pred(), levels=3, anchor_stride=8) == want
    finally:
        batch._cta_caps.clear()
        batch._cta_caps.update(saved)
