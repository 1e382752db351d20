"""Host logic of the batch API (latec_b200.batch) and the schedule cache:
the shared-buffer layout that lets one model-fit and one lane-coder launch
address every stage of every tensor, the least-recently-used plans, the
ctypes job records of the many-tensor stage calls (the C layouts of
include/latec_b200.h) and the autotuned CTA table's keys."""

import ctypes

import numpy as np


def _sizes(shapes, elem=4):
    from latec_b200 import levels
    from latec_b200.codec import buffer_sizes

    return [buffer_sizes(levels.plan_for(s, 3, 8, 1), 1, elem) for s in shapes]


def test_shared_buffers_pack_stages_and_align_slices():
    from latec_b200 import _lib, rans_model
    from latec_b200.batch import _ALIGN, _arenas

    shapes = [(40, 36), (9, 10, 11), (2, 2), (130, 70), (5, 6, 7, 8)]
    sizes = _sizes(shapes)
    views, bufs = _arenas(sizes, "cpu")
    ssz = ctypes.sizeof(_lib.StageStats)
    stage0 = np.cumsum([0] + [sz["stats"][0] // ssz for sz in sizes])
    for kind, (buf, offs) in bufs.items():
        esz = buf.element_size()
        base = buf.data_ptr()
        ends = []
        for j, sz in enumerate(sizes):
            v = views[j][kind]
            assert v.numel() == sz[kind][0]
            assert v.data_ptr() == base + offs[j] * esz
            ends.append(offs[j] + sz[kind][0])
            if kind == "stats":  # packed: a stage's global index = first stage + own index
                assert offs[j] * esz == stage0[j] * ssz
            elif kind == "hist_total":
                assert offs[j] == stage0[j] * 65536
            elif kind == "hist_seg":  # whole segment rows
                assert offs[j] % (2 * rans_model.HWIN) == 0
            else:
                assert (offs[j] * esz) % _ALIGN == 0
        # slices are disjoint and inside the buffer
        assert all(e <= o for e, o in zip(ends[:-1], offs[1:]))
        assert ends[-1] <= buf.numel()


def test_plan_cache_keeps_the_recent_schedules():
    from latec_b200 import levels

    old = levels._PLAN_CACHE
    levels._plans.clear()
    levels._PLAN_CACHE = 4
    try:
        first = levels.plan_for((20, 20), 2, 4)
        for n in range(21, 24):
            levels.plan_for((n, n), 2, 4)
        assert levels.plan_for((20, 20), 2, 4) is first  # a hit refreshes it
        levels.plan_for((30, 30), 2, 4)  # evicts the least recently used: (21, 21)
        assert len(levels._plans) == 4
        assert ((21, 21), 2, 4, 1) not in levels._plans
        assert levels.plan_for((20, 20), 2, 4) is first
    finally:
        levels._PLAN_CACHE = old
        levels._plans.clear()


def test_job_records_match_the_c_layout():
    from latec_b200 import _lib

    # latec_quant_params: 8 int32 + 2 double; the job records add pointers
    assert ctypes.sizeof(_lib.QuantParams) == 48
    assert ctypes.sizeof(_lib.EncodeJob) == 144
    assert ctypes.sizeof(_lib.DecodeJob) == 112
    assert _lib.EncodeJob.max_ctas.offset == 136
    assert _lib.DecodeJob.err.offset == 104


def test_size_classes_and_cap_lookup():
    from latec_b200 import batch

    assert [batch.size_class(n) for n in (1, 65535, 65536, 524287, 524288, (1 << 22) - 1,
                                          1 << 22, 1 << 30)] == [0, 0, 1, 1, 2, 2, 3, 3]
    caps = {(3, 4, 2): 296, (2, 8, 0): 148}
    assert batch.cta_cap(3, 4, 1 << 21, caps) == 296
    assert batch.cta_cap(2, 8, 1000, caps) == 148
    assert batch.cta_cap(3, 8, 1 << 21, caps) == 0  # no entry: the single-tensor grid
    saved = batch.cta_caps()
    try:
        batch._cta_caps.clear()
        batch._cta_caps[(2, 4, 3)] = 592
        assert batch.cta_cap(2, 4, 1 << 23) == 592 and batch.cta_caps() == {(2, 4, 3): 592}
    finally:
        batch._cta_caps.clear()
        batch._cta_caps.update(saved)
