"""Index plans of the tensor-core training GEMM (k_gemm_tc in
latec_b200/csrc/train_kernels.cu) and of the single-stack encoder's blocks
(k_stack_encode in rans_kernels.cu), restated on the CPU: every operand element
of a K chunk is staged exactly once into its own canonical slot, the split-K
slices tile [0, K) on 64-element boundaries, and the encoder's blocks visit the
symbols n - 1 ... 0 once each, in that order."""

import numpy as np
import pytest

GT_KC = 64
GT_THREADS = 256


def canon(r, k, R):
    """Element offset of (row r, column k) in the no-swizzle K-major layout."""
    return ((k >> 3) * (R >> 3) + (r >> 3)) * 64 + (r & 7) * 8 + (k & 7)


def items(R, k_contiguous):
    """(row, 8-wide chunk) of each staging item, in item order."""
    out = []
    for it in range(R * (GT_KC // 8)):
        if k_contiguous:
            g, lane = it >> 5, it & 31
            out.append(((g >> 1) * 8 + (lane & 7), (g & 1) * 4 + (lane >> 3)))
        else:
            out.append((it % R, it // R))
    return out


@pytest.mark.parametrize("R", [64, 128])
@pytest.mark.parametrize("k_contiguous", [False, True])
def test_staging_covers_each_slot_once(R, k_contiguous):
    seen = np.zeros(R * GT_KC, np.int32)
    for r, c in items(R, k_contiguous):
        assert 0 <= r < R and 0 <= c < GT_KC // 8
        base = canon(r, c * 8, R)
        assert base % 8 == 0  # one 16-byte BF16 store
        for e in range(8):
            assert canon(r, c * 8 + e, R) == base + e
        seen[base:base + 8] += 1
    assert (seen == 1).all()


@pytest.mark.parametrize("R", [64, 128])
@pytest.mark.parametrize("k_contiguous", [False, True])
def test_warp_access_pattern(R, k_contiguous):
    its = items(R, k_contiguous)
    for w0 in range(0, len(its), 32):
        warp = its[w0:w0 + 32]
        # the canonical stores of a warp fill whole 128-byte rows of 8 slots
        starts = sorted(canon(r, c * 8, R) for r, c in warp)
        groups = {s // 64 for s in starts}
        assert len(groups) * 8 == 32
        if k_contiguous:
            # 8 rows x 4 adjacent chunks: each row reads 32 contiguous floats
            rows = {}
            for r, c in warp:
                rows.setdefault(r, []).append(c)
            assert len(rows) == 8
            for cs in rows.values():
                cs = sorted(cs)
                assert cs == list(range(cs[0], cs[0] + 4))
        else:
            assert len({r for r, _ in warp}) == 32  # 32 consecutive rows, one column each


@pytest.mark.parametrize("K,splits", [(1, 1), (64, 1), (162, 1), (4097, 2), (20000, 5),
                                      (1 << 20, 256), (300000, 74)])
def test_split_k_slices(K, splits):
    per = ((K + splits - 1) // splits + GT_KC - 1) // GT_KC * GT_KC
    covered = []
    for z in range(splits):
        kb = per * z
        ke = min(kb + per, K)
        assert kb % GT_KC == 0
        if ke > kb:
            covered.append((kb, ke))
    assert covered[0][0] == 0 and covered[-1][1] == K
    for (a0, a1), (b0, b1) in zip(covered, covered[1:]):
        assert a1 == b0


def test_tmem_and_shared_budget():
    # per CTA: two buffers of (128 + NT) x 64 BF16; TMEM columns = NT
    for nt in (64, 128):
        smem = 2 * (128 + nt) * GT_KC * 2
        per_sm = min(228 * 1024 // (smem + 1024), 2048 // GT_THREADS)
        assert per_sm * nt <= 512  # resident CTAs never oversubscribe tensor memory


@pytest.mark.parametrize("n", [0, 1, 1023, 1024, 1025, 5000])
def test_stack_encoder_blocks(n):
    SB = 1024
    nb = (n + SB - 1) // SB
    order = []
    for b in range(nb):
        top = n - 1 - b * SB
        cnt = min(SB, n - b * SB)
        slots = [top - j for j in range(SB) if top - j >= 0]
        assert len(slots) == cnt
        order.extend(slots[:cnt])
    assert order == list(range(n - 1, -1, -1))
