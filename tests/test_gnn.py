"""The learned predictor (latec/gnn_predictor.py): host geometry against the
reference's own geometry (exact), and the CUDA forward against the float64
oracle and the reference module's float32 outputs."""

import numpy as np
import pytest

from tests.golden_io import load_npz

Z = load_npz("gnn.npz")
CASES = {c["name"]: c for c in Z["meta"]}

# float32 kernels vs the float64 oracle: accumulated float32 rounding only
# (the reference's own float32 run differs from the oracle by < 1e-7 on mu and
# < 1e-6 on log2 b).
MU_ATOL = 1e-5
LB_ATOL = 1e-4


def _geoms(c, device):
    from latec_b200 import gnn

    return gnn.build_stage_geoms(tuple(c["shape"]), c["levels"], c["stride"], c["block"],
                                 c["max_radius"], c["agg_level"], device=device)[0]


@pytest.mark.parametrize("name", sorted(CASES))
def test_geometry_matches_reference(name):
    c = CASES[name]
    geoms = _geoms(c, "cpu")
    assert len(geoms) == c["stages"]
    for s, g in enumerate(geoms):
        assert np.array_equal(g.query_idx_np, Z[f"{name}_q{s}"])
        assert np.array_equal(g.sp, Z[f"{name}_sp{s}"]) and np.array_equal(g.sn, Z[f"{name}_sn{s}"])
        assert np.array_equal(g.valid_p, Z[f"{name}_vp{s}"])
        assert np.array_equal(g.valid_n, Z[f"{name}_vn{s}"])


@pytest.mark.parametrize("d,agg", [(64, 1), (64, 2), (16, 3)])
def test_param_layout_matches_kernels(d, agg):
    from latec_b200 import _lib, gnn

    lib = _lib.load(require_gpu=False)
    n = sum(int(np.prod(s)) for s in gnn.param_shapes(d, agg).values())
    assert int(lib.latec_gnn_param_count(d, agg)) == n
    w = gnn.random_weights(3, d, agg)
    assert set(w) == set(gnn.param_shapes(d, agg))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_forward_matches_oracle_and_reference(name):
    from latec_b200 import gnn
    from oracle import gnn as ognn

    c = CASES[name]
    w = gnn.random_weights(c["seed"], 64, c["agg_level"])
    model = gnn.GNNModel(w, 64, c["agg_level"])
    out, E = gnn.run_stages(model, Z[f"{name}_x"], _geoms(c, None), eb=c["eb"])
    ogeoms = ognn.stage_geoms(tuple(c["shape"]), c["levels"], c["stride"], c["block"],
                              c["max_radius"], c["agg_level"])
    want, E64 = ognn.run_stages(w, Z[f"{name}_x"], ogeoms, c["agg_level"], eb=c["eb"])
    for s, ((mu, lb), (mu64, lb64)) in enumerate(zip(out, want)):
        mu, lb = mu.cpu().numpy(), lb.cpu().numpy()
        np.testing.assert_allclose(mu, mu64, rtol=0, atol=MU_ATOL)
        np.testing.assert_allclose(lb, lb64, rtol=0, atol=LB_ATOL)
        np.testing.assert_allclose(mu, Z[f"{name}_mu{s}"], rtol=0, atol=MU_ATOL)
        np.testing.assert_allclose(lb, Z[f"{name}_lb{s}"], rtol=0, atol=LB_ATOL)
    np.testing.assert_allclose(E.cpu().numpy()[..., :4], Z[f"{name}_E"], rtol=0, atol=1e-5)
    np.testing.assert_allclose(E.cpu().numpy(), E64, rtol=0, atol=1e-5)


@pytest.mark.gpu
def test_device_forward_is_deterministic_and_tiles():
    """Same bits on a second run, and the same bits when the message pass is
    split into query tiles (encoder and decoder must predict identically)."""
    from latec_b200 import gnn

    c = CASES["g2d"]
    w = gnn.random_weights(c["seed"], 64, 1)
    model = gnn.GNNModel(w, 64, 1)
    x = Z["g2d_x"]
    a, Ea = gnn.run_stages(model, x, _geoms(c, None), eb=c["eb"])
    b, Eb = gnn.run_stages(model, x, _geoms(c, None), eb=c["eb"])
    geoms_t = gnn.build_stage_geoms(tuple(c["shape"]), c["levels"], c["stride"], c["block"],
                                    c["max_radius"], 1, m_tile=7)[0]
    t, Et = gnn.run_stages(model, x, geoms_t, eb=c["eb"])
    for (m1, l1), (m2, l2), (m3, l3) in zip(a, b, t):
        assert np.array_equal(m1.cpu().numpy().view(np.uint32), m2.cpu().numpy().view(np.uint32))
        assert np.array_equal(l1.cpu().numpy().view(np.uint32), l2.cpu().numpy().view(np.uint32))
        assert np.array_equal(m1.cpu().numpy().view(np.uint32), m3.cpu().numpy().view(np.uint32))
    assert np.array_equal(Ea.cpu().numpy(), Eb.cpu().numpy())
    assert np.array_equal(Ea.cpu().numpy(), Et.cpu().numpy())


# BF16 operands (8-bit mantissa) in the message and finalisation MLPs: the
# predictions move by the rounding of those operands, well under these bounds
# (the codec's bound never depends on them: quantization enforces it).
BF16_MU_ATOL = 1e-2
BF16_LB_ATOL = 1e-1


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["g2d", "g3d", "g2d_agg2"])
def test_bf16_tensor_core_forward_close_to_oracle(name):
    from latec_b200 import gnn
    from oracle import gnn as ognn

    c = CASES[name]
    w = gnn.random_weights(c["seed"], 64, c["agg_level"])
    model = gnn.GNNModel(w, 64, c["agg_level"], precision="bf16")
    out, E = gnn.run_stages(model, Z[f"{name}_x"], _geoms(c, None), eb=c["eb"])
    again, E2 = gnn.run_stages(model, Z[f"{name}_x"], _geoms(c, None), eb=c["eb"])
    ogeoms = ognn.stage_geoms(tuple(c["shape"]), c["levels"], c["stride"], c["block"],
                              c["max_radius"], c["agg_level"])
    want, _ = ognn.run_stages(w, Z[f"{name}_x"], ogeoms, c["agg_level"], eb=c["eb"])
    assert int(model.tc_err.item()) == 0
    dmu = max(float(np.abs(m.cpu().numpy() - m64).max()) for (m, _), (m64, _) in zip(out, want))
    dlb = max(float(np.abs(l.cpu().numpy() - l64).max()) for (_, l), (_, l64) in zip(out, want))
    print(f"{name}: bf16 vs float64 oracle: max |d mu| {dmu:.3g}, max |d log2 b| {dlb:.3g}")
    assert dmu < BF16_MU_ATOL and dlb < BF16_LB_ATOL
    for (m1, l1), (m2, l2) in zip(out, again):  # deterministic
        assert np.array_equal(m1.cpu().numpy().view(np.uint32), m2.cpu().numpy().view(np.uint32))
    assert np.array_equal(E.cpu().numpy(), E2.cpu().numpy())


# E4M3 operands (3-bit mantissa) with per-channel weight and per-row
# activation scales in the message and finalisation MLPs.
FP8_MU_ATOL = 5e-2
FP8_LB_ATOL = 5e-1


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["g2d", "g3d", "g2d_agg2"])
def test_fp8_tensor_core_forward_close_to_oracle(name):
    from latec_b200 import gnn
    from oracle import gnn as ognn

    c = CASES[name]
    w = gnn.random_weights(c["seed"], 64, c["agg_level"])
    model = gnn.GNNModel(w, 64, c["agg_level"], precision="fp8")
    out, E = gnn.run_stages(model, Z[f"{name}_x"], _geoms(c, None), eb=c["eb"])
    again, _ = gnn.run_stages(model, Z[f"{name}_x"], _geoms(c, None), eb=c["eb"])
    ogeoms = ognn.stage_geoms(tuple(c["shape"]), c["levels"], c["stride"], c["block"],
                              c["max_radius"], c["agg_level"])
    want, _ = ognn.run_stages(w, Z[f"{name}_x"], ogeoms, c["agg_level"], eb=c["eb"])
    assert int(model.tc_err.item()) == 0
    dmu = max(float(np.abs(m.cpu().numpy() - m64).max()) for (m, _), (m64, _) in zip(out, want))
    dlb = max(float(np.abs(l.cpu().numpy() - l64).max()) for (_, l), (_, l64) in zip(out, want))
    print(f"{name}: fp8 vs float64 oracle: max |d mu| {dmu:.3g}, max |d log2 b| {dlb:.3g}")
    assert dmu < FP8_MU_ATOL and dlb < FP8_LB_ATOL
    for (m1, _), (m2, _) in zip(out, again):  # deterministic
        assert np.array_equal(m1.cpu().numpy().view(np.uint32), m2.cpu().numpy().view(np.uint32))
