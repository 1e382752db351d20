"""Pin the float64 GNN oracle to golden outputs of the reference GNN module
(tests/golden/make_gnn_golden.py): geometry exactly, predictions within
float32 rounding (the reference ran in float32)."""

import numpy as np
import pytest

from oracle import gnn as ognn
from tests.golden_io import load_npz

Z = load_npz("gnn.npz")
CASES = {c["name"]: c for c in Z["meta"]}

# The reference evaluates in float32: its per-stage outputs differ from the
# float64 restatement by accumulated float32 rounding only.
MU_ATOL = 1e-6
LB_ATOL = 1e-5


@pytest.mark.parametrize("name", sorted(CASES))
def test_geometry_matches_reference(name):
    c = CASES[name]
    geoms = ognn.stage_geoms(tuple(c["shape"]), c["levels"], c["stride"], c["block"],
                             c["max_radius"], c["agg_level"])
    assert len(geoms) == c["stages"]
    for s, g in enumerate(geoms):
        assert np.array_equal(g["query_idx"], Z[f"{name}_q{s}"])
        for k in ("sp", "sn", "vp", "vn"):
            assert np.array_equal(g[k], Z[f"{name}_{k}{s}"]), (s, k)


@pytest.mark.parametrize("name", sorted(CASES))
def test_forward_matches_reference(name):
    from latec_b200.gnn import random_weights

    c = CASES[name]
    w = random_weights(c["seed"], 64, c["agg_level"])
    geoms = ognn.stage_geoms(tuple(c["shape"]), c["levels"], c["stride"], c["block"],
                             c["max_radius"], c["agg_level"])
    out, E = ognn.run_stages(w, Z[f"{name}_x"], geoms, c["agg_level"], eb=c["eb"])
    for s, (mu, lb) in enumerate(out):
        np.testing.assert_allclose(mu, Z[f"{name}_mu{s}"], rtol=0, atol=MU_ATOL)
        np.testing.assert_allclose(lb, Z[f"{name}_lb{s}"], rtol=0, atol=LB_ATOL)
    np.testing.assert_allclose(E[..., :4], Z[f"{name}_E"], rtol=0, atol=1e-6)
