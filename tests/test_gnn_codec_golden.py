"""The learned codec against the reference learned codec, stage by stage.

tests/golden/gnn_codec.npz was recorded from the reference's own
``GNNCodec.compress`` (float32 on the CPU, gate on) with the checkpoint this
repository ships, by tests/golden/make_gnn_codec_golden.py. Here
``latec_b200.GNNCodec`` (float32 path, same checkpoint) codes the same fields
on the GPU, and its per-stage trace is compared with the recording
(latec/gnn_codec.py:1048-1336 is the loop both follow):

* the model's mu and Laplace scale per stage, within float32 tolerance (the
  two evaluate the same network in different summation orders, and later
  stages see the earlier stages' differences through the reconstruction);
* the gate's choice per stage (kind, direction, T, shift), equal except for
  at most one near-tie once the outputs have drifted apart; with
  ``gate_fine`` the finest sub-stages after the first apply the first one's
  choice (latec/gnn_codec.py:1229-1262);
* the quantized codes: identical except at points whose quotient
  (x - p) / 2eb lies within the two gated predictions' difference of a bin
  boundary (or whose reconstruction error lies that close to the bound);
  the scale levels: identical up to a few boundary points;
* the final reconstruction (equal to the reference's up to the predictions'
  float32 differences when every code agrees) and the error bound.
"""

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

CKPT = os.path.join(ROOT, "latec_b200", "checkpoints", "gnn_d64_agg1_synthetic.pt")


def _load():
    z = np.load(os.path.join(GOLDEN, "gnn_codec.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    return z, meta


CASES = [m["name"] for m in _load()[1]]


@pytest.mark.parametrize("name", CASES)
def test_gnn_codec_matches_reference_per_stage(name):
    import latec_b200 as lb
    from latec_b200.gnn_codec import gate_fields

    z, metas = _load()
    m = next(mm for mm in metas if mm["name"] == name)
    x = z[f"{name}/x"]
    codec = lb.GNNCodec(CKPT, device="cuda")
    codec.stage_trace = []
    fine = bool(m.get("gate_fine", False))
    stream = codec.compress(x, m["rel_eb"], levels=m["levels"], fp16=False, gate=True,
                            gate_fine=fine)
    tr = {t["stage"]: t for t in codec.stage_trace}
    report = []
    n_lv_diff = n_code = 0
    max_dp = 0.0
    gate_flips = 0
    g_last = None
    for k, s in enumerate(m["stages"]):
        t = tr[s]
        eb = m["ebs"][k]
        assert abs(t["eb"] - eb) <= 1e-15 * eb, (s, t["eb"], eb)
        mu_r, sc_r = z[f"{name}/{k}/mu"], z[f"{name}/{k}/scale"]
        mu, sc = t["mu"].cpu().numpy(), t["scale"].cpu().numpy()
        assert mu.shape == mu_r.shape, (s, mu.shape, mu_r.shape)
        # float32 agreement of the network's outputs (mu in [0, 1]; the scale
        # as log2): the two evaluate the same network in different summation
        # orders, and from the second level on each stage's inputs carry the
        # previous stages' differences through the reconstruction
        dmu = float(np.abs(mu.astype(np.float64) - mu_r).max())
        dsc = float(np.abs(np.log2(sc.astype(np.float64) / sc_r)).max())
        assert dmu <= 5e-4, (s, dmu)
        assert dsc <= 1e-2, (s, dsc)
        # the gate's choice: equal, except that one near-tie may flip once
        # the network's outputs have drifted apart
        g_ref = m["gates"][k]
        if g_ref is None:
            # gate_fine: the finest sub-stages after the first reuse its choice
            assert fine and g_last is not None, (s, "no gate recorded")
            g_ref = g_last
        g_last = g_ref
        g = list(gate_fields(int(t["word"].item())))
        if g != g_ref:
            gate_flips += 1
            assert gate_flips == 1 and dmu > 1e-5, ("gate", s, g, g_ref, dmu)
            report.append((s, len(mu), dmu, dsc, g_ref, g, None, None))
            continue
        # codes: identical except where the gated prediction's difference can
        # move the point across a bin boundary or across the bound check
        codes_r = z[f"{name}/{k}/codes"]
        codes = t["codes"].cpu().numpy().view(np.uint16).astype(np.int64)
        xs = t["x"].cpu().numpy().astype(np.float64)
        p_r = z[f"{name}/{k}/mu_g"].astype(np.float64)
        p_o = t["mu_gated"].cpu().numpy().astype(np.float64)
        w = 2.0 * eb
        max_dp = max(max_dp, float(np.abs(p_o - p_r).max()))
        band = np.abs(p_o - p_r) / w + 1e-9
        q = (xs - p_r) / w
        near_bin = np.abs(np.abs(q - np.floor(q)) - 0.5) <= band
        rec_r = p_r + w * np.rint(q)
        near_bound = np.abs(np.abs(xs - rec_r) - eb) <= np.abs(p_o - p_r) + 1e-9
        diff = codes != codes_r
        assert not (diff & ~near_bin & ~near_bound).any(), (s, int(diff.sum()))
        lv_r, lv = z[f"{name}/{k}/levels"], t["levels"].cpu().numpy()
        dl = int((lv != lv_r).sum())
        n_lv_diff += dl
        n_code += len(codes)
        report.append((s, len(mu), dmu, dsc, g_ref, g, int(diff.sum()), dl))
    print("\n".join(map(str, report)))
    assert n_lv_diff <= max(2, n_code // 500), report
    # the decoded field holds the bound (plus the float32 normalisation slack)
    back = codec.uncompress(stream).cpu().numpy()
    vmin, vmax = float(np.float32(x.min())), float(np.float32(x.max()))
    span = vmax - vmin
    slack = 2.0 ** -24 * (3.0 * span + max(abs(vmin), abs(vmax)))
    assert float(np.abs(back.astype(np.float64) - x).max()) <= m["eb_abs"] + slack
    if all(r[6] == 0 for r in report):
        # every code equal: the decoded field is the reference's
        # reconstruction up to the gated predictions' float32 differences (a
        # coded point is prediction + 2 eb q, an outlier its exact value)
        recon_r = z[f"{name}/recon"].reshape(x.shape).astype(np.float64) * span + vmin
        assert float(np.abs(back.reshape(x.shape) - recon_r).max()) <= max_dp * span + 4 * slack
