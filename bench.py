"""Benchmark: LATEC plain interpolation codec on B200.

Workload (one step = compress + decompress of the field through the public
API): 512^3 float32 power-law turbulence (E(k) ~ k^-5/3, unit variance) plus
3 random-hyperplane steps of amplitude 1, seeded synthetic data; cubic
InterpPredictor, levels=6, anchor_stride=64, absolute bound = 1e-4 x value
range. The 512 MiB input is larger than the 126 MB L2, so no flush is needed
between steps.

value  : input GB/s of the round trip with the field resident in HBM
         (bytes / (compress + decompress time)), CUDA events on the stream; the
         compressed stream stays in HBM too (stream_out="device").
e2e    : the same through host buffers: a page-locked host field in, the
         stream returned as a page-locked NumPy array, decoded from it back to
         a NumPy field; every host <-> device copy inside the timed region.
roofline: the dominant kernel, the fused encode of the finest level
         (k_lvl_enc, five sub-stages of stride 1 in one launch) -- algorithmic
         bytes 10 B per level point (read x, write recon, write the 16-bit
         code) + 4 B per coarser point (read once as a tap), over the launch's
         duration from CUDA event pairs the library records on the launching
         stream, against the measured HBM copy bandwidth. Beside it the
         finest-level decode, the coarser fused levels, the lane coders, the
         whole encode pass, and the codec-level fractions (N s + S bytes per
         direction over the compress / decompress time).
compat : the drop-in stream (the reference's single-stack rANS layout and
         zstd frame) on the same field.
cfg1, f64_256: the 512^2 SE-GRF configuration and the float64 256^3 variant.
cpu_baseline: the CPU oracle (NumPy restatement of the reference algorithm +
         C rANS coder) on a 128^3 sample of the same generator, 1 core.

``--impl reference`` times that CPU restatement of the reference path as its
own arm (rank 0 only under torchrun).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (512, 512, 512)
LEVELS, STRIDE, REL_EB = 6, 64, 1e-4
SAMPLE = (128, 128, 128)
METRIC = "compress/decompress GB/s and ratio at fixed abs eb (interp, 1 B200)"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


_NVML_CHILD = r"""
import json, select, sys, pynvml
pynvml.nvmlInit()
try:
    h = pynvml.nvmlDeviceGetHandleByPciBusId(sys.argv[1].encode())
except Exception:
    h = pynvml.nvmlDeviceGetHandleByIndex(int(sys.argv[2]))
mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
print("ready", flush=True)
rows = []
cmd = sys.stdin.readline().strip()
while cmd == "go":  # sample until "pause" or "stop"; "go" again resumes
    while True:
        try:
            rows.append((pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM), mx,
                         int(pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h))))
        except Exception:
            pass
        if select.select([sys.stdin], [], [], 0.002)[0]:
            cmd = sys.stdin.readline().strip()
            break
    if cmd == "pause":
        cmd = sys.stdin.readline().strip()
print(json.dumps(rows), flush=True)
"""


class ClockSampler:
    """SM clock and clock-event reasons during the timed region, read (never
    set) through NVML every 2 ms by a child process (so the sampling does not
    wait on this process's interpreter lock); nvidia-smi at 200 ms when NVML
    is missing."""

    # NVML clock-event reason bits
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap"}

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.proc = None
        self.child = None
        self.t = None
        try:  # NVML set-up (slow the first time) happens before the timed region
            self.child = self._start_child()
        except Exception:
            self.child = None

    def _start_child(self):
        import torch

        bus = ""
        try:
            p = torch.cuda.get_device_properties(self.idx)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        except Exception:
            pass
        c = subprocess.Popen([sys.executable, "-c", _NVML_CHILD, bus or "none", str(self.idx)],
                             stdin=subprocess.PIPE, stdout=subprocess.PIPE,
                             stderr=subprocess.DEVNULL, text=True)
        if c.stdout.readline().strip() != "ready":
            c.kill()
            c.wait()
            return None
        return c

    def __enter__(self):
        if self.child is not None:
            self._send("go")
            return self
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.idx)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._smi_read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _send(self, cmd):
        try:
            self.child.stdin.write(cmd + "\n")
            self.child.stdin.flush()
        except Exception:
            pass

    def pause(self):
        """Stop sampling between timed regions (NVML child only)."""
        if self.child is not None:
            self._send("pause")

    def resume(self):
        if self.child is not None:
            self._send("go")

    def _smi_read(self):
        bits = [0x8, 0x40, 0x20, 0x4]
        for line in self.proc.stdout:
            r = [v.strip() for v in line.split(",")]
            try:
                mask = sum(b for b, v in zip(bits, r[2:6]) if v.lower() == "active")
                self.rows.append((float(r[0]), float(r[1]), mask))
            except (ValueError, IndexError):
                continue

    def __exit__(self, *a):
        if self.child is not None:
            try:
                out, _ = self.child.communicate("stop\n", timeout=10)
                self.rows = [(float(s), float(m), int(b)) for s, m, b in json.loads(out or "[]")]
            except Exception:
                self.child.kill()
                self.child.wait()
            self.child = None
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.t is not None:
            self.t.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = sorted({n for _, _, m in self.rows for b, n in self.REASONS.items() if m & b})
        return {"sm_mhz": statistics.median(r[0] for r in self.rows),
                "sm_max_mhz": max(r[1] for r in self.rows), "reasons": reasons,
                "samples": len(self.rows)}


def make_field(device):
    import torch

    from latec_b200 import fields

    x = fields.turbulence_jumps(SHAPE, seed=0, device=device)
    mm = torch.aminmax(x)
    eb = REL_EB * (float(mm.max.item()) - float(mm.min.item()))
    return x, eb


def _timed(fn, steps):
    """Wall time per call of fn() over `steps` calls, the device synchronised
    on both sides (the public API includes host work)."""
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        out = fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / steps, out


def _roundtrip_leg(x, eb, levels, stride, steps, entropy="native"):
    """Compress + decompress of a device-resident field through the public
    API: GB/s of input each way, ratio, max error, and the codec-level
    fraction of the HBM roofline ((N s + S) bytes per direction)."""
    import latec_b200 as lb

    def pred():
        return lb.InterpPredictor("cubic", levels, stride, 1)

    # the native stream stays on the device; the compat stream's zstd frame
    # is built on the host, so it comes back as bytes
    where = "device" if entropy == "native" else "bytes"

    def enc():
        return lb.compress(x, eb, pred(), levels=levels, anchor_stride=stride, recon="none",
                           stream_out=where, entropy=entropy)[0]

    s = enc()  # warm-up: plans, tables, allocator
    lb.decompress(s, out="device")
    tc, s = _timed(enc, steps)
    td, out = _timed(lambda: lb.decompress(s, out="device"), steps)
    nbytes = x.numel() * x.element_size()
    err = float((out.double() - x.double()).abs().max().item())
    peak, kind = _peaks()
    sb = int(s.numel()) if entropy == "native" else len(s)
    return {"shape": list(x.shape), "dtype": str(x.dtype).replace("torch.", ""), "eb": eb,
            "entropy": entropy, "steps": steps,
            "compress_gbs": nbytes / tc / 1e9, "decompress_gbs": nbytes / td / 1e9,
            "roundtrip_gbs": nbytes / (tc + td) / 1e9, "compress_ms": tc * 1e3,
            "decompress_ms": td * 1e3, "ratio": nbytes / sb, "stream_bytes": sb,
            "max_abs_err": err, "bound_ok": err <= eb,
            "codec_roofline": {"compress_frac": (nbytes + sb) / tc / 1e9 / peak,
                               "decompress_frac": (nbytes + sb) / td / 1e9 / peak,
                               "bytes": "N s + S per direction", "peak": peak,
                               "peak_kind": kind}}


def cfg1_leg(dev, steps=20):
    """The reference's CPU-runnable configuration on the GPU: 512^2 float32
    SE-GRF (l = 16 px, seed 0), absolute eb 1e-3, cubic, levels 4, stride 16."""
    import torch

    from latec_b200 import fields

    x = torch.from_numpy(fields.grf_se((512, 512), 16.0, seed=0)).to(dev)
    out = _roundtrip_leg(x, 1e-3, 4, 16, steps)
    out["workload"] = "512^2 float32 SE-GRF l=16 seed 0, abs eb 1e-3, cubic, levels 4, stride 16"
    return out


def f64_leg(dev, steps=3):
    """The FP64 variant of the 3-D workload: 256^3 float64 turbulence + 3
    jumps, rel eb 1e-4 of the range, cubic, levels 6, stride 64 (prediction,
    reconstruction and bound check in float64)."""
    import torch

    from latec_b200 import fields

    x = fields.turbulence_jumps((256, 256, 256), seed=0, device=dev).double()
    mm = torch.aminmax(x)
    eb = REL_EB * (float(mm.max.item()) - float(mm.min.item()))
    out = _roundtrip_leg(x, eb, LEVELS, STRIDE, steps)
    out["workload"] = "256^3 float64 turbulence + 3 jumps, rel eb 1e-4, cubic, levels 6, stride 64"
    return out


def compat_leg(x, eb):
    """The drop-in stream (entropy="compat": the reference's single-stack rANS
    layout and level-9 zstd frame, readable by the reference decoder) on the
    512^3 workload: one timed round trip after a warm-up. The single-stack
    coder is serial by nature (one state chain per stage) and the zstd frame
    is built on the host."""
    import latec_b200 as lb

    out = _roundtrip_leg(x, eb, LEVELS, STRIDE, 1, entropy="compat")
    out["workload"] = "512^3 float32 turbulence + 3 jumps, rel eb 1e-4, compat stream"
    # where one compress spends its time: the device passes and the stage
    # coder (k_stack_encode) up to the payload download, then the host's
    # literal-zstd decisions and level-9 frame
    _s, st = lb.compress(x, eb, lb.InterpPredictor("cubic", LEVELS, STRIDE, 1), levels=LEVELS,
                         anchor_stride=STRIDE, recon="none", entropy="compat")
    out["compress_split_s"] = {"stages": st.get("predict_s"), "fit": st.get("fit_s"),
                               "rans_coder": st.get("rans_s"),
                               "host_literals_and_zstd_frame": st.get("download_s")}
    return out


def cpu_baseline(steps=1):
    """The oracle (NumPy restatement of the reference + C coder) on a sample."""
    import numpy as np

    from latec_b200 import fields
    from oracle import codec as ocodec

    x = fields.turbulence_jumps(SAMPLE, seed=0)
    eb = REL_EB * float(np.float64(x.max()) - np.float64(x.min()))
    best = None
    for _ in range(steps):
        t0 = time.perf_counter()
        stream, _st = ocodec.compress(x, eb, levels_=LEVELS, anchor_stride=STRIDE, mode="compat")
        ocodec.decompress(stream)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return x.nbytes / best / 1e9, x.nbytes / len(stream)


# DRAM bytes (read + write) of one encode pass (31 k_interp_quant and their
# compaction launches, the default per-stage path) on the 512^3 workload: an
# ncu capture of the pass on the 384^3 field of the same generator (1,752.8 MB
# for 56.6 M points), scaled by the points to 512^3; the per-stage kernels
# are unchanged since (same registers, same stack).
TRAFFIC_ENCODE_PASS = 4.155e9
TRAFFIC_SOURCE = ("ncu capture of the pass at 384^3 (dram__bytes_read.sum + "
                  "dram__bytes_write.sum), scaled by points to 512^3")
# The same for one launch of the opt-in fused finest-level encode (308.7 MB
# read + 277.5 MB written for the 49.5 M points of the 384^3 finest level).
TRAFFIC_FINEST_FUSED = (308.710144e6 + 277.469696e6) * (512.0 / 384.0) ** 3

GNN_SHAPE = (32, 32, 32, 32)
GNN_FULL_SHAPE = (128, 128, 64, 64)
GNN_CKPT = os.path.join(ROOT, "latec_b200", "checkpoints", "gnn_d64_agg1_synthetic.pt")
GNN_EB, GNN_LEVELS = 1e-3, 4


def gnn_leg(dev, steps=2):
    """Learned codec beside the plain one on one 32^4 chunk of the 4-D mixed
    field (0.5 anisotropic GRF + 0.5 turbulence+jumps; the reference's auto
    chunk of a 128x128x64x64 tensor), absolute eb 1e-3, levels 4, with the
    checkpoint trained by latec_b200.train on synthetic fields
    (latec_b200/checkpoints/gnn_d64_agg1_synthetic.pt).
    Wall time of compress + decompress through the public API with the field
    on the device."""
    import torch

    import latec_b200 as lb
    from latec_b200 import fields

    x = fields.mixed_4d(GNN_SHAPE, seed=3, device=dev)
    span = float(x.max().item()) - float(x.min().item())
    codec = lb.GNNCodec(checkpoint_path=GNN_CKPT, device=dev)
    rel = GNN_EB / span
    s = codec.compress(x, rel, levels=GNN_LEVELS)  # warm-up (geometry, tables)
    codec.uncompress(s)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        s = codec.compress(x, rel, levels=GNN_LEVELS)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(steps):
        out = codec.uncompress(s)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    err = float((out.to(dev) - x).abs().max().item())
    # float32 normalise / denormalise slack of the reference
    # (latec/gnn_codec.py:188-226): the bound is exact on the [0, 1] values
    vmin, vmax = float(x.min().item()), float(x.max().item())
    slack = 2.0 ** -24 * (3.0 * span + max(abs(vmin), abs(vmax)))
    si, _ = lb.compress(x, GNN_EB, lb.InterpPredictor("cubic", GNN_LEVELS, 16, 1),
                        levels=GNN_LEVELS, anchor_stride=16, recon="none")
    nbytes = x.numel() * 4
    return {"workload": "one 32^4 chunk of the 4-D mixed field, abs eb 1e-3, levels 4",
            "weights": "trained with latec_b200.train (hand-written forward/backward kernels), "
                       "797 AdamW steps of 16^4 x 4 + 128^2 x 16 synthetic fields; "
                       "latec_b200/checkpoints/gnn_d64_agg1_synthetic.pt",
            "ratio_gnn": nbytes / len(s), "ratio_interp": nbytes / len(si),
            "compress_gbs": nbytes * steps / (t1 - t0) / 1e9,
            "decompress_gbs": nbytes * steps / (t2 - t1) / 1e9,
            "max_abs_err": err, "bound": GNN_EB, "roundtrip_slack": slack, "dtype": "f32",
            "precision": gnn_precision(codec, x, rel),
            "full_tensor": gnn_full(dev, codec)}


def gnn_precision(codec, x, rel):
    """The same 32^4 chunk coded with the message MLPs in float32, BF16 and
    FP8 (the codec's fp16=False / fp16=True / fp8=True): stream bytes, and the
    model's predictions against the float32 run's, as max and RMS differences
    of mu and log2 b. At the first model stage every run sees the same coded
    anchors, so that stage isolates the network's precision; over all stages
    the later inputs also differ by the runs' own reconstructions. Errors are
    reported in the line instead of ending the bench."""
    import torch

    try:
        runs = {}
        for name, kw in (("f32", {"fp16": False}), ("bf16", {"fp16": True}),
                         ("fp8", {"fp16": True, "fp8": True})):
            codec.stage_trace = []
            try:
                s = codec.compress(x, rel, levels=GNN_LEVELS, **kw)
                trace = [(int(t["stage"]), t["mu"].double().reshape(-1),
                          torch.log2(t["scale"].double()).reshape(-1))
                         for t in codec.stage_trace]
            finally:
                codec.stage_trace = None
            runs[name] = (len(s), trace)

        def diff(a, b):
            d = (a - b).abs()
            return float(d.max().item()), float(d.pow(2).mean().sqrt().item())

        out = {"stream_bytes": {k: v[0] for k, v in runs.items()},
               "ratio": {k: x.numel() * 4 / v[0] for k, v in runs.items()}}
        ref = runs["f32"][1]
        for name in ("bf16", "fp8"):
            tr = runs[name][1]
            pairs = [(a, b) for a, b in zip(tr, ref) if a[0] == b[0] and a[1].numel() == b[1].numel()]
            # stage 0 holds the anchors, coded against 0 in every run
            first = next(((a, b) for a, b in pairs if a[0] > 0 and a[1].numel()), None)
            if first is None:
                continue
            mu_all = diff(torch.cat([a[1] for a, _ in pairs]), torch.cat([b[1] for _, b in pairs]))
            lb_all = diff(torch.cat([a[2] for a, _ in pairs]), torch.cat([b[2] for _, b in pairs]))
            out[name + "_vs_f32"] = {
                "first_model_stage": {"stage": first[0][0], "points": int(first[0][1].numel()),
                                      "mu_max": diff(first[0][1], first[1][1])[0],
                                      "mu_rms": diff(first[0][1], first[1][1])[1],
                                      "log2b_max": diff(first[0][2], first[1][2])[0],
                                      "log2b_rms": diff(first[0][2], first[1][2])[1]},
                "all_stages": {"stages": len(pairs), "mu_max": mu_all[0], "mu_rms": mu_all[1],
                               "log2b_max": lb_all[0], "log2b_rms": lb_all[1]}}
        out["units"] = "mu on the codec's normalised [0, 1] values; log2 b in bits"
        return out
    except Exception as e:  # a diagnostic leg: report, do not end the bench
        return {"error": f"{type(e).__name__}: {e}"}


def gnn_full(dev, codec):
    """The learned codec on the whole 128x128x64x64 4-D mixed field (256 MiB):
    64 chunks of 32^4 coded in same-shape batches; one timed round trip (the
    chunk geometry is already cached by the 32^4 leg)."""
    import torch

    import latec_b200 as lb
    from latec_b200 import fields
    from latec_b200.gnn_codec import read_stream

    x = fields.mixed_4d(GNN_FULL_SHAPE, seed=3, device=dev)
    vmin, vmax = float(x.min().item()), float(x.max().item())
    span = vmax - vmin
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s = codec.compress(x, GNN_EB / span, levels=GNN_LEVELS)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    out = codec.uncompress(s)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    err = float((out.to(dev) - x).abs().max().item())
    si, _ = lb.compress(x, GNN_EB, lb.InterpPredictor("cubic", GNN_LEVELS, 16, 1),
                        levels=GNN_LEVELS, anchor_stride=16, recon="none")
    nbytes = x.numel() * 4
    meta = read_stream(s)[0]
    return {"workload": "128x128x64x64 4-D mixed field (256 MiB), abs eb 1e-3, levels 4",
            "chunks": meta["chunks"], "chunk_batch": meta["chunk_batch"],
            "ratio_gnn": nbytes / len(s), "ratio_interp": nbytes / len(si),
            "compress_gbs": nbytes / (t1 - t0) / 1e9, "decompress_gbs": nbytes / (t2 - t1) / 1e9,
            "max_abs_err": err,
            "roundtrip_slack": 2.0 ** -24 * (3.0 * span + max(abs(vmin), abs(vmax)))}


def gnn_eval_1024(dev, ckpt=GNN_CKPT):
    """The learned codec against plain interpolation on a 1024^3 float32
    turbulence + jumps field (4 GiB, seed 5) at absolute eb 1e-4, auto levels
    (the learned codec's chunks of 128^3; interpolation at the same levels and
    stride): ratios, bound, one timed round trip each. Opt-in
    (``--gnn-eval-1024``): it holds about 40 GB on the device for a minute."""
    import torch

    import latec_b200 as lb
    from latec_b200 import fields
    from latec_b200.gnn_codec import read_stream

    x = fields.turbulence_jumps((1024, 1024, 1024), seed=5, device=dev)
    vmin, vmax = float(x.min().item()), float(x.max().item())
    span = vmax - vmin
    eb = 1e-4
    codec = lb.GNNCodec(checkpoint_path=ckpt, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s = codec.compress(x, eb / span)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    out = codec.uncompress(s)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    err = float((out.to(dev) - x).abs().max().item())
    del out
    meta = read_stream(s)[0]
    lv = int(meta["levels"])
    si, _ = lb.compress(x, eb, lb.InterpPredictor("cubic", lv, 1 << lv, 1), levels=lv,
                        anchor_stride=1 << lv, recon="none")
    nbytes = x.numel() * 4
    return {"workload": "1024^3 float32 turbulence + 3 jumps (seed 5), abs eb 1e-4, auto levels",
            "checkpoint": os.path.relpath(ckpt, ROOT), "levels": lv,
            "chunks": meta.get("chunks"), "chunk_batch": meta.get("chunk_batch"),
            "ratio_gnn": nbytes / len(s), "ratio_interp": nbytes / len(si),
            "compress_gbs": nbytes / (t1 - t0) / 1e9, "decompress_gbs": nbytes / (t2 - t1) / 1e9,
            "max_abs_err": err, "bound": eb,
            "roundtrip_slack": 2.0 ** -24 * (3.0 * span + max(abs(vmin), abs(vmax)))}


BATCH_N = 1000  # the whole multi-tensor population


def batch_shapes(n, seed=0):
    """The multi-tensor population: rank 2 or 3, volume log-uniform between
    64^2 and 256^3 (near-isotropic axes), 80 % float32 / 20 % float64, SE-GRF
    correlation length uniform in [2, 32]."""
    import numpy as np

    rs = np.random.RandomState(seed)
    out = []
    for i in range(n):
        rank = 2 if rs.rand() < 0.5 else 3
        vol = float(np.exp(rs.uniform(np.log(64 ** 2), np.log(256 ** 3))))
        edge = max(16, int(round(vol ** (1.0 / rank))))
        edge = min(edge, 4096 if rank == 2 else 256)
        shape = tuple(max(16, int(edge * f)) for f in rs.uniform(0.8, 1.25, rank))
        out.append((shape, rs.rand() < 0.2, float(rs.uniform(2, 32)), int(rs.randint(1 << 30))))
    return out


def shard(items, rank, world):
    """Independent units of a replicas-only job: rank r takes r, r + N, ..."""
    return list(items)[rank::world]


def reduce_over_ranks(values, op, world, device):
    """Sum or max of per-rank floats over all ranks (identity on one rank)."""
    if world == 1:
        return list(values)
    import torch
    import torch.distributed as dist

    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def batch_leg(dev, n=BATCH_N, rank=0, world=1):
    """Batched multi-tensor coding through the public API, tensors resident
    on the device: aggregate GB/s and per-tensor latency (compress +
    decompress), absolute eb 1e-3, cubic, levels 4, stride 16. Timed on the
    second pass over the tensors; the first (cold) pass is reported beside."""
    import torch

    import numpy as np

    import latec_b200 as lb
    from latec_b200 import fields

    tensors = []
    for shape, f64, ell, seed in shard(batch_shapes(n), rank, world):
        x = fields.grf_se(shape, ell, seed=seed, device=dev)
        tensors.append(x.double() if f64 else x)
    pred = lambda: lb.InterpPredictor("cubic", 4, 16, 1)  # noqa: E731
    # cold pass = warm-up: the first call at a new shape / model window builds
    # plans and entropy tables that later calls reuse
    torch.cuda.synchronize()
    tc0 = time.perf_counter()
    for x in tensors:
        s, _ = lb.compress(x, 1e-3, pred(), levels=4, anchor_stride=16, recon="none",
                           stream_out="device")
        lb.decompress(s, out="device")
    torch.cuda.synchronize()
    (cold,) = reduce_over_ranks([time.perf_counter() - tc0], "max", world, dev)
    lat, nbytes, sbytes = [], 0, 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for x in tensors:
        a = time.perf_counter()
        s, _ = lb.compress(x, 1e-3, pred(), levels=4, anchor_stride=16, recon="none",
                           stream_out="device")
        lb.decompress(s, out="device")
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - a)
        nbytes += x.numel() * x.element_size()
        sbytes += s.numel()
    total = time.perf_counter() - t0
    # the same tensors through the batch API: one compress_many and one
    # decompress_many call per rank, after the encode CTA caps are tuned for
    # the population's classes and one untimed call of each (the first call
    # puts every plan's stage descriptors on the device)
    from latec_b200 import _lib as blib

    tuned = lb.autotune_many(tensors, 1e-3, pred(), levels=4, anchor_stride=16)
    outs = lb.decompress_many(lb.compress_many(tensors, 1e-3, pred(), levels=4,
                                               anchor_stride=16, stream_out="device"),
                              out="device")
    del outs
    lib = blib.load()
    torch.cuda.synchronize()
    l0 = lib.latec_launch_count()
    tb0 = time.perf_counter()
    bs = lb.compress_many(tensors, 1e-3, pred(), levels=4, anchor_stride=16, stream_out="device")
    torch.cuda.synchronize()
    tb1 = time.perf_counter()
    l1 = lib.latec_launch_count()
    outs = lb.decompress_many(bs, out="device")
    torch.cuda.synchronize()
    tb2 = time.perf_counter()
    l2 = lib.latec_launch_count()
    del outs, bs
    # the tensors are sharded over the ranks: bytes add up, the slowest rank
    # sets the time
    nbytes, sbytes = reduce_over_ranks([nbytes, sbytes], "sum", world, dev)
    (total,) = reduce_over_ranks([total], "max", world, dev)
    tbc, tbd = reduce_over_ranks([tb1 - tb0, tb2 - tb1], "max", world, dev)
    lat_ms = np.sort(np.asarray(lat)) * 1e3
    return {"workload": f"{n} tensors sampled from the 1000-tensor population (rank 2/3, "
                        "volume log-uniform 64^2..256^3, 20 % float64, SE-GRF l 2..32), "
                        "abs eb 1e-3, cubic, levels 4, stride 16",
            "tensors": n, "bytes": nbytes, "gbs": nbytes / total / 1e9,
            "cold_pass_gbs": nbytes / cold / 1e9,
            "ratio": nbytes / sbytes, "latency_ms_p50": float(np.percentile(lat_ms, 50)),
            "latency_ms_p99": float(np.percentile(lat_ms, 99)),
            "mode": "serial loop over the public API per rank (one compress + decompress "
                    f"call per tensor), tensors sharded over {world} rank(s)",
            "latency_scope": "rank 0's tensors",
            "batch_api": {"call": "compress_many + decompress_many, one call each per rank",
                          "gbs": nbytes / (tbc + tbd) / 1e9,
                          "compress_gbs": nbytes / tbc / 1e9,
                          "decompress_gbs": nbytes / tbd / 1e9,
                          "launches_compress": int(l1 - l0),
                          "launches_decompress": int(l2 - l1),
                          "stage_launches": "one per stage index and kernel class over all "
                                            "tensors (latec_encode_stages_many / "
                                            "latec_decode_stages_many)",
                          "cta_caps": {"/".join(map(str, k)): v[0]
                                       for k, v in sorted(tuned.items())},
                          "cta_caps_key": "rank/value bytes/size class (points < 64Ki, "
                                          "< 512Ki, < 4Mi, larger)"}}


_CPU_SAMPLE = None


def _cpu_worker_init():
    """Process-pool initializer: each worker builds its own copy of the sample."""
    global _CPU_SAMPLE
    import numpy as np

    from latec_b200 import fields

    x = fields.turbulence_jumps(SAMPLE, seed=0)
    _CPU_SAMPLE = (x, REL_EB * float(np.float64(x.max()) - np.float64(x.min())))


def _cpu_roundtrip(_task):
    """One compress + decompress of the worker's sample with the CPU oracle
    (compat mode); returns (input bytes, stream bytes)."""
    from oracle import codec as ocodec

    x, eb = _CPU_SAMPLE
    s, _ = ocodec.compress(x, eb, levels_=LEVELS, anchor_stride=STRIDE, mode="compat")
    ocodec.decompress(s)
    return x.nbytes, len(s)


def run_reference(args, rank):
    """The reference arm: the CPU path on every host core. One worker process
    per core (spawned, one NumPy thread each) codes its own 128^3 sample per
    step; the step is the wall time of all workers' round trips, so the value
    is the host's whole-job throughput."""
    if rank != 0:
        return
    import multiprocessing as mp

    cores = (len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity")
             else os.cpu_count()) or 1
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    with mp.get_context("spawn").Pool(cores, initializer=_cpu_worker_init) as pool:
        tasks = range(cores)
        for _ in range(1 + args.warmup):  # the first map pays the workers' imports
            pool.map(_cpu_roundtrip, tasks, chunksize=1)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            res = pool.map(_cpu_roundtrip, tasks, chunksize=1)
        dt = (time.perf_counter() - t0) / max(1, args.steps)
    nbytes = sum(r[0] for r in res)
    v = nbytes / dt / 1e9
    sample = (f"{cores} x {SAMPLE[0]}^3 float32 samples of the same generator per step, one "
              f"per worker process (the GPU arm codes one {SHAPE[0]}^3 field per step; the "
              "full field is ~minutes per step on one core)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "ratio": res[0][0] / res[0][1],
        "config": {"workload": "plain interp codec, turbulence+3 jumps, cubic, levels 6, "
                               "stride 64, rel eb 1e-4", "shape": list(SAMPLE),
                   "samples_per_step": cores},
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": cores, "kind": "port",
                         "sample": sample, "nproc": os.cpu_count(),
                         "pinning": "one spawned worker process per core in the affinity "
                                    "mask, one NumPy thread each; not pinned to cores"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_profile(args, dev):
    """Warm-up plus timed device-resident round trips at --shape, with the
    per-phase wall times the codec records; used under ncu for launch lists."""
    import torch

    import latec_b200 as lb
    from latec_b200 import fields

    shape = tuple(args.shape) if args.shape else SHAPE
    x = fields.turbulence_jumps(shape, seed=0, device=dev)
    mm = torch.aminmax(x)
    eb = REL_EB * (float(mm.max.item()) - float(mm.min.item()))
    rows = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        a = time.perf_counter()
        stream, st = lb.compress(x, eb, lb.InterpPredictor("cubic", LEVELS, STRIDE, 1),
                                 levels=LEVELS, anchor_stride=STRIDE, recon="none")
        b = time.perf_counter()
        out = lb.decompress(stream, out="device")
        torch.cuda.synchronize()
        c = time.perf_counter()
        if i >= args.warmup:
            rows.append({"compress_ms": (b - a) * 1e3, "decompress_ms": (c - b) * 1e3,
                         "stages_ms": st["predict_s"] * 1e3, "entropy_ms": st["entropy_s"] * 1e3,
                         "fit_ms": st["fit_s"] * 1e3, "rans_ms": st["rans_s"] * 1e3,
                         "download_ms": st["download_s"] * 1e3,
                         "bytes": len(stream)})
        del out
    print(json.dumps({"profile": list(shape), "eb": eb, "ratio": x.numel() * 4 / len(stream),
                      "rows": rows}), flush=True)


def run_profile_gnn(args, dev):
    """The learned codec on one 32^4 chunk of the 4-D mixed field: warm-up
    round trips, then one compress + decompress inside a CUDA profiler range
    (``ncu --profile-from-start off`` captures only those launches)."""
    import torch

    import latec_b200 as lb
    from latec_b200 import fields

    x = fields.mixed_4d(GNN_SHAPE, seed=3, device=dev)
    rel = GNN_EB / (float(x.max().item()) - float(x.min().item()))
    codec = lb.GNNCodec(checkpoint_path=GNN_CKPT, device=dev)
    for _ in range(max(1, args.warmup)):
        codec.uncompress(codec.compress(x, rel, levels=GNN_LEVELS))
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    a = time.perf_counter()
    s = codec.compress(x, rel, levels=GNN_LEVELS)
    torch.cuda.synchronize()
    b = time.perf_counter()
    codec.uncompress(s)
    torch.cuda.synchronize()
    c = time.perf_counter()
    torch.cuda.cudart().cudaProfilerStop()
    print(json.dumps({"profile_gnn": list(GNN_SHAPE), "ratio": x.numel() * 4 / len(s),
                      "compress_ms": (b - a) * 1e3, "decompress_ms": (c - b) * 1e3}), flush=True)


def run_profile_batch(args, dev):
    """The batch API on the first ``--profile-batch`` tensors of the
    multi-tensor population: warm-up calls, then one compress_many +
    decompress_many inside a CUDA profiler range (``ncu --profile-from-start
    off`` captures only those launches)."""
    import torch

    import latec_b200 as lb
    from latec_b200 import fields

    tensors = []
    for shape, f64, ell, seed in batch_shapes(BATCH_N)[:args.profile_batch]:
        x = fields.grf_se(shape, ell, seed=seed, device=dev)
        tensors.append(x.double() if f64 else x)
    pred = lambda: lb.InterpPredictor("cubic", 4, 16, 1)  # noqa: E731
    for _ in range(max(1, args.warmup)):
        lb.decompress_many(lb.compress_many(tensors, 1e-3, pred(), levels=4, anchor_stride=16,
                                            stream_out="device"), out="device")
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    a = time.perf_counter()
    bs = lb.compress_many(tensors, 1e-3, pred(), levels=4, anchor_stride=16, stream_out="device")
    torch.cuda.synchronize()
    b = time.perf_counter()
    lb.decompress_many(bs, out="device")
    torch.cuda.synchronize()
    c = time.perf_counter()
    torch.cuda.cudart().cudaProfilerStop()
    nbytes = sum(x.numel() * x.element_size() for x in tensors)
    print(json.dumps({"profile_batch": len(tensors), "bytes": nbytes,
                      "compress_ms": (b - a) * 1e3, "decompress_ms": (c - b) * 1e3}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="latec_b200", choices=["latec_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gnn", action="store_true", help="skip the learned-codec leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the multi-tensor leg")
    ap.add_argument("--no-compat", action="store_true",
                    help="skip the reference-readable (compat) stream leg")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the 512^2 and float64 256^3 legs")
    ap.add_argument("--profile", action="store_true",
                    help="only warm-up + timed device round trips (for ncu launch lists)")
    ap.add_argument("--shape", type=int, nargs="+", default=None,
                    help="field shape for --profile (default 512 512 512)")
    ap.add_argument("--profile-gnn", action="store_true",
                    help="only the learned codec's round trip on one 32^4 chunk, inside a CUDA "
                         "profiler range (for ncu launch lists)")
    ap.add_argument("--profile-batch", type=int, default=0,
                    help="only the batch API on the first N population tensors, inside a CUDA "
                         "profiler range (for ncu launch lists)")
    ap.add_argument("--gnn-eval-1024", action="store_true",
                    help="only the learned codec against interpolation on a 1024^3 field "
                         "(one JSON line)")
    ap.add_argument("--gnn-ckpt", default=None,
                    help="checkpoint for --gnn-eval-1024 (default: the shipped one)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    import latec_b200 as lb
    from latec_b200 import _lib

    lib = _lib.load()
    if args.profile:
        return run_profile(args, dev)
    if args.profile_gnn:
        return run_profile_gnn(args, dev)
    if args.profile_batch:
        return run_profile_batch(args, dev)
    if args.gnn_eval_1024:
        print(json.dumps({"gnn_eval_1024": gnn_eval_1024(dev, args.gnn_ckpt or GNN_CKPT)}),
              flush=True)
        return 0
    x, eb = make_field(dev)
    nbytes = x.numel() * x.element_size()

    def pred():
        return lb.InterpPredictor("cubic", LEVELS, STRIDE, 1)

    def step_device():
        stream, st = lb.compress(x, eb, pred(), levels=LEVELS, anchor_stride=STRIDE, recon="none",
                                 stream_out="device")
        out = lb.decompress(stream, out="device")
        return stream, st, out

    for _ in range(max(3, args.warmup)):
        stream, st, out = step_device()
    del out
    # ---- device-resident timed region
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    l0 = lib.latec_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # clocks sampled during both timed regions (device-resident and end to
    # end), paused in between
    sampler = ClockSampler(local)  # NVML set-up before the timed region
    sampler.__enter__()
    ev0.record()
    tc = td = 0.0
    for _ in range(args.steps):
        a = time.perf_counter()
        stream, st = lb.compress(x, eb, pred(), levels=LEVELS, anchor_stride=STRIDE,
                                 recon="none", stream_out="device")
        b = time.perf_counter()
        out = lb.decompress(stream, out="device")
        torch.cuda.synchronize()
        c = time.perf_counter()
        tc += b - a
        td += c - b
        del out
    ev1.record()
    torch.cuda.synchronize()
    sampler.pause()
    launches = lib.latec_launch_count() - l0
    ms = ev0.elapsed_time(ev1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = world * nbytes / (ms / 1e3) / 1e9
    ratio = nbytes / len(stream)

    # ---- roofline. The dominant work is the encode pass (latec_encode_stages:
    # one k_interp_quant launch per stage and its outlier compaction, the
    # default per-stage launches), timed with CUDA events on the launching
    # stream. Beside it the opt-in fused finest level (k_lvl_enc / k_lvl_dec,
    # timed by the event pairs the library records around each fused launch),
    # the lane coders, and the codec-level fractions.
    from latec_b200 import codec as lcodec
    from latec_b200 import levels as llevels

    plan = llevels.plan_for(SHAPE, LEVELS, STRIDE, 1)
    enc = lcodec._Encoder(x.reshape((1,) + SHAPE), SHAPE, 1, 1, LEVELS, STRIDE, 1, 1 << 15,
                          "cubic", "native", 9, dev)
    ebs = llevels.stage_ebs(SHAPE, LEVELS, STRIDE, 1, eb, 0.9)
    import ctypes

    prm = lcodec._qparams(1, 1, 1 << 15, "cubic", 0, 1, False)
    eb_arr = (ctypes.c_double * len(plan))(*[float(e) for e in ebs])
    rc = torch.empty_like(x)
    b = enc.buf
    s_ptr = torch.cuda.current_stream().cuda_stream
    kms, kn = ctypes.c_double(), ctypes.c_uint32()

    def kernel_ms(kind):
        _lib.check(lib.latec_kernel_time(kind, ctypes.byref(kms), ctypes.byref(kn)))
        return kms.value / max(1, kn.value), int(kn.value)

    def encode_pass():
        _lib.check(lib.latec_encode_stages(plan.handle, ctypes.byref(prm), eb_arr, x.data_ptr(),
                                           rc.data_ptr(), b.codes.data_ptr(), b.outliers.data_ptr(),
                                           b.stats.data_ptr(), b.hist_seg.data_ptr(),
                                           b.hist_total.data_ptr(), b.ws.data_ptr(), b.ws.numel(),
                                           s_ptr))

    times = []
    for i in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        rc.zero_()
        e0.record()
        encode_pass()
        e1.record()
        torch.cuda.synchronize()
        if i:
            times.append(e0.elapsed_time(e1))
    pass_ms = statistics.median(times)
    # the opt-in fused finest level (tile mode 1) and the lane coders, timed
    # with events over whole round trips
    _lib.check(lib.latec_set_tile_mode(1))
    _lib.check(lib.latec_set_kernel_timing(1))
    for kind in range(6):
        kernel_ms(kind)
    for i in range(3):
        s_k, _ = lb.compress(x, eb, pred(), levels=LEVELS, anchor_stride=STRIDE, recon="none",
                             stream_out="device")
        out = lb.decompress(s_k, out="device")
    del out, s_k
    torch.cuda.synchronize()
    kt = {k: kernel_ms(k) for k in range(6)}
    _lib.check(lib.latec_set_kernel_timing(0))
    _lib.check(lib.latec_set_tile_mode(0))
    n_fine = sum(plan.counts[-5:])  # the finest level's five sub-stages
    n_coarse = sum(plan.counts) - n_fine
    es = 4  # float32
    enc_alg = n_fine * (es + es + 2) + n_coarse * es   # read x, write recon + code; coarse taps
    dec_alg = n_fine * (2 + es) + n_coarse * es        # read code, write recon; coarse taps
    enc_ms, n_enc = kt[0]
    dec_ms, n_dec = kt[1]
    peak, peak_kind = _peaks()
    alg_bytes = sum(plan.counts) * (es + es + 2)
    achieved = alg_bytes / (pass_ms / 1e3) / 1e9
    kernels = {
        "fused_finest_encode": {"kernel": "k_lvl_enc<float,1,1> (TMA planes; opt-in, tile mode 1)",
                                "launches": n_enc, "alg_bytes": enc_alg, "kernel_ms": enc_ms,
                                "achieved_gbs": enc_alg / (enc_ms / 1e3) / 1e9 if enc_ms else 0.0,
                                "frac": enc_alg / (enc_ms / 1e3) / 1e9 / peak if enc_ms else 0.0,
                                "traffic": TRAFFIC_FINEST_FUSED},
        "fused_finest_decode": {"kernel": "k_lvl_dec<float,1,1> (TMA planes; opt-in, tile mode 1)",
                                "launches": n_dec, "alg_bytes": dec_alg, "kernel_ms": dec_ms,
                                "achieved_gbs": dec_alg / (dec_ms / 1e3) / 1e9 if dec_ms else 0.0,
                                "frac": dec_alg / (dec_ms / 1e3) / 1e9 / peak if dec_ms else 0.0},
        # per round trip (three were timed): the lane rANS coder, one launch
        # each way
        "lane_encode_ms": kt[2][0] * kt[2][1] / 3, "lane_decode_ms": kt[3][0] * kt[3][1] / 3,
    }
    del rc, enc
    # the drop-in (reference-readable) stream on the same field
    compat_line = None if args.no_compat else compat_leg(x, eb)

    # ---- end to end through host buffers (pinned host input, bytes stream,
    # NumPy output)
    xh = torch.empty(SHAPE, dtype=torch.float32, pin_memory=True)
    xh.copy_(x.cpu())
    xh_np = xh
    del x
    torch.cuda.empty_cache()
    for _ in range(max(3, args.warmup)):  # first calls pay the page-locked allocations
        s_e, _ = lb.compress(xh_np, eb, pred(), levels=LEVELS, anchor_stride=STRIDE, recon="none",
                             stream_out="numpy")
        back = lb.decompress(s_e)
    del back
    torch.cuda.synchronize()
    sampler.resume()
    t0 = time.perf_counter()
    e_steps = max(1, args.steps)
    for _ in range(e_steps):
        s_e, _ = lb.compress(xh_np, eb, pred(), levels=LEVELS, anchor_stride=STRIDE, recon="none",
                             stream_out="numpy")
        back = lb.decompress(s_e)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / e_steps
    sampler.__exit__(None, None, None)
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = world * nbytes / e2e_s / 1e9
    assert back.shape == SHAPE

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, _r = cpu_baseline()
        cpu = {"value": v, "unit": "GB/s", "cores": 1, "kind": "port",
               "sample": f"{SAMPLE[0]}^3 float32 field of the same generator (the GPU codes "
                         f"{SHAPE[0]}^3), one compress + decompress round trip with the CPU "
                         "oracle (NumPy + C rANS, compat mode)",
               "nproc": os.cpu_count(), "pinning": "none: the NumPy restatement and the C "
                                                   "coder run on one thread"}
    cfg1_line = None if args.no_extra else cfg1_leg(dev)
    f64_line = None if args.no_extra else f64_leg(dev)
    gnn_line = None if args.no_gnn else gnn_leg(dev)
    batch_line = None if args.no_batch else batch_leg(dev, rank=rank, world=world)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "ratio": ratio, "stream_bytes": int(len(stream)),
        "compress_gbs": nbytes * args.steps / tc / 1e9, "decompress_gbs": nbytes * args.steps / td / 1e9,
        "config": {"workload": "plain interp codec: 512^3 float32 turbulence (k^-5/3) + 3 jumps, "
                               "cubic, levels 6, anchor_stride 64, abs eb = 1e-4 x range, "
                               "native 32-lane rANS",
                   "shape": list(SHAPE), "eb": eb, "parallelism": f"replicas x{world}",
                   "l2": "input 512 MiB > 126 MB L2, no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": TRAFFIC_ENCODE_PASS,
                     "traffic_source": TRAFFIC_SOURCE,
                     "kernel": "encode pass (latec_encode_stages): 31 k_interp_quant launches, "
                               "one per stage, and their outlier compaction; 134.2 M points",
                     "alg_bytes": alg_bytes, "pass_ms": pass_ms, "peak_kind": peak_kind,
                     "kernels": kernels},
        "codec_roofline": {"compress_frac": (nbytes + len(stream)) * args.steps / tc / 1e9 / peak,
                           "decompress_frac": (nbytes + len(stream)) * args.steps / td / 1e9 / peak,
                           "bytes": "N s + S per direction (read the field, write the stream; "
                                    "read the stream, write the field)"},
        "compat": compat_line,
        "cfg1": cfg1_line,
        "f64_256": f64_line,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "GB/s", "h2d_bytes_per_step": nbytes + len(s_e),
                "d2h_bytes_per_step": nbytes + len(s_e)},
        "gpu_launches": int(launches),
        "gnn": gnn_line,
        "batch": batch_line,
        "clocks": sampler.summary(),
    }), flush=True)


if __name__ == "__main__":
    main()
