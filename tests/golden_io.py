"""Readers for the committed golden vectors (written by tests/golden/make_golden.py)."""

import glob
import hashlib
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load_npz(name):
    z = np.load(os.path.join(GOLDEN, name))
    out = {k: z[k] for k in z.files}
    if "meta" in out:
        out["meta"] = json.loads(out["meta"].tobytes().decode())
    return out


def codec_case_names():
    return sorted(os.path.basename(p)[6:-4] for p in glob.glob(os.path.join(GOLDEN, "codec_*.npz")))


def schedule_cases():
    with open(os.path.join(GOLDEN, "schedule.json")) as f:
        return json.load(f)
