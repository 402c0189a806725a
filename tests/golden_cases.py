"""Loads the golden fixtures (generated from the reference by
tests/golden/make_golden.py)."""
import json
import os

import numpy as np

from gkc_b200 import synth

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def index():
    with open(os.path.join(HERE, "golden.json")) as f:
        return json.load(f)


def full_case(name):
    z = np.load(os.path.join(HERE, f"case_{name}.npz"))
    meta = index()["full"][name]
    return meta, {k: z[k] for k in z.files}


def multisets_from_case(d, nbins):
    out = [[] for _ in range(nbins)]
    for b, ln, o in zip(d["skm_bin"], d["skm_len"], d["skm_off"]):
        nb = (int(ln) + 3) // 4
        out[int(b)].append((int(ln), d["skm_bytes"][int(o):int(o) + nb].tobytes()))
    return out


def digest_case_reads(c):
    if c["gen"] == "iid":
        return synth.iid_reads(c["seed"], c["n_reads"], c["read_len"], c["n_rate"])
    g = synth.genome(c["seed"], c["genome_len"])
    n = c["coverage"] * c["genome_len"] // c["read_len"]
    return synth.short_reads(c["seed"], g, n, c["read_len"], c["err"])
