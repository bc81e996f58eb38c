"""The torch canonical form used by the full-size GPU tests equals the oracle's
numpy canonical form (CPU tensors here), and the recorded full-size digests
are well formed."""
import json
import os

import numpy as np

import canon
from gstar4d_b200 import workloads

HERE = os.path.dirname(os.path.abspath(__file__))


def test_torch_canonical_equals_oracle_canonical(oracle):
    pts = workloads.mixed(4000, seed=21)
    tets, _, _ = oracle.triangulate(pts, 64)
    # a shuffled copy with rotated vertex slots is the same mesh
    rng = np.random.default_rng(3)
    perm = rng.permutation(len(tets))
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    sh = tets[perm].copy()
    sh[:, 4:] = np.where(sh[:, 4:] >= 0, inv[np.clip(sh[:, 4:], 0, None)], -1)
    for t in (tets, sh):
        V, A = canon.canonical_torch(t)
        rV, rA = oracle.canonical(t)
        assert np.array_equal(V, rV) and np.array_equal(A, rA)
    assert canon.digest(*canon.canonical_torch(tets)) == canon.digest(*canon.canonical_torch(sh))


def test_fullsize_digests_recorded():
    with open(os.path.join(HERE, "golden", "fullsize.json")) as f:
        gold = json.load(f)
    for name in ("uniform100k", "degenerate500k", "mixed1m", "clustered8m"):
        rec = gold[name]
        assert rec["tets"] > 6 * rec["points"] * 0.8
        assert len(rec["V_sha256"]) == 64 and len(rec["A_sha256"]) == 64


def test_fullsize_digest_matches_oracle_on_the_100k_cloud(oracle):
    """The recorded digest of the 100k configuration is the oracle's result
    recomputed here (the larger ones take minutes on the CPU)."""
    with open(os.path.join(HERE, "golden", "fullsize.json")) as f:
        rec = json.load(f)["uniform100k"]
    pts, G = workloads.config_cloud("uniform100k")
    tets, _, _ = oracle.triangulate(pts, G)
    assert canon.digest(*canon.canonical_torch(tets)) == (rec["V_sha256"], rec["A_sha256"])
