"""Records the oracle's results on the full-size benchmark configurations as
digests (tests/golden/fullsize.json).

The full-size meshes (up to 54M tetrahedra for the 8M-point cloud) are too
large to commit and too slow for the CPU oracle to recompute on every GPU test
run, so this script triangulates each configuration once with the oracle
(oracle/, a C restatement of the reference pipeline whose predicates are pinned
to the reference's own code) and stores, per configuration: the tetrahedron
count and the SHA-256 digests of the canonical vertex and adjacency arrays
(tests/canon.py). The GPU tests canonicalise their own result and compare the
digests. Before writing, each result is certified by the oracle's validator
(Euler characteristic, orientation, local Delaunay with SoS, symmetric
adjacency) when the cloud is small enough to validate here.

Clouds come from gstar4d_b200.workloads with the configurations' seeds (numpy's
PCG64 streams are platform independent, so the GPU host regenerates the same
bytes); a digest of each cloud's coordinates is stored too and checked first.

    python tests/golden/gen_fullsize.py [name ...]
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))

OUT = os.path.join(HERE, "fullsize.json")

# name -> (workload, grid); seeds are the workloads' defaults (1)
CONFIGS = {
    "uniform100k": ("uniform100k", 256),
    "degenerate500k": ("degenerate500k", 512),
    "mixed1m": ("mixed1m", 512),
    "clustered8m": ("clustered8m", 1024),
}
VALIDATE_MAX = 1_100_000  # points; the validator is single-threaded


def cloud_digest(pts):
    return hashlib.sha256(np.ascontiguousarray(pts, dtype="<f8").tobytes()).hexdigest()


def main(names):
    from gstar4d_b200 import workloads
    from oracle import oracle_py
    import canon
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    for name in names:
        wl, G = CONFIGS[name]
        pts, _ = workloads.config_cloud(wl)
        t0 = time.time()
        tets, order, st = oracle_py.triangulate(pts, G)
        t1 = time.time()
        V, A = canon.canonical_torch(tets)
        dv, da = canon.digest(V, A)
        rec = {"points": int(len(pts)), "grid": G, "cloud_sha256": cloud_digest(pts), "tets": int(len(tets)),
               "V_sha256": dv, "A_sha256": da, "oracle_seconds": round(t1 - t0, 1),
               "oracle_threads": os.cpu_count(), "splay_loops": int(st["loops"])}
        if len(pts) <= VALIDATE_MAX:
            rank = np.empty(len(pts), np.int32)
            rank[order] = np.arange(len(pts), dtype=np.int32)
            rep = oracle_py.validate(pts, tets, rank)
            bad = {k: rep[k] for k in ("orient_fail", "insphere_fail", "adjacency_asym", "sos_fail")}
            assert rep["euler"] == 1 and not any(bad.values()), (name, rep)
            rec["validated"] = True
        else:
            rec["validated"] = False
        data[name] = rec
        print(name, json.dumps(rec), flush=True)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
            f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1:] or list(CONFIGS))
