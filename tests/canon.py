"""Canonical form of a tetrahedral mesh in torch (CPU or GPU) and its digest.

The same canonical form as oracle.canonical (sorted vertex ids per
tetrahedron, tetrahedra sorted lexicographically, adjacency rewritten as
canonical indices, -1 on the hull), computed with torch so that meshes of tens
of millions of tetrahedra canonicalise in a second on the GPU. The digest is
the SHA-256 of the int32 little-endian bytes of V then A, so a mesh can be
compared with an oracle result recorded as a digest in tests/golden/.
"""
import hashlib

import numpy as np


def canonical_torch(tets, device=None):
    """tets: (T, 8) int32 array or tensor [v0..v3, opp0..opp3]. Returns
    (V, A) as int32 numpy arrays, equal to oracle.canonical(tets)."""
    import torch
    t = torch.as_tensor(np.asarray(tets)) if not isinstance(tets, torch.Tensor) else tets
    if device is not None:
        t = t.to(device)
    if t.shape[0] == 0:
        z = np.zeros((0, 4), np.int32)
        return z, z.copy()
    v = t[:, :4].to(torch.int64)
    opp = t[:, 4:8].to(torch.int64)
    vs, srt = torch.sort(v, dim=1, stable=True)
    os_ = torch.gather(opp, 1, srt)
    # lexicographic order of the sorted rows: two stable passes on 46-bit keys
    # (vertex ids below 2^23)
    assert int(vs.max()) < (1 << 23)
    lo = (vs[:, 2] << 23) | vs[:, 3]
    hi = (vs[:, 0] << 23) | vs[:, 1]
    o1 = torch.sort(lo, stable=True).indices
    o2 = torch.sort(hi[o1], stable=True).indices
    order = o1[o2]
    new_index = torch.empty_like(order)
    new_index[order] = torch.arange(len(order), device=order.device)
    V = vs[order]
    O = os_[order]
    A = torch.where(O >= 0, new_index[O.clamp(min=0)], torch.full_like(O, -1))
    return V.to(torch.int32).cpu().numpy(), A.to(torch.int32).cpu().numpy()


def digest(V, A):
    """SHA-256 hex digests of the canonical vertex and adjacency arrays."""
    v = np.ascontiguousarray(V, dtype="<i4")
    a = np.ascontiguousarray(A, dtype="<i4")
    return hashlib.sha256(v.tobytes()).hexdigest(), hashlib.sha256(a.tobytes()).hexdigest()
