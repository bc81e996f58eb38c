"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker, and by bench.py for the timed CPU baseline. The product path
(gstar4d_b200) never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


class OraTet(ctypes.Structure):
    _fields_ = [("v", ctypes.c_int * 4), ("opp", ctypes.c_int * 4)]


class OraStats(ctypes.Structure):
    _fields_ = [
        ("points", ctypes.c_int), ("grid", ctypes.c_int), ("missing", ctypes.c_int),
        ("loops", ctypes.c_int), ("max_link", ctypes.c_int),
        ("voronoi_pairs", ctypes.c_longlong), ("workset_total", ctypes.c_longlong),
        ("star_insertions", ctypes.c_longlong), ("splay_insertions", ctypes.c_longlong),
        ("drowned", ctypes.c_longlong), ("proofs", ctypes.c_longlong),
        ("exact_calls", ctypes.c_longlong), ("consistency_repairs", ctypes.c_longlong),
        ("t_order", ctypes.c_double), ("t_pba", ctypes.c_double), ("t_star", ctypes.c_double),
        ("t_splay", ctypes.c_double), ("t_out", ctypes.c_double), ("t_total", ctypes.c_double),
        ("max_hist", ctypes.c_int),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def reference_root():
    """Where the reference sources are mounted: $REF_ROOT, else the container's
    default mount; None when absent (e.g. on the GPU host)."""
    root = os.environ.get("REF_ROOT", "/root/reference")
    return root if os.path.isdir(os.path.join(root, "GDelaunay")) else None


def build():
    """Builds liboracle.so (and oracle/_ref when the reference is mounted)."""
    subprocess.check_call(["make", "-s", "-C", HERE])
    root = reference_root()
    if root:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", "REF_ROOT=" + root])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", HERE])
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.ora_triangulate.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.POINTER(OraTet)), ctypes.POINTER(ctypes.c_int),
                                      vp, ctypes.POINTER(OraStats)]
        L.ora_validate.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, vp]
        L.ora_morton_order.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
        L.ora_edt.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
        L.ora_orient3d.argtypes = [vp, vp, vp, vp]
        L.ora_insphere.argtypes = [vp, vp, vp, vp, vp]
        L.ora_orient4_sos.argtypes = [vp, vp]
        L.ora_sos_only.argtypes = [vp, vp, vp]
        L.ora_free.argtypes = [vp]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def triangulate(points, grid, threads=0, input_order=True):
    """Returns (tets (T,8) int32 [v0..v3, opp0..opp3], sorted_to_input, stats dict)."""
    L = lib()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    n = len(pts)
    tp = ctypes.POINTER(OraTet)()
    nt = ctypes.c_int(0)
    order = np.zeros(n, dtype=np.int32)
    st = OraStats()
    rc = L.ora_triangulate(_ptr(pts), n, grid, threads, 1 if input_order else 0,
                           ctypes.byref(tp), ctypes.byref(nt), _ptr(order), ctypes.byref(st))
    if rc != 0:
        raise RuntimeError("oracle triangulation failed with status %d" % rc)
    if nt.value:
        flat = np.ctypeslib.as_array(ctypes.cast(tp, ctypes.POINTER(ctypes.c_int)), shape=(nt.value * 8,))
        tets = flat.reshape(-1, 8).copy()
    else:
        tets = np.zeros((0, 8), np.int32)
    L.ora_free(ctypes.cast(tp, ctypes.c_void_p))
    return tets, order, st.as_dict()


def validate(points, tets, rank):
    """Returns dict of the validator's counters (all failure counts must be 0)."""
    L = lib()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    t = np.ascontiguousarray(tets, dtype=np.int32)
    r = np.ascontiguousarray(rank, dtype=np.int32)
    rep = np.zeros(10, dtype=np.int64)
    L.ora_validate(_ptr(pts), len(pts), _ptr(r), _ptr(t), len(t), _ptr(rep))
    keys = ["euler", "orient_fail", "insphere_fail", "adjacency_asym", "sos_fail", "V", "E", "F", "T", "hull_faces"]
    return dict(zip(keys, rep.tolist()))


def morton_order(points, grid):
    L = lib()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    n = len(pts)
    order = np.zeros(n, np.int32)
    vox = np.zeros((n, 3), np.int32)
    rc = L.ora_morton_order(_ptr(pts), n, grid, _ptr(order), _ptr(vox))
    if rc:
        raise RuntimeError("morton order failed %d" % rc)
    return order, vox


def edt(voxel_sorted, grid):
    L = lib()
    v = np.ascontiguousarray(voxel_sorted, dtype=np.int32)
    site = np.zeros(grid ** 3, np.int32)
    rc = L.ora_edt(_ptr(v), len(v), grid, _ptr(site))
    if rc:
        raise RuntimeError("edt failed %d" % rc)
    return site


def orient3d(p4):
    a = np.ascontiguousarray(p4, dtype=np.float64).ravel()
    return lib().ora_orient3d(*[ctypes.c_void_p(a.ctypes.data + 24 * i) for i in range(4)])


def insphere(p5):
    a = np.ascontiguousarray(p5, dtype=np.float64).ravel()
    return lib().ora_insphere(*[ctypes.c_void_p(a.ctypes.data + 24 * i) for i in range(5)])


def orient4_sos(p5, idx5):
    a = np.ascontiguousarray(p5, dtype=np.float64).ravel()
    i = np.ascontiguousarray(idx5, dtype=np.int32)
    return lib().ora_orient4_sos(_ptr(a), _ptr(i))


def canonical(tets, n_points=None):
    """Canonical form of a tetrahedral mesh for bit-exact comparison.

    Each tet's vertices are sorted, tets are sorted lexicographically, and each
    tet's adjacency is rewritten as, for every sorted vertex position, the
    canonical index of the tet across the opposite face (-1 if none).
    Returns (V (T,4) int32, A (T,4) int32).
    """
    t = np.asarray(tets)
    if len(t) == 0:
        return np.zeros((0, 4), np.int32), np.zeros((0, 4), np.int32)
    v = t[:, :4].astype(np.int64)
    opp = t[:, 4:8].astype(np.int64)
    srt = np.argsort(v, axis=1, kind="stable")
    vs = np.take_along_axis(v, srt, axis=1)
    os_ = np.take_along_axis(opp, srt, axis=1)
    order = np.lexsort((vs[:, 3], vs[:, 2], vs[:, 1], vs[:, 0]))
    new_index = np.empty(len(t), np.int64)
    new_index[order] = np.arange(len(t))
    V = vs[order]
    O = os_[order]
    A = np.where(O >= 0, new_index[np.clip(O, 0, None)], -1)
    return V.astype(np.int32), A.astype(np.int32)
