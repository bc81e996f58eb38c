"""Python host mirror of the reference's entry points over the C ABI
(include/gstar4d.h, library gstar4d_b200/libgstar4d.so).

    gdel_init(config, points, scaled)   GDelaunay.cpp:47-60   (gdelInit)
    gdel_compute()                      GDelaunay.cpp:62-88   (gdelCompute)
    get_tetra_from_gpu()                GDelaunay.cpp:90-96   (getTetraFromGpu)
    gdel_deinit()                       GDelaunay.cpp:98-104  (gdelDeInit)

plus `Triangulator.triangulate` (points in, tetrahedra with adjacency out) and
the batched entry point. Failures raise G4DError carrying the C status code;
the CUDA library is required (there is no CPU fallback).
"""
import ctypes
import weakref
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgstar4d.so")

G4D_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "out of memory", 3: "iteration cap reached",
          4: "internal consistency error", 5: "CUDA error", 6: "star capacity exceeded",
          7: "coordinate exponent range too wide", 8: "no sm_100 device"}


class G4DError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (status %d): %s" % (STATUS.get(status, "?"), status, message))
        self.status = status


class Config(ctypes.Structure):
    """Mirrors Common/Config.h:59-79 plus the B200 options."""
    _fields_ = [("seed", ctypes.c_int), ("run_num", ctypes.c_int), ("grid_size", ctypes.c_int),
                ("point_num", ctypes.c_int), ("dist", ctypes.c_int), ("facet_max", ctypes.c_int),
                ("log_verbose", ctypes.c_int), ("log_stats", ctypes.c_int), ("log_timing", ctypes.c_int),
                ("do_check", ctypes.c_int), ("pred_thread_num", ctypes.c_int), ("pred_block_num", ctypes.c_int),
                ("do_sorting", ctypes.c_int), ("device", ctypes.c_int), ("index_space", ctypes.c_int),
                ("proposal", ctypes.c_int), ("max_splay_loops", ctypes.c_int)]


class CheckReport(ctypes.Structure):
    _fields_ = [(f, ctypes.c_longlong) for f in ("vertices", "edges", "triangles", "tets", "euler", "orient_fail",
                                                 "insphere_fail", "adjacency_fail")]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Stats(ctypes.Structure):
    _fields_ = [("t_init_ms", ctypes.c_double), ("t_pba_ms", ctypes.c_double), ("t_star_ms", ctypes.c_double),
                ("t_splay_ms", ctypes.c_double), ("t_out_ms", ctypes.c_double), ("t_total_ms", ctypes.c_double),
                ("star_insertions", ctypes.c_longlong), ("splay_insertions", ctypes.c_longlong),
                ("drowned", ctypes.c_longlong), ("proofs", ctypes.c_longlong),
                ("exact_predicates", ctypes.c_longlong), ("loops", ctypes.c_int), ("missing", ctypes.c_int),
                ("grid_size", ctypes.c_int), ("tets", ctypes.c_int), ("gpu_launches", ctypes.c_longlong),
                ("large_stars", ctypes.c_int), ("proposed", ctypes.c_int), ("pba_form", ctypes.c_int),
                ("block_pairs", ctypes.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


TET_DTYPE = np.dtype([("v", np.int32, 4), ("opp", np.int32, 4)])

_lib = None

EXPORTS = ["g4d_default_config", "g4d_create", "g4d_destroy", "g4d_last_error", "g4d_status_string",
           "g4d_triangulate", "g4d_triangulate_to", "g4d_triangulate_to_f32", "g4d_triangulate_device",
           "g4d_gdel_init",
           "g4d_gdel_compute", "g4d_get_tetra", "g4d_gdel_deinit", "g4d_get_stats", "g4d_triangulate_batch",
           "g4d_triangulate_batch_to", "g4d_triangulate_batch_device", "g4d_stream",
           "g4d_eval_predicates", "g4d_voronoi", "g4d_voronoi_noalloc", "g4d_proposal_train",
           "g4d_proposal_weights", "g4d_mlp_grad", "g4d_mlp_infer", "g4d_mlp_wait_probe", "g4d_make_points", "g4d_check_mesh", "g4d_check_tets", "g4d_free"]

MLP_PARAMS = 9473


def load():
    """Loads the CUDA library; raises if it was not built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("gstar4d CUDA library missing: build it with __graft_entry__.build() "
                           "(python -c 'import __graft_entry__ as g; g.build()')")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    L.g4d_default_config.argtypes = [ctypes.POINTER(Config)]
    L.g4d_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(Config)]
    L.g4d_destroy.argtypes = [vp]
    L.g4d_last_error.argtypes = [vp]
    L.g4d_last_error.restype = ctypes.c_char_p
    L.g4d_status_string.restype = ctypes.c_char_p
    L.g4d_triangulate_to.argtypes = [vp, vp, ip, vp, ip, ctypes.POINTER(ip), vp, ctypes.POINTER(Stats)]
    L.g4d_triangulate_to_f32.argtypes = [vp, vp, ip, vp, ip, ctypes.POINTER(ip), vp, ctypes.POINTER(Stats)]
    L.g4d_triangulate.argtypes = [vp, vp, ip, ctypes.POINTER(vp), ctypes.POINTER(ip), vp, ctypes.POINTER(Stats)]
    L.g4d_triangulate_device.argtypes = [vp, vp, ip, ctypes.POINTER(vp), ctypes.POINTER(ip), ctypes.POINTER(Stats)]
    L.g4d_gdel_init.argtypes = [vp, vp, vp, ip]
    L.g4d_gdel_compute.argtypes = [vp, dp, dp, dp, dp]
    L.g4d_get_tetra.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(ip)]
    L.g4d_gdel_deinit.argtypes = [vp]
    L.g4d_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.g4d_triangulate_batch.argtypes = [vp, vp, vp, ip, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                        ctypes.POINTER(Stats)]
    L.g4d_triangulate_batch_to.argtypes = [vp, vp, vp, ip, vp, ctypes.c_int64, vp, ctypes.POINTER(ctypes.c_int64),
                                           ctypes.POINTER(Stats)]
    L.g4d_triangulate_batch_device.argtypes = [vp, vp, vp, ip, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                               ctypes.POINTER(Stats)]
    L.g4d_eval_predicates.argtypes = [vp, ip, vp, vp, ip, vp]
    L.g4d_voronoi.argtypes = [vp, vp, ip, ip, vp]
    L.g4d_voronoi_noalloc.argtypes = [vp, ip, ip, vp, vp]
    fp = ctypes.POINTER(ctypes.c_float)
    L.g4d_proposal_train.argtypes = [vp, vp, ip, ip, ctypes.c_float, fp]
    L.g4d_proposal_weights.argtypes = [vp, vp, ip, ip]
    L.g4d_mlp_grad.argtypes = [vp, vp, vp, ip, vp, vp, fp]
    L.g4d_mlp_infer.argtypes = [vp, vp, ip, vp, vp]
    L.g4d_mlp_wait_probe.argtypes = [vp, ip]
    L.g4d_make_points.argtypes = [ip, ip, ip, ip, vp]
    L.g4d_check_mesh.argtypes = [vp, ctypes.POINTER(CheckReport)]
    L.g4d_check_tets.argtypes = [vp, vp, ip, vp, ip, ctypes.POINTER(CheckReport)]
    L.g4d_stream.argtypes = [vp]
    L.g4d_stream.restype = vp
    L.g4d_free.argtypes = [vp]
    _lib = L
    return L


def default_config(**kw):
    cfg = Config()
    load().g4d_default_config(ctypes.byref(cfg))
    for k, v in kw.items():
        setattr(cfg, k, int(v))
    return cfg


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class Triangulator:
    """One library context (device, stream, workspace). Not thread-safe: use one
    per host thread, as the C ABI requires."""

    def __init__(self, config=None, **kw):
        self._lib = load()
        self.config = config if config is not None else default_config(**kw)
        h = ctypes.c_void_p()
        st = self._lib.g4d_create(ctypes.byref(h), ctypes.byref(self.config))
        if st != G4D_OK:
            raise G4DError(st, "g4d_create failed")
        self._h = h
        self.last_stats = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.g4d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != G4D_OK:
            raise G4DError(st, self._lib.g4d_last_error(self._h).decode(errors="replace"))

    @property
    def stream(self):
        return self._lib.g4d_stream(self._h)

    def triangulate(self, points, out=None, want_order=False):
        """points: (n,3) float64 in input order. Returns (tets, order, stats):
        tets structured array (v[4], opp[4]) — or `out` filled in place —, the
        Morton order (sorted position -> input index) when want_order. float32
        points go through g4d_triangulate_to_f32 (widened on the device)."""
        n = len(points)
        nt = ctypes.c_int(0)
        order = np.empty(n, np.int32) if want_order else None
        stats = Stats()
        if getattr(points, "dtype", None) == np.float32:
            pts32 = np.ascontiguousarray(points, dtype=np.float32)
            own = out is None
            if own:  # about 6.8 tetrahedra per point; retried at the exact size if exceeded
                out = np.empty(int(7.5 * n) + 64, TET_DTYPE)
            st = self._lib.g4d_triangulate_to_f32(self._h, _ptr(pts32), n, _ptr(out), len(out), ctypes.byref(nt),
                                                  _ptr(order) if want_order else None, ctypes.byref(stats))
            if own and st == 1 and nt.value > len(out):
                out = np.empty(nt.value, TET_DTYPE)
                st = self._lib.g4d_triangulate_to_f32(self._h, _ptr(pts32), n, _ptr(out), len(out),
                                                      ctypes.byref(nt), _ptr(order) if want_order else None,
                                                      ctypes.byref(stats))
            self._check(st)
            self.last_stats = stats.as_dict()
            return out[:nt.value], order, self.last_stats
        pts = np.ascontiguousarray(points, dtype=np.float64)
        if out is None:
            tp = ctypes.c_void_p()
            st = self._lib.g4d_triangulate(self._h, _ptr(pts), n, ctypes.byref(tp), ctypes.byref(nt),
                                           _ptr(order) if want_order else None, ctypes.byref(stats))
            self._check(st)
            nbytes = max(nt.value * TET_DTYPE.itemsize, 1)
            out = np.frombuffer((ctypes.c_char * nbytes).from_address(tp.value), TET_DTYPE)[:nt.value].copy()
            self._lib.g4d_free(tp)
        else:
            st = self._lib.g4d_triangulate_to(self._h, _ptr(pts), n, _ptr(out), len(out), ctypes.byref(nt),
                                              _ptr(order) if want_order else None, ctypes.byref(stats))
            self._check(st)
            out = out[:nt.value]
        self.last_stats = stats.as_dict()
        return out, order, self.last_stats

    def triangulate_device(self, d_points_ptr, n):
        """Points already in HBM (device pointer to n*3 float64). Returns
        (device pointer to tets, ntet, stats)."""
        d = ctypes.c_void_p()
        nt = ctypes.c_int(0)
        stats = Stats()
        st = self._lib.g4d_triangulate_device(self._h, ctypes.c_void_p(d_points_ptr), int(n), ctypes.byref(d),
                                              ctypes.byref(nt), ctypes.byref(stats))
        self._check(st)
        self.last_stats = stats.as_dict()
        return d.value, nt.value, self.last_stats

    def eval_predicates(self, kind, points, idx=None):
        """Device predicate signs: kind 0 orient3d (sets of 4 points), 1 orient4
        with SoS (sets of 5 points + 5 indices), 2 orient4 without SoS."""
        pts = np.ascontiguousarray(points, dtype=np.float64)
        count = len(pts)
        out = np.zeros(count, np.int8)
        ia = np.ascontiguousarray(idx, dtype=np.int32) if idx is not None else None
        st = self._lib.g4d_eval_predicates(self._h, int(kind), _ptr(pts), _ptr(ia) if ia is not None else None,
                                           count, _ptr(out))
        self._check(st)
        return out

    def voronoi(self, points, grid):
        """Digital Voronoi grid (grid^3 packed site voxels, x fastest)."""
        pts = np.ascontiguousarray(points, dtype=np.float64)
        out = np.empty(grid ** 3, np.uint32)
        self._check(self._lib.g4d_voronoi(self._h, _ptr(pts), len(pts), int(grid), _ptr(out)))
        return out

    # ---- learned star proposal ---------------------------------------------------------
    def train_proposal(self, points, epochs=4, lr=2e-3):
        """Train the proposal model on one cloud (labels from the plain method);
        returns the last epoch's mean loss."""
        pts = np.ascontiguousarray(points, dtype=np.float64)
        loss = ctypes.c_float(0)
        self._check(self._lib.g4d_proposal_train(self._h, _ptr(pts), len(pts), int(epochs), float(lr),
                                                 ctypes.byref(loss)))
        return loss.value

    def proposal_weights(self, weights=None):
        """Current parameters (float32[9473]); with `weights`, replace them."""
        if weights is not None:
            w = np.ascontiguousarray(weights, dtype=np.float32)
            self._check(self._lib.g4d_proposal_weights(self._h, _ptr(w), len(w), 1))
            return w
        w = np.empty(MLP_PARAMS, np.float32)
        self._check(self._lib.g4d_proposal_weights(self._h, _ptr(w), MLP_PARAMS, 0))
        return w

    def mlp_grad(self, x_bf16, y, params):
        x = np.ascontiguousarray(x_bf16, dtype=np.uint16).reshape(-1, 16)
        yy = np.ascontiguousarray(y, dtype=np.float32)
        p = np.ascontiguousarray(params, dtype=np.float32)
        g = np.empty(MLP_PARAMS, np.float32)
        loss = ctypes.c_float(0)
        self._check(self._lib.g4d_mlp_grad(self._h, _ptr(x), _ptr(yy), len(x), _ptr(p), _ptr(g), ctypes.byref(loss)))
        return g, loss.value

    def mlp_infer(self, x_bf16, params):
        x = np.ascontiguousarray(x_bf16, dtype=np.uint16).reshape(-1, 16)
        p = np.ascontiguousarray(params, dtype=np.float32)
        out = np.empty(len(x), np.float32)
        self._check(self._lib.g4d_mlp_infer(self._h, _ptr(x), len(x), _ptr(p), _ptr(out)))
        return out

    def check_mesh(self):
        """The device validator (g4d_check_mesh) on the last single-cloud
        triangulation: dict of V, E, F, T, euler and the failure counts."""
        r = CheckReport()
        self._check(self._lib.g4d_check_mesh(self._h, ctypes.byref(r)))
        return r.as_dict()

    def check_tets(self, points, tets):
        """The device validator on a given mesh (g4d_check_tets): points (n,3)
        float64 and tets (structured TET_DTYPE, or (T, 8) int32)."""
        pts = np.ascontiguousarray(points, dtype=np.float64)
        t = np.asarray(tets)
        if t.dtype != TET_DTYPE:
            t = np.ascontiguousarray(t, dtype=np.int32).view(TET_DTYPE).reshape(-1)
        t = np.ascontiguousarray(t)
        r = CheckReport()
        self._check(self._lib.g4d_check_tets(self._h, _ptr(pts), len(pts), _ptr(t), len(t), ctypes.byref(r)))
        return r.as_dict()

    def mlp_wait_probe(self, limit):
        """Runs the tensor-core kernels' bounded wait on a phase nothing
        completes (g4d_mlp_wait_probe); raises G4DError (status 3) when it ran
        out, as it must."""
        self._check(self._lib.g4d_mlp_wait_probe(self._h, int(limit)))

    # ---- reference-shaped entry points ------------------------------------------------
    def gdel_init(self, points, scaled=None):
        """Like gdelInit: both arrays (n,3 float64, C-contiguous) are overwritten
        with the Morton-sorted order."""
        for a in (points, scaled):
            if a is not None and (a.dtype != np.float64 or not a.flags.c_contiguous):
                raise ValueError("points must be C-contiguous float64 arrays")
        st = self._lib.g4d_gdel_init(self._h, _ptr(points), _ptr(scaled) if scaled is not None else None,
                                     len(points))
        self._check(st)

    def gdel_compute(self):
        t = [ctypes.c_double() for _ in range(4)]
        st = self._lib.g4d_gdel_compute(self._h, *[ctypes.byref(x) for x in t])
        self._check(st)
        return tuple(x.value for x in t)

    def get_tetra_from_gpu(self):
        p = ctypes.c_void_p()
        nt = ctypes.c_int(0)
        self._check(self._lib.g4d_get_tetra(self._h, ctypes.byref(p), ctypes.byref(nt)))
        if nt.value == 0:
            return np.empty(0, TET_DTYPE)
        buf = (ctypes.c_char * (nt.value * TET_DTYPE.itemsize)).from_address(p.value)
        return np.frombuffer(buf, TET_DTYPE).copy()

    def stats(self):
        """Statistics of the last triangulation on this context."""
        st = Stats()
        self._check(self._lib.g4d_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def gdel_deinit(self):
        self._check(self._lib.g4d_gdel_deinit(self._h))

    def triangulate_batch(self, points, cloud_offsets, out=None):
        """Tetrahedra of many clouds: (tets, tet_offsets, stats), cloud c's
        tetrahedra are tets[tet_offsets[c]:tet_offsets[c+1]] with cloud-local
        input indices. With `out` (a TET_DTYPE array, best in pinned memory) the
        results are copied into it while later passes compute and tets is a
        view of it."""
        pts = np.ascontiguousarray(points, dtype=np.float64)
        offs = np.ascontiguousarray(cloud_offsets, dtype=np.int64)
        stats = Stats()
        nclouds = len(offs) - 1
        if out is not None:
            if out.dtype != TET_DTYPE or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous TET_DTYPE array")
            toffs = np.zeros(nclouds + 1, np.int64)
            nt = ctypes.c_int64()
            st = self._lib.g4d_triangulate_batch_to(self._h, _ptr(pts), _ptr(offs), nclouds, _ptr(out), len(out),
                                                    _ptr(toffs), ctypes.byref(nt), ctypes.byref(stats))
            self._check(st)
            self.last_stats = stats.as_dict()
            return out[: nt.value], toffs, self.last_stats
        tp, op = ctypes.c_void_p(), ctypes.c_void_p()
        st = self._lib.g4d_triangulate_batch(self._h, _ptr(pts), _ptr(offs), nclouds, ctypes.byref(tp),
                                             ctypes.byref(op), ctypes.byref(stats))
        self._check(st)
        toffs = np.frombuffer((ctypes.c_int64 * (nclouds + 1)).from_address(op.value), np.int64).copy()
        self._lib.g4d_free(op)
        total = int(toffs[-1])
        # the library's buffer becomes the array's memory (freed with the array)
        tets = _adopt(self._lib, tp.value, total * TET_DTYPE.itemsize, TET_DTYPE, total)
        self.last_stats = stats.as_dict()
        return tets, toffs, self.last_stats

    def triangulate_batch_device(self, d_points, cloud_offsets):
        """Batch on device-resident points (d_points: device address of n*3
        doubles). Returns (device address of the tetrahedra, their count, tet
        offsets per cloud, stats); the device buffer belongs to the context."""
        offs = np.ascontiguousarray(cloud_offsets, dtype=np.int64)
        tp, op = ctypes.c_void_p(), ctypes.c_void_p()
        stats = Stats()
        nclouds = len(offs) - 1
        st = self._lib.g4d_triangulate_batch_device(self._h, ctypes.c_void_p(int(d_points)), _ptr(offs), nclouds,
                                                    ctypes.byref(tp), ctypes.byref(op), ctypes.byref(stats))
        self._check(st)
        toffs = np.frombuffer((ctypes.c_int64 * (nclouds + 1)).from_address(op.value), np.int64).copy()
        self.last_stats = stats.as_dict()
        return tp.value, int(toffs[-1]), toffs, self.last_stats


def _adopt(lib, ptr, nbytes, dtype, count):
    """numpy view of a library-allocated buffer that frees it (g4d_free) when
    the last view is gone."""
    buf = (ctypes.c_char * max(nbytes, 1)).from_address(ptr)
    weakref.finalize(buf, lib.g4d_free, ctypes.c_void_p(ptr))
    return np.frombuffer(buf, dtype)[:count]


def make_points(n, grid, dist, seed):
    """The reference command line's points for -n -g -d -s (g4d_make_points):
    (n, 3) float64 holding float values in grid units [1, grid-2]."""
    out = np.empty((int(n), 3), np.float64)
    st = load().g4d_make_points(int(n), int(dist), int(grid), int(seed), _ptr(out))
    if st != G4D_OK:
        raise G4DError(st, "g4d_make_points(n=%d, dist=%d, grid=%d)" % (n, dist, grid))
    return out


def tets_as_array(tets):
    """Structured tets -> (T, 8) int32 [v0..v3, opp0..opp3]."""
    return np.concatenate([tets["v"], tets["opp"]], axis=1).astype(np.int32)


def triangulate(points, grid_size=0, **kw):
    with Triangulator(grid_size=grid_size, **kw) as t:
        tets, _, stats = t.triangulate(points)
    return tets, stats
