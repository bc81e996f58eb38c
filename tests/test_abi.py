"""The C-ABI library loads and exports every entry point include/gstar4d.h
declares (no device calls). CPU only."""
import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(REPO, "include", "gstar4d.h")).read()
    return sorted(set(re.findall(r"G4D_API\s+[\w\s\*]+?\b(g4d_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = _declared()
    for must in ("g4d_create", "g4d_triangulate", "g4d_gdel_init", "g4d_gdel_compute", "g4d_get_tetra",
                 "g4d_gdel_deinit", "g4d_triangulate_batch", "g4d_destroy", "g4d_free"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from gstar4d_b200 import api
    if not os.path.exists(api.LIB_PATH):
        import __graft_entry__
        __graft_entry__.build()
    lib = ctypes.CDLL(api.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(api.EXPORTS) == set(_declared())


def test_create_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from gstar4d_b200 import api
    lib = api.load()
    h = ctypes.c_void_p()
    cfg = api.default_config()
    assert lib.g4d_create(ctypes.byref(h), ctypes.byref(cfg)) == 8  # G4D_ERR_NODEVICE
    assert lib.g4d_status_string(8) == b"no sm_100 device"


def test_tet_layout_matches_reference_tetrahedron():
    from gstar4d_b200 import api
    # Tetrahedron { int _v[4]; int _opp[4]; } (Common/Geometry.h:147-150)
    assert api.TET_DTYPE.itemsize == 32
    assert api.TET_DTYPE.fields["opp"][1] == 16
