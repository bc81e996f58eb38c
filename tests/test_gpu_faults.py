"""Failure paths, made to happen on the host or by waits that run out; nothing
here faults, traps or hangs the GPU. Needs a B200.

  - the splaying loop cap (g4d_config.max_splay_loops) returns G4D_ERR_TIMEOUT
    where the reference would loop until its stars agree (GDelHost.cu:1393-1446);
  - workspace allocations that fail (G4D_FAIL_ALLOC_AFTER injects the failure
    into the k-th allocation of a new context) return G4D_ERR_NOMEM, and a
    context created afterwards works;
  - the tensor-core kernels' bounded mbarrier wait, given a phase that nothing
    completes, runs out, frees its tensor memory and returns G4D_ERR_TIMEOUT;
    the same context then runs the MLP kernels normally.
"""
import numpy as np
import pytest

from gstar4d_b200 import workloads

pytestmark = pytest.mark.gpu


def test_splay_loop_cap_returns_timeout(oracle):
    import gstar4d_b200
    pts = workloads.mixed(20000, seed=31)
    with gstar4d_b200.Triangulator(grid_size=64, max_splay_loops=1) as t:
        with pytest.raises(gstar4d_b200.G4DError) as e:
            t.triangulate(pts)
        assert e.value.status == 3
        assert "did not converge in 1 loops" in str(e.value)
    # the default cap lets the same cloud finish, bit-exact
    with gstar4d_b200.Triangulator(grid_size=64) as t:
        tets, _, st = t.triangulate(pts)
    assert st["loops"] > 1
    ref, _, _ = oracle.triangulate(pts, 64)
    g = oracle.canonical(gstar4d_b200.tets_as_array(tets))
    r = oracle.canonical(ref)
    assert np.array_equal(g[0], r[0]) and np.array_equal(g[1], r[1])


@pytest.mark.parametrize("after", [0, 4, 12, 24, 40])
def test_injected_allocation_failure_returns_nomem(monkeypatch, after):
    import gstar4d_b200
    pts = workloads.uniform(5000, seed=32)
    monkeypatch.setenv("G4D_FAIL_ALLOC_AFTER", str(after))
    t = gstar4d_b200.Triangulator(grid_size=64)
    monkeypatch.delenv("G4D_FAIL_ALLOC_AFTER")
    try:
        with pytest.raises(gstar4d_b200.G4DError) as e:
            t.triangulate(pts)
        assert e.value.status == 2, str(e.value)
    finally:
        t.close()
    with gstar4d_b200.Triangulator(grid_size=64) as t:
        tets, _, _ = t.triangulate(pts)
    assert len(tets) > 0


def test_tensor_core_wait_runs_out_and_context_stays_usable():
    import gstar4d_b200
    from oracle import mlp_oracle
    rng = np.random.default_rng(4)
    params = (rng.standard_normal(gstar4d_b200.api.MLP_PARAMS) * 0.2).astype(np.float32)
    x = mlp_oracle.bf16_bits(rng.standard_normal((300, 16)).astype(np.float32))
    with gstar4d_b200.Triangulator() as t:
        before = t.mlp_infer(x, params)
        with pytest.raises(gstar4d_b200.G4DError) as e:
            t.mlp_wait_probe(4096)
        assert e.value.status == 3
        after = t.mlp_infer(x, params)
    assert np.array_equal(before, after)
