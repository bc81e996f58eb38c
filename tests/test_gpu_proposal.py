"""Learned star proposal: the tensor-core MLP kernels against the FP64
restatement (oracle/mlp_oracle.py), and the proposal end to end. Needs a B200.

Tolerances: the kernels accumulate in FP32 and round to BF16 at the same points
as the restatement, so a value computed in FP32 can land on the other side of
a BF16 rounding boundary than its FP64 twin; logits agree to 2e-2 of their
scale, and every gradient block to 3e-2 relative error (Euclidean norm).
"""
import numpy as np
import pytest

from gstar4d_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mo():
    from oracle import mlp_oracle
    return mlp_oracle


@pytest.fixture(scope="module")
def tri():
    import gstar4d_b200
    t = gstar4d_b200.Triangulator()
    yield t
    t.close()


def test_mlp_inference_matches_restatement(tri, mo):
    bits, x = mo.sample_rows(1000, seed=11)  # 1000 rows: 7 full tiles and a partial one
    p = mo.init_params(seed=12)
    got = tri.mlp_infer(bits, p.astype(np.float32))
    exp = mo.logits(x, p.astype(np.float32).astype(np.float64))
    scale = np.abs(exp).max() + 1e-6
    assert np.abs(got - exp).max() <= 2e-2 * scale


def test_mlp_gradients_match_restatement(tri, mo):
    bits, x = mo.sample_rows(1000, seed=13)
    y = (np.random.default_rng(14).random(1000) < 0.4).astype(np.float32)
    p = mo.init_params(seed=15).astype(np.float32)
    g, loss = tri.mlp_grad(bits, y, p)
    eloss, eg, _ = mo.forward_backward(x, y, p.astype(np.float64), rounding=True)
    assert abs(loss - eloss) <= 1e-3 * max(1.0, abs(eloss))
    blocks = {"W1": (mo.P_W1, mo.P_B1), "b1": (mo.P_B1, mo.P_W2), "W2": (mo.P_W2, mo.P_B2),
              "b2": (mo.P_B2, mo.P_W3), "W3": (mo.P_W3, mo.P_B3), "b3": (mo.P_B3, mo.P_W4),
              "w4": (mo.P_W4, mo.P_B4), "b4": (mo.P_B4, mo.NPARAMS)}
    for name, (lo, hi) in blocks.items():
        err = np.linalg.norm(g[lo:hi] - eg[lo:hi]) / (np.linalg.norm(eg[lo:hi]) + 1e-12)
        assert err <= 3e-2, (name, err)


def test_learned_proposal_keeps_output_and_cuts_splaying(oracle):
    """Train on one mixed cloud, triangulate another with and without the
    proposal: identical tetrahedra and adjacency, fewer splaying insertions."""
    import gstar4d_b200
    train = workloads.mixed(200000, seed=21)
    test = workloads.mixed(200000, seed=22)
    with gstar4d_b200.Triangulator(grid_size=256) as t:
        loss0 = t.train_proposal(train, epochs=1, lr=2e-3)
        loss = t.train_proposal(train, epochs=4, lr=2e-3)
        assert np.isfinite(loss) and loss < loss0
        w = t.proposal_weights()
        plain, _, sp = t.triangulate(test)
    with gstar4d_b200.Triangulator(grid_size=256, proposal=1) as t:
        t.proposal_weights(w)
        learned, _, sl = t.triangulate(test)
    assert sl["proposed"] > 0
    g, r = oracle.canonical(gstar4d_b200.tets_as_array(learned)), oracle.canonical(gstar4d_b200.tets_as_array(plain))
    assert np.array_equal(g[0], r[0]) and np.array_equal(g[1], r[1])
    assert sl["splay_insertions"] < sp["splay_insertions"], (sl["splay_insertions"], sp["splay_insertions"])
