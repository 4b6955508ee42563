"""Learned start vector: the network's CUDA kernels against the CPU oracle (oracle/mlp.py,
itself pinned by finite differences), the sub-block compression, and what the trained
network gains over the standard start vector on held-out interaction variants.

Tolerances: GPU vs oracle forward outputs 1e-4 relative and gradients 2e-3 relative
(both compute in FP32 with BF16-rounded hidden activations; they differ in summation
order and in the exponential, and a BF16 rounding that lands the other way moves a value
by one BF16 ulp, 2^-8 relative, which the max over all entries can catch); the oracle's
float64 gradients vs central differences 1e-6 relative.
"""
import numpy as np
import pytest

from conftest import make_problem

SMALL = (8, 32, 16)   # n_in, width, n_out


def _rand_params(n_in, width, n_out, seed=0):
    from oracle.mlp import layout
    _, n = layout(n_in, width, n_out)
    return np.random.default_rng(seed).normal(0, 0.3, n).astype(np.float32)


def test_bf16_rounding_is_nearest_even():
    from oracle.mlp import bf16_round
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -7)                    # BF16 spacing at 1
    x = np.array([1.0, 1.0 + ulp / 2, 1.0 + 3 * ulp / 2, 1.0 + ulp / 4, -2.5, 3.0e-3], dtype=np.float32)
    r = bf16_round(x)
    assert r[0] == one and r[1] == one               # tie to even (1.0 has an even last bit)
    assert r[2] == one + 2 * ulp                     # tie to even (upwards)
    assert r[3] == one
    assert r[4] == np.float32(-2.5)
    assert abs(r[5] - 3.0e-3) <= 3.0e-3 * 2 ** -8


def test_oracle_gradients_match_finite_differences():
    from oracle.mlp import loss_and_grad
    n_in, width, n_out = 4, 6, 3
    p = _rand_params(n_in, width, n_out, 1).astype(np.float64)
    rng = np.random.default_rng(2)
    x, t = rng.normal(size=(5, n_in)), rng.normal(size=(5, n_out))
    _, g = loss_and_grad(p, x, t, n_in, width, n_out, bf16=False, dtype=np.float64)
    h = 1e-6
    fd = np.zeros_like(p)
    for i in range(len(p)):
        e = np.zeros_like(p)
        e[i] = h
        lp, _ = loss_and_grad(p + e, x, t, n_in, width, n_out, bf16=False, dtype=np.float64)
        lm, _ = loss_and_grad(p - e, x, t, n_in, width, n_out, bf16=False, dtype=np.float64)
        fd[i] = (lp - lm) / (2 * h)
    assert np.abs(g - fd).max() <= 1e-6 * max(np.abs(fd).max(), 1.0)


def test_subblocks_tile_the_parity_mask_and_compression_inverts():
    from nushellx_b200.learned.compress import SubBlocks, Compressor
    P = make_problem("fp_4p4n_0")
    sub = SubBlocks(P)
    assert np.array_equal(np.sort(sub.index), np.nonzero(P.lcoef)[0])
    g = np.random.default_rng(4).standard_normal(P.no_state) * P.lcoef
    g /= np.linalg.norm(g)
    comp = Compressor.from_reference(sub, g, 64)
    w = comp.compress(g)
    assert comp.K == 64 and np.all(w > 0)            # the reference compresses to its own norms
    assert np.allclose(np.sort(w)[::-1], np.sort(sub.norms(g))[::-1][:64])
    assert np.allclose(comp.compress(comp.decompress(w)), w)
    assert np.allclose(comp.compress(-g), w)          # sign convention


def test_compression_from_a_training_set():
    """Kept sub-blocks = largest mean weight over the training states; shapes = dominant
    singular vectors (independent of each state's overall sign); projections sign-aligned."""
    import torch
    from nushellx_b200.learned.compress import SubBlocks, Compressor
    P = make_problem("fp_4p4n_0")
    sub = SubBlocks(P)
    rng = np.random.default_rng(8)
    base = rng.standard_normal(P.no_state) * P.lcoef
    base /= np.linalg.norm(base)
    G = np.stack([(1 if i % 2 else -1) * (base * (1 + 0.05 * rng.standard_normal())
                                          + 1e-3 * rng.standard_normal(P.no_state) * P.lcoef) for i in range(24)])
    comp = Compressor.from_training(sub, torch.tensor(G, dtype=torch.float32), 64)
    assert comp.K == 64
    # the kept sub-blocks are the 64 heaviest by mean weight
    e = np.mean([sub.norms(g) ** 2 for g in G], axis=0)
    kept = {tuple(d) for d in comp.desc}
    heaviest = {tuple(sub.desc[i]) for i in np.argsort(-e)[:64]}
    assert kept == heaviest
    # unit shapes, one per kept sub-block
    assert np.allclose(np.sqrt(np.add.reduceat(comp.shapes ** 2, comp.start[:-1])), 1.0)
    W = np.stack([comp.compress(g) for g in G])
    lead = comp.rank[0]
    assert np.all(W[:, lead] > 0)                      # alternating overall signs are aligned
    assert np.corrcoef(W)[0, 1:].min() > 0.99           # the same state up to noise
    assert np.allclose(comp.compress(comp.decompress(W[3])), W[3])


@pytest.mark.gpu
def test_network_forward_and_gradients_match_the_oracle():
    from nushellx_b200.build import build
    from nushellx_b200.nsx import Network
    from oracle.mlp import forward, loss_and_grad
    build()
    n_in, width, n_out = SMALL
    net = Network(n_in, width, n_out, seed=3)
    p = _rand_params(n_in, width, n_out, 5)
    net.params = p
    assert np.array_equal(net.params, p)
    rng = np.random.default_rng(6)
    x = rng.uniform(-1, 1, (37, n_in)).astype(np.float32)
    t = rng.normal(size=(37, n_out)).astype(np.float32)
    y_ref, _ = forward(p, x, n_in, width, n_out)
    y = net.forward(x)
    assert np.abs(y - y_ref).max() <= 1e-4 * np.abs(y_ref).max()
    loss, g = net.gradients(x, t)
    loss_ref, g_ref = loss_and_grad(p, x, t, n_in, width, n_out)
    assert abs(loss - loss_ref) <= 1e-4 * loss_ref
    assert np.abs(g - g_ref).max() <= 2e-3 * np.abs(g_ref).max()
    # training lowers the loss
    l_end = net.train(x, t, 200, 1e-2)
    assert l_end < 0.5 * loss
    net.close()


@pytest.mark.gpu
def test_learned_start_saves_iterations_on_held_out_variants(tmp_path):
    """Sweep fp 4p+4n J=0+ over seeded variants, train on 48, compare on 12 held out:
    the learned start must need fewer Lanczos iterations on average than the standard
    start, and the eigenvalues must agree to the solve's accuracy regardless of the start."""
    from nushellx_b200.build import build
    from nushellx_b200.learned import pipeline as L
    build()
    data = str(tmp_path / "sweep.npz")
    model = str(tmp_path / "model.npz")
    L.sweep("fp_4p4n_0", 60, 11, 256, data, ntrain=48, log=lambda *a: None)
    stats = L.train(data, 48, model, width=256, steps=1500, lr=2e-3, log=lambda *a: None)
    assert stats["err_test"] < stats["err_mean_predictor"]   # the network beats predicting the mean
    learned = L.LearnedStart(model)
    P, fam, S = L.solver_and_family("fp_4p4n_0")
    lams = np.load(data)["lams"][48:60]
    rows = L.compare(S, fam, learned, lams, nev=10, tol=1e-6, log=lambda *a: None)
    it_std = np.mean([r["iter_standard"] for r in rows])
    it_l = np.mean([r["iter_learned"] for r in rows])
    print(f"mean iterations: standard {it_std:.1f}, learned {it_l:.1f}")
    assert it_l < it_std
    assert max(r["max_dE"] for r in rows) < 1e-5
    # fallback: a model for another vector space yields no start vector
    S2 = L.solver_and_family("sd_2p2n_0")[2]
    assert learned.start_vector(S2, lams[0]) is None
    S.close()
    S2.close()
    learned.close()
