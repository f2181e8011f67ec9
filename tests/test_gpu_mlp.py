"""The learned surrogate on the GPU against the FP64 oracle (oracle/mlp.py).

The oracle rounds every GEMM operand to bf16 where the GPU does, so training
gradients, energies and input gradients agree to fp32-accumulation level.
The engine tests show the gate (gate 0 = exact GAP everywhere) and what the
trained ensemble gains over the method without it, on a cell held out of the
training data: a low error and a small gated fraction, where an untrained
ensemble sends every site back to GAP."""
from __future__ import annotations

import numpy as np
import pytest

from _util import O
from oracle import mlp as M
from turbogap_b200 import synth
from turbogap_b200.hypers import carbon_hypers

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-30))


def _batch(seed, B, D, Dp):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(B, D)).astype(np.float32)
    y = rng.normal(size=B).astype(np.float32)
    g = (0.3 * rng.normal(size=(B, D))).astype(np.float32)
    X = np.zeros((B, Dp))
    X[:, :D] = x
    G = np.zeros((B, Dp))
    G[:, :D] = g
    return x, y, g, X, G


@pytest.mark.parametrize("D", [100, 324])
def test_batch_gradients_match_oracle(gpu, D):
    H, B, lam = 256, 256, 0.8
    m = gpu.Mlp(D, H, 2, seed=1)
    L = m.layout()
    Dp = L["Dp"]
    p = M.Params.random(D, Dp, H, seed=5)
    m.set_member(1, p.W1[:, :D], p.b1, p.W2, p.b2, p.w3, p.b3)
    x, y, g, X, G = _batch(7, B, D, Dp)
    loss, grads, E, Gg = m.batch_grads(1, x, y, g, lam)
    lo, go, Eo, Go = M.loss_and_grads(p, X, y.astype(np.float64), G, lam, D, bf16=True)
    assert abs(loss - lo) <= 2e-4 * abs(lo)
    assert rel(E, Eo) < 1e-4
    assert rel(Gg[:, :D], Go[:, :D]) < 1e-3
    W1g = grads[L["W1"]:L["W1"] + H * Dp].reshape(H, Dp)
    assert rel(W1g[:, :D], go["W1"][:, :D]) < 3e-3
    assert np.all(W1g[:, D:] == 0.0)
    assert rel(grads[L["b1"]:L["b1"] + H], go["b1"]) < 3e-3
    assert rel(grads[L["W2"]:L["W2"] + H * H].reshape(H, H), go["W2"]) < 3e-3
    assert rel(grads[L["b2"]:L["b2"] + H], go["b2"]) < 3e-3
    assert rel(grads[L["w3"]:L["w3"] + H], go["w3"]) < 3e-3
    assert abs(grads[L["b3"]] - go["b3"]) <= 1e-4 * max(1.0, abs(go["b3"]))
    m.close()


def test_adam_step_matches_oracle(gpu):
    D, H, B, lam, lr = 100, 128, 128, 0.5, 1e-3
    m = gpu.Mlp(D, H, 1, seed=2)
    Dp = m.layout()["Dp"]
    p = M.Params.random(D, Dp, H, seed=9)
    m.set_member(0, p.W1[:, :D], p.b1, p.W2, p.b2, p.w3, p.b3)
    m.set_normalisation(1.0, 0.0, 1.0)
    x, y, g, X, G = _batch(11, B, D, Dp)
    m.add_samples(x, y.astype(np.float64), g)
    m.train(1, batch=B, lr=lr, force_weight=lam, seed=0)
    _, go, _, _ = M.loss_and_grads(p, X, y.astype(np.float64), G, lam, D, bf16=True)
    M.adam_step(p, go, {}, lr)
    W1, b1, W2, b2, w3, b3 = m.get_member(0)
    # first Adam step moves each weight by ~lr sign(g): compare where g is not tiny
    for got, want, grad in ((W1, p.W1[:, :D], go["W1"][:, :D]), (W2, p.W2, go["W2"]),
                            (b1, p.b1, go["b1"]), (w3, p.w3, go["w3"])):
        big = np.abs(grad) > 1e-2 * np.abs(grad).max()
        assert big.mean() > 0.3
        assert np.max(np.abs(got - want)[big]) < 1e-5
    m.close()


# layer 2 as: one block-diagonal launch per tile column (H = 256), one dense
# block-diagonal GEMM (4 x 64 and 2 x 128: every member in one column tile), and
# one launch per member (4 x 128)
@pytest.mark.parametrize("D,H,nm", [(324, 256, 4), (324, 64, 4), (1224, 128, 2), (324, 128, 4)])
def test_predict_matches_oracle_ensemble(gpu, D, H, nm):
    m = gpu.Mlp(D, H, nm, seed=3)
    Dp = m.layout()["Dp"]
    members = [M.Params.random(D, Dp, H, seed=20 + k) for k in range(nm)]
    for k, p in enumerate(members):
        m.set_member(k, p.W1[:, :D], p.b1, p.W2, p.b2, p.w3, p.b3)
    sx, mu_e, se = 0.25, 0.1, 2.0          # powers of two: exact rescaling in bf16
    m.set_normalisation(sx, mu_e, se)
    rng = np.random.default_rng(4)
    delta = (sx * rng.normal(size=(300, D))).astype(np.float32)
    em, es, gm = m.predict(delta)
    X = np.zeros((300, Dp))
    X[:, :D] = delta / sx
    Es, Gs = [], []
    for p in members:
        E, G = M.forward(p, X, bf16=True, s1_bf16=True)
        Es.append(se * E + mu_e)
        Gs.append(se / sx * G[:, :D])
    Es, Gs = np.array(Es), np.array(Gs)
    # The oracle rounds to bf16 where the GPU does, so most rows agree to fp32
    # accumulation order (1e-8 to 1e-6). An activation that lands on a bf16
    # rounding boundary can round the other way and move its row by one bf16 step
    # of one hidden unit (up to about 6e-4 here); such rows are rare.
    de, ds = np.abs(em - Es.mean(0)), np.abs(es - Es.std(0))
    assert np.mean(de < 1e-4 * se) > 0.95 and np.mean(ds < 1e-4 * se) > 0.95
    assert de.max() < 2e-3 * se and ds.max() < 2e-3 * se
    assert rel(gm, Gs.mean(0)) < 2e-3
    m.close()


def test_training_reduces_loss(gpu):
    D, H = 64, 128
    rng = np.random.default_rng(0)
    A = rng.normal(size=(D, D)) / D
    c = rng.normal(size=D) / np.sqrt(D)
    x = rng.normal(size=(4096, D))
    E = 0.5 * np.einsum("nd,de,ne->n", x, A + A.T, x) / 2 + x @ c
    G = x @ ((A + A.T) / 2) + c
    m = gpu.Mlp(D, H, 2, seed=4)
    m.add_samples(x.astype(np.float32), E, G.astype(np.float32))
    loss = m.train(40, batch=256, lr=2e-3, force_weight=1.0, seed=1)
    assert np.all(np.isfinite(loss))
    assert loss[-1] < 0.05 * loss[0]
    em, _, gm = m.predict(x[:512].astype(np.float32))
    assert np.sqrt(np.mean((em - E[:512]) ** 2)) < 0.1 * E.std()
    assert rel(gm, G[:512]) < 0.3
    m.close()


def _carbon_engine(gpu, n_sparse=300, seed=31):
    from _util import sparse_block

    h = carbon_hypers()
    blk = sparse_block(h, n_sparse, seed=seed)
    gpu.soap_backend_begin(blk, key=777)
    st = synth.random_structure(216, 12.91, 1.2, seed=seed + 1)
    masses = np.full(216, 12.011 * 103.6426965268)
    eng = gpu.Engine(st.positions, st.species, masses, st.box, [777])
    eng.set_state(st.positions, synth.maxwell_velocities(masses, 600.0, seed))
    return eng, h, st


def test_engine_mixed_form(gpu):
    train_eng, h, st = _carbon_engine(gpu)
    D = h.dim
    # training data: exact steps of a 600 K run of one cell
    m = gpu.Mlp(D, 256, 4, seed=5)
    for _ in range(40):
        train_eng.md(1, 1.0)
        m.add_engine_samples(train_eng, 0)
    assert m.n_samples() == 40 * 216
    train_eng.close()
    # evaluated on a held-out cell (another seed, 10 steps into its own 600 K run)
    held = synth.random_structure(216, 12.91, 1.2, seed=977)
    masses = np.full(216, 12.011 * 103.6426965268)
    eng = gpu.Engine(held.positions, held.species, masses, held.box, [777])
    eng.set_state(held.positions, synth.maxwell_velocities(masses, 600.0, 978))
    eng.md(10, 1.0)
    e_ref, f_ref, v_ref = eng.compute()

    # gate 0: every site goes back to the exact kernel -> the exact result
    untrained = gpu.Mlp(D, 256, 4, seed=6)
    untrained.set_normalisation(*m_norm_from(m, untrained))
    gpu.engine_set_mlp(eng, 0, untrained, gate_ev=0.0)
    e0, f0, v0 = eng.compute()
    assert gpu.engine_mlp_stats(eng, 0) == (216, 216)
    assert np.max(np.abs(e0 - e_ref)) < 1e-9 and np.max(np.abs(f0 - f_ref)) < 1e-9

    # the method without training: an untrained ensemble, fully trusted
    gpu.engine_set_mlp(eng, 0, untrained, gate_ev=1e9)
    eu, fu, _ = eng.compute()
    sigma_e = untrained.normalisation()[2]
    gate_rel = 0.1 * sigma_e                             # gate on the data's energy scale
    gpu.engine_set_mlp(eng, 0, untrained, gate_ev=gate_rel)
    eng.compute()
    gated_untrained, _ = gpu.engine_mlp_stats(eng, 0)

    # trained ensemble
    loss = m.train(60, batch=256, lr=1e-3, force_weight=1.0, seed=2)
    assert loss[-1] < 0.1 * loss[0]
    gpu.engine_set_mlp(eng, 0, m, gate_ev=1e9)          # MLP everywhere
    em, fm, _ = eng.compute()
    gpu.engine_set_mlp(eng, 0, m, gate_ev=gate_rel)
    eng.compute()
    gated_trained, _ = gpu.engine_mlp_stats(eng, 0)
    gpu.engine_set_mlp(eng, 0, m, gate_ev=0.005)        # the production 5 meV gate
    eg, fg, _ = eng.compute()
    gpu.engine_set_mlp(eng, 0, None)

    rms = lambda a: float(np.sqrt(np.mean(np.square(a))))  # noqa: E731
    r_e_mlp, r_f_mlp = rms(em - e_ref), rms(fm - f_ref)
    r_e_gated, r_f_gated = rms(eg - e_ref), rms(fg - f_ref)
    r_e_untr, r_f_untr = rms(eu - e_ref), rms(fu - f_ref)
    print(f"sigma_E {sigma_e * 1e3:.2f} meV; trained: E {r_e_mlp * 1e3:.3f} meV/atom, "
          f"F {r_f_mlp * 1e3:.2f} meV/A; untrained: E {r_e_untr * 1e3:.3f}, F {r_f_untr * 1e3:.2f};"
          f" gated at {gate_rel * 1e3:.2f} meV: trained {gated_trained}/216, untrained "
          f"{gated_untrained}/216; 5 meV gate: E {r_e_gated * 1e3:.3f}, F {r_f_gated * 1e3:.2f}")
    # what training gains: 10x lower errors, and the gate keeps far more sites on the MLP
    assert r_e_mlp < 0.1 * r_e_untr and r_f_mlp < 0.1 * r_f_untr
    assert gated_untrained > 0.5 * 216 and gated_trained < 0.2 * 216
    # the accuracy targets of the mixed form: <= 1 meV/atom and <= 30 meV/A RMSE
    assert r_e_gated <= 1e-3 and r_f_gated <= 30e-3
    eng.close()
    m.close()
    untrained.close()


def m_norm_from(src, dst):
    """Normalisation of the trained network's data for an untrained ensemble."""
    src.train(0)   # sets the scales from the data set without updating weights
    return src.normalisation()
