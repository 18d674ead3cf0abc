"""The learned audit surrogate on the GPU: tensor-core forward and backward
against the CPU oracle, training, features, and the pruned executor (whose
every commit is still judged by the exact audit)."""
import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn
from oracle import surrogate_oracle as so

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _batch(seed, n):
    rng = np.random.default_rng(seed)
    feats = rng.normal(0, 1.5, (n, so.FEATURES)).astype(np.float32)
    labels = np.stack([rng.integers(0, 2, n), rng.uniform(0, 3, n)], 1).astype(np.float32)
    mean = rng.normal(0, 0.3, so.FEATURES).astype(np.float32)
    inv = rng.uniform(0.5, 1.5, so.FEATURES).astype(np.float32)
    return feats, labels, mean, inv


def _model(seed, mean, inv, bias_scale=0.1):
    m = br.Surrogate(seed=seed)
    p, _, _ = m.parameters()
    rng = np.random.default_rng(seed + 100)
    parts = so.unpack(p.astype(np.float64))
    parts["b1"][:] = rng.normal(0, bias_scale, 128)
    parts["b2"][:] = rng.normal(0, bias_scale, 128)
    parts["b3"][:2] = rng.normal(0, bias_scale, 2)
    m.load(so.pack(parts).astype(np.float32), mean, inv)
    return m


@pytest.mark.parametrize("n", [1, 127, 1000, 20000])
def test_forward_matches_oracle(gpu_lib, n):
    feats, _, mean, inv = _batch(n, n)
    m = _model(5, mean, inv)
    out = m.score(torch.from_numpy(feats).cuda()).cpu().numpy()
    params, _, _ = m.parameters()
    want, _ = so.forward(feats, params, mean, inv)
    scale = np.abs(want).max() + 1e-6
    # BF16 operands, FP32 accumulation: 1e-2 relative to the output scale.
    assert np.max(np.abs(out - want)) <= 1e-2 * scale, np.max(np.abs(out - want)) / scale


@pytest.mark.parametrize("n", [128, 3000])
def test_gradients_match_oracle(gpu_lib, n):
    feats, labels, mean, inv = _batch(11 + n, n)
    m = _model(9, mean, inv)
    g, loss = m.gradients(torch.from_numpy(feats).cuda(), torch.from_numpy(labels).cuda())
    params, _, _ = m.parameters()
    want, want_loss = so.gradients(feats, labels, params, mean, inv)
    assert abs(loss - want_loss) <= 1e-3 * abs(want_loss) + 1e-4
    for name, (o, shape) in so.OFF.items():
        k = int(np.prod(shape))
        a, b = g[o:o + k].astype(np.float64), want[o:o + k]
        err = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-12)
        assert err < 1e-2, (name, err)
    # the padding never receives a gradient
    parts = so.unpack(g.astype(np.float64))
    assert not parts["w1"][:, so.FEATURES:].any() and not parts["w3"][2:].any() and not parts["b3"][2:].any()


def test_training_learns_a_rule(gpu_lib):
    """Adam steps through the fused train kernel fit a separable rule."""
    rng = np.random.default_rng(1)
    n = 8192
    feats = rng.normal(0, 1, (n, so.FEATURES)).astype(np.float32)
    rule = (feats[:, 3] + 0.5 * feats[:, 7] > 0).astype(np.float32)
    labels = np.stack([rule, np.abs(feats[:, 1])], 1).astype(np.float32)
    m = br.Surrogate(seed=2)
    m.load(m.parameters()[0], np.zeros(so.FEATURES, np.float32), np.ones(so.FEATURES, np.float32))
    f, l = torch.from_numpy(feats).cuda(), torch.from_numpy(labels).cuda()
    first = m.train_step(f, l, 3e-3)
    for _ in range(300):
        last = m.train_step(f, l, 3e-3)
    assert last < 0.35 * first, (first, last)
    logits = m.score(f).cpu().numpy()[:, 0]
    assert np.mean((logits > 0) == (rule > 0)) > 0.95


def test_features_of_legal_edits(gpu_lib):
    mesh = syn.noisy_icosphere(3, 4)
    with br.AuditSession(mesh) as s:
        feats, cols = s.surrogate_features(24.0, 48.0)
        actions = s.actions()
    f = feats.cpu().numpy()
    assert f.shape == (len(actions), so.FEATURES) and len(cols) == len(actions)
    assert np.array_equal(cols["from"], actions["from"]) and np.array_equal(cols["to"], actions["to"])
    assert np.isfinite(f).all()
    pos = mesh.positions.astype(np.float64)
    lo, hi = pos.min(0), pos.max(0)
    center = ((lo + hi) * 0.5).astype(np.float32).astype(np.float64)
    radius = np.sqrt(((pos - center) ** 2).sum(1)).max()
    length = np.linalg.norm(pos[cols["to"]] - pos[cols["from"]], axis=1)
    np.testing.assert_allclose(f[:, 37], length * 24.0 / (2 * radius), rtol=1e-4)
    np.testing.assert_allclose(f[:, 39], length * 48.0 / (2 * radius), rtol=1e-4)
    assert (f[:, 33] >= 2).all() and (f[:, 42] >= 1).all()


def _c1_gates(screen=24.0, views=(8, 0, 0xB1172026), ss=8):
    return [br.eval_settings(screen, 2.0, views, ss, ss, 1.0), br.eval_settings(screen, 1.0, views, ss, ss, 1.0),
            br.eval_settings(screen, 2.0, views, ss, ss, 0.5), br.eval_settings(screen, 1.0, views, ss, ss, 0.5)]


def test_full_keep_equals_plain_batched_walk(gpu_lib):
    """Keeping every ranked edit is the plain batched walk, commit for commit."""
    mesh = syn.noisy_icosphere(3, 6)
    gates = _c1_gates()
    with br.AuditSession(mesh) as s:
        plain = s.execute(mesh.face_count // 3, 400, gates, batch=16)
        s.reset()
        m = br.Surrogate(seed=4)
        s.attach_surrogate(m)
        full = s.execute(mesh.face_count // 3, 400, gates, batch=16, keep_permille=1000)
    assert np.array_equal(plain["commits"], full["commits"]) and plain["trials"] == full["trials"]


def test_pruned_walk_passes_the_exact_audit(gpu_lib):
    """With an untrained (arbitrary) surrogate keeping 25%, every emitted
    state still passes the four gates: the exact audit judges each batch."""
    mesh = syn.noisy_icosphere(3, 8)
    gates = _c1_gates(screen=64.0)
    with br.AuditSession(mesh) as s:
        m = br.Surrogate(seed=12)
        s.attach_surrogate(m)
        r = s.execute(mesh.face_count // 4, 300, gates, batch=16, keep_permille=250)
        idx, pos = s.state()
        state = syn.Mesh(pos, idx)
        assert len(r["commits"]) > 0
        for g in gates:
            meas = br.evaluate(mesh, state, g, session=s)
            assert meas.passed == 1 and meas.complete == 1


def test_trained_surrogate_beats_untrained(gpu_lib):
    """What training buys: on held-out meshes at 96 px (where the exact audit
    rejects some candidates), the edits the trained network keeps (top 25%)
    hold far fewer exact rejections than those an untrained network keeps,
    and more accepted candidates than the base rate."""
    from blitzremesher_b200 import surrogate_train as st
    gates = st.c1_gates(screen=96.0, views=16)
    train = st.generate([2, 3], [1.0, 0.85], gates)
    held = st.generate([1001], [1.0, 0.85], gates)
    model = br.Surrogate(seed=1)
    st.fit(model, train, epochs=4, lr=1e-3)
    untrained = br.Surrogate(seed=1)
    untrained.load(untrained.parameters()[0], *st.normalisation(train.features))
    ours, base = st.pruning_stats(model, held), st.pruning_stats(untrained, held)
    assert base["kept_rejections"] > 0
    assert ours["kept_rejections"] * 2 <= base["kept_rejections"], (ours, base)
    assert ours["kept_acceptance"] > base["kept_acceptance"]
    assert ours["kept_acceptance"] >= ours["base_acceptance"]
