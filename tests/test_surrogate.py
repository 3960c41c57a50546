"""The surrogate network (include/negf_mlp.h) and the adaptive sampler.

CPU: node placement and quadrature helpers.  GPU: forward pass and gradients
of the network kernels against the NumPy oracle (oracle/mlp_oracle.py, BF16
operands mimicked, FP64 accumulation), training, and the gain of
surrogate-placed RGF nodes over a uniform grid on unseen devices."""
import numpy as np
import pytest

from negftrans_b200 import surrogate as S

WID = [17, 64, 48, 32, 1]


def test_curvature_nodes_follow_the_predicted_curvature():
    e = np.linspace(0.0, 30.0, 4096)
    t = 1.0 / (1.0 + np.exp(-(e - 12.0) / 0.3)) + 1.0 / (1.0 + np.exp(-(e - 21.0) / 0.3))
    nodes = S.curvature_nodes(e, t, 65)
    assert nodes[0] == 0.0 and nodes[-1] == 30.0
    assert np.all(np.diff(nodes) > 0) and 60 <= len(nodes) <= 65
    near = np.sum((np.abs(nodes - 12.0) < 1.5) | (np.abs(nodes - 21.0) < 1.5))
    assert near > 0.4 * len(nodes)   # 20 % of the window holds twice its share
    # a curve without curvature gives (nearly) uniform nodes
    flat = S.curvature_nodes(e, 0.1 * e, 33)
    np.testing.assert_allclose(np.diff(flat), 30.0 / 32, rtol=0.05)


def test_quadratures():
    e = np.linspace(0.0, 2.0, 9)
    assert abs(S.simpson(e, e ** 3) - 4.0) < 1e-12
    assert abs(S.trapezoid(e, 3 * e + 1) - 8.0) < 1e-12


def test_descriptors_of_a_sampled_device():
    (d,) = S.sample_devices(1, seed=5, nz=20)
    assert d.desc.shape == (16,)
    assert np.all(np.isfinite(d.desc))
    assert abs(d.desc[14] - d.Vg * 1e3) < 1e-12 and d.desc[15] == d.w
    assert 20.0 <= d.desc[14] <= 80.0 and 8.0 <= d.w <= 25.0


def _data(rng, n):
    x = rng.uniform(-1, 1, (n, WID[0])).astype(np.float32)
    t = (np.sin(3 * x[:, :1]) * np.cos(2 * x[:, 1:2]) + 0.3 * x[:, 2:3]).astype(np.float32)
    w = rng.uniform(0.5, 1.5, t.shape).astype(np.float32)
    return x, t, w


def _layers(flat):
    from oracle import mlp_oracle as M
    out = []
    for W, b in M.unpack(flat, WID):
        out += [W, b]
    return out


@pytest.mark.gpu
def test_mlp_forward_matches_oracle():
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(1)
    x, _, _ = _data(rng, 300)
    with S.MLP(WID, max_batch=128, seed=3) as net:
        y = net.forward(x)   # three chunks of max_batch rows
        ref, _ = M.forward(net.params.astype(np.float64), WID, x)
    assert np.max(np.abs(y - ref)) <= 2e-3 * np.max(np.abs(ref))


@pytest.mark.gpu
def test_mlp_gradient_matches_oracle():
    """Every layer's weight and bias gradient against the oracle with the same
    BF16 operand rounding (tight), and against the exact FP64 gradient (loose)."""
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(2)
    x, t, w = _data(rng, 200)
    with S.MLP(WID, max_batch=256, seed=4) as net:
        p = net.params.astype(np.float64)
        for rep in range(2):
            loss, g = net.grad(x, t, w)
            ref_loss, ref = M.loss_and_grad(p, WID, x, t, w, bf16_ops=True)
            assert abs(loss - ref_loss) <= 1e-4 * ref_loss
            for a, b in zip(_layers(g), _layers(ref)):
                assert np.linalg.norm(a - b) <= 5e-3 * np.linalg.norm(b) + 1e-7
        _, exact = M.loss_and_grad(p, WID, x, t, w, bf16_ops=False)
        for a, b in zip(_layers(g), _layers(exact)):
            assert np.linalg.norm(a - b) <= 5e-2 * np.linalg.norm(b) + 1e-6


@pytest.mark.gpu
def test_mlp_training_fits_a_smooth_function():
    rng = np.random.default_rng(3)
    x, t, w = _data(rng, 4096)
    with S.MLP(WID, max_batch=1024, seed=5) as net:
        l0, _ = net.grad(x[:1024], t[:1024], w[:1024])
        hist = net.train(x, t, w, steps=800, batch=512, lr=2e-3, seed=1)
        l1, _ = net.grad(x[:1024], t[:1024], w[:1024])
    assert len(hist) == 800 and np.all(np.isfinite(hist))
    assert l1 < 0.05 * l0


@pytest.mark.gpu
def test_surrogate_guided_sampling_on_unseen_devices():
    """Trained on RGF transmission and probe LDOS of 48 seeded QPC + disorder devices, the
    surrogate places the nodes of unseen devices.  Every node is an RGF solve,
    both node sets reach the 1e-4 integral tolerance, and the solve counts of
    the two methods are what the comparison reports (the measured ratio on
    this device family is recorded by bench.py --surrogate)."""
    train = S.sample_devices(48, seed=11, nz=60)
    e_train = S.training_energies(96)
    T, L = S.training_set(train, 96)
    assert T.shape == (48, 96) and np.all(T >= -1e-9)
    assert L.shape == (48, 96, S.N_PROBES) and np.all(np.isfinite(L)) and np.all(L > 0)
    sur = S.Surrogate(seed=0)
    try:
        hist = sur.fit(train, e_train, T, L, steps=(800, 200), lr=(1e-3, 2e-4), batch=2048)
        assert np.all(np.isfinite(hist)) and hist[-50:].mean() < 0.2 * hist[:50].mean()
        test = S.sample_devices(2, seed=99, nz=60)
        lp = sur.predict_ldos(test[0].desc, e_train)
        assert lp.shape == (96, S.N_PROBES) and np.all(np.isfinite(lp)) and np.all(lp >= 0)
        rows = S.compare(sur, test, tol=1e-4)
        for d in test:
            rgf = S.RGF(d)
            try:
                # the counts are those of RGF solves: the reference grid plus each candidate grid
                i_ref = S.reference_integral(rgf)
                n_u, err_u = S.solves_to_tolerance(rgf, i_ref, S.uniform_nodes, 1e-4)
                assert rgf.solves == 4097 + sum(S.CANDIDATES)
            finally:
                rgf.close()
    finally:
        sur.close()
    for r in rows:
        assert r["uniform"] is not None and r["adaptive"] is not None, r
        assert np.isfinite(r["surrogate_max_abs_err"])
