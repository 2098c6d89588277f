"""Learned absorbing layer: training gradients against an FP64 CPU MLP, the
tensor-core inference kernel against the same MLP on a real step, and the
C-PML fallback of the energy monitor."""

import numpy as np
import pytest

import gfb
from gfb import layer as gl
from gfb import mesh

pytestmark = pytest.mark.gpu


def bf16(x):
    """Round to the nearest BF16 value (ties to even), as the GPU does."""
    x = np.asarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def split(p):
    w1 = p[: 64 * 36].reshape(64, 36)
    w2 = p[64 * 36: 64 * 36 + 64 * 64].reshape(64, 64)
    w3 = p[64 * 36 + 64 * 64:].reshape(3, 64)
    return w1, w2, w3


def logits64(p, xh, rounded=True):
    """f(xh) = (y(xh) + y(-xh)) / 2 with y = W3 relu(W2 relu(W1 xh)), FP64,
    on the BF16-rounded weights (as the GPU uses them) unless rounded=False."""
    w1, w2, w3 = ((bf16(w) if rounded else w) for w in split(p))
    z = xh @ w1.T
    yp = np.maximum(np.maximum(z, 0) @ w2.T, 0) @ w3.T
    ym = np.maximum(np.maximum(-z, 0) @ w2.T, 0) @ w3.T
    return 0.5 * (yp + ym)


def softplus(f):
    return np.where(f > 20, f, np.log1p(np.exp(np.minimum(f, 20))))


def normalised(x_raw, sc):
    ch = np.array([sc[(q % 9) // 3] for q in range(36)])
    x = x_raw / ch
    n = np.linalg.norm(x, axis=1, keepdims=True)
    inv = np.where(n > 0, 1.0 / np.where(n > 0, n, 1.0), 0.0)
    return x * inv, inv


def loss64(p, x_raw, t_raw, sc, rounded=True):
    xh, inv = normalised(x_raw, sc)
    th = t_raw / sc[3] * inv
    c = -softplus(logits64(p, xh, rounded)) * xh[:, 3:6]
    e = c - th
    return 0.5 * np.sum(e * e)


def grad64(p, x, t, sc):
    """Analytic FP64 gradient of loss64 (backpropagation written out)."""
    w1, w2, w3 = (bf16(w) for w in split(p))
    xh, inv = normalised(x, sc)
    th = t / sc[3] * inv
    z = xh @ w1.T
    h1p, h1m = np.maximum(z, 0), np.maximum(-z, 0)
    h2p, h2m = np.maximum(h1p @ w2.T, 0), np.maximum(h1m @ w2.T, 0)
    f = 0.5 * (h2p @ w3.T + h2m @ w3.T)
    vh = xh[:, 3:6]
    e = -softplus(f) * vh - th
    dy = 0.5 * e * (-vh) / (1.0 + np.exp(-f))
    g3 = dy.T @ h2p + dy.T @ h2m
    dz2p = (dy @ w3) * (h2p > 0)
    dz2m = (dy @ w3) * (h2m > 0)
    g2 = dz2p.T @ h1p + dz2m.T @ h1m
    dz1 = (dz2p @ w2) * (z > 0) - (dz2m @ w2) * (z < 0)
    g1 = dz1.T @ xh
    return np.concatenate([g1.ravel(), g2.ravel(), g3.ravel()])


def test_training_gradient_matches_fp64_cpu_mlp():
    rng = np.random.default_rng(1)
    tr = gl.Trainer(n_net=3, capacity=16, seed=7)
    sc = np.array([2e-3, 5e-2, 1.3, 4e6], dtype=np.float32)
    tr.set_scales(sc)
    params, s = tr.params()
    np.testing.assert_array_equal(s, sc)
    n = 300
    x = (rng.standard_normal((n, 36)) * np.array([sc[(q % 9) // 3] for q in range(36)])).astype(np.float32)
    t = (rng.standard_normal((n, 3)) * sc[3]).astype(np.float32)
    for net in (0, 2):
        g, loss = tr.gradient(net, x, t)
        ref = grad64(params[net].astype(np.float64), x.astype(np.float64), t.astype(np.float64), sc.astype(np.float64))
        lref = loss64(params[net].astype(np.float64), x.astype(np.float64), t.astype(np.float64), sc.astype(np.float64))
        assert abs(loss - lref) <= 1e-4 * lref
        assert np.linalg.norm(g - ref) <= 1e-4 * np.linalg.norm(ref)
        # and the analytic FP64 gradient itself against central differences
        # of the FP64 loss, at the BF16-rounded weights without further
        # rounding, on parameters of all three layers
        pr = bf16(params[net])
        for q in (5, 64 * 36 + 100, 6592 - 1, 6592 - 70):
            step = 1e-6 * max(abs(pr[q]), 1e-3)
            p1, p2 = pr.copy(), pr.copy()
            p1[q] += step
            p2[q] -= step
            fd = (loss64(p1, x, t, sc, False) - loss64(p2, x, t, sc, False)) / (2 * step)
            assert abs(fd - ref[q]) <= 1e-3 * max(abs(ref[q]), 1e-3 * np.abs(ref).max())
    tr.close()


def thin_problem(nsteps=40, with_cpml=True):
    p = gl.PairSpec(ni=6, nj=5, nk=4, d=500.0, seed=4, src=(1400.0, 1200.0, 900.0), nsteps=nsteps)
    return gl.build_domain(p, 1, with_cpml=with_cpml), p


def test_inference_kernel_matches_fp64_mlp_on_a_step():
    """A layer with random parameters on a thin domain: the change of the
    acceleration of the layer nodes over one step, times their mass, equals
    the trapezoidal dashpot force the network gives for their features (only
    the newest tap is nonzero after a state overwrite).  BF16 activations on
    the tensor cores: 2e-2."""
    # legacy damping instead of C-PML: then the force the layer sees is the
    # whole force of the step, m a without the layer
    prob, _ = thin_problem(with_cpml=False)
    lay = gl.Layer(prob)
    assert lay.n_net == 10 and lay.node.size > 0
    rng = np.random.default_rng(3)
    tr = gl.Trainer(n_net=lay.n_net, capacity=8, seed=11)
    params, _ = tr.params()
    tr.close()
    n = prob["n_node"]
    u = rng.standard_normal((n, 3)) * 1e-3
    v = rng.standard_normal((n, 3)) * 1e-2
    a = rng.standard_normal((n, 3)) * 1e-1
    # output scale: damping of order m/dt/10 on these velocities, so the
    # correction is comparable with the elastic force and below the cap
    sc = np.array([1e-3, 1e-2, 1e-1, 1e7], dtype=np.float32)
    out = []
    for with_layer in (False, True):
        s = gfb.Solver(prob, dirs=[0], precision=gfb.FP32, record=False)
        if with_layer:
            gl.attach(s, lay, params, sc, threshold=1e30)
        s.set_state(0, 10, u, v, a)
        s.advance(1)
        out.append(s.state(0)[2])
        s.close()
    mass = np.zeros(n)
    np.add.at(mass, np.asarray(prob["ibool"]).ravel(), np.asarray(prob["mass"]).ravel())
    got = (out[1] - out[0])[lay.node] * mass[lay.node][:, None]
    # features: newest tap only, face frame, channel-scaled
    x = np.zeros((lay.node.size, 36))
    for j in range(3):
        ax = np.abs(lay.frame[:, j]).astype(int) - 1
        sg = np.sign(lay.frame[:, j])
        rows = np.arange(lay.node.size)
        x[:, 0 * 3 + j] = sg * u[lay.node][rows, ax] / sc[0]
        x[:, 1 * 3 + j] = sg * v[lay.node][rows, ax] / sc[1]
        x[:, 2 * 3 + j] = sg * a[lay.node][rows, ax] / sc[2]
    xh, _ = normalised(x * np.array([sc[(q % 9) // 3] for q in range(36)]), sc)
    dt = prob["dt"]
    want = np.zeros((lay.node.size, 3))
    for k in range(lay.n_net):
        sel = lay.net == k
        if not sel.any():
            continue
        damp = softplus(logits64(params[k].astype(np.float64), xh[sel])) * (sc[3] / sc[1])
        g = np.zeros((sel.sum(), 3))
        nodes = lay.node[sel]
        m = mass[nodes]
        for j in range(3):
            ax = np.abs(lay.frame[sel, j]).astype(int) - 1
            rows = np.arange(g.shape[0])
            d = np.minimum(damp[:, j], m / dt)
            # force of this step without the layer: m a_plain
            vbar = v[nodes][rows, ax] + 0.5 * dt * a[nodes][rows, ax] + 0.5 * dt * out[0][nodes][rows, ax]
            g[rows, ax] = -d * vbar / (1.0 + d * 0.5 * dt / m)
        want[sel] = g
    assert np.linalg.norm(got - want) <= 2e-2 * np.linalg.norm(want)


def test_layer_only_takes_energy_out_and_falls_back_on_non_finite_output():
    """The dashpot form does no positive work (the monitored residual stays
    <= 0 on a real run); a network whose output overflows to infinity is
    switched off by the monitor at once and the run stays finite (plain
    one-element C-PML from then on)."""
    prob, _ = thin_problem(nsteps=150)
    lay = gl.Layer(prob)
    tr = gl.Trainer(n_net=lay.n_net, capacity=8, seed=5)
    params, _ = tr.params()
    tr.close()
    sc = np.array([1e-3, 1e-2, 1e-1, 1e7], dtype=np.float32)
    s = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, record=False)
    gl.attach(s, lay, params, sc, threshold=1e-6)
    s.advance(150)
    active, resid = gl.status(s)
    assert active and resid <= 0.0
    s.close()
    big = params * 0.0
    for k in range(lay.n_net):
        w1, w2, w3 = gl_split(big[k])
        w1[0, 3] = 3e38   # overflows in the first layer
        w2[0, 0] = 3e38
        w3[0, 0] = 3e38
    s = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, record=False)
    gl.attach(s, lay, big, sc, threshold=1e-6)
    s.advance(150)
    active, resid = gl.status(s)
    assert not active
    for f in range(3):
        u, v, a = s.state(f)
        assert np.all(np.isfinite(u)) and np.all(np.isfinite(v))


def gl_split(p):
    w1 = p[: 64 * 36].reshape(64, 36)
    w2 = p[64 * 36: 64 * 36 + 64 * 64].reshape(64, 64)
    w3 = p[64 * 36 + 64 * 64:].reshape(3, 64)
    return w1, w2, w3


def test_trained_layer_reduces_reflection_against_thick_cpml():
    """End to end on small models: collect replays of two seeded pairs and
    fit the networks; fit the damping gains in closed loop on two further
    training models; then on a held-out model the reflection error of the
    thin domain (one-element C-PML) against the 10-element C-PML reference
    run is well below that of the thin domain without the layer, and the
    layer with its closed-loop gains beats the untrained layer (constant
    damping softplus(0) on every axis, unit gains)."""
    def pair(seed, steps):
        r = np.random.default_rng(seed)
        return gl.PairSpec(ni=6, nj=6, nk=4, d=500.0, seed=seed, f0=float(r.uniform(0.8, 1.2)),
                           src=(float(r.uniform(1.5, 4.5) * 500), float(r.uniform(1.5, 4.5) * 500),
                                float(r.uniform(1.0, 2.5) * 500)), nsteps=steps)
    p0 = pair(11, 10)
    n_net = gl.Layer(gl.build_domain(p0, 1)).n_net
    tr = gl.Trainer(n_net=n_net, capacity=2_000_000, seed=1)
    for k in range(2):
        gl.collect_pair(tr, pair(20 + k, 400), sample_stride=3, node_stride=2)
    assert tr.samples().sum() > 0
    base = tr.baseline_loss()
    loss = tr.fit(8, batch=2048, lr=1e-3, seed=2)
    assert loss[-1] < base
    params, scales = tr.params()
    tr.close()
    zero = params * 0.0

    cases = [gl.loop_case(pair(40 + k, 400), dirs=(0, 1, 2)) for k in range(2)]
    gains, e_fit, hist = gl.fit_gains(cases, zero, scales, max_evals=30)
    assert e_fit < hist[0][1]  # the closed loop lowered the training error
    assert gains.shape == (n_net, 3) and np.all(gains > 0)
    # the output-row factors of the replay-trained networks: never worse
    # than where they start (the networks as trained, with these gains)
    fitted, alpha, e_rows, hist_rows = gl.fit_output_layer(cases, params, scales, gains, max_evals=8)
    assert e_rows <= hist_rows[0][1] and np.all((alpha >= 0) & (alpha <= 4))
    assert np.isfinite(e_rows) and fitted.shape == params.shape

    test = gl.loop_case(pair(99, 500), dirs=(0, 1, 2))
    e_plain = gl.loop_error([test])
    e_replay = gl.loop_error([test], params, scales)
    e_untrained = gl.loop_error([test], zero, scales)
    e_learned = gl.loop_error([test], zero, scales, gains)
    rec, _, st = gl.run_domain(test.thin, zero, scales, gains)
    assert st[0]  # still active: no fallback was needed
    print(f"held-out: no layer {e_plain:.4f}, untrained {e_untrained:.4f}, replay-trained {e_replay:.4f}, "
          f"closed-loop gains {e_learned:.4f} (training {hist[0][1]:.4f} -> {e_fit:.4f}), gains {gains[sorted(set(gl.Layer(test.thin).net))]}")
    assert e_replay < 0.7 * e_plain, (e_replay, e_plain)
    assert e_learned < 0.7 * e_plain, (e_learned, e_plain)
    assert e_learned < e_untrained, (e_learned, e_untrained)
