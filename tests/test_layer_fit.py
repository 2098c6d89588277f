"""Closed-loop gain search of the learned layer (gfb.layer.fit_gains) on a
synthetic objective in place of whole runs: CPU only."""

import numpy as np

from gfb import layer as gl


def test_fit_gains_finds_the_minimum_of_a_separable_objective(monkeypatch):
    target = np.zeros((10, 3))
    target[4] = [1.0, -0.5, 0.25]
    target[9] = [2.0, 2.0, 2.0]
    calls = []

    def fake_loop_error(cases, params, scales, gains, scale_mult=1.0, device=0, planes=None):
        calls.append(np.array(gains))
        return float(np.sum((np.log(gains) - target) ** 2)) + 0.1

    monkeypatch.setattr(gl, "loop_error", fake_loop_error)
    params = np.zeros((10, gl.N_PARAMS), dtype=np.float32)
    gains, err, hist = gl.fit_gains([None], params, np.ones(4), nets=[4, 9], min_step=0.125, max_evals=500)
    assert gains.shape == (10, 3) and gains.dtype == np.float32
    np.testing.assert_allclose(np.log(gains[[4, 9]]), target[[4, 9]], atol=0.125)
    np.testing.assert_array_equal(gains[[0, 1, 2, 3, 5, 6, 7, 8]], 1.0)  # networks not fitted stay at 1
    assert hist[0] == (1, 3 * 2.0 ** 2 + 1.0 + 0.25 + 0.0625 + 0.1)  # the start: unit gains
    assert err < hist[0][1]
    assert all(e2 < e1 for (_, e1), (_, e2) in zip(hist, hist[1:]))  # only improvements are kept
    assert len(calls) >= hist[-1][0]


def test_fit_gains_respects_the_bound_and_the_evaluation_budget(monkeypatch):
    def fake_loop_error(cases, params, scales, gains, scale_mult=1.0, device=0, planes=None):
        return float(-np.sum(np.log(gains)))  # better without end: the bound stops it

    monkeypatch.setattr(gl, "loop_error", fake_loop_error)
    params = np.zeros((10, gl.N_PARAMS), dtype=np.float32)
    gains, err, hist = gl.fit_gains([None], params, np.ones(4), nets=[4], max_evals=400)
    np.testing.assert_allclose(np.log(gains[4]), gl.LOG_GAIN_BOUND, atol=1e-6)
    gains, err, hist = gl.fit_gains([None], params, np.ones(4), nets=[4], max_evals=5)
    assert hist[-1][0] <= 5


def test_fit_output_layer_finds_the_row_factors_of_a_synthetic_objective(monkeypatch):
    rng = np.random.default_rng(3)
    params = rng.normal(0.0, 0.1, size=(10, gl.N_PARAMS)).astype(np.float32)
    sl = slice(gl.W3_OFFSET, gl.W3_OFFSET + gl.N_OUT * gl.N_HID)
    want = np.ones((10, 3))
    want[4] = [0.0, 2.0, 1.5]
    want[9] = [0.5, 0.75, 3.0]
    target = gl.scale_output_rows(params, want)

    def fake_loop_error(cases, p, scales, gains, scale_mult=1.0, device=0, planes=None):
        return float(np.sum((p[:, sl] - target[:, sl]) ** 2))

    monkeypatch.setattr(gl, "loop_error", fake_loop_error)
    fitted, alpha, err, hist = gl.fit_output_layer([None], params, np.ones(4), nets=[4, 9], max_evals=300)
    np.testing.assert_allclose(alpha[[4, 9]], want[[4, 9]], atol=0.07)
    np.testing.assert_array_equal(alpha[[0, 1, 2, 3, 5, 6, 7, 8]], 1.0)
    assert err < 1e-2 * hist[0][1]
    assert all(e2 < e1 for (_, e1), (_, e2) in zip(hist, hist[1:]))
    keep = np.ones(gl.N_PARAMS, dtype=bool)
    keep[sl] = False
    np.testing.assert_array_equal(fitted[:, keep], params[:, keep])  # hidden layers untouched
    np.testing.assert_allclose(gl.scale_output_rows(params, np.zeros((10, 3)))[:, sl], 0.0)
