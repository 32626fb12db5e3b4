"""The surrogate's CPU oracle: its backward pass (without bf16 rounding) against
central finite differences of its forward pass, so that the GPU gradient
check compares against pinned formulas."""

import numpy as np
import pytest

import oracle.surrogate as O


def _tiny():
    from ionosphere_fdtd_b200.surrogate import architecture

    return [(L.fan_in, L.fan_out, L.act, L.expand) for L in architecture(inputs=3, width=5, depth=2, samples=8, t0=2, c0=3, channels=(2, 1), stride=2)]


def test_oracle_backward_matches_finite_differences():
    layers = _tiny()
    rng = np.random.default_rng(3)
    w = [rng.standard_normal((fo, fi)) * 0.7 for fi, fo, _, _ in layers]
    b = [rng.standard_normal(fo) * 0.1 for _, fo, _, _ in layers]
    x = rng.standard_normal((4, 3))
    t = rng.standard_normal((4, 8))

    def loss_of(ws, bs):
        pred, _ = O.forward(layers, ws, bs, x, use_bf16=False)
        return O.mse(pred, t)[0]

    pred, acts = O.forward(layers, w, b, x, use_bf16=False)
    _, grad = O.mse(pred, t)
    gw, gb = O.backward(layers, w, acts, grad, use_bf16=False)
    h = 1e-6
    for i in range(len(layers)):
        for idx in [(0, 0), (w[i].shape[0] - 1, w[i].shape[1] - 1)]:
            wp = [a.copy() for a in w]
            wm = [a.copy() for a in w]
            wp[i][idx] += h
            wm[i][idx] -= h
            fd = (loss_of(wp, b) - loss_of(wm, b)) / (2 * h)
            assert gw[i][idx] == pytest.approx(fd, rel=1e-5, abs=1e-9), (i, idx)
        bp = [a.copy() for a in b]
        bm = [a.copy() for a in b]
        bp[i][0] += h
        bm[i][0] -= h
        fd = (loss_of(w, bp) - loss_of(w, bm)) / (2 * h)
        assert gb[i][0] == pytest.approx(fd, rel=1e-5, abs=1e-9), i


def test_bf16_rounding_is_nearest_even():
    assert O.bf16(1.0 + 2.0**-8)[()] == 1.0  # tie, even mantissa kept
    assert O.bf16(1.0 + 3 * 2.0**-8)[()] == 1.0 + 2.0**-6  # tie, rounds to the even neighbour
    assert O.bf16(1.0 + 2.0**-9)[()] == 1.0


def test_architecture_checks_the_sample_count():
    from ionosphere_fdtd_b200.surrogate import architecture

    with pytest.raises(ValueError, match="samples"):
        architecture(samples=1000)


def test_receiver_geometry_round_trips_through_the_features():
    """A receiver placed at a bearing and great-circle distance from the source is
    encoded back to that distance and bearing (host geometry of the training data)."""

    from ionosphere_fdtd_b200.surrogate import _destination, encode_features

    rng = np.random.default_rng(4)
    rows = []
    truth = []
    for _ in range(200):
        lat, lon = float(rng.uniform(-80, 80)), float(rng.uniform(-180, 180))
        bearing, dist = float(rng.uniform(-180, 180)), float(rng.uniform(0.5, 12.0))
        lat2, lon2 = _destination(lat, lon, bearing, dist)
        assert -90.0 <= lat2 <= 90.0 and -180.0 <= lon2 < 180.0
        rows.append((-7.0, 62.5, 4.5, -2.0, lat, lon, lat2, lon2))
        truth.append((dist, bearing, lat))
    feats = encode_features(np.asarray(rows))
    truth = np.asarray(truth)
    np.testing.assert_allclose(feats[:, 4], truth[:, 0] / 10.0, rtol=0, atol=1e-9)
    np.testing.assert_allclose(feats[:, 5], np.cos(np.radians(truth[:, 1])), rtol=0, atol=1e-7)
    np.testing.assert_allclose(feats[:, 6], np.sin(np.radians(truth[:, 1])), rtol=0, atol=1e-7)
    np.testing.assert_allclose(feats[:, 7], np.sin(np.radians(truth[:, 2])), rtol=0, atol=1e-15)
    np.testing.assert_allclose(feats[:, :4], 0.0, atol=1e-15)  # centre of every parameter range
