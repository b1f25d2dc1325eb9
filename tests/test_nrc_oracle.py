"""CPU checks of the radiance-cache oracle (oracle/nrc_oracle.py): the
spherical-harmonic basis is orthonormal, the grid interpolation weights form a
partition of unity with in-range indices, and the analytic gradients of the
relative-L2 loss (weights and grid features) agree with float64 finite
differences of the same model without bf16 rounding."""
import numpy as np

import nrc_oracle as N


def test_sh_basis_is_orthonormal():
    rng = np.random.default_rng(0)
    d = rng.normal(size=(400000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    y = N.sh4(d.astype(np.float32)).astype(np.float64)
    gram = (y.T @ y) * (4 * np.pi / d.shape[0])
    assert np.abs(gram - np.eye(16)).max() < 0.03


def test_grid_weights_and_indices():
    rng = np.random.default_rng(1)
    p = rng.uniform(0, 1, (2000, 3)).astype(np.float32)
    p[:5] = [[0, 0, 0], [1, 1, 1], [1, 0, 1], [0.5, 0.5, 0.5], [1 - 1e-7, 0, 0]]
    corners = N.grid_corners(p)
    dense = [N.level_dense_side(s) for s in N.level_scales()]
    assert dense[0] > 0 and dense[-1] == 0  # coarse levels dense, fine ones hashed
    for idx, w in corners:
        assert np.allclose(w.sum(1), 1.0, atol=1e-5)
        assert idx.min() >= 0 and idx.max() < N.TABLE
    s = N.level_scales()
    assert abs(s[0] - 16) < 1e-4 and abs(s[-1] - 2048) < 0.1


def _problem(n=6, seed=2):
    rng = np.random.default_rng(seed)
    q = {"pos": rng.uniform(-1, 3, (n, 3)), "dir": rng.normal(size=(n, 3)), "normal": rng.normal(size=(n, 3)),
         "roughness": rng.uniform(0, 1, n), "diffuse": rng.uniform(0, 1, (n, 3)),
         "specular": rng.uniform(0, 1, (n, 3))}
    q["dir"] /= np.linalg.norm(q["dir"], axis=1, keepdims=True)
    q["normal"] /= np.linalg.norm(q["normal"], axis=1, keepdims=True)
    table = rng.uniform(-0.5, 0.5, (N.LEVELS, N.TABLE, 2)).astype(np.float32)
    ws = [w.astype(np.float64) * 3 for w in N.init_weights(seed)]
    target = rng.uniform(0.1, 2.0, (n, 3))
    return q, table, ws, target


def _loss64(q, table, ws, target, box=(-1.0, 0.25)):
    x, _ = N.encode(q, table, *box)
    acts, o, rgb = N.forward(x.astype(np.float64), ws, rnd=False)
    denom = rgb.copy() ** 2 + N.LOSS_EPS
    return float(np.mean((rgb - target) ** 2 / denom)), denom


def test_weight_gradients_match_finite_differences():
    q, table, ws, target = _problem()
    x, _ = N.encode(q, table, -1.0, 0.25)
    acts, o, rgb = N.forward(x.astype(np.float64), ws, rnd=False)
    _, do = N.loss_and_grad(o, rgb, target)
    grads, _ = N.backward(acts, ws, do, rnd=False)
    rng = np.random.default_rng(3)
    # The loss treats its denominator as a constant: finite differences
    # hold it fixed at the unperturbed value.
    _, denom = _loss64(q, table, ws, target)
    for l in range(6):
        rows = 3 if l == 5 else 64
        for _ in range(4):
            i, j = rng.integers(rows), rng.integers(64)
            h = 1e-6
            vals = []
            for sgn in (1, -1):
                wp = [w.copy() for w in ws]
                wp[l][i, j] += sgn * h
                a, oo, rr = N.forward(x.astype(np.float64), wp, rnd=False)
                vals.append(float(np.mean((rr - target) ** 2 / denom)))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - grads[l][i, j]) <= 1e-6 + 1e-4 * abs(fd), (l, i, j, fd, grads[l][i, j])


def test_grid_gradients_match_finite_differences():
    q, table, ws, target = _problem(n=3, seed=4)
    x, corners = N.encode(q, table, -1.0, 0.25)
    acts, o, rgb = N.forward(x.astype(np.float64), ws, rnd=False)
    _, do = N.loss_and_grad(o, rgb, target)
    _, dx = N.backward(acts, ws, do, rnd=False)
    gg = N.grid_backward(dx.astype(np.float32), corners)
    _, denom = _loss64(q, table, ws, target)
    t64 = table.astype(np.float64)
    checked = 0
    for l in (0, 7, 15):
        idx, w = corners[l]
        e = int(idx[0, 3])
        for j in range(2):
            h = 1e-4
            vals = []
            for sgn in (1, -1):
                tp = t64.copy()
                tp[l, e, j] += sgn * h
                xx, _ = N.encode(q, tp, -1.0, 0.25)
                a, oo, rr = N.forward(xx.astype(np.float64), ws, rnd=False)
                vals.append(float(np.mean((rr - target) ** 2 / denom)))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - gg[l, e, j]) <= 1e-6 + 2e-3 * abs(fd), (l, e, j, fd, gg[l, e, j])
            checked += 1
    assert checked == 6


def test_adam_step():
    p = np.array([1.0, -2.0, 0.5], np.float32)
    m = np.zeros(3, np.float32)
    v = np.zeros(3, np.float32)
    g = np.array([0.1, -0.2, 0.0], np.float32)
    N.adam(p, g, m, v, 1)
    # first bias-corrected step moves each parameter by lr * sign(g)
    assert np.allclose(p, [1.0 - 1e-2, -2.0 + 1e-2, 0.5], atol=1e-6)
