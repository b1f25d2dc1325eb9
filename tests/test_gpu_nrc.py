"""Radiance-cache kernels (tcgen05 forward / backward, Adam) against the
numpy oracle (oracle/nrc_oracle.py), through the C ABI.

Tolerances: both sides round activations, weights and gradients to bf16 at
the same points and accumulate in fp32, but in different orders, so values
agree to a few fp32 ulps except where a pre-rounding difference crosses a bf16
rounding boundary. Such a flip changes one activation by one bf16 ulp and,
through the exp output, the radiance by up to a few percent, so forward
outputs are bounded at 1e-4 relative for the median, 1e-3 for the 99.9th
percentile and 5e-2 for the maximum; gradient arrays are compared by their
relative Frobenius error (< 2e-2)."""
import numpy as np
import pytest

import nrc_oracle as N
from yaoray_b200.nrc import RadianceCache

pytestmark = pytest.mark.gpu
LO = np.array([-2.0, -1.0, -3.0], np.float32)
EXTENT = 8.0


def queries(n, seed):
    rng = np.random.default_rng(seed)
    q = {"pos": (LO + rng.uniform(0, EXTENT, (n, 3))).astype(np.float32),
         "dir": rng.normal(size=(n, 3)), "normal": rng.normal(size=(n, 3)),
         "roughness": rng.uniform(0, 1, n).astype(np.float32),
         "diffuse": rng.uniform(0, 1, (n, 3)).astype(np.float32),
         "specular": rng.uniform(0, 1, (n, 3)).astype(np.float32)}
    for k in ("dir", "normal"):
        q[k] = (q[k] / np.linalg.norm(q[k], axis=1, keepdims=True)).astype(np.float32)
    flat = np.concatenate([q["pos"], q["roughness"][:, None], q["dir"], q["normal"], q["diffuse"], q["specular"]], 1)
    return q, np.ascontiguousarray(flat, np.float32)


def params(seed, scale=2.0):
    rng = np.random.default_rng(seed)
    ws = N.init_weights(seed)
    w = np.zeros((6, 64, 64), np.float32)
    for l in range(6):
        w[l, :ws[l].shape[0]] = ws[l] * scale
    w[5, 3:] = 0.0
    grid = rng.uniform(-0.3, 0.3, (N.LEVELS, N.TABLE, 2)).astype(np.float32)
    return w, grid


def oracle_weights(w):
    return [N.bf16(w[l]) for l in range(5)] + [N.bf16(w[5, :16])]


def fp16(a):
    return a.astype(np.float16).astype(np.float32)


def rel_fro(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


@pytest.fixture(scope="module")
def cache(cuda):
    c = RadianceCache(LO, EXTENT, seed=3)
    yield c
    c.close()


def test_forward_matches_oracle(cuda, cache):
    import torch
    w, grid = params(11)
    cache.set_params(w, grid)
    q, flat = queries(3001, 1)  # a partial last tile
    out = cache.infer(torch.from_numpy(flat).to(cuda)).cpu().numpy()
    cache.check()
    x, _ = N.encode(q, fp16(grid), LO, np.float32(1.0 / EXTENT))
    _, o, rgb = N.forward(x, oracle_weights(w))
    rel = np.abs(out[:, :3] - rgb) / np.maximum(np.abs(rgb), 1e-6)
    assert np.median(rel) < 1e-4 and np.quantile(rel, 0.999) < 1e-3 and rel.max() < 5e-2, \
        (np.median(rel), np.quantile(rel, 0.999), rel.max())


@pytest.mark.parametrize("n", [1000, 40000])
def test_gradients_match_oracle(cuda, cache, n):
    import torch
    w, grid = params(12)
    cache.set_params(w, grid)
    q, flat = queries(n, 2)
    rng = np.random.default_rng(5)
    target = np.zeros((n, 4), np.float32)
    target[:, :3] = rng.uniform(0.05, 3.0, (n, 3))
    wg, gg, loss = cache.gradients(torch.from_numpy(flat).to(cuda), torch.from_numpy(target).to(cuda))
    x, corners = N.encode(q, fp16(grid), LO, np.float32(1.0 / EXTENT))
    ows = oracle_weights(w)
    acts, o, rgb = N.forward(x, ows)
    ref_loss, do = N.loss_and_grad(o, rgb, target[:, :3])
    grads, dx = N.backward(acts, ows, do)
    assert abs(loss / ref_loss - 1) < 1e-3
    for l in range(6):
        rows = 16 if l == 5 else 64
        assert rel_fro(wg[l, :rows], grads[l]) < 2e-2, (l, rel_fro(wg[l, :rows], grads[l]))
        assert not wg[l, rows:].any()
    ref_grid = N.grid_backward(dx.astype(np.float32), corners)
    assert rel_fro(gg, ref_grid) < 2e-2, rel_fro(gg, ref_grid)


def test_adam_step_matches_oracle(cuda, cache):
    import torch
    w, grid = params(13)
    cache.set_params(w, grid)
    q, flat = queries(2048, 3)
    target = np.full((2048, 4), 0.5, np.float32)
    qt, tt = torch.from_numpy(flat).to(cuda), torch.from_numpy(target).to(cuda)
    wg, gg, _ = cache.gradients(qt, tt)
    fresh = RadianceCache(LO, EXTENT, seed=3)  # step counter 0, zero moments
    fresh.set_params(w, grid)
    fresh.train_step(qt, tt)
    fresh.check()
    w_after, g_after = fresh.get_params()
    fresh.close()
    p = w.copy()
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    N.adam(p, wg, m, v, 1)
    diff = np.abs(w_after - p)
    assert (diff > 1e-5).mean() < 1e-3, (diff > 1e-5).mean()
    # the grid: lazy Adam over the entries the batch touched, the rest untouched
    p01 = np.clip((q["pos"] - LO) * np.float32(1.0 / EXTENT), 0.0, 1.0).astype(np.float32)
    mask = N.touched(N.grid_corners(p01))
    assert np.array_equal(g_after[~mask], grid[~mask])
    gp, gm, gv = grid.copy(), np.zeros_like(grid), np.zeros_like(grid)
    N.adam(gp, gg, gm, gv, 1, mask)
    gdiff = np.abs(g_after - gp)[mask]
    assert (gdiff > 1e-5).mean() < 1e-3, (gdiff > 1e-5).mean()
    assert (g_after[mask] != grid[mask]).mean() > 0.5  # the touched entries did move


def test_parameter_average_matches_oracle(cuda):
    import torch
    w, grid = params(17)
    c = RadianceCache(LO, EXTENT, seed=3)
    c.set_average_decay(0.9)
    c.set_params(w, grid)
    aw, ag = c.get_averaged_params()
    assert np.array_equal(aw, w) and np.array_equal(ag, grid)  # restarted at the parameters
    q, flat = queries(1024, 5)
    qt = torch.from_numpy(flat).to(cuda)
    tt = torch.from_numpy(np.full((1024, 4), 0.3, np.float32)).to(cuda)
    avg_w, avg_g = w.copy(), grid.copy()
    p01 = np.clip((q["pos"] - LO) * np.float32(1.0 / EXTENT), 0.0, 1.0).astype(np.float32)
    mask = N.touched(N.grid_corners(p01))  # the lazy grid optimiser updates these entries only
    for step in range(1, 5):
        c.train_step(qt, tt)
        pw, pg = c.get_params()
        N.average(avg_w, pw, step, 0.9)
        N.average(avg_g, pg, step, 0.9, mask)
    c.check()
    aw, ag = c.get_averaged_params()
    c.close()
    assert np.array_equal(aw, avg_w)
    assert np.array_equal(ag, avg_g)
    assert not np.array_equal(aw, pw)


def test_training_learns_a_radiance_function(cuda):
    import torch
    c = RadianceCache(LO, EXTENT, seed=4)

    def target_of(q):
        p, d = q["pos"], q["dir"]
        rgb = np.stack([0.6 + 0.4 * np.sin(0.9 * p[:, 0] + k) * np.cos(0.6 * p[:, 2]) + 0.2 * d[:, 1] * (k - 1)
                        for k in range(3)], 1)
        out = np.zeros((p.shape[0], 4), np.float32)
        out[:, :3] = np.maximum(rgb, 0.02) * (0.3 + q["diffuse"])
        return out

    vq, vflat = queries(8192, 99)
    vt = target_of(vq)
    vq_t = torch.from_numpy(vflat).to(cuda)

    def val_loss():
        pred = c.infer(vq_t).cpu().numpy()[:, :3]
        return float(np.mean((pred - vt[:, :3]) ** 2 / (pred ** 2 + 0.01)))

    before = val_loss()
    for step in range(300):
        q, flat = queries(16384, 1000 + step)
        c.train_step(torch.from_numpy(flat).to(cuda), torch.from_numpy(target_of(q)).to(cuda))
    c.check()
    after = val_loss()
    c.close()
    assert after < 0.1 * before, (before, after)
    assert after < 0.05, after


def test_copied_state_matches_and_trains_alike(cuda):
    """yrc_nrc_copy_state copies everything an optimiser step reads. Right
    after the copy, parameters, moving averages and inference are
    bit-identical. After the same further steps the two stay within the
    run-to-run spread of training (gradients are summed with fp32 atomics, so
    training is not bit-reproducible), far closer than a cache that got only
    the parameters (fresh Adam moments and step count)."""
    import torch
    a = RadianceCache(LO, EXTENT, seed=5)
    b = RadianceCache(LO, EXTENT, seed=6)
    c = RadianceCache(LO, EXTENT, seed=7)
    data = []
    rng = np.random.default_rng(8)
    for k in range(6):
        _, flat = queries(4096, 500 + k)
        data.append((torch.from_numpy(flat).to(cuda),
                     torch.from_numpy(rng.uniform(0.1, 2.0, (4096, 4)).astype(np.float32)).to(cuda)))
    for q, t in data[:3]:
        a.train_step(q, t)
    b.copy_from(a)
    c.set_params(*a.get_params())
    for x, y in zip(a.get_params() + a.get_averaged_params(), b.get_params() + b.get_averaged_params()):
        assert x.tobytes() == y.tobytes()
    _, flat = queries(2048, 77)
    qt = torch.from_numpy(flat).to(cuda)
    assert torch.equal(a.infer(qt), b.infer(qt))
    for q, t in data[3:]:
        for m in (a, b, c):
            m.train_step(q, t)
    for m in (a, b, c):
        m.check()
    wa, ga = a.get_params()
    wb, gb = b.get_params()
    wc, gc = c.get_params()
    copy_gap = rel_fro(wb, wa) + rel_fro(gb, ga)
    params_only_gap = rel_fro(wc, wa) + rel_fro(gc, ga)
    assert copy_gap < 1e-3 and copy_gap < 0.05 * params_only_gap, (copy_gap, params_only_gap)
    for m in (a, b, c):
        m.close()
