"""Device texture parity: SampleTexture4 and BuildTextureMipChain evaluated on
the GPU through the C ABI against the reference's golden vectors
(tests/golden/texture.npz) and the oracle.

Nearest and bilinear lookups and the mip chain are compared bit for bit (any
NaN matches any NaN). Trilinear and EWA lookups pick their level of detail
with log2f, whose last bit in the host C library differs from the device's
correctly rounded log2 for a few percent of arguments; that moves the blend
between two levels by one unit in the last place of the level, so they are
compared within 1e-5 absolute (texel values lie in [0, 1]) and most of them
must still match bit for bit."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from yaoray_b200 import texture as T
from yaoray_b200._lib import YrcError

GOLDEN = Path(__file__).resolve().parent / "golden"
LOD_TOL = 1e-5


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def same_values(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(bits(np.where(na, 0, a)), bits(np.where(nb, 0, b)))


def close_values(a, b, tol):
    """Same NaN positions, |a - b| <= tol elsewhere; returns the fraction of
    rows that match bit for bit."""
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb)
    a0, b0 = np.where(na, 0, a), np.where(nb, 0, b)
    assert np.max(np.abs(a0 - b0), initial=0.0) <= tol
    return float(np.mean(np.all(bits(a0) == bits(b0), axis=1)))


@pytest.mark.gpu
def test_device_texture_matches_reference_golden():
    f = dict(np.load(GOLDEN / "texture.npz"))
    exact_rows, rows = 0.0, 0
    for si in range(len(f["shapes"])):
        tx = f[f"t{si}_texels"]
        for wi, (ws, wt) in enumerate(f["wraps"]):
            uv, fp = f[f"t{si}_w{wi}_uv"], f[f"t{si}_w{wi}_fp"]
            for filt in range(4):
                got = T.sample(T.Texture(tx, filt, int(ws), int(wt)), uv, fp)
                want = f[f"t{si}_w{wi}_f{filt}"]
                if filt in (T.NEAREST, T.BILINEAR):
                    assert same_values(got, want), (si, wi, filt)
                else:
                    exact_rows += close_values(got, want, LOD_TOL) * len(uv)
                    rows += len(uv)
            mips = T.mip_chain(T.Texture(tx, T.BILINEAR, int(ws), int(wt)))
            expect = sorted((k for k in f if k.startswith(f"t{si}_w{wi}_mip")), key=lambda k: int(k.split("mip")[1]))
            assert len(mips) == 1 + len(expect)
            assert np.array_equal(bits(mips[0]), bits(tx))
            for a, k in zip(mips[1:], expect):
                assert np.array_equal(bits(a), bits(f[k])), (si, wi, k)
    assert exact_rows / rows > 0.9


@pytest.mark.gpu
@pytest.mark.parametrize("filt", [T.NEAREST, T.BILINEAR, T.TRILINEAR, T.EWA])
def test_device_texture_matches_oracle_large(filt):
    rng = np.random.default_rng(100 + filt)
    tx = rng.random((600, 1000, 4), dtype=np.float32)
    n = 100000
    uv = rng.uniform(-1.5, 2.5, (n, 2)).astype(np.float32)
    fp = (rng.standard_normal((n, 4)) * np.exp(rng.uniform(-12.0, -2.0, (n, 1)))).astype(np.float32)
    fp[: n // 10] = 0.0
    for ws, wt in [(T.REPEAT, T.MIRRORED_REPEAT), (T.CLAMP_TO_EDGE, T.REPEAT)]:
        got = T.sample(T.Texture(tx, filt, ws, wt), uv, fp)
        want = oracle.oracle_texture_sample(tx, filt, ws, wt, uv, fp)
        if filt in (T.NEAREST, T.BILINEAR):
            assert same_values(got, want)
        else:
            assert close_values(got, want, LOD_TOL) > 0.9


@pytest.mark.gpu
def test_device_mip_chain_matches_oracle_odd_sizes():
    rng = np.random.default_rng(5)
    for h, w in [(1, 1000), (777, 3), (129, 257)]:
        tx = rng.random((h, w, 4), dtype=np.float32)
        for ws, wt in [(T.REPEAT, T.REPEAT), (T.MIRRORED_REPEAT, T.CLAMP_TO_EDGE)]:
            got = T.mip_chain(T.Texture(tx, T.TRILINEAR, ws, wt))
            want = oracle.oracle_texture_mip_chain(tx, ws, wt)
            assert len(got) == 1 + len(want)
            for a, b in zip(got[1:], want):
                assert np.array_equal(bits(a), bits(b))


@pytest.mark.gpu
def test_device_texture_without_data_samples_black_with_alpha_one():
    uv = np.array([[0.5, 0.5], [3.0, -1.0]], np.float32)
    for filt in range(4):
        got = T.sample(T.Texture(np.zeros((0, 0, 4), np.float32), filt), uv, np.ones((2, 4), np.float32))
        assert np.array_equal(got, np.tile(np.array([0, 0, 0, 1], np.float32), (2, 1)))
    assert T.mip_chain(T.Texture(np.zeros((0, 0, 4), np.float32))) == []


def test_texture_eval_rejects_bad_modes():
    """Mode checks run before any CUDA call, so they need no device."""
    tx = np.ones((2, 2, 4), np.float32)
    with pytest.raises(YrcError):
        T.sample(T.Texture(tx, 4), np.zeros((1, 2), np.float32))
    with pytest.raises(YrcError):
        T.sample(T.Texture(tx, T.BILINEAR, 3, 0), np.zeros((1, 2), np.float32))
    assert T.sample(T.Texture(tx), np.zeros((0, 2), np.float32)).shape == (0, 4)
