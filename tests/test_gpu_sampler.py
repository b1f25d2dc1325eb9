"""Device sampling parity: the sampler, PCG32 and SeedForPixelSample code the
path-tracing kernels draw with, evaluated on the GPU through the C ABI and
compared bit for bit with the reference's golden vectors
(tests/golden/sampler.npz) and with the oracle on fresh seeded queries."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from yaoray_b200 import sampling
from yaoray_b200._lib import YrcError

GOLDEN = Path(__file__).resolve().parent / "golden"


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_device_sampler_matches_reference_golden(kind):
    f = dict(np.load(GOLDEN / "sampler.npz"))
    for seed in (0, 0x5EED1234):
        for spp in (1, 64):
            for d2 in (False, True):
                key = f"k{kind}_s{seed}_p{spp}_{'2d' if d2 else '1d'}"
                got = sampling.sampler_eval(kind, seed, spp, f["queries"], d2)
                assert np.array_equal(bits(got), bits(f[key])), key


@pytest.mark.gpu
def test_device_rng_and_pixel_seed_match_reference_golden():
    f = dict(np.load(GOLDEN / "sampler.npz"))
    got = sampling.rng_eval(f["rng_seeds"], 16)
    assert np.array_equal(bits(got), bits(f["rng_draws"]))
    seeds = sampling.pixel_seed_eval(0x1234, f["seed_pixel_queries"])
    assert np.array_equal(seeds, f["seed_pixel_values"])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_device_sampler_matches_oracle_random(kind):
    """Wider query ranges than the golden set: large pixels and sample
    indices, negative bounces, every dimension slot and lanes up to 64."""
    rng = np.random.default_rng(40 + kind)
    n = 20000
    q = np.stack([rng.integers(0, 4096, n), rng.integers(0, 4096, n), rng.integers(0, 1 << 16, n),
                  rng.integers(-2, 64, n), rng.integers(0, 16, n), rng.integers(0, 65, n)], 1).astype(np.int32)
    for seed in (7, 0xFFFFFFFFFFFFFFFF):
        for spp in (1, 3, 16, 1 << 16):
            for d2 in (False, True):
                a = sampling.sampler_eval(kind, seed, spp, q, d2)
                b = oracle.oracle_sampler(kind, seed, spp, q, d2)
                assert np.array_equal(bits(a), bits(b)), (seed, spp, d2)


@pytest.mark.gpu
def test_device_rng_and_pixel_seed_match_oracle_random():
    rng = np.random.default_rng(11)
    seeds = rng.integers(0, np.iinfo(np.uint64).max, 256, dtype=np.uint64, endpoint=True)
    got = sampling.rng_eval(seeds, 40)
    for s, row in zip(seeds, got):
        assert np.array_equal(bits(row), bits(oracle.oracle_rng(int(s), 40)))
    q = np.stack([rng.integers(-5, 8192, 512), rng.integers(-5, 8192, 512), rng.integers(0, 1 << 20, 512)], 1)
    vals = sampling.pixel_seed_eval(0xDEADBEEFCAFEF00D, q)
    for (x, y, s), v in zip(q, vals):
        assert oracle.oracle_seed_for_pixel_sample(0xDEADBEEFCAFEF00D, int(x), int(y), int(s)) == int(v)


def test_sampler_eval_rejects_bad_arguments():
    """Argument checks run before any CUDA call, so they need no device."""
    with pytest.raises(YrcError):
        sampling.sampler_eval(4, 0, 1, np.zeros((1, 6), np.int32), False)
    with pytest.raises(YrcError):
        sampling.sampler_eval(-1, 0, 1, np.zeros((1, 6), np.int32), True)
    assert sampling.sampler_eval(0, 0, 1, np.zeros((0, 6), np.int32), False).shape == (0,)
    assert sampling.rng_eval(np.zeros(0, np.uint64), 4).shape == (0, 4)
    assert sampling.pixel_seed_eval(0, np.zeros((0, 3), np.int64)).shape == (0,)
