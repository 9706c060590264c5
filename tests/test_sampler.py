"""Monte Carlo ensembles (gpop_sample_states): the Philox4x32-10 restatement against the published
known-answer vectors (CPU), and the device samples against it, their statistics, reproducibility,
and an ensemble fed to the propagation (GPU)."""
import numpy as np
import pytest

import philox_ref as P


def test_philox_known_answers():
    # Random123 known-answer vectors for philox4x32, 10 rounds
    kat = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, out in kat:
        assert P.philox4x32_10(ctr, key) == out


def _sample(ctx, n, seed, sr=10.0, sv=0.1):
    from gpu_util import host, zeros
    r = zeros(n, 3)
    v = zeros(n, 3)
    rn = np.array([7.0e6, 1.0e5, -2.0e5])
    vn = np.array([10.0, 7.5e3, 5.0])
    ctx.sample_states(rn, vn, sr, sv, seed, r, v)
    import torch
    torch.cuda.synchronize()
    return host(r), host(v), rn, vn


@pytest.fixture(scope="module")
def ctx():
    import opengpop_b200 as G
    c = G.Context()
    yield c
    c.close()


@pytest.mark.gpu
def test_samples_match_the_restatement(ctx):
    seed = 0x1234_5678_9ABC
    r, v, rn, vn = _sample(ctx, 4096, seed)
    for i in (0, 1, 17, 4095):
        z = P.normals(i, seed)
        # the sample is nominal + sigma z: compare it where it is formed (a few ulps of r, v)
        assert np.allclose(r[i], rn + 10.0 * z[:3], rtol=4e-16, atol=0)
        assert np.allclose(v[i], vn + 0.1 * z[3:], rtol=4e-16, atol=1e-13)


@pytest.mark.gpu
def test_sample_statistics_and_reproducibility(ctx):
    n = 1 << 18
    r, v, rn, vn = _sample(ctx, n, 7)
    z = np.concatenate([(r - rn) / 10.0, (v - vn) / 0.1], axis=1)
    assert np.abs(z.mean(axis=0)).max() < 5.0 / np.sqrt(n)
    assert np.abs(z.std(axis=0) - 1.0).max() < 5.0 / np.sqrt(2 * n)
    c = np.corrcoef(z.T)
    assert np.abs(c - np.eye(6)).max() < 5.0 / np.sqrt(n)
    r2, v2, _, _ = _sample(ctx, n, 7)
    r3, _, _, _ = _sample(ctx, n, 8)
    assert np.array_equal(r, r2) and np.array_equal(v, v2) and not np.array_equal(r, r3)


@pytest.mark.gpu
def test_ensemble_feeds_the_propagation(ctx):
    from gpu_util import dev, host
    import torch
    n = 2048
    r = torch.zeros(n, 3, dtype=torch.float64, device="cuda")
    v = torch.zeros_like(r)
    rn, vn = np.array([7.0e6, 0.0, 0.0]), np.array([0.0, 7.546e3, 0.0])
    ctx.sample_states(rn, vn, 0.0, 1.0, 99, r, v)  # velocity perturbations only, as the reference
    r0 = host(r)
    assert np.array_equal(r0, np.tile(rn, (n, 1)))
    ctx.propagate_device((2024, 1, 1, 0, 0, 0.0), 30.0, 120, r, v)
    spread = np.linalg.norm(host(r) - host(r).mean(axis=0), axis=1)
    assert np.all(np.isfinite(spread)) and 100.0 < np.median(spread) < 5.0e4
