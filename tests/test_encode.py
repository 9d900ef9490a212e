"""Host CKKS slot encoding (wg_encode_slots) against the reference encoder, coefficient for
coefficient: random complex slots, AES-style bit patterns and active-slot masks, at the scales
the AES circuit uses (the parameter scale, a quarter of it, a modulus, 1).  No GPU needed."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def plans(ref_mod):
    return ref_mod.RefPlans()


def _cases(N, rng):
    half = N // 2
    yield rng.uniform(-1, 1, half), rng.uniform(-1, 1, half)
    bits = rng.integers(0, 2, (2, half)).astype(np.float64)
    bits[:, 512:] = 0.0
    yield bits[0], bits[1]
    mask = np.zeros(half)
    mask[:512] = 1.0
    yield mask, np.zeros(half)
    yield np.full(half, 0.5), np.full(half, 0.5)


def test_encoder_matches_reference(wg, plans):
    N = plans.N
    rng = np.random.default_rng(4)
    q = plans.q
    scales = [plans.scale, plans.scale / 4.0, float(q[2]), float(q[12]), 1.0, 2.0 ** 45 + 12345.0]
    for re, im in _cases(N, rng):
        for sc in scales:
            level = 2
            want = plans.encode(re, im, sc, level)
            got = wg.encode_slots(N, re, im, sc, q[: level + 1])
            assert (got == want).all(), (sc, int((got != want).sum()))
