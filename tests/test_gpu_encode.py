"""CKKS slot encoding on the device (wg_encode_slots_device) against the reference's ckks_encode
(src/ckks/encoding/ckks_encoding.cpp:332-414) on the walsh15 chain: residue for residue, for
several plaintexts per call, on random complex slot vectors, on AES-style 0/1 bit planes at the
parameter scale, on a constant and on large values at a small scale; and the evaluation-form
output is the NTT of the coefficient-form one.  Decryption and decoding on the device
(wg_decrypt_decode) against the reference's ckks_decrypt, to FP64 rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_encoder_matches_reference(wg, ref_mod):
    import torch

    R = ref_mod.RefPlans()
    N, half = R.N, R.N // 2
    ctx = wg.Context(N, R.q, R.p, R.dnum)
    rng = np.random.default_rng(29)
    level = 3
    limbs = level + 1
    cases = [
        (2.0 ** 35, [(rng.uniform(-1, 1, half), rng.uniform(-1, 1, half)) for _ in range(3)]),
        (2.0 ** 37, [(rng.integers(0, 2, half).astype(np.float64), rng.integers(0, 2, half).astype(np.float64)),
                     (rng.integers(0, 2, half).astype(np.float64), np.zeros(half))]),
        (float(R.q[level]), [(np.full(half, 1.0), np.zeros(half))]),
        (2.0 ** 20, [(rng.uniform(-1e6, 1e6, half), rng.uniform(-1e6, 1e6, half))]),
    ]
    for scale, vecs in cases:
        re = np.stack([v[0] for v in vecs])
        im = np.stack([v[1] for v in vecs])
        outs = [torch.zeros(limbs * N, dtype=torch.int64, device="cuda") for _ in vecs]
        ctx.encode_slots_device(limbs, scale, re, im, outs)
        evals = [torch.zeros(limbs * N, dtype=torch.int64, device="cuda") for _ in vecs]
        ctx.encode_slots_device(limbs, scale, re, im, evals, eval_form=True)
        torch.cuda.synchronize()
        for k, (vr, vi) in enumerate(vecs):
            want = R.encode(vr, vi, scale, level)
            got = wg.to_host(outs[k])
            assert (got == want).all(), (scale, k, int((got != want).sum()))
            host = wg.encode_slots(N, vr, vi, scale, R.q[:limbs])
            assert (host.reshape(-1) == want).all()
            # evaluation form = forward NTT of the coefficients, limb by limb
            coeff = outs[k].clone()
            ctx.ntt_forward(coeff, limbs)
            torch.cuda.synchronize()
            assert (wg.to_host(evals[k]) == wg.to_host(coeff)).all(), (scale, k)


def test_device_decrypt_decode_matches_reference(wg, ref_mod):
    import torch

    R = ref_mod.RefPlans()
    N, half = R.N, R.N // 2
    s = R.secret_coeffs()
    ctx = wg.Context(N, R.q, R.p, R.dnum)
    rng = np.random.default_rng(31)
    for level, scale in ((3, 2.0 ** 35), (0, 2.0 ** 30)):
        n = (level + 1) * N
        vecs = [(rng.uniform(-1, 1, half), rng.uniform(-1, 1, half)) for _ in range(3)]
        pts = [torch.zeros(n, dtype=torch.int64, device="cuda") for _ in vecs]
        ctx.encode_slots_device(level + 1, scale, np.stack([v[0] for v in vecs]), np.stack([v[1] for v in vecs]),
                                pts, eval_form=True)
        cts = [(torch.zeros(n, dtype=torch.int64, device="cuda"), torch.zeros(n, dtype=torch.int64, device="cuda"))
               for _ in vecs]
        ctx.encrypt_symmetric(level, pts, s, cts, seed=5 + level)
        torch.cuda.synchronize()
        got = ctx.decrypt_decode(level, [scale] * len(vecs), cts, s)
        for k, (vr, vi) in enumerate(vecs):
            want = R.decrypt(level, scale, wg.to_host(cts[k][0]), wg.to_host(cts[k][1]))
            assert np.abs(got[k] - want).max() < 1e-9, (level, k, float(np.abs(got[k] - want).max()))
            assert np.abs(got[k] - (vr + 1j * vi)).max() < 1e-5, (level, k)
