"""The whole client-side setup of the XBOOT AES on the device: from the reference context's dense
secret and its bootstrapping sparse secret (the harness reads both out of the reference's
xboot14-sparse-1024 context), every switching key the bootstrapped AES uses is generated on the
device (wg_keygen_switch_key for the relinearisation, conjugation and all plan rotations;
wg_keygen_secret_switch for the dense-to-sparse and sparse-to-dense switches), the 1408 round-key
bits are encrypted on the device (wg_aes_xboot_encrypt_round_key_bits, the reference's
ckks_aes128_encrypt_expanded_round_key_bits with the first round key 4 levels up), and the XBOOT
AES-CTR then decrypts, under the reference's own decryption, to plain AES-128-CTR in every active
slot.  Only the linear-transform plans (and the EvalMod series) still come from the reference."""
import numpy as np
import pytest

from aes_util import encrypt_block, expand_key

pytestmark = pytest.mark.gpu


def test_device_generated_keys_and_key_bits_run_the_xboot_aes(wg, ref_mod):
    import torch

    R = ref_mod.RefPlans(bootstrap_keys=True, preset="xboot14-sparse")
    info = R.bts_info()
    N, K = R.N, len(R.p)
    s, sparse = R.secret_coeffs(), R.secret_coeffs(sparse=True)
    assert s is not None and sparse is not None
    ctx = wg.Context(N, R.q, R.p, R.dnum)
    ctx.keygen_switch_key(wg.WG_KEY_RELIN, 0, s, seed=101)
    ctx.keygen_switch_key(wg.WG_KEY_CONJ, 0, s, seed=102)
    for r in R.rotations():
        ctx.keygen_switch_key(wg.WG_KEY_ROTATION, int(r), s, seed=103)
    ctx.keygen_secret_switch(wg.WG_KEY_DENSE_TO_SPARSE, s, sparse, seed=104)
    ctx.keygen_secret_switch(wg.WG_KEY_SPARSE_TO_DENSE, sparse, s, seed=105)

    def stages(which):
        out = []
        for k in range(R.stages(which)):
            st = R.stage(which, k)
            out.append(wg.LtStage(ctx, st["qp_limbs"] - 1 - K, st["indices"], st["diagonals"], st["baby"],
                                  st["slot_count"], st["rescale"]))
        return out

    params = wg.BootstrapParams(info["s2c_depth"], info["depth"], info["evalmod_log_scale"], info["double_angle"],
                                info["active_slots"], info["slots"], info["scale"])
    s2c, c2s = stages(0), stages(1)
    rng = np.random.default_rng(211)
    ek = expand_key(bytes(rng.integers(0, 256, 16, dtype=np.uint8)))
    full = (info["depth"] + 1) * N
    key_bits = [(torch.zeros(full, dtype=torch.int64, device="cuda"),
                 torch.zeros(full, dtype=torch.int64, device="cuda")) for _ in range(1408)]
    kscales, klevels = ctx.aes_xboot_encrypt_round_key_bits(params, ek, 4, s, key_bits, seed=106)
    assert set(klevels[:128].tolist()) == {info["s2c_depth"] + 4} and set(klevels[128:].tolist()) == {info["s2c_depth"]}
    # a few key bits decrypt to their values under the reference's decryption
    for k in (0, 9, 700, 1407):
        m = (int(klevels[k]) + 1) * N
        z = R.decrypt(int(klevels[k]), float(kscales[k]), wg.to_host(key_bits[k][0])[:m], wg.to_host(key_bits[k][1])[:m])
        assert np.abs(z[:64].real - ((ek[k // 8] >> (k % 8)) & 1)).max() < 1e-3, k

    blocks = 40
    counters = bytes(rng.integers(0, 256, 16 * blocks, dtype=np.uint8))
    plain = bytes(rng.integers(0, 256, 16 * blocks, dtype=np.uint8))
    stream = b"".join(encrypt_block(ek, counters[16 * i:16 * i + 16]) for i in range(blocks))
    ciphertexts = bytes(x ^ y for x, y in zip(plain, stream))
    outs = [(torch.zeros(full, dtype=torch.int64, device="cuda"), torch.zeros(full, dtype=torch.int64, device="cuda"))
            for _ in range(128)]
    lv, sc = ctx.aes_ctr_xboot(params, s2c, c2s, info["coeffs"], key_bits, kscales, klevels, counters, ciphertexts,
                               blocks, outs)
    torch.cuda.synchronize()
    max_err, mismatched = 0.0, 0
    for bit in range(128):
        m = (lv[bit] + 1) * N
        z = R.decrypt(lv[bit], sc[bit], wg.to_host(outs[bit][0])[:m], wg.to_host(outs[bit][1])[:m])
        want = np.array([(plain[16 * b + bit // 8] >> (bit % 8)) & 1 for b in range(blocks)], dtype=np.float64)
        max_err = max(max_err, float(np.abs(z[:blocks].real - want).max()))
        mismatched += int((np.round(z[:blocks].real) != want).sum())
    print(f"device-generated setup: max error {max_err:.3e}")
    assert mismatched == 0 and max_err < 0.5


def test_device_encrypted_walsh_key_bits_decrypt_to_the_key(wg, ref_mod):
    """The Walsh AES's round-key bits encrypted on the device (wg_aes_walsh_encrypt_round_key_bits,
    the reference's ckks_aes128_encrypt_expanded_round_key_bits_walsh_complex_blocks,
    ckks_aes_ctr_walsh_sbox.cpp:981-1035) under the reference walsh15 context's secret: level S2C
    depth + 1, scale the parameter scale for rounds 0 and 10 and a quarter of it otherwise
    (:1010-1014), and each sampled bit decrypts, under the reference's decryption, to (v, v) in the
    first 512 slots and 0 elsewhere."""
    import json
    import os

    import torch

    plan = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "walsh15_plan.json")))
    R = ref_mod.RefPlans()
    assert [int(x) for x in R.q] == plan["q"]
    N = R.N
    s = R.secret_coeffs()
    b = plan["bootstrap"]
    params = wg.BootstrapParams(b["s2c_depth"], b["depth"], b["evalmod_log_scale"], b["double_angle"],
                                b["active_slots"], b["slots"], b["scale"])
    ctx = wg.Context(N, R.q, R.p, R.dnum)
    rng = np.random.default_rng(223)
    ek = expand_key(bytes(rng.integers(0, 256, 16, dtype=np.uint8)))
    level = b["s2c_depth"] + 1
    outs = [(torch.zeros((level + 1) * N, dtype=torch.int64, device="cuda"),
             torch.zeros((level + 1) * N, dtype=torch.int64, device="cuda")) for _ in range(1408)]
    sc, lv = ctx.aes_walsh_encrypt_round_key_bits(params, ek, 512, s, outs, seed=9)
    torch.cuda.synchronize()
    assert set(lv.tolist()) == {level}
    for k in range(1408):
        want = b["scale"] if (k < 128 or k >= 1280) else b["scale"] / 4.0
        assert sc[k] == want, k
    m = (level + 1) * N
    for k in (0, 5, 200, 700, 1279, 1300, 1407):
        v = (ek[k // 8] >> (k % 8)) & 1
        z = R.decrypt(level, float(sc[k]), wg.to_host(outs[k][0])[:m], wg.to_host(outs[k][1])[:m])
        assert np.abs(z[:512].real - v).max() < 1e-3 and np.abs(z[:512].imag - v).max() < 1e-3, k
        assert np.abs(z[512:]).max() < 1e-3, k
