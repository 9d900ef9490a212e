"""The XBOOT AES path on the device, on the reference's XBOOT parameter sets (AESXBoot15Config,
AESXBoot14SecureConfig and their 1024-active-slot variants, bootstrapping keys from the
reference):

* the pair bootstrap (wg_bootstrap_pair) against the reference's
  ckks_batch_bootstrap_evalmod_inplace (ckks_bootstrap_evalmod_inplace.cpp:393-414): two
  pairs in one call, both results residue for residue, same level and scale;
* AES-128-CTR with the XBOOT S-box (wg_aes_ctr_xboot, the reference's ckks_aes_ctr,
  ckks_aes_ctr.cpp:757-779) with the reference's encrypted round-key bits
  (ckks_aes128_encrypt_expanded_round_key_bits, first round key 4 levels up as its benchmark
  does): every output bit decrypts, in every active block slot, to the plaintext of plain
  AES-128-CTR with error below 0.5 (the reference benchmark's acceptance rule,
  bench/aes_bench.cpp:305-307);
* the circuit's own steps against the reference's, restated by the harness on the reference's
  public operations because the originals are file-internal: the initial public XOR of the
  counter bit planes (make_batched_initial_counter_state, ckks_aes_ctr.cpp:576-683; all-zero,
  all-one and varying planes) and one round's ShiftRows + MixColumns + AddRoundKey
  (ckks_aes_ctr.cpp:460-554), residue for residue with the same levels and scale labels;
* the serving path over XBOOT evaluations (wg_serve_create_xboot): three odd-sized requests
  queued within the batching window share one evaluation, each decrypting to its own plaintext.

The EvalMod polynomial is the one the reference context reports: the reference's own MPFR fit
(src/math/poly_approx.cpp:565)."""
import time

import numpy as np
import pytest

from aes_util import encrypt_block, expand_key

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["xboot15", "xboot15-sparse", "xboot14", "xboot14-sparse"])
def xb(request, wg, ref_mod):
    R = ref_mod.RefPlans(bootstrap_keys=True, preset=request.param)
    info = R.bts_info()
    N, K = R.N, len(R.p)
    ctx = wg.Context(N, R.q, R.p, R.dnum)
    for kind, wkind in ((2, wg.WG_KEY_RELIN), (1, wg.WG_KEY_CONJ), (4, wg.WG_KEY_SPARSE_TO_DENSE)):
        k, parts, lv = R.key(0, kind=kind)
        ctx.set_key(wkind, k, parts=parts, key_level=lv)
    ctx.set_key(wg.WG_KEY_DENSE_TO_SPARSE, R.key(0, kind=3)[0])
    for r in R.rotations():
        k, parts, lv = R.key(int(r))
        ctx.set_key(wg.WG_KEY_ROTATION, k, rotation=int(r), parts=parts, key_level=lv)

    def stages(which):
        out = []
        for k in range(R.stages(which)):
            st = R.stage(which, k)
            out.append(wg.LtStage(ctx, st["qp_limbs"] - 1 - K, st["indices"], st["diagonals"], st["baby"],
                                  st["slot_count"], st["rescale"]))
        return out

    params = wg.BootstrapParams(info["s2c_depth"], info["depth"], info["evalmod_log_scale"], info["double_angle"],
                                info["active_slots"], info["slots"], info["scale"])
    yield R, ctx, params, stages(0), stages(1), info
    del ctx


def test_pair_bootstrap_matches_reference(wg, xb):
    import torch

    R, ctx, params, s2c, c2s, info = xb
    N, lv, full = R.N, info["s2c_depth"], info["depth"] + 1
    rng = np.random.default_rng(83)
    qc = np.repeat(R.q[: lv + 1], N)
    draw = lambda: (rng.integers(0, 1 << 62, (lv + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)
    host = [((draw(), draw()), (draw(), draw())) for _ in range(2)]

    def dev(x):
        t = torch.zeros(full * N, dtype=torch.int64, device="cuda")
        t[: x.size] = wg.to_device(x)
        return t

    pairs = [((dev(c0[0]), dev(c0[1])), (dev(c1[0]), dev(c1[1]))) for c0, c1 in host]
    lvl, sc = ctx.bootstrap_pair(params, s2c, c2s, info["coeffs"], info["scale"], pairs)
    torch.cuda.synchronize()
    for i, (c0, c1) in enumerate(host):
        r0, r1, rl, rs = R.bootstrap_pair(lv, info["scale"], info["scale"], c0, c1)
        assert (lvl, sc) == (rl, rs), i
        n = (rl + 1) * N
        for which, (rb, ra) in enumerate((r0, r1)):
            gb, ga = wg.to_host(pairs[i][which][0])[:n], wg.to_host(pairs[i][which][1])[:n]
            assert (gb == rb).all(), (i, which, "b", int((gb != rb).sum()))
            assert (ga == ra).all(), (i, which, "a", int((ga != ra).sum()))


def test_xboot_aes_ctr_decrypts_to_plain_aes(wg, xb):
    import torch

    R, ctx, params, s2c, c2s, info = xb
    N, full = R.N, info["depth"] + 1
    rng = np.random.default_rng(91)
    ek = expand_key(bytes(rng.integers(0, 256, 16, dtype=np.uint8)))
    blocks = 40
    counters = bytes(rng.integers(0, 256, 16 * blocks, dtype=np.uint8))
    plain = bytes(rng.integers(0, 256, 16 * blocks, dtype=np.uint8))
    stream = b"".join(encrypt_block(ek, counters[16 * i:16 * i + 16]) for i in range(blocks))
    ciphertexts = bytes(x ^ y for x, y in zip(plain, stream))

    kbits, kscales, klevels = R.xboot_key_bits(ek, 4)
    key_bits = [(wg.to_device(b), wg.to_device(a)) for b, a in kbits]
    outs = [(torch.zeros(full * N, dtype=torch.int64, device="cuda"),
             torch.zeros(full * N, dtype=torch.int64, device="cuda")) for _ in range(128)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lv, sc = ctx.aes_ctr_xboot(params, s2c, c2s, info["coeffs"], key_bits, kscales, klevels, counters, ciphertexts,
                               blocks, outs)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    max_err, mismatched = 0.0, 0
    for bit in range(128):
        m = (lv[bit] + 1) * N
        z = R.decrypt(lv[bit], sc[bit], wg.to_host(outs[bit][0])[:m], wg.to_host(outs[bit][1])[:m])
        want = np.array([(plain[16 * b + bit // 8] >> (bit % 8)) & 1 for b in range(blocks)], dtype=np.float64)
        got = z[:blocks].real
        max_err = max(max_err, float(np.abs(got - want).max()))
        mismatched += int((np.round(got) != want).sum())
    print(f"{R.preset}: {blocks} blocks in {seconds:.2f} s on the device; max error {max_err:.3e}")
    assert mismatched == 0
    assert max_err < 0.5


def test_xboot_served_requests_share_an_evaluation(wg, xb):
    import torch

    R, ctx, params, s2c, c2s, info = xb
    N, full = R.N, info["depth"] + 1
    rng = np.random.default_rng(97)
    ek = expand_key(bytes(rng.integers(0, 256, 16, dtype=np.uint8)))
    kbits, kscales, klevels = R.xboot_key_bits(ek, 4)
    key_bits = [(wg.to_device(b), wg.to_device(a)) for b, a in kbits]
    srv = wg.Server.xboot(ctx, params, s2c, c2s, info["coeffs"], key_bits, kscales, klevels, workers=1,
                          batch_window_ms=300.0)
    try:
        reqs = []
        for blocks in (3, 17, 5):
            counters = bytes(rng.integers(0, 256, 16 * blocks, dtype=np.uint8))
            plain = bytes(rng.integers(0, 256, 16 * blocks, dtype=np.uint8))
            stream = b"".join(encrypt_block(ek, counters[16 * i:16 * i + 16]) for i in range(blocks))
            cts = bytes(x ^ y for x, y in zip(plain, stream))
            outs = [(torch.zeros(full * N, dtype=torch.int64, device="cuda"),
                     torch.zeros(full * N, dtype=torch.int64, device="cuda")) for _ in range(128)]
            reqs.append((blocks, plain, outs, srv.submit(counters, cts, outs)))
        offsets = []
        for blocks, plain, outs, rid in reqs:
            res = srv.wait(rid, 600)
            assert res["batch_requests"] == 3 and res["active_blocks"] == info["active_slots"]
            offsets.append(res["block_offset"])
            off = res["block_offset"]
            for bit in range(128):
                m = (res["levels"][bit] + 1) * N
                z = R.decrypt(res["levels"][bit], res["scales"][bit], wg.to_host(outs[bit][0])[:m],
                              wg.to_host(outs[bit][1])[:m])
                want = [(plain[16 * b + bit // 8] >> (bit % 8)) & 1 for b in range(blocks)]
                assert (np.round(z[off:off + blocks].real) == want).all(), (blocks, bit)
        assert offsets == [0, 3, 20]
    finally:
        srv.close()


def test_xboot_initial_state_matches_reference(wg, xb):
    import torch

    R, ctx, params, s2c, c2s, info = xb
    N = R.N
    rng = np.random.default_rng(101)
    ek = expand_key(bytes(rng.integers(0, 256, 16, dtype=np.uint8)))
    kbits, kscales, klevels = R.xboot_key_bits(ek, 4)
    # every slot filled on the sparse sets, so constant planes are all-zero or all-one there
    blocks = info["active_slots"] if info["active_slots"] <= 1024 else 40
    raw = rng.integers(0, 256, (blocks, 16), dtype=np.uint8)
    raw[:, 0] = 0x00
    raw[:, 1] = 0xFF
    raw[:, 2] = 0x0F
    counters = raw.tobytes()
    L = int(klevels[0])
    key_bits = [(wg.to_device(b), wg.to_device(a)) for b, a in kbits[:128]]
    outs = [(torch.zeros((L + 1) * N, dtype=torch.int64, device="cuda"),
             torch.zeros((L + 1) * N, dtype=torch.int64, device="cuda")) for _ in range(128)]
    lvl, sc = ctx.xboot_initial_state(params, key_bits, kscales[:128], klevels[:128], counters, blocks, outs)
    torch.cuda.synchronize()
    want, rl, rs = R.xboot_initial_state(kbits[:128], kscales[:128], L, counters, blocks)
    assert lvl == rl == L - 1
    n = (rl + 1) * N
    for k in range(128):
        assert sc[k] == rs[k], k
        assert (wg.to_host(outs[k][0])[:n] == want[k][0]).all(), (k, "b")
        assert (wg.to_host(outs[k][1])[:n] == want[k][1]).all(), (k, "a")


@pytest.mark.parametrize("mix", [True, False])
def test_xboot_linear_layer_matches_reference(wg, xb, mix):
    import torch

    R, ctx, params, s2c, c2s, info = xb
    N, level = R.N, info["s2c_depth"]
    rng = np.random.default_rng(103 + int(mix))
    qc = np.repeat(R.q[: level + 1], N)
    draw = lambda: (rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)
    state = [(draw(), draw()) for _ in range(128)]
    # distinct scale labels per input byte, to follow which operand's label each sum keeps
    scales = [info["scale"] * (1.0 + ((k // 8) % 3)) for k in range(128)]
    ek = expand_key(bytes(rng.integers(0, 256, 16, dtype=np.uint8)))
    kbits, kscales, klevels = R.xboot_key_bits(ek, 4)
    keys = kbits[128:256]
    kl = int(klevels[128])
    dev = lambda x: wg.to_device(x)
    ins = [(dev(b), dev(a)) for b, a in state]
    key_dev = [(dev(b), dev(a)) for b, a in keys]
    outs = [(torch.zeros((level + 1) * N, dtype=torch.int64, device="cuda"),
             torch.zeros((level + 1) * N, dtype=torch.int64, device="cuda")) for _ in range(128)]
    sc = ctx.xboot_linear_layer(level, scales, ins, key_dev, klevels[128:256], mix, outs)
    torch.cuda.synchronize()
    want, rs = R.xboot_linear(state, scales, level, keys, kl, mix)
    n = (level + 1) * N
    for k in range(128):
        assert sc[k] == rs[k], k
        assert (wg.to_host(outs[k][0])[:n] == want[k][0]).all(), (k, "b")
        assert (wg.to_host(outs[k][1])[:n] == want[k][1]).all(), (k, "a")
