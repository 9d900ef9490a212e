"""The mask-packed Walsh AES S-box on the device against the reference's
ckks_walsh_sbox_complex_blocks_mask_packed on its walsh15 bootstrapping context (its plans,
keys, segment rotation keys +-512 k and the EvalMod series it reports), for a batch of two S-box
instances of 8 lazy-bit ciphertexts each: all 8 output bits of every instance must match the
reference residue for residue, with the same level and scale."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bts(ref_mod):
    return ref_mod.RefPlans(bootstrap_keys=True)


def _setup(wg, bts):
    N, K = bts.N, len(bts.p)
    ctx = wg.Context(N, bts.q, bts.p, bts.dnum)
    for kind, wkind in ((2, wg.WG_KEY_RELIN), (1, wg.WG_KEY_CONJ), (4, wg.WG_KEY_SPARSE_TO_DENSE)):
        key, parts, kl = bts.key(0, kind=kind)
        ctx.set_key(wkind, key, parts=parts, key_level=kl)
    ctx.set_key(wg.WG_KEY_DENSE_TO_SPARSE, bts.key(0, kind=3)[0])
    for r in bts.rotations():
        key, parts, kl = bts.key(int(r))
        ctx.set_key(wg.WG_KEY_ROTATION, key, rotation=int(r), parts=parts, key_level=kl)
    stages = []
    for which in (0, 1):
        lst = []
        for k in range(bts.stages(which)):
            st = bts.stage(which, k)
            lst.append(wg.LtStage(ctx, st["qp_limbs"] - 1 - K, st["indices"], st["diagonals"], st["baby"],
                                  st["slot_count"], st["rescale"]))
        stages.append(lst)
    return ctx, stages


def test_walsh_sbox_matches_reference(wg, bts):
    import torch

    info = bts.bts_info()
    N = bts.N
    ctx, stages = _setup(wg, bts)
    params = wg.BootstrapParams(info["s2c_depth"], info["depth"], info["evalmod_log_scale"], info["double_angle"],
                                info["active_slots"], info["slots"], info["scale"])
    level = info["s2c_depth"]
    full = (info["depth"] + 1) * N
    rng = np.random.default_rng(21)
    qc = np.repeat(bts.q[: level + 1], N)
    count = 2
    host = [[((rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64),
              (rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)) for _ in range(8)]
            for _ in range(count)]
    bits = [[(wg.to_device(b), wg.to_device(a)) for b, a in inst] for inst in host]
    mk = lambda: torch.zeros(full, dtype=torch.int64, device="cuda")
    outs = [[(mk(), mk()) for _ in range(8)] for _ in range(count)]
    lv, sc = ctx.walsh_sbox(params, stages[0], stages[1], info["coeffs"], 512, level, info["scale"], bits, outs)
    torch.cuda.synchronize()
    for i in range(count):
        want = bts.walsh_sbox(512, level, info["scale"], host[i])
        for k in range(8):
            rb, ra, rl, rs = want[k]
            assert (lv[k], sc[k]) == (rl, rs), (i, k)
            n = (rl + 1) * N
            gb, ga = wg.to_host(outs[i][k][0])[:n], wg.to_host(outs[i][k][1])[:n]
            assert (gb == rb).all(), (i, k, "b", int((gb != rb).sum()))
            assert (ga == ra).all(), (i, k, "a", int((ga != ra).sum()))
