"""The XBOOT AES S-box on the device (wg_xboot_sbox) against the reference's
ckks_aes_xboot_sbox_impl (ckks_aes_ctr.cpp:280-336, restated by the harness on the reference's
own multiply / relinearize / rescale / integer operations) on the reference's XBOOT chain at
N = 2^15 (17 Q limbs, 5 P limbs, dnum 5) with its relinearisation key: for two S-box instances at
level 5, all 8 output bits must match residue for residue, with the same level and scale."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_xboot_sbox_matches_reference(wg, ref_mod):
    import torch

    R = ref_mod.RefXboot()
    N = R.N
    ctx = wg.Context(N, R.q, R.p, R.dnum)
    key, parts, kl = R.key(2)
    ctx.set_key(wg.WG_KEY_RELIN, key, parts=parts, key_level=kl)
    level, scale, count = 5, 2.0 ** 37, 2
    rng = np.random.default_rng(41)
    qc = np.repeat(R.q[: level + 1], N)
    draw = lambda: (rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)
    host = [[(draw(), draw()) for _ in range(8)] for _ in range(count)]
    bits = [[(wg.to_device(b), wg.to_device(a)) for b, a in inst] for inst in host]
    mk = lambda: torch.zeros((level + 1) * N, dtype=torch.int64, device="cuda")
    outs = [[(mk(), mk()) for _ in range(8)] for _ in range(count)]
    lv, sc = ctx.xboot_sbox(level, scale, bits, outs)
    torch.cuda.synchronize()
    for i in range(count):
        want = R.sbox(level, scale, host[i])
        for k in range(8):
            rb, ra, rl, rs = want[k]
            assert (lv[k], sc[k]) == (rl, rs), (i, k)
            n = (rl + 1) * N
            gb, ga = wg.to_host(outs[i][k][0])[:n], wg.to_host(outs[i][k][1])[:n]
            assert (gb == rb).all(), (i, k, "b", int((gb != rb).sum()))
            assert (ga == ra).all(), (i, k, "a", int((ga != ra).sum()))
