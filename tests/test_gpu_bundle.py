"""Keys and plans saved to a bundle file and loaded into a fresh context (wg_bundle_save /
wg_bundle_load) on the walsh15 chain: the fresh context rotates, relinearises and applies the
loaded linear-transform stage to the same residues as the original; a file for other
parameters is rejected."""
import numpy as np
import pytest

from params import WALSH15

pytestmark = pytest.mark.gpu


def test_bundle_round_trip_gives_the_same_results(wg, ref_mod, tmp_path):
    import torch

    R = ref_mod.RefCtx(1 << WALSH15["logN"], WALSH15["q_bits"], WALSH15["p_bits"], WALSH15["dnum"],
                       h=WALSH15["h"], rotations=[1, 4])
    N, K = R.N, len(R.p)
    a = wg.Context(N, R.q, R.p, R.dnum)
    for r in (1, 4):
        key, parts, kl = R.key(0, r)
        a.set_key(wg.WG_KEY_ROTATION, key, rotation=r, parts=parts, key_level=kl)
    key, parts, kl = R.key(2)
    a.set_key(wg.WG_KEY_RELIN, key, parts=parts, key_level=kl)
    level = 6
    rng = np.random.default_rng(41)
    mods = np.concatenate([R.q[: level + 1], R.p]).astype(np.uint64)
    idx = [0, 1, 4, 5]
    diags = (rng.integers(0, 1 << 62, (len(idx), mods.size, N), dtype=np.uint64) % mods[None, :, None]).astype(np.uint64)
    st = wg.LtStage(a, level, idx, diags, 4, 0, True)
    path = tmp_path / "walsh15.wgb"
    a.bundle_save(path, [st])

    b = wg.Context(N, R.q, R.p, R.dnum)
    loaded = b.bundle_load(path)
    assert len(loaded) == 1
    n = (level + 1) * N
    qc = np.repeat(R.q[: level + 1], N)
    draw = lambda: (rng.integers(0, 1 << 62, n, dtype=np.uint64) % qc).astype(np.uint64)
    x0, x1, x2 = draw(), draw(), draw()
    outs = []
    for ctx, stage in ((a, st), (b, loaded[0])):
        rb, ra = wg.to_device(x0), wg.to_device(x1)
        ctx.rotate(level, rb, ra, 4)
        c0, c1, c2 = wg.to_device(x0), wg.to_device(x1), wg.to_device(x2)
        ctx.relin(level, c0, c1, c2)
        lb, la = wg.to_device(x0), wg.to_device(x1)
        stage.apply([lb], [la])
        torch.cuda.synchronize()
        outs.append([wg.to_host(t) for t in (rb, ra, c0, c1, lb[: level * N], la[: level * N])])
    for k, (u, v) in enumerate(zip(outs[0], outs[1])):
        assert (u == v).all(), k

    other = wg.Context(N, R.q[:-1], R.p, R.dnum)
    with pytest.raises(wg.WalshGpuError):
        other.bundle_load(path)
