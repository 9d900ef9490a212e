"""Hoisted rotations on the device (wg_rotate_many) against the reference's hoisted evaluator.

The reference's ckks_hoist_ciphertext_a_qp_eval + ckks_hybrid_key_switch_hoisted_inplace
(ckks_keyswitch.cpp:344-373, 1072-1328) decompose `a` once and reuse the decomposition for
every rotation; the device entry point does the same.  Rotations by a multiple of the slot
count return the input unchanged.
"""
import numpy as np
import pytest

from params import WALSH15

pytestmark = pytest.mark.gpu

ROTS = [1, 8, 512, -512, 16383]


@pytest.fixture(scope="module")
def setup(wg, ref_mod):
    R = ref_mod.RefCtx(1 << WALSH15["logN"], WALSH15["q_bits"], WALSH15["p_bits"], WALSH15["dnum"],
                       rotations=ROTS)
    ctx = wg.Context(R.N, R.q, R.p, R.dnum)
    for r in ROTS:
        key, parts, kl = R.key(0, r)
        ctx.set_key(wg.WG_KEY_ROTATION, key, rotation=r, parts=parts, key_level=kl)
    return R, ctx


@pytest.mark.parametrize("level", [12, 6, 1, 0])
def test_rotate_many_matches_reference_hoisted(wg, setup, level):
    import torch

    R, ctx = setup
    N = R.N
    n = (level + 1) * N
    rng = np.random.default_rng(level)
    qcol = np.repeat(R.q[: level + 1], N)
    b = (rng.integers(0, 1 << 62, n, dtype=np.uint64) % qcol).astype(np.uint64)
    a = (rng.integers(0, 1 << 62, n, dtype=np.uint64) % qcol).astype(np.uint64)
    expect = R.hoisted_rotations(level, b, a, ROTS)
    rots = ROTS + [0, N // 2, -N]  # identity rotations mixed in
    out = torch.empty(len(rots) * 2 * n, dtype=torch.int64, device="cuda")
    ctx.rotate_many(level, wg.to_device(b), wg.to_device(a), rots, out)
    got = wg.to_host(out).reshape(len(rots), 2, n)
    for j, r in enumerate(ROTS):
        assert (got[j, 0] == expect[j, 0]).all(), (level, r, int((got[j, 0] != expect[j, 0]).sum()))
        assert (got[j, 1] == expect[j, 1]).all(), (level, r, int((got[j, 1] != expect[j, 1]).sum()))
    for j in range(len(ROTS), len(rots)):
        assert (got[j, 0] == b).all() and (got[j, 1] == a).all()


def test_rotate_many_missing_key_is_runtime_error(wg, setup):
    import torch

    R, ctx = setup
    n = R.N
    b = torch.zeros(n, dtype=torch.int64, device="cuda")
    out = torch.empty(4 * n, dtype=torch.int64, device="cuda")
    with pytest.raises(wg.WalshGpuError) as e:
        ctx.rotate_many(0, b, b.clone(), [1, 2], out)
    assert e.value.code == -2
