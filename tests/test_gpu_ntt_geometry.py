"""NTT geometries and their autotuner on the device, through the C ABI.

The context times four geometries of each transform phase when it is created (8 or 16
residues per thread, twiddle pairs staged in shared memory or read from the table) and keeps
the fastest per direction and phase.  Every geometry must give the oracle's words: each is
pinned in turn for both phases of both directions and checked on the walsh15 chain (N = 2^15,
13 Q + 4 P limbs: lazy 36..50-bit moduli and fully reduced 61-bit ones), on config 1
(N = 2^14, 16 limbs) and on a small ring (N = 2^10, whose whole limb is one tile).
"""
import numpy as np
import pytest

from params import CONFIG1, WALSH15

pytestmark = pytest.mark.gpu

SMALL_RING = {"logN": 10, "q_bits": [40, 50, 60], "p_bits": [61], "dnum": 1}


def _setup(wg, O, prm):
    N = 1 << prm["logN"]
    p, q = O.find_primes(prm["p_bits"], prm["q_bits"], N)
    return N, O.OracleCtx(N, q, p, prm["dnum"]), wg.Context(N, q, p, prm["dnum"])


@pytest.mark.parametrize("prm", [WALSH15, CONFIG1, SMALL_RING], ids=["walsh15", "config1", "n1024"])
def test_every_geometry_matches_the_oracle(wg, oracle_mod, prm):
    import torch

    N, o, ctx = _setup(wg, oracle_mod, prm)
    L, K = o.nq, len(o.p)
    x = o.uniform(L, 31)
    rng = np.random.default_rng(7)
    pp = np.concatenate([rng.integers(0, int(m), N, dtype=np.uint64) for m in o.p])
    want_q, want_p = o.ntt(x), o.ntt(pp, which=1)
    for geometry in range(4):
        for d in range(2):
            for ph in range(2):
                ctx.set_ntt_geometry(d, ph, geometry)
        dq, dp = wg.to_device(x), wg.to_device(pp)
        ctx.ntt_forward(dq, L)
        ctx.ntt_forward(dp, K, basis=1)
        torch.cuda.synchronize()
        assert (wg.to_host(dq) == want_q).all(), geometry
        assert (wg.to_host(dp) == want_p).all(), geometry
        ctx.ntt_inverse(dq, L)
        ctx.ntt_inverse(dp, K, basis=1)
        torch.cuda.synchronize()
        assert (wg.to_host(dq) == x).all(), geometry
        assert (wg.to_host(dp) == pp).all(), geometry
    # mixed choices per phase (forward rows 16-residue from the table, columns 8-residue staged)
    ctx.set_ntt_geometry(0, 0, 3)
    ctx.set_ntt_geometry(0, 1, 0)
    ctx.set_ntt_geometry(1, 0, 1)
    ctx.set_ntt_geometry(1, 1, 2)
    dq = wg.to_device(x)
    ctx.ntt_forward(dq, L)
    torch.cuda.synchronize()
    assert (wg.to_host(dq) == want_q).all()
    ctx.ntt_inverse(dq, L)
    torch.cuda.synchronize()
    assert (wg.to_host(dq) == x).all()
    for d in range(2):
        for ph in range(2):
            ctx.set_ntt_geometry(d, ph, -1)


def test_tuning_report(wg, oracle_mod):
    N, o, ctx = _setup(wg, oracle_mod, WALSH15)
    t = ctx.ntt_tuning()
    assert t["limbs"] >= 17
    ms = t["ms"]
    assert (ms > 0).all() and np.isfinite(ms).all()
    for d in range(2):
        for ph in range(2):
            g = t["chosen"][d][ph]
            assert 0 <= g < 4
            # the default geometry is replaced only by a fastest one at least 5 % faster
            if g == 0:
                assert (ms[d, ph, 1:] >= 0.95 * ms[d, ph, 0]).all()
            else:
                assert ms[d, ph, g] < 0.95 * ms[d, ph, 0] and ms[d, ph, g] == ms[d, ph, 1:].min()
    print("NTT tuning (N = 2^15, ms per phase over", t["limbs"], "limbs): chosen", t["chosen"])
    for d, dn in enumerate(("forward", "inverse")):
        for ph, pn in enumerate(("rows", "columns")):
            print(f"  {dn} {pn}: " + ", ".join(f"{ms[d, ph, g]:.4f}" for g in range(4)))
