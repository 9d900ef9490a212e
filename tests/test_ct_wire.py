"""Ciphertext wire records (wg_ct_wire_*, host only): a round trip returns the residues and
labels word for word; a damaged byte, a truncated record, a record from another modulus chain
or ring degree, and residues not below their moduli are rejected."""
import numpy as np
import pytest


def _chain(wg, N=1 << 12):
    p, q = wg.find_primes([55, 55], [40, 45, 45, 45, 50], N)
    return N, q


def _record(wg, N, q, level, npolys, seed=3):
    rng = np.random.default_rng(seed)
    polys = np.concatenate([rng.integers(0, int(q[l]), N, dtype=np.uint64) for _ in range(npolys)
                            for l in range(level + 1)])
    return polys, wg.ct_wire_encode(N, q, level, polys, 2.0 ** 40, secret_owner=1, encoding_state=0)


@pytest.mark.parametrize("level,npolys", [(0, 2), (3, 2), (4, 3)])
def test_round_trip(wg, level, npolys):
    N, q = _chain(wg)
    polys, rec = _record(wg, N, q, level, npolys)
    assert len(rec) == wg.lib().wg_ct_wire_bytes(N, level, npolys)
    out, lv, sc, owner, state = wg.ct_wire_decode(rec, N, q)
    assert (out == polys).all() and (lv, sc, owner, state) == (level, 2.0 ** 40, 1, 0)


def test_damage_and_mismatch_are_rejected(wg):
    N, q = _chain(wg)
    polys, rec = _record(wg, N, q, 2, 2)
    for pos in (0, 5, 20, 60, len(rec) // 2, len(rec) - 1):
        bad = bytearray(rec)
        bad[pos] ^= 0x10
        with pytest.raises(wg.InvalidArgument):
            wg.ct_wire_decode(bytes(bad), N, q)
    with pytest.raises(wg.InvalidArgument):
        wg.ct_wire_decode(rec[:-9], N, q)
    other_p, other_q = wg.find_primes([55, 55], [41, 45, 45, 45, 50], N)
    with pytest.raises(wg.InvalidArgument):
        wg.ct_wire_decode(rec, N, other_q)
    with pytest.raises(wg.InvalidArgument):
        wg.ct_wire_decode(rec, 2 * N, q)
    big = polys.copy()
    big[5] = q[0]  # not below its modulus
    with pytest.raises(wg.InvalidArgument):
        wg.ct_wire_decode(wg.ct_wire_encode(N, q, 2, big, 1.0), N, q)
