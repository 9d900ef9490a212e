"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference library compiled from its own sources (``make -C oracle ref``) through the
harness in oracle/ref_harness.cpp on small seeded inputs and stores inputs, the reference's
own (random) switching keys and the reference outputs:

    python tests/golden/make_golden.py

The reference's secrets come from the OS random source, so its keys cannot be regenerated
from a seed; they are stored with the fixture instead.  Parameters: N = 2^10, Q bits
[36, 61, 42, 42, 38] (the walsh15 chain's bit sizes, so Barrett products also land in
[q, 2q) sometimes), P bits [61, 61], dnum = 3.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

N = 1 << 10
Q_BITS = [36, 61, 42, 42, 38]
P_BITS = [61, 61]
DNUM = 3
ROTATION = 1


def main():
    O.build(ref=True)
    R = O.RefCtx(N, Q_BITS, P_BITS, DNUM, h=64, rotations=[ROTATION, 5])
    rng = np.random.default_rng(20261203)
    q = R.q
    L = len(q)

    def uniform(limbs):
        return np.concatenate([rng.integers(0, int(q[i]), N, dtype=np.uint64) for i in range(limbs)])

    out = {"N": np.array([N], np.uint64), "q": q, "p": R.p, "dnum": np.array([DNUM], np.uint64),
           "rotation": np.array([ROTATION], np.int64)}
    rot_key, parts, kl = R.key(0, ROTATION)
    conj_key, _, _ = R.key(1)
    relin_key, _, _ = R.key(2)
    out.update(rot_key=rot_key, conj_key=conj_key, relin_key=relin_key,
               key_parts=np.array([parts], np.uint64), key_level=np.array([kl], np.uint64))
    x = uniform(L)
    out["ntt_in"] = x
    out["ntt_fwd"] = R.ntt(x)
    out["ntt_inv"] = R.ntt(x, inverse=True)
    for level in (L - 1, 2):
        n = (level + 1) * N
        b, a, b2, a2 = uniform(level + 1), uniform(level + 1), uniform(level + 1), uniform(level + 1)
        out[f"l{level}_b"], out[f"l{level}_a"] = b, a
        out[f"l{level}_b2"], out[f"l{level}_a2"] = b2, a2
        rb, ra = R.rotate(level, b, a, ROTATION)
        out[f"l{level}_rot_b"], out[f"l{level}_rot_a"] = rb, ra
        cb, ca = R.conjugate(level, b, a)
        out[f"l{level}_conj_b"], out[f"l{level}_conj_a"] = cb, ca
        c0, c1, c2 = R.mul(level, b, a, b2, a2)
        out[f"l{level}_mul_c0"], out[f"l{level}_mul_c1"], out[f"l{level}_mul_c2"] = c0, c1, c2
        r0, r1 = R.relin(level, c0, c1, c2)
        out[f"l{level}_relin_b"], out[f"l{level}_relin_a"] = r0, r1
        s0, s1 = R.rescale(level, [r0, r1])
        out[f"l{level}_rescale_b"], out[f"l{level}_rescale_a"] = s0, s1
        assert n == b.size
    np.savez(os.path.join(HERE, "ref_n1024.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_n1024.npz"))


if __name__ == "__main__":
    main()
