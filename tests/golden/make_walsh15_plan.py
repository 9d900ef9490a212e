"""Write walsh15_plan.json: the public structure of the walsh15 bootstrapping context that the
device AES-CTR run needs besides key and plaintext values.

Generated from the reference compiled from its own sources (oracle/_ref, through oracle.RefPlans):
the prime chain, the EvalMod bootstrap parameters and its series coefficients (the reference's
own MPFR fit, src/math/poly_approx.cpp:565), the rotation-key set, every
SlotToCoeff (input scale ratio 1 and 2) and CoeffToSlot stage's shape (diagonal indices,
baby-step count, limbs, slot count, rescale flag), the switching-key shapes and the level and
scales of the encrypted AES key bits.  Values that do not steer the operation sequence (key
residues, diagonal residues, ciphertext residues) are not stored: the benchmark draws them at
random with these shapes, so it runs the same launches as a run on the reference's keys.

    python tests/golden/make_walsh15_plan.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def main():
    import oracle as O
    from aes_util import expand_key

    R = O.RefPlans(bootstrap_keys=True)
    info = R.bts_info()
    x2 = R.build_scaled_s2c(2)

    def stages(which):
        out = []
        for k in range(R.stages(which)):
            st = R.stage(which, k, with_diagonals=False)
            out.append({"qp_limbs": st["qp_limbs"], "indices": [int(i) for i in st["indices"]], "baby": st["baby"],
                        "slot_count": st["slot_count"], "rescale": st["rescale"]})
        return out

    keys = {}
    for name, kind, rot in (("relin", 2, 0), ("conj", 1, 0), ("dense_to_sparse", 3, 0), ("sparse_to_dense", 4, 0)):
        flat, parts, kl = R.key(rot, kind=kind)
        keys[name] = {"parts": parts, "key_level": kl, "words": int(flat.size)}
    rots = [int(r) for r in R.rotations()]
    flat, parts, kl = R.key(rots[0])
    keys["rotation"] = {"parts": parts, "key_level": kl, "words": int(flat.size)}
    # the encrypted key bits: level and per-bit scales do not depend on the key
    ek = expand_key(bytes(range(16)))
    _, kscales, klevel = R.aes_key_bits(ek, 512)
    plan = {
        "ring_degree": int(R.N), "q": [int(x) for x in R.q], "p": [int(x) for x in R.p], "dnum": int(R.dnum),
        "bootstrap": {k: (float(v) if k == "scale" else int(v)) for k, v in info.items() if k != "coeffs"},
        "evalmod_coeffs": [float(x) for x in info["coeffs"]],
        "rotations": rots,
        "s2c": stages(0), "s2c_x2": stages(x2), "c2s": stages(1),
        "keys": keys,
        "aes": {"key_level": int(klevel), "key_scales": [float(x) for x in kscales], "packing_block_count": 512,
                "packed_segment_count": 32, "active_blocks": 512},
    }
    with open(os.path.join(HERE, "walsh15_plan.json"), "w") as f:
        json.dump(plan, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", os.path.join(HERE, "walsh15_plan.json"))


if __name__ == "__main__":
    main()
