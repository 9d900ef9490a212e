"""Write xboot_plans.json: the public structure of the reference's XBOOT bootstrapping contexts
(AESXBoot15Config, AESXBoot15Sparse1024Config, AESXBoot14SecureConfig and
AESXBoot14SecureSparse1024Config) that a device XBOOT AES-CTR run needs besides key and plaintext
values.

Generated from the reference compiled from its own sources (oracle/_ref, through oracle.RefPlans)
like walsh15_plan.json: prime chain, EvalMod bootstrap parameters and series coefficients (from
the reference's own MPFR EvalMod fit, src/math/poly_approx.cpp:565), rotation-key set, every SlotToCoeff and
CoeffToSlot stage's shape, switching-key shapes, and the levels and scales of the encrypted
round-key bits (ckks_aes128_encrypt_expanded_round_key_bits with the first round key 4 levels up,
as the reference benchmark encrypts them).  Residues are not stored: the benchmark draws them at
random with these shapes.

    python tests/golden/make_xboot_plans.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def plan_of(O, preset, expand_key):
    R = O.RefPlans(bootstrap_keys=True, preset=preset)
    info = R.bts_info()

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
    _, kscales, klevels = R.xboot_key_bits(expand_key(bytes(range(16))), 4)
    return {
        "ring_degree": int(R.N), "q": [int(x) for x in R.q], "p": [int(x) for x in R.p], "dnum": int(R.dnum),
        "bootstrap": {k: (float(v) if k == "scale" else int(v)) for k, v in info.items() if k != "coeffs"},
        "evalmod_coeffs": [float(x) for x in info["coeffs"]],
        "rotations": rots,
        "s2c": stages(0), "c2s": stages(1),
        "keys": keys,
        "aes": {"key_levels": [int(x) for x in klevels], "key_scales": [float(x) for x in kscales],
                "first_round_key_level": 4},
    }


def main():
    import oracle as O
    from aes_util import expand_key

    plans = {preset: plan_of(O, preset, expand_key)
             for preset in ("xboot15", "xboot15-sparse", "xboot14", "xboot14-sparse")}
    path = os.path.join(HERE, "xboot_plans.json")
    with open(path, "w") as f:
        json.dump(plans, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", path)


if __name__ == "__main__":
    main()
