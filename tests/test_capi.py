"""The C ABI library loads and exports every entry point include/walsh_gpu.h declares.
Host-only entry points run without a GPU; nothing here launches a kernel."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "walsh_gpu.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wg_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def libwg():
    import walshgpu

    walshgpu.build()
    return walshgpu


def test_exports_every_declared_symbol(libwg):
    names = _declared()
    assert len(names) >= 20
    L = C.CDLL(libwg.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_library_does_not_link_the_oracle(libwg):
    out = subprocess.run(["readelf", "-d", libwg.LIB_PATH], capture_output=True, text=True, check=True).stdout
    needed = re.findall(r"\[(.*?)\]", "\n".join(l for l in out.splitlines() if "NEEDED" in l))
    assert not any("oracle" in n or "walshref" in n for n in needed), needed


def test_prime_chain_matches_oracle(libwg, oracle_mod):
    from params import CONFIG1, WALSH15

    for prm in (CONFIG1, WALSH15):
        N = 1 << prm["logN"]
        p, q = libwg.find_primes(prm["p_bits"], prm["q_bits"], N)
        po, qo = oracle_mod.find_primes(prm["p_bits"], prm["q_bits"], N)
        assert (p == po).all() and (q == qo).all()


def test_invalid_arguments_are_reported(libwg):
    with pytest.raises(libwg.InvalidArgument):
        libwg.find_primes([61], [50], 1000)  # N not a power of two
    assert libwg.lib().wg_version() >= 100


def test_context_without_gpu_fails_cleanly(libwg):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p, q = libwg.find_primes([55, 55], [50] * 3, 1024)
    with pytest.raises(libwg.WalshGpuError):
        libwg.Context(1024, q, p, 3)


def test_walsh15_plan_fixture_consistent(oracle_mod):
    """The bootstrap-structure fixture the benchmark builds its AES run from agrees with the
    library's prime generator and with the walsh15 shapes (limbs, slots, key sizes)."""
    import json

    plan = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "walsh15_plan.json")))
    N = plan["ring_degree"]
    p, q = oracle_mod.find_primes([61] * 4, [36, 61, 42, 42] + [38] * 7 + [50, 50], N)
    assert [int(x) for x in q] == plan["q"] and [int(x) for x in p] == plan["p"]
    K = len(plan["p"])
    for name in ("s2c", "s2c_x2", "c2s"):
        for st in plan[name]:
            assert 0 <= st["qp_limbs"] - 1 - K < len(plan["q"])
            assert all(0 <= i < N // 2 for i in st["indices"])
    for name, spec in plan["keys"].items():
        if name == "dense_to_sparse":
            assert spec["words"] == 4 * N
        else:
            assert spec["words"] == spec["parts"] * 2 * (spec["key_level"] + 1 + K) * N
    assert len(plan["aes"]["key_scales"]) == 11 * 128


def test_entry_points_reject_a_null_context(libwg):
    """Every context-taking entry point of the client setup, the XBOOT path and the bundle files
    returns an error status with a message for a null context (no exception crosses the ABI and
    no GPU is touched)."""
    L = libwg.lib()
    calls = {
        "wg_keygen_switch_key": lambda: L.wg_keygen_switch_key(None, 2, 1, None, None, None, 0, 3.2, None, None),
        "wg_keygen_secret_switch": lambda: L.wg_keygen_secret_switch(None, 3, None, None, None, None, 0, 3.2, None,
                                                                     None),
        "wg_encrypt_symmetric": lambda: L.wg_encrypt_symmetric(None, 0, 0, None, None, None, None, 0, 3.2, None, None,
                                                               None),
        "wg_encode_slots_device": lambda: L.wg_encode_slots_device(None, 0, 1, 1.0, None, None, None, 0, None),
        "wg_decrypt_decode": lambda: L.wg_decrypt_decode(None, 0, 0, None, None, None, None, None, None, None, None),
        "wg_bundle_save": lambda: L.wg_bundle_save(None, b"/nonexistent/x.wgb", None, 0),
        "wg_bundle_load": lambda: L.wg_bundle_load(None, b"/nonexistent/x.wgb", None, 0, None),
        "wg_bootstrap_pair": lambda: L.wg_bootstrap_pair(None, None, None, 0, None, 0, None, 0, 0, 1.0, None, None,
                                                         None, None, None, None, None),
        "wg_xboot_linear_layer": lambda: L.wg_xboot_linear_layer(None, 0, None, None, None, None, None, None, 1, None,
                                                                 None, None, None),
    }
    for name, call in calls.items():
        rc = call()
        assert rc != 0, name
        assert b"null context" in L.wg_last_error(), (name, L.wg_last_error())


def test_xboot_plan_fixture_consistent(oracle_mod):
    """The XBOOT bootstrap-structure fixture the benchmark's XBOOT sections build from agrees with
    the prime generator on the reference's XBOOT bit schedules (ckks_aes_params.hpp:133-209) and
    with its own shapes: stage limbs and diagonal indices, key sizes, and the round-key bits'
    levels (round 0 four levels above the S2C depth, the others at it) and scales."""
    import json

    plans = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "xboot_plans.json")))
    bits = {"xboot15": ([38] * 5, [38, 36, 36, 37, 37, 37] + [38] * 11),
            "xboot14": ([32], [31, 27, 30, 30, 30] + [31] * 6 + [27, 27])}
    assert set(plans) == {"xboot15", "xboot15-sparse", "xboot14", "xboot14-sparse"}
    for name, plan in plans.items():
        N = plan["ring_degree"]
        pb, qb = bits[name.split("-")[0]]
        p, q = oracle_mod.find_primes(pb, qb, N)
        assert [int(x) for x in q] == plan["q"] and [int(x) for x in p] == plan["p"], name
        K = len(plan["p"])
        b = plan["bootstrap"]
        assert b["slots"] == N // 2 and b["active_slots"] in (N // 2, 1024)
        for which in ("s2c", "c2s"):
            for st in plan[which]:
                assert 0 <= st["qp_limbs"] - 1 - K < len(plan["q"])
                assert all(0 <= i < st["slot_count"] for i in st["indices"])
        for kname, spec in plan["keys"].items():
            if kname == "dense_to_sparse":
                assert spec["words"] == 4 * N
            else:
                assert spec["words"] == spec["parts"] * 2 * (spec["key_level"] + 1 + K) * N
        lv = plan["aes"]["key_levels"]
        assert lv[:128] == [b["s2c_depth"] + 4] * 128 and lv[128:] == [b["s2c_depth"]] * 1280
        assert plan["aes"]["key_scales"] == [b["scale"]] * 1408


def test_header_is_clean_c11(tmp_path):
    """include/walsh_gpu.h is plain C (what a cgo / ctypes / JNI binding consumes): it compiles as
    C11 with every warning an error, and as C++."""
    src = tmp_path / "use_header.c"
    src.write_text('#include "walsh_gpu.h"\nint main(void) { return sizeof(wg_bootstrap_params) == 0; }\n')
    inc = os.path.join(ROOT, "include")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", inc, "-c", str(src), "-o",
                    str(tmp_path / "a.o")], check=True)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", inc, "-x", "c++", "-c", str(src), "-o",
                    str(tmp_path / "b.o")], check=True)
