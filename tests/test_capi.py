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
