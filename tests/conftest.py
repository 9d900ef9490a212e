"""Shared test setup.

* registers the ``gpu`` marker (tests that need a B200 and the built libwalshgpu.so);
* puts the oracle (test infrastructure) and the product package on sys.path;
* builds the oracle C library on first use, and the reference harness when its sources are
  present (they are not on GPU machines; tests needing it skip there).
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "aes-walsh-ckks_b200")
for p in (os.path.join(ROOT, "oracle"), PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built device library")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build(ref=False)
    return oracle


@pytest.fixture(scope="session")
def ref_mod(oracle_mod):
    if not oracle_mod.ref_available():
        if os.path.isdir(oracle_mod.REF_ROOT):
            subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle"), "ref",
                            "REF_ROOT=" + oracle_mod.REF_ROOT], check=True)
    if not oracle_mod.ref_available():
        pytest.skip("reference sources not available on this machine")
    return oracle_mod


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    return np.load(os.path.join(ROOT, "tests", "golden", "ref_n1024.npz"))


@pytest.fixture(scope="session")
def wg():
    import walshgpu

    walshgpu.lib()
    return walshgpu
