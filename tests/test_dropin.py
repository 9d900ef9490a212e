"""The reference-API layer (aes-walsh-ckks_b200/libckks_b200.so over the C ABI, headers under
aes-walsh-ckks_b200/shim/include) on the CPU:

* the reference's own benchmark driver, bench/aes_bench.cpp, compiles unchanged against the
  layer's headers and links with it (oracle/Makefile `dropin`, built where the reference
  sources are; its run on the device is tests/test_gpu_dropin.py);
* the layer's CKKSParams presets give the reference's modulus chains, P moduli, scale, depth,
  active slots, EvalMod K and DFT depths for all six AES parameter sets."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "aes-walsh-ckks_b200")
NAMES = ["walsh15", "xboot13", "xboot14", "xboot14-sparse", "xboot15", "xboot15-sparse"]


@pytest.fixture(scope="module")
def shim_presets(tmp_path_factory, wg):
    subprocess.run(["make", "-s", "-C", PKG, "libckks_b200.so"], check=True)
    exe = str(tmp_path_factory.mktemp("dropin") / "presets")
    subprocess.run(["g++", "-std=c++20", "-O1", "-I", os.path.join(PKG, "shim", "include"),
                    os.path.join(ROOT, "tests", "dropin", "presets.cpp"), "-o", exe, "-L", PKG, "-lckks_b200",
                    "-Wl,-rpath," + PKG], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return {d["name"]: d for d in (json.loads(line) for line in out.splitlines() if line.startswith("{"))}


def test_presets_match_reference(shim_presets, ref_mod):
    R = ref_mod.ref()
    R.ref_preset.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    for which, name in enumerate(NAMES):
        q, p = np.zeros(64, np.uint64), np.zeros(16, np.uint64)
        nq, np_, sc = C.c_size_t(), C.c_size_t(), C.c_double()
        info = np.zeros(5, np.uintp)
        assert R.ref_preset(which, q.ctypes.data, C.byref(nq), p.ctypes.data, C.byref(np_), C.byref(sc),
                            info.ctypes.data) == 0, name
        mine = shim_presets[name]
        assert mine["q"] == [int(x) for x in q[: nq.value]], name
        assert mine["p"] == [int(x) for x in p[: np_.value]], name
        assert mine["scale"] == sc.value, name
        assert [mine[k] for k in ("depth", "active", "k", "s2c", "c2s")] == [int(x) for x in info], name


def test_reference_benchmark_builds_against_the_layer(ref_mod):
    subprocess.run(["make", "-s", "-C", PKG, "libckks_b200.so"], check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "dropin", "REF_ROOT=" + ref_mod.REF_ROOT],
                   check=True)
    exe = os.path.join(ROOT, "oracle", "_ref", "aes_bench_b200")
    assert os.access(exe, os.X_OK)
    # without arguments the driver prints its usage and exits 2, before touching a device
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "walsh15" in r.stderr
