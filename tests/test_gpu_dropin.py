"""The reference's own benchmark driver (bench/aes_bench.cpp, unchanged) on the device, linked
against the reference-API layer (libckks_b200.so): the context, keys, plans, EvalMod series,
encrypted round-key bits, AES-CTR circuit and decryption all come from the device library.
Its RESULT line must report 0 mismatched blocks and a max error below 0.5 (the driver's own
acceptance rule, bench/aes_bench.cpp:305-307), with errors of the magnitude the reference
reports for its CPU run (walsh15: max 1.08e-05, average 2.77e-07).

The binary is built in the container that holds the reference sources (oracle/Makefile
`dropin`) and travels with the working tree; elsewhere the test is skipped."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "aes_bench_b200")
RESULT = re.compile(r"RESULT method=(\S+) parameter=(\S+) blocks=(\d+) seconds=([\d.]+) max_error=(\S+) "
                    r"average_error=(\S+) mismatches=(\d+) rotations=(\d+)")


def _run(command, timeout):
    if not os.access(EXE, os.X_OK):
        pytest.skip("the drop-in benchmark binary is built where the reference sources are")
    r = subprocess.run([EXE, command], capture_output=True, text=True, timeout=timeout)
    print(r.stdout[-2000:])
    assert r.returncode == 0, r.stderr[-2000:]
    m = RESULT.search(r.stdout)
    assert m, r.stdout[-2000:]
    return dict(method=m.group(1), parameter=m.group(2), blocks=int(m.group(3)), seconds=float(m.group(4)),
                max_error=float(m.group(5)), average_error=float(m.group(6)), mismatches=int(m.group(7)),
                rotations=int(m.group(8)))


def test_reference_benchmark_walsh15_on_the_device():
    res = _run("walsh15", 900)
    assert res["blocks"] == 1024 and res["mismatches"] == 0
    assert res["max_error"] < 1e-3 and res["average_error"] < 1e-5
    assert res["rotations"] == 65  # the reference context's rotation-key count for walsh15


def test_reference_benchmark_xboot15_sparse_on_the_device():
    res = _run("xboot15-sparse-1024", 900)
    assert res["blocks"] == 1024 and res["mismatches"] == 0 and res["max_error"] < 0.5
