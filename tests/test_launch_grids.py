"""Every job-table kernel is launched with the grid its body indexes.

Most batched kernels take one word per thread (grid_for: N / 256 blocks per job); the
elementwise ones take kWide words per thread (wide_index, grid_wide: N / 1024 blocks per job).
A one-word grid given to a wide kernel makes it index up to 4 N words past each job's limb, and a
wide grid given to a one-word kernel leaves three quarters of each limb untouched; neither shows
up as an error.  This reads the CUDA sources (no GPU, no build): each kernel whose body calls
wide_index must be launched only as `kernel<<<grid_wide(...)` or through `launch_jobs<true>`, and
every other launch through grid_wide or launch_jobs<true> must name a wide kernel."""
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "aes-walsh-ckks_b200", "csrc")


def _sources():
    out = {}
    for path in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh"))):
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        out[os.path.basename(path)] = text
    return out


def _body(text, start):
    """The brace-matched body that opens at the first '{' at or after start."""
    i = text.index("{", start)
    depth = 0
    for k in range(i, len(text)):
        if text[k] == "{":
            depth += 1
        elif text[k] == "}":
            depth -= 1
            if depth == 0:
                return text[i:k + 1]
    raise AssertionError("unbalanced braces")


def _kernels(src):
    """name -> True when the kernel's body (or a device helper it calls by name) uses wide_index."""
    helpers = {}
    for name, text in src.items():
        for m in re.finditer(r"__device__\s+__forceinline__\s+\w+\s+(\w+)\s*\(", text):
            helpers[m.group(1)] = "wide_index(" in _body(text, m.end())
    kernels = {}
    for name, text in src.items():
        for m in re.finditer(r"__global__[^{;]*?\b(kb_\w+)\s*\(", text):
            body = _body(text, m.end())
            wide = "wide_index(" in body or any(h for h, w in helpers.items() if w and re.search(rf"\b{h}\s*[<(]", body))
            assert kernels.get(m.group(1), wide) == wide, m.group(1)
            kernels[m.group(1)] = wide
    return kernels


def test_wide_kernels_are_found():
    kernels = _kernels(_sources())
    wide = sorted(k for k, w in kernels.items() if w)
    for k in ("kb_tensor", "kb_scalar", "kb_lincomb", "kb_pmul", "kb_copy", "kb_add"):
        assert k in wide, (k, wide)
    for k in ("kb_mac_group", "kb_giant", "kb_gather", "kb_linear"):
        assert kernels.get(k) is False, k


def test_every_launch_matches_the_kernel_grid():
    src = _sources()
    kernels = _kernels(src)
    wide = {k for k, w in kernels.items() if w}
    bad = []
    for fname, text in src.items():
        for m in re.finditer(r"\b(kb_\w+)\s*<<<\s*(\w+)", text):
            kernel, grid = m.group(1), m.group(2)
            if kernel not in kernels:
                continue
            want = "grid_wide" if kernel in wide else None
            if (want and grid != want) or (not want and grid == "grid_wide"):
                bad.append((fname, kernel, grid))
        for m in re.finditer(r"\blaunch_jobs\s*(<\s*true\s*>)?\s*\(([^;]*)\)\s*;", text):
            as_wide = m.group(1) is not None
            for kernel in re.findall(r"\b(kb_\w+)\b", m.group(2)):
                if kernel in kernels and (kernel in wide) != as_wide:
                    bad.append((fname, kernel, "launch_jobs<true>" if as_wide else "launch_jobs"))
        # a wide kernel named anywhere else (a function pointer handed to another launcher)
        for kernel in wide:
            for m in re.finditer(rf"\b{kernel}\b", text):
                after = text[m.end():m.end() + 8]
                before = text[max(0, m.start() - 200):m.start()]
                if after.lstrip().startswith("<<<") or after.lstrip().startswith("("):
                    continue  # a launch (checked above) or the definition
                if re.search(r"launch_jobs\s*<\s*true\s*>\s*\([^;]*$", before):
                    continue  # an argument of launch_jobs<true> (checked above)
                bad.append((fname, kernel, "named outside a checked launch"))
    assert not bad, bad
