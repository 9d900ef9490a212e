#!/usr/bin/env python
"""Benchmark: the walsh15 batched-ops workload on the device library.

One step = 64 ciphertexts of the AESWalsh15 parameter set (N = 2^15, Q chain 36|61|42,42|
38 x7|50,50, P = 4 x 61, dnum = 3) at seeded levels uniform in 1..12, each multiplied by a
partner ciphertext, relinearized, rescaled and rotated by a seeded index from the walsh15
AES rotation-key set (+-512 k, k = 1..31), through wg_batch_mul_relin_rescale_rotate.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl walsh|reference]

Prints one JSON line (rank 0).  Under torchrun every rank runs its own 64 ciphertexts
(replicas, weak scaling); the elapsed time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "aes-walsh-ckks_b200")
sys.path.insert(0, PKG)

METRIC = "walsh15 AES-CTR latency, blocks/s: batched vs plain GPU; NTT/KS % of HBM peak"
UNIT = "ciphertexts/s"
LOGN = 15
Q_BITS = [36, 61, 42, 42] + [38] * 7 + [50, 50]
P_BITS = [61] * 4
DNUM = 3
COUNT = 64
ROT_POOL = [512 * k for k in range(1, 32)] + [-512 * k for k in range(1, 32)]
WORKLOAD = ("walsh15 batched ops: 64 ciphertexts at seeded levels 1..12, each ct x ct multiply + "
            "relinearize + rescale + rotate by a seeded walsh15 AES rotation index")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="walsh", choices=["walsh", "reference"])
    ap.add_argument("--count", type=int, default=COUNT)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the op-by-op comparison pass")
    ap.add_argument("--no-probe", action="store_true", help="skip the per-kernel event-timing passes")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end pass")
    ap.add_argument("--no-bsgs", action="store_true", help="skip the CoeffToSlot / SlotToCoeff section")
    ap.add_argument("--e2e-chunk", type=int, default=16, help="ciphertexts per overlapped chunk (e2e)")
    return ap.parse_args()


def workload(seed, count):
    rng = np.random.default_rng(seed)
    levels = rng.integers(1, len(Q_BITS), count)
    rots = [int(r) for r in rng.choice(ROT_POOL, count)]
    return levels, rots


# ------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device, period_ms=50):
        self.device = device
        self.period_ms = period_ms
        self.rows = []
        self.proc = None
        self.first = threading.Event()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms",
                 str(self.period_ms), "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.first.wait(timeout=15.0)  # the timed region starts once sampling runs
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)
                self.first.set()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------------------------------
# CPU arms (reference compiled from its own sources, else the oracle port)
# ------------------------------------------------------------------------------------------
def cpu_run(levels, rots, seconds_budget, threads=None):
    """Time the reference CPU path on a bounded sample of the workload.  Returns a dict."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    threads = threads or os.cpu_count()
    N = 1 << LOGN
    sample = 8 if seconds_budget < 60 else 16
    lv, rt = np.asarray(levels[:sample]), list(rots[:sample])
    L = len(Q_BITS)
    stride = L * N
    if O.ref_available():
        kind = "reference"
        R = O.RefCtx(N, Q_BITS, P_BITS, DNUM, h=256, rotations=sorted(set(rt)))
        q = R.q
    else:
        kind = "port"
        p, q = O.find_primes(P_BITS, Q_BITS, N)
        o = O.OracleCtx(N, q, p, DNUM)
        rng = np.random.default_rng(5)
        ks = o.key_size()
        keys = {r: np.concatenate([rng.integers(0, int(q[0]), ks, dtype=np.uint64)]) for r in set(rt)}
        relin = rng.integers(0, int(q[0]), ks, dtype=np.uint64)
    rng = np.random.default_rng(7)
    mk = lambda: np.concatenate([rng.integers(0, int(q[i % L]), N, dtype=np.uint64) for i in range(sample * L)])
    yb, ya = mk(), mk()
    xb0, xa0 = mk(), mk()
    done, elapsed = 0, 0.0
    while elapsed < seconds_budget or done == 0:
        xb, xa = xb0.copy(), xa0.copy()
        t0 = time.perf_counter()
        if kind == "reference":
            import ctypes as C

            sec = C.c_double()
            rc = O.ref().ref_batched_ops(R.h, sample, np.ascontiguousarray(lv, dtype=np.uintp), xb, xa, yb, ya,
                                         np.ascontiguousarray(rt, dtype=np.int64), stride, threads, C.byref(sec))
            if rc != 0:
                raise RuntimeError(O.ref().ref_last_error().decode())
        else:
            o.batched_ops(lv, xb, xa, yb, ya, relin, [keys[r] for r in rt], rt, stride, threads)
        elapsed += time.perf_counter() - t0
        done += sample
        if elapsed > 4 * seconds_budget:
            break
    return {"value": done / elapsed, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{done} ciphertexts ({sample} per pass, the first {sample} of the seeded 64) in "
                      f"{elapsed:.1f} s with {threads} threads"}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    levels, rots = workload(args.seed, args.count)
    for _ in range(args.warmup):
        cpu_run(levels, rots, 0.0)
    t0 = time.perf_counter()
    vals = [cpu_run(levels, rots, 0.0) for _ in range(args.steps)]
    total = time.perf_counter() - t0
    v = float(np.mean([x["value"] for x in vals]))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / max(1, args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sampled": vals[0]["sample"]},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": vals[0]["cores"], "kind": vals[0]["kind"],
                             "sample": vals[0]["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# CoeffToSlot / SlotToCoeff (BSGS linear-transform stages)
# ------------------------------------------------------------------------------------------
SLOTS = 1 << (LOGN - 1)


def _two_sided(step, count):
    return [step * k for k in range(count)] + [SLOTS - step * k for k in range(1, count)]


# The walsh15 plans' stage shapes (level, diagonal indices, baby-step count, rescale), as the
# reference's plan builder lays them out for this parameter set.
S2C_STAGES = [(1, list(range(16)) + [SLOTS - k for k in range(1, 16)], 8, False),
              (1, _two_sided(16, 32), 256, False),
              (1, [512 * k for k in range(32)], 4096, True)]
C2S_STAGES = [(12, [1024 * k for k in range(16)], 8192, False),
              (12, _two_sided(64, 16), 512, True),
              (11, _two_sided(8, 8), 64, False),
              (11, list(range(8)) + [SLOTS - k for k in range(1, 8)], 8, True)]
BSGS_BATCH = 8


def bsgs_bench(wg, ctx, q, p, stream, timed, steps, warmup):
    """Config 3: CoeffToSlot (4 stages from level 12) and SlotToCoeff (3 stages at level 1) over
    a batch of 8 ciphertexts, diagonals with the plans' index sets (uniform residues), keys of
    the walsh15 key shape (uniform residues)."""
    import torch

    N = 1 << LOGN
    K = len(P_BITS)
    L = len(Q_BITS)
    mods = np.concatenate([q, p]).astype(np.uint64)
    rng = np.random.default_rng(31)
    need = set()
    for _, idx, baby, _ in S2C_STAGES + C2S_STAGES:
        need |= {i % baby for i in idx if i % baby} | {(i // baby) * baby for i in idx if i // baby}
    parts = ctx.parts(L - 1)
    for r in sorted(need):
        if not ctx.has_key(wg.WG_KEY_ROTATION, r):
            limb_mod = np.tile(np.repeat(mods, N), 2 * parts)
            ctx.set_key(wg.WG_KEY_ROTATION, (rng.integers(0, 1 << 62, limb_mod.size, dtype=np.uint64) % limb_mod)
                        .astype(np.uint64), rotation=r)

    def stages(spec):
        out = []
        for level, idx, baby, resc in spec:
            qp = np.concatenate([q[: level + 1], p])
            col = np.tile(np.repeat(qp, N), len(idx))
            d = (rng.integers(0, 1 << 62, col.size, dtype=np.uint64) % col).astype(np.uint64)
            out.append((wg.LtStage(ctx, level, idx, d, baby, SLOTS, resc), level, len(idx), baby))
        return out

    res = {}
    qcol = np.repeat(q, N)
    cts = torch.from_numpy(np.stack([(rng.integers(0, 1 << 62, L * N, dtype=np.uint64) % qcol).astype(np.uint64)
                                     for _ in range(2 * BSGS_BATCH)]).view(np.int64)).cuda()
    bs = [cts[2 * i] for i in range(BSGS_BATCH)]
    as_ = [cts[2 * i + 1] for i in range(BSGS_BATCH)]
    for name, spec in (("coeff_to_slot", C2S_STAGES), ("slot_to_coeff", S2C_STAGES)):
        sts = stages(spec)

        def run():
            for st, _, _, _ in sts:
                st.apply(bs, as_, stream)

        for _ in range(warmup):
            run()
        ms = timed(run, steps)
        per_stage = []
        for st, level, d, baby in sts:
            sms = timed(lambda: st.apply(bs, as_, stream), steps)
            per_stage.append({"level": level, "diagonals": d, "baby": baby, "ms": sms})
        # algorithmic bytes: each diagonal read once per batch, each rotation key once, each
        # ciphertext read and written once
        total_bytes = 0.0
        for (level, idx, baby, _), ps in zip(spec, per_stage):
            Lq, beta = level + 1, ctx.parts(level)
            R = len({i % baby for i in idx if i % baby} | {(i // baby) * baby for i in idx if i // baby})
            sb = 8.0 * N * (len(idx) * (Lq + K) + R * beta * 2 * (Lq + K) + BSGS_BATCH * 4 * Lq)
            ps["gbs"] = sb / (ps["ms"] * 1e6)
            total_bytes += sb
        res[name] = {"ciphertexts_per_s": BSGS_BATCH / (ms / 1000.0), "ms_per_batch": ms,
                     "algorithmic_gbs": total_bytes / (ms * 1e6), "stages": per_stage}
        for st, _, _, _ in sts:
            st.close()
    res["batch"] = BSGS_BATCH
    res["data"] = "diagonals with the walsh15 plans' index sets, uniform residues; uniform keys"
    return res


# ------------------------------------------------------------------------------------------
# device arm
# ------------------------------------------------------------------------------------------
def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    import walshgpu as wg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    N = 1 << LOGN
    L = len(Q_BITS)
    p, q = wg.find_primes(P_BITS, Q_BITS, N)
    ctx = wg.Context(N, q, p, DNUM, device=local)
    levels, rots = workload(args.seed + rank, args.count)
    # Switching keys: uniform residues of the key shape.  The work is independent of key
    # values; bit-exactness with real keys is covered by the parity tests.
    krng = np.random.default_rng(99)
    parts = ctx.parts(L - 1)
    mods = np.concatenate([q, p]).astype(np.uint64)

    def random_key():
        limb_mod = np.tile(np.repeat(mods, N), 2 * parts)
        return (krng.integers(0, 1 << 62, limb_mod.size, dtype=np.uint64) % limb_mod).astype(np.uint64)

    ctx.set_key(wg.WG_KEY_RELIN, random_key())
    for r in sorted(set(rots)):
        ctx.set_key(wg.WG_KEY_ROTATION, random_key(), rotation=r)
    stream = torch.cuda.current_stream()
    ctx.reserve(stream)

    count = args.count
    stride = L * N  # words per polynomial slot
    qcol = np.repeat(q, N)
    drng = np.random.default_rng(1000 + rank)

    def uniform_ct():
        return (drng.integers(0, 1 << 62, L * N, dtype=np.uint64) % qcol).astype(np.uint64)

    host_x = np.stack([np.stack([uniform_ct(), uniform_ct()]) for _ in range(count)])  # [ct][b,a][L*N]
    host_y = np.stack([np.stack([uniform_ct(), uniform_ct()]) for _ in range(count)])
    pristine = torch.from_numpy(host_x.view(np.int64)).cuda()
    work = torch.empty_like(pristine)
    dy = torch.from_numpy(host_y.view(np.int64)).cuda()
    xb = [work[i, 0] for i in range(count)]
    xa = [work[i, 1] for i in range(count)]
    yb = [dy[i, 0] for i in range(count)]
    ya = [dy[i, 1] for i in range(count)]

    work.copy_(pristine)
    plan = wg.BatchPlan(ctx, levels, xb, xa, yb, ya, rots)

    def step():
        # one graph replay of the whole batched pipeline; every step runs on the previous
        # step's outputs (same levels and shapes: the work does not depend on residue values)
        plan.launch(stream)

    def step_nograph():
        ctx.batch_mul_relin_rescale_rotate(levels, xb, xa, yb, ya, rots, stream=stream)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def timed(fn, k):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1) / k
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    for _ in range(args.warmup):
        step()
    launches0 = wg.launch_count()
    with ClockSampler(local) as clk:
        ms = timed(step, args.steps)
    launches = wg.launch_count() - launches0

    for _ in range(args.warmup):
        step_nograph()
    nograph_ms = timed(step_nograph, args.steps)

    # per-kernel-class device time over the same K steps (CUDA events on the launch stream,
    # so the un-captured batched call is used)
    kernels = {}
    for name, cls in ([] if args.no_probe else wg.KCLASS.items()):
        wg.probe_begin(cls, 60000)
        timed(step_nograph, args.steps)
        n, kms, kbytes = wg.probe_end()
        kernels[name] = {"launches": n, "ms": kms, "bytes": kbytes}
    probed_total = sum(v["ms"] for v in kernels.values())
    for v in kernels.values():
        v["share"] = v["ms"] / probed_total if probed_total else None
        v["gbs"] = v["bytes"] / (v["ms"] * 1e6) if v["ms"] else None
    dom_name = max(kernels, key=lambda k: kernels[k]["ms"]) if kernels else "ntt"
    dom = kernels.get(dom_name, {"ms": 0.0, "launches": 0, "bytes": 0.0, "gbs": None})
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    # DRAM traffic of the dominant kernel from the committed ncu capture summary (ratio of
    # dram__bytes to algorithmic bytes, scaled to this launch size)
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "ntt_phase_traffic.json")))
        if dom_name == "ntt" and dom["launches"]:
            traffic = tr["dram_traffic_over_algorithmic"] * dom["bytes"] / dom["launches"]
    except (OSError, ValueError, KeyError):
        pass
    roofline = {"kernel": dom_name, "bound": "hbm", "achieved": dom["gbs"], "peak": hbm, "unit": "GB/s",
                "frac": dom["gbs"] / hbm if dom["gbs"] else None, "traffic": traffic,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "avg_launch_us": 1000 * dom["ms"] / max(1, dom["launches"]),
                "bytes_per_launch": dom["bytes"] / max(1, dom["launches"])}

    # the same workload op by op (the plain per-operation GPU path)
    def plain_step():
        ctx.batch_mul_relin_rescale_rotate(levels, xb, xa, yb, ya, rots, stream=stream, plain=True)

    plain_ms, plain_launches = None, None
    if not args.no_plain:
        plain_step()
        plain_launches0 = wg.launch_count()
        plain_ms = timed(plain_step, max(1, args.steps // 2))
        plain_launches = (wg.launch_count() - plain_launches0) / max(1, args.steps // 2)

    # End to end through the C ABI with host buffers: H2D of each ciphertext's active limbs
    # (x and y), the batched pipeline, D2H of the rescaled and rotated results.  The batch is
    # cut into chunks, each with its own graph plan; chunk k's compute overlaps chunk k+1's
    # upload and chunk k-1's download (copy-in, compute and copy-out streams).
    pin_x = torch.from_numpy(host_x.view(np.int64)).pin_memory()
    pin_y = torch.from_numpy(host_y.view(np.int64)).pin_memory()
    pin_out = torch.empty((count, 2, stride), dtype=torch.int64).pin_memory()
    h2d = int(sum(4 * (int(lv) + 1) * N * 8 for lv in levels))
    d2h = int(sum(2 * int(lv) * N * 8 for lv in levels))
    chunk = max(1, min(args.e2e_chunk, count))
    bounds = [(i, min(count, i + chunk)) for i in range(0, count, chunk)]
    e2e_ms = None
    if not args.no_e2e:
        cplans = [wg.BatchPlan(ctx, levels[a:b], xb[a:b], xa[a:b], yb[a:b], ya[a:b], rots[a:b]) for a, b in bounds]
        s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
        ev = lambda: torch.cuda.Event()
        in_done = [ev() for _ in bounds]
        comp_done = [ev() for _ in bounds]
        out_done = [ev() for _ in bounds]
        for e in out_done:
            e.record(s_out)

        def e2e_step():
            start = ev()
            start.record(stream)
            s_in.wait_event(start)
            for k, (a, b) in enumerate(bounds):
                s_in.wait_event(out_done[k])  # the chunk's buffers are free again
                for i in range(a, b):
                    nb = (int(levels[i]) + 1) * N * 8
                    for j in range(2):
                        wg.memcpy_htod(work[i, j], pin_x[i, j].data_ptr(), nb, stream=s_in)
                        wg.memcpy_htod(dy[i, j], pin_y[i, j].data_ptr(), nb, stream=s_in)
                in_done[k].record(s_in)
                stream.wait_event(in_done[k])
                cplans[k].launch(stream)
                comp_done[k].record(stream)
                s_out.wait_event(comp_done[k])
                for i in range(a, b):
                    nb = int(levels[i]) * N * 8
                    for j in range(2):
                        wg.memcpy_dtoh(pin_out[i, j].data_ptr(), work[i, j], nb, stream=s_out)
                out_done[k].record(s_out)
            stream.wait_stream(s_out)

        for _ in range(args.warmup):
            e2e_step()
        e2e_ms = timed(e2e_step, args.steps)
        # the last chunk's results are back in pinned host memory and match the device copy
        torch.cuda.synchronize()
        i = count - 1
        nb = int(levels[i]) * N
        assert torch.equal(pin_out[i, 0, :nb], work[i, 0, :nb].cpu())
        for cp in cplans:
            cp.close()

    bsgs = None if args.no_bsgs else bsgs_bench(wg, ctx, q, p, stream, timed, max(1, args.steps // 2),
                                                args.warmup)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_run(levels, rots, 15.0)
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "unavailable", "sample": str(e)}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    value = count * world / (ms / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "ring_degree": N, "q_limbs": L, "p_limbs": len(P_BITS), "dnum": DNUM,
                   "ciphertexts_per_gpu": count, "levels": [int(x) for x in levels],
                   "rotation_keys": len(set(rots)), "keys": "uniform residues of the walsh15 key shape",
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2: ~0.9 GB of ciphertexts plus ~1.1 GB of keys per step",
                   "step": "one CUDA-graph replay of the batched pipeline on the previous step's outputs",
                   "e2e_chunk": chunk},
        "clocks": clk.summary(),
        "e2e": {"value": count * world / (e2e_ms / 1000.0) if e2e_ms else None, "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "gpu_launches": int(launches),
        "batched_nograph": {"value": count * world / (nograph_ms / 1000.0), "unit": UNIT, "ms_per_step": nograph_ms},
        "plain_per_op": {"value": count * world / (plain_ms / 1000.0) if plain_ms else None, "unit": UNIT,
                         "ms_per_step": plain_ms, "launches_per_step": plain_launches},
        "roofline": roofline,
        "kernels": kernels,
        "bsgs": bsgs,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
