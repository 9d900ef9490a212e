#!/usr/bin/env python
"""Benchmark: walsh15 homomorphic AES-128-CTR on the device library.

One step = one AES-CTR evaluation at the walsh15 parameter set (N = 2^15, Q chain
36|61|42,42|38 x7|50,50, P = 4 x 61, dnum = 3, EvalMod bootstrapping) over a slot-filling batch
of 1024 counter blocks (complex packing: block s in the real part and block 512 + s in the
imaginary part of slot s), through wg_aes_ctr_walsh: ten rounds of SubBytes (the 16 byte
positions as one batch of mask-packed Walsh S-boxes with bootstrapping), ShiftRows, MixColumns
and AddRoundKey on lazy bits, the final refresh and the XOR with the ciphertext blocks.  The
encrypted round-key bits and the switching keys stay device-resident; the step's counter and
ciphertext blocks come from host memory.  value = AES blocks per second over the K timed steps.

Key, diagonal and key-bit residues are uniform draws with the shapes of the reference's walsh15
context (tests/golden/walsh15_plan.json: stage shapes, rotation set, EvalMod series, key-bit
levels and scales): the launch sequence depends only on those shapes, levels and scales.
Bit-exactness and 0 decrypted mismatches on the reference's own keys are the parity tests'.

Further sections of the same JSON line:
  batched_ops   64 walsh15 ciphertexts at seeded levels, each ct x ct multiply + relinearize +
                rescale + rotate: one CUDA-graph replay vs the plain per-operation GPU path
  bsgs          CoeffToSlot / SlotToCoeff stages on 8 ciphertexts
  primitives    batched NTT at walsh15; the config-1 NTT and single rotation (N = 2^14, dnum 4)
  serving       Poisson stream of 2..1024-block requests through the continuous-batching service
  xboot_sbox    the XBOOT S-box (the other AES path's SubBytes) on 16 instances at xboot15
  cpu_baseline  the reference's SubBytes layer (16 S-box instances, OpenMP over instances as its
                AES does) on this host's cores, extrapolated to AES-CTR blocks/s

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl walsh|reference]

Prints one JSON line (rank 0).  Under torchrun every rank runs its own AES-CTR (replicas, weak
scaling); the elapsed time is the max over ranks.
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
PLAN_PATH = os.path.join(ROOT, "tests", "golden", "walsh15_plan.json")

METRIC = "walsh15 AES-CTR latency, blocks/s: batched vs plain GPU; NTT/KS % of HBM peak"
UNIT = "blocks/s"
LOGN = 15
Q_BITS = [36, 61, 42, 42] + [38] * 7 + [50, 50]
P_BITS = [61] * 4
DNUM = 3
ROUNDS = 10
SBOX_INSTANCES = 16  # byte positions per SubBytes layer
WORKLOAD = ("walsh15 AES-128-CTR: 1024 counter blocks per evaluation (2 x 512 complex-packed slots), "
            "10 rounds with batched Walsh S-boxes and EvalMod bootstrapping, final refresh and XOR")
OPS_COUNT = 64
ROT_POOL = [512 * k for k in range(1, 32)] + [-512 * k for k in range(1, 32)]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="walsh", choices=["walsh", "reference"])
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-probe", action="store_true", help="skip the per-kernel-class event-timing passes")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end pass")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-operation AES pass")
    ap.add_argument("--no-ops", action="store_true", help="skip the batched-ops section")
    ap.add_argument("--no-ntt", action="store_true", help="skip the NTT / rotation primitives section")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-requests section")
    ap.add_argument("--no-xboot", action="store_true", help="skip the XBOOT S-box section")
    ap.add_argument("--no-xboot-aes", action="store_true", help="skip the XBOOT AES-CTR section")
    ap.add_argument("--xboot-aes-steps", type=int, default=2, help="timed XBOOT AES-CTR evaluations (after one warm-up)")
    ap.add_argument("--no-keygen", action="store_true", help="skip the device key generation section")
    ap.add_argument("--serve-requests", type=int, default=32)
    ap.add_argument("--serve-mix-requests", type=int, default=10)
    ap.add_argument("--no-clocks", action="store_true",
                    help="do not sample nvidia-smi clocks (for runs under a profiler, which wants the GPU to itself)")
    ap.add_argument("--no-aes", action="store_true",
                    help="skip the AES-CTR headline (profiling runs of the NTT, batched-ops and XBOOT AES sections; "
                         "no headline value)")
    ap.add_argument("--no-bsgs", action="store_true", help="skip the CoeffToSlot / SlotToCoeff section")
    ap.add_argument("--ops-steps", type=int, default=50)
    ap.add_argument("--ops-count", type=int, default=OPS_COUNT)
    ap.add_argument("--e2e-chunk", type=int, default=16, help="ciphertexts per overlapped chunk (ops e2e)")
    return ap.parse_args()


def max_over_ranks(value, dist, device="cuda"):
    """The maximum of a per-rank time over all ranks (every rank gets it); the value itself on
    a single process."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_plan():
    with open(PLAN_PATH) as f:
        return json.load(f)


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
        if self.device is None:
            return self
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
# CPU: the reference's SubBytes layer (compiled from its own sources)
# ------------------------------------------------------------------------------------------
def _ref_sbox_setup():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if not O.ref_available():
        raise RuntimeError("the reference library (oracle/_ref) is not built")
    R = O.RefPlans(bootstrap_keys=True)
    info = R.bts_info()
    level = info["s2c_depth"]
    N = R.N
    rng = np.random.default_rng(17)
    qc = np.repeat(R.q[: level + 1], N)
    draw = lambda: (rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)
    bits = [(draw(), draw()) for _ in range(8)]
    return R, info, bits


def _layer_line(seconds, threads, layers):
    blocks = 2 * 512
    return {"value": blocks / (ROUNDS * seconds), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{layers} SubBytes layer(s) of {SBOX_INSTANCES} mask-packed Walsh S-box instances (the "
                      f"reference's ckks_walsh_sbox_complex_blocks_mask_packed, OpenMP over instances as its AES "
                      f"SubBytes runs them) on {threads} threads, {seconds:.2f} s per layer; AES-CTR time taken "
                      f"as {ROUNDS} layers for {blocks} blocks (its linear layers and final refresh not counted, "
                      f"which favours the reference)"}


def cpu_baseline():
    R, info, bits = _ref_sbox_setup()
    threads = os.cpu_count()
    sec = R.walsh_sbox_layer_seconds(512, info["s2c_depth"], info["scale"], bits, SBOX_INSTANCES, threads)
    return _layer_line(sec, threads, 1)


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    R, info, bits = _ref_sbox_setup()
    threads = os.cpu_count()
    level, scale = info["s2c_depth"], info["scale"]
    for _ in range(args.warmup):  # one instance each: pages in keys, plans and code
        R.walsh_sbox_layer_seconds(512, level, scale, bits, 1, threads)
    samples, t0 = [], time.perf_counter()
    for i in range(args.steps):
        samples.append(R.walsh_sbox_layer_seconds(512, level, scale, bits, SBOX_INSTANCES, threads))
        if time.perf_counter() - t0 > 200.0:  # keep the arm within a few minutes
            break
    sec = float(np.mean(samples))
    base = _layer_line(sec, threads, len(samples))
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sec, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sampled": base["sample"], "timed_layers": len(samples)},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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


def bsgs_bench(wg, ctx, q, p, stream, timed, steps, warmup, with_cpu=False):
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
    if with_cpu:
        res["reference_cpu"] = ref_bsgs_sample()
    return res


def ref_bsgs_sample():
    """Both plans on the reference's CPU path: its own walsh15 CoeffToSlot (from level 12) and
    SlotToCoeff (level 1) plans and rotation keys, every stage through its QP evaluator, on a
    batch of copies of one uniform ciphertext with OpenMP over ciphertexts."""
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        if not O.ref_available():
            return {"unavailable": "the reference library (oracle/_ref) is not built"}
        R = O.RefPlans()
        N, threads = R.N, os.cpu_count()
        rng = np.random.default_rng(43)
        out = {"cores": threads, "kind": "reference",
               "sample": f"{BSGS_BATCH} ciphertexts per plan, OpenMP over ciphertexts on {threads} threads"}
        for name, which, level in (("coeff_to_slot", 1, 12), ("slot_to_coeff", 0, 1)):
            qc = np.repeat(R.q[: level + 1], N)
            b, a = [(rng.integers(0, 1 << 62, qc.size, dtype=np.uint64) % qc).astype(np.uint64) for _ in range(2)]
            sec = R.plan_seconds(which, level, b, a, BSGS_BATCH, threads)
            out[name] = {"ciphertexts_per_s": BSGS_BATCH / sec, "seconds": sec}
        return out
    except Exception as e:  # reported, never required
        return {"unavailable": str(e)}


# ------------------------------------------------------------------------------------------
# batched ops: mul + relin + rescale + rotate on 64 ciphertexts, batched vs plain
# ------------------------------------------------------------------------------------------
def ops_bench(args, wg, torch, stream, timed, rank, local, with_cpu=False):
    N = 1 << LOGN
    L = len(Q_BITS)
    p, q = wg.find_primes(P_BITS, Q_BITS, N)
    ctx = wg.Context(N, q, p, DNUM, device=local)
    rng = np.random.default_rng(args.seed + rank)
    count = args.ops_count
    levels = rng.integers(1, L, count)
    rots = [int(r) for r in rng.choice(ROT_POOL, count)]
    # switching keys: uniform residues of the key shape (the work does not depend on them)
    krng = np.random.default_rng(99)
    parts = ctx.parts(L - 1)
    mods = np.concatenate([q, p]).astype(np.uint64)

    def random_key():
        limb_mod = np.tile(np.repeat(mods, N), 2 * parts)
        return (krng.integers(0, 1 << 62, limb_mod.size, dtype=np.uint64) % limb_mod).astype(np.uint64)

    ctx.set_key(wg.WG_KEY_RELIN, random_key())
    for r in sorted(set(rots)):
        ctx.set_key(wg.WG_KEY_ROTATION, random_key(), rotation=r)
    ctx.reserve(stream)
    stride = L * N
    qcol = np.repeat(q, N)
    drng = np.random.default_rng(1000 + rank)
    uniform_ct = lambda: (drng.integers(0, 1 << 62, L * N, dtype=np.uint64) % qcol).astype(np.uint64)
    host_x = np.stack([np.stack([uniform_ct(), uniform_ct()]) for _ in range(count)])  # [ct][b,a][L*N]
    host_y = np.stack([np.stack([uniform_ct(), uniform_ct()]) for _ in range(count)])
    work = torch.from_numpy(host_x.view(np.int64)).cuda()
    dy = torch.from_numpy(host_y.view(np.int64)).cuda()
    xb = [work[i, 0] for i in range(count)]
    xa = [work[i, 1] for i in range(count)]
    yb = [dy[i, 0] for i in range(count)]
    ya = [dy[i, 1] for i in range(count)]
    plan = wg.BatchPlan(ctx, levels, xb, xa, yb, ya, rots)
    steps = max(1, args.ops_steps)
    # one graph replay of the whole batched pipeline per step, on the previous step's outputs
    graph_step = lambda: plan.launch(stream)
    nograph_step = lambda: ctx.batch_mul_relin_rescale_rotate(levels, xb, xa, yb, ya, rots, stream=stream)
    plain_step = lambda: ctx.batch_mul_relin_rescale_rotate(levels, xb, xa, yb, ya, rots, stream=stream, plain=True)
    for _ in range(args.warmup):
        graph_step()
    l0 = wg.launch_count()
    graph_ms = timed(graph_step, steps)
    graph_launches = (wg.launch_count() - l0) / steps
    for _ in range(args.warmup):
        nograph_step()
    nograph_ms = timed(nograph_step, steps)
    # the same batched call with ModUp / ModDown as separate launches (no NTT column fusion)
    ctx.set_ntt_fusion(False)
    nograph_step()
    unfused_ms = timed(nograph_step, steps)
    ctx.set_ntt_fusion(True)
    plain_step()
    l0 = wg.launch_count()
    plain_ms = timed(plain_step, max(1, steps // 2))
    plain_launches = (wg.launch_count() - l0) / max(1, steps // 2)
    # NTT class over the batched call (CUDA events on the launch stream)
    wg.probe_begin(wg.KCLASS["ntt"], 60000)
    timed(nograph_step, 1)
    n, kms, kbytes = wg.probe_end()
    # end to end with host buffers: H2D of each ciphertext's active limbs, the pipeline in
    # chunks (compute of chunk k overlaps the upload of k+1 and the download of k-1), D2H
    e2e = None
    if not args.no_e2e:
        pin_x = torch.from_numpy(host_x.view(np.int64)).pin_memory()
        pin_y = torch.from_numpy(host_y.view(np.int64)).pin_memory()
        pin_out = torch.empty((count, 2, stride), dtype=torch.int64).pin_memory()
        chunk = max(1, min(args.e2e_chunk, count))
        bounds = [(i, min(count, i + chunk)) for i in range(0, count, chunk)]
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
        e2e_ms = timed(e2e_step, steps)
        torch.cuda.synchronize()
        i = count - 1
        nb = int(levels[i]) * N
        assert torch.equal(pin_out[i, 0, :nb], work[i, 0, :nb].cpu())
        for cp in cplans:
            cp.close()
        e2e = {"value": count / (e2e_ms / 1000.0), "unit": "ciphertexts/s", "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": int(sum(4 * (int(lv) + 1) * N * 8 for lv in levels)),
               "d2h_bytes_per_step": int(sum(2 * int(lv) * N * 8 for lv in levels)), "chunk": chunk}
    plan.close()
    K = len(P_BITS)
    alg = 0.0
    for lv in levels:
        lq = int(lv) + 1
        beta = ctx.parts(int(lv))
        alg += 8.0 * N * (4 * lq + 2 * beta * 2 * (lq + K) + 2 * lq)
    res = {
        "workload": f"{count} walsh15 ciphertexts at seeded levels 1..12, each ct x ct multiply + relinearize + "
                    f"rescale + rotate by a seeded walsh15 AES rotation index",
        "unit": "ciphertexts/s",
        "batched_graph": {"value": count / (graph_ms / 1000.0), "ms_per_step": graph_ms,
                          "launches_per_step": graph_launches},
        "batched_nograph": {"value": count / (nograph_ms / 1000.0), "ms_per_step": nograph_ms},
        "batched_nograph_unfused_keyswitch": {"value": count / (unfused_ms / 1000.0), "ms_per_step": unfused_ms,
                                              "fused_speedup": unfused_ms / nograph_ms},
        "plain_per_op": {"value": count / (plain_ms / 1000.0), "ms_per_step": plain_ms,
                         "launches_per_step": plain_launches},
        "batched_over_plain": plain_ms / graph_ms,
        "algorithmic_bytes_per_step": alg,
        "algorithmic_gbs": alg / (graph_ms * 1e6),
        "algorithmic_bytes_note": "per ciphertext 8 N [4 Lq (two inputs) + 2 beta 2 (Lq + K) (relin and "
                                  "rotation keys) + 2 Lq (output)]: the pipeline's compulsory traffic",
        "ntt": {"launches": n, "ms": kms, "gbs": kbytes / (kms * 1e6) if kms else None},
        "e2e": e2e, "steps": steps,
    }
    if with_cpu:
        res["reference_cpu"] = ref_ops_sample(levels, rots, args.seed + 41)
    return res, ctx, q, p


def ref_ops_sample(levels, rots, seed):
    """The batched-ops workload (same levels and rotation indices) on the reference's CPU path:
    its own multiply, relinearize, rescale and rotate per ciphertext with OpenMP over
    ciphertexts (ref_batched_ops), on a reference context of the same chain holding the
    relinearisation key and the rotation keys the workload uses; uniform residues."""
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        if not O.ref_available():
            return {"unavailable": "the reference library (oracle/_ref) is not built"}
        N, L, count = 1 << LOGN, len(Q_BITS), len(levels)
        R = O.RefCtx(N, Q_BITS, P_BITS, DNUM, rotations=sorted(set(int(r) for r in rots)))
        stride = L * N
        rng = np.random.default_rng(seed)
        qcol = np.tile(np.repeat(R.q, N), count)
        draw = lambda: (rng.integers(0, 1 << 62, count * stride, dtype=np.uint64) % qcol).astype(np.uint64)
        xb, xa, yb, ya = draw(), draw(), draw(), draw()
        threads = os.cpu_count()
        sec = R.batched_ops_seconds(levels, xb, xa, yb, ya, rots, stride, threads)
        return {"value": count / sec, "unit": "ciphertexts/s", "seconds": sec, "cores": threads, "kind": "reference",
                "sample": f"the whole workload ({count} ciphertexts, the same levels and rotation indices) through "
                          f"the reference's ckks_mul_inplace, ckks_relin_hybrid_inplace, ckks_rescale and "
                          f"ckks_rotate_inplace, OpenMP over ciphertexts on {threads} threads"}
    except Exception as e:  # reported, never required
        return {"unavailable": str(e)}


# ------------------------------------------------------------------------------------------
# primitives: batched NTT at walsh15, and the plain single-ciphertext config-1 primitives
# ------------------------------------------------------------------------------------------
def ntt_bench(wg, torch, stream, timed, local, steps, hbm):
    """Forward and inverse negacyclic NTT over batches of limbs, and one hybrid key switch
    (rotation by +1) of a single ciphertext.  Algorithmic bytes: 16 N B per limb-transform
    (each residue read and written once); a rotation moves 8 N [2 Lq + beta 2 (Lq + K) + 2 Lq] B
    (ciphertext in, evaluation key, ciphertext out)."""
    res = {}
    shapes = (("walsh15_batch", 15, Q_BITS, P_BITS, DNUM, 64),   # 64 polynomials x 13 limbs: 218 MB > L2
              ("config1", 14, [50] * 16, [50] * 4, 4, 2))         # one ciphertext (a, b) x 16 limbs
    for name, logn, qb, pb, dnum, polys in shapes:
        N = 1 << logn
        p, q = wg.find_primes(pb, qb, N)
        ctx = wg.Context(N, q, p, dnum, device=local)
        L, K = len(q), len(p)
        rng = np.random.default_rng(logn)
        qcol = np.repeat(q, N)
        host = np.stack([(rng.integers(0, 1 << 62, L * N, dtype=np.uint64) % qcol).astype(np.uint64)
                         for _ in range(polys)])
        data = torch.from_numpy(host.view(np.int64)).cuda()
        fwd = lambda: ctx.ntt_forward(data, L, polys=polys, stride=L * N, stream=stream)
        inv = lambda: ctx.ntt_inverse(data, L, polys=polys, stride=L * N, stream=stream)
        for _ in range(3):
            fwd()
            inv()
        tf, ti = timed(fwd, steps), timed(inv, steps)
        nbytes = 16.0 * N * L * polys
        entry = {"ring_degree": N, "limbs": L, "polynomials": polys,
                 "forward_us": 1000 * tf, "inverse_us": 1000 * ti,
                 "forward_gbs": nbytes / (tf * 1e6), "inverse_gbs": nbytes / (ti * 1e6),
                 "forward_frac": nbytes / (tf * 1e6) / hbm, "inverse_frac": nbytes / (ti * 1e6) / hbm}
        if name == "config1":
            parts = ctx.parts(L - 1)
            mods = np.concatenate([q, p]).astype(np.uint64)
            col = np.tile(np.repeat(mods, N), 2 * parts)
            ctx.set_key(wg.WG_KEY_ROTATION, (rng.integers(0, 1 << 62, col.size, dtype=np.uint64) % col)
                        .astype(np.uint64), rotation=1)
            rot = lambda: ctx.rotate(L - 1, data[0], data[1], 1, stream=stream)
            for _ in range(3):
                rot()
            tr = timed(rot, steps)
            rbytes = 8.0 * N * (2 * L + parts * 2 * (L + K) + 2 * L)
            entry.update({"rotation_us": 1000 * tr, "rotation_gbs": rbytes / (tr * 1e6),
                          "rotation_frac": rbytes / (tr * 1e6) / hbm, "dnum": dnum})
        res[name] = entry
    return res


def ref_config1_sample(repeats=5):
    """Config 1 on the reference's own CPU functions as it calls them for one ciphertext:
    forward and inverse NTT of both polynomials' 16 limbs (ntt_forward_rns_flat_inplace /
    ntt_inverse_rns_flat_inplace with the context's tables) and one rotation by +1
    (ckks_rotate_inplace) at level 15, N = 2^14, dnum 4; medians of `repeats` calls."""
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        if not O.ref_available():
            return {"unavailable": "the reference library (oracle/_ref) is not built"}
        R, lib = O.RefCtx(1 << 14, [50] * 16, [50] * 4, 4, rotations=(1,)), O.ref()
        N, L = R.N, len(R.q)
        rng = np.random.default_rng(14)
        qcol = np.repeat(R.q, N)
        b, a = [(rng.integers(0, 1 << 62, L * N, dtype=np.uint64) % qcol).astype(np.uint64) for _ in range(2)]

        def median(call):
            ts = []
            for _ in range(repeats):
                t0 = time.perf_counter()
                call()
                ts.append(time.perf_counter() - t0)
            return float(np.median(ts))

        def ntt(inverse):
            for x in (b, a):
                O._check(lib.ref_ctx_ntt(R.h, x, L, int(inverse), 0), "ref_ctx_ntt")

        tf = median(lambda: ntt(False))
        ti = median(lambda: ntt(True))
        tr = median(lambda: O._check(lib.ref_rotate(R.h, L - 1, b, a, 1), "ref_rotate"))
        return {"forward_us": 1e6 * tf, "inverse_us": 1e6 * ti, "rotation_us": 1e6 * tr, "cores": os.cpu_count(),
                "kind": "reference", "sample": f"one ciphertext (2 x {L} limbs), the reference's functions with "
                                              f"their own threading, median of {repeats} calls"}
    except Exception as e:  # reported, never required
        return {"unavailable": str(e)}


# ------------------------------------------------------------------------------------------
# AES-CTR on the device
# ------------------------------------------------------------------------------------------
class AesRun:
    """The walsh15 AES-CTR evaluation with real key material, all of it made by the library on
    the device: a seeded ternary secret of Hamming weight 256 and the sparse bootstrapping secret
    of weight 32, every switching key from them (wg_keygen_switch_key / wg_keygen_secret_switch,
    one seed per key), the SlotToCoeff (x1, x2 input scale) and CoeffToSlot plans
    (wg_dft_plan_create), the EvalMod series (wg_evalmod_fit) and the 1408 encrypted round-key
    bits of a seeded AES key (wg_aes_walsh_encrypt_round_key_bits).  The chain and bootstrap
    parameters are the walsh15 preset's (tests/golden/walsh15_plan.json).  Counter blocks and
    CTR ciphertexts of seeded plaintexts, so every output can be decrypted and checked against
    plain AES-128 (check())."""

    def __init__(self, wg, torch, plan, device, seed):
        N = plan["ring_degree"]
        q = np.array(plan["q"], dtype=np.uint64)
        p = np.array(plan["p"], dtype=np.uint64)
        self.N, self.wg, self.torch = N, wg, torch
        self.ctx = ctx = wg.Context(N, q, p, plan["dnum"], device=device)
        rng = np.random.default_rng(seed)

        def ternary(h):
            s = np.zeros(N, np.int8)
            pos = rng.choice(N, h, replace=False)
            s[pos] = rng.choice(np.array([-1, 1], np.int8), h)
            return s

        self.secret, self.low_secret = ternary(256), ternary(32)
        b = plan["bootstrap"]
        self.params = wg.BootstrapParams(b["s2c_depth"], b["depth"], b["evalmod_log_scale"], b["double_angle"],
                                         b["active_slots"], b["slots"], b["scale"])
        # the walsh15 preset's DFT literals (its scale schedules, bootstrap depths and EvalMod K)
        q0, scale = float(q[0]), b["scale"]
        K = wg.evalmod_k_bound(N, 32, -16.0)
        s2c = lambda ratio: wg.DftLiteral.make(False, b["s2c_depth"], (q0 * 0.5) / (scale * ratio),
                                               scale_groups=[[18, 20, 23]], active_slots=b["active_slots"])
        c2s = wg.DftLiteral.make(True, b["depth"], np.ldexp(scale, b["evalmod_log_scale"] - 36) / q0 / K,
                                 scale_groups=[[25, 25], [25, 25]], active_slots=b["active_slots"])
        self.s2c, self.s2c_x2, self.c2s = ctx.dft_plan(s2c(1)), ctx.dft_plan(s2c(2)), ctx.dft_plan(c2s)
        self.coeffs = wg.evalmod_fit(K, 100, 0, np.nextafter(0.25, 0.0), 128, 1e-10)["coeffs"]
        rots = set()
        for st in self.s2c + self.c2s:
            idx, _ = st.download()
            baby = st.info()["baby"]
            for d in idx.tolist():
                rots.update(r for r in (d % baby, d - d % baby) if r)
        a = plan["aes"]
        self.pbc, self.psc, self.acb = a["packing_block_count"], a["packed_segment_count"], a["active_blocks"]
        half = N // 2
        rots.update(r % half for k in range(1, self.psc) for r in (k * self.pbc, -k * self.pbc))
        self.rotations = sorted(r for r in rots if r)
        seeds = iter(rng.integers(1, 2**63, len(self.rotations) + 8).tolist())
        for r in self.rotations:
            ctx.keygen_switch_key(wg.WG_KEY_ROTATION, r, self.secret, seed=next(seeds))
        ctx.keygen_switch_key(wg.WG_KEY_CONJ, 0, self.secret, seed=next(seeds))
        ctx.keygen_switch_key(wg.WG_KEY_RELIN, 0, self.secret, seed=next(seeds))
        ctx.keygen_secret_switch(wg.WG_KEY_DENSE_TO_SPARSE, self.secret, self.low_secret, seed=next(seeds))
        ctx.keygen_secret_switch(wg.WG_KEY_SPARSE_TO_DENSE, self.low_secret, self.secret, seed=next(seeds))
        # a seeded AES key, its 1408 encrypted expanded-key bits on the device
        from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes

        self.aes_key = bytes(rng.integers(0, 256, 16, dtype=np.uint8))
        self._ecb = Cipher(algorithms.AES(self.aes_key), modes.ECB())
        self.kl = b["s2c_depth"] + 1
        n = (self.kl + 1) * N
        self.key_dev = torch.empty((1408, 2, n), dtype=torch.int64, device="cuda")
        self.key_bits = [(self.key_dev[k, 0], self.key_dev[k, 1]) for k in range(1408)]
        self.kscales, lv = ctx.aes_walsh_encrypt_round_key_bits(self.params, expand_key(self.aes_key), self.acb,
                                                                self.secret, self.key_bits, seed=next(seeds))
        assert (np.asarray(lv) == self.kl).all()
        full = (b["depth"] + 1) * N
        self.out_dev = torch.zeros((128, 2, full), dtype=torch.int64, device="cuda")
        self.outs = [(self.out_dev[k, 0], self.out_dev[k, 1]) for k in range(128)]
        self.blocks = 2 * self.acb
        # block_bytes[2i] counters, block_bytes[2i+1] CTR ciphertexts of plaintexts[i]
        self.plaintexts, self.block_bytes = [], []
        for _ in range(2):
            ctr = bytes(rng.integers(0, 256, 16 * self.blocks, dtype=np.uint8))
            pt = bytes(rng.integers(0, 256, 16 * self.blocks, dtype=np.uint8))
            e = self._ecb.encryptor()
            stream = e.update(ctr) + e.finalize()
            self.plaintexts.append(pt)
            self.block_bytes += [ctr, bytes(x ^ y for x, y in zip(pt, stream))]
        self.calls = 0
        self.last = None

    def step(self, stream, plain=False):
        k = self.calls % 2
        self.calls += 1
        self.last = k
        return self.ctx.aes_ctr_walsh(self.params, self.s2c, self.s2c_x2, self.c2s, self.coeffs, self.pbc, self.psc,
                                      self.key_bits, self.kscales, self.kl, self.block_bytes[2 * k],
                                      self.block_bytes[2 * k + 1], self.acb, self.outs, stream=stream, plain=plain)

    def check(self, levels, scales):
        """Decrypt the last evaluation's 128 output bits on the device and compare them with the
        plaintext the way the reference benchmark does (validate_walsh_outputs,
        bench/aes_bench.cpp:156-195): mismatched blocks, max and average |lane - bit|."""
        self.torch.cuda.synchronize()
        pt = np.frombuffer(self.plaintexts[self.last], dtype=np.uint8).reshape(self.blocks, 16)
        acb = self.acb
        err_max, err_sum, count = 0.0, 0.0, 0
        decoded = np.zeros((self.blocks, 16), np.uint8)
        for lvl in sorted(set(int(x) for x in levels)):
            bits = [i for i in range(128) if int(levels[i]) == lvl]
            z = self.ctx.decrypt_decode(lvl, [scales[i] for i in bits], [self.outs[i] for i in bits], self.secret)
            for j, bit in enumerate(bits):
                vals = np.concatenate([z[j, :acb].real, z[j, :acb].imag])  # block s, then block acb + s
                want = ((pt[:, bit // 8] >> (bit % 8)) & 1).astype(np.float64)
                e = np.abs(vals - want)
                err_max = max(err_max, float(e.max()))
                err_sum += float(e.sum())
                count += e.size
                decoded[:, bit // 8] |= ((vals >= 0.5).astype(np.uint8) << (bit % 8))
        mism = int((decoded != pt).any(axis=1).sum())
        return {"max_error": err_max, "average_error": err_sum / count, "mismatches": mism, "blocks": self.blocks}


def expand_key(key):
    """AES-128 key expansion (FIPS-197): the 176-byte schedule."""
    sbox = []
    for x in range(256):
        inv = 0
        for y in range(1, 256):
            a, b_, r = x, y, 0
            while b_:
                if b_ & 1:
                    r ^= a
                a = ((a << 1) ^ (0x1B if a & 0x80 else 0)) & 0xFF
                b_ >>= 1
            if r == 1:
                inv = y
                break
        v, out = inv, 0x63
        for _ in range(5):
            out ^= v
            v = ((v << 1) | (v >> 7)) & 0xFF
        sbox.append(out)
    w = list(key)
    rcon = 1
    for i in range(4, 44):
        t = w[4 * (i - 1): 4 * i]
        if i % 4 == 0:
            t = [sbox[t[1]] ^ rcon, sbox[t[2]], sbox[t[3]], sbox[t[0]]]
            rcon = ((rcon << 1) ^ (0x1B if rcon & 0x80 else 0)) & 0xFF
        w += [w[4 * (i - 4) + k] ^ t[k] for k in range(4)]
    return bytes(w)


# ------------------------------------------------------------------------------------------
# XBOOT S-box layer (the xboot15 chain's SubBytes: 16 instances)
# ------------------------------------------------------------------------------------------
XB_Q_BITS = [38, 36, 36, 37, 37, 37] + [38] * 11
XB_P_BITS = [38] * 5
XB_DNUM = 5


def xboot_bench(wg, torch, stream, timed, local, steps, with_cpu):
    """The XBOOT S-box (wg_xboot_sbox) on one SubBytes layer, 16 instances of 8 bit ciphertexts at
    level 5 of the xboot15 chain (N = 2^15, 17 Q + 5 P limbs, dnum 5; uniform residues, uniform
    relinearisation key of its shape); optionally one reference SubBytes layer (16 S-boxes
    side by side under OpenMP, the S-box restated in the harness on the reference's own
    operations) on the host cores."""
    N = 1 << 15
    p, q = wg.find_primes(XB_P_BITS, XB_Q_BITS, N)
    ctx = wg.Context(N, q, p, XB_DNUM, device=local)
    L, K = len(q), len(p)
    rng = np.random.default_rng(23)
    parts = ctx.parts(L - 1)
    col = np.tile(np.repeat(np.concatenate([q, p]).astype(np.uint64), N), 2 * parts)
    ctx.set_key(wg.WG_KEY_RELIN, (rng.integers(0, 1 << 62, col.size, dtype=np.uint64) % col).astype(np.uint64))
    level, scale, count = 5, 2.0 ** 37, 16
    qcol = torch.from_numpy(np.repeat(q[: level + 1], N).view(np.int64)).cuda()
    data = torch.randint(0, 1 << 62, (count, 8, 2, (level + 1) * N), dtype=torch.int64, device="cuda") % qcol
    bits = [[(data[i, k, 0], data[i, k, 1]) for k in range(8)] for i in range(count)]
    outs = [[(torch.empty((level + 1) * N, dtype=torch.int64, device="cuda"),
              torch.empty((level + 1) * N, dtype=torch.int64, device="cuda")) for _ in range(8)] for _ in range(count)]
    step = lambda: ctx.xboot_sbox(level, scale, bits, outs)
    step()
    l0 = wg.launch_count()
    ms = timed(step, steps)
    launches = (wg.launch_count() - l0) / steps
    ctx.set_ntt_fusion(0)  # the same layer with the separate launches around the NTTs
    step()
    unfused_ms = timed(step, steps)
    ctx.set_ntt_fusion(1)
    res = {"workload": "XBOOT S-box, one SubBytes layer: 16 instances of 8 bits at level 5 of the xboot15 chain "
                       "(255 monomials from 247 multiply+relin+rescale per instance, 8 integer combinations)",
           "ms_per_layer": ms, "sboxes_per_s": count / (ms / 1000.0),
           "launches_per_layer": launches, "output_level": level - 3,
           "unfused_ms_per_layer": unfused_ms, "fused_speedup": unfused_ms / ms}
    if with_cpu:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O

            if O.ref_available():
                R = O.RefXboot()
                qc = np.repeat(R.q[: level + 1], N)
                draw = lambda: (rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)
                one = [(draw(), draw()) for _ in range(8)]
                threads = os.cpu_count()
                t = R.sbox_layer_seconds(level, scale, one, count, threads)
                res["reference_cpu"] = {"s_per_subbytes_layer": t, "sboxes_per_s": count / t,
                                        "cores": threads, "kind": "reference",
                                        "sample": f"one SubBytes layer: {count} S-box instances on {threads} threads "
                                                  f"(OpenMP over instances, as the reference's SubBytes runs its "
                                                  f"16 byte positions), {t:.2f} s"}
        except Exception as e:  # reported, never required
            res["reference_cpu"] = {"unavailable": str(e)}
    return res


# ------------------------------------------------------------------------------------------
# XBOOT AES-CTR (xboot15-full: 16384 blocks per evaluation)
# ------------------------------------------------------------------------------------------
XBOOT_PLAN_PATH = os.path.join(ROOT, "tests", "golden", "xboot_plans.json")


class XbootAesRun:
    """Context, keys, bootstrap stages and encrypted round-key bits of one XBOOT N = 2^15 parameter
    set's shapes (uniform residues), and block bytes for every active slot."""

    def __init__(self, wg, torch, plan, device, seed):
        N = plan["ring_degree"]
        q = np.array(plan["q"], dtype=np.uint64)
        p = np.array(plan["p"], dtype=np.uint64)
        K = len(p)
        self.N, self.wg = N, wg
        self.ctx = ctx = wg.Context(N, q, p, plan["dnum"], device=device)
        rng = np.random.default_rng(seed)

        def residues(limb_mods, copies):
            col = np.tile(np.repeat(np.asarray(limb_mods, np.uint64), N), copies)
            return (rng.integers(0, 1 << 62, col.size, dtype=np.uint64) % col).astype(np.uint64)

        keys = plan["keys"]
        for name, kind in (("relin", wg.WG_KEY_RELIN), ("conj", wg.WG_KEY_CONJ),
                           ("sparse_to_dense", wg.WG_KEY_SPARSE_TO_DENSE)):
            k = keys[name]
            ctx.set_key(kind, residues(np.concatenate([q[: k["key_level"] + 1], p]), 2 * k["parts"]),
                        parts=k["parts"], key_level=k["key_level"])
        ctx.set_key(wg.WG_KEY_DENSE_TO_SPARSE, residues([q[0], p[0], q[0], p[0]], 1))
        rk = keys["rotation"]
        rkey = residues(np.concatenate([q[: rk["key_level"] + 1], p]), 2 * rk["parts"])
        for r in plan["rotations"]:
            ctx.set_key(wg.WG_KEY_ROTATION, rkey, rotation=int(r), parts=rk["parts"], key_level=rk["key_level"])

        def stages(spec):
            out = []
            for st in spec:
                level = st["qp_limbs"] - 1 - K
                d = residues(np.concatenate([q[: level + 1], p]), len(st["indices"]))
                out.append(wg.LtStage(ctx, level, st["indices"], d, st["baby"], st["slot_count"], st["rescale"]))
            return out

        self.s2c, self.c2s = stages(plan["s2c"]), stages(plan["c2s"])
        b = plan["bootstrap"]
        self.params = wg.BootstrapParams(b["s2c_depth"], b["depth"], b["evalmod_log_scale"], b["double_angle"],
                                         b["active_slots"], b["slots"], b["scale"])
        self.coeffs = np.asarray(plan["evalmod_coeffs"], dtype=np.float64)
        a = plan["aes"]
        self.klevels = np.asarray(a["key_levels"], dtype=np.int64)
        self.kscales = np.asarray(a["key_scales"], dtype=np.float64)
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        self.key_dev, self.key_bits = [], [None] * len(self.klevels)
        for lv in sorted(set(int(x) for x in self.klevels)):
            idx = [k for k in range(len(self.klevels)) if self.klevels[k] == lv]
            qcol = torch.from_numpy(np.repeat(q[: lv + 1], N).view(np.int64)).cuda()
            t = torch.randint(0, 1 << 62, (len(idx), 2, (lv + 1) * N), dtype=torch.int64, device="cuda",
                              generator=gen) % qcol
            self.key_dev.append(t)
            for j, k in enumerate(idx):
                self.key_bits[k] = (t[j, 0], t[j, 1])
        full = (b["depth"] + 1) * N
        self.out_dev = torch.zeros((128, 2, full), dtype=torch.int64, device="cuda")
        self.outs = [(self.out_dev[k, 0], self.out_dev[k, 1]) for k in range(128)]
        self.blocks = b["active_slots"]
        self.block_bytes = [bytes(rng.integers(0, 256, 16 * self.blocks, dtype=np.uint8)) for _ in range(3)]
        self.calls = 0

    def step(self, stream):
        c = self.block_bytes[self.calls % 3]
        x = self.block_bytes[(self.calls + 1) % 3]
        self.calls += 1
        return self.ctx.aes_ctr_xboot(self.params, self.s2c, self.c2s, self.coeffs, self.key_bits, self.kscales,
                                      self.klevels, c, x, self.blocks, self.outs, stream=stream)


def xboot_aes_bench(wg, torch, stream, timed, run, seed, steps, with_cpu, sbox_seconds=None):
    """AES-128-CTR with the XBOOT S-box (wg_aes_ctr_xboot) on xboot15-full: 16384 counter blocks
    per evaluation (every slot one block), ten rounds with 64 pair bootstraps after rounds 1..9
    and a final refresh.  Optionally one reference state refresh (64 pair bootstraps side by side
    under OpenMP) on the host cores, and an estimate of the reference's full evaluation from it
    and the SubBytes layer of the S-box section."""
    step = lambda: run.step(stream)
    step()
    l0 = wg.launch_count()
    ms = timed(step, steps)
    res = {"workload": "xboot15-full AES-128-CTR: 16384 counter blocks per evaluation (one block per slot), "
                       "XBOOT S-box on all 16 bytes per round, 64 pair bootstraps after rounds 1..9 and at the end",
           "shapes": "tests/golden/xboot_plans.json (the reference's xboot15 bootstrapping plan), uniform residues",
           "blocks": run.blocks, "ms_per_evaluation": ms, "blocks_per_s": run.blocks / (ms / 1000.0),
           "steps": steps, "launches_per_evaluation": (wg.launch_count() - l0) / steps,
           "pair_bootstraps_per_evaluation": 640, "sboxes_per_evaluation": 160}
    blocks = run.blocks
    torch.cuda.synchronize()
    if with_cpu:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O

            if O.ref_available():
                R = O.RefPlans(bootstrap_keys=True, preset="xboot15")
                lv, N = 2, R.N
                rng = np.random.default_rng(seed)
                qc = np.repeat(R.q[: lv + 1], N)
                draw = lambda: (rng.integers(0, 1 << 62, (lv + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)
                c0, c1 = (draw(), draw()), (draw(), draw())
                threads = os.cpu_count()
                tp = R.bootstrap_pair_layer_seconds(lv, R.scale, c0, c1, 64, threads)
                ref = {"s_per_refresh": tp, "cores": threads, "kind": "reference",
                       "sample": f"one state refresh: 64 pair bootstraps (ckks_batch_bootstrap_evalmod_inplace) on "
                                 f"{threads} threads (OpenMP over pairs, as the reference's refresh runs them), "
                                 f"{tp:.2f} s"}
                if sbox_seconds:
                    est = 10 * tp + 10 * sbox_seconds
                    ref.update({"estimated_s_per_evaluation": est, "estimated_blocks_per_s": blocks / est,
                                "estimate": "10 refreshes of 64 pairs + 10 SubBytes layers of 16 S-boxes at the "
                                            "timed layer times (its linear layers and XORs not counted, which "
                                            "favours the reference)"})
                res["reference_cpu"] = ref
        except Exception as e:  # reported, never required
            res["reference_cpu"] = {"unavailable": str(e)}
    return res


# ------------------------------------------------------------------------------------------
# served requests (config 5, walsh15 part): Poisson arrivals through the batching service
# ------------------------------------------------------------------------------------------
def serve_bench(wg, torch, aes, requests, seed, capacity_blocks, workers=2, window_ms=20.0, load=0.5):
    """Requests of log-uniform size in [2, 1024] blocks (even) arrive as a seeded Poisson stream
    at `load` x the full-slot capacity (the headline's measured blocks/s) in requests/s, are
    served by the continuous-batching service (wg_serve_*: `workers` concurrent evaluations,
    batching window) and timed from submission to completion."""
    rng = np.random.default_rng(seed)
    full = aes.out_dev.shape[2]
    srv = wg.Server(aes.ctx, aes.params, aes.s2c, aes.s2c_x2, aes.c2s, aes.coeffs, aes.pbc, aes.psc, aes.key_bits,
                    aes.kscales, aes.kl, workers=workers, batch_window_ms=window_ms)
    try:
        mk = lambda: [(torch.empty(full, dtype=torch.int64, device="cuda"),
                       torch.empty(full, dtype=torch.int64, device="cuda")) for _ in range(128)]
        # warm-up: one full evaluation per worker (worker streams, their scratch and caches)
        ids = [srv.submit(aes.block_bytes[0], aes.block_bytes[1], mk()) for _ in range(workers)]
        for i in ids:
            srv.wait(i)
        sizes = [2 * int(round(np.exp(rng.uniform(np.log(1), np.log(512))))) for _ in range(requests)]
        rate = load * capacity_blocks / float(np.mean(sizes))
        gaps = rng.exponential(1.0 / rate, requests)
        bufs = [mk() for _ in range(requests)]
        ids = []
        start = time.perf_counter()
        t = start
        for k, (n, gap) in enumerate(zip(sizes, gaps)):
            t += gap
            delay = t - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(aes.block_bytes[2][:16 * n], aes.block_bytes[3][:16 * n], bufs[k]))
        res = [srv.wait(i) for i in ids]
        wall = time.perf_counter() - start
    finally:
        srv.close()
    lat = np.array([r["latency_ms"] for r in res])
    queue = np.array([r["queue_ms"] for r in res])
    evaluations = sum(1.0 / r["batch_requests"] for r in res)
    return {"workload": f"{requests} requests, log-uniform 2..1024 blocks (even), Poisson arrivals at "
                        f"{load} x full-slot capacity; walsh15 alone (the mixed stream is serving_mix)",
            "workers": workers, "batch_window_ms": window_ms, "requests": requests, "blocks": int(sum(sizes)),
            "arrival_rate_per_s": rate, "offered_blocks_per_s": rate * float(np.mean(sizes)),
            "wall_s": wall, "blocks_per_s": sum(sizes) / wall,
            # blocks_per_s counts the final drain (the last requests' latency after the last
            # arrival); a server that keeps up shows flat latencies from the first quarter of the
            # stream to the last
            "arrival_span_s": float(np.sum(gaps)), "drain_s": wall - float(np.sum(gaps)),
            "latency_first_last_quarter_ms": [float(lat[: max(1, requests // 4)].mean()),
                                              float(lat[-max(1, requests // 4):].mean())],
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "mean": float(lat.mean()), "max": float(lat.max())},
            "queue_ms": {"p50": float(np.percentile(queue, 50)), "p99": float(np.percentile(queue, 99))},
            "evaluations": round(evaluations, 2), "requests_per_evaluation": requests / evaluations,
            "full_slot_capacity_blocks_per_s": capacity_blocks}


def keygen_bench(wg, torch, local, seed, with_cpu):
    """The client setup of xboot15 on the device: every switching key the bootstrapped AES uses
    (relinearisation, conjugation, the plan's rotations, both secret switches) generated from a
    seeded ternary secret, and the 1408 encrypted round-key bits; wall time of the host-synchronous
    calls.  Optionally the reference's encryption of the round-key bits on the host cores."""
    with open(XBOOT_PLAN_PATH) as f:
        plan = json.load(f)["xboot15"]
    N = plan["ring_degree"]
    q = np.array(plan["q"], dtype=np.uint64)
    p = np.array(plan["p"], dtype=np.uint64)
    ctx = wg.Context(N, q, p, plan["dnum"], device=local)
    rng = np.random.default_rng(seed)
    secret = np.zeros(N, np.int8)
    secret[rng.choice(N, 256, replace=False)] = rng.choice([-1, 1], 256).astype(np.int8)
    sparse = np.zeros(N, np.int8)
    sparse[rng.choice(N, 32, replace=False)] = rng.choice([-1, 1], 32).astype(np.int8)
    b = plan["bootstrap"]
    params = wg.BootstrapParams(b["s2c_depth"], b["depth"], b["evalmod_log_scale"], b["double_angle"],
                                b["active_slots"], b["slots"], b["scale"])
    full = (b["depth"] + 1) * N
    key_dev = torch.zeros((1408, 2, full), dtype=torch.int64, device="cuda")
    key_bits = [(key_dev[k, 0], key_dev[k, 1]) for k in range(1408)]
    ek = bytes(rng.integers(0, 256, 176, dtype=np.uint8))

    def keys(tag):
        ctx.keygen_switch_key(wg.WG_KEY_RELIN, 0, secret, seed=tag + 1)
        ctx.keygen_switch_key(wg.WG_KEY_CONJ, 0, secret, seed=tag + 2)
        for r in plan["rotations"]:
            ctx.keygen_switch_key(wg.WG_KEY_ROTATION, int(r), secret, seed=tag + 3)
        ctx.keygen_secret_switch(wg.WG_KEY_DENSE_TO_SPARSE, secret, sparse, seed=tag + 4)
        ctx.keygen_secret_switch(wg.WG_KEY_SPARSE_TO_DENSE, sparse, secret, seed=tag + 5)

    keys(0)  # warm-up (allocations, tables)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    keys(100)
    torch.cuda.synchronize()
    t_keys = time.perf_counter() - t0
    ctx.aes_xboot_encrypt_round_key_bits(params, ek, 4, secret, key_bits, seed=7)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.aes_xboot_encrypt_round_key_bits(params, ek, 4, secret, key_bits, seed=8)
    torch.cuda.synchronize()
    t_bits = time.perf_counter() - t0
    nkeys = len(plan["rotations"]) + 4
    res = {"workload": f"xboot15 client setup: {nkeys} switching keys (relinearisation, conjugation, "
                       f"{len(plan['rotations'])} rotations, both secret switches) and 1408 encrypted round-key bits",
           "keys_s": t_keys, "keys_per_s": nkeys / t_keys, "key_bits_s": t_bits}
    del key_dev, key_bits, ctx
    torch.cuda.synchronize()
    if with_cpu:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O

            if O.ref_available():
                t0 = time.perf_counter()
                R = O.RefPlans(bootstrap_keys=True, preset="xboot15")
                t_ctx = time.perf_counter() - t0
                t0 = time.perf_counter()
                R.xboot_key_bits(ek, 4)
                t_ref_bits = time.perf_counter() - t0
                res["reference_cpu"] = {"key_bits_s": t_ref_bits, "context_build_s": t_ctx, "cores": os.cpu_count(),
                                        "kind": "reference",
                                        "sample": "ckks_aes128_encrypt_expanded_round_key_bits (OpenMP) and the whole "
                                                  "xboot15 context build (keys, plans and EvalMod fit together)"}
        except Exception as e:  # reported, never required
            res["reference_cpu"] = {"unavailable": str(e)}
    return res


MIX_SETS = ("walsh15", "xboot15", "xboot15-sparse", "xboot14", "xboot14-sparse")
MIX_MAX_BLOCKS = {"walsh15": 1024, "xboot15": 16384, "xboot15-sparse": 1024, "xboot14": 8192, "xboot14-sparse": 1024}


def serve_mix_bench(wg, torch, aes, xruns, requests, seed, caps, eval_bytes, budget_frac=0.85, window_ms=20.0,
                    load=0.5):
    """Config 5's mixed stream over all five AES parameter sets: requests cycle through walsh15
    (log-uniform 2..1024 blocks, even), xboot15-full (1..16384), xboot15-sparse-1024 (1..1024),
    xboot14-full (1..8192) and xboot14-sparse-1024 (1..1024), arriving as one seeded Poisson
    stream whose offered work is `load` x the device in evaluation time (each request counted as
    one full evaluation of its set at the measured full-slot capacity).
    One continuous-batching server per set on the same device, keys resident, all admitted
    through one shared device-memory budget (budget_frac of the device memory left free once
    every set's keys, plans and request buffers are resident; each evaluation holds its measured
    working set, evaluation_bytes, and workers give their scratch back after each evaluation);
    the walsh15 server's streams have the highest scheduling priority, so its one-second
    evaluations are not queued behind the XBOOT ones."""
    rng = np.random.default_rng(seed)
    runs = dict(xruns, walsh15=aes)
    full = {k: r.out_dev.shape[2] for k, r in runs.items()}
    kinds = [MIX_SETS[k % len(MIX_SETS)] for k in range(requests)]
    sizes = []
    for kd in kinds:
        top = MIX_MAX_BLOCKS[kd] // (2 if kd == "walsh15" else 1)
        n = int(round(np.exp(rng.uniform(0.0, np.log(top)))))
        sizes.append(2 * n if kd == "walsh15" else n)
    # offered work in device time: a request can cost a whole evaluation of its set, whatever its
    # size (an XBOOT evaluation takes as long with 10 blocks as with 16384), so the arrival rate
    # is set from the sets' full-evaluation times rather than from blocks
    eval_s = {kd: MIX_MAX_BLOCKS[kd] / caps[kd] for kd in MIX_SETS}
    work = [eval_s[kd] for kd in kinds]
    mk = lambda n: [(torch.empty(n, dtype=torch.int64, device="cuda"), torch.empty(n, dtype=torch.int64, device="cuda"))
                    for _ in range(128)]
    # every request's output buffers first, then the budget: the device memory left over
    bufs = [mk(full[kd]) for kd in kinds]
    warm_bufs = {k: mk(full[k]) for k in runs}
    torch.cuda.synchronize()
    budget_bytes = budget_frac * torch.cuda.mem_get_info()[0]
    budget = wg.ServeBudget(int(budget_bytes))
    srv = {"walsh15": wg.Server(aes.ctx, aes.params, aes.s2c, aes.s2c_x2, aes.c2s, aes.coeffs, aes.pbc, aes.psc,
                                aes.key_bits, aes.kscales, aes.kl, workers=2, batch_window_ms=window_ms, priority=1,
                                budget=budget, eval_bytes=eval_bytes["walsh15"])}
    for k, r in xruns.items():
        srv[k] = wg.Server.xboot(r.ctx, r.params, r.s2c, r.c2s, r.coeffs, r.key_bits, r.kscales, r.klevels, workers=1,
                                 batch_window_ms=window_ms, budget=budget, eval_bytes=eval_bytes[k])
    try:
        warm = {k: srv[k].submit(runs[k].block_bytes[0][:32], runs[k].block_bytes[1][:32], warm_bufs[k]) for k in srv}
        for k, i in warm.items():
            srv[k].wait(i)
        rate = load / float(np.mean(work))
        gaps = rng.exponential(1.0 / rate, requests)
        ids = []
        start = time.perf_counter()
        t = start
        for k, (kd, n, gap) in enumerate(zip(kinds, sizes, gaps)):
            t += gap
            delay = t - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            src = runs[kd].block_bytes
            ids.append(srv[kd].submit(src[1][:16 * n], src[2][:16 * n], bufs[k]))
        res = [srv[kd].wait(i) for kd, i in zip(kinds, ids)]
        wall = time.perf_counter() - start
    finally:
        for v in srv.values():
            v.close()
        budget.close()
    offered = sum(sizes) / (sum(gaps) or 1.0)
    out = {"workload": f"{requests} requests cycling walsh15, xboot15-full, xboot15-sparse-1024, xboot14-full and "
                       f"xboot14-sparse-1024 (log-uniform sizes up to each set's slots), one Poisson stream at {load} "
                       f"x the device in evaluation time (each request counted as one full evaluation of its set); "
                       f"one server per set on the device, one shared "
                       f"device-memory budget of {budget_bytes / 2**30:.1f} GiB, walsh15 streams at the highest "
                       f"priority",
           "budget_gib": budget_bytes / 2**30, "evaluation_gib": {k: v / 2**30 for k, v in eval_bytes.items()},
           "evaluation_s": eval_s,
           "batch_window_ms": window_ms, "arrival_rate_per_s": rate, "wall_s": wall,
           "blocks_per_s": sum(sizes) / wall, "offered_blocks_per_s": offered}
    for kd in MIX_SETS:
        sel = [k for k in range(requests) if kinds[k] == kd]
        if not sel:
            continue
        lat = np.array([res[k]["latency_ms"] for k in sel])
        evaluations = sum(1.0 / res[k]["batch_requests"] for k in sel)
        out[kd] = {"requests": len(sel), "blocks": int(sum(sizes[k] for k in sel)),
                   "blocks_per_s": sum(sizes[k] for k in sel) / wall,
                   "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                  "max": float(lat.max())},
                   "requests_per_evaluation": len(sel) / evaluations,
                   "full_slot_capacity_blocks_per_s": caps[kd]}
    return out


def evaluation_capacity(run, stream, torch):
    """Full-slot blocks/s of one XBOOT evaluation (one warm-up, one timed)."""
    run.step(stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run.step(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return run.blocks / (e0.elapsed_time(e1) / 1000.0)


def evaluation_bytes(run, stream, torch):
    """Peak device bytes one evaluation of the run's context takes beyond its keys and plans:
    from a trimmed context, the largest drop of free device memory seen by a 2 ms poll during
    one evaluation, plus a quarter for what the poll misses; the admission estimate of the
    served mix.  The context is trimmed again afterwards."""
    run.ctx.trim(stream)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    low = [free0]
    done = threading.Event()

    def poll():
        while not done.is_set():
            low[0] = min(low[0], torch.cuda.mem_get_info()[0])
            time.sleep(0.002)

    th = threading.Thread(target=poll, daemon=True)
    th.start()
    run.step(stream)
    torch.cuda.synchronize()
    done.set()
    th.join()
    low[0] = min(low[0], torch.cuda.mem_get_info()[0])
    run.ctx.trim(stream)
    torch.cuda.synchronize()
    return int(1.25 * max(0, free0 - low[0]))


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
    stream = torch.cuda.current_stream()

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
        return max_over_ranks(e0.elapsed_time(e1) / k, dist)

    plan = load_plan()
    if args.no_aes:
        hbm = 6650.0
        try:
            hbm = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs", hbm))
        except (OSError, ValueError):
            pass
        prim = None if args.no_ntt else ntt_bench(wg, torch, stream, timed, local, 20, hbm)
        ops = bs = None
        if not args.no_ops:
            ops, octx, oq, op_ = ops_bench(args, wg, torch, stream, timed, rank, local)
            if not args.no_bsgs:
                bs = bsgs_bench(wg, octx, oq, op_, stream, timed, 2, args.warmup)
            del octx
        xaes = None
        if not args.no_xboot_aes:
            with open(XBOOT_PLAN_PATH) as f:
                xrun = XbootAesRun(wg, torch, json.load(f)["xboot15"], local, args.seed + 29 + rank)
            xaes = xboot_aes_bench(wg, torch, stream, timed, xrun, args.seed + 29 + rank, args.xboot_aes_steps, False)
            del xrun
        kg = None if args.no_keygen else keygen_bench(wg, torch, local, args.seed + 37 + rank, False)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": None, "unit": UNIT, "note": "--no-aes profiling run",
                              "primitives": prim, "batched_ops": ops, "bsgs": bs, "xboot_aes": xaes, "keygen": kg}),
                  flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    aes = AesRun(wg, torch, plan, local, args.seed + rank)
    N = aes.N
    aes_step = lambda: aes.step(stream)
    for _ in range(args.warmup):
        aes_step()
    # timed region: K evaluations, an event after each for the latency distribution
    barrier()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches0 = wg.launch_count()
    host0 = wg.host_stats()
    with ClockSampler(None if args.no_clocks else local) as clk:
        evs[0].record(stream)
        out_levels = out_scales = None
        for i in range(args.steps):
            out_levels, out_scales = aes_step()
            evs[i + 1].record(stream)
        barrier()
    launches = wg.launch_count() - launches0
    host1 = wg.host_stats()
    per_step = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    ms = max_over_ranks(evs[0].elapsed_time(evs[-1]) / args.steps, dist)
    value = aes.blocks * world / (ms / 1000.0)
    staged = (host1["stage_bytes"] - host0["stage_bytes"]) / args.steps
    # decrypt the last timed evaluation and check it against plain AES (outside the timing)
    correctness = aes.check(out_levels, out_scales)

    # the plain per-operation GPU path: the same circuit with every S-box instance and every
    # refresh bootstrap as its own call (the reference's call granularity), same output words
    aes_plain = None
    if not args.no_plain:
        ref_words = aes.out_dev.clone()
        aes.calls -= 1  # the same counter blocks as the last timed evaluation
        aes.step(stream, plain=True)
        torch.cuda.synchronize()
        same = bool(torch.equal(ref_words, aes.out_dev))
        plain_ms = timed(lambda: aes.step(stream, plain=True), max(1, args.steps // 4))
        aes_plain = {"value": aes.blocks * world / (plain_ms / 1000.0), "unit": UNIT, "ms_per_step": plain_ms,
                     "steps": max(1, args.steps // 4), "batched_over_plain": plain_ms / ms,
                     "same_output_words": same,
                     "path": "wg_aes_ctr_walsh_plain: 16 S-box calls per round and one bootstrap call per refresh "
                             "batch instead of one batched call each"}
    # the same evaluation with the key switches' ModUp / ModDown as separate launches
    aes_unfused = None
    if not args.no_plain:
        aes.ctx.set_ntt_fusion(False)
        aes_step()
        unfused_ms = timed(aes_step, max(1, args.steps // 4))
        aes.ctx.set_ntt_fusion(True)
        aes_unfused = {"value": aes.blocks * world / (unfused_ms / 1000.0), "unit": UNIT,
                       "ms_per_step": unfused_ms, "fused_speedup": unfused_ms / ms,
                       "path": "wg_aes_ctr_walsh with ModUp, ModDown, the rescale remainders, the combine "
                               "and the rescale finish as separate launches from the NTT phases "
                               "(wg_set_ntt_fusion 0)"}

    # end to end: the same call from host block bytes, plus the read-back of the 128 output
    # bit ciphertexts into pinned host memory, every step
    e2e = None
    if not args.no_e2e:
        full = aes.out_dev.shape[2]
        pinned = torch.empty((128, 2, full), dtype=torch.int64).pin_memory()
        d2h = [0]

        def e2e_step():
            lv, _ = aes_step()
            d2h[0] = 0
            for k in range(128):
                nb = (lv[k] + 1) * N * 8
                for j in range(2):
                    wg.memcpy_dtoh(pinned[k, j].data_ptr(), aes.out_dev[k, j], nb, stream=stream)
                d2h[0] += 2 * nb

        e2e_step()
        e2e_ms = timed(e2e_step, max(1, args.steps // 2))
        torch.cuda.synchronize()
        assert torch.equal(pinned[0, 0, :N], aes.out_dev[0, 0, :N].cpu())
        e2e = {"value": aes.blocks * world / (e2e_ms / 1000.0), "unit": UNIT, "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": int(2 * 16 * aes.blocks + staged), "d2h_bytes_per_step": int(d2h[0]),
               "h2d_detail": "counter and ciphertext blocks from host memory plus the slot encodings of their "
                             "bits staged by the library",
               "steps": max(1, args.steps // 2)}

    # per-kernel-class device time of one evaluation (CUDA events on the launch stream)
    kernels = {}
    for name, cls in ([] if args.no_probe else wg.KCLASS.items()):
        wg.probe_begin(cls, 65536)
        aes_step()
        torch.cuda.synchronize()
        n, kms, kbytes = wg.probe_end()
        kernels[name] = {"launches": n, "ms": kms, "bytes": kbytes}
    probed = sum(v["ms"] for v in kernels.values())
    for v in kernels.values():
        v["share"] = v["ms"] / probed if probed else None
        v["gbs"] = v["bytes"] / (v["ms"] * 1e6) if v["ms"] else None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    dom_name = max(kernels, key=lambda k: kernels[k]["ms"]) if kernels else "ntt"
    dom = kernels.get(dom_name, {"ms": 0.0, "launches": 0, "bytes": 0.0, "gbs": None})
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "ntt_phase_traffic.json")))
        if dom_name == "ntt" and dom["launches"]:
            traffic = tr["dram_traffic_over_algorithmic"] * dom["bytes"] / dom["launches"]
    except (OSError, ValueError, KeyError):
        pass
    ks = [kernels[k] for k in ("modup", "keymac", "moddown") if k in kernels]
    ks_ms, ks_bytes = sum(v["ms"] for v in ks), sum(v["bytes"] for v in ks)
    roofline = {"kernel": dom_name, "bound": "hbm", "achieved": dom["gbs"], "peak": hbm, "unit": "GB/s",
                "frac": dom["gbs"] / hbm if dom["gbs"] else None, "traffic": traffic,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "avg_launch_us": 1000 * dom["ms"] / max(1, dom["launches"]),
                "bytes_per_launch": dom["bytes"] / max(1, dom["launches"]),
                "keyswitch_kernels": {"gbs": ks_bytes / (ks_ms * 1e6) if ks_ms else None,
                                      "classes": "modup + key inner product + moddown, bytes each kernel "
                                                 "reads and writes (intermediates included)"}}

    prim = None if args.no_ntt else ntt_bench(wg, torch, stream, timed, local, 20, hbm)
    if prim and rank == 0 and world == 1 and not args.no_cpu_baseline:
        prim["config1"]["reference_cpu"] = ref_config1_sample()
    serving = None if args.no_serve else serve_bench(wg, torch, aes, args.serve_requests, args.seed + 17 + rank,
                                                     aes.blocks / (ms / 1000.0))
    xboot = None if args.no_xboot else xboot_bench(wg, torch, stream, timed, local, 5,
                                                     rank == 0 and world == 1 and not args.no_cpu_baseline)
    xboot_aes, serving_mix = None, None
    if not args.no_xboot_aes:
        sbox_s = ((xboot or {}).get("reference_cpu") or {}).get("s_per_subbytes_layer")
        with open(XBOOT_PLAN_PATH) as f:
            xrun = XbootAesRun(wg, torch, json.load(f)["xboot15"], local, args.seed + 29 + rank)
        xboot_aes = xboot_aes_bench(wg, torch, stream, timed, xrun, args.seed + 29 + rank, args.xboot_aes_steps,
                                    rank == 0 and world == 1 and not args.no_cpu_baseline, sbox_s)
        if not args.no_serve:
            xruns = {"xboot15": xrun}
            caps = {"walsh15": aes.blocks / (ms / 1000.0), "xboot15": xboot_aes["blocks_per_s"]}
            # every set's keys and plans resident, no evaluation scratch held between sections
            eval_bytes = {"walsh15": evaluation_bytes(aes, stream, torch),
                          "xboot15": evaluation_bytes(xrun, stream, torch)}
            with open(XBOOT_PLAN_PATH) as f:
                xplans = json.load(f)
            for name, key in (("xboot15-sparse", "xboot15-sparse"), ("xboot14", "xboot14"),
                              ("xboot14-sparse", "xboot14-sparse")):
                xruns[name] = XbootAesRun(wg, torch, xplans[key], local, args.seed + 41 + rank)
                caps[name] = evaluation_capacity(xruns[name], stream, torch)
                eval_bytes[name] = evaluation_bytes(xruns[name], stream, torch)
            serving_mix = serve_mix_bench(wg, torch, aes, xruns, args.serve_mix_requests, args.seed + 31 + rank,
                                          caps, eval_bytes)
            del xruns
        del xrun
        torch.cuda.synchronize()
    keygen = None
    if not args.no_keygen:
        try:
            keygen = keygen_bench(wg, torch, local, args.seed + 37 + rank,
                                  rank == 0 and world == 1 and not args.no_cpu_baseline)
        except Exception as e:  # a side section: reported, never fatal for the headline
            keygen = {"error": str(e)}
    ops, ops_ctx = None, None
    if not args.no_ops:
        ops, ops_ctx, q, p = ops_bench(args, wg, torch, stream, timed, rank, local,
                                       rank == 0 and world == 1 and not args.no_cpu_baseline)
    bsgs = None
    if not args.no_bsgs:
        if ops_ctx is None:
            p, q = wg.find_primes(P_BITS, Q_BITS, N)
            ops_ctx = wg.Context(N, q, p, DNUM, device=local)
        bsgs = bsgs_bench(wg, ops_ctx, q, p, stream, timed, 10, args.warmup,
                          rank == 0 and world == 1 and not args.no_cpu_baseline)
    if ops:
        # key switching against HBM: the batched mul + relin + rescale + rotate pipeline (two key
        # switches per ciphertext) at its compulsory bytes over the graph-replay time
        roofline["keyswitch"] = {"achieved": ops["algorithmic_gbs"], "peak": hbm, "unit": "GB/s",
                                 "frac": ops["algorithmic_gbs"] / hbm,
                                 "workload": "batched_ops (relin + rotation key switches dominate)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline()
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "unavailable", "sample": str(e)}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    per_sorted = sorted(per_step)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "ring_degree": N, "q_limbs": len(plan["q"]), "p_limbs": len(plan["p"]),
                   "dnum": plan["dnum"], "blocks_per_step": aes.blocks, "rounds": ROUNDS,
                   "keys": "made on the device from a seeded ternary secret (h = 256) and sparse secret (h = 32): "
                           f"{len(aes.rotations)} rotation keys, relin, conj, dense-to-sparse, sparse-to-dense",
                   "plans": "SlotToCoeff (x1, x2) and CoeffToSlot generated by the library (wg_dft_plan_create), "
                            "EvalMod series by wg_evalmod_fit, key bits of a seeded AES key encrypted on the device",
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2: 2.2 GB of encrypted key bits and 1.7 GB of rotation keys per step",
                   "step": "one wg_aes_ctr_walsh call on device-resident keys with host counter blocks"},
        "latency_ms": {"mean": float(np.mean(per_step)), "p50": per_sorted[len(per_sorted) // 2],
                       "p99": per_sorted[min(len(per_sorted) - 1, int(0.99 * len(per_sorted)))],
                       "min": per_sorted[0], "max": per_sorted[-1]},
        "clocks": clk.summary(),
        "e2e": e2e,
        "gpu_launches": int(launches),
        "output_levels": sorted(set(int(x) for x in out_levels)) if out_levels else None,
        "roofline": roofline,
        "kernels": kernels,
        "primitives": prim,
        "serving": serving,
        "xboot_sbox": xboot,
        "xboot_aes": xboot_aes,
        "serving_mix": serving_mix,
        "keygen": keygen,
        "batched_ops": ops,
        "bsgs": bsgs,
        "aes_plain": aes_plain,
        "aes_unfused_keyswitch": aes_unfused,
        "cpu_baseline": cpu,
    }
    line["correctness"] = dict(correctness, reference_result=REFERENCE_RESULT)
    line["summary"] = summary_keys(line)
    print(json.dumps(line), flush=True)


# The reference's own RESULT line for this workload (aes_bench walsh15 on 8 host cores).
REFERENCE_RESULT = {"seconds": 210.037, "max_error": 1.083466e-05, "average_error": 2.766340e-07, "mismatches": 0,
                    "cores": 8}


def summary_keys(line):
    """The headline figures and the device-over-reference ratio of every section in one short
    record at the end of the line (the part of the output that survives a truncated log)."""
    def ratio(dev, ref):
        try:
            return float(dev) / float(ref) if dev and ref else None
        except (TypeError, ValueError):
            return None

    def get(d, *path):
        for k in path:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    out = {"blocks_per_s": line["value"], "e2e_blocks_per_s": get(line, "e2e", "value"),
           "ntt_frac_of_hbm": get(line, "roofline", "frac"),
           "max_error": get(line, "correctness", "max_error"),
           "average_error": get(line, "correctness", "average_error"),
           "mismatches": get(line, "correctness", "mismatches")}
    cpu = line.get("cpu_baseline") or {}
    out["aes_vs_reference_cpu"] = ratio(line["value"], cpu.get("value"))
    c1 = get(line, "primitives", "config1") or {}
    r1 = c1.get("reference_cpu") or {}
    out["config1_ntt_fwd_vs_reference"] = ratio(r1.get("forward_us"), c1.get("forward_us"))
    out["config1_rotation_vs_reference"] = ratio(r1.get("rotation_us"), c1.get("rotation_us"))
    ops = line.get("batched_ops") or {}
    out["config2_graph_vs_reference"] = ratio(get(ops, "batched_graph", "value"), get(ops, "reference_cpu", "value"))
    out["config2_graph_vs_plain_gpu"] = ops.get("batched_over_plain")
    bs = line.get("bsgs") or {}
    out["config3_c2s_vs_reference"] = ratio(get(bs, "coeff_to_slot", "ciphertexts_per_s"),
                                           get(bs, "reference_cpu", "coeff_to_slot", "ciphertexts_per_s"))
    out["config3_s2c_vs_reference"] = ratio(get(bs, "slot_to_coeff", "ciphertexts_per_s"),
                                           get(bs, "reference_cpu", "slot_to_coeff", "ciphertexts_per_s"))
    xa = line.get("xboot_aes") or {}
    out["xboot_aes_vs_reference"] = ratio(xa.get("blocks_per_s"),
                                          get(xa, "reference_cpu", "estimated_blocks_per_s"))
    pl = line.get("aes_plain") or {}
    out["aes_batched_vs_plain_gpu"] = pl.get("batched_over_plain")
    out["aes_fused_vs_unfused_keyswitch"] = get(line, "aes_unfused_keyswitch", "fused_speedup")
    out["config2_fused_vs_unfused_keyswitch"] = get(ops, "batched_nograph_unfused_keyswitch", "fused_speedup")
    return out


if __name__ == "__main__":
    main()
