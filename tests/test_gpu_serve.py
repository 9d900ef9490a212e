"""The continuous-batching AES-CTR service (wg_serve_*) on the walsh15 bootstrapping context with
the reference's own keys and encrypted round-key bits.

A 6-block request is served alone, then again inside a mix that arrives within the server's
batching window: a 20-block
request and the same 6-block request share one evaluation, while a 1000-block request, which no
longer fits beside them, runs on the second worker at the same time.  Every request's output bit
ciphertexts must decrypt to its CTR plaintext with 0 mismatched bits against plain AES-128, the
6-block request must decrypt to the same bits alone and in the mix, and the two evaluations of
the mix must overlap in time."""
import numpy as np
import pytest

from aes_util import encrypt_block, expand_key

pytestmark = pytest.mark.gpu


def _request(rng, ek, blocks):
    counters = bytes(rng.integers(0, 256, 16 * blocks, dtype=np.uint8))
    plain = bytes(rng.integers(0, 256, 16 * blocks, dtype=np.uint8))
    stream = b"".join(encrypt_block(ek, counters[16 * i:16 * i + 16]) for i in range(blocks))
    return counters, bytes(x ^ y for x, y in zip(plain, stream)), plain


def _decrypt_bits(wg, R, outs, res, blocks):
    """bits[b][bit] of the request's blocks from its output ciphertexts."""
    N = R.N
    acb, off = res["active_blocks"], res["block_offset"]
    bits = np.zeros((blocks, 128), dtype=np.int64)
    for bit in range(128):
        lv, sc = res["levels"][bit], res["scales"][bit]
        m = (lv + 1) * N
        z = R.decrypt(lv, sc, wg.to_host(outs[bit][0])[:m], wg.to_host(outs[bit][1])[:m])
        for b in range(blocks):
            e = off + b
            bits[b, bit] = int(round(z[e].real if e < acb else z[e - acb].imag))
    return bits


def _plain_bits(plain, blocks):
    return np.array([[(plain[16 * b + bit // 8] >> (bit % 8)) & 1 for bit in range(128)] for b in range(blocks)])


@pytest.fixture(scope="module")
def walsh15_service(wg, ref_mod):
    """The reference walsh15 context's keys, plans and encrypted key bits on the device."""
    import torch

    R = ref_mod.RefPlans(bootstrap_keys=True)
    info = R.bts_info()
    N, K = R.N, len(R.p)
    rng = np.random.default_rng(77)
    ek = expand_key(bytes(rng.integers(0, 256, 16, dtype=np.uint8)))
    kflat, kscales, kl = R.aes_key_bits(ek, 512)

    ctx = wg.Context(N, R.q, R.p, R.dnum)
    for kind, wkind in ((2, wg.WG_KEY_RELIN), (1, wg.WG_KEY_CONJ), (4, wg.WG_KEY_SPARSE_TO_DENSE)):
        k, parts, lv = R.key(0, kind=kind)
        ctx.set_key(wkind, k, parts=parts, key_level=lv)
    ctx.set_key(wg.WG_KEY_DENSE_TO_SPARSE, R.key(0, kind=3)[0])
    for r in R.rotations():
        k, parts, lv = R.key(int(r))
        ctx.set_key(wg.WG_KEY_ROTATION, k, rotation=int(r), parts=parts, key_level=lv)
    x2 = R.build_scaled_s2c(2)

    def stages(which):
        out = []
        for k in range(R.stages(which)):
            st = R.stage(which, k)
            out.append(wg.LtStage(ctx, st["qp_limbs"] - 1 - K, st["indices"], st["diagonals"], st["baby"],
                                  st["slot_count"], st["rescale"]))
        return out

    s2c, s2c2, c2s = stages(0), stages(x2), stages(1)
    params = wg.BootstrapParams(info["s2c_depth"], info["depth"], info["evalmod_log_scale"], info["double_angle"],
                                info["active_slots"], info["slots"], info["scale"])
    n = (kl + 1) * N
    dev = torch.from_numpy(kflat.view(np.int64)).cuda().view(1408, 2, n)
    key_bits = [(dev[k, 0], dev[k, 1]) for k in range(1408)]
    full = (info["depth"] + 1) * N
    mk = lambda: [(torch.zeros(full, dtype=torch.int64, device="cuda"),
                   torch.zeros(full, dtype=torch.int64, device="cuda")) for _ in range(128)]
    return dict(R=R, rng=rng, ek=ek, ctx=ctx, params=params, s2c=s2c, s2c2=s2c2, c2s=c2s, coeffs=info["coeffs"],
                key_bits=key_bits, kscales=kscales, kl=kl, mk=mk)


def test_served_requests_alone_and_in_a_mix(wg, walsh15_service):
    S = walsh15_service
    R, rng, ek, mk = S["R"], S["rng"], S["ek"], S["mk"]
    # a 300 ms batching window: requests queued within it share an evaluation when they fit
    srv = wg.Server(S["ctx"], S["params"], S["s2c"], S["s2c2"], S["c2s"], S["coeffs"], 512, 32, S["key_bits"],
                    S["kscales"], S["kl"], workers=2, batch_window_ms=300.0)
    try:
        a_ctr, a_ct, a_plain = _request(rng, ek, 6)
        b_ctr, b_ct, b_plain = _request(rng, ek, 20)
        c_ctr, c_ct, c_plain = _request(rng, ek, 1000)

        outs_alone = mk()
        res_alone = srv.wait(srv.submit(a_ctr, a_ct, outs_alone), timeout=600)
        assert res_alone["batch_requests"] == 1 and res_alone["active_blocks"] == 512
        alone = _decrypt_bits(wg, R, outs_alone, res_alone, 6)
        assert (alone == _plain_bits(a_plain, 6)).all()

        ob, oa, oc = mk(), mk(), mk()
        ib = srv.submit(b_ctr, b_ct, ob)
        ia = srv.submit(a_ctr, a_ct, oa)
        ic = srv.submit(c_ctr, c_ct, oc)
        rb, ra, rc = srv.wait(ib, 600), srv.wait(ia, 600), srv.wait(ic, 600)
        # B and A share the first evaluation (A after B's 20 blocks); C runs on the other worker
        assert (rb["batch_requests"], rb["block_offset"]) == (2, 0)
        assert (ra["batch_requests"], ra["block_offset"], ra["active_blocks"]) == (2, 20, 512)
        assert (rc["batch_requests"], rc["block_offset"], rc["active_blocks"]) == (1, 0, 512)
        # the two evaluations overlapped: C started before B's evaluation finished
        assert rc["queue_ms"] < rb["latency_ms"]
        mixed = _decrypt_bits(wg, R, oa, ra, 6)
        assert (mixed == alone).all()
        assert (_decrypt_bits(wg, R, ob, rb, 20) == _plain_bits(b_plain, 20)).all()
        assert (_decrypt_bits(wg, R, oc, rc, 1000) == _plain_bits(c_plain, 1000)).all()
        print(f"alone {res_alone['latency_ms']:.0f} ms; mix: B {rb['latency_ms']:.0f} ms, A {ra['latency_ms']:.0f} ms, "
              f"C {rc['latency_ms']:.0f} ms (queued {rc['queue_ms']:.0f} ms)")
    finally:
        srv.close()


def test_servers_sharing_a_budget(wg, walsh15_service):
    """Two servers on one device (one at the highest stream priority) share a device-memory
    budget that admits one evaluation at a time: their evaluations run one after the other, and
    each request still decrypts to its plaintext."""
    S = walsh15_service
    R, rng, ek, mk = S["R"], S["rng"], S["ek"], S["mk"]
    budget = wg.ServeBudget(1 << 30)
    args = (S["ctx"], S["params"], S["s2c"], S["s2c2"], S["c2s"], S["coeffs"], 512, 32, S["key_bits"], S["kscales"],
            S["kl"])
    hi = wg.Server(*args, workers=1, priority=1, budget=budget, eval_bytes=1 << 30)
    lo = wg.Server(*args, workers=1, priority=0, budget=budget, eval_bytes=1 << 30)
    try:
        x_ctr, x_ct, x_plain = _request(rng, ek, 8)
        y_ctr, y_ct, y_plain = _request(rng, ek, 10)
        ox, oy = mk(), mk()
        ix = lo.submit(x_ctr, x_ct, ox)
        iy = hi.submit(y_ctr, y_ct, oy)
        rx, ry = lo.wait(ix, 600), hi.wait(iy, 600)
        first, second = (rx, ry) if rx["queue_ms"] <= ry["queue_ms"] else (ry, rx)
        # the second evaluation started only after the first had released the budget
        assert second["queue_ms"] >= first["latency_ms"] - 50.0
        assert (_decrypt_bits(wg, R, ox, rx, 8) == _plain_bits(x_plain, 8)).all()
        assert (_decrypt_bits(wg, R, oy, ry, 10) == _plain_bits(y_plain, 10)).all()
    finally:
        hi.close()
        lo.close()
        budget.close()
