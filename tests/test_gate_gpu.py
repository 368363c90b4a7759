"""GPU parity of the torus-32 gate bootstrap (FP64 FFT blind rotation, sample extract, key
switch) against the exact-integer oracle, through the C ABI: the extracted LWE and the
key-switched output are bit-exact; every gate's truth table; 64 random NAND gates."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_oracle
from gate_harness import TRUTH, OracleGate, declare_gate, decrypt

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.fixture(scope="module")
def gctx(pkg):
    c = pkg.GateContext(max_batch=256)
    c.keygen(11)
    yield c
    c.close()


@pytest.fixture(scope="module")
def gkeys(gctx):
    return gctx.export_keys()


def _bootstrap(pkg, ctx, a, b):
    p = ctx.params
    cnt = len(b)
    da, db = _dev(a), _dev(b)
    ext = torch.zeros((cnt, p.N + 1), dtype=torch.int32, device="cuda")
    oa = torch.zeros((cnt, p.n), dtype=torch.int32, device="cuda")
    ob = torch.zeros(cnt, dtype=torch.int32, device="cuda")
    pkg.call("cbs_gate_bootstrap_batch_device", ctx.handle, da.data_ptr(), db.data_ptr(), cnt, ext.data_ptr(),
             oa.data_ptr(), ob.data_ptr(), None)
    torch.cuda.synchronize()
    return _host(ext), _host(oa), _host(ob)


def test_keys_match_host_generation(pkg, gctx, gkeys):
    again = pkg.gate_generate_keys_host(gctx.params, 11)
    for k in gkeys:
        assert np.array_equal(gkeys[k], again[k])


def test_bootstrap_bit_exact(pkg, gctx, gkeys):
    p = gctx.params
    a, b = gctx.encrypt([1, 0, 1, 0], seed=3)
    ext, oa, ob = _bootstrap(pkg, gctx, a, b)
    og = OracleGate(declare_gate(load_oracle()), p, gkeys)
    want = og.blind_rotate(a, b)
    assert np.array_equal(ext, want)
    wa, wb = og.keyswitch(ext)
    assert np.array_equal(oa, wa) and np.array_equal(ob, wb)
    assert list(gctx.decrypt(oa, ob)) == [1, 0, 1, 0]


@pytest.mark.parametrize("gate", range(6))
def test_gate_truth_table(pkg, gctx, gate):
    p = gctx.params
    x = np.array([0, 0, 1, 1] * 2, np.uint8)
    y = np.array([0, 1, 0, 1] * 2, np.uint8)
    a1, b1 = gctx.encrypt(x, seed=100 + gate)
    a2, b2 = gctx.encrypt(y, seed=200 + gate)
    d = [_dev(v) for v in (a1, b1, a2, b2)]
    oa = torch.zeros((len(x), p.n), dtype=torch.int32, device="cuda")
    ob = torch.zeros(len(x), dtype=torch.int32, device="cuda")
    pkg.call("cbs_gate_eval_batch_device", gctx.handle, gate, *(t.data_ptr() for t in d), len(x), oa.data_ptr(),
             ob.data_ptr(), None)
    torch.cuda.synchronize()
    got = gctx.decrypt(_host(oa), _host(ob))
    assert list(got) == [TRUTH[gate](int(u), int(v)) for u, v in zip(x, y)]


def test_64_nand_gates_and_chaining(pkg, gctx):
    """64 independent NAND gates on uniform random bits, then a second layer fed by the first
    layer's outputs (bootstrapped ciphertexts are valid gate inputs)."""
    p = gctx.params
    rng = np.random.default_rng(64)
    x = rng.integers(0, 2, 64).astype(np.uint8)
    y = rng.integers(0, 2, 64).astype(np.uint8)
    a1, b1 = gctx.encrypt(x, seed=7)
    a2, b2 = gctx.encrypt(y, seed=8)
    d = [_dev(v) for v in (a1, b1, a2, b2)]
    oa = torch.zeros((64, p.n), dtype=torch.int32, device="cuda")
    ob = torch.zeros(64, dtype=torch.int32, device="cuda")
    pkg.call("cbs_gate_eval_batch_device", gctx.handle, 3, *(t.data_ptr() for t in d), 64, oa.data_ptr(),
             ob.data_ptr(), None)
    torch.cuda.synchronize()
    z = gctx.decrypt(_host(oa), _host(ob))
    assert np.array_equal(z, 1 - (x & y))
    # second layer: NAND(z_i, z_(i+1))
    a3 = oa.clone()
    b3 = ob.clone()
    a4 = torch.roll(oa, -1, 0).contiguous()
    b4 = torch.roll(ob, -1, 0).contiguous()
    oa2 = torch.zeros_like(oa)
    ob2 = torch.zeros_like(ob)
    pkg.call("cbs_gate_eval_batch_device", gctx.handle, 3, a3.data_ptr(), b3.data_ptr(), a4.data_ptr(),
             b4.data_ptr(), 64, oa2.data_ptr(), ob2.data_ptr(), None)
    torch.cuda.synchronize()
    assert np.array_equal(gctx.decrypt(_host(oa2), _host(ob2)), 1 - (z & np.roll(z, -1)))


def test_n2048_bit_exact(pkg):
    p = pkg.gate_default_params()
    p.N, p.n = 2048, 40
    ctx = pkg.GateContext(p, max_batch=4)
    ctx.keygen(12)
    keys = ctx.export_keys()
    a, b = ctx.encrypt([0, 1, 1], seed=9)
    ext, oa, ob = _bootstrap(pkg, ctx, a, b)
    og = OracleGate(declare_gate(load_oracle()), p, keys)
    assert np.array_equal(ext, og.blind_rotate(a, b))
    wa, wb = og.keyswitch(ext)
    assert np.array_equal(oa, wa) and np.array_equal(ob, wb)
    assert list(decrypt(keys["s_lwe"], oa, ob)) == [0, 1, 1]
    ctx.close()


def test_argument_checks(pkg, gctx):
    p = gctx.params
    a, b = gctx.encrypt([1], seed=1)
    da, db = _dev(a), _dev(b)
    out_a = torch.zeros((1, p.n), dtype=torch.int32, device="cuda")
    out_b = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib = pkg.load()
    st = lib.cbs_gate_eval_batch_device(gctx.handle, 9, da.data_ptr(), db.data_ptr(), da.data_ptr(), db.data_ptr(), 1,
                                        out_a.data_ptr(), out_b.data_ptr(), None)
    assert st == 1
    st = lib.cbs_gate_bootstrap_batch_device(gctx.handle, da.data_ptr(), db.data_ptr(), 1000, None, out_a.data_ptr(),
                                             out_b.data_ptr(), None)
    assert st == 2  # above max_batch


def test_ragged_two_parameter_sets_in_one_graph(pkg):
    """Requests of uneven size over two parameter sets (N=1024/n=636, N=2048/n=630), planned
    once and replayed from one captured CUDA graph: outputs equal the per-request launches
    bit for bit and decrypt to the input bits."""
    pa = pkg.gate_default_params()
    pb = pkg.gate_default_params()
    pb.N, pb.n = 2048, 630
    ctxs = [pkg.GateContext(pa, max_batch=64), pkg.GateContext(pb, max_batch=64)]
    for i, c in enumerate(ctxs):
        c.keygen(40 + i)
    sizes = [[1, 17, 5], [3, 33]]
    rng = np.random.default_rng(5)
    reqs, want = [[], []], []
    keep = []
    for i, c in enumerate(ctxs):
        for cnt in sizes[i]:
            bits = rng.integers(0, 2, cnt).astype(np.uint8)
            a, b = c.encrypt(bits, seed=int(rng.integers(1 << 30)))
            da, db = _dev(a), _dev(b)
            oa = torch.zeros((cnt, c.params.n), dtype=torch.int32, device="cuda")
            ob = torch.zeros(cnt, dtype=torch.int32, device="cuda")
            keep += [da, db, oa, ob]
            reqs[i].append((da.data_ptr(), db.data_ptr(), oa.data_ptr(), ob.data_ptr(), cnt))
            # per-request launch for comparison
            ra = torch.zeros_like(oa)
            rb = torch.zeros_like(ob)
            pkg.call("cbs_gate_bootstrap_batch_device", c.handle, da.data_ptr(), db.data_ptr(), cnt, None,
                     ra.data_ptr(), rb.data_ptr(), None)
            want.append((i, bits, oa, ob, ra, rb))
    ctxs[0].ragged_plan(reqs[0], grid_ctas=0)
    grid, ms = ctxs[0].ragged_autotune()  # the product's tile choice for set 0's plan
    assert grid >= 1 and ms > 0
    ctxs[1].ragged_plan(reqs[1], grid_ctas=3)  # fewer CTAs than ciphertexts: CTAs loop
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.graph(g):
        main = torch.cuda.current_stream()
        side.wait_stream(main)
        ctxs[0].ragged_launch(main.cuda_stream)
        with torch.cuda.stream(side):
            ctxs[1].ragged_launch(side.cuda_stream)
        main.wait_stream(side)
    for _ in range(2):
        for (_, _, oa, ob, _, _) in want:
            oa.zero_()
            ob.zero_()
        g.replay()
        torch.cuda.synchronize()
        for (i, bits, oa, ob, ra, rb) in want:
            assert torch.equal(oa, ra) and torch.equal(ob, rb)
            assert np.array_equal(ctxs[i].decrypt(_host(oa), _host(ob)), bits)
    del g
    for c in ctxs:
        c.close()


@pytest.mark.parametrize("mb", [2, 3])
def test_multibit_bootstrap_bit_exact(pkg, gctx, gkeys, mb):
    """Grouped (multi-bit) gate blind rotation against the oracle's exact grouped rotation with
    the same keys: the products stay below 2^52, so the FP64 result rounds to the exact one."""
    p = gctx.params
    gctx.set_multibit(mb)
    try:
        mbk = gctx.export_mb_bsk()
        a, b = gctx.encrypt([1, 0, 1, 1], seed=40 + mb)
        ext, oa, ob = _bootstrap(pkg, gctx, a, b)
    finally:
        gctx.set_multibit(1)
    og = OracleGate(declare_gate(load_oracle()), p, gkeys)
    want = og.blind_rotate_mb(a, b, mbk, mb)
    assert np.array_equal(ext, want)
    wa, wb = og.keyswitch(want)
    assert np.array_equal(oa, wa) and np.array_equal(ob, wb)


def test_multibit_nand_truth_table(pkg, gctx, gkeys):
    p = gctx.params
    rng = np.random.default_rng(12)
    x = rng.integers(0, 2, 64).astype(np.uint8)
    y = rng.integers(0, 2, 64).astype(np.uint8)
    a1, b1 = gctx.encrypt(x, seed=13)
    a2, b2 = gctx.encrypt(y, seed=14)
    gctx.set_multibit(2)
    try:
        da1, db1, da2, db2 = _dev(a1), _dev(b1), _dev(a2), _dev(b2)
        oa = torch.zeros((64, p.n), dtype=torch.int32, device="cuda")
        ob = torch.zeros(64, dtype=torch.int32, device="cuda")
        pkg.call("cbs_gate_eval_batch_device", gctx.handle, pkg.GATE_NAND, da1.data_ptr(), db1.data_ptr(),
                 da2.data_ptr(), db2.data_ptr(), 64, oa.data_ptr(), ob.data_ptr(), None)
        torch.cuda.synchronize()
    finally:
        gctx.set_multibit(1)
    assert np.array_equal(gctx.decrypt(_host(oa), _host(ob)), 1 - (x & y))
