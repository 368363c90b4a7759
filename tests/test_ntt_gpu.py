"""GPU parity: the Phantom 1-D NTT entry points through the C ABI vs the CPU oracle,
bit-exact, including odd batch sizes and the permute/out-of-place variants."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import oracle_primes, oracle_tables, rand_mod

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a: np.ndarray):
    return torch.from_numpy(a.view(np.int64)).cuda()


def _host(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


class Tabs:
    def __init__(self, oracle, n, q):
        self.n, self.q = n, q
        self.rp, self.rps, self.irp, self.irps, self.ninv = oracle_tables(oracle, n, q)
        self.d = {k: _dev(v) for k, v in dict(rp=self.rp, rps=self.rps, irp=self.irp, irps=self.irps,
                                              ninv=self.ninv[:1].copy(), ninvs=self.ninv[1:].copy()).items()}
        r = np.zeros(3, np.uint64)
        r[0] = q
        self.dmod = _dev(r)  # const_ratio unused by these kernels

    def p(self, k):
        return self.d[k].data_ptr()


CASES = [(1024, 50, 1), (2048, 54, 1), (4096, 50, 3)]


@pytest.mark.parametrize("n,bits,nprimes", CASES)
@pytest.mark.parametrize("batch", [1, 3, 17, 300])
def test_forward_inverse_bit_exact(lib, oracle, n, bits, nprimes, batch):
    for q in oracle_primes(oracle, n, bits, nprimes):
        t = Tabs(oracle, n, q)
        rng = np.random.default_rng(n + batch)
        a = rand_mod(rng, q, (batch, n))
        d = _dev(a.copy())
        assert lib.cbs_fnwt_1d_opt_batched(d.data_ptr(), t.p("rp"), t.p("rps"), t.dmod.data_ptr(), n, batch, None) == 0
        torch.cuda.synchronize()
        want = a.copy()
        oracle.orc_ntt_forward(want, batch, n, q, t.rp)
        assert (_host(d) == want).all()
        out = torch.empty_like(d)
        assert lib.cbs_inwt_1d_opt_outofplace_batched(out.data_ptr(), d.data_ptr(), t.p("irp"), t.p("irps"),
                                                      t.dmod.data_ptr(), t.p("ninv"), t.p("ninvs"), n, batch,
                                                      None) == 0
        assert lib.cbs_inwt_1d_opt_batched(d.data_ptr(), t.p("irp"), t.p("irps"), t.dmod.data_ptr(), t.p("ninv"),
                                           t.p("ninvs"), n, batch, None) == 0
        torch.cuda.synchronize()
        assert (_host(out) == a).all()
        assert (_host(d) == a).all()


def test_inverse_of_arbitrary_slots(lib, oracle):
    n = 2048
    q = oracle_primes(oracle, n, 54, 1)[0]
    t = Tabs(oracle, n, q)
    rng = np.random.default_rng(5)
    a = rand_mod(rng, q, (8, n))
    a[0, :] = 0
    a[1, :] = q - 1
    d = _dev(a.copy())
    assert lib.cbs_inwt_1d_opt_batched(d.data_ptr(), t.p("irp"), t.p("irps"), t.dmod.data_ptr(), t.p("ninv"),
                                       t.p("ninvs"), n, 8, None) == 0
    torch.cuda.synchronize()
    want = a.copy()
    oracle.orc_ntt_inverse(want, 8, n, q, t.irp, int(t.ninv[0]))
    assert (_host(d) == want).all()


def test_forward_out_of_place(lib, oracle):
    n = 2048
    q = oracle_primes(oracle, n, 54, 1)[0]
    t = Tabs(oracle, n, q)
    a = rand_mod(np.random.default_rng(9), q, (5, n))
    src = _dev(a.copy())
    dst = torch.zeros_like(src)
    assert lib.cbs_fnwt_1d_opt_outofplace_batched(dst.data_ptr(), src.data_ptr(), t.p("rp"), t.p("rps"),
                                                  t.dmod.data_ptr(), n, 5, None) == 0
    torch.cuda.synchronize()
    want = a.copy()
    oracle.orc_ntt_forward(want, 5, n, q, t.rp)
    assert (_host(dst) == want).all()
    assert (_host(src) == a).all()


@pytest.mark.parametrize("level", [0, 3, 10])
def test_inverse_permute_bit_exact(lib, oracle, level):
    n = 2048
    q = oracle_primes(oracle, n, 54, 1)[0]
    t = Tabs(oracle, n, q)
    maps = np.zeros(11 * n, np.uint32)
    oracle.orc_auto_maps(maps, n, 11)
    m = maps[level * n:(level + 1) * n].copy()
    # exercise the negation branch too: flag a few entries with +N
    m2 = m.copy()
    m2[::7] += n
    for mp in (m, m2):
        a = rand_mod(np.random.default_rng(level), q, (6, n))
        src = _dev(a)
        dst = torch.zeros_like(src)
        dmap = torch.from_numpy(mp.view(np.int32)).cuda()
        assert lib.cbs_inwt_1d_opt_permute_batched(dst.data_ptr(), src.data_ptr(), dmap.data_ptr(), t.p("irp"),
                                                   t.p("irps"), t.dmod.data_ptr(), t.p("ninv"), t.p("ninvs"), n, 6,
                                                   None) == 0
        torch.cuda.synchronize()
        want = np.zeros_like(a)
        oracle.orc_ntt_inverse_permute(want, a, mp, 6, n, q, t.irp, int(t.ninv[0]))
        assert (_host(dst) == want).all()


def test_large_batch_roundtrip(lib, oracle):
    """Full-size batch (2 x 256 ciphertexts x 6 digit polys) round trip; size-independent check."""
    n = 2048
    q = oracle_primes(oracle, n, 54, 1)[0]
    t = Tabs(oracle, n, q)
    batch = 3072
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randint(0, q, (batch, n), device="cuda", dtype=torch.int64, generator=g)
    y = x.clone()
    assert lib.cbs_fnwt_1d_opt_batched(y.data_ptr(), t.p("rp"), t.p("rps"), t.dmod.data_ptr(), n, batch, None) == 0
    assert lib.cbs_inwt_1d_opt_batched(y.data_ptr(), t.p("irp"), t.p("irps"), t.dmod.data_ptr(), t.p("ninv"),
                                       t.p("ninvs"), n, batch, None) == 0
    torch.cuda.synchronize()
    assert torch.equal(x, y)
    # spot-check a few rows against the oracle
    rows = [0, 1, batch // 2, batch - 1]
    a = x[rows].cpu().numpy().view(np.uint64).copy()
    z = x[rows].clone()
    assert lib.cbs_fnwt_1d_opt_batched(z.data_ptr(), t.p("rp"), t.p("rps"), t.dmod.data_ptr(), n, len(rows), None) == 0
    torch.cuda.synchronize()
    oracle.orc_ntt_forward(a, len(rows), n, q, t.rp)
    assert (_host(z) == a).all()
