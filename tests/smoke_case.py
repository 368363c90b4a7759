"""The smoke case run by __graft_entry__.smoke(): a small slice of the hot path on cuda:0
through the C ABI, checked bit-exactly against the CPU oracle."""
from __future__ import annotations


def run_smoke(pkg, torch, np) -> None:
    from conftest import load_oracle, oracle_primes, oracle_tables

    assert torch.cuda.is_available(), "smoke() needs cuda:0"
    torch.cuda.set_device(0)
    lib = pkg.load()
    oracle = load_oracle()

    # forward + inverse Phantom NTT at the CBS ring size
    n = 2048
    q = oracle_primes(oracle, n, 54, 1)[0]
    rp, rps, irp, irps, ninv = oracle_tables(oracle, n, q)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()  # noqa: E731
    d_rp, d_rps, d_irp, d_irps = dev(rp), dev(rps), dev(irp), dev(irps)
    d_ni, d_nis = dev(ninv[:1].copy()), dev(ninv[1:].copy())
    d_mod = dev(np.array([q, 0, 0], np.uint64))
    rng = np.random.default_rng(0)
    a = rng.integers(0, q, size=(4, n), dtype=np.uint64)
    x = dev(a.copy())
    pkg.call("cbs_fnwt_1d_opt_batched", x.data_ptr(), d_rp.data_ptr(), d_rps.data_ptr(), d_mod.data_ptr(), n, 4, None)
    torch.cuda.synchronize()
    want = a.copy()
    oracle.orc_ntt_forward(want, 4, n, q, rp)
    got = x.cpu().numpy().view(np.uint64)
    assert (got == want).all(), "forward NTT mismatch vs oracle"
    pkg.call("cbs_inwt_1d_opt_batched", x.data_ptr(), d_irp.data_ptr(), d_irps.data_ptr(), d_mod.data_ptr(),
             d_ni.data_ptr(), d_nis.data_ptr(), n, 4, None)
    torch.cuda.synchronize()
    assert (x.cpu().numpy().view(np.uint64) == a).all(), "inverse NTT mismatch"
    print("smoke: NTT N=2048 bit-exact vs oracle")
