"""The device generators compute the same values as the CPU oracle's
generator (so any sample of a benchmark workload can be checked)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,kw", [
    (0, dict(lo=-5, hi=1 << 40)),
    (1, dict(lo=0, hi=19)),
    (2, dict(x0=0.0, x1=0.1)),
    (3, dict(lo=0, hi=1_000_003)),
    (4, dict(lo=0, hi=100_000, x0=1.1)),
])
@pytest.mark.parametrize("row0", [0, 123_456])
def test_generators_match_oracle(kb, rt, oracle, kind, kw, row0):
    import torch
    n = 200_000
    dtype = {0: torch.int64, 1: torch.int32, 2: torch.float64, 3: torch.int64, 4: torch.int64}[kind]
    out = torch.empty(n, dtype=dtype, device="cuda")
    valid = torch.zeros((n + 31) // 32 * 4, dtype=torch.uint8, device="cuda")
    kb.gen_fill(rt, out, kind, 99, 5, row0=row0, null_fraction=0.02, valid=valid, **kw)
    rt.synchronize()
    want, wvalid = oracle.gen_column(kind, 99, 5, n, row0=row0, null_fraction=0.02, **kw)
    assert np.array_equal(out.cpu().numpy(), want)
    bits = np.unpackbits(valid.cpu().numpy(), bitorder="little")[:n]
    assert np.array_equal(bits, wvalid)


def test_permutation_is_a_bijection(kb, rt):
    import torch
    n = 1_000_000
    out = torch.empty(n, dtype=torch.int64, device="cuda")
    kb.gen_fill(rt, out, kb.GEN_PERMUTATION, 7, 1, lo=0, hi=n)
    rt.synchronize()
    assert torch.equal(torch.sort(out).values, torch.arange(n, device="cuda"))
