"""gpj_index_build_noalloc, the entry point for callers that cannot call
cudaMalloc (hosts that own the whole device memory pool, latency-critical
loops that avoid the device synchronisation of cudaMalloc/cudaFree).

Calls it through the C ABI and checks, on two calls in a row, that every
output equals the context-based gpj_index_build_async on the same input
(integer bitmaps: exact equality).  Kept in its own file, collected last.
"""
import numpy as np
import pytest
import torch

import oracle
from devmem import to_device

pytestmark = pytest.mark.gpu


def _buffers(n, levels, nl_cap):
    W = (n + 63) // 64
    mk = lambda k: torch.full((max(1, k),), -3, dtype=torch.int64, device="cuda")
    return {"S": mk(W), "LB": mk(W * levels), "E": mk(W), "Q": mk(W), "NL": mk(nl_cap),
            "sum": torch.full((4,), -3, dtype=torch.int64, device="cuda")}


def _index(gpj, b):
    ix = gpj.Index()
    ix.d_string, ix.d_leveled = b["S"].data_ptr(), b["LB"].data_ptr()
    ix.d_escape, ix.d_quote = b["E"].data_ptr(), b["Q"].data_ptr()
    ix.d_newline, ix.newline_capacity = b["NL"].data_ptr(), b["NL"].numel()
    return ix


@pytest.mark.parametrize("kind,size,offset", [("tweets", 5 << 20, 0), ("products", 3 << 20, 0),
                                              ("tweets", 777_777, 3), ("empty", 0, 0)])
def test_noalloc_matches_context_build(gpj, kind, size, offset):
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from gpjson_b200 import datagen
    data = {"tweets": lambda: datagen.tweets(21, size), "products": lambda: datagen.products(22, size),
            "empty": lambda: np.zeros(0, np.uint8)}[kind]()
    n, levels = data.size, 4
    nl_cap = n // 16 + 64
    t, ptr = to_device(data, offset)
    stream = torch.cuda.current_stream().cuda_stream

    # the warm-up a host that reserves all device memory makes before
    # reserving: the first call looks up the scratch array's address (and
    # CUDA's lazy loading places the module then)
    warm = _buffers(0, levels, 1)
    gpj.build_index_noalloc(ptr, 0, levels, _index(gpj, warm), warm["sum"].data_ptr(),
                            stream=stream)
    torch.cuda.synchronize()
    assert warm["sum"].cpu().tolist() == [1, 0, -1, 0]

    ref = _buffers(n, levels, nl_cap)
    with gpj.Context(0) as ctx:
        ctx.build_index_async(ptr, n, levels, _index(gpj, ref), ref["sum"].data_ptr(),
                              flags=1, stream=stream)
    torch.cuda.synchronize()

    for call in range(2):  # the shared scratch keeps the previous call's contents
        got = _buffers(n, levels, nl_cap)
        gpj.build_index_noalloc(ptr, n, levels, _index(gpj, got), got["sum"].data_ptr(),
                                flags=1, stream=stream)
        torch.cuda.synchronize()
        for k in ("S", "LB", "E", "Q", "NL", "sum"):
            assert torch.equal(got[k], ref[k]), (call, k)
    lines = int(ref["sum"][0])
    want = oracle.OracleIndex(data, levels)
    assert lines == want.num_lines
    assert np.array_equal(ref["NL"].cpu().numpy()[:lines], want.NL)


def test_noalloc_rejects_oversized_input(gpj):
    ix = gpj.Index()
    with pytest.raises(gpj.CapacityError, match="4 GiB"):
        gpj.build_index_noalloc(1 << 20, gpj.NOALLOC_MAX_BYTES + 1, 2, ix, 1 << 20)
