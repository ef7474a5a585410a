"""flsgpu_sum_alp_f64_noalloc: the f64 decode-and-sum for callers that
cannot allocate device memory (an engine with a fixed memory budget, a
thread capturing a CUDA graph, a plug-in that must not use the host
process's allocator).  Its scratch is a static device array inside the
library; the result must equal flsgpu_sum_alp_f64 (which takes caller
workspace) bit for bit, on consecutive calls, and columns larger than the
static limit must be refused before anything is launched.

This file is collected last on purpose (pytest orders files by name), so a
run that stops at the first failure has run every other test already; it
also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu

MAX_VECTORS = 262144  # FLSGPU_NOALLOC_MAX_VECTORS in include/flsgpu_b200.h


def _noalloc_sum(col, out, stream):
    f = F._fn("flsgpu_sum_alp_f64_noalloc")
    return f(C.byref(col.c), C.c_void_p(out.data_ptr()), None, C.c_void_p(stream))


def test_noalloc_sum_matches_workspace_sum_twice(cuda):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    # two different columns, so the second call must not see the first's partials
    for seed, n_vecs in ((21, 3000), (22, 700)):
        col = colgen.random_alp(seed, n_vecs, True, [6, 13, 21], [0, 2, 9])
        e = col["exceptions"]
        col["exceptions"] = np.where(np.isfinite(e), e, -2.25)  # NaN payloads are not summed bitwise
        d = F.make_alp_column(col, n_vecs * 1024, np.float64, device=cuda)
        want = F.sum_(d).cpu().numpy().view(np.uint64)[0]
        for _ in range(2):
            out = torch.full((1,), 7.0, dtype=torch.float64, device=cuda)
            assert _noalloc_sum(d, out, stream) == 0, F.lib().flsgpu_last_error()
            got = out.cpu().numpy().view(np.uint64)[0]
            assert got == want
        dec = B.alp_decode(col, n_vecs, np.float64)
        oracle = np.array([B.oracle().orc_tree_sum_f64(B.ptr(dec), n_vecs)]).view(np.uint64)[0]
        assert got == oracle


def test_noalloc_rejects_columns_beyond_the_static_limit(cuda):
    c = F.ALPColumnC()
    c.n_values = (MAX_VECTORS + 1) * 1024
    f = F._fn("flsgpu_sum_alp_f64_noalloc")
    assert f(C.byref(c), C.c_void_p(16), None, None) == 1
    assert b"static scratch limit" in F.lib().flsgpu_last_error()
