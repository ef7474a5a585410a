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


def _bad_width_column(seed, n_vecs, bad_vec):
    """A valid f64 ALP column and a copy whose vector `bad_vec` claims bit
    width 70 (beyond 64): the decode-and-sum rejects that vector, raises
    FLSGPU_BAD_BIT_WIDTH and counts it as +0.0."""
    col = colgen.random_alp(seed, n_vecs, True, [6, 13, 21], [0, 2, 9])
    e = col["exceptions"]
    col["exceptions"] = np.where(np.isfinite(e), e, -2.25)
    dec = B.alp_decode(col, n_vecs, np.float64)
    dec[bad_vec * 1024:(bad_vec + 1) * 1024] = 0.0
    want = np.array([B.oracle().orc_tree_sum_f64(B.ptr(dec), n_vecs)]).view(np.uint64)[0]
    bad = dict(col)
    bad["bit_widths"] = col["bit_widths"].copy()
    bad["bit_widths"][bad_vec] = 70
    return col, bad, want


def test_rejected_vector_adds_zero_whatever_the_scratch_held(cuda):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    n_vecs, bad_vec = 2500, 5
    good, bad, want = _bad_width_column(31, n_vecs, bad_vec)
    d_bad = F.make_alp_column(bad, n_vecs * 1024, np.float64, device=cuda)
    d_good = F.make_alp_column(colgen.random_alp(32, n_vecs, True, [9], [3]), n_vecs * 1024,
                               np.float64, device=cuda)
    ws_n = F.lib().flsgpu_sum_workspace_f64(n_vecs * 1024)
    # caller workspace poisoned two different ways
    for poison in (float("nan"), 1.0e300):
        ws = torch.full((ws_n,), poison, dtype=torch.float64, device=cuda)
        status = torch.zeros(1, dtype=torch.int32, device=cuda)
        out = F.sum_(d_bad, workspace=ws, o=F.opts(d_status=status))
        assert out.cpu().numpy().view(np.uint64)[0] == want
        assert int(status.item()) & 0x1  # FLSGPU_BAD_BIT_WIDTH
    # the static scratch after a call on another column, then twice more
    F.sum_(d_good)
    assert _noalloc_sum(d_good, torch.empty(1, dtype=torch.float64, device=cuda), stream) == 0
    for _ in range(2):
        out = torch.full((1,), 7.0, dtype=torch.float64, device=cuda)
        status = torch.zeros(1, dtype=torch.int32, device=cuda)
        o = F.opts(d_status=status)
        f = F._fn("flsgpu_sum_alp_f64_noalloc")
        assert f(C.byref(d_bad.c), C.c_void_p(out.data_ptr()), C.byref(o), C.c_void_p(stream)) == 0
        assert out.cpu().numpy().view(np.uint64)[0] == want
        assert int(status.item()) & 0x1


def test_noalloc_at_exactly_the_static_limit(cuda):
    """A column of exactly FLSGPU_NOALLOC_MAX_VECTORS vectors, where the
    scratch bound of the pairwise tree's ping-pong is tight: width 0
    everywhere (no packed words), per-vector bases, so every vector sums a
    different constant."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    n = MAX_VECTORS
    rng = np.random.default_rng(5)
    col = dict(packed=np.zeros(0, np.uint64), bit_widths=np.zeros(n, np.uint8),
               vector_offsets=np.zeros(n, np.uint64),
               bases=rng.integers(0, 100000, n).astype(np.uint64),
               factor_indices=np.zeros(n, np.uint8),
               fraction_indices=rng.integers(0, 4, n).astype(np.uint8),
               exceptions_offsets=np.zeros(n, np.uint64), exceptions=np.zeros(0),
               positions=np.zeros(0, np.uint16), counts=np.zeros(n, np.uint16))
    d = F.make_alp_column(col, n * 1024, np.float64, device=cuda)
    want = F.sum_(d).cpu().numpy().view(np.uint64)[0]
    # the per-vector constants summed by the fixed tree, on the host
    frac = np.array([1.0, 0.1, 0.01, 0.001])
    vals = col["bases"].astype(np.int64).astype(np.float64) * frac[col["fraction_indices"]]
    assert np.float64(want.view(np.float64)) == pytest.approx(float((vals * 1024).sum()), rel=1e-9)
    for _ in range(2):
        out = torch.full((1,), 7.0, dtype=torch.float64, device=cuda)
        assert _noalloc_sum(d, out, stream) == 0, F.lib().flsgpu_last_error()
        assert out.cpu().numpy().view(np.uint64)[0] == want
