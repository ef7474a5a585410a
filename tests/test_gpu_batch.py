"""Batched persistent decode and the fused pair query, bit-exact against the
oracle: columns of uneven length, type and bit width in one launch, the
same batch replayed from a captured CUDA graph, the per-column launch path,
and sum(A where B < median(B)) per (f64 ALP, u32 FFOR) pair."""
import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu


def _mixed_columns(seed, n_cols, cuda, max_vecs=40):
    rng = np.random.default_rng(seed)
    cols, wants = [], []
    for i in range(n_cols):
        kind = i % 6
        n_vecs = int(rng.integers(1, max_vecs))
        tail = int(rng.integers(0, 1024)) if i % 7 == 3 else 0
        n_values = n_vecs * 1024 - tail
        if kind in (0, 1):  # u32 / u64 FFOR, all widths
            bits = 32 if kind == 0 else 64
            c = colgen.random_ffor(seed * 100 + i, n_vecs, bits, range(bits + 1), n_values=n_values)
            d = F.make_ffor_column(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"],
                                   n_values, cuda)
            want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
        elif kind == 2:  # u32 BP
            c = colgen.random_ffor(seed * 100 + i, n_vecs, 32, range(33), n_values=n_values)
            d = F.make_ffor_column(c["packed"], c["bit_widths"], c["vector_offsets"], None,
                                   n_values, cuda)
            want = B.decode_bp(c["packed"], c["bit_widths"], c["vector_offsets"], 32)
        else:  # f64 / f32 ALP, plain or extended
            f64 = kind != 4
            dt = np.float64 if f64 else np.float32
            col = colgen.random_alp(seed * 100 + i, n_vecs, f64, range(0, 25), range(0, 30))
            ext = kind == 5
            c = B.to_extended(col, n_vecs, dt)[0] if ext else col
            d = F.make_alp_column(c, n_values, dt, extended=ext, device=cuda)
            want = B.alp_decode(c, n_vecs, dt, extended=ext)
        cols.append(d)
        wants.append(np.ascontiguousarray(want[:n_values]).view(np.uint8))
    return cols, wants


def _outs(cols, cuda):
    import torch
    return [torch.full((c.n_values,), -1, dtype=getattr(torch, F.TORCH_OF_BITS[c.dtype]),
                       device=cuda) for c in cols]


def _host_bytes(t):
    return t.cpu().numpy().view(np.uint8)


@pytest.mark.parametrize("mode", ["launch", "graph", "each"])
def test_batch_decode_matches_oracle(cuda, mode):
    import torch
    cols, wants = _mixed_columns(3, 60, cuda)
    outs = _outs(cols, cuda)
    b = F.Batch(cols, outs)
    assert b.total_vectors() == sum(c.n_vecs for c in cols)
    if mode == "launch":
        b.decompress()
    elif mode == "graph":
        b.capture()
        b.replay()
        torch.cuda.synchronize()
        for o in outs:
            o.fill_(-1)
        b.replay()  # a second replay decodes again from scratch
    else:
        b.decompress_each()
    torch.cuda.synchronize()
    for i, (o, w) in enumerate(zip(outs, wants)):
        assert np.array_equal(_host_bytes(o), w), f"column {i} ({cols[i].kind} {cols[i].dtype})"


def test_batch_with_empty_and_single_vector_columns(cuda):
    import torch
    cols, wants = _mixed_columns(5, 12, cuda, max_vecs=2)
    empty = F.make_ffor_column(np.zeros(0, np.uint32), np.zeros(0, np.uint8),
                               np.zeros(0, np.uint64), np.zeros(0, np.uint32), 0, cuda)
    cols = [empty] + cols[:6] + [empty] + cols[6:]
    wants = [np.zeros(0, np.uint8)] + wants[:6] + [np.zeros(0, np.uint8)] + wants[6:]
    outs = _outs(cols, cuda)
    b = F.Batch(cols, outs)
    b.decompress()
    torch.cuda.synchronize()
    for o, w in zip(outs, wants):
        assert np.array_equal(_host_bytes(o), w)


def _pair(seed, n_vecs, cuda, b_width_choices=range(0, 33)):
    col_a = colgen.random_alp(seed, n_vecs, True, range(8, 22), range(0, 20))
    e = col_a["exceptions"]
    col_a["exceptions"] = np.where(np.isfinite(e), e, 0.75)
    cb = colgen.random_ffor(seed + 7, n_vecs, 32, b_width_choices)
    a = F.make_alp_column(col_a, n_vecs * 1024, np.float64, device=cuda)
    b = F.make_ffor_column(cb["packed"], cb["bit_widths"], cb["vector_offsets"], cb["bases"],
                           n_vecs * 1024, cuda)
    av = B.alp_decode(col_a, n_vecs, np.float64)
    bv = B.decode_ffor(cb["packed"], cb["bit_widths"], cb["vector_offsets"], cb["bases"], 32)
    o = B.oracle()
    med = int(o.orc_median_u32(B.ptr(bv), bv.size))
    want = o.orc_tree_sum_masked_f64(B.ptr(av), B.ptr(bv), med, n_vecs)
    return a, b, med, want


@pytest.mark.parametrize("graph", [False, True])
def test_pair_query_median_and_masked_sum(cuda, graph):
    import torch
    rng = np.random.default_rng(8)
    pairs = [_pair(100 + i, int(rng.integers(1, 70)), cuda,
                   b_width_choices=[int(rng.integers(0, 33))] if i % 3 == 0 else range(0, 33))
             for i in range(24)]
    pairs.append(_pair(999, 2500, cuda))  # > 2048 vectors: two chunks in the pair reduction
    q = F.PairQuery([p[0] for p in pairs], [p[1] for p in pairs], cuda)
    if graph:
        q.capture()
        q.replay()
        torch.cuda.synchronize()
        q.results.zero_()
        q.replay()
    else:
        q.run()
    torch.cuda.synchronize()
    meds = q.medians.cpu().numpy().view(np.uint32)
    res = q.results.cpu().numpy()
    for i, (_, _, med, want) in enumerate(pairs):
        assert meds[i] == med, f"pair {i}"
        assert res[i].view(np.uint64) == np.float64(want).view(np.uint64), f"pair {i}"
    assert int(q.status.item()) == 0


def test_pair_query_ragged_lengths(cuda):
    """Columns whose length is not a multiple of 1024: the median and the
    masked sum cover only the valid values (the oracle sees the last vector
    padded with B = 0xFFFFFFFF, which is never below the median, and with the
    median taken over the n valid values)."""
    import torch
    o = B.oracle()
    pairs, wants = [], []
    for i, n_values in enumerate((1000, 5 * 1024 + 17, 3 * 1024 - 1)):
        n_vecs = (n_values + 1023) // 1024
        col_a = colgen.random_alp(300 + i, n_vecs, True, range(8, 22), range(0, 20))
        e = col_a["exceptions"]
        col_a["exceptions"] = np.where(np.isfinite(e), e, 0.75)
        cb = colgen.random_ffor(310 + i, n_vecs, 32, range(0, 33), n_values=n_values)
        a = F.make_alp_column(col_a, n_values, np.float64, device=cuda)
        b = F.make_ffor_column(cb["packed"], cb["bit_widths"], cb["vector_offsets"], cb["bases"],
                               n_values, cuda)
        av = B.alp_decode(col_a, n_vecs, np.float64)
        bv = B.decode_ffor(cb["packed"], cb["bit_widths"], cb["vector_offsets"], cb["bases"], 32)
        bv = np.ascontiguousarray(bv.astype(np.uint32))
        med = int(o.orc_median_u32(B.ptr(bv), n_values))
        bpad = bv.copy()
        bpad[n_values:] = 0xFFFFFFFF
        want = o.orc_tree_sum_masked_f64(B.ptr(av), B.ptr(bpad), med, n_vecs)
        pairs.append((a, b))
        wants.append((med, want))
    q = F.PairQuery([p[0] for p in pairs], [p[1] for p in pairs], cuda)
    q.run()
    torch.cuda.synchronize()
    meds = q.medians.cpu().numpy().view(np.uint32)
    res = q.results.cpu().numpy()
    for i, (med, want) in enumerate(wants):
        assert meds[i] == med, i
        assert res[i].view(np.uint64) == np.float64(want).view(np.uint64), i
    assert int(q.status.item()) == 0
