"""GPU parity of the BP / FFOR kernels against the oracle (bit-exact), on
the reference's test shapes: every bit width of u32 and u64, mixed widths
per vector, ragged tails, the FFOR-small benchmark column, fused sums,
magic-value scans, the synthetic compute kernel and the multi-column scan
(reference test-fls.sh / test-multi-column.sh sweeps)."""
import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu


def _col(c, dev, bp=False):
    return F.make_ffor_column(c["packed"], c["bit_widths"], c["vector_offsets"],
                              None if bp else c["bases"], c["n_values"], dev)


def _host(t, ut):
    return t.cpu().numpy().view(ut)


@pytest.mark.parametrize("bits", [32, 64])
def test_ffor_every_width(cuda, bits):
    ut = np.uint64 if bits == 64 else np.uint32
    for w in range(bits + 1):
        c = colgen.random_ffor(100 + w + bits, 9, bits, [w])
        got = _host(F.decompress(_col(c, cuda)), ut)
        want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
        assert np.array_equal(got, want), f"u{bits} w={w}"


@pytest.mark.parametrize("bits", [32, 64])
def test_bp_every_width(cuda, bits):
    ut = np.uint64 if bits == 64 else np.uint32
    for w in range(0, bits + 1, 3):
        c = colgen.random_ffor(300 + w + bits, 5, bits, [w])
        got = _host(F.decompress(_col(c, cuda, bp=True)), ut)
        want = B.decode_bp(c["packed"], c["bit_widths"], c["vector_offsets"], bits)
        assert np.array_equal(got, want), f"u{bits} w={w}"


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("variant", [F.VARIANT_AUTO, F.VARIANT_REGS, F.VARIANT_OCCUPANCY,
                                     F.VARIANT_STAGED])
def test_ffor_mixed_widths(cuda, bits, variant):
    ut = np.uint64 if bits == 64 else np.uint32
    c = colgen.random_ffor(7 + bits, 3000, bits, range(bits + 1))
    got = _host(F.decompress(_col(c, cuda), o=F.opts(variant=variant)), ut)
    want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("n_values", [1, 1000, 1025, 5 * 1024 - 3])
def test_ragged_tail_is_not_overwritten(cuda, bits, n_values):
    import torch
    ut = np.uint64 if bits == 64 else np.uint32
    n_vecs = (n_values + 1023) // 1024
    c = colgen.random_ffor(55, n_vecs, bits, [bits // 3, bits], n_values=n_values)
    out = torch.full((n_values + 2048,), -1, dtype=torch.int64 if bits == 64 else torch.int32,
                     device=cuda)
    F.decompress(_col(c, cuda), out=out[:n_values])
    got = _host(out, ut)
    want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
    assert np.array_equal(got[:n_values], want[:n_values])
    assert np.all(got[n_values:] == ut(np.iinfo(ut).max))


def test_ffor_small_config_roundtrip(cuda):
    """2^20 u32 values, 1024 vectors, w = 7: decode equals the input and the
    oracle's unffor."""
    vals, c = colgen.ffor_config1(1)
    assert set(c["bit_widths"].tolist()) == {7}
    got = _host(F.decompress(_col(c, cuda)), np.uint32)
    assert np.array_equal(got, vals)
    assert np.array_equal(got, B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"],
                                             c["bases"], 32))


@pytest.mark.parametrize("bits", [32, 64])
def test_fused_sum(cuda, bits):
    c = colgen.random_ffor(900 + bits, 2000, bits, range(bits + 1))
    want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
    s = int(F.sum_(_col(c, cuda)).cpu().numpy().view(np.uint64)[0])
    ref = int(want.astype(np.uint64).sum(dtype=np.uint64))
    assert s == ref


@pytest.mark.parametrize("bits", [32, 64])
def test_query_found_and_absent(cuda, bits):
    ut = np.uint64 if bits == 64 else np.uint32
    c = colgen.random_ffor(40 + bits, 300, bits, [3, 5], base_max=100)
    col = _col(c, cuda)
    vals = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
    present = int(vals[123457 % vals.size])
    absent = int(vals.max()) + 1
    assert int(F.query(col, present).item()) == 1
    assert int(F.query(col, absent).item()) == 0
    bp = _col(c, cuda, bp=True)
    raw = B.decode_bp(c["packed"], c["bit_widths"], c["vector_offsets"], bits)
    assert int(F.query(bp, int(raw[77])).item()) == 1
    assert int(F.query(bp, int(raw.max()) + 1).item()) == 0


@pytest.mark.parametrize("bits", [32, 64])
def test_compute_column_never_finds_one(cuda, bits):
    """compute_column ANDs every value with a runtime zero, so the magic
    value 1 is never seen (src/engine/kernels.cuh:75-88)."""
    c = colgen.random_ffor(60 + bits, 64, bits, [4, 9])
    assert int(F.compute(_col(c, cuda), 10).item()) == 0


@pytest.mark.parametrize("bits", [32, 64])
def test_multi_column(cuda, bits):
    ut = np.uint64 if bits == 64 else np.uint32
    n_vecs = 40
    cols = []
    for i in range(4):
        c = colgen.random_ffor(70 + i, n_vecs, bits, [0, 3], base_max=2)
        c["bit_widths"][:] = np.where(np.arange(n_vecs) % 2 == 0, 3, 0)
        nl = 1024 // bits
        c["vector_offsets"][:] = np.concatenate([[0], np.cumsum(c["bit_widths"].astype(np.uint64) * nl)[:-1]])
        c["packed"] = c["packed"][: int(c["bit_widths"].astype(np.int64).sum()) * nl]
        c["bases"][:] = 5
        cols.append(c)
    # width-0 vectors (odd ones) decode to the base 5 everywhere
    dcols = [_col(c, cuda) for c in cols]
    assert int(F.query_multi_column(dcols, 5).item()) == 1
    assert int(F.query_multi_column(dcols, 6).item()) == 0
    # the reference's own multi-column test queries the type's max: never found
    assert int(F.query_multi_column(dcols, int(np.iinfo(ut).max)).item()) == 0
    # break vector lanes of column 2 at every width-0 vector: no lane qualifies
    cols[2]["bases"][1::2] = 6
    dcols[2] = _col(cols[2], cuda)
    assert int(F.query_multi_column(dcols, 5).item()) == 0


@pytest.mark.parametrize("bits", [32, 64])
def test_corrupt_metadata_is_flagged_not_faulted(cuda, bits):
    import torch
    c = colgen.random_ffor(11, 16, bits, [5])
    c["bit_widths"][3] = bits + 1
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    F.decompress(_col(c, cuda), o=F.opts(d_status=status))
    assert int(status.item()) & F.BAD_BIT_WIDTH
    # a packed-size bound catches offsets that run past the array
    c = colgen.random_ffor(12, 16, bits, [5])
    status.zero_()
    F.decompress(_col(c, cuda), o=F.opts(d_status=status, n_packed_values=c["packed"].size - 1))
    assert int(status.item()) & F.BAD_OFFSET


@pytest.mark.parametrize("bp", [False, True])
def test_staged_decode_every_width_and_unaligned_vectors(cuda, bp):
    """The staged u64 decode (packed words brought into shared memory by bulk
    copies): every width 0..64, ragged tails, and a column whose vectors'
    packed words are not 16-byte aligned (odd word offsets), which take the
    register-held path."""
    import torch
    for w in range(65):
        c = colgen.random_ffor(700 + w, 7, 64, [w], n_values=7 * 1024 - 5)
        got = _host(F.decompress(_col(c, cuda, bp), o=F.opts(variant=F.VARIANT_STAGED)), np.uint64)
        want = (B.decode_bp(c["packed"], c["bit_widths"], c["vector_offsets"], 64) if bp else
                B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], 64))
        assert np.array_equal(got, want[:c["n_values"]]), w
    # odd word offsets: one spare word before every vector's packed words
    c = colgen.random_ffor(31, 40, 64, range(65))
    n_vecs = 40
    offs = c["vector_offsets"].astype(np.int64) + np.arange(1, n_vecs + 1)
    packed = np.zeros(int(c["packed"].size) + n_vecs + 1, np.uint64)
    for v in range(n_vecs):
        n = int(c["bit_widths"][v]) * 16
        o0 = int(c["vector_offsets"][v])
        packed[offs[v]:offs[v] + n] = c["packed"][o0:o0 + n]
    d = F.make_ffor_column(packed, c["bit_widths"], offs.astype(np.uint64),
                           None if bp else c["bases"], c["n_values"], cuda)
    got = _host(F.decompress(d, o=F.opts(variant=F.VARIANT_STAGED)), np.uint64)
    want = (B.decode_bp(c["packed"], c["bit_widths"], c["vector_offsets"], 64) if bp else
            B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], 64))
    assert np.array_equal(got, want)
    # a status word stays clear (no wait gave up)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    F.decompress(d, o=F.opts(variant=F.VARIANT_STAGED, d_status=status))
    assert int(status.item()) == 0


@pytest.mark.parametrize("bits", [32, 64])
def test_fused_sum_groups_and_edges(cuda, bits):
    """The integer sum adds each full vector's base once (1024 * base) when
    that is exact and sums value by value otherwise: exact (mod 2^64)
    against the oracle on long runs of one narrow width, on narrow and wide
    widths mixed, on u32 bases whose values wrap past 2^32 (every vector,
    and every third vector), on ragged tails and on a single partial
    vector; a bad width among narrow vectors is flagged and adds nothing."""
    import torch
    ut = np.uint64 if bits == 64 else np.uint32

    def ref(c, n_values=None):
        want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
        return int(want[:n_values].astype(np.uint64).sum(dtype=np.uint64))

    cases = [([3], 9000, None), ([1, 2, 9, 8, 30, 0], 9000, None), (range(9), 9001, 9001 * 1024 - 5),
             ([5], 7, 7 * 1024 - 1), ([0, 1], 1, 1)]
    for i, (widths, n_vecs, n_values) in enumerate(cases):
        c = colgen.random_ffor(1700 + i + bits, n_vecs, bits, widths, n_values=n_values)
        if i == 0 and bits == 32:
            c["bases"][:] = np.uint32(2 ** 32 - 3)  # every vector's values wrap
        s = int(F.sum_(_col(c, cuda)).cpu().numpy().view(np.uint64)[0])
        assert s == ref(c, c["n_values"]), (bits, i)
    # bases near the top of the u32 range on some vectors only
    if bits == 32:
        c = colgen.random_ffor(1790, 5000, 32, [4, 7])
        c["bases"][::3] = np.uint32(2 ** 32 - 1)
        assert int(F.sum_(_col(c, cuda)).cpu().numpy().view(np.uint64)[0]) == ref(c)
    # a bad width among narrow vectors: flagged, the rest summed
    c = colgen.random_ffor(1791 + bits, 6000, bits, [2])
    want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
    keep = np.ones(6000 * 1024, bool)
    keep[2500 * 1024:2501 * 1024] = False
    c["bit_widths"][2500] = bits + 1
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    s = int(F.sum_(_col(c, cuda), o=F.opts(d_status=status)).cpu().numpy().view(np.uint64)[0])
    assert int(status.item()) & F.BAD_BIT_WIDTH
    assert s == int(want[keep].astype(np.uint64).sum(dtype=np.uint64))


@pytest.mark.parametrize("bits", [32, 64])
def test_query_range_test_edges(cuda, bits):
    """The integer scan decides a vector on its metadata when the magic
    value lies outside [base, base + 2^w) (mod 2^bits): found exactly where
    the oracle's decode holds the value -- a vector's base (u = 0), its top
    value (u = 2^w - 1), values of vectors whose range wraps past 2^bits,
    width-0 vectors (only the base), full-width vectors (no test) -- and not
    found for values just outside a range or present only past n_values in
    the last, partial vector."""
    ut = np.uint64 if bits == 64 else np.uint32
    top = 2 ** bits
    rng = np.random.default_rng(bits)
    for widths in ([0, 3], [1, 7, bits], [5]):
        n_vecs = 64
        n_values = n_vecs * 1024 - 300
        c = colgen.random_ffor(2100 + bits + len(widths), n_vecs, bits, widths, n_values=n_values)
        # some bases near the top of the range, so that their values wrap
        c["bases"][::5] = ut(top - 3)
        vals = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
        inside = set(int(x) for x in vals[:n_values])
        col = _col(c, cuda)
        cands = set()
        for v in rng.choice(n_vecs - 1, 12, replace=False):
            w, base = int(c["bit_widths"][v]), int(c["bases"][v])
            cands |= {base, (base + 2 ** min(w, bits) - 1) % top, (base + 2 ** min(w, bits)) % top,
                      (base - 1) % top}
        cands |= set(int(x) for x in vals[n_values:n_vecs * 1024][:5])  # past n_values
        cands |= {0, top - 1, int(vals[n_values - 1])}
        for m in sorted(cands):
            got = int(F.query(col, m).item())
            assert got == (m in inside), (widths, m)


@pytest.mark.parametrize("bits", [32, 64])
def test_multi_column_range_test_and_skips(cuda, bits):
    """The multi-column scan decides a vector of a column on its metadata
    when the value lies outside the vector's range and stops decoding a
    vector's columns once no lane can qualify: same answers as the oracle's
    decode, per lane, on columns whose vectors mix width-0 runs of the
    value, narrow widths around it and wrapping bases; a corrupt width in a
    later column of a vector that already failed is still flagged."""
    import torch
    ut = np.uint64 if bits == 64 else np.uint32
    top = 2 ** bits
    n_vecs = 48
    nl = 1024 // bits
    rng = np.random.default_rng(5 + bits)

    def column(seed, widths, base_of):
        c = colgen.random_ffor(seed, n_vecs, bits, [0])
        c["bit_widths"][:] = widths
        c["vector_offsets"][:] = np.concatenate(
            [[0], np.cumsum(c["bit_widths"].astype(np.uint64) * nl)[:-1]])
        n = int(c["bit_widths"].astype(np.int64).sum()) * nl
        c["packed"] = rng.integers(0, 2 ** 63, max(n, 1), dtype=np.uint64).astype(ut)[:n]
        c["bases"][:] = [ut(base_of(v) % top) for v in range(n_vecs)]
        return c

    def lanes_equal(cols, value):
        lanes = 1024 // bits  # FastLanes lanes; lane l holds values l + lanes * k
        ok = False
        vals = [B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
                .reshape(n_vecs, 1024 // lanes, lanes) for c in cols]
        for v in range(n_vecs):
            every = np.ones(lanes, bool)
            for x in vals:
                every &= np.all(x[v] == ut(value % top), axis=0)
            ok |= bool(every.any())
        return ok

    value = 7
    widths_a = np.where(np.arange(n_vecs) % 3 == 0, 0, np.where(np.arange(n_vecs) % 3 == 1, 2, 5))
    cols = [column(2200 + bits, widths_a, lambda v: 7 if v % 3 == 0 else 6),
            column(2201 + bits, np.where(np.arange(n_vecs) % 2 == 0, 0, 3), lambda v: 7 if v % 4 else top - 2),
            column(2202 + bits, np.zeros(n_vecs, np.int64), lambda v: 7 if v != 9 else 8)]
    d = [_col(c, cuda) for c in cols]
    for m in (value, 6, 8, top - 2, 0):
        assert int(F.query_multi_column(d, m).item()) == int(lanes_equal(cols, m)), m
    # a corrupt width in the last column of vectors that fail on column 0
    cols[2]["bit_widths"][1] = bits + 1
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    F.query_multi_column([_col(c, cuda) for c in cols], 12345, o=F.opts(d_status=status))
    assert int(status.item()) & F.BAD_BIT_WIDTH
