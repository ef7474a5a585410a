"""GPU parity of the ALP / ALP-extended / ALP-RD kernels against the oracle,
bit for bit (every double's pattern), on the reference's test shapes:
compressed-level random columns over bit widths and exception counts
(test-alp.sh: patchers x exception counts 0..10 x widths 0..16), the
extremes (0 and 1024 exceptions per vector, full-width vectors), value-level
columns encoded by the oracle encoder, fused sums and scans."""
import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu


def _ut(f64):
    return np.uint64 if f64 else np.uint32


def _dt(f64):
    return np.float64 if f64 else np.float32


def _check(cuda, col, n_vecs, f64, extended=False, patcher=7, variant=F.VARIANT_AUTO):
    dt, ut = _dt(f64), _ut(f64)
    c = col
    if extended:
        c, _ = B.to_extended(col, n_vecs, dt)
    d = F.make_alp_column(c, n_vecs * 1024, dt, extended=extended, device=cuda)
    got = F.decompress(d, o=F.opts(patcher=patcher, variant=variant)).cpu().numpy().view(ut)
    want = B.alp_decode(c, n_vecs, dt, extended=extended).view(ut)
    return got, want


@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("extended", [False, True])
@pytest.mark.parametrize("variant", [F.VARIANT_REGS, F.VARIANT_OCCUPANCY, F.VARIANT_STAGED])
def test_alp_widths_and_exception_counts(cuda, f64, extended, variant):
    bits = 64 if f64 else 32
    for ec in [0, 1, 5, 10, 33, 70]:
        col = colgen.random_alp(1000 + ec, 64, f64, range(0, 17), [ec])
        got, want = _check(cuda, col, 64, f64, extended, variant=variant)
        assert np.array_equal(got, want), f"ec={ec}"
    col = colgen.random_alp(77, 256, f64, range(bits + 1), range(0, 40))
    got, want = _check(cuda, col, 256, f64, extended, variant=variant)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("f64", [True, False])
def test_alp_every_position_an_exception(cuda, f64):
    col = colgen.random_alp(5, 12, f64, [3, 17], [1024, 0, 1023, 512])
    for extended in (False, True):
        got, want = _check(cuda, col, 12, f64, extended)
        assert np.array_equal(got, want)


@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("patcher", [0, 1])
def test_patcher_none_and_dummy_skip_exceptions(cuda, f64, patcher):
    col = colgen.random_alp(15, 20, f64, [9], [7])
    got, want_patched = _check(cuda, col, 20, f64, patcher=patcher)
    nopatch = dict(col)
    nopatch["counts"] = np.zeros_like(col["counts"])
    _, want = _check(cuda, nopatch, 20, f64)
    assert np.array_equal(got, want)
    assert not np.array_equal(got, want_patched)


@pytest.mark.parametrize("f64,dmax", [(True, 4), (False, 3)])
def test_encoded_columns_roundtrip(cuda, f64, dmax):
    """Value-level data (ALP decode benchmark shape, scaled down), encoded by
    the oracle encoder with per-rowgroup sampling: GPU decode reproduces
    every input bit pattern and the oracle decode."""
    dt, ut = _dt(f64), _ut(f64)
    vals = colgen.alp_values(31, 150, f64, dmax)
    col = B.alp_encode(vals, rowgroup_vecs=100)
    assert col is not None
    for extended in (False, True):
        c, overflow = B.to_extended(col, 150, dt) if extended else (col, 0)
        d = F.make_alp_column(c, vals.size, dt, extended=extended, device=cuda)
        got = F.decompress(d).cpu().numpy().view(ut)
        assert np.array_equal(got, B.alp_decode(c, 150, dt, extended=extended).view(ut))
        if overflow == 0:
            assert np.array_equal(got, vals.view(ut))
        else:
            # vectors whose 64-bit lanes hold 64 exceptions cannot be expressed
            # in the extended layout; everything else round-trips
            bad = np.unique(np.nonzero(got != vals.view(ut))[0] // 1024)
            assert np.all(col["counts"][bad] >= 64)


def test_extended_overflow_matches_reference_cpu_decode(cuda):
    """A 64-bit lane with 64 exceptions overflows the 6-bit count field of
    the extended layout (src/flsgpu/structs.cuh:293-295); the GPU decode
    then matches the reference's CPU decode of that column (count = sum of
    lane fields), not the plain layout."""
    n_vecs = 3
    col = colgen.random_alp(9, n_vecs, True, [12], [0])
    pos = np.arange(0, 1024, 16, dtype=np.uint16)  # the whole of lane 0
    col["counts"] = np.array([0, 64, 0], np.uint16)
    col["exceptions_offsets"] = np.array([0, 0, 64], np.uint64)
    col["positions"] = pos
    col["exceptions"] = np.arange(64, dtype=np.float64) + 0.5
    x, ovf = B.to_extended(col, n_vecs, np.float64)
    assert ovf == 1
    got, want = _check(cuda, col, n_vecs, True, extended=True)
    assert np.array_equal(got, want)
    plain, _ = _check(cuda, col, n_vecs, True, extended=False)
    assert not np.array_equal(got, plain)


@pytest.mark.parametrize("extended", [False, True])
def test_fused_sum_f64_fixed_tree(cuda, extended):
    f64 = True
    vals = colgen.alp_values(41, 300, True, 4, exc_rate=0.0)
    col = B.alp_encode(vals, rowgroup_vecs=100)
    c = B.to_extended(col, 300, np.float64)[0] if extended else col
    d = F.make_alp_column(c, vals.size, np.float64, extended=extended, device=cuda)
    s = F.sum_(d).cpu().numpy().view(np.uint64)[0]
    dec = B.alp_decode(c, 300, np.float64, extended=extended)
    want = np.array([B.oracle().orc_tree_sum_f64(B.ptr(dec), 300)]).view(np.uint64)[0]
    assert s == want


def test_fused_sum_many_vectors(cuda):
    """> 2048 vectors exercises the multi-level pairwise reduction."""
    col = colgen.random_alp(3, 5000, True, [10, 20], [0, 3])
    # finite exceptions: NaN payloads are not preserved by IEEE additions
    e = col["exceptions"]
    col["exceptions"] = np.where(np.isfinite(e), e, 1.5)
    dec = B.alp_decode(col, 5000, np.float64)
    d = F.make_alp_column(col, 5000 * 1024, np.float64, device=cuda)
    s = F.sum_(d).cpu().numpy().view(np.uint64)[0]
    want = np.array([B.oracle().orc_tree_sum_f64(B.ptr(dec), 5000)]).view(np.uint64)[0]
    assert s == want


@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("extended", [False, True])
def test_query(cuda, f64, extended):
    dt = _dt(f64)
    vals = colgen.alp_values(51, 60, f64, 2)
    col = B.alp_encode(vals, rowgroup_vecs=100)
    c = B.to_extended(col, 60, dt)[0] if extended else col
    d = F.make_alp_column(c, vals.size, dt, extended=extended, device=cuda)
    exc_val = float(c["exceptions"][0]) if c["exceptions"].size else float(vals[5])
    assert int(F.query(d, float(vals[4321])).item()) == 1
    if not np.isnan(exc_val):
        assert int(F.query(d, exc_val).item()) == 1
    assert int(F.query(d, 0.3214).item()) == int(np.any(vals == dt(0.3214)))


@pytest.mark.parametrize("f64", [True, False])
def test_multi_column_alp(cuda, f64):
    dt = _dt(f64)
    n = 16 * 1024
    vals = np.full(n, 2.5, dt)
    vals[5000] = 7.25
    col = B.alp_encode(vals, rowgroup_vecs=100)
    d = F.make_alp_column(col, n, dt, device=cuda)
    assert int(F.query_multi_column([d, d, d], 2.5).item()) == 1
    assert int(F.query_multi_column([d, d], 7.25).item()) == 0


# ---------------------------------------------------------------------------
# ALP-RD
# ---------------------------------------------------------------------------
def rd_column(vals: np.ndarray, rowgroup_vecs: int = 100):
    """Encodes with the oracle's rd_encoder restatement (one dictionary per
    rowgroup) into the library's ALP-RD column layout."""
    o = B.oracle()
    import ctypes
    f64 = vals.dtype == np.float64
    ut = np.uint64 if f64 else np.uint32
    bits = 64 if f64 else 32
    n_vecs = vals.size // 1024
    rp, lp, rbw, lbw, ro, lo, dicts, di, eo, ex, ps, cnt = ([] for _ in range(12))
    roff = loff = eoff = 0
    st = B.RDState()
    for v in range(n_vecs):
        if v % rowgroup_vecs == 0:
            init = o.orc_rd_init_f64 if f64 else o.orc_rd_init_f32
            rg = np.ascontiguousarray(vals[v * 1024:])
            init(B.ptr(rg), rg.size, ctypes.byref(st))
            dicts.append(np.array(st.dict[:], np.uint16))
        vec = np.ascontiguousarray(vals[v * 1024:(v + 1) * 1024])
        right = np.zeros(1024, ut)
        left = np.zeros(1024, np.uint16)
        e = np.zeros(1024, np.uint16)
        p = np.zeros(1024, np.uint16)
        enc = o.orc_rd_encode_vector_f64 if f64 else o.orc_rd_encode_vector_f32
        n = enc(B.ptr(vec), ctypes.byref(st), B.ptr(right), B.ptr(left), B.ptr(e), B.ptr(p))
        rpk = B.pack(right, st.right_bw, bits)
        lpk = B.pack(left, st.left_bw, 16)
        rp.append(rpk)
        lp.append(lpk)
        rbw.append(st.right_bw)
        lbw.append(st.left_bw)
        ro.append(roff)
        lo.append(loff)
        roff += rpk.size
        loff += lpk.size
        di.append(len(dicts) - 1)
        eo.append(eoff)
        ex.append(e[:n])
        ps.append(p[:n])
        cnt.append(n)
        eoff += n
    return dict(right_packed=np.concatenate(rp).astype(ut), right_bw=np.array(rbw, np.uint8),
                right_offsets=np.array(ro, np.uint64), left_packed=np.concatenate(lp),
                left_bw=np.array(lbw, np.uint8), left_offsets=np.array(lo, np.uint64),
                dictionaries=np.concatenate(dicts), dictionary_indices=np.array(di, np.uint32),
                exceptions_offsets=np.array(eo, np.uint64), exceptions=np.concatenate(ex),
                positions=np.concatenate(ps), counts=np.array(cnt, np.uint16))


@pytest.mark.parametrize("f64", [True, False])
def test_alprd_roundtrip(cuda, f64):
    rng = np.random.default_rng(17)
    dt, ut = _dt(f64), _ut(f64)
    vals = rng.random(250 * 1024).astype(dt)
    vals[::97] = (rng.standard_normal(vals[::97].size) * 1e6).astype(dt)
    col = rd_column(vals)
    d = F.make_alprd_column(col, vals.size, dt, device=cuda)
    got = F.decompress(d).cpu().numpy().view(ut)
    assert np.array_equal(got, vals.view(ut))
    o = B.oracle()
    want = np.zeros(vals.size, dt)
    fn = o.orc_decode_rd_f64 if f64 else o.orc_decode_rd_f32
    fn(*[B.ptr(col[k]) for k in ["right_packed", "right_offsets", "right_bw", "left_packed",
                                  "left_offsets", "left_bw", "dictionaries", "dictionary_indices",
                                  "exceptions_offsets", "exceptions", "positions", "counts"]],
       250, B.ptr(want))
    assert np.array_equal(got, want.view(ut))
