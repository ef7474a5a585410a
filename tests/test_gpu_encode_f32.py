"""The f32 GPU ALP encoder (flsgpu_alp_encode_f32) against the oracle's
restatement of the reference's float encoder (pinned to alp::encode by
tests/test_oracle.py): per vector the pair of the plain search over its 32
samples, the exceptions (positions and values), the base and width of the
FFOR analysis and the packed words, word for word; the column decodes bit
for bit through flsgpu_decompress_alp_f32."""
import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu


def _check(vals, res, n_vecs):
    o = B.oracle()
    c = res.column
    host = lambda ptr, n, dt: F.device_array(ptr, max(n, 1), dt).cpu().numpy().view(dt)[:n]  # noqa: E731
    bw = host(c.ffor.bp.bit_widths, n_vecs, np.uint8)
    offs = host(c.ffor.bp.vector_offsets, n_vecs, np.uint64)
    base = host(c.ffor.bases, n_vecs, np.uint32)
    fac = host(c.factor_indices, n_vecs, np.uint8)
    exp = host(c.fraction_indices, n_vecs, np.uint8)
    counts = host(c.counts, n_vecs, np.uint16)
    eoffs = host(c.exceptions_offsets, n_vecs, np.uint64)
    packed = host(c.ffor.bp.packed_array, int(res.n_packed_words), np.uint32)
    exc = host(c.exceptions, int(res.n_exceptions), np.float32)
    pos = host(c.positions, int(res.n_exceptions), np.uint16)
    for i in range(n_vecs):
        vec = np.ascontiguousarray(vals[i * 1024:(i + 1) * 1024])
        r = o.orc_alp_vector_best_f32(B.ptr(vec), None)
        assert (int(exp[i]), int(fac[i])) == (r // 32, r % 32), i
        ints = np.zeros(1024, np.int32)
        ex = np.zeros(1024, np.float32)
        ps = np.zeros(1024, np.uint16)
        n = o.orc_alp_encode_vector_f32(B.ptr(vec), int(exp[i]), int(fac[i]), B.ptr(ints),
                                        B.ptr(ex), B.ptr(ps))
        assert counts[i] == n, i
        e0 = int(eoffs[i])
        assert np.array_equal(pos[e0:e0 + n], ps[:n]), i
        assert np.array_equal(exc[e0:e0 + n].view(np.uint32), ex[:n].view(np.uint32)), i
        mn = int(ints.min())
        w = int((int(ints.max()) - mn) % 2 ** 32).bit_length()
        assert bw[i] == w and int(base[i]) == mn % 2 ** 32, i
        buf = np.zeros(1024, np.uint32)
        o.orc_ffor_u32(B.ptr(ints.view(np.uint32)), B.ptr(buf), w, mn % 2 ** 32)
        assert np.array_equal(packed[int(offs[i]):int(offs[i]) + 32 * w], buf[:32 * w]), i


def test_f32_encoder_matches_oracle(cuda):
    import torch
    rng = np.random.default_rng(3)
    parts = [colgen.alp_values(31, 60, False, 3),                       # 1% exceptions
             colgen.alp_values(32, 20, False, 0, exc_rate=0.0),          # integers
             rng.random(5 * 1024).astype(np.float32),                    # full mantissa
             np.full(1024, np.nan, np.float32),                          # all exceptions
             np.concatenate([np.full(1023, np.inf, np.float32), [2.5]]).astype(np.float32),
             np.full(1024, -3.75, np.float32),                           # constant
             (np.round(rng.uniform(-1e5, 1e5, 1024), 2)).astype(np.float32)]
    vals = np.concatenate(parts).astype(np.float32)
    vals[100] = -0.0
    n_vecs = vals.size // 1024
    enc = F.AlpEncoder(seed=1)
    res = enc.encode_f32(torch.from_numpy(vals).to(cuda))
    _check(vals, res, n_vecs)
    col = F.encoded_column(res, vals.size, enc, dtype="f32")
    got = F.decompress(col).cpu().numpy().view(np.uint32)
    assert np.array_equal(got, vals.view(np.uint32))
    assert res.n_rd >= 5  # the full-mantissa vectors call for ALP-RD


def test_f32_encoder_bench_shape_round_trip(cuda):
    """The f32 column of the ALP decode benchmark at 2^20 values: integers in
    [-10^6, 10^6] times the float 10^-d (d in 0..3 per vector, the product
    ALP's decoder forms), 1% of positions random non-NaN patterns: exact
    decode and about the injected exceptions."""
    import torch
    rng = np.random.default_rng(77)
    n_vecs = 1024
    frac = np.array([1.0, 0.1, 0.01, 0.001], np.float32)
    ints = rng.integers(-10 ** 6, 10 ** 6 + 1, n_vecs * 1024).astype(np.float32)
    vals = (ints * np.repeat(frac[rng.integers(0, 4, n_vecs)], 1024)).astype(np.float32)
    m = rng.random(vals.size) < 0.01
    pat = rng.integers(0, 2 ** 32, int(m.sum()), dtype=np.uint64).astype(np.uint32)
    pat[np.isnan(pat.view(np.float32))] &= np.uint32(0xBFFFFFFF)
    vals.view(np.uint32)[m] = pat
    enc = F.AlpEncoder(seed=2)
    res = enc.encode_f32(torch.from_numpy(vals).to(cuda))
    got = F.decompress(F.encoded_column(res, vals.size, enc, dtype="f32")).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), vals.view(np.uint32))
    assert 0.8 * m.sum() < res.n_exceptions < 1.5 * m.sum()
    assert res.compressed_bytes < vals.nbytes * 0.8
