"""GPU ALP-RD encoder (flsgpu_alprd_encode_f64 / _f32) against the oracle's
restatement of rd_encoder::init and rd_encoder::encode (orc_rd_init_*,
orc_rd_encode_vector_*, pinned to the reference's rd.hpp by
tests/test_oracle.py): per rowgroup the cut, the left width and the
dictionary; per vector the packed right parts, the packed dictionary
indices, the exceptions and their positions, word for word; and the column
decodes bit for bit through flsgpu_decompress_alprd_*."""
import ctypes

import numpy as np
import pytest

import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu


def _values(kind, n_vecs, seed, f64=True):
    rng = np.random.default_rng(seed)
    n = n_vecs * 1024
    if kind == "uniform01":
        v = rng.random(n)
    elif kind == "wide":  # many distinct exponents: exceptions at every cut
        v = rng.standard_normal(n) * np.exp(rng.standard_normal(n) * 3)
    elif kind == "mantissa_noise":
        v = (rng.random(n) * 2.0 - 1.0) * 1000.0
    elif kind == "constant":
        v = np.full(n, 0.7)
    elif kind == "nine_ties":
        # nine exponents with equal counts in every sample: the dictionary
        # keeps the eight smaller left parts, the ninth is an exception
        e = np.arange(n) % 9
        v = (1.0 + rng.random(n)) * np.exp2(e - 20)
    elif kind == "specials":
        v = rng.random(n)
        v[rng.random(n) < 0.01] = np.nan
        v[rng.random(n) < 0.01] = -np.inf
        v[rng.random(n) < 0.01] = -0.0
    else:
        raise ValueError(kind)
    return v.astype(np.float64 if f64 else np.float32)


def _host(ptr, n, dt):
    return F.device_array(ptr, n, dt).cpu().numpy().view(dt)


def _check_column(vals, res, rg_vecs, f64):
    o = B.oracle()
    dt, ut, tb = (np.float64, np.uint64, 64) if f64 else (np.float32, np.uint32, 32)
    suf = "f64" if f64 else "f32"
    n_vecs = vals.size // 1024
    c = res.column
    rbw = _host(c.right.bit_widths, n_vecs, np.uint8)
    roff = _host(c.right.vector_offsets, n_vecs, np.uint64)
    lbw = _host(c.left.bit_widths, n_vecs, np.uint8)
    loff = _host(c.left.vector_offsets, n_vecs, np.uint64)
    di = _host(c.dictionary_indices, n_vecs, np.uint32)
    counts = _host(c.counts, n_vecs, np.uint16)
    eoff = _host(c.exceptions_offsets, n_vecs, np.uint64)
    n_rg = (n_vecs + rg_vecs - 1) // rg_vecs
    dicts = _host(c.dictionaries, n_rg * 8, np.uint16)
    right = _host(c.right.packed_array, max(int(res.n_right_words), 1), ut)
    left = _host(c.left.packed_array, max(int(res.n_left_words), 2), np.uint16)
    n_exc = int(res.n_exceptions)
    exc = _host(c.exceptions, max(n_exc, 1), np.uint16)
    pos = _host(c.positions, max(n_exc, 1), np.uint16)
    assert int(res.n_dictionaries) == n_rg
    nl = 1024 // tb
    rbuf = np.zeros(1024, ut)
    lbuf = np.zeros(1024, np.uint16)
    for r in range(n_rg):
        v0, v1 = r * rg_vecs, min(n_vecs, (r + 1) * rg_vecs)
        rg = np.ascontiguousarray(vals[v0 * 1024:v1 * 1024])
        st = B.RDState()
        getattr(o, f"orc_rd_init_{suf}")(B.ptr(rg), rg.size, ctypes.byref(st))
        ds = int(st.dict_size)
        assert list(dicts[8 * r:8 * r + ds]) == list(st.dict[:ds]), (r, dicts[8 * r:8 * r + 8])
        for v in range(v0, v1):
            assert di[v] == r and rbw[v] == st.right_bw and lbw[v] == st.left_bw, v
            vec = np.ascontiguousarray(vals[v * 1024:(v + 1) * 1024])
            rp = np.zeros(1024, ut)
            lp = np.zeros(1024, np.uint16)
            ex = np.zeros(1024, np.uint16)
            ps = np.zeros(1024, np.uint16)
            n = getattr(o, f"orc_rd_encode_vector_{suf}")(B.ptr(vec), ctypes.byref(st), B.ptr(rp),
                                                          B.ptr(lp), B.ptr(ex), B.ptr(ps))
            assert counts[v] == n, v
            getattr(o, f"orc_pack_u{tb}")(B.ptr(rp), B.ptr(rbuf), int(st.right_bw))
            nr = int(st.right_bw) * nl
            assert np.array_equal(right[int(roff[v]):int(roff[v]) + nr], rbuf[:nr]), v
            o.orc_pack_u16(B.ptr(lp), B.ptr(lbuf), int(st.left_bw))
            nlw = int(st.left_bw) * 64
            assert np.array_equal(left[int(loff[v]):int(loff[v]) + nlw], lbuf[:nlw]), v
            e0 = int(eoff[v])
            assert np.array_equal(exc[e0:e0 + n], ex[:n]) and np.array_equal(pos[e0:e0 + n], ps[:n]), v


@pytest.mark.parametrize("kind,n_vecs,rg", [
    ("uniform01", 250, 100), ("wide", 130, 100), ("mantissa_noise", 37, 1),
    ("constant", 5, 100), ("nine_ties", 24, 12), ("specials", 40, 13)])
@pytest.mark.parametrize("f64", [True, False])
def test_rd_encoder_matches_oracle_word_for_word(cuda, kind, n_vecs, rg, f64):
    import torch
    vals = _values(kind, n_vecs, 400 + n_vecs, f64)
    enc = F.AlpEncoder(seed=1)
    res = enc.encode_rd(torch.from_numpy(vals).to(cuda), rowgroup_vecs=rg)
    _check_column(vals, res, rg, f64)
    col = F.rd_encoded_column(res, vals.size, "f64" if f64 else "f32", enc)
    got = F.decompress(col).cpu().numpy()
    ut = np.uint64 if f64 else np.uint32
    assert np.array_equal(got.view(ut), vals.view(ut))


def test_rd_encoder_rejects_bad_arguments(cuda):
    import torch
    enc = F.AlpEncoder(seed=1)
    v = torch.zeros(2048, dtype=torch.float64, device=cuda)
    for rg in (0, 101):
        with pytest.raises(F.FlsgpuError):
            enc.encode_rd(v, rowgroup_vecs=rg)
    with pytest.raises(F.FlsgpuError):
        enc.encode_rd(v[:1000], rowgroup_vecs=100)
