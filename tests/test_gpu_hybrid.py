"""Hybrid ALP / ALP-RD columns (flsgpu_alp_encode_hybrid_f64,
flsgpu_decompress_alphybrid_f64): the GPU encoder sends the vectors that
call for ALP-RD to the ALP-RD encoder with a dictionary of their own and
keeps the others ALP.  Mode 0 (plain search) is checked against the oracle
vector by vector: the scheme is the oracle search's ALP-RD decision (best
estimate at the 48-bit limit, encoder.hpp:208-211), ALP vectors are byte
for byte the oracle encoder's, ALP-RD vectors are byte for byte
orc_rd_init_f64 + orc_rd_encode_vector_f64 run on the vector alone.  Every
column decodes bit for bit; the learned mode routes the network's ALP-RD
class to the ALP-RD encoder, keeps the ratio within 1% of the plain search
and falls back rarely on the vectors that ALP encodes well."""
import ctypes

import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu


def _host(ptr, n, dt):
    return F.device_array(ptr, max(n, 1), dt).cpu().numpy().view(dt)[:n]


def _oracle_label(vec):
    r = B.oracle().orc_alp_vector_best_f64(B.ptr(np.ascontiguousarray(vec)), None)
    return None if r < 0 else (r // 32, r % 32)


def _check_hybrid_against_oracle(res, vals):
    o = B.oracle()
    n_vecs = vals.size // 1024
    h = res.column
    a, r = h.alp, h.rd
    sch = _host(h.schemes, n_vecs, np.uint8)
    # ALP sub-column
    bw = _host(a.ffor.bp.bit_widths, n_vecs, np.uint8)
    offs = _host(a.ffor.bp.vector_offsets, n_vecs, np.uint64)
    base = _host(a.ffor.bases, n_vecs, np.uint64)
    fac = _host(a.factor_indices, n_vecs, np.uint8)
    exp = _host(a.fraction_indices, n_vecs, np.uint8)
    counts = _host(a.counts, n_vecs, np.uint16)
    eoffs = _host(a.exceptions_offsets, n_vecs, np.uint64)
    packed = _host(a.ffor.bp.packed_array, int(res.n_packed_words), np.uint64)
    exc = _host(a.exceptions, int(res.n_exceptions), np.float64)
    pos = _host(a.positions, int(res.n_exceptions), np.uint16)
    # ALP-RD sub-column
    rbw = _host(r.right.bit_widths, n_vecs, np.uint8)
    roff = _host(r.right.vector_offsets, n_vecs, np.uint64)
    lbw = _host(r.left.bit_widths, n_vecs, np.uint8)
    loff = _host(r.left.vector_offsets, n_vecs, np.uint64)
    di = _host(r.dictionary_indices, n_vecs, np.uint32)
    dicts = _host(r.dictionaries, 8 * n_vecs, np.uint16)
    rcounts = _host(r.counts, n_vecs, np.uint16)
    reoff = _host(r.exceptions_offsets, n_vecs, np.uint64)
    right = _host(r.right.packed_array, int(res.n_right_words), np.uint64)
    left = _host(r.left.packed_array, int(res.n_left_words), np.uint16)
    rexc = _host(r.exceptions, int(res.n_rd_exceptions), np.uint16)
    rpos = _host(r.positions, int(res.n_rd_exceptions), np.uint16)
    n_rd = 0
    for i in range(n_vecs):
        vec = np.ascontiguousarray(vals[i * 1024:(i + 1) * 1024])
        pair = _oracle_label(vec)
        if pair is None:
            n_rd += 1
            assert sch[i] == 1 and bw[i] == 0 and counts[i] == 0, i
            st = B.RDState()
            o.orc_rd_init_f64(B.ptr(vec), 1024, ctypes.byref(st))
            ds = int(st.dict_size)
            assert di[i] == i and rbw[i] == st.right_bw and lbw[i] == st.left_bw, i
            assert list(dicts[8 * i:8 * i + ds]) == list(st.dict[:ds]), i
            rp = np.zeros(1024, np.uint64)
            lp = np.zeros(1024, np.uint16)
            ex = np.zeros(1024, np.uint16)
            ps = np.zeros(1024, np.uint16)
            n = o.orc_rd_encode_vector_f64(B.ptr(vec), ctypes.byref(st), B.ptr(rp), B.ptr(lp),
                                           B.ptr(ex), B.ptr(ps))
            assert rcounts[i] == n, i
            buf = np.zeros(1024, np.uint64)
            o.orc_pack_u64(B.ptr(rp), B.ptr(buf), int(st.right_bw))
            nr = 16 * int(st.right_bw)
            assert np.array_equal(right[int(roff[i]):int(roff[i]) + nr], buf[:nr]), i
            lbuf = np.zeros(1024, np.uint16)
            o.orc_pack_u16(B.ptr(lp), B.ptr(lbuf), int(st.left_bw))
            nl = 64 * int(st.left_bw)
            assert np.array_equal(left[int(loff[i]):int(loff[i]) + nl], lbuf[:nl]), i
            e0 = int(reoff[i])
            assert np.array_equal(rexc[e0:e0 + n], ex[:n]) and np.array_equal(rpos[e0:e0 + n], ps[:n])
            continue
        assert sch[i] == 0 and rbw[i] == 0 and lbw[i] == 0 and rcounts[i] == 0, i
        assert (int(exp[i]), int(fac[i])) == pair, i
        ints = np.zeros(1024, np.int64)
        ex = np.zeros(1024, np.float64)
        ps = np.zeros(1024, np.uint16)
        n_exc = o.orc_alp_encode_vector_f64(B.ptr(vec), int(exp[i]), int(fac[i]), B.ptr(ints),
                                            B.ptr(ex), B.ptr(ps))
        assert n_exc == counts[i], i
        e0 = int(eoffs[i])
        assert np.array_equal(pos[e0:e0 + n_exc], ps[:n_exc])
        assert np.array_equal(exc[e0:e0 + n_exc].view(np.uint64), ex[:n_exc].view(np.uint64))
        mn = int(ints.min())
        w = int(int(ints.max()) - mn).bit_length()
        assert w == bw[i] and (mn & (2 ** 64 - 1)) == int(base[i]), i
        buf = np.zeros(1024, np.uint64)
        o.orc_ffor_u64(B.ptr(ints.view(np.uint64)), B.ptr(buf), w, mn & (2 ** 64 - 1))
        assert np.array_equal(packed[int(offs[i]):int(offs[i]) + 16 * w], buf[:16 * w]), i
    assert res.n_rd_vectors == n_rd and res.n_alp_vectors == n_vecs - n_rd
    return sch


def _decode(res, vals, enc):
    col = F.hybrid_column(res, vals.size, enc)
    return F.decompress(col).cpu().numpy().view(np.uint64)


def test_hybrid_plain_matches_oracle(cuda):
    import torch
    n_vecs = 400
    vals = colgen.learned_values(31, n_vecs)
    vals[3 * 1024 + 5] = np.nan
    vals[7 * 1024:8 * 1024] = np.random.default_rng(1).random(1024)  # full-mantissa noise
    enc = F.AlpEncoder(seed=1)
    res = enc.encode_hybrid(torch.from_numpy(vals).to(cuda), 0)
    sch = _check_hybrid_against_oracle(res, vals)
    assert 0 < sch.sum() < n_vecs
    assert np.array_equal(_decode(res, vals, enc), vals.view(np.uint64))


def test_hybrid_single_scheme_columns(cuda):
    """Pure ALP data gives no ALP-RD vector and the ALP-only encoder's bytes;
    uniform [0, 1) doubles with full mantissas are ALP-RD throughout."""
    import torch
    enc = F.AlpEncoder(seed=2)
    alp = colgen.alp_values(3, 60, True, 4, exc_rate=0.0)
    d = torch.from_numpy(alp).to(cuda)
    res = enc.encode_hybrid(d, 0)
    assert res.n_rd_vectors == 0
    hyb_words = _host(res.column.alp.ffor.bp.packed_array, int(res.n_packed_words), np.uint64).copy()
    assert np.array_equal(_decode(res, alp, enc), alp.view(np.uint64))
    only = enc.encode(d, 0)
    assert only.n_packed_words == res.n_packed_words
    assert np.array_equal(_host(only.column.ffor.bp.packed_array, int(only.n_packed_words),
                                np.uint64), hyb_words)
    rd = np.random.default_rng(4).random(50 * 1024)
    res = enc.encode_hybrid(torch.from_numpy(rd).to(cuda), 0)
    assert res.n_rd_vectors == 50 and res.n_packed_words == 0
    _check_hybrid_against_oracle(res, rd)
    assert np.array_equal(_decode(res, rd, enc), rd.view(np.uint64))


def test_hybrid_learned_routes_rd_and_keeps_ratio(cuda):
    import torch
    train = torch.from_numpy(colgen.learned_values(21, 16384)).to(cuda)
    test = colgen.learned_values(22, 2048)
    d_test = torch.from_numpy(test).to(cuda)
    enc = F.AlpEncoder(seed=5)
    enc.train(train, epochs=12, batch=1024, lr=3e-3)
    plain = enc.encode_hybrid(d_test, 0)
    p_bytes = plain.compressed_bytes
    p_sch = _host(plain.column.schemes, 2048, np.uint8).copy()
    p_cnt = _host(plain.column.alp.counts, 2048, np.uint16).copy()
    assert np.array_equal(_decode(plain, test, enc), test.view(np.uint64))
    learned = enc.encode_hybrid(d_test, 1)
    l_flags = _host(learned.d_flags, 2048, np.uint8).copy()
    assert np.array_equal(_decode(learned, test, enc), test.view(np.uint64))
    ratio_p, ratio_l = test.nbytes / p_bytes, test.nbytes / learned.compressed_bytes
    assert ratio_l >= 0.99 * ratio_p, (ratio_l, ratio_p)
    # ALP-RD vectors go to the ALP-RD encoder instead of the plain search:
    # most of the plain search's ALP-RD vectors are ALP-RD in the learned
    # column too, and they do not fall back
    rd_p = p_sch == 1
    rd_l = (l_flags & 2) != 0
    assert (rd_p & rd_l).sum() >= 0.9 * rd_p.sum(), ((rd_p & rd_l).sum(), rd_p.sum())
    # on the part of the data that ALP encodes well (ALP under the plain
    # search with at most 3% exceptions) the proposal rarely falls back
    friendly = (p_sch == 0) & (p_cnt <= 30)
    fb = (l_flags & 1) != 0
    assert friendly.sum() > 500
    assert (fb & friendly).sum() <= 0.05 * friendly.sum(), ((fb & friendly).sum(), friendly.sum())
    # and the hybrid column is smaller than the ALP-only one
    alp_only = enc.encode(d_test, 0)
    assert p_bytes < alp_only.compressed_bytes
