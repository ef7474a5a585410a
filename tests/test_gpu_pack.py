"""GPU FastLanes packing (flsgpu_ffor_encode_*) against the oracle's
restatement of fls::ffor / fls::pack (oracle/oracle.c, pinned against the
reference's own pack/ffor by tests/test_oracle.py): per-vector base and
width, packed words word for word, and decode round trips, at every width
of u16 / u32 / u64, for the three base rules."""
import numpy as np
import pytest

import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu

UT = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}
ST = {8: np.uint8, 16: np.int16, 32: np.int32, 64: np.int64}


def _values(rng, bits, n_vecs, widths, signed=False, zero_base=False):
    """Per vector: width from `widths`, base uniform (signed: around 0),
    values base + [0, 2^w) modulo 2^bits, with 0 and 2^w - 1 both present."""
    out = np.zeros(n_vecs * 1024, np.uint64)
    for v in range(n_vecs):
        w = int(widths[v % len(widths)])
        if zero_base:
            base = 0
        elif signed:
            base = int(rng.integers(-2 ** (bits - 2), 2 ** (bits - 2)))
        else:
            base = int(rng.integers(0, 2 ** bits, dtype=np.uint64))
        d = rng.integers(0, 2 ** w, 1024, dtype=np.uint64) if w else np.zeros(1024, np.uint64)
        if w:
            d[rng.integers(0, 1024)] = 2 ** w - 1   # the width is reached
            d[rng.integers(0, 1024)] = 0
        out[v * 1024:(v + 1) * 1024] = np.uint64(base % 2 ** 64) + d   # wraps mod 2^64
    if bits == 32:
        out &= np.uint64(0xFFFFFFFF)
    return out.astype(UT[bits])


def _expected(vals, bits, mode):
    o = B.oracle()
    ut = UT[bits]
    n_vecs = vals.size // 1024
    nl = 1024 // bits
    packed, bws, bases = [], [], []
    for v in range(n_vecs):
        vec = np.ascontiguousarray(vals[v * 1024:(v + 1) * 1024])
        if mode == F.BASE_SIGNED_MIN:
            mn = int(vec.view(ST[bits]).min()) % 2 ** bits
        elif mode == F.BASE_MIN:
            mn = int(vec.min())
        else:
            mn = 0
        d = (vec.astype(object) - mn) % 2 ** bits
        w = int(max(d)).bit_length()
        buf = np.zeros(1024, ut)
        if mode == F.BASE_ZERO or bits == 16:
            assert mn == 0 or bits == 16
            if bits == 16:
                dd = np.array([int(x) for x in d], ut)
                getattr(o, "orc_pack_u16")(B.ptr(dd), B.ptr(buf), w)
            else:
                getattr(o, f"orc_pack_u{bits}")(B.ptr(vec), B.ptr(buf), w)
        else:
            getattr(o, f"orc_ffor_u{bits}")(B.ptr(vec), B.ptr(buf), w, mn)
        packed.append(buf[:w * nl])
        bws.append(w)
        bases.append(mn)
    return (np.concatenate(packed) if packed else np.zeros(0, ut), np.array(bws),
            np.array(bases, dtype=object))


def _run(cuda, vals, bits, mode):
    import torch
    t = torch.from_numpy(vals.view(ST[bits])).to(cuda)
    r = F.ffor_encode(t, mode)
    bufs = r if isinstance(r, dict) else r.buffers
    got_packed = bufs["packed"].cpu().numpy().view(UT[bits])
    got_bw = bufs["bit_widths"].cpu().numpy()
    got_offs = bufs["vector_offsets"].cpu().numpy()
    return r, got_packed, got_bw, got_offs, bufs


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_ffor_encode_matches_oracle_every_width(cuda, bits, mode):
    rng = np.random.default_rng(bits * 10 + mode)
    widths = list(range(bits + 1))
    vals = _values(rng, bits, len(widths) * 2, widths, signed=(mode == 1), zero_base=(mode == 2))
    want_packed, want_bw, want_base = _expected(vals, bits, mode)
    col, packed, bw, offs, bufs = _run(cuda, vals, bits, mode)
    assert np.array_equal(bw, want_bw)
    nl = 1024 // bits
    assert np.array_equal(offs, np.concatenate([[0], np.cumsum(want_bw * nl)[:-1]]))
    assert np.array_equal(packed, want_packed)
    if mode != 2:
        got_base = bufs["bases"].cpu().numpy().view(UT[bits]).astype(object)
        assert [int(x) for x in got_base] == [int(x) for x in want_base]
    # round trip through the decoder
    got = F.decompress(col).cpu().numpy().view(UT[bits])
    assert np.array_equal(got, vals)


def test_bp_encode_u16_matches_oracle(cuda):
    rng = np.random.default_rng(16)
    n_vecs = 34
    vals = np.zeros(n_vecs * 1024, np.uint16)
    for v in range(n_vecs):
        w = v % 17
        vals[v * 1024:(v + 1) * 1024] = rng.integers(0, 2 ** w, 1024) if w else 0
    want_packed, want_bw, _ = _expected(vals, 16, F.BASE_ZERO)
    r, packed, bw, offs, _ = _run(cuda, vals, 16, F.BASE_ZERO)
    assert np.array_equal(bw, want_bw)
    assert np.array_equal(packed, want_packed)
    assert r.n_packed == want_packed.size


def test_ffor_encode_edges(cuda):
    import torch
    # constant vectors (width 0), the full unsigned range, one vector
    for bits, dt in ((32, torch.int32), (64, torch.int64)):
        z = torch.full((1024,), 7, dtype=dt, device=cuda)
        col = F.ffor_encode(z)
        assert col.n_packed == 0
        assert torch.equal(F.decompress(col), z)
        full = torch.tensor(np.array([0, -1] * 512, ST[bits]), device=cuda)
        col = F.ffor_encode(full)
        assert int(col.buffers["bit_widths"][0]) == bits
        assert torch.equal(F.decompress(col), full)
    with pytest.raises(F.FlsgpuError):
        F.ffor_encode(torch.zeros(1000, dtype=torch.int32, device=cuda))
