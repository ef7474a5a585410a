"""8- and 16-bit FastLanes columns (fls::pack / unpack / ffor / unffor for
uint8_t and uint16_t, src/fls/fls-bindings.hpp:8-52): the GPU decode
(flsgpu_decompress_{bp,ffor}_{u8,u16}) against the oracle at every width,
with mixed widths and ragged tails, and the GPU packer
(flsgpu_ffor_encode_u8 / _u16) word for word against the oracle's
fls::ffor / fls::pack restatement (pinned to the reference by
tests/test_oracle.py), round-tripping through the decode."""
import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu

UT = {8: np.uint8, 16: np.uint16}


def _oracle_decode(c, bits, bp):
    o = B.oracle()
    ut = UT[bits]
    n_vecs = c["bit_widths"].size
    out = np.zeros(n_vecs * 1024, ut)
    buf = np.zeros(1024, ut)
    pk = np.concatenate([c["packed"], np.zeros(1024, ut)])
    for v in range(n_vecs):
        src = np.ascontiguousarray(pk[int(c["vector_offsets"][v]):])
        if bp:
            getattr(o, f"orc_unpack_u{bits}")(B.ptr(src), B.ptr(buf), int(c["bit_widths"][v]))
        else:
            getattr(o, f"orc_unffor_u{bits}")(B.ptr(src), B.ptr(buf), int(c["bit_widths"][v]),
                                              int(c["bases"][v]))
        out[v * 1024:(v + 1) * 1024] = buf
    return out


@pytest.mark.parametrize("bits", [8, 16])
@pytest.mark.parametrize("bp", [False, True])
def test_small_decode_every_width(cuda, bits, bp):
    ut = UT[bits]
    for w in range(bits + 1):
        c = colgen.random_ffor(1300 + w + bits, 6, bits, [w])
        d = F.make_ffor_column(c["packed"], c["bit_widths"], c["vector_offsets"],
                               None if bp else c["bases"], c["n_values"], cuda)
        got = F.decompress(d).cpu().numpy().view(ut)
        assert np.array_equal(got, _oracle_decode(c, bits, bp)), (bits, bp, w)


@pytest.mark.parametrize("bits", [8, 16])
@pytest.mark.parametrize("n_values", [1, 1027, 9 * 1024 - 3, 40 * 1024])
def test_small_decode_mixed_widths_ragged(cuda, bits, n_values):
    import torch
    ut = UT[bits]
    n_vecs = (n_values + 1023) // 1024
    c = colgen.random_ffor(1400 + n_values, n_vecs, bits, range(bits + 1), n_values=n_values)
    d = F.make_ffor_column(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"],
                           n_values, cuda)
    pad = 4096
    out = torch.full((n_values + pad,), 0x5A, dtype=torch.uint8 if bits == 8 else torch.int16,
                     device=cuda)
    F.decompress(d, out=out[:n_values])
    got = out.cpu().numpy().view(ut)
    assert np.array_equal(got[:n_values], _oracle_decode(c, bits, False)[:n_values])
    assert np.all(got[n_values:] == ut(0x5A))  # nothing written past n_values


@pytest.mark.parametrize("bits", [8, 16])
@pytest.mark.parametrize("mode", [F.BASE_MIN, F.BASE_ZERO])
def test_small_encode_matches_oracle_and_round_trips(cuda, bits, mode):
    import torch
    ut = UT[bits]
    rng = np.random.default_rng(bits + 10 * mode)
    n_vecs = 3 * (bits + 1)
    vals = np.zeros(n_vecs * 1024, ut)
    for v in range(n_vecs):
        w = v % (bits + 1)
        base = 0 if mode == F.BASE_ZERO else int(rng.integers(0, 2 ** bits))
        d = rng.integers(0, 2 ** w, 1024) if w else np.zeros(1024, np.int64)
        if w:
            d[rng.integers(0, 1024)] = 2 ** w - 1
            d[rng.integers(0, 1024)] = 0
        vals[v * 1024:(v + 1) * 1024] = ((d + base) % 2 ** bits).astype(ut)
    t = torch.from_numpy(vals.view(np.int16) if bits == 16 else vals).to(cuda)
    col = F.ffor_encode(t, mode)
    o = B.oracle()
    nl = 1024 // bits
    packed = col.buffers["packed"].cpu().numpy().view(ut)
    bw = col.buffers["bit_widths"].cpu().numpy()
    offs = col.buffers["vector_offsets"].cpu().numpy()
    buf = np.zeros(1024, ut)
    for v in range(n_vecs):
        vec = np.ascontiguousarray(vals[v * 1024:(v + 1) * 1024])
        mn = 0 if mode == F.BASE_ZERO else int(vec.min())
        w = int(int(vec.max()) - mn).bit_length()
        assert bw[v] == w, v
        if mode == F.BASE_ZERO:
            getattr(o, f"orc_pack_u{bits}")(B.ptr(vec), B.ptr(buf), w)
        else:
            getattr(o, f"orc_ffor_u{bits}")(B.ptr(vec), B.ptr(buf), w, mn)
        assert np.array_equal(packed[int(offs[v]):int(offs[v]) + w * nl], buf[:w * nl]), v
    got = F.decompress(col).cpu().numpy().view(ut)
    assert np.array_equal(got, vals)
