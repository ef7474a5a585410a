"""Parity at the full benchmark sizes.

* FFOR at scale: one u32 column of 2^28 values and one u64 column of 2^27
  values per tested width, random packed words and bases generated on the
  device as the benchmark does; the whole column is decoded on the GPU and
  a strided sample of its vectors (the first, the last and every 1009th,
  spread over all warps of the persistent grid and over offsets past 2^32
  bytes) is compared word for word with the oracle's decode of the same
  packed words (fls::unffor restated, src/fls/fls-bindings.hpp:8-52).
* ALP / ALP-RD: f64 columns of 2^27 values (decimals with 1% random
  exceptions; uniform [0, 1) for ALP-RD) encoded by the GPU encoders and
  decoded by flsgpu_decompress_alp_f64 / _alprd_f64: the decode returns the
  column's values bit for bit (encode -> decode identity at full size).
"""
import numpy as np
import pytest

import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu

WIDTHS = {32: (0, 1, 7, 16, 31, 32), 64: (1, 5, 20, 33, 63, 64)}
N_VALUES = {32: 2 ** 28, 64: 2 ** 27}


@pytest.mark.parametrize("bits", [32, 64])
def test_ffor_full_size_sampled_against_oracle(cuda, bits):
    import torch
    ut = np.uint64 if bits == 64 else np.uint32
    n = N_VALUES[bits]
    n_vecs = n // 1024
    nl = 1024 // bits
    g = torch.Generator(device=cuda)
    g.manual_seed(77 + bits)
    sel = sorted(set([0, n_vecs - 1] + list(range(0, n_vecs, 1009))))
    sel_t = torch.tensor(sel, dtype=torch.int64, device=cuda)
    out = torch.empty(n, dtype=torch.int64 if bits == 64 else torch.int32, device=cuda)
    for w in WIDTHS[bits]:
        col = F._synthetic_ffor(bits, w, n, g, cuda)
        F.decompress(col, out=out)
        got = out.view(n_vecs, 1024)[sel_t].cpu().numpy().view(ut)
        if w:
            pk = col.buffers["packed"].view(n_vecs, w * nl)[sel_t].cpu().numpy().view(ut).ravel()
        else:
            pk = np.zeros(1, ut)
        bases = col.buffers["bases"][sel_t].cpu().numpy().view(ut)
        bw = np.full(len(sel), w, np.uint8)
        offs = (np.arange(len(sel), dtype=np.uint64) * np.uint64(w * nl))
        want = B.decode_ffor(pk, bw, offs, bases, bits).reshape(len(sel), 1024)
        assert np.array_equal(got, want), f"u{bits} w={w}"
        del col
        torch.cuda.synchronize()


def test_alp_f64_full_size_round_trip(cuda):
    import torch
    n = 2 ** 27
    nv = n // 1024
    g = torch.Generator(device=cuda)
    g.manual_seed(5)
    ints = torch.randint(-10 ** 6, 10 ** 6 + 1, (n,), dtype=torch.int64, device=cuda, generator=g)
    p10 = torch.tensor([1.0, 10.0, 100.0, 1000.0, 10000.0], dtype=torch.float64, device=cuda)
    d = torch.randint(0, 5, (nv,), device=cuda, generator=g).repeat_interleave(1024)
    vals = ints.double() / p10[d]
    m = torch.rand(n, device=cuda, generator=g) < 0.01
    pat = torch.randint(-2 ** 63, 2 ** 63 - 1, (n,), dtype=torch.int64, device=cuda, generator=g)
    pat = torch.where(torch.isnan(pat.view(torch.float64)), pat & ~(1 << 62), pat)
    vals.view(torch.int64)[m] = pat[m]
    del ints, d, m, pat
    enc = F.AlpEncoder(seed=1)
    res = enc.encode(vals, 0)
    assert int(res.n_exceptions) > n // 200  # the 1% patterns became exceptions
    col = F.encoded_column(res, n, enc)
    got = F.decompress(col)
    assert torch.equal(got.view(torch.int64), vals.view(torch.int64))
    # and through the lane-divided exception layout built on the GPU
    xcol = F.to_extended(col)
    got = F.decompress(xcol)
    assert torch.equal(got.view(torch.int64), vals.view(torch.int64))


def test_alprd_f64_full_size_round_trip(cuda):
    import torch
    n = 2 ** 27
    g = torch.Generator(device=cuda)
    g.manual_seed(6)
    vals = torch.rand(n, dtype=torch.float64, device=cuda, generator=g)
    enc = F.AlpEncoder(seed=1)
    res = enc.encode_rd(vals, rowgroup_vecs=100)
    assert int(res.n_dictionaries) == (n // 1024 + 99) // 100
    col = F.rd_encoded_column(res, n, "f64", enc)
    got = F.decompress(col)
    assert torch.equal(got.view(torch.int64), vals.view(torch.int64))
