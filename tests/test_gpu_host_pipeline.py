"""Pipelined decode of host-resident columns (flsgpu_host_*) against the
oracle, bit for bit: FFOR u32 / u64 and ALP f32 / f64 columns over several
chunks, with a ragged last vector and a chunk that is only partly used."""
import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("n_values", [7 * 1024, 9 * 1024 - 100, 1000])
def test_host_pipeline_ffor(cuda, bits, n_values):
    import torch
    ut = np.uint64 if bits == 64 else np.uint32
    n_vecs = (n_values + 1023) // 1024
    c = colgen.random_ffor(50 + bits, n_vecs, bits, range(bits + 1), n_values=n_values)
    sd = np.int64 if bits == 64 else np.int32
    t = [_pinned(c["packed"].view(sd) if c["packed"].size else np.zeros(1, sd)),
         _pinned(c["bit_widths"]), _pinned(c["vector_offsets"].view(np.int64)),
         _pinned(c["bases"].view(sd))]
    desc, kind, dt, keep = F.host_ffor_column(*t, n_values)
    out = torch.empty(n_values, dtype=torch.int64 if bits == 64 else torch.int32).pin_memory()
    pipe = F.HostPipeline(chunk_values=2048)  # several chunks per column
    pipe.decompress(desc, kind, dt, out)
    want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
    assert np.array_equal(out.numpy().view(ut), want[:n_values])


@pytest.mark.parametrize("f64", [True, False])
def test_host_pipeline_alp(cuda, f64):
    import torch
    n_vecs = 11
    col = colgen.random_alp(77, n_vecs, f64, range(0, 30), [0, 3, 40, 1024])
    dt = np.float64 if f64 else np.float32
    ut = np.uint64 if f64 else np.uint32
    n_values = n_vecs * 1024
    signed = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32,
              np.dtype(np.uint16): np.int16}
    keep = {k: _pinned(v.view(signed[v.dtype]) if v.dtype in signed else v)
            for k, v in col.items() if isinstance(v, np.ndarray)}
    bp = F.BPColumnC(n_values, n_vecs, keep["packed"].data_ptr(), keep["bit_widths"].data_ptr(),
                     keep["vector_offsets"].data_ptr())
    ff = F.FFORColumnC(n_values, bp, keep["bases"].data_ptr())
    exc = keep["exceptions"]
    c = F.ALPColumnC(n_values, ff, None, None, keep["factor_indices"].data_ptr(),
                     keep["fraction_indices"].data_ptr(), int(exc.numel()),
                     keep["exceptions_offsets"].data_ptr(), exc.data_ptr(),
                     keep["positions"].data_ptr(), keep["counts"].data_ptr())
    out = torch.empty(n_values, dtype=torch.float64 if f64 else torch.float32).pin_memory()
    pipe = F.HostPipeline(chunk_values=3072)
    pipe.decompress(c, "alp", "f64" if f64 else "f32", out)
    want = B.alp_decode(col, n_vecs, dt).view(ut)
    assert np.array_equal(out.numpy().view(ut), want)


def test_host_pipeline_async_series(cuda):
    """Several columns queued without waiting, then one sync: every output
    matches the oracle."""
    import torch
    pipe = F.HostPipeline(chunk_values=2048)
    jobs = []
    for i, (bits, n_values) in enumerate([(32, 5 * 1024 + 3), (64, 3 * 1024), (32, 2048)]):
        n_vecs = (n_values + 1023) // 1024
        c = colgen.random_ffor(70 + i, n_vecs, bits, range(bits + 1), n_values=n_values)
        sd = np.int64 if bits == 64 else np.int32
        t = [_pinned(c["packed"].view(sd)), _pinned(c["bit_widths"]),
             _pinned(c["vector_offsets"].view(np.int64)), _pinned(c["bases"].view(sd))]
        desc, kind, dt, keep = F.host_ffor_column(*t, n_values)
        out = torch.empty(n_values, dtype=torch.int64 if bits == 64 else torch.int32).pin_memory()
        pipe.decompress(desc, kind, dt, out, wait=False)
        jobs.append((c, bits, n_values, out, keep, desc))
    pipe.sync()
    for c, bits, n_values, out, *_ in jobs:
        ut = np.uint64 if bits == 64 else np.uint32
        want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
        assert np.array_equal(out.numpy().view(ut), want[:n_values])


def test_host_pipeline_rejects_offsets_outside_the_chunk(cuda):
    """A vector in the middle of a chunk whose packed words (or exceptions)
    lie outside the chunk's staged range is refused before any copy, with
    FLSGPU_ERR_INVALID_ARGUMENT: the decode would otherwise read outside the
    staging slot."""
    import torch
    n_vecs, bits = 6, 32
    c = colgen.random_ffor(90, n_vecs, bits, [5, 9])
    offs = c["vector_offsets"].copy()
    offs[1] = offs[4] + 10_000  # second vector of the first chunk points far past it
    t = [_pinned(c["packed"].view(np.int32)), _pinned(c["bit_widths"]),
         _pinned(offs.view(np.int64)), _pinned(c["bases"].view(np.int32))]
    desc, kind, dt, keep = F.host_ffor_column(*t, n_vecs * 1024)
    out = torch.empty(n_vecs * 1024, dtype=torch.int32).pin_memory()
    pipe = F.HostPipeline(chunk_values=3072)
    with pytest.raises(F.FlsgpuError) as e:
        pipe.decompress(desc, kind, dt, out)
    assert e.value.status == 1 and "outside its chunk" in str(e.value)

    col = colgen.random_alp(91, n_vecs, True, [8], [4])
    col["exceptions_offsets"] = col["exceptions_offsets"].copy()
    col["exceptions_offsets"][1] = 10_000
    signed = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32,
              np.dtype(np.uint16): np.int16}
    keep = {k: _pinned(v.view(signed[v.dtype]) if v.dtype in signed else v)
            for k, v in col.items() if isinstance(v, np.ndarray)}
    n_values = n_vecs * 1024
    bp = F.BPColumnC(n_values, n_vecs, keep["packed"].data_ptr(), keep["bit_widths"].data_ptr(),
                     keep["vector_offsets"].data_ptr())
    ac = F.ALPColumnC(n_values, F.FFORColumnC(n_values, bp, keep["bases"].data_ptr()), None, None,
                      keep["factor_indices"].data_ptr(), keep["fraction_indices"].data_ptr(),
                      int(keep["exceptions"].numel()), keep["exceptions_offsets"].data_ptr(),
                      keep["exceptions"].data_ptr(), keep["positions"].data_ptr(),
                      keep["counts"].data_ptr())
    outf = torch.empty(n_values, dtype=torch.float64).pin_memory()
    with pytest.raises(F.FlsgpuError) as e:
        F.HostPipeline(chunk_values=3072).decompress(ac, "alp", "f64", outf)
    assert e.value.status == 1 and "outside its chunk" in str(e.value)
