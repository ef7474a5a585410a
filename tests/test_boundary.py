"""The reference-facing layers above the C ABI:
  * the C++ drop-in shim (msc-thesis-project_b200/cpp/flsgpu_bindings.hpp):
    a test program written against the reference's API (host columns,
    copy_to_device, bindings::decompress_column / query_column /
    compute_column / query_multi_column, host::ALPColumn::
    create_extended_column, host::free_column) compiles, and decodes bit for
    bit like the oracle;
  * the device-side decoders (include/flsgpu_b200_device.cuh): user kernels
    in the reference's style (one thread per lane, Decompressor +
    unpack_next_into) compile and decode bit for bit like the oracle, one or
    four values per call;
  * the GPU conversion to the lane-divided exception layout
    (flsgpu_alp_to_extended_*) equals the oracle's restatement of
    create_extended_column, overflow of a 6-bit lane count included."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

ROOT = Path(__file__).resolve().parents[1]
NVCC = "/usr/local/cuda/bin/nvcc"
PKG = ROOT / "msc-thesis-project_b200"


def _compile(src: Path, out: Path, extra):
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
           "-Xcompiler", "-fPIC", "-shared", "-I", str(ROOT / "include"), *extra, "-o", str(out),
           str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


@pytest.fixture(scope="session")
def built(tmp_path_factory):
    d = tmp_path_factory.mktemp("boundary")
    F.lib()  # the library the shim links against is built
    shim = _compile(ROOT / "tests" / "cpp" / "shim_consumer.cu", d / "libshim.so",
                    ["-L", str(PKG), "-lflsgpu_b200", "-Xlinker", f"-rpath,{PKG}"])
    dev = _compile(ROOT / "tests" / "cpp" / "device_api_kernels.cu", d / "libdevapi.so", [])
    return shim, dev


def test_shim_and_device_header_build_and_export(built):
    shim, dev = built
    s = C.CDLL(str(shim))
    for n in ("shim_decompress_ffor_u32", "shim_decompress_ffor_u64", "shim_query_ffor_u32",
              "shim_compute_ffor_u64", "shim_query_multi_column_ffor_u32",
              "shim_decompress_alp_f32", "shim_decompress_alp_f64"):
        assert hasattr(s, n), n
    d = C.CDLL(str(dev))
    for k in ("bp_u32", "bp_u64", "ffor_u32", "ffor_u64", "alp_f32", "alp_f64", "alpx_f32",
              "alpx_f64"):
        assert hasattr(d, "user_decode_" + k), k


def test_shim_read_file_as(built, tmp_path):
    """data::arrays::read_file_as: whole vectors of the file, repeated when
    the file is shorter than the count asked for; errors as exceptions."""
    s = C.CDLL(str(built[0]))
    vals = np.random.default_rng(1).standard_normal(2500)
    path = tmp_path / "col.bin"
    vals.tofile(path)
    out = np.zeros(8192, np.float64)
    n = C.c_size_t(0)
    assert s.shim_read_file_f64(str(path).encode(), C.c_size_t(0), _p(out), C.byref(n)) == 0
    assert n.value == 2048 and np.array_equal(out[:2048], vals[:2048])
    assert s.shim_read_file_f64(str(path).encode(), C.c_size_t(7000), _p(out), C.byref(n)) == 0
    assert n.value == 6144
    assert np.array_equal(out[:6144], np.resize(vals, 6144))
    (tmp_path / "bad.bin").write_bytes(b"12345")
    assert s.shim_read_file_f64(str(tmp_path / "bad.bin").encode(), C.c_size_t(0), _p(out),
                                C.byref(n)) == 1
    assert s.shim_read_file_f64(str(tmp_path / "missing.bin").encode(), C.c_size_t(0), _p(out),
                                C.byref(n)) == 1


def _p(a):
    return C.c_void_p(a.ctypes.data) if a.size else C.c_void_p(16)


@pytest.mark.gpu
@pytest.mark.parametrize("bits", [32, 64])
def test_shim_ffor_decode_query_compute(cuda, built, bits):
    s = C.CDLL(str(built[0]))
    ut = np.uint64 if bits == 64 else np.uint32
    ct = C.c_uint64 if bits == 64 else C.c_uint32
    suf = f"u{bits}"
    c = colgen.random_ffor(900 + bits, 37, bits, range(bits + 1), n_values=37 * 1024 - 11)
    n = c["n_values"]
    offs = c["vector_offsets"].astype(np.uint64)
    out = np.zeros(n, ut)
    args = [_p(c["packed"]), C.c_size_t(c["packed"].size), _p(c["bit_widths"]), _p(offs),
            _p(c["bases"]), C.c_size_t(n)]
    assert getattr(s, f"shim_decompress_ffor_{suf}")(*args, _p(out)) == 0
    want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits)
    assert np.array_equal(out, want[:n])
    found = C.c_int(-1)
    assert getattr(s, f"shim_query_ffor_{suf}")(*args, ct(int(want[n // 2])), C.byref(found)) == 0
    assert found.value == 1
    missing = next(x for x in range(1, 1 << 20) if x not in set(want[:n].tolist()))
    assert getattr(s, f"shim_query_ffor_{suf}")(*args, ct(missing), C.byref(found)) == 0
    assert found.value == 0
    assert getattr(s, f"shim_compute_ffor_{suf}")(*args, C.byref(found)) == 0
    assert found.value == 0  # the reference's compute kernel never matches (it ANDs with 0)


@pytest.mark.gpu
def test_shim_query_multi_column(cuda, built):
    """The reference's host harness: ten copies with shuffled bit widths,
    scans over 1..10 of them.  With a single width every copy is the
    original column, so the result is the oracle's answer."""
    s = C.CDLL(str(built[0]))
    c = colgen.random_ffor(77, 20, 32, [0], base_max=4)
    c["bases"][:] = 3  # width 0: every value is 3
    offs = c["vector_offsets"].astype(np.uint64)
    args = [_p(c["packed"]), C.c_size_t(c["packed"].size), _p(c["bit_widths"]), _p(offs),
            _p(c["bases"]), C.c_size_t(c["n_values"])]
    found = C.c_int(-1)
    assert s.shim_query_multi_column_ffor_u32(*args, C.c_uint32(3), C.byref(found)) == 0
    assert found.value == 1
    assert s.shim_query_multi_column_ffor_u32(*args, C.c_uint32(4), C.byref(found)) == 0
    assert found.value == 0


@pytest.mark.gpu
@pytest.mark.parametrize("f64", [True, False])
@pytest.mark.parametrize("extended", [False, True])
def test_shim_alp_decode_and_create_extended_column(cuda, built, f64, extended):
    s = C.CDLL(str(built[0]))
    dt, ut = (np.float64, np.uint64) if f64 else (np.float32, np.uint32)
    n_vecs = 30
    col = colgen.random_alp(910, n_vecs, f64, range(0, 30), [0, 1, 7, 40])
    n = n_vecs * 1024
    out = np.zeros(n, dt)
    fn = getattr(s, "shim_decompress_alp_" + ("f64" if f64 else "f32"))
    # arrays converted once and kept alive across the call
    a = {k: np.ascontiguousarray(col[k], t) for k, t in
         (("packed", ut), ("bit_widths", np.uint8), ("vector_offsets", np.uint64), ("bases", ut),
          ("factor_indices", np.uint8), ("fraction_indices", np.uint8),
          ("exceptions_offsets", np.uint64), ("exceptions", dt), ("positions", np.uint16),
          ("counts", np.uint16))}
    rc = fn(_p(a["packed"]), C.c_size_t(a["packed"].size), _p(a["bit_widths"]),
            _p(a["vector_offsets"]), _p(a["bases"]), C.c_size_t(n), _p(a["factor_indices"]),
            _p(a["fraction_indices"]), C.c_size_t(a["exceptions"].size),
            _p(a["exceptions_offsets"]), _p(a["exceptions"]), _p(a["positions"]),
            _p(a["counts"]), C.c_int(1 if extended else 0), _p(out))
    assert rc == 0
    want = B.alp_decode(col, n_vecs, dt).view(ut)
    assert np.array_equal(out.view(ut), want)


def _user(built, name, col, out, nv):
    d = C.CDLL(str(built[1]))
    return getattr(d, "user_decode_" + name)(C.byref(col.c), C.c_void_p(out.data_ptr()),
                                             C.c_uint(nv))


@pytest.mark.gpu
@pytest.mark.parametrize("nv", [1, 4])
def test_device_decoders_match_oracle(cuda, built, nv):
    import torch
    for bits in (32, 64):
        ut = np.uint64 if bits == 64 else np.uint32
        td = torch.int64 if bits == 64 else torch.int32
        c = colgen.random_ffor(950 + bits, 23, bits, range(bits + 1))
        for bp in (False, True):
            d = F.make_ffor_column(c["packed"], c["bit_widths"], c["vector_offsets"],
                                   None if bp else c["bases"], c["n_values"], cuda)
            out = torch.zeros(c["n_values"], dtype=td, device=cuda)
            assert _user(built, f"{'bp' if bp else 'ffor'}_u{bits}", d, out, nv) == 0
            want = (B.decode_bp(c["packed"], c["bit_widths"], c["vector_offsets"], bits) if bp else
                    B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"], bits))
            assert np.array_equal(out.cpu().numpy().view(ut), want), (bits, bp)
    for f64 in (True, False):
        dt, ut = (np.float64, np.uint64) if f64 else (np.float32, np.uint32)
        n_vecs = 40
        col = colgen.random_alp(960, n_vecs, f64, range(0, 33), [0, 1, 5, 33, 40])
        want = B.alp_decode(col, n_vecs, dt).view(ut)
        for extended in (False, True):
            c2 = B.to_extended(col, n_vecs, dt)[0] if extended else col
            d = F.make_alp_column(c2, n_vecs * 1024, dt, extended=extended, device=cuda)
            out = torch.zeros(n_vecs * 1024, dtype=torch.float64 if f64 else torch.float32,
                              device=cuda)
            name = ("alpx_" if extended else "alp_") + ("f64" if f64 else "f32")
            assert _user(built, name, d, out, nv) == 0
            assert np.array_equal(out.cpu().numpy().view(ut), want), name


@pytest.mark.gpu
@pytest.mark.parametrize("f64", [True, False])
def test_gpu_to_extended_matches_oracle(cuda, f64):
    dt, ut = (np.float64, np.uint64) if f64 else (np.float32, np.uint32)
    n_vecs = 50
    # a vector whose every value is an exception overflows a 64-bit lane's
    # 6-bit count (64 exceptions per lane), as in the reference
    col = colgen.random_alp(970, n_vecs, f64, range(0, 20), [0, 3, 17, 64, 1024])
    want, _ = B.to_extended(col, n_vecs, dt)
    d = F.make_alp_column(col, n_vecs * 1024, dt, device=cuda)
    x = F.to_extended(d)
    n_exc = int(col["exceptions"].size)
    nl = 16 if f64 else 32
    got_exc = F.device_array(x.c.exceptions, n_exc, dt).cpu().numpy().view(ut)
    got_pos = F.device_array(x.c.positions, n_exc, np.uint16).cpu().numpy().view(np.uint16)
    got_oc = F.device_array(x.c.counts, n_vecs * nl, np.uint16).cpu().numpy().view(np.uint16)
    assert np.array_equal(got_exc, np.ascontiguousarray(want["exceptions"], dt).view(ut))
    assert np.array_equal(got_pos, want["positions"])
    assert np.array_equal(got_oc, want["offsets_counts"])
    # and it decodes as the oracle decodes the oracle's extended column
    got = F.decompress(x).cpu().numpy().view(ut)
    assert np.array_equal(got, B.alp_decode(want, n_vecs, dt, extended=True).view(ut))
