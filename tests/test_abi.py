"""The C-ABI library loads and exports every entry point that
include/flsgpu_b200.h declares; argument errors come back as status codes
(these calls return before touching the GPU)."""
import ctypes as C
import subprocess

import pytest

import flsgpu_b200 as F


def test_library_exports_every_declared_symbol():
    lib = F.lib()
    missing = [s for s in F.exported_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_nm_shows_the_symbols_as_defined_text():
    out = subprocess.run(["nm", "-D", "--defined-only", str(F.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    defined = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert set(F.exported_symbols()) <= defined


def test_abi_version_and_struct_sizes():
    assert F.lib().flsgpu_abi_version() == 1
    # field-for-field the reference's device structs on LP64
    assert C.sizeof(F.BPColumnC) == 40
    assert C.sizeof(F.FFORColumnC) == 56
    assert C.sizeof(F.ALPColumnC) == 56 + 8 + 8 * 9
    assert C.sizeof(F.DecodeOpts) == 40


def test_null_column_is_invalid_argument():
    f = F._fn("flsgpu_decompress_ffor_u32")
    assert f(None, None, None, None) == 1
    assert b"null column" in F.lib().flsgpu_last_error()


def test_bad_enum_is_rejected():
    col = F.FFORColumnC()
    o = F.opts(unpacker=99)
    f = F._fn("flsgpu_decompress_ffor_u32")
    assert f(C.byref(col), None, C.byref(o), None) == 1
    o = F.opts(patcher=42)
    assert f(C.byref(col), None, C.byref(o), None) == 1


def test_empty_column_is_a_no_op():
    col = F.FFORColumnC()
    f = F._fn("flsgpu_decompress_ffor_u64")
    assert f(C.byref(col), None, None, None) == 0


def test_multi_column_bounds():
    f = F._fn("flsgpu_query_multi_column_ffor_u32")
    cols = (F.FFORColumnC * 17)()
    assert f(cols, C.c_uint32(17), C.c_uint32(0), C.c_void_p(16), None, None) == 1
    assert f(cols, C.c_uint32(0), C.c_uint32(0), C.c_void_p(16), None, None) == 1


def test_decode_tuning_round_trip_and_checks():
    """The tuning state is host-only: set / get round trip, bad arguments
    rejected, the previous table restored."""
    before = F.tuning_get()
    try:
        F.tuning_set({"variant": {("f64", "alp"): F.VARIANT_OCCUPANCY},
                      "prefetch": {32: [3, 7, 32], 64: [0, 64]}})
        t = F.tuning_get()
        assert t["variant"][("f64", "alp")] == F.VARIANT_OCCUPANCY
        assert t["prefetch"][32] == [3, 7, 32] and t["prefetch"][64] == [0, 64]
        with pytest.raises(F.FlsgpuError):
            F.tuning_set({"variant": {("u32", "ffor"): F.VARIANT_AUTO}})
        with pytest.raises(F.FlsgpuError):
            F._check(F._fn("flsgpu_tuning_set_prefetch")(16, None))
    finally:
        F.tuning_set(before)
    assert F.tuning_get() == before
    hdr = F.tuning_header(before)
    assert "kPrefetch32[33]" in hdr and "kVariant[4][4]" in hdr
