"""ctypes loaders for the oracle (liboracle.so, oracle.c) and for the
reference's own CPU build (_ref/libflsref.so, build_ref.sh).

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libflsref.so"

P = C.c_void_p
SZ = C.c_size_t
I = C.c_int
U16 = C.c_uint16
U32 = C.c_uint32
U64 = C.c_uint64
F64 = C.c_double
F32 = C.c_float


def build_oracle(force: bool = False) -> Path:
    src = HERE / "oracle.c"
    if force or not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < src.stat().st_mtime:
        subprocess.check_call(
            ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off",
             "-o", str(ORACLE_SO), str(src), "-lm"])
    return ORACLE_SO


def reference_root() -> str:
    """The reference checkout: $FLSGPU_REFERENCE, default /root/reference."""
    return os.environ.get("FLSGPU_REFERENCE", "/root/reference")


def build_ref(reference: str | None = None) -> Path | None:
    reference = reference or reference_root()
    if not Path(reference, "src", "fls").is_dir():
        return REF_SO if REF_SO.exists() else None
    subprocess.check_call(["bash", str(HERE / "build_ref.sh"), reference])
    return REF_SO


class OracleInfo(C.Structure):
    _fields_ = [("n_packed", SZ), ("n_exceptions", SZ), ("compressed_bytes", SZ),
                ("compressed_bytes_extended", SZ), ("rd_rowgroup", SZ)]


class RDState(C.Structure):
    _fields_ = [("right_bw", C.c_uint8), ("left_bw", C.c_uint8),
                ("dict_size", C.c_uint8), ("dict", U16 * 8)]


_ORACLE_SIGS = {
    "orc_alp_vector_best_f32": (I, [P, P]),
    "orc_alp_encode_vector_f32": (I, [P, I, I, P, P, P]),
    "orc_pack_u8": (None, [P, P, I]), "orc_unpack_u8": (None, [P, P, I]),
    "orc_ffor_u8": (None, [P, P, I, C.c_uint8]), "orc_ffor_u16": (None, [P, P, I, U16]),
    "orc_unffor_u8": (None, [P, P, I, C.c_uint8]), "orc_unffor_u16": (None, [P, P, I, U16]),
    "orc_pack_u16": (None, [P, P, I]), "orc_pack_u32": (None, [P, P, I]),
    "orc_pack_u64": (None, [P, P, I]), "orc_unpack_u16": (None, [P, P, I]),
    "orc_unpack_u32": (None, [P, P, I]), "orc_unpack_u64": (None, [P, P, I]),
    "orc_ffor_u32": (None, [P, P, I, U32]), "orc_ffor_u64": (None, [P, P, I, U64]),
    "orc_unffor_u32": (None, [P, P, I, U32]), "orc_unffor_u64": (None, [P, P, I, U64]),
    "orc_falp_f32": (None, [P, P, I, U32, I, I]),
    "orc_falp_f64": (None, [P, P, I, U64, I, I]),
    "orc_decode_bp_u32": (None, [P, P, P, SZ, P]),
    "orc_decode_bp_u64": (None, [P, P, P, SZ, P]),
    "orc_decode_ffor_u32": (None, [P, P, P, P, SZ, P]),
    "orc_decode_ffor_u64": (None, [P, P, P, P, SZ, P]),
    "orc_decode_alp_f32": (None, [P] * 11 + [SZ, P]),
    "orc_decode_alp_f64": (None, [P] * 11 + [SZ, P]),
    "orc_alp_to_extended": (SZ, [I, P, P, P, SZ, P, P, P]),
    "orc_alp_encode_f64": (I, [P, SZ, SZ] + [P] * 10 + [P]),
    "orc_alp_encode_f32": (I, [P, SZ, SZ] + [P] * 10 + [P]),
    "orc_alp_rowgroup_topk_f64": (I, [P, SZ, P, P]),
    "orc_alp_rowgroup_topk_f32": (I, [P, SZ, P, P]),
    "orc_set_rd_as_alp": (None, [I]),
    "orc_alp_vector_best_f64": (I, [P, P]),
    "orc_alp_vector_choose_f64": (None, [P, I, P, P, P, P]),
    "orc_alp_encode_vector_f64": (I, [P, I, I, P, P, P]),
    "orc_rd_init_f64": (None, [P, SZ, P]), "orc_rd_init_f32": (None, [P, SZ, P]),
    "orc_rd_encode_vector_f64": (I, [P, P, P, P, P, P]),
    "orc_rd_encode_vector_f32": (I, [P, P, P, P, P, P]),
    "orc_rd_decode_vector_f64": (None, [P, P, P, I, P, P, I, P]),
    "orc_rd_decode_vector_f32": (None, [P, P, P, I, P, P, I, P]),
    "orc_decode_rd_f64": (None, [P] * 12 + [SZ, P]),
    "orc_decode_rd_f32": (None, [P] * 12 + [SZ, P]),
    "orc_tree_sum_f64": (F64, [P, SZ]),
    "orc_tree_sum_masked_f64": (F64, [P, P, U32, SZ]),
    "orc_tree_sum_f32": (F32, [P, SZ]),
    "orc_sum_u32": (U64, [P, SZ]), "orc_sum_u64": (U64, [P, SZ]),
    "orc_median_u32": (U32, [P, SZ]),
}

_REF_SIGS = {
    "ref_pack_u8": (None, [P, P, I]), "ref_unpack_u8": (None, [P, P, I]),
    "ref_ffor_u8": (None, [P, P, I, C.c_uint8]), "ref_ffor_u16": (None, [P, P, I, U16]),
    "ref_unffor_u8": (None, [P, P, I, C.c_uint8]), "ref_unffor_u16": (None, [P, P, I, U16]),
    "ref_pack_u16": (None, [P, P, I]), "ref_pack_u32": (None, [P, P, I]),
    "ref_pack_u64": (None, [P, P, I]), "ref_unpack_u16": (None, [P, P, I]),
    "ref_unpack_u32": (None, [P, P, I]), "ref_unpack_u64": (None, [P, P, I]),
    "ref_ffor_u32": (None, [P, P, I, U32]), "ref_ffor_u64": (None, [P, P, I, U64]),
    "ref_unffor_u32": (None, [P, P, I, U32]), "ref_unffor_u64": (None, [P, P, I, U64]),
    "ref_falp_f32": (None, [P, P, I, U32, I, I]),
    "ref_falp_f64": (None, [P, P, I, U64, I, I]),
    "ref_decode_ffor_u32": (None, [P, P, P, P, SZ, SZ, P]),
    "ref_decode_ffor_u64": (None, [P, P, P, P, SZ, SZ, P]),
    "ref_decode_alp_f64": (None, [P] * 10 + [SZ, SZ, P]),
    "ref_decode_alp_f32": (None, [P] * 10 + [SZ, SZ, P]),
    "ref_decode_alpx_f64": (None, [P] * 10 + [SZ, P]),
    "ref_decode_alpx_f32": (None, [P] * 10 + [SZ, P]),
    "ref_alp_to_extended_f64": (None, [P, P, P, SZ, SZ, P, P, P]),
    "ref_alp_to_extended_f32": (None, [P, P, P, SZ, SZ, P, P, P]),
    "ref_alp_encode_f64": (I, [P, SZ] + [P] * 11),
    "ref_alp_encode_f32": (I, [P, SZ] + [P] * 11),
    "ref_alp_topk_f64": (I, [P, SZ, P, P]), "ref_alp_topk_f32": (I, [P, SZ, P, P]),
    "ref_alp_encode_vector_f64": (I, [P, I, P, P, P, P, P, P, P]),
    "ref_rd_init_f64": (I, [P, SZ, P, P, P, P]),
    "ref_rd_roundtrip_f64": (I, [P, SZ, P, P, P, P, P, P]),
}


def _load(path: Path, sigs: dict) -> C.CDLL:
    lib = C.CDLL(str(path))
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_oracle = None
_ref = None


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_SO.exists():
            build_oracle()
        _oracle = _load(ORACLE_SO, _ORACLE_SIGS)
    return _oracle


def ref() -> C.CDLL | None:
    """The reference's own CPU build, or None when it was not built."""
    global _ref
    if _ref is None and REF_SO.exists():
        _ref = _load(REF_SO, _REF_SIGS)
    return _ref


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


# ---------------------------------------------------------------------------
# numpy conveniences over the oracle
# ---------------------------------------------------------------------------
UINT = {16: np.uint16, 32: np.uint32, 64: np.uint64}


def unpack(packed: np.ndarray, bw: int, bits: int, lib=None) -> np.ndarray:
    lib = lib or oracle()
    out = np.zeros(1024, UINT[bits])
    p = np.zeros(1024, UINT[bits])
    p[: packed.size] = packed
    getattr(lib, f"{'orc' if lib is oracle() else 'ref'}_unpack_u{bits}")(ptr(p), ptr(out), bw)
    return out


def pack(values: np.ndarray, bw: int, bits: int, lib=None) -> np.ndarray:
    lib = lib or oracle()
    out = np.zeros(1024, UINT[bits])
    v = np.ascontiguousarray(values, UINT[bits])
    getattr(lib, f"{'orc' if lib is oracle() else 'ref'}_pack_u{bits}")(ptr(v), ptr(out), bw)
    return out[: bw * (1024 // bits)].copy()


def alp_encode(values: np.ndarray, rowgroup_vecs: int = 100, rd_as_alp: bool = False):
    """Oracle ALP encode of a whole column (n % 1024 == 0).  Returns a dict of
    arrays in the reference's host::ALPColumn layout, or None when sampling
    selects ALP-RD for a rowgroup (as alp::encode throws).  With rd_as_alp
    such rowgroups keep their ALP top-k instead (an ALP-only encoder)."""
    lib = oracle()
    lib.orc_set_rd_as_alp(1 if rd_as_alp else 0)
    f64 = values.dtype == np.float64
    ut = np.uint64 if f64 else np.uint32
    n_vecs = values.size // 1024
    packed = np.zeros(n_vecs * 1024, ut)
    bw = np.zeros(n_vecs, np.uint8)
    offs = np.zeros(n_vecs, np.uint64)
    bases = np.zeros(n_vecs, ut)
    fac = np.zeros(n_vecs, np.uint8)
    exp = np.zeros(n_vecs, np.uint8)
    exc_offs = np.zeros(n_vecs, np.uint64)
    exc = np.zeros(n_vecs * 1024, values.dtype)
    pos = np.zeros(n_vecs * 1024, np.uint16)
    counts = np.zeros(n_vecs, np.uint16)
    info = OracleInfo()
    fn = lib.orc_alp_encode_f64 if f64 else lib.orc_alp_encode_f32
    rc = fn(ptr(np.ascontiguousarray(values)), n_vecs, rowgroup_vecs, ptr(packed), ptr(bw),
            ptr(offs), ptr(bases), ptr(fac), ptr(exp), ptr(exc_offs), ptr(exc), ptr(pos),
            ptr(counts), C.byref(info))
    if rc != 0:
        return None
    return dict(packed=packed[: info.n_packed].copy(), bit_widths=bw, vector_offsets=offs,
                bases=bases, factor_indices=fac, fraction_indices=exp,
                exceptions_offsets=exc_offs, exceptions=exc[: info.n_exceptions].copy(),
                positions=pos[: info.n_exceptions].copy(), counts=counts,
                compressed_bytes=info.compressed_bytes,
                compressed_bytes_extended=info.compressed_bytes_extended)


def alp_decode(col: dict, n_vecs: int, dtype, extended: bool = False) -> np.ndarray:
    lib = oracle()
    out = np.zeros(n_vecs * 1024, dtype)
    fn = lib.orc_decode_alp_f64 if dtype == np.float64 else lib.orc_decode_alp_f32
    fn(ptr(col["packed"]), ptr(col["bit_widths"]), ptr(col["vector_offsets"]),
       ptr(col["bases"]), ptr(col["factor_indices"]), ptr(col["fraction_indices"]),
       ptr(col["exceptions_offsets"]), ptr(col["exceptions"]), ptr(col["positions"]),
       None if extended else ptr(col["counts"]),
       ptr(col["offsets_counts"]) if extended else None, n_vecs, ptr(out))
    return out


def to_extended(col: dict, n_vecs: int, dtype):
    lib = oracle()
    bits = 64 if dtype == np.float64 else 32
    n_exc = col["exceptions"].size
    e = np.zeros(max(n_exc, 1), dtype)
    p = np.zeros(max(n_exc, 1), np.uint16)
    oc = np.zeros(n_vecs * (1024 // bits), np.uint16)
    ovf = lib.orc_alp_to_extended(bits, ptr(col["exceptions"]) if n_exc else None,
                                  ptr(col["positions"]) if n_exc else None, ptr(col["counts"]),
                                  n_vecs, ptr(e), ptr(p), ptr(oc))
    out = dict(col)
    out["exceptions"] = e[:n_exc].copy()
    out["positions"] = p[:n_exc].copy()
    out["offsets_counts"] = oc
    return out, int(ovf)


def decode_ffor(packed, bw, offs, bases, bits: int) -> np.ndarray:
    lib = oracle()
    n = bw.size
    out = np.zeros(n * 1024, UINT[bits])
    fn = lib.orc_decode_ffor_u32 if bits == 32 else lib.orc_decode_ffor_u64
    fn(ptr(packed), ptr(bw), ptr(offs), ptr(bases), n, ptr(out))
    return out


def decode_bp(packed, bw, offs, bits: int) -> np.ndarray:
    lib = oracle()
    n = bw.size
    out = np.zeros(n * 1024, UINT[bits])
    fn = lib.orc_decode_bp_u32 if bits == 32 else lib.orc_decode_bp_u64
    fn(ptr(packed), ptr(bw), ptr(offs), n, ptr(out))
    return out
