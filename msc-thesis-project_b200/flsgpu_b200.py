"""Python host interface of libflsgpu_b200.so (ctypes over the C ABI in
include/flsgpu_b200.h).

Device memory comes from torch tensors; the library never sees a torch
type: every call passes raw device pointers, sizes and a CUDA stream
handle.  The library must be built (build.py); importing this module on a
machine without it raises instead of falling back to anything else."""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Sequence

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libflsgpu_b200.so"

P = C.c_void_p
SZ = C.c_size_t


class Status(C.c_int):
    pass


STATUS_NAMES = {0: "OK", 1: "INVALID_ARGUMENT", 2: "UNSUPPORTED", 3: "MISALIGNED",
                4: "CORRUPT_COLUMN", 5: "CUDA", 6: "TIMEOUT", 7: "OUT_OF_MEMORY",
                8: "ENCODING"}

BAD_BIT_WIDTH, BAD_OFFSET, BAD_PARAMETER_INDEX, BAD_EXCEPTION = 1, 2, 4, 8

# reference enums (src/engine/enums.cuh:21-53)
UNPACKERS = ["Dummy", "OldFls", "SwitchCase", "Stateless", "StatelessBranchless",
             "StatefulCache", "StatefulLocal1", "StatefulLocal2", "StatefulLocal4",
             "StatefulShared1", "StatefulShared2", "StatefulShared4", "StatefulRegister1",
             "StatefulRegister2", "StatefulRegister4", "StatefulRegisterBranchless1",
             "StatefulRegisterBranchless2", "StatefulRegisterBranchless4",
             "StatefulBranchless"]
PATCHERS = ["None", "Dummy", "Stateless", "Stateful", "Naive", "NaiveBranchless",
            "PrefetchPosition", "PrefetchAll", "PrefetchAllBranchless"]
VARIANT_AUTO, VARIANT_DIRECT, VARIANT_STAGED = 0, 1, 2


class FlsgpuError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class BPColumnC(C.Structure):
    _fields_ = [("n_values", SZ), ("n_vecs", SZ), ("packed_array", P), ("bit_widths", P),
                ("vector_offsets", P)]


class FFORColumnC(C.Structure):
    _fields_ = [("n_values", SZ), ("bp", BPColumnC), ("bases", P)]


class ALPColumnC(C.Structure):
    _fields_ = [("n_values", SZ), ("ffor", FFORColumnC), ("factors", P), ("fractions", P),
                ("factor_indices", P), ("fraction_indices", P), ("n_exceptions", SZ),
                ("exceptions_offsets", P), ("exceptions", P), ("positions", P),
                ("counts", P)]


ALPXColumnC = ALPColumnC  # same layout; last field is offsets_counts


class ALPRDColumnC(C.Structure):
    _fields_ = [("n_values", SZ), ("right", BPColumnC), ("left", BPColumnC),
                ("dictionaries", P), ("dictionary_indices", P), ("n_exceptions", SZ),
                ("exceptions_offsets", P), ("exceptions", P), ("positions", P), ("counts", P)]


class DecodeOpts(C.Structure):
    _fields_ = [("unpack_n_vectors", C.c_uint32), ("unpack_n_values", C.c_uint32),
                ("unpacker", C.c_uint32), ("patcher", C.c_uint32), ("variant", C.c_uint32),
                ("reserved", C.c_uint32), ("d_status", P), ("n_packed_values", SZ)]


_lib = None


def lib() -> C.CDLL:
    """Loads the library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: run msc-thesis-project_b200/build.py")
        _lib = C.CDLL(str(LIB_PATH))
        _lib.flsgpu_last_error.restype = C.c_char_p
        _lib.flsgpu_abi_version.restype = C.c_uint32
        _lib.flsgpu_launch_count.restype = C.c_uint64
        _lib.flsgpu_sum_workspace_f64.restype = SZ
        _lib.flsgpu_sum_workspace_f64.argtypes = [SZ]
    return _lib


def exported_symbols() -> list[str]:
    """Entry points declared in include/flsgpu_b200.h."""
    hdr = (PKG.parent / "include" / "flsgpu_b200.h").read_text()
    import re
    return sorted(set(re.findall(r"\b(flsgpu_[a-z0-9_]+)\s*\(", hdr)))


def _check(status: int) -> None:
    if status != 0:
        raise FlsgpuError(status, lib().flsgpu_last_error().decode())


def _torch():
    import torch
    return torch


def _stream_handle(stream) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


def _dev(a: np.ndarray, device):
    torch = _torch()
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        t = torch.from_numpy(a.view(np.int64))
    elif a.dtype == np.uint32:
        t = torch.from_numpy(a.view(np.int32))
    elif a.dtype == np.uint16:
        t = torch.from_numpy(a.view(np.int16))
    else:
        t = torch.from_numpy(a)
    return t.to(device)


TORCH_OF_BITS = {"u32": "int32", "u64": "int64", "f32": "float32", "f64": "float64"}


@dataclass
class DeviceColumn:
    """Device-resident column: owns its torch buffers and exposes the
    ABI descriptor (`.c`)."""
    kind: str           # bp, ffor, alp, alpx, alprd
    dtype: str          # u32, u64, f32, f64
    n_values: int
    c: C.Structure
    buffers: dict = field(default_factory=dict)
    n_packed: int = 0

    @property
    def n_vecs(self) -> int:
        return (self.n_values + 1023) // 1024

    def compressed_bytes(self) -> int:
        """Bytes a full decode reads: packed words, per-vector metadata and
        exceptions (the algorithmic input bytes)."""
        return int(sum(t.numel() * t.element_size() for k, t in self.buffers.items()
                       if not k.startswith("_")))


def make_ffor_column(packed: np.ndarray, bit_widths: np.ndarray, offsets: np.ndarray,
                     bases: np.ndarray | None, n_values: int, device="cuda") -> DeviceColumn:
    dt = "u64" if packed.dtype == np.uint64 else "u32"
    bufs = {"packed": _dev(packed if packed.size else np.zeros(1, packed.dtype), device),
            "bit_widths": _dev(bit_widths.astype(np.uint8), device),
            "vector_offsets": _dev(offsets.astype(np.uint64), device)}
    n_vecs = bit_widths.size
    bp = BPColumnC(n_values, n_vecs, _ptr(bufs["packed"]), _ptr(bufs["bit_widths"]),
                   _ptr(bufs["vector_offsets"]))
    if bases is None:
        return DeviceColumn("bp", dt, n_values, bp, bufs, packed.size)
    bufs["bases"] = _dev(bases.astype(packed.dtype), device)
    return DeviceColumn("ffor", dt, n_values,
                        FFORColumnC(n_values, bp, _ptr(bufs["bases"])), bufs, packed.size)


def make_alp_column(col: dict, n_values: int, dtype, extended: bool = False,
                    device="cuda") -> DeviceColumn:
    """col: arrays in the reference's host::ALPColumn layout (as produced by
    the encoder), plus offsets_counts for the extended layout."""
    f64 = np.dtype(dtype) == np.float64
    ut = np.uint64 if f64 else np.uint32
    ffor = make_ffor_column(col["packed"].astype(ut), col["bit_widths"], col["vector_offsets"],
                            col["bases"].astype(ut), n_values, device)
    bufs = dict(ffor.buffers)
    n_exc = int(col["exceptions"].size)
    exc = col["exceptions"] if n_exc else np.zeros(1, dtype)
    pos = col["positions"] if n_exc else np.zeros(1, np.uint16)
    bufs.update({"factor_indices": _dev(col["factor_indices"].astype(np.uint8), device),
                 "fraction_indices": _dev(col["fraction_indices"].astype(np.uint8), device),
                 "exceptions_offsets": _dev(col["exceptions_offsets"].astype(np.uint64), device),
                 "exceptions": _dev(np.ascontiguousarray(exc, dtype), device),
                 "positions": _dev(pos.astype(np.uint16), device)})
    last = "offsets_counts" if extended else "counts"
    bufs[last] = _dev(col[last].astype(np.uint16), device)
    c = ALPColumnC(n_values, ffor.c, None, None, _ptr(bufs["factor_indices"]),
                   _ptr(bufs["fraction_indices"]), n_exc, _ptr(bufs["exceptions_offsets"]),
                   _ptr(bufs["exceptions"]), _ptr(bufs["positions"]), _ptr(bufs[last]))
    return DeviceColumn("alpx" if extended else "alp", "f64" if f64 else "f32", n_values, c,
                        bufs, ffor.n_packed)


def make_alprd_column(col: dict, n_values: int, dtype, device="cuda") -> DeviceColumn:
    f64 = np.dtype(dtype) == np.float64
    right = make_ffor_column(col["right_packed"], col["right_bw"], col["right_offsets"], None,
                             n_values, device)
    bufs = {"right_" + k: v for k, v in right.buffers.items()}
    lp = col["left_packed"].astype(np.uint16)
    if lp.size % 2:
        lp = np.concatenate([lp, np.zeros(1, np.uint16)])
    bufs["left_packed"] = _dev(lp if lp.size else np.zeros(2, np.uint16), device)
    bufs["left_bw"] = _dev(col["left_bw"].astype(np.uint8), device)
    bufs["left_offsets"] = _dev(col["left_offsets"].astype(np.uint64), device)
    bufs["dictionaries"] = _dev(col["dictionaries"].astype(np.uint16), device)
    bufs["dictionary_indices"] = _dev(col["dictionary_indices"].astype(np.uint32), device)
    n_exc = int(col["exceptions"].size)
    bufs["exceptions_offsets"] = _dev(col["exceptions_offsets"].astype(np.uint64), device)
    bufs["exceptions"] = _dev(col["exceptions"].astype(np.uint16) if n_exc
                              else np.zeros(1, np.uint16), device)
    bufs["positions"] = _dev(col["positions"].astype(np.uint16) if n_exc
                             else np.zeros(1, np.uint16), device)
    bufs["counts"] = _dev(col["counts"].astype(np.uint16), device)
    n_vecs = (n_values + 1023) // 1024
    left_c = BPColumnC(n_values, n_vecs, _ptr(bufs["left_packed"]), _ptr(bufs["left_bw"]),
                       _ptr(bufs["left_offsets"]))
    c = ALPRDColumnC(n_values, right.c, left_c, _ptr(bufs["dictionaries"]),
                     _ptr(bufs["dictionary_indices"]), n_exc, _ptr(bufs["exceptions_offsets"]),
                     _ptr(bufs["exceptions"]), _ptr(bufs["positions"]), _ptr(bufs["counts"]))
    return DeviceColumn("alprd", "f64" if f64 else "f32", n_values, c, bufs, right.n_packed)


def opts(unpacker: int = 18, patcher: int = 7, variant: int = VARIANT_AUTO,
         unpack_n_vectors: int = 1, unpack_n_values: int = 1, d_status=None,
         n_packed_values: int = 0) -> DecodeOpts:
    return DecodeOpts(unpack_n_vectors, unpack_n_values, unpacker, patcher, variant, 0,
                      _ptr(d_status), n_packed_values)


def _fn(name: str):
    f = getattr(lib(), name)
    f.restype = C.c_int
    return f


def decompress(col: DeviceColumn, out=None, o: DecodeOpts | None = None, stream=None):
    torch = _torch()
    if out is None:
        out = torch.empty(col.n_values, dtype=getattr(torch, TORCH_OF_BITS[col.dtype]),
                          device=col.buffers[next(iter(col.buffers))].device)
    f = _fn(f"flsgpu_decompress_{col.kind}_{col.dtype}")
    _check(f(C.byref(col.c), P(_ptr(out)), C.byref(o) if o is not None else None,
             P(_stream_handle(stream))))
    return out


def sum_(col: DeviceColumn, out=None, workspace=None, o: DecodeOpts | None = None, stream=None):
    """Decode fused with a sum: u64 (mod 2^64) for integer columns, f64 with
    the fixed reduction tree for f64 ALP columns."""
    torch = _torch()
    dev = col.buffers[next(iter(col.buffers))].device
    if col.dtype in ("u32", "u64"):
        out = out if out is not None else torch.empty(1, dtype=torch.int64, device=dev)
        f = _fn(f"flsgpu_sum_{col.kind}_{col.dtype}")
        _check(f(C.byref(col.c), P(_ptr(out)), C.byref(o) if o is not None else None,
                 P(_stream_handle(stream))))
        return out
    out = out if out is not None else torch.empty(1, dtype=torch.float64, device=dev)
    if workspace is None:
        workspace = torch.empty(lib().flsgpu_sum_workspace_f64(col.n_values),
                                dtype=torch.float64, device=dev)
    f = _fn(f"flsgpu_sum_{col.kind}_{col.dtype}")
    _check(f(C.byref(col.c), P(_ptr(out)), P(_ptr(workspace)),
             C.byref(o) if o is not None else None, P(_stream_handle(stream))))
    return out


_CT = {"u32": C.c_uint32, "u64": C.c_uint64, "f32": C.c_float, "f64": C.c_double}


def query(col: DeviceColumn, magic, found=None, o: DecodeOpts | None = None, stream=None):
    torch = _torch()
    dev = col.buffers[next(iter(col.buffers))].device
    if found is None:
        found = torch.zeros(1, dtype=torch.uint8, device=dev)
    f = _fn(f"flsgpu_query_{col.kind}_{col.dtype}")
    _check(f(C.byref(col.c), _CT[col.dtype](magic), P(_ptr(found)),
             C.byref(o) if o is not None else None, P(_stream_handle(stream))))
    return found


def compute(col: DeviceColumn, n_repetitions: int = 10, out=None, o=None, stream=None):
    torch = _torch()
    dev = col.buffers[next(iter(col.buffers))].device
    out = out if out is not None else torch.zeros(1, dtype=torch.uint8, device=dev)
    f = _fn(f"flsgpu_compute_{col.kind}_{col.dtype}")
    _check(f(C.byref(col.c), C.c_uint32(n_repetitions), P(_ptr(out)),
             C.byref(o) if o is not None else None, P(_stream_handle(stream))))
    return out


def query_multi_column(cols: Sequence[DeviceColumn], value, out=None, o=None, stream=None):
    torch = _torch()
    c0 = cols[0]
    dev = c0.buffers[next(iter(c0.buffers))].device
    out = out if out is not None else torch.zeros(1, dtype=torch.uint8, device=dev)
    arr = (type(c0.c) * len(cols))(*[c.c for c in cols])
    f = _fn(f"flsgpu_query_multi_column_{c0.kind}_{c0.dtype}")
    _check(f(arr, C.c_uint32(len(cols)), _CT[c0.dtype](value), P(_ptr(out)),
             C.byref(o) if o is not None else None, P(_stream_handle(stream))))
    return out


def launch_count() -> int:
    return int(lib().flsgpu_launch_count())
