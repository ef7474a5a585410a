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
VARIANT_AUTO, VARIANT_REGS, VARIANT_OCCUPANCY, VARIANT_STAGED = 0, 1, 2, 3


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
    """Entry points declared in include/*.h."""
    import re
    names = set()
    for hdr in sorted((PKG.parent / "include").glob("*.h")):
        names |= set(re.findall(r"\b(flsgpu_[a-z0-9_]+)\s*\(", hdr.read_text()))
    return sorted(names)


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


TORCH_OF_BITS = {"u8": "uint8", "u16": "int16", "u32": "int32", "u64": "int64", "f32": "float32",
                 "f64": "float64"}


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

    @property
    def device(self):
        for t in self.buffers.values():
            if hasattr(t, "device"):
                return t.device
        return _torch().device("cuda", _torch().cuda.current_device())

    def compressed_bytes(self) -> int:
        """Bytes a full decode reads: packed words, per-vector metadata and
        exceptions (the algorithmic input bytes)."""
        return int(sum(t.numel() * t.element_size() for k, t in self.buffers.items()
                       if not k.startswith("_")))


def make_ffor_column(packed: np.ndarray, bit_widths: np.ndarray, offsets: np.ndarray,
                     bases: np.ndarray | None, n_values: int, device="cuda") -> DeviceColumn:
    dt = {np.dtype(np.uint64): "u64", np.dtype(np.uint32): "u32", np.dtype(np.uint16): "u16",
          np.dtype(np.uint8): "u8"}[np.dtype(packed.dtype)]
    if dt in ("u8", "u16") and packed.size % (4 // packed.itemsize):
        packed = np.concatenate([packed, np.zeros(4 // packed.itemsize - packed.size % (4 // packed.itemsize), packed.dtype)])
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


BASE_MIN, BASE_SIGNED_MIN, BASE_ZERO = 0, 1, 2


def ffor_encode(values, base_mode: int = BASE_MIN, stream=None):
    """FastLanes FFOR / BP packing on the GPU (flsgpu_ffor_encode_*) of a
    device tensor of uint8 / int16 / int32 / int64 (read as u8 / u16 / u32 /
    u64), values.numel() % 1024 == 0.  Returns a DeviceColumn ("ffor", or
    "bp" for BASE_ZERO).  Synchronises to read the packed size."""
    torch = _torch()
    n = values.numel()
    bits = values.element_size() * 8
    n_vecs = n // 1024
    dev = values.device
    packed = torch.empty(max(n, 1), dtype=values.dtype, device=dev)
    bw = torch.empty(max(n_vecs, 1), dtype=torch.uint8, device=dev)
    offs = torch.empty(max(n_vecs, 1), dtype=torch.int64, device=dev)
    bases = torch.empty(max(n_vecs, 1), dtype=values.dtype, device=dev)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    f = _fn(f"flsgpu_ffor_encode_u{bits}")
    _check(f(P(_ptr(values)), C.c_size_t(n), C.c_uint32(base_mode), P(_ptr(packed)),
             P(_ptr(bw)), P(_ptr(offs)), P(_ptr(bases)), P(_ptr(total)),
             P(_stream_handle(stream))))
    n_packed = int(total.item())
    bufs = {"packed": packed[:n_packed], "bit_widths": bw[:n_vecs], "vector_offsets": offs[:n_vecs],
            "_keep": packed}
    bp = BPColumnC(n, n_vecs, _ptr(packed), _ptr(bw), _ptr(offs))
    if base_mode == BASE_ZERO:
        return DeviceColumn("bp", f"u{bits}", n, bp, bufs, n_packed)
    bufs["bases"] = bases[:n_vecs]
    return DeviceColumn("ffor", f"u{bits}", n, FFORColumnC(n, bp, _ptr(bases)), bufs, n_packed)


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


def to_extended(col: DeviceColumn, stream=None) -> DeviceColumn:
    """The lane-divided (ALPExtendedColumn) form of an ALP DeviceColumn,
    converted on the GPU (flsgpu_alp_to_extended_*); shares the packed
    words and metadata of `col`."""
    torch = _torch()
    f64 = col.dtype == "f64"
    n_exc = int(col.c.n_exceptions)
    dev = col.device
    exc = torch.empty(max(n_exc, 1), dtype=torch.float64 if f64 else torch.float32, device=dev)
    pos = torch.empty(max(n_exc, 1), dtype=torch.int16, device=dev)
    oc = torch.empty(max(col.n_vecs * (16 if f64 else 32), 1), dtype=torch.int16, device=dev)
    dst = ALPColumnC()
    _check(_fn(f"flsgpu_alp_to_extended_{col.dtype}")(C.byref(col.c), P(_ptr(exc)), P(_ptr(pos)),
                                                      P(_ptr(oc)), C.byref(dst),
                                                      P(_stream_handle(stream))))
    return DeviceColumn("alpx", col.dtype, col.n_values, dst,
                        {"_exc": exc, "_pos": pos, "_oc": oc, "_base": col}, col.n_packed)


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
                          device=col.device)
    f = _fn(f"flsgpu_decompress_{col.kind}_{col.dtype}")
    _check(f(C.byref(col.c), P(_ptr(out)), C.byref(o) if o is not None else None,
             P(_stream_handle(stream))))
    return out


def sum_(col: DeviceColumn, out=None, workspace=None, o: DecodeOpts | None = None, stream=None):
    """Decode fused with a sum: u64 (mod 2^64) for integer columns, f64 with
    the fixed reduction tree for f64 ALP columns."""
    torch = _torch()
    dev = col.device
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
    dev = col.device
    if found is None:
        found = torch.zeros(1, dtype=torch.uint8, device=dev)
    f = _fn(f"flsgpu_query_{col.kind}_{col.dtype}")
    _check(f(C.byref(col.c), _CT[col.dtype](magic), P(_ptr(found)),
             C.byref(o) if o is not None else None, P(_stream_handle(stream))))
    return found


def compute(col: DeviceColumn, n_repetitions: int = 10, out=None, o=None, stream=None):
    torch = _torch()
    dev = col.device
    out = out if out is not None else torch.zeros(1, dtype=torch.uint8, device=dev)
    f = _fn(f"flsgpu_compute_{col.kind}_{col.dtype}")
    _check(f(C.byref(col.c), C.c_uint32(n_repetitions), P(_ptr(out)),
             C.byref(o) if o is not None else None, P(_stream_handle(stream))))
    return out


def query_multi_column(cols: Sequence[DeviceColumn], value, out=None, o=None, stream=None):
    torch = _torch()
    c0 = cols[0]
    dev = c0.device
    out = out if out is not None else torch.zeros(1, dtype=torch.uint8, device=dev)
    arr = (type(c0.c) * len(cols))(*[c.c for c in cols])
    f = _fn(f"flsgpu_query_multi_column_{c0.kind}_{c0.dtype}")
    _check(f(arr, C.c_uint32(len(cols)), _CT[c0.dtype](value), P(_ptr(out)),
             C.byref(o) if o is not None else None, P(_stream_handle(stream))))
    return out


def launch_count() -> int:
    return int(lib().flsgpu_launch_count())


# ---------------------------------------------------------------------------
# host-resident columns, pipelined decode
# ---------------------------------------------------------------------------
def host_ffor_column(packed, bit_widths, offsets, bases, n_values: int) -> tuple:
    """An FFOR descriptor over host (CPU, ideally pinned) torch tensors;
    returns (descriptor, kind, dtype, tensors kept alive)."""
    bits = packed.element_size() * 8
    n_vecs = (n_values + 1023) // 1024
    bp = BPColumnC(n_values, n_vecs, packed.data_ptr(), bit_widths.data_ptr(), offsets.data_ptr())
    c = FFORColumnC(n_values, bp, bases.data_ptr())
    return c, "ffor", f"u{bits}", (packed, bit_widths, offsets, bases)


class HostPipeline:
    """Pipelined decode of host-resident columns into host memory
    (flsgpu_host_*): chunks of chunk_values values are copied in, decoded
    and copied out on three streams."""

    def __init__(self, chunk_values: int = 1 << 22):
        self.h = P()
        _check(_fn("flsgpu_host_pipeline_create")(SZ(chunk_values), C.byref(self.h)))

    def decompress(self, desc, kind: str, dtype: str, host_out, o: DecodeOpts | None = None,
                   wait: bool = True):
        """wait=False queues the column behind earlier ones (sync() waits);
        its host arrays must stay alive and untouched until then."""
        name = f"flsgpu_host_decompress_{kind}_{dtype}" + ("" if wait else "_async")
        _check(_fn(name)(self.h, C.byref(desc), P(host_out.data_ptr()),
                         C.byref(o) if o is not None else None))
        return host_out

    def sync(self):
        _check(_fn("flsgpu_host_pipeline_sync")(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            lib().flsgpu_host_pipeline_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# decode tuning and the autotuner
# ---------------------------------------------------------------------------
TYPE_CODES = {"u32": 0, "u64": 1, "f32": 2, "f64": 3}
KIND_CODES = {"bp": 0, "ffor": 1, "alp": 2, "alpx": 3}


def tuning_get() -> dict:
    """The process-wide decode tuning: {"variant": {(type, kind): variant},
    "prefetch": {lane_bits: sorted widths with L2 prefetch}}."""
    out = {"variant": {}, "prefetch": {}}
    v = C.c_uint32()
    for tn, tc in TYPE_CODES.items():
        for kn, kc in KIND_CODES.items():
            _check(_fn("flsgpu_tuning_get_variant")(C.c_uint32(tc), C.c_uint32(kc), C.byref(v)))
            out["variant"][(tn, kn)] = int(v.value)
    for lb in (32, 64):
        m = (C.c_uint64 * 2)()
        _check(_fn("flsgpu_tuning_get_prefetch")(C.c_uint32(lb), m))
        out["prefetch"][lb] = [w for w in range(lb + 1) if (m[w >> 6] >> (w & 63)) & 1]
    return out


def tuning_set(table: dict) -> None:
    """Installs a table of the tuning_get() shape (entries may be missing)."""
    for (tn, kn), var in table.get("variant", {}).items():
        _check(_fn("flsgpu_tuning_set_variant")(C.c_uint32(TYPE_CODES[tn]),
                                                C.c_uint32(KIND_CODES[kn]), C.c_uint32(var)))
    for lb, widths in table.get("prefetch", {}).items():
        m = (C.c_uint64 * 2)()
        for w in widths:
            m[w >> 6] |= 1 << (w & 63)
        _check(_fn("flsgpu_tuning_set_prefetch")(C.c_uint32(int(lb)), m))


def _synthetic_ffor(bits: int, w: int, n_values: int, g, dev) -> DeviceColumn:
    """Random packed words at width w (every value uniform in [0, 2^w)),
    random bases."""
    torch = _torch()
    n_vecs = n_values // 1024
    nl = 1024 // bits
    words = n_vecs * w * nl * (bits // 32)
    packed = torch.randint(-2 ** 31, 2 ** 31, (max(words, 2),), dtype=torch.int32, device=dev,
                           generator=g)
    packed = packed.view(torch.int64) if bits == 64 else packed
    bw = torch.full((n_vecs,), w, dtype=torch.uint8, device=dev)
    offs = torch.arange(n_vecs, dtype=torch.int64, device=dev) * (w * nl)
    bases = torch.randint(-2 ** 31, 2 ** 31, (n_vecs * (bits // 32),), dtype=torch.int32,
                          device=dev, generator=g)
    bases = bases.view(torch.int64) if bits == 64 else bases
    bp = BPColumnC(n_values, n_vecs, packed.data_ptr(), bw.data_ptr(), offs.data_ptr())
    return DeviceColumn("ffor", f"u{bits}", n_values, FFORColumnC(n_values, bp, bases.data_ptr()),
                        {"packed": packed[:max(words // (bits // 32), 1)], "bit_widths": bw,
                         "vector_offsets": offs, "bases": bases, "_keep": packed},
                        words // (bits // 32))


def _synthetic_alp(bits: int, w: int, n_values: int, exc_per_vec: int, g, dev) -> DeviceColumn:
    """An ALP column over a synthetic FFOR part: bases 2..20, factor /
    fraction indices in the lower half of their tables, exc_per_vec
    exceptions per vector at distinct spread positions."""
    torch = _torch()
    f = _synthetic_ffor(bits, w, n_values, g, dev)
    n_vecs = n_values // 1024
    it = torch.int64 if bits == 64 else torch.int32
    bases = torch.randint(2, 21, (n_vecs,), dtype=it, device=dev, generator=g)
    f.buffers["bases"] = bases
    f.c.bases = bases.data_ptr()
    nf, ne = (19, 21) if bits == 64 else (10, 11)
    fac = torch.randint(0, nf // 2 + 1, (n_vecs,), dtype=torch.uint8, device=dev, generator=g)
    fr = torch.randint(0, ne // 2 + 1, (n_vecs,), dtype=torch.uint8, device=dev, generator=g)
    k = exc_per_vec
    counts = torch.full((n_vecs,), k, dtype=torch.int16, device=dev)
    eoffs = torch.arange(n_vecs, dtype=torch.int64, device=dev) * k
    stride = 1024 // max(k, 1)
    shift = torch.randint(0, stride, (n_vecs, 1), device=dev, generator=g)
    pos = ((torch.arange(k, device=dev).view(1, -1) * stride + shift) % 1024).to(torch.int16)
    exc = torch.randn(max(n_vecs * k, 1), dtype=torch.float64 if bits == 64 else torch.float32,
                      device=dev, generator=g)
    pos = pos.reshape(-1) if k else torch.zeros(1, dtype=torch.int16, device=dev)
    c = ALPColumnC(n_values, f.c, None, None, fac.data_ptr(), fr.data_ptr(), n_vecs * k,
                   eoffs.data_ptr(), exc.data_ptr(), pos.data_ptr(), counts.data_ptr())
    bufs = dict(f.buffers)
    bufs.update({"factor_indices": fac, "fraction_indices": fr, "exceptions_offsets": eoffs,
                 "exceptions": exc[:n_vecs * k], "positions": pos[:n_vecs * k], "counts": counts})
    return DeviceColumn("alp", f"f{bits}", n_values, c, bufs, f.n_packed)


def autotune(values_32: int = 2 ** 26, values_64: int = 2 ** 25, reps: int = 5, stream=None,
             install: bool = True, alp_widths=None) -> dict:
    """Measures the decode variants on the current device and picks, per
    lane width and bit width, whether the decode prefetches the next
    vector's packed lines into L2, and per value type and column kind the
    kernel variant (register-rich or register-capped for occupancy).
    Columns are synthetic (random packed words, every width of the lane
    type; ALP columns at the given widths with 1% exceptions), each output
    larger than L2.  Time per configuration: the best of `reps` launches
    (CUDA events).  Returns the chosen table, the per-width GB/s of every
    configuration and the gain over the compiled defaults; installs the
    table unless install=False."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(2024)
    s = torch.cuda.current_stream() if stream is None else stream
    before = tuning_get()

    def best_ms(col, out, variant):
        o = opts(variant=variant)
        decompress(col, out=out, o=o, stream=s)
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            decompress(col, out=out, o=o, stream=s)
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return min(ts)

    def col_bytes(col):
        bits = int(col.dtype[1:])
        return col.compressed_bytes() + col.n_values * bits // 8

    report = {"ffor": {}, "alp": {}}
    table = {"variant": {}, "prefetch": {}}
    for bits, n in ((32, values_32), (64, values_64)):
        # the staged decode exists for 64-bit lanes only
        variants = (VARIANT_REGS, VARIANT_OCCUPANCY) + ((VARIANT_STAGED,) if bits == 64 else ())
        n -= n % 1024
        out = torch.empty(n, dtype=torch.int32 if bits == 32 else torch.int64, device=dev)
        per = {v: {} for v in variants}
        for w in range(bits + 1):
            col = _synthetic_ffor(bits, w, n, g, dev)
            for pf in (False, True):
                cur = tuning_get()["prefetch"][bits]
                tuning_set({"prefetch": {bits: sorted(set(cur) | {w}) if pf
                                         else [x for x in cur if x != w]}})
                for v in variants:
                    per[v][(w, pf)] = best_ms(col, out, v)
            del col
        totals = {v: sum(min(per[v][(w, False)], per[v][(w, True)]) for w in range(bits + 1))
                  for v in variants}
        var = min(variants, key=lambda v: totals[v])
        pf_widths = [w for w in range(bits + 1) if per[var][(w, True)] < per[var][(w, False)]]
        table["prefetch"][bits] = pf_widths
        table["variant"][(f"u{bits}", "ffor")] = var
        table["variant"][(f"u{bits}", "bp")] = var
        tuning_set({"prefetch": {bits: pf_widths}})
        nb = lambda w: (n * w // 8 + n // 1024 * (bits // 8 + 9) + n * bits // 8)  # noqa: E731
        report["ffor"][f"u{bits}"] = {
            "chosen_variant": var, "total_ms": {str(v): round(t, 4) for v, t in totals.items()},
            "gbs": {str(v): [round(nb(w) / (min(per[v][(w, False)], per[v][(w, True)]) / 1e3) / 1e9, 1)
                             for w in range(bits + 1)] for v in variants}}
        del out
    for bits, n in ((32, values_32), (64, values_64)):
        n -= n % 1024
        variants = (VARIANT_REGS, VARIANT_OCCUPANCY) + ((VARIANT_STAGED,) if bits == 64 else ())
        widths = alp_widths or ((8, 12, 16, 20, 24, 28) if bits == 32 else (8, 16, 20, 24, 32, 40, 48))
        out = torch.empty(n, dtype=torch.float32 if bits == 32 else torch.float64, device=dev)
        tot = {v: 0.0 for v in variants}
        gbs = {v: [] for v in variants}
        for w in widths:
            col = _synthetic_alp(bits, w, n, 10, g, dev)
            for v in variants:
                t = best_ms(col, out, v)
                tot[v] += t
                gbs[v].append(round(col_bytes(col) / (t / 1e3) / 1e9, 1))
            del col
        var = min(variants, key=lambda v: tot[v])
        table["variant"][(f"f{bits}", "alp")] = var
        table["variant"][(f"f{bits}", "alpx")] = var
        report["alp"][f"f{bits}"] = {"widths": list(widths), "chosen_variant": var,
                                     "total_ms": {str(v): round(t, 4) for v, t in tot.items()},
                                     "gbs": {str(v): g_ for v, g_ in gbs.items()}}
        del out
    if install:
        tuning_set(table)
    else:
        tuning_set(before)
    return {"table": table, "report": report, "defaults": before}


def tuning_header(table: dict) -> str:
    """The runtime part of a tuning table as the source of its compiled
    defaults (kPrefetch32, kPrefetch64, kVariant in autotune_table.h)."""
    def row(vals):
        return ", ".join(f"{v:2d}" for v in vals)
    p32 = [1 if w in table["prefetch"].get(32, []) else 0 for w in range(33)]
    p64 = [1 if w in table["prefetch"].get(64, []) else 0 for w in range(65)]
    var = [[table["variant"].get((tn, kn), VARIANT_REGS) for kn in KIND_CODES] for tn in TYPE_CODES]
    return ("constexpr unsigned char kPrefetch32[33] = {" + row(p32) + "};\n"
            "constexpr unsigned char kPrefetch64[65] = {" + row(p64) + "};\n"
            "constexpr unsigned char kVariant[4][4] = {" +
            ", ".join("{" + row(r) + "}" for r in var) + "};\n")


# ---------------------------------------------------------------------------
# batched persistent decode and the fused pair query
# ---------------------------------------------------------------------------
TYPE_CODE = {"u32": 0, "u64": 1, "f32": 2, "f64": 3}
ENCODING_CODE = {"bp": 0, "ffor": 1, "alp": 2, "alpx": 3}


class BatchColumnC(C.Structure):
    _fields_ = [("type", C.c_uint32), ("encoding", C.c_uint32), ("column", P), ("d_out", P)]


class Batch:
    """Many columns decoded by one persistent launch (or a replayed graph)."""

    def __init__(self, cols: Sequence[DeviceColumn], outs, o: DecodeOpts | None = None):
        self.cols = list(cols)
        self.outs = list(outs)
        arr = (BatchColumnC * len(cols))()
        for i, (c, out) in enumerate(zip(cols, outs)):
            arr[i] = BatchColumnC(TYPE_CODE[c.dtype], ENCODING_CODE[c.kind],
                                  C.cast(C.pointer(c.c), P), _ptr(out))
        self._arr = arr
        h = P()
        _check(_fn("flsgpu_batch_create")(arr, SZ(len(cols)), C.byref(o) if o is not None else None,
                                         C.byref(h)))
        self.h = h

    def decompress(self, stream=None):
        _check(_fn("flsgpu_batch_decompress")(self.h, P(_stream_handle(stream))))

    def decompress_each(self, sync_each: bool = False, stream=None):
        _check(_fn("flsgpu_batch_decompress_each")(self.h, C.c_int(int(sync_each)),
                                                  P(_stream_handle(stream))))

    def capture(self, stream=None):
        _check(_fn("flsgpu_batch_capture_graph")(self.h, P(_stream_handle(stream))))

    def replay(self, stream=None):
        _check(_fn("flsgpu_batch_replay")(self.h, P(_stream_handle(stream))))

    def total_vectors(self) -> int:
        f = lib().flsgpu_batch_total_vectors
        f.restype = SZ
        f.argtypes = [P]
        return int(f(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            f = lib().flsgpu_batch_destroy
            f.restype = None
            f.argtypes = [P]
            f(self.h)
            self.h = None


class PairQuery:
    """For each (A f64 ALP, B u32 FFOR) pair: sum(A where B < median(B))."""

    def __init__(self, a_cols: Sequence[DeviceColumn], b_cols: Sequence[DeviceColumn], device):
        torch = _torch()
        n = len(a_cols)
        self.a_cols, self.b_cols = list(a_cols), list(b_cols)
        self.results = torch.zeros(max(n, 1), dtype=torch.float64, device=device)
        self.medians = torch.zeros(max(n, 1), dtype=torch.int32, device=device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        aa = (ALPColumnC * max(n, 1))(*[c.c for c in a_cols])
        bb = (FFORColumnC * max(n, 1))(*[c.c for c in b_cols])
        h = P()
        _check(_fn("flsgpu_pair_query_create")(aa, bb, SZ(n), P(_ptr(self.results)),
                                              P(_ptr(self.medians)), P(_ptr(self.status)),
                                              C.byref(h)))
        self.h = h

    def run(self, stream=None):
        _check(_fn("flsgpu_pair_query_run")(self.h, P(_stream_handle(stream))))

    def capture(self, stream=None):
        _check(_fn("flsgpu_pair_query_capture_graph")(self.h, P(_stream_handle(stream))))

    def replay(self, stream=None):
        _check(_fn("flsgpu_pair_query_replay")(self.h, P(_stream_handle(stream))))

    def __del__(self):
        if getattr(self, "h", None):
            f = lib().flsgpu_pair_query_destroy
            f.restype = None
            f.argtypes = [P]
            f(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# GPU ALP encoder with the learned proposal, and the tensor-core GEMM
# ---------------------------------------------------------------------------
class EncodeResultC(C.Structure):
    _fields_ = [("column", ALPColumnC), ("n_packed_words", SZ), ("n_exceptions", SZ),
                ("compressed_bytes", SZ), ("n_fallback", SZ), ("n_rd", SZ),
                ("mean_bit_width", C.c_double)]


class HybridColumnC(C.Structure):
    _fields_ = [("n_values", SZ), ("alp", ALPColumnC), ("rd", ALPRDColumnC), ("schemes", P)]


class HybridEncodeResultC(C.Structure):
    _fields_ = [("column", HybridColumnC), ("n_alp_vectors", SZ), ("n_rd_vectors", SZ),
                ("n_packed_words", SZ), ("n_exceptions", SZ), ("n_right_words", SZ),
                ("n_left_words", SZ), ("n_rd_exceptions", SZ), ("compressed_bytes", SZ),
                ("n_fallback", SZ), ("mean_bit_width", C.c_double), ("d_flags", P)]


class RDEncodeResultC(C.Structure):
    _fields_ = [("column", ALPRDColumnC), ("n_right_words", SZ), ("n_left_words", SZ),
                ("n_exceptions", SZ), ("n_dictionaries", SZ), ("compressed_bytes", SZ)]


class AlpEncoder:
    """GPU ALP encoder for f64 columns; mode 0 = plain per-vector search,
    mode 1 = learned proposal verified on samples, with fallback."""

    def __init__(self, seed: int = 1):
        h = P()
        _check(_fn("flsgpu_alp_encoder_create")(C.c_uint32(seed), C.byref(h)))
        self.h = h

    def train(self, values, epochs=8, batch=1024, lr=2e-3, stream=None):
        lf, ll = C.c_float(), C.c_float()
        _check(_fn("flsgpu_alp_encoder_train")(self.h, P(_ptr(values)), SZ(values.numel()),
                                              C.c_uint32(epochs), C.c_uint32(batch),
                                              C.c_float(lr), C.byref(lf), C.byref(ll),
                                              P(_stream_handle(stream))))
        return lf.value, ll.value

    def encode(self, values, mode: int, stream=None) -> EncodeResultC:
        r = EncodeResultC()
        _check(_fn("flsgpu_alp_encode_f64")(self.h, P(_ptr(values)), SZ(values.numel()),
                                           C.c_uint32(mode), C.byref(r),
                                           P(_stream_handle(stream))))
        return r

    def encode_f32(self, values, stream=None) -> EncodeResultC:
        """ALP encode of an f32 column (float32 tensor) with the plain
        per-vector search; decodes with encoded_column(..., dtype="f32")."""
        r = EncodeResultC()
        _check(_fn("flsgpu_alp_encode_f32")(self.h, P(_ptr(values)), SZ(values.numel()),
                                           C.byref(r), P(_stream_handle(stream))))
        return r

    def encode_hybrid(self, values, mode: int, stream=None) -> HybridEncodeResultC:
        """Hybrid ALP / ALP-RD encode of an f64 column (mode 0 plain search,
        1 learned proposal); ALP-RD vectors get a dictionary of their own."""
        r = HybridEncodeResultC()
        _check(_fn("flsgpu_alp_encode_hybrid_f64")(self.h, P(_ptr(values)), SZ(values.numel()),
                                                  C.c_uint32(mode), C.byref(r),
                                                  P(_stream_handle(stream))))
        return r

    def encode_rd(self, values, rowgroup_vecs: int = 100, stream=None) -> RDEncodeResultC:
        """ALP-RD encode of an f64 (float64 tensor) or f32 (float32 tensor)
        column, one dictionary per rowgroup of rowgroup_vecs vectors."""
        r = RDEncodeResultC()
        suf = "f64" if values.element_size() == 8 else "f32"
        _check(_fn(f"flsgpu_alprd_encode_{suf}")(self.h, P(_ptr(values)), SZ(values.numel()),
                                                C.c_uint32(rowgroup_vecs), C.byref(r),
                                                P(_stream_handle(stream))))
        return r

    def propose(self, values, k=3, stream=None, layered=False):
        """Top-k proposed classes per vector (fused kernel; layered=True runs
        the layer-by-layer launches instead)."""
        torch = _torch()
        cand = torch.empty(values.numel() // 1024 * k, dtype=torch.int16, device=values.device)
        name = "flsgpu_alp_encoder_propose_layered" if layered else "flsgpu_alp_encoder_propose"
        _check(_fn(name)(self.h, P(_ptr(values)), SZ(values.numel()), C.c_uint32(k),
                         P(_ptr(cand)), P(_stream_handle(stream))))
        return cand.view(-1, k)

    def params(self) -> np.ndarray:
        f = lib().flsgpu_alp_encoder_param_count
        f.restype = SZ
        out = np.zeros(int(f()), np.float32)
        _check(_fn("flsgpu_alp_encoder_get_params")(self.h, out.ctypes.data_as(P)))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        _check(_fn("flsgpu_alp_encoder_set_params")(self.h, p.ctypes.data_as(P)))

    def gradients(self, features, labels, stream=None):
        torch = _torch()
        f = lib().flsgpu_alp_encoder_param_count
        f.restype = SZ
        g = torch.empty(int(f()), dtype=torch.float32, device=features.device)
        loss = C.c_float()
        _check(_fn("flsgpu_alp_encoder_gradients")(self.h, P(_ptr(features)), P(_ptr(labels)),
                                                  C.c_uint32(labels.numel()), P(_ptr(g)),
                                                  C.byref(loss), P(_stream_handle(stream))))
        return g, loss.value

    def save(self, path: str):
        _check(_fn("flsgpu_alp_encoder_save")(self.h, str(path).encode()))

    def load(self, path: str):
        _check(_fn("flsgpu_alp_encoder_load")(self.h, str(path).encode()))

    def __del__(self):
        if getattr(self, "h", None):
            f = lib().flsgpu_alp_encoder_destroy
            f.restype = None
            f.argtypes = [P]
            f(self.h)
            self.h = None


def encoded_column(res: EncodeResultC, n_values: int, keep=None, dtype: str = "f64") -> DeviceColumn:
    """The encoder's output as a decodable DeviceColumn (device arrays owned
    by the encoder; valid until its next encode)."""
    return DeviceColumn("alp", dtype, n_values, res.column, {"_owner": keep} if keep else {},
                        int(res.n_packed_words))


def rd_encoded_column(res: RDEncodeResultC, n_values: int, dtype: str = "f64",
                      keep=None) -> DeviceColumn:
    """The ALP-RD encoder's output as a decodable DeviceColumn (arrays owned
    by the encoder; valid until its next encode)."""
    return DeviceColumn("alprd", dtype, n_values, res.column, {"_owner": keep} if keep else {},
                        int(res.n_right_words))


def hybrid_column(res: HybridEncodeResultC, n_values: int, keep=None) -> DeviceColumn:
    """The hybrid encoder's output as a decodable DeviceColumn."""
    return DeviceColumn("alphybrid", "f64", n_values, res.column, {"_owner": keep} if keep else {},
                        int(res.n_packed_words))


def plain_labels(values, stream=None):
    torch = _torch()
    n = values.numel() // 1024
    lab = torch.empty(n, dtype=torch.int16, device=values.device)
    est = torch.empty(n, dtype=torch.int32, device=values.device)
    _check(_fn("flsgpu_alp_plain_labels")(P(_ptr(values)), SZ(values.numel()), P(_ptr(lab)),
                                         P(_ptr(est)), P(_stream_handle(stream))))
    return lab, est


def alp_features(values, stream=None):
    torch = _torch()
    out = torch.empty(values.numel() // 1024, 64, dtype=torch.bfloat16, device=values.device)
    _check(_fn("flsgpu_alp_features")(P(_ptr(values)), SZ(values.numel()), P(_ptr(out)),
                                     P(_stream_handle(stream))))
    return out


def gemm_bf16_tn(A, B, bias=None, relu=False, status=None, stream=None):
    """C = A @ B.T (+bias)(relu) on the tensor cores; A [M,K], B [N,K] bf16."""
    torch = _torch()
    M, K = A.shape
    N = B.shape[0]
    Cf = torch.empty(M, N, dtype=torch.float32, device=A.device)
    _check(_fn("flsgpu_gemm_bf16_tn")(P(_ptr(A)), C.c_int(A.stride(0)), P(_ptr(B)),
                                     C.c_int(B.stride(0)), C.c_int(M), C.c_int(N), C.c_int(K),
                                     P(_ptr(Cf)), None, C.c_int(N), P(_ptr(bias)),
                                     C.c_int(int(relu)), P(_ptr(status)),
                                     P(_stream_handle(stream))))
    return Cf


class _CudaArray:
    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 2}


def device_array(ptr: int, n: int, dtype):
    """A torch view of n elements of raw device memory (no copy)."""
    torch = _torch()
    typestr = np.dtype(dtype).str
    if n == 0:
        return torch.empty(0, dtype=getattr(torch, {"<u8": "int64", "<f8": "float64", "|u1": "uint8",
                                                      "<u2": "int16", "<u4": "int32"}.get(typestr, "uint8")),
                           device="cuda")
    return torch.as_tensor(_CudaArray(ptr, n, typestr), device="cuda")
