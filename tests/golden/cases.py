"""Seeded golden cases shared by gen_golden.py (run against the reference's
CPU build) and tests/test_oracle.py (run against the oracle).  Every input
is regenerated from a numpy seed, so fixtures hold only digests."""
from __future__ import annotations

import ctypes as C
import hashlib

import numpy as np

UT = {16: np.uint16, 32: np.uint32, 64: np.uint64}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:32]


def ptr(a):
    return None if a is None else a.ctypes.data


# ---------------------------------------------------------------------------
# FastLanes pack / unpack / unffor, every bit width of u16 / u32 / u64
# ---------------------------------------------------------------------------
def fls_cases():
    for bits in (16, 32, 64):
        for bw in range(bits + 1):
            yield {"bits": bits, "bw": bw, "seed": 1000 * bits + bw}


def run_fls(lib, pre, case):
    bits, bw = case["bits"], case["bw"]
    ut = UT[bits]
    rng = np.random.default_rng(case["seed"])
    vals = rng.integers(0, 2 ** bits, 1024, dtype=np.uint64).astype(ut)
    packed = np.zeros(1024, ut)
    getattr(lib, f"{pre}_pack_u{bits}")(ptr(vals), ptr(packed), bw)
    n = bw * 1024 // bits
    packed = packed[:n].copy()
    src = np.zeros(1024, ut)
    src[:n] = packed
    unpacked = np.zeros(1024, ut)
    getattr(lib, f"{pre}_unpack_u{bits}")(ptr(src), ptr(unpacked), bw)
    unffor = np.zeros(1024, ut)
    if bits > 16:
        base = int(rng.integers(0, 2 ** bits, dtype=np.uint64))
        getattr(lib, f"{pre}_unffor_u{bits}")(ptr(src), ptr(unffor), bw, base)
    return packed, unpacked, unffor


# ---------------------------------------------------------------------------
# falp (fused unFFOR + ALP scale), every width below the type width
# ---------------------------------------------------------------------------
def falp_cases():
    for bits in (32, 64):
        nf, ne = (19, 21) if bits == 64 else (10, 11)
        for bw in range(bits):
            for j in range(3):
                rng = np.random.default_rng(7 * bw + 1000 * bits + j)
                yield {"bits": bits, "bw": bw, "fac": int(rng.integers(0, nf)),
                       "exp": int(rng.integers(0, ne)), "seed": 50000 + 100 * bits + 3 * bw + j}


def run_falp(lib, pre, case):
    bits, bw = case["bits"], case["bw"]
    ut = UT[bits]
    ft = np.float64 if bits == 64 else np.float32
    rng = np.random.default_rng(case["seed"])
    packed = rng.integers(0, 2 ** bits, 1024, dtype=np.uint64).astype(ut)
    base = int(rng.integers(0, 2 ** min(bits, 24), dtype=np.uint64))
    out = np.zeros(1024, ft)
    getattr(lib, f"{pre}_falp_f{bits}")(ptr(packed), ptr(out), bw, base, case["fac"],
                                        case["exp"])
    return out.view(ut)


# ---------------------------------------------------------------------------
# ALP columns: integers uniform in [-10^6, 10^6] divided by 10^d, 1% of the
# positions replaced by random non-NaN bit patterns (config of the ALP
# decode benchmark, scaled down)
# ---------------------------------------------------------------------------
def make_alp_values(seed: int, n_vecs: int, f64: bool, dmax: int, uniform_d: bool,
                    exc_rate: float = 0.01) -> np.ndarray:
    rng = np.random.default_rng(seed)
    dt = np.float64 if f64 else np.float32
    bits = 64 if f64 else 32
    ut = UT[bits]
    ints = rng.integers(-10 ** 6, 10 ** 6 + 1, n_vecs * 1024)
    d = (np.full(n_vecs, int(rng.integers(0, dmax + 1))) if uniform_d
         else rng.integers(0, dmax + 1, n_vecs))
    vals = (ints / (10.0 ** np.repeat(d, 1024))).astype(dt)
    m = rng.random(vals.size) < exc_rate
    pat = rng.integers(0, 2 ** bits, int(m.sum()), dtype=np.uint64).astype(ut)
    f = pat.view(dt)
    pat[np.isnan(f)] &= ut((1 << bits) - 1 - (1 << (bits - 2)))
    v = vals.view(ut).copy()
    v[m] = pat
    return v.view(dt)


def alp_column_cases():
    i = 0
    for f64 in (True, False):
        for uniform_d in (True, False):
            for rep in range(2):
                yield {"f64": f64, "uniform_d": uniform_d, "n_vecs": 40 + 30 * rep,
                       "seed": 777 + i, "dmax": 4 if f64 else 3}
                i += 1


def case_values(case):
    return make_alp_values(case["seed"], case["n_vecs"], case["f64"], case["dmax"],
                           case["uniform_d"])


def _enc_buffers(n_vecs, f64):
    ut = np.uint64 if f64 else np.uint32
    dt = np.float64 if f64 else np.float32
    return dict(packed=np.zeros(n_vecs * 1024, ut), bit_widths=np.zeros(n_vecs, np.uint8),
                vector_offsets=np.zeros(n_vecs, np.uint64), bases=np.zeros(n_vecs, ut),
                factor_indices=np.zeros(n_vecs, np.uint8),
                fraction_indices=np.zeros(n_vecs, np.uint8),
                exceptions_offsets=np.zeros(n_vecs, np.uint64),
                exceptions=np.zeros(n_vecs * 1024, dt), positions=np.zeros(n_vecs * 1024, np.uint16),
                counts=np.zeros(n_vecs, np.uint16))


ENC_KEYS = ["packed", "bit_widths", "vector_offsets", "bases", "factor_indices",
            "fraction_indices", "exceptions_offsets", "exceptions", "positions", "counts"]


def run_ref_encode(r, case):
    vals = case_values(case)
    n_vecs = case["n_vecs"]
    b = _enc_buffers(n_vecs, case["f64"])
    sizes = np.zeros(4, np.uint64)
    fn = r.ref_alp_encode_f64 if case["f64"] else r.ref_alp_encode_f32
    rc = fn(ptr(vals), vals.size, *[ptr(b[k]) for k in ENC_KEYS], ptr(sizes))
    if rc != 0:
        return None
    b["packed"] = b["packed"][: int(sizes[0])]
    b["exceptions"] = b["exceptions"][: int(sizes[1])]
    b["positions"] = b["positions"][: int(sizes[1])]
    b["compressed_bytes"] = int(sizes[2])
    b["compressed_bytes_extended"] = int(sizes[3])
    return b


def run_orc_encode(o, case, rowgroup_vecs=0):
    from oracle import binding as B
    vals = case_values(case)
    return B.alp_encode(vals, rowgroup_vecs=rowgroup_vecs)


def full_width_vectors(case, enc) -> list[int]:
    """Vectors packed at the full type width.  There the reference's CPU
    falp (src/alp/falp.cpp:33293, :42198) differs from its GPU ALPFunctor
    and does not round-trip; digests exclude them."""
    full = 64 if case["f64"] else 32
    return [int(i) for i in np.nonzero(enc["bit_widths"] == full)[0]]


def mask_vectors(a: np.ndarray, vecs) -> np.ndarray:
    a = np.array(a, copy=True).reshape(-1)
    u = a.view(np.uint8).reshape(a.size // 1024 if a.size >= 1024 else 1, -1)
    for v in vecs:
        u[v, :] = 0
    return a


def run_ref_decode(r, case, enc):
    n_vecs = case["n_vecs"]
    dt = np.float64 if case["f64"] else np.float32
    out = np.zeros(n_vecs * 1024, dt)
    fn = r.ref_decode_alp_f64 if case["f64"] else r.ref_decode_alp_f32
    fn(*[ptr(enc[k]) for k in ENC_KEYS], 0, n_vecs, ptr(out))
    return out.view(UT[64 if case["f64"] else 32])


def run_ref_extended(r, case, enc):
    n_vecs = case["n_vecs"]
    f64 = case["f64"]
    dt = np.float64 if f64 else np.float32
    n_exc = enc["exceptions"].size
    e = np.zeros(max(n_exc, 1), dt)
    p = np.zeros(max(n_exc, 1), np.uint16)
    oc = np.zeros(n_vecs * (16 if f64 else 32), np.uint16)
    fn = r.ref_alp_to_extended_f64 if f64 else r.ref_alp_to_extended_f32
    fn(ptr(enc["exceptions"]), ptr(enc["positions"]), ptr(enc["counts"]), n_vecs, n_exc,
       ptr(e), ptr(p), ptr(oc))
    out = np.zeros(n_vecs * 1024, dt)
    fn = r.ref_decode_alpx_f64 if f64 else r.ref_decode_alpx_f32
    fn(ptr(enc["packed"]), ptr(enc["bit_widths"]), ptr(enc["vector_offsets"]), ptr(enc["bases"]),
       ptr(enc["factor_indices"]), ptr(enc["fraction_indices"]), ptr(enc["exceptions_offsets"]),
       ptr(e), ptr(p), ptr(oc), n_vecs, ptr(out))
    return {"x_exceptions": e[:n_exc], "x_positions": p[:n_exc], "x_offsets_counts": oc,
            "x_decoded": out}


# ---------------------------------------------------------------------------
# rowgroup sampling search (top-k combinations)
# ---------------------------------------------------------------------------
def topk_cases():
    for i in range(6):
        yield {"f64": i % 2 == 0, "seed": 4242 + i, "n_vecs": 100,
               "uniform_d": i % 3 != 2, "dmax": 4 if i % 2 == 0 else 3}


def run_topk(lib, pre, case):
    vals = case_values(case)
    ke = np.zeros(8, np.uint8)
    kf = np.zeros(8, np.uint8)
    if pre == "ref":
        fn = lib.ref_alp_topk_f64 if case["f64"] else lib.ref_alp_topk_f32
    else:
        fn = lib.orc_alp_rowgroup_topk_f64 if case["f64"] else lib.orc_alp_rowgroup_topk_f32
    k = fn(ptr(vals), vals.size, ptr(ke), ptr(kf))
    return [int(k)] + [[int(ke[i]), int(kf[i])] for i in range(max(k, 0))]


# ---------------------------------------------------------------------------
# ALP-RD: rowgroup init (cut + dictionary) and a vector round trip
# ---------------------------------------------------------------------------
def rd_cases():
    for i in range(4):
        yield {"seed": 9100 + i, "n_vecs": 12 + i, "kind": ["uniform01", "mantissa_noise",
                                                            "wide", "uniform01"][i]}


def rd_values(case):
    rng = np.random.default_rng(case["seed"])
    n = case["n_vecs"] * 1024
    if case["kind"] == "uniform01":
        return rng.random(n)
    if case["kind"] == "mantissa_noise":
        return (rng.random(n) * 2.0 - 1.0) * 1000.0
    return rng.standard_normal(n) * np.exp(rng.standard_normal(n) * 3)


def run_ref_rd(r, case):
    vals = rd_values(case)
    rbw = np.zeros(1, np.uint8)
    lbw = np.zeros(1, np.uint8)
    ds = np.zeros(1, np.uint8)
    dic = np.zeros(8, np.uint16)
    r.ref_rd_init_f64(ptr(vals), vals.size, ptr(rbw), ptr(lbw), ptr(ds), ptr(dic))
    vec = np.ascontiguousarray(vals[1024:2048])
    right = np.zeros(1024, np.uint64)
    left = np.zeros(1024, np.uint16)
    exc = np.zeros(1024, np.uint16)
    pos = np.zeros(1024, np.uint16)
    out = np.zeros(1024, np.float64)
    n_exc = r.ref_rd_roundtrip_f64(ptr(vals), vals.size, ptr(vec), ptr(right), ptr(left),
                                   ptr(exc), ptr(pos), ptr(out))
    return {"right_bw": int(rbw[0]), "left_bw": int(lbw[0]), "dict_size": int(ds[0]),
            "dict_sorted": sorted(int(x) for x in dic[: int(ds[0])]),
            "n_exc": int(n_exc), "right": digest(right), "decoded": digest(out.view(np.uint64)),
            "exc_positions": digest(pos[:n_exc])}
