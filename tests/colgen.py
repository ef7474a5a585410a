"""Seeded synthetic columns for the parity tests, generated at the
compressed level like the reference's own test fixtures
(src/engine/data.cuh:354-477: random packed words at a chosen width, random
bases, random ALP parameters and exceptions), or at the value level and
encoded with the oracle encoder."""
from __future__ import annotations

import numpy as np

from oracle import binding as B


def random_ffor(seed: int, n_vecs: int, bits: int, widths, base_max: int | None = None,
                n_values: int | None = None):
    """Random FastLanes column: per-vector width drawn from `widths`, random
    packed words (every value uniform in [0, 2^w)), random bases."""
    rng = np.random.default_rng(seed)
    ut = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}[bits]
    nl = 1024 // bits
    bw = rng.choice(np.asarray(list(widths)), n_vecs).astype(np.uint8)
    offs = np.zeros(n_vecs, np.uint64)
    offs[1:] = np.cumsum(bw.astype(np.uint64) * nl)[:-1]
    n_packed = int(bw.astype(np.int64).sum()) * nl
    packed = rng.integers(0, 2 ** bits, max(n_packed, 1), dtype=np.uint64).astype(ut)[:n_packed]
    hi = 2 ** bits if base_max is None else base_max
    bases = rng.integers(0, hi, n_vecs, dtype=np.uint64).astype(ut)
    return dict(packed=packed, bit_widths=bw, vector_offsets=offs, bases=bases,
                n_values=n_vecs * 1024 if n_values is None else n_values)


def ffor_config1(seed: int = 1):
    """2^20 uint32 values as 1024 vectors; per-vector base uniform in
    [0, 2^20), values base + uniform [0, 2^7); encoded with the oracle's
    analyze-FFOR (base = min, w = bits(max - min))."""
    rng = np.random.default_rng(seed)
    n_vecs = 1024
    base = rng.integers(0, 2 ** 20, n_vecs, dtype=np.uint64).astype(np.uint32)
    vals = (np.repeat(base, 1024) + rng.integers(0, 2 ** 7, n_vecs * 1024).astype(np.uint32))
    vals = vals.astype(np.uint32)
    return vals, ffor_encode(vals, 32)


def ffor_encode(vals: np.ndarray, bits: int):
    o = B.oracle()
    ut = np.uint64 if bits == 64 else np.uint32
    n_vecs = vals.size // 1024
    nl = 1024 // bits
    v = vals.reshape(n_vecs, 1024)
    mn = v.min(axis=1)
    delta = (v.max(axis=1) - mn).astype(np.uint64)
    bw = np.array([int(d).bit_length() for d in delta], np.uint8)
    offs = np.zeros(n_vecs, np.uint64)
    offs[1:] = np.cumsum(bw.astype(np.uint64) * nl)[:-1]
    packed = np.zeros(int(bw.astype(np.int64).sum()) * nl + 1, ut)
    buf = np.zeros(1024, ut)
    for i in range(n_vecs):
        row = np.ascontiguousarray(v[i], ut)
        getattr(o, f"orc_ffor_u{bits}")(B.ptr(row), B.ptr(buf), int(bw[i]), int(mn[i]))
        n = int(bw[i]) * nl
        packed[int(offs[i]): int(offs[i]) + n] = buf[:n]
    return dict(packed=packed[:-1], bit_widths=bw, vector_offsets=offs,
                bases=mn.astype(ut), n_values=vals.size)


def random_alp(seed: int, n_vecs: int, f64: bool, widths, exc_counts,
               fac_max: int | None = None, exp_max: int | None = None):
    """Compressed-level ALP column as the reference's generate_alp_column
    (data.cuh:437-477): random FFOR part with bases in [2, 20], factor /
    fraction indices in [0, COUNT/2], per-vector exception counts drawn from
    exc_counts, random bit patterns as exceptions at sorted random
    positions."""
    rng = np.random.default_rng(seed)
    bits = 64 if f64 else 32
    dt = np.float64 if f64 else np.float32
    col = random_ffor(seed + 1, n_vecs, bits, widths)
    col["bases"] = rng.integers(2, 21, n_vecs).astype(col["bases"].dtype)
    nf, ne = (19, 21) if f64 else (10, 11)
    col["factor_indices"] = rng.integers(0, (fac_max if fac_max is not None else nf // 2) + 1,
                                         n_vecs).astype(np.uint8)
    col["fraction_indices"] = rng.integers(0, (exp_max if exp_max is not None else ne // 2) + 1,
                                           n_vecs).astype(np.uint8)
    counts = rng.choice(np.asarray(list(exc_counts)), n_vecs).astype(np.uint16)
    eo = np.zeros(n_vecs, np.uint64)
    eo[1:] = np.cumsum(counts.astype(np.uint64))[:-1]
    n_exc = int(counts.astype(np.int64).sum())
    exc = rng.integers(0, 2 ** bits, max(n_exc, 1), dtype=np.uint64)
    exc = exc.astype(np.uint64 if f64 else np.uint32).view(dt)[:n_exc].copy()
    pos = np.zeros(n_exc, np.uint16)
    for i in range(n_vecs):
        c = int(counts[i])
        pos[int(eo[i]): int(eo[i]) + c] = np.sort(rng.permutation(1024)[:c])
    col.update(counts=counts, exceptions_offsets=eo, exceptions=exc, positions=pos)
    return col


def alp_values(seed: int, n_vecs: int, f64: bool, dmax: int, exc_rate: float = 0.01,
               per_vector_d: bool = True) -> np.ndarray:
    """Value-level ALP data: integers uniform in [-10^6, 10^6] / 10^d with d
    uniform per vector in [0, dmax], exc_rate of positions replaced by
    random non-NaN bit patterns."""
    rng = np.random.default_rng(seed)
    dt = np.float64 if f64 else np.float32
    bits = 64 if f64 else 32
    ut = np.uint64 if f64 else np.uint32
    ints = rng.integers(-10 ** 6, 10 ** 6 + 1, n_vecs * 1024)
    d = rng.integers(0, dmax + 1, n_vecs) if per_vector_d else np.full(n_vecs, dmax)
    vals = (ints / (10.0 ** np.repeat(d, 1024))).astype(dt)
    m = rng.random(vals.size) < exc_rate
    pat = rng.integers(0, 2 ** bits, int(m.sum()), dtype=np.uint64).astype(ut)
    f = pat.view(dt)
    pat[np.isnan(f)] &= ut((1 << bits) - 1 - (1 << (bits - 2)))
    v = vals.view(ut).copy()
    v[m] = pat
    return v.view(dt)


def learned_values(seed: int, n_vecs: int) -> np.ndarray:
    """Value-level f64 columns of the learned-proposal benchmark shape: per
    vector d in {0..6} decimal digits, scale 10^k (k in 0..8), Gaussian or
    uniform magnitude; 10% of the vectors are full-mantissa noise."""
    rng = np.random.default_rng(seed)
    d = rng.integers(0, 7, n_vecs)
    k = rng.integers(0, 9, n_vecs)
    gauss = rng.random(n_vecs) < 0.5
    noise = rng.random(n_vecs) < 0.1
    m = np.where(np.repeat(gauss, 1024), rng.standard_normal(n_vecs * 1024),
                 rng.uniform(-1.0, 1.0, n_vecs * 1024))
    scale = 10.0 ** np.repeat(k, 1024)
    dd = 10.0 ** np.repeat(d, 1024)
    vals = np.round(m * scale * dd) / dd
    vals = np.where(np.repeat(noise, 1024), m * scale, vals)
    return vals.astype(np.float64)
