"""The oracle (oracle/oracle.c, a CPU restatement of the reference's
codecs) against golden digests of the reference's own CPU code
(tests/golden/ref_golden.json, made by tests/golden/gen_golden.py), and,
when oracle/_ref was built, against the reference directly on fresh seeds."""
import json
from pathlib import Path

import numpy as np
import pytest

import cases
from oracle import binding as B

GOLD = json.loads((Path(__file__).parent / "golden" / "ref_golden.json").read_text())
ORC = B.oracle()


def test_fls_pack_unpack_unffor_all_widths():
    for g in GOLD["fls"]:
        packed, unpacked, unffor = cases.run_fls(ORC, "orc", g)
        assert cases.digest(packed) == g["packed"], g
        assert cases.digest(unpacked) == g["unpacked"], g
        assert cases.digest(unffor) == g["unffor"], g


def test_falp_all_widths_below_full():
    for g in GOLD["falp"]:
        assert cases.digest(cases.run_falp(ORC, "orc", g)) == g["out"], g


@pytest.mark.parametrize("idx", range(8))
def test_alp_encode_matches_reference_encoder(idx):
    g = GOLD["alp_encode"][idx]
    enc = cases.run_orc_encode(ORC, g, rowgroup_vecs=0)
    if g["rd"]:
        assert enc is None  # reference throws alp::EncodingException
        return
    for k in cases.ENC_KEYS:
        assert cases.digest(enc[k]) == g[k], k
    assert enc["compressed_bytes"] == g["compressed_bytes"]
    assert enc["compressed_bytes_extended"] == g["compressed_bytes_extended"]


def _enc_of(g):
    return cases.run_orc_encode(ORC, g, rowgroup_vecs=0)


def test_alp_decode_and_extended_layout():
    for g, gx in zip(GOLD["alp_decode"], GOLD["extended"]):
        enc = _enc_of(g)
        dt = np.float64 if g["f64"] else np.float32
        ut = np.uint64 if g["f64"] else np.uint32
        dec = B.alp_decode(enc, g["n_vecs"], dt)
        full = g["full_width_vectors"]
        assert cases.digest(cases.mask_vectors(dec.view(ut), full)) == g["out"]
        # encode -> decode round trip is exact
        assert np.array_equal(dec.view(ut), cases.case_values(g).view(ut))
        x, ovf = B.to_extended(enc, g["n_vecs"], dt)
        # lanes with 64 exceptions overflow the 6-bit count field (structs.cuh:293-295),
        # exactly as in the reference; the digests below include that behaviour
        assert cases.digest(x["exceptions"]) == gx["x_exceptions"]
        assert cases.digest(x["positions"]) == gx["x_positions"]
        assert cases.digest(x["offsets_counts"]) == gx["x_offsets_counts"]
        xd = B.alp_decode(x, g["n_vecs"], dt, extended=True).view(ut)
        assert cases.digest(cases.mask_vectors(xd, full)) == gx["x_decoded"]


def test_rowgroup_topk():
    for g in GOLD["topk"]:
        assert cases.run_topk(ORC, "orc", g) == g["result"], g


def test_rd_init_and_roundtrip():
    for g in GOLD["rd"]:
        vals = cases.rd_values(g)
        st = B.RDState()
        ORC.orc_rd_init_f64(B.ptr(vals), vals.size, B.ctypes.byref(st) if hasattr(B, "ctypes") else __import__("ctypes").byref(st))
        assert st.right_bw == g["right_bw"] and st.left_bw == g["left_bw"]
        assert st.dict_size == g["dict_size"]
        assert sorted(st.dict[: st.dict_size]) == g["dict_sorted"]
        vec = np.ascontiguousarray(vals[1024:2048])
        right = np.zeros(1024, np.uint64)
        left = np.zeros(1024, np.uint16)
        exc = np.zeros(1024, np.uint16)
        pos = np.zeros(1024, np.uint16)
        import ctypes
        n = ORC.orc_rd_encode_vector_f64(B.ptr(vec), ctypes.byref(st), B.ptr(right), B.ptr(left),
                                         B.ptr(exc), B.ptr(pos))
        assert n == g["n_exc"]
        assert cases.digest(right) == g["right"]
        assert cases.digest(pos[:n]) == g["exc_positions"]
        out = np.zeros(1024, np.float64)
        ORC.orc_rd_decode_vector_f64(B.ptr(right), B.ptr(left), (ctypes.c_uint16 * 8)(*st.dict),
                                     st.right_bw, B.ptr(exc), B.ptr(pos), n, B.ptr(out))
        assert cases.digest(out.view(np.uint64)) == g["decoded"]
        assert np.array_equal(out.view(np.uint64), vec.view(np.uint64))


# ---- directly against the reference CPU build, fresh seeds ----------------
needs_ref = pytest.mark.skipif(B.ref() is None, reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("seed", [11, 12, 13])
def test_encode_fresh_seeds_against_reference(seed):
    r = B.ref()
    for f64 in (True, False):
        case = {"f64": f64, "uniform_d": seed % 2 == 1, "n_vecs": 25, "seed": seed * 31,
                "dmax": 4 if f64 else 3}
        ref = cases.run_ref_encode(r, case)
        mine = cases.run_orc_encode(ORC, case)
        assert (ref is None) == (mine is None)
        if ref is None:
            continue
        for k in cases.ENC_KEYS:
            assert np.array_equal(np.asarray(ref[k]).view(np.uint8), np.asarray(mine[k]).view(np.uint8)), k


@needs_ref
def test_full_width_falp_quirk_is_known():
    """The reference's CPU full-width falp kernels (src/alp/falp.cpp:33293,
    :42198) differ from its GPU ALPFunctor; the oracle follows ALPFunctor.
    Pin that the difference exists so a change in either is noticed."""
    r = B.ref()
    rng = np.random.default_rng(5)
    packed = rng.integers(0, 2 ** 63, 1024, dtype=np.uint64)
    a = np.zeros(1024, np.float64)
    b = np.zeros(1024, np.float64)
    r.ref_falp_f64(B.ptr(packed), B.ptr(a), 64, 3, 2, 5)
    ORC.orc_falp_f64(B.ptr(packed), B.ptr(b), 64, 3, 2, 5)
    assert not np.array_equal(a.view(np.uint64), b.view(np.uint64))


@needs_ref
@pytest.mark.parametrize("bits", [8, 16])
def test_small_widths_pack_ffor_against_reference(bits):
    """u8 / u16 FastLanes (fls::pack / unpack / ffor / unffor,
    src/fls/fls-bindings.hpp:8-52) at every width: the oracle writes the
    reference's words and decodes its words."""
    r = B.ref()
    ut = np.uint8 if bits == 8 else np.uint16
    rng = np.random.default_rng(bits)
    for w in range(bits + 1):
        base = int(rng.integers(0, 2 ** bits))
        vals = ((rng.integers(0, 2 ** w, 1024) + base) % 2 ** bits).astype(ut)
        raw = rng.integers(0, 2 ** w, 1024).astype(ut)
        for fn_pack, args in ((f"pack_u{bits}", (raw,)), (f"ffor_u{bits}", (vals, base))):
            a = np.zeros(1024, ut)
            b = np.zeros(1024, ut)
            getattr(r, "ref_" + fn_pack)(B.ptr(args[0]), B.ptr(a), w, *args[1:])
            getattr(ORC, "orc_" + fn_pack)(B.ptr(args[0]), B.ptr(b), w, *args[1:])
            n = w * (1024 // bits)
            assert np.array_equal(a[:n], b[:n]), (fn_pack, w)
        packed = rng.integers(0, 2 ** bits, 1024).astype(ut)
        for fn, extra in ((f"unpack_u{bits}", ()), (f"unffor_u{bits}", (base,))):
            a = np.zeros(1024, ut)
            b = np.zeros(1024, ut)
            getattr(r, "ref_" + fn)(B.ptr(packed), B.ptr(a), w, *extra)
            getattr(ORC, "orc_" + fn)(B.ptr(packed), B.ptr(b), w, *extra)
            assert np.array_equal(a, b), (fn, w)
