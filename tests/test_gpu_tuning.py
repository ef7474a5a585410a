"""The decode autotuner on the device: it measures every configuration,
returns a complete table, installs it (and restores the previous one on
request), and decoding stays bit-exact under the table it picks."""
import numpy as np
import pytest

import colgen
import flsgpu_b200 as F
from oracle import binding as B

pytestmark = pytest.mark.gpu


def test_autotune_small_sizes_installs_a_complete_table(cuda):
    before = F.tuning_get()
    try:
        r = F.autotune(values_32=2 ** 18, values_64=2 ** 17, reps=1, alp_widths=(8, 20))
        t = r["table"]
        for tn, kn in (("u32", "ffor"), ("u32", "bp"), ("u64", "ffor"), ("u64", "bp"),
                       ("f32", "alp"), ("f32", "alpx"), ("f64", "alp"), ("f64", "alpx")):
            assert t["variant"][(tn, kn)] in (F.VARIANT_REGS, F.VARIANT_OCCUPANCY,
                                              F.VARIANT_STAGED)
        assert set(t["prefetch"]) == {32, 64}
        assert len(r["report"]["ffor"]["u32"]["gbs"][str(F.VARIANT_REGS)]) == 33
        assert len(r["report"]["ffor"]["u64"]["gbs"][str(F.VARIANT_OCCUPANCY)]) == 65
        now = F.tuning_get()
        for k, v in t["variant"].items():
            assert now["variant"][k] == v
        assert now["prefetch"][32] == t["prefetch"][32]
        # decode under the installed table is still exact
        for bits in (32, 64):
            ut = np.uint64 if bits == 64 else np.uint32
            c = colgen.random_ffor(90 + bits, 700, bits, range(bits + 1))
            col = F.make_ffor_column(c["packed"], c["bit_widths"], c["vector_offsets"],
                                     c["bases"], c["n_values"], cuda)
            got = F.decompress(col).cpu().numpy().view(ut)
            want = B.decode_ffor(c["packed"], c["bit_widths"], c["vector_offsets"], c["bases"],
                                 bits)
            assert np.array_equal(got, want)
        r2 = F.autotune(values_32=2 ** 16, values_64=2 ** 16, reps=1, install=False,
                        alp_widths=(8,))
        assert F.tuning_get() == now
        assert r2["defaults"] == now
    finally:
        F.tuning_set(before)
