"""Generates tests/golden/ref_golden.json from the reference's own CPU code
(oracle/_ref/libflsref.so, built from the reference sources by
oracle/build_ref.sh).

Inputs are regenerated from numpy seeds (tests/golden/cases.py), so the
fixture stores only case parameters and SHA-256 digests of the reference's
outputs.  Run from the repository root:

    bash oracle/build_ref.sh && python tests/golden/gen_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from oracle import binding as B  # noqa: E402
import cases  # noqa: E402


def main() -> None:
    r = B.ref()
    if r is None:
        raise SystemExit("oracle/_ref/libflsref.so not built")
    out = {"fls": [], "falp": [], "alp_encode": [], "alp_decode": [], "extended": [],
           "topk": [], "rd": []}
    for case in cases.fls_cases():
        packed, unpacked, unffor = cases.run_fls(r, "ref", case)
        out["fls"].append(dict(case, packed=cases.digest(packed), unpacked=cases.digest(unpacked),
                               unffor=cases.digest(unffor)))
    for case in cases.falp_cases():
        res = cases.run_falp(r, "ref", case)
        out["falp"].append(dict(case, out=cases.digest(res)))
    for case in cases.alp_column_cases():
        enc = cases.run_ref_encode(r, case)
        if enc is None:
            out["alp_encode"].append(dict(case, rd=True))
            continue
        out["alp_encode"].append(dict(case, rd=False, **{k: cases.digest(v) if isinstance(v, np.ndarray) else v
                                                      for k, v in enc.items()}))
        dec = cases.run_ref_decode(r, case, enc)
        full = cases.full_width_vectors(case, enc)
        out["alp_decode"].append(dict(case, out=cases.digest(cases.mask_vectors(dec, full)),
                                      full_width_vectors=full))
        ext = cases.run_ref_extended(r, case, enc)
        ext["x_decoded"] = cases.mask_vectors(ext["x_decoded"], full)
        out["extended"].append(dict(case, **{k: cases.digest(v) for k, v in ext.items()}))
    for case in cases.topk_cases():
        out["topk"].append(dict(case, result=cases.run_topk(r, "ref", case)))
    for case in cases.rd_cases():
        out["rd"].append(dict(case, **cases.run_ref_rd(r, case)))
    path = Path(__file__).resolve().parent / "ref_golden.json"
    path.write_text(json.dumps(out, indent=1, sort_keys=True))
    print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
