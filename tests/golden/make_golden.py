"""Regenerate the golden fixtures of the OLAP-core star-join.

Run where the reference tree is present (read only; its location is
$OLAP_REFERENCE_TREE); the GPU tests and the bench read only the JSON
written here.

* ``olapcore_queries.json`` — the ten query parameterisations of the
  reference's ``OLAPcore.sh`` (lines 3-12), parsed from that script, each
  with the grand total the reference published for SF=100 (parsed from the
  recorded GPU_OLAPcore output in ``GPU/plot/old.py``) and the grand total
  its CPU OLAPcore prints at SF=1 (the reference compiled from its sources by
  ``oracle/Makefile`` and run here through ``oracle/_ref``).
* ``olapcore_sf1_groups.json`` — per-group sums of the reference's own
  vector-wise static-vector thread body at SF=1 for the queries whose group
  count fits its int16 group ids.

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle  # noqa: E402  (test infrastructure)

REF = Path(os.environ.get("OLAP_REFERENCE_TREE", "/root/reference"))
OUT = Path(__file__).resolve().parent
FLAGS = ["d-sele", "d-bitmap", "d-groups", "s-sele", "s-bitmap", "s-groups", "p-sele",
         "p-bitmap", "p-groups", "c-sele", "c-bitmap", "c-groups", "sqlnum"]


def parse_queries() -> list[dict]:
    qs = []
    for line in (REF / "OLAPcore.sh").read_text().splitlines():
        if "--SF" not in line:
            continue
        kv = dict(re.findall(r"--([\w-]+)=([\d.]+)", line))
        # table order of the reference: customer, supplier, part, date
        q = {
            "sqlnum": int(kv["sqlnum"]),
            "sele": [float(kv[f"{t}-sele"]) for t in "cspd"],
            "bitmap": [int(kv[f"{t}-bitmap"]) for t in "cspd"],
            "groups": [int(kv[f"{t}-groups"]) for t in "cspd"],
            "sf_script": float(kv["SF"]),
        }
        qs.append(q)
    return qs


def parse_published() -> list[int]:
    text = (REF / "GPU" / "plot" / "old.py").read_text()
    blocks = text.split(">>> Generated data")[1:]
    totals = []
    for b in blocks:
        vals = {int(v) for v in re.findall(r"Result count of total selection rate [\d.e-]+% is (\d+)/", b)}
        assert len(vals) == 1, f"variants disagree in a published block: {vals}"
        totals.append(vals.pop())
    return totals


def main() -> None:
    oracle.build(with_reference=True)
    ref = oracle.ref_lib()
    qs = parse_queries()
    pub = parse_published()
    assert len(qs) == len(pub) == 10
    groups_out = {}
    for q, total in zip(qs, pub):
        q["total_sf100_published"] = total
        dv, fk, m1, m2 = oracle.gen_olapcore_compat(1.0, q["sele"], q["bitmap"], q["groups"],
                                                    use_reference=True)
        orders, factor, nd, gn = oracle.plan(q["sele"], q["bitmap"], q["groups"])
        q.update(orders=orders, factor=factor, dimvec_nums=nd, group_nums=gn)
        n = len(m1)
        dva = oracle._ptr_array(dv)
        fka = oracle._ptr_array(fk)
        o = np.array(orders + [0] * (4 - nd), np.int32)
        f = np.array(factor + [0] * (4 - nd), np.int32)
        q["total_sf1_reference"] = int(ref.ref_OLAPcore_vwm_sv(dva, fka, oracle._p(o), nd, oracle._p(f), n, gn,
                                                               oracle._p(m1), oracle._p(m2), 4))
        if gn <= 32766:
            gv = np.zeros(gn, np.uint32)
            ref.ref_vwm_sv_groups(dva, fka, oracle._p(o), nd, oracle._p(f), 0, n, oracle._p(m1),
                                  oracle._p(m2), oracle._p(gv))
            groups_out[str(q["sqlnum"])] = gv.astype(np.int64).tolist()
    (OUT / "olapcore_queries.json").write_text(json.dumps(qs, indent=1) + "\n")
    (OUT / "olapcore_sf1_groups.json").write_text(json.dumps(groups_out) + "\n")
    print(json.dumps([(q["sqlnum"], q["total_sf1_reference"], q["total_sf100_published"]) for q in qs]))


if __name__ == "__main__":
    main()
