"""Writes materials_subset.json: the records of the reference's material database
(src/materials-db.json of the reference) that the host-side material tests use, with each
parameter reduced to its value and unit. Run in a container that holds the reference:

    python tests/golden/make_material_fixtures.py /path/to/reference/src/materials-db.json
"""
import copy
import json
import os
import sys

IDS = ["uf9000ae", "abf_gl", "cu", "mcl_e_795g", "psr4000", "sac305", "si", "tim_gel", "eccobond3005", "mcl_e_705g",
       "mcl_e_795g_lh", "sn35ag", "cv5300", "ei6042"]


def values(o):
    if isinstance(o, dict):
        if "v" in o and not isinstance(o["v"], list):
            return {"v": o["v"], "u": o.get("u")}
        # s, c, n, r: a parameter's sources, confidence, note and remark (the Anand exponent n is a parameter)
        return {k: values(v) for k, v in o.items() if k not in ("s", "c", "n", "r") or isinstance(v, dict)}
    if isinstance(o, list):
        return [values(v) for v in o]
    return o


def expand(m, by_id):
    """A preset record (presetOf + override) as its complete record, as the tool's
    buildMaterialLibrary expands it: the base record, the preset's own fields, then each override
    path set."""
    if not m.get("presetOf"):
        return m
    r = copy.deepcopy(by_id[m["presetOf"]])
    r.update({k: copy.deepcopy(v) for k, v in m.items() if k != "override"})
    for path, val in (m.get("override") or {}).items():
        o = r
        ks = path.split(".")
        for k in ks[:-1]:
            o = o.setdefault(k, {})
        o[ks[-1]] = copy.deepcopy(val)
    return r


def main(path):
    db = json.load(open(path))
    by_id = {m["id"]: m for m in db["materials"]}
    out = {}
    for m in db["materials"]:
        if m["id"] in IDS:
            m = expand(m, by_id)
            out[m["id"]] = {k: values(m[k]) for k in ("elastic", "cte", "cteXY", "cteZ", "solidus", "anand") if k in m}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "materials_subset.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", dst, sorted(out))


if __name__ == "__main__":
    main(sys.argv[1])
