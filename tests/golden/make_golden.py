"""Extract the reference's golden values into tests/golden/golden.json.

Run once where the reference tree is available, giving its path as
argv[1] or in the PSCF_REFERENCE environment variable; the JSON it writes
is committed so that tests never read the reference at run time.

Sources (paths inside the reference project):
  tools/python/tests/outfile/in          converged 1-D lamellar run (thermo)
  tools/python/tests/sweep/out/{0..11}.out  BCC 'I m -3 m' 20^3 sweep
  src/space_groups_mod.f90               element tables of the groups used
                                          by the benchmark configurations
"""
import json
import os
import re
import sys
from fractions import Fraction

def reference_root() -> str:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PSCF_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py REFERENCE_TREE  (or set PSCF_REFERENCE)")
    return ref


REF = reference_root() if __name__ == "__main__" else None
HERE = os.path.dirname(os.path.abspath(__file__))


def read_out(path):
    """Parse a PSCF .out / param file: 'label' line followed by value line(s)."""
    lines = open(path).read().splitlines()
    vals = {}
    for i, ln in enumerate(lines):
        key = ln.strip()
        if re.fullmatch(r"[a-zA-Z_]+", key) and i + 1 < len(lines):
            nxt = lines[i + 1].split()
            try:
                vals[key] = [float(x.replace("D", "E")) for x in nxt]
            except ValueError:
                vals[key] = [x.strip("'") for x in nxt]
    return vals


def thermo(path):
    v = read_out(path)
    keys = ["block_length", "chi", "cell_param", "ngrid", "chain_step", "group_name",
            "f_Helmholtz", "f_homo", "pressure", "mu_chain", "stress", "N_star", "final_error"]
    return {k: v[k] for k in keys if k in v}


def group_table(src, name):
    """Elements (m, v) of one group of src/space_groups_mod.f90."""
    lines = open(src).read().splitlines()
    start = None
    for i, ln in enumerate(lines):
        if ln.strip().startswith("case(") and ("'" + name + "'") in ln:
            start = i
            break
    if start is None:
        raise KeyError(name)
    order = None
    elems = {}
    for ln in lines[start + 1:]:
        s = ln.strip()
        if s.startswith("case("):
            break
        m = re.match(r"g%order\s*=\s*(\d+)", s)
        if m:
            order = int(m.group(1))
        m = re.match(r"g%s\((\d+)\)%m\((\d),(\d)\)\s*=\s*([-0-9.]+)", s)
        if m:
            k, i, j, val = int(m.group(1)), int(m.group(2)), int(m.group(3)), float(m.group(4))
            elems.setdefault(k, {"m": {}, "v": {}})["m"][(i, j)] = val
        m = re.match(r"g%s\((\d+)\)%v\((\d)\)\s*=\s*([-0-9.]+)", s)
        if m:
            k, i, val = int(m.group(1)), int(m.group(2)), float(m.group(3))
            elems.setdefault(k, {"m": {}, "v": {}})["v"][i] = val
    out = []
    for k in range(1, order + 1):
        e = elems.get(k, {"m": {}, "v": {}})
        mat = [[int(round(e["m"].get((i, j), 0.0))) for j in (1, 2, 3)] for i in (1, 2, 3)]
        vec = [str(Fraction(e["v"].get(i, 0.0)).limit_denominator(48)) for i in (1, 2, 3)]
        out.append({"m": mat, "v": vec})
    return out


def main():
    g = {}
    g["lamellar_outfile"] = thermo(os.path.join(REF, "tools/python/tests/outfile/in"))
    g["bcc_sweep"] = [thermo(os.path.join(REF, "tools/python/tests/sweep/out/%d.out" % i)) for i in range(12)]
    src = os.path.join(REF, "src/space_groups_mod.f90")
    g["groups"] = {name: group_table(src, name)
                   for name in ["-1", "p 6 m m", "I m -3 m", "I a -3 d", "F d d d : 2", "I 41 3 2"]}
    g["source"] = {
        "lamellar_outfile": "tools/python/tests/outfile/in",
        "bcc_sweep": "tools/python/tests/sweep/out/{0..11}.out",
        "groups": "src/space_groups_mod.f90",
    }
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
