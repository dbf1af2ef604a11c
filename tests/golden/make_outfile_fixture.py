"""Copy the reference's output summary files into tests/golden/: the twelve
files of a sweep, tools/python/tests/sweep/out/0.out ... 11.out (BCC
I m -3 m 20^3, NR with N_cut, block length 0.39 -> 0.28 in steps of -0.01),
as sweep/0.out ... 11.out, and tools/python/tests/outfile/in (lamellar,
group -1) as lamellar.out.  Run once where the reference tree is available:
    python tests/golden/make_outfile_fixture.py REFERENCE_TREE
(or with the path in the PSCF_REFERENCE environment variable).
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = {f"tools/python/tests/sweep/out/{j}.out": f"sweep/{j}.out" for j in range(12)}
FILES["tools/python/tests/outfile/in"] = "lamellar.out"

if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PSCF_REFERENCE")
    if not ref:
        sys.exit("usage: make_outfile_fixture.py REFERENCE_TREE  (or set PSCF_REFERENCE)")
    os.makedirs(os.path.join(HERE, "sweep"), exist_ok=True)
    for src, dst in FILES.items():
        with open(os.path.join(ref, src)) as f:
            text = f.read()
        with open(os.path.join(HERE, dst), "w") as f:
            f.write(text)
        print("wrote", os.path.join(HERE, dst))
