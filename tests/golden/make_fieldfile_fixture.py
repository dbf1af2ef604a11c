"""Copy the reference's basis-format field file fixture
(tools/python/tests/fieldfile/rho: converged lamellar rho, group -1,
21 stars) into tests/golden/fieldfile_rho.txt.  Run once where the
reference tree is available:
    python tests/golden/make_fieldfile_fixture.py REFERENCE_TREE
(or with the path in the PSCF_REFERENCE environment variable).
"""
import os
import sys

DST = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fieldfile_rho.txt")

if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PSCF_REFERENCE")
    if not ref:
        sys.exit("usage: make_fieldfile_fixture.py REFERENCE_TREE  (or set PSCF_REFERENCE)")
    SRC = os.path.join(ref, "tools/python/tests/fieldfile/rho")
    with open(SRC) as f:
        text = f.read()
    with open(DST, "w") as f:
        f.write(text)
    print("wrote", DST)
