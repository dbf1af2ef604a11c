"""Copy the reference's basis-format field file fixture
(tools/python/tests/fieldfile/rho: converged lamellar rho, group -1,
21 stars) into tests/golden/fieldfile_rho.txt.  Run once where the
reference tree is available:  python tests/golden/make_fieldfile_fixture.py
"""
import os
import sys

SRC = os.path.join(sys.argv[1] if len(sys.argv) > 1 else "/root/reference", "tools/python/tests/fieldfile/rho")
DST = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fieldfile_rho.txt")

if __name__ == "__main__":
    with open(SRC) as f:
        text = f.read()
    with open(DST, "w") as f:
        f.write(text)
    print("wrote", DST)
