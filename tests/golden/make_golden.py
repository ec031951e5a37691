"""Regenerates tests/golden/ref_tables.txt from the reference's own headers.

Builds oracle/_ref/ref_tables (oracle/Makefile, target `ref`) from
element/GaussQuadrature.h and element/LagrangeShapeFuncs.h where they lie in the
reference checkout, runs it and stores its output (exact hexadecimal floats).
Usage: python tests/golden/make_golden.py [REFERENCE_DIR]
"""
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref", f"REF={ref}"], check=True)
    out = subprocess.run([str(ROOT / "oracle" / "_ref" / "ref_tables")], check=True, capture_output=True, text=True)
    (HERE / "ref_tables.txt").write_text(out.stdout)
    print(f"wrote {HERE / 'ref_tables.txt'} ({len(out.stdout.splitlines())} lines)")


if __name__ == "__main__":
    main()
