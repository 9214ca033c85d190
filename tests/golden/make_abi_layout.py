"""Writes tests/golden/abi_layout_reference.txt: tests/c/abi_layout.c
compiled against the reference's own C headers (wrapper/define/, read from
the reference tree in place) and run. The reference headers include
"monolis_utils.h" from the absent monolis_utils submodule only for its
logical constants; this library's include/monolis_utils.h stands in for it
(it defines nothing the listed structs contain).

    python tests/golden/make_abi_layout.py [--reference /path/to/monolis]
"""
import argparse
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    src = os.path.join(ROOT, "tests", "c", "abi_layout.c")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "abi_ref")
        subprocess.check_call(["gcc", "-std=c11", "-DABI_REFERENCE", "-I", os.path.join(args.reference, "wrapper",
                                                                                      "define"),
                               "-I", os.path.join(ROOT, "include"), src, "-o", exe])
        out = subprocess.check_output([exe], text=True)
    with open(os.path.join(HERE, "abi_layout_reference.txt"), "w") as f:
        f.write(out)
    print(f"{len(out.splitlines())} lines")


if __name__ == "__main__":
    main()
