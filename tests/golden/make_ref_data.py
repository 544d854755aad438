"""Copies the reference's only shipped seed sets into fixtures.

The reference repository ships three 97,336-seed point sets in its own text
.xyz format (data/100K-{blue,white,perturbed-grid}.xyz, README.md:15-25;
coordinates already in the reference frame [0,1000]^3).  The parity tests
need them on machines where the reference checkout is absent, so this
script stores each file unchanged, xz-compressed, as
tests/golden/ref_data_100k-<name>.xyz.xz; the tests decompress them and read
them through the library's own seed loader (rpd_seeds_load).

    RPD_REFERENCE_DIR=<reference checkout> python tests/golden/make_ref_data.py
"""
import lzma
import os
import sys

NAMES = ("blue", "white", "perturbed-grid")


def main():
    ref = os.environ.get("RPD_REFERENCE_DIR") or (sys.argv[1] if len(sys.argv) > 1 else None)
    if not ref:
        sys.exit("give the reference checkout (argument or RPD_REFERENCE_DIR)")
    here = os.path.dirname(os.path.abspath(__file__))
    for name in NAMES:
        src = os.path.join(ref, "data", f"100K-{name}.xyz")
        with open(src, "rb") as f:
            raw = f.read()
        dst = os.path.join(here, f"ref_data_100k-{name}.xyz.xz")
        with lzma.open(dst, "wb", preset=9) as f:
            f.write(raw)
        print(f"{src} -> {dst} ({len(raw)} bytes, {os.path.getsize(dst)} compressed)")


if __name__ == "__main__":
    main()
