"""Regenerate basis_sets.json from the reference's vendored basis-set data.

Run in a checkout that has the reference next to it:

    python gradscf_b200/basis_data/gen_basis_data.py <reference checkout>

(or set GRADSCF_REFERENCE to the checkout and give no argument).

It loads the reference's own snapshot parser
(src/gradscf/integrals/basis/data/__init__.py, functions
``load_basis_from_snapshot`` and friends at :262-298) straight from its file,
without importing the reference package, and stores the raw blocks
``[l, [exponent, c1, c2, ...], ...]`` it returns -- unsorted and unnormalised,
exactly as ``prepare_basis`` (src/gradscf/integrals/basis/library.py:30-46)
consumes them -- for the elements and basis names below.  The output is the
only basis data the package reads; the reference is not needed at run time.
"""
import importlib.util
import json
import sys
from pathlib import Path

BASES = ("sto-3g", "3-21g", "6-31g", "6-31g*", "cc-pvdz", "cc-pvtz")
ELEMENTS = ("H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne")


def main(reference_root):
    path = (Path(reference_root) / "src/gradscf/integrals/basis/data/__init__.py").resolve()
    spec = importlib.util.spec_from_file_location("_reference_basis_data", path)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    out = {}
    for name in BASES:
        out[name] = {}
        for symbol in ELEMENTS:
            try:
                out[name][symbol] = module.load_basis_from_snapshot(name, symbol)
            except KeyError:
                continue
    target = Path(__file__).with_name("basis_sets.json")
    target.write_text(json.dumps(out, separators=(",", ":")))
    print(f"wrote {target} ({target.stat().st_size} bytes)")


if __name__ == "__main__":
    import os
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GRADSCF_REFERENCE")
    if not root:
        sys.exit("give the reference checkout as the argument or in GRADSCF_REFERENCE")
    main(root)
