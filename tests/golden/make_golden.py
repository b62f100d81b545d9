"""Regenerate the golden fixtures in this folder.

* g01_water_rhf.json -- copied from the reference's published record
  reproducibility/ad_showcase/G01_water_rhf_gradient/gradscf.json (RHF/6-31G*
  Cartesian water: total energy and analytic nuclear gradient).
* h2_sto3g_jk.json -- the reference test tests/integrals/test_native_jk_dispatch.py:15-33
  inputs (H 0 0 0; H .2 -.1 .8 Angstrom, sto-3g, D = [[.8,-.2],[.3,.6]]) with the
  full-ERI einsum J/K computed by the oracle (libcint built from the reference sources).
* h2_general_jk.json -- tests/integrals/test_native_direct_parallel.py:16-34
  hand-written general-contraction basis with a d shell (both cart and sph),
  seeded nonsymmetric densities (default_rng(801), nvec 4), einsum J/K.

Usage: python tests/golden/make_golden.py <reference checkout>  (or GRADSCF_REFERENCE=<checkout>)
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from gradscf_b200 import basis as B  # noqa: E402
import oracle  # noqa: E402

GENERAL_BASIS = [[0, [2.0, 0.8, -0.2], [0.4, 0.3, 1.0]], [1, [0.8, 1.0]], [2, [0.6, 1.0]]]


def main(reference):
    here = Path(__file__).resolve().parent
    record = json.loads((Path(reference) / "reproducibility/ad_showcase/G01_water_rhf_gradient/gradscf.json").read_text())
    (here / "g01_water_rhf.json").write_text(json.dumps({
        "source": "reproducibility/ad_showcase/G01_water_rhf_gradient/gradscf.json",
        "basis": record["basis"], "cart": record["cart"], "symbols": record["symbols"],
        "coordinates_bohr": record["coordinates_bohr"], "energy_hartree": record["energy_hartree"],
        "gradient_hartree_per_bohr": record["gradient_hartree_per_bohr"]}, indent=1))

    top, par, _ = B.prepare_basis("H 0 0 0; H .2 -.1 .8", "sto-3g", cart=True)
    atm, bas, env = B.pack(top, par)
    d = np.array([[.8, -.2], [.3, .6]])
    j, k = oracle.full_jk(oracle.eri_s1(atm, bas, env, cart=True), d)
    (here / "h2_sto3g_jk.json").write_text(json.dumps({
        "atom": "H 0 0 0; H .2 -.1 .8", "basis": "sto-3g", "cart": True, "density": d.tolist(),
        "j": j.tolist(), "k": k.tolist()}, indent=1))

    out = {}
    for cart in (False, True):
        top, par, _ = B.prepare_basis("H 0 0 0; H 0.1 0.2 1.1", GENERAL_BASIS, cart=cart)
        atm, bas, env = B.pack(top, par)
        dens = np.random.default_rng(801).normal(size=(4, top.nao, top.nao))
        j, k = oracle.full_jk(oracle.eri_s1(atm, bas, env, cart=cart), dens)
        out["cart" if cart else "sph"] = {"density": dens.tolist(), "j": j.tolist(), "k": k.tolist()}
    out.update(atom="H 0 0 0; H 0.1 0.2 1.1", basis=GENERAL_BASIS, seed=801)
    (here / "h2_general_jk.json").write_text(json.dumps(out))
    print("golden fixtures written")


if __name__ == "__main__":
    import os
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GRADSCF_REFERENCE")
    if not root:
        sys.exit("give the reference checkout as the argument or in GRADSCF_REFERENCE")
    main(root)
