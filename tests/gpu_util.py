"""Shared helpers for the GPU parity tests (inputs + oracle calls)."""
import numpy as np

from gradscf_b200 import basis as B

WATER = "O 0 0 0; H 0 0.7572 0.5865; H 0 -0.7572 0.5865"


def tables(atom, basis, cart, unit="Angstrom"):
    top, par, sa = B.prepare_basis(atom, basis, unit=unit, cart=cart)
    atm, bas, env = B.pack(top, par)
    return top, par, sa, atm, bas, env


def psd_density(n, nocc, seed):
    c = np.random.default_rng(seed).normal(size=(n, nocc)) / np.sqrt(n)
    return c @ c.T
