"""Molecule parsing, named basis sets and libcint-layout tables (host side).

Mirrors the reference's input preparation so that the same ``atm/bas/env``
arrays reach both this package's GPU path and the CPU oracle:

* ``parse_molecule``  -- src/gradscf/data/molecule.py:101-180 ("Sym x y z"
  records separated by ';' or newlines, Angstrom or Bohr,
  ANGSTROM_TO_BOHR = 1.8897261245650618 as at :10).
* ``prepare_basis``   -- src/gradscf/integrals/basis/library.py:5-51 (raw,
  unsorted, unnormalised shells in atom order; general contractions kept).
* ``normalized_shell_coefficients`` -- basis/normalization.py:50-63.
* ``build_tables`` / ``pack`` -- backends/native/packing.py:17-47,78-95:
  nuclear atoms first, then one zero-charge centre atom per shell, ``env``
  data from offset 20, coefficients stored ``c.T.ravel()``.

Everything here is numpy; nothing touches the GPU.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass
from functools import lru_cache
from pathlib import Path

import numpy as np

ANGSTROM_TO_BOHR = 1.8897261245650618
ATM_SLOTS, BAS_SLOTS, PTR_ENV_START = 6, 8, 20

_SYMBOLS = ("H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si",
            "P", "S", "Cl", "Ar")
_Z = {s: i + 1 for i, s in enumerate(_SYMBOLS)}


@dataclass(frozen=True)
class Molecule:
    symbols: tuple
    coords_bohr: np.ndarray
    charges: np.ndarray

    @property
    def nelectron(self) -> int:
        return int(self.charges.sum())


def parse_molecule(atom, unit="Angstrom") -> Molecule:
    """Parse 'Sym x y z; ...' text or an iterable of (symbol, (x, y, z))."""
    if isinstance(atom, Molecule):
        return atom
    records = []
    if isinstance(atom, str):
        for raw in atom.replace(";", "\n").splitlines():
            line = raw.strip()
            if not line:
                continue
            parts = line.split()
            if len(parts) != 4:
                raise ValueError(f"Atom specification lines must have form 'Sym x y z'. Got {line!r}.")
            records.append((parts[0], tuple(float(v) for v in parts[1:])))
    else:
        for item in atom:
            if len(item) != 2:
                raise ValueError("Iterable atom specification must contain (symbol, (x,y,z)) pairs.")
            records.append((str(item[0]), tuple(float(v) for v in np.asarray(item[1]).reshape(3))))
    if not records:
        raise ValueError("Atom specification must contain at least one atom.")
    symbols = tuple(s.strip().capitalize() for s, _ in records)
    for s in symbols:
        if s not in _Z:
            raise ValueError(f"Unsupported element symbol {s!r}.")
    coords = np.asarray([xyz for _, xyz in records], dtype=np.float64)
    u = str(unit).strip().lower()
    if u.startswith("angs"):
        coords = coords * ANGSTROM_TO_BOHR
    elif not u.startswith("bohr"):
        raise ValueError(f"Unsupported unit={unit!r}. Expected 'Angstrom' or 'Bohr'.")
    return Molecule(symbols, coords, np.asarray([_Z[s] for s in symbols], dtype=np.float64))


@lru_cache(maxsize=1)
def _basis_library():
    path = Path(__file__).with_name("basis_data") / "basis_sets.json"
    return json.loads(path.read_text())


def _format_name(name: str) -> str:
    return str(name).lower().replace("-", "").replace("_", "").replace(" ", "")


def load_basis(name: str, symbol: str):
    """Raw blocks [l, [exp, c1, ...], ...] for a named basis and element."""
    lib = _basis_library()
    key = {_format_name(k): k for k in lib}.get(_format_name(name))
    if key is None:
        raise KeyError(f"Basis {name!r} is not bundled (have: {sorted(lib)}).")
    if symbol not in lib[key]:
        raise KeyError(f"Basis {name!r} has no data for {symbol!r}.")
    return [list(block) for block in lib[key][symbol]]


@dataclass(frozen=True)
class BasisTopology:
    """Static shell structure (src/gradscf/integrals/basis/types.py:6-28)."""
    angular_momenta: tuple
    primitive_counts: tuple
    contraction_counts: tuple
    nuclear_charges: tuple
    cart: bool = True

    @property
    def nao(self) -> int:
        return sum(((l + 1) * (l + 2) // 2 if self.cart else 2 * l + 1) * nc
                   for l, nc in zip(self.angular_momenta, self.contraction_counts))

    @property
    def nshell(self) -> int:
        return len(self.angular_momenta)


@dataclass(frozen=True)
class BasisParameters:
    """Raw basis values: coordinates in Bohr, exponents in Bohr^-2."""
    exponents: tuple
    coefficients: tuple
    centers: np.ndarray          # (nshell, 3)
    nuclear_coords: np.ndarray   # (natom, 3)

    def with_coordinates(self, nuclear_coords, shell_atoms):
        """Same basis, nuclei moved; shell centres follow their atoms."""
        nuclear_coords = np.asarray(nuclear_coords, dtype=np.float64)
        return BasisParameters(self.exponents, self.coefficients,
                               nuclear_coords[np.asarray(shell_atoms)], nuclear_coords)


def prepare_basis(atom, basis, *, unit="Angstrom", cart=True):
    """Parse a molecule and a named/explicit basis into topology + parameters.

    Returns ``(topology, parameters, shell_atoms)`` -- ``shell_atoms[s]`` is the
    nucleus shell ``s`` sits on (the reference keeps this implicit in the centre
    coordinates; forces need it to fold centre gradients onto nuclei).
    """
    mol = parse_molecule(atom, unit=unit)
    ls, nprim, nctr, exps, coefs, centers, shell_atoms = [], [], [], [], [], [], []
    for i, symbol in enumerate(mol.symbols):
        value = basis[symbol] if isinstance(basis, dict) else basis
        blocks = load_basis(value, symbol) if isinstance(value, str) else value
        for block in blocks:
            l, rows = int(block[0]), block[1:]
            if not rows or not isinstance(rows[0], (list, tuple)):
                raise ValueError("Expected nonrelativistic [l, [exponent, coefficients...], ...] shells.")
            data = np.asarray(rows, dtype=np.float64)
            if data.ndim != 2 or data.shape[1] < 2:
                raise ValueError("Each primitive requires an exponent and contraction coefficients.")
            ls.append(l)
            nprim.append(data.shape[0])
            nctr.append(data.shape[1] - 1)
            exps.append(data[:, 0].copy())
            coefs.append(data[:, 1:].copy())
            centers.append(mol.coords_bohr[i])
            shell_atoms.append(i)
    topology = BasisTopology(tuple(ls), tuple(nprim), tuple(nctr),
                             tuple(int(z) for z in mol.charges), bool(cart))
    parameters = BasisParameters(tuple(exps), tuple(coefs), np.asarray(centers).reshape(-1, 3),
                                 mol.coords_bohr.copy())
    return topology, parameters, np.asarray(shell_atoms, dtype=np.int64)


def radial_primitive_norm(l, exponents):
    a = np.asarray(exponents, dtype=np.float64)
    n = l + 1.5
    return 1.0 / np.sqrt(math.gamma(n) / (2.0 * (2.0 * a) ** n))


def normalized_shell_coefficients(l, exponents, coefficients):
    """Raw (nprim, nctr) coefficients -> normalised libcint env values."""
    a = np.asarray(exponents, dtype=np.float64)
    c = np.asarray(coefficients, dtype=np.float64)
    weighted = c * radial_primitive_norm(l, a)[:, None]
    metric = math.gamma(l + 1.5) / (2.0 * (a[:, None] + a[None, :]) ** (l + 1.5))
    norm2 = np.einsum("pi,pq,qi->i", weighted, metric, weighted)
    return weighted / np.sqrt(norm2)[None, :]


def build_tables(topology: BasisTopology):
    """ATM/BAS int32 tables and the env size (packing.py:78-95)."""
    nnuc = len(topology.nuclear_charges)
    nsh = len(topology.angular_momenta)
    atm = np.zeros((nnuc + nsh, ATM_SLOTS), dtype=np.int32)
    atm[:nnuc, 0] = topology.nuclear_charges
    atm[:, 2] = 1
    atm[:, 1] = PTR_ENV_START + np.arange(nnuc + nsh) * 3
    offset = PTR_ENV_START + 3 * (nnuc + nsh)
    bas = np.zeros((nsh, BAS_SLOTS), dtype=np.int32)
    for i, (l, np_, nc) in enumerate(zip(topology.angular_momenta, topology.primitive_counts,
                                          topology.contraction_counts)):
        bas[i, :4] = (nnuc + i, l, np_, nc)
        bas[i, 5] = offset
        bas[i, 6] = offset + np_
        offset += np_ + np_ * nc
    return atm, bas, offset


def pack(topology: BasisTopology, parameters: BasisParameters):
    """ATM/BAS/ENV with the current coordinates and normalised coefficients."""
    atm, bas, env_size = build_tables(topology)
    env = np.zeros(env_size, dtype=np.float64)
    coords = np.concatenate([np.asarray(parameters.nuclear_coords, dtype=np.float64).reshape(-1, 3),
                             np.asarray(parameters.centers, dtype=np.float64).reshape(-1, 3)])
    for i in range(len(atm)):
        env[atm[i, 1]:atm[i, 1] + 3] = coords[i]
    for i, (l, a, c) in enumerate(zip(topology.angular_momenta, parameters.exponents,
                                      parameters.coefficients)):
        norm = normalized_shell_coefficients(l, a, c)
        env[bas[i, 5]:bas[i, 5] + a.size] = a
        env[bas[i, 6]:bas[i, 6] + norm.size] = norm.T.ravel()
    return atm, bas, env


def ao_offsets(bas, cart):
    """AO offset of every shell (tables.h:71-73), length nbas+1."""
    l = bas[:, 1].astype(np.int64)
    nc = bas[:, 3].astype(np.int64)
    dim = (l + 1) * (l + 2) // 2 if cart else 2 * l + 1
    return np.concatenate([[0], np.cumsum(nc * dim)])


def nuclear_repulsion(charges, coords):
    z = np.asarray(charges, dtype=np.float64)
    r = np.asarray(coords, dtype=np.float64)
    e = 0.0
    for i in range(len(z)):
        for j in range(i):
            e += z[i] * z[j] / np.linalg.norm(r[i] - r[j])
    return e


def nuclear_repulsion_gradient(charges, coords):
    z = np.asarray(charges, dtype=np.float64)
    r = np.asarray(coords, dtype=np.float64)
    g = np.zeros_like(r)
    for i in range(len(z)):
        for j in range(len(z)):
            if i != j:
                d = r[i] - r[j]
                g[i] -= z[i] * z[j] * d / np.linalg.norm(d) ** 3
    return g
