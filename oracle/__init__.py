"""CPU ORACLE -- test infrastructure only.

ctypes bindings to oracle/_ref/libjk_oracle.so (the C restatement of the
reference's direct J/K driver in oracle/jk_oracle.c, linked against the
reference's vendored libcint compiled from source by oracle/Makefile), plus
numpy helpers built on them (full-ERI einsum J/K, RHF energy and gradient).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package, and only as the checker.  The product (gradscf_b200)
never imports it.
"""
from __future__ import annotations

import ctypes
from functools import lru_cache
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_ref" / "libjk_oracle.so"


class OracleError(RuntimeError):
    pass


@lru_cache(maxsize=1)
def lib():
    if not LIB_PATH.is_file():
        raise OracleError(f"oracle library missing: {LIB_PATH} (run `make -C oracle`)")
    h = ctypes.CDLL(str(LIB_PATH))
    h.oracle_last_error.restype = ctypes.c_char_p
    h.oracle_count_quartets.restype = ctypes.c_longlong
    return h


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(rc):
    if rc != 0:
        raise OracleError(lib().oracle_last_error().decode())


def _n(bas, cart):
    l = bas[:, 1].astype(np.int64)
    nc = bas[:, 3].astype(np.int64)
    return int(np.sum(nc * (((l + 1) * (l + 2) // 2) if cart else (2 * l + 1))))


def direct_jk(atm, bas, env, density, *, cart, cutoff=0.0, workers=1, with_j=True,
              with_k=True, return_calls=False):
    """The reference's GradSCFDirectJK restated in C: returns (J, K)."""
    atm, bas, env = _i32(atm), _i32(bas), _f64(env)
    d = _f64(density)
    shape = d.shape
    n = shape[-1]
    d = d.reshape(-1, n, n)
    nb = d.shape[0]
    nops = int(with_j) + int(with_k)
    out = np.zeros((nops, nb, n, n))
    calls = ctypes.c_longlong(0)
    _check(lib().oracle_direct_jk(_p(atm), len(atm), _p(bas), len(bas), _p(env), len(env), _p(d),
                                  nb, n, _p(out), int(cart), ctypes.c_double(cutoff), int(workers),
                                  int(with_j), int(with_k), ctypes.byref(calls)))
    j = out[0].reshape(shape) if with_j else np.zeros(shape)
    k = out[-1].reshape(shape) if with_k else np.zeros(shape)
    return (j, k, calls.value) if return_calls else (j, k)


def eri_s1(atm, bas, env, *, cart):
    atm, bas, env = _i32(atm), _i32(bas), _f64(env)
    n = _n(bas, cart)
    out = np.zeros((n, n, n, n))
    _check(lib().oracle_eri_s1(_p(atm), len(atm), _p(bas), len(bas), _p(env), len(env), int(cart),
                               _p(out)))
    return out


def eri_block(atm, bas, env, shls, *, cart):
    """libcint block for one shell quartet, returned as [p, q, r, s]."""
    atm, bas, env = _i32(atm), _i32(bas), _f64(env)
    dims = []
    for s in shls:
        l, nc = int(bas[s, 1]), int(bas[s, 3])
        dims.append(nc * (((l + 1) * (l + 2) // 2) if cart else (2 * l + 1)))
    out = np.zeros(int(np.prod(dims)))
    sh = _i32(shls)
    _check(lib().oracle_eri_block(_p(atm), len(atm), _p(bas), len(bas), _p(env), len(env),
                                  int(cart), _p(sh), _p(out)))
    return out.reshape(dims[::-1]).transpose(3, 2, 1, 0)


def full_jk(eri, density):
    """The reference tests' einsum oracle (test_native_direct_parallel.py:45-50)."""
    return (np.einsum("pqrs,...rs->...pq", eri, density),
            np.einsum("prqs,...rs->...pq", eri, density))


def int1e(atm, bas, env, which, *, cart):
    """which: 'ovlp' | 'kin' | 'nuc'."""
    atm, bas, env = _i32(atm), _i32(bas), _f64(env)
    n = _n(bas, cart)
    out = np.zeros((n, n))
    _check(lib().oracle_int1e(_p(atm), len(atm), _p(bas), len(bas), _p(env), len(env), int(cart),
                              {"ovlp": 0, "kin": 1, "nuc": 2}[which], _p(out)))
    return out


def int1e_ip(atm, bas, env, which, *, cart, atom=0):
    """which: 'ipovlp' | 'ipkin' | 'ipnuc' | 'iprinv' (about `atom`); shape (3, n, n)."""
    atm, bas, env = _i32(atm), _i32(bas), _f64(env)
    n = _n(bas, cart)
    out = np.zeros((3, n, n))
    _check(lib().oracle_int1e_ip(_p(atm), len(atm), _p(bas), len(bas), _p(env), len(env),
                                 int(cart), {"ipovlp": 0, "ipkin": 1, "ipnuc": 2, "iprinv": 3}[which],
                                 int(atom), _p(out)))
    return out


def schwarz_bounds(atm, bas, env, *, cart):
    atm, bas, env = _i32(atm), _i32(bas), _f64(env)
    out = np.zeros((len(bas), len(bas)))
    _check(lib().oracle_schwarz_bounds(_p(atm), len(atm), _p(bas), len(bas), _p(env), len(env),
                                       int(cart), _p(out)))
    return out


def count_quartets(bounds, cut):
    b = _f64(bounds)
    return int(lib().oracle_count_quartets(_p(b), b.shape[0], ctypes.c_double(cut)))


def direct_jk_geometry_vjp(atm, bas, env, density, cotangent, *, cart, with_j=True, with_k=True,
                           workers=1):
    """Reference gradscf_direct_jk_geometry_vjp_cpu_v2: env-sized gradient."""
    atm, bas, env = _i32(atm), _i32(bas), _f64(env)
    d = _f64(density)
    n = d.shape[-1]
    d = d.reshape(-1, n, n)
    v = _f64(cotangent)
    out = np.zeros(len(env))
    _check(lib().oracle_direct_jk_geometry_vjp(_p(atm), len(atm), _p(bas), len(bas), _p(env),
                                               len(env), _p(d), d.shape[0], n, _p(v), _p(out),
                                               int(cart), int(with_j), int(with_k), int(workers)))
    return out


def direct_jk_geometry_product(atm, bas, env, density, direction, vector=None, *, order, cart,
                               transpose=False, with_j=True, with_k=True, workers=1):
    """The reference's geometry products of J/K (csrc/direct_jk_geometry.cc:8-99).

    transpose=False (JVP): returns (J', K') with J' = d/du J (order 1) or
    d^2/(du dv) J (order 2, ``vector`` = v, env-sized), same for K.
    transpose=True (order 2 only): returns the env-sized coordinate gradient of
    sum(Jbar * dJ/du + Kbar * dK/du), ``vector`` = (Jbar, Kbar) cotangents of
    shape (with_j + with_k, nb, n, n)."""
    atm, bas, env = _i32(atm), _i32(bas), _f64(env)
    d = _f64(density)
    shape = d.shape
    n = shape[-1]
    d = d.reshape(-1, n, n)
    nb = d.shape[0]
    u = _f64(direction)
    nops = int(with_j) + int(with_k)
    if transpose:
        v = _f64(vector)
        out = np.zeros(len(env))
    else:
        v = _f64(vector) if vector is not None else np.zeros(len(env))
        out = np.zeros((nops, nb, n, n))
    _check(lib().oracle_direct_jk_geometry_product(
        _p(atm), len(atm), _p(bas), len(bas), _p(env), len(env), _p(d), nb, n, _p(u), _p(v), _p(out),
        int(order), int(bool(transpose)), int(cart), int(with_j), int(with_k), int(workers)))
    if transpose:
        return out
    j = out[0].reshape(shape) if with_j else np.zeros(shape)
    k = out[-1].reshape(shape) if with_k else np.zeros(shape)
    return j, k
