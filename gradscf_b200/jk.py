"""Direct J/K on the B200 through the C ABI, mirroring the reference's API.

Reference surface mirrored here (src/gradscf/integrals/...):
  * ``direct_jk(atm, bas, env, density, *, cart, cutoff, workers, with_j,
    with_k)`` -- backends/native/jk.py:399-446: (..., n, n) float64 or
    complex128 densities, complex split into real/imag batches, returns (J, K)
    with zeros for an operator that was not requested.
  * ``IntegralPlan.get_jk`` -- plan.py:71-92, ``make_plan`` -- plan.py:185-190.
  * ``NativeDirectBasis.get_jk`` -- backends/native/jk.py:98-107.
Arrays are torch tensors on a CUDA device (numpy inputs are moved there).
"""
from __future__ import annotations

import ctypes
from collections import OrderedDict
from dataclasses import dataclass
from numbers import Integral

import numpy as np
import torch

from . import _capi
from .basis import BasisParameters, BasisTopology, build_tables, pack

PRECISIONS = {"fp64": _capi.FP64, "split": _capi.SPLIT}
DEFAULT_FP32_CUT = 1e-6


def allreduce_partial(out, group=None):
    """Sum the ranks' partial J/K (or gradient) in place: one all-reduce
    over `group` (NCCL for CUDA tensors, gloo for CPU tensors)."""
    import torch.distributed as dist
    dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out


def _stream_handle(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


class DirectJKPlan:
    """Device-resident plan (``b200jk_plan_create``) for one molecule or a batch.

    ``molecules`` is a sequence of (atm, bas, env) libcint tables.  Densities
    and results use the packed layout: molecule m occupies
    ``[offsets[m], offsets[m] + nao[m]**2)`` of every matrix.
    """

    def __init__(self, molecules, *, cart, cutoff=0.0, device=None):
        lib = _capi.lib()
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        if dev.type != "cuda":
            raise ValueError("DirectJKPlan needs a CUDA device")
        self.device = dev
        self.cart = bool(cart)
        self.cutoff = float(cutoff)
        keep = []
        arr = (_capi.Molecule * len(molecules))()
        for i, (atm, bas, env) in enumerate(molecules):
            a = np.ascontiguousarray(atm, dtype=np.int32)
            b = np.ascontiguousarray(bas, dtype=np.int32)
            e = np.ascontiguousarray(env, dtype=np.float64)
            keep += [a, b, e]
            arr[i] = _capi.Molecule(a.ctypes.data, a.shape[0], b.ctypes.data, b.shape[0],
                                    e.ctypes.data, e.shape[0])
        self.natm = [int(np.asarray(m[0]).shape[0]) for m in molecules]
        handle = ctypes.c_void_p()
        with torch.cuda.device(dev):
            _capi.check(lib.b200jk_plan_create(arr, len(molecules), int(cart), float(cutoff),
                                               dev.index or 0, ctypes.byref(handle)))
        self._h = handle
        self.nmol = len(molecules)
        n = ctypes.c_int32()
        self.nao = []
        for m in range(self.nmol):
            _capi.check(lib.b200jk_plan_nao(self._h, m, ctypes.byref(n)))
            self.nao.append(n.value)
        offs = (ctypes.c_int64 * self.nmol)()
        _capi.check(lib.b200jk_plan_block_offsets(self._h, offs))
        self.offsets = list(offs)
        self.packed_size = self.offsets[-1] + self.nao[-1] ** 2
        q = ctypes.c_int64()
        _capi.check(lib.b200jk_plan_quartets(self._h, ctypes.byref(q)))
        self.quartets = q.value
        self.shard = (0, 1)
        self.group = None

    def set_shard(self, rank, world, group=None):
        """Evaluate only shard `rank` of `world` (contiguous cost-balanced
        blocks of every class pair's work items; ``b200jk_plan_set_shard``).
        Results of ``jk_packed`` / ``JKGraph.run`` are then summed over the
        ranks of `group` (one ``torch.distributed`` all-reduce, NCCL on GPUs)
        unless ``reduce=False`` is passed; ``(0, 1)`` restores the whole build."""
        with torch.cuda.device(self.device):
            _capi.check(_capi.lib().b200jk_plan_set_shard(self._h, int(rank), int(world)))
        self.shard = (int(rank), int(world))
        self.group = group

    def autotune(self, density, *, hermi=1, precision="split", fp32_cut=DEFAULT_FP32_CUT, reps=3, stream=None):
        """Pick each register-path class pair's kets per work item (32, 64 or
        128) by timing its kernels on `density` ((nb, packed_size), e.g. an SCF
        iteration's dD); ``b200jk_plan_autotune``.  Returns {class: kets}.
        Tune after ``set_shard`` and before creating a ``JKGraph``."""
        d = density.reshape(-1, self.packed_size).contiguous()
        if d.dtype != torch.float64 or d.device != self.device:
            raise ValueError("density must be float64 on the plan's device")
        chunks = (ctypes.c_int32 * _capi.NCLASS)()
        with torch.cuda.device(self.device):
            _capi.check(_capi.lib().b200jk_plan_autotune(
                self._h, ctypes.c_void_p(d.data_ptr()), d.shape[0], int(bool(hermi)), PRECISIONS[precision],
                float(fp32_cut), int(reps), _stream_handle(stream), chunks))
        return {"({}{}|{}{})".format(*_capi.QUARTET_CLASSES[c]): chunks[c]
                for c in range(_capi.NCLASS) if chunks[c] > 0}

    def reduce_shards(self, out):
        """Sum a sharded result over the ranks (in place); no-op when unsharded."""
        if self.shard[1] > 1:
            allreduce_partial(out, self.group)
        return out

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().b200jk_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- J/K ---------------------------------------------------------------
    def jk_packed(self, density, *, with_j=True, with_k=True, hermi=0, precision="fp64",
                  fp32_cut=DEFAULT_FP32_CUT, out=None, stream=None, check=True, reduce=True):
        """density: (nb, packed_size) float64 CUDA tensor -> (nops, nb, packed_size).
        On a sharded plan the partial results are all-reduced when `reduce`."""
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        d = density
        if d.dtype != torch.float64 or d.device != self.device or d.dim() != 2 or d.shape[1] != self.packed_size:
            raise ValueError("density must be a float64 (nb, packed_size) tensor on the plan's device")
        d = d.contiguous()
        nb = d.shape[0]
        nops = int(bool(with_j)) + int(bool(with_k))
        if out is None:
            out = torch.empty((nops, nb, self.packed_size), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            st = _stream_handle(stream)
            _capi.check(_capi.lib().b200jk_direct_jk(
                self._h, ctypes.c_void_p(d.data_ptr()), nb, ctypes.c_void_p(out.data_ptr()),
                int(bool(with_j)), int(bool(with_k)), int(bool(hermi)), PRECISIONS[precision],
                float(fp32_cut), st))
            if check:
                _capi.check(_capi.lib().b200jk_check_status(self._h, st))
        if reduce:
            self.reduce_shards(out)
        return out

    def jk(self, density, *, with_j=True, with_k=True, hermi=None, precision="fp64",
           fp32_cut=DEFAULT_FP32_CUT, stream=None):
        """Single-molecule convenience: (..., n, n) -> (J, K) of the same shape."""
        if self.nmol != 1:
            raise ValueError("jk() is for one-molecule plans; use jk_packed for batches")
        n = self.nao[0]
        d = torch.as_tensor(density, dtype=torch.float64, device=self.device)
        shape = d.shape
        if shape[-2:] != (n, n):
            raise ValueError("Density AO dimensions do not match the plan.")
        flat = d.reshape(-1, n * n)
        if hermi is None:
            hermi = bool(torch.equal(d, d.transpose(-1, -2)))
        out = self.jk_packed(flat, with_j=with_j, with_k=with_k, hermi=hermi, precision=precision,
                             fp32_cut=fp32_cut, stream=stream)
        j = out[0].reshape(shape) if with_j else torch.zeros_like(d)
        k = out[-1].reshape(shape) if with_k else torch.zeros_like(d)
        return j, k


class JKGraph:
    """A captured J/K build (``b200jk_graph_create``) on fixed buffers.

    ``run(density)`` copies the (nb, packed_size) density into the graph's
    input buffer and replays the captured build; the result lands in
    ``self.out`` (nops, nb, packed_size).
    """

    def __init__(self, plan: DirectJKPlan, nb=1, *, with_j=True, with_k=True, hermi=1,
                 precision="fp64", fp32_cut=DEFAULT_FP32_CUT):
        self.plan = plan
        nops = int(bool(with_j)) + int(bool(with_k))
        self.inp = torch.zeros((nb, plan.packed_size), dtype=torch.float64, device=plan.device)
        self.out = torch.zeros((nops, nb, plan.packed_size), dtype=torch.float64, device=plan.device)
        h = ctypes.c_void_p()
        with torch.cuda.device(plan.device):
            _capi.check(_capi.lib().b200jk_graph_create(
                plan._h, ctypes.c_void_p(self.inp.data_ptr()), nb, ctypes.c_void_p(self.out.data_ptr()),
                int(bool(with_j)), int(bool(with_k)), int(bool(hermi)), PRECISIONS[precision],
                float(fp32_cut), ctypes.byref(h)))
        self._h = h

    def run(self, density, stream=None, reduce=True):
        self.inp.copy_(density.reshape(self.inp.shape))
        return self.launch(stream, reduce)

    def launch(self, stream=None, reduce=True):
        """Replay on the current contents of ``self.inp``."""
        with torch.cuda.device(self.plan.device):
            _capi.check(_capi.lib().b200jk_graph_launch(self._h, _stream_handle(stream)))
        if reduce:
            self.plan.reduce_shards(self.out)
        return self.out

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().b200jk_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_PLAN_CACHE: "OrderedDict[tuple, DirectJKPlan]" = OrderedDict()


def cached_plan(atm, bas, env, *, cart, cutoff, device=None):
    """Plans keyed by table contents (coordinates included), LRU of 8."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    a = np.ascontiguousarray(atm, dtype=np.int32)
    b = np.ascontiguousarray(bas, dtype=np.int32)
    e = np.ascontiguousarray(env, dtype=np.float64)
    key = (a.tobytes(), b.tobytes(), e.tobytes(), bool(cart), float(cutoff), str(dev))
    plan = _PLAN_CACHE.get(key)
    if plan is None:
        plan = DirectJKPlan([(a, b, e)], cart=cart, cutoff=cutoff, device=dev)
        _PLAN_CACHE[key] = plan
        while len(_PLAN_CACHE) > 8:
            _PLAN_CACHE.popitem(last=False)
    else:
        _PLAN_CACHE.move_to_end(key)
    return plan


def direct_jk(atm, bas, env, density, *, cart, cutoff=0.0, workers=1, with_j=True, with_k=True,
              precision="fp64", fp32_cut=DEFAULT_FP32_CUT, device=None):
    """Contract J/K (backends/native/jk.py:399-446) on the GPU; returns (J, K)."""
    if not all(isinstance(f, (bool, np.bool_)) for f in (with_j, with_k)):
        raise ValueError("with_j and with_k must be static booleans.")
    if isinstance(workers, bool) or not isinstance(workers, Integral) or workers < 1:
        raise ValueError("workers must be a positive integer.")
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    d = torch.as_tensor(density, device=dev)
    n = d.shape[-1]
    if d.dim() < 2 or d.shape[-2:] != (n, n) or d.dtype not in (torch.float64, torch.complex128):
        raise ValueError("Direct J/K requires (...,n,n) float64/complex128 density.")
    if np.asarray(env).dtype != np.float64:
        raise ValueError("Direct J/K requires float64 environment.")
    if not (with_j or with_k):
        return torch.zeros_like(d), torch.zeros_like(d)
    plan = cached_plan(atm, bas, env, cart=cart, cutoff=cutoff, device=dev)
    if plan.nao[0] != n:
        raise ValueError("Direct J/K shape mismatch")
    flat = d.reshape(-1, n, n)
    count = flat.shape[0]
    real = torch.cat((flat.real, flat.imag), 0) if d.is_complex() else flat
    hermi = bool(torch.equal(real, real.transpose(-1, -2)))
    out = plan.jk_packed(real.reshape(real.shape[0], n * n).contiguous(), with_j=bool(with_j),
                         with_k=bool(with_k), hermi=hermi, precision=precision, fp32_cut=fp32_cut)
    out = out.reshape(out.shape[0], -1, n, n)
    if d.is_complex():
        out = torch.complex(out[:, :count], out[:, count:])
    out = out.reshape(int(with_j) + int(with_k), *d.shape)
    return (out[0] if with_j else torch.zeros_like(d), out[-1] if with_k else torch.zeros_like(d))


def _coordinate_rows(atm, vector, dev):
    """env-sized coordinate direction -> (natm, 3) rows per atm row.  Only the
    coordinate slots may be nonzero (csrc/direct_jk_geometry.cc:35-48)."""
    v = np.asarray(vector, dtype=np.float64)
    if v.ndim != 1:
        raise ValueError("Direct J/K geometry direction shape mismatch")
    if not np.all(np.isfinite(v)):
        raise ValueError("Direct J/K geometry input must be finite")
    a = np.asarray(atm)
    slots = (a[:, 1].astype(np.int64)[:, None] + np.arange(3)[None, :])
    allowed = np.zeros(v.shape[0], dtype=bool)
    allowed[slots.ravel()] = True
    if np.any(v[~allowed] != 0.0):
        raise ValueError("Direct J/K geometry supports coordinates only, not basis exponents/coefficients")
    return torch.as_tensor(v[slots], device=dev).contiguous(), slots


def _geometry_setup(atm, bas, env, density, cart, cutoff, with_j, with_k, dev):
    if not (with_j or with_k):
        raise ValueError("Invalid direct J/K geometry product")
    dev = torch.device("cuda", torch.cuda.current_device()) if dev is None else torch.device(dev)
    d = torch.as_tensor(density, dtype=torch.float64, device=dev)
    n = d.shape[-1]
    if d.dim() < 2 or d.shape[-2:] != (n, n) or not torch.isfinite(d).all():
        raise ValueError("Direct J/K geometry input must be finite (..., n, n) float64")
    plan = cached_plan(atm, bas, env, cart=cart, cutoff=cutoff, device=dev)
    if plan.nao[0] != n:
        raise ValueError("Direct J/K geometry density shape mismatch")
    return plan, d, n, dev


def direct_jk_geometry_jvp(atm, bas, env, density, direction, vector=None, *, cart, cutoff=0.0,
                           with_j=True, with_k=True, device=None):
    """Coordinate JVP of J/K at fixed density (the reference's
    gradscf_direct_jk_geometry_jvp_cpu_v1, csrc/direct_jk_geometry.cc:8-99):
    order 1, d/du (J, K), when ``vector`` is None; order 2, d^2/(du dv) (J, K),
    with ``vector`` = v.  ``direction`` / ``vector`` are env-sized, nonzero only
    at atm coordinate slots.  ``b200jk_direct_jk_geom_jvp``."""
    plan, d, n, dev = _geometry_setup(atm, bas, env, density, cart, cutoff, with_j, with_k, device)
    u, _ = _coordinate_rows(atm, direction, dev)
    v = _coordinate_rows(atm, vector, dev)[0] if vector is not None else None
    flat = d.reshape(-1, n * n).contiguous()
    nb = flat.shape[0]
    nops = int(bool(with_j)) + int(bool(with_k))
    out = torch.empty((nops, nb, n * n), dtype=torch.float64, device=dev)
    hermi = bool(torch.equal(flat.reshape(nb, n, n), flat.reshape(nb, n, n).transpose(-1, -2)))
    with torch.cuda.device(dev):
        st = _stream_handle()
        _capi.check(_capi.lib().b200jk_direct_jk_geom_jvp(
            plan._h, ctypes.c_void_p(flat.data_ptr()), nb, int(hermi), ctypes.c_void_p(u.data_ptr()),
            ctypes.c_void_p(v.data_ptr()) if v is not None else None, int(bool(with_j)), int(bool(with_k)),
            ctypes.c_void_p(out.data_ptr()), st))
    plan.reduce_shards(out)
    out = out.reshape(nops, *d.shape)
    return (out[0] if with_j else torch.zeros_like(d), out[-1] if with_k else torch.zeros_like(d))


def direct_jk_geometry_hvp(atm, bas, env, density, direction, cotangent, *, cart, cutoff=0.0,
                           with_j=True, with_k=True, device=None):
    """Order-2 coordinate VJP (the order-2 branch of the reference's
    gradscf_direct_jk_geometry_vjp_cpu_v2): the env-sized coordinate gradient
    of sum(Jbar * dJ/du + Kbar * dK/du), ``cotangent`` = (Jbar, Kbar) each
    shaped like the density.  ``b200jk_direct_jk_geom_hvp``."""
    plan, d, n, dev = _geometry_setup(atm, bas, env, density, cart, cutoff, with_j, with_k, device)
    u, slots = _coordinate_rows(atm, direction, dev)
    flat = d.reshape(-1, n * n).contiguous()
    nb = flat.shape[0]
    parts = []
    jbar, kbar = cotangent
    if with_j:
        parts.append(torch.as_tensor(jbar, dtype=torch.float64, device=dev).reshape(nb, n * n))
    if with_k:
        parts.append(torch.as_tensor(kbar, dtype=torch.float64, device=dev).reshape(nb, n * n))
    cot = torch.stack(parts).contiguous()
    g = torch.empty((plan.natm[0], 3), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        st = _stream_handle()
        _capi.check(_capi.lib().b200jk_direct_jk_geom_hvp(
            plan._h, ctypes.c_void_p(flat.data_ptr()), nb, ctypes.c_void_p(u.data_ptr()),
            ctypes.c_void_p(cot.data_ptr()), int(bool(with_j)), int(bool(with_k)),
            ctypes.c_void_p(g.data_ptr()), st))
    plan.reduce_shards(g)
    out = np.zeros(np.asarray(env).shape[0])
    np.add.at(out, slots.ravel(), g.cpu().numpy().ravel())
    return out


@dataclass(frozen=True)
class IntegralPlan:
    """Static topology + table layout (plan.py:50-92)."""
    topology: BasisTopology
    atm: np.ndarray
    bas: np.ndarray
    env_size: int

    def pack(self, parameters: BasisParameters):
        return pack(self.topology, parameters)

    def get_jk(self, parameters, density, *, screening_threshold=0.0, workers=1, with_j=True,
               with_k=True, omega=0.0, precision="fp64", fp32_cut=DEFAULT_FP32_CUT):
        omega = validate_omega(omega)
        atm, bas, env = self.pack(parameters)
        if omega:
            env = np.array(env, dtype=np.float64, copy=True)
            env[8] = omega  # libcint PTR_RANGE_OMEGA: erf(omega r)/r (plan.py:86-87)
        d = torch.as_tensor(density)
        if d.shape[-2:] != (self.topology.nao,) * 2:
            raise ValueError("Density AO dimensions do not match the plan.")
        return direct_jk(atm, bas, env, density, cart=self.topology.cart, cutoff=screening_threshold,
                         workers=workers, with_j=with_j, with_k=with_k, precision=precision,
                         fp32_cut=fp32_cut)


def validate_omega(omega):
    """Static nonnegative erf-Coulomb range parameter in inverse Bohr (plan.py:18-27)."""
    if isinstance(omega, (bool, np.bool_)) or not isinstance(omega, (int, float, np.integer, np.floating)):
        raise TypeError("omega must be a static real scalar.")
    omega = float(omega)
    if not np.isfinite(omega) or omega < 0 or omega > np.sqrt(np.finfo(np.float64).max) / 2:
        raise ValueError("omega must be finite, nonnegative and at most sqrt(float64.max)/2.")
    return omega


def make_plan(topology: BasisTopology) -> IntegralPlan:
    atm, bas, size = build_tables(topology)
    return IntegralPlan(topology, atm, bas, size)


@dataclass(frozen=True)
class NativeDirectBasis:
    """Bound (plan, parameters) J/K provider (backends/native/jk.py:70-107)."""
    plan: IntegralPlan
    parameters: BasisParameters

    @property
    def nao(self):
        return self.plan.topology.nao

    def get_jk(self, density, *, screening_threshold=0.0, workers=1, with_j=True, with_k=True,
               omega=0.0, precision="fp64", fp32_cut=DEFAULT_FP32_CUT):
        return self.plan.get_jk(self.parameters, density, screening_threshold=screening_threshold,
                                workers=workers, with_j=with_j, with_k=with_k, omega=omega,
                                precision=precision, fp32_cut=fp32_cut)

    def prepare_jk(self, *, cache_bytes=0, screening_threshold=0.0, workers=1, with_j=True, with_k=True,
                   omega=0.0, precision="fp64", fp32_cut=DEFAULT_FP32_CUT):
        """Bind one response action: density batch -> (J, K) (backends/native/jk.py:118-162).

        On CUDA arrays the reference's prepared action is the direct J/K
        (its ``platform_dependent`` default branch); here too.  The device
        plan for these tables is built on the first call and reused by every
        later one, so batches of response densities cost one launch set each.
        `cache_bytes` is accepted for signature compatibility; no ERIs are
        stored.
        """
        omega = validate_omega(omega)

        def action(density):
            return self.get_jk(density, screening_threshold=screening_threshold, workers=workers,
                               with_j=with_j, with_k=with_k, omega=omega, precision=precision,
                               fp32_cut=fp32_cut)
        return action


def rsh_jk(provider, density, coefficients, *, with_j=True, with_k=True, screening_threshold=0.0,
           workers=1, precision="fp64", fp32_cut=DEFAULT_FP32_CUT):
    """Range-separated-hybrid J/K (scf/rsh.py:62-85): the full Coulomb J and
    K_rsh = sr * K(full) + (lr - sr) * K(omega) for coefficients
    (omega, long_range, short_range)."""
    if len(coefficients) != 3:
        raise ValueError("RSH J/K requires (omega, long_range, short_range) coefficients.")
    omega, long_range, short_range = (float(v) for v in coefficients)
    if not all(np.isfinite(v) for v in (omega, long_range, short_range)) or omega <= 0.0:
        raise ValueError("RSH J/K requires finite coefficients and positive omega.")
    d = torch.as_tensor(density)
    coulomb = exchange = torch.zeros_like(d)
    opts = dict(screening_threshold=screening_threshold, workers=workers, precision=precision, fp32_cut=fp32_cut)
    if with_j or (with_k and short_range != 0.0):
        coulomb, full_k = provider.get_jk(density, with_j=with_j, with_k=with_k and short_range != 0.0,
                                          omega=0.0, **opts)
        if with_k:
            exchange = short_range * full_k
    if with_k and long_range != short_range:
        _, long_k = provider.get_jk(density, with_j=False, with_k=True, omega=omega, **opts)
        exchange = exchange + (long_range - short_range) * long_k
    if not with_j:
        coulomb = torch.zeros_like(d)
    return coulomb, exchange


def packed_eri_shape(n, ndim):
    """Shape of s8 (ndim 1) or s4 (ndim 2) packed ERIs of n AOs (molecular/jk.py)."""
    np_ = n * (n + 1) // 2
    return (np_ * (np_ + 1) // 2,) if ndim == 1 else (np_, np_)


def packed_eri(atm, bas, env, *, cart, aosym="s8", cutoff=0.0, device=None):
    """Exact packed ERIs on the GPU (the reference's plan.evaluate("eri", aosym=...)
    through csrc/packed_eri.cc): aosym "s8" -> (np(np+1)/2,), "s4" -> (np, np)."""
    if aosym not in ("s4", "s8"):
        raise ValueError("aosym must be 's4' or 's8'")
    plan = cached_plan(atm, bas, env, cart=cart, cutoff=cutoff, device=device)
    n = plan.nao[0]
    shape = packed_eri_shape(n, 1 if aosym == "s8" else 2)
    out = torch.empty(shape, dtype=torch.float64, device=plan.device)
    with torch.cuda.device(plan.device):
        _capi.check(_capi.lib().b200jk_packed_eri(plan._h, 1 if aosym == "s8" else 0,
                                                 ctypes.c_void_p(out.data_ptr()), out.numel(),
                                                 _stream_handle()))
    return out


def packed_jk(eri, density, *, with_j=True, with_k=True):
    """J/K from s8 or s4 packed ERIs (backends/native/jk.py packed_jk,
    csrc/packed_jk.cc): (..., n, n) float64 or complex128 densities -> (J, K)."""
    if not (with_j or with_k):
        raise ValueError("Packed J/K requires at least one selected operator")
    e = torch.as_tensor(eri)
    d = torch.as_tensor(density, device=e.device)
    n = d.shape[-1]
    if e.dtype != torch.float64 or e.dim() not in (1, 2) or tuple(e.shape) != packed_eri_shape(n, e.dim()):
        raise ValueError("Packed ERI/density shapes do not match.")
    flat = d.reshape(-1, n, n)
    count = flat.shape[0]
    real = torch.cat((flat.real, flat.imag), 0) if d.is_complex() else flat
    real = real.to(torch.float64).contiguous()
    nops = int(bool(with_j)) + int(bool(with_k))
    out = torch.empty((nops, real.shape[0], n, n), dtype=torch.float64, device=e.device)
    with torch.cuda.device(e.device):
        _capi.check(_capi.lib().b200jk_packed_jk(
            ctypes.c_void_p(e.contiguous().data_ptr()), 1 if e.dim() == 1 else 0, e.numel(), n,
            ctypes.c_void_p(real.data_ptr()), real.shape[0], ctypes.c_void_p(out.data_ptr()),
            int(bool(with_j)), int(bool(with_k)), _stream_handle()))
    if d.is_complex():
        out = torch.complex(out[:, :count], out[:, count:])
    out = out.reshape(nops, *d.shape)
    return (out[0] if with_j else torch.zeros_like(d), out[-1] if with_k else torch.zeros_like(d))


def build_jk_from_packed(eri, density):
    """molecular/jk.py build_jk_from_packed: J and K from s4/s8 packed ERIs."""
    return packed_jk(eri, density)
