"""ctypes driver of the C++ restatement (``oracle/cpu_ref.cpp``).

TEST INFRASTRUCTURE -- the checker, never the product.  The numpy oracle
(``oracle/port.py``) holds its catalog as Python lists and its sector blocks as
scipy CSR matrices, which does not scale to the 48-site checkerboard
(377,348,994 states, 15.7M orbits per sector).  This module runs the same
steps in OpenMP C++ on the host cores: the catalog (reference's two-pass
sweep with exact colex rank for any N <= 63), the sector filter and the
on-the-fly sector apply, plus a seeded ARPACK solve over that apply.  It is
pinned to ``oracle/port.py`` (which is pinned to the reference engine) by
``tests/test_oracle_cpp.py``.

The shared object is built by :func:`build` (``g++ -O3 -fopenmp``) into
``oracle/_build/`` (git-ignored; it travels with the working tree).
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_ref.cpp")
LIB = os.path.join(HERE, "_build", "librsed_cpu.so")
_lib = None


def build(force: bool = False) -> str:
    if not force and os.path.isfile(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    tmp = LIB + ".tmp"
    subprocess.run(["g++", "-O3", "-march=x86-64-v2", "-std=c++17", "-fopenmp", "-shared", "-fPIC", SRC, "-o", tmp],
                   check=True)
    os.replace(tmp, LIB)
    return LIB


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(build())
        P, I, I64, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
        L.rsedcpu_count_orbits.restype = I64
        L.rsedcpu_count_orbits.argtypes = [I, I, I, P, P, I]
        L.rsedcpu_catalog.argtypes = [I, I, I, P, P, I, P, P, P, P, P, P, I]
        L.rsedcpu_members.argtypes = [I, I, P, P, I, I64, P, P, I, P, D, P, I]
        L.rsedcpu_apply.argtypes = [I, I, I, I, P, P, P, P, P, I64, P, P, P, I, P, P, P, I, P, P, P, P, P, I]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def threads() -> int:
    return os.cpu_count() or 1


def catalog(n: int, k: int, perm0: np.ndarray, eta: np.ndarray, fermion: bool, nthreads: int = 0) -> dict:
    """Orbit catalog over all C(n, k) states: reprs, stab_mask, rep_rank,
    rep_sym (int32) and rep_amp (complex64), as in ``port.catalog``."""
    L = lib()
    ng = perm0.shape[0]
    perm = np.ascontiguousarray(perm0, dtype=np.uint8)
    angle = np.ascontiguousarray(np.angle(eta), dtype=np.float64)
    C = math.comb(n, k)
    nblk = (C + 65535) // 65536
    counts = np.zeros(nblk, dtype=np.int64)
    n_orb = L.rsedcpu_count_orbits(n, k, ng, _p(perm), _p(counts), nthreads or threads())
    reprs = np.zeros(n_orb, dtype=np.uint64)
    stab = np.zeros(n_orb, dtype=np.uint64)
    rep_rank = np.full(C, -1, dtype=np.int32)
    rep_sym = np.zeros(C, dtype=np.int32)
    rep_amp = np.zeros(C, dtype=np.complex64)
    L.rsedcpu_catalog(n, k, ng, _p(perm), _p(angle), int(fermion), _p(counts), _p(reprs), _p(stab), _p(rep_rank),
                      _p(rep_sym), _p(rep_amp), nthreads or threads())
    return dict(n=n, k=k, ng=ng, perm=perm, angle=angle, fermion=bool(fermion), reprs=reprs, stab_mask=stab,
                rep_rank=rep_rank, rep_sym=rep_sym, rep_amp=rep_amp)


def members(cat: dict, chi: np.ndarray, atol: float = 1e-12, nthreads: int = 0) -> np.ndarray:
    """uint64 sector bitmask per orbit for the rows of ``chi [n_sec, |G|]``."""
    chi = np.ascontiguousarray(np.atleast_2d(chi), dtype=np.complex128)
    out = np.zeros(len(cat["reprs"]), dtype=np.uint64)
    lib().rsedcpu_members(cat["n"], cat["ng"], _p(cat["perm"]), _p(cat["angle"]), int(cat["fermion"]),
                          len(cat["reprs"]), _p(cat["reprs"]), _p(cat["stab_mask"]), chi.shape[0], _p(chi),
                          float(atol), _p(out), nthreads or threads())
    return out


class SectorOperator:
    """``y = H^dagger x`` over the compact rows of one sector (the device
    kernel's pull form; ``H x`` for Hermitian blocks)."""

    def __init__(self, cat: dict, chi: np.ndarray, bilinear, density, nthreads: int = 0):
        self.cat = cat
        self.chi = np.ascontiguousarray(chi, dtype=np.complex128)
        mem = members(cat, self.chi[None, :], nthreads=nthreads)
        self.orbit_of_row = np.nonzero(mem & np.uint64(1))[0].astype(np.int32)
        self.row_of_orbit = np.full(len(cat["reprs"]), -1, dtype=np.int32)
        self.row_of_orbit[self.orbit_of_row] = np.arange(len(self.orbit_of_row), dtype=np.int32)
        self.n = len(self.orbit_of_row)
        self.ti = np.array([int(i) - 1 for (i, _, _) in bilinear], dtype=np.int32)
        self.tj = np.array([int(j) - 1 for (_, j, _) in bilinear], dtype=np.int32)
        self.tt = np.array([complex(t) for (_, _, t) in bilinear], dtype=np.complex128)
        self.di = np.array([int(i) - 1 for (i, _, _) in density] or [0], dtype=np.int32)
        self.dj = np.array([int(j) - 1 for (_, j, _) in density] or [0], dtype=np.int32)
        self.dv = np.array([complex(v) for (_, _, v) in density] or [0j], dtype=np.complex128)
        self.nd = len(density)
        self.nthreads = nthreads or threads()
        self.calls = 0

    def __call__(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.complex128).reshape(-1)
        y = np.empty(self.n, dtype=np.complex128)
        c = self.cat
        lib().rsedcpu_apply(c["n"], c["k"], c["ng"], int(c["fermion"]), _p(c["rep_rank"]), _p(c["rep_sym"]),
                            _p(c["rep_amp"]), _p(c["reprs"]), _p(c["stab_mask"]), self.n, _p(self.orbit_of_row),
                            _p(self.row_of_orbit), _p(self.chi), len(self.tt), _p(self.ti), _p(self.tj),
                            _p(self.tt), self.nd, _p(self.di), _p(self.dj), _p(self.dv), _p(x), _p(y),
                            self.nthreads)
        self.calls += 1
        return y


def solve(op: SectorOperator, nev: int, tol: float = 1e-10):
    """Lowest ``nev`` eigenvalues: ARPACK ``eigs(which="SR")`` with the
    reference's seeded ``v0`` (``symmetry_resolved_ed.py:2285-2299``)."""
    import scipy.sparse.linalg as spla

    n = op.n
    rng = np.random.default_rng(12345)
    v0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    v0 /= np.linalg.norm(v0)
    lin = spla.LinearOperator((n, n), matvec=op, dtype=np.complex128)
    vals, vecs = spla.eigs(lin, k=nev, which="SR", v0=v0, tol=tol)
    order = np.argsort(vals.real)
    return vals.real[order], vecs[:, order]
