"""Test oracle for the mcpi hot path (ctypes + numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by ``bench.py``'s CPU-baseline and reference legs. The
product package (``mcpi_b200``) never imports it.

Two libraries are wrapped:

* ``Orc``  -- ``oracle/liborc.so``: this directory's own C restatement
  (``mcpi_oracle.c``; every function cites the reference file:line it follows).
* ``Ref``  -- ``oracle/_ref/libmcpi_ref.so``: the reference's own C sources,
  compiled unmodified (``oracle/Makefile``). Present wherever it was built;
  the reference sources themselves are only needed to build it.

Arrays follow the reference layouts: ``IF[j + k*M]``,
``Map[i + k*nc + l*M*nc]``, ``Hint[k + s*M + q*M^2 + l*M^3]`` (flat, complex),
and ``Ho[k][l]`` as a 2-D numpy array (row k, column l).
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(HERE, "liborc.so")
REF_PATH = os.path.join(HERE, "_ref", "libmcpi_ref.so")
# the reference source tree: MCPI_REFERENCE_SRC, else "reference" beside the repository
REFERENCE_SRC = os.environ.get(
    "MCPI_REFERENCE_SRC", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))

_c_int_p = ct.POINTER(ct.c_int32)
_c_i64_p = ct.POINTER(ct.c_int64)
_c_dbl_p = ct.POINTER(ct.c_double)
_vp = ct.c_void_p


def build(ref: bool = True) -> None:
    """Compile liborc.so (and _ref/libmcpi_ref.so when the reference sources exist)."""
    targets = ["liborc.so"]
    if ref and os.path.exists(os.path.join(REFERENCE_SRC, "configurationsMap.h")):
        targets.append("ref")
        if os.path.exists(os.path.join(REFERENCE_SRC, "cuda", "hamiltonianMatrix.cuh")):
            targets.append("refcuda")
        if os.path.exists(os.path.join(HERE, "..", "mcpi_b200", "libmcpi_dropin.so")):
            targets.append("dropin")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_SRC}", *targets], check=True)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_vp)


def nc_of(N: int, M: int) -> int:
    from math import comb
    return comb(N + M - 1, N) if M >= 1 and N >= 0 else 0


# ---------------------------------------------------------------------------
# input generators (plain numpy; the oracle's C versions are Orc.perf_inputs etc.)
# ---------------------------------------------------------------------------

def symmetrize_hint8(h: np.ndarray, M: int) -> np.ndarray:
    """Average a flat M^4 complex tensor over the bosonic 8-fold group
    H[k,s,q,l] = H[s,k,q,l] = H[k,s,l,q] = conj(H[q,l,k,s]).
    Index flat = k + s*M + q*M^2 + l*M^3, i.e. array axes (l, q, s, k)."""
    t = h.reshape(M, M, M, M)  # axes: l q s k
    a = t
    b = t.transpose(0, 1, 3, 2)          # swap k,s
    c = t.transpose(1, 0, 2, 3)          # swap q,l
    d = t.transpose(1, 0, 3, 2)
    four = (a + b + c + d) / 4.0
    # conj(H[q,l,k,s]) : element (k,s,q,l) <- conj of element (q,l,k,s)
    # axes of four are (l,q,s,k); element (q,l,k,s) sits at [s,k,l,q]
    herm = np.conj(four.transpose(2, 3, 0, 1))
    return ((four + herm) / 2.0).reshape(-1).copy()


def random_inputs(N: int, M: int, seed: int):
    """Seeded random state (normalised complex normal), Hermitian Ho with N(0,1)
    entries, and an N(0,1) complex Hint averaged over the 8-fold bosonic group."""
    rng = np.random.default_rng(seed)
    nc = nc_of(N, M)
    C = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    C /= np.linalg.norm(C)
    A = rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))
    Ho = (A + A.conj().T) / 2.0
    H = rng.standard_normal(M ** 4) + 1j * rng.standard_normal(M ** 4)
    return C, Ho, symmetrize_hint8(H, M)


# ---------------------------------------------------------------------------
# restatement library
# ---------------------------------------------------------------------------

class Orc:
    def __init__(self, path: str = ORC_PATH):
        if not os.path.exists(path):
            build(ref=False)
        L = ct.CDLL(path)
        self.lib = L
        L.orc_nc.restype = ct.c_int64
        L.orc_nc.argtypes = [ct.c_int, ct.c_int]
        L.orc_ncmat.argtypes = [ct.c_int, ct.c_int, _vp]
        L.orc_index_to_fock.argtypes = [ct.c_int64, ct.c_int, ct.c_int, _vp]
        L.orc_fock_to_index.restype = ct.c_int64
        L.orc_fock_to_index.argtypes = [ct.c_int, ct.c_int, _vp]
        L.orc_setup_focks.argtypes = [ct.c_int, ct.c_int, _vp, ct.c_int]
        L.orc_one_one_map.argtypes = [ct.c_int, ct.c_int, _vp, _vp, ct.c_int]
        for f in (L.orc_one_two_strides, L.orc_two_two_strides):
            f.restype = ct.c_int64
            f.argtypes = [ct.c_int, ct.c_int, _vp, _vp]
        for f in (L.orc_one_two_map, L.orc_two_two_map):
            f.argtypes = [ct.c_int, ct.c_int, _vp, _vp, _vp, ct.c_int]
        L.orc_apply_h.argtypes = [ct.c_int, ct.c_int, ct.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                  _vp, _vp, _vp, _vp, ct.c_int64, ct.c_int64, ct.c_int]
        L.orc_obrho.argtypes = [ct.c_int, ct.c_int, _vp, _vp, _vp, _vp]
        L.orc_density_generic.argtypes = [ct.c_int, ct.c_int, ct.c_int, _vp, _vp, _vp]
        L.orc_density_rows.argtypes = [ct.c_int, ct.c_int, ct.c_int, _vp, _vp, _vp, ct.c_int64,
                                       ct.c_int64, ct.c_int]
        L.orc_apply_h_generic.argtypes = [ct.c_int, ct.c_int, _vp, _vp, _vp, _vp]
        L.orc_lieb_ho.argtypes = [ct.c_int, ct.c_double, _vp]
        L.orc_lieb_hint.argtypes = [ct.c_int, ct.c_double, _vp]
        L.orc_perf_inputs.argtypes = [ct.c_int, ct.c_int, _vp, _vp, _vp]
        L.orc_lanczos.restype = ct.c_int
        L.orc_lanczos.argtypes = [ct.c_int, ct.c_int, ct.c_int] + [_vp] * 8 + [
            ct.c_int, _vp, _vp, _vp, ct.c_int]
        L.orc_ground.restype = ct.c_double
        L.orc_ground.argtypes = [ct.c_int, ct.c_int, ct.c_int] + [_vp] * 8 + [
            ct.c_int, _vp, _vp, ct.c_int]

    # tables ---------------------------------------------------------------
    def nc(self, N, M):
        return int(self.lib.orc_nc(N, M))

    def ncmat(self, N, M):
        t = np.zeros((N + 1) * (M + 1), np.int32)
        self.lib.orc_ncmat(N, M, _ptr(t))
        return t

    def index_to_fock(self, k, N, M):
        v = np.zeros(M, np.int32)
        self.lib.orc_index_to_fock(k, N, M, _ptr(v))
        return v

    def fock_to_index(self, N, M, v):
        v = np.ascontiguousarray(v, np.int32)
        return int(self.lib.orc_fock_to_index(N, M, _ptr(v)))

    def focks(self, N, M, threads=0):
        IF = np.zeros(self.nc(N, M) * M, np.int32)
        assert self.lib.orc_setup_focks(N, M, _ptr(IF), threads or os.cpu_count()) == 0
        return IF

    def one_one_map(self, N, M, IF, threads=0):
        Map = np.zeros(self.nc(N, M) * M * M, np.int32)
        self.lib.orc_one_one_map(N, M, _ptr(IF), _ptr(Map), threads or os.cpu_count())
        return Map

    def one_two_map(self, N, M, IF, threads=0):
        nc = self.nc(N, M)
        stride = np.zeros(nc, np.int64)
        chunks = self.lib.orc_one_two_strides(N, M, _ptr(IF), _ptr(stride))
        Map = np.zeros(chunks * M * M, np.int32)
        self.lib.orc_one_two_map(N, M, _ptr(IF), _ptr(stride), _ptr(Map), threads or os.cpu_count())
        return Map, stride

    def two_two_map(self, N, M, IF, threads=0):
        nc = self.nc(N, M)
        stride = np.zeros(nc, np.int64)
        chunks = self.lib.orc_two_two_strides(N, M, _ptr(IF), _ptr(stride))
        Map = np.zeros(chunks * M * M, np.int32)
        self.lib.orc_two_two_map(N, M, _ptr(IF), _ptr(stride), _ptr(Map), threads or os.cpu_count())
        return Map, stride

    # operators ------------------------------------------------------------
    def apply_h(self, N, M, C, Ho, Hint, mode=2, IF=None, maps=None, row0=0, row1=None,
                threads=0, out=None):
        """mode 0: applyHconf (hash only), 1: applyHconf_X, 2: applyHconf_XX.
        maps = (Map, MapOT, strideOT, MapTT, strideTT) or None (hash lookups)."""
        nc = self.nc(N, M)
        if IF is None:
            IF = self.focks(N, M)
        Map = MapOT = sOT = MapTT = sTT = None
        if maps is not None:
            Map, MapOT, sOT, MapTT, sTT = maps
        C = np.ascontiguousarray(C, np.complex128)
        Ho = np.ascontiguousarray(Ho, np.complex128)
        Hint = np.ascontiguousarray(Hint, np.complex128)
        if out is None:
            out = np.zeros(nc, np.complex128)
        r1 = nc if row1 is None else row1
        rc = self.lib.orc_apply_h(N, M, mode, _ptr(IF), _ptr(Map), _ptr(MapOT), _ptr(sOT),
                                  _ptr(MapTT), _ptr(sTT), _ptr(C), _ptr(Ho), _ptr(Hint),
                                  _ptr(out), row0, r1, threads or os.cpu_count())
        assert rc == 0
        return out

    def obrho(self, N, M, C, IF=None, Map=None):
        if IF is None:
            IF = self.focks(N, M)
        rho = np.zeros(M * M, np.complex128)
        self.lib.orc_obrho(N, M, _ptr(IF), _ptr(Map), _ptr(np.ascontiguousarray(C)), _ptr(rho))
        return rho.reshape(M, M)

    def density(self, N, M, order, phi, psi):
        """Flat t1[k + l*M] or t2[k + s*M + q*M^2 + l*M^3] = <phi|a+..a..|psi>."""
        t = np.zeros(M ** (2 * order), np.complex128)
        self.lib.orc_density_generic(N, M, order, _ptr(np.ascontiguousarray(phi)),
                                     _ptr(np.ascontiguousarray(psi)), _ptr(t))
        return t

    def density_rows(self, N, M, order, phi, psi, row0, row1, threads=0):
        """density() with the ket restricted to rows [row0, row1): <phi| ... |psi_S>."""
        t = np.zeros(M ** (2 * order), np.complex128)
        rc = self.lib.orc_density_rows(N, M, order, _ptr(np.ascontiguousarray(phi)),
                                       _ptr(np.ascontiguousarray(psi)), _ptr(t), int(row0), int(row1),
                                       threads or os.cpu_count())
        assert rc == 0
        return t

    def apply_h_generic(self, N, M, Ho, Hint, psi):
        out = np.zeros(self.nc(N, M), np.complex128)
        self.lib.orc_apply_h_generic(N, M, _ptr(np.ascontiguousarray(Ho, np.complex128)),
                                     _ptr(np.ascontiguousarray(Hint, np.complex128)),
                                     _ptr(np.ascontiguousarray(psi)), _ptr(out))
        return out

    # inputs ---------------------------------------------------------------
    def lieb(self, M, g, L=1.0):
        Ho = np.zeros(M * M, np.complex128)
        Hint = np.zeros(M ** 4, np.complex128)
        self.lib.orc_lieb_ho(M, L, _ptr(Ho))
        self.lib.orc_lieb_hint(M, g, _ptr(Hint))
        return Ho.reshape(M, M), Hint

    def perf_inputs(self, N, M):
        C = np.zeros(self.nc(N, M), np.complex128)
        Ho = np.zeros(M * M, np.complex128)
        Hint = np.zeros(M ** 4, np.complex128)
        self.lib.orc_perf_inputs(N, M, _ptr(C), _ptr(Ho), _ptr(Hint))
        return C, Ho.reshape(M, M), Hint

    # Lanczos --------------------------------------------------------------
    def ground(self, N, M, Ho, Hint, C0, niter, mode=2, maps=None, IF=None, threads=0):
        if IF is None:
            IF = self.focks(N, M)
        Map = MapOT = sOT = MapTT = sTT = None
        if maps is not None:
            Map, MapOT, sOT, MapTT, sTT = maps
        C = np.array(C0, np.complex128, copy=True)
        it = ct.c_int(0)
        E = self.lib.orc_ground(N, M, mode, _ptr(IF), _ptr(Map), _ptr(MapOT), _ptr(sOT),
                                _ptr(MapTT), _ptr(sTT),
                                _ptr(np.ascontiguousarray(Ho, np.complex128)),
                                _ptr(np.ascontiguousarray(Hint, np.complex128)), niter,
                                _ptr(C), ct.byref(it), threads or os.cpu_count())
        return E, C, it.value

    def lanczos(self, N, M, Ho, Hint, C0, lm, mode=2, maps=None, IF=None, threads=0):
        if IF is None:
            IF = self.focks(N, M)
        Map = MapOT = sOT = MapTT = sTT = None
        if maps is not None:
            Map, MapOT, sOT, MapTT, sTT = maps
        nc = self.nc(N, M)
        lvec = np.zeros((lm, nc), np.complex128)
        lvec[0] = C0
        diag = np.zeros(lm, np.complex128)
        off = np.zeros(lm, np.complex128)
        it = self.lib.orc_lanczos(N, M, mode, _ptr(IF), _ptr(Map), _ptr(MapOT), _ptr(sOT),
                                  _ptr(MapTT), _ptr(sTT),
                                  _ptr(np.ascontiguousarray(Ho, np.complex128)),
                                  _ptr(np.ascontiguousarray(Hint, np.complex128)), lm,
                                  _ptr(lvec), _ptr(diag), _ptr(off), threads or os.cpu_count())
        return it, diag, off, lvec


# ---------------------------------------------------------------------------
# the reference compiled unmodified
# ---------------------------------------------------------------------------

def ref_available() -> bool:
    return os.path.exists(REF_PATH)


class Ref:
    """ctypes view of the reference's own functions. Ho / rho1 are passed as
    row-pointer arrays (the reference's Cmatrix = double complex **)."""

    def __init__(self, path: str = REF_PATH):
        if not os.path.exists(path):
            build(ref=True)
        L = ct.CDLL(path)
        self.lib = L
        L.NC.restype = ct.c_int
        L.NC.argtypes = [ct.c_int, ct.c_int]
        for name in ("setupNCmat", "setupFocks"):
            getattr(L, name).restype = _c_int_p
            getattr(L, name).argtypes = [ct.c_int, ct.c_int]
        L.IndexToFock.argtypes = [ct.c_int, ct.c_int, ct.c_int, _vp]
        L.FockToIndex.restype = ct.c_int
        L.FockToIndex.argtypes = [ct.c_int, ct.c_int, _vp, _vp]
        L.OneOneMap.restype = _c_int_p
        L.OneOneMap.argtypes = [ct.c_int, ct.c_int, _vp, _vp]
        for name in ("OneTwoMap", "TwoTwoMap"):
            getattr(L, name).restype = _c_int_p
            getattr(L, name).argtypes = [ct.c_int, ct.c_int, _vp, _vp, _vp]
        L.applyHconf.argtypes = [ct.c_int, ct.c_int] + [_vp] * 6
        L.applyHconf_X.argtypes = [ct.c_int, ct.c_int] + [_vp] * 9
        L.applyHconf_XX.argtypes = [ct.c_int, ct.c_int] + [_vp] * 10
        L.applyHconf_omp.argtypes = [ct.c_int, ct.c_int] + [_vp] * 10
        L.OBrho.argtypes = [ct.c_int, ct.c_int, _vp, _vp, _vp]
        L.OBrho_X.argtypes = [ct.c_int, ct.c_int] + [_vp] * 4
        L.OBrho_XM.argtypes = [ct.c_int, ct.c_int] + [_vp] * 5
        L.TBrho.argtypes = [ct.c_int, ct.c_int] + [_vp] * 4
        L.TBrho_X.argtypes = [ct.c_int, ct.c_int] + [_vp] * 7
        L.TBrho_XX.argtypes = [ct.c_int, ct.c_int] + [_vp] * 9
        L.setupHo.argtypes = [ct.c_int, ct.c_double, _vp]
        L.setupHint.argtypes = [ct.c_int, ct.c_double, _vp]
        L.ground.restype = ct.c_double
        L.ground.argtypes = [ct.c_int, ct.c_int, ct.c_int] + [_vp] * 9
        self._libc = ct.CDLL(None)
        self._libc.free.argtypes = [_vp]

    def _take(self, p, n):
        if n == 0 or not p:
            self._libc.free(ct.cast(p, _vp))
            return np.zeros(0, np.int32)
        a = np.ctypeslib.as_array(p, shape=(n,)).copy()
        self._libc.free(ct.cast(p, _vp))
        return a

    @staticmethod
    def _rows(mat: np.ndarray):
        """Cmatrix view: keeps `mat` alive through the returned tuple."""
        mat = np.ascontiguousarray(mat, np.complex128)
        ptrs = (_vp * mat.shape[0])(*[mat[i].ctypes.data for i in range(mat.shape[0])])
        return mat, ptrs

    def nc(self, N, M):
        return int(self.lib.NC(N, M))

    def ncmat(self, N, M):
        return self._take(self.lib.setupNCmat(N, M), (N + 1) * (M + 1))

    def focks(self, N, M):
        return self._take(self.lib.setupFocks(N, M), self.nc(N, M) * M)

    def index_to_fock(self, k, N, M):
        v = np.zeros(M, np.int32)
        self.lib.IndexToFock(k, N, M, _ptr(v))
        return v

    def fock_to_index(self, N, M, NCmat, v):
        return int(self.lib.FockToIndex(N, M, _ptr(NCmat), _ptr(np.ascontiguousarray(v, np.int32))))

    def one_one_map(self, N, M, NCmat, IF):
        return self._take(self.lib.OneOneMap(N, M, _ptr(NCmat), _ptr(IF)), self.nc(N, M) * M * M)

    def _two_map(self, fn, N, M, NCmat, IF, two_orbital):
        nc = self.nc(N, M)
        stride = np.zeros(nc, np.int32)
        p = fn(N, M, _ptr(NCmat), _ptr(IF), _ptr(stride))
        # total chunks counted exactly as the allocators do
        rows = IF.reshape(nc, M)
        if two_orbital:
            occ = (rows >= 1).astype(np.int64)
            cnt = (occ.sum(1) * (occ.sum(1) - 1)) // 2
        else:
            cnt = (rows >= 2).sum(1)
        total = int(cnt.sum()) * M * M
        return self._take(p, total), stride

    def one_two_map(self, N, M, NCmat, IF):
        return self._two_map(self.lib.OneTwoMap, N, M, NCmat, IF, False)

    def two_two_map(self, N, M, NCmat, IF):
        return self._two_map(self.lib.TwoTwoMap, N, M, NCmat, IF, True)

    def apply_h(self, variant, N, M, C, Ho, Hint, tables):
        """variant in {'plain','X','XX','omp'}; tables = dict with NCmat, IF, Map,
        MapOT, strideOT, MapTT, strideTT (as produced by this class)."""
        t = tables
        C = np.ascontiguousarray(C, np.complex128)
        Hint = np.ascontiguousarray(Hint, np.complex128)
        out = np.zeros_like(C)
        hom, hop = self._rows(Ho)
        if variant == "plain":
            self.lib.applyHconf(N, M, _ptr(t["NCmat"]), _ptr(t["IF"]), _ptr(C), hop,
                                _ptr(Hint), _ptr(out))
        elif variant == "X":
            self.lib.applyHconf_X(N, M, _ptr(t["Map"]), _ptr(t["MapOT"]), _ptr(t["strideOT"]),
                                  _ptr(t["NCmat"]), _ptr(t["IF"]), _ptr(C), hop, _ptr(Hint),
                                  _ptr(out))
        else:
            fn = self.lib.applyHconf_XX if variant == "XX" else self.lib.applyHconf_omp
            fn(N, M, _ptr(t["Map"]), _ptr(t["MapOT"]), _ptr(t["MapTT"]), _ptr(t["strideOT"]),
               _ptr(t["strideTT"]), _ptr(t["IF"]), _ptr(C), hop, _ptr(Hint), _ptr(out))
        return out

    def rho1(self, variant, N, M, C, tables):
        t = tables
        C = np.ascontiguousarray(C, np.complex128)
        rho = np.zeros((M, M), np.complex128)
        rm, rp = self._rows(rho)
        if variant == "plain":
            self.lib.OBrho(N, M, _ptr(t["NCmat"]), _ptr(C), rp)
        elif variant == "X":
            self.lib.OBrho_X(N, M, _ptr(t["NCmat"]), _ptr(t["IF"]), _ptr(C), rp)
        else:
            self.lib.OBrho_XM(N, M, _ptr(t["Map"]), _ptr(t["NCmat"]), _ptr(t["IF"]), _ptr(C), rp)
        return rm

    def rho2(self, variant, N, M, C, tables):
        t = tables
        C = np.ascontiguousarray(C, np.complex128)
        rho = np.zeros(M ** 4, np.complex128)
        if variant == "plain":
            self.lib.TBrho(N, M, _ptr(t["NCmat"]), _ptr(t["IF"]), _ptr(C), _ptr(rho))
        elif variant == "X":
            self.lib.TBrho_X(N, M, _ptr(t["Map"]), _ptr(t["MapOT"]), _ptr(t["strideOT"]),
                             _ptr(t["NCmat"]), _ptr(t["IF"]), _ptr(C), _ptr(rho))
        else:
            self.lib.TBrho_XX(N, M, _ptr(t["Map"]), _ptr(t["MapOT"]), _ptr(t["MapTT"]),
                              _ptr(t["strideOT"]), _ptr(t["strideTT"]), _ptr(t["NCmat"]),
                              _ptr(t["IF"]), _ptr(C), _ptr(rho))
        return rho

    def tables(self, N, M, two_orbital=True):
        NCmat = self.ncmat(N, M)
        IF = self.focks(N, M)
        Map = self.one_one_map(N, M, NCmat, IF)
        MapOT, sOT = self.one_two_map(N, M, NCmat, IF)
        d = dict(NCmat=NCmat, IF=IF, Map=Map, MapOT=MapOT, strideOT=sOT)
        if two_orbital:
            MapTT, sTT = self.two_two_map(N, M, NCmat, IF)
            d.update(MapTT=MapTT, strideTT=sTT)
        return d

    def lieb(self, M, g, L=1.0):
        Ho = np.zeros((M, M), np.complex128)
        hm, hp = self._rows(Ho)
        self.lib.setupHo(M, L, hp)
        Hint = np.zeros(M ** 4, np.complex128)
        self.lib.setupHint(M, g, _ptr(Hint))
        return hm, Hint

    def ground(self, N, M, Ho, Hint, C0, niter, tables):
        t = tables
        C = np.array(C0, np.complex128, copy=True)
        hm, hp = self._rows(Ho)
        E = self.lib.ground(niter, N, M, _ptr(t["IF"]), _ptr(t["strideOT"]), _ptr(t["strideTT"]),
                            _ptr(t["Map"]), _ptr(t["MapOT"]), _ptr(t["MapTT"]), hp,
                            _ptr(np.ascontiguousarray(Hint, np.complex128)), _ptr(C))
        return E, C


# ---------------------------------------------------------------------------
# the reference's own CUDA kernel (cuda/hamiltonianMatrix.cuh:60-626)
# ---------------------------------------------------------------------------
REFCUDA_PATH = os.path.join(HERE, "_ref", "libmcpi_refcuda.so")
REFCUDA_HOST_PATH = os.path.join(HERE, "_ref", "refcuda_host")


def refcuda_available() -> bool:
    return os.path.exists(REFCUDA_PATH) and os.path.exists(REFCUDA_HOST_PATH)


def _cuda_layout(Ho):
    # the kernel reads Ho[k + M*l] for the CPU reference's Ho[k][l]
    return np.ascontiguousarray(np.asarray(Ho, np.complex128).T)


def refcuda_host_apply_h(N, M, C, Ho, Hint, workdir):
    """H C from the reference CUDA kernel's source run on the host under
    AddressSanitizer (oracle/refcuda_host.cpp). Raises on any sanitizer report."""
    inp = os.path.join(workdir, f"refcuda_in_{N}_{M}.bin")
    outp = os.path.join(workdir, f"refcuda_out_{N}_{M}.bin")
    with open(inp, "wb") as f:
        f.write(np.ascontiguousarray(C, np.complex128).tobytes())
        f.write(_cuda_layout(Ho).tobytes())
        f.write(np.ascontiguousarray(Hint, np.complex128).tobytes())
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:halt_on_error=1:abort_on_error=0")
    r = subprocess.run([REFCUDA_HOST_PATH, str(N), str(M), inp, outp], env=env,
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"refcuda_host N={N} M={M} failed ({r.returncode}):\n{r.stderr[-4000:]}")
    return np.fromfile(outp, np.complex128)


class RefCuda:
    """ctypes view of oracle/_ref/libmcpi_refcuda.so: the reference CUDA kernel
    with its own int32 maps, launched as cuda/performanceTest.cu launches it."""

    def __init__(self, path: str = REFCUDA_PATH):
        L = ct.CDLL(path)
        L.refcuda_fits.restype = ct.c_int
        L.refcuda_fits.argtypes = [ct.c_int, ct.c_int]
        L.refcuda_map_bytes.restype = ct.c_int64
        L.refcuda_apply_h.restype = ct.c_int
        L.refcuda_apply_h.argtypes = [ct.c_int, ct.c_int, _vp, _vp, _vp, _vp, ct.c_int,
                                      ct.POINTER(ct.c_float), ct.c_char_p, ct.c_int]
        self.lib = L

    def fits(self, N, M) -> bool:
        return bool(self.lib.refcuda_fits(N, M))

    def apply_h(self, N, M, C, Ho, Hint, reps=0):
        """(out, ms per launch averaged over `reps` timed launches, map bytes)."""
        C = np.ascontiguousarray(C, np.complex128)
        Hint = np.ascontiguousarray(Hint, np.complex128)
        ho = _cuda_layout(Ho)
        out = np.zeros(nc_of(N, M), np.complex128)
        ms = ct.c_float(0.0)
        err = ct.create_string_buffer(512)
        rc = self.lib.refcuda_apply_h(N, M, _ptr(C), _ptr(ho), _ptr(Hint), _ptr(out), reps,
                                      ct.byref(ms), err, 512)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return out, float(ms.value), int(self.lib.refcuda_map_bytes())
