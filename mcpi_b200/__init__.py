"""mcpi_b200: B200-native multiconfigurational hot path for N bosons in M orbitals.

Python host layer over the C ABI of ``libmcpi_b200.so`` (include/mcpi_b200.h).
PyTorch supplies device memory and the CUDA stream; all arithmetic runs in the
library's CUDA kernels. There is no CPU fallback: importing works anywhere,
but every operation raises ``MCPIError`` unless the compiled library and a
CUDA device are present.

Two layers:

* ``FockSpace`` -- device-resident space (N, M): tables, H.psi, densities,
  transition densities, Lanczos, ground state. Tensors are torch complex128 /
  int32 on the space's device.
* reference-named functions (``NC``, ``setupNCmat``, ``setupFocks``,
  ``OneOneMap``, ``OneTwoMap``, ``TwoTwoMap``, ``applyHconf``, ``applyHconf_X``,
  ``applyHconf_XX``, ``applyHconf_omp``, ``OBrho_XM``, ``TBrho_XX``,
  ``lanczos``, ``ground``) taking and returning host numpy arrays in the
  reference layouts of configurationsMap.h, hamiltonianMatrix.h,
  onebodyMatrix.h, twobodyMatrix.h and groundStateLieb.c.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmcpi_b200.so")

VARIANT_MAPS = 0   # applyHconf_X / _XX / _omp and the reference CUDA kernel
VARIANT_HASH = 1   # applyHconf (plain): Rule 9 summed over every ordering

# space options (mcpi_space_set_option; meanings in include/mcpi_b200.h)
OPT_DENSE_PAIR_KERNEL = 1
OPT_NO_MOMENTUM_KERNEL = 2
OPT_CREATE_FORM = 3
OPT_NO_GEMM_KERNEL = 4
OPT_WAIT_LIMIT_KCYCLES = 5
OPT_TEST_STALL_GATHER = 6
OPT_NO_OCC_TABLES = 7
OPT_FUSED_HPSI = 8
OPT_FUSED_LEAD = 9
OPT_DIRECT_HPSI = 11


class MCPIError(RuntimeError):
    """A status other than MCPI_OK returned by the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(f"mcpi status {status}: {message}")
        self.status = status


_lib = None
_vp = ct.c_void_p


def lib():
    """The loaded libmcpi_b200.so (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MCPIError(-1, f"{LIB_PATH} not built (run __graft_entry__.build())")
    L = ct.CDLL(LIB_PATH)
    i, i64, d = ct.c_int, ct.c_int64, ct.c_double
    p64, p32, pd, pi = (ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int32), ct.POINTER(ct.c_double),
                        ct.POINTER(ct.c_int))
    sig = {
        "mcpi_status_string": (ct.c_char_p, [i]),
        "mcpi_last_error": (ct.c_char_p, []),
        "mcpi_nc": (i, [i, i, p64]),
        "mcpi_space_create": (i, [i, i, i, ct.POINTER(_vp)]),
        "mcpi_space_destroy": (i, [_vp]),
        "mcpi_space_set_stream": (i, [_vp, _vp]),
        "mcpi_space_sync": (i, [_vp]),
        "mcpi_space_set_option": (i, [_vp, i, i]),
        "mcpi_space_dims": (i, [_vp, pi, pi, p64]),
        "mcpi_ncmat": (i, [i, i, _vp]),
        "mcpi_index_to_fock": (i, [i, i, i64, _vp]),
        "mcpi_fock_to_index": (i, [i, i, _vp, p64]),
        "mcpi_focks": (i, [_vp, _vp]),
        "mcpi_one_one_map": (i, [_vp, _vp]),
        "mcpi_two_map_size": (i, [_vp, i, p64]),
        "mcpi_two_map": (i, [_vp, i, _vp, _vp]),
        "mcpi_set_integrals": (i, [_vp, _vp, _vp, i]),
        "mcpi_apply_h": (i, [_vp, _vp, _vp]),
        "mcpi_apply_h_adjoint": (i, [_vp, _vp, _vp]),
        "mcpi_apply_h_rows": (i, [_vp, _vp, i64, i64, _vp]),
        "mcpi_apply_h_host": (i, [_vp, i, _vp, _vp]),
        "mcpi_apply_h_profile": (i, [_vp, _vp, _vp, i, _vp]),
        "mcpi_rho1": (i, [_vp, _vp, _vp]),
        "mcpi_rho2": (i, [_vp, _vp, _vp]),
        "mcpi_trans_rho1": (i, [_vp, _vp, _vp, _vp]),
        "mcpi_trans_rho2": (i, [_vp, _vp, _vp, _vp]),
        "mcpi_dot": (i, [_vp, _vp, _vp, _vp]),
        "mcpi_lanczos": (i, [_vp, _vp, i, _vp, _vp, pi]),
        "mcpi_ground": (i, [_vp, _vp, i, pd, pi]),
        "mcpi_ground_lowmem": (i, [_vp, _vp, i, pd, pi]),
        "mcpi_tridiag_eig": (i, [i, _vp, _vp, _vp]),
        "mcpi_lieb_integrals": (i, [i, d, d, _vp, _vp]),
        "mcpi_batch_create": (i, [i, _vp, _vp, i, i, ct.POINTER(_vp)]),
        "mcpi_batch_member_size": (i, [_vp, i, p64]),
        "mcpi_batch_set_integrals": (i, [_vp, i, _vp, _vp, i]),
        "mcpi_batch_set_start": (i, [_vp, i, _vp]),
        "mcpi_batch_run": (i, [_vp, _vp, _vp]),
        "mcpi_batch_arena_bytes": (i, [_vp, ct.POINTER(ct.c_size_t)]),
        "mcpi_batch_set_schedule": (i, [_vp, i]),
        "mcpi_batch_schedule": (i, [_vp, ct.POINTER(ct.c_int), _vp]),
        "mcpi_batch_set_hpsi_schedule": (i, [_vp, i]),
        "mcpi_batch_hpsi_schedule": (i, [_vp, ct.POINTER(ct.c_int), _vp]),
        "mcpi_batch_destroy": (i, [_vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        L = lib()
        raise MCPIError(rc, L.mcpi_last_error().decode() or L.mcpi_status_string(rc).decode())


def _np_ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


def nc_of(N: int, M: int) -> int:
    """NC(N,M) = C(N+M-1, N) (configurationsMap.h:145-202)."""
    v = ct.c_int64(0)
    _check(lib().mcpi_nc(N, M, ct.byref(v)))
    return v.value


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------

def lieb_integrals(M: int, g: float, L: float = 1.0):
    """Lieb-Liniger plane-wave integrals (groundStateLieb.c:129-213):
    Ho (M, M) complex, Hint flat M^4 complex."""
    Ho = np.zeros((M, M), np.complex128)
    Hint = np.zeros(M ** 4, np.complex128)
    _check(lib().mcpi_lieb_integrals(M, float(g), float(L), _np_ptr(Ho), _np_ptr(Hint)))
    return Ho, Hint


def symmetrize_hint(h: np.ndarray, M: int) -> np.ndarray:
    """Average a flat Hint[k + s*M + q*M^2 + l*M^3] over the bosonic 8-fold group
    H[k,s,q,l] = H[s,k,q,l] = H[k,s,l,q] = conj(H[q,l,k,s]). The reference's
    folded rules read one representative per orbit, so they reproduce the full
    operator only for Hint with this symmetry."""
    t = h.reshape(M, M, M, M)            # axes (l, q, s, k)
    four = (t + t.transpose(0, 1, 3, 2) + t.transpose(1, 0, 2, 3) + t.transpose(1, 0, 3, 2)) / 4.0
    herm = np.conj(four.transpose(2, 3, 0, 1))
    return ((four + herm) / 2.0).reshape(-1).copy()


def random_problem(N: int, M: int, seed: int):
    """Seeded synthetic inputs: normalised complex-normal psi, Hermitian Ho with
    N(0,1) entries, N(0,1) complex Hint averaged over the 8-fold group."""
    rng = np.random.default_rng(seed)
    nc = nc_of(N, M)
    C = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    C /= np.linalg.norm(C)
    A = rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))
    Ho = (A + A.conj().T) / 2.0
    H = rng.standard_normal(M ** 4) + 1j * rng.standard_normal(M ** 4)
    return C, Ho, symmetrize_hint(H, M)


def tridiag_eig(d, e, vectors: bool = True):
    """Eigen-decomposition of the symmetric tridiagonal (d, e) with the
    LAPACKE_dstev('V') contract (groundStateLieb.c:435): ascending eigenvalues,
    z[k, j] = component k of eigenvector j. Host routine, no GPU needed."""
    d = np.array(d, np.float64, copy=True)
    n = d.size
    e = np.array(e, np.float64, copy=True) if n > 1 else np.zeros(1)
    z = np.zeros((n, n), np.float64) if vectors else None
    _check(lib().mcpi_tridiag_eig(n, _np_ptr(d), _np_ptr(e), _np_ptr(z) if vectors else None))
    return d, z


# ---------------------------------------------------------------------------
# device space
# ---------------------------------------------------------------------------

def _torch():
    import torch
    return torch


class FockSpace:
    """Fock space of N bosons in M orbitals on one CUDA device."""

    def __init__(self, N: int, M: int, device: int = 0):
        torch = _torch()
        if not torch.cuda.is_available():
            raise MCPIError(3, "no CUDA device: mcpi_b200 has no CPU path")
        self.N, self.M, self.device = N, M, device
        self.torch_device = torch.device("cuda", device)
        h = _vp()
        _check(lib().mcpi_space_create(N, M, device, ct.byref(h)))
        self._h = h
        self.nc = nc_of(N, M)
        self.P = M * (M + 1) // 2

    def close(self):
        if getattr(self, "_h", None):
            lib().mcpi_space_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # plumbing --------------------------------------------------------------
    def _stream(self):
        torch = _torch()
        s = torch.cuda.current_stream(self.torch_device).cuda_stream
        _check(lib().mcpi_space_set_stream(self._h, _vp(s)))

    def _vec(self, x, n=None):
        torch = _torch()
        n = self.nc if n is None else n
        if isinstance(x, np.ndarray):
            x = torch.from_numpy(np.ascontiguousarray(x, np.complex128))
        if x.dtype != torch.complex128 or x.device != self.torch_device or not x.is_contiguous():
            x = x.to(self.torch_device, torch.complex128).contiguous()
        if x.numel() != n:
            raise MCPIError(1, f"expected {n} complex entries, got {x.numel()}")
        return x

    def empty(self, n=None, dtype=None):
        torch = _torch()
        return torch.empty(self.nc if n is None else n, dtype=dtype or torch.complex128,
                           device=self.torch_device)

    def sync(self):
        _check(lib().mcpi_space_sync(self._h))

    def set_dense_pair_kernel(self, on: bool = True):
        """Force the dense pair-matrix H.psi kernel (applies at the next set_integrals)."""
        _check(lib().mcpi_space_set_option(self._h, 1, int(on)))

    def set_option(self, option: int, value: int):
        _check(lib().mcpi_space_set_option(self._h, int(option), int(value)))

    def set_momentum_kernel(self, on: bool = True):
        """Allow (default) or forbid the momentum-block H.psi kernel (next set_integrals)."""
        _check(lib().mcpi_space_set_option(self._h, 2, int(not on)))

    # tables ----------------------------------------------------------------
    def focks(self):
        """IF[j + i*M] (configurationsMap.h:309-344), int32 tensor."""
        torch = _torch()
        out = self.empty(self.nc * self.M, torch.int32)
        self._stream()
        _check(lib().mcpi_focks(self._h, _vp(out.data_ptr())))
        return out

    def one_one_map(self):
        """Map[i + k*nc + l*M*nc] (configurationsMap.h:348-417), int32 tensor."""
        torch = _torch()
        out = self.empty(self.nc * self.M * self.M, torch.int32)
        self._stream()
        _check(lib().mcpi_one_one_map(self._h, _vp(out.data_ptr())))
        return out

    def two_map(self, two_orbital: bool):
        """(MapOT, strideOT) or (MapTT, strideTT) (configurationsMap.h:617-762 /
        421-613); strides int64."""
        torch = _torch()
        n = ct.c_int64(0)
        self._stream()
        _check(lib().mcpi_two_map_size(self._h, int(two_orbital), ct.byref(n)))
        buf = self.empty(max(n.value, 1), torch.int32)
        stride = self.empty(self.nc, torch.int64)
        _check(lib().mcpi_two_map(self._h, int(two_orbital), _vp(stride.data_ptr()),
                                  _vp(buf.data_ptr())))
        return buf[: n.value], stride

    # operators -------------------------------------------------------------
    def set_integrals(self, Ho, Hint, variant: int = VARIANT_MAPS):
        Ho = np.ascontiguousarray(np.asarray(Ho, np.complex128).reshape(self.M, self.M))
        Hint = np.ascontiguousarray(np.asarray(Hint, np.complex128).reshape(-1))
        if Hint.size != self.M ** 4:
            raise MCPIError(1, "Hint must have M^4 entries")
        self._stream()
        _check(lib().mcpi_set_integrals(self._h, _np_ptr(Ho), _np_ptr(Hint), int(variant)))

    def apply_h(self, C, out=None):
        C = self._vec(C)
        out = self.empty() if out is None else out
        self._stream()
        _check(lib().mcpi_apply_h(self._h, _vp(C.data_ptr()), _vp(out.data_ptr())))
        return out

    def apply_h_host(self, states, outs):
        """outs[k] = H states[k] for host arrays (numpy complex128 or CPU torch
        tensors, nc entries, contiguous; page-locked memory copies fastest),
        pipelined through the device by mcpi_apply_h_host."""
        torch = _torch()
        if len(states) != len(outs):
            raise MCPIError(1, "states and outs differ in length")

        def ptr(x, writable):
            if isinstance(x, np.ndarray):
                if x.dtype != np.complex128 or not x.flags.c_contiguous or x.size != self.nc or \
                        (writable and not x.flags.writeable):
                    raise MCPIError(1, f"expected a contiguous complex128 array of {self.nc} entries")
                return x.ctypes.data
            if x.dtype != torch.complex128 or x.device.type != "cpu" or not x.is_contiguous() or x.numel() != self.nc:
                raise MCPIError(1, f"expected a contiguous CPU complex128 tensor of {self.nc} entries")
            return x.data_ptr()

        n = len(states)
        pin = (ct.c_void_p * max(n, 1))(*[ptr(x, False) for x in states])
        pout = (ct.c_void_p * max(n, 1))(*[ptr(x, True) for x in outs])
        self._stream()
        _check(lib().mcpi_apply_h_host(self._h, n, ct.cast(pin, ct.c_void_p), ct.cast(pout, ct.c_void_p)))
        return outs

    def apply_h_rows(self, C, row0: int, row1: int, out=None):
        """Rows [row0, row1) of H C (C the whole vector)."""
        C = self._vec(C)
        out = self.empty(row1 - row0) if out is None else out
        self._stream()
        _check(lib().mcpi_apply_h_rows(self._h, _vp(C.data_ptr()), row0, row1,
                                       _vp(out.data_ptr()) if row1 > row0 else None))
        return out

    def apply_h_profile(self, C, out=None, reps: int = 10):
        """Mean CUDA-event durations (ms) of the two H.psi kernels."""
        C = self._vec(C)
        out = self.empty() if out is None else out
        ms = np.zeros(2, np.float32)
        self._stream()
        _check(lib().mcpi_apply_h_profile(self._h, _vp(C.data_ptr()), _vp(out.data_ptr()), reps,
                                          _np_ptr(ms)))
        return float(ms[0]), float(ms[1])

    def apply_h_adjoint(self, C, out=None):
        C = self._vec(C)
        out = self.empty() if out is None else out
        self._stream()
        _check(lib().mcpi_apply_h_adjoint(self._h, _vp(C.data_ptr()), _vp(out.data_ptr())))
        return out

    def _dens(self, fn, order, *vecs):
        vecs = [self._vec(v) for v in vecs]
        out = self.empty(self.M ** (2 * order))
        self._stream()
        _check(fn(self._h, *[_vp(v.data_ptr()) for v in vecs], _vp(out.data_ptr())))
        return out

    def rho1(self, C):
        """rho1[k, l] = <a+_k a_l> (onebodyMatrix.h:190-251), (M, M) tensor."""
        return self._dens(lib().mcpi_rho1, 1, C).reshape(self.M, self.M)

    def rho2(self, C):
        """rho2[k + s*M + q*M^2 + l*M^3] = <a+_k a+_s a_q a_l> (twobodyMatrix.h:991-1487)."""
        return self._dens(lib().mcpi_rho2, 2, C)

    def trans_rho1(self, phi, psi):
        """t1[k, l] = <phi|a+_k a_l|psi>, (M, M) tensor."""
        return self._dens(lib().mcpi_trans_rho1, 1, phi, psi).reshape(self.M, self.M)

    def trans_rho2(self, phi, psi):
        """t2[k + s*M + q*M^2 + l*M^3] = <phi|a+_k a+_s a_q a_l|psi>."""
        return self._dens(lib().mcpi_trans_rho2, 2, phi, psi)

    def dot(self, a, b) -> complex:
        a, b = self._vec(a), self._vec(b)
        r = np.zeros(2)
        self._stream()
        _check(lib().mcpi_dot(self._h, _vp(a.data_ptr()), _vp(b.data_ptr()), _np_ptr(r)))
        return complex(r[0], r[1])

    # Lanczos ---------------------------------------------------------------
    def lanczos(self, C0, lm: int):
        """groundStateLieb.c:217-344. Returns (iters, alpha[lm] complex, beta[lm], lvec)."""
        torch = _torch()
        lvec = torch.empty((lm, self.nc), dtype=torch.complex128, device=self.torch_device)
        lvec[0].copy_(self._vec(C0))
        diag = np.zeros(lm, np.complex128)
        off = np.zeros(lm, np.float64)
        it = ct.c_int(0)
        self._stream()
        _check(lib().mcpi_lanczos(self._h, _vp(lvec.data_ptr()), lm, _np_ptr(diag), _np_ptr(off),
                                  ct.byref(it)))
        return it.value, diag, off, lvec

    def ground(self, C0, niter: int, lowmem: bool = False):
        """groundStateLieb.c:348-471. Returns (E0, ground-state tensor, iterations).
        lowmem: two-pass Lanczos that regenerates the Krylov vectors instead of
        storing them (mcpi_ground_lowmem)."""
        C = self._vec(C0).clone()
        E = ct.c_double(0.0)
        it = ct.c_int(0)
        self._stream()
        fn = lib().mcpi_ground_lowmem if lowmem else lib().mcpi_ground
        _check(fn(self._h, _vp(C.data_ptr()), niter, ct.byref(E), ct.byref(it)))
        return E.value, C, it.value


class Batch:
    """Many Lanczos ground-state solves advanced together and replayed as one
    CUDA graph (mcpi_batch_* in mcpi_b200.h). members: list of (N, M)."""

    def __init__(self, members, lm: int, device: int = 0):
        self.members = list(members)
        n = len(self.members)
        Ns = np.array([m[0] for m in self.members], np.int32)
        Ms = np.array([m[1] for m in self.members], np.int32)
        h = _vp()
        _check(lib().mcpi_batch_create(n, _np_ptr(Ns), _np_ptr(Ms), lm, device, ct.byref(h)))
        self._h = h
        self.lm = lm
        self.nc = []
        for k in range(n):
            v = ct.c_int64(0)
            _check(lib().mcpi_batch_member_size(self._h, k, ct.byref(v)))
            self.nc.append(v.value)

    def set_integrals(self, k, Ho, Hint, variant=VARIANT_MAPS):
        N, M = self.members[k]
        Ho = np.ascontiguousarray(np.asarray(Ho, np.complex128).reshape(M, M))
        Hint = np.ascontiguousarray(np.asarray(Hint, np.complex128).reshape(-1))
        _check(lib().mcpi_batch_set_integrals(self._h, k, _np_ptr(Ho), _np_ptr(Hint), int(variant)))

    def set_start(self, k, C):
        C = np.ascontiguousarray(C, np.complex128)
        if C.size != self.nc[k]:
            raise MCPIError(1, "start vector has the wrong length")
        _check(lib().mcpi_batch_set_start(self._h, k, _np_ptr(C)))

    def run(self):
        """Returns (E0 per member, Lanczos steps per member)."""
        E = np.zeros(len(self.members))
        it = np.zeros(len(self.members), np.int32)
        _check(lib().mcpi_batch_run(self._h, _np_ptr(E), _np_ptr(it)))
        return E, it

    def arena_bytes(self) -> int:
        v = ct.c_size_t(0)
        _check(lib().mcpi_batch_arena_bytes(self._h, ct.byref(v)))
        return v.value

    def set_schedule(self, tile_rows: int):
        """Pin the vector-stage tile (512, 1024, 2048) or 0 to autotune at the
        first run (before the first run only)."""
        _check(lib().mcpi_batch_set_schedule(self._h, int(tile_rows)))

    def schedule(self):
        """(tile rows in use or 0 before the first run, probe ms of the
        candidates 512 / 1024 / 2048 when autotuned, else zeros)."""
        t = ct.c_int(0)
        ms = np.zeros(3, np.float32)
        _check(lib().mcpi_batch_schedule(self._h, ct.byref(t), _np_ptr(ms)))
        return t.value, ms

    def set_hpsi_schedule(self, schedule: int):
        """Pin the batched H.psi schedule (0..3: bit 0 concurrent M groups, bit 1
        interleaved blocks) or -1 to autotune at the first run."""
        _check(lib().mcpi_batch_set_hpsi_schedule(self._h, int(schedule)))

    def hpsi_schedule(self):
        """(H.psi schedule in use or -1 before the first run, probe ms of
        schedules 0..3 when autotuned, else zeros)."""
        t = ct.c_int(0)
        ms = np.zeros(4, np.float32)
        _check(lib().mcpi_batch_hpsi_schedule(self._h, ct.byref(t), _np_ptr(ms)))
        return t.value, ms

    def close(self):
        if getattr(self, "_h", None):
            lib().mcpi_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# reference-named host API (numpy in / numpy out, device underneath)
# ---------------------------------------------------------------------------

_spaces: dict = {}


def _space(N, M) -> FockSpace:
    sp = _spaces.get((N, M))
    if sp is None:
        sp = _spaces[(N, M)] = FockSpace(N, M)
    return sp


def NC(N: int, M: int) -> int:
    return nc_of(N, M)


def setupNCmat(N: int, M: int) -> np.ndarray:
    t = np.zeros((N + 1) * (M + 1), np.int32)
    _check(lib().mcpi_ncmat(N, M, _np_ptr(t)))
    return t


def IndexToFock(k: int, N: int, M: int) -> np.ndarray:
    v = np.zeros(M, np.int32)
    _check(lib().mcpi_index_to_fock(N, M, k, _np_ptr(v)))
    return v


def FockToIndex(N: int, M: int, v) -> int:
    v = np.ascontiguousarray(v, np.int32)
    k = ct.c_int64(0)
    _check(lib().mcpi_fock_to_index(N, M, _np_ptr(v), ct.byref(k)))
    return k.value


def setupFocks(N: int, M: int) -> np.ndarray:
    return _space(N, M).focks().cpu().numpy()


def OneOneMap(N: int, M: int) -> np.ndarray:
    return _space(N, M).one_one_map().cpu().numpy()


def OneTwoMap(N: int, M: int):
    m, s = _space(N, M).two_map(False)
    return m.cpu().numpy(), s.cpu().numpy()


def TwoTwoMap(N: int, M: int):
    m, s = _space(N, M).two_map(True)
    return m.cpu().numpy(), s.cpu().numpy()


def _apply(N, M, C, Ho, Hint, variant):
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint, variant)
    out = sp.apply_h(C)
    return out.cpu().numpy()


def applyHconf(N, M, C, Ho, Hint):
    """hamiltonianMatrix.h:31-425 (hash-only variant)."""
    return _apply(N, M, C, Ho, Hint, VARIANT_HASH)


def applyHconf_X(N, M, C, Ho, Hint):
    """hamiltonianMatrix.h:431-887."""
    return _apply(N, M, C, Ho, Hint, VARIANT_MAPS)


def applyHconf_XX(N, M, C, Ho, Hint):
    """hamiltonianMatrix.h:891-1425."""
    return _apply(N, M, C, Ho, Hint, VARIANT_MAPS)


applyHconf_omp = applyHconf_XX


def OBrho_XM(N, M, C):
    """onebodyMatrix.h:190-251 -> (M, M) array rho[k][l]."""
    return _space(N, M).rho1(C).cpu().numpy()


def TBrho_XX(N, M, C):
    """twobodyMatrix.h:991-1487 -> flat M^4 array."""
    return _space(N, M).rho2(C).cpu().numpy()


def ground(Niter, N, M, Ho, Hint, C):
    """groundStateLieb.c:348-471 -> (E0, ground state)."""
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint, VARIANT_MAPS)
    E, psi, _ = sp.ground(C, Niter)
    return E, psi.cpu().numpy()
