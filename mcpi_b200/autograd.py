"""Derivatives of H.psi, for verification (torch.autograd.Function).

For out = H psi with H built from (Ho, Hint) as the reference builds it
(hamiltonianMatrix.h: nine two-body rules, each reading one representative
Hint entry with factor 1, 2 or 4 times the outer 1/2), and a real loss L with
torch's cotangent g = dL/dRe(out) + i dL/dIm(out):

* d/dpsi  : H^dagger g                              (mcpi_apply_h_adjoint)
* d/dHo   : conj(t1), t1[k][l] = <g| a+_k a_l |psi>  (mcpi_trans_rho1)
* d/dHint : conj(P^T G), G[(k,s),(q,l)] = <g| a+_k a+_s a_q a_l |psi>
            (mcpi_trans_rho2), P^T the transpose of the rule folding that maps
            Hint to the pair matrix -- so the gradient is exact for any Hint,
            symmetric or not, and zero on entries no rule reads.

The transition densities are the library's CUDA kernels; this module only
does the O(M^4) index bookkeeping of P^T on the host.
"""
from __future__ import annotations

import numpy as np
import torch

from . import VARIANT_HASH, VARIANT_MAPS, FockSpace


def pair_index(k: int, s: int, M: int) -> int:
    if k > s:
        k, s = s, k
    return k * M - (k * (k - 1)) // 2 + (s - k)


def fold_pullback(G: np.ndarray, M: int, N: int, variant: int = VARIANT_MAPS) -> np.ndarray:
    """P^T G: the flat M^4 array c with c[x] = sum over the pair-matrix entries
    built from Hint[x] of (their coefficient) * G at that entry. G is the P x P
    pair form (rows = creation pair, columns = annihilation pair). Mirrors the
    rule folding of the C library (capi.cpp build_pair_matrix)."""
    M2, M3 = M * M, M * M * M
    c = np.zeros(M ** 4, np.complex128)
    if N < 2:
        return c

    def h(k, s, q, l):
        return k + s * M + q * M2 + l * M3

    def pr(a, b):
        return pair_index(a, b, M)

    for k in range(M):
        c[h(k, k, k, k)] += 0.5 * G[pr(k, k), pr(k, k)]                          # R1
        for s in range(k + 1, M):
            c[h(k, s, k, s)] += 2.0 * G[pr(k, s), pr(k, s)]                       # R2
        for q in range(M):
            if q != k:
                c[h(k, k, q, q)] += 0.5 * G[pr(k, k), pr(q, q)]                   # R3
                c[h(k, k, k, q)] += G[pr(k, k), pr(k, q)]                         # R4
                c[h(k, q, q, q)] += G[pr(k, q), pr(q, q)]                         # R5
        for q in range(M):
            for l in range(q + 1, M):
                if q != k and l != k:
                    c[h(k, k, q, l)] += G[pr(k, k), pr(q, l)]                     # R6
    for k in range(M):
        for s in range(k + 1, M):
            for q in range(M):
                if q in (k, s):
                    continue
                c[h(k, s, q, q)] += G[pr(k, s), pr(q, q)]                         # R7
                for l in range(q + 1, M):
                    if l in (k, s):
                        continue
                    g = G[pr(k, s), pr(q, l)]                                     # R9
                    if variant == VARIANT_HASH:
                        for x in (h(k, s, q, l), h(s, k, q, l), h(k, s, l, q), h(s, k, l, q)):
                            c[x] += 0.5 * g
                    else:
                        c[h(k, s, q, l)] += 2.0 * g
    for s in range(M):
        for k in range(M):
            for l in range(M):
                if k != s and l != k and l != s:
                    c[h(k, s, s, l)] += 2.0 * G[pr(k, s), pr(s, l)]               # R8
    return c


def pair_form(t2: np.ndarray, M: int) -> np.ndarray:
    """t2[k + s*M + q*M^2 + l*M^3] -> G[pair(k,s), pair(q,l)]."""
    P = M * (M + 1) // 2
    T = t2.reshape(M, M, M, M)      # axes (l, q, s, k)
    G = np.zeros((P, P), np.complex128)
    for k in range(M):
        for s in range(k, M):
            for q in range(M):
                for l in range(q, M):
                    G[pair_index(k, s, M), pair_index(q, l, M)] = T[l, q, s, k]
    return G


class ApplyH(torch.autograd.Function):
    """out = H(Ho, Hint) psi on a FockSpace, differentiable in psi, Ho and Hint."""

    @staticmethod
    def forward(ctx, psi, Ho, Hint, space: FockSpace, variant: int = VARIANT_MAPS):
        ho = Ho.detach().cpu().numpy()
        hint = Hint.detach().cpu().numpy()
        space.set_integrals(ho, hint, variant)
        out = space.apply_h(psi.detach())
        ctx.space, ctx.variant = space, variant
        ctx.ho, ctx.hint = ho, hint
        ctx.save_for_backward(psi.detach())
        return out

    @staticmethod
    def backward(ctx, g):
        (psi,) = ctx.saved_tensors
        sp, M, N = ctx.space, ctx.space.M, ctx.space.N
        g = g.contiguous()
        sp.set_integrals(ctx.ho, ctx.hint, ctx.variant)
        grad_psi = sp.apply_h_adjoint(g)
        t1 = sp.trans_rho1(g, psi).cpu().numpy()                 # <g|a+_k a_l|psi>
        grad_ho = torch.from_numpy(np.conj(t1)).to(torch.complex128)
        t2 = sp.trans_rho2(g, psi).cpu().numpy()
        c = fold_pullback(pair_form(t2, M), M, N, ctx.variant)
        grad_hint = torch.from_numpy(np.conj(c))
        return grad_psi, grad_ho, grad_hint, None, None


def apply_h(psi, Ho, Hint, space: FockSpace, variant: int = VARIANT_MAPS):
    return ApplyH.apply(psi, Ho, Hint, space, variant)


def hellmann_feynman_lieb(rho2: np.ndarray, M: int, L: float = 1.0) -> float:
    """dE0/dg for the Lieb-Liniger Hamiltonian (Hint = g/L on momentum-conserving
    index tuples, groundStateLieb.c:183-211; the rules read only such tuples
    and every factor is symmetric there): 1/2 sum_{k+s=q+l} rho2[k,s,q,l] / L
    with rho2 of the normalised ground state."""
    T = rho2.reshape(M, M, M, M)    # axes (l, q, s, k)
    tot = 0.0 + 0.0j
    for k in range(M):
        for s in range(M):
            for q in range(M):
                for l in range(M):
                    if k + s == q + l:
                        tot += T[l, q, s, k]
    return float((0.5 * tot / L).real)
