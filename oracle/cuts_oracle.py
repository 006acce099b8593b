"""CPU restatement of GLU's momentum-space gluon measurements (CUTTYPE =
GLUON_PROPS, EXCEPTIONAL, FIELDS).  TEST INFRASTRUCTURE ONLY: the tests use
it as the checker of the GPU path; the product package never imports it.

Followed, in GLU's default build (SIN_MOM on, CUT_FORWARD off, CONDOR_MODE,
matrix contraction for the three-gluon vertex):

* lie fields       src/Matrix_Ops/exactQ.c:358-385 (Hermitian_proj, LINEAR)
* Fourier step     src/Cuts/cuts.c:35-97 (backward, unnormalised transform
                   of each colour component: sum_x A(x) e^{+ipx})
* momentum list    src/Cuts/cut_routines.c:60-81 (simorb_ratios), 84-104
                   (get_diagonal), 183-225 (cylinder_DF), 242-290
                   (cylinder_CJD), 294-370 (psq/hypercubic cuts,
                   safe_momenta), 373-441 (get_mom_veclist)
* p-space Landau   src/Cuts/pspace_landau.c:29-81
* propagators      src/Cuts/glueprop.c:33-146
* MOMgg g2, g3     src/Cuts/MOMgg.c:89-211 (contraction_matrices)

Parity of this restatement is pinned against GLU's own cuts_struct run
through the reference harness (tests/test_cuts_host.py).  Plain loops in
scalar libm arithmetic for the list, so small lattices only.
"""
from __future__ import annotations

import math

import numpy as np

TWOPI = 6.283185307179586
PREC_TOL = 3 * 1.0e-14
ND = 4

# GLU's cut_mode / momentum_cut_def / lie_field_def values (GLU_enum.h)
EXCEPTIONAL, NONEXCEPTIONAL, FIELDS, GLUON_PROPS = 0, 1, 2, 6
HYPERCUBIC_CUT, PSQ_CUT, CYLINDER_CUT, CYLINDER_AND_CONICAL_CUT = 0, 1, 2, 3
LINEAR_DEF, LOG_DEF = 0, 1


def hermitian_proj(U: np.ndarray) -> np.ndarray:
    """Traceless Hermitian part of -i U per matrix, (..., 3, 3)."""
    im = np.stack([U[..., 0, 0].imag, U[..., 1, 1].imag, U[..., 2, 2].imag], -1)
    Q = np.zeros_like(U)
    Q[..., 0, 0] = (2 * im[..., 0] - im[..., 1] - im[..., 2]) / 3.0
    Q[..., 1, 1] = (2 * im[..., 1] - im[..., 0] - im[..., 2]) / 3.0
    Q[..., 2, 2] = -Q[..., 0, 0].real - Q[..., 1, 1].real
    for a, b in ((0, 1), (0, 2), (1, 2)):
        Q[..., a, b] = -1j * (U[..., a, b] - np.conj(U[..., b, a])) / 2.0
        Q[..., b, a] = np.conj(Q[..., a, b])
    return Q


def momentum_fields(links: np.ndarray, dims) -> np.ndarray:
    """A_mu(p) = sum_x A_mu(x) e^{+ipx} for every p of the 0..2pi zone,
    (V, 4, 3, 3), site order x fastest."""
    Lx, Ly, Lz, Lt = (int(d) for d in dims)
    V = Lx * Ly * Lz * Lt
    Q = hermitian_proj(np.asarray(links).reshape(V, 4, 3, 3))
    A = Q.reshape(Lt, Lz, Ly, Lx, 4, 3, 3)
    A = np.fft.ifftn(A, axes=(0, 1, 2, 3)) * V
    return A.reshape(V, 4, 3, 3)


def _coords(i, dims):
    out = []
    for L in dims:
        out.append(i % L)
        i //= L
    return out


def _site(x, dims):
    s = 0
    for mu in reversed(range(ND)):
        s = s * dims[mu] + x[mu]
    return s


def _diagonal(i):
    return [1.0 if (i >> mu) & 1 else -1.0 for mu in range(ND)]


def _compute_p(n, dims):
    return [2.0 * math.sin(n[mu] * (TWOPI / dims[mu]) * 0.5) for mu in range(ND)]


def _cylinder_df(q, width):
    norm = 1.0 / (2.0 * math.sqrt(ND))
    for d in range(2 << (ND - 1)):
        x = _diagonal(d)
        sp = 0.0
        for nu in range(ND):
            sp += q[nu] * x[nu]
        sp *= norm
        mod = 0.0
        for nu in range(ND):
            t = q[nu] - sp * x[nu]
            mod += t * t
        if math.sqrt(mod) <= width:
            return True
    return False


def _cylinder_cjd(q, width, arc):
    qn = 0.0
    for mu in range(ND):
        qn += q[mu] * q[mu]
    if qn < PREC_TOL:
        return True
    qn = 1.0 / math.sqrt(qn)
    for d in range(2 << (ND - 1)):
        x = _diagonal(d)
        nn = 0.0
        for nu in range(ND):
            nn += x[nu] * x[nu]
        nn = qn / math.sqrt(nn)
        sp = 0.0
        for nu in range(ND):
            sp += q[nu] * x[nu] * nn
        theta = math.acos(sp)
        dq = math.sin(theta) / qn
        if dq <= width and theta <= arc * 0.01745329251994330:
            return True
    return False


def veclist(dims, dir=GLUON_PROPS, type=PSQ_CUT, max_mom=20, angle=0,
            cyl_width=1.0):
    """(MOM (n, 4) int, idx (n,)) of the momenta kept by the cut, in GLU's
    order (lexicographic in the -pi..pi zone, x fastest)."""
    dims = [int(d) for d in dims]
    if dir == NONEXCEPTIONAL:
        type = PSQ_CUT
    small = min(dims)
    rats = [small / d for d in dims]
    width = TWOPI * cyl_width / small
    moms, idx = [], []
    V = int(np.prod(dims))
    for i in range(V):
        x = _coords(i, dims)
        n = [x[mu] - dims[mu] // 2 for mu in range(ND)]
        psq = 0.0
        for mu in range(ND):
            t = rats[mu] * n[mu]
            psq += t * t
        if type == HYPERCUBIC_CUT:
            r = math.sqrt(max_mom)
            ok = all(abs(float(n[mu]) * rats[mu]) <= r for mu in range(ND))
        elif type == CYLINDER_CUT:
            ok = psq <= max_mom and _cylinder_df(_compute_p(n, dims), width)
        elif type == CYLINDER_AND_CONICAL_CUT:
            ok = psq <= max_mom and _cylinder_cjd(_compute_p(n, dims), width, angle)
        else:
            ok = psq <= max_mom
        if ok:
            moms.append(n)
            idx.append(_site([n[mu] + dims[mu] if n[mu] < 0 else n[mu]
                              for mu in range(ND)], dims))
    return np.array(moms, dtype=np.int64).reshape(-1, ND), np.array(idx, dtype=np.int64)


def _sin_mom(n, dims):
    return np.array([2.0 * math.sin(n[mu] * (TWOPI / dims[mu]) * 0.5)
                     for mu in range(ND)])


def correct_pspace(A: np.ndarray, moms, idx, dims) -> tuple[np.ndarray, float]:
    """A at the listed momenta times e^{i p_mu / 2}, and the printed p-space
    gauge error (mean over the list of |sum_mu,j p_mu A_mu(p)_j| / 9)."""
    dims = [int(d) for d in dims]
    B = A[idx].copy()
    err = 0.0
    for k, n in enumerate(moms):
        s = 0.0
        for mu in range(ND):
            c = 0.5 * n[mu] * (TWOPI / dims[mu])
            p = 2.0 * math.sin(c)
            B[k, mu] *= complex(math.cos(c), 0.5 * p)
            s += B[k, mu].sum() * p
        err += abs(s) / 9.0
    return B, err / max(len(moms), 1)


def _psq(n, dims):
    mom = _sin_mom(n, dims)
    t = float(np.sum(mom * mom))
    return mom, (1.0 if t < PREC_TOL else t)


def gluon_props(B, moms, dims):
    """(transverse, longitudinal) per listed momentum from the corrected
    fields B (n, 4, 3, 3)."""
    V = int(np.prod(dims))
    num = len(moms)
    g2 = 2.0 / (8 * 3 * V)
    g0 = 2.0 / (8 * 4 * V)
    gl = 2.0 / (8 * V)
    zero = num >> 1
    tr = np.zeros(num)
    lo = np.zeros(num)
    for i in list(range(zero)) + [zero]:
        mom, psq = _psq(moms[i], dims)
        T = L = 0.0
        for mu in range(ND):
            for nu in range(ND):
                t = np.sum(B[i, mu] * np.conj(B[i, nu])).real
                c = mom[mu] * mom[nu] * (1.0 / psq) * t
                T += -c if mu != nu else t - c
                L += c
        tr[i] = T * (g0 if i == zero else g2)
        lo[i] = L * gl
    for i in range(zero + 1, num):
        tr[i] = tr[num - i - 1]
        lo[i] = lo[num - i - 1]
    return tr, lo


def exceptional(B, moms, dims):
    """(g2, g3) of the MOMgg scheme per listed momentum."""
    V = int(np.prod(dims))
    num = len(moms)
    g2n = 2.0 / (8 * 3 * V)
    g0n = 2.0 / (8 * 4 * V)
    g3n = 4.0 / (2.0 * 3 * 8 * 3 * V)
    zp = (num - 1) // 2
    g2 = np.zeros(num)
    g3 = np.zeros(num)
    for i in range(num):
        c = num - i - 1
        t = 0.0
        for mu in range(ND):
            t += np.trace(B[i, mu] @ B[c, mu]).real
        g2[i] = t * (g0n if i == zp else g2n)
        mom, psq = _psq(moms[i], dims)
        AA = sum(B[i, mu] @ B[c, mu] for mu in range(ND))
        Ar = sum(B[zp, mu] * mom[mu] for mu in range(ND))
        AP = sum(B[i, mu] * mom[mu] for mu in range(ND))
        AM = sum(B[c, mu] * (-mom[mu] / psq) for mu in range(ND))
        val = (np.trace(AA @ Ar) + np.trace(Ar @ AP @ AM)) / psq
        g3[i] = val.real * g3n
    return g2, g3


def measure(links, dims, dir=GLUON_PROPS, type=PSQ_CUT, max_mom=20, angle=0,
            cyl_width=1.0):
    """dict(mom, out0, out1, pspace_err) as GLU's cuts_struct computes
    them; out0/out1 = transverse/longitudinal, g2/g3, or for FIELDS the
    corrected fields (n, 4, 3, 3) and None."""
    moms, idx = veclist(dims, dir, type, max_mom, angle, cyl_width)
    A = momentum_fields(links, dims)
    B, err = correct_pspace(A, moms, idx, dims)
    if dir == GLUON_PROPS:
        o0, o1 = gluon_props(B, moms, dims)
    elif dir == FIELDS:
        o0, o1 = B, None
    else:
        o0, o1 = exceptional(B, moms, dims)
    return dict(mom=moms, idx=idx, out0=o0, out1=o1, pspace_err=err)
