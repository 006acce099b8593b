"""CPU restatement of GLU's momentum-space gluon measurements (CUTTYPE =
GLUON_PROPS, EXCEPTIONAL, FIELDS).  TEST INFRASTRUCTURE ONLY: the tests use
it as the checker of the GPU path; the product package never imports it.

Followed, in GLU's default build (SIN_MOM on, CUT_FORWARD off, CONDOR_MODE,
matrix contraction for the three-gluon vertex):

* lie fields       src/Matrix_Ops/exactQ.c:358-385 (Hermitian_proj, LINEAR),
                   exactQ.c:157-240 with evalues.c:136-202, 317-349 and
                   effs.c:63-95 (exact_log_slow, LOGARITHMIC)
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


def _sq_root(z, R):
    """GLU's squarert (evalues.c:136-143): the real part of the root only."""
    t = np.sqrt(np.abs(z)) * np.cos(np.angle(z) * 0.5)
    return np.where((np.conj(R) * t).real < 0, -t, t)


def _cube_root(z):
    return np.cbrt(np.abs(z)) * (np.cos(np.angle(z) / 3.0) + 1j * np.sin(np.angle(z) / 3.0))


def su3_eigenvalues(U):
    """Eigenvalues_suNC (evalues.c:317-349) with Eigenvalues_su3_stab
    (evalues.c:185-202) near the identity, for U (..., 3, 3)."""
    rr3 = 1j * 1.7320508075688772
    tr = U[..., 0, 0] + U[..., 1, 1] + U[..., 2, 2]
    # generic branch
    a = -tr / 3.0
    ca = np.conj(a)
    Q = a * a + ca
    R = a * (Q + ca * 0.5) - 0.5
    res = _sq_root(R * R - Q * Q * Q, R)
    A = -_cube_root(R + res)
    with np.errstate(all="ignore"):
        B = np.where(A != 0, Q / np.where(A != 0, A, 1), 0)
    plus, minus = A + B, rr3 * (A - B)
    z0, z1 = plus - a, (minus - plus) * 0.5 - a
    # near-identity branch
    a2 = 1.0 - tr / 3.0
    b2 = -np.conj(a2)
    p = b2 + a2 * (2.0 - a2)
    q = (a2 * (1.0 - b2 - a2 * 2.0 * (1.0 - a2 / 3.0)) + b2) * 1.5
    r2 = _sq_root(q * q + p * p * p, p)
    u1 = _cube_root(r2 - q)
    with np.errstate(all="ignore"):
        u2 = np.where(u1.real != 0, -p / np.where(u1 != 0, u1, 1), 0)
    plus2, minus2 = u1 + u2, rr3 * (u1 - u2)
    s0, s1 = 1.0 + plus2 - a2, 1.0 + 0.5 * (minus2 - plus2) - a2
    stab = 1.0 - tr.real / 3.0 < 1e-12
    return np.where(stab, s0, z0), np.where(stab, s1, z1)


def exact_log(U: np.ndarray) -> np.ndarray:
    """Q with U = exp(iQ), Q traceless Hermitian (exact_log_slow,
    exactQ.c:157-240, f-constants effs.c:63-95); zero where GLU's routine
    returns without writing (all phases equal)."""
    e0, e1 = su3_eigenvalues(U)
    z0, z1 = np.angle(e0), np.angle(e1)
    z2 = -(z0 - z1)
    u = 0.5 * z0
    w = z1 + u
    cw, cu, su = np.cos(w), np.cos(u), np.sin(u)
    one1 = cu - 1j * su
    two1 = np.conj(one1) ** 2
    uu, ww = u * u, w * w
    with np.errstate(all="ignore"):
        denom = 1.0 / (9.0 * uu - ww)
        E0 = np.where(np.abs(w) < 1e-13, 1 - ww / 6.0 * (1 - ww / 20.0 * (1 - ww / 42.0)),
                      np.sin(w) / np.where(w != 0, w, 1))
        f0 = ((uu - ww) * two1 + one1 * (8.0 * uu * cw + 1j * 2.0 * u * (3.0 * uu + ww) * E0)) * denom
        f1 = (2 * u * two1 - one1 * (2.0 * u * cw - 1j * (3.0 * uu - ww) * E0)) * denom
        f2 = (two1 - one1 * (cw + 3.0 * 1j * u * E0)) * denom
        con = np.conj(f2)
        mod = 1.0 / (f1.imag * f2.real - f1.real * f2.imag)
        imf = (f0.imag * f2.real - f0.real * f2.imag) * mod
    trce = -1j * mod / 2.0
    Qm = np.zeros_like(U)
    for a, b in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2)):
        Qm[..., a, b] = trce * (con * U[..., a, b] - f2 * np.conj(U[..., b, a]))
    Qm[..., 0, 0] -= imf
    Qm[..., 1, 1] -= imf
    for a, b in ((0, 1), (0, 2), (1, 2)):
        Qm[..., b, a] = np.conj(Qm[..., a, b])
    Qm[..., 2, 2] = -(Qm[..., 0, 0] + Qm[..., 1, 1])
    same = (z0 == z1) & (z1 == z2)
    Qm[same] = 0
    return Qm


def momentum_fields(links: np.ndarray, dims, definition=LINEAR_DEF) -> np.ndarray:
    """A_mu(p) = sum_x A_mu(x) e^{+ipx} for every p of the 0..2pi zone,
    (V, 4, 3, 3), site order x fastest."""
    Lx, Ly, Lz, Lt = (int(d) for d in dims)
    V = Lx * Ly * Lz * Lt
    U = np.asarray(links).reshape(V, 4, 3, 3)
    Q = exact_log(U) if definition == LOG_DEF else hermitian_proj(U)
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
            cyl_width=1.0, definition=LINEAR_DEF):
    """dict(mom, out0, out1, pspace_err) as GLU's cuts_struct computes
    them; out0/out1 = transverse/longitudinal, g2/g3, or for FIELDS the
    corrected fields (n, 4, 3, 3) and None."""
    moms, idx = veclist(dims, dir, type, max_mom, angle, cyl_width)
    A = momentum_fields(links, dims, definition)
    B, err = correct_pspace(A, moms, idx, dims)
    if dir == GLUON_PROPS:
        o0, o1 = gluon_props(B, moms, dims)
    elif dir == FIELDS:
        o0, o1 = B, None
    else:
        o0, o1 = exceptional(B, moms, dims)
    return dict(mom=moms, idx=idx, out0=o0, out1=o1, pspace_err=err)
