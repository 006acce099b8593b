"""Seeded synthetic inputs with the shapes of the benchmark configurations.

GLU's benchmark inputs are heatbath configurations (beta 6.0, thousands of
sweeps) that take hours to generate on a CPU.  The stand-in used here keeps
their local value distribution exactly: the committed 8^4 GLU heatbath
configuration (beta 6.0, 500 sweeps, tests/golden/hb8.npz) is repeated
periodically to the requested extents (each a multiple of 8) and a seeded
random SU(3) gauge transformation is applied, so the solver starts from a
random point of the gauge orbit as GLU's RANDOM_TRANSFORM option does.
Plaquette and every gauge-invariant local observable equal those of the
heatbath configuration.

heatbath_config generates a genuine configuration of the requested extents
on the GPU with the library's heatbath (seconds at 32^3x64).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parents[1] / "tests" / "golden"


def base_config():
    g = np.load(GOLDEN / "hb8.npz")
    return g["links"].reshape(-1, 4, 3, 3), tuple(int(x) for x in g["dims"])


def random_su3(n: int, rng: np.random.Generator) -> np.ndarray:
    """n random SU(3) matrices: Gram-Schmidt of two Gaussian columns, third
    column the conjugate cross product."""
    z = rng.normal(size=(n, 3, 2)) + 1j * rng.normal(size=(n, 3, 2))
    c0 = z[:, :, 0] / np.linalg.norm(z[:, :, 0], axis=1, keepdims=True)
    c1 = z[:, :, 1] - np.sum(np.conj(c0) * z[:, :, 1], axis=1, keepdims=True) * c0
    c1 /= np.linalg.norm(c1, axis=1, keepdims=True)
    c2 = np.conj(np.cross(c0, c1))
    return np.stack([c0, c1, c2], axis=2)


def tiled_config(dims, seed: int = 2, transform: bool = True) -> np.ndarray:
    """Links of shape (V, 4, 3, 3) for dims (Lx, Ly, Lz, Lt)."""
    base, bd = base_config()
    Lx, Ly, Lz, Lt = (int(d) for d in dims)
    if any(L % b for L, b in zip((Lx, Ly, Lz, Lt), bd)):
        raise ValueError(f"extents {dims} must be multiples of {bd}")
    b = base.reshape(bd[3], bd[2], bd[1], bd[0], 4, 3, 3)
    t = np.tile(b, (Lt // bd[3], Lz // bd[2], Ly // bd[1], Lx // bd[0], 1, 1, 1))
    U = np.ascontiguousarray(t.reshape(-1, 4, 3, 3))
    if not transform:
        return U
    rng = np.random.default_rng(seed)
    V = U.shape[0]
    g = random_su3(V, rng).reshape(Lt, Lz, Ly, Lx, 3, 3)
    gd = np.conj(np.swapaxes(g, -1, -2))
    Ug = U.reshape(Lt, Lz, Ly, Lx, 4, 3, 3)
    out = np.empty_like(Ug)
    axis = {0: 3, 1: 2, 2: 1, 3: 0}
    for mu in range(4):
        gfwd = np.roll(gd, -1, axis=axis[mu])
        out[..., mu, :, :] = np.matmul(np.matmul(g, Ug[..., mu, :, :]), gfwd)
    return np.ascontiguousarray(out.reshape(-1, 4, 3, 3))


def _random_su3_torch(n: int, gen, device):
    """random_su3 on the device (torch), same construction."""
    import torch
    z = torch.randn((n, 3, 2), dtype=torch.complex128, generator=gen,
                    device=device)
    c0 = z[:, :, 0] / torch.linalg.vector_norm(z[:, :, 0], dim=1, keepdim=True)
    c1 = z[:, :, 1] - torch.sum(torch.conj(c0) * z[:, :, 1], dim=1,
                                keepdim=True) * c0
    c1 = c1 / torch.linalg.vector_norm(c1, dim=1, keepdim=True)
    c2 = torch.conj(torch.linalg.cross(c0, c1, dim=1))
    return torch.stack([c0, c1, c2], dim=2)


def tiled_config_device(dims, seed: int = 4, device="cuda"):
    """tiled_config built on the device (torch complex128, shape (V, 4, 3,
    3)), for lattices whose host-side construction would need tens of GB of
    host memory (64^3x128: 19.3 GB of links).  Seeded by a device generator:
    reproducible on the same GPU model, not bit-equal to the host version."""
    import torch
    base, bd = base_config()
    Lx, Ly, Lz, Lt = (int(d) for d in dims)
    if any(L % b for L, b in zip((Lx, Ly, Lz, Lt), bd)):
        raise ValueError(f"extents {dims} must be multiples of {bd}")
    b = torch.from_numpy(base.reshape(bd[3], bd[2], bd[1], bd[0], 4, 3, 3)).to(device)
    U = b.repeat(Lt // bd[3], Lz // bd[2], Ly // bd[1], Lx // bd[0], 1, 1, 1)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    V = Lx * Ly * Lz * Lt
    g = _random_su3_torch(V, gen, device).reshape(Lt, Lz, Ly, Lx, 3, 3)
    axis = {0: 3, 1: 2, 2: 1, 3: 0}
    for mu in range(4):
        gf = torch.roll(g, -1, dims=axis[mu]).conj().transpose(-1, -2)
        U[..., mu, :, :] = torch.matmul(torch.matmul(g, U[..., mu, :, :]), gf)
        del gf
    del g
    return U.reshape(V, 4, 3, 3)


def heatbath_config(dims, seed: int = 2, iterations: int = 1000, beta: float = 6.0,
                    n_or: int = 4) -> np.ndarray:
    """A heatbath configuration generated on the GPU (gfix_heatbath: GLU's
    hb_update algorithm, Kennedy-Pendleton heatbath plus n_or
    over-relaxation sweeps per iteration) from the unit start: the kind of
    input the benchmark configurations name (e.g. beta 6.0, 1000 sweeps).
    Reproducible for a given seed and build of the library."""
    import torch
    from .update import heatbath_device, unit_config
    d = torch.from_numpy(unit_config(dims).view(np.float64).reshape(-1).copy()).cuda()
    heatbath_device(d, dims, beta, iterations, n_or, seed=seed)
    return d.cpu().numpy().view(np.complex128).reshape(-1, 4, 3, 3)


def heatbath_config_device(dims, seed: int = 4, iterations: int = 200, beta: float = 6.0,
                           n_or: int = 4, device="cuda"):
    """A heatbath configuration generated on the GPU from the unit start
    without any host copy of the links (64^3x128 holds 19.3 GB of them):
    a device tensor of complex128, shape (V, 4, 3, 3).  The generator's own
    workspace is released afterwards."""
    import torch
    from . import _lib
    from .update import heatbath_device
    V = int(np.prod([int(d) for d in dims]))
    U = torch.zeros((V, 4, 3, 3), dtype=torch.complex128, device=device)
    for k in range(3):
        U[..., k, k] = 1.0
    heatbath_device(torch.view_as_real(U).reshape(-1), dims, beta, iterations, n_or,
                    seed=seed)
    _lib.load().gfix_update_release()
    return U
