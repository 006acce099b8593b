"""glu_b200: GLU's Fourier-accelerated Landau/Coulomb gauge fixing on B200.

The compute path is libglu_gfix.so (hand-written sm_100a kernels behind the
C ABI of include/glu_gfix.h); this package is its host-side mirror of GLU's
interface.  See glu_b200.gfix.
"""
from .gfix import (FACG, FASD, SENTINEL, Coulomb, Coulomb_FA, Landau,  # noqa
                   av_plaquette, coulomb_fix, gauge_functional, landau_fix,
                   latt_reunitU, observables, theta_test_lin)

__all__ = ["FACG", "FASD", "Landau", "Coulomb", "Coulomb_FA", "SENTINEL",
           "landau_fix", "coulomb_fix", "observables", "theta_test_lin",
           "gauge_functional", "av_plaquette", "latt_reunitU"]
