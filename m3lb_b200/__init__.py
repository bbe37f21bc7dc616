"""B200-native lattice-Boltzmann step of M3LB (D2Q9/D3Q27, Esoteric Pull,
BGK / TRT / MRT / central moments, Guo forcing, halfway bounce-back).

The compute path is ``libm3lb.so`` (hand-written sm_100a CUDA behind the C
ABI of ``include/m3lb.h``); :mod:`m3lb_b200.solver` mirrors the reference's
solver API on top of it.
"""
from .solver import (BGK, D2Q9, D3Q27, MRT, TRT, CellType, CentralMoments, Domain,  # noqa: F401
                     EsotericPull, FluidSolver, Guo, HighOrderEquilibrium, MomentCollision,
                     NoForcing, NullCollision, ProductFormEquilibrium, RawPopulations,
                     SecondOrderEquilibrium, ShiftedPopulations, opp)

__all__ = ["BGK", "D2Q9", "D3Q27", "MRT", "TRT", "CellType", "CentralMoments", "Domain",
           "EsotericPull", "FluidSolver", "Guo", "HighOrderEquilibrium", "MomentCollision",
           "NoForcing", "NullCollision", "ProductFormEquilibrium", "RawPopulations",
           "SecondOrderEquilibrium", "ShiftedPopulations", "opp"]
