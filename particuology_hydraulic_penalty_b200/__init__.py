"""B200-native D3Q19 PSC-IMB lattice-Boltzmann step (sm_100a CUDA behind a C ABI).

Drop-in for the hot path of wangjianfttt/particuology_Hydraulic-penalty-
(src/lbm_dem/psc3d.py): ``PscD3Q19``, ``SparsePscD3Q19``, ``Particle3D`` and
the lattice constants keep the reference's names and call surface.
"""

from .psc3d import C, CS2, OPP, W, Particle3D, PscD3Q19, SparsePscD3Q19, equilibrium, guo_force

__all__ = ["C", "CS2", "OPP", "W", "Particle3D", "PscD3Q19", "SparsePscD3Q19", "equilibrium", "guo_force"]
