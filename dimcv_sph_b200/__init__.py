"""B200-native DIMCV-SPH substep: neighbour grid, DFSPH, KVN/AKDE sampling and
Monte-Carlo VVPE as sm_100a CUDA kernels behind the reference's Python
operator surface (ParticleSystem / DIMCVSPHSolver / KarmanVortexSolver)."""
from .config_builder import SimConfig  # noqa: F401
from .params import Options, make_params  # noqa: F401

__version__ = "0.1.0"


def __getattr__(name):
    # the CUDA-backed classes import torch and load libdimcv lazily
    if name == "ParticleSystem":
        from .particle_system import ParticleSystem
        return ParticleSystem
    if name == "DIMCVSPHSolver":
        from .dimcv_sph import DIMCVSPHSolver
        return DIMCVSPHSolver
    if name == "KarmanVortexSolver":
        from .karman_vortex import KarmanVortexSolver
        return KarmanVortexSolver
    raise AttributeError(name)
