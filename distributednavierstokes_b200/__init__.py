"""distributednavierstokes_b200: the single-GPU finite-volume time step of
DistributedNavierStokes as hand-written sm_100a CUDA kernels behind a C ABI
(include/dnsb.h, libdnsb.so), with a host-side mirror of the reference's
setup/solve API (api.py).
"""
from .api import (  # noqa: F401
    RK3, Ensemble, State, VectorField, channelprofiles, channelstats, cfl_timestep, divergence,
    energyspectrum, exchange_halo, imex_update, interior, kinetic_energy, logger, maxdiv,
    momentum, noise, poisson, pressuregrad_component, pressuregrad_update, project,
    random_field, rescale_shell, scalarfield, setup, shell_count, shell_energies, shellforcing,
    solve, spectrumstats, step, vectorfield, velocityfield,
)

from .les import (  # noqa: F401
    les_cube, lescells, lessampler, load_snapshot, save_snapshot, sfs_from_cube, sfs_sample,
)

from . import spectral, spectral_io  # noqa: F401,E402  (the pseudo-spectral solver)

__version__ = "0.1.0"
