"""pm3_rs on B200: the molecular PM3 single point of pm3-rs, computed by the pm3gpu CUDA
library (sm_100a). Import-compatible with pm3-rs's ``pm3_rs`` for the single-point entry
points (``single_point``, ``gradient``, ``forces``), geometry optimisation (``optimize``) and the
Hessian and harmonic frequencies (``hessian``, ``frequencies``), plus batched forms (``batch``,
``optimize_batch``, ``numerical_hessian_batch``) for many molecules and ``batch_on_devices`` to
spread one batch over several GPUs."""
from .native import (ANGSTROM_TO_BOHR, EV_TO_HARTREE, BatchResult, batch, dipole, dipole_derivatives_batch, forces,
                     frequencies, gradient, hessian, ir_spectrum, numerical_hessian, numerical_hessian_batch, optimize,
                     optimize_batch, options, run, single_point)
from .sharding import batch_on_devices, partition

__all__ = ["single_point", "gradient", "forces", "batch", "batch_on_devices", "partition", "run", "options",
           "optimize", "optimize_batch", "hessian", "frequencies", "numerical_hessian", "numerical_hessian_batch",
           "dipole", "ir_spectrum", "dipole_derivatives_batch",
           "BatchResult", "ANGSTROM_TO_BOHR", "EV_TO_HARTREE"]
