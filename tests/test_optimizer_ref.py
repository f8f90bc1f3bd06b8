"""The CPU restatement of the reference's geometry optimiser (oracle/lbfgs_ref.py, the checker of
pm3gpu_optimize_batch) pinned to the reference's own test (src/optimizer.rs:363-386): the
distorted water relaxes to dHf = -53.4330121104622 kcal/mol (the reference asserts 0.005; the
restatement lands within 1e-6), converged, with the energy below the start."""
import numpy as np

import lbfgs_ref
from helpers import A2B, parse
from pm3_rs import _lib


def test_restated_optimiser_reproduces_the_reference_water_relaxation():
    z, xyz = parse("O 0.0 0.0 0.0; H 1.05 0.0 0.0; H -0.30 1.02 0.0")
    r = lbfgs_ref.optimize(z, xyz * A2B)
    assert r["converged"] and r["max_gradient"] < 1.0e-3
    assert abs(r["heat_of_formation_kcal"] - (-53.4330121104622)) < 1.0e-6
    start = lbfgs_ref.O.single_point(z, xyz * A2B)["total_ev"]
    assert r["energy_ev"] < start


def test_optimize_batch_rejects_bad_arguments_without_a_device():
    L = _lib.load()
    offs = np.array([0, 3], np.int32)
    z = np.array([8, 1, 1], np.int32)
    x = np.zeros(9)
    out = (_lib.OptResult * 1)()
    I32, D = np.ctypeslib.ctypes.POINTER(np.ctypeslib.ctypes.c_int32), np.ctypeslib.ctypes.POINTER(np.ctypeslib.ctypes.c_double)
    assert L.pm3gpu_optimize_batch(None, 1, offs.ctypes.data_as(I32), z.ctypes.data_as(I32), x.ctypes.data_as(D),
                                   None, None, out, None) == _lib.INVALID_INPUT
    d = _lib.OptOptions()
    L.pm3gpu_default_opt_options(np.ctypeslib.ctypes.byref(d))
    assert (d.max_iter, d.gtol, d.history) == (200, 1.0e-3, 8)
