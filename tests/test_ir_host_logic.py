"""The host arithmetic of pm3_rs.native.dipole_derivatives_batch and ir_spectrum on the CPU: the
device calls (batch, numerical_hessian_batch) are replaced by the oracle, so the displaced-geometry
bookkeeping, the fixed-origin correction mu_0 = mu_COM + Q R_COM, the projection onto the internal
modes and the intensities are checked here against the restatement and the reference's pins."""
import numpy as np
import pytest

import hessian_ref
import oracle as O
from helpers import A2B, parse
from pm3_rs import native
from test_ir_ref import AMMONIUM, MOPAC_WATER, WATER_MIN


class _FakeBatch:
    def __init__(self, offsets, z, xyz, opts):
        self.status = []
        dip = []
        per = opts if isinstance(opts, (list, tuple)) else [opts] * (len(offsets) - 1)
        for m in range(len(offsets) - 1):
            a0, a1 = offsets[m], offsets[m + 1]
            o = per[m]
            r = O.single_point(z[a0:a1], xyz[a0:a1], charge=o.charge, multiplicity=o.multiplicity, e_tol=o.e_tol,
                               p_tol=o.p_tol, max_scf=o.max_scf)
            dip.append(r["dipole_debye"])
            self.status.append(0)
        self.status = np.array(self.status)
        self.dipole_debye = np.array(dip)


@pytest.fixture
def oracle_device(monkeypatch):
    monkeypatch.setattr(native, "batch", lambda offsets, z, xyz, opts=None, **kw: _FakeBatch(
        np.asarray(offsets), np.asarray(z), np.asarray(xyz).reshape(-1, 3), opts))

    def fake_hessian(offsets, z, xyz, opts=None, step=1.0e-3, **kw):
        offsets = np.asarray(offsets)
        xyz = np.asarray(xyz).reshape(-1, 3)
        hs = [hessian_ref.numerical_hessian(z[offsets[m]:offsets[m + 1]], xyz[offsets[m]:offsets[m + 1]], step=step,
                                            charge=opts.charge, multiplicity=opts.multiplicity)
              for m in range(len(offsets) - 1)]
        return {"hessians": hs, "status": np.zeros(len(hs), np.int32)}

    monkeypatch.setattr(native, "numerical_hessian_batch", fake_hessian)
    monkeypatch.setattr(native, "atomic_masses", lambda numbers: [O.element(int(v))["mass"] for v in numbers])


def test_derivative_bookkeeping_and_origin(oracle_device):
    cases = [(parse(WATER_MIN), 0.0), (parse(AMMONIUM), 1.0)]
    offs = np.array([0, 3, 8], np.int32)
    z = np.concatenate([c[0][0] for c in cases]).astype(np.int32)
    x = np.concatenate([c[0][1] for c in cases]) * A2B
    opts = [native.options(charge=q) for _, q in cases]
    d = native.dipole_derivatives_batch(offs, z, x, opts)
    assert (d["status"] == 0).all()
    assert np.abs(d["derivatives"][0] - MOPAC_WATER).max() < 5.0e-5
    ref = hessian_ref.dipole_derivatives(z[3:], x[3:], charge=1.0)
    assert np.abs(d["derivatives"][1] - ref).max() < 1e-12
    assert np.abs(d["derivatives"][1].reshape(3, -1, 3).sum(axis=1) - np.eye(3)).max() < 1e-6


def test_ir_spectrum_host_arithmetic(oracle_device):
    z, x = parse(WATER_MIN)
    ir = native.ir_spectrum(z, x)
    f = np.array(ir["frequencies_cm"])
    inten = np.array(ir["intensities_km_per_mol"])
    assert ir["ndof"] == 9 and np.count_nonzero(f == 0.0) == 6
    assert (inten[f != 0.0] > 0.1).all() and np.abs(inten[f == 0.0]).max() < 1e-6
    assert np.abs(np.array(ir["dipole_derivatives_e"]) - MOPAC_WATER).max() < 5.0e-5
