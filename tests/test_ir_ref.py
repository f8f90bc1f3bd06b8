"""The CPU restatement of the dipole derivatives (oracle/hessian_ref.py: central differences of the
fixed-origin dipole under the tightened SCF, the checker of pm3_rs.native.dipole_derivatives_batch)
pinned to the reference's tests: MOPAC's own central-differenced dipole for the PM3 water minimum
(tests/molecules.rs:495-541, 5e-5 e) and the translational sum rule sum_A d mu_b / d R_Aa = Q d_ab
(src/ir.rs:438-470) on a cation; and the intensity constant the reference derives (src/ir.rs:60-80)."""
import numpy as np

import hessian_ref
from helpers import A2B, parse
from pm3_rs import native

MOPAC_WATER = np.array([[-0.64523, 0.0, 0.0, 0.32262, 0.0, 0.0, 0.32262, 0.0, 0.0],
                        [0.0, -0.29722, 0.0, 0.0, 0.14861, 0.12714, 0.0, 0.14861, -0.12714],
                        [0.0, 0.0, -0.19191, 0.0, -0.00274, 0.09595, 0.0, 0.00274, 0.09595]])
WATER_MIN = "O 0.0 0.0 0.10030517; H 0.0 0.76783584 -0.46070259; H 0.0 -0.76783584 -0.46070259"
AMMONIUM = "N 0 0 0; H 0.63 0.63 0.63; H -0.63 -0.63 0.63; H -0.63 0.63 -0.63; H 0.63 -0.63 -0.63"


def test_restated_derivatives_match_mopac():
    z, x = parse(WATER_MIN)
    d = hessian_ref.dipole_derivatives(z, x * A2B)
    assert np.abs(d - MOPAC_WATER).max() < 5.0e-5
    assert abs(d[0, 0]) > 0.5


def test_restated_derivatives_obey_the_sum_rule():
    z, x = parse(AMMONIUM)
    d = hessian_ref.dipole_derivatives(z, x * A2B, charge=1.0)
    assert np.abs(d.reshape(3, -1, 3).sum(axis=1) - np.eye(3)).max() < 1.0e-6


def test_intensity_constant():
    assert abs(native.KM_PER_MOL_PER_E2_PER_AMU - 974.88) < 0.01
