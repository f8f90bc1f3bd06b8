"""Spreading one batch over several GPUs (pm3_rs.sharding): the partition's balance and the gather
on CPU; the multi-device solve on one GPU with two contexts (the gather logic, not the scaling)."""
import numpy as np
import pytest

from helpers import A2B
from pm3_rs import _lib, native, sharding, workloads


def _batch(n, seed=11):
    mols = workloads.organic_batch(n, 5, 60, seed=seed)
    return workloads.pack(mols)


@pytest.fixture(scope="module")
def organics_4096():
    return _batch(4096)


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_partition_covers_every_molecule_once_and_balances_cost(parts, organics_4096):
    offs, z, _ = organics_4096
    P = sharding.partition(offs, z, parts)
    allm = np.concatenate(P)
    assert sorted(allm.tolist()) == list(range(4096))
    loads = sharding.part_loads(offs, z, P)
    # longest-processing-time rule: every part within one largest molecule of the mean
    largest = sharding.basis_sizes(offs, z).max() ** 3
    assert loads.max() - loads.min() <= largest
    assert loads.max() / loads.mean() < 1.01
    for p in P:
        assert np.all(np.diff(p) > 0)


def test_partition_of_uneven_sizes_and_empty_parts():
    mols = [workloads.organic(n, 3 + n) for n in (60, 5, 5, 5, 5)]
    offs, z, _ = workloads.pack(mols)
    P = sharding.partition(offs, z, 2)
    assert [0] in [p.tolist() for p in P]  # the one large molecule alone
    P = sharding.partition(offs, z, 8)  # more parts than molecules: some are empty
    assert sum(len(p) for p in P) == 5 and sum(len(p) == 0 for p in P) == 3
    with pytest.raises(ValueError):
        sharding.partition(offs, z, 0)


def test_gather_part_restores_the_molecules():
    offs, z, xyz = _batch(50)
    idx = np.array([3, 17, 42])
    so, sz, sx, atoms = sharding.gather_part(offs, z, xyz, idx)
    for j, m in enumerate(idx):
        assert np.array_equal(sz[so[j]:so[j + 1]], z[offs[m]:offs[m + 1]])
        assert np.array_equal(sx[so[j]:so[j + 1]], xyz[offs[m]:offs[m + 1]])
    assert len(atoms) == so[-1]


@pytest.mark.gpu
def test_batch_on_two_contexts_equals_one_batch():
    offs, z, xyz = _batch(96, seed=12)
    xyzb = xyz * A2B
    one = native.batch(offs, z, xyzb, native.options(), want_gradient=True)
    ctxs = [_lib.Context(0), _lib.Context(0)]
    try:
        two, parts = sharding.batch_on_devices(offs, z, xyzb, native.options(), devices=[0, 0], want_gradient=True,
                                               contexts=ctxs)
    finally:
        for c in ctxs:
            c.close()
    assert len(parts) == 2 and min(len(p) for p in parts) > 0
    # the per-CTA Fock build and the gradient kernel add per-atom terms with atomics, whose order
    # depends on scheduling: the two runs agree to rounding, not bit for bit (1e-8 eV/Bohr is
    # 4.4e-7 kcal/mol/A, below the 1e-6 kcal/mol/A parity bar)
    assert np.array_equal(one.status, two.status)
    assert np.abs(one.heat_of_formation_kcal - two.heat_of_formation_kcal).max() < 1e-9
    assert np.abs(one.charges - two.charges).max() < 1e-9
    assert np.abs(one.gradients - two.gradients).max() < 1e-8
