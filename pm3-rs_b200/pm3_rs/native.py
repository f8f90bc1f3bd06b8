"""PM3 API of pm3-rs (atomic units out, Angstrom in), running on the pm3gpu CUDA library.

Drop-in for ``pm3_rs.native`` of pm3-rs (python/pm3_rs/native.py:41-140 and
src/python.rs:253-357): same functions, signatures, dictionary keys and units, and the same
``ValueError`` on any failure (src/python.rs:22-24). ``method`` is one of ``"pm3"``, ``"pm3-d3"``,
``"pm3-d3h4"`` and ``"pm3-d3h4x"``, each optionally with ``"+mmok"`` (the post-SCF corrections of
src/corrections/, added to the energy, heat of formation and gradient) and ``field`` is ``None``:
external fields are outside this library's path, and asking for one raises rather than being
silently ignored.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _lib

PM3_EV = 27.211386245988
PM3_A0 = 0.529177210903
EV_TO_HARTREE = 1.0 / PM3_EV
ANGSTROM_TO_BOHR = 1.0 / PM3_A0

_REFERENCES = {"auto": 0, "": 0, "rhf": 1, "r": 1, "restricted": 1, "uhf": 2, "u": 2, "unrestricted": 2}


def _parse_reference(reference: str) -> int:
    key = str(reference).lower()
    if key not in _REFERENCES:
        raise ValueError(f"reference must be 'auto', 'rhf' or 'uhf' (got {reference!r})")
    return _REFERENCES[key]


# corrections::Variant::parse (src/corrections/mod.rs:180-191) -> PM3GPU_VARIANT_*
_VARIANTS = {"": 0, "pm3": 0, "pm3-d3": 1, "pm3-d3h4": 2, "pm3-d3h4x": 3}


def _check_method(method: str, field) -> dict:
    """The method string as option fields, parsed as src/python.rs:48-65 does: ``variant``
    (PM3GPU_VARIANT_*) and ``mmok`` (a ``+mmok`` suffix: MOPAC's amide term)."""
    m = str(method).strip().lower().replace(" ", "-").replace("_", "-")
    mmok = m.endswith("+mmok")
    if mmok:
        m = m[:-len("+mmok")]
    if m not in _VARIANTS:
        raise ValueError(f"method must be 'pm3', 'pm3-d3', 'pm3-d3h4' or 'pm3-d3h4x', each optionally with a "
                         f"'+mmok' suffix (got {method!r})")
    if field is not None:
        raise ValueError("an external field is not available on pm3gpu")
    return {"variant": _VARIANTS[m], "mmok": int(mmok)}


def _as_arrays(numbers, positions):
    z = np.ascontiguousarray(np.asarray(numbers).reshape(-1), dtype=np.int32)
    xyz = np.asarray(positions, dtype=np.float64)
    if xyz.size != 3 * len(z):
        raise ValueError("numbers and positions length mismatch")
    return z, np.ascontiguousarray(xyz.reshape(len(z), 3) * ANGSTROM_TO_BOHR)


def options(charge: float = 0.0, multiplicity: int = 1, reference: str = "auto", **overrides) -> _lib.Options:
    """Pm3Options with the reference's defaults (src/scf.rs:259-287) and the given overrides."""
    lib = _lib.load()
    o = _lib.Options()
    lib.pm3gpu_default_options(ctypes.byref(o))
    o.charge = float(charge)
    o.multiplicity = int(multiplicity)
    o.reference = _parse_reference(reference)
    for k, v in overrides.items():
        setattr(o, k, v)
    return o


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def run(z, xyz_bohr, opts: _lib.Options, want_density=False, want_mo_energies=False, want_gradient=False,
        device: int = 0, context: _lib.Context | None = None) -> dict:
    """run_pm3 on one molecule (Bohr in, eV out). Raises ValueError on any non-OK status.
    `context` selects a context other than the device's default one (e.g. one given its own
    parameter set with pm3gpu_set_parameters)."""
    ctx = context if context is not None else _lib.default_context(device)
    lib = ctx.lib
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(len(z), 3)
    nao = ctypes.c_int()
    lib.pm3gpu_result_sizes(len(z), _ip(z), ctypes.byref(nao))
    n = max(nao.value, 0)
    res = _lib.Result()
    charges = np.zeros(len(z))
    dens = np.zeros((n, n)) if want_density else None
    eps = np.zeros(n) if want_mo_energies else None
    if want_gradient:
        grad = np.zeros((len(z), 3))
        rc = lib.pm3gpu_gradient(ctx.ptr, len(z), _ip(z), _dp(xyz), ctypes.byref(opts), ctypes.byref(res),
                                 _dp(charges), _dp(grad))
    else:
        grad = None
        rc = lib.pm3gpu_single_point(ctx.ptr, len(z), _ip(z), _dp(xyz), ctypes.byref(opts), ctypes.byref(res),
                                     _dp(charges), _dp(dens), _dp(eps))
    if rc != _lib.OK:
        raise ValueError(ctx.last_error() or f"pm3gpu status {rc}")
    out = {name: getattr(res, name) for name, _ in _lib.Result._fields_}
    out["dipole_debye"] = list(res.dipole_debye)
    out["homo_ev"] = res.homo_ev if res.has_homo else None
    out["lumo_ev"] = res.lumo_ev if res.has_lumo else None
    out["converged"] = bool(res.converged)
    out["unrestricted"] = bool(res.unrestricted)
    out["charges"] = charges
    if dens is not None:
        out["density"] = dens
    if eps is not None:
        out["mo_energies"] = eps
    if grad is not None:
        out["gradient"] = grad
    return out


def single_point(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
                 reference: str = "auto", method: str = "pm3", field=None) -> dict:
    """PM3 single-point energy and properties (python/pm3_rs/native.py:41-83).

    Positions in Angstrom. Returns ``energy_hartree``, ``energy_ev``, ``heat_of_formation_kcal``,
    ``electronic_ev``, ``core_ev``, ``charges`` (Mulliken, e), ``dipole_debye`` ([x, y, z]),
    ``homo_ev``, ``lumo_ev``, ``converged`` and ``unrestricted``.
    """
    mo = _check_method(method, field)
    z, xyz = _as_arrays(numbers, positions)
    r = run(z, xyz, options(charge, multiplicity, reference, **mo))
    return {
        "energy_hartree": r["total_ev"] * EV_TO_HARTREE,
        "energy_ev": r["total_ev"],
        "heat_of_formation_kcal": r["heat_of_formation_kcal"],
        "electronic_ev": r["electronic_ev"],
        "core_ev": r["core_ev"],
        "charges": [float(q) for q in r["charges"]],
        "dipole_debye": [float(v) for v in r["dipole_debye"]],
        "homo_ev": r["homo_ev"],
        "lumo_ev": r["lumo_ev"],
        "converged": r["converged"],
        "unrestricted": r["unrestricted"],
    }


def gradient(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
             reference: str = "auto", method: str = "pm3", field=None) -> dict:
    """Energy and analytic gradient dE/dR (src/python.rs:299-357): Hartree/Bohr and eV/Angstrom."""
    mo = _check_method(method, field)
    z, xyz = _as_arrays(numbers, positions)
    r = run(z, xyz, options(charge, multiplicity, reference, **mo), want_gradient=True)
    g = r["gradient"]
    return {
        "energy_hartree": r["total_ev"] * EV_TO_HARTREE,
        "energy_ev": r["total_ev"],
        "heat_of_formation_kcal": r["heat_of_formation_kcal"],
        "gradient_hartree_per_bohr": (g * EV_TO_HARTREE).tolist(),
        "gradient_ev_per_angstrom": (g * ANGSTROM_TO_BOHR).tolist(),
    }


def forces(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
           reference: str = "auto", method: str = "pm3", field=None) -> dict:
    """Energy and forces (= -gradient), Hartree/Bohr and eV/Angstrom."""
    g = gradient(numbers, positions, charge, multiplicity, reference, method, field)
    return {
        "energy_hartree": g["energy_hartree"],
        "energy_ev": g["energy_ev"],
        "heat_of_formation_kcal": g["heat_of_formation_kcal"],
        "forces_hartree_per_bohr": (-np.asarray(g["gradient_hartree_per_bohr"])).tolist(),
        "forces_ev_per_angstrom": (-np.asarray(g["gradient_ev_per_angstrom"])).tolist(),
    }


class BatchResult:
    """Column arrays of a batched solve (one row per molecule)."""

    def __init__(self, results, charges, gradients, offsets):
        self.raw = list(results)
        self.status = np.array([r.status for r in results], dtype=np.int32)
        self.heat_of_formation_kcal = np.array([r.heat_of_formation_kcal for r in results])
        self.total_ev = np.array([r.total_ev for r in results])
        self.electronic_ev = np.array([r.electronic_ev for r in results])
        self.core_ev = np.array([r.core_ev for r in results])
        self.dipole_debye = np.array([list(r.dipole_debye) for r in results]).reshape(-1, 3)
        self.homo_ev = np.array([r.homo_ev if r.has_homo else np.nan for r in results])
        self.lumo_ev = np.array([r.lumo_ev if r.has_lumo else np.nan for r in results])
        self.iterations = np.array([r.iterations for r in results], dtype=np.int32)
        self.converged = np.array([bool(r.converged) for r in results])
        self.unrestricted = np.array([bool(r.unrestricted) for r in results])
        self.scf_paths_tried = np.array([r.scf_paths_tried for r in results], dtype=np.int32)
        self.charges = charges
        self.gradients = gradients
        self.offsets = offsets

    def charges_of(self, m: int) -> np.ndarray:
        return self.charges[self.offsets[m]:self.offsets[m + 1]]


def batch(offsets, z, xyz_bohr, opts=None, want_gradient=False, device: int = 0,
          context: _lib.Context | None = None) -> BatchResult:
    """run_pm3 over many molecules in one persistent launch. Molecule m owns atoms
    [offsets[m], offsets[m+1]) of z / xyz_bohr (Bohr). ``opts``: one Options or a list.
    ``context``: a context other than the device's default one."""
    ctx = context if context is not None else _lib.default_context(device)
    lib = ctx.lib
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    n_mol = len(offsets) - 1
    if opts is None:
        opts = options()
    per_mol = isinstance(opts, (list, tuple))
    if per_mol:
        arr = (_lib.Options * n_mol)(*opts)
        optp = ctypes.cast(arr, ctypes.POINTER(_lib.Options))
    else:
        arr = opts
        optp = ctypes.pointer(opts)
    results = (_lib.Result * max(n_mol, 1))()
    charges = np.zeros(len(z))
    grads = np.zeros((len(z), 3)) if want_gradient else None
    rc = lib.pm3gpu_batch(ctx.ptr, n_mol, _ip(offsets), _ip(z), _dp(xyz), optp, int(per_mol), results,
                          _dp(charges), _dp(grads))
    if rc != _lib.OK:
        raise ValueError(ctx.last_error() or f"pm3gpu status {rc}")
    return BatchResult(list(results)[:n_mol], charges, grads, offsets)


def optimize_batch(offsets, z, xyz_bohr, opts=None, max_iter: int = 200, gtol: float = 1.0e-3, history: int = 8,
                   want_gradient: bool = False, device: int = 0, context: _lib.Context | None = None) -> dict:
    """Geometry optimisation of many molecules at once (pm3gpu_optimize_batch): the reference's
    L-BFGS (src/optimizer.rs:77-221) per molecule, each round one batched SCF + gradient launch over
    every molecule's pending geometry. Bohr in and out. Returns ``positions_bohr`` (final, packed
    like the input), ``status``, ``converged``, ``iterations``, ``evaluations``, ``energy_ev``,
    ``heat_of_formation_kcal``, ``max_gradient`` (eV/Bohr) per molecule, and ``gradients`` when
    asked for."""
    ctx = context if context is not None else _lib.default_context(device)
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    z = np.ascontiguousarray(z, dtype=np.int32)
    x = np.ascontiguousarray(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)).copy()
    n_mol = len(offsets) - 1
    o = opts if opts is not None else options()
    oo = _lib.OptOptions(int(max_iter), float(gtol), int(history))
    res = (_lib.OptResult * max(n_mol, 1))()
    g = np.zeros_like(x) if want_gradient else None
    rc = ctx.lib.pm3gpu_optimize_batch(ctx.ptr, n_mol, _ip(offsets), _ip(z), _dp(x), ctypes.byref(o), ctypes.byref(oo),
                                       res, _dp(g) if g is not None else None)
    if rc != 0:
        raise ValueError(ctx.last_error() or f"pm3gpu status {rc}")
    r = np.ctypeslib.as_array(res)[:n_mol]
    out = {"positions_bohr": x, "status": r["status"].copy(), "converged": r["converged"].astype(bool),
           "iterations": r["iterations"].copy(), "evaluations": r["evaluations"].copy(),
           "energy_ev": r["energy_ev"].copy(), "heat_of_formation_kcal": r["heat_of_formation_kcal"].copy(),
           "max_gradient": r["max_gradient"].copy()}
    if g is not None:
        out["gradients"] = g
    return out


def optimize(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
             reference: str = "auto", method: str = "pm3", field=None, max_steps: int = 200,
             force_tol=None) -> dict:
    """Geometry optimisation (src/python.rs:430-486): positions in Angstrom; ``force_tol`` in
    eV/Angstrom (None keeps OptOptions' 1e-3 eV/Bohr). Same keys as the reference:
    ``positions_angstrom`` / ``positions``, ``energy_hartree``, ``energy_ev``,
    ``heat_of_formation_kcal``, ``converged``, ``iterations`` / ``steps``."""
    mo = _check_method(method, field)
    z, xyz = _as_arrays(numbers, positions)
    gtol = 1.0e-3 if force_tol is None else float(force_tol) * PM3_A0
    r = optimize_batch([0, len(z)], z, xyz, options(charge, multiplicity, reference, **mo),
                       max_iter=max_steps, gtol=gtol)
    if r["status"][0] != 0:
        raise ValueError(_lib.default_context().last_error() or f"pm3gpu status {int(r['status'][0])}")
    coords = (r["positions_bohr"] * PM3_A0).tolist()
    return {
        "positions_angstrom": coords,
        "positions": coords,
        "energy_hartree": float(r["energy_ev"][0]) * EV_TO_HARTREE,
        "energy_ev": float(r["energy_ev"][0]),
        "heat_of_formation_kcal": float(r["heat_of_formation_kcal"][0]),
        "converged": bool(r["converged"][0]),
        "iterations": int(r["iterations"][0]),
        "steps": int(r["iterations"][0]),
    }


def numerical_hessian_batch(offsets, z, xyz_bohr, opts=None, step: float = 1.0e-3, device: int = 0,
                            context: _lib.Context | None = None) -> dict:
    """Cartesian Hessians of many molecules by central differences of the analytic gradient
    (pm3gpu_numerical_hessian_batch; the reference's numerical_hessian, src/hessian.rs:268-319):
    every displaced geometry of every molecule runs in the batched SCF + gradient launch. Bohr in;
    returns ``hessians`` (one (3n, 3n) array per molecule, eV/Bohr^2) and ``status``."""
    ctx = context if context is not None else _lib.default_context(device)
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    z = np.ascontiguousarray(z, dtype=np.int32)
    x = np.ascontiguousarray(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3))
    n_mol = len(offsets) - 1
    o = opts if opts is not None else options()
    nd = 3 * np.diff(offsets).astype(np.int64)
    hoff = np.concatenate([[0], np.cumsum(nd * nd)])
    flat = np.zeros(int(hoff[-1]))
    status = np.zeros(max(n_mol, 1), dtype=np.int32)
    rc = ctx.lib.pm3gpu_numerical_hessian_batch(ctx.ptr, n_mol, _ip(offsets), _ip(z), _dp(x), ctypes.byref(o),
                                                float(step), _dp(flat), _ip(status))
    if rc != 0:
        raise ValueError(ctx.last_error() or f"pm3gpu status {rc}")
    hs = [flat[hoff[m]:hoff[m + 1]].reshape(nd[m], nd[m]) for m in range(n_mol)]
    return {"hessians": hs, "status": status[:n_mol].copy()}


def numerical_hessian(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
                      reference: str = "auto", step: float = 1.0e-3, method: str = "pm3") -> np.ndarray:
    """One molecule's gradient-difference Hessian (eV/Bohr^2), positions in Angstrom, ``step`` in
    Bohr (src/hessian.rs:268-319)."""
    mo = _check_method(method, None)
    z, xyz = _as_arrays(numbers, positions)
    r = numerical_hessian_batch([0, len(z)], z, xyz, options(charge, multiplicity, reference, **mo),
                                step=step)
    if r["status"][0] != 0:
        raise ValueError(_lib.default_context().last_error() or f"pm3gpu status {int(r['status'][0])}")
    return r["hessians"][0]


def hessian(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
            reference: str = "auto", method: str = "pm3", field=None, cphf_max_iter=None) -> dict:
    """Cartesian Hessian (src/python.rs:693-739): same signature and keys
    (``hessian_hartree_per_bohr2`` row-major 3N x 3N lists, ``ndof``). Computed by central
    differences of the analytic gradient with a 1e-3 Bohr step (the reference's numerical_hessian,
    which its own tests hold to 5e-3 eV/Bohr^2 of the CPHF one); ``cphf_max_iter`` caps CPHF
    iterations, which this path does not run."""
    _check_method(method, field)
    h = numerical_hessian(numbers, positions, charge, multiplicity, reference, 1.0e-3, method)
    return {"hessian_hartree_per_bohr2": (h * EV_TO_HARTREE).tolist(), "ndof": int(h.shape[0])}


def atomic_masses(numbers: Sequence[int]) -> list:
    """Tabulated atomic masses (amu) of the parameter set, one per atom."""
    elems, _ = _lib.standard_parameters()
    table = {int(e.z): float(e.mass) for e in elems}
    out = []
    for zv in np.asarray(numbers).reshape(-1):
        if int(zv) not in table:
            raise ValueError(f"no PM3 parameters for Z={int(zv)} on pm3gpu")
        out.append(table[int(zv)])
    return out


def frequencies(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
                reference: str = "auto", method: str = "pm3", field=None, cphf_max_iter=None) -> dict:
    """Harmonic vibrational frequencies (src/python.rs:498-556): ``frequencies_cm``,
    ``eigenvalues``, ``modes`` (mass-weighted, one row per degree of freedom), ``masses``,
    ``n_rigid`` and ``rigid_residual_cm``, from the gradient-difference Hessian (see ``hessian``)."""
    from . import vibrations

    _check_method(method, field)
    h = numerical_hessian(numbers, positions, charge, multiplicity, reference, 1.0e-3, method)
    masses = atomic_masses(numbers)
    vib = vibrations.vibrational_analysis(h, np.asarray(positions, dtype=np.float64).reshape(-1, 3), masses)
    return {
        "frequencies_cm": vib["frequencies_cm"],
        "eigenvalues": vib["eigenvalues"],
        "modes": vib["modes"].tolist(),
        "masses": masses,
        "n_rigid": vib["n_rigid"],
        "rigid_residual_cm": vib["rigid_residual_cm"],
    }


def d3_batch(offsets, z, xyz_bohr, d3_set: int = 1, want_gradient: bool = True, device: int = 0,
             context: _lib.Context | None = None) -> dict:
    """The D3 dispersion correction alone (pm3gpu_d3_batch; src/corrections/d3.rs:360-458) for many
    molecules: ``energy_ev`` per molecule and ``gradient`` (eV/Bohr, packed like the input).
    ``d3_set`` 1 = the PM3-D3 parameters, 2 = the PM3-D3H4 ones."""
    ctx = context if context is not None else _lib.default_context(device)
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    z = np.ascontiguousarray(z, dtype=np.int32)
    x = np.ascontiguousarray(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3))
    n_mol = len(offsets) - 1
    e = np.zeros(max(n_mol, 1))
    g = np.zeros_like(x) if want_gradient else None
    rc = ctx.lib.pm3gpu_d3_batch(ctx.ptr, n_mol, _ip(offsets), _ip(z), _dp(x), int(d3_set), _dp(e),
                                 _dp(g) if g is not None else None)
    if rc != 0:
        raise ValueError(ctx.last_error() or f"pm3gpu status {rc}")
    out = {"energy_ev": e[:n_mol].copy()}
    if g is not None:
        out["gradient"] = g
    return out


def corrections_batch(offsets, z, xyz_bohr, method: str = "pm3-d3h4", want_gradient: bool = True, device: int = 0,
                      context: _lib.Context | None = None) -> dict:
    """The post-SCF correction of a method variant alone (pm3gpu_corrections_batch; the
    CorrectionEnergies of src/corrections/mod.rs:193-235) for many molecules: ``d3_ev``, ``h4_ev``,
    ``hh_ev``, ``hx_ev`` and ``total_ev`` per molecule, ``gradient`` (eV/Bohr) of the total."""
    mo = _check_method(method, None)
    variant = mo["variant"]
    if variant == 0 or mo["mmok"]:
        raise ValueError("corrections_batch takes 'pm3-d3', 'pm3-d3h4' or 'pm3-d3h4x' (no '+mmok')")
    ctx = context if context is not None else _lib.default_context(device)
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    z = np.ascontiguousarray(z, dtype=np.int32)
    x = np.ascontiguousarray(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3))
    n_mol = len(offsets) - 1
    parts = np.zeros((max(n_mol, 1), 4))
    g = np.zeros_like(x) if want_gradient else None
    rc = ctx.lib.pm3gpu_corrections_batch(ctx.ptr, n_mol, _ip(offsets), _ip(z), _dp(x), variant, _dp(parts),
                                          _dp(g) if g is not None else None)
    if rc != 0:
        raise ValueError(ctx.last_error() or f"pm3gpu status {rc}")
    p = parts[:n_mol]
    out = {"d3_ev": p[:, 0].copy(), "h4_ev": p[:, 1].copy(), "hh_ev": p[:, 2].copy(), "hx_ev": p[:, 3].copy(),
           "total_ev": p[:, 0] + p[:, 1] + p[:, 2] + p[:, 3]}
    if g is not None:
        out["gradient"] = g
    return out


AU_DIPOLE_TO_DEBYE = 2.541746473  # constants.rs:64
DEBYE_TO_E_ANGSTROM = 0.2081943  # src/python.rs:2049
# N_A |dmu/dQ|^2 / (12 eps0 c^2) with dmu/dQ in e / sqrt(amu), in km/mol (src/ir.rs:60-80)
KM_PER_MOL_PER_E2_PER_AMU = (6.02214076e23 * (1.602176634e-19 ** 2 / 1.66053906660e-27)
                             / (12.0 * 8.8541878128e-12 * 2.99792458e8 ** 2) / 1000.0)


def _tightened(o: _lib.Options) -> _lib.Options:
    """tighten_scf_for_hessian (src/hessian.rs:169-175) on a copy."""
    t = _lib.Options.from_buffer_copy(o)
    t.e_tol = min(t.e_tol, 1.0e-12)
    t.p_tol = min(t.p_tol, 1.0e-11)
    t.max_scf = max(t.max_scf, 500)
    return t


def dipole_derivatives_batch(offsets, z, xyz_bohr, opts=None, step: float = 1.0e-3, device: int = 0,
                             context: _lib.Context | None = None) -> dict:
    """d mu / d R (elementary charges, one 3 x 3N array per molecule) by central differences of the
    dipole about a fixed origin, every displaced geometry of every molecule in one batched SCF
    launch under the tightened SCF. The reference's dipole_derivatives (src/ir.rs:103-190) solves
    three coupled-perturbed equations instead; its own tests hold that tensor to exactly this
    difference (src/ir.rs:393-436). ``opts``: one Options or a list, one per molecule. The GPU
    reports the dipole about the centre of mass; mu_0 = mu_COM + Q R_COM restores the fixed origin.
    Returns ``derivatives`` and ``status`` (the first failing displacement's)."""
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    z = np.ascontiguousarray(z, dtype=np.int32)
    x = np.ascontiguousarray(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3))
    n_mol = len(offsets) - 1
    base = opts if opts is not None else options()
    per = list(base) if isinstance(base, (list, tuple)) else [base] * n_mol
    masses = np.asarray(atomic_masses(z)) if len(z) else np.zeros(0)
    geo_z, geo_x, geo_o, geo_off = [], [], [], [0]
    for m in range(n_mol):
        a0, a1 = int(offsets[m]), int(offsets[m + 1])
        t = _tightened(per[m])
        for j in range(3 * (a1 - a0)):
            for sign in (1.0, -1.0):
                xd = x[a0:a1].copy()
                xd[j // 3, j % 3] += sign * step
                geo_z.append(z[a0:a1])
                geo_x.append(xd)
                geo_o.append(t)
                geo_off.append(geo_off[-1] + (a1 - a0))
    out = [np.zeros((3, 3 * int(offsets[m + 1] - offsets[m]))) for m in range(n_mol)]
    status = np.zeros(n_mol, dtype=np.int32)
    if geo_o:
        r = batch(np.array(geo_off, np.int32), np.concatenate(geo_z), np.concatenate(geo_x), geo_o,
                  device=device, context=context)
        g = 0
        for m in range(n_mol):
            a0, a1 = int(offsets[m]), int(offsets[m + 1])
            mm = masses[a0:a1]
            q = float(per[m].charge)
            for j in range(3 * (a1 - a0)):
                mu = []
                for _ in range(2):
                    if status[m] == 0 and r.status[g] != 0:
                        status[m] = r.status[g]
                    xd = geo_x[g]
                    com = (mm[:, None] * xd).sum(axis=0) / mm.sum()
                    mu.append(r.dipole_debye[g] / AU_DIPOLE_TO_DEBYE + q * com)
                    g += 1
                out[m][:, j] = (mu[0] - mu[1]) / (2.0 * step)
    for m in range(n_mol):
        if status[m] != 0:
            out[m][:] = 0.0
    return {"derivatives": out, "status": status}


def dipole(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1, reference: str = "auto",
           method: str = "pm3", field=None, operator: bool = False) -> dict:
    """The dipole and its nuclear derivatives (src/python.rs:2016-2083): ``dipole_debye``,
    ``dipole_e_angstrom``, ``centre_of_mass_angstrom`` (the origin of both) and ``derivatives_e``
    (3 x 3N, fixed origin, elementary charges; from ``dipole_derivatives_batch``). The AO moment
    matrices (``operator=True``) are not available here."""
    if operator:
        raise ValueError("the dipole operator matrices (operator=True) are not available on pm3gpu")
    mo = _check_method(method, field)
    z, xyz = _as_arrays(numbers, positions)
    o = options(charge, multiplicity, reference, **mo)
    r = run(z, xyz, o)
    d = dipole_derivatives_batch([0, len(z)], z, xyz, o)
    if d["status"][0] != 0:
        raise ValueError(_lib.default_context().last_error() or f"pm3gpu status {int(d['status'][0])}")
    m = np.asarray(atomic_masses(z))
    com = (m[:, None] * xyz).sum(axis=0) / m.sum()
    mu = [float(v) for v in r["dipole_debye"]]
    return {
        "dipole_debye": mu,
        "dipole_e_angstrom": [v * DEBYE_TO_E_ANGSTROM for v in mu],
        "centre_of_mass_angstrom": (com * PM3_A0).tolist(),
        "derivatives_e": d["derivatives"][0].tolist(),
    }


def ir_spectrum(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
                reference: str = "auto", method: str = "pm3", field=None, cphf_max_iter=None) -> dict:
    """Infrared spectrum (src/ir.rs:284-345, src/python.rs:1952-2003): ``frequencies_cm``,
    ``intensities_km_per_mol`` (N_A |d mu / d Q|^2 / (12 eps0 c^2), the modes projected onto the
    internal subspace first), ``dipole_derivatives_e`` (3 x 3N) and ``ndof``. Frequencies from the
    gradient-difference Hessian (see ``hessian``), derivatives from ``dipole_derivatives_batch``;
    ``cphf_max_iter`` caps CPHF iterations, which this path does not run."""
    from . import vibrations

    mo = _check_method(method, field)
    z, xyz = _as_arrays(numbers, positions)
    o = options(charge, multiplicity, reference, **mo)
    r = numerical_hessian_batch([0, len(z)], z, xyz, o, step=1.0e-3)
    if r["status"][0] != 0:
        raise ValueError(_lib.default_context().last_error() or f"pm3gpu status {int(r['status'][0])}")
    d = dipole_derivatives_batch([0, len(z)], z, xyz, o)
    if d["status"][0] != 0:
        raise ValueError(_lib.default_context().last_error() or f"pm3gpu status {int(d['status'][0])}")
    masses = np.asarray(atomic_masses(z))
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    vib = vibrations.vibrational_analysis(r["hessians"][0], pos, masses)
    basis = vibrations.rigid_body_basis(pos, masses)
    modes = vib["modes"]
    proj = modes - (np.stack(basis, axis=1) @ (np.stack(basis, axis=1).T @ modes) if basis else 0.0)
    root = np.sqrt(np.repeat(masses, 3))
    inv = np.where(root > 0.0, 1.0 / np.where(root > 0.0, root, 1.0), 0.0)
    dmu = d["derivatives"][0]
    dq = dmu @ (proj * inv[:, None])  # 3 x modes
    inten = KM_PER_MOL_PER_E2_PER_AMU * (dq ** 2).sum(axis=0)
    return {
        "frequencies_cm": vib["frequencies_cm"],
        "intensities_km_per_mol": inten.tolist(),
        "dipole_derivatives_e": dmu.tolist(),
        "ndof": len(vib["frequencies_cm"]),
    }


def orbitals(numbers: Sequence[int], positions, charge: float = 0.0, multiplicity: int = 1,
             reference: str = "auto", method: str = "pm3", field=None) -> dict:
    """The reference's orbitals (src/python.rs:559-688) returns every MO coefficient of the last
    iteration. The device eigensolvers form only the occupied eigenvectors the density needs, so
    the coefficients do not exist here: this raises, naming what is available instead (all MO
    energies through ``run(..., want_mo_energies=True)``, the density through ``want_density``)."""
    raise ValueError("orbitals: MO coefficients are not exported by pm3gpu (the eigensolvers form only the "
                     "occupied vectors); MO energies and the density come from run(..., want_mo_energies=True, "
                     "want_density=True)")


def molden(*args, **kwargs):
    """The reference's Molden writer (src/python.rs:1021-1066) needs the MO coefficients; see
    ``orbitals``."""
    raise ValueError("molden: MO coefficients are not exported by pm3gpu; see orbitals()")
