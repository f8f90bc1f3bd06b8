"""ctypes front end of the CPU oracle (``oracle/liboracle.so``) -- TEST INFRASTRUCTURE ONLY.

The oracle restates pm3-rs's CPU algorithm for the molecular PM3 single point (see
``pm3_oracle.cpp``). tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use it as the checker; the product package never imports it.

Dense eigensolves and GEMMs go through LAPACK ``dsyevd`` / BLAS ``dgemm`` taken from SciPy's
public Cython interface (``scipy.linalg.cython_lapack`` / ``cython_blas``), i.e. the OpenBLAS
bundled with SciPy, so the CPU baseline stays in the performance class of the reference's faer.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

ANGSTROM_TO_BOHR = 1.0 / 0.529177210903
EV_TO_HARTREE = 1.0 / 27.211386245988


class Options(ctypes.Structure):
    _fields_ = [
        ("charge", ctypes.c_double),
        ("multiplicity", ctypes.c_int),
        ("max_scf", ctypes.c_int),
        ("e_tol", ctypes.c_double),
        ("p_tol", ctypes.c_double),
        ("use_diis", ctypes.c_int),
        ("accelerator", ctypes.c_int),
        ("adiis_switch", ctypes.c_double),
        ("reference", ctypes.c_int),
        ("guess", ctypes.c_int),
        ("stability", ctypes.c_int),
        ("level_shift_ev", ctypes.c_double),
        ("damping", ctypes.c_double),
        ("scf_memory_mb", ctypes.c_int),
        ("variant", ctypes.c_int),
        ("mmok", ctypes.c_int),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("electronic_ev", ctypes.c_double),
        ("core_ev", ctypes.c_double),
        ("total_ev", ctypes.c_double),
        ("heat_of_formation_kcal", ctypes.c_double),
        ("dipole_debye", ctypes.c_double * 3),
        ("homo_ev", ctypes.c_double),
        ("lumo_ev", ctypes.c_double),
        ("has_homo", ctypes.c_int),
        ("has_lumo", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("unrestricted", ctypes.c_int),
        ("scf_paths_tried", ctypes.c_int),
        ("scf_improvement_ev", ctypes.c_double),
        ("n_occ", ctypes.c_int),
        ("n_beta", ctypes.c_int),
        ("nao", ctypes.c_int),
        ("last_change", ctypes.c_double),
    ]


_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _capsule_ptr(module, name):
    capsule = module.__pyx_capi__[name]
    get = ctypes.pythonapi.PyCapsule_GetPointer
    get.restype = ctypes.c_void_p
    get.argtypes = [ctypes.py_object, ctypes.c_char_p]
    get_name = ctypes.pythonapi.PyCapsule_GetName
    get_name.restype = ctypes.c_char_p
    get_name.argtypes = [ctypes.py_object]
    return get(capsule, get_name(capsule))


def lib():
    """Load liboracle.so and hand it SciPy's LAPACK/BLAS entry points."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `make -C oracle` (or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    L.oracle_set_lapack.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.oracle_default_options.argtypes = [ctypes.POINTER(Options)]
    L.oracle_nao.argtypes = [ctypes.c_int, _I]
    L.oracle_single_point.argtypes = [ctypes.c_int, _I, _D, ctypes.POINTER(Options), ctypes.POINTER(Result), _D, _D,
                                      _D, _D, ctypes.c_char_p, ctypes.c_int]
    L.oracle_element.argtypes = [ctypes.c_int, _D]
    L.oracle_pair.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D, _I, _I]
    L.oracle_core_hamiltonian.argtypes = [ctypes.c_int, _I, _D, _D]
    L.oracle_fock.argtypes = [ctypes.c_int, _I, _D, _D, _D, _D]
    L.oracle_core_core.argtypes = [ctypes.c_int, _I, _D]
    L.oracle_core_core.restype = ctypes.c_double
    L.oracle_fixed_density_gradient.argtypes = [ctypes.c_int, _I, _D, _D, _D, _D, ctypes.c_int, _D]
    L.oracle_eigh.argtypes = [ctypes.c_int, _D, _D, _D]
    L.oracle_set_parameters.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    L.oracle_reset_parameters.argtypes = []
    L.oracle_reset_parameters.restype = None
    L.oracle_d3.argtypes = [ctypes.c_int, _I, _D, ctypes.c_int, _D, _D, _D]
    L.oracle_corrections.argtypes = [ctypes.c_int, _I, _D, ctypes.c_int, ctypes.c_int, _D, _D]
    L.oracle_d3_c6.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
    L.oracle_d3_c6.restype = ctypes.c_double
    try:
        import scipy.linalg.cython_blas as cb
        import scipy.linalg.cython_lapack as cl

        L.oracle_set_lapack(_capsule_ptr(cl, "dsyevd"), _capsule_ptr(cb, "dgemm"))
    except Exception:  # pragma: no cover - SciPy is in the image; Jacobi fallback otherwise
        L.oracle_set_lapack(None, None)
    _lib = L
    return L


def set_parameters(elems, pairs):
    """Run later calls with the given parameter set (run_pm3's &Pm3Parameters): ctypes arrays of
    structures with the layout of oracle_element_params / oracle_pair_params (the GPU library's
    pm3gpu_element / pm3gpu_pair have the same layout)."""
    rc = lib().oracle_set_parameters(ctypes.cast(elems, ctypes.c_void_p), len(elems),
                                     ctypes.cast(pairs, ctypes.c_void_p), len(pairs))
    if rc != 0:
        raise OracleError(1, "bad parameter set")


def reset_parameters():
    """Back to Pm3Parameters::standard()."""
    lib().oracle_reset_parameters()


def _ip(a):
    return a.ctypes.data_as(_I)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def options(**kw) -> Options:
    o = Options()
    lib().oracle_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def nao(z) -> int:
    z = np.ascontiguousarray(z, dtype=np.int32)
    return lib().oracle_nao(len(z), _ip(z))


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"oracle status {code}: {msg}")
        self.code = code


def cut_short(z, xyz_bohr, max_scf, **opts) -> dict:
    """run_pm3 stopped after `max_scf` SCF iterations (no stability search): the state the
    reference's loop leaves (src/scf.rs:1290-1316) -- the density of the last iteration, its
    electronic energy from a fresh Fock matrix and the RMS change of the last step."""
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    n_ao = nao(z)
    o = options(max_scf=max_scf, stability=0, **opts)
    r = Result()
    charges = np.zeros(len(z))
    dens = np.zeros((n_ao, n_ao))
    err = ctypes.create_string_buffer(512)
    code = lib().oracle_single_point(len(z), _ip(z), _dp(xyz), ctypes.byref(o), ctypes.byref(r), _dp(charges),
                                     _dp(dens), None, None, err, 512)
    if code not in (0, 4):
        raise OracleError(code, err.value.decode())
    return {"electronic_ev": r.electronic_ev, "last_change": r.last_change, "iterations": r.iterations,
            "converged": bool(r.converged), "density": dens}


def single_point(z, xyz_bohr, want_density=False, want_gradient=False, **opts) -> dict:
    """run_pm3 on one molecule (positions in Bohr); returns a dict of results (eV, Debye)."""
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    n_ao = nao(z)
    if n_ao < 0:
        raise OracleError(2, "missing element")
    o = options(**opts)
    r = Result()
    charges = np.zeros(len(z))
    dens = np.zeros((n_ao, n_ao)) if want_density else None
    eps = np.zeros(n_ao)
    grad = np.zeros((len(z), 3)) if want_gradient else None
    err = ctypes.create_string_buffer(512)
    code = lib().oracle_single_point(len(z), _ip(z), _dp(xyz), ctypes.byref(o), ctypes.byref(r), _dp(charges),
                                     _dp(dens), _dp(eps), _dp(grad), err, 512)
    if code != 0:
        raise OracleError(code, err.value.decode())
    out = {k: getattr(r, k) for k, _ in Result._fields_}
    out["dipole_debye"] = list(r.dipole_debye)
    out["homo_ev"] = r.homo_ev if r.has_homo else None
    out["lumo_ev"] = r.lumo_ev if r.has_lumo else None
    out["charges"] = charges
    out["mo_energies"] = eps
    if dens is not None:
        out["density"] = dens
    if grad is not None:
        out["gradient"] = grad
    return out


def element(zv: int) -> dict:
    out = np.zeros(22)
    if lib().oracle_element(zv, _dp(out)) != 0:
        raise OracleError(2, f"missing element {zv}")
    keys = ["n_orb", "uss", "upp", "zs", "zp", "betas", "betap", "gss", "gsp", "gpp", "gp2", "hsp", "alpha", "core",
            "dd", "qq", "rho0", "rho1", "rho2", "e_isol", "eheat_ev", "mass"]
    return dict(zip(keys, out.tolist()))


def pair(za: int, zb: int, dvec):
    dv = np.ascontiguousarray(dvec, dtype=np.float64)
    w = np.zeros(100)
    e1b = np.zeros(16)
    e2a = np.zeros(16)
    s = np.zeros(16)
    na = ctypes.c_int()
    nb = ctypes.c_int()
    code = lib().oracle_pair(za, zb, _dp(dv), _dp(w), _dp(e1b), _dp(e2a), _dp(s), ctypes.byref(na), ctypes.byref(nb))
    if code != 0:
        raise OracleError(code, "pair")
    pa = na.value * (na.value + 1) // 2
    pb = nb.value * (nb.value + 1) // 2
    return {"w": w[: pa * pb].reshape(pa, pb), "e1b": e1b.reshape(4, 4), "e2a": e2a.reshape(4, 4),
            "s": s.reshape(4, 4), "na": na.value, "nb": nb.value}


def core_hamiltonian(z, xyz_bohr):
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64)
    n = nao(z)
    h = np.zeros((n, n))
    code = lib().oracle_core_hamiltonian(len(z), _ip(z), _dp(xyz), _dp(h))
    if code != 0:
        raise OracleError(code, "core hamiltonian")
    return h


def fock(z, xyz_bohr, p_tot, p_spin=None):
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64)
    pt = np.ascontiguousarray(p_tot, dtype=np.float64)
    ps = np.ascontiguousarray(0.5 * pt if p_spin is None else p_spin, dtype=np.float64)
    f = np.zeros_like(pt)
    code = lib().oracle_fock(len(z), _ip(z), _dp(xyz), _dp(pt), _dp(ps), _dp(f))
    if code != 0:
        raise OracleError(code, "fock")
    return f


def core_core(z, xyz_bohr) -> float:
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64)
    return lib().oracle_core_core(len(z), _ip(z), _dp(xyz))


def fixed_density_gradient(z, xyz_bohr, p_tot, pa=None, pb=None):
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64)
    pt = np.ascontiguousarray(p_tot, dtype=np.float64)
    uhf = pa is not None
    pa_ = np.ascontiguousarray(pa if uhf else pt, dtype=np.float64)
    pb_ = np.ascontiguousarray(pb if uhf else pt, dtype=np.float64)
    g = np.zeros((len(z), 3))
    code = lib().oracle_fixed_density_gradient(len(z), _ip(z), _dp(xyz), _dp(pt), _dp(pa_), _dp(pb_), int(uhf), _dp(g))
    if code != 0:
        raise OracleError(code, "gradient")
    return g


def eigh(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n))
    if lib().oracle_eigh(n, _dp(a), _dp(w), _dp(v)) != 0:
        raise OracleError(5, "eigh")
    return w, v


def d3(z, xyz_bohr, d3_set=1, want_gradient=True):
    """D3 dispersion (src/corrections/d3.rs) of one molecule: (energy eV, gradient eV/Bohr [n, 3]
    or None, coordination numbers [n]). d3_set 1 = PM3-D3 parameters, 2 = the PM3-D3H4 ones."""
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    e = np.zeros(1)
    g = np.zeros((len(z), 3)) if want_gradient else None
    cn = np.zeros(len(z))
    code = lib().oracle_d3(len(z), _ip(z), _dp(xyz), int(d3_set), _dp(e), _dp(g), _dp(cn))
    if code != 0:
        raise OracleError(code, "d3")
    return float(e[0]), g, cn


def d3_c6(zi, zj, cni, cnj) -> float:
    return lib().oracle_d3_c6(int(zi), int(zj), float(cni), float(cnj))


def corrections(z, xyz_bohr, variant, want_gradient=True, mmok=False):
    """The post-SCF correction of a method variant (0 none, 1 PM3-D3, 2 PM3-D3H4, 3 PM3-D3H4X;
    src/corrections/mod.rs:78-160), with the MMOK amide term when ``mmok``: (dict of the D3 / H4 /
    H-H / X parts, plus "mmok" when asked for, in eV; gradient of their sum in eV/Bohr [n, 3] or
    None)."""
    z = np.ascontiguousarray(z, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    parts = np.zeros(5)
    g = np.zeros((len(z), 3)) if want_gradient else None
    code = lib().oracle_corrections(len(z), _ip(z), _dp(xyz), int(variant), int(bool(mmok)), _dp(parts), _dp(g))
    if code != 0:
        raise OracleError(code, "corrections")
    names = ("d3", "h4", "hh", "hx", "mmok") if mmok else ("d3", "h4", "hh", "hx")
    return dict(zip(names, parts.tolist())), g
