"""ctypes bindings for the checkers under oracle/ (TEST INFRASTRUCTURE ONLY).

* ``Oracle``  -- the C restatement (tc_oracle.c), runtime sizes, FP64 or FP32.
* ``RefLib``  -- the reference's own CPU path compiled into oracle/_ref/ by
  oracle/Makefile (compile-time sizes; present only where the reference
  sources were available at build time).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs import this module.  The product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

HW2, VV4, COLLOC = 0, 1, 2
VISC_CROSS, VISC_NAIVE, VISC_GALERKIN = 0, 1, 2

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class OrcParams(C.Structure):
    _fields_ = [
        ("scheme", C.c_int), ("visc_type", C.c_int), ("turb", C.c_int),
        ("stab_type", C.c_int), ("fd_mode", C.c_int),
        ("NX", C.c_int), ("NY", C.c_int), ("NZ", C.c_int),
        ("visc", C.c_double), ("sour_dpdx", C.c_double), ("inv_length_scale", C.c_double),
        ("xmin", C.c_double), ("ymin", C.c_double), ("hx", C.c_double), ("hy", C.c_double),
        ("area", C.c_double),
    ]


def build_oracle() -> None:
    """Compile liborc_f64.so / liborc_f32.so (make oracle)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


_LIBS: dict = {}


def _orc_lib(precision: str):
    name = "liborc_f64.so" if precision == "f64" else "liborc_f32.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build_oracle()
    L = C.CDLL(path)
    L.orc_create.restype = C.c_void_p
    L.orc_create.argtypes = [C.POINTER(OrcParams), _dp, C.POINTER(C.c_int)]
    L.orc_destroy.argtypes = [C.c_void_p]
    vp = C.c_void_p
    for fn in ("orc_set_level", "orc_get_level"):
        getattr(L, fn).argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p]
    L.orc_get_flux.argtypes = [vp, C.c_int, _dp]
    L.orc_set_nu_t.argtypes = [vp, _dp]
    L.orc_get_nu_t.argtypes = [vp, _dp]
    L.orc_get_mesh.argtypes = [vp, C.c_char_p, _dp]
    L.orc_get_mesh.restype = C.c_int
    for fn in ("orc_apply_gradient", "orc_apply_divergence", "orc_unapply_gradient", "orc_pressure_solve",
               "orc_explicit_term"):
        getattr(L, fn).argtypes = [vp, _dp, _dp]
    L.orc_normalize_pressure.argtypes = [vp, _dp]
    L.orc_flux_fd.argtypes = [vp, _dp, C.c_int, C.c_int, _dp]
    L.orc_recalc_turb_visc.argtypes = [vp, _dp]
    L.orc_step.argtypes = [vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double,
                           C.POINTER(C.c_double)]
    L.orc_step.restype = C.c_int
    L.orc_integral.argtypes = [vp, C.c_int, _dp]
    L.orc_kinetic_energy.argtypes = [vp, C.c_int]
    L.orc_kinetic_energy.restype = C.c_double
    L.orc_cfl.argtypes = [vp, C.c_int, C.c_double, C.c_int]
    L.orc_cfl.restype = C.c_double
    L.orc_profiles.argtypes = [vp, C.c_int, _dp]
    L.orc_init_channel.argtypes = [vp, C.c_int, C.c_ulonglong, C.c_double, C.c_int]
    L.orc_mt64_fill.argtypes = [C.c_ulonglong, C.c_int, np.ctypeslib.ndpointer(dtype=np.uint64)]
    L.orc_mesh_tanh.argtypes = [C.c_int, C.c_double, C.c_double, _dp]
    for fn in ("orc_check_gradient_kernel", "orc_check_normalization_projection", "orc_check_matrix_symmetry",
               "orc_check_pressure_matrix"):
        getattr(L, fn).argtypes = [vp]
        getattr(L, fn).restype = C.c_double
    L.orc_check_pressure_solver.argtypes = [vp, C.c_int]
    L.orc_check_pressure_solver.restype = C.c_double
    L.orc_check_conservation.argtypes = [vp, C.c_int, _dp]
    L.orc_check_conservation.restype = C.c_double
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_get_threads.restype = C.c_int
    L.orc_real_size.restype = C.c_int
    L.orc_fft.argtypes = [C.c_int, C.c_int, _dp]
    L.orc_fft.restype = C.c_int
    _LIBS[name] = L
    return L


def mesh_tanh(n: int, gamma: float, H: float = 1.0) -> np.ndarray:
    """z_j = H (1 + tanh(gamma (2j/n - 1)) / tanh(gamma)), j = 0..n."""
    z = np.zeros(n + 1)
    _orc_lib("f64").orc_mesh_tanh(n, gamma, H, z)
    return z


def mt64(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint64)
    _orc_lib("f64").orc_mt64_fill(seed, n, out)
    return out


def set_threads(n: int) -> None:
    _orc_lib("f64").orc_set_threads(n)
    _orc_lib("f32").orc_set_threads(n)


def get_threads() -> int:
    return _orc_lib("f64").orc_get_threads()


def fft(x: np.ndarray, sign: int = -1) -> np.ndarray:
    a = np.ascontiguousarray(np.stack([x.real, x.imag], -1).reshape(-1), dtype=np.float64)
    rc = _orc_lib("f64").orc_fft(len(x), sign, a)
    if rc:
        raise ValueError("length must be 2^a 3^b")
    return a[0::2] + 1j * a[1::2]


class Oracle:
    """CPU restatement of the reference solver object (one instance per case)."""

    def __init__(self, p: dict, zz: np.ndarray, precision: str = "f64"):
        self.L = _orc_lib(precision)
        self.p = dict(p)
        s = OrcParams()
        for k, _ in OrcParams._fields_:
            setattr(s, k, p.get(k, 0))
        err = C.c_int(0)
        self.h = self.L.orc_create(C.byref(s), np.ascontiguousarray(zz, dtype=np.float64), C.byref(err))
        if err.value:
            raise RuntimeError(f"orc_create failed ({err.value})")
        self.NX, self.NY, self.NZ = p["NX"], p["NY"], p["NZ"]
        self.N = self.NX * self.NY * self.NZ

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def mesh(self, name: str) -> np.ndarray:
        out = np.zeros(3 * self.NZ + 8)
        n = self.L.orc_get_mesh(self.h, name.encode(), out)
        return out[:n].copy()

    def set_level(self, l, vel=None, p=None):
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        q = None if p is None else np.ascontiguousarray(p, dtype=np.float64)
        self.L.orc_set_level(self.h, l, None if v is None else v.ctypes.data, None if q is None else q.ctypes.data)

    def get_level(self, l):
        v = np.zeros((self.N, 3))
        q = np.zeros(self.N)
        self.L.orc_get_level(self.h, l, v.ctypes.data, q.ctypes.data)
        return v, q

    def get_flux(self, l):
        f = np.zeros((self.N, 3))
        self.L.orc_get_flux(self.h, l, f.reshape(-1))
        return f

    def set_nu_t(self, nt):
        self.L.orc_set_nu_t(self.h, np.ascontiguousarray(nt, dtype=np.float64))

    def get_nu_t(self):
        nt = np.zeros(self.N)
        self.L.orc_get_nu_t(self.h, nt)
        return nt

    def _v2s(self, fn, v, n_out):
        out = np.zeros(n_out)
        getattr(self.L, fn)(self.h, np.ascontiguousarray(v, dtype=np.float64).reshape(-1), out)
        return out

    def apply_gradient(self, p):
        return self._v2s("orc_apply_gradient", p, 3 * self.N).reshape(self.N, 3)

    def apply_divergence(self, v):
        return self._v2s("orc_apply_divergence", v, self.N)

    def unapply_gradient(self, v):
        return self._v2s("orc_unapply_gradient", v, self.N)

    def pressure_solve(self, rhs):
        return self._v2s("orc_pressure_solve", rhs, self.N)

    def normalize_pressure(self, p):
        q = np.ascontiguousarray(p, dtype=np.float64).copy()
        self.L.orc_normalize_pressure(self.h, q)
        return q

    def explicit_term(self, v):
        return self._v2s("orc_explicit_term", v, 3 * self.N).reshape(self.N, 3)

    def flux_fd(self, v, do_conv, do_visc):
        out = np.zeros(3 * self.N)
        self.L.orc_flux_fd(self.h, np.ascontiguousarray(v, dtype=np.float64).reshape(-1), do_conv, do_visc, out)
        return out.reshape(self.N, 3)

    def recalc_turb_visc(self, v):
        self.L.orc_recalc_turb_visc(self.h, np.ascontiguousarray(v, dtype=np.float64).reshape(-1))

    def step(self, t, tau, cur, order, cfr=None):
        d = C.c_double(0.0)
        rc = self.L.orc_step(self.h, t, tau, cur, order, 0 if cfr is None else 1, 0.0 if cfr is None else cfr,
                             C.byref(d))
        if rc:
            raise ValueError("bad bdf order")
        return d.value

    def integral(self, l):
        out = np.zeros(3)
        self.L.orc_integral(self.h, l, out)
        return out

    def kinetic_energy(self, l):
        return self.L.orc_kinetic_energy(self.h, l)

    def cfl(self, l, tau, mode=3):
        return self.L.orc_cfl(self.h, l, tau, mode)

    def profiles(self, l):
        out = np.zeros(12 * self.NZ)
        self.L.orc_profiles(self.h, l, out)
        return out.reshape(self.NZ, 12)

    def init_channel(self, l, seed=12345, amp=0.1, project=True):
        self.L.orc_init_channel(self.h, l, seed, amp, 1 if project else 0)

    def check(self, name, *args):
        fn = getattr(self.L, "orc_check_" + name)
        return fn(self.h, *args)

    def check_conservation(self):
        K = np.zeros(3)
        ediv = self.L.orc_check_conservation(self.h, 1, K)
        return ediv, K


class RefLib:
    """The reference's own CPU solver (compiled from its sources by oracle/Makefile)."""

    def __init__(self, variant: str):
        path = os.path.join(REF_DIR, f"libref_{variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.L = L = C.CDLL(path)
        for fn in ("ref_kind", "ref_nx", "ref_ny", "ref_nzmax", "ref_conv", "ref_turb", "ref_visc_naive",
                   "ref_real_size"):
            getattr(L, fn).restype = C.c_int
        self.kind = L.ref_kind()
        self.NX, self.NY, self.NZMAX = L.ref_nx(), L.ref_ny(), L.ref_nzmax()
        L.ref_set_level.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        L.ref_get_level.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        L.ref_get_flux.argtypes = [C.c_int, _dp]
        L.ref_set_nu_t.argtypes = [_dp]
        L.ref_get_nu_t.argtypes = [_dp]
        L.ref_step.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int]
        for fn in ("ref_explicit_term", "ref_apply_gradient", "ref_apply_divergence", "ref_unapply_gradient",
                   "ref_pressure_solve"):
            getattr(L, fn).argtypes = [_dp, _dp]
        L.ref_normalize_pressure.argtypes = [_dp]
        L.ref_recalc_turb_visc.argtypes = [_dp]
        L.ref_integral.argtypes = [C.c_int, _dp]
        L.ref_kinetic_energy.argtypes = [C.c_int]
        L.ref_kinetic_energy.restype = C.c_double
        L.ref_cfl.argtypes = [C.c_int, C.c_double, C.c_int]
        L.ref_cfl.restype = C.c_double
        L.ref_profiles.argtypes = [C.c_int, _dp]
        L.ref_get_mesh.argtypes = [C.c_char_p, _dp]
        L.ref_get_mesh.restype = C.c_int
        L.ref_set_threads.argtypes = [C.c_int]
        if self.kind != 2:
            L.ref_cfr_shift.argtypes = [C.c_int, C.c_double]
            L.ref_project.argtypes = [C.c_int]
        self.NZ = None

    def setup(self, p: dict, zz: np.ndarray):
        zz = np.ascontiguousarray(zz, dtype=np.float64)
        if self.kind == 2:
            self.L.ref_setup_colloc.argtypes = [C.c_int, _dp] + [C.c_double] * 6 + [C.c_int] * 3
            rc = self.L.ref_setup_colloc(p["NZ"], zz, p["visc"], p["sour_dpdx"], p["inv_length_scale"], p["hx"],
                                         p["hy"], p["area"], p.get("turb", 0), p.get("stab_type", 0),
                                         p.get("fd_mode", 1))
        else:
            self.L.ref_setup.argtypes = [C.c_int, _dp] + [C.c_double] * 6
            rc = self.L.ref_setup(p["NZ"], zz, p["visc"], p["sour_dpdx"], p["inv_length_scale"], p["hx"], p["hy"],
                                  p["area"])
        if rc:
            raise RuntimeError("ref setup failed")
        self.NZ = p["NZ"]
        self.N = self.NX * self.NY * self.NZ

    def mesh(self, name):
        out = np.zeros(3 * self.NZ + 8)
        n = self.L.ref_get_mesh(name.encode(), out)
        return out[:n].copy()

    def set_level(self, l, vel=None, p=None):
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        q = None if p is None else np.ascontiguousarray(p, dtype=np.float64)
        self.L.ref_set_level(l, None if v is None else v.ctypes.data, None if q is None else q.ctypes.data)

    def get_level(self, l):
        v = np.zeros((self.N, 3))
        q = np.zeros(self.N)
        self.L.ref_get_level(l, v.ctypes.data, q.ctypes.data)
        return v, q

    def get_flux(self, l):
        f = np.zeros(3 * self.N)
        self.L.ref_get_flux(l, f)
        return f.reshape(self.N, 3)

    def set_nu_t(self, nt):
        self.L.ref_set_nu_t(np.ascontiguousarray(nt, dtype=np.float64))

    def get_nu_t(self):
        nt = np.zeros(self.N)
        self.L.ref_get_nu_t(nt)
        return nt

    def step(self, t, tau, cur, order, cfr=None):
        """The reference's data::Step; with cfr, then the oracle driver's constant flow
        rate shift of u (staggered builds only: ref_cfr_shift)."""
        self.L.ref_step(t, tau, cur, order)
        if cfr is not None:
            self.L.ref_cfr_shift((cur + 1) % 4, C.c_double(cfr))

    def project(self, l):
        """Level l made divergence-free with the reference's own operators (staggered)."""
        self.L.ref_project(l)

    def _v2s(self, fn, v, n):
        out = np.zeros(n)
        getattr(self.L, fn)(np.ascontiguousarray(v, dtype=np.float64).reshape(-1), out)
        return out

    def explicit_term(self, v):
        return self._v2s("ref_explicit_term", v, 3 * self.N).reshape(self.N, 3)

    def apply_gradient(self, p):
        return self._v2s("ref_apply_gradient", p, 3 * self.N).reshape(self.N, 3)

    def apply_divergence(self, v):
        return self._v2s("ref_apply_divergence", v, self.N)

    def unapply_gradient(self, v):
        return self._v2s("ref_unapply_gradient", v, self.N)

    def pressure_solve(self, rhs):
        return self._v2s("ref_pressure_solve", rhs, self.N)

    def normalize_pressure(self, p):
        q = np.ascontiguousarray(p, dtype=np.float64).copy()
        self.L.ref_normalize_pressure(q)
        return q

    def recalc_turb_visc(self, v):
        self.L.ref_recalc_turb_visc(np.ascontiguousarray(v, dtype=np.float64).reshape(-1))

    def integral(self, l):
        out = np.zeros(3)
        self.L.ref_integral(l, out)
        return out

    def kinetic_energy(self, l):
        return self.L.ref_kinetic_energy(l)

    def cfl(self, l, tau, mode=3):
        return self.L.ref_cfl(l, tau, mode)

    def profiles(self, l):
        out = np.zeros(12 * self.NZ)
        self.L.ref_profiles(l, out)
        return out.reshape(self.NZ, 12)


def ref_available(variant: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{variant}.so"))


def channel_params(scheme: int, NX: int, NY: int, NZ: int, Lx: float, Ly: float, Re_b: float, gamma: float,
                   visc_type: int | None = None, turb: int = 0, stab_type: int = 0, fd_mode: int = 1,
                   sour_dpdx: float | None = None, H: float = 1.0):
    """Parameters + wall-normal mesh for a channel of half-height H (walls at z=0, 2H).

    nu = 2H/Re_b (bulk velocity 1).  Staggered: NZ cells, NZ+1 faces; collocated:
    NZ nodes.  The length scale for y+ is u_tau/nu with u_tau estimated from
    Re_tau ~ 0.09 Re_b^0.88 (Pope), only used by the Smagorinsky damping.
    """
    visc = 2.0 * H / Re_b
    if visc_type is None:
        visc_type = (VISC_GALERKIN if turb else VISC_CROSS) if scheme == COLLOC else (VISC_NAIVE if turb else VISC_CROSS)
    re_tau = 0.09 * Re_b ** 0.88
    u_tau = re_tau * visc / H
    if sour_dpdx is None:
        sour_dpdx = u_tau * u_tau / H
    if scheme == COLLOC:
        zz = mesh_tanh(NZ - 1, gamma, H)
        area = Lx * Ly * (zz[-1] - zz[0])
    else:
        zz = mesh_tanh(NZ, gamma, H)
        area = Lx * Ly * (zz[-1] - zz[0])
    p = dict(scheme=scheme, visc_type=visc_type, turb=turb, stab_type=stab_type, fd_mode=fd_mode,
             NX=NX, NY=NY, NZ=NZ, visc=visc, sour_dpdx=sour_dpdx, inv_length_scale=u_tau / visc,
             xmin=0.0, ymin=0.0, hx=Lx / NX, hy=Ly / NY, area=area)
    return p, zz
