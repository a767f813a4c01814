"""turbchannel_b200 -- B200 (sm_100a) per-time-step path of TurbChannel's channel solvers.

The product is the C-ABI shared library ``libturbch_b200.so`` (declared in
include/turbch.h).  This module is a thin ctypes mirror of the reference's solver
object (``struct data``, staggered/data_global_inc.h:11-76): ``Solver.Step``,
``CalcIntegral``, ``CalcKineticEnergy``, ``CalcCFL``, ``CalcProfiles`` and the
operator methods the reference's CPU/GPU self-checks call.  There is no CPU
fallback: constructing a Solver without the CUDA library or without a GPU raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libturbch_b200.so")

HW2, VV4, COLLOC = 0, 1, 2
VISC_CROSS, VISC_NAIVE, VISC_GALERKIN = 0, 1, 2
FP64, MIXED = 0, 1
TURB_NONE, TURB_SMAGORINSKY, TURB_MLP = 0, 1, 2


class TcParams(C.Structure):
    _fields_ = [
        ("scheme", C.c_int), ("precision", C.c_int), ("visc_type", C.c_int), ("turb_model", C.c_int),
        ("NX", C.c_int), ("NY", C.c_int), ("NZ", C.c_int),
        ("stab_type", C.c_int), ("fd_mode", C.c_int), ("device", C.c_int),
        ("visc", C.c_double), ("sour_dpdx", C.c_double), ("inv_length_scale", C.c_double),
        ("xmin", C.c_double), ("ymin", C.c_double), ("hx", C.c_double), ("hy", C.c_double),
        ("area", C.c_double), ("low_modes", C.c_int),
    ]


# Every entry point declared in include/turbch.h.
EXPORTS = [
    "tc_last_error", "tc_version", "tc_create", "tc_destroy", "tc_upload_level", "tc_download_level",
    "tc_download_flux", "tc_device_level", "tc_get_stream", "tc_sync", "tc_step", "tc_set_forcing",
    "tc_last_dpdx", "tc_set_turb_model", "tc_integral", "tc_kinetic_energy", "tc_cfl", "tc_profiles",
    "tc_diagnostics", "tc_op_explicit_term", "tc_op_apply_gradient", "tc_op_apply_divergence",
    "tc_op_unapply_gradient", "tc_op_pressure_solve", "tc_op_turb_visc", "tc_set_nu_t", "tc_get_nu_t",
    "tc_init_channel", "tc_mesh_tanh", "tc_phase_timing", "tc_phase_times", "tc_launch_count",
    "tc_op_pressure_solve_static", "tc_set_diag_fusion", "tc_set_fft_fusion", "tc_set_flux_staging", "tc_checkpoint_save", "tc_checkpoint_load",
    "tc_stats_accumulate", "tc_stats_read", "tc_stats_reset", "tc_run_graph", "tc_pressure_solve_device",
    "tc_srk_init", "tc_srk_step",
]
# Every entry point declared in include/turbch_les.h (learned LES closure).
EXPORTS_LES = [
    "tc_les_filter", "tc_les_samples", "tc_mlp_create", "tc_mlp_destroy", "tc_mlp_get_params", "tc_mlp_set_params",
    "tc_mlp_set_data", "tc_mlp_train", "tc_mlp_grad", "tc_mlp_forward", "tc_set_mlp_fusion",
]
MLP_NPAR = 4673
NPHASE = 8
PHASES = ["turb", "flux", "div_xfft", "yfft", "zsolve", "iyfft", "ixfft", "correct"]

_lib = None


class TcError(RuntimeError):
    pass


def load_library(path: str = LIB_PATH):
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise TcError(f"{path} not found: build it with `python -m turbchannel_b200.build`")
    L = C.CDLL(path)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
    L.tc_last_error.restype = C.c_char_p
    L.tc_version.restype = C.c_char_p
    L.tc_create.argtypes = [C.POINTER(TcParams), dp, C.POINTER(vp)]
    L.tc_destroy.argtypes = [vp]
    L.tc_upload_level.argtypes = [vp, ip, vp, vp]
    L.tc_download_level.argtypes = [vp, ip, vp, vp]
    L.tc_download_flux.argtypes = [vp, ip, vp]
    L.tc_device_level.argtypes = [vp, ip, C.POINTER(vp), C.POINTER(vp)]
    L.tc_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.tc_sync.argtypes = [vp]
    L.tc_step.argtypes = [vp, C.c_double, C.c_double, ip, ip]
    L.tc_set_forcing.argtypes = [vp, ip, C.c_double]
    L.tc_last_dpdx.argtypes = [vp, dp]
    L.tc_checkpoint_save.argtypes = [vp, C.c_char_p, ip, C.c_double]
    L.tc_checkpoint_load.argtypes = [vp, C.c_char_p, C.POINTER(ip), dp]
    L.tc_stats_accumulate.argtypes = [vp, ip, C.c_double]
    L.tc_stats_read.argtypes = [vp, vp, dp]
    L.tc_stats_reset.argtypes = [vp]
    L.tc_pressure_solve_device.argtypes = [vp, vp, vp]
    L.tc_run_graph.argtypes = [vp, C.c_double, ip, ip, ip, ip, C.c_double, C.c_double, C.POINTER(ip), dp]
    L.tc_set_turb_model.argtypes = [vp, ip, vp]
    L.tc_integral.argtypes = [vp, ip, vp]
    L.tc_kinetic_energy.argtypes = [vp, ip, dp]
    L.tc_cfl.argtypes = [vp, ip, C.c_double, ip, dp]
    L.tc_profiles.argtypes = [vp, ip, vp]
    L.tc_diagnostics.argtypes = [vp, ip, C.c_double, vp, dp, vp]
    for fn in ("tc_op_explicit_term", "tc_op_apply_gradient", "tc_op_apply_divergence", "tc_op_unapply_gradient",
               "tc_op_pressure_solve", "tc_op_turb_visc", "tc_op_pressure_solve_static"):
        getattr(L, fn).argtypes = [vp, vp, vp]
    L.tc_set_nu_t.argtypes = [vp, vp]
    L.tc_get_nu_t.argtypes = [vp, vp]
    L.tc_init_channel.argtypes = [vp, ip, C.c_ulonglong, C.c_double, ip]
    L.tc_mesh_tanh.argtypes = [ip, C.c_double, C.c_double, vp]
    L.tc_mesh_tanh.restype = None
    L.tc_phase_timing.argtypes = [vp, ip]
    L.tc_phase_times.argtypes = [vp, vp, C.POINTER(C.c_int)]
    L.tc_launch_count.argtypes = [vp, C.POINTER(C.c_ulonglong)]
    L.tc_set_diag_fusion.argtypes = [vp, ip]
    L.tc_set_fft_fusion.argtypes = [vp, ip]
    L.tc_set_flux_staging.argtypes = [vp, ip]
    L.tc_set_mlp_fusion.argtypes = [vp, ip]
    L.tc_srk_init.argtypes = [vp, ip, ip, vp, vp, ip, C.c_double]
    L.tc_srk_step.argtypes = [vp, C.c_double, C.c_double]
    ll = C.c_longlong
    L.tc_les_filter.argtypes = [vp, ip, ip, ip, vp]
    L.tc_les_samples.argtypes = [vp, ip, ip, ip, vp, vp]
    L.tc_mlp_create.argtypes = [ip, C.c_ulonglong, C.POINTER(vp)]
    L.tc_mlp_destroy.argtypes = [vp]
    L.tc_mlp_get_params.argtypes = [vp, vp]
    L.tc_mlp_set_params.argtypes = [vp, vp]
    L.tc_mlp_set_data.argtypes = [vp, vp, vp, ll]
    L.tc_mlp_train.argtypes = [vp, ip, ll, C.c_float, vp]
    L.tc_mlp_grad.argtypes = [vp, vp, vp, ll, vp, C.POINTER(C.c_float)]
    L.tc_mlp_forward.argtypes = [vp, vp, ll, vp]
    _lib = L
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def mesh_tanh(n: int, gamma: float, H: float = 1.0) -> np.ndarray:
    z = np.zeros(n + 1)
    load_library().tc_mesh_tanh(n, gamma, H, _ptr(z))
    return z


class Solver:
    """One solver object (the reference's ``data``) on one GPU.

    ``p`` holds the fields of tc_params (scheme, precision, visc_type, turb_model,
    NX, NY, NZ, stab_type, fd_mode, device, visc, sour_dpdx, inv_length_scale, xmin,
    ymin, hx, hy, area, low_modes); ``zz`` the wall-normal coordinates.
    """

    def __init__(self, p: dict, zz: np.ndarray):
        self.L = load_library()
        s = TcParams()
        for k, _ in TcParams._fields_:
            setattr(s, k, p.get(k, 0))
        self.p = dict(p)
        self.NX, self.NY, self.NZ = p["NX"], p["NY"], p["NZ"]
        self.N = self.NX * self.NY * self.NZ
        zz = np.ascontiguousarray(zz, dtype=np.float64)
        h = C.c_void_p()
        self._check(self.L.tc_create(C.byref(s), zz.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h)))
        self.h = h

    def _check(self, rc: int):
        if rc != 0:
            raise TcError(f"turbch error {rc}: {self.L.tc_last_error().decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.L.tc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- ring levels ----
    def upload_level(self, level: int, vel=None, p=None):
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        q = None if p is None else np.ascontiguousarray(p, dtype=np.float64)
        self._check(self.L.tc_upload_level(self.h, level, None if v is None else _ptr(v), None if q is None else _ptr(q)))

    def download_level(self, level: int):
        v = np.zeros((self.N, 3))
        q = np.zeros(self.N)
        self._check(self.L.tc_download_level(self.h, level, _ptr(v), _ptr(q)))
        return v, q

    def download_flux(self, level: int):
        f = np.zeros((self.N, 3))
        self._check(self.L.tc_download_flux(self.h, level, _ptr(f)))
        return f

    def device_level(self, level: int):
        v, p = C.c_void_p(), C.c_void_p()
        self._check(self.L.tc_device_level(self.h, level, C.byref(v), C.byref(p)))
        return v.value, p.value

    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self.L.tc_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def sync(self):
        self._check(self.L.tc_sync(self.h))

    # ---- the step (data::Step) ----
    def Step(self, t: float, tau: float, current_field: int, bdf_order: int):
        self._check(self.L.tc_step(self.h, t, tau, current_field, bdf_order))

    def set_forcing(self, mode: int, value: float):
        self._check(self.L.tc_set_forcing(self.h, mode, value))

    def last_dpdx(self) -> float:
        d = C.c_double()
        self._check(self.L.tc_last_dpdx(self.h, C.byref(d)))
        return d.value

    def save_checkpoint(self, path: str, current_field: int, t: float):
        """All four ring levels and the forcing state, for an exact restart."""
        self._check(self.L.tc_checkpoint_save(self.h, os.fsencode(path), current_field, t))

    def pressure_solve_device(self, rhs_ptr: int, p_ptr: int):
        """The pressure solve on device buffers (addresses, working precision), asynchronous
        on the solver's stream."""
        self._check(self.L.tc_pressure_solve_device(self.h, rhs_ptr, p_ptr))

    def run_graph(self, tau: float, current_field: int, nsteps: int, check_every: int = 8, cfl_mode: int = 3,
                  cfl_min: float = 0.0, cfl_max: float = float("inf")):
        """Up to nsteps order-3 steps as one device-controlled CUDA graph (see tc_run_graph);
        returns (steps done, CFL number of the last check)."""
        n, c = C.c_int(), C.c_double()
        self._check(self.L.tc_run_graph(self.h, tau, current_field, nsteps, check_every, cfl_mode, cfl_min, cfl_max,
                                        C.byref(n), C.byref(c)))
        return n.value, c.value

    def stats_accumulate(self, level: int, weight: float = 1.0):
        """Adds weight x the per-plane means of `level` to the device accumulator (no sync)."""
        self._check(self.L.tc_stats_accumulate(self.h, level, weight))

    def stats_read(self):
        """Weighted time means of the profiles (NZ, 12) and the total weight."""
        out = np.zeros(self.NZ * 12)
        w = C.c_double()
        self._check(self.L.tc_stats_read(self.h, _ptr(out), C.byref(w)))
        return out.reshape(self.NZ, 12), w.value

    def stats_reset(self):
        self._check(self.L.tc_stats_reset(self.h))

    def load_checkpoint(self, path: str):
        """Restores a checkpoint of a solver with the same scheme, precision and grid;
        returns (current_field, t)."""
        cf, t = C.c_int(), C.c_double()
        self._check(self.L.tc_checkpoint_load(self.h, os.fsencode(path), C.byref(cf), C.byref(t)))
        return cf.value, t.value

    def set_turb_model(self, kind: int, weights=None):
        """kind TURB_NONE / TURB_SMAGORINSKY / TURB_MLP (weights: MLP_NPAR float parameters)."""
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        self._check(self.L.tc_set_turb_model(self.h, kind, None if w is None else _ptr(w)))

    def set_mlp_fusion(self, mode: int):
        """1: the learned closure is evaluated inside the flux kernel; 0: a separate pass."""
        self._check(self.L.tc_set_mlp_fusion(self.h, mode))

    # ---- learned closure: training data ----
    def les_filter(self, level: int, width: int = 4, width_z: int = 1):
        """Box filter (width cells in x and y, width_z in z): 10 fields [k][Z][Y][X]
        (u, v, w, p, uu, vv, ww, uv, uw, vw)."""
        M = (self.NX // width) * (self.NY // width) * (self.NZ // width_z)
        out = np.zeros(10 * M, dtype=np.float32)
        self._check(self.L.tc_les_filter(self.h, level, width, width_z, _ptr(out)))
        return out.reshape(10, self.NZ // width_z, self.NY // width, self.NX // width)

    def les_samples(self, level: int, width: int = 4, width_z: int = 1):
        """Closure training samples of the filtered level: features (M, 6), targets nu*/nu (M,)."""
        M = (self.NX // width) * (self.NY // width) * (self.NZ // width_z)
        X = np.zeros((M, 6), dtype=np.float32)
        Y = np.zeros(M, dtype=np.float32)
        self._check(self.L.tc_les_samples(self.h, level, width, width_z, _ptr(X), _ptr(Y)))
        return X, Y

    # ---- diagnostics ----
    def CalcIntegral(self, level: int):
        out = np.zeros(3)
        self._check(self.L.tc_integral(self.h, level, _ptr(out)))
        return out

    def CalcKineticEnergy(self, level: int) -> float:
        d = C.c_double()
        self._check(self.L.tc_kinetic_energy(self.h, level, C.byref(d)))
        return d.value

    def CalcCFL(self, level: int, tau: float, mode: int = 3) -> float:
        d = C.c_double()
        self._check(self.L.tc_cfl(self.h, level, tau, mode, C.byref(d)))
        return d.value

    def CalcProfiles(self, level: int):
        out = np.zeros((self.NZ, 12))
        self._check(self.L.tc_profiles(self.h, level, _ptr(out)))
        return out

    def diagnostics(self, level: int, tau: float):
        integral = np.zeros(3)
        prof = np.zeros((self.NZ, 12))
        cfl = C.c_double()
        self._check(self.L.tc_diagnostics(self.h, level, tau, _ptr(integral), C.byref(cfl), _ptr(prof)))
        return integral, cfl.value, prof

    # ---- operators ----
    def _op(self, fn, x, nout):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(nout)
        self._check(getattr(self.L, fn)(self.h, _ptr(x), _ptr(out)))
        return out

    def ExplicitTerm(self, v):
        return self._op("tc_op_explicit_term", v, 3 * self.N).reshape(self.N, 3)

    def ApplyGradient(self, p):
        return self._op("tc_op_apply_gradient", p, 3 * self.N).reshape(self.N, 3)

    def ApplyDivergence(self, v):
        return self._op("tc_op_apply_divergence", v, self.N)

    def UnapplyGradient(self, v):
        return self._op("tc_op_unapply_gradient", v, self.N)

    def LinearSystemSolveFFT(self, rhs):
        return self._op("tc_op_pressure_solve", rhs, self.N)

    def RecalcTurbVisc(self, v):
        return self._op("tc_op_turb_visc", v, self.N)

    def set_nu_t(self, nt):
        nt = np.ascontiguousarray(nt, dtype=np.float64)
        self._check(self.L.tc_set_nu_t(self.h, _ptr(nt)))

    def get_nu_t(self):
        out = np.zeros(self.N)
        self._check(self.L.tc_get_nu_t(self.h, _ptr(out)))
        return out

    def set_diag_fusion(self, mode: int):
        """0 (default): separate diagnostics pass, 1: fused into the step, 2: fused while read every step."""
        self._check(self.L.tc_set_diag_fusion(self.h, mode))

    def set_fft_fusion(self, mode: int):
        """1 (default): the x- and y-FFTs of a plane in one cluster kernel where the grid has one, 0: separate kernels."""
        self._check(self.L.tc_set_fft_fusion(self.h, mode))

    def set_flux_staging(self, mode: int):
        """Float flux kernel ring fill: 0 (default) cp.async chunks, 1 TMA tensor boxes on tiles whose halo does not wrap."""
        self._check(self.L.tc_set_flux_staging(self.h, mode))

    def srk_init(self, method, stab_type: int = 1, alpha_tau: float = None):
        """Set up the segregated IMEX Runge-Kutta step (collocated_SRK data::Step) with a
        method of turbchannel_b200.imex (or any object with kind, S, E, I); alpha_tau
        defaults to half the method's limit for the StabType, as the reference's driver
        sets it (collocated_SRK/main.cpp:351-352)."""
        if alpha_tau is None:
            alpha_tau = method.alpha_tau(stab_type)
        E = np.ascontiguousarray(method.E, dtype=np.float64)
        I = np.ascontiguousarray(method.I, dtype=np.float64)
        self._check(self.L.tc_srk_init(self.h, int(method.kind), int(method.S), _ptr(E), _ptr(I), int(stab_type),
                                       float(alpha_tau)))

    def srk_step(self, t: float, tau: float):
        """One SRK step of ring level 0 (velocity, pressure); dp/dt in level 1's pressure."""
        self._check(self.L.tc_srk_step(self.h, float(t), float(tau)))

    def phase_timing(self, on: bool):
        self._check(self.L.tc_phase_timing(self.h, 1 if on else 0))

    def phase_times(self):
        ms = np.zeros(NPHASE)
        n = C.c_int()
        self._check(self.L.tc_phase_times(self.h, _ptr(ms), C.byref(n)))
        return ms, n.value

    def launch_count(self) -> int:
        n = C.c_ulonglong()
        self._check(self.L.tc_launch_count(self.h, C.byref(n)))
        return n.value

    def init_channel(self, level: int, seed: int = 12345, amp: float = 0.1, project: bool = True):
        self._check(self.L.tc_init_channel(self.h, level, seed, amp, 1 if project else 0))


class Mlp:
    """The learned closure's network on one GPU (include/turbch_les.h): BF16 tensor-core
    training (Adam) and inference kernels of the library."""

    def __init__(self, seed: int = 12345, device: int = 0):
        self.L = load_library()
        h = C.c_void_p()
        self._check(self.L.tc_mlp_create(device, seed, C.byref(h)))
        self.h = h

    def _check(self, rc: int):
        if rc != 0:
            raise TcError(f"turbch error {rc}: {self.L.tc_last_error().decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.L.tc_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(MLP_NPAR, dtype=np.float32)
        self._check(self.L.tc_mlp_get_params(self.h, _ptr(p)))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == MLP_NPAR
        self._check(self.L.tc_mlp_set_params(self.h, _ptr(p)))

    def set_data(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        self._check(self.L.tc_mlp_set_data(self.h, _ptr(X), _ptr(Y), len(Y)))

    def train(self, epochs: int, batch: int, lr: float) -> np.ndarray:
        loss = np.zeros(epochs, dtype=np.float32)
        self._check(self.L.tc_mlp_train(self.h, epochs, batch, lr, _ptr(loss)))
        return loss

    def grad(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        g = np.zeros(MLP_NPAR, dtype=np.float32)
        loss = C.c_float()
        self._check(self.L.tc_mlp_grad(self.h, _ptr(X), _ptr(Y), len(Y), _ptr(g), C.byref(loss)))
        return g, loss.value

    def forward(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros(len(X), dtype=np.float32)
        self._check(self.L.tc_mlp_forward(self.h, _ptr(X), len(X), _ptr(out)))
        return out


def channel_params(scheme: int, NX: int, NY: int, NZ: int, Lx: float, Ly: float, Re_b: float, gamma: float,
                   precision: int = FP64, visc_type: int | None = None, turb: int = 0, stab_type: int = 0,
                   fd_mode: int = 1, sour_dpdx: float | None = None, H: float = 1.0, device: int = 0):
    """Channel of half-height H between walls z = 0 and 2H, bulk velocity 1.

    nu = 2H / Re_b.  Staggered: NZ cells (NZ+1 faces); collocated: NZ nodes.
    The y+ length scale used by the Smagorinsky damping is u_tau/nu with
    Re_tau ~ 0.09 Re_b^0.88; sour_dpdx defaults to u_tau^2/H.
    """
    visc = 2.0 * H / Re_b
    if visc_type is None:
        visc_type = (VISC_GALERKIN if turb else VISC_CROSS) if scheme == COLLOC else (VISC_NAIVE if turb else VISC_CROSS)
    re_tau = 0.09 * Re_b ** 0.88
    u_tau = re_tau * visc / H
    if sour_dpdx is None:
        sour_dpdx = u_tau * u_tau / H
    n_int = NZ - 1 if scheme == COLLOC else NZ
    zz = H * (1.0 + np.tanh(gamma * (2.0 * np.arange(n_int + 1) / n_int - 1.0)) / np.tanh(gamma))
    area = Lx * Ly * (zz[-1] - zz[0])
    p = dict(scheme=scheme, precision=precision, visc_type=visc_type, turb_model=turb, NX=NX, NY=NY, NZ=NZ,
             stab_type=stab_type, fd_mode=fd_mode, device=device, visc=visc, sour_dpdx=sour_dpdx,
             inv_length_scale=u_tau / visc, xmin=0.0, ymin=0.0, hx=Lx / NX, hy=Ly / NY, area=area, low_modes=0)
    return p, zz


def run_adaptive(S: "Solver", t: float, tau: float, current_field: int, nsteps: int, cfl_min: float, cfl_max: float,
                 check_every: int = 8, cfl_mode: int = 3):
    """The reference driver's loop with CFL-adaptive dt (staggered/main.cpp:308-370): after
    a change of tau the BDF order restarts at 1 (tc_step ramps it), then order-3 steps run
    as device-controlled graphs (Solver.run_graph) that stop on the device when the CFL
    number leaves [cfl_min, cfl_max]; the host then halves tau until the CFL estimate is
    below cfl_max, or enlarges it by 1.5 below cfl_min, as the reference does.
    Returns (t, tau, current_field) after nsteps steps."""
    done, order, cur = 0, 1, current_field
    while done < nsteps:
        if order < 3 or nsteps - done < check_every:
            S.Step(t, tau, cur, order)
            t += tau
            cur = (cur + 1) % 4
            done += 1
            order = min(order + 1, 3)
            continue
        n, cfl = S.run_graph(tau, cur, (nsteps - done) // check_every * check_every, check_every, cfl_mode,
                             cfl_min, cfl_max)
        done += n
        t += n * tau  # n is a multiple of 4: the ring is back at `cur`
        if not np.isfinite(cfl):
            raise TcError(f"run_adaptive: non-finite CFL number after step {done}")
        if cfl > cfl_max:
            while cfl > cfl_max:
                cfl *= 0.5
                tau *= 0.5
            order = 1
        elif cfl < cfl_min:
            tau *= 1.5
            order = 1
    return t, tau, cur
