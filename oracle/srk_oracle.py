"""CPU restatement of the segregated IMEX Runge-Kutta step of the collocated scheme
(collocated_SRK/func_global.h:317-408, data::Step), in numpy over the collocated
operators of the C oracle (oracle_py.Oracle: explicit term, gradient, divergence +
pressure solve).

TEST INFRASTRUCTURE ONLY: the parity tests compare the product's tc_srk_step with this
restatement; nothing in the product imports it.

Differences from collocated_AB3 that the step needs, restated here:
  * the pressure normalisation of collocated_SRK/func_global.h:130-137 (shift
    sum(p vol) / area), applied on top of the oracle's AB3 normalisation (shift
    sum(p vol) hx hy / area); since sum(vol) = area the result is the SRK one;
  * the implicit part of the reference is empty (ImplicitTerm sets Ku = 0,
    ImplicitStage copies u*: func_global.h:310-315); it is kept literally here.
Vectors are (N, 3) arrays (the oracle's host layout), scalars (N,).
"""
from __future__ import annotations

import numpy as np

IMEX_A, IMEX_ARS, IMEX_CK = 0, 1, 2


def calc_d(S, A):
    """collocated_SRK/imex.cpp:37-46."""
    a_ss = A[S * S - 1]
    d = [1.0] + [0.0] * (S - 1)
    for j in range(1, S):
        for k in range(j):
            d[j] -= A[j * S + k] * d[k] / a_ss
    return d


class SrkOracle:
    def __init__(self, O, p: dict, zz: np.ndarray, kind: int, S: int, E, I, stab_type: int, alpha_tau: float):
        self.O = O
        self.kind, self.S = kind, S
        self.E, self.I = list(E), list(I)
        self.stab = stab_type
        self.alpha_tau = alpha_tau
        self.d = calc_d(S, self.I)
        NX, NY, NZ = p["NX"], p["NY"], p["NZ"]
        DZ = np.diff(np.asarray(zz, dtype=np.float64))
        cellh = np.empty(NZ)
        cellh[0] = 0.5 * DZ[0]
        cellh[NZ - 1] = 0.5 * DZ[NZ - 2]
        cellh[1:NZ - 1] = 0.5 * (DZ[:NZ - 2] + DZ[1:NZ - 1])
        self.vol = np.repeat(cellh * p["hx"] * p["hy"], NX * NY)  # GetCellVolume (func_global.h:116-128)
        self.area = p["area"]

    def unapply_gradient(self, v):
        """UnapplyGradient with the SRK normalisation (func_global.h:226-229, 130-137)."""
        q = self.O.unapply_gradient(v)
        return q - np.sum(q * self.vol) / self.area

    def step(self, tau, velocity, pressure, dpdt):
        """func_global.h:317-408; returns the new (velocity, pressure, dpdt)."""
        O, S, E, I = self.O, self.S, self.E, self.I
        velocity = np.array(velocity, dtype=np.float64)
        pressure = np.array(pressure, dtype=np.float64)
        dpdt = np.array(dpdt, dtype=np.float64)
        ass = I[S * S - 1]
        inv_ass = 1.0 / ass
        tau_stage = tau * ass
        inv_tau_stage = 1.0 / tau_stage
        alpha = self.alpha_tau / tau
        ck = self.kind == IMEX_CK
        zero_v = np.zeros_like(velocity)
        Ku = [zero_v.copy() for _ in range(S)]
        Kuhat = [zero_v.copy() for _ in range(S)]
        mujtilde = [np.zeros_like(pressure) for _ in range(S)]
        qj = [np.zeros_like(pressure) for _ in range(S)]
        pj = np.zeros_like(pressure)
        if self.kind in (IMEX_CK, IMEX_ARS):
            Kuhat[0] = O.explicit_term(velocity)
            gradp = O.apply_gradient(pressure)
            Ku[0] = zero_v.copy()
            Kuhat[0] = Kuhat[0] - gradp
        if ck:
            Ku[0] = zero_v.copy()  # ImplicitTerm
            nu1tilde = Ku[0] + Kuhat[0] + alpha * velocity
        j0 = 0 if self.kind == IMEX_A else 1
        for i in range(j0, S):
            buf = velocity.copy()
            for j in range(i):
                qi = tau * I[i * S + j]
                qe = tau * E[i * S + j]
                buf = buf + (qi * Ku[j] + qe * Kuhat[j])
            u = buf.copy()  # ImplicitStage
            Ku[i] = (u - buf) * inv_tau_stage
            Kuhat[i] = O.explicit_term(u)
            if self.stab == 0:
                pjhat = np.zeros_like(pressure)
                muj = pressure.copy()
                if ck:
                    muj = muj * (1.0 - self.alpha_tau * I[i * S])
                for j in range(j0, i):
                    muj = muj + inv_ass * I[i * S + j] * mujtilde[j]
                buf_s = muj - alpha * tau_stage * pressure
            else:
                muj = tau_stage * dpdt
                if ck:
                    muj = muj * (1.0 - self.alpha_tau * I[i * S])
                pjhat = pressure.copy()
                if ck:
                    pjhat = pjhat + tau * I[i * S] * dpdt
                for j in range(j0, i):
                    muj = muj + inv_ass * I[i * S + j] * mujtilde[j]
                    pjhat = pjhat + tau * I[i * S + j] * qj[j]
                buf_s = muj + pjhat - alpha * tau_stage * tau_stage * dpdt
            bufv = O.apply_gradient(buf_s)
            bufv = Ku[i] + Kuhat[i] - bufv + alpha * velocity
            if ck:
                bufv = bufv - self.d[i] * nu1tilde
            mujtilde[i] = self.unapply_gradient(bufv)
            pj = mujtilde[i] + buf_s
            mujtilde[i] = mujtilde[i] - alpha * tau_stage * (tau_stage * dpdt if self.stab else pressure)
            if self.stab:
                qj[i] = inv_tau_stage * (pj - pjhat)
            Kuhat[i] = Kuhat[i] - O.apply_gradient(pj)
        for j in range(S):
            qi = tau * I[S * S + j]
            qe = tau * E[S * S + j]
            velocity = velocity + (qi * Ku[j] + qe * Kuhat[j])
        pressure = pj
        if self.stab:
            dpdt = qj[S - 1]
        return velocity, pressure, dpdt


class RefSrk:
    """The reference's own collocated_SRK CPU solver (oracle/_ref/libref_srk_f64.so, built
    by `make -C oracle ref` from the read-only sources; x-y size fixed at the reference's
    NX = 128, NY = 64)."""

    def __init__(self, p: dict, zz, kind: int, S: int, E, I, stab_type: int, alpha_tau: float, threads: int = 0):
        import ctypes as C
        import os

        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_srk_f64.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        self.L.ref_srk_setup.argtypes = [C.c_int, dp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_int, C.c_int, dp, dp, C.c_int, C.c_double, C.c_int]
        self.L.ref_srk_set.argtypes = [dp, dp, dp]
        self.L.ref_srk_get.argtypes = [dp, dp, dp]
        self.L.ref_srk_step.argtypes = [C.c_double, C.c_double]
        if (p["NX"], p["NY"]) != (self.L.ref_srk_nx(), self.L.ref_srk_ny()):
            raise ValueError("the reference SRK build has NX, NY = %d, %d" % (self.L.ref_srk_nx(), self.L.ref_srk_ny()))
        self.N = p["NX"] * p["NY"] * p["NZ"]
        self._p = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(dp)
        self._keep = [np.ascontiguousarray(zz, dtype=np.float64), np.ascontiguousarray(E, dtype=np.float64),
                      np.ascontiguousarray(I, dtype=np.float64)]
        rc = self.L.ref_srk_setup(p["NZ"], self._keep[0].ctypes.data_as(dp), p["visc"], p["sour_dpdx"], p["hx"], p["hy"],
                                  p["area"], kind, S, self._keep[1].ctypes.data_as(dp), self._keep[2].ctypes.data_as(dp),
                                  stab_type, alpha_tau, threads)
        if rc:
            raise RuntimeError("ref_srk_setup failed")

    def step(self, t, tau, velocity, pressure, dpdt):
        v = np.ascontiguousarray(velocity, dtype=np.float64).reshape(-1).copy()
        p = np.ascontiguousarray(pressure, dtype=np.float64).copy()
        q = np.ascontiguousarray(dpdt, dtype=np.float64).copy()
        self.L.ref_srk_set(self._p(v), self._p(p), self._p(q))
        self.L.ref_srk_step(t, tau)
        import ctypes as C

        dp = C.POINTER(C.c_double)
        self.L.ref_srk_get(v.ctypes.data_as(dp), p.ctypes.data_as(dp), q.ctypes.data_as(dp))
        return v.reshape(self.N, 3), p, q
