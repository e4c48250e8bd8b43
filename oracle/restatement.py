"""ctypes bindings of the plain-C restatement (oracle/nz_oracle.c) -- TEST
INFRASTRUCTURE ONLY; used by tests/ as an independent checker."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libnzoracle.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        d, vp, i = C.c_double, C.c_void_p, C.c_int
        L.nzo_phase.restype = d
        L.nzo_phase.argtypes = [vp, d, d, d, vp, i, vp]
        L.nzo_rr2.argtypes = [i, vp, vp, d, d, i, vp]
        L.nzo_rr3_norm.restype = d
        L.nzo_rr3_norm.argtypes = [i, vp, vp, vp, d, d]
        L.nzo_wilson.argtypes = [vp, d, d, vp]
        L.nzo_lbc_viscosity.restype = d
        L.nzo_lbc_viscosity.argtypes = [vp, vp, d, d]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def phase(fluid, P, T, x, role, salinity=0.0):
    x = np.ascontiguousarray(x, dtype=np.float64)
    lnphi = np.zeros(fluid.nc)
    Z = lib().nzo_phase(C.byref(fluid), P, T, salinity, _p(x), int(role), _p(lnphi))
    return Z, lnphi


def rr2(z, K, init=0.5, tol=1e-12, maxit=80):
    z = np.ascontiguousarray(z, dtype=np.float64)
    K = np.ascontiguousarray(K, dtype=np.float64)
    b = C.c_double()
    ok = lib().nzo_rr2(z.size, _p(z), _p(K), init, tol, maxit, C.byref(b))
    return bool(ok), b.value


def rr3_norm(z, kg, kw, bg, bw):
    z, kg, kw = (np.ascontiguousarray(a, dtype=np.float64) for a in (z, kg, kw))
    return lib().nzo_rr3_norm(z.size, _p(z), _p(kg), _p(kw), bg, bw)


def lbc_viscosity(fluid, x, rho, T):
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().nzo_lbc_viscosity(C.byref(fluid), _p(x), rho, T)
