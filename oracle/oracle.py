"""ctypes binding of the CPU oracle (test infrastructure only: tests/, smoke() and the CPU legs
of bench.py).  Exposes the same Context API as the product library under the prefix oracle_."""
import ctypes as C
import os

import numpy as np

from ice_fem_2025a_b200 import abi
from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.OUT
        if not os.path.exists(path):
            _build.build()
        _lib = C.CDLL(path)
        _lib.oracle_assemble_mt.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.Time), C.c_int32, C.c_int64,
                                            C.POINTER(C.c_double)]
    return _lib


class OracleContext(abi.Context):
    def assemble_nohist(self, step, t=0.0, dt=1.0, du_dt=0.0, ddu_dt=0.0):
        tm = abi.Time(t, dt, du_dt, ddu_dt)
        self._check(self.lib.oracle_assemble_nohist(self.h, step, C.byref(tm)))

    def assemble_mt(self, step, nthreads, n_sample=0, t=0.0, dt=1.0, du_dt=0.0, ddu_dt=0.0):
        tm = abi.Time(t, dt, du_dt, ddu_dt)
        ms = C.c_double()
        self._check(self.lib.oracle_assemble_mt(self.h, step, C.byref(tm), nthreads, n_sample, C.byref(ms)))
        return ms.value

    def set_options(self, opts):
        self._check(self.lib.oracle_set_options(self.h, C.byref(opts)))
        self.opts = opts

    def shape(self, el):
        nip = 9 if self.mesh.dim == 2 else 27
        nen = self.mesh.nen
        N = np.empty((nip, nen)); G = np.empty((nip, self.mesh.dim, nen)); w = np.empty(nip)
        dp = C.POINTER(C.c_double)
        self._check(self.lib.oracle_shape(self.h, C.c_int64(el), N.ctypes.data_as(dp), G.ctypes.data_as(dp),
                                          w.ctypes.data_as(dp)))
        return N, G, w


    def shape2(self, el):
        """N [nip][nen], G [nip][dim][nen], G2 [nip][3 or 6][nen] (getShapeGrads2) and the weights of an element."""
        nip = 9 if self.mesh.dim == 2 else 27
        nen, dim = self.mesh.nen, self.mesh.dim
        ng = 3 if dim == 2 else 6
        N = np.empty((nip, nen)); G = np.empty((nip, dim, nen)); G2 = np.empty((nip, ng, nen)); w = np.empty(nip)
        dp = C.POINTER(C.c_double)
        self._check(self.lib.oracle_shape2(self.h, C.c_int64(el), N.ctypes.data_as(dp), G.ctypes.data_as(dp),
                                           G2.ctypes.data_as(dp), w.ctypes.data_as(dp)))
        return N, G, G2, w

    def face_shapes(self, group, face):
        """N [nq][nfn], weights [nq] and outward normals [nq][3] of a TriAxial face (group 0 side, 1 top)."""
        dim = self.mesh.dim
        nq, nfn = (3, 3) if dim == 2 else (9, 9)
        N = np.empty((nq, nfn)); w = np.empty(nq); n = np.empty((nq, 3))
        dp = C.POINTER(C.c_double)
        self._check(self.lib.oracle_face_shapes(self.h, int(group), C.c_int64(face), N.ctypes.data_as(dp),
                                                w.ctypes.data_as(dp), n.ctypes.data_as(dp)))
        return N, w, n


def context(mesh, mats, opts, use_kron=True) -> OracleContext:
    return OracleContext(lib(), "oracle_", mesh, mats, opts, use_kron=use_kron)


def return_map(mat, T, eps, epl_old, epl, hist0, damage, dt, tol_mode=0, tangent_mode=0):
    """Single material-point return map (SolidMaterial.cpp:200-269)."""
    dp = C.POINTER(C.c_double)
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    epl_old = np.ascontiguousarray(epl_old, dtype=np.float64)
    epl = np.array(epl, dtype=np.float64)
    h = C.c_double(hist0)
    D = np.empty(36)
    it = C.c_int64()
    diss = C.c_double()
    rc = lib().oracle_return_map(C.byref(mat), C.c_double(T), eps.ctypes.data_as(dp), epl_old.ctypes.data_as(dp),
                                 epl.ctypes.data_as(dp), C.byref(h), C.c_double(damage), C.c_double(dt),
                                 tol_mode, tangent_mode, D.ctypes.data_as(dp), C.byref(it), C.byref(diss))
    if rc != 0:
        raise abi.IfemError(rc, "return map")
    return epl, h.value, D.reshape(6, 6), it.value, diss.value


def return_map_vep(mat, T, eps, epl_old, epl, hist, h_old, dt, tol_mode=0):
    """Single material-point VEP return map (SolidMaterial.cpp:303-445).  Returns (epl, hist[4], DMat,
    iterations, DissRate, DamDissRate, f, K) with f, K the local residual and Jacobian at the solution."""
    dp = C.POINTER(C.c_double)
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    epl_old = np.ascontiguousarray(epl_old, dtype=np.float64)
    epl = np.array(epl, dtype=np.float64)
    h = np.array(hist, dtype=np.float64)
    assert h.size == 4
    D, f, K = np.empty(36), np.empty(8), np.empty(64)
    it = C.c_int64()
    diss, dd = C.c_double(), C.c_double()
    rc = lib().oracle_return_map_vep(C.byref(mat), C.c_double(T), eps.ctypes.data_as(dp), epl_old.ctypes.data_as(dp),
                                     epl.ctypes.data_as(dp), h.ctypes.data_as(dp), C.c_double(h_old), C.c_double(dt),
                                     tol_mode, D.ctypes.data_as(dp), C.byref(it), C.byref(diss), C.byref(dd),
                                     f.ctypes.data_as(dp), K.ctypes.data_as(dp))
    if rc != 0:
        raise abi.IfemError(rc, "VEP return map")
    return epl, h, D.reshape(6, 6), it.value, diss.value, dd.value, f, K.reshape(8, 8)


def energy_split(mat, T, e):
    dp = C.POINTER(C.c_double)
    e = np.ascontiguousarray(e, dtype=np.float64)
    Dd, Du, Sd, Su = np.empty(36), np.empty(36), np.empty(6), np.empty(6)
    en = C.c_double()
    rc = lib().oracle_energy_split(C.byref(mat), C.c_double(T), e.ctypes.data_as(dp), Dd.ctypes.data_as(dp),
                                   Du.ctypes.data_as(dp), Sd.ctypes.data_as(dp), Su.ctypes.data_as(dp), C.byref(en))
    if rc != 0:
        raise abi.IfemError(rc, "energy split")
    return Dd.reshape(6, 6), Du.reshape(6, 6), Sd, Su, en.value
