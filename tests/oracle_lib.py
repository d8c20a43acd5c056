"""ctypes access to the oracle (test infrastructure only).

- ``oracle/liblbm_oracle.so``: this project's CPU restatement of the reference
  step (lbm_oracle.cpp), FP32 or FP64.
- ``oracle/_ref/libpoplar_ref.so``: the reference's own lbm_codelets.cpp run on
  the host through ref_poplar_emu.cpp (cavity, LES + MRT only); present only
  where the reference tree was available at build time.
- ``oracle/_ref/libkernelcu_ref.so``: the reference's own kernel.cu kernels,
  run on a GPU.
"""
import ctypes as C
import os

import numpy as np

from conftest import ROOT, load_package

pkg = load_package()
Inputval = pkg.Inputval

ORACLE_SO = os.path.join(ROOT, "oracle", "liblbm_oracle.so")
POPLAR_REF_SO = os.path.join(ROOT, "oracle", "_ref", "libpoplar_ref.so")
KERNELCU_REF_SO = os.path.join(ROOT, "oracle", "_ref", "libkernelcu_ref.so")


class Ext(C.Structure):
    _fields_ = [("init_kind", C.c_int), ("use_double", C.c_int), ("seed", C.c_uint64),
                ("noise_amp", C.c_float), ("split", C.c_int), ("threads", C.c_int)]


_libs = {}


def _load(path, prefix):
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    vp = C.c_void_p
    if prefix in ("orc", "ref"):
        getattr(L, prefix + "_create").restype = vp
        getattr(L, prefix + "_create").argtypes = [C.POINTER(Inputval), C.POINTER(Ext)]
        getattr(L, prefix + "_step").argtypes = [vp, C.c_int]
        getattr(L, prefix + "_get").argtypes = [vp] + [vp] * 9
        getattr(L, prefix + "_destroy").argtypes = [vp]
        if prefix == "orc":
            L.orc_set_solid.argtypes = [vp, vp]
        getattr(L, prefix + "_decomposition").argtypes = [C.POINTER(Inputval), vp]
        getattr(L, prefix + "_set_move_decomp").argtypes = [C.c_int, vp, vp]
        getattr(L, prefix + "_inverse_mrt").argtypes = [vp, vp]
        getattr(L, prefix + "_slice_chunk").argtypes = [C.c_uint, vp] + [C.POINTER(C.c_int)] * 10
    if prefix == "orc":
        L.orc_set_arF.argtypes = [vp, vp]
        L.orc_tables.argtypes = [vp, vp, vp, vp]
        L.orc_noise.restype = C.c_double
        L.orc_noise.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.orc_profile.restype = C.c_float
        L.orc_profile.argtypes = [C.c_float, C.c_int, C.c_int, C.c_int, C.c_int]
    if prefix == "kref":
        L.kref_run.argtypes = [C.POINTER(Inputval), C.POINTER(Ext), C.c_int] + [vp] * 5
        L.kref_run_solid.argtypes = ([C.POINTER(Inputval), C.POINTER(Ext), C.c_int, vp] +
                                     [vp] * 5)
        L.kref_save_file.argtypes = ([C.POINTER(Inputval)] + [vp] * 5 +
                                     [C.c_int, C.c_int, C.c_char_p])
    _libs[path] = L
    return L


def oracle_lib():
    L = _load(ORACLE_SO, "orc")
    if L is None:
        raise RuntimeError("oracle/liblbm_oracle.so missing: run __graft_entry__.build()")
    return L


def poplar_ref_lib():
    return _load(POPLAR_REF_SO, "ref")


def kernelcu_ref_lib():
    return _load(KERNELCU_REF_SO, "kref")


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Run:
    """A CPU run of the oracle port ('orc') or of the reference codelets ('ref')."""

    def __init__(self, iv, init_kind=0, seed=1, amp=0.0, double=False, split=1, threads=0,
                 which="orc"):
        self.L = oracle_lib() if which == "orc" else poplar_ref_lib()
        if self.L is None:
            raise RuntimeError("reference build not available")
        self.p = which
        self.ext = Ext(init_kind, 1 if double else 0, seed, amp, split, threads)
        self.iv = iv
        self.h = getattr(self.L, which + "_create")(C.byref(iv), C.byref(self.ext))
        if not self.h:
            raise RuntimeError(f"{which}_create failed")
        self.shape = (iv.ny, iv.nz, iv.nx)

    def step(self, n):
        assert getattr(self.L, self.p + "_step")(self.h, int(n)) == 0

    def fields(self):
        ny, nz, nx = self.shape
        N = nx * ny * nz
        f = np.empty(N * 19)
        d, ux, uy, uz, pd, te = (np.empty(N) for _ in range(6))
        nt = np.empty(N, np.int32)
        ds = np.empty(N, np.int32)
        getattr(self.L, self.p + "_get")(self.h, *[_p(a) for a in (f, d, ux, uy, uz, pd, te, nt, ds)])
        r = dict(arF=f.reshape(ny, nz, nx, 19), den=d, ux=ux, uy=uy, uz=uz, pden=pd, tau_e=te,
                 ntype=nt, dstate=ds)
        for k in ("den", "ux", "uy", "uz", "pden", "tau_e", "ntype", "dstate"):
            r[k] = r[k].reshape(ny, nz, nx)
        return r

    def set_arF(self, arF):
        a = np.ascontiguousarray(arF, np.float64)
        assert self.L.orc_set_arF(self.h, _p(a)) == 0

    def set_solid(self, mask):
        """Solid voxels [ny][nz][nx] (or None); restarts from the initial state."""
        m = None if mask is None else np.ascontiguousarray(np.asarray(mask) != 0, np.uint8)
        assert self.L.orc_set_solid(self.h, _p(m)) == 0

    def close(self):
        if self.h:
            getattr(self.L, self.p + "_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernelcu_run(iv, nsteps, init_kind=0, seed=1, amp=0.0, solid=None):
    """Run the reference's kernel.cu on the GPU; returns arF, den, ux, uy, uz.
    solid: optional [ny][nz][nx] voxels made NODE_STRUCT."""
    L = kernelcu_ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libkernelcu_ref.so not built")
    ext = Ext(init_kind, 0, seed, amp, 1, 0)
    ny, nz, nx = iv.ny, iv.nz, iv.nx
    arF = np.empty((ny, nz, nx, 19), np.float32)
    out = [np.empty((ny, nz, nx), np.float32) for _ in range(4)]
    m = None if solid is None else np.ascontiguousarray(np.asarray(solid) != 0, np.uint8)
    rc = L.kref_run_solid(C.byref(iv), C.byref(ext), int(nsteps), _p(m), _p(arF),
                          *[_p(a) for a in out])
    if rc != 0:
        raise RuntimeError(f"kref_run failed with CUDA error {rc}")
    return dict(arF=arF, den=out[0], ux=out[1], uy=out[2], uz=out[3])


def rel_vel_err(u, ref):
    """Velocity error relative to the velocity field's magnitude maximum:
    max over components of max|u_c - ref_c| / max|ref|.  Each of u, ref is a
    (ux, uy, uz) triple.  (A per-component normalisation is ill-posed for a
    component that is ~0 by symmetry, e.g. u_z in the cavity.)"""
    r = [np.asarray(c, np.float64) for c in ref]
    mag = np.sqrt(r[0] ** 2 + r[1] ** 2 + r[2] ** 2).max()
    mag = mag if mag > 0 else 1.0
    return float(max(np.abs(np.asarray(a, np.float64) - b).max() for a, b in zip(u, r)) / mag)


def rel_field_err(a, b):
    """max |a - b| / max |b| (pointwise relative error on u ~ 0 is ill-posed)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))
