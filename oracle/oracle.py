"""ctypes binding of the CPU restatement (``liboracle.so``).

Test infrastructure only: tests, ``__graft_entry__.smoke`` and the CPU
baseline leg of ``bench.py`` use it as the checker.  The product package
(``vring_b200``) never imports it.

Arrays are exposed as numpy views in the reference's Fortran layouts
(column-major, theta fastest, reference ghost extents); index them as
``q1[i-1, j, k]`` for the Fortran element ``q1(i, j, k)`` of a field whose j and
k ranges start at 0.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

FIELDS = ["q1", "q2", "q3", "dq1", "dq2", "dq3", "ru1", "ru2", "ru3", "qrhs", "qcap",
          "pres", "prg", "rhs", "sol", "dph", "q1s", "q2s", "q3s", "dq3no", "corr1s",
          "corr2s", "corr3s", "corr3n", "csort", "tconv"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}


class Params(C.Structure):
    _fields_ = [("nth", C.c_int32), ("nr", C.c_int32), ("nz", C.c_int32),
                ("rmax", C.c_double), ("zmax", C.c_double), ("dt", C.c_double),
                ("re", C.c_double), ("pe", C.c_double), ("slip", C.c_double),
                ("wth_mode", C.c_int32), ("inflow_mode", C.c_int32), ("nthreads", C.c_int32)]


def build(force: bool = False) -> str:
    """Compile liboracle.so from vr_oracle.c with the committed Makefile."""
    src = os.path.join(_HERE, "vr_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, dp, i32, i64 = C.c_void_p, C.POINTER(C.c_double), C.c_int32, C.c_int64
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(Params)]
        L.orc_destroy.argtypes = [vp]
        L.orc_field.restype = dp
        L.orc_field.argtypes = [vp, i32, C.POINTER(C.c_int64)]
        L.orc_mesh.restype = dp
        L.orc_mesh.argtypes = [vp, i32]
        L.orc_coef.restype = dp
        L.orc_coef.argtypes = [vp, C.c_char_p]
        L.orc_set_clock.argtypes = [vp, i32, C.c_double, i64]
        L.orc_get_clock.argtypes = [vp, C.POINTER(i32), C.POINTER(C.c_double), C.POINTER(i64)]
        for n in ["ucoeff", "coesys", "hdnbc", "hdnl1", "hdnl2", "hdnl3", "step", "divq",
                  "upsol", "uppres", "laplace_solve"]:
            getattr(L, "orc_" + n).argtypes = [vp]
        L.orc_substep.argtypes = [vp, i32]
        L.orc_iterate.argtypes = [vp, i32]
        L.orc_solve_lap_thom.argtypes = [vp, vp, vp, vp, vp, i32]
        L.orc_solve_lap_par.argtypes = [vp, vp, vp, vp, vp, i32]
        L.orc_tripij.argtypes = [vp, vp, vp, vp, vp, i32, i32, i32, i32, i32]
        L.orc_solve_lap_bthom.argtypes = [vp, vp, vp, vp, vp, i32, i32]
        L.orc_fft_ptf.argtypes = [vp, vp, i32, i64]
        L.orc_fft_ftp.argtypes = [vp, vp, i32, i64]
        L.orc_fft_cos.argtypes = [vp, vp, i32, i32, i32]
        L.orc_vr_acos.restype = C.c_double
        L.orc_vr_acos.argtypes = [C.c_double]
        L.orc_part_create.restype = vp
        L.orc_part_create.argtypes = [vp, i32, i32, i32]
        L.orc_part_destroy.argtypes = [vp]
        L.orc_injc_part.restype = i32
        L.orc_injc_part.argtypes = [vp] + [C.c_double] * 7 + [i32]
        L.orc_remv_part.argtypes = [vp, i32]
        L.orc_iter_part.argtypes = [vp, vp, i32]
        L.orc_part_probe.argtypes = [vp, vp, C.c_double, C.c_double, C.c_double, vp]
        L.orc_part_cell.argtypes = [vp, C.c_double, C.c_double, C.c_double, vp, vp]
        L.orc_analysis.argtypes = [vp, i32, vp]
        L.orc_restart_save.restype = i32
        L.orc_restart_save.argtypes = [vp, C.c_char_p]
        L.orc_restart_load.restype = i32
        L.orc_restart_load.argtypes = [vp, C.c_char_p]
        L.orc_rng_uniform.restype = C.c_double
        L.orc_rng_uniform.argtypes = [C.POINTER(C.c_uint64)]
        L.orc_inlt_part.restype = i32
        L.orc_inlt_part.argtypes = [vp, vp, C.c_double, C.POINTER(C.c_uint64)]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """One single-rank run: mesh, fields, coefficient vectors and the clock."""

    def __init__(self, nth, nr, nz, rmax, zmax, dt, re, pe=1.0, slip=0.0, wth_mode=0,
                 inflow_mode=0, nthreads=0):
        self.params = Params(nth, nr, nz, rmax, zmax, dt, re, pe, slip, wth_mode, inflow_mode,
                             nthreads)
        self._h = lib().orc_create(C.byref(self.params))
        if not self._h:
            raise ValueError("oracle rejected the grid (need nth>=1, nr>=2, nz>=2)")
        self.nth, self.nr, self.nz = nth, nr, nz

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, name: str) -> np.ndarray:
        ext = (C.c_int64 * 4)()
        p = lib().orc_field(self._h, FIELD_ID[name], ext)
        shape = tuple(int(e) for e in ext)
        n = int(np.prod(shape))
        a = np.ctypeslib.as_array(p, shape=(n,)).reshape(shape, order="F")
        return a if shape[3] > 1 else a[..., 0]

    def mesh(self, which: str) -> np.ndarray:
        idx = {"rm": 0, "rc": 1, "zm": 2, "zc": 3, "thm": 4, "thc": 5}[which]
        n = {"rm": self.nr + 2, "rc": self.nr + 3, "zm": self.nz + 2, "zc": self.nz + 2,
             "thm": self.nth + 2, "thc": self.nth + 2}[which]
        return np.ctypeslib.as_array(lib().orc_mesh(self._h, idx), shape=(n,)).copy()

    def coef(self, name: str, n: int) -> np.ndarray:
        p = lib().orc_coef(self._h, name.encode())
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n,)).copy()

    def set_clock(self, irk: int, ntime: float, nstep: int = 0):
        lib().orc_set_clock(self._h, irk, ntime, nstep)

    def __getattr__(self, name):
        if name in ("ucoeff", "coesys", "hdnbc", "hdnl1", "hdnl2", "hdnl3", "step", "divq",
                    "upsol", "uppres", "laplace_solve"):
            fn = getattr(lib(), "orc_" + name)
            return lambda: fn(self._h)
        raise AttributeError(name)

    def substep(self, irk: int):
        lib().orc_substep(self._h, irk)

    def analysis(self, anlstp: int) -> np.ndarray:
        """analysis (run.F90:238-388): ntime, vortmax, swrlmax and the ten
        analysis.dat columns after them."""
        out = np.zeros(13)
        lib().orc_analysis(self._h, anlstp, _ptr(out))
        return out

    def restart_save(self, path: str) -> int:
        """restart_save (run.F90:390-460); 0 on success."""
        return lib().orc_restart_save(self._h, str(path).encode())

    def restart_load(self, path: str) -> int:
        """restart_load (run.F90:463-531); 0 on success, -2 on a grid mismatch."""
        return lib().orc_restart_load(self._h, str(path).encode())

    @property
    def clock(self):
        """(irk, ntime, nstep)"""
        irk, t, n = C.c_int32(), C.c_double(), C.c_int64()
        lib().orc_get_clock(self._h, C.byref(irk), C.byref(t), C.byref(n))
        return irk.value, t.value, n.value

    def iterate(self, nsteps: int):
        lib().orc_iterate(self._h, nsteps)


# ---- free-standing kernels -------------------------------------------------
def solve_lap_thom(rhs, aa, bb, cc):
    rhs, aa, bb, cc = (np.ascontiguousarray(x, dtype=np.float64) for x in (rhs, aa, bb, cc))
    sol = np.zeros_like(rhs)
    lib().orc_solve_lap_thom(_ptr(rhs), _ptr(sol), _ptr(aa), _ptr(bb), _ptr(cc), rhs.size)
    return sol


def solve_lap_par(rhs, aa, bb, cc):
    rhs, aa, bb, cc = (np.array(x, dtype=np.float64) for x in (rhs, aa, bb, cc))
    sol = np.zeros_like(rhs)
    lib().orc_solve_lap_par(_ptr(rhs), _ptr(sol), _ptr(aa), _ptr(bb), _ptr(cc), rhs.size)
    return sol


def tripij(ami, aci, api, fi):
    """Periodic solve of rows j (axis 0) over unknowns i (axis 1)."""
    nj, ni = fi.shape
    ld = nj + 1
    arrs = []
    for a in (ami, aci, api, fi, np.zeros_like(fi)):
        w = np.zeros((ld, ni + 1), order="F")
        w[1:, 1:] = a
        arrs.append(w)
    lib().orc_tripij(*[_ptr(w) for w in arrs], ld, 1, ni, 1, nj)
    return arrs[3][1:, 1:].copy()


def solve_lap_bthom(rhs, b1, b2, b3, m, n):
    rhs, b1, b2, b3 = (np.ascontiguousarray(x, dtype=np.float64) for x in (rhs, b1, b2, b3))
    sol = np.zeros_like(rhs)
    lib().orc_solve_lap_bthom(_ptr(rhs), _ptr(sol), _ptr(b1), _ptr(b2), _ptr(b3), m, n)
    return sol


def fft_ptf(a):
    """Packed forward real DFT along axis 0 of a Fortran-ordered array."""
    a = np.asfortranarray(a, dtype=np.float64)
    out = np.zeros_like(a, order="F")
    lib().orc_fft_ptf(_ptr(a), _ptr(out), a.shape[0], a.size // a.shape[0])
    return out


def fft_ftp(a):
    a = np.asfortranarray(a, dtype=np.float64)
    out = np.zeros_like(a, order="F")
    lib().orc_fft_ftp(_ptr(a), _ptr(out), a.shape[0], a.size // a.shape[0])
    return out


def fft_cos(a, direction):
    """DCT-II (+1, scaled 1/(2 nz)) / DCT-III (-1) along axis 1 of (nr, nz)."""
    a = np.asfortranarray(a, dtype=np.float64)
    out = np.zeros_like(a, order="F")
    lib().orc_fft_cos(_ptr(a), _ptr(out), a.shape[0], a.shape[1], direction)
    return out


def vr_acos(x: float) -> float:
    return lib().orc_vr_acos(float(x))


class OraclePart:
    """One particle class (part_tools.F90 type part) on an Oracle run."""

    def __init__(self, orc: Oracle, pid: int, naloc: int, mode: int = 0):
        class _P(C.Structure):
            _fields_ = [("id", C.c_int32), ("naloc", C.c_int32), ("nvar", C.c_int32),
                        ("nsubdt", C.c_int32), ("npart", C.c_int32), ("nlast", C.c_int32),
                        ("nfree", C.c_int32), ("nids", C.c_int32), ("r", C.c_double),
                        ("st", C.c_double), ("c", C.c_double),
                        ("u", C.POINTER(C.c_double)), ("v", C.POINTER(C.c_double)),
                        ("inflow", C.POINTER(C.c_double)),
                        ("isfre", C.POINTER(C.c_int32)), ("ifree", C.POINTER(C.c_int32)),
                        ("mode", C.c_int32), ("mint", C.POINTER(C.c_double)),
                        ("xint", C.POINTER(C.c_double))]
        self.orc = orc
        self._h = lib().orc_part_create(orc._h, pid, naloc, mode)
        self._s = C.cast(self._h, C.POINTER(_P)).contents
        self.naloc = naloc

    def close(self):
        if self._h:
            lib().orc_part_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def u(self):
        return np.ctypeslib.as_array(self._s.u, shape=(self.naloc * 117,)).reshape(
            (self.naloc, 117), order="F")

    @property
    def v(self):
        return np.ctypeslib.as_array(self._s.v, shape=(self.naloc * 3,)).reshape(
            (self.naloc, 3), order="F")

    @property
    def isfre(self):
        return np.ctypeslib.as_array(self._s.isfre, shape=(self.naloc + 1,))

    @property
    def mint(self):
        return np.ctypeslib.as_array(self._s.mint, shape=(9 * 27,)).reshape((9, 27), order="F")

    def __getattr__(self, name):
        if name in ("npart", "nlast", "nfree", "nsubdt", "st", "r", "c", "nids"):
            return getattr(self._s, name)
        raise AttributeError(name)

    def injc(self, x, y, z, u=0.0, v=0.0, w=0.0, c=None, icall=1):
        return lib().orc_injc_part(self._h, x, y, z, self._s.c if c is None else c, u, v, w,
                                   icall)

    def remv(self, ip):
        lib().orc_remv_part(self._h, ip)

    def iter_part(self, irk=1):
        lib().orc_iter_part(self.orc._h, self._h, irk)

    def inlt(self, r0, rng_state):
        """inlt_part (part_tools.F90:95-142); returns (injected, new rng state)."""
        st = C.c_uint64(rng_state)
        n = lib().orc_inlt_part(self.orc._h, self._h, r0, C.byref(st))
        return n, st.value

    @property
    def inflow(self):
        return np.ctypeslib.as_array(self._s.inflow, shape=(self.orc.nr + 2,))

    def probe(self, x, y, z):
        out = np.zeros(39)
        lib().orc_part_probe(self.orc._h, self._h, x, y, z, _ptr(out))
        return out

    def cell(self, x, y, z):
        idx = np.zeros(3, dtype=np.int32)
        th = np.zeros(1)
        lib().orc_part_cell(self.orc._h, x, y, z, _ptr(idx), _ptr(th))
        return idx, th[0]
