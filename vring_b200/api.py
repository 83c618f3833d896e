"""ctypes binding of ``lib/libvring_b200.so`` and the host-side mirror of the
reference's subroutine surface.

``Run`` stands for the reference's ``type(run) :: var`` (run.F90:14-22): it
owns one device context and exposes the routines of the RK3 core under the
reference's names (``ucoeff``, ``coesys``, ``hdnbc``, ``hdnl1``..``hdnl3``,
``step``, ``divq``, ``laplace_solve``, ``upsol``, ``uppres``, ``iterate``).
Fields are numpy arrays in the reference's Fortran layouts.

There is no CPU path: if the CUDA library cannot be loaded, or no device is
present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libvring_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "vring_b200.h")

VR_ABI_VERSION = 1
STATUS = {0: "VR_OK", 1: "VR_ERR_DESC", 2: "VR_ERR_OOM", 3: "VR_ERR_CUDA", 4: "VR_ERR_NONFINITE",
          5: "VR_ERR_TIMEOUT", 6: "VR_ERR_FIELD", 7: "VR_ERR_STATE", 8: "VR_ERR_ARG",
          9: "VR_ERR_CAPACITY", 10: "VR_ERR_NODEVICE", 11: "VR_ERR_SCRATCH", 12: "VR_ERR_IO"}
FIELD_ID = {"q1": 0, "q2": 1, "q3": 2, "dq1": 3, "dq2": 4, "dq3": 5, "ru1": 6, "ru2": 7, "ru3": 8,
            "pres": 11, "prg": 12, "rhs": 13, "dph": 15, "dq3no": 19, "corr3s": 22, "corr3n": 23,
            "csort": 24, "tconv": 25}
PRECISION = {"fp64": 0, "mixed": 1}
WTH = {"exact": 0, "wvnex": 0, "modified": 1}
INFLOW = {"off": 0, "reference": 1}


class VrError(RuntimeError):
    def __init__(self, code: int, msg: str = ""):
        super().__init__("%s: %s" % (STATUS.get(code, code), msg))
        self.code = code


class Desc(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("ntheta", C.c_int32), ("nr", C.c_int32),
                ("nz", C.c_int32), ("rmax", C.c_double), ("zmax", C.c_double), ("dt", C.c_double),
                ("re", C.c_double), ("pe", C.c_double), ("slip", C.c_double),
                ("precision", C.c_int32), ("theta_wavenumber", C.c_int32), ("inflow", C.c_int32),
                ("device", C.c_int32), ("flags", C.c_int32)]


class K2dDesc(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("nr", C.c_int32), ("nz", C.c_int32), ("zmax", C.c_double),
                ("faces", C.c_void_p), ("device", C.c_int32), ("flags", C.c_int32)]


class UnetDesc(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("nr", C.c_int32), ("nz", C.c_int32), ("ch", C.c_int32 * 4),
                ("pool", C.c_int32), ("device", C.c_int32), ("flags", C.c_int32)]


KRYLOV = {"cg": 0, "pcg": 1, "jacobi": 1, "bicgstab": 2, "fcg": 3, "learned": 3, "fcg_jacobi": 4}


def declared_symbols(header: str = HEADER) -> list[str]:
    """Every entry point ``include/vring_b200.h`` declares with VR_API."""
    txt = open(header).read()
    return re.findall(r"VR_API\s+[\w\s\*]+?\b(vr_\w+)\s*\(", txt)


_lib = None


def lib():
    """Load the CUDA library; raises when it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libvring_b200.so is not built (run vring_b200.build.build())")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, dp = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        L.vr_create.argtypes = [C.POINTER(Desc), C.POINTER(vp)]
        L.vr_destroy.argtypes = [vp]
        L.vr_last_error.restype = C.c_char_p
        L.vr_last_error.argtypes = [vp]
        L.vr_sync.argtypes = [vp]
        L.vr_field_extents.argtypes = [vp, i32, C.POINTER(i64)]
        L.vr_set_field.argtypes = [vp, i32, vp, C.POINTER(i64)]
        L.vr_get_field.argtypes = [vp, i32, vp, C.POINTER(i64)]
        L.vr_set_field_async.argtypes = [vp, i32, vp, C.POINTER(i64), vp]
        L.vr_get_field_async.argtypes = [vp, i32, vp, C.POINTER(i64), vp]
        L.vr_set_clock.argtypes = [vp, i32, dp, i64]
        L.vr_get_clock.argtypes = [vp, C.POINTER(i32), C.POINTER(dp), C.POINTER(i64)]
        for n in ("ucoeff", "coesys", "hdnbc", "hdnl1", "hdnl2", "hdnl3", "step", "divq",
                  "laplace_solve", "upsol", "uppres"):
            getattr(L, "vr_" + n).argtypes = [vp]
        L.vr_substep.argtypes = [vp, i32]
        L.vr_set_graphs.argtypes = [vp, i32]
        L.vr_set_slab_transforms.argtypes = [vp, i32]
        L.vr_iterate.argtypes = [vp, i32]
        L.vr_max_divergence.argtypes = [vp, C.POINTER(dp)]
        L.vr_check_finite.argtypes = [vp, C.POINTER(i64)]
        L.vr_clear_status.argtypes = [vp]
        L.vr_wait_selftest.argtypes = [vp, i64]
        L.vr_set_stream.argtypes = [vp, vp]
        L.vr_get_stream.argtypes = [vp, C.POINTER(vp)]
        L.vr_launch_count.argtypes = [vp, C.POINTER(i64)]
        L.vr_profile.argtypes = [vp, i32]
        L.vr_profile_read.argtypes = [vp, i32, C.POINTER(dp), C.POINTER(i64)]
        L.vr_analysis.argtypes = [vp, i32, vp, C.c_char_p]
        L.vr_format_e16_8.argtypes = [dp, C.c_char_p]
        L.vr_restart_save.argtypes = [vp, C.c_char_p, i32]
        L.vr_restart_load.argtypes = [vp, C.c_char_p, C.POINTER(i32)]
        L.vr_part_dump.argtypes = [vp, C.c_char_p]
        L.vr_part_set_dump.argtypes = [vp, i32, C.c_char_p]
        L.vr_part_restart_save.argtypes = [vp, C.c_char_p]
        L.vr_part_restart_load.argtypes = [vp, C.c_char_p]
        L.vr_part_create.argtypes = [vp, i32, i32, i32, C.POINTER(vp)]
        L.vr_part_destroy.argtypes = [vp]
        L.vr_part_info.argtypes = [vp, C.POINTER(dp), C.POINTER(dp), C.POINTER(dp), C.POINTER(i32)]
        L.vr_injc_part.argtypes = [vp, dp, dp, dp, dp, dp, dp, dp, i32, C.POINTER(i32)]
        L.vr_remv_part.argtypes = [vp, i32]
        L.vr_inlt_part.argtypes = [vp, dp, C.POINTER(C.c_uint64), C.POINTER(i32)]
        L.vr_part_set_inflow.argtypes = [vp, dp, C.c_uint64, i32]
        L.vr_iter_part.argtypes = [vp, i32]
        L.vr_part_attach.argtypes = [vp, i32]
        L.vr_part_set_order.argtypes = [vp, i32]
        L.vr_part_set_state.argtypes = [vp, vp, vp, vp, i32]
        L.vr_part_get_state.argtypes = [vp, vp, vp, vp, C.POINTER(i32)]
        L.vr_part_probe.argtypes = [vp, vp, i32, vp, vp]
        L.vr_solve_lap_thom.argtypes = [vp, vp, vp, vp, vp, i32, i32]
        L.vr_solve_lap_bthom.argtypes = [vp, vp, vp, vp, vp, i32, i32, i32]
        L.vr_solve_lap_thom_noalloc.argtypes = [vp, vp, vp, vp, vp, i32, i32, vp]
        L.vr_ens_create.argtypes = [C.POINTER(vp), i32, C.POINTER(vp)]
        L.vr_ens_destroy.argtypes = [vp]
        L.vr_ens_last_error.restype = C.c_char_p
        L.vr_ens_last_error.argtypes = [vp]
        L.vr_ens_iterate.argtypes = [vp, i32]
        L.vr_ens_sync.argtypes = [vp]
        L.vr_ens_launch_count.argtypes = [vp, C.POINTER(i64)]
        L.vr_ens_autotune.argtypes = [vp, i32]
        L.vr_autotune.argtypes = [vp, i32, C.POINTER(i32)]
        L.vr_set_tiles.argtypes = [vp, i32, i32]
        L.vr_k2d_create.argtypes = [C.POINTER(K2dDesc), C.POINTER(vp)]
        L.vr_k2d_destroy.argtypes = [vp]
        L.vr_k2d_last_error.restype = C.c_char_p
        L.vr_k2d_last_error.argtypes = [vp]
        L.vr_k2d_info.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), vp]
        L.vr_k2d_apply.argtypes = [vp, vp, vp]
        L.vr_k2d_apply_dev.argtypes = [vp, vp, vp, i32]
        L.vr_k2d_direct.argtypes = [vp, vp, vp]
        L.vr_k2d_direct_dev.argtypes = [vp, vp, vp]
        L.vr_k2d_solve.argtypes = [vp, i32, vp, vp, dp, i32, C.POINTER(i32), C.POINTER(dp), C.POINTER(dp)]
        L.vr_k2d_solve_dev.argtypes = [vp, i32, vp, vp, dp, i32, C.POINTER(i32), C.POINTER(dp)]
        L.vr_k2d_set_preconditioner.argtypes = [vp, vp]
        L.vr_k2d_set_smoothing.argtypes = [vp, C.c_double]
        L.vr_k2d_diag.argtypes = [vp, vp]
        L.vr_unet_create.argtypes = [C.POINTER(UnetDesc), C.c_uint64, C.POINTER(vp)]
        L.vr_unet_destroy.argtypes = [vp]
        L.vr_unet_last_error.restype = C.c_char_p
        L.vr_unet_last_error.argtypes = [vp]
        L.vr_unet_nparams.argtypes = [vp, C.POINTER(i64)]
        L.vr_unet_get_params.argtypes = [vp, vp]
        L.vr_unet_set_params.argtypes = [vp, vp]
        L.vr_unet_forward.argtypes = [vp, vp, vp]
        L.vr_unet_backward.argtypes = [vp, vp, vp, vp, vp]
        L.vr_unet_train_step.argtypes = [vp, vp, vp, i32, C.c_float, C.POINTER(dp)]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Run:
    """One single-rank vring run resident on a B200 (the reference's type(run))."""

    def __init__(self, ntheta, nr, nz, rmax, zmax, dt, re, pe=1.0, slip=0.0, precision="fp64",
                 theta_wavenumber="exact", inflow="off", device=0):
        self.desc = Desc(VR_ABI_VERSION, ntheta, nr, nz, rmax, zmax, dt, re, pe, slip,
                         PRECISION[precision], WTH[theta_wavenumber], INFLOW[inflow], device, 0)
        self._h = C.c_void_p()
        rc = lib().vr_create(C.byref(self.desc), C.byref(self._h))
        if rc:
            raise VrError(rc, "vr_create(%dx%dx%d)" % (ntheta, nr, nz))
        self.ntheta, self.nr, self.nz = ntheta, nr, nz
        self.dt = dt

    # -- lifetime -------------------------------------------------------------
    def close(self):
        # a context with live particle classes refuses (VR_ERR_STATE) and is kept
        if self._h and lib().vr_destroy(self._h) == 0:
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, rc, what):
        if rc:
            msg = lib().vr_last_error(self._h)
            raise VrError(rc, "%s: %s" % (what, msg.decode() if msg else ""))

    # -- state ----------------------------------------------------------------
    def extents(self, name: str) -> tuple:
        ext = (C.c_int64 * 4)()
        self._chk(lib().vr_field_extents(self._h, FIELD_ID[name], ext), "extents " + name)
        return tuple(int(e) for e in ext)

    def get(self, name: str) -> np.ndarray:
        ext = (C.c_int64 * 4)()
        self._chk(lib().vr_field_extents(self._h, FIELD_ID[name], ext), "extents " + name)
        shape = tuple(int(e) for e in ext)
        a = np.empty(shape, dtype=np.float64, order="F")
        self._chk(lib().vr_get_field(self._h, FIELD_ID[name], _p(a), ext), "get " + name)
        return a if shape[3] > 1 else a[..., 0]

    def set(self, name: str, value) -> None:
        ext = (C.c_int64 * 4)()
        self._chk(lib().vr_field_extents(self._h, FIELD_ID[name], ext), "extents " + name)
        shape = tuple(int(e) for e in ext)
        a = np.asfortranarray(np.broadcast_to(np.asarray(value, dtype=np.float64),
                                              shape if shape[3] > 1 else shape[:3]))
        self._chk(lib().vr_set_field(self._h, FIELD_ID[name], _p(a), ext), "set " + name)

    def set_ptr(self, name: str, host_ptr: int) -> None:
        """Copy a field from a raw host address (e.g. pinned memory)."""
        ext = (C.c_int64 * 4)()
        self._chk(lib().vr_field_extents(self._h, FIELD_ID[name], ext), "extents " + name)
        self._chk(lib().vr_set_field(self._h, FIELD_ID[name], C.c_void_p(host_ptr), ext), "set " + name)

    def get_ptr(self, name: str, host_ptr: int) -> None:
        ext = (C.c_int64 * 4)()
        self._chk(lib().vr_field_extents(self._h, FIELD_ID[name], ext), "extents " + name)
        self._chk(lib().vr_get_field(self._h, FIELD_ID[name], C.c_void_p(host_ptr), ext), "get " + name)

    def set_async(self, name: str, host_ptr: int, cuda_stream: int) -> None:
        """vr_set_field_async from pinned host memory on a caller's stream."""
        ext = (C.c_int64 * 4)()
        self._chk(lib().vr_field_extents(self._h, FIELD_ID[name], ext), "extents " + name)
        self._chk(lib().vr_set_field_async(self._h, FIELD_ID[name], C.c_void_p(host_ptr), ext,
                                           C.c_void_p(cuda_stream)), "set_async " + name)

    def get_async(self, name: str, host_ptr: int, cuda_stream: int) -> None:
        """vr_get_field_async into pinned host memory on a caller's stream."""
        ext = (C.c_int64 * 4)()
        self._chk(lib().vr_field_extents(self._h, FIELD_ID[name], ext), "extents " + name)
        self._chk(lib().vr_get_field_async(self._h, FIELD_ID[name], C.c_void_p(host_ptr), ext,
                                           C.c_void_p(cuda_stream)), "get_async " + name)

    def set_stream(self, cuda_stream_handle: int) -> None:
        """Queue the context's work on a caller's CUDA stream; 0 (which is also
        the handle of the legacy default stream) selects the context's own
        stream, so pass a created stream."""
        self._chk(lib().vr_set_stream(self._h, C.c_void_p(cuda_stream_handle or None)), "set_stream")

    @property
    def launch_count(self) -> int:
        n = C.c_int64()
        self._chk(lib().vr_launch_count(self._h, C.byref(n)), "launch_count")
        return n.value

    PROFILE_KINDS = ["hdnbc", "hdnl", "rhs", "tsweep", "rsweep", "zsweep", "divq", "fft", "dct",
                     "radial", "upsol", "uppres", "diag", "part", "pois_fwd", "pois_bwd"]

    def profile(self, enable: bool) -> None:
        self._chk(lib().vr_profile(self._h, 1 if enable else 0), "profile")

    def profile_read(self) -> dict:
        """{family: (total_ms, launches)} of the kernels recorded since profile(True)."""
        out = {}
        for k, name in enumerate(self.PROFILE_KINDS):
            t, n = C.c_double(), C.c_int64()
            self._chk(lib().vr_profile_read(self._h, k, C.byref(t), C.byref(n)), "profile_read")
            if n.value:
                out[name] = (t.value, n.value)
        return out

    def set_clock(self, irkstep: int, ntime: float, nstep: int = 0):
        self._chk(lib().vr_set_clock(self._h, irkstep, ntime, nstep), "set_clock")

    @property
    def clock(self):
        irk, t, n = C.c_int32(), C.c_double(), C.c_int64()
        self._chk(lib().vr_get_clock(self._h, C.byref(irk), C.byref(t), C.byref(n)), "get_clock")
        return irk.value, t.value, n.value

    # -- the reference's routines --------------------------------------------
    def __getattr__(self, name):
        if name in ("ucoeff", "coesys", "hdnbc", "hdnl1", "hdnl2", "hdnl3", "step", "divq",
                    "laplace_solve", "upsol", "uppres", "sync"):
            fn = getattr(lib(), "vr_" + name)
            return lambda: self._chk(fn(self._h), name)
        raise AttributeError(name)

    def analysis(self, anlstp: int, path=None) -> np.ndarray:
        """analysis (run.F90:238-388): ntime, vortmax, swrlmax and the ten
        analysis.dat columns after them; appends the line to path if given."""
        out = np.zeros(13)
        self._chk(lib().vr_analysis(self._h, anlstp, _p(out), None if path is None else str(path).encode()),
                  "analysis")
        return out

    def restart_save(self, path, full: bool = False) -> None:
        """restart_save (run.F90:390-460); full=True appends the whole state."""
        self._chk(lib().vr_restart_save(self._h, str(path).encode(), 1 if full else 0), "restart_save")

    def restart_load(self, path) -> bool:
        """restart_load (run.F90:463-531); True when the whole state was restored."""
        full = C.c_int32()
        self._chk(lib().vr_restart_load(self._h, str(path).encode(), C.byref(full)), "restart_load")
        return bool(full.value)

    def substep(self, irk: int):
        self._chk(lib().vr_substep(self._h, irk), "substep")

    def iterate(self, nsteps: int):
        self._chk(lib().vr_iterate(self._h, nsteps), "iterate")

    def max_divergence(self) -> float:
        v = C.c_double()
        self._chk(lib().vr_max_divergence(self._h, C.byref(v)), "max_divergence")
        return v.value

    def set_slab_transforms(self, on: bool):
        """The fused substep's transforms as slab cluster kernels, or apart (default)."""
        self._chk(lib().vr_set_slab_transforms(self._h, 1 if on else 0), "set_slab_transforms")

    def set_graphs(self, on: bool):
        """Replay each substep as a captured CUDA graph (default) or launch one by one."""
        self._chk(lib().vr_set_graphs(self._h, 1 if on else 0), "set_graphs")

    def clear_status(self):
        """Clear the device status word (bounded-wait timeouts) of the context."""
        self._chk(lib().vr_clear_status(self._h), "clear_status")

    def wait_selftest(self, limit_ns: int = 10_000_000) -> int:
        """Run a kernel whose bounded wait must run out; returns the status code
        (VR_ERR_TIMEOUT = 5 when the wait gave up as designed)."""
        return lib().vr_wait_selftest(self._h, int(limit_ns))

    def count_nonfinite(self) -> int:
        n = C.c_int64()
        rc = lib().vr_check_finite(self._h, C.byref(n))
        if rc not in (0, 4):
            self._chk(rc, "check_finite")
        return n.value


def solve_lap_thom(rhs, aa, bb, cc):
    """Batched Thomas solve on the GPU (tripar.F90:120-145); 2-D inputs are
    (nbatch, n) with one system per row."""
    arrs = [np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64) for x in (rhs, aa, bb, cc)]
    nb, n = arrs[0].shape
    sol = np.empty_like(arrs[0])
    rc = lib().vr_solve_lap_thom(_p(arrs[0]), _p(sol), _p(arrs[1]), _p(arrs[2]), _p(arrs[3]), n, nb)
    if rc:
        raise VrError(rc, "vr_solve_lap_thom")
    return sol.reshape(np.shape(rhs))


def solve_lap_bthom(rhs, b1, b2, b3, m, n):
    """Batched block Thomas (btrithom.F90:5-71); inputs (nbatch, m*n)."""
    arrs = [np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64) for x in (rhs, b1, b2, b3)]
    nb = arrs[0].shape[0]
    sol = np.empty_like(arrs[0])
    rc = lib().vr_solve_lap_bthom(_p(arrs[0]), _p(sol), _p(arrs[1]), _p(arrs[2]), _p(arrs[3]), m, n, nb)
    if rc:
        raise VrError(rc, "vr_solve_lap_bthom")
    return sol.reshape(np.shape(rhs))


class Part:
    """One particle class on a Run (part_tools.F90 ``type part``).

    ``u`` (naloc, 117) and ``v`` (naloc, 3) are the reference's state arrays;
    slots are 1-based in ``injc``/``remv`` as in the reference.
    """

    NVAR = 117

    def __init__(self, run: Run, pid: int, naloc: int, mode: int = 0):
        self.run, self.naloc = run, naloc
        self._h = C.c_void_p()
        run._chk(lib().vr_part_create(run._h, pid, naloc, mode, C.byref(self._h)), "vr_part_create")
        r, st, c, ns = C.c_double(), C.c_double(), C.c_double(), C.c_int32()
        self._chk(lib().vr_part_info(self._h, C.byref(r), C.byref(st), C.byref(c), C.byref(ns)))
        self.r, self.st, self.c, self.nsubdt = r.value, st.value, c.value, ns.value

    def _chk(self, rc, what="particles"):
        self.run._chk(rc, what)

    def close(self):
        if self._h:
            lib().vr_part_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def injc(self, x, y, z, u=0.0, v=0.0, w=0.0, c=None, icall=1) -> int:
        ip = C.c_int32()
        self._chk(lib().vr_injc_part(self._h, x, y, z, self.c if c is None else c, u, v, w, icall,
                                     C.byref(ip)), "injc_part")
        return ip.value

    def remv(self, ip: int) -> None:
        self._chk(lib().vr_remv_part(self._h, ip), "remv_part")

    def iter_part(self, irk: int = 1) -> None:
        self._chk(lib().vr_iter_part(self._h, irk), "iter_part")

    def set_order(self, order: int) -> None:
        """0: walk the slots in slot order (default); 1: grouped by cell."""
        self._chk(lib().vr_part_set_order(self._h, order), "part_set_order")

    def inlt(self, r0: float, rng_state: int):
        """inlt_part (part_tools.F90:95-142); returns (injected, new rng state)."""
        st, n = C.c_uint64(rng_state), C.c_int32()
        self._chk(lib().vr_inlt_part(self._h, r0, C.byref(st), C.byref(n)), "inlt_part")
        return n.value, st.value

    def set_inflow(self, r0: float, seed: int, on: bool = True) -> None:
        """Inflow injection every 10 steps inside Run.iterate (attached classes)."""
        self._chk(lib().vr_part_set_inflow(self._h, r0, seed, 1 if on else 0), "part_set_inflow")

    def dump(self, directory=None) -> None:
        """iter_part's dumps (part_tools.F90:444-491) into directory."""
        self._chk(lib().vr_part_dump(self._h, None if directory is None else str(directory).encode()), "part_dump")

    def set_dump(self, expstp: int, directory=None) -> None:
        self._chk(lib().vr_part_set_dump(self._h, expstp, None if directory is None else str(directory).encode()),
                  "part_set_dump")

    def restart_save(self, path) -> None:
        self._chk(lib().vr_part_restart_save(self._h, str(path).encode()), "part_restart_save")

    def restart_load(self, path) -> None:
        self._chk(lib().vr_part_restart_load(self._h, str(path).encode()), "part_restart_load")

    def attach(self, on: bool = True) -> None:
        self._chk(lib().vr_part_attach(self._h, 1 if on else 0), "part_attach")

    def set_state(self, u, v, isfre=None, nlast=None) -> None:
        u = np.asfortranarray(u, dtype=np.float64)
        v = np.asfortranarray(v, dtype=np.float64)
        assert u.shape == (self.naloc, self.NVAR) and v.shape == (self.naloc, 3)
        isf = None if isfre is None else np.ascontiguousarray(isfre, dtype=np.int32)
        self._chk(lib().vr_part_set_state(self._h, _p(u), _p(v), None if isf is None else _p(isf),
                                          self.naloc if nlast is None else nlast), "part_set_state")

    def state(self):
        """(u, v, isfre, {npart, nlast, nfree, nids}) copied to the host."""
        u = np.empty((self.naloc, self.NVAR), dtype=np.float64, order="F")
        v = np.empty((self.naloc, 3), dtype=np.float64, order="F")
        isf = np.empty(self.naloc, dtype=np.int32)
        cnt = (C.c_int32 * 4)()
        self._chk(lib().vr_part_get_state(self._h, _p(u), _p(v), _p(isf), cnt), "part_get_state")
        return u, v, isf, dict(zip(("npart", "nlast", "nfree", "nids"), list(cnt)))

    @property
    def counts(self) -> dict:
        cnt = (C.c_int32 * 4)()
        self._chk(lib().vr_part_get_state(self._h, None, None, None, cnt), "part_get_state")
        return dict(zip(("npart", "nlast", "nfree", "nids"), list(cnt)))

    def probe(self, xyz):
        """Interpolated velocity (n,3), gradient (n,3,3) [i,j] = du_i/dx_j,
        Hessian (n,3,3,3) and cell indices (n,3) at points xyz (n,3)."""
        xyz = np.ascontiguousarray(np.atleast_2d(xyz), dtype=np.float64)
        n = xyz.shape[0]
        out = np.empty((n, 39), dtype=np.float64)
        cells = np.empty((n, 3), dtype=np.int32)
        self._chk(lib().vr_part_probe(self._h, _p(xyz), n, _p(out), _p(cells)), "part_probe")
        vel = out[:, :3]
        dvel = out[:, 3:12].reshape(n, 3, 3, order="F")
        ddvel = out[:, 12:].reshape(n, 3, 3, 3, order="F")
        return vel, dvel, ddvel, cells


THOM_NOALLOC_MAX = 1 << 19


def solve_lap_thom_noalloc(rhs_ptr: int, sol_ptr: int, aa_ptr: int, bb_ptr: int, cc_ptr: int,
                           n: int, nbatch: int, cuda_stream: int = 0) -> None:
    """``vr_solve_lap_thom_noalloc``: the batched Thomas solve on device
    arrays (raw device addresses of n*nbatch doubles each), enqueued on
    ``cuda_stream`` without any device allocation; its scratch is a fixed
    array of THOM_NOALLOC_MAX doubles per device shared by all calls."""
    rc = lib().vr_solve_lap_thom_noalloc(C.c_void_p(rhs_ptr), C.c_void_p(sol_ptr), C.c_void_p(aa_ptr),
                                         C.c_void_p(bb_ptr), C.c_void_p(cc_ptr), n, nbatch,
                                         C.c_void_p(cuda_stream or None))
    if rc:
        raise VrError(rc, "vr_solve_lap_thom_noalloc(n=%d, nbatch=%d)" % (n, nbatch))


def format_e16_8(x: float) -> str:
    """gfortran's E16.8 edit descriptor, as the library writes analysis.dat."""
    buf = C.create_string_buffer(17)
    rc = lib().vr_format_e16_8(float(x), buf)
    if rc:
        raise VrError(rc, "vr_format_e16_8")
    return buf.value.decode()


class K2d:
    """The axisymmetric (Ntheta = 1) pressure operator on radial faces
    ``faces`` (nr+1 values, 0 .. rmax) and nz uniform cells on [0, zmax], with
    its GPU solvers (``vr_k2d_*``).  Host vectors are (nr, nz) arrays indexed
    [j, k], stored r fastest."""

    def __init__(self, faces, nz: int, zmax: float, device: int = 0):
        self.faces = np.ascontiguousarray(faces, dtype=np.float64)
        self.nr, self.nz, self.zmax = self.faces.size - 1, int(nz), float(zmax)
        d = K2dDesc(VR_ABI_VERSION, self.nr, self.nz, self.zmax, self.faces.ctypes.data, device, 0)
        self._h = C.c_void_p()
        rc = lib().vr_k2d_create(C.byref(d), C.byref(self._h))
        if rc:
            raise VrError(rc, "vr_k2d_create")

    def _chk(self, rc, what):
        if rc:
            raise VrError(rc, "%s: %s" % (what, (lib().vr_k2d_last_error(self._h) or b"").decode()))

    def close(self):
        if self._h:
            lib().vr_k2d_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _vec(self, a):
        return np.asfortranarray(np.asarray(a, dtype=np.float64).reshape(self.nr, self.nz, order="F"))

    def apply(self, x) -> np.ndarray:
        x = self._vec(x)
        y = np.empty_like(x)
        self._chk(lib().vr_k2d_apply(self._h, _p(x), _p(y)), "k2d_apply")
        return y

    def direct(self, f) -> np.ndarray:
        f = self._vec(f)
        x = np.empty_like(f)
        self._chk(lib().vr_k2d_direct(self._h, _p(f), _p(x)), "k2d_direct")
        return x

    def solve(self, f, method="cg", x0=None, tol=1e-10, maxit=1000000):
        """(x, iterations, relative residual, device ms)."""
        f = self._vec(f)
        # the library reads r fastest: keep the copy in Fortran order
        x = np.zeros_like(f) if x0 is None else np.array(self._vec(x0), order="F", copy=True)
        it, rr, ms = C.c_int32(), C.c_double(), C.c_double()
        self._chk(lib().vr_k2d_solve(self._h, KRYLOV[method], _p(f), _p(x), tol, maxit, C.byref(it),
                                     C.byref(rr), C.byref(ms)), "k2d_solve")
        return x, it.value, rr.value, ms.value

    def solve_dev(self, f_ptr: int, x_ptr: int, method="cg", tol=1e-10, maxit=1000000):
        it, rr = C.c_int32(), C.c_double()
        self._chk(lib().vr_k2d_solve_dev(self._h, KRYLOV[method], C.c_void_p(f_ptr), C.c_void_p(x_ptr), tol,
                                         maxit, C.byref(it), C.byref(rr)), "k2d_solve_dev")
        return it.value, rr.value

    def direct_dev(self, f_ptr: int, x_ptr: int) -> None:
        self._chk(lib().vr_k2d_direct_dev(self._h, C.c_void_p(f_ptr), C.c_void_p(x_ptr)), "k2d_direct_dev")

    def apply_dev(self, x_ptr: int, y_ptr: int, symmetric: bool = False) -> None:
        self._chk(lib().vr_k2d_apply_dev(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), 1 if symmetric else 0),
                  "k2d_apply_dev")

    def diag(self) -> np.ndarray:
        """diag(S) of the symmetric form, (nr, nz)."""
        d = np.empty((self.nr, self.nz), dtype=np.float64, order="F")
        self._chk(lib().vr_k2d_diag(self._h, _p(d)), "k2d_diag")
        return d

    def set_smoothing(self, omega: float) -> None:
        """Weight of the damped-Jacobi steps around the network (0: off)."""
        self._chk(lib().vr_k2d_set_smoothing(self._h, omega), "k2d_set_smoothing")

    def set_preconditioner(self, net) -> None:
        self._chk(lib().vr_k2d_set_preconditioner(self._h, net._h if net is not None else None),
                  "k2d_set_preconditioner")


class UNet:
    """The learned preconditioner (``vr_unet_*``): a 4-level linear U-Net with
    BF16 weights and activations and FP32 accumulation on an (nr, nz) grid."""

    CUDA_CORES = 1

    def __init__(self, nr: int, nz: int, ch=(16, 32, 48, 64), seed: int = 0, device: int = 0, flags: int = 0,
                 pool: int = 2):
        """pool: the pooling factor between levels (2 or 4); flags =
        UNet.CUDA_CORES runs the forward convolutions on the CUDA cores
        instead of the tensor cores."""
        self.nr, self.nz, self.ch, self.pool = int(nr), int(nz), tuple(int(c) for c in ch), int(pool)
        d = UnetDesc(VR_ABI_VERSION, self.nr, self.nz, (C.c_int32 * 4)(*self.ch), self.pool, device, flags)
        self._h = C.c_void_p()
        rc = lib().vr_unet_create(C.byref(d), seed, C.byref(self._h))
        if rc:
            raise VrError(rc, "vr_unet_create")
        n = C.c_int64()
        self._chk(lib().vr_unet_nparams(self._h, C.byref(n)), "unet_nparams")
        self.nparams = n.value

    def _chk(self, rc, what):
        if rc:
            raise VrError(rc, "%s: %s" % (what, (lib().vr_unet_last_error(self._h) or b"").decode()))

    def close(self):
        if self._h:
            lib().vr_unet_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        w = np.empty(self.nparams, dtype=np.float32)
        self._chk(lib().vr_unet_get_params(self._h, _p(w)), "unet_get_params")
        return w

    def set_params(self, w) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == self.nparams
        self._chk(lib().vr_unet_set_params(self._h, _p(w)), "unet_set_params")

    def _vec(self, a):
        return np.asfortranarray(np.asarray(a, dtype=np.float64).reshape(self.nr, self.nz, order="F"))

    def forward(self, x) -> np.ndarray:
        x = self._vec(x)
        y = np.empty_like(x)
        self._chk(lib().vr_unet_forward(self._h, _p(x), _p(y)), "unet_forward")
        return y

    def backward(self, x, g):
        """(dL/dw float32 (nparams,), dL/dx (nr, nz)) of L = sum(g * N(x))."""
        x, g = self._vec(x), self._vec(g)
        dw = np.empty(self.nparams, dtype=np.float32)
        dx = np.empty_like(x)
        self._chk(lib().vr_unet_backward(self._h, _p(x), _p(g), _p(dw), _p(dx)), "unet_backward")
        return dw, dx

    def train_step(self, k2d: K2d, e_ptr: int, nb: int, lr: float) -> float:
        """One Adam step on nb device-resident errors (nb x nr*nz doubles);
        returns the energy-norm loss before the step."""
        loss = C.c_double()
        self._chk(lib().vr_unet_train_step(self._h, k2d._h, C.c_void_p(e_ptr), nb, lr, C.byref(loss)),
                  "unet_train_step")
        return loss.value


class Ensemble:
    """Independent rings (Run objects on one device) stepped together: one
    CUDA graph launch per RK substep covering every ring (``vr_ens_*``)."""

    def __init__(self, runs):
        self.runs = list(runs)
        arr = (C.c_void_p * len(self.runs))(*[r._h.value for r in self.runs])
        self._h = C.c_void_p()
        rc = lib().vr_ens_create(arr, len(self.runs), C.byref(self._h))
        if rc:
            raise VrError(rc, "vr_ens_create")

    def _chk(self, rc, what):
        if rc:
            raise VrError(rc, "%s: %s" % (what, (lib().vr_ens_last_error(self._h) or b"").decode()))

    def close(self):
        if self._h:
            lib().vr_ens_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def iterate(self, nsteps: int) -> None:
        self._chk(lib().vr_ens_iterate(self._h, nsteps), "ens_iterate")

    def sync(self) -> None:
        self._chk(lib().vr_ens_sync(self._h), "ens_sync")

    def autotune(self, force: bool = False) -> None:
        self._chk(lib().vr_ens_autotune(self._h, 1 if force else 0), "ens_autotune")

    @property
    def launch_count(self) -> int:
        n = C.c_int64()
        self._chk(lib().vr_ens_launch_count(self._h, C.byref(n)), "ens_launch_count")
        return n.value


def autotune(run: Run, force: bool = False):
    """``vr_autotune``: the fastest (r, z) sweep tile variants for run's grid."""
    ch = (C.c_int32 * 2)()
    run._chk(lib().vr_autotune(run._h, 1 if force else 0, ch), "autotune")
    return ch[0], ch[1]


def set_tiles(run: Run, r_variant: int, z_variant: int) -> None:
    run._chk(lib().vr_set_tiles(run._h, r_variant, z_variant), "set_tiles")
