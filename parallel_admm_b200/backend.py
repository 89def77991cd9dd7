"""ctypes binding of ``libadmm_b200.so`` (the C ABI in ``include/admm_b200.h``).

``ADMMBackendB200`` mirrors the reference's backend contract for the ADMM GPU
path -- ``IADMMBackend`` (``src/solver/core/admm_backend.h:15-41``) together with
the ``Solver`` state accessors it exposes (``src/solver/solver.h:66-150``) -- and
``BVHB200`` mirrors ``ICollisionDetector`` (``src/contact/icollision_detector.h:19-47``).
Errors raise ``AdmmError`` instead of exiting the process.  The native library is
required: importing this module on a machine without the built ``.so`` raises.
"""
from __future__ import annotations

import ctypes
import os
import time
from typing import Dict, Optional

import numpy as np

from .scene import Scene

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libadmm_b200.so")

ABI_VERSION = 5
OK = 0
ERR_INVALID = -1
ERR_CUDA = -2
ERR_OOM = -3
ERR_CONTACT_OVERFLOW = -4
ERR_STACK_OVERFLOW = -5
ERR_NAN = -6
ERR_NOT_CONVERGED = -7
ERR_NO_DEVICE = -8
ERR_STATE = -9
ERR_TIMEOUT = -10

BUF_X, BUF_X0, BUF_V, BUF_P, BUF_UC, BUF_UE, BUF_Z, BUF_B, BUF_MXT = range(9)
PHASES = ("pre", "dcd", "local", "contact", "rhs", "jacobi", "residual", "final")
KERNELS = {"none": 0, "local": 1, "jacobi": 2, "rhs": 3, "contact_du": 4, "contact_gather": 5,
           "dcd_vf": 6, "dcd_ee": 7, "phases": 100}

_f = ctypes.POINTER(ctypes.c_float)
_i = ctypes.POINTER(ctypes.c_int32)
_d = ctypes.POINTER(ctypes.c_double)


class AdmmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


class AdmmB200Desc(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int32), ("n_vert", ctypes.c_int32), ("n_dyn", ctypes.c_int32),
        ("n_rows", ctypes.c_int32),
        ("x0", _f), ("v0", _f), ("mass", _f), ("is_fixed", _i),
        ("n_tri", ctypes.c_int32), ("tri_start_row", ctypes.c_int32),
        ("tri_inds", _i), ("tri_binv", _f), ("tri_w", _f),
        ("n_tet", ctypes.c_int32), ("tet_start_row", ctypes.c_int32),
        ("tet_inds", _i), ("tet_binv", _f), ("tet_w", _f),
        ("n_bend", ctypes.c_int32), ("bend_start_row", ctypes.c_int32),
        ("bend_offsets", _i), ("bend_inds", _i), ("bend_coeffs", _f), ("bend_rest_norm", _f), ("bend_w", _f),
        ("n_pin", ctypes.c_int32), ("pin_start_row", ctypes.c_int32),
        ("pin_inds", _i), ("pin_pos", _f), ("pin_w", _f),
        ("n_surf_tri", ctypes.c_int32), ("n_surf_edge", ctypes.c_int32), ("n_surf_vert", ctypes.c_int32),
        ("surf_tris", _i), ("surf_edges", _i), ("surf_verts", _i), ("contact_w", _f),
        ("dt", ctypes.c_float), ("g", ctypes.c_float), ("mu", ctypes.c_float), ("kappa", ctypes.c_float),
        ("beta", ctypes.c_float), ("thickness", ctypes.c_float),
        ("admm_max_iter", ctypes.c_int32), ("dcd_interval", ctypes.c_int32), ("gs_max_iter", ctypes.c_int32),
        ("jacobi_iter", ctypes.c_int32), ("max_contacts", ctypes.c_int32),
        ("enable_contact", ctypes.c_int32), ("warmstart_ue", ctypes.c_int32), ("warmstart_uc", ctypes.c_int32),
        ("residual_tol", ctypes.c_float), ("residual_check_every", ctypes.c_int32),
        ("bvh_refit", ctypes.c_int32), ("ell_lanes", ctypes.c_int32), ("jacobi_mode", ctypes.c_int32),
        ("broad_phase", ctypes.c_int32), ("global_solver", ctypes.c_int32), ("pcg_iter", ctypes.c_int32),
        ("vert_mu", ctypes.POINTER(ctypes.c_float)), ("query_lanes", ctypes.c_int32),
        ("contact_semantics", ctypes.c_int32), ("backend_semantics", ctypes.c_int32),
        ("damp_k_L", ctypes.c_float), ("damp_k_M", ctypes.c_float),
    ]


class AdmmStepStats(ctypes.Structure):
    _fields_ = [("frame", ctypes.c_int64), ("step_ms", ctypes.c_double), ("n_contacts", ctypes.c_int32),
                ("admm_iters", ctypes.c_int32), ("primal_residual", ctypes.c_double),
                ("dual_residual", ctypes.c_double), ("status", ctypes.c_int32), ("peak_contacts", ctypes.c_int32)]


class DescHolder:
    """Builds an ``AdmmB200Desc`` from a ``Scene`` and keeps its arrays alive."""

    def __init__(self, sc: Scene, **overrides):
        p = sc.params
        self.scene = sc
        keep = {}

        def arr(name, a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep[name] = a
            return a.ctypes.data_as(_f if dt == np.float32 else _i)

        d = AdmmB200Desc()
        d.abi_version = ABI_VERSION
        d.n_vert = sc.n_vert
        d.n_dyn = sc.n_dyn
        d.n_rows = sc.n_rows
        d.x0 = arr("x0", sc.verts, np.float32)
        d.v0 = None
        d.mass = arr("mass", sc.mass, np.float32)
        d.is_fixed = arr("fixed", sc.is_fixed, np.int32)
        d.n_tri, d.tri_start_row = len(sc.tri_inds), sc.tri_start_row
        d.tri_inds = arr("ti", sc.tri_inds, np.int32)
        d.tri_binv = arr("tb", sc.tri_binv, np.float32)
        d.tri_w = arr("tw", sc.tri_w, np.float32)
        d.n_tet, d.tet_start_row = len(sc.tet_inds), sc.tet_start_row
        d.tet_inds = arr("Ti", sc.tet_inds, np.int32)
        d.tet_binv = arr("Tb", sc.tet_binv, np.float32)
        d.tet_w = arr("Tw", sc.tet_w, np.float32)
        d.n_bend, d.bend_start_row = len(sc.bend_w), sc.bend_start_row
        d.bend_offsets = arr("bo", sc.bend_offsets, np.int32)
        d.bend_inds = arr("bi", sc.bend_inds, np.int32)
        d.bend_coeffs = arr("bc", sc.bend_coeffs, np.float32)
        d.bend_rest_norm = None
        d.bend_w = arr("bw", sc.bend_w, np.float32)
        d.n_pin, d.pin_start_row = len(sc.pin_inds), sc.pin_start_row
        d.pin_inds = arr("pi", sc.pin_inds, np.int32)
        d.pin_pos = arr("pp", sc.pin_pos, np.float32)
        d.pin_w = arr("pw", sc.pin_w, np.float32)
        d.n_surf_tri, d.n_surf_edge, d.n_surf_vert = len(sc.surf_tris), len(sc.surf_edges), len(sc.surf_verts)
        d.surf_tris = arr("st", sc.surf_tris, np.int32)
        d.surf_edges = arr("se", sc.surf_edges, np.int32)
        d.surf_verts = arr("sv", sc.surf_verts, np.int32)
        d.contact_w = arr("cw", sc.contact_w, np.float32)
        d.dt, d.g, d.mu, d.kappa, d.beta, d.thickness = p.dt, p.g, p.mu, p.kappa, p.beta, p.thickness
        d.admm_max_iter, d.dcd_interval, d.gs_max_iter = p.admm_max_iter, p.dcd_interval, p.gs_max_iter
        d.jacobi_iter, d.max_contacts = p.jacobi_iter, p.max_contacts
        d.enable_contact = int(p.enable_contact)
        d.warmstart_ue, d.warmstart_uc = int(p.warmstart_ue), int(p.warmstart_uc)
        d.residual_tol, d.residual_check_every = 0.0, 0
        d.bvh_refit = int(p.bvh_refit)
        d.ell_lanes = int(p.ell_lanes)
        d.jacobi_mode = int(p.jacobi_mode)
        d.broad_phase = int(p.broad_phase)
        d.global_solver = int(p.global_solver)
        d.pcg_iter = int(p.pcg_iter)
        d.query_lanes = int(getattr(p, "query_lanes", 0))
        d.contact_semantics = int(getattr(p, "contact_semantics", 0))
        d.backend_semantics = int(getattr(p, "backend_semantics", 0))
        d.damp_k_L = float(getattr(p, "damp_k_L", 1e-4))
        d.damp_k_M = float(getattr(p, "damp_k_M", 0.0))
        vm = getattr(sc, "vert_mu", None)
        d.vert_mu = arr("vm", vm, np.float32) if vm is not None else None
        for k, v in overrides.items():
            setattr(d, k, v)
        self.desc = d
        self._keep = keep


_lib = None


def lib():
    """Load the native library (fails loudly when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libadmm_b200.so not built at {LIB_PATH}: run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        sig = {
            "admm_b200_create": (ctypes.c_int, [ctypes.POINTER(AdmmB200Desc), ctypes.c_int, ctypes.POINTER(vp)]),
            "admm_b200_destroy": (None, [vp]),
            "admm_b200_errstr": (ctypes.c_char_p, [ctypes.c_int]),
            "admm_b200_last_error": (ctypes.c_char_p, [vp]),
            "admm_b200_step": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(AdmmStepStats)]),
            "admm_b200_step_async": (ctypes.c_int, [vp, ctypes.c_int]),
            "admm_b200_sync": (ctypes.c_int, [vp]),
            "admm_b200_set_state": (ctypes.c_int, [vp, _f, _f, ctypes.c_int]),
            "admm_b200_get_state": (ctypes.c_int, [vp, _f, _f, ctypes.c_int]),
            "admm_b200_reset": (ctypes.c_int, [vp]),
            "admm_b200_device_state": (ctypes.c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp)]),
            "admm_b200_read_buffer": (ctypes.c_int, [vp, ctypes.c_int, _f, ctypes.c_int]),
            "admm_b200_write_buffer": (ctypes.c_int, [vp, ctypes.c_int, _f, ctypes.c_int]),
            "admm_b200_local_step": (ctypes.c_int, [vp]),
            "admm_b200_global_step": (ctypes.c_int, [vp]),
            "admm_b200_jacobi": (ctypes.c_int, [vp, ctypes.c_int]),
            "admm_b200_pre_integration": (ctypes.c_int, [vp]),
            "admm_b200_contact_step": (ctypes.c_int, [vp]),
            "admm_b200_detect": (ctypes.c_int, [vp, _i]),
            "admm_b200_detect_host": (ctypes.c_int, [vp, _f, ctypes.c_int, _i]),
            "admm_b200_contacts": (ctypes.c_int, [vp, _i, _f, _f, _f, _f, ctypes.c_int, _i]),
            "admm_b200_contact_count": (ctypes.c_int, [vp, _i]),
            "admm_b200_max_slots": (ctypes.c_int, [vp, _i]),
            "admm_b200_peak_contact_count": (ctypes.c_int, [vp, _i]),
            "admm_b200_clear_contacts": (ctypes.c_int, [vp]),
            "admm_b200_residuals": (ctypes.c_int, [vp, _d, _d]),
            "admm_b200_last_step_device_ms": (ctypes.c_int, [vp, _f]),
            "admm_b200_set_profiling": (ctypes.c_int, [vp, ctypes.c_int]),
            "admm_b200_kernels_per_step": (ctypes.c_int, [vp, _i]),
            "admm_b200_kernels_fallback": (ctypes.c_int, [vp, _i]),
            "admm_b200_step_host": (ctypes.c_int, [vp, _f, _f, _f, _f, ctypes.c_int]),
            "admm_b200_phase_times": (ctypes.c_int, [vp, _d, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]),
            "admm_b200_set_probe": (ctypes.c_int, [vp, ctypes.c_int]),
            "admm_b200_probe_time": (ctypes.c_int, [vp, _d, ctypes.POINTER(ctypes.c_int64)]),
            "admm_b200_tuning": (ctypes.c_int, [vp, _i, _i, _f, _f]),
            "admm_b200_global_mode": (ctypes.c_int, [vp, _i, _i, _f, _f]),
            "admm_b200_set_preconditioner": (ctypes.c_int, [vp, _f, ctypes.c_int]),
            "admm_b200_set_rigid_track": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _f, _f]),
            "admm_b200_set_point_track": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _f, _f,
                                                         _f, ctypes.c_float]),
            "admm_b200_clear_tracks": (ctypes.c_int, [vp]),
            "admm_b200_jacobi_noalloc": (ctypes.c_int, [ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int,
                                                        vp]),
            "admm_b200_set_learned": (ctypes.c_int, [vp, ctypes.c_int, _f, _f, _f, _f, ctypes.c_int]),
            "admm_b200_vertex_order": (ctypes.c_int, [vp, _i, ctypes.c_int]),
            "admm_b200_learned_stats": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int64)]),
            "admm_b200_record_global": (ctypes.c_int, [vp, ctypes.c_int, _f, _f, _f, ctypes.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    """Names the header declares (used by the load test)."""
    return [
        "admm_b200_create", "admm_b200_destroy", "admm_b200_errstr", "admm_b200_last_error", "admm_b200_step",
        "admm_b200_step_async", "admm_b200_sync", "admm_b200_set_state", "admm_b200_get_state",
        "admm_b200_reset", "admm_b200_device_state", "admm_b200_read_buffer", "admm_b200_write_buffer",
        "admm_b200_local_step", "admm_b200_global_step", "admm_b200_jacobi", "admm_b200_pre_integration",
        "admm_b200_contact_step", "admm_b200_detect", "admm_b200_detect_host", "admm_b200_contacts",
        "admm_b200_contact_count", "admm_b200_max_slots", "admm_b200_peak_contact_count",
        "admm_b200_clear_contacts", "admm_b200_residuals", "admm_b200_last_step_device_ms",
        "admm_b200_set_profiling", "admm_b200_kernels_per_step", "admm_b200_kernels_fallback", "admm_b200_step_host",
        "admm_b200_phase_times", "admm_b200_set_probe", "admm_b200_probe_time", "admm_b200_tuning",
        "admm_b200_jacobi_noalloc", "admm_b200_global_mode", "admm_b200_set_preconditioner",
        "admm_b200_set_rigid_track", "admm_b200_set_point_track", "admm_b200_clear_tracks",
        "admm_b200_system", "admm_gnn_create", "admm_gnn_set_graph", "admm_gnn_destroy", "admm_gnn_num_params",
        "admm_gnn_set_params", "admm_gnn_get_params", "admm_gnn_forward", "admm_gnn_loss_grad", "admm_gnn_adam",
        "admm_b200_set_learned", "admm_b200_learned_stats", "admm_b200_record_global", "admm_gnn_outputs",
        "admm_gnn_backward", "admm_learn_create", "admm_learn_destroy", "admm_learn_loss_grad", "admm_learn_solve",
        "admm_learn_set_residual_weight",
        "admm_b200_vertex_order",
    ]


def _p(a: np.ndarray, ct=_f):
    return a.ctypes.data_as(ct)


class Handle:
    """Owns one ``AdmmB200*``."""

    def __init__(self, sc: Scene, device: int = 0, **overrides):
        self.holder = DescHolder(sc, **overrides)
        self.scene = sc
        self.h = ctypes.c_void_p()
        rc = lib().admm_b200_create(ctypes.byref(self.holder.desc), device, ctypes.byref(self.h))
        if rc != OK:
            raise AdmmError(rc, "admm_b200_create: " + lib().admm_b200_errstr(rc).decode())
        self.n_vert = sc.n_vert
        self.n_dyn = sc.n_dyn
        self.n_rows = sc.n_rows

    def check(self, rc: int, what: str, allow=()):
        if rc != OK and rc not in allow:
            raise AdmmError(rc, f"{what}: {lib().admm_b200_errstr(rc).decode()} "
                                f"[{lib().admm_b200_last_error(self.h).decode()}]")
        return rc

    def close(self):
        if self.h:
            lib().admm_b200_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rows(self, which: int) -> int:
        return {BUF_UC: self.n_dyn, BUF_B: self.n_dyn, BUF_UE: self.n_rows, BUF_Z: self.n_rows}.get(which, self.n_vert)

    def read(self, which: int) -> np.ndarray:
        n = self.rows(which)
        out = np.zeros((n, 3), np.float32)
        self.check(lib().admm_b200_read_buffer(self.h, which, _p(out), n), "read_buffer")
        return out

    def write(self, which: int, a: np.ndarray):
        n = self.rows(which)
        a = np.ascontiguousarray(a, np.float32).reshape(n, 3)
        self.check(lib().admm_b200_write_buffer(self.h, which, _p(a), n), "write_buffer")

    def step(self, n: int = 1, allow=()) -> Dict[str, float]:
        st = AdmmStepStats()
        rc = lib().admm_b200_step(self.h, n, ctypes.byref(st))
        self.check(rc, "step", allow=allow)
        return {"frame": st.frame, "step_ms": st.step_ms, "n_contacts": st.n_contacts, "iters": st.admm_iters,
                "primal": st.primal_residual, "dual": st.dual_residual, "status": st.status,
                "peak": st.peak_contacts}

    def step_async(self, n: int = 1):
        self.check(lib().admm_b200_step_async(self.h, n), "step_async")

    def sync(self):
        self.check(lib().admm_b200_sync(self.h), "sync")

    def get_state(self):
        x = np.zeros((self.n_vert, 3), np.float32)
        v = np.zeros((self.n_vert, 3), np.float32)
        self.check(lib().admm_b200_get_state(self.h, _p(x), _p(v), self.n_vert), "get_state")
        return x, v

    def set_state(self, x: np.ndarray, v: Optional[np.ndarray] = None):
        x = np.ascontiguousarray(x, np.float32)
        vv = None if v is None else np.ascontiguousarray(v, np.float32)
        self.check(lib().admm_b200_set_state(self.h, _p(x), None if vv is None else _p(vv), self.n_vert),
                   "set_state")

    def reset(self):
        self.check(lib().admm_b200_reset(self.h), "reset")

    def local_step(self):
        self.check(lib().admm_b200_local_step(self.h), "local_step")

    def global_step(self):
        self.check(lib().admm_b200_global_step(self.h), "global_step")

    def jacobi(self, sweeps: int):
        self.check(lib().admm_b200_jacobi(self.h, sweeps), "jacobi")

    def pre_integration(self):
        self.check(lib().admm_b200_pre_integration(self.h), "pre_integration")

    def contact_step(self):
        self.check(lib().admm_b200_contact_step(self.h), "contact_step")

    def detect(self, x: Optional[np.ndarray] = None, allow=()) -> int:
        cnt = ctypes.c_int32()
        if x is None:
            rc = lib().admm_b200_detect(self.h, ctypes.byref(cnt))
        else:
            xx = np.ascontiguousarray(x, np.float32)
            rc = lib().admm_b200_detect_host(self.h, _p(xx), self.n_vert, ctypes.byref(cnt))
        self.check(rc, "detect", allow=allow)
        return cnt.value

    def contacts(self) -> Dict[str, np.ndarray]:
        cnt = ctypes.c_int32()
        self.check(lib().admm_b200_contacts(self.h, None, None, None, None, None, 0, ctypes.byref(cnt)), "contacts")
        n = cnt.value
        k = max(n, 1)
        pairs = np.zeros((k, 4), np.int32)
        bary = np.zeros((k, 4), np.float32)
        nrm = np.zeros((k, 3), np.float32)
        pt = np.zeros((k, 3), np.float32)
        gap = np.zeros(k, np.float32)
        self.check(lib().admm_b200_contacts(self.h, _p(pairs, _i), _p(bary), _p(nrm), _p(pt), _p(gap), n,
                                            ctypes.byref(cnt)), "contacts")
        return {"pairs": pairs[:n], "bary": bary[:n], "normal": nrm[:n], "point": pt[:n], "gap": gap[:n]}

    def residuals(self):
        pr = ctypes.c_double()
        du = ctypes.c_double()
        self.check(lib().admm_b200_residuals(self.h, ctypes.byref(pr), ctypes.byref(du)), "residuals")
        return pr.value, du.value

    def last_step_device_ms(self) -> float:
        ms = ctypes.c_float()
        self.check(lib().admm_b200_last_step_device_ms(self.h, ctypes.byref(ms)), "last_step_device_ms")
        return ms.value

    def kernels_per_step(self) -> int:
        n = ctypes.c_int32()
        self.check(lib().admm_b200_kernels_per_step(self.h, ctypes.byref(n)), "kernels_per_step")
        return n.value

    def kernels_fallback(self) -> int:
        """Kernels of the plain solve that replaces a failed learned solve (0 unless learned)."""
        n = ctypes.c_int32()
        self.check(lib().admm_b200_kernels_fallback(self.h, ctypes.byref(n)), "kernels_fallback")
        return n.value

    def step_host(self, x_in: np.ndarray, v_in: Optional[np.ndarray], x_out: np.ndarray,
                  v_out: Optional[np.ndarray]) -> int:
        """One substep from/to host arrays (pinned for full speed), copies inside the call."""
        return self.check(lib().admm_b200_step_host(
            self.h, _p(x_in), None if v_in is None else _p(v_in), _p(x_out),
            None if v_out is None else _p(v_out), self.n_vert), "step_host",
            allow=(ERR_CONTACT_OVERFLOW, ERR_STACK_OVERFLOW))

    def set_profiling(self, on: bool):
        self.check(lib().admm_b200_set_profiling(self.h, 1 if on else 0), "set_profiling")

    def phase_times(self) -> Dict[str, Dict[str, float]]:
        ms = (ctypes.c_double * len(PHASES))()
        cnt = (ctypes.c_int64 * len(PHASES))()
        self.check(lib().admm_b200_phase_times(self.h, ms, cnt, len(PHASES)), "phase_times")
        return {p: {"ms": ms[i], "launches": cnt[i]} for i, p in enumerate(PHASES)}

    def set_probe(self, kernel: str):
        self.check(lib().admm_b200_set_probe(self.h, KERNELS[kernel]), "set_probe")

    def probe_time(self):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        self.check(lib().admm_b200_probe_time(self.h, ctypes.byref(ms), ctypes.byref(n)), "probe_time")
        return ms.value, n.value

    def tuning(self) -> Dict[str, float]:
        la, lr = ctypes.c_int32(), ctypes.c_int32()
        ma, mr = ctypes.c_float(), ctypes.c_float()
        self.check(lib().admm_b200_tuning(self.h, ctypes.byref(la), ctypes.byref(lr), ctypes.byref(ma),
                                          ctypes.byref(mr)), "tuning")
        return {"jacobi_lanes": la.value, "rhs_lanes": lr.value, "jacobi_ms": ma.value, "rhs_ms": mr.value}

    def set_preconditioner(self, blocks: np.ndarray):
        """Per-vertex 3x3 blocks (n_dyn x 9 or n_dyn x 3 x 3) for global_solver 2."""
        blk = np.ascontiguousarray(blocks, np.float32).reshape(self.n_dyn, 9)
        self.check(lib().admm_b200_set_preconditioner(self.h, _p(blk), self.n_dyn), "set_preconditioner")

    def set_learned(self, omega: np.ndarray, beta: np.ndarray, m: Optional[np.ndarray] = None,
                    theta: Optional[np.ndarray] = None):
        """Learned global step (global_solver 3): per-sweep (omega, beta), per-vertex m and theta."""
        om = np.ascontiguousarray(omega, np.float32).ravel()
        be = np.ascontiguousarray(beta, np.float32).ravel()
        if len(om) != len(be):
            raise ValueError("omega and beta need one entry per sweep")
        mm = None if m is None else np.ascontiguousarray(m, np.float32).reshape(self.n_dyn)
        th = None if theta is None else np.ascontiguousarray(theta, np.float32).reshape(self.n_dyn)
        self.check(lib().admm_b200_set_learned(self.h, len(om), _p(om), _p(be), None if mm is None else _p(mm),
                                               None if th is None else _p(th), self.n_dyn), "set_learned")

    def vertex_order(self) -> np.ndarray:
        """The caller's index of each internal vertex row (the library's storage order)."""
        out = np.zeros(self.n_vert, np.int32)
        self.check(lib().admm_b200_vertex_order(self.h, _p(out, _i), self.n_vert), "vertex_order")
        return out

    def learned_stats(self) -> Dict[str, int]:
        out = (ctypes.c_int64 * 4)()
        self.check(lib().admm_b200_learned_stats(self.h, out), "learned_stats")
        return {"substeps": out[0], "fallbacks": out[1], "solves": out[2], "failed_solves": out[3]}

    def record_global(self, iteration: int, allow=()):
        """One substep; (b, x_cur, x_last) of its global step number `iteration` (n_dyn x 3 each)."""
        nd = self.n_dyn
        b = np.zeros((nd, 3), np.float32)
        xc = np.zeros((nd, 3), np.float32)
        xl = np.zeros((nd, 3), np.float32)
        self.check(lib().admm_b200_record_global(self.h, iteration, _p(b), _p(xc), _p(xl), nd), "record_global",
                   allow)
        return b, xc, xl

    def set_rigid_track(self, v_begin: int, v_end: int, pos: np.ndarray, quat_xyzw: np.ndarray):
        """Static vertices [v_begin, v_end) follow pos[f] + quat[f] * rest (one row per frame)."""
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        quat = np.ascontiguousarray(quat_xyzw, np.float32).reshape(-1, 4)
        if len(pos) != len(quat):
            raise ValueError("pos and quat need one row per frame")
        self.check(lib().admm_b200_set_rigid_track(self.h, v_begin, v_end, len(pos), _p(pos), _p(quat)),
                   "set_rigid_track")

    def set_point_track(self, v_begin: int, v_end: int, points: np.ndarray, rot: np.ndarray,
                        translate: np.ndarray, scale: float):
        """Static vertices [v_begin, v_end) follow translate + rot (scale * points[f])."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, v_end - v_begin, 3)
        r = np.ascontiguousarray(rot, np.float32).reshape(9)
        t = np.ascontiguousarray(translate, np.float32).reshape(3)
        self.check(lib().admm_b200_set_point_track(self.h, v_begin, v_end, len(pts), _p(pts), _p(r), _p(t),
                                                   float(scale)), "set_point_track")

    def clear_tracks(self):
        self.check(lib().admm_b200_clear_tracks(self.h), "clear_tracks")

    def global_mode(self) -> Dict[str, float]:
        """Global-step mode: persistent kernel (and its grid) or one kernel per sweep."""
        pe, nb = ctypes.c_int32(), ctypes.c_int32()
        ms, mp = ctypes.c_float(), ctypes.c_float()
        self.check(lib().admm_b200_global_mode(self.h, ctypes.byref(pe), ctypes.byref(nb), ctypes.byref(ms),
                                               ctypes.byref(mp)), "global_mode")
        return {"mode": {0: "sweeps", 1: "persistent", 3: "tiled"}.get(pe.value, "?"), "persistent": pe.value == 1,
                "blocks": nb.value, "ms_sweeps": ms.value, "ms_persist": mp.value}

    def max_slots(self) -> int:
        n = ctypes.c_int32()
        self.check(lib().admm_b200_max_slots(self.h, ctypes.byref(n)), "max_slots")
        return n.value

    def peak_contact_count(self) -> int:
        n = ctypes.c_int32()
        self.check(lib().admm_b200_peak_contact_count(self.h, ctypes.byref(n)), "peak_contact_count")
        return n.value


# ----------------------------------------------------------------------------
# Mirrors of the reference contracts
# ----------------------------------------------------------------------------

class ADMMBackendB200:
    """Backend with the reference's ``IADMMBackend`` call order.

    ``apply_config`` -> ``add_constraints`` -> ``addPins`` -> ``set_constraint_dim``
    -> ``finalize_constraints`` -> ``init(verts, mass, dt)`` -> ``set_sync_to_host``
    -> ``step()`` ... -> ``reset()`` (``src/app/app_initializer.cpp:142-211``).  Here
    the constraint records come as a ``Scene`` (the per-type arrays the reference's
    ``convert_constraint2device`` builds, ``admm_impl_gpu.cu:61-96``).
    """

    def __init__(self, device: int = 0):
        self.device = device
        self._scene: Optional[Scene] = None
        self._cfg: Dict[str, object] = {}
        self._pins = set()
        self._dim: Optional[int] = None
        self._finalized = False
        self._h: Optional[Handle] = None
        self.sync_to_host = True
        self.m_vertices: Optional[np.ndarray] = None
        self.m_velocities: Optional[np.ndarray] = None
        self.step_metrics = []
        self.step_cnt = 0

    # IADMMBackend::apply_config (admm_backend.h:30)
    def apply_config(self, **cfg):
        if self._h is not None:
            raise AdmmError(ERR_STATE, "apply_config must come before init")
        self._cfg.update(cfg)

    # Solver::add_constraints (solver.h:96) -- records of one scene
    def add_constraints(self, scene: Scene):
        self._scene = scene

    # Solver::addPins (solver.h:150)
    def addPins(self, pin_inds):
        self._pins.update(int(p) for p in pin_inds)

    # IADMMBackend::set_constraint_dim (admm_backend.h:37)
    def set_constraint_dim(self, n: int):
        self._dim = int(n)

    # IADMMBackend::finalize_constraints (admm_backend.h:34)
    def finalize_constraints(self):
        if self._scene is None:
            raise AdmmError(ERR_STATE, "finalize_constraints before add_constraints")
        if self._dim is not None and self._dim != self._scene.n_rows:
            raise AdmmError(ERR_INVALID, f"constraint dim {self._dim} != rows {self._scene.n_rows}")
        self._finalized = True

    # Solver::init(verts, mass, dt) (solver.h:66-90) -> precompute
    def init(self, verts=None, mass=None, dt=None):
        if not self._finalized:
            raise AdmmError(ERR_STATE, "init before finalize_constraints")
        sc = self._scene
        if verts is not None:
            sc.verts = np.ascontiguousarray(verts, np.float32)
        if mass is not None:
            sc.mass = np.ascontiguousarray(mass, np.float32)
        if dt is not None:
            sc.params.dt = float(dt)
        if self._pins:
            sc.is_fixed = sc.is_fixed.copy()
            sc.is_fixed[sorted(p for p in self._pins if p < sc.n_vert)] = 1
        for k, v in self._cfg.items():
            setattr(sc.params, k, v)
        self._h = Handle(sc, self.device)
        self.m_vertices, self.m_velocities = self._h.get_state()

    def precompute(self):
        if self._h is None:
            self.init()

    def set_sync_to_host(self, enabled: bool):
        self.sync_to_host = bool(enabled)

    # IADMMBackend::step (admm_backend.h:17)
    def step(self):
        if self._h is None:
            raise AdmmError(ERR_STATE, "step before init")
        t0 = time.perf_counter()
        st = self._h.step(1, allow=(ERR_CONTACT_OVERFLOW, ERR_STACK_OVERFLOW))
        if self.sync_to_host:
            self.m_vertices, self.m_velocities = self._h.get_state()
        self.step_cnt += 1
        self.step_metrics.append({"frame": self.step_cnt, "step_ms": (time.perf_counter() - t0) * 1e3,
                                  "n_contacts": st["n_contacts"], "admm_iters": st["iters"],
                                  "primal_residual": st["primal"], "dual_residual": st["dual"],
                                  "status": st["status"]})
        return st

    def reset(self):
        self._h.reset()
        self.step_cnt = 0
        self.m_vertices, self.m_velocities = self._h.get_state()

    def getVertices(self):
        if not self.sync_to_host:
            self.m_vertices, self.m_velocities = self._h.get_state()
        return self.m_vertices

    def getVelocities(self):
        if not self.sync_to_host:
            self.m_vertices, self.m_velocities = self._h.get_state()
        return self.m_velocities

    def write_step_metrics_csv(self, path: str):
        """Solver::write_step_metrics_csv (solver.h:38-46), with residual columns added."""
        with open(path, "w") as f:
            f.write("frame,step_ms,n_contacts,admm_iters,primal_residual,dual_residual\n")
            for m in self.step_metrics:
                f.write(f"{m['frame']},{m['step_ms']},{m['n_contacts']},{m['admm_iters']},"
                        f"{m['primal_residual']},{m['dual_residual']}\n")

    @property
    def handle(self) -> Handle:
        return self._h

    def collision_detector(self) -> "BVHB200":
        return BVHB200(self._h)


class BVHB200:
    """ICollisionDetector over a handle (``src/contact/icollision_detector.h:19-47``)."""

    def __init__(self, h: Handle):
        self._h = h

    def detect(self, pos: np.ndarray):
        self._h.detect(pos, allow=(ERR_CONTACT_OVERFLOW, ERR_STACK_OVERFLOW))

    def contact_count(self) -> int:
        n = ctypes.c_int32()
        self._h.check(lib().admm_b200_contact_count(self._h.h, ctypes.byref(n)), "contact_count")
        return n.value

    def kernels_fallback(self) -> int:
        """Kernels of the plain solve that replaces a failed learned solve (0 unless learned)."""
        n = ctypes.c_int32()
        self.check(lib().admm_b200_kernels_fallback(self.h, ctypes.byref(n)), "kernels_fallback")
        return n.value

    def step_host(self, x_in: np.ndarray, v_in: Optional[np.ndarray], x_out: np.ndarray,
                  v_out: Optional[np.ndarray]) -> int:
        """One substep from/to host arrays (pinned for full speed), copies inside the call."""
        return self.check(lib().admm_b200_step_host(
            self.h, _p(x_in), None if v_in is None else _p(v_in), _p(x_out),
            None if v_out is None else _p(v_out), self.n_vert), "step_host",
            allow=(ERR_CONTACT_OVERFLOW, ERR_STACK_OVERFLOW))

    def set_profiling(self, on: bool):
        self.check(lib().admm_b200_set_profiling(self.h, 1 if on else 0), "set_profiling")

    def phase_times(self) -> Dict[str, Dict[str, float]]:
        ms = (ctypes.c_double * len(PHASES))()
        cnt = (ctypes.c_int64 * len(PHASES))()
        self.check(lib().admm_b200_phase_times(self.h, ms, cnt, len(PHASES)), "phase_times")
        return {p: {"ms": ms[i], "launches": cnt[i]} for i, p in enumerate(PHASES)}

    def set_probe(self, kernel: str):
        self.check(lib().admm_b200_set_probe(self.h, KERNELS[kernel]), "set_probe")

    def probe_time(self):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        self.check(lib().admm_b200_probe_time(self.h, ctypes.byref(ms), ctypes.byref(n)), "probe_time")
        return ms.value, n.value

    def max_slots(self) -> int:
        return self._h.max_slots()

    def peak_contact_count(self) -> int:
        return self._h.peak_contact_count()

    def points(self) -> np.ndarray:
        """Exactly max_slots() rows, unused slots zero (icollision_detector.h:35-39)."""
        c = self._h.contacts()
        out = np.zeros((self.max_slots(), 3), np.float32)
        out[:len(c["point"])] = c["point"]
        return out

    def normals(self) -> np.ndarray:
        c = self._h.contacts()
        out = np.zeros((self.max_slots(), 3), np.float32)
        out[:len(c["normal"])] = c["normal"]
        return out

    def clear(self):
        self._h.check(lib().admm_b200_clear_contacts(self._h.h), "clear")
