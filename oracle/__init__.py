"""Oracle: FP64 CPU restatement of ClothCraft's reference CPU path.

TEST INFRASTRUCTURE ONLY. The product library (clothcraft_b200) never imports,
links or calls anything here; tests, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py use it as the checker
and as the timed CPU baseline.

Parity is pinned against the reference's own known-answer tests (tests/ogc.rs,
tests/ogc_bvh.rs, tests/ogc_cache.rs, tests/vbd.rs, src/vbd/coloring.rs,
src/vbd/prediction.rs, src/ogc/world.rs tests), ported in tests/test_oracle_*.py.
The Rust reference cannot be compiled in this environment (no cargo/rustc),
so no compiled copy of the reference exists to compare against.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from clothcraft_b200 import abi
from clothcraft_b200.abi import read_contacts, ContactResult  # noqa: F401
from clothcraft_b200.abi import (c_double_p, c_uint32_p, c_uint8_p, c_uint64_p, cc_candidates, cc_contacts,
                                 cc_grab, cc_mesh, cc_metrics, cc_ogc_settings, cc_surface, cc_vbd_settings)

from .build import build as _build

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = _build()
        L = C.CDLL(str(path))
        vp = C.c_void_p
        sig = {
            "or_global_last_error": (C.c_int32, [C.c_char_p, C.c_uint64]),
            "or_last_error": (C.c_int32, [vp, C.c_char_p, C.c_uint64]),
            "or_world_last_error": (C.c_int32, [vp, C.c_char_p, C.c_uint64]),
            "or_set_threads": (C.c_int32, [vp, C.c_int32]),
            "or_solver_create": (C.c_int32, [C.POINTER(cc_mesh), C.POINTER(cc_surface), c_double_p, c_double_p,
                                             C.c_uint64, C.POINTER(vp)]),
            "or_solver_destroy": (None, [vp]),
            "or_solver_moving": (C.c_uint64, [vp]),
            "or_solver_total": (C.c_uint64, [vp]),
            "or_solver_world": (vp, [vp]),
            "or_solver_step": (C.c_int32, [vp, c_double_p, c_double_p, c_double_p, C.POINTER(cc_vbd_settings),
                                           C.POINTER(cc_grab), C.POINTER(cc_metrics)]),
            "or_solver_set_learned_correction": (C.c_int32, [vp, C.POINTER(C.c_float), C.c_uint64]),
            "or_solver_colors": (C.c_int32, [vp, c_double_p, C.c_double, C.POINTER(cc_ogc_settings),
                                             C.POINTER(cc_grab), c_uint32_p, c_uint32_p]),
            "or_solver_local_blocks": (C.c_int32, [vp, c_double_p, C.c_double, C.POINTER(cc_vbd_settings),
                                                   C.POINTER(cc_grab), c_double_p, c_double_p, c_double_p,
                                                   c_double_p, c_double_p]),
            "or_world_create": (C.c_int32, [c_double_p, C.c_uint64, c_uint32_p, C.c_uint64, C.c_uint64,
                                            c_uint32_p, C.c_uint64, C.POINTER(vp)]),
            "or_world_destroy": (None, [vp]),
            "or_world_validate_start": (C.c_int32, [vp, c_double_p]),
            "or_world_detect": (C.c_int32, [vp, c_double_p, C.c_double, C.POINTER(cc_ogc_settings),
                                            C.POINTER(cc_contacts)]),
            "or_world_detect_unpruned": (C.c_int32, [vp, c_double_p, C.c_double, C.POINTER(cc_ogc_settings),
                                                     C.POINTER(cc_contacts)]),
            "or_world_candidates": (C.c_int32, [vp, c_double_p, C.c_double, C.POINTER(cc_candidates)]),
            "or_world_edges": (C.c_uint64, [vp, c_uint32_p]),
            "or_activation_jet1": (None, [C.c_double, C.c_double, C.c_double, c_double_p]),
            "or_activation": (C.c_double, [C.c_double, C.c_double, C.c_double]),
            "or_contact_value": (C.c_double, [C.c_uint8, C.c_uint8, C.c_double, c_double_p, C.c_double,
                                              C.c_double]),
            "or_contact_block": (None, [C.c_uint8, C.c_uint8, C.c_double, c_double_p, C.c_uint32, C.c_double,
                                        C.c_double, c_double_p, c_double_p, c_double_p]),
            "or_membrane_element": (None, [c_double_p, c_double_p, C.c_double, C.POINTER(abi.cc_material),
                                           c_double_p, c_double_p, c_double_p]),
            "or_bending_element": (None, [c_double_p, C.c_double, c_double_p, C.POINTER(abi.cc_material),
                                          c_double_p, c_double_p, c_double_p]),
            "or_closest_triangle": (C.c_int32, [c_double_p, c_double_p]),
            "or_closest_segments": (None, [c_double_p, c_double_p]),
            "or_segment_triangle": (C.c_int32, [c_double_p]),
            "or_edge_feasible": (C.c_int32, [c_double_p, C.c_uint64, c_uint32_p, C.c_uint64, c_double_p,
                                             C.c_uint32, C.c_uint32]),
            "or_bvh_create": (vp, [c_double_p, c_uint8_p, C.c_uint64]),
            "or_bvh_destroy": (None, [vp]),
            "or_bvh_refit_dynamic": (None, [vp, c_double_p, C.c_uint64]),
            "or_bvh_pairs": (C.c_uint64, [vp, vp, C.c_double, C.c_int32, c_uint32_p, C.c_uint64]),
            "or_bvh_query": (C.c_uint64, [vp, c_double_p, C.c_int32, c_uint32_p, C.c_uint64]),
            "or_bounds_distance_squared": (C.c_double, [c_double_p, c_double_p]),
            "or_prediction_create": (vp, []),
            "or_prediction_destroy": (None, [vp]),
            "or_prediction_guess": (None, [vp, c_double_p, c_double_p, C.c_uint64, C.c_double,
                                           C.POINTER(cc_vbd_settings), c_double_p]),
            "or_prediction_record": (None, [vp, c_double_p, c_double_p, c_double_p, C.c_uint64, C.c_double,
                                            C.POINTER(cc_vbd_settings)]),
            "or_greedy_colors": (C.c_uint32, [C.c_uint64, c_uint64_p, c_uint32_p, C.POINTER(cc_contacts),
                                              C.POINTER(cc_grab), c_uint32_p]),
            "or_extension_percent": (None, [C.POINTER(cc_mesh), c_double_p, c_double_p]),
            "or_newton_step": (C.c_int32, [vp, c_double_p, c_double_p, C.POINTER(cc_vbd_settings), C.c_int32,
                                           C.c_int32, C.c_double, C.c_double, C.c_int32, c_double_p, c_double_p,
                                           C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
            "or_step_gradient": (C.c_int32, [vp, c_double_p, c_double_p, C.POINTER(cc_vbd_settings), c_double_p,
                                             C.c_int32, c_double_p, c_double_p]),
            "or_mlp_parameter_count": (C.c_uint64, []),
            "or_mlp_forward": (C.c_int32, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_uint64, c_double_p]),
            "or_mlp_gradients": (C.c_int32, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                             C.c_uint64, c_double_p, c_double_p]),
            "or_learned_features": (C.c_int32, [vp, c_double_p, c_double_p, C.c_double, C.POINTER(cc_vbd_settings),
                                                C.POINTER(C.c_float)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


class OracleError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__("[%d] %s" % (code, message))
        self.code = code
        self.message = message


def _global_error(code):
    buf = C.create_string_buffer(1024)
    lib().or_global_last_error(buf, 1024)
    return OracleError(code, buf.value.decode())


def f64p(a):
    return abi.ptr(a, C.c_double)


def u32p(a):
    return abi.ptr(a, C.c_uint32)


def grab_c(grab):
    """grab: None or dict(vertices, weights, target, stiffness)."""
    if grab is None:
        return None
    g = cc_grab()
    for k in range(3):
        g.vertices[k] = int(grab["vertices"][k])
        g.weights[k] = float(grab["weights"][k])
        g.target[k] = float(grab["target"][k])
    g.stiffness = float(grab["stiffness"])
    return g


def _byref_or_null(obj, ctype):
    return C.byref(obj) if obj is not None else C.cast(None, C.POINTER(ctype))


class World:
    """OgcWorld (src/ogc/world.rs) on the oracle."""

    def __init__(self, x, triangles, moving, excluded=(), _handle=None, _owner=None):
        L = lib()
        if _handle is not None:
            self.h = _handle
            self._owner = _owner
            self.owned = False
        else:
            x = abi.as_f64(x).reshape(-1, 3)
            t = abi.as_u32(triangles).reshape(-1, 3)
            ex = abi.as_u32(np.asarray(excluded, dtype=np.uint32).reshape(-1, 2))
            h = C.c_void_p()
            rc = L.or_world_create(f64p(x), len(x), u32p(t), len(t), int(moving), u32p(ex), len(ex), C.byref(h))
            if rc != 0:
                raise _global_error(rc)
            self.h = h
            self.owned = True
        self.n_all = None
        self.moving = int(moving)

    def __del__(self):
        if getattr(self, "owned", False) and self.h:
            lib().or_world_destroy(self.h)
            self.h = None

    def _err(self, rc):
        buf = C.create_string_buffer(1024)
        lib().or_world_last_error(self.h, buf, 1024)
        return OracleError(rc, buf.value.decode())

    def validate_start(self, x):
        x = abi.as_f64(x).reshape(-1, 3)
        rc = lib().or_world_validate_start(self.h, f64p(x))
        if rc != 0:
            raise self._err(rc)

    def detect(self, x, query_radius, settings: cc_ogc_settings, prune: bool = True) -> ContactResult:
        x = abi.as_f64(x).reshape(-1, 3)
        fn = lib().or_world_detect if prune else lib().or_world_detect_unpruned
        r = read_contacts(lambda out: fn(self.h, f64p(x), float(query_radius), C.byref(settings), C.byref(out)),
                          self.moving)
        if isinstance(r, int):
            raise self._err(r)
        return r

    def candidates(self, x, radius):
        x = abi.as_f64(x).reshape(-1, 3)
        cap = 1 << 14
        while True:
            vf = np.zeros((cap, 2), np.uint32)
            ee = np.zeros((cap, 2), np.uint32)
            out = cc_candidates(cap, cap, u32p(vf), u32p(ee), 0, 0)
            rc = lib().or_world_candidates(self.h, f64p(x), float(radius), C.byref(out))
            if rc == abi.CC_ERR_CAPACITY:
                cap = max(int(out.n_vf), int(out.n_ee)) + 1
                continue
            if rc != 0:
                raise self._err(rc)
            return vf[:out.n_vf].copy(), ee[:out.n_ee].copy()

    def edges(self):
        n = lib().or_world_edges(self.h, None)
        e = np.zeros((n, 2), np.uint32)
        lib().or_world_edges(self.h, u32p(e))
        return e


class Solver:
    """VbdSolver (src/vbd.rs) on the oracle, driven through the C entry points."""

    def __init__(self, scene, threads: int = 1):
        L = lib()
        m, self._keep_m = scene.mesh.to_c()
        if scene.obstacle is not None:
            o, self._keep_o = scene.obstacle.to_c()
            op = C.byref(o)
        else:
            op = C.cast(None, C.POINTER(cc_surface))
        x0 = abi.as_f64(scene.x0)
        v0 = abi.as_f64(scene.v0)
        h = C.c_void_p()
        rc = L.or_solver_create(C.byref(m), op, f64p(x0), f64p(v0), scene.n, C.byref(h))
        if rc != 0:
            raise _global_error(rc)
        self.h = h
        self.n = scene.n
        self.total = int(L.or_solver_total(h))
        self.obstacle_x = None if scene.obstacle is None else abi.as_f64(scene.obstacle.vertices)
        self._pinned = np.asarray(scene.mesh.pinned).astype(bool)
        L.or_set_threads(h, int(threads))
        self.world = World(None, None, self.n, _handle=L.or_solver_world(h), _owner=self)

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_solver_destroy(self.h)
            self.h = None

    def set_threads(self, threads: int):
        lib().or_set_threads(self.h, int(threads))

    def _err(self, rc):
        buf = C.create_string_buffer(1024)
        lib().or_last_error(self.h, buf, 1024)
        return OracleError(rc, buf.value.decode())

    def positions(self, x):
        """OgcWorld::positions: cloth followed by the fixed obstacle."""
        x = abi.as_f64(x).reshape(-1, 3)
        return x if self.obstacle_x is None else np.ascontiguousarray(np.concatenate([x, self.obstacle_x]))

    def step(self, x, v, time, settings: cc_vbd_settings, grab=None):
        """Returns (x, v, time, metrics); raises OracleError (state untouched)."""
        x = abi.as_f64(x).copy()
        v = abi.as_f64(v).copy()
        t = C.c_double(time)
        m = cc_metrics()
        g = grab_c(grab)
        rc = lib().or_solver_step(self.h, f64p(x), f64p(v), C.byref(t), C.byref(settings),
                                  _byref_or_null(g, cc_grab), C.byref(m))
        if rc != 0:
            raise self._err(rc)
        return x, v, t.value, m.as_dict()

    def set_learned_correction(self, corr):
        """Network output ([free vertices, 3] float32, vertex order) that the
        next step with init_mode = 1 turns into the library's learned guess."""
        c = np.ascontiguousarray(corr, dtype=np.float32).reshape(-1, 3)
        rc = lib().or_solver_set_learned_correction(self.h, c.ctypes.data_as(C.POINTER(C.c_float)), c.shape[0])
        if rc != 0:
            raise self._err(rc)

    def newton_step(self, x_old, v_old, settings: cc_vbd_settings, newton_iterations=30, pcg_iterations=250,
                    abs_tol=1e-6, rel_tol=1e-4, threads=8):
        """FP64 Newton-PCG step (src/solver.rs:422-646) with the OGC contacts
        detected at x_old frozen. Returns (x, residual_rms, converged, iterations)."""
        xo = abi.as_f64(x_old)
        vo = abi.as_f64(v_old)
        out = np.zeros((self.n, 3))
        res = C.c_double()
        conv = C.c_int32()
        its = C.c_int32()
        rc = lib().or_newton_step(self.h, f64p(xo), f64p(vo), C.byref(settings), newton_iterations, pcg_iterations,
                                  abs_tol, rel_tol, threads, f64p(out), C.byref(res), C.byref(conv), C.byref(its))
        if rc != 0:
            raise OracleError(rc, "Newton step failed")
        return out, res.value, bool(conv.value), its.value

    def learned_features(self, x, v, time, settings: cc_vbd_settings):
        """The 24 learned-guess features of the step starting at (x, v, time)
        with this solver's prediction history; [free vertices, 24] float32."""
        x = abi.as_f64(x)
        v = abi.as_f64(v)
        rows = int(np.count_nonzero(~self._pinned)) if hasattr(self, "_pinned") else None
        if rows is None:
            raise OracleError(1, "solver built without pin information")
        out = np.zeros((rows, 24), np.float32)
        rc = lib().or_learned_features(self.h, f64p(x), f64p(v), float(time), C.byref(settings),
                                       out.ctypes.data_as(C.POINTER(C.c_float)))
        if rc != 0:
            raise OracleError(rc, "feature evaluation failed")
        return out

    def step_gradient(self, x_old, v_old, settings: cc_vbd_settings, x_eval, threads=8):
        """Objective and gradient (pinned dofs zero) of the step from
        (x_old, v_old) at x_eval, OGC contacts detected at x_old frozen."""
        xo = abi.as_f64(x_old)
        vo = abi.as_f64(v_old)
        xe = abi.as_f64(x_eval)
        g = np.zeros((self.n, 3))
        e = C.c_double()
        rc = lib().or_step_gradient(self.h, f64p(xo), f64p(vo), C.byref(settings), f64p(xe), threads, C.byref(e),
                                    f64p(g))
        if rc != 0:
            raise OracleError(rc, "objective evaluation failed")
        return e.value, g

    def relative_residual(self, x_old, v_old, settings: cc_vbd_settings, x_eval, threads=8):
        """||grad E(x_eval)|| / ||grad E(y)|| over free vertices, y the
        inertial target (the step's convergence measure)."""
        xo = abi.as_f64(x_old).reshape(-1, 3)
        vo = abi.as_f64(v_old).reshape(-1, 3)
        damp = 1.0 + settings.damping * settings.dt
        g = np.array([settings.gravity[0], settings.gravity[1], settings.gravity[2]])
        y = xo + (vo * settings.dt + g * settings.dt * settings.dt) / damp
        _, gx = self.step_gradient(xo, vo, settings, x_eval, threads)
        _, gy = self.step_gradient(xo, vo, settings, y, threads)
        return float(np.linalg.norm(gx) / np.linalg.norm(gy))

    def colors(self, x_all, query_radius, ogc: cc_ogc_settings, grab=None):
        x_all = abi.as_f64(x_all)
        out = np.zeros(self.n, np.uint32)
        nc = C.c_uint32()
        g = grab_c(grab)
        rc = lib().or_solver_colors(self.h, f64p(x_all), float(query_radius), C.byref(ogc),
                                    _byref_or_null(g, cc_grab), u32p(out), C.byref(nc))
        if rc != 0:
            raise self._err(rc)
        return out, int(nc.value)

    def local_blocks(self, x_all, query_radius, settings: cc_vbd_settings, grab=None, targets=None, inertia=None):
        x_all = abi.as_f64(x_all)
        n = self.n
        e = np.zeros(n)
        g = np.zeros((n, 3))
        h = np.zeros((n, 9))
        t = None if targets is None else abi.as_f64(targets)
        m = None if inertia is None else abi.as_f64(inertia)
        gr = grab_c(grab)
        rc = lib().or_solver_local_blocks(self.h, f64p(x_all), float(query_radius), C.byref(settings),
                                          _byref_or_null(gr, cc_grab), f64p(t), f64p(m), f64p(e), f64p(g), f64p(h))
        if rc != 0:
            raise self._err(rc)
        return e, g, h.reshape(n, 3, 3)


class Bvh:
    """Bvh over explicit boxes (src/ogc/bvh.rs), for tests/ogc_bvh.rs."""

    def __init__(self, boxes, dynamic):
        self.boxes = abi.as_f64(boxes).reshape(-1, 6)
        d = np.ascontiguousarray(dynamic, dtype=np.uint8)
        self.h = lib().or_bvh_create(f64p(self.boxes), abi.ptr(d, C.c_uint8), len(self.boxes))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_bvh_destroy(self.h)
            self.h = None

    def refit_dynamic(self, boxes):
        b = abi.as_f64(boxes).reshape(-1, 6)
        lib().or_bvh_refit_dynamic(self.h, f64p(b), len(b))

    def pairs(self, other, radius, same=False):
        cap = 1 << 16
        out = np.zeros((cap, 2), np.uint32)
        k = lib().or_bvh_pairs(self.h, (other or self).h, float(radius), int(same), u32p(out), cap)
        assert k <= cap
        return out[:k].copy()

    def query(self, box6, dynamic_only):
        cap = 1 << 16
        out = np.zeros(cap, np.uint32)
        b = abi.as_f64(box6)
        k = lib().or_bvh_query(self.h, f64p(b), int(dynamic_only), u32p(out), cap)
        return out[:k].copy()


def mlp_forward(params, features):
    """FP64 forward of the 24-64-64-64-3 GELU MLP (parameters and features float32)."""
    p = np.ascontiguousarray(params, np.float32)
    f = np.ascontiguousarray(features, np.float32)
    out = np.zeros((f.shape[0], 3))
    lib().or_mlp_forward(p.ctypes.data_as(C.POINTER(C.c_float)), f.ctypes.data_as(C.POINTER(C.c_float)), f.shape[0],
                         f64p(out))
    return out


def mlp_gradients(params, features, targets):
    """FP64 gradient and value of mean_s |MLP(f_s) - t_s|^2."""
    p = np.ascontiguousarray(params, np.float32)
    f = np.ascontiguousarray(features, np.float32)
    t = np.ascontiguousarray(targets, np.float32)
    g = np.zeros(p.size)
    loss = C.c_double()
    rc = lib().or_mlp_gradients(p.ctypes.data_as(C.POINTER(C.c_float)), f.ctypes.data_as(C.POINTER(C.c_float)),
                                t.ctypes.data_as(C.POINTER(C.c_float)), f.shape[0], f64p(g), C.byref(loss))
    if rc != 0:
        raise OracleError(rc, "MLP gradient failed")
    return g, loss.value
