"""Host mirror of the reference's step interface, over the CUDA C ABI.

    VbdSolver(scene)                 ~ VbdSolver::new          (src/vbd.rs:101-192)
    VbdSolver.step(...)              ~ VbdSolver::step / GpuVbd::step (src/vbd.rs:250, src/gpu_vbd.rs:125)
    OgcWorld(x, triangles, moving)   ~ OgcWorld::new           (src/ogc/world.rs:126)
    OgcWorld.detect(...)             ~ OgcWorld::detect        (src/ogc/world.rs:308)
    OgcWorld.validate_start(...)     ~ OgcWorld::validate_start (src/ogc/world.rs:242)

Errors raise VbdError and leave the caller's state untouched, as the
reference's Result<_, String> does.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, native
from .abi import cc_candidates, cc_grab, cc_mesh, cc_metrics, cc_surface


class VbdError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__("[%d] %s" % (code, message))
        self.code = code
        self.message = message


def _f64p(a):
    return abi.ptr(a, C.c_double)


def _u32p(a):
    return abi.ptr(a, C.c_uint32)


def _grab_c(grab):
    if grab is None:
        return None
    g = cc_grab()
    for k in range(3):
        g.vertices[k] = int(grab["vertices"][k])
        g.weights[k] = float(grab["weights"][k])
        g.target[k] = float(grab["target"][k])
    g.stiffness = float(grab["stiffness"])
    return g


def _ref(obj, ctype):
    return C.byref(obj) if obj is not None else C.cast(None, C.POINTER(ctype))


def _settings_c(settings):
    return settings.to_c() if hasattr(settings, "to_c") else settings


def _ogc_c(settings):
    return settings.ogc_c() if hasattr(settings, "ogc_c") else settings


class OgcWorld:
    """OgcWorld on the GPU."""

    def __init__(self, x, triangles, moving, excluded=(), _handle=None, _owner=None):
        L = native.load()
        self._owner = _owner
        if _handle is not None:
            self.h = _handle
            self.owned = False
        else:
            x = abi.as_f64(x).reshape(-1, 3)
            t = abi.as_u32(triangles).reshape(-1, 3)
            ex = abi.as_u32(np.asarray(excluded, dtype=np.uint32).reshape(-1, 2))
            h = C.c_void_p()
            rc = L.cc_world_create(_f64p(x), len(x), _u32p(t), len(t), int(moving), _u32p(ex), len(ex), C.byref(h))
            if rc != 0:
                raise _global_error(rc)
            self.h = h
            self.owned = True
        self.moving = int(moving)

    def __del__(self):
        if getattr(self, "owned", False) and self.h:
            native.load().cc_world_destroy(self.h)
            self.h = None

    def _err(self, rc):
        buf = C.create_string_buffer(1024)
        native.load().cc_world_last_error(self.h, buf, 1024)
        return VbdError(rc, buf.value.decode())

    def validate_start(self, x):
        x = abi.as_f64(x).reshape(-1, 3)
        rc = native.load().cc_world_validate_start(self.h, _f64p(x))
        if rc != 0:
            raise self._err(rc)

    def detect(self, x, query_radius, settings) -> abi.ContactResult:
        x = abi.as_f64(x).reshape(-1, 3)
        s = _ogc_c(settings)
        L = native.load()
        r = abi.read_contacts(lambda out: L.cc_world_detect(self.h, _f64p(x), float(query_radius), C.byref(s),
                                                             C.byref(out)), self.moving)
        if isinstance(r, int):
            raise self._err(r)
        return r

    def candidates(self, x, radius):
        """Fresh broad-phase pairs at an exact search radius, sorted."""
        x = abi.as_f64(x).reshape(-1, 3)
        cap = 1 << 14
        while True:
            vf = np.zeros((cap, 2), np.uint32)
            ee = np.zeros((cap, 2), np.uint32)
            out = cc_candidates(cap, cap, _u32p(vf), _u32p(ee), 0, 0)
            rc = native.load().cc_world_candidates(self.h, _f64p(x), float(radius), C.byref(out))
            if rc == abi.CC_ERR_CAPACITY:
                cap = max(int(out.n_vf), int(out.n_ee)) + 1
                continue
            if rc != 0:
                raise self._err(rc)
            return vf[:out.n_vf].copy(), ee[:out.n_ee].copy()

    def set_tree_rebuild_period(self, period: int):
        """LBVH policy at a candidate rebuild: 0 refits the first build's
        trees (the reference's tree), k >= 1 rebuilds them every k-th time."""
        rc = native.load().cc_world_set_tree_rebuild_period(self.h, int(period))
        if rc != 0:
            raise self._err(rc)

    def edges(self):
        L = native.load()
        n = L.cc_world_edges(self.h, None)
        e = np.zeros((n, 2), np.uint32)
        L.cc_world_edges(self.h, _u32p(e))
        return e


def _global_error(rc):
    buf = C.create_string_buffer(1024)
    native.load().cc_global_last_error(buf, 1024)
    return VbdError(rc, buf.value.decode())


class VbdSolver:
    """VbdSolver with the whole step (detection included) on the GPU."""

    def __init__(self, scene):
        L = native.load()
        m, self._keep_m = scene.mesh.to_c()
        if scene.obstacle is not None:
            o, self._keep_o = scene.obstacle.to_c()
            op = C.byref(o)
        else:
            op = C.cast(None, C.POINTER(cc_surface))
        x0 = abi.as_f64(scene.x0)
        v0 = abi.as_f64(scene.v0)
        h = C.c_void_p()
        rc = L.cc_solver_create(C.byref(m), op, _f64p(x0), _f64p(v0), scene.n, C.byref(h))
        if rc != 0:
            raise _global_error(rc)
        self.h = h
        self.n = scene.n
        self.total = int(L.cc_solver_total(h))
        self.obstacle_x = None if scene.obstacle is None else abi.as_f64(scene.obstacle.vertices)
        self.world = OgcWorld(None, None, self.n, _handle=L.cc_solver_world(h), _owner=self)

    @classmethod
    def batch(cls, instances):
        """Many independent scenes stepped as one solver (cc_batch_create);
        state arrays hold the instances' vertices in order."""
        L = native.load()
        keep = []
        k = len(instances)
        meshes = (cc_mesh * k)()
        obst = (cc_surface * k)()
        xs = (abi.c_double_p * k)()
        vs = (abi.c_double_p * k)()
        for i, sc in enumerate(instances):
            m, km = sc.mesh.to_c()
            meshes[i] = m
            keep.append(km)
            if sc.obstacle is not None:
                o, ko = sc.obstacle.to_c()
                obst[i] = o
                keep.append(ko)
            x = abi.as_f64(sc.x0)
            v = abi.as_f64(sc.v0)
            keep += [x, v]
            xs[i] = _f64p(x)
            vs[i] = _f64p(v)
        h = C.c_void_p()
        rc = L.cc_batch_create(meshes, obst, xs, vs, k, C.byref(h))
        if rc != 0:
            raise _global_error(rc)
        self = cls.__new__(cls)
        self.h = h
        self.n = int(L.cc_solver_moving(h))
        self.total = int(L.cc_solver_total(h))
        obs = [sc.obstacle.vertices for sc in instances if sc.obstacle is not None]
        self.obstacle_x = abi.as_f64(np.concatenate(obs)) if obs else None
        self.world = OgcWorld(None, None, self.n, _handle=L.cc_solver_world(h), _owner=self)
        return self

    def instances(self):
        """(first vertex, vertex count) of each batched instance."""
        L = native.load()
        k = int(L.cc_batch_instances(self.h, None, None, 0))
        f = (C.c_uint64 * max(k, 1))()
        c = (C.c_uint64 * max(k, 1))()
        L.cc_batch_instances(self.h, f, c, k)
        return [(int(f[i]), int(c[i])) for i in range(k)]

    def __del__(self):
        if getattr(self, "h", None):
            native.load().cc_solver_destroy(self.h)
            self.h = None

    def _err(self, rc):
        buf = C.create_string_buffer(1024)
        native.load().cc_last_error(self.h, buf, 1024)
        return VbdError(rc, buf.value.decode())

    def positions(self, x):
        """OgcWorld::positions: cloth followed by the fixed obstacle."""
        x = abi.as_f64(x).reshape(-1, 3)
        return x if self.obstacle_x is None else np.ascontiguousarray(np.concatenate([x, self.obstacle_x]))

    def step(self, x, v, time, settings, grab=None):
        """One step from host arrays. Returns (x, v, time, metrics)."""
        x = abi.as_f64(x).copy()
        v = abi.as_f64(v).copy()
        t = C.c_double(time)
        m = cc_metrics()
        s = _settings_c(settings)
        g = _grab_c(grab)
        rc = native.load().cc_solver_step(self.h, _f64p(x), _f64p(v), C.byref(t), C.byref(s), _ref(g, cc_grab),
                                          C.byref(m))
        if rc != 0:
            raise self._err(rc)
        return x, v, t.value, m.as_dict()

    def step_into(self, x, v, time, settings, grab=None):
        """One step from host arrays, in place: x and v (C-contiguous float64
        [n, 3]; pinned memory makes the copies plain DMA) receive the new
        state, only when the step succeeds. Returns (time, metrics)."""
        for a in (x, v):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
                    and a.flags.writeable and a.shape == (self.n, 3)):
                raise ValueError("step_into needs writable C-contiguous float64 arrays of shape (%d, 3)" % self.n)
        t = C.c_double(time)
        m = cc_metrics()
        s = _settings_c(settings)
        g = _grab_c(grab)
        rc = native.load().cc_solver_step(self.h, _f64p(x), _f64p(v), C.byref(t), C.byref(s), _ref(g, cc_grab),
                                          C.byref(m))
        if rc != 0:
            raise self._err(rc)
        return t.value, m.as_dict()

    # device-resident stepping
    def set_state(self, x, v, time):
        x = abi.as_f64(x)
        v = abi.as_f64(v)
        rc = native.load().cc_solver_set_state(self.h, _f64p(x), _f64p(v), float(time))
        if rc != 0:
            raise self._err(rc)

    def get_state(self):
        x = np.zeros((self.n, 3))
        v = np.zeros((self.n, 3))
        t = C.c_double()
        rc = native.load().cc_solver_get_state(self.h, _f64p(x), _f64p(v), C.byref(t))
        if rc != 0:
            raise self._err(rc)
        return x, v, t.value

    # learned initial guess
    def set_mlp(self, mlp, precision=1):
        """Attach an Mlp (clothcraft_b200.learned.Mlp) for init_mode = 1;
        precision 0 = FP32 CUDA cores, 1 = FP16 tensor cores. None detaches."""
        self._mlp = mlp  # keep the network alive while attached
        rc = native.load().cc_solver_set_mlp(self.h, None if mlp is None else mlp.h, int(precision))
        if rc != 0:
            raise self._err(rc)

    def set_lanes(self, lanes: int):
        """Threads per vertex solve (1..32), or 0 to autotune on the next step.
        Two solvers give bitwise-identical steps only with the same lanes."""
        rc = native.load().cc_solver_set_lanes(self.h, int(lanes))
        if rc != 0:
            raise self._err(rc)
        return self

    def set_profiling(self, enable: bool):
        """Time each iteration's colour sweeps (metrics sweep_ms) with
        device-clock stamps written by the sweep kernels' first and last
        colour blocks, and the detection phases with CUDA events."""
        native.load().cc_solver_set_profiling(self.h, 1 if enable else 0)
        return self

    def set_graphs(self, enable: bool):
        """Launch each step's iteration chunks as CUDA graphs (bitwise the
        results of direct launches)."""
        native.load().cc_solver_set_graphs(self.h, 1 if enable else 0)
        return self

    def set_lanes32(self, lanes: int):
        """Threads per vertex solve of the FP32-assembly sweep (4, 8, 16 or 32,
        optionally | cap << 8), or 0 to autotune on the next FP32 step."""
        rc = native.load().cc_solver_set_lanes32(self.h, int(lanes))
        if rc != 0:
            raise self._err(rc)
        return self

    def last_step_trace(self):
        """(relative residual after each iteration, NaN where not evaluated;
        vertices clipped in each iteration) of the last step."""
        r = np.zeros(256)
        c = np.zeros(256, np.uint32)
        native.load().cc_solver_last_step_trace(self.h, _f64p(r), _u32p(c), 256)
        return r, c

    @property
    def free_vertices(self) -> int:
        return int(native.load().cc_solver_free_vertices(self.h))

    def step_sample(self, settings, features, targets, grab=None):
        """step_resident that also writes the step's training sample into the
        CUDA float32 tensors features [free, 24] and targets [free, 3]."""
        import torch

        rows = self.free_vertices
        for t, w in ((features, 24), (targets, 3)):
            if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and tuple(t.shape) == (rows, w)):
                raise ValueError("sample buffers must be contiguous CUDA float32 [%d, %d]" % (rows, w))
        torch.cuda.synchronize()
        m = cc_metrics()
        s = _settings_c(settings)
        g = _grab_c(grab)
        rc = native.load().cc_solver_step_sample(self.h, C.byref(s), _ref(g, cc_grab), C.c_void_p(features.data_ptr()),
                                                 C.c_void_p(targets.data_ptr()), C.byref(m))
        if rc != 0:
            raise self._err(rc)
        return m.as_dict()

    def step_resident(self, settings, grab=None):
        m = cc_metrics()
        s = _settings_c(settings)
        g = _grab_c(grab)
        rc = native.load().cc_solver_step_resident(self.h, C.byref(s), _ref(g, cc_grab), C.byref(m))
        if rc != 0:
            raise self._err(rc)
        return m.as_dict()

    def newton_step(self, x_old, v_old, settings, newton_iterations=30, pcg_iterations=500, abs_tol=1e-6,
                    rel_tol=1e-4):
        """FP64 Newton reference step on the GPU from (x_old, v_old) with the
        step's OGC contacts frozen (src/solver.rs:422-646 plus the contact
        terms). Returns (x, report dict); the solver's state is not changed."""
        x_old = abi.as_f64(x_old)
        v_old = abi.as_f64(v_old)
        out = np.zeros((self.n, 3))
        rep = abi.cc_newton_report()
        s = _settings_c(settings)
        rc = native.load().cc_solver_newton_step(self.h, _f64p(x_old), _f64p(v_old), C.byref(s),
                                                 int(newton_iterations), int(pcg_iterations), float(abs_tol),
                                                 float(rel_tol), _f64p(out), C.byref(rep))
        if rc != 0:
            raise self._err(rc)
        return out, rep.as_dict()

    def colors(self, x_all, query_radius, ogc, grab=None):
        x_all = abi.as_f64(x_all)
        out = np.zeros(self.n, np.uint32)
        nc = C.c_uint32()
        g = _grab_c(grab)
        o = _ogc_c(ogc)
        rc = native.load().cc_solver_colors(self.h, _f64p(x_all), float(query_radius), C.byref(o), _ref(g, cc_grab),
                                            _u32p(out), C.byref(nc))
        if rc != 0:
            raise self._err(rc)
        return out, int(nc.value)

    def local_blocks(self, x_all, query_radius, settings, grab=None, targets=None, inertia=None):
        x_all = abi.as_f64(x_all)
        n = self.n
        e = np.zeros(n)
        g = np.zeros((n, 3))
        h = np.zeros((n, 9))
        t = None if targets is None else abi.as_f64(targets)
        m = None if inertia is None else abi.as_f64(inertia)
        s = _settings_c(settings)
        gr = _grab_c(grab)
        rc = native.load().cc_solver_local_blocks(self.h, _f64p(x_all), float(query_radius), C.byref(s),
                                                  _ref(gr, cc_grab), _f64p(t), _f64p(m), _f64p(e), _f64p(g),
                                                  _f64p(h))
        if rc != 0:
            raise self._err(rc)
        return e, g, h.reshape(n, 3, 3)
