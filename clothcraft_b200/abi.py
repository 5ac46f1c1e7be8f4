"""ctypes mirror of include/clothcraft.h (structure layouts only).

Kept free of any library loading so that both the CUDA library binding and
test tooling can share one definition of the C structures.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

CC_OK = 0
CC_ERR_INVALID_ARGUMENT = 1
CC_ERR_INVALID_STATE = 2
CC_ERR_CONTACT = 3
CC_ERR_NON_FINITE = 4
CC_ERR_CAPACITY = 5
CC_ERR_CUDA = 6
CC_ERR_DEVICE_TIMEOUT = 7

KIND_NAMES = ("PointPoint", "PointEdge", "PointFace", "EdgeEdge")

c_double_p = C.POINTER(C.c_double)
c_uint32_p = C.POINTER(C.c_uint32)
c_uint8_p = C.POINTER(C.c_uint8)
c_uint64_p = C.POINTER(C.c_uint64)


class cc_material(C.Structure):
    _fields_ = [(name, C.c_double) for name in (
        "warp", "weft", "shear", "compression_ratio", "compression_transition",
        "bend_warp", "bend_weft", "density", "thickness", "grain_degrees")]


class cc_mesh(C.Structure):
    _fields_ = [
        ("n_vertices", C.c_uint64),
        ("n_triangles", C.c_uint64),
        ("triangles", c_uint32_p),
        ("inv_dm", c_double_p),
        ("area", c_double_p),
        ("triangle_material", c_uint32_p),
        ("n_hinges", C.c_uint64),
        ("hinges", c_uint32_p),
        ("hinge_weight", c_double_p),
        ("hinge_across", c_double_p),
        ("hinge_material", c_uint32_p),
        ("n_materials", C.c_uint64),
        ("materials", C.POINTER(cc_material)),
        ("masses", c_double_p),
        ("pinned", c_uint8_p),
        ("pin_positions", c_double_p),
        ("n_stitches", C.c_uint64),
        ("stitch_offsets", c_uint32_p),
        ("stitch_vertices", c_uint32_p),
        ("stitch_weights", c_double_p),
        ("stitch_stiffness", c_double_p),
    ]


class cc_surface(C.Structure):
    _fields_ = [
        ("n_vertices", C.c_uint64),
        ("vertices", c_double_p),
        ("n_triangles", C.c_uint64),
        ("triangles", c_uint32_p),
    ]


class cc_ogc_settings(C.Structure):
    _fields_ = [("radius", C.c_double), ("stiffness", C.c_double),
                ("relaxation", C.c_double), ("refresh_fraction", C.c_double)]


class cc_vbd_settings(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("iterations", C.c_uint32),
        ("init_mode", C.c_uint32),
        ("damping", C.c_double),
        ("gravity", C.c_double * 3),
        ("contact", cc_ogc_settings),
        ("residual_tolerance", C.c_double),
        ("residual_check_every", C.c_uint32),
        ("stall_refresh", C.c_uint32),
        ("acceleration", C.c_double),
        ("sweep_precision", C.c_uint32),
        ("reserved1", C.c_uint32),
    ]


CC_SWEEP_FP64 = 0
CC_SWEEP_FP32 = 1


class cc_grab(C.Structure):
    _fields_ = [
        ("vertices", C.c_uint32 * 3),
        ("reserved0", C.c_uint32),
        ("weights", C.c_double * 3),
        ("target", C.c_double * 3),
        ("stiffness", C.c_double),
    ]


class cc_metrics(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "time_s", "dt_s", "step_ms", "detection_ms", "solve_ms", "gpu_compute_ms",
        "refit_ms", "candidates_ms", "narrow_ms")] + [(n, C.c_uint64) for n in (
            "candidate_pairs", "aabb_rejections", "iterations", "contacts", "contact_terms",
            "detection_updates", "broad_phase_rebuilds", "truncated_vertices", "colors")] + [
        (n, C.c_double) for n in (
            "minimum_distance_m", "max_seam_gap_m", "extension_p95_percent",
            "extension_max_percent", "residual_rms_n")] + [
        ("has_residual", C.c_int32), ("reserved0", C.c_int32),
        ("sweep_ms", C.c_double)] + [(n, C.c_uint64) for n in (
            "sweep_launches", "vertex_solves", "kernel_launches", "contact_incidence")] + [
        ("color_ms", C.c_double), ("color_rounds", C.c_uint64),
        ("relative_residual", C.c_double), ("initial_relative_residual", C.c_double),
        ("has_relative_residual", C.c_int32), ("init_used", C.c_int32),
        ("init_energy_adaptive", C.c_double), ("init_energy_learned", C.c_double),
        ("init_ms", C.c_double), ("relative_force_residual", C.c_double)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved0"}
        d["residual_rms_n"] = d["residual_rms_n"] if d.pop("has_residual") else None
        if not d.pop("has_relative_residual"):
            d["relative_residual"] = d["initial_relative_residual"] = d["relative_force_residual"] = None
        return d


class cc_newton_report(C.Structure):
    _fields_ = [
        ("converged", C.c_int32),
        ("iterations", C.c_uint32),
        ("pcg_iterations", C.c_uint64),
        ("residual_rms_n", C.c_double),
        ("objective_j", C.c_double),
        ("relative_force_residual", C.c_double),
        ("contact_terms", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["converged"] = bool(d["converged"])
        return d


class cc_contacts(C.Structure):
    _fields_ = [
        ("contact_capacity", C.c_uint64),
        ("incident_capacity", C.c_uint64),
        ("radii_capacity", C.c_uint64),
        ("kinds", c_uint8_p),
        ("vertices", c_uint32_p),
        ("counts", c_uint8_p),
        ("mollifier_epsilon", c_double_p),
        ("incident_offsets", c_uint64_p),
        ("incident", c_uint32_p),
        ("radii", c_double_p),
        ("n_contacts", C.c_uint64),
        ("n_incident", C.c_uint64),
        ("active_contacts", C.c_uint64),
        ("vertex_face_candidates", C.c_uint64),
        ("edge_edge_candidates", C.c_uint64),
        ("candidate_pairs", C.c_uint64),
        ("aabb_rejections", C.c_uint64),
        ("minimum_distance", C.c_double),
        ("broad_phase_rebuilt", C.c_int32),
        ("reserved0", C.c_int32),
    ]


class cc_candidates(C.Structure):
    _fields_ = [
        ("vf_capacity", C.c_uint64), ("ee_capacity", C.c_uint64),
        ("vf", c_uint32_p), ("ee", c_uint32_p),
        ("n_vf", C.c_uint64), ("n_ee", C.c_uint64),
    ]


def ptr(a: np.ndarray | None, ctype):
    """Pointer to a contiguous numpy array (or NULL)."""
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


def as_f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def as_u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


class ContactResult(dict):
    """ContactSet fields as numpy arrays / scalars."""


def read_contacts(call, moving: int, contact_hint: int = 4096) -> ContactResult:
    """Two-call protocol around a cc_contacts-filling function."""
    cap = contact_hint
    while True:
        out = cc_contacts()
        kinds = np.zeros(cap, np.uint8)
        verts = np.zeros((cap, 4), np.uint32)
        counts = np.zeros(cap, np.uint8)
        eps = np.zeros(cap)
        inc_off = np.zeros(moving + 1, np.uint64)
        inc = np.zeros(4 * cap, np.uint32)
        radii = np.zeros(max(moving, 1))
        out.contact_capacity = cap
        out.incident_capacity = 4 * cap
        out.radii_capacity = moving
        out.kinds = ptr(kinds, C.c_uint8)
        out.vertices = ptr(verts, C.c_uint32)
        out.counts = ptr(counts, C.c_uint8)
        out.mollifier_epsilon = ptr(eps, C.c_double)
        out.incident_offsets = ptr(inc_off, C.c_uint64)
        out.incident = ptr(inc, C.c_uint32)
        out.radii = ptr(radii, C.c_double)
        rc = call(out)
        if rc == CC_ERR_CAPACITY:
            cap = max(int(out.n_contacts), int(out.n_incident) // 4 + 1, 2 * cap)
            continue
        if rc != CC_OK:
            return rc
        k = int(out.n_contacts)
        r = ContactResult(
            kinds=kinds[:k].copy(), vertices=verts[:k].copy(), counts=counts[:k].copy(), epsilon=eps[:k].copy(),
            incident_offsets=inc_off.copy(), incident=inc[:int(out.n_incident)].copy(), radii=radii[:moving].copy(),
            active_contacts=int(out.active_contacts), vertex_face_candidates=int(out.vertex_face_candidates),
            edge_edge_candidates=int(out.edge_edge_candidates), candidate_pairs=int(out.candidate_pairs),
            aabb_rejections=int(out.aabb_rejections), minimum_distance=float(out.minimum_distance),
            broad_phase_rebuilt=bool(out.broad_phase_rebuilt))
        return r
