"""Seeded synthetic scenes: cloth meshes, obstacles and step settings.

Mesh formulas follow the reference's model builder (src/model.rs:124-227):
inverse rest matrices, area/3 mass lumping, hinge pairing and weight
3|e|^2/(A1+A2), across = normalised perpendicular of the rest edge. Grid
sheets here may use one uniform diagonal and more than 128 cells, which the
reference's Pattern::build does not allow, so the mesh is written directly
with the same formulas. `pattern_build` reproduces Pattern::build itself
(alternating diagonals) for the reference's own test fixtures.

All scenes are generated from seeds; no external dataset is involved.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi


# --------------------------------------------------------------- materials
@dataclass
class Material:
    """Material (src/model.rs:7-38); defaults are the reference defaults."""
    warp: float = 350.0
    weft: float = 180.0
    shear: float = 45.0
    compression_ratio: float = 0.15
    compression_transition: float = 0.005
    bend_warp: float = 0.00008
    bend_weft: float = 0.00004
    density: float = 0.2
    thickness: float = 0.001
    grain_degrees: float = 0.0

    @staticmethod
    def stvk_mapped(mu: float = 1.0e4, lam: float = 2.0e4, bending: float = 1e-5,
                    density: float = 0.2) -> "Material":
        """StVK (mu, lambda) mapped onto the reference law: warp = weft = lambda + 2 mu,
        shear = mu, compression_ratio = 1 (pure quadratic). This equals StVK without
        the lambda*E11*E22 coupling, which the reference law cannot express."""
        return Material(warp=lam + 2 * mu, weft=lam + 2 * mu, shear=mu, compression_ratio=1.0,
                        compression_transition=0.005, bend_warp=bending, bend_weft=bending,
                        density=density, thickness=0.001, grain_degrees=0.0)

    def to_c(self) -> abi.cc_material:
        return abi.cc_material(self.warp, self.weft, self.shear, self.compression_ratio,
                               self.compression_transition, self.bend_warp, self.bend_weft,
                               self.density, self.thickness, self.grain_degrees)


# -------------------------------------------------------------------- mesh
@dataclass
class Mesh:
    """Cloth mesh arrays in the layout of cc_mesh."""
    uv: np.ndarray                 # [n,2]
    triangles: np.ndarray          # [T,3] uint32
    inv_dm: np.ndarray             # [T,4]
    area: np.ndarray               # [T]
    triangle_material: np.ndarray  # [T] uint32
    hinges: np.ndarray             # [H,4] uint32
    hinge_weight: np.ndarray       # [H]
    hinge_across: np.ndarray       # [H,2]
    hinge_material: np.ndarray     # [H] uint32
    materials: list
    rest_area: np.ndarray          # [n]
    masses: np.ndarray             # [n]
    pinned: np.ndarray             # [n] uint8
    pin_positions: np.ndarray      # [n,3]
    stitch_offsets: np.ndarray = field(default_factory=lambda: np.zeros(1, np.uint32))
    stitch_vertices: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    stitch_weights: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    stitch_stiffness: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))

    @property
    def n(self) -> int:
        return int(self.uv.shape[0])

    def to_c(self):
        """Return (cc_mesh, keepalive); keep the second object alive while the
        struct is in use."""
        arrays = dict(
            triangles=abi.as_u32(self.triangles), inv_dm=abi.as_f64(self.inv_dm),
            area=abi.as_f64(self.area), triangle_material=abi.as_u32(self.triangle_material),
            hinges=abi.as_u32(self.hinges).reshape(-1, 4), hinge_weight=abi.as_f64(self.hinge_weight),
            hinge_across=abi.as_f64(self.hinge_across).reshape(-1, 2),
            hinge_material=abi.as_u32(self.hinge_material), masses=abi.as_f64(self.masses),
            pinned=np.ascontiguousarray(self.pinned, dtype=np.uint8),
            pin_positions=abi.as_f64(self.pin_positions),
            stitch_offsets=abi.as_u32(self.stitch_offsets), stitch_vertices=abi.as_u32(self.stitch_vertices),
            stitch_weights=abi.as_f64(self.stitch_weights), stitch_stiffness=abi.as_f64(self.stitch_stiffness),
        )
        mats = (abi.cc_material * max(1, len(self.materials)))(*[m.to_c() for m in self.materials])
        m = abi.cc_mesh()
        m.n_vertices = self.n
        m.n_triangles = len(self.triangles)
        m.triangles = abi.ptr(arrays["triangles"], C.c_uint32)
        m.inv_dm = abi.ptr(arrays["inv_dm"], C.c_double)
        m.area = abi.ptr(arrays["area"], C.c_double)
        m.triangle_material = abi.ptr(arrays["triangle_material"], C.c_uint32)
        m.n_hinges = len(arrays["hinges"])
        m.hinges = abi.ptr(arrays["hinges"], C.c_uint32)
        m.hinge_weight = abi.ptr(arrays["hinge_weight"], C.c_double)
        m.hinge_across = abi.ptr(arrays["hinge_across"], C.c_double)
        m.hinge_material = abi.ptr(arrays["hinge_material"], C.c_uint32)
        m.n_materials = len(self.materials)
        m.materials = C.cast(mats, C.POINTER(abi.cc_material))
        m.masses = abi.ptr(arrays["masses"], C.c_double)
        m.pinned = abi.ptr(arrays["pinned"], C.c_uint8)
        m.pin_positions = abi.ptr(arrays["pin_positions"], C.c_double)
        m.n_stitches = len(self.stitch_stiffness)
        m.stitch_offsets = abi.ptr(arrays["stitch_offsets"], C.c_uint32)
        m.stitch_vertices = abi.ptr(arrays["stitch_vertices"], C.c_uint32)
        m.stitch_weights = abi.ptr(arrays["stitch_weights"], C.c_double)
        m.stitch_stiffness = abi.ptr(arrays["stitch_stiffness"], C.c_double)
        return m, (arrays, mats)


@dataclass
class Obstacle:
    """Fixed obstacle, SurfaceMesh (src/avatar.rs:8-11)."""
    vertices: np.ndarray   # [m,3]
    triangles: np.ndarray  # [f,3]

    def to_c(self):
        v = abi.as_f64(self.vertices)
        t = abi.as_u32(self.triangles)
        s = abi.cc_surface(len(v), abi.ptr(v, C.c_double), len(t), abi.ptr(t, C.c_uint32))
        return s, (v, t)


def inverse_rest(uv: np.ndarray, tri: np.ndarray):
    """DMat2::from_cols(r1-r0, r2-r0).inverse() and 0.5|det| per triangle, in
    glam's operation order (determinant, recip, cofactors)."""
    r0, r1, r2 = uv[tri[:, 0]], uv[tri[:, 1]], uv[tri[:, 2]]
    e1 = r1 - r0
    e2 = r2 - r0
    a, b = e1[:, 0], e1[:, 1]
    c, d = e2[:, 0], e2[:, 1]
    det = a * d - c * b
    inv = 1.0 / det
    inv_dm = np.stack([d * inv, b * -inv, c * -inv, a * inv], axis=1)
    area = 0.5 * np.abs(det)
    return inv_dm, area


def build_hinges(uv: np.ndarray, tri: np.ndarray, area: np.ndarray):
    """Hinge pairing of Pattern::build (src/model.rs:193-211): a hinge is made
    when the second triangle of an edge is visited, [a, b, c, d] with a->b the
    edge in that triangle, c its opposite vertex and d the first triangle's."""
    T = len(tri)
    if T == 0:
        return (np.zeros((0, 4), np.uint32), np.zeros(0), np.zeros((0, 2)))
    k0 = np.arange(3)
    a = tri[:, k0].reshape(-1).astype(np.int64)
    b = tri[:, (k0 + 1) % 3].reshape(-1).astype(np.int64)
    c = tri[:, (k0 + 2) % 3].reshape(-1).astype(np.int64)
    t_of = np.repeat(np.arange(T), 3)
    n = int(max(a.max(), b.max())) + 1
    key = np.minimum(a, b) * n + np.maximum(a, b)
    order = np.argsort(key, kind="stable")
    ks = key[order]
    same = np.nonzero(ks[1:] == ks[:-1])[0]
    if len(same) and np.any(np.diff(same) == 1):
        raise ValueError("non-manifold edge with more than two triangles")
    first = order[same]
    second = order[same + 1]
    # hinges are emitted in visiting order of the second half-edge
    emit = np.argsort(second, kind="stable")
    first, second = first[emit], second[emit]
    ha, hb, hc, hd = a[second], b[second], c[second], c[first]
    edge = uv[hb] - uv[ha]
    weight = 3.0 * (edge[:, 0] * edge[:, 0] + edge[:, 1] * edge[:, 1]) / (area[t_of[first]] + area[t_of[second]])
    across = np.stack([-edge[:, 1], edge[:, 0]], axis=1)
    across = across / np.sqrt((across * across).sum(axis=1))[:, None]
    hinges = np.stack([ha, hb, hc, hd], axis=1).astype(np.uint32)
    return hinges, weight, across


def build_mesh(uv: np.ndarray, tri: np.ndarray, material: Material) -> Mesh:
    """One panel: rest data, hinges, lumped masses (src/model.rs:164-214)."""
    uv = np.ascontiguousarray(uv, dtype=np.float64)
    tri = np.ascontiguousarray(tri, dtype=np.uint32)
    n = len(uv)
    inv_dm, area = inverse_rest(uv, tri.astype(np.int64))
    rest_area = np.zeros(n)
    for k in range(3):  # accumulate area/3 in triangle order
        np.add.at(rest_area, tri[:, k].astype(np.int64), area / 3.0)
    hinges, weight, across = build_hinges(uv, tri.astype(np.int64), area)
    return Mesh(
        uv=uv, triangles=tri, inv_dm=inv_dm, area=area,
        triangle_material=np.zeros(len(tri), np.uint32),
        hinges=hinges, hinge_weight=weight, hinge_across=across,
        hinge_material=np.zeros(len(hinges), np.uint32), materials=[material],
        rest_area=rest_area, masses=rest_area * material.density,
        pinned=np.zeros(n, np.uint8), pin_positions=np.zeros((n, 3)))


def concat_meshes(meshes: list) -> Mesh:
    """Panels side by side with their own materials (GarmentTemplate::compile,
    src/garment/template.rs:320-370)."""
    off = 0
    parts = dict(uv=[], triangles=[], inv_dm=[], area=[], triangle_material=[], hinges=[],
                 hinge_weight=[], hinge_across=[], hinge_material=[], rest_area=[], masses=[],
                 pinned=[], pin_positions=[])
    materials = []
    for m in meshes:
        mat0 = len(materials)
        materials.extend(m.materials)
        parts["uv"].append(m.uv)
        parts["triangles"].append(m.triangles.astype(np.int64) + off)
        parts["inv_dm"].append(m.inv_dm)
        parts["area"].append(m.area)
        parts["triangle_material"].append(m.triangle_material + mat0)
        parts["hinges"].append(m.hinges.astype(np.int64) + off)
        parts["hinge_weight"].append(m.hinge_weight)
        parts["hinge_across"].append(m.hinge_across)
        parts["hinge_material"].append(m.hinge_material + mat0)
        parts["rest_area"].append(m.rest_area)
        parts["masses"].append(m.masses)
        parts["pinned"].append(m.pinned)
        parts["pin_positions"].append(m.pin_positions)
        off += m.n
    cat = {k: np.concatenate(v) for k, v in parts.items()}
    return Mesh(uv=cat["uv"], triangles=cat["triangles"].astype(np.uint32), inv_dm=cat["inv_dm"],
                area=cat["area"], triangle_material=cat["triangle_material"].astype(np.uint32),
                hinges=cat["hinges"].astype(np.uint32).reshape(-1, 4), hinge_weight=cat["hinge_weight"],
                hinge_across=cat["hinge_across"].reshape(-1, 2),
                hinge_material=cat["hinge_material"].astype(np.uint32), materials=materials,
                rest_area=cat["rest_area"], masses=cat["masses"], pinned=cat["pinned"].astype(np.uint8),
                pin_positions=cat["pin_positions"])


def grid_triangles(nx: int, ny: int, alternate: bool) -> np.ndarray:
    """Cells of an nx x ny vertex grid. alternate=True is Pattern::build's
    checkerboard of diagonals (src/model.rs:164-176); False splits every cell
    on the same diagonal [a,b,d],[a,d,c]."""
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="xy")
    i = i.reshape(-1)
    j = j.reshape(-1)
    a = j * nx + i
    b = a + 1
    c = a + nx
    d = c + 1
    t1 = np.stack([a, b, d], axis=1)
    t2 = np.stack([a, d, c], axis=1)
    if alternate:
        odd = (i + j) % 2 == 1
        t1[odd] = np.stack([a, b, c], axis=1)[odd]
        t2[odd] = np.stack([b, d, c], axis=1)[odd]
    return np.stack([t1, t2], axis=1).reshape(-1, 3).astype(np.uint32)


def grid_uv(nx: int, ny: int, width: float, height: float) -> np.ndarray:
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    return np.stack([width * i.reshape(-1) / (nx - 1), height * j.reshape(-1) / (ny - 1)], axis=1)


def pattern_build(width: float, height: float, nx_cells: int, ny_cells: int, material: Material) -> Mesh:
    """Pattern::build (src/model.rs:124-227) without its 128-cell limit check."""
    return build_mesh(grid_uv(nx_cells + 1, ny_cells + 1, width, height),
                      grid_triangles(nx_cells + 1, ny_cells + 1, alternate=True), material)


def euler_xyz(deg) -> np.ndarray:
    """Rotation R = Rx * Ry * Rz (Placement, src/garment/template.rs:76-92)."""
    rx, ry, rz = (math.radians(float(d)) for d in deg)
    cx, sx, cy, sy, cz, sz = math.cos(rx), math.sin(rx), math.cos(ry), math.sin(ry), math.cos(rz), math.sin(rz)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rx @ Ry @ Rz


def icosphere(subdivisions: int, radius: float, center=(0.0, 0.0, 0.0)) -> Obstacle:
    """Outward-oriented icosphere: 10*4^s + 2 vertices, 20*4^s faces."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        new = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new
    v = np.array(verts) * radius + np.asarray(center, dtype=np.float64)
    return Obstacle(vertices=v, triangles=np.array(faces, dtype=np.uint32))


def capsule(radius: float, height: float, segments: int = 32, rings: int = 8, cylinder_rings: int = 24,
            center=(0.0, 0.0, 0.0)) -> Obstacle:
    """Closed capsule along y: a cylinder of `height` between two hemispheres."""
    c = np.asarray(center, dtype=np.float64)
    rows = []
    half = 0.5 * height
    for k in range(rings - 1, 0, -1):  # bottom hemisphere, pole excluded
        phi = -0.5 * math.pi * k / rings
        rows.append((radius * math.cos(phi), -half + radius * math.sin(phi)))
    for k in range(cylinder_rings + 1):
        rows.append((radius, -half + height * k / cylinder_rings))
    for k in range(1, rings):
        phi = 0.5 * math.pi * k / rings
        rows.append((radius * math.cos(phi), half + radius * math.sin(phi)))
    verts = [c + np.array([0.0, -half - radius, 0.0])]
    for r, y in rows:
        for s in range(segments):
            th = 2 * math.pi * s / segments
            verts.append(c + np.array([r * math.cos(th), y, r * math.sin(th)]))
    verts.append(c + np.array([0.0, half + radius, 0.0]))
    faces = []
    R = len(rows)
    idx = lambda ring, s: 1 + ring * segments + (s % segments)
    for s in range(segments):
        faces.append((0, idx(0, s), idx(0, s + 1)))
    for ring in range(R - 1):
        for s in range(segments):
            a, b = idx(ring, s), idx(ring, s + 1)
            cc, d = idx(ring + 1, s), idx(ring + 1, s + 1)
            faces += [(a, cc, b), (b, cc, d)]
    top = len(verts) - 1
    for s in range(segments):
        faces.append((top, idx(R - 1, s + 1), idx(R - 1, s)))
    return Obstacle(vertices=np.array(verts), triangles=np.array(faces, dtype=np.uint32))


# ------------------------------------------------------------------ scenes
@dataclass
class StepSettings:
    """VbdSettings (src/vbd.rs:18-36) with OgcSettings (src/ogc/world.rs:45-54)."""
    dt: float = 1.0 / 240.0
    iterations: int = 16
    damping: float = 1.5
    gravity: tuple = (0.0, -9.81, 0.0)
    radius: float = 0.003
    stiffness: float = 100000.0
    relaxation: float = 0.45
    refresh_fraction: float = 0.01
    init_mode: int = 0  # 0 adaptive (reference), 1 learned
    residual_tolerance: float = 0.0
    residual_check_every: int = 0
    stall_refresh: int = 0
    acceleration: float = 0.0  # Chebyshev rho; 0 = off (the reference)
    sweep_precision: int = 0  # 0 FP64 sweeps (the CPU path's arithmetic), 1 FP32 element assembly

    def to_c(self) -> abi.cc_vbd_settings:
        s = abi.cc_vbd_settings()
        s.dt = self.dt
        s.iterations = self.iterations
        s.init_mode = self.init_mode
        s.residual_tolerance = self.residual_tolerance
        s.residual_check_every = self.residual_check_every
        s.stall_refresh = self.stall_refresh
        s.acceleration = self.acceleration
        s.sweep_precision = self.sweep_precision
        s.damping = self.damping
        for k in range(3):
            s.gravity[k] = self.gravity[k]
        s.contact = abi.cc_ogc_settings(self.radius, self.stiffness, self.relaxation, self.refresh_fraction)
        return s

    def ogc_c(self) -> abi.cc_ogc_settings:
        return abi.cc_ogc_settings(self.radius, self.stiffness, self.relaxation, self.refresh_fraction)


@dataclass
class Scene:
    name: str
    mesh: Mesh
    obstacle: Obstacle | None
    x0: np.ndarray
    v0: np.ndarray
    settings: StepSettings
    steps: int
    note: str = ""

    @property
    def n(self) -> int:
        return self.mesh.n


def _rotation_about(angle_x_deg: float, angle_z_deg: float) -> np.ndarray:
    ax, az = math.radians(angle_x_deg), math.radians(angle_z_deg)
    Rx = np.array([[1, 0, 0], [0, math.cos(ax), -math.sin(ax)], [0, math.sin(ax), math.cos(ax)]])
    Rz = np.array([[math.cos(az), -math.sin(az), 0], [math.sin(az), math.cos(az), 0], [0, 0, 1]])
    return Rz @ Rx


def sheet(nx: int, side: float, height: float, material: Material, *, jitter: float = 0.0,
          tilt_deg: tuple = (0.0, 0.0), seed: int = 0, pins=()) -> tuple:
    """Square nx x nx vertex sheet of `side` metres, horizontal at y=height
    (x,z centred on the origin), uniform diagonal, optional seeded jitter and
    tilt about x then z through its centre. Returns (mesh, x0)."""
    mesh = build_mesh(grid_uv(nx, nx, side, side), grid_triangles(nx, nx, alternate=False), material)
    uv = mesh.uv
    x = np.stack([uv[:, 0] - 0.5 * side, np.full(len(uv), height), uv[:, 1] - 0.5 * side], axis=1)
    if tilt_deg != (0.0, 0.0):
        R = _rotation_about(*tilt_deg)
        c = np.array([0.0, height, 0.0])
        x = (x - c) @ R.T + c
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        x = x + rng.uniform(-jitter, jitter, size=x.shape)
    for p in pins:
        mesh.pinned[p] = 1
        mesh.pin_positions[p] = x[p]
    return mesh, np.ascontiguousarray(x)


def config0(seed: int = 0, n_side: int = 64) -> Scene:
    """64x64 sheet (4,096 v / 7,938 t), 0.5 m, y=0.3, jitter U(+-1e-4) m, two
    adjacent corners pinned, icosphere r=0.1 (2,562 v) at the origin; dt 1/60,
    20 iterations, contact radius 2 mm, stiffness 1e4 N/m, 200 steps."""
    mesh, x = sheet(n_side, 0.5, 0.3, Material.stvk_mapped(), jitter=1e-4, seed=seed, pins=(0, n_side - 1))
    return Scene("sheet64_sphere", mesh, icosphere(4, 0.1), x, np.zeros_like(x),
                 StepSettings(dt=1 / 60, iterations=20, damping=1.5, radius=0.002, stiffness=1e4), 200)


def config1(seed: int = 1, n_side: int = 256) -> Scene:
    """256x256 sheet (65,536 v / 130,050 t), 1 m, y=0.5, seeded tilt U(+-30 deg)
    about x and z, icosphere r=0.3 below; self-contact radius 1 mm, 30
    iterations, dt 1/60, 300 steps."""
    rng = np.random.default_rng(seed)
    tilt = tuple(float(a) for a in rng.uniform(-30.0, 30.0, size=2))
    mesh, x = sheet(n_side, 1.0, 0.5, Material.stvk_mapped(), tilt_deg=tilt, seed=seed)
    return Scene("sheet256_fold", mesh, icosphere(4, 0.3), x, np.zeros_like(x),
                 StepSettings(dt=1 / 60, iterations=30, damping=1.5, radius=0.001, stiffness=1e4), 300,
                 note="tilt_deg=%.3f,%.3f" % tilt)


def config4(seed: int = 4, n_side: int = 1024) -> Scene:
    """1024x1024 sheet (1,048,576 v / 2,093,058 t), 1 m, four corners pinned
    (driven inward at 0.2 m/s by the caller), radius 0.5 mm, 40 iterations."""
    c = (0, n_side - 1, n_side * (n_side - 1), n_side * n_side - 1)
    mesh, x = sheet(n_side, 1.0, 0.5, Material.stvk_mapped(), jitter=1e-5, seed=seed, pins=c)
    return Scene("sheet1024_crumple", mesh, None, x, np.zeros_like(x),
                 StepSettings(dt=1 / 60, iterations=40, damping=1.5, radius=0.0005, stiffness=1e4), 120)


def poisson_disk(width: float, height: float, r: float, seed: int, boundary_step: float | None = None,
                 k: int = 30) -> tuple:
    """Seeded Poisson-disk sample of the rectangle [0,w]x[0,h] with minimum
    spacing r (Bridson 2007: background grid of cell r/sqrt 2, k annulus
    candidates per active point, tested together). The perimeter is sampled
    first at a fixed step (default r) so that two panels of the same size share
    their edge points exactly; interior points keep a distance >= r from all
    points. Returns (points, number of perimeter points first in the list)."""
    rng = np.random.default_rng(seed)
    step = r if boundary_step is None else boundary_step
    border = []
    for (x0, y0, x1, y1) in ((0, 0, width, 0), (width, 0, width, height), (width, height, 0, height),
                             (0, height, 0, 0)):
        m = max(1, int(round(math.hypot(x1 - x0, y1 - y0) / step)))
        for i in range(m):  # corners once (start of each side)
            t = i / m
            border.append((x0 + t * (x1 - x0), y0 + t * (y1 - y0)))
    border = np.asarray(border)
    cell = r / math.sqrt(2.0)
    gw, gh = int(math.ceil(width / cell)) + 1, int(math.ceil(height / cell)) + 1
    grid = -np.ones((gw, gh), dtype=np.int64)
    cap = len(border) + int(2.0 * width * height / (r * r)) + 16
    pts = np.empty((cap, 2))
    count = 0

    def put(p):
        nonlocal count
        pts[count] = p
        grid[min(int(p[0] / cell), gw - 1), min(int(p[1] / cell), gh - 1)] = count
        count += 1
        return count - 1

    for p in border:
        put(p)
    nbr = int(math.ceil(3.0 * r / cell)) + 1
    active = [put((rng.uniform(r, width - r), rng.uniform(r, height - r)))]
    r2 = r * r
    while active:
        j = int(rng.integers(len(active)))
        base = pts[active[j]]
        ang = rng.uniform(0.0, 2.0 * math.pi, k)
        rad = r * np.sqrt(rng.uniform(1.0, 4.0, k))
        cand = base + np.stack([rad * np.cos(ang), rad * np.sin(ang)], axis=1)
        ok = ((cand[:, 0] >= 0.5 * r) & (cand[:, 0] <= width - 0.5 * r) & (cand[:, 1] >= 0.5 * r) &
              (cand[:, 1] <= height - 0.5 * r))
        gx, gy = int(base[0] / cell), int(base[1] / cell)
        ids = grid[max(gx - nbr, 0):gx + nbr + 1, max(gy - nbr, 0):gy + nbr + 1].ravel()
        near = pts[ids[ids >= 0]]
        bsel = border[(np.abs(border[:, 0] - base[0]) < 3 * r) & (np.abs(border[:, 1] - base[1]) < 3 * r)]
        near = np.concatenate([near, bsel]) if len(bsel) else near
        if len(near):
            d2 = ((cand[:, None, :] - near[None, :, :]) ** 2).sum(axis=2).min(axis=1)
            ok &= d2 >= r2
        hit = np.nonzero(ok)[0]
        if len(hit):
            active.append(put(cand[hit[0]]))
        else:
            active[j] = active[-1]
            active.pop()
    return pts[:count].copy(), len(border)


def delaunay_panel(uv: np.ndarray) -> np.ndarray:
    """Delaunay triangles of the panel points (scipy Qhull), counter-clockwise,
    without degenerate (area < 1e-12 of the mean) triangles."""
    from scipy.spatial import Delaunay

    tri = Delaunay(uv).simplices.astype(np.int64)
    a, b, c = uv[tri[:, 0]], uv[tri[:, 1]], uv[tri[:, 2]]
    cr = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])
    tri[cr < 0] = tri[cr < 0][:, [0, 2, 1]]
    keep = np.abs(cr) > 1e-12 * np.abs(cr).mean()
    return tri[keep].astype(np.uint32)


def config3(seed: int = 3, spacing: float = 0.0036) -> Scene:
    """Sewn garment proxy: two 0.6 x 0.7 m panels (seeded Poisson-disk points,
    ~20k each, Delaunay triangles) 5 cm either side of a fixed vertical
    capsule (r 0.15 m, cylinder 1.2 m), joined along both side edges and the
    outer shoulders by 1e3 N/m penalty sewing springs [(a,+1),(b,-1)] whose
    vertex pairs are excluded from contact (src/vbd.rs:128-144). Material as
    config 0, contact radius 1 mm, dt 1/60, 20 iterations."""
    W, H = 0.6, 0.7
    mat = Material.stvk_mapped()
    panels, borders = [], []
    for side in range(2):
        uv, nb = poisson_disk(W, H, spacing, seed * 1009 + side, boundary_step=spacing)
        tri = delaunay_panel(uv)
        if side == 1:
            tri = tri[:, [0, 2, 1]]  # back panel faces outward
        panels.append(build_mesh(uv, tri, mat))
        borders.append(nb)
    mesh = concat_meshes(panels)
    n0 = panels[0].n
    cap_r, cap_h, gap = 0.15, 1.2, 0.05
    y0 = 0.5 * cap_h + cap_r - H  # top edge level with the capsule's top
    xs = []
    for side, zsign in ((0, 1.0), (1, -1.0)):
        uv = panels[side].uv
        xs.append(np.stack([uv[:, 0] - 0.5 * W, y0 + uv[:, 1], np.full(len(uv), zsign * (cap_r + gap))], axis=1))
    x = np.ascontiguousarray(np.concatenate(xs))
    # seams: perimeter points are identical on both panels (same order, same uv)
    ub = panels[0].uv[:borders[0]]
    assert np.array_equal(ub, panels[1].uv[:borders[1]])
    side_seam = (np.abs(ub[:, 0]) < 1e-12) | (np.abs(ub[:, 0] - W) < 1e-12)
    shoulder = (np.abs(ub[:, 1] - H) < 1e-12) & ((ub[:, 0] <= 0.2 + 1e-12) | (ub[:, 0] >= W - 0.2 - 1e-12))
    ids = np.nonzero(side_seam | shoulder)[0]
    mesh.stitch_offsets = np.arange(0, 2 * len(ids) + 1, 2, dtype=np.uint32)
    mesh.stitch_vertices = np.stack([ids, ids + n0], axis=1).ravel().astype(np.uint32)
    mesh.stitch_weights = np.tile([1.0, -1.0], len(ids))
    mesh.stitch_stiffness = np.full(len(ids), 1e3)
    return Scene("garment_capsule", mesh, capsule(cap_r, cap_h), x, np.zeros_like(x),
                 StepSettings(dt=1 / 60, iterations=20, damping=1.5, radius=0.001, stiffness=1e4), 120,
                 note="seed=%d, %d stitches" % (seed, len(ids)))


def config2_instances(seed: int = 2, count: int = 96, sides=(32, 320), pitch: float = 3.0) -> list:
    """Batched uneven instances: `count` square sheets whose vertex side is
    drawn from U{sides} (1k-102k vertices each, ~3.6M in total for 96), at the
    config-0 vertex spacing (0.5 m / 63 cells), 1-4 random corners pinned,
    moduli x U(0.5, 2) of config 0's, each with its own icosphere below it
    (r = 0.2 side, sheet 0.6 side above its centre). Instances sit on a
    10-wide grid `pitch` m apart, so no two come within contact range.
    Contact radius 2 mm, stiffness 1e4 N/m, dt 1/60 s, 20 iterations."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(sides[0], sides[1] + 1))
        side = (n - 1) * (0.5 / 63)
        scale = float(rng.uniform(0.5, 2.0))
        mat = Material.stvk_mapped(mu=1.0e4 * scale, lam=2.0e4 * scale)
        corners = np.array([0, n - 1, n * (n - 1), n * n - 1])
        pins = tuple(int(c) for c in np.sort(rng.choice(corners, int(rng.integers(1, 5)), replace=False)))
        mesh, x = sheet(n, side, 0.6 * side, mat, jitter=1e-4, seed=seed * 100003 + k, pins=pins)
        off = np.array([(k % 10) * pitch, 0.0, (k // 10) * pitch])
        x = np.ascontiguousarray(x + off)
        mesh.pin_positions[list(pins)] += off
        obs = icosphere(3, 0.2 * side, center=tuple(off))
        out.append(Scene("batch%d_sheet%d" % (k, n), mesh, obs, x, np.zeros_like(x),
                         StepSettings(dt=1 / 60, iterations=20, damping=1.5, radius=0.002, stiffness=1e4), 120,
                         note="side %d, pins %s, moduli x%.3f" % (n, pins, scale)))
    return out


def batch_scene(instances: list) -> Scene:
    """The union of instances as one scene (vertex order = instance order,
    obstacles concatenated), the layout cc_batch_create builds."""
    mesh = concat_meshes([sc.mesh for sc in instances])
    so, sv, sw, sk = [np.zeros(1, np.uint32)], [], [], []
    off, base = 0, 0
    for sc in instances:
        m = sc.mesh
        so.append(m.stitch_offsets[1:].astype(np.int64) + base)
        sv.append(m.stitch_vertices.astype(np.int64) + off)
        sw.append(m.stitch_weights)
        sk.append(m.stitch_stiffness)
        base += len(m.stitch_vertices)
        off += m.n
    mesh.stitch_offsets = np.concatenate(so).astype(np.uint32)
    mesh.stitch_vertices = np.concatenate(sv).astype(np.uint32)
    mesh.stitch_weights = np.concatenate(sw).astype(np.float64)
    mesh.stitch_stiffness = np.concatenate(sk).astype(np.float64)
    verts, faces, ob = [], [], 0
    for sc in instances:
        if sc.obstacle is not None:
            verts.append(sc.obstacle.vertices)
            faces.append(sc.obstacle.triangles.astype(np.int64) + ob)
            ob += len(sc.obstacle.vertices)
    obs = Obstacle(np.concatenate(verts), np.concatenate(faces).astype(np.uint32)) if verts else None
    x = np.ascontiguousarray(np.concatenate([sc.x0 for sc in instances]))
    v = np.ascontiguousarray(np.concatenate([sc.v0 for sc in instances]))
    return Scene("batch%d" % len(instances), mesh, obs, x, v, instances[0].settings, instances[0].steps,
                 note="%d instances, %d vertices" % (len(instances), len(x)))


def partition_instances(sizes, parts: int) -> list:
    """Greedy longest-first bin packing of instances (by vertex count) onto
    `parts` GPUs: returns, per part, the ascending instance indices."""
    loads = [0] * parts
    bins = [[] for _ in range(parts)]
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        p = min(range(parts), key=lambda q: (loads[q], q))
        bins[p].append(i)
        loads[p] += sizes[i]
    return [sorted(b) for b in bins]


def driven_corners(sc: Scene, x: np.ndarray, time: float, speed: float = 0.2) -> np.ndarray:
    """Config-4 kinematics: the pinned corners move toward the sheet's centre
    at `speed` m/s; returns x with the pinned rows set for `time`. The caller
    edits the pinned positions between steps (the reference has no driven
    pins; this invalidates the adaptive-guess history every step)."""
    pins = np.nonzero(sc.mesh.pinned)[0]
    start = sc.mesh.pin_positions[pins]
    centre = sc.x0.mean(axis=0)
    d = centre - start
    d[:, 1] = 0.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = x.copy()
    out[pins] = start + d * (speed * time)
    return out


def small_sheet(n_side: int = 16, seed: int = 0, obstacle: bool = True, iterations: int = 20,
                radius: float = 0.002, height: float = 0.3, side: float = 0.5, pins=None) -> Scene:
    """Reduced config-0 style scene for fast parity tests."""
    if pins is None:
        pins = (0, n_side - 1)
    mesh, x = sheet(n_side, side, height, Material.stvk_mapped(), jitter=1e-4, seed=seed, pins=pins)
    obs = icosphere(2, 0.1) if obstacle else None
    return Scene("sheet%d" % n_side, mesh, obs, x, np.zeros_like(x),
                 StepSettings(dt=1 / 60, iterations=iterations, damping=1.5, radius=radius, stiffness=1e4), 10)


# ---------------------------------------------- reference test fixtures
def resting_patch(offset=(0.0, 0.0, 0.0)) -> Scene:
    """tests/common/mod.rs:8-36: a 3x3-cell 0.12 m patch of the default fabric
    rotated 90 deg about x, 50 micrometres outside the 3 mm shell of a
    one-triangle floor."""
    off = np.asarray(offset, dtype=np.float64)
    mesh = pattern_build(0.12, 0.12, 3, 3, Material())
    R = euler_xyz((90.0, 0.0, 0.0))
    local = np.stack([mesh.uv[:, 0], -mesh.uv[:, 1], np.zeros(mesh.n)], axis=1)
    x = local @ R.T + (off + np.array([-0.06, 0.00305, 0.06]))
    floor = Obstacle(vertices=np.array([[-1.0, 0.0, -1.0], [1.0, 0.0, -1.0], [0.0, 0.0, 1.0]]) + off,
                     triangles=np.array([[0, 1, 2]], dtype=np.uint32))
    return Scene("resting_patch", mesh, floor, np.ascontiguousarray(x), np.zeros((mesh.n, 3)),
                 StepSettings(dt=1 / 60), 60)


def demo_left_panel(nx_cells: int = 2, ny_cells: int = 2) -> Scene:
    """tests/vbd.rs:35-43: the left panel of the two-panel demo template
    (0.4 x 0.6 m, default fabric, placed at (-0.4, 1, 0)) with 2x2 cells and no
    pins or seams."""
    mesh = pattern_build(0.4, 0.6, nx_cells, ny_cells, Material())
    x = np.stack([mesh.uv[:, 0], -mesh.uv[:, 1], np.zeros(mesh.n)], axis=1) + np.array([-0.4, 1.0, 0.0])
    return Scene("demo_left", mesh, None, np.ascontiguousarray(x), np.zeros((mesh.n, 3)), StepSettings(), 1)
