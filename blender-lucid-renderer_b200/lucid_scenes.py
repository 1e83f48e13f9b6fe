"""Seeded synthetic scenes in the Lucid scene-JSON schema.

The schema is the one `PyRenderer::loadSceneFromJsonString` reads
(LucidRenderer/cpp_renderer/include/pybind_renderer.hpp:1258-1542) and that
the Blender exporter writes (LucidRenderer/scene_export.py): ``meshes`` with
``vertices``, ``triangles``, optional ``triangle_normals`` + ``smooth``,
``material`` {base_color, metallic, roughness, emission, transmission, ior,
node_tree, use_nodes, volume}, ``native_lights`` (POINT/SUN/SPOT/AREA) and
``environment``.  Volumes reference a raw float32 sidecar grid file.

Every generator returns ``(scene_dict, camera)`` where camera is the
``set_camera`` argument tuple (pos, dir, up, fov_deg) flattened to 10 floats.
No public dataset is used: every scene is procedural and seeded.
"""
from __future__ import annotations

import math
import os

import numpy as np

F32 = np.float32


def _fmt_array(a: np.ndarray) -> str:
    """JSON text of a float array with 9 significant digits (float32 round-trip)."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        return "[" + ",".join("%.9g" % v for v in a) + "]"
    return "[" + ",".join(_fmt_array(r) for r in a) + "]"


def _fmt_int_array(a: np.ndarray) -> str:
    a = np.asarray(a, dtype=np.int64)
    if a.ndim == 1:
        return "[" + ",".join(str(int(v)) for v in a) + "]"
    return "[" + ",".join(_fmt_int_array(r) for r in a) + "]"


def _fmt_value(v) -> str:
    import json
    if isinstance(v, np.ndarray):
        return _fmt_int_array(v) if v.dtype.kind in "iu" else _fmt_array(v)
    if isinstance(v, dict):
        return "{" + ",".join(json.dumps(k) + ":" + _fmt_value(x) for k, x in v.items()) + "}"
    if isinstance(v, (list, tuple)):
        return "[" + ",".join(_fmt_value(x) for x in v) + "]"
    if isinstance(v, (float, np.floating)):
        return "%.9g" % float(v)
    return json.dumps(v)


def to_json(scene: dict) -> str:
    """Serialise a scene dict (numpy arrays allowed) to the reference JSON schema."""
    return _fmt_value(scene)


def material(base=(0.8, 0.8, 0.8), metallic=0.0, roughness=0.5, emission=(0.0, 0.0, 0.0),
             transmission=0.0, ior=1.45) -> dict:
    return {"base_color": [float(x) for x in base], "metallic": float(metallic),
            "roughness": float(roughness), "emission": [float(x) for x in emission],
            "transmission": float(transmission), "ior": float(ior)}


def quad(p0, p1, p2, p3):
    """Two triangles (p0,p1,p2), (p0,p2,p3)."""
    v = np.array([p0, p1, p2, p3], dtype=np.float64)
    t = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int64)
    return v, t


def box(size, center, rot_y_deg=0.0):
    """Axis-aligned box (12 triangles) rotated about y and placed with its base at center.y."""
    sx, sy, sz = size
    c = np.array([[x, y, z] for x in (-sx / 2, sx / 2) for y in (0.0, sy) for z in (-sz / 2, sz / 2)])
    a = math.radians(rot_y_deg)
    R = np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])
    v = c @ R.T + np.asarray(center, dtype=np.float64)
    # corner index = 4*ix + 2*iy + iz
    faces = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    t = []
    for f in faces:
        t += [[f[0], f[1], f[2]], [f[0], f[2], f[3]]]
    return v, np.array(t, dtype=np.int64)


def mesh(v, t, mat, normals=None, smooth=False) -> dict:
    m = {"vertices": np.asarray(v, dtype=np.float64), "triangles": np.asarray(t, dtype=np.int64),
         "material": mat}
    if normals is not None:
        m["triangle_normals"] = np.asarray(normals, dtype=np.float64)
        m["smooth"] = bool(smooth)
    return m


# ---------------------------------------------------------------------------
# Config 1: Cornell box, 36 triangles
# ---------------------------------------------------------------------------
def cornell_box():
    """Unit-cube room (10 triangles, front open), two boxes of 12 triangles
    (0.3 and 0.6 high, rotated -17 and +17 degrees about y) and a 0.25 x 0.2
    ceiling quad light (2 triangles, emission 17 warm white).  Walls are
    Principled diffuse (roughness 1, metallic 0).  Camera: 40 degree vertical
    fov looking down -z into the room."""
    white, red, green = (0.73, 0.73, 0.73), (0.63, 0.065, 0.05), (0.14, 0.45, 0.09)
    meshes = []
    wall = lambda col: material(col, 0.0, 1.0)
    meshes.append(mesh(*quad((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0)), wall(white)))      # floor
    meshes.append(mesh(*quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)), wall(white)))      # ceiling
    meshes.append(mesh(*quad((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)), wall(white)))      # back
    meshes.append(mesh(*quad((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1)), wall(red)))        # left
    meshes.append(mesh(*quad((1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0)), wall(green)))      # right
    meshes.append(mesh(*box((0.3, 0.3, 0.3), (0.66, 0.0, 0.62), -17.0), wall(white)))        # short box
    meshes.append(mesh(*box((0.3, 0.6, 0.3), (0.34, 0.0, 0.36), 17.0), wall(white)))         # tall box
    lv, lt = quad((0.375, 0.999, 0.4), (0.625, 0.999, 0.4), (0.625, 0.999, 0.6), (0.375, 0.999, 0.6))
    meshes.append(mesh(lv, lt, material((0.78, 0.78, 0.78), 0.0, 1.0, emission=(17.0, 12.0, 4.0))))
    scene = {"meshes": meshes, "native_lights": [],
             "environment": {"color": [0.0, 0.0, 0.0], "strength": 1.0}}
    camera = (0.5, 0.5, 1.95, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 40.0)
    return scene, camera


# ---------------------------------------------------------------------------
# Icospheres and value-noise fBm
# ---------------------------------------------------------------------------
def icosphere(levels: int):
    """Unit icosphere with 20 * 4**levels triangles (Blender's 'subdivisions'
    = levels + 1)."""
    p = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
         (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, dtype=np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array(f, dtype=np.int64)
    for _ in range(levels):
        e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = verts[uniq[:, 0]] + verts[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(verts)
        verts = np.concatenate([verts, mid])
        n = len(faces)
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        ab, bc, ca = inv[:n] + base, inv[n:2 * n] + base, inv[2 * n:] + base
        faces = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1),
                                np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)])
    return verts, faces


def _value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise in [-1, 1] on the integer lattice (hash-based)."""
    i = np.floor(p).astype(np.int64)
    f = p - i
    f = f * f * (3 - 2 * f)

    def h(ix, iy, iz):
        x = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761)
        x = (x ^ (x >> 13)) * 1274126177
        x = x ^ (x >> 16)
        return (x & 0xFFFF).astype(np.float64) / 32767.5 - 1.0

    out = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = ((f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) *
                     (f[:, 2] if dz else 1 - f[:, 2]))
                out = out + w * h(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
    return out


def fbm(p: np.ndarray, seed: int, octaves: int = 4) -> np.ndarray:
    out, amp, freq, norm = 0.0, 1.0, 1.0, 0.0
    for o in range(octaves):
        out = out + amp * _value_noise(p * freq, seed + o)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return out / norm


def vertex_normals(v: np.ndarray, t: np.ndarray) -> np.ndarray:
    fn = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    vn = np.zeros_like(v)
    for k in range(3):
        np.add.at(vn, t[:, k], fn)
    vn /= np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-12)
    return vn


def displaced_sphere(levels, radius, center, amp_frac, seed):
    v, t = icosphere(levels)
    d = fbm(v * 2.5, seed)
    v = v * (radius * (1.0 + amp_frac * d))[:, None] + np.asarray(center)
    vn = vertex_normals(v, t)
    return v, t, vn[t]


def write_constant_grid(path: str, dims=(8, 8, 8), value: float = 1.0) -> None:
    np.full(int(np.prod(dims)), value, dtype=np.float32).tofile(path)


def volume_box_mesh(bmin, bmax, density, color, anisotropy, sidecar, dims=(8, 8, 8)) -> dict:
    """A volume-boundary-only cube (Material Output Surface unlinked, Volume
    linked) carrying a constant-density grid that fills its bbox."""
    size = np.asarray(bmax, dtype=np.float64) - np.asarray(bmin, dtype=np.float64)
    v, t = box(tuple(size), (bmin[0] + size[0] / 2, bmin[1], bmin[2] + size[2] / 2), 0.0)
    node_tree = {"nodes": [
        {"name": "Material Output", "type": "ShaderNodeOutputMaterial",
         "inputs": [{"name": "Surface", "type": "SHADER"}, {"name": "Volume", "type": "SHADER"}]},
        {"name": "Principled Volume", "type": "ShaderNodeVolumePrincipled", "inputs": []}],
        "links": [{"from_node": "Principled Volume", "from_socket": "Volume",
                   "to_node": "Material Output", "to_socket": "Volume"}]}
    mat = material((0.8, 0.8, 0.8), 0.0, 0.5)
    mat["node_tree"] = node_tree
    mat["use_nodes"] = False
    mat["volume"] = {"color": [float(c) for c in color], "absorption_color": [0.0, 0.0, 0.0],
                     "density": float(density), "anisotropy": float(anisotropy),
                     "smoke_grid": {"dims": list(dims), "world_min": [float(x) for x in bmin],
                                    "world_max": [float(x) for x in bmax], "sidecar_path": sidecar}}
    return mesh(v, t, mat)


# ---------------------------------------------------------------------------
# Config 2: ~1M-triangle procedural scene
# ---------------------------------------------------------------------------
def procedural_scene(seed: int = 2, n_spheres: int = 200, levels: int = 4, emissive_levels: int = 3,
                     workdir: str | None = None, extent: float = 30.0):
    """200 fBm-displaced icospheres (5120 triangles each, Blender subdivision
    5; displacement 5% of radius; radii U[0.2, 1.5] m) on a 2-triangle 100 m
    ground; per-object Principled params (base U[0.05,0.95]^3, roughness
    U[0.02,1], metallic Bern(0.3), IOR 1.45, transmission Bern(0.1));
    16 point, 4 spot (30 degree cone, 5 degree blend), 1 sun, 8 rectangle area
    lights and 2 emissive icospheres (1280 triangles each); one homogeneous
    volume box (sigma_t 0.5/m, albedo 0.8, g 0.3) encoded as a constant 8^3
    grid inside a volume-boundary-only cube.  The sun is a delta light: the
    reference ignores Blender's sun angle."""
    rng = np.random.default_rng(seed)
    meshes = [mesh(*quad((-50, 0, -50), (-50, 0, 50), (50, 0, 50), (50, 0, -50)),
                   material((0.5, 0.5, 0.5), 0.0, 0.8))]
    centers = []
    for i in range(n_spheres):
        r = rng.uniform(0.2, 1.5)
        for _ in range(100):
            c = np.array([rng.uniform(-extent, extent), r, rng.uniform(-extent, extent)])
            if all(np.linalg.norm(c - c2) > r + r2 for c2, r2 in centers):
                break
        centers.append((c, r))
        v, t, tn = displaced_sphere(levels, r, c, 0.05, seed * 1000 + i)
        base = rng.uniform(0.05, 0.95, 3)
        rough = rng.uniform(0.02, 1.0)
        metal = float(rng.random() < 0.3)
        trans = float(rng.random() < 0.1)
        meshes.append(mesh(v, t, material(base, metal, rough, transmission=trans, ior=1.45), tn, True))
    for k in range(2):
        c = np.array([rng.uniform(-extent / 2, extent / 2), 4.0 + 2.0 * k, rng.uniform(-extent / 2, extent / 2)])
        v, t = icosphere(emissive_levels)
        v = v * 0.6 + c
        meshes.append(mesh(v, t, material((0.9, 0.9, 0.9), 0.0, 1.0, emission=(12.0, 10.0, 8.0)),
                           vertex_normals(v, t)[t], True))
    workdir = workdir or os.getcwd()
    sidecar = os.path.join(workdir, "procedural_volume_grid_%d.f32" % seed)
    write_constant_grid(sidecar, (8, 8, 8), 1.0)
    meshes.append(volume_box_mesh((-4.0, 0.0, -4.0), (4.0, 3.0, 4.0), 0.5, (0.8, 0.8, 0.8), 0.3, sidecar))
    lights = []
    for i in range(16):
        lights.append({"type": "POINT", "name": "Point.%03d" % i,
                       "position": [rng.uniform(-extent, extent), rng.uniform(1.5, 6.0), rng.uniform(-extent, extent)],
                       "color": list(rng.uniform(0.6, 1.0, 3)), "energy": float(rng.uniform(200, 800)),
                       "radius": 0.0})
    for i in range(4):
        pos = np.array([rng.uniform(-extent / 2, extent / 2), 8.0, rng.uniform(-extent / 2, extent / 2)])
        lights.append({"type": "SPOT", "name": "Spot.%03d" % i, "position": list(pos),
                       "direction": [0.0, -1.0, 0.0], "color": [1.0, 0.95, 0.9],
                       "energy": 2000.0, "spot_size": math.radians(30.0), "spot_blend": 5.0 / 30.0, "radius": 0.0})
    sd = np.array([-0.4, -1.0, -0.3])
    lights.append({"type": "SUN", "name": "Sun", "direction": list(sd / np.linalg.norm(sd)),
                   "color": [1.0, 0.95, 0.85], "energy": 3.0, "angle": math.radians(0.5)})
    for i in range(8):
        pos = np.array([rng.uniform(-extent, extent), rng.uniform(3.0, 7.0), rng.uniform(-extent, extent)])
        lights.append({"type": "AREA", "name": "Area.%03d" % i, "position": list(pos),
                       "direction": [0.0, -1.0, 0.0], "right": [1.0, 0.0, 0.0], "up": [0.0, 0.0, 1.0],
                       "shape": "RECTANGLE", "size": float(rng.uniform(0.5, 2.0)), "size_y": float(rng.uniform(0.5, 2.0)),
                       "color": [1.0, 1.0, 1.0], "energy": float(rng.uniform(300, 1500))})
    scene = {"meshes": meshes, "native_lights": lights,
             "environment": {"color": [0.25, 0.32, 0.45], "strength": 1.0}}
    camera = (0.0, 9.0, 42.0, 0.0, -0.22, -1.0, 0.0, 1.0, 0.0, 45.0)
    return scene, camera


# ---------------------------------------------------------------------------
# Small scenes for targeted parity cases
# ---------------------------------------------------------------------------
def all_lights_scene(workdir: str | None = None, with_volume: bool = True):
    """A floor, a glass sphere, a near-mirror metal sphere, a rough metal box
    and every native light type (soft and hard point, spot, sun, square /
    rectangle / disk / ellipse area lights) plus an emissive triangle and,
    optionally, a volume box — every light, BSDF and volume branch of the
    reference integrators is reachable."""
    meshes = [mesh(*quad((-5, 0, -5), (-5, 0, 5), (5, 0, 5), (5, 0, -5)), material((0.6, 0.6, 0.6), 0.0, 0.7))]
    v, t = icosphere(2)
    meshes.append(mesh(v * 0.5 + np.array([-1.0, 0.5, 0.0]), t, material((1, 1, 1), 0.0, 0.05, transmission=1.0, ior=1.5),
                       vertex_normals(v, t)[t], True))
    meshes.append(mesh(v * 0.45 + np.array([0.3, 0.45, -0.5]), t, material((0.95, 0.8, 0.5), 1.0, 0.02)))
    meshes.append(mesh(*box((0.6, 0.6, 0.6), (1.3, 0.0, 0.6), 30.0), material((0.3, 0.5, 0.8), 0.7, 0.35)))
    meshes.append(mesh(np.array([[-2.0, 0.01, 1.5], [-1.2, 0.01, 1.5], [-1.6, 0.8, 1.6]]), np.array([[0, 1, 2]]),
                       material((0.9, 0.9, 0.9), 0.0, 1.0, emission=(6.0, 3.0, 1.0))))
    if with_volume:
        workdir = workdir or os.getcwd()
        sidecar = os.path.join(workdir, "all_lights_grid.f32")
        write_constant_grid(sidecar, (4, 4, 4), 1.0)
        meshes.append(volume_box_mesh((0.2, 0.0, 0.8), (1.2, 1.0, 1.8), 1.5, (0.9, 0.7, 0.5), 0.3, sidecar, (4, 4, 4)))
    lights = [
        {"type": "POINT", "position": [0.0, 2.5, 1.0], "color": [1.0, 0.9, 0.8], "energy": 120.0, "radius": 0.0},
        {"type": "POINT", "position": [-1.5, 1.8, -1.0], "color": [0.8, 0.9, 1.0], "energy": 80.0, "radius": 0.2},
        {"type": "SPOT", "position": [1.5, 3.0, -0.5], "direction": [-0.3, -1.0, 0.1], "color": [1.0, 1.0, 0.9],
         "energy": 300.0, "spot_size": math.radians(40.0), "spot_blend": 0.2},
        {"type": "SUN", "direction": [0.3, -1.0, -0.4], "color": [1.0, 0.95, 0.9], "energy": 1.5},
        {"type": "AREA", "position": [0.0, 3.0, 0.0], "direction": [0.0, -1.0, 0.0], "right": [1, 0, 0], "up": [0, 0, 1],
         "shape": "SQUARE", "size": 0.8, "color": [1, 1, 1], "energy": 60.0},
        {"type": "AREA", "position": [2.5, 1.5, 1.5], "direction": [-1.0, 0.0, 0.0], "right": [0, 0, 1], "up": [0, 1, 0],
         "shape": "RECTANGLE", "size": 1.0, "size_y": 0.5, "color": [1, 0.7, 0.7], "energy": 40.0},
        {"type": "AREA", "position": [-2.5, 1.5, 0.5], "direction": [1.0, 0.0, 0.0], "right": [0, 0, 1], "up": [0, 1, 0],
         "shape": "DISK", "size": 0.7, "color": [0.7, 1, 0.7], "energy": 40.0},
        {"type": "AREA", "position": [0.0, 1.2, -2.5], "direction": [0.0, 0.0, 1.0], "right": [1, 0, 0], "up": [0, 1, 0],
         "shape": "ELLIPSE", "size": 1.2, "size_y": 0.6, "color": [0.7, 0.7, 1], "energy": 40.0},
    ]
    scene = {"meshes": meshes, "native_lights": lights,
             "environment": {"color": [0.1, 0.12, 0.15], "strength": 1.0}}
    camera = (0.0, 1.6, 5.0, 0.0, -0.25, -1.0, 0.0, 1.0, 0.0, 45.0)
    return scene, camera


def mirror_point_light_scene():
    """Mirror floor + diffuse back wall + a point light (the reference's
    createMirrorPointLightScene regression shape, test_utils.hpp:277-330)."""
    meshes = [mesh(*quad((-2, 0, -2), (-2, 0, 2), (2, 0, 2), (2, 0, -2)), material((0.9, 0.9, 0.9), 1.0, 0.0)),
              mesh(*quad((-2, 0, -2), (2, 0, -2), (2, 3, -2), (-2, 3, -2)), material((0.7, 0.7, 0.7), 0.0, 1.0))]
    lights = [{"type": "POINT", "position": [0.0, 1.5, 0.0], "color": [1, 1, 1], "energy": 100.0, "radius": 0.0}]
    scene = {"meshes": meshes, "native_lights": lights, "environment": {"color": [0, 0, 0], "strength": 1.0}}
    camera = (0.0, 1.0, 4.0, 0.0, -0.2, -1.0, 0.0, 1.0, 0.0, 50.0)
    return scene, camera


def material_preview_scene(seed: int = 0):
    """A material-preview shot: a subdivision-4 icosphere (5,120 triangles,
    smooth normals) with seeded random Principled parameters on a plane,
    lit by a square area light and a dim environment."""
    rng = np.random.default_rng(seed)
    v, t = icosphere(4)
    mat = material(tuple(rng.uniform(0.05, 0.95, 3)), float(rng.random() < 0.3), float(rng.uniform(0.02, 1.0)),
                   transmission=float(rng.random() < 0.1))
    meshes = [mesh(*quad((-3, 0, -3), (-3, 0, 3), (3, 0, 3), (3, 0, -3)), material((0.5, 0.5, 0.5), 0.0, 0.8)),
              mesh(v * 0.8 + np.array([0.0, 0.8, 0.0]), t, mat, vertex_normals(v, t)[t], True)]
    lights = [{"type": "AREA", "position": [1.5, 3.0, 2.0], "direction": [-0.4, -1.0, -0.5], "right": [1, 0, 0],
               "up": [0, 0, 1], "shape": "SQUARE", "size": 1.5, "color": [1, 1, 1], "energy": 200.0}]
    scene = {"meshes": meshes, "native_lights": lights, "environment": {"color": [0.2, 0.22, 0.25], "strength": 1.0}}
    camera = (0.0, 1.2, 3.2, 0.0, -0.15, -1.0, 0.0, 1.0, 0.0, 40.0)
    return scene, camera


def _grid_quad(origin, du, dv, nu, nv, skip=None):
    """A planar quad origin + [0,1]^2 (du, dv) split into nu x nv cells (two
    triangles each); `skip(i, j)` leaves cells out (openings)."""
    o, du, dv = (np.asarray(a, np.float64) for a in (origin, du, dv))
    verts, tris = [], []
    for j in range(nv):
        for i in range(nu):
            if skip is not None and skip(i, j):
                continue
            p0 = o + du * (i / nu) + dv * (j / nv)
            p1 = o + du * ((i + 1) / nu) + dv * (j / nv)
            p2 = o + du * ((i + 1) / nu) + dv * ((j + 1) / nv)
            p3 = o + du * (i / nu) + dv * ((j + 1) / nv)
            b = len(verts)
            verts += [p0, p1, p2, p3]
            tris += [[b, b + 1, b + 2], [b, b + 2, b + 3]]
    return np.array(verts), np.array(tris, dtype=np.int64)


def _grid_quad_fast(origin, du, dv, nu, nv):
    """_grid_quad without openings, vectorised: (nu + 1) x (nv + 1) shared
    vertices, two triangles per cell."""
    o, du, dv = (np.asarray(a, np.float64) for a in (origin, du, dv))
    i, j = np.meshgrid(np.arange(nu + 1) / nu, np.arange(nv + 1) / nv)
    verts = o + i.reshape(-1, 1) * du + j.reshape(-1, 1) * dv
    ci, cj = np.meshgrid(np.arange(nu), np.arange(nv))
    a = (cj * (nu + 1) + ci).reshape(-1)
    b, c, d = a + 1, a + nu + 2, a + nu + 1
    tris = np.stack([np.stack([a, b, c], 1), np.stack([a, c, d], 1)], 1).reshape(-1, 3)
    return verts, tris.astype(np.int64)


def cornell_variant(seed: int, triangles: int):
    """A seeded variant of the Cornell box with about `triangles` triangles:
    the five walls split into k x k grids, wall colours and box rotations
    varied, the same two boxes, ceiling light and camera."""
    rng = np.random.default_rng(seed)
    k = max(1, int(round(np.sqrt(max(triangles - 26, 10) / 10.0))))
    jitter = lambda c: tuple(float(x) for x in np.clip(np.asarray(c) * rng.uniform(0.8, 1.2, 3), 0.0, 0.95))
    white, red, green = jitter((0.73, 0.73, 0.73)), jitter((0.63, 0.065, 0.05)), jitter((0.14, 0.45, 0.09))
    wall = lambda col: material(col, 0.0, 1.0)
    meshes = [mesh(*_grid_quad_fast((0, 0, 0), (0, 0, 1), (1, 0, 0), k, k), wall(white)),   # floor
              mesh(*_grid_quad_fast((0, 1, 0), (1, 0, 0), (0, 0, 1), k, k), wall(white)),   # ceiling
              mesh(*_grid_quad_fast((0, 0, 0), (1, 0, 0), (0, 1, 0), k, k), wall(white)),   # back
              mesh(*_grid_quad_fast((0, 0, 0), (0, 1, 0), (0, 0, 1), k, k), wall(red)),     # left
              mesh(*_grid_quad_fast((1, 0, 0), (0, 0, 1), (0, 1, 0), k, k), wall(green)),   # right
              mesh(*box((0.3, 0.3, 0.3), (0.66, 0.0, 0.62), float(rng.uniform(-30, 0))), wall(white)),
              mesh(*box((0.3, 0.6, 0.3), (0.34, 0.0, 0.36), float(rng.uniform(0, 30))), wall(white))]
    lv, lt = quad((0.375, 0.999, 0.4), (0.625, 0.999, 0.4), (0.625, 0.999, 0.6), (0.375, 0.999, 0.6))
    meshes.append(mesh(lv, lt, material((0.78, 0.78, 0.78), 0.0, 1.0, emission=(17.0, 12.0, 4.0))))
    scene = {"meshes": meshes, "native_lights": [], "environment": {"color": [0.0, 0.0, 0.0], "strength": 1.0}}
    camera = (0.5, 0.5, 1.95, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 40.0)
    return scene, camera


def hard_indirect_scene():
    """A 12 x 12 x 4 m room (diffuse walls, albedo 0.6; glossy floor,
    roughness 0.2) lit only through a 0.5 m wide, 2.25 m high door gap from
    an adjoining 4 x 12 m room holding a 1 m^2 area light and a 2 x 2 m roof
    opening for the sun.  Walls are tessellated into 0.25 m cells (about
    20k triangles); the environment is black.  Camera: 1280x720 framing,
    60 degree vertical field of view, inside the main room."""
    wall = material((0.6, 0.6, 0.6), 0.0, 1.0)
    floor_m = material((0.6, 0.6, 0.6), 0.0, 0.2)
    c = 4   # cells per metre
    meshes = []
    add = lambda vt, m: meshes.append(mesh(vt[0], vt[1], m))
    # main room: x in [0, 12], z in [0, 12], y in [0, 4]
    add(_grid_quad((0, 0, 0), (0, 0, 12), (12, 0, 0), 12 * c, 12 * c), floor_m)            # floor (normal +y)
    add(_grid_quad((0, 4, 0), (12, 0, 0), (0, 0, 12), 12 * c, 12 * c), wall)               # ceiling
    add(_grid_quad((0, 0, 0), (12, 0, 0), (0, 4, 0), 12 * c, 4 * c), wall)                 # z = 0
    add(_grid_quad((0, 0, 12), (0, 4, 0), (12, 0, 0), 4 * c, 12 * c), wall)                # z = 12
    add(_grid_quad((0, 0, 0), (0, 4, 0), (0, 0, 12), 4 * c, 12 * c), wall)                 # x = 0
    door = lambda i, j: 23 <= j <= 24 and i <= 8     # z in [5.75, 6.25], y in [0, 2.25]
    add(_grid_quad((12, 0, 0), (0, 4, 0), (0, 0, 12), 4 * c, 12 * c, skip=door), wall)    # x = 12, with the gap
    # adjoining room: x in [12, 16]
    add(_grid_quad((12, 0, 0), (0, 0, 12), (4, 0, 0), 12 * c, 4 * c), wall)
    hole = lambda i, j: 4 <= i < 12 and 4 <= j < 12    # x in [13, 15], z in [1, 3]
    add(_grid_quad((12, 4, 0), (4, 0, 0), (0, 0, 12), 4 * c, 12 * c, skip=hole), wall)
    add(_grid_quad((12, 0, 0), (4, 0, 0), (0, 4, 0), 4 * c, 4 * c), wall)
    add(_grid_quad((12, 0, 12), (0, 4, 0), (4, 0, 0), 4 * c, 4 * c), wall)
    add(_grid_quad((16, 0, 0), (0, 0, 12), (0, 4, 0), 12 * c, 4 * c), wall)
    lights = [
        {"type": "SUN", "direction": [-0.25, -1.0, 0.35], "color": [1.0, 0.95, 0.85], "energy": 6.0},
        {"type": "AREA", "position": [14.0, 3.8, 9.0], "direction": [0.0, -1.0, 0.0], "right": [1, 0, 0],
         "up": [0, 0, 1], "shape": "SQUARE", "size": 1.0, "color": [1.0, 1.0, 1.0], "energy": 300.0},
    ]
    scene = {"meshes": meshes, "native_lights": lights, "environment": {"color": [0.0, 0.0, 0.0], "strength": 1.0}}
    camera = (2.0, 1.7, 1.5, 0.9, -0.1, 0.42, 0.0, 1.0, 0.0, 60.0)
    return scene, camera


def scene_triangle_count(scene: dict) -> int:
    return int(sum(len(m["triangles"]) for m in scene["meshes"]))


# ---------------------------------------------------------------------------
# Array form of a scene (lucid_cuda_load_scene_arrays)
# ---------------------------------------------------------------------------
_JSON_ROUNDING = [True]


def _json_f32(a) -> np.ndarray:
    """float32 values exactly as the JSON loader reads this module's JSON
    text: 9 significant digits, parsed as a double, then rounded to float
    (with json_rounding off in scene_arrays: rounded to float directly)."""
    a = np.asarray(a, dtype=np.float64)
    if not _JSON_ROUNDING[0]:
        return a.astype(np.float32)
    return np.char.mod("%.9g", a).astype(np.float64).astype(np.float32)


def _surface_linked(nt) -> bool:
    """The loader's test for a linked Material Output Surface socket (a
    node tree with no nodes, or no output node, counts as linked)."""
    if not isinstance(nt, dict) or "nodes" not in nt or not nt["nodes"]:
        return True
    links = {(l["to_node"], l["to_socket"]) for l in nt.get("links", [])}
    for n in nt["nodes"]:
        if n.get("type", "") != "ShaderNodeOutputMaterial":
            continue
        for i in n.get("inputs", []):
            if i.get("name", "") == "Surface":
                return (n.get("name", ""), "Surface") in links
        return False
    return True


def scene_arrays(scene: dict, json_rounding: bool = True) -> dict:
    """The scene as plain arrays with every default filled in, read as the
    JSON loader reads to_json(scene), so that both uploads give the same
    scene bit for bit.  json_rounding=False rounds values to float32
    directly (fast; a last-bit difference from the JSON form is possible)."""
    _JSON_ROUNDING[0] = json_rounding
    try:
        return _scene_arrays(scene)
    finally:
        _JSON_ROUNDING[0] = True


def _scene_arrays(scene: dict) -> dict:
    meshes = []
    for m in scene.get("meshes", []):
        mat = m.get("material", {})
        vol = mat.get("volume") or {}
        sg = vol.get("smoke_grid") if isinstance(vol.get("smoke_grid"), dict) else None
        grid = None
        dims, wmin, wmax = (0, 0, 0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)
        if sg and all(k in sg for k in ("dims", "world_min", "world_max", "sidecar_path")):
            dims, wmin, wmax = tuple(int(x) for x in sg["dims"]), sg["world_min"], sg["world_max"]
            if os.path.exists(sg["sidecar_path"]):
                grid = np.fromfile(sg["sidecar_path"], dtype=np.float32)[: int(np.prod(dims))].copy()
        nt = mat.get("node_tree")
        tn = m.get("triangle_normals")
        meshes.append({
            "vertices": _json_f32(np.asarray(m.get("vertices", np.zeros((0, 3)))).reshape(-1, 3)).ravel(),
            "triangles": np.asarray(m.get("triangles", np.zeros((0, 3))), dtype=np.int32).reshape(-1).copy(),
            "triangle_normals": None if tn is None else _json_f32(np.asarray(tn).reshape(-1, 9)).ravel(),
            "smooth": bool(m.get("smooth", False)),
            "base_color": _json_f32(mat.get("base_color", [0.8, 0.8, 0.8])),
            "metallic": _json_f32(mat.get("metallic", 0.0)), "roughness": _json_f32(mat.get("roughness", 0.5)),
            "emission": _json_f32(mat.get("emission", [0.0, 0.0, 0.0])),
            "transmission": _json_f32(mat.get("transmission", 0.0)), "ior": _json_f32(mat.get("ior", 1.45)),
            "surface": True if nt is None else _surface_linked(nt),
            "volume_density": _json_f32(vol.get("density", 0.0)), "volume_anisotropy": _json_f32(vol.get("anisotropy", 0.0)),
            "volume_color": _json_f32(vol.get("color", [1.0, 1.0, 1.0])),
            "volume_absorption": _json_f32(vol.get("absorption_color", [0.0, 0.0, 0.0])),
            "volume_dims": dims, "volume_world_min": _json_f32(wmin), "volume_world_max": _json_f32(wmax),
            "volume_grid": grid})
    lights = []
    types = {"POINT": 1, "SUN": 2, "SPOT": 3, "AREA": 4}
    shapes = {"SQUARE": 0, "RECTANGLE": 1, "DISK": 2, "ELLIPSE": 3}
    for l in scene.get("native_lights", scene.get("lights", [])):
        size = l.get("size", 1.0)
        lights.append({
            "type": types.get(l.get("type", "POINT"), 0), "position": _json_f32(l.get("position", [0.0, 0.0, 0.0])),
            "direction": _json_f32(l.get("direction", [0.0, 0.0, 1.0])), "color": _json_f32(l.get("color", [1.0, 1.0, 1.0])),
            "energy": _json_f32(l.get("energy", 1.0)), "radius": _json_f32(l.get("radius", 0.0)),
            "spot_size": _json_f32(l.get("spot_size", np.float32(np.pi / 4.0))),
            "spot_blend": _json_f32(l.get("spot_blend", 0.0)), "size": _json_f32(size),
            "size_y": _json_f32(l.get("size_y", size)), "shape": shapes.get(l.get("shape", "SQUARE"), 0),
            "right": _json_f32(l.get("right", [1.0, 0.0, 0.0])), "up": _json_f32(l.get("up", [0.0, 1.0, 0.0]))})
    env = scene.get("environment")
    if isinstance(env, dict):
        col = _json_f32(env.get("color", [0.05, 0.05, 0.05])) if isinstance(env.get("color"), (list, tuple, np.ndarray)) \
            else np.full(3, np.float32(0.05))
        environment = (col * _json_f32(env.get("strength", 1.0))).astype(np.float32)
    else:
        environment = np.full(3, np.float32(0.05))
    return {"meshes": meshes, "lights": lights, "environment": environment}


# ---------------------------------------------------------------------------
# Node-graph materials (use_nodes) with UV checker textures
# ---------------------------------------------------------------------------
def _sock(name, value=None):
    s = {"name": name, "type": "RGBA" if isinstance(value, (list, tuple)) else "VALUE"}
    if value is not None:
        s["default_value"] = list(value) if isinstance(value, (list, tuple)) else float(value)
    return s


def _tree(nodes, links):
    return {"nodes": nodes, "links": [{"from_node": a, "from_socket": b, "to_node": c, "to_socket": d}
                                      for a, b, c, d in links]}


def _out(surface_from, socket="BSDF"):
    return ({"name": "Material Output", "type": "ShaderNodeOutputMaterial",
             "inputs": [_sock("Surface"), _sock("Volume")]}, (surface_from, socket, "Material Output", "Surface"))


def textured_scene():
    """Quads whose materials come from node graphs: a checker floor (Base
    Color <- Checker, UVs 0..4), a Mix of a checker and an RGB node on the back
    wall (a Diffuse BSDF), an emissive checker panel (Emission <- Checker), a
    Principled panel whose scalars come from the graph, and a box with a node
    tree but use_nodes off; lit by a point light and the panel."""
    meshes = []
    uv = np.array([[[0, 0], [4, 0], [4, 4]], [[0, 0], [4, 4], [0, 4]]], dtype=np.float64)
    # floor: Principled, Base Color <- Checker (Color1/Color2 constants, scale 2)
    out, link = _out("Principled BSDF")
    floor_mat = material((0.1, 0.1, 0.1))
    floor_mat["use_nodes"] = True
    floor_mat["node_tree"] = _tree([
        out,
        {"name": "Principled BSDF", "type": "ShaderNodeBsdfPrincipled",
         "inputs": [_sock("Base Color", (0.5, 0.5, 0.5, 1.0)), _sock("Metallic", 0.0), _sock("Roughness", 0.7),
                    _sock("IOR", 1.5), _sock("Transmission Weight", 0.0), _sock("Emission Color", (0, 0, 0, 1)),
                    _sock("Emission Strength", 0.0)]},
        {"name": "Checker Texture", "type": "ShaderNodeTexChecker",
         "inputs": [_sock("Color1", (0.9, 0.8, 0.7, 1.0)), _sock("Color2", (0.1, 0.2, 0.3, 1.0)), _sock("Scale", 2.0)]}],
        [link, ("Checker Texture", "Color", "Principled BSDF", "Base Color")])
    m = mesh(*quad((-2, 0, -2), (2, 0, -2), (2, 0, 2), (-2, 0, 2)), floor_mat)
    m["triangle_uvs"] = uv
    meshes.append(m)
    # back wall: Diffuse BSDF, Color <- Mix(Checker, RGB, fac 0.3)
    out, link = _out("Diffuse BSDF")
    wall_mat = material((0.5, 0.5, 0.5), 0.3, 0.2)
    wall_mat["use_nodes"] = True
    wall_mat["node_tree"] = _tree([
        out,
        {"name": "Diffuse BSDF", "type": "ShaderNodeBsdfDiffuse", "inputs": [_sock("Color", (0.8, 0.8, 0.8, 1.0))]},
        {"name": "Mix", "type": "ShaderNodeMix", "inputs": [_sock("Fac", 0.3), _sock("A"), _sock("B")]},
        {"name": "Checker Texture", "type": "ShaderNodeTexChecker", "inputs": [_sock("Scale", 3.0)]},
        {"name": "RGB", "type": "ShaderNodeRGB", "inputs": [], "outputs": [{"name": "Color", "default_value": [0.2, 0.6, 0.3, 1.0]}]}],
        [link, ("Mix", "Result", "Diffuse BSDF", "Color"), ("Checker Texture", "Color", "Mix", "A"),
         ("RGB", "Color", "Mix", "B")])
    m = mesh(*quad((-2, 0, -2), (-2, 2.5, -2), (2, 2.5, -2), (2, 0, -2)), wall_mat)
    m["triangle_uvs"] = uv * 0.5
    meshes.append(m)
    # emissive panel: Emission shader, Color <- Checker, strength 4
    out, link = _out("Emission", "Emission")
    panel = material((0.0, 0.0, 0.0))
    panel["use_nodes"] = True
    panel["node_tree"] = _tree([
        out,
        {"name": "Emission", "type": "ShaderNodeEmission", "inputs": [_sock("Color"), _sock("Strength", 4.0)]},
        {"name": "Checker Texture", "type": "ShaderNodeTexChecker",
         "inputs": [_sock("Color1", (1.0, 0.9, 0.7, 1.0)), _sock("Color2", (0.0, 0.0, 0.0, 1.0)), _sock("Scale", 1.5)]}],
        [link, ("Checker Texture", "Color", "Emission", "Color")])
    m = mesh(*quad((-1.5, 1.0, -1.99), (-0.5, 1.0, -1.99), (-0.5, 2.0, -1.99), (-1.5, 2.0, -1.99)), panel)
    m["triangle_uvs"] = np.array([[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]], dtype=np.float64)
    meshes.append(m)
    # glossy Principled panel: all scalars from the graph (the JSON fields are ignored)
    out, link = _out("Principled BSDF")
    gl = material((0.9, 0.1, 0.1), 0.0, 0.9)
    gl["use_nodes"] = True
    gl["node_tree"] = _tree([
        out,
        {"name": "Principled BSDF", "type": "ShaderNodeBsdfPrincipled",
         "inputs": [_sock("Base Color", (0.7, 0.75, 0.8, 1.0)), _sock("Metallic", 1.0), _sock("Roughness", 0.25),
                    _sock("IOR", 1.45), _sock("Emission Color", (0.0, 0.0, 0.0, 1.0)), _sock("Emission Strength", 0.0)]}],
        [link])
    meshes.append(mesh(*quad((0.5, 0.2, -1.0), (1.8, 0.2, -1.0), (1.8, 1.5, -1.6), (0.5, 1.5, -1.6)), gl))
    # a node tree present but use_nodes off: the JSON fields apply
    bx = material((0.3, 0.5, 0.8), 0.0, 0.4)
    bx["use_nodes"] = False
    bx["node_tree"] = floor_mat["node_tree"]
    meshes.append(mesh(*box((0.6, 0.6, 0.6), (-0.8, 0.0, 0.3), 20.0), bx))
    lights = [{"type": "POINT", "position": [0.5, 2.2, 1.0], "color": [1, 1, 1], "energy": 150.0, "radius": 0.05}]
    scene = {"meshes": meshes, "native_lights": lights, "environment": {"color": [0.05, 0.05, 0.06], "strength": 1.0}}
    camera = (0.0, 1.2, 4.5, 0.0, -0.15, -1.0, 0.0, 1.0, 0.0, 50.0)
    return scene, camera
