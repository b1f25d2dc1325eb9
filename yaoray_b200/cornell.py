"""Cornell-box scene of the plain-MIS configuration: a 5.56-unit box of five
wall quads, a short box (1.65 tall, rotated -17 degrees about y) and a tall
box (3.3 tall, +17 degrees) — 34 triangles — plus a 1.3 x 1.05 quad area
light (2 more triangles) emitting (17, 12, 4); Lambertian red
(0.63, 0.065, 0.05), green (0.14, 0.45, 0.09) and white 0.73; pinhole camera
with a 40 degree vertical fov; 256 x 256, 64 spp Owen-scrambled Sobol (seed
0), max depth 8 (Russian roulette from depth 3 is built into the path
integrator).

`pbrt_text()` writes it as a PBRT v4 "trianglemesh" file for the reference's
own frontend; `scene()` builds the same RenderSceneIR directly (the tests
check both agree field by field with what the reference compiles).
"""
from __future__ import annotations

import math

import numpy as np

from .accel import SceneGeometry
from .render import EMISSIVE_DTYPE, OWEN_SOBOL, SUBSURFACE, RenderScene, build_bssrdf_table, default_material

SIZE = 5.56
WHITE = (0.73, 0.73, 0.73)
RED = (0.63, 0.065, 0.05)
GREEN = (0.14, 0.45, 0.09)
LIGHT_L = (17.0, 12.0, 4.0)
EYE = (2.78, 2.73, -8.0)
LOOK = (2.78, 2.73, 0.0)
FOV = 40.0


def _box(cx, cz, w, h, d, deg):
    """Axis box rotated about y by `deg` around its centre: 8 corners, 12
    triangles wound outward."""
    a = math.radians(deg)
    ca, sa = math.cos(a), math.sin(a)
    pts = []
    for y in (0.0, h):
        for (x, z) in ((-w / 2, -d / 2), (w / 2, -d / 2), (w / 2, d / 2), (-w / 2, d / 2)):
            pts.append((round(cx + ca * x + sa * z, 4), y, round(cz - sa * x + ca * z, 4)))
    tris = [[0, 2, 1], [0, 3, 2],          # bottom
            [4, 5, 6], [4, 6, 7],          # top
            [0, 1, 5], [0, 5, 4],          # front
            [1, 2, 6], [1, 6, 5],          # right
            [2, 3, 7], [2, 7, 6],          # back
            [3, 0, 4], [3, 4, 7]]          # left
    return pts, tris


def shapes():
    """[(material name, points, triangles, emission or None)] in file order."""
    s = SIZE
    quad = [[0, 1, 2], [0, 2, 3]]
    out = [
        ("white", [(0, 0, 0), (s, 0, 0), (s, 0, s), (0, 0, s)], quad, None),            # floor
        ("white", [(0, s, 0), (0, s, s), (s, s, s), (s, s, 0)], quad, None),            # ceiling
        ("white", [(0, 0, s), (s, 0, s), (s, s, s), (0, s, s)], quad, None),            # back
        ("red", [(s, 0, 0), (s, s, 0), (s, s, s), (s, 0, s)], quad, None),              # left (image left)
        ("green", [(0, 0, 0), (0, 0, s), (0, s, s), (0, s, 0)], quad, None),            # right
    ]
    p, t = _box(1.85, 1.69, 1.65, 1.65, 1.65, -17.0)
    out.append(("white", p, t, None))
    p, t = _box(3.69, 3.51, 1.65, 3.30, 1.65, 17.0)
    out.append(("white", p, t, None))
    y = s - 0.005
    lx0, lx1, lz0, lz1 = 2.13, 3.43, 2.27, 3.32
    out.append(("white", [(lx0, y, lz0), (lx0, y, lz1), (lx1, y, lz1), (lx1, y, lz0)], quad, LIGHT_L))
    return out


def pbrt_text(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8) -> str:
    lines = [
        "# Cornell box: 34 scene triangles + a 2-triangle area light.",
        f"LookAt {EYE[0]} {EYE[1]} {EYE[2]}  {LOOK[0]} {LOOK[1]} {LOOK[2]}  0 1 0",
        f'Camera "perspective" "float fov" [{FOV}]',
        f'Sampler "sobol" "integer pixelsamples" [{spp}]',
        f'Integrator "path" "integer maxdepth" [{max_depth}]',
        f'Film "rgb" "integer xresolution" [{width}] "integer yresolution" [{height}] "string filename" ["cornell.exr"]',
        "WorldBegin",
    ]
    for name, rgb in (("white", WHITE), ("red", RED), ("green", GREEN)):
        lines.append(f'MakeNamedMaterial "{name}" "string type" ["diffuse"] "rgb reflectance" [{rgb[0]} {rgb[1]} {rgb[2]}]')
    for name, pts, tris, emission in shapes():
        lines.append("AttributeBegin")
        if emission is not None:
            lines.append(f'AreaLightSource "diffuse" "rgb L" [{emission[0]} {emission[1]} {emission[2]}]')
        lines.append(f'NamedMaterial "{name}"')
        flat_p = " ".join(f"{c}" for pt in pts for c in pt)
        flat_i = " ".join(str(i) for tri in tris for i in tri)
        lines.append(f'Shape "trianglemesh" "point3 P" [{flat_p}] "integer indices" [{flat_i}]')
        lines.append("AttributeEnd")
    lines.append("WorldEnd")
    return "\n".join(lines) + "\n"


def camera() -> dict:
    """The camera basis the reference derives from LookAt + fov (forward,
    right = forward x up, true up = right x forward)."""
    eye = np.array(EYE, np.float32)
    fwd = np.array(LOOK, np.float32) - eye
    fwd = fwd / np.float32(np.sqrt(np.float32(np.dot(fwd, fwd))))
    right = np.cross(fwd, np.array([0, 1, 0], np.float32)).astype(np.float32)
    right = right / np.float32(np.sqrt(np.float32(np.dot(right, right))))
    up = np.cross(right, fwd).astype(np.float32)
    return {"origin": tuple(map(float, eye)), "forward": tuple(map(float, fwd)), "right": tuple(map(float, right)),
            "up": tuple(map(float, up)), "fov_y_radians": float(np.float32(FOV) * np.float32(math.pi) / np.float32(180))}


def scene(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8) -> RenderScene:
    """The RenderSceneIR the reference compiles from `pbrt_text()`."""
    # Named materials in the order the reference's compiler emits them.
    names = {"green": 0, "red": 1, "white": 2}
    mats = np.stack([default_material(reflectance=GREEN), default_material(reflectance=RED),
                     default_material(reflectance=WHITE)])
    meshes, emissive = [], []
    light_mat = None
    for k, (name, pts, tris, em) in enumerate(shapes()):
        meshes.append((np.array(pts, np.float32), np.array(tris, np.uint32)))
        if em is not None:
            light_mat = k
    geom = SceneGeometry.from_meshes(meshes)
    prims = geom.primitives
    for k, (name, pts, tris, em) in enumerate(shapes()):
        prims[k]["material_index"] = names[name]
    # The emitting shape gets its own material carrying the emission.
    lm = default_material(reflectance=WHITE, emission=LIGHT_L)
    mats = np.concatenate([mats, lm[None]])
    prims[light_mat]["material_index"] = len(mats) - 1
    p = geom.positions
    idx = geom.indices.reshape(-1, 3)
    first = prims[light_mat]["first_index"] // 3
    count = prims[light_mat]["index_count"] // 3
    area = np.float32(0)
    for t in range(first, first + count):
        a, b, c = p[idx[t, 0]], p[idx[t, 1]], p[idx[t, 2]]
        cr = np.cross(b - a, c - a).astype(np.float32)
        area = np.float32(area + np.float32(np.sqrt(np.float32(np.dot(cr, cr)))) * np.float32(0.5))
    em = np.zeros(1, EMISSIVE_DTYPE)
    em[0]["primitive_index"] = light_mat
    em[0]["radiance"] = LIGHT_L
    em[0]["area"] = area
    return RenderScene(geom, mats, camera(), width, height, spp=spp, max_depth=max_depth, seed=0,
                       sampler=OWEN_SOBOL, emissive=em)


# The reference compiler's "Skin1" subsurface preset, per scene unit
# (src/frontend/pbrt/scene_compiler_special_materials.cpp:33-35).
SKIN1_SIGMA_A = (0.032, 0.17, 0.48)
SKIN1_SIGMA_S = (0.74, 0.88, 1.01)


def subsurface_scene(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8,
                     scale: float = 1.0, eta: float = 1.33) -> RenderScene:
    """The Cornell box with the tall box made of a subsurface material (the
    Skin1 coefficients times `scale`, relative index `eta`) and its
    100 x 64 beam-diffusion profile table, as the reference's compiler would
    build it from `Material "subsurface"`."""
    s = scene(width, height, spp, max_depth)
    m = default_material(kind=SUBSURFACE, sigma_a=np.float32(scale) * np.array(SKIN1_SIGMA_A, np.float32),
                         sigma_s=np.float32(scale) * np.array(SKIN1_SIGMA_S, np.float32), bssrdf_eta=eta,
                         bssrdf_index=0)
    s.materials = np.concatenate([s.materials, m[None]])
    tall_box = 6  # shapes(): five walls, short box, tall box, light
    s.geometry.primitives[tall_box]["material_index"] = len(s.materials) - 1
    s.bssrdf_tables = [build_bssrdf_table(eta)]
    return s


def _checker(n: int, tiles: int, a, b) -> np.ndarray:
    y, x = np.mgrid[0:n, 0:n]
    on = ((x * tiles // n) + (y * tiles // n)) % 2 == 0
    tex = np.where(on[..., None], np.array([*a, 1.0], np.float32), np.array([*b, 1.0], np.float32))
    return tex.astype(np.float32)


def _bump_normal_map(n: int, waves: int = 4, slope: float = 0.35) -> np.ndarray:
    """A tangent-space normal map of sine bumps, encoded n * 0.5 + 0.5."""
    v, u = (np.mgrid[0:n, 0:n] + 0.5) / n
    nx = slope * np.sin(2.0 * np.pi * waves * u)
    ny = slope * np.cos(2.0 * np.pi * waves * v)
    nz = np.ones_like(nx)
    ln = np.sqrt(nx * nx + ny * ny + nz * nz)
    enc = np.stack([nx / ln, ny / ln, nz / ln], -1) * 0.5 + 0.5
    return np.concatenate([enc, np.ones((n, n, 1))], -1).astype(np.float32)


def textured_scene(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8,
                   filters=(3, 2, 1, 0), seed: int = 7) -> RenderScene:
    """The Cornell box with textured surfaces: the floor carries a checker
    reflectance texture (filters[0], repeat), the back wall a noise texture
    (filters[1], mirrored repeat), the red wall a coarse texture
    (filters[2], clamp to edge), the short box a checker (filters[3],
    repeat), and the tall box a tangent-space normal map (bilinear) with
    per-vertex tangents. Every wall and box has planar uvs spanning several
    texture repeats."""
    from .texture import Texture

    s = scene(width, height, spp, max_depth)
    g = s.geometry
    rng = np.random.default_rng(seed)
    nv = g.positions.shape[0]
    uvs = np.zeros((nv, 2), np.float32)
    tangents = np.zeros((nv, 4), np.float32)
    tangents[:, 3] = 1.0
    prims = g.primitives
    idx = g.indices
    # Planar uvs per shape: walls and boxes are parameterised by the two
    # axes of largest extent, in units of 1.39 (a quarter of the box).
    for k in range(7):
        first, count = int(prims[k]["first_index"]), int(prims[k]["index_count"])
        verts = np.unique(idx[first:first + count])
        p = g.positions[verts]
        ext = p.max(0) - p.min(0)
        if k >= 5:  # boxes: (x + z, y)
            uvs[verts, 0] = (p[:, 0] + p[:, 2]) / 1.39
            uvs[verts, 1] = p[:, 1] / 1.39
        else:
            a, b = np.argsort(-ext)[:2]
            uvs[verts, 0] = p[:, a] / 1.39
            uvs[verts, 1] = p[:, b] / 1.39
        prims[k]["flags"] = prims[k]["flags"] | 2
    # Tall box: tangents along its rotated x axis (17 degrees about y).
    a = math.radians(17.0)
    first, count = int(prims[6]["first_index"]), int(prims[6]["index_count"])
    verts = np.unique(idx[first:first + count])
    tangents[verts, 0:3] = (math.cos(a), 0.0, -math.sin(a))
    tangents[verts, 3] = np.where(np.arange(verts.size) % 2 == 0, 1.0, -1.0)
    prims[6]["flags"] = prims[6]["flags"] | 4
    noise = (0.35 + 0.6 * rng.random((23, 37, 4))).astype(np.float32)
    noise[..., 3] = 1.0
    coarse = (0.3 + 0.7 * rng.random((5, 3, 4))).astype(np.float32)
    s.textures = [
        Texture(_checker(64, 8, (0.9, 0.9, 0.85), (0.15, 0.2, 0.3)), filters[0], 0, 0),
        Texture(noise, filters[1], 2, 2),
        Texture(coarse, filters[2], 1, 1),
        Texture(_checker(16, 4, (0.95, 0.6, 0.3), (0.3, 0.5, 0.9)), filters[3], 0, 0),
        Texture(_bump_normal_map(32), 1, 0, 0),
    ]
    white, red = s.materials[2].copy(), s.materials[1].copy()
    new = []
    for base, key, t in ((white, "reflectance_texture", 0), (white, "reflectance_texture", 1),
                         (red, "reflectance_texture", 2), (white, "reflectance_texture", 3),
                         (white, "normal_map", 4)):
        m = base.copy()
        m[key] = t
        if key == "normal_map":
            m["normal_scale"] = 0.8
        new.append(m)
    base_index = len(s.materials)
    s.materials = np.concatenate([s.materials, np.stack(new)])
    for shape, k in ((0, 0), (2, 1), (3, 2), (5, 3), (6, 4)):  # floor, back, red wall, short box, tall box
        prims[shape]["material_index"] = base_index + k
    s.uvs = uvs
    s.tangents = tangents
    return s


def _append_quad(s: RenderScene, corners, material: int, uv_scale: float = 3.0) -> None:
    """Appends a two-triangle quad (corners in order) with uvs spanning
    uv_scale repeats as a new mesh primitive of material `material`."""
    from . import _lib

    g = s.geometry
    base = g.positions.shape[0]
    g.positions = np.concatenate([g.positions, np.asarray(corners, np.float32)])
    first = g.indices.size
    g.indices = np.concatenate([g.indices, (np.array([0, 1, 2, 0, 2, 3], np.uint32) + base)])
    prim = np.zeros(1, _lib.PRIM_DTYPE)
    prim[0]["first_index"], prim[0]["index_count"] = first, 6
    prim[0]["material_index"], prim[0]["flags"] = material, 2
    g.primitives = np.concatenate([g.primitives, prim])
    quad_uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32) * np.float32(uv_scale)
    s.uvs = np.concatenate([s.uvs, quad_uv])
    tg = np.zeros((4, 4), np.float32)
    tg[:, 3] = 1.0
    s.tangents = np.concatenate([s.tangents, tg])
    if s.normals is not None:
        s.normals = np.concatenate([s.normals, np.zeros((4, 3), np.float32)])


def cutout_scene(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8) -> RenderScene:
    """textured_scene() plus three panes that exercise alpha and shadows: a
    screen in front of the boxes whose alpha texture (red channel, bilinear)
    cuts round holes, a pane under the light with constant alpha 0.2 (cut out
    everywhere: camera and shadow rays skip it), and a thin-glass pane whose
    reflectance is textured (shadow rays through it take the textured
    transmittance)."""
    from .render import THIN_DIELECTRIC
    from .texture import Texture

    s = textured_scene(width, height, spp, max_depth)
    n = 32
    v, u = (np.mgrid[0:n, 0:n] + 0.5) / n
    holes = ((u - 0.5) ** 2 + (v - 0.5) ** 2) > 0.09
    alpha_tex = np.stack([holes.astype(np.float32), 0.5 * np.ones((n, n)), u, np.ones((n, n))], -1).astype(np.float32)
    s.textures = s.textures + [Texture(alpha_tex, 1, 0, 0),
                               Texture(_checker(8, 2, (0.9, 0.7, 0.5), (0.4, 0.8, 0.95)), 0, 0, 0)]
    t_alpha, t_glass = len(s.textures) - 2, len(s.textures) - 1
    white = s.materials[2].copy()
    screen = white.copy()
    screen["alpha_texture"] = t_alpha
    ghost = white.copy()
    ghost["alpha"] = 0.2
    glass = default_material(kind=THIN_DIELECTRIC, reflectance=(1.0, 1.0, 1.0), ior=1.5)
    glass["reflectance_texture"] = t_glass
    base = len(s.materials)
    s.materials = np.concatenate([s.materials, np.stack([screen, ghost, glass])])
    _append_quad(s, [(0.6, 0.4, 1.0), (4.9, 0.4, 1.0), (4.9, 3.9, 1.0), (0.6, 3.9, 1.0)], base, 2.0)
    _append_quad(s, [(1.6, 5.2, 1.8), (3.9, 5.2, 1.8), (3.9, 5.2, 3.9), (1.6, 5.2, 3.9)], base + 1)
    _append_quad(s, [(0.8, 2.2, 0.6), (2.0, 2.2, 0.6), (2.0, 2.2, 2.9), (0.8, 2.2, 2.9)], base + 2, 1.0)
    return s


def instanced_cutout_scene(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8) -> RenderScene:
    """cutout_scene() traversed as a two-level scene: every primitive is an
    explicit instance, the identity except for the normal-mapped tall box,
    mirrored in x about its centre (a negative-determinant transform: its
    tangent frame flips orientation), and the cut-out screen, moved 0.3
    towards the camera and tilted 10 degrees about x."""
    from . import _lib

    s = cutout_scene(width, height, spp, max_depth)
    g = s.geometry
    n = g.primitives.size
    eye = np.eye(4, dtype=np.float32)
    inst = np.zeros(n, _lib.INSTANCE_DTYPE)
    for k in range(n):
        m = eye.copy()
        if k == 6:  # tall box: x -> 2 cx - x
            first, count = int(g.primitives[k]["first_index"]), int(g.primitives[k]["index_count"])
            cx = float(g.positions[np.unique(g.indices[first:first + count])][:, 0].mean())
            m[0, 0] = -1.0
            m[0, 3] = 2.0 * cx
        elif k == n - 3:  # the screen (first of the three appended panes)
            a = math.radians(10.0)
            m[1, 1], m[1, 2], m[2, 1], m[2, 2] = math.cos(a), -math.sin(a), math.sin(a), math.cos(a)
            m[2, 3] = -0.3
        inst[k]["primitive"] = k
        inst[k]["object_to_world"] = m.T.reshape(16)  # column-major
    g.instances = inst
    return s


def measured_scene(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8) -> RenderScene:
    """The Cornell box with both boxes made of a measured (RGL-layout) BRDF:
    the seeded synthetic tensors of measured.synthetic_brdf()."""
    from .measured import synthetic_brdf
    from .render import MEASURED

    s = scene(width, height, spp, max_depth)
    m = default_material(kind=MEASURED, reflectance=WHITE, measured_index=0, uroughness=0.3, vroughness=0.3)
    s.materials = np.concatenate([s.materials, m[None]])
    for box in (5, 6):
        s.geometry.primitives[box]["material_index"] = len(s.materials) - 1
    s.measured = [synthetic_brdf(3)]
    return s


def analytic_scene(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8,
                   many: bool = False) -> RenderScene:
    """The Cornell box lit by analytic lights as well as its area light:
    a point, a spot and a distant light (selected through the power alias
    table), or with many=True twelve point and spot lights spread under the
    ceiling (more than 8 local lights: selected through the light tree)."""
    from .render import ANALYTIC_DTYPE

    s = scene(width, height, spp, max_depth)
    if many:
        rng = np.random.default_rng(11)
        a = np.zeros(12, ANALYTIC_DTYPE)
        a["kind"] = np.where(np.arange(12) % 3 == 2, 1, 0)
        a["position"] = np.stack([rng.uniform(0.5, 5.0, 12), rng.uniform(3.5, 5.3, 12), rng.uniform(0.5, 5.0, 12)], 1)
        a["direction"] = (0.0, -1.0, 0.0)
        a["intensity"] = rng.uniform(0.5, 2.5, (12, 3))
        a["cone_angle"] = np.float32(math.cos(math.radians(40.0)))
        a["cone_cos_inner"] = np.float32(math.cos(math.radians(25.0)))
    else:
        a = np.zeros(3, ANALYTIC_DTYPE)
        a[0] = (0, (1.2, 4.5, 2.0), (0, 0, 0), (6.0, 5.0, 4.0), 0.0, 0.0)
        a[1] = (1, (4.0, 5.0, 3.5), (-0.3, -1.0, 0.1), (12.0, 12.0, 16.0), math.cos(math.radians(30.0)),
                math.cos(math.radians(20.0)))
        a[2] = (2, (0, 0, 0), (0.2, -1.0, 0.6), (0.6, 0.55, 0.5), 0.0, 0.0)
    s.analytic = a
    return s


def write_tga(path, rgb: np.ndarray) -> None:
    """Writes an (h, w, 3) uint8 image as an uncompressed 24-bit TGA, top row
    first."""
    h, w, _ = rgb.shape
    header = bytes([0, 0, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0, w & 255, w >> 8, h & 255, h >> 8, 24, 0x20])
    with open(path, "wb") as f:
        f.write(header + np.ascontiguousarray(rgb[..., ::-1], np.uint8).tobytes())


def pbrt_text_textured(width: int, height: int, spp: int, max_depth: int, floor_tex: str, wall_tex: str) -> str:
    """pbrt_text() with image-map textures: the floor's reflectance from
    `floor_tex` (bilinear) and the back wall's from `wall_tex` (the
    frontend's default EWA filter), both with uvs spanning 3 repeats."""
    lines = pbrt_text(width, height, spp, max_depth).splitlines()
    world = lines.index("WorldBegin")
    tex = [f'Texture "floorimg" "spectrum" "imagemap" "string filename" ["{floor_tex}"] "string filter" ["bilinear"]',
           f'Texture "wallimg" "spectrum" "imagemap" "string filename" ["{wall_tex}"]',
           'MakeNamedMaterial "floortex" "string type" ["diffuse"] "texture reflectance" ["floorimg"]',
           'MakeNamedMaterial "walltex" "string type" ["diffuse"] "texture reflectance" ["wallimg"]']
    out = lines[:world + 1] + tex
    shape = 0
    for line in lines[world + 1:]:
        if line.startswith('NamedMaterial "white"') and shape in (0, 2):
            line = 'NamedMaterial "floortex"' if shape == 0 else 'NamedMaterial "walltex"'
        if line.startswith('Shape "trianglemesh"'):
            if shape in (0, 2):
                line += ' "point2 uv" [0 0 3 0 3 3 0 3]'
            shape += 1
        out.append(line)
    return "\n".join(out) + "\n"
