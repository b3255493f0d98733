"""Seeded synthetic scenes for the spectral path: the PBRT-profile inputs the benchmarks use.

``cornell_box()`` is the 36-triangle Cornell-style box (256x256, 64 spp, depth 8) and
``mixed_scene()`` the ~1.44M-triangle mixed-material mesh scene (1920x1080, 16 spp, depth 16).
Both return a ``Scene`` holding numpy arrays in the layout of ``rp_scene_desc``; ``Scene.desc()``
produces the C description (the arrays stay owned by the Scene).

Light spectra follow rypath's PBRT blackbody normalisation (src/pbrt_render.cpp:883-935): the
Planck shape divided by its 830 nm value, scaled by ``scale / sum(shape * ybar)`` over the
1 nm CIE table.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import abi

DATA = Path(__file__).resolve().parent / "data"
WAVELENGTHS = np.arange(360, 831, dtype=np.float64)


def sobol_tables() -> bytes:
    blob = (DATA / "pbrt_sobol_tables.bin").read_bytes()
    assert len(blob) == abi.RP_SOBOL_TABLE_BYTES
    return blob


def cie_xyz() -> np.ndarray:
    return np.frombuffer((DATA / "cie_xyz_1931.bin").read_bytes(), dtype="<f8").reshape(471, 3)


def blackbody_shape(kelvin: float) -> np.ndarray:
    """Planck radiance over its 830 nm value (src/pbrt_render.cpp:890-905)."""
    c2 = 6.62606957e-34 * 299792458.0 / 1.3806488e-23 * 1e9
    ref = 830.0
    ref_factor = -math.expm1(-(c2 / ref) / kelvin)
    out = np.empty(471)
    for i, w in enumerate(WAVELENGTHS):
        delta = c2 * (ref - w) / (ref * w)
        out[i] = (ref / w) ** 5 * math.exp(-delta / kelvin) * ref_factor / -math.expm1(-(c2 / w) / kelvin)
    return out


def blackbody_emission(kelvin: float, scale: float) -> np.ndarray:
    shape = blackbody_shape(kelvin)
    norm = float(np.sum(shape * cie_xyz()[:, 1]))
    return (shape * (scale / norm)).astype(np.float32)


def knots_from_curve(values, count: int = 32) -> np.ndarray:
    """A 32-bin spectrum as `count` knots evenly spaced on 360..830 nm."""
    w = np.linspace(360.0, 830.0, count, dtype=np.float32)
    v = np.asarray(values, dtype=np.float32)
    if v.ndim == 0:
        v = np.full(count, float(v), dtype=np.float32)
    return np.stack([w, v], axis=1).astype(np.float32)


@dataclass
class Scene:
    name: str
    width: int
    height: int
    spp: int
    positions: np.ndarray  # (V, 3) f32
    triangles: np.ndarray  # (T, 3) u32
    instances: list = field(default_factory=list)
    materials: list = field(default_factory=list)
    knots: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.float32))
    emissions: list = field(default_factory=list)  # (radiance[471], two_sided)
    positional: list = field(default_factory=list)  # dicts
    environment: np.ndarray | None = None
    camera: tuple = ((0, 0, 0), (0, 0, -1), (1, 0, 0), (0, -1, 0))
    filter_kind: int = abi.FILTER_BOX
    filter_radius: tuple = (0.5, 0.5)
    max_depth: int = 8
    light_sampler: int = abi.LIGHTS_BVH
    hero_wavelengths: int = abi.HERO_VISIBLE
    normals: np.ndarray | None = None
    # homogeneous media (scalar transport): dicts of sigma_a, sigma_s, emission (471 each), g
    media: list = field(default_factory=list)
    camera_medium: int = abi.RP_NONE
    transport: int = abi.TRANSPORT_HERO
    # thin lens (radius 0: pinhole): radius, focal distance, camera x / y axes
    lens: tuple = (0.0, 1e6, (1.0, 0.0, 0.0), (0.0, 1.0, 0.0))
    filter_sigma: float = 0.5
    images: object = None  # images.ImageSet: image textures and the environment image
    # RenderModel: MODEL_PBRT, or MODEL_DEMO (camera = (origin, forward, right, up) of a look-at
    # pose, film_scale = tan(fov / 2), materials' 8-knot reflectance, the unit sky)
    model: int = abi.MODEL_PBRT
    film_scale: float = 1.0
    # bilinear patches ((N, 4) vertex indices p00 p10 p01 p11, instance-local like triangles)
    # and analytic shapes (abi.Analytic records), referenced by the instances' ranges
    patches: np.ndarray | None = None
    analytics: list = field(default_factory=list)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def triangle_count(self) -> int:
        return int(self.triangles.shape[0])

    def desc(self) -> abi.SceneDesc:
        keep = []

        def arr(a, ctype):
            a = np.ascontiguousarray(a)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(ctype))

        d = abi.SceneDesc()
        d.abi_version = abi.RP_ABI_VERSION
        pos = np.ascontiguousarray(self.positions, dtype=np.float32)
        tri = np.ascontiguousarray(self.triangles, dtype=np.uint32)
        d.vertex_count, d.positions = pos.shape[0], arr(pos, C.c_float)
        d.triangle_count, d.triangles = tri.shape[0], arr(tri, C.c_uint32)
        if self.normals is not None:
            nrm = np.ascontiguousarray(self.normals, dtype=np.float32)
            d.normal_count, d.normals = nrm.shape[0], arr(nrm, C.c_float)
        inst = (abi.Instance * max(1, len(self.instances)))()
        for i, x in enumerate(self.instances):
            inst[i] = x
        keep.append(inst)
        d.instance_count, d.instances = len(self.instances), C.cast(inst, C.POINTER(abi.Instance))
        mats = (abi.Material * max(1, len(self.materials)))()
        for i, x in enumerate(self.materials):
            mats[i] = x
        keep.append(mats)
        d.material_count, d.materials = len(self.materials), C.cast(mats, C.POINTER(abi.Material))
        kn = np.ascontiguousarray(self.knots, dtype=np.float32).reshape(-1, 2)
        keep.append(kn)
        d.knot_count = kn.shape[0]
        d.knots = kn.ctypes.data_as(C.POINTER(abi.Knot))
        em = (abi.AreaEmission * max(1, len(self.emissions)))()
        for i, (rad, two) in enumerate(self.emissions):
            em[i].radiance[:] = [float(v) for v in np.asarray(rad, np.float32)]
            em[i].two_sided = int(two)
        keep.append(em)
        d.emission_count, d.emissions = len(self.emissions), C.cast(em, C.POINTER(abi.AreaEmission))
        pl = (abi.PositionalLight * max(1, len(self.positional)))()
        for i, L in enumerate(self.positional):
            pl[i].position[:] = list(L["position"])
            pl[i].intensity[:] = [float(v) for v in np.asarray(L["intensity"], np.float32)]
            pl[i].kind = L["kind"]
            pl[i].light_from_world[:] = list(L.get("light_from_world", (1, 0, 0, 0, 1, 0, 0, 0, 1)))
            pl[i].cos_falloff_start = L.get("cos_falloff_start", 1.0)
            pl[i].cos_falloff_end = L.get("cos_falloff_end", 0.0)
        keep.append(pl)
        d.positional_count = len(self.positional)
        d.positional = C.cast(pl, C.POINTER(abi.PositionalLight))
        md = (abi.Medium * max(1, len(self.media)))()
        for i, m in enumerate(self.media):
            for name in ("sigma_a", "sigma_s", "emission"):
                getattr(md[i], name)[:] = [float(v) for v in np.broadcast_to(np.asarray(m.get(name, 0.0), np.float32),
                                                                             (471,))]
            md[i].g = float(m.get("g", 0.0))
        keep.append(md)
        d.medium_count, d.media = len(self.media), C.cast(md, C.POINTER(abi.Medium))
        d.camera_medium = self.camera_medium
        if self.environment is not None:
            d.environment = arr(np.asarray(self.environment, np.float32), C.c_float)
        o, corner, dx, dy = self.camera
        d.camera.origin[:] = list(o)
        d.camera.corner[:] = list(corner)
        d.camera.dx[:] = list(dx)
        d.camera.dy[:] = list(dy)
        d.filter_kind = self.filter_kind
        d.filter_x_radius, d.filter_y_radius = self.filter_radius
        d.filter_sigma = self.filter_sigma
        d.lens_radius, d.focal_distance = self.lens[0], self.lens[1]
        d.lens_x[:] = list(self.lens[2])
        d.lens_y[:] = list(self.lens[3])
        d.max_depth = self.max_depth
        d.light_sampler = self.light_sampler
        d.transport = self.transport
        d.hero_wavelengths = self.hero_wavelengths
        tables = C.create_string_buffer(sobol_tables(), abi.RP_SOBOL_TABLE_BYTES)
        keep.append(tables)
        d.sobol_tables = C.cast(tables, C.c_void_p)
        d.model, d.film_scale = self.model, self.film_scale
        if self.patches is not None and len(self.patches):
            pt = np.ascontiguousarray(self.patches, dtype=np.uint32).reshape(-1, 4)
            d.patch_count, d.patches = pt.shape[0], arr(pt, C.c_uint32)
        if self.analytics:
            an = (abi.Analytic * len(self.analytics))(*self.analytics)
            keep.append(an)
            d.analytic_count, d.analytics = len(self.analytics), C.cast(an, C.POINTER(abi.Analytic))
        if self.images is not None:
            im = self.images.to_c(keep)
            keep.append(im)
            d.images = C.pointer(im)
        self._keep = keep
        return d


def identity_instance(vertex_begin, triangle_begin, triangle_count, material, emission=abi.RP_NONE):
    inst = abi.Instance()
    inst.matrix[:] = [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0]
    inst.vertex_begin, inst.triangle_begin, inst.triangle_count = vertex_begin, triangle_begin, triangle_count
    inst.material, inst.emission = material, emission
    inst.reverse_orientation = 0
    inst.normal_begin = abi.RP_NONE
    inst.inside_medium = inst.outside_medium = abi.RP_NONE
    inst.patch_begin = inst.analytic_begin = abi.RP_NONE
    inst.patch_count = inst.analytic_count = 0
    return inst


def diffuse_material(knot_begin, knot_count=32):
    m = abi.Material()
    m.scattering, m.kind, m.knot_begin, m.knot_count = abi.DIFFUSE, abi.REFLECTANCE_KNOTS, knot_begin, knot_count
    m.remap_roughness = 1
    return m


def thin_lens(origin, target, up, radius, focal_distance=None):
    """PerspectiveLens (src/render.hpp:159-164) of a pinhole_camera pose: aperture radius, focal
    distance (default: the distance to target) and the camera's x / y axes in world space."""
    o = np.asarray(origin, np.float64)
    f = np.asarray(target, np.float64) - o
    dist = float(np.linalg.norm(f))
    f /= dist
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    return (float(radius), float(focal_distance or dist), tuple(r.astype(np.float32)), tuple(u.astype(np.float32)))


def pinhole_camera(origin, target, up, vfov_degrees, width, height):
    """A PBRT perspective camera as the raster basis of RasterCamera (src/render.hpp:152)."""
    o = np.asarray(origin, np.float64)
    f = np.asarray(target, np.float64) - o
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    aspect = width / height
    # PBRT's fov spans the shorter image axis.
    t = math.tan(math.radians(vfov_degrees) / 2)
    tx, ty = (t * aspect, t) if aspect >= 1 else (t, t / aspect)
    corner = f - tx * r + ty * u
    dx = 2 * tx * r
    dy = -2 * ty * u
    return tuple(o.astype(np.float32)), tuple(corner.astype(np.float32)), tuple(dx.astype(np.float32)), tuple(
        dy.astype(np.float32))


def _box(lo, hi):
    """12 outward-wound triangles of an axis-aligned box."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float32)
    t = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [3, 7, 6], [3, 6, 2], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.uint32)
    return v, t


def _quad(a, b, c, d):
    return np.array([a, b, c, d], np.float32), np.array([[0, 1, 2], [0, 2, 3]], np.uint32)


def cornell_box(width=256, height=256, spp=64, max_depth=8) -> Scene:
    """Cornell-style box: 5 walls (10 tris), two boxes (24 tris), one quad light (2 tris)."""
    parts = []  # (verts, tris, material, emission)
    # walls, wound so their geometric normals face the interior
    parts.append(_quad((-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1)) + (0, None))    # floor
    parts.append(_quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)) + (0, None))    # ceiling
    parts.append(_quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)) + (0, None))  # back
    parts.append(_quad((-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1)) + (1, None))  # left (red)
    parts.append(_quad((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)) + (2, None))      # right (green)
    # short and tall boxes (axis aligned)
    parts.append(_box((0.10, 0.0, -0.10), (0.70, 0.60, 0.50)) + (0, None))
    parts.append(_box((-0.75, 0.0, -0.70), (-0.15, 1.20, -0.10)) + (0, None))
    # light quad just below the ceiling, facing down
    parts.append(_quad((-0.25, 1.98, -0.25), (0.25, 1.98, -0.25), (0.25, 1.98, 0.25), (-0.25, 1.98, 0.25))
                 + (3, 0))
    positions, triangles, instances = [], [], []
    vb = tb = 0
    for verts, tris, mat, emission in parts:
        positions.append(verts)
        triangles.append(tris)
        instances.append(identity_instance(vb, tb, len(tris), mat,
                                           abi.RP_NONE if emission is None else emission))
        vb += len(verts)
        tb += len(tris)
    positions = np.concatenate(positions)
    triangles = np.concatenate(triangles)
    w = np.linspace(360, 830, 32)
    white = knots_from_curve(0.73)
    red = knots_from_curve(np.interp(w, [360, 560, 610, 830], [0.05, 0.05, 0.65, 0.70]))
    green = knots_from_curve(np.interp(w, [360, 470, 530, 580, 830], [0.05, 0.08, 0.55, 0.10, 0.05]))
    black = knots_from_curve(0.0)
    knots = np.concatenate([white, red, green, black])
    materials = [diffuse_material(0), diffuse_material(32), diffuse_material(64), diffuse_material(96)]
    light = blackbody_emission(6500.0, 17.0)
    scene = Scene("cornell_box", width, height, spp, positions, triangles, instances, materials, knots,
                  emissions=[(light, False)], max_depth=max_depth)
    scene.camera = pinhole_camera((0, 1, 3.94), (0, 1, 0), (0, 1, 0), 40.0, width, height)
    return scene


def mix_material(first, second, amount):
    """A mix of materials `first` and `second` (indices): second where the alpha hash is below amount."""
    m = abi.Material()
    m.scattering, m.kind = abi.MIX, abi.REFLECTANCE_CONSTANT
    m.first_material, m.second_material, m.mix_amount = first, second, amount
    return m


def _append_knots(scene, values):
    begin = scene.knots.shape[0]
    scene.knots = np.concatenate([scene.knots, knots_from_curve(values)])
    return begin


def cornell_pass_through(width=256, height=256, spp=64, max_depth=8, pane=True, invisible_light=True,
                         mixes=True) -> Scene:
    """The Cornell-style box with the hero transport's pass-through and mix surfaces.

    pane: a null-interface quad across the box opening (camera and shadow rays cross it);
    invisible_light: the area light is an invisible emitter (rays pass through it, light
    sampling still reaches it); mixes: the short box is mix(white, rough conductor, 0.35), the
    tall box mix(mix(white, glass, 0.5), red, 0.7).
    """
    scene = cornell_box(width, height, spp, max_depth)
    scene.name = "cornell_pass_through"
    if invisible_light:
        scene.instances[-1].invisible_emitter = 1
    if mixes:
        conductor = abi.Material()
        conductor.scattering, conductor.kind, conductor.scalar_value = abi.CONDUCTOR, abi.REFLECTANCE_CONSTANT, 1.0
        conductor.eta_begin, conductor.eta_count = _append_knots(scene, 0.25), 32
        conductor.k_begin, conductor.k_count = _append_knots(scene, 3.2), 32
        conductor.optical_extensions, conductor.u_roughness, conductor.v_roughness = 3, 0.3, 0.3
        conductor.remap_roughness = 1
        glass = abi.Material()
        glass.scattering, glass.kind, glass.scalar_value = abi.DIELECTRIC, abi.REFLECTANCE_CONSTANT, 1.0
        glass.eta_begin, glass.eta_count, glass.optical_extensions = _append_knots(scene, 1.5), 32, 1
        base = len(scene.materials)
        scene.materials += [conductor, glass]
        scene.materials.append(mix_material(0, base, 0.35))          # base + 2: short box
        scene.materials.append(mix_material(0, base + 1, 0.5))       # base + 3: inner mix
        scene.materials.append(mix_material(base + 3, 1, 0.7))       # base + 4: tall box
        scene.instances[5].material = base + 2
        scene.instances[6].material = base + 4
    if pane:
        verts, tris = _quad((-1, 0.3, 0.8), (1, 0.3, 0.8), (1, 1.7, 0.8), (-1, 1.7, 0.8))
        interface = abi.Material()
        interface.scattering, interface.kind = abi.INTERFACE, abi.REFLECTANCE_CONSTANT
        scene.materials.append(interface)
        scene.instances.append(identity_instance(scene.positions.shape[0], scene.triangles.shape[0], 2,
                                                 len(scene.materials) - 1))
        scene.positions = np.concatenate([scene.positions, verts])
        scene.triangles = np.concatenate([scene.triangles, tris])
    return scene


CORNELL_FEATURES = ("point", "spot", "environment", "cauchy", "env_image", "texture")


def cauchy_dielectric(scene, a=1.5, b_um2=0.004):
    """A smooth dielectric whose eta follows Cauchy's n = a + b / lambda^2 (lambda in um), as
    32 sampled knots (rypath has no Cauchy model; a sampled eta spectrum stands in)."""
    w = np.linspace(360, 830, 32)
    m = abi.Material()
    m.scattering, m.kind, m.scalar_value = abi.DIELECTRIC, abi.REFLECTANCE_CONSTANT, 1.0
    m.eta_begin, m.eta_count, m.optical_extensions = _append_knots(scene, a + b_um2 / (w / 1000.0) ** 2), 32, 1
    m.k_begin = m.k_count = 0
    m.u_roughness = m.v_roughness = 0.0
    m.remap_roughness = 1
    return m


def cornell_features(feature, width=32, height=32, spp=4, max_depth=8) -> Scene:
    """The Cornell-style box with one light or material feature of the mixed-material scene, so
    that each can be checked on its own:

    point: the area light replaced by a blackbody point light below the ceiling;
    spot: the area light replaced by a spot light pointing down at the short box;
    environment: the area light replaced by a constant environment seen through the open front;
    cauchy: the tall box made of a smooth dispersive (Cauchy) dielectric, the short box of a
    rough conductor, under the area light;
    env_image: the area light replaced by an equal-area octahedral sky image (float texels,
    a bright sun shining in through the open front), sampled by its importance tables;
    texture: image reflectance on the back wall (sRGB 8-bit, trilinear, tiled), the floor (float,
    EWA) and the tall box (half, point, clamped), and RGB (sigmoid) reflectance on the short box,
    under the area light.
    """
    if feature not in CORNELL_FEATURES:
        raise ValueError(f"unknown feature {feature!r}")
    scene = cornell_box(width, height, spp, max_depth)
    scene.name = f"cornell_{feature}"
    if feature in ("point", "spot", "environment", "env_image"):
        scene.instances[-1].emission = abi.RP_NONE  # the quad stays, as a black diffuse panel
        scene.emissions = []
    if feature == "point":
        scene.positional = [{"kind": abi.POINT_LIGHT, "position": (0.2, 1.7, 0.3),
                             "intensity": blackbody_emission(3200, 3.0)}]
    elif feature == "spot":
        scene.positional = [_spot((-0.1, 1.9, 0.4), (0.4, 0.6, 0.2), 20.0, 30.0, blackbody_emission(5000, 8.0))]
    elif feature == "environment":
        scene.environment = (1.5 * blackbody_shape(9000) / blackbody_shape(9000).max()).astype(np.float32)
    elif feature == "texture":
        textured_cornell(scene)
    elif feature == "env_image":
        from . import images

        scene.images = images.ImageSet()
        scene.images.environment_image = scene.images.add_image(images.sky_image(32, seed=3), wrap=abi.WRAP_CLAMP)
        scene.images.environment_scale = 1.5
    else:
        conductor = abi.Material()
        conductor.scattering, conductor.kind, conductor.scalar_value = abi.CONDUCTOR, abi.REFLECTANCE_CONSTANT, 1.0
        conductor.eta_begin, conductor.eta_count = _append_knots(scene, 0.4), 32
        conductor.k_begin, conductor.k_count = _append_knots(scene, 3.0), 32
        conductor.optical_extensions, conductor.u_roughness, conductor.v_roughness = 3, 0.2, 0.2
        conductor.remap_roughness = 1
        base = len(scene.materials)
        scene.materials += [conductor, cauchy_dielectric(scene)]
        scene.instances[5].material = base
        scene.instances[6].material = base + 1
    return scene


def conductor_material(scene, eta, k, u, v, remap=True):
    """A GGX conductor with constant optical constants (32 knots each, extended)."""
    m = abi.Material()
    m.scattering, m.kind, m.scalar_value = abi.CONDUCTOR, abi.REFLECTANCE_CONSTANT, 1.0
    m.eta_begin, m.eta_count = _append_knots(scene, eta), 32
    m.k_begin, m.k_count = _append_knots(scene, k), 32
    m.optical_extensions, m.u_roughness, m.v_roughness = 3, u, v
    m.remap_roughness = int(remap)
    return m


def dielectric_material(scene, eta, roughness, remap=True):
    """A GGX dielectric with a constant eta (32 knots, extended)."""
    m = abi.Material()
    m.scattering, m.kind, m.scalar_value = abi.DIELECTRIC, abi.REFLECTANCE_CONSTANT, 1.0
    m.eta_begin, m.eta_count, m.optical_extensions = _append_knots(scene, eta), 32, 1
    m.u_roughness = m.v_roughness = roughness
    m.remap_roughness = int(remap)
    return m


def cornell_microfacets(width=32, height=32, spp=4, max_depth=8, transport=abi.TRANSPORT_SCALAR) -> Scene:
    """The Cornell-style box with every microfacet case of the transport: the short box a rough
    anisotropic conductor, the tall box rough glass (eta 1.5), the right wall a smooth (Dirac)
    mirror, under the area light."""
    scene = cornell_box(width, height, spp, max_depth)
    scene.name = "cornell_microfacets"
    base = len(scene.materials)
    scene.materials += [conductor_material(scene, 0.2, 3.4, 0.3, 0.08), dielectric_material(scene, 1.5, 0.04),
                        conductor_material(scene, 1.1, 4.0, 0.0, 0.0)]
    scene.instances[5].material = base
    scene.instances[6].material = base + 1
    scene.instances[4].material = base + 2
    scene.transport = transport
    return scene


def _procedural_instance(material, vertex_begin=0, patches=(0, 0), analytics=(0, 0), matrix=None):
    inst = identity_instance(vertex_begin, 0, 0, material)
    inst.patch_begin, inst.patch_count = patches
    inst.analytic_begin, inst.analytic_count = analytics
    if matrix is not None:
        inst.matrix[:] = [float(v) for v in np.asarray(matrix, np.float32).reshape(-1)]
    return inst


def _rotation_y(degrees, translation=(0, 0, 0), scale=(1, 1, 1)):
    c, s = math.cos(math.radians(degrees)), math.sin(math.radians(degrees))
    r = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]]) @ np.diag(scale)
    return np.concatenate([r, np.asarray(translation, np.float64)[:, None]], axis=1)


def add_patches(scene: Scene, corners, material, matrix=None) -> None:
    """Append an instance of bilinear patches; `corners` is (N, 4, 3), each p00 p10 p01 p11."""
    corners = np.asarray(corners, np.float32).reshape(-1, 4, 3)
    begin = 0 if scene.patches is None else scene.patches.shape[0]
    vb = scene.positions.shape[0]
    idx = np.arange(4 * corners.shape[0], dtype=np.uint32).reshape(-1, 4)
    scene.positions = np.concatenate([scene.positions, corners.reshape(-1, 3)])
    scene.patches = idx if scene.patches is None else np.concatenate([scene.patches, idx])
    scene.instances.append(_procedural_instance(material, vb, patches=(begin, corners.shape[0]), matrix=matrix))


def add_analytics(scene: Scene, records, material, matrix=None) -> None:
    """Append an instance of analytic shapes (abi.Analytic records)."""
    begin = len(scene.analytics)
    scene.analytics = list(scene.analytics) + list(records)
    scene.instances.append(_procedural_instance(material, analytics=(begin, len(records)), matrix=matrix))


def analytic(subtype, radius, z_min=-1.0, z_max=1.0, phi_max=2 * math.pi, inner_radius=0.0, height=0.0):
    a = abi.Analytic()
    a.kind, a.subtype = abi.PRIMITIVE_ANALYTIC, subtype
    a.radius, a.z_min, a.z_max, a.phi_max, a.inner_radius, a.height = radius, z_min, z_max, phi_max, inner_radius, height
    return a


def cornell_shapes(width=32, height=32, spp=4, max_depth=8, transport=abi.TRANSPORT_HERO) -> Scene:
    """The Cornell-style box with procedural primitives: the left wall a planar bilinear patch,
    a warped patch 'sail' in front of the back wall (rotated instance), the tall box replaced by
    a capped cylinder (a cylinder and a holed disk, axis along +y by the instance rotation), and
    a rough-glass ellipsoid (a sphere scaled by the instance) on the short box."""
    scene = cornell_box(width, height, spp, max_depth)
    scene.name = "cornell_shapes"
    # left wall: the patch of its quad's corners, replacing its two triangles
    scene.instances[3].triangle_count = 0
    add_patches(scene, [[(-1, 0, -1), (-1, 2, -1), (-1, 0, 1), (-1, 2, 1)]], 1)
    add_patches(scene, [[(-0.6, 0.9, -0.1), (0.2, 1.1, -0.05), (-0.7, 1.7, -0.15), (0.3, 1.6, 0.1)]], 2,
                matrix=_rotation_y(12.0, (0.1, 0.0, -0.75)))
    scene.instances[6].triangle_count = 0  # the tall box
    axis_y = np.array([[1, 0, 0, -0.45], [0, 0, 1, 0.0], [0, -1, 0, -0.4]])
    add_analytics(scene, [analytic(abi.ANALYTIC_CYLINDER, 0.28, 0.0, 1.1),
                          analytic(abi.ANALYTIC_DISK, 0.28, 0, 0, 2 * math.pi, 0.08, 1.1)], 0, matrix=axis_y)
    scene.materials.append(dielectric_material(scene, 1.5, 0.05))
    add_analytics(scene, [analytic(abi.ANALYTIC_SPHERE, 0.2, -0.2, 0.2)], len(scene.materials) - 1,
                  matrix=_rotation_y(30.0, (0.4, 0.78, 0.2), (1.0, 0.8, 1.2)))
    scene.transport = transport
    return scene


def shape_furnace(kind, width=16, height=16, spp=4, rho=0.5, transport=abi.TRANSPORT_HERO) -> Scene:
    """One convex diffuse object of constant reflectance rho under a constant environment of
    radiance 1 at every wavelength (kind: 'sphere', 'disk', 'cylinder' -- open, seen from the
    side -- or 'patch', a flat one): no ray leaving it meets it again, so every camera ray that
    hits it returns rho on average and every other 1."""
    scene = Scene(f"furnace_{kind}", width, height, spp, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32),
                  [], [], max_depth=8)
    m = abi.Material()
    m.scattering, m.kind, m.scalar_value = abi.DIFFUSE, abi.REFLECTANCE_CONSTANT, rho
    scene.materials = [m]
    tilt = _rotation_y(25.0, (0, 0, 0))
    if kind == "sphere":
        add_analytics(scene, [analytic(abi.ANALYTIC_SPHERE, 0.6, -0.6, 0.6)], 0, matrix=tilt)
    elif kind == "disk":
        add_analytics(scene, [analytic(abi.ANALYTIC_DISK, 0.7, 0, 0, 2 * math.pi, 0.2, 0.1)], 0,
                      matrix=np.array([[1, 0, 0, 0], [0, 0.8, 0.6, 0], [0, -0.6, 0.8, 0]]))
    elif kind == "cylinder":
        add_analytics(scene, [analytic(abi.ANALYTIC_CYLINDER, 0.4, -0.6, 0.6)], 0,
                      matrix=np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, -1, 0, 0]]))
    else:
        add_patches(scene, [[(-0.7, -0.6, 0.2), (0.7, -0.5, -0.1), (-0.6, 0.7, -0.2), (0.8, 0.8, -0.5)]], 0,
                    matrix=tilt)  # a parallelogram: flat
    scene.environment = np.ones(471, np.float32)
    scene.camera = pinhole_camera((0, 0, 3.0), (0, 0, 0), (0, 1, 0), 40.0, width, height)
    scene.transport = transport
    return scene


def triangle_frames(positions, triangles, uvs):
    """PBRT's triangle texture partials (dp/du, dp/dv from the vertices' uvs; for a degenerate
    uv parameterisation a frame around the geometric normal), per triangle, as (T, 6) float32."""
    p = np.asarray(positions, np.float64)[np.asarray(triangles)]
    t = np.asarray(uvs, np.float64)[np.asarray(triangles)]
    duv02, duv12 = t[:, 0] - t[:, 2], t[:, 1] - t[:, 2]
    dp02, dp12 = p[:, 0] - p[:, 2], p[:, 1] - p[:, 2]
    det = duv02[:, 0] * duv12[:, 1] - duv02[:, 1] * duv12[:, 0]
    safe = np.where(np.abs(det) < 1e-9, 1.0, det)
    dpdu = (duv12[:, 1:2] * dp02 - duv02[:, 1:2] * dp12) / safe[:, None]
    dpdv = (duv02[:, 0:1] * dp12 - duv12[:, 0:1] * dp02) / safe[:, None]
    n = np.cross(p[:, 2] - p[:, 0], p[:, 1] - p[:, 0])
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    sign = np.copysign(1.0, n[:, 2])
    a = -1 / (sign + n[:, 2])
    b = n[:, 0] * n[:, 1] * a
    fu = np.stack([1 + sign * n[:, 0] ** 2 * a, sign * b, -sign * n[:, 0]], 1)
    fv = np.stack([b, sign + n[:, 1] ** 2 * a, -n[:, 1]], 1)
    bad = (np.abs(det) < 1e-9)[:, None] | (np.linalg.norm(np.cross(dpdu, dpdv), axis=1) == 0)[:, None]
    dpdu, dpdv = np.where(bad, fu, dpdu), np.where(bad, fv, dpdv)
    return np.concatenate([dpdu, dpdv], axis=1).astype(np.float32)


def texture_camera(origin, target, up):
    """TextureCamera (src/texture_footprint.hpp:9-12) of a look-at pose: world_from_camera's
    columns are the camera's right, up and forward axes (row-major), camera_from_world its
    transpose."""
    o, t = np.asarray(origin, np.float64), np.asarray(target, np.float64)
    f = (t - o) / np.linalg.norm(t - o)
    r = np.cross(np.asarray(up, np.float64), f)
    r /= np.linalg.norm(r)
    u = np.cross(f, r)
    m = np.stack([r, u, f], axis=1)
    return tuple(m.reshape(-1).astype(np.float32)), tuple(m.T.reshape(-1).astype(np.float32))


def textured_cornell(scene: Scene) -> None:
    """Give the Cornell box's back wall, floor and tall box image reflectance (see
    cornell_features("texture")): per-vertex uvs by planar projection, PBRT triangle frames, the
    texture camera of the box's pose, and three seeded images."""
    from . import images

    rng = np.random.default_rng(11)
    pos = scene.positions.astype(np.float64)
    # planar projections: floor / ceiling / boxes' tops on (x, z), walls on (x, y) or (z, y)
    uv = np.stack([0.5 * pos[:, 0] + 0.5, 0.5 * pos[:, 1]], 1)
    for inst in (scene.instances[0], scene.instances[1]):
        vs = slice(inst.vertex_begin, inst.vertex_begin + 4)
        uv[vs] = np.stack([0.5 * pos[vs, 0] + 0.5, 0.5 * pos[vs, 2] + 0.5], 1)
    for k in (3, 4):
        inst = scene.instances[k]
        vs = slice(inst.vertex_begin, inst.vertex_begin + 4)
        uv[vs] = np.stack([0.5 * pos[vs, 2] + 0.5, 0.5 * pos[vs, 1]], 1)
    tall = scene.instances[6]
    vs = slice(tall.vertex_begin, tall.vertex_begin + 8)
    uv[vs] = np.stack([(pos[vs, 0] + pos[vs, 2]) * 0.8 + 0.5, pos[vs, 1] / 1.2], 1)
    s = images.ImageSet()
    yy, xx = np.mgrid[0:64, 0:64]
    check = ((xx // 8 + yy // 8) % 2).astype(np.float64)
    base = np.stack([0.15 + 0.7 * check, 0.2 + 0.5 * (1 - check), 0.3 + 0.2 * rng.uniform(size=(64, 64))], 2)
    codes = [np.round(np.clip(c, 0, 1) * 255).astype(np.uint8) for c in images.box_pyramid(base)]
    back = s.add_image(codes, abi.TEXELS_SRGB8, abi.WRAP_REPEAT, abi.TEXTURE_TRILINEAR, uvscale=(3.0, 2.0))
    stripes = np.stack([0.3 + 0.6 * ((xx % 16) < 8), np.full((64, 64), 0.5), 0.2 + 0.7 * (yy / 63.0)], 2)
    floor = s.add_image([c.astype(np.float32) for c in images.box_pyramid(stripes[:32, :32])], abi.TEXELS_FLOAT,
                        abi.WRAP_REPEAT, abi.TEXTURE_EWA, uvscale=(2.0, 2.0), uvdelta=(0.25, 0.0))
    noise = rng.uniform(0.05, 0.95, (16, 16, 3)).astype(np.float32)
    box = s.add_image(noise, abi.TEXELS_HALF, abi.WRAP_CLAMP, abi.TEXTURE_POINT)
    first = len(scene.materials)
    for index in (back, floor, box):
        m = abi.Material()
        m.scattering, m.kind, m.image_texture = abi.DIFFUSE, abi.REFLECTANCE_IMAGE, index
        m.remap_roughness = 1
        scene.materials.append(m)
    # the short box: PBRT RGB reflectance (sigmoid polynomial coefficients, a warm orange)
    rgb = abi.Material()
    rgb.scattering, rgb.kind, rgb.remap_roughness = abi.DIFFUSE, abi.REFLECTANCE_RGB, 1
    rgb.coefficients[:] = [-2.0e-4, 0.24, -68.0]
    scene.materials.append(rgb)
    scene.instances[2].material = first
    scene.instances[0].material = first + 1
    scene.instances[6].material = first + 2
    scene.instances[5].material = first + 3
    s.uvs = uv.astype(np.float32)
    s.instance_uv_begin = [inst.vertex_begin for inst in scene.instances]
    s.frames = triangle_frames(scene.positions, scene.triangles, s.uvs)
    s.instance_frame_begin = [inst.triangle_begin for inst in scene.instances]
    s.world_from_camera, s.camera_from_world = texture_camera((0, 1, 3.94), (0, 1, 0), (0, 1, 0))
    scene.images = s


def demo_camera(origin, target, up, vfov_degrees):
    """The demo model's camera slots (src/metal_render.mm:194-204): origin and the unit
    forward / right / up of the look-at pose (double, rounded to binary32), and
    tan(vfov / 2)."""
    o, t, u = (np.asarray(v, np.float32).astype(np.float64) for v in (origin, target, up))  # RenderCamera is binary32
    f = (t - o) / np.linalg.norm(t - o)
    r = np.cross(f, u)
    r /= np.linalg.norm(r)
    up2 = np.cross(r, f)
    scale = float(np.float32(math.tan(float(np.float32(vfov_degrees)) * (math.pi / 360.0))))
    return (tuple(np.float32(o)), tuple(f.astype(np.float32)), tuple(r.astype(np.float32)),
            tuple(up2.astype(np.float32))), scale


def demo_material(reflectance):
    m = abi.Material()
    m.scattering, m.kind = abi.DIFFUSE, abi.REFLECTANCE_KNOTS
    m.reflectance[:] = [float(v) for v in reflectance]
    m.remap_roughness = 1
    return m


def _demo_box(offset, scale, angle):
    """A unit box placement of the demo scene (box_transform, src/render.cpp:821-827), in binary32
    with the C library's cosf / sinf."""
    libm = C.CDLL("libm.so.6")
    libm.cosf.restype = libm.sinf.restype = C.c_float
    libm.cosf.argtypes = libm.sinf.argtypes = [C.c_float]
    f = np.float32
    x, y, z = (f(v) for v in offset)
    w, h, d = (f(v) for v in scale)
    c, s = f(libm.cosf(f(angle))), f(libm.sinf(f(angle)))
    return [float(v) for v in (c * w, 0, s * d, x, 0, h, 0, y, -s * w, 0, c * d, z)]


def demo_scene(width=256, height=192, spp=128, max_depth=5) -> Scene:
    """rypath's `--render-demo` scene (demo-v1, make_demo_scene, src/render.cpp:2060-2106): a
    floor and two walls, three rotated boxes, six 8-knot diffuse reflectances, under the demo
    model's unit sky, through its look-at camera; scalar transport, depth 5."""
    quads = [((-3, 0, -3), (-3, 0, 3), (3, 0, 3), (3, 0, -3)),
             ((-3, 0, -3), (3, 0, -3), (3, 3.2, -3), (-3, 3.2, -3)),
             ((-3, 0, 3), (-3, 0, -3), (-3, 3.2, -3), (-3, 3.2, 3))]
    cube = np.array([(-0.5, 0, -0.5), (0.5, 0, -0.5), (0.5, 0, 0.5), (-0.5, 0, 0.5),
                     (-0.5, 1, -0.5), (0.5, 1, -0.5), (0.5, 1, 0.5), (-0.5, 1, 0.5)], np.float32)
    cube_tris = np.array([(0, 1, 2), (0, 2, 3), (4, 6, 5), (4, 7, 6), (0, 4, 5), (0, 5, 1), (1, 5, 6), (1, 6, 2),
                          (2, 6, 7), (2, 7, 3), (3, 7, 4), (3, 4, 0)], np.uint32)
    positions = [np.array(q, np.float32) for q in quads] + [cube]
    triangles = [np.array([(0, 1, 2), (0, 2, 3)], np.uint32)] * 3 + [cube_tris]
    vb = np.cumsum([0] + [len(p) for p in positions])
    tb = np.cumsum([0] + [len(t) for t in triangles])
    instances = [identity_instance(int(vb[i]), int(tb[i]), 2, i) for i in range(3)]
    for k, box in enumerate([((-1.25, -0.05, -0.6), (1.25, 2.25, 1.25), 0.18),
                             ((0.25, -0.05, 0.8), (1.45, 1.08, 1.3), -0.24),
                             ((1.4, -0.05, -1.5), (1.07, 1.55, 1.06), 0.44)]):
        inst = identity_instance(int(vb[3]), int(tb[3]), 12, 3 + k)
        inst.matrix[:] = _demo_box(*box)
        instances.append(inst)
    reflectances = [(0.54, 0.54, 0.55, 0.58, 0.61, 0.63, 0.65, 0.65), (0.69, 0.68, 0.67, 0.65, 0.64, 0.62, 0.61, 0.61),
                    (0.34, 0.34, 0.36, 0.43, 0.55, 0.61, 0.63, 0.63), (0.10, 0.10, 0.16, 0.52, 0.40, 0.09, 0.06, 0.06),
                    (0.07, 0.08, 0.09, 0.13, 0.39, 0.73, 0.72, 0.72), (0.32, 0.47, 0.72, 0.23, 0.11, 0.08, 0.09, 0.09)]
    scene = Scene("demo_v1", width, height, spp, np.concatenate(positions), np.concatenate(triangles), instances,
                  [demo_material(r) for r in reflectances], max_depth=max_depth)
    scene.camera, scene.film_scale = demo_camera((4.1, 3.0, 6.2), (0, 1, -0.45), (0, 1, 0), 42.0)
    scene.model = abi.MODEL_DEMO
    scene.transport = abi.TRANSPORT_SCALAR
    return scene


def demo_microfacets(width=64, height=48, spp=8, max_depth=5) -> Scene:
    """The demo scene with its three boxes made a rough conductor, smooth glass and rough glass
    (the demo model shades conductors and dielectrics with rho = 1 and the unit sky)."""
    scene = demo_scene(width, height, spp, max_depth)
    scene.name = "demo_microfacets"
    base = len(scene.materials)
    scene.materials += [conductor_material(scene, 0.25, 3.1, 0.12, 0.12), dielectric_material(scene, 1.45, 0.0),
                        dielectric_material(scene, 1.6, 0.1)]
    for k in range(3):
        scene.instances[3 + k].material = base + k
    return scene


def demo_floor(reflectance=None, width=1, height=1) -> Scene:
    """The demo model's analytic fixtures (tests/render_tests.cpp): with reflectance None, the
    bare sky (no geometry); else an unbounded-looking Lambertian floor under the unit sky, seen
    straight down from above, so every path hits the floor once and then escapes."""
    if reflectance is None:
        scene = Scene("demo_sky", width, height, 1, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32), [], [],
                      max_depth=5)
    else:
        big = 1e4
        pos = np.array([(-big, 0, -big), (-big, 0, big), (big, 0, big), (big, 0, -big)], np.float32)
        scene = Scene("demo_floor", width, height, 1, pos, np.array([(0, 1, 2), (0, 2, 3)], np.uint32),
                      [identity_instance(0, 0, 2, 0)], [demo_material(reflectance)], max_depth=5)
    scene.camera, scene.film_scale = demo_camera((0, 1, 0), (0, 0, 0.0001), (0, 0, 1), 1.0)
    scene.model = abi.MODEL_DEMO
    scene.transport = abi.TRANSPORT_SCALAR
    return scene


def with_environment_image(scene: Scene, width=256, seed=2, scale=0.03) -> Scene:
    """Replace a scene's constant environment by a seeded equal-area octahedral sky image
    (float texels, images.sky_image) of the given size and radiance scale, the sky's zenith
    along the scene's +y."""
    from . import images

    s = scene.images if scene.images is not None else images.ImageSet()
    s.environment_image = s.add_image(images.sky_image(width, seed=seed), abi.TEXELS_FLOAT, abi.WRAP_CLAMP)
    s.environment_scale = scale
    # environment frame: world +y is the map's +z (zenith), world +z its +x
    s.environment_from_world = (0, 0, 1, 1, 0, 0, 0, 1, 0)
    scene.images = s
    scene.environment = None
    scene.name = scene.name + "_env_image"
    return scene


def crop(scene: Scene, x0: int, y0: int, width: int, height: int) -> Scene:
    """The window [x0, x0 + width) x [y0, y0 + height) of a scene's film as a scene of its own:
    the same geometry, lights and materials, its raster camera narrowed to the window."""
    if not (0 <= x0 and 0 <= y0 and width > 0 and height > 0 and x0 + width <= scene.width
            and y0 + height <= scene.height):
        raise ValueError("crop window outside the film")
    import copy

    out = copy.copy(scene)
    o, corner, dx, dy = (np.asarray(v, np.float64) for v in scene.camera)
    corner = corner + (x0 / scene.width) * dx + (y0 / scene.height) * dy
    dx = dx * (width / scene.width)
    dy = dy * (height / scene.height)
    out.camera = tuple(tuple(v.astype(np.float32)) for v in (o, corner, dx, dy))
    out.width, out.height = width, height
    out.name = f"{scene.name}_crop"
    out._keep = []
    return out


def cornell_fog(width=1024, height=1024, spp=64, max_depth=32, sigma_s_mean=0.5, albedo=0.9, g=0.7) -> Scene:
    """The Cornell-style box filled with a homogeneous medium, rendered by the scalar transport.

    The box interior is closed at the open front by a null interface quad (inside: the medium,
    outside: vacuum), so camera rays enter the medium there.  sigma_s ramps linearly over the
    spectrum around its mean (+-20%), sigma_a = sigma_s (1 - albedo) / albedo, HG asymmetry g.
    """
    scene = cornell_box(width, height, spp, max_depth)
    scene.name = "cornell_fog"
    sigma_s = sigma_s_mean * (1.0 + 0.2 * np.linspace(-1.0, 1.0, 471))
    sigma_a = sigma_s * (1.0 - albedo) / albedo
    scene.media = [dict(sigma_a=sigma_a.astype(np.float32), sigma_s=sigma_s.astype(np.float32), emission=0.0, g=g)]
    # front interface: the plane z = 1 over the box opening, normal +z (towards the camera)
    verts, tris = _quad((-1, 0, 1), (1, 0, 1), (1, 2, 1), (-1, 2, 1))
    interface = abi.Material()
    interface.scattering, interface.kind = abi.INTERFACE, abi.REFLECTANCE_CONSTANT
    scene.materials.append(interface)
    inst = identity_instance(scene.positions.shape[0], scene.triangles.shape[0], 2, len(scene.materials) - 1)
    inst.inside_medium, inst.outside_medium = 0, abi.RP_NONE
    scene.instances.append(inst)
    # every other surface keeps the medium on both sides: inside == outside (no change)
    scene.positions = np.concatenate([scene.positions, verts])
    scene.triangles = np.concatenate([scene.triangles, tris])
    scene.transport = abi.TRANSPORT_SCALAR
    return scene


def cornell_groups(width=512, height=512, spp=32, max_depth=8, seed=1, start=0.5):
    """The Cornell-style box with 16 reflectance groups of 32 knots each, for differentiation.

    Groups: the 5 walls, the 6 faces of the short box, and the tall box's faces with its top
    and bottom sharing a group (5), 16 in all; the light keeps its black material.  Returns
    (scene, truth): ``scene`` starts every group at the constant ``start`` reflectance and
    ``truth`` (same geometry) holds seeded smooth ground-truth spectra in [0.1, 0.9].
    Materials 0..15 are the groups.
    """
    base = cornell_box(width, height, spp, max_depth)
    positions, triangles, instances = [], [], []
    group_of_triangle = [0, 0, 1, 1, 2, 2, 3, 3, 4, 4]  # walls (floor, ceiling, back, left, right)
    group_of_triangle += [5 + f // 2 for f in range(12)]  # short box: 6 faces
    tall = [11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16]  # faces z0, z1, y0, y1, x0, x1
    tall = [t if t != 16 else 11 for t in tall]  # x1 face joins the z0 face's group
    group_of_triangle += [t for t in tall]
    # one instance per triangle of the groups, then the light
    rng = np.random.default_rng(seed)
    # world-space corners of every triangle (triangle indices are local to their instance)
    corners = []
    for inst in base.instances:
        for t in range(inst.triangle_count):
            corners.append(base.positions[inst.vertex_begin + base.triangles[inst.triangle_begin + t]])
    light_inst = base.instances[-1]
    for t in range(34):
        positions.append(corners[t])
        triangles.append(np.array([[0, 1, 2]], np.uint32))
        instances.append(identity_instance(3 * t, t, 1, group_of_triangle[t]))
    lv = np.concatenate(corners[34:36])
    positions.append(lv)
    triangles.append(np.array([[0, 1, 2], [3, 4, 5]], np.uint32))
    instances.append(identity_instance(3 * 34, 34, 2, 16, light_inst.emission))
    positions = np.concatenate(positions).astype(np.float32)
    triangles = np.concatenate(triangles)
    # rebase triangle vertex indices to instance-local ones
    w = np.linspace(360.0, 830.0, 32)

    def make(values_per_group):
        knots = np.concatenate([knots_from_curve(v) for v in values_per_group] + [knots_from_curve(0.0)])
        materials = [diffuse_material(32 * g) for g in range(17)]
        sc = Scene("cornell_groups", width, height, spp, positions.copy(), triangles.copy(), list(instances),
                   materials, knots, emissions=list(base.emissions), max_depth=max_depth)
        sc.camera = base.camera
        return sc

    truth_values = []
    for _ in range(16):
        anchors = rng.uniform(0.1, 0.9, 6)
        truth_values.append(np.interp(w, np.linspace(360, 830, 6), anchors))
    return make([np.full(32, start)] * 16), make(truth_values)


def view_batch(scene: Scene, count=64, seed=1, min_size=(256, 256), max_size=(1280, 720), spp=(4, 8, 16, 32, 64),
               target=(0.0, 0.35, 0.0), distance=(2.2, 4.0), vfov=40.0):
    """Seeded camera views of one scene for batched rendering: uniform resolutions between
    min_size and max_size, sample counts drawn from ``spp``, and poses on a sphere around
    ``target`` (distance range, elevation 5..45 degrees, any azimuth).  Returns a list of
    ``renderer.View`` with consecutive film offsets."""
    from . import renderer

    rng = np.random.default_rng(seed)
    views = []
    for _ in range(count):
        w = int(rng.integers(min_size[0], max_size[0] + 1))
        h = int(rng.integers(min_size[1], max_size[1] + 1))
        n = int(rng.choice(spp))
        r = float(rng.uniform(*distance))
        az = float(rng.uniform(0, 2 * math.pi))
        el = math.radians(float(rng.uniform(5, 45)))
        eye = (target[0] + r * math.cos(el) * math.sin(az), target[1] + r * math.sin(el),
               target[2] + r * math.cos(el) * math.cos(az))
        views.append(renderer.View(pinhole_camera(eye, target, (0, 1, 0), vfov, w, h), w, h, 0, n))
    renderer.pack_views(views)
    return views


def slab_scene(media, planes, camera_medium=abi.RP_NONE, environment=1.0, max_depth=1, materials=None,
               positional=None) -> Scene:
    """Analytic medium scenes in the style of rypath's medium tests (tests/medium_render_tests.cpp:24-85).

    A 1x1 film looks along +z from the origin through a nearly collimated camera; each plane is
    a 32x32 quad at z with its normal along +z (positive) or -z, bounding media through
    (inside, outside) medium ids, with material 0 the null interface unless given.
    """
    positions, triangles, instances = [], [], []
    mats = [abi.Material()]
    mats[0].scattering, mats[0].kind = abi.INTERFACE, abi.REFLECTANCE_CONSTANT
    for m in materials or []:
        mats.append(m)
    for plane in planes:
        z, positive = plane["z"], plane["positive"]
        inside, outside = plane.get("media", (abi.RP_NONE, abi.RP_NONE))
        v = np.array([[-16, -16, z], [16, -16, z], [16, 16, z], [-16, 16, z]], np.float32)
        t = np.array([[0, 1, 2], [0, 2, 3]] if positive else [[0, 2, 1], [0, 3, 2]], np.uint32)
        inst = identity_instance(sum(len(p) for p in positions), sum(len(x) for x in triangles), 2,
                                 plane.get("material", 0), plane.get("emission", abi.RP_NONE))
        inst.inside_medium, inst.outside_medium = inside, outside
        inst.reverse_orientation = int(plane.get("reverse", False))
        if "matrix" in plane:
            inst.matrix[:] = list(plane["matrix"])
        positions.append(v)
        triangles.append(t)
        instances.append(inst)
    scene = Scene("slab", 1, 1, 1, np.concatenate(positions) if positions else np.zeros((0, 3), np.float32),
                  np.concatenate(triangles) if triangles else np.zeros((0, 3), np.uint32), instances, mats,
                  environment=np.full(471, environment, np.float32), max_depth=max_depth)
    scene.camera = ((0.0, 0.0, 0.0), (-1e-7, -1e-7, 1.0), (2e-7, 0.0, 0.0), (0.0, 2e-7, 0.0))
    scene.media = media
    scene.camera_medium = camera_medium
    scene.positional = positional or []
    scene.transport = abi.TRANSPORT_SCALAR
    return scene


# ------------------------------------------------------------------ mixed-material scene
def icosphere(subdivisions: int):
    t = (1 + 5 ** 0.5) / 2
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t],
                  [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                  [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                  [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(subdivisions):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        edges.sort(axis=1)
        unique, inverse = np.unique(edges, axis=0, return_inverse=True)
        inverse = inverse.reshape(-1)
        mid = v[unique[:, 0]] + v[unique[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        n = len(f)
        a = base + inverse[:n]
        b = base + inverse[n:2 * n]
        c = base + inverse[2 * n:]
        f = np.concatenate([np.stack([f[:, 0], a, c], 1), np.stack([f[:, 1], b, a], 1),
                            np.stack([f[:, 2], c, b], 1), np.stack([a, b, c], 1)])
    return v, f


def uv_sphere(n_phi=32, n_theta=33):
    """Latitude-longitude sphere with 2*n_phi*(n_theta-1) triangles (2048 by default)."""
    verts = [[0, 0, 1]]
    for i in range(1, n_theta):
        th = math.pi * i / n_theta
        for j in range(n_phi):
            ph = 2 * math.pi * j / n_phi
            verts.append([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
    verts.append([0, 0, -1])
    verts = np.array(verts, np.float64)
    tris = []
    for j in range(n_phi):
        tris.append([0, 1 + j, 1 + (j + 1) % n_phi])
    for i in range(n_theta - 2):
        r0, r1 = 1 + i * n_phi, 1 + (i + 1) * n_phi
        for j in range(n_phi):
            j1 = (j + 1) % n_phi
            tris.append([r0 + j, r1 + j, r1 + j1])
            tris.append([r0 + j, r1 + j1, r0 + j1])
    last = len(verts) - 1
    r0 = 1 + (n_theta - 2) * n_phi
    for j in range(n_phi):
        tris.append([r0 + j, last, r0 + (j + 1) % n_phi])
    return verts, np.array(tris, np.int64)


def _smooth_random_curve(rng, lo, hi, count=32):
    """A smooth random spectrum: a few random Gaussian bumps, mapped into [lo, hi]."""
    w = np.linspace(0, 1, count)
    y = np.zeros(count)
    for _ in range(3):
        y += rng.uniform(-1, 1) * np.exp(-((w - rng.uniform(0, 1)) ** 2) / (2 * rng.uniform(0.05, 0.3) ** 2))
    y = (y - y.min()) / max(1e-6, y.max() - y.min())
    return lo + (hi - lo) * y


def mixed_scene(width=1920, height=1080, spp=16, max_depth=16, seed=1, subdivisions=8,
                sphere_count=64) -> Scene:
    rng = np.random.default_rng(seed)
    positions, triangles, instances, materials = [], [], [], []
    knots = []

    def add_knots(k):
        begin = sum(len(x) for x in knots)
        knots.append(np.asarray(k, np.float32))
        return begin

    def random_material():
        r = rng.uniform()
        if r < 0.4:
            return diffuse_material(add_knots(knots_from_curve(_smooth_random_curve(rng, 0.05, 0.9))))
        m = abi.Material()
        m.remap_roughness = 1
        if r < 0.8:
            m.scattering = abi.CONDUCTOR
            m.kind = abi.REFLECTANCE_CONSTANT
            m.scalar_value = 1.0
            m.eta_begin = add_knots(knots_from_curve(_smooth_random_curve(rng, 0.2, 1.8)))
            m.eta_count = 32
            m.k_begin = add_knots(knots_from_curve(_smooth_random_curve(rng, 2.0, 4.5)))
            m.k_count = 32
            m.optical_extensions = 3
            rough = rng.uniform(0.05, 0.5)
            m.u_roughness = m.v_roughness = rough
        else:
            m.scattering = abi.DIELECTRIC
            m.kind = abi.REFLECTANCE_CONSTANT
            m.scalar_value = 1.0
            w = np.linspace(360, 830, 32)
            cauchy = 1.5 + 0.004 / (w / 1000.0) ** 2
            m.eta_begin = add_knots(knots_from_curve(cauchy))
            m.eta_count = 32
            m.optical_extensions = 1
            m.k_begin = m.k_count = 0
            m.u_roughness = m.v_roughness = 0.0
        return m

    vb = tb = 0

    def add_mesh(v, f, material):
        nonlocal vb, tb
        positions.append(np.asarray(v, np.float32))
        triangles.append(np.asarray(f, np.uint32))
        materials.append(material)
        instances.append(identity_instance(vb, tb, len(f), len(materials) - 1))
        vb += len(v)
        tb += len(f)

    # displaced icosphere at the origin
    v, f = icosphere(subdivisions)
    d = np.zeros(len(v))
    for _ in range(6):
        k = rng.normal(size=3) * rng.uniform(2, 9)
        d += np.sin(v @ k + rng.uniform(0, 2 * math.pi))
    v = v * (1 + 0.02 * d / 6)[:, None]
    add_mesh(v, f, random_material())
    # random spheres around it, on a ring above the ground
    sv, sf = uv_sphere()
    for i in range(sphere_count):
        radius = rng.uniform(0.08, 0.3)
        ang = rng.uniform(0, 2 * math.pi)
        dist = rng.uniform(1.5, 4.0)
        center = np.array([dist * math.cos(ang), -1.0 + radius + rng.uniform(0, 1.2), dist * math.sin(ang)])
        add_mesh(sv * radius + center, sf, random_material())
    # ground plane
    g = 12.0
    add_mesh(np.array([[-g, -1, -g], [-g, -1, g], [g, -1, g], [g, -1, -g]]), np.array([[0, 1, 2], [0, 2, 3]]),
             diffuse_material(add_knots(knots_from_curve(0.5))))
    scene = Scene("mixed_material", width, height, spp, np.concatenate(positions), np.concatenate(triangles),
                  instances, materials, np.concatenate(knots), max_depth=max_depth)
    # 2 point + 2 spot lights with blackbody intensities
    def blackbody_intensity(kelvin, scale):
        return blackbody_emission(kelvin, scale)

    scene.positional = [
        {"kind": abi.POINT_LIGHT, "position": (3.0, 4.0, 3.0), "intensity": blackbody_intensity(3200, 60.0)},
        {"kind": abi.POINT_LIGHT, "position": (-4.0, 3.0, 1.0), "intensity": blackbody_intensity(5000, 40.0)},
        _spot((0.0, 5.0, 0.5), (0.0, 0.0, 0.0), 25.0, 30.0, blackbody_intensity(6500, 120.0)),
        _spot((-2.0, 3.0, 4.0), (0.0, -0.5, 0.0), 15.0, 20.0, blackbody_intensity(4000, 80.0)),
    ]
    scene.environment = (0.03 * blackbody_shape(9000) / blackbody_shape(9000).max()).astype(np.float32)
    scene.camera = pinhole_camera((0.0, 1.2, 5.5), (0.0, -0.1, 0.0), (0, 1, 0), 38.0, width, height)
    return scene


def _spot(position, target, start_deg, end_deg, intensity):
    """Spot light whose light_from_world maps the spot axis to +z (src/render.hpp:183-191)."""
    p = np.asarray(position, np.float64)
    z = np.asarray(target, np.float64) - p
    z /= np.linalg.norm(z)
    helper = np.array([1.0, 0, 0]) if abs(z[0]) < 0.9 else np.array([0, 1.0, 0])
    x = np.cross(helper, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    m = np.stack([x, y, z])  # rows: world -> light
    return {"kind": abi.SPOT_LIGHT, "position": tuple(p), "intensity": intensity,
            "light_from_world": tuple(m.reshape(-1)), "cos_falloff_start": math.cos(math.radians(start_deg)),
            "cos_falloff_end": math.cos(math.radians(end_deg))}
