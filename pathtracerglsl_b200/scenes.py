"""Synthetic workloads, as SceneDescription / RenderStrategy dicts in the reference's shapes.

* ``cornell()``  — the Cornell box workload: interior [-1,1]x[0,2]x[-1,1] of five Lambert
  quads (front open), a 0.5x0.5 ceiling area light at y=1.99 with radiance 15, a Lambert
  sphere and a smooth dielectric sphere (IOR 1.5); pinhole at (0,1,4) -> (0,1,0), vertical
  fov 40 degrees; 256x256, 64 spp, max depth 8, roulette from depth 3, MIS.
* ``furnace()``  — the open furnace: a Lambert sphere of albedo 0.8 in a unit white
  environment (expected radiance 0.8 on the sphere, 1.0 on the sky).
"""
import math


def _quad(corner, e1, e2, material):
    return {"type": "quad", "parameters": {"corner": corner, "edge1": e1, "edge2": e2}, "material": material}


def cornell(direct="mis", max_depth=8, rr_start=3):
    scene = {
        "id": "cornell-c1",
        "ambientSpace": {"type": "euclidean"},
        "objects": [
            # edges ordered so cross(edge1, edge2) points into the box
            _quad([-1, 0, 1], [2, 0, 0], [0, 0, -2], "white"),    # floor, +y
            _quad([-1, 2, -1], [2, 0, 0], [0, 0, 2], "white"),    # ceiling, -y
            _quad([-1, 0, -1], [2, 0, 0], [0, 2, 0], "white"),    # back, +z
            _quad([-1, 0, 1], [0, 0, -2], [0, 2, 0], "red"),      # left, +x
            _quad([1, 0, -1], [0, 0, 2], [0, 2, 0], "green"),     # right, -x
            {"type": "sphere", "parameters": {"center": [-0.4, 0.3, -0.3], "radius": 0.3}, "material": "matte"},
            {"type": "sphere", "parameters": {"center": [0.4, 0.3, 0.3], "radius": 0.3}, "material": "glass"},
        ],
        "materials": {
            "white": {"model": "lambert", "albedo": [0.75, 0.75, 0.75]},
            "red": {"model": "lambert", "albedo": [0.75, 0.25, 0.25]},
            "green": {"model": "lambert", "albedo": [0.25, 0.75, 0.25]},
            "matte": {"model": "lambert", "albedo": [0.75, 0.75, 0.75]},
            "glass": {"model": "dielectric", "ior": 1.5},
        },
        # cross(edge1, edge2) = -y: the panel emits downward (one-sided quad light)
        "lights": [{"kind": "quad", "corner": [-0.25, 1.99, -0.25], "edge1": [0.5, 0, 0],
                    "edge2": [0, 0, 0.5], "emission": 15.0}],
    }
    strategy = {
        "id": "pt-" + direct if direct != "none" else "pt",
        "measurement": {"camera": {"type": "pinhole", "fov": math.radians(40.0),
                                   "position": [0, 1, 4], "target": [0, 1, 0]},
                        "maxBounces": max_depth},
        "estimator": {"directLighting": direct,
                      "russianRoulette": {"startDepth": rr_start} if rr_start is not None else None,
                      "accumulation": {"type": "average"}},
        "view": {"tonemap": {"type": "none"}},
    }
    return scene, strategy


CORNELL_SIZE = (256, 256, 64)   # width, height, spp


def cornell_rough(direct="mis", roughness=0.3, max_depth=8, rr_start=3):
    """The Cornell box with the remaining surface occupants: the glass sphere a rough
    dielectric (IOR 1.5, tinted), the matte sphere a mirror (Schlick F0)."""
    scene, strategy = cornell(direct, max_depth, rr_start)
    scene = dict(scene, id="cornell-rough")
    scene["materials"] = dict(scene["materials"],
                              matte={"model": "mirror", "f0": [0.95, 0.85, 0.6]},
                              glass={"model": "rough_dielectric", "ior": 1.5, "roughness": roughness,
                                     "transmittance": [1.0, 0.95, 0.9]})
    return scene, strategy


def cornell_mesh_light(direct="mis", emitter="panel", max_depth=8, rr_start=3):
    """The Cornell box lit by an emissive mesh object in place of the authored quad light
    (the mesh light's one route: an emissive Lambert material on a mesh object).
    ``panel``: the same 0.5x0.5 ceiling panel (radiance 15, emitting downward), fanned into
    four triangles of unequal area around an off-centre point, so the image equals the
    quad-lit box's; ``sphere``: an outward-wound level-2 icosphere (320 triangles) of
    radius 0.15 under the ceiling, radiance 6."""
    scene, strategy = cornell(direct, max_depth, rr_start)
    scene = dict(scene, id="cornell-mesh-" + emitter, lights=[])
    if emitter == "panel":
        y = 1.99
        pos = [[0.1, y, -0.05], [-0.25, y, -0.25], [0.25, y, -0.25], [0.25, y, 0.25], [-0.25, y, 0.25]]
        # (centre, corner i, corner i+1): cross(b - a, c - a) points down (-y)
        idx = [[0, 1, 2], [0, 2, 3], [0, 3, 4], [0, 4, 1]]
        obj = {"kind": "mesh", "positions": pos, "indices": idx, "material": "lamp", "closed": False}
        lamp = {"model": "lambert", "albedo": [0.0, 0.0, 0.0], "emission": 15.0}
    else:
        v, f = icosphere(2)
        v = v * 0.15 + _np.array([0.0, 1.6, 0.0])
        obj = {"kind": "mesh", "positions": v.tolist(), "indices": f.tolist(), "material": "lamp", "closed": True}
        lamp = {"model": "lambert", "albedo": [0.0, 0.0, 0.0], "emission": 6.0}
    scene["objects"] = list(scene["objects"]) + [obj]
    scene["materials"] = dict(scene["materials"], lamp=lamp)
    return scene, strategy


def many_lights(direct="mis", selection="bvh", n=64, seed=0, fog=False, max_depth=6, rr_start=3):
    """The Cornell walls lit by many small lamps: ``n`` emissive instanced spheres in two
    batches (warm and cool, radii U(0.02, 0.05) in the upper half; under
    lightSelection 'bvh' every instance is a light of the tree), the ceiling quad light at
    radiance 5 and a fanned mesh panel; a GGX sphere and a rough glass sphere below.
    ``fog`` fills the box with a thin scattering medium (medium events query the tree
    without a normal)."""
    scene, strategy = cornell(direct, max_depth, rr_start)
    rng = _np.random.RandomState(seed)
    objects = list(scene["objects"][:5])
    objects.append({"type": "sphere", "parameters": {"center": [-0.4, 0.3, -0.3], "radius": 0.3}, "material": "metal"})
    objects.append({"type": "sphere", "parameters": {"center": [0.4, 0.3, 0.3], "radius": 0.3}, "material": "frost"})
    materials = dict(scene["materials"],
                     metal={"model": "ggx", "f0": [0.9, 0.8, 0.6], "roughness": 0.4},
                     frost={"model": "rough_dielectric", "ior": 1.5, "roughness": 0.3})
    for b, (col, le) in enumerate((([1.0, 0.6, 0.3], 40.0), ([0.3, 0.6, 1.0], 25.0))):
        pl = [{"position": [float(rng.uniform(-0.9, 0.9)), float(rng.uniform(0.8, 1.9)), float(rng.uniform(-0.9, 0.6))],
               "scale": float(rng.uniform(0.02, 0.05))} for _ in range(n // 2)]
        objects.append({"kind": "instanced", "placements": pl,
                        "prototype": {"type": "sphere", "parameters": {"center": [0, 0, 0], "radius": 1.0},
                                      "material": f"lamp{b}"}})
        materials[f"lamp{b}"] = {"model": "lambert", "albedo": [0.0, 0.0, 0.0], "emission": [le * c for c in col]}
    y = 1.98
    objects.append({"kind": "mesh", "material": "panel", "closed": False,
                    "positions": [[0.55, y, 0.45], [0.3, y, 0.3], [0.8, y, 0.3], [0.8, y, 0.6], [0.3, y, 0.6]],
                    "indices": [[0, 1, 2], [0, 2, 3], [0, 3, 4], [0, 4, 1]]})
    materials["panel"] = {"model": "lambert", "albedo": [0.0, 0.0, 0.0], "emission": [4.0, 8.0, 4.0]}
    lights = [dict(scene["lights"][0], emission=5.0)]
    scene = dict(scene, id=f"many-lights-{n}", objects=objects, materials=materials, lights=lights)
    if fog:
        scene["materials"]["fog"] = {"model": "none", "medium": {"sigma_a": [0.02, 0.02, 0.02],
                                                                 "sigma_s": [0.15, 0.15, 0.15], "phase_g": 0.3}}
        scene["ambientMedium"] = "fog"
    strategy = dict(strategy, id=strategy["id"] + "-" + selection,
                    estimator=dict(strategy["estimator"], lightSelection=selection))
    return scene, strategy


def het_fog(direct="nee", kind="ground", max_depth=12, rr_start=4):
    """Heterogeneous media in the Cornell walls (the reference's groundfog and fogblobs
    demos, as closed rooms):
    ``ground``: ambient ground fog sigma_s(p) = gain exp(-falloff y)(0.6 + 0.4 sin 4x sin 4z),
    gain 1.2, falloff 1.5, majorant 2.0 (delta tracking, ratio-tracked shadows);
    ``blobs``: two merging coloured Gaussian puffs inside a null-interface sphere, majorant 6
    (the field exceeds it at the puff centres: the clamped, rendered medium);
    ``absorb``: an absorbing-only field sigma_a(p) = 0.8 (1 + sin 3x) / 2 + 0.1 filling the
    room (the ratio-tracked pass-through).
    The ceiling quad light and a point light light the room."""
    scene, strategy = cornell(direct, max_depth, rr_start)
    objects = list(scene["objects"][:5]) + [
        {"type": "sphere", "parameters": {"center": [0.5, 0.3, 0.2], "radius": 0.3}, "material": "matte"}]
    materials = {k: scene["materials"][k] for k in ("white", "red", "green", "matte")}
    lights = [dict(scene["lights"][0], emission=12.0), {"kind": "point", "position": [-0.5, 1.5, 0.4], "emission": 1.5}]
    scene = dict(scene, id="het-" + kind, objects=objects, materials=materials, lights=lights)
    if kind == "ground":
        materials["fog"] = {"model": "none", "medium": {
            "sigma_a": [0.02, 0.02, 0.02],
            "sigma_s": {"kind": "glsl", "source": "u_fog_gain * exp(-u_fog_falloff * p.y) * (0.6 + 0.4 * sin(4.0 * p.x) * sin(4.0 * p.z))",
                        "params": [{"param": "fog.gain", "default": 1.2}, {"param": "fog.falloff", "default": 1.5}]},
            "majorant": 2.0, "phase_g": 0.3}}
        scene["ambientMedium"] = "fog"
    elif kind == "blobs":
        src = ("vec3(1.0, 0.7, 0.4) * u_blob_gain * (exp(-u_blob_sharp * dot(p - vec3(-0.25, 1.1, -0.2), p - vec3(-0.25, 1.1, -0.2)))"
               " + exp(-u_blob_sharp * dot(p - vec3(0.2, 0.9, -0.2), p - vec3(0.2, 0.9, -0.2))))")
        materials["puff"] = {"model": "none", "medium": {
            "sigma_a": [0.05, 0.05, 0.05],
            "sigma_s": {"kind": "glsl", "source": src,
                        "params": [{"param": "blob.gain", "default": 6.0}, {"param": "blob.sharp", "default": 14.0}]},
            "majorant": 6.0, "phase_g": 0.2}}
        objects.append({"type": "sphere", "parameters": {"center": [0.0, 1.0, -0.2], "radius": 0.65}, "material": "puff"})
    else:
        materials["smoke"] = {"model": "none", "medium": {
            "sigma_a": {"kind": "glsl", "source": "0.8 * (1.0 + sin(3.0 * p.x)) * 0.5 + 0.1"}, "majorant": 1.0}}
        scene["ambientMedium"] = "smoke"
    strategy = dict(strategy, estimator=dict(strategy["estimator"], volumeSampling="delta-tracking"))
    return scene, strategy


def furnace(direct="mis", max_depth=8):
    scene = {
        "id": "furnace-c1",
        "ambientSpace": {"type": "euclidean"},
        "objects": [{"type": "sphere", "parameters": {"center": [0, 0, 0], "radius": 1.0}, "material": "gray"}],
        "materials": {"gray": {"model": "lambert", "albedo": [0.8, 0.8, 0.8]}},
        "lights": [],
        "environment": {"type": "constant", "color": [1, 1, 1], "intensity": 1.0, "sampleAsLight": True},
    }
    strategy = {
        "id": "pt-" + direct if direct != "none" else "pt",
        "measurement": {"camera": {"type": "pinhole", "fov": math.radians(40.0),
                                   "position": [0, 0, 4], "target": [0, 0, 0]},
                        "maxBounces": max_depth},
        "estimator": {"directLighting": direct, "russianRoulette": None, "accumulation": {"type": "average"}},
        "view": {"tonemap": {"type": "none"}},
    }
    return scene, strategy


# ---------------------------------------------------------------------------------- meshes
import numpy as _np


def icosphere(level):
    """Subdivided icosahedron on the unit sphere: 20*4^level triangles, 10*4^level+2 vertices."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = _np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                   [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], _np.float64)
    f = _np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                   [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                   [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], _np.int64)
    v /= _np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        nv = len(v)
        edges = _np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = _np.minimum(edges[:, 0], edges[:, 1]) * nv + _np.maximum(edges[:, 0], edges[:, 1])
        uniq, inv = _np.unique(key, return_inverse=True)
        a, b = uniq // nv, uniq % nv
        mid = v[a] + v[b]
        mid /= _np.linalg.norm(mid, axis=1, keepdims=True)
        v = _np.concatenate([v, mid])
        m = inv.reshape(3, -1).T + nv          # midpoints of (01, 12, 20)
        f = _np.concatenate([_np.stack([f[:, 0], m[:, 0], m[:, 2]], 1), _np.stack([f[:, 1], m[:, 1], m[:, 0]], 1),
                             _np.stack([f[:, 2], m[:, 2], m[:, 1]], 1), m])
    return v, f


def _hash3(ix, iy, iz, seed):
    h = (ix.astype(_np.uint32) * _np.uint32(73856093)) ^ (iy.astype(_np.uint32) * _np.uint32(19349663)) \
        ^ (iz.astype(_np.uint32) * _np.uint32(83492791)) ^ _np.uint32(seed * 2654435761 & 0xFFFFFFFF)
    h = h ^ (h >> _np.uint32(13))
    h = h * _np.uint32(1274126177)
    h = h ^ (h >> _np.uint32(16))
    return (h & _np.uint32(0xFFFFFF)).astype(_np.float64) / float(1 << 24)


def value_noise(p, seed, freq=4.0):
    """Seeded 3D value noise in [-1, 1]: hashed lattice values, smoothstep-trilinear."""
    q = p * freq
    i0 = _np.floor(q).astype(_np.int64)
    fq = q - i0
    w = fq * fq * (3.0 - 2.0 * fq)
    out = _np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                h = _hash3(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz, seed)
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out += wx * wy * wz * h
    return 2.0 * out - 1.0


def sky_table(width=1024, height=512, seed=0, sun_radiance=5.0e3, sun_diameter_deg=0.5):
    """Procedural equirect sky (row 0 = +Y pole): a zenith-to-horizon gradient, a dark
    ground half, and a seeded sun disc of the given radiance and angular diameter."""
    rng = _np.random.RandomState(seed)
    j = (_np.arange(height) + 0.5) / height
    i = (_np.arange(width) + 0.5) / width
    theta = _np.pi * j[:, None] * _np.ones((1, width))
    phi = (i[None, :] - 0.5) * 2.0 * _np.pi * _np.ones((height, 1))
    d = _np.stack([_np.cos(phi) * _np.sin(theta), _np.cos(theta), _np.sin(phi) * _np.sin(theta)], -1)
    up = _np.clip(d[..., 1], 0.0, 1.0)
    zen = _np.array([0.25, 0.45, 0.95])
    hor = _np.array([0.9, 0.95, 1.0])
    sky = hor[None, None, :] * (1 - up[..., None]) ** 2 + zen[None, None, :] * (1 - (1 - up[..., None]) ** 2)
    ground = _np.array([0.08, 0.07, 0.06])
    table = _np.where(d[..., 1:2] >= 0.0, sky, ground[None, None, :] * _np.ones_like(sky))
    sun_el = rng.uniform(0.35, 1.0)
    sun_az = rng.uniform(0, 2 * _np.pi)
    sd = _np.array([_np.cos(sun_az) * _np.cos(sun_el), _np.sin(sun_el), _np.sin(sun_az) * _np.cos(sun_el)])
    cosang = d @ sd
    half = _np.radians(sun_diameter_deg) / 2.0
    table = table + (cosang >= _np.cos(half))[..., None] * sun_radiance * _np.array([1.0, 0.95, 0.85])
    return table.astype(_np.float32), sd


def mesh_scene(level=8, instances=16, seed=0, width=1920, height=1080, spp=256, max_depth=12,
               env_size=(1024, 512), direct="mis", accel="cwbvh"):
    """The mesh workload: a noise-displaced level-`level` icosphere (GGX conductor,
    F0 (0.9, 0.6, 0.3), per-triangle alpha ~ U(0.05, 0.5)) instanced `instances` times
    by seeded similarities over a Lambert ground plane (albedo 0.5), lit by a procedural
    equirect sky with a sun lobe of radiance 5e3 over 0.5 degrees."""
    rng = _np.random.RandomState(seed)
    v, f = icosphere(level)
    v = v * (1.0 + 0.05 * value_noise(v, seed))[:, None]
    alpha = rng.uniform(0.05, 0.5, len(f)).astype(_np.float32)
    placements = []
    cells = _np.arange(instances)
    grid = int(_np.ceil(_np.sqrt(instances)))
    for k in cells:
        gx, gz = k % grid, k // grid
        s = float(rng.uniform(0.5, 1.1))
        x = (gx - (grid - 1) / 2.0) * 2.6 + float(rng.uniform(-0.3, 0.3))
        z = (gz - (grid - 1) / 2.0) * 2.6 + float(rng.uniform(-0.3, 0.3))
        axis = rng.normal(size=3)
        placements.append({"position": [x, s * 1.05, z], "scale": s,
                           "rotation": {"axis": list(axis / _np.linalg.norm(axis)), "angle": float(rng.uniform(0, 6.28))}})
    table, sun = sky_table(env_size[0], env_size[1], seed)
    scene = {
        "id": "mesh-c2",
        "ambientSpace": {"type": "euclidean"},
        "objects": [
            {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 0.0}, "material": "ground"},
            {"kind": "instanced",
             "prototype": {"kind": "mesh", "positions": v.astype(_np.float32).reshape(-1),
                           "indices": f.astype(_np.uint32).reshape(-1), "material": "metal",
                           "triangleAlpha": alpha},
             "placements": placements},
        ],
        "materials": {"ground": {"model": "lambert", "albedo": [0.5, 0.5, 0.5]},
                      "metal": {"model": "ggx", "f0": [0.9, 0.6, 0.3], "roughness": 0.5}},
        "lights": [],
        "environment": {"type": "image", "table": table, "intensity": 1.0, "sampleAsLight": True},
    }
    extent = grid * 1.3
    strategy = {
        "id": "pt-" + direct,
        "measurement": {"camera": {"type": "pinhole", "fov": math.radians(45.0),
                                   "position": [0.0, extent * 1.1, extent * 2.2], "target": [0.0, 0.6, 0.0]},
                        "maxBounces": max_depth},
        "estimator": {"directLighting": direct, "russianRoulette": {"startDepth": 3},
                      "meshTraversal": accel, "accumulation": {"type": "average"}},
        "view": {"tonemap": {"type": "none"}},
    }
    return scene, strategy, (width, height, spp)


# ------------------------------------------------------------------------- scene batches
def batch_scene(seed, max_spheres=200):
    """One seeded Cornell-style scene of the batched workload: the Cornell box's five
    walls and ceiling light with 1..`max_spheres` non-overlapping spheres of radius
    U(0.05, 0.3) inside it (count log-uniform), each with a material drawn uniformly from
    Lambert (albedo U(0.2, 0.9) per channel), smooth dielectric (IOR U(1.3, 1.8)) and GGX
    (alpha U(0.05, 0.6), F0 = albedo); resolution 128..1024 squared (log-uniform, a
    multiple of 16), spp 16..256 (a power of two) and max depth 4..32.
    Returns (scene, strategy, (width, height, spp))."""
    rng = _np.random.RandomState(1000 + seed)
    base, strategy = cornell()
    objects = list(base["objects"][:5])
    materials = {k: base["materials"][k] for k in ("white", "red", "green")}
    n = int(round(math.exp(rng.uniform(0.0, math.log(max_spheres)))))
    n = max(1, min(max_spheres, n))
    placed = []
    for k in range(n):
        r = float(rng.uniform(0.05, 0.3))
        for _attempt in range(200):
            c = _np.array([rng.uniform(-1 + r, 1 - r), rng.uniform(r, 1.9 - r), rng.uniform(-1 + r, 1 - r)])
            if all(_np.linalg.norm(c - pc) > r + pr + 1e-3 for pc, pr in placed):
                break
            if _attempt % 20 == 19:
                r = max(0.02, r * 0.8)
        else:
            continue
        placed.append((c, r))
        kind = int(rng.randint(3))
        name = f"s{k}"
        if kind == 0:
            materials[name] = {"model": "lambert", "albedo": [float(a) for a in rng.uniform(0.2, 0.9, 3)]}
        elif kind == 1:
            materials[name] = {"model": "dielectric", "ior": float(rng.uniform(1.3, 1.8))}
        else:
            alpha = float(rng.uniform(0.05, 0.6))
            materials[name] = {"model": "ggx", "f0": [float(a) for a in rng.uniform(0.2, 0.9, 3)],
                               "roughness": math.sqrt(alpha)}
        objects.append({"type": "sphere", "parameters": {"center": [float(x) for x in c], "radius": r},
                        "material": name})
    scene = dict(base, id=f"batch-{seed}", objects=objects, materials=materials)
    res = int(round(math.exp(rng.uniform(math.log(128), math.log(1024))) / 16.0)) * 16
    spp = int(2 ** rng.randint(4, 9))
    depth = int(rng.randint(4, 33))
    strategy = dict(strategy, id=f"batch-{seed}-pt-mis",
                    measurement=dict(strategy["measurement"], maxBounces=depth))
    return scene, strategy, (res, res, spp)


BATCH_SIZE = 64


def batch_scenes(n=BATCH_SIZE, seed=0, max_spheres=200):
    """The batched workload: `n` seeded Cornell-style scenes (``batch_scene``)."""
    return [batch_scene(seed * 100003 + k, max_spheres) for k in range(n)]


# ------------------------------------------------------------------------- adjoint workload
def adjoint_box_scene():
    """The adjoint's check scene: the Cornell box without roulette, with a Lambert sphere,
    a GGX sphere and a grey scattering medium behind a null interface."""
    sc, st = cornell(direct="mis", rr_start=None)
    sc = dict(sc)
    sc["objects"] = list(sc["objects"][:5]) + [
        {"type": "sphere", "parameters": {"center": [-0.45, 0.35, -0.3], "radius": 0.35}, "material": "matte"},
        {"type": "sphere", "parameters": {"center": [0.45, 0.3, 0.2], "radius": 0.3}, "material": "metal"},
        {"type": "sphere", "parameters": {"center": [0.0, 1.1, -0.3], "radius": 0.3}, "material": "fog"},
    ]
    sc["materials"] = dict(sc["materials"], matte={"model": "lambert", "albedo": [0.7, 0.5, 0.3]},
                           metal={"model": "ggx", "f0": [0.9, 0.6, 0.3], "roughness": 0.5},
                           fog={"model": "none", "medium": {"sigma_a": [0.3] * 3, "sigma_s": [1.7] * 3,
                                                            "phase_g": 0.5}})
    return sc, st


def adjoint_scene(seed=0, n_spheres=64, width=256, height=256, spp_primal=64, spp_adjoint=16, max_depth=8):
    """The inverse-rendering workload: the Cornell box's walls and ceiling light with
    `n_spheres` seeded non-overlapping spheres of radius U(0.06, 0.16), each with its own
    material drawn uniformly from Lambert (albedo U(0.2, 0.9) per channel), GGX (alpha
    U(0.05, 0.6), F0 (0.9, 0.6, 0.3)) and smooth dielectric (IOR U(1.3, 1.8)), plus one
    sphere of radius 0.3 holding a grey homogeneous medium behind a null interface
    (sigma_t 2.0, single-scattering albedo 0.9, HG g 0.6).  MIS, no roulette, max depth 8.
    Returns (scene, strategy, (width, height, spp_primal, spp_adjoint))."""
    rng = _np.random.RandomState(7000 + seed)
    base, strategy = cornell(rr_start=None, max_depth=max_depth)
    objects = list(base["objects"][:5])
    materials = {k: base["materials"][k] for k in ("white", "red", "green")}
    fog_c, fog_r = _np.array([0.0, 1.0, -0.2]), 0.3
    placed = [(fog_c, fog_r)]
    k = 0
    while k < n_spheres:
        r = float(rng.uniform(0.06, 0.16))
        c = _np.array([rng.uniform(-1 + r, 1 - r), rng.uniform(r, 1.9 - r), rng.uniform(-1 + r, 1 - r)])
        if not all(_np.linalg.norm(c - pc) > r + pr + 1e-3 for pc, pr in placed):
            continue
        placed.append((c, r))
        kind = int(rng.randint(3))
        name = f"s{k}"
        if kind == 0:
            materials[name] = {"model": "lambert", "albedo": [float(a) for a in rng.uniform(0.2, 0.9, 3)]}
        elif kind == 1:
            alpha = float(rng.uniform(0.05, 0.6))
            materials[name] = {"model": "ggx", "f0": [0.9, 0.6, 0.3], "roughness": math.sqrt(alpha)}
        else:
            materials[name] = {"model": "dielectric", "ior": float(rng.uniform(1.3, 1.8))}
        objects.append({"type": "sphere", "parameters": {"center": [float(x) for x in c], "radius": r},
                        "material": name})
        k += 1
    materials["fog"] = {"model": "none", "medium": {"sigma_a": [0.2, 0.2, 0.2], "sigma_s": [1.8, 1.8, 1.8],
                                                    "phase_g": 0.6}}
    objects.append({"type": "sphere", "parameters": {"center": [float(x) for x in fog_c], "radius": fog_r},
                    "material": "fog"})
    scene = dict(base, id=f"adjoint-{seed}", objects=objects, materials=materials)
    strategy = dict(strategy, id="adjoint-pt-mis")
    return scene, strategy, (width, height, spp_primal, spp_adjoint)


# ------------------------------------------------------------------------- media + spectral workload
def media_scene(width=1024, height=1024, spp=512, max_depth=64, spectral=True, lambda_range=(380.0, 780.0)):
    """The media and spectral workload: a sphere of radius 1 with a dielectric boundary
    (IOR 1.33) holding a chromatic homogeneous medium (sigma_t (0.5, 1.0, 2.0), single-scattering
    albedo 0.9, HG g 0.6); a second sphere of radius 1 behind a null interface holding a grey
    medium of sigma_t 2.0 (albedo 0.9, isotropic); a Lambert ground plane (albedo 0.5); lit by a
    spherical light of radius 0.05 emitting a 3000 K blackbody spectrum and a 1 x 1 quad light
    of radiance 20; NEE with equiangular placement in the media (the area-light extension),
    roulette from depth 3, max depth 64; spectral with four hero wavelengths over 380-780 nm.
    Returns (scene, strategy, (width, height, spp))."""
    st_rgb = [0.5, 1.0, 2.0]
    scene = {
        "id": "media-c3",
        "objects": [
            {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 0.0}, "material": "ground"},
            {"type": "sphere", "parameters": {"center": [-1.15, 1.0, 0.0], "radius": 1.0}, "material": "glass_medium"},
            {"type": "sphere", "parameters": {"center": [1.15, 1.0, 0.0], "radius": 1.0}, "material": "grey_fog"},
        ],
        "materials": {
            "ground": {"model": "lambert", "albedo": [0.5, 0.5, 0.5]},
            "glass_medium": {"model": "dielectric", "ior": 1.33,
                             "medium": {"sigma_a": [0.1 * v for v in st_rgb], "sigma_s": [0.9 * v for v in st_rgb],
                                        "phase_g": 0.6}},
            "grey_fog": {"model": "none", "medium": {"sigma_a": [0.2] * 3, "sigma_s": [1.8] * 3, "phase_g": 0.0}},
        },
        "lights": [
            {"kind": "sphere", "position": [0.0, 2.4, 1.2], "radius": 0.05,
             "emission": {"blackbody": {"kelvin": 3000.0, "scale": 400.0}}},
            # cross(edge1, edge2) = -y: the 1 x 1 panel emits downward
            {"kind": "quad", "corner": [-0.5, 3.5, -0.5], "edge1": [1.0, 0.0, 0.0], "edge2": [0.0, 0.0, 1.0],
             "emission": 20.0},
        ],
    }
    meas = {"camera": {"type": "pinhole", "fov": math.radians(45.0), "position": [0.0, 1.4, 5.5],
                       "target": [0.0, 0.9, 0.0]},
            "maxBounces": max_depth}
    if spectral:
        meas["color"] = "spectral"
        meas["wavelengthRange"] = list(lambda_range)
    strategy = {"id": "pt-nee-eq", "measurement": meas,
                "estimator": {"directLighting": "nee", "russianRoulette": {"startDepth": 3},
                              "volumeSampling": "analytic", "mediumLightSampling": "equiangular",
                              "equiangularAreaLights": True, "wavelengths": "visible"},
                "view": {"tonemap": {"type": "none"}}}
    return scene, strategy, (width, height, spp)
