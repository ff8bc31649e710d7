"""The reference's witness scenes and strategies, as SceneDescription / RenderStrategy dicts.

Transcribed from the reference's test fixtures (tests/witnesses/scenes/*.ts); each
matches one of the snapshot programs compiled into ``oracle/_ref`` so the CUDA path,
the oracle and the reference's own program can be compared on identical inputs.
"""

CORNELL_OBJECTS = [   # tests/witnesses/scenes/cornellBox.ts:6-53
    {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 0.0}, "material": "white"},
    {"type": "plane", "parameters": {"normal": [0, -1, 0], "offset": 2.0}, "material": "white"},
    {"type": "plane", "parameters": {"normal": [0, 0, 1], "offset": 2.0}, "material": "white"},
    {"type": "plane", "parameters": {"normal": [1, 0, 0], "offset": 1.5}, "material": "red"},
    {"type": "plane", "parameters": {"normal": [-1, 0, 0], "offset": 1.5}, "material": "green"},
    {"type": "plane", "parameters": {"normal": [0, 0, -1], "offset": 5.0}, "material": "white"},
    {"type": "box", "parameters": {"center": [-0.5, 0.6, -0.5], "halfSize": [0.3, 0.6, 0.3]}, "material": "white"},
    {"type": "sphere", "parameters": {"center": [0.5, 0.4, 0.3], "radius": 0.4}, "material": "clay"},
]
CEILING_QUAD = {"kind": "quad", "corner": [-0.5, 1.98, -0.5], "edge1": [1.0, 0.0, 0.0],
                "edge2": [0.0, 0.0, 1.0], "emission": 15.0}

# areaLightScenes.ts:23-36 (cornell-area) and :66-77 (cornell-area-glass)
CORNELL_AREA = {
    "id": "cornell-area", "ambientSpace": {"type": "euclidean"},
    "objects": CORNELL_OBJECTS,
    "materials": {
        "white": {"model": "lambert", "albedo": [0.73, 0.73, 0.73]},
        "red": {"model": "lambert", "albedo": [0.65, 0.05, 0.05]},
        "green": {"model": "lambert", "albedo": [0.12, 0.45, 0.15]},
        "clay": {"model": "lambert", "albedo": {"param": "clay.albedo", "default": [0.8, 0.4, 0.2]}},
    },
    "lights": [CEILING_QUAD],
}
CORNELL_AREA_GLASS = dict(CORNELL_AREA, id="cornell-area-glass",
                          objects=[dict(o, material="glass") if o["material"] == "clay" else o for o in CORNELL_OBJECTS],
                          materials={
                              "white": {"model": "lambert", "albedo": [0.73, 0.73, 0.73]},
                              "red": {"model": "lambert", "albedo": [0.65, 0.05, 0.05]},
                              "green": {"model": "lambert", "albedo": [0.12, 0.45, 0.15]},
                              "glass": {"model": "dielectric", "ior": 1.5},
                          })


def _area_strategy(sid, direct, bounces=10):
    return {"id": sid,
            "measurement": {"camera": {"type": "pinhole", "fov": {"param": "camera.fov", "default": 0.8}},
                            "maxBounces": bounces},
            "estimator": {"directLighting": direct, "russianRoulette": {"startDepth": 3},
                          "accumulation": {"type": "average"}},
            "view": {"tonemap": {"type": "reinhard"}}}


CORNELL_AREA_MIS = _area_strategy("pt-mis", "mis")
CORNELL_AREA_NEE = _area_strategy("pt-nee", "nee")
CORNELL_AREA_PT = _area_strategy("pt", "none")

# envScenes.ts:81-122 (furnace-sky)
FURNACE_SKY = {
    "id": "furnace-sky", "ambientSpace": {"type": "euclidean"},
    "objects": [{"type": "sphere", "parameters": {"center": [0, 0, 0], "radius": 1}, "material": "gray"}],
    "materials": {"gray": {"model": "lambert", "albedo": [0.4, 0.4, 0.4]}},
    "lights": [],
    "environment": {"type": "constant", "color": [1, 1, 1], "intensity": 1.0, "sampleAsLight": True},
}
FURNACE_SKY_MIS = {"id": "pt-mis",
                   "measurement": {"camera": {"type": "pinhole", "fov": {"param": "camera.fov", "default": 0.8}},
                                   "maxBounces": 32},
                   "estimator": {"directLighting": "mis", "russianRoulette": None, "accumulation": {"type": "average"}},
                   "view": {"tonemap": {"type": "none"}}}
FURNACE_SKY_NEE = dict(FURNACE_SKY_MIS, id="pt-nee",
                       estimator=dict(FURNACE_SKY_MIS["estimator"], directLighting="nee"))

# dielectricWitness.ts:14-56 (F-ETA)
ETA = {
    "id": "eta", "ambientSpace": {"type": "euclidean"},
    "objects": [
        {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 0.0}, "material": "water"},
        {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 1.0}, "material": "glow"},
    ],
    "materials": {"water": {"model": "dielectric", "ior": 1.33},
                  "glow": {"model": "lambert", "albedo": [0, 0, 0], "emission": [1.0, 1.0, 1.0]}},
    "lights": [],
}
ETA_STRATEGY = {"id": "pathtracer",
                "measurement": {"camera": {"type": "pinhole", "fov": 0.6, "position": [0, 1, 0.05], "target": [0, -1, 0]},
                                "maxBounces": 4},
                "estimator": {"directLighting": "none", "russianRoulette": None, "accumulation": {"type": "average"}},
                "view": {"tonemap": {"type": "reinhard"}}}

# mediaWitness.ts:22-57 (F-SLAB)
SLAB = {
    "id": "slab", "ambientSpace": {"type": "euclidean"},
    "objects": [
        {"type": "plane", "parameters": {"normal": [0, 0, 1], "offset": 2.0}, "material": "screen"},
        {"type": "box", "parameters": {"center": [0, 0, -0.5], "halfSize": [4, 4, 0.5]}, "material": "ink"},
    ],
    "materials": {"screen": {"model": "lambert", "albedo": [0, 0, 0], "emission": [1.0, 1.0, 1.0]},
                  "ink": {"model": "none", "medium": {"sigma_a": [1.0, 2.0, 4.0]}}},
    "lights": [],
}
SLAB_STRATEGY = {"id": "pathtracer",
                 "measurement": {"camera": {"type": "pinhole", "fov": 0.6}, "maxBounces": 4},
                 "estimator": {"directLighting": "none", "russianRoulette": None, "accumulation": {"type": "average"}},
                 "view": {"tonemap": {"type": "reinhard"}}}

# areaLightScenes.ts:95-126 (fog-area, X-FOG)
FOG_AREA = dict(CORNELL_AREA, id="fog-area",
                materials=dict(CORNELL_AREA["materials"],
                               haze={"model": "none", "medium": {"sigma_a": [0.05, 0.05, 0.05],
                                                                 "sigma_s": [0.4, 0.4, 0.4], "phase_g": 0.6}}),
                ambientMedium="haze")
FOG_AREA_MIS = _area_strategy("pt-mis", "mis", bounces=16)
FOG_AREA_NEE = _area_strategy("pt-nee", "nee", bounces=16)

# mediaWitness.ts:113-160 (haze)
HAZE = {
    "id": "haze", "ambientSpace": {"type": "euclidean"},
    "objects": [
        {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 0.0}, "material": "gray"},
        {"type": "plane", "parameters": {"normal": [0, -1, 0], "offset": 2.5}, "material": "gray"},
        {"type": "plane", "parameters": {"normal": [0, 0, 1], "offset": 2.5}, "material": "gray"},
        {"type": "plane", "parameters": {"normal": [1, 0, 0], "offset": 2.5}, "material": "gray"},
        {"type": "plane", "parameters": {"normal": [-1, 0, 0], "offset": 2.5}, "material": "gray"},
        {"type": "plane", "parameters": {"normal": [0, 0, -1], "offset": 6.0}, "material": "gray"},
        {"type": "box", "parameters": {"center": [-1.2, 1.2, -2.4], "halfSize": [0.4, 0.4, 0.05]}, "material": "panel"},
    ],
    "materials": {
        "gray": {"model": "lambert", "albedo": [0.5, 0.5, 0.5]},
        "panel": {"model": "lambert", "albedo": [0, 0, 0], "emission": [4.0, 4.0, 4.0]},
        "fog": {"model": "none", "medium": {"sigma_a": [0.02, 0.02, 0.02], "sigma_s": [0.4, 0.4, 0.4],
                                            "phase_g": {"param": "haze.g", "default": 0.7}}},
    },
    "lights": [{"kind": "point", "position": [0.8, 2.2, -1.0], "emission": 10}],
    "ambientMedium": "fog",
}
HAZE_NEE = {"id": "pt-nee",
            "measurement": {"camera": {"type": "pinhole", "fov": 0.9}, "maxBounces": 24},
            "estimator": {"directLighting": "nee", "russianRoulette": {"startDepth": 4},
                          "volumeSampling": "analytic", "accumulation": {"type": "average"}},
            "view": {"tonemap": {"type": "reinhard"}}}

# areaLightScenes.ts:177-230 (orb: sphere light through the sampleAsLight route)
ORB = {
    "id": "orb", "ambientSpace": {"type": "euclidean"},
    "objects": [
        {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 0.0}, "material": "ground"},
        {"type": "sphere", "parameters": {"center": [0.0, 1.6, 0.0], "radius": 0.25}, "material": "glow"},
        {"type": "box", "parameters": {"center": [-0.7, 0.4, 0.0], "halfSize": [0.35, 0.4, 0.35]}, "material": "slate"},
        {"type": "sphere", "parameters": {"center": [0.75, 0.45, 0.35], "radius": 0.45}, "material": "glass"},
    ],
    "materials": {
        "ground": {"model": "lambert", "albedo": [0.45, 0.44, 0.42]},
        "glow": {"model": "lambert", "albedo": [0, 0, 0], "emission": [22.0, 20.0, 17.0]},
        "slate": {"model": "lambert", "albedo": [0.25, 0.27, 0.3]},
        "glass": {"model": "dielectric", "ior": 1.5},
    },
    "lights": [],
    "environment": {"type": "constant", "color": [0.03, 0.035, 0.05], "intensity": 1.0},
}

ORB_NEE = {"id": "pt-nee",
           "measurement": {"camera": {"type": "pinhole", "fov": 0.8, "position": [0, 1.3, 3.4], "target": [0, 0.7, 0]},
                           "maxBounces": 12},
           "estimator": {"directLighting": "nee", "russianRoulette": {"startDepth": 3}, "accumulation": {"type": "average"}},
           "view": {"tonemap": {"type": "reinhard"}}}

# ggxScenes.ts:16-75 (veach-mis: GGX plates under three sphere lights)
VEACH = {
    "id": "veach-mis", "ambientSpace": {"type": "euclidean"},
    "objects": [
        {"type": "quad", "parameters": {"corner": [-1.8, 1.113, -0.54], "edge1": [0.0, -0.125, 0.38], "edge2": [3.6, 0.0, 0.0]}, "material": "plate1"},
        {"type": "quad", "parameters": {"corner": [-1.8, 0.769, 0.156], "edge1": [0.0, -0.099, 0.388], "edge2": [3.6, 0.0, 0.0]}, "material": "plate2"},
        {"type": "quad", "parameters": {"corner": [-1.8, 0.457, 0.853], "edge1": [0.0, -0.074, 0.393], "edge2": [3.6, 0.0, 0.0]}, "material": "plate3"},
        {"type": "quad", "parameters": {"corner": [-1.8, 0.173, 1.551], "edge1": [0.0, -0.047, 0.397], "edge2": [3.6, 0.0, 0.0]}, "material": "plate4"},
        {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 0.35}, "material": "floor"},
    ],
    "materials": {
        "plate1": {"model": "ggx", "f0": [0.95, 0.93, 0.88], "roughness": 0.1},
        "plate2": {"model": "ggx", "f0": [0.95, 0.93, 0.88], "roughness": 0.22},
        "plate3": {"model": "ggx", "f0": [0.95, 0.93, 0.88], "roughness": 0.38},
        "plate4": {"model": "ggx", "f0": [0.95, 0.93, 0.88], "roughness": 0.6},
        "floor": {"model": "lambert", "albedo": [0.18, 0.18, 0.2]},
    },
    "lights": [
        {"kind": "sphere", "position": [-1.15, 2.3, -1.9], "radius": 0.035, "emission": [150, 127.5, 105]},
        {"kind": "sphere", "position": [0.0, 2.3, -1.9], "radius": 0.14, "emission": [8.46, 9.4, 7.99]},
        {"kind": "sphere", "position": [1.15, 2.3, -1.9], "radius": 0.5, "emission": [0.592, 0.666, 0.74]},
    ],
    "environment": {"type": "constant", "color": [0.015, 0.015, 0.02], "intensity": 1.0},
}
VEACH_MIS = {"id": "pt-mis",
             "measurement": {"camera": {"type": "pinhole", "fov": 0.8, "position": [0, 1.3, 5.5], "target": [0, 0.55, 0]},
                             "maxBounces": 6},
             "estimator": {"directLighting": "mis", "russianRoulette": {"startDepth": 3}, "accumulation": {"type": "average"}},
             "view": {"tonemap": {"type": "reinhard"}}}

# twoLightScene.ts:17-80 (point lights under the power CDF)
TWO_LIGHT = {
    "id": "two-light", "ambientSpace": {"type": "euclidean"},
    "objects": [
        {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 0.0}, "material": "floor"},
        {"type": "plane", "parameters": {"normal": [0, 0, 1], "offset": 3.0}, "material": "floor"},
        {"type": "sphere", "parameters": {"center": [-0.75, 0.5, 0], "radius": 0.5}, "material": "ivory"},
        {"type": "sphere", "parameters": {"center": [0.75, 0.5, 0], "radius": 0.5}, "material": "ivory"},
    ],
    "materials": {"floor": {"model": "lambert", "albedo": [0.6, 0.6, 0.6]},
                  "ivory": {"model": "lambert", "albedo": [0.82, 0.78, 0.68]}},
    "lights": [{"kind": "point", "position": [-2.5, 3.0, 1.5], "emission": [26, 14.3, 6.5]},
               {"kind": "point", "position": [2.5, 2.5, 1.5], "emission": [4.9, 7.7, 14]}],
    "environment": {"type": "none"},
}
TWO_LIGHT_POWER = {"id": "power",
                   "measurement": {"camera": {"type": "pinhole", "fov": 0.9, "position": [0, 1.2, 4], "target": [0, 0.5, 0]},
                                   "maxBounces": 6},
                   "estimator": {"directLighting": "nee", "russianRoulette": None, "lightSelection": "power",
                                 "accumulation": {"type": "average"}},
                   "view": {"tonemap": {"type": "reinhard"}}}
HAZE_NEE["measurement"]["camera"].update({"position": [0, 1.2, 5], "target": [0, 1.2, -1]})

# (scene, strategy, snapshot program, camera parameters of that program)
CASES = {
    "cornell_area_glass_pt_mis": (CORNELL_AREA_GLASS, CORNELL_AREA_MIS),
    "cornell_area_glass_pt_nee": (CORNELL_AREA_GLASS, CORNELL_AREA_NEE),
    "cornell_area_glass_pt": (CORNELL_AREA_GLASS, CORNELL_AREA_PT),
    "cornell_area_pt_mis": (CORNELL_AREA, CORNELL_AREA_MIS),
    "furnace_sky_pt_mis": (FURNACE_SKY, FURNACE_SKY_MIS),
    "furnace_sky_pt_nee": (FURNACE_SKY, FURNACE_SKY_NEE),
    "eta_witness": (ETA, ETA_STRATEGY),
    "slab_witness": (SLAB, SLAB_STRATEGY),
    "fog_area_pt_mis": (FOG_AREA, FOG_AREA_MIS),
    "fog_area_pt_nee": (FOG_AREA, FOG_AREA_NEE),
    "veach_mis": (VEACH, VEACH_MIS),
    "orb_pt_nee": (ORB, ORB_NEE),
    "two_light_power": (TWO_LIGHT, TWO_LIGHT_POWER),
    "haze_pt_nee": (HAZE, HAZE_NEE),
}
