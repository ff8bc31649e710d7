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
