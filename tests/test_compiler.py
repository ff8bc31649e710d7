"""The host compiler: validation diagnostics and packing (Validator / Planner mirror)."""
import pytest

import ref_scenes
from pathtracerglsl_b200 import abi, scenes
from pathtracerglsl_b200.compiler import CompileError, Compiler


def test_cornell_packs_regions_materials_and_light():
    sc, st = scenes.cornell()
    r, pk = Compiler().compile(sc, st)
    assert len(pk.regions) == 8              # 5 walls + 2 spheres + the desugared light quad
    assert len(pk.lights) == 1
    assert r.program.direct == abi.DIRECT_MIS
    assert r.program.max_bounces == 8 and r.program.rr_start == 3


def test_material_order_and_synthesized_light_material():
    # reference order: authored materials in declaration order, then light materials
    r, pk = Compiler().compile(ref_scenes.FOG_AREA, ref_scenes.FOG_AREA_MIS)
    assert pk.material_names == ["white", "red", "green", "clay", "haze"]
    assert len(pk.materials) == 6
    assert pk.ambient_material == 4


def test_unknown_material_model_is_an_error():
    sc, st = scenes.cornell()
    sc = dict(sc, materials=dict(sc["materials"], white={"model": "velvet"}))
    with pytest.raises(CompileError) as e:
        Compiler().compile(sc, st)
    assert any(d.code == "unknown-model" for d in e.value.diagnostics)


def test_equiangular_pins_like_the_reference_validator():
    sc, st = scenes.cornell()
    st = dict(st, estimator=dict(st["estimator"], mediumLightSampling="equiangular"))
    with pytest.raises(CompileError) as e:
        Compiler().compile(sc, st)
    codes = [d.code for d in e.value.diagnostics]
    assert "invalid-setting" in codes


def test_negative_max_bounces_rejected():
    sc, st = scenes.cornell()
    st = dict(st, measurement=dict(st["measurement"], maxBounces=-1))
    with pytest.raises(CompileError):
        Compiler().compile(sc, st)
