"""Host-side scene handling of the CUDA library (no GPU needed): the JSON
loader, light list and CDF built by lucid_cuda_inspect_scene must equal the
CPU oracle's restatement of loadSceneFromJsonString + SceneLights bit for
bit, and malformed scenes must be rejected with an error status."""
import json

import numpy as np
import pytest

import lucid_capi
import lucid_scenes as ls
from oracle_ctypes import Oracle

SCENES = {
    "cornell": lambda wd: ls.cornell_box(),
    "all_lights": lambda wd: ls.all_lights_scene(workdir=wd),
    "mirror": lambda wd: ls.mirror_point_light_scene(),
    "procedural_small": lambda wd: ls.procedural_scene(seed=5, n_spheres=6, levels=2, emissive_levels=1,
                                                       workdir=wd, extent=6.0),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_lights_and_cdf_match_oracle(name, workdir):
    sc, _ = SCENES[name](workdir)
    js = ls.to_json(sc)
    counts, cdf, area, em = lucid_capi.inspect_scene(js)
    o = Oracle()
    assert o.load_scene_json(js)
    ocdf, oarea, oem = o.scene_lights()
    assert counts[:6] == o.scene_stats()
    assert np.array_equal(cdf.view(np.uint32), ocdf.view(np.uint32))
    assert np.array_equal(area.view(np.uint32), oarea.view(np.uint32))
    assert np.array_equal(em.view(np.uint32), oem.view(np.uint32))
    if len(cdf):
        assert cdf[-1] == pytest.approx(1.0, rel=1e-5)
        assert np.all(np.diff(cdf) >= 0)


def test_light_unit_conversions(workdir):
    """parseNativeLights (pybind_renderer.hpp:1597-1736): W -> radiance."""
    import math
    lights = [
        {"type": "POINT", "position": [0, 1, 0], "energy": 100.0, "radius": 0.0},
        {"type": "POINT", "position": [0, 1, 0], "energy": 100.0, "radius": 0.5},
        {"type": "SUN", "direction": [0, -1, 0], "energy": 3.0},
        {"type": "SPOT", "position": [0, 2, 0], "direction": [0, -1, 0], "energy": 50.0,
         "spot_size": math.radians(60)},
        {"type": "AREA", "position": [0, 2, 0], "direction": [0, -1, 0], "size": 2.0, "shape": "SQUARE",
         "energy": 40.0},
        {"type": "AREA", "position": [0, 2, 0], "direction": [0, -1, 0], "size": 2.0, "shape": "DISK",
         "energy": 40.0},
    ]
    sc = {"meshes": [], "native_lights": lights}
    counts, cdf, area, em = lucid_capi.inspect_scene(json.dumps(sc))
    assert counts[3] == 6
    assert em[0, 0] == pytest.approx(100.0 / (4 * math.pi), rel=1e-6)
    a = 4 * math.pi * 0.25
    assert area[1] == pytest.approx(a, rel=1e-6)
    assert em[1, 0] == pytest.approx(100.0 / (math.pi * a), rel=1e-6)
    assert em[2, 0] == pytest.approx(3.0)
    assert em[3, 0] == pytest.approx(50.0 / (2 * math.pi * (1 - math.cos(math.radians(30)))), rel=1e-5)
    assert em[4, 0] == pytest.approx(40.0 / (math.pi * 4.0), rel=1e-6)
    assert area[5] == pytest.approx(math.pi, rel=1e-6)
    assert list(area[[0, 2, 3]]) == [1.0, 1.0, 1.0]   # point-like lights: 1 m^2 in the CDF


@pytest.mark.parametrize("bad", [
    "{not json",
    json.dumps({"meshes": [{"vertices": [[0, 0, 0], [1, 0, 0], [0, 1, 0]], "triangles": [[0, 1, 5]]}]}),
    json.dumps({"meshes": [{"vertices": [[0, 0, 0]], "triangles": [[0, 0, "x"]]}]}),
])
def test_malformed_scenes_rejected(bad):
    with pytest.raises(lucid_capi.LucidError):
        lucid_capi.inspect_scene(bad)


def test_empty_and_volume_boundary(workdir):
    counts, cdf, _, _ = lucid_capi.inspect_scene(json.dumps({"meshes": []}))
    assert counts[:6] == [0, 0, 0, 0, 0, 0] and len(cdf) == 0
    sc, _ = ls.all_lights_scene(workdir=workdir)
    counts, _, _, _ = lucid_capi.inspect_scene(ls.to_json(sc))
    assert counts[4] == 1 and counts[5] == 1   # one boundary-only mesh carrying one grid volume
