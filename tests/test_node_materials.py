"""Node-graph materials (use_nodes, node_evaluator.cpp) in the oracle, on
the CPU: the restated evaluator's answers on small hand-made graphs, and
that a textured scene renders differently from its use_nodes-off twin."""
from __future__ import annotations

import copy

import numpy as np

import lucid_scenes as ls


def _oracle(scene, cam, algo="mis"):
    from oracle_ctypes import Oracle
    o = Oracle(device_math=True, canonical_ties=True)
    assert o.load_scene_json(ls.to_json(scene))
    o.set_camera(*cam)
    o.set_algorithm(algo)
    return o


def test_albedo_pass_shows_the_checker(oracle_lib):
    scene, cam = ls.textured_scene()
    o = _oracle(scene, cam)
    alb = o.render_debug(1, 64, 48)
    # the floor's albedo takes exactly the checker's two colours
    colours = {tuple(round(float(x), 5) for x in p[:3]) for p in alb.reshape(-1, 4)}
    assert (0.9, 0.8, 0.7) in colours and (0.1, 0.2, 0.3) in colours
    # the wall: Mix(Checker with its default colours, RGB (0.2, 0.6, 0.3)), factor 0.3
    assert (0.62, 0.74, 0.65) in colours and (0.2, 0.32, 0.23) in colours
    # the panel's emission pass shows strength 4 x Color1 and black squares
    em = o.render_debug(2, 64, 48)
    ecols = {tuple(round(float(x), 5) for x in p[:3]) for p in em.reshape(-1, 4)}
    assert (4.0, 3.6, 2.8) in ecols


def test_use_nodes_off_keeps_the_json_fields(oracle_lib):
    scene, cam = ls.textured_scene()
    off = copy.deepcopy(scene)
    for m in off["meshes"]:
        m["material"]["use_nodes"] = False
    a = _oracle(scene, cam).render_debug(1, 32, 24)
    b = _oracle(off, cam).render_debug(1, 32, 24)
    assert not np.array_equal(a, b)
    colours = {tuple(round(float(x), 5) for x in p[:3]) for p in b.reshape(-1, 4)}
    assert (0.1, 0.1, 0.1) in colours          # the floor's own base_color
