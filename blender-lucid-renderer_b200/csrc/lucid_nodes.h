// lucid_nodes.h — material node graphs compiled to device programs.
//
// The reference evaluates a material's node graph by name at every hit
// (src/node_evaluator.cpp:168-740, called from getMaterialParams,
// integrator/path_tracer.hpp:45-72).  Everything in that evaluator except the
// Checker texture is independent of the hit, so the loader folds it to
// constants once; what remains (a Checker somewhere below the Base Color or
// the emission colour) becomes a short program of CONST / CHECKER / MIX /
// SCALE steps over the hit's UV that the shading kernels run.  Folding and
// the device steps use the same float operations in the same order, so a
// folded value equals the evaluated one bit for bit.
#pragma once

#include <nlohmann/json.hpp>
#include <string>
#include <vector>

#include "lucid_types.h"

namespace lucid {


// A material's values under use_nodes: the five scalars folded, albedo and
// emission each either a constant (n == 0) or a program of n steps (two
// float4 per step in `ops`: {kind, operand a, operand b, k}, {rgb, 0}).
struct NodeMaterial {
    float albedo[3], emission[3];        // the values at uv (0, 0)
    float metallic, roughness, transmission, ior;
    int albedo_start = 0, albedo_n = 0, emission_start = 0, emission_n = 0;
};

// Compiles `node_tree` (a valid tree: an object with a non-empty "nodes"
// array) and appends its programs to `ops`.  Throws std::runtime_error when a
// program would exceed kTexMaxOps steps.
NodeMaterial compile_node_material(const nlohmann::json& node_tree, std::vector<float4>& ops);

// Host evaluation of a program (the device steps, same float operations).
void eval_tex_program(const float4* ops, int n, float u, float v, float out[3]);

}  // namespace lucid
