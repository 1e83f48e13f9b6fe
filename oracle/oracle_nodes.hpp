// oracle_nodes.hpp — restatement of the reference's material node evaluator
// (LucidRenderer/cpp_renderer/src/node_evaluator.cpp:41-740) for the oracle.
//
// TEST INFRASTRUCTURE ONLY (the checker for the CUDA material programs).
// Like the reference, it walks the node graph by name on every query:
// Principled / Emission / Diffuse BSDF, RGB, Mix (constant factor) and
// Checker texture nodes; anything else evaluates to 0.8 grey.  One
// difference, on purpose: a cycle in the graph (the reference recurses until
// its stack overflows) stops at depth kNodeDepth with the grey default.
#pragma once

#include <cmath>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

namespace orc {

struct V2 {
    float x = 0.0f, y = 0.0f;
};

struct SockVal {   // SocketValue (core/material.hpp:36-70)
    enum Type { FLOAT, VEC3, VEC4, STRING, BOOL, NONE };
    Type type = NONE;
    float f = 0.0f;
    float v3[3] = {0, 0, 0};
    float v4[3] = {0, 0, 0};
};
struct Sock {      // NodeSocket (core/material.hpp:74-83)
    std::string name;
    SockVal def;
    bool linked = false;
    std::string lnode, lsock;
};
struct Node {      // MaterialNode (core/material.hpp:88-102)
    std::string name, type;
    std::vector<Sock> in, out;
    const Sock* input(const std::string& n) const {
        for (const auto& s : in)
            if (s.name == n) return &s;
        return nullptr;
    }
};
struct NodeTree {  // NodeTree (core/material.hpp:107-128)
    std::vector<Node> nodes;
    bool valid = false;
    const Node* find(const std::string& n) const {
        for (const auto& x : nodes)
            if (x.name == n) return &x;
        return nullptr;
    }
    const Node* output() const {
        for (const auto& x : nodes)
            if (x.type == "ShaderNodeOutputMaterial") return &x;
        return nullptr;
    }
};

// parseSocketValue (node_evaluator.cpp:41-70)
inline SockVal parse_sock_val(const nlohmann::json& j) {
    SockVal v;
    if (j.is_number()) {
        v.type = SockVal::FLOAT;
        v.f = j.get<float>();
    } else if (j.is_array()) {
        if (j.size() == 3) {
            v.type = SockVal::VEC3;
            for (int k = 0; k < 3; ++k) v.v3[k] = j[k].get<float>();
        } else if (j.size() == 4) {
            v.type = SockVal::VEC4;
            for (int k = 0; k < 3; ++k) v.v4[k] = j[k].get<float>();
        }
    } else if (j.is_boolean()) {
        v.type = SockVal::BOOL;
    } else if (j.is_string()) {
        v.type = SockVal::STRING;
    }
    return v;
}

// parseNodeTree (node_evaluator.cpp:82-158): links give each input socket its
// source (the last link to a socket wins).
inline NodeTree parse_node_tree(const nlohmann::json& nt) {
    NodeTree t;
    if (!nt.contains("nodes") || !nt.is_object()) return t;
    std::vector<std::pair<std::pair<std::string, std::string>, std::pair<std::string, std::string>>> links;
    if (nt.contains("links"))
        for (const auto& l : nt["links"])
            links.push_back({{l["to_node"].get<std::string>(), l["to_socket"].get<std::string>()},
                             {l["from_node"].get<std::string>(), l["from_socket"].get<std::string>()}});
    for (const auto& nj : nt["nodes"]) {
        Node n;
        n.name = nj.value("name", "");
        n.type = nj.value("type", "");
        if (nj.contains("inputs"))
            for (const auto& ij : nj["inputs"]) {
                Sock s;
                s.name = ij.value("name", "");
                if (ij.contains("default_value")) s.def = parse_sock_val(ij["default_value"]);
                for (const auto& l : links)
                    if (l.first.first == n.name && l.first.second == s.name) {
                        s.linked = true;
                        s.lnode = l.second.first;
                        s.lsock = l.second.second;
                    }
                n.in.push_back(s);
            }
        if (nj.contains("outputs"))
            for (const auto& oj : nj["outputs"]) {
                Sock s;
                s.name = oj.value("name", "");
                if (oj.contains("default_value")) s.def = parse_sock_val(oj["default_value"]);
                n.out.push_back(s);
            }
        t.nodes.push_back(n);
    }
    t.valid = !t.nodes.empty();
    return t;
}

constexpr int kNodeDepth = 32;

struct C3 {
    float r, g, b;
};
inline C3 grey() { return C3{0.8f, 0.8f, 0.8f}; }

// An unlinked colour socket's value: VEC4 (rgb of rgba) or VEC3, else `fb`.
inline C3 sock_color(const SockVal& v, C3 fb) {
    if (v.type == SockVal::VEC4) return C3{v.v4[0], v.v4[1], v.v4[2]};
    if (v.type == SockVal::VEC3) return C3{v.v3[0], v.v3[1], v.v3[2]};
    return fb;
}

// evaluateNode (node_evaluator.cpp:168-404)
inline C3 eval_node(const NodeTree& t, const std::string& name, const std::string& sock, V2 uv, int depth = 0) {
    const Node* n = t.find(name);
    if (!n || depth >= kNodeDepth) return grey();
    auto linked_or = [&](const Sock* s, C3 fb) {
        if (!s) return fb;
        if (s->linked) return eval_node(t, s->lnode, s->lsock, uv, depth + 1);
        return sock_color(s->def, fb);
    };
    if (n->type == "ShaderNodeBsdfPrincipled") {
        if (sock == "BSDF") {
            const Sock* s = n->input("Base Color");
            if (!s) return grey();
            return linked_or(s, grey());
        }
        if (sock == "Base Color") {
            const Sock* s = n->input("Base Color");
            if (s && !s->linked) return sock_color(s->def, grey());
            return grey();
        }
    } else if (n->type == "ShaderNodeEmission") {
        if (sock == "Emission") {
            const Sock* cs = n->input("Color");
            const Sock* ss = n->input("Strength");
            C3 c{1.0f, 1.0f, 1.0f};
            float k = 1.0f;
            if (cs) c = linked_or(cs, c);
            if (ss && !ss->linked && ss->def.type == SockVal::FLOAT) k = ss->def.f;
            return C3{c.r * k, c.g * k, c.b * k};
        }
    } else if (n->type == "ShaderNodeBsdfDiffuse") {
        if (sock == "BSDF") {
            const Sock* s = n->input("Color");
            if (!s) return grey();
            return linked_or(s, grey());
        }
    } else if (n->type == "ShaderNodeRGB") {
        for (const auto& o : n->out)
            if (o.name == "Color" && o.def.type != SockVal::NONE) {
                if (o.def.type == SockVal::VEC4) return C3{o.def.v4[0], o.def.v4[1], o.def.v4[2]};
                if (o.def.type == SockVal::VEC3) return C3{o.def.v3[0], o.def.v3[1], o.def.v3[2]};
            }
        return C3{1.0f, 1.0f, 1.0f};
    } else if (n->type == "ShaderNodeMix" || n->type == "ShaderNodeMixRGB") {
        const Sock* fs = n->input("Fac");
        float fac = 0.5f;
        if (fs && !fs->linked && fs->def.type == SockVal::FLOAT) fac = fs->def.f;
        C3 a = linked_or(n->input("A"), C3{0.0f, 0.0f, 0.0f});
        C3 b = linked_or(n->input("B"), C3{1.0f, 1.0f, 1.0f});
        return C3{a.r * (1.0f - fac) + b.r * fac, a.g * (1.0f - fac) + b.g * fac, a.b * (1.0f - fac) + b.b * fac};
    } else if (n->type == "ShaderNodeTexChecker") {
        C3 c1 = linked_or(n->input("Color1"), C3{0.8f, 0.8f, 0.8f});
        C3 c2 = linked_or(n->input("Color2"), C3{0.2f, 0.2f, 0.2f});
        const Sock* ss = n->input("Scale");
        float scale = 5.0f;
        if (ss && !ss->linked && ss->def.type == SockVal::FLOAT) scale = ss->def.f;
        float u = uv.x * scale, v = uv.y * scale;
        int cu = static_cast<int>(std::floor(u)) % 2, cv = static_cast<int>(std::floor(v)) % 2;
        if (cu < 0) cu += 2;
        if (cv < 0) cv += 2;
        return (cu + cv) % 2 == 0 ? c1 : c2;
    } else if (n->type == "ShaderNodeOutputMaterial") {
        const Sock* s = n->input("Surface");
        if (s && s->linked) return eval_node(t, s->lnode, s->lsock, uv, depth + 1);
    }
    return grey();
}

// The Principled node behind the Material Output's Surface link, if any.
inline const Node* surface_principled(const NodeTree& t, const Node** shader = nullptr) {
    if (shader) *shader = nullptr;
    const Node* o = t.output();
    if (!o) return nullptr;
    const Sock* s = o->input("Surface");
    if (!s || !s->linked) return nullptr;
    const Node* sh = t.find(s->lnode);
    if (shader) *shader = sh;
    return sh && sh->type == "ShaderNodeBsdfPrincipled" ? sh : nullptr;
}

// getAlbedoFromNodeTree (:420-456)
inline C3 node_albedo(const NodeTree& t, V2 uv) {
    if (!t.valid) return grey();
    const Node* o = t.output();
    if (!o) return grey();
    const Sock* s = o->input("Surface");
    if (!s || !s->linked) return grey();
    return eval_node(t, s->lnode, s->lsock, uv);
}

// getEmissionFromNodeTree (:475-533)
inline C3 node_emission(const NodeTree& t, V2 uv) {
    const C3 zero{0.0f, 0.0f, 0.0f};
    if (!t.valid) return zero;
    const Node* sh = nullptr;
    const Node* p = surface_principled(t, &sh);
    if (sh && sh->type == "ShaderNodeEmission") {
        const Sock* s = t.output()->input("Surface");
        return eval_node(t, s->lnode, "Emission", uv);
    }
    if (!p) return zero;
    const Sock* es = p->input("Emission Color");
    if (!es) es = p->input("Emission");
    if (!es) return zero;
    const Sock* ks = p->input("Emission Strength");
    float k = 0.0f;
    if (ks && ks->def.type == SockVal::FLOAT) k = ks->def.f;
    C3 c;
    if (es->linked) c = eval_node(t, es->lnode, es->lsock, uv);
    else if (es->def.type == SockVal::VEC4) c = C3{es->def.v4[0], es->def.v4[1], es->def.v4[2]};
    else if (es->def.type == SockVal::VEC3) c = C3{es->def.v3[0], es->def.v3[1], es->def.v3[2]};
    else return zero;
    return C3{c.r * k, c.g * k, c.b * k};
}

// getTransmission / IOR / Metallic / Roughness FromNodeTree (:548-740): an
// unlinked FLOAT input of the Principled node, else the default.
inline float node_scalar(const NodeTree& t, const char* name, const char* alt, float fb) {
    if (!t.valid) return fb;
    const Node* p = surface_principled(t);
    if (!p) return fb;
    const Sock* s = p->input(name);
    if (!s && alt) s = p->input(alt);
    if (s && !s->linked && s->def.type == SockVal::FLOAT) return s->def.f;
    return fb;
}

}  // namespace orc
