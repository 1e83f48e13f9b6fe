// lucid_nodes.cpp — node graph parsing, folding and program emission (see
// lucid_nodes.h).  Semantics: parseNodeTree / parseSocketValue
// (node_evaluator.cpp:41-158), evaluateNode (:168-404) and the get*FromNodeTree
// queries (:420-740).  Compiled with -ffp-contract=off.
#include "lucid_nodes.h"

#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>

namespace lucid {

namespace {

using json = nlohmann::json;

struct SVal {
    enum Kind { FLOAT, VEC3, VEC4, OTHER, NONE } kind = NONE;
    float f = 0.0f;
    float c[3] = {0, 0, 0};   // VEC3 xyz or VEC4 rgb
};
struct Socket {
    std::string name;
    SVal def;
    bool linked = false;
    std::string from_node, from_socket;
};
struct Node {
    std::string name, type;
    std::vector<Socket> in, out;
    const Socket* input(const char* n) const {
        for (const auto& s : in)
            if (s.name == n) return &s;
        return nullptr;
    }
};
struct Graph {
    std::vector<Node> nodes;
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

SVal parse_value(const json& j) {
    SVal v;
    if (j.is_number()) {
        v.kind = SVal::FLOAT;
        v.f = j.get<float>();
    } else if (j.is_array() && (j.size() == 3 || j.size() == 4)) {
        v.kind = j.size() == 3 ? SVal::VEC3 : SVal::VEC4;
        for (int k = 0; k < 3; ++k) v.c[k] = j[k].get<float>();
    } else if (j.is_boolean() || j.is_string()) {
        v.kind = SVal::OTHER;
    }
    return v;
}

Graph parse_graph(const json& nt) {
    Graph g;
    std::map<std::pair<std::string, std::string>, std::pair<std::string, std::string>> links;
    if (nt.contains("links"))
        for (const auto& l : nt["links"])
            links[{l["to_node"].get<std::string>(), l["to_socket"].get<std::string>()}] = {
                l["from_node"].get<std::string>(), l["from_socket"].get<std::string>()};
    for (const auto& nj : nt["nodes"]) {
        Node n;
        n.name = nj.value("name", "");
        n.type = nj.value("type", "");
        for (const char* side : {"inputs", "outputs"}) {
            if (!nj.contains(side)) continue;
            for (const auto& sj : nj[side]) {
                Socket s;
                s.name = sj.value("name", "");
                if (sj.contains("default_value")) s.def = parse_value(sj["default_value"]);
                if (side[0] == 'i') {
                    auto it = links.find({n.name, s.name});
                    if (it != links.end()) {
                        s.linked = true;
                        s.from_node = it->second.first;
                        s.from_socket = it->second.second;
                    }
                    n.in.push_back(s);
                } else {
                    n.out.push_back(s);
                }
            }
        }
        g.nodes.push_back(n);
    }
    return g;
}

// A compiled colour: a constant or the index (within the program) of a step.
struct CVal {
    bool is_const = true;
    float c[3] = {0.8f, 0.8f, 0.8f};
    int step = -1;
};
CVal konst(float r, float g, float b) {
    CVal v;
    v.c[0] = r; v.c[1] = g; v.c[2] = b;
    return v;
}
CVal grey() { return konst(0.8f, 0.8f, 0.8f); }

constexpr int kMaxDepth = 32;   // a cyclic graph stops here (grey)

struct Program {
    std::vector<float4> steps;   // two float4 per step
    int count() const { return (int)steps.size() / 2; }
    int emit(int kind, int a, int b, float k, const float* c) {
        if (count() >= kTexMaxOps) throw std::runtime_error("material node graph exceeds the device program size");
        float4 s0, s1;
        int bits[3] = {kind, a, b};
        std::memcpy(&s0.x, &bits[0], 4);
        std::memcpy(&s0.y, &bits[1], 4);
        std::memcpy(&s0.z, &bits[2], 4);
        s0.w = k;
        s1.x = c ? c[0] : 0.0f; s1.y = c ? c[1] : 0.0f; s1.z = c ? c[2] : 0.0f; s1.w = 0.0f;
        steps.push_back(s0);
        steps.push_back(s1);
        return count() - 1;
    }
    int operand(const CVal& v) { return v.is_const ? emit(TEX_CONST, 0, 0, 0.0f, v.c) : v.step; }
};

CVal color_of(const SVal& v, CVal fb) {
    if (v.kind == SVal::VEC4 || v.kind == SVal::VEC3) return konst(v.c[0], v.c[1], v.c[2]);
    return fb;
}

CVal compile(const Graph& g, Program& P, const std::string& name, const std::string& sock, int depth);

// An input socket: its linked source, its own colour, or `fb`.
CVal input_color(const Graph& g, Program& P, const Socket* s, CVal fb, int depth) {
    if (!s) return fb;
    if (s->linked) return compile(g, P, s->from_node, s->from_socket, depth + 1);
    return color_of(s->def, fb);
}

CVal compile(const Graph& g, Program& P, const std::string& name, const std::string& sock, int depth) {
    const Node* n = g.find(name);
    if (!n || depth >= kMaxDepth) return grey();
    if (n->type == "ShaderNodeBsdfPrincipled") {
        if (sock == "BSDF") {
            const Socket* s = n->input("Base Color");
            return s ? input_color(g, P, s, grey(), depth) : grey();
        }
        if (sock == "Base Color") {
            const Socket* s = n->input("Base Color");
            return (s && !s->linked) ? color_of(s->def, grey()) : grey();
        }
    } else if (n->type == "ShaderNodeEmission") {
        if (sock == "Emission") {
            CVal c = input_color(g, P, n->input("Color"), konst(1.0f, 1.0f, 1.0f), depth);
            const Socket* ss = n->input("Strength");
            float k = 1.0f;
            if (ss && !ss->linked && ss->def.kind == SVal::FLOAT) k = ss->def.f;
            if (c.is_const) return konst(c.c[0] * k, c.c[1] * k, c.c[2] * k);
            CVal r;
            r.is_const = false;
            r.step = P.emit(TEX_SCALE, c.step, 0, k, nullptr);
            return r;
        }
    } else if (n->type == "ShaderNodeBsdfDiffuse") {
        if (sock == "BSDF") {
            const Socket* s = n->input("Color");
            return s ? input_color(g, P, s, grey(), depth) : grey();
        }
    } else if (n->type == "ShaderNodeRGB") {
        for (const auto& o : n->out)
            if (o.name == "Color" && (o.def.kind == SVal::VEC4 || o.def.kind == SVal::VEC3))
                return konst(o.def.c[0], o.def.c[1], o.def.c[2]);
        return konst(1.0f, 1.0f, 1.0f);
    } else if (n->type == "ShaderNodeMix" || n->type == "ShaderNodeMixRGB") {
        const Socket* fs = n->input("Fac");
        float fac = 0.5f;
        if (fs && !fs->linked && fs->def.kind == SVal::FLOAT) fac = fs->def.f;
        CVal a = input_color(g, P, n->input("A"), konst(0.0f, 0.0f, 0.0f), depth);
        CVal b = input_color(g, P, n->input("B"), konst(1.0f, 1.0f, 1.0f), depth);
        if (a.is_const && b.is_const)
            return konst(a.c[0] * (1.0f - fac) + b.c[0] * fac, a.c[1] * (1.0f - fac) + b.c[1] * fac,
                         a.c[2] * (1.0f - fac) + b.c[2] * fac);
        const int ia = P.operand(a), ib = P.operand(b);
        CVal r;
        r.is_const = false;
        r.step = P.emit(TEX_MIX, ia, ib, fac, nullptr);
        return r;
    } else if (n->type == "ShaderNodeTexChecker") {
        CVal c1 = input_color(g, P, n->input("Color1"), konst(0.8f, 0.8f, 0.8f), depth);
        CVal c2 = input_color(g, P, n->input("Color2"), konst(0.2f, 0.2f, 0.2f), depth);
        const Socket* ss = n->input("Scale");
        float scale = 5.0f;
        if (ss && !ss->linked && ss->def.kind == SVal::FLOAT) scale = ss->def.f;
        const int i1 = P.operand(c1), i2 = P.operand(c2);
        CVal r;
        r.is_const = false;
        r.step = P.emit(TEX_CHECKER, i1, i2, scale, nullptr);
        return r;
    } else if (n->type == "ShaderNodeOutputMaterial") {
        const Socket* s = n->input("Surface");
        if (s && s->linked) return compile(g, P, s->from_node, s->from_socket, depth + 1);
    }
    return grey();
}

// The Principled node the Material Output's Surface is linked to, and the
// linked shader node itself.
const Node* surface_shader(const Graph& g, const Socket** surf) {
    *surf = nullptr;
    const Node* o = g.output();
    if (!o) return nullptr;
    const Socket* s = o->input("Surface");
    if (!s || !s->linked) return nullptr;
    *surf = s;
    return g.find(s->from_node);
}

float principled_scalar(const Graph& g, const char* name, const char* alt, float fb) {
    const Socket* surf;
    const Node* sh = surface_shader(g, &surf);
    if (!sh || sh->type != "ShaderNodeBsdfPrincipled") return fb;
    const Socket* s = sh->input(name);
    if (!s && alt) s = sh->input(alt);
    if (s && !s->linked && s->def.kind == SVal::FLOAT) return s->def.f;
    return fb;
}

// getAlbedoFromNodeTree (node_evaluator.cpp:420-456)
CVal compile_albedo(const Graph& g, Program& P) {
    const Socket* surf;
    surface_shader(g, &surf);
    if (!surf) return grey();
    return compile(g, P, surf->from_node, surf->from_socket, 0);
}

// getEmissionFromNodeTree (node_evaluator.cpp:475-533)
CVal compile_emission(const Graph& g, Program& P) {
    const CVal zero = konst(0.0f, 0.0f, 0.0f);
    const Socket* surf;
    const Node* sh = surface_shader(g, &surf);
    if (!sh) return zero;
    if (sh->type == "ShaderNodeEmission") return compile(g, P, surf->from_node, "Emission", 0);
    if (sh->type != "ShaderNodeBsdfPrincipled") return zero;
    const Socket* es = sh->input("Emission Color");
    if (!es) es = sh->input("Emission");
    if (!es) return zero;
    const Socket* ks = sh->input("Emission Strength");
    float k = 0.0f;
    if (ks && ks->def.kind == SVal::FLOAT) k = ks->def.f;
    CVal c;
    if (es->linked) c = compile(g, P, es->from_node, es->from_socket, 0);
    else if (es->def.kind == SVal::VEC4 || es->def.kind == SVal::VEC3) c = konst(es->def.c[0], es->def.c[1], es->def.c[2]);
    else return zero;
    if (c.is_const) return konst(c.c[0] * k, c.c[1] * k, c.c[2] * k);
    CVal r;
    r.is_const = false;
    r.step = P.emit(TEX_SCALE, c.step, 0, k, nullptr);
    return r;
}

}  // namespace

void eval_tex_program(const float4* ops, int n, float u, float v, float out[3]) {
    float val[kTexMaxOps][3];
    for (int i = 0; i < n && i < kTexMaxOps; ++i) {
        const float4 s0 = ops[2 * i], s1 = ops[2 * i + 1];
        int kind, a, b;
        std::memcpy(&kind, &s0.x, 4);
        std::memcpy(&a, &s0.y, 4);
        std::memcpy(&b, &s0.z, 4);
        const float k = s0.w;
        if (kind == TEX_CONST) {
            val[i][0] = s1.x; val[i][1] = s1.y; val[i][2] = s1.z;
        } else if (kind == TEX_CHECKER) {
            int cu = static_cast<int>(std::floor(u * k)) % 2, cv = static_cast<int>(std::floor(v * k)) % 2;
            if (cu < 0) cu += 2;
            if (cv < 0) cv += 2;
            const int src = (cu + cv) % 2 == 0 ? a : b;
            for (int c = 0; c < 3; ++c) val[i][c] = val[src][c];
        } else if (kind == TEX_MIX) {
            for (int c = 0; c < 3; ++c) val[i][c] = val[a][c] * (1.0f - k) + val[b][c] * k;
        } else {
            for (int c = 0; c < 3; ++c) val[i][c] = val[a][c] * k;
        }
    }
    for (int c = 0; c < 3; ++c) out[c] = n > 0 ? val[n - 1][c] : 0.0f;
}

NodeMaterial compile_node_material(const json& node_tree, std::vector<float4>& ops) {
    const Graph g = parse_graph(node_tree);
    NodeMaterial m;
    m.metallic = principled_scalar(g, "Metallic", nullptr, 0.0f);
    m.roughness = principled_scalar(g, "Roughness", nullptr, 0.5f);
    m.transmission = principled_scalar(g, "Transmission", "Transmission Weight", 0.0f);
    m.ior = principled_scalar(g, "IOR", nullptr, 1.45f);
    for (int which = 0; which < 2; ++which) {
        Program P;
        const CVal v = which == 0 ? compile_albedo(g, P) : compile_emission(g, P);
        float* dst = which == 0 ? m.albedo : m.emission;
        if (v.is_const) {
            for (int c = 0; c < 3; ++c) dst[c] = v.c[c];
            continue;
        }
        // the program's last step is the value; keep only steps up to it
        P.steps.resize((size_t)(v.step + 1) * 2);
        eval_tex_program(P.steps.data(), P.count(), 0.0f, 0.0f, dst);
        const int start = (int)ops.size() / 2;
        ops.insert(ops.end(), P.steps.begin(), P.steps.end());
        if (which == 0) { m.albedo_start = start; m.albedo_n = P.count(); }
        else { m.emission_start = start; m.emission_n = P.count(); }
    }
    return m;
}

}  // namespace lucid
