// MRay scene JSON loader (host code): the subset of GPUSceneJson
// (GPUSceneJson.cpp:150-560) and SceneIO (RayLib/SceneIO.cpp:78-226) that
// the hot path consumes, producing an mrb_scene_desc and a pinhole camera.
//
//   Cameras          "Pinhole" (GPUCameraPinhole.cu:40-78: fov in degrees,
//                    the vertical fov re-derived from the horizontal one)
//   Lights           "Null" (boundary), "Primitive" (radiance, primitive,
//                    accelerator) placed by LightSurfaces
//   Mediums          "Vacuum", "Homogeneous" (IOR; absorption and
//                    scattering must be zero)
//   Transforms       "Identity", "Single" with layout "matrix4x4" (row or
//                    column major) or "trs" (GPUTransformSingle.cu:45-100),
//                    applied to positions and normals at load time
//   Materials        "Lambert" (constant albedo), "LambertC", "Metal",
//                    "Unreal" (constant parameters), "Refract"
//   Primitives       "Triangle" from the in-node loaders ".nodeTriangle" /
//                    ".nodeTriangleIndexed" (RayLib/BasicSurfaceLoaders.cpp),
//                    optional "cullFace" (default true)
//   Accelerators     any type name (they all map to the LBVH group)
//   Surfaces, LightSurfaces, CameraSurfaces, BaseMedium, BaseBoundaryLight
//
// Nodes may list several ids ("id": [a, b, ...]); their attributes are then
// arrays with one entry per id (SceneNodeJson).  The JSON may carry // and
// /* */ comments and trailing commas, as MRay's scene files do.  Anything
// outside this subset (file-based meshes, spheres, textures, other lights
// and cameras) is rejected with MRB_E_UNSUPPORTED and a message naming it.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <exception>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mrb200.h"
#include "common.cuh"

namespace mrb {
namespace {

// ---------------------------------------------------------------------------
// JSON value and a tolerant recursive-descent parser
// ---------------------------------------------------------------------------
struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double n = 0.0;
    std::string s;
    std::vector<JVal> a;
    std::vector<std::pair<std::string, JVal>> o;  // insertion order kept

    const JVal* get(const char* key) const {
        if (kind != Obj) return nullptr;
        for (const auto& kv : o)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    bool is_arr() const { return kind == Arr; }
    bool is_num() const { return kind == Num; }
};

struct JParser {
    const char* p;
    const char* end;
    std::string err;
    int line = 1;

    void skip() {
        for (;;) {
            while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) {
                if (*p == '\n') line++;
                p++;
            }
            if (p + 1 < end && p[0] == '/' && p[1] == '/') {
                while (p < end && *p != '\n') p++;
                continue;
            }
            if (p + 1 < end && p[0] == '/' && p[1] == '*') {
                p += 2;
                while (p + 1 < end && !(p[0] == '*' && p[1] == '/')) {
                    if (*p == '\n') line++;
                    p++;
                }
                p = (p + 1 < end) ? p + 2 : end;
                continue;
            }
            return;
        }
    }
    bool fail(const char* what) {
        if (err.empty()) err = std::string(what) + " at line " + std::to_string(line);
        return false;
    }
    bool parse_string(std::string& out) {
        if (p >= end || *p != '"') return fail("expected a string");
        p++;
        while (p < end && *p != '"') {
            if (*p == '\\' && p + 1 < end) {
                p++;
                switch (*p) {
                    case 'n': out.push_back('\n'); break;
                    case 't': out.push_back('\t'); break;
                    case 'r': out.push_back('\r'); break;
                    case 'b': out.push_back('\b'); break;
                    case 'f': out.push_back('\f'); break;
                    case 'u':
                        // \uXXXX outside ASCII is not used by scene files
                        if (p + 4 < end) {
                            out.push_back(static_cast<char>(std::strtol(std::string(p + 1, 4).c_str(),
                                                                        nullptr, 16) & 0x7F));
                            p += 4;
                        }
                        break;
                    default: out.push_back(*p); break;
                }
                p++;
            } else {
                if (*p == '\n') line++;
                out.push_back(*p++);
            }
        }
        if (p >= end) return fail("unterminated string");
        p++;
        return true;
    }
    bool parse(JVal& v, int depth = 0) {
        if (depth > 64) return fail("nesting too deep");
        skip();
        if (p >= end) return fail("unexpected end of input");
        const char c = *p;
        if (c == '{') {
            v.kind = JVal::Obj;
            p++;
            for (;;) {
                skip();
                if (p < end && *p == '}') {
                    p++;
                    return true;
                }
                std::string key;
                if (!parse_string(key)) return false;
                skip();
                if (p >= end || *p != ':') return fail("expected ':'");
                p++;
                JVal child;
                if (!parse(child, depth + 1)) return false;
                v.o.emplace_back(std::move(key), std::move(child));
                skip();
                if (p < end && *p == ',') {
                    p++;
                    continue;
                }
                if (p < end && *p == '}') {
                    p++;
                    return true;
                }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = JVal::Arr;
            p++;
            for (;;) {
                skip();
                if (p < end && *p == ']') {
                    p++;
                    return true;
                }
                JVal child;
                if (!parse(child, depth + 1)) return false;
                v.a.push_back(std::move(child));
                skip();
                if (p < end && *p == ',') {
                    p++;
                    continue;
                }
                if (p < end && *p == ']') {
                    p++;
                    return true;
                }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = JVal::Str;
            return parse_string(v.s);
        }
        if (end - p >= 4 && std::strncmp(p, "true", 4) == 0) {
            v.kind = JVal::Bool;
            v.b = true;
            p += 4;
            return true;
        }
        if (end - p >= 5 && std::strncmp(p, "false", 5) == 0) {
            v.kind = JVal::Bool;
            p += 5;
            return true;
        }
        if (end - p >= 4 && std::strncmp(p, "null", 4) == 0) {
            v.kind = JVal::Null;
            p += 4;
            return true;
        }
        if (c == '-' || c == '+' || (c >= '0' && c <= '9') || c == '.') {
            char* q = nullptr;
            const std::string tok(p, static_cast<size_t>(std::min<ptrdiff_t>(end - p, 64)));
            v.n = std::strtod(tok.c_str(), &q);
            if (q == tok.c_str()) return fail("bad number");
            v.kind = JVal::Num;
            p += (q - tok.c_str());
            return true;
        }
        return fail("unexpected character");
    }
};

// ---------------------------------------------------------------------------
// scene nodes
// ---------------------------------------------------------------------------
struct LoadError {
    int code;
    std::string msg;
};

struct NodeRef {
    const JVal* node = nullptr;
    uint32_t inner = 0;
    bool multi = false;
};

// GenIdLookup: node id -> (node, index inside a multi-id node)
void build_lookup(const JVal* arr, const char* what, std::map<uint32_t, NodeRef>& out) {
    if (!arr) return;
    if (!arr->is_arr()) throw LoadError{MRB_E_ARG, std::string(what) + " must be an array"};
    for (const JVal& n : arr->a) {
        const JVal* id = n.get("id");
        if (!id) throw LoadError{MRB_E_ARG, std::string(what) + ": node without \"id\""};
        if (id->is_arr()) {
            for (size_t i = 0; i < id->a.size(); i++) {
                if (!id->a[i].is_num()) throw LoadError{MRB_E_ARG, std::string(what) + ": bad id"};
                out[static_cast<uint32_t>(id->a[i].n)] = NodeRef{&n, static_cast<uint32_t>(i), true};
            }
        } else if (id->is_num()) {
            out[static_cast<uint32_t>(id->n)] = NodeRef{&n, 0, false};
        } else {
            throw LoadError{MRB_E_ARG, std::string(what) + ": bad id"};
        }
    }
}

std::string node_type(const NodeRef& r) {
    const JVal* t = r.node->get("type");
    return (t && t->kind == JVal::Str) ? t->s : std::string();
}

// the value of `key` for this id: a multi-id node lists one entry per id
// (SceneNodeJson); a value that is not such a list is taken as shared
const JVal* field(const NodeRef& r, const char* key) {
    const JVal* v = r.node->get(key);
    if (!v) return nullptr;
    if (r.multi && v->is_arr() && v->a.size() == r.node->get("id")->a.size())
        return &v->a[r.inner];
    return v;
}

double num(const JVal* v, const char* what) {
    if (!v || !v->is_num()) throw LoadError{MRB_E_ARG, std::string("expected a number for ") + what};
    return v->n;
}
void vec(const JVal* v, int n, double* out, const char* what) {
    if (!v || !v->is_arr() || v->a.size() != static_cast<size_t>(n))
        throw LoadError{MRB_E_ARG, std::string("expected ") + std::to_string(n) +
                                       " numbers for " + what};
    for (int i = 0; i < n; i++) out[i] = num(&v->a[i], what);
}
bool boolean(const JVal* v, bool dflt) {
    if (!v) return dflt;
    if (v->kind == JVal::Bool) return v->b;
    if (v->is_num()) return v->n != 0.0;
    throw LoadError{MRB_E_ARG, "expected a boolean"};
}

struct Mat4 {
    double m[4][4];
    static Mat4 identity() {
        Mat4 r{};
        for (int i = 0; i < 4; i++) r.m[i][i] = 1.0;
        return r;
    }
    Mat4 operator*(const Mat4& b) const {
        Mat4 r{};
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++)
                for (int k = 0; k < 4; k++) r.m[i][j] += m[i][k] * b.m[k][j];
        return r;
    }
};

// CPUTransformSingle::InitializeGroup (GPUTransformSingle.cu:45-100)
Mat4 transform_of(const std::map<uint32_t, NodeRef>& tl, uint32_t id) {
    const auto it = tl.find(id);
    if (it == tl.end()) throw LoadError{MRB_E_ARG, "transform " + std::to_string(id) + " not found"};
    const NodeRef& r = it->second;
    const std::string type = node_type(r);
    if (type == "Identity") return Mat4::identity();
    if (type != "Single") throw LoadError{MRB_E_UNSUPPORTED, "transform type '" + type + "'"};
    const JVal* lay = r.node->get("layout");
    const std::string layout = (lay && lay->kind == JVal::Str) ? lay->s : "";
    if (layout == "matrix4x4") {
        const JVal* mv = field(r, "matrix");
        if (!mv || !mv->is_arr()) throw LoadError{MRB_E_ARG, "transform: matrix missing"};
        // nested rows or a flat list of 16
        std::vector<double> a;
        for (const JVal& e : mv->a) {
            if (e.is_arr()) {
                for (const JVal& x : e.a) a.push_back(num(&x, "matrix"));
            } else {
                a.push_back(num(&e, "matrix"));
            }
        }
        if (a.size() != 16) throw LoadError{MRB_E_ARG, "transform: matrix needs 16 numbers"};
        const JVal* mj = r.node->get("major");
        const bool rowMajor = mj && mj->kind == JVal::Str && mj->s == "row";
        Mat4 M{};
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) M.m[i][j] = rowMajor ? a[i * 4 + j] : a[j * 4 + i];
        return M;
    }
    if (layout == "trs") {
        double t[3], rdeg[3], sc[3];
        vec(field(r, "translate"), 3, t, "translate");
        vec(field(r, "rotate"), 3, rdeg, "rotate");
        vec(field(r, "scale"), 3, sc, "scale");
        const double k = 3.14159265358979323846 / 180.0;
        auto rot = [&](int axis, double ang) {
            Mat4 R = Mat4::identity();
            const double c = std::cos(ang * k), s = std::sin(ang * k);
            const int a0 = (axis + 1) % 3, a1 = (axis + 2) % 3;
            R.m[a0][a0] = c;
            R.m[a0][a1] = -s;
            R.m[a1][a0] = s;
            R.m[a1][a1] = c;
            return R;
        };
        Mat4 S = Mat4::identity(), T = Mat4::identity();
        for (int i = 0; i < 3; i++) {
            S.m[i][i] = sc[i];
            T.m[i][3] = t[i];
        }
        // M = T * Rz * Ry * Rx * S
        return T * (rot(2, rdeg[2]) * (rot(1, rdeg[1]) * (rot(0, rdeg[0]) * S)));
    }
    throw LoadError{MRB_E_UNSUPPORTED, "transform layout '" + layout + "'"};
}

struct SceneBuild {
    std::map<uint32_t, NodeRef> prims, mats, lights, cams, accels, xforms, media;
    std::vector<float> pos, nrm, uv;
    std::vector<uint32_t> idx, triMat;
    std::vector<uint8_t> cull;
    std::vector<mrb_material> materials;
    std::vector<float> mediumIor;
    std::map<uint32_t, uint32_t> matIndex, lightIndex, mediumIndex;
    uint32_t baseMedium = 0;
    std::vector<mrb_camera> cameras;

    const NodeRef& find(const std::map<uint32_t, NodeRef>& m, uint32_t id, const char* what) {
        const auto it = m.find(id);
        if (it == m.end()) throw LoadError{MRB_E_ARG, std::string(what) + " " + std::to_string(id) + " not found"};
        return it->second;
    }

    // GPUMediumVacuum / GPUMediumHomogeneous (IOR only)
    uint32_t medium(uint32_t id) {
        const auto it = mediumIndex.find(id);
        if (it != mediumIndex.end()) return it->second;
        const NodeRef& r = find(media, id, "medium");
        const std::string type = node_type(r);
        float ior = 1.0f;
        if (type == "Homogeneous") {
            ior = static_cast<float>(num(field(r, "ior"), "ior"));
            for (const char* k : {"absorption", "scattering"}) {
                const JVal* v = field(r, k);
                if (!v) continue;
                double c[3];
                vec(v, 3, c, k);
                if (c[0] != 0.0 || c[1] != 0.0 || c[2] != 0.0)
                    throw LoadError{MRB_E_UNSUPPORTED, std::string("medium ") + std::to_string(id) +
                                                           ": non-zero " + k + " (IOR-only media)"};
            }
        } else if (type != "Vacuum") {
            throw LoadError{MRB_E_UNSUPPORTED, "medium type '" + type + "'"};
        }
        const uint32_t k = static_cast<uint32_t>(mediumIor.size());
        mediumIor.push_back(ior);
        mediumIndex[id] = k;
        return k;
    }

    static void put3(float* dst, const JVal* v, const char* what) {
        if (v && v->kind == JVal::Obj)
            throw LoadError{MRB_E_UNSUPPORTED, std::string(what) + " given as a texture"};
        double c[3];
        vec(v, 3, c, what);
        for (int i = 0; i < 3; i++) dst[i] = static_cast<float>(c[i]);
    }
    static float scalar(const JVal* v, const char* what) {
        if (v && v->kind == JVal::Obj)
            throw LoadError{MRB_E_UNSUPPORTED, std::string(what) + " given as a texture"};
        return static_cast<float>(num(v, what));
    }

    uint32_t material(uint32_t id) {
        const auto it = matIndex.find(id);
        if (it != matIndex.end()) return it->second;
        const NodeRef& r = find(mats, id, "material");
        const std::string type = node_type(r);
        mrb_material m{};
        if (type == "Lambert" || type == "LambertC") {
            m.type = (type == "Lambert") ? MRB_MAT_LAMBERT : MRB_MAT_LAMBERTC;
            put3(m.albedo, field(r, "albedo"), "albedo");
            if (r.node->get("normal"))
                throw LoadError{MRB_E_UNSUPPORTED, "material " + std::to_string(id) + ": normal map"};
        } else if (type == "Metal") {  // MetalGlassMaterials.cu:11-14
            m.type = MRB_MAT_METAL;
            put3(m.eta, field(r, "eta"), "eta");
            put3(m.k, field(r, "k"), "k");
            put3(m.specular, field(r, "specular"), "specular");
            m.roughness = scalar(field(r, "roughness"), "roughness");
        } else if (type == "Unreal") {  // UnrealMaterial.cu:95-99
            m.type = MRB_MAT_UNREAL;
            put3(m.albedo, field(r, "albedo"), "albedo");
            m.roughness = scalar(field(r, "roughness"), "roughness");
            m.metallic = scalar(field(r, "metallic"), "metallic");
            m.specular[0] = scalar(field(r, "specular"), "specular");
            if (r.node->get("normal"))
                throw LoadError{MRB_E_UNSUPPORTED, "material " + std::to_string(id) + ": normal map"};
        } else if (type == "Refract") {  // SimpleMaterials.cu:99-100
            m.type = MRB_MAT_REFRACT;
            put3(m.albedo, field(r, "albedo"), "albedo");
            m.medium = medium(static_cast<uint32_t>(num(field(r, "medium"), "medium")));
        } else {
            throw LoadError{MRB_E_UNSUPPORTED, "material type '" + type + "'"};
        }
        const uint32_t k = static_cast<uint32_t>(materials.size());
        materials.push_back(m);
        matIndex[id] = k;
        return k;
    }

    uint32_t light_material(uint32_t id, const NodeRef& r) {
        const auto it = lightIndex.find(id);
        if (it != lightIndex.end()) return it->second;
        mrb_material m{};
        m.type = MRB_MAT_LIGHT;
        put3(m.radiance, field(r, "radiance"), "radiance");
        const uint32_t k = static_cast<uint32_t>(materials.size());
        materials.push_back(m);
        lightIndex[id] = k;
        return k;
    }

    // InNodeTriLoader / InNodeTriLoaderIndexed (RayLib/BasicSurfaceLoaders.cpp)
    void primitive(uint32_t id, const Mat4& M, uint32_t mat) {
        const NodeRef& r = find(prims, id, "primitive");
        const std::string type = node_type(r);
        if (type != "Triangle")
            throw LoadError{MRB_E_UNSUPPORTED, "primitive type '" + type + "' (triangles only)"};
        const JVal* nm = r.node->get("name");
        const std::string name = (nm && nm->kind == JVal::Str) ? nm->s : "";
        const bool indexed = (name == ".nodeTriangleIndexed" || name == "nodeTriangleIndexed");
        if (!indexed && name != ".nodeTriangle" && name != "nodeTriangle")
            throw LoadError{MRB_E_UNSUPPORTED, "primitive " + std::to_string(id) + ": surface '" +
                                                   name + "' needs a file loader (in-node triangles only)"};
        auto list = [&](const char* key, int n, std::vector<double>& out, bool required) {
            const JVal* v = field(r, key);
            if (!v) {
                if (required) throw LoadError{MRB_E_ARG, std::string("primitive: ") + key + " missing"};
                return;
            }
            if (!v->is_arr()) throw LoadError{MRB_E_ARG, std::string("primitive: bad ") + key};
            for (const JVal& e : v->a) {
                double c[3];
                vec(&e, n, c, key);
                for (int i = 0; i < n; i++) out.push_back(c[i]);
            }
        };
        std::vector<double> P, N, T;
        list("position", 3, P, true);
        list("normal", 3, N, true);
        list("uv", 2, T, false);
        const size_t nv = P.size() / 3;
        if (N.size() != P.size()) throw LoadError{MRB_E_ARG, "primitive: normal count differs from position count"};
        if (!T.empty() && T.size() / 2 != nv) throw LoadError{MRB_E_ARG, "primitive: uv count differs"};
        std::vector<uint32_t> I;
        if (indexed) {
            const JVal* iv = field(r, "index");
            if (!iv || !iv->is_arr()) throw LoadError{MRB_E_ARG, "primitive: index missing"};
            for (const JVal& e : iv->a) {
                const double x = num(&e, "index");
                if (x < 0 || x >= double(nv)) throw LoadError{MRB_E_ARG, "primitive: index out of range"};
                I.push_back(static_cast<uint32_t>(x));
            }
        } else {
            for (size_t i = 0; i < nv; i++) I.push_back(static_cast<uint32_t>(i));
        }
        if (I.size() % 3 != 0) throw LoadError{MRB_E_ARG, "primitive: not a whole number of triangles"};
        const bool cullFace = boolean(field(r, "cullFace"), true);
        // normals go through the inverse transpose of the 3x3 part
        double A[3][3], inv[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) A[i][j] = M.m[i][j];
        const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                           A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
        if (det == 0.0) throw LoadError{MRB_E_ARG, "transform is singular"};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                const int i1 = (j + 1) % 3, i2 = (j + 2) % 3, j1 = (i + 1) % 3, j2 = (i + 2) % 3;
                inv[i][j] = (A[i1][j1] * A[i2][j2] - A[i1][j2] * A[i2][j1]) / det;
            }
        const uint32_t base = static_cast<uint32_t>(pos.size() / 3);
        for (size_t v = 0; v < nv; v++) {
            const double* p = &P[3 * v];
            const double* n = &N[3 * v];
            double wn[3], len = 0.0;
            for (int i = 0; i < 3; i++) {
                const double wp = M.m[i][0] * p[0] + M.m[i][1] * p[1] + M.m[i][2] * p[2] + M.m[i][3];
                pos.push_back(static_cast<float>(wp));
                // (A^-1)^T n: row i of the transpose is column i of A^-1
                wn[i] = inv[0][i] * n[0] + inv[1][i] * n[1] + inv[2][i] * n[2];
                len += wn[i] * wn[i];
            }
            len = std::sqrt(len);
            for (int i = 0; i < 3; i++) nrm.push_back(static_cast<float>(len > 0.0 ? wn[i] / len : wn[i]));
            uv.push_back(T.empty() ? 0.0f : static_cast<float>(T[2 * v]));
            uv.push_back(T.empty() ? 0.0f : static_cast<float>(T[2 * v + 1]));
        }
        for (size_t t = 0; t < I.size() / 3; t++) {
            for (int k = 0; k < 3; k++) idx.push_back(base + I[3 * t + k]);
            triMat.push_back(mat);
            cull.push_back(cullFace ? 1 : 0);
        }
    }
};

const JVal* section(const JVal& root, const char* key, bool required) {
    const JVal* v = root.get(key);
    if (!v && required) throw LoadError{MRB_E_ARG, std::string("scene: \"") + key + "\" missing"};
    return v;
}

uint32_t uid(const JVal* v, const char* what) {
    const double x = num(v, what);
    if (x < 0 || x > 4294967295.0) throw LoadError{MRB_E_ARG, std::string("bad id for ") + what};
    return static_cast<uint32_t>(x);
}

// GPUCameraPinhole group initialisation (GPUCameraPinhole.cu:40-78)
mrb_camera pinhole(const NodeRef& r, const Mat4& M) {
    const std::string type = node_type(r);
    if (type != "Pinhole") throw LoadError{MRB_E_UNSUPPORTED, "camera type '" + type + "'"};
    double pos[3], gz[3], up[3], planes[2], fov[2];
    vec(field(r, "position"), 3, pos, "position");
    vec(field(r, "gaze"), 3, gz, "gaze");
    vec(field(r, "up"), 3, up, "up");
    vec(field(r, "planes"), 2, planes, "planes");
    vec(field(r, "fov"), 2, fov, "fov");
    mrb_camera c{};
    for (int i = 0; i < 3; i++) {
        c.position[i] = static_cast<float>(M.m[i][0] * pos[0] + M.m[i][1] * pos[1] + M.m[i][2] * pos[2] + M.m[i][3]);
        c.gaze[i] = static_cast<float>(M.m[i][0] * gz[0] + M.m[i][1] * gz[1] + M.m[i][2] * gz[2] + M.m[i][3]);
        c.up[i] = static_cast<float>(M.m[i][0] * up[0] + M.m[i][1] * up[1] + M.m[i][2] * up[2]);
    }
    c.near_far[0] = static_cast<float>(planes[0]);
    c.near_far[1] = static_cast<float>(planes[1]);
    // fov in degrees; the vertical one follows from the horizontal one and
    // the ratio of the two given values
    const float degToRad = 0.017453292519943295f;
    const float fx = static_cast<float>(fov[0]), fy = static_cast<float>(fov[1]);
    c.fov[0] = fx * degToRad;
    const float aspect = fy / fx;
    c.fov[1] = 2.0f * std::atan(std::tan(c.fov[0] * 0.5f) * aspect);
    return c;
}

// GPUSceneJson::GenerateConstructionData (GPUSceneJson.cpp:150-560) for the
// subset described at the top of this file
void load(const JVal& root, SceneBuild& b) {
    build_lookup(section(root, "Primitives", true), "Primitives", b.prims);
    build_lookup(section(root, "Materials", true), "Materials", b.mats);
    build_lookup(section(root, "Lights", true), "Lights", b.lights);
    build_lookup(section(root, "Cameras", true), "Cameras", b.cams);
    build_lookup(section(root, "Accelerators", true), "Accelerators", b.accels);
    build_lookup(section(root, "Transforms", true), "Transforms", b.xforms);
    build_lookup(section(root, "Mediums", true), "Mediums", b.media);
    const JVal* tex = root.get("Textures");
    if (tex && tex->is_arr() && !tex->a.empty())
        throw LoadError{MRB_E_UNSUPPORTED, "textures"};
    // the base medium first: it is medium 0 unless a material named it before
    b.baseMedium = b.medium(uid(section(root, "BaseMedium", true), "BaseMedium"));
    if (const JVal* bl = root.get("BaseBoundaryLight")) {
        const NodeRef& r = b.find(b.lights, uid(bl, "BaseBoundaryLight"), "light");
        if (node_type(r) != "Null")
            throw LoadError{MRB_E_UNSUPPORTED, "boundary light '" + node_type(r) + "' (Null only)"};
    }
    // Surfaces (SceneIO::LoadSurface, RayLib/SceneIO.cpp:78-140)
    const JVal* surfs = section(root, "Surfaces", true);
    if (!surfs->is_arr()) throw LoadError{MRB_E_ARG, "Surfaces must be an array"};
    for (const JVal& sn : surfs->a) {
        uint32_t tr, acc;
        const JVal *mv, *pv;
        bool sorted = false;
        if (sn.is_arr()) {
            if (sn.a.size() < 4) throw LoadError{MRB_E_ARG, "surface array needs 4 entries"};
            tr = uid(&sn.a[0], "transform");
            acc = uid(&sn.a[1], "accelerator");
            mv = &sn.a[2];
            pv = &sn.a[3];
        } else {
            tr = uid(sn.get("transform"), "transform");
            acc = uid(sn.get("accelerator"), "accelerator");
            mv = sn.get("material");
            pv = sn.get("primitive");
            sorted = true;
        }
        b.find(b.accels, acc, "accelerator");
        std::vector<std::pair<uint32_t, uint32_t>> pairs;  // (material, primitive)
        if (mv && mv->is_arr()) {
            if (!pv || !pv->is_arr() || pv->a.size() != mv->a.size())
                throw LoadError{MRB_E_ARG, "surface: material and primitive lists differ in size"};
            for (size_t i = 0; i < mv->a.size(); i++)
                pairs.push_back({uid(&mv->a[i], "material"), uid(&pv->a[i], "primitive")});
        } else {
            pairs.push_back({uid(mv, "material"), uid(pv, "primitive")});
        }
        if (sorted) std::sort(pairs.begin(), pairs.end());
        const Mat4 M = transform_of(b.xforms, tr);
        for (const auto& mp : pairs) b.primitive(mp.second, M, b.material(mp.first));
    }
    // LightSurfaces (SceneIO::LoadLightSurface, RayLib/SceneIO.cpp:142-193)
    if (const JVal* ls = root.get("LightSurfaces")) {
        if (!ls->is_arr()) throw LoadError{MRB_E_ARG, "LightSurfaces must be an array"};
        for (const JVal& ln : ls->a) {
            const uint32_t lid = uid(ln.get("light"), "light");
            const NodeRef& r = b.find(b.lights, lid, "light");
            const std::string type = node_type(r);
            if (type == "Null") continue;
            if (type != "Primitive")
                throw LoadError{MRB_E_UNSUPPORTED, "light type '" + type + "' (primitive lights only)"};
            const Mat4 M = ln.get("transform") ? transform_of(b.xforms, uid(ln.get("transform"), "transform"))
                                               : Mat4::identity();
            b.find(b.accels, uid(field(r, "accelerator"), "accelerator"), "accelerator");
            b.primitive(uid(field(r, "primitive"), "primitive"), M, b.light_material(lid, r));
        }
    }
    // CameraSurfaces (SceneIO::LoadCameraSurface, RayLib/SceneIO.cpp:195-222)
    if (const JVal* cs = root.get("CameraSurfaces")) {
        if (!cs->is_arr()) throw LoadError{MRB_E_ARG, "CameraSurfaces must be an array"};
        for (const JVal& cn : cs->a) {
            const NodeRef& r = b.find(b.cams, uid(cn.get("camera"), "camera"), "camera");
            const Mat4 M = cn.get("transform") ? transform_of(b.xforms, uid(cn.get("transform"), "transform"))
                                               : Mat4::identity();
            b.cameras.push_back(pinhole(r, M));
        }
    }
    if (b.idx.empty()) throw LoadError{MRB_E_ARG, "scene has no triangles"};
}

}  // namespace
}  // namespace mrb

struct mrb_json_scene {
    mrb::SceneBuild b;
};

extern "C" {

int mrb_json_scene_load(const char* text, size_t length, mrb_json_scene** out) {
    if (!text || !out) {
        mrb::set_error("mrb_json_scene_load: missing argument");
        return MRB_E_ARG;
    }
    *out = nullptr;
    mrb::JVal root;
    mrb::JParser ps{text, text + length, std::string(), 1};
    if (!ps.parse(root)) {
        mrb::set_error("scene JSON: %s", ps.err.c_str());
        return MRB_E_ARG;
    }
    if (root.kind != mrb::JVal::Obj) {
        mrb::set_error("scene JSON: the top level must be an object");
        return MRB_E_ARG;
    }
    std::unique_ptr<mrb_json_scene> js(new mrb_json_scene());
    try {
        mrb::load(root, js->b);
    } catch (const mrb::LoadError& e) {
        mrb::set_error("scene JSON: %s", e.msg.c_str());
        return e.code;
    } catch (const std::exception& e) {
        mrb::set_error("scene JSON: %s", e.what());
        return MRB_E_ARG;
    }
    *out = js.release();
    return 0;
}

int mrb_json_scene_load_file(const char* path, mrb_json_scene** out) {
    if (!path || !out) {
        mrb::set_error("mrb_json_scene_load_file: missing argument");
        return MRB_E_ARG;
    }
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        mrb::set_error("scene JSON: cannot open '%s'", path);
        return MRB_E_ARG;
    }
    std::string text;
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    std::fclose(f);
    return mrb_json_scene_load(text.data(), text.size(), out);
}

void mrb_json_scene_destroy(mrb_json_scene* js) { delete js; }

int mrb_json_scene_get(const mrb_json_scene* js, mrb_scene_desc* desc, uint32_t* camera_count) {
    if (!js) return MRB_E_ARG;
    const mrb::SceneBuild& b = js->b;
    if (desc) {
        desc->vertex_count = static_cast<uint32_t>(b.pos.size() / 3);
        desc->triangle_count = static_cast<uint32_t>(b.idx.size() / 3);
        desc->positions = b.pos.data();
        desc->normals = b.nrm.data();
        desc->uvs = b.uv.data();
        desc->indices = b.idx.data();
        desc->tri_material = b.triMat.data();
        desc->tri_cull = b.cull.data();
        desc->material_count = static_cast<uint32_t>(b.materials.size());
        desc->materials = b.materials.data();
        desc->medium_count = static_cast<uint32_t>(b.mediumIor.size());
        desc->medium_ior = b.mediumIor.data();
        desc->base_medium = b.baseMedium;
    }
    if (camera_count) *camera_count = static_cast<uint32_t>(b.cameras.size());
    return 0;
}

int mrb_json_scene_camera(const mrb_json_scene* js, uint32_t index, mrb_camera* cam) {
    if (!js || !cam) return MRB_E_ARG;
    if (index >= js->b.cameras.size()) {
        mrb::set_error("scene JSON: camera %u of %zu", index, js->b.cameras.size());
        return MRB_E_ARG;
    }
    *cam = js->b.cameras[index];
    return 0;
}

}  // extern "C"
