// OBJ meshes for the reference's asset scenes (host code): lux_obj_load.
//
// Follows the reference's loader (util/obj_loader.cpp:636-1328) over its bundled parser's
// geometry (tinyobjloader 2.0, vendored as util/tiny_obj_loader.h, with its fast_float
// number parsing: numbers are read as correctly rounded doubles, then rounded to float,
// which strtod followed by a cast reproduces):
//   * faces are split into triangles on import: a quad (0,1,2,3) into (0,1,2),(0,2,3)
//     when |v2 - v0|^2 < |v3 - v1|^2, else (0,1,3),(1,2,3) (exportGroupsToShape); larger
//     polygons, which the reference's assets do not hold, become fans (the bundled
//     parser clips ears, so such faces may split differently);
//   * triangles with an out-of-range vertex index, a non-finite position or an area of at
//     most 1e-12 are skipped and counted;
//   * every (position, used normal, used texcoord) corner becomes one mesh vertex, in
//     first-use order; normals are the source normal (normalised) where it is finite and
//     nonzero, else the area-weighted sum of the faces at the position (smooth mode),
//     else zero;
//   * the placement is translate(target) * scale(s) * translate(-anchor) over the mesh
//     box (make_obj_placement_transform, :388-423).
// The arithmetic is written operation by operation as the reference's (float, no
// contraction on the host's baseline ISA).

#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/lux_gpu.h"

namespace lux {
int fail(int status, const std::string& message);
}

namespace {

struct P3 {
    float x, y, z;
};
P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
P3 cross(P3 a, P3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
float length2(P3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
P3 normalize(P3 v) {  // core/vec3.cuh normalize: v * (1 / length), zero kept
    float len = std::sqrt(length2(v));
    if (!(len > 0)) return v;
    float inv = 1.0f / len;
    return {v.x * inv, v.y * inv, v.z * inv};
}
bool finite(P3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }

struct Corner {
    int v, t, n;  // 0-based; -1 absent
};

struct Face {
    Corner c[3];
    int name;  // index into names, -1 for no usemtl
};

bool iprefix(const std::string& s, size_t at, const char* word) {
    size_t n = std::strlen(word);
    if (s.size() - at < n) return false;
    for (size_t i = 0; i < n; ++i)
        if (std::tolower(static_cast<unsigned char>(s[at + i])) != word[i]) return false;
    return true;
}

// One whitespace-delimited number (parseReal): a correctly rounded double, rounded to
// float; "nan" reads as 0 and "inf" / "infinity" as the largest double (infinite as a
// float), as the bundled parser maps them; missing or malformed fields read as fallback.
float read_real(const char*& p, const char* end, float fallback) {
    while (p < end && (*p == ' ' || *p == '\t')) ++p;
    const char* q = p;
    while (q < end && *q != ' ' && *q != '\t' && *q != '\r') ++q;
    float value = fallback;
    if (q > p) {
        std::string token(p, q);
        size_t at = token[0] == '+' || token[0] == '-' ? 1 : 0;
        if (iprefix(token, at, "nan")) {
            value = 0.0f;
        } else if (iprefix(token, at, "inf")) {
            const double big = token[0] == '-' ? -1.7976931348623157e308 : 1.7976931348623157e308;
            value = static_cast<float>(big);
        } else {
            char* stop = nullptr;
            double d = std::strtod(token.c_str(), &stop);
            if (stop != token.c_str()) value = static_cast<float>(d);
        }
    }
    p = q;
    return value;
}

// 1-based or negative (relative) index; 0 is invalid for positions.
bool fix_index(long idx, int count, int* out) {
    if (idx > 0) {
        *out = static_cast<int>(idx - 1);
        return true;
    }
    if (idx == 0) {
        *out = -1;
        return false;
    }
    *out = count + static_cast<int>(idx);
    return true;
}

bool parse_corner(const std::string& token, int nv, int nt, int nn, Corner* c) {
    c->v = c->t = c->n = -1;
    long field[3] = {0, 0, 0};
    bool present[3] = {false, false, false};
    size_t start = 0;
    for (int k = 0; k < 3 && start <= token.size(); ++k) {
        size_t slash = token.find('/', start);
        std::string part = token.substr(start, slash == std::string::npos ? std::string::npos
                                                                            : slash - start);
        if (!part.empty()) {
            field[k] = std::strtol(part.c_str(), nullptr, 10);
            present[k] = true;
        }
        if (slash == std::string::npos) break;
        start = slash + 1;
    }
    if (!present[0] || !fix_index(field[0], nv, &c->v)) return false;
    if (present[1]) fix_index(field[1], nt, &c->t);
    if (present[2]) fix_index(field[2], nn, &c->n);
    return true;
}

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return {};
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

bool keyword(const std::string& line, const char* kw, std::string* payload) {
    size_t n = std::strlen(kw);
    if (line.size() < n || line.compare(0, n, kw) != 0) return false;
    if (line.size() > n && line[n] != ' ' && line[n] != '\t') return false;
    *payload = line.size() > n ? trim(line.substr(n)) : std::string();
    return true;
}

struct CornerKey {
    int v, n, t;
    bool operator==(const CornerKey& o) const { return v == o.v && n == o.n && t == o.t; }
};
struct CornerHash {
    size_t operator()(const CornerKey& k) const {
        uint64_t h = static_cast<uint32_t>(k.v);
        h = h * 1099511628211ull ^ static_cast<uint32_t>(k.n);
        h = h * 1099511628211ull ^ static_cast<uint32_t>(k.t);
        return static_cast<size_t>(h);
    }
};

template <typename T>
T* copy_out(const std::vector<T>& v) {
    T* p = static_cast<T*>(std::malloc(sizeof(T) * (v.empty() ? 1 : v.size())));
    if (p && !v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

}  // namespace

extern "C" void lux_obj_mesh_free(lux_obj_mesh* m) {
    if (!m) return;
    std::free(m->vertices);
    std::free(m->normals);
    std::free(m->uvs);
    std::free(m->indices);
    std::free(m->material_ids);
    delete m;
}

extern "C" int lux_obj_load(const char* path, const lux_obj_options* opt, lux_obj_mesh** out) {
    if (!path || !opt || !out) return lux::fail(LUX_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (opt->normal_mode < 0 || opt->normal_mode > 2 || opt->scale_mode < 0 || opt->scale_mode > 2)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "unknown OBJ normal or scale mode");
    if (opt->binding_count < 0 || (opt->binding_count > 0 && (!opt->binding_names || !opt->binding_ids)))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "bad OBJ material bindings");
    if (opt->scale_mode != LUX_OBJ_SCALE_NONE && !(std::isfinite(opt->target_extent) && opt->target_extent > 0))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT,
                         "OBJ placement target_extent must be finite and positive when scaling is enabled");
    if (opt->ground_to_y && !std::isfinite(opt->target_y))
        return lux::fail(LUX_ERR_INVALID_ARGUMENT,
                         "OBJ placement target_y must be finite when grounding is enabled");
    std::ifstream file(path, std::ios::binary);
    if (!file) return lux::fail(LUX_ERR_INVALID_ARGUMENT, std::string("Cannot open OBJ file [") + path + "]");
    std::ostringstream text;
    text << file.rdbuf();
    const std::string src = text.str();

    std::unordered_map<std::string, int> bindings;
    for (int i = 0; i < opt->binding_count; ++i) bindings[opt->binding_names[i]] = opt->binding_ids[i];
    const bool bound = !bindings.empty();

    std::vector<P3> positions, normals;
    std::vector<float> texcoords;  // 2 per entry
    std::vector<Face> faces;
    std::vector<std::string> names;
    std::unordered_map<std::string, int> name_index;
    int current = -1;
    bool unnamed_face = false;

    std::istringstream lines(src);
    std::string raw;
    while (std::getline(lines, raw)) {
        size_t hash = raw.find('#');
        std::string line = trim(hash == std::string::npos ? raw : raw.substr(0, hash));
        if (line.empty()) continue;
        std::string payload;
        if (keyword(line, "v", &payload)) {
            const char* p = payload.c_str();
            const char* e = p + payload.size();
            P3 v;
            v.x = read_real(p, e, 0.0f);
            v.y = read_real(p, e, 0.0f);
            v.z = read_real(p, e, 0.0f);
            positions.push_back(v);
        } else if (keyword(line, "vn", &payload)) {
            const char* p = payload.c_str();
            const char* e = p + payload.size();
            P3 n;
            n.x = read_real(p, e, 0.0f);
            n.y = read_real(p, e, 0.0f);
            n.z = read_real(p, e, 0.0f);
            normals.push_back(n);
        } else if (keyword(line, "vt", &payload)) {
            const char* p = payload.c_str();
            const char* e = p + payload.size();
            texcoords.push_back(read_real(p, e, 0.0f));
            texcoords.push_back(read_real(p, e, 0.0f));
        } else if (keyword(line, "usemtl", &payload)) {
            if (payload.empty()) {
                current = -1;
                continue;
            }
            if (bound && !bindings.count(payload))
                return lux::fail(LUX_ERR_INVALID_ARGUMENT, "OBJ usemtl '" + payload + "' has no material binding");
            auto it = name_index.find(payload);
            if (it == name_index.end()) {
                it = name_index.emplace(payload, static_cast<int>(names.size())).first;
                names.push_back(payload);
            }
            current = it->second;
        } else if (keyword(line, "f", &payload)) {
            std::istringstream tokens(payload);
            std::vector<Corner> poly;
            std::string tok;
            const int nt = static_cast<int>(texcoords.size() / 2);
            while (tokens >> tok) {
                Corner c;
                if (!parse_corner(tok, static_cast<int>(positions.size()), nt,
                                  static_cast<int>(normals.size()), &c))
                    return lux::fail(LUX_ERR_INVALID_ARGUMENT, "Failed parse `f' line in OBJ file");
                poly.push_back(c);
            }
            if (poly.size() < 3) continue;
            if (current < 0) unnamed_face = true;
            if (poly.size() == 4) {
                for (const Corner& c : poly)
                    if (c.v < 0 || c.v >= static_cast<int>(positions.size()))
                        return lux::fail(LUX_ERR_INVALID_ARGUMENT, "OBJ face with invalid vertex index");
                const P3 v0 = positions[poly[0].v], v1 = positions[poly[1].v];
                const P3 v2 = positions[poly[2].v], v3 = positions[poly[3].v];
                const P3 e02 = sub(v2, v0), e13 = sub(v3, v1);
                if (length2(e02) < length2(e13)) {
                    faces.push_back(Face{{poly[0], poly[1], poly[2]}, current});
                    faces.push_back(Face{{poly[0], poly[2], poly[3]}, current});
                } else {
                    faces.push_back(Face{{poly[0], poly[1], poly[3]}, current});
                    faces.push_back(Face{{poly[1], poly[2], poly[3]}, current});
                }
            } else {
                for (size_t k = 1; k + 1 < poly.size(); ++k)
                    faces.push_back(Face{{poly[0], poly[k], poly[k + 1]}, current});
            }
        }
    }
    if (bound && opt->default_material < 0 && unnamed_face)
        return lux::fail(LUX_ERR_INVALID_ARGUMENT,
                         "OBJ face has no usemtl tag while material bindings are required");

    const int nv = static_cast<int>(positions.size());
    const int nn = static_cast<int>(normals.size());
    const int nt = static_cast<int>(texcoords.size() / 2);
    auto normal_usable = [&](int ni) {
        return ni >= 0 && ni < nn && finite(normals[ni]) && length2(normals[ni]) > 1e-20f;
    };
    auto texcoord_usable = [&](int ti) {
        return ti >= 0 && ti < nt && std::isfinite(texcoords[2 * ti]) &&
               std::isfinite(texcoords[2 * ti + 1]);
    };

    lux_obj_mesh* m = new (std::nothrow) lux_obj_mesh();
    if (!m) return lux::fail(LUX_ERR_OUT_OF_MEMORY, "OBJ mesh allocation failed");
    std::vector<Face> kept;
    std::vector<P3> smooth(opt->normal_mode == LUX_OBJ_NORMALS_SMOOTH ? nv : 0, P3{0, 0, 0});
    for (const Face& f : faces) {
        bool valid = true, fin = true;
        for (const Corner& c : f.c) valid = valid && c.v >= 0 && c.v < nv;
        if (!valid) {
            ++m->skipped_invalid;
            continue;
        }
        for (const Corner& c : f.c) fin = fin && finite(positions[c.v]);
        if (!fin) {
            ++m->skipped_nonfinite;
            continue;
        }
        const P3 v0 = positions[f.c[0].v], v1 = positions[f.c[1].v], v2 = positions[f.c[2].v];
        const P3 n = cross(sub(v1, v0), sub(v2, v0));
        if (0.5f * std::sqrt(length2(n)) <= 1e-12f) {  // triangle_area
            ++m->skipped_degenerate;
            continue;
        }
        if (opt->normal_mode == LUX_OBJ_NORMALS_SMOOTH) {
            for (const Corner& c : f.c) {
                P3& s = smooth[c.v];
                s = {s.x + n.x, s.y + n.y, s.z + n.z};
            }
        }
        Face g = f;
        if (opt->reverse_orientation) std::swap(g.c[1], g.c[2]);
        kept.push_back(g);
    }

    std::vector<float> verts, norms, uvs;
    std::vector<uint32_t> indices;
    std::vector<int32_t> mids;
    std::unordered_map<CornerKey, uint32_t, CornerHash> vertex_of;
    const float flip = opt->reverse_orientation ? -1.0f : 1.0f;
    auto corner_vertex = [&](const Corner& c) -> uint32_t {
        const bool use_n = opt->normal_mode != LUX_OBJ_NORMALS_FACE && normal_usable(c.n);
        const bool use_t = texcoord_usable(c.t);
        CornerKey key{c.v, use_n ? c.n : -1, use_t ? c.t : -1};
        auto it = vertex_of.find(key);
        if (it != vertex_of.end()) return it->second;
        const uint32_t index = static_cast<uint32_t>(verts.size() / 3);
        vertex_of.emplace(key, index);
        const P3 p = positions[c.v];
        verts.insert(verts.end(), {p.x, p.y, p.z});
        P3 nrm{0, 0, 0};
        if (opt->normal_mode != LUX_OBJ_NORMALS_FACE) {
            if (use_n) {
                nrm = normalize(normals[c.n]);
                nrm = {nrm.x * flip, nrm.y * flip, nrm.z * flip};
            } else if (opt->normal_mode == LUX_OBJ_NORMALS_SMOOTH && length2(smooth[c.v]) > 0) {
                nrm = normalize(smooth[c.v]);
                nrm = {nrm.x * flip, nrm.y * flip, nrm.z * flip};
            }
        }
        norms.insert(norms.end(), {nrm.x, nrm.y, nrm.z});
        float u = use_t ? texcoords[2 * c.t] : 0.0f, v = use_t ? texcoords[2 * c.t + 1] : 0.0f;
        if (use_t && opt->flip_texcoord_v) v = 1.0f - v;
        uvs.insert(uvs.end(), {u, v});
        return index;
    };
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (const Face& f : kept) {
        for (const Corner& c : f.c) {
            const uint32_t i = corner_vertex(c);
            indices.push_back(i);
            const float* p = &verts[3 * size_t(i)];
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::fmin(lo[a], p[a]);
                hi[a] = std::fmax(hi[a], p[a]);
            }
        }
        int material = opt->default_material;
        if (bound && f.name >= 0) material = bindings[names[f.name]];
        mids.push_back(material);
    }
    if (kept.empty()) {
        lux_obj_mesh_free(m);
        return LUX_OK;
    }

    // make_obj_placement_transform: s on the diagonal, translation target + s * -anchor.
    float s = 1.0f;
    const float ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    if (opt->scale_mode != LUX_OBJ_SCALE_NONE) {
        float source = opt->scale_mode == LUX_OBJ_SCALE_X_EXTENT
                           ? ext[0]
                           : std::fmax(ext[0], std::fmax(ext[1], ext[2]));
        if (source > 0) s = opt->target_extent / source;
    }
    float anchor[3] = {0, 0, 0}, target[3] = {0, 0, 0};
    if (opt->center_xz) {
        anchor[0] = (lo[0] + hi[0]) * 0.5f;
        anchor[2] = (lo[2] + hi[2]) * 0.5f;
    }
    if (opt->ground_to_y) {
        anchor[1] = lo[1];
        target[1] = opt->target_y;
    }
    std::memset(m->object_to_world, 0, sizeof(m->object_to_world));
    for (int r = 0; r < 3; ++r) {
        m->object_to_world[4 * r + r] = s;
        m->object_to_world[4 * r + 3] = s * -anchor[r] + target[r];
    }
    for (int a = 0; a < 3; ++a) {
        m->bounds[a] = lo[a];
        m->bounds[3 + a] = hi[a];
    }
    m->vertex_count = static_cast<int32_t>(verts.size() / 3);
    m->triangle_count = static_cast<int32_t>(kept.size());
    m->vertices = copy_out(verts);
    m->normals = copy_out(norms);
    m->uvs = copy_out(uvs);
    m->indices = copy_out(indices);
    m->material_ids = copy_out(mids);
    if (!m->vertices || !m->normals || !m->uvs || !m->indices || !m->material_ids) {
        lux_obj_mesh_free(m);
        return lux::fail(LUX_ERR_OUT_OF_MEMORY, "OBJ mesh allocation failed");
    }
    *out = m;
    return LUX_OK;
}
