// Wavefront OBJ meshes for the scene description: the reference's importer semantics
// (src/io/obj_importer.cpp: `v`, `vt`, `vn`, `f` records, 1-based and negative indices, fan
// triangulation of polygons, one vertex per distinct (position, uv, normal) corner, normals kept
// only when every vertex has a non-zero one) followed by TriangleMesh::toPrimitives
// (src/geometry/mesh.cpp:14-38) as flat arrays: 9 floats of vertices per triangle and, with
// normals, 9 floats of normals made unit as the Triangle constructor does
// (include/render/geometry/triangle.h:28-33).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <new>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "rbr_b200.h"

struct rbr_mesh {
    std::vector<float> vertices;  // 9 per triangle
    std::vector<float> normals;   // 9 per triangle, or empty
};

namespace {

struct P3 {
    float x, y, z;
};

// 1-based or negative (relative to the end) OBJ index -> 0-based, -1 when absent or invalid.
int resolve(int idx, size_t count) {
    if (idx > 0) return idx <= static_cast<int>(count) ? idx - 1 : -1;
    if (idx < 0) {
        const int r = static_cast<int>(count) + idx;
        return r >= 0 ? r : -1;
    }
    return -1;
}

// "v", "v/vt", "v//vn" or "v/vt/vn"
void corner(const std::string& tok, int& v, int& vt, int& vn) {
    v = vt = vn = 0;
    const size_t a = tok.find('/');
    v = std::atoi(tok.substr(0, a).c_str());
    if (a == std::string::npos) return;
    const size_t b = tok.find('/', a + 1);
    const std::string t = tok.substr(a + 1, b == std::string::npos ? std::string::npos : b - a - 1);
    if (!t.empty()) vt = std::atoi(t.c_str());
    if (b != std::string::npos) {
        const std::string n = tok.substr(b + 1);
        if (!n.empty()) vn = std::atoi(n.c_str());
    }
}

// Vec3::normalized: v * (1 / length), zero for a zero vector.
P3 unit(P3 v) {
    const float len = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    if (!(len > 0.0f)) return P3{0.0f, 0.0f, 0.0f};
    const float inv = 1.0f / len;
    return P3{v.x * inv, v.y * inv, v.z * inv};
}

rbr_status parse(const std::string& text, rbr_mesh& mesh, std::string& err) {
    std::vector<P3> pos, nrm;
    size_t nuv = 0;
    std::map<std::tuple<int, int, int>, int> cache;
    std::vector<P3> vpos, vnrm;
    std::vector<int> index;
    bool any_normals = false;
    auto emit = [&](int v, int vt, int vn) {
        const auto key = std::make_tuple(v, vt, vn);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
        const int i = static_cast<int>(vpos.size());
        vpos.push_back(pos[v]);
        vnrm.push_back(vn >= 0 ? nrm[vn] : P3{0.0f, 0.0f, 0.0f});
        any_normals = any_normals || vn >= 0;
        cache[key] = i;
        return i;
    };
    std::istringstream in(text);
    std::string line;
    int lineno = 0;
    while (std::getline(in, line)) {
        ++lineno;
        std::istringstream ls(line);
        std::string tag;
        if (!(ls >> tag) || tag[0] == '#') continue;
        if (tag == "v" || tag == "vn") {
            float x, y, z;
            if (ls >> x >> y >> z) (tag == "v" ? pos : nrm).push_back(P3{x, y, z});
        } else if (tag == "vt") {
            float u;
            if (ls >> u) ++nuv;
        } else if (tag == "f") {
            std::vector<int> c;
            std::string tok;
            while (ls >> tok) {
                int v, vt, vn;
                corner(tok, v, vt, vn);
                const int pi = resolve(v, pos.size());
                if (pi < 0) {
                    err = "invalid vertex index on line " + std::to_string(lineno);
                    return RBR_ERR_INVALID_ARGUMENT;
                }
                c.push_back(emit(pi, resolve(vt, nuv), resolve(vn, nrm.size())));
            }
            for (size_t i = 1; i + 1 < c.size(); ++i) {
                index.push_back(c[0]);
                index.push_back(c[i]);
                index.push_back(c[i + 1]);
            }
        }
    }
    if (index.empty()) {
        err = "no faces";
        return RBR_ERR_INVALID_ARGUMENT;
    }
    bool normals = any_normals;
    for (const P3& n : vnrm)
        if (normals && n.x * n.x + n.y * n.y + n.z * n.z == 0.0f) normals = false;
    mesh.vertices.resize(index.size() * 3);
    if (normals) mesh.normals.resize(index.size() * 3);
    for (size_t k = 0; k < index.size(); ++k) {
        const P3 p = vpos[index[k]];
        mesh.vertices[3 * k] = p.x;
        mesh.vertices[3 * k + 1] = p.y;
        mesh.vertices[3 * k + 2] = p.z;
        if (normals) {
            const P3 n = unit(vnrm[index[k]]);
            mesh.normals[3 * k] = n.x;
            mesh.normals[3 * k + 1] = n.y;
            mesh.normals[3 * k + 2] = n.z;
        }
    }
    return RBR_OK;
}

void put_error(const std::string& e, char* buf, size_t len) {
    if (!buf || !len) return;
    std::strncpy(buf, e.c_str(), len - 1);
    buf[len - 1] = '\0';
}

rbr_status finish(rbr_status st, rbr_mesh* m, rbr_mesh** out, const std::string& err, char* ebuf, size_t elen) {
    if (st != RBR_OK) {
        delete m;
        put_error(err, ebuf, elen);
        return st;
    }
    *out = m;
    return RBR_OK;
}

}  // namespace

extern "C" {

rbr_status rbr_mesh_parse_obj(const char* text, size_t length, rbr_mesh** out, char* error, size_t error_len) {
    if (!text || !out) return RBR_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    rbr_mesh* m = new (std::nothrow) rbr_mesh();
    if (!m) return RBR_ERR_OUT_OF_MEMORY;
    std::string err;
    const rbr_status st = parse(std::string(text, length), *m, err);
    return finish(st, m, out, err, error, error_len);
}

rbr_status rbr_mesh_load_obj(const char* path, rbr_mesh** out, char* error, size_t error_len) {
    if (!path || !out) return RBR_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::ifstream f(path);
    if (!f.is_open()) {
        put_error(std::string("could not open OBJ file: ") + path, error, error_len);
        return RBR_ERR_INVALID_ARGUMENT;
    }
    std::stringstream buf;
    buf << f.rdbuf();
    const std::string text = buf.str();
    return rbr_mesh_parse_obj(text.data(), text.size(), out, error, error_len);
}

uint32_t rbr_mesh_triangles(const rbr_mesh* m) { return m ? static_cast<uint32_t>(m->vertices.size() / 9) : 0; }
const float* rbr_mesh_triangle_vertices(const rbr_mesh* m) { return m ? m->vertices.data() : nullptr; }
const float* rbr_mesh_triangle_normals(const rbr_mesh* m) {
    return (m && !m->normals.empty()) ? m->normals.data() : nullptr;
}
void rbr_mesh_destroy(rbr_mesh* m) { delete m; }

}  // extern "C"
