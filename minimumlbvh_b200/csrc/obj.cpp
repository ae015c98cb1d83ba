// OBJ / MTL reader for the path tracer's input (host code, no reference
// counterpart in this repository's dependencies: the reference reads its scene
// with a third-party OBJ library, main_gpu.cpp:209-282). It produces what the
// reference's loop produces from that library's output: one Triangle per
// triangle (minimum_lbvh.h:207-210) and one TriangleAttrib (main_gpu.cu:10-15)
// with the corner normals, reflectance = the material's Kd and emissive = its
// Ke, or reflectance 0.5 and no emission for faces without a material.
//
// Supported: `v`, `vn`, `vt` (ignored), `f` with `v`, `v/vt`, `v//vn`,
// `v/vt/vn` corners and negative (relative) indices, `mtllib`, `usemtl`,
// `newmtl` / `Kd` / `Ke` in the material library; other statements are
// skipped. A face of four corners is split along its shorter diagonal, a face
// of more corners into a fan around its first corner. Corners without a
// normal get a zero shading normal (the reference's shaders do not read them).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "capi_internal.h"

struct mlbvh_obj_mesh {
    std::vector<mlbvh_triangle> tris;
    std::vector<mlbvh_triangle_attrib> attribs;
};

namespace mlbvh {

namespace {

struct Material {
    float kd[3] = {0.5f, 0.5f, 0.5f};
    float ke[3] = {0.0f, 0.0f, 0.0f};
    bool known = false;
};

struct Corner {
    long v = 0, n = 0;  // 1-based after resolution, 0 = none
};

std::string dirname_of(const std::string& p)
{
    const size_t s = p.find_last_of("/\\");
    return s == std::string::npos ? std::string() : p.substr(0, s + 1);
}

std::string trim(const std::string& s)
{
    size_t a = 0, b = s.size();
    while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r')) ++a;
    while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r')) --b;
    return s.substr(a, b - a);
}

bool read_lines(const std::string& path, std::vector<std::string>& lines)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::string cur;
    char buf[65536];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0)
        for (size_t i = 0; i < got; ++i) {
            if (buf[i] == '\n') {
                lines.push_back(cur);
                cur.clear();
            } else {
                cur.push_back(buf[i]);
            }
        }
    if (!cur.empty()) lines.push_back(cur);
    std::fclose(f);
    return true;
}

void read_mtl(const std::string& path, std::map<std::string, Material>& mats)
{
    std::vector<std::string> lines;
    if (!read_lines(path, lines)) return;  // a missing library leaves faces at the default material
    Material* cur = nullptr;
    for (const std::string& raw : lines) {
        const std::string l = trim(raw);
        if (l.empty() || l[0] == '#') continue;
        if (l.compare(0, 7, "newmtl ") == 0) {
            cur = &mats[trim(l.substr(7))];
            cur->known = true;
        } else if (cur && (l.compare(0, 3, "Kd ") == 0 || l.compare(0, 3, "Ke ") == 0)) {
            float* dst = l[1] == 'd' ? cur->kd : cur->ke;
            float x = 0, y = 0, z = 0;
            const int k = std::sscanf(l.c_str() + 3, "%f %f %f", &x, &y, &z);
            if (k >= 1) dst[0] = dst[1] = dst[2] = x;  // one value: grey
            if (k == 3) {
                dst[1] = y;
                dst[2] = z;
            }
        }
    }
}

// 1-based index of corner token component (negative: relative to `count`).
long resolve(long i, size_t count) { return i < 0 ? (long)count + i + 1 : i; }

bool parse_corner(const char* tok, size_t nv, size_t nn, Corner& c)
{
    long v = 0, t = 0, n = 0;
    const char* p = tok;
    char* end = nullptr;
    v = std::strtol(p, &end, 10);
    if (end == p) return false;
    p = end;
    if (*p == '/') {
        ++p;
        if (*p != '/') {
            t = std::strtol(p, &end, 10);
            p = end;
        }
        if (*p == '/') {
            ++p;
            n = std::strtol(p, &end, 10);
            p = end;
        }
    }
    (void)t;
    c.v = resolve(v, nv);
    c.n = n ? resolve(n, nn) : 0;
    return c.v >= 1 && (size_t)c.v <= nv && c.n >= 0 && (size_t)c.n <= nn;
}

}  // namespace

mlbvh_status obj_load(const char* path, mlbvh_obj_mesh** out)
{
    if (!path || !out) return fail(MLBVH_ERR_INVALID_ARG, "null path or output pointer");
    *out = nullptr;
    std::vector<std::string> lines;
    if (!read_lines(path, lines)) return fail(MLBVH_ERR_INVALID_ARG, "cannot open the OBJ file");
    const std::string dir = dirname_of(path);
    std::map<std::string, Material> mats;
    std::vector<float> pos, nrm;
    const Material fallback;
    const Material* mat = &fallback;
    mlbvh_obj_mesh* m = new mlbvh_obj_mesh;
    std::vector<Corner> face;
    char tok[256];
    for (size_t li = 0; li < lines.size(); ++li) {
        const std::string l = trim(lines[li]);
        if (l.size() < 2 || l[0] == '#') continue;
        if (l[0] == 'v' && l[1] == ' ') {
            float x = 0, y = 0, z = 0;
            std::sscanf(l.c_str() + 2, "%f %f %f", &x, &y, &z);
            pos.insert(pos.end(), {x, y, z});
        } else if (l[0] == 'v' && l[1] == 'n') {
            float x = 0, y = 0, z = 0;
            std::sscanf(l.c_str() + 3, "%f %f %f", &x, &y, &z);
            nrm.insert(nrm.end(), {x, y, z});
        } else if (l.compare(0, 7, "mtllib ") == 0) {
            read_mtl(dir + trim(l.substr(7)), mats);
        } else if (l.compare(0, 7, "usemtl ") == 0) {
            auto it = mats.find(trim(l.substr(7)));
            mat = it != mats.end() && it->second.known ? &it->second : &fallback;
        } else if (l[0] == 'f' && l[1] == ' ') {
            face.clear();
            const char* p = l.c_str() + 2;
            int used = 0;
            while (std::sscanf(p, "%255s%n", tok, &used) == 1) {
                Corner c;
                if (!parse_corner(tok, pos.size() / 3, nrm.size() / 3, c)) {
                    delete m;
                    char msg[96];
                    std::snprintf(msg, sizeof(msg), "bad face corner on OBJ line %zu", li + 1);
                    return fail(MLBVH_ERR_INVALID_ARG, msg);
                }
                face.push_back(c);
                p += used;
            }
            if (face.size() < 3) continue;
            auto corner_pos = [&](const Corner& c, int a) { return pos[3 * (c.v - 1) + a]; };
            auto emit = [&](int a, int b, int c) {
                const Corner* cs[3] = {&face[a], &face[b], &face[c]};
                mlbvh_triangle t;
                mlbvh_triangle_attrib at;
                for (int k = 0; k < 3; ++k)
                    for (int d = 0; d < 3; ++d) {
                        t.vs[k][d] = corner_pos(*cs[k], d);
                        at.shadingNormals[k][d] = cs[k]->n ? nrm[3 * (cs[k]->n - 1) + d] : 0.0f;
                    }
                for (int d = 0; d < 3; ++d) {
                    at.reflectance[d] = mat->kd[d];
                    at.emissive[d] = mat->ke[d];
                }
                m->tris.push_back(t);
                m->attribs.push_back(at);
            };
            if (face.size() == 4) {
                // the shorter diagonal: |v2 - v0| against |v3 - v1|
                double d02 = 0, d13 = 0;
                for (int a = 0; a < 3; ++a) {
                    const double x = (double)corner_pos(face[2], a) - corner_pos(face[0], a);
                    const double y = (double)corner_pos(face[3], a) - corner_pos(face[1], a);
                    d02 += x * x;
                    d13 += y * y;
                }
                if (d02 <= d13) {
                    emit(0, 1, 2);
                    emit(0, 2, 3);
                } else {
                    emit(0, 1, 3);
                    emit(1, 2, 3);
                }
            } else {
                for (size_t k = 1; k + 1 < face.size(); ++k) emit(0, (int)k, (int)k + 1);
            }
        }
    }
    *out = m;
    return MLBVH_OK;
}

}  // namespace mlbvh

using namespace mlbvh;

extern "C" {

mlbvh_status mlbvh_obj_load(const char* path, mlbvh_obj_mesh** mesh)
{
    clear_error();
    return obj_load(path, mesh);
}

uint32_t mlbvh_obj_triangle_count(const mlbvh_obj_mesh* mesh) { return mesh ? (uint32_t)mesh->tris.size() : 0u; }

const mlbvh_triangle* mlbvh_obj_triangles(const mlbvh_obj_mesh* mesh)
{
    return mesh && !mesh->tris.empty() ? mesh->tris.data() : nullptr;
}

const mlbvh_triangle_attrib* mlbvh_obj_attribs(const mlbvh_obj_mesh* mesh)
{
    return mesh && !mesh->attribs.empty() ? mesh->attribs.data() : nullptr;
}

void mlbvh_obj_free(mlbvh_obj_mesh* mesh) { delete mesh; }

}  // extern "C"
