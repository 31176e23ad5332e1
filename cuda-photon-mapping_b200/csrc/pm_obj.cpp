// pm_obj.cpp -- OBJ / MTL scene import into pm_scene_desc.
//
// Model, material and light semantics follow the reference's loader and
// initializer (CudaPhotonMapping/ObjLoader.cpp:18-320, Initializer.cu:62-100):
//   * a model is a run of consecutive face lines; the first line after a face
//     line that is not itself a face line closes it (a blank or comment line
//     included, ObjLoader.cpp:169-185);
//   * its name is the last 'g' / 'o' name seen (initially "n1"); a name already
//     taken gets '1' appended, and the appended name carries on (:173-176);
//   * its material is the one the last 'usemtl' selected, carried across
//     models until the next 'usemtl' (:181-183, :207-216): Material()'s
//     defaults (diffuse 1, specular 1, emission 0, shininess 16, index 1,
//     opaque 1; Material.cuh:4-31) overridden by the first 'newmtl' block of
//     that name in the 'mtllib' file: Kd, Ks, Ke, Ns, Ni, d (opaque) and Tr
//     (opaque = 1 - Tr), later lines winning (ObjLoader.cpp:4-87);
//   * vertex indices are 1-based, negative ones count back from the end
//     (:103-121);
//   * a quad (v0 v1 v2 v3) is the triangles (v0 v1 v3), (v1 v2 v3), in that
//     order, as the reference intersects it (Model.cuh:400-423);
//   * the light is the model named "light" (Initializer.cu:70), intensity 1.
// Where the reference loader is undefined or wrong this one follows the OBJ
// format instead: position-only faces ("f 1 2 3") and faces with texture
// indices parse correctly (the reference assigns their indices by a running
// counter), faces without normals get the triangle's flat normal (the
// reference leaves them uninitialised), faces of more than 4 vertices become
// a fan (the reference cannot intersect them), a model may mix triangles and
// quads (the reference takes the last face's size for all), and a line of
// whitespace only counts as blank (the reference re-applies the previous
// line's keyword to it).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/pm_api.h"

struct pm_obj_scene {
    std::vector<float> pos, nrm, mats;   // 9 + 9 floats per triangle, 12 per model
    std::vector<int32_t> model;          // per triangle
    std::vector<std::string> names;      // per model
    int32_t light = -1;
};

namespace {

struct Mat {
    float kd[3] = {1.f, 1.f, 1.f}, ks[3] = {1.f, 1.f, 1.f}, ke[3] = {0.f, 0.f, 0.f};
    float ior = 1.f, opaque = 1.f, shininess = 16.f;
};

void set_err(char* err, int len, const std::string& msg) {
    if (err && len > 0) {
        std::snprintf(err, (size_t)len, "%s", msg.c_str());
    }
}

std::string join(const std::string& dir, const std::string& f) { return dir.empty() ? f : dir + "/" + f; }

void strip_cr(std::string& s) {
    while (!s.empty() && (s.back() == '\r' || s.back() == '\n')) s.pop_back();
}

bool read3(std::istringstream& ss, float* v) { return static_cast<bool>(ss >> v[0] >> v[1] >> v[2]); }

// the first 'newmtl name' block of the file; false when the file cannot be read
bool load_material(const std::string& path, const std::string& name, Mat& m) {
    std::ifstream f(path);
    if (!f.is_open()) return false;
    std::string line, key;
    bool in = false;
    while (std::getline(f, line)) {
        strip_cr(line);
        std::istringstream ss(line);
        if (!(ss >> key)) continue;
        if (key == "newmtl") {
            if (in) break;
            std::string n;
            ss >> n;
            in = n == name;
            continue;
        }
        if (!in) continue;
        float v[3], x;
        if (key == "Kd" && read3(ss, v)) std::memcpy(m.kd, v, sizeof v);
        else if (key == "Ks" && read3(ss, v)) std::memcpy(m.ks, v, sizeof v);
        else if (key == "Ke" && read3(ss, v)) std::memcpy(m.ke, v, sizeof v);
        else if (key == "d" && (ss >> x)) m.opaque = x;
        else if (key == "Tr" && (ss >> x)) m.opaque = 1.f - x;
        else if (key == "Ns" && (ss >> x)) m.shininess = x;
        else if (key == "Ni" && (ss >> x)) m.ior = x;
    }
    return true;
}

// "a", "a/b", "a//c", "a/b/c" -> position and normal index (0: absent)
bool parse_vertex(const std::string& tok, long& vp, long& vn) {
    vp = 0;
    vn = 0;
    const char* s = tok.c_str();
    char* end = nullptr;
    vp = std::strtol(s, &end, 10);
    if (end == s) return false;
    if (*end == 0) return true;
    if (*end != '/') return false;
    s = end + 1;
    if (*s != '/') {   // texture index: parsed and ignored
        std::strtol(s, &end, 10);
        if (end == s) return false;
        s = end;
        if (*s == 0) return true;
        if (*s != '/') return false;
    }
    s++;
    if (*s == 0) return true;
    vn = std::strtol(s, &end, 10);
    return end != s && *end == 0;
}

bool resolve(long idx, size_t count, size_t& out) {
    long r = idx > 0 ? idx - 1 : (long)count + idx;
    if (idx == 0 || r < 0 || (size_t)r >= count) return false;
    out = (size_t)r;
    return true;
}

}  // namespace

extern "C" {

int pm_obj_load(const char* dir, const char* file, pm_obj_scene** out, char* err, int err_len) {
    if (!file || !out) return PM_ERR_INVALID;
    *out = nullptr;
    const std::string d = dir ? dir : "";
    std::ifstream f(join(d, file));
    if (!f.is_open()) {
        set_err(err, err_len, "cannot open " + join(d, file));
        return PM_ERR_IO;
    }
    pm_obj_scene* S = new pm_obj_scene();
    std::vector<float> vpos, vnrm;
    std::string mtllib, name = "n1", line, key;
    std::set<std::string> taken;
    Mat mat;
    bool in_faces = false;
    size_t tri_start = 0;
    long lineno = 0;
    auto fail = [&](int code, const std::string& msg) {
        set_err(err, err_len, join(d, file) + ":" + std::to_string(lineno) + ": " + msg);
        delete S;
        return code;
    };
    auto close_model = [&]() {
        const int32_t m = (int32_t)S->names.size();
        if (taken.count(name)) name += '1';
        taken.insert(name);
        S->names.push_back(name);
        const float mm[12] = {mat.kd[0], mat.kd[1], mat.kd[2], mat.ks[0], mat.ks[1], mat.ks[2],
                              mat.ke[0], mat.ke[1], mat.ke[2], mat.ior, mat.opaque, mat.shininess};
        S->mats.insert(S->mats.end(), mm, mm + 12);
        for (size_t t = tri_start; t < S->model.size(); t++) S->model[t] = m;
        tri_start = S->model.size();
        in_faces = false;
    };
    while (std::getline(f, line)) {
        lineno++;
        strip_cr(line);
        std::istringstream ss(line);
        if (!(ss >> key)) key.clear();
        if (in_faces && key != "f") close_model();
        if (key == "mtllib") {
            ss >> mtllib;
        } else if (key == "g" || key == "o") {
            std::string n;
            if (ss >> n) name = n;
        } else if (key == "usemtl") {
            std::string n;
            ss >> n;
            mat = Mat();
            if (!load_material(join(d, mtllib), n, mat)) return fail(PM_ERR_IO, "cannot open material file " + mtllib);
        } else if (key == "v" || key == "vn") {
            float v[3];
            if (!read3(ss, v)) return fail(PM_ERR_INVALID, "expected three numbers");
            (key == "v" ? vpos : vnrm).insert((key == "v" ? vpos : vnrm).end(), v, v + 3);
        } else if (key == "f") {
            std::vector<size_t> ip, in;
            bool all_n = true;
            std::string tok;
            while (ss >> tok) {
                long a, c;
                size_t p, q = 0;
                if (!parse_vertex(tok, a, c)) return fail(PM_ERR_INVALID, "bad face vertex '" + tok + "'");
                if (!resolve(a, vpos.size() / 3, p)) return fail(PM_ERR_INVALID, "vertex index out of range");
                if (c != 0 && !resolve(c, vnrm.size() / 3, q)) return fail(PM_ERR_INVALID, "normal index out of range");
                ip.push_back(p);
                in.push_back(q);
                all_n = all_n && c != 0;
            }
            const size_t nv = ip.size();
            if (nv < 3) return fail(PM_ERR_INVALID, "a face needs at least 3 vertices");
            std::vector<int> corners;   // triangles as corner triples of this face
            if (nv == 4) corners = {0, 1, 3, 1, 2, 3};
            else for (size_t i = 1; i + 1 < nv; i++) corners.insert(corners.end(), {0, (int)i, (int)i + 1});
            for (size_t t = 0; t < corners.size(); t += 3) {
                const float* v[3];
                for (int k = 0; k < 3; k++) v[k] = &vpos[3 * ip[corners[t + k]]];
                float n[3] = {0.f, 0.f, 0.f};
                if (!all_n) {
                    const float e1[3] = {v[1][0] - v[0][0], v[1][1] - v[0][1], v[1][2] - v[0][2]};
                    const float e2[3] = {v[2][0] - v[0][0], v[2][1] - v[0][1], v[2][2] - v[0][2]};
                    n[0] = e1[1] * e2[2] - e1[2] * e2[1];
                    n[1] = e1[2] * e2[0] - e1[0] * e2[2];
                    n[2] = e1[0] * e2[1] - e1[1] * e2[0];
                    const float l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                    if (l > 0.f) for (float& x : n) x /= l;
                }
                for (int k = 0; k < 3; k++) {
                    S->pos.insert(S->pos.end(), v[k], v[k] + 3);
                    const float* nk = all_n ? &vnrm[3 * in[corners[t + k]]] : n;
                    S->nrm.insert(S->nrm.end(), nk, nk + 3);
                }
                S->model.push_back(-1);
            }
            in_faces = true;
        }
    }
    if (in_faces) close_model();
    if (S->model.empty()) return fail(PM_ERR_INVALID, "no faces");
    for (size_t m = 0; m < S->names.size(); m++)
        if (S->names[m] == "light") { S->light = (int32_t)m; break; }
    *out = S;
    return PM_OK;
}

int pm_obj_desc(const pm_obj_scene* s, float default_ior, pm_scene_desc* out) {
    if (!s || !out) return PM_ERR_INVALID;
    if (s->light < 0) return PM_ERR_INVALID;
    std::memset(out, 0, sizeof *out);
    out->ntri = (int32_t)s->model.size();
    out->tri_pos = s->pos.data();
    out->tri_nrm = s->nrm.data();
    out->tri_model = s->model.data();
    out->tri_diffuse = nullptr;
    out->nmodel = (int32_t)s->names.size();
    out->materials = s->mats.data();
    out->light_model = s->light;
    out->light_intensity[0] = out->light_intensity[1] = out->light_intensity[2] = 1.f;
    out->default_ior = default_ior;
    return PM_OK;
}

int32_t pm_obj_model_count(const pm_obj_scene* s) { return s ? (int32_t)s->names.size() : 0; }

const char* pm_obj_model_name(const pm_obj_scene* s, int32_t m) {
    if (!s || m < 0 || (size_t)m >= s->names.size()) return nullptr;
    return s->names[(size_t)m].c_str();
}

int32_t pm_obj_light_model(const pm_obj_scene* s) { return s ? s->light : -1; }

void pm_obj_free(pm_obj_scene* s) { delete s; }

}  // extern "C"
