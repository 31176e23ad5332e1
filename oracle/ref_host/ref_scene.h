// ref_scene.h -- the reference's own scene objects built from a triangle soup.
//
// TEST INFRASTRUCTURE ONLY.  Shared by the two host harnesses (ref_driver.cu,
// the render / gather / OBJ pins; ref_trace.cu, the photon-tracer pin).  Both
// include the reference sources before this file.  One Model per model index
// (CPM/Initializer.cu:11-16 assigns model ids in model order), built with the
// reference's ModelConstructInfo / Model / AABB constructors; the light is the
// reference's LightSource owned by the light model.
#pragma once
#include <vector>

namespace ref_host {

struct HostScene {
    std::vector<cpm::vec3*> pos, nrm;
    std::vector<Model> models;
    LightSource light;
    Camera camera;
    ~HostScene() {
        for (auto p : pos) delete[] p;
        for (auto p : nrm) delete[] p;
    }
};

inline cpm::vec3 V(const float* p) { return cpm::vec3(p[0], p[1], p[2]); }

// Triangle soup sorted by model: 9 floats of positions and of normals per
// triangle, tri_model[t] = model index; mats = 12 floats per model (diffuse3,
// specular3, emission3, ior, opaque, shininess).
inline HostScene* make_scene(int ntri, const float* pos, const float* nrm, const int* tri_model, int nmodel,
                             const float* mats, int light_model, const float* light_intensity) {
    HostScene* s = new HostScene();
    s->models.reserve(nmodel);
    for (int m = 0; m < nmodel; m++) {
        int first = -1, count = 0;
        for (int t = 0; t < ntri; t++) if (tri_model[t] == m) { if (first < 0) first = t; count++; }
        cpm::vec3* P = new cpm::vec3[3 * count];
        cpm::vec3* N = new cpm::vec3[3 * count];
        for (int i = 0; i < 3 * count; i++) { P[i] = V(pos + 9 * first + 3 * i); N[i] = V(nrm + 9 * first + 3 * i); }
        s->pos.push_back(P); s->nrm.push_back(N);
        ModelConstructInfo mci;
        mci.positions = P; mci.normals = N; mci.texcoords = nullptr;
        mci.size = 3 * count; mci.primitives_size = count; mci.type = ModelType::Triangle; mci.smooth = false;
        const float* q = mats + 12 * m;
        Material mat;
        mat.diffuse = V(q); mat.specular = V(q + 3); mat.emission = V(q + 6);
        mat.refr_index = q[9]; mat.opaque = q[10]; mat.shininess = q[11];
        mci.material = mat;
        AABB box(P, 3 * count);
        s->models.push_back(Model(mci, m, box));
    }
    s->light = LightSource();
    s->light.intensity = V(light_intensity);
    s->light.model_owner = &s->models[light_model];
    return s;
}

}  // namespace ref_host
