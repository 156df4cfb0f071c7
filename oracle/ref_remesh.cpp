// oracle/ref_remesh.cpp -- plain C entry points over the reference's own CPU
// remeshers (kenji-tojo/diffsoup src/remesh.cpp TriangleSoupSplitter and
// src/remesh_clip.cpp TriangleSoupSplitterClip, compiled unmodified beside
// this file into oracle/_ref/libremesh_ref.so by oracle/Makefile).
//
// TEST INFRASTRUCTURE ONLY: the checker of the GPU remesher
// (diffsoup_b200/csrc/remesh.cu).  The calls mirror the reference's bindings
// (src/main.cpp:308-388): run the splitter, then read its sizes and arrays.
#include <cstring>

#include "remesh.h"
#include "remesh_clip.h"

namespace {

struct Result {
    int nv = 0, nt = 0;
    float* verts = nullptr;
    int* faces = nullptr;
    int* map = nullptr;
    int* flag = nullptr;
};

template <class Splitter>
Result* collect(Splitter& s) {
    Result* r = new Result;
    r->nv = s.getNumVertices();
    r->nt = s.getNumTriangles();
    r->verts = new float[(size_t)r->nv * 3];
    r->faces = new int[(size_t)r->nt * 3];
    r->map = new int[(size_t)r->nt];
    r->flag = new int[(size_t)r->nt];
    s.exportToFlatArrays(r->verts, r->faces);
    s.getFaceMapping(r->map);
    s.getSameAsOriginal(r->flag);
    return r;
}

}  // namespace

extern "C" {

// main.cpp:308-340: split_triangle_soup(verts, faces, numSplits, tau)
void* remref_split_world(const float* verts, const int* faces, int nv, int nt, int num_splits, float tau) {
    diffsoup::TriangleSoupSplitter s(verts, faces, nv, nt);
    s.splitLongEdges(num_splits, tau);
    return collect(s);
}

// main.cpp:342-388: split_triangle_soup_clip(mvp, verts, faces, valid, numSplits, tau_ratio, aspectWH)
void* remref_split_clip(const float* mvp, const float* verts, const int* faces, const int* valid, int nv, int nt,
                        int num_splits, float tau_ratio, float aspect_wh) {
    diffsoup::TriangleSoupSplitterClip s(mvp, verts, faces, nv, nt, valid);
    s.splitLongEdges(num_splits, tau_ratio, aspect_wh);
    return collect(s);
}

void remref_sizes(void* h, int* nv, int* nt) {
    const Result* r = static_cast<const Result*>(h);
    *nv = r->nv;
    *nt = r->nt;
}

void remref_export(void* h, float* verts, int* faces, int* map, int* flag) {
    const Result* r = static_cast<const Result*>(h);
    std::memcpy(verts, r->verts, sizeof(float) * 3 * (size_t)r->nv);
    std::memcpy(faces, r->faces, sizeof(int) * 3 * (size_t)r->nt);
    std::memcpy(map, r->map, sizeof(int) * (size_t)r->nt);
    std::memcpy(flag, r->flag, sizeof(int) * (size_t)r->nt);
}

void remref_free(void* h) {
    Result* r = static_cast<Result*>(h);
    delete[] r->verts;
    delete[] r->faces;
    delete[] r->map;
    delete[] r->flag;
    delete r;
}

}  // extern "C"
