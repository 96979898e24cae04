// TEST INFRASTRUCTURE: the reference's ObjImporter::load + TriangleMesh::toPrimitives on one
// file, written to stdout as int64 count (-1: the importer failed), int32 has_normals, then
// 9 floats of vertices and (with normals) 9 floats of normals per triangle. A separate process
// because the importer's stream parsing is run in isolation from the test process.
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "render/geometry/triangle.h"
#include "render/io/obj_importer.h"

using namespace render;

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    TriangleMesh mesh;
    int64_t n = -1;
    int32_t has = 0;
    if (!ObjImporter::load(argv[1], mesh)) {
        std::fwrite(&n, 8, 1, stdout);
        std::fwrite(&has, 4, 1, stdout);
        return 0;
    }
    const auto prims = mesh.toPrimitives(nullptr);
    n = static_cast<int64_t>(prims.size());
    std::vector<float> v, nn;
    for (const auto& p : prims) {
        const auto* t = static_cast<const Triangle*>(p.get());
        for (const Vec3* q : {&t->v0, &t->v1, &t->v2}) v.insert(v.end(), {q->x, q->y, q->z});
        if (t->hasNormals) {
            has = 1;
            for (const Vec3* q : {&t->n0, &t->n1, &t->n2}) nn.insert(nn.end(), {q->x, q->y, q->z});
        }
    }
    std::fwrite(&n, 8, 1, stdout);
    std::fwrite(&has, 4, 1, stdout);
    std::fwrite(v.data(), 4, v.size(), stdout);
    if (has) std::fwrite(nn.data(), 4, nn.size(), stdout);
    return 0;
}
