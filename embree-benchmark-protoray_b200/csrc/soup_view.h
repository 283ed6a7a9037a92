// Indexed form of a triangle soup parsed from an OBJ file, shared by the host
// parser (obj_soup.cpp) and the GPU mesh builder (mesh_build.cu).  An OBJ is
// an indexed mesh; the soup's 100-byte triangle records are its expansion, so
// the builder uploads this form (positions-only files: 12 bytes per triangle
// plus 12 per vertex) and expands it on the device.
#pragma once

#include <cstdint>

struct prt_soup;

namespace prt_b200 {

struct SoupIndexed
{
    const float* v;         // positions, 3 floats each
    long long nv;
    const float* vt;        // texcoords, 2 floats each
    long long nvt;
    const float* vn;        // normals, 3 floats each
    long long nvn;
    // per triangle, 3 corners of cornerInts ints: the 0-based position index,
    // and with cornerInts == 3 also the texcoord and normal index (-1: none)
    const int* corners;
    int cornerInts;         // 1 or 3
    const int* mat;         // per triangle material id
    long long triCount;
};

// The indexed form of a soup from prt_soup_load_obj (false for a null soup).
bool soup_indexed(const prt_soup* soup, SoupIndexed* out);

} // namespace prt_b200
