// FP32 binned-SAH BVH for the host CPU — TEST / BASELINE INFRASTRUCTURE ONLY.
//
// Embree 3, which the reference renderers call for every closest-hit and
// any-hit query (accel/embree/embree_intersector_single.h:29-60,
// accel/embree/embree_intersector_stream.h:30-104), is not installed in this
// image and its version is not pinned by the reference.  This intersector
// stands in for it so that the reference's own CPU renderers (diffuse,
// diffuseStream) can be compiled and timed on the host cores: a binary
// binned-SAH BVH (12 bins, leaves of up to 4 triangles) with an ordered
// stack traversal and a Moller-Trumbore triangle test in single precision.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace prt_oracle {

struct Bvh32
{
    struct Node
    {
        float lo[3], hi[3];
        int offset;   // internal: right child; leaf: first triangle
        int count;    // internal: 0; leaf: triangle count
        int axis;     // internal: split axis
        int pad;
    };
    struct Tri
    {
        float v0[3], e1[3], e2[3];
        int prim;
    };

    std::vector<Node> nodes;
    std::vector<Tri> tris;

    struct Ref
    {
        float lo[3], hi[3], c[3];
        int prim;
    };

    void build(const float* pos, const int* idx, int nt)
    {
        nodes.clear();
        tris.clear();
        if (nt <= 0) return;
        std::vector<Ref> refs(nt);
        for (int p = 0; p < nt; ++p)
        {
            Ref& r = refs[p];
            for (int k = 0; k < 3; ++k)
            {
                float a = pos[3 * idx[3 * p + 0] + k], b = pos[3 * idx[3 * p + 1] + k], c = pos[3 * idx[3 * p + 2] + k];
                r.lo[k] = std::min(a, std::min(b, c));
                r.hi[k] = std::max(a, std::max(b, c));
                r.c[k] = 0.5f * (r.lo[k] + r.hi[k]);
            }
            r.prim = p;
        }
        nodes.reserve(2 * nt);
        buildRec(refs, 0, nt);
        tris.resize(nt);
        for (int i = 0; i < nt; ++i)
        {
            int p = refs[i].prim;
            Tri& t = tris[i];
            const float* a = pos + 3 * idx[3 * p + 0];
            const float* b = pos + 3 * idx[3 * p + 1];
            const float* c = pos + 3 * idx[3 * p + 2];
            for (int k = 0; k < 3; ++k)
            {
                t.v0[k] = a[k];
                t.e1[k] = b[k] - a[k];
                t.e2[k] = c[k] - a[k];
            }
            t.prim = p;
        }
    }

    static float area(const float* lo, const float* hi)
    {
        float d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
        if (d0 < 0 || d1 < 0 || d2 < 0) return 0.f;
        return d0 * d1 + d1 * d2 + d2 * d0;
    }

    int buildRec(std::vector<Ref>& refs, int first, int count)
    {
        int ni = (int)nodes.size();
        nodes.push_back(Node());
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = first; i < first + count; ++i)
            for (int k = 0; k < 3; ++k)
            {
                lo[k] = std::min(lo[k], refs[i].lo[k]);
                hi[k] = std::max(hi[k], refs[i].hi[k]);
                clo[k] = std::min(clo[k], refs[i].c[k]);
                chi[k] = std::max(chi[k], refs[i].c[k]);
            }
        for (int k = 0; k < 3; ++k)
        {
            nodes[ni].lo[k] = lo[k];
            nodes[ni].hi[k] = hi[k];
        }
        auto makeLeaf = [&]() {
            nodes[ni].offset = first;
            nodes[ni].count = count;
            nodes[ni].axis = 0;
        };
        if (count <= 2) { makeLeaf(); return ni; }

        const int B = 12;
        float bestCost = FLT_MAX;
        int bestAxis = -1, bestSplit = -1;
        for (int k = 0; k < 3; ++k)
        {
            float ext = chi[k] - clo[k];
            if (!(ext > 0)) continue;
            int bc[B] = {0};
            float blo[B][3], bhi[B][3];
            for (int b = 0; b < B; ++b)
                for (int j = 0; j < 3; ++j) { blo[b][j] = FLT_MAX; bhi[b][j] = -FLT_MAX; }
            float scale = B / ext;
            for (int i = first; i < first + count; ++i)
            {
                int b = std::min(B - 1, (int)((refs[i].c[k] - clo[k]) * scale));
                bc[b]++;
                for (int j = 0; j < 3; ++j)
                {
                    blo[b][j] = std::min(blo[b][j], refs[i].lo[j]);
                    bhi[b][j] = std::max(bhi[b][j], refs[i].hi[j]);
                }
            }
            float rA[B];
            int rC[B];
            float alo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ahi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            int acc = 0;
            for (int b = B - 1; b > 0; --b)
            {
                acc += bc[b];
                for (int j = 0; j < 3; ++j) { alo[j] = std::min(alo[j], blo[b][j]); ahi[j] = std::max(ahi[j], bhi[b][j]); }
                rA[b] = area(alo, ahi);
                rC[b] = acc;
            }
            float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            int lc = 0;
            for (int b = 0; b < B - 1; ++b)
            {
                lc += bc[b];
                for (int j = 0; j < 3; ++j) { llo[j] = std::min(llo[j], blo[b][j]); lhi[j] = std::max(lhi[j], bhi[b][j]); }
                if (lc == 0 || rC[b + 1] == 0) continue;
                float cost = area(llo, lhi) * lc + rA[b + 1] * rC[b + 1];
                if (cost < bestCost) { bestCost = cost; bestAxis = k; bestSplit = b; }
            }
        }
        if (bestAxis < 0)
        {
            if (count <= 4) { makeLeaf(); return ni; }
            // all centroids coincide: split the list in the middle
            int half = count / 2;
            nodes[ni].axis = 0;
            nodes[ni].count = 0;
            buildRec(refs, first, half);
            int r = buildRec(refs, first + half, count - half);
            nodes[ni].offset = r;
            return ni;
        }
        // SAH with unit traversal and intersection costs
        float parentArea = area(lo, hi);
        if (count <= 4 && parentArea * count <= parentArea + bestCost) { makeLeaf(); return ni; }
        float ext = chi[bestAxis] - clo[bestAxis];
        float scale = B / ext;
        auto mid = std::partition(refs.begin() + first, refs.begin() + first + count, [&](const Ref& r) {
            int b = std::min(B - 1, (int)((r.c[bestAxis] - clo[bestAxis]) * scale));
            return b <= bestSplit;
        });
        int lcount = (int)(mid - (refs.begin() + first));
        if (lcount == 0 || lcount == count) lcount = count / 2;
        nodes[ni].axis = bestAxis;
        nodes[ni].count = 0;
        buildRec(refs, first, lcount);
        int r = buildRec(refs, first + lcount, count - lcount);
        nodes[ni].offset = r;
        return ni;
    }

    // Closest hit over (0, tfar]; returns true and updates tfar/prim/u/v.
    bool intersect(const float org[3], const float dir[3], float& tfar, int& prim, float& u, float& v,
                   int64_t* nodeCount = nullptr) const
    {
        if (nodes.empty()) return false;
        float inv[3];
        int neg[3];
        for (int k = 0; k < 3; ++k)
        {
            inv[k] = 1.0f / dir[k];
            neg[k] = inv[k] < 0;
        }
        int stack[96];
        int sp = 0;
        int ni = 0;
        bool found = false;
        for (;;)
        {
            const Node& n = nodes[ni];
            if (nodeCount) (*nodeCount)++;
            float t0 = 0.f, t1 = tfar;
            for (int k = 0; k < 3; ++k)
            {
                float a = (n.lo[k] - org[k]) * inv[k];
                float b = (n.hi[k] - org[k]) * inv[k];
                float l = neg[k] ? b : a, h = neg[k] ? a : b;
                t0 = l > t0 ? l : t0;
                t1 = h < t1 ? h : t1;
            }
            if (t0 <= t1 * 1.0000004f)
            {
                if (n.count > 0)
                {
                    for (int i = n.offset; i < n.offset + n.count; ++i)
                    {
                        const Tri& t = tris[i];
                        float p[3] = {dir[1] * t.e2[2] - dir[2] * t.e2[1], dir[2] * t.e2[0] - dir[0] * t.e2[2],
                                      dir[0] * t.e2[1] - dir[1] * t.e2[0]};
                        float det = t.e1[0] * p[0] + t.e1[1] * p[1] + t.e1[2] * p[2];
                        if (det == 0.f) continue;
                        float id = 1.0f / det;
                        float s[3] = {org[0] - t.v0[0], org[1] - t.v0[1], org[2] - t.v0[2]};
                        float uu = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * id;
                        if (uu < 0.f || uu > 1.f) continue;
                        float q[3] = {s[1] * t.e1[2] - s[2] * t.e1[1], s[2] * t.e1[0] - s[0] * t.e1[2],
                                      s[0] * t.e1[1] - s[1] * t.e1[0]};
                        float vv = (dir[0] * q[0] + dir[1] * q[1] + dir[2] * q[2]) * id;
                        if (vv < 0.f || uu + vv > 1.f) continue;
                        float tt = (t.e2[0] * q[0] + t.e2[1] * q[1] + t.e2[2] * q[2]) * id;
                        if (!(tt > 0.f) || !(tt < tfar)) continue;
                        tfar = tt;
                        prim = t.prim;
                        u = uu;
                        v = vv;
                        found = true;
                    }
                }
                else
                {
                    int l = ni + 1, r = n.offset;
                    if (neg[n.axis]) std::swap(l, r);
                    if (sp < 96) stack[sp++] = r;
                    ni = l;
                    continue;
                }
            }
            if (sp == 0) break;
            ni = stack[--sp];
        }
        return found;
    }
};

} // namespace prt_oracle
