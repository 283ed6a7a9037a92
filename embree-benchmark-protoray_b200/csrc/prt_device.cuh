// Device-side building blocks of the B200 diffuse path tracer: records, RNG,
// camera, compressed 8-wide BVH node layout, watertight traversal and the
// diffuse bounce.  Everything here is __device__ code included by the kernels.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

namespace prt_b200 {

// ---------------------------------------------------------------------------
// Small float3 helpers.  Arithmetic that decides a path's trajectory uses the
// explicitly rounded intrinsics so that every kernel that replays a path
// (forward wavefront, megakernel, adjoint) computes bit-identical rays no
// matter how the compiler fuses the surrounding code.
// ---------------------------------------------------------------------------

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return f3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return f3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ float3 mul(float3 a, float s) { return f3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)); }
__device__ __forceinline__ float dot(float3 a, float3 b)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float3 cross(float3 a, float3 b)
{
    return f3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
              __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float3 normalize(float3 a)
{
    float l2 = dot(a, a);
    float inv = __frcp_rn(__fsqrt_rn(l2));
    return mul(a, inv);
}
// a + s*b, rounded after each operation
__device__ __forceinline__ float3 madd(float3 a, float s, float3 b) { return add(a, mul(b, s)); }

// ---------------------------------------------------------------------------
// Records.  RayRec/HitRec keep the 32-byte / 16-byte layouts of the reference
// GPU interface (core/ray_cuda.cuh:23-80): a miss is t < 0.
// ---------------------------------------------------------------------------

struct RayRec
{
    float ox, oy, oz, tnear;
    float dx, dy, dz, tfar;
};

struct HitRec
{
    float t;
    int primId;
    float u, v;
};

// Wavefront path record (32 bytes, two 16-byte words):
//   w0 = {org.xyz, pixel id (int bits)}, w1 = {dir.xyz, RNG state (uint bits)}
struct PathRec
{
    float4 w0;
    float4 w1;
};

// ---------------------------------------------------------------------------
// RNG: Murmur3 mixing of (pixel, pass) then an LCG stream
// (sampling/random_sampler.cuh:29-103 and sampling/random_sampler.h:44-73).
// uint32 -> float rounds to nearest as the reference CPU code does
// (math/math.h:179), so GPU and CPU draw identical sample values.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t murmur_mix(uint32_t h, uint32_t k)
{
    k *= 0xcc9e2d51u;
    k = __funnelshift_l(k, k, 15);
    k *= 0x1b873593u;
    h ^= k;
    h = __funnelshift_l(h, h, 13) * 5u + 0xe6546b64u;
    return h;
}

__device__ __forceinline__ uint32_t murmur_fin(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

__device__ __forceinline__ uint32_t rng_seed(int pass, int pixel)
{
    return murmur_fin(murmur_mix(murmur_mix(0u, (uint32_t)pixel), (uint32_t)pass));
}

__device__ __forceinline__ float rng_next(uint32_t& s)
{
    s = s * 1664525u + 1013904223u;
    return __fmul_rn(__uint2float_rn(s), 0x1.0p-32f);
}

// ---------------------------------------------------------------------------
// Camera (fields of ThinLensCameraCuda, camera/thin_lens_camera_cuda.h:23-30)
// ---------------------------------------------------------------------------

struct CameraDev
{
    float3 origin;
    float3 basisU, basisV;
    float3 imageO, imageDx, imageDy;
    float lensRadius, focalDistance;
    float invW, invH;
    int width, height;
};

// Primary ray for pixel (x, y) of pass `pass`: pixel jitter and lens sample
// are the first two 2D draws (render/renderer_single.h:112-119); the pinhole
// camera is used when the lens radius is 0 (render/device_cpu_impl.cpp:86-97).
__device__ __forceinline__ void camera_ray(const CameraDev& cam, int x, int y, uint32_t& rng, float3& org, float3& dir)
{
    float jx = rng_next(rng);
    float jy = rng_next(rng);
    float lx = rng_next(rng);
    float ly = rng_next(rng);
    float ix = __fmul_rn(__fadd_rn((float)x, jx), cam.invW);
    float iy = __fmul_rn(__fadd_rn((float)y, jy), cam.invH);
    float3 d = add(add(cam.imageO, mul(cam.imageDx, ix)), mul(cam.imageDy, iy));
    if (cam.lensRadius == 0.0f)
    {
        org = cam.origin;
        dir = normalize(d);
    }
    else
    {
        // uniformSampleDisk (sampling/shape_sampler.h:114-124)
        float r = __fsqrt_rn(lx);
        float s, c;
        sincosf(__fmul_rn(2.0f * 3.14159265358979f, ly), &s, &c);
        float dx = __fmul_rn(__fmul_rn(r, c), cam.lensRadius);
        float dy = __fmul_rn(__fmul_rn(r, s), cam.lensRadius);
        float3 begin = add(add(cam.origin, mul(cam.basisU, dx)), mul(cam.basisV, dy));
        float3 end = add(cam.origin, mul(d, cam.focalDistance));
        org = begin;
        dir = normalize(sub(end, begin));
    }
}

// ---------------------------------------------------------------------------
// Compressed 8-wide BVH node (80 bytes = 5 x 16 B).
//   q0 = {origin.xyz, exponents x|y|z (biased by 127, bytes 0..2) | imask << 24}
//   q1 = {child node base, triangle base, meta[0..3], meta[4..7]}
//   q2 = {qlo.x[0..3], qlo.x[4..7], qlo.y[0..3], qlo.y[4..7]}
//   q3 = {qlo.z[0..3], qlo.z[4..7], qhi.x[0..3], qhi.x[4..7]}
//   q4 = {qhi.y[0..3], qhi.y[4..7], qhi.z[0..3], qhi.z[4..7]}
// A child box is origin + q * 2^e per axis (8-bit q).  meta per slot:
//   0                       empty slot
//   0x20 | (24 + slot)      internal child (stored at base + rank among
//                           internal slots of lower index, imask bit = slot)
//   unary(n) << 5 | offset  leaf with n in 1..3 triangles at triBase+offset
// Triangles are stored in leaf order, 48 bytes each: {v0, primId}, {v1, 0},
// {v2, 0}.
// Slot s is given to the child that comes first for rays whose direction
// octant is s; traversal pops hits in the order of (slot ^ (7 - octant)).
// ---------------------------------------------------------------------------

// PRT_NODE_PAD pads nodes to 128 bytes (one L1 line each) instead of 80.
#ifndef PRT_NODE_PAD
#define PRT_NODE_PAD 0
#endif

struct Bvh8Node
{
    uint4 q[5];
#if PRT_NODE_PAD
    uint4 pad[3];
#endif
};

struct TriRec
{
    float4 v0, v1, v2;
};

struct SceneDev
{
    const Bvh8Node* nodes;
    const TriRec* tris;
    const float* albedo;   // per original triangle id, or nullptr (constant 0.8)
    int triCount;
    int hasRoot;           // 0 for an empty scene
    int leafTris;          // most triangles in one leaf (the build's leaf size)
    int deferTris;         // one-triangle leaves and fewer than 2^27 triangles: deferred triangle tests
};

// Leaf-order triangle indices the deferred-test queue can hold (27 bits; the
// other 5 bits of a queue entry hold the owner lane).
constexpr int kDeferMaxTris = 1 << 27;

// Per-ray constants for traversal.
struct TravRay
{
    float3 org;
    float3 dir;
    float3 inv;
    uint32_t octinv;   // 7 - octant of dir
    int kx, ky, kz;    // watertight shear axes
    float Sx, Sy, Sz;
};

__device__ __forceinline__ void trav_setup(TravRay& r, float3 org, float3 dir)
{
    r.org = org;
    r.dir = dir;
    const float tiny = 1e-30f;
    r.inv.x = 1.0f / (fabsf(dir.x) > tiny ? dir.x : copysignf(tiny, dir.x));
    r.inv.y = 1.0f / (fabsf(dir.y) > tiny ? dir.y : copysignf(tiny, dir.y));
    r.inv.z = 1.0f / (fabsf(dir.z) > tiny ? dir.z : copysignf(tiny, dir.z));
    uint32_t oct = (dir.x < 0.f ? 1u : 0u) | (dir.y < 0.f ? 2u : 0u) | (dir.z < 0.f ? 4u : 0u);
    r.octinv = 7u - oct;
    float ax = fabsf(dir.x), ay = fabsf(dir.y), az = fabsf(dir.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    float dkz = kz == 0 ? dir.x : (kz == 1 ? dir.y : dir.z);
    if (dkz < 0.f) { int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    float dkx = kx == 0 ? dir.x : (kx == 1 ? dir.y : dir.z);
    float dky = ky == 0 ? dir.x : (ky == 1 ? dir.y : dir.z);
    r.Sx = dkx / dkz;
    r.Sy = dky / dkz;
    r.Sz = 1.0f / dkz;
}

__device__ __forceinline__ float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2(1) 2013).
// Accepts t in (tnear, tbest) — or t == tbest with a lower primitive id, so
// that exact ties resolve the same way in every traversal order.  On a hit
// returns true and sets t (and the barycentrics b1 -> u, b2 -> v, the
// reference's convention, geometry/triangle_mesh.cpp:69-71).
__device__ __forceinline__ bool tri_test(const TravRay& r, float3 v0, float3 v1, float3 v2, float tnear, float tbest,
                                         int prim, int bestPrim, float& t, float& u, float& v)
{
    float3 A = sub(v0, r.org), B = sub(v1, r.org), C = sub(v2, r.org);
    float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
    float Ax = comp(A, r.kx) - r.Sx * Akz, Ay = comp(A, r.ky) - r.Sy * Akz;
    float Bx = comp(B, r.kx) - r.Sx * Bkz, By = comp(B, r.ky) - r.Sy * Bkz;
    float Cx = comp(C, r.kx) - r.Sx * Ckz, Cy = comp(C, r.ky) - r.Sy * Ckz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f)
    {
        // edge case: recompute the edge functions in double precision
        double CxBy = (double)Cx * (double)By, CyBx = (double)Cy * (double)Bx;
        U = (float)(CxBy - CyBx);
        double AxCy = (double)Ax * (double)Cy, AyCx = (double)Ay * (double)Cx;
        V = (float)(AxCy - AyCx);
        double BxAy = (double)Bx * (double)Ay, ByAx = (double)By * (double)Ax;
        W = (float)(BxAy - ByAx);
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    float det = U + V + W;
    if (det == 0.f) return false;
    float T = U * (r.Sz * Akz) + V * (r.Sz * Bkz) + W * (r.Sz * Ckz);
    // sign-aware range check without dividing
    uint32_t sgn = __float_as_uint(det) & 0x80000000u;
    float Ts = __uint_as_float(__float_as_uint(T) ^ sgn);
    float dets = fabsf(det);
    if (!(Ts > tnear * dets) || Ts > tbest * dets) return false;
    float rcp = 1.0f / det;
    float tt = T * rcp;
    if (!(tt > tnear)) return false;
    if (tt > tbest || (tt == tbest && prim >= bestPrim)) return false;
    t = tt;
    u = V * rcp;
    v = W * rcp;
    return true;
}

// Three-input float max / min (one instruction each on sm_100).
__device__ __forceinline__ float fmax3(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float fmin3(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Byte j of x as a float, exactly: 2^23 + byte built with a byte permute,
// minus 2^23 (avoids the slower integer-to-float conversion).
__device__ __forceinline__ float byte_f(uint32_t x, int j)
{
    return __uint_as_float(__byte_perm(x, 0x4b000000u, 0x7440u + (uint32_t)j)) - 8388608.0f;
}

// Byte j of x in mantissa bits 8..15 of 1.0f: exactly 1 + q * 2^-15, one
// byte permute.  A child plane is then fma(u, 2^15 * s * inv, (p - o) * inv -
// 2^15 * s * inv); the subtraction's rounding moves a plane by at most 2^-9
// of a quantization step, which the build's 2^-8-step margin covers.
__device__ __forceinline__ float byte_unit(uint32_t x, int j)
{
    return __uint_as_float(__byte_perm(x, 0x3f800000u, 0x7604u + ((uint32_t)j << 4)));
}

#ifndef PRT_FAST_DECODE
#define PRT_FAST_DECODE 1
#endif

// Paired FP32 FMA of sm_100 (fma.rn.f32x2): two child planes per instruction.
#ifndef PRT_FFMA2
#define PRT_FFMA2 0
#endif

// {a0, a1} * {s, s} + {o, o}, each lane rounded once, as two fmaf calls would.
__device__ __forceinline__ float2 ffma2(float a0, float a1, float s, float o)
{
    unsigned long long a, b, c, d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(a) : "f"(a0), "f"(a1));
    asm("mov.b64 %0, {%1, %1};" : "=l"(b) : "f"(s));
    asm("mov.b64 %0, {%1, %1};" : "=l"(c) : "f"(o));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(d));
    return r;
}

// Intersection of the ray with the 8 child boxes of a node.  Returns the hit
// mask: bits 24..31 internal children (traversal order), bits 0..23 triangles
// relative to the node's triangle base.
__device__ __forceinline__ uint32_t node_hits(const TravRay& r, const uint4* q, float tnear, float tfar)
{
    float px = __uint_as_float(q[0].x), py = __uint_as_float(q[0].y), pz = __uint_as_float(q[0].z);
    uint32_t e = q[0].w;
    // 2^(e-127), times 2^15 for the fast plane decode (the build keeps e <= 100)
    const uint32_t eb = PRT_FAST_DECODE ? 15u : 0u;
    float sx = __uint_as_float(((e & 0xffu) + eb) << 23);
    float sy = __uint_as_float((((e >> 8) & 0xffu) + eb) << 23);
    float sz = __uint_as_float((((e >> 16) & 0xffu) + eb) << 23);
    float aix = sx * r.inv.x, aiy = sy * r.inv.y, aiz = sz * r.inv.z;
    float aox = (px - r.org.x) * r.inv.x, aoy = (py - r.org.y) * r.inv.y, aoz = (pz - r.org.z) * r.inv.z;
    if (PRT_FAST_DECODE)
    {
        aox -= aix;
        aoy -= aiy;
        aoz -= aiz;
    }
    // For a negative direction component the far plane is the low plane:
    // select per axis which byte array feeds the near / far distance.
    bool nx = r.inv.x < 0.f, ny = r.inv.y < 0.f, nz = r.inv.z < 0.f;
    uint32_t loX[2] = {q[2].x, q[2].y}, loY[2] = {q[2].z, q[2].w}, loZ[2] = {q[3].x, q[3].y};
    uint32_t hiX[2] = {q[3].z, q[3].w}, hiY[2] = {q[4].x, q[4].y}, hiZ[2] = {q[4].z, q[4].w};
    uint32_t meta[2] = {q[1].z, q[1].w};
    const uint32_t octinv4 = r.octinv * 0x01010101u;
    uint32_t hits = 0;
    const float tfarp = tfar * 1.0000004f;
#pragma unroll
    for (int h = 0; h < 2; ++h)
    {
        uint32_t nearX = nx ? hiX[h] : loX[h], farX = nx ? loX[h] : hiX[h];
        uint32_t nearY = ny ? hiY[h] : loY[h], farY = ny ? loY[h] : hiY[h];
        uint32_t nearZ = nz ? hiZ[h] : loZ[h], farZ = nz ? loZ[h] : hiZ[h];
        // per byte: internal children (low 5 meta bits 24..31) put one bit at
        // 24 + (slot ^ octinv); leaves put their unary triangle count at their
        // triangle offset; empty slots (meta 0) contribute nothing
        uint32_t m4 = meta[h];
        uint32_t inner4 = ((m4 & (m4 << 1)) & 0x10101010u) >> 4;           // 1 per internal byte
        uint32_t index4 = (m4 ^ (octinv4 & (inner4 * 0xffu))) & 0x1f1f1f1fu;
        uint32_t bits4 = (m4 >> 5) & 0x07070707u;
        if (PRT_FFMA2 && PRT_FAST_DECODE)
        {
#pragma unroll
            for (int j = 0; j < 4; j += 2)
            {
                const float2 nX = ffma2(byte_unit(nearX, j), byte_unit(nearX, j + 1), aix, aox);
                const float2 nY = ffma2(byte_unit(nearY, j), byte_unit(nearY, j + 1), aiy, aoy);
                const float2 nZ = ffma2(byte_unit(nearZ, j), byte_unit(nearZ, j + 1), aiz, aoz);
                const float2 fX = ffma2(byte_unit(farX, j), byte_unit(farX, j + 1), aix, aox);
                const float2 fY = ffma2(byte_unit(farY, j), byte_unit(farY, j + 1), aiy, aoy);
                const float2 fZ = ffma2(byte_unit(farZ, j), byte_unit(farZ, j + 1), aiz, aoz);
                const float t0a = fmax3(nX.x, nY.x, fmaxf(nZ.x, tnear)), t1a = fmin3(fX.x, fY.x, fminf(fZ.x, tfarp));
                const float t0b = fmax3(nX.y, nY.y, fmaxf(nZ.y, tnear)), t1b = fmin3(fX.y, fY.y, fminf(fZ.y, tfarp));
                if (t0a <= t1a * 1.0000008f)
                    hits |= ((bits4 >> (8 * j)) & 0xffu) << ((index4 >> (8 * j)) & 0xffu);
                if (t0b <= t1b * 1.0000008f)
                    hits |= ((bits4 >> (8 * j + 8)) & 0xffu) << ((index4 >> (8 * j + 8)) & 0xffu);
            }
            continue;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            float tnx, tny, tnz, tfx, tfy, tfz;
            if (PRT_FAST_DECODE)
            {
                tnx = fmaf(byte_unit(nearX, j), aix, aox);
                tny = fmaf(byte_unit(nearY, j), aiy, aoy);
                tnz = fmaf(byte_unit(nearZ, j), aiz, aoz);
                tfx = fmaf(byte_unit(farX, j), aix, aox);
                tfy = fmaf(byte_unit(farY, j), aiy, aoy);
                tfz = fmaf(byte_unit(farZ, j), aiz, aoz);
            }
            else
            {
                tnx = fmaf(byte_f(nearX, j), aix, aox);
                tny = fmaf(byte_f(nearY, j), aiy, aoy);
                tnz = fmaf(byte_f(nearZ, j), aiz, aoz);
                tfx = fmaf(byte_f(farX, j), aix, aox);
                tfy = fmaf(byte_f(farY, j), aiy, aoy);
                tfz = fmaf(byte_f(farZ, j), aiz, aoz);
            }
            float t0 = fmax3(tnx, tny, fmaxf(tnz, tnear));
            float t1 = fmin3(tfx, tfy, fminf(tfz, tfarp));
            // t0 >= tnear >= 0: one relative slack covers rounding on both sides
            if (t0 <= t1 * 1.0000008f) hits |= ((bits4 >> (8 * j)) & 0xffu) << ((index4 >> (8 * j)) & 0xffu);
        }
    }
    return hits;
}

// Node test for trees with one-triangle leaves (the default build): every
// non-empty child owns exactly one hit bit, so the test sets bit `slot` of an
// 8-bit mask per child hit instead of assembling the general mask from the
// meta bytes.  Non-empty slots have bit 5 of their meta byte set (0x20 for an
// internal child, a unary count of 1 for a leaf); leaf triangles are stored in
// slot order, so the triangle of leaf slot j is triBase + popc(leafMask below j).
// Returns internal hits at bits 24 + (slot ^ octinv) as node_hits does, leaf
// hits as slot bits 0..7, and the node's leaf-slot mask in leafMask.
// octinv: the octant code that orders the internal hit bits (the ray's own in
// per-lane traversal; one shared by a warp in packet traversal).  kPair: the
// planes of two children per paired FP32 FMA (fma.rn.f32x2); faster where the
// kernel has registers to spare for the paired coefficients, slower where they
// make it spill heavily (closest-hit ray queries, the first bounce of the
// diffuse2 kernel).  Both give the same results: each lane of a paired FMA is
// rounded once, as fmaf is.
template <bool kPair = false>
__device__ __forceinline__ uint32_t node_hits1(const TravRay& r, const uint4* q, float tnear, float tfar,
                                               uint32_t& leafMask, uint32_t octinv)
{
    float px = __uint_as_float(q[0].x), py = __uint_as_float(q[0].y), pz = __uint_as_float(q[0].z);
    uint32_t e = q[0].w;
    float sx = __uint_as_float(((e & 0xffu) + 15u) << 23);
    float sy = __uint_as_float((((e >> 8) & 0xffu) + 15u) << 23);
    float sz = __uint_as_float((((e >> 16) & 0xffu) + 15u) << 23);
    float aix = sx * r.inv.x, aiy = sy * r.inv.y, aiz = sz * r.inv.z;
    float aox = (px - r.org.x) * r.inv.x - aix, aoy = (py - r.org.y) * r.inv.y - aiy, aoz = (pz - r.org.z) * r.inv.z - aiz;
    bool nx = r.inv.x < 0.f, ny = r.inv.y < 0.f, nz = r.inv.z < 0.f;
    uint32_t loX[2] = {q[2].x, q[2].y}, loY[2] = {q[2].z, q[2].w}, loZ[2] = {q[3].x, q[3].y};
    uint32_t hiX[2] = {q[3].z, q[3].w}, hiY[2] = {q[4].x, q[4].y}, hiZ[2] = {q[4].z, q[4].w};
    const float tfarp = tfar * 1.0000004f;
    uint32_t c8 = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h)
    {
        uint32_t nearX = nx ? hiX[h] : loX[h], farX = nx ? loX[h] : hiX[h];
        uint32_t nearY = ny ? hiY[h] : loY[h], farY = ny ? loY[h] : hiY[h];
        uint32_t nearZ = nz ? hiZ[h] : loZ[h], farZ = nz ? loZ[h] : hiZ[h];
        if constexpr (kPair)
        {
#pragma unroll
            for (int j = 0; j < 4; j += 2)
            {
                const float2 nX = ffma2(byte_unit(nearX, j), byte_unit(nearX, j + 1), aix, aox);
                const float2 nY = ffma2(byte_unit(nearY, j), byte_unit(nearY, j + 1), aiy, aoy);
                const float2 nZ = ffma2(byte_unit(nearZ, j), byte_unit(nearZ, j + 1), aiz, aoz);
                const float2 fX = ffma2(byte_unit(farX, j), byte_unit(farX, j + 1), aix, aox);
                const float2 fY = ffma2(byte_unit(farY, j), byte_unit(farY, j + 1), aiy, aoy);
                const float2 fZ = ffma2(byte_unit(farZ, j), byte_unit(farZ, j + 1), aiz, aoz);
                const float t0a = fmax3(nX.x, nY.x, fmaxf(nZ.x, tnear)), t1a = fmin3(fX.x, fY.x, fminf(fZ.x, tfarp));
                const float t0b = fmax3(nX.y, nY.y, fmaxf(nZ.y, tnear)), t1b = fmin3(fX.y, fY.y, fminf(fZ.y, tfarp));
                if (t0a <= t1a * 1.0000008f) c8 |= 1u << (4 * h + j);
                if (t0b <= t1b * 1.0000008f) c8 |= 1u << (4 * h + j + 1);
            }
        }
        else
        {
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                float tnx = fmaf(byte_unit(nearX, j), aix, aox);
                float tny = fmaf(byte_unit(nearY, j), aiy, aoy);
                float tnz = fmaf(byte_unit(nearZ, j), aiz, aoz);
                float tfx = fmaf(byte_unit(farX, j), aix, aox);
                float tfy = fmaf(byte_unit(farY, j), aiy, aoy);
                float tfz = fmaf(byte_unit(farZ, j), aiz, aoz);
                float t0 = fmax3(tnx, tny, fmaxf(tnz, tnear));
                float t1 = fmin3(tfx, tfy, fminf(tfz, tfarp));
                if (t0 <= t1 * 1.0000008f) c8 |= 1u << (4 * h + j);
            }
        }
    }
    // bit 5 of each meta byte -> one bit per slot (multiply gathers bytes 0..3 into bits 24..27)
    const uint32_t ne = ((((q[1].z >> 5) & 0x01010101u) * 0x01020408u) >> 24) |
                        (((((q[1].w >> 5) & 0x01010101u) * 0x01020408u) >> 24) << 4);
    c8 &= ne;
    const uint32_t imask = q[0].w >> 24;
    leafMask = ne & ~imask;
    // internal hits: bit slot -> bit slot ^ octinv (three conditional swaps)
    uint32_t in8 = c8 & imask;
    const uint32_t o = octinv;
    uint32_t sw = ((in8 & 0x55u) << 1) | ((in8 >> 1) & 0x55u);
    in8 = (o & 1u) ? sw : in8;
    sw = ((in8 & 0x33u) << 2) | ((in8 >> 2) & 0x33u);
    in8 = (o & 2u) ? sw : in8;
    sw = ((in8 & 0x0fu) << 4) | ((in8 >> 4) & 0x0fu);
    in8 = (o & 4u) ? sw : in8;
    return (in8 << 24) | (c8 & leafMask);
}

// Traversal stack: the first kShared entries of each thread live in shared
// memory (one column per thread), deeper entries spill to local memory.  A
// node visit pushes at most one node group and one postponed triangle group,
// so a tree of L 8-wide levels needs at most 2L entries.
#ifndef PRT_STACK_SHARED
#define PRT_STACK_SHARED 8
#endif
constexpr int kShared = PRT_STACK_SHARED;
constexpr int kLocal = 64 - PRT_STACK_SHARED;
constexpr int kStackMax = kShared + kLocal;

struct TravStack
{
    uint2* sh;         // shared base for this thread: sh[i * stride]
    int stride;
    uint2 loc[kLocal];
    int sp;
    bool overflow;

    __device__ __forceinline__ void push(uint2 v)
    {
        if (sp < kShared) sh[sp * stride] = v;
        else if (sp < kStackMax) loc[sp - kShared] = v;
        else { overflow = true; return; }
        ++sp;
    }
    __device__ __forceinline__ uint2 pop()
    {
        --sp;
        return sp < kShared ? sh[sp * stride] : loc[sp - kShared];
    }
};

// Closest hit (anyHit = false) or any hit (anyHit = true) over (tnear, tfar].
// Returns the leaf-order triangle index of the hit (or -1), with t/u/v/prim.
// Resumable traversal state of one ray.  A step visits one 8-wide node and
// tests the triangles of its hit leaves; `done` is set when no node groups
// remain (or, for any-hit queries, at the first hit).
struct TravState
{
    uint2 ng;       // current node group: {child base, hit bits 24..31 | imask bits 0..7}
    float tHit;     // closest hit so far (starts at tfar)
    int primHit;    // original triangle id of the hit (INT_MAX: none)
    int triHit;     // leaf-order triangle index of the hit (-1: none)
    float uHit, vHit;
    bool done;
};

__device__ __forceinline__ void trav_init(TravState& s, const SceneDev& sc, float tfar, TravStack& st)
{
    s.ng = make_uint2(0u, 0x80000000u);   // root group: one internal "child" at base 0
    s.tHit = tfar;
    s.primHit = 0x7fffffff;
    s.triHit = -1;
    s.uHit = 0.f;
    s.vHit = 0.f;
    s.done = !sc.hasRoot;
    st.sp = 0;
}

// Triangle postponement (Ylitie et al. 2017): while a ray still has child
// nodes to visit, it defers its triangle tests (pushing the triangle group
// on the stack) if fewer than this many lanes of the warp are testing
// triangles at that moment, so triangle tests run with more lanes together.
// Off by default: on the 1.4M-triangle terrain at 1080p it measured 1.65
// Grays/s off vs 1.62 with thresholds of 12 and 16 lanes.
// Prefetch of the next child node into L1 (on by default if measured faster).
#ifndef PRT_PREFETCH
#define PRT_PREFETCH 0
#endif

#ifndef PRT_POSTPONE_MIN
#define PRT_POSTPONE_MIN 0
#endif

template <bool anyHit>
__device__ __forceinline__ void trav_step(TravState& s, const SceneDev& sc, const TravRay& r, float tnear, TravStack& st,
                                          uint32_t* nodeVisits = nullptr, uint32_t* triTests = nullptr,
                                          bool anyHitRt = false)
{
    uint2 ng = s.ng;
    uint32_t tbits, tbase;
    if (ng.y & 0xff000000u)
    {
        // visit the next child node of the group
        uint32_t b = 31u - __clz(ng.y & 0xff000000u);
        ng.y &= ~(1u << b);
        uint32_t slot = (b - 24u) ^ r.octinv;
        uint32_t rel = __popc((ng.y & 0xffu) & ((1u << slot) - 1u));
        uint32_t nodeIdx = ng.x + rel;
        if (ng.y & 0xff000000u) st.push(ng);
        const uint4* qp = reinterpret_cast<const uint4*>(sc.nodes + nodeIdx);
        uint4 q[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) q[k] = __ldg(qp + k);
        uint32_t hits = node_hits(r, q, tnear, s.tHit);
        if (nodeVisits) ++*nodeVisits;
        ng = make_uint2(q[1].x, (hits & 0xff000000u) | (q[0].w >> 24));
        if (PRT_PREFETCH && (ng.y & 0xff000000u))
        {
            // start fetching the child visited next while the triangles are tested
            uint32_t nb = 31u - __clz(ng.y & 0xff000000u);
            uint32_t ns = (nb - 24u) ^ r.octinv;
            uint32_t nidx = ng.x + __popc((ng.y & 0xffu) & ((1u << ns) - 1u));
            const char* np = reinterpret_cast<const char*>(sc.nodes + nidx);
            asm volatile("prefetch.global.L1 [%0];" ::"l"(np));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(np + 64));
        }
        tbits = hits & 0x00ffffffu;
        tbase = q[1].y;
        if (PRT_POSTPONE_MIN > 0 && tbits && (ng.y & 0xff000000u) &&
            __popc(__activemask()) < PRT_POSTPONE_MIN)
        {
            st.push(make_uint2(tbase, tbits));   // a triangle group: no bits above 23
            tbits = 0;
        }
    }
    else
    {
        // a postponed triangle group popped from the stack
        tbase = ng.x;
        tbits = ng.y;
        ng = make_uint2(0u, 0u);
    }
    while (tbits)
    {
        uint32_t tb = 31u - __clz(tbits);
        tbits &= ~(1u << tb);
        int ti = (int)(tbase + tb);
        const float4* tp = reinterpret_cast<const float4*>(sc.tris + ti);
        float4 a = __ldg(tp), bq = __ldg(tp + 1), c = __ldg(tp + 2);
        int prim = __float_as_int(a.w);
        float t, u, v;
        if (triTests) ++*triTests;
        if (tri_test(r, f3(a.x, a.y, a.z), f3(bq.x, bq.y, bq.z), f3(c.x, c.y, c.z), tnear, s.tHit, prim, s.primHit,
                     t, u, v))
        {
            s.tHit = t;
            s.primHit = prim;
            s.uHit = u;
            s.vHit = v;
            s.triHit = ti;
            if (anyHit || anyHitRt)
            {
                s.done = true;
                return;
            }
        }
    }
    if (!(ng.y & 0xff000000u))
    {
        if (st.sp == 0)
        {
            s.done = true;
            return;
        }
        ng = st.pop();   // a node group, or a postponed triangle group (bits 0..23 only)
    }
    s.ng = ng;
}

// ---- deferred triangle tests -------------------------------------------------
//
// With one-triangle leaves a node visit finds a triangle for only a few lanes
// of a warp, so testing triangles in the visiting lane runs the test with ~3 of
// 32 lanes.  In the deferred mode a node visit only queues its hit triangles
// (leaf-order index + owner lane) in a per-warp ring in shared memory; once 32
// are pending, the whole warp tests them, one per lane, with the owner's ray
// fetched by shuffles, and the owners' closest hits are merged with one 64-bit
// shared-memory atomicMin on (t bits, primitive id): positive floats order as
// their bit patterns and the id breaks exact ties the way tri_test does.  Node
// culling uses the owner's tHit as of the last merge, which can only be larger
// than the final one, so no node that holds the closest hit is skipped.
#ifndef PRT_DEFER_TRIS
#define PRT_DEFER_TRIS 1
#endif
#ifndef PRT_DEFER_FLUSH
#define PRT_DEFER_FLUSH 32
#endif

constexpr uint32_t kTriQCap = 512;   // > 31 pending + 8 triangles x 32 lanes from one step
constexpr uint32_t kTriQMask = kTriQCap - 1;

struct TriQueue
{
    unsigned long long key[32];   // per owner lane: (t bits << 32) | primitive id
    uint32_t tri[kTriQCap];       // leaf-order triangle index << 5 | owner lane
    float u[32], v[32];
    int ti[32];
};

__device__ __forceinline__ unsigned long long hit_key(float t, int prim)
{
    return ((unsigned long long)__float_as_uint(t) << 32) | (uint32_t)prim;
}

// One node visit of the deferred mode: returns the node's hit triangles
// (tbase + set bits of tbits) instead of testing them.
#ifndef PRT_LEAF1_HITS
#define PRT_LEAF1_HITS 1
#endif

// tbits: the hit leaf slots (PRT_LEAF1_HITS) with the node's leaf-slot mask in
// leafMask, or triangle offset bits with leafMask = 0.
template <bool kPair = false>
__device__ __forceinline__ void trav_visit(TravState& s, const SceneDev& sc, const TravRay& r, float tnear, TravStack& st,
                                           uint32_t& tbase, uint32_t& tbits, uint32_t& leafMask,
                                           uint32_t* nodeVisits = nullptr)
{
    uint2 ng = s.ng;
    uint32_t b = 31u - __clz(ng.y & 0xff000000u);
    ng.y &= ~(1u << b);
    uint32_t slot = (b - 24u) ^ r.octinv;
    uint32_t rel = __popc((ng.y & 0xffu) & ((1u << slot) - 1u));
    uint32_t nodeIdx = ng.x + rel;
    if (ng.y & 0xff000000u) st.push(ng);
    const uint4* qp = reinterpret_cast<const uint4*>(sc.nodes + nodeIdx);
    uint4 q[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) q[k] = __ldg(qp + k);
    uint32_t hits;
    if (PRT_LEAF1_HITS)
    {
        hits = node_hits1<kPair>(r, q, tnear, s.tHit, leafMask, r.octinv);
    }
    else
    {
        hits = node_hits(r, q, tnear, s.tHit);
        leafMask = 0;
    }
    if (nodeVisits) ++*nodeVisits;
    ng = make_uint2(q[1].x, (hits & 0xff000000u) | (q[0].w >> 24));
    tbits = hits & 0x00ffffffu;
    tbase = q[1].y;
    if (!(ng.y & 0xff000000u))
    {
        if (st.sp == 0)
        {
            s.done = true;
            s.ng = ng;
            return;
        }
        ng = st.pop();
    }
    s.ng = ng;
}

// Warp-collective: appends every lane's triangles to the ring at tail
// (leafMask != 0: tbits are leaf slots, see trav_visit).
__device__ __forceinline__ void triq_push(TriQueue& q, uint32_t& tail, uint32_t tbase, uint32_t tbits, uint32_t leafMask,
                                          unsigned lane)
{
    const unsigned FULL = 0xffffffffu;
    const uint32_t n = __popc(tbits);
    uint32_t x = n;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        const uint32_t y = __shfl_up_sync(FULL, x, off);
        if ((int)lane >= off) x += y;
    }
    uint32_t pos = tail + x - n;
    while (tbits)
    {
        const uint32_t bit = __ffs(tbits) - 1u;
        tbits &= tbits - 1u;
        q.tri[pos & kTriQMask] = ((tbase + (leafMask ? __popc(leafMask & ((1u << bit) - 1u)) : bit)) << 5) | lane;
        ++pos;
    }
    tail += __shfl_sync(FULL, x, 31);
}

// Warp-collective: tests the m (<= 32) oldest queued triangles, one per lane,
// and merges each owner's closest hit into its traversal state.  The owner's
// ray, tnear and triangle array (lanes of a batch may traverse different
// scenes) come from the owner lane by shuffles.
__device__ __forceinline__ void triq_flush(TriQueue& q, uint32_t& head, uint32_t m, const TriRec* tris, const TravRay& r,
                                           float tnear, TravState& ts, unsigned lane, uint32_t* triTests = nullptr)
{
    const unsigned FULL = 0xffffffffu;
    const bool act = lane < m;
    uint32_t tri = 0;
    int own = 0;
    if (act)
    {
        const uint32_t e = q.tri[(head + lane) & kTriQMask];
        tri = e >> 5;
        own = (int)(e & 31u);
    }
    head += m;
    TravRay o;
    o.org.x = __shfl_sync(FULL, r.org.x, own);
    o.org.y = __shfl_sync(FULL, r.org.y, own);
    o.org.z = __shfl_sync(FULL, r.org.z, own);
    o.Sx = __shfl_sync(FULL, r.Sx, own);
    o.Sy = __shfl_sync(FULL, r.Sy, own);
    o.Sz = __shfl_sync(FULL, r.Sz, own);
    const int kp = __shfl_sync(FULL, r.kx | (r.ky << 2) | (r.kz << 4), own);
    o.kx = kp & 3;
    o.ky = (kp >> 2) & 3;
    o.kz = kp >> 4;
    const float tb = __shfl_sync(FULL, ts.tHit, own);
    const int bp = __shfl_sync(FULL, ts.primHit, own);
    const float tn = __shfl_sync(FULL, tnear, own);
    const TriRec* otris = reinterpret_cast<const TriRec*>(
        __shfl_sync(FULL, reinterpret_cast<unsigned long long>(tris), own));
    const unsigned long long mine = hit_key(ts.tHit, ts.primHit);
    q.key[lane] = mine;
    __syncwarp();
    bool hit = false;
    float t = 0.f, u = 0.f, v = 0.f;
    int prim = 0;
    if (act)
    {
        const float4* tp = reinterpret_cast<const float4*>(otris + tri);
        const float4 a = __ldg(tp), bq = __ldg(tp + 1), c = __ldg(tp + 2);
        prim = __float_as_int(a.w);
        if (triTests) ++*triTests;
        hit = tri_test(o, f3(a.x, a.y, a.z), f3(bq.x, bq.y, bq.z), f3(c.x, c.y, c.z), tn, tb, prim, bp, t, u, v);
        if (hit) atomicMin(&q.key[own], hit_key(t, prim));
    }
    __syncwarp();
    if (hit && q.key[own] == hit_key(t, prim))
    {
        q.u[own] = u;
        q.v[own] = v;
        q.ti[own] = (int)tri;
    }
    __syncwarp();
    const unsigned long long k = q.key[lane];
    if (k != mine)
    {
        ts.tHit = __uint_as_float((uint32_t)(k >> 32));
        ts.primHit = (int)(uint32_t)k;
        ts.uHit = q.u[lane];
        ts.vHit = q.v[lane];
        ts.triHit = q.ti[lane];
    }
    __syncwarp();
}

// Warp-collective traversal with deferred triangle tests, for trees with
// one-triangle leaves: runs node steps until no lane of the warp is traversing
// or, when mayStop, until refillMin lanes are idle; every queued test is merged
// before it returns.  active: this lane holds a ray.  anyHit: this lane's ray
// is an occlusion query, which stops at the first merged hit (its later queued
// tests are still merged, which can only move the hit nearer).  The counter
// pointers (node visits, triangle tests per lane; steps, running-lane steps and
// flushes per warp) may be null.
template <bool kPair = false>
__device__ __forceinline__ void warp_trav_deferred(TriQueue& q, TravState& ts, const SceneDev& sc, const TravRay& r,
                                                   float tnear, TravStack& st, bool active, bool mayStop, int refillMin,
                                                   unsigned lane, uint32_t* cNodes = nullptr, uint32_t* cTris = nullptr,
                                                   unsigned long long* cSteps = nullptr,
                                                   unsigned long long* cLaneSteps = nullptr,
                                                   unsigned long long* cFlushes = nullptr, bool anyHit = false)
{
    const unsigned FULL = 0xffffffffu;
    uint32_t head = 0, tail = 0;
    for (;;)
    {
        uint32_t tbase = 0, tbits = 0, lmask = 0;
        if (cSteps)
        {
            *cLaneSteps += __popc(__ballot_sync(FULL, active && !ts.done));
            *cSteps += 1;
        }
        if (active && !ts.done) trav_visit<kPair>(ts, sc, r, tnear, st, tbase, tbits, lmask, cNodes);
        if (__any_sync(FULL, tbits != 0)) triq_push(q, tail, tbase, tbits, lmask, lane);
        while (tail - head >= (uint32_t)PRT_DEFER_FLUSH)
        {
            triq_flush(q, head, min(32u, tail - head), sc.tris, r, tnear, ts, lane, cTris);
            if (cFlushes) *cFlushes += 1;
            if (anyHit && ts.triHit >= 0) ts.done = true;
        }
        const unsigned running = __ballot_sync(FULL, active && !ts.done);
        if (running == 0) break;
        if (mayStop && 32 - __popc(running) >= refillMin) break;
    }
    while (tail != head)
    {
        triq_flush(q, head, min(32u, tail - head), sc.tris, r, tnear, ts, lane, cTris);
        if (cFlushes) *cFlushes += 1;
    }
}

// Closest hit (anyHit = false) or any hit (anyHit = true) over (tnear, tfar].
// Returns the leaf-order triangle index of the hit (or -1), with t/u/v/prim.
template <bool anyHit>
__device__ __forceinline__ int traverse(const SceneDev& sc, const TravRay& r, float tnear, float tfar, TravStack& st,
                                        float& tHit, int& primHit, float& uHit, float& vHit)
{
    TravState s;
    trav_init(s, sc, tfar, st);
    while (!s.done) trav_step<anyHit>(s, sc, r, tnear, st);
    tHit = s.tHit;
    primHit = s.primHit;
    uHit = s.uHit;
    vHit = s.vHit;
    return s.triHit;
}

// Post-intersection shading and the diffuse bounce
// (geometry/triangle_mesh.cpp:59-100 + render/diffuse_integrator_single.h:57-63):
// hit point, eps = max(t, max|p|) * 0x1.fp-18 (core/ray.h:71-76), geometric
// normal flipped against the ray, frame from makeFrame (math/basis3.h:128-137),
// cosine-weighted direction (sampling/shape_sampler.h:50-74), and the origin
// offset by eps along the new direction (core/ray.h:47-52).
// Shading frame of a hit: point p, offset eps, geometric normal N facing the
// ray, and the tangents U, V of makeFrame.
struct HitFrame
{
    float3 p;
    float eps;
    float3 U, V, N;
};

__device__ __forceinline__ HitFrame hit_frame(const TriRec* tris, int triIdx, float3 org, float3 dir, float t)
{
    HitFrame h;
    h.p = madd(org, t, dir);
    float m = fmaxf(fabsf(h.p.x), fmaxf(fabsf(h.p.y), fabsf(h.p.z)));
    h.eps = __fmul_rn(fmaxf(t, m), 0x1.fp-18f);
    const float4* tp = reinterpret_cast<const float4*>(tris + triIdx);
    float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
    float3 p0 = f3(a.x, a.y, a.z), p1 = f3(b.x, b.y, b.z), p2 = f3(c.x, c.y, c.z);
    float3 Ng = normalize(cross(sub(p1, p0), sub(p2, p0)));
    if (dot(Ng, dir) > 0.0f) Ng = f3(-Ng.x, -Ng.y, -Ng.z);
    // makeFrame
    float3 U0 = f3(0.0f, Ng.z, -Ng.y);
    float3 U1 = f3(-Ng.z, 0.0f, Ng.x);
    h.U = normalize(dot(U0, U0) > dot(U1, U1) ? U0 : U1);
    h.V = normalize(cross(Ng, h.U));
    h.N = Ng;
    return h;
}

// A cosine-weighted direction about the frame (two RNG draws) and the ray
// origin offset along it.
__device__ __forceinline__ void sample_bounce(const HitFrame& h, uint32_t& rng, float3& org, float3& dir)
{
    float sx = rng_next(rng);
    float sy = rng_next(rng);
    float cosT = __fsqrt_rn(sx);
    float sinT = __fsqrt_rn(__fsub_rn(1.0f, sx));
    float sphi, cphi;
    sincosf(__fmul_rn(2.0f * 3.14159265358979f, sy), &sphi, &cphi);
    float lx = __fmul_rn(cphi, sinT), ly = __fmul_rn(sphi, sinT);
    dir = add(add(mul(h.U, lx), mul(h.V, ly)), mul(h.N, cosT));
    org = madd(h.p, h.eps, dir);
}

__device__ __forceinline__ void diffuse_bounce(const TriRec* tris, int triIdx, float3& org, float3& dir, float t,
                                               uint32_t& rng)
{
    HitFrame h = hit_frame(tris, triIdx, org, dir, t);
    sample_bounce(h, rng, org, dir);
}

// Fire-and-forget vector add into the accumulation buffer (sm_90+).
__device__ __forceinline__ void red_add_v4(float4* addr, float a, float b, float c, float d)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

} // namespace prt_b200
