// Driver around ProtoRay's own CPU renderers — TEST / BASELINE INFRASTRUCTURE ONLY.
//
// This file is compiled together with the reference's unmodified sources
// (renderers, integrators, samplers, cameras, scene and .mesh loader, frame
// buffer) into oracle/_ref/libprotoray_ref.so by oracle/Makefile.  It exposes
// a small C interface that the test suite uses to generate golden vectors and
// that the benchmark's CPU-baseline leg uses to time the reference renderers.
//
// The reference renderers reach their acceleration structure through
// IntersectorSingle / IntersectorStream<N> (core/intersector_single.h:23-31,
// core/intersector_stream.h:23-31).  Their only implementations in the
// reference are Embree 3 wrappers (accel/embree/*), and Embree is absent here,
// so project intersectors implement those interfaces instead:
//   * OracleIntersector: the FP64 watertight BVH of prt_oracle.c (parity);
//   * FastIntersector over the 8-wide AVX2 BVH with 4-triangle leaves of
//     cpu_bvh8.hpp (timing; the class of structure the reference asks Embree
//     for, bvh8.triangle4), or over the scalar binary FP32 BVH of
//     cpu_bvh32.hpp (timing, for comparison).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "render/scene.h"
#include "render/renderer_single.h"
#include "render/diffuse_integrator_single.h"
#include "render/diffuse2_integrator_single.h"
#include "render/diffuse_renderer_stream.h"
#include "sampling/random_sampler.h"
#include "sampling/random_sampler_simd.h"
#include "camera/pinhole_camera.h"
#include "camera/thin_lens_camera.h"
#include "core/intersector_single.h"
#include "core/intersector_stream.h"
#include "image/frame_buffer.h"
#include "main/build/obj_loader.h"
#include "geometry/triangle_mesh_builder.h"
#include "sys/blob.h"

#include "prt_oracle.h"
#include "cpu_bvh32.hpp"
#include "cpu_bvh8.hpp"

using namespace prt;

namespace {

const int kStream = 2048;   // defaultRayStreamSize on AVX2 (core/ray_stream.h:27-35)

struct SceneHandle
{
    ref<Scene> scene;
    std::vector<float> pos;
    std::vector<int> idx;
    or_scene* fp64 = nullptr;
    prt_oracle::Bvh32 bvh;
    prt_oracle::Bvh8 bvh8;
    bool bvh8Built = false;
    std::string error;
};

class OracleIntersector : public IntersectorSingle
{
    const or_scene* s;

public:
    explicit OracleIntersector(const or_scene* s) : s(s) {}

    void intersect(Ray& ray, Hit& hit, RayStats& stats, RayHint) override
    {
        stats.rayCount++;
        double org[3] = {ray.org.x, ray.org.y, ray.org.z};
        double dir[3] = {ray.dir.x, ray.dir.y, ray.dir.z};
        or_hit h;
        if (or_intersect(s, org, dir, 0.0, (double)ray.far, &h))
        {
            ray.far = (float)h.t;
            hit.primId = h.primId;
            hit.u = (float)h.u;
            hit.v = (float)h.v;
        }
    }

    void occluded(Ray& ray, RayStats& stats, RayHint) override
    {
        stats.rayCount++;
        double org[3] = {ray.org.x, ray.org.y, ray.org.z};
        double dir[3] = {ray.dir.x, ray.dir.y, ray.dir.z};
        if (or_occluded(s, org, dir, 0.0, (double)ray.far)) ray.far = 0.0f;
    }
};

// Closest-hit / any-hit queries of the two timing BVHs behind one interface.
struct FastBvh
{
    const prt_oracle::Bvh32* b32 = nullptr;
    const prt_oracle::Bvh8* b8 = nullptr;

    bool intersect(const float org[3], const float dir[3], float& t, int& prim, float& u, float& v) const
    {
        return b8 ? b8->intersect(org, dir, t, prim, u, v) : b32->intersect(org, dir, t, prim, u, v);
    }
    bool occluded(const float org[3], const float dir[3], float t) const
    {
        if (b8) return b8->occluded(org, dir, t);
        float u, v;
        int prim;
        return b32->intersect(org, dir, t, prim, u, v);
    }
};

class FastIntersectorSingle : public IntersectorSingle
{
    FastBvh bvh;

public:
    explicit FastIntersectorSingle(FastBvh b) : bvh(b) {}

    void intersect(Ray& ray, Hit& hit, RayStats& stats, RayHint) override
    {
        stats.rayCount++;
        float org[3] = {ray.org.x, ray.org.y, ray.org.z}, dir[3] = {ray.dir.x, ray.dir.y, ray.dir.z};
        float t = ray.far, u = 0, v = 0;
        int prim = -1;
        if (bvh.intersect(org, dir, t, prim, u, v))
        {
            ray.far = t;
            hit.primId = prim;
            hit.u = u;
            hit.v = v;
        }
    }

    void occluded(Ray& ray, RayStats& stats, RayHint) override
    {
        stats.rayCount++;
        float org[3] = {ray.org.x, ray.org.y, ray.org.z}, dir[3] = {ray.dir.x, ray.dir.y, ray.dir.z};
        if (bvh.occluded(org, dir, ray.far)) ray.far = 0.0f;
    }
};

// The stream interface of the reference's stream renderers, one ray at a time
// (Embree's rtcIntersectNp traverses incoherent streams ray by ray as well).
template <int N>
class FastIntersectorStream : public IntersectorStream<N>
{
    FastBvh bvh;

public:
    explicit FastIntersectorStream(FastBvh b) : bvh(b) {}

    void intersect(RayStream<N>& rays, HitStream<N>& hits, int count, RayStats& stats, RayHint) override
    {
        stats.rayCount += count;
        float* ox = rays.getOrgX(); float* oy = rays.getOrgY(); float* oz = rays.getOrgZ();
        float* dx = rays.getDirX(); float* dy = rays.getDirY(); float* dz = rays.getDirZ();
        float* far = rays.getFar();
        int* pid = hits.getPrimId(); float* hu = hits.getU(); float* hv = hits.getV();
        for (int i = 0; i < count; ++i)
        {
            float org[3] = {ox[i], oy[i], oz[i]}, dir[3] = {dx[i], dy[i], dz[i]};
            float t = far[i], u = 0, v = 0;
            int prim = -1;
            if (bvh.intersect(org, dir, t, prim, u, v))
            {
                far[i] = t;
                pid[i] = prim;
                hu[i] = u;
                hv[i] = v;
            }
        }
    }

    void occluded(RayStream<N>& rays, int count, RayStats& stats, RayHint) override
    {
        stats.rayCount += count;
        for (int i = 0; i < count; ++i)
        {
            float org[3] = {rays.getOrgX()[i], rays.getOrgY()[i], rays.getOrgZ()[i]};
            float dir[3] = {rays.getDirX()[i], rays.getDirY()[i], rays.getDirZ()[i]};
            if (bvh.occluded(org, dir, rays.getFar()[i])) rays.getFar()[i] = 0.0f;
        }
    }
};

// Raw sums/weights of the reference accumulation buffer (protected members,
// image/accum_buffer.h:36-40) read through a member pointer of a derived type.
struct AccumPeek : AccumBuffer3f
{
    static float* const* sums(const AccumBuffer3f& a) { return a.*(&AccumPeek::sum); }
    static const float* weights(const AccumBuffer3f& a) { return a.*(&AccumPeek::weight); }
};

Basis3f viewBasis(float angleX, float angleY)
{
    // main/render/render_window.cpp:309
    return Basis3f(one).rotateV(angleY).rotateU(angleX);
}

Props cameraProps(const float view[8], int W, int H)
{
    Props camera;
    camera.set("type", view[6] == 0.0f ? "pinhole" : "thinlens");
    camera.set("position", Vec3f(view[0], view[1], view[2]));
    camera.set("basis", viewBasis(view[3], view[4]));
    camera.set("fov", view[5]);
    camera.set("aspectRatio", (float)W / (float)H);
    camera.set("lensRadius", view[6]);
    camera.set("focalDistance", view[7]);
    return camera;
}

// render/device_cpu_impl.cpp:86-97
Camera* makeCamera(const Props& p)
{
    std::string type = p.get<std::string>("type");
    float lensRadius = p.get("lensRadius", 0.0f);
    if (type == "pinhole" || lensRadius == 0.0f) return new PinholeCamera(p);
    return new ThinLensCamera(p);
}

} // namespace

extern "C" {

void* ref_scene_open(const char* path, char* err, int errlen)
{
    try
    {
        SceneHandle* h = new SceneHandle;
        Props props;
        h->scene = makeRef<Scene>(std::string(path), props);
        const TriangleMesh& m = *h->scene->shape;
        int nt = m.getPrimCount(), nv = m.getVertexCount();
        h->idx.resize(3 * (size_t)nt);
        std::memcpy(h->idx.data(), m.indices.getData(), sizeof(int) * 3 * (size_t)nt);
        h->pos.resize(3 * (size_t)nv);
        for (int i = 0; i < nv; ++i)
        {
            Vec3f p = m.getPosition(i);
            h->pos[3 * i + 0] = p.x; h->pos[3 * i + 1] = p.y; h->pos[3 * i + 2] = p.z;
        }
        return h;
    }
    catch (const std::exception& e)
    {
        if (err && errlen > 0) { std::snprintf(err, errlen, "%s", e.what()); }
        return nullptr;
    }
}

void ref_scene_close(void* handle)
{
    SceneHandle* h = (SceneHandle*)handle;
    if (!h) return;
    or_scene_destroy(h->fp64);
    delete h;
}

int ref_scene_info(void* handle, int* triCount, int* vertCount, float* lo, float* hi)
{
    SceneHandle* h = (SceneHandle*)handle;
    Box3f b = h->scene->getBounds();
    *triCount = h->scene->shape->getPrimCount();
    *vertCount = h->scene->shape->getVertexCount();
    lo[0] = b.low.x; lo[1] = b.low.y; lo[2] = b.low.z;
    hi[0] = b.high.x; hi[1] = b.high.y; hi[2] = b.high.z;
    return 0;
}

// Copies the loaded mesh (positions, indices) so tests can compare it with the writer.
void ref_scene_arrays(void* handle, float* pos, int* idx)
{
    SceneHandle* h = (SceneHandle*)handle;
    std::memcpy(pos, h->pos.data(), sizeof(float) * h->pos.size());
    std::memcpy(idx, h->idx.data(), sizeof(int) * h->idx.size());
}

// accel: 0 = FP64 oracle BVH, 1 = 8-wide AVX2 BVH (4-triangle leaves),
// 2 = scalar binary FP32 SAH BVH.  Returns build seconds.
double ref_scene_build(void* handle, int accel)
{
    SceneHandle* h = (SceneHandle*)handle;
    auto t0 = std::chrono::steady_clock::now();
    int nt = (int)(h->idx.size() / 3), nv = (int)(h->pos.size() / 3);
    if (accel == 0 && !h->fp64) h->fp64 = or_scene_create(h->pos.data(), nv, h->idx.data(), nt);
    if (accel == 1 && !h->bvh8Built)
    {
        h->bvh8.build(h->pos.data(), h->idx.data(), nt);
        h->bvh8Built = true;
    }
    if (accel == 2 && h->bvh.nodes.empty()) h->bvh.build(h->pos.data(), h->idx.data(), nt);
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Renders `frames` frames with a reference renderer, one sample per pixel per
// frame as the reference's render loop does (main/render/render_window.cpp:204-256).
//   renderer: "diffuse", "diffuseFast", "diffuse2", "diffuse2Fast", "diffuseStream", "diffuseStreamFast"
//   accel:    0 = FP64 oracle BVH, 1 = 8-wide AVX2 BVH, 2 = scalar binary FP32 BVH
//   view:     {pos.xyz, angleX, angleY, fovY, radius, focus}
//   sums:     W*H*4 floats (r,g,b,weight) or NULL
//   stats:    [0] rays, [1] seconds (sum of the renderer's own frame timers),
//             [2] Mrays/s averaged over frames after dropping the first frames/6
// Returns 0 on success, -1 on error (message in err).
int ref_render(void* handle, const char* renderer, int accel, int W, int H, int frames, int maxDepth,
               const float view[8], float* sums, double* stats, char* err, int errlen)
{
    SceneHandle* h = (SceneHandle*)handle;
    try
    {
        ref_scene_build(handle, accel);
        FastBvh fast;
        if (accel == 1) fast.b8 = &h->bvh8;
        else fast.b32 = &h->bvh;
        std::string type(renderer);
        Props props;
        props.set("type", type);
        props.set("imageSize", Vec2i(W, H));
        props.set("spp", frames);
        props.set("maxDepth", maxDepth);

        Props cam = cameraProps(view, W, H);
        std::unique_ptr<Camera> camera(makeCamera(cam));
        FrameBuffer fb(Vec2i(W, H), 0);
        fb.clear();

        ref<const Scene> scene = h->scene;
        ref<Renderer> r;
        if (type == "diffuse2" || type == "diffuse2Fast")
        {
            ref<IntersectorSingle> isect;
            if (accel == 0) isect = makeRef<OracleIntersector>(h->fp64);
            else isect = makeRef<FastIntersectorSingle>(fast);
            // render/renderer_factory_single.cpp (diffuse2 / diffuse2Fast)
            if (type == "diffuse2")
                r = makeRef<RendererSingle<Diffuse2IntegratorSingle<ShadingContext, RandomSampler>, RandomSampler>>(scene, isect, props);
            else
                r = makeRef<RendererSingle<Diffuse2IntegratorSingle<SimpleShadingContext, RandomSampler>, RandomSampler, false>>(scene, isect, props);
        }
        else if (type == "diffuse" || type == "diffuseFast")
        {
            ref<IntersectorSingle> isect;
            if (accel == 0) isect = makeRef<OracleIntersector>(h->fp64);
            else isect = makeRef<FastIntersectorSingle>(fast);
            // render/renderer_factory_single.cpp:56-59
            if (type == "diffuse")
                r = makeRef<RendererSingle<DiffuseIntegratorSingle<ShadingContext, RandomSampler>, RandomSampler>>(scene, isect, props);
            else
                r = makeRef<RendererSingle<DiffuseIntegratorSingle<SimpleShadingContext, RandomSampler>, RandomSampler, false>>(scene, isect, props);
        }
        else if (type == "diffuseStream" || type == "diffuseStreamFast")
        {
            if (accel == 0) throw std::invalid_argument("stream renderers use a FP32 BVH (accel 1 or 2)");
            ref<IntersectorStream<kStream>> isect = makeRef<FastIntersectorStream<kStream>>(fast);
            // render/renderer_factory_stream.cpp:91-94 (streamTileX 64, streamTileY 2048/64)
            if (type == "diffuseStream")
                r = makeRef<DiffuseRendererStream<ShadingContextSimd, RandomSamplerSimd, true, kStream, 64, kStream / 64>>(scene, isect, props);
            else
                r = makeRef<DiffuseRendererStream<SimpleShadingContextSimd, RandomSamplerSimd, false, kStream, 64, kStream / 64>>(scene, isect, props);
        }
        else
        {
            throw std::invalid_argument("invalid renderer type");
        }

        double rays = 0, seconds = 0, mraySum = 0;
        int counted = 0;
        int warmup = frames / 6;   // main/render/render_window.cpp:43,262
        for (int f = 0; f < frames; ++f)
        {
            Props st;
            r->render(camera.get(), &fb, st);
            double ray = (double)st.get<int64_t>("ray");
            double mray = st.get<double>("mray");
            rays += ray;
            if (mray > 0) seconds += ray / (mray * 1e6);
            if (f + 1 > warmup) { mraySum += mray; counted++; }
        }
        if (stats)
        {
            stats[0] = rays;
            stats[1] = seconds;
            stats[2] = counted ? mraySum / counted : 0.0;
        }
        if (sums)
        {
            float* const* s = AccumPeek::sums(fb.getColor());
            const float* w = AccumPeek::weights(fb.getColor());
            for (int i = 0; i < W * H; ++i)
            {
                sums[4 * i + 0] = s[0][i];
                sums[4 * i + 1] = s[1][i];
                sums[4 * i + 2] = s[2][i];
                sums[4 * i + 3] = w[i];
            }
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
        return -1;
    }
}

// Primary-hit query through RendererSingle::queryRay (render/renderer_single.h:137-163).
// ray: {org.xyz, dir.xyz, far}; out: {primId, dist, p.xyz, Ng.xyz}.  Returns 1 on hit.
int ref_query_ray(void* handle, const float ray[7], float* out)
{
    SceneHandle* h = (SceneHandle*)handle;
    ref_scene_build(handle, 0);
    Props props;
    props.set("imageSize", Vec2i(8, 8));
    ref<IntersectorSingle> isect = makeRef<OracleIntersector>(h->fp64);
    RendererSingle<DiffuseIntegratorSingle<ShadingContext, RandomSampler>, RandomSampler> r(h->scene, isect, props);
    Ray rr;
    rr.org = Vec3f(ray[0], ray[1], ray[2]);
    rr.dir = Vec3f(ray[3], ray[4], ray[5]);
    rr.far = ray[6];
    Props res = r.queryRay(rr);
    if (res.isEmpty()) return 0;
    out[0] = (float)res.get<int>("primId");
    out[1] = res.get<float>("dist");
    Vec3f p = res.get<Vec3f>("p"), Ng = res.get<Vec3f>("Ng");
    out[2] = p.x; out[3] = p.y; out[4] = p.z;
    out[5] = Ng.x; out[6] = Ng.y; out[7] = Ng.z;
    return 1;
}

// Closest hits (accel 1 or 2) or occlusion (any != 0) of n rays through a
// timing BVH, for checking it against the FP64 oracle.  rays: n x 8 floats
// (org, tnear ignored, dir, tfar); out: n x 4 floats (t or -1, primId bits,
// u, v), or n floats (1 occluded, 0 free) for occlusion.
void ref_fast_trace(void* handle, int accel, int any, const float* rays, int n, float* out)
{
    SceneHandle* h = (SceneHandle*)handle;
    ref_scene_build(handle, accel);
    FastBvh fast;
    if (accel == 1) fast.b8 = &h->bvh8;
    else fast.b32 = &h->bvh;
    for (int i = 0; i < n; ++i)
    {
        const float* r = rays + 8 * (size_t)i;
        float org[3] = {r[0], r[1], r[2]}, dir[3] = {r[4], r[5], r[6]};
        if (any)
        {
            out[i] = fast.occluded(org, dir, r[7]) ? 1.0f : 0.0f;
            continue;
        }
        float t = r[7], u = 0, v = 0;
        int prim = -1;
        float* o = out + 4 * (size_t)i;
        if (fast.intersect(org, dir, t, prim, u, v))
        {
            o[0] = t;
            std::memcpy(&o[1], &prim, 4);
            o[2] = u;
            o[3] = v;
        }
        else
        {
            o[0] = -1.0f;
            std::memcpy(&o[1], &prim, 4);
            o[2] = o[3] = 0.0f;
        }
    }
}

// `protoray build` of the reference, split at its two seams so that each can
// be compared on its own: ObjLoader::load (main/build/obj_loader.cpp:35-53)
// and TriangleMeshBuilder + saveBlob (geometry/triangle_mesh_builder.cpp:23-44,
// main/build/build.cpp:98-118).
static_assert(sizeof(FatTriangle) == 100, "FatTriangle is 3 x 32-byte vertices + matId");

struct RefSoup
{
    TriangleSoup soup;
};

// Parses an OBJ file.  Returns nullptr when ObjLoader::load returns false.
void* ref_obj_load(const char* path, int* triCount, int* nameCount, int* nameBytes)
{
    RefSoup* h = new RefSoup;
    ObjLoader loader;
    if (!loader.load(path, h->soup))
    {
        delete h;
        return nullptr;
    }
    *triCount = (int)h->soup.triangles.getSize();
    *nameCount = (int)h->soup.materialNames.getSize();
    size_t bytes = 0;
    for (int i = 0; i < *nameCount; ++i) bytes += h->soup.materialNames[i].size() + 1;
    *nameBytes = (int)bytes;
    return h;
}

// Copies the soup out: FatTriangle records, and the material names each
// followed by a '\n'.
void ref_soup_get(void* handle, void* tris, char* names)
{
    RefSoup* h = (RefSoup*)handle;
    std::memcpy(tris, h->soup.triangles.getData(), sizeof(FatTriangle) * (size_t)h->soup.triangles.getSize());
    for (int i = 0; i < (int)h->soup.materialNames.getSize(); ++i)
    {
        const std::string& s = h->soup.materialNames[i];
        std::memcpy(names, s.data(), s.size());
        names += s.size();
        *names++ = '\n';
    }
}

void ref_soup_free(void* handle) { delete (RefSoup*)handle; }

// TriangleMeshBuilder over a soup given as FatTriangle records and
// '\n'-terminated material names; writes the .mesh blob and returns the
// builder's own time in milliseconds (negative on failure).
double ref_build_soup(const void* tris, int n, const char* names, int nameCount, const char* meshPath)
{
    try
    {
        TriangleSoup soup;
        soup.triangles.alloc(n);
        std::memcpy(soup.triangles.getData(), tris, sizeof(FatTriangle) * (size_t)n);
        const char* p = names;
        for (int i = 0; i < nameCount; ++i)
        {
            const char* e = std::strchr(p, '\n');
            soup.materialNames.pushBack(std::string(p, e - p));
            p = e + 1;
        }
        TriangleMesh mesh;
        auto t0 = std::chrono::steady_clock::now();
        TriangleMeshBuilder(soup, mesh);
        auto t1 = std::chrono::steady_clock::now();
        saveBlob(meshPath, mesh);
        return std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    catch (const std::exception&)
    {
        return -1.0;
    }
}

// ---- known-answer vectors from the reference's own code ----

// RandomSampler::setSample + n get1D draws (sampling/random_sampler.h:44-63).
void ref_rng(int pass, int pixel, int n, unsigned* states, float* values)
{
    RandomSampler s;
    s.init(4, 0, 1);
    RandomSampler::State st;
    s.setSample(st, pass, pixel);
    if (n > 0) states[0] = st.s;
    for (int i = 0; i < n; ++i)
    {
        values[i] = s.get1D(st, i);
        states[i + 1] = st.s;
    }
}

// Camera fields (camera/pinhole_camera.h:34-47, camera/thin_lens_camera.h:29-36):
// out = origin, U, V, N, imageO, imageDx, imageDy (7 x 3 floats), lensRadius, focalDistance.
void ref_camera(const float view[8], int W, int H, float* out)
{
    Props p = cameraProps(view, W, H);
    ThinLensCamera c(p);
    Vec3f v[7] = {c.origin, c.basis.U, c.basis.V, c.basis.N, c.imageO, c.imageDx, c.imageDy};
    for (int i = 0; i < 7; ++i) { out[3 * i] = v[i].x; out[3 * i + 1] = v[i].y; out[3 * i + 2] = v[i].z; }
    out[21] = c.lensRadius;
    out[22] = c.focalDistance;
}

// Primary rays exactly as RendererSingle::renderTile makes them for pass
// `pass` (render/renderer_single.h:107-124), in raster order; 8 floats per
// ray {org.xyz, 0, dir.xyz, far}.
void ref_primary_rays(const float view[8], int W, int H, int pass, float* rays)
{
    Props cp = cameraProps(view, W, H);
    std::unique_ptr<Camera> camera(makeCamera(cp));
    FrameBuffer fb(Vec2i(W, H), 0);
    RandomSampler sampler;
    sampler.init(4, 0, W * H);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            Vec2i pixel(x, y);
            int pixelIndex = x + y * W;
            RandomSampler::State st;
            sampler.setSample(st, pass, pixelIndex);
            CameraSample cs;
            Vec2f ps = sampler.get2D(st, IntegratorBase::sampleDimPixel);
            cs.image = (toFloat(pixel) + ps) * fb.getInvSize();
            cs.lens = sampler.get2D(st, IntegratorBase::sampleDimLens);
            Ray ray;
            camera->getRay(ray, cs);
            float* r = rays + 8 * (size_t)pixelIndex;
            r[0] = ray.org.x; r[1] = ray.org.y; r[2] = ray.org.z; r[3] = 0.0f;
            r[4] = ray.dir.x; r[5] = ray.dir.y; r[6] = ray.dir.z; r[7] = ray.far;
        }
}

// cosineSampleHemisphere (sampling/shape_sampler.h:50-74)
void ref_cosine_sample(float sx, float sy, float* out)
{
    Vec3f d = cosineSampleHemisphere(Vec2f(sx, sy));
    out[0] = d.x; out[1] = d.y; out[2] = d.z;
}

// makeFrame (math/basis3.h:128-145); out = U, V
void ref_make_frame(const float N[3], float* out)
{
    Basis3f f = makeFrame(Vec3f(N[0], N[1], N[2]));
    out[0] = f.U.x; out[1] = f.U.y; out[2] = f.U.z;
    out[3] = f.V.x; out[4] = f.V.y; out[5] = f.V.z;
}

// TriangleMesh::postIntersect + the bounce of DiffuseIntegratorSingle
// (geometry/triangle_mesh.cpp:59-153, render/diffuse_integrator_single.h:57-63).
// ray: {org.xyz, dir.xyz}; out: p.xyz, eps, Ng.xyz, U.xyz, V.xyz, next org.xyz, next dir.xyz
void ref_shade(void* handle, const float ray[6], float t, int primId, float u, float v, float sx, float sy, float* out)
{
    SceneHandle* h = (SceneHandle*)handle;
    Ray r;
    r.org = Vec3f(ray[0], ray[1], ray[2]);
    r.dir = Vec3f(ray[3], ray[4], ray[5]);
    r.far = t;
    Hit hit;
    hit.primId = primId;
    hit.u = u;
    hit.v = v;
    ShadingContext ctx;
    h->scene->postIntersect(r, hit, ctx);
    Ray next;
    next.init(ctx.p, ctx.getFrame() * cosineSampleHemisphere(Vec2f(sx, sy)), ctx.eps);
    float vals[19] = {ctx.p.x, ctx.p.y, ctx.p.z, ctx.eps, ctx.Ng.x, ctx.Ng.y, ctx.Ng.z,
                      ctx.f.U.x, ctx.f.U.y, ctx.f.U.z, ctx.f.V.x, ctx.f.V.y, ctx.f.V.z,
                      next.org.x, next.org.y, next.org.z, next.dir.x, next.dir.y, next.dir.z};
    std::memcpy(out, vals, sizeof(vals));
}

} // extern "C"
