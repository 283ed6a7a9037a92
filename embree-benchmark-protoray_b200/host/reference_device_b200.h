// DeviceB200 for the reference tree: the class a maintainer adds beside
// render/device_cuda.{h,cpp} so that `protoray render ... -dev b200` runs the
// reference's own render loop on the B200 path tracer.  It is written against
// the reference's headers (Device, Props, ThinLensCamera, Surface) and the C
// ABI in include/prt_b200.h; main/render/render.cpp selects it with one
// more `-dev` branch (render.cpp:200-214).
#pragma once

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "render/device.h"
#include "camera/thin_lens_camera.h"
#include "prt_b200.h"

namespace prt {

class DeviceB200 : public Device
{
    prt_ctx* ctx = nullptr;
    int maxDepth = 6;
    int accumulate = 1;
    Vec2i size = Vec2i(0, 0);
    Box3f bounds;

    void check(int st) const
    {
        if (st == PRT_OK) return;
        std::string msg = ctx ? prt_last_error(ctx) : "prt_create failed";
        if (st == PRT_EINVAL) throw std::invalid_argument(msg);
        throw std::runtime_error(msg);
    }

public:
    DeviceB200() { check(prt_create(0, &ctx)); }
    ~DeviceB200() { prt_destroy(ctx); }

    std::string getInfo()
    {
        char b[256];
        check(prt_get_info(ctx, b, sizeof(b)));
        return b;
    }

    void initScene(const std::string& path, const Props&)
    {
        float lo[3], hi[3];
        check(prt_load_mesh_file(ctx, path.c_str(), lo, hi));
        bounds = Box3f(Vec3f(lo[0], lo[1], lo[2]), Vec3f(hi[0], hi[1], hi[2]));
    }

    Box3f getSceneBounds() { return bounds; }

    void initRenderer(const Props& props, Props& stats)
    {
        std::string type = props.get("type");
        if (type != "diffuse" && type != "diffuseFast" && type != "diffuse2" && type != "diffuse2Fast")
            throw std::invalid_argument("invalid renderer type");
        accumulate = type == "diffuse" || type == "diffuse2";
        check(prt_set_integrator(ctx, type.rfind("diffuse2", 0) == 0 ? PRT_INTEGRATOR_DIFFUSE2 : PRT_INTEGRATOR_DIFFUSE));
        maxDepth = props.get("maxDepth", 6);
        check(prt_set_build_quality(ctx, props.exists("no-sbvh") ? 0 : 1));
        prt_build_stats bs;
        check(prt_build_accel(ctx, &bs));
        stats.set("buildMs", bs.buildMs);
        stats.set("buildMprim", bs.buildMprim);
    }

    void render(Props& stats)
    {
        prt_render_stats rs;
        check(prt_render(ctx, 1, maxDepth, accumulate, &rs));   // one pass per frame
        stats.set("mray", rs.mray);
        stats.set("ray", (int64_t)rs.rays);
    }

    Props queryRay(const Ray& ray)
    {
        prt_ray r = {{ray.org.x, ray.org.y, ray.org.z}, 0.0f, {ray.dir.x, ray.dir.y, ray.dir.z}, ray.far};
        prt_hit h;
        float p[3], Ng[3];
        check(prt_query_ray(ctx, &r, &h, p, Ng));
        Props res;
        if (h.t < 0) return res;
        res.set("primId", h.primId);
        res.set("dist", h.t);
        res.set("p", Vec3f(p[0], p[1], p[2]));
        res.set("Ng", Vec3f(Ng[0], Ng[1], Ng[2]));
        return res;
    }

    Props queryPixel(int x, int y) { return Props(); }

    void initCamera(const Props& props)
    {
        ThinLensCamera c(props);   // the reference's own camera set-up
        prt_camera cam = {{c.origin.x, c.origin.y, c.origin.z},
                          {c.basis.U.x, c.basis.U.y, c.basis.U.z},
                          {c.basis.V.x, c.basis.V.y, c.basis.V.z},
                          {c.imageO.x, c.imageO.y, c.imageO.z},
                          {c.imageDx.x, c.imageDx.y, c.imageDx.z},
                          {c.imageDy.x, c.imageDy.y, c.imageDy.z},
                          c.lensRadius,
                          c.focalDistance};
        check(prt_set_camera(ctx, &cam));
    }

    void initFrame(const Vec2i& s, const Props&)
    {
        size = s;
        check(prt_init_frame(ctx, s.x, s.y));
    }

    void initToneMapper(const Props&) {}

    void clearFrame() { check(prt_clear(ctx)); }

    void blitFrame(Surface& dest)
    {
        std::vector<uint32_t> px((size_t)size.x * size.y);
        check(prt_read_ldr(ctx, px.data()));
        for (int y = 0; y < dest.height; ++y)
            std::memcpy((char*)dest.data + y * (ptrdiff_t)dest.pitch, px.data() + (size_t)y * size.x, size.x * 4);
    }
};

} // namespace prt
