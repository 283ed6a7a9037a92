// DeviceB200: the reference's Device interface (render/device.h:29-54) on the
// B200 path tracer's C ABI.  Errors become the exception types the reference
// throws for the same conditions (std::invalid_argument for bad arguments,
// render/device_cuda.cpp:63,92; std::runtime_error otherwise).
#include "device_b200.h"

#include <cmath>
#include <cstring>

namespace prt_host {

void DeviceB200::check(int status) const
{
    if (status == PRT_OK) return;
    std::string msg = ctx_ ? prt_last_error(ctx_) : "prt_create failed";
    if (status == PRT_EINVAL) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

DeviceB200::DeviceB200(int device)
{
    int st = prt_create(device, &ctx_);
    if (st != PRT_OK) throw std::runtime_error("cannot create a B200 context on device " + std::to_string(device));
}

DeviceB200::~DeviceB200()
{
    if (ctx_) prt_destroy(ctx_);
}

std::string DeviceB200::getInfo()
{
    char buf[256];
    check(prt_get_info(ctx_, buf, sizeof(buf)));
    return buf;
}

void DeviceB200::initScene(const std::string& path, const Props&)
{
    check(prt_load_mesh_file(ctx_, path.c_str(), bounds_.lo, bounds_.hi));
}

void DeviceB200::initRenderer(const Props& props, Props& stats)
{
    // the renderer names of the reference's diffuse renderers
    // (render/renderer_factory_single.cpp:56-59, render/device_cuda.cpp:51-93)
    std::string type = props.get("type", "diffuse");
    if (type != "diffuse" && type != "diffuseFast" && type != "diffuse2" && type != "diffuse2Fast")
        throw std::invalid_argument("invalid renderer type");
    accumulate_ = type == "diffuse" || type == "diffuse2";
    check(prt_set_integrator(ctx_, type.rfind("diffuse2", 0) == 0 ? PRT_INTEGRATOR_DIFFUSE2 : PRT_INTEGRATOR_DIFFUSE));
    maxDepth_ = props.getInt("maxDepth", 6);   // render/diffuse_integrator_single.h:35
    passesPerFrame_ = props.getInt("sppPerFrame", 1);
    if (passesPerFrame_ < 1) throw std::invalid_argument("sppPerFrame must be positive");
    // -no-sbvh: the reference's switch off its high-quality build (accel/embree/embree_intersector.cpp:24)
    check(prt_set_build_quality(ctx_, props.exists("no-sbvh") ? 0 : 1));
    prt_build_stats bs;
    check(prt_build_accel(ctx_, &bs));
    stats.set("buildMs", bs.buildMs);
    stats.set("buildMprim", bs.buildMprim);
}

void DeviceB200::render(Props& stats)
{
    prt_render_stats rs;
    check(prt_render(ctx_, passesPerFrame_, maxDepth_, accumulate_, &rs));
    stats.set("mray", rs.mray);
    stats.set("ray", rs.rays);
    stats.set("spp", passesPerFrame_);
}

Props DeviceB200::queryRay(const float org[3], const float dir[3], float far)
{
    prt_ray r;
    std::memcpy(r.org, org, 12);
    r.tnear = 0.0f;
    std::memcpy(r.dir, dir, 12);
    r.tfar = far;
    prt_hit h;
    float p[3], Ng[3];
    check(prt_query_ray(ctx_, &r, &h, p, Ng));
    Props res;
    if (h.t < 0) return res;
    res.set("primId", h.primId);
    res.set("dist", h.t);
    std::ostringstream sp, sn;
    sp << p[0] << "," << p[1] << "," << p[2];
    sn << Ng[0] << "," << Ng[1] << "," << Ng[2];
    res.set("p", sp.str());
    res.set("Ng", sn.str());
    return res;
}

// Renderer::queryPixel (render/renderer.h:57-81): a ray through the pixel
// centre, plus its depth along the view direction.
Props DeviceB200::queryPixel(int x, int y)
{
    prt_camera cam;
    prt_view v;
    std::memcpy(&v, &view_, sizeof(v));
    check(prt_camera_from_view(&v, width_, height_, &cam));
    float ix = ((float)x + 0.5f) / (float)width_, iy = ((float)y + 0.5f) / (float)height_;
    float d[3], c[3];
    for (int k = 0; k < 3; ++k)
    {
        d[k] = cam.imageO[k] + ix * cam.imageDx[k] + iy * cam.imageDy[k];
        c[k] = cam.imageO[k] + 0.5f * cam.imageDx[k] + 0.5f * cam.imageDy[k];
    }
    float ld = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    float lc = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    for (int k = 0; k < 3; ++k)
    {
        d[k] /= ld;
        c[k] /= lc;
    }
    Props res = queryRay(cam.origin, d, 3.4028235e38f);
    if (!res.exists("dist")) return res;
    res.set("depth", res.getDouble("dist", 0) * (d[0] * c[0] + d[1] * c[1] + d[2] * c[2]));
    return res;
}

void DeviceB200::initCamera(const View& view)
{
    view_ = view;
    prt_view v;
    std::memcpy(&v, &view, sizeof(v));
    prt_camera cam;
    check(prt_camera_from_view(&v, width_, height_, &cam));
    check(prt_set_camera(ctx_, &cam));
}

void DeviceB200::initFrame(int width, int height, const Props&)
{
    width_ = width;
    height_ = height;
    check(prt_init_frame(ctx_, width, height));
}

void DeviceB200::initToneMapper(const Props& props)
{
    // the reference supports only "none" (render/device_cpu_impl.cpp:105-117)
    std::string type = props.get("type", "none");
    if (type != "none") throw std::invalid_argument("invalid tone mapper type");
}

void DeviceB200::clearFrame() { check(prt_clear(ctx_)); }

void DeviceB200::blitFrame(std::vector<uint32_t>& bgra)
{
    bgra.resize((size_t)width_ * height_);
    check(prt_read_ldr(ctx_, bgra.data()));
}

} // namespace prt_host
