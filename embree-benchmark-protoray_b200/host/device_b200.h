// C++ host side of the B200 path tracer: a Device interface with the
// reference's methods (render/device.h:29-54) and its B200 implementation
// over the C ABI (include/prt_b200.h).
//
// Props is a small string-keyed property bag standing in for the reference's
// Props (sys/props.h): values are kept as strings and converted on get, and
// "W,H"-style pairs parse like Value::get<Vec2i> (sys/value.h:159-176).
#pragma once

#include <cstdint>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/prt_b200.h"

namespace prt_host {

class Props
{
    std::map<std::string, std::string> items_;
    std::vector<std::string> order_;

public:
    template <class T>
    void set(const std::string& name, const T& value)
    {
        std::ostringstream s;
        s.precision(9);
        s << value;
        if (!items_.count(name)) order_.push_back(name);
        items_[name] = s.str();
    }
    void set(const std::string& name, const std::string& value)
    {
        if (!items_.count(name)) order_.push_back(name);
        items_[name] = value;
    }
    void set(const std::string& name, const char* value) { set(name, std::string(value)); }
    bool exists(const std::string& name) const { return items_.count(name) != 0; }
    std::string get(const std::string& name, const std::string& def = "") const
    {
        auto it = items_.find(name);
        return it == items_.end() ? def : it->second;
    }
    int getInt(const std::string& name, int def) const
    {
        auto it = items_.find(name);
        return it == items_.end() || it->second.empty() ? def : std::stoi(it->second);
    }
    double getDouble(const std::string& name, double def) const
    {
        auto it = items_.find(name);
        return it == items_.end() || it->second.empty() ? def : std::stod(it->second);
    }
    // "1920,1080" or "1920 1080"
    bool getPair(const std::string& name, int& a, int& b) const
    {
        auto it = items_.find(name);
        if (it == items_.end()) return false;
        std::string v = it->second;
        for (char& c : v)
            if (c == ',' || c == 'x') c = ' ';
        std::istringstream s(v);
        return bool(s >> a >> b);
    }
    const std::vector<std::string>& keys() const { return order_; }
};

struct Box3f
{
    float lo[3] = {0, 0, 0};
    float hi[3] = {0, 0, 0};
};

// Camera view (main/render/view.h:25-33)
struct View
{
    float pos[3];
    float angleX, angleY, fovY, radius, focus;
};

// Device interface of the reference (render/device.h:29-54).
class Device
{
public:
    virtual ~Device() {}
    virtual std::string getInfo() = 0;
    virtual void initScene(const std::string& path, const Props& props) = 0;
    virtual Box3f getSceneBounds() = 0;
    virtual void initRenderer(const Props& props, Props& stats) = 0;
    virtual void render(Props& stats) = 0;
    virtual Props queryPixel(int x, int y) = 0;
    virtual Props queryRay(const float org[3], const float dir[3], float far) = 0;
    virtual void initCamera(const View& view) = 0;
    virtual void initFrame(int width, int height, const Props& props) = 0;
    virtual void initToneMapper(const Props& props) = 0;
    virtual void clearFrame() = 0;
    // BGRA8 pixels, width*height, raster order (DeviceCuda::blitFrame, render/device_cuda.cpp:214-230)
    virtual void blitFrame(std::vector<uint32_t>& bgra) = 0;
};

class DeviceB200 : public Device
{
    prt_ctx* ctx_ = nullptr;
    int width_ = 0, height_ = 0;
    int maxDepth_ = 6;
    int accumulate_ = 1;
    int passesPerFrame_ = 1;
    Box3f bounds_;
    View view_{};

    void check(int status) const;

public:
    explicit DeviceB200(int device = 0);
    ~DeviceB200() override;
    DeviceB200(const DeviceB200&) = delete;
    DeviceB200& operator=(const DeviceB200&) = delete;

    std::string getInfo() override;
    void initScene(const std::string& path, const Props& props) override;
    Box3f getSceneBounds() override { return bounds_; }
    // props: type (diffuse | diffuseFast | diffuse2 | diffuse2Fast), maxDepth (default 6), sppPerFrame (default 1)
    void initRenderer(const Props& props, Props& stats) override;
    // one frame: sppPerFrame passes; stats: mray, ray, spp
    void render(Props& stats) override;
    Props queryPixel(int x, int y) override;
    Props queryRay(const float org[3], const float dir[3], float far) override;
    void initCamera(const View& view) override;
    void initFrame(int width, int height, const Props& props) override;
    void initToneMapper(const Props& props) override;
    void clearFrame() override;
    void blitFrame(std::vector<uint32_t>& bgra) override;

    prt_ctx* handle() { return ctx_; }
};

} // namespace prt_host
