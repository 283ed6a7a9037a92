// protoray — command line of the B200 path tracer with the reference's
// `protoray render` and `protoray build` interfaces (main/main.cpp:43-69,
// main/render/render.cpp, main/build/build.cpp):
//
//   protoray render scene.mesh [-r diffuse|diffuseFast] [-spp N] [-size W,H]
//       [-maxDepth D] [-dev b200] [-view K] [-benchmark PREFIX | -o PREFIX]
//       [-warmup N] [-sppPerFrame K] [-c config] [-checkpoint] [-runtime S] [-no-mtl] ...
//
// Options are `-name value` or `-name=value`; a bare argument is the scene
// (sys/option.cpp:37-93).  Unknown options are kept as properties, as in the
// reference.  The render loop renders frames until `spp` samples per pixel,
// drops the first spp/6 frames from the averaged stats in benchmark mode
// (main/render/render_window.cpp:43,143-144), and on exit writes the averaged
// stats as `stats_<name>=<value>` lines (<prefix>.txt), the per-frame stats
// (<prefix>.csv) and the image (<prefix>.ppm) (render_window.cpp:145-162,
// 227-255).  Only offscreen rendering exists (the reference's window mode is
// unsupported too, main/render/window.cpp:129-133).
//
//   protoray build input.obj|input.mesh [-o output] [-t mesh] [-threads N]
//
// parses the OBJ on host threads and builds the indexed mesh on the GPU from
// the OBJ's indexed form (prt_soup_load_obj + prt_build_mesh_soup), then
// writes the .mesh blob; the output
// defaults to the input name with its extension replaced by the type
// (build.cpp:84-85).  A .mesh input is read and written back.  Unlike the
// reference, which ignores ObjLoader::load's result and writes an empty mesh
// for a malformed OBJ (build.cpp:100-104), an OBJ error ends the command with
// status 1 and no output file.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "device_b200.h"

using namespace prt_host;

namespace {

struct Option
{
    std::string name, value;
};

std::vector<Option> parse_args(const std::vector<std::string>& args)
{
    std::vector<Option> opts;
    Option cur;
    bool pending = false;
    for (const std::string& a0 : args)
    {
        if (a0.size() > 1 && a0[0] == '-' && std::isalpha((unsigned char)a0[1]))
        {
            if (pending) opts.push_back(cur);
            std::string a = a0.substr(a0.find_first_not_of('-'));
            size_t eq = a.find('=');
            if (eq != std::string::npos)
            {
                opts.push_back({a.substr(0, eq), a.substr(eq + 1)});
                pending = false;
            }
            else
            {
                cur = {a, ""};
                pending = true;
            }
        }
        else
        {
            if (!pending) cur.name.clear();
            cur.value = a0;
            opts.push_back(cur);
            pending = false;
        }
    }
    if (pending) opts.push_back(cur);
    return opts;
}

std::vector<std::string> read_config(const std::string& path)
{
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open config file " + path);
    std::vector<std::string> words;
    std::string w;
    while (f >> w) words.push_back(w);
    return words;
}

std::string dir_of(const std::string& p)
{
    size_t s = p.find_last_of("/\\");
    return s == std::string::npos ? "" : p.substr(0, s + 1);
}

std::string base_of(const std::string& p)
{
    size_t d = p.find_last_of('.');
    size_t s = p.find_last_of("/\\");
    if (d == std::string::npos || (s != std::string::npos && d < s)) return p;
    return p.substr(0, d);
}

struct Settings
{
    std::string scene, device = "b200", renderer = "diffuse", prefix = "render";
    int width = 1024, height = 576, viewId = 0;
    bool benchmark = false;
    Props props;
};

bool apply(const std::vector<Option>& opts, Settings& s, const std::string& inputPath)
{
    for (const Option& o : opts)
    {
        if (o.name.empty()) s.scene = inputPath + o.value;
        else if (o.name == "c" || o.name == "config")
        {
            if (!apply(parse_args(read_config(o.value)), s, dir_of(o.value))) return false;
        }
        else if (o.name == "dev" || o.name == "device" || o.name == "e" || o.name == "engine") s.device = o.value;
        else if (o.name == "r" || o.name == "renderer") s.renderer = o.value;
        else if (o.name == "s" || o.name == "size")
        {
            Props p;
            p.set("v", o.value);
            if (!p.getPair("v", s.width, s.height)) return false;
        }
        else if (o.name == "dw" || o.name == "df")
        {
            std::cerr << "GUI not supported" << std::endl;
            return false;
        }
        else if (o.name == "do") {}
        else if (o.name == "benchmark" || o.name == "bench")
        {
            s.benchmark = true;
            s.prefix = o.value.empty() ? "benchmark" : o.value;
        }
        else if (o.name == "o" || o.name == "out" || o.name == "output") s.prefix = o.value;
        else if (o.name == "view")
        {
            s.viewId = std::stoi(o.value);
            if (s.viewId < 0 || s.viewId >= 10) return false;
        }
        else s.props.set(o.name, o.value);
    }
    return true;
}

// .view files: 10 x View (main/render/view.cpp:38-47); a missing file leaves
// the default view of main/render/render_window.cpp:400-426.
View load_view(const std::string& path, int id, const Box3f& b, bool& found)
{
    View v;
    float c[3], sz[3];
    for (int k = 0; k < 3; ++k)
    {
        c[k] = (b.lo[k] + b.hi[k]) * 0.5f;
        sz[k] = b.hi[k] - b.lo[k];
    }
    float mx = std::max(sz[0], std::max(sz[1], sz[2]));
    v.pos[0] = c[0];
    v.pos[1] = c[1];
    v.pos[2] = 1.7f * mx + c[2];
    v.angleX = v.angleY = 0.0f;
    v.fovY = 45.0f * (3.14159265358979f / 180.0f);
    v.radius = 0.0f;
    float d[3] = {c[0] - v.pos[0], c[1] - v.pos[1], c[2] - v.pos[2]};
    v.focus = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    found = false;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return v;
    View all[10];
    size_t n = std::fread(all, sizeof(View), 10, f);
    std::fclose(f);
    if (n == 10)
    {
        found = true;
        return all[id];
    }
    return v;
}

void save_ppm(const std::string& path, const std::vector<uint32_t>& px, int w, int h)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fprintf(f, "P6\n%d %d\n255\n", w, h);
    // the reference writes the bytes of each BGRA pixel in memory order
    // (image/image_io.cpp:55-64)
    for (uint32_t p : px)
    {
        std::fputc((int)(p & 0xff), f);
        std::fputc((int)((p >> 8) & 0xff), f);
        std::fputc((int)((p >> 16) & 0xff), f);
    }
    std::fclose(f);
}

int main_render(const std::vector<std::string>& args)
{
    Settings s;
    if (!apply(parse_args(args), s, "")) return 1;
    if (s.scene.empty())
    {
        std::cerr << "Scene not specified" << std::endl;
        return 1;
    }
    // render/render.cpp:182-187
    if (s.width <= 0 || s.width % 8 != 0 || s.height <= 0 || s.height % 8 != 0)
    {
        std::cerr << "Resolution must be multiple of 8" << std::endl;
        return 1;
    }
    if (s.device != "b200" && s.device != "cuda")
    {
        std::cerr << "Invalid device: " << s.device << std::endl;
        return 1;
    }
    std::ofstream log(s.prefix + ".log");
    auto say = [&](const std::string& m) {
        std::cout << m << std::endl;
        log << m << std::endl;
    };

    DeviceB200 dev(0);
    say("Device: " + dev.getInfo());
    dev.initScene(s.scene, s.props);
    dev.initFrame(s.width, s.height, s.props);
    Props rp = s.props;
    rp.set("type", s.renderer);
    Props buildStats;
    dev.initRenderer(rp, buildStats);
    say("Build: " + buildStats.get("buildMs") + " ms, " + buildStats.get("buildMprim") + " Mprim/s");

    bool found = false;
    View view = load_view(base_of(s.scene) + ".view", s.viewId, dev.getSceneBounds(), found);
    say(found ? "Loaded view " + std::to_string(s.viewId) : std::string("Default view"));
    dev.initCamera(view);
    dev.clearFrame();

    int maxSpp = s.props.getInt("spp", 0);
    int warmupSpp = s.props.getInt("warmup", maxSpp / 6);
    if (maxSpp <= 0)
    {
        std::cerr << "-spp N is required (offscreen rendering)" << std::endl;
        return 1;
    }
    std::vector<std::string> names;
    std::vector<std::vector<double>> values;
    auto record = [&](const Props& st) {
        for (const std::string& k : st.keys())
        {
            size_t i = 0;
            while (i < names.size() && names[i] != k) ++i;
            if (i == names.size())
            {
                names.push_back(k);
                values.emplace_back();
            }
            values[i].push_back(st.getDouble(k, 0.0));
        }
    };
    // -checkpoint: an image at every power-of-two spp; -runtime T: stop after T
    // seconds (main/render/render_window.cpp:39-41, 279-304)
    const bool checkpoint = s.props.exists("checkpoint");
    const double runtime = s.props.getDouble("runtime", 1e300);
    int spp = 0;
    auto t0 = std::chrono::steady_clock::now();
    while (spp < maxSpp)
    {
        Props st;
        auto f0 = std::chrono::steady_clock::now();
        dev.render(st);
        auto f1 = std::chrono::steady_clock::now();
        double frameMs = std::chrono::duration<double, std::milli>(f1 - f0).count();
        spp += st.getInt("spp", 1);
        st.set("renderMs", frameMs);
        st.set("fps", 1000.0 / frameMs);
        if (spp > warmupSpp || !s.benchmark) record(st);
        if (checkpoint && (spp & (spp - 1)) == 0)
        {
            char name[32];
            std::snprintf(name, sizeof(name), "%06dspp", spp);
            std::vector<uint32_t> px;
            dev.blitFrame(px);
            save_ppm(s.prefix + "_" + name + ".ppm", px, s.width, s.height);
        }
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= runtime) break;
    }
    double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    say("Rendered " + std::to_string(spp) + " spp in " + std::to_string(total) + " s");

    // averaged stats (StatsRecorder::getAverage, main/render/stats_recorder.cpp:48-64)
    Props avg = buildStats;
    for (size_t i = 0; i < names.size(); ++i)
    {
        double sum = 0;
        for (double v : values[i]) sum += v;
        avg.set(names[i], values[i].empty() ? 0.0 : sum / values[i].size());
    }
    for (const std::string& k : avg.keys()) say("Average " + k + "=" + avg.get(k));
    if (s.benchmark)
    {
        std::ofstream txt(s.prefix + ".txt");
        for (const std::string& k : avg.keys()) txt << "stats_" << k << "=" << avg.get(k) << "\n";
        std::ofstream csv(s.prefix + ".csv");
        for (size_t i = 0; i < names.size(); ++i) csv << (i ? "," : "") << names[i];
        csv << "\n";
        size_t rows = 0;
        for (auto& v : values) rows = std::max(rows, v.size());
        for (size_t t = 0; t < rows; ++t)
        {
            for (size_t i = 0; i < names.size(); ++i)
            {
                if (i) csv << ",";
                if (t < values[i].size())
                {
                    char b[64];
                    std::snprintf(b, sizeof(b), "%f", values[i][t]);
                    csv << b;
                }
            }
            csv << "\n";
        }
    }
    std::vector<uint32_t> px;
    dev.blitFrame(px);
    save_ppm(s.prefix + ".ppm", px, s.width, s.height);
    say("Saved " + s.prefix + ".ppm");
    return 0;
}

// .mesh re-save (build.cpp:92-96): the blob is parsed (geometry/triangle_mesh.cpp:305-320)
// and written back without anything that follows it.
int resave_mesh(const std::string& input, const std::string& output)
{
    std::ifstream f(input, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + input);
    std::vector<char> data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    auto need = [&](size_t at, size_t n) {
        if (at + n > data.size()) throw std::runtime_error("unexpected end of stream: " + input);
    };
    auto geti = [&](size_t at) {
        int v;
        need(at, 4);
        std::memcpy(&v, &data[at], 4);
        return v;
    };
    if (geti(0) != 0x04df8666) throw std::runtime_error("file has wrong blob ID: " + input);
    need(0, 38);
    const int tri = geti(28), vert = geti(32);
    if (tri < 0 || vert < 0) throw std::runtime_error("negative element count: " + input);
    const int stride = 3 + (data[36] ? 3 : 0) + (data[37] ? 2 : 0);
    size_t at = 38 + 16 * (size_t)tri + 4 * (size_t)stride * vert;
    const int names = geti(at);
    at += 4;
    for (int i = 0; i < names; ++i)
    {
        const int len = geti(at);
        if (len < 0) throw std::runtime_error("negative string length: " + input);
        need(at + 4, (size_t)len);
        at += 4 + (size_t)len;
    }
    std::ofstream o(output, std::ios::binary);
    if (!o.write(data.data(), (std::streamsize)at)) throw std::runtime_error("cannot write " + output);
    return 0;
}

int main_build(const std::vector<std::string>& args)
{
    // build.log beside the working directory, as the reference (build.cpp:41)
    std::ofstream log("build.log");
    auto say = [&](const std::string& m) {
        std::cout << m << std::endl;
        log << m << std::endl;
    };
    std::string type = "mesh", input, output;
    int threads = 0;
    for (const Option& opt : parse_args(args))
    {
        if (opt.name.empty())
        {
            if (!input.empty()) throw std::invalid_argument("Multiple inputs");
            input = opt.value;
        }
        else if (opt.name == "o")
        {
            if (!output.empty()) throw std::invalid_argument("Multiple outputs");
            output = opt.value;
        }
        else if (opt.name == "t")
            type = opt.value;
        else if (opt.name == "threads")
            threads = std::stoi(opt.value);
        else
            say("Option: " + opt.name + " = " + opt.value);
    }
    if (output.empty()) output = input.substr(0, input.find_last_of('.')) + "." + type;
    const std::string ext = input.substr(input.find_last_of('.') + 1);
    if (ext != "mesh" && ext != "obj")
    {
        std::cerr << "Error: Unsupported input format" << std::endl;
        return 1;
    }
    if (type != "mesh")
    {
        std::cerr << "Error: Invalid type" << std::endl;
        return 1;
    }
    if (ext == "mesh") return resave_mesh(input, output);

    const auto t0 = std::chrono::steady_clock::now();
    prt_soup* soup = nullptr;
    char err[512];
    if (prt_soup_load_obj(input.c_str(), threads, &soup, err, sizeof(err)) != PRT_OK)
        throw std::runtime_error(std::string(err) + " (" + input + ")");
    struct SoupFree
    {
        prt_soup* s;
        ~SoupFree() { prt_soup_free(s); }
    } soupFree{soup};
    const auto t1 = std::chrono::steady_clock::now();
    int degenerate = 0;
    prt_soup_info(soup, nullptr, nullptr, &degenerate);
    if (degenerate > 0) say("Removed " + std::to_string(degenerate) + " degenerate triangles");

    DeviceB200 dev(0);
    prt_mesh_info info;
    int st = prt_build_mesh_soup(dev.handle(), soup, &info);
    if (st != PRT_OK) throw std::runtime_error(prt_last_error(dev.handle()));
    st = prt_save_built_mesh(dev.handle(), output.c_str());
    if (st != PRT_OK) throw std::runtime_error(prt_last_error(dev.handle()));
    const double parseMs = std::chrono::duration<double, std::milli>(t1 - t0).count();
    say("Built " + output + ": " + std::to_string(info.triCount) + " triangles, " + std::to_string(info.vertCount) +
        " unique vertices (OBJ " + std::to_string(parseMs) + " ms, build " + std::to_string(info.buildMs) + " ms)");
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    std::vector<std::string> args(argv + 1, argv + argc);
    if (args.empty() || (args[0] != "render" && args[0] != "build"))
    {
        std::cout << "Usage: protoray render scene.mesh [options]" << std::endl;
        std::cout << "       protoray build input.obj [-o output.mesh]" << std::endl;
        return args.empty() ? 0 : 1;
    }
    const std::string cmd = args[0];
    args.erase(args.begin());
    if (args.empty())
    {
        std::cout << "Usage: protoray " << cmd << " [options]" << std::endl;
        return 0;
    }
    try
    {
        return cmd == "build" ? main_build(args) : main_render(args);
    }
    catch (const std::exception& e)
    {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }
}
