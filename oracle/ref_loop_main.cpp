// The reference's own render loop driving the B200 device — TEST
// INFRASTRUCTURE ONLY (an integration check of the drop-in boundary).
//
// oracle/Makefile links this file with the reference's unmodified
// RenderWindow / Window / StatsRecorder / ViewSet (main/render/*.cpp) and the
// reference's sys/ and image/ code, plus DeviceB200
// (embree-benchmark-protoray_b200/host/reference_device_b200.h), the class a
// maintainer adds beside render/device_cuda.{h,cpp}.  The steps below are the
// ones mainRender takes once it has picked a device
// (main/render/render.cpp:200-243): initScene, initFrame, initRenderer, then
// RenderWindow::run in offscreen mode.  The reference's option parser
// (sys/option.cpp) is not linked (its TextReader includes the original
// sys/ref.h, which GCC rejects), so the options come positionally:
//
//   protoray_refloop <scene.mesh> <width> <height> <spp> <maxDepth> <renderer> <resultPrefix>
//
// With a result prefix the loop runs in benchmark mode, as `-benchmark
// <prefix>` does: frames after the first spp/6 are averaged, and it writes
// <prefix>.txt (stats_<name>=<value>), <prefix>.csv and <prefix>.ppm.
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>

#include "sys/logging.h"
#include "sys/filesystem.h"
#include "main/render/render_window.h"
#include "reference_device_b200.h"

using namespace prt;

int main(int argc, char* argv[])
{
    if (argc != 8)
    {
        std::fprintf(stderr, "usage: %s scene.mesh width height spp maxDepth renderer resultPrefix\n", argv[0]);
        return 2;
    }
    try
    {
        initLogging();
        const std::string sceneFilename = argv[1];
        const Vec2i imageSize(std::atoi(argv[2]), std::atoi(argv[3]));
        const std::string rendererId = argv[6];
        const std::string resultPrefix = argv[7];
        Props props;
        props.set("spp", std::atoi(argv[4]));
        props.set("maxDepth", std::atoi(argv[5]));
        props.set("benchmark", resultPrefix);

        ref<Device> device = makeRef<DeviceB200>();
        Log() << "Device: " << device->getInfo();
        device->initScene(sceneFilename, props);
        device->initFrame(imageSize, props);

        Props rendererProps = props;
        rendererProps.set("type", rendererId);
        rendererProps.set("imageSize", imageSize);
        Props buildStats;
        device->initRenderer(rendererProps, buildStats);

        const std::string sceneBase = getFilenameBase(sceneFilename);
        props.set("viewFile", sceneBase + ".view");
        props.set("view", 0);
        props.set("poiFile", sceneBase + ".poi");
        props.set("output", resultPrefix);

        RenderWindow window(imageSize.x, imageSize.y, displayModeOffscreen, device, props, buildStats);
        window.setTitle("ProtoRay");
        window.run();
    }
    catch (const std::exception& e)
    {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
