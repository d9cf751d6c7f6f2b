// bbcli_gpu: the reference CLI's render route (cli/main.cpp:191-297: scene ->
// BVH -> filter, camera, sampler -> Integrator::Create -> Render -> image)
// with the GPU tree and the GPU integrator in place of BVH and
// PathIntegrator. As in the CLI (cli/main.cpp:199-203), each input is first
// looked up in the built-in sample registry (Sample::Get, cli/samples.h:37-48)
// and otherwise read as an XML scene file by the CLI's own scene loader
// (LoadScene, cli/scene_loader.cpp:2147), with OBJ and glTF models through its
// model loader (cli/model_loader.cpp); those two are compiled against this
// project's XML, OBJ and glTF readers (bulbit_b200/cpp/scene_io), which stand
// in for pugixml, tinyobjloader and tinygltf. A scene that fails to load is
// reported and skipped, as the CLI does. The options that apply to the path
// tracer are the CLI's (cli/main.cpp:8-33): -t -o -s -b -i -r. Images are
// written as Radiance .hdr (flat RGBE scanlines) or .pfm; other extensions
// are saved as .hdr.
//
// Build: compile with the reference's include directory and flags, link the
// reference library objects, the CLI's builders, loaders and sample scenes,
// the scene_io readers, bulbit_gpu.cpp and libbulbit_b200.so.

#include "bulbit_gpu.hpp"

#include "bulbit/parallel.h"
#include "samples.h"
#include "scene_loader.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <filesystem>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace bulbit;

namespace
{

double Seconds(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

bool EndsWith(const std::string& s, const char* suffix)
{
    size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

// Portable float map: rows bottom to top, little-endian floats.
bool WritePfm(const Image3& img, const std::string& path)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    std::fprintf(f, "PF\n%d %d\n-1.0\n", img.width, img.height);
    std::vector<float> row(size_t(img.width) * 3);
    for (int32 y = img.height - 1; y >= 0; --y)
    {
        for (int32 x = 0; x < img.width; ++x)
        {
            const RGBSpectrum& p = img(x, y);
            row[3 * x + 0] = float(p.r);
            row[3 * x + 1] = float(p.g);
            row[3 * x + 2] = float(p.b);
        }
        std::fwrite(row.data(), sizeof(float), row.size(), f);
    }
    return std::fclose(f) == 0;
}

// Radiance RGBE, uncompressed scanlines, top row first: each pixel is the
// three channels scaled by 2^-e to below 256 plus the biased exponent e.
bool WriteHdr(const Image3& img, const std::string& path)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    std::fprintf(f, "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n", img.height, img.width);
    std::vector<unsigned char> row(size_t(img.width) * 4);
    for (int32 y = 0; y < img.height; ++y)
    {
        for (int32 x = 0; x < img.width; ++x)
        {
            const RGBSpectrum& p = img(x, y);
            double c[3] = { std::max(0.0, double(p.r)), std::max(0.0, double(p.g)), std::max(0.0, double(p.b)) };
            double v = std::max(c[0], std::max(c[1], c[2]));
            unsigned char* o = &row[4 * size_t(x)];
            if (!(v >= 1e-32) || !std::isfinite(v))
            {
                o[0] = o[1] = o[2] = o[3] = 0;
                continue;
            }
            int e;
            double m = std::frexp(v, &e); // v = m 2^e, m in [0.5, 1)
            double scale = m * 256.0 / v;
            for (int k = 0; k < 3; ++k)
            {
                o[k] = static_cast<unsigned char>(std::min(255.0, c[k] * scale));
            }
            o[3] = static_cast<unsigned char>(e + 128);
        }
        std::fwrite(row.data(), 1, row.size(), f);
    }
    return std::fclose(f) == 0;
}

void PrintHelp()
{
    std::printf(
        "\nUsage:\n"
        "  bbcli_gpu [options] <scene.xml | sample_name> [<scene.xml | sample_name>...]\n\n"
        "Options:\n"
        "  -t <num_threads>          Host threads (scene set-up, film)  (default: hardware concurrency)\n"
        "  -o <output_file>          Output file name, .hdr or .pfm  (default: from scene or generated)\n"
        "  -s <samples_per_pixel>    Samples per pixel  (default: from scene)\n"
        "  -b <max_bounces>          Maximum path bounces  (default: from scene)\n"
        "  -i <integrator>           Integrator by index; 0 (path tracing) is the one on the GPU\n"
        "  -r <image_scale>          Scale the output image resolution  (default: 1)\n"
        "  --tree <reference|device|split|device-split>  GPU tree: the reference's SAH tree (default),\n"
        "                            a linear BVH built on the GPU, or the SAH tree over split\n"
        "                            references built on the host or on the GPU\n"
        "  --list-samples            List the built-in sample scenes\n"
        "  --help                    Show this help message\n\n");
}

} // namespace

int main(int argc, const char* argv[])
{
    if (argc <= 1 || std::string(argv[1]) == "--help")
    {
        PrintHelp();
        return 0;
    }

    int32 num_threads = int32(std::thread::hardware_concurrency());
    std::string output_file;
    int32 spp = 0, max_bounces = -1, integrator_index = -1;
    float scale = 1;
    bulbit_gpu::GpuTree tree = bulbit_gpu::GpuTree::Reference;
    std::vector<std::string> inputs;

    for (int i = 1; i < argc; ++i)
    {
        std::string a = argv[i];
        auto value = [&](const char* what) -> const char* {
            if (i + 1 >= argc)
            {
                std::fprintf(stderr, "Error: %s needs a value\n", what);
                std::exit(1);
            }
            return argv[++i];
        };
        if (a == "-t") num_threads = std::max(1, std::atoi(value("-t")));
        else if (a == "-o") output_file = value("-o");
        else if (a == "-s") spp = std::atoi(value("-s"));
        else if (a == "-b") max_bounces = std::atoi(value("-b"));
        else if (a == "-i") integrator_index = std::atoi(value("-i"));
        else if (a == "-r") scale = float(std::atof(value("-r")));
        else if (a == "--tree")
        {
            std::string t = value("--tree");
            if (t == "reference") tree = bulbit_gpu::GpuTree::Reference;
            else if (t == "device") tree = bulbit_gpu::GpuTree::DeviceLinear;
            else if (t == "split") tree = bulbit_gpu::GpuTree::SplitReferences;
            else if (t == "device-split") tree = bulbit_gpu::GpuTree::DeviceSplitReferences;
            else
            {
                std::fprintf(stderr, "Error: unknown tree '%s'\n", t.c_str());
                return 1;
            }
        }
        else if (a == "--list-samples")
        {
            for (const auto& kv : Sample::samples)
            {
                std::printf("  %s\n", kv.first.c_str());
            }
            return 0;
        }
        else if (!a.empty() && a[0] == '-')
        {
            std::fprintf(stderr, "Error: unknown option '%s'\n", a.c_str());
            return 1;
        }
        else inputs.push_back(a);
    }
    if (inputs.empty())
    {
        std::fprintf(stderr, "Error: No sample name provided.\n");
        return 1;
    }

    ThreadPool::global_thread_pool = std::make_unique<ThreadPool>(num_threads);
    int failures = 0;

    for (const std::string& input : inputs)
    {
        std::printf("\n--- %s ---\n", input.c_str());
        auto t0 = std::chrono::steady_clock::now();
        RendererInfo ri;
        bool loaded = Sample::Get(&ri, input);
        if (!loaded)
        {
            // LoadScene changes into the file's directory while it reads, so
            // it gets an absolute path (a bare file name has no parent).
            std::error_code ec;
            std::filesystem::path path = std::filesystem::absolute(input, ec);
            loaded = !ec && LoadScene(&ri, path);
        }
        if (!loaded)
        {
            std::fprintf(stderr, "Failed to load scene or sample: %s\n", input.c_str());
            ++failures;
            continue;
        }
        if (spp > 0) ri.camera_info.sampler_info.spp = spp;
        if (max_bounces >= 0) ri.integrator_info.max_bounces = max_bounces;
        if (integrator_index >= 0 && integrator_index < int32(IntegratorType::count))
        {
            ri.integrator_info.type = IntegratorType(integrator_index);
        }
        ri.camera_info.film_info.resolution *= scale;
        std::printf("Loading scene.. %.3fs\n", Seconds(t0));
        std::printf("Primitives: %zu, Lights: %zu\n", ri.scene.GetPrimitives().size(), ri.scene.GetLights().size());

        try
        {
            auto t1 = std::chrono::steady_clock::now();
            bulbit_gpu::GpuBVH accel(ri.scene.GetPrimitives(), tree);
            std::printf("Building acceleration structure (GPU).. %.3fs\n", Seconds(t1));

            Allocator alloc;
            Filter* filter = Filter::Create(alloc, ri.camera_info.film_info.filter_info);
            Camera* camera = filter ? Camera::Create(alloc, ri.camera_info, filter) : nullptr;
            Sampler* sampler = Sampler::Create(alloc, ri.camera_info.sampler_info);
            if (!filter || !camera || !sampler)
            {
                std::fprintf(stderr, "Failed to create pixel filter, camera or sampler\n");
                ++failures;
                continue;
            }

            t1 = std::chrono::steady_clock::now();
            Integrator* integrator =
                bulbit_gpu::CreateGpuIntegrator(alloc, ri.integrator_info, &accel, ri.scene.GetLights(), sampler);
            if (!integrator)
            {
                std::fprintf(stderr, "Failed to create integrator: type %d has no GPU implementation "
                                     "(path tracing, -i 0, has)\n",
                             int(ri.integrator_info.type));
                alloc.delete_object(sampler);
                alloc.delete_object(camera);
                alloc.delete_object(filter);
                ++failures;
                continue;
            }
            std::printf("Initializing integrator.. %.3fs\n", Seconds(t1));

            t1 = std::chrono::steady_clock::now();
            Rendering* rendering = integrator->Render(alloc, camera);
            rendering->WaitAndLogProgress();
            double render_s = Seconds(t1);
            const bbg_render_stats& st = dynamic_cast<bulbit_gpu::GpuPathIntegrator&>(*integrator).LastStats();
            std::printf("\nComplete %.3fs (device %.1f ms, %lld paths, %lld + %lld rays)\n", render_s, st.device_ms,
                        (long long)st.paths, (long long)st.closest_rays, (long long)st.shadow_rays);

            Image3 image = rendering->GetFilm().GetRenderedImage();
            std::string filename = output_file.empty() ? ri.camera_info.film_info.filename : output_file;
            if (filename.empty())
            {
                filename = "bbcli_gpu_" + input + "_" + std::to_string(image.width) + "x" +
                           std::to_string(image.height) + "_s" + std::to_string(ri.camera_info.sampler_info.spp) +
                           "_d" + std::to_string(ri.integrator_info.max_bounces) + ".hdr";
            }
            if (!EndsWith(filename, ".hdr") && !EndsWith(filename, ".pfm"))
            {
                std::printf("Warning: only .hdr and .pfm are written; saving as .hdr\n");
                size_t dot = filename.find_last_of('.');
                size_t slash = filename.find_last_of('/');
                if (dot != std::string::npos && (slash == std::string::npos || dot > slash)) filename.resize(dot);
                filename += ".hdr";
            }
            bool ok = EndsWith(filename, ".pfm") ? WritePfm(image, filename) : WriteHdr(image, filename);
            if (!ok)
            {
                std::fprintf(stderr, "Failed to write %s\n", filename.c_str());
                ++failures;
            }
            else
            {
                std::printf("Wrote %s\n", filename.c_str());
            }

            alloc.delete_object(rendering);
            alloc.delete_object(integrator);
            alloc.delete_object(sampler);
            alloc.delete_object(camera);
            alloc.delete_object(filter);
        }
        catch (const std::exception& e)
        {
            std::fprintf(stderr, "%s: %s\n", input.c_str(), e.what());
            ++failures;
        }
    }
    return failures == 0 ? 0 : 1;
}
