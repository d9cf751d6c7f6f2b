// Test infrastructure (the oracle): renders a built-in sample scene of the
// reference CLI (Sample::Get, cli/samples.h:37-48) or an XML scene file read
// by the CLI's scene loader (LoadScene, cli/scene_loader.cpp:2147) through the
// reference's own route (cli/main.cpp:191-297: BVH, Filter/Camera/
// Sampler::Create, Integrator::Create, Render) on the host threads, and writes
// the image as a .pfm. The GPU CLI's output is compared against it.
//
//   cli_ref [-t threads] [-s spp] [-b max_bounces] [-r scale] -o out.pfm <scene.xml | sample_name>

#include "bulbit/bulbit.h"
#include "bulbit/parallel.h"
#include "samples.h"
#include "scene_loader.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace bulbit;

int main(int argc, const char* argv[])
{
    int32 threads = int32(std::thread::hardware_concurrency()), spp = 0, bounces = -1;
    float scale = 1;
    std::string out, input;
    for (int i = 1; i < argc; ++i)
    {
        std::string a = argv[i];
        if (i + 1 < argc && a == "-t") threads = std::atoi(argv[++i]);
        else if (i + 1 < argc && a == "-s") spp = std::atoi(argv[++i]);
        else if (i + 1 < argc && a == "-b") bounces = std::atoi(argv[++i]);
        else if (i + 1 < argc && a == "-r") scale = float(std::atof(argv[++i]));
        else if (i + 1 < argc && a == "-o") out = argv[++i];
        else input = a;
    }
    if (input.empty() || out.empty())
    {
        std::fprintf(stderr, "usage: cli_ref [-t n] [-s spp] [-b bounces] [-r scale] -o out.pfm <scene.xml | sample>\n");
        return 2;
    }
    ThreadPool::global_thread_pool = std::make_unique<ThreadPool>(std::max(1, threads));

    RendererInfo ri;
    if (!Sample::Get(&ri, input) && !LoadScene(&ri, std::filesystem::absolute(input)))
    {
        std::fprintf(stderr, "cannot load scene or sample %s\n", input.c_str());
        return 1;
    }
    if (spp > 0) ri.camera_info.sampler_info.spp = spp;
    if (bounces >= 0) ri.integrator_info.max_bounces = bounces;
    ri.camera_info.film_info.resolution *= scale;

    std::printf("primitives %zu lights %zu\n", ri.scene.GetPrimitives().size(), ri.scene.GetLights().size());
    BVH accel(ri.scene.GetPrimitives());
    Allocator alloc;
    Filter* filter = Filter::Create(alloc, ri.camera_info.film_info.filter_info);
    Camera* camera = Camera::Create(alloc, ri.camera_info, filter);
    Sampler* sampler = Sampler::Create(alloc, ri.camera_info.sampler_info);
    Integrator* integrator = Integrator::Create(alloc, ri.integrator_info, &accel, ri.scene.GetLights(), sampler);
    if (!filter || !camera || !sampler || !integrator)
    {
        std::fprintf(stderr, "set-up failed\n");
        return 1;
    }
    auto t0 = std::chrono::steady_clock::now();
    Rendering* rendering = integrator->Render(alloc, camera);
    rendering->Wait();
    std::printf("render_s %.3f threads %d\n",
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(), int(threads));
    Image3 img = rendering->GetFilm().GetRenderedImage();

    FILE* f = std::fopen(out.c_str(), "wb");
    if (!f) return 1;
    std::fprintf(f, "PF\n%d %d\n-1.0\n", img.width, img.height);
    std::vector<float> row(size_t(img.width) * 3);
    for (int32 y = img.height - 1; y >= 0; --y)
    {
        for (int32 x = 0; x < img.width; ++x)
        {
            row[3 * x + 0] = float(img(x, y).r);
            row[3 * x + 1] = float(img(x, y).g);
            row[3 * x + 2] = float(img(x, y).b);
        }
        std::fwrite(row.data(), sizeof(float), row.size(), f);
    }
    std::fclose(f);

    alloc.delete_object(rendering);
    alloc.delete_object(integrator);
    alloc.delete_object(sampler);
    alloc.delete_object(camera);
    alloc.delete_object(filter);
    return 0;
}
