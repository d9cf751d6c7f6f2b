// Test-infrastructure stubs for the oracle build of the reference renderer.
//
// The reference links stb (image files) and nanovdb (volumes) through
// FetchContent; neither is present here and neither is on the path-tracer
// path. These definitions replace them so the reference library links:
//   * image reads report "no file" (an empty image) and writes do nothing, so
//     the reflectance tables of src/bxdf/microfacet.cpp:239 are always
//     recomputed in memory (deterministic, never loaded from a lossy file);
//   * NanoVDBMedium members abort if ever reached (no config uses volumes;
//     the CLI's scene loader reaches the constructor only after reading a
//     NanoVDB file, which the nanovdb shim refuses).
#include "bulbit/image.h"
#include "bulbit/image3d.h"
#include "bulbit/media.h"

#include <cstdio>
#include <cstdlib>

namespace bulbit
{

Image1 ReadImage1(const std::filesystem::path&, int32, bool, std::function<Image1::Type(Image1::Type)>)
{
    return Image1{};
}
Image3 ReadImage3(const std::filesystem::path&, bool, std::function<Image3::Type(Image3::Type)>)
{
    return Image3{};
}
Image4 ReadImage4(const std::filesystem::path&, bool, std::function<Image4::Type(Image4::Type)>)
{
    return Image4{};
}
void WriteImage(const Image3&, const std::filesystem::path&, ToneMappingCallback*) {}
void WriteImage(const Image1&, const std::filesystem::path&, ToneMappingCallback*) {}

Image3D1 ReadImage3D(const std::filesystem::path&, int32, Point3i, bool, std::function<Image3D1::Type(Image3D1::Type)>)
{
    return Image3D1{};
}
Image3D3 ReadImage3D(const std::filesystem::path&, Point3i, bool, std::function<Image3D3::Type(Image3D3::Type)>)
{
    return Image3D3{};
}
void WriteImage3D(const Image3D1&, const std::filesystem::path&) {}
void WriteImage3D(const Image3D3&, const std::filesystem::path&) {}

[[noreturn]] static void NoVolumes()
{
    std::fprintf(stderr, "oracle build: NanoVDB volumes are not available\n");
    std::abort();
}

NanoVDBMedium::NanoVDBMedium(const Transform&, Spectrum, Spectrum, Float, Float g,
                             nanovdb::GridHandle<nanovdb::HostBuffer>, nanovdb::GridHandle<nanovdb::HostBuffer>, Float,
                             Float, Float)
    : Medium(TypeIndexOf<NanoVDBMedium>())
    , phase{ g }
{
    NoVolumes();
}
void NanoVDBMedium::Destroy() {}
bool NanoVDBMedium::IsEmissive() const { NoVolumes(); }
MediumSample NanoVDBMedium::SamplePoint(Point3) const { NoVolumes(); }
DDAMajorantIterator NanoVDBMedium::SampleRay(Ray, Float) const { NoVolumes(); }
RayMajorantIterator* NanoVDBMedium::SampleRay(Ray, Float, Allocator&) const { NoVolumes(); }

} // namespace bulbit
