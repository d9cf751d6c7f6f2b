// Test-infrastructure shim (oracle build only); see ../NanoVDB.h. The CLI's
// scene loader reads NanoVDB volume files through nanovdb::io::readGrids
// (cli/scene_loader.cpp, "nanovdb" media); volumes are not on the path-tracer
// path, so reading one reports an error, which the loader catches.
#pragma once
#include "../NanoVDB.h"

#include <stdexcept>
#include <string>
#include <vector>

namespace nanovdb
{
namespace io
{
inline std::vector<GridHandle<HostBuffer>> readGrids(const std::string& filename)
{
    throw std::runtime_error("NanoVDB volume files are not read in this build: " + filename);
}
} // namespace io
} // namespace nanovdb
