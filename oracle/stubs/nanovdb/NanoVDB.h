// Test-infrastructure shim (oracle build only): the volume types that the
// reference's media header names. Volumes are not on the path-tracer path, so
// the shim only has to make the declarations compile; nothing constructs them.
#pragma once
namespace nanovdb
{
struct HostBuffer {};
template <typename B> struct GridHandle {};
struct FloatGrid {};
} // namespace nanovdb
