// Stand-in for the un-vendored assimp importer header, used only to compile the
// reference sources as a test oracle. It declares the names that
// src/bvh/bvh_IO.cpp:13-15,24-70 uses; ReadFile always reports failure, so the
// oracle only ever sees geometry injected directly or built from sphere/box lines.
#pragma once
#include <string>
#include <assimp/scene.h>

namespace Assimp
{
class Importer
{
public:
    const aiScene* ReadFile(const std::string&, unsigned int) { return nullptr; }
    const char*    GetErrorString() const { return "mesh import is not available in the oracle build"; }
};
} // namespace Assimp
