// Stand-in post-process flags for the oracle build (see Importer.hpp).
#pragma once
enum aiPostProcessSteps
{
    aiProcess_Triangulate       = 0x8,
    aiProcess_GenSmoothNormals  = 0x40
};
