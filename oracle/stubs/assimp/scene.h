// Stand-in scene types for the oracle build (see Importer.hpp).
#pragma once

struct aiVector3D { float x, y, z; };
struct aiFace     { unsigned int mNumIndices; unsigned int* mIndices; };
struct aiMesh
{
    unsigned int mNumVertices;
    aiVector3D*  mVertices;
    aiVector3D*  mNormals;
    unsigned int mNumFaces;
    aiFace*      mFaces;
};
struct aiNode {};
struct aiScene
{
    unsigned int mFlags;
    aiNode*      mRootNode;
    unsigned int mNumMeshes;
    aiMesh**     mMeshes;
};
#define AI_SCENE_FLAGS_INCOMPLETE 0x1
