// build_displaced_mesh (displaced_tessellation.cpp) calls BaseMesh::triangle,
// which lives in base_mesh.cpp beside the OBJ loader; that file is not part of
// the oracle build, and the oracle never calls build_displaced_mesh. This
// stand-in only resolves the symbol, and aborts if it is ever reached.
#include "base_mesh.h"

#include <cstdio>
#include <cstdlib>

dmap::BaseTriangle dmap::BaseMesh::triangle(int) const
{
    std::fprintf(stderr, "BaseMesh::triangle is not part of the oracle build\n");
    std::abort();
}
