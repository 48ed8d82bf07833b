// tree.cu -- octree build and walks (placeholder until the device tree lands).
#include "handle.cuh"

struct TreeBuffers {};
void tree_alloc(nv_handle *) {}
void tree_free(nv_handle *) {}
void launch_tree_build(nv_handle *) {}
void launch_tree_walk(nv_handle *) {}
void launch_closest_tree(nv_handle *) {}
int tree_dump(nv_handle *, int, void *, int, int *n) { *n = 0; return NV_ERR_UNSUPPORTED; }
