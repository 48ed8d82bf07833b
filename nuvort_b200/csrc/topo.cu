// topo.cu -- topology stages (placeholder until the device resolvers land).
#include "handle.cuh"

struct TopoBuffers {};
void topo_alloc(nv_handle *) {}
void topo_free(nv_handle *) {}
void launch_pinsert(nv_handle *) {}
void launch_pclose(nv_handle *, bool) {}
void launch_precon(nv_handle *) {}
void launch_premove(nv_handle *) {}
