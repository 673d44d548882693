// h3g_mixed.cu — split-precision pruning path (not built yet: mixed_available() is false).
#include "h3g_mixed.h"

namespace h3g {

bool mixed_available() { return false; }
void mixed_configure() {}
h3g_status mixed_alloc(MixedWork&, std::vector<void*>&, int, int, int, int) { return H3G_ERR_CUDA; }
int mixed_prepare(const Topo&, const Model&, const Work&, const MixedWork&, cudaStream_t) { return 0; }
int launch_inside_mixed(const Topo&, const Model&, const Work&, const MixedWork&, const int*, int, cudaStream_t) { return 0; }
int launch_root_mixed(const Topo&, const Model&, const Work&, const MixedWork&, cudaStream_t) { return 0; }
int launch_outside_mixed(const Topo&, const Model&, const Work&, const MixedWork&, const int*, int, cudaStream_t) { return 0; }
int launch_accumA_mixed(const Topo&, const Model&, const Work&, const MixedWork&, cudaStream_t) { return 0; }

}  // namespace h3g
