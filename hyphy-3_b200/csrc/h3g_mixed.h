// h3g_mixed.h — split-precision (tensor-core) pruning path: FP32 partials with
// per-pattern power-of-two exponents, contractions on tcgen05, FP64 for the
// model, the root log-sum and every reduction.
#pragma once
#include <vector>
#include "../../include/h3g.h"
#include "h3g_common.cuh"

namespace h3g {

struct MixedWork {
    float* D = nullptr;      // [NI][M][Pp][64]  pattern-major FP32 partials
    float* Ms = nullptr;     // [NI][M][Pp][64]
    float* U = nullptr;      // [NI][M][Pp][64]
    float* Vf = nullptr;     // [n][M][Pp][64]
    int* Ecum = nullptr;     // [NI][M][Pp]
    int* Eown = nullptr;     // [NI][M][Pp]
    int* Eu = nullptr;       // [NI][M][Pp] exponent of the stored outside partial
    int* Ev = nullptr;       // [n][M][Pp]  exponent of the stored Vf
    float* Phi = nullptr;    // [M][n][64*64] tf32-rounded high part of P (row-major)
    float* Plo = nullptr;    // [M][n][64*64] remainder
    float* PThi = nullptr;   // transposes
    float* PTlo = nullptr;
};

bool mixed_available();
void mixed_configure();
h3g_status mixed_alloc(MixedWork& mw, std::vector<void*>& owned, int n, int NI, int M, int Pp);
int mixed_prepare(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, cudaStream_t s);
int launch_inside_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, const int* d_nodes, int count, cudaStream_t s);
int launch_root_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, cudaStream_t s);
int launch_outside_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, const int* d_nodes, int count, cudaStream_t s);
int launch_accumA_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, cudaStream_t s);

}  // namespace h3g
