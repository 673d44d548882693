// h3g_kernels.h — host-callable launchers of the device pipeline (one per stage).
// Each returns the number of kernels it enqueued on the stream.
#pragma once
#include "h3g_common.cuh"

namespace h3g {

void fp64_configure();
int launch_build_P(const Topo& t, const Model& md, const Work& w, cudaStream_t s);
int launch_prep_given_P(const Topo& t, const Work& w, cudaStream_t s);
int launch_inside_fp64(const Topo& t, const Model& md, const Work& w, const int* d_nodes, int count, cudaStream_t s);
int launch_root(const Topo& t, const Model& md, const Work& w, cudaStream_t s);
int launch_outside_fp64(const Topo& t, const Model& md, const Work& w, const int* d_nodes, int count, int want_v, cudaStream_t s);
// d_branches NULL: every branch (grid over all node ids)
int launch_accumA_fp64(const Topo& t, const Model& md, const Work& w, const int* d_branches, int count, cudaStream_t s);
int launch_frechet(const Topo& t, const Model& md, const Work& w, int want_global, cudaStream_t s);
int launch_global(const Topo& t, const Model& md, const Work& w, cudaStream_t s);
int launch_dir(const Topo& t, const Model& md, const Work& w, cudaStream_t s);
int launch_small(const Topo& t, const Model& md, const Work& w, int grads, cudaStream_t s);
void eigen_configure();
// Model eigensystems on the device (h3g_eigen.cu): Q [nmod][64*64] padded, pi [64] -> lam, U, U^T, V.
int launch_model_eig(const double* Q, const double* pi, int S, int nmod, double* lam, double* U, double* UT, double* V,
                     cudaStream_t s);
int launch_pack_result(const Topo& t, const Model& md, const Work& w, int grads, int global, double* dst, cudaStream_t s);

}  // namespace h3g
