// h3g_eigen.cu — the main engine's model eigensystems on the device.
//
// For every model k of an installed model table: A = D^1/2 Q_k D^-1/2 with D = diag(pi) (pi
// floored at 1e-12), its symmetric part, diagonalised by the parallel cyclic Jacobi of
// h3g_jacobi.cuh; lambda clamped to <= 0; U_pi = D^-1/2 E and V_pi = E^T D^1/2.  This is the
// reference's MG94Matrix::update eigen step (rate_matrix.hpp:229-249, Eigen's
// SelfAdjointEigenSolver there).  The outputs are the engine's padded 64 x 64 layouts (lam, U,
// U^T, V); padding states stay decoupled (zero coupling, eigenvalue 0, zero rows and columns of
// U and V), so they add nothing to P(t) = U diag(e^{lambda t}) V.
#include "h3g_common.cuh"
#include "h3g_jacobi.cuh"
#include "h3g_kernels.h"

namespace h3g {

namespace {

constexpr int kET = 256;
constexpr int kEigMaxSweeps = 30;
constexpr size_t kModelEigSmem = size_t(2) * SP * jac::LD * sizeof(double);

// grid (nmod), block 256: one model per CTA.
__global__ void __launch_bounds__(kET) k_model_eig(const double* __restrict__ Q, const double* __restrict__ pi, int S,
                                                   double* lam, double* U, double* UT, double* V) {
    pdl_enter();
    extern __shared__ __align__(16) double sm[];
    constexpr int LD = jac::LD;
    double* A = sm;
    double* E = sm + SP * LD;
    __shared__ double sq[SP], isq[SP];
    __shared__ jac::Scratch js;
    const int tid = threadIdx.x, k = blockIdx.x;
    const double* Qk = Q + size_t(k) * SP2;
    if (tid < SP) {
        const double r = tid < S ? sqrt(fmax(pi[tid], 1e-12)) : 0.0;
        sq[tid] = r;
        isq[tid] = tid < S ? 1.0 / r : 0.0;
    }
    __syncthreads();
    for (int e = tid; e < SP2; e += kET) {
        const int i = e >> 6, j = e & 63;
        A[i * LD + j] = (i < S && j < S) ? sq[i] * Qk[e] * isq[j] : 0.0;
        E[i * LD + j] = i == j ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int e = tid; e < SP2; e += kET) {            // symmetric part (rate_matrix.hpp:236-237)
        const int i = e >> 6, j = e & 63;
        if (i < j) {
            const double m = 0.5 * (A[i * LD + j] + A[j * LD + i]);
            A[i * LD + j] = m;
            A[j * LD + i] = m;
        }
    }
    __syncthreads();
    jac::sweeps<kET>(A, E, js, kEigMaxSweeps);
    double* lk = lam + size_t(k) * SP;
    double* Uk = U + size_t(k) * SP2;
    double* UTk = UT + size_t(k) * SP2;
    double* Vk = V + size_t(k) * SP2;
    if (tid < SP) lk[tid] = tid < S ? fmin(A[tid * LD + tid], 0.0) : 0.0;
    for (int e = tid; e < SP2; e += kET) {
        const int a = e >> 6, b = e & 63;
        const bool real = a < S && b < S;
        const double u = real ? isq[a] * E[a * LD + b] : 0.0;     // U_pi[i = a][k = b]
        Uk[e] = u;
        UTk[size_t(b) * SP + a] = u;
        Vk[e] = real ? E[b * LD + a] * sq[b] : 0.0;                // V_pi[k = a][j = b]
    }
}

}  // namespace

void eigen_configure() {
    cudaFuncSetAttribute(k_model_eig, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kModelEigSmem));
}

int launch_model_eig(const double* Q, const double* pi, int S, int nmod, double* lam, double* U, double* UT, double* V,
                     cudaStream_t s) {
    launch_k(k_model_eig, nmod, kET, kModelEigSmem, s, Q, pi, S, lam, U, UT, V);
    return 1;
}

}  // namespace h3g
