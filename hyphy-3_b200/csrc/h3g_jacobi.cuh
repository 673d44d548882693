// h3g_jacobi.cuh — parallel cyclic Jacobi for a symmetric 64x64 FP64 matrix held in shared
// memory by one CTA, shared by the per-site fits' eigensystems (h3g_fel.cu) and the main
// engine's model eigensystems (h3g_eigen.cu).
//
// Golub & Van Loan, "Matrix Computations" (Alg. 8.5.1 / 8.5.3): one sweep = 63 rounds of 32
// disjoint rotations (p_k, q_k) covering all 64 indices (circle schedule).  Warp 0 computes the
// round's rotations (t from one square root and one divide, c = rsqrt(1 + t^2)); then every 2x2
// block (I, J) of A is replaced by R_I^T A_IJ R_J in one pass, the diagonal blocks by their exact
// annihilated values a_pp - t a_pq, a_qq + t a_pq and 0, and the columns of E by E R.  Two
// barriers per round.  The sweeps stop when the off-diagonal mass is below 1e-30 of the total.
#pragma once

#include "h3g_common.cuh"

namespace h3g {
namespace jac {

constexpr int LD = SP + 1;                // padded row stride: column walks hit 32 distinct banks

struct Scratch {                          // shared-memory scratch of one round
    double c[32], s[32], t[32], apq[32], app[32], aqq[32];
    int p[32], q[32];
    double red[32];
};

template <int NT>
__device__ __forceinline__ double block_sum_or_max(double v, double* red, bool is_max) {
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = is_max ? fmax(v, w) : v + w;
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) red[warp] = v;
    __syncthreads();
    double r = red[0];
    for (int k = 1; k < NT / 32; ++k) r = is_max ? fmax(r, red[k]) : r + red[k];
    __syncthreads();
    return r;
}

// A (symmetric, [64][LD]) is diagonalised in place; E ([64][LD]) is multiplied by the rotations
// (start it at the identity, or at a warm-start basis with A already rotated into it).
// NT threads (a multiple of 32, at least 64).
template <int NT>
__device__ void sweeps(double* A, double* E, Scratch& js, int max_sweeps) {
    const int tid = threadIdx.x;
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int e = tid; e < SP2; e += NT) {
            const int i = e >> 6, j = e & 63;
            const double x = A[i * LD + j] * A[i * LD + j];
            tot += x;
            if (i != j) off += x;
        }
        off = block_sum_or_max<NT>(off, js.red, false);
        tot = block_sum_or_max<NT>(tot, js.red, false);
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int round = 0; round < SP - 1; ++round) {
            if (tid < 32) {
                int p, q;
                if (tid == 0) { p = SP - 1; q = round; }
                else { p = (round + tid) % (SP - 1); q = (round - tid + (SP - 1)) % (SP - 1); }
                if (p > q) { const int tmp = p; p = q; q = tmp; }
                const double apq = A[p * LD + q], app = A[p * LD + p], aqq = A[q * LD + q];
                double c = 1.0, s = 0.0, t = 0.0;
                if (fabs(apq) >= 1e-300) {
                    // t = tan(theta) of the smaller rotation, tau = (a_qq - a_pp) / (2 a_pq):
                    // t = sign(tau) / (|tau| + sqrt(1 + tau^2)) = 2 a_pq sign(d) / (|d| + sqrt(d^2 + 4 a_pq^2)), d = a_qq - a_pp
                    const double d = aqq - app;
                    const double tt = 2.0 * apq / (fabs(d) + sqrt(d * d + 4.0 * apq * apq));
                    t = d >= 0.0 ? tt : -tt;
                    c = rsqrt(1.0 + t * t);
                    s = t * c;
                }
                js.p[tid] = p; js.q[tid] = q; js.c[tid] = c; js.s[tid] = s;
                js.t[tid] = t; js.apq[tid] = apq; js.app[tid] = app; js.aqq[tid] = aqq;
            }
            __syncthreads();
            for (int e = tid; e < 32 * 32; e += NT) {      // block (I, J) of A
                const int I = e >> 5, J = e & 31;
                const int pI = js.p[I], qI = js.q[I], pJ = js.p[J], qJ = js.q[J];
                if (I == J) {
                    A[pI * LD + pI] = js.app[I] - js.t[I] * js.apq[I];
                    A[qI * LD + qI] = js.aqq[I] + js.t[I] * js.apq[I];
                    A[pI * LD + qI] = 0.0;
                    A[qI * LD + pI] = 0.0;
                    continue;
                }
                const double cI = js.c[I], sI = js.s[I], cJ = js.c[J], sJ = js.s[J];
                const double a = A[pI * LD + pJ], b = A[pI * LD + qJ], cc = A[qI * LD + pJ], dd = A[qI * LD + qJ];
                const double m0 = cJ * a - sJ * b, m1 = sJ * a + cJ * b;      // [a b; c d] R_J
                const double m2 = cJ * cc - sJ * dd, m3 = sJ * cc + cJ * dd;
                A[pI * LD + pJ] = cI * m0 - sI * m2;                        // R_I^T (...)
                A[pI * LD + qJ] = cI * m1 - sI * m3;
                A[qI * LD + pJ] = sI * m0 + cI * m2;
                A[qI * LD + qJ] = sI * m1 + cI * m3;
            }
            for (int e = tid; e < 32 * SP; e += NT) {      // columns p, q of E
                const int k = e >> 6, i = e & 63;
                const int p = js.p[k], q = js.q[k];
                const double c = js.c[k], s = js.s[k];
                const double ekp = E[i * LD + p], ekq = E[i * LD + q];
                E[i * LD + p] = c * ekp - s * ekq;
                E[i * LD + q] = s * ekp + c * ekq;
            }
            __syncthreads();
        }
    }
}

}  // namespace jac
}  // namespace h3g
