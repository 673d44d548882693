// h3g_fp64.cu — FP64 kernels of the likelihood + adjoint-gradient pipeline.
//
// Per evaluation (one CUDA stream, level-synchronous over the tree):
//   k_build_P      P_{m,b} = sum_k c_k clamp(U_k diag(e^{lam_k tau}) V_k), dP = d P / d t
//                  (rate_matrix.hpp:251-257, likelihood.hpp:1118-1127, busted.hpp:1191-1216),
//                  FP64 tensor-core products
//   k_inside       one launch per height level: D_u = prod_c P_c D_c with power-of-two
//                  rescaling, then the message P_u D_u for the parent (likelihood.hpp:500-597)
//   k_root         L = pi . D_root, log-sum-exp over rate classes, per-pattern scale
//                  factors f = w * post / L (likelihood.hpp:599-610, busted.hpp:1346-1375)
//   k_outside      one launch per depth level: V_c = 2^{e_u} U_u o prod_{s != c} P_s D_s,
//                  U_c = P_c^T V_c (likelihood.hpp:612-761)
//   k_accumA       A_{m,b} = sum_p f V D^T  (likelihood.hpp:1435 generalised)
//   k_frechet      dlnL/dt_b = <A, dP>; spectral Frechet pieces U^T A V^T o E
//                  (likelihood.hpp:1428-1471)
//   k_hsum, k_dir, k_small   fixed-order reductions -> lnL, gradients
// All reductions run in a fixed order, so repeated evaluations are bit-identical.
#include <cstdlib>
#include "h3g_common.cuh"
#include "h3g_kernels.h"
#include "h3g_mixed.h"
#include "h3g_tc.cuh"

namespace h3g {

__device__ __forceinline__ int renorm64(double (&v)[SP]) {
    double mx = 0.0;
#pragma unroll
    for (int i = 0; i < SP; ++i) mx = fmax(mx, v[i]);
    if (mx > 0.0 && mx < 0x1p-256) {
        const int sh = -ilogb(mx) - 1;    // brings the max into [0.5, 1)
#pragma unroll
        for (int i = 0; i < SP; ++i) v[i] = ldexp(v[i], sh);
        return sh;
    }
    return 0;
}

// v *= P_c * leaf_vector(c, p): a column of P_c, a masked column sum or the row sums.
__device__ __forceinline__ void mul_leaf_msg(double (&v)[SP], const Topo& t, const Work& w, int m, int c, int p) {
    const int tx = t.taxon[c];
    const double* PTc = w.PT + mat_off(m, c, t.n);
    const int st = tx < 0 ? -1 : int(t.states[size_t(tx) * t.Pp + p]);
    if (st >= 0) {
        const double2* r = reinterpret_cast<const double2*>(PTc + st * SP);
#pragma unroll
        for (int i = 0; i < SP / 2; ++i) { double2 x = __ldg(r + i); v[2 * i] *= x.x; v[2 * i + 1] *= x.y; }
        return;
    }
    const uint64_t mk = tx < 0 ? t.all_mask : t.masks[size_t(tx) * t.Pp + p];
    if (mk == 0 || (mk & t.all_mask) == t.all_mask) {
        const double2* r = reinterpret_cast<const double2*>(w.rs + (size_t(m) * t.n + c) * SP);
#pragma unroll
        for (int i = 0; i < SP / 2; ++i) { double2 x = __ldg(r + i); v[2 * i] *= x.x; v[2 * i + 1] *= x.y; }
        return;
    }
#pragma unroll
    for (int i = 0; i < SP; ++i) {
        double s = 0.0;
        for (uint64_t b = mk; b; b &= b - 1) s += __ldg(PTc + (__ffsll((long long)b) - 1) * SP + i);
        v[i] *= s;
    }
}

__device__ __forceinline__ void stage_matrix(double* __restrict__ s, const double* __restrict__ g, int tid, int nthr) {
    const double2* g2 = reinterpret_cast<const double2*>(g);
    double2* s2 = reinterpret_cast<double2*>(s);
    for (int k = tid; k < SP2 / 2; k += nthr) s2[k] = __ldg(g2 + k);
}

// --------------------------------------------------- FP64 tensor-core products
// 64x64x64 products on the FP64 tensor cores (mma.sync m8n8k4 .f64; tcgen05 has no FP64
// kind) by the 8 warps of a 256-thread CTA: warp w owns rows 16(w/2) .. +16 and columns
// 32(w%2) .. +32 as 2 x 4 tiles of 8x8, operands and results stay in registers between
// the k steps.  Both operands are row-major in shared memory with a padded stride of 68
// doubles: the fragment loads of a half-warp, (row + lane/4) * 68 + k + lane%4 and
// (k + lane%4) * 68 + col + lane/4, fall in 16 different banks.
constexpr int LDM = SP + 4;

struct Frag64 {
    double v[2][4][2];        // C[r0 + 8i + lane/4][c0 + 8j + 2(lane%4) + e]
};

__device__ __forceinline__ void frag_zero(Frag64& f) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) f.v[i][j][0] = f.v[i][j][1] = 0.0;
}
// position of f.v[i][j][e] in the 64x64 result
__device__ __forceinline__ int frag_row(int i) { return 16 * (int(threadIdx.x) >> 6) + 8 * i + ((threadIdx.x & 31) >> 2); }
__device__ __forceinline__ int frag_col(int j, int e) {
    return 32 * ((int(threadIdx.x) >> 5) & 1) + 8 * j + 2 * (threadIdx.x & 3) + e;
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// c = X Y, X and Y [64][LDM] in shared memory
__device__ __forceinline__ void mm64(const double* __restrict__ X, const double* __restrict__ Y, Frag64& c) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int r0 = 16 * (wp >> 1), c0 = 32 * (wp & 1), g = lane >> 2, q = lane & 3;
    frag_zero(c);
#pragma unroll 4
    for (int k = 0; k < SP; k += 4) {
        double a[2], b[4];
#pragma unroll
        for (int i = 0; i < 2; ++i) a[i] = X[(r0 + 8 * i + g) * LDM + k + q];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Y[(k + q) * LDM + c0 + 8 * j + g];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma(c.v[i][j][0], c.v[i][j][1], a[i], b[j]);
    }
}

// ------------------------------------------------------------------ build P
// grid (n, M): one CTA per branch and rate class computes the whole 64x64
// P_{m,b} = sum_k c_k clamp(U_k diag(e^{lam_k tau}) V_k) and
// dP_{m,b} = sum_k c_k r_m conv_k Q_k clamp(P_k), model by model, as two FP64
// tensor-core products per model (mm64).
// dynamic smem: 2 x 64 x LDM doubles (U e then Q; V then clamp(P_k)).
// kMixed: the split-precision path's operands instead of the FP64 P and P^T, from P staged in
// shared memory: the BF16 hi/mid/lo tiles of P and P^T in the tcgen05 K-major layout (16-byte
// stores of 8 consecutive K), FP32 P^T and the row sums (FP64 and FP32); thread 0 of CTA (0, 0)
// starts the evaluation's epoch of the persistent passes.
template <bool kMixed>
__global__ void __launch_bounds__(256) k_build_P(Topo t, Model md, Work w, MixedWork mw) {
    pdl_enter();
    extern __shared__ __align__(16) double sm[];
    double* sX = sm;                 // U_k diag(e), then Q_k
    double* sY = sm + SP * LDM;      // V_k, then clamp(P_k)
    __shared__ double se[SP];
    const int b = blockIdx.x, m = blockIdx.y, tid = threadIdx.x;
    if (kMixed && b == 0 && m == 0 && tid == 0) {        // a new evaluation: new epoch, fresh item counters
        mw.sync[0] += 1;
        mw.sync[1] = 0;
        mw.sync[2] = 0;
    }
    if (b == t.root) return;
    const BranchModels bm = branch_models(md, b);
    Frag64 accP, accD;
    frag_zero(accP);
    frag_zero(accD);
    for (int k = bm.k0; k < bm.k1; ++k) {
        const double cw = class_weight(md, bm, k);
        const double cv = time_conv(md, k);
        const double rate = md.rates[m];
        const double tau = rate * w.bl[b] * cv;
        __syncthreads();                          // the previous model's products are done
        if (tid < SP) se[tid] = exp(md.lam[size_t(k) * SP + tid] * tau);
        __syncthreads();
        {
            const double* U = md.U + size_t(k) * SP2;
            const double* V = md.V + size_t(k) * SP2;
            for (int e = tid; e < SP2; e += 256) {
                const int r = e >> 6, l = e & 63;
                sX[r * LDM + l] = __ldg(U + e) * se[l];
                sY[r * LDM + l] = __ldg(V + e);
            }
        }
        __syncthreads();
        Frag64 pk;
        mm64(sX, sY, pk);                         // P_k = (U e) V
        __syncthreads();                          // every warp is done with U e and V
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const double x = fmax(pk.v[i][j][e], 0.0);
                    accP.v[i][j][e] = fma(cw, x, accP.v[i][j][e]);
                    sY[frag_row(i) * LDM + frag_col(j, e)] = x;
                }
        {
            const double* Q = md.Q + size_t(k) * SP2;
            for (int e = tid; e < SP2; e += 256) sX[(e >> 6) * LDM + (e & 63)] = __ldg(Q + e);
        }
        __syncthreads();
        Frag64 qp;
        mm64(sX, sY, qp);                         // Q clamp(P_k)
        const double sc = cw * rate * cv;
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) accD.v[i][j][e] = fma(sc, qp.v[i][j][e], accD.v[i][j][e]);
    }
    const size_t o = mat_off(m, b, t.n);
    if constexpr (!kMixed) {
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int r = frag_row(i), c = frag_col(j, 0);
                *reinterpret_cast<double2*>(w.P + o + r * SP + c) = make_double2(accP.v[i][j][0], accP.v[i][j][1]);
                *reinterpret_cast<double2*>(w.dP + o + r * SP + c) = make_double2(accD.v[i][j][0], accD.v[i][j][1]);
                w.PT[o + c * SP + r] = accP.v[i][j][0];
                w.PT[o + (c + 1) * SP + r] = accP.v[i][j][1];
            }
    } else {
        __syncthreads();                          // every warp is done reading sX (Q) and sY
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int r = frag_row(i), c = frag_col(j, 0);
                *reinterpret_cast<double2*>(w.dP + o + r * SP + c) = make_double2(accD.v[i][j][0], accD.v[i][j][1]);
                sX[r * LDM + c] = accP.v[i][j][0];
                sX[r * LDM + c + 1] = accP.v[i][j][1];
            }
        __syncthreads();
        // chunk c: row c / 8 of the tile, K = 8 (c % 8) .. +8
        for (int c = tid; c < SP * (SP / 8); c += 256) {
            const int r = c >> 3, k0 = (c & 7) * 8;
            const uint32_t off = tc::kmajor_off16(SP, r, k0) / 2;
            float x[8];
            uint32_t hw[3][4];
            // P tile: row r = output state i, K = input state j
#pragma unroll
            for (int e = 0; e < 8; ++e) x[e] = float(sX[r * LDM + k0 + e]);
#pragma unroll
            for (int e = 0; e < 4; ++e) tc::split3x2(x[2 * e], x[2 * e + 1], hw[0][e], hw[1][e], hw[2][e]);
#pragma unroll
            for (int q = 0; q < 3; ++q)
                *reinterpret_cast<uint4*>(mw.Bp[q] + o + off) = make_uint4(hw[q][0], hw[q][1], hw[q][2], hw[q][3]);
            // P^T tile: row r = input state j, K = output state i; FP32 P^T row r
#pragma unroll
            for (int e = 0; e < 8; ++e) x[e] = float(sX[(k0 + e) * LDM + r]);
#pragma unroll
            for (int e = 0; e < 4; ++e) tc::split3x2(x[2 * e], x[2 * e + 1], hw[0][e], hw[1][e], hw[2][e]);
#pragma unroll
            for (int q = 0; q < 3; ++q)
                *reinterpret_cast<uint4*>(mw.Bpt[q] + o + off) = make_uint4(hw[q][0], hw[q][1], hw[q][2], hw[q][3]);
            float4* pt = reinterpret_cast<float4*>(mw.PT32 + o + size_t(r) * SP + k0);
            pt[0] = make_float4(x[0], x[1], x[2], x[3]);
            pt[1] = make_float4(x[4], x[5], x[6], x[7]);
        }
        if (tid < SP) {
            double rs = 0.0;
            for (int j = 0; j < SP; ++j) rs += sX[tid * LDM + j];
            w.rs[(size_t(m) * t.n + b) * SP + tid] = rs;
            mw.rs32[(size_t(m) * t.n + b) * SP + tid] = float(rs);
        }
    }
}

// Row sums of P_{m,b} (the message of a leaf with missing data).  grid (n, M), block 64.
__global__ void k_rowsum(Topo t, Model md, Work w) {
    pdl_enter();
    const int b = blockIdx.x, m = blockIdx.y, r = threadIdx.x;
    if (b == t.root) return;
    const double* PT = w.PT + mat_off(m, b, t.n) + r;
    double s = 0.0;
    for (int j = 0; j < SP; ++j) s += PT[j * SP];     // sum_j P[r][j], read along PT rows
    w.rs[(size_t(m) * t.n + b) * SP + r] = s;
}

// Caller-supplied P (compute_tree_log_likelihood_from_P): derive PT and row sums.
__global__ void k_prep_given_P(Topo t, Work w) {
    pdl_enter();
    const int b = blockIdx.x, tid = threadIdx.x;
    if (b == t.root) return;
    const double* P = w.P + mat_off(0, b, t.n);
    double* PT = w.PT + mat_off(0, b, t.n);
    for (int e = tid; e < SP2; e += blockDim.x) PT[(e % SP) * SP + e / SP] = P[e];
    if (tid < SP) {
        double s = 0.0;
        for (int j = 0; j < SP; ++j) s += P[tid * SP + j];
        w.rs[size_t(b) * SP + tid] = s;
    }
}

// ------------------------------------------------------------------- inside
// CTA = 8 warps x 32 patterns; warp g owns states [8g, 8g+8) of its 32 patterns
// (lane = pattern), so every global access of a partial is a coalesced 256-byte row.
constexpr int kTileP = 32;      // patterns per CTA in the FP64 pruning kernels
constexpr int kGroups = 8;      // state groups (warps) per CTA

// v[q] *= message of leaf child c for states [8g, 8g+8) of pattern p.
__device__ __forceinline__ void mul_leaf8(double (&v)[8], const Topo& t, const Work& w, int m, int c, int p, int g) {
    const int tx = t.taxon[c];
    const double* PTc = w.PT + mat_off(m, c, t.n);
    const int st = tx < 0 ? -1 : int(t.states[size_t(tx) * t.Pp + p]);
    const double* src;
    if (st >= 0) {
        src = PTc + st * SP + 8 * g;
    } else {
        const uint64_t mk = tx < 0 ? t.all_mask : t.masks[size_t(tx) * t.Pp + p];
        if (mk == 0 || (mk & t.all_mask) == t.all_mask) {
            src = w.rs + (size_t(m) * t.n + c) * SP + 8 * g;
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                double s = 0.0;
                for (uint64_t b = mk; b; b &= b - 1) s += __ldg(PTc + (__ffsll((long long)b) - 1) * SP + 8 * g + q);
                v[q] *= s;
            }
            return;
        }
    }
    const double2* s2 = reinterpret_cast<const double2*>(src);
#pragma unroll
    for (int q = 0; q < 4; ++q) { const double2 x = __ldg(s2 + q); v[2 * q] *= x.x; v[2 * q + 1] *= x.y; }
}

// Power-of-two renormalisation of a 64-state column spread over the 8 warps:
// returns the shift applied (same on every warp of a lane).
__device__ __forceinline__ int renorm_cols(double (&v)[8], double* smax, int g, int lane) {
    double mx = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) mx = fmax(mx, v[q]);
    smax[g * kTileP + lane] = mx;
    __syncthreads();
    double all = 0.0;
#pragma unroll
    for (int k = 0; k < kGroups; ++k) all = fmax(all, smax[k * kTileP + lane]);
    __syncthreads();
    if (all > 0.0 && all < 0x1p-256) {
        const int sh = -ilogb(all) - 1;
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = ldexp(v[q], sh);
        return sh;
    }
    return 0;
}

// Partial tiles of the FP64 pruning CTAs in shared memory: [64 states][32 patterns] with a row
// stride of kDL = 36 doubles, so the B-fragment loads (k + lane%4) * 36 + col + lane/4 of a half-warp
// fall in 16 different banks.
constexpr int kDL = kTileP + 4;

__device__ __forceinline__ void cp_async16_f64(double* dst, const double* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;"
                 ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))), "l"(src) : "memory");
}

// Stage a 64x64 matrix row-major with the padded stride LDM (k_build_P's operand layout) by 16-byte
// cp.async, one commit group: the copy runs while the CTA loads and multiplies its partials;
// stage_wait() before the product reads it.
__device__ __forceinline__ void stage_matrix_pad_async(double* __restrict__ s, const double* __restrict__ g, int tid, int nthr) {
    for (int e = tid; e < SP2 / 2; e += nthr) {
        const int r = e / (SP / 2), c2 = e % (SP / 2);
        cp_async16_f64(s + r * LDM + 2 * c2, g + 2 * e);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// dst[i][p] = sum_k sM[i][k] sX[k][p] for the CTA's 64 x 32 tile on the FP64 tensor cores
// (mma.sync m8n8k4): warp w owns output rows 8w .. 8w+7, all 32 columns as four 8x8 tiles,
// 16 k steps of 4.  sM [64][LDM] row-major, sX [64][kDL]; dst has row stride `stride`
// (state-major partials), each thread storing two adjacent patterns as one 16-byte write.
__device__ __forceinline__ void tile_mm_store(const double* __restrict__ sM, const double* __restrict__ sX,
                                              double* __restrict__ dst, size_t stride) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
    double c[4][2];
#pragma unroll
    for (int j = 0; j < 4; ++j) c[j][0] = c[j][1] = 0.0;
    const double* arow = sM + (8 * wp + g) * LDM + q;
#pragma unroll 4
    for (int k = 0; k < SP; k += 4) {
        const double a = arow[k];
        const double* brow = sX + (k + q) * kDL + g;
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(c[j][0], c[j][1], a, brow[8 * j]);
    }
    double* d = dst + size_t(8 * wp + g) * stride + 2 * q;
#pragma unroll
    for (int j = 0; j < 4; ++j) *reinterpret_cast<double2*>(d + 8 * j) = make_double2(c[j][0], c[j][1]);
}

// grid (Pp/32, nodes in level, M), block 256, dynamic smem (64*LDM + 64*kDL + 8*32) doubles.
__global__ void __launch_bounds__(256) k_inside(Topo t, Model md, Work w, const int* __restrict__ nodes) {
    pdl_enter();
    extern __shared__ __align__(16) double sm[];
    double* sP = sm;                     // P_u row-major [64][LDM]
    double* sD = sm + SP * LDM;          // D_u tile [64][kDL]
    double* smax = sD + SP * kDL;        // [8][32]
    const int u = nodes[blockIdx.y], m = blockIdx.z, tid = threadIdx.x;
    const int g = tid >> 5, lane = tid & 31;
    const int p = blockIdx.x * kTileP + lane;
    const int iu = t.iidx[u], M = md.M;
    const size_t Pp = size_t(t.Pp);
    const bool root = (u == t.root);
    if (!root) stage_matrix_pad_async(sP, w.P + mat_off(m, u, t.n), tid, 256);
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = (8 * g + q) < t.S ? 1.0 : 0.0;
    int ecum = 0, eown = 0;
    for (int k = t.ch_off[u]; k < t.ch_off[u + 1]; ++k) {
        const int c = t.ch[k];
        if (t.leaf[c]) {
            mul_leaf8(v, t, w, m, c, p, g);
        } else {
            const int ic = t.iidx[c];
            const double* src = w.Ms + part_off(ic, m, M, t.Pp) + size_t(8 * g) * Pp + p;
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] *= src[q * Pp];
            ecum += w.Ecum[col_off(ic, m, M, t.Pp) + p];
        }
        eown += renorm_cols(v, smax, g, lane);
    }
    double* dst = w.D + part_off(iu, m, M, t.Pp) + size_t(8 * g) * Pp + p;
#pragma unroll
    for (int q = 0; q < 8; ++q) dst[q * Pp] = v[q];
    if (g == 0) {
        w.Eown[col_off(iu, m, M, t.Pp) + p] = eown;
        w.Ecum[col_off(iu, m, M, t.Pp) + p] = ecum + eown;
    }
    if (root) return;
#pragma unroll
    for (int q = 0; q < 8; ++q) sD[(8 * g + q) * kDL + lane] = v[q];
    stage_wait();
    __syncthreads();
    // message to the parent: (P_u D_u)_i = sum_j P[i][j] D_j
    tile_mm_store(sP, sD, w.Ms + part_off(iu, m, M, t.Pp) + size_t(blockIdx.x) * kTileP, Pp);
}

// --------------------------------------------------------------------- root
__global__ void k_root(Topo t, Model md, Work w) {
    pdl_enter();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= t.Pp) return;
    const int ir = t.iidx[t.root], M = md.M;
    const double wt = t.w[p];
    double L[kMaxRateClasses], ll[kMaxRateClasses];
    for (int m = 0; m < M; ++m) {
        const double* D = w.D + part_off(ir, m, M, t.Pp) + p;
        double s = 0.0;
        for (int i = 0; i < SP; ++i) s = fma(md.pi[i], D[size_t(i) * t.Pp], s);
        L[m] = s;
        ll[m] = s > 0.0 ? log(s) - double(w.Ecum[col_off(ir, m, M, t.Pp) + p]) * 0.69314718055994530942 : -1e20;
    }
    double site = -1e20, contrib = 0.0;
    bool ok = false;
    if (M == 1) {
        if (L[0] > 0.0) {
            ok = true; site = ll[0]; contrib = wt * ll[0];
            w.f[p] = wt / L[0];
        } else {
            w.f[p] = 0.0;
        }
        w.rw[p] = 0.0;
    } else {
        double mx = -INFINITY;
        for (int m = 0; m < M; ++m)
            if (md.rate_w[m] > 1e-12 && L[m] > 0.0) mx = fmax(mx, log(md.rate_w[m]) + ll[m]);
        double post[kMaxRateClasses], se = 0.0;
        for (int m = 0; m < M; ++m) {
            post[m] = 0.0;
            if (mx > -1e19 && md.rate_w[m] > 1e-12 && L[m] > 0.0) { post[m] = exp(log(md.rate_w[m]) + ll[m] - mx); se += post[m]; }
        }
        if (mx > -1e19 && se > 0.0) { ok = true; site = mx + log(se); contrib = wt * site; }
        for (int m = 0; m < M; ++m) {
            const double pw = ok ? post[m] / se : 0.0;
            w.f[size_t(m) * t.Pp + p] = (ok && pw > 1e-12) ? wt * pw / L[m] : 0.0;
            w.rw[size_t(m) * t.Pp + p] = ok ? wt * pw / md.rate_w[m] : 0.0;
        }
    }
    if (!ok && md.sentinel) contrib = wt * -1e20;
    w.contrib[p] = contrib;
    w.site[p] = site;
}

// ------------------------------------------------------------------ outside
// One CTA per (child c of a node at this depth, 32-pattern tile, rate class):
// V_c = 2^{e_u} U_u o prod_{s != c} (P_s D_s), then U_c = P_c^T V_c for internal c.
// grid (Pp/32, children in level, M), block 256, dynamic smem (64*64 + 64*32 + 8*32) doubles.
__global__ void __launch_bounds__(256) k_outside(Topo t, Model md, Work w, const int* __restrict__ kids, int want_v) {
    pdl_enter();
    extern __shared__ __align__(16) double sm[];
    double* sPT = sm;                    // P_c^T row-major [64][LDM]
    double* sV = sm + SP * LDM;          // V_c tile [64][kDL]
    double* smax = sV + SP * kDL;
    const int c = kids[blockIdx.y], m = blockIdx.z, tid = threadIdx.x;
    const int g = tid >> 5, lane = tid & 31;
    const int p = blockIdx.x * kTileP + lane;
    const int u = t.parent[c], iu = t.iidx[u], M = md.M;
    const size_t Pp = size_t(t.Pp);
    const bool internal = !t.leaf[c];
    if (internal) stage_matrix_pad_async(sPT, w.PT + mat_off(m, c, t.n), tid, 256);
    double v[8];
    if (u == t.root) {
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = md.pi[8 * g + q];
    } else {
        const double* src = w.U + part_off(iu, m, M, t.Pp) + size_t(8 * g) * Pp + p;
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = src[q * Pp];
    }
    int ev = w.Eown[col_off(iu, m, M, t.Pp) + p];
    for (int k = t.ch_off[u]; k < t.ch_off[u + 1]; ++k) {
        const int s = t.ch[k];
        if (s == c) continue;
        if (t.leaf[s]) {
            mul_leaf8(v, t, w, m, s, p, g);
        } else {
            const double* src = w.Ms + part_off(t.iidx[s], m, M, t.Pp) + size_t(8 * g) * Pp + p;
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] *= src[q * Pp];
        }
        ev -= renorm_cols(v, smax, g, lane);
    }
    if (ev != 0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = ldexp(v[q], ev);
    }
    if (want_v) {
        const double fp = w.f[size_t(m) * Pp + p];
        double* dst = w.Vf + part_off(vslot(t, c), m, M, t.Pp) + size_t(8 * g) * Pp + p;
#pragma unroll
        for (int q = 0; q < 8; ++q) dst[q * Pp] = fp * v[q];
    }
    if (!internal) return;
#pragma unroll
    for (int q = 0; q < 8; ++q) sV[(8 * g + q) * kDL + lane] = v[q];
    stage_wait();
    __syncthreads();
    // U_c = P_c^T V_c : (U_c)_i = sum_j PT[i][j] V_j
    tile_mm_store(sPT, sV, w.U + part_off(t.iidx[c], m, M, t.Pp) + size_t(blockIdx.x) * kTileP, Pp);
}

// ------------------------------------------------------------------ accum A
// A_{m,b,chunk} = sum_{p in chunk} Vf_b[:, p] D_b[:, p]^T on the FP64 tensor cores: C = X Y^T with
// X = Vf (64 states x patterns), Y = D, K = the pattern axis.  8 warps as mm64 (warp w: rows
// 16(w/2) .. +16, columns 32(w%2) .. +32, 2 x 4 tiles of 8x8), 32 patterns per stage, stages
// double-buffered by 16-byte cp.async (a leaf's 0/1 vectors are written from its states and
// masks instead).  grid (branches, M, nchunk), block 256; `branches` lists the branches (NULL: every
// node id, the root skipped).
constexpr int kAccP = 32;                                      // patterns per stage
constexpr int kAL = kAccP + 4;                                 // row stride of a staged tile (doubles)
constexpr size_t kAccStage = size_t(2) * SP * kAL;             // V and D tiles of one stage
static const size_t kAccSmemF = 2 * kAccStage * sizeof(double);

__global__ void __launch_bounds__(256) k_accumA(Topo t, Model md, Work w, const int* __restrict__ branches) {
    pdl_enter();
    extern __shared__ __align__(16) double smA[];
    const int b = branches ? branches[blockIdx.x] : int(blockIdx.x), m = blockIdx.y, ck = blockIdx.z, tid = threadIdx.x;
    if (b == t.root) return;
    const int M = md.M;
    const size_t Pp = size_t(t.Pp);
    const int p_begin = ck * w.chunk, p_end = min(t.Pp, p_begin + w.chunk);
    const int nst = (p_end - p_begin) / kAccP;
    const bool lf = t.leaf[b];
    const int tx = lf ? t.taxon[b] : -1;
    const double* Vb = w.Vf + part_off(vslot(t, b), m, M, t.Pp);
    const double* Db = lf ? nullptr : w.D + part_off(t.iidx[b], m, M, t.Pp);

    // stage `st` of the chunk into buffer st & 1: 64 state rows x 32 patterns of Vf (and D)
    auto stage = [&](int st) {
        double* sV = smA + size_t(st & 1) * kAccStage;
        double* sD = sV + SP * kAL;
        const size_t p0 = size_t(p_begin) + size_t(st) * kAccP;
        for (int c = tid; c < SP * (kAccP / 2); c += 256) {
            const int r = c / (kAccP / 2), q2 = c % (kAccP / 2);
            cp_async16_f64(sV + r * kAL + 2 * q2, Vb + size_t(r) * Pp + p0 + 2 * q2);
            if (!lf) cp_async16_f64(sD + r * kAL + 2 * q2, Db + size_t(r) * Pp + p0 + 2 * q2);
        }
        if (lf) {
            // pattern p0 + (tid % 32), states 8 (tid / 32) .. +8 of the leaf's 0/1 vector
            const int pp = tid & 31, j0 = 8 * (tid >> 5);
            const size_t p = p0 + pp;
            const int sv = tx < 0 ? -1 : int(t.states[size_t(tx) * Pp + p]);
            const uint64_t mk = (tx < 0 || sv >= 0) ? 0 : t.masks[size_t(tx) * Pp + p];
            const bool all = tx < 0 || (sv < 0 && (mk == 0 || (mk & t.all_mask) == t.all_mask));
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int j = j0 + q;
                double d = 0.0;
                if (j < t.S) d = all ? 1.0 : (sv >= 0 ? (sv == j ? 1.0 : 0.0) : (((mk >> j) & 1) ? 1.0 : 0.0));
                sD[j * kAL + pp] = d;
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    const int lane = tid & 31, wp = tid >> 5, g = lane >> 2, q = lane & 3;
    const int r0 = 16 * (wp >> 1), c0 = 32 * (wp & 1);
    Frag64 acc;
    frag_zero(acc);
    if (nst > 0) stage(0);
    for (int st = 0; st < nst; ++st) {
        if (st + 1 < nst) stage(st + 1);
        else asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();
        const double* sV = smA + size_t(st & 1) * kAccStage;
        const double* sD = sV + SP * kAL;
#pragma unroll
        for (int k = 0; k < kAccP; k += 4) {
            double a[2], bb[4];
#pragma unroll
            for (int i = 0; i < 2; ++i) a[i] = sV[(r0 + 8 * i + g) * kAL + k + q];
#pragma unroll
            for (int j = 0; j < 4; ++j) bb[j] = sD[(c0 + 8 * j + g) * kAL + k + q];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc.v[i][j][0], acc.v[i][j][1], a[i], bb[j]);
        }
        __syncthreads();                         // the buffer is refilled by the next iteration's stage
    }
    double* dst = w.Apart + ((size_t(b) * M + m) * w.nchunk + ck) * SP2;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
            *reinterpret_cast<double2*>(dst + frag_row(i) * SP + frag_col(j, 0)) = make_double2(acc.v[i][j][0], acc.v[i][j][1]);
}

__device__ __forceinline__ double block_sum_256(double x, double* red) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = x;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) for (int i = 0; i < 8; ++i) s += red[i];
    return s;   // valid on thread 0
}

// A_{m,b} = sum of the chunk partials in chunk order, and dlnL/dt_b's term
// <A_{m,b}, dP_{m,b}>.  grid (n, M), block 256.
__global__ void __launch_bounds__(256) k_areduce(Topo t, Model md, Work w) {
    pdl_enter();
    __shared__ double red[8];
    const int b = blockIdx.x, m = blockIdx.y, tid = threadIdx.x, n = t.n, M = md.M;
    if (b == t.root) return;
    const double* Ap = w.Apart + (size_t(b) * M + m) * w.nchunk * SP2;
    const double* dP = w.dP + mat_off(m, b, n);
    double* Af = w.Afull + (size_t(b) * M + m) * SP2;
    double g = 0.0;
    for (int e = tid; e < SP2; e += 256) {
        double s = 0.0;
        for (int ck = 0; ck < w.nchunk; ++ck) s += Ap[size_t(ck) * SP2 + e];
        Af[e] = s;
        g = fma(s, dP[e], g);
    }
    g = block_sum_256(g, red);
    if (tid == 0) w.gt[size_t(m) * n + b] = g;
}

// ------------------------------------------------------------------ frechet
// grid (G, M, nmod): CTA (g, m, k) walks the branches b = g, g+G, ... that use
// model k (test branches for k < K, background branches for k = K), computes
// the spectral transform At = U_k^T A_{m,b} V_k^T (two FP64 tensor-core products,
// mm64) and accumulates H += c_k At o E(lambda, tau_b) in registers
// (likelihood.hpp:1428-1471), plus the diagonal sums for d/dc_k and the d mu term.
// block 256, dynamic smem 3 x 64 x LDM doubles (U_k^T, V_k^T, A then T).
__global__ void __launch_bounds__(256) k_frechet(Topo t, Model md, Work w, int G) {
    pdl_enter();
    extern __shared__ __align__(16) double sm[];
    double* sUT = sm;                     // U_k^T: sUT[r][l] = U[l][r]
    double* sVT = sm + SP * LDM;          // V_k^T: sVT[l][c] = V[c][l]
    double* sA = sm + 2 * SP * LDM;       // A_{m,b}, then T = U^T A
    __shared__ double se[SP];
    __shared__ double red[8];
    const int g = blockIdx.x, m = blockIdx.y, k = blockIdx.z, tid = threadIdx.x, n = t.n, M = md.M;
    for (int e = tid; e < SP2; e += 256) {
        const int x = e >> 6, y = e & 63;                 // coalesced reads of U[x][y], V[x][y]
        sUT[y * LDM + x] = md.U[size_t(k) * SP2 + e];
        sVT[y * LDM + x] = md.V[size_t(k) * SP2 + e];
    }
    const double* lam = md.lam + size_t(k) * SP;
    Frag64 H;
    frag_zero(H);
    double dg = 0.0, dq = 0.0;
    for (int b = g; b < n; b += G) {
        if (b == t.root) continue;
        const BranchModels bm = branch_models(md, b);
        if (k < bm.k0 || k >= bm.k1) continue;
        const double cw = class_weight(md, bm, k);
        const double tau = md.rates[m] * w.bl[b] * time_conv(md, k);
        __syncthreads();                                  // the previous branch is done with sA
        {
            const double* A = w.Afull + (size_t(b) * M + m) * SP2;
            for (int e = tid; e < SP2; e += 256) sA[(e >> 6) * LDM + (e & 63)] = __ldg(A + e);
        }
        if (tid < SP) se[tid] = exp(lam[tid] * tau);
        __syncthreads();
        Frag64 T;
        mm64(sUT, sA, T);                                 // T = U^T A
        __syncthreads();                                  // every warp is done with A: T overwrites it
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                *reinterpret_cast<double2*>(sA + frag_row(i) * LDM + frag_col(j, 0)) = make_double2(T.v[i][j][0], T.v[i][j][1]);
        __syncthreads();
        Frag64 At;
        mm64(sA, sVT, At);                                // At = T V^T
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = frag_row(i);
            const double li = lam[r], ei = se[r];
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int c = frag_col(j, e);
                    const double d = li - lam[c], ej = se[c], a = At.v[i][j][e];
                    const double E = fabs(d) < 1e-9 ? tau * ei : (ei - ej) / d;
                    H.v[i][j][e] = fma(cw * a, E, H.v[i][j][e]);
                    if (r == c) {
                        dg += ei * a;
                        dq += cw * tau * li * ei * a;
                    }
                }
        }
    }
    double* Hp = w.Hpart + ((size_t(k) * M + m) * G + g) * SP2;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
            *reinterpret_cast<double2*>(Hp + frag_row(i) * SP + frag_col(j, 0)) = make_double2(H.v[i][j][0], H.v[i][j][1]);
    dg = block_sum_256(dg, red);
    dq = block_sum_256(dq, red);
    if (tid == 0) {
        const size_t o = (size_t(k) * M + m) * G + g;
        w.gc[o] = dg;
        w.stg[o] = dq;
    }
}

// H_k[e] = sum over (m, g) of the per-CTA partials (fixed order: four interleaved
// running sums, combined pairwise), then the directional contractions
// dirpart[x][k][block] = sum over this block's 256 entries of H_k o G_{x,k}.
// grid (nmod, 16), block 256.
__global__ void __launch_bounds__(256) k_hsum(Topo t, Model md, Work w, int G) {
    pdl_enter();
    __shared__ double red[8];
    const int k = blockIdx.x, e = blockIdx.y * 256 + threadIdx.x, M = md.M, nt = M * G;
    const double* hp = w.Hpart + size_t(k) * nt * SP2 + e;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int i = 0;
    for (; i + 4 <= nt; i += 4) {
        s0 += hp[size_t(i) * SP2];
        s1 += hp[size_t(i + 1) * SP2];
        s2 += hp[size_t(i + 2) * SP2];
        s3 += hp[size_t(i + 3) * SP2];
    }
    for (; i < nt; ++i) s0 += hp[size_t(i) * SP2];
    const double h = (s0 + s1) + (s2 + s3);
    w.H[size_t(k) * SP2 + e] = h;
    for (int x = 0; x < md.ndirs; ++x) {
        const double v = block_sum_256(h * w.G[(size_t(x) * md.nmod + k) * SP2 + e], red);
        if (threadIdx.x == 0) w.dirpart[(size_t(x) * md.nmod + k) * 17 + blockIdx.y] = v;
    }
}

// G_{x,k} = V_k dQ_{x,k} U_k, rows [16rb, 16rb+16); block 0 also stores
// d mu = -sum_i pi_i dQ_ii.  Depends on the model only, so it runs on a side
// stream alongside the pruning passes.  grid (ndirs, nmod, 4), block 256,
// dynamic smem (64*64 + 16*64 + 16*64) doubles.
__global__ void __launch_bounds__(256) k_dir(Topo t, Model md, Work w) {
    pdl_enter();
    extern __shared__ __align__(16) double sm[];
    double* sX = sm;                 // dQ, later U_k
    double* sY = sm + SP2;           // (V dQ)[rows, :]
    double* sVr = sY + 16 * SP;      // V_k rows of the block
    __shared__ double red[8];
    const int x = blockIdx.x, k = blockIdx.y, rb = blockIdx.z, tid = threadIdx.x;
    const bool own = x >= md.ndirs_dense;                 // a per-model direction: model x - ndirs_dense only
    if (own && k != x - md.ndirs_dense) {
        double* Gz = w.G + (size_t(x) * md.nmod + k) * SP2 + size_t(16 * rb) * SP;
        for (int e = tid; e < 16 * SP; e += 256) Gz[e] = 0.0;
        if (rb == 0 && tid == 0) w.dirpart[(size_t(x) * md.nmod + k) * 17 + 16] = 0.0;
        return;
    }
    const double* dQ = own ? md.dQ + (size_t(md.ndirs_dense) * md.nmod + k) * SP2 : md.dQ + (size_t(x) * md.nmod + k) * SP2;
    stage_matrix(sX, dQ, tid, 256);
    for (int e = tid; e < 16 * SP; e += 256) sVr[e] = md.V[size_t(k) * SP2 + size_t(16 * rb) * SP + e];
    __syncthreads();
    const int r = tid >> 4, c0 = (tid & 15) * 4;   // 16 rows x 64 columns, 4 per thread
    double acc[4] = {0, 0, 0, 0};
    for (int l = 0; l < SP; ++l) {
        const double a = sVr[r * SP + l];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] = fma(a, sX[l * SP + c0 + q], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) sY[r * SP + c0 + q] = acc[q];
    double dmu = 0.0;
    if (rb == 0 && tid < SP) dmu = -md.pi[tid] * dQ[tid * SP + tid];
    __syncthreads();
    stage_matrix(sX, md.U + size_t(k) * SP2, tid, 256);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = 0.0;
    for (int l = 0; l < SP; ++l) {
        const double a = sY[r * SP + l];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] = fma(a, sX[l * SP + c0 + q], acc[q]);
    }
    double* Gx = w.G + (size_t(x) * md.nmod + k) * SP2 + size_t(16 * rb + r) * SP + c0;
#pragma unroll
    for (int q = 0; q < 4; ++q) Gx[q] = acc[q];
    dmu = block_sum_256(dmu, red);
    if (rb == 0 && tid == 0) w.dirpart[(size_t(x) * md.nmod + k) * 17 + 16] = dmu;
}

// Fixed-order reductions of the small per-branch / per-pattern partials.
// One block of 256 threads.
__global__ void __launch_bounds__(256) k_small(Topo t, Model md, Work w, int grads) {
    pdl_enter();
    __shared__ double red[8];
    const int tid = threadIdx.x, n = t.n, M = md.M;
    // lnL: per-thread Neumaier over a strided slice, then a fixed tree
    double s = 0.0, c = 0.0;
    for (int p = tid; p < t.Pp; p += 256) {
        const double x = w.contrib[p], y = s + x;
        c += fabs(s) >= fabs(x) ? (s - y) + x : (x - y) + s;
        s = y;
    }
    double tot = block_sum_256(s + c, red);
    if (tid == 0) { w.out[0] = tot; w.out[1] = w.err ? double(*w.err) : 0.0; }
    if (!grads) return;
    for (int b = tid; b < n; b += 256) {
        double g = 0.0;
        if (b != t.root) for (int m = 0; m < M; ++m) g += w.gt[size_t(m) * n + b];
        w.out[2 + b] = g;
    }
    for (int k = 0; k < md.nmod; ++k) {
        double a = 0.0, z = 0.0;
        for (int idx = tid; idx < M * w.ngroups; idx += 256) {
            a += w.gc[size_t(k) * M * w.ngroups + idx];
            z += w.stg[size_t(k) * M * w.ngroups + idx];
        }
        a = block_sum_256(a, red);
        z = block_sum_256(z, red);
        if (tid == 0) {
            w.out[2 + n + k] = a;                 // d lnL / d (class or background weight of model k)
            w.out[2 + n + md.nmod + k] = z;
        }
    }
    for (int m = 0; m < M; ++m) {
        double a = 0.0;
        for (int p = tid; p < t.Pp; p += 256) a += w.rw[size_t(m) * t.Pp + p];
        a = block_sum_256(a, red);
        if (tid == 0) w.out[2 + n + 2 * md.nmod + m] = a;
    }
}

// ------------------------------------------------------------------ launch
static const size_t kPruneSmem = (SP * LDM + SP * kDL + kGroups * kTileP) * sizeof(double);
static const size_t kDirSmem = (2 * SP2 + 16 * SP) * sizeof(double);
static const size_t kBuildSmem = size_t(2) * SP * LDM * sizeof(double);
static const size_t kFrechetSmem = size_t(3) * SP * LDM * sizeof(double);

void fp64_configure() {
    cudaFuncSetAttribute(k_build_P<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kBuildSmem));
    cudaFuncSetAttribute(k_build_P<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kBuildSmem));
    cudaFuncSetAttribute(k_inside, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kPruneSmem));
    cudaFuncSetAttribute(k_outside, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kPruneSmem));
    cudaFuncSetAttribute(k_frechet, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kFrechetSmem));
    cudaFuncSetAttribute(k_dir, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kDirSmem));
    cudaFuncSetAttribute(k_accumA, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kAccSmemF));
}

int launch_build_P(const Topo& t, const Model& md, const Work& w, cudaStream_t s) {
    launch_k(k_build_P<false>, dim3(t.n, md.M), 256, kBuildSmem, s, t, md, w, MixedWork{});
    launch_k(k_rowsum, dim3(t.n, md.M), SP, 0, s, t, md, w);
    return 2;
}
int launch_build_P_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, cudaStream_t s) {
    launch_k(k_build_P<true>, dim3(t.n, md.M), 256, kBuildSmem, s, t, md, w, mw);
    return 1;
}
int launch_prep_given_P(const Topo& t, const Work& w, cudaStream_t s) {
    launch_k(k_prep_given_P, t.n, 256, 0, s, t, w);
    return 1;
}
int launch_inside_fp64(const Topo& t, const Model& md, const Work& w, const int* d_nodes, int count, cudaStream_t s) {
    launch_k(k_inside, dim3(t.Pp / kTileP, count, md.M), 256, kPruneSmem, s, t, md, w, d_nodes);
    return 1;
}
int launch_root(const Topo& t, const Model& md, const Work& w, cudaStream_t s) {
    launch_k(k_root, (t.Pp + 127) / 128, 128, 0, s, t, md, w);
    return 1;
}
int launch_outside_fp64(const Topo& t, const Model& md, const Work& w, const int* d_kids, int count, int want_v, cudaStream_t s) {
    launch_k(k_outside, dim3(t.Pp / kTileP, count, md.M), 256, kPruneSmem, s, t, md, w, d_kids, want_v);
    return 1;
}
int launch_accumA_fp64(const Topo& t, const Model& md, const Work& w, const int* d_branches, int count, cudaStream_t s) {
    const int* none = nullptr;
    launch_k(k_accumA, dim3(d_branches ? count : t.n, md.M, w.nchunk), 256, kAccSmemF, s, t, md, w,
             d_branches ? d_branches : none);
    return 1;
}
int launch_frechet(const Topo& t, const Model& md, const Work& w, int want_global, cudaStream_t s) {
    launch_k(k_areduce, dim3(t.n, md.M), 256, 0, s, t, md, w);
    if (!want_global) return 1;
    launch_k(k_frechet, dim3(w.ngroups, md.M, md.nmod), 256, kFrechetSmem, s, t, md, w, w.ngroups);
    return 2;
}
int launch_global(const Topo& t, const Model& md, const Work& w, cudaStream_t s) {
    launch_k(k_hsum, dim3(md.nmod, SP2 / 256), 256, 0, s, t, md, w, w.ngroups);
    return 1;
}
int launch_dir(const Topo& t, const Model& md, const Work& w, cudaStream_t s) {
    if (md.ndirs <= 0) return 0;
    launch_k(k_dir, dim3(md.ndirs, md.nmod, 4), 256, kDirSmem, s, t, md, w);
    return 1;
}
// The evaluation's results as one FP64 vector on the device, in the order
// [lnl, grad_t (n, root 0), grad_dir (ndirs), grad_class_w (K), grad_rate_w (M), failed]:
// every entry is a sum over site patterns (grad_dir's d mu term multiplies one such sum by a
// model constant), so vectors of pattern shards add up to the whole alignment's.  The directional
// gradient is assembled here from the 16 Frechet partials per (direction, model) exactly as the
// host does for h3g_eval.  One block.
__global__ void k_pack_result(Topo t, Model md, Work w, int grads, int global, double* dst) {
    const int tid = threadIdx.x, n = t.n, K = md.K, M = md.M, nmod = md.nmod, ndirs = md.ndirs;
    const double* out = w.out;
    if (tid == 0) {
        dst[0] = out[0];
        dst[1 + n + ndirs + K + M] = out[1] != 0.0 ? 1.0 : 0.0;
    }
    for (int b = tid; b < n; b += blockDim.x) dst[1 + b] = (grads && b != t.root) ? out[2 + b] : 0.0;
    for (int x = tid; x < ndirs; x += blockDim.x) {
        double g = 0.0;
        if (global)
            for (int k = 0; k < nmod; ++k) {
                const double* d = w.dirpart + (size_t(x) * nmod + k) * 17;
                double v = 0.0;
                for (int q = 0; q < 16; ++q) v += d[q];
                if (md.time_mode == 1) v -= d[16] / fmax(md.mu[k], 1e-12) * out[2 + n + nmod + k];
                g += v;
            }
        dst[1 + n + x] = g;
    }
    for (int k = tid; k < K; k += blockDim.x) dst[1 + n + ndirs + k] = global ? out[2 + n + k] : 0.0;
    for (int m = tid; m < M; m += blockDim.x) dst[1 + n + ndirs + K + m] = grads ? out[2 + n + 2 * nmod + m] : 0.0;
}

int launch_pack_result(const Topo& t, const Model& md, const Work& w, int grads, int global, double* dst, cudaStream_t s) {
    launch_k(k_pack_result, 1, 256, 0, s, t, md, w, grads, global, dst);
    return 1;
}

int launch_small(const Topo& t, const Model& md, const Work& w, int grads, cudaStream_t s) {
    launch_k(k_small, 1, 256, 0, s, t, md, w, grads);
    return 1;
}

bool pdl_enabled() {
    static const bool on = [] { const char* e = std::getenv("H3G_NO_PDL"); return !(e && e[0] == '1'); }();
    return on;
}

}  // namespace h3g
