// h3g_fel.cu — batched device evaluator for FEL per-site fits.
//
// The reference evaluates one pattern at a time on the CPU: for every trial
// (alpha, beta) it re-eigensolves MG94 at omega = beta / alpha, builds the
// transition matrix of every branch and prunes the single pattern
// (analyses/fel.hpp:276-308, :365-383).  Here one optimiser step of every
// pattern is evaluated in one batch:
//
//   k_fel_eig   one CTA per distinct omega of the batch: the symmetric form
//               of Q(omega) = Qs + omega Qn is diagonalised by the parallel
//               (round-robin) cyclic Jacobi method in shared memory; the
//               slot receives lambda (clamped <= 0), U_pi and V_pi.
//   k_fel_lnl   one CTA per request: single-pattern pruning in the spectral
//               domain.  The message of branch b is
//               U (e^{lambda a t_b} o (V L_b)), two 64x64 mat-vecs from shared
//               memory, so no transition matrix is ever formed.  The tree is
//               walked depth-first; open partials live on a per-CTA stack,
//               with power-of-two rescaling when a partial falls below 2^-256.
//
// Everything is FP64: FEL results are compared with the reference's.
#include <algorithm>
#include <cmath>
#include <new>
#include <type_traits>
#include <vector>

#include "h3g_common.cuh"
#include "h3g_fel.h"
#include "h3g_jacobi.cuh"

namespace h3g {

Topo problem_topo(h3g_problem* pr, int S);         // h3g_capi.cu
cudaStream_t problem_stream(h3g_problem* pr);      // h3g_capi.cu

namespace {

constexpr int kFT = 256;                  // threads per CTA
constexpr int LD = jac::LD;               // padded row stride: column walks hit 32 distinct banks
constexpr int kMaxSweeps = 30;
constexpr int kMaxDepth = 1024;           // open internal nodes on the traversal stack
constexpr size_t kEigSmem = size_t(2) * SP * LD * sizeof(double);

struct FelModel {
    int S;
    const double* Qs;     // [S][S]
    const double* Qn;     // [S][S]
    const double* sq;     // [64] sqrt(max(pi, 1e-12)), 0 on padding
    const double* isq;    // [64] 1 / sq, 0 on padding
    const double* pi;     // [64]
    double* lam;          // [slots][64]
    double* U;            // [slots][64*64]
    double* V;            // [slots][64*64]
    const uint8_t* bg;    // [n] 1 on a background branch (requests with a background eigensystem)
};

// ----------------------------------------------------------------- eigensystems
// grid n_eig, block 256.  Jacobi rotations as in Golub & Van Loan (Alg. 8.5.3);
// one sweep = 63 rounds of 32 disjoint pairs (circle schedule), each round
// A <- A J (columns) then A <- J^T A (rows), E <- E J.
// Warm start: when prev[r] >= 0 the eigenvectors E0 of that slot (E0 = D^1/2 U)
// are the starting basis: A <- E0^T A E0, E <- E0.  A pattern's next omega is
// usually close to its last one, so the rotated matrix is nearly diagonal and
// the sweeps needed drop from ~8 to 2-3.
__global__ void __launch_bounds__(kFT) k_fel_eig(FelModel f, const double* __restrict__ omega, const int* __restrict__ slot,
                                                 const int* __restrict__ prev) {
    pdl_enter();
    extern __shared__ __align__(16) double sm[];
    double* A = sm;
    double* E = sm + SP * LD;
    __shared__ jac::Scratch js;
    const int tid = threadIdx.x, S = f.S;
    const double om = omega[blockIdx.x];
    const int sl = slot[blockIdx.x];
    for (int e = tid; e < SP2; e += kFT) {
        const int i = e >> 6, j = e & 63;
        double v = 0.0;
        if (i < S && j < S && i != j) v = f.sq[i] * (f.Qs[i * S + j] + om * f.Qn[i * S + j]) * f.isq[j];
        A[i * LD + j] = v;
        E[i * LD + j] = i == j ? 1.0 : 0.0;
    }
    __syncthreads();
    if (tid < S) {
        double row = 0.0;
        for (int j = 0; j < S; ++j)
            if (j != tid) row += f.Qs[tid * S + j] + om * f.Qn[tid * S + j];
        A[tid * LD + tid] = -row;
    }
    __syncthreads();
    for (int e = tid; e < SP2; e += kFT) {        // symmetric part (rate_matrix.hpp:236-237)
        const int i = e >> 6, j = e & 63;
        if (i < j) {
            const double m = 0.5 * (A[i * LD + j] + A[j * LD + i]);
            A[i * LD + j] = m;
            A[j * LD + i] = m;
        }
    }
    __syncthreads();
    const int pv = prev[blockIdx.x];
    if (pv >= 0) {
        const double* U0 = f.U + size_t(pv) * SP2;
        for (int e = tid; e < SP2; e += kFT) {
            const int i = e >> 6, k = e & 63;
            E[i * LD + k] = i < S ? f.sq[i] * U0[e] : (i == k ? 1.0 : 0.0);
        }
        __syncthreads();
        const int i = tid & 63, kq = (tid >> 6) * 16;
        double acc[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) acc[m] = 0.0;
        for (int j = 0; j < SP; ++j) {                   // T = A E0, row i, columns kq..kq+15
            const double aij = A[i * LD + j];
#pragma unroll
            for (int m = 0; m < 16; ++m) acc[m] = fma(aij, E[j * LD + kq + m], acc[m]);
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 16; ++m) A[i * LD + kq + m] = acc[m];
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 16; ++m) acc[m] = 0.0;
        for (int j = 0; j < SP; ++j) {                   // B = E0^T T, row k = i, columns kq..kq+15
            const double ejk = E[j * LD + i];
#pragma unroll
            for (int m = 0; m < 16; ++m) acc[m] = fma(ejk, A[j * LD + kq + m], acc[m]);
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 16; ++m) A[i * LD + kq + m] = acc[m];
        __syncthreads();
        for (int e = tid; e < SP2; e += kFT) {           // re-symmetrise the rounding
            const int a = e >> 6, b = e & 63;
            if (a < b) {
                const double m = 0.5 * (A[a * LD + b] + A[b * LD + a]);
                A[a * LD + b] = m;
                A[b * LD + a] = m;
            }
        }
        __syncthreads();
    }
    jac::sweeps<kFT>(A, E, js, kMaxSweeps);
    double* lam = f.lam + size_t(sl) * SP;
    double* U = f.U + size_t(sl) * SP2;
    double* V = f.V + size_t(sl) * SP2;
    if (tid < SP) lam[tid] = fmin(A[tid * LD + tid], 0.0);
    for (int e = tid; e < SP2; e += kFT) {
        const int a = e >> 6, b = e & 63;
        U[e] = f.isq[a] * E[a * LD + b];                  // U_pi[i = a][k = b]
        V[e] = E[b * LD + a] * f.sq[b];                   // V_pi[k = a][j = b]
    }
}

// ---------------------------------------------------------------- likelihoods
// A request evaluates one pattern with NC eigensystems mixed at the
// transition-matrix level, P_b = sum_c w_c U_c diag(e^{lambda_c a t_b}) V_c:
// NC = 1 for FEL (one omega), NC = 2 for MEME (the p1 / p+ components,
// meme.hpp:221-245).  The message of branch b is sum_c w_c U_c (e_c o (V_c L_b)).
struct FelReqs {
    const int* pattern;
    const double* a;      // time scale (the site's alpha)
    const int* slot;      // eigensystem of component 0
    const int* slot2;     // component 1 (NC = 2)
    const double* w1;     // weight of component 0 (NC = 2); component 1 gets 1 - w1
    const int* slot_bg;   // eigensystem of the background branches (BG)
};

template <int NC>
struct Spectral {
    double* U[NC];        // shared [64][LD]
    double* V[NC];
    double* part[NC];     // [4][64] quarter sums of a mat-vec
    double* x[NC];        // [64]
    double* lam[NC];      // [64] lambda * a
    double w[NC];
};

constexpr size_t spectral_doubles(int nc) { return size_t(nc) * (2 * SP * LD + 6 * SP); }
// EBF pass: two class eigensystems, plus the background's when NT = 3
constexpr size_t ebf_smem(int nt) { return (spectral_doubles(nt) + 3 * SP) * sizeof(double); }
static_assert(ebf_smem(3) + kMaxDepth * sizeof(int) + 16 * sizeof(double) <= 227 * 1024, "EBF pass must fit one CTA");

// carve shared memory and stage request r's eigensystems (NC = 3: the third is the
// background's, weight 1); returns the first free double
template <int NC>
__device__ double* spectral_setup(Spectral<NC>& sp, double* sm, const FelModel& f, const FelReqs& q, int r) {
    const int tid = threadIdx.x;
    double* z = sm;
    int sl[NC];
    sl[0] = q.slot[r];
    if constexpr (NC >= 2) {
        sl[1] = q.slot2[r];
        sp.w[0] = q.w1[r];
        sp.w[1] = 1.0 - q.w1[r];
    } else {
        sp.w[0] = 1.0;
    }
    if constexpr (NC == 3) {
        sl[2] = q.slot_bg[r];
        sp.w[2] = 1.0;
    }
    const double a = q.a[r];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        sp.U[c] = z; z += SP * LD;
        sp.V[c] = z; z += SP * LD;
        sp.part[c] = z; z += 4 * SP;
        sp.x[c] = z; z += SP;
        sp.lam[c] = z; z += SP;
        const double* gU = f.U + size_t(sl[c]) * SP2;
        const double* gV = f.V + size_t(sl[c]) * SP2;
        for (int e = tid; e < SP2; e += kFT) {
            const int i = e >> 6, j = e & 63;
            sp.U[c][i * LD + j] = gU[e];
            sp.V[c][i * LD + j] = gV[e];
        }
        if (tid < SP) sp.lam[c][tid] = f.lam[size_t(sl[c]) * SP + tid] * a;
    }
    return z;
}

// maximum over the 64 threads that own a state vector (named barrier 1)
__device__ __forceinline__ double max64(double v, double* r2) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) r2[threadIdx.x >> 5] = v;
    asm volatile("bar.sync 1, 64;" ::: "memory");
    const double m = fmax(r2[0], r2[1]);
    asm volatile("bar.sync 1, 64;" ::: "memory");
    return m;
}

// Depth-first pruning of pattern p (ev: 2 node + 1 opens an internal node,
// 2 node closes a node and sends its message to the parent's partial).  Open
// partials live on stk with power-of-two exponents in sexp.  NC = 2: every
// branch mixes the two class eigensystems; NC = 3: a branch flagged in bgf uses
// the third (background) one alone.  STORE: the two class messages of every
// non-root node are written to msg[node][c][64], the background message in
// both slots of a background branch (the outside pass of k_meme_ebf reads
// them).  On return stk[0..63] holds the root partial and sexp[0] its exponent.
template <int NC, bool STORE>
__device__ void prune(const Spectral<NC>& sp, double* sL, const Topo& t, const double* __restrict__ bl,
                      const uint8_t* __restrict__ bgf, const int* __restrict__ ev, int n_ev, double* stk, int* sexp,
                      double* red, int p, double* msg) {
    const int tid = threadIdx.x, S = t.S, row = tid & 63, qd = tid >> 6;
    int sp_ = -1;
    for (int k = 0; k < n_ev; ++k) {
        const int code = ev[k], node = code >> 1;
        if (code & 1) {                                    // open an internal node: partial = 1
            ++sp_;
            if (tid < SP) stk[sp_ * SP + tid] = tid < S ? 1.0 : 0.0;
            if (tid == 0) sexp[sp_] = 0;
            continue;
        }
        int Ev = 0;
        if (t.leaf[node]) {                                // x_c = V_c * leaf vector
            if (tid < SP) {
                const int tx = t.taxon[node];
                int st = -1;
                uint64_t mk = t.all_mask;
                if (tx >= 0) {
                    st = t.states[size_t(tx) * t.Pp + p];
                    if (st < 0) mk = t.masks[size_t(tx) * t.Pp + p];
                }
                const bool all = mk == 0 || (mk & t.all_mask) == t.all_mask;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    double s = 0.0;
                    if (st >= 0) {
                        s = sp.V[c][tid * LD + st];
                    } else {
                        for (int j = 0; j < S; ++j)
                            if (all || ((mk >> j) & 1)) s += sp.V[c][tid * LD + j];
                    }
                    sp.x[c][tid] = s;
                }
            }
        } else {                                           // x_c = V_c * L(node), pop it
            if (tid < SP) sL[tid] = stk[sp_ * SP + tid];
            __syncthreads();
            Ev = sexp[sp_];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                double s = 0.0;
#pragma unroll
                for (int j = 0; j < 16; ++j) s = fma(sp.V[c][row * LD + 16 * qd + j], sL[16 * qd + j], s);
                sp.part[c][qd * SP + row] = s;
            }
            __syncthreads();
            if (tid < SP) {
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    sp.x[c][tid] = (sp.part[c][tid] + sp.part[c][SP + tid]) + (sp.part[c][2 * SP + tid] + sp.part[c][3 * SP + tid]);
            }
            --sp_;
        }
        if (tid < SP) {
#pragma unroll
            for (int c = 0; c < NC; ++c) sp.x[c][tid] *= exp(sp.lam[c][tid] * bl[node]);
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < NC; ++c) {                     // U_c x_c
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 16; ++j) s = fma(sp.U[c][row * LD + 16 * qd + j], sp.x[c][16 * qd + j], s);
            sp.part[c][qd * SP + row] = s;
        }
        __syncthreads();
        if (tid < SP) {
            // the two warps that own the partial multiply, take its maximum between
            // themselves (named barrier 1, 64 threads) and rescale; the other warps go on
            const bool bgn = NC == 3 && bgf[node] != 0;
            double mc[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c)
                mc[c] = (sp.part[c][tid] + sp.part[c][SP + tid]) + (sp.part[c][2 * SP + tid] + sp.part[c][3 * SP + tid]);
            double m = 0.0;
#pragma unroll
            for (int c = 0; c < (NC == 3 ? 2 : NC); ++c) {
                m += sp.w[c] * mc[c];
                if constexpr (STORE) msg[(size_t(node) * 3 + c) * SP + tid] = tid < S ? fmax(bgn ? mc[NC - 1] : mc[c], 0.0) : 0.0;
            }
            if (bgn) m = mc[NC - 1];
            m = tid < S ? fmax(m, 0.0) : 0.0;
            double v = stk[sp_ * SP + tid] * m;
            double w = v;
            for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_xor_sync(0xffffffffu, w, o));
            if ((tid & 31) == 0) red[tid >> 5] = w;
            asm volatile("bar.sync 1, 64;" ::: "memory");
            const double mx = fmax(red[0], red[1]);
            if (mx > 0.0 && mx < 0x1p-256) {
                v *= 0x1p256;
                if (tid == 0) sexp[sp_] += 256;
            }
            stk[sp_ * SP + tid] = v;
            if (tid == 0) sexp[sp_] += Ev;
        }
    }
    __syncthreads();
}

// Level-synchronous pruning, one warp per node: the log-likelihood of each
// request, or the reference's -1e20 for L <= 0.  Nodes are grouped by height
// (leaves first, the root last); the nodes of one level are independent, so
// the warps of a CTA take them in parallel and the chain of dependent steps
// is the tree's height instead of its node count.  Lane l owns states l and
// l + 32.  A node's message sum_c w_c U_c (e_c o (V_c D)) goes to the CTA's
// workspace row; its partial D is the product of its children's rows,
// rescaled by 2^256 whenever its maximum falls below 2^-256 (exponents summed
// over the tree).  With BG, a branch flagged in f.bg uses the request's
// background eigensystem alone (weight 1) instead of the NC tested ones.
// Persistent: CTA b evaluates requests b, b + grid, ...
struct LevelPlan {
    int H;                    // levels: 0 = leaves ... H - 1 = the root alone
    const int* off;           // [H + 1]
    const int* nodes;         // [n] nodes ordered by level
};

constexpr int kLvT = 512;
constexpr int kLvW = kLvT / 32;

// nc tested components, plus the background's eigensystem when bg
constexpr size_t lv_smem(int nc, bool bg) {
    return (size_t(nc + (bg ? 1 : 0)) * (2 * SP * LD + SP) + size_t(kLvW) * (nc + 1) * SP) * sizeof(double);
}
static_assert(lv_smem(2, true) <= 227 * 1024, "three eigensystems must fit one CTA");

__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int NC, bool BG>
__global__ void __launch_bounds__(kLvT) k_site_lnl(FelModel f, Topo t, const double* __restrict__ bl, LevelPlan lp,
                                                   double* __restrict__ work, FelReqs q, int n_req, double* __restrict__ out) {
    constexpr int NT = NC + (BG ? 1 : 0);                 // eigensystems per request; the last is the background's
    pdl_enter();
    extern __shared__ __align__(16) double sm[];
    __shared__ int sE;
    __shared__ double sL;
    double* U[NT];
    double* V[NT];
    double* lam[NT];
    double* z = sm;
#pragma unroll
    for (int c = 0; c < NT; ++c) {
        U[c] = z; z += SP * LD;
        V[c] = z; z += SP * LD;
        lam[c] = z; z += SP;
    }
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, S = t.S;
    double* dv = z + size_t(warp) * (NC + 1) * SP;        // this warp's partial
    double* xv = dv + SP;                                  // [NC][64] spectral coordinates
    double* msg = work + size_t(blockIdx.x) * t.n * SP;
    const int s0 = lane, s1 = lane + 32;
    for (int r = blockIdx.x; r < n_req; r += gridDim.x) {
        int sl[NT];
        double w[NC];
        sl[0] = q.slot[r];
        if constexpr (NC == 2) {
            sl[1] = q.slot2[r];
            w[0] = q.w1[r];
            w[1] = 1.0 - q.w1[r];
        } else {
            w[0] = 1.0;
        }
        if constexpr (BG) sl[NT - 1] = q.slot_bg[r];
        const double a = q.a[r];
        const int p = q.pattern[r];
        __syncthreads();                                   // the previous request is done with shared memory
#pragma unroll
        for (int c = 0; c < NT; ++c) {
            const double* gU = f.U + size_t(sl[c]) * SP2;
            const double* gV = f.V + size_t(sl[c]) * SP2;
            for (int e = tid; e < SP2; e += kLvT) {
                const int i = e >> 6, j = e & 63;
                U[c][i * LD + j] = gU[e];
                V[c][i * LD + j] = gV[e];
            }
            if (tid < SP) lam[c][tid] = f.lam[size_t(sl[c]) * SP + tid] * a;
        }
        if (tid == 0) { sE = 0; sL = 0.0; }
        __syncthreads();
        for (int h = 0; h < lp.H; ++h) {
            const int b1 = lp.off[h + 1];
            for (int i = lp.off[h] + warp; i < b1; i += kLvW) {
                const int u = lp.nodes[i];
                // the branch above u: the tested components, or the background one alone
                const bool bgn = BG && f.bg[u] != 0;
                const int ncu = bgn ? 1 : NC;
                double x[NC][2];
                if (t.leaf[u]) {                           // x_c = V_c * leaf vector
                    const int tx = t.taxon[u];
                    int st = -1;
                    uint64_t mk = t.all_mask;
                    if (tx >= 0) {
                        st = t.states[size_t(tx) * t.Pp + p];
                        if (st < 0) mk = t.masks[size_t(tx) * t.Pp + p];
                    }
                    const bool all = mk == 0 || (mk & t.all_mask) == t.all_mask;
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        if (c >= ncu) break;
                        const double* Vc = bgn ? V[NT - 1] : V[c];
                        double a0 = 0.0, a1 = 0.0;
                        if (st >= 0) {
                            a0 = Vc[s0 * LD + st];
                            a1 = Vc[s1 * LD + st];
                        } else {
                            for (int j = 0; j < S; ++j)
                                if (all || ((mk >> j) & 1)) { a0 += Vc[s0 * LD + j]; a1 += Vc[s1 * LD + j]; }
                        }
                        x[c][0] = a0;
                        x[c][1] = a1;
                    }
                } else {                                   // D = product of the children's messages
                    double d0 = s0 < S ? 1.0 : 0.0, d1 = s1 < S ? 1.0 : 0.0;
                    int E = 0;
                    const int e1 = t.ch_off[u + 1];
                    for (int e = t.ch_off[u]; e < e1; ++e) {
                        const double* mc = msg + size_t(t.ch[e]) * SP;
                        d0 *= mc[s0];
                        d1 *= mc[s1];
                        const double mx = warp_max(fmax(d0, d1));
                        if (mx > 0.0 && mx < 0x1p-256) {
                            d0 *= 0x1p256;
                            d1 *= 0x1p256;
                            E += 256;
                        }
                    }
                    if (lane == 0 && E) atomicAdd(&sE, E);
                    if (u == t.root) {                     // L = pi . D
                        const double v = warp_sum((s0 < S ? f.pi[s0] * d0 : 0.0) + (s1 < S ? f.pi[s1] * d1 : 0.0));
                        if (lane == 0) sL = v;
                        continue;
                    }
                    dv[s0] = d0;
                    dv[s1] = d1;
                    __syncwarp();
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        if (c >= ncu) break;
                        const double* Vc = bgn ? V[NT - 1] : V[c];
                        double a0 = 0.0, a1 = 0.0;
                        const double* v0 = Vc + s0 * LD;
                        const double* v1 = Vc + s1 * LD;
#pragma unroll 16
                        for (int j = 0; j < SP; ++j) {
                            const double dj = dv[j];
                            a0 = fma(v0[j], dj, a0);
                            a1 = fma(v1[j], dj, a1);
                        }
                        x[c][0] = a0;
                        x[c][1] = a1;
                    }
                }
                const double tb = bl[u];
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if (c >= ncu) break;
                    const double* lc = bgn ? lam[NT - 1] : lam[c];
                    xv[c * SP + s0] = x[c][0] * exp(lc[s0] * tb);
                    xv[c * SP + s1] = x[c][1] * exp(lc[s1] * tb);
                }
                __syncwarp();
                double m0 = 0.0, m1 = 0.0;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if (c >= ncu) break;
                    double a0 = 0.0, a1 = 0.0;
                    const double* u0 = (bgn ? U[NT - 1] : U[c]) + s0 * LD;
                    const double* u1 = (bgn ? U[NT - 1] : U[c]) + s1 * LD;
                    const double* xc = xv + c * SP;
#pragma unroll 16
                    for (int j = 0; j < SP; ++j) {
                        const double xj = xc[j];
                        a0 = fma(u0[j], xj, a0);
                        a1 = fma(u1[j], xj, a1);
                    }
                    const double wc = bgn ? 1.0 : w[c];
                    m0 += wc * a0;
                    m1 += wc * a1;
                }
                __syncwarp();                              // dv / xv are reused by this warp's next node
                msg[size_t(u) * SP + s0] = s0 < S ? fmax(m0, 0.0) : 0.0;
                msg[size_t(u) * SP + s1] = s1 < S ? fmax(m1, 0.0) : 0.0;
            }
            __syncthreads();                               // this level's messages are visible to the next
        }
        if (tid == 0) out[r] = sL > 0.0 ? log(sL) - double(sE) * 0.69314718055994530942 : -1e20;
    }
}

// grid n_req, block 256: MEME's empirical Bayes factors (meme.hpp:484-588).  For
// every branch b the reference re-prunes the pattern twice, with b alone in
// class 1 and alone in class +; the likelihood is linear in b's message, so
// both follow from one inside-outside pass: L_c(b) = top_b . M_c(b), where
// top_b = O_parent o (product of b's siblings' messages) and O is the outside
// vector (pi at the root, P_mix^T top below).  Every vector may carry any
// positive factor common to both classes, so the outside pass normalises by
// the maximum instead of tracking exponents.  ebf[r][b] for every non-root b.
// NT = 3: background branches (f.bg) use the request's background
// eigensystem alone and get ebf 1 (meme.hpp:497-552).
template <int NT>
__global__ void __launch_bounds__(kFT) k_meme_ebf(FelModel f, Topo t, const double* __restrict__ bl, const int* __restrict__ ev,
                                                  int n_ev, int depth, double* __restrict__ stack, FelReqs q,
                                                  double* __restrict__ msg_all, double* __restrict__ ebf_all) {
    pdl_enter();
    extern __shared__ __align__(16) double sm[];
    __shared__ int sexp[kMaxDepth];
    __shared__ double red[kFT / 32], r2[2], r4[4];
    const int tid = threadIdx.x, S = t.S, r = blockIdx.x, n = t.n, row = tid & 63, qd = tid >> 6;
    Spectral<NT> sp;
    double* sL = spectral_setup<NT>(sp, sm, f, q, r);
    double* ou = sL + SP;                                  // outside vector of the open node
    double* top = ou + SP;
    double* stk = stack + size_t(r) * depth * SP;
    double* msg = msg_all + size_t(r) * n * 3 * SP;        // [node][M_1 | M_+ | O or prefix][64]
    double* ebf = ebf_all + size_t(r) * n;
    __syncthreads();
    prune<NT, true>(sp, sL, t, bl, f.bg, ev, n_ev, stk, sexp, red, q.pattern[r], msg);
    const double w0 = sp.w[0], w1 = sp.w[1];
    if (tid == 0) ebf[t.root] = 1.0;
    for (int k = 0; k < n_ev; ++k) {                       // internal nodes in pre-order
        const int code = ev[k];
        if (!(code & 1)) continue;
        const int u = code >> 1;
        if (tid < SP) ou[tid] = tid >= S ? 0.0 : (u == t.root ? f.pi[tid] : msg[(size_t(u) * 3 + 2) * SP + tid]);
        const int c0 = t.ch_off[u], c1 = t.ch_off[u + 1];
        if (tid < SP) {                                    // prefix products into each child's third slot
            double acc = ou[tid];
            for (int i = c0; i < c1; ++i) {
                const size_t b = size_t(t.ch[i]) * 3 * SP;
                msg[b + 2 * SP + tid] = acc;
                acc *= w0 * msg[b + tid] + w1 * msg[b + SP + tid];
                const double mx = max64(acc, r2);
                if (mx > 0.0) acc /= mx;
            }
        }
        __syncthreads();
        double suf = tid < S ? 1.0 : 0.0;
        for (int i = c1 - 1; i >= c0; --i) {               // suffix products, children in reverse
            const int c = t.ch[i];
            const size_t b = size_t(c) * 3 * SP;
            const bool bgc = NT == 3 && f.bg[c] != 0;
            if (tid < SP) {
                double tv = msg[b + 2 * SP + tid] * suf;
                const double mx = max64(tv, r2);
                if (mx > 0.0) tv /= mx;
                top[tid] = tv;
                double s1 = tv * msg[b + tid], s2 = tv * msg[b + SP + tid];
                for (int o = 16; o > 0; o >>= 1) {
                    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                }
                if ((tid & 31) == 0) { r4[2 * (tid >> 5)] = s1; r4[2 * (tid >> 5) + 1] = s2; }
                asm volatile("bar.sync 1, 64;" ::: "memory");
                if (tid == 0) {
                    const double L1 = r4[0] + r4[2], Lp = r4[1] + r4[3];
                    double e = 0.0;
                    if (L1 > 0.0 && Lp > 0.0) e = exp(fmin(fmax(log(Lp) - log(L1), -50.0), 50.0));
                    else if (!(L1 > 0.0) && Lp > 0.0) e = 1e6;
                    ebf[c] = bgc ? 1.0 : e;
                }
                suf *= w0 * msg[b + tid] + w1 * msg[b + SP + tid];
                const double ms = max64(suf, r2);
                if (ms > 0.0) suf /= ms;
            }
            __syncthreads();
            if (!t.leaf[c]) {                              // O_c = sum_k w_k V_k^T (e_k o (U_k^T top))
#pragma unroll
                for (int m = 0; m < NT; ++m) {
                    double s = 0.0;
#pragma unroll
                    for (int j = 0; j < 16; ++j) s = fma(sp.U[m][(16 * qd + j) * LD + row], top[16 * qd + j], s);
                    sp.part[m][qd * SP + row] = s;
                }
                __syncthreads();
                if (tid < SP) {
#pragma unroll
                    for (int m = 0; m < NT; ++m)
                        sp.x[m][tid] = ((sp.part[m][tid] + sp.part[m][SP + tid]) + (sp.part[m][2 * SP + tid] + sp.part[m][3 * SP + tid])) *
                                       exp(sp.lam[m][tid] * bl[c]);
                }
                __syncthreads();
#pragma unroll
                for (int m = 0; m < NT; ++m) {
                    double s = 0.0;
#pragma unroll
                    for (int j = 0; j < 16; ++j) s = fma(sp.V[m][(16 * qd + j) * LD + row], sp.x[m][16 * qd + j], s);
                    sp.part[m][qd * SP + row] = s;
                }
                __syncthreads();
                if (tid < SP) {
                    double o = 0.0;
#pragma unroll
                    for (int m = 0; m < 2; ++m)
                        o += sp.w[m] * ((sp.part[m][tid] + sp.part[m][SP + tid]) + (sp.part[m][2 * SP + tid] + sp.part[m][3 * SP + tid]));
                    if (bgc) {
                        const int m = NT - 1;
                        o = (sp.part[m][tid] + sp.part[m][SP + tid]) + (sp.part[m][2 * SP + tid] + sp.part[m][3 * SP + tid]);
                    }
                    msg[b + 2 * SP + tid] = tid < S ? fmax(o, 0.0) : 0.0;
                }
                __syncthreads();
            }
        }
    }
}

}  // namespace

struct FelDevice {
    h3g_problem* pr = nullptr;
    cudaStream_t s = nullptr;
    int S = 0, n = 0, n_ev = 0, depth = 1, max_req = 0, n_slots = 0;
    Topo t{};
    FelModel f{};
    double* d_bl = nullptr;
    uint8_t* d_bg = nullptr;              // [n] background flags of the run
    int* d_ev = nullptr;
    double* d_stack = nullptr;            // EBF pass: [kEbfChunk][depth][64] open partials
    int* d_lv = nullptr;                  // level plan: [H + 1] offsets, then [n] nodes
    int H = 0;
    double* d_work = nullptr;             // level-synchronous pruning: [grid][n][64] messages
    int grid[2][2] = {{1, 1}, {1, 1}};    // persistent CTAs per [tested components - 1][background]
    unsigned char* d_req = nullptr;       // per batch: [om | a | w1 | eslot | eprev | pat | slot | slot2 | slot_bg], packed to the batch's sizes
    unsigned char* h_req = nullptr;       // pinned mirror
    double* d_out = nullptr;
    double* h_out = nullptr;
    double* d_msg = nullptr;              // EBF pass: [kEbfChunk][n][3][64], allocated on first use
    double* d_ebf = nullptr;              // [kEbfChunk][n]
    double* h_ebf = nullptr;
    size_t h2d = 0, d2h = 0;              // bytes moved by the batches so far
    int launches = 0;                     // kernels launched so far
    std::vector<void*> owned;
    std::vector<uint8_t> bg_host;
    std::vector<int> order;               // requests grouped by kernel: (1, -), (2, -), (1, bg), (2, bg)
    ~FelDevice() {
        for (void* p : owned) cudaFree(p);
        if (h_req) cudaFreeHost(h_req);
        if (h_out) cudaFreeHost(h_out);
        if (h_ebf) cudaFreeHost(h_ebf);
    }
    // a batch holds up to max_req requests and three eigensolves per request
    size_t req_bytes() const { return 5 * size_t(max_req) * sizeof(double) + 10 * size_t(max_req) * sizeof(int); }
};

constexpr int kEbfChunk = 256;

namespace {

// Buffers that depend on the problem (traversals, levels) and on the run's sizes
// (requests per batch, eigensystem slots), not on the model.
FelDevice* fel_device_alloc(h3g_problem* pr, const FelProblemView& v, int max_requests, int n_slots, std::string* err) {
    auto* d = new (std::nothrow) FelDevice;
    if (!d) { *err = "host allocation failed"; return nullptr; }
    d->pr = pr;
    d->s = problem_stream(pr);
    d->n = v.n;
    d->max_req = std::max(1, max_requests);
    d->n_slots = std::max(1, n_slots);
    // depth-first events in the children CSR order
    std::vector<int> ev;
    ev.reserve(2 * size_t(v.n));
    int open = 0, deepest = 1;
    std::vector<std::pair<int, int>> stk{{v.root, 0}};
    ev.push_back(2 * v.root + 1);
    open = 1;
    while (!stk.empty()) {
        auto& [u, k] = stk.back();
        if (k < v.ch_off[u + 1] - v.ch_off[u]) {
            const int c = v.ch[v.ch_off[u] + k++];
            if (v.leaf[c]) {
                ev.push_back(2 * c);
            } else {
                ev.push_back(2 * c + 1);
                deepest = std::max(deepest, ++open);
                stk.push_back({c, 0});
            }
        } else {
            if (u != v.root) { ev.push_back(2 * u); --open; }
            stk.pop_back();
        }
    }
    if (deepest > kMaxDepth) { *err = "tree deeper than 1024 internal levels"; delete d; return nullptr; }
    d->n_ev = int(ev.size());
    d->depth = deepest;
    // levels by height: a node's children all sit on lower levels; the root alone on the top one
    std::vector<int> height(v.n, 0);
    for (int e : ev) {                    // a node closes after all of its descendants
        if (e & 1) continue;
        const int u = e >> 1;
        for (int c = v.ch_off[u]; c < v.ch_off[u + 1]; ++c) height[u] = std::max(height[u], height[v.ch[c]] + 1);
    }
    for (int c = v.ch_off[v.root]; c < v.ch_off[v.root + 1]; ++c) height[v.root] = std::max(height[v.root], height[v.ch[c]] + 1);
    d->H = height[v.root] + 1;
    std::vector<int> lv(size_t(d->H) + 1 + v.n, 0);
    for (int u = 0; u < v.n; ++u) ++lv[size_t(height[u]) + 1];
    for (int h = 0; h < d->H; ++h) lv[size_t(h) + 1] += lv[size_t(h)];
    {
        std::vector<int> fill(lv.begin(), lv.begin() + d->H);
        for (int u = 0; u < v.n; ++u) lv[size_t(d->H) + 1 + size_t(fill[size_t(height[u])]++)] = u;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, v.device);
    auto take = [&](auto** ptr, size_t count) -> bool {
        void* q = nullptr;
        if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(**ptr)) != cudaSuccess) return false;
        d->owned.push_back(q);
        *ptr = static_cast<std::remove_reference_t<decltype(*ptr)>>(q);
        return true;
    };
    double *qs = nullptr, *qn = nullptr, *dsq = nullptr, *disq = nullptr, *dpi = nullptr;
    bool ok = take(&qs, SP2) && take(&qn, SP2) && take(&dsq, SP) && take(&disq, SP) && take(&dpi, SP) &&
              take(&d->f.lam, size_t(d->n_slots) * SP) && take(&d->f.U, size_t(d->n_slots) * SP2) &&
              take(&d->f.V, size_t(d->n_slots) * SP2) && take(&d->d_bl, v.n) && take(&d->d_bg, v.n) &&
              take(&d->d_ev, ev.size()) &&
              take(&d->d_stack, size_t(kEbfChunk) * d->depth * SP) && take(&d->d_out, d->max_req) &&
              take(&d->d_lv, lv.size()) && take(&d->d_work, size_t(2) * std::max(sms, 1) * v.n * SP);
    void* rq = nullptr;
    ok = ok && cudaMalloc(&rq, d->req_bytes()) == cudaSuccess;
    if (rq) d->owned.push_back(rq);
    d->d_req = static_cast<unsigned char*>(rq);
    ok = ok && cudaMallocHost(reinterpret_cast<void**>(&d->h_req), d->req_bytes()) == cudaSuccess &&
         cudaMallocHost(reinterpret_cast<void**>(&d->h_out), d->max_req * sizeof(double)) == cudaSuccess;
    if (!ok) { *err = "device allocation failed"; delete d; return nullptr; }
    d->f.Qs = qs; d->f.Qn = qn; d->f.sq = dsq; d->f.isq = disq; d->f.pi = dpi; d->f.bg = d->d_bg;
    ok = cudaMemcpyAsync(d->d_ev, ev.data(), ev.size() * sizeof(int), cudaMemcpyHostToDevice, d->s) == cudaSuccess &&
         cudaMemcpyAsync(d->d_lv, lv.data(), lv.size() * sizeof(int), cudaMemcpyHostToDevice, d->s) == cudaSuccess &&
         cudaStreamSynchronize(d->s) == cudaSuccess;
    static bool configured = false;
    if (ok && !configured) {
        ok = cudaFuncSetAttribute(k_fel_eig, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kEigSmem)) == cudaSuccess &&
             cudaFuncSetAttribute(k_site_lnl<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(lv_smem(1, false))) == cudaSuccess &&
             cudaFuncSetAttribute(k_site_lnl<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(lv_smem(2, false))) == cudaSuccess &&
             cudaFuncSetAttribute(k_site_lnl<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(lv_smem(1, true))) == cudaSuccess &&
             cudaFuncSetAttribute(k_site_lnl<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(lv_smem(2, true))) == cudaSuccess &&
             cudaFuncSetAttribute(k_meme_ebf<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ebf_smem(2))) == cudaSuccess &&
             cudaFuncSetAttribute(k_meme_ebf<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ebf_smem(3))) == cudaSuccess;
        configured = ok;
    }
    int per[2][2] = {{0, 0}, {0, 0}};
    ok = ok && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[0][0], k_site_lnl<1, false>, kLvT, lv_smem(1, false)) == cudaSuccess &&
         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[1][0], k_site_lnl<2, false>, kLvT, lv_smem(2, false)) == cudaSuccess &&
         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[0][1], k_site_lnl<1, true>, kLvT, lv_smem(1, true)) == cudaSuccess &&
         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[1][1], k_site_lnl<2, true>, kLvT, lv_smem(2, true)) == cudaSuccess;
    if (!ok) { *err = std::string("FEL set-up: ") + cudaGetErrorString(cudaGetLastError()); delete d; return nullptr; }
    for (int c = 0; c < 2; ++c)
        for (int b = 0; b < 2; ++b)       // the workspace holds 2 x SMs CTAs
            d->grid[c][b] = std::max(1, std::min(per[c][b], 2) * std::max(sms, 1));
    return d;
}

}  // namespace

FelDevice* fel_device_create(h3g_problem* pr, int S, const double* pi, const double* Qs, const double* Qn,
                             const double* branch_lengths, const uint8_t* background, int max_requests, int n_slots,
                             std::string* err) {
    FelProblemView v;
    if (!fel_problem_view(pr, &v) || S < 1 || S > SP) { *err = "invalid problem"; return nullptr; }
    FelDevice*& cached = problem_fel_device(pr);
    if (cached && (cached->max_req < max_requests || cached->n_slots < n_slots)) {
        fel_device_free(cached);
        cached = nullptr;
    }
    if (!cached) cached = fel_device_alloc(pr, v, max_requests, n_slots, err);
    FelDevice* d = cached;
    if (!d) return nullptr;
    // the run's model: rates, frequencies, branch lengths
    d->S = S;
    d->f.S = S;
    d->t = problem_topo(pr, S);
    d->h2d = d->d2h = 0;
    d->launches = 0;
    std::vector<double> sq(SP, 0.0), isq(SP, 0.0), pp(SP, 0.0);
    for (int i = 0; i < S; ++i) {
        sq[i] = std::sqrt(std::max(pi[i], 1e-12));
        isq[i] = 1.0 / sq[i];
        pp[i] = pi[i];
    }
    d->bg_host.assign(size_t(v.n), 0);
    if (background)
        for (int i = 0; i < v.n; ++i) d->bg_host[size_t(i)] = i != v.root && background[i] ? 1 : 0;
    cudaStream_t s = d->s;
    const bool ok =
        cudaMemcpyAsync(d->d_bg, d->bg_host.data(), size_t(v.n), cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(const_cast<double*>(d->f.Qs), Qs, size_t(S) * S * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(const_cast<double*>(d->f.Qn), Qn, size_t(S) * S * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(const_cast<double*>(d->f.sq), sq.data(), SP * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(const_cast<double*>(d->f.isq), isq.data(), SP * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(const_cast<double*>(d->f.pi), pp.data(), SP * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(d->d_bl, branch_lengths, v.n * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) {
        *err = std::string("FEL set-up: ") + cudaGetErrorString(cudaGetLastError());
        fel_device_free(d);
        cached = nullptr;
        return nullptr;
    }
    return d;
}

namespace {

// Validate a batch, pack it into one host-to-device copy in `order` and launch
// the eigensolves.  Returns the request views (in packed order) through q.
bool stage_batch(FelDevice* d, int n_eig, const double* eig_omega, const int* eig_slot, const int* eig_prev, int n_req,
                 const int* req_pattern, const double* req_a, const int* req_slot, const int* req_slot2, const double* req_w1,
                 const int* req_slot_bg, const std::vector<int>& order, FelReqs* q, std::string* err) {
    if (n_eig > 3 * d->max_req || n_req > d->max_req || n_eig < 0 || n_req < 0) { *err = "FEL batch too large"; return false; }
    for (int i = 0; i < n_eig; ++i)
        if (eig_slot[i] < 0 || eig_slot[i] >= d->n_slots || eig_prev[i] < -1 || eig_prev[i] >= d->n_slots) {
            *err = "FEL eigensystem slot out of range";
            return false;
        }
    for (int i = 0; i < n_req; ++i) {
        const bool mix = req_slot2 && req_slot2[i] >= 0;
        if (req_slot[i] < 0 || req_slot[i] >= d->n_slots || req_pattern[i] < 0 || req_pattern[i] >= d->t.P ||
            (mix && req_slot2[i] >= d->n_slots) || (req_slot_bg && req_slot_bg[i] >= d->n_slots) || !(req_a[i] > 0.0) ||
            (req_w1 && !(req_w1[i] >= 0.0 && req_w1[i] <= 1.0))) {
            *err = "FEL request out of range";
            return false;
        }
    }
    const size_t o_a = size_t(n_eig) * sizeof(double), o_w = o_a + size_t(n_req) * sizeof(double);
    const size_t o_es = o_w + size_t(n_req) * sizeof(double), o_pv = o_es + size_t(n_eig) * sizeof(int);
    const size_t o_pat = o_pv + size_t(n_eig) * sizeof(int), o_sl = o_pat + size_t(n_req) * sizeof(int);
    const size_t o_s2 = o_sl + size_t(n_req) * sizeof(int), o_sb = o_s2 + size_t(n_req) * sizeof(int);
    const size_t bytes = o_sb + size_t(n_req) * sizeof(int);
    unsigned char* h = d->h_req;
    std::copy(eig_omega, eig_omega + n_eig, reinterpret_cast<double*>(h));
    std::copy(eig_slot, eig_slot + n_eig, reinterpret_cast<int*>(h + o_es));
    std::copy(eig_prev, eig_prev + n_eig, reinterpret_cast<int*>(h + o_pv));
    for (int k = 0; k < n_req; ++k) {
        const int i = order[k];
        reinterpret_cast<double*>(h + o_a)[k] = req_a[i];
        reinterpret_cast<double*>(h + o_w)[k] = req_w1 ? req_w1[i] : 1.0;
        reinterpret_cast<int*>(h + o_pat)[k] = req_pattern[i];
        reinterpret_cast<int*>(h + o_sl)[k] = req_slot[i];
        reinterpret_cast<int*>(h + o_s2)[k] = req_slot2 ? req_slot2[i] : -1;
        reinterpret_cast<int*>(h + o_sb)[k] = req_slot_bg ? req_slot_bg[i] : -1;
    }
    cudaStream_t s = d->s;
    if (cudaMemcpyAsync(d->d_req, h, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) {
        *err = std::string("FEL batch copy: ") + cudaGetErrorString(cudaGetLastError());
        return false;
    }
    d->h2d += bytes;
    unsigned char* g = d->d_req;
    if (n_eig > 0) {
        launch_k(k_fel_eig, n_eig, kFT, kEigSmem, s, d->f, reinterpret_cast<const double*>(g),
                 reinterpret_cast<const int*>(g + o_es), reinterpret_cast<const int*>(g + o_pv));
        ++d->launches;
    }
    *q = FelReqs{reinterpret_cast<const int*>(g + o_pat), reinterpret_cast<const double*>(g + o_a),
                 reinterpret_cast<const int*>(g + o_sl), reinterpret_cast<const int*>(g + o_s2),
                 reinterpret_cast<const double*>(g + o_w), reinterpret_cast<const int*>(g + o_sb)};
    return true;
}

FelReqs offset(const FelReqs& q, int k) {
    return FelReqs{q.pattern + k, q.a + k, q.slot + k, q.slot2 + k, q.w1 + k, q.slot_bg + k};
}

}  // namespace

bool fel_device_eval(FelDevice* d, int n_eig, const double* eig_omega, const int* eig_slot, const int* eig_prev, int n_req,
                     const int* req_pattern, const double* req_a, const int* req_slot, const int* req_slot2,
                     const double* req_w1, const int* req_slot_bg, double* lnl_out, std::string* err) {
    if (n_req == 0 && n_eig == 0) return true;
    // group the requests by kernel: tested components (1 or 2) x background eigensystem (no / yes)
    auto& order = d->order;
    order.clear();
    int start[5] = {0, 0, 0, 0, 0};
    for (int g = 0; g < 4; ++g) {
        const bool two = g & 1, bg = g >> 1;
        for (int i = 0; i < n_req; ++i)
            if ((req_slot2 && req_slot2[i] >= 0) == two && (req_slot_bg && req_slot_bg[i] >= 0) == bg) order.push_back(i);
        start[g + 1] = int(order.size());
    }
    FelReqs q{};
    if (!stage_batch(d, n_eig, eig_omega, eig_slot, eig_prev, n_req, req_pattern, req_a, req_slot, req_slot2, req_w1,
                     req_slot_bg, order, &q, err))
        return false;
    cudaStream_t s = d->s;
    const LevelPlan lp{d->H, d->d_lv, d->d_lv + d->H + 1};
    const double* bl = d->d_bl;
    for (int g = 0; g < 4; ++g) {
        const int k0 = start[g], cnt = start[g + 1] - start[g];
        if (cnt == 0) continue;
        const FelReqs qg = offset(q, k0);
        double* o = d->d_out + k0;
        const int grid = std::min(cnt, d->grid[g & 1][g >> 1]);
        switch (g) {
            case 0: launch_k(k_site_lnl<1, false>, grid, kLvT, lv_smem(1, false), s, d->f, d->t, bl, lp, d->d_work, qg, cnt, o); break;
            case 1: launch_k(k_site_lnl<2, false>, grid, kLvT, lv_smem(2, false), s, d->f, d->t, bl, lp, d->d_work, qg, cnt, o); break;
            case 2: launch_k(k_site_lnl<1, true>, grid, kLvT, lv_smem(1, true), s, d->f, d->t, bl, lp, d->d_work, qg, cnt, o); break;
            default: launch_k(k_site_lnl<2, true>, grid, kLvT, lv_smem(2, true), s, d->f, d->t, bl, lp, d->d_work, qg, cnt, o); break;
        }
        ++d->launches;
    }
    d->d2h += size_t(n_req) * sizeof(double);
    const bool ok = cudaGetLastError() == cudaSuccess &&
                    (n_req == 0 || cudaMemcpyAsync(d->h_out, d->d_out, n_req * sizeof(double), cudaMemcpyDeviceToHost, s) == cudaSuccess) &&
                    cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) { *err = std::string("FEL batch: ") + cudaGetErrorString(cudaGetLastError()); return false; }
    for (int k = 0; k < n_req; ++k) lnl_out[order[k]] = d->h_out[k];
    return true;
}

bool fel_device_ebf(FelDevice* d, int n_eig, const double* eig_omega, const int* eig_slot, const int* eig_prev, int n_req,
                    const int* req_pattern, const double* req_a, const int* req_slot, const int* req_slot2,
                    const double* req_w1, const int* req_slot_bg, double* ebf_out, std::string* err) {
    if (n_req > kEbfChunk) { *err = "EBF batch larger than 256 requests"; return false; }
    for (int i = 0; i < n_req; ++i)
        if (req_slot2[i] < 0 || (req_slot_bg && req_slot_bg[i] < 0)) {
            *err = "EBF request needs two components (and the background's when one is given)";
            return false;
        }
    if (!d->d_msg) {
        void *m = nullptr, *e = nullptr;
        bool ok = cudaMalloc(&m, size_t(kEbfChunk) * d->n * 3 * SP * sizeof(double)) == cudaSuccess;
        if (m) d->owned.push_back(m);
        ok = ok && cudaMalloc(&e, size_t(kEbfChunk) * d->n * sizeof(double)) == cudaSuccess;
        if (e) d->owned.push_back(e);
        ok = ok && cudaMallocHost(reinterpret_cast<void**>(&d->h_ebf), size_t(kEbfChunk) * d->n * sizeof(double)) == cudaSuccess;
        if (!ok) { *err = "EBF scratch allocation failed"; return false; }
        d->d_msg = static_cast<double*>(m);
        d->d_ebf = static_cast<double*>(e);
    }
    auto& order = d->order;
    order.resize(n_req);
    for (int i = 0; i < n_req; ++i) order[i] = i;
    FelReqs q{};
    if (!stage_batch(d, n_eig, eig_omega, eig_slot, eig_prev, n_req, req_pattern, req_a, req_slot, req_slot2, req_w1,
                     req_slot_bg, order, &q, err))
        return false;
    cudaStream_t s = d->s;
    const size_t bytes = size_t(n_req) * d->n * sizeof(double);
    d->launches += n_req > 0;
    if (n_req > 0)
        launch_k(req_slot_bg ? k_meme_ebf<3> : k_meme_ebf<2>, n_req, kFT, ebf_smem(req_slot_bg ? 3 : 2), s, d->f, d->t,
                 static_cast<const double*>(d->d_bl), static_cast<const int*>(d->d_ev), d->n_ev, d->depth, d->d_stack, q,
                 d->d_msg, d->d_ebf);
    d->d2h += bytes;
    const bool ok = cudaGetLastError() == cudaSuccess &&
                    (n_req == 0 || cudaMemcpyAsync(d->h_ebf, d->d_ebf, bytes, cudaMemcpyDeviceToHost, s) == cudaSuccess) &&
                    cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) { *err = std::string("EBF batch: ") + cudaGetErrorString(cudaGetLastError()); return false; }
    std::copy(d->h_ebf, d->h_ebf + size_t(n_req) * d->n, ebf_out);
    return true;
}

int fel_device_max_ebf(const FelDevice* d) { return std::min(kEbfChunk, d->max_req); }

void fel_device_transfer(const FelDevice* d, size_t* h2d, size_t* d2h, int* launches) {
    *h2d = d->h2d;
    *d2h = d->d2h;
    *launches = d->launches;
}

void fel_device_destroy(FelDevice* d) {
    if (d && d->s) cudaStreamSynchronize(d->s);
}

void fel_device_free(FelDevice* d) {
    if (d && d->s) cudaStreamSynchronize(d->s);
    delete d;
}

}  // namespace h3g
