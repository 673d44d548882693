// h3g_common.cuh — device-side layout shared by the FP64 and mixed-precision paths.
//
// HBM layout (one problem = one tree x one compressed alignment):
//   states / masks     [T][Pp]              leaf observations, taxon-major so a
//                                           pattern tile of one taxon is contiguous
//   P, PT, dP          [M][n][64*64]        per rate class and branch, 61 states
//                                           zero-padded to 64 (PT = transpose)
//   D, Ms, U           [NI][M][64][Pp]      inside partial, P*D message to the
//                                           parent, outside partial; state-major so
//                                           a warp reading one state of 32
//                                           consecutive patterns is coalesced
//   Ecum, Eown         [NI][M][Pp]          power-of-two scaling exponents
//   Vf                 [n][M][64][Pp]       outside vector at the top of each branch
//                                           times w_p * posterior_m / L_m
// Leaves never get a partial: their message P_b * leaf_vector is a column of P_b
// (a row of PT_b), a masked column sum, or the P_b row sums for missing data.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace h3g {

// Programmatic dependent launch: every evaluation kernel is launched with
// programmatic stream serialisation, so its CTAs may start while the previous
// kernel drains.  Each kernel first waits for the previous grid to complete
// (and its writes to become visible) before touching global memory, then lets
// the next kernel's CTAs launch into the SM space its own CTAs leave free.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

bool pdl_enabled();   // false when H3G_NO_PDL=1

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

constexpr int SP = 64;       // padded state count (61 sense codons -> 64)
constexpr int SP2 = SP * SP; // one padded matrix
constexpr int TP = 128;      // pattern padding granule (the mixed path's CTA tile)
constexpr int kMaxRateClasses = 16;

struct Topo {
    int n, root, NI, T, P, Pp, S;
    const int* ch_off;       // [n+1] children CSR, children in increasing id order
    const int* ch;
    const int* parent;       // [n] parent id, -1 at the root
    const int* iidx;         // [n] internal-node slot, -1 for leaves
    const uint8_t* leaf;     // [n]
    const int* taxon;        // [n] alignment row of a leaf, -1 = missing
    const int8_t* states;    // [T][Pp]
    const uint64_t* masks;   // [T][Pp]
    const double* w;         // [Pp] pattern weights, 0 on padding
    uint64_t all_mask;
    // per-item descriptors of the persistent passes, one load each instead of a chain of lookups
    const int2* kdesc;       // [children CSR] {child, code}: code = taxon (>= 0) or -1 for a leaf, -(2 + iidx) for an internal child
    const int4* in_info;     // [internal nodes, inside order] {u, iidx[u], first child slot, end}
    const int4* out_info;    // [2 x children, outside order] {c, u, iidx[u], iidx[c] or -1}, {first sibling slot, end, 0, 0}
    // chains of the persistent passes: the items are chain heads; a CTA carries a chain's
    // message in registers from one node to the next
    const int* in_next;      // [inside position] position of the parent when its only internal child is this node, else -1
    const int* in_heads;     // [chains] inside position of each chain's first node, inside order
    const int* out_next;     // [outside position] position of this node's deepest internal child, else -1
    const int* out_heads;    // [chains] outside position of each chain's first node, outside order
    // subtree checkpointing: Vf slot of each node (NULL: the node id).  With checkpoints, iidx and vidx
    // map checkpoint nodes to persistent slots [0, ncp) and every other node to a scratch slot that
    // the nodes of other blocks reuse
    const int* vidx;
    int ncp;
};

__device__ __forceinline__ int vslot(const Topo& t, int b) { return t.vidx ? t.vidx[b] : b; }

struct Model {
    int M, K, has_bg, nmod, time_mode, ndirs, sentinel;
    int ndirs_dense;         // the first ndirs_dense directions act on every model; direction ndirs_dense + k acts
                             // on model k alone (one matrix each, stored after the dense ones)
    const double* pi;        // [64]
    const double* Q;         // [nmod][64*64]
    const double* QT;        // [nmod][64*64] transpose of Q
    const double* lam;       // [nmod][64]
    const double* U;         // [nmod][64*64]
    const double* UT;        // [nmod][64*64] transpose of U
    const double* V;         // [nmod][64*64]
    const double* mu;        // [nmod]
    const double* class_w;   // [K]
    const double* bg_w;      // [nmod - K] background mixing weights
    const double* rates;     // [M]
    const double* rate_w;    // [M]
    const uint8_t* is_test;  // [n] or null
    const int* br_off;       // [n + 1] or null: branch b mixes classes [br_off[b], br_off[b + 1]) with class_w
    const double* dQ;        // [ndirs_dense][nmod][64*64], then [nmod][64*64] for the per-model directions
};

struct Work {
    const double* bl;        // [n]
    double* P;               // [M][n][64*64]
    double* PT;              // [M][n][64*64]
    double* dP;              // [M][n][64*64]
    double* rs;              // [M][n][64] row sums of P
    double* D;               // [NI][M][64][Pp]
    double* Ms;              // [NI][M][64][Pp]
    double* U;               // [NI][M][64][Pp]
    int* Ecum;               // [NI][M][Pp]
    int* Eown;               // [NI][M][Pp]
    double* Vf;              // [n][M][64][Pp]
    double* f;               // [M][Pp]   w_p * post_{m,p} / L_{m,p}
    double* contrib;         // [Pp]      this pattern's term of lnL
    double* site;            // [Pp]      per-pattern lnL
    double* rw;              // [M][Pp]   w_p * post_{m,p} / rho_m
    int nchunk, chunk;
    double* Apart;           // [n][M][nchunk][64*64]
    double* Afull;           // [n][M][64*64] A_{m,b} summed over chunks
    double* gt;              // [M][n]    <A_{m,b}, dP_{m,b}>
    int ngroups;             // branch groups G of the Frechet kernel
    double* Hpart;           // [nmod][M][G][64*64] per-CTA partial H
    double* gc;              // [K][M][G] <A_{m,b}, P_k(tau)> summed over a branch group
    double* stg;             // [nmod][M][G] c_k * tau * <A_{m,b}, Q_k P_k(tau)> summed over a branch group
    double* H;               // [nmod][64*64]
    double* dirpart;         // [ndirs][nmod][17]: 16 partials of sum (V dQ U) o H, then d mu = -sum pi_i dQ_ii
    double* G;               // [ndirs][nmod][64*64] V_k dQ_x U_k (depends on the model only)
    double* out;             // [2 + n + 2 nmod + M] lnl | error flag | grad_t | gc (per model) | stg | grad_rate_w
    int* err;                // sticky device error flags (bounded waits that expired)
};

__device__ __forceinline__ size_t mat_off(int m, int b, int n) { return (size_t(m) * n + b) * SP2; }
__device__ __forceinline__ size_t part_off(int ii, int m, int M, int Pp) { return (size_t(ii) * M + m) * SP * size_t(Pp); }
__device__ __forceinline__ size_t col_off(int ii, int m, int M, int Pp) { return (size_t(ii) * M + m) * size_t(Pp); }

// The classes a branch mixes and the weight of class k on it: a per-branch range of the class
// table (br_off), else the K test classes on test branches and the background classes elsewhere.
struct BranchModels {
    int k0, k1;
    bool test;
};
__device__ __forceinline__ BranchModels branch_models(const Model& md, int b) {
    if (md.br_off) return {md.br_off[b], md.br_off[b + 1], true};
    const bool test = md.is_test == nullptr || md.is_test[b] != 0;
    return {test ? 0 : md.K, test ? md.K : md.nmod, test};
}
__device__ __forceinline__ double class_weight(const Model& md, const BranchModels& bm, int k) {
    return bm.test ? md.class_w[k] : md.bg_w[k - md.K];
}

__device__ __forceinline__ double time_conv(const Model& md, int k) {
    return md.time_mode == 1 ? 3.0 / fmax(md.mu[k], 1e-12) : 1.0;
}

}  // namespace h3g
