// h3g_mixed.h — split-precision (tensor-core) pruning path.
//
// Partials are FP32 in block-floating-point form: every stored vector (one
// node, one pattern, one rate class) is normalised to a maximum in [0.5, 1)
// and carries an int32 exponent E with  true value = stored * 2^-E.  The
// 61x61 contractions run on tcgen05 (kind::f16, BF16 operands) as the six
// leading products of a three-term BF16 split of both operands
// (hh + hm + mh + hl + lh + mm), accumulated in FP32 in TMEM.
// The model (eigensystems, P assembly), rate-class mixing, the root log-sum
// and every reduction stay in FP64.
#pragma once
#include <vector>
#include "../../include/h3g.h"
#include "h3g_common.cuh"

namespace h3g {

struct MixedWork {
    float* D = nullptr;      // [NI][M][64][Pp]  inside partial (normalised)
    float* Ms = nullptr;     // [NI][M][64][Pp]  message P*D to the parent (normalised)
    float* U = nullptr;      // [NI][M][64][Pp]  outside partial below the parent branch (normalised)
    float* Vf = nullptr;     // [n][M][64][Pp]   f * V * 2^(EL - EV - ED) (gradient operand, O(1) scale)
    int* ED = nullptr;       // [NI][M][Pp]      exponent of D
    int* EM = nullptr;       // [NI][M][Pp]      exponent of Ms
    int* EU = nullptr;       // [NI][M][Pp]      exponent of U
    uint16_t* Bp[3] = {nullptr, nullptr, nullptr};   // [M][n][64*64] BF16 hi/mid/lo of P (rows = out state,
                                                     //   K = in state) as a tcgen05 K-major tile
    uint16_t* Bpt[3] = {nullptr, nullptr, nullptr};  // same for P^T
    float* PT32 = nullptr;   // [M][n][64*64]    FP32 P^T row-major (leaf messages)
    float* rs32 = nullptr;   // [M][n][64]       FP32 row sums of P
    int* flag_in = nullptr;  // [NI][M][Pp/128]  epoch of the evaluation whose inside item is stored
    int* flag_out = nullptr; // [NI][M][Pp/128]  same for the outside item (U of an internal node)
    int* sync = nullptr;     // [4]              epoch, inside and outside item counters
};

// Limit of the persistent passes' waits on another item's flag: polls before the wait gives up
// (the kernel then records H3G_ERR_TIMEOUT's flag and carries on), and a skew added to the
// awaited epoch (nonzero only to test that path: no item publishes that value).
struct WaitCfg {
    uint32_t polls = 1u << 22;
    int skew = 0;
    int ctas_per_sm = 2;      // persistent grid: resident CTAs per SM (1 or 2; the kernels' resources admit 2)
};

bool mixed_available();
void mixed_configure();
// Element counts of the mixed path's buffers: part = NI M 64 Pp, vf = n M 64 Pp, cols = NI M Pp,
// mats = M n 64 64, rs = M n 64, flags = NI M Pp / 128 (or the maxima over the problems a workspace serves).
struct MixedSizes {
    size_t part = 0, vf = 0, cols = 0, mats = 0, rs = 0, flags = 0;
};
// the buffers' zeroing is enqueued on st (the stream the evaluations run on)
h3g_status mixed_alloc(MixedWork& mw, std::vector<void*>& owned, const MixedSizes& z, cudaStream_t st);
// caller-supplied P: the split-precision operands from w.P / w.rs (new epoch included)
int mixed_prepare(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, cudaStream_t s);
// P, dP and the split-precision operands in one launch (h3g_fp64.cu); the FP64 P and P^T are not stored
int launch_build_P_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, cudaStream_t s);
// count: chains of the pass (Topo::in_heads / out_heads)
int launch_inside_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, int count, WaitCfg wc,
                        cudaStream_t s);
int launch_root_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, cudaStream_t s);
int launch_outside_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, int count, WaitCfg wc,
                         cudaStream_t s);
// d_branches NULL: every branch (grid over all node ids)
int launch_accumA_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, const int* d_branches,
                        int count, cudaStream_t s);
// new epoch and item counters for the next persistent launch of the same evaluation
int mixed_new_epoch(const MixedWork& mw, cudaStream_t s);

}  // namespace h3g
