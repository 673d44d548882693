// h3g_mixed.cu — split-precision pruning on the sm_100a tensor cores.
//
// One CTA = 128 patterns x one node (inside) or one child (outside), 512
// threads: four threads share each pattern row (16 states each); the row is
// also TMEM lane r of the accumulator, read back by the warp that owns that
// lane quadrant.  Per-pattern rescaling combines the four partial maxima
// through shared memory.  The 61x61 contraction is a
// tcgen05.mma (M=128 patterns, N=64 states, K=64 states) issued by one thread:
// A = the CTA's partial tile, written by the threads into shared memory as a
// K-major BF16 hi/mid/lo triple; B = the branch's P (or P^T) tile, prepared
// once per evaluation in the same layout and brought in by the bulk-copy (TMA)
// engine.  The six leading products of the split accumulate in FP32 in TMEM,
// which reproduces an FP32 contraction to about 2^-24.
#include <algorithm>
#include <type_traits>

#include "h3g_mixed.h"
#include "h3g_tc.cuh"

namespace h3g {

namespace {

constexpr int MT = 128;                       // patterns per CTA = MMA M
constexpr uint32_t kIdesc = tc::idesc_bf16(MT, SP);
constexpr size_t kTileBytes = size_t(MT) * SP * 2;       // 16 KB per BF16 term
constexpr size_t kBBytes = size_t(SP) * SP * 2;          // 8 KB per BF16 term
constexpr int kKSteps = SP / 16;                                 // K = 16 per kind::f16 MMA
constexpr uint32_t kTmemCols = kKSteps * SP;                     // one 64-column accumulator per K step

__device__ __forceinline__ size_t mat_off_f(int m, int b, int n) { return (size_t(m) * n + b) * SP2; }

// Thread layout of the pruning CTAs: 16 warps; warp w serves TMEM lane quadrant
// q = w % 4 (patterns 32q .. 32q+31 of the tile, lane = pattern) and state group
// g = w / 4 (states 16g .. 16g+15).  Four threads share one pattern row.
constexpr int kThreads = 512;
constexpr int kSG = 16;                                           // states per thread
constexpr size_t kMxSmem = 3 * kTileBytes + 3 * kBBytes + 4 * MT * sizeof(float) + 64;

struct Lane {
    int r;      // row in the tile (pattern), also the TMEM lane
    int g;      // state group
    int q;      // lane quadrant
    int warp;
};
__device__ __forceinline__ Lane lane_of(int tid) {
    Lane l;
    l.warp = tid >> 5;
    l.q = l.warp & 3;
    l.g = l.warp >> 2;
    l.r = 32 * l.q + (tid & 31);
    return l;
}

// Exact power-of-two scale factor 2^k for |k| <= 126.
__device__ __forceinline__ float pow2f(int k) { return __int_as_float((127 + k) << 23); }

__device__ __forceinline__ void scale_pow2(float (&v)[kSG], int sh) {
    for (int rem = sh; rem != 0;) {
        const int step = rem > 126 ? 126 : (rem < -126 ? -126 : rem);
        const float f = pow2f(step);
#pragma unroll
        for (int i = 0; i < kSG; ++i) v[i] *= f;
        rem -= step;
    }
}

// Normalise the pattern row (spread over the 4 state groups) to a maximum in
// [0.5, 1); returns the shift s (v_new = v * 2^s), identical on all 4 threads.
__device__ __forceinline__ int renorm_row(float (&v)[kSG], float* smax, const Lane& l) {
    float mx = 0.f;
#pragma unroll
    for (int i = 0; i < kSG; ++i) mx = fmaxf(mx, v[i]);
    smax[l.g * MT + l.r] = mx;
    __syncthreads();
    mx = fmaxf(fmaxf(smax[l.r], smax[MT + l.r]), fmaxf(smax[2 * MT + l.r], smax[3 * MT + l.r]));
    __syncthreads();
    if (!(mx > 0.f) || !(mx < INFINITY)) return 0;
    const int sh = -ilogbf(mx) - 1;
    scale_pow2(v, sh);
    return sh;
}

// After a node's last child product the product that follows renormalises anyway: skip the
// exchange when every thread's 16 states reach 2^-64 (power-of-two scaling is exact, so the results
// are the same), renormalise otherwise.  Without this guard, products at extreme branch lengths ran
// into the FP32 subnormal range and the gradient operand's scale overflowed.
__device__ __forceinline__ int renorm_if_small(float (&v)[kSG], float* smax, const Lane& l) {
    float mx = 0.f;
#pragma unroll
    for (int i = 0; i < kSG; ++i) mx = fmaxf(mx, v[i]);
    if (__syncthreads_and(mx >= 0x1p-64f)) return 0;
    return renorm_row(v, smax, l);
}

// Where this thread's 16 states of a child's message live: a contiguous
// row of PT32 / rs32 for a leaf (one-hot or fully ambiguous codon), a masked
// sum of PT32 rows (partially ambiguous codon), or the child's stored message
// (stride Pp) with its exponent.  Splitting address resolution from the loads
// lets a thread put the loads of two children in flight together.
struct MsgSrc {
    const float* src;
    size_t stride;      // 1 (leaf row) or Pp (stored message)
    uint64_t mk;        // != 0: masked sum of PT32 rows starting at src
    int E;              // exponent of a stored message
};
__device__ __forceinline__ MsgSrc msg_src(const Topo& t, const MixedWork& mw, int m, int M, int2 d, int p, int g, size_t so) {
    MsgSrc r{nullptr, 1, 0, 0};
    const int c = d.x;
    if (d.y >= -1) {
        const int tx = d.y;
        const float* PTc = mw.PT32 + mat_off_f(m, c, t.n);
        const int st = tx < 0 ? -1 : int(t.states[size_t(tx) * t.Pp + p]);
        if (st >= 0) {
            r.src = PTc + st * SP + kSG * g;
        } else {
            const uint64_t mk = tx < 0 ? t.all_mask : t.masks[size_t(tx) * t.Pp + p];
            if (mk == 0 || (mk & t.all_mask) == t.all_mask) {
                r.src = mw.rs32 + (size_t(m) * t.n + c) * SP + kSG * g;
            } else {
                r.src = PTc + kSG * g;
                r.mk = mk;
            }
        }
    } else {
        const int ic = -(d.y + 2);
        r.src = mw.Ms + part_off(ic, m, M, t.Pp) + so;
        r.stride = size_t(t.Pp);
        r.E = __ldcg(mw.EM + col_off(ic, m, M, t.Pp) + p);
    }
    return r;
}
__device__ __forceinline__ void msg_load(const MsgSrc& r, float (&a)[kSG]) {
    if (r.stride != 1) {                // a message written by another CTA of this launch: read through L2
#pragma unroll
        for (int i = 0; i < kSG; ++i) a[i] = __ldcg(r.src + i * r.stride);
    } else if (r.mk == 0) {
        const float4* s4 = reinterpret_cast<const float4*>(r.src);
#pragma unroll
        for (int q4 = 0; q4 < kSG / 4; ++q4) {
            const float4 x = __ldg(s4 + q4);
            a[4 * q4] = x.x; a[4 * q4 + 1] = x.y; a[4 * q4 + 2] = x.z; a[4 * q4 + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < kSG; ++i) a[i] = 0.f;
        for (uint64_t b = r.mk; b; b &= b - 1) {
            const float4* r4 = reinterpret_cast<const float4*>(r.src + (__ffsll((long long)b) - 1) * SP);
#pragma unroll
            for (int q4 = 0; q4 < kSG / 4; ++q4) {
                const float4 x = __ldg(r4 + q4);
                a[4 * q4] += x.x; a[4 * q4 + 1] += x.y; a[4 * q4 + 2] += x.z; a[4 * q4 + 3] += x.w;
            }
        }
    }
}

__device__ __forceinline__ void load_part(float (&v)[kSG], const float* src, size_t stride) {
#pragma unroll
    for (int i = 0; i < kSG; ++i) v[i] = __ldcg(src + i * stride);
}
__device__ __forceinline__ void store_part(const float (&v)[kSG], float* dst, size_t stride) {
#pragma unroll
    for (int i = 0; i < kSG; ++i) dst[i * stride] = v[i];
}

// Shared-memory block of one tensor-core contraction.
struct TcTile {
    unsigned char* A[3];   // BF16 hi / mid / lo of the CTA's 128 x 64 partial tile
    unsigned char* B[3];   // BF16 hi / mid / lo of the 64 x 64 transition tile
    float* smax;           // [4][128] per-group row maxima
    uint64_t* bars;        // [0] B tile arrival, [1] MMA completion
    uint32_t* slot;        // TMEM base address written by tcgen05.alloc
};

__device__ __forceinline__ TcTile carve(unsigned char* sm) {
    TcTile s;
    for (int q = 0; q < 3; ++q) s.A[q] = sm + q * kTileBytes;
    for (int q = 0; q < 3; ++q) s.B[q] = sm + 3 * kTileBytes + q * kBBytes;
    s.smax = reinterpret_cast<float*>(sm + 3 * kTileBytes + 3 * kBBytes);
    s.bars = reinterpret_cast<uint64_t*>(s.smax + 4 * MT);
    s.slot = reinterpret_cast<uint32_t*>(s.bars + 2);
    return s;
}

// Once per persistent CTA: barriers and TMEM.  All threads call.
__device__ __forceinline__ void tc_setup(const TcTile& s) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        tc::mbar_init(&s.bars[0], 1);
        tc::mbar_init(&s.bars[1], 1);
        tc::mbar_fence_init();
    }
    if ((tid >> 5) == 0) tc::tmem_alloc(s.slot, kTmemCols);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
}
__device__ __forceinline__ void tc_teardown(const TcTile& s) {
    tc::tc_fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(*s.slot, kTmemCols);
}
// Per item: bring the branch's B tile terms in with the bulk-copy engine (thread 0).
// The previous item's MMAs, the last readers of the B tiles, completed in its tc_run.
__device__ __forceinline__ void tc_load_b(const TcTile& s, uint16_t* const (&b)[3], size_t off) {
    if (threadIdx.x == 0) {
        tc::fence_async_smem();
        tc::mbar_expect_tx(&s.bars[0], uint32_t(3 * kBBytes));
        for (int q = 0; q < 3; ++q) tc::bulk_g2s(s.B[q], b[q] + off, uint32_t(kBBytes), &s.bars[0]);
    }
}

// Write this thread's 16 states of its row into the K-major A tiles as a BF16 split.
__device__ __forceinline__ void tc_write_part(const TcTile& s, const float (&v)[kSG], const Lane& l) {
#pragma unroll
    for (int kc = 0; kc < kSG / 8; ++kc) {
        uint32_t w[3][4];
#pragma unroll
        for (int e = 0; e < 4; ++e) tc::split3x2(v[8 * kc + 2 * e], v[8 * kc + 2 * e + 1], w[0][e], w[1][e], w[2][e]);
        const uint32_t off = tc::kmajor_off16(MT, l.r, kSG * l.g + 8 * kc);
#pragma unroll
        for (int q = 0; q < 3; ++q)
            *reinterpret_cast<uint4*>(s.A[q] + off) = make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
    }
}

// s = fl(a + b) and e = (a + b) - s exactly (Knuth's two-sum; no fast-math reassociation here)
__device__ __forceinline__ float two_sum(float a, float b, float& e) {
    const float s = a + b, bb = s - a;
    e = (a - (s - bb)) + (b - bb);
    return s;
}

// out = A * B^T for this thread's row and state group: issue (one thread),
// wait (all), read the four per-K-step accumulators from TMEM and add them with compensated FP32 sums.
__device__ __forceinline__ void tc_run(const TcTile& s, float (&o)[kSG], const Lane& l, int* err, uint32_t phase) {
    const int tid = threadIdx.x;
    tc::fence_async_smem();
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *s.slot;
    if (tid == 0) {
        const bool got_b = tc::mbar_wait(&s.bars[0], phase);
        if (got_b) {
            const uint32_t lboA = (MT / 8) * 128, lboB = (SP / 8) * 128;
            // Each K step accumulates into its own TMEM columns: the five small split
            // products first (their rounding is ~2^-8 below the result), hi*hi last,
            // so every accumulator takes at most one add at full magnitude.
            const int pa[6] = {1, 2, 0, 1, 0, 0}, pb[6] = {1, 0, 2, 0, 1, 0};   // mm lh hl mh hm hh
#pragma unroll
            for (int ks = 0; ks < kKSteps; ++ks) {
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    const uint64_t da = tc::smem_desc(tc::smem_u32(s.A[pa[q]]) + 2 * ks * lboA, lboA, 128);
                    const uint64_t db = tc::smem_desc(tc::smem_u32(s.B[pb[q]]) + 2 * ks * lboB, lboB, 128);
                    tc::mma_bf16(tmem + uint32_t(ks * SP), da, db, kIdesc, q == 0 ? 0u : 1u);
                }
            }
        } else {
            atomicOr(err, 1);
        }
        tc::mma_commit(&s.bars[1]);
    }
    if (!tc::mbar_wait(&s.bars[1], phase) && (tid & 31) == 0) atomicOr(err, 2);
    tc::tc_fence_after();
    const uint32_t row = tmem + (uint32_t(32 * l.q) << 16) + uint32_t(kSG * l.g);
    // read back in two halves of 8 columns (fewer live registers)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        float t8[kKSteps][8];
#pragma unroll
        for (int ks = 0; ks < kKSteps; ++ks) tc::tmem_ld8(row + uint32_t(ks * SP + 8 * h), t8[ks]);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            // the four K-step sums added with their rounding errors carried (error-free two-sums in
            // FP32): the FP64 sum's result without its conversions, which limited the pass's throughput
            float e1, e2, e3;
            const float s1 = two_sum(t8[0][i], t8[1][i], e1);
            const float s2 = two_sum(t8[2][i], t8[3][i], e2);
            const float sm = two_sum(s1, s2, e3);
            o[8 * h + i] = sm + ((e1 + e2) + e3);
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
}

// ------------------------------------------------------------ P preparation
// grid (n, M), block 256: BF16 hi/mid/lo tiles of P and P^T, FP32 P^T and row sums.
__global__ void __launch_bounds__(256) k_prep_mx(Topo t, Model md, Work w, MixedWork mw) {
    pdl_enter();
    const int b = blockIdx.x, m = blockIdx.y, tid = threadIdx.x;
    if (b == 0 && m == 0 && tid == 0) {        // a new evaluation: new epoch, fresh item counters
        mw.sync[0] += 1;
        mw.sync[1] = 0;
        mw.sync[2] = 0;
    }
    if (b == t.root) return;
    const double* P = w.P + mat_off(m, b, t.n);
    const size_t o = mat_off_f(m, b, t.n);
    for (int e = tid; e < SP2; e += 256) {
        const int i = e >> 6, j = e & 63;
        const float x = float(P[e]);             // P[i][j]
        const tc::Bf16x3 sp = tc::split3(x);
        const uint16_t terms[3] = {sp.hi, sp.mid, sp.lo};
        // inside contraction: row i (output state), K = j;  outside (P^T): row j, K = i
        const uint32_t oi = tc::kmajor_off16(SP, i, j) / 2, ot = tc::kmajor_off16(SP, j, i) / 2;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            mw.Bp[q][o + oi] = terms[q];
            mw.Bpt[q][o + ot] = terms[q];
        }
        mw.PT32[o + size_t(j) * SP + i] = x;
    }
    if (tid < SP) mw.rs32[(size_t(m) * t.n + b) * SP + tid] = float(w.rs[(size_t(m) * t.n + b) * SP + tid]);
}

// --------------------------------------------------- persistent pass machinery
// The inside and outside passes are each ONE launch of persistent CTAs (two per
// SM).  A work item is (node, rate class, 128-pattern tile); items are claimed
// from a counter in tree order (children before parents for the inside pass,
// parents before children for the outside pass), so an item only ever waits for
// items that running CTAs have already claimed.  An item waits for the items
// it reads with a per-(node, class, tile) flag that holds the evaluation's
// epoch once the item's partials are in memory.  This replaces one launch and
// one grid-wide wait per tree level with per-tile dependencies.
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// next item for this CTA (all threads call)
__device__ __forceinline__ int claim(int* ctr, int* s_item) {
    __syncthreads();
    if (threadIdx.x == 0) *s_item = atomicAdd(ctr, 1);
    __syncthreads();
    return *s_item;
}
// thread 0: bounded wait (wc.polls polls) until an item's flag holds this evaluation's epoch
// (plus wc.skew: a nonzero skew waits for a value no item publishes, the test of this path)
__device__ __forceinline__ void wait_item(const int* flag, int epoch, int* err, const WaitCfg& wc) {
    const int want = epoch + wc.skew;
    for (uint32_t it = 0; ld_acquire(flag) != want; ++it) {
        if (it >= wc.polls) { atomicOr(err, 32); return; }
        __nanosleep(64);
    }
}
// all threads: the partials are stored; make them visible and raise the flag.  Every thread's stores
// precede the CTA barrier, the barrier synchronises them with thread 0, and thread 0's release store
// (st.release.gpu, cumulative) orders all of them before the flag for a reader that acquires it
// (wait_item's ld.acquire.gpu followed by its CTA barrier): no separate __threadfence is needed.
__device__ __forceinline__ void publish(int* flag, int epoch) {
    __syncthreads();
    if (threadIdx.x == 0) st_release(flag, epoch);
}
// all threads: the item's partials are stored; make them visible, raise its flag, and
// claim the CTA's next item in the same step (the item being published waits for nothing
// more, so holding the next claim meanwhile cannot block anyone)
__device__ __forceinline__ int publish_and_claim(int* flag, int epoch, int* ctr, int* s_item) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const int next = atomicAdd(ctr, 1);
        st_release(flag, epoch);                  // ordered as in publish()
        *s_item = next;
    }
    __syncthreads();
    return *s_item;
}

// ------------------------------------------------------------------ inside
// Persistent: grid min(items, 2 x SMs), block 512; items (chain, m, tile) in the order of
// t.in_heads (chains by the height of their first node, the root's last).  A chain runs up
// the tree while the parent's only internal child is the node just finished.
__global__ void __launch_bounds__(kThreads, 2) k_inside_mx(Topo t, Model md, Work w, MixedWork mw, int n_items, WaitCfg wc) {
    pdl_enter();
    extern __shared__ __align__(1024) unsigned char smraw[];
    __shared__ int s_item;
    const TcTile s = carve(smraw);
    const Lane l = lane_of(threadIdx.x);
    const int M = md.M, ntile = t.Pp / MT;
    const size_t Pp = size_t(t.Pp);
    const int epoch = __ldcg(mw.sync);
    tc_setup(s);
    uint32_t phase = 0;
    int item = claim(mw.sync + 1, &s_item);
    while (item < n_items) {
        const int tile = item % ntile, rest = item / ntile, m = rest % M;
        const int p = tile * MT + l.r;
        const size_t so = size_t(kSG * l.g) * Pp + p;     // this thread's first state of the pattern column
        int pos = t.in_heads[rest / M];
        int carried = -1;                                 // the chain's previous node, whose message v holds
        float v[kSG];
        int E = 0, iu = 0;
        for (;;) {
            const int4 info = t.in_info[pos];
            const int u = info.x, k0 = info.z, k1 = info.w;
            iu = info.y;
            const bool root = u == t.root;
            if (!root) tc_load_b(s, mw.Bp, mat_off_f(m, u, t.n));
            if (carried < 0) {
                if (threadIdx.x == 0)
                    for (int k = k0; k < k1; ++k) {
                        const int code = t.kdesc[k].y;
                        // a checkpoint slot (below t.ncp) was written by an earlier launch: no wait
                        if (code <= -2 && -(code + 2) >= t.ncp)
                            wait_item(mw.flag_in + (size_t(-(code + 2)) * M + m) * ntile + tile, epoch, w.err, wc);
                    }
                __syncthreads();
                // the first two children's messages load together (padding states are zero in every
                // message), then one product and one renormalisation; further children one at a time.
                // The product with the last child is renormalised only when it is small (renorm_if_small)
                const MsgSrc s0 = msg_src(t, mw, m, M, t.kdesc[k0], p, l.g, so);
                E = s0.E;
                if (k0 + 1 < k1) {
                    const MsgSrc s1 = msg_src(t, mw, m, M, t.kdesc[k0 + 1], p, l.g, so);
                    float b[kSG];
                    msg_load(s0, v);
                    msg_load(s1, b);
#pragma unroll
                    for (int i = 0; i < kSG; ++i) v[i] *= b[i];
                    E += s1.E;
                } else {
                    msg_load(s0, v);
                }
                E += k0 + 2 < k1 ? renorm_row(v, s.smax, l) : renorm_if_small(v, s.smax, l);
                for (int k = k0 + 2; k < k1; ++k) {
                    const MsgSrc sr = msg_src(t, mw, m, M, t.kdesc[k], p, l.g, so);
                    float a[kSG];
                    msg_load(sr, a);
#pragma unroll
                    for (int i = 0; i < kSG; ++i) v[i] *= a[i];
                    E += sr.E + (k + 1 < k1 ? renorm_row(v, s.smax, l) : renorm_if_small(v, s.smax, l));
                }
            } else {
                // a chain node: its only internal child is the previous node (message in v, exponent E);
                // the other children are leaves (the last product again through renorm_if_small)
                const int k_last = t.kdesc[k1 - 1].x == carried ? k1 - 2 : k1 - 1;
                for (int k = k0; k < k1; ++k) {
                    const int2 d = t.kdesc[k];
                    if (d.x == carried) continue;
                    const MsgSrc sr = msg_src(t, mw, m, M, d, p, l.g, so);
                    float a[kSG];
                    msg_load(sr, a);
#pragma unroll
                    for (int i = 0; i < kSG; ++i) v[i] *= a[i];
                    E += sr.E + (k != k_last ? renorm_row(v, s.smax, l) : renorm_if_small(v, s.smax, l));
                }
            }
            store_part(v, mw.D + part_off(iu, m, M, t.Pp) + so, Pp);
            if (l.g == 0) mw.ED[col_off(iu, m, M, t.Pp) + p] = E;
            if (root) break;
            tc_write_part(s, v, l);
            tc_run(s, v, l, w.err, phase);                // v: the message to the parent
            phase ^= 1u;
            const int sh = renorm_row(v, s.smax, l);
            E += sh;
            store_part(v, mw.Ms + part_off(iu, m, M, t.Pp) + so, Pp);
            if (l.g == 0) mw.EM[col_off(iu, m, M, t.Pp) + p] = E;
            const int nxt = t.in_next[pos];
            if (nxt < 0) break;
            // the parent has no other internal child: it is next, with this message in registers
            // (its flag is never read, so none is raised)
            carried = u;
            pos = nxt;
        }
        item = publish_and_claim(mw.flag_in + (size_t(iu) * M + m) * ntile + tile, epoch, mw.sync + 1, &s_item);
    }
    tc_teardown(s);
}

// --------------------------------------------------------------------- root
__global__ void k_root_mx(Topo t, Model md, Work w, MixedWork mw) {
    pdl_enter();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= t.Pp) return;
    const int ir = t.iidx[t.root], M = md.M;
    const double wt = t.w[p];
    double L[kMaxRateClasses], ll[kMaxRateClasses];
    for (int m = 0; m < M; ++m) {
        const float* D = mw.D + part_off(ir, m, M, t.Pp) + p;
        double s = 0.0;
        for (int i = 0; i < SP; ++i) s = fma(md.pi[i], double(D[size_t(i) * t.Pp]), s);
        L[m] = s;
        ll[m] = s > 0.0 ? log(s) - double(mw.ED[col_off(ir, m, M, t.Pp) + p]) * 0.69314718055994530942 : -1e20;
    }
    double site = -1e20, contrib = 0.0;
    bool ok = false;
    if (M == 1) {
        if (L[0] > 0.0) { ok = true; site = ll[0]; contrib = wt * ll[0]; w.f[p] = wt / L[0]; }
        else w.f[p] = 0.0;
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
// Persistent like the inside pass; items (chain, m, tile) in the order of t.out_heads (chains
// by the depth of their first node's parent).  A chain runs down the tree through each
// node's deepest internal child.
__global__ void __launch_bounds__(kThreads, 2) k_outside_mx(Topo t, Model md, Work w, MixedWork mw, int n_items, WaitCfg wc) {
    pdl_enter();
    extern __shared__ __align__(1024) unsigned char smraw[];
    __shared__ int s_item;
    const TcTile s = carve(smraw);
    const Lane l = lane_of(threadIdx.x);
    const int M = md.M, ntile = t.Pp / MT;
    const size_t Pp = size_t(t.Pp);
    const int epoch = __ldcg(mw.sync);
    const int ir = t.iidx[t.root];
    tc_setup(s);
    uint32_t phase = 0;
    int item = claim(mw.sync + 2, &s_item);
    while (item < n_items) {
        const int tile = item % ntile, rest = item / ntile, m = rest % M;
        const int p = tile * MT + l.r;
        const size_t so = size_t(kSG * l.g) * Pp + p;
        int pos = t.out_heads[rest / M];
        bool carried = false;                             // v holds the parent's outside vector (chain)
        float v[kSG];
        int EV = 0, last = -1;
        for (;;) {
            const int4 oi = t.out_info[2 * pos], oj = t.out_info[2 * pos + 1];
            const int c = oi.x, u = oi.y, iu = oi.z, ic = oi.w, k0 = oj.x, k1 = oj.y;
            const bool internal = ic >= 0;
            if (internal) tc_load_b(s, mw.Bpt, mat_off_f(m, c, t.n));
            if (!carried) {
                if (threadIdx.x == 0 && u != t.root && iu >= t.ncp)
                    wait_item(mw.flag_out + (size_t(iu) * M + m) * ntile + tile, epoch, w.err, wc);
                __syncthreads();
                if (u == t.root) {
#pragma unroll
                    for (int i = 0; i < kSG; ++i) v[i] = float(md.pi[kSG * l.g + i]);
                    EV = 0;
                } else {
                    load_part(v, mw.U + part_off(iu, m, M, t.Pp) + so, Pp);
                    EV = __ldcg(mw.EU + col_off(iu, m, M, t.Pp) + p);
                }
            }
            // times every sibling's message, renormalised after each (after the last only when it is
            // small: the gradient operand carries its scale in EV, and U_c is renormalised after its product)
            const int k_last = t.kdesc[k1 - 1].x == c ? k1 - 2 : k1 - 1;
            for (int k = k0; k < k1; ++k) {
                const int2 sb = t.kdesc[k];
                if (sb.x == c) continue;
                const MsgSrc sr = msg_src(t, mw, m, M, sb, p, l.g, so);
                float a[kSG];
                msg_load(sr, a);
#pragma unroll
                for (int i = 0; i < kSG; ++i) v[i] *= a[i];
                EV += sr.E + (k != k_last ? renorm_row(v, s.smax, l) : renorm_if_small(v, s.smax, l));
            }
            // gradient operand: f * V_true * D-scale, with V_true = v * 2^-EV and D_true = D * 2^-ED_c
            const int EL = mw.ED[col_off(ir, m, M, t.Pp) + p];
            const int EDc = internal ? mw.ED[col_off(ic, m, M, t.Pp) + p] : 0;
            const double scale = ldexp(w.f[size_t(m) * Pp + p], EL - EV - EDc);
            float* vf = mw.Vf + part_off(vslot(t, c), m, M, t.Pp) + so;
#pragma unroll
            for (int i = 0; i < kSG; ++i) vf[i * Pp] = v[i] * float(scale);
            if (!internal) break;                          // a leaf: no outside vector below it
            tc_write_part(s, v, l);
            tc_run(s, v, l, w.err, phase);                // v: U_c, the outside vector at c
            phase ^= 1u;
            EV += renorm_row(v, s.smax, l);
            store_part(v, mw.U + part_off(ic, m, M, t.Pp) + so, Pp);
            if (l.g == 0) mw.EU[col_off(ic, m, M, t.Pp) + p] = EV;
            const int nxt = t.out_next[pos];
            if (nxt < 0) { last = ic; break; }
            // c's other children read U_c: raise its flag, then go on with the deepest internal
            // child, U_c kept in registers
            publish(mw.flag_out + (size_t(ic) * M + m) * ntile + tile, epoch);
            carried = true;
            pos = nxt;
        }
        item = last >= 0 ? publish_and_claim(mw.flag_out + (size_t(last) * M + m) * ntile + tile, epoch, mw.sync + 2, &s_item)
                         : claim(mw.sync + 2, &s_item);
    }
    tc_teardown(s);
}

// ------------------------------------------------------------------ accum A
// A_{m,b,chunk}[i][j] = sum_p Vf[i][p] D[j][p] on the tensor cores: the K
// dimension of the MMA is the pattern axis.  Both operands are split into
// BF16 hi/mid/lo; the V terms are stacked as one 192-row K-major tile
// [lo | hi | mid], so two M=128 operands cover all six leading products with
// four MMAs per K step (N = 64 states of D):
//   acc0 += [hi; mid] x D_hi      rows 0-63: hi*hi   rows 64-127: mid*hi
//   acc1 += [hi; mid] x D_mid                hi*mid              mid*mid
//   acc2 += [lo; hi]  x D_hi                 lo*hi               (unused)
//   acc3 += [lo; hi]  x D_lo                 (unused)            hi*lo
// A[i][.] = acc0[i] + acc1[i] + acc2[i] + acc0[64+i] + acc1[64+i] + acc3[64+i].
// Leaf branches have 0/1 leaf vectors (exact in BF16): only acc0 and acc2.
// Every kADrain tiles (1024 patterns) the accumulators are drained into FP64 registers, so no
// FP32 accumulator takes more than 4 * kADrain = 64 additions: a truncation bias below 2e-6 relative
// even if every addition truncated by half an ulp (gradient errors against FP64 measured 0.8-3e-6;
// draining every 256 patterns kept them at 0.6-1e-6 and cost 11 % of the kernel in FP64 conversions).
//
// Pipeline (one CTA per SM, 16 warps): the FP32 V and D tiles of 64 patterns
// stream into a kRing-deep shared-memory ring by 16-byte cp.async (one commit
// group per tile); the threads split the oldest ring slot into one of two
// BF16 MMA stages; one thread issues the MMAs of that stage asynchronously.
// Copies for tiles k+1 .. k+3, the split of tile k and the MMAs of tile k-1 overlap.
// grid (n, M, nchunk), block 512 (warp w: TMEM lane quadrant w % 4, column quarter w / 4).
constexpr int kAccThreads = 512;
constexpr int kAT = 64;                                   // patterns per tile (MMA K per tile)
constexpr int kADrain = 16;                               // tiles per FP32 accumulation group
constexpr int kRing = 4;                                  // FP32 tiles in flight
constexpr uint32_t kVRows = 3 * SP;                       // stacked V terms
constexpr uint32_t kVLbo = (kVRows / 8) * 128;            // K-chunk stride in the V stack
constexpr uint32_t kDLbo = (SP / 8) * 128;                // K-chunk stride in a D term
constexpr size_t kVStage = size_t(kVRows) * kAT * 2;      // 24 KB
constexpr size_t kDTerm = size_t(SP) * kAT * 2;           // 8 KB
constexpr size_t kStage = kVStage + 3 * kDTerm;           // 48 KB per BF16 MMA stage
// FP32 row of a tile, unpadded: its 16-byte chunk j sits at position j ^ (row & 7), so the 16-byte
// reads of 8 consecutive rows hit 8 different bank groups (the padding this replaces cost the 4th ring slot)
constexpr uint32_t kRawRow = kAT * 4;
constexpr size_t kRawOp = size_t(SP) * kRawRow;           // 16 KB per operand
constexpr size_t kRawSlot = 2 * kRawOp;                   // V and D
constexpr size_t kAccSmem = 2 * kStage + kRing * kRawSlot + 8 * 2 + 16;
// Two TMEM accumulator sets of 4 x 64 columns (all 512 columns: the shared memory above admits one
// CTA per SM), so one group's drain overlaps the next group's products.
constexpr uint32_t kAccSet = 256;

struct Split8 { uint4 hi, mid, lo; };
__device__ __forceinline__ Split8 split8(const float (&x)[8]) {
    uint32_t h[4], md[4], lo[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) tc::split3x2(x[2 * e], x[2 * e + 1], h[e], md[e], lo[e]);
    return {make_uint4(h[0], h[1], h[2], h[3]), make_uint4(md[0], md[1], md[2], md[3]), make_uint4(lo[0], lo[1], lo[2], lo[3])};
}

// The 8 patterns of state row j of a leaf's 0/1 vector, from the tile's states
// (8 bytes at st) and masks (8 words at mk) staged in shared memory.
__device__ __forceinline__ void leaf_row8_smem(const Topo& t, int tx, int j, const unsigned char* st, const uint64_t* mk,
                                               float (&d)[8]) {
    if (j >= t.S) {
#pragma unroll
        for (int x = 0; x < 8; ++x) d[x] = 0.f;
        return;
    }
    if (tx < 0) {
#pragma unroll
        for (int x = 0; x < 8; ++x) d[x] = 1.f;
        return;
    }
    const uint64_t st8 = *reinterpret_cast<const uint64_t*>(st);
#pragma unroll
    for (int x = 0; x < 8; ++x) {
        const int s = int(int8_t(uint8_t(st8 >> (8 * x))));
        bool on;
        if (s >= 0) {
            on = s == j;
        } else {
            const uint64_t m = mk[x];
            on = m == 0 || (m & t.all_mask) == t.all_mask || ((m >> j) & 1);
        }
        d[x] = on ? 1.f : 0.f;
    }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void ld_row8(const unsigned char* raw, int row, int kc, float (&x)[8]) {
    const unsigned char* rb = raw + row * kRawRow;
    const float4 a = *reinterpret_cast<const float4*>(rb + (((2 * kc) ^ (row & 7)) << 4));
    const float4 b = *reinterpret_cast<const float4*>(rb + (((2 * kc + 1) ^ (row & 7)) << 4));
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w; x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
}

__global__ void __launch_bounds__(kAccThreads, 1) k_accumA_mx(Topo t, Model md, Work w, MixedWork mw,
                                                              const int* __restrict__ branches) {
    pdl_enter();
    extern __shared__ __align__(1024) unsigned char smraw[];
    const int b = branches ? branches[blockIdx.x] : int(blockIdx.x), m = blockIdx.y, ck = blockIdx.z, tid = threadIdx.x;
    if (b == t.root) return;
    const int M = md.M, warp = tid >> 5, lane = tid & 31;
    const size_t Pp = size_t(t.Pp);
    const int p_begin = ck * w.chunk, p_end = min(t.Pp, p_begin + w.chunk);
    const int ntile = (p_end - p_begin) / kAT;
    const bool lf = t.leaf[b];
    const int tx = lf ? t.taxon[b] : -1;
    const float* Vb = mw.Vf + part_off(vslot(t, b), m, M, t.Pp);
    const float* Db = lf ? nullptr : mw.D + part_off(t.iidx[b], m, M, t.Pp);
    unsigned char* ring = smraw + 2 * kStage;
    uint64_t* mma_bar = reinterpret_cast<uint64_t*>(ring + kRing * kRawSlot);   // [2]
    uint32_t* slot = reinterpret_cast<uint32_t*>(mma_bar + 2);
    if (tid == 0) {
        for (int q = 0; q < 2; ++q) tc::mbar_init(&mma_bar[q], 1);
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc(slot, 2 * kAccSet);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *slot;

    // all threads stream tile `tile` into ring slot tile % kRing with 16-byte cp.async
    // (256-byte state-row segments, two rows per warp instruction); one commit group per tile
    auto produce = [&](int tile) {
        if (tile < ntile) {
            unsigned char* dst = ring + (tile % kRing) * kRawSlot;
            const size_t p0 = size_t(p_begin) + size_t(tile) * kAT;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int c = tid + kAccThreads * q, r = c >> 4, c16 = c & 15;
                const int pc = (c16 ^ (r & 7)) * 16;
                cp_async16(dst + r * kRawRow + pc, Vb + size_t(r) * Pp + p0 + 4 * c16);
                if (!lf) cp_async16(dst + kRawOp + r * kRawRow + pc, Db + size_t(r) * Pp + p0 + 4 * c16);
            }
            if (lf && tx >= 0 && tid < 36) {
                // a leaf's states (64 B) and masks (512 B) of the tile, in the unused D area of the slot
                const size_t o = size_t(tx) * Pp + p0;
                if (tid < 4) cp_async16(dst + kRawOp + tid * 16, t.states + o + 16 * tid);
                else cp_async16(dst + kRawOp + 64 + (tid - 4) * 16, t.masks + o + 2 * (tid - 4));
            }
        }
        cp_async_commit();
    };

    // split item of this thread: state row 8 (tid / 64) + tid % 8, 8-pattern chunk (tid / 8) % 8
    const int row = 8 * (tid >> 6) + (tid & 7), kc = (tid >> 3) & 7;
    const int lq = warp & 3, cq = warp >> 2;
    const bool top = lq < 2;
    double dacc[16];
#pragma unroll
    for (int x = 0; x < 16; ++x) dacc[x] = 0.0;

    // Accumulator group G (tiles kADrain G .. kADrain G + kADrain - 1) runs on TMEM set G & 1; draining it
    // waits for the commit of its last tile and adds the set into the FP64 registers.
    auto drain = [&](int G) {
        const int kl = min(ntile, (G + 1) * kADrain) - 1;
        if (kl < 0) return;
        if (!tc::mbar_wait(&mma_bar[kl & 1], uint32_t((kl >> 1) & 1)) && lane == 0) atomicOr(w.err, 8);
        tc::tc_fence_after();
        const uint32_t rowaddr = tmem + kAccSet * uint32_t(G & 1) + (uint32_t(32 * lq) << 16) + uint32_t(16 * cq);
        // acc0, acc1 (internal branches) and acc2 (top rows) / acc3 (bottom rows, internal branches)
        const uint32_t cols[3] = {0u, 64u, top ? 128u : 192u};
        const bool use[3] = {true, !lf, top || !lf};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (!use[a]) continue;
            float v16[16];
            tc::tmem_ld16(rowaddr + cols[a], v16);
            tc::tmem_wait_ld();
#pragma unroll
            for (int x = 0; x < 16; ++x) dacc[x] += double(v16[x]);
        }
        tc::tc_fence_before();
        __syncthreads();
        tc::tc_fence_after();
    };
    for (int q = 0; q < kRing - 1; ++q) produce(q);
    for (int kt = 0; kt < ntile; ++kt) {
        const int st = kt & 1, sl = kt % kRing;
        produce(kt + kRing - 1);                 // slot of tile kt-1, released by the barrier of iteration kt-1
        cp_async_wait<kRing - 1>();              // this thread's copies of tile kt have landed
        __syncthreads();                         // ... and everyone else's
        unsigned char* VS = smraw + st * kStage;
        unsigned char* DS = VS + kVStage;
        const unsigned char* raw = ring + sl * kRawSlot;
        if (kt >= 2 && !tc::mbar_wait(&mma_bar[st], uint32_t(((kt - 2) >> 1) & 1)) && lane == 0) atomicOr(w.err, 4);
        {
            const uint32_t rg = uint32_t(row >> 3) * 128 + uint32_t(row & 7) * 16;
            float x[8];
            ld_row8(raw, row, kc, x);
            const Split8 sv = split8(x);
            *reinterpret_cast<uint4*>(VS + kc * kVLbo + 0 * 1024 + rg) = sv.lo;
            *reinterpret_cast<uint4*>(VS + kc * kVLbo + 1 * 1024 + rg) = sv.hi;
            *reinterpret_cast<uint4*>(VS + kc * kVLbo + 2 * 1024 + rg) = sv.mid;
            if (lf) {
                leaf_row8_smem(t, tx, row, raw + kRawOp + 8 * kc, reinterpret_cast<const uint64_t*>(raw + kRawOp + 64) + 8 * kc, x);
                uint32_t h[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) h[e] = tc::bf16x2_bits(x[2 * e], x[2 * e + 1]);
                *reinterpret_cast<uint4*>(DS + kc * kDLbo + rg) = make_uint4(h[0], h[1], h[2], h[3]);
            } else {
                ld_row8(raw + kRawOp, row, kc, x);
                const Split8 sd = split8(x);
                *reinterpret_cast<uint4*>(DS + kc * kDLbo + rg) = sd.hi;
                *reinterpret_cast<uint4*>(DS + kDTerm + kc * kDLbo + rg) = sd.mid;
                *reinterpret_cast<uint4*>(DS + 2 * kDTerm + kc * kDLbo + rg) = sd.lo;
            }
        }
        tc::fence_async_smem();
        tc::tc_fence_before();
        __syncthreads();
        tc::tc_fence_after();
        if (tid == 0) {
            const uint32_t vs = tc::smem_u32(VS), ds = tc::smem_u32(DS);
            const bool first = (kt % kADrain) == 0;
            const uint32_t set = tmem + kAccSet * uint32_t((kt / kADrain) & 1);     // this group's accumulators
#pragma unroll
            for (int ks = 0; ks < kAT / 16; ++ks) {
                const uint32_t acc = (first && ks == 0) ? 0u : 1u;
                const uint64_t a1 = tc::smem_desc(vs + 1024 + 2 * ks * kVLbo, kVLbo, 128);   // [hi; mid]
                const uint64_t a2 = tc::smem_desc(vs + 2 * ks * kVLbo, kVLbo, 128);          // [lo; hi]
                const uint64_t bh = tc::smem_desc(ds + 2 * ks * kDLbo, kDLbo, 128);
                tc::mma_bf16(set + 0, a1, bh, kIdesc, acc);
                tc::mma_bf16(set + 128, a2, bh, kIdesc, acc);
                if (!lf) {
                    const uint64_t bm = tc::smem_desc(ds + uint32_t(kDTerm) + 2 * ks * kDLbo, kDLbo, 128);
                    const uint64_t bl = tc::smem_desc(ds + uint32_t(2 * kDTerm) + 2 * ks * kDLbo, kDLbo, 128);
                    tc::mma_bf16(set + 64, a1, bm, kIdesc, acc);
                    tc::mma_bf16(set + 192, a2, bl, kIdesc, acc);
                }
            }
            tc::mma_commit(&mma_bar[st]);
        }
        // the previous group's accumulators drain while this tile's products run on the other set
        if ((kt % kADrain) == 0 && kt > 0) drain(kt / kADrain - 1);
    }
    drain((ntile - 1) / kADrain);
    // combine the two halves of each state row in shared memory (stages are idle now), write coalesced
    double* sA = reinterpret_cast<double*>(smraw);              // [64][65]
    const int i = 32 * lq + lane - (top ? 0 : 64);
    if (!top) {
#pragma unroll
        for (int x = 0; x < 16; ++x) sA[i * 65 + 16 * cq + x] = dacc[x];
    }
    __syncthreads();
    if (top) {
#pragma unroll
        for (int x = 0; x < 16; ++x) sA[i * 65 + 16 * cq + x] += dacc[x];
    }
    __syncthreads();
    double* dst = w.Apart + ((size_t(b) * M + m) * w.nchunk + ck) * SP2;
    for (int e = tid; e < SP2; e += kAccThreads) dst[e] = sA[(e >> 6) * 65 + (e & 63)];
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 2 * kAccSet);
}

}  // namespace

bool mixed_available() { return true; }

void mixed_configure() {
    cudaFuncSetAttribute(k_accumA_mx, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kAccSmem));
    cudaFuncSetAttribute(k_inside_mx, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kMxSmem));
    cudaFuncSetAttribute(k_outside_mx, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kMxSmem));
}

h3g_status mixed_alloc(MixedWork& mw, std::vector<void*>& owned, const MixedSizes& z, cudaStream_t st) {
    auto take = [&](auto** ptr, size_t count) -> bool {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(**ptr)) != cudaSuccess) return false;
        owned.push_back(p);
        *ptr = static_cast<std::remove_reference_t<decltype(*ptr)>>(p);
        return true;
    };
    const size_t part = z.part, cols = z.cols, mats = z.mats;
    bool ok = take(&mw.D, part) && take(&mw.Ms, part) && take(&mw.U, part) && take(&mw.Vf, z.vf) &&
              take(&mw.ED, cols) && take(&mw.EM, cols) && take(&mw.EU, cols) && take(&mw.PT32, mats) &&
              take(&mw.rs32, z.rs);
    // partials start at zero (their padding states 61 .. 63 are then zero before any evaluation)
    // on the evaluations' stream: a default-stream memset is not ordered before the kernels of a
    // non-blocking stream, and one landing after the first evaluation has begun clears published flags
    ok = ok && cudaMemsetAsync(mw.D, 0, part * sizeof(float), st) == cudaSuccess &&
         cudaMemsetAsync(mw.Ms, 0, part * sizeof(float), st) == cudaSuccess &&
         cudaMemsetAsync(mw.U, 0, part * sizeof(float), st) == cudaSuccess &&
         cudaMemsetAsync(mw.Vf, 0, z.vf * sizeof(float), st) == cudaSuccess;
    for (int q = 0; q < 3 && ok; ++q) ok = take(&mw.Bp[q], mats) && take(&mw.Bpt[q], mats);
    const size_t flags = z.flags;
    ok = ok && take(&mw.flag_in, flags) && take(&mw.flag_out, flags) && take(&mw.sync, 4);
    ok = ok && cudaMemsetAsync(mw.flag_in, 0, flags * sizeof(int), st) == cudaSuccess &&
         cudaMemsetAsync(mw.flag_out, 0, flags * sizeof(int), st) == cudaSuccess &&
         cudaMemsetAsync(mw.sync, 0, 4 * sizeof(int), st) == cudaSuccess;
    return ok ? H3G_OK : H3G_ERR_OOM;
}

int mixed_prepare(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, cudaStream_t s) {
    launch_k(k_prep_mx, dim3(t.n, md.M), 256, 0, s, t, md, w, mw);
    return 1;
}
static int persistent_ctas(int items, int per_sm) {
    static int sms = [] {
        int dev = 0, v = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v;
    }();
    return std::max(1, std::min(items, std::max(1, std::min(per_sm, 2)) * sms));
}
int launch_inside_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, int count, WaitCfg wc,
                        cudaStream_t s) {
    const int items = count * md.M * (t.Pp / MT);
    launch_k(k_inside_mx, persistent_ctas(items, wc.ctas_per_sm), kThreads, kMxSmem, s, t, md, w, mw, items, wc);
    return 1;
}
int launch_root_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, cudaStream_t s) {
    launch_k(k_root_mx, (t.Pp + 127) / 128, 128, 0, s, t, md, w, mw);
    return 1;
}
int launch_outside_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, int count, WaitCfg wc,
                         cudaStream_t s) {
    const int items = count * md.M * (t.Pp / MT);
    launch_k(k_outside_mx, persistent_ctas(items, wc.ctas_per_sm), kThreads, kMxSmem, s, t, md, w, mw, items, wc);
    return 1;
}
int launch_accumA_mixed(const Topo& t, const Model& md, const Work& w, const MixedWork& mw, const int* d_branches,
                        int count, cudaStream_t s) {
    const int* none = nullptr;
    launch_k(k_accumA_mx, dim3(d_branches ? count : t.n, md.M, w.nchunk), kAccThreads, kAccSmem, s, t, md, w, mw,
             d_branches ? d_branches : none);
    return 1;
}

// A new epoch and fresh item counters between two persistent launches of one evaluation (the blocks of
// a checkpoint plan reuse scratch slots, whose flags then hold an older epoch).
__global__ void k_new_epoch_mx(MixedWork mw) {
    pdl_enter();
    if (threadIdx.x == 0) {
        mw.sync[0] += 1;
        mw.sync[1] = 0;
        mw.sync[2] = 0;
    }
}

int mixed_new_epoch(const MixedWork& mw, cudaStream_t s) {
    launch_k(k_new_epoch_mx, 1, 32, 0, s, mw);
    return 1;
}

}  // namespace h3g
