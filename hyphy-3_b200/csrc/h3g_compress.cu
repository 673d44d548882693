// h3g_compress.cu — Alignment::finalize's codon translation, nucleotide counts
// and site-pattern compression on the device (h3g_alignment_compress*).
//
// The reference translates every (taxon, codon) on the host and inserts each
// codon column, as a vector of (state, mask) pairs, into an unordered_map in
// column order (include/hyphy/core/alignment.hpp:665-722, :1021-1078).  Here:
//
//   k_translate  grid (128-codon groups, taxa / 32), block 256.  The block's
//                32 x 384-character strip of the [taxa][nucleotides] input is
//                staged in shared memory with 16-byte loads; for each 32-codon
//                tile a lane translates one codon (lane = column, warp = 4 taxa),
//                adds its hash contribution and nucleotide counts in
//                registers and leaves the 16-bit key in shared memory; the
//                tile is then stored column-major ([column][taxon], 64
//                contiguous bytes per warp).
//   k_insert     one thread per unresolved column: open addressing on the
//                column hash, the slot keeps its smallest column (atomicMin).
//   k_verify     one warp per unresolved column: full comparison with its
//                slot's smallest column; equal columns are resolved, the
//                others (hash collisions) go to the next round with a new seed.
//   scan         representatives (columns resolved to themselves) numbered in
//                column order = the reference's first-occurrence order.
//   k_assign / k_gather   site -> pattern, weights, pattern-major states/masks.
//
// Key of a cell (16 bits): 0x8000 | s for the unambiguous sense codon s, else the
// id of its set of compatible sense codons among the distinct sets the genetic
// code gives (a host table over the 4096 IUPAC triples; stops, '!' and gaps map to
// the set of every sense codon).  Equal keys <=> equal (state, mask).  A column's
// hash is sum over taxa t of Z[key_t] x salt_t mod 2^64 (Zobrist-style: Z random per
// key, salt_t random and odd per taxon and round, both from the SplitMix64
// generator of Steele, Lea, Flood, OOPSLA 2014), so a column differing in one taxon
// never collides; all columns equal in content share every round's hash and slot,
// so they are resolved together, to their first occurrence.
#include <algorithm>
#include <climits>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/h3g.h"

namespace h3g {

cudaStream_t ctx_stream(h3g_ctx* ctx);                        // h3g_capi.cu
int ctx_device(h3g_ctx* ctx);
h3g_status ctx_fail(h3g_ctx* ctx, h3g_status st, const std::string& msg);
void*& ctx_compress_scratch(h3g_ctx* ctx);

namespace {

constexpr uint16_t kResolved = 0x8000;
constexpr int kTile = 32;                 // columns and taxa per translate tile
constexpr int kTilesPerBlock = 4;         // column tiles a translate block walks (amortises its table loads)
constexpr int kMaxRounds = 4096;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per codon position p and character (host_pos_tables), fields that add without
// carries over the three characters of a codon: bits 0-5 the unambiguous codon index
// 16 n0 + 4 n1 + n2 (this position's part), bits 8-9 the number of unambiguous
// characters, bits 12-23 the IUPAC sets (position 0 in 20-23 ... 2 in 12-15, the
// index of the ambiguity table), bits 28-29 the number of '!'.  Nucleotide counts are
// 10-bit fields of two words, field 4 p + n (0-5 in lo, 6-11 in hi); per unambiguous
// codon both increments come from one table.
struct Tables {
    const uint32_t* pos;      // [3][256]
    const int8_t* sense;      // [64]
    const uint64_t* inc;      // [64][2] count increments of an unambiguous codon (lo, hi)
    const uint16_t* cid;      // [4096] key of three IUPAC sets
    const uint64_t* z;        // [4096 + 64] random value per key (4096 + s for the sense codon s)
    uint16_t all_id;          // key of the set of every sense codon
};

__device__ __forceinline__ int zindex(uint16_t key) { return (key & 0x8000) ? 4096 + (key & 63) : key; }
__device__ __forceinline__ uint64_t salt_of(uint64_t seed, uint64_t t) { return mix64(seed + t) | 1ull; }

constexpr int kStrip = 3 * kTile * kTilesPerBlock;       // characters of a row a block translates (384)
constexpr int kStripBytes = kStrip + 16;                  // staged from its 16-byte-aligned start (400)

__global__ void __launch_bounds__(256) k_translate(const unsigned char* __restrict__ seqs, size_t stride, int T, int C,
                                                   const unsigned char* __restrict__ seqs_end, Tables tb, uint64_t seed,
                                                   uint16_t* __restrict__ keys, uint64_t* __restrict__ hash,
                                                   unsigned long long* __restrict__ counts) {
    __shared__ __align__(16) unsigned char raw[kTile][kStripBytes];   // the block's strip of each taxon's row
    __shared__ uint16_t ks[kTile][kTile + 2];              // [column][taxon] of the current tile
    __shared__ uint64_t hp[8][kTile];                      // per warp, per column: hash over the warp's taxa
    __shared__ uint32_t pos[3][256];
    __shared__ uint64_t inc[64][2];
    __shared__ int8_t sense[64];
    __shared__ unsigned int cnt[12];
    __shared__ int off[kTile];                             // where each row's strip starts in raw
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int t0 = blockIdx.y * kTile, nt = min(kTile, T - t0);
    const int cb0 = blockIdx.x * kTilesPerBlock * kTile;
    const int nbytes = 3 * min(kTile * kTilesPerBlock, C - cb0);
#pragma unroll
    for (int p = 0; p < 3; ++p) pos[p][tid] = tb.pos[p * 256 + tid];
    if (tid < 128) inc[tid >> 1][tid & 1] = tb.inc[tid];
    if (tid < 64) sense[tid] = tb.sense[tid];
    if (tid < 12) cnt[tid] = 0;
    if (tid < kTile) off[tid] = int(reinterpret_cast<uintptr_t>(seqs + size_t(t0 + min(tid, nt - 1)) * stride + 3 * size_t(cb0)) & 15);
    __syncthreads();
    // stage the strips: 16-byte loads from each row's aligned start; a chunk that would leave the
    // input buffer is read byte by byte within the row's strip
    for (int e = tid; e < kTile * (kStripBytes / 16); e += 256) {
        const int r = e / (kStripBytes / 16), k = e - r * (kStripBytes / 16);
        if (r >= nt) continue;
        const unsigned char* p0 = seqs + size_t(t0 + r) * stride + 3 * size_t(cb0);
        const unsigned char* a = p0 - off[r] + 16 * k;
        if (16 * k >= off[r] + nbytes) continue;           // past this row's strip
        uint4 v;
        if (a >= seqs && a + 16 <= seqs_end) {
            v = __ldg(reinterpret_cast<const uint4*>(a));
        } else {
            unsigned char b[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const unsigned char* q = a + i;
                b[i] = (q >= p0 && q < p0 + nbytes) ? __ldg(q) : 0;
            }
            memcpy(&v, b, 16);
        }
        *reinterpret_cast<uint4*>(&raw[r][16 * k]) = v;
    }
    uint64_t salt[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) salt[k] = salt_of(seed, uint64_t(t0 + warp + 8 * k));
    uint64_t clo = 0, chi = 0;                             // 10-bit nucleotide counters
    __syncthreads();
    for (int tile = 0; tile < kTilesPerBlock; ++tile) {
        const int c0 = cb0 + tile * kTile;
        if (c0 >= C) break;
        const int ncol = min(kTile, C - c0);
        const bool col_ok = lane < ncol;
        uint64_t h = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {                      // taxon warp + 8 k, codon c0 + lane
            const int r = warp + 8 * k;
            uint16_t key = 0;
            if (col_ok && r < nt) {
                const unsigned char* q = &raw[r][off[r] + 3 * (tile * kTile + lane)];
                const uint32_t u0 = pos[0][q[0]], u1 = pos[1][q[1]], u2 = pos[2][q[2]];
                const uint32_t S = u0 + u1 + u2;
                if (((S >> 8) & 3) == 3) {                 // three unambiguous nucleotides
                    const int ci = int(S & 63);
                    const int sv = sense[ci];
                    key = sv >= 0 ? uint16_t(kResolved | sv) : tb.all_id;   // a stop: every sense codon
                    clo += inc[ci][0];
                    chi += inc[ci][1];
                } else {
                    key = (S >> 28) ? tb.all_id : __ldg(tb.cid + ((S >> 12) & 4095));   // '!', or the ambiguity table
                    const uint32_t u[3] = {u0, u1, u2};
#pragma unroll
                    for (int p = 0; p < 3; ++p)            // the unambiguous characters among them
                        if (u[p] & 0x100) {
                            const int f = 4 * p + int((u[p] >> (4 - 2 * p)) & 3);
                            if (f < 6) clo += uint64_t(1) << (10 * f);
                            else chi += uint64_t(1) << (10 * (f - 6));
                        }
                }
                h += __ldg(tb.z + zindex(key)) * salt[k];
            }
            ks[lane][r] = key;
        }
        hp[warp][lane] = h;
        __syncthreads();
        if (tid < kTile && tid < ncol) {
            uint64_t t = 0;
#pragma unroll
            for (int w = 0; w < 8; ++w) t += hp[w][tid];
            atomicAdd(reinterpret_cast<unsigned long long*>(hash + c0 + tid), (unsigned long long)t);
        }
        for (int j = warp; j < ncol; j += 8)               // column-major stores, lane = taxon
            if (lane < nt) keys[size_t(c0 + j) * T + t0 + lane] = ks[j][lane];
        __syncthreads();                                   // ks / hp are rewritten by the next tile
    }
    // counts: per warp (10-bit fields hold at most 32 lanes x 16 codons), then per block
    for (int o = 16; o > 0; o >>= 1) {
        clo += __shfl_xor_sync(0xffffffffu, clo, o);
        chi += __shfl_xor_sync(0xffffffffu, chi, o);
    }
    if (lane == 0)
        for (int f = 0; f < 12; ++f) {
            const unsigned x = unsigned(((f < 6 ? clo : chi) >> (10 * (f < 6 ? f : f - 6))) & 0x3ff);
            if (x) atomicAdd(&cnt[f], x);
        }
    __syncthreads();
    if (tid < 12 && cnt[tid]) atomicAdd(counts + tid, (unsigned long long)cnt[tid]);
}

// one warp per listed column: its hash under a new seed, from the stored keys
__global__ void __launch_bounds__(256) k_rehash(const uint16_t* __restrict__ keys, int T, const int* __restrict__ list, int n,
                                                const uint64_t* __restrict__ z, uint64_t seed, uint64_t* __restrict__ hash) {
    const int lane = threadIdx.x & 31;
    const int i = int((size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    const int c = list[i];
    uint64_t h = 0;
    for (int t = lane; t < T; t += 32) h += __ldg(z + zindex(keys[size_t(c) * T + t])) * salt_of(seed, uint64_t(t));
    h = warp_sum_u64(h);
    if (lane == 0) hash[c] = h;
}

// list == nullptr: columns 0..n-1
__global__ void k_insert(const uint64_t* __restrict__ hash, const int* __restrict__ list, int n, uint64_t hmask,
                         uint64_t* __restrict__ tkey, int* __restrict__ tfirst, uint64_t tmask, int* __restrict__ slot_of) {
    const int i = int(size_t(blockIdx.x) * blockDim.x + threadIdx.x);
    if (i >= n) return;
    const int c = list ? list[i] : i;
    uint64_t h = hash[c] & hmask;
    if (h == 0) h = 1;                                     // 0 marks an empty slot
    uint64_t s = mix64(h) & tmask;
    for (uint64_t probe = 0; probe <= tmask; ++probe) {    // the table holds at least twice the columns
        const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(tkey + s), 0ull, (unsigned long long)h);
        if (prev == 0ull || prev == h) {
            atomicMin(tfirst + s, c);
            slot_of[c] = int(s);
            return;
        }
        s = (s + 1) & tmask;
    }
}

// one warp per listed column: equal to its slot's smallest column -> resolved, else to the next list
__global__ void __launch_bounds__(256) k_verify(const uint16_t* __restrict__ keys, int T, const int* __restrict__ list, int n,
                                                const int* __restrict__ tfirst, const int* __restrict__ slot_of,
                                                int* __restrict__ rep, int* __restrict__ next, int* __restrict__ n_next) {
    const int lane = threadIdx.x & 31;
    const int i = int((size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    const int c = list ? list[i] : i;
    const int r = tfirst[slot_of[c]];
    bool same = true;
    if (r != c)                                            // warp-uniform; every lane takes every step
        for (int t0 = 0; t0 < T; t0 += 32) {
            const int t = t0 + lane;
            const bool eq = t >= T || keys[size_t(c) * T + t] == keys[size_t(r) * T + t];
            if (!__all_sync(0xffffffffu, eq)) {
                same = false;
                break;
            }
        }
    if (lane == 0) {
        if (same) {
            rep[c] = r;
        } else {
            next[atomicAdd(n_next, 1)] = c;
        }
    }
}

__global__ void k_rep_flags(const int* __restrict__ rep, int C, int* __restrict__ flags) {
    const int c = int(size_t(blockIdx.x) * blockDim.x + threadIdx.x);
    if (c < C) flags[c] = rep[c] == c ? 1 : 0;
}

// exclusive scan of 1024-element blocks; block totals to sums
__global__ void __launch_bounds__(1024) k_scan_block(const int* __restrict__ in, int* __restrict__ out, int n, int* __restrict__ sums) {
    __shared__ int wsum[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i = blockIdx.x * 1024 + tid;
    const int v = i < n ? in[i] : 0;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        wsum[lane] = w;
    }
    __syncthreads();
    const int before = (warp > 0 ? wsum[warp - 1] : 0) + x - v;
    if (i < n) out[i] = before;
    if (tid == 1023) sums[blockIdx.x] = wsum[31];
}

__global__ void k_scan_add(int* __restrict__ out, int n, const int* __restrict__ offsets) {
    const int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < n) out[i] += offsets[blockIdx.x];
}

__global__ void k_total(const int* __restrict__ in, const int* __restrict__ ex, int n, long long* __restrict__ total) {
    *total = (long long)ex[n - 1] + in[n - 1];
}

__global__ void k_assign(const int* __restrict__ rep, const int* __restrict__ pid, int C, int* __restrict__ s2p,
                         int* __restrict__ weight, int* __restrict__ first) {
    const int c = int(size_t(blockIdx.x) * blockDim.x + threadIdx.x);
    if (c >= C) return;
    const int r = rep[c], p = pid[r];
    s2p[c] = p;
    atomicAdd(weight + p, 1);
    if (r == c) first[p] = c;
}

// one warp per pattern: its representative column's keys as states and masks
__global__ void __launch_bounds__(256) k_gather(const uint16_t* __restrict__ keys, int T, const int* __restrict__ first, int P,
                                                const uint64_t* __restrict__ set_of, int8_t* __restrict__ states,
                                                uint64_t* __restrict__ masks) {
    const int lane = threadIdx.x & 31;
    const int p = int((size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (p >= P) return;
    const int r = first[p];
    for (int t = lane; t < T; t += 32) {
        const uint16_t k = keys[size_t(r) * T + t];
        const bool res = (k & kResolved) != 0;
        states[size_t(p) * T + t] = res ? int8_t(k & 0x3f) : int8_t(-1);
        masks[size_t(p) * T + t] = res ? (uint64_t(1) << (k & 0x3f)) : __ldg(set_of + k);
    }
}

// ------------------------------------------------------------------ host

// genetic_code.hpp: IUPAC sets over A C G T (U = T), anything else every nucleotide
uint8_t iupac(unsigned char ch) {
    switch (ch >= 'a' && ch <= 'z' ? ch - 32 : ch) {
        case 'A': return 1; case 'C': return 2; case 'G': return 4; case 'T': case 'U': return 8;
        case 'R': return 1 | 4; case 'Y': return 2 | 8; case 'S': return 2 | 4; case 'W': return 1 | 8;
        case 'K': return 4 | 8; case 'M': return 1 | 2; case 'B': return 2 | 4 | 8; case 'D': return 1 | 4 | 8;
        case 'H': return 1 | 2 | 8; case 'V': return 1 | 2 | 4;
        default: return 15;
    }
}

// [3][256]: see Tables::pos
std::vector<uint32_t> host_pos_tables() {
    std::vector<uint32_t> tab(3 * 256);
    for (int p = 0; p < 3; ++p)
        for (int ch = 0; ch < 256; ++ch) {
            const bool bang = ch == '!';
            const uint8_t m = bang ? 15 : iupac((unsigned char)ch);
            uint32_t v = uint32_t(m) << (20 - 4 * p);
            if (!bang && (m == 1 || m == 2 || m == 4 || m == 8)) v |= (uint32_t(__builtin_ctz(m)) << (4 - 2 * p)) | (1u << 8);
            if (bang) v |= 1u << 28;
            tab[size_t(p) * 256 + size_t(ch)] = v;
        }
    return tab;
}

// [64][2]: count increments (10-bit field 4 p + n; 0-5 in lo, 6-11 in hi) of codon 16 n0 + 4 n1 + n2
std::vector<uint64_t> host_codon_increments() {
    std::vector<uint64_t> inc(128, 0);
    for (int c = 0; c < 64; ++c) {
        const int n[3] = {c >> 4, (c >> 2) & 3, c & 3};
        for (int p = 0; p < 3; ++p) {
            const int f = 4 * p + n[p];
            if (f < 6) inc[size_t(2 * c)] += uint64_t(1) << (10 * f);
            else inc[size_t(2 * c + 1)] += uint64_t(1) << (10 * (f - 6));
        }
    }
    return inc;
}

// random value per key: SplitMix64 outputs, distinct
std::vector<uint64_t> host_zobrist() {
    std::vector<uint64_t> z(4096 + 64);
    uint64_t x = 0x6A09E667F3BCC908ull;
    for (auto& v : z) {
        uint64_t q = (x += 0x9E3779B97F4A7C15ull);
        q = (q ^ (q >> 30)) * 0xBF58476D1CE4E5B9ull;
        q = (q ^ (q >> 27)) * 0x94D049BB133111EBull;
        v = q ^ (q >> 31);
    }
    return z;
}

// compatible sense codons of IUPAC sets (m0, m1, m2): all when the three are every
// nucleotide or when none is a sense codon (genetic_code.hpp:82-109); as key ids into
// the list of distinct sets (id 0 = every sense codon)
void host_sets(const int8_t* sense, uint64_t all, std::vector<uint16_t>* cid, std::vector<uint64_t>* set_of) {
    cid->assign(4096, 0);
    set_of->assign(1, all);
    for (int m = 0; m < 4096; ++m) {
        const int m0 = (m >> 8) & 15, m1 = (m >> 4) & 15, m2 = m & 15;
        uint64_t out = 0;
        for (int c = 0; c < 64; ++c)
            if (((m0 >> (c >> 4)) & 1) && ((m1 >> ((c >> 2) & 3)) & 1) && ((m2 >> (c & 3)) & 1) && sense[c] >= 0)
                out |= uint64_t(1) << sense[c];
        if ((m0 == 15 && m1 == 15 && m2 == 15) || out == 0) out = all;
        size_t id = 0;
        while (id < set_of->size() && (*set_of)[id] != out) ++id;
        if (id == set_of->size()) set_of->push_back(out);
        (*cid)[size_t(m)] = uint16_t(id);
    }
}

struct Scratch {
    int device = -1;
    size_t cap_cells = 0, cap_cols = 0, cap_table = 0, cap_seq = 0, cap_out = 0, cap_out_cols = 0;
    uint16_t* keys = nullptr;
    uint16_t* cid = nullptr;
    uint64_t *hash = nullptr, *tkey = nullptr, *set_of = nullptr;
    int *tfirst = nullptr, *slot_of = nullptr, *rep = nullptr, *list_a = nullptr, *list_b = nullptr, *flags = nullptr,
        *pid = nullptr, *scan_tmp = nullptr, *n_next = nullptr;
    uint32_t* pos = nullptr;
    uint64_t* inc = nullptr;
    uint64_t* z = nullptr;
    int8_t* sense = nullptr;
    unsigned long long* counts = nullptr;
    long long* total = nullptr;
    unsigned char* seqs = nullptr;                          // host-memory entry: staged input
    int *s2p = nullptr, *weight = nullptr, *first = nullptr; // host-memory entry: staged outputs
    int8_t* pst = nullptr;
    uint64_t* pmk = nullptr;
    int8_t code_sense[64] = {};
    int code_S = -1;
    void* pinned = nullptr;                                 // [n_next | total | counts]
    cudaEvent_t ev[5] = {};                                 // stage boundaries when profiling
    std::vector<void*> owned;
    ~Scratch() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        for (void* p : owned) cudaFree(p);
        if (pinned) cudaFreeHost(pinned);
    }
};

// (re)allocate p for n elements, releasing what it held
template <class T>
bool alloc_to(Scratch* s, T*& p, size_t n) {
    if (p) {
        auto it = std::find(s->owned.begin(), s->owned.end(), static_cast<void*>(p));
        if (it != s->owned.end()) s->owned.erase(it);
        cudaFree(p);
        p = nullptr;
    }
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return false;
    s->owned.push_back(q);
    p = static_cast<T*>(q);
    return true;
}

Scratch* scratch_for(h3g_ctx* ctx) {
    void*& slot = ctx_compress_scratch(ctx);
    if (!slot) {
        auto* s = new (std::nothrow) Scratch;
        if (!s) return nullptr;
        s->device = ctx_device(ctx);
        if (cudaMallocHost(&s->pinned, 16 * sizeof(long long)) != cudaSuccess) { delete s; return nullptr; }
        void* q = nullptr;
        bool ok = true;
        auto take = [&](size_t bytes) -> void* {
            if (!ok || cudaMalloc(&q, bytes) != cudaSuccess) { ok = false; return nullptr; }
            s->owned.push_back(q);
            return q;
        };
        s->pos = static_cast<uint32_t*>(take(3 * 256 * sizeof(uint32_t)));
        s->inc = static_cast<uint64_t*>(take(128 * sizeof(uint64_t)));
        s->z = static_cast<uint64_t*>(take((4096 + 64) * sizeof(uint64_t)));
        s->sense = static_cast<int8_t*>(take(64));
        s->cid = static_cast<uint16_t*>(take(4096 * sizeof(uint16_t)));
        s->set_of = static_cast<uint64_t*>(take(4097 * sizeof(uint64_t)));
        s->counts = static_cast<unsigned long long*>(take(12 * sizeof(unsigned long long)));
        s->total = static_cast<long long*>(take(sizeof(long long)));
        s->n_next = static_cast<int*>(take(sizeof(int)));
        if (!ok) { delete s; return nullptr; }
        const std::vector<uint32_t> pos = host_pos_tables();
        const std::vector<uint64_t> inc = host_codon_increments(), z = host_zobrist();
        if (cudaMemcpy(s->pos, pos.data(), pos.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(s->inc, inc.data(), inc.size() * sizeof(uint64_t), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(s->z, z.data(), z.size() * sizeof(uint64_t), cudaMemcpyHostToDevice) != cudaSuccess ||
            // a copy from pageable memory may return before its DMA lands, and the kernels run on a
            // non-blocking stream that does not wait for the default stream
            cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess) {
            delete s;
            return nullptr;
        }
        slot = s;
    }
    return static_cast<Scratch*>(slot);
}

// exclusive scan of n ints on the stream; levels[k] holds the block sums of level k
bool scan(const int* in, int* out, int n, std::vector<int*>& tmp, size_t level, cudaStream_t st, int* launches) {
    const int nb = (n + 1023) / 1024;
    int* sums = tmp[level];
    int* sums_ex = tmp[level] + nb;
    k_scan_block<<<nb, 1024, 0, st>>>(in, out, n, sums);
    ++*launches;
    if (nb > 1) {
        if (!scan(sums, sums_ex, nb, tmp, level + 1, st, launches)) return false;
        k_scan_add<<<nb, 1024, 0, st>>>(out, n, sums_ex);
        ++*launches;
    }
    return cudaGetLastError() == cudaSuccess;
}

h3g_status run(h3g_ctx* ctx, Scratch* s, int T, int64_t n_nuc, const unsigned char* d_seqs, size_t stride, const h3g_genetic_code* code,
               int* d_s2p, int* d_weight, int* d_first, int8_t* d_states, uint64_t* d_masks, h3g_compress_info* info) {
    cudaStream_t st = ctx_stream(ctx);
    const int C = int(n_nuc / 3);
    // genetic code tables (re-uploaded when the code changes)
    uint64_t all = code->S >= 64 ? ~uint64_t(0) : ((uint64_t(1) << code->S) - 1);
    if (s->code_S != code->S || std::memcmp(s->code_sense, code->codon_to_sense, 64) != 0) {
        std::vector<uint16_t> cid;
        std::vector<uint64_t> set_of;
        host_sets(code->codon_to_sense, all, &cid, &set_of);
        if (cudaMemcpyAsync(s->sense, code->codon_to_sense, 64, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(s->cid, cid.data(), 4096 * sizeof(uint16_t), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(s->set_of, set_of.data(), set_of.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return ctx_fail(ctx, H3G_ERR_CUDA, "alignment compression: genetic code upload failed");
        std::memcpy(s->code_sense, code->codon_to_sense, 64);
        s->code_S = code->S;
    }
    // working sets
    size_t table = 1;
    while (table < 2 * size_t(C)) table <<= 1;
    std::vector<size_t> lv;                                // scan levels: block sums (and their scans)
    for (size_t n = size_t(C); n > 1024; n = (n + 1023) / 1024) lv.push_back(2 * ((n + 1023) / 1024));
    lv.push_back(2);
    size_t scan_need = 0;
    for (size_t x : lv) scan_need += x;
    const size_t cells = size_t(C) * size_t(T);
    bool ok = true;
    if (s->cap_cells < cells) {
        s->cap_cells = 0;
        ok = alloc_to(s, s->keys, cells);
        if (ok) s->cap_cells = cells;
    }
    if (ok && s->cap_cols < size_t(C)) {
        s->cap_cols = 0;
        ok = alloc_to(s, s->hash, size_t(C)) && alloc_to(s, s->slot_of, size_t(C)) && alloc_to(s, s->rep, size_t(C)) &&
             alloc_to(s, s->list_a, size_t(C)) && alloc_to(s, s->list_b, size_t(C)) && alloc_to(s, s->flags, size_t(C)) &&
             alloc_to(s, s->pid, size_t(C)) && alloc_to(s, s->scan_tmp, scan_need + 64);
        if (ok) s->cap_cols = size_t(C);
    }
    if (ok && s->cap_table < table) {
        s->cap_table = 0;
        ok = alloc_to(s, s->tkey, table) && alloc_to(s, s->tfirst, table);
        if (ok) s->cap_table = table;
    }
    if (!ok) return ctx_fail(ctx, H3G_ERR_OOM, "alignment compression: device allocation failed");
    std::vector<int*> tmp;
    {
        int* p = s->scan_tmp;
        for (size_t x : lv) { tmp.push_back(p); p += x; }
    }
    const Tables tb{s->pos, s->sense, s->inc, s->cid, s->z, 0};
    const bool prof = info->profile != 0;
    if (prof && !s->ev[0])
        for (auto& e : s->ev)
            if (cudaEventCreate(&e) != cudaSuccess) return ctx_fail(ctx, H3G_ERR_CUDA, "alignment compression: event creation failed");
    auto mark = [&](int k) {
        if (prof) cudaEventRecord(s->ev[k], st);
    };
    const uint64_t hmask = (info->hash_bits <= 0 || info->hash_bits >= 64) ? ~uint64_t(0) : ((uint64_t(1) << info->hash_bits) - 1);
    // translate, hash, count
    bool cu = cudaMemsetAsync(s->hash, 0, size_t(C) * sizeof(uint64_t), st) == cudaSuccess &&
              cudaMemsetAsync(s->counts, 0, 12 * sizeof(unsigned long long), st) == cudaSuccess;
    const dim3 tg((C + kTile * kTilesPerBlock - 1) / (kTile * kTilesPerBlock), (T + kTile - 1) / kTile);
    int launches = 0;
    mark(0);
    const unsigned char* seqs_end = d_seqs + size_t(T - 1) * stride + size_t(n_nuc);
    k_translate<<<tg, 256, 0, st>>>(d_seqs, stride, T, C, seqs_end, tb, 0x243F6A8885A308D3ull, s->keys, s->hash, s->counts);
    ++launches;
    mark(1);
    // rounds: insert the unresolved columns, keep those equal to their slot's smallest column
    auto* pin = static_cast<long long*>(s->pinned);
    int* list = nullptr;                                   // nullptr: every column
    int n_list = C, rounds = 0;
    int* lists[2] = {s->list_a, s->list_b};
    while (cu && n_list > 0) {
        if (++rounds > kMaxRounds) return ctx_fail(ctx, H3G_ERR_NUMERIC, "alignment compression: column hashes did not separate");
        if (rounds > 1) {
            k_rehash<<<(n_list + 7) / 8, 256, 0, st>>>(s->keys, T, list, n_list, s->z,
                                                      0x243F6A8885A308D3ull + 0x9E3779B97F4A7C15ull * rounds, s->hash);
            ++launches;
        }
        cu = cudaMemsetAsync(s->tkey, 0, table * sizeof(uint64_t), st) == cudaSuccess &&
             cudaMemsetAsync(s->tfirst, 0x7f, table * sizeof(int), st) == cudaSuccess &&
             cudaMemsetAsync(s->n_next, 0, sizeof(int), st) == cudaSuccess;
        int* next = lists[rounds & 1];
        k_insert<<<(n_list + 255) / 256, 256, 0, st>>>(s->hash, list, n_list, hmask, s->tkey, s->tfirst, uint64_t(table - 1), s->slot_of);
        k_verify<<<(n_list + 7) / 8, 256, 0, st>>>(s->keys, T, list, n_list, s->tfirst, s->slot_of, s->rep, next, s->n_next);
        launches += 2;
        cu = cu && cudaMemcpyAsync(pin, s->n_next, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
             cudaStreamSynchronize(st) == cudaSuccess;
        if (!cu) break;
        n_list = int(*reinterpret_cast<int*>(pin));
        list = next;
    }
    if (!cu) return ctx_fail(ctx, H3G_ERR_CUDA, std::string("alignment compression: ") + cudaGetErrorString(cudaGetLastError()));
    // pattern numbers in first-site order
    mark(2);
    k_rep_flags<<<(C + 255) / 256, 256, 0, st>>>(s->rep, C, s->flags);
    if (!scan(s->flags, s->pid, C, tmp, 0, st, &launches))
        return ctx_fail(ctx, H3G_ERR_CUDA, "alignment compression: scan launch failed");
    k_total<<<1, 1, 0, st>>>(s->flags, s->pid, C, s->total);
    launches += 2;
    mark(3);
    cu = cudaMemcpyAsync(pin + 1, s->total, sizeof(long long), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaMemcpyAsync(pin + 2, s->counts, 12 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaStreamSynchronize(st) == cudaSuccess;
    if (!cu) return ctx_fail(ctx, H3G_ERR_CUDA, std::string("alignment compression: ") + cudaGetErrorString(cudaGetLastError()));
    const int P = int(pin[1]);
    cu = cudaMemsetAsync(d_weight, 0, size_t(P) * sizeof(int), st) == cudaSuccess;
    int* first = d_first ? d_first : s->flags;             // the flags are no longer needed
    k_assign<<<(C + 255) / 256, 256, 0, st>>>(s->rep, s->pid, C, d_s2p, d_weight, first);
    k_gather<<<(P + 7) / 8, 256, 0, st>>>(s->keys, T, first, P, s->set_of, d_states, d_masks);
    launches += 2;
    info->launches = launches;
    mark(4);
    if (!cu || cudaGetLastError() != cudaSuccess)
        return ctx_fail(ctx, H3G_ERR_CUDA, std::string("alignment compression: ") + cudaGetErrorString(cudaGetLastError()));
    for (double& x : info->stage_ms) x = 0.0;
    if (prof) {
        if (cudaEventSynchronize(s->ev[4]) != cudaSuccess)
            return ctx_fail(ctx, H3G_ERR_CUDA, "alignment compression: event synchronisation failed");
        for (int k = 0; k < 4; ++k) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, s->ev[k], s->ev[k + 1]);
            info->stage_ms[k] = ms;
        }
    }
    info->n_patterns = P;
    for (int k = 0; k < 12; ++k) info->pos_counts[k] = pin[2 + k];
    info->rounds = rounds;
    return H3G_OK;
}

h3g_status check_args(h3g_ctx* ctx, int n_taxa, int64_t n_nuc, const void* seqs, size_t row_stride, const h3g_genetic_code* code,
                      const void* s2p, const void* w, const void* st, const void* mk, const h3g_compress_info* info) {
    if (!ctx) return H3G_ERR_ARG;
    if (!seqs || !code || !code->codon_to_sense || !s2p || !w || !st || !mk || !info)
        return ctx_fail(ctx, H3G_ERR_ARG, "alignment compression: null argument");
    if (n_taxa < 1 || n_nuc < 3 || n_nuc % 3 != 0 || row_stride < size_t(n_nuc))
        return ctx_fail(ctx, H3G_ERR_ARG, "alignment compression: needs taxa, a positive multiple of 3 nucleotides and row_stride >= n_nuc");
    if (n_nuc / 3 > int64_t(INT_MAX / 2) || int64_t(n_taxa) * (n_nuc / 3) > (int64_t(1) << 40))
        return ctx_fail(ctx, H3G_ERR_ARG, "alignment compression: alignment too large");
    if (code->S < 1 || code->S > 63) return ctx_fail(ctx, H3G_ERR_ARG, "alignment compression: the code needs 1..63 sense codons");
    int seen = 0;
    for (int c = 0; c < 64; ++c) {
        if (code->codon_to_sense[c] < -1 || code->codon_to_sense[c] >= code->S)
            return ctx_fail(ctx, H3G_ERR_ARG, "alignment compression: codon_to_sense out of range");
        seen += code->codon_to_sense[c] >= 0;
    }
    if (seen != code->S) return ctx_fail(ctx, H3G_ERR_ARG, "alignment compression: codon_to_sense must list S sense codons");
    return H3G_OK;
}

}  // namespace

void compress_scratch_free(void* p) { delete static_cast<Scratch*>(p); }

}  // namespace h3g

using namespace h3g;

extern "C" h3g_status h3g_alignment_compress_device(h3g_ctx* ctx, int n_taxa, int64_t n_nuc, const char* d_seqs, size_t row_stride,
                                                    const h3g_genetic_code* code, int32_t* d_site_to_pattern,
                                                    int32_t* d_pattern_weight, int32_t* d_pattern_first_site,
                                                    int8_t* d_pattern_states, uint64_t* d_pattern_masks, h3g_compress_info* info) {
    const h3g_status a = check_args(ctx, n_taxa, n_nuc, d_seqs, row_stride, code, d_site_to_pattern, d_pattern_weight,
                                    d_pattern_states, d_pattern_masks, info);
    if (a != H3G_OK) return a;
    if (cudaSetDevice(ctx_device(ctx)) != cudaSuccess) return ctx_fail(ctx, H3G_ERR_CUDA, "alignment compression: no device");
    Scratch* s = scratch_for(ctx);
    if (!s) return ctx_fail(ctx, H3G_ERR_OOM, "alignment compression: scratch allocation failed");
    return run(ctx, s, n_taxa, n_nuc, reinterpret_cast<const unsigned char*>(d_seqs), row_stride, code, d_site_to_pattern,
               d_pattern_weight, d_pattern_first_site, d_pattern_states, d_pattern_masks, info);
}

extern "C" h3g_status h3g_alignment_compress(h3g_ctx* ctx, int n_taxa, int64_t n_nuc, const char* seqs, size_t row_stride,
                                             const h3g_genetic_code* code, int32_t* site_to_pattern, int32_t* pattern_weight,
                                             int32_t* pattern_first_site, int8_t* pattern_states, uint64_t* pattern_masks,
                                             h3g_compress_info* info) {
    const h3g_status a = check_args(ctx, n_taxa, n_nuc, seqs, row_stride, code, site_to_pattern, pattern_weight, pattern_states,
                                    pattern_masks, info);
    if (a != H3G_OK) return a;
    if (cudaSetDevice(ctx_device(ctx)) != cudaSuccess) return ctx_fail(ctx, H3G_ERR_CUDA, "alignment compression: no device");
    Scratch* s = scratch_for(ctx);
    if (!s) return ctx_fail(ctx, H3G_ERR_OOM, "alignment compression: scratch allocation failed");
    cudaStream_t st = ctx_stream(ctx);
    const size_t C = size_t(n_nuc / 3), T = size_t(n_taxa);
    // staged input ([taxa][n_nuc], packed) and outputs sized for C patterns
    bool ok = true;
    if (s->cap_seq < T * size_t(n_nuc)) {
        s->cap_seq = 0;
        ok = alloc_to(s, s->seqs, T * size_t(n_nuc));
        if (ok) s->cap_seq = T * size_t(n_nuc);
    }
    if (ok && (s->cap_out < C * T || s->cap_out_cols < C)) {
        s->cap_out = s->cap_out_cols = 0;
        ok = alloc_to(s, s->s2p, C) && alloc_to(s, s->weight, C) && alloc_to(s, s->first, C) && alloc_to(s, s->pst, C * T) &&
             alloc_to(s, s->pmk, C * T);
        if (ok) {
            s->cap_out = C * T;
            s->cap_out_cols = C;
        }
    }
    if (!ok) return ctx_fail(ctx, H3G_ERR_OOM, "alignment compression: device allocation failed");
    if (cudaMemcpy2DAsync(s->seqs, size_t(n_nuc), seqs, row_stride, size_t(n_nuc), T, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return ctx_fail(ctx, H3G_ERR_CUDA, "alignment compression: input copy failed");
    const h3g_status r = run(ctx, s, n_taxa, n_nuc, s->seqs, size_t(n_nuc), code, s->s2p, s->weight, s->first, s->pst, s->pmk, info);
    if (r != H3G_OK) return r;
    const size_t P = size_t(info->n_patterns);
    const bool cu =
        cudaMemcpyAsync(site_to_pattern, s->s2p, C * sizeof(int32_t), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
        cudaMemcpyAsync(pattern_weight, s->weight, P * sizeof(int32_t), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
        (!pattern_first_site ||
         cudaMemcpyAsync(pattern_first_site, s->first, P * sizeof(int32_t), cudaMemcpyDeviceToHost, st) == cudaSuccess) &&
        cudaMemcpyAsync(pattern_states, s->pst, P * T, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
        cudaMemcpyAsync(pattern_masks, s->pmk, P * T * sizeof(uint64_t), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
        cudaStreamSynchronize(st) == cudaSuccess;
    if (!cu) return ctx_fail(ctx, H3G_ERR_CUDA, std::string("alignment compression: ") + cudaGetErrorString(cudaGetLastError()));
    return H3G_OK;
}
