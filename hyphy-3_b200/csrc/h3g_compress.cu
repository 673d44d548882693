// h3g_compress.cu — Alignment::finalize's codon translation, nucleotide counts
// and site-pattern compression on the device (h3g_alignment_compress*).
//
// The reference translates every (taxon, codon) on the host and inserts each
// codon column, as a vector of (state, mask) pairs, into an unordered_map in
// column order (include/hyphy/core/alignment.hpp:665-722, :1021-1078).  Here:
//
//   k_translate  grid (columns / 32, taxa / 32), block 256.  A 32-taxon x
//                96-character tile of the [taxa][nucleotides] input is staged
//                in shared memory; each warp translates one codon column of
//                the tile (lane = taxon) to a 64-bit key, writes the keys
//                column-major ([column][taxon], 256 contiguous bytes per warp)
//                and adds the column's hash contribution; unambiguous
//                nucleotides are counted per codon position with warp ballots.
//   k_insert     one thread per unresolved column: open addressing on the
//                column hash, the slot keeps its smallest column (atomicMin).
//   k_verify     one warp per unresolved column: full comparison with its
//                slot's smallest column; equal columns are resolved, the
//                others (hash collisions) go to the next round with a new seed.
//   scan         representatives (columns resolved to themselves) numbered in
//                column order = the reference's first-occurrence order.
//   k_assign / k_gather   site -> pattern, weights, pattern-major states/masks.
//
// Key of a cell: the mask of compatible sense codons, with bit 63 set when the
// codon is unambiguous (state s, mask 1 << s); with at most 63 sense codons this
// encodes (state, mask) exactly.  A column's hash is the sum over taxa of
// mix(key xor mix(seed + taxon)), mix the SplitMix64 finaliser (Steele, Lea,
// Flood, OOPSLA 2014); all columns equal in content share every round's hash
// and slot, so they are resolved together, to their first occurrence.
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

constexpr uint64_t kResolved = uint64_t(1) << 63;
constexpr int kTile = 32;                 // columns and taxa per translate tile
constexpr int kRowBytes = 100;            // 96 characters, padded: row i starts at bank 25 i mod 32
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

// Character classes (bits 0-3 IUPAC set over A C G T, bit 4 '!', bit 7 an unambiguous
// nucleotide, bits 5-6 its index); see host_char_classes.
struct Tables {
    const uint8_t* cls;       // [256]
    const int8_t* sense;      // [64]
    const uint64_t* amb;      // [4096] compatible sense codons of three IUPAC sets
    uint64_t all;             // every sense codon
};

__global__ void __launch_bounds__(256) k_translate(const unsigned char* __restrict__ seqs, size_t stride, int T, int C,
                                                   Tables tb, uint64_t seed, uint64_t* __restrict__ keys,
                                                   uint64_t* __restrict__ hash, unsigned long long* __restrict__ counts) {
    __shared__ unsigned char raw[kTile][kRowBytes];
    __shared__ uint8_t cls[256];
    __shared__ int8_t sense[64];
    __shared__ unsigned int cnt[12];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int c0 = blockIdx.x * kTile, t0 = blockIdx.y * kTile;
    const int ncol = min(kTile, C - c0), nt = min(kTile, T - t0);
    cls[tid] = tb.cls[tid];
    if (tid < 64) sense[tid] = tb.sense[tid];
    if (tid < 12) cnt[tid] = 0;
    for (int e = tid; e < kTile * 3 * kTile; e += 256) {
        const int r = e / (3 * kTile), b = e - r * (3 * kTile);
        unsigned char v = 0;
        if (r < nt && b < 3 * ncol) v = seqs[size_t(t0 + r) * stride + 3 * size_t(c0) + b];
        raw[r][b] = v;
    }
    __syncthreads();
    const bool valid_t = lane < nt;
    const uint64_t salt = mix64(seed + uint64_t(t0 + lane));
    for (int j = warp; j < ncol; j += 8) {
        const uint8_t a0 = cls[raw[lane][3 * j]], a1 = cls[raw[lane][3 * j + 1]], a2 = cls[raw[lane][3 * j + 2]];
        uint64_t key;
        if (a0 & a1 & a2 & 0x80) {                         // three unambiguous nucleotides
            const int s = sense[16 * ((a0 >> 5) & 3) + 4 * ((a1 >> 5) & 3) + ((a2 >> 5) & 3)];
            key = s >= 0 ? (kResolved | (uint64_t(1) << s)) : tb.all;   // a stop: every sense codon
        } else if ((a0 | a1 | a2) & 0x10) {               // '!'
            key = tb.all;
        } else {
            key = tb.amb[((a0 & 15) << 8) | ((a1 & 15) << 4) | (a2 & 15)];
        }
        // nucleotide counts per codon position (ballots over the warp's valid taxa)
#pragma unroll
        for (int p = 0; p < 3; ++p) {
            const uint8_t a = p == 0 ? a0 : (p == 1 ? a1 : a2);
            const int nuc = (valid_t && (a & 0x80)) ? ((a >> 5) & 3) : -1;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const unsigned m = __ballot_sync(0xffffffffu, nuc == b);
                if (lane == 0 && m) atomicAdd(&cnt[4 * p + b], unsigned(__popc(m)));
            }
        }
        const size_t col = size_t(c0 + j);
        if (valid_t) keys[col * T + t0 + lane] = key;
        const uint64_t h = warp_sum_u64(valid_t ? mix64(key ^ salt) : 0ull);
        if (lane == 0) atomicAdd(reinterpret_cast<unsigned long long*>(hash + col), (unsigned long long)h);
    }
    __syncthreads();
    if (tid < 12 && cnt[tid]) atomicAdd(counts + tid, (unsigned long long)cnt[tid]);
}

// one warp per listed column: its hash under a new seed, from the stored keys
__global__ void __launch_bounds__(256) k_rehash(const uint64_t* __restrict__ keys, int T, const int* __restrict__ list, int n,
                                                uint64_t seed, uint64_t* __restrict__ hash) {
    const int lane = threadIdx.x & 31;
    const int i = int((size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    const int c = list[i];
    uint64_t h = 0;
    for (int t = lane; t < T; t += 32) h += mix64(keys[size_t(c) * T + t] ^ mix64(seed + uint64_t(t)));
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
__global__ void __launch_bounds__(256) k_verify(const uint64_t* __restrict__ keys, int T, const int* __restrict__ list, int n,
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
__global__ void __launch_bounds__(256) k_gather(const uint64_t* __restrict__ keys, int T, const int* __restrict__ first, int P,
                                                int8_t* __restrict__ states, uint64_t* __restrict__ masks) {
    const int lane = threadIdx.x & 31;
    const int p = int((size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (p >= P) return;
    const int r = first[p];
    for (int t = lane; t < T; t += 32) {
        const uint64_t k = keys[size_t(r) * T + t], m = k & ~kResolved;
        states[size_t(p) * T + t] = (k & kResolved) ? int8_t(__ffsll((long long)m) - 1) : int8_t(-1);
        masks[size_t(p) * T + t] = m;
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

std::vector<uint8_t> host_char_classes() {
    std::vector<uint8_t> cls(256);
    for (int ch = 0; ch < 256; ++ch) {
        uint8_t m = iupac((unsigned char)ch), v = m;
        if (m == 1 || m == 2 || m == 4 || m == 8) v |= uint8_t(0x80 | ((__builtin_ctz(m) & 3) << 5));
        if (ch == '!') v = 0x10 | 15;
        cls[size_t(ch)] = v;
    }
    return cls;
}

// compatible sense codons of IUPAC sets (m0, m1, m2): all when the three are every
// nucleotide or when none is a sense codon (genetic_code.hpp:82-109)
std::vector<uint64_t> host_ambiguity(const int8_t* sense, uint64_t all) {
    std::vector<uint64_t> amb(4096);
    for (int m = 0; m < 4096; ++m) {
        const int m0 = (m >> 8) & 15, m1 = (m >> 4) & 15, m2 = m & 15;
        uint64_t out = 0;
        for (int c = 0; c < 64; ++c)
            if (((m0 >> (c >> 4)) & 1) && ((m1 >> ((c >> 2) & 3)) & 1) && ((m2 >> (c & 3)) & 1) && sense[c] >= 0)
                out |= uint64_t(1) << sense[c];
        amb[size_t(m)] = (m0 == 15 && m1 == 15 && m2 == 15) || out == 0 ? all : out;
    }
    return amb;
}

struct Scratch {
    int device = -1;
    size_t cap_cells = 0, cap_cols = 0, cap_table = 0, cap_seq = 0, cap_out = 0, cap_out_cols = 0;
    uint64_t *keys = nullptr, *hash = nullptr, *tkey = nullptr, *amb = nullptr;
    int *tfirst = nullptr, *slot_of = nullptr, *rep = nullptr, *list_a = nullptr, *list_b = nullptr, *flags = nullptr,
        *pid = nullptr, *scan_tmp = nullptr, *n_next = nullptr;
    uint8_t* cls = nullptr;
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
    std::vector<void*> owned;
    ~Scratch() {
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
        s->cls = static_cast<uint8_t*>(take(256));
        s->sense = static_cast<int8_t*>(take(64));
        s->amb = static_cast<uint64_t*>(take(4096 * sizeof(uint64_t)));
        s->counts = static_cast<unsigned long long*>(take(12 * sizeof(unsigned long long)));
        s->total = static_cast<long long*>(take(sizeof(long long)));
        s->n_next = static_cast<int*>(take(sizeof(int)));
        if (!ok) { delete s; return nullptr; }
        const std::vector<uint8_t> cls = host_char_classes();
        if (cudaMemcpy(s->cls, cls.data(), 256, cudaMemcpyHostToDevice) != cudaSuccess) { delete s; return nullptr; }
        slot = s;
    }
    return static_cast<Scratch*>(slot);
}

// exclusive scan of n ints on the stream; levels[k] holds the block sums of level k
bool scan(const int* in, int* out, int n, std::vector<int*>& tmp, size_t level, cudaStream_t st) {
    const int nb = (n + 1023) / 1024;
    int* sums = tmp[level];
    int* sums_ex = tmp[level] + nb;
    k_scan_block<<<nb, 1024, 0, st>>>(in, out, n, sums);
    if (nb > 1) {
        if (!scan(sums, sums_ex, nb, tmp, level + 1, st)) return false;
        k_scan_add<<<nb, 1024, 0, st>>>(out, n, sums_ex);
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
        const std::vector<uint64_t> amb = host_ambiguity(code->codon_to_sense, all);
        if (cudaMemcpyAsync(s->sense, code->codon_to_sense, 64, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(s->amb, amb.data(), 4096 * sizeof(uint64_t), cudaMemcpyHostToDevice, st) != cudaSuccess ||
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
    const Tables tb{s->cls, s->sense, s->amb, all};
    const uint64_t hmask = (info->hash_bits <= 0 || info->hash_bits >= 64) ? ~uint64_t(0) : ((uint64_t(1) << info->hash_bits) - 1);
    // translate, hash, count
    bool cu = cudaMemsetAsync(s->hash, 0, size_t(C) * sizeof(uint64_t), st) == cudaSuccess &&
              cudaMemsetAsync(s->counts, 0, 12 * sizeof(unsigned long long), st) == cudaSuccess;
    const dim3 tg((C + kTile - 1) / kTile, (T + kTile - 1) / kTile);
    k_translate<<<tg, 256, 0, st>>>(d_seqs, stride, T, C, tb, 0x243F6A8885A308D3ull, s->keys, s->hash, s->counts);
    // rounds: insert the unresolved columns, keep those equal to their slot's smallest column
    auto* pin = static_cast<long long*>(s->pinned);
    int* list = nullptr;                                   // nullptr: every column
    int n_list = C, rounds = 0;
    int* lists[2] = {s->list_a, s->list_b};
    while (cu && n_list > 0) {
        if (++rounds > kMaxRounds) return ctx_fail(ctx, H3G_ERR_NUMERIC, "alignment compression: column hashes did not separate");
        if (rounds > 1)
            k_rehash<<<(n_list + 7) / 8, 256, 0, st>>>(s->keys, T, list, n_list, 0x243F6A8885A308D3ull + 0x9E3779B97F4A7C15ull * rounds,
                                                      s->hash);
        cu = cudaMemsetAsync(s->tkey, 0, table * sizeof(uint64_t), st) == cudaSuccess &&
             cudaMemsetAsync(s->tfirst, 0x7f, table * sizeof(int), st) == cudaSuccess &&
             cudaMemsetAsync(s->n_next, 0, sizeof(int), st) == cudaSuccess;
        int* next = lists[rounds & 1];
        k_insert<<<(n_list + 255) / 256, 256, 0, st>>>(s->hash, list, n_list, hmask, s->tkey, s->tfirst, uint64_t(table - 1), s->slot_of);
        k_verify<<<(n_list + 7) / 8, 256, 0, st>>>(s->keys, T, list, n_list, s->tfirst, s->slot_of, s->rep, next, s->n_next);
        cu = cu && cudaMemcpyAsync(pin, s->n_next, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
             cudaStreamSynchronize(st) == cudaSuccess;
        if (!cu) break;
        n_list = int(*reinterpret_cast<int*>(pin));
        list = next;
    }
    if (!cu) return ctx_fail(ctx, H3G_ERR_CUDA, std::string("alignment compression: ") + cudaGetErrorString(cudaGetLastError()));
    // pattern numbers in first-site order
    k_rep_flags<<<(C + 255) / 256, 256, 0, st>>>(s->rep, C, s->flags);
    if (!scan(s->flags, s->pid, C, tmp, 0, st))
        return ctx_fail(ctx, H3G_ERR_CUDA, "alignment compression: scan launch failed");
    k_total<<<1, 1, 0, st>>>(s->flags, s->pid, C, s->total);
    cu = cudaMemcpyAsync(pin + 1, s->total, sizeof(long long), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaMemcpyAsync(pin + 2, s->counts, 12 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaStreamSynchronize(st) == cudaSuccess;
    if (!cu) return ctx_fail(ctx, H3G_ERR_CUDA, std::string("alignment compression: ") + cudaGetErrorString(cudaGetLastError()));
    const int P = int(pin[1]);
    cu = cudaMemsetAsync(d_weight, 0, size_t(P) * sizeof(int), st) == cudaSuccess;
    int* first = d_first ? d_first : s->flags;             // the flags are no longer needed
    k_assign<<<(C + 255) / 256, 256, 0, st>>>(s->rep, s->pid, C, d_s2p, d_weight, first);
    k_gather<<<(P + 7) / 8, 256, 0, st>>>(s->keys, T, first, P, d_states, d_masks);
    if (!cu || cudaGetLastError() != cudaSuccess)
        return ctx_fail(ctx, H3G_ERR_CUDA, std::string("alignment compression: ") + cudaGetErrorString(cudaGetLastError()));
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
