// h3g_noalloc.cu — log-likelihood from caller-supplied transition matrices
// without any device allocation.
//
// Some callers cannot allocate GPU memory while they run: code executing
// inside a framework that owns the whole device pool (a serving process that
// pre-reserves HBM, a host that forbids cudaMalloc after start-up), or code
// that must not introduce allocation-driven synchronisation.  For them
// h3g_eval_from_P_noalloc runs the same inside pass as h3g_eval_from_P, with
// every intermediate (topology tables, padded transition matrices, partial
// likelihoods, scaling exponents, per-pattern terms) carved out of one
// file-scope __device__ array of kNoallocScratchBytes that each GPU loading
// the library holds until the process exits.
//
// Set-up: the first call on a device looks up the device address of that
// array (cudaGetSymbolAddress) with the device current; make that first call
// before any stream capture.  Every call shares the array and it keeps the
// previous call's contents, so calls that overlap on the GPU (two streams, two
// host threads) race and must be serialised by the caller.
#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/h3g.h"
#include "h3g_common.cuh"
#include "h3g_kernels.h"

namespace {

constexpr size_t kNoallocScratchBytes = size_t(32) << 20;   // 32 MiB per device
constexpr int kNoallocMaxNodes = 1024;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Patterns arrive pattern-major [P][T]; the pruning kernels read them
// taxon-major [T][Pp] with the padding columns marked missing.
__global__ void k_noalloc_patterns(const int8_t* st_pm, const uint64_t* mk_pm, int P, int T, int Pp,
                                   int8_t* st, uint64_t* mk) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= size_t(T) * Pp) return;
    const int t = int(i / Pp), p = int(i % Pp);
    st[i] = p < P ? st_pm[size_t(p) * T + t] : int8_t(-1);
    mk[i] = p < P ? mk_pm[size_t(p) * T + t] : ~uint64_t(0);
}

struct Carver {
    unsigned char* base;
    size_t used = 0;
    template <class T> T* take(size_t count) {
        used = (used + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + used);
        used += count * sizeof(T);
        return p;
    }
};

}  // namespace

extern "C" h3g_status h3g_eval_from_P_noalloc(int device, void* cuda_stream, int n_nodes, const int32_t* parent,
                                              const uint8_t* is_leaf, const int32_t* leaf_taxon, int n_taxa,
                                              int n_patterns, const int8_t* states, const uint64_t* masks,
                                              const double* weights, int S, const double* P, const double* pi,
                                              double* lnl, double* site_lnl) {
    using namespace h3g;
    if (device < 0 || device >= kMaxDevices || !parent || !is_leaf || !leaf_taxon || !P || !pi || !lnl) return H3G_ERR_ARG;
    if (n_nodes < 2 || n_nodes > kNoallocMaxNodes || S < 1 || S > SP || n_taxa < 0 || n_patterns < 0) return H3G_ERR_ARG;
    if (n_patterns > 0 && (!states || !masks || !weights)) return H3G_ERR_ARG;
    const int n = n_nodes, T = n_taxa;
    // topology tables on the stack: children CSR in increasing id order, internal
    // slots, heights for the level-synchronous inside pass
    int ch_off[kNoallocMaxNodes + 1], ch[kNoallocMaxNodes], iidx[kNoallocMaxNodes], taxon[kNoallocMaxNodes];
    int order[kNoallocMaxNodes], height[kNoallocMaxNodes], in_nodes[kNoallocMaxNodes], in_off[kNoallocMaxNodes + 1];
    int fill[kNoallocMaxNodes];
    int root = -1, NI = 0;
    std::memset(ch_off, 0, sizeof(int) * (n + 1));
    for (int i = 0; i < n; ++i) {
        const int p = parent[i];
        if (p < 0) { if (root >= 0) return H3G_ERR_ARG; root = i; continue; }
        if (p >= n || p == i || is_leaf[p]) return H3G_ERR_ARG;
        ch_off[p + 1]++;
    }
    if (root < 0 || is_leaf[root]) return H3G_ERR_ARG;
    for (int i = 0; i < n; ++i) { ch_off[i + 1] += ch_off[i]; fill[i] = ch_off[i]; }
    for (int i = 0; i < n; ++i) if (parent[i] >= 0) ch[fill[parent[i]]++] = i;
    int cnt = 0;
    order[cnt++] = root;
    for (int q = 0; q < cnt; ++q)
        for (int k = ch_off[order[q]]; k < ch_off[order[q] + 1]; ++k) {
            if (cnt >= n) return H3G_ERR_ARG;
            order[cnt++] = ch[k];
        }
    if (cnt != n) return H3G_ERR_ARG;
    int H = 0;
    for (int q = n - 1; q >= 0; --q) {
        const int u = order[q];
        height[u] = 0;
        for (int k = ch_off[u]; k < ch_off[u + 1]; ++k) height[u] = std::max(height[u], height[ch[k]] + 1);
        if (!is_leaf[u] && ch_off[u] == ch_off[u + 1]) height[u] = 1;
        if (!is_leaf[u]) H = std::max(H, height[u]);
    }
    for (int i = 0; i < n; ++i) {
        iidx[i] = is_leaf[i] ? -1 : NI++;
        taxon[i] = -1;
        if (is_leaf[i]) {
            if (leaf_taxon[i] >= T) return H3G_ERR_ARG;
            taxon[i] = leaf_taxon[i] < 0 ? -1 : leaf_taxon[i];
        }
    }
    int m = 0;
    in_off[0] = 0;
    for (int h = 1; h <= H; ++h) {
        for (int i = 0; i < n; ++i) if (!is_leaf[i] && height[i] == h) in_nodes[m++] = i;
        in_off[h] = m;
    }
    for (size_t k = 0; k < size_t(n_patterns) * T; ++k)
        if (states[k] >= S) return H3G_ERR_ARG;
    for (int p = 0; p < n_patterns; ++p)
        if (!(weights[p] >= 0.0) || !std::isfinite(weights[p])) return H3G_ERR_ARG;
    const int Pp = std::max(TP, (n_patterns + TP - 1) / TP * TP);

    // one-time set-up per device: the device address of the scratch array
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return H3G_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return H3G_ERR_CUDA;
    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[device]) {
            void* addr = nullptr;
            if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr) {
                cudaSetDevice(prev);
                return H3G_ERR_CUDA;
            }
            g_scratch_addr[device] = addr;
            h3g::fp64_configure();   // shared-memory limits of the pruning kernels on this device
        }
        scratch = static_cast<unsigned char*>(g_scratch_addr[device]);
    }

    Carver c{scratch};
    Topo t{};
    Model md{};
    Work w{};
    t.n = n; t.root = root; t.NI = NI; t.T = T; t.P = n_patterns; t.Pp = Pp; t.S = S;
    t.all_mask = S >= 64 ? ~uint64_t(0) : ((uint64_t(1) << S) - 1);
    int* d_ch_off = c.take<int>(n + 1);
    int* d_ch = c.take<int>(std::max(n, 1));
    int* d_iidx = c.take<int>(n);
    int* d_taxon = c.take<int>(n);
    uint8_t* d_leaf = c.take<uint8_t>(n);
    int* d_in_nodes = c.take<int>(std::max(m, 1));
    int8_t* d_st_pm = c.take<int8_t>(std::max<size_t>(size_t(n_patterns) * T, 1));
    uint64_t* d_mk_pm = c.take<uint64_t>(std::max<size_t>(size_t(n_patterns) * T, 1));
    int8_t* d_st = c.take<int8_t>(std::max<size_t>(size_t(T) * Pp, 1));
    uint64_t* d_mk = c.take<uint64_t>(std::max<size_t>(size_t(T) * Pp, 1));
    double* d_w = c.take<double>(Pp);
    double* d_pi = c.take<double>(SP);
    w.P = c.take<double>(size_t(n) * SP2);
    w.PT = c.take<double>(size_t(n) * SP2);
    w.rs = c.take<double>(size_t(n) * SP);
    w.D = c.take<double>(size_t(NI) * SP * Pp);
    w.Ms = c.take<double>(size_t(NI) * SP * Pp);
    w.Ecum = c.take<int>(size_t(NI) * Pp);
    w.Eown = c.take<int>(size_t(NI) * Pp);
    w.f = c.take<double>(Pp);
    w.rw = c.take<double>(Pp);
    w.contrib = c.take<double>(Pp);
    w.site = c.take<double>(Pp);
    w.out = c.take<double>(2 + size_t(n) + 3);
    if (c.used > kNoallocScratchBytes) { cudaSetDevice(prev); return H3G_ERR_ARG; }   // problem exceeds the 32 MiB scratch

    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    ok(cudaMemcpyAsync(d_ch_off, ch_off, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(d_ch, ch, sizeof(int) * std::max(ch_off[n], 1), cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(d_iidx, iidx, sizeof(int) * n, cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(d_taxon, taxon, sizeof(int) * n, cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(d_leaf, is_leaf, n, cudaMemcpyHostToDevice, s));
    if (m > 0) ok(cudaMemcpyAsync(d_in_nodes, in_nodes, sizeof(int) * m, cudaMemcpyHostToDevice, s));
    // the scratch keeps the previous call's contents: zero what is read before written
    ok(cudaMemsetAsync(d_w, 0, sizeof(double) * Pp, s));
    ok(cudaMemsetAsync(d_pi, 0, sizeof(double) * SP, s));
    ok(cudaMemsetAsync(w.P, 0, sizeof(double) * size_t(n) * SP2, s));
    if (n_patterns > 0) {
        ok(cudaMemcpyAsync(d_st_pm, states, size_t(n_patterns) * T, cudaMemcpyHostToDevice, s));
        ok(cudaMemcpyAsync(d_mk_pm, masks, sizeof(uint64_t) * size_t(n_patterns) * T, cudaMemcpyHostToDevice, s));
        ok(cudaMemcpyAsync(d_w, weights, sizeof(double) * n_patterns, cudaMemcpyHostToDevice, s));
    }
    ok(cudaMemcpyAsync(d_pi, pi, sizeof(double) * S, cudaMemcpyHostToDevice, s));
    for (int b = 0; b < n; ++b) {
        if (b == root) continue;
        ok(cudaMemcpy2DAsync(w.P + size_t(b) * SP2, SP * sizeof(double), P + size_t(b) * S * S, S * sizeof(double),
                             S * sizeof(double), S, cudaMemcpyHostToDevice, s));
    }
    if (T > 0) {
        const size_t total = size_t(T) * Pp;
        k_noalloc_patterns<<<unsigned((total + 255) / 256), 256, 0, s>>>(d_st_pm, d_mk_pm, n_patterns, T, Pp, d_st, d_mk);
    }
    t.ch_off = d_ch_off; t.ch = d_ch; t.iidx = d_iidx; t.leaf = d_leaf; t.taxon = d_taxon;
    t.states = d_st; t.masks = d_mk; t.w = d_w;
    md.M = 1; md.K = 1; md.nmod = 1; md.sentinel = 1; md.pi = d_pi;
    launch_prep_given_P(t, w, s);
    for (int h = 0; h < H; ++h) {
        const int k = in_off[h + 1] - in_off[h];
        if (k) launch_inside_fp64(t, md, w, d_in_nodes + in_off[h], k, s);
    }
    launch_root(t, md, w, s);
    launch_small(t, md, w, 0, s);
    ok(cudaGetLastError());
    ok(cudaMemcpyAsync(lnl, w.out, sizeof(double), cudaMemcpyDeviceToHost, s));
    if (site_lnl && n_patterns > 0) ok(cudaMemcpyAsync(site_lnl, w.site, sizeof(double) * n_patterns, cudaMemcpyDeviceToHost, s));
    ok(cudaStreamSynchronize(s));
    cudaSetDevice(prev);
    return e == cudaSuccess ? H3G_OK : H3G_ERR_CUDA;
}
