// h3_oracle.hpp — CPU oracle for the MG94xREV codon likelihood core.
//
// TEST INFRASTRUCTURE ONLY.  This is a plain FP64 restatement of the
// reference engine (veg/hyphy-3, header-only C++ with Eigen) written without
// Eigen, used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
// leg as the checker.  The product library never links or calls it.
//
// Every function cites the reference file:line it restates.  Parity is pinned
// against the reference's own known answers (tests/golden/): the MG94 point
// log-likelihood on cd2_reduced (benchmarks/ground_truth/
// cd2_reduced_point_truth.json, asserted in tests/test_core.cpp:95-124), the
// alignment statistics asserted in tests/test_core.cpp:12-37, and the finite
// difference gradient tests (tests/test_core.cpp:149-223,
// tests/test_cpp_autograd.cpp:47-104).
#pragma once

#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <limits>
#include <list>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace h3o {

// ---------------------------------------------------------------- matrices
struct Mat {
    int r = 0, c = 0;
    std::vector<double> a;
    Mat() = default;
    Mat(int r_, int c_, double v = 0.0) : r(r_), c(c_), a(size_t(r_) * c_, v) {}
    double& operator()(int i, int j) { return a[size_t(i) * c + j]; }
    double operator()(int i, int j) const { return a[size_t(i) * c + j]; }
    static Mat eye(int n) { Mat m(n, n); for (int i = 0; i < n; ++i) m(i, i) = 1.0; return m; }
};

inline Mat matmul(const Mat& A, const Mat& B) {
    Mat C(A.r, B.c);
    for (int i = 0; i < A.r; ++i)
        for (int k = 0; k < A.c; ++k) {
            double a = A(i, k);
            if (a == 0.0) continue;
            const double* b = &B.a[size_t(k) * B.c];
            double* c = &C.a[size_t(i) * C.c];
            for (int j = 0; j < B.c; ++j) c[j] += a * b[j];
        }
    return C;
}
inline Mat transpose(const Mat& A) {
    Mat T(A.c, A.r);
    for (int i = 0; i < A.r; ++i) for (int j = 0; j < A.c; ++j) T(j, i) = A(i, j);
    return T;
}
// y = A x
inline void matvec(const Mat& A, const double* x, double* y) {
    for (int i = 0; i < A.r; ++i) {
        const double* row = &A.a[size_t(i) * A.c];
        double s = 0.0;
        for (int j = 0; j < A.c; ++j) s += row[j] * x[j];
        y[i] = s;
    }
}
// y = A^T x
inline void matvec_t(const Mat& A, const double* x, double* y) {
    for (int j = 0; j < A.c; ++j) y[j] = 0.0;
    for (int i = 0; i < A.r; ++i) {
        const double* row = &A.a[size_t(i) * A.c];
        double xi = x[i];
        for (int j = 0; j < A.c; ++j) y[j] += row[j] * xi;
    }
}

// Neumaier compensated summation (likelihood.hpp:33-51).
struct Neumaier {
    double s = 0.0, c = 0.0;
    void add(double x) {
        double t = s + x;
        if (std::fabs(s) >= std::fabs(x)) c += (s - t) + x; else c += (x - t) + s;
        s = t;
    }
    double value() const { return s + c; }
};

// ------------------------------------------------------------ genetic code
// Nucleotide coding A=0 C=1 G=2 T=3 (types.hpp:34-43).
inline int nuc_index(char ch) {
    switch (ch) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': case 'U': case 'u': return 3;
        default: return -1;
    }
}
// IUPAC bitmask A=1 C=2 G=4 T=8 (types.hpp:47-67).
inline unsigned iupac_bits(char ch) {
    switch (std::toupper(static_cast<unsigned char>(ch))) {
        case 'A': return 1; case 'C': return 2; case 'G': return 4; case 'T': case 'U': return 8;
        case 'R': return 5; case 'Y': return 10; case 'S': return 6; case 'W': return 9;
        case 'K': return 12; case 'M': return 3; case 'B': return 14; case 'D': return 13;
        case 'H': return 11; case 'V': return 7;
        default: return 15;
    }
}

// Sense-codon table and codon-pair difference records (genetic_code.hpp:127-200).
struct Code {
    std::string name;
    int S = 0;
    char aa[64];        // amino acid of codon index 16*n1+4*n2+n3, '*' for stop
    int sense[64];      // codon index -> sense index or -1
    int codon[64];      // sense index -> codon index
    struct Diff { int nd = 0; bool syn = false; int pos[3] = {-1, -1, -1}, from[3] = {-1, -1, -1}, to[3] = {-1, -1, -1}; };
    std::vector<Diff> diff; // S*S, row-major [from][to]

    // Standard code (NCBI table 1) as amino-acid letters in TCAG-major codon order,
    // the order in which the table is conventionally printed.
    static Code make(const std::string& which) {
        static const char* tcag = "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG";
        static const int to_tcag[4] = {2, 1, 3, 0}; // A C G T -> position in T C A G
        Code c;
        c.name = which;
        for (int n1 = 0; n1 < 4; ++n1) for (int n2 = 0; n2 < 4; ++n2) for (int n3 = 0; n3 < 4; ++n3)
            c.aa[16 * n1 + 4 * n2 + n3] = tcag[16 * to_tcag[n1] + 4 * to_tcag[n2] + to_tcag[n3]];
        auto set = [&](const char* trip, char a) {
            c.aa[16 * nuc_index(trip[0]) + 4 * nuc_index(trip[1]) + nuc_index(trip[2])] = a;
        };
        std::string w = which;
        std::transform(w.begin(), w.end(), w.begin(), ::tolower);
        if (w == "universal" || w == "standard" || w == "1") {
        } else if (w == "vertebrate-mtdna" || w == "vertebrate_mtdna" || w == "2") {
            set("AGA", '*'); set("AGG", '*'); set("ATA", 'M'); set("TGA", 'W');
        } else {
            throw std::runtime_error("oracle: unsupported genetic code " + which);
        }
        int s = 0;
        for (int i = 0; i < 64; ++i) {
            c.codon[i] = -1;
            if (c.aa[i] == '*') { c.sense[i] = -1; continue; }
            c.sense[i] = s; c.codon[s] = i; ++s;
        }
        c.S = s;
        c.diff.assign(size_t(s) * s, Diff{});
        for (int u = 0; u < s; ++u) for (int v = 0; v < s; ++v) {
            if (u == v) continue;
            Diff& d = c.diff[size_t(u) * s + v];
            int cu = c.codon[u], cv = c.codon[v];
            for (int p = 0; p < 3; ++p) {
                int sh = 2 * (2 - p);
                int a = (cu >> sh) & 3, b = (cv >> sh) & 3;
                if (a != b) { d.pos[d.nd] = p; d.from[d.nd] = a; d.to[d.nd] = b; ++d.nd; }
            }
            d.syn = (c.aa[cu] == c.aa[cv]);
        }
        return c;
    }
    const Diff& df(int u, int v) const { return diff[size_t(u) * S + v]; }
    uint64_t all_sense() const { return S >= 64 ? ~uint64_t(0) : ((uint64_t(1) << S) - 1); }
    int triplet_sense(char a, char b, char c3) const {
        int x = nuc_index(a), y = nuc_index(b), z = nuc_index(c3);
        if (x < 0 || y < 0 || z < 0) return -1;
        return sense[16 * x + 4 * y + z];
    }
    // genetic_code.hpp:82-109
    uint64_t triplet_mask(char a, char b, char c3) const {
        if (a == '!' || b == '!' || c3 == '!') return all_sense();
        unsigned m1 = iupac_bits(a), m2 = iupac_bits(b), m3 = iupac_bits(c3);
        if (m1 == 15 && m2 == 15 && m3 == 15) return all_sense();
        uint64_t m = 0;
        for (int i = 0; i < 4; ++i) if (m1 >> i & 1)
            for (int j = 0; j < 4; ++j) if (m2 >> j & 1)
                for (int k = 0; k < 4; ++k) if (m3 >> k & 1) {
                    int s = sense[16 * i + 4 * j + k];
                    if (s >= 0) m |= uint64_t(1) << s;
                }
        return m ? m : all_sense();
    }
    int codon_nuc(int s, int pos) const { return (codon[s] >> (2 * (2 - pos))) & 3; }
};

// --------------------------------------------------------------- alignment
struct Alignment {
    std::vector<std::string> names;
    std::vector<std::string> seqs;
    std::string embedded_tree;
    Code code;
    int n_codons = 0;
    // pattern store: states[p * T + t], masks[p * T + t]
    int T = 0, P = 0;
    std::vector<int8_t> states;
    std::vector<uint64_t> masks;
    std::vector<double> weights;
    std::vector<int> site_pattern;    // alignment.hpp site_to_pattern
    double nuc_freq[4] = {0, 0, 0, 0};
    double pos_freq[3][4] = {};   // CF3x4-corrected (alignment.hpp:1017)
    std::vector<double> pi;       // codon_frequencies_f3x4

    // alignment.hpp:665-723 (finalize) + :893-1019 (frequencies) + :1021-1078 (patterns)
    void finalize(const std::string& code_name = "Universal") {
        code = Code::make(code_name);
        if (seqs.empty()) throw std::runtime_error("Empty alignment");
        T = int(seqs.size());
        size_t L = seqs[0].size();
        for (auto& s : seqs) if (s.size() != L) throw std::runtime_error("Sequences have unequal lengths in alignment");
        if (L % 3) throw std::runtime_error("Nucleotide alignment length is not a multiple of 3");
        n_codons = int(L / 3);
        std::vector<int8_t> cs(size_t(T) * n_codons);
        std::vector<uint64_t> cm(size_t(T) * n_codons);
        for (int t = 0; t < T; ++t) for (int c = 0; c < n_codons; ++c) {
            const char* x = &seqs[t][3 * c];
            int s = code.triplet_sense(x[0], x[1], x[2]);
            cs[size_t(t) * n_codons + c] = int8_t(s);
            cm[size_t(t) * n_codons + c] = s >= 0 ? (uint64_t(1) << s) : code.triplet_mask(x[0], x[1], x[2]);
        }
        frequencies();
        // first-occurrence pattern order
        std::map<std::pair<std::vector<int8_t>, std::vector<uint64_t>>, int> seen;
        states.clear(); masks.clear(); weights.clear(); site_pattern.clear(); P = 0;
        std::vector<int8_t> ks(T); std::vector<uint64_t> km(T);
        for (int c = 0; c < n_codons; ++c) {
            for (int t = 0; t < T; ++t) { ks[t] = cs[size_t(t) * n_codons + c]; km[t] = cm[size_t(t) * n_codons + c]; }
            auto key = std::make_pair(ks, km);
            auto it = seen.find(key);
            if (it == seen.end()) {
                site_pattern.push_back(P);
                seen.emplace(key, P++);
                states.insert(states.end(), ks.begin(), ks.end());
                masks.insert(masks.end(), km.begin(), km.end());
                weights.push_back(1.0);
            } else {
                site_pattern.push_back(it->second);
                weights[it->second] += 1.0;
            }
        }
    }

    void frequencies() {
        double nc[4] = {0, 0, 0, 0}, pc[3][4] = {};
        for (auto& s : seqs)
            for (int c = 0; c < n_codons; ++c)
                for (int p = 0; p < 3; ++p) {
                    int n = nuc_index(s[3 * c + p]);
                    if (n >= 0) { nc[n] += 1; pc[p][n] += 1; }
                }
        double tot = nc[0] + nc[1] + nc[2] + nc[3];
        if (tot > 0) for (int b = 0; b < 4; ++b) nuc_freq[b] = nc[b] / tot;
        bool pad = false;
        for (int b = 0; b < 4; ++b) if (nuc_freq[b] < 1e-8) { nuc_freq[b] = 1e-8; pad = true; }
        if (pad) { double z = nuc_freq[0] + nuc_freq[1] + nuc_freq[2] + nuc_freq[3]; for (int b = 0; b < 4; ++b) nuc_freq[b] /= z; }
        double emp[3][4] = {};
        for (int p = 0; p < 3; ++p) {
            double z = pc[p][0] + pc[p][1] + pc[p][2] + pc[p][3];
            if (z > 0) for (int b = 0; b < 4; ++b) emp[p][b] = pc[p][b] / z;
            bool pd = false;
            for (int b = 0; b < 4; ++b) if (emp[p][b] < 1e-8) { emp[p][b] = 1e-8; pd = true; }
            if (pd) { double s = emp[p][0] + emp[p][1] + emp[p][2] + emp[p][3]; for (int b = 0; b < 4; ++b) emp[p][b] /= s; }
        }
        // CF3x4 fixed point (alignment.hpp:962-1018)
        const int S = code.S;
        pi.assign(S, 0.0);
        double cur[3][4];
        std::copy(&emp[0][0], &emp[0][0] + 12, &cur[0][0]);
        auto product_freqs = [&]() {
            double z = 0;
            for (int s = 0; s < S; ++s) {
                pi[s] = cur[0][code.codon_nuc(s, 0)] * cur[1][code.codon_nuc(s, 1)] * cur[2][code.codon_nuc(s, 2)];
                z += pi[s];
            }
            if (z > 0) for (int s = 0; s < S; ++s) pi[s] /= z;
        };
        for (int it = 0; it < 200; ++it) {
            double prev[3][4];
            std::copy(&cur[0][0], &cur[0][0] + 12, &prev[0][0]);
            product_freqs();
            double q[3][4] = {};
            for (int s = 0; s < S; ++s) for (int p = 0; p < 3; ++p) q[p][code.codon_nuc(s, p)] += pi[s];
            for (int p = 0; p < 3; ++p) {
                for (int b = 0; b < 4; ++b) cur[p][b] *= emp[p][b] / std::max(q[p][b], 1e-12);
                double z = cur[p][0] + cur[p][1] + cur[p][2] + cur[p][3];
                if (z > 0) for (int b = 0; b < 4; ++b) cur[p][b] /= z;
            }
            double d = 0;
            for (int p = 0; p < 3; ++p) for (int b = 0; b < 4; ++b) d = std::max(d, std::fabs(cur[p][b] - prev[p][b]));
            if (d < 1e-14) break;
        }
        product_freqs();
        std::copy(&cur[0][0], &cur[0][0] + 12, &pos_freq[0][0]);
    }
};

inline std::string read_text(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("Could not open alignment file: " + path);
    std::stringstream ss; ss << f.rdbuf();
    return ss.str();
}

// FASTA: '>' header lines, sequence lines concatenated with whitespace removed.
inline Alignment parse_fasta(const std::string& text) {
    Alignment a;
    std::string line; std::istringstream in(text);
    int cur = -1;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) continue;
        if (line[0] == '>') {
            std::string nm = line.substr(1);
            while (!nm.empty() && std::isspace(static_cast<unsigned char>(nm.back()))) nm.pop_back();
            size_t b = 0; while (b < nm.size() && std::isspace(static_cast<unsigned char>(nm[b]))) ++b;
            a.names.push_back(nm.substr(b)); a.seqs.emplace_back(); cur = int(a.seqs.size()) - 1;
        } else if (cur >= 0) {
            for (char ch : line) if (!std::isspace(static_cast<unsigned char>(ch))) a.seqs[cur] += ch;
        }
    }
    return a;
}

// Minimal NEXUS reader: TAXLABELS, MATRIX (sequential or interleaved) and the first TREE.
inline Alignment parse_nexus(const std::string& raw) {
    // strip [...] comments
    std::string t; t.reserve(raw.size());
    int depth = 0; char q = 0;
    for (char ch : raw) {
        if (q) { t += ch; if (ch == q) q = 0; continue; }
        if (depth == 0 && (ch == '\'' || ch == '"')) { q = ch; t += ch; continue; }
        if (ch == '[') { ++depth; continue; }
        if (ch == ']' && depth > 0) { --depth; continue; }
        if (depth == 0) t += (ch == '\r') ? '\n' : ch;
    }
    auto upper = [](std::string s) { for (auto& ch : s) ch = char(std::toupper(static_cast<unsigned char>(ch))); return s; };
    std::string T = upper(t);
    Alignment a;
    auto unq = [](std::string s) {
        if (s.size() >= 2 && (s[0] == '\'' || s[0] == '"') && s.back() == s[0]) s = s.substr(1, s.size() - 2);
        return s;
    };
    auto tokens = [&](const std::string& body) {
        std::vector<std::pair<std::string, bool>> out; // token, starts_line
        size_t i = 0; bool nl = true;
        while (i < body.size()) {
            char ch = body[i];
            if (ch == '\n') { nl = true; ++i; continue; }
            if (std::isspace(static_cast<unsigned char>(ch))) { ++i; continue; }
            std::string tok;
            if (ch == '\'' || ch == '"') {
                char qq = ch; tok += ch; ++i;
                while (i < body.size() && body[i] != qq) tok += body[i++];
                if (i < body.size()) tok += body[i++];
            } else {
                while (i < body.size() && !std::isspace(static_cast<unsigned char>(body[i]))) tok += body[i++];
            }
            out.push_back({tok, nl}); nl = false;
        }
        return out;
    };
    std::vector<std::string> labels;
    size_t tl = T.find("TAXLABELS");
    if (tl != std::string::npos) {
        size_t e = T.find(';', tl);
        for (auto& tk : tokens(t.substr(tl + 9, e - tl - 9))) labels.push_back(unq(tk.first));
    }
    size_t mx = T.find("MATRIX");
    if (mx == std::string::npos) throw std::runtime_error("NEXUS: no MATRIX");
    size_t me = t.find(';', mx);
    auto toks = tokens(t.substr(mx + 6, me - mx - 6));
    std::unordered_map<std::string, int> idx;
    for (auto& l : labels) { idx[l] = int(a.names.size()); a.names.push_back(l); a.seqs.emplace_back(); }
    int cur = -1;
    for (auto& [tok, starts] : toks) {
        std::string u = unq(tok);
        auto it = idx.find(u);
        bool is_name = labels.empty() ? starts : (it != idx.end());
        if (is_name) {
            if (it == idx.end()) { idx[u] = int(a.names.size()); a.names.push_back(u); a.seqs.emplace_back(); it = idx.find(u); }
            cur = it->second;
        } else if (cur >= 0) {
            a.seqs[cur] += tok;
        }
    }
    size_t tr = T.find("BEGIN TREES");
    if (tr != std::string::npos) {
        size_t k = T.find("TREE ", tr + 11);
        if (k != std::string::npos) {
            size_t eq = t.find('=', k);
            size_t sc = t.find(';', eq);
            std::string nw = t.substr(eq + 1, sc - eq - 1);
            size_t b = 0; while (b < nw.size() && std::isspace(static_cast<unsigned char>(nw[b]))) ++b;
            a.embedded_tree = nw.substr(b) + ";";
        }
    }
    return a;
}

inline Alignment load_alignment(const std::string& path, const std::string& code_name = "Universal") {
    std::string txt = read_text(path);
    size_t b = 0; while (b < txt.size() && std::isspace(static_cast<unsigned char>(txt[b]))) ++b;
    Alignment a = (txt.compare(b, 6, "#NEXUS") == 0 || txt.compare(b, 6, "#nexus") == 0) ? parse_nexus(txt) : parse_fasta(txt);
    a.finalize(code_name);
    return a;
}

// -------------------------------------------------------------------- tree
// Node ids follow the reference parser's creation order: '(' opens an
// internal node, a label before ',' or ')' creates a leaf (tree.hpp:273-585).
struct Tree {
    std::vector<int> parent;
    std::vector<std::vector<int>> children;
    std::vector<std::string> name;
    std::vector<double> bl;
    std::vector<char> leaf;
    std::vector<int> post;
    int root = -1;
    int n() const { return int(parent.size()); }

    int add() { parent.push_back(-1); children.emplace_back(); name.emplace_back(); bl.push_back(0.0); leaf.push_back(0); return n() - 1; }
    void label(int id, std::string tok) {
        size_t lb = tok.find('{'), rb = tok.find('}');
        if (lb != std::string::npos && rb != std::string::npos && rb > lb) tok.erase(lb, rb - lb + 1);
        size_t col = std::string::npos; char q = 0;
        for (size_t k = 0; k < tok.size(); ++k) {
            char ch = tok[k];
            if (q) { if (ch == q) q = 0; continue; }
            if (ch == '\'' || ch == '"') { q = ch; continue; }
            if (ch == ':') { col = k; break; }
        }
        std::string nm = col == std::string::npos ? tok : tok.substr(0, col);
        if (col != std::string::npos) { try { bl[id] = std::stod(tok.substr(col + 1)); } catch (...) { bl[id] = 0.0; } }
        if (nm.size() >= 2 && (nm[0] == '\'' || nm[0] == '"') && nm.back() == nm[0]) nm = nm.substr(1, nm.size() - 2);
        name[id] = nm;
    }
    static Tree parse(std::string s, bool keep_rooted = true) {
        Tree tr;
        while (!s.empty() && (s.back() == ';' || std::isspace(static_cast<unsigned char>(s.back())))) s.pop_back();
        std::string c; bool cm = false; char q = 0;
        for (char ch : s) {
            if (q) { c += ch; if (ch == q) q = 0; continue; }
            if (cm) { if (ch == ']') cm = false; continue; }
            if (ch == '[') { cm = true; continue; }
            if (ch == '\'' || ch == '"') { q = ch; c += ch; continue; }
            if (!std::isspace(static_cast<unsigned char>(ch))) c += ch;
        }
        std::vector<int> st; std::string tok; q = 0;
        for (size_t i = 0; i < c.size(); ++i) {
            char ch = c[i];
            if (q) { tok += ch; if (ch == q) q = 0; continue; }
            if (ch == '\'' || ch == '"') { q = ch; tok += ch; continue; }
            if (ch == ';') break;
            if (ch == '(') {
                int id = tr.add();
                if (!st.empty()) { tr.children[st.back()].push_back(id); tr.parent[id] = st.back(); }
                st.push_back(id);
            } else if (ch == ',' || ch == ')') {
                if (!tok.empty()) {
                    int id = tr.add(); tr.leaf[id] = 1; tr.label(id, tok); tok.clear();
                    if (!st.empty()) { tr.children[st.back()].push_back(id); tr.parent[id] = st.back(); }
                }
                if (ch == ')') {
                    if (st.empty()) throw std::runtime_error("Invalid Newick tree: unbalanced parentheses");
                    int cur = st.back(); st.pop_back();
                    size_t j = i + 1; std::string it; char iq = 0;
                    while (j < c.size()) {
                        char cj = c[j];
                        if (iq) { it += cj; if (cj == iq) iq = 0; ++j; continue; }
                        if (cj == '\'' || cj == '"') { iq = cj; it += cj; ++j; continue; }
                        if (cj == ',' || cj == ')' || cj == '(' || cj == ';') break;
                        it += cj; ++j;
                    }
                    if (!it.empty()) { tr.label(cur, it); i = j - 1; }
                }
            } else tok += ch;
        }
        if (!st.empty()) throw std::runtime_error("Invalid Newick tree: unbalanced parentheses");
        if (tr.n() == 0) throw std::runtime_error("Failed to parse Newick tree: empty tree");
        for (int i = 0; i < tr.n(); ++i) if (tr.parent[i] < 0) tr.root = i;
        if (!keep_rooted) tr.unroot();
        tr.order();
        return tr;
    }
    void order() {
        post.clear();
        std::vector<std::pair<int, size_t>> stk{{root, 0}};
        while (!stk.empty()) {
            auto& [u, k] = stk.back();
            if (k < children[u].size()) { int c = children[u][k++]; stk.push_back({c, 0}); }
            else { post.push_back(u); stk.pop_back(); }
        }
    }
    // tree.hpp:591-690 (model tags are not tracked by the oracle)
    void unroot() {
        if (root < 0 || n() <= 3 || children[root].size() != 2) return;
        int c0 = children[root][0], c1 = children[root][1], ab, ot;
        if (!leaf[c0]) { ab = c0; ot = c1; } else if (!leaf[c1]) { ab = c1; ot = c0; } else return;
        bl[ot] += bl[ab];
        std::vector<int> nc;
        if (ab == c0) { nc = children[ab]; nc.push_back(ot); } else { nc.push_back(ot); for (int g : children[ab]) nc.push_back(g); }
        children[root] = nc;
        std::vector<int> remap(n(), -1); int k = 0;
        for (int i = 0; i < n(); ++i) if (i != ab) remap[i] = k++;
        Tree t2;
        for (int i = 0; i < n(); ++i) if (i != ab) {
            int id = t2.add(); t2.name[id] = name[i]; t2.bl[id] = bl[i]; t2.leaf[id] = leaf[i];
        }
        t2.root = remap[root];
        for (int i = 0; i < n(); ++i) if (i != ab) for (int cc : children[i]) {
            t2.children[remap[i]].push_back(remap[cc]); t2.parent[remap[cc]] = remap[i];
        }
        t2.parent[t2.root] = -1; t2.bl[t2.root] = 0.0;
        *this = t2;
    }
};

// leaf -> alignment row: exact, case-insensitive, then unique prefix (likelihood.hpp:106-161)
inline std::vector<int> leaf_map(const Tree& tr, const Alignment& a) {
    auto low = [](std::string s) { for (auto& c : s) c = char(std::tolower(static_cast<unsigned char>(c))); return s; };
    std::vector<int> m(tr.n(), -1); int leaves = 0, hit = 0;
    for (int i = 0; i < tr.n(); ++i) {
        if (!tr.leaf[i]) continue;
        ++leaves;
        std::string nm = tr.name[i];
        int f = -1;
        for (size_t t = 0; t < a.names.size(); ++t) if (a.names[t] == nm) { f = int(t); break; }
        if (f < 0) for (size_t t = 0; t < a.names.size(); ++t) if (low(a.names[t]) == low(nm)) { f = int(t); break; }
        if (f < 0 && nm.size() >= 3) {
            int cnt = 0, last = -1; std::string ln = low(nm);
            for (size_t t = 0; t < a.names.size(); ++t) {
                std::string ls = low(a.names[t]);
                if ((ls.size() > ln.size() && ls.compare(0, ln.size(), ln) == 0) ||
                    (ls.size() >= 3 && ln.size() > ls.size() && ln.compare(0, ls.size(), ls) == 0)) { ++cnt; last = int(t); }
            }
            if (cnt == 1) f = last;
        }
        m[i] = f; if (f >= 0) ++hit;
    }
    if (leaves > 0 && hit == 0) throw std::runtime_error("Phylogenetic tree leaves do not match any sequences in alignment!");
    return m;
}

// ----------------------------------------------------------------- MG94xREV
// An eigensystem handed to the oracle instead of its own (U_pi, V_pi, lambda): lets a test
// compare another engine that diagonalises Q with a different solver like with like, the
// eigensolver's own floor being pinned separately.
struct GivenEigen {
    std::vector<double> U, V, lam;     // S x S, S x S (row-major), S
};

struct Params {
    double alpha = 1.0, beta = 1.0;
    double theta[5] = {1, 1, 1, 1, 1}; // AC AT CG CT GT (AG == 1)
    double delta = 0.0, psi = 0.0;
    std::shared_ptr<const GivenEigen> eig;   // null: the oracle's own Jacobi eigensystem
};

inline void nuc_rates(const Params& p, double r[4][4]) {
    const double AC = p.theta[0], AT = p.theta[1], CG = p.theta[2], CT = p.theta[3], GT = p.theta[4];
    double t[4][4] = {{0, AC, 1, AT}, {AC, 0, CG, CT}, {1, CG, 0, GT}, {AT, CT, GT, 0}};
    std::copy(&t[0][0], &t[0][0] + 16, &r[0][0]);
}

// Cyclic Jacobi eigensolver for a symmetric matrix (Golub & Van Loan,
// "Matrix Computations", 4th ed., Alg. 8.5.3 with the threshold strategy).
// On return A's diagonal holds eigenvalues and the columns of V eigenvectors.
inline void jacobi_eigen(Mat A, std::vector<double>& w, Mat& V) {
    const int n = A.r;
    V = Mat::eye(n);
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) { double x = A(i, j) * A(i, j); tot += x; if (i != j) off += x; }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; ++p) for (int q = p + 1; q < n; ++q) {
            double apq = A(p, q);
            if (std::fabs(apq) < 1e-300) continue;
            const double app = A(p, p), aqq = A(q, q);
            double tau = (aqq - app) / (2.0 * apq);
            double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
            double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
            for (int k = 0; k < n; ++k) {
                double akp = A(k, p), akq = A(k, q);
                A(k, p) = c * akp - s * akq; A(k, q) = s * akp + c * akq;
            }
            for (int k = 0; k < n; ++k) {
                double apk = A(p, k), aqk = A(q, k);
                A(p, k) = c * apk - s * aqk; A(q, k) = s * apk + c * aqk;
            }
            for (int k = 0; k < n; ++k) {
                double vkp = V(k, p), vkq = V(k, q);
                V(k, p) = c * vkp - s * vkq; V(k, q) = s * vkp + c * vkq;
            }
            // the rotation annihilates a_pq; set the 2x2 block to its exact values (Alg. 8.5.1)
            A(p, p) = app - t * apq; A(q, q) = aqq + t * apq; A(p, q) = 0.0; A(q, p) = 0.0;
        }
    }
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = A(i, i);
}

struct MG94 {
    int S = 0;
    Mat Q, U, Vp;           // Q, U_pi = D^-1/2 E, V_pi = E^T D^1/2
    std::vector<double> lam, pi;
    double mu = 0.0;        // scale_factor = -sum pi_i Q_ii (stored, not applied)

    // rate_matrix.hpp:165-249
    void update(const Params& p, const double pos[3][4], const std::vector<double>& pi_in, const Code& code) {
        S = code.S; pi = pi_in;
        double r[4][4]; nuc_rates(p, r);
        Q = Mat(S, S);
        for (int i = 0; i < S; ++i) for (int j = 0; j < S; ++j) {
            if (i == j) continue;
            const auto& d = code.df(i, j);
            double rm = d.syn ? p.alpha : p.beta;
            if (d.nd == 1) Q(i, j) = rm * r[d.from[0]][d.to[0]] * pos[d.pos[0]][d.to[0]];
            else if (d.nd == 2 && p.delta > 0)
                Q(i, j) = rm * p.delta * r[d.from[0]][d.to[0]] * r[d.from[1]][d.to[1]] * pos[d.pos[0]][d.to[0]] * pos[d.pos[1]][d.to[1]];
            else if (d.nd == 3 && p.psi > 0)
                Q(i, j) = rm * p.psi * r[d.from[0]][d.to[0]] * r[d.from[1]][d.to[1]] * r[d.from[2]][d.to[2]] *
                          pos[d.pos[0]][d.to[0]] * pos[d.pos[1]][d.to[1]] * pos[d.pos[2]][d.to[2]];
        }
        for (int i = 0; i < S; ++i) { double s = 0; for (int j = 0; j < S; ++j) if (j != i) s += Q(i, j); Q(i, i) = -s; }
        mu = 0; for (int i = 0; i < S; ++i) mu -= pi[i] * Q(i, i);
        std::vector<double> sq(S), isq(S);
        for (int i = 0; i < S; ++i) { sq[i] = std::sqrt(std::max(pi[i], 1e-12)); isq[i] = 1.0 / sq[i]; }
        Mat A(S, S);
        for (int i = 0; i < S; ++i) for (int j = 0; j < S; ++j) A(i, j) = sq[i] * Q(i, j) * isq[j];
        for (int i = 0; i < S; ++i) for (int j = i + 1; j < S; ++j) { double m = 0.5 * (A(i, j) + A(j, i)); A(i, j) = A(j, i) = m; }
        Mat E; jacobi_eigen(A, lam, E);
        for (auto& l : lam) l = std::min(l, 0.0);
        U = Mat(S, S); Vp = Mat(S, S);
        for (int i = 0; i < S; ++i) for (int j = 0; j < S; ++j) { U(i, j) = isq[i] * E(i, j); Vp(j, i) = E(i, j) * sq[i]; }
        if (p.eig) {
            if (p.eig->U.size() != size_t(S) * S || p.eig->V.size() != size_t(S) * S || p.eig->lam.size() != size_t(S))
                throw std::runtime_error("given eigensystem has the wrong size");
            std::copy(p.eig->U.begin(), p.eig->U.end(), U.a.begin());
            std::copy(p.eig->V.begin(), p.eig->V.end(), Vp.a.begin());
            lam = p.eig->lam;
        }
    }
    // rate_matrix.hpp:251-257
    Mat P(double t) const {
        Mat W(S, S);
        for (int i = 0; i < S; ++i) for (int k = 0; k < S; ++k) W(i, k) = U(i, k) * std::exp(lam[k] * t);
        Mat R = matmul(W, Vp);
        for (auto& x : R.a) x = std::max(x, 0.0);
        return R;
    }
};

// d Q / d x as used by the Frechet gradients (likelihood.hpp:1537-1576)
inline Mat dQ_beta(const Params& p, const double pos[3][4], const Code& code) {
    double r[4][4]; nuc_rates(p, r);
    Mat d(code.S, code.S);
    for (int i = 0; i < code.S; ++i) {
        double s = 0;
        for (int j = 0; j < code.S; ++j) {
            if (i == j) continue;
            const auto& df = code.df(i, j);
            if (df.nd == 1 && !df.syn) { d(i, j) = r[df.from[0]][df.to[0]] * pos[df.pos[0]][df.to[0]]; s += d(i, j); }
        }
        d(i, i) = -s;
    }
    return d;
}
inline Mat dQ_theta(int u, int v, double alpha, double beta, const double pos[3][4], const Code& code) {
    Mat d(code.S, code.S);
    for (int i = 0; i < code.S; ++i) {
        double s = 0;
        for (int j = 0; j < code.S; ++j) {
            if (i == j) continue;
            const auto& df = code.df(i, j);
            if (df.nd != 1) continue;
            int f = df.from[0], t = df.to[0];
            if ((f == u && t == v) || (f == v && t == u)) { d(i, j) = (df.syn ? alpha : beta) * pos[df.pos[0]][t]; s += d(i, j); }
        }
        d(i, i) = -s;
    }
    return d;
}
static const int kThetaPairs[5][2] = {{0, 1}, {0, 3}, {1, 2}, {1, 3}, {2, 3}}; // AC AT CG CT GT

// ------------------------------------------------- single-pattern inside-outside
// Per-pattern restatement of the batched two-pass traversal
// (likelihood.hpp:479-762) with the same 1e-150 / 1e150 scaling scheme.
struct Pass {
    std::vector<std::vector<double>> D, V, PD, U;
    std::vector<int> boost;
    std::vector<double> lscale;
    double L = 0, logL = 0;
};

// likelihood.hpp:54-87
inline void leaf_vector(const Alignment& a, int p, int taxon, int S, double* out) {
    if (taxon < 0) { std::fill(out, out + S, 1.0); return; }
    int st = a.states[size_t(p) * a.T + taxon];
    if (st >= 0 && st < S) { std::fill(out, out + S, 0.0); out[st] = 1.0; return; }
    uint64_t m = a.masks[size_t(p) * a.T + taxon];
    const uint64_t all = S >= 64 ? ~uint64_t(0) : ((uint64_t(1) << S) - 1);
    if (m == 0 || (m & all) == all) { std::fill(out, out + S, 1.0); return; }
    for (int s = 0; s < S; ++s) out[s] = (m >> s & 1) ? 1.0 : 0.0;
}

constexpr double kThresh = 1e-150, kUp = 1e150, kDown = 1e-150, kLogScaler = 345.38776394910684;

inline void rescale(double* x, int S, int& count) {
    double mx = *std::max_element(x, x + S);
    while (mx < kThresh && mx > 0.0) { for (int i = 0; i < S; ++i) x[i] *= kUp; mx *= kUp; ++count; }
}

inline void inside_outside(const Tree& tr, const Alignment& a, int p, const std::vector<int>& l2t,
                           const std::vector<Mat>& Pb, const std::vector<double>& pi, int S, Pass& w, bool outside) {
    const int n = tr.n();
    w.D.assign(n, std::vector<double>(S)); w.PD.assign(n, std::vector<double>(S));
    w.boost.assign(n, 0); w.lscale.assign(n, 0.0);
    for (int u : tr.post) {
        if (tr.leaf[u]) { leaf_vector(a, p, l2t[u], S, w.D[u].data()); continue; }
        auto& D = w.D[u];
        std::fill(D.begin(), D.end(), 1.0);
        for (int c : tr.children[u]) {
            matvec(Pb[c], w.D[c].data(), w.PD[c].data());
            for (int i = 0; i < S; ++i) D[i] *= w.PD[c][i];
            w.lscale[u] += w.lscale[c];
            rescale(D.data(), S, w.boost[u]);
        }
        rescale(D.data(), S, w.boost[u]);
        w.lscale[u] -= w.boost[u] * kLogScaler;
    }
    double L = 0; for (int i = 0; i < S; ++i) L += w.D[tr.root][i] * pi[i];
    w.L = L;
    w.logL = L > 0 ? std::log(L) + w.lscale[tr.root] : -1e20;
    if (!outside) return;
    w.U.assign(n, std::vector<double>(S)); w.V.assign(n, std::vector<double>(S));
    w.U[tr.root] = pi;
    for (auto it = tr.post.rbegin(); it != tr.post.rend(); ++it) {
        int u = *it;
        if (tr.leaf[u]) continue;
        const auto& ch = tr.children[u];
        const size_t k = ch.size();
        if (!k) continue;
        std::vector<std::vector<double>> pref(k, std::vector<double>(S, 1.0)), suff(k, std::vector<double>(S, 1.0));
        std::vector<int> pb(k, 0), sb(k, 0);
        for (size_t i = 1; i < k; ++i) {
            for (int s = 0; s < S; ++s) pref[i][s] = pref[i - 1][s] * w.PD[ch[i - 1]][s];
            pb[i] = pb[i - 1]; rescale(pref[i].data(), S, pb[i]);
        }
        for (size_t i = k - 1; i > 0; --i) {
            for (int s = 0; s < S; ++s) suff[i - 1][s] = suff[i][s] * w.PD[ch[i]][s];
            sb[i - 1] = sb[i]; rescale(suff[i - 1].data(), S, sb[i - 1]);
        }
        for (size_t i = 0; i < k; ++i) {
            int c = ch[i];
            auto& Vc = w.V[c];
            for (int s = 0; s < S; ++s) Vc[s] = w.U[u][s] * pref[i][s] * suff[i][s];
            int net = w.boost[u] - pb[i] - sb[i];
            for (; net > 0; --net) for (int s = 0; s < S; ++s) Vc[s] *= kUp;
            for (; net < 0; ++net) for (int s = 0; s < S; ++s) Vc[s] *= kDown;
            matvec_t(Pb[c], Vc.data(), w.U[c].data());
        }
    }
}

// ------------------------------------------------- 64-pattern tile inside-outside
// The reference's batched form (likelihood.hpp:295-340 workspaces, :479-762
// compute_inside_outside_batch_in_place): every node holds S x B matrices for a
// tile of B <= 64 patterns (element (s, b) at s * B + b), the child messages and
// the outside vectors are S x S by S x B products, and the 1e150 rescaling runs
// per column exactly as in the per-pattern form above, so both forms give the
// same numbers (the products sum over k in the same order as matvec / matvec_t).
constexpr int kTile = 64;   // likelihood.hpp:1155 tile_size

struct TilePass {
    int B = 0;
    std::vector<std::vector<double>> D, PD, U, V;   // [node][S * B]
    std::vector<std::vector<int>> boost;            // [node][B]
    std::vector<std::vector<double>> lscale;        // [node][B]
    std::vector<std::vector<double>> pref, suff;    // [child slot][S * B]
    std::vector<std::vector<int>> pb, sb;           // [child slot][B]
    std::vector<double> L, logL;                    // [B]
};

// C = op(A) X with op(A) = A (Trans = false) or A^T, A S x S, X and C S x B: 4 x 4
// register blocks, every entry summed over k = 0, 1, ... from 0.0 (the order of matvec)
template <bool Trans>
inline void gemm_tile_blocked(const Mat& A, const double* X, double* C, int S, int B) {
    auto a_at = [&](int i, int k) { return Trans ? A.a[size_t(k) * A.c + i] : A.a[size_t(i) * A.c + k]; };
    for (int i0 = 0; i0 < S; i0 += 4) {
        const int ni = std::min(4, S - i0);
        for (int b0 = 0; b0 < B; b0 += 4) {
            const int nb = std::min(4, B - b0);
            double acc[4][4] = {{0.0}};
            if (ni == 4 && nb == 4) {
                for (int k = 0; k < S; ++k) {
                    const double* x = X + size_t(k) * B + b0;
                    const double a0 = a_at(i0, k), a1 = a_at(i0 + 1, k), a2 = a_at(i0 + 2, k), a3 = a_at(i0 + 3, k);
                    for (int q = 0; q < 4; ++q) {
                        acc[0][q] += a0 * x[q]; acc[1][q] += a1 * x[q];
                        acc[2][q] += a2 * x[q]; acc[3][q] += a3 * x[q];
                    }
                }
            } else {
                for (int k = 0; k < S; ++k)
                    for (int r = 0; r < ni; ++r) {
                        const double a = a_at(i0 + r, k);
                        for (int q = 0; q < nb; ++q) acc[r][q] += a * X[size_t(k) * B + b0 + q];
                    }
            }
            for (int r = 0; r < ni; ++r)
                for (int q = 0; q < nb; ++q) C[size_t(i0 + r) * B + b0 + q] = acc[r][q];
        }
    }
}
// C = A X  (A S x S, X and C S x B)
inline void gemm_tile(const Mat& A, const double* X, double* C, int S, int B) { gemm_tile_blocked<false>(A, X, C, S, B); }
// C = A^T X
inline void gemm_tile_t(const Mat& A, const double* X, double* C, int S, int B) { gemm_tile_blocked<true>(A, X, C, S, B); }
// A += Y Z^T over the tile (Y, Z S x B): 4 x 4 register blocks summed over b
inline void gemm_tile_acc_nt(const double* Y, const double* Z, Mat& A, int S, int B) {
    for (int i0 = 0; i0 < S; i0 += 4) {
        const int ni = std::min(4, S - i0);
        for (int j0 = 0; j0 < S; j0 += 4) {
            const int nj = std::min(4, S - j0);
            double acc[4][4] = {{0.0}};
            for (int b = 0; b < B; ++b) {
                double y[4], z[4];
                for (int r = 0; r < 4; ++r) y[r] = r < ni ? Y[size_t(i0 + r) * B + b] : 0.0;
                for (int q = 0; q < 4; ++q) z[q] = q < nj ? Z[size_t(j0 + q) * B + b] : 0.0;
                for (int r = 0; r < 4; ++r)
                    for (int q = 0; q < 4; ++q) acc[r][q] += y[r] * z[q];
            }
            for (int r = 0; r < ni; ++r)
                for (int q = 0; q < nj; ++q) A.a[size_t(i0 + r) * A.c + j0 + q] += acc[r][q];
        }
    }
}
// per column: multiply by 1e150 while the column maximum is in (0, 1e-150), counting steps
inline void rescale_cols(double* X, int S, int B, int* count) {
    for (int b = 0; b < B; ++b) {
        double mx = 0.0;
        for (int s = 0; s < S; ++s) mx = std::max(mx, X[size_t(s) * B + b]);
        while (mx < kThresh && mx > 0.0) {
            for (int s = 0; s < S; ++s) X[size_t(s) * B + b] *= kUp;
            mx *= kUp;
            ++count[b];
        }
    }
}

inline void inside_outside_tile(const Tree& tr, const Alignment& a, int p0, int B, const std::vector<int>& l2t,
                                const std::vector<Mat>& Pb, const std::vector<double>& pi, int S, TilePass& w, bool outside) {
    const int n = tr.n();
    const size_t SB = size_t(S) * B;
    if (w.B != B || int(w.D.size()) != n || (w.D.empty() ? 0 : w.D[0].size()) != SB) {
        w.B = B;
        w.D.assign(n, std::vector<double>(SB)); w.PD.assign(n, std::vector<double>(SB));
        w.U.assign(n, std::vector<double>(SB)); w.V.assign(n, std::vector<double>(SB));
        w.boost.assign(n, std::vector<int>(B)); w.lscale.assign(n, std::vector<double>(B));
        w.L.assign(B, 0.0); w.logL.assign(B, 0.0);
    }
    std::vector<double> col(S);
    for (int u : tr.post) {
        auto& D = w.D[u];
        std::fill(w.boost[u].begin(), w.boost[u].end(), 0);
        std::fill(w.lscale[u].begin(), w.lscale[u].end(), 0.0);
        if (tr.leaf[u]) {                                             // likelihood.hpp:505-512
            for (int b = 0; b < B; ++b) {
                leaf_vector(a, p0 + b, l2t[u], S, col.data());
                for (int s = 0; s < S; ++s) D[size_t(s) * B + b] = col[s];
            }
            continue;
        }
        std::fill(D.begin(), D.end(), 1.0);                           // likelihood.hpp:568-595
        for (int c : tr.children[u]) {
            gemm_tile(Pb[c], w.D[c].data(), w.PD[c].data(), S, B);
            const auto& M = w.PD[c];
            for (size_t e = 0; e < SB; ++e) D[e] *= M[e];
            for (int b = 0; b < B; ++b) w.lscale[u][b] += w.lscale[c][b];
            rescale_cols(D.data(), S, B, w.boost[u].data());
        }
        rescale_cols(D.data(), S, B, w.boost[u].data());
        for (int b = 0; b < B; ++b) w.lscale[u][b] -= w.boost[u][b] * kLogScaler;
    }
    for (int b = 0; b < B; ++b) {                                     // likelihood.hpp:599-608
        double L = 0;
        for (int s = 0; s < S; ++s) L += w.D[tr.root][size_t(s) * B + b] * pi[s];
        w.L[b] = L;
        w.logL[b] = L > 0 ? std::log(L) + w.lscale[tr.root][b] : -1e20;
    }
    if (!outside) return;
    for (int s = 0; s < S; ++s) for (int b = 0; b < B; ++b) w.U[tr.root][size_t(s) * B + b] = pi[s];   // :611
    for (auto it = tr.post.rbegin(); it != tr.post.rend(); ++it) {
        const int u = *it;
        if (tr.leaf[u]) continue;
        const auto& ch = tr.children[u];
        const size_t k = ch.size();
        if (!k) continue;
        if (w.pref.size() < k) {
            w.pref.resize(k); w.suff.resize(k); w.pb.resize(k); w.sb.resize(k);
        }
        for (size_t i = 0; i < k; ++i) {
            w.pref[i].assign(SB, 1.0); w.suff[i].assign(SB, 1.0);
            w.pb[i].assign(B, 0); w.sb[i].assign(B, 0);
        }
        for (size_t i = 1; i < k; ++i) {                              // :707-722 prefix products
            const auto& M = w.PD[ch[i - 1]];
            for (size_t e = 0; e < SB; ++e) w.pref[i][e] = w.pref[i - 1][e] * M[e];
            w.pb[i] = w.pb[i - 1];
            rescale_cols(w.pref[i].data(), S, B, w.pb[i].data());
        }
        for (size_t i = k - 1; i > 0; --i) {                          // :724-739 suffix products
            const auto& M = w.PD[ch[i]];
            for (size_t e = 0; e < SB; ++e) w.suff[i - 1][e] = w.suff[i][e] * M[e];
            w.sb[i - 1] = w.sb[i];
            rescale_cols(w.suff[i - 1].data(), S, B, w.sb[i - 1].data());
        }
        for (size_t i = 0; i < k; ++i) {                              // :741-759
            const int c = ch[i];
            auto& Vc = w.V[c];
            for (size_t e = 0; e < SB; ++e) Vc[e] = w.U[u][e] * w.pref[i][e] * w.suff[i][e];
            for (int b = 0; b < B; ++b) {
                int net = w.boost[u][b] - w.pb[i][b] - w.sb[i][b];
                for (; net > 0; --net) for (int s = 0; s < S; ++s) Vc[size_t(s) * B + b] *= kUp;
                for (; net < 0; ++net) for (int s = 0; s < S; ++s) Vc[size_t(s) * B + b] *= kDown;
            }
            gemm_tile_t(Pb[c], Vc.data(), w.U[c].data(), S, B);
        }
    }
}

inline int n_threads_for(int items) {
#ifdef _OPENMP
    return std::max(1, std::min(omp_get_max_threads(), items));
#else
    (void)items; return 1;
#endif
}

// likelihood.hpp:766-806 : lnL from given transition matrices (zero-likelihood
// patterns contribute weight * -1e20).
inline double loglik_from_P(const Tree& tr, const Alignment& a, const std::vector<Mat>& Pb,
                            const std::vector<double>& pi, std::vector<double>* site = nullptr) {
    const int S = a.code.S, P = a.P;
    auto l2t = leaf_map(tr, a);
    std::vector<double> pl(P);
    #pragma omp parallel num_threads(n_threads_for(P))
    {
        Pass w;
        #pragma omp for schedule(static)
        for (int p = 0; p < P; ++p) { inside_outside(tr, a, p, l2t, Pb, pi, S, w, false); pl[p] = w.logL; }
    }
    Neumaier acc;
    for (int p = 0; p < P; ++p) acc.add(a.weights[p] * pl[p]);
    if (site) *site = pl;
    return acc.value();
}

// likelihood.hpp:257-292
inline double mg94_loglik(const Tree& tr, const Alignment& a, const MG94& m, double branch_scale = 1.0,
                          const std::vector<double>* bl = nullptr) {
    std::vector<Mat> Pb(tr.n(), Mat::eye(a.code.S));
    for (int i = 0; i < tr.n(); ++i) if (i != tr.root) Pb[i] = m.P((bl ? (*bl)[i] : tr.bl[i]) * branch_scale);
    return loglik_from_P(tr, a, Pb, m.pi);
}

// ------------------------------------------------------------ nucleotide GTR
// alignment.hpp:832-890 (to_nucleotide_alignment): per nucleotide site the IUPAC set of every taxon
// is the pattern key; state = the unambiguous nucleotide (char_to_nuc) or -1, mask = the set; patterns
// in first-occurrence order; the codon alignment's nucleotide frequencies are kept.
inline Alignment nucleotide_patterns(const Alignment& a) {
    Alignment r;
    r.names = a.names; r.seqs = a.seqs; r.code = a.code; r.T = a.T; r.n_codons = 0;
    std::copy(a.nuc_freq, a.nuc_freq + 4, r.nuc_freq);
    const size_t L = a.seqs.empty() ? 0 : a.seqs[0].size();
    std::map<std::string, int> seen;
    std::string key(size_t(a.T), 'N');
    for (size_t site = 0; site < L; ++site) {
        for (int t = 0; t < a.T; ++t) key[size_t(t)] = char('A' + iupac_bits(a.seqs[size_t(t)][site]));
        auto it = seen.find(key);
        if (it == seen.end()) {
            seen.emplace(key, r.P);
            r.site_pattern.push_back(r.P++);
            for (int t = 0; t < a.T; ++t) {
                const char ch = a.seqs[size_t(t)][site];
                r.states.push_back(int8_t(nuc_index(ch)));
                r.masks.push_back(uint64_t(iupac_bits(ch)));
            }
            r.weights.push_back(1.0);
        } else {
            r.site_pattern.push_back(it->second);
            r.weights[size_t(it->second)] += 1.0;
        }
    }
    return r;
}

// rate_matrix.hpp:14-104: GTR with theta_AG = 1, Q normalised to mean rate 1, symmetric
// eigensystem of diag(sqrt pi) Q diag(1 / sqrt pi) (pi floored at 1e-12), eigenvalues <= 0,
// P(t) = U diag(e^{lambda t}) V clamped at 0
struct GTR {
    double pi[4] = {0.25, 0.25, 0.25, 0.25};
    double scale = 1.0;
    std::vector<double> lam;
    Mat Q{4, 4}, U{4, 4}, V{4, 4};
    void update(const double theta[5], const double freq[4]) {
        const double AC = theta[0], AT = theta[1], CG = theta[2], CT = theta[3], GT = theta[4];
        const double r[4][4] = {{0, AC, 1, AT}, {AC, 0, CG, CT}, {1, CG, 0, GT}, {AT, CT, GT, 0}};
        double sq[4], isq[4];
        for (int i = 0; i < 4; ++i) { pi[i] = freq[i]; sq[i] = std::sqrt(std::max(pi[i], 1e-12)); isq[i] = 1.0 / sq[i]; }
        Q = Mat(4, 4);
        for (int i = 0; i < 4; ++i) {
            double row = 0;
            for (int j = 0; j < 4; ++j) if (i != j) { Q(i, j) = r[i][j] * pi[j]; row += Q(i, j); }
            Q(i, i) = -row;
        }
        double avg = 0;
        for (int i = 0; i < 4; ++i) avg -= pi[i] * Q(i, i);
        if (avg > 0) { scale = avg; for (auto& x : Q.a) x /= avg; }
        Mat Sm(4, 4);
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) Sm(i, j) = sq[i] * Q(i, j) * isq[j];
        for (int i = 0; i < 4; ++i) for (int j = i + 1; j < 4; ++j) { const double m = 0.5 * (Sm(i, j) + Sm(j, i)); Sm(i, j) = m; Sm(j, i) = m; }
        Mat E;
        jacobi_eigen(Sm, lam, E);
        for (auto& l : lam) l = std::min(l, 0.0);
        for (int i = 0; i < 4; ++i) for (int k = 0; k < 4; ++k) { U(i, k) = isq[i] * E(i, k); V(k, i) = E(i, k) * sq[i]; }
    }
    Mat P(double t) const {
        Mat out(4, 4);
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) {
            double x = 0;
            for (int k = 0; k < 4; ++k) x += U(i, k) * std::exp(lam[k] * t) * V(k, j);
            out(i, j) = std::max(x, 0.0);
        }
        return out;
    }
};

// likelihood.hpp:181-254 (compute_gtr_log_likelihood): per pattern L = pi . D_root, weight x
// (log L + scale) or weight x -1e20 when L <= 0, Neumaier sum over the patterns in order
inline double gtr_loglik(const Tree& tr, const Alignment& nuc, const GTR& g, const std::vector<double>& bl,
                         std::vector<double>* site = nullptr) {
    std::vector<Mat> Pb(tr.n(), Mat::eye(4));
    for (int i = 0; i < tr.n(); ++i) if (i != tr.root) Pb[i] = g.P(bl[i]);
    const std::vector<double> pi(g.pi, g.pi + 4);
    const auto l2t = leaf_map(tr, nuc);
    std::vector<double> pl(size_t(nuc.P));
    #pragma omp parallel num_threads(n_threads_for(nuc.P))
    {
        Pass w;
        #pragma omp for schedule(static)
        for (int p = 0; p < nuc.P; ++p) { inside_outside(tr, nuc, p, l2t, Pb, pi, 4, w, false); pl[size_t(p)] = w.logL; }
    }
    Neumaier acc;
    for (int p = 0; p < nuc.P; ++p) acc.add(nuc.weights[size_t(p)] * pl[size_t(p)]);
    if (site) *site = pl;
    return acc.value();
}

// ------------------------------------------------ general mixture evaluation
// One engine for the three reference gradient entry points:
//   * compute_branch_length_gradients   (likelihood.hpp:1102-1211): K=1, M=1, raw time
//   * compute_joint_frechet_gradients   (likelihood.hpp:1228-1594): K=1, M=1, tau = t*3/mu,
//     optional test/background partition, global gradients with the d mu term
//   * BUSTED compute_busted_branch_gradients (busted.hpp:1138-1429): K omega classes mixed
//     at the P level on test branches, background model elsewhere, M synonymous-rate
//     classes as separate passes with a root log-sum-exp, raw time.
// Global gradients for omega classes / mixture weights / thetas extend the same
// spectral Frechet formula (likelihood.hpp:1428-1520) to the mixture.
struct MixSpec {
    std::vector<Params> classes;       // K test-branch models
    std::vector<double> class_w;       // K mixing weights at the P level
    bool has_bg = false; Params bg;    // background model for non-test branches
    std::vector<char> is_test;         // per node (empty = all test)
    std::vector<double> rates{1.0}, rate_w{1.0};
    bool normalized_time = false;      // tau = t * 3 / mu (per model)
    bool want_global = false;
    bool zero_l_sentinel = false;      // true: L<=0 contributes w * -1e20 to lnL
    bool tiled = false;                // true: 64-pattern tiles with S x B GEMMs (the reference's batched shape)
    std::vector<int> branch_classes;   // empty, or n + 1 offsets: branch b mixes classes [bc[b], bc[b+1]) (aBSREL,
                                       // absrel.hpp:262-276: P_b = sum_k w_bk P(omega_bk, t_b))
};
struct MixResult {
    double lnl = 0;
    std::vector<double> grad_t;        // per node (root 0)
    std::vector<double> grad_beta;     // per test class k (d/d beta_k)
    double grad_beta_bg = 0;
    std::vector<double> grad_class_w;  // d/d c_k (raw partials)
    double grad_theta[5] = {0, 0, 0, 0, 0};
    std::vector<double> grad_rate_w;   // d/d rho_m (raw partials)
    std::vector<double> site_lnl;
};

inline MixResult mixture_eval(const Tree& tr, const Alignment& a, const MixSpec& sp, const std::vector<double>& bl) {
    const int S = a.code.S, n = tr.n(), P = a.P;
    const int K = int(sp.classes.size()), M = int(sp.rates.size());
    auto l2t = leaf_map(tr, a);
    auto test = [&](int b) { return sp.is_test.empty() ? true : bool(sp.is_test[b]); };
    // the test classes branch b mixes: all K, or its own range of them
    auto kb0 = [&](int b) { return sp.branch_classes.empty() ? 0 : sp.branch_classes[size_t(b)]; };
    auto kb1 = [&](int b) { return sp.branch_classes.empty() ? K : sp.branch_classes[size_t(b) + 1]; };
    std::vector<MG94> mk(K); for (int k = 0; k < K; ++k) mk[k].update(sp.classes[k], a.pos_freq, a.pi, a.code);
    MG94 mbg; if (sp.has_bg) mbg.update(sp.bg, a.pos_freq, a.pi, a.code);
    auto conv = [&](const MG94& m) { return sp.normalized_time ? 3.0 / std::max(m.mu, 1e-12) : 1.0; };
    // per (m, b): P, dP/dt, and the per-class (class, tau) used
    std::vector<std::vector<Mat>> Pm(M, std::vector<Mat>(n, Mat::eye(S))), dPm(M, std::vector<Mat>(n, Mat(S, S)));
    std::vector<std::vector<std::vector<Mat>>> Pk(M, std::vector<std::vector<Mat>>(n));
    // every (m, b) is independent: built in parallel, same values as a serial loop
    #pragma omp parallel for schedule(dynamic) num_threads(n_threads_for(M * n))
    for (int mb = 0; mb < M * n; ++mb) {
        const int m = mb / n, b = mb % n;
        if (b == tr.root) continue;
        double r = sp.rates[m];
        if (test(b)) {
            Pm[m][b] = Mat(S, S);
            Pk[m][b].resize(K);
            for (int k = kb0(b); k < kb1(b); ++k) {
                double cv = conv(mk[k]);
                Mat Pkb = mk[k].P(r * bl[b] * cv);
                Mat QP = matmul(mk[k].Q, Pkb);
                for (size_t e = 0; e < Pkb.a.size(); ++e) {
                    Pm[m][b].a[e] += sp.class_w[k] * Pkb.a[e];
                    dPm[m][b].a[e] += sp.class_w[k] * r * cv * QP.a[e];
                }
                Pk[m][b][k] = std::move(Pkb);
            }
        } else {
            double cv = conv(mbg);
            Mat Pb = mbg.P(r * bl[b] * cv);
            Mat QP = matmul(mbg.Q, Pb);
            for (size_t e = 0; e < QP.a.size(); ++e) dPm[m][b].a[e] = r * cv * QP.a[e];
            Pm[m][b] = std::move(Pb);
        }
    }
    MixResult res;
    res.grad_t.assign(n, 0.0);
    res.site_lnl.assign(P, 0.0);
    std::vector<double> pat_ll(P, 0.0);
    std::vector<std::vector<double>> pat_g(n, std::vector<double>(P, 0.0));
    std::vector<std::vector<double>> pat_rw(M, std::vector<double>(P, 0.0));
    // A_{m,b} = sum_p f_{m,p} V D^T, accumulated per thread then reduced in thread order
    const bool G = sp.want_global;
    // per pattern: combine the rate passes (root log-sum-exp, busted.hpp:1342-1375); post[m] = posterior
    // of rate class m; false when the pattern has zero likelihood (no gradient terms)
    auto combine = [&](int p, const double* Lm, const double* logLm, double* post) {
        const double wt = a.weights[p];
        for (int m = 0; m < M; ++m) post[m] = 0.0;
        bool ok = false;
        if (M == 1) {
            if (Lm[0] > 0) { pat_ll[p] = wt * logLm[0]; post[0] = 1.0; ok = true; }
            else if (sp.zero_l_sentinel) pat_ll[p] = wt * -1e20;
            res.site_lnl[p] = Lm[0] > 0 ? logLm[0] : -1e20;
        } else {
            double mx = -std::numeric_limits<double>::infinity();
            for (int m = 0; m < M; ++m)
                if (sp.rate_w[m] > 1e-12 && Lm[m] > 0) mx = std::max(mx, std::log(sp.rate_w[m]) + logLm[m]);
            res.site_lnl[p] = -1e20;
            if (mx > -1e19) {
                double se = 0;
                for (int m = 0; m < M; ++m)
                    if (sp.rate_w[m] > 1e-12 && Lm[m] > 0) { post[m] = std::exp(std::log(sp.rate_w[m]) + logLm[m] - mx); se += post[m]; }
                if (se > 0) {
                    pat_ll[p] = wt * (mx + std::log(se));
                    res.site_lnl[p] = mx + std::log(se);
                    for (int m = 0; m < M; ++m) post[m] /= se;
                    ok = true;
                }
            }
            if (!ok && sp.zero_l_sentinel) pat_ll[p] = wt * -1e20;
        }
        return ok;
    };
    std::vector<std::vector<Mat>> Athr;
    if (sp.tiled) {
        // likelihood.hpp:1151-1197: OpenMP over 64-pattern tiles, per branch the S x B product dP * D
        // and (w / L) V . (dP D) per pattern; the A_b accumulation is (f V) D^T over the tile
        if (M > 64) throw std::runtime_error("tiled mixture_eval: at most 64 rate classes");
        const int ntile = (P + kTile - 1) / kTile;
        const int nt = n_threads_for(ntile);
        Athr.resize(G ? nt : 0);
        #pragma omp parallel num_threads(nt)
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            if (G) Athr[tid].assign(size_t(M) * n, Mat(S, S));
            std::vector<TilePass> w(M);
            std::vector<double> dPD(size_t(S) * kTile), fv(size_t(S) * kTile);
            std::vector<double> Lm(M), logLm(M), post(size_t(M) * kTile), f(size_t(M) * kTile);
            std::vector<char> ok(kTile);
            #pragma omp for schedule(static)
            for (int t = 0; t < ntile; ++t) {
                const int p0 = t * kTile, B = std::min(kTile, P - p0);
                for (int m = 0; m < M; ++m)
                    if (M == 1 || sp.rate_w[m] > 1e-12) inside_outside_tile(tr, a, p0, B, l2t, Pm[m], a.pi, S, w[m], true);
                for (int b = 0; b < B; ++b) {
                    for (int m = 0; m < M; ++m) {
                        const bool on = M == 1 || sp.rate_w[m] > 1e-12;
                        Lm[m] = on ? w[m].L[b] : 0.0;
                        logLm[m] = on ? w[m].logL[b] : -1e20;
                    }
                    double pm[64];
                    ok[b] = combine(p0 + b, Lm.data(), logLm.data(), pm);
                    for (int m = 0; m < M; ++m) {
                        post[size_t(m) * kTile + b] = pm[m];
                        const bool use = ok[b] && !(pm[m] <= 1e-12 && M > 1);
                        f[size_t(m) * kTile + b] = use ? a.weights[p0 + b] * pm[m] / w[m].L[b] : 0.0;
                        if (use && M > 1) pat_rw[m][p0 + b] = a.weights[p0 + b] * pm[m] / sp.rate_w[m];
                    }
                }
                for (int m = 0; m < M; ++m) {
                    bool any = false;
                    for (int b = 0; b < B; ++b) any = any || f[size_t(m) * kTile + b] != 0.0;
                    if (!any) continue;
                    const double* fm = &f[size_t(m) * kTile];
                    for (int br = 0; br < n; ++br) {
                        if (br == tr.root) continue;
                        const auto& Vb = w[m].V[br];
                        const auto& Db = w[m].D[br];
                        gemm_tile(dPm[m][br], Db.data(), dPD.data(), S, B);
                        for (int b = 0; b < B; ++b) {
                            if (fm[b] == 0.0) continue;
                            double g = 0;
                            for (int s = 0; s < S; ++s) g += Vb[size_t(s) * B + b] * dPD[size_t(s) * B + b];
                            pat_g[br][p0 + b] += fm[b] * g;
                        }
                        if (G) {
                            // A += (f V) D^T : S x B by B x S
                            Mat& A = Athr[tid][size_t(m) * n + br];
                            for (int s = 0; s < S; ++s)
                                for (int b = 0; b < B; ++b) fv[size_t(s) * B + b] = fm[b] * Vb[size_t(s) * B + b];
                            gemm_tile_acc_nt(fv.data(), Db.data(), A, S, B);
                        }
                    }
                }
            }
        }
    } else {
    int nt = n_threads_for(P);
    Athr.resize(G ? nt : 0);
    #pragma omp parallel num_threads(nt)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        if (G) Athr[tid].assign(size_t(M) * n, Mat(S, S));
        std::vector<Pass> w(M);
        std::vector<double> tmp(S);
        #pragma omp for schedule(static)
        for (int p = 0; p < P; ++p) {
            double wt = a.weights[p];
            std::vector<double> post(M, 0.0);
            for (int m = 0; m < M; ++m)
                if (M == 1 || sp.rate_w[m] > 1e-12) inside_outside(tr, a, p, l2t, Pm[m], a.pi, S, w[m], true);
            bool ok = false;
            if (M == 1) {
                if (w[0].L > 0) { pat_ll[p] = wt * w[0].logL; post[0] = 1.0; ok = true; }
                else if (sp.zero_l_sentinel) pat_ll[p] = wt * -1e20;
                res.site_lnl[p] = w[0].L > 0 ? w[0].logL : -1e20;
            } else {
                double mx = -std::numeric_limits<double>::infinity();
                for (int m = 0; m < M; ++m)
                    if (sp.rate_w[m] > 1e-12 && w[m].L > 0) mx = std::max(mx, std::log(sp.rate_w[m]) + w[m].logL);
                res.site_lnl[p] = -1e20;
                if (mx > -1e19) {
                    double se = 0;
                    for (int m = 0; m < M; ++m)
                        if (sp.rate_w[m] > 1e-12 && w[m].L > 0) { post[m] = std::exp(std::log(sp.rate_w[m]) + w[m].logL - mx); se += post[m]; }
                    if (se > 0) {
                        pat_ll[p] = wt * (mx + std::log(se));
                        res.site_lnl[p] = mx + std::log(se);
                        for (int m = 0; m < M; ++m) post[m] /= se;
                        ok = true;
                    }
                }
                if (!ok && sp.zero_l_sentinel) pat_ll[p] = wt * -1e20;
            }
            if (!ok) continue;
            for (int m = 0; m < M; ++m) {
                if (post[m] <= 1e-12 && M > 1) continue;
                if (M > 1) pat_rw[m][p] = wt * post[m] / sp.rate_w[m];
                double f = wt * post[m] / w[m].L;
                for (int b = 0; b < n; ++b) {
                    if (b == tr.root) continue;
                    matvec(dPm[m][b], w[m].D[b].data(), tmp.data());
                    double g = 0; for (int s = 0; s < S; ++s) g += w[m].V[b][s] * tmp[s];
                    pat_g[b][p] += f * g;
                    if (G) {
                        Mat& A = Athr[tid][size_t(m) * n + b];
                        const auto& Vb = w[m].V[b]; const auto& Db = w[m].D[b];
                        for (int i = 0; i < S; ++i) { double vi = f * Vb[i]; if (vi == 0) continue; double* row = &A.a[size_t(i) * S]; for (int j = 0; j < S; ++j) row[j] += vi * Db[j]; }
                    }
                }
            }
        }
    }
    }
    Neumaier acc; for (int p = 0; p < P; ++p) acc.add(pat_ll[p]);
    res.lnl = acc.value();
    std::vector<double> dL_dtau(n, 0.0);
    for (int b = 0; b < n; ++b) {
        if (b == tr.root) continue;
        Neumaier g; for (int p = 0; p < P; ++p) g.add(pat_g[b][p]);
        res.grad_t[b] = g.value();
    }
    res.grad_rate_w.assign(M, 0.0);
    if (M > 1) for (int m = 0; m < M; ++m) { Neumaier g; for (int p = 0; p < P; ++p) g.add(pat_rw[m][p]); res.grad_rate_w[m] = g.value(); }
    if (!G) return res;
    std::vector<Mat> A(size_t(M) * n, Mat(S, S));
    for (auto& th : Athr) for (size_t i = 0; i < A.size(); ++i) for (size_t e = 0; e < A[i].a.size(); ++e) A[i].a[e] += th[i].a[e];
    // spectral Frechet accumulation H = sum_b (U^T A_b V^T) o E(lambda, tau_b) (likelihood.hpp:1428-1471)
    auto frechetE = [&](const MG94& mm, double tau, Mat& E) {
        E = Mat(S, S);
        for (int i = 0; i < S; ++i) for (int j = 0; j < S; ++j) {
            double d = mm.lam[i] - mm.lam[j];
            E(i, j) = std::fabs(d) < 1e-9 ? tau * std::exp(mm.lam[i] * tau) : (std::exp(mm.lam[i] * tau) - std::exp(mm.lam[j] * tau)) / d;
        }
    };
    std::vector<Mat> Hk(K, Mat(S, S)); Mat Hbg(S, S);
    std::vector<double> sum_tau_g(K, 0.0); double sum_tau_g_bg = 0.0;
    res.grad_class_w.assign(K, 0.0);
    // (m, b) in fixed chunks summed in order inside each chunk, the chunks in order afterwards:
    // deterministic whatever the thread count
    const int nmb = M * n, kChunk = 32, nch = (nmb + kChunk - 1) / kChunk;
    std::vector<std::vector<Mat>> Hk_c(nch, std::vector<Mat>(K, Mat(S, S)));
    std::vector<Mat> Hbg_c(nch, Mat(S, S));
    std::vector<std::vector<double>> stg_c(nch, std::vector<double>(K, 0.0)), gcw_c(nch, std::vector<double>(K, 0.0));
    std::vector<double> stgbg_c(nch, 0.0);
    #pragma omp parallel for schedule(dynamic) num_threads(n_threads_for(nch))
    for (int ch = 0; ch < nch; ++ch)
    for (int mb = ch * kChunk; mb < std::min(nmb, (ch + 1) * kChunk); ++mb) {
        const int m = mb / n, b = mb % n;
        if (b == tr.root) continue;
        const Mat& Ab = A[size_t(m) * n + b];
        double r = sp.rates[m];
        if (test(b)) {
            for (int k = kb0(b); k < kb1(b); ++k) {
                double tau = r * bl[b] * conv(mk[k]);
                // d/dc_k : <A, P_k>
                double s = 0; for (size_t e = 0; e < Ab.a.size(); ++e) s += Ab.a[e] * Pk[m][b][k].a[e];
                gcw_c[ch][k] += s;
                Mat At = matmul(matmul(transpose(mk[k].U), Ab), transpose(mk[k].Vp));
                Mat E; frechetE(mk[k], tau, E);
                for (size_t e = 0; e < At.a.size(); ++e) Hk_c[ch][k].a[e] += sp.class_w[k] * At.a[e] * E.a[e];
                // tau * dlnL/dtau through this class, for the d mu term
                Mat QP = matmul(mk[k].Q, Pk[m][b][k]);
                double g = 0; for (size_t e = 0; e < Ab.a.size(); ++e) g += Ab.a[e] * QP.a[e];
                stg_c[ch][k] += sp.class_w[k] * tau * g;
            }
        } else {
            double tau = r * bl[b] * conv(mbg);
            Mat At = matmul(matmul(transpose(mbg.U), Ab), transpose(mbg.Vp));
            Mat E; frechetE(mbg, tau, E);
            for (size_t e = 0; e < At.a.size(); ++e) Hbg_c[ch].a[e] += At.a[e] * E.a[e];
            Mat QP = matmul(mbg.Q, Pm[m][b]);
            double g = 0; for (size_t e = 0; e < Ab.a.size(); ++e) g += Ab.a[e] * QP.a[e];
            stgbg_c[ch] += tau * g;
        }
    }
    for (int ch = 0; ch < nch; ++ch) {
        for (int k = 0; k < K; ++k) {
            for (size_t e = 0; e < Hk[k].a.size(); ++e) Hk[k].a[e] += Hk_c[ch][k].a[e];
            res.grad_class_w[k] += gcw_c[ch][k];
            sum_tau_g[k] += stg_c[ch][k];
        }
        for (size_t e = 0; e < Hbg.a.size(); ++e) Hbg.a[e] += Hbg_c[ch].a[e];
        sum_tau_g_bg += stgbg_c[ch];
    }
    auto part = [&](const MG94& mm, const Mat& H, double sum_tg, const Mat& dQ) {
        Mat Mx = matmul(matmul(mm.Vp, dQ), mm.U);
        double p1 = 0; for (size_t e = 0; e < Mx.a.size(); ++e) p1 += Mx.a[e] * H.a[e];
        double p2 = 0;
        if (sp.normalized_time) {
            double dmu = 0; for (int i = 0; i < S; ++i) dmu -= mm.pi[i] * dQ(i, i);
            p2 = -(dmu / std::max(mm.mu, 1e-12)) * sum_tg;
        }
        return p1 + p2;
    };
    res.grad_beta.assign(K, 0.0);
    for (int k = 0; k < K; ++k) res.grad_beta[k] = part(mk[k], Hk[k], sum_tau_g[k], dQ_beta(sp.classes[k], a.pos_freq, a.code));
    if (sp.has_bg) res.grad_beta_bg = part(mbg, Hbg, sum_tau_g_bg, dQ_beta(sp.bg, a.pos_freq, a.code));
    for (int x = 0; x < 5; ++x) {
        double g = 0;
        for (int k = 0; k < K; ++k)
            g += part(mk[k], Hk[k], sum_tau_g[k], dQ_theta(kThetaPairs[x][0], kThetaPairs[x][1], sp.classes[k].alpha, sp.classes[k].beta, a.pos_freq, a.code));
        if (sp.has_bg)
            g += part(mbg, Hbg, sum_tau_g_bg, dQ_theta(kThetaPairs[x][0], kThetaPairs[x][1], sp.bg.alpha, sp.bg.beta, a.pos_freq, a.code));
        res.grad_theta[x] = g;
    }
    return res;
}

// likelihood.hpp:1102-1211
inline std::pair<double, std::vector<double>> branch_length_gradients(const Tree& tr, const Alignment& a, const Params& p,
                                                                      std::vector<double> bl) {
    if (bl.empty()) bl = tr.bl;
    MixSpec sp; sp.classes = {p}; sp.class_w = {1.0};
    auto r = mixture_eval(tr, a, sp, bl);
    return {r.lnl, r.grad_t};
}

// likelihood.hpp:1228-1594 (grad_branches = conv * dL/dtau; globals include the d mu term)
inline MixResult joint_frechet_gradients(const Tree& tr, const Alignment& a, const Params& p, std::vector<double> bl,
                                         const std::vector<char>* is_test = nullptr, double omega_bg = -1.0) {
    if (bl.empty()) bl = tr.bl;
    MixSpec sp; sp.classes = {p}; sp.class_w = {1.0}; sp.normalized_time = true; sp.want_global = true;
    if (is_test && int(is_test->size()) == tr.n() && omega_bg >= 0.0) {
        sp.has_bg = true; sp.bg = p; sp.bg.beta = omega_bg; sp.is_test = *is_test;
    }
    return mixture_eval(tr, a, sp, bl);
}


// ------------------------------------------------------------------ FEL
// Per-site fixed-effects likelihood fits (analyses/fel.hpp:230-446, fast path
// with every branch tested) and the two scalar optimisers it uses
// (opt/nelder_mead.hpp:24-105 Brent1D, :111-229 NelderMead2D), restated.

// opt/nelder_mead.hpp:24-105 — Brent's parabolic / golden-section minimiser on [min(ax,cx), max(ax,cx)]
template <class F>
inline std::pair<double, double> brent1d(F&& f, double ax, double bx, double cx, double tol = 1e-4, int max_iter = 60) {
    const double CGOLD = 0.3819660, ZEPS = 1e-10;
    double a = std::min(ax, cx), b = std::max(ax, cx);
    double v = bx, w = v, x = v, e = 0.0;
    double fx = f(x), fv = fx, fw = fx;
    for (int iter = 0; iter < max_iter; ++iter) {
        const double xm = 0.5 * (a + b), tol1 = tol * std::fabs(x) + ZEPS, tol2 = 2.0 * tol1;
        if (std::fabs(x - xm) <= (tol2 - 0.5 * (b - a))) break;
        double d = 0.0;
        if (std::fabs(e) > tol1) {
            double r = (x - w) * (fx - fv), q = (x - v) * (fx - fw), pp = (x - v) * q - (x - w) * r;
            q = 2.0 * (q - r);
            if (q > 0.0) pp = -pp;
            q = std::fabs(q);
            const double etemp = e;
            e = d;
            if (std::fabs(pp) >= std::fabs(0.5 * q * etemp) || pp <= q * (a - x) || pp >= q * (b - x)) {
                e = (x >= xm) ? a - x : b - x;
                d = CGOLD * e;
            } else {
                d = pp / q;
                const double u = x + d;
                if (u - a < tol2 || b - u < tol2) d = (xm - x >= 0.0) ? std::fabs(tol1) : -std::fabs(tol1);
            }
        } else {
            e = (x >= xm) ? a - x : b - x;
            d = CGOLD * e;
        }
        const double u = (std::fabs(d) >= tol1) ? x + d : x + ((d >= 0.0) ? std::fabs(tol1) : -std::fabs(tol1));
        const double fu = f(u);
        if (fu <= fx) {
            if (u >= x) a = x; else b = x;
            v = w; fv = fw; w = x; fw = fx; x = u; fx = fu;
        } else {
            if (u < x) a = u; else b = u;
            if (fu <= fw || w == x) { v = w; fv = fw; w = u; fw = fu; }
            else if (fu <= fv || v == x || v == w) { v = u; fv = fu; }
        }
    }
    return {x, fx};
}

struct NMPoint { double a = 0, b = 0, f = 0; };

// stable order of three simplex vertices by f (what std::sort does on three elements in libstdc++)
inline void sort3(std::array<NMPoint, 3>& s) {
    for (int i = 1; i < 3; ++i) {
        NMPoint v = s[i]; int j = i;
        while (j > 0 && v.f < s[j - 1].f) { s[j] = s[j - 1]; --j; }
        s[j] = v;
    }
}

// opt/nelder_mead.hpp:111-229 — bounded 2-D Nelder-Mead
template <class F>
inline NMPoint nelder_mead2d(F&& f, double init_a, double init_b, double lb = 1e-4, double ub = 1000.0,
                             double tol = 1e-4, int max_iter = 100) {
    auto clamp = [&](double v) { return std::clamp(v, lb, ub); };
    auto eval = [&](double a, double b) { const double ca = clamp(a), cb = clamp(b); return NMPoint{ca, cb, f(ca, cb)}; };
    const double step_a = std::max(0.1, 0.2 * init_a), step_b = std::max(0.1, 0.2 * init_b);
    std::array<NMPoint, 3> s = {eval(init_a, init_b), eval(init_a + step_a, init_b), eval(init_a, init_b + step_b)};
    const double alpha = 1.0, gamma = 2.0, rho = 0.5, sigma = 0.5;
    for (int iter = 0; iter < max_iter; ++iter) {
        sort3(s);
        if (std::fabs(s[2].f - s[0].f) < tol && std::fabs(s[2].a - s[0].a) < tol && std::fabs(s[2].b - s[0].b) < tol) break;
        const double c_a = 0.5 * (s[0].a + s[1].a), c_b = 0.5 * (s[0].b + s[1].b);
        const NMPoint r = eval(c_a + alpha * (c_a - s[2].a), c_b + alpha * (c_b - s[2].b));
        if (r.f < s[0].f) {
            const NMPoint e = eval(c_a + gamma * (r.a - c_a), c_b + gamma * (r.b - c_b));
            s[2] = (e.f < r.f) ? e : r;
        } else if (r.f < s[1].f) {
            s[2] = r;
        } else {
            const bool outside = r.f < s[2].f;
            const NMPoint c = outside ? eval(c_a + rho * (r.a - c_a), c_b + rho * (r.b - c_b))
                                      : eval(c_a + rho * (s[2].a - c_a), c_b + rho * (s[2].b - c_b));
            const double ref_f = outside ? r.f : s[2].f;
            if (c.f < ref_f) {
                s[2] = c;
            } else {
                s[1] = eval(s[0].a + sigma * (s[1].a - s[0].a), s[0].b + sigma * (s[1].b - s[0].b));
                s[2] = eval(s[0].a + sigma * (s[2].a - s[0].a), s[0].b + sigma * (s[2].b - s[0].b));
            }
        }
    }
    sort3(s);
    return s[0];
}

struct FelSite {
    double alpha = 0, beta = 0, alpha_null = 0, lrt = 0, p_value = 1, total_bl = 0, lnl_alt = 0, lnl_null = 0;
    int evals = 0;
};
struct FelRun {
    double conversion = 1.0, tested_length = 0.0;
    std::vector<double> bl;           // branch lengths in FEL time (x conversion)
    std::vector<FelSite> patterns;
};

// fel.hpp:230-273 (every branch tested): t_b <- t_b * 3 / scale_factor(base model)
inline FelRun fel_prepare(const Tree& tr, const Alignment& a, const Params& base) {
    FelRun r;
    MG94 m0; m0.update(base, a.pos_freq, a.pi, a.code);
    r.conversion = m0.mu > 1e-12 ? 3.0 / m0.mu : 1.0;
    r.bl.assign(tr.n(), 0.0);
    for (int i = 0; i < tr.n(); ++i) if (i != tr.root) { r.tested_length += tr.bl[i]; r.bl[i] = tr.bl[i] * r.conversion; }
    return r;
}

// fel.hpp:326-446 (analyze_pattern, num_background == 0)
inline FelSite fel_pattern(const Tree& tr, const Alignment& a, const std::vector<int>& l2t, const Params& base,
                           const FelRun& run, int p) {
    FelSite res;
    int first = -1; bool invariant = true;
    for (int t = 0; t < a.T; ++t) {
        const int st = a.states[size_t(p) * a.T + t];
        if (st >= 0) { if (first == -1) first = st; else if (st != first) { invariant = false; break; } }
    }
    if (invariant) return res;
    const int S = a.code.S, n = tr.n();
    MG94 mg; double cached = -1.0;
    std::vector<Mat> Pb(n, Mat::eye(S));
    Pass w;
    auto lnl = [&](double aa, double bb) {
        ++res.evals;
        const double as = std::max(aa, 1e-12), om = bb / as;
        if (std::fabs(om - cached) > 1e-12) {
            Params q = base; q.alpha = 1.0; q.beta = om;
            mg.update(q, a.pos_freq, a.pi, a.code);
            cached = om;
        }
        for (int i = 0; i < n; ++i) if (i != tr.root) Pb[i] = mg.P(as * run.bl[i]);
        inside_outside(tr, a, p, l2t, Pb, mg.pi, S, w, false);
        return w.logL;
    };
    static const double grid[12][2] = {{0.01, 0.1}, {1.0, 0.1}, {1.0, 0.5}, {1.0, 1.0}, {1.0, 5.0}, {10.0, 0.1},
                                       {0.01, 0.5}, {0.01, 5.0}, {10.0, 0.5}, {10.0, 1.0}, {10.0, 50.0}, {100.0, 1.0}};
    double best = -1e20, ba = 1.0, bb = 1.0;
    for (auto& g : grid) { const double l = lnl(g[0], g[1]); if (l > best) { best = l; ba = g[0]; bb = g[1]; } }
    const NMPoint alt = nelder_mead2d([&](double x, double y) { return -lnl(x, y); }, ba, bb, 1e-4, 1000.0, 1e-4, 100);
    res.alpha = alt.a; res.beta = alt.b; res.lnl_alt = -alt.f;
    const double init_null = (std::min(res.alpha, 100.0) + 3.0 * std::min(res.beta, 100.0)) / 4.0;
    double best_null = lnl(init_null, init_null), best_na = init_null;
    for (double c : {0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0}) { const double l = lnl(c, c); if (l > best_null) { best_null = l; best_na = c; } }
    const auto nul = brent1d([&](double x) { return -lnl(x, x); }, 1e-4, std::clamp(best_na, 0.01, 45.0), 50.0, 1e-4, 60);
    res.alpha_null = nul.first; res.lnl_null = -nul.second;
    double lrt = 0.0;
    if (res.lnl_alt > -1e10 && res.lnl_null > -1e10) lrt = std::max(0.0, 2.0 * (res.lnl_alt - res.lnl_null));
    res.lrt = lrt;
    res.p_value = std::erfc(std::sqrt(lrt / 2.0));
    res.total_bl = res.alpha_null * run.tested_length;
    return res;
}

// fel.hpp:778-833 (run): every pattern, in parallel
inline FelRun fel_run(const Tree& tr, const Alignment& a, const Params& base, int max_patterns = -1) {
    FelRun run = fel_prepare(tr, a, base);
    const auto l2t = leaf_map(tr, a);
    const int P = max_patterns < 0 ? a.P : std::min(a.P, max_patterns);
    run.patterns.assign(P, FelSite{});
    #pragma omp parallel for schedule(dynamic) num_threads(n_threads_for(P))
    for (int p = 0; p < P; ++p) run.patterns[p] = fel_pattern(tr, a, l2t, base, run, p);
    return run;
}

// ------------------------------------------------------------------ MEME
// Mixed-effects model of episodic selection per site (analyses/meme.hpp:166-632,
// every branch tested), restated with the N-dimensional Nelder-Mead it uses
// (opt/nelder_mead.hpp:209-357).

template <int D>
struct NMPointN { std::array<double, D> x{}; double f = 0.0; };

// opt/nelder_mead.hpp:209-357 — bounded Nelder-Mead: the best of init and the grid
// starts a simplex of D perturbed vertices; reflection 1, expansion 2,
// contraction 0.5, shrink 0.5; converged when both the f-spread and the
// coordinate spread of best vs worst vertex are below tol.
template <int D, class F>
inline NMPointN<D> nelder_mead_nd(F&& f, const std::array<double, D>& init, const std::array<double, D>& lb,
                                  const std::array<double, D>& ub, double tol, int max_iter,
                                  const std::vector<std::array<double, D>>& grid) {
    using Pt = NMPointN<D>;
    auto eval = [&](const std::array<double, D>& v) {
        Pt q;
        for (int d = 0; d < D; ++d) q.x[d] = std::clamp(v[d], lb[d], ub[d]);
        q.f = f(q.x);
        return q;
    };
    Pt best = eval(init);
    for (const auto& g : grid) { Pt q = eval(g); if (q.f < best.f) best = q; }
    std::array<Pt, D + 1> s;
    s[0] = best;
    for (int d = 0; d < D; ++d) {
        std::array<double, D> x = best.x;
        const double step = std::max(0.05, 0.2 * std::fabs(best.x[d]));
        if (best.x[d] + step <= ub[d]) x[d] += step; else x[d] -= step;
        s[d + 1] = eval(x);
    }
    auto by_f = [](const Pt& a, const Pt& b) { return a.f < b.f; };
    for (int iter = 0; iter < max_iter; ++iter) {
        std::sort(s.begin(), s.end(), by_f);
        double dx = 0.0;
        for (int d = 0; d < D; ++d) dx = std::max(dx, std::fabs(s[D].x[d] - s[0].x[d]));
        if (std::fabs(s[D].f - s[0].f) < tol && dx < tol) break;
        std::array<double, D> c{};
        for (int i = 0; i < D; ++i) for (int d = 0; d < D; ++d) c[d] += s[i].x[d];
        for (int d = 0; d < D; ++d) c[d] /= double(D);
        std::array<double, D> xr;
        for (int d = 0; d < D; ++d) xr[d] = c[d] + 1.0 * (c[d] - s[D].x[d]);
        const Pt r = eval(xr);
        if (r.f < s[0].f) {
            std::array<double, D> xe;
            for (int d = 0; d < D; ++d) xe[d] = c[d] + 2.0 * (r.x[d] - c[d]);
            const Pt e = eval(xe);
            s[D] = (e.f < r.f) ? e : r;
        } else if (r.f < s[D - 1].f) {
            s[D] = r;
        } else {
            const bool outside = r.f < s[D].f;
            std::array<double, D> xc;
            for (int d = 0; d < D; ++d) xc[d] = c[d] + 0.5 * ((outside ? r.x[d] : s[D].x[d]) - c[d]);
            const Pt cc = eval(xc);
            if (cc.f < (outside ? r.f : s[D].f)) {
                s[D] = cc;
            } else {
                for (int i = 1; i <= D; ++i) {
                    std::array<double, D> xs;
                    for (int d = 0; d < D; ++d) xs[d] = s[0].x[d] + 0.5 * (s[i].x[d] - s[0].x[d]);
                    s[i] = eval(xs);
                }
            }
        }
    }
    std::sort(s.begin(), s.end(), by_f);
    return s[0];
}

// ------------------------------------------------------------ FEL, branch subsets
// fel.hpp:215-266 (partition_branches, prepare_branch_lengths) and :462-572
// (analyze_pattern with num_background > 0), without bridge resolutions.

struct FelSubsetSite {
    double alpha = 0, beta = 0, beta_nuisance = 0, alpha_null = 0, lrt = 0, p_value = 1, total_bl = 0;
    double lnl_alt = 0, lnl_null = 0;
    int evals = 0;
};
struct FelSubsetRun {
    double conversion = 1.0, bg_conversion = 1.0, tested_length = 0.0, bg_length = 0.0;
    std::vector<double> bl;           // branch lengths in FEL time
    std::vector<char> tested;         // per node; the root's entry is 0
    std::vector<FelSubsetSite> patterns;
};

// tested branches t * 3 / mu(base); background ones t * 3 / mu(alpha 1, beta bg_omega) when
// bg_omega > 0, else as the tested ones (fel.hpp:230-266)
inline FelSubsetRun fel_prepare_tested(const Tree& tr, const Alignment& a, const Params& base, const std::vector<char>& tested,
                                       double bg_omega = -1.0) {
    FelSubsetRun r;
    MG94 m0; m0.update(base, a.pos_freq, a.pi, a.code);
    r.conversion = m0.mu > 1e-12 ? 3.0 / m0.mu : 1.0;
    r.bg_conversion = r.conversion;
    r.tested.assign(tr.n(), 0);
    bool any_bg = false;
    for (int i = 0; i < tr.n(); ++i)
        if (i != tr.root) { r.tested[i] = tested[i] ? 1 : 0; any_bg = any_bg || !tested[i]; }
    if (any_bg && bg_omega > 0.0) {
        Params q = base; q.alpha = 1.0; q.beta = bg_omega;
        MG94 mb; mb.update(q, a.pos_freq, a.pi, a.code);
        if (mb.mu > 1e-12) r.bg_conversion = 3.0 / mb.mu;
    }
    r.bl.assign(tr.n(), 0.0);
    for (int i = 0; i < tr.n(); ++i) {
        if (i == tr.root) continue;
        if (r.tested[i]) { r.tested_length += tr.bl[i]; r.bl[i] = tr.bl[i] * r.conversion; }
        else { r.bg_length += tr.bl[i]; r.bl[i] = tr.bl[i] * r.bg_conversion; }
    }
    return r;
}

// fel.hpp:462-572: the likelihood builds MG94(alpha = a, beta = b_test) for the tested branches
// and MG94(a, b_bg) for the others at the FEL-time lengths, one model for all when
// |b_test - b_bg| < 1e-9; 3-D Nelder-Mead for the alternative, 2-D for the null (beta = alpha)
inline FelSubsetSite fel_pattern_subset(const Tree& tr, const Alignment& a, const std::vector<int>& l2t, const Params& base,
                                        const FelSubsetRun& run, int p) {
    FelSubsetSite res;
    int first = -1; bool invariant = true;
    for (int t = 0; t < a.T; ++t) {
        const int st = a.states[size_t(p) * a.T + t];
        if (st >= 0) { if (first == -1) first = st; else if (st != first) { invariant = false; break; } }
    }
    if (invariant) return res;
    const int S = a.code.S, n = tr.n();
    std::vector<Mat> Pb(n, Mat::eye(S));
    Pass w;
    MG94 mt, mb;
    auto lnl = [&](double aa, double bt, double bb) {
        ++res.evals;
        Params qt = base; qt.alpha = aa; qt.beta = bt;
        mt.update(qt, a.pos_freq, a.pi, a.code);
        const bool same = std::fabs(bt - bb) < 1e-9;
        if (!same) { Params qb = base; qb.alpha = aa; qb.beta = bb; mb.update(qb, a.pos_freq, a.pi, a.code); }
        for (int i = 0; i < n; ++i)
            if (i != tr.root) Pb[i] = (same || run.tested[i]) ? mt.P(run.bl[i]) : mb.P(run.bl[i]);
        inside_outside(tr, a, p, l2t, Pb, mt.pi, S, w, false);
        return w.logL;
    };
    using A3 = std::array<double, 3>;
    using A2 = std::array<double, 2>;
    static const double g3[12][3] = {{0.01, 0.1, 0.1}, {1.0, 0.1, 0.1}, {1.0, 0.5, 0.5},   {1.0, 1.0, 1.0},
                                     {1.0, 5.0, 5.0},  {10.0, 0.1, 0.1}, {0.01, 0.5, 0.5}, {0.01, 5.0, 5.0},
                                     {10.0, 0.5, 0.5}, {10.0, 1.0, 1.0}, {10.0, 50.0, 50.0}, {100.0, 1.0, 1.0}};
    double best = -1e20;
    A3 init = {1.0, 1.0, 1.0};
    for (const auto& g : g3) {
        const double l = lnl(g[0], g[1], g[2]);
        if (l > best) { best = l; init = {g[0], g[1], g[2]}; }
    }
    const auto alt = nelder_mead_nd<3>([&](const A3& x) { return -lnl(x[0], x[1], x[2]); }, init, A3{1e-4, 1e-4, 1e-4},
                                       A3{1000.0, 1000.0, 1000.0}, 1e-4, 100, {});
    res.alpha = alt.x[0]; res.beta = alt.x[1]; res.beta_nuisance = alt.x[2]; res.lnl_alt = -alt.f;
    const double ina = (std::min(res.alpha, 100.0) + 3.0 * std::min(res.beta, 100.0)) / 4.0, inb = res.beta_nuisance;
    double best_null = lnl(ina, ina, inb);
    A2 initn = {ina, inb};
    for (double ca : {0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0})
        for (double cb : {inb, 0.1, 1.0, 5.0}) {
            const double l = lnl(ca, ca, cb);
            if (l > best_null) { best_null = l; initn = {ca, cb}; }
        }
    const auto nul = nelder_mead_nd<2>([&](const A2& x) { return -lnl(x[0], x[0], x[1]); }, initn, A2{1e-4, 1e-4},
                                       A2{1000.0, 1000.0}, 1e-4, 80, {});
    res.alpha_null = nul.x[0]; res.lnl_null = -nul.f;
    double lrt = 0.0;
    if (res.lnl_alt > -1e10 && res.lnl_null > -1e10) lrt = std::max(0.0, 2.0 * (res.lnl_alt - res.lnl_null));
    res.lrt = lrt;
    res.p_value = std::erfc(std::sqrt(lrt / 2.0));
    res.total_bl = res.alpha_null * run.tested_length;
    return res;
}

// one likelihood of the subset model (for checks of the device evaluator)
inline double fel_subset_lnl(const Tree& tr, const Alignment& a, const Params& base, const FelSubsetRun& run, int p,
                             double aa, double bt, double bb) {
    const auto l2t = leaf_map(tr, a);
    const int S = a.code.S, n = tr.n();
    std::vector<Mat> Pb(n, Mat::eye(S));
    Pass w;
    MG94 mt, mb;
    Params qt = base; qt.alpha = aa; qt.beta = bt;
    mt.update(qt, a.pos_freq, a.pi, a.code);
    const bool same = std::fabs(bt - bb) < 1e-9;
    if (!same) { Params qb = base; qb.alpha = aa; qb.beta = bb; mb.update(qb, a.pos_freq, a.pi, a.code); }
    for (int i = 0; i < n; ++i)
        if (i != tr.root) Pb[i] = (same || run.tested[i]) ? mt.P(run.bl[i]) : mb.P(run.bl[i]);
    inside_outside(tr, a, p, l2t, Pb, mt.pi, S, w, false);
    return w.logL;
}

// fel.hpp:778-833 (run) with a background: every pattern, in parallel
inline FelSubsetRun fel_run_tested(const Tree& tr, const Alignment& a, const Params& base, const std::vector<char>& tested,
                                   double bg_omega = -1.0, int max_patterns = -1) {
    FelSubsetRun run = fel_prepare_tested(tr, a, base, tested, bg_omega);
    const auto l2t = leaf_map(tr, a);
    const int P = max_patterns < 0 ? a.P : std::min(a.P, max_patterns);
    run.patterns.assign(P, FelSubsetSite{});
    #pragma omp parallel for schedule(dynamic) num_threads(n_threads_for(P))
    for (int p = 0; p < P; ++p) run.patterns[p] = fel_pattern_subset(tr, a, l2t, base, run, p);
    return run;
}

struct MemeSite {
    double alpha = 0, beta1 = 0, p1 = 1, beta_plus = 0, p_plus = 0, lrt = 0, p_value = 1, beta_bg = 0;
    int bus = 0;                      // branches with EBF >= 100
    double total_bl = 0, lnl_meme = 0, lnl_fel = 0, p_vs_fel = 1, fel_alpha = 0, fel_beta = 0;
    int evals = 0;
    std::vector<double> ebf;          // per node, 1 where not computed
};
struct MemeRun {
    FelRun fel;                       // conversion, FEL-time branch lengths, the FEL fit of every pattern
    double mu_s = 0, mu_n = 0;        // scale factor = alpha mu_s + beta mu_n
    std::vector<MemeSite> patterns;
};

// meme.hpp:484-588: for every non-root branch b, the pattern's likelihood with b
// alone in class 1 (P1) and alone in class + (Pp), every other branch mixed (Pm);
// ebf[b] = exp(clamp(lnL_+ - lnL_1, -50, 50)), 1e6 when only lnL_1 is the zero
// sentinel, 0 when lnL_+ is.
inline void meme_branch_ebf(const Tree& tr, const Alignment& a, const std::vector<int>& l2t, int p, const std::vector<Mat>& P1,
                            const std::vector<Mat>& Pp, std::vector<Mat>& Pm, const std::vector<double>& pi,
                            std::vector<double>& ebf, const std::vector<char>* tested = nullptr) {
    const int S = a.code.S, n = tr.n();
    Pass w;
    ebf.assign(n, 1.0);
    for (int b = 0; b < n; ++b) {
        if (b == tr.root || (tested && !(*tested)[b])) continue;       // background branches keep 1
        const Mat keep = Pm[b];
        Pm[b] = P1[b];
        inside_outside(tr, a, p, l2t, Pm, pi, S, w, false);
        const double l1 = w.logL;
        Pm[b] = Pp[b];
        inside_outside(tr, a, p, l2t, Pm, pi, S, w, false);
        const double lp = w.logL;
        Pm[b] = keep;
        double e = 1.0;
        if (l1 > -1e10 && lp > -1e10) e = std::exp(std::clamp(lp - l1, -50.0, 50.0));
        else if (l1 <= -1e10 && lp > -1e10) e = 1e6;
        else e = 0.0;
        ebf[b] = e;
    }
}

// The branch EBFs of pattern p at given (alpha, omega1, p1, beta+) and FEL-time branch lengths;
// with tested (per node, non-empty) the other branches use omega beta_bg / alpha and keep EBF 1.
inline std::vector<double> meme_ebf_at(const Tree& tr, const Alignment& a, const Params& base, const std::vector<double>& bl,
                                       int p, double alpha, double omega1, double p1, double beta_plus,
                                       const std::vector<char>& tested = {}, double beta_bg = 0.0) {
    const int S = a.code.S, n = tr.n();
    const double ap = std::max(alpha, 1e-12);
    Params q1 = base; q1.alpha = 1.0; q1.beta = omega1;
    Params qp = base; qp.alpha = 1.0; qp.beta = beta_plus / ap;
    Params qb = base; qb.alpha = 1.0; qb.beta = beta_bg / ap;
    MG94 m1, mp, mb;
    m1.update(q1, a.pos_freq, a.pi, a.code);
    mp.update(qp, a.pos_freq, a.pi, a.code);
    if (!tested.empty()) mb.update(qb, a.pos_freq, a.pi, a.code);
    std::vector<Mat> P1(n, Mat::eye(S)), Pp(n, Mat::eye(S)), Pm(n, Mat::eye(S));
    for (int i = 0; i < n; ++i) {
        if (i == tr.root) continue;
        P1[i] = m1.P(ap * bl[i]);
        Pp[i] = mp.P(ap * bl[i]);
        if (!tested.empty() && !tested[i]) { Pm[i] = mb.P(ap * bl[i]); continue; }
        for (size_t e = 0; e < Pm[i].a.size(); ++e) Pm[i].a[e] = p1 * P1[i].a[e] + (1.0 - p1) * Pp[i].a[e];
    }
    std::vector<double> ebf;
    meme_branch_ebf(tr, a, leaf_map(tr, a), p, P1, Pp, Pm, a.pi, ebf, tested.empty() ? nullptr : &tested);
    return ebf;
}

// One MEME log-likelihood of pattern p (meme.hpp:219-272): tested branches mix omega1 and
// beta+ / alpha with (p1, 1 - p1); with tested non-empty the others use beta_bg / alpha alone.
inline double meme_lnl_at(const Tree& tr, const Alignment& a, const Params& base, const std::vector<double>& bl, int p,
                          double alpha, double omega1, double p1, double beta_plus, const std::vector<char>& tested,
                          double beta_bg) {
    const int S = a.code.S, n = tr.n();
    Params q1 = base; q1.alpha = alpha; q1.beta = alpha * omega1;
    Params qp = base; qp.alpha = alpha; qp.beta = beta_plus;
    Params qb = base; qb.alpha = alpha; qb.beta = beta_bg;
    MG94 m1, mp, mb;
    m1.update(q1, a.pos_freq, a.pi, a.code);
    mp.update(qp, a.pos_freq, a.pi, a.code);
    if (!tested.empty()) mb.update(qb, a.pos_freq, a.pi, a.code);
    std::vector<Mat> Pm(n, Mat::eye(S));
    for (int i = 0; i < n; ++i) {
        if (i == tr.root) continue;
        if (!tested.empty() && !tested[i]) { Pm[i] = mb.P(bl[i]); continue; }
        const Mat A = m1.P(bl[i]), B = mp.P(bl[i]);
        for (size_t e = 0; e < Pm[i].a.size(); ++e) Pm[i].a[e] = p1 * A.a[e] + (1.0 - p1) * B.a[e];
    }
    Pass w;
    inside_outside(tr, a, p, leaf_map(tr, a), Pm, m1.pi, S, w, false);
    return w.logL;
}

// The FEL fit a MEME search starts from (FelSite or FelSubsetSite).
struct MemeFelStart { double alpha = 0, beta = 0, beta_nuisance = 0, alpha_null = 0, lnl_alt = 0; };

// meme.hpp:166-632.  tested: per node, empty when every branch is tested; with a background the
// background branches evolve under omega beta_bg / alpha alone, beta_bg free in both models
// (5-D alternative from the grid with beta_bg = FEL's beta_nuisance, 4-D null), EBF 1 on them.
inline MemeSite meme_pattern_tested(const Tree& tr, const Alignment& a, const std::vector<int>& l2t, const Params& base,
                                    const std::vector<double>& bl, const std::vector<char>& tested, const MemeFelStart& fel,
                                    double mu_s, double mu_n, int p) {
    MemeSite res;
    const int S = a.code.S, n = tr.n();
    bool has_bg = false;
    for (int i = 0; i < n; ++i) if (i != tr.root && !tested.empty() && !tested[i]) has_bg = true;
    res.ebf.assign(n, 1.0);
    res.fel_alpha = fel.alpha; res.fel_beta = fel.beta; res.lnl_fel = fel.lnl_alt;
    int first = -1; bool invariant = true;
    for (int t = 0; t < a.T; ++t) {
        const int st = a.states[size_t(p) * a.T + t];
        if (st >= 0) { if (first == -1) first = st; else if (st != first) { invariant = false; break; } }
    }
    if (invariant) { res.lnl_fel = 0.0; return res; }
    // eigensystems of Q(omega) = Qs + omega Qn, reused when omega repeats exactly
    // (least recently used at the front; a hit moves to the back, so the models
    // returned by the current call are never the ones evicted)
    std::list<std::pair<double, MG94>> cache;
    auto model = [&](double om) -> const MG94& {
        for (auto it = cache.begin(); it != cache.end(); ++it)
            if (it->first == om) { cache.splice(cache.end(), cache, it); return cache.back().second; }
        if (cache.size() >= 8) cache.pop_front();
        Params q = base; q.alpha = 1.0; q.beta = om;
        cache.emplace_back(om, MG94{});
        cache.back().second.update(q, a.pos_freq, a.pi, a.code);
        return cache.back().second;
    };
    std::vector<Mat> P1(n, Mat::eye(S)), Pp(n, Mat::eye(S)), Pm(n, Mat::eye(S));
    Pass w;
    auto build = [&](double al, double w1, double p1, double bp, double bbg) {
        const double ap = std::max(al, 1e-12);
        const MG94& m1 = model(w1);
        const MG94& mp = model(bp / ap);
        const MG94& mb = has_bg ? model(bbg / ap) : m1;
        for (int i = 0; i < n; ++i) {
            if (i == tr.root) continue;
            P1[i] = m1.P(ap * bl[i]);
            Pp[i] = mp.P(ap * bl[i]);
            if (has_bg && !tested[i]) { Pm[i] = mb.P(ap * bl[i]); continue; }
            for (size_t e = 0; e < Pm[i].a.size(); ++e) Pm[i].a[e] = p1 * P1[i].a[e] + (1.0 - p1) * Pp[i].a[e];
        }
    };
    const std::vector<double>& pi = a.pi;
    auto lnl = [&](double al, double w1, double p1, double bp, double bbg) {
        ++res.evals;
        build(al, w1, p1, bp, bbg);
        inside_outside(tr, a, p, l2t, Pm, pi, S, w, false);
        return w.logL;
    };
    using A5 = std::array<double, 5>;
    using A4 = std::array<double, 4>;
    using A3 = std::array<double, 3>;
    // start grid (meme.hpp:282-312)
    const double af = std::clamp(fel.alpha, 1e-4, 10000.0), bf = std::clamp(fel.beta, 1e-4, 100000.0);
    const double bg0 = (has_bg && fel.beta_nuisance > 0.0) ? std::clamp(fel.beta_nuisance, 1e-4, 100000.0) : bf;
    const double w10 = std::clamp(bf / std::max(af, 1e-4), 0.0, 1.0);
    std::vector<A4> grid;
    if (af >= bf) {
        grid = {{af, w10, 0.75, bf}, {af, 0.0, 0.75, bf}, {af, 0.0, 0.95, af * 0.5}, {af, 0.25, 0.85, af * 0.9}};
        const double bp1 = std::max(af * 1.5, bf * 2.0), bp2 = std::max(af * 2.5, bf * 4.0), bp3 = std::max(af * 4.0, bf * 8.0);
        for (double pp : {0.05, 0.10, 0.20}) {
            grid.push_back({af, w10, 1.0 - pp, bp1});
            grid.push_back({af, w10, 1.0 - pp, bp2});
            grid.push_back({af, w10, 1.0 - pp, bp3});
        }
    } else {
        grid = {{af, w10, 0.75, bf}, {af, 0.0, 0.75, bf}, {af, 0.25, 0.50, bf * 2.0}, {af, 0.25, 0.75, bf * 5.0},
                {af, 0.10, 0.90, bf * 15.0}, {af, 0.00, 0.95, bf * 30.0}, {af, 1.00, 0.01, std::max(bf, af * 1.5)}};
    }
    const A4 lb4 = {1e-4, 0.0, 1e-6, 1e-4}, ub4 = {10000.0, 1.0, 1.0 - 1e-6, 100000.0};
    const A5 lb5 = {1e-4, 0.0, 1e-6, 1e-4, 1e-4}, ub5 = {10000.0, 1.0, 1.0 - 1e-6, 100000.0, 100000.0};
    auto obj4 = [&](const A4& x) { return -lnl(x[0], x[1], x[2], x[3], 0.0); };
    auto obj5 = [&](const A5& x) { return -lnl(x[0], x[1], x[2], x[3], x[4]); };
    double omega1 = w10;
    if (has_bg) {
        // meme.hpp:318-337
        std::vector<A5> grid5;
        for (const auto& g : grid) grid5.push_back({g[0], g[1], g[2], g[3], bg0});
        const auto alt = nelder_mead_nd<5>(obj5, grid5[0], lb5, ub5, 1e-5, 800, grid5);
        res.alpha = alt.x[0]; omega1 = alt.x[1]; res.p1 = alt.x[2]; res.beta_plus = alt.x[3]; res.beta_bg = alt.x[4];
        res.lnl_meme = -alt.f;
    } else {
        // meme.hpp:338-354
        const auto alt = nelder_mead_nd<4>(obj4, grid[0], lb4, ub4, 1e-5, 800, grid);
        res.alpha = alt.x[0]; omega1 = alt.x[1]; res.p1 = alt.x[2]; res.beta_plus = alt.x[3]; res.beta_bg = 0.0;
        res.lnl_meme = -alt.f;
    }
    res.beta1 = res.alpha * omega1; res.p_plus = 1.0 - res.p1;
    if (res.beta_plus > res.alpha && res.p_plus > 1e-6) {
        double lnl_null = -1e20, a_null = res.alpha, w_null = omega1, p_null = res.p1, bg_null = res.beta_bg;
        const double an = std::clamp(fel.alpha_null, 1e-4, 50.0);
        if (has_bg) {
            // null model beta+ = alpha, beta_bg free (meme.hpp:364-405)
            std::vector<A4> ng = {{res.alpha, omega1, res.p1, res.beta_bg}, {an, 1.0, 0.5, bg0}, {an, omega1, res.p1, bg0},
                                  {std::clamp(res.alpha, 1e-4, 50.0), 1.0, 0.5, res.beta_bg}};
            for (double c : {0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0, 20.0}) {
                ng.push_back({c, 0.5, 0.5, res.beta_bg}); ng.push_back({c, 0.0, 0.9, res.beta_bg});
            }
            const auto nul = nelder_mead_nd<4>([&](const A4& x) { return -lnl(x[0], x[1], x[2], x[0], x[3]); }, ng[0], lb4, ub4,
                                               1e-5, 800, ng);
            lnl_null = -nul.f; a_null = nul.x[0]; w_null = nul.x[1]; p_null = nul.x[2]; bg_null = nul.x[3];
            if (lnl_null > res.lnl_meme && std::isfinite(lnl_null)) {
                const std::vector<A5> wg = {{a_null, w_null, p_null, a_null, bg_null}, {a_null, w_null, 0.99, a_null, bg_null}};
                const auto alt2 = nelder_mead_nd<5>(obj5, wg[0], lb5, ub5, 1e-5, 800, wg);
                if (-alt2.f > res.lnl_meme) {
                    res.alpha = alt2.x[0]; omega1 = alt2.x[1]; res.p1 = alt2.x[2]; res.beta_plus = alt2.x[3];
                    res.beta_bg = alt2.x[4];
                    res.beta1 = res.alpha * omega1; res.p_plus = 1.0 - res.p1; res.lnl_meme = -alt2.f;
                }
            }
        } else {
            // null model beta+ = alpha (meme.hpp:406-452)
            std::vector<A3> ng = {{res.alpha, omega1, res.p1}, {an, 1.0, 0.5}, {an, omega1, res.p1},
                                  {std::clamp(res.alpha, 1e-4, 50.0), 1.0, 0.5}};
            for (double c : {0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0, 20.0}) { ng.push_back({c, 0.5, 0.5}); ng.push_back({c, 0.0, 0.9}); }
            const A3 lb3 = {1e-4, 0.0, 1e-6}, ub3 = {10000.0, 1.0, 1.0 - 1e-6};
            const auto nul = nelder_mead_nd<3>([&](const A3& x) { return -lnl(x[0], x[1], x[2], x[0], 0.0); }, ng[0], lb3, ub3,
                                               1e-5, 800, ng);
            lnl_null = -nul.f; a_null = nul.x[0]; w_null = nul.x[1]; p_null = nul.x[2];
            if (lnl_null > res.lnl_meme && std::isfinite(lnl_null)) {
                // warm-started alternative (meme.hpp:436-452)
                const std::vector<A4> wg = {{a_null, w_null, p_null, a_null}, {a_null, w_null, 0.99, a_null}};
                const auto alt2 = nelder_mead_nd<4>(obj4, wg[0], lb4, ub4, 1e-5, 800, wg);
                if (-alt2.f > res.lnl_meme) {
                    res.alpha = alt2.x[0]; omega1 = alt2.x[1]; res.p1 = alt2.x[2]; res.beta_plus = alt2.x[3];
                    res.beta1 = res.alpha * omega1; res.p_plus = 1.0 - res.p1; res.lnl_meme = -alt2.f;
                }
            }
        }
        // meme.hpp:456-482
        if (lnl_null <= -1e10 || res.lnl_meme <= -1e10 || !std::isfinite(lnl_null) || !std::isfinite(res.lnl_meme)) {
            res.lrt = 0.0; res.p_value = 1.0;
        } else if (lnl_null > res.lnl_meme) {
            res.alpha = a_null; res.beta1 = a_null * w_null; res.p1 = p_null; res.beta_plus = a_null; res.beta_bg = bg_null;
            res.p_plus = 1.0 - p_null; res.lnl_meme = lnl_null; omega1 = w_null;
            res.lrt = 0.0; res.p_value = 2.0 / 3.0;
        } else if (std::fabs(res.lnl_meme - lnl_null) <= 1e-12) {
            res.lrt = 0.0; res.p_value = 2.0 / 3.0;
        } else {
            res.lrt = 2.0 * (res.lnl_meme - lnl_null);
            res.p_value = (2.0 / 3.0) * (0.45 * std::erfc(std::sqrt(res.lrt / 2.0)) + 0.55 * std::exp(-res.lrt / 2.0));
        }
        // empirical Bayes factors of the tested branches (meme.hpp:484-588); the background model
        // takes beta_bg, or beta1 when that is not positive
        build(res.alpha, omega1, res.p1, res.beta_plus, res.beta_bg > 0.0 ? res.beta_bg : res.beta1);
        meme_branch_ebf(tr, a, l2t, p, P1, Pp, Pm, pi, res.ebf, has_bg ? &tested : nullptr);
        for (int b = 0; b < n; ++b)
            if (b != tr.root && res.ebf[b] >= 100.0) ++res.bus;
    } else {
        res.lrt = 0.0; res.p_value = 2.0 / 3.0;
    }
    // meme.hpp:607-634
    const double d_fel = 2.0 * (res.lnl_meme - res.lnl_fel);
    res.p_vs_fel = d_fel > 0.0 ? std::exp(-d_fel / 2.0) : 1.0;
    const double test_rate = (res.p1 * (res.alpha * mu_s + res.beta1 * mu_n) + res.p_plus * (res.alpha * mu_s + res.beta_plus * mu_n)) / 3.0;
    const double bg_rate = has_bg ? (res.alpha * mu_s + (res.beta_bg > 0.0 ? res.beta_bg : res.beta1) * mu_n) / 3.0 : test_rate;
    double tbl = 0.0;
    for (int b = 0; b < n; ++b)
        if (b != tr.root) tbl += bl[b] * ((has_bg && !tested[b]) ? bg_rate : test_rate);
    res.total_bl = tbl;
    return res;
}

// meme.hpp:166-632 with num_background == 0
inline MemeSite meme_pattern(const Tree& tr, const Alignment& a, const std::vector<int>& l2t, const Params& base,
                             const MemeRun& run, int p) {
    const FelSite& f = run.fel.patterns[p];
    const MemeFelStart fs{f.alpha, f.beta, 0.0, f.alpha_null, f.lnl_alt};
    return meme_pattern_tested(tr, a, l2t, base, run.fel.bl, {}, fs, run.mu_s, run.mu_n, p);
}

// meme.hpp:150-164, :620-660 (run): FEL baseline then MEME for every pattern, in parallel
inline MemeRun meme_run(const Tree& tr, const Alignment& a, const Params& base, int max_patterns = -1) {
    MemeRun run;
    run.fel = fel_run(tr, a, base, max_patterns);
    Params ps = base; ps.alpha = 1.0; ps.beta = 0.0;
    Params pn = base; pn.alpha = 0.0; pn.beta = 1.0;
    MG94 ms, mn;
    ms.update(ps, a.pos_freq, a.pi, a.code);
    mn.update(pn, a.pos_freq, a.pi, a.code);
    run.mu_s = ms.mu; run.mu_n = mn.mu;
    const auto l2t = leaf_map(tr, a);
    const int P = int(run.fel.patterns.size());
    run.patterns.assign(P, MemeSite{});
    #pragma omp parallel for schedule(dynamic) num_threads(n_threads_for(P))
    for (int p = 0; p < P; ++p) run.patterns[p] = meme_pattern(tr, a, l2t, base, run, p);
    return run;
}

// meme.hpp:84-92, :150-164, :620-660 with branch sets: tested (MEME) and fel_tested (its FEL baseline,
// partitioned with {T}-tag detection in the reference); every length converted by the base model's rate
struct MemeTestedRun {
    std::vector<double> bl;
    std::vector<MemeFelStart> fel;
    double mu_s = 0, mu_n = 0;
    std::vector<MemeSite> patterns;
};
inline MemeTestedRun meme_run_tested(const Tree& tr, const Alignment& a, const Params& base, const std::vector<char>& tested,
                                     const std::vector<char>& fel_tested, int max_patterns = -1) {
    MemeTestedRun run;
    const FelRun fr = fel_prepare(tr, a, base);
    run.bl = fr.bl;
    bool fel_bg = false;
    for (int i = 0; i < tr.n(); ++i) if (i != tr.root && !fel_tested[i]) fel_bg = true;
    FelSubsetRun sr;
    sr.bl = fr.bl; sr.tested = fel_tested; sr.conversion = sr.bg_conversion = fr.conversion;
    Params ps = base; ps.alpha = 1.0; ps.beta = 0.0;
    Params pn = base; pn.alpha = 0.0; pn.beta = 1.0;
    MG94 ms, mn;
    ms.update(ps, a.pos_freq, a.pi, a.code);
    mn.update(pn, a.pos_freq, a.pi, a.code);
    run.mu_s = ms.mu; run.mu_n = mn.mu;
    const auto l2t = leaf_map(tr, a);
    const int P = max_patterns < 0 ? a.P : std::min(a.P, max_patterns);
    run.fel.assign(P, MemeFelStart{});
    run.patterns.assign(P, MemeSite{});
    #pragma omp parallel for schedule(dynamic) num_threads(n_threads_for(P))
    for (int p = 0; p < P; ++p) {
        if (fel_bg) {
            const FelSubsetSite f = fel_pattern_subset(tr, a, l2t, base, sr, p);
            run.fel[p] = MemeFelStart{f.alpha, f.beta, f.beta_nuisance, f.alpha_null, f.lnl_alt};
        } else {
            const FelSite f = fel_pattern(tr, a, l2t, base, fr, p);
            run.fel[p] = MemeFelStart{f.alpha, f.beta, 0.0, f.alpha_null, f.lnl_alt};
        }
        run.patterns[p] = meme_pattern_tested(tr, a, l2t, base, run.bl, tested, run.fel[p], run.mu_s, run.mu_n, p);
    }
    return run;
}

// ------------------------------------------------------------ BUSTED E-steps
// busted.hpp:509-660 (evaluate_log_l), :662-975 (compute_expected_weights) and
// :978-1134 (compute_expected_syn_weights) without the error sink (eps_sink = 0)
// and without bridge resolutions.  Test branches mix the K omega classes at
// the P level, other branches use the background model; synonymous-rate
// classes are separate passes combined per site by log-sum-exp.  bl are the
// branch lengths already multiplied by s (raw time, alpha_m * bl per class).
struct BustedEStep {
    double lnl = 0.0;
    std::vector<double> weights, syn_weights, pattern_ll;
};
inline BustedEStep busted_estep(const Tree& tr, const Alignment& a, const Params& base, const std::vector<double>& bl,
                                const std::vector<double>& omegas, const std::vector<double>& weights,
                                const std::vector<double>& syn_rates, const std::vector<double>& syn_weights,
                                const std::vector<char>& is_test, double omega_bg) {
    const int S = a.code.S, n = tr.n(), P = a.P, K = int(omegas.size()), M = int(syn_rates.size());
    const auto l2t = leaf_map(tr, a);
    auto test = [&](int b) { return is_test.empty() ? b != tr.root : bool(is_test[b]); };
    int n_test = 0;
    for (int b = 0; b < n; ++b) if (b != tr.root && test(b)) ++n_test;
    std::vector<MG94> mk(K);
    for (int k = 0; k < K; ++k) { Params q = base; q.alpha = 1.0; q.beta = omegas[k]; mk[k].update(q, a.pos_freq, a.pi, a.code); }
    MG94 mbg;
    if (n_test + 1 < n) { Params q = base; q.alpha = 1.0; q.beta = omega_bg; mbg.update(q, a.pos_freq, a.pi, a.code); }
    std::vector<std::vector<std::vector<Mat>>> Pc(M, std::vector<std::vector<Mat>>(K, std::vector<Mat>(n, Mat::eye(S))));
    std::vector<std::vector<Mat>> Pmix(M, std::vector<Mat>(n, Mat::eye(S)));
    for (int m = 0; m < M; ++m)
        for (int b = 0; b < n; ++b) {
            if (b == tr.root) continue;
            const double t = syn_rates[m] * bl[b];
            for (int k = 0; k < K; ++k) Pc[m][k][b] = mk[k].P(t);
            if (test(b)) {
                Pmix[m][b] = Mat(S, S);
                for (int k = 0; k < K; ++k)
                    for (size_t e = 0; e < Pmix[m][b].a.size(); ++e) Pmix[m][b].a[e] += weights[k] * Pc[m][k][b].a[e];
            } else {
                Pmix[m][b] = mbg.P(t);
            }
        }
    BustedEStep r;
    r.pattern_ll.assign(P, -1e20);
    std::vector<std::vector<double>> wacc(K, std::vector<double>(P, 0.0)), sacc(M, std::vector<double>(P, 0.0));
    std::vector<double> wt_w(P, 0.0), wt_s(P, 0.0);
    #pragma omp parallel num_threads(n_threads_for(P))
    {
        std::vector<Pass> w(M);
        std::vector<double> pd(S);
        #pragma omp for schedule(static)
        for (int p = 0; p < P; ++p) {
            const double wt = a.weights[p];
            std::vector<double> post(M, 0.0);
            double mx = -1e300;
            for (int m = 0; m < M; ++m) {
                if (syn_weights[m] <= 1e-12 && M > 1) continue;
                inside_outside(tr, a, p, l2t, Pmix[m], a.pi, S, w[m], true);
                if (w[m].L > 0.0) mx = std::max(mx, (M > 1 ? std::log(syn_weights[m]) : 0.0) + w[m].logL);
            }
            if (!(mx > -1e19)) continue;
            double se = 0.0;
            for (int m = 0; m < M; ++m)
                if ((M == 1 || syn_weights[m] > 1e-12) && w[m].L > 0.0) { post[m] = std::exp((M > 1 ? std::log(syn_weights[m]) : 0.0) + w[m].logL - mx); se += post[m]; }
            if (!(se > 0.0)) continue;
            r.pattern_ll[p] = M == 1 ? w[0].logL : mx + std::log(se);
            for (int m = 0; m < M; ++m) { post[m] /= se; sacc[m][p] = wt * post[m]; }
            wt_s[p] = wt;
            // busted.hpp:822-860: per test branch and class, w_k * post_m * V . (P_k D) / L_m
            for (int b = 0; b < n; ++b) {
                if (b == tr.root || !test(b)) continue;
                for (int k = 0; k < K; ++k)
                    for (int m = 0; m < M; ++m) {
                        if (post[m] <= 1e-12 || !(w[m].L > 0.0)) continue;
                        matvec(Pc[m][k][b], w[m].D[b].data(), pd.data());
                        double dot = 0.0;
                        for (int i = 0; i < S; ++i) dot += w[m].V[b][i] * pd[i];
                        wacc[k][p] += wt * weights[k] * post[m] * dot / w[m].L;
                    }
                wt_w[p] += wt;
            }
        }
    }
    Neumaier ll;
    for (int p = 0; p < P; ++p) ll.add(a.weights[p] * r.pattern_ll[p]);
    r.lnl = ll.value();
    auto normalise = [](std::vector<double> acc, double total, const std::vector<double>& old) {
        if (!(total > 0.0)) return old;
        double sum = 0.0;
        for (auto& x : acc) { x = std::clamp(x / total, 1e-6, 1.0 - 1e-6); sum += x; }
        for (auto& x : acc) x /= sum;
        return acc;
    };
    std::vector<double> wk(K, 0.0), sm(M, 0.0);
    double tw = 0.0, ts = 0.0;
    for (int p = 0; p < P; ++p) {
        for (int k = 0; k < K; ++k) wk[k] += wacc[k][p];
        for (int m = 0; m < M; ++m) sm[m] += sacc[m][p];
        tw += wt_w[p];
        ts += wt_s[p];
    }
    r.weights = K <= 1 ? std::vector<double>{1.0} : normalise(wk, tw, weights);
    r.syn_weights = M <= 1 ? std::vector<double>{1.0} : normalise(sm, ts, syn_weights);
    return r;
}

} // namespace h3o
