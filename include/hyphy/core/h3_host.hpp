// h3_host.hpp — host-side data model for the B200 likelihood core.
//
// Mirrors the reference's public core types so callers of
// hyphy::core::LikelihoodEngine keep their code:
//   GeneticCode      genetic_code.hpp:14-200  (sense codons, StepDiff table, IUPAC masks)
//   Alignment        alignment.hpp:33-1078    (FASTA / NEXUS loading, CF3x4, pattern compression)
//   Tree / TreeNode  tree.hpp:22-892          (Newick parsing, node ids, post-order, unrooting)
//   MG94Parameters   rate_matrix.hpp:106-118
//   MG94Matrix       rate_matrix.hpp:120-258  (generator, symmetric eigensystem, P(t))
// Dense matrices are a small row-major type (no Eigen); the symmetric
// eigensolver is Householder tridiagonalisation followed by implicit-shift QL
// (Wilkinson & Reinsch, Handbook for Automatic Computation vol. II, tred2/tql2).
#pragma once

#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <memory>
#include <regex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace hyphy::core {

using Scalar = double;
constexpr int32_t INVALID_INDEX = -1;

// ------------------------------------------------------------------ dense
struct Matrix {
    int rows_ = 0, cols_ = 0;
    std::vector<double> v;
    Matrix() = default;
    Matrix(int r, int c, double x = 0.0) : rows_(r), cols_(c), v(size_t(r) * c, x) {}
    static Matrix Identity(int n) { Matrix m(n, n); for (int i = 0; i < n; ++i) m(i, i) = 1.0; return m; }
    static Matrix Zero(int r, int c) { return Matrix(r, c); }
    int rows() const { return rows_; }
    int cols() const { return cols_; }
    double& operator()(int i, int j) { return v[size_t(i) * cols_ + j]; }
    double operator()(int i, int j) const { return v[size_t(i) * cols_ + j]; }
    const double* data() const { return v.data(); }
    double* data() { return v.data(); }
};
using Vector = std::vector<double>;

// ------------------------------------------------------------- nucleotides
inline constexpr int8_t char_to_nuc(char c) {
    switch (c) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': case 'U': case 'u': return 3;
        default: return -1;
    }
}
// IUPAC ambiguity code -> 4-bit set over {A,C,G,T}; anything unknown is all four.
inline uint8_t char_to_iupac_mask(char c) {
    static const std::array<uint8_t, 26> tab = [] {
        std::array<uint8_t, 26> t{};
        t.fill(0xF);
        auto put = [&](char ch, uint8_t m) { t[ch - 'A'] = m; };
        put('A', 1); put('C', 2); put('G', 4); put('T', 8); put('U', 8);
        put('R', 1 | 4); put('Y', 2 | 8); put('S', 2 | 4); put('W', 1 | 8); put('K', 4 | 8); put('M', 1 | 2);
        put('B', 2 | 4 | 8); put('D', 1 | 4 | 8); put('H', 1 | 2 | 8); put('V', 1 | 2 | 4);
        return t;
    }();
    unsigned char u = static_cast<unsigned char>(std::toupper(static_cast<unsigned char>(c)));
    return (u >= 'A' && u <= 'Z') ? tab[u - 'A'] : uint8_t(0xF);
}

// ------------------------------------------------------------ genetic code
class GeneticCode {
public:
    struct StepDiff {
        int8_t num_diffs = 0;
        bool synonymous = false;
        int8_t diff_pos[3] = {-1, -1, -1};
        int8_t diff_from[3] = {-1, -1, -1};
        int8_t diff_to[3] = {-1, -1, -1};
    };
    std::string name;
    int num_sense_codons = 0;
    std::vector<std::string> sense_codons;
    std::vector<char> sense_codon_aa;
    int8_t codon64_to_sense[64];
    std::vector<std::vector<StepDiff>> diff_matrix;

    // `aa64` lists the amino acid of each codon in A,C,G,T-major order
    // (index 16*n1 + 4*n2 + n3), '*' marking stops.
    GeneticCode(std::string nm, const std::string& aa64) : name(std::move(nm)) {
        static const char N[4] = {'A', 'C', 'G', 'T'};
        for (int c = 0; c < 64; ++c) {
            codon64_to_sense[c] = -1;
            if (aa64[c] == '*') continue;
            codon64_to_sense[c] = int8_t(sense_codons.size());
            sense_codons.push_back(std::string{N[c >> 4], N[(c >> 2) & 3], N[c & 3]});
            sense_codon_aa.push_back(aa64[c]);
        }
        num_sense_codons = int(sense_codons.size());
        const int S = num_sense_codons;
        diff_matrix.assign(S, std::vector<StepDiff>(S));
        for (int a = 0; a < S; ++a)
            for (int b = 0; b < S; ++b) {
                if (a == b) continue;
                StepDiff& d = diff_matrix[a][b];
                for (int p = 0; p < 3; ++p)
                    if (sense_codons[a][p] != sense_codons[b][p]) {
                        d.diff_pos[d.num_diffs] = int8_t(p);
                        d.diff_from[d.num_diffs] = char_to_nuc(sense_codons[a][p]);
                        d.diff_to[d.num_diffs] = char_to_nuc(sense_codons[b][p]);
                        ++d.num_diffs;
                    }
                d.synonymous = sense_codon_aa[a] == sense_codon_aa[b];
            }
    }

    uint64_t all_sense_mask() const { return num_sense_codons >= 64 ? ~uint64_t(0) : ((uint64_t(1) << num_sense_codons) - 1); }

    int8_t triplet_to_sense(char c1, char c2, char c3) const {
        int a = char_to_nuc(c1), b = char_to_nuc(c2), c = char_to_nuc(c3);
        if ((a | b | c) < 0) return -1;
        return codon64_to_sense[16 * a + 4 * b + c];
    }

    // Set of sense codons compatible with an ambiguous triplet; stops, gaps and
    // all-N resolve to every sense codon (genetic_code.hpp:82-109).
    uint64_t resolve_triplet_mask(char c1, char c2, char c3) const {
        const uint64_t all = all_sense_mask();
        if (c1 == '!' || c2 == '!' || c3 == '!') return all;
        const uint8_t m[3] = {char_to_iupac_mask(c1), char_to_iupac_mask(c2), char_to_iupac_mask(c3)};
        if (m[0] == 0xF && m[1] == 0xF && m[2] == 0xF) return all;
        uint64_t out = 0;
        for (int c = 0; c < 64; ++c)
            if ((m[0] >> (c >> 4) & 1) && (m[1] >> ((c >> 2) & 3) & 1) && (m[2] >> (c & 3) & 1) && codon64_to_sense[c] >= 0)
                out |= uint64_t(1) << codon64_to_sense[c];
        return out ? out : all;
    }

    static std::shared_ptr<const GeneticCode> universal() { return from_name("Universal"); }
    static std::shared_ptr<const GeneticCode> from_name(const std::string& nm) {
        std::string k = nm;
        std::transform(k.begin(), k.end(), k.begin(), ::tolower);
        static const std::string standard = standard_acgt();
        static auto uni = std::make_shared<const GeneticCode>("Universal", standard);
        static auto vmt = std::make_shared<const GeneticCode>("Vertebrate-mtDNA", vertebrate_mt(standard));
        if (k == "universal" || k == "standard" || k == "default" || k == "1" || k == "transl_table=1") return uni;
        if (k == "vertebrate-mtdna" || k == "vertebrate_mtdna" || k == "2" || k == "transl_table=2") return vmt;
        throw std::runtime_error("Unknown genetic code: '" + nm + "'");
    }

private:
    // NCBI translation table 1, re-indexed from its customary T,C,A,G print order.
    static std::string standard_acgt() {
        const char* tcag = "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG";
        const int pos[4] = {2, 1, 3, 0};
        std::string s(64, '?');
        for (int c = 0; c < 64; ++c) s[c] = tcag[16 * pos[c >> 4] + 4 * pos[(c >> 2) & 3] + pos[c & 3]];
        return s;
    }
    static std::string vertebrate_mt(std::string s) {
        auto at = [&](const char* t) -> char& { return s[16 * char_to_nuc(t[0]) + 4 * char_to_nuc(t[1]) + char_to_nuc(t[2])]; };
        at("AGA") = '*'; at("AGG") = '*'; at("ATA") = 'M'; at("TGA") = 'W';
        return s;
    }
};

// --------------------------------------------------------------- alignment
struct SitePattern {
    std::vector<int8_t> states;            // sense index per taxon, -1 when not a resolved sense codon
    std::vector<uint64_t> ambiguous_masks; // compatible sense codons per taxon
    size_t weight = 0;
    std::vector<size_t> sites;
};

struct Sequence {
    std::string name;
    std::string raw_seq;
};

class Alignment {
public:
    std::vector<std::string> taxon_names;
    std::vector<Sequence> sequences;
    size_t num_taxa = 0, num_codons = 0, num_nucleotides = 0;
    std::shared_ptr<const GeneticCode> code;
    std::string embedded_tree_newick;
    std::vector<SitePattern> patterns;
    std::vector<size_t> site_to_pattern;
    double nuc_frequencies[4] = {0, 0, 0, 0};
    double pos_nuc_frequencies[3][4] = {};   // CF3x4-corrected positional frequencies
    Vector codon_frequencies_f3x4;

    void add_sequence(const std::string& nm, const std::string& seq) {
        taxon_names.push_back(nm);
        sequences.push_back({nm, seq});
    }

    static Alignment load(const std::string& path, std::shared_ptr<const GeneticCode> gc = nullptr) {
        std::ifstream f(path, std::ios::binary);
        if (!f) throw std::runtime_error("Could not open alignment file: " + path);
        std::stringstream ss; ss << f.rdbuf();
        return from_text(ss.str(), gc);
    }
    static Alignment from_fasta(const std::string& path) { return load(path); }
    static Alignment from_nexus(const std::string& path) { return load(path); }

    // finalize = false leaves the sequences as read (load_unfinalized, alignment.hpp:648-650)
    static Alignment from_text(const std::string& text, std::shared_ptr<const GeneticCode> gc = nullptr, bool finalize = true) {
        Alignment a;
        size_t b = text.find_first_not_of(" \t\r\n");
        if (b != std::string::npos && (text.compare(b, 6, "#NEXUS") == 0 || text.compare(b, 6, "#nexus") == 0))
            a.read_nexus(text);
        else
            a.read_fasta(text);
        if (finalize) a.finalize(gc);
        else if (gc) a.code = gc;
        return a;
    }
    static Alignment load_unfinalized(const std::string& path) {
        std::ifstream f(path, std::ios::binary);
        if (!f) throw std::runtime_error("Could not open alignment file: " + path);
        std::stringstream ss; ss << f.rdbuf();
        return from_text(ss.str(), nullptr, false);
    }

    // alignment.hpp:665-723
    void finalize(std::shared_ptr<const GeneticCode> gc = nullptr) {
        code = gc ? gc : (code ? code : GeneticCode::universal());
        if (sequences.empty()) throw std::runtime_error("Empty alignment");
        num_taxa = sequences.size();
        num_nucleotides = sequences[0].raw_seq.size();
        taxon_names.clear();
        for (auto& s : sequences) {
            if (s.raw_seq.size() != num_nucleotides) throw std::runtime_error("Sequences have unequal lengths in alignment");
            taxon_names.push_back(s.name);
        }
        if (num_nucleotides % 3) throw std::runtime_error("Nucleotide alignment length is not a multiple of 3 (in-frame codons required)");
        num_codons = num_nucleotides / 3;
        compute_frequencies();
        compress_patterns();
    }

    size_t taxon_index(const std::string& raw) const {
        std::string nm = raw;
        if (nm.size() >= 2 && (nm.front() == '\'' || nm.front() == '"') && nm.back() == nm.front()) nm = nm.substr(1, nm.size() - 2);
        auto low = [](std::string s) { for (auto& c : s) c = char(std::tolower(static_cast<unsigned char>(c))); return s; };
        for (size_t i = 0; i < taxon_names.size(); ++i) if (taxon_names[i] == nm) return i;
        std::string ln = low(nm);
        for (size_t i = 0; i < taxon_names.size(); ++i) if (low(taxon_names[i]) == ln) return i;
        if (ln.size() >= 3) {
            size_t hit = size_t(-1), count = 0;
            for (size_t i = 0; i < taxon_names.size(); ++i) {
                std::string ls = low(taxon_names[i]);
                bool pre = (ls.size() > ln.size() && ls.compare(0, ln.size(), ln) == 0) ||
                           (ls.size() >= 3 && ln.size() > ls.size() && ln.compare(0, ls.size(), ls) == 0);
                if (pre) { hit = i; ++count; }
            }
            if (count == 1) return hit;
        }
        return size_t(-1);
    }

private:
    void read_fasta(const std::string& text) {
        std::istringstream in(text);
        std::string line;
        while (std::getline(in, line)) {
            if (!line.empty() && line.back() == '\r') line.pop_back();
            if (line.empty()) continue;
            if (line[0] == '>') {
                size_t s = line.find_first_not_of(" \t", 1), e = line.find_last_not_of(" \t");
                add_sequence(s == std::string::npos ? "" : line.substr(s, e - s + 1), "");
            } else if (!sequences.empty()) {
                for (char c : line) if (!std::isspace(static_cast<unsigned char>(c))) sequences.back().raw_seq += c;
            }
        }
    }

    // NEXUS subset: TAXLABELS, MATRIX (sequential or interleaved) and the first TREE statement.
    void read_nexus(const std::string& raw) {
        std::string body;
        body.reserve(raw.size());
        int depth = 0; char quote = 0;
        for (char c : raw) {
            if (quote) { body += c; if (c == quote) quote = 0; continue; }
            if (!depth && (c == '\'' || c == '"')) { quote = c; body += c; continue; }
            if (c == '[') { ++depth; continue; }
            if (c == ']' && depth) { --depth; continue; }
            if (!depth) body += (c == '\r' ? '\n' : c);
        }
        std::string up(body);
        for (auto& c : up) c = char(std::toupper(static_cast<unsigned char>(c)));
        struct Tok { std::string s; bool line_start; };
        auto lex = [](std::string_view sv) {
            std::vector<Tok> out; bool ls = true;
            for (size_t i = 0; i < sv.size();) {
                char c = sv[i];
                if (c == '\n') { ls = true; ++i; continue; }
                if (std::isspace(static_cast<unsigned char>(c))) { ++i; continue; }
                size_t j = i;
                if (c == '\'' || c == '"') { j = sv.find(c, i + 1); j = (j == std::string_view::npos) ? sv.size() : j + 1; }
                else while (j < sv.size() && !std::isspace(static_cast<unsigned char>(sv[j]))) ++j;
                out.push_back({std::string(sv.substr(i, j - i)), ls});
                ls = false; i = j;
            }
            return out;
        };
        auto unquote = [](std::string s) {
            if (s.size() >= 2 && (s[0] == '\'' || s[0] == '"') && s.back() == s[0]) s = s.substr(1, s.size() - 2);
            return s;
        };
        std::unordered_map<std::string, size_t> row;
        size_t tl = up.find("TAXLABELS");
        if (tl != std::string::npos) {
            size_t e = up.find(';', tl);
            for (auto& t : lex(std::string_view(body).substr(tl + 9, e - tl - 9))) {
                std::string nm = unquote(t.s);
                row.emplace(nm, sequences.size());
                add_sequence(nm, "");
            }
        }
        const bool labelled = !row.empty();
        size_t mx = up.find("MATRIX");
        if (mx == std::string::npos) throw std::runtime_error("NEXUS file has no MATRIX block");
        size_t me = body.find(';', mx);
        long cur = -1;
        for (auto& t : lex(std::string_view(body).substr(mx + 6, me - mx - 6))) {
            std::string nm = unquote(t.s);
            auto it = row.find(nm);
            bool is_label = labelled ? it != row.end() : t.line_start;
            if (is_label) {
                if (it == row.end()) { it = row.emplace(nm, sequences.size()).first; add_sequence(nm, ""); }
                cur = long(it->second);
            } else if (cur >= 0) {
                sequences[size_t(cur)].raw_seq += t.s;
            }
        }
        size_t tb = up.find("BEGIN TREES");
        if (tb != std::string::npos) {
            size_t ts = up.find("TREE ", tb + 11);
            if (ts != std::string::npos) {
                size_t eq = body.find('=', ts), sc = body.find(';', eq);
                std::string nw = body.substr(eq + 1, sc - eq - 1);
                size_t s = nw.find_first_not_of(" \t\n");
                embedded_tree_newick = (s == std::string::npos ? std::string() : nw.substr(s)) + ";";
            }
        }
    }

    // alignment.hpp:893-1019 — empirical nucleotide and positional frequencies, then CF3x4.
    void compute_frequencies() {
        double pc[3][4] = {};
        for (auto& s : sequences)
            for (size_t i = 0; i < 3 * num_codons; ++i) {
                int n = char_to_nuc(s.raw_seq[i]);
                if (n >= 0) pc[i % 3][n] += 1;
            }
        frequencies_from_counts(pc);
    }

public:
    // alignment.hpp:832-890: the nucleotide patterns of this alignment (num_codons = 0): per site
    // the IUPAC set of every taxon is the key, state = the unambiguous nucleotide or -1, mask = the
    // set; patterns in first-occurrence order; this alignment's nucleotide frequencies are kept.
    Alignment to_nucleotide_alignment() const {
        if (num_codons == 0 && !patterns.empty()) return *this;
        Alignment r;
        r.taxon_names = taxon_names;
        r.sequences = sequences;
        r.num_taxa = num_taxa;
        r.num_nucleotides = num_nucleotides;
        r.num_codons = 0;
        r.code = code;
        r.embedded_tree_newick = embedded_tree_newick;
        std::copy(nuc_frequencies, nuc_frequencies + 4, r.nuc_frequencies);
        std::unordered_map<std::string, size_t> seen;
        r.site_to_pattern.assign(num_nucleotides, 0);
        std::string key(num_taxa, 'N');
        for (size_t site = 0; site < num_nucleotides; ++site) {
            for (size_t t = 0; t < num_taxa; ++t) key[t] = char('A' + char_to_iupac_mask(sequences[t].raw_seq[site]));
            auto [it, fresh] = seen.emplace(key, r.patterns.size());
            if (fresh) {
                SitePattern p;
                p.states.resize(num_taxa);
                p.ambiguous_masks.resize(num_taxa);
                for (size_t t = 0; t < num_taxa; ++t) {
                    const char ch = sequences[t].raw_seq[site];
                    p.states[t] = char_to_nuc(ch);
                    p.ambiguous_masks[t] = char_to_iupac_mask(ch);
                }
                r.patterns.push_back(std::move(p));
            }
            r.patterns[it->second].weight += 1;
            r.patterns[it->second].sites.push_back(site);
            r.site_to_pattern[site] = it->second;
        }
        return r;
    }

    // alignment.hpp:911-1019 from the counts of unambiguous nucleotides per codon position
    void frequencies_from_counts(const double pc[3][4]) {
        double nc[4];
        for (int b = 0; b < 4; ++b) nc[b] = pc[0][b] + pc[1][b] + pc[2][b];
        auto floor_norm = [](double* f) {
            bool pad = false;
            for (int b = 0; b < 4; ++b) if (f[b] < 1e-8) { f[b] = 1e-8; pad = true; }
            if (pad) { double z = f[0] + f[1] + f[2] + f[3]; for (int b = 0; b < 4; ++b) f[b] /= z; }
        };
        double tot = nc[0] + nc[1] + nc[2] + nc[3];
        for (int b = 0; b < 4; ++b) nuc_frequencies[b] = tot > 0 ? nc[b] / tot : 0.0;
        floor_norm(nuc_frequencies);
        double target[3][4];
        for (int p = 0; p < 3; ++p) {
            double z = pc[p][0] + pc[p][1] + pc[p][2] + pc[p][3];
            for (int b = 0; b < 4; ++b) target[p][b] = z > 0 ? pc[p][b] / z : 0.0;
            floor_norm(target[p]);
        }
        const int S = code->num_sense_codons;
        std::vector<std::array<int, 3>> nucs(S);
        for (int s = 0; s < S; ++s)
            for (int p = 0; p < 3; ++p) nucs[s][p] = char_to_nuc(code->sense_codons[s][p]);
        codon_frequencies_f3x4.assign(S, 0.0);
        double x[3][4];
        std::copy(&target[0][0], &target[0][0] + 12, &x[0][0]);
        auto codon_product = [&]() {
            double z = 0;
            for (int s = 0; s < S; ++s) z += (codon_frequencies_f3x4[s] = x[0][nucs[s][0]] * x[1][nucs[s][1]] * x[2][nucs[s][2]]);
            if (z > 0) for (auto& v : codon_frequencies_f3x4) v /= z;
        };
        // fixed point: rescale positional weights until the sense-codon marginals match the
        // empirical positional frequencies (at most 200 steps, 1e-14 tolerance)
        for (int it = 0; it < 200; ++it) {
            double prev[3][4];
            std::copy(&x[0][0], &x[0][0] + 12, &prev[0][0]);
            codon_product();
            double marg[3][4] = {};
            for (int s = 0; s < S; ++s) for (int p = 0; p < 3; ++p) marg[p][nucs[s][p]] += codon_frequencies_f3x4[s];
            double change = 0;
            for (int p = 0; p < 3; ++p) {
                for (int b = 0; b < 4; ++b) x[p][b] *= target[p][b] / std::max(marg[p][b], 1e-12);
                double z = x[p][0] + x[p][1] + x[p][2] + x[p][3];
                if (z > 0) for (int b = 0; b < 4; ++b) x[p][b] /= z;
                for (int b = 0; b < 4; ++b) change = std::max(change, std::fabs(x[p][b] - prev[p][b]));
            }
            if (change < 1e-14) break;
        }
        codon_product();
        std::copy(&x[0][0], &x[0][0] + 12, &pos_nuc_frequencies[0][0]);
    }

private:
    // alignment.hpp:1021-1078 — unique columns in first-occurrence order.
    void compress_patterns() {
        const size_t T = num_taxa;
        std::vector<int8_t> st(T * num_codons);
        std::vector<uint64_t> mk(T * num_codons);
        for (size_t t = 0; t < T; ++t)
            for (size_t c = 0; c < num_codons; ++c) {
                const char* x = &sequences[t].raw_seq[3 * c];
                int8_t s = code->triplet_to_sense(x[0], x[1], x[2]);
                st[c * T + t] = s;
                mk[c * T + t] = s >= 0 ? (uint64_t(1) << s) : code->resolve_triplet_mask(x[0], x[1], x[2]);
            }
        struct Key { const int8_t* s; const uint64_t* m; size_t T; };
        struct Hash {
            size_t operator()(const Key& k) const {
                uint64_t h = 1469598103934665603ull;
                for (size_t i = 0; i < k.T; ++i) { h ^= uint64_t(uint8_t(k.s[i])) + (k.m[i] * 0x9E3779B97F4A7C15ull); h *= 1099511628211ull; }
                return size_t(h);
            }
        };
        struct Eq {
            bool operator()(const Key& a, const Key& b) const {
                return std::equal(a.s, a.s + a.T, b.s) && std::equal(a.m, a.m + a.T, b.m);
            }
        };
        std::unordered_map<Key, size_t, Hash, Eq> seen;
        patterns.clear();
        site_to_pattern.assign(num_codons, 0);
        for (size_t c = 0; c < num_codons; ++c) {
            Key k{&st[c * T], &mk[c * T], T};
            auto [it, fresh] = seen.emplace(k, patterns.size());
            if (fresh) {
                SitePattern p;
                p.states.assign(k.s, k.s + T);
                p.ambiguous_masks.assign(k.m, k.m + T);
                patterns.push_back(std::move(p));
            }
            patterns[it->second].weight += 1;
            patterns[it->second].sites.push_back(c);
            site_to_pattern[c] = it->second;
        }
    }
};

// -------------------------------------------------------------------- tree
struct TreeNode {
    int32_t id = INVALID_INDEX;
    std::string name;
    int32_t parent_id = INVALID_INDEX;
    std::vector<int32_t> children;
    Scalar branch_length = 0.0;
    bool is_leaf = false;
    std::string model_tag;
};

class Tree {
public:
    std::vector<TreeNode> nodes;
    int32_t root_id = INVALID_INDEX;
    std::vector<int32_t> post_order;
    std::unordered_map<std::string, int32_t> leaf_name_to_id;

    size_t num_nodes() const { return nodes.size(); }
    size_t num_leaves() const { return leaf_name_to_id.size(); }

    static Tree from_newick_file(const std::string& path, bool keep_rooted = true) {
        std::ifstream f(path);
        if (!f) throw std::runtime_error("Could not open Newick file: " + path);
        std::stringstream ss; ss << f.rdbuf();
        return from_newick(ss.str(), keep_rooted);
    }

    // Node ids follow the order in which the Newick text introduces nodes: an
    // opening parenthesis creates an internal node, a label before ',' or ')'
    // creates a leaf (tree.hpp:273-585).  The ids index branch-length and
    // gradient vectors, so they must match the reference's.
    static Tree from_newick(std::string_view text, bool keep_rooted = true) {
        std::string s;
        {
            bool comment = false; char quote = 0;
            for (char c : text) {
                if (quote) { s += c; if (c == quote) quote = 0; continue; }
                if (comment) { if (c == ']') comment = false; continue; }
                if (c == '[') { comment = true; continue; }
                if (c == '\'' || c == '"') { quote = c; s += c; continue; }
                if (!std::isspace(static_cast<unsigned char>(c))) s += c;
            }
            while (!s.empty() && s.back() == ';') s.pop_back();
        }
        Tree tr;
        std::vector<int32_t> open;
        auto new_node = [&](bool leaf) {
            TreeNode nd; nd.id = int32_t(tr.nodes.size()); nd.is_leaf = leaf;
            if (!open.empty()) { nd.parent_id = open.back(); tr.nodes[size_t(open.back())].children.push_back(nd.id); }
            tr.nodes.push_back(nd);
            return nd.id;
        };
        auto scan_label = [&](size_t i) {   // returns one past the label starting at i
            char quote = 0;
            for (; i < s.size(); ++i) {
                char c = s[i];
                if (quote) { if (c == quote) quote = 0; continue; }
                if (c == '\'' || c == '"') { quote = c; continue; }
                if (c == ',' || c == ')' || c == '(' || c == ';') break;
            }
            if (quote) throw std::runtime_error("Invalid Newick tree: unterminated quoted label");
            return i;
        };
        size_t i = 0;
        while (i < s.size()) {
            char c = s[i];
            if (c == ';') break;
            if (c == '(') { open.push_back(new_node(false)); ++i; continue; }
            if (c == ',') { ++i; continue; }
            if (c == ')') {
                if (open.empty()) throw std::runtime_error("Invalid Newick tree: unbalanced parentheses");
                int32_t id = open.back(); open.pop_back();
                size_t e = scan_label(i + 1);
                tr.apply_label(id, s.substr(i + 1, e - i - 1));
                i = e; continue;
            }
            size_t e = scan_label(i);
            int32_t id = new_node(true);
            tr.apply_label(id, s.substr(i, e - i));
            i = e;
        }
        if (!open.empty()) throw std::runtime_error("Invalid Newick tree: unbalanced parentheses");
        if (tr.nodes.empty()) throw std::runtime_error("Failed to parse Newick tree: empty tree");
        for (auto& nd : tr.nodes) if (nd.parent_id == INVALID_INDEX) tr.root_id = nd.id;
        int counter = 1;
        std::unordered_map<std::string, int> used;
        for (auto& nd : tr.nodes) if (nd.is_leaf && !nd.name.empty()) used[nd.name] = 1;
        for (auto& nd : tr.nodes) {
            if (!nd.is_leaf && (nd.name.empty() || used.count(nd.name))) {
                std::string cand;
                do cand = "Node" + std::to_string(counter++); while (used.count(cand));
                nd.name = cand;
            } else if (nd.is_leaf && nd.name.empty()) {
                std::string cand;
                do cand = "Leaf" + std::to_string(counter++); while (used.count(cand));
                nd.name = cand;
            }
            used[nd.name] = 1;
        }
        if (!keep_rooted) tr.unroot_if_bifurcating();
        tr.finish();
        return tr;
    }

    // Collapse a two-child root into a multifurcating root (tree.hpp:591-690).
    void unroot_if_bifurcating() {
        if (root_id == INVALID_INDEX || nodes.size() <= 3 || nodes[root_id].children.size() != 2) return;
        int32_t c0 = nodes[root_id].children[0], c1 = nodes[root_id].children[1];
        int32_t ab, other;
        if (!nodes[c0].is_leaf && !nodes[c1].is_leaf) {
            bool swap = nodes[c1].model_tag.empty() && !nodes[c0].model_tag.empty();
            ab = swap ? c1 : c0; other = swap ? c0 : c1;
        } else if (!nodes[c0].is_leaf) { ab = c0; other = c1; }
        else if (!nodes[c1].is_leaf) { ab = c1; other = c0; }
        else return;
        nodes[other].branch_length += nodes[ab].branch_length;
        if (nodes[other].model_tag.empty()) nodes[other].model_tag = nodes[ab].model_tag;
        std::vector<int32_t> kids;
        if (ab == c0) { kids = nodes[ab].children; kids.push_back(other); }
        else { kids.push_back(other); kids.insert(kids.end(), nodes[ab].children.begin(), nodes[ab].children.end()); }
        nodes[root_id].children = kids;
        std::vector<int32_t> remap(nodes.size(), INVALID_INDEX);
        std::vector<TreeNode> keep;
        for (auto& nd : nodes) if (nd.id != ab) { remap[size_t(nd.id)] = int32_t(keep.size()); keep.push_back(nd); }
        root_id = remap[size_t(root_id)];
        for (auto& nd : keep) {
            nd.id = remap[size_t(nd.id)];
            for (auto& c : nd.children) c = remap[size_t(c)];
        }
        for (auto& nd : keep) for (auto c : nd.children) keep[size_t(c)].parent_id = nd.id;
        keep[size_t(root_id)].parent_id = INVALID_INDEX;
        keep[size_t(root_id)].branch_length = 0.0;
        nodes = std::move(keep);
    }

    void finish() {
        leaf_name_to_id.clear();
        for (auto& nd : nodes) if (nd.is_leaf) leaf_name_to_id[nd.name] = nd.id;
        post_order.clear();
        if (root_id == INVALID_INDEX) return;
        std::vector<std::pair<int32_t, size_t>> st{{root_id, 0}};
        while (!st.empty()) {
            auto& [u, k] = st.back();
            if (k < nodes[size_t(u)].children.size()) { int32_t c = nodes[size_t(u)].children[k++]; st.push_back({c, 0}); }
            else { post_order.push_back(u); st.pop_back(); }
        }
    }

    struct BranchSelection {
        std::vector<bool> is_selected;            // per node id; the root is never selected
        std::vector<std::string> selected_names;  // in node-id order
        std::vector<std::string> unselected_names;
        size_t num_selected = 0;
        size_t num_unselected = 0;
    };

    // tree.hpp:893-1075: which branches a site analysis tests.  Precedence: a regex (matched,
    // case-insensitive, against the node name or its {tag}), then explicit names or tags, then
    // spec: "All" (every branch; with auto_detect, only the branches tagged {T}/{test}/
    // {foreground}/{fg} when any is), "all-branches", "Internal", "Leaves" / "terminal" /
    // "tips", "Unlabeled" / "untagged", a comma-separated list of names, tags and those
    // keywords, or one name or tag (a regex when nothing matches it exactly and it holds
    // regex metacharacters).  Names, tags and keywords compare case-insensitively, with
    // surrounding braces and blanks removed.
    BranchSelection select_branches(const std::string& spec = "All", const std::string& regex_str = "",
                                    const std::vector<std::string>& explicit_names = {},
                                    bool auto_detect_test_tags_when_all = false, bool throw_on_empty = true) const;

private:
    void apply_label(int32_t id, std::string tok) {
        TreeNode& nd = nodes[size_t(id)];
        size_t lb = tok.find('{'), rb = tok.find('}');
        if (lb != std::string::npos && rb != std::string::npos && rb > lb) {
            nd.model_tag = tok.substr(lb + 1, rb - lb - 1);
            tok.erase(lb, rb - lb + 1);
        }
        size_t colon = std::string::npos; char quote = 0;
        for (size_t k = 0; k < tok.size(); ++k) {
            if (quote) { if (tok[k] == quote) quote = 0; continue; }
            if (tok[k] == '\'' || tok[k] == '"') { quote = tok[k]; continue; }
            if (tok[k] == ':') { colon = k; break; }
        }
        std::string nm = tok.substr(0, colon);
        if (colon != std::string::npos) {
            try { nd.branch_length = std::stod(tok.substr(colon + 1)); } catch (...) { nd.branch_length = 0.0; }
        }
        if (nm.size() >= 2 && (nm.front() == '\'' || nm.front() == '"') && nm.back() == nm.front()) nm = nm.substr(1, nm.size() - 2);
        nd.name = nm;
    }
};

inline Tree::BranchSelection Tree::select_branches(const std::string& spec, const std::string& regex_str,
                                                   const std::vector<std::string>& explicit_names,
                                                   bool auto_detect_test_tags_when_all, bool throw_on_empty) const {
    auto lower = [](std::string s) {
        for (auto& ch : s) ch = char(std::tolower(static_cast<unsigned char>(ch)));
        return s;
    };
    auto unbrace = [](const std::string& s) {
        const auto blank = [](char ch) { return ch == ' ' || ch == '\t' || ch == '\r' || ch == '\n'; };
        size_t b = 0, e = s.size();
        while (b < e && blank(s[b])) ++b;
        while (e > b && blank(s[e - 1])) --e;
        if (e - b >= 2 && s[b] == '{' && s[e - 1] == '}') {
            ++b; --e;
            while (b < e && blank(s[b])) ++b;
            while (e > b && blank(s[e - 1])) --e;
        }
        return s.substr(b, e - b);
    };
    auto fg = [](const std::string& t) { return t == "t" || t == "test" || t == "foreground" || t == "fg"; };
    auto bg = [](const std::string& t) { return t == "r" || t == "ref" || t == "reference" || t == "background" || t == "bg"; };
    auto regex_match = [&](const std::regex& re, const TreeNode& nd) {
        return std::regex_search(nd.name, re) || (!nd.model_tag.empty() && std::regex_search(nd.model_tag, re));
    };
    BranchSelection sel;
    sel.is_selected.assign(nodes.size(), false);
    auto each = [&](auto&& pick) {
        for (const auto& nd : nodes)
            if (nd.id != root_id) sel.is_selected[size_t(nd.id)] = pick(nd);
    };
    if (!regex_str.empty()) {
        const std::regex re(regex_str, std::regex::icase);
        each([&](const TreeNode& nd) { return regex_match(re, nd); });
    } else if (!explicit_names.empty()) {
        std::unordered_set<std::string> want;
        for (const auto& item : explicit_names) {
            const std::string k = lower(unbrace(item));
            if (!k.empty()) want.insert(k);
        }
        each([&](const TreeNode& nd) {
            const std::string tag = lower(nd.model_tag);
            return want.count(lower(nd.name)) > 0 || (!tag.empty() && want.count(tag) > 0);
        });
    } else {
        const std::string mode = unbrace(spec), m = lower(mode);
        if (m.empty() || m == "all") {
            bool tagged = false;
            if (auto_detect_test_tags_when_all)
                for (const auto& nd : nodes)
                    if (nd.id != root_id && fg(lower(nd.model_tag))) tagged = true;
            each([&](const TreeNode& nd) { return tagged ? fg(lower(nd.model_tag)) : true; });
        } else if (m == "all-branches" || m == "all_branches") {
            each([](const TreeNode&) { return true; });
        } else if (m == "internal") {
            each([](const TreeNode& nd) { return !nd.is_leaf; });
        } else if (m == "leaves" || m == "terminal" || m == "tips") {
            each([](const TreeNode& nd) { return nd.is_leaf; });
        } else if (m == "unlabeled" || m == "untagged") {
            each([](const TreeNode& nd) { return nd.model_tag.empty(); });
        } else if (mode.find(',') != std::string::npos) {
            std::unordered_set<std::string> tok;
            std::stringstream ss(mode);
            for (std::string item; std::getline(ss, item, ',');) {
                const std::string k = lower(unbrace(item));
                if (!k.empty()) tok.insert(k);
            }
            auto any = [&](auto&& pred) {
                for (const auto& k : tok)
                    if (pred(k)) return true;
                return false;
            };
            each([&](const TreeNode& nd) {
                const std::string name = lower(nd.name), tag = lower(nd.model_tag);
                if (tok.count(name) || (!tag.empty() && tok.count(tag))) return true;
                if (tok.count("internal") && !nd.is_leaf) return true;
                if ((tok.count("leaves") || tok.count("terminal")) && nd.is_leaf) return true;
                if ((tok.count("unlabeled") || tok.count("untagged")) && nd.model_tag.empty()) return true;
                if (fg(tag) && any(fg)) return true;
                return bg(tag) && any(bg);
            });
        } else {
            bool hit = false;
            each([&](const TreeNode& nd) {
                const std::string name = lower(nd.name), tag = lower(nd.model_tag);
                const bool ok = (!tag.empty() && tag == m) || name == m || (fg(m) && fg(tag)) || (bg(m) && bg(tag));
                hit = hit || ok;
                return ok;
            });
            if (!hit && spec.find_first_of(".*+?^$[]()|\\") != std::string::npos) {
                try {
                    const std::regex re(spec, std::regex::icase);
                    each([&](const TreeNode& nd) { return regex_match(re, nd); });
                } catch (const std::regex_error&) {
                }
            }
        }
    }
    for (const auto& nd : nodes) {
        if (nd.id == root_id) continue;
        if (sel.is_selected[size_t(nd.id)]) {
            sel.selected_names.push_back(nd.name);
            ++sel.num_selected;
        } else {
            sel.unselected_names.push_back(nd.name);
            ++sel.num_unselected;
        }
    }
    if (throw_on_empty && sel.num_selected == 0 && nodes.size() > 1)
        throw std::runtime_error("No branches matched '--branches " + (regex_str.empty() ? spec : regex_str) + "'.");
    return sel;
}

// ----------------------------------------------------------------- MG94xREV
struct MG94Parameters {
    Scalar alpha = 1.0;
    Scalar beta = 1.0;
    Scalar theta_AC = 1.0, theta_AT = 1.0, theta_CG = 1.0, theta_CT = 1.0, theta_GT = 1.0; // theta_AG == 1
    Scalar delta = 0.0;
    Scalar psi = 0.0;
};

inline void exchangeabilities(const MG94Parameters& p, double r[4][4]) {
    const double m[4][4] = {{0, p.theta_AC, 1, p.theta_AT},
                            {p.theta_AC, 0, p.theta_CG, p.theta_CT},
                            {1, p.theta_CG, 0, p.theta_GT},
                            {p.theta_AT, p.theta_CT, p.theta_GT, 0}};
    std::copy(&m[0][0], &m[0][0] + 16, &r[0][0]);
}

// Symmetric eigendecomposition A = Z diag(d) Z^T.  Householder reduction to
// tridiagonal form followed by the implicit-shift QL iteration.
inline void symmetric_eigen(int n, std::vector<double> a, std::vector<double>& d, std::vector<double>& Z) {
    auto A = [&](int i, int j) -> double& { return a[size_t(i) * n + j]; };
    d.assign(n, 0.0);
    std::vector<double> e(n, 0.0);
    for (int j = 0; j < n; ++j) d[j] = A(n - 1, j);
    for (int i = n - 1; i > 0; --i) {
        double scale = 0.0, h = 0.0;
        for (int k = 0; k < i; ++k) scale += std::fabs(d[k]);
        if (scale == 0.0) {
            e[i] = d[i - 1];
            for (int j = 0; j < i; ++j) { d[j] = A(i - 1, j); A(i, j) = 0.0; A(j, i) = 0.0; }
        } else {
            for (int k = 0; k < i; ++k) { d[k] /= scale; h += d[k] * d[k]; }
            double f = d[i - 1];
            double g = f > 0 ? -std::sqrt(h) : std::sqrt(h);
            e[i] = scale * g;
            h -= f * g;
            d[i - 1] = f - g;
            for (int j = 0; j < i; ++j) e[j] = 0.0;
            for (int j = 0; j < i; ++j) {
                f = d[j];
                A(j, i) = f;
                g = e[j] + A(j, j) * f;
                for (int k = j + 1; k <= i - 1; ++k) { g += A(k, j) * d[k]; e[k] += A(k, j) * f; }
                e[j] = g;
            }
            f = 0.0;
            for (int j = 0; j < i; ++j) { e[j] /= h; f += e[j] * d[j]; }
            double hh = f / (h + h);
            for (int j = 0; j < i; ++j) e[j] -= hh * d[j];
            for (int j = 0; j < i; ++j) {
                f = d[j]; g = e[j];
                for (int k = j; k <= i - 1; ++k) A(k, j) -= (f * e[k] + g * d[k]);
                d[j] = A(i - 1, j);
                A(i, j) = 0.0;
            }
        }
        d[i] = h;
    }
    for (int i = 0; i < n - 1; ++i) {
        A(n - 1, i) = A(i, i);
        A(i, i) = 1.0;
        double h = d[i + 1];
        if (h != 0.0) {
            for (int k = 0; k <= i; ++k) d[k] = A(k, i + 1) / h;
            for (int j = 0; j <= i; ++j) {
                double g = 0.0;
                for (int k = 0; k <= i; ++k) g += A(k, i + 1) * A(k, j);
                for (int k = 0; k <= i; ++k) A(k, j) -= g * d[k];
            }
        }
        for (int k = 0; k <= i; ++k) A(k, i + 1) = 0.0;
    }
    for (int j = 0; j < n; ++j) { d[j] = A(n - 1, j); A(n - 1, j) = 0.0; }
    A(n - 1, n - 1) = 1.0;
    e[0] = 0.0;
    // implicit QL on the tridiagonal (d, e), rotations accumulated into A
    for (int i = 1; i < n; ++i) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    double f = 0.0, tst1 = 0.0;
    const double eps = std::ldexp(1.0, -52);
    for (int l = 0; l < n; ++l) {
        tst1 = std::max(tst1, std::fabs(d[l]) + std::fabs(e[l]));
        int m = l;
        while (m < n && std::fabs(e[m]) > eps * tst1) ++m;
        if (m == n) m = n - 1;
        if (m > l) {
            int guard = 0;
            do {
                if (++guard > 200) throw std::runtime_error("MG94 eigendecomposition failed");
                double g = d[l];
                double p = (d[l + 1] - g) / (2.0 * e[l]);
                double r = std::hypot(p, 1.0);
                if (p < 0) r = -r;
                d[l] = e[l] / (p + r);
                d[l + 1] = e[l] * (p + r);
                double dl1 = d[l + 1];
                double h = g - d[l];
                for (int i = l + 2; i < n; ++i) d[i] -= h;
                f += h;
                p = d[m];
                double c = 1.0, c2 = 1.0, c3 = 1.0, el1 = e[l + 1], s = 0.0, s2 = 0.0;
                for (int i = m - 1; i >= l; --i) {
                    c3 = c2; c2 = c; s2 = s;
                    g = c * e[i];
                    h = c * p;
                    r = std::hypot(p, e[i]);
                    e[i + 1] = s * r;
                    s = e[i] / r;
                    c = p / r;
                    p = c * d[i] - s * g;
                    d[i + 1] = h + s * (c * g + s * d[i]);
                    for (int k = 0; k < n; ++k) {
                        h = A(k, i + 1);
                        A(k, i + 1) = s * A(k, i) + c * h;
                        A(k, i) = c * A(k, i) - s * h;
                    }
                }
                p = -s * s2 * c3 * el1 * e[l] / dl1;
                e[l] = s * p;
                d[l] = c * p;
            } while (std::fabs(e[l]) > eps * tst1);
        }
        d[l] += f;
        e[l] = 0.0;
    }
    Z = std::move(a);
}

class MG94Matrix {
public:
    int S = 0;
    Matrix Q;
    Vector pi, sqrt_pi, inv_sqrt_pi, eigenvalues;
    Matrix U_pi, V_pi;
    Scalar scale_factor = 1.0;

    // rate_matrix.hpp:165-249: single-nucleotide changes weighted by
    // (alpha | beta) * theta * target positional frequency; double/triple hits
    // only with delta/psi > 0; the mean rate is stored but not applied.
    // with_eigen = false builds the generator only (the device diagonalises it):
    // eigenvalues, U_pi and V_pi stay empty.
    void update(const MG94Parameters& p, const double pos[3][4], const Vector& codon_freqs,
                const GeneticCode& code = *GeneticCode::universal(), bool with_eigen = true) {
        S = code.num_sense_codons;
        pi = codon_freqs;
        double r[4][4];
        exchangeabilities(p, r);
        Q = Matrix(S, S);
        for (int i = 0; i < S; ++i) {
            double row = 0.0;
            for (int j = 0; j < S; ++j) {
                if (i == j) continue;
                const auto& d = code.diff_matrix[i][j];
                double w = d.synonymous ? p.alpha : p.beta, q = 0.0;
                if (d.num_diffs == 1) q = w;
                else if (d.num_diffs == 2 && p.delta > 0) q = w * p.delta;
                else if (d.num_diffs == 3 && p.psi > 0) q = w * p.psi;
                if (q == 0.0) continue;
                for (int k = 0; k < d.num_diffs; ++k) q *= r[d.diff_from[k]][d.diff_to[k]] * pos[d.diff_pos[k]][d.diff_to[k]];
                Q(i, j) = q;
                row += q;
            }
            Q(i, i) = -row;
        }
        scale_factor = 0.0;
        for (int i = 0; i < S; ++i) scale_factor -= pi[size_t(i)] * Q(i, i);
        if (!with_eigen) {
            eigenvalues.clear(); U_pi = Matrix(); V_pi = Matrix();
            return;
        }
        sqrt_pi.resize(S); inv_sqrt_pi.resize(S);
        for (int i = 0; i < S; ++i) { sqrt_pi[i] = std::sqrt(std::max(pi[i], 1e-12)); inv_sqrt_pi[i] = 1.0 / sqrt_pi[i]; }
        std::vector<double> sym(size_t(S) * S);
        for (int i = 0; i < S; ++i)
            for (int j = 0; j < S; ++j) sym[size_t(i) * S + j] = sqrt_pi[i] * Q(i, j) * inv_sqrt_pi[j];
        for (int i = 0; i < S; ++i)
            for (int j = i + 1; j < S; ++j) {
                double m = 0.5 * (sym[size_t(i) * S + j] + sym[size_t(j) * S + i]);
                sym[size_t(i) * S + j] = sym[size_t(j) * S + i] = m;
            }
        std::vector<double> Z;
        symmetric_eigen(S, std::move(sym), eigenvalues, Z);
        for (auto& l : eigenvalues) l = std::min(l, 0.0);
        U_pi = Matrix(S, S); V_pi = Matrix(S, S);
        for (int i = 0; i < S; ++i)
            for (int k = 0; k < S; ++k) {
                U_pi(i, k) = inv_sqrt_pi[i] * Z[size_t(i) * S + k];
                V_pi(k, i) = Z[size_t(i) * S + k] * sqrt_pi[i];
            }
    }

    Matrix transition_matrix(Scalar t) const {
        Matrix P(S, S);
        std::vector<double> ex(S);
        for (int k = 0; k < S; ++k) ex[k] = std::exp(eigenvalues[k] * t);
        for (int i = 0; i < S; ++i)
            for (int k = 0; k < S; ++k) {
                double u = U_pi(i, k) * ex[k];
                if (u == 0.0) continue;
                for (int j = 0; j < S; ++j) P(i, j) += u * V_pi(k, j);
            }
        for (auto& x : P.v) x = std::max(x, 0.0);
        return P;
    }
};

// ------------------------------------------------------------------- GTR
// rate_matrix.hpp:14-21
struct GTRParameters {
    Scalar theta_AC = 1.0, theta_AT = 1.0, theta_CG = 1.0, theta_CT = 1.0, theta_GT = 1.0;   // theta_AG = 1
};

// rate_matrix.hpp:23-104: nucleotide GTR normalised to mean rate 1 (scale_factor), symmetric
// eigensystem of diag(sqrt pi) Q diag(1 / sqrt pi) with pi floored at 1e-12, eigenvalues clamped
// <= 0, P(t) = U_pi diag(e^{lambda t}) V_pi clamped at 0.
class GTRMatrix {
public:
    Matrix Q{4, 4};
    Vector pi = Vector(4, 0.0), sqrt_pi = Vector(4, 0.0), inv_sqrt_pi = Vector(4, 0.0), eigenvalues = Vector(4, 0.0);
    Matrix U_pi{4, 4}, V_pi{4, 4};
    Scalar scale_factor = 1.0;

    void update(const GTRParameters& p, const double freq[4]) {
        const double r[4][4] = {{0.0, p.theta_AC, 1.0, p.theta_AT},
                                {p.theta_AC, 0.0, p.theta_CG, p.theta_CT},
                                {1.0, p.theta_CG, 0.0, p.theta_GT},
                                {p.theta_AT, p.theta_CT, p.theta_GT, 0.0}};
        for (int i = 0; i < 4; ++i) {
            pi[i] = freq[i];
            sqrt_pi[i] = std::sqrt(std::max(pi[i], 1e-12));
            inv_sqrt_pi[i] = 1.0 / sqrt_pi[i];
        }
        Q = Matrix(4, 4);
        for (int i = 0; i < 4; ++i) {
            double row = 0.0;
            for (int j = 0; j < 4; ++j)
                if (i != j) { Q(i, j) = r[i][j] * pi[j]; row += Q(i, j); }
            Q(i, i) = -row;
        }
        double avg = 0.0;
        for (int i = 0; i < 4; ++i) avg -= pi[i] * Q(i, i);
        scale_factor = 1.0;
        if (avg > 0.0) {
            scale_factor = avg;
            for (auto& x : Q.v) x /= avg;
        }
        std::vector<double> sym(16);
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) sym[size_t(i) * 4 + j] = sqrt_pi[i] * Q(i, j) * inv_sqrt_pi[j];
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j) {
                const double m = 0.5 * (sym[size_t(i) * 4 + j] + sym[size_t(j) * 4 + i]);
                sym[size_t(i) * 4 + j] = sym[size_t(j) * 4 + i] = m;
            }
        std::vector<double> Z;
        symmetric_eigen(4, std::move(sym), eigenvalues, Z);
        for (auto& l : eigenvalues) l = std::min(l, 0.0);
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 4; ++k) {
                U_pi(i, k) = inv_sqrt_pi[i] * Z[size_t(i) * 4 + k];
                V_pi(k, i) = Z[size_t(i) * 4 + k] * sqrt_pi[i];
            }
    }
    void update(const GTRParameters& p, const Vector& freq) { update(p, freq.data()); }

    Matrix transition_matrix(Scalar t) const {
        Matrix P(4, 4);
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                double x = 0.0;
                for (int k = 0; k < 4; ++k) x += U_pi(i, k) * std::exp(eigenvalues[k] * t) * V_pi(k, j);
                P(i, j) = std::max(x, 0.0);
            }
        return P;
    }
};

} // namespace hyphy::core
