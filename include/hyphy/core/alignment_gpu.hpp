// alignment_gpu.hpp — Alignment::finalize (include/hyphy/core/alignment.hpp:665-722)
// with the codon translation, the nucleotide counts and the site-pattern compression
// (alignment.hpp:893-911, :1021-1078) on the device through h3g_alignment_compress.
//
// finalize_on_device(aln) fills the same fields as aln.finalize(): num_taxa,
// num_codons, num_nucleotides, patterns (states, ambiguous_masks, weight, sites in
// column order), site_to_pattern, and the frequencies, computed on the host from the
// device's counts (the 3 x 4 CF3x4 fixed point is not worth a launch).
#pragma once

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "likelihood_gpu.hpp"

namespace hyphy::core {

inline void finalize_on_device(Alignment& a, std::shared_ptr<const GeneticCode> gc = nullptr) {
    a.code = gc ? gc : (a.code ? a.code : GeneticCode::universal());
    if (a.sequences.empty()) throw std::runtime_error("Empty alignment");
    a.num_taxa = a.sequences.size();
    a.num_nucleotides = a.sequences[0].raw_seq.size();
    a.taxon_names.clear();
    for (auto& s : a.sequences) {
        if (s.raw_seq.size() != a.num_nucleotides) throw std::runtime_error("Sequences have unequal lengths in alignment");
        a.taxon_names.push_back(s.name);
    }
    if (a.num_nucleotides % 3) throw std::runtime_error("Nucleotide alignment length is not a multiple of 3 (in-frame codons required)");
    a.num_codons = a.num_nucleotides / 3;
    const size_t T = a.num_taxa, L = a.num_nucleotides, C = a.num_codons;
    std::vector<char> rows(T * L);
    for (size_t t = 0; t < T; ++t) std::memcpy(rows.data() + t * L, a.sequences[t].raw_seq.data(), L);
    const h3g_genetic_code code{a.code->num_sense_codons, a.code->codon64_to_sense};
    std::vector<int32_t> s2p(C), weight(C);
    std::vector<int8_t> states(C * T);
    std::vector<uint64_t> masks(C * T);
    h3g_compress_info info{};
    auto& eng = gpu_detail::Engine::get();
    eng.check(h3g_alignment_compress(eng.ctx(), int(T), int64_t(L), rows.data(), L, &code, s2p.data(), weight.data(), nullptr,
                                     states.data(), masks.data(), &info));
    const size_t P = size_t(info.n_patterns);
    a.patterns.assign(P, SitePattern{});
    for (size_t p = 0; p < P; ++p) {
        a.patterns[p].states.assign(states.begin() + std::ptrdiff_t(p * T), states.begin() + std::ptrdiff_t((p + 1) * T));
        a.patterns[p].ambiguous_masks.assign(masks.begin() + std::ptrdiff_t(p * T), masks.begin() + std::ptrdiff_t((p + 1) * T));
        a.patterns[p].weight = weight[p];
        a.patterns[p].sites.reserve(size_t(weight[p]));
    }
    a.site_to_pattern.assign(C, 0);
    for (size_t c = 0; c < C; ++c) {
        a.site_to_pattern[c] = size_t(s2p[c]);
        a.patterns[size_t(s2p[c])].sites.push_back(c);
    }
    double pc[3][4];
    for (int p = 0; p < 3; ++p)
        for (int b = 0; b < 4; ++b) pc[p][b] = double(info.pos_counts[4 * p + b]);
    a.frequencies_from_counts(pc);
}

}  // namespace hyphy::core
