// h3g_sitefit.cpp — the lockstep loop shared by the FEL and MEME drivers.
#include "h3g_sitefit.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>

namespace h3g::sitefit {

uint64_t bits_of(double x) {
    uint64_t u;
    std::memcpy(&u, &x, sizeof u);
    return u;
}

h3g_status run_lockstep(FelDevice* dev, std::vector<Site>& sites, std::vector<Fit>& fits, const LockstepOptions& opt,
                        LockstepState& state, std::string* err) {
    const int N = int(sites.size());
    const int C = opt.components;
    if (C < 2 || C > 3) { *err = "components must be 2 or 3"; return H3G_ERR_STATE; }
    const int temp_base = slots_needed(N, 0, C);
    for (int i = 0; i < N; ++i) {
        sites[i].resume = fits[i].h;
        sites[i].pending = nullptr;
    }
    // start every fit: it runs to its first evaluation
    for (int i = 0; i < N; ++i) {
        std::coroutine_handle<> h = sites[i].resume;
        sites[i].resume = {};
        h.resume();
        if (fits[i].h.promise().error) { *err = "optimiser failed"; return H3G_ERR_NUMERIC; }
    }
    auto& shared = state.shared;                        // omega bits -> shared slot (whole run)
    std::unordered_map<uint64_t, int> users;           // omega bits -> sites requesting it this batch
    std::unordered_map<uint64_t, int> temp;            // omega bits -> pool slot (this batch)
    std::vector<uint64_t> keys;
    std::vector<int> admitted, req_pat, req_slot, req_slot2, req_slot3, eig_slot, eig_prev;
    std::vector<double> req_a, req_w1, eig_om, lnl;
    std::vector<Req*> req_ptr;
    const size_t n_slots = size_t(slots_needed(N, opt.temp_slots, C));
    if (state.written.size() < n_slots) {
        state.written.resize(n_slots, -1);
        state.solved.resize(n_slots, 0);
    }
    auto& written = state.written;
    auto& solved = state.solved;
    int& batch = state.batch;
    for (;;) {
        users.clear();
        bool any = false;
        for (int i = 0; i < N; ++i) {
            Site& s = sites[i];
            if (!s.pending) continue;
            any = true;
            keys.clear();
            for (const Req& r : *s.pending)
                for (int c = 0; c < 3; ++c) {
                    if (!req_has(r, c)) continue;
                    if (c >= C) { *err = "a request has more components than the run"; return H3G_ERR_STATE; }
                    const double om = req_omega(r, c);
                    if (s.slot[c] >= 0 && std::fabs(om - s.cached[c]) <= opt.cache_tol) continue;
                    keys.push_back(bits_of(om));
                }
            std::sort(keys.begin(), keys.end());
            keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
            for (uint64_t k : keys) ++users[k];
        }
        if (!any) break;
        temp.clear();
        admitted.clear(); req_pat.clear(); req_slot.clear(); req_slot2.clear(); req_slot3.clear(); req_a.clear(); req_w1.clear();
        eig_om.clear(); eig_slot.clear(); eig_prev.clear(); req_ptr.clear();
        int temp_used = 0;
        bool mixed = false, background = false;
        auto solve = [&](double om, int slot, int prev) {
            eig_om.push_back(om);
            eig_slot.push_back(slot);
            eig_prev.push_back(prev);
        };
        for (int i = 0; i < N; ++i) {
            Site& s = sites[i];
            if (!s.pending) continue;
            const int k = int(s.pending->size());
            if (int(req_pat.size()) + k > opt.max_requests) continue;       // next batch
            const bool single = k == 1;
            int need = 0;                                                    // eigensystems of the site's requests
            for (const Req& r : *s.pending)
                for (int c = 0; c < C; ++c) need += req_has(r, c) ? 1 : 0;
            if (!single && temp_used + need > opt.temp_slots) continue;     // next batch
            admitted.push_back(i);
            int flip_slot[3] = {-1, -1, -1};
            double flip_om[3] = {0.0, 0.0, 0.0};
            bool first = true;
            for (Req& r : *s.pending) {
                int sl[3] = {-1, -1, -1};
                for (int c = 0; c < C; ++c) {
                    if (!req_has(r, c)) continue;
                    const double om = req_omega(r, c);
                    if (s.slot[c] >= 0 && std::fabs(om - s.cached[c]) <= opt.cache_tol) { sl[c] = s.slot[c]; continue; }
                    const uint64_t key = bits_of(om);
                    int slot = -1;
                    if (auto it = shared.find(key); it != shared.end()) {
                        slot = it->second;
                    } else if (users[key] >= 2 && int(shared.size()) < kSharedSlots) {
                        slot = int(shared.size());
                        shared.emplace(key, slot);
                        solve(om, slot, -1);                // shared slots start from the identity
                    } else if (!single) {
                        if (auto t = temp.find(key); t != temp.end()) {
                            slot = t->second;
                        } else {
                            if (first) {                    // into the site's other buffer, current afterwards
                                slot = own_slot(i, 1 - s.buf[c], c, C);
                                flip_slot[c] = slot;
                                flip_om[c] = om;
                            } else {
                                slot = temp_base + temp_used++;
                            }
                            temp.emplace(key, slot);
                            solve(om, slot, s.slot[c]);     // warm start from the site's current eigensystem
                        }
                    } else {
                        slot = own_slot(i, s.buf[c], c, C);
                        solve(om, slot, s.slot[c]);         // in place when the current one is the site's own
                    }
                    if (single) { s.slot[c] = slot; s.cached[c] = om; }
                    sl[c] = slot;
                }
                first = false;
                req_pat.push_back(s.pattern);
                req_a.push_back(r.a);
                req_w1.push_back(sl[1] >= 0 ? r.w1 : 1.0);
                req_slot.push_back(sl[0]);
                req_slot2.push_back(sl[1]);
                req_slot3.push_back(sl[2]);
                req_ptr.push_back(&r);
                mixed = mixed || sl[1] >= 0;
                background = background || sl[2] >= 0;
            }
            for (int c = 0; c < C; ++c)
                if (flip_slot[c] >= 0) {
                    s.buf[c] ^= 1;
                    s.slot[c] = flip_slot[c];
                    s.cached[c] = flip_om[c];
                }
        }
        if (admitted.empty()) { *err = "a pattern's requests exceed one device batch"; return H3G_ERR_STATE; }
        // one launch solves every slot at most once, reads no slot it writes (an in-place warm
        // start excepted), and every request reads slots solved in this or an earlier batch
        for (size_t e = 0; e < eig_slot.size(); ++e) {
            if (written[size_t(eig_slot[e])] == batch) { *err = "an eigensystem slot is solved twice in one batch"; return H3G_ERR_STATE; }
            written[size_t(eig_slot[e])] = batch;
        }
        for (size_t e = 0; e < eig_prev.size(); ++e) {
            const int pv = eig_prev[e];
            if (pv < 0) continue;
            if ((written[size_t(pv)] == batch && pv != eig_slot[e]) || !solved[size_t(pv)]) {
                *err = "a warm start reads a slot solved in the same batch";
                return H3G_ERR_STATE;
            }
        }
        for (size_t e = 0; e < eig_slot.size(); ++e) solved[size_t(eig_slot[e])] = 1;
        for (size_t r = 0; r < req_slot.size(); ++r)
            if (!solved[size_t(req_slot[r])] || (req_slot2[r] >= 0 && !solved[size_t(req_slot2[r])]) ||
                (req_slot3[r] >= 0 && !solved[size_t(req_slot3[r])])) {
                *err = "a request reads an eigensystem that was never solved";
                return H3G_ERR_STATE;
            }
        ++batch;
        lnl.assign(req_pat.size(), 0.0);
        if (!fel_device_eval(dev, int(eig_om.size()), eig_om.data(), eig_slot.data(), eig_prev.data(), int(req_pat.size()),
                             req_pat.data(), req_a.data(), req_slot.data(), mixed ? req_slot2.data() : nullptr,
                             mixed ? req_w1.data() : nullptr, background ? req_slot3.data() : nullptr, lnl.data(), err))
            return H3G_ERR_CUDA;
        for (size_t r = 0; r < req_ptr.size(); ++r) req_ptr[r]->lnl = lnl[r];
        const bool small = int(req_pat.size()) <= opt.spec_threshold;
        for (int i : admitted) {
            Site& s = sites[i];
            s.pending = nullptr;
            s.speculate = small;
            std::coroutine_handle<> h = s.resume;
            s.resume = {};
            h.resume();
            if (fits[i].h.promise().error) {
                try {
                    std::rethrow_exception(fits[i].h.promise().error);
                } catch (const std::exception& e) {
                    *err = std::string("optimiser failed: ") + e.what();
                } catch (...) {
                    *err = "optimiser failed";
                }
                return H3G_ERR_NUMERIC;
            }
        }
    }
    for (int i = 0; i < N; ++i)
        if (!fits[i].h.done()) { *err = "a pattern did not finish"; return H3G_ERR_STATE; }
    return H3G_OK;
}

}  // namespace h3g::sitefit
