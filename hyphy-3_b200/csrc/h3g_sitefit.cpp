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
                        std::string* err) {
    const int N = int(sites.size());
    const int own_base = kSharedSlots, temp_base = kSharedSlots + 2 * N;
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
    std::unordered_map<uint64_t, int> shared;          // omega bits -> shared slot (whole run)
    std::unordered_map<uint64_t, int> users;           // omega bits -> sites requesting it this batch
    std::unordered_map<uint64_t, int> temp;            // omega bits -> pool slot (this batch)
    std::vector<uint64_t> keys;
    std::vector<int> admitted, req_pat, req_slot, req_slot2, eig_slot, eig_prev;
    std::vector<double> req_a, req_w1, eig_om, lnl;
    std::vector<Req*> req_ptr;
    for (;;) {
        users.clear();
        bool any = false;
        for (int i = 0; i < N; ++i) {
            Site& s = sites[i];
            if (!s.pending) continue;
            any = true;
            keys.clear();
            for (const Req& r : *s.pending)
                for (int c = 0; c < (r.om2 >= 0.0 ? 2 : 1); ++c) {
                    const double om = c ? r.om2 : r.om1;
                    if (s.slot[c] >= 0 && std::fabs(om - s.cached[c]) <= opt.cache_tol) continue;
                    keys.push_back(bits_of(om));
                }
            std::sort(keys.begin(), keys.end());
            keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
            for (uint64_t k : keys) ++users[k];
        }
        if (!any) break;
        temp.clear();
        admitted.clear(); req_pat.clear(); req_slot.clear(); req_slot2.clear(); req_a.clear(); req_w1.clear();
        eig_om.clear(); eig_slot.clear(); eig_prev.clear(); req_ptr.clear();
        int temp_used = 0;
        bool mixed = false;
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
            if (!single && temp_used + 2 * k > opt.temp_slots) continue;    // next batch
            admitted.push_back(i);
            for (Req& r : *s.pending) {
                const int nc = r.om2 >= 0.0 ? 2 : 1;
                int sl[2] = {-1, -1};
                for (int c = 0; c < nc; ++c) {
                    const double om = c ? r.om2 : r.om1;
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
                            slot = temp_base + temp_used++;
                            temp.emplace(key, slot);
                            solve(om, slot, s.slot[c]);     // warm start from the site's last eigensystem
                        }
                    } else {
                        slot = own_base + 2 * i + c;
                        solve(om, slot, s.slot[c]);         // in place when the site's last one was its own
                    }
                    if (single) { s.slot[c] = slot; s.cached[c] = om; }
                    sl[c] = slot;
                }
                req_pat.push_back(s.pattern);
                req_a.push_back(r.a);
                req_w1.push_back(nc == 2 ? r.w1 : 1.0);
                req_slot.push_back(sl[0]);
                req_slot2.push_back(sl[1]);
                req_ptr.push_back(&r);
                mixed = mixed || nc == 2;
            }
        }
        if (admitted.empty()) { *err = "a pattern's requests exceed one device batch"; return H3G_ERR_STATE; }
        lnl.assign(req_pat.size(), 0.0);
        if (!fel_device_eval(dev, int(eig_om.size()), eig_om.data(), eig_slot.data(), eig_prev.data(), int(req_pat.size()),
                             req_pat.data(), req_a.data(), req_slot.data(), mixed ? req_slot2.data() : nullptr,
                             mixed ? req_w1.data() : nullptr, lnl.data(), err))
            return H3G_ERR_CUDA;
        for (size_t r = 0; r < req_ptr.size(); ++r) req_ptr[r]->lnl = lnl[r];
        for (int i : admitted) {
            Site& s = sites[i];
            s.pending = nullptr;
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
