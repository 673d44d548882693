// h3g_fel.h — FEL per-site fits: the batched device evaluator (h3g_fel.cu) and
// the host driver that runs one optimiser per pattern (h3g_fel_driver.cpp).
// Plain C++ (no device code), so the driver builds with the host compiler.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/h3g.h"

namespace h3g {

// Host view of an uploaded problem (h3g_capi.cu).
struct FelProblemView {
    int n = 0, root = -1, T = 0, P = 0;
    const int* parent = nullptr;      // [n]
    const uint8_t* leaf = nullptr;    // [n]
    const int* taxon = nullptr;       // [n] alignment row of each leaf, -1 otherwise
    const int* ch_off = nullptr;      // [n + 1] children CSR
    const int* ch = nullptr;
    const int8_t* states = nullptr;   // [P][T] as uploaded
    int device = 0;
};
bool fel_problem_view(h3g_problem* pr, FelProblemView* v);
void fel_set_error(h3g_problem* pr, const std::string& msg);

// Device evaluator.  Eigensystem slots hold (lambda, U, V) of
// Q(omega) = Qs + omega Qn.  A request evaluates one pattern's log-likelihood
// at time scale a with the eigensystem in its slot, or, when slot2 >= 0, with
// the two eigensystems mixed at the transition-matrix level with weights
// (w1, 1 - w1).  When slot_bg >= 0 the branches flagged in the run's
// background[] use that eigensystem alone.  req_slot2 / req_w1 / req_slot_bg
// may be null (no request has that component).
struct FelDevice;
// background[n_nodes] (may be null: none) flags the branches a request's
// background eigensystem applies to; the root's flag is ignored
FelDevice* fel_device_create(h3g_problem* pr, int S, const double* pi, const double* Qs, const double* Qn,
                             const double* branch_lengths, const uint8_t* background, int max_requests, int n_slots,
                             std::string* err);
// eig_prev[i] >= 0: slot whose eigenvectors start the solve (warm start), -1: from the identity
bool fel_device_eval(FelDevice* d, int n_eig, const double* eig_omega, const int* eig_slot, const int* eig_prev, int n_req,
                     const int* req_pattern, const double* req_a, const int* req_slot, const int* req_slot2,
                     const double* req_w1, const int* req_slot_bg, double* lnl_out, std::string* err);
// MEME's empirical Bayes factors of every branch for two-component requests
// (at most fel_device_max_ebf(d) per call): ebf_out[r * n_nodes + b].  With
// req_slot_bg (every entry >= 0) the background branches use that eigensystem
// and get factor 1.
int fel_device_max_ebf(const FelDevice* d);
bool fel_device_ebf(FelDevice* d, int n_eig, const double* eig_omega, const int* eig_slot, const int* eig_prev, int n_req,
                    const int* req_pattern, const double* req_a, const int* req_slot, const int* req_slot2,
                    const double* req_w1, const int* req_slot_bg, double* ebf_out, std::string* err);
void fel_device_transfer(const FelDevice* d, size_t* h2d, size_t* d2h, int* launches);   // bytes moved, kernels launched
// ends a run: the evaluator stays with its problem (problem_fel_device) and a
// later fel_device_create with the same problem and no larger sizes reuses its
// device buffers instead of allocating them again
void fel_device_destroy(FelDevice* d);
void fel_device_free(FelDevice* d);                 // release (problem destruction)
FelDevice*& problem_fel_device(h3g_problem* pr);    // h3g_capi.cu
// record a whole run's transfers, kernel launches and host wall time where
// h3g_last_eval_transfer / h3g_last_eval_stats report them (h3g_capi.cu)
void fel_record_transfer(h3g_problem* pr, size_t h2d, size_t d2h, int launches, double ms);

}  // namespace h3g
