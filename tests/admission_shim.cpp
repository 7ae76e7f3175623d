// C entry points over zeknox_b200/csrc/admission.h for tests/test_admission.py
// (built with g++ by the test; host code only).
#include <string.h>

#include "admission.h"

static std::vector<zk::AdmitJob> jobs_of(const double *est, const double *budget, const uint64_t *bytes, size_t n) {
    std::vector<zk::AdmitJob> q(n);
    for (size_t i = 0; i < n; i++) q[i] = zk::AdmitJob{est[i], budget[i], bytes[i]};
    return q;
}

extern "C" long shim_pick(const double *est, const double *budget, const uint64_t *bytes, size_t n,
                          const double *running, size_t nr, uint64_t in_use, uint64_t budget_bytes) {
    return zk::admission_pick(jobs_of(est, budget, bytes, n), std::vector<double>(running, running + nr), in_use,
                              budget_bytes);
}

// Charges job `pick`; writes the queue's and the running jobs' budgets back.
extern "C" void shim_charge(const double *est, double *budget, const uint64_t *bytes, size_t n, double *running,
                            size_t nr, long pick) {
    std::vector<zk::AdmitJob> q = jobs_of(est, budget, bytes, n);
    std::vector<double> r(running, running + nr);
    zk::admission_charge(q, r, pick);
    for (size_t i = 0; i < n; i++) budget[i] = q[i].budget_s;
    if (nr) memcpy(running, r.data(), nr * sizeof(double));
}
