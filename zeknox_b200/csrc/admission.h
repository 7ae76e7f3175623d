// The served commits' admission rule, as plain host code (no CUDA), so that
// the dispatcher in serve.cu and a CPU test use the same function.
//
// Every job carries an estimate of its GPU time alone (est_s) and a delay
// budget (budget_s, a fraction of its own estimate, reduced as later jobs are
// charged to it).  Jobs are queued in submission order.  A candidate at queue
// position q would delay the running jobs and the queued jobs before it; it
// may start if its est_s fits in the remaining budget of every one of them
// (so the oldest job, with nothing running, always may), and if its bytes fit
// the HBM budget next to the memory that the oldest queued job is waiting for.
// Among the candidates that may start, the shortest goes first (the earliest
// of equal ones).  Starting a job charges its est_s to every job it delays.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <vector>

namespace zk {

struct AdmitJob {
    double est_s = 0;     // estimated GPU time alone
    double budget_s = 0;  // delay it may still take from later jobs
    uint64_t bytes = 0;   // device bytes it needs to start (resident tree + running buffers)
};

// Index in `queue` of the job to start now, or -1 if none may start until a
// job completes or memory is released.
inline long admission_pick(const std::vector<AdmitJob> &queue, const std::vector<double> &running_budgets,
                           uint64_t in_use, uint64_t budget_bytes) {
    if (queue.empty()) return -1;
    // memory held back for the oldest job while it waits for it
    const uint64_t head = queue.front().bytes;
    const uint64_t reserve = in_use + head > budget_bytes ? head : 0;
    double room = 1e300;  // smallest budget among the jobs a candidate would delay
    for (double b : running_budgets) room = b < room ? b : room;
    long pick = -1;
    double best = 1e300;
    for (size_t q = 0; q < queue.size(); q++) {
        const AdmitJob &J = queue[q];
        const uint64_t need = J.bytes + (q == 0 ? 0 : reserve);
        if (J.est_s <= room && in_use + need <= budget_bytes && J.est_s < best) {
            best = J.est_s;
            pick = (long)q;
        }
        room = J.budget_s < room ? J.budget_s : room;
    }
    return pick;
}

// Charge a started job (queue position `pick`) to the jobs it delays: every
// running job and every queued job before it.
inline void admission_charge(std::vector<AdmitJob> &queue, std::vector<double> &running_budgets, long pick) {
    const double est = queue[(size_t)pick].est_s;
    for (double &b : running_budgets) b -= est;
    for (long q = 0; q < pick; q++) queue[(size_t)q].budget_s -= est;
}

}  // namespace zk
