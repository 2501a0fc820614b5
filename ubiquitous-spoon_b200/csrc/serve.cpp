// Serving loop over the instance and batch API (include/chanfast_cuda.h):
// channel-flow solves of different grids, Reynolds numbers and step counts
// arrive over time; each is admitted when the device-memory budget and the
// slot limit allow, stays resident on the device, is advanced together with
// every other resident solve by one batched launch per substep stage, and is
// retired on its own as soon as it has run its steps.  Requests that arrive
// while others run join the next round: continuous batching.  While the set
// of solves advancing by a full quantum stays the same from round to round,
// its recorded batch (per-instance records uploaded once, two steps replayed
// as one CUDA graph) is replayed; it is formed again, without launch-shape
// trials, only when that set changes.
#include <algorithm>
#include <chrono>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "chanfast_cuda.h"

namespace {

struct Active {
    int index;           // request index
    cf_instance* inst;
    int remaining;       // RK3 steps left
};

double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" int cf_serve(const cf_request* reqs, int n, double hbm_budget_bytes, int max_active, int quantum,
                        void* stream, cf_done_fn on_done, void* user, cf_result* results)
{
    if (!reqs || n < 0 || !results || max_active <= 0 || quantum <= 0 || !(hbm_budget_bytes > 0.0))
        return CF_EINVAL;
    for (int q = 0; q < n; q++) {
        results[q].admit_s = results[q].finish_s = -1.0;
        results[q].status = CF_OK;
        results[q].steps_done = 0;
        if (q > 0 && reqs[q].arrival_s < reqs[q - 1].arrival_s) return CF_EINVAL;   // arrival order
        if (reqs[q].nsteps < 0 || reqs[q].cfg.scheme != CF_SCHEME_CHANFAST) return CF_EINVAL;
    }
    cudaStream_t st = (cudaStream_t) stream;
    bool own = false;
    if (!st) {
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return CF_ECUDA;
        own = true;
    }
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<Active> active;
    cf_batch* batch = nullptr;              // recorded batch of the full-quantum set
    std::vector<cf_instance*> batch_set;
    auto drop_batch = [&]() {
        if (batch) cf_batch_destroy(batch);
        batch = nullptr;
        batch_set.clear();
    };
    std::vector<double> bytes(n, 0.0);
    double used = 0.0;
    int next = 0, done = 0, rc = CF_OK;

    auto retire = [&](size_t a, int status) {
        Active& A = active[a];
        if (std::find(batch_set.begin(), batch_set.end(), A.inst) != batch_set.end()) drop_batch();
        cf_result& R = results[A.index];
        R.status = status;
        R.finish_s = seconds_since(t0);
        if (on_done) on_done(A.index, A.inst, user);
        cf_destroy(A.inst);
        used -= bytes[A.index];
        active.erase(active.begin() + a);
        done++;
    };

    while (done < n && rc == CF_OK) {
        // admit every request that has arrived, in order, while memory and slots allow
        const double now = seconds_since(t0);
        while (next < n && reqs[next].arrival_s <= now && (int) active.size() < max_active) {
            const cf_request& Q = reqs[next];
            const double need = (double) cf_instance_bytes(&Q.cfg);
            if (need > hbm_budget_bytes) {   // can never fit: fail it now
                results[next].status = CF_ENOMEM;
                results[next].admit_s = results[next].finish_s = seconds_since(t0);
                if (on_done) on_done(next, nullptr, user);
                next++;
                done++;
                continue;
            }
            if (used + need > hbm_budget_bytes) break;   // wait for a retirement
            cf_instance* inst = nullptr;
            int s = cf_create(&Q.cfg, st, &inst);
            if (s == CF_OK) s = cf_init_fields(inst, Q.seed, Q.amp, Q.c_amp);
            results[next].admit_s = seconds_since(t0);
            bytes[next] = need;
            if (s != CF_OK) {
                if (inst) cf_destroy(inst);
                results[next].status = s;
                results[next].finish_s = results[next].admit_s;
                if (on_done) on_done(next, nullptr, user);
                done++;
            } else {
                used += need;
                active.push_back(Active{next, inst, Q.nsteps});
            }
            next++;
        }
        // retire solves with nothing left to run (zero-step requests)
        for (size_t a = 0; a < active.size();) {
            if (active[a].remaining == 0) retire(a, CF_OK);
            else a++;
        }
        if (active.empty()) {
            if (next < n) {   // idle until the next arrival
                const double wait = reqs[next].arrival_s - seconds_since(t0);
                if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
            }
            continue;
        }
        // one round: every resident solve advances min(quantum, its remaining) steps;
        // at most two batched calls (a full quantum, and the solves finishing sooner)
        const int q_full = quantum;
        int q_short = quantum;
        for (const Active& A : active) q_short = std::min(q_short, A.remaining);
        for (int pass = 0; pass < 2 && rc == CF_OK; pass++) {
            const int steps = pass == 0 ? q_full : q_short;
            if (pass == 1 && q_short == q_full) break;
            std::vector<cf_instance*> group;
            for (const Active& A : active)
                if ((pass == 0 && A.remaining >= q_full) || (pass == 1 && A.remaining < q_full))
                    group.push_back(A.inst);
            if (group.empty()) continue;
            int s;
            if (pass == 0) {   // the full-quantum set: its recorded batch
                if (group != batch_set) {
                    drop_batch();
                    s = cf_batch_create_opts(group.data(), (int) group.size(), st, CF_BATCH_NO_TUNE, &batch);
                    if (s != CF_OK) {
                        rc = s;
                        break;
                    }
                    batch_set = group;
                }
                s = cf_batch_run(batch, steps);
            } else {
                s = cf_batch_step(group.data(), (int) group.size(), 3 * steps, st);
            }
            if (s != CF_OK) {
                rc = s;
                break;
            }
            for (Active& A : active)
                if ((pass == 0 && A.remaining >= q_full) || (pass == 1 && A.remaining < q_full)) {
                    A.remaining -= steps;
                    results[A.index].steps_done += steps;
                }
        }
        if (rc != CF_OK) break;
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            rc = CF_ECUDA;
            break;
        }
        for (size_t a = 0; a < active.size();) {
            // a solve whose state went NaN / Inf retires at once with that status
            const int s = cf_sync(active[a].inst);
            if (s == CF_ENONFINITE) retire(a, CF_ENONFINITE);
            else if (s != CF_OK) {
                rc = s;
                break;
            } else if (active[a].remaining <= 0) retire(a, CF_OK);
            else a++;
        }
    }
    drop_batch();
    for (size_t a = active.size(); a-- > 0;) retire(a, rc == CF_OK ? CF_OK : rc);
    if (own) cudaStreamDestroy(st);
    return rc;
}
