// server.cu -- continuous batching of (r, s-set, d-range) search jobs.
//
// Jobs arrive at any time (submit).  A job is admitted when the device
// memory its r needs fits the budget: the sieve workspace for its degree
// range and, for degrees above 24, a scanner for its r (per-s F, ACC and
// transform buffers for `slots` resident s).  Scanners are shared by every
// job with the same r and are released when idle, so jobs of very different
// r are resident together.  On admission the job is sieved (degrees 2..24 or
// its own maximum); s with a factor there are finished at once, the others
// enter the scanner queue for degrees 25..maxd.  step() advances every
// scanner by a few degrees (each s keeps its state on the device between
// steps and retires at its first factor); poll() returns finished jobs.
// Results are per s in the reference's line format.
#include "gf2e_internal.cuh"

#include <algorithm>
#include <chrono>
#include <cinttypes>
#include <deque>
#include <map>
#include <string>
#include <vector>

namespace {

constexpr int SIEVE_DMAX = 24;

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

std::string hexmask(const uint64_t *w, size_t n) {
    static const char *dig = "0123456789abcdef";
    long long d = -1;
    for (size_t i = n; i-- > 0;)
        if (w[i]) { d = (long long)(i * 64 + 63 - __builtin_clzll(w[i])); break; }
    if (d < 0) return "0";
    std::string s;
    for (long long k = d / 4; k >= 0; k--) s += dig[(w[k >> 4] >> ((k & 15) * 4)) & 0xF];
    return s;
}

struct Job {
    uint64_t id, r, dmax, L0, Lmax;
    std::vector<uint64_t> s;
    std::vector<std::string> lines;       // per s, in submission order
    size_t remaining = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    bool admitted = false;
};

struct RClass {
    gf2e_scanner *sc = nullptr;
    size_t bytes = 0;
    int users = 0;                        // admitted jobs still needing it
};

}  // namespace

namespace gf2e {
cudaStream_t scanner_stream(gf2e_scanner *S);
}  // namespace gf2e

namespace {

}  // namespace

struct gf2e_server {
    size_t budget = 0, used = 0;
    cudaEvent_t ev_caller = nullptr;                 // caller's stream at the start of a step
    std::vector<cudaEvent_t> ev_join;                // each scanner's stream at its end
    int slots = 64;
    int block = 1;                                   // blocked-DDF block size of the scanners
    uint64_t next_tag = 1;
    std::map<uint64_t, Job> jobs;                    // by id
    std::deque<uint64_t> waiting;                    // ids not yet admitted
    std::map<uint64_t, RClass> rclass;               // by r
    std::map<uint64_t, std::pair<uint64_t, size_t>> tag_owner;   // tag -> (job, index)
    std::deque<uint64_t> finished;                   // job ids
    void *sieve_ws = nullptr;
    size_t sieve_ws_bytes = 0;
    uint64_t *best = nullptr;
    size_t best_words = 0;
    uint64_t sd_pairs_sieve = 0;
    uint64_t sd_pairs_scan_retired = 0;              // scanned pairs of destroyed scanners
    std::vector<gf2e_scan_result> res;
    std::vector<uint64_t> tags, masks;
};

namespace {

const size_t MASK_CAP = 2048;

int admit(gf2e_server &S, Job &J, cudaStream_t st) {
    // sieve the job's s values (degrees 2..min(dmax, 24)) on the shared workspace
    const int dsieve = (int)std::min<uint64_t>(J.dmax, SIEVE_DMAX);
    uint64_t smax = 0;
    for (uint64_t s : J.s) smax = std::max(smax, s);
    if (smax + 1 > S.best_words) {
        cudaFree(S.best);
        S.best = nullptr;
        cudaError_t e = cudaMalloc(&S.best, (smax + 1) * 8);
        if (e != cudaSuccess) return gf2e::cuda_status(e, "server best[]");
        S.best_words = smax + 1;
    }
    GF2E_TRY(gf2e_sieve_fill(S.best, smax, st));
    GF2E_TRY(gf2e_sieve_run(J.r, 2, dsieve, smax, S.best, S.sieve_ws, S.sieve_ws_bytes, st));
    std::vector<uint64_t> best(smax + 1);
    cudaError_t e = cudaMemcpyAsync(best.data(), S.best, (smax + 1) * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "server sieve readback");
    S.sd_pairs_sieve += (uint64_t)J.s.size() * (uint64_t)(dsieve - 1);
    std::vector<uint64_t> deep;
    std::vector<size_t> deep_idx;
    J.lines.assign(J.s.size(), std::string());
    for (size_t i = 0; i < J.s.size(); i++) {
        uint64_t k = best[J.s[i]];
        char buf[96];
        if (k != ~0ull) {
            snprintf(buf, sizeof buf, "%" PRIu64 " %u p%" PRIx64, (uint64_t)J.s[i],
                     (unsigned)(k >> 48), (uint64_t)(k & 0xFFFFFFFFFFFFull));
            J.lines[i] = buf;
        } else if (J.dmax <= (uint64_t)SIEVE_DMAX) {
            snprintf(buf, sizeof buf, "%" PRIu64 " u", J.s[i]);
            J.lines[i] = buf;
        } else {
            deep.push_back(J.s[i]);
            deep_idx.push_back(i);
        }
    }
    J.remaining = deep.size();
    J.admitted = true;
    J.t_admit = now_s();
    if (!deep.empty()) {
        RClass &rc = S.rclass[J.r];
        if (!rc.sc) {
            GF2E_TRY(gf2e_scanner_create_blocked(J.r, S.slots, S.block, &rc.sc));
            gf2e_scanner_footprint_blocked(J.r, S.slots, S.block, &rc.bytes);
            S.used += rc.bytes;
        }
        rc.users++;
        uint64_t tag0 = S.next_tag;
        S.next_tag += deep.size();
        for (size_t q = 0; q < deep.size(); q++) S.tag_owner[tag0 + q] = {J.id, deep_idx[q]};
        GF2E_TRY(gf2e_scanner_submit(rc.sc, deep.data(), (int)deep.size(), SIEVE_DMAX, J.dmax,
                                     J.L0, J.Lmax, tag0));
    } else {
        J.t_done = now_s();
        S.finished.push_back(J.id);
    }
    return GF2E_OK;
}

int try_admit(gf2e_server &S, cudaStream_t st) {
    while (!S.waiting.empty()) {
        Job &J = S.jobs[S.waiting.front()];
        size_t need = 0;
        if (J.dmax > (uint64_t)SIEVE_DMAX && !S.rclass[J.r].sc)
            gf2e_scanner_footprint_blocked(J.r, S.slots, S.block, &need);
        if (S.used + need > S.budget && S.used > 0) break;      // wait for memory
        S.waiting.pop_front();
        GF2E_TRY(admit(S, J, st));
    }
    return GF2E_OK;
}

}  // namespace

extern "C" {

int gf2e_server_create(size_t budget_bytes, int slots_per_r, gf2e_server **out) {
    return gf2e_server_create_blocked(budget_bytes, slots_per_r, 1, out);
}

int gf2e_server_create_blocked(size_t budget_bytes, int slots_per_r, int block,
                               gf2e_server **out) {
    if (!out || slots_per_r < 1) return gf2e::invalid("server: bad arguments");
    if (!(block == 1 || (block >= 2 && block <= 62 && !(block & 1))))
        return gf2e::invalid("server: block size must be 1 or even in 2..62");
    gf2e_server *S = new gf2e_server;
    S->slots = slots_per_r;
    S->block = block;
    int st = gf2e_sieve_workspace_size(SIEVE_DMAX, &S->sieve_ws_bytes);
    if (st != GF2E_OK) { delete S; return st; }
    cudaError_t e = cudaMalloc(&S->sieve_ws, S->sieve_ws_bytes);
    if (e != cudaSuccess) { delete S; return gf2e::cuda_status(e, "server sieve workspace"); }
    S->budget = budget_bytes > S->sieve_ws_bytes ? budget_bytes - S->sieve_ws_bytes : 0;
    S->res.resize(4096);
    S->tags.resize(4096);
    S->masks.resize(4096 * MASK_CAP);
    *out = S;
    return GF2E_OK;
}

int gf2e_server_destroy(gf2e_server *S) {
    if (!S) return GF2E_OK;
    if (S->ev_caller) cudaEventDestroy(S->ev_caller);
    for (cudaEvent_t ev : S->ev_join) cudaEventDestroy(ev);
    for (auto &kv : S->rclass)
        if (kv.second.sc) gf2e_scanner_destroy(kv.second.sc);
    cudaFree(S->sieve_ws);
    cudaFree(S->best);
    delete S;
    return GF2E_OK;
}

int gf2e_server_submit(gf2e_server *S, uint64_t job_id, uint64_t r, const uint64_t *s_host,
                       int ns, uint64_t dmax, uint64_t L0, uint64_t Lmax) {
    if (!S || !s_host || ns < 1 || dmax < 2) return gf2e::invalid("server submit: bad arguments");
    if (S->jobs.count(job_id)) return gf2e::invalid("server submit: duplicate job id");
    if (r < 5 || !(r & 1) || r >= (1ull << 31)) return gf2e::invalid("server submit: bad r");
    for (int i = 0; i < ns; i++)
        if (!(s_host[i] >= 1 && 2 * s_host[i] < r))
            return gf2e::invalid("server submit: s outside 1..(r-1)/2");
    Job J;
    J.id = job_id;
    J.r = r;
    J.dmax = dmax;
    J.L0 = L0 ? L0 : 64;
    J.Lmax = Lmax ? Lmax : 4096;
    J.s.assign(s_host, s_host + ns);
    J.t_submit = now_s();
    S->jobs[job_id] = J;
    S->waiting.push_back(job_id);
    return GF2E_OK;
}

int gf2e_server_step(gf2e_server *S, int degrees, void *stream) {
    if (!S) return gf2e::invalid("null server");
    cudaStream_t st = (cudaStream_t)stream;
    GF2E_TRY(try_admit(*S, st));
    // scanners of different r are independent: each steps on its own stream,
    // after the caller's prior work, and the caller waits for all of them
    if (!S->ev_caller) {
        cudaError_t e = cudaEventCreateWithFlags(&S->ev_caller, cudaEventDisableTiming);
        if (e != cudaSuccess) return gf2e::cuda_status(e, "server event");
    }
    cudaError_t e = cudaEventRecord(S->ev_caller, st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "server stream order");
    size_t nj = 0;
    for (auto it = S->rclass.begin(); it != S->rclass.end(); ++it) {
        RClass &rc = it->second;
        if (!rc.sc) continue;
        cudaStream_t own = gf2e::scanner_stream(rc.sc);
        e = cudaStreamWaitEvent(own, S->ev_caller, 0);
        if (e != cudaSuccess) return gf2e::cuda_status(e, "server stream order");
        GF2E_TRY(gf2e_scanner_step(rc.sc, degrees, own));
        if (nj == S->ev_join.size()) {
            cudaEvent_t ev;
            e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e != cudaSuccess) return gf2e::cuda_status(e, "server event");
            S->ev_join.push_back(ev);
        }
        e = cudaEventRecord(S->ev_join[nj], own);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, S->ev_join[nj], 0);
        if (e != cudaSuccess) return gf2e::cuda_status(e, "server stream join");
        nj++;
        for (;;) {
            int n = 0;
            GF2E_TRY(gf2e_scanner_poll(rc.sc, S->res.data(), S->tags.data(), S->masks.data(),
                                       MASK_CAP, (int)S->res.size(), &n));
            for (int k = 0; k < n; k++) {
                auto own = S->tag_owner.find(S->tags[k]);
                if (own == S->tag_owner.end()) continue;
                Job &J = S->jobs[own->second.first];
                size_t i = own->second.second;
                S->tag_owner.erase(own);
                const gf2e_scan_result &R = S->res[k];
                char buf[64];
                if (R.status == 1) {
                    snprintf(buf, sizeof buf, "%" PRIu64 " %" PRIu64 " p", R.s, R.d);
                    J.lines[i] = buf + hexmask(&S->masks[(size_t)k * MASK_CAP], R.mask_words);
                } else if (R.status == 2) {
                    snprintf(buf, sizeof buf, "%" PRIu64 " u", R.s);
                    J.lines[i] = buf;
                } else {
                    snprintf(buf, sizeof buf, "%" PRIu64 " r%" PRIu64 "-%" PRIu64, R.s, R.rlo, R.rhi);
                    J.lines[i] = buf;
                }
                if (--J.remaining == 0) {
                    J.t_done = now_s();
                    S->finished.push_back(J.id);
                    if (--rc.users == 0) {
                        // keep the scanner only while someone needs it
                        int q = 0, a = 0;
                        gf2e_scanner_status(rc.sc, &q, &a, nullptr, nullptr);
                        if (q == 0 && a == 0) {
                            uint64_t pairs = 0;
                            gf2e_scanner_status(rc.sc, nullptr, nullptr, nullptr, &pairs);
                            S->sd_pairs_scan_retired += pairs;
                            gf2e_scanner_destroy(rc.sc);
                            rc.sc = nullptr;
                            S->used -= rc.bytes;
                        }
                    }
                }
            }
            if (n < (int)S->res.size()) break;
        }
    }
    return try_admit(*S, st);
}

int gf2e_server_status(const gf2e_server *S, int *waiting, int *active, int *finished,
                       size_t *used_bytes) {
    if (!S) return gf2e::invalid("null server");
    int act = 0;
    for (auto &kv : S->jobs)
        if (kv.second.admitted && kv.second.remaining) act++;
    if (waiting) *waiting = (int)S->waiting.size();
    if (active) *active = act;
    if (finished) *finished = (int)S->finished.size();
    if (used_bytes) *used_bytes = S->used;
    return GF2E_OK;
}

int gf2e_server_pairs(const gf2e_server *S, uint64_t *sieved, uint64_t *scanned) {
    if (!S) return gf2e::invalid("null server");
    uint64_t sc = S->sd_pairs_scan_retired;
    for (auto &kv : S->rclass) {
        uint64_t p = 0;
        if (kv.second.sc) gf2e_scanner_status(kv.second.sc, nullptr, nullptr, nullptr, &p);
        sc += p;
    }
    if (sieved) *sieved = S->sd_pairs_sieve;
    if (scanned) *scanned = sc;
    return GF2E_OK;
}

int gf2e_server_poll(gf2e_server *S, uint64_t *job_ids, double *latency_s, int cap, int *nout) {
    if (!S || !job_ids || !nout) return gf2e::invalid("server poll: bad arguments");
    int k = 0;
    while (k < cap && !S->finished.empty()) {
        uint64_t id = S->finished.front();
        S->finished.pop_front();
        job_ids[k] = id;
        if (latency_s) latency_s[k] = S->jobs[id].t_done - S->jobs[id].t_submit;
        k++;
    }
    *nout = k;
    return GF2E_OK;
}

int gf2e_server_job_lines(gf2e_server *S, uint64_t job_id, char *buf, size_t cap,
                          size_t *needed) {
    if (!S || !needed) return gf2e::invalid("server job lines: bad arguments");
    auto it = S->jobs.find(job_id);
    if (it == S->jobs.end()) return gf2e::invalid("unknown job %llu", (unsigned long long)job_id);
    std::string all;
    for (auto &l : it->second.lines) { all += l; all += '\n'; }
    *needed = all.size() + 1;
    if (buf && cap >= all.size() + 1) memcpy(buf, all.c_str(), all.size() + 1);
    return GF2E_OK;
}

int gf2e_server_release(gf2e_server *S, uint64_t job_id) {
    if (!S) return gf2e::invalid("null server");
    S->jobs.erase(job_id);
    return GF2E_OK;
}

}  // extern "C"
