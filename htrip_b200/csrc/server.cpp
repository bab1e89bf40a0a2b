// Request server over many resident map sessions (include/htrip_b200.h,
// htrip_server_*).  Written on top of the index C ABI only.
//
// The reference serves one robot team per process: its simulator keeps a
// front and a back MinPlusOracle, applies onBatchCellsOpened on a worker
// thread and swaps them, while queries read the front copy
// (robot_simulator.cpp:897-1045, :1478-1545).  Here one process keeps many
// maps resident in HBM and serves their requests with continuous batching:
//
//  * Every session has a FIFO of requests.  Requests of one session run in
//    arrival order and never overlap (an opening mutates the index a query
//    reads); requests of different sessions are independent.
//  * Two workers, one for queries and one for openings, each with its own
//    stream and scratch (htrip_batch).  A worker takes, from every idle
//    session whose oldest request is of its kind, the run of such requests
//    at the head of the queue: all of those queries go into ONE launch of
//    the persistent query kernel (htrip_query_batch); the openings of one
//    session are merged into one onBatchCellsOpened (the closure of the
//    union equals the closure after the calls in turn) and all sessions'
//    openings advance level by level together (htrip_open_batch).  Requests
//    that arrive while a launch is on the GPU wait for the next one.
//  * Memory: sessions are admitted against an HBM budget by the estimated
//    footprint of their index (htrip_estimate_bytes).  When a new session
//    or a request for an offloaded session needs room, idle sessions are
//    offloaded to host memory, least recently used first
//    (htrip_offload / htrip_restore); when even that cannot make room the
//    new session is refused with HTRIP_ERR_OOM.
//  * Double-buffered sessions (htrip_server_config::double_buffer), the
//    reference simulator's protocol for every session: the session holds a
//    front index that queries read and a back index that openings update;
//    queries never wait behind the session's openings.  The open worker
//    applies to the back the batch it still lacks (the last one published)
//    merged with the new openings, then swaps the two; a back index is never
//    updated while a query launch may still read it.  Each query reports
//    the number of the session's openings its result includes.
//  * Latency of a request = time from its submission to its result being
//    in host memory and marked done.
#include "../../include/htrip_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

enum Kind { kQuery = 0, kOpen = 1 };

struct SReq {
    uint64_t ticket = 0;
    int kind = kQuery;
    int64_t sid = 0;
    std::vector<int32_t> rc;  // viewpoints or cells
    uint16_t* out = nullptr;  // query result (k*k), caller memory
    Clock::time_point t0, t1;
    uint64_t version = 0;     // query: openings its result includes; opening: its number
    bool done = false;
    htrip_status status = HTRIP_OK;
    std::string error;
};

struct Session {
    int64_t id = 0;
    htrip_index* h = nullptr;   // the index (double-buffered: the front one, queried)
    std::vector<uint8_t> grid;  // the session's observed grid (CellState) as h has it
    int rows = 0, cols = 0;
    std::deque<SReq*> q;        // requests (double-buffered: the queries)
    bool busy = false;
    bool resident = true;
    uint64_t bytes = 0;
    uint64_t last_use = 0;
    uint64_t opens_submitted = 0;
    // double-buffered sessions
    bool dbuf = false;
    htrip_index* hb = nullptr;    // the back index (updated by openings)
    std::vector<uint8_t> grid_b;  // the grid as hb has it
    std::deque<SReq*> oq;         // queued openings
    bool qbusy = false, obusy = false;
    int reads = 0, reads_b = 0;   // query launches in flight on h / on hb
    uint64_t version = 0;         // openings published into h
    std::vector<int32_t> pending; // cells of the last published batch (hb lacks them)
};

bool idle(const Session& s) { return s.dbuf ? !s.qbusy && !s.obusy && s.reads == 0 && s.reads_b == 0 : !s.busy; }
bool drained(const Session& s) { return s.q.empty() && s.oq.empty() && idle(s); }

}  // namespace

struct htrip_server {
    int device = 0;
    uint64_t budget = 0;
    int max_per_launch = 128;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<int64_t, Session> sessions;
    std::unordered_map<uint64_t, std::unique_ptr<SReq>> reqs;
    uint64_t next_ticket = 1;
    int64_t next_sid = 1;
    uint64_t tick = 0;
    uint64_t resident_bytes = 0;
    bool stop = false;
    uint64_t completions = 0;  // launches finished (wakes workers waiting for memory)
    bool dbuf = false;         // new sessions are double-buffered
    htrip_server_stats st{};
    htrip_batch* batch[2] = {nullptr, nullptr};
    std::thread worker[2];
};

namespace {

thread_local std::string t_err;

htrip_status sfail(htrip_status s, const std::string& m) {
    t_err = m;
    return s;
}

// Offloads idle resident sessions, least recently used first, until `need`
// more bytes fit under the budget.  Caller holds mu.  False if impossible.
bool make_room(htrip_server* S, uint64_t need, int64_t keep) {
    while (S->resident_bytes + need > S->budget) {
        Session* victim = nullptr;
        for (auto& kv : S->sessions) {
            Session& s = kv.second;
            if (!s.resident || !idle(s) || s.id == keep || !s.q.empty() || !s.oq.empty()) continue;
            if (!victim || s.last_use < victim->last_use) victim = &s;
        }
        if (!victim)  // sessions with queued work only if nothing else is left
            for (auto& kv : S->sessions) {
                Session& s = kv.second;
                if (!s.resident || !idle(s) || s.id == keep) continue;
                if (!victim || s.last_use < victim->last_use) victim = &s;
            }
        if (!victim) return false;
        if (htrip_offload(victim->h) != HTRIP_OK) return false;
        if (victim->hb && htrip_offload(victim->hb) != HTRIP_OK) return false;
        victim->resident = false;
        S->resident_bytes -= victim->bytes;
        S->st.evictions++;
        S->st.resident_sessions--;
    }
    return true;
}

// Brings `s` back to the device (caller holds mu; s is busy).
htrip_status ensure_resident(htrip_server* S, Session& s) {
    if (s.resident) return HTRIP_OK;
    if (!make_room(S, s.bytes, s.id)) return sfail(HTRIP_ERR_OOM, "no room to restore the session within the budget");
    htrip_status r = htrip_restore(s.h);
    if (r == HTRIP_OK && s.hb) r = htrip_restore(s.hb);
    if (r != HTRIP_OK) return sfail(r, htrip_last_error());
    s.resident = true;
    S->resident_bytes += s.bytes;
    S->st.restores++;
    S->st.resident_sessions++;
    return HTRIP_OK;
}

// Whether worker `kind` can take session s now.
bool takes(const Session& s, int kind) {
    if (!s.dbuf) return !s.busy && !s.q.empty() && s.q.front()->kind == kind;
    if (kind == kQuery) return !s.qbusy && !s.q.empty();
    return !s.obusy && !s.oq.empty() && s.reads_b == 0;
}

bool has_work(htrip_server* S, int kind) {
    for (auto& kv : S->sessions)
        if (takes(kv.second, kind)) return true;
    return false;
}

void worker_loop(htrip_server* S, int kind) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_work.wait(lk, [&] { return S->stop || has_work(S, kind); });
        if (S->stop && !has_work(S, kind)) return;
        // Take the head runs of every idle session, oldest sessions' work first.
        struct Item {
            Session* s;
            std::vector<SReq*> r;
            htrip_index* h = nullptr;         // the index the launch reads or updates
            const uint8_t* grid = nullptr;
        };
        std::vector<Item> items;
        int taken = 0;
        std::vector<Session*> cand;
        for (auto& kv : S->sessions)
            if (takes(kv.second, kind)) cand.push_back(&kv.second);
        auto head = [kind](const Session* s) { return (s->dbuf && kind == kOpen ? s->oq : s->q).front()->t0; };
        std::sort(cand.begin(), cand.end(), [&](const Session* a, const Session* b) { return head(a) < head(b); });
        for (Session* s : cand) {
            if (taken >= S->max_per_launch) break;
            Item it{s, {}};
            for (SReq* r : (s->dbuf && kind == kOpen ? s->oq : s->q)) {
                if (r->kind != kind || taken >= S->max_per_launch) break;
                it.r.push_back(r);
                ++taken;
            }
            if (!s->dbuf) s->busy = true;
            else if (kind == kQuery) s->qbusy = true;
            else s->obusy = true;
            s->last_use = ++S->tick;
            items.push_back(std::move(it));
        }
        // Residency (rare path: only when sessions were offloaded).  A
        // session that cannot be brought back now - the budget is held by
        // sessions busy in this launch or in the other worker's - stays
        // queued for a later launch; with nothing ready at all the worker
        // waits for some launch to finish before it tries again.
        std::vector<Item> ready;
        for (auto& it : items) {
            Session& s = *it.s;
            if (ensure_resident(S, s) != HTRIP_OK) {
                if (!s.dbuf) s.busy = false;
                else if (kind == kQuery) s.qbusy = false;
                else s.obusy = false;
                continue;
            }
            if (s.dbuf && kind == kQuery) {  // the published state, read until the launch ends
                it.h = s.h;
                it.grid = s.grid.data();
                ++s.reads;
                for (SReq* r : it.r) r->version = s.version;
            } else if (s.dbuf) {
                it.h = s.hb;
                it.grid = s.grid_b.data();
            } else {
                it.h = s.h;
                it.grid = s.grid.data();
            }
            ready.push_back(std::move(it));
        }
        if (ready.empty()) {
            const uint64_t seen = S->completions;
            S->cv_work.wait(lk, [&] { return S->stop || S->completions != seen; });
            continue;
        }
        lk.unlock();
        htrip_status rs = HTRIP_OK;
        std::string err;
        const auto tb = Clock::now();
        if (!ready.empty()) {
            if (kind == kQuery) {
                std::vector<htrip_query_request> qr;
                for (auto& it : ready)
                    for (SReq* r : it.r)
                        qr.push_back({it.h, r->rc.data(), (int32_t)(r->rc.size() / 2), it.grid, it.s->rows,
                                      it.s->cols, r->out});
                rs = htrip_query_batch(S->batch[kind], qr.data(), (int32_t)qr.size());
            } else {
                std::vector<std::vector<int32_t>> merged(ready.size());
                std::vector<htrip_open_request> orq;
                for (size_t i = 0; i < ready.size(); ++i) {
                    Session& s = *ready[i].s;
                    // double-buffered: the back first catches up with the last published batch
                    if (s.dbuf) merged[i] = s.pending;
                    std::vector<uint8_t>& g = s.dbuf ? s.grid_b : s.grid;
                    auto mark = [&](const std::vector<int32_t>& rc) {  // the caller's protocol: Free before the call
                        for (size_t c = 0; c + 1 < rc.size(); c += 2) {
                            const int32_t rr = rc[c], cc = rc[c + 1];
                            if (rr >= 0 && cc >= 0 && rr < s.rows && cc < s.cols) g[(size_t)rr * s.cols + cc] = 1;
                        }
                    };
                    mark(merged[i]);
                    for (SReq* r : ready[i].r) {
                        mark(r->rc);
                        merged[i].insert(merged[i].end(), r->rc.begin(), r->rc.end());
                    }
                    orq.push_back({ready[i].h, merged[i].data(), (int32_t)(merged[i].size() / 2), g.data(), s.rows,
                                   s.cols});
                }
                rs = htrip_open_batch(S->batch[kind], orq.data(), (int32_t)orq.size());
            }
            if (rs != HTRIP_OK) err = htrip_last_error();
        }
        const auto t1 = Clock::now();
        lk.lock();
        for (auto& it : ready) {
            Session& s = *it.s;
            std::vector<int32_t> batch;
            for (SReq* r : it.r) {
                r->status = rs;
                r->error = err;
                r->t1 = t1;
                r->done = true;
                (s.dbuf && kind == kOpen ? s.oq : s.q).pop_front();
                if (s.dbuf && kind == kOpen) batch.insert(batch.end(), r->rc.begin(), r->rc.end());
            }
            if (!s.dbuf) {
                s.busy = false;
            } else if (kind == kQuery) {
                if (it.h == s.h) --s.reads;  // the index may have been swapped meanwhile
                else --s.reads_b;
                s.qbusy = false;
            } else {
                s.obusy = false;
                if (rs == HTRIP_OK) {  // publish: the back becomes the front
                    std::swap(s.h, s.hb);
                    std::swap(s.grid, s.grid_b);
                    std::swap(s.reads, s.reads_b);
                    s.version += it.r.size();
                    s.pending = std::move(batch);
                }
            }
            s.last_use = ++S->tick;
        }
        const double busy = std::chrono::duration<double>(t1 - tb).count();
        if (kind == kQuery) {
            S->st.launches_query++;
            S->st.busy_query_us += (uint64_t)(busy * 1e6);
        } else {
            S->st.launches_open++;
            S->st.busy_open_us += (uint64_t)(busy * 1e6);
        }
        S->completions++;
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

// The plain per-call baseline: one worker, one request at a time in global
// arrival order, each through the single-index calls (htrip_query_all_pairs
// / htrip_open_cells) - no batching, no overlap.
void worker_loop_plain(htrip_server* S) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        auto any = [&] {
            for (auto& kv : S->sessions)
                if (!kv.second.q.empty()) return true;
            return false;
        };
        S->cv_work.wait(lk, [&] { return S->stop || any(); });
        if (S->stop && !any()) return;
        Session* s = nullptr;
        for (auto& kv : S->sessions) {
            Session& c = kv.second;
            if (!c.q.empty() && (!s || c.q.front()->t0 < s->q.front()->t0)) s = &c;
        }
        SReq* r = s->q.front();
        s->busy = true;
        s->last_use = ++S->tick;
        htrip_status rs = ensure_resident(S, *s);  // one session at a time: only fails if it alone cannot fit
        std::string err = rs != HTRIP_OK ? t_err : std::string();
        lk.unlock();
        if (rs == HTRIP_OK) {
            const int32_t n = (int32_t)(r->rc.size() / 2);
            if (r->kind == kQuery) {
                rs = htrip_query_all_pairs(s->h, r->rc.data(), n, s->grid.data(), s->rows, s->cols, r->out);
            } else {
                for (int32_t c = 0; c < n; ++c) {
                    const int32_t rr = r->rc[2 * c], cc = r->rc[2 * c + 1];
                    if (rr >= 0 && cc >= 0 && rr < s->rows && cc < s->cols) s->grid[(size_t)rr * s->cols + cc] = 1;
                }
                rs = htrip_open_cells(s->h, r->rc.data(), n, s->grid.data(), s->rows, s->cols);
            }
            if (rs != HTRIP_OK) err = htrip_last_error();
        }
        const auto t1 = Clock::now();
        lk.lock();
        r->status = rs;
        r->error = err;
        r->t1 = t1;
        r->done = true;
        s->q.pop_front();
        s->busy = false;
        if (r->kind == kQuery) S->st.launches_query++;
        else S->st.launches_open++;
        S->completions++;
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

htrip_status submit(htrip_server* S, int64_t sid, int kind, const int32_t* rc, int32_t n, uint16_t* out,
                    uint64_t* ticket) {
    auto r = std::make_unique<SReq>();
    r->kind = kind;
    r->sid = sid;
    r->rc.assign(rc, rc + 2 * (size_t)n);
    r->out = out;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->sessions.find(sid);
    if (it == S->sessions.end()) return sfail(HTRIP_ERR_INVALID, "unknown session " + std::to_string(sid));
    r->ticket = S->next_ticket++;
    r->t0 = Clock::now();
    SReq* p = r.get();
    S->reqs[p->ticket] = std::move(r);
    Session& s = it->second;
    if (kind == kOpen) p->version = ++s.opens_submitted;
    else p->version = s.opens_submitted;  // single-buffered: every earlier opening
    (s.dbuf && kind == kOpen ? s.oq : s.q).push_back(p);
    if (kind == kQuery) S->st.requests_query++;
    else S->st.requests_open++;
    *ticket = p->ticket;
    S->cv_work.notify_all();
    return HTRIP_OK;
}

}  // namespace

extern "C" {

const char* htrip_server_last_error(void) { return t_err.c_str(); }

htrip_status htrip_server_create(const htrip_server_config* cfg, htrip_server** out) {
    if (!cfg || !out) return sfail(HTRIP_ERR_INVALID, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return sfail(HTRIP_ERR_NO_DEVICE, "no CUDA device");
    }
    if (cfg->device < 0 || cfg->device >= ndev) return sfail(HTRIP_ERR_INVALID, "bad device ordinal");
    auto* S = new htrip_server();
    S->device = cfg->device;
    S->max_per_launch = cfg->max_requests_per_launch > 0 ? cfg->max_requests_per_launch : 128;
    S->budget = cfg->hbm_budget_bytes;
    S->dbuf = cfg->double_buffer != 0 && !cfg->plain_per_call;
    if (S->budget == 0) {
        size_t fr = 0, tot = 0;
        cudaSetDevice(S->device);
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            delete S;
            return sfail(HTRIP_ERR_CUDA, "cudaMemGetInfo failed");
        }
        S->budget = (uint64_t)(fr * 0.80);
    }
    for (int k = 0; k < 2; ++k) {
        // queries on a high-priority stream: the cooperative query launch gets
        // the SMs ahead of the openings' many small kernels
        const htrip_status r = htrip_batch_create_priority(S->device, k == kQuery ? 1 : 0, &S->batch[k]);
        if (r != HTRIP_OK) {
            const std::string e = htrip_last_error();
            for (auto* b : S->batch) htrip_batch_destroy(b);
            delete S;
            return sfail(r, e);
        }
    }
    if (cfg->plain_per_call) S->worker[0] = std::thread(worker_loop_plain, S);
    else
        for (int k = 0; k < 2; ++k) S->worker[k] = std::thread(worker_loop, S, k);
    *out = S;
    return HTRIP_OK;
}

htrip_status htrip_server_destroy(htrip_server* S) {
    if (!S) return HTRIP_OK;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        // finish the queued work first
        S->cv_done.wait(lk, [&] {
            for (auto& kv : S->sessions)
                if (!drained(kv.second)) return false;
            return true;
        });
        S->stop = true;
        S->cv_work.notify_all();
    }
    for (auto& w : S->worker)
        if (w.joinable()) w.join();
    for (auto& kv : S->sessions) {
        htrip_destroy(kv.second.h);
        htrip_destroy(kv.second.hb);
    }
    for (auto* b : S->batch) htrip_batch_destroy(b);
    delete S;
    return HTRIP_OK;
}

htrip_status htrip_server_add_session(htrip_server* S, htrip_config cfg, const uint8_t* observed, int32_t rows,
                                      int32_t cols, int64_t* session) {
    if (!S || !observed || !session) return sfail(HTRIP_ERR_INVALID, "null argument");
    uint64_t est = 0;
    htrip_status r = htrip_estimate_bytes(cfg, rows, cols, &est);
    if (r != HTRIP_OK) return sfail(r, htrip_last_error());
    if (S->dbuf) est *= 2;  // front and back index
    std::lock_guard<std::mutex> lk(S->mu);
    if (est > S->budget) return sfail(HTRIP_ERR_OOM, "session needs " + std::to_string(est) + " bytes; budget is " +
                                                         std::to_string(S->budget));
    if (!make_room(S, est, -1))
        return sfail(HTRIP_ERR_OOM, "session of " + std::to_string(est) + " bytes refused: budget " +
                                        std::to_string(S->budget) + " bytes held by busy sessions");
    htrip_index* h = nullptr;
    htrip_index* hb = nullptr;
    r = htrip_create(cfg, S->device, &h);
    if (r == HTRIP_OK) r = htrip_build(h, observed, rows, cols);
    if (r == HTRIP_OK && S->dbuf) r = htrip_clone(h, &hb);
    if (r != HTRIP_OK) {
        const std::string e = htrip_last_error();
        htrip_destroy(h);
        htrip_destroy(hb);
        return sfail(r, e);
    }
    Session s;
    s.id = S->next_sid++;
    s.h = h;
    s.hb = hb;
    s.dbuf = S->dbuf;
    if (s.dbuf) s.grid_b.assign(observed, observed + (size_t)rows * cols);
    s.grid.assign(observed, observed + (size_t)rows * cols);
    s.rows = rows;
    s.cols = cols;
    s.bytes = est;
    s.last_use = ++S->tick;
    S->resident_bytes += est;
    S->st.sessions++;
    S->st.resident_sessions++;
    *session = s.id;
    S->sessions.emplace(s.id, std::move(s));
    return HTRIP_OK;
}

htrip_status htrip_server_remove_session(htrip_server* S, int64_t sid) {
    if (!S) return sfail(HTRIP_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->sessions.find(sid);
    if (it == S->sessions.end()) return sfail(HTRIP_ERR_INVALID, "unknown session " + std::to_string(sid));
    S->cv_done.wait(lk, [&] { return drained(it->second); });
    if (it->second.resident) {
        S->resident_bytes -= it->second.bytes;
        S->st.resident_sessions--;
    }
    S->st.sessions--;
    htrip_destroy(it->second.h);
    htrip_destroy(it->second.hb);
    S->sessions.erase(it);
    return HTRIP_OK;
}

htrip_status htrip_server_submit_query(htrip_server* S, int64_t sid, const int32_t* vps, int32_t k, uint16_t* out,
                                       uint64_t* ticket) {
    if (!S || !ticket || k < 0 || (k > 0 && (!vps || !out))) return sfail(HTRIP_ERR_INVALID, "bad arguments");
    return submit(S, sid, kQuery, vps, k, out, ticket);
}

htrip_status htrip_server_submit_open(htrip_server* S, int64_t sid, const int32_t* rc, int32_t n, uint64_t* ticket) {
    if (!S || !ticket || n < 0 || (n > 0 && !rc)) return sfail(HTRIP_ERR_INVALID, "bad arguments");
    return submit(S, sid, kOpen, rc, n, nullptr, ticket);
}

htrip_status htrip_server_wait(htrip_server* S, uint64_t ticket, double* latency_ms) {
    return htrip_server_wait_version(S, ticket, latency_ms, nullptr);
}

htrip_status htrip_server_wait_version(htrip_server* S, uint64_t ticket, double* latency_ms, uint64_t* version) {
    if (!S) return sfail(HTRIP_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return sfail(HTRIP_ERR_INVALID, "unknown ticket " + std::to_string(ticket));
    SReq* r = it->second.get();
    S->cv_done.wait(lk, [&] { return r->done; });
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t1 - r->t0).count();
    if (version) *version = r->version;
    const htrip_status st = r->status;
    const std::string e = r->error;
    S->reqs.erase(it);
    if (st != HTRIP_OK) return sfail(st, e);
    return HTRIP_OK;
}

htrip_status htrip_server_get_stats(htrip_server* S, htrip_server_stats* out) {
    if (!S || !out) return sfail(HTRIP_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->st;
    out->resident_bytes = S->resident_bytes;
    out->budget_bytes = S->budget;
    return HTRIP_OK;
}

htrip_status htrip_server_run_trace(htrip_server* S, const htrip_server_request* reqs, const double* arrival_s,
                                    int32_t n, double* latency_ms, double* wall_s) {
    if (!S || n < 0 || (n > 0 && (!reqs || !arrival_s || !latency_ms))) return sfail(HTRIP_ERR_INVALID, "bad arguments");
    std::vector<uint64_t> tickets(n, 0);
    std::vector<htrip_status> sub(n, HTRIP_OK);
    const auto start = Clock::now();
    for (int i = 0; i < n; ++i) {
        const auto due = start + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
        // sleep until shortly before the arrival, then spin: a submitter
        // spinning through every gap would hold a core the workers need (and
        // under a CPU quota, get every thread of the process throttled)
        if (due - Clock::now() > std::chrono::microseconds(300))
            std::this_thread::sleep_until(due - std::chrono::microseconds(200));
        while (Clock::now() < due) {
        }
        const htrip_server_request& q = reqs[i];
        sub[i] = q.kind == kQuery ? htrip_server_submit_query(S, q.session, q.rc, q.n, q.out, &tickets[i])
                                  : htrip_server_submit_open(S, q.session, q.rc, q.n, &tickets[i]);
    }
    htrip_status first = HTRIP_OK;
    std::string first_err;
    for (int i = 0; i < n; ++i) {
        latency_ms[i] = -1.0;
        htrip_status r = sub[i];
        if (r == HTRIP_OK) r = htrip_server_wait(S, tickets[i], &latency_ms[i]);
        if (r != HTRIP_OK && first == HTRIP_OK) {
            first = r;
            first_err = "request " + std::to_string(i) + ": " + t_err;
        }
    }
    if (wall_s) *wall_s = std::chrono::duration<double>(Clock::now() - start).count();
    if (first != HTRIP_OK) return sfail(first, first_err);
    return HTRIP_OK;
}

}  // extern "C"
