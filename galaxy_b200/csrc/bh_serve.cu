// SPDX-License-Identifier: Apache-2.0
// Native continuous-batching server over the public C ABI (galaxy_bh.h).
//
// Two host threads, each owning a device handle (and so a stream) of the
// same GPU.  The stager takes submitted requests (initial state records,
// config, dt, step count) in arrival order as soon as the device-memory
// footprint of the active set, the staged requests and the newcomer fits
// the budget; it uploads and checks the newcomer's state and solves its
// boundary acceleration while the rounds go on, then hands the state to the
// serving loop's handle.  The serving loop admits staged requests between
// rounds; admitted simulations stay resident and advance together, a round
// of fused KDK steps at a time, in one batch (one launch per stage for all
// of them).  A round stops at the smallest remaining step count, so finished
// simulations leave and staged ones join between rounds.  Finished results
// are copied back and queued for galaxy_bh_serve_poll.  Each simulation's
// result equals its result alone: batch members never interact.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "bh_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct ServeRequest {
    uint64_t id = 0;
    std::vector<GpuEvolveState> records;  // initial state, then the result
    bh_config cfg{};
    double dt = 0.0;
    uint32_t n = 0, steps = 0, remaining = 0;
    int status = BH_OK;
    double submitted_s = 0.0, admitted_s = -1.0, finished_s = -1.0;
    bh_state* st = nullptr;
};

}  // namespace

struct bh_server {
    bh_device* dev = nullptr;    // the serving loop's handle: rounds of steps
    bh_device* dev2 = nullptr;   // the stager's handle: uploads and boundary solves
    bh_serve_config sc{};
    Clock::time_point t0;
    std::thread loop, stager;
    std::mutex mu;
    std::condition_variable cv_in, cv_out, cv_stage;
    // submitted -> (stager: state uploaded, checked, boundary-solved) staged
    // -> (loop) active -> done
    std::deque<std::unique_ptr<ServeRequest>> submitted, staged, done;
    // the active members' sizes and configs, published by the loop for the
    // stager's budget check
    std::vector<uint32_t> active_n;
    std::vector<bh_config> active_cfg;
    bool stopping = false;
    int pollers = 0;  // polls inside galaxy_bh_serve_poll (stop waits for them)
    uint64_t next_id = 1;
    uint64_t rounds = 0, particle_steps = 0, completed = 0;
    double busy_s = 0.0;
    double admit_s = 0.0, solve_s = 0.0, form_s = 0.0, readback_s = 0.0;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

void finish(bh_server* s, std::unique_ptr<ServeRequest> r) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->status == BH_OK) ++s->completed;
    s->done.push_back(std::move(r));
    s->cv_out.notify_all();
}

void release_state(std::unique_ptr<ServeRequest>& r) {
    if (r->st) galaxy_bh_state_destroy(r->st);
    r->st = nullptr;
}

// Re-forms *b over the active requests, reusing its arena when it is large
// enough (the arena grows to the largest active set and stays).
int form_batch(bh_server* s, std::vector<std::unique_ptr<ServeRequest>>& active, bh_batch** b) {
    std::vector<bh_state*> states;
    std::vector<bh_config> cfgs;
    for (auto& r : active) {
        states.push_back(r->st);
        cfgs.push_back(r->cfg);
    }
    return gbh::batch_reform(s->dev, b, states.data(), cfgs.data(), (uint32_t)states.size());
}

// Whether `cand` joins the active members and the staged requests inside
// the budget (caller holds s->mu); *alone_too_big when it can never fit.
bool fits_budget(bh_server* s, const ServeRequest& cand, bool* alone_too_big) {
    std::vector<uint32_t> counts(s->active_n);
    std::vector<bh_config> cfgs(s->active_cfg);
    for (auto& r : s->staged) {
        counts.push_back(r->n);
        cfgs.push_back(r->cfg);
    }
    counts.push_back(cand.n);
    cfgs.push_back(cand.cfg);
    uint64_t bytes = 0, alone = 0;
    *alone_too_big = false;
    if (galaxy_bh_batch_footprint(counts.data(), cfgs.data(), (uint32_t)counts.size(), &bytes) !=
        BH_OK)
        return false;
    if (bytes <= s->sc.budget_bytes) return true;
    if (galaxy_bh_batch_footprint(&cand.n, &cand.cfg, 1, &alone) == BH_OK &&
        alone > s->sc.budget_bytes)
        *alone_too_big = true;
    return false;
}

constexpr size_t kStageAhead = 4;  // requests the stager prepares ahead of admission

// The stager: in arrival order, for the requests that fit the budget next to
// the active and the already staged ones, uploads and checks the initial
// state and runs its boundary solve (rebuild + force on the stager's own
// tree, reused from request to request) on the stager's handle and stream,
// so that this host work and its copies
// overlap the rounds the loop keeps running; then hands the state to the
// loop's handle.  A simulation's result does not depend on where its solve
// ran: the tree kernels are the same.
void stage_loop(bh_server* s) {
    // pinned staging of the records: an upload from pageable memory goes
    // through the driver's shared bounce buffers, which would hold up the
    // serving loop's own small uploads behind this one
    GpuEvolveState* pinned = nullptr;
    size_t pinned_n = 0;
    // one tree, pointed at each newcomer in turn: its arena grows to the
    // largest request solved and is then reused
    bh_tree* tree = nullptr;
    while (true) {
        std::unique_ptr<ServeRequest> r;
        int rc = BH_OK;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            bool too_big = false;
            s->cv_stage.wait(lk, [&] {
                return s->stopping ||
                       (!s->submitted.empty() && s->staged.size() < kStageAhead &&
                        (fits_budget(s, *s->submitted.front(), &too_big) || too_big));
            });
            if (s->stopping) break;
            r = std::move(s->submitted.front());
            s->submitted.pop_front();
            if (too_big) rc = BH_CAPACITY_OVERFLOW;  // alone it can never fit
        }
        const double t0 = s->now();
        const GpuEvolveState* src = r->records.data();
        if (rc == BH_OK) {
            if (pinned_n < r->n) {
                if (pinned) cudaFreeHost(pinned);
                pinned = nullptr;
                pinned_n = 0;
                if (cudaMallocHost((void**)&pinned, sizeof(GpuEvolveState) * (size_t)r->n) ==
                    cudaSuccess)
                    pinned_n = r->n;
                else
                    cudaGetLastError();  // upload from the pageable copy instead
            }
            if (pinned_n >= r->n) {
                std::memcpy(pinned, src, sizeof(GpuEvolveState) * (size_t)r->n);
                src = pinned;
            }
            rc = galaxy_bh_state_create(s->dev2, src, r->n, &r->st, nullptr);
        }
        const double t1 = s->now();
        if (rc == BH_OK) {
            rc = gbh::tree_retarget(s->dev2, &tree, r->st, &r->cfg);
            if (rc == BH_OK) rc = galaxy_bh_tree_rebuild(s->dev2, r->st, tree, &r->cfg, nullptr);
            bh_config fc = r->cfg;
            fc.flags |= BH_FLAG_NO_STATS;
            if (rc == BH_OK) rc = galaxy_bh_force(s->dev2, r->st, tree, &fc, nullptr);
            if (rc == BH_OK) rc = gbh::state_move(r->st, s->dev);
        }
        const double t2 = s->now();
        if (rc != BH_OK) {
            release_state(r);
            r->status = rc;
            r->finished_s = s->now();
            finish(s, std::move(r));
            std::lock_guard<std::mutex> lk(s->mu);
            s->admit_s += t1 - t0;
            s->solve_s += t2 - t1;
            continue;
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->admit_s += t1 - t0;
        s->solve_s += t2 - t1;
        s->staged.push_back(std::move(r));
        s->cv_in.notify_all();
    }
    if (tree) galaxy_bh_tree_destroy(tree);
    if (pinned) cudaFreeHost(pinned);
}

void serve_loop(bh_server* s) {
    std::vector<std::unique_ptr<ServeRequest>> active;
    bh_batch* batch = nullptr;
    // publishes the active set for the stager's budget check (caller holds mu)
    auto publish = [&]() {
        s->active_n.clear();
        s->active_cfg.clear();
        for (auto& r : active) {
            s->active_n.push_back(r->n);
            s->active_cfg.push_back(r->cfg);
        }
        s->cv_stage.notify_all();
    };
    auto fail_all_active = [&](int rc) {
        for (auto& r : active) {
            release_state(r);
            r->status = rc;
            r->finished_s = s->now();
            finish(s, std::move(r));
        }
        active.clear();
        if (batch) galaxy_bh_batch_destroy(batch);
        batch = nullptr;
        std::lock_guard<std::mutex> lk(s->mu);
        publish();
    };
    while (true) {
        // admission: staged requests join in arrival order (the stager kept
        // the active set plus every staged request inside the budget)
        bool joined = false;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stopping) break;
            if (s->staged.empty() && active.empty()) {
                s->cv_in.wait_for(lk, std::chrono::milliseconds(50));
                continue;
            }
            while (!s->staged.empty() && active.size() < s->sc.max_members) {
                std::unique_ptr<ServeRequest> r = std::move(s->staged.front());
                s->staged.pop_front();
                r->admitted_s = s->now();
                r->remaining = r->steps;
                active.push_back(std::move(r));
                joined = true;
            }
            if (joined) publish();
        }
        if (joined) {
            // every member holds its boundary acceleration: the newcomers'
            // from their staged solves, the others' from their last step
            const double tf = s->now();
            const int rc = form_batch(s, active, &batch);
            {
                std::lock_guard<std::mutex> lk(s->mu);
                s->form_s += s->now() - tf;
            }
            if (rc != BH_OK) {
                fail_all_active(rc);
                continue;
            }
        }
        uint32_t r_steps = s->sc.round_steps;
        uint64_t bodies = 0;
        std::vector<double> dts;
        for (auto& r : active) {
            r_steps = std::min(r_steps, r->remaining);
            bodies += r->n;
            dts.push_back(r->dt);
        }
        const double tb = s->now();
        int rc = galaxy_bh_batch_step(s->dev, batch, dts.data(), r_steps);
        if (rc != BH_OK) {
            fail_all_active(rc);
            continue;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->busy_s += s->now() - tb;
            ++s->rounds;
            s->particle_steps += bodies * r_steps;
        }
        std::vector<std::unique_ptr<ServeRequest>> still;
        bool left = false;
        const double tr = s->now();
        for (auto& r : active) {
            r->remaining -= r_steps;
            if (r->remaining == 0) {
                r->status = galaxy_bh_read_state(s->dev, r->st, r->records.data(), r->n, nullptr);
                r->finished_s = s->now();
                release_state(r);
                finish(s, std::move(r));
                left = true;
            } else {
                still.push_back(std::move(r));
            }
        }
        active = std::move(still);
        const double tf = s->now();
        if (left) {
            {
                std::lock_guard<std::mutex> lk(s->mu);
                publish();
            }
            // re-formed batches step at once: every member's acceleration
            // buffer holds its boundary acceleration
            if ((rc = form_batch(s, active, &batch)) != BH_OK) fail_all_active(rc);
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->readback_s += tf - tr;
            s->form_s += s->now() - tf;
        }
    }
    if (batch) galaxy_bh_batch_destroy(batch);
    for (auto& r : active) release_state(r);
}

}  // namespace

using gbh::set_error_message;

extern "C" int galaxy_bh_serve_start(int ordinal, const bh_serve_config* config,
                                     bh_server** out) {
    if (!config || !out) return set_error_message(BH_INVALID_ARG, "null argument");
    *out = nullptr;
    if (config->round_steps == 0 || config->max_members == 0 || config->budget_bytes == 0)
        return set_error_message(BH_INVALID_ARG,
                                 "serve config needs a budget, round_steps and max_members");
    bh_device* dev = nullptr;
    bh_device* dev2 = nullptr;
    int rc = galaxy_bh_device_open(ordinal, &dev);
    if (rc != BH_OK) return rc;
    if ((rc = galaxy_bh_device_open(ordinal, &dev2)) != BH_OK) {
        galaxy_bh_device_close(dev);
        return rc;
    }
    bh_server* s = new bh_server();
    s->dev = dev;
    s->dev2 = dev2;
    s->sc = *config;
    s->t0 = Clock::now();
    s->loop = std::thread(serve_loop, s);
    s->stager = std::thread(stage_loop, s);
    *out = s;
    return BH_OK;
}

extern "C" int galaxy_bh_serve_submit(bh_server* s, const GpuEvolveState* host, uint32_t n,
                                      const bh_config* cfg, double dt, uint32_t steps,
                                      uint64_t* request_id) {
    if (!s || !host || !cfg || !request_id)
        return set_error_message(BH_INVALID_ARG, "null argument");
    if (n < 2 || steps == 0)
        return set_error_message(BH_INVALID_ARG, "a request needs n >= 2 bodies and steps >= 1");
    auto r = std::make_unique<ServeRequest>();
    r->records.assign(host, host + n);
    r->cfg = *cfg;
    r->dt = dt;
    r->n = n;
    r->steps = steps;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return set_error_message(BH_INVALID_ARG, "server is stopping");
    r->id = s->next_id++;
    r->submitted_s = s->now();
    *request_id = r->id;
    s->submitted.push_back(std::move(r));
    s->cv_in.notify_all();
    s->cv_stage.notify_all();
    return BH_OK;
}

extern "C" int galaxy_bh_serve_poll(bh_server* s, uint32_t timeout_ms, bh_serve_result* res,
                                    GpuEvolveState* out, uint32_t capacity) {
    if (!s || !res) return set_error_message(BH_INVALID_ARG, "null argument");
    std::unique_ptr<ServeRequest> taken;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->stopping) return set_error_message(BH_INVALID_ARG, "server stopped");
        ++s->pollers;
        // leaves the wait on a result, on the timeout, or when stop begins
        auto leave = [&](int status, const char* msg) {
            --s->pollers;
            s->cv_out.notify_all();
            return set_error_message(status, msg);
        };
        const bool ready = s->cv_out.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] {
            return !s->done.empty() || s->stopping;
        });
        if (s->stopping) return leave(BH_INVALID_ARG, "server stopped");
        if (!ready) return leave(BH_TIMEOUT, "no finished request within the timeout");
        const ServeRequest& r = *s->done.front();
        res->request_id = r.id;
        res->n = r.n;
        if (r.status == BH_OK && (!out || capacity < r.n))  // kept for a retry with room
            return leave(BH_INVALID_ARG, "result buffer smaller than the request");
        taken = std::move(s->done.front());
        s->done.pop_front();
        --s->pollers;
        s->cv_out.notify_all();
    }
    // the copy and the release of the records run without the server's lock
    const ServeRequest& r = *taken;
    res->status = (uint32_t)r.status;
    res->steps = r.steps;
    res->submitted_s = r.submitted_s;
    res->admitted_s = r.admitted_s;
    res->finished_s = r.finished_s;
    if (r.status == BH_OK) std::memcpy(out, r.records.data(), sizeof(GpuEvolveState) * r.n);
    return BH_OK;
}

extern "C" int galaxy_bh_serve_stats(bh_server* s, bh_serve_stats* out) {
    if (!s || !out) return set_error_message(BH_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out->rounds = s->rounds;
    out->particle_steps = s->particle_steps;
    out->completed = s->completed;
    out->busy_seconds = s->busy_s;
    out->elapsed_seconds = s->now();
    out->admit_seconds = s->admit_s;
    out->solve_seconds = s->solve_s;
    out->form_seconds = s->form_s;
    out->readback_seconds = s->readback_s;
    return BH_OK;
}

extern "C" int galaxy_bh_serve_stop(bh_server* s) {
    if (!s) return BH_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->cv_in.notify_all();
        s->cv_stage.notify_all();
        s->cv_out.notify_all();  // waiting polls return "server stopped"
    }
    if (s->stager.joinable()) s->stager.join();
    if (s->loop.joinable()) s->loop.join();
    for (auto& r : s->staged) release_state(r);  // dropped with the unfinished ones
    s->staged.clear();
    {
        // no poll may still be inside the server when it is freed
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_out.wait(lk, [&] { return s->pollers == 0; });
    }
    galaxy_bh_device_close(s->dev);
    galaxy_bh_device_close(s->dev2);
    delete s;
    return BH_OK;
}
