// The serving loop: a native request loop over diagrams kept resident on one
// GPU.  No counterpart in the reference, which triangulates one caller's
// image per call; this is the form a service wraps around its incremental
// object (Delaunay, src/cuda/delaunay.cu) when many clients share a device.
//
// `slots` worker threads each own a CUDA stream, a workspace context that
// every diagram the slot runs shares (idl_delaunay_set_workspace) and a batch
// context.  Scheduling and memory admission are the policy of scheduler.h,
// run under the server's lock; a worker executes what it is handed:
//   * a group of new diagrams (reference mode): one pass of the batched
//     pipeline (idl_triangulate_batch's) triangulates all of them; each
//     object is reset and takes its image's labels (idl_delaunay_adopt) --
//     bit for bit the state an (x, y)-ordered insert reaches -- and the
//     request's result (triangle count; with `fetch`, the grid and triangle
//     rows) comes from the batch, whose per-image results equal the
//     single-image pipeline's; the object's own topology follows lazily.  If
//     the batch rejects the group, each request runs on its own
//     (idl_delaunay_insert_ordered) so that only the bad one fails;
//   * an insert (or a new diagram in exact mode): idl_delaunay_insert_ordered
//     into the object, then finalise (with `fetch`, into the caller's host
//     grid, triangles kept for idl_server_wait);
// and synchronises its stream, so a result is complete when it is reported.
// All of it is C++: a request costs a Python caller one call to submit and
// one to collect.
#include "context.cuh"
#include "scheduler.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using namespace idl::serve;

int64_t clock_ns()
{
    return std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Outcome {
    bool done = false;
    int status = IDL_OK;
    std::string error;
    int kind = NEW;
    int64_t diagram = -1, n_seeds = 0, n_triangles = 0, arrival_ns = 0, start_ns = 0, done_ns = 0;
    std::vector<int32_t> tris;   // 5 int32 per triangle, when fetched
};

struct Slot {
    cudaStream_t stream = nullptr;
    idl_context* ws = nullptr;
    idl_context* batch = nullptr;
};

void check_status(int st)
{
    if (st != IDL_OK) throw idl::Error(st, idl_last_error());
}

}  // namespace

struct idl_server {
    int device = 0;
    int mode = IDL_MODE_REFERENCE;
    Scheduler sched;
    std::mutex mu;
    std::condition_variable work_cv, done_cv;
    std::unordered_map<int64_t, Outcome> outcomes;
    std::vector<Slot> slots;
    std::vector<std::thread> workers;
    int running = 0;   // workers executing a work list
    bool closing = false;
    bool submitted = false;

    idl_server(int64_t budget, int P, int n_slots) : sched(budget, P, (int64_t)n_slots * slot_reserve(P)) {}
};

namespace {

void deliver_failures(idl_server& S, std::vector<Failed>& failed)
{
    for (auto& f : failed) {
        Outcome& o = S.outcomes[f.req.id];
        o.done = true;
        o.kind = f.req.kind;
        o.diagram = f.req.diagram;
        o.arrival_ns = f.req.arrival_ns;
        o.done_ns = clock_ns();
        if (f.reason == FAIL_BUDGET) {
            o.status = IDL_ERR_BUDGET;
            o.error = "request needs " + std::to_string(f.req.need) + " bytes; the budget of " +
                      std::to_string(S.sched.budget()) + " bytes cannot hold it" +
                      (f.req.need > S.sched.budget() ? "" : " with nothing left to evict");
        } else {
            o.status = IDL_ERR_NOT_RESIDENT;
            o.error = "diagram " + std::to_string(f.req.diagram) + " is not resident";
        }
    }
    if (!failed.empty()) S.done_cv.notify_all();
    failed.clear();
}

// One request on the slot's stream; the outcome's status says how it ended.
// `batch_tris` >= 0: a new diagram that is image `image` of the batch just
// triangulated on the slot's batch context, with that many triangles -- the
// object adopts its labels and the result (and fetched grid and rows) comes
// from the batch; the object's own topology follows lazily when an insert
// needs it.  For a new diagram, obj_out receives the object used (fresh or
// pooled, or null if none could be created) and cap_out / dev_bytes its
// allocations.
void execute(idl_server& S, Slot& slot, const Item& it, int64_t batch_tris, int image, int64_t start, Outcome& o,
             void*& obj_out, Capacity& cap_out, int64_t& dev_bytes)
{
    const bool adopt = batch_tris >= 0;
    const Request& r = it.req;
    const int P = S.sched.padding();
    idl_delaunay* obj = static_cast<idl_delaunay*>(it.obj);
    o.kind = r.kind;
    o.diagram = r.diagram;
    o.arrival_ns = r.arrival_ns;
    o.start_ns = start;
    try {
        const int64_t n = r.n_seeds();
        const int32_t* xy = n ? r.seeds.data() : nullptr;
        if (r.kind == NEW) {
            const int64_t ms = n + SEED_HEADROOM;
            if (obj) {
                cap_out = it.cap;
            } else {
                const int Wc = class_dim(r.W), Hc = class_dim(r.H);
                check_status(idl_delaunay_create(S.device, Wc, Hc, ms, P, S.mode, &obj));
                cap_out = capacity(Wc, Hc, ms, P);
            }
            obj_out = obj;
            check_status(idl_delaunay_set_stream(obj, slot.stream));
            check_status(idl_delaunay_set_workspace(obj, slot.ws));
            check_status(idl_delaunay_reset(obj, r.W, r.H, ms, P));
            if (adopt) check_status(idl_delaunay_adopt(obj, slot.batch, image));
            else check_status(idl_delaunay_insert_ordered(obj, xy, n, nullptr, 1, nullptr));
            o.n_seeds = n;
        } else {
            check_status(idl_delaunay_set_stream(obj, slot.stream));
            check_status(idl_delaunay_set_workspace(obj, slot.ws));
            check_status(idl_delaunay_insert_ordered(obj, xy, n, nullptr, 0, nullptr));
            o.n_seeds = it.base_seeds + n;
        }
        if (adopt) {
            o.n_triangles = batch_tris;
            if (r.fetch) {
                o.tris.resize((size_t)batch_tris * 5);
                idl::batch_fetch(*slot.batch, image, r.grid_out, o.tris.data(), (int64_t)o.tris.size());
            }
        } else if (r.fetch) {
            check_status(idl_delaunay_finalise(obj, r.grid_out, &o.n_triangles, nullptr));
            o.tris.resize((size_t)o.n_triangles * 5);
            int64_t got = 0;
            check_status(idl_delaunay_triangles(obj, 0, o.tris.data(), (int64_t)o.tris.size(), &got));
        } else {
            check_status(idl_delaunay_finalise_device(obj, &o.n_triangles, nullptr, nullptr, nullptr, nullptr));
        }
        IDL_CUDA(cudaStreamSynchronize(slot.stream));
        if (r.kind == NEW) {
            int64_t info[IDL_DI_COUNT];
            check_status(idl_delaunay_info(obj, info, IDL_DI_COUNT));
            dev_bytes = info[IDL_DI_DEVICE_BYTES];
        }
        o.status = IDL_OK;
    } catch (const idl::Error& e) {
        o.status = e.status;
        o.error = e.what();
    } catch (const std::exception& e) {
        o.status = IDL_ERR_INTERNAL;
        o.error = e.what();
    }
    o.done_ns = clock_ns();
    o.done = true;
}

// A group of new diagrams whose batch succeeded: every object is made ready
// (fresh or pooled, reset to its canvas), then all adopt their images at once
// (idl_delaunay_adopt_group: one launch, one wait), and the fetched results
// are copied from the batch with one more wait for the whole group.  A
// request whose object cannot be made ready fails alone.
void execute_group(idl_server& S, Slot& slot, const std::vector<Item>& work, const std::vector<int64_t>& batch_tris,
                   int64_t start, std::vector<Outcome>& outs, std::vector<void*>& objs, std::vector<Capacity>& caps,
                   std::vector<int64_t>& dev_bytes)
{
    const int P = S.sched.padding();
    std::vector<idl_delaunay*> ready;
    std::vector<int> images;
    for (size_t k = 0; k < work.size(); ++k) {
        const Request& r = work[k].req;
        Outcome& o = outs[k];
        o.kind = r.kind;
        o.diagram = r.diagram;
        o.arrival_ns = r.arrival_ns;
        o.start_ns = start;
        idl_delaunay* obj = static_cast<idl_delaunay*>(work[k].obj);
        try {
            const int64_t ms = r.n_seeds() + SEED_HEADROOM;
            if (obj) {
                caps[k] = work[k].cap;
            } else {
                const int Wc = class_dim(r.W), Hc = class_dim(r.H);
                check_status(idl_delaunay_create(S.device, Wc, Hc, ms, P, S.mode, &obj));
                caps[k] = capacity(Wc, Hc, ms, P);
            }
            objs[k] = obj;
            check_status(idl_delaunay_set_stream(obj, slot.stream));
            check_status(idl_delaunay_set_workspace(obj, slot.ws));
            check_status(idl_delaunay_reset(obj, r.W, r.H, ms, P));
            o.n_seeds = r.n_seeds();
            ready.push_back(obj);
            images.push_back((int)k);
        } catch (const idl::Error& e) {
            o.status = e.status;
            o.error = e.what();
            o.done_ns = clock_ns();
            o.done = true;
        } catch (const std::exception& e) {
            o.status = IDL_ERR_INTERNAL;
            o.error = e.what();
            o.done_ns = clock_ns();
            o.done = true;
        }
    }
    if (ready.empty()) return;
    int status = IDL_OK;
    std::string error;
    try {
        check_status(idl_delaunay_adopt_group(ready.data(), images.data(), (int)ready.size(), slot.batch));
        for (int k : images) {
            outs[k].n_triangles = batch_tris[k];
            if (work[k].req.fetch) {
                outs[k].tris.resize((size_t)batch_tris[k] * 5);
                idl::batch_fetch(*slot.batch, k, work[k].req.grid_out, outs[k].tris.data(),
                                 (int64_t)outs[k].tris.size());
            }
        }
        IDL_CUDA(cudaStreamSynchronize(slot.stream));
        for (size_t j = 0; j < ready.size(); ++j) {
            int64_t info[IDL_DI_COUNT];
            check_status(idl_delaunay_info(ready[j], info, IDL_DI_COUNT));
            dev_bytes[images[j]] = info[IDL_DI_DEVICE_BYTES];
        }
    } catch (const idl::Error& e) {
        status = e.status;
        error = e.what();
    } catch (const std::exception& e) {
        status = IDL_ERR_INTERNAL;
        error = e.what();
    }
    const int64_t done = clock_ns();
    for (int k : images) {
        outs[k].status = status;
        outs[k].error = error;
        outs[k].done_ns = done;
        outs[k].done = true;
    }
}

void destroy_all(std::vector<void*>& objs)
{
    for (void* p : objs) idl_delaunay_destroy(static_cast<idl_delaunay*>(p));
    objs.clear();
}

void worker_loop(idl_server* Sp, int index)
{
    idl_server& S = *Sp;
    Slot& slot = S.slots[index];
    cudaSetDevice(S.device);
    std::vector<Item> work;
    std::vector<Failed> failed;
    std::vector<void*> to_free;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S.mu);
            for (;;) {
                const bool got = S.sched.next(work, failed, to_free);
                deliver_failures(S, failed);
                if (got) break;
                if (!to_free.empty()) {
                    lk.unlock();
                    destroy_all(to_free);
                    lk.lock();
                    continue;
                }
                if (S.closing && S.sched.queued() == 0) return;
                S.done_cv.notify_all();   // a drain may be waiting for this state
                S.work_cv.wait(lk);
            }
            ++S.running;
        }
        destroy_all(to_free);
        const int64_t start = clock_ns();
        // a group of new diagrams: one pass of the batched pipeline for all
        // of them; if it rejects the group (a request's bad seeds), each runs
        // on its own so that only the bad one fails
        std::vector<int64_t> batch_tris(work.size(), -1);
        if (work[0].req.kind == NEW && S.mode == IDL_MODE_REFERENCE) {
            std::vector<int32_t> dims, seeds;
            std::vector<int64_t> counts;
            for (auto& it : work) {
                dims.push_back(it.req.W);
                dims.push_back(it.req.H);
                counts.push_back(it.req.n_seeds());
                seeds.insert(seeds.end(), it.req.seeds.begin(), it.req.seeds.end());
            }
            try {
                idl::triangulate_batch_keep(*slot.batch, (int)work.size(), dims.data(), counts.data(),
                                            seeds.empty() ? nullptr : seeds.data(), S.sched.padding(),
                                            batch_tris.data());
            } catch (const std::exception&) {
                std::fill(batch_tris.begin(), batch_tris.end(), -1);
            }
            std::lock_guard<std::mutex> lk(S.mu);
            S.sched.count_group((int)work.size());
        }
        // a whole group that the batch took: adopt all of its images at once
        const bool grouped = work[0].req.kind == NEW && S.mode == IDL_MODE_REFERENCE &&
                             std::all_of(batch_tris.begin(), batch_tris.end(), [](int64_t t) { return t >= 0; });
        std::vector<Outcome> outs(grouped ? work.size() : 0);
        std::vector<void*> g_objs(outs.size(), nullptr);
        std::vector<Capacity> g_caps(outs.size());
        std::vector<int64_t> g_bytes(outs.size(), 0);
        if (grouped) execute_group(S, slot, work, batch_tris, start, outs, g_objs, g_caps, g_bytes);
        for (size_t k = 0; k < work.size(); ++k) {
            const Item& it = work[k];
            Outcome o;
            void* obj = nullptr;
            Capacity cap;
            int64_t dev_bytes = 0;
            if (grouped) {
                o = std::move(outs[k]);
                obj = g_objs[k];
                cap = g_caps[k];
                dev_bytes = g_bytes[k];
            } else {
                execute(S, slot, it, batch_tris[k], (int)k, start, o, obj, cap, dev_bytes);
            }
            void* drop = nullptr;
            {
                std::lock_guard<std::mutex> lk(S.mu);
                if (it.req.kind == NEW)
                    drop = S.sched.finish_new(it, o.status == IDL_OK, obj, cap, dev_bytes, o.done_ns);
                else
                    S.sched.finish_insert(it, o.status == IDL_OK, o.n_seeds, o.done_ns);
                S.outcomes[it.req.id] = std::move(o);
            }
            if (drop) idl_delaunay_destroy(static_cast<idl_delaunay*>(drop));
            S.done_cv.notify_all();
            S.work_cv.notify_all();
        }
        std::lock_guard<std::mutex> lk(S.mu);
        --S.running;
        S.done_cv.notify_all();
    }
}

void check_server(const idl_server* s)
{
    if (!s) idl::invalid("server handle must not be NULL");
}

void take_seeds(const int32_t* xy, int64_t n, Request& r)
{
    if (n < 0) idl::invalid("seed count must not be negative");
    if (n > MAX_REQUEST_SEEDS)
        idl::invalid("a request holds at most " + std::to_string(MAX_REQUEST_SEEDS) + " seeds");
    if (n > 0 && !xy) idl::invalid("seeds must not be NULL");
    r.seeds.assign(xy, xy + 2 * n);
}

void release_slots(idl_server* s)
{
    for (auto& sl : s->slots) {
        if (sl.ws) idl_context_destroy(sl.ws);
        if (sl.batch) idl_context_destroy(sl.batch);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    s->slots.clear();
}

}  // namespace

extern "C" {

int64_t idl_server_clock_ns(void) { return clock_ns(); }

int idl_server_create(int device, int64_t budget_bytes, int slots, int border_padding, int mode, idl_server** out)
{
    IDL_API_BEGIN
    if (!out) idl::invalid("out must not be NULL");
    *out = nullptr;
    if (slots < 1 || slots > 64) idl::invalid("slots must lie in [1, 64]");
    if (budget_bytes <= 0) idl::invalid("budget_bytes must be positive");
    if (mode != IDL_MODE_REFERENCE && mode != IDL_MODE_EXACT)
        idl::invalid("a server runs in IDL_MODE_REFERENCE or IDL_MODE_EXACT");
    int dev = device;
    if (dev < 0) IDL_CUDA(cudaGetDevice(&dev));
    const int P = border_padding >= 0 ? border_padding : IDL_DEFAULT_BORDER_PADDING;
    idl::DeviceGuard g(dev);
    auto* s = new idl_server(budget_bytes, P, slots);
    s->device = dev;
    s->mode = mode;
    try {
        s->slots.resize(slots);
        for (auto& sl : s->slots) {
            IDL_CUDA(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
            check_status(idl_context_create(dev, &sl.ws));
            check_status(idl_context_create(dev, &sl.batch));
            check_status(idl_context_set_stream(sl.ws, sl.stream));
            check_status(idl_context_set_stream(sl.batch, sl.stream));
            // workers overlap: tile rounds as plain launches, not a device-filling grid
            sl.ws->persistent_rounds = false;
            sl.batch->persistent_rounds = false;
            // inserts as tile rounds: plain launches that overlap the other
            // workers' work, where the persistent kernel would hold the whole
            // device (measured: twice the insert throughput with 8 workers)
            check_status(idl_context_set_schedule(sl.ws, -1));
            // grouped new diagrams likewise, as cell-list tile rounds (48 x 48
            // tiles, 8 passes per round) to convergence: measured 3 329 req/s
            // on the saturated stream against 2 853 with one tile round and
            // the persistent kernel for the tail
            check_status(idl_context_set_schedule(sl.batch, -1));
            check_status(idl_context_set_tile(sl.batch, 8, nullptr));
        }
        for (int i = 0; i < slots; ++i) s->workers.emplace_back(worker_loop, s, i);
    } catch (...) {
        release_slots(s);
        delete s;
        throw;
    }
    *out = s;
    IDL_API_END
}

int idl_server_set_schedule(idl_server* s, int group_rounds, int insert_rounds)
{
    IDL_API_BEGIN
    check_server(s);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->submitted) throw idl::Error(IDL_ERR_STATE, "the schedule is set before the first request");
    for (auto& sl : s->slots) {
        check_status(idl_context_set_schedule(sl.batch, group_rounds));
        check_status(idl_context_set_schedule(sl.ws, insert_rounds));
    }
    IDL_API_END
}

int idl_server_set_tile(idl_server* s, int shape)
{
    IDL_API_BEGIN
    check_server(s);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->submitted) throw idl::Error(IDL_ERR_STATE, "the tile shape is set before the first request");
    for (auto& sl : s->slots) check_status(idl_context_set_tile(sl.batch, shape, nullptr));
    IDL_API_END
}

int idl_server_destroy(idl_server* s)
{
    IDL_API_BEGIN
    if (!s) return IDL_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->closing = true;
    }
    s->work_cv.notify_all();
    for (auto& t : s->workers) t.join();
    idl::DeviceGuard g(s->device);
    std::vector<void*> objs = s->sched.release_all();
    destroy_all(objs);
    release_slots(s);
    delete s;
    IDL_API_END
}

int idl_server_submit_new(idl_server* s, int width, int height, const int32_t* seeds_xy, int64_t n, int fetch,
                          int32_t* grid_out, int64_t arrival_ns, int64_t* request_out, int64_t* diagram_out)
{
    IDL_API_BEGIN
    check_server(s);
    if (width <= 0 || height <= 0 || width > MAX_SIDE || height > MAX_SIDE)
        idl::invalid("dimensions must lie in [1, " + std::to_string(MAX_SIDE) + "]");
    if (fetch && !grid_out) idl::invalid("fetch needs grid_out");
    Request r;
    take_seeds(seeds_xy, n, r);
    r.W = width;
    r.H = height;
    r.fetch = fetch != 0;
    r.grid_out = fetch ? grid_out : nullptr;
    r.arrival_ns = arrival_ns > 0 ? arrival_ns : clock_ns();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->closing) throw idl::Error(IDL_ERR_STATE, "server is closing");
        s->sched.add_new(r);
        s->submitted = true;
        s->outcomes[r.id] = Outcome{};
        if (request_out) *request_out = r.id;
        if (diagram_out) *diagram_out = r.diagram;
    }
    s->work_cv.notify_one();
    IDL_API_END
}

int idl_server_submit_insert(idl_server* s, int64_t diagram, const int32_t* seeds_xy, int64_t n, int fetch,
                             int32_t* grid_out, int64_t arrival_ns, int64_t* request_out)
{
    IDL_API_BEGIN
    check_server(s);
    if (fetch && !grid_out) idl::invalid("fetch needs grid_out");
    Request r;
    take_seeds(seeds_xy, n, r);
    r.diagram = diagram;
    r.fetch = fetch != 0;
    r.grid_out = fetch ? grid_out : nullptr;
    r.arrival_ns = arrival_ns > 0 ? arrival_ns : clock_ns();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->closing) throw idl::Error(IDL_ERR_STATE, "server is closing");
        if (!s->sched.add_insert(r))
            throw idl::Error(IDL_ERR_NOT_RESIDENT, "diagram " + std::to_string(diagram) + " is not resident");
        s->outcomes[r.id] = Outcome{};
        if (request_out) *request_out = r.id;
    }
    s->work_cv.notify_one();
    IDL_API_END
}

int idl_server_wait(idl_server* s, int64_t request, double timeout_s, int64_t* result_out, int32_t* tris_out,
                    int64_t capacity)
{
    IDL_API_BEGIN
    check_server(s);
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->outcomes.find(request) == s->outcomes.end())
        idl::invalid("request " + std::to_string(request) + " is unknown or already collected");
    auto ready = [&] {   // done, or collected meanwhile by another thread
        auto f = s->outcomes.find(request);
        return f == s->outcomes.end() || f->second.done;
    };
    if (timeout_s < 0) s->done_cv.wait(lk, ready);
    else if (!s->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
        throw idl::Error(IDL_ERR_STATE, "request " + std::to_string(request) + " not finished within the timeout");
    auto found = s->outcomes.find(request);
    if (found == s->outcomes.end()) idl::invalid("request " + std::to_string(request) + " was already collected");
    Outcome& o = found->second;
    if (result_out) {
        const int64_t v[IDL_SR_COUNT] = {o.status,      o.kind,       o.diagram,  o.n_seeds,
                                         o.n_triangles, o.arrival_ns, o.start_ns, o.done_ns};
        for (int i = 0; i < IDL_SR_COUNT; ++i) result_out[i] = v[i];
    }
    if (tris_out && !o.tris.empty()) {
        if (capacity < (int64_t)o.tris.size())   // the outcome stays, for a retry with room
            idl::invalid("triangle buffer holds " + std::to_string(capacity) + " int32, " +
                         std::to_string(o.tris.size()) + " needed");
        std::copy(o.tris.begin(), o.tris.end(), tris_out);
    }
    const int status = o.status;
    const std::string error = o.error;
    s->outcomes.erase(request);
    lk.unlock();
    if (status != IDL_OK) throw idl::Error(status, error);
    IDL_API_END
}

int idl_server_drain(idl_server* s)
{
    IDL_API_BEGIN
    check_server(s);
    std::unique_lock<std::mutex> lk(s->mu);
    s->done_cv.wait(lk, [&] { return s->sched.queued() == 0 && s->running == 0; });
    IDL_API_END
}

int idl_server_recycle(idl_server* s, int64_t diagram, int* recycled_out)
{
    IDL_API_BEGIN
    check_server(s);
    std::lock_guard<std::mutex> lk(s->mu);
    const bool ok = s->sched.recycle(diagram);
    if (recycled_out) *recycled_out = ok;
    IDL_API_END
}

int idl_server_info(idl_server* s, int64_t* info_out, int count)
{
    IDL_API_BEGIN
    check_server(s);
    if (!info_out) idl::invalid("info_out must not be NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    int64_t resident = 0;
    for (auto& kv : s->sched.diagrams()) resident += kv.second.obj != nullptr;
    const int64_t v[IDL_SI_COUNT] = {s->sched.used(),          s->sched.budget(),        resident,
                                     (int64_t)s->sched.pooled(), (int64_t)s->sched.queued(), s->sched.stat(ST_GROUPS),
                                     s->sched.stat(ST_GROUPED), s->sched.stat(ST_NEW_OBJECTS), s->sched.stat(ST_REUSED),
                                     s->sched.stat(ST_EVICTED), s->sched.stat(ST_FREED)};
    for (int i = 0; i < count && i < IDL_SI_COUNT; ++i) info_out[i] = v[i];
    IDL_API_END
}

int idl_server_resident(idl_server* s, int64_t* ids_out, int64_t capacity, int64_t* n_out)
{
    IDL_API_BEGIN
    check_server(s);
    std::lock_guard<std::mutex> lk(s->mu);
    int64_t n = 0;
    for (auto& kv : s->sched.diagrams()) {
        if (!kv.second.obj && kv.second.pins == 0) continue;
        if (ids_out && n < capacity) ids_out[n] = kv.first;
        ++n;
    }
    if (n_out) *n_out = n;
    IDL_API_END
}

}  // extern "C"
