// Admission and scheduling policy of the serving loop (server.cu), as plain
// host C++ with no CUDA dependency: the worker threads of the server call it
// under their lock, and a host-only test drives it directly.
//
// State: a FIFO queue of requests ("new": create a diagram of W x H from a
// seed set; "insert": add seeds to a resident diagram), the diagrams (an
// opaque object handle each, its device bytes and allocation capacity, busy
// and pin counts), a pool of idle objects kept for reuse, and the bytes
// charged against the budget.
//
// Policy:
//   * requests are taken in queue order, but one that cannot run yet (its
//     diagram busy or not yet created, or its memory does not fit) is passed
//     over, not waited on;
//   * a new diagram takes the smallest pooled object it fits in (the rule of
//     idl_delaunay_reset: every allocation's size, not the sides) if that
//     object is at most twice its own footprint, else fresh budget, else
//     budget freed by retiring idle diagrams (least recently used first) into
//     the pool and, failing that, by dropping pooled objects, largest first;
//   * queued new diagrams that fit are grouped with the first (up to
//     GROUP_MAX, one 4128^2 atlas of padded canvases, MAX_REQUEST_SEEDS
//     seeds) so that one pass of the batched pipeline serves them all;
//   * a new diagram whose own footprint exceeds the budget fails at once;
//     one that does not fit while nothing is running (so nothing can free
//     memory) fails too, instead of waiting for good.
#pragma once

#include <algorithm>
#include <cstdint>
#include <deque>
#include <list>
#include <string>
#include <unordered_map>
#include <vector>

namespace idl {
namespace serve {

constexpr int GROUP_MAX = 16;               // new diagrams propagated in one launch, at most
constexpr int64_t SEED_HEADROOM = 50000;    // seed capacity beyond a new diagram's own seeds
constexpr int SIZE_CLASS = 128;             // object canvases are rounded up to multiples of this
constexpr int MAX_SIDE = 4096;              // largest request a worker's scratch is reserved for
constexpr int64_t MAX_REQUEST_SEEDS = 200000;

enum Kind { NEW = 0, INSERT = 1 };
enum Failure { FAIL_NONE = 0, FAIL_BUDGET = 1, FAIL_NOT_RESIDENT = 2 };

inline int class_dim(int v) { return (v + SIZE_CLASS - 1) / SIZE_CLASS * SIZE_CLASS; }

// Device allocations of an incremental object: label planes, padded raster
// and pixel outputs in bytes, and seed slots.
struct Capacity {
    int64_t planes = 0, raster = 0, pixels = 0, seeds = 0;
    bool fits(const Capacity& need) const
    {
        return need.planes <= planes && need.raster <= raster && need.pixels <= pixels && need.seeds <= seeds;
    }
    int64_t bytes() const { return planes + raster + pixels + seeds * 32; }
};

inline Capacity capacity(int W, int H, int64_t max_seeds, int P)
{
    const int64_t Wd = (int64_t)W + 2 * P, Hd = (int64_t)H + 2 * P;
    Capacity c;
    c.planes = (Wd + 31) / 32 * 32 * Hd * 8;
    c.raster = Wd * Hd * 4;
    c.pixels = (int64_t)W * H * 9;
    c.seeds = max_seeds;
    return c;
}

// Scratch a context grows to triangulate a canvas of Wd x Hd with `seeds`
// seeds: micro-tile lists and bitmaps, hash table, work lists, triangle rows.
inline int64_t scratch_bytes(int64_t Wd, int64_t Hd, int64_t seeds)
{
    const int64_t n_mt = ((Wd + 7) / 8) * ((Hd + 7) / 8);
    int64_t hash = 1024;
    while (hash < 8 * seeds + 1024) hash <<= 1;
    // hash table (32 B a slot) and the grouping and triangle rows sized by it
    // (24 B a slot); the tile rounds' three change bitmaps
    return n_mt * 8 + n_mt / 4 + 16 * (Wd + Hd) + 56 * hash + 48 * seeds + Wd * Hd / 8 +
           3 * ((Wd + 127) / 32 + 1) * 4 * Hd;
}

// Memory one worker slot holds at most: its diagram workspace, and its batch
// context triangulating a full group (one atlas of MAX_SIDE^2 padded, its
// label planes, raster and composed grids, seed arrays).
inline int64_t slot_reserve(int P)
{
    const int64_t Wd = MAX_SIDE + 2 * P, Hd = Wd;
    const int64_t pitch = (Wd + 31) / 32 * 32;
    const int64_t px = (int64_t)MAX_SIDE * MAX_SIDE;
    return 2 * scratch_bytes(Wd, Hd, MAX_REQUEST_SEEDS) + pitch * Hd * 8 + px * 16 + 32 * MAX_REQUEST_SEEDS;
}

struct Request {
    int64_t id = -1;
    int kind = NEW;
    int64_t diagram = -1;
    int W = 0, H = 0;                 // new: the canvas; insert: the diagram's, filled in at submit
    std::vector<int32_t> seeds;       // x, y pairs
    bool fetch = false;
    int32_t* grid_out = nullptr;
    int64_t need = 0;                 // new: bytes charged for a fresh object
    int64_t arrival_ns = 0;
    int64_t n_seeds() const { return (int64_t)seeds.size() / 2; }
};

// One request handed to a worker.  New: `obj` is the pooled object to reset
// (with `bytes` and `cap`), or null for a fresh one.  Insert: `obj` is the
// diagram's object and `base_seeds` its seed count before the request.
struct Item {
    Request req;
    void* obj = nullptr;
    int64_t bytes = 0;
    Capacity cap;
    int64_t base_seeds = 0;
};

struct Failed {
    Request req;
    int reason = FAIL_NONE;
};

struct Diagram {
    void* obj = nullptr;
    int64_t bytes = 0;
    Capacity cap;
    bool busy = false;
    int pins = 0;                     // queued or running requests
    int64_t last_used = 0;
    int64_t n_seeds = 0;
    int W = 0, H = 0;
};

struct Pooled {
    void* obj = nullptr;
    int64_t bytes = 0;
    Capacity cap;
};

enum Stat { ST_GROUPS, ST_GROUPED, ST_NEW_OBJECTS, ST_REUSED, ST_EVICTED, ST_FREED, ST_COUNT };

class Scheduler {
public:
    Scheduler(int64_t budget, int padding, int64_t reserved) : budget_(budget), P_(padding), used_(reserved) {}

    int padding() const { return P_; }
    int64_t budget() const { return budget_; }
    int64_t used() const { return used_; }
    int64_t stat(int k) const { return stats_[k]; }
    size_t queued() const { return queue_.size(); }
    size_t pooled() const { return pool_.size(); }
    const std::unordered_map<int64_t, Diagram>& diagrams() const { return diagrams_; }

    int64_t fresh_bytes(int W, int H, int64_t n) const
    {
        return capacity(class_dim(W), class_dim(H), n + SEED_HEADROOM, P_).bytes();
    }

    // Queue a new diagram; fills in id, diagram and need.
    void add_new(Request& r)
    {
        r.kind = NEW;
        r.id = next_id_++;
        r.diagram = next_diagram_++;
        r.need = fresh_bytes(r.W, r.H, r.n_seeds());
        Diagram d;
        d.pins = 1;
        d.W = r.W;
        d.H = r.H;
        diagrams_[r.diagram] = d;
        queue_.push_back(r);
    }

    // Queue an insert; false (nothing queued) if the diagram is not resident.
    bool add_insert(Request& r)
    {
        auto it = diagrams_.find(r.diagram);
        if (it == diagrams_.end()) return false;
        r.kind = INSERT;
        r.id = next_id_++;
        r.W = it->second.W;
        r.H = it->second.H;
        it->second.pins += 1;
        queue_.push_back(r);
        return true;
    }

    bool any_busy() const
    {
        for (auto& kv : diagrams_)
            if (kv.second.busy) return true;
        return false;
    }
    bool idle() const { return queue_.empty() && !any_busy(); }

    // Next work: a group of new diagrams or one insert, in `work` (true), or
    // nothing runnable now (false).  Requests that can never run go to
    // `failed`; objects to destroy (outside any lock) to `to_free`.
    bool next(std::vector<Item>& work, std::vector<Failed>& failed, std::vector<void*>& to_free)
    {
        work.clear();
        for (;;) {
            for (size_t i = 0; i < queue_.size(); ++i) {
                Request& r = queue_[i];
                auto dit = diagrams_.find(r.diagram);
                if (dit == diagrams_.end()) {       // target's creation failed
                    failed.push_back(Failed{r, FAIL_NOT_RESIDENT});
                    queue_.erase(queue_.begin() + i);
                    --i;
                    continue;
                }
                Diagram& d = dit->second;
                if (r.kind == NEW) {
                    if (r.need > budget_) {
                        failed.push_back(Failed{r, FAIL_BUDGET});
                        diagrams_.erase(dit);
                        queue_.erase(queue_.begin() + i);
                        --i;
                        continue;
                    }
                    Item it;
                    if (!place(r, it, to_free)) continue;
                    d.busy = true;
                    it.req = std::move(r);
                    queue_.erase(queue_.begin() + i);
                    work.push_back(std::move(it));
                    group_more(i, work, to_free);
                    return true;
                }
                if (d.busy || !d.obj) continue;     // running, or its creation has not run yet
                d.busy = true;
                Item it;
                it.obj = d.obj;
                it.base_seeds = d.n_seeds;
                it.req = std::move(r);
                queue_.erase(queue_.begin() + i);
                work.push_back(std::move(it));
                return true;
            }
            if (queue_.empty() || any_busy()) return false;
            // Nothing runs, so nothing can free memory: the first new
            // diagram that did not fit never will.
            bool dropped = false;
            for (size_t i = 0; i < queue_.size(); ++i)
                if (queue_[i].kind == NEW) {
                    failed.push_back(Failed{queue_[i], FAIL_BUDGET});
                    diagrams_.erase(queue_[i].diagram);
                    queue_.erase(queue_.begin() + i);
                    dropped = true;
                    break;
                }
            if (!dropped) return false;
        }
    }

    void count_group(int n)
    {
        stats_[ST_GROUPS] += 1;
        stats_[ST_GROUPED] += n;
    }

    // A new diagram ran.  ok: `obj` (with allocation `cap` and `dev_bytes`
    // on the device) is resident; returns null.  Otherwise the diagram is
    // dropped, its charge released, and `obj` returned for destruction.
    void* finish_new(const Item& it, bool ok, void* obj, const Capacity& cap, int64_t dev_bytes, int64_t now)
    {
        const int64_t charged = it.obj ? it.bytes : it.req.need;
        auto dit = diagrams_.find(it.req.diagram);
        if (!ok || dit == diagrams_.end()) {
            used_ -= charged;
            if (dit != diagrams_.end()) diagrams_.erase(dit);
            return obj;
        }
        Diagram& d = dit->second;
        const int64_t actual = std::max(dev_bytes, charged);
        d.obj = obj;
        d.bytes = actual;
        d.cap = cap;
        d.busy = false;
        d.pins -= 1;
        d.last_used = now;
        d.n_seeds = it.req.n_seeds();
        used_ += actual - charged;
        stats_[it.obj ? ST_REUSED : ST_NEW_OBJECTS] += 1;
        return nullptr;
    }

    // An insert ran; ok: the diagram now holds `n_seeds` seeds.
    void finish_insert(const Item& it, bool ok, int64_t n_seeds, int64_t now)
    {
        auto dit = diagrams_.find(it.req.diagram);
        if (dit == diagrams_.end()) return;
        dit->second.busy = false;
        dit->second.pins -= 1;
        dit->second.last_used = now;
        if (ok) dit->second.n_seeds = n_seeds;
    }

    // Retire an idle diagram now, keeping its object for reuse.
    bool recycle(int64_t diagram)
    {
        auto dit = diagrams_.find(diagram);
        if (dit == diagrams_.end() || dit->second.busy || dit->second.pins) return false;
        if (dit->second.obj) pool_.push_back(Pooled{dit->second.obj, dit->second.bytes, dit->second.cap});
        diagrams_.erase(dit);
        return true;
    }

    // Every object held (resident and pooled), for teardown.
    std::vector<void*> release_all()
    {
        std::vector<void*> out;
        for (auto& kv : diagrams_)
            if (kv.second.obj) out.push_back(kv.second.obj);
        for (auto& p : pool_) out.push_back(p.obj);
        diagrams_.clear();
        pool_.clear();
        return out;
    }

    // Test hooks: place an object directly (as a finished new diagram would).
    int64_t insert_resident(void* obj, int64_t bytes, const Capacity& cap, int W, int H, int64_t last_used)
    {
        const int64_t id = next_diagram_++;
        Diagram d;
        d.obj = obj;
        d.bytes = bytes;
        d.cap = cap;
        d.last_used = last_used;
        d.W = W;
        d.H = H;
        diagrams_[id] = d;
        used_ += bytes;
        return id;
    }
    void set_busy(int64_t diagram, bool busy) { diagrams_.at(diagram).busy = busy; }

private:
    bool take_pooled(const Request& r, const Capacity& need, Item& out)
    {
        auto best = pool_.end();
        for (auto it = pool_.begin(); it != pool_.end(); ++it)
            if (it->bytes <= 2 * r.need && it->cap.fits(need) && (best == pool_.end() || it->bytes < best->bytes))
                best = it;
        if (best == pool_.end()) return false;
        out.obj = best->obj;
        out.bytes = best->bytes;
        out.cap = best->cap;
        pool_.erase(best);
        return true;
    }

    bool place(const Request& r, Item& out, std::vector<void*>& to_free)
    {
        const Capacity need = capacity(r.W, r.H, r.n_seeds() + SEED_HEADROOM, P_);
        if (take_pooled(r, need, out)) return true;
        if (used_ + r.need <= budget_) {
            used_ += r.need;                    // charged now, corrected when the object exists
            return true;
        }
        std::vector<std::pair<int64_t, int64_t>> idle;   // (last used, diagram)
        for (auto& kv : diagrams_)
            if (kv.second.obj && !kv.second.busy && kv.second.pins == 0)
                idle.emplace_back(kv.second.last_used, kv.first);
        std::sort(idle.begin(), idle.end());
        for (auto& e : idle) {
            Diagram& d = diagrams_[e.second];
            pool_.push_back(Pooled{d.obj, d.bytes, d.cap});
            diagrams_.erase(e.second);
            stats_[ST_EVICTED] += 1;
            if (take_pooled(r, need, out)) return true;
        }
        pool_.sort([](const Pooled& a, const Pooled& b) { return a.bytes > b.bytes; });
        while (!pool_.empty() && used_ + r.need > budget_) {
            used_ -= pool_.front().bytes;
            to_free.push_back(pool_.front().obj);
            pool_.pop_front();
            stats_[ST_FREED] += 1;
        }
        if (used_ + r.need > budget_) return false;
        used_ += r.need;
        return true;
    }

    // Further queued new diagrams, from queue position `from`, for the launch
    // of work[0], while they fit the group limits and the budget.
    void group_more(size_t from, std::vector<Item>& work, std::vector<void*>& to_free)
    {
        auto padded = [&](const Request& q) { return (int64_t)(q.W + 2 * P_ + 1) * (q.H + 2 * P_ + 1); };
        int64_t area = padded(work[0].req), seeds = work[0].req.n_seeds();
        const int64_t limit = (int64_t)(MAX_SIDE + 2 * P_ + 1) * (MAX_SIDE + 2 * P_ + 1);
        for (size_t j = from; j < queue_.size() && (int)work.size() < GROUP_MAX;) {
            Request& q = queue_[j];
            if (q.kind != NEW || q.need > budget_ || area + padded(q) > limit ||
                seeds + q.n_seeds() > MAX_REQUEST_SEEDS) {
                ++j;
                continue;
            }
            Item it;
            if (!place(q, it, to_free)) break;
            diagrams_[q.diagram].busy = true;
            area += padded(q);
            seeds += q.n_seeds();
            it.req = std::move(q);
            queue_.erase(queue_.begin() + j);
            work.push_back(std::move(it));
        }
    }

    int64_t budget_;
    int P_;
    int64_t used_;
    std::deque<Request> queue_;
    std::unordered_map<int64_t, Diagram> diagrams_;
    std::list<Pooled> pool_;
    int64_t next_id_ = 0, next_diagram_ = 0;
    int64_t stats_[ST_COUNT] = {};
};

}  // namespace serve
}  // namespace idl
