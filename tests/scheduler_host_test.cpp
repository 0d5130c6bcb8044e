// Host-only checks of the serving loop's admission and scheduling policy
// (integer_delauney_b200/csrc/scheduler.h), driven without a GPU: object
// handles are fake pointers and "execution" is a call to finish_*.
// Built and run by tests/test_scheduler_host.py; exits non-zero on failure.
#include "scheduler.h"

#include <cstdio>
#include <cstdlib>

using namespace idl::serve;

static int failures = 0;
#define CHECK(cond)                                                              \
    do {                                                                         \
        if (!(cond)) {                                                           \
            std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                          \
        }                                                                        \
    } while (0)

static const int P = 16;

static Request new_req(int W = 200, int H = 150, int n = 100)
{
    Request r;
    r.W = W;
    r.H = H;
    r.seeds.assign(2 * (size_t)n, 0);
    return r;
}

static Request ins_req(int64_t diagram, int n = 1)
{
    Request r;
    r.diagram = diagram;
    r.seeds.assign(2 * (size_t)n, 0);
    return r;
}

static void* fake(int i) { return reinterpret_cast<void*>((uintptr_t)(0x1000 + 16 * i)); }

static void test_capacity_rules()
{
    CHECK(class_dim(1) == 128 && class_dim(129) == 256 && class_dim(128) == 128);
    CHECK(capacity(256, 256, 1000, 16).bytes() < capacity(512, 256, 1000, 16).bytes());
    CHECK(capacity(512, 256, 1000, 16).bytes() < capacity(512, 256, 100000, 16).bytes());
    CHECK(capacity(256, 256, 1000, 0).bytes() < capacity(256, 256, 1000, 16).bytes());
    // reuse is decided by the sizes of the allocations, not by the sides
    const Capacity c = capacity(512, 256, 1000, 16);
    CHECK(c.fits(capacity(256, 512, 1000, 16)) && c.fits(capacity(300, 300, 900, 16)));
    CHECK(!c.fits(capacity(600, 300, 1000, 16)) && !c.fits(capacity(256, 256, 1001, 16)));
    CHECK(slot_reserve(16) > capacity(4096, 4096, 0, 16).planes);
}

static void test_busy_diagram_is_passed_over()
{
    Scheduler s(1ll << 40, P, 0);
    const int64_t d7 = s.insert_resident(fake(7), 10, Capacity{}, 100, 100, 0);
    s.set_busy(d7, true);
    Request ins = ins_req(d7);
    CHECK(s.add_insert(ins));
    Request nw = new_req();
    s.add_new(nw);
    std::vector<Item> work;
    std::vector<Failed> failed;
    std::vector<void*> to_free;
    CHECK(s.next(work, failed, to_free));
    CHECK(work.size() == 1 && work[0].req.id == nw.id && work[0].req.kind == NEW);
    CHECK(s.queued() == 1 && failed.empty());
    // the insert runs once its diagram is free
    s.set_busy(d7, false);
    CHECK(s.next(work, failed, to_free));
    CHECK(work.size() == 1 && work[0].req.id == ins.id && work[0].obj == fake(7));
    CHECK(work[0].req.W == 100 && work[0].req.H == 100);
}

static void test_insert_waits_for_its_diagram_creation()
{
    Scheduler s(1ll << 40, P, 0);
    Request nw = new_req(300, 200, 500);
    s.add_new(nw);
    Request ins = ins_req(nw.diagram, 20);
    CHECK(s.add_insert(ins));
    std::vector<Item> work;
    std::vector<Failed> failed;
    std::vector<void*> to_free;
    CHECK(s.next(work, failed, to_free) && work.size() == 1 && work[0].req.id == nw.id);
    Item created = work[0];
    std::vector<Item> none;
    CHECK(!s.next(none, failed, to_free));          // the diagram is being created
    const Capacity cap = capacity(384, 256, 500 + SEED_HEADROOM, P);
    CHECK(s.finish_new(created, true, fake(1), cap, created.req.need, 5) == nullptr);
    CHECK(s.next(work, failed, to_free) && work[0].req.id == ins.id && work[0].obj == fake(1));
    CHECK(work[0].base_seeds == 500);
    s.finish_insert(work[0], true, 520, 6);
    CHECK(s.diagrams().at(nw.diagram).n_seeds == 520 && s.idle());
    CHECK(s.stat(ST_NEW_OBJECTS) == 1);
}

static void test_idle_diagram_evicted_and_its_object_reused()
{
    const int64_t need = capacity(256, 256, 100 + SEED_HEADROOM, P).bytes();
    Scheduler s(need + need / 2, P, 0);
    const int64_t old = s.insert_resident(fake(1), need, capacity(256, 256, 100 + SEED_HEADROOM, P), 256, 256, 1);
    Request nw = new_req(200, 150, 100);
    s.add_new(nw);
    std::vector<Item> work;
    std::vector<Failed> failed;
    std::vector<void*> to_free;
    CHECK(s.next(work, failed, to_free));
    CHECK(work.size() == 1 && work[0].obj == fake(1) && work[0].bytes == need);
    CHECK(s.stat(ST_EVICTED) == 1 && s.diagrams().count(old) == 0 && to_free.empty());
    CHECK(s.used() == need);                          // the reused object's bytes, charged once
    CHECK(s.finish_new(work[0], true, work[0].obj, work[0].cap, need, 2) == nullptr);
    CHECK(s.stat(ST_REUSED) == 1 && s.used() == need);
}

static void test_least_recently_used_goes_first()
{
    const Capacity cap = capacity(256, 256, 100 + SEED_HEADROOM, P);
    Scheduler s(2 * cap.bytes() + cap.bytes() / 2, P, 0);
    const int64_t a = s.insert_resident(fake(1), cap.bytes(), cap, 256, 256, 20);   // used later
    const int64_t b = s.insert_resident(fake(2), cap.bytes(), cap, 256, 256, 10);   // used earlier
    Request nw = new_req(256, 256, 100);
    s.add_new(nw);
    std::vector<Item> work;
    std::vector<Failed> failed;
    std::vector<void*> to_free;
    CHECK(s.next(work, failed, to_free) && work[0].obj == fake(2));
    CHECK(s.diagrams().count(a) == 1 && s.diagrams().count(b) == 0);
}

static void test_pool_dropped_when_nothing_fits()
{
    const Capacity small = capacity(128, 128, 100 + SEED_HEADROOM, P);
    const int64_t need = capacity(1024, 1024, 100 + SEED_HEADROOM, P).bytes();
    Scheduler s(need + small.bytes() / 2, P, 0);
    const int64_t d = s.insert_resident(fake(3), small.bytes(), small, 128, 128, 0);
    CHECK(s.recycle(d));                              // idle: into the pool
    CHECK(s.pooled() == 1);
    Request nw = new_req(1000, 1000, 100);
    s.add_new(nw);
    std::vector<Item> work;
    std::vector<Failed> failed;
    std::vector<void*> to_free;
    CHECK(s.next(work, failed, to_free));
    CHECK(work[0].obj == nullptr && to_free.size() == 1 && to_free[0] == fake(3));
    CHECK(s.stat(ST_FREED) == 1 && s.pooled() == 0 && s.used() == need);
}

static void test_failures()
{
    const int64_t need = capacity(256, 256, 100 + SEED_HEADROOM, P).bytes();
    Scheduler s(need / 2, P, 0);
    Request big = new_req(200, 200, 100);            // can never fit
    s.add_new(big);
    Request none = ins_req(12345);
    CHECK(!s.add_insert(none));                       // unknown diagram: nothing queued
    std::vector<Item> work;
    std::vector<Failed> failed;
    std::vector<void*> to_free;
    CHECK(!s.next(work, failed, to_free));
    CHECK(failed.size() == 1 && failed[0].req.id == big.id && failed[0].reason == FAIL_BUDGET);
    CHECK(s.diagrams().empty() && s.queued() == 0);
    // an insert queued behind a creation that fails
    Scheduler t(1ll << 40, P, 0);
    Request nw = new_req();
    t.add_new(nw);
    Request ins = ins_req(nw.diagram);
    CHECK(t.add_insert(ins));
    failed.clear();
    CHECK(t.next(work, failed, to_free));
    const int64_t used_before = t.used();
    CHECK(t.finish_new(work[0], false, fake(9), Capacity{}, 0, 1) == fake(9));   // returned for destruction
    CHECK(t.used() == used_before - nw.need);
    CHECK(!t.next(work, failed, to_free));
    CHECK(failed.size() == 1 && failed[0].req.id == ins.id && failed[0].reason == FAIL_NOT_RESIDENT);
}

static void test_queued_new_diagrams_share_one_group()
{
    Scheduler s(1ll << 40, P, 0);
    std::vector<int64_t> ids;
    for (int i = 0; i < 20; ++i) {
        Request r = new_req(100 + i, 100, 50);
        s.add_new(r);
        ids.push_back(r.id);
    }
    Request ins = ins_req(0);
    CHECK(s.add_insert(ins));
    std::vector<Item> work;
    std::vector<Failed> failed;
    std::vector<void*> to_free;
    CHECK(s.next(work, failed, to_free));
    CHECK((int)work.size() == GROUP_MAX);
    for (int i = 0; i < GROUP_MAX; ++i) CHECK(work[i].req.id == ids[i]);
    CHECK(s.next(work, failed, to_free) && work.size() == 4);   // the rest, the insert still waits
    // two full-size canvases do not share one atlas
    Scheduler t(1ll << 40, P, 0);
    Request a = new_req(4096, 4096, 10), b = new_req(4096, 4096, 10);
    t.add_new(a);
    t.add_new(b);
    CHECK(t.next(work, failed, to_free) && work.size() == 1);
    // nor do groups exceed the seed limit
    Scheduler u(1ll << 40, P, 0);
    Request c = new_req(1000, 1000, 150000), d = new_req(1000, 1000, 60000), e = new_req(100, 100, 10);
    u.add_new(c);
    u.add_new(d);
    u.add_new(e);
    CHECK(u.next(work, failed, to_free) && work.size() == 2 && work[1].req.id == e.id);
}

static void test_waits_while_something_runs_fails_when_nothing_does()
{
    const int64_t need = capacity(256, 256, 100 + SEED_HEADROOM, P).bytes();
    Scheduler s(need + need / 2, P, 0);
    Request a = new_req(256, 256, 100), b = new_req(256, 256, 100);
    s.add_new(a);
    std::vector<Item> work;
    std::vector<Failed> failed;
    std::vector<void*> to_free;
    CHECK(s.next(work, failed, to_free) && work.size() == 1);
    Item running = work[0];
    s.add_new(b);
    CHECK(!s.next(work, failed, to_free) && failed.empty());   // a is running: b waits
    CHECK(s.finish_new(running, true, fake(1), capacity(256, 256, 100 + SEED_HEADROOM, P), need, 3) == nullptr);
    CHECK(s.next(work, failed, to_free) && work[0].req.id == b.id && work[0].obj == fake(1));
    // reserved workspace leaves no room and nothing runs: fails instead of waiting
    Scheduler t(need + need / 2, P, need);
    Request c = new_req(256, 256, 100);
    t.add_new(c);
    CHECK(!t.next(work, failed, to_free) && failed.size() == 1 && failed[0].reason == FAIL_BUDGET);
}

int main()
{
    test_capacity_rules();
    test_busy_diagram_is_passed_over();
    test_insert_waits_for_its_diagram_creation();
    test_idle_diagram_evicted_and_its_object_reused();
    test_least_recently_used_goes_first();
    test_pool_dropped_when_nothing_fits();
    test_failures();
    test_queued_new_diagrams_share_one_group();
    test_waits_while_something_runs_fails_when_nothing_does();
    if (failures) {
        std::fprintf(stderr, "%d checks failed\n", failures);
        return 1;
    }
    // the figures the Python layer mirrors (serving.slot_reserve, estimate_bytes(workspace=False))
    std::printf("slot_reserve %d %lld\n", 16, (long long)slot_reserve(16));
    std::printf("slot_reserve %d %lld\n", 0, (long long)slot_reserve(0));
    std::printf("fresh %d %d %lld %d %lld\n", 300, 200, 5000LL, 16, (long long)capacity(300, 200, 5000, 16).bytes());
    std::printf("fresh %d %d %lld %d %lld\n", 4096, 17, 1LL, 0, (long long)capacity(4096, 17, 1, 0).bytes());
    std::printf("scheduler: all checks passed\n");
    return 0;
}
