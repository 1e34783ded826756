// The serving loop's bookkeeping (loom_b200/csrc/request_book.hpp) on the
// host, without a GPU: cancelling queued and in-flight requests, the
// watchdog's expiry by submission time, the hand-out of failures and the
// device-memory budget of admitted requests.
// Prints "ok" and returns 0 when every check holds.
#include "request_book.hpp"

#include <cstdio>
#include <deque>
#include <vector>

using namespace loom_b200;

namespace
{
struct Req
{
    uint64_t                ticket = 0;
    SteadyClock::time_point born{};
    int                     fail = 0;
};

int failures = 0;

void
check(bool ok, const char* what)
{
    if(!ok)
    {
        std::printf("FAIL: %s\n", what);
        ++failures;
    }
}

constexpr int kCancelled = -8;
constexpr int kTimeout   = -9;

struct Budget
{
    uint64_t limit = 0, used = 0;
};

void
test_budget()
{
    Budget b{1000, 0};
    check(request_bytes(10, 40, 25) == 500, "bytes: n x per-thread + 4 x table words");
    check(budget_take(&b, 600), "take what fits");
    check(!budget_take(&b, 500), "refuse what does not fit");
    check(b.used == 600, "a refusal takes nothing");
    check(budget_take(&b, 400) && b.used == 1000, "take up to the limit");
    budget_give(&b, 600);
    check(b.used == 400, "give back");
    check(!budget_take(&b, 1001), "larger than the limit never fits");
    budget_give(&b, 5000);
    check(b.used == 0, "giving back more than held clamps at zero");
    Budget* none = nullptr;
    check(budget_take(none, ~0ull), "no budget: everything fits");
    budget_give(none, 7);
    Budget big{~0ull, ~0ull - 10};
    check(!budget_take(&big, 11) && budget_take(&big, 10), "no overflow near the top");
}
} // namespace

int
main()
{
    const auto t0 = SteadyClock::now();
    std::deque<Req>     queued;
    std::vector<Req>    flight;
    std::deque<Failure> failed;
    for(uint64_t t = 1; t <= 3; ++t) queued.push_back({t, t0, 0});
    for(uint64_t t = 4; t <= 5; ++t) flight.push_back({t, t0, 0});

    // a queued request leaves at once and is reported
    check(cancel_request(queued, flight, 2, kCancelled, failed), "cancel queued");
    check(queued.size() == 2 && queued[0].ticket == 1 && queued[1].ticket == 3, "queue order kept");
    check(failed.size() == 1 && failed[0].ticket == 2 && failed[0].code == kCancelled, "queued failure");
    // one in flight is marked, reported later by the harvest
    check(cancel_request(queued, flight, 5, kCancelled, failed), "cancel in flight");
    check(flight[1].fail == kCancelled && failed.size() == 1, "in flight marked, not reported");
    // twice, or an unknown ticket: refused
    check(!cancel_request(queued, flight, 5, kCancelled, failed), "second cancel refused");
    check(!cancel_request(queued, flight, 2, kCancelled, failed), "cancelled ticket gone");
    check(!cancel_request(queued, flight, 99, kCancelled, failed), "unknown ticket refused");

    // watchdog off: nothing expires
    check(expire_requests(queued, flight, t0 + std::chrono::hours(1), 0, kTimeout, failed) == 0, "timeout 0 is off");
    // not yet due
    check(expire_requests(queued, flight, t0 + std::chrono::microseconds(500), 1000, kTimeout, failed) == 0,
          "young requests stay");
    // due: the queued ones leave, the unmarked one in flight is marked; the
    // one cancelled by the caller keeps its reason
    const uint64_t k = expire_requests(queued, flight, t0 + std::chrono::milliseconds(2), 1000, kTimeout, failed);
    check(k == 3, "three expire");
    check(queued.empty(), "queue emptied");
    check(flight[0].fail == kTimeout && flight[1].fail == kCancelled, "in-flight reasons");
    check(failed.size() == 3 && failed[1].ticket == 1 && failed[2].ticket == 3 && failed[2].code == kTimeout,
          "expired queued requests reported in order");

    // hand-out, oldest first, in pieces
    uint64_t tk[2];
    int32_t  cd[2];
    check(drain_failures(failed, tk, cd, 2) == 2 && tk[0] == 2 && cd[0] == kCancelled && tk[1] == 1, "first two");
    check(drain_failures(failed, tk, nullptr, 2) == 1 && tk[0] == 3, "the rest, codes skipped");
    check(drain_failures(failed, tk, cd, 2) == 0, "empty");

    test_budget();
    if(failures == 0) std::printf("ok\n");
    return failures == 0 ? 0 : 1;
}
