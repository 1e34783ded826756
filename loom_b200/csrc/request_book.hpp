// Host bookkeeping of the serving loop (no CUDA): requests the caller
// cancels, requests a host-side watchdog expires, and the device-memory
// budget that admitted requests hold.
//
// Loom has neither (its streams have no request boundary,
// src/vm/bve.hpp:1208-1270).  The server's threads cannot be taken back
// from the device once admitted, so a request ends in one of two ways:
// still queued, it leaves the queue at once; in flight, it is marked and
// dropped by the harvest after its threads have finished (its outputs are
// not copied out and its ticket never comes back as completed).  Either way
// its ticket is reported once as a failure with the reason.
#pragma once

#include <chrono>
#include <cstdint>
#include <deque>
#include <vector>

namespace loom_b200
{
using SteadyClock = std::chrono::steady_clock;

/// A ticket that will not complete, and why (a LOOM_B200_ERR_* code).
struct Failure
{
    uint64_t ticket;
    int      code;
};

/// Ends request `ticket` with `code`.  `Req` has `ticket`, `born` (its
/// submission time) and `fail` (0 while it may still complete).  Returns
/// false when the ticket is neither queued nor in flight, or was ended
/// already.
template <typename Req>
bool
cancel_request(std::deque<Req>&      queued,
               std::vector<Req>&     flight,
               uint64_t              ticket,
               int                   code,
               std::deque<Failure>&  failed)
{
    for(auto it = queued.begin(); it != queued.end(); ++it)
        if(it->ticket == ticket)
        {
            failed.push_back({ticket, code});
            queued.erase(it);
            return true;
        }
    for(Req& r: flight)
        if(r.ticket == ticket)
        {
            if(r.fail) return false;
            r.fail = code;
            return true;
        }
    return false;
}

/// The watchdog: ends with `code` every request submitted more than
/// `timeout_us` microseconds before `now` (0: off).  Returns how many it
/// ended.
template <typename Req>
uint64_t
expire_requests(std::deque<Req>&        queued,
                std::vector<Req>&       flight,
                SteadyClock::time_point now,
                uint64_t                timeout_us,
                int                     code,
                std::deque<Failure>&    failed)
{
    if(timeout_us == 0) return 0;
    const auto limit = std::chrono::microseconds(timeout_us);
    uint64_t   k     = 0;
    for(auto it = queued.begin(); it != queued.end();)
        if(now - it->born > limit)
        {
            failed.push_back({it->ticket, code});
            it = queued.erase(it);
            ++k;
        }
        else
            ++it;
    for(Req& r: flight)
        if(!r.fail && now - r.born > limit)
        {
            r.fail = code;
            ++k;
        }
    return k;
}

/// Device bytes a request holds while admitted: per thread its state and
/// its column entries (`per_thread`), plus its table words.
inline uint64_t
request_bytes(uint64_t n, uint64_t per_thread, uint64_t table_words)
{
    return n * per_thread + 4 * table_words;
}

/// Takes `bytes` from a budget (`limit`, `used`) when they fit; a NULL
/// budget always fits.
template <typename Budget>
bool
budget_take(Budget* b, uint64_t bytes)
{
    if(!b) return true;
    if(bytes > b->limit || b->used > b->limit - bytes) return false;
    b->used += bytes;
    return true;
}

/// Gives `bytes` back to a budget (NULL: nothing to do).
template <typename Budget>
void
budget_give(Budget* b, uint64_t bytes)
{
    if(b) b->used -= bytes < b->used ? bytes : b->used;
}

/// Hands out up to `max` failures, oldest first; returns how many.
inline uint32_t
drain_failures(std::deque<Failure>& failed, uint64_t* tickets, int32_t* codes, uint32_t max)
{
    uint32_t k = 0;
    while(k < max && !failed.empty())
    {
        if(tickets) tickets[k] = failed.front().ticket;
        if(codes) codes[k] = failed.front().code;
        failed.pop_front();
        ++k;
    }
    return k;
}
} // namespace loom_b200
