// Serving: continuous batching of Loom kernel invocations on the regrouping
// engine.
//
// Loom's streams keep a fixed set of thread rows busy by exchanging halted
// rows for new inputs (StreamFacade::exchange, src/vm/bve.hpp:1208-1270) and
// spread requests over workers (mp::Shop, src/vm/mp.hpp:316-385).  A server
// here does the same for whole requests on one GPU:
//
//  * a request is an instance: n threads, its input columns (host arrays),
//    an optional table header and body (the scene of a render request);
//  * requests are admitted in arrival order while their thread state fits:
//    a free request slot, room in the column rings (every array input and
//    output is a ring of `ring_threads` entries indexed by thread id), and
//    room for the table body in the table arena;
//  * the device runs slices of `slice_rounds` rounds of the regrouping
//    megakernel; between slices the parked threads stay in the queues on the
//    device, so a request admitted now joins the threads of every request in
//    flight, and they share warps whenever they stand at the same block;
//  * after each slice the per-instance completion counters come back; a
//    request whose threads all finished has its outputs copied to the host
//    and frees its slot, ring range and table space;
//  * the caller can cancel a request, and a host-side watchdog cancels the
//    requests older than a timeout (request_book.hpp); a cancelled request
//    in flight is dropped once its threads have finished.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <vector>

#include "request_book.hpp"
#include "runtime_iface.h"

using namespace loom_b200;

namespace
{
#define SV_CUDA(call)                                     \
    do                                                    \
    {                                                     \
        if((call) != cudaSuccess) return LOOM_B200_ERR_CUDA; \
    } while(0)

size_t
tbytes(int t)
{
    switch(t)
    {
    case LOOM_B200_B8:
    case LOOM_B200_I8:
    case LOOM_B200_U8: return 1;
    case LOOM_B200_I16:
    case LOOM_B200_U16: return 2;
    case LOOM_B200_I32:
    case LOOM_B200_U32:
    case LOOM_B200_F32: return 4;
    default: return 8;
    }
}

__global__ void
serve_reset(RegroupCtl* ctl, unsigned* qcnt, unsigned* qhead, unsigned num_queues)
{
    for(unsigned i = threadIdx.x; i < 3 * num_queues; i += blockDim.x)
    {
        if(i < 2 * num_queues)
            qcnt[i] = 0u;
        else
            qhead[i - 2 * num_queues] = 0u;
    }
    if(threadIdx.x == 0)
    {
        ctl->bar_count  = 0u;
        ctl->bar_gen    = 0u;
        ctl->done       = 0u;
        ctl->pad0       = 0u;
        ctl->cursor     = 0ull;
        ctl->admit_end  = 0ull;
        ctl->next_round = 0ull;
        ctl->t_first    = ~0ull;
        ctl->t_last     = 0ull;
    }
}

/// Before a slice: the threads parked by the previous slice wait in the
/// queues of parity round0 & 1; clear the other parity and the pop cursors
/// and admit new inputs up to the population.
__global__ void
serve_resume(RegroupCtl*        ctl,
             unsigned*          qcnt,
             unsigned*          qhead,
             unsigned           num_queues,
             unsigned           round0,
             unsigned long long n,
             unsigned long long cap)
{
    if(threadIdx.x != 0) return;
    const unsigned     cur    = round0 & 1u, nxt = cur ^ 1u;
    unsigned long long parked = 0;
    for(unsigned b = 0; b < num_queues; ++b)
    {
        parked += qcnt[cur * num_queues + b];
        qcnt[nxt * num_queues + b] = 0u;
        qhead[b]                   = 0u;
    }
    ctl->bar_count = 0u;
    ctl->done      = 0u;
    ctl->t_first   = ~0ull;
    ctl->t_last    = 0ull;
    const unsigned long long c    = ctl->cursor;
    const unsigned long long room = parked < cap ? cap - parked : 0ull;
    ctl->admit_end                = c + room < n ? c + room : n;
}

struct Request
{
    uint64_t              ticket;
    uint64_t              n;
    std::vector<const void*> inputs;
    std::vector<void*>    outputs;
    std::vector<uint32_t> header;
    const uint32_t*       body       = nullptr;
    uint64_t              body_words = 0;
    SteadyClock::time_point born{}; // submission time, for the watchdog
    int                     fail = 0; // LOOM_B200_ERR_* once cancelled
    uint64_t                bytes  = 0;     // budget bytes while admitted
    bool                    waited = false; // has waited for the budget
    // in flight
    uint32_t slot     = 0;
    uint64_t vstart   = 0;
    uint64_t arena_at = 0;
};

/// First-fit allocator over the words of the table arena.
struct Arena
{
    std::map<uint64_t, uint64_t> free; // start -> length

    void
    init(uint64_t words)
    {
        free.clear();
        if(words) free[0] = words;
    }

    bool
    alloc(uint64_t words, uint64_t* at)
    {
        if(words == 0)
        {
            *at = 0;
            return true;
        }
        for(auto it = free.begin(); it != free.end(); ++it)
            if(it->second >= words)
            {
                *at                 = it->first;
                const uint64_t rest = it->second - words;
                const uint64_t next = it->first + words;
                free.erase(it);
                if(rest) free[next] = rest;
                return true;
            }
        return false;
    }

    void
    release(uint64_t at, uint64_t words)
    {
        if(words == 0) return;
        auto it = free.emplace(at, words).first;
        auto nx = std::next(it);
        if(nx != free.end() && it->first + it->second == nx->first)
        {
            it->second += nx->second;
            free.erase(nx);
        }
        if(it != free.begin())
        {
            auto pv = std::prev(it);
            if(pv->first + pv->second == it->first)
            {
                pv->second += it->second;
                free.erase(it);
            }
        }
    }
};

const KernelEntry*
find_entry(const char* name)
{
    for(int i = 0; i < kRegistrySize; ++i)
        if(std::strcmp(kRegistry[i]->info->name, name) == 0) return kRegistry[i];
    return nullptr;
}
} // namespace

struct loom_b200_server
{
    const KernelEntry*    e = nullptr;
    loom_b200_opts        opts{};
    loom_b200_server_cfg  cfg{};
    std::vector<uint32_t> forms;
    cudaStream_t          stream = nullptr;
    int                   sms    = 0;
    unsigned              grid = 0, block = 0;
    uint64_t              cap  = 0; // population
    uint64_t              mask = 0; // ring_threads - 1

    // device memory
    char*               d_state    = nullptr;
    unsigned*           d_qcnt     = nullptr;
    unsigned*           d_qhead    = nullptr;
    RegroupCtl*         d_ctl      = nullptr;
    unsigned*           d_status   = nullptr;
    unsigned long long* d_counters = nullptr;
    unsigned*           d_done     = nullptr; // per slot
    unsigned long long* d_starts   = nullptr; // max_requests + 1
    unsigned*           d_ids      = nullptr; // max_requests
    unsigned*           d_table    = nullptr; // headers, then the arena
    std::vector<void*>  d_cols;               // one ring per input (array form) and output
    uint64_t            device_bytes = 0;

    // host side; the results of a slice come back into pinned memory, so
    // that starting a slice does not wait for it
    std::deque<Request>     queued;
    std::vector<Request>    flight; // in virtual-start order
    std::vector<uint32_t>   free_slots;
    Arena                   arena;
    unsigned*               h_done     = nullptr; // pinned, max_requests
    RegroupCtl*             h_ctl      = nullptr; // pinned
    unsigned*               h_status   = nullptr; // pinned
    unsigned long long*     h_counters = nullptr; // pinned, 8
    cudaEvent_t             ev_a = nullptr, ev_k = nullptr, ev_b = nullptr;
    bool                    launched   = false; // a slice runs, not harvested yet
    uint64_t                per_thread = 0;     // budget bytes per thread of a request
    std::vector<unsigned long long> h_starts;
    std::vector<unsigned>   h_ids;
    std::deque<uint64_t>    done_q; // completed tickets not handed out yet
    std::deque<Failure>     failed_q; // cancelled tickets not handed out yet
    uint64_t                timeout_us = 0; // watchdog (0: off)
    uint64_t                vnext      = 0;
    uint64_t                next_round = 0;
    uint64_t                ticket     = 0;
    loom_b200_server_stats  st{};
};

namespace
{
int
dalloc(loom_b200_server* s, void** p, size_t bytes)
{
    if(bytes == 0) bytes = 16;
    if(cudaMalloc(p, bytes) != cudaSuccess)
    {
        *p = nullptr;
        return LOOM_B200_ERR_OOM;
    }
    s->device_bytes += bytes;
    return LOOM_B200_OK;
}

void
free_all(loom_b200_server* s)
{
    cudaFreeHost(s->h_done);
    cudaFreeHost(s->h_ctl);
    cudaFreeHost(s->h_status);
    cudaFreeHost(s->h_counters);
    if(s->ev_a) cudaEventDestroy(s->ev_a);
    if(s->ev_k) cudaEventDestroy(s->ev_k);
    if(s->ev_b) cudaEventDestroy(s->ev_b);
    cudaFree(s->d_state);
    cudaFree(s->d_qcnt);
    cudaFree(s->d_qhead);
    cudaFree(s->d_ctl);
    cudaFree(s->d_status);
    cudaFree(s->d_counters);
    cudaFree(s->d_done);
    cudaFree(s->d_starts);
    cudaFree(s->d_ids);
    cudaFree(s->d_table);
    for(void* p: s->d_cols) cudaFree(p);
}

/// Copies `count` entries starting at ring position `pos` between a host
/// array and a device ring of `ring` entries of `eb` bytes, in at most two
/// pieces.
int
ring_copy(void* ring_dev, const void* host_src, void* host_dst, uint64_t pos, uint64_t count,
          uint64_t ring, size_t eb, cudaStream_t st)
{
    const uint64_t first = std::min<uint64_t>(count, ring - pos);
    char*          d     = static_cast<char*>(ring_dev);
    if(host_src)
    {
        const char* h = static_cast<const char*>(host_src);
        SV_CUDA(cudaMemcpyAsync(d + pos * eb, h, first * eb, cudaMemcpyHostToDevice, st));
        if(count > first)
            SV_CUDA(cudaMemcpyAsync(d, h + first * eb, (count - first) * eb, cudaMemcpyHostToDevice, st));
    }
    else
    {
        char* h = static_cast<char*>(host_dst);
        SV_CUDA(cudaMemcpyAsync(h, d + pos * eb, first * eb, cudaMemcpyDeviceToHost, st));
        if(count > first)
            SV_CUDA(cudaMemcpyAsync(h + first * eb, d, (count - first) * eb, cudaMemcpyDeviceToHost, st));
    }
    return LOOM_B200_OK;
}

uint64_t
tid_base(const loom_b200_server* s)
{
    return s->flight.empty() ? s->vnext : s->flight.front().vstart;
}

/// Admits queued requests in arrival order while they fit.
int
admit(loom_b200_server* s)
{
    const loom_b200_kernel_info& info = *s->e->info;
    const uint64_t               ring = s->mask + 1;
    while(!s->queued.empty() && !s->free_slots.empty())
    {
        Request& r = s->queued.front();
        if(s->vnext + r.n > tid_base(s) + ring) break; // ring full until older requests finish
        if(!budget_take(s->cfg.budget, r.bytes))
        {
            // the budget is held by requests in flight (of this server or
            // of others sharing the budget): wait, in arrival order
            if(!r.waited) s->st.budget_waits += 1;
            r.waited = true;
            break;
        }
        uint64_t at = 0;
        if(!s->arena.alloc(r.body_words, &at))
        {
            budget_give(s->cfg.budget, r.bytes);
            break;
        }
        s->st.held_bytes += r.bytes;
        r.slot     = s->free_slots.back();
        r.vstart   = s->vnext;
        r.arena_at = at;
        s->free_slots.pop_back();
        const uint64_t pos = r.vstart & s->mask;
        for(uint32_t i = 0; i < info.num_inputs; ++i)
            if(s->forms[i] == LOOM_B200_IN_ARRAY)
            {
                const int rc = ring_copy(s->d_cols[i], r.inputs[i], nullptr, pos, r.n, ring,
                                         tbytes(info.input_types[i]), s->stream);
                if(rc) return rc;
            }
        if(s->cfg.header_words)
        {
            std::vector<uint32_t> hdr = r.header;
            if(s->cfg.reloc_word >= 0)
                hdr[s->cfg.reloc_word] += static_cast<uint32_t>(
                    uint64_t(s->cfg.max_requests) * s->cfg.header_words + at);
            // header bytes live in the request (kept until completion)
            r.header = hdr;
            SV_CUDA(cudaMemcpyAsync(s->d_table + uint64_t(r.slot) * s->cfg.header_words,
                                    r.header.data(),
                                    s->cfg.header_words * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice,
                                    s->stream));
        }
        if(r.body_words)
            SV_CUDA(cudaMemcpyAsync(s->d_table + uint64_t(s->cfg.max_requests) * s->cfg.header_words + at,
                                    r.body,
                                    r.body_words * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice,
                                    s->stream));
        SV_CUDA(cudaMemsetAsync(s->d_done + r.slot, 0, sizeof(unsigned), s->stream));
        s->h_done[r.slot] = 0u;
        s->vnext += r.n;
        s->st.admitted += 1;
        s->flight.push_back(std::move(r));
        s->queued.pop_front();
    }
    return LOOM_B200_OK;
}
} // namespace

extern "C" {

int
loom_b200_server_create(const char*                 kernel,
                        const loom_b200_opts*       opts,
                        const loom_b200_server_cfg* cfg,
                        void*                       stream,
                        loom_b200_server**          out)
{
    if(!kernel || !cfg || !out) return LOOM_B200_ERR_INVALID;
    *out                  = nullptr;
    const KernelEntry* e  = find_entry(kernel);
    if(!e) return LOOM_B200_ERR_NOT_FOUND;
    const loom_b200_kernel_info& info = *e->info;
    const uint64_t ring = cfg->ring_threads;
    if(ring < 32 || ring > (1ull << 31) || (ring & (ring - 1)) != 0) return LOOM_B200_ERR_INVALID;
    if(cfg->max_requests == 0 || cfg->max_requests > (1u << 20)) return LOOM_B200_ERR_INVALID;
    if(cfg->reloc_word >= static_cast<int32_t>(cfg->header_words)) return LOOM_B200_ERR_INVALID;
    if(info.num_inputs > static_cast<uint32_t>(kMaxIn) ||
       info.num_inputs + info.num_outputs > static_cast<uint32_t>(kMaxCols))
        return LOOM_B200_ERR_INVALID;

    int dev = 0, sms = 0;
    if(cudaGetDevice(&dev) != cudaSuccess) return LOOM_B200_ERR_NO_DEVICE;
    if(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return LOOM_B200_ERR_NO_DEVICE;

    auto* s = new(std::nothrow) loom_b200_server;
    if(!s) return LOOM_B200_ERR_OOM;
    s->e      = e;
    s->cfg    = *cfg;
    s->stream = static_cast<cudaStream_t>(stream);
    s->sms    = sms;
    s->mask   = ring - 1;
    if(opts) s->opts = *opts;
    loom_b200_opts& o = s->opts;
    if(o.block_size == 0 || o.block_size % 32 != 0 || o.block_size > 1024) o.block_size = 256;
    if(o.utr_lanes == 0 || o.utr_lanes > 32) o.utr_lanes = 16;
    if(o.period == 0) o.period = 1024;
    if(o.burst == 0) o.burst = 32;
    if(o.spread_lanes == 0) o.spread_lanes = 33;
    if(o.max_steps == 0) o.max_steps = 1ull << 40;
    if(s->cfg.slice_rounds == 0) s->cfg.slice_rounds = 4;
    s->forms.assign(info.num_inputs, LOOM_B200_IN_ARRAY);
    if(cfg->forms)
        for(uint32_t i = 0; i < info.num_inputs; ++i)
        {
            if(cfg->forms[i] > LOOM_B200_IN_INSTANCE || cfg->forms[i] == LOOM_B200_IN_BROADCAST)
            {
                delete s;
                return LOOM_B200_ERR_INVALID;
            }
            s->forms[i] = cfg->forms[i];
        }
    s->cap = (o.population ? o.population : (1ull << 21));
    s->cap = std::min<uint64_t>((s->cap + 31) / 32 * 32, ring);

    // launch shape: the largest CTA up to the requested size that fits
    unsigned block = o.block_size;
    int      ctas  = 0;
    for(;;)
    {
        if(e->regroup_occupancy(static_cast<int>(block), o.profile != 0, o.max_regs, 0u, true, &ctas) != cudaSuccess)
        {
            delete s;
            return LOOM_B200_ERR_CUDA;
        }
        if(ctas > 0 || block <= 32) break;
        block /= 2;
    }
    if(ctas <= 0)
    {
        delete s;
        return LOOM_B200_ERR_INVALID;
    }
    if(o.ctas_per_sm) ctas = std::min<int>(ctas, static_cast<int>(o.ctas_per_sm));
    s->grid  = static_cast<unsigned>(ctas * sms);
    s->block = block;

    const uint64_t B  = e->num_queues;
    const uint64_t mr = cfg->max_requests;
    int            rc = LOOM_B200_OK;
    rc = rc ? rc : dalloc(s, reinterpret_cast<void**>(&s->d_state), 2 * e->row_bytes * s->cap);
    rc = rc ? rc : dalloc(s, reinterpret_cast<void**>(&s->d_qcnt), 2 * B * sizeof(unsigned));
    rc = rc ? rc : dalloc(s, reinterpret_cast<void**>(&s->d_qhead), B * sizeof(unsigned));
    rc = rc ? rc : dalloc(s, reinterpret_cast<void**>(&s->d_ctl), sizeof(RegroupCtl));
    rc = rc ? rc : dalloc(s, reinterpret_cast<void**>(&s->d_status), sizeof(unsigned));
    const size_t cbytes = (8 + 2 * static_cast<size_t>(info.num_blocks)) * sizeof(unsigned long long);
    rc = rc ? rc : dalloc(s, reinterpret_cast<void**>(&s->d_counters), cbytes);
    rc = rc ? rc : dalloc(s, reinterpret_cast<void**>(&s->d_done), mr * sizeof(unsigned));
    rc = rc ? rc : dalloc(s, reinterpret_cast<void**>(&s->d_starts), (mr + 1) * sizeof(unsigned long long));
    rc = rc ? rc : dalloc(s, reinterpret_cast<void**>(&s->d_ids), mr * sizeof(unsigned));
    rc = rc ? rc
            : dalloc(s, reinterpret_cast<void**>(&s->d_table),
                     (mr * cfg->header_words + cfg->table_words) * sizeof(uint32_t));
    s->d_cols.assign(info.num_inputs + info.num_outputs, nullptr);
    for(uint32_t i = 0; i < info.num_inputs && !rc; ++i)
        if(s->forms[i] == LOOM_B200_IN_ARRAY)
            rc = dalloc(s, &s->d_cols[i], ring * tbytes(info.input_types[i]));
    for(uint32_t j = 0; j < info.num_outputs && !rc; ++j)
        rc = dalloc(s, &s->d_cols[info.num_inputs + j], ring * tbytes(info.output_types[j]));
    if(!rc)
    {
        serve_reset<<<1, 256, 0, s->stream>>>(s->d_ctl, s->d_qcnt, s->d_qhead, e->num_queues);
        if(cudaGetLastError() != cudaSuccess ||
           cudaMemsetAsync(s->d_status, 0, sizeof(unsigned), s->stream) != cudaSuccess ||
           cudaMemsetAsync(s->d_counters, 0, cbytes, s->stream) != cudaSuccess ||
           cudaStreamSynchronize(s->stream) != cudaSuccess)
            rc = LOOM_B200_ERR_CUDA;
    }
    if(rc)
    {
        free_all(s);
        delete s;
        return rc;
    }
    if(!rc &&
       (cudaMallocHost(reinterpret_cast<void**>(&s->h_done), mr * sizeof(unsigned)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&s->h_ctl), sizeof(RegroupCtl)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&s->h_status), sizeof(unsigned)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&s->h_counters), 8 * sizeof(unsigned long long)) != cudaSuccess))
        rc = LOOM_B200_ERR_OOM;
    if(!rc && (cudaEventCreate(&s->ev_a) != cudaSuccess || cudaEventCreate(&s->ev_k) != cudaSuccess ||
               cudaEventCreateWithFlags(&s->ev_b, cudaEventDisableTiming) != cudaSuccess))
        rc = LOOM_B200_ERR_CUDA;
    if(rc)
    {
        free_all(s);
        delete s;
        return rc;
    }
    std::memset(s->h_done, 0, mr * sizeof(unsigned));
    // budget bytes per thread: the thread state (K::state_size) and the
    // thread's entries in the column rings
    s->per_thread = info.state_size;
    for(uint32_t i = 0; i < info.num_inputs; ++i)
        if(s->forms[i] == LOOM_B200_IN_ARRAY) s->per_thread += tbytes(info.input_types[i]);
    for(uint32_t j = 0; j < info.num_outputs; ++j) s->per_thread += tbytes(info.output_types[j]);
    s->arena.init(cfg->table_words);
    for(uint32_t i = 0; i < mr; ++i) s->free_slots.push_back(static_cast<uint32_t>(mr - 1 - i));
    s->st.device_bytes = s->device_bytes;
    *out               = s;
    return LOOM_B200_OK;
}

int
loom_b200_server_destroy(loom_b200_server* s)
{
    if(!s) return LOOM_B200_OK;
    cudaStreamSynchronize(s->stream);
    for(const Request& r: s->flight) budget_give(s->cfg.budget, r.bytes);
    free_all(s);
    delete s;
    return LOOM_B200_OK;
}

int
loom_b200_server_submit(loom_b200_server* s, const loom_b200_request* r, uint64_t* ticket)
{
    if(!s || !r) return LOOM_B200_ERR_INVALID;
    const loom_b200_kernel_info& info = *s->e->info;
    if(r->n == 0 || r->n > s->mask + 1) return LOOM_B200_ERR_BUDGET;
    if(!r->outputs) return LOOM_B200_ERR_INVALID;
    if(s->cfg.header_words && !r->header) return LOOM_B200_ERR_INVALID;
    if(r->body_words > s->cfg.table_words) return LOOM_B200_ERR_BUDGET;
    Request q;
    q.ticket = ++s->ticket;
    q.n      = r->n;
    q.born   = SteadyClock::now();
    q.inputs.assign(info.num_inputs, nullptr);
    for(uint32_t i = 0; i < info.num_inputs; ++i)
        if(s->forms[i] == LOOM_B200_IN_ARRAY)
        {
            if(!r->inputs || !r->inputs[i]) return LOOM_B200_ERR_INVALID;
            q.inputs[i] = r->inputs[i];
        }
    q.outputs.assign(r->outputs, r->outputs + info.num_outputs);
    for(void* p: q.outputs)
        if(!p) return LOOM_B200_ERR_INVALID;
    if(s->cfg.header_words) q.header.assign(r->header, r->header + s->cfg.header_words);
    q.body       = r->body;
    q.body_words = r->body ? r->body_words : 0;
    q.bytes      = request_bytes(q.n, s->per_thread, s->cfg.header_words + q.body_words);
    if(s->cfg.budget && q.bytes > s->cfg.budget->limit) return LOOM_B200_ERR_BUDGET;
    if(ticket) *ticket = q.ticket;
    s->queued.push_back(std::move(q));
    s->st.submitted += 1;
    return LOOM_B200_OK;
}

namespace
{
/// Admits what fits and starts a slice on the server's stream (with
/// `ctas_per_sm` CTAs per SM, 0: the server's own shape) without waiting:
/// the completion counters, control block, status and counters come back
/// into pinned host memory behind it.  Nothing starts when no request is in
/// flight.
int
slice_launch(loom_b200_server* s, unsigned ctas_per_sm)
{
    if(s->launched) return LOOM_B200_OK;
    if(int rc = admit(s)) return rc;
    if(s->flight.empty()) return LOOM_B200_OK;
    const loom_b200_kernel_info& info = *s->e->info;

    // instance table of this slice: requests in flight, in thread order
    const size_t m = s->flight.size();
    s->h_starts.resize(m + 1);
    s->h_ids.resize(m);
    for(size_t i = 0; i < m; ++i)
    {
        s->h_starts[i] = s->flight[i].vstart;
        s->h_ids[i]    = s->flight[i].slot;
    }
    s->h_starts[m] = s->vnext;
    SV_CUDA(cudaMemcpyAsync(s->d_starts, s->h_starts.data(), (m + 1) * sizeof(unsigned long long),
                            cudaMemcpyHostToDevice, s->stream));
    SV_CUDA(cudaMemcpyAsync(s->d_ids, s->h_ids.data(), m * sizeof(unsigned), cudaMemcpyHostToDevice,
                            s->stream));

    const loom_b200_opts& o = s->opts;
    RegroupLaunch         L{};
    Columns&              c = L.params.cols;
    for(uint32_t i = 0; i < info.num_inputs; ++i)
    {
        c.form[i] = s->forms[i];
        c.p[i]    = s->d_cols[i];
    }
    for(uint32_t j = 0; j < info.num_outputs; ++j)
        c.p[info.num_inputs + j] = s->d_cols[info.num_inputs + j];
    c.inst_start = s->d_starts;
    c.num_inst   = static_cast<unsigned>(m);
    c.table      = s->d_table;
    c.ring_mask  = s->mask;
    c.tid_base   = tid_base(s);
    c.inst_id    = s->d_ids;
    L.params.state         = s->d_state;
    L.params.qcnt          = s->d_qcnt;
    L.params.qhead         = s->d_qhead;
    L.params.ctl           = s->d_ctl;
    L.params.status        = s->d_status;
    L.params.counters      = s->d_counters;
    L.params.n             = s->vnext;
    L.params.max_rounds    = o.max_steps;
    L.params.barrier_spins = o.barrier_spins ? o.barrier_spins : (1ull << 25);
    L.params.cap           = static_cast<unsigned>(s->cap);
    L.params.utr           = o.utr_lanes;
    L.params.period        = o.period;
    L.params.burst         = o.burst;
    L.params.spread        = o.spread_lanes;
    L.params.refill        = o.no_refill ? 0u : 1u;
    L.params.prefetch      = o.no_prefetch ? 0u : 1u;
    L.params.cost_model    = o.cost_model;
    L.params.schedule      = o.schedule;
    L.params.defer_lanes   = o.defer_lanes;
    L.params.spin_iters    = o.spin_iters;
    L.params.refill_lanes  = o.refill_lanes;
    L.params.round0        = static_cast<unsigned>(s->next_round);
    // beside other servers' slices: one round, an ordinary launch (no grid
    // barrier to wait at), so that the GPU runs the slices together;
    // cooperative launches do not share the GPU with other kernels
    L.params.slice_rounds  = ctas_per_sm ? 1u : s->cfg.slice_rounds;
    L.ordinary             = ctas_per_sm != 0u;
    L.params.inst_done     = s->d_done;
    L.grid                 = s->grid;
    if(ctas_per_sm)
    {
        // never more CTAs per SM than fit (cooperative launches need every
        // CTA resident at once)
        int fit = 0;
        SV_CUDA(s->e->regroup_occupancy(static_cast<int>(s->block), o.profile != 0, o.max_regs, 0u, true, &fit));
        const unsigned c = std::min<unsigned>(ctas_per_sm, static_cast<unsigned>(std::max(fit, 1)));
        L.grid           = c * static_cast<unsigned>(s->sms);
    }
    L.block   = s->block;
    L.regs    = o.max_regs;
    L.profile = o.profile != 0;
    L.stream  = s->stream;
    SV_CUDA(cudaEventRecord(s->ev_a, s->stream));
    serve_resume<<<1, 32, 0, s->stream>>>(s->d_ctl, s->d_qcnt, s->d_qhead, s->e->num_queues,
                                          static_cast<unsigned>(s->next_round), s->vnext, s->cap);
    SV_CUDA(cudaGetLastError());
    SV_CUDA(s->e->regroup(L));
    SV_CUDA(cudaEventRecord(s->ev_k, s->stream));
    SV_CUDA(cudaMemcpyAsync(s->h_done, s->d_done, s->cfg.max_requests * sizeof(unsigned),
                            cudaMemcpyDeviceToHost, s->stream));
    SV_CUDA(cudaMemcpyAsync(s->h_ctl, s->d_ctl, sizeof(RegroupCtl), cudaMemcpyDeviceToHost, s->stream));
    SV_CUDA(cudaMemcpyAsync(s->h_status, s->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
    SV_CUDA(cudaMemcpyAsync(s->h_counters, s->d_counters, 8 * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, s->stream));
    SV_CUDA(cudaEventRecord(s->ev_b, s->stream));
    s->launched = true;
    return LOOM_B200_OK;
}

/// Waits for the slice started by slice_launch, then copies out the
/// requests whose threads all finished and frees what they held.
int
slice_harvest(loom_b200_server* s)
{
    if(!s->launched) return LOOM_B200_OK;
    s->launched = false;
    const loom_b200_kernel_info& info = *s->e->info;
    const uint64_t               ring = s->mask + 1;
    SV_CUDA(cudaEventSynchronize(s->ev_b));
    float ms = 0.f;
    if(cudaEventElapsedTime(&ms, s->ev_a, s->ev_k) == cudaSuccess) s->st.busy_ms += ms;
    const unsigned status = *s->h_status;
    s->next_round      = s->h_ctl->next_round;
    s->st.slice_t0_ns  = s->h_ctl->t_first;
    s->st.slice_t1_ns  = s->h_ctl->t_last;
    s->st.slices      += 1;
    s->st.status      |= status;
    s->st.thread_instr = s->h_counters[0];
    s->st.warp_instr   = s->h_counters[1];
    s->st.rounds       = s->h_counters[5];
    if(status) return LOOM_B200_ERR_DEVICE;

    // harvest: requests whose threads all finished
    uint32_t             k = 0;
    std::vector<Request> keep;
    keep.reserve(s->flight.size());
    for(Request& r: s->flight)
    {
        if(s->h_done[r.slot] < r.n)
        {
            keep.push_back(std::move(r));
            continue;
        }
        budget_give(s->cfg.budget, r.bytes);
        s->st.held_bytes -= r.bytes;
        if(r.fail)
        {
            // cancelled in flight: its threads have finished, so its slot,
            // ring range, arena words and budget are free; nothing is copied out
            s->arena.release(r.arena_at, r.body_words);
            s->free_slots.push_back(r.slot);
            s->failed_q.push_back({r.ticket, r.fail});
            continue;
        }
        const uint64_t pos = r.vstart & s->mask;
        for(uint32_t j = 0; j < info.num_outputs; ++j)
        {
            const int rc = ring_copy(s->d_cols[info.num_inputs + j], nullptr, r.outputs[j], pos, r.n,
                                     ring, tbytes(info.output_types[j]), s->stream);
            if(rc) return rc;
        }
        s->arena.release(r.arena_at, r.body_words);
        s->free_slots.push_back(r.slot);
        s->st.completed += 1;
        s->st.threads += r.n;
        s->done_q.push_back(r.ticket);
        ++k;
    }
    s->flight.swap(keep);
    if(k) SV_CUDA(cudaStreamSynchronize(s->stream));
    return LOOM_B200_OK;
}
} // namespace

int
loom_b200_server_step(loom_b200_server* s, uint64_t* done, uint32_t max_done, uint32_t* n_done)
{
    if(!s) return LOOM_B200_ERR_INVALID;
    if(n_done) *n_done = 0;
    int rc = LOOM_B200_OK;
    if(!s->launched)
    {
        expire_requests(s->queued, s->flight, SteadyClock::now(), s->timeout_us, LOOM_B200_ERR_TIMEOUT,
                        s->failed_q);
        rc = slice_launch(s, 0u);
    }
    if(!rc) rc = slice_harvest(s);
    uint32_t k = 0;
    while(done && k < max_done && !s->done_q.empty())
    {
        done[k++] = s->done_q.front();
        s->done_q.pop_front();
    }
    if(n_done) *n_done = k;
    return rc;
}

int
loom_b200_server_launch(loom_b200_server* s, uint32_t ctas_per_sm)
{
    if(!s) return LOOM_B200_ERR_INVALID;
    if(s->launched) return LOOM_B200_OK;
    expire_requests(s->queued, s->flight, SteadyClock::now(), s->timeout_us, LOOM_B200_ERR_TIMEOUT,
                    s->failed_q);
    return slice_launch(s, ctas_per_sm);
}

int
loom_b200_server_cancel(loom_b200_server* s, uint64_t ticket)
{
    if(!s) return LOOM_B200_ERR_INVALID;
    return cancel_request(s->queued, s->flight, ticket, LOOM_B200_ERR_CANCELLED, s->failed_q)
               ? LOOM_B200_OK
               : LOOM_B200_ERR_INVALID;
}

int
loom_b200_server_set_timeout(loom_b200_server* s, uint64_t timeout_us)
{
    if(!s) return LOOM_B200_ERR_INVALID;
    s->timeout_us = timeout_us;
    return LOOM_B200_OK;
}

int
loom_b200_server_failed(loom_b200_server* s, uint64_t* tickets, int32_t* codes, uint32_t max, uint32_t* n)
{
    if(!s || !n) return LOOM_B200_ERR_INVALID;
    *n = drain_failures(s->failed_q, tickets, codes, max);
    return LOOM_B200_OK;
}

int
loom_b200_server_get_stats(const loom_b200_server* s, loom_b200_server_stats* st)
{
    if(!s || !st) return LOOM_B200_ERR_INVALID;
    *st           = s->st;
    st->queued    = s->queued.size();
    st->in_flight = s->flight.size();
    st->unreported = s->done_q.size();
    return LOOM_B200_OK;
}

} // extern "C"
