// C-ABI runtime of libloom_b200: kernel registry, handles, device memory and
// launches of the plain and regrouping engines.
//
// The handle plays the role of Loom's backend facades (cuda::MemoryFacade /
// StreamFacade, Loom src/vm/cuda.hpp:1029-1327): it owns the device columns
// and the regrouping workspace (RAII on the host side of the ABI), copies
// inputs in and outputs out, and runs the kernel to completion on the device
// without per-round host round trips.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "runtime_iface.h"

using namespace loom_b200;

namespace
{
thread_local std::string g_last_error;

int
cuda_fail(cudaError_t e, const char* what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    if(e == cudaErrorMemoryAllocation) return LOOM_B200_ERR_OOM;
    if(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return LOOM_B200_ERR_NO_DEVICE;
    return LOOM_B200_ERR_CUDA;
}

#define LB_CUDA(call)                                  \
    do                                                 \
    {                                                  \
        const cudaError_t e_ = (call);                 \
        if(e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while(0)

size_t
type_bytes(int t)
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
regroup_reset(RegroupCtl*        ctl,
              unsigned*          qcnt,
              unsigned*          qhead,
              unsigned           num_blocks,
              unsigned long long first,
              unsigned long long admit_end)
{
    for(unsigned i = threadIdx.x; i < 3 * num_blocks; i += blockDim.x)
    {
        if(i < 2 * num_blocks)
            qcnt[i] = 0u;
        else
            qhead[i - 2 * num_blocks] = 0u;
    }
    if(threadIdx.x == 0)
    {
        ctl->bar_count = 0u;
        ctl->bar_gen   = 0u;
        ctl->done      = 0u;
        ctl->pad0      = 0u;
        ctl->cursor    = first;
        ctl->admit_end = admit_end;
        ctl->t_first   = ~0ull;
        ctl->t_last    = 0ull;
    }
}

/// Per-group means of a float column, summed in thread order: output row r
/// of instance i covers threads starts[i] + (r - out_starts[i]) * group[i]
/// and the group[i] - 1 after it; without instances every row covers
/// `group` threads from r * group.  Each warp takes 32 consecutive rows.
/// Where they lie in one instance, their group is a power of two from 4 to
/// kTileGroupMax and their samples start on a 16-byte boundary (f32), the
/// warp reads those samples with coalesced 16-byte loads into a padded
/// shared-memory tile (row stride group + 1: no bank conflicts) and each
/// lane then sums its row from there; otherwise each lane reads its row
/// from global memory.  Either way a row's samples are added one after the
/// other in thread order, so the means are the same bits.
constexpr unsigned kTileGroupMax = 64;
constexpr unsigned kMeanWarps    = 4; // warps per CTA of group_mean

template <typename T>
__device__ __forceinline__ void
row_of(const unsigned long long          r,
       const unsigned                    group,
       const unsigned long long* __restrict__ starts,
       const unsigned* __restrict__           inst_group,
       const unsigned long long* __restrict__ out_starts,
       const unsigned                    num_inst,
       unsigned long long&               t0,
       unsigned&                         g,
       unsigned&                         inst)
{
    t0   = r * group;
    g    = group;
    inst = 0;
    if(num_inst)
    {
        unsigned lo = 0, hi = num_inst; // out_starts[lo] <= r < out_starts[hi]
        while(hi - lo > 1)
        {
            const unsigned mid = (lo + hi) >> 1;
            if(out_starts[mid] <= r)
                lo = mid;
            else
                hi = mid;
        }
        g    = inst_group[lo];
        t0   = starts[lo] + (r - out_starts[lo]) * g;
        inst = lo;
    }
}

template <typename T>
__global__ void __launch_bounds__(32 * kMeanWarps)
group_mean(const T* __restrict__                  in,
           T* __restrict__                        out,
           const unsigned long long               rows,
           const unsigned                         group,
           const unsigned long long* __restrict__ starts,
           const unsigned* __restrict__           inst_group,
           const unsigned long long* __restrict__ out_starts,
           const unsigned                         num_inst)
{
    __shared__ float          s_tile[kMeanWarps][32 * (kTileGroupMax + 1)];
    const unsigned            lane = threadIdx.x & 31u;
    const unsigned            wib  = threadIdx.x >> 5;
    const unsigned long long  r0   = (static_cast<unsigned long long>(blockIdx.x) * kMeanWarps + wib) * 32ull;
    if(r0 >= rows) return;
    const unsigned            nr = rows - r0 < 32ull ? static_cast<unsigned>(rows - r0) : 32u;
    const unsigned long long  r  = r0 + lane;
    unsigned long long        t0 = 0;
    unsigned                  g = 0, inst = 0;
    if(lane < nr) row_of<T>(r, group, starts, inst_group, out_starts, num_inst, t0, g, inst);
    // the tile applies when every row of the warp has the first row's
    // instance (hence group), the group is a power of two in [4, 64] and
    // the first row's samples start on a 16-byte boundary
    const unsigned long long base = __shfl_sync(0xffffffffu, t0, 0);
    const unsigned           g0   = __shfl_sync(0xffffffffu, g, 0);
    const unsigned           i0   = __shfl_sync(0xffffffffu, inst, 0);
    bool tiled = sizeof(T) == 4 && g0 >= 4u && g0 <= kTileGroupMax && (g0 & (g0 - 1u)) == 0u &&
                 (reinterpret_cast<unsigned long long>(in + base) & 15ull) == 0ull;
    tiled = __all_sync(0xffffffffu, !tiled || lane >= nr || inst == i0) && tiled;
    if(tiled)
    {
        if constexpr(sizeof(T) == 4)
        {
            float*         tile = s_tile[wib];
            const unsigned sh   = static_cast<unsigned>(__ffs(static_cast<int>(g0))) - 1u; // log2(g0)
            const unsigned n4   = nr * g0 / 4u;                                           // float4 of the tile
            const float4*  src  = reinterpret_cast<const float4*>(in + base);
            for(unsigned e4 = lane; e4 < n4; e4 += 32u)
            {
                const float4   v   = __ldg(src + e4);
                const unsigned e   = 4u * e4;
                const unsigned row = e >> sh;
                const unsigned j   = e & (g0 - 1u);
                float*         d   = tile + row * (g0 + 1u) + j;
                d[0]               = v.x;
                d[1]               = v.y;
                d[2]               = v.z;
                d[3]               = v.w;
            }
            __syncwarp();
            if(lane < nr)
            {
                const float* row = tile + lane * (g0 + 1u);
                float        acc = 0.0f;
                for(unsigned j = 0; j < g0; ++j) acc = acc + row[j];
                out[r] = static_cast<T>(acc / static_cast<float>(g0));
            }
        }
        return;
    }
    if(lane >= nr) return;
    T acc = T(0);
    for(unsigned j = 0; j < g; ++j) acc = acc + __ldg(in + t0 + j);
    out[r] = acc / static_cast<T>(g);
}

/// Grid of group_mean over `rows` rows.
unsigned
mean_blocks(const unsigned long long rows)
{
    return static_cast<unsigned>((rows + 32ull * kMeanWarps - 1) / (32ull * kMeanWarps));
}

/// Launch counters: 8 totals, then thread and warp instructions per block.
size_t
counter_bytes(const KernelEntry& e)
{
    return (8 + 2 * static_cast<size_t>(e.info->num_blocks)) * sizeof(unsigned long long);
}

constexpr unsigned long long kDefaultMaxSteps    = 1ull << 40;
constexpr unsigned long long kBarrierSpins       = 1ull << 25;
constexpr unsigned long long kDefaultStateBudget = 8ull << 30; // queue state bytes
constexpr unsigned           kDefaultPlainBlock  = 256;
constexpr unsigned           kDefaultRegroupBlock = 256;
constexpr unsigned           kDefaultUtr         = 16;
constexpr unsigned           kDefaultPeriod      = 1024;
constexpr unsigned           kDefaultBurst       = 32;
constexpr unsigned           kDefaultSpread      = 33;
constexpr unsigned           kMaxDynSmem         = 227u * 1024u; // shared memory one CTA may use
} // namespace

struct loom_b200_handle
{
    const KernelEntry* e = nullptr;
    loom_b200_opts     opts{};
    uint64_t           capacity = 0;
    int                device   = 0;
    int                sms      = 0;
    cudaStream_t       stream   = nullptr;
    cudaEvent_t        ev0 = nullptr, ev1 = nullptr;

    // staging columns for run_host
    std::vector<void*> d_in, d_out;
    // device bookkeeping
    unsigned*           d_status   = nullptr;
    unsigned long long* d_counters = nullptr; // 8 counters, then 2 per block (profiled launches)
    // regrouping workspace: the queues with their state, sized for `ws_cap`
    // entries per queue
    uint64_t            ws_cap  = 0;
    char*               d_state = nullptr;
    unsigned*           d_qcnt  = nullptr;
    unsigned*           d_qhead = nullptr;
    RegroupCtl*         d_ctl   = nullptr;

    // device copies of instance starts and table for launch_host
    void*  d_starts     = nullptr;
    size_t starts_bytes = 0;
    void*  d_table      = nullptr;
    size_t table_bytes  = 0;
    // launch_host_mean: the rows of the group means (and their offsets)
    void*  d_rows       = nullptr;
    size_t rows_bytes   = 0;
    // launch_host pipeline: copy streams and one event per stage of a chunk
    cudaStream_t             s_in = nullptr, s_out = nullptr;
    std::vector<cudaEvent_t> chunk_ev;

    // CUDA graph of the regrouping launch sequence (opts.graph)
    cudaStream_t    cap_stream   = nullptr;
    cudaGraphExec_t graph_exec   = nullptr;
    RegroupLaunch   graph_key{};
    uint64_t        graph_admit  = 0;
    bool            graph_broken = false; // capture refused: launch directly

    loom_b200_stats stats{};
    unsigned        last_grid     = 0;
    uint64_t        last_cap      = 0; // queue capacity of the last launch (0: plain)
    bool            pending       = false; // launched, counters not read yet
    uint64_t        launches      = 0;
    uint64_t        plain_threads = 0;
};

namespace
{
void
free_ws(loom_b200_handle* h)
{
    cudaFree(h->d_state);
    cudaFree(h->d_qcnt);
    cudaFree(h->d_qhead);
    h->d_state = nullptr;
    h->d_qcnt = h->d_qhead = nullptr;
    h->ws_cap = 0;
}

/// Population rounded up to whole tiles (keeps every queue column aligned).
uint64_t
round_cap(uint64_t cap)
{
    return (cap + 31) / 32 * 32;
}

/// Whether a regrouping launch never parks a thread: schedules 2 and 3 with
/// no period limit keep every thread in its lane until it halts.
bool
never_parks(const loom_b200_opts& o)
{
    return o.mode == LOOM_B200_REGROUP && (o.schedule == 2u || o.schedule == 3u) &&
           o.period == LOOM_B200_PERIOD_UNBOUNDED;
}

/// Whether a regrouping launch runs the megakernel's parking form: every
/// launch but those that never park and do not prefetch (the never-park
/// form is compiled without prefetch).
bool
park_form(const loom_b200_opts& o)
{
    return !(never_parks(o) && o.no_prefetch);
}

/// Threads in flight of a regrouping launch: the requested population, or
/// as many as the queue state of kDefaultStateBudget bytes holds.  A launch
/// that never parks keeps its threads in registers: its queues get one tile
/// each, which nothing writes, and it admits every input in its one round.
uint64_t
population(const loom_b200_handle* h, uint64_t n)
{
    if(never_parks(h->opts)) return 32;
    uint64_t p = h->opts.population ? h->opts.population : n;
    const uint64_t fit = kDefaultStateBudget / (2 * h->e->row_bytes) / 32 * 32;
    if(!h->opts.population && fit && p > fit) p = fit;
    return round_cap(std::min<uint64_t>(p, n));
}

int
ensure_ws(loom_b200_handle* h, uint64_t cap)
{
    if(cap <= h->ws_cap) return LOOM_B200_OK;
    free_ws(h);
    const KernelEntry& e = *h->e;
    const uint64_t     B = e.num_queues;
    LB_CUDA(cudaMalloc(&h->d_state, 2 * e.row_bytes * cap));
    LB_CUDA(cudaMalloc(&h->d_qcnt, 2 * B * sizeof(unsigned)));
    LB_CUDA(cudaMalloc(&h->d_qhead, B * sizeof(unsigned)));
    h->ws_cap = cap;
    return LOOM_B200_OK;
}

/// Grows a device buffer to at least `bytes` (contents are not kept).
int
grow(void** p, size_t* have, size_t bytes)
{
    if(bytes <= *have) return LOOM_B200_OK;
    cudaFree(*p);
    *p    = nullptr;
    *have = 0;
    LB_CUDA(cudaMalloc(p, bytes));
    *have = bytes;
    return LOOM_B200_OK;
}

void
normalise(loom_b200_opts& o)
{
    if(o.block_size == 0 || o.block_size % 32 != 0 || o.block_size > 1024)
        o.block_size = o.mode == LOOM_B200_REGROUP ? kDefaultRegroupBlock
                                                   : kDefaultPlainBlock;
    if(o.utr_lanes == 0 || o.utr_lanes > 32) o.utr_lanes = kDefaultUtr;
    if(o.period == 0) o.period = kDefaultPeriod;
    if(o.burst == 0) o.burst = kDefaultBurst;
    if(o.spread_lanes == 0) o.spread_lanes = kDefaultSpread;
    if(o.max_steps == 0) o.max_steps = kDefaultMaxSteps;
}

int
finish_launch(loom_b200_handle* h)
{
    if(!h->pending) return h->stats.status ? LOOM_B200_ERR_DEVICE : LOOM_B200_OK;
    LB_CUDA(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    LB_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    unsigned long long c[8];
    unsigned           status = 0;
    LB_CUDA(cudaMemcpy(c, h->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
    LB_CUDA(cudaMemcpy(&status, h->d_status, sizeof(status), cudaMemcpyDeviceToHost));
    loom_b200_stats& s = h->stats;
    s.launches     = h->launches;
    s.thread_instr = c[0];
    s.warp_instr   = c[1];
    s.parks        = c[2];
    s.state_bytes  = c[3];
    s.rounds       = c[5];
    s.threads      = c[4] + h->plain_threads;
    s.status       = status;
    s.grid         = h->last_grid;
    s.ms           = ms;
    h->pending     = false;
    return status ? LOOM_B200_ERR_DEVICE : LOOM_B200_OK;
}

/// The regrouping launch sequence (queue reset, engine kernel) as a CUDA
/// graph: captured on first use, replayed while the launch arguments stay
/// the same, re-captured when they change.  Where capture is refused the
/// handle falls back to direct launches for good.
int
launch_graph(loom_b200_handle* h, const RegroupLaunch& L, uint64_t admit, cudaStream_t stream)
{
    const uint64_t first = L.params.cols.tid_base;
    const bool same = h->graph_exec && h->graph_admit == admit && h->graph_key.grid == L.grid &&
                      h->graph_key.block == L.block && h->graph_key.profile == L.profile &&
                      h->graph_key.regs == L.regs &&
                      std::memcmp(&h->graph_key.params, &L.params, sizeof(RegroupParams)) == 0;
    if(!same)
    {
        if(h->graph_exec)
        {
            cudaGraphExecDestroy(h->graph_exec);
            h->graph_exec = nullptr;
        }
        if(!h->cap_stream && cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking) != cudaSuccess)
        {
            h->graph_broken = true;
            return LOOM_B200_ERR_CUDA;
        }
        RegroupLaunch C = L;
        C.stream        = h->cap_stream;
        cudaGraph_t g   = nullptr;
        cudaError_t err = cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal);
        if(err == cudaSuccess)
        {
            regroup_reset<<<1, 256, 0, h->cap_stream>>>(h->d_ctl, h->d_qcnt, h->d_qhead,
                                                        h->e->num_queues, first, admit);
            cudaError_t e1 = cudaGetLastError();
            cudaError_t e2 = h->e->regroup(C);
            cudaError_t e3 = cudaStreamEndCapture(h->cap_stream, &g);
            err            = e1 != cudaSuccess ? e1 : e2 != cudaSuccess ? e2 : e3;
        }
        if(err == cudaSuccess) err = cudaGraphInstantiate(&h->graph_exec, g, 0);
        if(g) cudaGraphDestroy(g);
        if(err != cudaSuccess)
        {
            cudaGetLastError(); // the refusal is not an error of the launch
            h->graph_exec   = nullptr;
            h->graph_broken = true;
            return LOOM_B200_ERR_CUDA;
        }
        h->graph_key   = L;
        h->graph_admit = admit;
        h->stats.graph_captures += 1;
    }
    LB_CUDA(cudaGraphLaunch(h->graph_exec, stream));
    h->stats.graph_launches += 1;
    return LOOM_B200_OK;
}

/// Launch with every pointer of `L` on the device: Loom threads
/// [first, first + L.n), inputs and outputs indexed by the thread id.
/// `graph` allows the regrouping launch to replay a CUDA graph.
int
launch(loom_b200_handle* h, const loom_b200_launch& L, cudaStream_t stream, uint64_t first = 0, bool graph = true)
{
    const KernelEntry&           e    = *h->e;
    const loom_b200_kernel_info& info = *e.info;
    const uint64_t               n    = L.n;
    if(n == 0) return LOOM_B200_OK;
    if(n >= (1ull << 32))
    {
        g_last_error = "at most 2^32 - 1 threads per launch";
        return LOOM_B200_ERR_INVALID;
    }
    if(info.num_inputs > static_cast<uint32_t>(kMaxIn) ||
       info.num_inputs + info.num_outputs > static_cast<uint32_t>(kMaxCols))
    {
        g_last_error = "too many columns";
        return LOOM_B200_ERR_INVALID;
    }
    Columns cols{};
    int     c = 0;
    for(uint32_t i = 0; i < info.num_inputs; ++i)
    {
        const loom_b200_input& in = L.inputs[i];
        if(in.form > LOOM_B200_IN_INSTANCE ||
           (in.form == LOOM_B200_IN_ARRAY && in.ptr == nullptr))
        {
            g_last_error = "bad input column";
            return LOOM_B200_ERR_INVALID;
        }
        cols.form[i]  = in.form;
        cols.value[i] = in.value;
        cols.p[c++]   = const_cast<void*>(in.ptr);
    }
    for(uint32_t i = 0; i < info.num_outputs; ++i)
    {
        if(L.outputs[i] == nullptr)
        {
            g_last_error = "output column is NULL";
            return LOOM_B200_ERR_INVALID;
        }
        cols.p[c++] = L.outputs[i];
    }
    cols.inst_start = reinterpret_cast<const unsigned long long*>(L.instance_starts);
    cols.num_inst   = L.instance_starts ? L.num_instances : 0u;
    cols.table      = L.table;
    cols.tid_base   = first; // thread ids in flight lie in [first, first + n)
    const loom_b200_opts& o = h->opts;
    // a regrouping handle runs launches below plain_below threads on the
    // plain engine (the persistent megakernel does not pay for them)
    const bool regroup = o.mode == LOOM_B200_REGROUP && n >= o.plain_below;
    if(regroup)
    {
        // the workspace is reallocated only between launches
        const uint64_t cap = population(h, n);
        if(cap > h->ws_cap)
        {
            LB_CUDA(cudaStreamSynchronize(stream));
            const int rc = ensure_ws(h, cap);
            if(rc) return rc;
        }
    }
    LB_CUDA(cudaEventRecord(h->ev0, stream));
    if(regroup)
    {
        const uint64_t cap = population(h, n);
        // the largest CTA size up to the requested one that fits on an SM
        unsigned block = o.block_size;
        int      ctas  = 0;
        for(;;)
        {
            const unsigned    dyn = o.bulk_restore ? bulk_stage_bytes(block / 32u, e.max_stage_row) : 0u;
            const cudaError_t oe  = dyn > kMaxDynSmem ? cudaErrorInvalidValue
                                                      : e.regroup_occupancy(static_cast<int>(block), o.profile != 0,
                                                                            o.max_regs, dyn, park_form(o), &ctas);
            if(oe == cudaErrorInvalidValue && dyn > kMaxDynSmem && block > 32)
            {
                block /= 2; // the staging area of this many warps does not fit
                continue;
            }
            if(oe == cudaErrorInvalidValue)
            {
                g_last_error = dyn ? "bulk_restore: the staging area does not fit in shared memory"
                                   : "register cap not compiled for this kernel (loom_b200_kernel_reg_caps)";
                return LOOM_B200_ERR_INVALID;
            }
            LB_CUDA(oe);
            if(ctas > 0 || block <= 32) break;
            block /= 2;
        }
        if(ctas <= 0)
        {
            g_last_error = "regroup kernel does not fit on an SM";
            return LOOM_B200_ERR_INVALID;
        }
        if(o.ctas_per_sm) ctas = std::min<int>(ctas, static_cast<int>(o.ctas_per_sm));
        RegroupLaunch L{};
        L.params.cols          = cols;
        L.params.state         = h->d_state;
        L.params.qcnt          = h->d_qcnt;
        L.params.qhead         = h->d_qhead;
        L.params.ctl           = h->d_ctl;
        L.params.status        = h->d_status;
        L.params.counters      = h->d_counters;
        L.params.n             = first + n; // end of the thread range
        L.params.max_rounds    = o.max_steps;
        L.params.barrier_spins = o.barrier_spins ? o.barrier_spins : kBarrierSpins;
        L.params.phantoms      = o.fault_phantom_ctas;
        L.params.cap           = static_cast<unsigned>(cap);
        L.params.utr           = o.utr_lanes;
        L.params.period        = o.period;
        L.params.burst         = o.burst;
        L.params.spread        = o.spread_lanes;
        L.params.refill        = o.no_refill ? 0u : 1u;
        L.params.prefetch      = o.no_prefetch ? 0u : 1u;
        L.params.cost_model    = o.cost_model;
        L.params.schedule      = o.schedule;
        L.params.defer_lanes   = o.defer_lanes;
        L.params.bulk_restore  = o.bulk_restore;
        L.params.spin_iters    = o.spin_iters;
        L.params.refill_lanes  = o.refill_lanes;
        L.dyn_smem             = o.bulk_restore ? bulk_stage_bytes(block / 32u, e.max_stage_row) : 0u;
        L.grid                 = static_cast<unsigned>(ctas * h->sms);
        L.block                = block;
        L.regs                 = o.max_regs;
        L.park                 = park_form(o);
        L.profile              = o.profile != 0;
        L.stream               = stream;
        const uint64_t admit = first + (never_parks(o) ? n : std::min<uint64_t>(n, cap));
        if(!(graph && o.graph && !h->graph_broken && launch_graph(h, L, admit, stream) == LOOM_B200_OK))
        {
            regroup_reset<<<1, 256, 0, stream>>>(h->d_ctl, h->d_qcnt, h->d_qhead, e.num_queues, first, admit);
            LB_CUDA(cudaGetLastError());
            LB_CUDA(e.regroup(L));
        }
        h->last_grid = L.grid;
        h->last_cap  = cap;
    }
    else
    {
        h->last_cap = 0;
        PlainLaunch L{};
        L.cols      = cols;
        L.first     = first;
        L.n         = n;
        L.max_steps = o.mode == LOOM_B200_REGROUP ? kDefaultMaxSteps : o.max_steps; // regroup: max_steps counts rounds
        L.status    = h->d_status;
        L.counters  = h->d_counters;
        L.block     = o.block_size;
        L.profile   = o.profile != 0;
        L.stream    = stream;
        LB_CUDA(e.plain(L));
        h->last_grid = static_cast<unsigned>((n + o.block_size - 1) / o.block_size);
        h->plain_threads += n;
    }
    LB_CUDA(cudaEventRecord(h->ev1, stream));
    h->pending = true;
    h->launches += 1;
    return LOOM_B200_OK;
}
} // namespace

extern "C" {

int
loom_b200_version(void)
{
    return LOOM_B200_ABI_VERSION;
}

const char*
loom_b200_error_string(int code)
{
    switch(code)
    {
    case LOOM_B200_OK: return "ok";
    case LOOM_B200_ERR_INVALID:
        return g_last_error.empty() ? "invalid argument" : g_last_error.c_str();
    case LOOM_B200_ERR_NOT_FOUND: return "kernel not compiled into libloom_b200";
    case LOOM_B200_ERR_CUDA:
    case LOOM_B200_ERR_OOM:
    case LOOM_B200_ERR_NO_DEVICE:
        return g_last_error.empty() ? "CUDA error" : g_last_error.c_str();
    case LOOM_B200_ERR_DEVICE: return "device status word set (see stats.status)";
    case LOOM_B200_ERR_BUDGET: return "request exceeds the device memory budget";
    case LOOM_B200_ERR_CANCELLED: return "request cancelled";
    case LOOM_B200_ERR_TIMEOUT: return "watchdog expired";
    default: return "unknown error";
    }
}

int
loom_b200_kernel_count(void)
{
    return kRegistrySize;
}

int
loom_b200_kernel_get(int index, const loom_b200_kernel_info** info)
{
    if(!info || index < 0 || index >= kRegistrySize) return LOOM_B200_ERR_INVALID;
    *info = kRegistry[index]->info;
    return LOOM_B200_OK;
}

int
loom_b200_kernel_find(const char* name, const loom_b200_kernel_info** info)
{
    if(!name || !info) return LOOM_B200_ERR_INVALID;
    for(int i = 0; i < kRegistrySize; ++i)
        if(std::strcmp(kRegistry[i]->info->name, name) == 0)
        {
            *info = kRegistry[i]->info;
            return LOOM_B200_OK;
        }
    return LOOM_B200_ERR_NOT_FOUND;
}

int
loom_b200_kernel_find_digest(const char* digest, const loom_b200_kernel_info** info)
{
    if(!digest || !info) return LOOM_B200_ERR_INVALID;
    for(int i = 0; i < kRegistrySize; ++i)
        if(std::strcmp(kRegistry[i]->info->ir_digest, digest) == 0)
        {
            *info = kRegistry[i]->info;
            return LOOM_B200_OK;
        }
    return LOOM_B200_ERR_NOT_FOUND;
}

int
loom_b200_create(const char*           kernel,
                 uint64_t              capacity,
                 const loom_b200_opts* opts,
                 loom_b200_handle**    out)
{
    if(!kernel || !out) return LOOM_B200_ERR_INVALID;
    *out = nullptr;
    const KernelEntry* e = nullptr;
    for(int i = 0; i < kRegistrySize; ++i)
        if(std::strcmp(kRegistry[i]->info->name, kernel) == 0) e = kRegistry[i];
    if(!e) return LOOM_B200_ERR_NOT_FOUND;
    int ndev = 0;
    const cudaError_t ce = cudaGetDeviceCount(&ndev);
    if(ce != cudaSuccess || ndev == 0)
    {
        g_last_error = ce != cudaSuccess ? cudaGetErrorString(ce) : "no CUDA device";
        return LOOM_B200_ERR_NO_DEVICE;
    }
    auto* h = new(std::nothrow) loom_b200_handle();
    if(!h) return LOOM_B200_ERR_OOM;
    h->e        = e;
    h->capacity = capacity;
    if(opts) h->opts = *opts;
    normalise(h->opts);
    auto fail = [&](int rc)
    {
        loom_b200_destroy(h);
        return rc;
    };
    if(cudaGetDevice(&h->device) != cudaSuccess) return fail(LOOM_B200_ERR_CUDA);
    if(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device) !=
       cudaSuccess)
        return fail(LOOM_B200_ERR_CUDA);
    if(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
       cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess)
        return fail(LOOM_B200_ERR_CUDA);
    if(cudaMalloc(&h->d_status, sizeof(unsigned)) != cudaSuccess ||
       cudaMalloc(&h->d_counters, counter_bytes(*e)) != cudaSuccess ||
       cudaMalloc(&h->d_ctl, sizeof(RegroupCtl)) != cudaSuccess)
        return fail(LOOM_B200_ERR_OOM);
    if(cudaMemset(h->d_counters, 0, counter_bytes(*e)) != cudaSuccess ||
       cudaMemset(h->d_status, 0, sizeof(unsigned)) != cudaSuccess)
        return fail(LOOM_B200_ERR_CUDA);
    const loom_b200_kernel_info& info = *e->info;
    h->d_in.assign(info.num_inputs, nullptr);
    h->d_out.assign(info.num_outputs, nullptr);
    if(capacity)
    {
        for(uint32_t i = 0; i < info.num_inputs; ++i)
            if(cudaMalloc(&h->d_in[i], capacity * type_bytes(info.input_types[i])) !=
               cudaSuccess)
                return fail(LOOM_B200_ERR_OOM);
        for(uint32_t i = 0; i < info.num_outputs; ++i)
            if(cudaMalloc(&h->d_out[i], capacity * type_bytes(info.output_types[i])) !=
               cudaSuccess)
                return fail(LOOM_B200_ERR_OOM);
    }
    *out = h;
    return LOOM_B200_OK;
}

int
loom_b200_destroy(loom_b200_handle* h)
{
    if(!h) return LOOM_B200_OK;
    if(h->stream) cudaStreamSynchronize(h->stream);
    free_ws(h);
    for(void* p: h->d_in) cudaFree(p);
    for(void* p: h->d_out) cudaFree(p);
    cudaFree(h->d_status);
    cudaFree(h->d_counters);
    cudaFree(h->d_starts);
    cudaFree(h->d_table);
    cudaFree(h->d_rows);
    cudaFree(h->d_ctl);
    for(cudaEvent_t ev: h->chunk_ev) cudaEventDestroy(ev);
    if(h->s_in) cudaStreamDestroy(h->s_in);
    if(h->s_out) cudaStreamDestroy(h->s_out);
    if(h->ev0) cudaEventDestroy(h->ev0);
    if(h->ev1) cudaEventDestroy(h->ev1);
    if(h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    if(h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if(h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return LOOM_B200_OK;
}

int
loom_b200_set_opts(loom_b200_handle* h, const loom_b200_opts* opts)
{
    if(!h || !opts) return LOOM_B200_ERR_INVALID;
    if(h->pending)
    {
        const int rc = finish_launch(h);
        if(rc != LOOM_B200_OK && rc != LOOM_B200_ERR_DEVICE) return rc;
    }
    h->opts = *opts;
    normalise(h->opts);
    return LOOM_B200_OK;
}

int
loom_b200_get_opts(const loom_b200_handle* h, loom_b200_opts* opts)
{
    if(!h || !opts) return LOOM_B200_ERR_INVALID;
    *opts = h->opts;
    return LOOM_B200_OK;
}

int
loom_b200_launch_device(loom_b200_handle* h, const loom_b200_launch* L, void* stream)
{
    if(!h || !L || (!L->inputs && h->e->info->num_inputs) || !L->outputs)
        return LOOM_B200_ERR_INVALID;
    return launch(h, *L, static_cast<cudaStream_t>(stream));
}

namespace
{
/// Copies the instance offsets and the table of a host launch to the
/// handle's device buffers on `st` and points `D` at them.
int
stage_tables(loom_b200_handle* h, const loom_b200_launch& L, loom_b200_launch& D, cudaStream_t st)
{
    if(L.instance_starts)
    {
        const size_t bytes = (static_cast<size_t>(L.num_instances) + 1) * sizeof(uint64_t);
        int rc = grow(&h->d_starts, &h->starts_bytes, bytes);
        if(rc) return rc;
        LB_CUDA(cudaMemcpyAsync(h->d_starts, L.instance_starts, bytes, cudaMemcpyHostToDevice, st));
        D.instance_starts = static_cast<const uint64_t*>(h->d_starts);
    }
    if(L.table)
    {
        const size_t bytes = L.table_words * sizeof(uint32_t);
        int rc = grow(&h->d_table, &h->table_bytes, bytes);
        if(rc) return rc;
        LB_CUDA(cudaMemcpyAsync(h->d_table, L.table, bytes, cudaMemcpyHostToDevice, st));
        D.table = static_cast<const uint32_t*>(h->d_table);
    }
    return LOOM_B200_OK;
}

/// Chunks of a host launch: 1 when the host copies are small, else enough
/// that each chunk's copies overlap the neighbouring chunks' kernels.
uint64_t
host_chunks(const loom_b200_handle* h, uint64_t n, uint64_t copy_bytes)
{
    uint64_t c = h->opts.host_chunks ? h->opts.host_chunks : (copy_bytes >= (32ull << 20) ? 8 : 1);
    c = std::min<uint64_t>(c, std::max<uint64_t>(1, n / 1024));
    return std::max<uint64_t>(c, 1);
}

int
ensure_copy_streams(loom_b200_handle* h, size_t events)
{
    if(!h->s_in) LB_CUDA(cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking));
    if(!h->s_out) LB_CUDA(cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking));
    while(h->chunk_ev.size() < events)
    {
        cudaEvent_t ev = nullptr;
        LB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        h->chunk_ev.push_back(ev);
    }
    return LOOM_B200_OK;
}
} // namespace

int
loom_b200_launch_host(loom_b200_handle* h, const loom_b200_launch* L)
{
    if(!h || !L || (!L->inputs && h->e->info->num_inputs) || !L->outputs)
        return LOOM_B200_ERR_INVALID;
    const uint64_t n = L->n;
    if(n > h->capacity)
    {
        g_last_error = "n exceeds the handle's capacity";
        return LOOM_B200_ERR_INVALID;
    }
    if(n == 0) return LOOM_B200_OK;
    const loom_b200_kernel_info& info = *h->e->info;
    std::vector<loom_b200_input> din(L->inputs, L->inputs + info.num_inputs);
    uint64_t                     per_thread = 0;
    for(uint32_t i = 0; i < info.num_inputs; ++i)
        if(din[i].form == LOOM_B200_IN_ARRAY && din[i].ptr) per_thread += type_bytes(info.input_types[i]);
    for(uint32_t j = 0; j < info.num_outputs; ++j) per_thread += type_bytes(info.output_types[j]);
    const uint64_t chunks = host_chunks(h, n, n * per_thread);

    // Pipeline of `chunks` ranges of threads: the inputs of range k go in on
    // s_in, its kernel runs on the handle's stream once they arrived, its
    // outputs come back on s_out once it finished, so range k's copies
    // overlap the kernels of ranges k - 1 and k + 1.  One range is the plain
    // sequence copy in, launch, copy out.
    if(chunks > 1)
    {
        const int rc = ensure_copy_streams(h, 2 * chunks + 1);
        if(rc) return rc;
    }
    cudaStream_t s_in  = chunks > 1 ? h->s_in : h->stream;
    cudaStream_t s_out = chunks > 1 ? h->s_out : h->stream;
    loom_b200_launch D = *L;
    for(uint32_t i = 0; i < info.num_inputs; ++i)
        if(din[i].form == LOOM_B200_IN_ARRAY && din[i].ptr) din[i].ptr = h->d_in[i];
    D.inputs  = din.data();
    D.outputs = h->d_out.data();
    if(int rc = stage_tables(h, *L, D, s_in)) return rc;
    const uint64_t step = (n + chunks - 1) / chunks;
    for(uint64_t k = 0; k < chunks; ++k)
    {
        const uint64_t a = k * step, b = std::min<uint64_t>(n, a + step);
        if(a >= b) break;
        for(uint32_t i = 0; i < info.num_inputs; ++i)
            if(L->inputs[i].form == LOOM_B200_IN_ARRAY && L->inputs[i].ptr)
            {
                const size_t eb = type_bytes(info.input_types[i]);
                LB_CUDA(cudaMemcpyAsync(static_cast<char*>(h->d_in[i]) + a * eb,
                                        static_cast<const char*>(L->inputs[i].ptr) + a * eb,
                                        (b - a) * eb, cudaMemcpyHostToDevice, s_in));
            }
        if(chunks > 1)
        {
            LB_CUDA(cudaEventRecord(h->chunk_ev[2 * k], s_in));
            LB_CUDA(cudaStreamWaitEvent(h->stream, h->chunk_ev[2 * k], 0));
        }
        loom_b200_launch C = D;
        C.n                = b - a;
        if(int rc = launch(h, C, h->stream, a, chunks == 1)) return rc;
        if(chunks > 1)
        {
            LB_CUDA(cudaEventRecord(h->chunk_ev[2 * k + 1], h->stream));
            LB_CUDA(cudaStreamWaitEvent(s_out, h->chunk_ev[2 * k + 1], 0));
        }
        for(uint32_t j = 0; j < info.num_outputs; ++j)
        {
            const size_t eb = type_bytes(info.output_types[j]);
            LB_CUDA(cudaMemcpyAsync(static_cast<char*>(L->outputs[j]) + a * eb,
                                    static_cast<const char*>(h->d_out[j]) + a * eb, (b - a) * eb,
                                    cudaMemcpyDeviceToHost, s_out));
        }
    }
    LB_CUDA(cudaStreamSynchronize(s_out));
    LB_CUDA(cudaStreamSynchronize(h->stream));
    return finish_launch(h);
}

int
loom_b200_group_mean(uint32_t type, const void* in, void* out, uint64_t rows, uint32_t group, void* stream)
{
    if(!in || !out || group == 0 || (type != LOOM_B200_F32 && type != LOOM_B200_F64))
        return LOOM_B200_ERR_INVALID;
    if(rows == 0) return LOOM_B200_OK;
    const unsigned blocks = mean_blocks(rows);
    auto           st     = static_cast<cudaStream_t>(stream);
    if(type == LOOM_B200_F32)
        group_mean<float><<<blocks, 32 * kMeanWarps, 0, st>>>(static_cast<const float*>(in), static_cast<float*>(out),
                                                             rows, group, nullptr, nullptr, nullptr, 0u);
    else
        group_mean<double><<<blocks, 32 * kMeanWarps, 0, st>>>(static_cast<const double*>(in), static_cast<double*>(out),
                                                   rows, group, nullptr, nullptr, nullptr, 0u);
    LB_CUDA(cudaGetLastError());
    return LOOM_B200_OK;
}

int
loom_b200_launch_host_mean(loom_b200_handle* h, const loom_b200_launch* L, const loom_b200_mean* M)
{
    if(!h || !L || !M || (!L->inputs && h->e->info->num_inputs) || !L->outputs)
        return LOOM_B200_ERR_INVALID;
    const uint64_t               n    = L->n;
    const loom_b200_kernel_info& info = *h->e->info;
    if(n > h->capacity)
    {
        g_last_error = "n exceeds the handle's capacity";
        return LOOM_B200_ERR_INVALID;
    }
    for(uint32_t j = 0; j < info.num_outputs; ++j)
        if(info.output_types[j] != LOOM_B200_F32 && info.output_types[j] != LOOM_B200_F64)
        {
            g_last_error = "group means need float outputs";
            return LOOM_B200_ERR_INVALID;
        }
    // output rows: per instance its threads / its group, in instance order
    std::vector<unsigned long long> out_starts;
    uint64_t                        rows = 0;
    if(M->instance_group)
    {
        if(!L->instance_starts || L->num_instances == 0)
        {
            g_last_error = "instance_group needs instance_starts";
            return LOOM_B200_ERR_INVALID;
        }
        out_starts.resize(L->num_instances + 1);
        for(uint32_t i = 0; i < L->num_instances; ++i)
        {
            const uint64_t t = L->instance_starts[i + 1] - L->instance_starts[i];
            const uint32_t g = M->instance_group[i];
            if(g == 0 || t % g != 0)
            {
                g_last_error = "an instance's threads are not a multiple of its group";
                return LOOM_B200_ERR_INVALID;
            }
            out_starts[i] = rows;
            rows += t / g;
        }
        out_starts[L->num_instances] = rows;
        if(L->instance_starts[L->num_instances] != n)
        {
            g_last_error = "instance_starts must end at n";
            return LOOM_B200_ERR_INVALID;
        }
    }
    else
    {
        if(M->group == 0 || n % M->group != 0)
        {
            g_last_error = "n is not a multiple of the group";
            return LOOM_B200_ERR_INVALID;
        }
        rows = n / M->group;
    }
    if(n == 0) return LOOM_B200_OK;

    std::vector<loom_b200_input> din(L->inputs, L->inputs + info.num_inputs);
    for(uint32_t i = 0; i < info.num_inputs; ++i)
        if(din[i].form == LOOM_B200_IN_ARRAY && din[i].ptr)
        {
            LB_CUDA(cudaMemcpyAsync(h->d_in[i], din[i].ptr, n * type_bytes(info.input_types[i]),
                                    cudaMemcpyHostToDevice, h->stream));
            din[i].ptr = h->d_in[i];
        }
    loom_b200_launch D = *L;
    D.inputs           = din.data();
    D.outputs          = h->d_out.data();
    if(int rc = stage_tables(h, *L, D, h->stream)) return rc;
    if(int rc = launch(h, D, h->stream)) return rc;

    // the reduction: row buffers, and for instances the row offsets and
    // group sizes, all in one device buffer
    size_t row_bytes = 0;
    for(uint32_t j = 0; j < info.num_outputs; ++j) row_bytes += rows * type_bytes(info.output_types[j]);
    const size_t meta = M->instance_group ? (out_starts.size() * 8 + L->num_instances * 4) : 0;
    if(int rc = grow(&h->d_rows, &h->rows_bytes, (row_bytes + 255) / 256 * 256 + meta)) return rc;
    char*                     base = static_cast<char*>(h->d_rows);
    const unsigned long long* d_os = nullptr;
    const unsigned*           d_g  = nullptr;
    if(meta)
    {
        char* m = base + (row_bytes + 255) / 256 * 256;
        LB_CUDA(cudaMemcpyAsync(m, out_starts.data(), out_starts.size() * 8, cudaMemcpyHostToDevice, h->stream));
        LB_CUDA(cudaMemcpyAsync(m + out_starts.size() * 8, M->instance_group, L->num_instances * 4,
                                cudaMemcpyHostToDevice, h->stream));
        d_os = reinterpret_cast<const unsigned long long*>(m);
        d_g  = reinterpret_cast<const unsigned*>(m + out_starts.size() * 8);
    }
    const auto*    d_st   = static_cast<const unsigned long long*>(h->d_starts);
    const unsigned blocks = mean_blocks(rows);
    size_t         off    = 0;
    for(uint32_t j = 0; j < info.num_outputs; ++j)
    {
        const size_t eb = type_bytes(info.output_types[j]);
        if(info.output_types[j] == LOOM_B200_F32)
            group_mean<float><<<blocks, 32 * kMeanWarps, 0, h->stream>>>(
                static_cast<const float*>(h->d_out[j]), reinterpret_cast<float*>(base + off), rows, M->group,
                d_os ? d_st : nullptr, d_g, d_os, d_os ? L->num_instances : 0u);
        else
            group_mean<double><<<blocks, 32 * kMeanWarps, 0, h->stream>>>(
                static_cast<const double*>(h->d_out[j]), reinterpret_cast<double*>(base + off), rows, M->group,
                d_os ? d_st : nullptr, d_g, d_os, d_os ? L->num_instances : 0u);
        LB_CUDA(cudaGetLastError());
        LB_CUDA(cudaMemcpyAsync(L->outputs[j], base + off, rows * eb, cudaMemcpyDeviceToHost, h->stream));
        off += rows * eb;
    }
    LB_CUDA(cudaStreamSynchronize(h->stream));
    return finish_launch(h);
}

int
loom_b200_run_host(loom_b200_handle*  h,
                   const void* const* inputs,
                   void* const*       outputs,
                   uint64_t           n)
{
    if(!h || (!inputs && h->e->info->num_inputs) || !outputs)
        return LOOM_B200_ERR_INVALID;
    std::vector<loom_b200_input> in(h->e->info->num_inputs);
    for(size_t i = 0; i < in.size(); ++i)
        in[i] = loom_b200_input{inputs[i],
                                inputs[i] ? LOOM_B200_IN_ARRAY : LOOM_B200_IN_IOTA,
                                0u,
                                0ull};
    loom_b200_launch L{};
    L.inputs  = in.data();
    L.outputs = outputs;
    L.n       = n;
    return loom_b200_launch_host(h, &L);
}

int
loom_b200_run_device(loom_b200_handle*  h,
                     const void* const* inputs,
                     void* const*       outputs,
                     uint64_t           n,
                     void*              stream)
{
    if(!h || (!inputs && h->e->info->num_inputs) || !outputs)
        return LOOM_B200_ERR_INVALID;
    std::vector<loom_b200_input> in(h->e->info->num_inputs);
    for(size_t i = 0; i < in.size(); ++i)
        in[i] = loom_b200_input{inputs[i],
                                inputs[i] ? LOOM_B200_IN_ARRAY : LOOM_B200_IN_IOTA,
                                0u,
                                0ull};
    loom_b200_launch L{};
    L.inputs  = in.data();
    L.outputs = outputs;
    L.n       = n;
    return launch(h, L, static_cast<cudaStream_t>(stream));
}

int
loom_b200_sync(loom_b200_handle* h)
{
    if(!h) return LOOM_B200_ERR_INVALID;
    return finish_launch(h);
}

int
loom_b200_get_stats(loom_b200_handle* h, loom_b200_stats* stats)
{
    if(!h || !stats) return LOOM_B200_ERR_INVALID;
    const int rc = finish_launch(h);
    if(rc != LOOM_B200_OK && rc != LOOM_B200_ERR_DEVICE) return rc;
    *stats = h->stats;
    return LOOM_B200_OK;
}

int
loom_b200_device_bytes(const loom_b200_handle* h, uint64_t* bytes)
{
    if(!h || !bytes) return LOOM_B200_ERR_INVALID;
    const loom_b200_kernel_info& info = *h->e->info;
    uint64_t b = 0;
    if(h->capacity)
    {
        for(uint32_t i = 0; i < info.num_inputs; ++i) b += h->capacity * type_bytes(info.input_types[i]);
        for(uint32_t i = 0; i < info.num_outputs; ++i) b += h->capacity * type_bytes(info.output_types[i]);
    }
    b += sizeof(unsigned) + counter_bytes(*h->e) + sizeof(RegroupCtl);
    if(h->ws_cap) b += 2 * h->e->row_bytes * h->ws_cap + 3ull * h->e->num_queues * sizeof(unsigned);
    b += h->starts_bytes + h->table_bytes + h->rows_bytes;
    *bytes = b;
    return LOOM_B200_OK;
}

int
loom_b200_get_block_stats(loom_b200_handle* h,
                          uint64_t*         thread_instr,
                          uint64_t*         warp_instr,
                          uint32_t          num_blocks)
{
    if(!h || !thread_instr || !warp_instr || num_blocks != h->e->info->num_blocks)
        return LOOM_B200_ERR_INVALID;
    const int rc = finish_launch(h);
    if(rc != LOOM_B200_OK && rc != LOOM_B200_ERR_DEVICE) return rc;
    std::vector<unsigned long long> c(2 * static_cast<size_t>(num_blocks));
    LB_CUDA(cudaMemcpy(c.data(), h->d_counters + 8, c.size() * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost));
    for(uint32_t b = 0; b < num_blocks; ++b)
    {
        thread_instr[b] = c[2 * b];
        warp_instr[b]   = c[2 * b + 1];
    }
    return LOOM_B200_OK;
}

int
loom_b200_kernel_reg_caps(const char* kernel, uint32_t* caps, uint32_t max_caps, uint32_t* num_caps)
{
    if(!kernel || !num_caps || (!caps && max_caps)) return LOOM_B200_ERR_INVALID;
    for(int i = 0; i < kRegistrySize; ++i)
        if(std::strcmp(kRegistry[i]->info->name, kernel) == 0)
        {
            const KernelEntry& e = *kRegistry[i];
            for(uint32_t c = 0; c < max_caps && c < e.num_reg_caps; ++c) caps[c] = e.reg_caps[c];
            *num_caps = e.num_reg_caps;
            return LOOM_B200_OK;
        }
    return LOOM_B200_ERR_NOT_FOUND;
}

int
loom_b200_kernel_queues(const char* kernel, uint32_t* num_queues, const loom_b200_queue_layout** queues)
{
    if(!kernel || !num_queues || !queues) return LOOM_B200_ERR_INVALID;
    for(int i = 0; i < kRegistrySize; ++i)
        if(std::strcmp(kRegistry[i]->info->name, kernel) == 0)
        {
            *num_queues = kRegistry[i]->num_queues;
            *queues     = kRegistry[i]->queues;
            return LOOM_B200_OK;
        }
    g_last_error = "kernel not compiled into libloom_b200";
    return LOOM_B200_ERR_NOT_FOUND;
}

namespace
{
/// Parked rows per queue after the handle's last launch, and the parity of
/// the state half that holds them: the megakernel parks a round's leftovers
/// in the half of the next round, whose number it leaves in the control
/// block; the counts of that half survive the launch.
int
parked_state(loom_b200_handle* h, std::vector<unsigned>& counts, unsigned& parity)
{
    const int rc = finish_launch(h);
    if(rc != LOOM_B200_OK && rc != LOOM_B200_ERR_DEVICE) return rc;
    const unsigned B = h->e->num_queues;
    counts.assign(B, 0u);
    parity = 0;
    if(h->last_cap == 0 || !h->d_qcnt) return LOOM_B200_OK;
    RegroupCtl ctl{};
    LB_CUDA(cudaMemcpy(&ctl, h->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
    parity = static_cast<unsigned>(ctl.next_round & 1ull);
    LB_CUDA(cudaMemcpy(counts.data(), h->d_qcnt + parity * B, B * sizeof(unsigned), cudaMemcpyDeviceToHost));
    for(unsigned& c : counts)
        if(c > h->last_cap) c = static_cast<unsigned>(h->last_cap); // rows past capacity were never written
    return LOOM_B200_OK;
}
} // namespace

int
loom_b200_parked_counts(loom_b200_handle* h, uint32_t* counts, uint32_t max_queues, uint32_t* num_queues)
{
    if(!h || (!counts && max_queues)) return LOOM_B200_ERR_INVALID;
    std::vector<unsigned> c;
    unsigned              parity = 0;
    const int             rc     = parked_state(h, c, parity);
    if(rc) return rc;
    for(uint32_t q = 0; q < max_queues && q < c.size(); ++q) counts[q] = c[q];
    if(num_queues) *num_queues = static_cast<uint32_t>(c.size());
    return LOOM_B200_OK;
}

int
loom_b200_parked_dump(loom_b200_handle* h,
                      uint32_t          queue,
                      void* const*      cols,
                      uint32_t*         tids,
                      uint64_t          max_rows,
                      uint64_t*         rows)
{
    if(!h || !rows || queue >= h->e->num_queues) return LOOM_B200_ERR_INVALID;
    *rows = 0;
    std::vector<unsigned> c;
    unsigned              parity = 0;
    const int             rc     = parked_state(h, c, parity);
    if(rc) return rc;
    const uint64_t n = std::min<uint64_t>(c[queue], max_rows);
    if(n == 0) return LOOM_B200_OK;
    const loom_b200_queue_layout& ql   = h->e->queues[queue];
    const QueueSegment&           seg  = h->e->segments[queue];
    const uint64_t                cap  = h->last_cap;
    const char*                   half = h->d_state + parity * h->e->row_bytes * cap;
    for(uint32_t k = 0; cols && k < ql.num_cols; ++k)
    {
        if(!cols[k]) continue;
        const size_t width = type_bytes(ql.types[k]);
        LB_CUDA(cudaMemcpy2D(cols[k], width, half + seg.col_off[k] * cap + seg.col_sub[k], seg.col_width[k],
                             width, n, cudaMemcpyDeviceToHost));
    }
    if(tids)
        LB_CUDA(cudaMemcpy2D(tids, sizeof(uint32_t), half + seg.tid_off * cap + seg.tid_sub, seg.tid_width,
                             sizeof(uint32_t), n, cudaMemcpyDeviceToHost));
    *rows = n;
    return LOOM_B200_OK;
}

int
loom_b200_reset_stats(loom_b200_handle* h)
{
    if(!h) return LOOM_B200_ERR_INVALID;
    const int rc = finish_launch(h);
    if(rc != LOOM_B200_OK && rc != LOOM_B200_ERR_DEVICE) return rc;
    LB_CUDA(cudaMemset(h->d_counters, 0, counter_bytes(*h->e)));
    LB_CUDA(cudaMemset(h->d_status, 0, sizeof(unsigned)));
    h->stats         = loom_b200_stats{};
    h->launches      = 0;
    h->plain_threads = 0;
    return LOOM_B200_OK;
}

} // extern "C"
