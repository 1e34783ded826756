// loom_b200_launch_static: the regrouping engine with its workspace in a
// fixed device array instead of memory from cudaMalloc.
//
// Who needs it: a caller that may not allocate device memory at the point
// of the call.  cudaMalloc can synchronise the whole device and can fail
// outright when another allocator of the process (a framework's caching
// allocator, a memory pool sized to the whole GPU) has already reserved the
// free memory, so a plugin or callback that runs inside such a host, or a
// service that must not stall on the allocator, brings its own input and
// output buffers and cannot create a handle (loom_b200_create allocates its
// queues and bookkeeping).  Here the queues, their state and the engine's
// control words live in `g_scratch`, a file-scope device array of
// LOOM_B200_STATIC_SCRATCH_BYTES that every GPU which loads this library
// holds until the process exits.
//
// The array is one per device and shared by every call: each call clears
// the words that must start at zero (queue counters, pop cursors, the grid
// barrier, the admission cursor, the status word) before its launch, and the
// queue state needs no clearing because every row is written before it is
// read.  Two calls whose launches overlap on the GPU (different streams,
// different host threads) race on the array and give wrong results; the
// call returns only after its launch finished, so calls made one after
// another from one host thread never overlap.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "runtime_iface.h"

using namespace loom_b200;

/// The workspace.  Device code could name it directly; host code must not:
/// on the host `g_scratch` is a stand-in symbol, not a device address, so
/// the launch below passes the address returned by cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[LOOM_B200_STATIC_SCRATCH_BYTES];

namespace
{
// Layout of the array: control words, then the queue counters, then the
// queue state (both parities), each part on a 256-byte boundary.
constexpr size_t kCtlOff      = 0;   // RegroupCtl
constexpr size_t kStatusOff   = 64;  // unsigned status word
constexpr size_t kCountersOff = 128; // 8 x unsigned long long
constexpr size_t kQueueOff    = 256; // qcnt [2][B], then qhead [B]

constexpr size_t
align256(size_t x)
{
    return (x + 255) / 256 * 256;
}

// The defaults of loom_b200_create for the regrouping engine.
constexpr unsigned           kBlock    = 256;
constexpr unsigned           kUtr      = 16;
constexpr unsigned           kPeriod   = 1024;
constexpr unsigned           kBurst    = 32;
constexpr unsigned           kSpread   = 33;
constexpr unsigned long long kMaxSteps = 1ull << 40;
constexpr unsigned long long kSpins    = 1ull << 25;

constexpr int kMaxDevices = 64;

/// Device address of g_scratch and SM count, per device, set up on the
/// first call made with that device current.
struct DeviceSlot
{
    unsigned char* scratch = nullptr;
    int            sms     = 0;
};
DeviceSlot g_slots[kMaxDevices];
std::mutex g_setup;

int
setup(int device, DeviceSlot* out)
{
    std::lock_guard<std::mutex> lock(g_setup);
    DeviceSlot&                 s = g_slots[device];
    if(s.scratch == nullptr)
    {
        void* ptr = nullptr;
        if(cudaGetSymbolAddress(&ptr, g_scratch) != cudaSuccess) return LOOM_B200_ERR_CUDA;
        int sms = 0;
        if(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
            return LOOM_B200_ERR_CUDA;
        s.sms     = sms;
        s.scratch = static_cast<unsigned char*>(ptr);
    }
    *out = s;
    return LOOM_B200_OK;
}

/// Clears what a launch reads before writing: the control block, status,
/// counters, the queue counters of both parities and the pop cursors.
__global__ void
static_reset(unsigned char* base, unsigned num_queues, unsigned long long admit_end)
{
    auto* ctl      = reinterpret_cast<RegroupCtl*>(base + kCtlOff);
    auto* qwords   = reinterpret_cast<unsigned*>(base + kQueueOff);
    auto* counters = reinterpret_cast<unsigned long long*>(base + kCountersOff);
    for(unsigned i = threadIdx.x; i < 3 * num_queues; i += blockDim.x) qwords[i] = 0u;
    if(threadIdx.x < 8) counters[threadIdx.x] = 0ull;
    if(threadIdx.x == 0)
    {
        *reinterpret_cast<unsigned*>(base + kStatusOff) = 0u;
        ctl->bar_count = 0u;
        ctl->bar_gen   = 0u;
        ctl->done      = 0u;
        ctl->pad0      = 0u;
        ctl->cursor    = 0ull;
        ctl->admit_end = admit_end;
    }
}

const KernelEntry*
find(const char* name)
{
    for(int i = 0; i < kRegistrySize; ++i)
        if(std::strcmp(kRegistry[i]->info->name, name) == 0) return kRegistry[i];
    return nullptr;
}
} // namespace

extern "C" int
loom_b200_launch_static(const char*             kernel,
                        const loom_b200_launch* L,
                        const loom_b200_opts*   opts,
                        void*                   stream_,
                        uint32_t*               status_out)
{
    if(status_out) *status_out = 0u;
    if(!kernel || !L) return LOOM_B200_ERR_INVALID;
    const KernelEntry* e = find(kernel);
    if(!e) return LOOM_B200_ERR_NOT_FOUND;
    const loom_b200_kernel_info& info = *e->info;
    const uint64_t               n    = L->n;
    if(n == 0) return LOOM_B200_OK;
    if(n >= (1ull << 32)) return LOOM_B200_ERR_INVALID; // thread ids are 32-bit
    if(info.num_inputs > static_cast<uint32_t>(kMaxIn) ||
       info.num_inputs + info.num_outputs > static_cast<uint32_t>(kMaxCols))
        return LOOM_B200_ERR_INVALID;
    if(!L->inputs && info.num_inputs) return LOOM_B200_ERR_INVALID;
    if(!L->outputs) return LOOM_B200_ERR_INVALID;

    // columns, as loom_b200_launch_device reads them
    Columns cols{};
    int     c = 0;
    for(uint32_t i = 0; i < info.num_inputs; ++i)
    {
        const loom_b200_input& in = L->inputs[i];
        if(in.form > LOOM_B200_IN_INSTANCE || (in.form == LOOM_B200_IN_ARRAY && in.ptr == nullptr))
            return LOOM_B200_ERR_INVALID;
        cols.form[i]  = in.form;
        cols.value[i] = in.value;
        cols.p[c++]   = const_cast<void*>(in.ptr);
    }
    for(uint32_t i = 0; i < info.num_outputs; ++i)
    {
        if(L->outputs[i] == nullptr) return LOOM_B200_ERR_INVALID;
        cols.p[c++] = L->outputs[i];
    }
    cols.inst_start = reinterpret_cast<const unsigned long long*>(L->instance_starts);
    cols.num_inst   = L->instance_starts ? L->num_instances : 0u;
    cols.table      = L->table;

    loom_b200_opts o{};
    if(opts) o = *opts;
    if(o.block_size == 0 || o.block_size % 32 != 0 || o.block_size > 1024) o.block_size = kBlock;
    if(o.utr_lanes == 0 || o.utr_lanes > 32) o.utr_lanes = kUtr;
    if(o.period == 0) o.period = kPeriod;
    if(o.burst == 0) o.burst = kBurst;
    if(o.spread_lanes == 0) o.spread_lanes = kSpread;
    if(o.max_steps == 0) o.max_steps = kMaxSteps;

    // population: what the caller asked for, else as many threads in flight
    // as the array holds; a request beyond the array is refused
    const size_t   queue_words = 3ull * e->num_queues * sizeof(unsigned);
    const size_t   state_off   = align256(kQueueOff + queue_words);
    const uint64_t per_slot    = 2ull * e->row_bytes;
    if(state_off >= LOOM_B200_STATIC_SCRATCH_BYTES) return LOOM_B200_ERR_BUDGET;
    const uint64_t fit = (LOOM_B200_STATIC_SCRATCH_BYTES - state_off) / per_slot / 32 * 32;
    uint64_t       cap;
    if(o.population)
    {
        cap = (std::min<uint64_t>(o.population, n) + 31) / 32 * 32;
        if(cap > fit) return LOOM_B200_ERR_BUDGET;
    }
    else
    {
        if(fit == 0) return LOOM_B200_ERR_BUDGET;
        cap = std::min<uint64_t>((n + 31) / 32 * 32, fit);
    }

    int device = 0;
    if(cudaGetDevice(&device) != cudaSuccess) return LOOM_B200_ERR_NO_DEVICE;
    if(device < 0 || device >= kMaxDevices) return LOOM_B200_ERR_INVALID;
    DeviceSlot slot;
    if(const int rc = setup(device, &slot)) return rc;

    unsigned block = o.block_size;
    int      ctas  = 0;
    for(;;)
    {
        if(e->regroup_occupancy(static_cast<int>(block), false, 0u, 0u, true, &ctas) != cudaSuccess)
            return LOOM_B200_ERR_CUDA;
        if(ctas > 0 || block <= 32) break;
        block /= 2;
    }
    if(ctas <= 0) return LOOM_B200_ERR_INVALID;
    if(o.ctas_per_sm) ctas = std::min<int>(ctas, static_cast<int>(o.ctas_per_sm));

    unsigned char* base = slot.scratch;
    RegroupLaunch  R{};
    R.params.cols          = cols;
    R.params.state         = reinterpret_cast<char*>(base + state_off);
    R.params.qcnt          = reinterpret_cast<unsigned*>(base + kQueueOff);
    R.params.qhead         = reinterpret_cast<unsigned*>(base + kQueueOff) + 2 * e->num_queues;
    R.params.ctl           = reinterpret_cast<RegroupCtl*>(base + kCtlOff);
    R.params.status        = reinterpret_cast<unsigned*>(base + kStatusOff);
    R.params.counters      = reinterpret_cast<unsigned long long*>(base + kCountersOff);
    R.params.n             = n;
    R.params.max_rounds    = o.max_steps;
    R.params.barrier_spins = o.barrier_spins ? o.barrier_spins : kSpins;
    R.params.phantoms      = 0u;
    R.params.cap           = static_cast<unsigned>(cap);
    R.params.utr           = o.utr_lanes;
    R.params.period        = o.period;
    R.params.burst         = o.burst;
    R.params.spread        = o.spread_lanes;
    R.params.refill        = o.no_refill ? 0u : 1u;
    R.params.prefetch      = o.no_prefetch ? 0u : 1u;
    R.params.cost_model    = o.cost_model;
    R.params.schedule      = o.schedule;
    R.grid                 = static_cast<unsigned>(ctas * slot.sms);
    R.block                = block;
    R.profile              = false;
    R.stream               = static_cast<cudaStream_t>(stream_);

    static_reset<<<1, 256, 0, R.stream>>>(base, e->num_queues, std::min<uint64_t>(n, cap));
    if(cudaGetLastError() != cudaSuccess) return LOOM_B200_ERR_CUDA;
    if(e->regroup(R) != cudaSuccess) return LOOM_B200_ERR_CUDA;
    unsigned status = 0;
    if(cudaMemcpyAsync(&status, R.params.status, sizeof status, cudaMemcpyDeviceToHost, R.stream) !=
           cudaSuccess ||
       cudaStreamSynchronize(R.stream) != cudaSuccess)
        return LOOM_B200_ERR_CUDA;
    if(status_out) *status_out = status;
    return status ? LOOM_B200_ERR_DEVICE : LOOM_B200_OK;
}
