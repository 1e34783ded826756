/* loom_b200.h — C ABI of the B200 execution backend for Loom kernels.
 *
 * Loom selects a backend by C++ template alias and has no FFI of its own:
 *   vm::bse::function<K>          Loom src/vm/bse.hpp:648-649
 *   vm::cuda::function<K>(n)      Loom src/vm/cuda.hpp:1581-1582
 *   vm::cuda::stream<K>(n)        Loom src/vm/cuda.hpp:1584-1586
 *   vm::simd::hybrid_function<K>  Loom src/vm/simd.hpp:4311-4318
 * The functions below are the boundary those aliases bind to on B200: the
 * C++ front end (loom_b200.hpp) and the Python binding (loom_b200.api) call
 * only these entry points.  Plain pointers and sizes; no exceptions cross the
 * ABI; every call returns LOOM_B200_OK (0) or a negative error code.
 * A handle is not thread-safe: one host thread drives it at a time
 * (Loom's facades have the same rule, src/vm/mp.hpp:67-132).
 */
#ifndef LOOM_B200_H
#define LOOM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LOOM_B200_ABI_VERSION 1

/* ------------------------------------------------------------ error codes */
#define LOOM_B200_OK 0
#define LOOM_B200_ERR_INVALID (-1)   /* bad argument */
#define LOOM_B200_ERR_NOT_FOUND (-2) /* kernel name not compiled in */
#define LOOM_B200_ERR_CUDA (-3)      /* CUDA runtime error */
#define LOOM_B200_ERR_OOM (-4)       /* device allocation failed */
#define LOOM_B200_ERR_DEVICE (-5)    /* device status word non-zero */
#define LOOM_B200_ERR_BUDGET (-6)    /* request exceeds the memory budget */
#define LOOM_B200_ERR_NO_DEVICE (-7) /* no CUDA device visible */
#define LOOM_B200_ERR_CANCELLED (-8) /* request cancelled */
#define LOOM_B200_ERR_TIMEOUT (-9)   /* host-side watchdog expired */

/* Device status bits (loom_b200_stats.status).  Device code never traps:
 * it records one of these and finishes the launch. */
#define LOOM_B200_STATUS_STEP_LIMIT 1u      /* a thread exceeded max_steps */
#define LOOM_B200_STATUS_ASSERT_FP 2u       /* ops::assert_fp saw NaN/inf */
#define LOOM_B200_STATUS_QUEUE_OVERRUN 4u   /* a work-queue index was out of range */
#define LOOM_B200_STATUS_BARRIER_TIMEOUT 8u /* a bounded grid-barrier wait ran out */

/* ------------------------------------------------------------ scalar types */
enum loom_b200_type
{
    LOOM_B200_B8  = 0,
    LOOM_B200_I8  = 1,
    LOOM_B200_U8  = 2,
    LOOM_B200_I16 = 3,
    LOOM_B200_U16 = 4,
    LOOM_B200_I32 = 5,
    LOOM_B200_U32 = 6,
    LOOM_B200_I64 = 7,
    LOOM_B200_U64 = 8,
    LOOM_B200_F32 = 9,
    LOOM_B200_F64 = 10
};

/* Static description of a compiled kernel.  Mirrors the compile-time facts
 * of loom::vm::kernel_blank (Loom src/vm/core.hpp:939-1031): inputs/outputs
 * (input_vars/output_vars), num_blocks, state_size. */
typedef struct loom_b200_kernel_info
{
    const char*        name;          /* registry name, e.g. "fib_u64" */
    const char*        ir_digest;     /* structural digest of the text IR (16 hex) */
    uint32_t           num_inputs;
    uint32_t           num_outputs;
    const int*         input_types;   /* enum loom_b200_type */
    const int*         output_types;
    const char* const* input_names;
    const char* const* output_names;
    uint32_t           num_blocks;
    uint32_t           num_regs;      /* Loom registers incl. PC (reg_names) */
    uint32_t           state_size;    /* K::state_size in bytes */
    uint32_t           state_cols;    /* registers live at some block entry */
    const uint32_t*    block_instrs;  /* static instruction count per block */
    const uint32_t*    block_live_bytes; /* live-in bytes per block */
} loom_b200_kernel_info;

/* Execution form. */
#define LOOM_B200_PERIOD_UNBOUNDED 0xffffffffu /* opts.period: no period limit */
#define LOOM_B200_PLAIN 0u   /* one CUDA thread per Loom thread, hardware reconvergence */
#define LOOM_B200_REGROUP 1u /* persistent megakernel, threads regrouped by PC */

/* Launch options; zero-initialise and set what you need (0 = default). */
typedef struct loom_b200_opts
{
    uint32_t mode;        /* LOOM_B200_PLAIN or LOOM_B200_REGROUP */
    uint32_t block_size;  /* CUDA threads per CTA (multiple of 32) */
    uint32_t utr_lanes;   /* regroup: keep running in registers while the
                             largest same-PC group has >= utr_lanes lanes
                             (the GPU form of Loom's UTR, simd.hpp:3273-3292) */
    uint32_t period;      /* regroup: max block steps per tile per round;
                             LOOM_B200_PERIOD_UNBOUNDED with schedule 2 or 3:
                             a warp never parks, so the launch runs one round,
                             admits every input at once and needs no queue
                             state (a few KB instead of 2 x row bytes per
                             thread in flight) */
    uint32_t burst;       /* regroup: blocks a lane runs between two votes */
    uint32_t spread_lanes; /* regroup: when the majority block holds at least
                              this many lanes, every live lane runs the
                              burst (33 = majority lanes only) */
    uint32_t no_refill;   /* regroup: halted lanes without a prefetched input
                             wait for the next vote instead of claiming one */
    uint32_t graph;       /* regroup: capture the launch sequence (queue reset
                             + engine kernel) into a CUDA graph on first use
                             and replay it while the launch arguments stay
                             the same */
    uint64_t population;  /* regroup: resident thread slots; 0 = all inputs */
    uint64_t max_steps;   /* plain: per-thread block-step guard; regroup:
                             rounds of the megakernel (a tile runs at most
                             `period` block steps per round); 0 = 2^40 */
    uint32_t profile;     /* collect lane-efficiency counters (slower) */
    uint32_t no_prefetch; /* regroup: do not prefetch each lane's next input */
    uint32_t ctas_per_sm; /* regroup: resident CTAs per SM; 0 = occupancy max */
    uint32_t fault_phantom_ctas; /* fault injection for tests: the grid barrier
                                    also waits for this many CTAs that do not
                                    exist, so its bounded wait must run out */
    uint64_t barrier_spins; /* regroup: polls before a barrier wait gives up
                               (0 = default, about 7 s) */
    uint32_t cost_model;  /* regroup: per-block quorum from a cost model (a
                             long block runs only with enough lanes, else its
                             lanes park and come back as full warps) */
    uint32_t schedule;    /* regroup: 0 runs the largest same-block group
                             (Loom's majority rule); 1 runs the group at the
                             block earliest in program order, so lagging lanes
                             catch up and merge; 2 steps one block at a time
                             in that order without votes or parking (a
                             reconvergence stack in software, plus refill);
                             3 runs each warp's lanes along their own paths
                             under the hardware's reconvergence, as the plain
                             engine does, and gives the warp new threads when
                             all its lanes have finished (use a large burst) */
    uint32_t host_chunks; /* launch_host: split the threads into this many
                             ranges whose host copies overlap the kernels of
                             the neighbouring ranges (0 = 8 ranges when the
                             copies reach 32 MB, else 1) */
    uint32_t max_regs;    /* regroup: registers per thread of the megakernel,
                             one of the caps compiled for the kernel
                             (loom_b200_kernel_reg_caps); 0 = its default */
    uint64_t plain_below; /* regroup: launches of fewer threads run the plain
                             engine, for workloads too small or too uniform
                             for the persistent megakernel to pay (Loom's
                             hybrid backend likewise falls back to predicated
                             execution where regrouping does not pay,
                             src/vm/simd.hpp:4163-4194); 0 = never */
    uint32_t defer_lanes; /* regroup, schedule 2: a long block of the kernel
                             (the longest few, >= 96 instructions) runs only
                             once this many of the warp's lanes stand at it,
                             or when no other block is left; its lanes wait
                             while the others catch up (0 = off) */
    uint32_t bulk_restore; /* regroup: full tiles of parked threads come back
                              through shared memory, one bulk copy (TMA,
                              cp.async.bulk, no multicast) per 16-byte slot
                              column, instead of 128-bit loads from HBM; the
                              CTA size is halved until the staging area
                              fits in shared memory; runs at the default
                              register cap (max_regs is ignored) */
    uint32_t spin_iters;  /* regroup, schedule 2: iterations of a loop on one
                             block a lane runs within one step (0 = 1024);
                             kernels of at most 300 instructions run 16
                             (spin_iters 1-16), 64 (17-64) or 1024, counts
                             compiled into their code: a few let halted
                             lanes take new threads sooner, many save the
                             step's cost */
    uint32_t refill_lanes; /* regroup, schedule 2: a warp's burst of steps
                              ends as soon as this many of its lanes have
                              halted, so that the threads that replace them
                              start together (0: every burst runs its full
                              length) */
} loom_b200_opts;

/* Counters of the launches since the last reset. */
typedef struct loom_b200_stats
{
    uint64_t launches;
    uint64_t threads;      /* Loom threads completed */
    uint64_t thread_instr; /* VM instructions executed, summed over threads */
    uint64_t warp_instr;   /* VM instructions issued, summed over warp steps;
                              lane efficiency = thread_instr / (32 * warp_instr) */
    uint64_t rounds;       /* regroup rounds (grid barriers) */
    uint64_t parks;        /* threads written to the state file */
    uint64_t state_bytes;  /* algorithmic state bytes moved (saves + restores) */
    uint32_t status;       /* OR of LOOM_B200_STATUS_* */
    uint32_t grid;         /* CTAs of the last launch */
    double   ms;           /* device time of the last launch (CUDA events) */
    uint64_t graph_captures; /* CUDA graphs captured (opts.graph) */
    uint64_t graph_launches; /* launches replayed from a graph */
} loom_b200_stats;

/* Input column forms (loom_b200_input.form). */
#define LOOM_B200_IN_ARRAY 0u      /* ptr[tid] */
#define LOOM_B200_IN_IOTA 1u       /* the thread index tid */
#define LOOM_B200_IN_BROADCAST 2u  /* `value` (its low bytes) for every thread */
#define LOOM_B200_IN_LOCAL_IOTA 3u /* tid minus the first thread of its instance */
#define LOOM_B200_IN_INSTANCE 4u   /* index of the thread's instance */

typedef struct loom_b200_input
{
    const void* ptr;  /* LOOM_B200_IN_ARRAY: the column */
    uint32_t    form; /* LOOM_B200_IN_* */
    uint32_t    pad;
    uint64_t    value; /* LOOM_B200_IN_BROADCAST: the bit pattern */
} loom_b200_input;

/* One launch over n threads that may belong to several instances of the
 * kernel (render requests, input batches): instance i owns threads
 * [instance_starts[i], instance_starts[i + 1]).  Threads of different
 * instances that stand at the same basic block share warps.  `table` is the
 * read-only table of 32-bit words that the tab op reads (a Loom extension,
 * loom_b200/frontend/b200_ops.hpp). */
typedef struct loom_b200_launch
{
    const loom_b200_input* inputs;          /* one per kernel input */
    void* const*           outputs;         /* one per kernel output */
    uint64_t               n;
    const uint64_t*        instance_starts; /* num_instances + 1 offsets, or NULL */
    uint32_t               num_instances;
    uint32_t               pad;
    const uint32_t*        table;           /* or NULL */
    uint64_t               table_words;
} loom_b200_launch;

typedef struct loom_b200_handle loom_b200_handle;

/* ------------------------------------------------------------ registry */
int         loom_b200_version(void);
const char* loom_b200_error_string(int code);
int         loom_b200_kernel_count(void);
int         loom_b200_kernel_get(int index, const loom_b200_kernel_info** info);
int         loom_b200_kernel_find(const char* name, const loom_b200_kernel_info** info);
/* Register caps compiled for the kernel's regrouping megakernel (values for
 * opts.max_regs), the default first: *num_caps receives their number, up to
 * max_caps of them go to caps. */
int         loom_b200_kernel_reg_caps(const char* kernel, uint32_t* caps, uint32_t max_caps, uint32_t* num_caps);
/* Finds a compiled kernel by the structural digest of its IR (16 hex
 * digits, loom_b200/frontend/ir_emit.hpp: structural_digest): how the C++
 * front end binds a Loom kernel type to its compiled code. */
int         loom_b200_kernel_find_digest(const char* digest, const loom_b200_kernel_info** info);

/* ------------------------------------------------------------ function
 * Replaces vm::cuda::function<K>(n)(inputs...) (Loom src/vm/cuda.hpp:
 * 1406-1462, MemoryFacade::set_inputs/get_outputs 1060-1148): one handle per
 * kernel and capacity; inputs are column arrays (one pointer per
 * K::input_vars entry), outputs likewise; outputs keep input order. */
int loom_b200_create(const char*             kernel,
                     uint64_t                capacity,
                     const loom_b200_opts*   opts,
                     loom_b200_handle**      out);
int loom_b200_destroy(loom_b200_handle* h);
int loom_b200_set_opts(loom_b200_handle* h, const loom_b200_opts* opts);
int loom_b200_get_opts(const loom_b200_handle* h, loom_b200_opts* opts);

/* Host columns in, host columns out; copies and launch are inside the call,
 * which returns after the outputs are on the host.  A NULL input column
 * means "iota": input value = thread index. */
int loom_b200_run_host(loom_b200_handle*  h,
                       const void* const* inputs,
                       void* const*       outputs,
                       uint64_t           n);

/* Device columns in and out, enqueued on `stream` (a cudaStream_t; NULL is
 * the CUDA default stream, as everywhere in CUDA); returns without
 * synchronising. */
int loom_b200_run_device(loom_b200_handle*  h,
                         const void* const* inputs,
                         void* const*       outputs,
                         uint64_t           n,
                         void*              stream);

/* General launch on device memory: every pointer of `L` (array inputs,
 * outputs, instance_starts, table) is a device pointer; asynchronous on
 * `stream`. */
int loom_b200_launch_device(loom_b200_handle* h, const loom_b200_launch* L, void* stream);

/* General launch on host memory: array inputs, outputs, instance_starts and
 * the table are host arrays; the call copies them in, runs the kernel,
 * copies the outputs back and returns after they arrived.  Large copies
 * are pipelined (opts.host_chunks): the threads run as consecutive ranges,
 * and while range k runs, the inputs of range k + 1 go in and the outputs
 * of range k - 1 come back (pinned host memory lets the copies overlap). */
int loom_b200_launch_host(loom_b200_handle* h, const loom_b200_launch* L);

/* Per-group means of float outputs: for launches whose threads are samples
 * of one result, e.g. a render request with one thread per pixel-sample and
 * `group` samples per pixel, which Loom's render path turns into an image
 * (src/benchmarks/render.hpp:223-230).  Output row r is the mean of threads
 * r * group .. r * group + group - 1, summed in thread order and divided by
 * the group size, in the output's own float type.  With instance_group,
 * instance i's rows cover instance_group[i] threads each and follow the rows
 * of instance i - 1 (each instance's thread count must be a multiple of its
 * group). */
typedef struct loom_b200_mean
{
    uint32_t        group;          /* threads per row (without instance_group) */
    uint32_t        pad;
    const uint32_t* instance_group; /* threads per row of each instance (host), or NULL */
} loom_b200_mean;

/* loom_b200_launch_host whose outputs are the group means of `M`: every
 * output must be f32 or f64, and the host output arrays hold one row per
 * group.  Only the rows are copied back. */
int loom_b200_launch_host_mean(loom_b200_handle* h, const loom_b200_launch* L, const loom_b200_mean* M);

/* The same reduction of one device column of `type` (LOOM_B200_F32 or
 * LOOM_B200_F64) with a uniform group: out[r] for r < rows from
 * in[r * group ...]; asynchronous on `stream`. */
int loom_b200_group_mean(uint32_t type, const void* in, void* out, uint64_t rows, uint32_t group, void* stream);

int loom_b200_sync(loom_b200_handle* h);
int loom_b200_get_stats(loom_b200_handle* h, loom_b200_stats* stats);
int loom_b200_reset_stats(loom_b200_handle* h);
/* Device memory the handle holds now: its staging columns, the regrouping
 * engine's queues with their state, control words, counters and the copies
 * of instance offsets and table made by launch_host.  Loom's facades size
 * their device columns by the stream size (src/vm/cuda.hpp:86-118); this is
 * the figure a caller budgets against. */
int loom_b200_device_bytes(const loom_b200_handle* h, uint64_t* bytes);
/* Per basic block, over the profiled launches (opts.profile) since the last
 * reset: VM instructions executed summed over threads, and issued summed
 * over warp steps (lane efficiency of block b = thread_instr[b] / (32 *
 * warp_instr[b])).  num_blocks must equal the kernel's.  Replaces reading
 * Loom's per-instruction debug trace (src/vm/dbg.hpp:920-1143) for the
 * question of where lanes go idle. */
int loom_b200_get_block_stats(loom_b200_handle* h,
                              uint64_t*         thread_instr,
                              uint64_t*         warp_instr,
                              uint32_t          num_blocks);

/* ------------------------------------------------------------ state inspection
 * The regrouping engine's work queues read back after a launch: at which
 * Loom block each parked thread waits and the registers it carries there.
 * This takes the place of Loom's inspector (src/vm/dbg.hpp:918-933
 * print_state, 1143 inspect), which steps one thread on the CPU and prints
 * its PC label and registers: here the rows are every thread the engine
 * parked.  Threads stay parked when a launch ends before they finish, i.e.
 * when opts.max_steps (for the regrouping engine: rounds of the megakernel)
 * runs out; the launch then reports LOOM_B200_STATUS_STEP_LIMIT and its
 * queues keep their rows until the handle's next launch.  After a launch
 * that finished every thread the queues are empty. */

/* One work queue: the block it holds threads for and their live registers.
 * A block ending in a dispatch on a register the callers set (a subroutine
 * such as Loom's RNG block) has one more queue per caller: `context` is the
 * value the caller set, restored without being stored (-1 for a block's own
 * queue). */
typedef struct loom_b200_queue_layout
{
    uint32_t           block;    /* Loom block index (0 = START) */
    int32_t            context;  /* dispatch context, or -1 */
    uint32_t           num_cols; /* live registers saved per parked thread */
    const uint32_t*    regs;     /* register index of each column (IR order, PC = 0) */
    const int*         types;    /* enum loom_b200_type of each column */
    const char* const* names;    /* register name of each column */
} loom_b200_queue_layout;

/* The queues of a compiled kernel (static; no GPU needed). */
int loom_b200_kernel_queues(const char*                    kernel,
                            uint32_t*                      num_queues,
                            const loom_b200_queue_layout** queues);

/* Threads parked in each queue at the end of the handle's last launch
 * (waits for it; zero for the plain engine).  Writes min(max_queues, the
 * kernel's queues) counts and the kernel's queue count. */
int loom_b200_parked_counts(loom_b200_handle* h,
                            uint32_t*         counts,
                            uint32_t          max_queues,
                            uint32_t*         num_queues);

/* Copies up to max_rows parked rows of one queue to host memory: column c
 * into cols[c] (num_cols arrays of the column's type; NULL skips a column,
 * or all when cols is NULL) and the low 32 bits of each row's thread index
 * into tids (may be NULL).  *rows receives the rows copied. */
int loom_b200_parked_dump(loom_b200_handle* h,
                          uint32_t          queue,
                          void* const*      cols,
                          uint32_t*         tids,
                          uint64_t          max_rows,
                          uint64_t*         rows);

/* ------------------------------------------------------------ serving
 * Continuous batching of requests on the regrouping engine.  Replaces the
 * exchange loop of Loom's streams (StreamFacade::exchange, Loom
 * src/vm/bve.hpp:1208-1270; tests/stream_wrapper.hpp:33-80) and the worker
 * pool that feeds them (mp::Shop, src/vm/mp.hpp:316-385) for whole
 * requests: a request (an instance of n threads) is admitted in arrival
 * order as soon as its thread state fits (a request slot, n entries of the
 * column rings, its table body in the arena), joins the threads already in
 * flight in the running megakernel, and its outputs come back when its last
 * thread finished.  The device runs slices of `slice_rounds` regroup rounds;
 * between slices the parked threads stay resident in the device queues.
 * A server is driven by one host thread; every call is synchronous on the
 * server's stream. */
typedef struct loom_b200_server loom_b200_server;

/* A device-memory budget for the thread state of admitted requests, shared
 * by the servers that point to it (drive them from one host thread).  A
 * request holds n x (state_size + its column bytes per thread) plus its
 * header and body bytes from admission until it completes or is dropped:
 * Loom's per-thread state is K::state_size (src/vm/core.hpp:1026-1030), and
 * its streams bound the rows in flight by the stream size
 * (src/vm/simd.hpp:2803-2903).  A request that does not fit waits in the
 * queue (arrival order); one larger than the whole limit is refused at
 * submit with LOOM_B200_ERR_BUDGET. */
typedef struct loom_b200_budget
{
    uint64_t limit; /* bytes */
    uint64_t used;  /* bytes held by admitted requests (maintained by the servers) */
} loom_b200_budget;

typedef struct loom_b200_server_cfg
{
    uint64_t        ring_threads; /* entries of each column ring: a power of
                                     two in [32, 2^31]; bounds the threads of
                                     the requests in flight */
    uint64_t        table_words;  /* words of the table arena for request bodies */
    uint32_t        header_words; /* table words per request header (0: none);
                                     the header of the request in slot i sits
                                     at word i * header_words, and the
                                     INSTANCE input form gives i */
    int32_t         reloc_word;   /* header word holding an offset into the
                                     request's body; the server adds the
                                     body's table position (-1: none) */
    uint32_t        max_requests; /* request slots (in flight at once) */
    uint32_t        slice_rounds; /* regroup rounds per slice (0: 4) */
    const uint32_t* forms;        /* one LOOM_B200_IN_* per kernel input
                                     (ARRAY, IOTA, LOCAL_IOTA, INSTANCE);
                                     NULL: every input an ARRAY */
    loom_b200_budget* budget;     /* shared thread-state budget, or NULL */
} loom_b200_server_cfg;

typedef struct loom_b200_request
{
    uint64_t           n;          /* threads (<= ring_threads) */
    const void* const* inputs;     /* host arrays of the ARRAY-form inputs */
    void* const*       outputs;    /* host arrays that receive the outputs */
    const uint32_t*    header;     /* header_words words (copied at submit) */
    const uint32_t*    body;       /* body_words words, or NULL */
    uint64_t           body_words;
} loom_b200_request;

typedef struct loom_b200_server_stats
{
    uint64_t submitted, admitted, completed;
    uint64_t threads;      /* threads of the completed requests */
    uint64_t slices;       /* megakernel launches */
    uint64_t rounds;       /* regroup rounds over all slices */
    uint64_t queued;       /* submitted, not admitted */
    uint64_t in_flight;    /* admitted, not completed */
    uint64_t unreported;   /* completed, ticket not returned by step yet */
    uint64_t device_bytes; /* device memory the server holds */
    uint64_t thread_instr, warp_instr; /* with opts.profile: lane efficiency */
    uint32_t status;       /* OR of LOOM_B200_STATUS_* */
    uint32_t pad;
    uint64_t budget_waits; /* requests that waited for the budget at least once */
    uint64_t held_bytes;   /* budget bytes held by this server's requests in flight */
    double   busy_ms;      /* device time of the slices (CUDA events on the server's stream) */
    uint64_t slice_t0_ns;  /* the last slice's first CTA start and its end, */
    uint64_t slice_t1_ns;  /* on the GPU's global timer (ns): slices of
                              servers whose intervals intersect ran at once */
} loom_b200_server_stats;

/* `opts`: engine options (population = resident threads; 0: 2^21);
 * `stream`: a cudaStream_t (NULL: the CUDA default stream). */
int loom_b200_server_create(const char*                 kernel,
                            const loom_b200_opts*       opts,
                            const loom_b200_server_cfg* cfg,
                            void*                       stream,
                            loom_b200_server**          out);
int loom_b200_server_destroy(loom_b200_server* s);
/* Queues a request; its host arrays must stay valid until its ticket comes
 * back from loom_b200_server_step (or from loom_b200_server_failed).
 * LOOM_B200_ERR_BUDGET: larger than the ring or the arena. */
int loom_b200_server_submit(loom_b200_server* s, const loom_b200_request* r, uint64_t* ticket);
/* Admits what fits, runs one slice, copies out the requests that finished
 * and returns up to max_done of their tickets (the rest on later calls).
 * After loom_b200_server_launch it completes the slice that call started. */
int loom_b200_server_step(loom_b200_server* s, uint64_t* done, uint32_t max_done, uint32_t* n_done);
/* Admits what fits and starts the next slice without waiting for it, so
 * that the slices of several servers (each on its own stream) run on the
 * GPU at the same time; the next loom_b200_server_step completes it.  With
 * ctas_per_sm > 0 the slice has that many CTAs per SM and runs one round as
 * an ordinary launch (no grid barrier, so it shares the SMs with the other
 * servers' slices; a cooperative launch would not); 0 keeps the server's
 * own launch shape and slice length.  Nothing is launched when no request
 * is in flight or admissible. */
int loom_b200_server_launch(loom_b200_server* s, uint32_t ctas_per_sm);
int loom_b200_server_get_stats(const loom_b200_server* s, loom_b200_server_stats* st);
/* Cancels a request (no counterpart in Loom, whose streams have no request
 * boundary).  A queued request leaves the queue at once.  The threads of a
 * request in flight cannot be taken back from the device: they run to their
 * end, and the request is dropped then (its outputs are not written and its
 * ticket never comes back from loom_b200_server_step).  Either way the
 * ticket comes back once from loom_b200_server_failed with
 * LOOM_B200_ERR_CANCELLED, after which its host arrays are no longer used.
 * LOOM_B200_ERR_INVALID: the ticket is not pending or was cancelled already. */
int loom_b200_server_cancel(loom_b200_server* s, uint64_t ticket);
/* Host-side watchdog: at each loom_b200_server_step, a request submitted
 * more than timeout_us microseconds earlier and not completed is cancelled
 * as above, with LOOM_B200_ERR_TIMEOUT (0, the default: off). */
int loom_b200_server_set_timeout(loom_b200_server* s, uint64_t timeout_us);
/* Hands out up to max tickets of cancelled or timed-out requests, oldest
 * first, with their LOOM_B200_ERR_* code (either array may be NULL). */
int loom_b200_server_failed(loom_b200_server* s, uint64_t* tickets, int32_t* codes, uint32_t max, uint32_t* n);

/* ------------------------------------------------------------ no allocation
 * No counterpart in the reference: Loom's backends allocate their device
 * memory themselves.
 *
 * Runs `kernel` on the regrouping engine like loom_b200_launch_device, but
 * allocates nothing: no cudaMalloc, no cudaFree, no handle.  It is for
 * callers that must not allocate device memory at the point of the call,
 * for instance a plugin inside a host whose caching allocator or memory pool
 * already holds the free memory (cudaMalloc would fail there), or code that
 * must not stall on cudaMalloc's implicit device synchronisation.  The
 * caller passes device pointers for every input, output, instance offset
 * and table of `L`; the engine's queues and control words live in a fixed
 * device array of LOOM_B200_STATIC_SCRATCH_BYTES that each GPU which loads
 * this library holds until the process exits.
 *
 * Limits: at most 2^32 - 1 threads; the threads in flight (`population` of
 * `opts`, or, when that is 0, as many as the array holds) need 2 x row
 * bytes of queue state each (a few tens of bytes for small kernels, 2832 for
 * sphere_pt_f32), and a population the array cannot hold is refused with
 * LOOM_B200_ERR_BUDGET.  `opts` may be NULL (defaults of loom_b200_create);
 * its mode, profile, graph and fault_phantom_ctas fields are ignored.
 *
 * The first call on a device looks up the array's device address (and so
 * loads it onto that device): make that first call before any stream
 * capture.  The address is kept for the life of the process; a process that
 * calls cudaDeviceReset discards the array with the device's other state and
 * must not call this entry point on that device again.  The call waits for
 * its launch before it returns.  Every call shares the array and clears what
 * must start at zero;
 * calls whose launches overlap on the GPU (other streams, other host
 * threads) race on it.  The call returns after the launch finished on
 * `stream` (NULL: the CUDA default stream); *status_out (may be NULL)
 * receives the device status bits, and a non-zero status returns
 * LOOM_B200_ERR_DEVICE. */
#define LOOM_B200_STATIC_SCRATCH_BYTES (64ull << 20)
int loom_b200_launch_static(const char*             kernel,
                            const loom_b200_launch* L,
                            const loom_b200_opts*   opts,
                            void*                   stream,
                            uint32_t*               status_out);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* LOOM_B200_H */
