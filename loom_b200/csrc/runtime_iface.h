// Interface between the hand-written runtime (runtime.cu) and the generated
// per-kernel translation units (gen/*.cu).
#pragma once

#include <cuda_runtime.h>

#include "engine/regroup.cuh"
#include "loom_b200.h"

namespace loom_b200
{
struct PlainLaunch
{
    Columns             cols;
    unsigned long long  first; // Loom threads [first, first + n)
    unsigned long long  n;
    unsigned long long  max_steps;
    unsigned*           status;
    unsigned long long* counters;
    unsigned            block;
    bool                profile;
    cudaStream_t        stream;
};

struct RegroupLaunch
{
    RegroupParams params;
    unsigned      grid;
    unsigned      block;
    unsigned      regs; // register cap of the megakernel (0: the kernel's default)
    bool          profile;
    // a one-round slice (params.slice_rounds == 1) waits at no grid
    // barrier, so it may be an ordinary launch, which can run on the GPU
    // beside other kernels; every other launch is cooperative (its CTAs
    // resident together, as the grid barrier between rounds needs)
    bool          ordinary = false;
    unsigned      dyn_smem = 0; // dynamic shared memory (bulk_restore's staging)
    // false: the launch never parks (schedule 2 or 3, no period), does not
    // prefetch and runs the megakernel compiled without queue code
    bool          park = true;
    cudaStream_t  stream;
};

/// Where one queue's columns lie in a row of the regrouping state: the
/// values of column c sit in slots of col_width[c] bytes per entry (16 for
/// four 32-bit values packed together), `cap` slots from byte
/// `col_off[c] * cap` of the state half of the round's parity, at byte
/// col_sub[c] of each slot; the thread ids (low 32 bits) likewise at
/// tid_off / tid_sub / tid_width.
struct QueueSegment
{
    const unsigned long long* col_off;
    const unsigned*           col_sub;
    const unsigned*           col_width;
    unsigned long long        tid_off;
    unsigned                  tid_sub;
    unsigned                  tid_width;
};

/// One compiled kernel: its descriptor and the launchers of both engines.
struct KernelEntry
{
    const loom_b200_kernel_info* info;
    unsigned long long           row_bytes;  // queue bytes per entry, summed over queues
    unsigned                     num_queues; // work queues of the regrouping engine
    cudaError_t (*plain)(const PlainLaunch&);
    cudaError_t (*regroup)(const RegroupLaunch&);
    cudaError_t (*regroup_occupancy)(int block, bool profile, unsigned regs, unsigned dyn_smem, bool park,
                                     int* ctas_per_sm);
    const loom_b200_queue_layout* queues;   // num_queues entries
    const QueueSegment*           segments; // num_queues entries
    const unsigned*               reg_caps; // compiled register caps, default first
    unsigned                      num_reg_caps;
    unsigned                      max_stage_row; // K::kMaxStageRow (bulk_restore staging per entry)
};

extern const KernelEntry* const kRegistry[];
extern const int                kRegistrySize;
} // namespace loom_b200
