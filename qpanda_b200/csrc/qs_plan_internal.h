// qs_plan_internal.h - the fusion plan's structure, shared by the planner
// (qs_plan.cpp) and the batched executor (qs_batch.cu).
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <vector>

#include "../../include/qpanda_b200.h"

typedef std::complex<double> cd;

struct PlanBlock {
    int k = 0;
    int q[5] = {0, 0, 0, 0, 0};          // ascending global qubits
    std::vector<cd> U;                   // 32 x 32 row-major
    std::vector<size_t> gates;           // indices into the gate list, in application order
};

// A pass of the tiled kernel: one read and one write of the state, applying
// up to 3 consecutive blocks (sub-blocks) whose qubits lie in the 12 tile qubits.
struct PlanPass {
    int T[12] = {0};                     // ascending global qubits of the tile
    size_t first = 0, count = 0;         // its blocks: blocks[first, first + count)
    int rows[3][7] = {};                 // each block's other tile qubits in row-bit order (qs_tile_row_orders)
};

struct qs_plan {
    int n = 0;
    int max_k = 5;
    qs_plan_opts opts;
    std::vector<qs_gate> gates;
    std::vector<PlanBlock> blocks;
    std::vector<PlanPass> passes;        // tiled kernel only
    int dev = -1;                        // device holding mats
    void *mats = nullptr;                // [blocks][2][64][64] bf16
    cudaStream_t mats_stream = nullptr;  // stream-ordered mats: freed with cudaFreeAsync on it
    bool mats_async = false;
    // the last tiled schedule (qs_plan_tiled_schedule) and what it was for
    std::vector<struct qs_tiled_desc> sched;
    std::vector<int> sched_dst;
    size_t sched_first = 0, sched_count = 0;
    int sched_remap = -1;
};


// A plan with the same structure as `proto` (same passes and blocks) for a
// gate list with the same operations on the same qubits - only angles may
// differ - with the block unitaries recomputed.  QS_ERR_ARG if the gate
// pattern differs.
int qs_plan_rebind(const qs_plan *proto, const qs_gate *gates, size_t count, qs_plan **out);
// 2 x 64 x 64 BF16 bits (hi, lo) of block b's real matrix form.
void qs_plan_block_bf16(const qs_plan *P, size_t b, uint16_t *out);

struct qs_tiled_desc;
// Launch descriptors of tiled passes [first, first + count) of P on an
// n-qubit state (buffers and norm pointers left empty), and for each pass
// the buffer it writes: -1 in place, 0 the state's own, 1 the spare (reading
// the other).  With remap (qs_plan_opts.remap), passes ping-pong through the
// spare buffer, each writing the layout that makes its own stores (1) or the
// next pass's loads (2) contiguous tiles, and the last writes the natural
// order; the state's own buffer holds the result.  Pure host code (also used by the CPU
// emulation test of the tiled passes).
int qs_plan_tiled_schedule(const qs_plan *P, int n, size_t first, size_t count, int remap,
                           std::vector<qs_tiled_desc> &descs, std::vector<int> &dst);
