// qs_fused.h - host interface of the fused-block tensor-core kernel.
#pragma once
#include <stdint.h>

struct qs_state;

// One fused 5-qubit block: qubits ascending, and the device address of its
// matrix as BF16 bits [2][64][64] (hi then lo) of the real form R of U.
struct qs_fused_desc {
    int qpos[5];
    const void *mat_dev;
    // norm tracking buffers (device, qs_fused_grid() doubles each; may be null)
    const double *norm0;         // input-norm partials of the plan's first pass
    const double *prev_out;      // output-norm partials of the previous pass
    double *in_parts;            // this pass: input-norm partials
    double *out_parts;           // this pass: output-norm partials
};

// CTAs of one fused pass on s (the number of norm partials per pass).
int qs_fused_grid(const qs_state *s);

// After a plan's last pass: scales the state by sqrt(sum(norm0) /
// sum(last_out)) when the two sums (nparts partials each) differ by more than
// 2^-21 relative, decided on the device; complex64 states only (no-op
// otherwise).
int qs_launch_norm_fix(qs_state *s, const double *norm0, const double *last_out, int nparts);

// Launch one block on a complex64 state (n >= 12) on the state's stream.
// err_dev: device int set to 1 if a bounded wait inside the kernel expired.
int qs_launch_fused(qs_state *s, const qs_fused_desc *d, int *err_dev);

// One tiled pass: 12 tile positions T (ascending) and nsub (1..3) blocks,
// each on 5 of them (in the column-bit order of its matrix), applied in
// order; mat_dev holds the blocks' BF16 [2][64][64] matrices back to back.
struct qs_tiled_desc {
    int T[12];
    int nsub;
    int qpos[3][5];
    int has_rows;                // rows[b] = block b's other tile qubits in row-bit order (else ascending)
    int rows[3][7];
    const void *mat_dev;
    const double *norm0;
    const double *prev_out;
    double *in_parts;
    double *out_parts;
    // Where the results go (qs_tile::StoreMap): with has_write, tile bit l
    // (l-th of T) is written at position wtile[l] and tile index bit i at
    // wpos[i] (wmode 2) or 12 + i (wmode 1); otherwise in place.
    int has_write;
    int wtile[12];
    int wmode;
    int wpos[52];
    // Results go to amp_in -> amp_out (device, state-size, distinct) when
    // both are set; in place in the state's buffer otherwise.  Passes with
    // has_write need distinct buffers: a tile's results land where other
    // tiles are still to be read.
    const void *amp_in;
    void *amp_out;
    size_t first_block;          // the plan's index of block 0 of the pass (host bookkeeping)
    int threads_per_row;         // 1: 128 threads per lane, a row each; 2: 256, half a row each
};

int qs_tiled_grid(const qs_state *s);
// Row-bit orders for a pass's blocks that keep warp-wide accesses coalesced
// and the shared-memory stores free of bank conflicts as far as possible
// (qs_tile_layout.cu).  rows[b][i] = global qubit of row bit i.  wtile: the
// write position of each tile bit (NULL: written where read); input_mode 0
// for k_fused_tile's tile-order staging, 1 for k_batch's per-row loads.
int qs_tile_row_orders(int n, const int *T, int nsub, const int (*qpos)[5], int (*rows)[7],
                       const int *wtile = nullptr, int input_mode = 0);
int qs_launch_tiled(qs_state *s, const qs_tiled_desc *d, int *err_dev);
// The same pass on k_tile_tmem (qs_tile_tmem.cu): the tile in tensor memory
// as the MMAs' A operand.  QS_ERR_UNSUPPORTED, with nothing launched and no
// error recorded, for a pass it does not take (then use qs_launch_tiled).
int qs_launch_tiled_tmem(qs_state *s, const qs_tiled_desc *d, int *err_dev);
