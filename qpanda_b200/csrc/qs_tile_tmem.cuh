// qs_tile_tmem.cuh - layout of the tiled pass that keeps the tile in tensor
// memory (k_tile_tmem, qs_tile_tmem.cu).
//
// The pass is the same as k_fused_tile's (qs_fused2.cu): 12 tile qubits, up to
// three 5-qubit blocks applied to each 4096-amplitude tile between one read
// and one write of the state.  What differs is where the operands live:
//   * the tile is the MMA's A operand and sits in tensor memory: TMEM lane r
//     holds row r of the block's 128 x 32 complex view, as BF16 hi/lo pairs
//     written with tcgen05.st by the thread that owns the row;
//   * each block's 64 x 64 real matrix (hi and lo) is the B operand in shared
//     memory, loaded once per CTA;
// so a block costs the tensor cores 24 KB of shared-memory operand reads
// (three products of an 8 KB matrix) instead of 72 KB.
//
// Rows and warps.  Row r's bits 0..4 are a warp's lanes, bits 5..6 the four
// warps of a 128-thread lane group (warp w may only touch TMEM lanes
// 32w..32w+31).  Each block has its own assignment of the 12 tile bits to its
// 5 columns (register index bits), 5 lane bits and 2 warp bits: block 0's
// suits the gather, the last block's the stores.  Between two blocks the
// group's 4096 amplitudes go through its staging buffer - each thread writes
// its row's 32 results at their tile positions and reads its row of the next
// block - with a per-transition XOR swizzle that keeps both the write and the
// read phases of a half warp on distinct banks.  A block's matrix is this
// kernel's column order, a bit permutation of the plan's, applied when the
// CTA loads it.
//
// Staging.  Copies land in a 32 KB staging buffer per lane group in tile
// order, with stage bits 1..3 XOR'd by a linear function f of stage bits
// >= 4 (swizzle); each thread then gathers its own block-0 row.  f is chosen
// per pass so that the lanes of one shared-memory phase read distinct banks,
// and being constant on the 8 consecutive chunks of a quarter warp's copy it
// keeps the copies conflict-free.  The buffer is free from the gather until
// the last exchange, after which the next tile's copies are issued into it.
#pragma once

#include <stdint.h>

namespace qs_tmem {

constexpr int kMaxSub = 3;

struct TLayout {
    uint64_t tmask;              // the 12 tile positions (read side) as a mask
    int8_t tpos[12];             // read position of tile bit t (ascending)
    int32_t nsub;
    int32_t pair_in;             // block 0's register bit 0 is tile bit 0: gather column pairs (16 B)
    int32_t vec_out;             // last block's register bit 0 is written at position 0: 16-byte stores
    // gather: stage slot (in amplitudes) of row part and column part, XOR'd
    uint16_t s_lane[5];          // lane bit i of block 0
    uint16_t s_warp[2];          // warp bit v
    uint16_t s_col[32];          // register (column) index j of block 0
    // copies: chunk c = 128 k + t of the tile (tile indices 2c, 2c+1) goes to
    // stage chunk c ^ cf_t(t) ^ cf_k[k]; its global offset is g_t(t) | gk[k]
    uint64_t g_bit[7];           // global offset of chunk bit b (tile bit b + 1), b < 7
    uint64_t gk[16];             // global offset of tile bits 8..11 = k
    uint16_t cf_bit[7];          // stage-chunk XOR of chunk bit b, b < 7
    uint16_t cf_k[16];           // stage-chunk XOR of k
    // exchange before block b + 1 through the staging buffer: block b's value
    // of register j of thread (warp w, lane l) is written at slot
    // xw(w, l) ^ xw_col[b][j]; block b + 1's register j is read from
    // xr(w, l) ^ xr_col[b][j]; xw / xr are XORs of the lane and warp parts
    uint16_t xw_lane[kMaxSub - 1][5], xw_warp[kMaxSub - 1][2], xw_col[kMaxSub - 1][32];
    uint16_t xr_lane[kMaxSub - 1][5], xr_warp[kMaxSub - 1][2], xr_col[kMaxSub - 1][32];
    // matrix of block b: register bit p is matrix index bit mperm[b][p]
    int8_t mperm[kMaxSub][5];
    // stores of the last block: global offsets of its lane bits, warp bits and register index
    uint64_t o_lane[5];
    uint64_t o_warp[2];
    uint64_t o_col[32];
};

// Matrix index (in the plan's order) of a register-order complex index.
__host__ __device__ inline uint32_t tmem_matrix_index(uint32_t jr, const int8_t *perm)
{
    uint32_t j = 0;
    for (int p = 0; p < 5; ++p) j |= ((jr >> p) & 1u) << perm[p];
    return j;
}

// Byte offset of element (n, k) of a 64 x 64 BF16 operand in the K-major,
// 128-byte-swizzled layout the UMMA descriptors describe.
__host__ __device__ inline uint32_t tmem_b_offset(uint32_t n, uint32_t k)
{
    return n * 128 + ((((k >> 3) ^ (n & 7)) & 7) << 4) + ((k & 7) << 1);
}

}  // namespace qs_tmem

struct qs_tiled_desc;
// Host: the TLayout of a tiled pass for k_tile_tmem.  QS_OK, or
// QS_ERR_UNSUPPORTED when the pass does not fit this kernel (tile bit 0 not
// at position 0: its 16-byte copies need adjacent pairs), in which case the
// caller runs the shared-memory kernel.  n: qubits.
int qs_tmem_layout_build(int n, const qs_tiled_desc *d, qs_tmem::TLayout *L);
