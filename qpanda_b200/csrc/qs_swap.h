// qs_swap.h - host interface of the in-place half-slice swap (qs_swap.cu).
#pragma once
#include <stddef.h>

#include <cuda_runtime.h>

// Swap, element for element, rows [r0, r0 + nr) x bytes [c0, c0 + w) of two
// regions of rows `width` bytes wide and `pitch` bytes apart, starting at a
// and b (device memory of this GPU, or a peer's that this GPU can address).
// w must be a power-of-two count of 8-byte units (16-byte ones are used when
// every size and both bases allow).  Asynchronous on `stream`.
int qs_launch_swap_halves(void *a, void *b, size_t width, size_t pitch, size_t r0, size_t nr, size_t c0,
                          size_t w, cudaStream_t stream);
