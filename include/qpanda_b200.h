/*
 * qpanda_b200.h - C ABI of the B200 state-vector gate backend.
 *
 * This is the thin, plain-C layer between the C++ host code (the QuantumGates
 * subclass in qpanda_b200/host/) and the sm_100a CUDA kernels.  Every entry
 * point takes plain pointers and sizes; no C++ or torch types cross it.
 *
 * Each entry point below cites the reference interface it replaces, as
 * "path:line" inside the QPanda 2018 SDK tree (QPandaSDK/...).  The reference
 * reached its GPU code through dlsym() by name with C++ reference arguments
 * (QPandaSDK/GPUEmulator/GPUGatesDecl.h:38-75); this header replaces that
 * with a real extern "C" ABI.
 *
 * Conventions
 *  - Qubit q is bit q of the amplitude index (little-endian), as in
 *    QPandaSDK/QuantumInstructionHandle/CPUQuantumGates.cpp.
 *  - Amplitudes are interleaved complex (re, im): complex64 = 2 x float,
 *    complex128 = 2 x double.
 *  - Return value: QS_OK (0) on success, a negative QS_ERR_* code otherwise;
 *    qs_last_error() then holds a message for the calling thread.
 *  - Calls that return host-visible results (measure, probabilities, samples,
 *    get_state, norms) synchronize the state's stream.  Gate calls are
 *    asynchronous on that stream; an error in an asynchronous kernel is
 *    reported by the next synchronizing call.
 */
#ifndef QPANDA_B200_H
#define QPANDA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define QS_OK               0
#define QS_ERR_ARG         -1   /* bad argument: qubit out of range, duplicate qubit, bad dtype */
#define QS_ERR_CUDA        -2   /* CUDA runtime error */
#define QS_ERR_OOM         -3   /* device memory exhausted */
#define QS_ERR_UNSUPPORTED -4   /* valid request this build does not provide */
#define QS_ERR_NOT_UNITARY -5   /* matrix failed the |det|==1 check (CPUQuantumGates.cpp:1182-1186) */
#define QS_ERR_STATE       -6   /* state handle is unusable (e.g. a measured probability of 0) */
#define QS_ERR_IO          -7   /* a file could not be opened or written */

/* ---- element types ----------------------------------------------------- */
#define QS_C64   0              /* complex64: float re, float im  */
#define QS_C128  1              /* complex128: double re, double im */

/* ---- gate records (one per reference QuantumGates method) -------------- */
/* Operation codes.  Each names the QuantumGates virtual it reproduces
 * (QPandaSDK/QuantumInstructionHandle/QuantumGates.h). */
#define QS_OP_H         1   /* Hadamard(qn)                         QuantumGates.h:56,87   */
#define QS_OP_X         2   /* NOT(qn)                              QuantumGates.h:396,409 */
#define QS_OP_RX        3   /* RX(qn, theta, dagger)                QuantumGates.h:115,146 */
#define QS_OP_RY        4   /* RY(qn, theta, dagger)                QuantumGates.h:163,176 */
#define QS_OP_RZ        5   /* RZ(qn, theta, dagger)                QuantumGates.h:194,211 */
#define QS_OP_CNOT      6   /* CNOT(q[0]=control, q[1]=target)      QuantumGates.h:229,242 */
#define QS_OP_CR        7   /* CR(q[0], q[1], theta, dagger)        QuantumGates.h:261     */
#define QS_OP_ISWAP     8   /* iSWAP(q[0], q[1], dagger)            QuantumGates.h:274,292 */
#define QS_OP_SQISWAP   9   /* sqiSWAP(q[0], q[1], dagger)          QuantumGates.h:310,328 */
#define QS_OP_TOFFOLI  10   /* toffoli(q[0], q[1] controls, q[2])   QuantumGates.h:425     */
#define QS_OP_CSWAP    11   /* controlSwap(q[0] control, q[1], q[2]) QuantumGates.h:345    */
#define QS_OP_SWAP     12   /* SWAP(q[0], q[1]); no reference method: QRunes writes it as 3 CNOTs */

#define QS_MAX_CTRL    16

/* One gate.  q[] holds the operands in the order of the reference method's
 * arguments; ctrl[0..nctrl) are the extra control qubits of a QRunes CONTROL
 * block (the reference passes them with the target appended,
 * QPandaSDK/QuantumInstructionHandle/Instruction.cpp:62,155,243); the gate then
 * acts on the subspace where every control qubit is 1.  dagger follows the
 * reference's iDagger argument.  96 bytes, 8-byte aligned. */
typedef struct qs_gate {
    int32_t op;
    int32_t dagger;
    int32_t q[3];
    int32_t nctrl;
    int32_t ctrl[QS_MAX_CTRL];
    double  theta;
} qs_gate;

typedef struct qs_state qs_state;   /* opaque: one state vector resident in HBM */

/* ---- errors ------------------------------------------------------------- */
/* Message for the last failing call on this thread ("" if none). */
const char *qs_last_error(void);
/* Library build string (architecture, version). */
const char *qs_version(void);

/* ---- state lifetime ----------------------------------------------------- */
/* Allocate 2^n_qubits amplitudes of dtype on the current CUDA device and set
 * |0...0>.  stream: a cudaStream_t (NULL = the legacy default stream).
 * Replaces QuantumGates::initState (QuantumGates.h:376;
 * CPUQuantumGates.cpp:1136-1157; GPU: GPUEmulator/GPUGates.cu:1208-1299). */
int qs_create(int n_qubits, int dtype, void *stream, qs_state **out);
/* As qs_create, with stream-ordered memory: the state's buffers come from
 * cudaMallocAsync on `stream` and go back with cudaFreeAsync in qs_destroy, so
 * creating and destroying states never synchronizes the device (serving). */
int qs_create_async(int n_qubits, int dtype, void *stream, qs_state **out);
/* Free the state.  Replaces QuantumGates::destroyState (QuantumGates.h:438). */
int qs_destroy(qs_state *s);
int qs_num_qubits(const qs_state *s, int *n_qubits);
int qs_dtype(const qs_state *s, int *dtype);
/* Device address of the amplitude array (for zero-copy interop). */
int qs_device_ptr(const qs_state *s, void **dev_ptr);
int qs_set_stream(qs_state *s, void *stream);
int qs_synchronize(qs_state *s);

/* |0...0>.  Replaces endGate, which the dispatcher sends before every run
 * (CPUQuantumGates.cpp:1445-1453; QuantumInstructionHandleAPI.cpp:96-100). */
int qs_reset_zero(qs_state *s);
/* Copy a host state in (host_dtype QS_C64 or QS_C128; converted as needed). */
int qs_set_state(qs_state *s, const void *host_amps, int host_dtype);
/* Copy the state out.  Replaces getQState's data path (QuantumGates.h:46;
 * CPUQuantumGates.cpp:64-82; GPUGates.cu:2160-2169) without the 6-digit text. */
int qs_get_state(qs_state *s, void *host_out, int host_dtype);

/* ---- gates (reference conventions, CPUQuantumGates.cpp) ----------------- */
/* Apply one gate record.  Conventions follow CPUQuantumGates.cpp: RZ is
 * diag(e^{-i t/2}, e^{+i t/2}) (:524-570), CR multiplies |11> by e^{+i t}
 * (:773-825), iSWAP maps |01> -> +i|10> (:838-899), H and sqiSWAP use
 * SQ2 = 0.707106781186548 (:36).  Controlled iSWAP / sqiSWAP, which the
 * reference leaves as no-ops (:914-922, :1054-1062), act on the control=1
 * subspace here. */
int qs_gate_apply(qs_state *s, const qs_gate *g);
/* Apply count gate records in order (one launch per gate, no fusion). */
int qs_gates_apply(qs_state *s, const qs_gate *g, size_t count);

/* ---- generic unitaries (the kernels the gate records lower to) --------- */
/* Dense 2x2 on qubit q, row-major complex m = {m00, m01, m10, m11} as 8
 * doubles (re, im), acting where all bits of ctrl_mask are 1.  Replaces
 * unitarySingleQubitGate (QuantumGates.h:367; CPUQuantumGates.cpp:1170-1212),
 * whose stride is POW2(qn-1) in the reference; this entry uses 2^q. */
int qs_apply_1q(qs_state *s, int q, const double m[8], uint64_t ctrl_mask);
/* Same with the reference's unitarity check |det| within 1e-6 of 1. */
int qs_apply_unitary_1q(qs_state *s, int q, const double m[8]);
/* Dense 4x4 on (q0, q1); basis index b = bit(q0) + 2*bit(q1); row-major
 * complex m as 32 doubles. */
int qs_apply_2q(qs_state *s, int q0, int q1, const double m[32], uint64_t ctrl_mask);
/* 2x2 on the pair {|a=1,b=0>, |a=0,b=1>} (iSWAP / sqiSWAP / SWAP family),
 * m row-major over (a-set, b-set). */
int qs_apply_exchange(qs_state *s, int a, int b, const double m[8], uint64_t ctrl_mask);
/* Multiply every amplitude whose index has all bits of mask set by
 * (re + i im): CR / CZ / controlled phase. */
int qs_apply_phase(qs_state *s, uint64_t mask, double re, double im);

/* ---- measurement and probabilities (FP64 accumulation) ------------------ */
/* P(qubit q == 0) = sum |a|^2 over bit q == 0. */
int qs_prob_zero(qs_state *s, int q, double *p0);
/* qubitMeasure with the uniform u supplied by the caller (QuantumGates.h:356;
 * CPUQuantumGates.cpp:1071-1126): outcome = ((float)u > p0), then the kept
 * half is scaled by 1/sqrt(p) and the other half zeroed.  The reference draws
 * u from its 16807 generator (QuantumGates.cpp:46-85). */
int qs_measure(qs_state *s, int q, double u, int *outcome);
/* Full marginal distribution over m qubits: out[idx] (2^m doubles, host),
 * idx bit j = qubit qubits[j].  This is the un-truncated vector that
 * pMeasure builds (QuantumGates.h:75; CPUQuantumGates.cpp:159-190). */
int qs_probs(qs_state *s, const int *qubits, int m, double *out);
/* qs_probs into a device buffer of 2^m doubles, asynchronous on the state's stream. */
int qs_probs_device(qs_state *s, const int *qubits, int m, double *dev_out);
/* pMeasure as the reference returns it: the marginal sorted by descending
 * probability and cut to the first 10 entries (CPUQuantumGates.cpp:178-189).
 * idx_out/p_out hold up to 10 entries; *count receives how many. */
int qs_pmeasure(qs_state *s, const int *qubits, int m, uint64_t *idx_out,
                double *p_out, int *count);
/* Shots: for each shot s, measure qubits[0], qubits[1], ... in order with
 * uniforms u[s*m + k] under qubitMeasure semantics (sequential collapse and
 * renormalisation), without modifying the state.  out[s] bit k = outcome of
 * qubits[k].  Equivalent to re-running the circuit once per shot with
 * terminal MEASUREs, as QPandaSDK::run does (QPandaAPI.cpp:173-182). */
int qs_sample(qs_state *s, const int *qubits, int m, const double *u,
              size_t shots, uint64_t *out);
/* sum |a|^2 */
int qs_norm2(qs_state *s, double *norm2);
/* <a|b> = sum conj(a_i) b_i, FP64 accumulation; a and b may differ in dtype. */
int qs_inner(qs_state *a, qs_state *b, double *re, double *im);
/* max_i |a_i - b_i| and sum_i |a_i - b_i|^2 on the device (dtypes may differ). */
int qs_diff(qs_state *a, qs_state *b, double *max_abs, double *sum_sq);

/* Measurement of qubit q for callers that cannot allocate memory when they
 * measure.  No counterpart in the reference.  qs_measure keeps its reduction
 * partials in scratch that qs_create allocated; this entry point allocates
 * nothing (no cudaMalloc, cudaFree or allocating library call) and needs no
 * qs_state, for a serving loop that reserved all device memory up front, a
 * framework whose own allocator owns the device memory, or a caller that holds
 * the amplitudes in a buffer of its own.  amp: 2^n_qubits amplitudes of dtype
 * on the current device (8-byte aligned for complex64, 16-byte for
 * complex128), collapsed in place: with p0 = P(qubit q == 0) summed in FP64,
 * the outcome is 1 when (float)u > p0, else 0; the half of the state with the
 * outcome is scaled by 1/sqrt(p) (p = p0 or 1 - p0) and the other half set to
 * zero.  outcome_dev / p0_dev: device words that receive the outcome (-1 if
 * the selected outcome has probability 0, state left unchanged) and p0.
 * Asynchronous on `stream`.  Its partial sums live in a fixed 512 KB device
 * array compiled into the library (held on every GPU that loads it until
 * exit), which limits states to at most 32 qubits; larger ones are rejected
 * with QS_ERR_ARG.  The first call on a device looks up that array's address
 * (cudaGetSymbolAddress) and keeps it: make that call before any stream
 * capture on the device, and do not reset the device (cudaDeviceReset)
 * between calls.  All calls share the array, so calls that overlap on the GPU
 * (unordered streams) race; calls ordered on one stream do not. */
int qs_measure_noalloc(void *amp, int n_qubits, int dtype, int q, double u,
                       int *outcome_dev, double *p0_dev, void *stream);

/* ---- fused path: gate runs -> dense 5-qubit blocks on the tensor cores ---- */
/* The reference applies every gate as its own pass over the state
 * (QuantumInstructionGet.cpp:104-124 -> one CPUQuantumGates method each).  A
 * plan groups the gate list into dense blocks of up to max_k (<= 5) qubits,
 * each applied in one pass as a 32x32 complex contraction on the tensor cores
 * (split-BF16 x3 products, FP32 accumulation) for complex64 states of at
 * least 12 qubits; other states run the plan's gates through the per-gate
 * kernels.  No reference counterpart (the reference has no gate fusion). */
typedef struct qs_plan qs_plan;
/* Single-block passes: one dense block of up to max_k qubits per pass. */
int qs_plan_create(int n_qubits, const qs_gate *gates, size_t count, int max_k, qs_plan **out);

#define QS_PLAN_SINGLE 1   /* one 5-qubit block per read+write of the state */
#define QS_PLAN_TILED  2   /* up to max_sub 5-qubit blocks per read+write, within 12 tile qubits */
typedef struct qs_plan_opts {
    int block_qubits;      /* fusion width of one block, 1..5 */
    int tile_qubits;       /* tiled passes: qubits per tile (12) */
    int max_sub;           /* tiled passes: blocks per pass, 1..3 */
    int low_qubits;        /* tiled passes: qubits 0..low_qubits-1 always in the tile (1..5) */
    int kernel;            /* QS_PLAN_SINGLE or QS_PLAN_TILED */
    int remap;             /* tiled passes of states of >= 20 qubits: 0 = in place (default); 1 = every
                              pass but the last writes its tiles as contiguous runs into a second
                              state-size buffer (held by the state from its first such plan until
                              qs_destroy or qs_release_spare) and the last writes the natural order
                              back; 2 = as 1, but each pass writes the layout in which the next pass's
                              tiles are contiguous (loads stream, stores scatter; measured slower) */
    int threads_per_row;   /* tiled passes: 1 = each of a lane's 128 threads owns a row of the tile (default);
                              2 = 256 threads per lane, two per row, each with 16 of its 32 columns
                              (measured slower on both tiled kernels: 3-4 % with the tile in shared
                              memory, 20 % with it in tensor memory, where 64 registers a thread spill) */
    int tile_in_tmem;      /* tiled passes: 1 = the tile is the MMAs' A operand in tensor memory and the
                              block matrices the B operand in shared memory (default), for every pass
                              with position 0 in its tile; other passes, and 0, keep the tile in
                              shared memory */
} qs_plan_opts;
/* Defaults: 5-qubit blocks, tiled passes of 12 qubits with up to 2 blocks
 * (a pass of 3 blocks saves a pass but runs on a kernel with fewer resident
 * CTAs, and measured slower overall), qubits 0..2 in every tile, in place,
 * one thread per tile row.  Fill a qs_plan_opts with this call before
 * changing fields: the struct may gain fields at its end. */
int qs_plan_default_opts(qs_plan_opts *opts);
int qs_plan_create_ex(int n_qubits, const qs_gate *gates, size_t count, const qs_plan_opts *opts,
                      qs_plan **out);
/* Pick a circuit's plan options by measurement: plans of `gates` with
 * tile_in_tmem 0 and 1, max_sub 2 and 3 and low_qubits 2 and 3 - and 1 for a
 * remapping base, whose passes read the qubits they share with the previous
 * pass as contiguous runs anyway - (the other fields from *base, or the
 * defaults when base is NULL) are each applied to
 * s once untimed and `reps` times timed with CUDA events on the state's
 * stream; *best gets the options of the fastest and *best_ms (may be NULL)
 * its mean time per application.  Overwrites the state: reset it after.
 * States below 12 qubits have no tiled passes: *best = the base options.
 * No reference counterpart (the reference applies gates one at a time). */
int qs_plan_autotune(qs_state *s, const qs_gate *gates, size_t count, const qs_plan_opts *base, int reps,
                     qs_plan_opts *best, double *best_ms);
/* Kernel launches (passes) the plan makes per application. */
int qs_plan_launches(const qs_plan *plan, size_t *n_launches);
int qs_plan_destroy(qs_plan *plan);
int qs_plan_info(const qs_plan *plan, size_t *n_blocks, size_t *n_gates);
/* Block i: its 5 qubits (ascending) and its 32x32 unitary, row-major complex
 * as 2048 doubles (either output may be NULL).  Row/column index bit b is
 * qubit qubits[b]. */
int qs_plan_block(const qs_plan *plan, size_t i, int *k, int *qubits, double *matrix);
/* Pass i of a tiled plan: its number of blocks (1..3), its 12 tile qubits
 * (ascending) and each block's 5 qubits, row-major [3][5] (rows past
 * *n_blocks untouched).  Any output may be NULL.  QS_ERR_ARG for a plan
 * without tiled passes or i out of range.  No reference counterpart:
 * introspection of this backend's fusion plan. */
int qs_plan_pass(const qs_plan *plan, size_t i, int *n_blocks, int *tile_qubits, int *block_qubits);
/* Apply every block in order (asynchronous, on the state's stream).  The
 * norm is kept to the input's: each pass rescales by the drift of the one
 * before, and after the last pass the state is rescaled on the device when
 * its norm differs from the input's by more than 2^-21 relative. */
int qs_plan_apply(qs_state *s, qs_plan *plan);
/* Apply launches (passes) [first, first + count) only (for timing or
 * interleaving); a range that ends at the plan's last pass ends with the
 * closing rescale. */
int qs_plan_apply_range(qs_state *s, qs_plan *plan, size_t first, size_t count);
/* Synchronize and report whether a bounded wait inside a fused pass expired
 * since the last qs_plan_apply (QS_ERR_STATE) - a watchdog, not expected. */
int qs_plan_status(qs_state *s);
/* Self-test of the bounded waits above: one kernel waits wait_us
 * microseconds (1 us .. 2 s) on an mbarrier that nothing arrives on, gives up,
 * and sets the word that qs_plan_status reads, which then returns
 * QS_ERR_STATE; the context stays usable.  Asynchronous on the state's
 * stream.  No reference counterpart (the reference's kernels have no
 * waits). */
int qs_watchdog_selftest(qs_state *s, unsigned wait_us);
/* Free the second state-size buffer that plans with remap = 1 keep with the
 * state (no-op when there is none).  No reference counterpart. */
int qs_release_spare(qs_state *s);

/* ---- result formats ------------------------------------------------------ */
/* Write the state to "<path_prefix>.fullstate" (binary = 0) or
 * "<path_prefix>.fullstate.binary" (binary = 1), streamed from the device in
 * chunks (the whole state never sits in host memory at once).
 * Text: the reference's getQState text, one line per amplitude,
 *   "state[i].real = <re> state[i].imag = <im>\n" with the default C++ stream
 *   formatting (6 significant digits), which QCommandRun::saveQstate writes
 *   verbatim (QPandaSDK/QuantumCommandControl/QCommand.cpp:402-428,
 *   CPUQuantumGates.cpp:64-82).
 * Binary: per amplitude the record { double real; double imag; } in native
 *   byte order, index order - the layout QCommandRun::saveQstateBinary declares
 *   (QCommand.cpp:437-480); the reference fills it by parsing the text lines
 *   with atof, which yields 0.0 and an unset imaginary part, so its files do
 *   not hold the amplitudes; this writer stores the amplitudes.
 * complex64 states are widened to double for both.  Synchronizes the state's
 * stream.  QS_ERR_IO if the file cannot be written. */
int qs_write_fullstate(qs_state *s, const char *path_prefix, int binary);

/* The result text of QPandaSDK::getResult (QPandaAPI.cpp:220-238): one line
 * "<key> <value>\n" per outcome, the key as a width-bit binary string, most
 * significant bit first (QPandaSDK::integerToBinary, QPandaAPI.cpp:295-305),
 * the value with the default stream formatting, lines in ascending key order
 * (the reference's std::map<string, double>).  For PMEASURE results the keys
 * are pMeasure indices (width = number of measured qubits); for MEASURE
 * results they are the classical-register bit strings read as numbers
 * (width = number of registers) and the values their frequencies.  Writes at
 * most cap bytes including the terminating NUL into buf (buf may be NULL to
 * query); *needed receives the full length including the NUL.  Duplicate keys
 * are rejected (QS_ERR_ARG), as a map cannot hold them. */
int qs_format_outcomes(const uint64_t *keys, const double *values, size_t count, int width, char *buf,
                       size_t cap, size_t *needed);

/* ---- batched circuits: many circuits in one persistent launch ---------- */
/* The reference runs one program per QPandaSDK::run (QPandaAPI.cpp:131-211); a
 * parameter sweep is a host loop over runs.  A batch holds many independent
 * circuits (up to 24 qubits each; narrower than 12 are padded with idle
 * qubits), each with its own state in HBM and its own fused plan, and runs
 * them all from |0...0> in one persistent kernel launch (captured in a CUDA
 * graph when use_graph is set): the CTAs take whole circuits from a queue.
 * After a run, qs_batch_zz gives every circuit's nearest-neighbour
 * <Z_i Z_{i+1}> (i = 0..n-2), i.e. P00 + P11 - P01 - P10 of the pMeasure
 * marginal on (i, i+1) (CPUQuantumGates.cpp:159-190).  No reference
 * counterpart beyond that loop. */
typedef struct qs_batch qs_batch;
#define QS_BATCH_LONGEST_FIRST 0
#define QS_BATCH_INPUT_ORDER   1
typedef struct qs_batch_opts {
    int max_sub;           /* fused blocks per pass, 1..3 (default 2: three CTAs per SM) */
    int low_qubits;        /* qubits 0..low_qubits-1 in every tile, 1..5 */
    int order;             /* QS_BATCH_LONGEST_FIRST or QS_BATCH_INPUT_ORDER */
    int use_graph;         /* capture the launch in a CUDA graph and replay it */
    int block_qubits;      /* fusion width: gates are grouped into blocks of at most 4 or 5 qubits
                              (default 5; applied as 5-qubit blocks either way) */
    int tile_in_tmem;      /* with max_sub <= 2: 1 = the tile in tensor memory as the MMAs' A operand
                              (k_batch_tmem, default), 0 = in shared memory (k_batch) */
} qs_batch_opts;
/* Defaults (2 blocks per pass, 3 low qubits, longest first, graph, 5-qubit
 * fusion, the tile in tensor memory).  Fill a qs_batch_opts with this call before changing fields: the
 * struct may gain fields at its end. */
int qs_batch_default_opts(qs_batch_opts *opts);
/* Circuit c has n_qubits[c] qubits and gates[offsets[c] .. offsets[c+1]). */
int qs_batch_create(int n_circuits, const int *n_qubits, const qs_gate *gates, const size_t *offsets,
                    const qs_batch_opts *opts, qs_batch **out);
/* Run every circuit from |0...0> (asynchronous on `stream`). */
int qs_batch_run(qs_batch *b, void *stream);
/* Synchronize; copy the <Z_i Z_{i+1}> of all circuits, concatenated in
 * circuit order (out may be NULL to query *count). */
int qs_batch_zz(qs_batch *b, double *out, size_t *count);
/* offsets[c] = first output of circuit c in qs_batch_zz's array; n+1 entries. */
int qs_batch_zz_offsets(const qs_batch *b, size_t *offsets);
/* Final state of circuit c (2^n_qubits[c] amplitudes) to the host. */
int qs_batch_state(qs_batch *b, int circuit, void *host_out, int host_dtype);
int qs_batch_info(const qs_batch *b, size_t *state_bytes, size_t *passes_total);
int qs_batch_destroy(qs_batch *b);
/* Autotuner: build and time candidate options (fusion width 4 or 5 qubits,
 * blocks per pass 1..3, lowest tile qubits 3 or 5, queue order) on every
 * stride-th circuit and write the fastest to *best (with use_graph set) and
 * its time per run to *best_ms. */
int qs_batch_autotune(int n_circuits, const int *n_qubits, const qs_gate *gates, const size_t *offsets,
                      int stride, qs_batch_opts *best, double *best_ms);
/* The same, with the result kept in a text file: cache_path holds one line
 * per tuning, keyed by the device (name, SM count) and the sampled circuits'
 * gate pattern (operations and qubits; angles do not change the timing).  A
 * key found there is returned without timing anything (*from_cache = 1); a
 * new one is tuned and appended (*from_cache = 0).  No reference counterpart. */
int qs_batch_autotune_cached(int n_circuits, const int *n_qubits, const qs_gate *gates, const size_t *offsets,
                             int stride, const char *cache_path, qs_batch_opts *best, double *best_ms,
                             int *from_cache);

/* ---- sharded states: 2^g shards of 2^(n-g) amplitudes ------------------- */
/* For states beyond one GPU (33 qubits and up in complex64).  The top g
 * physical positions of the amplitude index select the shard; logical qubit
 * q sits at physical position pos[q] (qs_sharded_positions).  Gates on local
 * positions run on every shard without communication; a gate on a global
 * qubit first swaps it with a local position the gate does not use - the two
 * shards that differ in that rank bit exchange half of their slices.  The
 * reference has no counterpart (it caps programs at 30 qubits,
 * QPandaAPI.cpp:87).
 * A process holds some of the shards (ranks[0..n_ranks), on the current
 * device): two local shards swap in place with one kernel; a shard whose
 * partner is elsewhere swaps with it over peer memory (qs_sharded_set_peer)
 * or calls `exchange` for each piece (at most 256 MB) of its half:
 * send `bytes` of device memory at `send` to shard `partner`, receive as many
 * from it into `recv` (distinct device buffers of the library), and return 0
 * once `recv` holds them - e.g. an NCCL send/receive pair on `stream`
 * followed by a stream synchronization.  Shard 0 starts in |0...0>, the
 * others at zero. */
typedef struct qs_sharded qs_sharded;
typedef int (*qs_exchange_fn)(void *ctx, int shard, int partner, const void *send, void *recv, size_t bytes,
                              void *stream);
int qs_sharded_create(int n_qubits, int n_global, int dtype, const int *ranks, int n_ranks,
                      qs_exchange_fn exchange, void *ctx, qs_sharded **out);
/* Apply gate records (logical qubits); synchronous at every swap. */
int qs_sharded_apply(qs_sharded *s, const qs_gate *gates, size_t count);
/* Peer swaps with shard `partner`, whose amplitudes this process can address
 * at `partner_amp`: a peer GPU's buffer (peer access enabled) or an IPC
 * mapping (cudaIpcOpenMemHandle) of another process's shard, 16-byte aligned
 * (qs_device_ptr of that shard, exported by its owner).  A swap with that
 * partner then runs as one kernel on each side that reads and writes both
 * halves in place - over NVLink when the partner is another GPU - with no
 * staging buffer, packing or exchange call: the side with the rank bit 0
 * swaps the first half of the rows, the other side the second.  Before and
 * after each such swap this side calls barrier(ctx, shard, partner), which
 * returns 0 once the partner has made the same call (this side's earlier work
 * on its shard is complete before the first call, its part of the swap before
 * the second).  Replaces the exchange function for that partner.  The
 * reference has no counterpart. */
typedef int (*qs_barrier_fn)(void *ctx, int shard, int partner);
int qs_sharded_set_peer(qs_sharded *s, int partner, void *partner_amp, qs_barrier_fn barrier, void *ctx);
/* The local shard with these rank bits (a qs_state of n - g qubits). */
int qs_sharded_shard(qs_sharded *s, int rank, qs_state **shard);
/* pos[q] = physical position of logical qubit q (n entries). */
int qs_sharded_positions(const qs_sharded *s, int *pos);
/* Swaps so far, and bytes this process's shards sent plus received. */
int qs_sharded_info(const qs_sharded *s, size_t *swaps, size_t *bytes_moved);
int qs_sharded_destroy(qs_sharded *s);

/* ---- request loop: continuous batching on one GPU ----------------------- */
/* Requests (a circuit, plus 1024-style shots or the full probability vector)
 * are submitted at any time; `slots` worker threads with their own streams
 * take them in arrival order (or up to `bypass` places past a head that does
 * not fit yet) when their HBM footprint - state, scratch and, for
 * probabilities, the output vector - fits `hbm_budget_bytes` beside the
 * requests already on the device.  Requests overlap on the GPU; states use
 * stream-ordered memory.  A request's result does not depend on what else
 * runs.  The reference's counterpart is one QPandaSDK::run per program
 * (QPandaAPI.cpp:131-211) and its remote cloud mode
 * (QuantumCloudHTTP.cpp:117-191). */
typedef struct qs_server qs_server;
#define QS_REQ_SHOTS 1     /* sample shots of all qubits (qs_sample semantics) into out_host */
#define QS_REQ_PROBS 2     /* full 2^n probability vector, held on the device */
#define QS_MAX_QUBITS_SERVED 32
typedef struct qs_server_opts {
    size_t hbm_budget_bytes;
    int slots;             /* concurrent requests (worker threads / streams), 1..64 */
    int bypass;            /* admission may skip this many non-fitting requests */
} qs_server_opts;
int qs_server_default_opts(qs_server_opts *opts);
int qs_server_create(const qs_server_opts *opts, qs_server **out);
/* Queue a request; returns at once with its id.  For QS_REQ_SHOTS, uniforms
 * holds shots x n_qubits values (u[s*n + k] for qubit k of shot s) and
 * out_host receives the shots; out_host must stay valid until the request is
 * done.  QS_ERR_OOM if the request alone exceeds the budget. */
int qs_server_submit(qs_server *srv, int n_qubits, const qs_gate *gates, size_t count, int kind,
                     const double *uniforms, size_t shots, uint64_t *out_host, uint64_t *id);
/* Block until the request is done; latency = submit -> result ready, service =
 * admitted -> result ready.  Returns the request's status. */
int qs_server_wait(qs_server *srv, uint64_t id, double *latency_s, double *service_s);
/* Copy a QS_REQ_PROBS result (2^n doubles) to the host. */
int qs_server_fetch_probs(qs_server *srv, uint64_t id, double *host_out);
/* Forget a finished request and free its held result. */
int qs_server_release(qs_server *srv, uint64_t id);
int qs_server_stats(qs_server *srv, size_t *served, size_t *max_concurrent, size_t *hbm_in_use);
/* Stop: queued requests end with QS_ERR_STATE, running ones finish. */
int qs_server_destroy(qs_server *srv);

#ifdef __cplusplus
}
#endif
#endif /* QPANDA_B200_H */
