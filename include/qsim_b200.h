/*
 * libqsim_b200 -- C ABI of the B200 statevector tile executor.
 *
 * Drop-in boundary for the native module of qgpusim's custom backend
 * (pybind11 module ``qgpusim_cuda``, qgpusim/backends/custom/qgpusim_cuda/src/bindings.cpp:1004-1092).
 * Every function returns 0 on success or a negative status; the message of the last
 * failure on the calling thread is returned by qs_last_error().  Message texts follow the
 * reference's std::runtime_error messages where the reference has one.
 *
 * Complex numbers are interleaved (re, im) in the state's precision unless stated:
 * QS_C64 = complex64 (StatevectorF32), QS_C128 = complex128 (Statevector).
 * Gate matrices are row-major; for 2-qubit gates the index is b_q0 + 2*b_q1
 * (kernels.cu:54-55,108-114).  Qubit arguments of tile ops are bit positions in the
 * state's current layout (after permute()).
 */
#ifndef QSIM_B200_H
#define QSIM_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define QS_API __attribute__((visibility("default")))
#else
#define QS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define QS_C64 0
#define QS_C128 1

#define QS_MODE_COOPERATIVE 0 /* apply_tile_cooperative */
#define QS_MODE_GRAPHED 1     /* apply_tile_graphed     */
#define QS_MODE_SEQUENTIAL 2  /* apply_tile_dev         */

#define QS_OP_1Q 1
#define QS_OP_2Q 2

#define QS_ERR_INVALID -1 /* bad argument */
#define QS_ERR_CUDA -2    /* CUDA runtime error */
#define QS_ERR_DEVICE -3  /* a kernel reported an error word (bounded wait expired) */

typedef struct qs_state qs_state;

/* One tile op: ('1q', q0, U) or ('2q', q0, q1, U) of bindings.cpp:182-220.
 * U points to 4 or 16 complex entries in the state's precision; u_on_device = 1 when U
 * is a device pointer.  The executor copies U before returning (no borrowed pointer). */
typedef struct {
  int kind; /* QS_OP_1Q or QS_OP_2Q */
  int q0;
  int q1;
  int u_on_device;
  const void* U;
} qs_op;

typedef struct {
  int m;          /* local (staged) bits per sweep; c64 <= 13, c128 <= 12 */
  int k;          /* lowest physical bits always staged (>= 1) */
  int hill_iters; /* planner search effort */
  int grid_mult;  /* resident blocks per SM used by the pass kernel (0 = occupancy) */
  int jit;        /* plan-time specialised kernels in graphed mode: 0 auto (complex64,
                     >= 20 qubits), 1 always (complex64), -1 never */
  int jit_lr;     /* register bits per thread of the specialised kernels (3..6; 6: 64 amplitudes
                     per thread, 2^(m-6) threads per group) */
  int jit_blocks; /* specialised kernels: 1 double-buffered block per SM, 2 single-buffered
                     blocks per SM, 3 one block of two teams over three buffers */
  int jit_packed; /* specialised kernels: FP32x2 arithmetic on two amplitudes (1) or scalar (0) */
  unsigned long long wait_limit_ns; /* limit of every bounded device wait of this state's kernels
                                       (grid barriers of cooperative launches, tensor-core
                                       completion waits); 0 = the default, 20 s.  A wait that
                                       expires sets an error word; the call that observes it
                                       returns QS_ERR_DEVICE and the state stays usable. */
  int jit_async;  /* 1: while the specialised kernels of a new circuit structure compile (on a
                     background thread), the generic pass kernel runs the same plan (needs
                     jit_lr = 5 and jit_packed = 0); later flushes use the specialised kernels
                     once they are ready.  0 (default): the first flush waits for the compile. */
  int pad;
} qs_config;

typedef struct {
  unsigned long long gates;          /* ops accepted */
  unsigned long long sweeps;         /* full-state passes run by the pass kernel */
  unsigned long long perm_sweeps;    /* of which: in-place permutation passes */
  unsigned long long gate_sweeps;    /* per-gate kernel sweeps (sequential mode / per-gate API) */
  unsigned long long launches;       /* kernel launches (graph launches count once) */
  unsigned long long graph_replays;  /* cached graph launches */
  unsigned long long graph_builds;   /* graph captures */
  unsigned long long flushes;        /* planned executions */
  unsigned long long permutes;       /* permute() calls */
  unsigned long long plans;          /* pass plans computed (cache misses) */
  unsigned long long jit_compile_ms; /* host time spent compiling specialised kernels */
  unsigned long long jit_modules;    /* kernel modules prepared for specialised programs */
  unsigned long long jit_disk_hits;  /* of which read from the on-disk kernel cache */
  unsigned long long jit_pending_flushes; /* flushes run by the generic kernel while compiling */
} qs_stats;

/* Library */
QS_API const char* qs_last_error(void);
/* Fault injection for tests of the error paths (no counterpart in the reference, whose only
 * failure handling is catching out-of-memory exceptions in its benchmark driver,
 * benches/run_benchmarks.py:192-213): the k-th next device or pinned-host allocation made by
 * the library fails with a CUDA out-of-memory error and allocates nothing (k <= 0: off). */
QS_API int qs_debug_fail_alloc(int k);
/* Waits until every background compile of specialised kernels (qs_config.jit_async) has ended. */
QS_API int qs_jit_wait(void);
QS_API int qs_version(void);
QS_API int qs_device_count(int* out);

/* Statevector(num_qubits) / StatevectorF32(num_qubits): bindings.cpp:92-110, 645-658 */
QS_API int qs_create(int num_qubits, int dtype, qs_state** out);
/* ~Statevector: bindings.cpp:112-122 */
QS_API int qs_destroy(qs_state* s);
/* num_qubits / dim properties: bindings.cpp:1023-1024 */
QS_API int qs_num_qubits(const qs_state* s, int* out);
QS_API int qs_dim(const qs_state* s, unsigned long long* out);
QS_API int qs_dtype(const qs_state* s, int* out);

/* reset(): bindings.cpp:577-582 */
QS_API int qs_reset(qs_state* s);
/* synchronize(): bindings.cpp:585-587 (executes queued ops, waits, checks error words) */
QS_API int qs_synchronize(qs_state* s);
/* to_numpy(): bindings.cpp:547-560 -- state in the current layout, nbytes = dim * elem */
QS_API int qs_copy_to_host(qs_state* s, void* dst, unsigned long long nbytes);
/* from_numpy(psi): bindings.cpp:563-574 (also offered for complex64) */
QS_API int qs_copy_from_host(qs_state* s, const void* src, unsigned long long nbytes);

/* permute(layout_old, layout_new): bindings.cpp:434-483, scatter semantics of
 * kernels.cu:165-185.  Recorded as a relabelling; data moves (in place, bit-exact) when
 * the state is next observed. */
QS_API int qs_permute(qs_state* s, const int* layout_old, const int* layout_new, int n);

/* apply_tile_cooperative / apply_tile_graphed / apply_tile_dev: bindings.cpp:223-373 */
QS_API int qs_apply_tile(qs_state* s, const qs_op* ops, int nops, int mode);
/* apply_1q / apply_2q / apply_1q_dev / apply_2q_dev: bindings.cpp:499-544, 589-608 */
QS_API int qs_apply_1q(qs_state* s, int target_qubit, const void* U, int u_on_device);
QS_API int qs_apply_2q(qs_state* s, int q0, int q1, const void* U, int u_on_device);
/* apply_diagonal_1q(target, phase0, phase1): bindings.cpp:611-619; phases complex128 */
QS_API int qs_apply_diagonal_1q(qs_state* s, int target_qubit, const double* phase0, const double* phase1);

/* Run queued ops now (asynchronously on the state's stream). */
QS_API int qs_flush(qs_state* s);
/* Run queued ops and move the data to the current layout (asynchronously). */
QS_API int qs_materialize(qs_state* s);
/* Dense 64x64 unitary on layout positions 0..5 (no counterpart in the reference executor;
 * the k=6 fused-gate form of the north-star design): U is a host complex128 matrix, row-major,
 * row/column index sum_j b_j 2^j over positions j = 0..5.  Complex64 states of >= 13 qubits.
 * One sweep on the tensor cores (tcgen05 MMAs, operands split into BF16 high and low parts,
 * FP32 accumulation in tensor memory); queued gates run first and the layout is materialised. */
QS_API int qs_apply_dense6(qs_state* s, const double* U);
/* Dense 2^k x 2^k unitary (k = 1..6) on k arbitrary layout positions qubits[0..k-1] of a
 * complex64 state of >= 13 qubits, in one tensor-core sweep (no counterpart in the reference
 * executor: the fused k-qubit blocks of the north-star design).  U: host complex128, row-major,
 * row/column index sum_j b_{qubits[j]} 2^j.  Applied as the 64x64 unitary U (x) I on the block's
 * bits and the lowest other physical bits; a tile of the kernel is 2^13 amplitudes over those six
 * bits and the seven lowest other bits (coalesced copies for any positions).  Queued gates run
 * first; no data is moved to another layout. */
QS_API int qs_apply_dense(qs_state* s, int k, const int* qubits, const double* U);
/* Measurement sampling (the runner's "sampling" task, runner.py:25-27, 74; the reference's custom
 * backend has none): `shots` basis indices (layout order, bit p = position p) drawn from |psi|^2,
 * returned ascending in out (host, shots entries).  Queued gates run first.  seed selects the
 * counter-based random stream (same seed, same state -> same indices). */
QS_API int qs_sample(qs_state* s, unsigned long long shots, unsigned long long seed, unsigned long long* out);
/* The tensor-core operand qs_apply_dense6 builds from U (host only; 65536 bytes into out):
 * the 128x128 real form W (row 2r+q, column 2s+p: q,p = 0 real / 1 imaginary part) split into
 * BF16 high and low parts, in the canonical K-major layout (8-row x 16-byte core matrices,
 * K-chunks 128 B apart, 8-row groups 2048 B apart), high part first. */
QS_API int qs_dense6_weights(const double* U, void* out);
/* Device address of the amplitudes in the current layout (executes queued ops and
 * pending data movement, then synchronises).  Valid until the next call on s. */
QS_API int qs_device_ptr(qs_state* s, void** out);
/* Stream used by s (cudaStream_t); NULL selects the state's own non-blocking stream. */
QS_API int qs_set_stream(qs_state* s, void* stream);
QS_API int qs_get_stream(qs_state* s, void** out);
QS_API int qs_set_config(qs_state* s, const qs_config* cfg);
QS_API int qs_get_config(qs_state* s, qs_config* cfg);
QS_API int qs_get_stats(qs_state* s, qs_stats* out);
QS_API int qs_reset_stats(qs_state* s);
/* Current layout relabelling: out[p] = physical bit holding layout position p. */
QS_API int qs_get_pos2bit(qs_state* s, int* out, int n);

/* Reductions in FP64: sum |psi|^2 and <a|b> (states of equal size; a complex64 and a
 * complex128 state may be paired, e.g. to measure a single-precision run against a
 * double-precision one). */
QS_API int qs_norm_squared(qs_state* s, double* out);
QS_API int qs_inner_product(qs_state* a, qs_state* b, double* re, double* im);

/* Adjoint differentiation (no counterpart in the reference executor).
 * qs_expect_zz_x: lam <- H psi and energy = <psi|H|psi> (FP64) for
 * H = sum_i a_i Z_i Z_{(i+1) mod n} + b_i X_i; psi and lam are states of equal size/dtype. */
QS_API int qs_expect_zz_x(qs_state* psi, qs_state* lam, const double* a, const double* b, double* energy);

/* One gate of a circuit for the reverse sweep.  U: host complex128 matrix (4 or 16
 * entries, row-major, index b_q0 + 2*b_q1) of the forward gate; gen: generator of a
 * parameterised rotation R(theta) = exp(-i theta G / 2): 0 none, 1 X, 2 Y, 3 Z. */
typedef struct {
  int kind; /* QS_OP_1Q or QS_OP_2Q */
  int q0;
  int q1;
  int gen;
  int grad_index; /* slot of dE/dtheta in grads (ignored when gen == 0) */
  int pad;
  const double* U;
} qs_adj_op;

/* Reverse sweep: psi holds U|0>, lam holds H psi (qs_expect_zz_x).  For k = nops-1 .. 0:
 * grads[grad_index] += Im <lam|G|psi> (FP64), then psi <- U_k^dagger psi, lam <- U_k^dagger lam.
 * Ops use layout positions of the states (identity layout after qs_expect_zz_x).
 * grads (host, ngrads doubles) is overwritten. */
QS_API int qs_adjoint_sweep(qs_state* psi, qs_state* lam, const qs_adj_op* ops, int nops, double* grads,
                            int ngrads);

/* Adjoint gradient with the plan-time specialised kernels (complex64 states, FP64 energy and
 * gradient; no counterpart in the reference).  psi = U|0...0> runs as one graphed tile; one
 * kernel then writes the stacked state Phi = psi (+) H psi (n + 1 qubits, Phi[2x] = psi[x],
 * Phi[2x + 1] = (H psi)[x]) and the energy; the reverse sweep is ONE planned program over Phi
 * (both states uncomputed by the same U_k^dagger), whose kernels add Im <lam|G|psi> before
 * each rotation into per-gate FP64 terms.  Plans and kernels follow the circuit's structure
 * (gate kinds, qubits, generators, slots): new parameter values reuse them.  10 <= n <= 33.
 * cfg (optional): m, k and hill_iters of the plans and jit_lr (5 or 6 register bits per
 * thread; the reverse program holds the lam bit in one of them); other fields ignored. */
typedef struct qs_grad qs_grad;
QS_API int qs_grad_create(int num_qubits, const qs_adj_op* ops, int nops, int nparams, const qs_config* cfg,
                          qs_grad** out);
/* Same structure as at creation, any matrices: energy and grads (nparams doubles, overwritten;
 * NULL: the energy only, no reverse sweep).  QS_ERR_INVALID when the structure differs. */
QS_API int qs_grad_run(qs_grad* g, const qs_adj_op* ops, int nops, const double* a, const double* b, double* energy,
                       double* grads);
/* Sweeps of the last forward run and of the reverse program, register phases of the
 * reverse program, gradient terms (one per rotation). */
QS_API int qs_grad_info(const qs_grad* g, int* fwd_sweeps, int* rev_sweeps, int* rev_phases, int* terms);
/* Execution counters of the handle (launches, sweeps, graph builds, kernel compiles). */
QS_API int qs_grad_stats(qs_grad* g, qs_stats* out);
QS_API int qs_grad_destroy(qs_grad* g);
/* Compiles the reverse program's kernels on the host only (NVRTC; tests): sweeps and the
 * compiler's resource log (registers, spills) in logbuf. */
QS_API int qs_grad_jit_check(int num_qubits, const qs_adj_op* ops, int nops, int nparams, const qs_config* cfg,
                             int* sweeps, char* logbuf, int logcap);
/* Host interpretation of the reverse program (CPU tests of its planning, scalar weights and
 * term placement): psi = U|0> and lam = H psi given (complex64, 2^n each), grads out.
 * 10 <= n <= 22. */
QS_API int qs_grad_emulate(int num_qubits, const qs_adj_op* ops, int nops, int nparams, const qs_config* cfg,
                           const void* psi, const void* lam, double* grads);

/* Module-level apply_1q_gate / apply_2q_gate (bindings.cpp:931-1001): gate on a raw
 * device array psi of 2^num_qubits amplitudes; U is a host matrix; stream may be NULL. */
QS_API int qs_apply_1q_gate(void* psi, int dtype, const void* U, int target_qubit, int num_qubits, void* stream);
QS_API int qs_apply_2q_gate(void* psi, int dtype, const void* U, int q0, int q1, int num_qubits, void* stream);
/* Reference permute kernel semantics on raw device arrays (out-of-place scatter,
 * kernels.cu:165-185): out[sum_p bit_p(i) << map_old_to_new[p]] = in[i]. */
QS_API int qs_permute_scatter(const void* in, void* out, int dtype, int num_qubits, const int* map_old_to_new,
                       void* stream);

/* Allocation-free gate application (no counterpart in the reference).
 * For callers that cannot allocate device memory -- code that runs inside a framework
 * whose allocator already holds the device memory it may use, or that must not trigger the
 * device-wide synchronisation cudaMalloc/cudaFree imply -- this applies ops (host
 * matrices, physical bit positions) to a caller-owned device state psi of 2^num_qubits
 * amplitudes with the same sweep kernel as qs_apply_tile's cooperative mode, and allocates
 * nothing: its program and grid-barrier words live in one fixed 1 MiB device array that
 * every GPU loading the library holds until exit.  Calls whose encoded program exceeds that
 * array (about 20,000 gates) are rejected with an error asking to split them.
 * psi must be 16-byte aligned device memory of the current device (or managed memory):
 * the kernel moves amplitudes in 16-byte units; other pointers are rejected with
 * QS_ERR_INVALID before anything is launched.  Errors name this entry point.
 * The first call on a device looks up the array's device address (with that device
 * current) and keeps it for the life of the process; make that first call before any stream
 * capture, and do not call this entry point again after cudaDeviceReset on that device.
 * All calls share the array: it is reset at the start of each call, and calls that overlap
 * on the GPU (other streams, other host threads) race -- serialise them.  The call returns
 * after the work on `stream` (NULL: the legacy default stream) has finished. */
QS_API int qs_apply_ops_noalloc(void* psi, int dtype, int num_qubits, const qs_op* ops, int nops, void* stream);

/* LQR flat tiling of a depth-sorted gate list (host only; replaces the Python loops of
 * LazyQubitReordering.flat_tiling / tile_construction / greedy_qubit_mapping and
 * extract_tiles, qgpusim/transpiler/passes.py:89-272).  targets[i] = bit mask of gate i's
 * qubits (num_qubits <= 64), in the order of passes.py:359-368's stable depth sort.  Out:
 * order[k] = input index of the k-th scheduled gate, tile_of[k] = its tile, tile_masks[t] =
 * the qubit set of tile t (room for ngates entries), *ntiles. */
QS_API int qs_lqr_flat_tiling(int num_qubits, int nL, const unsigned long long* targets, int ngates, int* order,
                              int* tile_of, unsigned long long* tile_masks, int* ntiles);

/* Gate fusion of a tile's op list on the host (replaces the Python loop of fuse_tile_ops,
 * qgpusim/backends/custom/backend.py:88-200; same result: consecutive gates on the same qubit /
 * the same ordered qubit pair multiplied, U_new = U @ U_prev).  in: nin ops with host matrices
 * of dtype; out: room for nin ops, whose U point into mats (room for nin * 16 entries of
 * dtype); *nout = fused count.  Device matrices are rejected (fuse those on the caller side). */
QS_API int qs_fuse_ops(int dtype, const qs_op* in, int nin, qs_op* out, void* mats, int* nout);

/* Gate ids of qs_prepare_ops / qs_gate_matrix: the named gates of the reference's circuits
 * (qiskit names), QS_GATE_MATRIX = a caller-supplied matrix. */
#define QS_GATE_MATRIX 0
#define QS_GATE_ID 1
#define QS_GATE_H 2
#define QS_GATE_X 3
#define QS_GATE_Y 4
#define QS_GATE_Z 5
#define QS_GATE_S 6
#define QS_GATE_SDG 7
#define QS_GATE_T 8
#define QS_GATE_TDG 9
#define QS_GATE_SX 10
#define QS_GATE_RX 11
#define QS_GATE_RY 12
#define QS_GATE_RZ 13
#define QS_GATE_P 14
#define QS_GATE_U 15
#define QS_GATE_CX 32
#define QS_GATE_CY 33
#define QS_GATE_CZ 34
#define QS_GATE_CP 35
#define QS_GATE_CRZ 36
#define QS_GATE_SWAP 37
#define QS_GATE_RZZ 38

/* Matrix of a named gate (host only; replaces op.to_matrix() behind the reference's gate cache,
 * qgpusim/backends/custom/backend.py:37-76): params[0..2] its angles; out receives 4 or 16
 * complex128 entries (row-major, index b_q0 + 2*b_q1), *arity 1 or 2. */
QS_API int qs_gate_matrix(int gate_id, const double* params, double* out, int* arity);
/* A tile's op list prepared in one call (host only; replaces the per-gate loop of the
 * reference's native branch, backend.py:432-451, its matrix cache and fuse_tile_ops,
 * backend.py:16-200): gate i is gate_id[i] with params[3i..3i+2] on layout positions q0[i]
 * (and q1[i] >= 0 for two-qubit gates; -1 otherwise); QS_GATE_MATRIX gates read 4 or 16
 * complex128 entries at custom + 32 i (doubles).  fuse != 0 fuses as qs_fuse_ops does.  out (room
 * for ngates ops) receives the ops with U pointing into mats (room for 16 ngates entries of
 * dtype); *nout = their count. */
QS_API int qs_prepare_ops(int dtype, int ngates, const int* gate_id, const double* params, const int* q0,
                          const int* q1, const double* custom, int fuse, qs_op* out, void* mats, int* nout);

/* Planner inspection (host only, no GPU needed): plan the ops of a tile list for an
 * n-qubit state and report sweeps / phases.  ops use physical bits. */
QS_API int qs_plan_info(int num_qubits, int dtype, const qs_op* ops, int nops, const qs_config* cfg,
                 int* sweeps, int* phases);
/* Host emulation of the planned program (tests of the planner, no GPU needed):
 * applies ops to the host state psi (2^n entries, dtype precision). */
QS_API int qs_plan_emulate(int num_qubits, int dtype, const qs_op* ops, int nops, const qs_config* cfg, void* psi);
/* Generate and compile (NVRTC, sm_100a, host only) the specialised kernels of the planned
 * complex64 program for ops; returns QS_ERR_INVALID with the compiler log on failure.
 * log (optional, logcap bytes) receives the compiler log (ptxas resource usage). */
QS_API int qs_jit_check(int num_qubits, const qs_op* ops, int nops, const qs_config* cfg, int* sweeps, char* log,
                        int logcap);
/* Host emulation of the in-place permutation program: perm[b] = destination bit. */
QS_API int qs_perm_emulate(int num_qubits, int dtype, const int* perm, const qs_config* cfg, void* psi,
                    int* sweeps);

/* ---- Batched variational workload (no counterpart in the reference executor) ----------
 * Energy E_i = <psi_i|H_i|psi_i> and the full adjoint gradient dE_i/dtheta of many
 * independent circuits of uneven qubit count, in ONE persistent cooperative launch per
 * batch: psi_i = U_i |0...0> (complex64), H_i = sum_j a_j Z_j Z_{(j+1) mod n} + b_j X_j,
 * FP64 energies and gradients.  Instances up to small_max qubits run entirely in shared
 * memory; larger ones stream their states from an HBM arena in planned passes. */
typedef struct qs_batch qs_batch;
typedef struct {
  int num_qubits;       /* 2 .. 26 */
  const qs_adj_op* ops; /* the circuit (qubit indices = bit positions); gen marks rotations */
  int nops;
  int nparams;          /* gradient slots: grad_index < nparams */
  const double* a;      /* observable coefficients, num_qubits each */
  const double* b;
} qs_batch_instance;
typedef struct {
  int m;             /* staged bits per group of the arena instances (9 .. 13) */
  int small_max;     /* instances with num_qubits <= small_max run in shared memory (0 .. 13) */
  int chunk;         /* groups per work item (>= 1) */
  int threads;       /* threads per block: 256 or 512 */
  int blocks_per_sm; /* cap on resident blocks per SM (0: as many as fit) */
  int pad;
  unsigned long long wait_limit_ns; /* limit of the kernel's dependency waits (0: 10 s) */
} qs_batch_config;
/* Plan and encode the batch, allocate its device program, arena and outputs (cfg NULL:
 * m 13, small_max 13, chunk 4, 256 threads). */
QS_API int qs_batch_create(const qs_batch_instance* insts, int ninst, const qs_batch_config* cfg, qs_batch** out);
/* New gate matrices / observables for the same instance shapes (re-encodes the program). */
QS_API int qs_batch_set_params(qs_batch* b, const qs_batch_instance* insts, int ninst);
/* Launch the batch on stream (NULL: legacy default stream).  ms (optional): device time of
 * the launch, waiting for it. */
QS_API int qs_batch_run(qs_batch* b, void* stream, float* ms);
/* Wait for the device, then copy energies (ninst) and gradients (concatenated in instance
 * order, nparams each); QS_ERR_DEVICE when a dependency wait of the kernel timed out. */
QS_API int qs_batch_results(qs_batch* b, double* energies, double* grads);
QS_API int qs_batch_info(const qs_batch* b, int* nitems, int* nparams_total, long long* arena_bytes, int* grid);
QS_API int qs_batch_destroy(qs_batch* b);
/* Host-side plan of a batch (no device work): per instance five ints in stats[5 * i ..]:
 * passes, passes run in register phases, register phases, gates, work items. */
QS_API int qs_batch_describe(const qs_batch_instance* insts, int ninst, const qs_batch_config* cfg, int* stats);
/* Host emulation of the same device program (items in list order, FP64 states): tests of
 * the batch planner and encoder without a GPU. */
QS_API int qs_batch_emulate(const qs_batch_instance* insts, int ninst, const qs_batch_config* cfg, double* energies,
                            double* grads);

#ifdef __cplusplus
}
#endif

#endif /* QSIM_B200_H */
