// Host-side planning for the pass kernel: classification of gates, pass (sweep)
// selection, register-phase selection, in-place permutation decomposition and the
// encoding of a device program.
#pragma once
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

#include "qsim.h"

namespace qsb {

using cplx = std::complex<double>;

// A gate queued for execution, at physical bits.
struct QOp {
  int arity = 1;          // 1 or 2
  int q0 = 0, q1 = -1;    // physical bits; matrix index b_q0 + 2 b_q1
  cplx U[16];             // row-major 2x2 (first 4) or 4x4
};

// A gate after classification (see GateKind).
struct COp {
  GateKind kind = GK_NONE;
  int a = -1, b = -1;     // physical bits in role order
  int ncoef = 0;
  cplx coef[16];
  uint64_t touch = 0;     // physical bits read or written
  uint64_t need = 0;      // physical bits that must be staged (pass) / held in registers (phase)
};

COp classify(const QOp& op);

// Rewrites the gates of one planned pass as s * V (one entry of V exactly 1, as many
// entries as possible in {0, +-1, +-i}) and multiplies the product of the scalars into one
// gate of the pass.  The classification (need/touch bits) of every gate is unchanged.
// diag_absorbs = false: diagonal gates never absorb the product (they keep unit-modulus
// entries); a pass of diagonal gates only then drops its product, a unit-modulus phase.
void extract_pass_scalars(std::vector<QOp>& ops, const std::vector<int>& pass_ops, bool diag_absorbs = true);

struct PlanConfig {
  int m = 13;             // local bits per pass
  int r = 5;              // register bits per thread
  int k = 3;              // lowest physical bits always staged (contiguous runs of 2^k amplitudes)
  int hill_iters = 16;    // hill-climbing rounds when choosing the staged / register sets (and
                          // restarts of the staged-set search)
  bool pair_bit = false;  // physical bit 0 is a register bit of every phase (packed kernels)
  int lookahead = 2;      // staged-set choice: greedy passes looked ahead over the 4 best candidates
  int phase_lookahead = 16;  // register sets: every set scored, and among this many best the one after
                            // which greedy phases finish the pass soonest (0: hill climbing only)
};

struct PlannedPhase {
  std::vector<int> rbits;  // local bits held in registers
  std::vector<int> ops;    // indices into the op list, in execution order
};

struct PlannedPass {
  std::vector<int> sbits;        // staged physical bits (ascending), size m
  std::vector<int> ops;          // op indices in execution order
  std::vector<PlannedPhase> phases;
  std::vector<int> store_src;    // optional: output local bit j <- input local bit store_src[j]
};

// Split ops (in order) into passes and phases.
std::vector<PlannedPass> plan_passes(const std::vector<COp>& ops, int n, const PlanConfig& cfg);

// Order of a phase's thread bits (local bits not in registers): the lowest five (the lane
// bits) cover as many shared-memory bank classes of the dtype's swizzle as possible, taking
// bits of `prefer`, then bits outside `avoid` (masks of local bits) first.
std::vector<int> order_thread_bits(const std::vector<int>& tb, int dtype, uint64_t avoid = 0, uint64_t prefer = 0);

// In-place bit permutation as a sequence of gate-free passes.  perm[b] = destination
// physical bit of the data now at physical bit b.
std::vector<PlannedPass> plan_permutation(const std::vector<int>& perm, int n, const PlanConfig& cfg);

// Encoded program (host copy) and its structure hash (coefficient values excluded).
struct Program {
  std::vector<uint8_t> bytes;
  uint64_t structure_hash = 0;
  int npass = 0;
  int threads = 0;        // block size (max over passes of 2^(m - r))
  size_t max_smem = 0;    // bytes of shared memory per block
  bool has_gates = false;  // at least one gate instruction
  // Gradient programs only (the reverse sweep of an adjoint gradient over the stacked state
  // psi (+) lam, physical bit 0 selecting lam; empty otherwise), per gate instruction: the
  // generator of a parameterised rotation (0 none, 1 X, 2 Y, 3 Z) and the index of its
  // gradient term Im <lam|G|psi> (-1 none).  Terms are numbered in instruction order.
  std::vector<int8_t> grad_gen;
  std::vector<int32_t> grad_term;
  int nterm = 0;
};

// r_req: register bits per thread (the generic kernel's fixed value when <= 0:
// 5 for complex64, 4 for complex128; specialised kernels may use others).
Program encode_program(const std::vector<PlannedPass>& passes, const std::vector<COp>& ops,
                       int n, int dtype, int r_req = 0);

// The per-pass scalar extraction of ops (which keeps every gate's planned shape, so the plan
// made from the original gates stays valid), then the encoded program of the passes.
Program build_program(std::vector<QOp>& ops, const std::vector<PlannedPass>& passes, int n, int dtype, int r);

// Reference interpretation of a program on host memory (used by CPU tests of the planner).
void emulate_program(const uint8_t* prog, void* state, int n, int dtype);

// ---- adjoint gradient over the stacked state -------------------------------------------
// A gate of the forward circuit (qubit indices = bit positions of the n-qubit state) with
// its parameter: gen 0 none, 1 X, 2 Y, 3 Z (R(theta) = exp(-i theta G / 2)), slot = index of
// dE/dtheta.
struct GradOp {
  QOp op;
  int gen = 0, slot = -1;
};

// Reverse-sweep program over Phi = psi (+) lam on n + 1 qubits (physical bit 0 selects lam,
// circuit qubit q is physical bit q + 1): the circuit's gates as U^dagger in reverse order;
// before each parameterised gate its term Im <lam|G|psi> is accumulated, term t weighing
// term_w[t] (the squared magnitude of the scalars extracted before it) into gradient slot
// term_slot[t].
struct GradProgram {
  Program prog;
  std::vector<int> term_slot;
  std::vector<double> term_w;
};

// Planned passes of the reverse sweep (gate classes and bits only: reusable for any
// parameter values of the same structure) and the structure's signature.
std::vector<PlannedPass> plan_grad_passes(const std::vector<GradOp>& fwd, int n, const PlanConfig& cfg,
                                          uint64_t* signature);
uint64_t grad_signature(const std::vector<GradOp>& fwd, int n, const PlanConfig& cfg);
// Whether a plan made for other matrix values of the same circuit holds these values' gates
// (every gate's register needs met in its phase).
bool grad_plan_fits(const std::vector<GradOp>& fwd, const std::vector<PlannedPass>& passes);
GradProgram build_grad_program(const std::vector<GradOp>& fwd, int n, const std::vector<PlannedPass>& passes,
                               int r);

// Host interpretation of a gradient program on Phi (complex64, 2^(n+1) amplitudes, the
// program's own coefficients): terms[t] (FP64, unweighted) as the specialised kernels
// accumulate them.
void emulate_grad_program(const GradProgram& g, void* phi, double* terms);

}  // namespace qsb
