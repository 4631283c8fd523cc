// Batched variational workload: energy and full adjoint gradient of many independent
// circuits of uneven qubit count in one persistent launch.
//
// Device program (one buffer): header, instances, passes, gates, work items, observable
// coefficients.  Every instance is a circuit on n qubits applied to |0...0>, an
// observable H = sum_i a_i Z_i Z_{(i+1) mod n} + b_i X_i, and parameter slots.
//
//  * n <= small_max: one work item (SMALL) holds psi and lam = H psi in shared memory for
//    the whole forward sweep, the energy and the reverse sweep; nothing touches HBM but the
//    results.
//  * larger n: the states live in an arena in HBM; the gates are planned into passes (2^m
//    amplitudes staged per group, as in the tile executor), and the work items are
//    FWD (groups of one forward pass), HAM (lam = H psi and the energy, by amplitude
//    chunks) and BWD (groups of one reverse pass over psi and lam, accumulating
//    Im <lam|G|psi> per parameterised gate).
//  * Items are taken from a global counter in list order; an item waits (bounded) until
//    the items of its instance's earlier stages are complete.  The list is ordered by stage
//    across instances, so an item's prerequisites were all taken before it, by blocks that
//    are resident (cooperative launch): the waits end.
#pragma once
#include "qsim.h"

namespace qsb {

constexpr int kBatchMaxQubits = 26;  // qubits per instance
constexpr int kBatchMaxLocal = 13;   // staged bits per group (complex64: 64 KiB per state)

enum BatchGateKind : uint8_t {
  BG_1Q = 1,      // u: 2x2 row-major on q0 (staged)
  BG_DIAG1 = 2,   // u: 2 diagonal entries on q0 (staged or fixed by the group)
  BG_DIAG2 = 3,   // u: 4 diagonal entries, index b_q0 + 2 b_q1 (staged or fixed)
  BG_2Q = 4,      // u: 4x4 row-major, index b_q0 + 2 b_q1; both staged, or one fixed when the
                  // matrix is block-diagonal in that qubit (controlled gates)
};

enum BatchItemKind : int32_t { BI_SMALL = 0, BI_FWD = 1, BI_HAM = 2, BI_BWD = 3 };

struct BatchGate {
  uint8_t kind;
  uint8_t q0, q1;
  uint8_t gen;       // generator of R(theta) = exp(-i theta G / 2): 0 none, 1 X, 2 Y, 3 Z
  int32_t grad;      // parameter slot within the instance (gen != 0)
  float2 u[16];      // forward matrix (BG_1Q: 4 entries, BG_DIAG2: 4, BG_2Q: 16)
};

constexpr int kBatchRegBits = 4;     // register bits per thread in a phase (16 amplitudes per state)
constexpr int kBatchMaxPhases = 16;  // phases per pass run in registers (more: per-gate path)

// A register phase of a pass: each thread holds the 2^nr amplitudes whose local bits rbit vary
// (per state), the other local bits (tbit, lane bits first) select the thread's slot.  The
// phase's gates act on register bits or on bits fixed per slot or per group.
struct BatchPhase {
  int8_t rbit[kBatchRegBits];
  int8_t tbit[kBatchMaxLocal];
  int8_t nr;                // register bits (kBatchRegBits unless the pass is smaller)
  int8_t pad[3];
  int32_t gate0, ngate;     // gates (forward order), index into the gate array
};

struct BatchPass {
  int32_t m;         // staged bits
  int32_t gate0;     // first gate (forward order), index into the gate array
  int32_t ngate;
  int32_t phase0;    // register phases of the pass (their gates are gate0 .. gate0 + ngate)
  int32_t nphase;    // 0: the pass runs gate by gate in shared memory
  int8_t sbit[kBatchMaxLocal];      // qubit of local bit j (ascending)
  int8_t gbit[kBatchMaxQubits];     // qubit of group bit j (ascending), n - m of them
  int8_t pad[1];
};

struct BatchInst {
  int32_t n;
  int32_t m;                // staged bits of the instance's passes (n for SMALL)
  int32_t npass, pass0;     // passes (arena instances) or 1 pseudo-pass of all gates (SMALL)
  int32_t nparam;
  int32_t grad0;            // first gradient slot in the output
  int32_t coef0;            // a[n] then b[n] (doubles) in the coefficient table
  int32_t pad;
  int64_t psi, lam;         // arena offsets (complex64 amplitudes); -1 for SMALL
};

struct BatchItem {
  int32_t inst;
  int32_t kind;             // BatchItemKind
  int32_t pass;             // pass index within the instance (FWD/BWD)
  int32_t first, count;     // groups (FWD/BWD) or 2^m-amplitude chunks (HAM)
  int32_t need;             // items of this instance completed before this one may start
};

struct BatchHeader {
  int32_t ninst, npass, ngate, nitem, ncoef;
  int32_t off_inst, off_pass, off_gate, off_item, off_coef;  // byte offsets
  int32_t m;                // staged bits of arena instances
  int32_t small_max;        // instances with n <= small_max are SMALL
  int32_t mbuf;             // shared buffers hold 2^mbuf amplitudes each (psi, then lam)
  int32_t nphase;
  int32_t off_phase;
  int32_t pad;
};

}  // namespace qsb
