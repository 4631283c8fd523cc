// Internal header of the B200 statevector tile executor (libqsim_b200.so).
//
// Vocabulary
//   state      2^n complex amplitudes (complex64 or complex128) in HBM.
//   physical bit  bit position p of the amplitude index in memory.
//   virtual position  bit position as seen by the caller after permute() calls; the
//              executor maps it to a physical bit (pos2bit) and moves data only when the
//              state is observed (copy-out, device pointer export).
//   sweep / pass  one read + write of the whole state.  A pass stages groups of 2^m
//              amplitudes (one value of the n-m "group bits", all values of the m "local
//              bits" S) in shared memory and applies every gate of the pass to them.
//   phase      inside a pass, a choice of r local bits held in registers by each thread
//              (2^r amplitudes per thread); gates whose data bits are register bits run
//              entirely in registers.  Diagonal gates and controls need no register bit.
#pragma once
#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

namespace qsb {

constexpr int kMaxQubits = 40;
constexpr int kMaxM = 16;          // local bits per pass (group of 2^m amplitudes)
constexpr int kMaxR = 5;           // register bits per thread
constexpr int kFixed = 64;         // operand >= kFixed: physical bit (operand - kFixed), value fixed per thread

enum GateKind : uint8_t {
  GK_NONE = 0,
  // 1-qubit: operand a
  GK_1Q_DENSE = 1,   // coef: u00 u01 u10 u11
  GK_1Q_REAL = 2,    // all entries real; coef as dense (imag parts zero)
  GK_1Q_REIM = 3,    // u00,u11 real, u01,u10 imaginary (RX-like)
  GK_1Q_DIAG = 4,    // coef: d0 d1   (operand may be fixed)
  GK_1Q_X = 5,       // pure bit flip, no coef
  // 2-qubit: operands a = q0, b = q1 (matrix index b_q0 + 2 b_q1)
  GK_2Q_DENSE = 16,  // coef: 16 entries row-major
  GK_2Q_DIAG = 17,   // coef: 4 diagonal entries (operands may be fixed)
  GK_2Q_CX = 18,     // a = control (may be fixed), b = target; flip target when control = 1
  GK_2Q_CU = 19,     // a = control (may be fixed), b = target; coef: 2x2 applied when control = 1
  GK_2Q_SWAP = 20,   // exchange the two bits
};

struct GateInstr {
  uint8_t kind;
  uint8_t a;         // register bit index (< r) or kFixed + physical bit
  uint8_t b;
  uint8_t pad;
  int32_t coef;      // offset in complex entries into the coefficient table
};

struct PhaseDesc {
  int8_t rbit[kMaxR];    // local bit held by register bit j
  int8_t tbit[kMaxM];    // local bit of thread-index bit j (m - r of them)
  int8_t pad[3];
  int32_t gate0;         // first gate instruction of the phase
  int32_t ngate;
};

struct PassDesc {
  int32_t m;             // local bits
  int32_t r;             // register bits
  int32_t phase0;        // first phase of the pass
  int32_t nphase;
  int32_t ngbits;        // group bits = n - m
  int32_t store_perm;    // 1: output local bit j takes input local bit store_src[j]
  int8_t sbit[kMaxM];    // physical bit of local bit j (ascending)
  int8_t gbit[kMaxQubits];  // physical bit of group-index bit j (ascending)
  int8_t store_src[kMaxM];
};

// Device program: arrays of passes, phases, gates and coefficients in one buffer.
struct ProgramHeader {
  int32_t npass, nphase, ngate, ncoef;
  int32_t off_pass, off_phase, off_gate, off_coef;   // byte offsets from program start
  int32_t n;             // qubits
  int32_t dtype;         // 0 c64, 1 c128
  int32_t max_threads;   // block size used for every pass
  int32_t pad;
};

// Error word layout written by kernels (host reads after a launch).
enum DeviceError : uint32_t {
  DERR_NONE = 0,
  DERR_BARRIER_TIMEOUT = 1,
  DERR_BAD_PROGRAM = 2,
};

}  // namespace qsb
