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
#ifdef __CUDACC_RTC__
// compiled by NVRTC (kernels generated at plan time): no standard headers
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
#else
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#endif

namespace qsb {

constexpr int kMaxQubits = 40;
constexpr int kMaxM = 16;          // local bits per pass (group of 2^m amplitudes)
constexpr int kMaxR = 6;           // register bits per thread (the generic kernels use 5 / 4)
constexpr int kFixed = 64;         // operand >= kFixed: physical bit (operand - kFixed), value fixed per thread
// dynamic shared-memory limit requested for the pass kernels (two 64 KiB group buffers);
// static tables take about 30 KiB more, within the 227 KiB per block
constexpr int kMaxDynamicSmem = 160 * 1024;
// limit of every bounded device-side wait (grid barriers, group copies of the two-team kernels)
constexpr unsigned long long kDeviceWaitLimitNs = 20ull * 1000ull * 1000ull * 1000ull;  // 20 s

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
  DERR_LOAD_TIMEOUT = 3,   // a team's wait for its group copies expired (pass kernel, two teams)
};

#ifndef __CUDACC_RTC__
inline const char* device_error_name(uint32_t w) {
  switch (w) {
    case DERR_BARRIER_TIMEOUT: return "a grid barrier wait expired";
    case DERR_BAD_PROGRAM: return "the device program was rejected by the kernel";
    case DERR_LOAD_TIMEOUT: return "a wait for group copies expired";
    default: return "a bounded device wait expired";
  }
}
#endif

// Bank-spreading swizzle of a local amplitude index inside the shared-memory group.
// complex64: XOR bits 1..3 with a fold of bits 4.. (bit 0 kept so aligned pairs stay together);
// complex128: XOR bits 0..2 with a fold of bits 3..  Both are XOR-linear, so
// swz(a | b) = swz(a) ^ swz(b) for disjoint a, b.
__host__ __device__ inline uint32_t swz64(uint32_t l) {
  uint32_t f = (l >> 4) ^ (l >> 7) ^ (l >> 10) ^ (l >> 13);
  return l ^ ((f & 7u) << 1);
}
__host__ __device__ inline uint32_t swz128(uint32_t l) {
  uint32_t f = (l >> 3) ^ (l >> 6) ^ (l >> 9) ^ (l >> 12);
  return l ^ (f & 7u);
}

}  // namespace qsb
