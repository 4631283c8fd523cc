// Conversion of the C ABI's op descriptors (qs_op) into planner ops, shared by the state's
// tile API and the allocation-free entry point.
#pragma once
#include <vector>

#include "../../include/qsim_b200.h"
#include "plan.h"

namespace qsb {

// Validates an op list as parse_tile_ops does (bindings.cpp:182-220), with messages
// "<who>: invalid q0", "<who>: q0 == q1", "<who>: unknown op kind: k", ... (std::invalid_argument),
// and reads the matrices (dtype precision).  pos2bit (optional) maps layout positions to
// physical bits.  Device matrices are read back when allow_device, rejected otherwise.
std::vector<QOp> convert_abi_ops(const qs_op* ops, int nops, int n, int dtype, const char* who, const int* pos2bit,
                                 bool allow_device);

}  // namespace qsb
