// Gate fusion of a tile's op list on the host: consecutive gates on the same qubit (1q) or on
// the same ordered qubit pair (2q) are multiplied, U_new = U @ U_prev, with the semantics of
// fuse_tile_ops (qgpusim/backends/custom/backend.py:88-200).  The reference scans the fused
// list for later ops that touch the qubits; here the index of the last fused entry touching
// each qubit is kept, which is the same test (a 1q gate fuses into that entry when it is a 1q
// gate on the same qubit; a 2q gate fuses into the later of its two qubits' entries when that
// entry is a 2q gate on the same ordered pair), so each op costs O(1) plus its matrix product.
#include <algorithm>
#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qsim_b200.h"
#include "kernels.h"

namespace {

int fail(const std::string& msg) {
  qsb::set_last_error(msg);
  return QS_ERR_INVALID;
}

template <typename R>
int fuse(const qs_op* in, int nin, qs_op* out, void* mats, int* nout) {
  using Cx = std::complex<R>;
  Cx* M = static_cast<Cx*>(mats);  // 16 entries per output slot
  int maxq = -1;
  for (int i = 0; i < nin; ++i) {
    const qs_op& o = in[i];
    if (o.u_on_device) return fail("qs_fuse_ops: device matrices are not fused on the host");
    if (!o.U) return fail("qs_fuse_ops: null matrix");
    if (o.kind == QS_OP_1Q) {
      if (o.q0 < 0) return fail("qs_fuse_ops: invalid q0");
      maxq = o.q0 > maxq ? o.q0 : maxq;
    } else if (o.kind == QS_OP_2Q) {
      if (o.q0 < 0 || o.q1 < 0) return fail("qs_fuse_ops: invalid qubit");
      if (o.q0 == o.q1) return fail("qs_fuse_ops: q0 == q1");
      maxq = std::max(maxq, std::max(o.q0, o.q1));
    } else {
      return fail("qs_fuse_ops: unknown op kind: " + std::to_string(o.kind));
    }
  }
  std::vector<int> last(maxq + 1, -1);  // last fused entry touching each qubit
  int n = 0;
  Cx tmp[16];
  for (int i = 0; i < nin; ++i) {
    const qs_op& o = in[i];
    const Cx* U = static_cast<const Cx*>(o.U);
    if (o.kind == QS_OP_1Q) {
      const int idx = last[o.q0];
      if (idx >= 0 && out[idx].kind == QS_OP_1Q && out[idx].q0 == o.q0) {
        Cx* P = M + 16 * idx;  // U @ P, 2x2 row-major
        for (int r = 0; r < 2; ++r)
          for (int c = 0; c < 2; ++c) tmp[2 * r + c] = U[2 * r] * P[c] + U[2 * r + 1] * P[2 + c];
        std::memcpy(P, tmp, 4 * sizeof(Cx));
        continue;
      }
      std::memcpy(M + 16 * n, U, 4 * sizeof(Cx));
      out[n] = o;
      out[n].q1 = -1;
      out[n].U = M + 16 * n;
      last[o.q0] = n++;
    } else {
      const int idx = std::max(last[o.q0], last[o.q1]);
      if (idx >= 0 && out[idx].kind == QS_OP_2Q && out[idx].q0 == o.q0 && out[idx].q1 == o.q1) {
        Cx* P = M + 16 * idx;  // U @ P, 4x4 row-major
        for (int r = 0; r < 4; ++r)
          for (int c = 0; c < 4; ++c) {
            Cx s = U[4 * r] * P[c];
            for (int k = 1; k < 4; ++k) s += U[4 * r + k] * P[4 * k + c];
            tmp[4 * r + c] = s;
          }
        std::memcpy(P, tmp, 16 * sizeof(Cx));
        continue;
      }
      std::memcpy(M + 16 * n, U, 16 * sizeof(Cx));
      out[n] = o;
      out[n].U = M + 16 * n;
      last[o.q0] = last[o.q1] = n++;
    }
  }
  *nout = n;
  return 0;
}

}  // namespace

extern "C" int qs_fuse_ops(int dtype, const qs_op* in, int nin, qs_op* out, void* mats, int* nout) {
  if (nin < 0 || (nin > 0 && (!in || !out || !mats)) || !nout) return fail("qs_fuse_ops: invalid argument");
  if (dtype == QS_C64) return fuse<float>(in, nin, out, mats, nout);
  if (dtype == QS_C128) return fuse<double>(in, nin, out, mats, nout);
  return fail("qs_fuse_ops: dtype must be QS_C64 or QS_C128");
}
