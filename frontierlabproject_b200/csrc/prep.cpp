// Host preparation of a tile's op list in one call (the per-gate Python loop of the reference's
// native branch, qgpusim/backends/custom/backend.py:432-451, and its gate-matrix cache and
// fusion, backend.py:16-200): each gate's matrix is built from its name and parameters, the list
// is optionally fused (fuse.cpp: consecutive gates on the same qubit / ordered pair multiplied,
// U_new = U @ U_prev) and packed into qs_op entries whose matrices live in the caller's buffer.
//
// The matrices are the textbook definitions in the little-endian convention of the reference's
// gates (matrix index b_q0 + 2*b_q1, q0 the control of controlled gates), evaluated in double
// precision with the same operations, in the same order, as frontierlabproject_b200/gates.py,
// then rounded to the state's precision: the entries equal those of the Python gate table.
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qsim_b200.h"
#include "kernels.h"

namespace {

using cd = std::complex<double>;

int fail(const std::string& msg) {
  qsb::set_last_error(msg);
  return QS_ERR_INVALID;
}

// Python's complex * float: the float promoted to (f, 0.0), then the full complex product
cd mulf(cd z, double f) { return cd(z.real() * f - z.imag() * 0.0, z.real() * 0.0 + z.imag() * f); }
// cmath.exp(1j * y) for a real y
cd expi(double y) { return std::exp(cd(0.0 * y, y)); }

// d x d row-major matrix of gate id (QS_GATE_*) with parameters p; false for an unknown id
bool gate_matrix(int id, const double* p, cd* U, int* arity) {
  const double s2 = 1.0 / std::sqrt(2.0);
  auto one = [&](cd a, cd b, cd c, cd d) {
    *arity = 1;
    U[0] = a; U[1] = b; U[2] = c; U[3] = d;
    return true;
  };
  auto diag4 = [&](cd a, cd b, cd c, cd d) {
    *arity = 2;
    for (int i = 0; i < 16; ++i) U[i] = 0.0;
    U[0] = a; U[5] = b; U[10] = c; U[15] = d;
    return true;
  };
  // control on matrix bit 0 (q0), 2x2 block on indices 1 and 3
  auto ctrl = [&](cd a, cd b, cd c, cd d) {
    *arity = 2;
    for (int i = 0; i < 16; ++i) U[i] = 0.0;
    U[0] = 1.0; U[10] = 1.0;
    U[5] = a; U[7] = b; U[13] = c; U[15] = d;
    return true;
  };
  const cd I(0.0, 1.0);
  switch (id) {
    case QS_GATE_ID: return one(1.0, 0.0, 0.0, 1.0);
    case QS_GATE_H: return one(s2, s2, s2, -s2);
    case QS_GATE_X: return one(0.0, 1.0, 1.0, 0.0);
    case QS_GATE_Y: return one(0.0, cd(-0.0, -1.0), cd(0.0, 1.0), 0.0);
    case QS_GATE_Z: return one(1.0, 0.0, 0.0, -1.0);
    case QS_GATE_S: return one(1.0, 0.0, 0.0, I);
    case QS_GATE_SDG: return one(1.0, 0.0, 0.0, cd(-0.0, -1.0));
    case QS_GATE_T: return one(1.0, 0.0, 0.0, std::exp(cd(0.0, M_PI) / 4.0));
    case QS_GATE_TDG: return one(1.0, 0.0, 0.0, std::exp(cd(-0.0, -M_PI) / 4.0));
    case QS_GATE_SX: return one(cd(0.5, 0.5), cd(0.5, -0.5), cd(0.5, -0.5), cd(0.5, 0.5));
    case QS_GATE_RX: {
      const double a = std::cos(p[0] / 2), b = std::sin(p[0] / 2);
      const cd mib = mulf(cd(-0.0, -1.0), b);
      return one(a, mib, mib, a);
    }
    case QS_GATE_RY: {
      const double a = std::cos(p[0] / 2), b = std::sin(p[0] / 2);
      return one(a, -b, b, a);
    }
    case QS_GATE_RZ:
      return one(std::exp(mulf(cd(-0.0, -0.5), p[0])), 0.0, 0.0, std::exp(mulf(cd(0.0, 0.5), p[0])));
    case QS_GATE_P: return one(1.0, 0.0, 0.0, std::exp(mulf(I, p[0])));
    case QS_GATE_U: {
      const double th = p[0], ph = p[1], la = p[2];
      const double a = std::cos(th / 2), b = std::sin(th / 2);
      return one(a, mulf(-std::exp(mulf(I, la)), b), mulf(std::exp(mulf(I, ph)), b), mulf(std::exp(mulf(I, ph + la)), a));
    }
    case QS_GATE_CX: return ctrl(0.0, 1.0, 1.0, 0.0);
    case QS_GATE_CY: return ctrl(0.0, cd(-0.0, -1.0), cd(0.0, 1.0), 0.0);
    case QS_GATE_CZ: return diag4(1.0, 1.0, 1.0, -1.0);
    case QS_GATE_CP: return diag4(1.0, 1.0, 1.0, std::exp(mulf(I, p[0])));
    case QS_GATE_CRZ:
      return ctrl(std::exp(mulf(cd(-0.0, -0.5), p[0])), 0.0, 0.0, std::exp(mulf(cd(0.0, 0.5), p[0])));
    case QS_GATE_SWAP:
      *arity = 2;
      for (int i = 0; i < 16; ++i) U[i] = 0.0;
      U[0] = 1.0; U[6] = 1.0; U[9] = 1.0; U[15] = 1.0;
      return true;
    case QS_GATE_RZZ: {
      const cd e0 = std::exp(mulf(cd(-0.0, -0.5), p[0])), e1 = std::exp(mulf(cd(0.0, 0.5), p[0]));
      return diag4(e0, e1, e1, e0);
    }
    default: return false;
  }
}

template <typename R>
int prepare(int ngates, const int* gid, const double* params, const int* q0, const int* q1, const double* custom,
            int fuse, qs_op* out, void* mats, int* nout) {
  using Cx = std::complex<R>;
  Cx* M = static_cast<Cx*>(mats);
  // unfused ops first: packed into out[] with matrices in their own slots of mats
  std::vector<qs_op> raw(ngates);
  std::vector<Cx> rawm(fuse ? 16 * (size_t)ngates : 0);
  Cx* dst = fuse ? rawm.data() : M;
  cd U[16];
  for (int i = 0; i < ngates; ++i) {
    int arity = 0;
    if (gid[i] == QS_GATE_MATRIX) {
      if (!custom) return fail("qs_prepare_ops: gate " + std::to_string(i) + " needs a custom matrix");
      arity = q1[i] >= 0 ? 2 : 1;
      const double* c = custom + 32 * (size_t)i;
      for (int k = 0; k < (arity == 1 ? 4 : 16); ++k) U[k] = cd(c[2 * k], c[2 * k + 1]);
    } else if (!gate_matrix(gid[i], params + 3 * (size_t)i, U, &arity)) {
      return fail("qs_prepare_ops: unknown gate id " + std::to_string(gid[i]));
    }
    if ((arity == 2) != (q1[i] >= 0)) return fail("qs_prepare_ops: gate " + std::to_string(i) + " has the wrong arity");
    if (q0[i] < 0 || (arity == 2 && q0[i] == q1[i])) return fail("qs_prepare_ops: invalid qubits of gate " + std::to_string(i));
    Cx* m = dst + 16 * (size_t)i;
    for (int k = 0; k < (arity == 1 ? 4 : 16); ++k) m[k] = Cx((R)U[k].real(), (R)U[k].imag());
    raw[i] = qs_op{arity == 1 ? QS_OP_1Q : QS_OP_2Q, q0[i], arity == 1 ? -1 : q1[i], 0, m};
  }
  if (!fuse) {
    std::memcpy(out, raw.data(), sizeof(qs_op) * (size_t)ngates);
    *nout = ngates;
    return 0;
  }
  return qs_fuse_ops(sizeof(R) == 4 ? QS_C64 : QS_C128, raw.data(), ngates, out, mats, nout);
}

}  // namespace

extern "C" int qs_gate_matrix(int gate_id, const double* params, double* out, int* arity) {
  if (!out || !arity) return fail("qs_gate_matrix: null argument");
  static const double zero[3] = {0.0, 0.0, 0.0};
  cd U[16];
  if (!gate_matrix(gate_id, params ? params : zero, U, arity)) return fail("qs_gate_matrix: unknown gate id " + std::to_string(gate_id));
  for (int k = 0; k < (*arity == 1 ? 4 : 16); ++k) {
    out[2 * k] = U[k].real();
    out[2 * k + 1] = U[k].imag();
  }
  return 0;
}

extern "C" int qs_prepare_ops(int dtype, int ngates, const int* gate_id, const double* params, const int* q0,
                              const int* q1, const double* custom, int fuse, qs_op* out, void* mats, int* nout) {
  if (ngates < 0 || !nout || (ngates > 0 && (!gate_id || !params || !q0 || !q1 || !out || !mats)))
    return fail("qs_prepare_ops: invalid argument");
  if (ngates == 0) {
    *nout = 0;
    return 0;
  }
  if (dtype == QS_C64) return prepare<float>(ngates, gate_id, params, q0, q1, custom, fuse, out, mats, nout);
  if (dtype == QS_C128) return prepare<double>(ngates, gate_id, params, q0, q1, custom, fuse, out, mats, nout);
  return fail("qs_prepare_ops: dtype must be QS_C64 or QS_C128");
}
