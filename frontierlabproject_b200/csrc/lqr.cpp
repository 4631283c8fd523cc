// Lazy qubit reordering (LQR) flat tiling on qubit bit masks: Alg. 1 (flat tiling with the
// forced single-gate tile), Alg. 2 (tile construction) and Alg. 3 (greedy qubit mapping) of
// qgpusim/transpiler/passes.py:89-243, and the tile extraction of passes.py:247-272.  The
// gates arrive depth-sorted (passes.py:359-420 computes and sorts the depths); every set of
// the reference is a 64-bit mask here, so one tile costs one scan of the remaining gates.
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/qsim_b200.h"
#include "kernels.h"

namespace {

int fail(const char* msg) {
  qsb::set_last_error(msg);
  return QS_ERR_INVALID;
}

inline int popc64(uint64_t x) { return __builtin_popcountll(x); }

// lowest qubits of `from` outside `s` added to `s` until it has `nL` qubits
uint64_t fill_lowest(uint64_t s, uint64_t from, int nL) {
  for (int q = 0; q < 64 && popc64(s) < nL; ++q)
    if (((from >> q) & 1ull) && !((s >> q) & 1ull)) s |= 1ull << q;
  return s;
}

}  // namespace

extern "C" int qs_lqr_flat_tiling(int num_qubits, int nL, const unsigned long long* targets, int ngates,
                                  int* order, int* tile_of, unsigned long long* tile_masks, int* ntiles) {
  if (num_qubits < 1 || num_qubits > 64 || nL < 1 || ngates < 0 || (ngates > 0 && (!targets || !order || !tile_of)) ||
      !tile_masks || !ntiles)
    return fail("qs_lqr_flat_tiling: invalid argument");
  const uint64_t Q = num_qubits == 64 ? ~0ull : ((1ull << num_qubits) - 1);
  std::vector<int> remaining(ngates), next;
  for (int i = 0; i < ngates; ++i) {
    if (targets[i] & ~Q) return fail("qs_lqr_flat_tiling: gate qubit out of range");
    remaining[i] = i;
  }
  std::vector<uint64_t> ql_of(ngates);
  int nsched = 0;
  uint64_t QL = fill_lowest(0, Q, nL);  // the lowest min(nL, n) qubits
  std::vector<int> picked;
  while (!remaining.empty()) {
    // Alg. 2: gates whose qubits are all still available in QL, in order
    picked.clear();
    uint64_t avail = QL;
    for (int g : remaining) {
      const uint64_t t = targets[g];
      if ((t & ~avail) == 0) {
        picked.push_back(g);
      } else {
        avail &= ~t;
        if (!avail) break;
      }
    }
    if (picked.empty()) {
      // forced tile: the first remaining gate alone, QL = its qubits + the lowest others
      const int first = remaining[0];
      QL = targets[first];
      if (popc64(QL) < nL) QL = fill_lowest(QL, Q, nL);
      picked.push_back(first);
    }
    for (int g : picked) {
      order[nsched] = g;
      ql_of[nsched] = QL;
      ++nsched;
    }
    // remove the picked gates (both lists are in schedule order)
    next.clear();
    size_t k = 0;
    for (int g : remaining) {
      if (k < picked.size() && picked[k] == g) { ++k; continue; }
      next.push_back(g);
    }
    remaining.swap(next);
    if (remaining.empty()) break;
    // Alg. 3: greedy mapping of the next tile's qubits
    uint64_t chosen = 0;
    avail = Q;
    for (int g : remaining) {
      const uint64_t t = targets[g];
      if ((t & ~avail) == 0 && popc64(chosen | t) <= nL) {
        chosen |= t;
      } else {
        avail &= ~t;
        if (!avail) break;
      }
    }
    QL = chosen ? fill_lowest(chosen, Q, nL) : 0ull;
  }
  // tiles: runs of consecutive scheduled gates with the same qubit set
  int nt = 0;
  for (int s = 0; s < nsched; ++s) {
    if (s == 0 || ql_of[s] != ql_of[s - 1]) tile_masks[nt++] = ql_of[s];
    tile_of[s] = nt - 1;
  }
  *ntiles = nt;
  return 0;
}
