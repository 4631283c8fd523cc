// Pass / phase planning and program encoding for the pass kernel.
#include "plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace qsb {

static inline uint64_t bit(int p) { return 1ull << p; }
static inline int popc(uint64_t x) { return __builtin_popcountll(x); }

static bool is_zero(const cplx& z) { return z.real() == 0.0 && z.imag() == 0.0; }
static bool is_one(const cplx& z) { return z.real() == 1.0 && z.imag() == 0.0; }

COp classify(const QOp& op) {
  COp c;
  const cplx* U = op.U;
  if (op.arity == 1) {
    c.a = op.q0;
    c.touch = bit(op.q0);
    if (is_zero(U[1]) && is_zero(U[2])) {
      c.kind = GK_1Q_DIAG; c.ncoef = 2; c.coef[0] = U[0]; c.coef[1] = U[3];
      c.need = 0;
      return c;
    }
    c.need = bit(op.q0);
    if (is_zero(U[0]) && is_zero(U[3]) && is_one(U[1]) && is_one(U[2])) {
      c.kind = GK_1Q_X; c.ncoef = 0;
      return c;
    }
    c.ncoef = 4;
    for (int i = 0; i < 4; ++i) c.coef[i] = U[i];
    bool real = true, reim = true;
    for (int i = 0; i < 4; ++i) if (U[i].imag() != 0.0) real = false;
    if (U[0].imag() != 0.0 || U[3].imag() != 0.0 || U[1].real() != 0.0 || U[2].real() != 0.0) reim = false;
    c.kind = real ? GK_1Q_REAL : (reim ? GK_1Q_REIM : GK_1Q_DENSE);
    return c;
  }
  // two-qubit; index = b_q0 + 2 b_q1
  const int q0 = op.q0, q1 = op.q1;
  c.touch = bit(q0) | bit(q1);
  auto M = [&](int r, int col) { return U[4 * r + col]; };
  bool diag = true;
  for (int r = 0; r < 4; ++r)
    for (int col = 0; col < 4; ++col)
      if (r != col && !is_zero(M(r, col))) diag = false;
  if (diag) {
    c.kind = GK_2Q_DIAG; c.a = q0; c.b = q1; c.ncoef = 4;
    for (int i = 0; i < 4; ++i) c.coef[i] = M(i, i);
    c.need = 0;
    return c;
  }
  // SWAP
  {
    static const int P[4] = {0, 2, 1, 3};
    bool sw = true;
    for (int r = 0; r < 4; ++r)
      for (int col = 0; col < 4; ++col) {
        cplx want = (col == P[r]) ? cplx(1, 0) : cplx(0, 0);
        if (M(r, col) != want) sw = false;
      }
    if (sw) {
      c.kind = GK_2Q_SWAP; c.a = q0; c.b = q1; c.ncoef = 0; c.need = c.touch;
      return c;
    }
  }
  // controlled on matrix bit cb (0 -> q0, 1 -> q1): identity where that bit is 0 and
  // no coupling between the two halves.
  for (int cb = 0; cb < 2; ++cb) {
    const int cm = 1 << cb, tm = 1 << (1 - cb);
    bool ok = true;
    for (int r = 0; r < 4 && ok; ++r)
      for (int col = 0; col < 4 && ok; ++col) {
        const bool rc = r & cm, cc = col & cm;
        if (!rc || !cc) {
          cplx want = (r == col && !rc) ? cplx(1, 0) : cplx(0, 0);
          if (M(r, col) != want) ok = false;
        }
      }
    if (!ok) continue;
    // block on the control = 1 half: rows/cols cm and cm|tm
    cplx u00 = M(cm, cm), u01 = M(cm, cm | tm), u10 = M(cm | tm, cm), u11 = M(cm | tm, cm | tm);
    c.a = cb == 0 ? q0 : q1;
    c.b = cb == 0 ? q1 : q0;
    c.need = bit(c.b);
    if (is_zero(u00) && is_zero(u11) && is_one(u01) && is_one(u10)) {
      c.kind = GK_2Q_CX; c.ncoef = 0;
    } else {
      c.kind = GK_2Q_CU; c.ncoef = 4;
      c.coef[0] = u00; c.coef[1] = u01; c.coef[2] = u10; c.coef[3] = u11;
    }
    return c;
  }
  c.kind = GK_2Q_DENSE; c.a = q0; c.b = q1; c.ncoef = 16;
  for (int i = 0; i < 16; ++i) c.coef[i] = U[i];
  c.need = c.touch;
  return c;
}

// ---------------------------------------------------------------------------------
// helpers of the per-pass scalar extraction
// ---------------------------------------------------------------------------------
namespace {

cplx snap(cplx z, double scale) {
  const double eps = 1e-14 * scale;
  return cplx(std::abs(z.real()) < eps ? 0.0 : z.real(), std::abs(z.imag()) < eps ? 0.0 : z.imag());
}

}  // namespace

// ---------------------------------------------------------------------------------
// Per-pass scalar extraction: each gate with coefficients is written s * V with one entry
// of V exactly 1, choosing the entry that leaves the most entries in {0, +-1, +-i} (an
// add instead of a multiply in the specialised kernels): H = (1/sqrt2)[[1,1],[1,-1]],
// RX(t) = cos(t/2)[[1,-i tan],[-i tan,1]], SX = ((1+i)/2)[[1,-i],[-i,1]], RZ = e^{-it/2}
// diag(1, e^{it}).  The product of a pass's scalars is multiplied into one gate of the
// same pass, so magnitudes stay bounded in single precision and the state is unchanged.
// ---------------------------------------------------------------------------------
namespace {

int entry_cost(const cplx& z) {
  const double r = z.real(), i = z.imag();
  if (r == 0.0 && i == 0.0) return 0;
  if ((i == 0.0 && (r == 1.0 || r == -1.0)) || (r == 0.0 && (i == 1.0 || i == -1.0))) return 1;
  if (i == 0.0 || r == 0.0) return 2;
  return 4;
}

int matrix_cost(const cplx* U, int d) {
  int c = 0;
  for (int e = 0; e < d * d; ++e) c += entry_cost(U[e]);
  return c;
}

bool carries_coefficients(const QOp& o) {
  // permutations (X, CX, SWAP) carry none; everything else is multiplied entry by entry
  const int d = o.arity == 1 ? 2 : 4;
  for (int e = 0; e < d * d; ++e) {
    const cplx z = o.U[e];
    if (!(z == cplx(0, 0) || z == cplx(1, 0))) return true;
  }
  return false;
}

// the rewritten gate keeps the shape the planner used: same staged/register needs, same
// operand roles, same diagonal / controlled / dense family
bool same_shape(const QOp& o, const cplx* V) {
  QOp b = o;
  const int d = o.arity == 1 ? 2 : 4;
  for (int k = 0; k < d * d; ++k) b.U[k] = V[k];
  const COp x = classify(o), y = classify(b);
  if (x.need != y.need || x.touch != y.touch || x.a != y.a || x.b != y.b) return false;
  if (o.arity == 2) return x.kind == y.kind;
  return (x.kind == GK_1Q_DIAG) == (y.kind == GK_1Q_DIAG) && (x.kind == GK_1Q_X) == (y.kind == GK_1Q_X);
}

}  // namespace

Program build_program(std::vector<QOp>& ops, const std::vector<PlannedPass>& passes, int n, int dtype, int r) {
  for (const PlannedPass& ps : passes) extract_pass_scalars(ops, ps.ops);
  std::vector<COp> cops;
  cops.reserve(ops.size());
  for (const QOp& o : ops) cops.push_back(classify(o));
  return encode_program(passes, cops, n, dtype, r);
}

void extract_pass_scalars(std::vector<QOp>& ops, const std::vector<int>& pass_ops, bool diag_absorbs) {
  cplx total(1.0, 0.0);
  int absorber = -1, absorber_cost = -1;
  // Dividing a gate by its pivot p scales the state by 1/|p| until the pass's scalar is
  // multiplied back in.  log2 of that running factor is kept within +-kMaxLog2 at every gate
  // (whichever gate absorbs the product, the state stays within 2^(+-2 kMaxLog2) of its
  // norm: far inside the single-precision exponent range); a gate whose pivot would leave
  // the band keeps its matrix.
  constexpr double kMaxLog2 = 24.0;
  double log2_scale = 0.0;
  for (int oi : pass_ops) {
    QOp& o = ops[oi];
    const int d = o.arity == 1 ? 2 : 4;
    if (!carries_coefficients(o)) continue;
    double scale = 0.0;
    for (int e = 0; e < d * d; ++e) scale = std::max(scale, std::abs(o.U[e]));
    if (scale == 0.0) continue;
    int best = matrix_cost(o.U, d);
    int best_e = -1;
    double best_mag = 0.0;
    cplx bestV[16];
    for (int e = 0; e < d * d; ++e) {
      const double mag = std::abs(o.U[e]);
      if (mag < 1e-6 * scale) continue;  // keep scaled entries bounded
      const double step = -std::log2(mag);
      if (std::abs(log2_scale + step) > kMaxLog2) continue;
      cplx V[16];
      for (int k = 0; k < d * d; ++k) V[k] = snap(o.U[k] / o.U[e], scale / mag);
      for (int k = 0; k < d * d; ++k)  // entries equal to the pivot divide to exactly one
        if (o.U[k] == o.U[e]) V[k] = cplx(1.0, 0.0);
      V[e] = cplx(1.0, 0.0);
      const int c = matrix_cost(V, d);
      // among pivots of equal cost the first, unless a later one is far larger (RX(t) within
      // about 0.008 of t = pi pivots on its sine, not on its vanishing cosine); the choice, and
      // with it the zero/one/real/imaginary class of every entry, stays the same for most
      // parameter values, so the specialised kernels are reused across parameter changes
      if ((c < best || (c == best && best_e >= 0 && mag > 256.0 * best_mag)) && same_shape(o, V)) {
        best = c;
        best_e = e;
        best_mag = mag;
        for (int k = 0; k < d * d; ++k) bestV[k] = V[k];
      }
    }
    if (best_e >= 0) {
      total *= o.U[best_e];
      log2_scale -= std::log2(best_mag);
      for (int k = 0; k < d * d; ++k) o.U[k] = bestV[k];
    }
    // absorber: a gate whose shape survives scaling, and whose cost grows least
    const COp c0 = classify(o);
    bool can_absorb = o.arity == 1 || c0.kind == GK_2Q_DIAG || c0.kind == GK_2Q_DENSE;
    if (!diag_absorbs && (c0.kind == GK_1Q_DIAG || c0.kind == GK_2Q_DIAG)) can_absorb = false;
    if (!can_absorb) continue;
    int grow = 0;
    for (int k = 0; k < d * d; ++k) grow += (o.U[k] == cplx(0, 0)) ? 0 : 4 - entry_cost(o.U[k]);
    if (absorber < 0 || grow < absorber_cost) { absorber = oi; absorber_cost = grow; }
  }
  if (total == cplx(1.0, 0.0)) return;
  if (absorber < 0 && !diag_absorbs && std::abs(std::abs(total) - 1.0) < 1e-9) return;  // a phase
  if (absorber < 0) throw std::runtime_error("planner: no gate of the pass can absorb its scalar");
  QOp& a = ops[absorber];
  const int d = a.arity == 1 ? 2 : 4;
  for (int k = 0; k < d * d; ++k) a.U[k] *= total;
}

// ---------------------------------------------------------------------------------
// Greedy + hill-climbing choice of a bit set of size `cap` (containing `forced`) that
// executes the longest dependency-closed run of the remaining ops; `restarts` perturbed
// climbs from the best set found (iterated local search).
// ---------------------------------------------------------------------------------
namespace {

struct Scan {
  const std::vector<COp>& ops;
  uint64_t universe;   // bits whose blocking ends the scan
  // phases: among sets executing equally many gates, prefer those that also hold the
  // controls and diagonal bits of the executed gates (register renames / half multiplies)
  bool soft = false;
  // ops (in order) executable with staged set S
  void run(const std::vector<int>& rem, uint64_t S, std::vector<int>& out) const {
    out.clear();
    uint64_t blocked = 0;
    for (int i : rem) {
      const COp& o = ops[i];
      if (o.touch & blocked) { blocked |= o.touch; }
      else if ((o.need & ~S) == 0) { out.push_back(i); }
      else { blocked |= o.touch; }
      if ((blocked & universe) == universe) break;
    }
  }
  size_t count(const std::vector<int>& rem, uint64_t S) const {
    size_t c = 0, inside = 0;
    uint64_t blocked = 0;
    for (int i : rem) {
      const COp& o = ops[i];
      if (o.touch & blocked) { blocked |= o.touch; }
      else if ((o.need & ~S) == 0) { ++c; if ((o.touch & ~S) == 0) ++inside; }
      else { blocked |= o.touch; }
      if ((blocked & universe) == universe) break;
    }
    return soft ? (c << 8) + inside : c;
  }
};

uint64_t choose_set(const Scan& sc, const std::vector<int>& rem, uint64_t candidates, uint64_t forced,
                    int cap, int iters, int restarts = 0,
                    std::vector<std::pair<size_t, uint64_t>>* optima = nullptr) {
  uint64_t S = forced;
  // greedy seed in op order
  uint64_t blocked = 0;
  std::vector<uint64_t> lookahead;
  for (int i : rem) {
    const COp& o = sc.ops[i];
    if (o.touch & blocked) { blocked |= o.touch; if (o.need) lookahead.push_back(o.need); continue; }
    if ((o.need & ~S) == 0) continue;
    if (popc(S | o.need) <= cap) S |= o.need;
    else { blocked |= o.touch; lookahead.push_back(o.need); }
    if ((blocked & sc.universe) == sc.universe) break;
  }
  // fill with bits the blocked ops need next, then the lowest free bits
  for (uint64_t nd : lookahead) {
    if (popc(S) >= cap) break;
    if (popc(S | nd) <= cap) S |= nd;
  }
  for (int p = 0; p < 64 && popc(S) < cap; ++p)
    if ((candidates & bit(p)) && !(S & bit(p))) S |= bit(p);
  // first-improvement hill climbing over single-bit swaps (at most `iters` improvements)
  auto climb = [&](uint64_t& X) {
    size_t bx = sc.count(rem, X);
    for (int it = 0; it < iters; ++it) {
      bool improved = false;
      for (int a = 0; a < 64 && !improved; ++a) {
        if (!(X & bit(a)) || (forced & bit(a))) continue;
        for (int b = 0; b < 64; ++b) {
          if (!(candidates & bit(b)) || (X & bit(b))) continue;
          uint64_t T = (X & ~bit(a)) | bit(b);
          size_t c = sc.count(rem, T);
          if (c > bx) { bx = c; X = T; improved = true; break; }
        }
      }
      if (!improved) break;
    }
    return bx;
  };
  size_t best = climb(S);
  if (optima) optima->push_back({best, S});
  // iterated local search: restart the climb from the best set with three random bit swaps
  // (a fixed xorshift sequence per call: plans are deterministic), keep strict improvements
  uint64_t rng = 0x9E3779B97F4A7C15ull ^ ((uint64_t)rem.size() * 0xBF58476D1CE4E5B9ull);
  auto next = [&rng]() {
    rng ^= rng << 13;
    rng ^= rng >> 7;
    rng ^= rng << 17;
    return rng;
  };
  std::vector<int> in, out;
  for (int r = 0; r < restarts; ++r) {
    uint64_t T = S;
    for (int k = 0; k < 3; ++k) {
      in.clear();
      out.clear();
      for (int p = 0; p < 64; ++p) {
        if ((T & bit(p)) && !(forced & bit(p))) in.push_back(p);
        else if ((candidates & bit(p)) && !(T & bit(p))) out.push_back(p);
      }
      if (in.empty() || out.empty()) break;
      const int a = in[next() % in.size()], b = out[next() % out.size()];
      T = (T & ~bit(a)) | bit(b);
    }
    const size_t c = climb(T);
    if (optima) optima->push_back({c, T});
    if (c > best) { best = c; S = T; }
  }
  return S;
}

std::vector<int> bits_of(uint64_t m) {
  std::vector<int> v;
  for (int p = 0; p < 64; ++p) if (m & bit(p)) v.push_back(p);
  return v;
}

}  // namespace

// Every r-subset of the staged bits (containing `forced`): the register set of a phase that
// executes the most gates (soft score of Scan).
static uint64_t choose_phase_exhaustive(const Scan& sc, const std::vector<int>& rem, uint64_t Smask, uint64_t forced,
                                        int r, std::vector<std::pair<size_t, uint64_t>>* top = nullptr) {
  std::vector<int> free_bits;
  for (int p : bits_of(Smask))
    if (!(forced & bit(p))) free_bits.push_back(p);
  const int need = r - __builtin_popcountll(forced);
  const int nf = (int)free_bits.size();
  uint64_t best = 0;
  size_t best_v = 0;
  bool have = false;
  std::vector<int> idx(need);
  for (int i = 0; i < need; ++i) idx[i] = i;
  if (need <= 0 || need > nf) return forced;
  for (;;) {
    uint64_t R = forced;
    for (int i : idx) R |= bit(free_bits[i]);
    const size_t v = sc.count(rem, R);
    if (!have || v > best_v) { best = R; best_v = v; have = true; }
    if (top) top->push_back({v, R});
    int i = need - 1;
    while (i >= 0 && idx[i] == nf - need + i) --i;
    if (i < 0) break;
    ++idx[i];
    for (int j = i + 1; j < need; ++j) idx[j] = idx[j - 1] + 1;
  }
  return best;
}

static std::vector<PlannedPhase> plan_phases(const std::vector<COp>& ops, const std::vector<int>& pass_ops,
                                             const std::vector<int>& sbits, int r, int iters, bool pair_bit,
                                             int lookahead) {
  // Phases choose register bits among the staged physical bits; op need masks are
  // physical, so the phase set is a physical mask, converted to local bits at the end.
  uint64_t Smask = 0;
  for (int p : sbits) Smask |= bit(p);
  const int rr = std::min<int>(r, (int)sbits.size());
  Scan sc{ops, Smask, true};
  std::vector<PlannedPhase> phases;
  std::vector<int> rem = pass_ops, taken, rest;
  while (!rem.empty()) {
    const uint64_t forced = (pair_bit && (Smask & 1ull)) ? 1ull : 0ull;
    std::vector<std::pair<size_t, uint64_t>> top;
    uint64_t R = 0;
    if (lookahead <= 0) {
      R = choose_set(sc, rem, Smask, forced, rr, iters);
    } else {
      // every register set is scored; among the `lookahead` best, the one after which greedy
      // phases (best set each) finish the pass soonest
      R = choose_phase_exhaustive(sc, rem, Smask, forced, rr, &top);
      std::stable_sort(top.begin(), top.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
      if ((int)top.size() > lookahead) top.resize(lookahead);
      int best_np = 1 << 30;
      std::vector<int> r1, r2, tk;
      auto drop = [&](const std::vector<int>& rr0, uint64_t X, std::vector<int>& out) {
        sc.run(rr0, X, tk);
        out.clear();
        size_t t2 = 0;
        for (int i : rr0) {
          if (t2 < tk.size() && tk[t2] == i) { ++t2; continue; }
          out.push_back(i);
        }
      };
      for (const auto& c : top) {
        drop(rem, c.second, r1);
        int np = 1;
        while (!r1.empty() && np < best_np) {
          const uint64_t X = choose_phase_exhaustive(sc, r1, Smask, forced, rr);
          drop(r1, X, r2);
          r1.swap(r2);
          ++np;
        }
        if (np < best_np) { best_np = np; R = c.second; }
      }
    }
    sc.run(rem, R, taken);
    if (taken.empty()) throw std::runtime_error("planner: phase made no progress");
    PlannedPhase ph;
    for (int p : bits_of(R)) {
      auto it = std::find(sbits.begin(), sbits.end(), p);
      ph.rbits.push_back((int)(it - sbits.begin()));
    }
    ph.ops = taken;
    phases.push_back(ph);
    rest.clear();
    size_t t = 0;
    for (int i : rem) {
      if (t < taken.size() && taken[t] == i) { ++t; continue; }
      rest.push_back(i);
    }
    rem.swap(rest);
  }
  return phases;
}

std::vector<PlannedPass> plan_passes(const std::vector<COp>& ops, int n, const PlanConfig& cfg) {
  std::vector<PlannedPass> out;
  if (ops.empty()) return out;
  const int m = std::min(cfg.m, n);
  const int k = std::min(cfg.k, m);
  const uint64_t all = (n >= 64) ? ~0ull : (bit(n) - 1);
  const uint64_t forced = (k >= 64) ? ~0ull : (bit(k) - 1);
  Scan sc{ops, all};
  std::vector<int> rem(ops.size()), taken, rest;
  for (size_t i = 0; i < ops.size(); ++i) rem[i] = (int)i;
  while (!rem.empty()) {
    uint64_t S = all;
    if (m < n) {
      // lookahead: among the 4 best distinct local optima of the search, the set after which
      // `lookahead` more greedy passes execute the most gates
      std::vector<std::pair<size_t, uint64_t>> opt;
      S = choose_set(sc, rem, all, forced, m, cfg.hill_iters, cfg.hill_iters, cfg.lookahead > 0 ? &opt : nullptr);
      if (cfg.lookahead > 0 && opt.size() > 1) {
        std::stable_sort(opt.begin(), opt.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        std::vector<std::pair<size_t, uint64_t>> cand;
        for (const auto& o : opt) {
          bool dup = false;
          for (const auto& c : cand) dup = dup || c.second == o.second;
          if (!dup) cand.push_back(o);
          if (cand.size() == 4) break;
        }
        std::vector<int> r1, r2, tk;
        auto drop = [&](const std::vector<int>& r, uint64_t X, std::vector<int>& out) {
          sc.run(r, X, tk);
          out.clear();
          size_t t2 = 0;
          for (int i : r) {
            if (t2 < tk.size() && tk[t2] == i) { ++t2; continue; }
            out.push_back(i);
          }
          return tk.size();
        };
        size_t best_v = 0;
        for (const auto& c : cand) {
          size_t v = drop(rem, c.second, r1);
          for (int d = 0; d < cfg.lookahead && !r1.empty(); ++d) {
            const uint64_t S2 = choose_set(sc, r1, all, forced, m, cfg.hill_iters, 4);
            v += drop(r1, S2, r2);
            r1.swap(r2);
          }
          if (v > best_v) { best_v = v; S = c.second; }
        }
      }
    }
    sc.run(rem, S, taken);
    if (taken.empty()) throw std::runtime_error("planner: pass made no progress");
    PlannedPass ps;
    ps.sbits = bits_of(S);
    ps.ops = taken;
    ps.phases = plan_phases(ops, taken, ps.sbits, cfg.r, cfg.hill_iters, cfg.pair_bit, cfg.phase_lookahead);
    out.push_back(std::move(ps));
    rest.clear();
    size_t t = 0;
    for (int i : rem) {
      if (t < taken.size() && taken[t] == i) { ++t; continue; }
      rest.push_back(i);
    }
    rem.swap(rest);
  }
  return out;
}

std::vector<PlannedPass> plan_permutation(const std::vector<int>& perm, int n, const PlanConfig& cfg) {
  // perm[b] = destination bit of the data at bit b.  Cycles are packed into passes whose
  // staged set (always holding the k lowest bits) has at most m bits; a cycle longer than
  // the free room is split: (c0 .. cL-1) = (c0 c_{j+1} .. c_{L-1}) after (c0 .. c_j), and
  // the pieces are placed first-fit (each after its cycle's previous piece).
  std::vector<PlannedPass> out;
  const int m = std::min(cfg.m, n);
  const int k = std::min(cfg.k, m);
  std::vector<int> cur(n);
  for (int b = 0; b < n; ++b) cur[b] = perm[b];
  // pieces: each a list of positions (c0, c1, ..., c_{L-1}) meaning data at c_i -> c_{i+1}
  std::vector<std::vector<int>> pieces;
  std::vector<bool> seen(n, false);
  for (int b = 0; b < n; ++b) {
    if (seen[b] || cur[b] == b) { seen[b] = true; continue; }
    std::vector<int> cyc;
    int x = b;
    while (!seen[x]) { seen[x] = true; cyc.push_back(x); x = cur[x]; }
    pieces.push_back(cyc);
  }
  auto extra = [&](const std::vector<int>& c) {
    int e = 0;
    for (int p : c) if (p >= k) ++e;
    return e;
  };
  const int room = m - k;
  // split long cycles
  std::vector<std::vector<int>> fitted;
  std::vector<int> cyc_of;  // cycle index of each piece
  for (size_t ci = 0; ci < pieces.size(); ++ci) {
    std::vector<int> cyc = pieces[ci];
    while (extra(cyc) > room) {
      // take the longest prefix c0..cj with extra() <= room
      std::vector<int> head;
      for (size_t i = 0; i < cyc.size(); ++i) {
        head.push_back(cyc[i]);
        if (extra(head) > room) { head.pop_back(); break; }
      }
      if (head.size() < 2) throw std::runtime_error("planner: cannot split permutation cycle");
      fitted.push_back(head);
      cyc_of.push_back((int)ci);
      std::vector<int> tail;
      tail.push_back(cyc[0]);
      for (size_t i = head.size(); i < cyc.size(); ++i) tail.push_back(cyc[i]);
      cyc.swap(tail);
    }
    if (cyc.size() >= 2) { fitted.push_back(cyc); cyc_of.push_back((int)ci); }
  }
  // first fit: each piece joins the earliest pass after its cycle's previous piece whose
  // positions it does not share and whose staged set keeps room
  std::vector<std::vector<std::vector<int>>> groups;
  std::vector<uint64_t> gmask;
  std::vector<int> last_pass(pieces.size(), -1);
  const uint64_t low = (k >= 64) ? ~0ull : (bit(k) - 1);
  for (size_t pi = 0; pi < fitted.size(); ++pi) {
    const auto& pc = fitted[pi];
    uint64_t pm = 0;
    for (int p : pc) pm |= bit(p);
    int g = last_pass[cyc_of[pi]] + 1;
    for (; g < (int)groups.size(); ++g)
      if (!(gmask[g] & pm) && popc((gmask[g] | pm) & ~low) <= room) break;
    if (g == (int)groups.size()) { groups.push_back({}); gmask.push_back(0); }
    groups[g].push_back(pc);
    gmask[g] |= pm;
    last_pass[cyc_of[pi]] = g;
  }
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    uint64_t S = gmask[gi] | ((k >= 64) ? ~0ull : (bit(k) - 1));
    // fill to m with the lowest free bits (keeps the group count at 2^(n-m))
    for (int p = 0; p < n && popc(S) < m; ++p) S |= bit(p);
    PlannedPass ps;
    ps.sbits = bits_of(S);
    std::vector<int> dest(n);
    for (int b = 0; b < n; ++b) dest[b] = b;
    for (auto& pc : groups[gi])
      for (size_t i = 0; i < pc.size(); ++i) dest[pc[i]] = pc[(i + 1) % pc.size()];
    ps.store_src.assign(ps.sbits.size(), 0);
    for (size_t u = 0; u < ps.sbits.size(); ++u) {
      int d = dest[ps.sbits[u]];
      auto it = std::find(ps.sbits.begin(), ps.sbits.end(), d);
      ps.store_src[it - ps.sbits.begin()] = (int)u;
    }
    out.push_back(std::move(ps));
  }
  return out;
}

// ---------------------------------------------------------------------------------
// Encoding
// ---------------------------------------------------------------------------------
static uint64_t fnv(uint64_t h, const void* p, size_t n) {
  const uint8_t* b = (const uint8_t*)p;
  for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
  return h;
}

// Thread-bit order: the first five (the lane bits) cover as many shared-memory bank
// classes as possible, given the swizzle of the dtype.
std::vector<int> order_thread_bits(const std::vector<int>& tb, int dtype, uint64_t avoid, uint64_t prefer) {
  auto cls = [&](int j) {
    if (dtype == 0) return j == 0 ? 0 : 1 + (j - 1) % 3;
    return j % 3;
  };
  // candidates in preference order: `prefer`, then bits outside `avoid`, then the rest
  std::vector<int> rest;
  for (int j : tb)
    if ((prefer >> j) & 1ull) rest.push_back(j);
  for (int pass = 0; pass < 2; ++pass)
    for (int j : tb)
      if (!((prefer >> j) & 1ull) && ((avoid >> j) & 1ull) == (uint64_t)pass) rest.push_back(j);
  std::vector<int> out;
  std::vector<bool> covered(4, false);
  for (int c = 0; c < 4 && out.size() < 5; ++c) {
    for (size_t i = 0; i < rest.size(); ++i) {
      int kc = cls(rest[i]);
      if (!covered[kc]) {
        covered[kc] = true;
        out.push_back(rest[i]);
        rest.erase(rest.begin() + i);
        break;
      }
    }
  }
  std::sort(out.begin(), out.end());
  while (out.size() < 5 && !rest.empty()) { out.push_back(rest.front()); rest.erase(rest.begin()); }
  for (int j : rest) out.push_back(j);
  return out;
}

Program encode_program(const std::vector<PlannedPass>& passes, const std::vector<COp>& ops, int n,
                       int dtype, int r_req) {
  Program prog;
  std::vector<PassDesc> pd;
  std::vector<PhaseDesc> phd;
  std::vector<GateInstr> gi;
  std::vector<cplx> coef;
  int threads = 32;
  size_t smem = 0;
  const size_t esz = dtype == 0 ? 8 : 16;
  for (const PlannedPass& ps : passes) {
    PassDesc d;
    std::memset(&d, 0, sizeof(d));
    d.m = (int)ps.sbits.size();
    // register bits per thread are fixed by the dtype (the kernel's template parameter);
    // 2^(r - item bits) = 16 load/store items per thread
    const int r = r_req > 0 ? r_req : (dtype == 0 ? 5 : 4);
    if (d.m < r || d.m - r > 9) throw std::runtime_error("encoder: pass size outside the kernel's geometry");
    d.r = r;
    d.phase0 = (int)phd.size();
    d.nphase = (int)ps.phases.size();
    uint64_t S = 0;
    for (int j = 0; j < d.m; ++j) { d.sbit[j] = (int8_t)ps.sbits[j]; S |= bit(ps.sbits[j]); }
    int g = 0;
    for (int p = 0; p < n; ++p) if (!(S & bit(p))) d.gbit[g++] = (int8_t)p;
    d.ngbits = g;
    d.store_perm = ps.store_src.empty() ? 0 : 1;
    for (size_t j = 0; j < ps.store_src.size(); ++j) d.store_src[j] = (int8_t)ps.store_src[j];
    threads = std::max(threads, 1 << (d.m - r));
    smem = std::max(smem, (size_t)2 * (esz << d.m));  // two group buffers (double buffering)
    for (const PlannedPhase& ph : ps.phases) {
      PhaseDesc h;
      std::memset(&h, 0, sizeof(h));
      if ((int)ph.rbits.size() != r) throw std::runtime_error("encoder: register count differs within a pass");
      std::vector<int> tb;
      uint64_t Rl = 0;
      for (int j = 0; j < r; ++j) { h.rbit[j] = (int8_t)ph.rbits[j]; Rl |= bit(ph.rbits[j]); }
      for (int j = 0; j < d.m; ++j) if (!(Rl & bit(j))) tb.push_back(j);
      // controls of controlled gates held by a thread bit: off the lane bits where the bank
      // classes allow (a warp-uniform control costs no per-amplitude select)
      uint64_t avoid = 0;
      for (int oi : ph.ops) {
        const COp& o = ops[oi];
        if (o.kind != GK_2Q_CX && o.kind != GK_2Q_CU) continue;
        for (int j = 0; j < d.m; ++j)
          if (ps.sbits[j] == o.a && !(Rl & bit(j))) avoid |= bit(j);
      }
      // the pass's last phase: lanes over local bits 0-2 (the lowest physical bits), so its
      // registers can be stored to global memory in contiguous 64-byte runs
      const bool last = &ph == &ps.phases.back();
      tb = order_thread_bits(tb, dtype, avoid, last ? 7ull : 0ull);
      for (size_t j = 0; j < tb.size(); ++j) h.tbit[j] = (int8_t)tb[j];
      h.gate0 = (int)gi.size();
      h.ngate = (int)ph.ops.size();
      // physical bit -> register index for this phase
      int reg_of_phys[kMaxQubits];
      for (int p = 0; p < kMaxQubits; ++p) reg_of_phys[p] = -1;
      for (int j = 0; j < r; ++j) reg_of_phys[ps.sbits[ph.rbits[j]]] = j;
      auto opnd = [&](int p) -> uint8_t {
        return reg_of_phys[p] >= 0 ? (uint8_t)reg_of_phys[p] : (uint8_t)(kFixed + p);
      };
      for (int oi : ph.ops) {
        const COp& o = ops[oi];
        GateInstr g2;
        std::memset(&g2, 0, sizeof(g2));
        g2.kind = o.kind;
        g2.a = opnd(o.a);
        g2.b = o.b >= 0 ? opnd(o.b) : 0;
        g2.coef = (int)coef.size();
        for (int c = 0; c < o.ncoef; ++c) coef.push_back(o.coef[c]);
        gi.push_back(g2);
      }
      phd.push_back(h);
    }
    pd.push_back(d);
  }
  ProgramHeader hdr;
  std::memset(&hdr, 0, sizeof(hdr));
  hdr.npass = (int)pd.size();
  hdr.nphase = (int)phd.size();
  hdr.ngate = (int)gi.size();
  hdr.ncoef = (int)coef.size();
  hdr.n = n;
  hdr.dtype = dtype;
  hdr.max_threads = threads;
  auto align16 = [](size_t x) { return (x + 15) & ~size_t(15); };
  size_t off = align16(sizeof(hdr));
  hdr.off_pass = (int)off; off = align16(off + pd.size() * sizeof(PassDesc));
  hdr.off_phase = (int)off; off = align16(off + phd.size() * sizeof(PhaseDesc));
  hdr.off_gate = (int)off; off = align16(off + gi.size() * sizeof(GateInstr));
  hdr.off_coef = (int)off; off = align16(off + coef.size() * esz);
  prog.bytes.assign(off, 0);
  std::memcpy(prog.bytes.data(), &hdr, sizeof(hdr));
  if (!pd.empty()) std::memcpy(prog.bytes.data() + hdr.off_pass, pd.data(), pd.size() * sizeof(PassDesc));
  if (!phd.empty()) std::memcpy(prog.bytes.data() + hdr.off_phase, phd.data(), phd.size() * sizeof(PhaseDesc));
  if (!gi.empty()) std::memcpy(prog.bytes.data() + hdr.off_gate, gi.data(), gi.size() * sizeof(GateInstr));
  uint64_t h = 1469598103934665603ull;
  h = fnv(h, prog.bytes.data(), hdr.off_coef);  // everything except coefficient values
  if (dtype == 0) {
    float* cf = (float*)(prog.bytes.data() + hdr.off_coef);
    for (size_t i = 0; i < coef.size(); ++i) { cf[2 * i] = (float)coef[i].real(); cf[2 * i + 1] = (float)coef[i].imag(); }
  } else {
    double* cf = (double*)(prog.bytes.data() + hdr.off_coef);
    for (size_t i = 0; i < coef.size(); ++i) { cf[2 * i] = coef[i].real(); cf[2 * i + 1] = coef[i].imag(); }
  }
  prog.structure_hash = h;
  prog.has_gates = !gi.empty();
  prog.npass = (int)pd.size();
  prog.threads = threads;
  prog.max_smem = smem;
  return prog;
}

// ---------------------------------------------------------------------------------
// Host interpretation of a program: gate semantics by physical bit, no thread mapping.
// ---------------------------------------------------------------------------------
// A diagonal gate whose bits are all fixed in its phase: the specialised kernels apply it as a
// per-thread factor, at a point of the phase of their choosing (it commutes with the phase).
static bool fixed_diag_instr(const GateInstr& g) {
  return (g.kind == GK_1Q_DIAG && g.a >= kFixed) || (g.kind == GK_2Q_DIAG && g.a >= kFixed && g.b >= kFixed);
}

// gen / term (optional): gradient annotations of a gradient program; psi is then the stacked
// state (bit 0 selects lam) and terms[t] receives Im <lam|G|psi> before gate t's instruction
// (the terms of fixed diagonal gates at the start of their phase, as the kernels take them).
template <typename R>
static void emulate_t(const uint8_t* prog, std::complex<R>* psi, int n, const int8_t* gen = nullptr,
                      const int32_t* term = nullptr, double* terms = nullptr) {
  using C = std::complex<R>;
  const ProgramHeader* hdr = (const ProgramHeader*)prog;
  const PassDesc* pd = (const PassDesc*)(prog + hdr->off_pass);
  const PhaseDesc* phd = (const PhaseDesc*)(prog + hdr->off_phase);
  const GateInstr* gi = (const GateInstr*)(prog + hdr->off_gate);
  const C* cf = (const C*)(prog + hdr->off_coef);
  const uint64_t dim = 1ull << n;
  std::vector<C> tmp;
  // Im sum_x conj(lam(x)) (G psi)(x), G on physical bit pb (psi at even, lam at odd indices)
  auto grad_term = [&](int pb, int g) {
    const uint64_t mp = 1ull << pb;
    double s = 0.0;
    for (uint64_t i = 0; i < dim; i += 2) {
      const std::complex<double> l(psi[i | 1].real(), psi[i | 1].imag());
      std::complex<double> v;
      if (g == 3) {
        v = std::complex<double>(psi[i].real(), psi[i].imag());
        if (i & mp) v = -v;
      } else {
        const std::complex<double> o(psi[i ^ mp].real(), psi[i ^ mp].imag());
        v = g == 1 ? o : ((i & mp) ? std::complex<double>(0, 1) * o : std::complex<double>(0, -1) * o);
      }
      s += std::imag(std::conj(l) * v);
    }
    return s;
  };
  for (int p = 0; p < hdr->npass; ++p) {
    const PassDesc& d = pd[p];
    for (int h = 0; h < d.nphase; ++h) {
      const PhaseDesc& ph = phd[d.phase0 + h];
      auto phys = [&](uint8_t o) -> int { return o >= kFixed ? o - kFixed : d.sbit[ph.rbit[o]]; };
      if (gen)
        for (int g = 0; g < ph.ngate; ++g) {
          const int k = ph.gate0 + g;
          if (gen[k] && fixed_diag_instr(gi[k])) terms[term[k]] = grad_term(phys(gi[k].a), gen[k]);
        }
      for (int g = 0; g < ph.ngate; ++g) {
        const GateInstr& G = gi[ph.gate0 + g];
        if (gen && gen[ph.gate0 + g] && !fixed_diag_instr(G))
          terms[term[ph.gate0 + g]] = grad_term(phys(G.a), gen[ph.gate0 + g]);
        const C* c = cf + G.coef;
        const int a = phys(G.a);
        const uint64_t ma = 1ull << a;
        switch (G.kind) {
          case GK_1Q_DENSE: case GK_1Q_REAL: case GK_1Q_REIM:
            for (uint64_t i = 0; i < dim; ++i) if (!(i & ma)) {
              C x0 = psi[i], x1 = psi[i | ma];
              psi[i] = c[0] * x0 + c[1] * x1; psi[i | ma] = c[2] * x0 + c[3] * x1;
            }
            break;
          case GK_1Q_DIAG:
            for (uint64_t i = 0; i < dim; ++i) psi[i] *= (i & ma) ? c[1] : c[0];
            break;
          case GK_1Q_X:
            for (uint64_t i = 0; i < dim; ++i) if (!(i & ma)) std::swap(psi[i], psi[i | ma]);
            break;
          default: {
            const int b = phys(G.b);
            const uint64_t mb = 1ull << b;
            if (G.kind == GK_2Q_DIAG) {
              for (uint64_t i = 0; i < dim; ++i) psi[i] *= c[((i & ma) ? 1 : 0) + ((i & mb) ? 2 : 0)];
            } else if (G.kind == GK_2Q_CX) {
              for (uint64_t i = 0; i < dim; ++i) if ((i & ma) && !(i & mb)) std::swap(psi[i], psi[i | mb]);
            } else if (G.kind == GK_2Q_CU) {
              for (uint64_t i = 0; i < dim; ++i) if ((i & ma) && !(i & mb)) {
                C x0 = psi[i], x1 = psi[i | mb];
                psi[i] = c[0] * x0 + c[1] * x1; psi[i | mb] = c[2] * x0 + c[3] * x1;
              }
            } else if (G.kind == GK_2Q_SWAP) {
              for (uint64_t i = 0; i < dim; ++i) if ((i & ma) && !(i & mb)) std::swap(psi[i], psi[(i ^ ma) | mb]);
            } else if (G.kind == GK_2Q_DENSE) {
              for (uint64_t i = 0; i < dim; ++i) if (!(i & ma) && !(i & mb)) {
                const uint64_t idx[4] = {i, i | ma, i | mb, i | ma | mb};
                C x[4] = {psi[idx[0]], psi[idx[1]], psi[idx[2]], psi[idx[3]]};
                for (int rr = 0; rr < 4; ++rr)
                  psi[idx[rr]] = c[4 * rr] * x[0] + c[4 * rr + 1] * x[1] + c[4 * rr + 2] * x[2] + c[4 * rr + 3] * x[3];
              }
            } else {
              throw std::runtime_error("emulator: unknown gate kind");
            }
          }
        }
      }
    }
    if (d.store_perm) {
      tmp.assign(psi, psi + dim);
      // output local bit j takes input local bit store_src[j]
      for (uint64_t i = 0; i < dim; ++i) {
        uint64_t o = i;
        for (int j = 0; j < d.m; ++j) o &= ~(1ull << d.sbit[j]);
        for (int j = 0; j < d.m; ++j)
          if (i & (1ull << d.sbit[d.store_src[j]])) o |= 1ull << d.sbit[j];
        psi[o] = tmp[i];
      }
    }
  }
}

void emulate_program(const uint8_t* prog, void* state, int n, int dtype) {
  if (dtype == 0) emulate_t<float>(prog, (std::complex<float>*)state, n);
  else emulate_t<double>(prog, (std::complex<double>*)state, n);
}

}  // namespace qsb

// ---------------------------------------------------------------------------------
// Adjoint gradient: the reverse sweep as one program over the stacked state
// ---------------------------------------------------------------------------------
namespace qsb {

namespace {

// The circuit's gates as U^dagger in reverse order, at physical bits q + 1.
std::vector<QOp> reverse_ops(const std::vector<GradOp>& fwd) {
  std::vector<QOp> r;
  r.reserve(fwd.size());
  for (size_t k = fwd.size(); k-- > 0;) {
    const QOp& o = fwd[k].op;
    QOp d;
    d.arity = o.arity;
    d.q0 = o.q0 + 1;
    d.q1 = o.arity == 2 ? o.q1 + 1 : -1;
    const int dd = o.arity == 1 ? 2 : 4;
    for (int i = 0; i < dd; ++i)
      for (int j = 0; j < dd; ++j) d.U[i * dd + j] = std::conj(o.U[j * dd + i]);
    r.push_back(d);
  }
  return r;
}

// Classes of the reverse gates.  A parameterised X or Y rotation stays a register gate even
// where its matrix is diagonal (theta = 0): its gradient term pairs amplitudes across its bit.
std::vector<COp> classify_grad(const std::vector<QOp>& rev, const std::vector<GradOp>& fwd) {
  std::vector<COp> c;
  c.reserve(rev.size());
  const size_t N = fwd.size();
  for (size_t i = 0; i < N; ++i) {
    COp o = classify(rev[i]);
    const int g = fwd[N - 1 - i].gen;
    if (g == 1 || g == 2) o.need |= bit(rev[i].q0);
    c.push_back(o);
  }
  return c;
}

PlanConfig grad_cfg(const PlanConfig& cfg) {
  PlanConfig pc = cfg;
  pc.pair_bit = true;  // the lam bit is a register bit of every phase
  return pc;
}

}  // namespace

uint64_t grad_signature(const std::vector<GradOp>& fwd, int n, const PlanConfig& cfg) {
  const std::vector<COp> c = classify_grad(reverse_ops(fwd), fwd);
  uint64_t h = 1469598103934665603ull;
  auto mix = [&h](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
  mix((uint64_t)n); mix((uint64_t)cfg.m); mix((uint64_t)cfg.r); mix((uint64_t)cfg.k);
  mix((uint64_t)cfg.hill_iters); mix((uint64_t)cfg.lookahead);
  for (const COp& o : c) {
    mix(((uint64_t)o.kind << 16) | ((uint64_t)(o.a & 0xff) << 8) | (uint64_t)(o.b & 0xff));
    mix(o.need);
  }
  for (const GradOp& g : fwd) mix((uint64_t)g.gen);
  return h;
}

std::vector<PlannedPass> plan_grad_passes(const std::vector<GradOp>& fwd, int n, const PlanConfig& cfg,
                                          uint64_t* signature) {
  const std::vector<COp> c = classify_grad(reverse_ops(fwd), fwd);
  std::vector<PlannedPass> passes = plan_passes(c, n + 1, grad_cfg(cfg));
  for (const PlannedPass& ps : passes) {
    if (ps.sbits.empty() || ps.sbits[0] != 0 || !ps.store_src.empty())
      throw std::runtime_error("gradient planner: a pass does not stage the lam bit");
    for (const PlannedPhase& ph : ps.phases)
      if (std::find(ph.rbits.begin(), ph.rbits.end(), 0) == ph.rbits.end())
        throw std::runtime_error("gradient planner: a phase does not hold the lam bit in registers");
  }
  if (signature) *signature = grad_signature(fwd, n, cfg);
  return passes;
}

bool grad_plan_fits(const std::vector<GradOp>& fwd, const std::vector<PlannedPass>& passes) {
  const std::vector<COp> c = classify_grad(reverse_ops(fwd), fwd);
  size_t seen = 0;
  for (const PlannedPass& ps : passes)
    for (const PlannedPhase& ph : ps.phases) {
      uint64_t R = 0;
      for (int j : ph.rbits) R |= bit(ps.sbits[j]);
      for (int oi : ph.ops) {
        if (oi < 0 || (size_t)oi >= c.size() || (c[oi].need & ~R)) return false;
        ++seen;
      }
    }
  return seen == c.size();
}

GradProgram build_grad_program(const std::vector<GradOp>& fwd, int n, const std::vector<PlannedPass>& passes,
                               int r) {
  std::vector<QOp> rev = reverse_ops(fwd);
  const std::vector<QOp> orig = rev;
  // scalar extraction with unit-modulus diagonals: the per-thread factors of diagonal gates
  // on fixed bits (applied wherever the kernel places them in their phase) leave magnitudes
  // alone, so a term's weight only depends on the register gates before it
  for (const PlannedPass& ps : passes) extract_pass_scalars(rev, ps.ops, false);
  const std::vector<COp> c = classify_grad(rev, fwd);
  GradProgram g;
  g.prog = encode_program(passes, c, n + 1, 0, r);
  const size_t N = fwd.size();
  // squared magnitude of the scalar each gate's rewrite took out
  std::vector<double> r2(N, 1.0);
  for (size_t i = 0; i < N; ++i) {
    const int d = rev[i].arity == 1 ? 2 : 4;
    int e = 0;
    for (int k = 1; k < d * d; ++k)
      if (std::abs(rev[i].U[k]) > std::abs(rev[i].U[e])) e = k;
    if (std::abs(rev[i].U[e]) > 0.0) r2[i] = std::norm(orig[i].U[e]) / std::norm(rev[i].U[e]);
  }
  const ProgramHeader* hdr = (const ProgramHeader*)g.prog.bytes.data();
  const GateInstr* gi = (const GateInstr*)(g.prog.bytes.data() + hdr->off_gate);
  g.prog.grad_gen.assign(hdr->ngate, 0);
  g.prog.grad_term.assign(hdr->ngate, -1);
  double f2 = 1.0;  // |actual / carried|^2 of both halves before the current instruction
  int k = 0;
  for (const PlannedPass& ps : passes)
    for (const PlannedPhase& ph : ps.phases) {
      const double start = f2;
      for (int oi : ph.ops) {
        const GradOp& src = fwd[N - 1 - (size_t)oi];
        const bool hoisted = fixed_diag_instr(gi[k]);
        if (hoisted && std::abs(r2[oi] - 1.0) > 1e-9)
          throw std::runtime_error("gradient program: a diagonal gate on fixed bits rescales the state");
        if (src.gen) {
          if (src.op.arity != 1) throw std::runtime_error("gradient program: parameterised gates are single-qubit");
          g.prog.grad_gen[k] = (int8_t)src.gen;
          g.prog.grad_term[k] = g.prog.nterm++;
          g.term_slot.push_back(src.slot);
          g.term_w.push_back(hoisted ? start : f2);
        }
        f2 *= r2[oi];
        ++k;
      }
    }
  if (k != hdr->ngate) throw std::runtime_error("gradient program: instruction count mismatch");
  return g;
}

void emulate_grad_program(const GradProgram& g, void* phi, double* terms) {
  const ProgramHeader* hdr = (const ProgramHeader*)g.prog.bytes.data();
  emulate_t<float>(g.prog.bytes.data(), (std::complex<float>*)phi, hdr->n, g.prog.grad_gen.data(),
                   g.prog.grad_term.data(), terms);
}

}  // namespace qsb
