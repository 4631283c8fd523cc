// Batched variational workload: host planning, encoding, execution and CPU emulation
// (device program layout: batch.h; kernel: kern_batch.cu).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/qsim_b200.h"
#include "batch.h"
#include "kernels.h"
#include "plan.h"

using namespace qsb;

namespace {

struct BErr {
  std::string msg;
  int code;
};
#define BCK(call)                                                                          \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) throw BErr{std::string("CUDA error: ") + cudaGetErrorString(_e), QS_ERR_CUDA}; \
  } while (0)

template <typename F>
int bguard(F&& f) {
  try {
    f();
    return 0;
  } catch (const BErr& e) {
    set_last_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return QS_ERR_INVALID;
  }
}

[[noreturn]] void bad(const std::string& m) { throw BErr{m, QS_ERR_INVALID}; }

constexpr uint64_t kBatchWaitNs = 10ull * 1000ull * 1000ull * 1000ull;  // 10 s per dependency wait

struct Cfg {
  int m = 13, small_max = 13, chunk = 4, threads = 256, bps = 0;
  uint64_t wait_ns = kBatchWaitNs;
};

Cfg cfg_of(const qs_batch_config* c) {
  Cfg k;
  if (c) {
    k.m = c->m; k.small_max = c->small_max; k.chunk = c->chunk; k.threads = c->threads; k.bps = c->blocks_per_sm;
    if (c->wait_limit_ns) k.wait_ns = c->wait_limit_ns;
  }
  if (k.m < 9 || k.m > kBatchMaxLocal) bad("batch: m must be in 9..13");
  if (k.small_max < 0 || k.small_max > kBatchMaxLocal) bad("batch: small_max must be in 0..13");
  if (k.chunk < 1) bad("batch: chunk must be >= 1");
  if (k.threads != 256 && k.threads != 512) bad("batch: threads must be 256 or 512");
  if (k.bps < 0 || k.bps > 8) bad("batch: blocks_per_sm must be in 0..8");
  return k;
}

// Gate of an instance, as given (forward matrix in complex128).
struct IGate {
  QOp op;
  int gen = 0, grad = 0;
};

struct Inst {
  int n = 0, nparam = 0;
  std::vector<IGate> gates;
  std::vector<double> a, b;
};

std::vector<Inst> read_instances(const qs_batch_instance* insts, int ninst) {
  if (!insts || ninst < 1) bad("batch: no instances");
  std::vector<Inst> out(ninst);
  for (int i = 0; i < ninst; ++i) {
    const qs_batch_instance& s = insts[i];
    Inst& d = out[i];
    d.n = s.num_qubits;
    if (d.n < 2 || d.n > kBatchMaxQubits) bad("batch: instance " + std::to_string(i) + ": num_qubits must be in 2..26");
    if (s.nparams < 0) bad("batch: nparams < 0");
    if (s.nops < 0 || (s.nops > 0 && !s.ops)) bad("batch: null ops");
    if (!s.a || !s.b) bad("batch: null observable coefficients");
    d.nparam = s.nparams;
    d.a.assign(s.a, s.a + d.n);
    d.b.assign(s.b, s.b + d.n);
    for (int k = 0; k < s.nops; ++k) {
      const qs_adj_op& o = s.ops[k];
      IGate g;
      if (!o.U) bad("batch: null gate matrix");
      if (o.kind == QS_OP_1Q) {
        if (o.q0 < 0 || o.q0 >= d.n) bad("batch: invalid q0");
        g.op.arity = 1;
        g.op.q0 = o.q0;
        for (int e = 0; e < 4; ++e) g.op.U[e] = cplx(o.U[2 * e], o.U[2 * e + 1]);
      } else if (o.kind == QS_OP_2Q) {
        if (o.q0 < 0 || o.q0 >= d.n || o.q1 < 0 || o.q1 >= d.n) bad("batch: invalid q0/q1");
        if (o.q0 == o.q1) bad("batch: q0 == q1");
        g.op.arity = 2;
        g.op.q0 = o.q0;
        g.op.q1 = o.q1;
        for (int e = 0; e < 16; ++e) g.op.U[e] = cplx(o.U[2 * e], o.U[2 * e + 1]);
      } else {
        bad("batch: unknown op kind " + std::to_string(o.kind));
      }
      if (o.gen < 0 || o.gen > 3) bad("batch: gen must be 0..3");
      if (o.gen) {
        if (o.kind != QS_OP_1Q) bad("batch: parameterised gates must be single-qubit rotations");
        if (o.grad_index < 0 || o.grad_index >= d.nparam) bad("batch: grad_index out of range");
        g.gen = o.gen;
        g.grad = o.grad_index;
      }
      d.gates.push_back(g);
    }
  }
  return out;
}

// A single-qubit gate applied as a diagonal (its qubit need not be staged): diagonal, and
// not the rotation of an X or Y generator (whose gradient needs the pairs).
bool diag1(const IGate& ig) {
  return ig.op.arity == 1 && classify(ig.op).kind == GK_1Q_DIAG && (ig.gen == 0 || ig.gen == 3);
}

BatchGate encode_gate(const IGate& ig) {
  BatchGate g;
  std::memset(&g, 0, sizeof(g));
  const COp c = classify(ig.op);
  g.q0 = (uint8_t)ig.op.q0;
  g.q1 = (uint8_t)(ig.op.arity == 2 ? ig.op.q1 : 0);
  g.gen = (uint8_t)ig.gen;
  g.grad = ig.gen ? ig.grad : 0;
  auto f2 = [](cplx z) { return float2{(float)z.real(), (float)z.imag()}; };
  // A diagonal unitary is stored divided by its first entry (a phase): the states then carry a
  // phase common to psi and lam, which cancels in the energy <psi|H psi> and in every term
  // Im <lam|G|psi>; the kernel skips the multiplies by the exact 1 this leaves.
  auto unit_first = [](cplx* d, int k) {
    const cplx d0 = d[0];
    if (std::abs(std::abs(d0) - 1.0) > 1e-9) return;
    for (int e = 0; e < k; ++e) d[e] /= d0;
    d[0] = cplx(1.0, 0.0);
  };
  if (ig.op.arity == 1) {
    if (diag1(ig)) {
      g.kind = BG_DIAG1;
      cplx d[2] = {ig.op.U[0], ig.op.U[3]};
      unit_first(d, 2);
      g.u[0] = f2(d[0]);
      g.u[1] = f2(d[1]);
    } else {
      g.kind = BG_1Q;
      for (int e = 0; e < 4; ++e) g.u[e] = f2(ig.op.U[e]);
    }
  } else if (c.kind == GK_2Q_DIAG) {
    g.kind = BG_DIAG2;
    cplx d[4] = {ig.op.U[0], ig.op.U[5], ig.op.U[10], ig.op.U[15]};
    unit_first(d, 4);
    for (int e = 0; e < 4; ++e) g.u[e] = f2(d[e]);
  } else {
    g.kind = BG_2Q;
    for (int e = 0; e < 16; ++e) g.u[e] = f2(ig.op.U[e]);
  }
  return g;
}

// Staging requirement of a gate in the batch kernel (bits that must be local).
uint64_t need_of(const IGate& ig) {
  const COp c = classify(ig.op);
  if (ig.op.arity == 1) return diag1(ig) ? 0ull : (1ull << ig.op.q0);
  if (c.kind == GK_2Q_DIAG) return 0ull;
  // controlled gates may keep the control fixed (block-diagonal in it): the planner's need
  return c.need;
}

struct Encoded {
  std::vector<uint8_t> bytes;
  int nitem = 0, nparam_total = 0, mbuf = 0;
  size_t arena_amps = 0;
  std::vector<int> grad0;   // per instance
};

// plans: optional per-instance cache (structure signature, planned passes)
using PlanCache = std::vector<std::pair<uint64_t, std::vector<PlannedPass>>>;

Encoded encode_batch(const std::vector<Inst>& insts, const Cfg& cfg, PlanCache* plans = nullptr) {
  const int ninst = (int)insts.size();
  std::vector<BatchInst> bi(ninst);
  std::vector<BatchPass> bp;
  std::vector<BatchGate> bg;
  std::vector<double> coef;
  Encoded E;
  E.grad0.resize(ninst);
  std::vector<BatchPhase> bph;
  // per instance: stage list (kind, pass, items)
  struct Stage { int kind, pass, nitems; };
  std::vector<std::vector<Stage>> stages(ninst);

  // Passes of instance i with m staged bits and kBatchRegBits register bits per phase.  Plans
  // depend on the gates' staging requirements and commutation (touch masks), not on matrix
  // values: the cached plan of the same structure is reused (parameter updates).
  auto plan_instance = [&](const Inst& in, int i, int m, PlanCache* cache) {
    std::vector<COp> cops;
    for (const IGate& g : in.gates) {
      COp c = classify(g.op);
      c.need = need_of(g);
      cops.push_back(c);
    }
    PlanConfig pc;
    pc.m = m;
    pc.r = std::min(kBatchRegBits, m);
    pc.k = std::min(3, m);
    pc.lookahead = 0;  // many small instances: planning time matters more than a sweep or two
    pc.phase_lookahead = 0;
    uint64_t sig = 1469598103934665603ull ^ (uint64_t)m;
    for (const COp& c : cops) {
      const uint64_t w[3] = {c.need, c.touch, (uint64_t)c.kind};
      for (uint64_t v : w) { sig ^= v; sig *= 1099511628211ull; }
    }
    if (cache && (size_t)i < cache->size() && (*cache)[i].first == sig) return (*cache)[i].second;
    std::vector<PlannedPass> passes = plan_passes(cops, in.n, pc);
    if (cache) {
      if (cache->size() <= (size_t)i) cache->resize(i + 1);
      (*cache)[i] = {sig, passes};
    }
    return passes;
  };

  // Encode one pass: its gates in phase order, and its register phases unless a gate cannot
  // run in registers there (then the kernel runs the pass gate by gate in shared memory).
  auto emit_pass = [&](const PlannedPass& ps, const Inst& in) {
    BatchPass p;
    std::memset(&p, 0, sizeof(p));
    p.m = (int)ps.sbits.size();
    p.gate0 = (int)bg.size();
    uint64_t S = 0;
    int8_t loc[kBatchMaxQubits];
    for (int q = 0; q < kBatchMaxQubits; ++q) loc[q] = -1;
    for (int j = 0; j < p.m; ++j) {
      p.sbit[j] = (int8_t)ps.sbits[j];
      S |= 1ull << ps.sbits[j];
      loc[ps.sbits[j]] = (int8_t)j;
    }
    int gj = 0;
    for (int q = 0; q < in.n; ++q) if (!(S >> q & 1ull)) p.gbit[gj++] = (int8_t)q;
    const int nr = std::min(kBatchRegBits, p.m);
    bool regs = (int)ps.phases.size() <= kBatchMaxPhases && p.m - nr <= kBatchMaxLocal;
    std::vector<BatchPhase> mine;
    int count = 0;
    for (const PlannedPhase& ph : ps.phases) {
      BatchPhase h;
      std::memset(&h, 0, sizeof(h));
      h.nr = (int8_t)nr;
      if ((int)ph.rbits.size() != nr) regs = false;
      uint32_t R = 0;
      for (int j = 0; j < (int)ph.rbits.size() && j < kBatchRegBits; ++j) {
        h.rbit[j] = (int8_t)ph.rbits[j];
        R |= 1u << ph.rbits[j];
      }
      std::vector<int> tb;
      for (int j = 0; j < p.m; ++j) if (!(R >> j & 1u)) tb.push_back(j);
      tb = order_thread_bits(tb, 0);
      for (size_t j = 0; j < tb.size(); ++j) h.tbit[j] = (int8_t)tb[j];
      h.gate0 = (int)bg.size();
      h.ngate = (int)ph.ops.size();
      auto reg = [&](int q) { return loc[q] >= 0 && (R >> loc[q] & 1u); };
      for (int oi : ph.ops) {
        const BatchGate g = encode_gate(in.gates[oi]);
        // register path: 1q on a register bit; 2q with exactly one register operand (the
        // other fixed: controlled gates); diagonals anywhere
        if (g.kind == BG_1Q && !reg(g.q0)) regs = false;
        if (g.kind == BG_2Q && (reg(g.q0) == reg(g.q1))) regs = false;
        bg.push_back(g);
        ++count;
      }
      mine.push_back(h);
    }
    p.ngate = count;
    if (ps.phases.empty()) {  // (no phases planned: gates in pass order)
      for (int oi : ps.ops) bg.push_back(encode_gate(in.gates[oi]));
      p.ngate = (int)ps.ops.size();
      regs = false;
    }
    if (regs) {
      p.phase0 = (int)bph.size();
      p.nphase = (int)mine.size();
      bph.insert(bph.end(), mine.begin(), mine.end());
    }
    bp.push_back(p);
  };
  size_t arena = 0;
  int grad = 0;
  for (int i = 0; i < ninst; ++i) {
    const Inst& in = insts[i];
    BatchInst& b = bi[i];
    std::memset(&b, 0, sizeof(b));
    b.n = in.n;
    b.nparam = in.nparam;
    b.grad0 = grad;
    E.grad0[i] = grad;
    grad += in.nparam;
    b.coef0 = (int)coef.size();
    coef.insert(coef.end(), in.a.begin(), in.a.end());
    coef.insert(coef.end(), in.b.begin(), in.b.end());
    b.pass0 = (int)bp.size();
    b.m = in.n <= cfg.small_max ? in.n : std::min(cfg.m, in.n);
    if (in.n <= cfg.small_max) {
      // all qubits staged: one pass (its register phases planned like any other pass)
      std::vector<PlannedPass> one = plan_instance(in, i, in.n, plans);
      if (one.size() == 1 && (int)one[0].sbits.size() == in.n) {
        emit_pass(one[0], in);
      } else {
        BatchPass p;
        std::memset(&p, 0, sizeof(p));
        p.m = in.n;
        p.gate0 = (int)bg.size();
        p.ngate = (int)in.gates.size();
        for (int j = 0; j < in.n; ++j) p.sbit[j] = (int8_t)j;
        for (const IGate& g : in.gates) bg.push_back(encode_gate(g));
        bp.push_back(p);
      }
      b.npass = 1;
      b.psi = b.lam = -1;
      stages[i].push_back({BI_SMALL, 0, 1});
      continue;
    }
    const int m = std::min(cfg.m, in.n);
    if (in.n - m > 14) bad("batch: instance of " + std::to_string(in.n) + " qubits needs m >= " + std::to_string(in.n - 14));
    std::vector<PlannedPass> passes = plan_instance(in, i, m, plans);
    for (const PlannedPass& ps : passes) {
      if ((int)ps.sbits.size() != m || ps.sbits[0] != 0) bad("batch: planner returned an unexpected staged set");
      emit_pass(ps, in);
    }
    b.npass = (int)passes.size();
    arena = (arena + 1) & ~size_t(1);  // 16-byte aligned states
    b.psi = (int64_t)arena;
    arena += size_t(1) << in.n;
    b.lam = (int64_t)arena;
    arena += size_t(1) << in.n;
    const int groups = 1 << (in.n - m);
    const int items = (groups + cfg.chunk - 1) / cfg.chunk;
    for (int p = 0; p < b.npass; ++p) stages[i].push_back({BI_FWD, p, items});
    stages[i].push_back({BI_HAM, 0, items});
    for (int p = b.npass - 1; p >= 0; --p) stages[i].push_back({BI_BWD, p, items});
  }
  // work items: stage-major across the arena instances, then the shared-memory instances
  std::vector<BatchItem> items;
  size_t max_st = 0;
  for (auto& s : stages) max_st = std::max(max_st, s.size());
  std::vector<int> done_before(ninst, 0);
  auto emit = [&](int i, const Stage& st) {
    const int n = insts[i].n;
    const int m = std::min(cfg.m, n);
    const int units = st.kind == BI_SMALL ? 1 : 1 << (n - m);
    for (int k = 0; k < st.nitems; ++k) {
      BatchItem it;
      it.inst = i;
      it.kind = st.kind;
      it.pass = st.pass;
      it.first = k * cfg.chunk;
      it.count = std::min(cfg.chunk, units - it.first);
      if (st.kind == BI_SMALL) { it.first = 0; it.count = 1; }
      it.need = done_before[i];
      items.push_back(it);
    }
    done_before[i] += st.nitems;
  };
  for (size_t s = 0; s < max_st; ++s)
    for (int i = 0; i < ninst; ++i)
      if (stages[i].size() > s && stages[i][s].kind != BI_SMALL) emit(i, stages[i][s]);
  for (int i = 0; i < ninst; ++i)
    if (stages[i][0].kind == BI_SMALL) emit(i, stages[i][0]);

  BatchHeader h;
  std::memset(&h, 0, sizeof(h));
  h.ninst = ninst;
  h.npass = (int)bp.size();
  h.ngate = (int)bg.size();
  h.nitem = (int)items.size();
  h.ncoef = (int)coef.size();
  h.m = cfg.m;
  h.small_max = cfg.small_max;
  int mbuf = 1;
  for (const Inst& in : insts) mbuf = std::max(mbuf, in.n <= cfg.small_max ? in.n : std::min(cfg.m, in.n));
  h.mbuf = mbuf;
  auto align = [](size_t x) { return (x + 15) & ~size_t(15); };
  size_t off = align(sizeof(h));
  h.off_inst = (int)off; off = align(off + bi.size() * sizeof(BatchInst));
  h.off_pass = (int)off; off = align(off + bp.size() * sizeof(BatchPass));
  h.off_gate = (int)off; off = align(off + bg.size() * sizeof(BatchGate));
  h.off_item = (int)off; off = align(off + items.size() * sizeof(BatchItem));
  h.off_coef = (int)off; off = align(off + coef.size() * sizeof(double));
  h.nphase = (int)bph.size();
  h.off_phase = (int)off; off = align(off + bph.size() * sizeof(BatchPhase));
  E.bytes.assign(off, 0);
  if (!bph.empty()) std::memcpy(E.bytes.data() + h.off_phase, bph.data(), bph.size() * sizeof(BatchPhase));
  std::memcpy(E.bytes.data(), &h, sizeof(h));
  std::memcpy(E.bytes.data() + h.off_inst, bi.data(), bi.size() * sizeof(BatchInst));
  std::memcpy(E.bytes.data() + h.off_pass, bp.data(), bp.size() * sizeof(BatchPass));
  std::memcpy(E.bytes.data() + h.off_gate, bg.data(), bg.size() * sizeof(BatchGate));
  std::memcpy(E.bytes.data() + h.off_item, items.data(), items.size() * sizeof(BatchItem));
  std::memcpy(E.bytes.data() + h.off_coef, coef.data(), coef.size() * sizeof(double));
  E.nitem = h.nitem;
  E.nparam_total = grad;
  E.mbuf = mbuf;
  E.arena_amps = arena;
  return E;
}

// ---- host emulation of the device program (same items, same order, FP64 states) ------
using cd = std::complex<double>;
cd c2(float2 v) { return cd(v.x, v.y); }

struct Emu {
  const uint8_t* b;
  const BatchHeader* h;
  std::vector<cd> arena;
  std::vector<double> grads, energy;

  static int qbit(const int8_t* loc, int q, uint32_t x, uint64_t gb) {
    return loc[q] >= 0 ? (int)((x >> loc[q]) & 1u) : (int)((gb >> q) & 1ull);
  }
  static void pairs(cd m0, cd m1, cd m2, cd m3, int gen, bool rev, cd* A, cd* L, int m, int j, double& acc) {
    for (uint32_t i0 = 0; i0 < (1u << m); ++i0) {
      if (i0 >> j & 1u) continue;
      const uint32_t i1 = i0 | (1u << j);
      const cd p0 = A[i0], p1 = A[i1];
      A[i0] = m0 * p0 + m1 * p1;
      A[i1] = m2 * p0 + m3 * p1;
      if (rev) {
        const cd l0 = L[i0], l1 = L[i1];
        cd g0 = 0, g1 = 0;
        if (gen == 1) { g0 = p1; g1 = p0; }
        else if (gen == 2) { g0 = cd(0, -1) * p1; g1 = cd(0, 1) * p0; }
        else if (gen == 3) { g0 = p0; g1 = -p1; }
        acc += std::imag(std::conj(l0) * g0 + std::conj(l1) * g1);
        L[i0] = m0 * l0 + m1 * l1;
        L[i1] = m2 * l0 + m3 * l1;
      }
    }
  }
  void gate(const BatchGate& g, bool rev, cd* A, cd* L, int m, uint64_t gb, const int8_t* loc, double* gslot) {
    double acc = 0;
    auto M = [&](int r, int c, int d) { return rev ? std::conj(c2(g.u[d * c + r])) : c2(g.u[d * r + c]); };
    if (g.kind == BG_1Q) {
      pairs(M(0, 0, 2), M(0, 1, 2), M(1, 0, 2), M(1, 1, 2), g.gen, rev, A, L, m, loc[g.q0], acc);
    } else if (g.kind == BG_DIAG1 || g.kind == BG_DIAG2) {
      for (uint32_t x = 0; x < (1u << m); ++x) {
        const int b0 = qbit(loc, g.q0, x, gb);
        const int v = g.kind == BG_DIAG2 ? b0 + 2 * qbit(loc, g.q1, x, gb) : b0;
        const cd d = rev ? std::conj(c2(g.u[v])) : c2(g.u[v]);
        if (rev && g.gen == 3) acc += (b0 ? -1.0 : 1.0) * std::imag(std::conj(L[x]) * A[x]);
        A[x] *= d;
        if (rev) L[x] *= d;
      }
    } else {
      const int j0 = loc[g.q0], j1 = loc[g.q1];
      if (j0 >= 0 && j1 >= 0) {
        for (uint32_t base = 0; base < (1u << m); ++base) {
          if ((base >> j0 & 1u) || (base >> j1 & 1u)) continue;
          const uint32_t idx[4] = {base, base | (1u << j0), base | (1u << j1), base | (1u << j0) | (1u << j1)};
          cd x[4], y[4];
          for (int c = 0; c < 4; ++c) { x[c] = A[idx[c]]; y[c] = L ? L[idx[c]] : cd(); }
          for (int r = 0; r < 4; ++r) {
            cd s = 0, t = 0;
            for (int c = 0; c < 4; ++c) { s += M(r, c, 4) * x[c]; t += M(r, c, 4) * y[c]; }
            A[idx[r]] = s;
            if (rev) L[idx[r]] = t;
          }
        }
      } else if (j1 >= 0) {
        const int f = (int)((gb >> g.q0) & 1ull);
        pairs(M(f, f, 4), M(f, f + 2, 4), M(f + 2, f, 4), M(f + 2, f + 2, 4), 0, rev, A, L, m, j1, acc);
      } else if (j0 >= 0) {
        const int f = (int)((gb >> g.q1) & 1ull);
        pairs(M(2 * f, 2 * f, 4), M(2 * f, 2 * f + 1, 4), M(2 * f + 1, 2 * f, 4), M(2 * f + 1, 2 * f + 1, 4), 0, rev,
              A, L, m, j0, acc);
      }
    }
    if (rev && g.gen) *gslot += acc;
  }
  static double ham(const cd* psi, cd* lam, int n, uint64_t x0, uint64_t x1, const double* a, const double* b) {
    double e = 0;
    for (uint64_t x = x0; x < x1; ++x) {
      double d = 0;
      for (int i = 0; i < n; ++i) {
        const int j = i + 1 == n ? 0 : i + 1;
        d += (((x >> i) ^ (x >> j)) & 1ull) ? -a[i] : a[i];
      }
      cd v = d * psi[x];
      for (int i = 0; i < n; ++i) v += b[i] * psi[x ^ (1ull << i)];
      lam[x] = v;
      e += std::real(std::conj(psi[x]) * v);
    }
    return e;
  }

  void run() {
    h = (const BatchHeader*)b;
    const BatchInst* insts = (const BatchInst*)(b + h->off_inst);
    const BatchPass* passes = (const BatchPass*)(b + h->off_pass);
    const BatchGate* gates = (const BatchGate*)(b + h->off_gate);
    const BatchItem* items = (const BatchItem*)(b + h->off_item);
    const double* coef = (const double*)(b + h->off_coef);
    std::vector<int> done(h->ninst, 0);
    std::vector<cd> A(size_t(1) << h->mbuf), L(size_t(1) << h->mbuf);
    for (int k = 0; k < h->nitem; ++k) {
      const BatchItem& it = items[k];
      if (done[it.inst] < it.need) throw std::runtime_error("batch emulation: item order violates a dependency");
      const BatchInst& in = insts[it.inst];
      const int n = in.n;
      const double* a = coef + in.coef0;
      const double* bb = a + n;
      double* gout = grads.data() + in.grad0;
      if (it.kind == BI_HAM) {
        const uint64_t chunk = 1ull << in.m;
        energy[it.inst] += ham(arena.data() + in.psi, arena.data() + in.lam, n, it.first * chunk,
                               (uint64_t)(it.first + it.count) * chunk, a, bb);
      } else {
        const BatchPass& ps = passes[in.pass0 + it.pass];
        int8_t loc[kBatchMaxQubits];
        for (int q = 0; q < kBatchMaxQubits; ++q) loc[q] = -1;
        for (int j = 0; j < ps.m; ++j) loc[ps.sbit[j]] = (int8_t)j;
        const BatchGate* gs = gates + ps.gate0;
        if (it.kind == BI_SMALL) {
          std::fill(A.begin(), A.end(), cd(0));
          A[0] = 1;
          for (int g = 0; g < ps.ngate; ++g) gate(gs[g], false, A.data(), L.data(), n, 0, loc, nullptr);
          energy[it.inst] += ham(A.data(), L.data(), n, 0, 1ull << n, a, bb);
          for (int g = ps.ngate - 1; g >= 0; --g) gate(gs[g], true, A.data(), L.data(), n, 0, loc, gout + gs[g].grad);
        } else {
          const bool rev = it.kind == BI_BWD;
          const int m = ps.m;
          for (int grp = it.first; grp < it.first + it.count; ++grp) {
            uint64_t gb = 0;
            for (int j = 0; j < n - m; ++j) if (grp >> j & 1) gb |= 1ull << ps.gbit[j];
            std::vector<uint64_t> off(size_t(1) << m);
            for (uint32_t l = 0; l < (1u << m); ++l) {
              uint64_t o = gb;
              for (int j = 0; j < m; ++j) if (l >> j & 1u) o |= 1ull << ps.sbit[j];
              off[l] = o;
            }
            for (uint32_t l = 0; l < (1u << m); ++l) {
              A[l] = (!rev && it.pass == 0) ? cd(gb == 0 && l == 0 ? 1.0 : 0.0) : arena[in.psi + off[l]];
              if (rev) L[l] = arena[in.lam + off[l]];
            }
            if (!rev)
              for (int g = 0; g < ps.ngate; ++g) gate(gs[g], false, A.data(), L.data(), m, gb, loc, nullptr);
            else
              for (int g = ps.ngate - 1; g >= 0; --g) gate(gs[g], true, A.data(), L.data(), m, gb, loc, gout + gs[g].grad);
            for (uint32_t l = 0; l < (1u << m); ++l) {
              arena[in.psi + off[l]] = A[l];
              if (rev) arena[in.lam + off[l]] = L[l];
            }
          }
        }
      }
      done[it.inst] += 1;
    }
  }
};

}  // namespace

struct qs_batch {
  Cfg cfg;
  std::vector<int> n, nparam;
  Encoded enc;
  PlanCache plans;             // per instance: reused by parameter updates of the same structure
  uint8_t* d_prog = nullptr;
  void* d_arena = nullptr;
  double* d_grads = nullptr;   // nparam_total, then ninst energies
  unsigned* d_ctl = nullptr;   // next item, error word, done count per instance
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int grid = 0;
  ~qs_batch() {
    if (d_prog) cudaFree(d_prog);
    if (d_arena) cudaFree(d_arena);
    if (d_grads) cudaFree(d_grads);
    if (d_ctl) cudaFree(d_ctl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

extern "C" {

int qs_batch_create(const qs_batch_instance* insts, int ninst, const qs_batch_config* cfg, qs_batch** out) {
  return bguard([&] {
    if (!out) bad("batch: null output handle");
    *out = nullptr;
    const Cfg c = cfg_of(cfg);
    auto in = read_instances(insts, ninst);
    std::unique_ptr<qs_batch> b(new qs_batch);
    b->cfg = c;
    for (auto& x : in) { b->n.push_back(x.n); b->nparam.push_back(x.nparam); }
    b->enc = encode_batch(in, c, &b->plans);
    BCK(dev_malloc((void**)&b->d_prog, b->enc.bytes.size()));
    BCK(cudaMemcpy(b->d_prog, b->enc.bytes.data(), b->enc.bytes.size(), cudaMemcpyHostToDevice));
    if (b->enc.arena_amps) BCK(dev_malloc(&b->d_arena, b->enc.arena_amps * sizeof(float2)));
    BCK(dev_malloc((void**)&b->d_grads, (b->enc.nparam_total + ninst) * sizeof(double)));
    BCK(dev_malloc((void**)&b->d_ctl, (2 + ninst) * sizeof(unsigned)));
    BCK(cudaEventCreate(&b->ev0));
    BCK(cudaEventCreate(&b->ev1));
    *out = b.release();
  });
}

int qs_batch_set_params(qs_batch* b, const qs_batch_instance* insts, int ninst) {
  return bguard([&] {
    if (!b) bad("batch: null handle");
    if (ninst != (int)b->n.size()) bad("batch: instance count differs from the batch's");
    auto in = read_instances(insts, ninst);
    for (int i = 0; i < ninst; ++i)
      if (in[i].n != b->n[i] || in[i].nparam != b->nparam[i]) bad("batch: instance shapes differ from the batch's");
    Encoded e = encode_batch(in, b->cfg, &b->plans);
    if (e.arena_amps != b->enc.arena_amps || e.nparam_total != b->enc.nparam_total)
      bad("batch: instance shapes differ from the batch's");
    BCK(cudaDeviceSynchronize());
    if (e.bytes.size() > b->enc.bytes.size()) {
      BCK(cudaFree(b->d_prog));
      b->d_prog = nullptr;
      BCK(dev_malloc((void**)&b->d_prog, e.bytes.size()));
    }
    b->enc = std::move(e);
    BCK(cudaMemcpy(b->d_prog, b->enc.bytes.data(), b->enc.bytes.size(), cudaMemcpyHostToDevice));
  });
}

int qs_batch_run(qs_batch* b, void* stream, float* ms) {
  return bguard([&] {
    if (!b) bad("batch: null handle");
    cudaStream_t s = (cudaStream_t)stream;
    const int ninst = (int)b->n.size();
    BCK(cudaMemsetAsync(b->d_grads, 0, (b->enc.nparam_total + ninst) * sizeof(double), s));
    BCK(cudaMemsetAsync(b->d_ctl, 0, (2 + ninst) * sizeof(unsigned), s));
    BCK(cudaEventRecord(b->ev0, s));
    BCK(launch_batch(b->d_prog, b->d_arena, b->d_grads, b->d_grads + b->enc.nparam_total, b->d_ctl,
                     b->cfg.threads, b->enc.mbuf, b->cfg.bps, b->cfg.wait_ns, s, &b->grid));
    BCK(cudaEventRecord(b->ev1, s));
    if (ms) {
      BCK(cudaEventSynchronize(b->ev1));
      BCK(cudaEventElapsedTime(ms, b->ev0, b->ev1));
    }
  });
}

int qs_batch_results(qs_batch* b, double* energies, double* grads) {
  return bguard([&] {
    if (!b) bad("batch: null handle");
    const int ninst = (int)b->n.size();
    BCK(cudaDeviceSynchronize());
    unsigned err = 0;
    BCK(cudaMemcpy(&err, b->d_ctl + 1, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (err) throw BErr{"batch: a dependency wait of the batch kernel timed out (error word " + std::to_string(err) + ")",
                        QS_ERR_DEVICE};
    if (grads) BCK(cudaMemcpy(grads, b->d_grads, b->enc.nparam_total * sizeof(double), cudaMemcpyDeviceToHost));
    if (energies)
      BCK(cudaMemcpy(energies, b->d_grads + b->enc.nparam_total, ninst * sizeof(double), cudaMemcpyDeviceToHost));
  });
}

int qs_batch_info(const qs_batch* b, int* nitems, int* nparams_total, long long* arena_bytes, int* grid) {
  return bguard([&] {
    if (!b) bad("batch: null handle");
    if (nitems) *nitems = b->enc.nitem;
    if (nparams_total) *nparams_total = b->enc.nparam_total;
    if (arena_bytes) *arena_bytes = (long long)(b->enc.arena_amps * sizeof(float2));
    if (grid) *grid = b->grid;
  });
}

int qs_batch_destroy(qs_batch* b) {
  return bguard([&] { delete b; });
}

int qs_batch_describe(const qs_batch_instance* insts, int ninst, const qs_batch_config* cfg, int* stats) {
  return bguard([&] {
    if (!stats) bad("batch_describe: null stats");
    const Cfg c = cfg_of(cfg);
    auto in = read_instances(insts, ninst);
    Encoded e = encode_batch(in, c);
    BatchHeader h;
    std::memcpy(&h, e.bytes.data(), sizeof(h));
    const BatchInst* bi = reinterpret_cast<const BatchInst*>(e.bytes.data() + h.off_inst);
    const BatchPass* bp = reinterpret_cast<const BatchPass*>(e.bytes.data() + h.off_pass);
    const BatchItem* it = reinterpret_cast<const BatchItem*>(e.bytes.data() + h.off_item);
    for (int i = 0; i < ninst; ++i) {
      int* s = stats + 5 * i;
      s[0] = bi[i].npass;
      s[1] = s[2] = s[3] = s[4] = 0;
      for (int p = bi[i].pass0; p < bi[i].pass0 + bi[i].npass; ++p) {
        s[1] += bp[p].nphase > 0;
        s[2] += bp[p].nphase;
        s[3] += bp[p].ngate;
      }
    }
    for (int k = 0; k < h.nitem; ++k) stats[5 * it[k].inst + 4] += 1;
  });
}

int qs_batch_emulate(const qs_batch_instance* insts, int ninst, const qs_batch_config* cfg, double* energies,
                     double* grads) {
  return bguard([&] {
    const Cfg c = cfg_of(cfg);
    auto in = read_instances(insts, ninst);
    Encoded e = encode_batch(in, c);
    Emu emu;
    emu.b = e.bytes.data();
    emu.arena.assign(e.arena_amps, cd(0));
    emu.grads.assign(e.nparam_total, 0.0);
    emu.energy.assign(ninst, 0.0);
    emu.run();
    if (energies) std::copy(emu.energy.begin(), emu.energy.end(), energies);
    if (grads) std::copy(emu.grads.begin(), emu.grads.end(), grads);
  });
}

}  // extern "C"
