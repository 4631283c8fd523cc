// Plan-time specialisation of pass kernels (see jit.h).
#include "jit.h"

#include <cerrno>
#include <cuda.h>
#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <cstring>
#include <future>
#include <list>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <thread>
#include <unordered_map>

namespace qsb {

namespace {

// ---- NVRTC (dlopen: the library is optional at load time) ---------------------------
struct Nvrtc {
  void* h = nullptr;
  int (*create)(void**, const char*, const char*, int, const char* const*, const char* const*) = nullptr;
  int (*compile)(void*, int, const char* const*) = nullptr;
  int (*cubin_size)(void*, size_t*) = nullptr;
  int (*cubin)(void*, char*) = nullptr;
  int (*log_size)(void*, size_t*) = nullptr;
  int (*log)(void*, char*) = nullptr;
  int (*destroy)(void**) = nullptr;
  int (*version)(int*, int*) = nullptr;
  std::string why;
  bool ok = false;
  Nvrtc() {
    const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
    for (const char* n : names) {
      h = dlopen(n, RTLD_NOW | RTLD_LOCAL);
      if (h) break;
    }
    if (!h) { why = "NVRTC (libnvrtc.so.12) not found"; return; }
    create = (decltype(create))dlsym(h, "nvrtcCreateProgram");
    compile = (decltype(compile))dlsym(h, "nvrtcCompileProgram");
    cubin_size = (decltype(cubin_size))dlsym(h, "nvrtcGetCUBINSize");
    cubin = (decltype(cubin))dlsym(h, "nvrtcGetCUBIN");
    log_size = (decltype(log_size))dlsym(h, "nvrtcGetProgramLogSize");
    log = (decltype(log))dlsym(h, "nvrtcGetProgramLog");
    destroy = (decltype(destroy))dlsym(h, "nvrtcDestroyProgram");
    version = (decltype(version))dlsym(h, "nvrtcVersion");
    ok = create && compile && cubin_size && cubin && log_size && log && destroy;
    if (!ok) why = "NVRTC symbols missing";
  }
};

Nvrtc& nvrtc() {
  static Nvrtc n;
  return n;
}

// ---- driver entry points through the runtime (no link-time libcuda dependency) -------
struct Driver {
  CUresult (*load)(CUmodule*, const void*) = nullptr;
  CUresult (*unload)(CUmodule) = nullptr;
  CUresult (*get_fn)(CUfunction*, CUmodule, const char*) = nullptr;
  CUresult (*set_attr)(CUfunction, CUfunction_attribute, int) = nullptr;
  CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                     void**, void**) = nullptr;
  bool ok = false;
  std::string why;
  Driver() {
    auto get = [&](const char* name, void** fp) {
      cudaDriverEntryPointQueryResult q;
      cudaError_t e = cudaGetDriverEntryPointByVersion(name, fp, 12000, cudaEnableDefault, &q);
      return e == cudaSuccess && q == cudaDriverEntryPointSuccess && *fp;
    };
    ok = get("cuModuleLoadData", (void**)&load) && get("cuModuleUnload", (void**)&unload) &&
         get("cuModuleGetFunction", (void**)&get_fn) && get("cuFuncSetAttribute", (void**)&set_attr) &&
         get("cuLaunchKernel", (void**)&launch);
    if (!ok) why = "CUDA driver entry points unavailable";
  }
};

Driver& driver() {
  static Driver d;
  return d;
}

std::string csrc_dir() {
  Dl_info info;
  if (dladdr((void*)&jit_available, &info) && info.dli_fname) {
    std::string p(info.dli_fname);
    size_t s = p.rfind('/');
    return (s == std::string::npos ? std::string(".") : p.substr(0, s)) + "/csrc";
  }
  return "csrc";
}

int cls_of(float re, float im) {
  if (re == 0.0f && im == 0.0f) return 0;
  if (im == 0.0f) return re == 1.0f ? 1 : (re == -1.0f ? 2 : 5);
  if (re == 0.0f) return im == 1.0f ? 3 : (im == -1.0f ? 4 : 6);
  return 7;
}

uint64_t fnv(uint64_t h, const void* p, size_t n) {
  const uint8_t* b = (const uint8_t*)p;
  for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
  return h;
}

// ---- code generation ------------------------------------------------------------------
struct Ent {
  int cls = 0;          // 0 zero, 1 one, 2 minus one, 3 +i, 4 -i, 5 real, 6 imaginary, 7 general
  std::string var;      // coefficient variable for classes 5..7
  int off = -1;         // its entry of the coefficient table (-1: a per-thread value)
};

struct Gen {
  std::ostringstream o;
  const float* coef = nullptr;  // interleaved complex64 table
  int nvar = 0;
  bool used_fa = false;  // the phase accumulated diagonal factors of non-register bits in `fa`
  int kbase = 0, kcount = 0;  // coefficients [kbase, kbase + kcount) arrive as a kernel parameter

  // expression of coefficient `off`: the pass's parameter block (constant bank, an operand
  // of the arithmetic instruction itself) or, past its capacity, a load from the table
  std::string kref(int off) const {
    if (off >= kbase && off < kbase + kcount) return "kp->k[" + std::to_string(off - kbase) + "]";
    return "LK(" + std::to_string(off) + ")";
  }
  // coefficient off + v for a run-time v in [0, n)
  std::string kref_dyn(int off, int n, const std::string& v) const {
    if (off >= kbase && off + n <= kbase + kcount) return "kp->k[" + std::to_string(off - kbase) + "+" + v + "]";
    return "LK(" + std::to_string(off) + "+" + v + ")";
  }

  Ent coef_ent(int off) {
    Ent e;
    e.cls = cls_of(coef[2 * off], coef[2 * off + 1]);
    if (e.cls >= 5) {
      e.var = "k" + std::to_string(nvar++);
      e.off = off;
      o << "const float2 " << e.var << " = " << kref(off) << ";";
    }
    return e;
  }

  // ---- packed registers (FP32x2 arithmetic on two amplitudes) ----
  // packed: the phase's registers are R[q] / I[q] (real / imaginary parts of registers 2q and
  // 2q + 1); gates that do not act on register bit 0 update both lanes with one packed
  // instruction, gates on bit 0 read and write single lanes (LDA / STA).
  bool packed = false;
  std::vector<uint32_t> splats;               // parameter-block splats: entry * 4 + component
  std::unordered_map<uint32_t, int> splat_idx;
  int splat_cap = 0;                          // splats that fit the parameter block

  // {v, v} for component comp (0: x, 1: y, 2: -x, 3: -y) of e: a parameter-block entry
  // (constant bank operand) when e is a table entry and the block has room, else built from
  // the variable
  std::string splat(const Ent& e, int comp) {
    if (e.off >= 0) {
      const uint32_t key = (uint32_t)e.off * 4u + (uint32_t)comp;
      auto it = splat_idx.find(key);
      int j = -1;
      if (it != splat_idx.end()) {
        j = it->second;
      } else if ((int)splats.size() < splat_cap) {
        j = (int)splats.size();
        splats.push_back(key);
        splat_idx[key] = j;
      }
      if (j >= 0) return "kp->s[" + std::to_string(j) + "]";
    }
    static const char* c[4] = {".x", ".y", ".x", ".y"};
    const std::string v = std::string(comp >= 2 ? "-" : "") + e.var + c[comp];
    return "make_float2(" + v + "," + v + ")";
  }

  // packed sum_c row[c] * x_c: real part (comp 0) or imaginary part (comp 1); xr / xi name
  // the operands' packed real / imaginary parts.  Unit entries are adds (a negated one a
  // multiply-add by M1 = {-1, -1}), the others multiply-adds with splatted coefficients.
  std::string plin(const Ent* row, const std::vector<std::string>& xr, const std::vector<std::string>& xi,
                   int comp) {
    struct Term {
      std::string k;  // splatted coefficient; empty: +-1
      std::string x;
      bool neg;
    };
    std::vector<Term> ts;
    for (size_t c = 0; c < xr.size(); ++c) {
      const Ent& e = row[c];
      const std::string& R = xr[c];
      const std::string& I = xi[c];
      switch (e.cls) {
        case 0: break;
        case 1: ts.push_back({"", comp ? I : R, false}); break;
        case 2: ts.push_back({"", comp ? I : R, true}); break;
        case 3: ts.push_back(comp ? Term{"", R, false} : Term{"", I, true}); break;   // +i
        case 4: ts.push_back(comp ? Term{"", R, true} : Term{"", I, false}); break;   // -i
        case 5: ts.push_back({splat(e, 0), comp ? I : R, false}); break;
        case 6:
          if (comp) ts.push_back({splat(e, 1), R, false});
          else ts.push_back({splat(e, 3), I, false});
          break;
        default:
          if (comp) {
            ts.push_back({splat(e, 0), I, false});
            ts.push_back({splat(e, 1), R, false});
          } else {
            ts.push_back({splat(e, 0), R, false});
            ts.push_back({splat(e, 3), I, false});
          }
      }
    }
    if (ts.empty()) return "make_float2(0.f,0.f)";
    std::string acc;
    auto first = std::find_if(ts.begin(), ts.end(), [](const Term& t) { return t.k.empty() && !t.neg; });
    if (first != ts.end()) {
      acc = first->x;
      ts.erase(first);
    } else {
      const Term t = ts.front();
      ts.erase(ts.begin());
      acc = t.k.empty() ? "__fmul2_rn(" + t.x + ",M1)" : "__fmul2_rn(" + t.k + "," + t.x + ")";
    }
    for (const Term& t : ts) {
      if (t.k.empty())
        acc = t.neg ? "__ffma2_rn(" + t.x + ",M1," + acc + ")" : "__fadd2_rn(" + acc + "," + t.x + ")";
      else
        acc = "__ffma2_rn(" + t.k + "," + t.x + "," + acc + ")";
    }
    return acc;
  }

  // register access in the emitted loops: a[i] (interleaved) or one lane of R / I (packed)
  std::string rd(const std::string& i) const { return packed ? "LDA(" + i + ")" : "a[" + i + "]"; }
  std::string wr(const std::string& i, const std::string& v) const {
    return packed ? "STA(" + i + "," + v + ");" : "a[" + i + "]=" + v + ";";
  }
  static Ent cst(int cls) { Ent e; e.cls = cls; return e; }
  Ent cls_ent(int off) const { return cst(cls_of(coef[2 * off], coef[2 * off + 1])); }

  // ---- bit-flip frame of the phase ----
  // mask[j] names a warp-uniform bool: when true, register index i holds the amplitude of
  // logical register index i ^ (1 << j).  A bit flip conditioned on a warp-uniform fixed bit
  // (a CX whose control is a group or warp-index bit) only toggles mask[j]; later gates on
  // bit j run as their X-conjugated version under the mask, and the phase's stores land at
  // the flipped addresses.  Empty name: mask known to be false.
  std::string mask[kMaxR];
  int nmask = 0;
  std::ostringstream post;  // declarations emitted after the current gate's block
  void reset_masks() {
    for (auto& m : mask) m.clear();
  }
  // mask[j] ^= cond (cond: a bool-valued expression)
  void toggle_mask(int j, const std::string& cond) {
    const std::string v = "m" + std::to_string(nmask++);
    post << "const bool " << v << "=" << (mask[j].empty() ? "(bool)(" + cond + ")" : "(" + mask[j] + "!=(bool)(" + cond + "))")
         << ";";
    mask[j] = v;
  }
  // entries of X^c M X^c for the d x d matrix m (bit k of c flips matrix bit k)
  static void conjugate(Ent* m, int d, unsigned c) {
    if (!c) return;
    Ent t[16];
    for (int r = 0; r < d; ++r)
      for (int col = 0; col < d; ++col) t[r * d + col] = m[(r ^ c) * d + (col ^ c)];
    for (int e = 0; e < d * d; ++e) m[e] = t[e];
  }
  // body(c) under every value of the masks of the register bits `bits` (bit k of c = mask of
  // bits[k]); the versions update the same registers in place
  void masked(const std::vector<int>& bits, const std::function<void(unsigned)>& body, size_t k = 0,
              unsigned c = 0) {
    if (k == bits.size()) {
      o << "{";
      body(c);
      o << "}";
      return;
    }
    if (bits[k] < 0 || bits[k] >= kMaxR || mask[bits[k]].empty()) {
      masked(bits, body, k + 1, c);
      return;
    }
    o << "if(" << mask[bits[k]] << "){";
    masked(bits, body, k + 1, c | (1u << k));
    o << "}else{";
    masked(bits, body, k + 1, c);
    o << "}";
  }

  // Multiplies every entry of the d x d matrix m by the phase factor fa (per-thread values):
  // the gate then also applies the phase's diagonal factor of its fixed bits.
  void fold(Ent* m, int d) {
    static const char* unit[5] = {"", "fa", "make_float2(-fa.x,-fa.y)", "make_float2(-fa.y,fa.x)",
                                  "make_float2(fa.y,-fa.x)"};
    for (int e = 0; e < d * d; ++e) {
      if (m[e].cls == 0) continue;
      const std::string v = "f" + std::to_string(nvar++);
      if (m[e].cls <= 4) {
        o << "const float2 " << v << "=" << unit[m[e].cls] << ";";
      } else {
        const std::string& k = m[e].var;
        o << "const float2 " << v << "=make_float2(fa.x*" << k << ".x-fa.y*" << k << ".y,fa.x*" << k << ".y+fa.y*"
          << k << ".x);";
      }
      m[e].cls = 7;
      m[e].var = v;
    }
  }

  // Arithmetic instructions per amplitude that folding fa into the d x d matrix m adds
  // (lin's terms: a leading +x is a move, a leading -x / +-ix one instruction per component,
  // other unit and real/imaginary terms one per component, general terms two).
  static double fold_added(const Ent* m, int d) {
    auto term = [](int cls, bool first) {
      if (cls == 0) return 0;
      if (cls == 1) return first ? 0 : 2;
      if (cls <= 4) return first ? 1 : 2;
      return cls == 7 ? 4 : 2;
    };
    double added = 0;
    for (int r = 0; r < d; ++r) {
      bool first = true;
      for (int c = 0; c < d; ++c) {
        const int cls = m[r * d + c].cls;
        if (!cls) continue;
        added += term(7, first) - term(cls, first);
        first = false;
      }
    }
    return added / d;
  }

  // linear combination sum_c row[c] * x_c; empty string when all terms vanish
  static std::string lin(const Ent* row, const char* const* x, int n) {
    std::string re, im;
    int nz = 0, last = -1;
    for (int c = 0; c < n; ++c) {
      const Ent& e = row[c];
      const std::string X(x[c]);
      const std::string& k = e.var;
      switch (e.cls) {
        case 0: continue;
        case 1: re += "+" + X + ".x"; im += "+" + X + ".y"; break;
        case 2: re += "-" + X + ".x"; im += "-" + X + ".y"; break;
        case 3: re += "-" + X + ".y"; im += "+" + X + ".x"; break;
        case 4: re += "+" + X + ".y"; im += "-" + X + ".x"; break;
        case 5: re += "+" + k + ".x*" + X + ".x"; im += "+" + k + ".x*" + X + ".y"; break;
        case 6: re += "-" + k + ".y*" + X + ".y"; im += "+" + k + ".y*" + X + ".x"; break;
        default:
          re += "+" + k + ".x*" + X + ".x-" + k + ".y*" + X + ".y";
          im += "+" + k + ".x*" + X + ".y+" + k + ".y*" + X + ".x";
      }
      ++nz;
      last = c;
    }
    if (nz == 0) return "make_float2(0.f,0.f)";
    if (nz == 1 && row[last].cls == 1) return x[last];
    return "make_float2(" + re + "," + im + ")";
  }

  static bool is_identity(const Ent* m, int d) {
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c)
        if (m[r * d + c].cls != (r == c ? 1 : 0)) return false;
    return true;
  }

  // 2x2 on register bit J
  void pairs(int J, const Ent* m) {
    if (is_identity(m, 2)) return;
    if (packed && J > 0) { ppairs(J, m, ""); return; }
    static const char* x[2] = {"x0", "x1"};
    const std::string B = std::to_string(1 << J);
    o << "\n#pragma unroll\nfor(int i=0;i<NR;++i) if(!(i&" << B << ")){const float2 x0=" << rd("i") << ",x1="
      << rd("i|" + B) << ";" << wr("i", lin(m, x, 2)) << wr("i|" + B, lin(m + 2, x, 2)) << "}\n";
  }
  // 2x2 on register bit J, applied where the runtime condition holds (selects, no divergence)
  void pairs_sel(int J, const Ent* m, const std::string& cond) {
    if (is_identity(m, 2)) return;
    if (packed && J > 0) { ppairs(J, m, cond); return; }
    static const char* x[2] = {"x0", "x1"};
    const std::string B = std::to_string(1 << J);
    o << "\n#pragma unroll\nfor(int i=0;i<NR;++i) if(!(i&" << B << ")){const float2 x0=" << rd("i") << ",x1="
      << rd("i|" + B) << ";const float2 y0=" << lin(m, x, 2) << ",y1=" << lin(m + 2, x, 2) << ";"
      << wr("i", "(" + cond + ")?y0:x0") << wr("i|" + B, "(" + cond + ")?y1:x1") << "}\n";
  }
  // packed 2x2 on register bit J >= 1 (both lanes at once); cond: applied where it holds
  void ppairs(int J, const Ent* m, const std::string& cond) {
    const std::string b = std::to_string(1 << (J - 1));
    const std::vector<std::string> xr = {"r0", "r1"}, xi = {"i0", "i1"};
    o << "\n#pragma unroll\nfor(int q=0;q<NQ;++q) if(!(q&" << b << ")){const float2 r0=R[q],i0=I[q],r1=R[q|" << b
      << "],i1=I[q|" << b << "];";
    const std::string y0 = plin(m, xr, xi, 0), y1 = plin(m, xr, xi, 1), y2 = plin(m + 2, xr, xi, 0),
                      y3 = plin(m + 2, xr, xi, 1);
    if (cond.empty()) {
      o << "R[q]=" << y0 << ";I[q]=" << y1 << ";R[q|" << b << "]=" << y2 << ";I[q|" << b << "]=" << y3 << ";}\n";
    } else {
      o << "const float2 y0=" << y0 << ",y1=" << y1 << ",y2=" << y2 << ",y3=" << y3 << ";const bool c_=(bool)("
        << cond << ");R[q]=c_?y0:r0;I[q]=c_?y1:i0;R[q|" << b << "]=c_?y2:r1;I[q|" << b << "]=c_?y3:i1;}\n";
    }
  }
  // 4x4 on register bits (JA = matrix bit 0, JB = matrix bit 1)
  void quads(int JA, int JB, const Ent* m) {
    if (is_identity(m, 4)) return;
    if (packed && JA > 0 && JB > 0) { pquads(JA, JB, m); return; }
    static const char* x[4] = {"x0", "x1", "x2", "x3"};
    const std::string A = std::to_string(1 << JA), B = std::to_string(1 << JB),
                      AB = std::to_string((1 << JA) | (1 << JB));
    o << "\n#pragma unroll\nfor(int i=0;i<NR;++i) if(!(i&" << AB << ")){const float2 x0=" << rd("i") << ",x1="
      << rd("i|" + A) << ",x2=" << rd("i|" + B) << ",x3=" << rd("i|" + AB) << ";";
    o << wr("i", lin(m, x, 4)) << wr("i|" + A, lin(m + 4, x, 4)) << wr("i|" + B, lin(m + 8, x, 4))
      << wr("i|" + AB, lin(m + 12, x, 4)) << "}\n";
  }
  // packed 4x4 on register bits JA, JB >= 1
  void pquads(int JA, int JB, const Ent* m) {
    const std::string A = std::to_string(1 << (JA - 1)), B = std::to_string(1 << (JB - 1)),
                      AB = std::to_string((1 << (JA - 1)) | (1 << (JB - 1)));
    const std::vector<std::string> xr = {"r0", "r1", "r2", "r3"}, xi = {"i0", "i1", "i2", "i3"};
    o << "\n#pragma unroll\nfor(int q=0;q<NQ;++q) if(!(q&" << AB << ")){const float2 r0=R[q],i0=I[q],r1=R[q|" << A
      << "],i1=I[q|" << A << "],r2=R[q|" << B << "],i2=I[q|" << B << "],r3=R[q|" << AB << "],i3=I[q|" << AB << "];";
    const std::string idx[4] = {"q", "q|" + A, "q|" + B, "q|" + AB};
    std::string y[8];
    for (int r = 0; r < 4; ++r) {
      y[2 * r] = plin(m + 4 * r, xr, xi, 0);
      y[2 * r + 1] = plin(m + 4 * r, xr, xi, 1);
    }
    for (int r = 0; r < 4; ++r) o << "R[" << idx[r] << "]=" << y[2 * r] << ";I[" << idx[r] << "]=" << y[2 * r + 1] << ";";
    o << "}\n";
  }
  // every amplitude times a (possibly selected) scalar
  void scale(const Ent& d) {
    if (d.cls == 1) return;
    if (packed) {
      const std::vector<std::string> xr = {"r0"}, xi = {"i0"};
      o << "\n#pragma unroll\nfor(int q=0;q<NQ;++q){const float2 r0=R[q],i0=I[q];R[q]=" << plin(&d, xr, xi, 0)
        << ";I[q]=" << plin(&d, xr, xi, 1) << ";}\n";
      return;
    }
    static const char* x[1] = {"x0"};
    o << "\n#pragma unroll\nfor(int i=0;i<NR;++i){const float2 x0=a[i];a[i]=" << lin(&d, x, 1) << ";}\n";
  }
};

// complex coefficients a gate instruction reads from the table
int coef_entries(uint8_t kind) {
  switch (kind) {
    case GK_1Q_DENSE: case GK_1Q_REAL: case GK_1Q_REIM: case GK_2Q_DIAG: case GK_2Q_CU: return 4;
    case GK_1Q_DIAG: return 2;
    case GK_2Q_DENSE: return 16;
    default: return 0;
  }
}

// Coefficients travel as a by-value kernel parameter of each pass kernel (constant bank 0):
// up to 4000 complex64 entries, 32 000 bytes, within the 32 764-byte parameter limit.
constexpr int kParamCoefs = 4000;

// The contiguous range of the coefficient table that pass p reads (count capped at
// kParamCoefs; entries past the cap are loaded from the table).
void pass_coef_range(const uint8_t* b, int p, int* base, int* count) {
  const ProgramHeader* hdr = (const ProgramHeader*)b;
  const PassDesc& pd = ((const PassDesc*)(b + hdr->off_pass))[p];
  const PhaseDesc* phs = (const PhaseDesc*)(b + hdr->off_phase);
  const GateInstr* gis = (const GateInstr*)(b + hdr->off_gate);
  int lo = 0, hi = -1;
  for (int h = 0; h < pd.nphase; ++h) {
    const PhaseDesc& ph = phs[pd.phase0 + h];
    for (int gi = 0; gi < ph.ngate; ++gi) {
      const GateInstr& g = gis[ph.gate0 + gi];
      const int ne = coef_entries(g.kind);
      if (!ne) continue;
      if (hi < 0 || g.coef < lo) lo = g.coef;
      hi = std::max(hi, g.coef + ne);
    }
  }
  *base = hi < 0 ? 0 : lo;
  *count = hi < 0 ? 0 : std::min(hi - lo, kParamCoefs);
}

std::string bitcond(int phys) { return "((pb>>" + std::to_string(phys) + ")&1ull)"; }

// Diagonal gate whose bits are all fixed per thread: a factor of the phase scalar fa.
bool fixed_diag(const GateInstr& g) {
  return (g.kind == GK_1Q_DIAG && g.a >= kFixed) || (g.kind == GK_2Q_DIAG && g.a >= kFixed && g.b >= kFixed);
}

// Entry classes of an unconditional register gate that acts on every amplitude of the thread
// (so it can absorb the phase scalar); false for other gates.  d = matrix dimension.
bool absorber_matrix(const Gen& G, const GateInstr& g, Ent* m, int* d) {
  const int c = g.coef;
  const bool fa = g.a >= kFixed, fb = g.b >= kFixed;
  switch (g.kind) {
    case GK_1Q_DENSE: case GK_1Q_REAL: case GK_1Q_REIM:
      *d = 2;
      for (int e = 0; e < 4; ++e) m[e] = G.cls_ent(c + e);
      return true;
    case GK_1Q_DIAG:
      if (fa) return false;
      *d = 2;
      m[0] = G.cls_ent(c); m[1] = Gen::cst(0); m[2] = Gen::cst(0); m[3] = G.cls_ent(c + 1);
      return true;
    case GK_2Q_DENSE:
      *d = 4;
      for (int e = 0; e < 16; ++e) m[e] = G.cls_ent(c + e);
      return true;
    case GK_2Q_DIAG:
      if (fa || fb) return false;
      *d = 4;
      for (int e = 0; e < 16; ++e) m[e] = Gen::cst(0);
      for (int e = 0; e < 4; ++e) m[5 * e] = G.cls_ent(c + e);
      return true;
    case GK_2Q_CU:
      if (fa) return false;
      *d = 4;
      for (int r = 0; r < 4; ++r)
        for (int col = 0; col < 4; ++col) m[4 * r + col] = Gen::cst((r == col && !(r & 1)) ? 1 : 0);
      m[5] = G.cls_ent(c); m[7] = G.cls_ent(c + 1); m[13] = G.cls_ent(c + 2); m[15] = G.cls_ent(c + 3);
      return true;
    default:
      return false;
  }
}

// fold: the gate also applies the phase scalar fa (it must be an absorber_matrix gate)
void gen_gate(Gen& G, const GateInstr& g, const PassDesc& pd, const PhaseDesc& ph, bool fold = false) {
  auto& o = G.o;
  o << "{";
  const bool fa = g.a >= kFixed, fb = g.b >= kFixed;
  const int c = g.coef;
  // whether a fixed bit is uniform across the warp (group bit or warp-index bit)
  auto warp_uniform = [&](int phys) {
    for (int j = 0; j < 5 && j < pd.m - pd.r; ++j)
      if (pd.sbit[ph.tbit[j]] == phys) return false;
    return true;
  };
  // the gate's matrix, X-conjugated under the bit-flip frame of its register operands
  auto pairs_m = [&](int J, const Ent* m0) {
    G.masked({J}, [&](unsigned cm) {
      Ent m[4];
      std::copy(m0, m0 + 4, m);
      Gen::conjugate(m, 2, cm);
      if (fold) G.fold(m, 2);
      G.pairs(J, m);
    });
  };
  auto quads_m = [&](int A, int B, const Ent* m0) {
    G.masked({A, B}, [&](unsigned cm) {
      Ent m[16];
      std::copy(m0, m0 + 16, m);
      Gen::conjugate(m, 4, cm);
      if (fold) G.fold(m, 4);
      G.quads(A, B, m);
    });
  };
  switch (g.kind) {
    case GK_1Q_DENSE: case GK_1Q_REAL: case GK_1Q_REIM: {
      Ent m[4] = {G.coef_ent(c), G.coef_ent(c + 1), G.coef_ent(c + 2), G.coef_ent(c + 3)};
      pairs_m(g.a, m);
      break;
    }
    case GK_1Q_X: {
      // packed registers: X on the lane bit only flips the frame (the stores swap the lanes)
      if (G.packed && g.a == 0) {
        G.toggle_mask(0, "true");
        break;
      }
      // register rename; X commutes with the frame
      Ent m[4] = {Gen::cst(0), Gen::cst(1), Gen::cst(1), Gen::cst(0)};
      G.pairs(g.a, m);
      break;
    }
    case GK_1Q_DIAG: {
      if (!fa) {
        Ent m[4] = {G.coef_ent(c), Gen::cst(0), Gen::cst(0), G.coef_ent(c + 1)};
        pairs_m(g.a, m);
      } else {
        // a diagonal gate on a non-register bit commutes with every gate of the phase:
        // its per-thread factor joins the phase's accumulated scalar
        o << "const float2 d=" << bitcond(g.a - kFixed) << "?" << G.kref(c + 1) << ":" << G.kref(c) << ";"
          << "fa=make_float2(fa.x*d.x-fa.y*d.y,fa.x*d.y+fa.y*d.x);";
        G.used_fa = true;
      }
      break;
    }
    case GK_2Q_DENSE: {
      Ent m[16];
      for (int e = 0; e < 16; ++e) m[e] = G.coef_ent(c + e);
      quads_m(g.a, g.b, m);
      break;
    }
    case GK_2Q_SWAP: {
      // register rename; the frame bits swap with the data
      Ent m[16];
      const int P[4] = {0, 2, 1, 3};
      for (int r = 0; r < 4; ++r)
        for (int col = 0; col < 4; ++col) m[4 * r + col] = Gen::cst(col == P[r] ? 1 : 0);
      G.quads(g.a, g.b, m);
      std::swap(G.mask[g.a], G.mask[g.b]);
      break;
    }
    case GK_2Q_DIAG: {
      if (!fa && !fb) {
        Ent m[16];
        for (int e = 0; e < 16; ++e) m[e] = Gen::cst(0);
        for (int e = 0; e < 4; ++e) m[5 * e] = G.coef_ent(c + e);
        quads_m(g.a, g.b, m);
      } else if (fa && fb) {
        o << "const int v=(int)" << bitcond(g.a - kFixed) << "+2*(int)" << bitcond(g.b - kFixed)
          << ";const float2 d=" << G.kref_dyn(c, 4, "v") << ";"
          << "fa=make_float2(fa.x*d.x-fa.y*d.y,fa.x*d.y+fa.y*d.x);";
        G.used_fa = true;
      } else {
        // one fixed bit selects a diagonal 2x2 on the register bit
        const int J = fa ? g.b : g.a;
        const std::string cond = bitcond((fa ? g.a : g.b) - kFixed);
        // entries indexed b_a + 2 b_b
        const int lo0 = fa ? c + 0 : c + 0, hi0 = fa ? c + 2 : c + 1;   // fixed bit = 0
        const int lo1 = fa ? c + 1 : c + 2, hi1 = fa ? c + 3 : c + 3;   // fixed bit = 1
        o << "const float2 d0=" << cond << "?" << G.kref(lo1) << ":" << G.kref(lo0) << ";const float2 d1=" << cond
          << "?" << G.kref(hi1) << ":" << G.kref(hi0) << ";";
        Ent m[4];
        m[0].cls = 7; m[0].var = "d0";
        m[3].cls = 7; m[3].var = "d1";
        pairs_m(J, m);
      }
      break;
    }
    case GK_2Q_CX: case GK_2Q_CU: {
      if (fold && (g.kind != GK_2Q_CU || fa)) throw std::runtime_error("jit: gate cannot absorb the phase scalar");
      Ent u[4];
      if (g.kind == GK_2Q_CX) {
        u[0] = Gen::cst(0); u[1] = Gen::cst(1); u[2] = Gen::cst(1); u[3] = Gen::cst(0);
      } else {
        for (int e = 0; e < 4; ++e) u[e] = G.coef_ent(c + e);
      }
      if (!fa) {
        // control a (matrix bit 0), target b (matrix bit 1): U acts on indices 1 and 3
        Ent m[16];
        for (int r = 0; r < 4; ++r)
          for (int col = 0; col < 4; ++col) m[4 * r + col] = Gen::cst((r == col && !(r & 1)) ? 1 : 0);
        m[4 * 1 + 1] = u[0]; m[4 * 1 + 3] = u[1]; m[4 * 3 + 1] = u[2]; m[4 * 3 + 3] = u[3];
        if (g.kind == GK_2Q_CX) {
          // register rename; a flipped control flips the target's frame bit
          G.quads(g.a, g.b, m);
          if (!G.mask[g.a].empty()) G.toggle_mask(g.b, G.mask[g.a]);
        } else {
          quads_m(g.a, g.b, m);
        }
      } else {
        const int P = g.a - kFixed;
        if (g.kind == GK_2Q_CX && warp_uniform(P)) {
          // bit flip under a warp-uniform condition: frame only, no data movement
          G.toggle_mask(g.b, bitcond(P));
        } else if (warp_uniform(P)) {
          o << "if(" << bitcond(P) << "){";
          pairs_m(g.b, u);
          o << "}";
        } else if (g.kind == GK_2Q_CX) {
          G.pairs_sel(g.b, u, bitcond(P));  // X commutes with the frame
        } else {
          G.masked({g.b}, [&](unsigned cm) {
            Ent m[4];
            std::copy(u, u + 4, m);
            Gen::conjugate(m, 2, cm);
            G.pairs_sel(g.b, m, bitcond(P));
          });
        }
      }
      break;
    }
    default:
      throw std::runtime_error("jit: unknown gate kind " + std::to_string((int)g.kind));
  }
  o << "}\n" << G.post.str();
  G.post.str("");
}

// Gradient programs: before a parameterised gate (generator gen on the instruction's operand),
// the thread's part of Im <lam|G|psi> over its registers (register bit A holds the lam bit)
// into a phase-scope accumulator gt<local>; the accumulators are reduced over the warp in
// batches (gen_term_flush: independent shuffle chains).  A fixed operand only occurs for Z (a
// diagonal gate): its sign is the thread's bit.  Under a flipped frame bit the registers of
// the gate's bit hold X-conjugated data: X G X = -G for Y and Z.
void gen_term(Gen& G, const GateInstr& g, int gen, int local, int A, std::vector<int>* pending) {
  auto& o = G.o;
  if (A < 0 || !G.mask[A].empty()) throw std::runtime_error("jit: the lam bit is not a plain register bit");
  const std::string AM = std::to_string(1 << A);
  const std::string v = "gt" + std::to_string(local);
  o << "float " << v << "=0.f;{";
  if (g.a >= kFixed) {
    if (gen != 3) throw std::runtime_error("jit: an X or Y rotation on a fixed bit");
    o << "\n#pragma unroll\nfor(int i=0;i<NR;++i) if(!(i&" << AM << ")){const float2 p=a[i],l=a[i|" << AM
      << "];" << v << "+=l.x*p.y-l.y*p.x;}\nif(" << bitcond(g.a - kFixed) << ")" << v << "=-" << v << ";";
  } else {
    const int J = g.a;
    if (J == A) throw std::runtime_error("jit: a gate on the lam bit");
    const std::string JM = std::to_string(1 << J), AJ = std::to_string((1 << A) | (1 << J));
    G.masked({J}, [&](unsigned cm) {
      const bool flip = cm != 0 && gen != 1;
      o << "\n#pragma unroll\nfor(int i=0;i<NR;++i) if(!(i&" << AJ << ")){const float2 p0=a[i],p1=a[i|" << JM
        << "],l0=a[i|" << AM << "],l1=a[i|" << AJ << "];" << v << (flip ? "-=" : "+=");
      if (gen == 1) o << "(l0.x*p1.y-l0.y*p1.x)+(l1.x*p0.y-l1.y*p0.x);}\n";
      else if (gen == 2) o << "(l1.x*p0.x+l1.y*p0.y)-(l0.x*p1.x+l0.y*p1.y);}\n";
      else o << "(l0.x*p0.y-l0.y*p0.x)-(l1.x*p1.y-l1.y*p1.x);}\n";
    });
  }
  o << "}\n";
  pending->push_back(local);
}

// accumulators live at once (registers) before a flush
constexpr int kTermBatch = 4;

// Warp sums of the pending term accumulators, interleaved per shuffle distance; lane 0 adds
// them to its warp's row of the block's terms (no shared-memory atomics: one writer per row).
void gen_term_flush(Gen& G, std::vector<int>* pending, int nt) {
  if (pending->empty()) return;
  auto& o = G.o;
  for (int d = 16; d >= 1; d >>= 1)
    for (int t : *pending) o << "gt" << t << "+=__shfl_xor_sync(0xffffffffu,gt" << t << "," << d << ");";
  o << "if((threadIdx.x&31u)==0u){double* gw=ga+(threadIdx.x>>5)*" << nt << ";";
  for (int t : *pending) o << "gw[" << t << "]+=(double)gt" << t << ";";
  o << "}\n";
  pending->clear();
}

const char* kPrelude = R"(
#include "pass_body.cuh"
__device__ __forceinline__ float2 ldk_(const float2* p) {
  float2 v;
  asm volatile("ld.global.nc.v2.f32 {%0,%1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}
#define LK(i) ldk_(K + (i))
#define LDA(i) (((i)&1)?make_float2(R[(i)>>1].y,I[(i)>>1].y):make_float2(R[(i)>>1].x,I[(i)>>1].x))
#define STA(i,v) do{const float2 t_=(v);if((i)&1){R[(i)>>1].y=t_.x;I[(i)>>1].y=t_.y;}else{R[(i)>>1].x=t_.x;I[(i)>>1].x=t_.y;}}while(0)
)";

}  // namespace

JitKernels::~JitKernels() {
  Driver& d = driver();
  if (d.ok)
    for (void* m : modules) d.unload((CUmodule)m);
}

bool jit_available(std::string* why) {
  if (!nvrtc().ok) { if (why) *why = nvrtc().why; return false; }
  if (!driver().ok) { if (why) *why = driver().why; return false; }
  return true;
}

uint64_t jit_key(const Program& prog, const JitConfig& cfg) {
  const ProgramHeader* hdr = (const ProgramHeader*)prog.bytes.data();
  const float* cf = (const float*)(prog.bytes.data() + hdr->off_coef);
  uint64_t h = fnv(1469598103934665603ull, prog.bytes.data(), hdr->off_coef);
  std::vector<uint8_t> cls(hdr->ncoef);
  for (int i = 0; i < hdr->ncoef; ++i) cls[i] = (uint8_t)cls_of(cf[2 * i], cf[2 * i + 1]);
  h = fnv(h, cls.data(), cls.size());
  h = fnv(h, &cfg.blocks, sizeof(cfg.blocks));
  if (!prog.grad_gen.empty()) {
    h = fnv(h, prog.grad_gen.data(), prog.grad_gen.size());
    h = fnv(h, prog.grad_term.data(), prog.grad_term.size() * sizeof(int32_t));
  }
  const int pk = cfg.packed ? 1 : 0;
  return fnv(h, &pk, sizeof(pk));
}

std::string jit_source(const Program& prog, int pass_begin, int pass_end, uint64_t key, const JitConfig& cfg,
                       std::vector<std::vector<uint32_t>>* splats_out) {
  const uint8_t* b = prog.bytes.data();
  const ProgramHeader* hdr = (const ProgramHeader*)b;
  if (hdr->dtype != 0) throw std::runtime_error("jit: complex64 programs only");
  const PassDesc* pds = (const PassDesc*)(b + hdr->off_pass);
  const PhaseDesc* phs = (const PhaseDesc*)(b + hdr->off_phase);
  const GateInstr* gis = (const GateInstr*)(b + hdr->off_gate);
  Gen G;
  G.coef = (const float*)(b + hdr->off_coef);
  G.o << kPrelude;
  char kname[64];
  const bool grad = !prog.grad_gen.empty();
  for (int p = pass_begin; p < pass_end; ++p) {
    const PassDesc& pd = pds[p];
    pass_coef_range(b, p, &G.kbase, &G.kcount);
    // gradient programs: the pass's terms [t0, t0 + nt) (numbered in instruction order)
    int t0 = 0, nt = 0;
    if (grad) {
      int lo = -1, hi = -1;
      for (int h = 0; h < pd.nphase; ++h) {
        const PhaseDesc& ph = phs[pd.phase0 + h];
        for (int gi = 0; gi < ph.ngate; ++gi) {
          const int t = prog.grad_term[ph.gate0 + gi];
          if (t < 0) continue;
          if (lo < 0) lo = t;
          hi = t + 1;
        }
      }
      if (lo >= 0) { t0 = lo; nt = hi - lo; }
    }
    // packed registers when every phase holds local bit 0 in register bit 0
    bool packed = cfg.packed && pd.nphase > 0 && !pd.store_perm && !grad;
    for (int h = 0; h < pd.nphase && packed; ++h)
      if (phs[pd.phase0 + h].rbit[0] != 0) packed = false;
    G.packed = packed;
    G.splats.clear();
    G.splat_idx.clear();
    G.splat_cap = packed ? std::max(0, kParamCoefs - std::max(1, G.kcount)) : 0;
    // the pass's struct X is generated first: its splats size the parameter block
    std::ostringstream outer;
    outer.swap(G.o);
    G.o << "struct X" << p << "{const KP" << p << "* kp;" << (grad ? "double* ga;" : "")
        << "\nstatic constexpr bool kPacked=" << (packed ? "true" : "false") << ";\n";
    // swizzled byte offsets of each phase's register bits: immediates
    G.o << "template<typename Real,int LR>__device__ __forceinline__ void reg_offsets(const qsb::PhaseDesc*,int h,"
        << "uint32_t (&B)[LR])const{switch(h){";
    for (int h = 0; h < pd.nphase; ++h) {
      const PhaseDesc& ph = phs[pd.phase0 + h];
      G.o << "case " << h << ":";
      for (int j = 0; j < pd.r; ++j) G.o << "B[" << j << "]=" << swz64(1u << ph.rbit[j]) * 8u << "u;";
      G.o << "break;";
    }
    G.o << "default:break;}}\n";
    if (packed) {
      G.o << "template<int LR>__device__ __forceinline__ uint32_t run_packed(const uint8_t* prog,int h,"
          << "float2 (&R)[1<<(LR-1)],float2 (&I)[1<<(LR-1)],uint64_t pb)const{constexpr int NR=1<<LR;"
          << "constexpr int NQ=NR/2;const float2 M1=make_float2(-1.f,-1.f);(void)M1;(void)NR;"
          << "const float2* K=(const float2*)(prog+((const qsb::ProgramHeader*)prog)->off_coef);switch(h){\n";
    } else {
      // register bit holding local bit 0 per phase (16-byte pair accesses), -1 if none
      G.o << "template<int LR>__device__ __forceinline__ int pair_reg(const qsb::PhaseDesc*,int h)const{switch(h){";
      for (int h = 0; h < pd.nphase; ++h) {
        const PhaseDesc& ph = phs[pd.phase0 + h];
        int jr = -1;
        for (int j = 0; j < pd.r; ++j)
          if (ph.rbit[j] == 0) jr = j;
        if (jr >= 0) G.o << "case " << h << ":return " << jr << ";";
      }
      G.o << "default:return -1;}}\n";
      // group copies: physical offset and swizzled byte offset of item row v of thread 0
      {
        const int T = 1 << (pd.m - pd.r), V = 1 << (pd.r - 1);
        G.o << "template<int V>__device__ __forceinline__ void copy_offsets(uint64_t (&P)[V],uint32_t (&D)[V])const{";
        for (int v = 0; v < V; ++v) {
          const uint32_t lv = ((uint32_t)v * (uint32_t)T) << 1;
          uint64_t q = 0;
          for (int j = 0; j < pd.m; ++j)
            if ((lv >> j) & 1u) q |= 1ull << pd.sbit[j];
          G.o << "P[" << v << "]=" << q << "ull;D[" << v << "]=" << swz64(lv) * 8u << "u;";
        }
        G.o << "}\n";
      }
      // physical offset (amplitudes) and local bit of each register bit per phase (the last
      // phase stores straight to global memory)
      G.o << "template<int LR>__device__ __forceinline__ void phys_offsets(int h,uint64_t (&P)[LR],uint32_t (&L)[LR])"
          << "const{switch(h){";
      for (int h = 0; h < pd.nphase; ++h) {
        const PhaseDesc& ph = phs[pd.phase0 + h];
        G.o << "case " << h << ":";
        for (int j = 0; j < pd.r; ++j)
          G.o << "P[" << j << "]=" << (1ull << pd.sbit[ph.rbit[j]]) << "ull;L[" << j << "]=" << (1u << ph.rbit[j])
              << "u;";
        G.o << "break;";
      }
      G.o << "default:break;}}\n";
      G.o << "template<typename C,int LR>__device__ __forceinline__ uint32_t run("
          << "const uint8_t* prog,const qsb::PhaseDesc*,int,int h,C (&a)[1<<LR],uint64_t pb)const{constexpr int NR=1<<LR;"
          << "const float2* K=(const float2*)(prog+((const qsb::ProgramHeader*)prog)->off_coef);switch(h){\n";
    }
    for (int h = 0; h < pd.nphase; ++h) {
      const PhaseDesc& ph = phs[pd.phase0 + h];
      G.o << "case " << h << ":{\nfloat2 fa=make_float2(1.f,0.f);\n";
      G.used_fa = false;
      G.reset_masks();
      // Diagonal gates on fixed bits commute with every gate of the phase: their factors
      // are accumulated first, then folded into the register gate where that costs least
      // (else one multiply of every amplitude at the end of the phase).
      // gradient programs: the register bit of the lam bit (local bit 0)
      int A = -1;
      for (int j = 0; j < pd.r; ++j)
        if (ph.rbit[j] == 0) A = j;
      std::vector<int> pending;  // the phase's term accumulators not yet reduced
      auto term = [&](int gi) {
        const int k = ph.gate0 + gi;
        if (!grad || !prog.grad_gen[k]) return;
        gen_term(G, gis[k], prog.grad_gen[k], prog.grad_term[k] - t0, A, &pending);
        if ((int)pending.size() >= kTermBatch) gen_term_flush(G, &pending, std::max(1, nt));
      };
      // Z rotations on fixed bits: their terms are taken at the phase start (the registers are
      // untouched yet; Z of a fixed bit commutes with the phase) and all share the thread's sum
      // gb_ = sum_i Im(conj(lam_i) psi_i), signed by the bit.  For a bit that is uniform over the
      // warp (a group or warp-index bit) one warp sum gw_ of gb_ serves every such term.
      const int ntr = std::max(1, nt);
      bool have_base = false, have_wsum = false;
      auto fixed_z_term = [&](int gi) {
        const int k = ph.gate0 + gi;
        if (!grad || !prog.grad_gen[k]) return;
        const GateInstr& g = gis[k];
        if (prog.grad_gen[k] != 3) throw std::runtime_error("jit: an X or Y rotation on a fixed bit");
        if (A < 0) throw std::runtime_error("jit: the lam bit is not a register bit");
        const int P = g.a - kFixed, local = prog.grad_term[k] - t0;
        if (!have_base) {
          G.o << "float gb_=0.f;\n#pragma unroll\nfor(int i=0;i<NR;++i) if(!(i&" << (1 << A)
              << ")){const float2 p=a[i],l=a[i|" << (1 << A) << "];gb_+=l.x*p.y-l.y*p.x;}\n";
          have_base = true;
        }
        bool uniform = true;
        for (int j = 0; j < 5 && j < pd.m - pd.r; ++j)
          if (pd.sbit[ph.tbit[j]] == P) uniform = false;
        if (uniform) {
          if (!have_wsum) {
            G.o << "float gw_=gb_;gw_+=__shfl_xor_sync(0xffffffffu,gw_,16);gw_+=__shfl_xor_sync(0xffffffffu,gw_,8);"
                << "gw_+=__shfl_xor_sync(0xffffffffu,gw_,4);gw_+=__shfl_xor_sync(0xffffffffu,gw_,2);"
                << "gw_+=__shfl_xor_sync(0xffffffffu,gw_,1);\n";
            have_wsum = true;
          }
          G.o << "if((threadIdx.x&31u)==0u)ga[(threadIdx.x>>5)*" << ntr << "+" << local << "]+=(double)("
              << bitcond(P) << "?-gw_:gw_);\n";
        } else {
          G.o << "float gt" << local << "=" << bitcond(P) << "?-gb_:gb_;\n";
          pending.push_back(local);
          if ((int)pending.size() >= kTermBatch) gen_term_flush(G, &pending, ntr);
        }
      };
      for (int gi = 0; gi < ph.ngate; ++gi)
        if (fixed_diag(gis[ph.gate0 + gi])) {
          fixed_z_term(gi);
          gen_gate(G, gis[ph.gate0 + gi], pd, ph);
        }
      int absorber = -1;
      if (G.used_fa) {
        // packed kernels: only gates on register bit 0 (single-lane arithmetic) absorb; the
        // separate packed multiply costs two instructions per amplitude
        double best = packed ? 2.0 : 4.0;  // instructions per amplitude of the separate multiply
        for (int gi = 0; gi < ph.ngate; ++gi) {
          const GateInstr& gg = gis[ph.gate0 + gi];
          if (packed && gg.a != 0 && (gg.kind < GK_2Q_DENSE || gg.b != 0)) continue;
          Ent m[16];
          int d = 0;
          if (!absorber_matrix(G, gg, m, &d)) continue;
          const double added = Gen::fold_added(m, d);
          if (added < best) { best = added; absorber = gi; }
        }
      }
      for (int gi = 0; gi < ph.ngate; ++gi)
        if (!fixed_diag(gis[ph.gate0 + gi])) {
          term(gi);
          gen_gate(G, gis[ph.gate0 + gi], pd, ph, gi == absorber);
        }
      if (G.used_fa && absorber < 0) {
        Ent d;
        d.cls = 7;
        d.var = "fa";
        G.scale(d);
      }
      gen_term_flush(G, &pending, std::max(1, nt));
      // local bits left flipped by the phase's bit-flip frame
      G.o << "return 0u";
      for (int j = 0; j < pd.r; ++j)
        if (!G.mask[j].empty()) G.o << "|(" << G.mask[j] << "?" << (1u << ph.rbit[j]) << "u:0u)";
      G.o << ";}\n";
    }
    G.o << "default:break;}return 0u;}};\n";
    const std::string xs = G.o.str();
    G.o.swap(outer);
    G.o << "struct KP" << p << "{float2 k[" << std::max(1, G.kcount) << "];";
    if (!G.splats.empty()) G.o << "float2 s[" << G.splats.size() << "];";
    G.o << "};\n" << xs;
    if (splats_out) splats_out->push_back(G.splats);
    std::snprintf(kname, sizeof(kname), "qp_%016llx_%d", (unsigned long long)key, p);
    // blocks == 1: double-buffered group loads; blocks == 2: one buffer per block; blocks == 3:
    // two teams per block over three buffers.  The bound is the block size every pass of the
    // program is launched with (>= this pass's threads per team).  The pass's coefficients
    // are the by-value parameter kp (constant bank): the arithmetic reads them as operands,
    // with no load instruction and no register.
    const bool teams = cfg.blocks == 3;
    const int per_sm = teams ? 1 : cfg.blocks == 4 ? 2 : cfg.blocks;  // resident blocks per SM
    const bool all_active_g = (1 << (pd.m - pd.r)) == hdr->max_threads;
    if (grad) {
      // the block's terms in shared memory (zeroed before the pass body's first barrier),
      // added to the program's term array once at the end
      if (cfg.blocks != 2 || !all_active_g || pd.nphase == 0)
        throw std::runtime_error("jit: gradient programs run single-buffered blocks with every thread active");
      // one row of terms per warp (rows: max_threads / 32)
      const int ntr = std::max(1, nt), rows = hdr->max_threads / 32;
      if (hdr->max_threads % 32) throw std::runtime_error("jit: gradient programs need whole warps");
      G.o << "extern \"C\" __global__ void __launch_bounds__(" << hdr->max_threads << ",2) " << kname
          << "(const uint8_t* __restrict__ prog,float2* __restrict__ psi,unsigned* __restrict__ err,"
          << "double* __restrict__ gterm,const __grid_constant__ KP" << p << " kp){__shared__ double ga_["
          << rows * ntr << "];for(int j=threadIdx.x;j<" << rows * ntr << ";j+=blockDim.x)ga_[j]=0.0;const X" << p
          << " ex{&kp,ga_};qsb::pass_body_direct<float," << pd.r << ",X" << p << "," << pd.nphase << ">(ex,prog,psi,"
          << p << ");__syncthreads();for(int j=threadIdx.x;j<" << nt << ";j+=blockDim.x){double v=0.0;"
          << "for(int w=0;w<" << rows << ";++w)v+=ga_[w*" << ntr << "+j];if(v!=0.0)atomicAdd(gterm+" << t0
          << "+j,v);}}\n";
      continue;
    }
    G.o << "extern \"C\" __global__ void __launch_bounds__("
        << (teams ? 2 : 1) * hdr->max_threads << "," << per_sm << ") " << kname
        << "(const uint8_t* __restrict__ prog,float2* __restrict__ psi,unsigned* __restrict__ err,"
        << "const __grid_constant__ KP" << p << " kp){const X" << p << " ex{&kp};";
    const bool all_active = (1 << (pd.m - pd.r)) == hdr->max_threads;
    if (teams)
      G.o << "qsb::pass_body_teams<float," << pd.r << ",X" << p << "," << pd.nphase << ","
          << (!packed && all_active && pd.nphase > 0 ? "true" : "false") << ">(ex,prog,psi," << p << ",err,"
          << kDeviceWaitLimitNs << "ull);}\n";
    else if (cfg.blocks == 2 && !packed && all_active && pd.nphase > 0)
      G.o << "qsb::pass_body_direct<float," << pd.r << ",X" << p << "," << pd.nphase << ">(ex,prog,psi," << p
          << ");}\n";
    else
      G.o << "qsb::pass_body<float," << pd.r << ",X" << p << "," << (cfg.blocks != 2 ? "true" : "false") << ","
          << pd.nphase << ">(ex,prog,psi," << p << "," << p + 1 << ",nullptr,err,0ull);}\n";
  }
  return G.o.str();
}

namespace {

// NVRTC options; entry 3 is replaced by the include path of the device headers.  No line
// tables: they add a quarter to the compile time and nothing to the code.
constexpr int kNumOpts = 7;
const char* const kCompileOpts[kNumOpts] = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device",
                                            "-I<csrc>", "--extra-device-vectorization", "--disable-warnings",
                                            "--ptxas-options=-v"};

bool compile_source(const std::string& src, std::vector<char>* cubin, std::string* log, bool verbose = false) {
  Nvrtc& nv = nvrtc();
  void* prog = nullptr;
  if (nv.create(&prog, src.c_str(), "qsim_jit.cu", 0, nullptr, nullptr) != 0) {
    if (log) *log = "nvrtcCreateProgram failed";
    return false;
  }
  const std::string inc = "-I" + csrc_dir();
  const char* opts[kNumOpts];
  for (int i = 0; i < kNumOpts; ++i) opts[i] = kCompileOpts[i];
  opts[3] = inc.c_str();
  const int rc = nv.compile(prog, verbose ? kNumOpts : kNumOpts - 1, opts);
  size_t ls = 0;
  nv.log_size(prog, &ls);
  std::string lg(ls, '\0');
  if (ls) nv.log(prog, &lg[0]);
  if (log) *log = lg;
  bool ok = rc == 0;
  if (ok && cubin) {
    size_t cs = 0;
    nv.cubin_size(prog, &cs);
    cubin->resize(cs);
    nv.cubin(prog, cubin->data());
  }
  nv.destroy(&prog);
  return ok;
}

std::mutex g_mu;
std::list<std::shared_ptr<JitKernels>> g_cache;  // most recent first

// ---- compiled kernels kept on disk across processes -----------------------------------
// A cubin is stored under the FNV-1a hash of everything that determines it: the generated
// source, the device headers it includes, the compile options and the NVRTC version.
// $QSIM_JIT_CACHE names the directory ("0" or "off": no disk cache); by default
// $XDG_CACHE_HOME/qsim_b200/jit or ~/.cache/qsim_b200/jit.
uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ull) {
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

std::string read_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return std::string();
  std::ostringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

std::string disk_cache_dir() {
  const char* e = std::getenv("QSIM_JIT_CACHE");
  if (e) {
    if (!*e || !std::strcmp(e, "0") || !std::strcmp(e, "off")) return std::string();
    return e;
  }
  const char* x = std::getenv("XDG_CACHE_HOME");
  const char* home = std::getenv("HOME");
  std::string base = (x && *x) ? std::string(x) : (home && *home ? std::string(home) + "/.cache" : std::string());
  return base.empty() ? base : base + "/qsim_b200/jit";
}

bool make_dirs(const std::string& dir) {
  std::string cur;
  size_t i = 0;
  while (i <= dir.size()) {
    const size_t j = dir.find('/', i);
    cur = dir.substr(0, j == std::string::npos ? dir.size() : j);
    if (!cur.empty()) {
      struct stat st;
      if (stat(cur.c_str(), &st) != 0 && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return false;
    }
    if (j == std::string::npos) break;
    i = j + 1;
  }
  return true;
}

// the part of a kernel's cache key that does not depend on its source
uint64_t disk_key_base(const char* const* opts, int nopts) {
  static uint64_t base = 0;
  static std::once_flag once;
  std::call_once(once, [&] {
    std::string k = read_file(csrc_dir() + "/qsim.h") + read_file(csrc_dir() + "/pass_body.cuh");
    for (int i = 0; i < nopts; ++i) k += std::string("\n") + opts[i];
    int major = 0, minor = 0;
    if (nvrtc().version) nvrtc().version(&major, &minor);
    k += "\nnvrtc " + std::to_string(major) + "." + std::to_string(minor);
    base = fnv1a(k);
  });
  return base;
}

std::string disk_path(const std::string& dir, const std::string& src, uint64_t base) {
  char name[40];
  std::snprintf(name, sizeof(name), "/qp_%016llx.cubin", (unsigned long long)fnv1a(src, base));
  return dir + name;
}

bool disk_load(const std::string& path, std::vector<char>* cubin) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) return false;
  const std::streamsize n = f.tellg();
  if (n <= 0) return false;
  cubin->resize((size_t)n);
  f.seekg(0);
  return (bool)f.read(cubin->data(), n);
}

void disk_store(const std::string& path, const std::vector<char>& cubin) {
  const size_t slash = path.rfind('/');
  if (slash == std::string::npos || !make_dirs(path.substr(0, slash))) return;
  const std::string tmp = path + "." + std::to_string((long long)getpid()) + ".tmp";
  {
    std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
    if (!f) return;
    f.write(cubin.data(), (std::streamsize)cubin.size());
    if (!f) { std::remove(tmp.c_str()); return; }
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

}  // namespace

// Two teams need whole warps per team (named barriers count warps): programs whose team
// would be smaller than a warp run one buffer per block instead.
JitConfig jit_effective(const Program& prog, const JitConfig& cfg) {
  JitConfig e = cfg;
  const ProgramHeader* hdr = (const ProgramHeader*)prog.bytes.data();
  if (e.blocks == 3 && hdr->max_threads % 32 != 0) e.blocks = 2;
  return e;
}

bool jit_compile_check(const Program& prog, std::string* log, const JitConfig& cfg_in) {
  if (!nvrtc().ok) { if (log) *log = nvrtc().why; return false; }
  const JitConfig cfg = jit_effective(prog, cfg_in);
  const ProgramHeader* hdr = (const ProgramHeader*)prog.bytes.data();
  return compile_source(jit_source(prog, 0, hdr->npass, jit_key(prog, cfg), cfg), nullptr, log, true);
}

std::shared_ptr<JitKernels> jit_get(const Program& prog, const JitConfig& cfg_in) {
  std::string why;
  if (!jit_available(&why)) throw std::runtime_error("jit: " + why);
  const JitConfig cfg = jit_effective(prog, cfg_in);
  const uint64_t key = jit_key(prog, cfg);
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto it = g_cache.begin(); it != g_cache.end(); ++it)
      if ((*it)->key == key) {
        auto k = *it;
        g_cache.erase(it);
        g_cache.push_front(k);
        return k;
      }
  }
  const auto t0 = std::chrono::steady_clock::now();
  const ProgramHeader* hdr = (const ProgramHeader*)prog.bytes.data();
  const int npass = hdr->npass;
  unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nchunk = std::max(1, std::min<int>(npass, (int)std::min(hw, 32u)));
  std::vector<std::vector<char>> cubins(nchunk);
  std::vector<std::vector<std::vector<uint32_t>>> splats(nchunk);
  std::vector<std::string> logs(nchunk);
  std::vector<int> ok(nchunk, 0);
  std::vector<std::pair<int, int>> range(nchunk);
  for (int c = 0; c < nchunk; ++c) range[c] = {npass * c / nchunk, npass * (c + 1) / nchunk};
  const std::string dir = disk_cache_dir();
  const uint64_t base = dir.empty() ? 0 : disk_key_base(kCompileOpts, kNumOpts - 1);
  std::vector<int> hit(nchunk, 0);
  {
    std::vector<std::thread> th;
    for (int c = 0; c < nchunk; ++c)
      th.emplace_back([&, c] {
        try {
          const std::string src = jit_source(prog, range[c].first, range[c].second, key, cfg, &splats[c]);
          const std::string path = dir.empty() ? std::string() : disk_path(dir, src, base);
          if (!path.empty() && disk_load(path, &cubins[c])) {
            ok[c] = 1;
            hit[c] = 1;
            return;
          }
          ok[c] = compile_source(src, &cubins[c], &logs[c]);
          if (ok[c] && !path.empty()) disk_store(path, cubins[c]);
        } catch (const std::exception& e) {
          logs[c] = e.what();
        }
      });
    for (auto& t : th) t.join();
  }
  for (int c = 0; c < nchunk; ++c)
    if (!ok[c]) throw std::runtime_error("jit: NVRTC compilation failed:\n" + logs[c].substr(0, 4000));
  auto k = std::make_shared<JitKernels>();
  k->key = key;
  k->blocks = cfg.blocks;
  k->grad = !prog.grad_gen.empty();
  for (int c = 0; c < nchunk; ++c) k->disk_hits += hit[c];
  k->chunks = nchunk;
  k->cbase.resize(npass);
  k->ccount.resize(npass);
  for (int p = 0; p < npass; ++p) pass_coef_range(prog.bytes.data(), p, &k->cbase[p], &k->ccount[p]);
  for (int c = 0; c < nchunk; ++c)
    for (auto& v : splats[c]) k->splats.push_back(std::move(v));
  if ((int)k->splats.size() != npass) throw std::runtime_error("jit: parameter layout of a pass missing");
  Driver& d = driver();
  char kname[64];
  for (int c = 0; c < nchunk; ++c) {
    CUmodule mod;
    if (d.load(&mod, cubins[c].data()) != CUDA_SUCCESS) throw std::runtime_error("jit: cuModuleLoadData failed");
    k->modules.push_back(mod);
    for (int p = range[c].first; p < range[c].second; ++p) {
      std::snprintf(kname, sizeof(kname), "qp_%016llx_%d", (unsigned long long)key, p);
      CUfunction f;
      if (d.get_fn(&f, mod, kname) != CUDA_SUCCESS) throw std::runtime_error("jit: kernel not found");
      // two teams: three complex64 groups of at most 2^13 amplitudes
      const int dyn = cfg.blocks == 3 ? 3 * (8 << 13) : kMaxDynamicSmem;
      if (d.set_attr(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, dyn) != CUDA_SUCCESS)
        throw std::runtime_error("jit: cannot raise the shared-memory limit");
      k->functions.push_back(f);
    }
  }
  k->compile_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache.push_front(k);
  while (g_cache.size() > 8) g_cache.pop_back();
  return k;
}

namespace {
// compiles started by jit_try_get and not yet collected, by kernel key (guarded by g_mu)
std::unordered_map<uint64_t, std::shared_future<std::shared_ptr<JitKernels>>> g_inflight;
}  // namespace

std::shared_ptr<JitKernels> jit_try_get(const Program& prog, const JitConfig& cfg_in) {
  std::string why;
  if (!jit_available(&why)) throw std::runtime_error("jit: " + why);
  const JitConfig cfg = jit_effective(prog, cfg_in);
  const uint64_t key = jit_key(prog, cfg);
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto it = g_cache.begin(); it != g_cache.end(); ++it)
    if ((*it)->key == key) {
      auto k = *it;
      g_cache.erase(it);
      g_cache.push_front(k);
      return k;
    }
  auto it = g_inflight.find(key);
  if (it != g_inflight.end()) {
    if (it->second.wait_for(std::chrono::seconds(0)) != std::future_status::ready) return nullptr;
    auto fut = it->second;
    g_inflight.erase(it);
    return fut.get();  // the compiled kernels (also in the cache now), or the compile's error
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("jit: no current device");
  Program copy = prog;
  // the compiling thread makes the same device current (its driver calls load the modules there)
  g_inflight.emplace(key, std::async(std::launch::async, [copy, cfg_in, dev]() {
                            if (cudaSetDevice(dev) != cudaSuccess) throw std::runtime_error("jit: cannot set the device");
                            return jit_get(copy, cfg_in);
                          }).share());
  return nullptr;
}

void jit_wait_all() {
  std::vector<std::shared_future<std::shared_ptr<JitKernels>>> futs;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto& kv : g_inflight) futs.push_back(kv.second);
  }
  for (auto& f : futs) f.wait();
}

cudaError_t jit_launch(const JitKernels& k, int p, const uint8_t* d_prog, const void* host_coef, void* psi,
                       unsigned* err, int threads, size_t smem_double, int sms, cudaStream_t stream, double* gterm) {
  static const float2 kNone = {0.f, 0.f};
  // the driver copies the parameter block (the pass's coefficients) at the launch call
  const float2* hc = (const float2*)host_coef;
  const void* kp = k.ccount[p] > 0 ? (const void*)(hc + k.cbase[p]) : (const void*)&kNone;
  const std::vector<uint32_t>& sp = k.splats[p];
  thread_local std::vector<float2> block;
  if (!sp.empty()) {
    // coefficient range, then the splats {v, v} of the packed arithmetic
    const int nk = std::max(1, k.ccount[p]);
    block.assign((size_t)nk + sp.size(), float2{0.f, 0.f});
    for (int i = 0; i < k.ccount[p]; ++i) block[i] = hc[k.cbase[p] + i];
    for (size_t j = 0; j < sp.size(); ++j) {
      const float2 c = hc[sp[j] >> 2];
      const unsigned comp = sp[j] & 3u;
      const float v = comp == 0 ? c.x : comp == 1 ? c.y : comp == 2 ? -c.x : -c.y;
      block[nk + j] = float2{v, v};
    }
    kp = block.data();
  }
  void* args[] = {(void*)&d_prog, (void*)&psi, (void*)&err, const_cast<void*>(kp), nullptr};
  if (k.grad) {
    if (!gterm) return cudaErrorInvalidValue;
    args[3] = (void*)&gterm;
    args[4] = const_cast<void*>(kp);
  }
  const unsigned smem = (unsigned)jit_smem_bytes(k.blocks, smem_double);
  const bool teams = k.blocks == 3;
  const int per_sm = teams ? 1 : k.blocks == 4 ? 2 : k.blocks;
  CUresult r = driver().launch((CUfunction)k.functions[p], (unsigned)(per_sm * sms), 1, 1,
                               (unsigned)((teams ? 2 : 1) * threads), 1, 1, smem, (CUstream)stream, args, nullptr);
  if (r == CUDA_SUCCESS) return cudaSuccess;
  // launch-time rejections (configuration) are reported as such, not as a kernel failure
  if (r == CUDA_ERROR_INVALID_VALUE || r == CUDA_ERROR_LAUNCH_OUT_OF_RESOURCES) return cudaErrorInvalidConfiguration;
  return cudaErrorLaunchFailure;
}

}  // namespace qsb
