// pmb_jit.cu — per-signature fused group-by kernels compiled at run time with NVRTC.
//
// The reference generates a fused aggregate kernel per query signature at run time and caches
// the compiled pipeline (crates/polars-metal-kernels/src/aggregate_fused/emitter.rs:189-393,
// cache.rs:81-208). This is the B200 counterpart for the whole filter -> group_by -> aggregate
// row program: the host emits straight-line CUDA for the query's predicate, key and record
// updates (literal offsets and dtypes), NVRTC compiles it for sm_100a together with the kernel
// skeleton (pmb_jit_skeleton.cuh), and the cubin is cached by source text for the process.
// NVRTC is loaded with dlopen; if it is missing or a compile fails, the caller runs the prebuilt
// generic kernel instead (same results, slower), so a JIT problem never changes results.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "pmb_groupby.h"
#include "pmb_jit.h"

namespace {

#include "pmb_jit_sources.inc"  // kDeviceHeader, kSkeleton, ... (generated from the .cuh files by the build)

// ---------------------------------------------------------------------------- NVRTC via dlopen
typedef int nvrtcResult_t;
typedef struct _nvrtcProgram* nvrtcProgram_t;
struct Nvrtc {
  bool tried = false, ok = false;
  nvrtcResult_t (*create)(nvrtcProgram_t*, const char*, const char*, int, const char* const*, const char* const*);
  nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char* const*);
  nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t*);
  nvrtcResult_t (*log)(nvrtcProgram_t, char*);
  nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t*);
  nvrtcResult_t (*cubin)(nvrtcProgram_t, char*);
  nvrtcResult_t (*destroy)(nvrtcProgram_t*);
};

Nvrtc g_nv;
std::mutex g_mu;
std::unordered_map<std::string, cudaKernel_t> g_cache;
std::unordered_map<std::string, std::string> g_fail;  // source -> compile error (do not retry)

bool load_nvrtc() {
  if (g_nv.tried) return g_nv.ok;
  g_nv.tried = true;
  const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
  void* lib = nullptr;
  for (const char* n : names)
    if ((lib = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
  if (!lib) return false;
  g_nv.create = (decltype(g_nv.create))dlsym(lib, "nvrtcCreateProgram");
  g_nv.compile = (decltype(g_nv.compile))dlsym(lib, "nvrtcCompileProgram");
  g_nv.log_size = (decltype(g_nv.log_size))dlsym(lib, "nvrtcGetProgramLogSize");
  g_nv.log = (decltype(g_nv.log))dlsym(lib, "nvrtcGetProgramLog");
  g_nv.cubin_size = (decltype(g_nv.cubin_size))dlsym(lib, "nvrtcGetCUBINSize");
  g_nv.cubin = (decltype(g_nv.cubin))dlsym(lib, "nvrtcGetCUBIN");
  g_nv.destroy = (decltype(g_nv.destroy))dlsym(lib, "nvrtcDestroyProgram");
  g_nv.ok = g_nv.create && g_nv.compile && g_nv.log_size && g_nv.log && g_nv.cubin_size && g_nv.cubin && g_nv.destroy;
  return g_nv.ok;
}

// ---------------------------------------------------------------------------- code generation
const char* ctype(int dt) {
  switch (dt) {
    case PMB_BOOL: return "bool";
    case PMB_I8: return "signed char";
    case PMB_I16: return "short";
    case PMB_I32: return "int";
    case PMB_I64: return "long long";
    case PMB_U8: return "unsigned char";
    case PMB_U16: return "unsigned short";
    case PMB_U32: return "unsigned int";
    case PMB_U64: return "unsigned long long";
    case PMB_F32: return "float";
    default: return "double";
  }
}

std::string lit_i64(long long v) {
  if (v == (long long)0x8000000000000000LL) return "(-9223372036854775807LL - 1LL)";
  return std::to_string(v) + "LL";
}
std::string lit_f64(double v) {
  if (v != v) return "__longlong_as_double(0x7FF8000000000000LL)";
  if (v == 1.0 / 0.0) return "__longlong_as_double(0x7FF0000000000000LL)";
  if (v == -1.0 / 0.0) return "__longlong_as_double((long long)0xFFF0000000000000ULL)";
  char buf[64];
  snprintf(buf, sizeof buf, "%a", v);  // exact hexadecimal literal
  return buf;
}

struct Gen {
  const DQuery& q;
  const JitPlan& P;
  std::ostringstream o;
  std::vector<bool> need_val, need_bits, need_valid, field_col, pred_col, key_col;
  JitSLayout S;
  int tmp = 0;

  Gen(const DQuery& q_, const JitPlan& p_) : q(q_), P(p_) {
    pmb_jit_slayout(q, &S);
    pred_col.assign(q.n_cols, false);
    key_col.assign(q.n_cols, false);
    need_val.assign(q.n_cols, false);
    need_bits.assign(q.n_cols, false);
    need_valid.assign(q.n_cols, false);
    field_col.assign(q.n_cols, false);
  }

  std::string v(int c) { return "r.v" + std::to_string(c); }
  std::string ok(int c) { return q.col[c].valid ? "r.ok" + std::to_string(c) : std::string("true"); }
  // validity of column c in a row the filter kept: the filter may already imply it
  std::string okk(int c) { return ((q.valid_if_kept >> c) & 1u) ? std::string("true") : ok(c); }

  void mark_leaf(const DLeaf& L) {
    if (L.col >= 0) need_val[L.col] = need_valid[L.col] = pred_col[L.col] = true;
  }
  void mark() {
    for (int i = 0; i < q.prog.n_terms; i++) {
      const DTerm& T = q.prog.term[i];
      mark_leaf(T.lhs.a);
      if (T.lhs.arith >= 0) mark_leaf(T.lhs.b);
      if (T.kind == T_CMP) {
        mark_leaf(T.rhs.a);
        if (T.rhs.arith >= 0) mark_leaf(T.rhs.b);
      }
    }
    for (int k = 0; k < q.n_keys; k++) {
      need_bits[q.key[k].col] = need_valid[q.key[k].col] = key_col[q.key[k].col] = true;
      need_val[q.key[k].col] = true;
    }
    for (int f = 0; f < q.n_fields; f++) {
      if (q.field[f].kind == F_LEN) continue;
      int c = q.field[f].col;
      need_val[c] = need_valid[c] = field_col[c] = true;
    }
  }

  std::string load_val(int c) {
    const DCol& C = q.col[c];
    std::string d = std::to_string(P.doff[c]);
    if (C.dtype == PMB_BOOL) return "(((st[" + d + " + (lr >> 3)] >> (lr & 7)) & 1) != 0)";
    return "reinterpret_cast<const " + std::string(ctype(C.dtype)) + "*>(st + " + d + ")[lr]";
  }
  std::string load_valid(int c) {
    // the bit of row lr from the unit's 32-bit validity word of rows lr & ~31 (voff is 16-aligned)
    std::string vo = std::to_string(P.voff[c]);
    return "(((reinterpret_cast<const unsigned int*>(st + " + vo + ")[lr >> 5] >> (lr & 31)) & 1u) != 0u)";
  }

  void row_struct() {
    o << "struct JRow {\n";
    for (int c = 0; c < q.n_cols; c++) {
      if (need_val[c]) o << "  " << ctype(q.col[c].dtype) << " v" << c << ";\n";
      if (need_valid[c] && q.col[c].valid) o << "  bool ok" << c << ";\n";
    }
    o << "};\n";
  }

  // leaf value in compare dtype dt: returns (value expr, valid expr)
  std::pair<std::string, std::string> leaf(const DLeaf& L, int dt) {
    if (L.col < 0) return {dt == PMB_F64 ? lit_f64(L.f) : lit_i64(L.i), "true"};
    std::string x = dt == PMB_F64 ? "((double)" + v(L.col) + ")" : "((long long)" + v(L.col) + ")";
    return {x, ok(L.col)};
  }

  // emits statements for an operand; returns (value var, valid var)
  std::pair<std::string, std::string> operand(const DOperand& op, int dt, std::ostringstream& b) {
    auto a = leaf(op.a, dt);
    if (op.arith < 0) return a;
    auto c = leaf(op.b, dt);
    int id = tmp++;
    std::string xv = "x" + std::to_string(id), ov = "o" + std::to_string(id);
    const char* T = dt == PMB_F64 ? "double" : "long long";
    b << "    bool " << ov << " = " << a.second << " && " << c.second << ";\n";
    if (dt == PMB_F64) {
      switch (op.arith) {
        case PMB_ARITH_ADD: b << "    " << T << " " << xv << " = " << a.first << " + " << c.first << ";\n"; break;
        case PMB_ARITH_SUB: b << "    " << T << " " << xv << " = " << a.first << " - " << c.first << ";\n"; break;
        case PMB_ARITH_MUL: b << "    " << T << " " << xv << " = " << a.first << " * " << c.first << ";\n"; break;
        case PMB_ARITH_TRUEDIV: b << "    " << T << " " << xv << " = " << a.first << " / " << c.first << ";\n"; break;
        case PMB_ARITH_FLOORDIV:
          b << "    " << T << " " << xv << " = floor(" << a.first << " / " << c.first << ");\n";
          break;
        default: b << "    " << T << " " << xv << " = j_mod_f(" << a.first << ", " << c.first << ");\n"; break;
      }
    } else {
      switch (op.arith) {
        case PMB_ARITH_ADD:
        case PMB_ARITH_SUB:
        case PMB_ARITH_MUL: {
          const char* sym = op.arith == PMB_ARITH_ADD ? "+" : (op.arith == PMB_ARITH_SUB ? "-" : "*");
          b << "    " << T << " " << xv << " = (long long)((unsigned long long)" << a.first << " " << sym
            << " (unsigned long long)" << c.first << ");\n";
          break;
        }
        case PMB_ARITH_FLOORDIV:
          b << "    " << T << " " << xv << " = j_fdiv_i(" << a.first << ", " << c.first << ", " << ov << ");\n";
          break;
        default:
          b << "    " << T << " " << xv << " = j_mod_i(" << a.first << ", " << c.first << ", " << ov << ");\n";
          break;
      }
    }
    return {xv, ov};
  }

  // "x is a multiple of d" for a signed 64-bit x and a literal d != 0 without a division: with
  // |d| = 2^k * o (o odd), the low k bits of x are zero and, for o > 1, x * o^-1 + c <= 2c modulo
  // 2^64 where c = floor((2^63 - 1) / o) (the multiplicative-inverse divisibility test of Granlund
  // and Montgomery, 1994, in its signed form; Lemire, Kaser and Kurz, 2019)
  static std::string divisible(const std::string& x, long long d) {
    unsigned long long a = d < 0 ? 0ULL - (unsigned long long)d : (unsigned long long)d;
    int k = 0;
    while (((a >> k) & 1ULL) == 0ULL) k++;
    const unsigned long long o = a >> k;
    std::string e = "(";
    if (k > 0) e += "((unsigned long long)(" + x + ") & " + std::to_string((1ULL << k) - 1ULL) + "ULL) == 0ULL";
    if (o > 1) {
      unsigned long long inv = o;  // Newton iteration for the inverse modulo 2^64 (5 steps from 3 bits)
      for (int i = 0; i < 5; i++) inv *= 2ULL - o * inv;
      const unsigned long long c = 0x7FFFFFFFFFFFFFFFULL / o;
      if (k > 0) e += " && ";
      e += "((unsigned long long)(" + x + ") * " + std::to_string(inv) + "ULL + " + std::to_string(c) + "ULL) <= " +
           std::to_string(2 * c) + "ULL";
    }
    if (k == 0 && o == 1) e += "true";
    return e + ")";
  }

  std::string predicate(std::ostringstream& b) {
    const DProgram& PR = q.prog;
    if (PR.n_ops == 0) return "true";
    std::vector<std::pair<std::string, std::string>> stack;  // (T, F) expressions
    for (int i = 0; i < PR.n_ops; i++) {
      int op = PR.ops[i];
      if (op >= 0) {
        const DTerm& T = PR.term[op];
        std::string t = "t" + std::to_string(op), f = "f" + std::to_string(op);
        switch (T.kind) {
          case T_CMP: {
            // `x % c == 0` / `!= 0` with an integer literal c: whether the remainder is zero does
            // not depend on the sign convention, so C's truncated remainder (a multiply-based
            // divisibility test for a constant divisor) gives the floor-mod verdict; the divisor
            // is not zero, so the remainder is valid exactly when x is
            if (T.dtype != PMB_F64 && (T.op == PMB_CMP_EQ || T.op == PMB_CMP_NE) && T.lhs.arith == PMB_ARITH_MOD &&
                T.lhs.b.col < 0 && T.lhs.b.i != 0 && T.lhs.b.i != -1 && T.rhs.arith < 0 && T.rhs.a.col < 0 &&
                T.rhs.a.i == 0) {
              auto x = leaf(T.lhs.a, T.dtype);
              b << "    bool " << t << "v = " << x.second << ";\n";
              b << "    bool " << t << "c = " << (T.op == PMB_CMP_EQ ? "" : "!") << divisible(x.first, T.lhs.b.i) << ";\n";
              b << "    bool " << t << " = " << t << "v && " << t << "c, " << f << " = " << t << "v && !" << t << "c;\n";
              break;
            }
            auto l = operand(T.lhs, T.dtype, b);
            auto r = operand(T.rhs, T.dtype, b);
            const char* sym[] = {"==", "!=", "<", "<=", ">", ">="};
            b << "    bool " << t << "v = " << l.second << " && " << r.second << ";\n";
            b << "    bool " << t << "c = " << l.first << " " << sym[T.op] << " " << r.first << ";\n";
            b << "    bool " << t << " = " << t << "v && " << t << "c, " << f << " = " << t << "v && !" << t << "c;\n";
            break;
          }
          case T_BOOLCOL: {
            int c = T.lhs.a.col;
            b << "    bool " << t << " = " << ok(c) << " && " << v(c) << ", " << f << " = " << ok(c) << " && !" << v(c)
              << ";\n";
            break;
          }
          case T_ISNULL:
          case T_ISNOTNULL: {
            int c = T.lhs.a.col;
            std::string isnull = "!(" + ok(c) + ")";
            if (T.kind == T_ISNULL) b << "    bool " << t << " = " << isnull << ", " << f << " = !" << t << ";\n";
            else b << "    bool " << t << " = !(" << isnull << "), " << f << " = !" << t << ";\n";
            break;
          }
          default:
            b << "    bool " << t << " = " << (T.lhs.a.i ? "true" : "false") << ", " << f << " = !" << t << ";\n";
        }
        stack.push_back({t, f});
      } else if (op == OP_NOT) {
        std::swap(stack.back().first, stack.back().second);
      } else {
        auto y = stack.back();
        stack.pop_back();
        auto x = stack.back();
        stack.pop_back();
        if (op == OP_AND) stack.push_back({"(" + x.first + " && " + y.first + ")", "(" + x.second + " || " + y.second + ")"});
        else stack.push_back({"(" + x.first + " || " + y.first + ")", "(" + x.second + " && " + y.second + ")"});
      }
    }
    return stack.back().first;
  }

  std::string raw_bits(int c) {
    switch (q.col[c].dtype) {
      case PMB_BOOL: return "(unsigned long long)(" + v(c) + " ? 1u : 0u)";
      case PMB_I8: case PMB_U8: return "(unsigned long long)(unsigned char)" + v(c);
      case PMB_I16: case PMB_U16: return "(unsigned long long)(unsigned short)" + v(c);
      case PMB_I32: case PMB_U32: return "(unsigned long long)(unsigned int)" + v(c);
      case PMB_F32: return "(unsigned long long)__float_as_uint(" + v(c) + ")";
      case PMB_F64: return "(unsigned long long)__double_as_longlong(" + v(c) + ")";
      default: return "(unsigned long long)" + v(c);
    }
  }

  // value of a field's column in the field's arithmetic type
  std::string fval(const DField& F) {
    int c = F.col, dt = q.col[c].dtype;
    switch (F.kind) {
      case F_SUM_DD: return "(double)" + v(c);
      case F_SUM_I:
        if (dt == PMB_BOOL) return "(unsigned long long)(" + v(c) + " ? 1u : 0u)";
        if (pmb_is_signed(dt)) return "(unsigned long long)(long long)" + v(c);
        return "(unsigned long long)" + v(c);
      case F_MIN_I:
      case F_MAX_I:
        if (dt == PMB_BOOL) return "(long long)(" + v(c) + " ? 1 : 0)";
        return "(long long)" + v(c);
      case F_MIN_U:
      case F_MAX_U: return "(unsigned long long)" + v(c);
      case F_MIN_F: return "j_minkey((double)" + v(c) + ")";
      default: return "j_maxkey((double)" + v(c) + ")";
    }
  }

  std::string at(int off, const char* T) { return "reinterpret_cast<" + std::string(T) + "*>(rec + " + std::to_string(off) + ")"; }

  // ---- global-table record (layout of the plan: u64 words, shared with the prebuilt kernels)
  void apply_global(std::ostringstream& b) {
    // pack 32-bit counters sharing a 64-bit word into one add
    std::vector<std::pair<int, std::string>> words;  // (word offset, increment expression)
    for (int i = 0; i < q.n_fields; i++) {
      const DField& F = q.field[i];
      std::string okc = F.kind == F_LEN ? std::string("true") : okk(F.col);
      if (F.kind == F_LEN || F.kind == F_CNT) {
        std::string inc = F.kind == F_LEN ? "1ULL" : "(" + okc + " ? 1ULL : 0ULL)";
        int w = F.off & ~7;
        std::string sh = (F.off & 4) ? " << 32" : "";
        bool found = false;
        for (auto& p : words)
          if (p.first == w) {
            p.second += " + (" + inc + sh + ")";
            found = true;
          }
        if (!found) words.push_back({w, "(" + inc + sh + ")"});
        continue;
      }
      b << "  if (" << okc << ") {\n";
      switch (F.kind) {
        case F_SUM_FX: {
          std::string slot = std::to_string(F.fx_slot);
          b << "    double xv = (double)" << v(F.col) << ";\n    unsigned fl = pmb_fx_flag(xv);\n";
          b << "    if (fl) pmb_rec_or32(rec, " << F.off + 16 << ", fl);\n";
          b << "    else if (pmb_fx_in_range(xv, P.fx_e[" << slot << "])) {\n      unsigned long long w0, w1;\n";
          b << "      pmb_fx_words(xv, P.fx[" << slot << "], w0, w1);\n";
          b << "      if (w0) pmb_red_add(" << at(F.off, "unsigned long long") << ", w0);\n";
          b << "      if (w1) pmb_red_add(" << at(F.off + 8, "unsigned long long") << ", w1);\n    }\n";
          break;
        }
        case F_SUM_DD:
          b << "    dd_atomic_add(" << at(F.off, "double") << ", " << at(F.off + 8, "double") << ", " << fval(F) << ");\n";
          break;
        case F_SUM_I: b << "    pmb_red_add(" << at(F.off, "unsigned long long") << ", " << fval(F) << ");\n"; break;
        default: {
          bool mn = F.kind == F_MIN_I || F.kind == F_MIN_U || F.kind == F_MIN_F;
          const char* T = (F.kind == F_MIN_U || F.kind == F_MAX_U) ? "unsigned long long" : "long long";
          // no read first: cold keys rarely skip an update, and a reduction (red) does not wait
          b << "    " << (mn ? "pmb_red_min(" : "pmb_red_max(") << at(F.off, T) << ", (" << T << ")(" << fval(F) << "));\n";
        }
      }
      b << "  }\n";
    }
    for (auto& p : words)
      b << "  pmb_red_add(reinterpret_cast<unsigned long long*>(rec + " << p.first << "), " << p.second << ");\n";
  }

  // ---- shared-memory record: native 32-bit atomics and 64-bit min/max only
  void apply_shared(std::ostringstream& b) {
    for (int i = 0; i < q.n_fields; i++) {
      const DField& F = q.field[i];
      const int so = S.off[i];
      if (F.kind == F_LEN) {
        b << "  atomicAdd(" << at(so, "unsigned int") << ", 1u);\n";
        continue;
      }
      b << "  if (" << okk(F.col) << ") {\n";
      switch (F.kind) {
        case F_CNT: b << "    atomicAdd(" << at(so, "unsigned int") << ", 1u);\n"; break;
        case F_SUM_FX: {
          std::string slot = std::to_string(F.fx_slot);
          b << "    double xv = (double)" << v(F.col) << ";\n    unsigned fl = pmb_fx_flag(xv);\n";
          b << "    if (fl) { if ((*reinterpret_cast<volatile unsigned int*>(rec + " << so + 12 << ") & fl) != fl) atomicOr("
            << at(so + 12, "unsigned int") << ", fl); }\n";
          b << "    else if (pmb_fx_in_range(xv, P.fx_e[" << slot << "])) {\n      unsigned long long a, b_, c;\n";
          b << "      pmb_fx_split(xv, P.fx[" << slot << "], a, b_, c);\n";
          b << "      pmb_s_add96(" << at(so, "unsigned int") << ", (unsigned)a, (unsigned)b_, (unsigned)c);\n    }\n";
          break;
        }
        case F_SUM_I:
          b << "    unsigned long long x = " << fval(F) << ";\n    pmb_s_add64(" << at(so, "unsigned int")
            << ", (unsigned)x, (unsigned)(x >> 32));\n";
          break;
        case F_SUM_DD:
          b << "    dd_atomic_add(" << at(so, "double") << ", " << at(so + 8, "double") << ", " << fval(F) << ");\n";
          break;
        default: {
          bool mn = F.kind == F_MIN_I || F.kind == F_MIN_U || F.kind == F_MIN_F;
          const char* T = (F.kind == F_MIN_U || F.kind == F_MAX_U) ? "unsigned long long" : "long long";
          b << "    " << T << " val = " << fval(F) << ";\n";
          b << "    if (val " << (mn ? "<" : ">") << " *reinterpret_cast<volatile " << T << "*>(rec + " << so << ")) "
            << (mn ? "atomicMin(" : "atomicMax(") << at(so, T) << ", val);\n";
        }
      }
      b << "  }\n";
    }
  }

  // d += s for shared-memory records with one owner
  void sfold(std::ostringstream& b) {
    for (int i = 0; i < q.n_fields; i++) {
      const DField& F = q.field[i];
      std::string d = std::to_string(S.off[i]);
      auto U = [&](int off) { return "reinterpret_cast<unsigned int*>(d + " + std::to_string(off) + ")"; };
      auto CU = [&](int off) { return "reinterpret_cast<const unsigned int*>(s + " + std::to_string(off) + ")"; };
      switch (F.kind) {
        case F_LEN:
        case F_CNT: b << "  *" << U(S.off[i]) << " += *" << CU(S.off[i]) << ";\n"; break;
        case F_SUM_FX:
          b << "  pmb_s_fold96(" << U(S.off[i]) << ", " << CU(S.off[i]) << ");\n";
          b << "  *" << U(S.off[i] + 12) << " |= *" << CU(S.off[i] + 12) << ";\n";
          break;
        case F_SUM_I: b << "  pmb_s_fold64(" << U(S.off[i]) << ", " << CU(S.off[i]) << ");\n"; break;
        case F_SUM_DD:
          b << "  dd_plain_add(reinterpret_cast<double*>(d + " << d << "), reinterpret_cast<double*>(d + " << S.off[i] + 8
            << "), *reinterpret_cast<const double*>(s + " << d << "));\n";
          b << "  *reinterpret_cast<double*>(d + " << S.off[i] + 8 << ") += *reinterpret_cast<const double*>(s + "
            << S.off[i] + 8 << ");\n";
          break;
        default: {
          bool mn = F.kind == F_MIN_I || F.kind == F_MIN_U || F.kind == F_MIN_F;
          const char* T = (F.kind == F_MIN_U || F.kind == F_MAX_U) ? "unsigned long long" : "long long";
          b << "  { " << T << " x = *reinterpret_cast<const " << T << "*>(s + " << d << ");\n";
          b << "    if (x " << (mn ? "<" : ">") << " *reinterpret_cast<" << T << "*>(d + " << d << ")) *reinterpret_cast<"
            << T << "*>(d + " << d << ") = x; }\n";
        }
      }
    }
  }

  // shared-memory record s into global-table record d
  void merge_sg(std::ostringstream& b) {
    for (int i = 0; i < q.n_fields; i++) {
      const DField& F = q.field[i];
      const int so = S.off[i];
      std::string gd = std::to_string(F.off);
      auto CU = [&](int off) { return "*reinterpret_cast<const unsigned int*>(s + " + std::to_string(off) + ")"; };
      auto GU64 = [&](int off) { return "reinterpret_cast<unsigned long long*>(d + " + std::to_string(off) + ")"; };
      switch (F.kind) {
        case F_LEN:
        case F_CNT:
          b << "  { unsigned int x = " << CU(so) << "; if (x) pmb_rec_add32(d, " << gd << ", x); }\n";
          break;
        case F_SUM_FX:
          // the 96-bit partial P: its low 32 bits, and P >> 32 as a signed 64-bit word
          b << "  { unsigned fl = " << CU(so + 12) << "; if (fl) pmb_rec_or32(d, " << F.off + 16 << ", fl);\n";
          b << "    unsigned w0 = " << CU(so) << ";\n    unsigned long long hi = ((unsigned long long)" << CU(so + 8)
            << " << 32) | " << CU(so + 4) << ";\n";
          b << "    if (w0) pmb_red_add(" << GU64(F.off) << ", (unsigned long long)w0);\n";
          b << "    if (hi) pmb_red_add(" << GU64(F.off + 8) << ", hi); }\n";
          break;
        case F_SUM_I:
          b << "  { unsigned long long x = ((unsigned long long)" << CU(so + 4) << " << 32) | " << CU(so)
            << "; if (x) pmb_red_add(" << GU64(F.off) << ", x); }\n";
          break;
        case F_SUM_DD:
          b << "  { double hi = *reinterpret_cast<const double*>(s + " << so << "), lo = *reinterpret_cast<const double*>(s + "
            << so + 8 << ");\n";
          b << "    if (hi != 0.0) dd_atomic_add(reinterpret_cast<double*>(d + " << gd << "), reinterpret_cast<double*>(d + "
            << F.off + 8 << "), hi);\n";
          b << "    if (lo != 0.0) atomicAdd(reinterpret_cast<double*>(d + " << F.off + 8 << "), lo); }\n";
          break;
        default: {
          bool mn = F.kind == F_MIN_I || F.kind == F_MIN_U || F.kind == F_MIN_F;
          bool uns = F.kind == F_MIN_U || F.kind == F_MAX_U;
          const char* T = uns ? "unsigned long long" : "long long";
          std::string ident = uns ? (mn ? "0xFFFFFFFFFFFFFFFFULL" : "0ULL")
                                  : (mn ? "0x7FFFFFFFFFFFFFFFLL" : "(long long)0x8000000000000000ULL");
          b << "  { " << T << " x = *reinterpret_cast<const " << T << "*>(s + " << so << ");\n";
          b << "    if (x != " << ident << ") " << (mn ? "pmb_red_min" : "pmb_red_max") << "(reinterpret_cast<" << T
            << "*>(d + " << gd << "), x); }\n";
        }
      }
    }
  }

  // shared-memory record s written as a global-table record d (plain stores: d is not shared)
  void store_sg(std::ostringstream& b) {
    for (int i = 0; i < q.n_fields; i++) {
      const DField& F = q.field[i];
      const int so = S.off[i];
      auto CU = [&](int off) { return "(*reinterpret_cast<const unsigned int*>(s + " + std::to_string(off) + "))"; };
      auto D = [&](const char* T, int off) {
        return "*reinterpret_cast<" + std::string(T) + "*>(d + " + std::to_string(off) + ")";
      };
      switch (F.kind) {
        case F_LEN:
        case F_CNT: b << "  " << D("unsigned int", F.off) << " = " << CU(so) << ";\n"; break;
        case F_SUM_FX:
          b << "  " << D("unsigned long long", F.off) << " = (unsigned long long)" << CU(so) << ";\n";
          b << "  " << D("unsigned long long", F.off + 8) << " = ((unsigned long long)" << CU(so + 8) << " << 32) | "
            << CU(so + 4) << ";\n";
          b << "  " << D("unsigned int", F.off + 16) << " = " << CU(so + 12) << ";\n";
          break;
        case F_SUM_I:
          b << "  " << D("unsigned long long", F.off) << " = ((unsigned long long)" << CU(so + 4) << " << 32) | " << CU(so)
            << ";\n";
          break;
        case F_SUM_DD:
          b << "  " << D("double", F.off) << " = *reinterpret_cast<const double*>(s + " << so << ");\n";
          b << "  " << D("double", F.off + 8) << " = *reinterpret_cast<const double*>(s + " << so + 8 << ");\n";
          break;
        default:
          b << "  " << D("unsigned long long", F.off) << " = *reinterpret_cast<const unsigned long long*>(s + " << so
            << ");\n";
      }
    }
  }

  // the top-level filter's row functions. A row's values (the predicate's columns and the first
  // `n_out` columns, the outputs) are read once into a JCRow (j_cload), its verdict is taken from
  // those registers (j_ckeep), and the kept row is written from them (j_cscatter; every lane of
  // the warp calls it: the validity words are OR-ed warp-wide). Reading the columns once matters:
  // a second read at the scatter, after the tile's look-back, mostly missed L2 (1.48x the
  // algorithmic DRAM reads on the hash workload's filter).
  std::string compact_funcs(int n_out) {
    std::ostringstream b;
    mark();
    std::ostringstream body;
    std::string keep = predicate(body);
    std::vector<bool> use(q.n_cols, false);
    for (int c = 0; c < q.n_cols; c++) use[c] = pred_col[c] || c < n_out;
    b << "struct JCRow {\n";
    for (int c = 0; c < q.n_cols; c++) {
      if (!use[c]) continue;
      b << "  " << (q.col[c].dtype == PMB_BOOL ? "bool" : ctype(q.col[c].dtype)) << " v" << c << ";\n";
      if (q.col[c].valid) b << "  bool ok" << c << ";\n";
    }
    b << "};\n";
    b << "__device__ __forceinline__ void j_cload(const JCParams& P, long long row, JCRow& r) {\n";
    for (int c = 0; c < q.n_cols; c++) {
      if (!use[c]) continue;
      const DCol& C = q.col[c];
      const std::string cs = std::to_string(c);
      if (C.dtype == PMB_BOOL)
        b << "  r.v" << cs << " = ((P.col_data[" << cs << "][row >> 3] >> (row & 7)) & 1) != 0;\n";
      else
        b << "  r.v" << cs << " = reinterpret_cast<const " << ctype(C.dtype) << "*>(P.col_data[" << cs << "])[row];\n";
      if (C.valid) b << "  r.ok" << cs << " = ((P.col_valid[" << cs << "][row >> 3] >> (row & 7)) & 1) != 0;\n";
    }
    b << "}\n";
    b << "__device__ __forceinline__ bool j_ckeep(const JCRow& r) {\n" << body.str() << "  return " << keep << ";\n}\n";
    b << "__device__ __forceinline__ void j_cscatter(const JCParams& P, const JCRow& r, bool keep, long long p, "
         "long long p_first) {\n";
    for (int c = 0; c < n_out && c < q.n_cols; c++) {
      const DCol& C = q.col[c];
      const std::string cs = std::to_string(c);
      if (C.dtype == PMB_BOOL) {
        b << "  jc_set_bits(reinterpret_cast<unsigned int*>(P.out_data[" << cs << "]), p, p_first, keep && r.v" << cs
          << ");\n";
      } else {
        const std::string T = ctype(C.dtype);
        b << "  if (keep) reinterpret_cast<" << T << "*>(P.out_data[" << cs << "])[p] = r.v" << cs << ";\n";
      }
      if (C.valid)
        b << "  jc_set_bits(P.out_valid[" << cs << "], p, p_first, keep && r.ok" << cs << ");\n";
      else
        b << "  jc_set_bits(P.out_valid[" << cs << "], p, p_first, keep);\n";
    }
    b << "}\n";
    return b.str();
  }

  // the aggregated columns of row `row`, read straight from the columns (a gather)
  void gather(std::ostringstream& b) {
    for (int c = 0; c < q.n_cols; c++) {
      if (!field_col[c]) continue;
      const DCol& C = q.col[c];
      const std::string cs = std::to_string(c);
      if (C.dtype == PMB_BOOL)
        b << "  r.v" << cs << " = ((P.col_data[" << cs << "][row >> 3] >> (row & 7)) & 1) != 0;\n";
      else
        b << "  r.v" << cs << " = reinterpret_cast<const " << ctype(C.dtype) << "*>(P.col_data[" << cs << "])[row];\n";
      if (C.valid) b << "  r.ok" << cs << " = ((P.col_valid[" << cs << "][row >> 3] >> (row & 7)) & 1) != 0;\n";
    }
  }

  // range report of the exact float sums: status bit and the largest exponent seen
  void fxcheck(std::ostringstream& b) {
    for (int i = 0; i < q.n_fields; i++) {
      const DField& F = q.field[i];
      if (F.kind != F_SUM_FX) continue;
      std::string slot = std::to_string(F.fx_slot);
      b << "  if (" << okk(F.col) << ") {\n    double xv = (double)" << v(F.col) << ";\n";
      b << "    if (!pmb_fx_flag(xv) && !pmb_fx_in_range(xv, P.fx_e[" << slot << "])) {\n";
      b << "      unsigned ex = (unsigned)pmb_fx_expo(xv);\n";
      b << "      if (ex > *(volatile unsigned int*)&P.status[4 + " << slot << "]) atomicMax(&P.status[4 + " << slot
        << "], ex);\n";
      b << "      if (!(*(volatile unsigned int*)P.status & PMB_ST_FXRANGE)) atomicOr(P.status, PMB_ST_FXRANGE);\n    }\n  }\n";
    }
  }

  void loads_of(std::ostringstream& b, const std::vector<bool>& want) {
    for (int c = 0; c < q.n_cols; c++) {
      if (!want[c]) continue;
      b << "  r.v" << c << " = " << load_val(c) << ";\n";
      if (q.col[c].valid) b << "  r.ok" << c << " = " << load_valid(c) << ";\n";
    }
  }

  std::string build() {
    mark();
    // columns of the predicate and keys (classification) and of the keys alone
    std::vector<bool> pk(q.n_cols, false), kc(q.n_cols, false);
    for (int c = 0; c < q.n_cols; c++) pk[c] = pred_col[c] || key_col[c];
    for (int k = 0; k < q.n_keys; k++) kc[q.key[k].col] = true;
    o << "#define J_WAIT_NS " << P.wait_ns << "\n";
    o << "#define J_NT " << P.nt << "\n#define J_NBUF " << P.nbuf << "\n#define J_OFF_BARS " << P.off_bars
      << "\n#define J_OFF_BUF " << P.off_buf << "\n#define J_BUF_BYTES " << P.buf_bytes << "\n#define J_OFF_Q " << P.off_q
      << "\n#define J_OFF_TKEYS " << P.off_tkeys << "\n#define J_OFF_TVAL " << P.off_tval << "\n#define J_TKEY " << P.tkey
      << "\n#define J_TNB " << P.tnb
      << "\n#define J_OFF_SRECS " << P.off_srecs << "\n#define J_H " << P.hot_cap << "\n#define J_SW " << P.warm_cap
      << "\n#define J_SREC " << S.bytes << "\n#define J_SREC_WORDS " << S.bytes / 4 << "\n#define J_LEN_SOFF " << (S.off.empty() ? 0 : S.off[0])
      << "\n#define J_REC " << q.rec_bytes << "\n";
    o << "__constant__ unsigned int J_SIDENT[" << S.ident.size() << "] = {";
    for (size_t i = 0; i < S.ident.size(); i++) o << (i ? ", " : "") << S.ident[i] << "u";
    o << "};\n";
    o << R"(
__device__ __forceinline__ long long j_minkey(double x) {
  return isnan(x) ? (long long)0x8000000000000000ULL : pmb_f64_key(x);
}
__device__ __forceinline__ long long j_maxkey(double x) { return isnan(x) ? 0x7FFFFFFFFFFFFFFFLL : pmb_f64_key(x); }
__device__ __forceinline__ double j_mod_f(double a, double b) {
  double r = fmod(a, b);
  if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
  return r;
}
__device__ __forceinline__ long long j_mod_i(long long a, long long b, bool& ok) {
  if (b == 0) { ok = false; return 0; }
  if (b == -1) return 0;
  long long m = a % b;
  if (m != 0 && ((m < 0) != (b < 0))) m += b;
  return m;
}
__device__ __forceinline__ long long j_fdiv_i(long long a, long long b, bool& ok) {
  if (b == 0) { ok = false; return 0; }
  if (a == (-9223372036854775807LL - 1LL) && b == -1) return a;
  long long d = a / b;
  if ((a % b != 0) && ((a < 0) != (b < 0))) d -= 1;
  return d;
}
)";
    row_struct();
    // bulk copies of one 128-row unit into a warp buffer (inputs are read once: evict-first in L2)
    o << "__device__ __forceinline__ void j_issue_unit(const JParams& P, unsigned char* st, long long u, "
         "unsigned long long* bar, unsigned long long pol) {\n";
    o << "  mbar_arrive_expect_tx(bar, " << P.tx_bytes << "u);\n";
    for (int c = 0; c < q.n_cols; c++) {
      const DCol& C = q.col[c];
      int db = C.elem ? 128 * C.elem : 16;
      o << "  bulk_g2s_hint(st + " << P.doff[c] << ", P.col_data[" << c << "] + u * " << db << "LL, " << db
        << "u, bar, pol);\n";
      if (C.valid) o << "  bulk_g2s_hint(st + " << P.voff[c] << ", P.col_valid[" << c << "] + u * 16LL, 16u, bar, pol);\n";
    }
    o << "}\n";
    // plain copy of the partial last unit (lanes of one warp)
    o << "__device__ void j_copy_unit(const JParams& P, unsigned char* st, long long row0, int rows) {\n";
    o << "  const int lane = threadIdx.x & 31;\n";
    for (int c = 0; c < q.n_cols; c++) {
      const DCol& C = q.col[c];
      if (C.elem)
        o << "  for (int i = lane; i < rows * " << C.elem << "; i += 32) st[" << P.doff[c] << " + i] = P.col_data[" << c
          << "][row0 * " << C.elem << " + i];\n";
      else
        o << "  for (int i = lane; i < (rows + 7) / 8; i += 32) st[" << P.doff[c] << " + i] = P.col_data[" << c
          << "][row0 / 8 + i];\n";
      if (C.valid)
        o << "  for (int i = lane; i < (rows + 7) / 8; i += 32) st[" << P.voff[c] << " + i] = P.col_valid[" << c
          << "][row0 / 8 + i];\n";
    }
    o << "}\n";
    // predicate + key columns and the filter verdict
    std::ostringstream body;
    std::string keep = predicate(body);
    o << "__device__ __forceinline__ bool j_load_pk(const JParams& P, const unsigned char* st, int lr, JRow& r) {\n";
    loads_of(o, pk);
    o << body.str() << "  return " << keep << ";\n}\n";
    o << "__device__ __forceinline__ void j_load_key(const JParams& P, const unsigned char* st, int lr, JRow& r) {\n";
    loads_of(o, kc);
    o << "}\n";
    o << "__device__ __forceinline__ void j_load_vals(const JParams& P, const unsigned char* st, int lr, JRow& r) {\n";
    loads_of(o, field_col);
    o << "}\n";
    o << "__device__ __forceinline__ void j_fxcheck(const JParams& P, const JRow& r) {\n";
    fxcheck(o);
    o << "}\n";
    // key
    o << "__device__ __forceinline__ unsigned long long j_key(const JRow& r) {\n  unsigned long long k = 0ULL;\n";
    // (keys wider than 64 bits never use it: the partitioned kernel reads packed sort keys)
    for (int i = 0; i < q.n_keys && q.key_bits <= 64; i++) {
      const DKey& K = q.key[i];
      std::string mask = K.bits < 64 ? std::to_string((1ULL << K.bits) - 1ULL) + "ULL" : "0xFFFFFFFFFFFFFFFFULL";
      std::string put = "k |= (" + raw_bits(K.col) + " & " + mask + ") << " + std::to_string(K.data_off) + ";";
      if (K.nullable)
        o << "  if (!" << ok(K.col) << ") k |= 1ULL << " << K.null_off << "; else " << put << "\n";
      else
        o << "  " << put << "\n";
    }
    o << "  return k;\n}\n";
    // hash of a packed key: MurmurHash3's 32-bit finalizer for keys of at most 32 bits (its word
    // repeated, so that the high and the low bits both vary), the 64-bit finalizer otherwise
    if (q.key_bits <= 32)
      o << "__device__ __forceinline__ unsigned long long j_hash(unsigned long long k) {\n"
           "  const unsigned x = pmb_fmix32((unsigned)k);\n  return ((unsigned long long)x << 32) | x;\n}\n";
    else
      o << "__device__ __forceinline__ unsigned long long j_hash(unsigned long long k) { return pmb_fmix64(k); }\n";
    o << "__device__ __forceinline__ void j_shared(const JParams& P, unsigned char* rec, const JRow& r) {\n";
    apply_shared(o);
    o << "}\n__device__ __forceinline__ void j_global(const JParams& P, unsigned char* rec, const JRow& r) {\n";
    apply_global(o);
    o << "}\n__device__ __forceinline__ void j_sfold(unsigned char* d, const unsigned char* s) {\n";
    sfold(o);
    o << "}\n__device__ __forceinline__ void j_merge_sg(const JParams& P, unsigned char* d, const unsigned char* s) {\n";
    merge_sg(o);
    o << "}\n__device__ __forceinline__ void j_store_sg(unsigned char* d, const unsigned char* s) {\n";
    store_sg(o);
    o << "}\n__device__ __forceinline__ void j_gather(const JParams& P, long long row, JRow& r) {\n";
    gather(o);
    o << "}\n";
    return o.str();
  }
};

}  // namespace

// Shared-memory record layout of the run-time kernel: 8-byte fields (min/max, double-double sums)
// first, then 32-bit words (counters; exact float sums as three carry-chained words and a flag
// word; integer sums as two carry-chained words).
void pmb_jit_slayout(const DQuery& q, JitSLayout* S) {
  S->off.assign(q.n_fields, 0);
  int off = 0;
  for (int pass = 0; pass < 2; pass++)
    for (int i = 0; i < q.n_fields; i++) {
      int k = q.field[i].kind;
      bool eight = k == F_SUM_DD || k == F_MIN_I || k == F_MAX_I || k == F_MIN_U || k == F_MAX_U || k == F_MIN_F ||
                   k == F_MAX_F;
      if (eight != (pass == 0)) continue;
      S->off[i] = off;
      off += k == F_SUM_DD || k == F_SUM_FX ? 16 : (eight || k == F_SUM_I ? 8 : 4);
    }
  // records sit at random slots: a stride of 2 mod 4 words spreads them over 16 bank pairs (a
  // multiple of 16 words would put every record's field in the same two banks)
  S->bytes = (off + 7) & ~7;
  if (S->bytes % 16 == 0) S->bytes += 8;
  S->ident.assign(S->bytes / 4, 0u);
  for (int i = 0; i < q.n_fields; i++) {
    int k = q.field[i].kind, w = S->off[i] / 4;
    if (k == F_MIN_I || k == F_MIN_F) {
      S->ident[w] = 0xFFFFFFFFu;
      S->ident[w + 1] = 0x7FFFFFFFu;
    } else if (k == F_MAX_I || k == F_MAX_F) {
      S->ident[w + 1] = 0x80000000u;
    } else if (k == F_MIN_U) {
      S->ident[w] = S->ident[w + 1] = 0xFFFFFFFFu;
    }
  }
}

bool pmb_jit_enabled(int64_t n_rows) {
  const char* e = getenv("PMB_JIT");
  if (e && e[0] == '0') return false;
  if (e && e[0] == '1') return true;
  return n_rows >= (1LL << 21);
}

// The hash kernel's skeleton text: the embedded one, or (for kernel development) the text of the
// file PMB_JIT_SKELETON names, which must define the same kernel and parameter block
static std::string hash_skeleton() {
  if (const char* path = getenv("PMB_JIT_SKELETON")) {
    if (FILE* f = fopen(path, "rb")) {
      std::string t;
      char buf[65536];
      size_t n;
      while ((n = fread(buf, 1, sizeof buf, f)) > 0) t.append(buf, n);
      fclose(f);
      if (t.find("__device__ __forceinline__ long long j_gresolve") != std::string::npos) return t;
    }
  }
  return std::string(kSkeleton);
}

std::string pmb_jit_source(const CompiledQuery& cq, const JitPlan& J) {
  Gen g(cq.dq, J);
  // order: device helpers, the skeleton's parameter block, the generated row program, the kernel
  std::string skel = hash_skeleton();
  size_t cut = skel.find("__device__ __forceinline__ long long j_gresolve");
  return std::string(kDeviceHeader) + "\n" + skel.substr(0, cut) + "\n" + g.build() + "\n" + skel.substr(cut);
}

int pmb_plan_jit(pmb_handle* h, const CompiledQuery& cq, bool have_sketch, int max_smem_optin, JitPlan* J) {
  const DQuery& q = cq.dq;
  memset(J, 0, sizeof(*J));
  J->nt = 1024;
  J->nbuf = 1;
  J->wait_ns = 0;
  if (const char* e = getenv("PMB_WAIT_NS")) J->wait_ns = std::max(0, std::min(atoi(e), 100000));
  if (const char* e = getenv("PMB_NT")) {
    int v = atoi(e);
    if (v == 256 || v == 512 || v == 1024) J->nt = v;
  }
  if (const char* e = getenv("PMB_NBUF")) {
    int v = atoi(e);
    if (v == 1 || v == 2) J->nbuf = v;
  }
  const int W = J->nt / 32;
  int off = 0, tx = 0;
  for (int c = 0; c < q.n_cols; c++) {
    int db = q.col[c].elem ? 128 * q.col[c].elem : 16;
    J->doff[c] = off;
    off += db;
    tx += db;
    J->voff[c] = -1;
    if (q.col[c].valid) {
      J->voff[c] = off;
      off += 16;
      tx += 16;
    }
  }
  J->buf_bytes = (int)pmb_align((size_t)off, 128);
  J->tx_bytes = tx;
  JitSLayout S;
  pmb_jit_slayout(q, &S);
  J->srec = S.bytes;
  const int budget = max_smem_optin - 1024;
  int used = 0;
  for (;;) {
    J->off_bars = 0;
    J->off_buf = (int)pmb_align((size_t)(8 * W * J->nbuf), 128);
    J->off_q = J->off_buf + W * J->nbuf * J->buf_bytes;
    used = J->off_q + W * 128 * 4;
    if (used <= budget) break;
    if (J->nbuf == 1) return pmb_fail(h, PMB_E_UNSUPPORTED, "query touches too many columns for the unit buffers");
    J->nbuf = 1;
  }
  // hot keys: one record per warp each; warm keys: the largest count whose table and records fit.
  // The sampled-key table: buckets of 4 keys and 4 16-bit values, filled to at most 50% (a key
  // sits in its first bucket unless that one was full, so most lookups read one bucket).
  J->tkey = q.key_bits <= 32 ? 4 : 8;
  auto buckets = [](int keys) { return keys ? ((keys / 2 + 2) + 1) & ~1 : 0; };
  auto tbytes = [&](int keys) { return buckets(keys) * 4 * (J->tkey + 2); };
  // 24 hot keys (a record per warp each): measured best on the hash workload (100M rows, Zipf 1.1
  // over 1M keys): 1.48 ms against 1.55 ms with 8 and 1.54 ms with 48
  int hot = have_sketch ? 24 : 0;
  if (const char* e = getenv("PMB_HOT")) hot = std::max(0, std::min(atoi(e), 64));
  while (hot > 0 && (int)pmb_align((size_t)used, 16) + tbytes(hot) + 32 + W * hot * J->srec > budget) hot /= 2;
  int warm = 0;
  if (have_sketch) {
    // at most 2^14 warm keys: the sampled-key table's 16-bit values keep bits 14-15 for flags
    for (int sw = 16384; sw >= 32; sw -= 32) {
      int need = (int)pmb_align((size_t)used, 16) + tbytes(hot + sw) + 32 + (W * hot + sw) * J->srec;
      if (need <= budget) {
        warm = sw;
        break;
      }
    }
  }
  if (const char* e = getenv("PMB_SMEM_SLOTS")) {
    int v = atoi(e);
    if (v >= 0 && v < warm) warm = v;
  }
  J->hot_cap = hot;
  J->warm_cap = warm;
  J->tnb = buckets(hot + warm);
  J->off_tkeys = (int)pmb_align((size_t)used, 16);
  J->off_tval = J->off_tkeys + J->tnb * 4 * J->tkey;
  J->off_srecs = (int)pmb_align((size_t)(J->off_tval + J->tnb * 8), 16);
  J->smem = J->off_srecs + (W * hot + warm) * J->srec;
  return PMB_OK;
}

// NVRTC: source -> sm_100a cubin; false with the compiler log on failure
static bool jit_compile(const std::string& src, std::vector<char>& cubin, std::string& log) {
  if (!load_nvrtc()) {
    log = "NVRTC not available";
    return false;
  }
  nvrtcProgram_t prog;
  if (g_nv.create(&prog, src.c_str(), "pmb_jit.cu", 0, nullptr, nullptr) != 0) {
    log = "nvrtcCreateProgram failed";
    return false;
  }
  // PMB_JIT_DEBUG=2 also asks ptxas for its resource report (registers, spills, shared memory)
  const char* dbg = getenv("PMB_JIT_DEBUG");
  const bool verbose = dbg && dbg[0] == '2';
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-diag-suppress=177", "--ptxas-options=-v"};
  int rc = g_nv.compile(prog, verbose ? 5 : 4, opts);
  size_t n = 0;
  g_nv.log_size(prog, &n);
  log.assign(n, '\0');
  if (n) g_nv.log(prog, &log[0]);
  if (rc != 0) {
    g_nv.destroy(&prog);
    return false;
  }
  size_t cn = 0;
  g_nv.cubin_size(prog, &cn);
  cubin.resize(cn);
  g_nv.cubin(prog, cubin.data());
  g_nv.destroy(&prog);
  return true;
}

// compiled kernel `name` of a source (cached by source text)
static int jit_kernel(pmb_handle* h, const std::string& src, const char* name, cudaKernel_t* out) {
  *out = nullptr;
  const std::string key = std::string(name) + "\n" + src;
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_cache.find(key);
  if (it != g_cache.end()) {
    *out = it->second;
    return PMB_OK;
  }
  if (g_fail.count(src)) return pmb_fail(h, PMB_E_UNSUPPORTED, "JIT compile failed earlier for this signature");
  std::vector<char> cubin;
  std::string log;
  if (!jit_compile(src, cubin, log)) {
    g_fail[src] = log;
    if (getenv("PMB_JIT_DEBUG")) fprintf(stderr, "pmb jit compile failed:\n%s\n---- source ----\n%s\n", log.c_str(), src.c_str());
    return pmb_fail(h, PMB_E_UNSUPPORTED, "JIT compile failed: " + log.substr(0, 400));
  }
  cudaLibrary_t lib;
  PMB_CUDA(h, cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
  cudaKernel_t k;
  PMB_CUDA(h, cudaLibraryGetKernel(&k, lib, name));
  g_cache[key] = k;
  *out = k;
  if (getenv("PMB_JIT_DEBUG")) fprintf(stderr, "pmb jit: compiled a %zu-byte cubin (%zu cached)\n", cubin.size(), g_cache.size());
  return PMB_OK;
}

// The signature of a hash kernel as bytes: the query descriptor without what only the launch
// parameters carry (buffer addresses, row count, fixed-point widths and ranges; only whether a
// column has a validity bitmap reaches the source), the launch plan, and the skeleton's origin.
// Equal signatures generate equal source, so a repeated query skips generating its source text
// (about 0.1 ms of host time per call, spent while the device waits for the launch).
static std::string hash_signature(const CompiledQuery& cq, const JitPlan& J) {
  DQuery d = cq.dq;
  d.n_rows = 0;
  memset(d.fx_e, 0, sizeof(d.fx_e));
  for (int c = 0; c < PMB_MAX_COLS; c++) {
    d.col[c].data = nullptr;
    d.col[c].valid = d.col[c].valid ? reinterpret_cast<const uint8_t*>(1) : nullptr;
  }
  for (int f = 0; f < PMB_MAX_FIELDS; f++) d.field[f].fx = 0;
  std::string k(reinterpret_cast<const char*>(&d), sizeof d);
  k.append(reinterpret_cast<const char*>(&J), sizeof J);
  if (const char* path = getenv("PMB_JIT_SKELETON")) k.append(path);
  return k;
}

int pmb_jit_hash_kernel(pmb_handle* h, const CompiledQuery& cq, const JitPlan& J, cudaKernel_t* out) {
  static std::mutex sig_mu;
  static std::unordered_map<std::string, cudaKernel_t> by_sig;
  const std::string sig = hash_signature(cq, J);
  {
    std::lock_guard<std::mutex> lock(sig_mu);
    auto it = by_sig.find(sig);
    if (it != by_sig.end()) {
      *out = it->second;
      return PMB_OK;
    }
  }
  const int rc = jit_kernel(h, pmb_jit_source(cq, J), "pmb_jit_hash_agg", out);
  if (rc == PMB_OK) {
    std::lock_guard<std::mutex> lock(sig_mu);
    by_sig[sig] = *out;
  }
  return rc;
}

int pmb_plan_jit_batch(pmb_handle* h, const CompiledQuery& cq, int nt, int nbuf, int max_smem_optin, JitPlan* J,
                       int warm_max) {
  const DQuery& q = cq.dq;
  memset(J, 0, sizeof(*J));
  J->nt = nt;
  J->nbuf = nbuf;
  const int W = nt / 32;
  int off = 0, tx = 0;
  for (int c = 0; c < q.n_cols; c++) {
    int db = q.col[c].elem ? 128 * q.col[c].elem : 16;
    J->doff[c] = off;
    off += db;
    tx += db;
    J->voff[c] = -1;
    if (q.col[c].valid) {
      J->voff[c] = off;
      off += 16;
      tx += 16;
    }
  }
  J->buf_bytes = (int)pmb_align((size_t)off, 128);
  J->tx_bytes = tx;
  JitSLayout S;
  pmb_jit_slayout(q, &S);
  J->srec = S.bytes;
  const int budget = max_smem_optin - 1024;
  // fewer buffers per warp when wide rows do not leave room for them
  while (nbuf > 1 && (int)pmb_align((size_t)(8 * W * nbuf), 128) + W * nbuf * J->buf_bytes + W * 128 * 4 +
                             64 + W * J->srec > budget)
    nbuf--;
  J->nbuf = nbuf;
  J->off_bars = 0;
  J->off_buf = (int)pmb_align((size_t)(8 * W * nbuf), 128);
  J->off_q = J->off_buf + W * nbuf * J->buf_bytes;
  const int used = J->off_q + W * 128 * 4;
  if (used > budget) return pmb_fail(h, PMB_E_UNSUPPORTED, "query touches too many columns for the unit buffers");
  // hot keys: 8 per item, one record per warp each; warm: the largest power of two that fits
  int hot = 8;
  while (hot > 0 && (int)pmb_align((size_t)used, 16) + 64 + W * hot * J->srec > budget) hot /= 2;
  int warm = 0;
  for (int sw = 1 << 14; sw >= 64; sw /= 2)
    if ((warm_max <= 0 || sw <= warm_max) &&
        (int)pmb_align((size_t)used, 16) + 8 * sw + 64 + (W * hot + sw) * J->srec <= budget) {
      warm = sw;
      break;
    }
  J->hot_cap = hot;
  J->warm_cap = warm;
  J->tkey = 8;
  J->tnb = 0;
  J->off_tkeys = (int)pmb_align((size_t)used, 16);
  J->off_tval = J->off_tkeys + 8 * warm;
  J->off_srecs = (int)pmb_align((size_t)(J->off_tval + 64), 16);
  J->smem = J->off_srecs + (W * hot + warm) * J->srec;
  return PMB_OK;
}

// source of the partitioned aggregation: device helpers, the parameter block, the generated row
// functions and pmb_jit_part.cuh (not the hash kernel)
static std::string part_source(const CompiledQuery& cq, const JitPlan& J, int key_words, bool cas64) {
  Gen g(cq.dq, J);
  std::string skel(kSkeleton);
  size_t cut = skel.find("__device__ __forceinline__ long long j_gresolve");
  return "#define JP_W " + std::to_string(key_words) + "\n#define JP_CAS64 " + (cas64 ? "1" : "0") + "\n" +
         std::string(kDeviceHeader) + "\n" + skel.substr(0, cut) + "\n" + g.build() + "\n" + std::string(kPartSkeleton);
}

int pmb_jit_part_kernel(pmb_handle* h, const CompiledQuery& cq, int key_words, bool cas64, JitPlan* J,
                        cudaKernel_t* out) {
  int rc = pmb_plan_jit_batch(h, cq, 1024, 1, h->max_smem_optin, J);
  if (rc) return rc;
  return jit_kernel(h, part_source(cq, *J, key_words, cas64 && key_words == 1), "pmb_jit_part_agg", out);
}

// the top-level filter's compaction (pmb_jit_compact.cuh): device helpers, the parameter block,
// the generated row functions of the hash skeleton's prefix, the compaction's own parameter block
// and helpers, its generated row functions, then its kernel
std::string pmb_jit_compact_source(const CompiledQuery& cq, const JitPlan& J, int n_out) {
  Gen g(cq.dq, J);
  std::string skel(kSkeleton);
  const size_t cut = skel.find("__device__ __forceinline__ long long j_gresolve");
  std::string comp(kCompactSkeleton);
  const size_t kcut = comp.find("extern \"C\" __global__");
  Gen g2(cq.dq, J);
  return std::string(kDeviceHeader) + "\n" + skel.substr(0, cut) + "\n" + g.build() + "\n" + comp.substr(0, kcut) +
         "\n" + g2.compact_funcs(n_out) + "\n" + comp.substr(kcut);
}

int pmb_jit_compact_kernel(pmb_handle* h, const CompiledQuery& cq, int n_out, cudaKernel_t* out) {
  JitPlan J;
  int rc = pmb_plan_jit_batch(h, cq, 1024, 1, h->max_smem_optin, &J);
  if (rc) return rc;
  return jit_kernel(h, pmb_jit_compact_source(cq, J, n_out), "pmb_jit_compact", out);
}

int pmb_jit_batch_kernel(pmb_handle* h, const CompiledQuery& cq, const JitPlan& J, cudaKernel_t* out) {
  return jit_kernel(h, "#define PMB_EXPLICIT_RED 1\n" + pmb_jit_source(cq, J) + "\n" + std::string(kBatchSkeleton),
                    "pmb_jit_batch_agg", out);
}

// Internal check (not part of the C ABI in pmb.h): generates and compiles the run-time kernel of
// a query with NVRTC, without a GPU. Column pointers are not read, only their dtypes and whether
// a validity bitmap is present. Returns PMB_OK, or an error with the compiler log in `log`.
// mode 0: the hash kernel, 1: the batched kernel, 2: the partitioned aggregation (one- and
// two-word packed keys)
static int debug_compile(const pmb_query* q, const pmb_column* cols, int32_t n_cols, char* log, int64_t log_cap,
                         int mode) {
  const bool batch = mode == 1;
  pmb_handle h;
  CompiledQuery cq;
  int rc = pmb_compile_groupby(&h, q, cols, n_cols, &cq);
  std::string msg;
  if (rc == PMB_OK) {
    static const uint8_t dummy[16] = {0};
    for (int c = 0; c < cq.dq.n_cols; c++) {
      cq.dq.col[c].data = dummy;
      cq.dq.col[c].valid = cols[cq.map.user[c]].validity ? dummy : nullptr;
    }
    if (mode == 3) {
      // the query of a top-level filter (pmb_filter.cu): every column an output, no keys or
      // aggregates, the predicate only
      CompiledQuery fq;
      memset(&fq.dq, 0, sizeof(DQuery));
      for (int c = 0; c < n_cols; c++) fq.map.user.push_back(c);
      if (q->predicate) rc = pmb_compile_predicate(&h, q->predicate, &fq.map, cols, n_cols, &fq.dq.prog);
      fq.dq.n_cols = (int)fq.map.user.size();
      fq.dq.n_rows = n_cols ? cols[0].length : 0;
      for (int c = 0; c < fq.dq.n_cols; c++) {
        fq.dq.col[c].dtype = cols[fq.map.user[c]].dtype;
        fq.dq.col[c].elem = pmb_dtype_bytes(fq.dq.col[c].dtype);
        fq.dq.col[c].data = dummy;
        fq.dq.col[c].valid = cols[fq.map.user[c]].validity ? dummy : nullptr;
      }
      cq = fq;
      JitPlan J;
      if (rc == PMB_OK) rc = pmb_plan_jit_batch(&h, cq, 1024, 1, 232448, &J);
      if (rc != PMB_OK) msg = h.err;
      std::vector<char> cubin;
      if (rc == PMB_OK && !jit_compile(pmb_jit_compact_source(cq, J, n_cols), cubin, msg)) rc = PMB_E_UNSUPPORTED;
      else if (rc == PMB_OK && getenv("PMB_JIT_DEBUG") && getenv("PMB_JIT_DEBUG")[0] == '2') fprintf(stderr, "%s\n", msg.c_str());
    } else if (mode == 2) {
      JitPlan J;
      rc = pmb_plan_jit_batch(&h, cq, 1024, 1, 232448, &J);
      if (rc != PMB_OK) msg = h.err;
      for (int v = 0; v < 3 && rc == PMB_OK; v++) {
        std::vector<char> cubin;
        if (!jit_compile(part_source(cq, J, v == 2 ? 2 : 1, v == 1), cubin, msg)) rc = PMB_E_UNSUPPORTED;
        else if (getenv("PMB_JIT_DEBUG") && getenv("PMB_JIT_DEBUG")[0] == '2') fprintf(stderr, "%s\n", msg.c_str());
      }
    } else if (cq.dq.key_bits > 64) {
      rc = PMB_E_UNSUPPORTED;
      msg = "128-bit keys use the prebuilt kernel";
    } else {
      JitPlan J;
      rc = batch ? pmb_plan_jit_batch(&h, cq, 1024, 2, 232448, &J) : pmb_plan_jit(&h, cq, true, 232448, &J);
      if (rc == PMB_OK) {
        std::vector<char> cubin;
        const std::string src = batch ? "#define PMB_EXPLICIT_RED 1\n" + pmb_jit_source(cq, J) + "\n" + std::string(kBatchSkeleton)
                                      : pmb_jit_source(cq, J);
        if (const char* e = getenv("PMB_JIT_DEBUG"))
          if (e[0] == '2') fprintf(stderr, "%s\n", src.c_str());  // the generated source, for inspection
        if (!jit_compile(src, cubin, msg)) rc = PMB_E_UNSUPPORTED;
        else if (getenv("PMB_JIT_DEBUG") && getenv("PMB_JIT_DEBUG")[0] == '2') fprintf(stderr, "%s\n", msg.c_str());
      } else {
        msg = h.err;
      }
    }
  } else {
    msg = h.err;
  }
  if (log && log_cap > 0) {
    size_t n = std::min<size_t>(msg.size(), (size_t)log_cap - 1);
    memcpy(log, msg.data(), n);
    log[n] = 0;
  }
  return rc;
}

extern "C" int pmb_debug_jit_compile(const pmb_query* q, const pmb_column* cols, int32_t n_cols, char* log,
                                     int64_t log_cap) {
  return debug_compile(q, cols, n_cols, log, log_cap, 0);
}
// the same for the batched kernel (pmb_jit_batch.cuh)
extern "C" int pmb_debug_jit_compile_batch(const pmb_query* q, const pmb_column* cols, int32_t n_cols, char* log,
                                           int64_t log_cap) {
  return debug_compile(q, cols, n_cols, log, log_cap, 1);
}
// the same for the top-level filter's compaction (pmb_jit_compact.cuh) of every column by the
// query's predicate (keys and aggregates of the query are ignored)
extern "C" int pmb_debug_jit_compile_compact(const pmb_query* q, const pmb_column* cols, int32_t n_cols, char* log,
                                             int64_t log_cap) {
  return debug_compile(q, cols, n_cols, log, log_cap, 3);
}
// the same for the partitioned strategy's aggregation kernel (pmb_jit_part.cuh)
extern "C" int pmb_debug_jit_compile_part(const pmb_query* q, const pmb_column* cols, int32_t n_cols, char* log,
                                          int64_t log_cap) {
  return debug_compile(q, cols, n_cols, log, log_cap, 2);
}

int pmb_jit_launch(pmb_handle* h, cudaKernel_t k, const CompiledQuery& cq, const JitPlan& J, const HashParams& P,
                   int grid, const uint8_t* ttab, int tnb) {
  JitParams A;
  memset(&A, 0, sizeof(A));
  for (int c = 0; c < cq.dq.n_cols; c++) {
    A.col_data[c] = cq.dq.col[c].data;
    A.col_valid[c] = cq.dq.col[c].valid;
  }
  A.n_rows = cq.dq.n_rows;
  A.n_units = (cq.dq.n_rows + 127) / 128;
  A.gprobe = (int)std::min<unsigned long long>(P.gcap / 4, 256);     // buckets of 4 slots
  A.occ_limit = (unsigned)std::min<unsigned long long>(P.gcap - P.gcap / 5, 0xFFFFFFFFull);  // 80% full
  A.gkeys = P.gkeys;
  A.grecs = P.grecs;
  A.gcap = P.gcap;
  A.status = P.status;
  A.hot_keys = P.hot_keys;
  A.hot_n = P.hot_n;
  A.warm_keys = P.warm_keys;
  A.warm_n = P.warm_n;
  A.kstats = P.kstats;
  A.ttab = ttab;
  A.tnb = ttab ? tnb : 0;
  for (int i = 0; i < cq.dq.n_fields; i++)
    if (cq.dq.field[i].kind == F_SUM_FX) {
      A.fx[cq.dq.field[i].fx_slot] = cq.dq.field[i].fx;
      A.fx_e[cq.dq.field[i].fx_slot] = cq.dq.fx_e[cq.dq.field[i].fx_slot];
    }
  PMB_CUDA(h, cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, J.smem));
  void* args[] = {&A};
  pmb_kernel_begin(h, "hash_agg");
  cudaError_t e = cudaLaunchKernel((const void*)k, dim3(grid), dim3(J.nt), args, (size_t)J.smem, h->stream);
  pmb_kernel_end(h);
  PMB_CUDA(h, e);
  return PMB_OK;
}
