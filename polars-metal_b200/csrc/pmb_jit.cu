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

uint64_t next_pow2_u64(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

#include "pmb_jit_sources.inc"  // kDeviceHeader, kSkeleton (generated from the .cuh files by the build)

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
  std::vector<bool> need_val, need_bits, need_valid, field_col;
  int tmp = 0;

  Gen(const DQuery& q_, const JitPlan& p_) : q(q_), P(p_) {
    need_val.assign(q.n_cols, false);
    need_bits.assign(q.n_cols, false);
    need_valid.assign(q.n_cols, false);
    field_col.assign(q.n_cols, false);
  }

  std::string v(int c) { return "r.v" + std::to_string(c); }
  std::string ok(int c) { return q.col[c].valid ? "r.ok" + std::to_string(c) : std::string("true"); }

  void mark_leaf(const DLeaf& L) {
    if (L.col >= 0) need_val[L.col] = need_valid[L.col] = true;
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
      need_bits[q.key[k].col] = need_valid[q.key[k].col] = true;
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
    std::string vo = std::to_string(P.voff[c]);
    return "(((st[" + vo + " + (lr >> 3)] >> (lr & 7)) & 1) != 0)";
  }

  void row_struct() {
    o << "struct JRow {\n";
    for (int c = 0; c < q.n_cols; c++) {
      if (need_val[c]) o << "  " << ctype(q.col[c].dtype) << " v" << c << ";\n";
      if (need_valid[c] && q.col[c].valid) o << "  bool ok" << c << ";\n";
    }
    o << "};\n";
  }

  // exact float sums: report values outside the slot's range (the call is then re-run wider)
  void fx_check(std::ostringstream& b) {
    for (int i = 0; i < q.n_fields; i++) {
      const DField& F = q.field[i];
      if (F.kind != F_SUM_FX) continue;
      std::string slot = std::to_string(F.fx_slot);
      b << "  if (check && " << ok(F.col) << ") {\n    double xv = (double)" << v(F.col) << ";\n";
      b << "    if (!pmb_fx_flag(xv) && !pmb_fx_in_range(xv, P.fx_e[" << slot << "])) { atomicOr(P.status, PMB_ST_FXRANGE); "
        << "atomicMax(&P.status[4 + " << slot << "], (unsigned)pmb_fx_expo(xv)); }\n  }\n";
    }
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

  void loads(std::ostringstream& b, bool fields_only) {
    for (int c = 0; c < q.n_cols; c++) {
      if (fields_only ? !field_col[c] : !need_val[c]) continue;
      b << "  r.v" << c << " = " << load_val(c) << ";\n";
      if (q.col[c].valid) b << "  r.ok" << c << " = " << load_valid(c) << ";\n";
    }
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

  void apply(std::ostringstream& b, int mode) {  // 0 private, 1 shared, 2 global
    // global: pack 32-bit counters sharing a 64-bit word into one add
    std::vector<std::pair<int, std::string>> words;  // (word offset, increment expression)
    for (int i = 0; i < q.n_fields; i++) {
      const DField& F = q.field[i];
      std::string okc = F.kind == F_LEN ? std::string("true") : ok(F.col);
      if (F.kind == F_LEN || F.kind == F_CNT) {
        std::string inc = F.kind == F_LEN ? "1ULL" : "(" + okc + " ? 1ULL : 0ULL)";
        if (mode == 0) b << "  *" << at(F.off, "unsigned int") << " += (unsigned int)" << inc << ";\n";
        else if (mode == 1) b << "  if (" << inc << ") atomicAdd(" << at(F.off, "unsigned int") << ", 1u);\n";
        else {
          int w = F.off & ~7;
          std::string sh = (F.off & 4) ? " << 32" : "";
          bool found = false;
          for (auto& p : words)
            if (p.first == w) {
              p.second += " + (" + inc + sh + ")";
              found = true;
            }
          if (!found) words.push_back({w, "(" + inc + sh + ")"});
        }
        continue;
      }
      if (F.kind == F_SUM_FX) {
        std::string hi = at(F.off, "double"), lo = at(F.off + 8, "double"), slot = std::to_string(F.fx_slot);
        b << "  if (" << okc << ") {\n    double xv = (double)" << v(F.col) << ";\n";
        if (mode == 0) b << "    dd_plain_add(" << hi << ", " << lo << ", xv);\n";
        else if (mode == 1) b << "    dd_atomic_add(" << hi << ", " << lo << ", xv);\n";
        else {
          b << "    unsigned fl = pmb_fx_flag(xv);\n";
          b << "    if (fl) atomicOr(" << at(F.off + 24, "unsigned int") << ", fl);\n";
          b << "    else if (pmb_fx_in_range(xv, P.fx_e[" << slot << "])) {\n      unsigned long long a, b_, c;\n";
          b << "      pmb_fx_split(xv, P.fx[" << slot << "], a, b_, c);\n";
          b << "      if (a) atomicAdd(" << at(F.off, "unsigned long long") << ", a);\n";
          b << "      if (b_) atomicAdd(" << at(F.off + 8, "unsigned long long") << ", b_);\n";
          b << "      if (c) atomicAdd(" << at(F.off + 16, "unsigned long long") << ", c);\n    }\n";
        }
        b << "  }\n";
        continue;
      }
      std::string x = fval(F);
      b << "  if (" << okc << ") {\n";
      switch (F.kind) {
        case F_SUM_DD:
          if (mode == 0) b << "    dd_plain_add(" << at(F.off, "double") << ", " << at(F.off + 8, "double") << ", " << x << ");\n";
          else b << "    dd_atomic_add(" << at(F.off, "double") << ", " << at(F.off + 8, "double") << ", " << x << ");\n";
          break;
        case F_SUM_I:
          if (mode == 0) b << "    *" << at(F.off, "unsigned long long") << " += " << x << ";\n";
          else b << "    atomicAdd(" << at(F.off, "unsigned long long") << ", " << x << ");\n";
          break;
        default: {
          bool mn = F.kind == F_MIN_I || F.kind == F_MIN_U || F.kind == F_MIN_F;
          const char* T = (F.kind == F_MIN_U || F.kind == F_MAX_U) ? "unsigned long long" : "long long";
          const char* cmp = mn ? "<" : ">";
          b << "    " << T << " val = " << x << ";\n";
          if (mode == 0) {
            b << "    if (val " << cmp << " *" << at(F.off, T) << ") *" << at(F.off, T) << " = val;\n";
          } else {
            std::string rd = mode == 1 ? "*reinterpret_cast<volatile " + std::string(T) + "*>(rec + " + std::to_string(F.off) + ")"
                                       : "*" + at(F.off, T);
            b << "    if (val " << cmp << " " << rd << ") " << (mn ? "atomicMin(" : "atomicMax(") << at(F.off, T)
              << ", val);\n";
          }
        }
      }
      b << "  }\n";
    }
    for (auto& p : words)
      b << "  atomicAdd(reinterpret_cast<unsigned long long*>(rec + " << p.first << "), " << p.second << ");\n";
  }

  void merge(std::ostringstream& b, bool global) {
    for (int i = 0; i < q.n_fields; i++) {
      const DField& F = q.field[i];
      std::string d = std::to_string(F.off);
      switch (F.kind) {
        case F_LEN:
        case F_CNT:
          if (global) b << "  { unsigned int x = *reinterpret_cast<const unsigned int*>(s + " << d << "); if (x) atomicAdd(reinterpret_cast<unsigned int*>(d + " << d << "), x); }\n";
          else b << "  *reinterpret_cast<unsigned int*>(d + " << d << ") += *reinterpret_cast<const unsigned int*>(s + " << d << ");\n";
          break;
        case F_SUM_DD:
          b << "  { double hi = *reinterpret_cast<const double*>(s + " << d << "), lo = *reinterpret_cast<const double*>(s + " << F.off + 8 << ");\n";
          if (global)
            b << "    if (hi != 0.0) dd_atomic_add(reinterpret_cast<double*>(d + " << d << "), reinterpret_cast<double*>(d + " << F.off + 8 << "), hi);\n"
              << "    if (lo != 0.0) atomicAdd(reinterpret_cast<double*>(d + " << F.off + 8 << "), lo); }\n";
          else
            b << "    dd_plain_add(reinterpret_cast<double*>(d + " << d << "), reinterpret_cast<double*>(d + " << F.off + 8 << "), hi);\n"
              << "    *reinterpret_cast<double*>(d + " << F.off + 8 << ") += lo; }\n";
          break;
        case F_SUM_FX: {
          std::string hs = std::to_string(F.off), ls = std::to_string(F.off + 8), slot = std::to_string(F.fx_slot);
          b << "  { double hi = *reinterpret_cast<const double*>(s + " << hs << "), lo = *reinterpret_cast<const double*>(s + "
            << ls << ");\n";
          if (!global) {
            b << "    dd_plain_add(reinterpret_cast<double*>(d + " << hs << "), reinterpret_cast<double*>(d + " << ls
              << "), hi);\n    *reinterpret_cast<double*>(d + " << ls << ") += lo; }\n";
          } else {
            // a double-double partial of at most 2^(94 - F - E) values splits exactly into limbs
            b << "    unsigned fl = pmb_fx_flag(hi);\n";
            b << "    if (fl) atomicOr(reinterpret_cast<unsigned int*>(d + " << F.off + 24 << "), fl);\n";
            b << "    else {\n      double parts[2] = {hi, lo};\n      for (int t = 0; t < 2; t++) {\n";
            b << "        if (parts[t] == 0.0 || !isfinite(parts[t])) continue;\n        unsigned long long a, b_, c;\n";
            b << "        pmb_fx_split(parts[t], P.fx[" << slot << "], a, b_, c);\n";
            b << "        if (a) atomicAdd(reinterpret_cast<unsigned long long*>(d + " << F.off << "), a);\n";
            b << "        if (b_) atomicAdd(reinterpret_cast<unsigned long long*>(d + " << F.off + 8 << "), b_);\n";
            b << "        if (c) atomicAdd(reinterpret_cast<unsigned long long*>(d + " << F.off + 16 << "), c);\n";
            b << "      }\n    }\n  }\n";
          }
          break;
        }
        case F_SUM_I:
          if (global) b << "  { unsigned long long x = *reinterpret_cast<const unsigned long long*>(s + " << d << "); if (x) atomicAdd(reinterpret_cast<unsigned long long*>(d + " << d << "), x); }\n";
          else b << "  *reinterpret_cast<unsigned long long*>(d + " << d << ") += *reinterpret_cast<const unsigned long long*>(s + " << d << ");\n";
          break;
        default: {
          bool mn = F.kind == F_MIN_I || F.kind == F_MIN_U || F.kind == F_MIN_F;
          bool uns = F.kind == F_MIN_U || F.kind == F_MAX_U;
          const char* T = uns ? "unsigned long long" : "long long";
          std::string ident = uns ? (mn ? "0xFFFFFFFFFFFFFFFFULL" : "0ULL")
                                  : (mn ? "0x7FFFFFFFFFFFFFFFLL" : "(long long)0x8000000000000000ULL");
          b << "  { " << T << " x = *reinterpret_cast<const " << T << "*>(s + " << d << ");\n";
          if (global)
            b << "    if (x != " << ident << ") " << (mn ? "atomicMin" : "atomicMax") << "(reinterpret_cast<" << T << "*>(d + " << d << "), x); }\n";
          else
            b << "    if (x " << (mn ? "<" : ">") << " *reinterpret_cast<" << T << "*>(d + " << d << ")) *reinterpret_cast<" << T << "*>(d + " << d << ") = x; }\n";
        }
      }
    }
  }

  std::string build(const std::vector<uint64_t>& ident) {
    mark();
    o << "#define J_NT " << P.nt << "\n#define J_OFF_BUF " << P.off_buf << "\n#define J_BUF_BYTES " << P.buf_bytes
      << "\n#define J_OFF_SKEYS " << P.off_skeys << "\n#define J_OFF_SRECS " << P.off_srecs << "\n#define J_S " << P.S
      << "\n#define J_HOT_CAP " << P.hot_cap << "\n#define J_HOT_LUT " << std::max(P.hot_lut, 1)
      << "\n#define J_OFF_HOT_LUT " << P.off_hot_lut << "\n#define J_OFF_HOT_RECS " << P.off_hot_recs
      << "\n#define J_REC " << q.rec_bytes << "\n#define J_REC_WORDS " << q.rec_bytes / 8 << "\n#define J_LEN_OFF "
      << q.field[0].off << "\n";
    o << "__constant__ unsigned long long J_IDENT[" << ident.size() << "] = {";
    for (size_t i = 0; i < ident.size(); i++) o << (i ? ", " : "") << ident[i] << "ULL";
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
    // bulk copies of one 128-row unit into a warp's buffer
    o << "__device__ __forceinline__ void j_issue_unit(const JParams& P, unsigned char* st, long long u, unsigned long long* bar) {\n";
    o << "  mbar_arrive_expect_tx(bar, " << P.tx_bytes << "u);\n";
    for (int c = 0; c < q.n_cols; c++) {
      const DCol& C = q.col[c];
      int db = C.elem ? 128 * C.elem : 16;
      o << "  bulk_g2s(st + " << P.doff[c] << ", P.col_data[" << c << "] + u * " << db << "LL, " << db << "u, bar);\n";
      if (C.valid) o << "  bulk_g2s(st + " << P.voff[c] << ", P.col_valid[" << c << "] + u * 16LL, 16u, bar);\n";
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
    // row loads + predicate
    std::ostringstream body;
    std::string keep = predicate(body);
    o << "__device__ __forceinline__ bool j_load(const JParams& P, const unsigned char* st, int lr, JRow& r, bool check) {\n";
    loads(o, false);
    o << body.str() << "  bool keep = " << keep << ";\n";
    o << "  if (keep) {\n";
    fx_check(o);
    o << "  }\n  return keep;\n}\n";
    o << "__device__ __forceinline__ void j_load_vals(const JParams& P, const unsigned char* st, int lr, JRow& r) {\n";
    loads(o, true);
    o << "}\n";
    // key
    o << "__device__ __forceinline__ unsigned long long j_key(const JRow& r) {\n  unsigned long long k = 0ULL;\n";
    for (int i = 0; i < q.n_keys; i++) {
      const DKey& K = q.key[i];
      std::string mask = K.bits < 64 ? std::to_string((1ULL << K.bits) - 1ULL) + "ULL" : "0xFFFFFFFFFFFFFFFFULL";
      std::string put = "k |= (" + raw_bits(K.col) + " & " + mask + ") << " + std::to_string(K.data_off) + ";";
      if (K.nullable)
        o << "  if (!" << ok(K.col) << ") k |= 1ULL << " << K.null_off << "; else " << put << "\n";
      else
        o << "  " << put << "\n";
    }
    o << "  return k;\n}\n";
    // record updates
    const char* names[] = {"j_private", "j_shared", "j_global"};
    for (int m = 0; m < 3; m++) {
      o << "__device__ __forceinline__ void " << names[m] << "(const JParams& P, unsigned char* rec, const JRow& r) {\n";
      apply(o, m);
      o << "}\n";
    }
    o << "__device__ __forceinline__ void j_merge_private(unsigned char* d, const unsigned char* s) {\n";
    merge(o, false);
    o << "}\n__device__ __forceinline__ void j_merge_global(const JParams& P, unsigned char* d, const unsigned char* s) {\n";
    merge(o, true);
    o << "}\n";
    return o.str();
  }
};

}  // namespace

bool pmb_jit_enabled(int64_t n_rows) {
  const char* e = getenv("PMB_JIT");
  if (e && e[0] == '0') return false;
  if (e && e[0] == '1') return true;
  return n_rows >= (1LL << 21);
}

std::string pmb_jit_source(const CompiledQuery& cq, const JitPlan& J) {
  Gen g(cq.dq, J);
  // order: device helpers, the skeleton's parameter block, the generated row program, the kernel
  std::string skel(kSkeleton);
  size_t cut = skel.find("__device__ __forceinline__ long long j_gresolve");
  return std::string(kDeviceHeader) + "\n" + skel.substr(0, cut) + "\n" + g.build(cq.rec_init) + "\n" + skel.substr(cut);
}

int pmb_plan_jit(pmb_handle* h, const CompiledQuery& cq, bool have_sketch, int max_smem_optin, JitPlan* J) {
  const DQuery& q = cq.dq;
  memset(J, 0, sizeof(*J));
  J->nt = 1024;
  if (const char* e = getenv("PMB_NT")) {
    int v = atoi(e);
    if (v == 256 || v == 512 || v == 1024) J->nt = v;
  }
  const int W = J->nt / 32, rec = q.rec_bytes;
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
  const int budget = max_smem_optin - 1024;
  J->off_buf = (int)pmb_align((size_t)(8 * W), 128);
  int used = J->off_buf + W * J->buf_bytes;
  if (used > budget) return pmb_fail(h, PMB_E_UNSUPPORTED, "query touches too many columns for the unit buffers");
  // hot tier: per-warp records of the heaviest sample keys (up to 32 KB), then the warm table
  int hot = have_sketch ? 32 : 0;
  if (const char* e = getenv("PMB_HOT")) hot = std::max(0, std::min(atoi(e), 128));
  while (hot > 0 && (W * hot * rec > (32 << 10) || used + W * hot * rec + 16 * hot > budget)) hot /= 2;
  J->hot_cap = hot;
  J->hot_lut = hot ? (int)next_pow2_u64((uint64_t)(2 * hot)) : 0;
  J->off_hot_lut = (int)pmb_align((size_t)used, 16);
  J->off_hot_recs = (int)pmb_align((size_t)(J->off_hot_lut + 12 * J->hot_lut), 16);
  used = J->off_hot_recs + W * hot * rec;
  int S = 0;
  if (have_sketch) {
    S = 1;
    while (used + (2 * S) * (8 + rec) + 16 <= budget && 2 * S <= 4096) S *= 2;
    if (S < 64) S = 0;
  }
  if (const char* e = getenv("PMB_SMEM_SLOTS")) {
    int v = atoi(e);
    if (v == 0) S = 0;
    else if (v > 0 && v < S) S = (int)next_pow2_u64((uint64_t)v);
  }
  J->S = S;
  J->off_skeys = (int)pmb_align((size_t)used, 16);
  J->off_srecs = J->off_skeys + 8 * S;
  J->smem = J->off_srecs + S * rec;
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
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-diag-suppress=177"};
  int rc = g_nv.compile(prog, 4, opts);
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

int pmb_jit_hash_kernel(pmb_handle* h, const CompiledQuery& cq, const JitPlan& J, cudaKernel_t* out) {
  *out = nullptr;
  std::string src = pmb_jit_source(cq, J);
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_cache.find(src);
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
  PMB_CUDA(h, cudaLibraryGetKernel(&k, lib, "pmb_jit_hash_agg"));
  g_cache[src] = k;
  *out = k;
  if (getenv("PMB_JIT_DEBUG")) fprintf(stderr, "pmb jit: compiled a %zu-byte cubin (%zu cached)\n", cubin.size(), g_cache.size());
  return PMB_OK;
}

// Internal check (not part of the C ABI in pmb.h): generates and compiles the run-time kernel of
// a query with NVRTC, without a GPU. Column pointers are not read, only their dtypes and whether
// a validity bitmap is present. Returns PMB_OK, or an error with the compiler log in `log`.
extern "C" int pmb_debug_jit_compile(const pmb_query* q, const pmb_column* cols, int32_t n_cols, char* log,
                                     int64_t log_cap) {
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
    if (cq.dq.key_bits > 64) {
      rc = PMB_E_UNSUPPORTED;
      msg = "128-bit keys use the prebuilt kernel";
    } else {
      JitPlan J;
      rc = pmb_plan_jit(&h, cq, true, 232448, &J);
      if (rc == PMB_OK) {
        std::vector<char> cubin;
        if (!jit_compile(pmb_jit_source(cq, J), cubin, msg)) rc = PMB_E_UNSUPPORTED;
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

int pmb_jit_launch(pmb_handle* h, cudaKernel_t k, const CompiledQuery& cq, const JitPlan& J, const HashParams& P,
                   int grid) {
  JitParams A;
  memset(&A, 0, sizeof(A));
  for (int c = 0; c < cq.dq.n_cols; c++) {
    A.col_data[c] = cq.dq.col[c].data;
    A.col_valid[c] = cq.dq.col[c].valid;
  }
  A.n_rows = cq.dq.n_rows;
  A.n_units = (cq.dq.n_rows + 127) / 128;
  A.gprobe = P.gprobe;
  A.gkeys = P.gkeys;
  A.grecs = P.grecs;
  A.gcap = P.gcap;
  A.status = P.status;
  A.hot_keys = P.hot_keys;
  A.hot_n = P.hot_n;
  A.warm_keys = P.warm_keys;
  A.warm_n = P.warm_n;
  A.kstats = P.kstats;
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
