// program.cpp -- bytecode validation and micro-op compilation (see program.hpp).
#include "program.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace gpum {

namespace {

enum SrcOp : uint32_t {
  OP_CONST = 0, OP_PARAM = 1, OP_DATA = 2, OP_ADD = 3, OP_SUB = 4, OP_MUL = 5,
  OP_DIV = 6, OP_NEG = 7, OP_EXP = 8, OP_LOG = 9, OP_SQRT = 10, OP_POW = 11,
  OP_LGAMMA = 12
};

// The reference dispatches every unknown opcode to POW
// (cpu_native.rs:103, chain_kernel.rs:109-111); normalise it here.
inline uint32_t norm_op(uint32_t op) {
  return (op <= OP_SQRT || op == OP_LGAMMA) ? op : OP_POW;
}
inline bool is_push(uint32_t op) { return op <= OP_DATA; }
inline bool is_unary(uint32_t op) {
  return (op >= OP_NEG && op <= OP_SQRT) || op == OP_LGAMMA;
}
inline bool is_binary(uint32_t op) { return !is_push(op) && !is_unary(op); }

std::string fmt(const char* f, long a, long b = 0) {
  char buf[256];
  std::snprintf(buf, sizeof buf, f, a, b);
  return buf;
}

}  // namespace

int validate_program(const uint32_t* code, size_t n_code, size_t n_consts,
                     uint32_t n_params, uint32_t n_cols, bool allow_data, int* depth,
                     std::string* err) {
  *depth = 0;
  if (n_code % 2 != 0) {
    *err = "bytecode length must be even (opcode/argument pairs)";
    return 1;
  }
  if (n_code > 0 && code == nullptr) {
    *err = "bytecode pointer is NULL";
    return 1;
  }
  const size_t n = n_code / 2;
  int sp = 0, maxd = 0;
  for (size_t pc = 0; pc < n; ++pc) {
    const uint32_t op = norm_op(code[2 * pc]);
    const uint32_t arg = code[2 * pc + 1];
    if (is_push(op)) {
      if (op == OP_CONST && arg >= n_consts) {
        *err = fmt("instruction %ld: constant index %ld out of range", (long)pc, arg);
        return 1;
      }
      if (op == OP_PARAM && arg >= n_params) {
        *err = fmt("instruction %ld: parameter index %ld out of range", (long)pc, arg);
        return 1;
      }
      if (op == OP_DATA && (!allow_data || arg >= n_cols)) {
        *err = allow_data
                   ? fmt("instruction %ld: data column %ld out of range", (long)pc, arg)
                   : fmt("instruction %ld: the prior may not read data (column %ld)",
                         (long)pc, arg);
        return 1;
      }
      ++sp;
    } else if (is_unary(op)) {
      if (sp < 1) {
        *err = fmt("instruction %ld: stack underflow", (long)pc);
        return 1;
      }
    } else {
      if (sp < 2) {
        *err = fmt("instruction %ld: stack underflow", (long)pc);
        return 1;
      }
      --sp;
    }
    if (sp > maxd) maxd = sp;
    if (maxd > kMaxStack) {
      *err = fmt("stack depth %ld exceeds the interpreter limit %ld", maxd, kMaxStack);
      return 1;
    }
  }
  if (n > 0 && sp < 1) {
    *err = "program leaves an empty stack";
    return 1;
  }
  *depth = maxd;
  return 0;
}

int compile_program(const uint32_t* code, size_t n_code, const double* consts,
                    size_t n_consts, uint32_t n_params, uint32_t n_cols,
                    bool allow_data, UProg* out, std::string* err) {
  *out = UProg();
  int depth = 0;
  if (validate_program(code, n_code, n_consts, n_params, n_cols, allow_data, &depth,
                       err))
    return 1;
  if (n_params > (uint32_t)kMaxIndex || n_cols > (uint32_t)kMaxIndex) {
    *err = "more than 2047 parameters or data columns";
    return 1;
  }
  if (n_consts > 0 && consts == nullptr) {
    *err = "constant pool pointer is NULL";
    return 1;
  }
  const size_t n = n_code / 2;
  out->depth = depth;
  out->n_src = (int)n;
  for (size_t i = 0; i < n_consts; ++i) out->consts.push_back((float)consts[i]);

  // Stack depth before each source instruction.
  std::vector<int> before(n + 1, 0);
  std::vector<uint32_t> op(n), arg(n);
  int sp = 0;
  for (size_t pc = 0; pc < n; ++pc) {
    op[pc] = norm_op(code[2 * pc]);
    arg[pc] = code[2 * pc + 1];
    before[pc] = sp;
    if (is_push(op[pc])) ++sp;
    else if (is_binary(op[pc])) --sp;
    if (op[pc] == OP_DATA) out->uses_data = true;
  }

  // Repeated subtrees.  In postfix order a subtree is the contiguous range
  // [start[pc], pc] that ends at its root; two subtrees compute the same value
  // when their instruction ranges match (constants compared by value).
  std::vector<size_t> start(n, 0);
  {
    std::vector<size_t> st;
    for (size_t pc = 0; pc < n; ++pc) {
      if (is_push(op[pc])) {
        start[pc] = pc;
      } else if (is_unary(op[pc])) {
        start[pc] = st.back();
        st.pop_back();
      } else {
        st.pop_back();
        start[pc] = st.back();
        st.pop_back();
      }
      st.push_back(start[pc]);
    }
  }
  auto same_range = [&](size_t a, size_t b, size_t len) {
    for (size_t k = 0; k < len; ++k) {
      if (op[a + k] != op[b + k]) return false;
      if (op[a + k] == OP_CONST) {
        if (consts[arg[a + k]] != consts[arg[b + k]]) return false;
      } else if (is_push(op[a + k]) && arg[a + k] != arg[b + k]) {
        return false;
      }
    }
    return true;
  };
  // LOG(1 + EXP(a)) and LOG(EXP(a) + 1): the instructions other than `a` are
  // not emitted (omit), and the LOG emits the softplus of `a` into the slot
  // of the LOG's result -- in place when `a` sits there (EXP first), from the
  // slot above when the constant 1 was pushed first.
  std::vector<char> omit(n, 0);
  std::vector<int> softplus_kind(n, 0);
  auto is_one = [&](size_t i) { return op[i] == OP_CONST && consts[arg[i]] == 1.0; };
  for (size_t pc = 2; pc < n; ++pc) {
    if (op[pc] != OP_LOG || op[pc - 1] != OP_ADD) continue;
    const size_t r = pc - 2;            // the ADD's right operand root
    if (start[r] == 0) continue;
    const size_t l = start[r] - 1;      // its left operand root
    if (start[l] == l && is_one(l) && op[r] == OP_EXP && r >= 1) {
      omit[l] = omit[r] = omit[pc - 1] = 1;
      softplus_kind[pc] = K_SOFTPLUS1;
    } else if (start[r] == r && is_one(r) && op[l] == OP_EXP) {
      omit[l] = omit[r] = omit[pc - 1] = 1;
      softplus_kind[pc] = K_SOFTPLUS;
    }
  }
  // A push that is the left operand of an ADD, SUB or MUL whose right operand
  // is a subtree of two or more instructions: the push is deferred to the
  // operation (defer_kind at the operation, the push's index in defer_src).
  // Excluded: the softplus's parts, and acc + p*x, which stays one
  // multiply-add.
  std::vector<char> deferred(n, 0);
  std::vector<int> defer_kind(n, 0);
  std::vector<size_t> defer_src(n, 0);
  for (size_t q = 2; q < n; ++q) {
    const uint32_t b = op[q];
    if (b != OP_ADD && b != OP_SUB && b != OP_MUL) continue;
    const size_t r = q - 1;           // right operand root
    const size_t pc = start[r] - 1;   // left operand root, when it is a push
    if (start[r] == 0 || !is_push(op[pc]) || r - start[r] + 1 < 2 || omit[pc] || omit[q])
      continue;
    const bool fma = b == OP_ADD && q == pc + 4 && op[pc + 3] == OP_MUL &&
                     ((op[pc + 1] == OP_PARAM && op[pc + 2] == OP_DATA) ||
                      (op[pc + 1] == OP_DATA && op[pc + 2] == OP_PARAM));
    if (fma) continue;
    const int bi = b == OP_ADD ? 0 : (b == OP_SUB ? 1 : 2);
    const int base = op[pc] == OP_CONST ? K_ADD_C1 : (op[pc] == OP_PARAM ? K_ADD_P1 : K_ADD_D1);
    deferred[pc] = 1;
    defer_kind[q] = base + bi;
    defer_src[q] = pc;
  }
  // save_end[pc] = k + 1 when the first copy of saved subtree k ends at pc;
  // load_at[pc] = k + 1 when a later copy of it starts at pc (skipped).
  std::vector<int> save_end(n, 0), load_at(n, 0);
  std::vector<size_t> load_root(n, 0);
  std::vector<char> skipped(n, 0);
  {
    std::vector<size_t> roots;
    for (size_t pc = 0; pc < n && depth <= kMaxSavedDepth; ++pc)
      if (!is_push(op[pc]) && !omit[pc] && pc - start[pc] + 1 >= (size_t)kMinSaved)
        roots.push_back(pc);
    // Largest subtrees first: a smaller one inside a skipped copy is gone.
    std::stable_sort(roots.begin(), roots.end(), [&](size_t a, size_t b) {
      return a - start[a] > b - start[b];
    });
    std::vector<char> used(n, 0);
    for (size_t ri = 0; ri < roots.size() && out->n_saves < kMaxSaves; ++ri) {
      const size_t r = roots[ri], len = r - start[r] + 1;
      if (used[r] || skipped[r]) continue;
      std::vector<size_t> occ;
      for (size_t rj = ri; rj < roots.size(); ++rj) {
        const size_t q = roots[rj];
        if (q - start[q] + 1 != len || used[q] || skipped[q]) continue;
        if (same_range(start[r], start[q], len)) occ.push_back(q);
      }
      for (size_t q : occ) used[q] = 1;
      if (occ.size() < 2) continue;
      std::sort(occ.begin(), occ.end());
      const int k = out->n_saves++;
      save_end[occ[0]] = k + 1;
      for (size_t o = 1; o < occ.size(); ++o) {
        load_at[start[occ[o]]] = k + 1;
        load_root[start[occ[o]]] = occ[o];
        for (size_t i = start[occ[o]]; i <= occ[o]; ++i) skipped[i] = 1;
      }
    }
  }

  auto add_const = [&](float v) -> int {
    out->consts.push_back(v);
    return (int)out->consts.size() - 1;
  };
  auto emit = [&](uint32_t kind, int slot, uint32_t a0, uint32_t a1) {
    out->uops.push_back(uop_word(kind, (uint32_t)slot, a0, a1));
  };
  static const uint32_t kBin[5] = {K_ADD, K_SUB, K_MUL, K_DIV, K_POW};
  auto bin_index = [](uint32_t o) -> int {
    return o == OP_POW ? 4 : (int)(o - OP_ADD);
  };

  size_t pc = 0;
  // After each emitted group (fused groups never straddle the end of a saved
  // subtree, whose root is an operation that ends its group): keep the value.
  auto after = [&](size_t next) {
    const int k = save_end[next - 1];
    if (k) emit(k == 1 ? K_SAVE0 : K_SAVE1, before[start[next - 1]], 0, 0);
  };
  while (pc < n) {
    const uint32_t o = op[pc];
    if (load_at[pc]) {  // a later copy of a saved subtree
      const int k = load_at[pc];
      emit(k == 1 ? K_LOAD0 : K_LOAD1, before[pc], 0, 0);
      pc = load_root[pc] + 1;
      after(pc);
      continue;
    }
    if (omit[pc] || deferred[pc]) {  // the 1, EXP and ADD of a softplus; a deferred push
      ++pc;
      continue;
    }
    if (defer_kind[pc]) {
      const size_t src = defer_src[pc];
      emit((uint32_t)defer_kind[pc], before[src], arg[src], 0);
      ++pc;
      after(pc);
      continue;
    }
    if (softplus_kind[pc]) {
      emit((uint32_t)softplus_kind[pc], before[pc] - 1, 0, 0);
      ++pc;
      after(pc);
      continue;
    }
    // acc + p*x  or  acc + x*p  -> one multiply-add into the accumulator slot.
    if (pc + 3 < n && before[pc] >= 1 && op[pc + 2] == OP_MUL && op[pc + 3] == OP_ADD &&
        ((o == OP_PARAM && op[pc + 1] == OP_DATA && arg[pc + 1] <= (uint32_t)kMaxA1) ||
         (o == OP_DATA && op[pc + 1] == OP_PARAM && arg[pc] <= (uint32_t)kMaxA1))) {
      const uint32_t p = o == OP_PARAM ? arg[pc] : arg[pc + 1];
      const uint32_t x = o == OP_PARAM ? arg[pc + 1] : arg[pc];
      emit(K_FMA_PD, before[pc] - 1, p, x);
      pc += 4;
      after(pc);
      continue;
    }
    // push followed by the binary op that consumes it: fold the operand.
    if (is_push(o) && pc + 1 < n && is_binary(op[pc + 1])) {
      const uint32_t b = op[pc + 1];
      const int slot = before[pc] - 1;
      if (o == OP_CONST && b == OP_POW && consts[arg[pc]] == 2.0) {
        emit(K_SQR, slot, 0, 0);
      } else if (o == OP_CONST && b == OP_DIV && consts[arg[pc]] != 0.0 &&
                 std::isfinite(consts[arg[pc]]) &&
                 std::ldexp(1.0, std::ilogb(consts[arg[pc]])) ==
                     std::fabs(consts[arg[pc]])) {
        // Division by a power of two is exactly a multiply by its reciprocal.
        emit(K_MUL_C, slot, (uint32_t)add_const((float)(1.0 / consts[arg[pc]])), 0);
      } else {
        const uint32_t base = o == OP_CONST ? K_ADD_C : (o == OP_PARAM ? K_ADD_P : K_ADD_D);
        emit(base + (uint32_t)bin_index(b), slot, arg[pc], 0);
      }
      pc += 2;
      after(pc);
      continue;
    }
    switch (o) {
      case OP_CONST: emit(K_PUSH_C, before[pc], arg[pc], 0); break;
      case OP_PARAM: emit(K_PUSH_P, before[pc], arg[pc], 0); break;
      case OP_DATA: emit(K_PUSH_D, before[pc], arg[pc], 0); break;
      case OP_NEG: emit(K_NEG, before[pc] - 1, 0, 0); break;
      case OP_EXP: emit(K_EXP, before[pc] - 1, 0, 0); break;
      case OP_LOG: emit(K_LOG, before[pc] - 1, 0, 0); break;
      case OP_SQRT: emit(K_SQRT, before[pc] - 1, 0, 0); break;
      case OP_LGAMMA: emit(K_LGAMMA, before[pc] - 1, 0, 0); break;
      default: emit(kBin[bin_index(o)], before[pc] - 2, 0, 0); break;
    }
    ++pc;
    after(pc);
  }
  // Runs of multiply-adds into one slot become one K_DOT over a term table
  // (the same fmaf sequence in the same order, so the value is unchanged).
  {
    std::vector<uint32_t> merged;
    merged.reserve(out->uops.size());
    size_t i = 0;
    while (i < out->uops.size()) {
      const uint32_t w = out->uops[i];
      const uint32_t id = w & kCaseMask, kind = id % NKIND, slot = id / NKIND;
      size_t j = i + 1;
      if (kind == K_FMA_PD)
        while (j < out->uops.size() && (out->uops[j] & kCaseMask) == id &&
               j - i < (size_t)kDotCount)
          ++j;
      if (kind == K_FMA_PD && j - i >= 2 &&
          out->terms.size() + (j - i) + 1 <= (size_t)kMaxTerms) {
        // A parameter pushed into the same slot just before starts the sum.
        const bool from_param = !merged.empty() &&
                                (merged.back() & kCaseMask) == slot * NKIND + K_PUSH_P;
        const uint32_t t0 = (uint32_t)out->terms.size();
        if (from_param) {
          out->terms.push_back((merged.back() >> kCaseBits) & 0x7FFu);
          merged.pop_back();
        }
        for (size_t k = i; k < j; ++k)
          out->terms.push_back(((out->uops[k] >> kCaseBits) & 0x7FFu) |
                               ((out->uops[k] >> 22) << 11));
        uint32_t a1 = (uint32_t)(j - i);
        // A K_SAVE0 of the sum right after it becomes the K_DOT's save flag.
        if (j < out->uops.size() && (out->uops[j] & kCaseMask) == slot * NKIND + K_SAVE0) {
          a1 |= kDotSave;
          ++j;
        }
        merged.push_back(uop_word(from_param ? K_DOTP : K_DOT, slot, t0, a1));
        i = j;
      } else if (kind == K_LOAD0 && j < out->uops.size() &&
                 ((out->uops[j] & kCaseMask) == (slot - 1) * NKIND + K_SOFTPLUS1 ||
                  (out->uops[j] & kCaseMask) == slot * NKIND + K_SOFTPLUS ||
                  (out->uops[j] & kCaseMask) == slot * NKIND + K_EXP)) {
        // The loaded value feeds only this operation: read it from the save.
        const uint32_t nid = out->uops[j] & kCaseMask;
        const uint32_t nk = nid % NKIND, ns = nid / NKIND;
        merged.push_back(uop_word(nk == K_EXP ? K_EXP_SV : K_SOFTPLUS_SV, ns, 0, 0));
        i = j + 1;
      } else {
        merged.push_back(w);
        ++i;
      }
    }
    out->uops.swap(merged);
  }
  if ((int)out->uops.size() > kMaxUops) {
    *err = fmt("program compiles to %ld micro-ops, limit %ld", (long)out->uops.size(),
               kMaxUops);
    return 1;
  }
  if ((int)out->consts.size() > kMaxConsts) {
    *err = fmt("constant pool of %ld entries exceeds %ld", (long)out->consts.size(),
               kMaxConsts);
    return 1;
  }
  return 0;
}

int compile_grad_program(const uint32_t* code, size_t n_code, uint32_t n_params,
                         UGradProg* out, std::string* err) {
  *out = UGradProg();
  if (n_params > (uint32_t)kMaxGradParams) {
    *err = fmt("the interpreter's gradient takes at most %ld parameters (%ld here); the "
               "compiled engine has no such limit",
               kMaxGradParams, (long)n_params);
    return 1;
  }
  const size_t n = n_code / 2;
  std::vector<uint32_t> st;  // refs on the stack
  auto ref = [](uint32_t type, uint32_t idx) { return type | (idx << 2); };
  for (size_t pc = 0; pc < n; ++pc) {
    const uint32_t op = norm_op(code[2 * pc]), arg = code[2 * pc + 1];
    if (is_push(op)) {
      if (arg >= 4096) {
        *err = "operand index beyond the interpreter's gradient (4096)";
        return 1;
      }
      st.push_back(ref(op == OP_CONST ? GREF_CONST : op == OP_PARAM ? GREF_PARAM : GREF_DATA,
                       arg));
      continue;
    }
    if ((int)out->nodes.size() >= kMaxGradNodes) {
      *err = fmt("the interpreter's gradient takes at most %ld operations (more here); the "
                 "compiled engine has no such limit",
                 kMaxGradNodes);
      return 1;
    }
    uint32_t a = 0, b = 0;
    if (is_unary(op)) {
      a = st.back();
      st.pop_back();
    } else {
      b = st.back();
      st.pop_back();
      a = st.back();
      st.pop_back();
    }
    out->nodes.push_back(op | (a << 4) | (b << 18));
    st.push_back(ref(GREF_NODE, (uint32_t)out->nodes.size() - 1));
  }
  if (!st.empty()) {
    out->root = st.front();
    out->has_root = true;
  }
  return 0;
}

}  // namespace gpum

