// codegen.cpp -- bytecode -> CUDA C model functions (see codegen.hpp).
//
// Generated interface (all __device__ __forceinline__):
//   void   gm_mat_obs(const float* x, long long ld, float* m)  materialized
//          data-only operations of one observation (once per session)
//   void   gm_data(const float* xo, int T, float* d)     per observation
//   void   gm_data2(const float* xo, int T, float2* d)   observation pair
//   void   gm_hoist(const float* p, float* h)            per chain
//   float  gm_value(const float* d, const float* p, const float* h)
//   float2 gm_value2(const float2* d, const float2* pp, const float2* hh)
//   void   gm_value4l(const float* xo, const float* p, const float* h,
//                     float* out)  four observations, chain-lane body
//   float  gm_value_grad(d, p, h, float* gp, float* gh)  gp/gh accumulated
//   void   gm_value_grad4l(const float* xo, int nv, p, h, float* gp, float* gh,
//                          float* out)  four observations, chain-lane body
//   void   gm_hoist_grad(const float* p, const float* gh, float* gp)
//   double gm_prior(const double* p)
//   double gm_prior_grad(const double* p, double* g)     g accumulated
// `xo` points at this lane's observation in the shared-memory tile; column j
// is xo[j*GM_T] (data columns, then the materialized columns).
#include "codegen.hpp"

#include "program.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <sstream>
#include <tuple>

namespace gpum {

namespace {

enum : uint32_t { O_C = 0, O_P = 1, O_D = 2, O_ADD = 3, O_SUB = 4, O_MUL = 5, O_DIV = 6,
                  O_NEG = 7, O_EXP = 8, O_LOG = 9, O_SQRT = 10, O_POW = 11, O_LGAMMA = 12 };
enum : uint8_t { DEP_P = 1, DEP_D = 2 };

struct Node {
  uint32_t op;
  int a = -1, b = -1;
  uint32_t arg = 0;
  double c = 0.0;
  uint8_t dep = 0;
};

inline uint32_t norm(uint32_t op) { return (op <= O_SQRT || op == O_LGAMMA) ? op : O_POW; }
inline bool unary(uint32_t op) { return (op >= O_NEG && op <= O_SQRT) || op == O_LGAMMA; }

double fold(uint32_t op, double a, double b) {
  switch (op) {
    case O_ADD: return a + b;
    case O_SUB: return a - b;
    case O_MUL: return a * b;
    case O_DIV: return a / b;
    case O_NEG: return -a;
    case O_EXP: return std::exp(a);
    case O_LOG: return std::log(a);
    case O_SQRT: return std::sqrt(a);
    case O_LGAMMA: return std::lgamma(a);
    default: return std::pow(a, b);
  }
}

struct Graph {
  std::vector<Node> n;
  std::map<std::tuple<uint32_t, int, int, uint32_t, uint64_t>, int> memo;
  int add(Node x) {
    uint64_t bits = 0;
    if (x.op == O_C) std::memcpy(&bits, &x.c, sizeof bits);
    auto key = std::make_tuple(x.op, x.a, x.b, x.arg, bits);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
    n.push_back(x);
    memo[key] = (int)n.size() - 1;
    return (int)n.size() - 1;
  }
  // Build from a validated program; returns the root (or -1 if empty).
  int build(const uint32_t* code, size_t n_code, const double* consts) {
    std::vector<int> st;
    for (size_t pc = 0; pc < n_code / 2; ++pc) {
      const uint32_t op = norm(code[2 * pc]), arg = code[2 * pc + 1];
      Node x;
      x.op = op;
      if (op == O_C) {
        x.c = consts[arg];
        st.push_back(add(x));
      } else if (op == O_P || op == O_D) {
        x.arg = arg;
        x.dep = op == O_P ? DEP_P : DEP_D;
        st.push_back(add(x));
      } else if (unary(op)) {
        const int a = st.back();
        st.pop_back();
        if (n[a].op == O_C && n[a].dep == 0) {
          Node k;
          k.op = O_C;
          k.c = fold(op, n[a].c, 0.0);
          st.push_back(add(k));
        } else {
          x.a = a;
          x.dep = n[a].dep;
          st.push_back(add(x));
        }
      } else {
        const int b = st.back();
        st.pop_back();
        const int a = st.back();
        st.pop_back();
        if (n[a].op == O_C && n[b].op == O_C) {
          Node k;
          k.op = O_C;
          k.c = fold(op, n[a].c, n[b].c);
          st.push_back(add(k));
        } else {
          x.a = a;
          x.b = b;
          x.dep = n[a].dep | n[b].dep;
          st.push_back(add(x));
        }
      }
    }
    return st.empty() ? -1 : st.front();  // the result is slot 0
  }
  std::vector<char> reachable(int root) const {
    std::vector<char> r(n.size(), 0);
    if (root < 0) return r;
    r[root] = 1;
    for (int i = root; i >= 0; --i) {
      if (!r[i]) continue;
      if (n[i].a >= 0) r[n[i].a] = 1;
      if (n[i].b >= 0) r[n[i].b] = 1;
    }
    return r;
  }
};

std::string flit(double v) {
  const float f = (float)v;
  if (std::isnan(f)) return "__int_as_float(0x7fffffff)";
  if (std::isinf(f)) return f > 0 ? "__int_as_float(0x7f800000)" : "__int_as_float(0xff800000)";
  char buf[64];
  std::snprintf(buf, sizeof buf, "%af", (double)f);
  return buf;
}

std::string dlit(double v) {
  if (std::isnan(v)) return "__longlong_as_double(0x7fffffffffffffffll)";
  if (std::isinf(v))
    return v > 0 ? "__longlong_as_double(0x7ff0000000000000ll)"
                 : "__longlong_as_double(0xfff0000000000000ll)";
  char buf[64];
  std::snprintf(buf, sizeof buf, "%a", v);
  return buf;
}

bool is_const2(const Graph& g, int i) { return g.n[i].op == O_C && g.n[i].c == 2.0; }

// A constant divisor +-2^k whose reciprocal is a normal float: x / c and
// x * (1 / c) are the same correctly rounded value, so the division becomes
// a product.  Returns the reciprocal's literal, or "".
std::string pow2_recip(const Graph& g, int b) {
  if (b < 0 || g.n[b].op != O_C || g.n[b].c == 0.0 || !std::isfinite(g.n[b].c)) return "";
  int e = 0;
  const double m = std::frexp(g.n[b].c, &e);
  if (std::fabs(m) != 0.5 || e - 1 < -125 || e - 1 > 125) return "";
  return flit(1.0 / g.n[b].c);
}

// Emits the value of `i` from child names.
std::string op_expr(const Graph& g, int i, const std::string& a, const std::string& b,
                    bool f32) {
  const char* sfx = f32 ? "f" : "";
  switch (g.n[i].op) {
    case O_ADD: return "(" + a + " + " + b + ")";
    case O_SUB: return "(" + a + " - " + b + ")";
    case O_MUL: return "(" + a + " * " + b + ")";
    case O_DIV: {
      const std::string r = pow2_recip(g, g.n[i].b);
      if (!r.empty()) return "(" + a + " * " + (f32 ? r : dlit(1.0 / g.n[g.n[i].b].c)) + ")";
      return "(" + a + " / " + b + ")";
    }
    case O_NEG: return "(-" + a + ")";
    case O_EXP: return std::string("exp") + sfx + "(" + a + ")";
    case O_LOG: return std::string("log") + sfx + "(" + a + ")";
    case O_SQRT: return std::string("sqrt") + sfx + "(" + a + ")";
    case O_LGAMMA: return std::string("lgamma") + sfx + "(" + a + ")";
    default:
      if (is_const2(g, g.n[i].b)) return "(" + a + " * " + a + ")";
      return std::string("pow") + sfx + "(" + a + ", " + b + ")";
  }
}

// Paired (float2) value of `i` from child names: two observations at once.
std::string op_expr2(const Graph& g, int i, const std::string& a, const std::string& b) {
  switch (g.n[i].op) {
    case O_ADD: return "gm2_add(" + a + ", " + b + ")";
    case O_SUB: return "gm2_sub(" + a + ", " + b + ")";
    case O_MUL: return "gm2_mul(" + a + ", " + b + ")";
    case O_DIV: {
      const std::string r = pow2_recip(g, g.n[i].b);
      if (!r.empty()) return "gm2_mul(" + a + ", gm2(" + r + "))";
      return "gm2_div(" + a + ", " + b + ")";
    }
    case O_NEG: return "gm2_neg(" + a + ")";
    case O_EXP: return "gm2_exp(" + a + ")";
    case O_LOG: return "gm2_log(" + a + ")";
    case O_SQRT: return "gm2_sqrt(" + a + ")";
    case O_LGAMMA: return "gm2_lgamma(" + a + ")";
    default:
      if (is_const2(g, g.n[i].b)) return "gm2_mul(" + a + ", " + a + ")";
      return "gm2_pow(" + a + ", " + b + ")";
  }
}

// Local-derivative contributions of node i with adjoint `G` to its children,
// as (child, expression) pairs (cpu_native.rs:217-277).  `rb`, when given, is
// the reciprocal of a DIV node's divisor (the divisions become products).
std::vector<std::pair<int, std::string>> adjoints(const Graph& g, int i, const std::string& G,
                                                  const std::string& v, const std::string& a,
                                                  const std::string& b, bool f32,
                                                  const std::string& rb = "") {
  const Node& x = g.n[i];
  const std::string one = f32 ? "1.0f" : "1.0";
  const std::string half = f32 ? "0.5f" : "0.5";
  const std::string zero = f32 ? "0.0f" : "0.0";
  const char* sfx = f32 ? "f" : "";
  std::vector<std::pair<int, std::string>> out;
  switch (x.op) {
    case O_ADD: out = {{x.a, G}, {x.b, G}}; break;
    case O_SUB: out = {{x.a, G}, {x.b, "(-" + G + ")"}}; break;
    case O_MUL: out = {{x.a, G + " * " + b}, {x.b, G + " * " + a}}; break;
    case O_DIV:
      if (!rb.empty())
        out = {{x.a, G + " * " + rb}, {x.b, "(-" + G + " * " + v + " * " + rb + ")"}};
      else
        out = {{x.a, G + " / " + b}, {x.b, "(-" + G + " * " + v + " / " + b + ")"}};
      break;
    case O_NEG: out = {{x.a, "(-" + G + ")"}}; break;
    case O_EXP: out = {{x.a, G + " * " + v}}; break;
    case O_LOG: out = {{x.a, G + " / " + a}}; break;
    case O_SQRT: out = {{x.a, G + " * " + half + " / " + v}}; break;
    case O_LGAMMA:
      out = {{x.a, G + " * " + std::string(f32 ? "gm_digammaf(" : "gm_digamma(") + a + ")"}};
      break;
    default:
      if (is_const2(g, x.b)) {
        out = {{x.a, G + " * " + (f32 ? std::string("2.0f") : std::string("2.0")) + " * " + a}};
      } else {
        out = {{x.a, G + " * " + b + " * pow" + sfx + "(" + a + ", " + b + " - " + one + ")"},
               {x.b, "((" + a + " > " + zero + ") ? " + G + " * " + v + " * log" + sfx + "(" +
                         a + ") : " + zero + ")"}};
      }
      break;
  }
  return out;
}

}  // namespace

int generate_model(const uint32_t* code, size_t n_code, const double* consts,
                   const uint32_t* prior_code, size_t n_prior, const double* prior_consts,
                   uint32_t n_params, uint32_t n_cols, GenModel* out, std::string* err) {
  *out = GenModel();
  Graph g;
  const int root = g.build(code, n_code, consts);
  const std::vector<char> live = g.reachable(root);
  const int N = (int)g.n.size();

  // Names and storage classes.
  std::vector<std::string> name(N);
  std::vector<int> hslot(N, -1), dslot(N, -1);
  std::set<int> need_h, need_d;  // referenced from per-observation code
  auto is_pd = [&](int i) { return g.n[i].dep == (DEP_P | DEP_D); };
  auto is_h = [&](int i) { return g.n[i].dep == DEP_P && g.n[i].op != O_P; };
  auto is_d = [&](int i) { return g.n[i].dep == DEP_D; };
  for (int i = 0; i < N; ++i) {
    if (!live[i]) continue;
    if (is_pd(i)) {
      for (int c : {g.n[i].a, g.n[i].b}) {
        if (c < 0) continue;
        if (is_h(c)) need_h.insert(c);
        if (is_d(c)) need_d.insert(c);
      }
    }
  }
  if (root >= 0 && is_h(root)) need_h.insert(root);
  if (root >= 0 && is_d(root)) need_d.insert(root);
  for (int i : need_h) hslot[i] = out->n_hoist++;
  // Division by a parameter-only value (exp(ls), a parameter, ...): the value
  // functions multiply by its reciprocal, hoisted once per chain into a slot
  // of its own (the gradient keeps the division and its adjoints).
  std::vector<int> rslot(N, -1);
  for (int i = 0; i < N; ++i) {
    if (!live[i] || g.n[i].dep != (DEP_P | DEP_D) || g.n[i].op != O_DIV) continue;
    const int b = g.n[i].b;
    if (b >= 0 && g.n[b].dep == DEP_P && rslot[b] < 0) rslot[b] = out->n_hoist++;
  }
  auto recip = [&](int i) {  // hoisted reciprocal slot of node i's divisor, or -1
    const Node& x = g.n[i];
    return x.op == O_DIV && x.b >= 0 ? rslot[x.b] : -1;
  };
  for (int i : need_d) dslot[i] = out->n_data++;
  // Data-only operations that per-observation code reads (lgamma(y + 1),
  // x^2, ...) are computed once per session into extra f32 columns n_cols,
  // n_cols + 1, ... (gm_mat_obs below); every per-observation function then
  // loads them like data columns.  col_of(i): the column of a data value.
  std::vector<int> mcol(N, -1);
  for (int i : need_d)
    if (g.n[i].op != O_D) mcol[i] = (int)n_cols + out->n_mat++;
  auto col_of = [&](int i) { return g.n[i].op == O_D ? (int)g.n[i].arg : mcol[i]; };
  for (int i = 0; i < N; ++i) {
    const Node& x = g.n[i];
    if (x.op == O_C) name[i] = flit(x.c);
    else if (x.op == O_P) name[i] = "p[" + std::to_string(x.arg) + "]";
    else name[i] = "v" + std::to_string(i);
  }
  auto ref_obs = [&](int i) -> std::string {  // name inside per-observation code
    if (hslot[i] >= 0) return "h[" + std::to_string(hslot[i]) + "]";
    if (dslot[i] >= 0) return "d[" + std::to_string(dslot[i]) + "]";
    return name[i];
  };

  // Use counts, and LOG(1 + EXP(a)) chains whose inner nodes feed nothing
  // else: the value functions evaluate them as one accurate softplus(a).
  std::vector<int> uses(N, 0);
  for (int i = 0; i < N; ++i) {
    if (!live[i]) continue;
    if (g.n[i].a >= 0) ++uses[g.n[i].a];
    if (g.n[i].b >= 0) ++uses[g.n[i].b];
  }
  if (root >= 0) ++uses[root];
  std::vector<int> softplus_arg(N, -1);
  std::vector<char> softplus_inner(N, 0);
  auto is_one = [&](int i) { return i >= 0 && g.n[i].op == O_C && g.n[i].c == 1.0; };
  for (int i = 0; i < N; ++i) {
    if (!live[i] || !is_pd(i) || g.n[i].op != O_LOG) continue;
    const int j = g.n[i].a;
    if (!is_pd(j) || g.n[j].op != O_ADD || uses[j] != 1) continue;
    const int k = is_one(g.n[j].a) ? g.n[j].b : (is_one(g.n[j].b) ? g.n[j].a : -1);
    if (k < 0 || !is_pd(k) || g.n[k].op != O_EXP || uses[k] != 1) continue;
    softplus_arg[i] = g.n[k].a;
    softplus_inner[j] = softplus_inner[k] = 1;
  }

  // LOG(X + Y) with X, Y scaled exponentials (EXP(a), EXP(a) * c, c * EXP(a)
  // or EXP(a) / c; c a parameter-only or constant weight that is positive by
  // construction) feeding nothing else: the value functions evaluate it as
  // logaddexp(a +- log c1, b +- log c2), the log weights hoisted per chain.
  std::vector<int> pos_memo(N, -1);
  std::function<bool(int)> positive = [&](int i) -> bool {
    if (i < 0) return false;
    if (pos_memo[i] >= 0) return pos_memo[i] != 0;
    const Node& x = g.n[i];
    bool r = false;
    if (x.op == O_C) r = x.c > 0.0;
    else if (x.dep != DEP_P) r = false;
    else if (x.op == O_EXP) r = true;
    else if (x.op == O_ADD || x.op == O_MUL || x.op == O_DIV) r = positive(x.a) && positive(x.b);
    else if (x.op == O_SQRT) r = positive(x.a);
    pos_memo[i] = r ? 1 : 0;
    return r;
  };
  struct ScaledExp {
    int expo = -1, exp_node = -1, weight = -1, sign = 1;
  };
  auto scaled_exp = [&](int X, ScaledExp* o) -> bool {
    if (X < 0 || !is_pd(X) || uses[X] != 1) return false;
    const Node& x = g.n[X];
    auto is_exp = [&](int e) { return e >= 0 && g.n[e].op == O_EXP && is_pd(e) && uses[e] == 1; };
    if (x.op == O_EXP && is_exp(X)) {
      *o = ScaledExp{x.a, X, -1, 1};
      return true;
    }
    if (x.op == O_MUL) {
      for (int side = 0; side < 2; ++side) {
        const int e = side ? x.b : x.a, c = side ? x.a : x.b;
        if (is_exp(e) && positive(c)) {
          *o = ScaledExp{g.n[e].a, e, c, 1};
          return true;
        }
      }
    }
    if (x.op == O_DIV && is_exp(x.a) && positive(x.b)) {
      *o = ScaledExp{g.n[x.a].a, x.a, x.b, -1};
      return true;
    }
    return false;
  };
  std::vector<ScaledExp> lse_x(N), lse_y(N);
  std::vector<char> lse(N, 0), lse_skip(N, 0);
  std::vector<int> lslot(N, -1);
  for (int i = 0; i < N; ++i) {
    if (!live[i] || !is_pd(i) || g.n[i].op != O_LOG || softplus_arg[i] >= 0) continue;
    const int j = g.n[i].a;
    if (j < 0 || !is_pd(j) || g.n[j].op != O_ADD || uses[j] != 1) continue;
    ScaledExp X, Y;
    if (!scaled_exp(g.n[j].a, &X) || !scaled_exp(g.n[j].b, &Y)) continue;
    lse[i] = 1;
    lse_x[i] = X;
    lse_y[i] = Y;
    lse_skip[j] = lse_skip[g.n[j].a] = lse_skip[g.n[j].b] = 1;
    lse_skip[X.exp_node] = lse_skip[Y.exp_node] = 1;
    for (int w : {X.weight, Y.weight})
      if (w >= 0 && g.n[w].op != O_C && lslot[w] < 0) lslot[w] = out->n_hoist++;
  }
  // The term a +- log c of a scaled exponential, for a given reference to a.
  auto lse_term = [&](const ScaledExp& e, const std::string& a, bool paired,
                      const std::string& hname) -> std::string {
    if (e.weight < 0) return a;
    const Node& w = g.n[e.weight];
    const std::string lw =
        w.op == O_C ? (paired ? "gm2(" + flit(std::log(w.c)) + ")" : flit(std::log(w.c)))
                    : hname + "[" + std::to_string(lslot[e.weight]) + "]";
    if (paired) return std::string(e.sign > 0 ? "gm2_add(" : "gm2_sub(") + a + ", " + lw + ")";
    return "(" + a + (e.sign > 0 ? " + " : " - ") + lw + ")";
  };

  // Linear predictor for the tensor cores: the per-observation node with the
  // most data columns that is affine in the data with parameter-only
  // coefficients, sum_c coef_c(theta) x_c + offset(theta).  Over a tile of
  // observations and a block of chains it is a matrix product (chains x
  // columns times columns x observations); the value kernel gm_iter_value_tc
  // runs it on the tensor cores and evaluates the rest of the expression
  // (the tail, gm_tc_tail2) with the node replaced by its product.
  struct AffTerm {
    double c;
    int pn;  // c * value(pn); pn = -1: the constant c
  };
  struct Aff {
    bool ok = false;
    std::map<int, std::vector<AffTerm>> col;  // data column -> coefficient terms
    std::vector<AffTerm> off;
  };
  std::vector<Aff> aff(N);
  auto scaled = [](const std::vector<AffTerm>& v, double c, int pn) {
    std::vector<AffTerm> o;
    for (const AffTerm& t : v) {
      if (pn >= 0 && t.pn >= 0) return std::vector<AffTerm>{{0.0, -2}};  // product of two
      o.push_back({t.c * c, pn >= 0 ? pn : t.pn});
    }
    return o;
  };
  auto bad_terms = [](const std::vector<AffTerm>& v) {
    for (const AffTerm& t : v)
      if (t.pn == -2) return true;
    return false;
  };
  for (int i = 0; i < N; ++i) {
    if (!live[i]) continue;
    const Node& x = g.n[i];
    Aff& r = aff[i];
    if (x.op == O_C) {
      r.ok = true;
      r.off.push_back({x.c, -1});
    } else if ((x.dep & DEP_D) == 0) {  // parameter-only
      r.ok = true;
      r.off.push_back({1.0, i});
    } else if (is_d(i)) {  // a data column (given or materialized)
      const int c = col_of(i);
      if (c >= 0) {
        r.ok = true;
        r.col[c].push_back({1.0, -1});
      }
    } else if ((x.op == O_ADD || x.op == O_SUB) && aff[x.a].ok && aff[x.b].ok) {
      r = aff[x.a];
      const double sg = x.op == O_ADD ? 1.0 : -1.0;
      for (auto& kv : aff[x.b].col)
        for (const AffTerm& t : kv.second) r.col[kv.first].push_back({sg * t.c, t.pn});
      for (const AffTerm& t : aff[x.b].off) r.off.push_back({sg * t.c, t.pn});
    } else if (x.op == O_NEG && aff[x.a].ok) {
      r = aff[x.a];
      for (auto& kv : r.col)
        for (AffTerm& t : kv.second) t.c = -t.c;
      for (AffTerm& t : r.off) t.c = -t.c;
    } else if (x.op == O_MUL && aff[x.a].ok && aff[x.b].ok) {
      // one side free of data: scale the other side by it
      const bool a_scalar = (g.n[x.a].dep & DEP_D) == 0, b_scalar = (g.n[x.b].dep & DEP_D) == 0;
      if (a_scalar == b_scalar) continue;
      const int k = a_scalar ? x.a : x.b, o = a_scalar ? x.b : x.a;
      const double kc = g.n[k].op == O_C ? g.n[k].c : 1.0;
      const int kp = g.n[k].op == O_C ? -1 : k;
      Aff t;
      t.ok = true;
      for (auto& kv : aff[o].col) t.col[kv.first] = scaled(kv.second, kc, kp);
      t.off = scaled(aff[o].off, kc, kp);
      bool bad = bad_terms(t.off);
      for (auto& kv : t.col) bad = bad || bad_terms(kv.second);
      if (!bad) r = t;
    } else if (x.op == O_DIV && aff[x.a].ok && (g.n[x.a].dep & DEP_D) && g.n[x.b].op == O_C &&
               g.n[x.b].c != 0.0 && std::isfinite(g.n[x.b].c)) {
      // division by a constant: the coefficients scaled by its reciprocal
      const double kc = 1.0 / g.n[x.b].c;
      for (auto& kv : aff[x.a].col) r.col[kv.first] = scaled(kv.second, kc, -1);
      r.off = scaled(aff[x.a].off, kc, -1);
      r.ok = true;
    }
  }
  int tc_root = -1;
  for (int i = 0; i < N; ++i) {
    if (!live[i] || !is_pd(i) || !aff[i].ok) continue;
    if (tc_root < 0 || aff[i].col.size() >= aff[tc_root].col.size()) tc_root = i;
  }
  std::vector<char> in_tc(N, 0);  // nodes of the linear predictor's subtree
  if (tc_root >= 0) {
    in_tc[tc_root] = 1;
    for (int i = tc_root; i >= 0; --i) {
      if (!in_tc[i]) continue;
      if (g.n[i].a >= 0) in_tc[g.n[i].a] = 1;
      if (g.n[i].b >= 0) in_tc[g.n[i].b] = 1;
    }
    bool ok = aff[tc_root].col.size() >= 6;
    // per-observation values inside the subtree must feed nothing outside it
    for (int i = 0; i < N && ok; ++i) {
      if (!live[i] || in_tc[i]) continue;
      for (int c : {g.n[i].a, g.n[i].b})
        if (c >= 0 && c != tc_root && in_tc[c] && is_pd(c)) ok = false;
    }
    if (!ok) tc_root = -1;
  }
  std::vector<int> tc_cols;  // column of each product column (-1: the ones column)
  if (tc_root >= 0) {
    for (auto& kv : aff[tc_root].col) tc_cols.push_back(kv.first);
    bool has_off = false;
    for (const AffTerm& t : aff[tc_root].off) has_off = has_off || t.pn >= 0 || t.c != 0.0;
    if (has_off) tc_cols.push_back(-1);
    if (tc_cols.size() > 96) tc_root = -1;  // the shared-memory operands' limit
  }

  std::ostringstream s;
  s << "#define GM_NP " << n_params << "\n";
  s << "#define GM_NH " << std::max(1, out->n_hoist) << "\n";
  s << "#define GM_ND " << std::max(1, out->n_data) << "\n";
  // The tile height is fixed by the column count, so column offsets are
  // compile-time immediates in the generated loads.
  s << "#define GM_T " << tile_obs(n_cols + (uint32_t)out->n_mat) << "\n";
  s << "#define GM_NCOLS " << n_cols << "\n";
  s << "#define GM_NMAT " << std::max(1, out->n_mat) << "\n";
  s << "#define GM_HAS_MAT " << (out->n_mat > 0 ? 1 : 0) << "\n";

  // gm_mat_obs: the materialized data-only operations of one observation
  // from its data columns (x[j * ld]), computed as the per-observation code
  // would compute them.
  s << "__device__ __forceinline__ void gm_mat_obs(const float* __restrict__ x, long long ld, "
       "float* __restrict__ m) {\n";
  for (int i = 0; i < N; ++i) {
    if (!live[i] || !is_d(i)) continue;
    const Node& x = g.n[i];
    std::string e = x.op == O_D ? "x[" + std::to_string(x.arg) + " * ld]"
                                : op_expr(g, i, name[x.a], x.b >= 0 ? name[x.b] : "", true);
    s << "  const float " << name[i] << " = " << e << ";\n";
    if (mcol[i] >= 0) s << "  m[" << mcol[i] - (int)n_cols << "] = " << name[i] << ";\n";
  }
  s << "  (void)x; (void)ld; (void)m;\n}\n";

  // gm_data: the data values per-observation code reads, one observation.
  s << "__device__ __forceinline__ void gm_data(const float* __restrict__ xo, int T, "
       "float* __restrict__ d) {\n";
  for (int i : need_d)
    s << "  d[" << dslot[i] << "] = xo[" << col_of(i) << " * GM_T];\n";
  s << "  (void)xo; (void)T; (void)d;\n}\n";

  // gm_hoist: parameter-only subexpressions, once per chain.
  auto emit_hoist_body = [&](std::ostringstream& o) {
    for (int i = 0; i < N; ++i) {
      if (!live[i] || !is_h(i)) continue;
      const Node& x = g.n[i];
      o << "  const float " << name[i] << " = "
        << op_expr(g, i, name[x.a], x.b >= 0 ? name[x.b] : "", true) << ";\n";
    }
  };
  s << "__device__ __forceinline__ void gm_hoist(const float* __restrict__ p, "
       "float* __restrict__ h) {\n";
  emit_hoist_body(s);
  for (int i : need_h) s << "  h[" << hslot[i] << "] = " << name[i] << ";\n";
  for (int i = 0; i < N; ++i)
    if (rslot[i] >= 0) s << "  h[" << rslot[i] << "] = 1.0f / " << name[i] << ";\n";
  for (int i = 0; i < N; ++i)
    if (lslot[i] >= 0) s << "  h[" << lslot[i] << "] = logf(" << name[i] << ");\n";
  s << "  (void)p; (void)h;\n}\n";

  // Per-observation forward code (`fused`: with the softplus rewrite, for
  // the value functions; the gradient keeps every node).
  auto emit_fwd = [&](std::ostringstream& o, bool fused) {
    for (int i = 0; i < N; ++i) {
      if (!live[i] || !is_pd(i)) continue;
      if (fused && (softplus_inner[i] || lse_skip[i])) continue;
      const Node& x = g.n[i];
      if (fused && lse[i]) {
        o << "  const float " << name[i] << " = gm_logaddexp("
          << lse_term(lse_x[i], ref_obs(lse_x[i].expo), false, "h") << ", "
          << lse_term(lse_y[i], ref_obs(lse_y[i].expo), false, "h") << ");\n";
        ++out->n_fwd;
        continue;
      }
      o << "  const float " << name[i] << " = "
        << (fused && softplus_arg[i] >= 0
                ? "gm_softplus(" + ref_obs(softplus_arg[i]) + ")"
                : fused && recip(i) >= 0
                      ? "(" + ref_obs(x.a) + " * h[" + std::to_string(recip(i)) + "])"
                      : op_expr(g, i, ref_obs(x.a), x.b >= 0 ? ref_obs(x.b) : "", true))
        << ";\n";
      ++out->n_fwd;
    }
  };
  const std::string rootv = root < 0 ? std::string("0.0f") : ref_obs(root);
  s << "__device__ __forceinline__ float gm_value(const float* __restrict__ d, "
       "const float* __restrict__ p, const float* __restrict__ h) {\n";
  emit_fwd(s, true);
  s << "  (void)d; (void)p; (void)h;\n  return " << rootv << ";\n}\n";

  // gm_value4l: four consecutive observations xo .. xo + 3 (the chain-lane
  // body), evaluated node by node in lockstep so that only the running
  // values stay live; each data column is loaded (16 bytes, a broadcast: every
  // lane reads the same address) at its first use, materialized data-only
  // operations included.  xo is 16-byte aligned: a multiple of 4 observations
  // into a tile whose column stride GM_T * 4 is a multiple of 128 bytes.
  s << "__device__ __forceinline__ void gm_value4l(const float* __restrict__ xo, "
       "const float* __restrict__ p, const float* __restrict__ h, "
       "float* __restrict__ out) {\n";
  {
    std::vector<char> loaded(N, 0);
    auto ref4 = [&](int i, int k) -> std::string {
      const Node& x = g.n[i];
      if (x.op == O_C) return name[i];
      if (hslot[i] >= 0) return "h[" + std::to_string(hslot[i]) + "]";
      if (x.op == O_P) return name[i];
      if (dslot[i] >= 0) {
        if (!loaded[i]) {
          s << "  const float4 q_" << name[i] << " = *reinterpret_cast<const float4*>(xo + "
            << col_of(i) << " * GM_T);\n";
          loaded[i] = 1;
        }
        return "q_" + name[i] + "." + "xyzw"[k];
      }
      return name[i] + "_" + std::to_string(k);
    };
    for (int i = 0; i < N; ++i) {
      if (!live[i] || !is_pd(i) || softplus_inner[i] || lse_skip[i]) continue;
      const Node& x = g.n[i];
      if (lse[i]) {
        std::string ta[4], tb[4];
        for (int k = 0; k < 4; ++k) {
          ta[k] = lse_term(lse_x[i], ref4(lse_x[i].expo, k), false, "h");
          tb[k] = lse_term(lse_y[i], ref4(lse_y[i].expo, k), false, "h");
        }
        for (int k = 0; k < 4; ++k)
          s << "  const float " << name[i] << "_" << k << " = gm_logaddexp(" << ta[k] << ", "
            << tb[k] << ");\n";
        continue;
      }
      std::string a[4], b[4];
      for (int k = 0; k < 4; ++k) {  // loads first, so they precede the four uses
        const int ca = softplus_arg[i] >= 0 ? softplus_arg[i] : x.a;
        a[k] = ref4(ca, k);
        if (softplus_arg[i] < 0 && x.b >= 0) b[k] = ref4(x.b, k);
      }
      for (int k = 0; k < 4; ++k)
        s << "  const float " << name[i] << "_" << k << " = "
          << (softplus_arg[i] >= 0 ? "gm_softplus(" + a[k] + ")"
              : recip(i) >= 0      ? "(" + a[k] + " * h[" + std::to_string(recip(i)) + "])"
                                   : op_expr(g, i, a[k], b[k], true))
          << ";\n";
    }
    for (int k = 0; k < 4; ++k)
      s << "  out[" << k << "] = " << (root < 0 ? std::string("0.0f") : ref4(root, k))
        << ";\n";
  }
  s << "  (void)xo; (void)p; (void)h;\n}\n";

  // Paired versions (two observations per call) of gm_data and gm_value.
  // Leaves that do not depend on the observation (constants, parameters,
  // hoisted values) appear as broadcast pairs; a product used only by one sum
  // is fused into it (FFMA2), the contraction the scalar code gets from
  // --fmad=true.
  {
    auto ref2 = [&](int i) -> std::string {
      const Node& x = g.n[i];
      if (x.op == O_C) return "gm2(" + flit(x.c) + ")";
      if (x.op == O_P) return "pp[" + std::to_string(x.arg) + "]";
      if (hslot[i] >= 0) return "hh[" + std::to_string(hslot[i]) + "]";
      if (dslot[i] >= 0) return "d[" + std::to_string(dslot[i]) + "]";
      return name[i];
    };
    s << "__device__ __forceinline__ void gm_data2(const float* __restrict__ xo, int T, "
         "float2* __restrict__ d) {\n";
    for (int i : need_d)
      s << "  d[" << dslot[i] << "] = *reinterpret_cast<const float2*>(xo + " << col_of(i)
        << " * GM_T);\n";
    s << "  (void)xo; (void)T; (void)d;\n}\n";
    auto fusable = [&](int c) {
      return c >= 0 && is_pd(c) && g.n[c].op == O_MUL && uses[c] == 1 && c != root;
    };
    std::vector<char> fused(N, 0);
    for (int i = 0; i < N; ++i) {
      if (!live[i] || !is_pd(i) || g.n[i].op != O_ADD) continue;
      if (fusable(g.n[i].a)) fused[g.n[i].a] = 1;
      else if (fusable(g.n[i].b)) fused[g.n[i].b] = 1;
    }
    // x * y - softplus(a), with the product and the softplus feeding nothing
    // else, is one gm2_fma_nsoftplus (value functions only).
    std::vector<char> nsp_fold(N, 0), nsp_skip(N, 0);
    for (int i = 0; i < N; ++i) {
      if (!live[i] || !is_pd(i) || g.n[i].op != O_SUB) continue;
      const int a = g.n[i].a, b = g.n[i].b;
      if (!fusable(a) || fused[a] || b < 0 || softplus_arg[b] < 0 || uses[b] != 1 || b == root)
        continue;
      nsp_fold[i] = 1;
      nsp_skip[a] = nsp_skip[b] = 1;
    }
    // The paired value of node i with the references R (rewrites included);
    // value_node(i): whether the paired value function evaluates node i.
    auto value_node = [&](int i) {
      return live[i] && is_pd(i) && !fused[i] && !softplus_inner[i] && !nsp_skip[i] &&
             !lse_skip[i];
    };
    auto value2_expr = [&](int i, const std::function<std::string(int)>& R) -> std::string {
      const Node& x = g.n[i];
      if (lse[i])
        return "gm2_logaddexp(" + lse_term(lse_x[i], R(lse_x[i].expo), true, "hh") + ", " +
               lse_term(lse_y[i], R(lse_y[i].expo), true, "hh") + ")";
      if (nsp_fold[i]) {
        const Node& m = g.n[x.a];
        return "gm2_fma_nsoftplus(" + R(m.a) + ", " + R(m.b) + ", " + R(softplus_arg[x.b]) + ")";
      }
      if (softplus_arg[i] >= 0) return "gm2_softplus(" + R(softplus_arg[i]) + ")";
      if (recip(i) >= 0) return "gm2_mul(" + R(x.a) + ", hh[" + std::to_string(recip(i)) + "])";
      if (x.op == O_ADD && (fused[x.a] || (x.b >= 0 && fused[x.b]))) {
        const int m = fused[x.a] ? x.a : x.b, o = fused[x.a] ? x.b : x.a;
        return "gm2_fma(" + R(g.n[m].a) + ", " + R(g.n[m].b) + ", " + R(o) + ")";
      }
      return op_expr2(g, i, R(x.a), x.b >= 0 ? R(x.b) : "");
    };
    s << "__device__ __forceinline__ float2 gm_value2(const float2* __restrict__ d, "
         "const float2* __restrict__ pp, const float2* __restrict__ hh) {\n";
    for (int i = 0; i < N; ++i)
      if (value_node(i))
        s << "  const float2 " << name[i] << " = " << value2_expr(i, ref2) << ";\n";
    const std::string root2 = root < 0 ? std::string("gm2(0.0f)") : ref2(root);
    s << "  (void)d; (void)pp; (void)hh;\n  return " << root2 << ";\n}\n";

    // The tensor-core value path.  A linear predictor that is itself a
    // product folded into an FFMA2 of its consumer keeps the FP32 path.
    if (tc_root >= 0 && fused[tc_root]) tc_root = -1;
    if (tc_root >= 0) {
      // gm_tc_tail2: the paired value with the linear predictor's pair `eta`;
      // t[k] = the k-th data column the tail reads (gm_tc_tailvals).
      std::vector<int> tslot(N, -1), tail_cols;
      auto refT = [&](int i) -> std::string {
        if (i == tc_root) return "eta";
        const Node& x = g.n[i];
        if (x.op == O_C) return "gm2(" + flit(x.c) + ")";
        if (x.op == O_P) return "pp[" + std::to_string(x.arg) + "]";
        if (hslot[i] >= 0) return "hh[" + std::to_string(hslot[i]) + "]";
        if (dslot[i] >= 0) {
          if (tslot[i] < 0) {
            tslot[i] = (int)tail_cols.size();
            tail_cols.push_back(col_of(i));
          }
          return "t[" + std::to_string(tslot[i]) + "]";
        }
        return name[i];
      };
      std::ostringstream body;
      for (int i = 0; i < N; ++i)
        if (value_node(i) && !in_tc[i])
          body << "  const float2 " << name[i] << " = " << value2_expr(i, refT) << ";\n";
      const std::string rootT = refT(root);
      const int K = (int)tc_cols.size(), KP = (K + 7) / 8 * 8, NT = (int)tail_cols.size();
      // Observations per tile and pipeline stages: the largest that fit
      // shared memory (stages of [hi | lo | tail] x TN, the coefficient
      // operand [hi | lo] x 128 chains, the reduction buffer).
      // Epilogue warps: four per column part, each part a multiple of 16
      // columns of the tile.
      int EW = 16;
      if (const char* e = std::getenv("GPUM_B200_TC_WARPS")) {
        const int v = std::atoi(e);
        if (v == 8 || v == 12 || v == 16) EW = v;
      }
      const int parts = EW / 4;
      int TN = 0, S = 0;
      for (int tn = 256 / (16 * parts) * (16 * parts); tn >= 16 * parts && !TN; tn -= 16 * parts) {
        for (int st : {3, 2}) {
          if (tc_smem_bytes(KP, NT, tn, st) <= 231424) {
            TN = tn;
            S = st;
            break;
          }
        }
      }
      if (TN == 0) tc_root = -1;
      if (tc_root >= 0) {
        out->tc = true;
        out->tc_k = K;
        out->tc_kp = KP;
        out->tc_ntail = NT;
        out->tc_tn = TN;
        out->tc_stages = S;
        out->tc_warps = EW;
        s << "#define GM_TC 1\n#define GM_TC_EW " << EW << "\n#define GM_TC_K " << K
          << "\n#define GM_TC_KP " << KP
          << "\n#define GM_TC_NTAIL " << NT << "\n#define GM_TC_NT1 " << std::max(NT, 1)
          << "\n#define GM_TC_TN " << TN << "\n#define GM_TC_STAGES " << S << "\n";
        // gm_tc_colvals / gm_tc_tailvals: one observation's product columns
        // and tail columns from the column-major data (x[c * ld]).
        s << "__device__ __forceinline__ void gm_tc_colvals(const float* __restrict__ x, "
             "long long ld, float* __restrict__ v) {\n";
        for (int k = 0; k < K; ++k)
          s << "  v[" << k << "] = "
            << (tc_cols[k] < 0 ? std::string("1.0f")
                               : "x[" + std::to_string(tc_cols[k]) + " * ld]")
            << ";\n";
        s << "  (void)x; (void)ld;\n}\n";
        s << "__device__ __forceinline__ void gm_tc_tailvals(const float* __restrict__ x, "
             "long long ld, float* __restrict__ t) {\n";
        for (int k = 0; k < NT; ++k)
          s << "  t[" << k << "] = x[" << tail_cols[k] << " * ld];\n";
        s << "  (void)x; (void)ld; (void)t;\n}\n";
        // gm_tc_coef: the coefficients of one chain (the ones column's is the
        // offset), from its parameters.
        s << "__device__ __forceinline__ void gm_tc_coef(const float* __restrict__ p, "
             "float* __restrict__ a) {\n";
        emit_hoist_body(s);
        auto term_sum = [&](const std::vector<AffTerm>& ts) {
          std::string e;
          for (const AffTerm& t : ts) {
            std::string v = t.pn < 0 ? flit(t.c)
                            : t.c == 1.0 ? name[t.pn]
                            : t.c == -1.0 ? "(-" + name[t.pn] + ")"
                                          : "(" + flit(t.c) + " * " + name[t.pn] + ")";
            e = e.empty() ? v : "(" + e + " + " + v + ")";
          }
          return e.empty() ? std::string("0.0f") : e;
        };
        for (int k = 0; k < K; ++k)
          s << "  a[" << k << "] = "
            << term_sum(tc_cols[k] < 0 ? aff[tc_root].off : aff[tc_root].col[tc_cols[k]])
            << ";\n";
        s << "  (void)p;\n}\n";
        s << "__device__ __forceinline__ float2 gm_tc_tail2(float2 eta, "
             "const float2* __restrict__ t, const float2* __restrict__ pp, "
             "const float2* __restrict__ hh) {\n"
          << body.str() << "  (void)eta; (void)t; (void)pp; (void)hh;\n  return " << rootT
          << ";\n}\n";
      }
    }
    if (tc_root < 0) s << "#define GM_TC 0\n";
  }

  // Value + gradient: forward, then adjoints in reverse order.
  s << "__device__ __forceinline__ float gm_value_grad(const float* __restrict__ d, "
       "const float* __restrict__ p, const float* __restrict__ h, float* __restrict__ gp, "
       "float* __restrict__ gh) {\n";
  {
    std::ostringstream f;
    const int nf = out->n_fwd;
    emit_fwd(f, false);
    out->n_fwd = nf;
    s << f.str();
    // Adjoints of per-observation nodes: the first contribution assigns
    // (0 + x is not x in IEEE arithmetic, so adding to a zero would cost an
    // instruction per edge), later ones accumulate.
    std::vector<char> has_adj(N, 0);
    for (int i = 0; i < N; ++i)
      if (live[i] && is_pd(i)) s << "  float g" << i << " = 0.0f;\n";
    auto sink = [&](int c, const std::string& e) {
      if (c < 0 || !(g.n[c].dep & DEP_P)) return;
      if (g.n[c].op == O_P) s << "  gp[" << g.n[c].arg << "] += " << e << ";\n";
      else if (hslot[c] >= 0) s << "  gh[" << hslot[c] << "] += " << e << ";\n";
      else if (!has_adj[c]) {
        s << "  g" << c << " = " << e << ";\n";
        has_adj[c] = 1;
      } else {
        s << "  g" << c << " += " << e << ";\n";
      }
    };
    if (root >= 0 && (g.n[root].dep & DEP_P)) {
      if (is_pd(root)) {
        s << "  g" << root << " = 1.0f;\n";
        has_adj[root] = 1;
      } else {
        sink(root, "1.0f");
      }
    }
    for (int i = N - 1; i >= 0; --i) {
      if (!live[i] || !is_pd(i)) continue;
      const Node& x = g.n[i];
      const std::string G = "g" + std::to_string(i);
      for (auto& ce : adjoints(g, i, G, name[i], ref_obs(x.a), x.b >= 0 ? ref_obs(x.b) : "",
                               true))
        sink(ce.first, ce.second);
    }
    s << "  (void)d; (void)p; (void)h; (void)gp; (void)gh;\n  return " << rootv << ";\n}\n";
  }

  // gm_value_grad4l: values and adjoints of four consecutive observations
  // xo .. xo + 3 for the chain-lane gradient body, node by node in lockstep
  // (forward as gm_value_grad, no value rewrites).  The reverse sweep reloads
  // the data columns it needs (gm_lds4v) rather than keeping the forward's
  // loads live.  Observations k >= nv (a partial last quad) read observation
  // 0's data and enter the sweep with adjoint 0.
  s << "__device__ __forceinline__ void gm_value_grad4l(const float* __restrict__ xo, int nv, "
       "const float* __restrict__ p, const float* __restrict__ h, float* __restrict__ gp, "
       "float* __restrict__ gh, float* __restrict__ out) {\n";
  {
    std::vector<char> fl(N, 0), rl(N, 0);
    auto data4 = [&](int i, int k, bool reload) -> std::string {
      std::vector<char>& L = reload ? rl : fl;
      const std::string q = (reload ? "r_" : "q_") + name[i];
      if (!L[i]) {
        s << "  const float4 " << q << " = "
          << (reload ? "gm_lds4v(" : "*reinterpret_cast<const float4*>(") << "xo + " << col_of(i)
          << " * GM_T);\n";
        s << "  const float " << q << "_0 = " << q << ".x;\n";
        for (int j = 1; j < 4; ++j)
          s << "  const float " << q << "_" << j << " = nv > " << j << " ? " << q << "."
            << "xyzw"[j] << " : " << q << ".x;\n";
        L[i] = 1;
      }
      return q + "_" + std::to_string(k);
    };
    auto ref4g = [&](int i, int k, bool reload) -> std::string {
      const Node& x = g.n[i];
      if (x.op == O_C || x.op == O_P) return name[i];
      if (hslot[i] >= 0) return "h[" + std::to_string(hslot[i]) + "]";
      if (dslot[i] >= 0) return data4(i, k, reload);
      return name[i] + "_" + std::to_string(k);
    };
    for (int i = 0; i < N; ++i) {
      if (!live[i] || !is_pd(i)) continue;
      const Node& x = g.n[i];
      std::string a[4], b[4];
      for (int k = 0; k < 4; ++k) {
        a[k] = ref4g(x.a, k, false);
        if (x.b >= 0) b[k] = ref4g(x.b, k, false);
      }
      const std::string rb = recip(i) >= 0 ? "h[" + std::to_string(recip(i)) + "]" : "";
      for (int k = 0; k < 4; ++k)
        s << "  const float " << name[i] << "_" << k << " = "
          << (rb.empty() ? op_expr(g, i, a[k], b[k], true) : "(" + a[k] + " * " + rb + ")")
          << ";\n";
    }
    for (int i = 0; i < N; ++i)
      if (live[i] && is_pd(i))
        for (int k = 0; k < 4; ++k) s << "  float g" << i << "_" << k << " = 0.0f;\n";
    std::vector<char> has_adj(N, 0);
    auto sink4 = [&](int c, const std::string* e) {
      if (c < 0 || !(g.n[c].dep & DEP_P)) return;
      for (int k = 0; k < 4; ++k) {
        if (g.n[c].op == O_P) s << "  gp[" << g.n[c].arg << "] += " << e[k] << ";\n";
        else if (hslot[c] >= 0) s << "  gh[" << hslot[c] << "] += " << e[k] << ";\n";
        else
          s << "  g" << c << "_" << k << (has_adj[c] ? " += " : " = ") << e[k] << ";\n";
      }
      if (g.n[c].op != O_P && hslot[c] < 0) has_adj[c] = 1;
    };
    if (root >= 0 && (g.n[root].dep & DEP_P)) {
      std::string w[4];
      for (int k = 0; k < 4; ++k)
        w[k] = k == 0 ? "1.0f" : "(nv > " + std::to_string(k) + " ? 1.0f : 0.0f)";
      if (is_pd(root)) {
        for (int k = 0; k < 4; ++k) s << "  g" << root << "_" << k << " = " << w[k] << ";\n";
        has_adj[root] = 1;
      } else {
        sink4(root, w);
      }
    }
    for (int i = N - 1; i >= 0; --i) {
      if (!live[i] || !is_pd(i)) continue;
      const Node& x = g.n[i];
      std::vector<std::vector<std::pair<int, std::string>>> ce(4);
      for (int k = 0; k < 4; ++k) {
        const std::string G = "g" + std::to_string(i) + "_" + std::to_string(k);
        const std::string v = name[i] + "_" + std::to_string(k);
        ce[k] = adjoints(g, i, G, v, ref4g(x.a, k, true), x.b >= 0 ? ref4g(x.b, k, true) : "",
                         true, recip(i) >= 0 ? "h[" + std::to_string(recip(i)) + "]" : "");
      }
      for (size_t j = 0; j < ce[0].size(); ++j) {
        std::string e[4];
        for (int k = 0; k < 4; ++k) e[k] = ce[k][j].second;
        sink4(ce[0][j].first, e);
      }
    }
    for (int k = 0; k < 4; ++k)
      s << "  out[" << k << "] = " << (root < 0 ? std::string("0.0f") : ref4g(root, k, false))
        << ";\n";
  }
  s << "  (void)xo; (void)nv; (void)p; (void)h; (void)gp; (void)gh;\n}\n";

  // Chain rule through the hoisted parameter-only nodes, once per chain.
  s << "__device__ __forceinline__ void gm_hoist_grad(const float* __restrict__ p, "
       "const float* __restrict__ gh, float* __restrict__ gp) {\n";
  emit_hoist_body(s);
  for (int i = 0; i < N; ++i)
    if (live[i] && is_h(i))
      s << "  float a" << i << " = " << (hslot[i] >= 0 ? "gh[" + std::to_string(hslot[i]) + "]"
                                                       : std::string("0.0f"))
        << ";\n";
  for (int i = N - 1; i >= 0; --i) {
    if (!live[i] || !is_h(i)) continue;
    const Node& x = g.n[i];
    for (auto& ce : adjoints(g, i, "a" + std::to_string(i), name[i], name[x.a],
                             x.b >= 0 ? name[x.b] : "", true)) {
      const int c = ce.first;
      if (c < 0 || !(g.n[c].dep & DEP_P)) continue;
      if (g.n[c].op == O_P) s << "  gp[" << g.n[c].arg << "] += " << ce.second << ";\n";
      else s << "  a" << c << " += " << ce.second << ";\n";
    }
  }
  s << "  (void)p; (void)gh; (void)gp;\n}\n";

  // Prior in f64 (parameters only).
  Graph pg;
  const int proot = pg.build(prior_code, n_prior, prior_consts);
  const std::vector<char> plive = pg.reachable(proot);
  std::vector<std::string> pn(pg.n.size());
  for (size_t i = 0; i < pg.n.size(); ++i) {
    const Node& x = pg.n[i];
    if (x.op == O_C) pn[i] = dlit(x.c);
    else if (x.op == O_P) pn[i] = "p[" + std::to_string(x.arg) + "]";
    else if (x.op == O_D) {
      *err = "the prior may not read data";
      return 1;
    } else pn[i] = "w" + std::to_string(i);
  }
  auto emit_prior_fwd = [&](std::ostringstream& o) {
    for (size_t i = 0; i < pg.n.size(); ++i) {
      if (!plive[i] || pg.n[i].op <= O_D) continue;
      const Node& x = pg.n[i];
      o << "  const double " << pn[i] << " = "
        << op_expr(pg, (int)i, pn[x.a], x.b >= 0 ? pn[x.b] : "", false) << ";\n";
    }
  };
  const std::string proot_v = proot < 0 ? std::string("0.0") : pn[proot];
  s << "__device__ __forceinline__ double gm_prior(const double* __restrict__ p) {\n";
  emit_prior_fwd(s);
  s << "  (void)p;\n  return " << proot_v << ";\n}\n";
  s << "__device__ __forceinline__ double gm_prior_grad(const double* __restrict__ p, "
       "double* __restrict__ g) {\n";
  emit_prior_fwd(s);
  for (size_t i = 0; i < pg.n.size(); ++i)
    if (plive[i] && pg.n[i].op > O_D) s << "  double a" << i << " = 0.0;\n";
  if (proot >= 0 && (pg.n[proot].dep & DEP_P)) {
    if (pg.n[proot].op == O_P) s << "  g[" << pg.n[proot].arg << "] += 1.0;\n";
    else s << "  a" << proot << " = 1.0;\n";
  }
  for (int i = (int)pg.n.size() - 1; i >= 0; --i) {
    if (!plive[i] || pg.n[i].op <= O_D || !(pg.n[i].dep & DEP_P)) continue;
    const Node& x = pg.n[i];
    for (auto& ce : adjoints(pg, i, "a" + std::to_string(i), pn[i], pn[x.a],
                             x.b >= 0 ? pn[x.b] : "", false)) {
      const int c = ce.first;
      if (c < 0 || !(pg.n[c].dep & DEP_P)) continue;
      if (pg.n[c].op == O_P) s << "  g[" << pg.n[c].arg << "] += " << ce.second << ";\n";
      else s << "  a" << c << " += " << ce.second << ";\n";
    }
  }
  s << "  (void)p; (void)g;\n  return " << proot_v << ";\n}\n";

  out->source = s.str();
  out->np = (int)n_params;
  out->has_grad = true;
  return 0;
}

}  // namespace gpum
