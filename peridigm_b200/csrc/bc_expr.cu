// Prescribed-displacement functions: the compiler of the boundary-condition
// bodies (bc_expr.cuh), the per-step kernel that evaluates them at a step's
// current and previous times, and pd_expr_eval.
//
// Language (the subset of C the reference's input decks use for "Value"):
//   body      := statement*
//   statement := 'if' '(' expr ')' statement ['else' statement]
//              | '{' statement* '}'
//              | ['double'|'float'|'int'] name '=' expr [';']
//              | ';'
//   expr      := or;  or := and ('||' and)*;  and := cmp ('&&' cmp)*
//   cmp       := sum (('<'|'<='|'>'|'>='|'=='|'!=') sum)*
//   sum       := prod (('+'|'-') prod)*;  prod := unary (('*'|'/'|'%') unary)*
//   unary     := ('-'|'+'|'!') unary | power;  power := primary ['^' unary]
//   primary   := number | name | function '(' expr [',' expr] ')' | '(' expr ')'
// '^' is exponentiation (right associative, above unary minus: -2^2 = -4);
// comparisons and logical operators give 1 or 0.
#include <cuda_runtime.h>

#include <cctype>
#include <cstdlib>
#include <cstring>

#include "bc_expr.cuh"
#include "pd_internal.cuh"

namespace pdb {

namespace {

struct Tok {
  enum Kind { END, NUM, NAME, OP } kind = END;
  std::string s;
  double num = 0.0;
  size_t pos = 0;
};

struct Compiler {
  std::string src;
  size_t p = 0;
  Tok tok;
  std::vector<int32_t>* code;
  std::vector<double>* konst;
  int64_t base = 0;
  std::vector<std::string> vars{"x", "y", "z", "t", "value"};
  int depth = 0, max_depth = 0;
  std::string err;

  bool fail(const std::string& m) {
    if (err.empty()) err = m + " at offset " + std::to_string(tok.pos);
    return false;
  }
  void next() {
    while (p < src.size() && std::isspace((unsigned char)src[p])) ++p;
    tok = Tok();
    tok.pos = p;
    if (p >= src.size()) return;
    const char ch = src[p];
    if (std::isdigit((unsigned char)ch) || (ch == '.' && p + 1 < src.size() && std::isdigit((unsigned char)src[p + 1]))) {
      char* end = nullptr;
      tok.num = std::strtod(src.c_str() + p, &end);
      tok.kind = Tok::NUM;
      p = (size_t)(end - src.c_str());
      return;
    }
    if (std::isalpha((unsigned char)ch) || ch == '_') {
      size_t q = p;
      while (q < src.size() && (std::isalnum((unsigned char)src[q]) || src[q] == '_')) ++q;
      tok.kind = Tok::NAME;
      tok.s = src.substr(p, q - p);
      p = q;
      return;
    }
    static const char* two[] = {"<=", ">=", "==", "!=", "&&", "||"};
    for (const char* t : two)
      if (src.compare(p, 2, t) == 0) {
        tok.kind = Tok::OP;
        tok.s = t;
        p += 2;
        return;
      }
    tok.kind = Tok::OP;
    tok.s = std::string(1, ch);
    ++p;
  }
  bool is(const char* op) const { return tok.kind == Tok::OP && tok.s == op; }
  bool is_name(const char* s) const { return tok.kind == Tok::NAME && tok.s == s; }
  bool expect(const char* op) {
    if (!is(op)) return fail(std::string("expected '") + op + "'");
    next();
    return true;
  }
  void emit(int32_t op, int32_t arg, int dd) {
    code->push_back(op | (arg << 8));
    depth += dd;
    if (depth > max_depth) max_depth = depth;
  }
  int64_t here() const { return (int64_t)code->size() - base; }
  void patch(int64_t at, int64_t target) {
    int32_t& w = (*code)[(size_t)(base + at)];
    w = (w & 0xff) | (int32_t)(target << 8);
  }
  static int f1_id(const std::string& s) {
    static const char* names[] = {"sin", "cos", "tan", "asin", "acos", "atan", "sinh", "cosh",
                                  "tanh", "exp", "log", "log10", "sqrt", "abs", "floor", "ceil"};
    for (int k = 0; k < 16; ++k)
      if (s == names[k]) return k;
    if (s == "fabs") return XF_ABS;
    return -1;
  }
  static int f2_id(const std::string& s) {
    static const char* names[] = {"pow", "atan2", "fmod", "min", "max"};
    for (int k = 0; k < 5; ++k)
      if (s == names[k]) return k;
    return -1;
  }
  int var_id(const std::string& s, bool create) {
    for (size_t k = 0; k < vars.size(); ++k)
      if (vars[k] == s) return (int)k;
    if (!create) return -1;
    if ((int)vars.size() >= kExprVars) return -2;
    vars.push_back(s);
    return (int)vars.size() - 1;
  }

  bool primary() {
    if (tok.kind == Tok::NUM) {
      konst->push_back(tok.num);
      emit(XO_CONST, (int32_t)(konst->size() - 1), +1);
      next();
      return true;
    }
    if (is("(")) {
      next();
      if (!expr()) return false;
      return expect(")");
    }
    if (tok.kind == Tok::NAME) {
      const std::string name = tok.s;
      next();
      if (is("(")) {
        next();
        const int f1 = f1_id(name), f2 = f2_id(name);
        if (f1 < 0 && f2 < 0) return fail("unknown function '" + name + "'");
        if (!expr()) return false;
        if (f2 >= 0) {
          if (!expect(",")) return false;
          if (!expr()) return false;
          emit(XO_F2, f2, -1);
        } else {
          emit(XO_F1, f1, 0);
        }
        return expect(")");
      }
      const int v = var_id(name, false);
      if (v < 0) return fail("unknown variable '" + name + "'");
      emit(XO_LOAD, v, +1);
      return true;
    }
    return fail(tok.kind == Tok::END ? "unexpected end" : "unexpected '" + tok.s + "'");
  }
  bool power() {
    if (!primary()) return false;
    if (is("^")) {
      next();
      if (!unary()) return false;
      emit(XO_POW, 0, -1);
    }
    return true;
  }
  bool unary() {
    if (is("-") || is("+") || is("!")) {
      const std::string op = tok.s;
      next();
      if (!unary()) return false;
      if (op == "-") emit(XO_NEG, 0, 0);
      if (op == "!") emit(XO_NOT, 0, 0);
      return true;
    }
    return power();
  }
  bool binary_level(int level) {
    // 0: ||, 1: &&, 2: comparisons, 3: + -, 4: * / %
    static const char* ops[5][6] = {{"||"}, {"&&"}, {"<", "<=", ">", ">=", "==", "!="}, {"+", "-"}, {"*", "/", "%"}};
    static const int32_t codes[5][6] = {{XO_OR}, {XO_AND}, {XO_LT, XO_LE, XO_GT, XO_GE, XO_EQ, XO_NE},
                                        {XO_ADD, XO_SUB}, {XO_MUL, XO_DIV, XO_MOD}};
    auto sub = [&]() { return level == 4 ? unary() : binary_level(level + 1); };
    if (!sub()) return false;
    for (;;) {
      int hit = -1;
      for (int k = 0; k < 6 && ops[level][k]; ++k)
        if (is(ops[level][k])) hit = k;
      if (hit < 0) return true;
      next();
      if (!sub()) return false;
      emit(codes[level][hit], 0, -1);
    }
  }
  bool expr() { return binary_level(0); }

  bool statement() {
    if (is(";")) {
      next();
      return true;
    }
    if (is("{")) {
      next();
      while (!is("}")) {
        if (tok.kind == Tok::END) return fail("expected '}'");
        if (!statement()) return false;
      }
      next();
      return true;
    }
    if (is_name("if")) {
      next();
      if (!expect("(")) return false;
      if (!expr()) return false;
      if (!expect(")")) return false;
      const int64_t jz = here();
      emit(XO_JZ, 0, -1);
      if (!statement()) return false;
      if (is_name("else")) {
        next();
        const int64_t jmp = here();
        emit(XO_JMP, 0, 0);
        patch(jz, here());
        if (!statement()) return false;
        patch(jmp, here());
      } else {
        patch(jz, here());
      }
      return true;
    }
    if (is_name("double") || is_name("float") || is_name("int")) next();
    if (tok.kind != Tok::NAME) return fail("expected a statement");
    const std::string name = tok.s;
    if (name == "if" || name == "else" || f1_id(name) >= 0 || f2_id(name) >= 0)
      return fail("'" + name + "' cannot be assigned");
    next();
    if (!expect("=")) return false;
    if (!expr()) return false;
    const int v = var_id(name, true);
    if (v == -2) return fail("more than " + std::to_string(kExprVars) + " variables");
    emit(XO_STORE, v, -1);
    if (is(";")) next();
    return true;
  }
};

}  // namespace

bool expr_compile(const std::string& body_in, std::vector<int32_t>& code, std::vector<double>& konst, int64_t* start,
                  std::string* err) {
  const size_t code0 = code.size(), konst0 = konst.size();
  Compiler cp;
  cp.src = body_in.find("value") == std::string::npos ? "value = " + body_in : body_in;
  cp.code = &code;
  cp.konst = &konst;
  cp.base = (int64_t)code.size();
  cp.next();
  bool ok = true;
  while (ok && cp.tok.kind != Tok::END) ok = cp.statement();
  if (ok && cp.max_depth > kExprStack) ok = cp.fail("expression nested too deeply");
  if (ok) {
    cp.emit(XO_END, 0, 0);
    if (((int64_t)code.size() >> 23) != 0 || ((int64_t)konst.size() >> 23) != 0) ok = cp.fail("too many functions");
  }
  if (!ok) {
    code.resize(code0);
    konst.resize(konst0);
    if (err) *err = "boundary-condition function: " + cp.err;
    return false;
  }
  *start = cp.base;
  return true;
}

// One evaluation's prescribed values of the function dofs: cp[k] = (u_k(t_c),
// u_k(t_p)) at the times the Verlet epilogue of evaluation `step` uses.
// step >= 0: the times of the Verlet epilogue of evaluation `step`; step < 0:
// the given times t0 (current) and dt (previous), a quasi-static load step's.
__global__ void k_bc_expr(int64_t nd, const int32_t* __restrict__ dofs, const int32_t* __restrict__ start,
                          const int32_t* __restrict__ code, const double* __restrict__ konst,
                          const double4* __restrict__ xv, int64_t step, double t0, double dt, double2* __restrict__ cp,
                          int max_ops, int* __restrict__ status) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nd) return;
  const int64_t k = dofs[q];
  const double4 x = xv[k / 3];
  const double tc = step < 0 ? t0 : __dadd_rn(t0, __dmul_rn((double)(step + 1), dt));
  const double tp = step < 0 ? dt : (step == 0 ? t0 : __dadd_rn(t0, __dmul_rn((double)step, dt)));
  bool ok1 = false, ok2 = false;
  const int32_t* prog = code + start[q];
  const double cur = expr_run(prog, konst, x.x, x.y, x.z, tc, max_ops, &ok1);
  const double prev = expr_run(prog, konst, x.x, x.y, x.z, tp, max_ops, &ok2);
  if (!ok1 || !ok2) atomicOr(status, ST_NONFINITE_BC);
  cp[k] = make_double2(cur, prev);
}

cudaError_t launch_bc_expr_at(pd_ctx* c, double t_cur, double t_prev) {
  return launch_bc_expr(c, -1, t_cur, t_prev);
}

cudaError_t launch_bc_expr(pd_ctx* c, int64_t step, double t0, double dt) {
  if (c->n_bc_expr == 0) return cudaSuccess;
  const int64_t nd = c->n_bc_expr;
  k_bc_expr<<<(unsigned)((nd + 127) / 128), 128, 0, c->stream>>>(nd, c->bc_dofs.p, c->bc_start.p, c->bc_code.p,
                                                                  c->bc_konst.p, c->xv.p, step, t0, dt, c->bc_cp.p,
                                                                  (int)c->h_bc_code.size() + 1, c->status.p);
  return cudaGetLastError();
}

}  // namespace pdb

extern "C" int pd_expr_eval(const char* function, double x, double y, double z, double t, double* value) {
  if (!function || !value) return PD_ERR_ARG;
  std::vector<int32_t> code;
  std::vector<double> konst;
  int64_t start = 0;
  if (!pdb::expr_compile(function, code, konst, &start, nullptr)) return PD_ERR_ARG;
  bool ok = false;
  *value = pdb::expr_run(code.data() + start, konst.data(), x, y, z, t, (int)code.size() + 1, &ok);
  return ok ? PD_OK : PD_ERR_ARG;
}
