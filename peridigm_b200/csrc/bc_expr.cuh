// Prescribed-value functions of x, y, z and t: the bodies the reference
// compiles with its run-time compiler for a boundary condition's "Value"
// string (src/core/Peridigm_BoundaryCondition.cpp:68-84 declares the
// variables x, y, z, t and value; :157-160 and :217-220 prepend "value = "
// when the string does not mention value). Here the body is compiled on the
// host to a short stack program (ExprOp words: opcode in the low 8 bits,
// operand above) over a table of FP64 constants, and run by expr_run on the
// device for every prescribed degree of freedom, or on the host by
// pd_expr_eval.
#pragma once

#include <math.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace pdb {

enum ExprOp : int32_t {
  XO_END = 0,
  XO_CONST,  // push constant [operand]
  XO_LOAD,   // push variable [operand]
  XO_STORE,  // pop into variable [operand]
  XO_ADD,
  XO_SUB,
  XO_MUL,
  XO_DIV,
  XO_POW,
  XO_MOD,
  XO_NEG,
  XO_NOT,
  XO_LT,
  XO_LE,
  XO_GT,
  XO_GE,
  XO_EQ,
  XO_NE,
  XO_AND,
  XO_OR,
  XO_F1,   // one-argument function [operand]
  XO_F2,   // two-argument function [operand]
  XO_JZ,   // pop; jump to [operand] when zero
  XO_JMP,  // jump to [operand]
};
enum ExprF1 : int32_t {
  XF_SIN = 0, XF_COS, XF_TAN, XF_ASIN, XF_ACOS, XF_ATAN, XF_SINH, XF_COSH, XF_TANH,
  XF_EXP, XF_LOG, XF_LOG10, XF_SQRT, XF_ABS, XF_FLOOR, XF_CEIL,
};
enum ExprF2 : int32_t { XF_POW2 = 0, XF_ATAN2, XF_FMOD, XF_MIN, XF_MAX };

// Variables 0-4 are x, y, z, t, value; 5.. the body's own.
constexpr int kExprVars = 16;
constexpr int kExprStack = 32;
constexpr int kExprVarValue = 4;

__host__ __device__ inline double expr_f1(int f, double a) {
  switch (f) {
    case XF_SIN: return sin(a);
    case XF_COS: return cos(a);
    case XF_TAN: return tan(a);
    case XF_ASIN: return asin(a);
    case XF_ACOS: return acos(a);
    case XF_ATAN: return atan(a);
    case XF_SINH: return sinh(a);
    case XF_COSH: return cosh(a);
    case XF_TANH: return tanh(a);
    case XF_EXP: return exp(a);
    case XF_LOG: return log(a);
    case XF_LOG10: return log10(a);
    case XF_SQRT: return sqrt(a);
    case XF_ABS: return fabs(a);
    case XF_FLOOR: return floor(a);
    default: return ceil(a);
  }
}
__host__ __device__ inline double expr_f2(int f, double a, double b) {
  switch (f) {
    case XF_POW2: return pow(a, b);
    case XF_ATAN2: return atan2(a, b);
    case XF_FMOD: return fmod(a, b);
    case XF_MIN: return fmin(a, b);
    default: return fmax(a, b);
  }
}

// Runs the program at code[0..] (jump targets relative to code) and returns
// value. The compiler checks the stack depth, variable and constant indices
// and jump targets of every program, and bodies have no loops, so a program
// runs at most its own length in operations; max_ops bounds it regardless
// (*ok = false when reached).
__host__ __device__ inline double expr_run(const int32_t* code, const double* konst, double x, double y, double z,
                                           double t, int max_ops, bool* ok) {
  double s[kExprStack];
  double v[kExprVars];
  v[0] = x, v[1] = y, v[2] = z, v[3] = t;
  for (int k = 4; k < kExprVars; ++k) v[k] = 0.0;
  int sp = 0, pc = 0;
  for (int n = 0; n < max_ops; ++n) {
    const int32_t w = code[pc++];
    const int op = w & 0xff, arg = w >> 8;
    switch (op) {
      case XO_END: *ok = true; return v[kExprVarValue];
      case XO_CONST: s[sp++] = konst[arg]; break;
      case XO_LOAD: s[sp++] = v[arg]; break;
      case XO_STORE: v[arg] = s[--sp]; break;
      case XO_NEG: s[sp - 1] = -s[sp - 1]; break;
      case XO_NOT: s[sp - 1] = s[sp - 1] == 0.0 ? 1.0 : 0.0; break;
      case XO_F1: s[sp - 1] = expr_f1(arg, s[sp - 1]); break;
      case XO_F2: --sp; s[sp - 1] = expr_f2(arg, s[sp - 1], s[sp]); break;
      case XO_JZ: if (s[--sp] == 0.0) pc = arg; break;
      case XO_JMP: pc = arg; break;
      default: {
        const double b = s[--sp], a = s[sp - 1];
        double r;
        switch (op) {
          case XO_ADD: r = a + b; break;
          case XO_SUB: r = a - b; break;
          case XO_MUL: r = a * b; break;
          case XO_DIV: r = a / b; break;
          case XO_POW: r = pow(a, b); break;
          case XO_MOD: r = fmod(a, b); break;
          case XO_LT: r = a < b ? 1.0 : 0.0; break;
          case XO_LE: r = a <= b ? 1.0 : 0.0; break;
          case XO_GT: r = a > b ? 1.0 : 0.0; break;
          case XO_GE: r = a >= b ? 1.0 : 0.0; break;
          case XO_EQ: r = a == b ? 1.0 : 0.0; break;
          case XO_NE: r = a != b ? 1.0 : 0.0; break;
          case XO_AND: r = (a != 0.0 && b != 0.0) ? 1.0 : 0.0; break;
          default: r = (a != 0.0 || b != 0.0) ? 1.0 : 0.0; break;  // XO_OR
        }
        s[sp - 1] = r;
      }
    }
  }
  *ok = false;
  return NAN;
}

// Compiles a body (with "value = " prepended when it does not contain
// "value") into code/konst (appended; jump targets relative to the program's
// first word, which is returned in *start). Returns false with a message on
// a syntax error, an unknown name, or a body deeper than kExprStack or with
// more than kExprVars variables.
bool expr_compile(const std::string& body, std::vector<int32_t>& code, std::vector<double>& konst, int64_t* start,
                  std::string* err);

}  // namespace pdb
