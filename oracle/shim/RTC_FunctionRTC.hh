// Stand-in for Trilinos' run-time expression compiler. The oracle uses the
// built-in influence functions only; every user-expression call fails, which
// makes the reference raise its own "invalid influence function" error.
#pragma once
#include <string>
namespace PG_RuntimeCompiler {
class Function {
 public:
  Function(int, const std::string& = "") {}
  bool addVar(const std::string&, const std::string&) { return true; }
  bool addBody(const std::string&) { return false; }
  bool varValueFill(int, double) { return false; }
  bool execute() { return false; }
  double getValueOfVar(const std::string&) { return 0.0; }
  std::string getErrors() { return "run-time expressions are not available in the oracle build"; }
};
}  // namespace PG_RuntimeCompiler
