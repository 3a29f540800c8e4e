// Stand-in for Teuchos_Assert.hpp: the assertion macros throw std::logic_error
// (the reference's behaviour) or abort, so reference error paths stay visible.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <stdexcept>
// The reference writes some uses without a trailing semicolon, so each macro
// expands to a plain block.
#define TEUCHOS_TEST_FOR_EXCEPT_MSG(cond, msg)                           \
  { if (cond) { std::ostringstream os_; os_ << msg;                       \
                throw std::logic_error(os_.str()); } }
#define TEUCHOS_TEST_FOR_EXCEPTION(cond, ex, msg)                        \
  { if (cond) { std::ostringstream os_; os_ << msg;                       \
                throw ex(os_.str()); } }
#define TEUCHOS_TEST_FOR_TERMINATION(cond, msg)                          \
  { if (cond) { std::fprintf(stderr, "%s\n", std::string(msg).c_str());   \
                std::abort(); } }
