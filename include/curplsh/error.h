// error.h -- status-code to exception bridge for the C++ drop-in headers.
// The reference aborts or exits on errors (include/internal/assertions.h:7-14);
// these wrappers throw std::runtime_error carrying curplsh_last_error().
#pragma once
#include <stdexcept>
#include <string>

#include "../curplsh_b200.h"

namespace curplsh {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc) {
  if (rc != CURPLSH_OK) throw Error(rc, std::string("curplsh: ") + curplsh_last_error());
}

}  // namespace curplsh
