// Errors and status codes shared by the host code (hs::Error equivalent, include/hsolve/error.hpp).
#pragma once

#include <cstdint>
#include <sstream>
#include <stdexcept>
#include <string>

#include "hsg.h"

namespace hsg {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& msg) : std::runtime_error(msg), status_(status) {}
  int status() const noexcept { return status_; }

 private:
  int status_;
};

#define HSG_THROW(status, msg)                 \
  do {                                         \
    std::ostringstream hsg_os_;                \
    hsg_os_ << msg;                            \
    throw ::hsg::Error((status), hsg_os_.str()); \
  } while (0)

#define HSG_REQUIRE(cond, status, msg) \
  do {                                 \
    if (!(cond)) HSG_THROW(status, msg); \
  } while (0)

void set_last_error(const std::string& msg);

// Kernel launches issued by this library (exported as hsg_kernel_launches).
void note_launches(long long count);

// Runs f(), mapping exceptions to status codes and recording the message (C ABI wrapper).
template <class F>
int guarded(F&& f) noexcept {
  try {
    f();
    set_last_error("");
    return HSG_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status();
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return HSG_OUT_OF_MEMORY_BUDGET;
  } catch (const std::invalid_argument& e) {
    set_last_error(e.what());
    return HSG_INVALID_INPUT;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return HSG_INTERNAL;
  } catch (...) {
    set_last_error("unknown exception");
    return HSG_INTERNAL;
  }
}

}  // namespace hsg
