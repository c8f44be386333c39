// Thread-local error state and the exception -> error-code plumbing shared by
// every C ABI translation unit (same conventions as scl-core's
// scl/binding/c_api/core/internal.hpp:307-343: failures set a per-thread
// message, success clears it, exceptions never cross the ABI).
#pragma once

#include "engine.hpp"
#include "scl_core.h"

namespace sclabi {
void set_last_error(scl_error_t code, const char* message) noexcept;
void clear_last_error() noexcept;
// Maps the active exception to an error code and records its message.
scl_error_t handle_exception() noexcept;
}  // namespace sclabi

#define SCL_API_CHECK_NULL(ptr, msg)                                    \
  do {                                                                  \
    if ((ptr) == nullptr) {                                             \
      ::sclabi::set_last_error(SCL_ERROR_NULL_POINTER, (msg));          \
      return SCL_ERROR_NULL_POINTER;                                    \
    }                                                                   \
  } while (0)

#define SCL_API_CHECK(cond, code, msg)                                  \
  do {                                                                  \
    if (!(cond)) {                                                      \
      ::sclabi::set_last_error((code), (msg));                          \
      return (code);                                                    \
    }                                                                   \
  } while (0)

#define SCL_API_TRY try {
#define SCL_API_CATCH \
  }                   \
  catch (...) { return ::sclabi::handle_exception(); }

#define SCL_API_RETURN_OK          \
  do {                             \
    ::sclabi::clear_last_error();  \
    return SCL_OK;                 \
  } while (0)
