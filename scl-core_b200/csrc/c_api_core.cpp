// Core C ABI: version, build configuration and thread-local error state.
// Replaces scl/binding/c_api/core/core.cpp:17-120,240-326.
#include <cstring>
#include <new>
#include <stdexcept>

#include "abi.hpp"

namespace sclabi {
namespace {
constexpr size_t kMsgLen = 512;
thread_local scl_error_t t_code = SCL_OK;
thread_local char t_msg[kMsgLen] = {0};
}  // namespace

void set_last_error(scl_error_t code, const char* message) noexcept {
  t_code = code;
  if (message) {
    std::strncpy(t_msg, message, kMsgLen - 1);
    t_msg[kMsgLen - 1] = '\0';
  } else {
    t_msg[0] = '\0';
  }
}

void clear_last_error() noexcept {
  t_code = SCL_OK;
  t_msg[0] = '\0';
}

scl_error_t handle_exception() noexcept {
  try {
    throw;
  } catch (const sclgpu::Error& e) {
    set_last_error(e.code, e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error(SCL_ERROR_OUT_OF_MEMORY, "Memory allocation failed (std::bad_alloc)");
    return SCL_ERROR_OUT_OF_MEMORY;
  } catch (const std::length_error& e) {
    set_last_error(SCL_ERROR_INVALID_ARGUMENT, e.what());
    return SCL_ERROR_INVALID_ARGUMENT;
  } catch (const std::out_of_range& e) {
    set_last_error(SCL_ERROR_RANGE_ERROR, e.what());
    return SCL_ERROR_RANGE_ERROR;
  } catch (const std::logic_error& e) {
    set_last_error(SCL_ERROR_INVALID_ARGUMENT, e.what());
    return SCL_ERROR_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    set_last_error(SCL_ERROR_UNKNOWN, e.what());
    return SCL_ERROR_UNKNOWN;
  } catch (...) {
    set_last_error(SCL_ERROR_UNKNOWN, "Unknown exception (not derived from std::exception)");
    return SCL_ERROR_UNKNOWN;
  }
}
}  // namespace sclabi

extern "C" {

SCL_EXPORT const char* scl_get_version(void) { return "1.0.0"; }

SCL_EXPORT const char* scl_get_build_config(void) {
  return SCL_REAL_TYPE_NAME "+" SCL_INDEX_TYPE_NAME "+cuda-sm_100a";
}

SCL_EXPORT const char* scl_get_last_error(void) {
  return sclabi::t_msg[0] != '\0' ? sclabi::t_msg : "No error";
}

SCL_EXPORT scl_error_t scl_get_last_error_code(void) { return sclabi::t_code; }

SCL_EXPORT void scl_clear_error(void) { sclabi::clear_last_error(); }

SCL_EXPORT scl_bool_t scl_is_ok(scl_error_t code) { return code == SCL_OK ? SCL_TRUE : SCL_FALSE; }

SCL_EXPORT scl_bool_t scl_is_error(scl_error_t code) { return code != SCL_OK ? SCL_TRUE : SCL_FALSE; }

}  // extern "C"
