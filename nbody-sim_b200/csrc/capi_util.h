// capi_util.h -- error plumbing shared by the extern "C" entry points.
#pragma once
#include <exception>
#include <new>
#include <string>

#include "../../include/nbody_b200.h"

namespace nb {

void set_error(const std::string& msg);

struct ArgError : std::exception {
  std::string msg;
  int code;
  explicit ArgError(std::string m, int c = NBODY_ERR_ARG) : msg(std::move(m)), code(c) {}
  const char* what() const noexcept override { return msg.c_str(); }
};

}  // namespace nb

// Wraps an entry point body: maps C++ exceptions onto NBODY_ERR_* codes.
#define NBODY_API_BODY(...)                                              \
  try {                                                                  \
    __VA_ARGS__;                                                         \
    return NBODY_OK;                                                     \
  } catch (const nb::ArgError& e) {                                      \
    nb::set_error(e.msg);                                                \
    return e.code;                                                       \
  } catch (const nb::CudaError& e) {                                     \
    nb::set_error(e.what());                                             \
    return NBODY_ERR_CUDA;                                               \
  } catch (const std::bad_alloc&) {                                      \
    nb::set_error("host allocation failed");                             \
    return NBODY_ERR_ARG;                                                \
  } catch (const std::exception& e) {                                    \
    nb::set_error(e.what());                                             \
    return NBODY_ERR_ARG;                                                \
  }

#define NBODY_REQUIRE(cond, msg) \
  do {                           \
    if (!(cond)) throw nb::ArgError(msg); \
  } while (0)
