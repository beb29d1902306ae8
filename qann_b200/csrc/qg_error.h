// Status codes and the exception type every layer of the library throws and
// the C-ABI turns back into status codes.
#pragma once

#include <stdexcept>
#include <string>

namespace qg {

// Error classes mirror the exception types the reference's Python layer maps:
// std::invalid_argument -> ValueError, std::logic_error -> RuntimeError,
// std::runtime_error -> RuntimeError / IOError (reference bindings/python_bindings.cpp).
enum Status : int {
    kOk = 0,
    kInvalidArgument = 1,
    kLogicError = 2,
    kRuntimeError = 3,
    kCudaError = 4,
    kOutOfMemory = 5,
    kUnsupported = 6,
};

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void require(bool ok, const std::string& msg, int status = kInvalidArgument) {
    if (!ok) throw Error(status, msg);
}

} // namespace qg
