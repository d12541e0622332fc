// Error model of the cusignal_cpp API (ZKX/cusignal_cpp/include/cusignal/runtime/errors.h:18-41,
// 83-96): the numeric ErrorCode values are part of the public contract, so they are kept;
// ProjectError carries one of them.  Shape and parameter errors are thrown as
// std::invalid_argument, as the reference's operators do.
#pragma once

#include <stdexcept>
#include <string>

namespace cusignal {

enum class ErrorCode : int {
    SUCCESS = 0,
    INVALID_ARGUMENT = 1001,
    INVALID_SHAPE = 1002,
    INVALID_DTYPE = 1003,
    UNSUPPORTED_OPERATION = 1004,
    CONFIG_ERROR = 1005,
    CUDA_DRIVER_ERROR = 2001,
    CUDA_RUNTIME_ERROR = 2002,
    OUT_OF_MEMORY = 2003,
    BACKEND_ERROR = 2099,
    EXECUTION_FAILED = 2100,
    SYNC_FAILED = 2101,
    ACCURACY_FAILED = 3001,
    RESOURCE_FAILED = 3002,
    IO_ERROR = 4001,
    INTERNAL_ERROR = 9001,
    UPSTREAM_STEP_FAILED = 9002,
    OK = SUCCESS,
    INVALID_CONFIG = CONFIG_ERROR,
    UNSUPPORTED = UNSUPPORTED_OPERATION,
    ALLOCATION_FAILED = OUT_OF_MEMORY,
};

class ProjectError : public std::runtime_error {
public:
    ProjectError(ErrorCode code, const std::string& message)
        : std::runtime_error(message), code_(code) {}
    ErrorCode code() const noexcept { return code_; }

private:
    ErrorCode code_;
};

}  // namespace cusignal
