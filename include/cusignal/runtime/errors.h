// Error model of the cusignal_cpp API (ZKX/cusignal_cpp/include/cusignal/runtime/errors.h:18-41,
// 44-123): the numeric ErrorCode values and their names are part of the public contract,
// so they are kept; ProjectError carries an Error (code, message, backend report).  Shape and parameter errors are thrown as
// std::invalid_argument, as the reference's operators do.
#pragma once

#include <stdexcept>
#include <string>
#include <utility>

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

inline const char* error_code_name(ErrorCode code)
{
    switch (code) {
    case ErrorCode::SUCCESS: return "SUCCESS";
    case ErrorCode::INVALID_ARGUMENT: return "INVALID_ARGUMENT";
    case ErrorCode::INVALID_SHAPE: return "INVALID_SHAPE";
    case ErrorCode::INVALID_DTYPE: return "INVALID_DTYPE";
    case ErrorCode::UNSUPPORTED_OPERATION: return "UNSUPPORTED_OPERATION";
    case ErrorCode::CONFIG_ERROR: return "CONFIG_ERROR";
    case ErrorCode::CUDA_DRIVER_ERROR: return "CUDA_DRIVER_ERROR";
    case ErrorCode::CUDA_RUNTIME_ERROR: return "CUDA_RUNTIME_ERROR";
    case ErrorCode::OUT_OF_MEMORY: return "OUT_OF_MEMORY";
    case ErrorCode::BACKEND_ERROR: return "BACKEND_ERROR";
    case ErrorCode::EXECUTION_FAILED: return "EXECUTION_FAILED";
    case ErrorCode::SYNC_FAILED: return "SYNC_FAILED";
    case ErrorCode::ACCURACY_FAILED: return "ACCURACY_FAILED";
    case ErrorCode::RESOURCE_FAILED: return "RESOURCE_FAILED";
    case ErrorCode::IO_ERROR: return "IO_ERROR";
    case ErrorCode::INTERNAL_ERROR: return "INTERNAL_ERROR";
    case ErrorCode::UPSTREAM_STEP_FAILED: return "UPSTREAM_STEP_FAILED";
    }
    return "INTERNAL_ERROR";
}

inline int error_code_value(ErrorCode code) noexcept { return static_cast<int>(code); }

// What a failing backend call reported ("NA" when the error did not come from one).
struct BackendError {
    std::string code{"NA"};
    std::string name{"NA"};
    std::string message{"NA"};
};

// A project error: its code, a message, the backend's own report and whether the
// failure left the process in a state that can continue (safe_exit).
struct Error {
    ErrorCode code{ErrorCode::SUCCESS};
    std::string message;
    BackendError backend;
    bool safe_exit{true};
};

class ProjectError : public std::runtime_error {
public:
    explicit ProjectError(Error error) : std::runtime_error(error.message), error_(std::move(error)) {}
    ProjectError(ErrorCode code, const std::string& message) : ProjectError(Error{code, message, {}, true}) {}
    const Error& detail() const noexcept { return error_; }
    ErrorCode code() const noexcept { return error_.code; }

private:
    Error error_;
};

[[noreturn]] inline void throw_error(ErrorCode code, std::string message, BackendError backend = {},
                                     bool safe_exit = true)
{
    if (message.empty()) message = std::string("operation failed: ") + error_code_name(code);
    throw ProjectError(Error{code, std::move(message), std::move(backend), safe_exit});
}

// The inverse of error_code_name; an unknown name is a configuration error.
inline ErrorCode parse_error_code(const std::string& name)
{
    static const ErrorCode all[] = {
        ErrorCode::SUCCESS, ErrorCode::INVALID_ARGUMENT, ErrorCode::INVALID_SHAPE, ErrorCode::INVALID_DTYPE,
        ErrorCode::UNSUPPORTED_OPERATION, ErrorCode::CONFIG_ERROR, ErrorCode::CUDA_DRIVER_ERROR,
        ErrorCode::CUDA_RUNTIME_ERROR, ErrorCode::OUT_OF_MEMORY, ErrorCode::BACKEND_ERROR,
        ErrorCode::EXECUTION_FAILED, ErrorCode::SYNC_FAILED, ErrorCode::ACCURACY_FAILED,
        ErrorCode::RESOURCE_FAILED, ErrorCode::IO_ERROR, ErrorCode::INTERNAL_ERROR,
        ErrorCode::UPSTREAM_STEP_FAILED};
    for (ErrorCode c : all)
        if (name == error_code_name(c)) return c;
    throw_error(ErrorCode::CONFIG_ERROR, "unknown error code name: " + name);
}

}  // namespace cusignal
