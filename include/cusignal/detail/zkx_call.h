// Maps a libzkx_rd status to the cusignal_cpp exception contract: shape/parameter
// errors become std::invalid_argument, everything else a ProjectError with the same
// ErrorCode number.
#pragma once

#include <zkx_rd.h>

#include <cusignal/runtime/errors.h>

#include <stdexcept>
#include <string>

namespace cusignal::detail {

inline void zkx_check(int status)
{
    if (status == ZKX_SUCCESS) return;
    const std::string msg = zkx_last_error();
    if (status == ZKX_INVALID_ARGUMENT || status == ZKX_INVALID_SHAPE) throw std::invalid_argument(msg);
    throw ProjectError(static_cast<ErrorCode>(status), msg);
}

}  // namespace cusignal::detail
