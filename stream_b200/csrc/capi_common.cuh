// Helpers shared by the extern "C" translation units.
#pragma once

#include <exception>
#include <string>

#include "common.cuh"

#define SB_EXPORT __attribute__((visibility("default")))

namespace sb {
// Thread-local text of the last failure seen at the C boundary.
std::string& last_error_text();
}  // namespace sb

// Run f, converting any exception into a status code (0 = ok) and recording
// its message for stream_b200_last_error().
template <typename F>
inline int sb_guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::invalid_argument& e) {
        sb::last_error_text() = e.what();
        return (int)sb::ST_BAD_INPUT;
    } catch (const std::exception& e) {
        sb::last_error_text() = e.what();
        return (int)sb::ST_CUDA_ERROR;
    } catch (...) {
        sb::last_error_text() = "unknown error";
        return (int)sb::ST_CUDA_ERROR;
    }
}
