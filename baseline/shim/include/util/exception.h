/*
 * Stand-in for the reference's external Logging package (an empty git
 * submodule in the reference tree), for compiling the reference's CUDA_BLAS
 * sources into the GPU baseline: LOGGING_CHECK(cond, fmt, args...) and
 * LOGGING_THROW(fmt, args...) throw std::runtime_error with the format string
 * as the message (the arguments are dropped).
 */
#pragma once

#include <stdexcept>

namespace baseline_shim
{
template <typename... Args> [[noreturn]] inline void raise(const char* msg, Args&&...)
{
    throw std::runtime_error(msg);
}
[[noreturn]] inline void raise() { throw std::runtime_error("check failed"); }
}  // namespace baseline_shim

#define LOGGING_CHECK(cond, ...)                                                                   \
    do                                                                                             \
    {                                                                                              \
        if (!(cond))                                                                               \
        {                                                                                          \
            ::baseline_shim::raise(__VA_ARGS__);                                                   \
        }                                                                                          \
    } while (0)

#define LOGGING_THROW(...) ::baseline_shim::raise(__VA_ARGS__)
