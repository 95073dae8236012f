/*
 * Stand-in for the reference's external Logging package (an empty git
 * submodule in the reference tree).  The reference's checks spell errors as
 * LOGGING_CHECK(cond, fmt, args...) / LOGGING_THROW(fmt, args...); for the
 * oracle build both only need to throw, so the format arguments are dropped
 * and the format string becomes the exception message.
 *
 * Test infrastructure only: this header is used to compile the reference's
 * NATIVE sources into oracle/_ref, never by the B200 library.
 */
#pragma once

#include <stdexcept>

namespace oracle_shim
{
template <typename... Args> [[noreturn]] inline void fail(const char* msg, Args&&...)
{
    throw std::invalid_argument(msg);
}
[[noreturn]] inline void fail() { throw std::invalid_argument("check failed"); }
}  // namespace oracle_shim

#define LOGGING_CHECK(cond, ...)                                                                   \
    do                                                                                             \
    {                                                                                              \
        if (!(cond))                                                                               \
        {                                                                                          \
            ::oracle_shim::fail(__VA_ARGS__);                                                      \
        }                                                                                          \
    } while (0)

#define LOGGING_THROW(...) ::oracle_shim::fail(__VA_ARGS__)
