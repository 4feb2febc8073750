// Failure handling shared by the extern "C" entry points: every call catches its own exceptions and turns them into
// an nb_status; the message of the last failure on this host thread is kept for nereus_b200_last_error().
#pragma once

#include <new>
#include <string>

#include "nb_solver.h"

namespace nb
{
namespace capi
{
extern thread_local std::string g_error;

inline int Fail(int code, const std::string &msg)
{
    g_error = msg;
    return code;
}

// the nb_status of an exception
inline int StatusOf(std::exception_ptr ep)
{
    try
    {
        std::rethrow_exception(ep);
    }
    catch (const nb::InputError &e)
    {
        return Fail(NB_BAD_INPUT, e.what());
    }
    catch (const nb::CudaError &e)
    {
        if (e.code == cudaErrorMemoryAllocation) return Fail(NB_OUT_OF_MEMORY, e.what());
        if (e.code == cudaErrorNoDevice || e.code == cudaErrorInsufficientDriver ||
            e.code == cudaErrorNoKernelImageForDevice)
            return Fail(NB_NO_DEVICE, e.what());
        return Fail(NB_DEVICE_ERROR, e.what());
    }
    catch (const std::bad_alloc &)
    {
        return Fail(NB_OUT_OF_MEMORY, "host allocation failed");
    }
    catch (const std::exception &e)
    {
        return Fail(NB_DEVICE_ERROR, e.what());
    }
    catch (...)
    {
        return Fail(NB_DEVICE_ERROR, "unknown failure");
    }
}

template <typename F> int Guard(F &&f)
{
    try
    {
        return f();
    }
    catch (...)
    {
        return StatusOf(std::current_exception());
    }
}
} // namespace capi
} // namespace nb
