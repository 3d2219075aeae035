// abi_guard.h -- no C++ exception crosses the C ABI.
//
// Every exported entry point runs its body through NEO_ABI_GUARD: a failed
// host allocation (std::bad_alloc, e.g. copying a large CCS or witness)
// becomes NEO_ERR_OOM and any other exception (a thread that could not be
// started, a library error) NEO_ERR_INVARIANT, instead of unwinding into the
// caller's C, Rust or Python frames (which would terminate the process).
#pragma once
#include <exception>
#include <new>
#include "../../include/neo_gpu.h"

#define NEO_ABI_GUARD(call)             \
    try {                               \
        return (call);                  \
    } catch (const std::bad_alloc&) {   \
        return NEO_ERR_OOM;             \
    } catch (...) {                     \
        return NEO_ERR_INVARIANT;       \
    }
