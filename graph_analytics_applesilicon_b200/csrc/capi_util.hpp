// capi_util.hpp -- exception-to-status guard shared by the C ABI files.
#pragma once

#include <exception>
#include <string>

#include "common.cuh"
#include "graph_host.hpp"

namespace gb {
extern thread_local std::string g_lastError;
int guardStatus(const std::exception_ptr& ep);
void toC(HostCsr&& g, gb_csr* out);
HostCsr fromC(const gb_csr* g);
// Releases an array of gb_csr_load_pinned (page-locked); false for any other pointer.
bool freePinnedArray(void* p);

template <class F>
int guard(F&& f) {
    try {
        f();
        return GB_OK;
    } catch (...) {
        return guardStatus(std::current_exception());
    }
}
}  // namespace gb
