// Definitions shared by the translation units that implement the C ABI.
#pragma once

#include <functional>

#include "mpm_field.h"
#include "mpm_krylov.h"

struct mpm_field {
    mpm::Field* impl;
    mpm::BatchSolver* solver;
};

namespace mpm {
// Runs f, mapping exceptions to a status code and the thread's last-error text.
int capi_guard(const std::function<void()>& f);
}  // namespace mpm
