// Opaque handle behind the C ABI (include/psp_b200.h).
#pragma once
#include "solver.hpp"

struct psp_cu_handle {
    psp_b200::Helmholtz* solver;
};
