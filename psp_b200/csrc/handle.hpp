// Opaque handle behind the C ABI (include/psp_b200.h).
#pragma once
#include "host_io.hpp"
#include "solver.hpp"

struct psp_cu_handle {
    psp_b200::Helmholtz* solver;
    psp_b200::HostIo io;  // host-buffer entry points: pinned staging and device scratch
};
