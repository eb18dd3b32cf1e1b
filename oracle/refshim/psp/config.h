// ORACLE — test infrastructure only.  The configuration header the
// reference's CMake build generates (cmake/config.h.cmake of the
// reference): directories for the parallel VTK writers, no Ritz printing.
#pragma once
#define HAVE_MKDIR
