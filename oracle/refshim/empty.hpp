// ORACLE — test infrastructure only: stands for the Elemental headers that
// psp/environment.hpp includes by macro; the reference's code needs nothing
// from them beyond clique.hpp.
#pragma once
