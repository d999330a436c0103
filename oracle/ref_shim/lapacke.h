// lapacke.h stand-in -- TEST INFRASTRUCTURE ONLY.  src/pes/include/pes.hpp
// includes it, but src/pes/pes.cpp calls no LAPACK routine.
#pragma once
