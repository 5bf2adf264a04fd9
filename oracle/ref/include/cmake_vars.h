// ORACLE — TEST INFRASTRUCTURE ONLY: the header CMake would configure from
// the reference's cmake_vars.h.in (project version 2.0).
#define FREECFD_VERSION_MAJOR 2
#define FREECFD_VERSION_MINOR 0
