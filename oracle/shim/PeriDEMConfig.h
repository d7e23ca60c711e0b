// Stand-in for the configure-time header the reference's CMake generates.
// ORACLE TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cstddef>
#define PERIDEM_VERSION_MAJOR 0
#define PERIDEM_VERSION_MINOR 2
#define PERIDEM_VERSION_PATCH 1
const size_t MAJOR_VERSION = PERIDEM_VERSION_MAJOR;
const size_t MINOR_VERSION = PERIDEM_VERSION_MINOR;
const size_t UPDATE_VERSION = PERIDEM_VERSION_PATCH;
