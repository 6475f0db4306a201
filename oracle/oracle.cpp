// CPU oracle shared library (liboracle.so): the restated reference arithmetic.
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg as the checker, never by the product library.
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "oracle_system.hpp"

#define ORC_API(name) orc_##name
#include "oracle_capi.inc"
