/*
 * Force-included prelude for compiling the reference sbd headers (oracle recipe).
 *
 * TEST INFRASTRUCTURE ONLY. The reference headers are not self-contained:
 * framework/type_def.h needs SIZE_MAX before <cstdint> is seen by every
 * translation unit, several headers use std::mt19937 / std::chrono /
 * std::iota / omp_get_* without including their headers, and
 * chemistry/tpb/davidson.h uses an unqualified `endl`. This prelude supplies
 * exactly those declarations so that the unmodified headers compile.
 */
#ifndef SBDX_ORACLE_REF_PRELUDE_H
#define SBDX_ORACLE_REF_PRELUDE_H
#include <cstdint>
#include <climits>
#include <cmath>
#include <cassert>
#include <chrono>
#include <random>
#include <numeric>
#include <algorithm>
#include <vector>
#include <string>
#include <iostream>
#include <omp.h>
namespace sbd { using std::endl; }
#endif
