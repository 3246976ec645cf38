// ref_access_prelude.hpp — forced include (g++ -include) for every reference
// build.  TEST INFRASTRUCTURE ONLY.  It includes the standard headers the
// reference uses first, with access control intact, and only then turns
// `private` into `public`, so the harness can read Simulation's grid and clock
// (simulation.hpp:149-224) without touching the reference's sources.
#include <assert.h>
#include <omp.h>
#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include <Eigen/Core>
#include <Eigen/Dense>

#ifdef MATTER_REF_CUBIC
#include "ref_cubic_prelude.hpp"
#endif

#define private public
