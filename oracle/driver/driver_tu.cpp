// The reference's own driver (app/driver_main.hpp: run_application, the time
// loop and its key=value report) compiled against the single-box AMReX shim.
// TEST INFRASTRUCTURE ONLY.
//
// Two builds of this file (oracle/Makefile, targets driver-ref and
// driver-bridge):
//   * ECG_DRIVER_BRIDGE undefined: the reference's numerics, as
//     src/euler_compare_app.cpp:41-62 includes them;
//   * ECG_DRIVER_BRIDGE defined: the same headers, then include/ecg_bridge.hpp,
//     which sends run_application's hot-path calls to libecg.so (linked).
// Arguments are the reference executable's: key=value pairs.
#include "amrex_shim.hpp"

#include <Eigen/Dense>
#include <Eigen/IterativeLinearSolvers>
#include <Eigen/Sparse>
#include <Eigen/SparseLU>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cctype>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <limits>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

enum ConservedComponent { Rho = 0, Mx = 1, My = 2, E = 3, NCons = 4 };

#include "euler_compare/core/solver_types.hpp"
#include "euler_compare/core/diagnostics.hpp"
#include "euler_compare/core/run_config.hpp"
#include "euler_compare/core/config_reader.hpp"
#include "euler_compare/problems/problem_setup_boundary.hpp"
#include "euler_compare/numerics/explicit_update.hpp"
#include "euler_compare/imex/imex_source_map_helpers.hpp"
#include "euler_compare/imex/imex_pressure_helpers.hpp"
#include "euler_compare/imex/imex_bdltv20_updates.hpp"
#include "euler_compare/io/output_cases.hpp"

}  // namespace

#ifdef ECG_DRIVER_BRIDGE
#include "ecg_bridge.hpp"
#endif

#include "euler_compare/app/driver_main.hpp"

int main(int argc, char* argv[])
{
  try {
    return euler_compare::run_application(argc, argv);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "amrex::Abort: %s\n", e.what());
    return 2;
  }
}
