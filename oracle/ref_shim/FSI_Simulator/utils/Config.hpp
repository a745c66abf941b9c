// Stand-in for the reference's include/FSI_Simulator/utils/Config.hpp when
// its fluid-step sources are compiled into oracle/_ref.  The reference reads
// these structs from JSON through nlohmann-json (not installed here); the
// checker fills them directly.  Fields, defaults and getCf() are those of
// Config.hpp:17-22 (BoundaryCondition), :64-101 (2D) and :124-159 (3D), the
// interface the fluid step reads; the solid-solver fields are left out.
// The reference's Config.hpp also brings in common/Types.hpp (through
// fem/FemConfig.hpp), whose real / vec2_t / vec3_t aliases FsiCoupling2D.cu
// uses; they are restated here (Types.hpp:16-20, real = double).
#pragma once

#include <string>
#include <vector>

#include <glm/glm.hpp>

#include "FSI_Simulator/lbm/LbmDataTypes.cuh"

namespace fsi {

using real = double;
using vec2_t = glm::dvec2;
using vec3_t = glm::dvec3;

struct BoundaryCondition {
    std::vector<int> position;
    lbm::LbmNodeFlag flag;
};

struct SimulationParameters2D {
    int dimension = 2;
    double fluid_viscosity = 0.001;
    double fluid_density = 1000.0;
    int fluid_nx = 400;
    int fluid_ny = 400;
    double fluid_dx = 1.0;
    double total_time = 10.0;
    double dt = 0.001;
    std::vector<BoundaryCondition> boundaries;
    std::vector<float> boundary_velocities;

    // rho_f dx^2 converted to float, then * dx / dt^2 in double, to float
    float getCf() const
    {
        float cm = fluid_density * fluid_dx * fluid_dx;
        return cm * fluid_dx / (dt * dt);
    }
};

struct SimulationParameters3D {
    int dimension = 3;
    double fluid_viscosity = 0.001;
    double fluid_density = 1000.0;
    int fluid_nx = 128;
    int fluid_ny = 128;
    int fluid_nz = 128;
    double fluid_dx = 1.0;
    double total_time = 10.0;
    double dt = 0.001;
    std::vector<BoundaryCondition> boundaries;
    std::vector<float> boundary_velocities;

    // rho_f dx^3 converted to float, then * dx / dt^2 in double, to float
    float getCf() const
    {
        float cm = fluid_density * fluid_dx * fluid_dx * fluid_dx;
        return cm * fluid_dx / (dt * dt);
    }
};

} // namespace fsi
