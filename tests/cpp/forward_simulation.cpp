// The forward example's main program (examples/smoke/forward/main.cpp) over
// include/xayah/forward_simulation.hpp: runs the 128 x 192 x 128 double-jet
// scene and prints the metrics every `every` steps as one JSON line each.
//   forward_simulation [steps=960] [every=60] [pcg]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>

#include "xayah/forward_simulation.hpp"

int main(int argc, char** argv) {
    namespace ex = xayah::smoke::examples::forward;
    try {
        const long steps = argc > 1 ? std::atol(argv[1]) : 960;
        const long every = argc > 2 ? std::atol(argv[2]) : 60;
        ex::ForwardSimulationOptions options{};
        if (argc > 3 && std::strcmp(argv[3], "pcg") == 0) options.pressure_solver = xayah::smoke::PressureSolver::jacobi_pcg;
        ex::ForwardSimulation simulation{options};
        for (long step = 0; step < steps; ++step) {
            simulation.step();
            const ex::ForwardSimulationMetrics& m = simulation.metrics;
            if (m.step % every != 0) continue;
            std::printf("{\"step\": %llu, \"physical_time\": %.17g, \"density_mass\": %.17g, \"density_maximum\": %.17g, "
                        "\"temperature_maximum\": %.17g, \"maximum_velocity\": %.17g, \"cfl\": %.17g, "
                        "\"pre_projection_divergence_rms\": %.17g, \"post_projection_divergence_rms\": %.17g, \"divergence_ratio\": %.17g, "
                        "\"step_milliseconds\": %.6f, \"average_step_milliseconds\": %.6f}\n",
                        static_cast<unsigned long long>(m.step), m.physical_time, m.density_mass, m.density_maximum, m.temperature_maximum,
                        m.maximum_velocity, m.cfl, m.pre_projection_divergence_rms, m.post_projection_divergence_rms, m.divergence_ratio,
                        m.step_milliseconds, m.average_step_milliseconds);
        }
        return 0;
    } catch (const std::exception& error) {
        std::fprintf(stderr, "forward_simulation failed: %s\n", error.what());
        return 1;
    }
}
