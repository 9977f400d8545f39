// dgswemv2-b200-serial: the reference's serial driver (source/dgswemv2-serial.cpp) for the rkdg_swe
// problem on the GPU. Usage: dgswemv2-b200-serial input_file
//
// Runs Serial::GpuSimulation<SWE::RKDG::GpuProblem>: reads the `.15` YAML file and its ADCIRC mesh,
// steps ceil(run_time / dt) times, prints the elapsed time like the reference, then the L2 error when
// the input names a function set with an analytic solution.
#include <chrono>
#include <iomanip>
#include <iostream>

#include "../../include/dgsw_rkdg_problem.hpp"

int main(int argc, char* argv[]) {
    if (argc != 2) {
        std::cerr << "Usage\n"
                  << "    /path/to/dgswemv2-b200-serial input_file\n";
        return 1;
    }
    try {
        Serial::GpuSimulation<SWE::RKDG::GpuProblem> simulation{std::string(argv[1])};
        auto t1 = std::chrono::high_resolution_clock::now();
        simulation.Run();
        dgsw::check(dgsw_rkdg_synchronize(simulation.discretization().handle.get()), "dgsw_rkdg_synchronize");
        auto t2 = std::chrono::high_resolution_clock::now();
        std::cout << "Time Elapsed (in us): " << std::chrono::duration_cast<std::chrono::microseconds>(t2 - t1).count()
                  << "\n";
        if (simulation.input().b200.function_set != 0) simulation.ComputeL2Residual();
        simulation.Finalize();
    } catch (const dgsw::Error& e) {
        std::cerr << e.what() << "\n";
        return 2 + e.status();
    } catch (const std::exception& e) {
        std::cerr << e.what();
        return 2;
    }
    return 0;
}
