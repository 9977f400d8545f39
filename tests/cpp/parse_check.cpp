// Test driver for the C++ host side (include/dgsw_rkdg_problem.hpp): parses a `.15` input file and its
// ADCIRC mesh without a GPU and prints what it read, one "key value" per line, then the host-only
// topology of the mesh (dgsw_mesh_topology) as counts and checksums. Errors print "error <status>
// <message>" and exit 3. With a second argument (a directory), the mesh arrays the reader produced are
// also written there as raw little-endian files (<name>.bin) plus an index (arrays.txt: name, type,
// element count), so that a test can hand exactly these arrays to the library and to the oracle.
#include <cstdint>
#include <fstream>
#include <iostream>

#include "../../include/dgsw_rkdg_problem.hpp"

static uint64_t fnv(const void* p, size_t n, uint64_t h = 1469598103934665603ull) {
    const unsigned char* c = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
    return h;
}

struct Dump {
    std::string dir;
    std::ofstream index;
    explicit Dump(const std::string& d) : dir(d), index(d + "/arrays.txt") {}
    template <typename T>
    void put(const std::string& name, const char* type, const std::vector<T>& v) {
        std::ofstream f(dir + "/" + name + ".bin", std::ios::binary);
        if (!v.empty()) f.write((const char*)v.data(), (std::streamsize)(v.size() * sizeof(T)));
        index << name << " " << type << " " << v.size() << "\n";
    }
};

int main(int argc, char** argv) {
    if (argc != 2 && argc != 3) return 1;
    try {
        dgsw::InputParameters in(argv[1]);
        const auto& pi = in.problem_input;
        std::cout.precision(17);
        std::cout << "p " << in.polynomial_order << "\n"
                  << "mesh_format " << in.mesh_input.mesh_format << "\n"
                  << "mesh_file " << in.mesh_input.mesh_file_name << "\n"
                  << "bcis_file " << in.mesh_input.bc_is_file_name << "\n"
                  << "coordinate_system " << in.mesh_input.coordinate_system << "\n"
                  << "run_time " << in.stepper_input.run_time << "\n"
                  << "dt " << in.stepper_input.dt << "\n"
                  << "order " << in.stepper_input.order << "\n"
                  << "nstages " << in.stepper_input.nstages << "\n"
                  << "name " << pi.name << "\n"
                  << "g " << pi.g << "\n"
                  << "rho_air " << pi.rho_air << "\n"
                  << "ic_type " << pi.ic_type << "\n"
                  << "ic_const " << pi.ze_initial << " " << pi.qx_initial << " " << pi.qy_initial << "\n"
                  << "function_source " << pi.function_source << "\n"
                  << "wetting_drying " << pi.wetting_drying << "\n"
                  << "h_o " << pi.h_o << "\n"
                  << "slope_limiting " << pi.slope_limiting << "\n"
                  << "sl_M " << pi.sl_M << "\n"
                  << "sl_nu " << pi.sl_nu << "\n"
                  << "spherical " << pi.spherical << "\n"
                  << "writing_vtk " << in.writer_input.writing_vtk_output << " "
                  << in.writer_input.vtk_output_freq_step << "\n"
                  << "writing_vtu " << in.writer_input.writing_vtu_output << " "
                  << in.writer_input.vtu_output_freq_step << "\n"
                  << "writing_modal " << in.writer_input.writing_modal_output << " "
                  << in.writer_input.modal_output_freq_step << "\n"
                  << "function_set " << in.b200.function_set << "\n"
                  << "precision " << in.b200.precision << "\n"
                  << "n_params " << in.b200.function_parameters.size() << "\n"
                  << "bottom_friction " << pi.bottom_friction << " " << pi.friction_coefficient << "\n"
                  << "manning_file " << pi.manning_data_file << "\n"
                  << "ramp_duration " << in.stepper_input.ramp_duration << "\n";
        dgsw::AdcircMesh M = dgsw::read_adcirc(dgsw::input_relative(in.input_dir, in.mesh_input.mesh_file_name));
        dgsw::read_bcis(dgsw::input_relative(in.input_dir, in.mesh_input.bc_is_file_name), M);
        dgsw::project_spherical(in, M);
        std::cout << "projected_xyz_hash " << fnv(M.node_xyz.data(), M.node_xyz.size() * 8) << "\n";
        if (pi.bottom_friction == DGSW_FRICTION_MANNING)
            dgsw::read_manning(dgsw::input_relative(in.input_dir, pi.manning_data_file), M);
        std::cout << "n_forcing " << M.forcing.size() << "\n";
        for (size_t b = 0; b < M.forcing.size(); ++b) {
            const auto& F = M.forcing[b];
            std::cout << "forcing_" << b << " " << F.type << " " << F.nodes.size() << " " << F.frequency.size() << " "
                      << fnv(F.nodes.data(), F.nodes.size() * 4) << " "
                      << fnv(F.frequency.data(), F.frequency.size() * 8,
                             fnv(F.forcing_fact.data(), F.forcing_fact.size() * 8,
                                 fnv(F.equilib_arg.data(), F.equilib_arg.size() * 8)))
                      << " " << fnv(F.amplitude.data(), F.amplitude.size() * 8) << " "
                      << fnv(F.phase.data(), F.phase.size() * 8) << "\n";
        }
        std::cout << "manning_hash " << fnv(M.node_manning_n.data(), M.node_manning_n.size() * 8) << "\n"
                  << "n_levee_pairs " << M.levee_nodes.size() / 2 << "\n"
                  << "levee_hash " << fnv(M.levee_nodes.data(), M.levee_nodes.size() * 4) << " "
                  << fnv(M.levee_data.data(), M.levee_data.size() * 8) << "\n";
        std::cout << "mesh_name " << M.name << "\n"
                  << "n_nodes " << M.n_nodes() << "\n"
                  << "n_elems " << M.n_elems() << "\n"
                  << "n_segments " << M.seg_type.size() << "\n"
                  << "node_xyz_hash " << fnv(M.node_xyz.data(), M.node_xyz.size() * 8) << "\n"
                  << "elem_nodes_hash " << fnv(M.elem_nodes.data(), M.elem_nodes.size() * 4) << "\n"
                  << "elem_ids_hash " << fnv(M.elem_names.data(), M.elem_names.size() * 4) << "\n"
                  << "seg_type_hash " << fnv(M.seg_type.data(), M.seg_type.size() * 4) << "\n"
                  << "seg_nodes_hash " << fnv(M.seg_nodes.data(), M.seg_nodes.size() * 4) << "\n";
        if (argc == 3) {
            Dump D(argv[2]);
            D.put("node_xyz", "f64", M.node_xyz);
            D.put("elem_nodes", "i32", M.elem_nodes);
            D.put("elem_ids", "u32", M.elem_names);
            D.put("seg_type", "i32", M.seg_type);
            D.put("seg_offsets", "i64", M.seg_offsets);
            D.put("seg_nodes", "i32", M.seg_nodes);
            D.put("node_manning_n", "f64", M.node_manning_n);
            D.put("levee_nodes", "i32", M.levee_nodes);
            D.put("levee_data", "f64", M.levee_data);
            for (size_t b = 0; b < M.forcing.size(); ++b) {
                const auto& F = M.forcing[b];
                const std::string k = "forcing" + std::to_string(b) + "_";
                D.put(k + "type", "i32", std::vector<int32_t>{F.type});
                D.put(k + "nodes", "i32", F.nodes);
                D.put(k + "frequency", "f64", F.frequency);
                D.put(k + "forcing_fact", "f64", F.forcing_fact);
                D.put(k + "equilib_arg", "f64", F.equilib_arg);
                D.put(k + "amplitude", "f64", F.amplitude);
                D.put(k + "phase", "f64", F.phase);
            }
        }
        const dgsw_mesh m = M.view();
        int64_t ni = 0, nb = 0;
        dgsw::check(dgsw_mesh_topology(&m, nullptr, nullptr, &ni, nullptr, &nb, nullptr), "dgsw_mesh_topology");
        std::vector<int32_t> nbr(3 * M.n_elems()), intf(4 * ni), bnd(3 * nb);
        std::vector<uint8_t> bt(3 * M.n_elems());
        dgsw::check(dgsw_mesh_topology(&m, nbr.data(), bt.data(), &ni, intf.data(), &nb, bnd.data()),
                    "dgsw_mesh_topology");
        std::cout << "n_interfaces " << ni << "\n"
                  << "n_boundaries " << nb << "\n"
                  << "neighbors_hash " << fnv(nbr.data(), nbr.size() * 4) << "\n"
                  << "btype_hash " << fnv(bt.data(), bt.size()) << "\n"
                  << "interfaces_hash " << fnv(intf.data(), intf.size() * 4) << "\n"
                  << "boundaries_hash " << fnv(bnd.data(), bnd.size() * 4) << "\n";
    } catch (const dgsw::Error& e) {
        std::cout << "error " << e.status() << " " << e.what() << "\n";
        return 3;
    } catch (const std::exception& e) {
        std::cout << "error -1 " << e.what() << "\n";
        return 3;
    }
    return 0;
}
