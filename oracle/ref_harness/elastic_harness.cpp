// Test-infrastructure driver for the reference's elastic CPU solver (cuda/src/cpp).
//
// This file is part of the ORACLE, not of the product. It is compiled together with the
// reference's own, unmodified sources (grid_parameter.cpp, grid_energy.cpp, forward.cpp,
// forward_simulation.cpp, inverse.cpp, input_processing.cpp) by oracle/Makefile, and it
// replaces only the reference's file-driven main (cuda/src/cpp/main_host_FDM_2D.tpp:11-285)
// with a binary-file protocol, so that tests can inject arbitrary media, one source and
// arbitrary receivers and read back the traces, the energy records, the final fields and
// the per-grid coefficients.
//
// The call sequence is the reference's (main_host_FDM_2D.tpp):
//   ns_input_derived_variables                           (:36)
//   dx = num/den, dt given                               (:56-57)
//   set_grid_parameters / set_forward_operators / set_grid_pointers for NN,MN,NM,MM (:96-103)
//   Map_inv_prmt = caller's padded rho/vp/vs             (replaces :134-140)
//   retrieve_forward_parameter, define_parameters_energy, adjust_parameters_energy_periodic,
//   make_density_reciprocal                              (:146-168)
//   process_src_locations / process_rcv_locations        (:202-221)
//   forward_simulation_periodic_y<cpst_N,cpst_S>         (:238-241, forward_simulation.cpp:21)
//
// Input file (little endian):  int64 ih[32]; float64 dh[8]; float64 rho[P], vp[P], vs[P];
//                              int64 rcv[n_rcv][6]  (type_x, type_y, num_x, den_x, num_y, den_y)
//   ih: 0 magic 0x5457454C, 1 Mx, 2 My, 3 Mx_prmt, 4 My_prmt, 5 num_dx, 6 den_dx, 7 num_dxM,
//       8 den_dxM, 9 Nt, 10 cpst_N, 11 cpst_S (char code), 12 src_type_x, 13 src_type_y,
//       14..17 src num_x, den_x, num_y, den_y, 18 n_rcv, 19 quiet,
//       20 boundary type of both x ends (0 = 'F'; another letter selects the reference's
//          SAT interface branch of secure_bdry, grid_drvt.tpp:575-693),
//       21 untimed warm-up passes: the whole run of Nt steps is made this many times from rest
//          before the timed pass (the outputs are those of the timed pass, identical to them)
//       22 1: observed traces follow the receiver table (float64 [n_rcv][2][Nt], the second
//          field ignored on single-field grids); after the run the reference's
//          calculate_data_misfit (forward.cpp:414-445) compares them with the recorded traces
//   dh: 0 dt, 1 central_f, 2 time_delay
// Optional third argument: a folder into which the reference's own writers put their files
// after the run (output_solution_record and output_energy, forward.cpp:215-325, with the text
// output that bool_visual selects).
// With ih[22] = 1 the output file ends with the total misfit and one misfit per receiver (input
// order).
//   P = (Mx_prmt + 2) * (My_prmt + 2)  (the reference's padded model layout, inverse.cpp:79-90)
// Output file: float64 loop_seconds; E_k[Nt]; E_p0[Nt]; E_p1[Nt]; traces[n_rcv][2][Nt];
//              fields NN, MN, NM, MM0, MM1 (reference sizes, row-major, x slow);
//              coefficients NN(mu) MN(1/rho) NM(1/rho) MM(lambda) MM(2mu);
//              energy weights NN MN NM MM(P1) MM(P2).

#include "forward.hpp"
#include "inverse.hpp"

#include <chrono>
#include <cstdio>
#include <cstdint>
#include <vector>
#include <unistd.h>
#include <fcntl.h>

namespace {

template <int N, char S>
void run_cpst(Class_Forward_Specs &fwd) { fwd.forward_simulation_periodic_y<N, S>(); }

bool dispatch_cpst(Class_Forward_Specs &fwd, int n, char s)
{
    if (n == 0 && s == '0') { run_cpst<0, '0'>(fwd); return true; }
    if (n == -3 && s == 'C') { run_cpst<-3, 'C'>(fwd); return true; }
    if (n == -3 && s == 'R') { run_cpst<-3, 'R'>(fwd); return true; }
    if (n == 3 && s == 'C') { run_cpst<3, 'C'>(fwd); return true; }
    if (n == 3 && s == 'R') { run_cpst<3, 'R'>(fwd); return true; }
    if (n == 6 && s == 'C') { run_cpst<6, 'C'>(fwd); return true; }
    if (n == 6 && s == 'R') { run_cpst<6, 'R'>(fwd); return true; }
    return false;
}

// the previous run's energy records must be released before allocate_memory accepts them again
void reset_record(run_time_vector<double> &v, int Nt)
{
    run_time_vector<double> gone(std::move(v));
    v.allocate_memory(Nt);
}

template <typename T>
void put(std::FILE *f, const T *p, size_t n) { std::fwrite(p, sizeof(T), n, f); }

void put_vec(std::FILE *f, run_time_vector<ns_type::host_precision> &v)
{
    std::vector<double> tmp(v.length);
    for (int i = 0; i < v.length; i++) tmp[i] = (double)v.ptr[i];
    put(f, tmp.data(), tmp.size());
}

} // namespace

int main(int argc, char **argv)
{
    if (argc != 3 && argc != 4) { std::fprintf(stderr, "usage: %s input.bin output.bin [folder]\n", argv[0]); return 2; }
    std::FILE *fi = std::fopen(argv[1], "rb");
    if (!fi) { std::fprintf(stderr, "cannot open %s\n", argv[1]); return 2; }
    int64_t ih[32];
    double dh[8];
    if (std::fread(ih, sizeof(ih), 1, fi) != 1 || std::fread(dh, sizeof(dh), 1, fi) != 1) return 2;
    if (ih[0] != 0x5457454C) { std::fprintf(stderr, "bad magic\n"); return 2; }

    using namespace ns_input;
    soln_M_sizes = {(int)ih[1], (int)ih[2]};
    prmt_M_sizes = {(int)ih[3], (int)ih[4]};
    num_dx_soln = (int)ih[5]; den_dx_soln = (int)ih[6];
    num_dx_prmt = (int)ih[7]; den_dx_prmt = (int)ih[8];
    Nt = (int)ih[9];
    const int cpst_N = (int)ih[10];
    const char cpst_S = (char)ih[11];
    const int n_rcv = (int)ih[18];
    const bool quiet = ih[19] != 0;

    bdry_type_L = {'F', 'F'};
    bdry_type_R = {'F', 'F'};
    c_energy = 'Y';
    bool_energy = true;
    bool_visual = false;
    ns_input_derived_variables();
    // ns_input_derived_variables asserts four 'F' sides (namespace_input.hpp:155-160); the x
    // boundary type is only read by secure_bdry, so the interface branch is selected after it
    if (ih[20] != 0 && ih[20] != 'F') {
        Map_bdry_type[{'x', 'L'}] = (char)ih[20];
        Map_bdry_type[{'x', 'R'}] = (char)ih[20];
    }

    dx = static_cast<double>(num_dx_soln) / static_cast<double>(den_dx_soln);
    dt = dh[0];
    central_f = dh[1];
    time_delay = dh[2];

    const long P = PADDED_inv_prmt_size;
    std::vector<double> rho(P), vp(P), vs(P);
    if (std::fread(rho.data(), 8, P, fi) != (size_t)P || std::fread(vp.data(), 8, P, fi) != (size_t)P ||
        std::fread(vs.data(), 8, P, fi) != (size_t)P) { std::fprintf(stderr, "short model\n"); return 2; }
    std::vector<int64_t> rcv((size_t)n_rcv * 6);
    if (n_rcv > 0 && std::fread(rcv.data(), 8, rcv.size(), fi) != rcv.size()) { std::fprintf(stderr, "short rcv\n"); return 2; }
    const bool misfit = ih[22] == 1;
    std::vector<double> obs(misfit ? (size_t)n_rcv * 2 * Nt : 0);
    if (misfit && !obs.empty() && std::fread(obs.data(), 8, obs.size(), fi) != obs.size()) { std::fprintf(stderr, "short obs\n"); return 2; }
    std::fclose(fi);

    int saved_stdout = -1;
    if (quiet) {   // the reference prints per-grid strides and progress lines; keep the test logs clean
        std::fflush(stdout);
        saved_stdout = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        dup2(devnull, 1);
        close(devnull);
    }

    reset_record(Record_E_k, Nt);
    reset_record(Record_E_p0, Nt);
    reset_record(Record_E_p1, Nt);

    Class_Forward_Specs Fwd_Specs;
    Class_Inverse_Specs Inv_Specs;
    std::array<Class_Grid, 4> Grids;
    constexpr auto types = ns_forward::define_Array_Grid_types();
    for (int g = 0; g < 4; g++) Fwd_Specs.Map_Grid_pointers[types.at(g)] = &Grids.at(g);
    for (const auto &t : types) Fwd_Specs.Map_Grid_pointers.at(t)->set_grid_parameters(t, bool_energy);
    for (const auto &t : types) Fwd_Specs.Map_Grid_pointers.at(t)->set_forward_operators();
    for (const auto &t : types) Fwd_Specs.Map_Grid_pointers.at(t)->set_grid_pointers(Fwd_Specs.Map_Grid_pointers);

    const char *names[3] = {"rho", "vp", "vs"};
    const std::vector<double> *src_arrays[3] = {&rho, &vp, &vs};
    for (int k = 0; k < 3; k++) {
        auto &v = Inv_Specs.Map_inv_prmt[names[k]];
        v.allocate_memory(P);
        for (long i = 0; i < P; i++) v.ptr[i] = (*src_arrays[k])[i];
    }
    for (const auto &t : types) Fwd_Specs.Map_Grid_pointers.at(t)->retrieve_forward_parameter(Inv_Specs);
    for (const auto &t : types) Fwd_Specs.Map_Grid_pointers.at(t)->define_parameters_energy();
    for (const auto &t : types) Fwd_Specs.Map_Grid_pointers.at(t)->adjust_parameters_energy_periodic();
    for (const auto &t : types) {
        auto *g = Fwd_Specs.Map_Grid_pointers.at(t);
        if (g->grid_name == "Vx" || g->grid_name == "Vy") g->make_density_reciprocal(Inv_Specs);
    }

    struct_src_input src{};
    src.src_index = 0;
    src.src_grid_type = {(char)ih[12], (char)ih[13]};
    src.src_location = {(int)ih[14], (int)ih[15], (int)ih[16], (int)ih[17]};
    Fwd_Specs.process_src_locations(src);

    std::vector<struct_rcv_input> rcv_in;
    for (int r = 0; r < n_rcv; r++) {
        struct_rcv_input ri{};
        ri.src_index = 0;
        ri.rcv_index = r;
        ri.rcv_grid_type = {(char)rcv[r * 6 + 0], (char)rcv[r * 6 + 1]};
        ri.rcv_location = {(int)rcv[r * 6 + 2], (int)rcv[r * 6 + 3], (int)rcv[r * 6 + 4], (int)rcv[r * 6 + 5]};
        rcv_in.push_back(ri);
    }
    for (const auto &t : types) {
        Fwd_Specs.Map_grid_N_rcvs[t] = 0;
        Fwd_Specs.Map_grid_struct_rcv_forward[t] = {};
        Fwd_Specs.Map_grid_record_rcv[t] = {};
        Fwd_Specs.Map_grid_RESULT_rcv[t] = {};
        Fwd_Specs.Map_grid_misfit_rcv[t] = {};
    }
    Fwd_Specs.process_rcv_locations(rcv_in);

    double loop_seconds = 0.0;
    const int64_t passes = 1 + (ih[21] > 0 ? ih[21] : 0);
    for (int64_t pass = 0; pass < passes; pass++) {
        for (auto &g : Grids)
            for (int f = 0; f < g.N_soln; f++) g.Vec_soln.at(f).set_constant(0.);
        Record_E_k.set_constant(0.);
        Record_E_p0.set_constant(0.);
        Record_E_p1.set_constant(0.);
        if (Nt > 0) {
            auto t0 = std::chrono::steady_clock::now();
            if (!dispatch_cpst(Fwd_Specs, cpst_N, cpst_S)) { std::fprintf(stderr, "bad cpst\n"); return 2; }
            auto t1 = std::chrono::steady_clock::now();
            loop_seconds = std::chrono::duration<double>(t1 - t0).count();
        }
    }

    // the observed traces into the reference's record matrices, receiver by receiver in input
    // order (grouped per grid type in input order, as process_rcv_locations stored them)
    std::vector<double> misfit_rcv;
    if (misfit) {
        std::map<std::array<char, 2>, int> k_of;
        for (int r = 0; r < n_rcv; r++) {
            std::array<char, 2> t = rcv_in[r].rcv_grid_type;
            int k = k_of[t]++;
            auto &M = Fwd_Specs.Map_grid_record_rcv.at(t).at(k);
            for (int f = 0; f < M.rows; f++)
                for (int it = 0; it < Nt; it++) M.at(f, it) = (ns_type::host_precision)obs[((size_t)r * 2 + f) * Nt + it];
        }
        Fwd_Specs.calculate_data_misfit();
        std::map<std::array<char, 2>, int> k2;
        for (int r = 0; r < n_rcv; r++) {
            std::array<char, 2> t = rcv_in[r].rcv_grid_type;
            misfit_rcv.push_back(Fwd_Specs.Map_grid_misfit_rcv.at(t).at(k2[t]++));
        }
    }
    if (argc == 4) {   // the reference's own writers (main_host_FDM_2D.tpp:270-272)
        bool_visual = true;
        Fwd_Specs.output_solution_record(argv[3]);
        Fwd_Specs.output_energy(argv[3]);
    }

    if (quiet) {
        std::fflush(stdout);
        dup2(saved_stdout, 1);
        close(saved_stdout);
    }

    std::FILE *fo = std::fopen(argv[2], "wb");
    if (!fo) return 2;
    put(fo, &loop_seconds, 1);
    put(fo, Record_E_k.ptr, (size_t)Nt);
    put(fo, Record_E_p0.ptr, (size_t)Nt);
    put(fo, Record_E_p1.ptr, (size_t)Nt);

    // receivers in input order; the reference groups them per grid type in input order
    std::map<std::array<char, 2>, int> seen;
    std::vector<double> trace((size_t)2 * Nt);
    for (int r = 0; r < n_rcv; r++) {
        std::array<char, 2> t = rcv_in[r].rcv_grid_type;
        int k = seen[t]++;
        auto &M = Fwd_Specs.Map_grid_RESULT_rcv.at(t).at(k);
        std::fill(trace.begin(), trace.end(), 0.0);
        for (int f = 0; f < M.rows; f++)
            for (int it = 0; it < Nt; it++) trace[(size_t)f * Nt + it] = (double)M.at(f, it);
        put(fo, trace.data(), trace.size());
    }

    Class_Grid &NN = *Fwd_Specs.Map_Grid_pointers.at({'N', 'N'});
    Class_Grid &MN = *Fwd_Specs.Map_Grid_pointers.at({'M', 'N'});
    Class_Grid &NM = *Fwd_Specs.Map_Grid_pointers.at({'N', 'M'});
    Class_Grid &MM = *Fwd_Specs.Map_Grid_pointers.at({'M', 'M'});
    put_vec(fo, NN.Vec_soln.at(0));
    put_vec(fo, MN.Vec_soln.at(0));
    put_vec(fo, NM.Vec_soln.at(0));
    put_vec(fo, MM.Vec_soln.at(0));
    put_vec(fo, MM.Vec_soln.at(1));
    put_vec(fo, NN.Vec_prmt.at(0));
    put_vec(fo, MN.Vec_prmt.at(0));
    put_vec(fo, NM.Vec_prmt.at(0));
    put_vec(fo, MM.Vec_prmt.at(0));
    put_vec(fo, MM.Vec_prmt.at(1));
    put(fo, NN.Vec_prmt_enrg.at(0).ptr, (size_t)NN.Vec_prmt_enrg.at(0).length);
    put(fo, MN.Vec_prmt_enrg.at(0).ptr, (size_t)MN.Vec_prmt_enrg.at(0).length);
    put(fo, NM.Vec_prmt_enrg.at(0).ptr, (size_t)NM.Vec_prmt_enrg.at(0).length);
    put(fo, MM.Vec_prmt_enrg.at(0).ptr, (size_t)MM.Vec_prmt_enrg.at(0).length);
    put(fo, MM.Vec_prmt_enrg.at(1).ptr, (size_t)MM.Vec_prmt_enrg.at(1).length);
    if (misfit) {
        const double total = Fwd_Specs.data_misfit;
        put(fo, &total, 1);
        put(fo, misfit_rcv.data(), misfit_rcv.size());
    }
    std::fclose(fo);
    return 0;
}
