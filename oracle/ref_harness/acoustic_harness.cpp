// Test-infrastructure driver for the reference's single-core acoustic solver (singlecore/).
//
// This file is part of the ORACLE, not of the product. oracle/Makefile compiles it as the only
// translation unit that includes the reference's unmodified singlecore/src/cpp/namespaces.hpp
// (which defines its fields as non-inline globals, so one simulation runs per process).
// It replaces singlecore/src/main_cpp/cpu_acoustic.cpp's main, which never parses its command
// line and hard-codes dt (cpu_acoustic.cpp:78), with a binary-file protocol:
//   * the single-rank geometry that main derives at cpu_acoustic.cpp:72-157 is set directly
//     (pad 1 on N grids and 2 on M grids, namespaces.hpp map_len_LIR);
//   * the coefficients (1/rho on Vx and Vy, 1/beta = kappa on P, cpu_acoustic.cpp:178-180)
//     come from the caller, per grid point, instead of constants;
//   * the time loop calls the reference's own actions in the reference's order
//     (cpu_acoustic.cpp:247-344): copy_to_halo, take_drvt, update_soln, the P source at
//     t = (it + 1/2) dt - delay, then the records;
//   * any number of receivers are read straight from the solution arrays after each step
//     (the reference keeps one receiver per mesh, namespaces.hpp:329-330).
//
// Input file (little endian): int64 ih[16]; float64 dh[8]; float64 prmt_Vx[(Nx+1)*Ny],
//   prmt_Vy[Nx*(Ny+1)], prmt_P[Nx*Ny]; int64 rcv[n_rcv][3] (mesh 0=Vx 1=Vy 2=P, ix, iy)
//   ih: 0 magic 0x54574143, 1 Nel_x, 2 Nel_y, 3 Nt, 4 cpst char ('0','3','6'), 5 src ix (P cell),
//       6 src iy, 7 n_rcv, 8 quiet
//   dh: 0 dx, 1 dt, 2 central_f, 3 time_delay
// Output file: float64 loop_seconds; energy[3][Nt] (Vx, Vy, P sums); traces[n_rcv][Nt];
//   fields Vx, Vy, P (unpadded, row-major, x slow).

#include <array>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fcntl.h>
#include <unistd.h>
#include <vector>

#include "namespaces.hpp"

namespace {

template <typename T>
void put(std::FILE *f, const T *p, size_t n) { std::fwrite(p, sizeof(T), n, f); }

// unpadded (ix, iy) of mesh -> padded 2D index; pads: N grid 1, M grid 2
long padded_index(class_mesh &m, long ix, long iy)
{
    const long px = ns_config::map_bgn.at('x').at(m.T_x);
    const long py = ns_config::map_bgn.at('y').at(m.T_y);
    return m.hst_soln.convert_index(ix + px, iy + py);
}

} // namespace

int main(int argc, char **argv)
{
    if (argc != 3) { std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]); return 2; }
    std::FILE *fi = std::fopen(argv[1], "rb");
    if (!fi) return 2;
    int64_t ih[16];
    double dh[8];
    if (std::fread(ih, sizeof(ih), 1, fi) != 1 || std::fread(dh, sizeof(dh), 1, fi) != 1) return 2;
    if (ih[0] != 0x54574143) { std::fprintf(stderr, "bad magic\n"); return 2; }
    const long Nx = ih[1], Ny = ih[2];
    const int n_rcv = (int)ih[7];
    const bool quiet = ih[8] != 0;

    std::vector<double> in_vx((Nx + 1) * Ny), in_vy(Nx * (Ny + 1)), in_p(Nx * Ny);
    if (std::fread(in_vx.data(), 8, in_vx.size(), fi) != in_vx.size() ||
        std::fread(in_vy.data(), 8, in_vy.size(), fi) != in_vy.size() ||
        std::fread(in_p.data(), 8, in_p.size(), fi) != in_p.size()) return 2;
    std::vector<int64_t> rcv((size_t)n_rcv * 3);
    if (n_rcv > 0 && std::fread(rcv.data(), 8, rcv.size(), fi) != rcv.size()) return 2;
    std::fclose(fi);

    int saved_stdout = -1;
    if (quiet) {
        std::fflush(stdout);
        saved_stdout = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        dup2(devnull, 1);
        close(devnull);
    }

    using namespace ns_config;
    ns_mpi::rank = 0;
    ns_mpi::size = 1;
    Nt = (int)ih[3];
    char_cpst = (char)ih[4];
    dx = dh[0];
    dt = dh[1];
    central_f = dh[2];
    time_delay = dh[3];
    multiple = 1;
    src_loc_i_base_ppw = ih[5];
    src_loc_j_base_ppw = ih[6];
    rcv_loc_i_base_ppw = 0;
    rcv_loc_j_base_ppw = 0;

    // single-rank geometry (one subdomain = the whole periodic domain)
    const long nel[2] = {Nx, Ny};
    const char dirs[2] = {'x', 'y'};
    for (int d = 0; d < 2; d++) {
        const char dir = dirs[d];
        map_Nel_entire.at(dir) = (int)nel[d];
        map_Nel.at(dir) = (int)nel[d];
        map_bgn_entire.at(dir).at('M') = 0;
        map_end_entire.at(dir).at('M') = (int)nel[d];
        map_bgn_entire.at(dir).at('N') = 0;
        map_end_entire.at(dir).at('N') = (int)nel[d] + 1;
        map_len_LIR[dir]['N']['I'] = (int)nel[d] + 1;
        map_len_LIR[dir]['N']['L'] = 1;
        map_len_LIR[dir]['N']['R'] = 1;
        map_len_LIR[dir]['M']['I'] = (int)nel[d];
        map_len_LIR[dir]['M']['L'] = 2;
        map_len_LIR[dir]['M']['R'] = 2;
        for (char T : {'N', 'M'}) {
            auto &lir = map_len_LIR.at(dir).at(T);
            map_len.at(dir).at(T) = lir.at('L') + lir.at('I') + lir.at('R');
            map_bgn.at(dir).at(T) = lir.at('L');
            map_end.at(dir).at(T) = map_len.at(dir).at(T) - lir.at('R');
        }
    }

    for (auto field : {"prmt", "soln", "rths"})
        for (auto mesh : {"Vx", "Vy", "P"}) {
            std::array<char, 2> t = mesh2char.at(mesh);
            ns_fields::field2mesh2resource.at(field).at(mesh)->allocate_memory(
                {(long)map_len.at('x').at(t[0]), (long)map_len.at('y').at(t[1])});
        }
    for (auto mesh : {"Vx", "Vy", "P"}) {
        ns_fields::mesh2signal.at(mesh)->allocate_memory((long)Nt);
        ns_fields::mesh2energy.at(mesh)->allocate_memory((long)Nt);
    }
    ns_energy::prepare_energy_weight();

    ns_meshes::mesh_Vx.initialize('N', 'M');
    ns_meshes::mesh_Vy.initialize('M', 'N');
    ns_meshes::mesh_P.initialize('M', 'M');

    class_mesh *meshes[3] = {&ns_meshes::mesh_Vx, &ns_meshes::mesh_Vy, &ns_meshes::mesh_P};
    const std::vector<double> *coefs[3] = {&in_vx, &in_vy, &in_p};
    const long sx[3] = {Nx + 1, Nx, Nx}, sy[3] = {Ny, Ny + 1, Ny};
    for (int m = 0; m < 3; m++)
        for (long ix = 0; ix < sx[m]; ix++)
            for (long iy = 0; iy < sy[m]; iy++)
                meshes[m]->hst_prmt.at(padded_index(*meshes[m], ix, iy)) =
                    (ns_prcs::precision)(*coefs[m])[ix * sy[m] + iy];

    std::vector<long> rcv_index(n_rcv);
    std::vector<int> rcv_mesh(n_rcv);
    for (int r = 0; r < n_rcv; r++) {
        rcv_mesh[r] = (int)rcv[r * 3];
        rcv_index[r] = padded_index(*meshes[rcv_mesh[r]], rcv[r * 3 + 1], rcv[r * 3 + 2]);
    }
    std::vector<double> traces((size_t)n_rcv * Nt);
    std::vector<double> energy((size_t)3 * Nt);

    using ns_meshes::mesh_P;
    using ns_meshes::mesh_Vx;
    using ns_meshes::mesh_Vy;
    auto t0 = std::chrono::steady_clock::now();
    for (int it = 0; it < Nt; it++) {
        ns_action::copy_to_halo<'x'>(mesh_P);
        for (long ix = map_bgn.at('x').at('N'); ix < map_end.at('x').at('N'); ix++)
            for (long iy = map_bgn.at('y').at('M'); iy < map_end.at('y').at('M'); iy++) {
                ns_action::take_drvt<'x', 'N'>(ix, iy, mesh_Vx, mesh_P);
                ns_action::update_soln(ix, iy, mesh_Vx);
            }
        ns_action::copy_to_halo<'y'>(mesh_P);
        for (long ix = map_bgn.at('x').at('M'); ix < map_end.at('x').at('M'); ix++)
            for (long iy = map_bgn.at('y').at('N'); iy < map_end.at('y').at('N'); iy++) {
                ns_action::take_drvt<'y', 'N'>(ix, iy, mesh_Vy, mesh_P);
                ns_action::update_soln(ix, iy, mesh_Vy);
            }
        ns_action::copy_to_halo<'x'>(mesh_Vx);
        ns_action::copy_to_halo<'y'>(mesh_Vy);
        for (long ix = map_bgn.at('x').at('M'); ix < map_end.at('x').at('M'); ix++)
            for (long iy = map_bgn.at('y').at('M'); iy < map_end.at('y').at('M'); iy++) {
                ns_action::take_drvt<'x', 'M'>(ix, iy, mesh_P, mesh_Vx);
                ns_action::take_drvt<'y', 'M'>(ix, iy, mesh_P, mesh_Vy);
                ns_action::update_soln(ix, iy, mesh_P);
            }
        if (mesh_P.bool_src) {
            const double t = (it + 1 - 1. / 2.) * dt - time_delay;
            const double A = (1 - 2 * M_PI * M_PI * central_f * central_f * t * t) *
                             exp(-M_PI * M_PI * central_f * central_f * t * t);
            mesh_P.hst_soln(mesh_P.I_SRC) += A * dt / (dx * dx);
        }
        for (int r = 0; r < n_rcv; r++)
            traces[(size_t)r * Nt + it] = (double)meshes[rcv_mesh[r]]->hst_soln(rcv_index[r]);
        const char *names[3] = {"Vx", "Vy", "P"};
        for (int m = 0; m < 3; m++) {
            auto &soln = meshes[m]->hst_soln;
            auto &prmt = meshes[m]->hst_prmt;
            auto &w = ns_fields::mesh2weight_energy.at(names[m])->acc;
            double e = 0.;
            for (long i = 0; i < soln.length; i++) e += soln(i) * prmt(i) * soln(i) * w(i);
            energy[(size_t)m * Nt + it] = e;
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    double loop_seconds = std::chrono::duration<double>(t1 - t0).count();

    if (quiet) {
        std::fflush(stdout);
        dup2(saved_stdout, 1);
        close(saved_stdout);
    }

    std::FILE *fo = std::fopen(argv[2], "wb");
    if (!fo) return 2;
    put(fo, &loop_seconds, 1);
    put(fo, energy.data(), energy.size());
    put(fo, traces.data(), traces.size());
    for (int m = 0; m < 3; m++) {
        std::vector<double> out((size_t)sx[m] * sy[m]);
        for (long ix = 0; ix < sx[m]; ix++)
            for (long iy = 0; iy < sy[m]; iy++)
                out[ix * sy[m] + iy] = (double)meshes[m]->hst_soln.at(padded_index(*meshes[m], ix, iy));
        put(fo, out.data(), out.size());
    }
    std::fclose(fo);
    return 0;
}
