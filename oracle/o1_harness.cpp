// O1 harness: drives the UNMODIFIED reference (prateekbansal97/MD) step by
// step.  TEST INFRASTRUCTURE: built by oracle/Makefile into oracle/_ref/, used
// only by tests, by __graft_entry__.smoke()'s checker and by bench.py's CPU
// baseline / reference arm.  Never linked into the product library.
//
// The reference's System keeps every energy and force routine private
// (include/System/System.h:78-170) and init() prints six digits only
// (src/System/init.cpp:67-79), so this translation unit is compiled with
// -Dprivate=public and replays init()'s sequence (src/System/init.cpp:10-64)
// with two overrides the workloads need: the Ewald tolerance and the PME mesh.
//
// usage:
//   o1_harness PRMTOP RST7 OUTDIR [--tol T] [--grid NX NY NZ] [--no-allpairs]
//                                  [--dump-grids] [--bench K] [--bench-warmup W]
// writes OUTDIR/energies.txt ("name value" with %.17g), forces.bin (3N f64,
// calculate_forces result), forces_pme.bin (3N f64, gather_forces_pme
// result), grid_q.bin / grid_phi.bin (with --dump-grids), info.txt.
// With --bench K it times K force evaluations (PME chain + list energies +
// calculate_forces) and prints one JSON line with per-step seconds.
#include "System/System.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using clk = std::chrono::steady_clock;

static double secs(clk::time_point a, clk::time_point b)
{
    return std::chrono::duration<double>(b - a).count();
}

static void write_bin(const std::string& path, const double* p, size_t n)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { std::perror(path.c_str()); std::exit(2); }
    std::fwrite(p, sizeof(double), n, f);
    std::fclose(f);
}

// PME chain exactly as init() runs it (src/System/init.cpp:59-64)
static void pme_chain(md::System& s, bool first)
{
    s.spread_charge_pme();
    if (first) s.init_pme_resources();
    s.perform_forward_fft();
    s.solve_poisson_kspace();
    s.perform_backward_fft();
    s.gather_forces_pme();
}

// calculate_energies() (src/System/System.cpp:9-23) with the O(N^2)
// all-pairs Coulomb optionally left out
static void list_energies(md::System& s, bool allpairs)
{
    s.calculate_bond_energy();
    s.calculate_angle_energy();
    s.calculate_dihedral_energy();
    s.calculate_UB_energy();
    s.calculate_improper_energy();
    s.calculate_CMAP_energy();
    s.calculate_LJ_energy_pairlist();
    if (allpairs) s.calculate_EE_energy();
    s.calculate_EE_energy_pairlist();
    s.calculate_EE_energy_pairlist_with_cutoff();
    s.calculate_EE_ewald_direct_term();
    s.calculate_EE_ewald_self_term();
}

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s PRMTOP RST7 OUTDIR [options]\n", argv[0]);
        return 2;
    }
    std::string prm = argv[1], rst = argv[2], out = argv[3];
    double tol = 1e-5;
    int gx = 0, gy = 0, gz = 0;
    bool allpairs = true, dump = false;
    int bench = 0, bench_warm = 1;
    for (int i = 4; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--tol")) tol = std::atof(argv[++i]);
        else if (!std::strcmp(argv[i], "--grid")) { gx = std::atoi(argv[++i]); gy = std::atoi(argv[++i]); gz = std::atoi(argv[++i]); }
        else if (!std::strcmp(argv[i], "--no-allpairs")) allpairs = false;
        else if (!std::strcmp(argv[i], "--dump-grids")) dump = true;
        else if (!std::strcmp(argv[i], "--bench")) bench = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--bench-warmup")) bench_warm = std::atoi(argv[++i]);
        else { std::fprintf(stderr, "unknown option %s\n", argv[i]); return 2; }
    }

    auto t0 = clk::now();
    auto top = md::AmberTopology::AmberTopology::read_topology_coordinates(prm, rst);
    md::System s(top);
    auto t_read = clk::now();

    // src/System/init.cpp:12-35 (cutoffs, switch, cells, shift tables, lists)
    s.build_nonbonded_cache();
    const auto b = s.topology_.get_box_dimensions();
    s.set_box(b[0], b[1], b[2]);
    s.set_lj_cutoff(10.0);
    s.set_lj_skin_(2.0);
    s.set_lj_switch_radius(9.0);
    s.set_ee_cutoff(10.0);
    s.set_ee_skin(2.0);
    s.setup_neighbor_rebuild_threshold_lj();
    s.setup_neighbor_rebuild_threshold_ee();
    s.init_box();
    s.precompute_lj_energy_force_shift();
    auto t_pl0 = clk::now();
    s.setup_pairlists();
    auto t_pl1 = clk::now();
    s.copy_ref_coords_lj();
    s.copy_ref_coords_ee();

    // src/System/init.cpp:53-56, tolerance and mesh overridden
    s.set_ewald_error_tolerance(tol);
    s.calculate_ewald_alpha();
    s.calculate_ewald_nnodes();
    if (gx > 0) {
        s.newald_mesh_x = gx; s.newald_mesh_y = gy; s.newald_mesh_z = gz;
        s.newald_total = gx * gy * gz;
    }

    if (bench > 0) {
        // warm-up evaluations, then K timed ones; pairlist built once above
        std::vector<double> t_step, t_pme, t_en, t_f;
        bool first = true;
        for (int it = 0; it < bench_warm + bench; ++it) {
            auto a = clk::now();
            std::fill(s.forces_.begin(), s.forces_.end(), 0.0);
            pme_chain(s, first);
            first = false;
            auto c = clk::now();
            list_energies(s, false);
            auto d = clk::now();
            s.calculate_forces();
            auto e = clk::now();
            if (it >= bench_warm) {
                t_step.push_back(secs(a, e));
                t_pme.push_back(secs(a, c));
                t_en.push_back(secs(c, d));
                t_f.push_back(secs(d, e));
            }
        }
        double sum = 0, sp = 0, se = 0, sf = 0;
        for (size_t i = 0; i < t_step.size(); ++i) { sum += t_step[i]; sp += t_pme[i]; se += t_en[i]; sf += t_f[i]; }
        double n = (double)t_step.size();
        std::printf("{\"natoms\": %lu, \"pairs\": %zu, \"steps\": %d, \"s_per_step\": %.6f, "
                    "\"s_pme_chain\": %.6f, \"s_list_energies\": %.6f, \"s_calculate_forces\": %.6f, "
                    "\"s_pairlist\": %.6f, \"s_read\": %.6f, \"mesh\": [%d, %d, %d]}\n",
                    (unsigned long)s.natoms_, s.lj_pairs_.size(), bench, sum / n, sp / n, se / n, sf / n,
                    secs(t_pl0, t_pl1), secs(t0, t_read), s.newald_mesh_x, s.newald_mesh_y, s.newald_mesh_z);
        return 0;
    }

    // PME chain as init() runs it; forces_ holds only the PME forces here
    s.spread_charge_pme();
    if (dump) write_bin(out + "/grid_q.bin", s.pme_grid_charge_.data(), s.pme_grid_charge_.size());
    s.init_pme_resources();
    s.perform_forward_fft();
    s.solve_poisson_kspace();
    s.perform_backward_fft();
    if (dump) write_bin(out + "/grid_phi.bin", s.pme_grid_charge_.data(), s.pme_grid_charge_.size());
    s.gather_forces_pme();
    write_bin(out + "/forces_pme.bin", s.forces_.data(), s.forces_.size());
    auto t_pme = clk::now();

    list_energies(s, allpairs);
    auto t_en = clk::now();
    s.calculate_forces();
    auto t_f = clk::now();
    write_bin(out + "/forces.bin", s.forces_.data(), s.forces_.size());

    FILE* f = std::fopen((out + "/energies.txt").c_str(), "w");
    if (!f) { std::perror("energies.txt"); return 2; }
    std::fprintf(f, "bond %.17g\n", s.bond_energies_);
    std::fprintf(f, "angle %.17g\n", s.angle_energy_);
    std::fprintf(f, "dihedral %.17g\n", s.dihedral_energy_);
    std::fprintf(f, "ub %.17g\n", s.urey_bradley_energy_);
    std::fprintf(f, "improper %.17g\n", s.improper_energy_);
    std::fprintf(f, "cmap %.17g\n", s.CMAP_energy_);
    std::fprintf(f, "vdw %.17g\n", s.LJ_energy_pairlist_);
    if (allpairs) std::fprintf(f, "ee %.17g\n", s.EE_energy_);
    std::fprintf(f, "ee_pairlist %.17g\n", s.EE_energy_pairlist_);
    std::fprintf(f, "ee_cutoff %.17g\n", s.EE_energy_pairlist_cutoff_);
    std::fprintf(f, "ee_direct %.17g\n", s.EE_energy_pairlist_ewald_direct_);
    std::fprintf(f, "ee_self %.17g\n", s.EE_energy_pairlist_ewald_self_);
    std::fclose(f);

    f = std::fopen((out + "/info.txt").c_str(), "w");
    std::fprintf(f, "natoms %lu\npairs %zu\nalpha %.17g\nmesh %d %d %d\ntol %.17g\n"
                    "t_read %.6f\nt_pairlist %.6f\nt_pme %.6f\nt_energies %.6f\nt_forces %.6f\n",
                 (unsigned long)s.natoms_, s.lj_pairs_.size(), s.ewald_alpha_, s.newald_mesh_x,
                 s.newald_mesh_y, s.newald_mesh_z, s.ewald_error_tolerance_, secs(t0, t_read),
                 secs(t_pl0, t_pl1), secs(t_pl1, t_pme), secs(t_pme, t_en), secs(t_en, t_f));
    std::fclose(f);
    return 0;
}
