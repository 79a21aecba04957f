// ref_on_mdf: the reference's own md::System, built from its unmodified
// sources with src/System/System.cpp replaced by MdfBackend.cpp, so that its
// calculate_energies() and calculate_forces() run on libmdf.  TEST
// INFRASTRUCTURE (oracle/Makefile -> oracle/_ref/ref_on_mdf): the GPU test
// compares what it writes with the golden fixtures of the reference on the
// CPU.
//
// It replays System::init()'s set-up (src/System/init.cpp:12-56) with the
// same two overrides as the O1 harness (Ewald tolerance, PME mesh), then
// calls the System's own calculate_energies() and calculate_forces() - the
// members MdfBackend.cpp defines - and writes, in the O1 harness's format,
// OUTDIR/energies.txt ("name value", %.17g) and OUTDIR/forces.bin (3N f64).
// With --repeat K the pair of calls runs K times (positions unchanged), so a
// test can check that re-evaluation gives the same bits.
//
// usage: ref_on_mdf PRMTOP RST7 OUTDIR [--tol T] [--grid NX NY NZ] [--repeat K]
#include "System/System.h"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s PRMTOP RST7 OUTDIR [--tol T] [--grid NX NY NZ] [--repeat K]\n", argv[0]);
        return 2;
    }
    std::string prm = argv[1], rst = argv[2], out = argv[3];
    double tol = 1e-5;
    int gx = 0, gy = 0, gz = 0, repeat = 1;
    for (int i = 4; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--tol")) tol = std::atof(argv[++i]);
        else if (!std::strcmp(argv[i], "--grid")) { gx = std::atoi(argv[++i]); gy = std::atoi(argv[++i]); gz = std::atoi(argv[++i]); }
        else if (!std::strcmp(argv[i], "--repeat")) repeat = std::atoi(argv[++i]);
        else { std::fprintf(stderr, "unknown option %s\n", argv[i]); return 2; }
    }
    try {
        auto top = md::AmberTopology::AmberTopology::read_topology_coordinates(prm, rst);
        md::System s(top);
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
        s.set_ewald_error_tolerance(tol);
        s.calculate_ewald_alpha();
        s.calculate_ewald_nnodes();
        if (gx > 0) {
            s.newald_mesh_x = gx; s.newald_mesh_y = gy; s.newald_mesh_z = gz;
            s.newald_total = gx * gy * gz;
        }
        std::vector<double> first;
        for (int it = 0; it < repeat; ++it) {
            s.calculate_energies();
            s.calculate_forces();
            if (it == 0) first = s.forces_;
            else if (first != s.forces_) {
                std::fprintf(stderr, "re-evaluation %d changed the forces\n", it);
                return 3;
            }
        }
        FILE* f = std::fopen((out + "/forces.bin").c_str(), "wb");
        if (!f) { std::perror("forces.bin"); return 2; }
        std::fwrite(s.forces_.data(), sizeof(double), s.forces_.size(), f);
        std::fclose(f);
        f = std::fopen((out + "/energies.txt").c_str(), "w");
        if (!f) { std::perror("energies.txt"); return 2; }
        std::fprintf(f, "bond %.17g\n", s.bond_energies_);
        std::fprintf(f, "angle %.17g\n", s.angle_energy_);
        std::fprintf(f, "dihedral %.17g\n", s.dihedral_energy_);
        std::fprintf(f, "ub %.17g\n", s.urey_bradley_energy_);
        std::fprintf(f, "improper %.17g\n", s.improper_energy_);
        std::fprintf(f, "cmap %.17g\n", s.CMAP_energy_);
        std::fprintf(f, "vdw %.17g\n", s.LJ_energy_pairlist_);
        std::fprintf(f, "ee %.17g\n", s.EE_energy_);
        std::fprintf(f, "ee_pairlist %.17g\n", s.EE_energy_pairlist_);
        std::fprintf(f, "ee_cutoff %.17g\n", s.EE_energy_pairlist_cutoff_);
        std::fprintf(f, "ee_direct %.17g\n", s.EE_energy_pairlist_ewald_direct_);
        std::fprintf(f, "ee_self %.17g\n", s.EE_energy_pairlist_ewald_self_);
        std::fclose(f);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_on_mdf: %s\n", e.what());
        return 1;
    }
    return 0;
}
