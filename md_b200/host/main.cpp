// mdb200: the reference's command line (apps/main.cpp: ./md <prmtop> [coords])
// on the GPU engine.  Reads the topology and coordinates, evaluates the
// energies and forces once and prints them the way the reference's init()
// does (src/System/init.cpp), with full precision.  Options go beyond the
// reference: PHYSICAL semantics, mixed precision, minimisation, dynamics.
//
//   mdb200 <prmtop> [coords] [--physical] [--mixed] [--tol T] [--grid NX NY NZ]
//          [--device D] [--minimize ITERS] [--md STEPS DT_PS] [--rst7-out PATH]
//          [--forces-out PATH] [--dump-topology DIR]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>

#include "amber_topology.hpp"
#include "system.hpp"

using namespace mdb200;

static void usage()
{
    std::cerr << "Usage: mdb200 <prmtop> [coords] [--physical] [--mixed] [--tol T] [--grid NX NY NZ] "
                 "[--device D] [--minimize ITERS] [--md STEPS DT_PS] [--rst7-out PATH] [--forces-out PATH] "
                 "[--dump-topology DIR]\n";
}

template <typename T>
static void dump(const std::string& dir, const char* name, const std::vector<T>& v)
{
    std::ofstream f(dir + "/" + name + ".bin", std::ios::binary);
    if (!v.empty()) f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
    if (!f) throw std::runtime_error(std::string("cannot write ") + name);
}

static void dump_topology(const FlatTopology& o, const std::string& dir)
{
    dump(dir, "charge", o.charge); dump(dir, "type", o.type); dump(dir, "nb_index", o.nb_index);
    dump(dir, "lj_a", o.lj_a); dump(dir, "lj_b", o.lj_b); dump(dir, "lj14_a", o.lj14_a); dump(dir, "lj14_b", o.lj14_b);
    dump(dir, "bond_atoms", o.bond_atoms); dump(dir, "bond_k", o.bond_k); dump(dir, "bond_r0", o.bond_r0);
    dump(dir, "ub_atoms", o.ub_atoms); dump(dir, "ub_k", o.ub_k); dump(dir, "ub_r0", o.ub_r0);
    dump(dir, "angle_atoms", o.angle_atoms); dump(dir, "angle_k", o.angle_k);
    dump(dir, "angle_theta0", o.angle_theta0);
    dump(dir, "dihedral_atoms", o.dihedral_atoms); dump(dir, "dihedral_k", o.dihedral_k);
    dump(dir, "dihedral_n", o.dihedral_n); dump(dir, "dihedral_phase", o.dihedral_phase);
    dump(dir, "improper_atoms", o.improper_atoms); dump(dir, "improper_k", o.improper_k);
    dump(dir, "improper_phase", o.improper_phase);
    dump(dir, "cmap_atoms", o.cmap_atoms); dump(dir, "cmap_set", o.cmap_set); dump(dir, "cmap_coeff", o.cmap_coeff);
    dump(dir, "excl_pairs", o.excl_pairs); dump(dir, "pairs14", o.pairs14);
    dump(dir, "scee14", o.scee14); dump(dir, "scnb14", o.scnb14);
}

int main(int argc, char* argv[])
{
    if (argc < 2) {
        usage();
        return 1;
    }
    std::string prmtop = argv[1], coords, rst7_out, forces_out, dump_dir;
    int sem = MDF_SEM_REFERENCE, prec = MDF_PREC_FP64, device = 0, min_iters = 0, grid[3] = {0, 0, 0};
    long long md_steps = 0;
    double tol = 1e-6, dt = 0.0005;
    int a = 2;
    if (argc > 2 && argv[2][0] != '-') coords = argv[a++];
    for (; a < argc; ++a) {
        const std::string o = argv[a];
        auto need = [&](int k) {
            if (a + k >= argc) {
                usage();
                std::exit(1);
            }
        };
        if (o == "--physical") sem = MDF_SEM_PHYSICAL;
        else if (o == "--reference") sem = MDF_SEM_REFERENCE;
        else if (o == "--mixed") prec = MDF_PREC_MIXED;
        else if (o == "--tol") { need(1); tol = std::atof(argv[++a]); }
        else if (o == "--grid") { need(3); for (int d = 0; d < 3; ++d) grid[d] = std::atoi(argv[++a]); }
        else if (o == "--device") { need(1); device = std::atoi(argv[++a]); }
        else if (o == "--minimize") { need(1); min_iters = std::atoi(argv[++a]); }
        else if (o == "--md") { need(2); md_steps = std::atoll(argv[++a]); dt = std::atof(argv[++a]); }
        else if (o == "--rst7-out") { need(1); rst7_out = argv[++a]; }
        else if (o == "--forces-out") { need(1); forces_out = argv[++a]; }
        else if (o == "--dump-topology") { need(1); dump_dir = argv[++a]; }
        else { usage(); return 1; }
    }
    try {
        const auto t0 = std::chrono::steady_clock::now();
        AmberTopology top = AmberTopology::read(prmtop, coords);
        const auto t1 = std::chrono::steady_clock::now();
        if (!dump_dir.empty()) {
            const FlatTopology flat = flatten(top, sem);
            const auto t2 = std::chrono::steady_clock::now();
            std::printf("read %d atoms in %.3f s, flattened in %.3f s\n", top.natoms,
                        std::chrono::duration<double>(t1 - t0).count(), std::chrono::duration<double>(t2 - t1).count());
            dump_topology(flat, dump_dir);
            return 0;
        }
        std::vector<double> mass = top.mass;
        System sys(std::move(top), sem, prec, device);
        sys.set_ewald_error_tolerance(tol);
        if (grid[0] > 0) sys.set_pme_grid(grid[0], grid[1], grid[2]);
        sys.init();
        std::printf("nX: %d nY: %d nZ: %d\n", sys.mesh(0), sys.mesh(1), sys.mesh(2));
        if (min_iters > 0) {
            mdf_min_report r;
            if (mdf_minimize_lbfgs(sys.context(), min_iters, 1.0, 0.1, 8, &r) != MDF_OK)
                throw std::runtime_error(mdf_last_error(sys.context()));
            std::printf("minimised (L-BFGS): %d iterations, %d evaluations, E %.10g -> %.10g, max |F| %.6g\n",
                        r.iterations, r.evaluations, r.e_initial, r.e_final, r.fmax_final);
        }
        if (md_steps > 0) {
            mdf_md_report r;
            if (mdf_md_init(sys.context(), mass.data(), nullptr, 300.0, 1) != MDF_OK ||
                mdf_md_run(sys.context(), md_steps, dt, 10, 10, nullptr, 0, &r) != MDF_OK)
                throw std::runtime_error(mdf_last_error(sys.context()));
            std::printf("dynamics: %lld steps in %.3f s (%.1f steps/s), E_total %.10g -> %.10g\n",
                        (long long)r.steps, r.wall_s, r.steps / r.wall_s, r.pe_first + r.ke_first,
                        r.pe_last + r.ke_last);
            if (!rst7_out.empty() &&
                mdf_md_write_rst7(sys.context(), rst7_out.c_str(), "mdb200", md_steps * dt) != MDF_OK)
                throw std::runtime_error(mdf_last_error(sys.context()));
        }
        sys.calculate_energies();
        std::printf("\nBond: %.17g\nAngle: %.17g\nCosineDihedral: %.17g\nUrey-Bradley: %.17g\nImpropers: %.17g\n"
                    "CMAP energy: %.17g\nVDW: %.17g\n",
                    sys.bond_energies(), sys.angle_energy(), sys.dihedral_energy(), sys.urey_bradley_energy(),
                    sys.improper_energy(), sys.CMAP_energy(), sys.LJ_energy_pairlist());
        if (sem == MDF_SEM_REFERENCE)
            std::printf("EE: %.17g\nEE pairlist: %.17g\nEE_energy_pairlist_cutoff_ %.17g\n"
                        "EE_energy_pairlist_ewald_direct_ %.17g\nEE_energy_pairlist_ewald_self_ %.17g\n",
                        sys.EE_energy(), sys.EE_energy_pairlist(), sys.EE_energy_pairlist_cutoff(),
                        sys.EE_energy_pairlist_ewald_direct(), sys.EE_energy_pairlist_ewald_self());
        else
            std::printf("VDW14: %.17g\nEE direct: %.17g\nEE14: %.17g\nEE exclusions: %.17g\nEE self: %.17g\n"
                        "EE reciprocal: %.17g\nTotal: %.17g\n",
                        sys.energies().e[MDF_E_VDW14], sys.energies().e[MDF_E_EE_DIRECT],
                        sys.energies().e[MDF_E_EE14], sys.energies().e[MDF_E_EE_EXCL],
                        sys.energies().e[MDF_E_EE_SELF], sys.energies().e[MDF_E_EE_RECIP], sys.energies().total);
        sys.calculate_forces();
        const auto& f = sys.forces();
        std::printf("Calculated Forces!\n%.17g %.17g %.17g\n", f[0], f[1], f[2]);
        if (!forces_out.empty()) {
            std::ofstream fo(forces_out, std::ios::binary);
            fo.write(reinterpret_cast<const char*>(f.data()), (std::streamsize)(f.size() * sizeof(double)));
        }
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 2;
    }
    return 0;
}
