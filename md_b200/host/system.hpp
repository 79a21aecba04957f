// mdb200::System: the reference's md::System interface (include/System/
// System.h:33-190) on libmdf.  The same construction from a parsed topology,
// init() with the reference's settings (src/System/init.cpp: cutoff 10 A,
// skin 2 A, LJ switch at 9 A, Ewald tolerance 1e-6, the reference's mesh
// formula), calculate_energies() and calculate_forces() filling the energy
// members and forces_ (force, not gradient, kcal/mol/A, 3N atom-major) the
// reference fills.  Every evaluation runs on the GPU through the C ABI; there
// is no CPU path.  Errors throw std::runtime_error with the library's message.
#pragma once

#include <string>
#include <vector>

#include "amber_topology.hpp"
#include "mdf.h"

namespace mdb200 {

class System {
public:
    // semantics: MDF_SEM_REFERENCE (the reference as it runs) or
    // MDF_SEM_PHYSICAL; precision: MDF_PREC_FP64 or MDF_PREC_MIXED.
    explicit System(AmberTopology topology, int semantics = MDF_SEM_REFERENCE, int precision = MDF_PREC_FP64,
                    int device = 0);
    ~System();
    System(const System&) = delete;
    System& operator=(const System&) = delete;

    // settings (before init(); the reference's setters, include/System/System.h:45-53)
    void set_box(double Lx, double Ly, double Lz);
    void set_lj_cutoff(double rc) { cutoff_ = rc; }
    void set_lj_skin_(double skin) { skin_ = skin; }
    void set_lj_switch_radius(double r) { switch_ = r; }
    void set_ewald_error_tolerance(double tol) { tol_ = tol; }
    void set_pme_grid(int nx, int ny, int nz) { grid_[0] = nx; grid_[1] = ny; grid_[2] = nz; }

    void init();                  // creates the GPU context and builds the pairlist
    void calculate_energies();    // src/System/System.cpp:9-23
    void calculate_forces();      // src/System/System.cpp:25-39
    void set_coordinates(const std::vector<double>& xyz);   // positions changed by the caller

    const std::vector<double>& forces() const { return forces_; }
    const mdf_energies& energies() const { return e_; }
    const AmberTopology& get_topology() const { return topology_; }
    mdf_ctx* context() const { return ctx_; }
    int mesh(int d) const { return mesh_[d]; }

    // the reference's energy members, by their names
    double bond_energies() const { return e_.e[MDF_E_BOND]; }
    double angle_energy() const { return e_.e[MDF_E_ANGLE]; }
    double dihedral_energy() const { return e_.e[MDF_E_DIHEDRAL]; }
    double urey_bradley_energy() const { return e_.e[MDF_E_UB]; }
    double improper_energy() const { return e_.e[MDF_E_IMPROPER]; }
    double CMAP_energy() const { return e_.e[MDF_E_CMAP]; }
    double LJ_energy_pairlist() const { return e_.e[MDF_E_VDW]; }
    double EE_energy() const { return e_.e[MDF_E_EE]; }
    double EE_energy_pairlist() const { return e_.e[MDF_E_EE_PAIRLIST]; }
    double EE_energy_pairlist_cutoff() const { return e_.e[MDF_E_EE_CUTOFF]; }
    double EE_energy_pairlist_ewald_direct() const { return e_.e[MDF_E_EE_DIRECT]; }
    double EE_energy_pairlist_ewald_self() const { return e_.e[MDF_E_EE_SELF]; }

private:
    void check(int rc) const;

    AmberTopology topology_;
    FlatTopology flat_;
    int semantics_, precision_, device_;
    double box_[3] = {0, 0, 0};
    double cutoff_ = 10.0, skin_ = 2.0, switch_ = 9.0, tol_ = 1e-6;
    int grid_[3] = {0, 0, 0}, mesh_[3] = {0, 0, 0};
    mdf_ctx* ctx_ = nullptr;
    std::vector<double> forces_;
    mdf_energies e_{};
};

}  // namespace mdb200
