// MdfBackend.cpp — the reference's System::calculate_energies() and
// System::calculate_forces() evaluated by libmdf on the GPU.
//
// This is the file a maintainer of prateekbansal97/MD adds as
// src/System/MdfBackend.cpp and compiles INSTEAD of src/System/System.cpp
// (which holds only those two members, src/System/System.cpp:9-39) in the
// reserved ENABLE_CUDA slot (CMakeLists.txt:140-160), linking libmdf.so.
// Nothing else in the reference changes: System::init() and every caller
// keep calling the same private members, which now read the reference's own
// parsed state (topology_, q_, type_, nb_flat_, the term lists, the box and
// the cutoffs) and write forces_ and the energy members
// (include/System/System.h:176-188) from the device evaluation.
//
// In this repository it is test infrastructure: oracle/Makefile compiles it
// with the unmodified reference sources into oracle/_ref/ref_on_mdf, and a
// GPU test checks that the reference's own System, running on libmdf,
// reproduces the reference's CPU numbers (golden fixtures).
//
// Semantics are the reference's as it runs (MDF_SEM_REFERENCE): the term
// lists are whatever its loaders produced, its exclusion lists (per atom,
// Atom::get_excluded_atoms) are passed through as they are, and its pairlist
// rebuild rule (System::ljpairs_needs_rebuild, src/System/NonBondedUtils.cpp:
// 87-100) decides when the device list is rebuilt.  The environment variable
// MD_MDF_PRECISION=mixed selects libmdf's mixed-precision path (FP64 by
// default); MD_MDF_DEVICE picks the CUDA device (default 0).
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "System/System.h"
#include "mdf.h"

namespace md
{
namespace
{
struct MdfState {
    mdf_ctx* ctx = nullptr;   // mdf_create copied the topology; nothing else is kept
};

// One libmdf context per System object (System has no member for it; the
// reference's header is left untouched).
std::map<const System*, MdfState>& registry()
{
    static std::map<const System*, MdfState> r;
    return r;
}

void check(int rc, const mdf_ctx* ctx, const char* what)
{
    if (rc != MDF_OK)
        throw std::runtime_error(std::string("libmdf ") + what + ": " + mdf_status_string(rc) + ": " +
                                 mdf_last_error(ctx));
}

int env_int(const char* name, int def)
{
    const char* v = std::getenv(name);
    return v && *v ? std::atoi(v) : def;
}
}  // namespace

// The first evaluation of a System builds its device context from the
// System's private state (so it happens inside a member); later calls upload
// the current coordinates and rebuild the device pairlist when the
// reference's own rule asks for it.
void System::calculate_energies()
{
    bool fresh = false;
    mdf_ctx* ctx = nullptr;
    {
        auto& st = registry()[this];
        if (!st.ctx) {
            // ---- flatten the reference's parsed topology into mdf_topology
            std::vector<int32_t> type32(type_.begin(), type_.end());
            std::vector<int32_t> nb32(nb_flat_.begin(), nb_flat_.end());
            auto& tp = topology_;
            std::vector<int32_t> bond_atoms, ub_atoms, angle_atoms, dih_atoms, imp_atoms, cmap_atoms, cmap_set;
            std::vector<double> bond_k, bond_r0, ub_k, ub_r0, angle_k, angle_t0, dih_k, dih_n, dih_ph, imp_k, imp_ph;
            for (const auto& b : tp.get_harmonic_bonds()) {
                bond_atoms.push_back(b.get_atomA_index());
                bond_atoms.push_back(b.get_atomB_index());
                bond_k.push_back(b.get_Bond_force_constant());
                bond_r0.push_back(b.get_Bond_equil_length());
            }
            for (const auto& u : tp.get_harmonic_UBs()) {
                ub_atoms.push_back(u.get_atomA_index());
                ub_atoms.push_back(u.get_atomB_index());
                ub_k.push_back(u.get_UB_force_constant());
                ub_r0.push_back(u.get_UB_equil_value());
            }
            for (const auto& a : tp.get_harmonic_angles()) {
                angle_atoms.push_back(a.get_atomA_index());
                angle_atoms.push_back(a.get_atomB_index());
                angle_atoms.push_back(a.get_atomC_index());
                angle_k.push_back(a.get_Angle_force_constant());
                angle_t0.push_back(a.get_Angle_equil_angle());
            }
            for (const auto& d : tp.get_cosine_dihedrals()) {
                dih_atoms.push_back(d.get_atomA_index());
                dih_atoms.push_back(d.get_atomB_index());
                dih_atoms.push_back(d.get_atomC_index());
                dih_atoms.push_back(d.get_atomD_index());
                dih_k.push_back(d.get_Dihedral_force_constant());
                dih_n.push_back(d.get_Dihedral_Periodicity());
                dih_ph.push_back(d.get_Dihedral_phase());
            }
            for (const auto& m : tp.get_harmonic_impropers()) {
                imp_atoms.push_back(m.get_atomA_index());
                imp_atoms.push_back(m.get_atomB_index());
                imp_atoms.push_back(m.get_atomC_index());
                imp_atoms.push_back(m.get_atomD_index());
                imp_k.push_back(m.get_IMP_force_constant());
                imp_ph.push_back(m.get_IMP_phase_value());
            }
            for (const auto& c : tp.get_cmaps()) {
                const int idx[5] = {c.get_atomA_index(), c.get_atomB_index(), c.get_atomC_index(),
                                    c.get_atomD_index(), c.get_atomE_index()};
                cmap_atoms.insert(cmap_atoms.end(), idx, idx + 5);
                cmap_set.push_back(c.get_parameter_set() - 1);   // the reference's sets are 1-based
            }
            // CMAP tables: the reference's bicubic patches from its grids
            // (src/AmberTopology/CreateNonBondedFromParsed.cpp:46-117)
            const auto& res = tp.get_charmm_cmap_resolutions();
            const int nsets = (int)res.size(), cres = nsets ? res[0] : 24;
            std::vector<double> grids, coeff;
            if (!tp.get_cmaps().empty()) {
                for (int k = 1; k <= nsets; ++k) {
                    const auto& g = tp.get_cmap_grid_data(k);
                    grids.insert(grids.end(), g.begin(), g.end());
                }
                coeff.assign((size_t)nsets * cres * cres * 16, 0.0);
                check(mdf_cmap_coefficients(nsets, cres, grids.data(), coeff.data()), nullptr, "CMAP table");
            }
            // exclusions as the reference holds them (per atom)
            std::vector<int32_t> excl;
            auto& atoms = tp.get_atom_list();
            for (size_t i = 0; i < atoms.size(); ++i)
                for (int j : atoms[i].get_excluded_atoms())
                    if (j > (int)i && j < (int)atoms.size()) {
                        excl.push_back((int32_t)i);
                        excl.push_back(j);
                    }

            mdf_topology t;
            std::memset(&t, 0, sizeof(t));
            t.natoms = (int32_t)q_.size();
            t.charge = q_.data();
            t.type = type32.data();
            t.ntypes = nTypes_;
            t.nb_index = nb32.data();
            t.n_ljpair = (int32_t)tp.get_lennard_jones_Acoefs_().size();
            t.lj_a = tp.get_lennard_jones_Acoefs_().data();
            t.lj_b = tp.get_lennard_jones_Bcoefs_().data();
            const bool have14 = tp.get_lennard_jones_14_Acoefs_().size() == (size_t)t.n_ljpair;
            t.lj14_a = have14 ? tp.get_lennard_jones_14_Acoefs_().data() : nullptr;
            t.lj14_b = have14 ? tp.get_lennard_jones_14_Bcoefs_().data() : nullptr;
            t.n_bonds = (int32_t)bond_k.size();
            t.bond_atoms = bond_atoms.data(); t.bond_k = bond_k.data(); t.bond_r0 = bond_r0.data();
            t.n_ub = (int32_t)ub_k.size();
            t.ub_atoms = ub_atoms.data(); t.ub_k = ub_k.data(); t.ub_r0 = ub_r0.data();
            t.n_angles = (int32_t)angle_k.size();
            t.angle_atoms = angle_atoms.data(); t.angle_k = angle_k.data(); t.angle_theta0 = angle_t0.data();
            t.n_dihedrals = (int32_t)dih_k.size();
            t.dihedral_atoms = dih_atoms.data(); t.dihedral_k = dih_k.data(); t.dihedral_n = dih_n.data();
            t.dihedral_phase = dih_ph.data();
            t.n_impropers = (int32_t)imp_k.size();
            t.improper_atoms = imp_atoms.data(); t.improper_k = imp_k.data(); t.improper_phase = imp_ph.data();
            t.n_cmaps = (int32_t)cmap_set.size();
            t.cmap_atoms = cmap_atoms.data(); t.cmap_set = cmap_set.data();
            t.cmap_nsets = nsets; t.cmap_res = cres; t.cmap_coeff = coeff.empty() ? nullptr : coeff.data();
            t.n_excl = (int32_t)(excl.size() / 2);
            t.excl_pairs = excl.data();

            // ---- run parameters: the System's own settings
            mdf_params p;
            mdf_params_default(&p);
            p.semantics = MDF_SEM_REFERENCE;
            const char* prec = std::getenv("MD_MDF_PRECISION");
            p.precision = (prec && !std::strcmp(prec, "mixed")) ? MDF_PREC_MIXED : MDF_PREC_FP64;
            p.device = env_int("MD_MDF_DEVICE", 0);
            p.box[0] = boxLx_; p.box[1] = boxLy_; p.box[2] = boxLz_;
            p.cutoff = lj_cutoff_;
            p.skin = lj_skin_;
            p.switch_radius = lj_use_switch_ ? lj_switch_ : 0.0;
            p.ewald_tol = ewald_error_tolerance_;
            p.ewald_alpha = ewald_alpha_;           // set by calculate_ewald_alpha() (0: libmdf uses the same formula)
            p.grid[0] = newald_mesh_x; p.grid[1] = newald_mesh_y; p.grid[2] = newald_mesh_z;
            check(mdf_create(&t, &p, &st.ctx), nullptr, "mdf_create");
            check(mdf_set_positions(st.ctx, topology_.get_coordinates().data()), st.ctx, "positions");
            check(mdf_build_pairlist(st.ctx), st.ctx, "pairlist");
            copy_ref_coords_lj();   // the reference's rebuild reference point
            fresh = true;
        }
        ctx = st.ctx;
    }
    if (!fresh) {
        check(mdf_set_positions(ctx, topology_.get_coordinates().data()), ctx, "positions");
        if (ljpairs_needs_rebuild()) {
            check(mdf_build_pairlist(ctx), ctx, "pairlist");
            copy_ref_coords_lj();
        }
    }
    mdf_energies e;
    check(mdf_compute(ctx, MDF_COMPUTE_ENERGY, nullptr, &e), ctx, "energies");
    bond_energies_ = e.e[MDF_E_BOND];
    angle_energy_ = e.e[MDF_E_ANGLE];
    dihedral_energy_ = e.e[MDF_E_DIHEDRAL];
    urey_bradley_energy_ = e.e[MDF_E_UB];
    improper_energy_ = e.e[MDF_E_IMPROPER];
    CMAP_energy_ = e.e[MDF_E_CMAP];
    LJ_energy_pairlist_ = e.e[MDF_E_VDW];
    EE_energy_ = e.e[MDF_E_EE];
    EE_energy_pairlist_ = e.e[MDF_E_EE_PAIRLIST];
    EE_energy_pairlist_cutoff_ = e.e[MDF_E_EE_CUTOFF];
    EE_energy_pairlist_ewald_direct_ = e.e[MDF_E_EE_DIRECT];
    EE_energy_pairlist_ewald_self_ = e.e[MDF_E_EE_SELF];
}

void System::calculate_forces()
{
    auto& st = registry()[this];
    if (!st.ctx) {
        // first evaluation of this System: the energy member sets the context up
        calculate_energies();
    } else {
        check(mdf_set_positions(st.ctx, topology_.get_coordinates().data()), st.ctx, "positions");
        if (ljpairs_needs_rebuild()) {
            check(mdf_build_pairlist(st.ctx), st.ctx, "pairlist");
            copy_ref_coords_lj();
        }
    }
    // clear_forces() + every calculate_forces_* member: forces_ is overwritten
    check(mdf_compute(st.ctx, MDF_COMPUTE_FORCES, forces_.data(), nullptr), st.ctx, "forces");
}

// Releases the context of a System that is going away (call from ~System in a
// build that owns the registry's lifetime; process exit releases it too).
void mdf_release(const System* s)
{
    auto it = registry().find(s);
    if (it == registry().end()) return;
    mdf_destroy(it->second.ctx);
    registry().erase(it);
}
}  // namespace md
