// Amber prmtop / rst7 reader and the flattening into mdf_topology.
//
// The host side of the drop-in: the reference reads a prmtop and an rst7
// (AmberTopology::read_topology_coordinates,
// include/AmberTopology/AmberTopology.h:33; src/AmberTopology/AmberTopology.cpp,
// TopologyParser.cpp) and turns the parsed sections into term objects
// (src/AmberTopology/CreateBondedFromParsed.cpp,
// CreateNonBondedFromParsed.cpp).  This reader keeps the same inputs and the
// same post-processing, with the semantics switch:
//   REFERENCE  the reference as it runs: the term loaders stop one tuple early
//              (loop bound i + w < size, CreateBondedFromParsed.cpp:11,74,100,
//              126,152,178,220,262; impropers keep every tuple, :41) and the
//              exclusion lists stay empty (CreateNonBondedFromParsed.cpp:33-36);
//   PHYSICAL   every tuple; exclusions from EXCLUDED_ATOMS_LIST plus the 1-4
//              set of the proper dihedrals without the exclude-1-4 flag, SCEE
//              and SCNB per 1-4 pair the largest over its dihedrals
//              (CreateNonBondedFromParsed.cpp:124-169).
// Numbers are read as whitespace-separated tokens per %FLAG section.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "mdf.h"

namespace mdb200 {

// Internal charge unit of the reference: prmtop charge / 18.2206899283247
// (src/AmberTopology/TopologyParser.cpp:52); the Coulomb constant is its square.
constexpr double kAmberChargeScale = 18.2206899283247;

struct AmberTopology {
    std::string title;
    int natoms = 0, ntypes = 0;
    std::vector<double> charge;        // internal unit
    std::vector<double> mass;          // amu
    std::vector<int> type;             // 0-based
    std::vector<int> nb_index;         // [ntypes^2], 1-based, 0 = none
    std::vector<double> lj_a, lj_b, lj14_a, lj14_b;
    std::vector<double> bond_k, bond_r0, angle_k, angle_t0, ub_k, ub_r0;
    std::vector<double> dih_k, dih_n, dih_phase, scee, scnb, imp_k, imp_phase;
    // tuples, 0-based atoms and types, in file order (hydrogen lists first)
    std::vector<int> bonds;            // 3 per bond: i, j, type (BONDS_INC_HYDROGEN then _WITHOUT_)
    std::vector<int> angles;           // 4 per angle
    std::vector<int> dihedrals;        // 7 per dihedral: i, j, k, l, type, exclude-1-4 flag, improper flag
    std::vector<int> nbonds_part, nangles_part, ndih_part;   // tuple counts of the two lists each
    std::vector<int> ub;               // 3 per term
    std::vector<int> impropers;        // 5 per term: i, j, k, l, type
    std::vector<int> cmaps;            // 6 per term: 5 atoms, set (0-based)
    int cmap_res = 24;
    std::vector<std::vector<double>> cmap_grids;   // [nsets][res*res]
    std::vector<std::vector<int>> excluded;        // per atom, 0-based partners
    double box[3] = {0, 0, 0};
    std::vector<double> coords;        // [3N] from the rst7 (or empty)

    // read_topology_coordinates: prmtop, then the rst7 if a path is given
    static AmberTopology read(const std::string& prmtop, const std::string& rst7 = "");
    void read_coordinates(const std::string& rst7);
};

// Owning flattened topology: the arrays behind one mdf_topology.
struct FlatTopology {
    std::vector<double> charge, lj_a, lj_b, lj14_a, lj14_b;
    std::vector<int32_t> type, nb_index;
    int ntypes = 0;
    std::vector<int32_t> bond_atoms, ub_atoms, angle_atoms, dihedral_atoms, improper_atoms, cmap_atoms, cmap_set;
    std::vector<double> bond_k, bond_r0, ub_k, ub_r0, angle_k, angle_theta0, dihedral_k, dihedral_n,
        dihedral_phase, improper_k, improper_phase, cmap_coeff;
    int cmap_nsets = 0, cmap_res = 24;
    std::vector<int32_t> excl_pairs, pairs14;
    std::vector<double> scee14, scnb14;

    mdf_topology view() const;   // pointers into this object
};

// semantics: MDF_SEM_REFERENCE or MDF_SEM_PHYSICAL.  The CMAP table comes from
// mdf_cmap_coefficients (REFERENCE) or mdf_cmap_coefficients_spline (PHYSICAL).
FlatTopology flatten(const AmberTopology& t, int semantics);

}  // namespace mdb200
