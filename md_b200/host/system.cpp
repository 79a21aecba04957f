// mdb200::System on libmdf (see system.hpp).
#include "system.hpp"

#include <cmath>
#include <stdexcept>
#include <utility>

namespace mdb200 {

System::System(AmberTopology topology, int semantics, int precision, int device)
    : topology_(std::move(topology)), semantics_(semantics), precision_(precision), device_(device)
{
    for (int d = 0; d < 3; ++d) box_[d] = topology_.box[d];
    forces_.assign(3 * (size_t)topology_.natoms, 0.0);
}

System::~System()
{
    if (ctx_) mdf_destroy(ctx_);
}

void System::check(int rc) const
{
    if (rc != MDF_OK) throw std::runtime_error(std::string("libmdf: ") + mdf_status_string(rc) + ": " +
                                               mdf_last_error(ctx_));
}

void System::set_box(double Lx, double Ly, double Lz)
{
    box_[0] = Lx; box_[1] = Ly; box_[2] = Lz;
    if (ctx_) check(mdf_set_box(ctx_, box_));
}

void System::init()
{
    if (topology_.coords.size() != 3 * (size_t)topology_.natoms)
        throw std::runtime_error("no coordinates: read the topology with an rst7");
    flat_ = flatten(topology_, semantics_);
    mdf_params p;
    mdf_params_default(&p);
    p.semantics = semantics_;
    p.precision = precision_;
    p.device = device_;
    for (int d = 0; d < 3; ++d) {
        p.box[d] = box_[d];
        p.grid[d] = grid_[d];
    }
    p.cutoff = cutoff_;
    p.skin = skin_;
    p.switch_radius = switch_;
    p.ewald_tol = tol_;
    // the reference's mesh formula (src/System/PBC.cpp:93-99) when none is set
    const double alpha = std::sqrt(-std::log(2.0 * tol_)) / cutoff_;
    for (int d = 0; d < 3; ++d)
        mesh_[d] = grid_[d] > 0 ? grid_[d] : (int)((2 * alpha * box_[d]) / (3 * std::pow(tol_, 0.2)));
    const mdf_topology t = flat_.view();
    if (ctx_) mdf_destroy(ctx_);
    ctx_ = nullptr;
    const int rc = mdf_create(&t, &p, &ctx_);
    if (rc != MDF_OK) throw std::runtime_error(std::string("libmdf: ") + mdf_last_error(nullptr));
    check(mdf_set_positions(ctx_, topology_.coords.data()));
    check(mdf_build_pairlist(ctx_));
}

void System::set_coordinates(const std::vector<double>& xyz)
{
    if (xyz.size() != 3 * (size_t)topology_.natoms) throw std::runtime_error("coordinate count");
    topology_.coords = xyz;
    if (ctx_) check(mdf_set_positions(ctx_, topology_.coords.data()));
}

void System::calculate_energies()
{
    if (!ctx_) init();
    check(mdf_compute(ctx_, MDF_COMPUTE_ENERGY, nullptr, &e_));
}

void System::calculate_forces()
{
    if (!ctx_) init();
    check(mdf_compute(ctx_, MDF_COMPUTE_FORCES, forces_.data(), nullptr));
}

}  // namespace mdb200
