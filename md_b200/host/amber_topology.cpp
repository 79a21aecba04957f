// Amber prmtop / rst7 reader and flattening (see amber_topology.hpp).
#include "amber_topology.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>

namespace mdb200 {

namespace {

// The whole file in memory (NUL-terminated) and, per %FLAG name, the byte
// range of its body.  Numbers are parsed in place: no per-line strings, no
// stream objects (a 960,000-atom prmtop is ~100 MB).
struct Sections {
    std::string buf;
    std::map<std::string, std::pair<size_t, size_t>> range;   // [begin, end) of the body
    bool has(const std::string& name) const { return range.count(name) != 0; }
};

std::string slurp(const std::string& path, const char* what)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error(std::string("cannot open ") + what + " " + path);
    std::string buf;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (n > 0) {
        buf.resize((size_t)n);
        if (std::fread(&buf[0], 1, (size_t)n, f) != (size_t)n) {
            std::fclose(f);
            throw std::runtime_error(std::string("cannot read ") + what + " " + path);
        }
    }
    std::fclose(f);
    return buf;   // std::string keeps a NUL after the last byte
}

Sections read_sections(const std::string& path)
{
    Sections s;
    s.buf = slurp(path, "prmtop");
    const char* d = s.buf.data();
    const size_t n = s.buf.size();
    std::string cur;
    size_t pos = 0;
    while (pos < n) {
        const char* nl = static_cast<const char*>(std::memchr(d + pos, '\n', n - pos));
        const size_t end = nl ? (size_t)(nl - d) : n;
        if (end - pos >= 5 && std::strncmp(d + pos, "%FLAG", 5) == 0) {
            if (!cur.empty()) s.range[cur].second = pos;
            size_t p = pos + 5;
            while (p < end && (d[p] == ' ' || d[p] == '\t')) ++p;
            size_t q = p;
            while (q < end && d[q] != ' ' && d[q] != '\t' && d[q] != '\r') ++q;
            cur.assign(d + p, q - p);
            s.range[cur] = {end < n ? end + 1 : n, n};
        }
        pos = end + 1;
    }
    if (!cur.empty()) s.range[cur].second = n;
    return s;
}

// Calls fn(token_start) for every whitespace-separated token of the section's
// body, skipping its %FORMAT / %COMMENT lines.  Returns false if the section
// is absent.
template <typename Fn>
bool for_each_token(const Sections& s, const std::string& name, Fn&& fn)
{
    auto it = s.range.find(name);
    if (it == s.range.end()) return false;
    const char* d = s.buf.data();
    size_t p = it->second.first;
    const size_t e = it->second.second;
    bool line_start = true;
    while (p < e) {
        const char c = d[p];
        if (c == '\n') {
            line_start = true;
            ++p;
            continue;
        }
        if (line_start && c == '%') {   // %FORMAT / %COMMENT line
            while (p < e && d[p] != '\n') ++p;
            continue;
        }
        line_start = false;
        if (c == ' ' || c == '\t' || c == '\r') {
            ++p;
            continue;
        }
        const size_t next = fn(d + p);
        p += next;
    }
    return true;
}

template <typename T>
std::vector<T> numbers(const Sections& s, const std::string& name, bool required = true)
{
    std::vector<T> v;
    const bool found = for_each_token(s, name, [&](const char* tok) -> size_t {
        char* end = nullptr;
        const double x = std::strtod(tok, &end);
        if (end == tok) {
            size_t k = 0;
            while (tok[k] && tok[k] != ' ' && tok[k] != '\n') ++k;
            throw std::runtime_error("bad number '" + std::string(tok, k) + "' in " + name);
        }
        v.push_back(static_cast<T>(x));
        return (size_t)(end - tok);
    });
    if (!found && required) throw std::runtime_error("prmtop section missing: " + name);
    return v;
}

// First line of a text section (the title).
std::string first_line(const Sections& s, const std::string& name)
{
    auto it = s.range.find(name);
    if (it == s.range.end()) return "";
    const char* d = s.buf.data();
    size_t p = it->second.first;
    const size_t e = it->second.second;
    while (p < e) {
        const char* nl = static_cast<const char*>(std::memchr(d + p, '\n', e - p));
        const size_t end = nl ? (size_t)(nl - d) : e;
        if (d[p] != '%') return std::string(d + p, end - p);
        p = end + 1;
    }
    return "";
}

void require(bool ok, const std::string& what)
{
    if (!ok) throw std::runtime_error("prmtop: " + what);
}

}  // namespace

AmberTopology AmberTopology::read(const std::string& prmtop, const std::string& rst7)
{
    const Sections s = read_sections(prmtop);
    AmberTopology t;
    t.title = first_line(s, "TITLE");
    const auto ptr = numbers<long long>(s, "POINTERS");
    require(ptr.size() >= 2, "POINTERS too short");
    t.natoms = (int)ptr[0];
    t.ntypes = (int)ptr[1];
    const int N = t.natoms;
    // long double divide, as the reference does (TopologyParser.cpp:49-52)
    for_each_token(s, "CHARGE", [&](const char* tok) -> size_t {
        char* end = nullptr;
        const long double v = std::strtold(tok, &end);
        if (end == tok) throw std::runtime_error("bad number in CHARGE");
        t.charge.push_back((double)(v / 18.2206899283247L));
        return (size_t)(end - tok);
    });
    t.mass = numbers<double>(s, "MASS");
    for (int ty : numbers<int>(s, "ATOM_TYPE_INDEX")) t.type.push_back(ty - 1);
    t.nb_index = numbers<int>(s, "NONBONDED_PARM_INDEX");
    require((int)t.charge.size() == N && (int)t.mass.size() == N && (int)t.type.size() == N, "per-atom arrays");
    require((int)t.nb_index.size() == t.ntypes * t.ntypes, "NONBONDED_PARM_INDEX size");
    t.lj_a = numbers<double>(s, "LENNARD_JONES_ACOEF");
    t.lj_b = numbers<double>(s, "LENNARD_JONES_BCOEF");
    t.lj14_a = numbers<double>(s, "LENNARD_JONES_14_ACOEF", false);
    t.lj14_b = numbers<double>(s, "LENNARD_JONES_14_BCOEF", false);
    if (t.lj14_a.empty()) {
        t.lj14_a = t.lj_a;
        t.lj14_b = t.lj_b;
    }
    t.bond_k = numbers<double>(s, "BOND_FORCE_CONSTANT");
    t.bond_r0 = numbers<double>(s, "BOND_EQUIL_VALUE");
    t.angle_k = numbers<double>(s, "ANGLE_FORCE_CONSTANT");
    t.angle_t0 = numbers<double>(s, "ANGLE_EQUIL_VALUE");
    t.dih_k = numbers<double>(s, "DIHEDRAL_FORCE_CONSTANT");
    t.dih_n = numbers<double>(s, "DIHEDRAL_PERIODICITY");
    t.dih_phase = numbers<double>(s, "DIHEDRAL_PHASE");
    t.scee = numbers<double>(s, "SCEE_SCALE_FACTOR", false);
    t.scnb = numbers<double>(s, "SCNB_SCALE_FACTOR", false);
    if (t.scee.empty()) t.scee.assign(t.dih_k.size(), 1.2);
    if (t.scnb.empty()) t.scnb.assign(t.dih_k.size(), 2.0);
    t.ub_k = numbers<double>(s, "CHARMM_UREY_BRADLEY_FORCE_CONSTANT", false);
    t.ub_r0 = numbers<double>(s, "CHARMM_UREY_BRADLEY_EQUIL_VALUE", false);
    t.imp_k = numbers<double>(s, "CHARMM_IMPROPER_FORCE_CONSTANT", false);
    t.imp_phase = numbers<double>(s, "CHARMM_IMPROPER_PHASE", false);

    // bonds / angles / dihedrals: coordinate indices (3 * atom), 1-based types
    for (const char* name : {"BONDS_INC_HYDROGEN", "BONDS_WITHOUT_HYDROGEN"}) {
        const auto v = numbers<int>(s, name);
        require(v.size() % 3 == 0, std::string(name) + " length");
        for (size_t k = 0; k < v.size(); k += 3) {
            t.bonds.push_back(v[k] / 3);
            t.bonds.push_back(v[k + 1] / 3);
            t.bonds.push_back(v[k + 2] - 1);
        }
        t.nbonds_part.push_back((int)(v.size() / 3));
    }
    for (const char* name : {"ANGLES_INC_HYDROGEN", "ANGLES_WITHOUT_HYDROGEN"}) {
        const auto v = numbers<int>(s, name);
        require(v.size() % 4 == 0, std::string(name) + " length");
        for (size_t k = 0; k < v.size(); k += 4) {
            for (int a = 0; a < 3; ++a) t.angles.push_back(v[k + a] / 3);
            t.angles.push_back(v[k + 3] - 1);
        }
        t.nangles_part.push_back((int)(v.size() / 4));
    }
    for (const char* name : {"DIHEDRALS_INC_HYDROGEN", "DIHEDRALS_WITHOUT_HYDROGEN"}) {
        const auto v = numbers<int>(s, name);
        require(v.size() % 5 == 0, std::string(name) + " length");
        for (size_t k = 0; k < v.size(); k += 5) {
            t.dihedrals.push_back(std::abs(v[k]) / 3);
            t.dihedrals.push_back(std::abs(v[k + 1]) / 3);
            t.dihedrals.push_back(std::abs(v[k + 2]) / 3);
            t.dihedrals.push_back(std::abs(v[k + 3]) / 3);
            t.dihedrals.push_back(v[k + 4] - 1);
            t.dihedrals.push_back(v[k + 2] < 0 ? 1 : 0);   // no 1-4 interaction
            t.dihedrals.push_back(v[k + 3] < 0 ? 1 : 0);   // improper (Amber style)
        }
        t.ndih_part.push_back((int)(v.size() / 5));
    }
    {
        const auto v = numbers<int>(s, "CHARMM_UREY_BRADLEY", false);
        for (size_t k = 0; k + 2 < v.size(); k += 3) {
            t.ub.push_back(v[k] - 1);
            t.ub.push_back(v[k + 1] - 1);
            t.ub.push_back(v[k + 2] - 1);
        }
    }
    {
        const auto v = numbers<int>(s, "CHARMM_IMPROPERS", false);
        for (size_t k = 0; k + 4 < v.size(); k += 5)
            for (int a = 0; a < 5; ++a) t.impropers.push_back(v[k + a] - 1);
    }
    {
        const auto cnt = numbers<int>(s, "CHARMM_CMAP_COUNT", false);
        const auto res = numbers<int>(s, "CHARMM_CMAP_RESOLUTION", false);
        const int nsets = cnt.size() >= 2 ? cnt[1] : 0;
        if (!res.empty()) t.cmap_res = res[0];
        for (int k = 0; k < nsets; ++k) {
            char nm[64];
            std::snprintf(nm, sizeof(nm), "CHARMM_CMAP_PARAMETER_%02d", k + 1);
            auto g = numbers<double>(s, nm);
            require((int)g.size() == t.cmap_res * t.cmap_res, std::string(nm) + " size");
            t.cmap_grids.push_back(std::move(g));
        }
        const auto v = numbers<int>(s, "CHARMM_CMAP_INDEX", false);
        for (size_t k = 0; k + 5 < v.size(); k += 6) {
            for (int a = 0; a < 5; ++a) t.cmaps.push_back(v[k + a] - 1);
            t.cmaps.push_back(v[k + 5] - 1);
        }
    }
    {
        const auto nex = numbers<int>(s, "NUMBER_EXCLUDED_ATOMS");
        const auto lst = numbers<int>(s, "EXCLUDED_ATOMS_LIST");
        require((int)nex.size() == N, "NUMBER_EXCLUDED_ATOMS size");
        t.excluded.assign(N, {});
        size_t p = 0;
        for (int i = 0; i < N; ++i)
            for (int k = 0; k < nex[i]; ++k, ++p) {
                require(p < lst.size(), "EXCLUDED_ATOMS_LIST too short");
                if (lst[p] > 0) t.excluded[i].push_back(lst[p] - 1);
            }
    }
    {
        const auto b = numbers<double>(s, "BOX_DIMENSIONS", false);
        if (b.size() >= 4)
            for (int d = 0; d < 3; ++d) t.box[d] = b[1 + d];
    }
    if (!rst7.empty()) t.read_coordinates(rst7);
    return t;
}

// ASCII restart: title, natoms (and time), 3N coordinates in 12-character
// fields six per line, then (velocities and) the box line.
void AmberTopology::read_coordinates(const std::string& path)
{
    const std::string buf = slurp(path, "coordinates");
    const char* d = buf.data();
    const size_t nb = buf.size();
    auto line_end = [&](size_t p) {
        const char* nl = static_cast<const char*>(std::memchr(d + p, '\n', nb - p));
        return nl ? (size_t)(nl - d) : nb;
    };
    size_t p = line_end(0) + 1;   // title
    if (p > nb) throw std::runtime_error("rst7 too short");
    const size_t e2 = line_end(p);
    const int n = std::atoi(std::string(d + p, e2 - p).c_str());
    if (n != natoms) throw std::runtime_error("rst7 atom count differs from the prmtop");
    std::vector<double> vals;
    vals.reserve(3 * (size_t)n + 6);
    p = e2 + 1;
    while (p < nb) {
        size_t e = line_end(p);
        if (e > p && d[e - 1] == '\r') --e;
        // fixed 12-character fields
        for (size_t q = p; q < e; q += 12) {
            char fld[13];
            const size_t w = std::min<size_t>(12, e - q);
            std::memcpy(fld, d + q, w);
            fld[w] = 0;
            size_t k = 0;
            while (k < w && fld[k] == ' ') ++k;
            if (k == w) continue;
            vals.push_back(std::strtod(fld, nullptr));
        }
        p = line_end(p) + 1;
    }
    if (vals.size() < 3 * (size_t)n) throw std::runtime_error("rst7 has too few coordinates");
    coords.assign(vals.begin(), vals.begin() + 3 * (size_t)n);
    // box: the last line's first three fields when the file carries one
    const size_t rest = vals.size() - 3 * (size_t)n;
    if (rest == 6 || rest == 3 * (size_t)n + 6)
        for (int d = 0; d < 3; ++d) box[d] = vals[vals.size() - 6 + d];
}

mdf_topology FlatTopology::view() const
{
    mdf_topology t{};
    t.natoms = (int32_t)charge.size();
    t.charge = charge.data();
    t.type = type.data();
    t.ntypes = ntypes;
    t.nb_index = nb_index.data();
    t.n_ljpair = (int32_t)lj_a.size();
    t.lj_a = lj_a.data(); t.lj_b = lj_b.data(); t.lj14_a = lj14_a.data(); t.lj14_b = lj14_b.data();
    t.n_bonds = (int32_t)bond_k.size(); t.bond_atoms = bond_atoms.data(); t.bond_k = bond_k.data();
    t.bond_r0 = bond_r0.data();
    t.n_ub = (int32_t)ub_k.size(); t.ub_atoms = ub_atoms.data(); t.ub_k = ub_k.data(); t.ub_r0 = ub_r0.data();
    t.n_angles = (int32_t)angle_k.size(); t.angle_atoms = angle_atoms.data(); t.angle_k = angle_k.data();
    t.angle_theta0 = angle_theta0.data();
    t.n_dihedrals = (int32_t)dihedral_k.size(); t.dihedral_atoms = dihedral_atoms.data();
    t.dihedral_k = dihedral_k.data(); t.dihedral_n = dihedral_n.data(); t.dihedral_phase = dihedral_phase.data();
    t.n_impropers = (int32_t)improper_k.size(); t.improper_atoms = improper_atoms.data();
    t.improper_k = improper_k.data(); t.improper_phase = improper_phase.data();
    t.n_cmaps = (int32_t)cmap_set.size(); t.cmap_atoms = cmap_atoms.data(); t.cmap_set = cmap_set.data();
    t.cmap_nsets = cmap_nsets; t.cmap_res = cmap_res; t.cmap_coeff = cmap_coeff.data();
    t.n_excl = (int32_t)(excl_pairs.size() / 2); t.excl_pairs = excl_pairs.data();
    t.n_pairs14 = (int32_t)scee14.size(); t.pairs14 = pairs14.data();
    t.scee14 = scee14.data(); t.scnb14 = scnb14.data();
    return t;
}

FlatTopology flatten(const AmberTopology& t, int semantics)
{
    const bool ref = semantics == MDF_SEM_REFERENCE;
    FlatTopology o;
    o.charge = t.charge;
    o.type.assign(t.type.begin(), t.type.end());
    o.ntypes = t.ntypes;
    o.nb_index.assign(t.nb_index.begin(), t.nb_index.end());
    o.lj_a = t.lj_a; o.lj_b = t.lj_b; o.lj14_a = t.lj14_a; o.lj14_b = t.lj14_b;

    // REFERENCE: each loader drops its list's last tuple (per list: the
    // hydrogen and non-hydrogen lists separately)
    auto keep = [&](int count) { return ref && count > 0 ? count - 1 : count; };
    {
        size_t base = 0;
        for (int part : t.nbonds_part) {
            for (int k = 0; k < keep(part); ++k) {
                const int* b = &t.bonds[3 * (base + k)];
                o.bond_atoms.push_back(b[0]); o.bond_atoms.push_back(b[1]);
                o.bond_k.push_back(t.bond_k.at(b[2])); o.bond_r0.push_back(t.bond_r0.at(b[2]));
            }
            base += part;
        }
    }
    {
        size_t base = 0;
        for (int part : t.nangles_part) {
            for (int k = 0; k < keep(part); ++k) {
                const int* a = &t.angles[4 * (base + k)];
                for (int q = 0; q < 3; ++q) o.angle_atoms.push_back(a[q]);
                o.angle_k.push_back(t.angle_k.at(a[3])); o.angle_theta0.push_back(t.angle_t0.at(a[3]));
            }
            base += part;
        }
    }
    std::vector<const int*> dkept;
    {
        size_t base = 0;
        for (int part : t.ndih_part) {
            for (int k = 0; k < keep(part); ++k) {
                const int* d = &t.dihedrals[7 * (base + k)];
                dkept.push_back(d);
                for (int q = 0; q < 4; ++q) o.dihedral_atoms.push_back(d[q]);
                o.dihedral_k.push_back(t.dih_k.at(d[4]));
                o.dihedral_n.push_back(t.dih_n.at(d[4]));
                o.dihedral_phase.push_back(t.dih_phase.at(d[4]));
            }
            base += part;
        }
    }
    const int nub = (int)(t.ub.size() / 3);
    for (int k = 0; k < keep(nub); ++k) {
        o.ub_atoms.push_back(t.ub[3 * k]); o.ub_atoms.push_back(t.ub[3 * k + 1]);
        o.ub_k.push_back(t.ub_k.at(t.ub[3 * k + 2])); o.ub_r0.push_back(t.ub_r0.at(t.ub[3 * k + 2]));
    }
    const int nimp = (int)(t.impropers.size() / 5);
    for (int k = 0; k < nimp; ++k) {   // the improper loader keeps every tuple
        for (int q = 0; q < 4; ++q) o.improper_atoms.push_back(t.impropers[5 * k + q]);
        o.improper_k.push_back(t.imp_k.at(t.impropers[5 * k + 4]));
        o.improper_phase.push_back(t.imp_phase.at(t.impropers[5 * k + 4]));
    }
    const int ncm = (int)(t.cmaps.size() / 6);
    for (int k = 0; k < keep(ncm); ++k) {
        for (int q = 0; q < 5; ++q) o.cmap_atoms.push_back(t.cmaps[6 * k + q]);
        o.cmap_set.push_back(t.cmaps[6 * k + 5]);
    }
    o.cmap_nsets = (int)t.cmap_grids.size();
    o.cmap_res = t.cmap_res;
    {
        std::vector<double> grids;
        for (const auto& g : t.cmap_grids) grids.insert(grids.end(), g.begin(), g.end());
        o.cmap_coeff.assign((size_t)o.cmap_nsets * o.cmap_res * o.cmap_res * 16, 0.0);
        if (o.cmap_nsets > 0) {
            const int rc = ref ? mdf_cmap_coefficients(o.cmap_nsets, o.cmap_res, grids.data(), o.cmap_coeff.data())
                               : mdf_cmap_coefficients_spline(o.cmap_nsets, o.cmap_res, grids.data(),
                                                              o.cmap_coeff.data());
            if (rc != MDF_OK) throw std::runtime_error("CMAP coefficient table failed");
        }
    }
    if (!ref) {
        // pairs as sorted 64-bit keys (min << 32 | max): the order of a set of
        // pairs, built with one sort instead of a tree insert per pair
        auto key = [](int a, int b) {
            return ((unsigned long long)(unsigned)std::min(a, b) << 32) | (unsigned)std::max(a, b);
        };
        auto sort_unique = [](std::vector<unsigned long long>& v) {
            std::sort(v.begin(), v.end());
            v.erase(std::unique(v.begin(), v.end()), v.end());
        };
        std::vector<unsigned long long> ex, near;
        for (int i = 0; i < t.natoms; ++i)
            for (int j : t.excluded[i]) ex.push_back(key(i, j));
        for (size_t k = 0; k < o.bond_atoms.size(); k += 2) near.push_back(key(o.bond_atoms[k], o.bond_atoms[k + 1]));
        for (size_t k = 0; k < o.angle_atoms.size(); k += 3) near.push_back(key(o.angle_atoms[k], o.angle_atoms[k + 2]));
        sort_unique(near);
        // 1-4 pairs with the largest SCEE / SCNB over the dihedrals that generate them
        std::vector<std::pair<unsigned long long, std::pair<double, double>>> cand;
        for (const int* d : dkept) {
            if (d[5] || d[6]) continue;
            const auto kk = key(d[0], d[3]);
            if (std::binary_search(near.begin(), near.end(), kk)) continue;
            cand.push_back({kk, {t.scee.at(d[4]), t.scnb.at(d[4])}});
        }
        std::sort(cand.begin(), cand.end(),
                  [](const auto& x, const auto& y) { return x.first < y.first; });
        std::vector<std::pair<unsigned long long, std::pair<double, double>>> p14;
        for (const auto& c : cand) {
            if (!p14.empty() && p14.back().first == c.first)
                p14.back().second = {std::max(p14.back().second.first, c.second.first),
                                     std::max(p14.back().second.second, c.second.second)};
            else
                p14.push_back(c);
        }
        for (const auto& kv : p14) ex.push_back(kv.first);
        sort_unique(ex);
        o.excl_pairs.reserve(2 * ex.size());
        for (unsigned long long e : ex) {
            o.excl_pairs.push_back((int)(e >> 32));
            o.excl_pairs.push_back((int)(e & 0xffffffffu));
        }
        for (const auto& kv : p14) {
            o.pairs14.push_back((int)(kv.first >> 32));
            o.pairs14.push_back((int)(kv.first & 0xffffffffu));
            o.scee14.push_back(kv.second.first);
            o.scnb14.push_back(kv.second.second);
        }
    }
    return o;
}

}  // namespace mdb200
