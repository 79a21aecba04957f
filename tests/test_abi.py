"""The C ABI library: it loads without a GPU, exports every function that
include/mdf.h declares, its host-only utilities agree with the oracle, and
it refuses to run (rather than falling back to the CPU) without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from md_b200 import abi, engine
from oracle import oracle as O
from tests import helpers as H

HEADER = os.path.join(H.ROOT, "include", "mdf.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(mdf_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = engine.library()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(engine.EXPORTS) == names


def test_params_default_are_the_reference_init_values():
    p = engine.default_params()
    assert p.cutoff == 10.0 and p.skin == 2.0 and p.switch_radius == 9.0
    assert p.ewald_tol == 1e-6
    assert p.coulomb_const == H.KC
    assert p.semantics == abi.MDF_SEM_REFERENCE


def test_status_strings():
    lib = engine.library()
    for k, v in abi.STATUS.items():
        assert lib.mdf_status_string(k).decode() == v


def test_cmap_coefficients_match_oracle():
    s = H.system("tiny")
    a = engine.cmap_coefficients(5, 24, s.cmap_grids)
    b = O.cmap_coeff(5, 24, s.cmap_grids)
    assert np.array_equal(a, b)


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_create_fails_loudly_without_gpu():
    s = H.system("tiny")
    flat = H.flat(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    with pytest.raises(engine.MDFError) as e:
        engine.Engine(flat, s.box)
    assert e.value.status == 2   # MDF_ERR_CUDA


def test_invalid_topology_rejected_before_device_work():
    # a bad atom index is caught on the host; without a GPU the device check
    # comes first, so accept either status but never success
    s = H.system("tiny")
    flat = H.flat(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    flat.bond_atoms = flat.bond_atoms.copy()
    flat.bond_atoms[0] = 10 ** 6
    flat._struct = None
    with pytest.raises(engine.MDFError) as e:
        engine.Engine(flat, s.box)
    assert e.value.status in (1, 2)


def test_cmap_spline_table_is_c1_and_interpolates():
    """PHYSICAL CMAP table: patches meet with equal value and slope along every
    cell edge (the reference's do not), hit the grid at the corners, and
    interpolate a smooth periodic surface to 1e-3."""
    res = 24
    ph = np.arange(res) * 2 * np.pi / res
    grid = 2 * np.cos(ph)[:, None] * np.sin(2 * ph)[None, :] + np.cos(ph[:, None] + ph[None, :])
    C = engine.cmap_coefficients_spline(1, res, grid.reshape(1, -1)).reshape(res, res, 4, 4)
    R = engine.cmap_coefficients(1, res, grid.reshape(1, -1)).reshape(res, res, 4, 4)
    p = lambda t: np.array([1, t, t * t, t ** 3])
    d = lambda t: np.array([0, 1, 2 * t, 3 * t * t])
    e_ref = e_edge = e_slope = e_corner = e_int = 0.0
    for i in range(res):
        for j in range(res):
            e_corner = max(e_corner, abs(p(0) @ C[i, j] @ p(0) - grid[i, j]))
            for v in (0.0, 0.4, 0.8):
                a, b = C[i, j], C[(i + 1) % res, j]
                e_edge = max(e_edge, abs(p(1) @ a @ p(v) - p(0) @ b @ p(v)))
                e_slope = max(e_slope, abs(d(1) @ a @ p(v) - d(0) @ b @ p(v)))
                e_ref = max(e_ref, abs(p(1) @ R[i, j] @ p(v) - p(0) @ R[(i + 1) % res, j] @ p(v)))
            x, y = (i + 0.5) * 2 * np.pi / res, (j + 0.5) * 2 * np.pi / res
            e_int = max(e_int, abs(p(0.5) @ C[i, j] @ p(0.5) - (2 * np.cos(x) * np.sin(2 * y) + np.cos(x + y))))
    assert e_edge < 1e-12 and e_slope < 1e-12 and e_corner < 1e-12
    assert e_int < 1e-3
    assert e_ref > 0.1      # the reference's table is discontinuous along cell edges


@pytest.mark.parametrize("lang,std", [("c", "c99"), ("c++", "c++11")])
def test_header_is_plain_c_and_cxx(lang, std, tmp_path):
    """include/mdf.h compiles warning-free as C99 and as C++11 (the C ABI a
    C, Fortran-interop or older C++ caller binds), and the struct sizes the C
    compiler sees match the ctypes mirror."""
    import subprocess
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    src = tmp_path / "probe.c"
    src.write_text('#include <stdio.h>\n#include "mdf.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(mdf_params), sizeof(mdf_energies), '
                   'sizeof(mdf_md_report), sizeof(mdf_min_report), sizeof(mdf_topology), sizeof(mdf_tune_report));'
                   ' return 0; }\n')
    exe = tmp_path / "probe"
    cc = "gcc" if lang == "c" else "g++"
    r = subprocess.run([cc, "-x", lang, "-std=" + std, "-Wall", "-Wextra", "-Werror", "-I" + inc, str(src), "-o",
                        str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    sizes = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert sizes == [C.sizeof(abi.mdf_params), C.sizeof(abi.mdf_energies), C.sizeof(abi.mdf_md_report),
                     C.sizeof(abi.mdf_min_report), C.sizeof(abi.mdf_topology), C.sizeof(abi.mdf_tune_report)]
