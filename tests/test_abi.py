"""CPU checks of the drop-in boundary: the built library loads and exports every
entry point include/h3d.h declares; the Python binding and the synthetic density
generator behave without a GPU."""
import os
import re
import subprocess

import numpy as np

import homo3d_b200 as H
from homo3d_b200 import density

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "h3d.h")).read()
    return sorted(set(re.findall(r"H3D_API\s+[\w\s\*]*?\b(h3d_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert len(syms) >= 30
    for s in ("h3d_create", "h3d_v_cycle", "h3d_solve", "h3d_elastic_matrix", "h3d_sensitivity",
              "h3d_oc_update", "h3d_symmetrize"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    L = H.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", H.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (h3d_\w+)", out))
    for s in declared_symbols():
        assert s in exported, s
        assert hasattr(L, s)
    # nothing else leaks out of the library
    assert exported == set(declared_symbols())


def test_binding_signatures_cover_the_header():
    bound = set(H._SIGS) | {"h3d_last_error", "h3d_stream", "h3d_mma_last_error", "h3d_warmnet_last_error",
                            "h3d_lockstep_last_error"}
    assert bound == set(declared_symbols())


def test_cpp_shim_compiles_and_links(tmp_path):
    src = tmp_path / "drv.cpp"
    src.write_text(
        '#include "h3d.hpp"\n'
        "int main() {\n"
        "  homo::HomoConfig c; c.reso[0] = c.reso[1] = c.reso[2] = 16;\n"
        "  (void)c;\n"
        "  void (homo::Homogenization::*f)(double (*)[6]) = &homo::Homogenization::elasticMatrix;\n"
        "  (void)f; return 0;\n"
        "}\n")
    out = tmp_path / "drv"
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(out),
                        "-L", os.path.dirname(H.LIB_PATH), "-lh3d"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_buffer_extent_rule():
    assert H._extent((4, 5, 6)) == 120
    assert H._extent((4, 5, 6), 8) == 3 + 8 * (4 + 5 * 5) + 1


def test_reference_resolution_rule():
    assert H.reference_resolution((80, 96, 100)) == (96, 96, 112)
    assert H.reference_resolution((320, 512, 1000)) == (320, 512, 1024)


def test_synthetic_density_is_seeded_symmetric_and_on_volume():
    a = density.synthetic_density(16, seed=3, vol=0.3)
    b = density.synthetic_density(16, seed=3, vol=0.3)
    c = density.synthetic_density(16, seed=4, vol=0.3)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert abs(a.mean() - 0.3) <= 1e-6
    assert a.min() >= 1e-3 and a.max() <= 1.0
    for ax in range(3):
        assert np.allclose(a, np.flip(a, axis=ax), atol=1e-12)
    assert np.allclose(a, np.transpose(a, (1, 0, 2)), atol=1e-12)
    assert np.allclose(a, np.transpose(a, (2, 1, 0)), atol=1e-12)


def test_splitmix64_known_values():
    # published first outputs of SplitMix64 seeded with 0
    r = density.SplitMix64(0)
    assert r.next_u64() == 0xE220A8397B1DCDAF
    assert r.next_u64() == 0x6E789E6AA1B965F4
