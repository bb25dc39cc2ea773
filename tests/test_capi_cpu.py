"""Host-side logic of the C ABI; runs without a GPU."""
import ctypes as C
import os

import numpy as np
import pytest

from vpfft_b200 import capi, fixtures


def test_library_exports_every_declared_symbol(lib):
    names = capi.declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_status_strings(lib):
    assert b"sm_100a" in lib.vpfft_version()
    for s in range(12):
        assert lib.vpfft_status_string(s)


def test_no_device_is_an_error_not_a_fallback(lib):
    if capi.device_count() > 0:
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    st = lib.vpfft_grid_create(8, 8, 8, None, None, capi.PREC_FP64, C.byref(h))
    assert st == capi.ERR_NO_DEVICE
    assert b"no CPU fallback" in lib.vpfft_last_error(None)


def test_unsupported_sizes_rejected(lib):
    h = C.c_void_p()
    for dims in [(7, 8, 8), (8, 0, 8), (1024, 8, 8), (8, 8, 11)]:
        assert lib.vpfft_grid_create(*dims, None, None, capi.PREC_FP64, C.byref(h)) == \
            capi.ERR_UNSUPPORTED_SIZE


def test_solver_option_defaults_and_checks(lib):
    """The reference's NR constants by default, the mixed-precision certificate
    bound 1e-5; options out of range are refused before any device work."""
    o = capi.solver_options()
    assert (o.nr_epsilon, o.nr_max_iter, o.nr_max_resolved) == (5e-4, 100, 1e9)
    assert (o.init_nr_epsilon, o.init_nr_max_iter) == (5e-4, 1000)
    assert o.mixed_certify_step == 1e-5 and o.green_operator == 0
    assert capi.solver_options(mixed_certify_step=0.0).mixed_certify_step == 0.0
    h = C.c_void_p()
    for bad in (-1e-6, 0.5, float("nan")):
        opt = capi.solver_options(mixed_certify_step=bad)
        st = lib.vpfft_grid_create(8, 8, 8, None, C.byref(opt), capi.PREC_MIXED, C.byref(h))
        assert st == capi.ERR_INVALID_ARGUMENT, bad
        assert b"mixed_certify_step" in lib.vpfft_last_error(None)
    opt = capi.solver_options(green_operator=3)
    assert lib.vpfft_grid_create(8, 8, 8, None, C.byref(opt), capi.PREC_MIXED,
                                 C.byref(h)) == capi.ERR_INVALID_ARGUMENT


def test_material_defaults_are_the_reference_constants(lib):
    m = capi.Material()
    lib.vpfft_material_default(C.byref(m))
    assert list(m.gamma_dot_base) == [15.5] * 12
    assert list(m.rate_sensitivity) == [10] * 12
    assert list(m.crss) == [11.0] * 12
    assert list(m.theta0) == [430.0] * 12 and list(m.theta1) == [110.0] * 12
    o = capi.SolverOptions()
    lib.vpfft_solver_options_default(C.byref(o))
    assert (o.init_nr_epsilon, o.init_nr_max_iter, o.nr_epsilon, o.nr_max_resolved,
            o.nr_max_iter) == (5e-4, 1000, 5e-4, 1e9, 100)


def _brute_voronoi(nx, ny, nz, ng, seed):
    M = (1 << 64) - 1
    s = seed
    pts = []
    for _ in range(ng):
        vals = []
        for _ in range(6):
            s = (s + 0x9E3779B97F4A7C15) & M
            z = s
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
            vals.append(((z ^ (z >> 31)) >> 11) * 2.0 ** -53)
        pts.append((vals[0] * nx, vals[1] * ny, vals[2] * nz))
    pts = np.array(pts)
    idx = np.indices((nx, ny, nz)).reshape(3, -1).T.astype(float)
    L = np.array([nx, ny, nz], float)
    d = np.abs(idx[:, None, :] - pts[None])
    d = np.minimum(d, L - d)
    return np.argmin((d ** 2).sum(-1), axis=1)


@pytest.mark.parametrize("dims,ng,seed", [((12, 10, 8), 7, 1), ((16, 16, 16), 64, 3),
                                          ((20, 6, 9), 200, 9), ((5, 5, 5), 1, 0)])
def test_voronoi_fixture_is_exact_periodic_voronoi(lib, dims, ng, seed):
    R, g = fixtures.polycrystal(*dims, ng, seed, with_grains=True)
    assert np.array_equal(g, _brute_voronoi(*dims, ng, seed))
    Rm = R.reshape(-1, 3, 3)
    assert np.abs(np.einsum("nij,nkj->nik", Rm, Rm) - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(Rm) - 1).max() < 1e-14
    R2 = fixtures.polycrystal(*dims, ng, seed)
    assert np.array_equal(R, R2)


def test_orientations_uniform_on_so3(lib):
    # For uniform rotations E[R] = 0 and E[R_ij^2] = 1/3.
    R = fixtures.polycrystal(40, 40, 40, 20000, 5).reshape(-1, 9)
    _, first = np.unique(fixtures.polycrystal(40, 40, 40, 20000, 5, True)[1], return_index=True)
    Ru = R[first]
    assert np.abs(Ru.mean(axis=0)).max() < 0.03
    assert np.abs((Ru ** 2).mean(axis=0) - 1 / 3).max() < 0.03


def test_edot_round_trip(lib):
    L = np.array([[1.0, 0.3, -0.2], [0.5, -0.4, 0.1], [0.0, 0.7, -0.6]])
    e = fixtures.edot_from_matrix(L)
    D = fixtures.matrix_from_edot(e)
    np.testing.assert_allclose(D, 0.5 * (L + L.T) - np.eye(3) * np.trace(L) / 3, atol=1e-15)
    np.testing.assert_allclose(fixtures.edot_from_matrix(np.diag([1, -0.5, -0.5])),
                               [-1.5 / np.sqrt(2), -1.5 / np.sqrt(6), 0, 0, 0], atol=1e-15)


CONFIG_OK = """# test input
GridDimension 16 16 8
InputStrainRate
  -0.5 0 0
  0 -0.5 0
  0 0 1
MaxNRIter 100
TimeStep 0.03
NumTimeIter 4
NRTolerence 1e-5
TwoGrainInit
CRSS 1 1 1 1 1 1 1 1 1 1 1 2
GammaDotBase 1
RateSensitivity 10 10 10 10 10 10 10 10 10 10 10 20
Tau0 1
Theta0 20
HardeningMatrix 1.4
VoxelLength 1 1 2
Precision MIXED
"""


def test_config_file(lib, tmp_path):
    from vpfft_b200 import ConfigFile

    p = tmp_path / "in.config"
    p.write_text(CONFIG_OK)
    cf = ConfigFile()
    assert cf.Read(str(p)), cf.error
    assert (cf.NumX, cf.NumY, cf.NumZ) == (16, 16, 8)
    np.testing.assert_array_equal(cf.InputStrainRate, np.diag([-0.5, -0.5, 1.0]))
    assert cf.MaxNRIter == 100 and cf.NumTimeIter == 4
    assert cf.TimeStep == 0.03 and cf.NRTolerence == 1e-5  # double, not float
    assert cf.CRSS[0] == 1.0 and cf.CRSS[11] == 2.0      # indices 0..11
    assert list(cf.RateSensitivity[-2:]) == [10, 20]
    assert cf.InitMethod == ConfigFile.eInitTwoGrain
    assert np.allclose(cf.VoxelLength, [1, 1, 2]) and cf.precision == "mixed"
    assert cf.material.hardening[143] == 1.4


@pytest.mark.parametrize("edit,msg", [
    (lambda s: s.replace("MaxNRIter 100\n", ""), "MaxNRIter"),
    (lambda s: s.replace("TwoGrainInit\n", ""), "initialization scheme"),
    (lambda s: s.replace("CRSS 1 1 1 1 1 1 1 1 1 1 1 2", "CRSS 1 1 1"), "CRSS"),
    (lambda s: s + "Bogus 3\n", "not recognized"),
    (lambda s: s.replace("TwoGrainInit", "FileInit /nonexistent/file"), "not found"),
])
def test_config_errors(lib, tmp_path, edit, msg):
    from vpfft_b200 import ConfigFile

    p = tmp_path / "bad.config"
    p.write_text(edit(CONFIG_OK))
    cf = ConfigFile()
    assert not cf.Read(str(p))
    assert msg in cf.error


def test_headers_compile_as_c_and_cpp(tmp_path):
    """include/*.h is plain C; the C++ facade header compiles too."""
    import subprocess

    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    src = tmp_path / "t.c"
    src.write_text('#include "vpfft_capi.h"\nint main(void){vpfft_material m; (void)m; return 0;}\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", inc, "-c", str(src), "-o",
                    str(tmp_path / "t.o")], check=True)
    cpp = tmp_path / "t.cpp"
    cpp.write_text('#include "vpfft/MaterialGrid.hpp"\nint main(){return 0;}\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", inc, "-c", str(cpp), "-o",
                    str(tmp_path / "t2.o")], check=True)
