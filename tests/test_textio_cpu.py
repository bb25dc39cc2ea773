"""The reference's text formats (CPU): our writers and readers against the
reference's own routines run on the same numbers (tests/golden/io, written by
tests/golden/make_io_golden.py).  Bar: files byte-identical; values read back
bit-identical."""
import os

import numpy as np
import pytest

from vpfft_b200 import capi, textio

IO = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "io")
DIMS = (6, 5, 4)
N = 6 * 5 * 4


def raw(name, width):
    return np.fromfile(os.path.join(IO, name), dtype=np.float64).reshape(N, width)


def text(name):
    with open(os.path.join(IO, name), "rb") as f:
        return f.read()


@pytest.mark.parametrize("kind,re,im,ref", [
    ("stress", "in_S.bin", None, "stress.txt"),
    ("lagrange", "in_L.bin", None, "lagrange.txt"),
    ("strain", "in_D.bin", "in_D.bin", "strain.txt"),
    ("polarization", "in_P.bin", "in_P.bin", "polarization.txt"),
])
def test_print_field_matches_reference_bytes(lib, tmp_path, kind, re, im, ref):
    if im is None:
        r, i = raw(re, 5), None
    else:
        c = raw(re, 10).reshape(N, 5, 2)
        r, i = np.ascontiguousarray(c[:, :, 0]), np.ascontiguousarray(c[:, :, 1])
    out = tmp_path / f"{kind}.txt"
    textio.print_field(out, kind, DIMS, r, i)
    assert out.read_bytes() == text(ref)


def test_random_material_write_and_read(lib, tmp_path):
    out = tmp_path / "rm.txt"
    textio.WriteRandomMaterial(out, DIMS, raw("in_R.bin", 9), raw("in_S.bin", 5))
    assert out.read_bytes() == text("random_material.txt")
    R, S = textio.ReadRandomMaterial(os.path.join(IO, "random_material.txt"), DIMS)
    assert np.array_equal(R, raw("read_R.bin", 9))
    assert np.array_equal(S, raw("read_S.bin", 5))


def test_euler_texture_reader_matches_reference(lib):
    R = textio.ReadRicardoData(os.path.join(IO, "texture.txt"), DIMS)
    assert np.array_equal(R, raw("texture_R.bin", 9))
    # proper rotations
    M = R.reshape(N, 3, 3)
    assert np.allclose(np.einsum("nij,nkj->nik", M, M), np.eye(3), atol=1e-6)


def test_io_errors(lib, tmp_path):
    with pytest.raises(capi.VpfftError) as e:
        textio.ReadRandomMaterial(tmp_path / "missing.txt", DIMS)
    assert e.value.status == capi.ERR_IO
    short = tmp_path / "short.txt"
    short.write_text("1 2 3\n")
    with pytest.raises(capi.VpfftError) as e:
        textio.ReadRandomMaterial(short, DIMS)
    assert e.value.status == capi.ERR_IO
    bad = tmp_path / "bad_texture.txt"
    bad.write_text("10 20 30 7 1 1 0 1\n" * N)  # x = 7 > 6
    with pytest.raises(capi.VpfftError) as e:
        textio.ReadRicardoData(bad, DIMS)
    assert e.value.status == capi.ERR_IO


def test_two_grain_microstructure_matches_reference(lib):
    from vpfft_b200 import fixtures

    ref = np.fromfile(os.path.join(IO, "two_grain_R.bin"), dtype=np.float64).reshape(70, 9)
    assert np.array_equal(fixtures.two_grain(7, 5, 2), ref)
