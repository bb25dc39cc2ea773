"""A C++ caller written against the reference's class and method names
(VPFFT::DataStructures::MaterialGrid, include/vpfft/MaterialGrid.hpp) is
compiled with g++, linked with libvpfft_b200.so and run on the GPU: the
configuration-1 case (16^3, 8 grains, n = 10, uniaxial tension, one increment,
FP64) through SendDataAndInitialize / SetVoxelLength / RunSingleStrainStep,
then RunVPFFT.  Its <sigma> must match the reference's run (golden c1_16)
within 1e-9 relative, its stress field within 1e-7 per voxel, and its
Stress_Strain.txt must have one line per increment."""
import os
import subprocess

import numpy as np
import pytest

from vpfft_b200 import capi

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>
#include "vpfft/MaterialGrid.hpp"

using VPFFT::DataStructures::MaterialGrid;
using VPFFT::LinearAlgebra::EigenRep;
using VPFFT::LinearAlgebra::SMatrix3x3;

int main(int argc, char** argv) {
  // argv: orientations.bin edot(5) max_iter dt eps stress_out.bin stress_strain.txt
  const int n = 16 * 16 * 16;
  std::vector<SMatrix3x3> R(n);
  std::ifstream f(argv[1], std::ios::binary);
  f.read(reinterpret_cast<char*>(R.data()), sizeof(SMatrix3x3) * n);
  std::vector<EigenRep> S(n);
  EigenRep edot(atof(argv[2]), atof(argv[3]), atof(argv[4]), atof(argv[5]), atof(argv[6]));
  vpfft_material m;
  vpfft_material_default(&m);
  for (int s = 0; s < VPFFT_NUM_SLIP_SYSTEMS; ++s) {
    m.gamma_dot_base[s] = 1.0; m.rate_sensitivity[s] = 10; m.crss[s] = 1.0;
    m.tau0[s] = 1.0; m.tau1[s] = 0.5; m.theta0[s] = 20.0; m.theta1[s] = 1.0;
  }
  try {
    MaterialGrid g(16, 16, 16, &m);
    g.SendDataAndInitialize(R.data(), S.data());
    g.SetVoxelLength(1, 1, 1);
    EigenRep avg = g.RunSingleStrainStep(edot, atoi(argv[7]), atof(argv[8]), atof(argv[9]));
    std::printf("%.17g %.17g %.17g %.17g %.17g\n", avg(0), avg(1), avg(2), avg(3), avg(4));
    std::vector<EigenRep> out = g.Stress();
    std::ofstream o(argv[10], std::ios::binary);
    o.write(reinterpret_cast<const char*>(out.data()), sizeof(EigenRep) * n);
    MaterialGrid g2(16, 16, 16, &m);
    g2.SendDataAndInitialize(R.data(), S.data());
    g2.RunVPFFT(edot, 5, 2, atof(argv[8]), atof(argv[9]), argv[11]);
  } catch (const VPFFT::Error& e) {
    std::fprintf(stderr, "VPFFT::Error %d: %s\n", (int)e.status, e.what());
    return 1;
  }
  return 0;
}
"""


def test_cpp_caller_runs_configuration_1(golden, lib, tmp_path):
    g = golden("c1_16")
    src = tmp_path / "caller.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(capi.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe), "-L", libdir, "-lvpfft_b200", f"-Wl,-rpath,{libdir}"],
                   check=True)
    rin = tmp_path / "R.bin"
    np.ascontiguousarray(g["R_in"], "<f8").tofile(rin)
    sout, ss = tmp_path / "S.bin", tmp_path / "Stress_Strain.txt"
    e = [repr(float(x)) for x in g["edot"]]
    r = subprocess.run([str(exe), str(rin), *e, str(int(g["max_iter"])), repr(float(g["dt"])),
                        repr(float(g["eps"])), str(sout), str(ss)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    avg = np.array([float(t) for t in r.stdout.split()])
    ref = g["avg_stress"][0]
    assert np.linalg.norm(avg - ref) <= 1e-9 * np.linalg.norm(ref)
    sigma = np.fromfile(sout, "<f8").reshape(-1, 5)
    rel = np.linalg.norm(sigma - g["sigma"], axis=1) / np.linalg.norm(g["sigma"], axis=1)
    assert rel.max() <= 1e-7
    assert len(ss.read_text().strip().splitlines()) == 2
