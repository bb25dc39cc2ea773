"""A run driven by the reference's configuration file (ConfigFile, Config.h:
21-85), wired to MaterialGrid:

    python -m vpfft_b200.run_config <config> [--out DIR] [--print-fields]

GridDimension sets the RVE; TwoGrainInit builds the reference's two-grain
microstructure (UnitTester::SetMaterialGrid, UnitTester.cpp:46-74), FileInit
reads the Euler-angle texture named by the following line (ReadRicardoData,
UnitTester.cpp:237-265); CRSS, GammaDotBase, RateSensitivity, Tau0, Tau1,
Theta0, Theta1 and HardeningMatrix set the material; VoxelLength and
Precision are this implementation's additions.  The increments run as
RunVPFFT (MaterialGrid.cpp:1202-1228) with InputStrainRate (projected on the
deviatoric basis), NumTimeIter, TimeStep, and the fixed-point limits MaxIter
and ConvergenceEpsilon (defaults 100 and 1e-5, the values the reference's
drivers pass).  MaxNRIter and NRTolerence are read but, as in the reference,
do not change the Newton-Raphson constants.  Writes Stress_Strain.txt (and
with --print-fields the four Print* dumps) into the output directory.
"""
from __future__ import annotations

import argparse
import os
import sys

from . import fixtures, textio
from .config import ConfigFile
from .material_grid import MaterialGrid


def run(config_path: str, out_dir: str = ".", print_fields: bool = False):
    cfg = ConfigFile()
    if not cfg.Read(config_path):
        raise ValueError(f"{config_path}: {cfg.error}")
    dims = (cfg.NumX, cfg.NumY, cfg.NumZ)
    if cfg.InitMethod == ConfigFile.eInitFile:
        src = cfg.InputMicrostructureFilename
        if not os.path.isabs(src):
            src = os.path.join(os.path.dirname(os.path.abspath(config_path)), src)
        R = textio.ReadRicardoData(src, dims)
    else:
        R = fixtures.two_grain(*dims)
    grid = MaterialGrid(*dims, material=cfg.material, precision=cfg.precision)
    grid.SendDataAndInitialize(R)
    grid.SetVoxelLength(*cfg.VoxelLength)
    edot = fixtures.edot_from_matrix(cfg.InputStrainRate)
    os.makedirs(out_dir, exist_ok=True)
    rows = grid.RunVPFFT(edot, cfg.MaxIter, cfg.NumTimeIter, cfg.TimeStep,
                         cfg.ConvergenceEpsilon, os.path.join(out_dir, "Stress_Strain.txt"))
    if print_fields:
        grid.PrintStrain(os.path.join(out_dir, "Strain.txt"))
        grid.PrintStress(os.path.join(out_dir, "Stress.txt"))
        grid.PrintLagrangeMultiplier(os.path.join(out_dir, "LagrangeMultiplier.txt"))
        grid.PrintPolarization(os.path.join(out_dir, "Polarization.txt"))
    return grid, rows


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("config")
    ap.add_argument("--out", default=".")
    ap.add_argument("--print-fields", action="store_true")
    a = ap.parse_args(argv)
    grid, rows = run(a.config, a.out, a.print_fields)
    for step, strain, stress in rows:
        print(step, " ".join(f"{v:.6g}" for v in stress))
    grid.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
