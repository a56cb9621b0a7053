"""Writes tests/golden/amr_workload.par with the reference's own input
generators (amss-ncku-python: setup.generate_AMSSNCKU_input,
numerical_grid.append_AMSSNCKU_cgh_input,
renew_puncture_parameter.append_AMSSNCKU_BSSN_input), fed the settings of the
amr workload: a 96^3 static level on [-48, 48]^3 and 6 moving levels of 48
cells per side around Brill-Lindquist punctures m = 0.5 at (-3, 0, 0) and
(3, 0, 0), no symmetry, Courant 0.25, dissipation 0.1, Lousto initial data.

Every other setting is the reference's shipped AMSS_NCKU_Input.py.  The
generators import matplotlib for plots this script never draws; a stand-in
module satisfies the import.  Run: python tests/golden/make_parfile.py
(needs the reference tree mounted; the output is committed).
"""
import importlib.util
import os
import shutil
import sys
import tempfile
import types

import numpy as np

REF = "/root/reference/amss-ncku-python"
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "amr_workload.par")


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    tmp = tempfile.mkdtemp()
    inp = _load("AMSS_NCKU_Input", os.path.join(REF, "AMSS_NCKU_Input.py"))
    inp.File_directory = tmp
    inp.Symmetry = "no-symmetry"
    inp.Initial_Data_Method = "Lousto-Analytical"
    inp.puncture_data_set = "Manually"
    inp.Courant_Factor = 0.25
    inp.Dissipation = 0.1
    inp.refinement_level = 0
    inp.devide_factor = 2.0
    inp.static_grid_type = "Linear"
    inp.moving_grid_type = "Linear"
    inp.grid_level = 7
    inp.static_grid_level = 1
    inp.moving_grid_level = 6
    inp.static_grid_number = 96
    inp.moving_grid_number = 48
    inp.largest_box_xyz_max = np.array([48.0, 48.0, 48.0])
    inp.largest_box_xyz_min = np.array([-48.0, -48.0, -48.0])
    inp.puncture_number = 2
    inp.position_BH = np.array([[-3.0, 0.0, 0.0], [3.0, 0.0, 0.0]])
    inp.momentum_BH = np.zeros((2, 3))
    inp.parameter_BH = np.array([[0.5, 0.0, 0.0], [0.5, 0.0, 0.0]])
    inp.dimensionless_spin_BH = np.zeros((2, 3))
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = mpl.pyplot
    sys.path.insert(0, REF)
    cwd = os.getcwd()
    os.chdir(tmp)
    try:
        setup = _load("setup", os.path.join(REF, "setup.py"))
        setup.generate_AMSSNCKU_input()
        grid = _load("numerical_grid", os.path.join(REF, "numerical_grid.py"))
        grid.append_AMSSNCKU_cgh_input()
        renew = _load("renew_puncture_parameter", os.path.join(REF, "renew_puncture_parameter.py"))
        renew.append_AMSSNCKU_BSSN_input(tmp, tmp)
    finally:
        os.chdir(cwd)
    shutil.copy(os.path.join(tmp, "AMSS-NCKU.input"), OUT)
    shutil.rmtree(tmp)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
