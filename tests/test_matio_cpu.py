"""MATLAB v5 output files in the reference's layout: variable names, shapes
and values survive a write/read round trip, and the file names follow the
reference's strcat patterns."""
import os

import numpy as np

from elastodynamicebem_b200 import matio


def test_output_stem():
    assert matio.output_stem("sphereUniform", 3, "SA", 7) == os.path.join("./outputData", "sphereUniform3_SA_7")
    assert matio.output_stem("barH3", 2, "NEW") == os.path.join("./outputData", "barH32_NEW")


def test_density_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    phi = rng.normal(size=(20, 3 * 32))                  # (nT, 3N)
    f = str(tmp_path / "screenTest2_SA_7_density.mat")
    matio.save_density(f, phi)
    import scipy.io
    raw = scipy.io.loadmat(f)
    assert raw["density"].shape == (96, 20)               # 3N x nT, as the reference saves it
    assert np.array_equal(raw["density"][:, 5], phi[5])
    assert np.array_equal(matio.load_density(f), phi)


def test_block_and_field_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    E = rng.normal(size=(12, 12))
    f = str(tmp_path / "b_matrixE3.mat")
    matio.save_matrix_block(f, E)
    assert np.array_equal(matio.load_matrix_block(f), E)
    u = rng.normal(size=(4, 5, 3))                        # (times, points, 3)
    g = str(tmp_path / "b_A_campoVett.mat")
    matio.save_campo_vett(g, u)
    import scipy.io
    cell = scipy.io.loadmat(g)["campoVett"]
    assert cell.shape == (5, 4) and cell[2, 1].shape == (3, 1)
    assert np.array_equal(cell[2, 1][:, 0], u[1, 2])
    assert np.array_equal(matio.load_campo_vett(g), u)
