"""The results file of a multigroup solve (MultigroupSolver.write_results: the reference's
LionboltHDF5.f90 layout, written without the HDF5 library) holds exactly the solver's fluence and
dose, and the oracle's within 1e-5."""
import numpy as np
import pytest

import oracle as O
from helpers import rel_l2
from lionbolt_b200 import MultigroupSolver
from lionbolt_b200 import lionbolt_hdf5 as H
from lionbolt_b200 import problems as P

pytestmark = pytest.mark.gpu


def test_results_file_of_a_multigroup_solve(tmp_path):
    prob = P.multigroup_box(n=(4, 4, 8), size=(4.0, 4.0, 8.0), G=3, Ng=4, Nc=8, slab=(2.0, 4.0))
    mg = MultigroupSolver().set_problem(prob)
    mg.solve("GMRES", m=20, rtol=1e-8)
    flux, dose = mg.results()
    path = mg.write_results(str(tmp_path / "lb.h5"), particle="Photon")
    f = H.read(path)
    ph = f["photon"]
    assert ph.attrs["number_of_energy_dofs"] == prob.G and np.array_equal(ph["energy_grid"], prob.energy)
    for g in range(prob.G):
        assert np.array_equal(ph["fluence"][f"energy_{g + 1}"], flux[g])
    assert np.array_equal(ph["uncollided_fluence"]["energy_1"], prob.unc)
    assert np.array_equal(f["dose_deposition"], dose)
    # against the FP64 oracle's group loop
    o = O.Oracle(prob.mesh)
    assert o.set_angular(prob.k, prob.w, prob.Ls) == 0
    fo, do, _ = o.multigroup(prob, "GMRES", m=20, rtol=1e-11)
    assert rel_l2(f["dose_deposition"], do) < 1e-5
    for g in range(prob.G):
        assert rel_l2(ph["fluence"][f"energy_{g + 1}"], fo[g]) < 1e-5
