"""k-point SCF of one cell with device members (chfsi.Context per k-point,
kpoint_scf.DeviceMember) against the same loop on oracle members: energies
per iteration at 1e-10 Ha, integrated charge N_e."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "chemrust-scf_b200"))
import kpoint_scf  # noqa: E402
from test_kpoint_scf import CELL, KPTS, _run, _systems  # noqa: E402


def test_device_kpoint_scf_matches_oracle_members(chfsi):
    kpts = KPTS[:3]
    w = np.full(len(kpts), 1.0 / len(kpts))
    ref = _run(_systems(kpts), w, 0, 1, None, 4)
    systems = [chfsi.SyntheticSystem(kpt=k, **CELL) for k in kpts]
    got = kpoint_scf.run_device_kpoint_scf(chfsi, systems, w, 10, max_iter=4, tol_per_atom=1e-14)
    print("k-point SCF energies: device %s oracle %s" % (got["energies"], ref["energies"]))
    np.testing.assert_allclose(got["energies"], ref["energies"], atol=1e-10, rtol=0)
    assert abs(got["charge"] - systems[0].n_elec) < 1e-8
