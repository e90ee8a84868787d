"""Engine and oracle trajectories of the same beam recorded as ArtiSynth
print-state files (active nodes, t = 0 and every step) and compared with the
restated CompareStateFiles: within the parity bars (positions 1e-8,
velocities 1e-6 relative)."""
import numpy as np
import pytest

from artisynth_core_b200 import statefile as S
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import MechSystemSolver, NeoHookeanMaterial

from helpers import oracle_model

pytestmark = pytest.mark.gpu


def test_engine_and_oracle_state_files_agree(b200, oracle, tmp_path):
    wl = W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33), cells=(6, 2, 2))
    wl.build_mesh()
    steps = 8
    m = wl.model()
    ms = MechSystemSolver(m, tol=1e-13)
    w = S.StateWriter(str(tmp_path / "gpu.out"), fmt="%.15g")
    S.write_model_trajectory(w, "TetBeam BackwardEuler", m, ms, wl.h, steps)
    w.close()
    om = oracle_model(oracle, wl)
    active = np.where(wl.fixed == 0)[0]
    x = wl.rest.copy()
    v = np.zeros_like(x)
    w = S.StateWriter(str(tmp_path / "oracle.out"), fmt="%.15g")
    w.header("TetBeam BackwardEuler", int(active.size))
    w.state(0.0, v[active], x[active])
    t = 0.0
    for _ in range(steps):
        st, _, _ = om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, solver=1)
        assert st == 0
        t += wl.h
        w.state(t, v[active], x[active])
    w.close()
    ve, pe = S.compare_files(str(tmp_path / "gpu.out"), str(tmp_path / "oracle.out"), show_level=-1)
    assert pe <= 1e-8 and ve <= 1e-6, (pe, ve)
