"""gdfv_residual_norms against the oracle: the Linf and L2 residual norms Eilmer
reports (e4/fluidblock.d:861-909, e4/simcore.d:1193-1212) of dU/dt of the last
step's predictor stage, which is R(U) of the state before that step."""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def _oracle_norms(orc, nsteps, threeD, mhd):
    """Norms of R(U) on the oracle's state after nsteps - 1 steps."""
    assert orc.run(nsteps - 1) == 0
    R = orc.residual(orc.all_U())
    nq = 10 if mhd else 5
    linf = np.zeros(nq)
    l2 = 0.0
    l2_vars = [0, 1, 2] + ([3] if threeD else []) + [4] + ([5, 6] if mhd else [])
    off = 0
    for (nic, njc, nkc) in orc.blocks:
        n = nic * njc * nkc
        Rb = R[off:off + nq * n].reshape(nq, n)
        off += nq * n
        linf = np.maximum(linf, np.abs(Rb).max(axis=1))
        l2 += float(sum((Rb[q] ** 2).sum() for q in l2_vars))
    return linf, np.sqrt(l2)


@pytest.mark.parametrize("name", ["inflow_fp64", "mhd_tube_fp64", "inflow_fp32"])
def test_residual_norms_match_oracle(name):
    """FP64 form: Linf to 1e-13 and L2 (summed in another order) to 1e-12 relative.  The
    predictor derivative is not pinned bit for bit by the state parity: an ulp of dU/dt
    rounds away in U0 + dt*dU/dt.  Float-flux form: the residual is a difference of
    nearly equal float fluxes, so its norms agree to 1e-4 relative."""
    nsteps = 6
    if name == "mhd_tube_fp64":
        case, threeD, mhd = cases.mhd_shock_tube(N=64), False, True
    else:
        prec = "fp32" if name.endswith("fp32") else "fp64"
        case, threeD, mhd = cases.c2_inflow_box(n=(40, 24, 20), precision=prec), True, False
    orc = cases.build_oracle(case)
    sim = cases.build_gpu(case)
    assert sim.run(max_step=nsteps) == nsteps
    linf, l2 = sim.residual_norms()
    linf_o, l2_o = _oracle_norms(orc, nsteps, threeD, mhd)
    assert linf.shape == linf_o.shape
    rel = np.abs(linf - linf_o) / np.maximum(linf_o, 1e-300)
    print(name, "Linf relative difference", rel, "L2", abs(l2 - l2_o) / l2_o)
    if name.endswith("fp64"):
        assert np.all(rel <= 1e-13), rel
        assert abs(l2 - l2_o) <= 1e-12 * l2_o, (l2, l2_o)
    else:
        assert np.all(np.abs(linf - linf_o) <= 1e-4 * np.maximum(linf_o, 1e-300))
        assert abs(l2 - l2_o) <= 1e-4 * l2_o
    # a second call returns the same figures (deterministic reduction order)
    linf2, l22 = sim.residual_norms()
    assert np.array_equal(linf, linf2) and l2 == l22
    sim.close()
