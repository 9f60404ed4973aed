"""The GPU sweep against the 1-D MT analytic answer and the oracle.

The reference's serial MT example (serial/gen_mesh.f90, 50 x 50 x 121 nodes,
1.2 M unknowns) with both MT sheet sources (gen_rhs oper_mode 2 and 3,
src/aphid.f90:590-619) at 0.01, 0.1 and 1 Hz: six systems in one batched
sweep through aphid_gpu_sweep_sources, mixed precision with escalation
(AUTO) to a true FP64 residual of 1e-8, and the reference's own complex128
recurrence (FP64) for comparison.  The surface impedance tensor of each
solution must match
  - the analytic layered-earth impedance (mt.layered_impedance with the
    mesh's H = 0 bottom) within the discretisation tolerance of
    tests/test_mt_analytic_cpu.py (1.5% in rho_a, 0.75 deg in phase), and
  - the oracle's discrete impedance, solved to 1e-12 on a 5 x 5 horizontal
    cut of the same mesh (the solution is laterally uniform), within 2e-6
    relative: the 1e-8 residual target and the complex64 inner solves leave
    the impedance that close to the FP64 answer.
The receiver gather's E at the surface node is the EM_grid mean of the two
edges, the same numbers the host forms from the full E field.
"""
import numpy as np
import pytest

from aphid_git_b200 import Solver, model, mt
from test_mt_analytic_cpu import FREQS, TOL_PHASE, TOL_RHO, oracle_impedance

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mt_sweeps():
    xn, yn, zn, sig, ks = model.serial_mt_model(50)
    om = [2 * np.pi * f for f in FREQS for _ in (2, 3)]
    sos = [0, 1] * len(FREQS)
    out = {}
    with Solver() as s:
        s.set_nodes(xn, yn, zn)
        s.set_model("R", sig)
        for prec in ("auto", "fp64"):
            X, infos = s.sweep(om, [2, 3], sos, precision=prec, target=1e-8, max_it=20000)
            ic = 25
            E, H = s.sweep_receivers([[ic + 1, ic + 1, ks + 1]])
            fields = [mt.surface_fields((50, 50, len(zn)), ks, w, *s.gen_fields(w, x), ic, ic)
                      for w, x in zip(om, X)]
            out[prec] = (infos, fields, E)
    return out, (zn, ks, sig)


@pytest.mark.parametrize("prec", ["auto", "fp64"])
def test_gpu_mt_impedance_matches_analytic_and_oracle(mt_sweeps, prec):
    out, (zn, ks, sig) = mt_sweeps
    infos, fields, _ = out[prec]
    for s, inf in enumerate(infos):
        assert inf["status_name"] == "converged", (prec, s, inf)
        assert inf["true_rel_resid"] < 1e-8 * (1.05 if prec == "fp64" else 1.0), inf
    for q, f in enumerate(FREQS):
        (e1, h1), (e2, h2) = fields[2 * q], fields[2 * q + 1]
        z = mt.tensor(e1, h1, e2, h2)
        za = mt.layered_impedance(f, zn[ks:], np.asarray(sig[0, 0, ks:], np.float64), bottom="wall")
        rho, ph = mt.apparent_resistivity(z[0, 1], f)
        rho_a, ph_a = mt.apparent_resistivity(za, f)
        assert abs(rho / rho_a - 1) < TOL_RHO, (prec, f, rho, rho_a)
        assert abs(ph - ph_a) < TOL_PHASE, (prec, f, ph, ph_a)
        zo = oracle_impedance(f)[0][0]
        for a, b in ((0, 1), (1, 0)):
            assert abs(z[a, b] / zo[a, b] - 1) < 2e-6, (prec, f, a, b, z[a, b], zo[a, b])
        assert abs(z[0, 0]) < 1e-6 * abs(z[0, 1]) and abs(z[1, 1]) < 1e-6 * abs(z[0, 1])


def test_gpu_receiver_gather_matches_host_fields(mt_sweeps):
    out, _ = mt_sweeps
    infos, fields, E = out["auto"]
    for s, (e, _) in enumerate(fields):
        assert np.allclose(E[s, 0, :2], e[:2], rtol=1e-12, atol=0), (s, E[s, 0], e)
