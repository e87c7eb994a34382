"""Parity at the configurations' sizes and at convergence: the GPU's SIMPLEC
solve against the oracle's on the flat neutral ABL of the oracle case (32 x
32 x 48, 300 outer iterations), on a small hill run to the steady criterion,
and on the 128 x 128 x 64 hill at full size (one iteration, one residual
evaluation, one V-cycle, one line solve). The mixed-precision form (FP32
inner solves) is compared with the oracle's FP64 steady state field by
field. The GPU's converged neutral ABL is checked against the physics the
reference's Neutral_ABL_Flat regression checks
(Tests/Canonical_RANS/Neutral_ABL_Flat/README.md:17-22)."""
import math

import numpy as np
import pytest

import oracle
from ablsteadyrans_b200 import workloads

FIELDS = ("u", "v", "w", "p", "theta", "tke")
LOCS = (1, 2, 4, 0, 0, 0)


def oracle_case(inst):
    """The oracle's copy of an instance (metrics from its node heights), ghosts filled."""
    g = inst.grid
    J, ax, ay, az, _ = oracle.metrics(g, inst.z)
    oc = oracle.Case(g, inst.z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.z0map)
    oc.q = {f: a.copy() for f, a in inst.q.items()}
    oracle.fill_ghosts(oc, inst.bc, inst.physics)
    return oc


def gpu_stage(ctx, oc, inst, options=None):
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    dc = DeviceCase.from_oracle(oc)
    st = SimplecStage(ctx, dc, inst.bc, inst.physics, options if options is not None else inst.options)
    st.fill_ghosts()
    return dc, st


def field_errors(grid, got, ref):
    """Per field: max |got - ref| over the valid points / max |ref| (the
    field's scale; 1 for a field that is zero everywhere)."""
    out = {}
    for f, loc in zip(FIELDS, LOCS):
        v = grid.valid(loc)
        scale = float(np.abs(ref[f][v]).max())
        out[f] = float(np.abs(got[f][v] - ref[f][v]).max()) / (scale if scale > 0 else 1.0)
    return out


def run_oracle(oc, inst, cfls):
    """The oracle's SIMPLEC iterations at the given CFL per iteration (the
    GPU driver's sequence, so both take the same pseudo-time steps)."""
    for cfl in cfls:
        dt = oracle.local_dtau(oc, cfl, phys=inst.physics)
        rc, info, _ = oracle.simplec_iterate(oc, inst.bc, inst.physics, inst.options, dt)
        assert rc == 0
    return info


def closure_length(oc, inst):
    oracle.fill_ghosts(oc, inst.bc, inst.physics)
    return oracle.closure_fields(oc, inst.bc, inst.physics)["length"]


def gpu_closure_length(st):
    st.fill_ghosts()
    st.residual()
    cf, _ = st.turbulence(closure=True, surface=False)
    return cf["length"]


@pytest.mark.gpu
def test_gpu_config0_300_iterations_match_oracle(ctx):
    """The oracle case itself (flat, 32 x 32 x 48, log-law inflow u* = 0.4
    m/s, z0 = 0.1 m, the k-L closure and neutral MOST, no Coriolis): 300
    outer iterations of the SER driver on the GPU, and the oracle's 300 at
    the same CFL per iteration; U, V, W, p, k, theta and the closure's
    length L agree within 1e-6 relative."""
    from ablsteadyrans_b200.driver import Driver
    inst = workloads.config0()
    oc = oracle_case(inst)
    dc, st = gpu_stage(ctx, oc, inst)
    try:
        drv = Driver(st)
        for _ in range(300):
            assert drv.step() != "diverged"
        cfls = [h[0] for h in drv.history]
        oracle.set_threads(oracle.max_threads())
        run_oracle(oc, inst, cfls)
        got = {f: dc.host(f) for f in FIELDS}
        err = field_errors(inst.grid, got, oc.q)
        v = inst.grid.valid(0)
        Lg, Lo = gpu_closure_length(st), closure_length(oc, inst)
        err["L"] = float(np.abs(Lg[v] - Lo[v]).max() / np.abs(Lo[v]).max())
        print("config 0, 300 iterations, GPU vs oracle:", err)
        for f, e in err.items():
            assert e <= 1e-6, (f, e)
    finally:
        st.close()
