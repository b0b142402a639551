"""The routed build's error-budget check (fjb_set_route_check): a sampled
FP64 re-build of the FP32 queue estimates its error in G; within budget the
routed result stands, over budget the same build re-runs the FP32 units in
FP64 on the device (eager and captured builds alike).  Bars: the 1e-8
budget for routed results, the plain FP64 bar (1e-11) once re-routed."""

import numpy as np
import pytest

from felizjueves_b200 import configs
from felizjueves_b200.fock import FockEngine

pytestmark = pytest.mark.gpu


def _setup(cuda):
    import torch
    w = configs.cluster(3, 5)
    eng = FockEngine(w.basis)
    eng.plan(w.D, 0.0, 4)
    return w, eng, torch.tensor(w.D, device=cuda)


def test_checked_routed_build_within_budget(cuda, lib_built, oracle_lib):
    import torch
    from felizjueves_b200 import _lib, router
    w, eng, D = _setup(cuda)
    G = eng.build(D, precision=_lib.FJB_ROUTED, threshold=1e-7)[2]
    torch.cuda.synchronize()
    est, rerouted = eng.route_check()
    assert router.route_stats(eng)[0] > 0
    assert not rerouted and 0.0 < est <= 1e-8
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    assert np.abs(G.cpu().numpy() - (Jo - 0.5 * Ko)).max() <= 1e-8


@pytest.mark.parametrize("graph", [False, True])
def test_over_budget_reroutes_to_fp64(cuda, lib_built, oracle_lib, graph):
    """A budget no FP32 unit can meet: the build re-runs its FP32 queue in
    FP64 and G is the plain FP64 build's, to the FP64 bar."""
    import torch
    from felizjueves_b200 import _lib
    w, eng, D = _setup(cuda)
    eng.set_route_check(1e-30, 4)
    G = eng.build(D, precision=_lib.FJB_ROUTED, threshold=1e30, graph=graph)[2]
    torch.cuda.synchronize()
    est, rerouted = eng.route_check()
    assert rerouted and est > 1e-30
    Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
    assert np.abs(G.cpu().numpy() - (Jo - 0.5 * Ko)).max() <= 1e-11


def test_check_off_keeps_fp32(cuda, lib_built):
    """budget 0 turns the check off: an all-FP32 build keeps FP32 accuracy
    (its error is far above the FP64 bar) and reports no check."""
    import torch
    from felizjueves_b200 import _lib
    w, eng, D = _setup(cuda)
    G64 = eng.build(D)[2].clone()
    eng.set_route_check(0.0, 16)
    G32 = eng.build(D, precision=_lib.FJB_ROUTED, threshold=1e30)[2]
    torch.cuda.synchronize()
    assert float((G32 - G64).abs().max()) > 1e-11
    with pytest.raises(Exception):
        eng.route_check()
