"""The uneven molecule batch (config c4) as one captured CUDA graph: every
molecule's G equals its own direct build's (FP64, to rounding: the atomics'
order differs), the routed batch with the learned router installed stays in
the 1e-8 budget, and per-molecule device times are read back after a replay."""

import numpy as np
import pytest

from felizjueves_b200 import configs

pytestmark = pytest.mark.gpu


def test_batch_graph_matches_oracle(cuda, lib_built, oracle_lib):
    """Each molecule of a captured batch against the oracle directly: the
    FP64 graph within the screened build's bar (tau = 1e-12: every skipped
    term is below tau by the proved bounds), the routed graph within the
    1e-8 budget."""
    import torch
    from felizjueves_b200 import _lib
    from felizjueves_b200.batch import BatchBuilder
    ws = [configs.cluster(n, 4200 + n) for n in (3, 2, 4)]
    bb = BatchBuilder(ws)
    Go = []
    for w in ws:
        Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
        Go.append(Jo - 0.5 * Ko)
    for name, prec, thr, bar in (("fp64", _lib.FJB_FP64, 0.0, 1e-9),
                                 ("routed", _lib.FJB_ROUTED, 1e-9, 1e-8)):
        bb.capture(name, prec, thr)
        bb.replay(name)
        torch.cuda.synchronize()
        for g, go in zip(bb.G(), Go):
            assert float(np.abs(g.cpu().numpy() - go).max()) <= bar, name


def test_batch_graph_matches_per_molecule_builds(cuda, lib_built):
    import torch
    from felizjueves_b200 import _lib
    from felizjueves_b200.batch import BatchBuilder
    ws = [configs.cluster(n, 4100 + n) for n in (2, 3, 4, 3, 2)]
    bb = BatchBuilder(ws)
    ref = []
    for eng, D in zip(bb.engines, bb.D):
        ref.append(eng.build(D)[2].clone())
    bb.capture("fp64", _lib.FJB_FP64)
    for rep in range(2):
        bb.replay("fp64")
        torch.cuda.synchronize()
        for g, r in zip(bb.G(), ref):
            assert float((g - r).abs().max()) <= 1e-12
    ms = bb.device_ms()
    assert ms.shape == (5,) and np.all(ms > 0)
    bb.capture("routed", _lib.FJB_ROUTED, 1e-9)
    bb.replay("routed")
    torch.cuda.synchronize()
    for g, r in zip(bb.G(), ref):
        assert float((g - r).abs().max()) <= 1e-8


def test_merged_batch_matches_oracle(cuda, lib_built, oracle_lib):
    """The batched build -- one launch per class for every molecule, a
    class-sorted queue over all of them -- against the oracle, molecule by
    molecule (FP64 at the screened bar, routed within the 1e-8 budget), eager
    and replayed from its graph."""
    import torch
    from felizjueves_b200 import _lib
    from felizjueves_b200.batch import BatchBuilder
    ws = [configs.cluster(n, 4300 + n) for n in (3, 2, 4, 2)]
    bb = BatchBuilder(ws)
    Go = []
    for w in ws:
        Jo, Ko = oracle_lib.jk(oracle_lib.OracleBasis.of(w.basis), w.D)
        Go.append(Jo - 0.5 * Ko)
    bb.build_merged(_lib.FJB_FP64)
    torch.cuda.synchronize()
    st = bb.merged_stats()
    assert st["class_launches"] <= 55 and st["units"] > 0
    for g, go in zip(bb.G(), Go):
        assert float(np.abs(g.cpu().numpy() - go).max()) <= 1e-9
    for name, prec, thr, bar in (("m64", _lib.FJB_FP64, 0.0, 1e-9), ("m32", _lib.FJB_ROUTED, 1e-9, 1e-8)):
        bb.capture_merged(name, prec, thr)
        for o in bb.out:
            o[2].fill_(float("nan"))
        bb.replay(name)
        torch.cuda.synchronize()
        for g, go in zip(bb.G(), Go):
            assert float(np.abs(g.cpu().numpy() - go).max()) <= bar, name
    bb.close()


def test_merged_batch_learned_router_matches_loop(cuda, lib_built):
    """With a network installed on the first molecule, the batched build
    routes every molecule by it: the same network installed on each
    molecule's own handle makes the per-molecule routed builds take the
    same routing decisions, so the two agree to FP64 rounding."""
    import torch
    from felizjueves_b200 import _lib, router
    from felizjueves_b200.batch import BatchBuilder
    ws = [configs.cluster(n, 4400 + n) for n in (3, 2, 3)]
    bb = BatchBuilder(ws)
    X = np.random.default_rng(0).normal(size=(64, 12)).astype(np.float32)
    mlp = router.MLP(router.init_params(X, seed=3))
    for eng in bb.engines:
        router.install(eng, mlp, threshold=1e-9, margin=0.5)
        eng.set_route_check(0.0, 16)  # the batch has no per-build check
    bb.build_loop(_lib.FJB_ROUTED, 1e-9)
    torch.cuda.synchronize()
    loop = [g.clone() for g in bb.G()]
    bb.capture_merged("mlp", _lib.FJB_ROUTED, 1e-9)
    bb.replay("mlp")
    torch.cuda.synchronize()
    for g, h in zip(bb.G(), loop):
        assert float((g - h).abs().max()) <= 1e-11
    bb.close()
