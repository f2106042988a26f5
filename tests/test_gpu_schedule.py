"""Launch schedules and CUDA-graph replay on the GPU. Every schedule the autotuner can pick (CTA count, CTAs per
SM, unit deal) gives the same solutions and diagnostics bit for bit, in FP64 and in mixed precision; the tuner
returns one of them and caches it; schedule="auto" solves like the default; and a captured launch replayed with
new inputs written into its static tensors equals the eager solve of those inputs."""

import pytest
import torch

from mit_jax_b200 import autotune
from mit_jax_b200 import cg2d as cg
from mit_jax_b200.graph import GraphedSolve
from mit_jax_b200.synthetic import make_batch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def workload():
    syn, B = make_batch(90, 4, with_cotangent=True)
    dev = torch.device("cuda")
    ex = cg.default_exchanger(syn.L)
    ops = tuple(torch.as_tensor(B[k]).to(dev) for k in cg.OPS)
    b = torch.as_tensor(B["b"]).to(dev)
    mask = cg._interior_mask(syn.L, dev)
    w = torch.where(mask, torch.as_tensor(B["w"]).to(dev), torch.zeros((), dtype=torch.float64, device=dev))
    norms = torch.as_tensor(B["cg2dNorm"]).to(dev)
    G = cg.GroupSpec(ex, ops, [b, w], [torch.zeros_like(b), torch.zeros_like(w)], [1e-12, 1e-12], [300, 300],
                     norms)
    return ex, G


def _same(r0, r1):
    for (x0, _, d0), (x1, _, d1) in zip(r0[0], r1[0]):
        torch.testing.assert_close(x1, x0, rtol=0, atol=0)
        assert torch.equal(d1, d0)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_every_candidate_schedule_is_bitwise_equal(workload, precision):
    _, G = workload
    ref = cg.solve_groups([G], precision=precision)
    recs = cg.diag_records(ref[0][0][2])
    assert all(r["status"] == "ok" for r in recs)
    ran = 0
    for cand in autotune.candidates(torch.cuda.get_device_properties(0).multi_processor_count):
        try:
            res = cg.solve_groups([G], precision=precision, **cand)
        except cg.capi.Cg2dError as e:           # a pipeline too deep for the shared memory is refused, not run
            assert e.status == cg.capi.CG2D_UNSUPPORTED, e
            continue
        _same(ref, res)
        ran += 1
    assert ran >= 12


def test_fp64_builds_for_one_and_two_ctas_per_sm_are_bitwise_equal():
    """One right-hand side, batch 8 LLC90 (1248 work units, at least 8 per SM): the default launch takes the FP64
    build for 2 CTAs per SM (96 registers a thread), ctas_per_sm 1 the build for one CTA per SM and ctas_per_sm 2
    the first again. Solutions and diagnostics are the same bit for bit."""
    syn, B = make_batch(90, 8)
    dev = torch.device("cuda")
    ex = cg.default_exchanger(syn.L)
    ops = tuple(torch.as_tensor(B[k]).to(dev) for k in cg.OPS)
    b = torch.as_tensor(B["b"]).to(dev)
    G = cg.GroupSpec(ex, ops, [b], [torch.zeros_like(b)], [1e-12], [300], torch.as_tensor(B["cg2dNorm"]).to(dev))
    ref = cg.solve_groups([G], precision="f64")
    assert all(r["status"] == "ok" for r in cg.diag_records(ref[0][0][2]))
    for cps in (1, 2):
        _same(ref, cg.solve_groups([G], precision="f64", ctas_per_sm=cps))


def test_tune_picks_a_candidate_and_caches_it(workload, monkeypatch):
    _, G = workload
    monkeypatch.delenv("MIT_JAX_B200_TUNE_CACHE", raising=False)
    monkeypatch.setattr(autotune, "_CACHE", {})
    report = []
    sched = autotune.tune([G], precision="mixed", report=report)
    cands = autotune.candidates(torch.cuda.get_device_properties(0).multi_processor_count)
    assert sched in cands and len(report) == len(cands)
    assert min(ms for _, ms in report if ms is not None) == dict((str(c), ms) for c, ms in report)[str(sched)]
    again = []
    assert autotune.tune([G], precision="mixed", report=again) == sched and again == []
    _same(cg.solve_groups([G], precision="mixed"), cg.solve_groups([G], precision="mixed", schedule="auto"))


def test_graph_replay_equals_eager_on_new_inputs(workload):
    ex, G = workload
    norms = G.norm

    def post(res):
        return cg.edge_products(ex, res[0][1][0], res[0][0][0], norms)

    gs = GraphedSolve([G], precision="mixed", post=post)
    b_orig = G.b[0].clone()
    try:
        for scale in (1.0, 0.5):
            G.b[0].copy_(b_orig * scale + (1.0 - scale) * G.b[1])
            res, extra = gs.replay()
            eager = cg.solve_groups([G], precision="mixed")
            _same(eager, res)
            for a, e in zip(extra, post(eager)):
                torch.testing.assert_close(a, e, rtol=0, atol=0)
            assert gs.status() == cg.capi.CG2D_OK
    finally:
        G.b[0].copy_(b_orig)
