"""Batched persistent assembly against single-problem assembly (run on a B200)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _problems():
    from bempp_cuda.shapes import ellipsoid

    rng = np.random.default_rng(3)
    out = []
    for level in (1, 2, 3, 2, 3, 1):
        axes = rng.uniform(0.5, 1.5, 3)
        out.append((ellipsoid(level, *axes), float(rng.uniform(1.0, 16.0))))
    return out


def _single(grid, k, interface="cuda", kind="slp"):
    from bempp_cuda import operators
    from bempp_cuda.space import function_space

    sp = function_space(grid, "DP", 0)
    if kind == "slp":
        return operators.boundary.helmholtz.single_layer(sp, sp, sp, k, device_interface=interface).weak_form().tensor
    slp = operators.boundary.helmholtz.single_layer(sp, sp, sp, k, device_interface=interface)
    dlp = operators.boundary.helmholtz.double_layer(sp, sp, sp, k, device_interface=interface)
    ident = operators.boundary.sparse.identity(sp, sp, sp)
    return (dlp - 0.5 * ident - 1j * k * slp).weak_form().tensor


def _rel(a, b):
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


@pytest.mark.parametrize("rows,bps", [(32, 4), (8, 2), (16, 6)])
def test_batch_fp64_matches_single_assemblies(rows, bps):
    from bempp_cuda.batch import BatchAssembler

    probs = _problems()
    ba = BatchAssembler([g for g, _ in probs], [k for _, k in probs], precision="fp64", rows_per_item=rows,
                        blocks_per_sm=bps)
    ba.launch()
    torch.cuda.synchronize()
    for (g, k), out in zip(probs, ba.outputs):
        assert _rel(out, _single(g, k)) < 1e-13


def test_batch_mixed_and_complex_wavenumbers():
    from bempp_cuda.batch import BatchAssembler

    probs = _problems()
    ks = [k if i % 2 else k + 0.7j for i, (_, k) in enumerate(probs)]
    precisions = ["mixed" if i % 3 else "fp64" for i in range(len(probs))]
    ba = BatchAssembler([g for g, _ in probs], ks, precision=precisions)
    ba.launch()
    torch.cuda.synchronize()
    for (g, _), k, prec, out in zip(probs, ks, precisions, ba.outputs):
        ref = _single(g, k)
        assert _rel(out, ref) < (1e-6 if prec == "mixed" else 1e-13)


def test_batch_combined_field_with_identity():
    from bempp_cuda.batch import BatchAssembler

    probs = _problems()[:3]
    ba = BatchAssembler([g for g, _ in probs], [k for _, k in probs], kernel="helmholtz_combined_field",
                        identity=-0.5)
    ba.launch()
    torch.cuda.synchronize()
    for (g, k), out in zip(probs, ba.outputs):
        assert _rel(out, _single(g, k, kind="combined")) < 1e-12


def test_graph_replay_and_multi_rhs_products():
    from bempp_cuda.batch import BatchAssembler

    probs = _problems()
    ba = BatchAssembler([g for g, _ in probs], [k for _, k in probs], precision="mixed")
    rng = np.random.default_rng(9)
    rhs = [torch.as_tensor(rng.standard_normal((g.number_of_elements, 8)) +
                           1j * rng.standard_normal((g.number_of_elements, 8)), device="cuda") for g, _ in probs]
    prods = [torch.empty_like(x) for x in rhs]
    ba.capture(rhs, prods)
    for out in ba.outputs:
        out.zero_()
    ba.replay()
    torch.cuda.synchronize()
    for (g, k), out, x, y in zip(probs, ba.outputs, rhs, prods):
        ref = _single(g, k, "cuda_mixed")
        assert _rel(out, ref) < 1e-12
        assert _rel(y, ref @ x) < 1e-12


def test_autotune_picks_a_timed_shape():
    from bempp_cuda.batch import BatchAssembler

    probs = _problems()
    ba = BatchAssembler([g for g, _ in probs], [k for _, k in probs])
    shape, timings = ba.autotune(rows=(16, 32), blocks=(2, 4), repeats=1)
    assert shape in timings and timings[shape] == min(timings.values())
    ba.launch()
    torch.cuda.synchronize()
    g, k = probs[0]
    assert _rel(ba.outputs[0], _single(g, k)) < 1e-13


def test_batch_rejects_bad_problem_lists():
    import ctypes

    from bempp_cuda import _lib
    from bempp_cuda.batch import BatchAssembler
    from bempp_cuda.device import current_stream

    probs = _problems()[:2]
    ba = BatchAssembler([g for g, _ in probs], [k for _, k in probs])
    ba._problems[1].pair_begin += 1  # pair ranges no longer contiguous
    rc = _lib.load().bemppcuda_batch_launch(ctypes.byref(ba.args), current_stream())
    assert rc == _lib.ERR_INVALID and "singular pairs" in _lib.last_error()
    torch.cuda.synchronize()
