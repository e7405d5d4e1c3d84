"""The ``cuda`` device interface, with the signatures of the reference back end.

Each function mirrors ``bempp_cl/core/numba_assemblers.py`` one for one, so
that ``bempp_cl.core.dispatcher`` can route ``device_interface="cuda"`` (or
"cuda_mixed") here exactly as it routes "numba":

* ``singular_assembler``  <- numba_assemblers.py:6-55 (dispatcher.py:4-19)
* ``dense_assembler``     <- numba_assemblers.py:58-112 (dispatcher.py:22-37)
* ``potential_assembler`` <- numba_assemblers.py:115-164 (dispatcher.py:40-55)

Same ownership rules: the first two accumulate into the caller's host
``result`` array; ``potential_assembler`` returns an evaluator that returns a
fresh (kernel_dimension, npoints) array.  Unsupported operators raise
ValueError like the reference dispatcher does for unknown interfaces.

``assemble_dense`` is the fused whole-matrix replacement of
core/dense_assembler.py:49-98 (regular and singular parts on the device,
one device-to-host copy).
"""

import numpy as _np
import torch as _torch

from . import _lib
from .assembly import (
    assemble_dense_device,
    evaluate_potential_device,
    kernel_ids,
    kernel_params,
    note_fp64_fallback,
    precision_of,
    regular_into,
    result_dtype,
)
from .device import DeviceSingularRule, current_stream, device_grid, device_space, ptr, require_cuda


def _torch_dtype(np_dtype):
    return _torch.complex128 if _np.dtype(np_dtype).kind == "c" else _torch.float64


def singular_assembler(
    device_interface,
    operator_descriptor,
    grid,
    domain,
    dual_to_range,
    test_points,
    trial_points,
    quad_weights,
    test_elements,
    trial_elements,
    test_offsets,
    trial_offsets,
    weights_offsets,
    number_of_quad_points,
    kernel_options,
    result,
):
    """Accumulate per-pair singular values into the flat host array ``result``."""
    require_cuda()
    precision_of(device_interface)
    kernel, assembly = kernel_ids(operator_descriptor)
    rule = DeviceSingularRule(
        [
            test_points,
            trial_points,
            quad_weights,
            test_elements,
            trial_elements,
            test_offsets,
            trial_offsets,
            weights_offsets,
            number_of_quad_points,
        ]
    )
    values = _torch.zeros(result.shape, dtype=_torch_dtype(result.dtype), device="cuda")
    args = _lib.SingularArgs()
    args.kernel = kernel
    args.assembly = assembly
    args.is_complex = 1 if values.is_complex() else 0
    p = kernel_params(kernel_options)
    for i in range(4):
        args.params[i] = float(p[i])
    args.grid = device_grid(grid).record()
    args.test = device_space(dual_to_range).record()
    args.trial = device_space(domain).record()
    rule.fill(args)
    args.values = ptr(values)
    args.dense = None
    args.ld = 0
    args.diag_shift = 0.0
    _lib.check(_lib.load().bemppcuda_assemble_singular(args, current_stream()))
    result += values.cpu().numpy().astype(result.dtype, copy=False)


def dense_assembler(device_interface, operator_descriptor, domain, dual_to_range, parameters, result):
    """Accumulate the regular-pair part into the host matrix ``result``."""
    require_cuda()
    precision = precision_of(device_interface)
    dev = _torch.zeros(result.shape, dtype=_torch_dtype(result.dtype), device="cuda")
    try:
        regular_into(dev, operator_descriptor, domain, dual_to_range, parameters, precision=precision,
                     result_is_zero=True)
    except _lib.BemppCudaError as exc:
        if exc.status == _lib.ERR_UNSUPPORTED and precision == _lib.MIXED:
            note_fp64_fallback(operator_descriptor, "regular-pair")
            regular_into(dev, operator_descriptor, domain, dual_to_range, parameters, precision=_lib.FP64,
                         result_is_zero=True)
        else:
            raise
    result += dev.cpu().numpy().astype(result.dtype, copy=False)


def potential_assembler(device_interface, space, operator_descriptor, points, parameters):
    """Return ``evaluator(x)`` giving the (kernel_dimension, npoints) potential."""
    require_cuda()
    precision_of(device_interface)
    kernel_ids(operator_descriptor)
    pts = _np.asarray(points, dtype=_np.float64)
    is_complex = operator_descriptor.is_complex

    def evaluator(x):
        res = evaluate_potential_device(space, operator_descriptor, pts, _np.asarray(x, dtype=_np.complex128), parameters)
        out = res.cpu().numpy()
        return out if is_complex else out.real.copy()

    return evaluator


def assemble_dense(domain, dual_to_range, parameters, operator_descriptor, device_interface):
    """Whole dense weak form on the device, returned as a host ndarray."""
    dev = assemble_dense_device(domain, dual_to_range, parameters, operator_descriptor, device_interface)
    out = dev.cpu().numpy()
    return out
