"""Register the ``cuda`` device interface inside an installed bempp_cl.

bempp_cl selects back ends by the prefix of ``device_interface`` in
bempp_cl/core/dispatcher.py:4-55 and raises ValueError for anything other
than "numba" / "opencl".  ``install()`` wraps the three dispatcher functions
so that "cuda" and "cuda_mixed" go to ``bempp_cuda.cuda_assemblers`` and every
other value reaches the original functions unchanged.  It also wraps
``bempp_cl.core.dense_assembler.assemble_dense`` (core/dense_assembler.py:49)
so a cuda weak form is assembled whole on the device (regular and singular
parts fused, one copy back) instead of pair-list by pair-list through the
host.  User scripts then run unchanged apart from the device_interface
string:

    import bempp_cuda.plugin; bempp_cuda.plugin.install()
    op = bempp_cl.api.operators.boundary.helmholtz.single_layer(
        sp, sp, sp, 5.0, assembler="dense", device_interface="cuda")
    op.weak_form()
"""

_installed = False


def _is_cuda(device_interface):
    return device_interface is not None and str(device_interface).split("_")[0] == "cuda"


def install():
    """Idempotently patch bempp_cl's dispatcher and dense assembler."""
    global _installed
    if _installed:
        return
    from bempp_cl.core import dispatcher as _dispatcher
    from bempp_cl.core import dense_assembler as _dense

    from . import cuda_assemblers as _cuda

    orig_singular = _dispatcher.singular_assembler_dispatcher
    orig_dense = _dispatcher.dense_assembler_dispatcher
    orig_potential = _dispatcher.potential_dispatcher
    orig_assemble_dense = _dense.assemble_dense

    def singular_assembler_dispatcher(device_interface, *args):
        if _is_cuda(device_interface):
            return _cuda.singular_assembler(device_interface, *args)
        return orig_singular(device_interface, *args)

    def dense_assembler_dispatcher(device_interface, *args):
        if _is_cuda(device_interface):
            return _cuda.dense_assembler(device_interface, *args)
        return orig_dense(device_interface, *args)

    def potential_dispatcher(device_interface, *args):
        if _is_cuda(device_interface):
            return _cuda.potential_assembler(device_interface, *args)
        return orig_potential(device_interface, *args)

    def assemble_dense(domain, dual_to_range, parameters, operator_descriptor, device_interface):
        if _is_cuda(device_interface):
            return _cuda.assemble_dense(domain, dual_to_range, parameters, operator_descriptor, device_interface)
        return orig_assemble_dense(domain, dual_to_range, parameters, operator_descriptor, device_interface)

    _dispatcher.singular_assembler_dispatcher = singular_assembler_dispatcher
    _dispatcher.dense_assembler_dispatcher = dense_assembler_dispatcher
    _dispatcher.potential_dispatcher = potential_dispatcher
    _dense.assemble_dense = assemble_dense
    _installed = True


def installed():
    return _installed
