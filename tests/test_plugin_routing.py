"""``bempp_cuda.plugin.install`` routes the cuda interface and leaves others alone.

bempp_cl is not importable everywhere these tests run, so a minimal stand-in
package with the two patched modules (dispatcher, dense_assembler) is put in
sys.modules; the routing logic is what is under test.
"""

import sys
import types

import pytest


@pytest.fixture
def fake_bempp(monkeypatch):
    calls = []
    root = types.ModuleType("bempp_cl")
    core = types.ModuleType("bempp_cl.core")
    disp = types.ModuleType("bempp_cl.core.dispatcher")
    dense = types.ModuleType("bempp_cl.core.dense_assembler")

    def make(name):
        def fn(device_interface, *args):
            if device_interface.split("_")[0] not in ("numba", "opencl"):
                raise ValueError("Device interface must be one of 'numba', 'opencl'.")
            calls.append(("orig", name, device_interface))
            return name
        return fn

    disp.singular_assembler_dispatcher = make("singular")
    disp.dense_assembler_dispatcher = make("dense")
    disp.potential_dispatcher = make("potential")

    def assemble_dense(domain, dual, params, desc, device_interface):
        calls.append(("orig", "assemble_dense", device_interface))
        return "host"

    dense.assemble_dense = assemble_dense
    root.core = core
    core.dispatcher = disp
    core.dense_assembler = dense
    for name, mod in [("bempp_cl", root), ("bempp_cl.core", core), ("bempp_cl.core.dispatcher", disp),
                      ("bempp_cl.core.dense_assembler", dense)]:
        monkeypatch.setitem(sys.modules, name, mod)
    from bempp_cuda import cuda_assemblers, plugin

    monkeypatch.setattr(plugin, "_installed", False)
    for fname in ("singular_assembler", "dense_assembler", "potential_assembler", "assemble_dense"):
        monkeypatch.setattr(cuda_assemblers, fname,
                            (lambda n: (lambda *a, **k: calls.append(("cuda", n, a[0] if a else None)) or "cuda"))(fname))
    plugin.install()
    yield disp, dense, calls


def test_cuda_interfaces_route_to_bempp_cuda(fake_bempp):
    disp, dense, calls = fake_bempp
    assert disp.dense_assembler_dispatcher("cuda", 1, 2) == "cuda"
    assert disp.singular_assembler_dispatcher("cuda_mixed", 1) == "cuda"
    assert disp.potential_dispatcher("cuda", 1) == "cuda"
    assert dense.assemble_dense(None, None, None, None, "cuda") == "cuda"
    assert [c[0] for c in calls] == ["cuda"] * 4


def test_other_interfaces_untouched(fake_bempp):
    disp, dense, calls = fake_bempp
    assert disp.dense_assembler_dispatcher("numba", 1) == "dense"
    assert dense.assemble_dense(None, None, None, None, "numba") == "host"
    with pytest.raises(ValueError):
        disp.potential_dispatcher("vulkan", 1)
    assert all(c[0] == "orig" for c in calls)


def test_install_is_idempotent(fake_bempp):
    from bempp_cuda import plugin

    disp, _, _ = fake_bempp
    first = disp.dense_assembler_dispatcher
    plugin.install()
    assert disp.dense_assembler_dispatcher is first
