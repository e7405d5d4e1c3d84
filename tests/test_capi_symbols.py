"""The C-ABI library loads and exports every function declared in include/bemppcuda.h."""

import ctypes
import os
import re

from conftest import ROOT


def _declared():
    text = open(os.path.join(ROOT, "include", "bemppcuda.h")).read()
    return sorted(set(re.findall(r"^(?:int|int64_t)\s+(bemppcuda_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = _declared()
    for required in ("bemppcuda_assemble_regular", "bemppcuda_assemble_singular", "bemppcuda_evaluate_potential",
                     "bemppcuda_grid_geometry", "bemppcuda_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from bempp_cuda import _lib

    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name


def test_struct_layout_matches_header():
    """Compile a probe against the header with gcc and compare sizes / offsets."""
    import subprocess
    import tempfile

    from bempp_cuda import _lib

    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "bemppcuda.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(bemppcuda_regular_args), sizeof(bemppcuda_singular_args),
         sizeof(bemppcuda_potential_args), sizeof(bemppcuda_space), offsetof(bemppcuda_regular_args, result),
         offsetof(bemppcuda_singular_args, diag_shift), offsetof(bemppcuda_potential_args, workspace_bytes),
         offsetof(bemppcuda_regular_args, phase_radius), sizeof(bemppcuda_batch_problem),
         sizeof(bemppcuda_batch_args), offsetof(bemppcuda_batch_args, rows_per_item), sizeof(bemppcuda_shape_args),
         offsetof(bemppcuda_shape_args, incident), offsetof(bemppcuda_shape_args, lambda),
         offsetof(bemppcuda_shape_args, workspace_bytes), offsetof(bemppcuda_potential_args, phase_radius),
         offsetof(bemppcuda_regular_args, result_is_zero), offsetof(bemppcuda_singular_args, mirror_weights_offset),
         sizeof(bemppcuda_matmat_problem), sizeof(bemppcuda_matmat_args), offsetof(bemppcuda_matmat_args, blocks),
         sizeof(bemppcuda_identity_args), offsetof(bemppcuda_identity_args, nelements),
         offsetof(bemppcuda_identity_args, values));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as tmp:
        c = os.path.join(tmp, "probe.c")
        exe = os.path.join(tmp, "probe")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    mine = [ctypes.sizeof(_lib.RegularArgs), ctypes.sizeof(_lib.SingularArgs), ctypes.sizeof(_lib.PotentialArgs),
            ctypes.sizeof(_lib.Space), _lib.RegularArgs.result.offset, _lib.SingularArgs.diag_shift.offset,
            _lib.PotentialArgs.workspace_bytes.offset, _lib.RegularArgs.phase_radius.offset,
            ctypes.sizeof(_lib.BatchProblem), ctypes.sizeof(_lib.BatchArgs), _lib.BatchArgs.rows_per_item.offset,
            ctypes.sizeof(_lib.ShapeArgs), _lib.ShapeArgs.incident.offset, _lib.ShapeArgs.lam.offset,
            _lib.ShapeArgs.workspace_bytes.offset, _lib.PotentialArgs.phase_radius.offset,
            _lib.RegularArgs.result_is_zero.offset, _lib.SingularArgs.mirror_weights_offset.offset,
            ctypes.sizeof(_lib.MatmatProblem), ctypes.sizeof(_lib.MatmatArgs), _lib.MatmatArgs.blocks.offset,
            ctypes.sizeof(_lib.IdentityArgs), _lib.IdentityArgs.nelements.offset, _lib.IdentityArgs.values.offset]
    assert [int(x) for x in out] == mine


def test_last_error_is_callable_without_gpu():
    from bempp_cuda import _lib

    assert isinstance(_lib.last_error(), str)
    assert _lib.load().bemppcuda_version() >= 100
