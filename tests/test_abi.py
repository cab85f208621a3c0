"""CPU checks of the C ABI: the library loads without a GPU, exports every
function include/mosscap_b200.h declares, and the ctypes mirrors of the
structs match the C layout. No compute call is made."""
import ctypes
import os
import subprocess
import tempfile

import pytest

from mosscap_b200 import capi


def test_library_exports_every_declared_function():
    lib = capi.load()
    declared = capi.declared_functions()
    assert "mc_time_step" in declared and "mc_compute_dt" in declared
    missing = [f for f in declared if not hasattr(lib, f)]
    assert not missing, missing
    assert lib.mc_abi_version() == 1


def test_struct_layout_matches_header():
    src = r"""
#include <stddef.h>
#include <stdio.h>
#include "mosscap_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(mc_grid), offsetof(mc_grid, dx), offsetof(mc_grid, bc),
         offsetof(mc_grid, bc_const), sizeof(mc_scheme));
  printf("%zu %zu %zu\n", offsetof(mc_scheme, gamma), offsetof(mc_scheme, max_cfl), sizeof(mc_clock));
  return 0;
}
"""
    inc = os.path.join(os.path.dirname(capi.HEADER))
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-std=c99", "-I", inc, c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    vals = [int(x) for x in out]
    assert vals[0] == ctypes.sizeof(capi.McGrid)
    assert vals[1] == capi.McGrid.dx.offset
    assert vals[2] == capi.McGrid.bc.offset
    assert vals[3] == capi.McGrid.bc_const.offset
    assert vals[4] == ctypes.sizeof(capi.McScheme)
    assert vals[5] == capi.McScheme.gamma.offset
    assert vals[6] == capi.McScheme.max_cfl.offset
    assert vals[7] == ctypes.sizeof(capi.McClock)


def test_enum_values_are_reference_ordinals():
    # source/Reconstruct.hpp:10-27, Riemann.hpp:10-14, TimeStepping.hpp:10-14, State.hpp:62-70
    text = open(capi.HEADER).read()
    for name, val in [("MC_RECON_WENO5Z", 3), ("MC_LIMITER_MINMOD", 2), ("MC_RIEMANN_HLLC", 2),
                      ("MC_STEPPER_SSPRK4", 2), ("MC_BC_ZEROGRAD", 4), ("MC_BC_USERFN", 6)]:
        assert f"{name} = {val}" in text
    assert capi.RECON["weno5z"] == 3 and capi.BOUNDARY["constant"] == 5


def test_slab_and_batch_form_entry_points_reject_bad_arguments():
    """Argument checks of the adjoint's slab entry points, the batch's
    launch-form switch, the host-resident step and the slab overlap switch,
    which fail before any device call."""
    lib = capi.load()
    INVALID = 1  # MC_ERR_INVALID_ARGUMENT
    assert capi.STATUS_NAMES[INVALID] == "MC_ERR_INVALID_ARGUMENT"
    hook = capi.COMM_FN(lambda user, op, bufs, count, stream: 0)
    uid = ctypes.create_string_buffer(128)
    assert lib.mc_adjoint_set_slab_hook(None, hook, None, 0, 1) == INVALID
    assert lib.mc_adjoint_set_slab_decomposition(None, uid, 0, 1) == INVALID
    assert lib.mc_batch_set_stage_launches(None, 1) == INVALID
    dt = ctypes.c_double()
    assert lib.mc_step_host(None, None, None, None, ctypes.byref(dt), None) == INVALID
    assert lib.mc_set_slab_overlap(None, 1) == INVALID
    n = ctypes.c_int32()
    assert lib.mc_batch_stage_launches(None, ctypes.byref(n)) == INVALID
    # the hook operation codes are the header's
    text = open(capi.HEADER).read()
    for name, val in [("MC_COMM_HALO", capi.COMM_HALO), ("MC_COMM_MIN_U64", capi.COMM_MIN_U64),
                      ("MC_COMM_SUM_F64", capi.COMM_SUM_F64), ("MC_COMM_MIN_I64", capi.COMM_MIN_I64)]:
        assert f"{name} = {val}" in text
