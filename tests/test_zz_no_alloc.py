"""mc_time_step_noalloc against mc_time_step, through the C ABI.

mc_time_step_noalloc exists for callers that cannot call cudaMalloc (their
device memory belongs to a pool allocator, or they must not synchronise the
device mid-run): it takes its stage buffers from a fixed 16 MiB static device
array instead of a context. Its results must equal the context-based entry
point's bit for bit, on consecutive calls (the static array keeps the previous
call's contents). This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

from mosscap_b200 import problems as P

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


@pytest.mark.parametrize("case", ["kh2d_weno_hllc", "sod1d_tracer", "sedov3d_ppm_hll"])
def test_noalloc_matches_context_entry_point(gpu_lib, case):
    from mosscap_b200 import capi
    from mosscap_b200.hydro import HydroSim
    lib = gpu_lib
    if case == "kh2d_weno_hllc":
        p = P.kelvin_helmholtz_2d(96, seed=4)
    elif case == "sod1d_tracer":
        base = P.sod_1d(512)
        q = np.concatenate([base.Q, (0.3 + 0.2 * np.sin(np.arange(base.Q.shape[-1]) / 9.0))
                            .reshape(1, 1, 1, -1) * base.Q[:1]], axis=0)
        p = base.with_scheme(num_tracers=1, Q=q)
    else:
        p = P.sedov_3d(24)
    ref = HydroSim(p)           # mc_create + mc_time_step (allocating path)
    ref.fill_bcs()
    q2 = ref.Q.clone()          # the same filled state for the static path
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        dt = ref.compute_dt()
        ref.time_step(dt)
        st = lib.mc_time_step_noalloc(ctypes.byref(ref._grid), ctypes.byref(ref._scheme),
                                      ctypes.c_void_p(q2.data_ptr()), dt, stream)
        capi.check(st, "mc_time_step_noalloc")
        torch.cuda.synchronize()
        a, b = ref.get_Q(), q2.cpu().numpy()
        assert np.array_equal(_bits(a), _bits(b)), f"call {call}: {np.count_nonzero(_bits(a) != _bits(b))} differ"


def test_noalloc_rejects_oversize(gpu_lib):
    from mosscap_b200 import capi
    from mosscap_b200.hydro import HydroSim
    p = P.kelvin_helmholtz_2d(600, seed=0)  # 2 x 4 x 606^2 doubles > 16 MiB
    sim = HydroSim(p)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = gpu_lib.mc_time_step_noalloc(ctypes.byref(sim._grid), ctypes.byref(sim._scheme),
                                      ctypes.c_void_p(sim.Q.data_ptr()), 1e-4, stream)
    assert st == 4  # MC_ERR_OUT_OF_MEMORY
    assert b"16 MiB" in gpu_lib.mc_last_error()
    with pytest.raises(capi.McError):
        capi.check(st, "mc_time_step_noalloc")
